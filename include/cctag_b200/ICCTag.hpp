// Header-only C++ shim with the reference's public API (src/cctag/ICCTag.hpp,
// Params.hpp, CCTagMarkersBank.hpp, CCTag.hpp status codes) on top of the C ABI
// of cctag_b200 (include/cctag_b200.h).  No OpenCV, Boost or Eigen: the image
// is any type with `data`, `cols`, `rows` and `step` members (cv::Mat works) or
// a GrayView; the marker list is any container with clear() and push_back(T*)
// (boost::ptr_list<ICCTag> works) or a std::vector<std::unique_ptr<ICCTag>>.
//
//   cctag::Parameters params(3);
//   std::vector<std::unique_ptr<cctag::ICCTag>> markers;
//   cctag::cctagDetection(markers, 0, frameId, cctag::GrayView{ptr, w, h, w}, params);
//   for (auto& m : markers) if (m->getStatus() == cctag::status::id_reliable) ...
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../cctag_b200.h"

namespace cctag {

using MarkerID = int;
static constexpr MarkerID UndefinedMarkerID{-1};

namespace status {
// CCTag.hpp:416-426
static const int id_reliable = 1;
static const int too_few_outer_points = -1;
static const int no_collected_cuts = -1;
static const int no_selected_cuts = -2;
static const int opti_has_diverged = -3;
static const int id_not_reliable = -4;
static const int degenerate = -5;
}  // namespace status

namespace numerical {
namespace geometry {
// Minimal ellipse value type: parameters and conic matrix (row-major).
class Ellipse {
public:
    Ellipse() = default;
    explicit Ellipse(const cctagb_ellipse& e) : _e(e) {}
    struct Center {
        float _x, _y;
        float x() const { return _x; }
        float y() const { return _y; }
    };
    Center center() const { return Center{_e.cx, _e.cy}; }
    float a() const { return _e.a; }
    float b() const { return _e.b; }
    float angle() const { return _e.angle; }
    float matrix(int r, int c) const { return _e.m[r * 3 + c]; }

private:
    cctagb_ellipse _e{};
};
}  // namespace geometry
}  // namespace numerical

namespace logtime {
// Stand-in for the reference's logtime::Mgmt: keeps named durations (ms).
class Mgmt {
public:
    explicit Mgmt(std::size_t = 0) {}
    void log(const char* name, float ms) { _entries.emplace_back(name, ms); }
    void print(std::ostream& os) const
    {
        for (const auto& e : _entries) os << e.first << ": " << e.second << " ms\n";
    }
    const std::vector<std::pair<std::string, float>>& entries() const { return _entries; }

private:
    std::vector<std::pair<std::string, float>> _entries;
};
}  // namespace logtime

// Params.hpp:108-255: same member names and defaults.
struct Parameters {
    explicit Parameters(std::size_t nCrowns = 3)
    {
        cctagb_params_default(&_p, int(nCrowns));
        sync_from();
    }
    float _cannyThrLow, _cannyThrHigh;
    std::size_t _distSearch;
    int _thrGradientMagInVote;
    float _angleVoting, _ratioVoting, _averageVoteMin, _thrMedianDistanceEllipse;
    std::size_t _maximumNbSeeds, _maximumNbCandidatesLoopTwo, _nCrowns, _nCircles, _minPointsSegmentCandidate,
        _minVotesToSelectCandidate;
    float _threshRobustEstimationOfOuterEllipse, _ellipseGrowingEllipticHullWidth;
    std::size_t _windowSizeOnInnerEllipticSegment, _numberOfMultiresLayers, _numberOfProcessedMultiresLayers,
        _nSamplesOuterEllipse, _numCutsInIdentStep, _numSamplesOuterEdgePointsRefinement, _cutsSelectionTrials,
        _sampleCutLength, _imagedCenterNGridSample;
    float _imagedCenterNeighbourSize, _minIdentProba;
    bool _useLMDif, _searchForAnotherSegment, _writeOutput, _doIdentification;
    uint32_t _maxEdges;
    bool _useCuda = true;
    std::size_t _pinnedCounters = 100, _pinnedNearbyPoints = 60;
    std::string _debugDir;

    void setDebugDir(const std::string& d) { _debugDir = d; }
    void setUseCuda(bool) { _useCuda = true; }  // the B200 path is the only path

    cctagb_params to_c() const
    {
        cctagb_params p = _p;
        p.cannyThrLow = _cannyThrLow;
        p.cannyThrHigh = _cannyThrHigh;
        p.distSearch = int(_distSearch);
        p.thrGradientMagInVote = _thrGradientMagInVote;
        p.angleVoting = _angleVoting;
        p.ratioVoting = _ratioVoting;
        p.averageVoteMin = _averageVoteMin;
        p.thrMedianDistanceEllipse = _thrMedianDistanceEllipse;
        p.maximumNbSeeds = int(_maximumNbSeeds);
        p.maximumNbCandidatesLoopTwo = int(_maximumNbCandidatesLoopTwo);
        p.nCrowns = int(_nCrowns);
        p.nCircles = int(2 * _nCrowns);
        p.minPointsSegmentCandidate = int(_minPointsSegmentCandidate);
        p.minVotesToSelectCandidate = int(_minVotesToSelectCandidate);
        p.threshRobustEstimationOfOuterEllipse = _threshRobustEstimationOfOuterEllipse;
        p.ellipseGrowingEllipticHullWidth = _ellipseGrowingEllipticHullWidth;
        p.windowSizeOnInnerEllipticSegment = int(_windowSizeOnInnerEllipticSegment);
        p.numberOfMultiresLayers = int(_numberOfMultiresLayers);
        p.numberOfProcessedMultiresLayers = int(_numberOfProcessedMultiresLayers);
        p.nSamplesOuterEllipse = int(_nSamplesOuterEllipse);
        p.numCutsInIdentStep = int(_numCutsInIdentStep);
        p.numSamplesOuterEdgePointsRefinement = int(_numSamplesOuterEdgePointsRefinement);
        p.cutsSelectionTrials = int(_cutsSelectionTrials);
        p.sampleCutLength = int(_sampleCutLength);
        p.imagedCenterNGridSample = int(_imagedCenterNGridSample);
        p.imagedCenterNeighbourSize = _imagedCenterNeighbourSize;
        p.minIdentProba = _minIdentProba;
        p.useLMDif = _useLMDif;
        p.searchForAnotherSegment = _searchForAnotherSegment;
        p.writeOutput = _writeOutput;
        p.doIdentification = _doIdentification;
        p.maxEdges = _maxEdges;
        return p;
    }

    // Reads the reference's Boost-XML parameter file shape
    // (<CCTagsParams><_cannyThrLow>0.01</_cannyThrLow>...).  Unknown tags are
    // ignored; returns false if the file cannot be opened.
    bool readXml(const std::string& path)
    {
        std::ifstream f(path);
        if (!f) return false;
        std::stringstream ss;
        ss << f.rdbuf();
        const std::string s = ss.str();
        auto num = [&](const char* tag, double& v) {
            const std::string open = std::string("<") + tag + ">";
            const std::size_t a = s.find(open);
            if (a == std::string::npos) return false;
            v = std::atof(s.c_str() + a + open.size());
            return true;
        };
        double v;
#define CCTAGB_XML(field) \
    if (num(#field, v)) field = static_cast<decltype(field)>(v);
        CCTAGB_XML(_cannyThrLow) CCTAGB_XML(_cannyThrHigh) CCTAGB_XML(_distSearch) CCTAGB_XML(_thrGradientMagInVote)
        CCTAGB_XML(_angleVoting) CCTAGB_XML(_ratioVoting) CCTAGB_XML(_averageVoteMin)
        CCTAGB_XML(_thrMedianDistanceEllipse) CCTAGB_XML(_maximumNbSeeds) CCTAGB_XML(_maximumNbCandidatesLoopTwo)
        CCTAGB_XML(_nCrowns) CCTAGB_XML(_minPointsSegmentCandidate) CCTAGB_XML(_minVotesToSelectCandidate)
        CCTAGB_XML(_threshRobustEstimationOfOuterEllipse) CCTAGB_XML(_ellipseGrowingEllipticHullWidth)
        CCTAGB_XML(_windowSizeOnInnerEllipticSegment) CCTAGB_XML(_numberOfMultiresLayers)
        CCTAGB_XML(_numberOfProcessedMultiresLayers) CCTAGB_XML(_nSamplesOuterEllipse)
        CCTAGB_XML(_numCutsInIdentStep) CCTAGB_XML(_numSamplesOuterEdgePointsRefinement)
        CCTAGB_XML(_cutsSelectionTrials) CCTAGB_XML(_sampleCutLength) CCTAGB_XML(_imagedCenterNGridSample)
        CCTAGB_XML(_imagedCenterNeighbourSize) CCTAGB_XML(_minIdentProba) CCTAGB_XML(_useLMDif)
        CCTAGB_XML(_searchForAnotherSegment) CCTAGB_XML(_writeOutput) CCTAGB_XML(_doIdentification)
        CCTAGB_XML(_maxEdges)
#undef CCTAGB_XML
        _nCircles = 2 * _nCrowns;
        return true;
    }

private:
    void sync_from()
    {
        _cannyThrLow = _p.cannyThrLow;
        _cannyThrHigh = _p.cannyThrHigh;
        _distSearch = std::size_t(_p.distSearch);
        _thrGradientMagInVote = _p.thrGradientMagInVote;
        _angleVoting = _p.angleVoting;
        _ratioVoting = _p.ratioVoting;
        _averageVoteMin = _p.averageVoteMin;
        _thrMedianDistanceEllipse = _p.thrMedianDistanceEllipse;
        _maximumNbSeeds = std::size_t(_p.maximumNbSeeds);
        _maximumNbCandidatesLoopTwo = std::size_t(_p.maximumNbCandidatesLoopTwo);
        _nCrowns = std::size_t(_p.nCrowns);
        _nCircles = std::size_t(_p.nCircles);
        _minPointsSegmentCandidate = std::size_t(_p.minPointsSegmentCandidate);
        _minVotesToSelectCandidate = std::size_t(_p.minVotesToSelectCandidate);
        _threshRobustEstimationOfOuterEllipse = _p.threshRobustEstimationOfOuterEllipse;
        _ellipseGrowingEllipticHullWidth = _p.ellipseGrowingEllipticHullWidth;
        _windowSizeOnInnerEllipticSegment = std::size_t(_p.windowSizeOnInnerEllipticSegment);
        _numberOfMultiresLayers = std::size_t(_p.numberOfMultiresLayers);
        _numberOfProcessedMultiresLayers = std::size_t(_p.numberOfProcessedMultiresLayers);
        _nSamplesOuterEllipse = std::size_t(_p.nSamplesOuterEllipse);
        _numCutsInIdentStep = std::size_t(_p.numCutsInIdentStep);
        _numSamplesOuterEdgePointsRefinement = std::size_t(_p.numSamplesOuterEdgePointsRefinement);
        _cutsSelectionTrials = std::size_t(_p.cutsSelectionTrials);
        _sampleCutLength = std::size_t(_p.sampleCutLength);
        _imagedCenterNGridSample = std::size_t(_p.imagedCenterNGridSample);
        _imagedCenterNeighbourSize = _p.imagedCenterNeighbourSize;
        _minIdentProba = _p.minIdentProba;
        _useLMDif = _p.useLMDif != 0;
        _searchForAnotherSegment = _p.searchForAnotherSegment != 0;
        _writeOutput = _p.writeOutput != 0;
        _doIdentification = _p.doIdentification != 0;
        _maxEdges = _p.maxEdges;
    }
    cctagb_params _p;
};

// CCTagMarkersBank.hpp: built-in bank for nCrowns, or a text file of ratios.
class CCTagMarkersBank {
public:
    explicit CCTagMarkersBank(std::size_t nCrowns) : _nCrowns(nCrowns) {}
    explicit CCTagMarkersBank(const std::string& file) { read(file); }
    void read(const std::string& file)
    {
        std::ifstream in(file);
        if (!in.good()) throw std::ios_base::failure("Unable to open the bank file: " + file);
        std::string line;
        while (std::getline(in, line)) {
            std::vector<float> rr;
            std::stringstream ss(line);
            float v;
            while (ss >> v) rr.push_back(v);
            if (!rr.empty()) _markers.push_back(rr);
        }
    }
    const std::vector<std::vector<float>>& getMarkers() const { return _markers; }
    bool builtin() const { return _markers.empty(); }

private:
    std::size_t _nCrowns = 3;
    std::vector<std::vector<float>> _markers;
};

// ICCTag.hpp:28-82
class ICCTag {
public:
    ICCTag() = default;
    virtual float x() const = 0;
    virtual float y() const = 0;
    virtual MarkerID id() const = 0;
    virtual int getStatus() const = 0;
    virtual const numerical::geometry::Ellipse& rescaledOuterEllipse() const = 0;
    virtual ~ICCTag() = default;
    virtual ICCTag* clone() const = 0;

protected:
    float _x{0.f};
    float _y{0.f};
    MarkerID _id{UndefinedMarkerID};
    int _status{-1};
};

inline ICCTag* new_clone(const ICCTag& a) { return a.clone(); }

class CCTag : public ICCTag {
public:
    explicit CCTag(const cctagb_marker& m) : _m(m), _ellipse(m.outer)
    {
        _x = m.x;
        _y = m.y;
        _id = m.id;
        _status = m.status;
    }
    float x() const override { return _x; }
    float y() const override { return _y; }
    MarkerID id() const override { return _id; }
    int getStatus() const override { return _status; }
    const numerical::geometry::Ellipse& rescaledOuterEllipse() const override { return _ellipse; }
    ICCTag* clone() const override { return new CCTag(*this); }
    float quality() const { return _m.quality; }
    int pyramidLevel() const { return _m.pyramidLevel; }
    float scale() const { return _m.scale; }
    const float* homography() const { return _m.homography; }
    bool operator<(const CCTag& o) const { return _id < o._id; }

private:
    cctagb_marker _m;
    numerical::geometry::Ellipse _ellipse;
};

struct GrayView {
    const unsigned char* data;
    int cols, rows;
    std::size_t step;
};

namespace detail {

// pipeId -> handle registry (the reference keeps one CUDA pipeline per pipeId,
// Detection.cpp:61-67,732-760); a handle grows when a larger frame arrives.
struct Registry {
    struct Entry {
        cctagb_handle* h = nullptr;
        int w = 0, hgt = 0;
        std::vector<float> bank;
        int bank_rows = 0;
    };
    std::mutex mu;
    std::map<int, Entry> pipes;
    ~Registry()
    {
        for (auto& kv : pipes)
            if (kv.second.h) cctagb_destroy(kv.second.h);
    }
    static Registry& get()
    {
        static Registry r;
        return r;
    }
};

inline void detect_impl(std::vector<cctagb_marker>& out, int pipeId, std::size_t frame, const GrayView& g,
                        const Parameters& params, logtime::Mgmt* durations, const CCTagMarkersBank* pBank)
{
    Registry& reg = Registry::get();
    std::lock_guard<std::mutex> lock(reg.mu);
    Registry::Entry& e = reg.pipes[pipeId];
    const cctagb_params cp = params.to_c();
    if (!e.h || g.cols > e.w || g.rows > e.hgt) {
        if (e.h) cctagb_destroy(e.h);
        e.h = nullptr;
        const cctagb_status st = cctagb_create(&cp, g.cols, g.rows, 1, &e.h);
        if (st != CCTAGB_OK) throw std::runtime_error(std::string("cctagb_create: ") + cctagb_status_string(st));
        e.w = g.cols;
        e.hgt = g.rows;
        e.bank_rows = 0;
    }
    if (pBank && !pBank->builtin()) {
        std::vector<float> flat;
        for (const auto& r : pBank->getMarkers()) flat.insert(flat.end(), r.begin(), r.end());
        const int rows = int(pBank->getMarkers().size());
        if (flat != e.bank) {
            const cctagb_status st = cctagb_set_bank(e.h, flat.data(), rows, rows ? int(flat.size() / rows) : 0);
            if (st != CCTAGB_OK) throw std::runtime_error(cctagb_last_error_string(e.h));
            e.bank = flat;
            e.bank_rows = rows;
        }
    }
    int n = 0;
    cctagb_stats stats{};
    out.resize(256);
    cctagb_status st = cctagb_detect(e.h, g.data, g.cols, g.rows, g.step, int(frame), out.data(), int(out.size()),
                                     &n, &stats);
    if (st == CCTAGB_BAD_ARG && n > int(out.size())) {
        out.resize(size_t(n));
        st = cctagb_detect(e.h, g.data, g.cols, g.rows, g.step, int(frame), out.data(), int(out.size()), &n, &stats);
    }
    if (st != CCTAGB_OK) throw std::runtime_error(cctagb_last_error_string(e.h));
    out.resize(size_t(n));
    if (durations) {
        durations->log("image stage (device)", stats.ms_image_stage);
        durations->log("candidates (host)", stats.ms_host_candidates);
        durations->log("identification (device)", stats.ms_identify);
        durations->log("total", stats.ms_total);
    }
}

template <class M>
GrayView view_of(const M& m)
{
    return GrayView{reinterpret_cast<const unsigned char*>(m.data), int(m.cols), int(m.rows), std::size_t(m.step)};
}
inline GrayView view_of(const GrayView& g) { return g; }

template <class Container>
void fill(Container& markers, const std::vector<cctagb_marker>& out)
{
    markers.clear();
    for (const auto& m : out) markers.push_back(new CCTag(m));
}
inline void fill(std::vector<std::unique_ptr<ICCTag>>& markers, const std::vector<cctagb_marker>& out)
{
    markers.clear();
    for (const auto& m : out) markers.emplace_back(new CCTag(m));
}

}  // namespace detail

// ICCTag.hpp:125-131
template <class Container, class Image>
void cctagDetection(Container& markers, int pipeId, std::size_t frame, const Image& graySrc,
                    const Parameters& params, logtime::Mgmt* durations = nullptr,
                    const CCTagMarkersBank* pBank = nullptr)
{
    std::vector<cctagb_marker> out;
    detail::detect_impl(out, pipeId, frame, detail::view_of(graySrc), params, durations, pBank);
    detail::fill(markers, out);
}

// ICCTag.hpp:103-110: a missing parameter file prints a message and returns
// with an empty list (ICCTag.cpp:51-54).
template <class Container, class Image>
void cctagDetection(Container& markers, int pipeId, std::size_t frame, const Image& graySrc, std::size_t nRings = 3,
                    logtime::Mgmt* durations = nullptr, const std::string& parameterFile = "",
                    const std::string& cctagBankFilename = "")
{
    Parameters params(nRings);
    if (!parameterFile.empty() && !params.readXml(parameterFile)) {
        std::cerr << "\nThe input parameter file \"" << parameterFile << "\" is missing" << std::endl;
        return;
    }
    if (!cctagBankFilename.empty()) {
        CCTagMarkersBank bank(cctagBankFilename);
        cctagDetection(markers, pipeId, frame, graySrc, params, durations, &bank);
    } else {
        cctagDetection(markers, pipeId, frame, graySrc, params, durations, nullptr);
    }
}

}  // namespace cctag
