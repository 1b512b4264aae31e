// Reference-style use of the drop-in API: cctag::cctagDetection with
// cctag::Parameters and a list of ICCTag, on a raw 8-bit frame read from a file
// (width height then w*h bytes), printing one line per marker.
#include <cstdio>
#include <fstream>
#include <memory>
#include <vector>

#include "cctag_b200/ICCTag.hpp"

struct Frame {  // a minimal cv::Mat look-alike
    std::vector<unsigned char> buf;
    unsigned char* data;
    int cols, rows;
    size_t step;
};

template <class T>
struct PtrList {  // boost::ptr_list look-alike: owns raw pointers
    std::vector<std::unique_ptr<T>> v;
    void clear() { v.clear(); }
    void push_back(T* p) { v.emplace_back(p); }
};

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    std::ifstream in(argv[1], std::ios::binary);
    int w = 0, h = 0;
    in.read(reinterpret_cast<char*>(&w), 4);
    in.read(reinterpret_cast<char*>(&h), 4);
    Frame f;
    f.buf.resize(size_t(w) * h);
    in.read(reinterpret_cast<char*>(f.buf.data()), f.buf.size());
    f.data = f.buf.data();
    f.cols = w;
    f.rows = h;
    f.step = size_t(w);

    cctag::Parameters params(3);
    PtrList<cctag::ICCTag> markers;
    cctag::logtime::Mgmt durations(25);
    cctag::cctagDetection(markers, 0, 0, f, params, &durations);
    for (const auto& m : markers.v)
        std::printf("%d %d %.4f %.4f %.3f %.3f\n", m->id(), m->getStatus(), m->x(), m->y(),
                    m->rescaledOuterEllipse().a(), m->rescaledOuterEllipse().b());
    // the nRings overload with a missing parameter file returns an empty list
    std::vector<std::unique_ptr<cctag::ICCTag>> none;
    cctag::cctagDetection(none, 1, 0, f, 3, nullptr, "/nonexistent/params.xml");
    return none.empty() ? 0 : 1;
}
