"""Regression logs in the reference's format, so that its regression harness
and this library can check each other.

The reference's regression tool (``applications/regression/TestLog.h``,
``TestLog.cpp``, ``Regression.cpp``) stores, per input file, a ``FileLog``
(file name, the ``cctag::Parameters`` used, one ``FrameLog`` per frame with the
frame number, the detection time and the detected tags' id, status, x, y and
quality) as a Boost XML archive, and compares two such logs frame by frame:
tags with status < 1 are dropped, the rest sorted by id (duplicate ids fail),
then every tag must agree in reliability, id and position within epsilon.

``FileLog.save`` writes that archive layout (``class_id``/``tracking_level``/
``version`` on the first element of each class, ``count``/``item_version`` in
collections); ``FileLog.load`` reads it (attributes are not required);
``compare`` applies the checker's rules.
"""
from __future__ import annotations

import time
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field

import numpy as np

# Params.hpp serialize() order (cctag::Parameters), with the library field
# each maps to (None: written with the reference's default, not used here).
PARAM_FIELDS = [
    ("_cannyThrLow", "cannyThrLow", float), ("_cannyThrHigh", "cannyThrHigh", float),
    ("_distSearch", "distSearch", int), ("_thrGradientMagInVote", "thrGradientMagInVote", int),
    ("_angleVoting", "angleVoting", float), ("_ratioVoting", "ratioVoting", float),
    ("_averageVoteMin", "averageVoteMin", float), ("_thrMedianDistanceEllipse", "thrMedianDistanceEllipse", float),
    ("_maximumNbSeeds", "maximumNbSeeds", int), ("_maximumNbCandidatesLoopTwo", "maximumNbCandidatesLoopTwo", int),
    ("_nCrowns", "nCrowns", int), ("_minPointsSegmentCandidate", "minPointsSegmentCandidate", int),
    ("_minVotesToSelectCandidate", "minVotesToSelectCandidate", int),
    ("_threshRobustEstimationOfOuterEllipse", "threshRobustEstimationOfOuterEllipse", float),
    ("_ellipseGrowingEllipticHullWidth", "ellipseGrowingEllipticHullWidth", float),
    ("_windowSizeOnInnerEllipticSegment", "windowSizeOnInnerEllipticSegment", int),
    ("_numberOfMultiresLayers", "numberOfMultiresLayers", int),
    ("_numberOfProcessedMultiresLayers", "numberOfProcessedMultiresLayers", int),
    ("_nSamplesOuterEllipse", "nSamplesOuterEllipse", int), ("_numCutsInIdentStep", "numCutsInIdentStep", int),
    ("_numSamplesOuterEdgePointsRefinement", "numSamplesOuterEdgePointsRefinement", int),
    ("_cutsSelectionTrials", "cutsSelectionTrials", int), ("_sampleCutLength", "sampleCutLength", int),
    ("_imagedCenterNGridSample", "imagedCenterNGridSample", int),
    ("_imagedCenterNeighbourSize", "imagedCenterNeighbourSize", float), ("_minIdentProba", "minIdentProba", float),
    ("_useLMDif", "useLMDif", int), ("_searchForAnotherSegment", "searchForAnotherSegment", int),
    ("_writeOutput", "writeOutput", int), ("_doIdentification", "doIdentification", int),
    ("_maxEdges", "maxEdges", int), ("_useCuda", None, int), ("_pinnedCounters", None, int),
    ("_pinnedNearbyPoints", None, int),
]
_PARAM_EXTRA_DEFAULTS = {"_useCuda": 1, "_pinnedCounters": 100, "_pinnedNearbyPoints": 60}

ARCHIVE_VERSION = "17"


def _fmt(v, kind):
    if kind is float:
        return np.format_float_positional(np.float32(v), unique=True, trim="-") if np.isfinite(v) else repr(v)
    return str(int(v))


@dataclass
class DetectedTag:
    id: int
    status: int
    x: float
    y: float
    quality: float


@dataclass
class FrameLog:
    frame: int
    elapsedTime: float
    tags: list = field(default_factory=list)


@dataclass
class FileLog:
    filename: str
    parameters: dict                       # reference field name -> value
    frameLogs: list = field(default_factory=list)

    # -- writing ---------------------------------------------------------------
    def to_xml(self) -> str:
        out = ['<?xml version="1.0" encoding="UTF-8" standalone="yes" ?>', "<!DOCTYPE boost_serialization>",
               f'<boost_serialization signature="serialization::archive" version="{ARCHIVE_VERSION}">',
               '<FileLog class_id="0" tracking_level="0" version="0">',
               f"\t<filename>{_escape(self.filename)}</filename>",
               '\t<parameters class_id="1" tracking_level="0" version="0">']
        for name, _, kind in PARAM_FIELDS:
            out.append(f"\t\t<{name}>{_fmt(self.parameters[name], kind)}</{name}>")
        out.append("\t</parameters>")
        out.append('\t<frameLogs class_id="2" tracking_level="0" version="0">')
        out.append(f"\t\t<count>{len(self.frameLogs)}</count>")
        out.append("\t\t<item_version>0</item_version>")
        first_frame, first_tags, first_tag = True, True, True
        for fl in self.frameLogs:
            out.append('\t\t<item class_id="3" tracking_level="0" version="0">' if first_frame else "\t\t<item>")
            first_frame = False
            out.append(f"\t\t\t<frame>{int(fl.frame)}</frame>")
            out.append(f"\t\t\t<elapsedTime>{_fmt(fl.elapsedTime, float)}</elapsedTime>")
            out.append('\t\t\t<tags class_id="4" tracking_level="0" version="0">' if first_tags else "\t\t\t<tags>")
            first_tags = False
            out.append(f"\t\t\t\t<count>{len(fl.tags)}</count>")
            out.append("\t\t\t\t<item_version>0</item_version>")
            for t in fl.tags:
                out.append('\t\t\t\t<item class_id="5" tracking_level="0" version="0">' if first_tag
                           else "\t\t\t\t<item>")
                first_tag = False
                out.append(f"\t\t\t\t\t<id>{int(t.id)}</id>")
                out.append(f"\t\t\t\t\t<status>{int(t.status)}</status>")
                out.append(f"\t\t\t\t\t<x>{_fmt(t.x, float)}</x>")
                out.append(f"\t\t\t\t\t<y>{_fmt(t.y, float)}</y>")
                out.append(f"\t\t\t\t\t<quality>{_fmt(t.quality, float)}</quality>")
                out.append("\t\t\t\t</item>")
            out.append("\t\t\t</tags>")
            out.append("\t\t</item>")
        out.append("\t</frameLogs>")
        out.append("</FileLog>")
        out.append("</boost_serialization>")
        return "\n".join(out) + "\n"

    def save(self, path) -> None:
        with open(path, "w", encoding="utf-8") as f:
            f.write(self.to_xml())

    # -- reading ---------------------------------------------------------------
    @staticmethod
    def from_xml(text: str) -> "FileLog":
        # ElementTree does not accept the DOCTYPE without a DTD; drop it.
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("<!DOCTYPE"))
        root = ET.fromstring(text)
        fl = root.find("FileLog")
        if fl is None:
            raise ValueError("not a FileLog archive")
        params = {}
        pe = fl.find("parameters")
        for name, _, kind in PARAM_FIELDS:
            el = pe.find(name) if pe is not None else None
            if el is not None and el.text is not None:
                params[name] = int(float(el.text)) if kind is int else float(np.float32(el.text))
        frames = []
        for item in _items(fl.find("frameLogs")):
            tags = [DetectedTag(int(t.findtext("id")), int(t.findtext("status")), float(t.findtext("x")),
                                float(t.findtext("y")), float(t.findtext("quality")))
                    for t in _items(item.find("tags"))]
            frames.append(FrameLog(int(item.findtext("frame")), float(item.findtext("elapsedTime")), tags))
        return FileLog(fl.findtext("filename") or "", params, frames)

    @staticmethod
    def load(path) -> "FileLog":
        with open(path, encoding="utf-8") as f:
            return FileLog.from_xml(f.read())


def _items(coll):
    if coll is None:
        return []
    n = int(coll.findtext("count") or 0)
    items = coll.findall("item")
    if len(items) != n:
        raise ValueError(f"collection count {n} but {len(items)} items")
    return items


def _escape(s: str) -> str:
    return s.replace("&", "&amp;").replace("<", "&lt;").replace(">", "&gt;")


def parameters_of(params) -> dict:
    """Reference-named parameter dict from a ``cctag_b200.Params`` struct."""
    out = {}
    for name, lib, kind in PARAM_FIELDS:
        if lib is None:
            out[name] = _PARAM_EXTRA_DEFAULTS[name]
        else:
            v = getattr(params, lib)
            out[name] = int(v) if kind is int else float(np.float32(v))
    return out


def detect_frames(detector, filename: str, frames, params) -> FileLog:
    """FileLog of a sequence of gray frames run through ``detector`` (the
    reference's FileLog::detect, one FrameLog per frame)."""
    log = FileLog(filename, parameters_of(params))
    for i, gray in enumerate(frames):
        t0 = time.perf_counter()
        markers, _ = detector.detect(gray, frame_id=i)
        dt = time.perf_counter() - t0
        log.frameLogs.append(FrameLog(i, dt, [DetectedTag(m.id, m.status, m.x, m.y, m.quality) for m in markers]))
    return log


class CheckError(RuntimeError):
    pass


def _sorted_reliable(tags):
    kept = sorted((t for t in tags if t.status >= 1), key=lambda t: t.id)
    if any(a.id == b.id for a, b in zip(kept, kept[1:])):
        raise CheckError("duplicate IDs")
    return kept


def compare(reference: FileLog, test: FileLog, epsilon: float) -> dict:
    """The reference checker's rules; raises CheckError on the first
    mismatch, else returns the mean / stdev of the quality and elapsed-time
    differences (test - reference)."""
    if reference.filename != test.filename:
        raise CheckError("mismatching filenames")
    if reference.parameters.get("_nCrowns") != test.parameters.get("_nCrowns"):
        raise CheckError("mismatching parameters")
    if len(reference.frameLogs) != len(test.frameLogs):
        raise CheckError("mismatching frame counts")
    for log in (reference, test):
        if any(a.frame > b.frame for a, b in zip(log.frameLogs, log.frameLogs[1:])):
            raise CheckError("frames not monotonic")
    dq, dt = [], []
    for k, (rf, tf) in enumerate(zip(reference.frameLogs, test.frameLogs)):
        if len(rf.tags) != len(tf.tags):
            raise CheckError(f"different # of tags in frame {k}")
        rt, tt = _sorted_reliable(rf.tags), _sorted_reliable(tf.tags)
        dt.append(tf.elapsedTime - rf.elapsedTime)
        if len(rt) != len(tt):
            raise CheckError(f"tags of different status in frame {k}")
        for a, b in zip(rt, tt):
            dq.append(b.quality - a.quality)
            ra, rb = a.status == 1, b.status == 1
            if ra != rb:
                raise CheckError(f"tags of different status in frame {k}")
            if ra and rb:
                if a.id != b.id:
                    raise CheckError(f"tags with different IDs frame {k}")
                if abs(a.x - b.x) > epsilon or abs(a.y - b.y) > epsilon:
                    raise CheckError(f"tags at different positions in frame {k}")
    return {"quality_diff_mean": float(np.mean(dq)) if dq else 0.0,
            "quality_diff_stdev": float(np.std(dq)) if dq else 0.0,
            "elapsed_diff_mean": float(np.mean(dt)) if dt else 0.0,
            "elapsed_diff_stdev": float(np.std(dt)) if dt else 0.0}
