"""Python face of the drop-in ISSLScoringModule (include/issl_b200_module.hpp).

Mirrors the reference's `ISSLScoringModule(const cracklingConfig&)` + `run(vector<guideResults>&)`
(include/ISSLScoringModule.hpp:15-29): run() scores the guides that pass processGuide
(lib/ISSLScoringModule.cpp:488-513) and writes mitOfftargetscore, cfdOfftargetscore and
passedOffTargetScore in place. The work happens in the C++ class inside libissl_b200.so.
"""
from __future__ import annotations

import ctypes as C
import sys
from dataclasses import dataclass, field
from typing import List

import numpy as np

from ._lib import OT_METHODS, check, lib

OPTIMISATION = {"ultralow": 0, "low": 1, "medium": 2, "high": 3}  # include/util.hpp:21


@dataclass
class GuideResults:
    """The guideResults fields (include/util.hpp:112-140) the off-target module reads/writes."""
    seq: str = "-"
    isUnique: bool = False
    consensusCount: int = 0
    passedBowtie2: str = "?"
    passedOffTargetScore: str = "?"
    mitOfftargetscore: float = -sys.float_info.max
    cfdOfftargetscore: float = -sys.float_info.max


@dataclass
class CracklingConfig:
    """The cracklingConfig fields the module uses: input.offtargetSites, offTarget.{enabled,
    method, scoreThreshold, memoryMapped}, general.optimisation, consensus.n (threads/pageLen are
    accepted and unused). memoryMapped keeps the lists in host memory (Index.open_mapped)."""
    offtargetSites: str
    method: str = "mitAndCfd"
    scoreThreshold: float = 75.0
    enabled: bool = True
    optimisation: str = "ultralow"
    consensusN: int = 0
    threads: int = 0
    memoryMapped: bool = False
    extra: dict = field(default_factory=dict)


class ISSLScoringModule:
    def __init__(self, config: CracklingConfig):
        if config.method not in OT_METHODS:
            raise RuntimeError("Scoring method is not valid.")
        self.config = config

    def run(self, candidateGuides: List[GuideResults]) -> None:
        cfg = self.config
        n = len(candidateGuides)
        stride = max([len(g.seq) for g in candidateGuides] + [20]) + 1
        buf = b"".join(g.seq.encode().ljust(stride, b"\0") for g in candidateGuides)
        uniq = np.array([1 if g.isUnique else 0 for g in candidateGuides] + [0], np.uint8)
        cons = np.array([g.consensusCount for g in candidateGuides] + [0], np.int8)
        bt2 = bytes(ord(g.passedBowtie2[0]) for g in candidateGuides) + b"\0"
        mit = np.array([g.mitOfftargetscore for g in candidateGuides] + [0.0])
        cfd = np.array([g.cfdOfftargetscore for g in candidateGuides] + [0.0])
        code = C.create_string_buffer(bytes(ord(g.passedOffTargetScore[0]) for g in candidateGuides) + b"\0")
        f = C.POINTER(C.c_double)
        check(lib().issl_module_run(cfg.offtargetSites.encode(), OT_METHODS[cfg.method], cfg.scoreThreshold,
                                    OPTIMISATION[cfg.optimisation], cfg.consensusN,
                                    int(cfg.enabled) | (2 if cfg.memoryMapped else 0), n, buf, stride,
                                    uniq.ctypes.data_as(C.POINTER(C.c_uint8)),
                                    cons.ctypes.data_as(C.POINTER(C.c_int8)), bt2, mit.ctypes.data_as(f),
                                    cfd.ctypes.data_as(f), code))
        for i, g in enumerate(candidateGuides):
            g.mitOfftargetscore = float(mit[i])
            g.cfdOfftargetscore = float(cfd[i])
            g.passedOffTargetScore = chr(code.raw[i])


def release_all() -> None:
    """Drops the indexes the module keeps resident between run() calls."""
    check(lib().issl_module_release_all())
