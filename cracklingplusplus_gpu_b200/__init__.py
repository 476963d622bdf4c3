"""B200-native ISSL off-target scoring (Crackling++ specificity path).

The compute path is the in-tree native library ``libissl_b200.so`` (CUDA kernels for sm_100a
behind the C ABI declared in ``include/issl_b200.h``). This package is a thin ctypes layer over it:
there is no Python or CPU fallback, and importing the bindings fails loudly when the library has
not been built (``python -m cracklingplusplus_gpu_b200.build``).

Python mirrors of the reference's interfaces:
  * ``Index``              -- a resident index: ``Index.open(path)`` replaces the per-call .issl read
                              of lib/ISSLScoringModule.cpp:72-150; ``score()`` is the scoring loop
  * ``ISSLScoringModule``  -- same constructor/run() contract as include/ISSLScoringModule.hpp:15-29
                              (through ``issl_module_run``, the C entry point behind the
                              header-only C++ class of include/issl_b200_module.hpp)
  * ``OT_METHODS`` / ``CLI_METHODS`` -- otScoreMethod numbering and the CLI's method words

Beyond the reference: ``Batch`` scores many guide sets (each with its own method, threshold and
mismatch bound) in one graph-captured pass; ``Index.autotune`` sweeps the scan's tile and staging
parameters per bucket-size class; ``Server`` admits guide-set requests by device-memory footprint
and scores them with continuous batching over several in-flight slots.
"""
from __future__ import annotations

from ._lib import (  # noqa: F401
    CLI_METHODS,
    OT_METHODS,
    IsslError,
    lib,
    library_path,
)
from .batch import Batch  # noqa: F401
from .index import Index, ScoreResult, SynthSpec, extract_offtargets, tables  # noqa: F401
from .module import CracklingConfig, GuideResults, ISSLScoringModule  # noqa: F401
from .server import Server  # noqa: F401
from .slice_configs import SLICE_CONFIGS, slice_masks  # noqa: F401
