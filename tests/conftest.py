"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (REPO, os.path.join(REPO, "oracle"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the native CUDA path)")


@pytest.fixture(scope="session")
def penalties():
    pen = json.load(open(os.path.join(GOLDEN, "penalties.json")))
    masks = np.array([k for k, _ in pen["mit"]], np.uint64)
    vals = np.array([float.fromhex(v) for _, v in pen["mit"]])
    pos = np.array([float.fromhex(v) for v in pen["cfd_pos"]])
    pam = np.array([float.fromhex(v) for v in pen["cfd_pam"]])
    return {"mit_masks": masks, "mit_vals": vals, "cfd_pos": pos, "cfd_pam": pam, "raw": pen}


@pytest.fixture(scope="session")
def oracle(penalties):
    import pyoracle
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    pyoracle.set_cfd_tables(penalties["cfd_pos"], penalties["cfd_pam"])
    return pyoracle


@pytest.fixture(scope="session")
def native():
    from cracklingplusplus_gpu_b200 import build
    build.build()
    import cracklingplusplus_gpu_b200 as pkg
    pkg.lib()
    return pkg


def load_case(name):
    z = np.load(os.path.join(GOLDEN, f"case_{name}.npz"))
    meta = json.loads(str(z["meta"]))
    return z, meta


CASE_NAMES = ["c0_small", "c1_small", "c2_small", "c4_small"]


def c0_full_index():
    """Config 0 at its stated size, regenerated from its seed in the reference's site order."""
    import synth
    from cracklingplusplus_gpu_b200.slice_configs import slice_masks
    z, meta = load_case("c0_full")
    sites, occ, queries = synth.make_case(meta["seed"], meta["n_sites"], meta["n_queries"], repeat_frac=0.0,
                                          planted_into_sites=True)
    order = synth.reference_order(sites)
    occ_of = dict(zip(sites.tolist(), occ.tolist()))
    occ_sorted = np.array([occ_of[int(s)] for s in order.tolist()], np.uint32)
    np.testing.assert_array_equal(queries, z["queries"])
    return z, meta, order, occ_sorted, np.array(slice_masks(meta["config"]), np.uint64)


def extract_fixture(root):
    """Writes the extraction fixture's input files under `root`; returns (input paths as the
    reference was given them, the reference's output bytes, meta)."""
    z, meta = load_case("extract")
    for i, rel in enumerate(meta["inputs"]):
        p = os.path.join(root, rel)
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "wb") as f:
            f.write(z[f"input_{i}"].tobytes())
    return [os.path.join(root, a) for a in meta["args"]], z["output"].tobytes(), meta
