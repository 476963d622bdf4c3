"""Pins the CPU oracle against the reference's own outputs (CPU only).

The golden fixtures were produced by the reference's binaries (oracle/_ref, compiled from the
reference sources) -- see tests/golden/make_golden.py. The oracle must reproduce them bit for bit:
same MIT table, byte-identical index files, identical scores, accept codes, counts and distinct
counts for every method and threshold, early exits included.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import CASE_NAMES, GOLDEN, REPO, c0_full_index, load_case

METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}


def test_mit_table_formula_matches_reference_table(oracle, penalties):
    masks, vals = oracle.mit_table()
    assert len(masks) == 6195
    np.testing.assert_array_equal(masks, penalties["mit_masks"])
    np.testing.assert_array_equal(vals, penalties["mit_vals"])  # bit-exact


def test_golden_penalties_cross_checked_against_legacy_index(penalties):
    raw = penalties["raw"]
    assert raw["legacy_pairs_equal"] is True
    assert raw["legacy_header"][:3] == [39, 20, 43] and raw["legacy_header"][5] == 6195
    assert penalties["cfd_pam"][0b1010] == 1.0  # PAM NGG


def test_encoding(oracle):
    assert oracle.encode("ACGTACGTACGTACGTACGT") == sum(((j % 4) << (2 * j)) for j in range(20))
    # every non-CGT byte encodes as A (lowercase included)
    assert oracle.encode("NNNNNNNNNNNNNNNNNNNN") == 0
    assert oracle.encode("cgtacgtacgtacgtacgta") == 0


@pytest.mark.parametrize("name", CASE_NAMES)
def test_builder_reproduces_reference_index(oracle, name):
    z, meta = load_case(name)
    ix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "x.issl")
        ix.write(p)
        digest = hashlib.sha256(open(p, "rb").read()).hexdigest()
    assert digest == meta["index_sha256"]


def _check_case(oracle, ix, z, meta):
    exits = 0
    for meth in meta["methods"]:
        for t in meta["thresholds"]:
            k = f"{meth}_{t}"
            tm, tc, cnt, dist = ix.score(z["queries"], METHODS[meth], t)
            ms, cs, codes = oracle.finalise(METHODS[meth], t, tm, tc)
            np.testing.assert_array_equal(ms, z["mit_" + k], err_msg=k)
            np.testing.assert_array_equal(cs, z["cfd_" + k], err_msg=k)
            assert codes == z["code_" + k].tobytes(), k
            np.testing.assert_array_equal(cnt, z["count_" + k], err_msg=k)
            assert dist == int(z["distinct_" + k][0]), k
            exits += int((codes == b"0" * len(codes)) is False)
    return exits


@pytest.mark.parametrize("name", CASE_NAMES)
def test_oracle_scores_equal_reference(oracle, name):
    z, meta = load_case(name)
    ix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    _check_case(oracle, ix, z, meta)


def test_oracle_tiny_genome_equals_reference(oracle):
    z, meta = load_case("tiny")
    ix = oracle.Index.load(os.path.join(GOLDEN, "tiny_genome.issl"))
    _check_case(oracle, ix, z, meta)


@pytest.mark.parametrize("name", CASE_NAMES)
def test_candidate_set_equals_bruteforce(oracle, name):
    """Every sample slice config leaves some slice free of any <=4 mismatch positions, so the
    ISSL candidate set equals the brute-force set; with no early exit the sums agree."""
    z, _ = load_case(name)
    ix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    tm, tc, cnt, _ = ix.score(z["queries"], METHODS["mitAndCfd"], 1e-9)  # threshold ~0: no exit
    bm, bc, bcnt = oracle.bruteforce(z["sites"], z["occ"], z["queries"])
    np.testing.assert_array_equal(cnt, bcnt)
    np.testing.assert_allclose(tm, bm, rtol=1e-12, atol=0)
    np.testing.assert_allclose(tc, bc, rtol=1e-12, atol=0)


def test_early_exit_is_exercised(oracle):
    """The golden cases must include guides that stop early (scores depend on the stop point)."""
    z, meta = load_case("c2_small")  # 20% repeat-derived guides
    ix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    tm_full, tc_full, _, _ = ix.score(z["queries"], METHODS["mitAndCfd"], 1e-9)
    tm_exit, tc_exit, _, _ = ix.score(z["queries"], METHODS["mitAndCfd"], 99.0)
    assert np.sum(tm_exit < tm_full) > 20 and np.sum(tc_exit < tc_full) > 20


def _knife_entries(oracle):
    z, meta = load_case("knife")
    ix = oracle.Index.build(z["sites"], z["occ"], z["masks"])
    return z, meta, ix


def test_oracle_equals_reference_on_knife_edge_thresholds(oracle):
    """Thresholds whose maximum_sum sits within a few ulps of a running sum: the oracle's
    one-at-a-time sums reproduce the reference's scores, codes and counts bit for bit."""
    z, meta, ix = _knife_entries(oracle)
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "k.issl")
        ix.write(p)
        assert hashlib.sha256(open(p, "rb").read()).hexdigest() == meta["index_sha256"]
    for i in range(len(z["guide"])):
        g, m, thr = int(z["guide"][i]), int(z["method"][i]), float(z["threshold"][i])
        tm, tc, cnt, _ = ix.score(z["queries"][g:g + 1], m, thr)
        ms, cs, code = oracle.finalise(m, thr, tm, tc)
        assert (ms[0], cs[0], code[0], int(cnt[0])) == (z["mit"][i], z["cfd"][i], z["code"][i], int(z["count"][i])), i


def test_knife_edge_fixture_has_teeth(oracle):
    """The knife-edge fixture exercises the reference's rounding: for many entries a decision
    taken on exactly summed totals would differ, in every method, and the recorded flag agrees
    with a recomputation from the oracle's trace of the guide."""
    import knife_edge
    z, meta, ix = _knife_entries(oracle)
    names = list(knife_edge.METHODS)
    assert int(z["exact_differs"].sum()) > 100
    assert set(z["method"][z["exact_differs"]].tolist()) == set(range(5))
    for i in range(0, len(z["guide"]), 7):
        mt, ct, _ = ix.trace(int(z["queries"][int(z["guide"][i])]))
        assert knife_edge.exact_decision_differs(names[int(z["method"][i])], float(z["threshold"][i]), mt, ct) == \
            bool(z["exact_differs"][i])


def test_oracle_equals_reference_config0_full(oracle):
    z, meta, sites, occ, masks = c0_full_index()
    ix = oracle.Index.build(sites, occ, masks)
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "c0.issl")
        ix.write(p)
        assert hashlib.sha256(open(p, "rb").read()).hexdigest() == meta["index_sha256"]
    for meth, ts in meta["thresholds"].items():
        for t in ts:
            k = f"{meth}_{t}"
            tm, tc, cnt, dist = ix.score(z["queries"], METHODS[meth], t)
            ms, cs, codes = oracle.finalise(METHODS[meth], t, tm, tc)
            np.testing.assert_array_equal(ms, z["mit_" + k], err_msg=k)
            np.testing.assert_array_equal(cs, z["cfd_" + k], err_msg=k)
            assert codes == z["code_" + k].tobytes(), k
            np.testing.assert_array_equal(cnt, z["count_" + k], err_msg=k)
            assert dist == int(z["distinct_" + k][0]), k


def test_slice_configs_match_fixture_masks():
    from cracklingplusplus_gpu_b200.slice_configs import slice_masks
    for name in CASE_NAMES:
        z, meta = load_case(name)
        assert [int(m) for m in z["masks"]] == slice_masks(meta["config"])


REF_BIN = os.path.join(REPO, "oracle", "_ref")
from refpath import REFERENCE as REF_SRC  # noqa: E402  (oracle/ is on the path, conftest.py)


@pytest.mark.skipif(not (os.path.isdir(REF_SRC) and os.path.exists(os.path.join(REF_BIN, "ref_module_driver"))),
                    reason="needs the reference checkout and oracle/_ref binaries")
def test_oracle_equals_live_reference_on_fresh_case(oracle, tmp_path):
    """A case not in the fixtures, run through the reference binaries here and now."""
    import synth
    from make_golden import ref_build_index, ref_cli, ref_module
    from cracklingplusplus_gpu_b200.slice_configs import SLICE_CONFIGS
    sites, occ, queries = synth.make_case(97, 8000, 80, repeat_frac=0.1, n_seeds=10)
    idx = str(tmp_path / "f.issl")
    seqs = ref_build_index(sites, occ, SLICE_CONFIGS["slice-8-20"], idx, str(tmp_path))
    ix = oracle.Index.load(idx)
    qs = [synth.sig_to_seq(q) for q in queries.tolist()]
    for meth, cli in [("mitAndCfd", "and"), ("avgMitCfd", "avg")]:
        m, c, codes = ref_module(idx, qs, meth, 90.0, str(tmp_path))
        cnt, distinct = ref_cli(idx, qs, cli, 90.0, str(tmp_path))
        tm, tc, ocnt, odist = ix.score(queries, METHODS[meth], 90.0)
        ms, cs, ocodes = oracle.finalise(METHODS[meth], 90.0, tm, tc)
        np.testing.assert_array_equal(ms, m)
        np.testing.assert_array_equal(cs, c)
        assert ocodes == codes.tobytes()
        np.testing.assert_array_equal(ocnt, cnt)
        assert odist == distinct
