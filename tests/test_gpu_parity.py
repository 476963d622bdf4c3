"""Parity of the CUDA path with the reference (golden fixtures) and the oracle. Needs a GPU.

Bar: accept codes, per-guide occurrence counts and distinct-site counts bit-exact; MIT and CFD
scores within 1e-12 relative of the reference's double sums (the GPU sums in a different order);
scores of a method's unused component exactly -1.
"""
from __future__ import annotations

import hashlib
import os
import subprocess

import numpy as np
import pytest

from conftest import CASE_NAMES, GOLDEN, c0_full_index, load_case

pytestmark = pytest.mark.gpu

RTOL = 1e-12
METHODS = {"mit": 0, "cfd": 1, "mitAndCfd": 2, "mitOrCfd": 3, "avgMitCfd": 4}


def assert_matches(res, mit, cfd, codes, counts=None, distinct=None, tag=""):
    assert res.code == bytes(codes), f"{tag}: accept codes differ"
    np.testing.assert_allclose(res.mit, mit, rtol=RTOL, atol=0, err_msg=tag)
    np.testing.assert_allclose(res.cfd, cfd, rtol=RTOL, atol=0, err_msg=tag)
    if counts is not None:
        np.testing.assert_array_equal(res.count, counts, err_msg=tag)
    if distinct is not None:
        assert res.distinct == distinct, tag


def check_golden(ix, z, meta):
    q = z["queries"]
    for meth in meta["methods"]:
        for t in meta["thresholds"]:
            k = f"{meth}_{t}"
            res = ix.score(q, meth, t)
            assert_matches(res, z["mit_" + k], z["cfd_" + k], z["code_" + k].tobytes(), z["count_" + k],
                           int(z["distinct_" + k][0]), tag=f"{meta['name']} {k}")


@pytest.fixture(scope="module")
def oracle_arrays(oracle):
    cache = {}

    def get(name):
        if name not in cache:
            z, _ = load_case(name)
            cache[name] = oracle.Index.build(z["sites"], z["occ"], z["masks"]).arrays()
        return cache[name]
    return get


@pytest.mark.parametrize("name", CASE_NAMES)
def test_golden_case(native, oracle_arrays, name):
    z, meta = load_case(name)
    with native.Index.from_arrays(*oracle_arrays(name)) as ix:
        check_golden(ix, z, meta)


def test_config0_full_size(native, tmp_path):
    """Config 0 at its stated size (1,000,000 sites, slice-4-5, 1,000 planted guides), built on the
    GPU from the seeded sites: the index file equals the reference builder's byte for byte and
    every method's results equal the reference's (module scores and codes, CLI counts and
    distinct-site counts)."""
    z, meta, sites, occ, masks = c0_full_index()
    with native.Index.build(sites, occ, masks) as ix:
        p = str(tmp_path / "c0.issl")
        ix.save(p)
        assert hashlib.sha256(open(p, "rb").read()).hexdigest() == meta["index_sha256"]
        for meth, ts in meta["thresholds"].items():
            for t in ts:
                k = f"{meth}_{t}"
                res = ix.score(z["queries"], meth, t)
                assert_matches(res, z["mit_" + k], z["cfd_" + k], z["code_" + k].tobytes(), z["count_" + k],
                               int(z["distinct_" + k][0]), tag=f"c0_full {k}")


@pytest.mark.parametrize("spec", [
    dict(seed=1235, n_sites=2_000_000, n_queries=2000),  # the benchmark's composition
    dict(seed=7, n_sites=300_000, n_queries=600, repeat_frac=0.2, n_repeat_seeds=50, repeat_query_frac=0.2,
         planted_into_sites=True),
])
def test_host_generator_equals_device_generator(native, oracle, spec):
    """The benchmark's reference arm builds its index without the library: the oracle's host
    restatement of the seeded generator (oracle/synth_oracle.c) must give the device generator's
    sites, occurrence counts and guides exactly."""
    ix, q = native.Index.synth(native.SynthSpec(slice_config="slice-8-20", **spec))
    with ix:
        sigs, _, _, lists = ix.export()
    n = len(sigs)
    occ = np.zeros(n, np.uint32)
    occ[(lists[:n] & 0xFFFFFFFF).astype(np.int64)] = (lists[:n] >> 32).astype(np.uint32)
    hs, ho, hq = oracle.synth(spec["seed"], spec["n_sites"], spec["n_queries"], repeat_frac=spec.get("repeat_frac", 0.05),
                              n_repeat_seeds=spec.get("n_repeat_seeds", 10000), copied_frac=0.5,
                              repeat_query_frac=spec.get("repeat_query_frac", 0.0),
                              planted_into_sites=spec.get("planted_into_sites", False))
    np.testing.assert_array_equal(hs, sigs)
    np.testing.assert_array_equal(ho, occ)
    np.testing.assert_array_equal(hq, q)


def test_tiny_genome_from_reference_file(native):
    z, meta = load_case("tiny")
    with native.Index.open(os.path.join(GOLDEN, "tiny_genome.issl")) as ix:
        check_golden(ix, z, meta)


@pytest.mark.parametrize("name", CASE_NAMES)
def test_gpu_builder_equals_reference_builder(native, oracle_arrays, name, tmp_path):
    z, meta = load_case(name)
    with native.Index.build(z["sites"], z["occ"], z["masks"]) as ix:
        for a, b in zip(ix.export(), oracle_arrays(name)):
            np.testing.assert_array_equal(a, b)
        p = str(tmp_path / "g.issl")
        ix.save(p)
        assert hashlib.sha256(open(p, "rb").read()).hexdigest() == meta["index_sha256"]


def test_ascii_guides_equal_signatures(native):
    from cracklingplusplus_gpu_b200.index import decode
    z, meta = load_case("c0_small")
    with native.Index.open(os.path.join(GOLDEN, "tiny_genome.issl")) as ix:
        q = load_case("tiny")[0]["queries"]
        seqs = [decode(s) + "AGG" for s in q]  # 23-mers: only the first 20 nt are scored
        a = ix.score(seqs, "and", 75.0)
        b = ix.score(q, "and", 75.0)
        assert a.code == b.code
        np.testing.assert_array_equal(a.mit, b.mit)
        np.testing.assert_array_equal(a.cfd, b.cfd)
        # any byte other than C, G, T encodes as A
        c = ix.score(["acgtNNNNacgtRYKMacgt", "AAAAAAAAAAAAAAAAAAAA"], "and", 75.0)
        assert c.code[0] == c.code[1]
        assert c.mit[0] == c.mit[1] and c.cfd[0] == c.cfd[1]


@pytest.mark.parametrize("max_dist", [0, 1, 2, 3])
def test_max_dist_filter(native, oracle, oracle_arrays, max_dist):
    z, _ = load_case("c1_small")
    arrays = oracle_arrays("c1_small")
    oix = oracle.Index.from_arrays(*arrays)
    with native.Index.from_arrays(*arrays) as ix:
        for meth in ["mitAndCfd", "avgMitCfd"]:
            tm, tc, cnt, dist = oix.score(z["queries"], METHODS[meth], 90.0, max_dist=max_dist)
            ms, cs, codes = oracle.finalise(METHODS[meth], 90.0, tm, tc)
            res = ix.score(z["queries"], meth, 90.0, max_dist=max_dist)
            assert_matches(res, ms, cs, codes, cnt, dist, tag=f"max_dist={max_dist} {meth}")


def _neighbourhood_index(oracle):
    """A site plus all its 1- and 2-substitution neighbours (1,770 sites within distance 2) and
    random background: guides near the centre have far more hits than a warp holds."""
    import synth
    rng_sites = synth.random_sigs(synth.Stream(5, 1), 3000)
    centre = int(rng_sites[0])
    nbrs = set()
    for p in range(20):
        for d in range(1, 4):
            v = centre ^ (d << (2 * p))
            nbrs.add(v)
            for p2 in range(p + 1, 20):
                for d2 in range(1, 4):
                    nbrs.add(v ^ (d2 << (2 * p2)))
    sites = np.array(sorted(nbrs | {centre} | set(int(s) for s in rng_sites)), np.uint64)
    occ = synth.occurrences(synth.Stream(5, 2), len(sites))
    from cracklingplusplus_gpu_b200.slice_configs import slice_masks
    masks = np.array(slice_masks("slice-8-20"), np.uint64)
    queries = np.array([centre, centre ^ (1 << 10), centre ^ (2 << 30) ^ (1 << 4)] + [int(s) for s in rng_sites[1:40]],
                       np.uint64)
    return sites, occ, masks, queries


def test_many_hits_block_scorer_and_early_exit(native, oracle):
    sites, occ, masks, queries = _neighbourhood_index(oracle)
    oix = oracle.Index.build(sites, occ, masks)
    with native.Index.from_arrays(*oix.arrays()) as ix:
        for meth in METHODS:
            for t in [1e-9, 20.0, 50.0, 90.0, 99.99]:
                tm, tc, cnt, dist = oix.score(queries, METHODS[meth], t)
                ms, cs, codes = oracle.finalise(METHODS[meth], t, tm, tc)
                res = ix.score(queries, meth, t)
                assert_matches(res, ms, cs, codes, cnt, dist, tag=f"{meth} t={t}")
        _, _, cnt, _ = oix.score(queries, 2, 1e-9)
        assert int(np.max(cnt)) > 1000  # the centre guides go through the block scorer


def test_synthetic_device_workload_against_oracle(native, oracle):
    spec = native.SynthSpec(seed=7, n_sites=200_000, slice_config="slice-8-20", n_queries=3000,
                            repeat_frac=0.05, n_repeat_seeds=300, repeat_query_frac=0.2)
    ix, q = native.Index.synth(spec)
    with ix:
        arrays = ix.export()
        assert len(np.unique(arrays[0])) == spec.n_sites  # distinct sites
        oix = oracle.Index.from_arrays(*arrays)
        for meth, t in [("mitAndCfd", 75.0), ("mitOrCfd", 90.0), ("avgMitCfd", 50.0), ("cfd", 99.0), ("mit", 75.0)]:
            tm, tc, cnt, dist = oix.score(q, METHODS[meth], t)
            ms, cs, codes = oracle.finalise(METHODS[meth], t, tm, tc)
            res = ix.score(q, meth, t)
            assert_matches(res, ms, cs, codes, cnt, dist, tag=f"synth {meth} {t}")


def test_planted_workload_has_every_distance(native, oracle):
    spec = native.SynthSpec(seed=3, n_sites=50_000, slice_config="slice-4-5", n_queries=1000,
                            planted_into_sites=True)
    ix, q = native.Index.synth(spec)
    with ix:
        sigs = ix.export()[0]
        s = set(int(x) for x in sigs)
        copied = [int(x) for x in q if int(x) in s]
        assert len(copied) >= 450  # exact site copies (their mutants were added to the sites)
        x = np.array(copied[:200], np.uint64)[:, None] ^ sigs[None, :]
        mism = ((x | (x >> np.uint64(1))) & np.uint64(0x5555555555555555))
        d = np.array([[bin(int(v)).count("1") for v in row] for row in mism[:50]])
        nearest_nonzero = [sorted(set(r.tolist()) - {0})[0] for r in d]
        assert set(nearest_nonzero) >= {1, 2, 3, 4}


def test_empty_and_single_guide(native):
    with native.Index.open(os.path.join(GOLDEN, "tiny_genome.issl")) as ix:
        r = ix.score([], "and", 75.0)
        assert r.code == b"" and r.distinct == 0
        r = ix.score(["GATTACAGATTACAGATTAC"], "mit", 75.0)
        assert len(r.code) == 1 and r.cfd[0] == -1


def test_repeated_and_interleaved_calls_are_identical(native, oracle_arrays):
    z, _ = load_case("c2_small")
    with native.Index.from_arrays(*oracle_arrays("c2_small")) as ix:
        a = ix.score(z["queries"], "and", 90.0)
        ix.score(z["queries"][::-1][:17], "cfd", 50.0)
        b = ix.score(z["queries"], "and", 90.0)
        assert a.code == b.code
        np.testing.assert_array_equal(a.mit, b.mit)  # deterministic, bit for bit
        np.testing.assert_array_equal(a.cfd, b.cfd)
        np.testing.assert_array_equal(a.count, b.count)


def test_module_filter_matches_reference(native):
    z, meta = load_case("tiny")
    from cracklingplusplus_gpu_b200.index import decode
    flags = z["filter_flags"]
    seqs = [decode(s) + "TGG" for s in z["queries"]]
    path = os.path.join(GOLDEN, "tiny_genome.issl")
    for level in ["ultralow", "low", "medium", "high"]:
        guides = [native.GuideResults(seq=s, isUnique=bool(f[0]), consensusCount=int(f[1]), passedBowtie2=chr(f[2]))
                  for s, f in zip(seqs, flags)]
        mod = native.ISSLScoringModule(native.CracklingConfig(path, method="mitAndCfd", scoreThreshold=75.0,
                                                              optimisation=level, consensusN=2))
        mod.run(guides)
        codes = bytes(ord(g.passedOffTargetScore) for g in guides)
        assert codes == z[f"filter_code_{level}"].tobytes(), level
        np.testing.assert_allclose([g.mitOfftargetscore for g in guides], z[f"filter_mit_{level}"], rtol=RTOL)
        np.testing.assert_allclose([g.cfdOfftargetscore for g in guides], z[f"filter_cfd_{level}"], rtol=RTOL)
    guides = [native.GuideResults(seq=s) for s in seqs]
    native.ISSLScoringModule(native.CracklingConfig(path, enabled=False)).run(guides)
    assert bytes(ord(g.passedOffTargetScore) for g in guides) == z["disabled_code"].tobytes()


DROPIN = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "module_dropin")


def _run_dropin(index, seqs, flags, method, threshold, level, consensus_n, enabled, tmp):
    """oracle/_ref/module_dropin: the reference's module driver, built with the reference's own
    types and include/dropin/ISSLScoringModule.hpp over libissl_b200.so (oracle/Makefile)."""
    gp, out = tmp / "guides.tsv", tmp / "out.tsv"
    gp.write_text("".join(f"{s}\t{u}\t{c}\t{chr(b)}\n" for s, (u, c, b) in zip(seqs, flags)))
    subprocess.run([DROPIN, index, str(gp), method, repr(threshold), level, str(consensus_n), str(enabled), str(out)],
                   check=True, capture_output=True)
    rows = [ln.split("\t") for ln in out.read_text().splitlines()]
    return (np.array([float(r[1]) for r in rows]), np.array([float(r[2]) for r in rows]),
            bytes(ord(r[3]) for r in rows))


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="oracle/_ref/module_dropin is built where the reference is")
def test_dropin_module_with_reference_types(native, tmp_path):
    """ISSLScoringModule as a Crackling++ pipeline would build it (src/CracklingPlusPlus.cpp:74-81):
    the reference's cracklingConfig / guideResults, run() on a vector<guideResults>, every method
    and threshold, every optimisation level of the processGuide filter, and the disabled module --
    equal to the reference module's own outputs."""
    from cracklingplusplus_gpu_b200.index import decode
    z, meta = load_case("tiny")
    index = os.path.join(GOLDEN, "tiny_genome.issl")
    seqs = [decode(s) + "TGG" for s in z["queries"]]
    plain = [(1, 0, ord("?"))] * len(seqs)
    for meth in meta["methods"]:
        for t in meta["thresholds"]:
            k = f"{meth}_{t}"
            m, c, codes = _run_dropin(index, seqs, plain, meth, t, "ultralow", 0, 1, tmp_path)
            assert codes == z["code_" + k].tobytes(), k
            np.testing.assert_allclose(m, z["mit_" + k], rtol=RTOL, atol=0, err_msg=k)
            np.testing.assert_allclose(c, z["cfd_" + k], rtol=RTOL, atol=0, err_msg=k)
    flags = [tuple(int(v) for v in f) for f in z["filter_flags"]]
    for level in ["ultralow", "low", "medium", "high"]:
        m, c, codes = _run_dropin(index, seqs, flags, "mitAndCfd", 75.0, level, 2, 1, tmp_path)
        assert codes == z[f"filter_code_{level}"].tobytes(), level
        np.testing.assert_allclose(m, z[f"filter_mit_{level}"], rtol=RTOL, atol=0, err_msg=level)
        np.testing.assert_allclose(c, z[f"filter_cfd_{level}"], rtol=RTOL, atol=0, err_msg=level)
    m, c, codes = _run_dropin(index, seqs, plain, "mitAndCfd", 75.0, "ultralow", 0, 0, tmp_path)
    assert codes == z["disabled_code"].tobytes()


def test_cli_output_matches_reference_format(native, tmp_path):
    from cracklingplusplus_gpu_b200.index import decode
    z, meta = load_case("tiny")
    qfile = tmp_path / "q.txt"
    qfile.write_text("".join(decode(s) + "\n" for s in z["queries"]))
    cli = os.path.join(os.path.dirname(native.library_path()), "issl_score_offtargets")
    for meth, word in [("mitAndCfd", "and"), ("mit", "mit"), ("cfd", "cfd")]:
        out = tmp_path / f"{word}.tsv"
        r = subprocess.run([cli, os.path.join(GOLDEN, "tiny_genome.issl"), str(qfile), "4", "75", word, str(out)],
                           capture_output=True, text=True, check=True)
        k = f"{meth}_75.0"
        lines = [ln for ln in r.stdout.splitlines() if "\t" in ln]
        assert len(lines) == len(z["queries"])
        for ln, s, m, c in zip(lines, z["queries"], z["mit_" + k], z["cfd_" + k]):
            want_m = "-1" if meth == "cfd" else f"{m:f}"
            want_c = "-1" if meth == "mit" else f"{c:f}"
            assert ln == f"{decode(s)}\t{want_m}\t{want_c}"
        rows = [ln.split("\t") for ln in out.read_text().splitlines()[1:]]
        assert [int(r[3]) for r in rows] == [int(c) for c in z["count_" + k]]
        assert f"Distinct off-targets: {int(z['distinct_' + k][0])}" in r.stderr


def test_corrupt_indexes_rejected(native, oracle_arrays, tmp_path):
    sigs, masks, sizes, lists = oracle_arrays("c0_small")
    good = tmp_path / "good.issl"
    with native.Index.from_arrays(sigs, masks, sizes, lists) as ix:
        ix.save(str(good))
    raw = good.read_bytes()
    trunc = tmp_path / "trunc.issl"
    trunc.write_bytes(raw[: len(raw) - 1000])
    with pytest.raises(native.IsslError) as e:
        native.Index.open(str(trunc))
    assert e.value.code == -2
    bad_sizes = sizes.copy()
    bad_sizes[0] += 1
    with pytest.raises(native.IsslError) as e:
        native.Index.from_arrays(sigs, masks, bad_sizes, lists)
    assert e.value.code == -3
    swapped = lists.copy()
    swapped[[0, -1]] = swapped[[-1, 0]]  # two entries in each other's bucket
    with pytest.raises(native.IsslError) as e:
        native.Index.from_arrays(sigs, masks, sizes, swapped)
    assert e.value.code == -3
    with pytest.raises(native.IsslError) as e:
        native.Index.from_arrays(sigs, masks, sizes, lists).score(["A" * 20], "and", 75.0, max_dist=5)
    assert e.value.code == -1


def test_mixed_slice_widths_use_generic_scan(native, oracle):
    """Slices of different widths (the format allows it) go through the mixed-width scan."""
    import synth
    sites, occ, queries = synth.make_case(21, 30000, 200, repeat_frac=0.1, n_seeds=20)
    masks = synth.masks_from_strings([
        "11111100000000000000", "00000011111110000000", "00000000000001111111",
        "10101010101010101010", "01010101010101010101", "11110000111100001111",
    ])
    oix = oracle.Index.build(sites, occ, masks)
    with native.Index.from_arrays(*oix.arrays()) as ix:
        for meth, t in [("mitAndCfd", 75.0), ("avgMitCfd", 95.0), ("cfd", 99.0)]:
            tm, tc, cnt, dist = oix.score(queries, METHODS[meth], t)
            ms, cs, codes = oracle.finalise(METHODS[meth], t, tm, tc)
            assert_matches(ix.score(queries, meth, t), ms, cs, codes, cnt, dist, tag=f"mixed {meth}")


def test_large_occurrence_counts_read_from_the_site_table(native, oracle):
    """List entries carry occurrence counts up to 6; larger ones are read from the per-site
    table. Counts spread over 0..100000 exercise both paths against the oracle."""
    import synth
    from cracklingplusplus_gpu_b200.slice_configs import slice_masks
    sites = np.unique(synth.random_sigs(synth.Stream(9, 1), 30000))
    rng = np.random.default_rng(4)
    occ = np.where(rng.random(len(sites)) < 0.5, rng.integers(0, 7, len(sites)),
                   rng.integers(7, 100000, len(sites))).astype(np.uint32)
    masks = np.array(slice_masks("slice-8-20"), np.uint64)
    oix = oracle.Index.build(sites, occ, masks)
    queries = np.concatenate([sites[:300], synth.random_sigs(synth.Stream(9, 2), 300)])
    with native.Index.build(sites, occ, masks) as ix:
        for a, b in zip(ix.export(), oix.arrays()):
            np.testing.assert_array_equal(a, b)
        for meth, t in [("mitAndCfd", 50.0), ("avgMitCfd", 99.0), ("cfd", 75.0)]:
            tm, tc, cnt, dist = oix.score(queries, METHODS[meth], t)
            ms, cs, codes = oracle.finalise(METHODS[meth], t, tm, tc)
            res = ix.score(queries, meth, t)
            assert_matches(res, ms, cs, codes, cnt, dist, tag=f"large occ {meth} {t}")
        assert int(np.max(cnt)) >= 7


def test_four_byte_entries_match(native, oracle_arrays, monkeypatch):
    """Indexes too large for 8-byte list entries keep 4-byte ones and read signatures from the
    site table; forced here on a small case, the results are the same."""
    z, meta = load_case("c1_small")
    monkeypatch.setenv("ISSL_ENTRY_BYTES", "4")
    with native.Index.from_arrays(*oracle_arrays("c1_small")) as ix4:
        assert ix4.info().entry_bytes == 4
        check_golden(ix4, z, meta)
    monkeypatch.setenv("ISSL_ENTRY_BYTES", "8")
    with native.Index.build(z["sites"], z["occ"], z["masks"]) as ix8:
        assert ix8.info().entry_bytes == 8
        for a, b in zip(ix8.export(), oracle_arrays("c1_small")):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", ["c4_small", "c2_small"])
def test_capacity_path_conditions(native, oracle_arrays, monkeypatch, name):
    """The conditions of the largest-index path on small cases: 4-byte list entries (signatures
    read from the site table, which checks every scored site's distance independently of the
    scan), guides scored in many chunks, and a range of scan unit sizes, staging depths, grids and
    slice waves. Every call matches the reference fixtures and finds no site farther than 4
    mismatches from its guide (a call that did would fail with ISSL_ERR_INTERNAL)."""
    z, meta = load_case(name)
    monkeypatch.setenv("ISSL_ENTRY_BYTES", "4")
    monkeypatch.setenv("ISSL_MAX_GUIDES_PER_RUN", "37")
    with native.Index.from_arrays(*oracle_arrays(name)) as ix:
        assert ix.info().entry_bytes == 4
        for chunk, stages, bps, fw in [((256, 256, 256), 2, 0, 0), ((512, 1024, 256), 4, 0, 2), ((1024, 512, 512), 3, 2, 1)]:
            ix.set_tuning(chunk, stages, bps, fw)
            for meth in meta["methods"]:
                for t in [50.0, 99.9]:
                    k = f"{meth}_{t}"
                    res = ix.score(z["queries"], meth, t)
                    assert_matches(res, z["mit_" + k], z["cfd_" + k], z["code_" + k].tobytes(), z["count_" + k],
                                   int(z["distinct_" + k][0]), tag=f"{name} {k} {chunk} {stages} {bps} {fw}")
                    assert ix.last_stats().dropped_hits == 0
