"""Regenerates the golden fixtures under tests/golden/ from the reference itself.

Run here (where the reference checkout and its compiled binaries exist), never on the GPU
host:   make -C oracle ref && python tests/golden/make_golden.py

Outputs
  penalties.json     MIT (mask, score) pairs and CFD position/PAM tables read from the
                     reference's lib/otScorePenalties.cpp:3-6199, :6201-6527, :6529-6546,
                     cross-checked against the 6,195 (mask, score) pairs embedded in the
                     reference's legacy test index tests/data/test_genome_offTargets_indexed.issl
  tiny_genome.issl   the reference's ISSLCreateIndex run on tests/data/test_genome_offTargets.fa
                     with sample/slice-4-5.txt
  case_*.npz         per case: the index inputs' digest, the queries, and the reference's
                     outputs (ISSLScoringModule::run scores at %.17g and accept codes for every
                     method and threshold; ISSLScoreOfftargets per-query counts and distinct
                     site count)
  case_knife.npz     thresholds on the reference's own running sums (knife_edge.py), one
                     (guide, method, threshold) per entry, scored by the same two binaries
  case_c0_full.npz   config 0 at its stated size (1M sites, slice-4-5, 1,000 guides): outputs
                     only, the sites are regenerated from the seed
  case_extract.npz   the reference's ExtractOfftargets on a small genome collection: the input
                     files and its output file

python tests/golden/make_golden.py [names...] regenerates only the named fixtures.
"""
from __future__ import annotations

import glob
import hashlib
import json
import os
import re
import shutil
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(REPO, "oracle", "_ref")
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))
from refpath import REFERENCE as REF  # noqa: E402

import synth  # noqa: E402
from cracklingplusplus_gpu_b200.slice_configs import SLICE_CONFIGS  # noqa: E402

MODULE_METHODS = ["mit", "cfd", "mitAndCfd", "mitOrCfd", "avgMitCfd"]
CLI_NAME = {"mit": "mit", "cfd": "cfd", "mitAndCfd": "and", "mitOrCfd": "or", "avgMitCfd": "avg"}


def parse_penalties():
    src = open(os.path.join(REF, "lib", "otScorePenalties.cpp")).read()
    mit_block = src[src.index("precalculatedMITScores"):src.index("cfdPosPenalties")]
    pairs = re.findall(r"\{\s*(\d+)\s*,\s*([0-9eE+.\-]+)\s*\}", mit_block)
    mit = [(int(k), float(v)) for k, v in pairs]

    def array(name, n):
        blk = src[src.index(name):]
        blk = blk[blk.index("{") + 1:blk.index("};")]
        blk = re.sub(r"//[^\n]*", "", blk)
        vals = [float(x) for x in re.findall(r"[0-9]+\.[0-9]+(?:[eE][+\-]?\d+)?|\b\d+\b", blk)]
        assert len(vals) == n, (name, len(vals))
        return vals

    return mit, array("cfdPosPenalties[320]", 320), array("cfdPamPenalties[16]", 16)


def legacy_mit_pairs():
    raw = open(os.path.join(REF, "tests", "data", "test_genome_offTargets_indexed.issl"), "rb").read()
    hdr = struct.unpack_from("<6Q", raw, 0)
    n_pairs = hdr[5]
    # legacy layout: a 6-word header, then the (mask, score) pairs
    pairs = [struct.unpack_from("<Qd", raw, 48 + 16 * i) for i in range(n_pairs)]
    return hdr, pairs


def run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed: {r.stderr[-2000:]}")
    return r


def ref_build_index(sites, occ, masks_str, out_path, tmp):
    """Reference ISSLCreateIndex on a sorted site text file (duplicates encode occurrences)."""
    seqs = [synth.sig_to_seq(s) for s in sites.tolist()]
    lines = []
    for s, o in zip(seqs, occ.tolist()):
        lines.extend([s] * int(o))
    lines.sort()
    sites_txt = os.path.join(tmp, "sites.txt")
    with open(sites_txt, "w") as f:
        f.write("\n".join(lines) + "\n")
    sc = os.path.join(tmp, "slices.txt")
    with open(sc, "w") as f:
        f.write("\n".join(masks_str) + "\n")
    run([os.path.join(REF_BIN, "ISSLCreateIndex"), sites_txt, sc, "20", out_path], cwd=tmp)
    return sorted(set(seqs))


def ref_module(index, guides, method, threshold, tmp, optimisation="ultralow", consensus_n=0,
               enabled=1, flags=None):
    gp = os.path.join(tmp, "guides.tsv")
    with open(gp, "w") as f:
        for i, g in enumerate(guides):
            u, c, b = flags[i] if flags else (1, 0, "?")
            f.write(f"{g}\t{u}\t{c}\t{b}\n")
    out = os.path.join(tmp, "module_out.tsv")
    run([os.path.join(REF_BIN, "ref_module_driver"), index, gp, method, repr(threshold), optimisation,
         str(consensus_n), str(enabled), out], cwd=tmp)
    mit, cfd, codes = [], [], []
    for line in open(out):
        _, m, c, code = line.rstrip("\n").split("\t")
        mit.append(float(m))
        cfd.append(float(c))
        codes.append(ord(code))
    return np.array(mit), np.array(cfd), np.array(codes, np.uint8)


def ref_cli(index, queries, method_cli, threshold, tmp):
    qp = os.path.join(tmp, "queries.txt")
    with open(qp, "w") as f:
        f.write("".join(q + "\n" for q in queries))
    work = tempfile.mkdtemp(dir=tmp)
    # the build without FMA contraction: its sums are rounded as the reference's release build rounds them
    r = run([os.path.join(REF_BIN, "ISSLScoreOfftargets_exact"), index, qp, "4", repr(threshold), method_cli,
             "cli_out.txt"], cwd=work)
    out_files = [p for p in glob.glob(os.path.join(work, "*")) if p.endswith("cli_out.txt") and os.path.isfile(p)]
    assert len(out_files) == 1, out_files
    counts = []
    for line in open(out_files[0]):
        if line.startswith("#"):
            continue
        counts.append(int(line.rstrip("\n").split("\t")[3]))
    distinct = int(re.search(r"Distinct off-targets: (\d+)", r.stderr).group(1))
    shutil.rmtree(work)
    return np.array(counts, np.uint64), distinct


THRESHOLDS = [50.0, 75.0, 90.0, 99.0, 99.9]

CASES = [
    # name, seed, n_sites, n_queries, slice config, repeat fraction, planted into sites
    ("c0_small", 11, 20000, 240, "slice-4-5", 0.05, True),
    ("c1_small", 12, 40000, 240, "slice-8-20", 0.05, False),
    ("c2_small", 13, 12000, 160, "slice-10-37", 0.20, False),
    ("c4_small", 14, 30000, 160, "slice-8-28", 0.05, False),
]


def make_case(name, seed, n_sites, n_queries, cfg, rep, planted, tmp):
    sites, occ, queries = synth.make_case(seed, n_sites, n_queries, repeat_frac=rep, n_seeds=40,
                                          planted_into_sites=planted,
                                          repeat_query_frac=0.2 if cfg == "slice-10-37" else 0.0)
    idx_path = os.path.join(tmp, f"{name}.issl")
    sorted_seqs = ref_build_index(sites, occ, SLICE_CONFIGS[cfg], idx_path, tmp)
    # canonical site order: the reference builder's (sorted text) order
    sig_sorted = np.array([synth.seq_to_sig(s) for s in sorted_seqs], np.uint64)
    occ_map = dict(zip(sites.tolist(), occ.tolist()))
    occ_sorted = np.array([occ_map[int(s)] for s in sig_sorted], np.uint32)
    digest = hashlib.sha256(open(idx_path, "rb").read()).hexdigest()
    qseqs = [synth.sig_to_seq(q) for q in queries.tolist()]
    # 23-mer guides (protospacer + NGG) for the module path: only the first 20 nt are scored
    guides = [q + "AGG" for q in qseqs]
    arrays = {"sites": sig_sorted, "occ": occ_sorted, "queries": queries.astype(np.uint64),
              "masks": synth.masks_from_strings(SLICE_CONFIGS[cfg])}
    meta = {"name": name, "config": cfg, "index_sha256": digest, "thresholds": THRESHOLDS,
            "methods": MODULE_METHODS}
    for meth in MODULE_METHODS:
        for t in THRESHOLDS:
            m, c, codes = ref_module(idx_path, guides, meth, t, tmp)
            cnt, distinct = ref_cli(idx_path, qseqs, CLI_NAME[meth], t, tmp)
            key = f"{meth}_{t}"
            arrays[f"mit_{key}"] = m
            arrays[f"cfd_{key}"] = c
            arrays[f"code_{key}"] = codes
            arrays[f"count_{key}"] = cnt
            arrays[f"distinct_{key}"] = np.array([distinct], np.uint64)
    np.savez_compressed(os.path.join(HERE, f"case_{name}.npz"), meta=json.dumps(meta), **arrays)
    print(f"{name}: {len(sig_sorted)} sites, {len(queries)} queries, index {digest[:12]}")


def make_tiny(tmp):
    """The reference's own tiny genome fixture through the reference's own builder."""
    fa = os.path.join(REF, "tests", "data", "test_genome_offTargets.fa")
    sc = os.path.join(tmp, "s45.txt")
    with open(sc, "w") as f:
        f.write("\n".join(SLICE_CONFIGS["slice-4-5"]) + "\n")
    shutil.copy(fa, os.path.join(tmp, "ot.txt"))
    out = os.path.join(HERE, "tiny_genome.issl")
    run([os.path.join(REF_BIN, "ISSLCreateIndex"), os.path.join(tmp, "ot.txt"), sc, "20", out], cwd=tmp)
    sites = sorted(set(l.strip() for l in open(fa) if l.strip()))
    qs = [l.strip() for l in open(os.path.join(REF, "sample", "test_queries.txt")) if l.strip()]
    # the reference sample queries (blank lines removed), every indexed site, and one- and
    # two-substitution variants of the first sites
    variants = []
    for s in sites[:12]:
        v1 = s[:5] + ("A" if s[5] != "A" else "C") + s[6:]
        v2 = v1[:13] + ("G" if v1[13] != "G" else "T") + v1[14:]
        variants += [v1, v2]
    queries = qs + sites + variants
    arrays = {"queries": np.array([synth.seq_to_sig(q) for q in queries], np.uint64)}
    meta = {"name": "tiny", "config": "slice-4-5", "thresholds": THRESHOLDS, "methods": MODULE_METHODS,
            "index_sha256": hashlib.sha256(open(out, "rb").read()).hexdigest()}
    guides = [q + "TGG" for q in queries]
    # processGuide filter coverage: alternate uniqueness / consensus / bowtie2 flags
    flags = [(i % 2, i % 4, "0" if i % 5 == 0 else "1") for i in range(len(guides))]
    for meth in MODULE_METHODS:
        for t in THRESHOLDS:
            m, c, codes = ref_module(out, guides, meth, t, tmp)
            cnt, distinct = ref_cli(out, queries, CLI_NAME[meth], t, tmp)
            key = f"{meth}_{t}"
            arrays[f"mit_{key}"], arrays[f"cfd_{key}"], arrays[f"code_{key}"] = m, c, codes
            arrays[f"count_{key}"] = cnt
            arrays[f"distinct_{key}"] = np.array([distinct], np.uint64)
    for level in ["ultralow", "low", "medium", "high"]:
        m, c, codes = ref_module(out, guides, "mitAndCfd", 75.0, tmp, optimisation=level, consensus_n=2,
                                 flags=flags)
        arrays[f"filter_mit_{level}"], arrays[f"filter_cfd_{level}"], arrays[f"filter_code_{level}"] = m, c, codes
    arrays["filter_flags"] = np.array([[u, cn, ord(b)] for u, cn, b in flags], np.int64)
    m, c, codes = ref_module(out, guides, "mitAndCfd", 75.0, tmp, enabled=0)
    arrays["disabled_mit"], arrays["disabled_cfd"], arrays["disabled_code"] = m, c, codes
    np.savez_compressed(os.path.join(HERE, "case_tiny.npz"), meta=json.dumps(meta), **arrays)
    print(f"tiny: {len(sites)} sites, {len(queries)} queries")


KNIFE = {"name": "knife", "seed": 15, "n_sites": 40000, "n_queries": 400, "config": "slice-8-20",
         "repeat_frac": 0.3, "n_seeds": 30, "repeat_query_frac": 0.5, "guides": 24, "min_hits": 20}


def _oracle(pen_pos, pen_pam):
    import pyoracle
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
    pyoracle.set_cfd_tables(pen_pos, pen_pam)
    return pyoracle


def make_knife(tmp, pen_pos, pen_pam):
    """Thresholds on the reference's own running sums (knife_edge.py): per selected guide and
    method, thresholds whose maximum_sum is within a few ulps of the rounded running quantity at
    the last hit and at an interior hit, and every threshold between the rounded and the exactly
    summed quantity. Each (guide, method, threshold) is scored by the reference module and CLI."""
    from concurrent.futures import ThreadPoolExecutor

    import knife_edge
    K = KNIFE
    sites, occ, queries = synth.make_case(K["seed"], K["n_sites"], K["n_queries"], repeat_frac=K["repeat_frac"],
                                          n_seeds=K["n_seeds"], planted_into_sites=False,
                                          repeat_query_frac=K["repeat_query_frac"])
    idx_path = os.path.join(tmp, "knife.issl")
    sorted_seqs = ref_build_index(sites, occ, SLICE_CONFIGS[K["config"]], idx_path, tmp)
    sig_sorted = np.array([synth.seq_to_sig(x) for x in sorted_seqs], np.uint64)
    occ_map = dict(zip(sites.tolist(), occ.tolist()))
    occ_sorted = np.array([occ_map[int(x)] for x in sig_sorted], np.uint32)
    ora = _oracle(pen_pos, pen_pam)
    oix = ora.Index.load(idx_path)  # the reference-built index, read by the pinned oracle
    traces = {}

    def trace(g):
        if g not in traces:
            traces[g] = oix.trace(int(queries[g]))
        return traces[g]

    sel = [g for g in range(len(queries)) if len(trace(g)[0]) >= K["min_hits"]][:K["guides"]]
    ent = knife_edge.entries(trace, sel)
    qseqs = [synth.sig_to_seq(x) for x in queries.tolist()]

    def one(i):
        g, meth, t, _ = ent[i]
        wd = os.path.join(tmp, f"k{i}")
        os.makedirs(wd, exist_ok=True)
        m, c, code = ref_module(idx_path, [qseqs[g] + "AGG"], meth, t, wd)
        cnt, _ = ref_cli(idx_path, [qseqs[g]], CLI_NAME[meth], t, wd)
        shutil.rmtree(wd)
        return m[0], c[0], code[0], cnt[0]

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        res = list(pool.map(one, range(len(ent))))
    differs = [knife_edge.exact_decision_differs(meth, t, *trace(g)[:2]) for g, meth, t, _ in ent]
    arrays = {"sites": sig_sorted, "occ": occ_sorted, "queries": queries.astype(np.uint64),
              "masks": synth.masks_from_strings(SLICE_CONFIGS[K["config"]]),
              "guide": np.array([e[0] for e in ent], np.int32),
              "method": np.array([knife_edge.METHODS[e[1]] for e in ent], np.int8),
              "threshold": np.array([e[2] for e in ent], np.float64),
              "aimed_hit": np.array([e[3] for e in ent], np.int32),
              "mit": np.array([r[0] for r in res]), "cfd": np.array([r[1] for r in res]),
              "code": np.array([r[2] for r in res], np.uint8), "count": np.array([r[3] for r in res], np.uint64),
              "exact_differs": np.array(differs, bool)}
    meta = dict(K, index_sha256=hashlib.sha256(open(idx_path, "rb").read()).hexdigest())
    np.savez_compressed(os.path.join(HERE, "case_knife.npz"), meta=json.dumps(meta), **arrays)
    print(f"knife: {len(ent)} (guide, method, threshold) entries on {len(sel)} guides, "
          f"{sum(differs)} where exact sums would decide differently")


C0_FULL = {"name": "c0_full", "seed": 1234, "n_sites": 1_000_000, "n_queries": 1000, "config": "slice-4-5",
           "thresholds": {"mitAndCfd": [50.0, 75.0, 90.0], "mit": [75.0], "cfd": [75.0], "mitOrCfd": [75.0],
                          "avgMitCfd": [75.0]}}


def make_c0_full(tmp):
    """Config 0 at its stated size: 1,000,000 i.i.d. sites (GC 41%), slice-4-5, 1,000 queries (500
    copied from the sites, whose 0-4-substitution mutants join the site set, 500 random). Only
    the outputs are stored: the sites are regenerated from the seed (synth.make_case) in the test."""
    C = C0_FULL
    sites, occ, queries = synth.make_case(C["seed"], C["n_sites"], C["n_queries"], repeat_frac=0.0,
                                          planted_into_sites=True)
    idx_path = os.path.join(tmp, "c0_full.issl")
    ref_build_index(sites, occ, SLICE_CONFIGS[C["config"]], idx_path, tmp)
    qseqs = [synth.sig_to_seq(x) for x in queries.tolist()]
    guides = [x + "AGG" for x in qseqs]
    arrays = {"queries": queries.astype(np.uint64)}
    for meth, ts in C["thresholds"].items():
        for t in ts:
            m, c, codes = ref_module(idx_path, guides, meth, t, tmp)
            cnt, distinct = ref_cli(idx_path, qseqs, CLI_NAME[meth], t, tmp)
            key = f"{meth}_{t}"
            arrays[f"mit_{key}"], arrays[f"cfd_{key}"], arrays[f"code_{key}"] = m, c, codes
            arrays[f"count_{key}"] = cnt
            arrays[f"distinct_{key}"] = np.array([distinct], np.uint64)
    meta = dict(C, index_sha256=hashlib.sha256(open(idx_path, "rb").read()).hexdigest())
    np.savez_compressed(os.path.join(HERE, "case_c0_full.npz"), meta=json.dumps(meta), **arrays)
    print(f"c0_full: {C['n_sites']} sites, {len(queries)} queries, index {meta['index_sha256'][:12]}")


def extract_inputs(seed=21):
    """A small genome collection for the extractor, every input form the reference reads: a FASTA
    file with CRLF lines, lower-case stretches, N runs and copied stretches (duplicate sites); a
    plain file of one sequence per line; a directory holding a FASTA file with an empty record line
    and a plain file without a final newline. Returns {relative path: bytes}."""
    st = synth.Stream(seed, 31)

    def genome(n):
        b = bytearray(np.frombuffer(b"ACGT", np.uint8)[synth.gc41_bases(st.uniform(n)).astype(np.int64)].tobytes())
        for _ in range(n // 2000):  # copied stretches
            a, c = (int(x) for x in st.below(2, n - 200))
            b[c:c + 150] = b[a:a + 150]
        for _ in range(n // 5000):  # N runs
            a, k = int(st.below(1, n - 50)[0]), 1 + int(st.below(1, 40)[0])
            b[a:a + k] = b"N" * k
        for _ in range(n // 8000):  # soft-masked (lower-case) stretches
            a = int(st.below(1, n - 300)[0])
            b[a:a + 300] = bytes(b[a:a + 300]).lower()
        return bytes(b[:n])

    fa = b""
    for r in range(3):
        g = genome(30000 + 7000 * r)
        fa += b">chr%d synthetic\r\n" % r + b"".join(g[i:i + 60] + b"\r\n" for i in range(0, len(g), 60))
    lines = b"\n".join(genome(400 + 50 * i) for i in range(20)) + b"\n"
    a_fa = b">x\n" + genome(5000) + b"\n>y\n\n" + genome(3000) + b"\n"
    b_txt = genome(2500)
    return {"g.fa": fa, "lines.txt": lines, "more/a.fa": a_fa, "more/b.txt": b_txt}


def make_extract(tmp):
    """The reference's own ExtractOfftargets (built with read-only std::regex / <cctype> stand-ins
    for its two Boost headers, oracle/Makefile) on extract_inputs(): its output file, byte for byte."""
    inputs = extract_inputs()
    root = os.path.join(tmp, "extract_in")
    for rel, data in inputs.items():
        os.makedirs(os.path.dirname(os.path.join(root, rel)), exist_ok=True)
        with open(os.path.join(root, rel), "wb") as f:
            f.write(data)
    out = os.path.join(tmp, "extract_out.txt")
    env = dict(os.environ, TMPDIR=os.path.join(tmp, "extract_tmp"))  # its fixed temp directory name
    os.makedirs(env["TMPDIR"], exist_ok=True)
    r = subprocess.run([os.path.join(REF_BIN, "ExtractOfftargets"), out, os.path.join(root, "g.fa"),
                        os.path.join(root, "lines.txt"), os.path.join(root, "more")], env=env, capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError(f"ExtractOfftargets failed: {r.stderr[-2000:]}")
    data = open(out, "rb").read()
    arrays = {f"input_{i}": np.frombuffer(v, np.uint8) for i, v in enumerate(inputs.values())}
    meta = {"name": "extract", "inputs": list(inputs), "args": ["g.fa", "lines.txt", "more"],
            "output_sha256": hashlib.sha256(data).hexdigest(), "lines": data.count(b"\n")}
    np.savez_compressed(os.path.join(HERE, "case_extract.npz"), meta=json.dumps(meta),
                        output=np.frombuffer(data, np.uint8), **arrays)
    print(f"extract: {meta['lines']} sites from {sum(len(v) for v in inputs.values())} input bytes")


def main():
    mit, pos, pam = parse_penalties()
    hdr, legacy = legacy_mit_pairs()
    assert len(mit) == 6195 and len(legacy) == 6195
    assert sorted(mit) == sorted(legacy), "legacy index MIT pairs differ from otScorePenalties"
    payload = {
        "source": "lib/otScorePenalties.cpp (reference), cross-checked against the (mask, score) pairs "
                  "embedded in tests/data/test_genome_offTargets_indexed.issl",
        "legacy_header": list(hdr),
        "legacy_pairs_equal": True,
        "mit": [[k, v.hex()] for k, v in sorted(mit)],
        "cfd_pos": [v.hex() for v in pos],
        "cfd_pam": [v.hex() for v in pam],
    }
    with open(os.path.join(HERE, "penalties.json"), "w") as f:
        json.dump(payload, f, indent=0)
    print("penalties.json:", len(mit), "MIT pairs")
    only = set(sys.argv[1:])  # optional: names of the fixtures to regenerate
    with tempfile.TemporaryDirectory() as tmp:
        if not only or "tiny" in only:
            make_tiny(tmp)
        for c in CASES:
            if not only or c[0] in only:
                make_case(*c, tmp)
        if not only or "knife" in only:
            make_knife(tmp, pos, pam)
        if not only or "c0_full" in only:
            make_c0_full(tmp)
        if not only or "extract" in only:
            make_extract(tmp)


if __name__ == "__main__":
    main()
