"""GPU off-target extraction (ExtractOfftargets) against its CPU restatement, and the FASTA ->
index pipeline against the oracle builder and, when it was built, the reference's own
ISSLCreateIndex run on the extracted list. Needs a GPU."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import extract_oracle as eo
from conftest import REPO

pytestmark = pytest.mark.gpu


def test_extraction_equals_reference_extractor(native, tmp_path):
    """The reference's own ExtractOfftargets output (case_extract.npz: FASTA with CRLF lines, N runs,
    lower case and repeats, a plain file of lines, a directory), byte for byte."""
    from conftest import extract_fixture
    paths, want, meta = extract_fixture(str(tmp_path / "in"))
    out = tmp_path / "out.txt"
    n = native.extract_offtargets(paths, str(out))
    assert n == meta["lines"]
    assert out.read_bytes() == want


def _genome(rng, n):
    s = np.array(list("ACGT"))[rng.choice(4, n, p=[0.295, 0.205, 0.205, 0.295])]
    s = "".join(s)
    # repeats (duplicate sites), N runs, lower-case stretches
    for _ in range(n // 2000):
        a, b = rng.integers(0, n - 200, 2)
        s = s[:b] + s[a:a + 150] + s[b + 150:]
    for _ in range(n // 5000):
        a = int(rng.integers(0, n - 50))
        s = s[:a] + "N" * int(rng.integers(1, 40)) + s[a + 40:]
    for _ in range(n // 8000):
        a = int(rng.integers(0, n - 300))
        s = s[:a] + s[a:a + 300].lower() + s[a + 300:]
    return s[:n]


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    rng = np.random.default_rng(17)
    d = tmp_path_factory.mktemp("genome")
    fa = d / "g.fa"
    with open(fa, "w", newline="") as f:
        for r in range(3):
            f.write(f">chr{r} synthetic\r\n")
            g = _genome(rng, 30000 + 7000 * r)
            for i in range(0, len(g), 60):
                f.write(g[i:i + 60] + "\r\n")
    txt = d / "lines.txt"
    txt.write_text("\n".join(_genome(rng, 400 + 50 * i) for i in range(20)) + "\n")
    sub = d / "more"
    sub.mkdir()
    (sub / "a.fa").write_text(">x\n" + _genome(rng, 5000) + "\n>y\n\n" + _genome(rng, 3000) + "\n")
    (sub / "b.txt").write_text(_genome(rng, 2500))  # no final newline
    return [str(fa), str(txt), str(sub)]


def _big_genome(rng, n):
    """Like _genome, built with array operations (megabase sizes)."""
    b = np.frombuffer(b"ACGT", np.uint8)[rng.choice(4, n, p=[0.295, 0.205, 0.205, 0.295])].copy()
    for _ in range(n // 20000):
        a, c = rng.integers(0, n - 200, 2)
        b[c:c + 150] = b[a:a + 150]
    for _ in range(n // 50000):
        a = int(rng.integers(0, n - 50))
        b[a:a + int(rng.integers(1, 40))] = ord("N")
    for _ in range(n // 80000):
        a = int(rng.integers(0, n - 300))
        b[a:a + 300] += 32  # lower case
    return b.tobytes()


def test_large_inputs_parsed_in_pieces(native, tmp_path):
    """Inputs above 8 MB are cut at line starts and parsed by all host threads: FASTA records
    with CRLF lines and blank lines inside a record, and a plain file of many lines without a
    final newline must still give exactly the restatement's output."""
    rng = np.random.default_rng(23)
    fa = tmp_path / "big.fa"
    with open(fa, "wb") as f:
        for r in range(4):
            f.write(b">rec%d\r\n" % r)
            g = _big_genome(rng, 3_000_000 + 100_000 * r)
            f.write(b"\r\n".join(g[i:i + 70] for i in range(0, len(g), 70)) + b"\r\n")
            if r == 1:
                f.write(b"\n  \n")
    txt = tmp_path / "big.txt"
    with open(txt, "wb") as f:
        f.write(b"\n".join(_big_genome(rng, 1000 + (i % 7) * 300) for i in range(7000)))
    inputs = [str(fa), str(txt)]
    assert os.path.getsize(fa) > 8 << 20 and os.path.getsize(txt) > 8 << 20
    out = str(tmp_path / "ot.txt")
    n = native.extract_offtargets(inputs, out)
    want = eo.extract_text(inputs)
    assert n == want.count(b"\n") and n > 100000
    assert open(out, "rb").read() == want


def test_extraction_equals_restatement(native, inputs, tmp_path):
    out = str(tmp_path / "ot.txt")
    n = native.extract_offtargets(inputs, out)
    want = eo.extract_text(inputs)
    got = open(out, "rb").read()
    assert n == want.count(b"\n") and n > 1000
    assert got == want


def test_sequences_to_index_equals_reference_builder(native, oracle, inputs, tmp_path):
    from cracklingplusplus_gpu_b200.slice_configs import SLICE_CONFIGS, slice_masks
    import synth
    sites = eo.extract(inputs)
    uniq, occ = np.unique(np.array(sites), return_counts=True)
    sigs = np.array([synth.seq_to_sig(s) for s in uniq.tolist()], np.uint64)
    masks = np.array(slice_masks("slice-8-20"), np.uint64)
    ix, n = native.Index.from_sequences(inputs, masks)
    with ix:
        assert n == len(sites)
        got = str(tmp_path / "gpu.issl")
        ix.save(got)
    want = str(tmp_path / "oracle.issl")
    oracle.Index.build(sigs, occ.astype(np.uint32), masks).write(want)
    assert open(got, "rb").read() == open(want, "rb").read()
    ref = os.path.join(REPO, "oracle", "_ref", "ISSLCreateIndex")
    if os.path.exists(ref):  # the reference's own builder on the extracted list
        ot = tmp_path / "ot.txt"
        ot.write_bytes(eo.extract_text(inputs))
        sc = tmp_path / "slices.txt"
        sc.write_text("\n".join(SLICE_CONFIGS["slice-8-20"]) + "\n")
        out = tmp_path / "ref.issl"
        subprocess.run([ref, str(ot), str(sc), "20", str(out)], cwd=tmp_path, check=True, capture_output=True)
        assert open(got, "rb").read() == out.read_bytes()


def test_no_sites_and_missing_inputs(native, tmp_path):
    empty = tmp_path / "e.txt"
    empty.write_text("NNNNNNNNNNNNNNNNNNNNNNNNNNNNNN\nACGT\n")
    out = str(tmp_path / "o.txt")
    assert native.extract_offtargets([str(empty)], out) == 0
    assert open(out, "rb").read() == b""
    with pytest.raises(native.IsslError):
        native.extract_offtargets([str(tmp_path / "missing.fa")], out)
