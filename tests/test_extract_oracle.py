"""The extraction oracle (oracle/extract_oracle.py) on hand-made inputs whose sites follow from
the reference's rules by hand: forward and reverse patterns, overlaps, sequence breaks, FASTA
records, plain-text lines, case and line endings; and on the fixture made by the reference's own
ExtractOfftargets. No GPU."""
from __future__ import annotations

import hashlib

import extract_oracle as eo
from conftest import extract_fixture


def test_oracle_equals_reference_extractor(tmp_path):
    """case_extract.npz holds the output of the reference's ExtractOfftargets (tests/golden/
    make_golden.py): the restatement reproduces it byte for byte."""
    paths, want, meta = extract_fixture(str(tmp_path))
    assert hashlib.sha256(want).hexdigest() == meta["output_sha256"]
    assert eo.extract_text(paths) == want

F20 = "ACGTACGTACGTACGTACGT"


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return str(p)


def test_forward_site_needs_acg_start_and_rgg_tail(tmp_path):
    assert eo.extract([write(tmp_path, "a.txt", F20 + "AGG\n")]) == [F20]
    assert eo.extract([write(tmp_path, "b.txt", F20 + "TGG\n")]) == [F20]       # N of NGG is any base
    assert eo.extract([write(tmp_path, "b2.txt", F20 + "ATG\n")]) == []         # [AG]G tail
    assert eo.extract([write(tmp_path, "c.txt", "T" + F20[1:] + "AGG\n")]) == []  # T first: no site


def test_reverse_site_is_the_reverse_complement(tmp_path):
    # C[CT][ACGT] + 19 bases + [TGC]: the site is the first 20 bases of the match's reverse complement
    m = "CCA" + "ACGTTGCAACGTTGCAACG" + "T"
    assert len(m) == 23
    assert eo.extract([write(tmp_path, "r.txt", m + "\n")]) == [eo.rc(m)[:20]]
    assert eo.rc(m)[:20] == "ACGTTGCAACGTTGCAACGT"


def test_overlapping_matches_and_duplicates_kept(tmp_path):
    assert eo.extract([write(tmp_path, "g.txt", "G" * 25 + "\n")]) == ["G" * 20] * 3


def test_breaks_records_lines_case_and_crlf(tmp_path):
    site = F20 + "AGG"
    fa = write(tmp_path, "x.fa", ">r1\r\n" + site[:10].lower() + "\r\n" + site[10:] + "\r\n>r2\n" +
               site[:12] + "\n>r3\n" + site[12:] + "\n")
    # r1: the site split over two lines and lower-cased is still found; r2/r3: a record boundary breaks it
    assert eo.extract([fa]) == [F20]
    plain = write(tmp_path, "y.txt", site[:12] + "\n" + site[12:] + "\n" + site + "NACGT\n")
    assert eo.extract([plain]) == [F20]  # lines are separate sequences; N stops nothing outside the site
    d = tmp_path / "dir"
    d.mkdir()
    (d / "1.txt").write_text(site + "\n")
    (d / "2.fa").write_text(">h\n" + site + "\n")
    assert eo.extract([str(d)]) == [F20, F20]
