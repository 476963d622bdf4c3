"""Test infrastructure only: a CPU restatement of the reference's off-target extraction
(ExtractOfftargets/ExtractOfftargets.cpp), used by tests/ as the checker of the GPU extractor.

The reference's own binary cannot be built here (it needs Boost.Regex and Boost.Algorithm, which
are not installed); this restatement runs the reference's two regular expressions verbatim with
Python's `re` (the same lookahead semantics) and follows its input rules line by line:
  * inputs: files, or directories whose files are all read                     (:38-59)
  * a file whose first line starts with '>' is FASTA: every later line is trimmed and upper-cased,
    a line starting with '>' starts a new sequence, others are appended        (:66-90)
  * any other file: every line, trimmed and upper-cased, is one sequence       (:91-102)
  * forward matches: the first 20 bases of each match                          (:16, :124-138)
  * reverse matches: the first 20 bases of each match's reverse complement     (:17, :140-154)
    (rc: lib/util.cpp:50-64)
  * output: every match, sorted, one per line, duplicates kept                 (:160-365)
"""
from __future__ import annotations

import os
import re

FWD = re.compile(r"(?=([ACG][ACGT]{19}[ACGT][AG]G))")   # ExtractOfftargets.cpp:16
BWD = re.compile(r"(?=(C[CT][ACGT][ACGT]{19}[TGC]))")   # ExtractOfftargets.cpp:17
_COMP = str.maketrans("acgtrymkbdhvACGTRYMKBDHV", "tgcayrkmvhdbTGCAYRKMVHDB")  # lib/util.cpp:47-48
_WS = " \t\n\v\f\r"


def rc(s: str) -> str:
    return s[::-1].translate(_COMP)


def _lines(data: bytes):
    # std::getline on '\n'; a final line without a newline is still a line
    parts = data.split(b"\n")
    if parts and parts[-1] == b"":
        parts.pop()
    return [p.decode("latin-1") for p in parts]


def sequences(path: str):
    lines = _lines(open(path, "rb").read())
    if not lines:
        return []
    out = []
    if lines[0].startswith(">"):
        cur = []
        for ln in lines[1:]:
            t = ln.strip(_WS).upper()
            if t.startswith(">"):
                out.append("".join(cur))
                cur = []
            else:
                cur.append(t)
        out.append("".join(cur))
    else:
        out = [ln.strip(_WS).upper() for ln in lines]
    return out


def expand(inputs):
    files = []
    for p in inputs:
        if os.path.isfile(p):
            files.append(p)
        elif os.path.isdir(p):
            files += sorted(os.path.join(p, f) for f in os.listdir(p))
        else:
            raise FileNotFoundError(p)
    return files


def extract(inputs):
    """Every off-target site of the inputs, sorted, duplicates kept (list of 20-char strings)."""
    sites = []
    for f in expand(inputs):
        for s in sequences(f):
            sites += [m.group(1)[:20] for m in FWD.finditer(s)]
            sites += [rc(m.group(1))[:20] for m in BWD.finditer(s)]
    sites.sort()
    return sites


def extract_text(inputs) -> bytes:
    return "".join(s + "\n" for s in extract(inputs)).encode()
