"""Writes cfd_tables.inc (the CFD penalty tables as exact hexadecimal doubles).

The CFD model (Doench et al. 2016) scores a mismatching position by a penalty indexed by
position and by the guide / reverse-complemented off-target base pair, and the PAM by its
last two bases. The values must equal the reference's cfdPosPenalties[320] and
cfdPamPenalties[16] (lib/otScorePenalties.cpp:6201-6546) bit for bit; they are taken from
the golden fixture tests/golden/penalties.json, which tests/golden/make_golden.py extracts
from the reference. Layout kept: index (pos << 4) | (guide_base << 2) | (offtarget_base ^ 3).
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "..", "tests", "golden", "penalties.json")


def main():
    pen = json.load(open(SRC))
    pos = [float.fromhex(x) for x in pen["cfd_pos"]]
    pam = [float.fromhex(x) for x in pen["cfd_pam"]]
    out = ["// Generated by gen_cfd_tables.py -- CFD penalties as exact doubles.",
           "// index = (position << 4) | (guide base << 2) | (off-target base ^ 3); A=0 C=1 G=2 T=3",
           "static const double kCfdPos[320] = {"]
    for p in range(20):
        out.append("    " + ", ".join(v.hex() for v in pos[16 * p:16 * p + 16]) + ",")
    out.append("};")
    out.append("// index = (second-to-last PAM base << 2) | last PAM base; NGG = 0xA")
    out.append("static const double kCfdPam[16] = {")
    out.append("    " + ", ".join(v.hex() for v in pam) + ",")
    out.append("};")
    with open(os.path.join(HERE, "cfd_tables.inc"), "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
