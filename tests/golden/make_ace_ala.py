"""Writes ace_ala_nme.json: the atoms of QUICK's ACE-(ALA)n-NME benchmark
inputs (example/benchmarks/ACE_ALA_NME/ala{n}.in of the QUICK tree), the
molecules of QUICK's published HF energies.  Run where the QUICK tree exists:

    python tests/golden/make_ace_ala.py [QUICK_ROOT]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from quick_b200.molecule import parse_quick_input  # noqa: E402


def main(quick_root):
    out = {}
    for n in (1, 2, 3, 5):
        path = os.path.join(quick_root, "example", "benchmarks", "ACE_ALA_NME", "ala%d.in" % n)
        with open(path) as fh:
            text = fh.read()
        m = parse_quick_input(text)
        out["ala%d" % n] = dict(keywords=text.splitlines()[0], symbols=m.symbols,
                                xyz_angstrom=m.xyz_angstrom.tolist())
    with open(os.path.join(HERE, "ace_ala_nme.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "oracle"))
    from build_ref import quick_root
    main(sys.argv[1] if len(sys.argv) > 1 else quick_root())
