"""Extract the basis-set data this package ships from QUICK's basis library.

QUICK reads Gaussian-style basis files (``basis/6-31GS`` and friends) at run
time.  The GPU host that runs this package does not have those files, so the
numbers for the elements used by the workloads (H, C, N, O) are extracted once
into ``basis_sets.json`` next to this script.  The JSON keeps every shell in
file order with its label (S, P, SP, D, F), exponents and contraction
coefficients as the decimal strings of the file, so that parsing them later
gives bit-identical doubles to what QUICK's list-directed ``read`` sees.

Usage (only where the QUICK tree is present):
    python quick_b200/data/make_basis.py QUICK_ROOT   (or with $QUICK_ROOT set)
"""
import json
import os
import sys

# basis name -> QUICK basis file name (``basis/<file>``)
FILES = {
    "6-31G": "6-31G",
    "6-31G*": "6-31GS",
    "6-31G**": "6-31GSS",
    "cc-pVTZ": "CC-PVTZ",
}
ELEMENTS = ("H", "C", "N", "O")


def parse(path):
    """Parse one QUICK basis file into {element: [shell, ...]}.

    Mirrors the grammar readbasis accepts (src/basis.f90:54-96): a line
    ``<symbol> 0`` opens an element, each following ``<label> <nprim> <scale>``
    line opens a shell with ``nprim`` primitive lines (two columns, three for
    SP), and any other line (``****``) closes the element.
    """
    out = {}
    with open(path) as fh:
        lines = fh.read().splitlines()
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        i += 1
        if len(tok) == 2 and tok[1] == "0" and tok[0].isalpha():
            elem = tok[0].upper()
            shells = []
            while i < len(lines):
                t = lines[i].split()
                if len(t) != 3 or not t[0].isalpha():
                    break
                label, nprim = t[0].upper(), int(t[1])
                i += 1
                prims = []
                for _ in range(nprim):
                    prims.append(lines[i].split())
                    i += 1
                shells.append({"label": label, "prims": prims})
            out[elem] = shells
    return out


def main(basis_dir):
    data = {}
    for name, fname in FILES.items():
        parsed = parse(os.path.join(basis_dir, fname))
        data[name] = {e: parsed[e] for e in ELEMENTS if e in parsed}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_sets.json")
    with open(dst, "w") as fh:
        json.dump(data, fh, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    # the QUICK tree from the argument or $QUICK_ROOT
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("QUICK_ROOT")
    if not root:
        sys.exit("usage: make_basis.py QUICK_ROOT (or set QUICK_ROOT)")
    main(os.path.join(root, "basis"))
