"""Records molecules of the reference's own fullerene library as test inputs.

The GPU box has no reference checkout, so the drop-in driver tests cannot
read its FullereneLib there.  This script reads a selection of the
reference's .cc1 files (count line, then "C idx x y z flag neighbours...")
and stores each molecule's atom coordinates, flag and neighbour indices in
tests/golden/fullerenes.npz; tests/test_drivers.py writes them back out in
the same layout (six decimals, as in the library, so the numbers the
programs parse are unchanged) into a temporary FullereneLib for both the
reference programs and the *_gpu drivers.

Run (where the reference checkout is present; REF overrides its path):
    python tests/golden/gen_fullerenes.py
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "fullerenes.npz"
REF = Path(os.environ.get("REF", Path(__file__).resolve().parents[3] / "reference"))

# (library sub-directory, file) -- the molecules the driver tests use
FILES = [("C60-76", "C60-Ih.cc1"), ("C60-76", "C70-D5h.cc1"), ("C60-76", "C72-D6d.cc1"),
         ("C84", "C84-No.01-D2.cc1"), ("C84", "C84-No.24-D6h.cc1")]


def parse_cc1(path: Path):
    tok = path.read_text().split("\n")
    n = int(tok[0].split()[0])
    xyz, flag, nbr = [], [], []
    for ln in tok[1:]:
        f = ln.split()
        if not f:
            continue
        xyz.append([float(v) for v in f[2:5]])
        flag.append(int(f[5]))
        nbr.append([int(v) for v in f[6:]])
        if len(xyz) == n:
            break
    k = max(len(b) for b in nbr)
    nb = np.full((n, k), -1, np.int32)
    for i, b in enumerate(nbr):
        nb[i, :len(b)] = b
    return np.array(xyz), np.array(flag, np.int32), nb


def main() -> None:
    out = {}
    for sub, fn in FILES:
        xyz, flag, nb = parse_cc1(REF / "FullereneLib" / sub / fn)
        key = fn[:-4]
        out[f"{key}/dir"] = np.array(sub)
        out[f"{key}/xyz"] = xyz
        out[f"{key}/flag"] = flag
        out[f"{key}/nbr"] = nb
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({len(FILES)} molecules)")


if __name__ == "__main__":
    main()
