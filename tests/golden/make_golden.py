"""Generates tests/golden/testcoul_fit2.npz from the reference's fixture.

Source: PIMC++/examples/testcoul.dm of the reference (a real squarer output:
Coulomb e-p, LOG r grid 0.0025..10 with 250 points, fits 0..3, 7 tau levels
1/64..1).  The file is parsed here with a plain numpy reader written
independently of both the oracle and the CUDA library's reader, and the raw
arrays the DavidPA reader must reproduce are stored:

  potential  [250]              the "BEGIN potential" block
  u_fit2     [ntau][nukj][250]  the NMax == 2 table, derv = 1 (file order)
  du_fit2    [ntau][nukj][250]  the NMax == 2 table, derv = 2
  grid       (r_start, r_end, n), tau grid (tau_min, tau_max, ntau)

Run: python tests/golden/make_golden.py [path/to/testcoul.dm]
(default: $PIMC_REFERENCE_ROOT/PIMC++/examples/testcoul.dm)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_SRC = os.path.join(os.environ.get("PIMC_REFERENCE_ROOT", ""), "PIMC++", "examples", "testcoul.dm")


def parse(path):
    with open(path) as f:
        lines = f.read().split("\n")
    out = {}

    def numbers_from(i, count):
        vals = []
        while len(vals) < count:
            vals.extend(float(t) for t in lines[i].split())
            i += 1
        return np.array(vals[:count])

    for i, line in enumerate(lines):
        toks = line.split()
        if toks[:2] == ["BEGIN", "potential"]:
            out["potential"] = numbers_from(i + 1, 250)
        if toks[:2] == ["GRID", "1"] and "grid" not in out:
            out["grid"] = np.array([float(toks[3]), float(toks[4]), 250.0])
        if toks[:2] == ["GRID", "3"] and "taugrid" not in out:
            out["taugrid"] = np.array([float(toks[3]), float(toks[4]), 7.0])
        if line.strip().startswith("BEGIN density matrix table"):
            rest = line.split("fit=")[1]
            fit = int(rest.split()[0])
            derv = int(rest.split("=")[-1])
            if fit != 2:
                continue
            nukj = 6
            vals = numbers_from(i + 1, 7 * nukj * 250).reshape(7, nukj, 250)
            out["u_fit2" if derv == 1 else "du_fit2"] = vals
    return out


def main(src=DEFAULT_SRC):
    d = parse(src)
    np.savez_compressed(os.path.join(HERE, "testcoul_fit2.npz"), **d)
    print({k: v.shape for k, v in d.items()})


if __name__ == "__main__":
    main(*sys.argv[1:])
