"""Regenerate the golden fixtures of this directory from the reference's own files.

Run where the reference tree is available, with its path as the argument:

    python tests/golden/make_golden.py <path to the reference tree>

* sod_exact_t0.4.txt   -- analysis/sod.ana unchanged: the exact Sod solution the
  reference ships (x, rho, u, p at t=0.4, gamma=1.4, diaphragm at 0).
* sodtest_column.txt   -- from analysis/sodtest.dat (the reference's stored Sod
  run, nx=8 ny=200 nz=8, step 375, t=0.4): the column x=-0.005, z=-0.005 as
  (y, rho, p, vy).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    src = os.path.join(ref, "analysis", "sod.ana")
    a = np.loadtxt(src)
    np.savetxt(os.path.join(HERE, "sod_exact_t0.4.txt"), a, fmt="%.6E",
               header="x rho u p  (analysis/sod.ana: exact Sod solution, gamma=1.4, t=0.4)")
    rows = []
    with open(os.path.join(ref, "analysis", "sodtest.dat")) as f:
        for line in f:
            if line.lstrip().startswith("#"):
                continue
            t = line.split()
            rows.append([float(v) for v in t[:9]])
    d = np.array(rows)
    m = np.isclose(d[:, 0], -0.005) & np.isclose(d[:, 2], -0.005)
    col = d[m][:, [1, 3, 4, 6]]
    np.savetxt(os.path.join(HERE, "sodtest_column.txt"), col, fmt="%.8E",
               header="y rho p vy  (analysis/sodtest.dat column x=-0.005 z=-0.005, t=0.4)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference tree>")
    main(sys.argv[1])
