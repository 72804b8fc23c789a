"""Generate the boundary-condition golden fixture from the reference itself.

Runs CarpetX's BoundaryCondition (CarpetX/src/boundaries*.cxx compiled
unmodified into oracle/_ref/libref_bc.so, see oracle/Makefile) on the seeded
cases of tests/boundary_cases.py and stores, per case, the seed and the
reference's values at the FAB points outside the domain interior (the input
is regenerated from the seed; the other points are left unchanged):

  boundary_golden.npz   <seed>_out for seeds 0..NCASES-1

Usage:  make -C oracle ref && python tests/golden/make_boundary_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import RefBoundary  # noqa: E402
from boundary_cases import fab_data, outside_mask, random_bc_case  # noqa: E402

NCASES = 64


def main():
    ref = RefBoundary()
    rec = {}
    for seed in range(NCASES):
        spec, lo, hi = random_bc_case(seed, max_n=6, max_ghost=2, max_comp=2)
        a = fab_data(seed, len(spec["dirichlet"]), lo, hi)
        ref.boundary(spec, a, lo, hi)
        rec[f"{seed:04d}_out"] = a[:, outside_mask(spec, lo, hi)]
    np.savez_compressed(os.path.join(HERE, "boundary_golden.npz"), **rec)


if __name__ == "__main__":
    main()
