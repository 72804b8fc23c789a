"""Generate the golden fixtures from the reference operators themselves.

Runs the reference prolongation (CarpetX/src/prolongate_3d_rf2*.cxx compiled
unmodified into oracle/_ref/libref_prolong.so, see oracle/Makefile) on seeded
inputs and stores inputs and outputs:

  prolong_golden.npz   every registered operator (9 families x orders x 8
                       centerings) per var on a small random box, plus per
                       group for the ENO and linear-fallback families
  config1_sha256.txt   SHA-256 of the reference output of the order-3
                       vertex-centred single-box case (35^3 coarse -> 64^3 fine)

Usage:  make -C oracle ref && python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import RefOracle  # noqa: E402
from helpers import ALL_OPS, box_shape, random_case  # noqa: E402
from config1 import config1_case  # noqa: E402


def main():
    ref = RefOracle()
    rng = np.random.default_rng(20261203)
    rec = {}
    n = 0
    for typ, order, it in ALL_OPS:
        modes = [0, 1] if typ in ("eno", "poly-cons3lfb", "poly-eno3lfb") else [0]
        for pg in modes:
            kind = "jumps" if typ in ("eno", "poly-cons3lfb", "poly-eno3lfb", "minmod") else "normal"
            c = random_case(rng, ref, typ, order, it, ncomp=2 if pg else 1, max_n=6, kind=kind)
            fine = np.full((c["ncomp"],) + box_shape(c["flo"], c["fhi"]), np.nan)
            ref.prolong(typ, order, it, pg, c["crse"], c["clo"], c["chi"], fine, c["flo"],
                        c["fhi"], c["rlo"], c["rhi"], c["ncomp"])
            key = f"{n:04d}"
            rec[key + "_meta"] = np.array([order, it, pg, c["ncomp"], *c["clo"], *c["chi"],
                                           *c["flo"], *c["fhi"], *c["rlo"], *c["rhi"]], np.int32)
            rec[key + "_type"] = np.array(typ)
            rec[key + "_crse"] = c["crse"]
            rec[key + "_fine"] = fine
            n += 1
    np.savez_compressed(os.path.join(HERE, "prolong_golden.npz"), **rec)
    c = config1_case()
    fine = np.zeros((1,) + box_shape(c["flo"], c["fhi"]))
    ref.prolong("interpolate", 3, 0, 0, c["crse"], c["clo"], c["chi"], fine, c["flo"], c["fhi"],
                c["flo"], c["fhi"], 1)
    with open(os.path.join(HERE, "config1_sha256.txt"), "w") as f:
        f.write(hashlib.sha256(np.ascontiguousarray(fine).tobytes()).hexdigest() + "\n")
    print(f"{n} cases written")


if __name__ == "__main__":
    main()
