"""Regenerates tests/golden/*.npz from the CPU oracle.

These fixtures pin the oracle against itself (regression); the reference
ships no outputs and cannot be built here (no Fortran compiler), so they are
NOT reference outputs.  Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tabi-pb_b200"), os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from tabipb import surface as S  # noqa: E402


def main():
    pos, nrm, fc = S.icosphere(3, 2.0)
    chr_ = np.zeros((1, 3))
    q = np.array([1.0])
    xyz, tq, ar, b = O.form_matrix(pos, nrm, fc, chr_, q, 1.0)
    T = O.Tree(xyz, tq, ar, b, 3, 100, 0.8)
    kap = O.kappa(0.15, 80.0)
    res = T.dgmres(kap, 80.0, T.bvct, iprcd=1, tol=1e-4, nthreads=4)
    se, ce = T.energy(chr_, q, kap, 80.0, 1.0, res["x"], nthreads=4)
    np.savez_compressed(os.path.join(HERE, "born_l3.npz"), x=res["x"], iter=res["iter"],
                        soleng=se, orderarr=T.orderarr, err_hist=res["err_hist"])
    print("born_l3", res["iter"], se)


if __name__ == "__main__":
    main()
