"""Writes tests/golden/proteins.npz: the atoms of the reference's own test
inputs, src/test_proteins/1a63.pqr (2,065 atoms) and 4mn3.pqr (997 atoms),
as readin.f90:29-86 reads them (x, y, z, charge, radius, each REAL*4).

The reference tree is not available where the tests run, so its two inputs
travel as this fixture; the tests write them back as PQR files for the host
driver.  Run from the repository root with the reference checked out at
REFERENCE (default /root/reference):

    python tests/golden/make_proteins.py [REFERENCE]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "tabi-pb_b200"))

from tabipb import surface as S  # noqa: E402


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    out = {}
    for name in ("1a63", "4mn3"):
        xyz, q, r = S.read_pqr(os.path.join(ref, "src", "test_proteins", name + ".pqr"))
        out[name] = np.concatenate([xyz, q[:, None], r[:, None]], axis=1).astype(np.float32)
        print(name, out[name].shape[0], "atoms, net charge", round(float(q.sum()), 3))
    np.savez_compressed(os.path.join(HERE, "proteins.npz"), **out)


if __name__ == "__main__":
    main()
