"""Golden vectors of the reference's low-order A11 operator.

MatMult_MFStokes_A11LowOrder (src/stokes_operators.c:1207-1278) applies
MFStokesWrapper_A11PC (src/stokes_operators_mf.c:353-488) built with
ONEPOINTQ_LOWORDER_OPERATORS (:61): the Q2 element action with the Jacobian
evaluated once at the element centre.  This script runs the reference's own
compiled kernel (oracle/_ref, built from the pTatin3d sources) on a seeded
deformed 4x3x5 mesh and stores x, coords, eta and y = sum_e A_e x.

    python tests/golden/make_loworder_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402
from ptatin3d_b200 import mesh as M  # noqa: E402


def main():
    dims = (4, 3, 5)
    c = M.perturb_interior(M.uniform_coords(*dims), *dims, frac=0.2, seed=11)
    rng = np.random.default_rng(12)
    eta = 10.0 ** rng.uniform(-1, 1, size=(dims[0] * dims[1] * dims[2], 27))
    x = rng.uniform(-1, 1, size=c.size)
    R = Reference()
    R.setup(dims, c, eta)
    y = R.a11_raw(x, "loworder")
    np.savez_compressed(os.path.join(HERE, "loworder_4x3x5.npz"), dims=np.array(dims), coords=c, eta=eta, x=x, y=y)


if __name__ == "__main__":
    main()
