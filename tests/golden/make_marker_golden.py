"""Golden vectors of the reference's material-point -> Gauss-point projections.

pTatin_EvaluateRheologyNonlinearities (src/rheology.c:150-185) sets the
Gauss-point viscosity and density from the markers by one of: P0 averages
(arithmetic 0, harmonic 10, geometric 20; MPntPStokesProj_P0,
src/material_point_utils.c:2567-2808), the Q1 projection (1;
SwarmUpdateGaussPropertiesLocalL2Projection_Q1_MPntPStokes, :604-891) or the
one-to-one map (4; :803-840).  This script runs the reference's own compiled
functions (oracle/_ref, built from the pTatin3d sources) on seeded markers of
a 3x2x4 mesh and stores inputs and outputs:

  dense   8 markers per element, plus markers on element faces and corners
  sparse  5 markers in all (elements without markers: P0 gives 0/0, Q1 gives
          0 on nodes without weight)
  one2one 27 markers per element in Gauss-point order

    python tests/golden/make_marker_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402
from ptatin3d_b200 import mesh as M  # noqa: E402

DIMS = (3, 2, 4)
TYPES = (0, 10, 20, 1)


def markers(seed, n, nel):
    rng = np.random.default_rng(seed)
    wil = rng.integers(0, nel, size=n).astype(np.int32)
    xi = rng.uniform(-1.0, 1.0, size=(n, 3))
    eta = 10.0 ** rng.uniform(-3.0, 3.0, size=n)
    rho = rng.uniform(0.9, 1.1, size=n)
    return wil, xi, eta, rho


def main():
    nel = DIMS[0] * DIMS[1] * DIMS[2]
    R = Reference()
    R.setup(DIMS, M.uniform_coords(*DIMS), np.ones(27 * nel))
    out = {"dims": np.array(DIMS)}
    wil, xi, eta, rho = markers(21, 8 * nel, nel)
    # markers on faces, edges and corners of the reference element
    edge = np.array([[1, 1, 1], [-1, -1, -1], [1, -1, 0], [0, 0, 1], [-1, 0.5, -1]], dtype=np.float64)
    wil = np.concatenate([wil, np.arange(5, dtype=np.int32) * 4])
    xi = np.concatenate([xi, edge])
    eta = np.concatenate([eta, [1.0, 2.0, 3.0, 4.0, 5.0]])
    rho = np.concatenate([rho, [1.0, 1.01, 1.02, 1.03, 1.04]])
    for case, (w, x, e, r) in (("dense", (wil, xi, eta, rho)), ("sparse", markers(22, 5, nel))):
        out[f"{case}_wil"], out[f"{case}_xi"], out[f"{case}_eta"], out[f"{case}_rho"] = w, x, e, r
        for t in TYPES:
            eq, rq = R.marker_project(t, w, x, e, r)
            out[f"{case}_{t}_eta_q"], out[f"{case}_{t}_rho_q"] = eq, rq
    rng = np.random.default_rng(23)
    e27, r27 = 10.0 ** rng.uniform(-1, 1, size=27 * nel), rng.uniform(0.9, 1.1, size=27 * nel)
    w27 = np.repeat(np.arange(nel, dtype=np.int32), 27)
    eq, rq = R.marker_project(4, w27, None, e27, r27)
    out.update(one2one_wil=w27, one2one_eta=e27, one2one_rho=r27, one2one_eta_q=eq, one2one_rho_q=rq)
    np.savez_compressed(os.path.join(HERE, "markers_3x2x4.npz"), **out)


if __name__ == "__main__":
    main()
