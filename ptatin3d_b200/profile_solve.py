"""One short device-resident Stokes solve, for profiling its kernel mix.

    python -m ptatin3d_b200.profile_solve [m] [iterations] [precision]

The C2 construction (unit cube, 8 sinkers of radius 0.1, viscosity contrast
1e4, density +1 %, free slip walls and base, free surface top), 4 Galerkin
levels, Chebyshev(3)/Jacobi, geometric-mean Schur weighting; stops after
`iterations` FGMRES iterations.
"""
import sys

import numpy as np
import torch

from . import PREC_F32, PREC_F64, SCHUR_ETA_GEOMEAN
from . import mesh as M
from .solver import StokesSolver, max_levels


def main(argv):
    m = int(argv[1]) if len(argv) > 1 else 32
    its = int(argv[2]) if len(argv) > 2 else 60
    prec = PREC_F32 if (len(argv) > 3 and argv[3] == "32") else PREC_F64
    bits = M.FREE_SLIP & ~M.bc_bit(M.FACE_KMAX, 2)
    c = M.uniform_coords(m, m, m)
    qp = M.qp_coords(c, m, m, m)
    cen, r = M.random_sinkers(8, 1, 0.1)
    S = StokesSolver(m, m, m, bits, nlevels=min(4, max_levels(m)), rtol=1e-12, max_it=its, mg_precision=prec,
                     schur_eta=SCHUR_ETA_GEOMEAN)
    S.setup(c, M.sinker_eta(qp, cen, r, 1.0, 1e4))
    S.set_rhs_body_force(M.sinker_density(qp, cen, r, 1.0, 1.01))
    u, p, st = S.solve(raise_on_noconv=False)
    torch.cuda.synchronize()
    print(f"{st['iterations']} iterations, |r|/|r0| = {st['rfinal'] / st['r0']:.3e}, "
          f"setup {st['setup_ms']:.1f} ms, solve {st['solve_ms']:.1f} ms")
    S.destroy()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
