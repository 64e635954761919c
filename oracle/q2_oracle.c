/*
 * CPU oracle: a plain-C restatement of pTatin3d's matrix-free Q2-P1disc
 * Stokes operators on a structured (DMDA) hexahedral mesh.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is compiled into
 * oracle/liboracle.so and called only from tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg.  No product code links or calls it.
 *
 * What it restates (reference paths are relative to the pTatin3d tree):
 *   - Q2 element layout, lexicographic 27-node connectivity on the node
 *     lattice:            src/dmda_element_q2p1.c:368-468
 *   - 1-D Q2 basis B and derivative D at the 3 Gauss points, weights:
 *                         src/stokes_operators_tensor.c:200-214,
 *                         src/element_utils_q2.c:276-333
 *   - A11 apply, sum-factorised tensor form (contract coords -> J, invert,
 *     contract u -> grad, symmetric-gradient action, transposed contraction):
 *                         src/stokes_operators_tensor.c:40-288
 *   - diag(A11):          src/stokes_operators_mf.c:67-131 +
 *                         src/stokes_q2p1_mf_operators_diag_def.c:120-218
 *   - A12 (grad) / A21 (div) with the P1 "global relative" pressure basis:
 *                         src/stokes_operators_mf.c:788-933,
 *                         src/stokes_q2p1_mf_operators_def.c:423-537,
 *                         src/element_utils_q2.c:183-224
 *   - scaled pressure-mass Schur approximation, per element 4x4:
 *                         src/stokes_assembly.c:299-450
 *   - DMDA trilinear prolongation on the Q2 node lattice (factor 2) and its
 *     transpose, PETSc DMCreateInterpolation as called from
 *                         src/ptatin_driver_linear_ts.c:986-990
 *
 * The "raw" operators below add element contributions into y and do not
 * touch Dirichlet rows/columns; the MatMult Dirichlet convention
 * (src/stokes_operators.c:1176,1201 and src/dmda_bcs.c:500-611) is applied by
 * the callers through o_bc_* helpers.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int mx, my, mz; /* elements per direction */
} o_mesh;

/* node lattice sizes */
static inline int o_nx(const o_mesh *m) { return 2 * m->mx + 1; }
static inline int o_ny(const o_mesh *m) { return 2 * m->my + 1; }
static inline int o_nz(const o_mesh *m) { return 2 * m->mz + 1; }

/* 1-D Gauss-Legendre rule on [-1,1] and the Q2 Lagrange basis (nodes -1,0,1)
 * evaluated there.  Row = quadrature point, column = basis function. */
static double GP[3], GW[3], BAS[3][3], DER[3][3], WQ[27];
static int tables_ready = 0;

static void o_tables(void)
{
  if (tables_ready) return;
  GP[0] = -sqrt(3.0 / 5.0); GP[1] = 0.0; GP[2] = sqrt(3.0 / 5.0);
  GW[0] = 5.0 / 9.0; GW[1] = 8.0 / 9.0; GW[2] = 5.0 / 9.0;
  for (int q = 0; q < 3; q++) {
    double s = GP[q];
    BAS[q][0] = 0.5 * (s * s - s);
    BAS[q][1] = 1.0 - s * s;
    BAS[q][2] = 0.5 * (s * s + s);
    DER[q][0] = s - 0.5;
    DER[q][1] = -2.0 * s;
    DER[q][2] = s + 0.5;
  }
  for (int k = 0; k < 3; k++)
    for (int j = 0; j < 3; j++)
      for (int i = 0; i < 3; i++) WQ[i + 3 * j + 9 * k] = GW[i] * GW[j] * GW[k];
  tables_ready = 1;
}

/* global node ids of element e, local node n = a + 3b + 9c (x fastest) */
static void o_element_nodes(const o_mesh *m, long e, long nid[27])
{
  int nx = o_nx(m), ny = o_ny(m);
  long ei = e % m->mx, ej = (e / m->mx) % m->my, ek = e / ((long)m->mx * m->my);
  for (int c = 0; c < 3; c++)
    for (int b = 0; b < 3; b++)
      for (int a = 0; a < 3; a++)
        nid[a + 3 * b + 9 * c] = (2 * ei + a) + (long)nx * ((2 * ej + b) + (long)ny * (2 * ek + c));
}

/* Apply the 3-D tensor product  out[f][c][b][a] (+)= Z[c][k] Y[b][j] X[a][i] in[f][k][j][i]
 * for nf fields; trans selects the transposed 1-D matrices.  Follows the
 * three-stage contraction of src/stokes_operators_tensor.c:40-92. */
static void o_contract(int nf, const double X[3][3], const double Y[3][3], const double Z[3][3], int trans,
                       const double *in, double *out)
{
  double x1[3][3], y1[3][3], z1[3][3];
  for (int r = 0; r < 3; r++)
    for (int s = 0; s < 3; s++) {
      x1[r][s] = trans ? X[s][r] : X[r][s];
      y1[r][s] = trans ? Y[s][r] : Y[r][s];
      z1[r][s] = trans ? Z[s][r] : Z[r][s];
    }
  for (int f = 0; f < nf; f++) {
    const double *u = in + 27 * f;
    double t1[27], t2[27];
    for (int k = 0; k < 3; k++)
      for (int j = 0; j < 3; j++)
        for (int a = 0; a < 3; a++) {
          double acc = 0.0;
          for (int i = 0; i < 3; i++) acc += x1[a][i] * u[i + 3 * j + 9 * k];
          t1[a + 3 * j + 9 * k] = acc;
        }
    for (int k = 0; k < 3; k++)
      for (int b = 0; b < 3; b++)
        for (int a = 0; a < 3; a++) {
          double acc = 0.0;
          for (int j = 0; j < 3; j++) acc += y1[b][j] * t1[a + 3 * j + 9 * k];
          t2[a + 3 * b + 9 * k] = acc;
        }
    for (int c = 0; c < 3; c++)
      for (int b = 0; b < 3; b++)
        for (int a = 0; a < 3; a++) {
          double acc = 0.0;
          for (int k = 0; k < 3; k++) acc += z1[c][k] * t2[a + 3 * b + 9 * k];
          out[27 * f + a + 3 * b + 9 * c] += acc;
        }
  }
}

/* gather 27 nodes x 3 components into field-major [3][27] */
static void o_gather3(const double *v, const long nid[27], double *el)
{
  for (int n = 0; n < 27; n++)
    for (int f = 0; f < 3; f++) el[27 * f + n] = v[3 * nid[n] + f];
}

/* grad[d][f][q] = d(field f)/d(xi_d) at quadrature point q */
static void o_ref_gradient(const double *el, double grad[3][3][27])
{
  memset(grad, 0, sizeof(double) * 3 * 3 * 27);
  o_contract(3, DER, BAS, BAS, 0, el, &grad[0][0][0]);
  o_contract(3, BAS, DER, BAS, 0, el, &grad[1][0][0]);
  o_contract(3, BAS, BAS, DER, 0, el, &grad[2][0][0]);
}

/* Per-QP Jacobian J[d][l] = dx_l/dxi_d; returns inverse in place of J
 * (iJ[k][d] = dxi_k/dx_d ... stored the same way as the reference:
 * after inversion jac[r][s] holds (J^{-1})[r][s]) and detJ.
 * Cofactor inverse as in src/stokes_operators_tensor.c:94-125. */
static void o_invert(double a[3][3], double *det_out)
{
  double c00 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
  double c10 = -(a[1][0] * a[2][2] - a[2][0] * a[1][2]);
  double c20 = a[1][0] * a[2][1] - a[2][0] * a[1][1];
  double det = a[0][0] * c00 + a[0][1] * c10 + a[0][2] * c20;
  double r = 1.0 / det;
  double inv[3][3];
  inv[0][0] = r * c00;
  inv[0][1] = -r * (a[0][1] * a[2][2] - a[2][1] * a[0][2]);
  inv[0][2] = r * (a[0][1] * a[1][2] - a[1][1] * a[0][2]);
  inv[1][0] = r * c10;
  inv[1][1] = r * (a[0][0] * a[2][2] - a[2][0] * a[0][2]);
  inv[1][2] = -r * (a[0][0] * a[1][2] - a[1][0] * a[0][2]);
  inv[2][0] = r * c20;
  inv[2][1] = -r * (a[0][0] * a[2][1] - a[2][0] * a[0][1]);
  inv[2][2] = r * (a[0][0] * a[1][1] - a[1][0] * a[0][1]);
  memcpy(a, inv, sizeof inv);
  *det_out = det;
}

/* geometry of one element at the 27 QPs: inverse Jacobian and detJ */
static void o_geometry(const double *elx, double iJ[27][3][3], double detJ[27])
{
  double g[3][3][27];
  o_ref_gradient(elx, g);
  for (int q = 0; q < 27; q++) {
    double a[3][3];
    for (int d = 0; d < 3; d++)
      for (int l = 0; l < 3; l++) a[d][l] = g[d][l][q];
    o_invert(a, &detJ[q]);
    memcpy(iJ[q], a, sizeof a);
  }
}

/* ---------------------------------------------------------------- A11 ---- */
/* y += A11_elements(u).  Follows src/stokes_operators_tensor.c:181-288: the
 * quadrature action computes dux[k][l] = sum_d du[d][l] iJ[k][d], the
 * symmetric strain, tau = 2 eta eps, and dv[k][l] = w detJ sum_m tau[m][l] iJ[m][k]
 * (src/stokes_operators_tensor.c:127-179). */
void o_a11_apply(int mx, int my, int mz, const double *coords, const double *eta, const double *u, double *y)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], elu[81], elv[81];
    double iJ[27][3][3], detJ[27], gu[3][3][27], dv[3][3][27];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_gather3(u, nid, elu);
    o_geometry(elx, iJ, detJ);
    o_ref_gradient(elu, gu);
    const double *eq = eta + 27 * e;
    for (int q = 0; q < 27; q++) {
      double dux[3][3], tau[3][3];
      for (int l = 0; l < 3; l++)
        for (int k = 0; k < 3; k++)
          dux[k][l] = gu[0][l][q] * iJ[q][k][0] + gu[1][l][q] * iJ[q][k][1] + gu[2][l][q] * iJ[q][k][2];
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) tau[k][l] = eq[q] * (dux[k][l] + dux[l][k]);
      double s = WQ[q] * detJ[q];
      for (int l = 0; l < 3; l++)
        for (int k = 0; k < 3; k++)
          dv[k][l][q] = s * (tau[0][l] * iJ[q][0][k] + tau[1][l] * iJ[q][1][k] + tau[2][l] * iJ[q][2][k]);
    }
    memset(elv, 0, sizeof elv);
    o_contract(3, DER, BAS, BAS, 1, &dv[0][0][0], elv);
    o_contract(3, BAS, DER, BAS, 1, &dv[1][0][0], elv);
    o_contract(3, BAS, BAS, DER, 1, &dv[2][0][0], elv);
    for (int n = 0; n < 27; n++)
      for (int f = 0; f < 3; f++) y[3 * nid[n] + f] += elv[27 * f + n];
  }
}

/* physical shape-function gradients at QP q: dN[d][n] = dN_n/dx_d */
static void o_phys_grad(const double iJ[3][3], int q, double dN[3][27])
{
  int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
  for (int n = 0; n < 27; n++) {
    int a = n % 3, b = (n / 3) % 3, c = n / 9;
    double g0 = DER[qi][a] * BAS[qj][b] * BAS[qk][c];
    double g1 = BAS[qi][a] * DER[qj][b] * BAS[qk][c];
    double g2 = BAS[qi][a] * BAS[qj][b] * DER[qk][c];
    for (int d = 0; d < 3; d++) dN[d][n] = iJ[d][0] * g0 + iJ[d][1] * g1 + iJ[d][2] * g2;
  }
}

/* y += diag(A11_elements): per dof (n,l): sum_q w detJ eta (|grad N_n|^2 + (dN_n/dx_l)^2)
 * (src/stokes_q2p1_mf_operators_diag_def.c:120-218). */
void o_a11_diag(int mx, int my, int mz, const double *coords, const double *eta, double *y)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], iJ[27][3][3], detJ[27], acc[81];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_geometry(elx, iJ, detJ);
    memset(acc, 0, sizeof acc);
    for (int q = 0; q < 27; q++) {
      double dN[3][27];
      o_phys_grad(iJ[q], q, dN);
      double s = WQ[q] * detJ[q] * eta[27 * e + q];
      for (int n = 0; n < 27; n++) {
        double sq = dN[0][n] * dN[0][n] + dN[1][n] * dN[1][n] + dN[2][n] * dN[2][n];
        for (int l = 0; l < 3; l++) acc[3 * n + l] += s * (sq + dN[l][n] * dN[l][n]);
      }
    }
    for (int n = 0; n < 27; n++)
      for (int l = 0; l < 3; l++) y[3 * nid[n] + l] += acc[3 * n + l];
  }
}

/* P1 "global relative" pressure basis at reference point (qi,qj,qk):
 * N = [1, xh, yh, zh], xh = (x(xi) - mean of the 27 nodes)/L with
 * L from mid-face node differences (src/element_utils_q2.c:183-224). */
static void o_pressure_basis(const double *elx, int q, double Np[4])
{
  int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
  double xq[3] = {0, 0, 0}, avg[3] = {0, 0, 0};
  for (int n = 0; n < 27; n++) {
    int a = n % 3, b = (n / 3) % 3, c = n / 9;
    double N = BAS[qi][a] * BAS[qj][b] * BAS[qk][c];
    for (int d = 0; d < 3; d++) {
      xq[d] += N * elx[27 * d + n];
      avg[d] += elx[27 * d + n];
    }
  }
  double L[3];
  L[0] = elx[27 * 0 + 14] - elx[27 * 0 + 12];
  L[1] = elx[27 * 1 + 16] - elx[27 * 1 + 10];
  L[2] = elx[27 * 2 + 22] - elx[27 * 2 + 4];
  Np[0] = 1.0;
  for (int d = 0; d < 3; d++) Np[1 + d] = (xq[d] - avg[d] / 27.0) / L[d];
}

/* y_u += A12 p : y_(n,d) += - sum_q w detJ dN_n/dx_d p(q)
 * (src/stokes_q2p1_mf_operators_def.c:423-515) */
void o_a12_apply(int mx, int my, int mz, const double *coords, const double *p, double *yu)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], iJ[27][3][3], detJ[27], acc[81];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_geometry(elx, iJ, detJ);
    memset(acc, 0, sizeof acc);
    for (int q = 0; q < 27; q++) {
      double dN[3][27], Np[4];
      o_phys_grad(iJ[q], q, dN);
      o_pressure_basis(elx, q, Np);
      double pq = Np[0] * p[4 * e] + Np[1] * p[4 * e + 1] + Np[2] * p[4 * e + 2] + Np[3] * p[4 * e + 3];
      double s = WQ[q] * detJ[q];
      for (int n = 0; n < 27; n++)
        for (int d = 0; d < 3; d++) acc[3 * n + d] += -s * dN[d][n] * pq;
    }
    for (int n = 0; n < 27; n++)
      for (int d = 0; d < 3; d++) yu[3 * nid[n] + d] += acc[3 * n + d];
  }
}

/* y_p += A21 u : y_(e,i) += - sum_q w detJ Np_i div u(q)
 * (src/stokes_q2p1_mf_operators_def.c:517-537) */
void o_a21_apply(int mx, int my, int mz, const double *coords, const double *u, double *yp)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], elu[81], iJ[27][3][3], detJ[27];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_gather3(u, nid, elu);
    o_geometry(elx, iJ, detJ);
    for (int q = 0; q < 27; q++) {
      double dN[3][27], Np[4], div = 0.0;
      o_phys_grad(iJ[q], q, dN);
      o_pressure_basis(elx, q, Np);
      for (int n = 0; n < 27; n++)
        for (int d = 0; d < 3; d++) div += dN[d][n] * elu[27 * d + n];
      double s = WQ[q] * detJ[q];
      for (int i = 0; i < 4; i++) yp[4 * e + i] += -s * Np[i] * div;
    }
  }
}

/* Scaled pressure mass matrix, one dense 4x4 block per element:
 * S_e[i][j] = - sum_q (1/eta_q) w detJ Np_i Np_j  (src/stokes_assembly.c:299-450).
 * Output S[nel][4][4]. */
void o_schur_mass(int mx, int my, int mz, const double *coords, const double *eta, double *S)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], iJ[27][3][3], detJ[27];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_geometry(elx, iJ, detJ);
    double *Se = S + 16 * e;
    memset(Se, 0, 16 * sizeof(double));
    for (int q = 0; q < 27; q++) {
      double Np[4];
      o_pressure_basis(elx, q, Np);
      double s = -WQ[q] * detJ[q] / eta[27 * e + q];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) Se[4 * i + j] += s * Np[i] * Np[j];
    }
  }
}

/* Element stiffness matrix of A11 (81x81, dof order 3n+l), used to build
 * assembled coarse operators (src/stokes_assembly.c:115-297). */
void o_a11_element_matrix(const double *elcoords /* [27][3] */, const double *eta_e /* [27] */, double *K)
{
  o_tables();
  double elx[81];
  for (int n = 0; n < 27; n++)
    for (int f = 0; f < 3; f++) elx[27 * f + n] = elcoords[3 * n + f];
  double iJ[27][3][3], detJ[27];
  o_geometry(elx, iJ, detJ);
  memset(K, 0, 81 * 81 * sizeof(double));
  for (int q = 0; q < 27; q++) {
    double dN[3][27];
    o_phys_grad(iJ[q], q, dN);
    double s = WQ[q] * detJ[q] * eta_e[q];
    /* a(v,u) = sum eta (du_l/dx_k + du_k/dx_l) dv_l/dx_k */
    for (int n = 0; n < 27; n++)
      for (int l = 0; l < 3; l++)
        for (int mm = 0; mm < 27; mm++)
          for (int f = 0; f < 3; f++) {
            double v = 0.0;
            /* column dof (mm,f) contributes to dux[k][f] = dN[k][mm] */
            for (int k = 0; k < 3; k++) {
              double duxkl = (f == l) ? dN[k][mm] : 0.0; /* dux[k][l] from column (mm,f) */
              double duxlk = (k == f) ? dN[l][mm] : 0.0; /* dux[l][k] */
              v += dN[k][n] * (duxkl + duxlk);
            }
            K[(3 * n + l) * 81 + 3 * mm + f] += s * v;
          }
  }
}

/* ------------------------------------------------- MG transfer (DMDA) --- */
/* Prolongation from a coarse node lattice (cnx,cny,cnz) to the fine one
 * (2c-1 per direction), ndof components interleaved: fine node at an even
 * index copies the coarse node, at an odd index averages its two coarse
 * neighbours, tensor product in 3-D (trilinear on the node lattice). */
void o_prolong(int cnx, int cny, int cnz, int ndof, const double *xc, double *xf)
{
  int fnx = 2 * cnx - 1, fny = 2 * cny - 1, fnz = 2 * cnz - 1;
  for (int k = 0; k < fnz; k++)
    for (int j = 0; j < fny; j++)
      for (int i = 0; i < fnx; i++) {
        int i0 = i / 2, i1 = (i + 1) / 2, j0 = j / 2, j1 = (j + 1) / 2, k0 = k / 2, k1 = (k + 1) / 2;
        double wi = (i0 == i1) ? 1.0 : 0.5, wj = (j0 == j1) ? 1.0 : 0.5, wk = (k0 == k1) ? 1.0 : 0.5;
        for (int d = 0; d < ndof; d++) {
          double acc = 0.0;
          int ii[2] = {i0, i1}, jj[2] = {j0, j1}, kk[2] = {k0, k1};
          int ni = (i0 == i1) ? 1 : 2, nj = (j0 == j1) ? 1 : 2, nk = (k0 == k1) ? 1 : 2;
          for (int c = 0; c < nk; c++)
            for (int b = 0; b < nj; b++)
              for (int a = 0; a < ni; a++)
                acc += wi * wj * wk * xc[(long)ndof * (ii[a] + (long)cnx * (jj[b] + (long)cny * kk[c])) + d];
          xf[(long)ndof * (i + (long)fnx * (j + (long)fny * k)) + d] = acc;
        }
      }
}

/* Restriction = transpose of o_prolong: xc = P^T xf */
void o_restrict(int cnx, int cny, int cnz, int ndof, const double *xf, double *xc)
{
  int fnx = 2 * cnx - 1, fny = 2 * cny - 1, fnz = 2 * cnz - 1;
  memset(xc, 0, sizeof(double) * (size_t)ndof * cnx * cny * cnz);
  for (int k = 0; k < fnz; k++)
    for (int j = 0; j < fny; j++)
      for (int i = 0; i < fnx; i++) {
        int i0 = i / 2, i1 = (i + 1) / 2, j0 = j / 2, j1 = (j + 1) / 2, k0 = k / 2, k1 = (k + 1) / 2;
        double wi = (i0 == i1) ? 1.0 : 0.5, wj = (j0 == j1) ? 1.0 : 0.5, wk = (k0 == k1) ? 1.0 : 0.5;
        int ii[2] = {i0, i1}, jj[2] = {j0, j1}, kk[2] = {k0, k1};
        int ni = (i0 == i1) ? 1 : 2, nj = (j0 == j1) ? 1 : 2, nk = (k0 == k1) ? 1 : 2;
        for (int d = 0; d < ndof; d++) {
          double v = xf[(long)ndof * (i + (long)fnx * (j + (long)fny * k)) + d];
          for (int c = 0; c < nk; c++)
            for (int b = 0; b < nj; b++)
              for (int a = 0; a < ni; a++)
                xc[(long)ndof * (ii[a] + (long)cnx * (jj[b] + (long)cny * kk[c])) + d] += wi * wj * wk * v;
        }
      }
}

/* ------------------------------------------- coefficient hierarchy --- */
/* The reference's coefficient hierarchy for Gauss-point viscosity
 * (SwarmUpdateGaussPropertiesLocalL2Projection_Q1_MPntPStokes_Hierarchy,
 * src/material_point_utils.c:1267-1420, projection types -1/0 with
 * -mp_hierarchy_projection_type 0).  The Q2 node lattice is treated as a Q1
 * lattice with one scalar per node. */

/* Q1 shape functions of the element at reference point xi (element_utils_q1.c:32-47),
 * mapped to the element's Q2 corner nodes 0,2,6,8,18,20,24,26 */
static void o_q1_corner_weights(const double xi[3], double w[27])
{
  for (int n = 0; n < 27; n++) w[n] = 0.0;
  for (int c = 0; c < 2; c++)
    for (int b = 0; b < 2; b++)
      for (int a = 0; a < 2; a++)
        w[2 * a + 3 * (2 * b) + 9 * (2 * c)] = 0.125 * (a ? 1.0 + xi[0] : 1.0 - xi[0]) *
                                               (b ? 1.0 + xi[1] : 1.0 - xi[1]) * (c ? 1.0 + xi[2] : 1.0 - xi[2]);
}

/* fine level: nodal field v = A / B with, per element and Gauss point q,
 * A_n += N_n(q) eta_q, B_n += N_n(q); N = the Q1 corner weights at the corners
 * and 1 at the 19 other Q2 nodes
 * (_BuildQ1CoefficientProjection_QuadraturePoints_MPntPStokes_FineGrid, :1138-1257) */
void o_eta_project_nodes(int mx, int my, int mz, const double *eta, double *v)
{
  o_tables();
  o_mesh m = {mx, my, mz};
  long nx = 2 * mx + 1, ny = 2 * my + 1, nn = nx * ny * (2 * mz + 1);
  double *B = (double *)calloc((size_t)nn, sizeof(double));
  memset(v, 0, sizeof(double) * (size_t)nn);
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    o_element_nodes(&m, e, nid);
    for (int q = 0; q < 27; q++) {
      double xi[3] = {GP[q % 3], GP[(q / 3) % 3], GP[q / 9]}, w[27];
      o_q1_corner_weights(xi, w);
      for (int n = 0; n < 27; n++) {
        const int corner = (n % 3 != 1) && ((n / 3) % 3 != 1) && (n / 9 != 1);
        const double N = corner ? w[n] : 1.0;
        v[nid[n]] += N * eta[27 * e + q];
        B[nid[n]] += N;
      }
    }
  }
  for (long i = 0; i < nn; i++) v[i] /= B[i];
  free(B);
}

/* next coarser level: vc = (P^T vf) ./ (P^T 1) (MatRestrict with DMCreateInterpolationScale, :1379-1394) */
void o_eta_restrict_nodes(int cnx, int cny, int cnz, const double *vf, double *vc)
{
  long fn = (long)(2 * cnx - 1) * (2 * cny - 1) * (2 * cnz - 1), cn = (long)cnx * cny * cnz;
  double *ones = (double *)malloc(sizeof(double) * (size_t)fn), *den = (double *)malloc(sizeof(double) * (size_t)cn);
  for (long i = 0; i < fn; i++) ones[i] = 1.0;
  o_restrict(cnx, cny, cnz, 1, vf, vc);
  o_restrict(cnx, cny, cnz, 1, ones, den);
  for (long i = 0; i < cn; i++) vc[i] /= den[i];
  free(ones);
  free(den);
}

/* Gauss-point values of a level from its nodal field: Q1 interpolation of the
 * 8 corner values, clamped to the range of the element's 27 nodal values
 * (_SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_InterpolateToQuadratePoints, :894-1030) */
void o_eta_nodes_to_qp(int mx, int my, int mz, const double *v, double *eta)
{
  o_tables();
  o_mesh m = {mx, my, mz};
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    o_element_nodes(&m, e, nid);
    double lo = 1e32, hi = -1e32;
    for (int n = 0; n < 27; n++) {
      if (v[nid[n]] < lo) lo = v[nid[n]];
      if (v[nid[n]] > hi) hi = v[nid[n]];
    }
    for (int q = 0; q < 27; q++) {
      double xi[3] = {GP[q % 3], GP[(q / 3) % 3], GP[q / 9]}, w[27], s = 0.0;
      o_q1_corner_weights(xi, w);
      for (int n = 0; n < 27; n++) s += w[n] * v[nid[n]];
      if (s < lo) s = lo;
      if (s > hi) s = hi;
      eta[27 * e + q] = s;
    }
  }
}

/* --------------------------------------------- Dirichlet conventions --- */
/* x_local[k] = 0 where mask[k] (src/dmda_bcs.c:500-526) */
void o_bc_zero(long n, const uint8_t *mask, double *x)
{
  for (long k = 0; k < n; k++)
    if (mask[k]) x[k] = 0.0;
}

/* y[k] = x[k] where mask[k]   (scale 1, src/dmda_bcs.c:574-611) */
void o_bc_insert_matmult(long n, const uint8_t *mask, const double *x, double *y)
{
  for (long k = 0; k < n; k++)
    if (mask[k]) y[k] = x[k];
}

/* y[k] = value where mask[k]  (src/dmda_bcs.c:409-) */
void o_bc_insert_value(long n, const uint8_t *mask, double value, double *y)
{
  for (long k = 0; k < n; k++)
    if (mask[k]) y[k] = value;
}

/* ------------------------------------------------------- body force --- */
/* bu_(n,l) += sum_q w detJ N_n(q) rho_q g_l  (the body-force term of the
 * velocity residual, src/stokes_form_function.c:99-243) */
void o_body_force(int mx, int my, int mz, const double *coords, const double *rho, double gx, double gy, double gz,
                  double *bu)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  double g[3] = {gx, gy, gz};
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], iJ[27][3][3], detJ[27];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_geometry(elx, iJ, detJ);
    for (int q = 0; q < 27; q++) {
      int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
      double s = WQ[q] * detJ[q] * rho[27 * e + q];
      for (int n = 0; n < 27; n++) {
        double N = BAS[qi][n % 3] * BAS[qj][(n / 3) % 3] * BAS[qk][n / 9];
        for (int l = 0; l < 3; l++) bu[3 * nid[n] + l] += s * N * g[l];
      }
    }
  }
}

/* Body-force terms of the Stokes residual from Gauss-point forces
 * (the Be / Be arrays of FormFunctionLocal_U and FormFunctionLocal_P,
 * src/stokes_form_function.c:99-243, 357-450):
 *   bu[3n+l] += sum_q w detJ N_n(q) fu[e][q][l],   bp[4e+k] += sum_q w detJ Np_k(q) fp[e][q]  */
void o_force_u(int mx, int my, int mz, const double *coords, const double *fu, double *bu)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], iJ[27][3][3], detJ[27];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_geometry(elx, iJ, detJ);
    for (int q = 0; q < 27; q++) {
      int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
      double s = WQ[q] * detJ[q];
      for (int n = 0; n < 27; n++) {
        double N = BAS[qi][n % 3] * BAS[qj][(n / 3) % 3] * BAS[qk][n / 9];
        for (int l = 0; l < 3; l++) bu[3 * nid[n] + l] += s * N * fu[81 * e + 3 * q + l];
      }
    }
  }
}

void o_force_p(int mx, int my, int mz, const double *coords, const double *fp, double *bp)
{
  o_mesh m = {mx, my, mz};
  o_tables();
  long nel = (long)mx * my * mz;
  for (long e = 0; e < nel; e++) {
    long nid[27];
    double elx[81], iJ[27][3][3], detJ[27];
    o_element_nodes(&m, e, nid);
    o_gather3(coords, nid, elx);
    o_geometry(elx, iJ, detJ);
    for (int q = 0; q < 27; q++) {
      double Np[4];
      o_pressure_basis(elx, q, Np);
      for (int k = 0; k < 4; k++) bp[4 * e + k] += WQ[q] * detJ[q] * Np[k] * fp[27 * e + q];
    }
  }
}
