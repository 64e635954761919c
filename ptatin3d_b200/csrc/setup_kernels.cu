// Solver set-up kernels (run once per solve, FP64, one thread per element or node).
//
//   s_schur_blocks : inverse of the viscosity-scaled pressure mass matrix,
//                    dense 4x4 per element for P1disc
//                    (src/stokes_assembly.c:299-450 assembles the same blocks
//                    with 1/eta per quadrature point; the element geometric
//                    mean of eta is the alternative weighting)
//   s_body_force   : velocity right-hand side from a density field and gravity,
//                    b_(n,l) = sum_q w detJ N_n rho_q g_l (the body-force part of
//                    FormFunctionLocal_U, src/stokes_form_function.c:99-243)
//   s_restrict_eta : Gauss-point viscosity of a coarse level from the next finer
//                    one (geometric mean over the fine points nearest each coarse
//                    point; keeps eta positive across contrasts of 1e5)
//   s_inject_coords: coarse coordinates by injection on the node lattice
//                    (src/dmda_project_coords.c:73-95)
#include <cuda_runtime.h>

#include "p3d_internal.h"
#include "q2_tile.cuh"
#include "solver_internal.h"

namespace p3d {

static int sgrid(size_t n)
{
  size_t g = (n + 127) / 128;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

// Q2 basis / derivative at the Gauss points
__host__ __device__ __forceinline__ double bq(int q, int a)
{
  if (q == 1) return a == 1 ? 1.0 : 0.0;
  if (q == 0) return a == 0 ? P3D_B0 : (a == 1 ? P3D_B1 : P3D_B2);
  return a == 0 ? P3D_B2 : (a == 1 ? P3D_B1 : P3D_B0);
}
__host__ __device__ __forceinline__ double dq(int q, int a)
{
  const double s = 0.77459666924148337704;
  if (q == 1) return a == 0 ? -0.5 : (a == 1 ? 0.0 : 0.5);
  if (q == 0) return a == 0 ? -s - 0.5 : (a == 1 ? 2.0 * s : -s + 0.5);
  return a == 0 ? s - 0.5 : (a == 1 ? -2.0 * s : s + 0.5);
}

struct QPGeom {
  double detJ, w, xq[3];
};

// element nodes (whole-mesh lattice) -> detJ and physical position of Gauss point q
__device__ QPGeom qp_geom(const double X[27][3], int q)
{
  int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, xq[3] = {0, 0, 0};
  for (int n = 0; n < 27; n++) {
    int a = n % 3, b = (n / 3) % 3, c = n / 9;
    double g0 = dq(qi, a) * bq(qj, b) * bq(qk, c);
    double g1 = bq(qi, a) * dq(qj, b) * bq(qk, c);
    double g2 = bq(qi, a) * bq(qj, b) * dq(qk, c);
    double N = bq(qi, a) * bq(qj, b) * bq(qk, c);
    for (int l = 0; l < 3; l++) {
      J[0][l] += g0 * X[n][l];
      J[1][l] += g1 * X[n][l];
      J[2][l] += g2 * X[n][l];
      xq[l] += N * X[n][l];
    }
  }
  QPGeom r;
  r.detJ = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  r.w = w1d(qi) * w1d(qj) * w1d(qk);
  for (int l = 0; l < 3; l++) r.xq[l] = xq[l];
  return r;
}

__device__ void gather_element(int mx, int my, size_t e, const double *coords, double X[27][3])
{
  int ex = e % mx, ey = (e / mx) % my, ez = e / ((size_t)mx * my);
  int nx = 2 * mx + 1, ny = 2 * my + 1;
  for (int n = 0; n < 27; n++) {
    size_t g = (size_t)(2 * ex + n % 3) + (size_t)nx * ((size_t)(2 * ey + (n / 3) % 3) + (size_t)ny * (2 * ez + n / 9));
    for (int l = 0; l < 3; l++) X[n][l] = coords[3 * g + l];
  }
}

__global__ void k_schur_blocks(int mx, int my, int mz, const double *__restrict__ coords, const double *__restrict__ eta,
                               int geomean, double *__restrict__ Binv)
{
  size_t nel = (size_t)mx * my * mz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
    double X[27][3];
    gather_element(mx, my, e, coords, X);
    double avg[3] = {0, 0, 0};
    for (int n = 0; n < 27; n++)
      for (int l = 0; l < 3; l++) avg[l] += X[n][l];
    for (int l = 0; l < 3; l++) avg[l] /= 27.0;
    double L[3] = {X[14][0] - X[12][0], X[16][1] - X[10][1], X[22][2] - X[4][2]};
    double S[4][4] = {};
    double eg = 0.0;
    if (geomean) {
      for (int q = 0; q < 27; q++) eg += log(eta[27 * e + q]);
      eg = exp(eg / 27.0);
    }
    for (int q = 0; q < 27; q++) {
      QPGeom g = qp_geom(X, q);
      double Np[4] = {1.0, (g.xq[0] - avg[0]) / L[0], (g.xq[1] - avg[1]) / L[1], (g.xq[2] - avg[2]) / L[2]};
      double s = -g.w * g.detJ / (geomean ? eg : eta[27 * e + q]);
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) S[i][j] += s * Np[i] * Np[j];
    }
    // Gauss-Jordan inverse with partial pivoting of the 4x4 block
    double A[4][8];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 8; j++) A[i][j] = j < 4 ? S[i][j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; c++) {
      int piv = c;
      for (int r = c + 1; r < 4; r++)
        if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
      if (piv != c)
        for (int j = 0; j < 8; j++) { double t = A[c][j]; A[c][j] = A[piv][j]; A[piv][j] = t; }
      double inv = 1.0 / A[c][c];
      for (int j = 0; j < 8; j++) A[c][j] *= inv;
      for (int r = 0; r < 4; r++)
        if (r != c) {
          double f = A[r][c];
          for (int j = 0; j < 8; j++) A[r][j] -= f * A[c][j];
        }
    }
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) Binv[16 * e + 4 * i + j] = A[i][4 + j];
  }
}

__global__ void k_body_force(int mx, int my, int mz, const double *__restrict__ coords, const double *__restrict__ rho,
                             double g0, double g1, double g2, double *__restrict__ bu)
{
  size_t nel = (size_t)mx * my * mz;
  int nx = 2 * mx + 1, ny = 2 * my + 1;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
    double X[27][3];
    gather_element(mx, my, e, coords, X);
    double acc[27] = {};
    for (int q = 0; q < 27; q++) {
      QPGeom g = qp_geom(X, q);
      int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
      double s = g.w * g.detJ * rho[27 * e + q];
      for (int n = 0; n < 27; n++) acc[n] += s * bq(qi, n % 3) * bq(qj, (n / 3) % 3) * bq(qk, n / 9);
    }
    int ex = e % mx, ey = (e / mx) % my, ez = e / ((size_t)mx * my);
    for (int n = 0; n < 27; n++) {
      size_t node = (size_t)(2 * ex + n % 3) + (size_t)nx * ((size_t)(2 * ey + (n / 3) % 3) + (size_t)ny * (2 * ez + n / 9));
      if (g0 != 0.0) atomicAdd(bu + 3 * node + 0, acc[n] * g0);
      if (g1 != 0.0) atomicAdd(bu + 3 * node + 1, acc[n] * g1);
      if (g2 != 0.0) atomicAdd(bu + 3 * node + 2, acc[n] * g2);
    }
  }
}

__global__ void k_restrict_eta(int mxc, int myc, int mzc, const double *__restrict__ ef, double *__restrict__ ec)
{
  size_t nel = (size_t)mxc * myc * mzc;
  const int mxf = 2 * mxc, myf = 2 * myc;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < nel * 27; idx += (size_t)gridDim.x * blockDim.x) {
    size_t e = idx / 27;
    int q = idx % 27;
    int E[3] = {(int)(e % mxc), (int)((e / mxc) % myc), (int)(e / ((size_t)mxc * myc))};
    int Q[3] = {q % 3, (q / 3) % 3, q / 9};
    // per direction: candidate (child offset, fine Gauss index) pairs
    int nc[3], ch[3][2], fq[3][2];
    for (int d = 0; d < 3; d++) {
      if (Q[d] == 0) { nc[d] = 1; ch[d][0] = 0; fq[d][0] = 0; }
      else if (Q[d] == 2) { nc[d] = 1; ch[d][0] = 1; fq[d][0] = 2; }
      else { nc[d] = 2; ch[d][0] = 0; fq[d][0] = 2; ch[d][1] = 1; fq[d][1] = 0; }
    }
    double lsum = 0.0;
    int cnt = 0;
    for (int c = 0; c < nc[2]; c++)
      for (int b = 0; b < nc[1]; b++)
        for (int a = 0; a < nc[0]; a++) {
          size_t fe = (size_t)(2 * E[0] + ch[0][a]) + (size_t)mxf * ((size_t)(2 * E[1] + ch[1][b]) + (size_t)myf * (2 * E[2] + ch[2][c]));
          int fqq = fq[0][a] + 3 * fq[1][b] + 9 * fq[2][c];
          lsum += log(ef[27 * fe + fqq]);
          cnt++;
        }
    ec[idx] = exp(lsum / cnt);
  }
}

__global__ void k_inject(int cnx, int cny, int cnz, const double *__restrict__ cf, double *__restrict__ cc)
{
  size_t n = (size_t)cnx * cny * cnz;
  int fnx = 2 * cnx - 1, fny = 2 * cny - 1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    int I = i % cnx, J = (i / cnx) % cny, K = i / ((size_t)cnx * cny);
    size_t f = (size_t)(2 * I) + (size_t)fnx * ((size_t)(2 * J) + (size_t)fny * (2 * K));
    for (int l = 0; l < 3; l++) cc[3 * i + l] = cf[3 * f + l];
  }
}

void s_schur_blocks(int mx, int my, int mz, const double *coords, const double *eta, int geomean, double *Binv,
                    cudaStream_t s)
{
  k_schur_blocks<<<sgrid((size_t)mx * my * mz), 128, 0, s>>>(mx, my, mz, coords, eta, geomean, Binv);
  count_launch(1);
}
void s_body_force(int mx, int my, int mz, const double *coords, const double *rho, double g[3], double *bu, cudaStream_t s)
{
  k_body_force<<<sgrid((size_t)mx * my * mz), 128, 0, s>>>(mx, my, mz, coords, rho, g[0], g[1], g[2], bu);
  count_launch(1);
}
void s_restrict_eta(int mxc, int myc, int mzc, const double *eta_f, double *eta_c, cudaStream_t s)
{
  k_restrict_eta<<<sgrid((size_t)mxc * myc * mzc * 27), 128, 0, s>>>(mxc, myc, mzc, eta_f, eta_c);
  count_launch(1);
}
void s_inject_coords(int cnx, int cny, int cnz, const double *cf, double *cc, cudaStream_t s)
{
  k_inject<<<sgrid((size_t)cnx * cny * cnz), 128, 0, s>>>(cnx, cny, cnz, cf, cc);
  count_launch(1);
}

} // namespace p3d
