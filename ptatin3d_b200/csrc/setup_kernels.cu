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
//   s_eta_project / s_eta_to_qp: the reference's Q1 projection hierarchy of
//                    Gauss-point viscosity (nodal projection, scaled
//                    restriction, clamped interpolation back to Gauss points)
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

// ---- the reference's Q1 projection hierarchy of Gauss-point viscosity
// (src/material_point_utils.c:1138-1257, 1379-1394, 894-1030)
__device__ __forceinline__ double q1w(int corner, double xi, double eta, double zeta)
{
  const int a = corner & 1, b = (corner >> 1) & 1, c = corner >> 2;
  return 0.125 * (a ? 1.0 + xi : 1.0 - xi) * (b ? 1.0 + eta : 1.0 - eta) * (c ? 1.0 + zeta : 1.0 - zeta);
}
__device__ __forceinline__ double gp1(int i) { return i == 0 ? -0.77459666924148337704 : (i == 1 ? 0.0 : 0.77459666924148337704); }

// A_n += N_n(q) eta_q, B_n += N_n(q): Q1 corner weights at the 8 corners, 1 at the other Q2 nodes
__global__ void k_eta_project(int mx, int my, int mz, const double *__restrict__ eta, double *__restrict__ A,
                              double *__restrict__ B)
{
  const size_t nel = (size_t)mx * my * mz;
  const int nx = 2 * mx + 1, ny = 2 * my + 1;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
    const int ex = e % mx, ey = (e / mx) % my, ez = e / ((size_t)mx * my);
    double sc[8] = {}, wc[8] = {}, se = 0.0;
    for (int q = 0; q < 27; q++) {
      const double v = eta[27 * e + q], xi = gp1(q % 3), et = gp1((q / 3) % 3), ze = gp1(q / 9);
      se += v;
      for (int c = 0; c < 8; c++) {
        const double w = q1w(c, xi, et, ze);
        sc[c] += w * v;
        wc[c] += w;
      }
    }
    for (int n = 0; n < 27; n++) {
      const int a = n % 3, b = (n / 3) % 3, c = n / 9;
      const size_t g = (size_t)(2 * ex + a) + (size_t)nx * ((size_t)(2 * ey + b) + (size_t)ny * (2 * ez + c));
      if (a != 1 && b != 1 && c != 1) {
        const int corner = (a >> 1) | ((b >> 1) << 1) | ((c >> 1) << 2);
        atomicAdd(A + g, sc[corner]);
        atomicAdd(B + g, wc[corner]);
      } else {
        atomicAdd(A + g, se);
        atomicAdd(B + g, 27.0);
      }
    }
  }
}
__global__ void k_divide(size_t n, double *__restrict__ a, const double *__restrict__ b)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) a[i] /= b[i];
}
// Gauss-point values from the nodal field: Q1 interpolation of the corners, clamped to the element's nodal range
__global__ void k_eta_to_qp(int mx, int my, int mz, const double *__restrict__ v, double *__restrict__ eta)
{
  const size_t nel = (size_t)mx * my * mz;
  const int nx = 2 * mx + 1, ny = 2 * my + 1;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
    const int ex = e % mx, ey = (e / mx) % my, ez = e / ((size_t)mx * my);
    double lo = 1e32, hi = -1e32, vc[8];
    for (int n = 0; n < 27; n++) {
      const int a = n % 3, b = (n / 3) % 3, c = n / 9;
      const double x = v[(size_t)(2 * ex + a) + (size_t)nx * ((size_t)(2 * ey + b) + (size_t)ny * (2 * ez + c))];
      lo = fmin(lo, x);
      hi = fmax(hi, x);
      if (a != 1 && b != 1 && c != 1) vc[(a >> 1) | ((b >> 1) << 1) | ((c >> 1) << 2)] = x;
    }
    for (int q = 0; q < 27; q++) {
      const double xi = gp1(q % 3), et = gp1((q / 3) % 3), ze = gp1(q / 9);
      double s = 0.0;
      for (int c = 0; c < 8; c++) s += q1w(c, xi, et, ze) * vc[c];
      eta[27 * e + q] = fmin(fmax(s, lo), hi);
    }
  }
}

void s_eta_project(int mx, int my, int mz, const double *eta, double *A, double *B, cudaStream_t s)
{
  const size_t nn = (size_t)(2 * mx + 1) * (2 * my + 1) * (2 * mz + 1);
  cudaMemsetAsync(A, 0, nn * 8, s);
  cudaMemsetAsync(B, 0, nn * 8, s);
  k_eta_project<<<sgrid((size_t)mx * my * mz), 128, 0, s>>>(mx, my, mz, eta, A, B);
  k_divide<<<sgrid(nn), 128, 0, s>>>(nn, A, B);
  count_launch(2);
}
__global__ void k_fill(size_t n, double v, double *__restrict__ a)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) a[i] = v;
}
void s_fill(size_t n, double v, double *a, cudaStream_t s)
{
  k_fill<<<sgrid(n), 128, 0, s>>>(n, v, a);
  count_launch(1);
}
void s_divide(size_t n, double *a, const double *b, cudaStream_t s)
{
  k_divide<<<sgrid(n), 128, 0, s>>>(n, a, b);
  count_launch(1);
}
void s_eta_to_qp(int mx, int my, int mz, const double *v, double *eta, cudaStream_t s)
{
  k_eta_to_qp<<<sgrid((size_t)mx * my * mz), 128, 0, s>>>(mx, my, mz, v, eta);
  count_launch(1);
}

// ---- residual body-force terms on a (possibly ghosted) local lattice
__device__ void gather_element_g(int gx, int gy, int ox, int oy, int oz, int ex, int ey, int ez, const double *coords,
                                 double X[27][3])
{
  for (int n = 0; n < 27; n++) {
    size_t g = (size_t)(ox + 2 * ex + n % 3) + (size_t)gx * ((size_t)(oy + 2 * ey + (n / 3) % 3) + (size_t)gy * (oz + 2 * ez + n / 9));
    for (int l = 0; l < 3; l++) X[n][l] = coords[3 * g + l];
  }
}
// ru[3n+l] -= sum_q w detJ N_n(q) fu[e][q][l]
__global__ void k_force_u(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, const double *__restrict__ coords,
                          const double *__restrict__ fu, double *__restrict__ ru)
{
  size_t nel = (size_t)mx * my * mz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
    const int ex = e % mx, ey = (e / mx) % my, ez = e / ((size_t)mx * my);
    double X[27][3];
    gather_element_g(gx, gy, ox, oy, oz, ex, ey, ez, coords, X);
    double acc[27][3] = {};
    for (int q = 0; q < 27; q++) {
      QPGeom g = qp_geom(X, q);
      const int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
      const double s = g.w * g.detJ;
      const double f0 = fu[81 * e + 3 * q], f1 = fu[81 * e + 3 * q + 1], f2 = fu[81 * e + 3 * q + 2];
      for (int n = 0; n < 27; n++) {
        const double N = s * bq(qi, n % 3) * bq(qj, (n / 3) % 3) * bq(qk, n / 9);
        acc[n][0] += N * f0; acc[n][1] += N * f1; acc[n][2] += N * f2;
      }
    }
    for (int n = 0; n < 27; n++) {
      size_t node = (size_t)(ox + 2 * ex + n % 3) + (size_t)gx * ((size_t)(oy + 2 * ey + (n / 3) % 3) + (size_t)gy * (oz + 2 * ez + n / 9));
      for (int l = 0; l < 3; l++) atomicAdd(ru + 3 * node + l, -acc[n][l]);
    }
  }
}
// rp[4e+k] -= sum_q w detJ Np_k(q) fp[e][q]  (Np = [1, xh, yh, zh], the global-relative P1 basis)
__global__ void k_force_p(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, const double *__restrict__ coords,
                          const double *__restrict__ fp, double *__restrict__ rp)
{
  size_t nel = (size_t)mx * my * mz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
    const int ex = e % mx, ey = (e / mx) % my, ez = e / ((size_t)mx * my);
    double X[27][3];
    gather_element_g(gx, gy, ox, oy, oz, ex, ey, ez, coords, X);
    double avg[3] = {0, 0, 0};
    for (int n = 0; n < 27; n++)
      for (int l = 0; l < 3; l++) avg[l] += X[n][l];
    for (int l = 0; l < 3; l++) avg[l] /= 27.0;
    const double L[3] = {X[14][0] - X[12][0], X[16][1] - X[10][1], X[22][2] - X[4][2]};
    double acc[4] = {0, 0, 0, 0};
    for (int q = 0; q < 27; q++) {
      QPGeom g = qp_geom(X, q);
      const double s = g.w * g.detJ * fp[27 * e + q];
      acc[0] += s;
      for (int l = 0; l < 3; l++) acc[1 + l] += s * (g.xq[l] - avg[l]) / L[l];
    }
    for (int k = 0; k < 4; k++) rp[4 * e + k] -= acc[k];
  }
}

void s_force_u(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, const double *coords, const double *fu,
               double *ru, cudaStream_t s)
{
  k_force_u<<<sgrid((size_t)mx * my * mz), 128, 0, s>>>(mx, my, mz, gx, gy, ox, oy, oz, coords, fu, ru);
  count_launch(1);
}
void s_force_p(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, const double *coords, const double *fp,
               double *rp, cudaStream_t s)
{
  k_force_p<<<sgrid((size_t)mx * my * mz), 128, 0, s>>>(mx, my, mz, gx, gy, ox, oy, oz, coords, fp, rp);
  count_launch(1);
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
