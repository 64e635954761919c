// In-place inverse of the dense coarse-grid operator (symmetric positive
// definite, row-major n x n) by blocked Gauss-Jordan elimination.
//
// Pivots are taken in panels P = [k0, k0+b), b <= 32.  One panel step is the
// block sweep
//     A_PP <- A_PP^{-1}              A_PR <- A_PP^{-1} A_PR
//     A_RP <- -A_RP A_PP^{-1}        A_RR <- A_RR - A_RP A_PP^{-1} A_PR
// (R = the other indices); sweeping every panel in turn leaves A^{-1}.  No
// pivoting: the blocks met are Schur complements of an SPD matrix.  Per panel
// the kernels are
//     k_gj_cols    C = A[:, P]                      (n x b, kept before A changes)
//     k_gj_pivot   A_PP^{-1} (one CTA, scalar Gauss-Jordan in shared memory)
//     k_gj_rows    W = A_PP^{-1} A[P, :], with W[:, P] = A_PP^{-1}
//     k_gj_update  rows in P: A = W; other rows: A = A - C W (columns in P: -C W),
//                  a rank-b update in 32 x 32 shared-memory tiles
// so that an n = 2187 coarse inverse (4^3 Q2 elements) takes 69 panel steps
// instead of 2187 scalar ones.
#include <cuda_runtime.h>

#include <algorithm>

#include "p3d_internal.h"
#include "solver_internal.h"

namespace p3d {

constexpr int GJB = 32;

__global__ void k_gj_cols(int n, int k0, int b, const double *__restrict__ A, double *__restrict__ C)
{
  const size_t total = (size_t)n * b;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t i = idx / b;
    const int p = idx % b;
    C[i * GJB + p] = A[i * n + k0 + p];
  }
}

// one CTA of GJB x GJB threads
__global__ void __launch_bounds__(GJB *GJB) k_gj_pivot(int n, int k0, int b, const double *__restrict__ A,
                                                        double *__restrict__ Pinv)
{
  __shared__ double M[GJB][GJB + 1];
  __shared__ double col[GJB], row[GJB];
  const int i = threadIdx.y, j = threadIdx.x;
  const bool in = i < b && j < b;
  M[i][j] = in ? A[(size_t)(k0 + i) * n + k0 + j] : 0.0;
  __syncthreads();
  for (int k = 0; k < b; k++) {
    if (i == 0 && j < b) row[j] = M[k][j];
    if (j == 0 && i < b) col[i] = M[i][k];
    __syncthreads();
    if (in) {
      const double piv = row[k];
      double v;
      if (i == k) v = (j == k) ? 1.0 / piv : row[j] / piv;
      else if (j == k) v = -col[i] / piv;
      else v = M[i][j] - col[i] * row[j] / piv;
      M[i][j] = v;
    }
    __syncthreads();
  }
  if (in) Pinv[i * GJB + j] = M[i][j];
}

__global__ void k_gj_rows(int n, int k0, int b, const double *__restrict__ A, const double *__restrict__ Pinv,
                          double *__restrict__ W)
{
  const size_t total = (size_t)b * n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int p = idx / n, j = idx % n;
    double s;
    if (j >= k0 && j < k0 + b) {
      s = Pinv[p * GJB + (j - k0)];
    } else {
      s = 0.0;
      for (int q = 0; q < b; q++) s += Pinv[p * GJB + q] * A[(size_t)(k0 + q) * n + j];
    }
    W[(size_t)p * n + j] = s;
  }
}

// 32 x 32 output tile per CTA of 32 x 8 threads (4 rows per thread)
__global__ void __launch_bounds__(256) k_gj_update(int n, int k0, int b, double *__restrict__ A, const double *__restrict__ C,
                                                   const double *__restrict__ W)
{
  __shared__ double Ct[GJB][GJB + 1]; // [tile row][p]
  __shared__ double Wt[GJB][GJB + 1]; // [p][tile col]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = blockIdx.x * GJB + tx, i0 = blockIdx.y * GJB;
  for (int r = ty; r < GJB; r += 8) {
    const int i = i0 + r;
    Ct[r][tx] = (i < n && tx < b) ? C[(size_t)i * GJB + tx] : 0.0;
    Wt[r][tx] = (r < b && j < n) ? W[(size_t)r * n + j] : 0.0;
  }
  __syncthreads();
  if (j >= n) return;
  const bool jp = j >= k0 && j < k0 + b;
  for (int r = ty; r < GJB; r += 8) {
    const int i = i0 + r;
    if (i >= n) break;
    const size_t g = (size_t)i * n + j;
    if (i >= k0 && i < k0 + b) {
      A[g] = Wt[i - k0][tx];
    } else {
      double acc = 0.0;
#pragma unroll 8
      for (int p = 0; p < GJB; p++) acc += Ct[r][p] * Wt[p][tx];
      A[g] = (jp ? 0.0 : A[g]) - acc;
    }
  }
}

// scratch: GJB*n (C) + GJB*n (W) + GJB*GJB (pivot inverse) doubles
size_t dense_inverse_scratch(int n) { return (size_t)2 * GJB * n + GJB * GJB; }

int dense_inverse_spd(int n, double *A, double *scratch, cudaStream_t s)
{
  double *C = scratch, *W = scratch + (size_t)GJB * n, *Pinv = scratch + (size_t)2 * GJB * n;
  const int g1 = (int)std::min<size_t>(((size_t)n * GJB + 255) / 256, 148 * 8);
  const dim3 tb(GJB, 8), tg((n + GJB - 1) / GJB, (n + GJB - 1) / GJB);
  for (int k0 = 0; k0 < n; k0 += GJB) {
    const int b = n - k0 < GJB ? n - k0 : GJB;
    k_gj_cols<<<g1, 256, 0, s>>>(n, k0, b, A, C);
    k_gj_pivot<<<1, dim3(GJB, GJB), 0, s>>>(n, k0, b, A, Pinv);
    k_gj_rows<<<g1, 256, 0, s>>>(n, k0, b, A, Pinv, W);
    k_gj_update<<<tg, tb, 0, s>>>(n, k0, b, A, C, W);
    count_launch(4);
  }
  return cuda_check(cudaGetLastError(), "dense inverse");
}

} // namespace p3d
