// Galerkin coarse operators of the velocity multigrid as 27-point block stencils.
//
// With trilinear transfers on the node lattice (coarse node I <-> fine node 2I),
// the Galerkin product Ac = P^T A P of a Q2 operator couples each coarse node
// only with its 27 lattice neighbours: P spreads node I over fine nodes
// 2I-1..2I+1, A couples those with fine nodes 2I-2..2I+2 (a Q2 element spans
// three lattice nodes per direction), and P^T gathers them back onto coarse
// nodes I-1..I+1.  The same holds for P^T Ac P, so every coarse level of the
// hierarchy is a variable-coefficient 27-point stencil of 3x3 blocks:
//
//   G[((o*3 + r)*3 + c) * nn + i]   o = (dk+1)*9 + (dj+1)*3 + (di+1)   neighbour
//                                   r, c = row / column velocity component
//
// stored entry-major so that the threads of a warp read consecutive nodes'
// coefficients (coalesced).  The reference forms the same operators with
// PETSc's MatPtAP on assembled matrices (OP_TYPE_GALERKIN,
// src/ptatin_driver_linear_ts.c:712-762); here they are formed matrix-free
// by probing: nodes coloured by (I mod 3, J mod 3, K mod 3) have at most one
// member in any 27-neighbourhood, so 27 colours x 3 components = 81 applies of
// the finer operator recover every coefficient.
#include <cuda_runtime.h>

#include "p3d_internal.h"
#include "q2_tile.cuh"
#include "solver_internal.h"

namespace p3d {

static int ggrid(size_t n)
{
  size_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

#define G_LOOP(i, n) for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

// y = G x (overwrites y); accumulation in T.  A block covers 32 consecutive
// nodes with 9 warps, one per (row component r, neighbour plane dk): each
// thread sums the 9 neighbours of its plane (27 coalesced coefficient loads,
// the x values shared through L1), and the three plane partials of a row meet
// in shared memory.  Nine independent load streams per node keep enough bytes
// in flight to stream the coefficients even on the small coarse levels.
constexpr int STENCIL_NODES = 32;
template <typename T>
__device__ __forceinline__ void stencil_apply_body(int nx, int ny, int nz, const T *__restrict__ G, const T *__restrict__ x,
                                                   T *__restrict__ y)
{
  __shared__ T part[9][STENCIL_NODES];
  const size_t nn = (size_t)nx * ny * nz;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5; // w = 3 r + (dk + 1)
  const int r = w / 3, dk = w % 3 - 1;
  const size_t i = (size_t)blockIdx.x * STENCIL_NODES + lane;
  T a = 0;
  if (i < nn) {
    const int I = i % nx, J = (i / nx) % ny, K = i / ((size_t)nx * ny);
    if (K + dk >= 0 && K + dk < nz) {
#pragma unroll
      for (int o9 = 0; o9 < 9; o9++) {
        const int di = o9 % 3 - 1, dj = o9 / 3 - 1;
        if (I + di < 0 || I + di >= nx || J + dj < 0 || J + dj >= ny) continue;
        const long long j = (long long)i + di + (long long)nx * (dj + (long long)ny * dk);
        const T *g = G + ((size_t)((dk + 1) * 9 + o9) * 9 + 3 * r) * nn + i;
        a += g[0] * x[3 * j] + g[nn] * x[3 * j + 1] + g[2 * nn] * x[3 * j + 2];
      }
    }
  }
  part[w][lane] = a;
  __syncthreads();
  if (dk == -1 && i < nn) y[3 * i + r] = part[w][lane] + part[w + 1][lane] + part[w + 2][lane];
}
template <typename T>
__global__ void __launch_bounds__(9 * STENCIL_NODES) k_stencil_apply(int nx, int ny, int nz, const T *__restrict__ G,
                                                                    const T *__restrict__ x, T *__restrict__ y)
{
  stencil_apply_body<T>(nx, ny, nz, G, x, y);
}
// over the members of a group (blockIdx.y = member): a = G, b = x, out = y
template <typename T>
__global__ void __launch_bounds__(9 * STENCIL_NODES) k_stencil_apply_group(const __grid_constant__ TGroup<T> P, int nx, int ny,
                                                                          int nz)
{
  stencil_apply_body<T>(nx, ny, nz, P.a[blockIdx.y], P.b[blockIdx.y], P.out[blockIdx.y]);
}

// probe vector: component d of every node of colour (ci,cj,ck), zero on Dirichlet dofs
__global__ void k_probe_vec(int nx, int ny, int nz, int ci, int cj, int ck, int d, uint32_t dir, double *__restrict__ x)
{
  const size_t nn = (size_t)nx * ny * nz;
  G_LOOP(i, nn)
  {
    const int I = i % nx, J = (i / nx) % ny, K = i / ((size_t)nx * ny);
    const bool on = (I % 3 == ci) && (J % 3 == cj) && (K % 3 == ck) &&
                    !is_dirichlet(dir, I, J, K, 0, 0, 0, nx - 1, ny - 1, nz - 1, d);
    x[3 * i] = (d == 0 && on) ? 1.0 : 0.0;
    x[3 * i + 1] = (d == 1 && on) ? 1.0 : 0.0;
    x[3 * i + 2] = (d == 2 && on) ? 1.0 : 0.0;
  }
}

// column (colour, d) of the probed operator -> the stencil entries of that neighbour
__global__ void k_probe_scatter(int nx, int ny, int nz, int ci, int cj, int ck, int d, const double *__restrict__ y,
                                double *__restrict__ G)
{
  const size_t nn = (size_t)nx * ny * nz;
  G_LOOP(i, nn)
  {
    const int I = i % nx, J = (i / nx) % ny, K = i / ((size_t)nx * ny);
    // the colour's member among the neighbours: offset in {-1,0,1} per direction
    const int ti = (ci - I % 3 + 3) % 3, tj = (cj - J % 3 + 3) % 3, tk = (ck - K % 3 + 3) % 3;
    const int di = ti == 2 ? -1 : ti, dj = tj == 2 ? -1 : tj, dk = tk == 2 ? -1 : tk;
    if (I + di < 0 || I + di >= nx || J + dj < 0 || J + dj >= ny || K + dk < 0 || K + dk >= nz) continue;
    const int o = (dk + 1) * 9 + (dj + 1) * 3 + (di + 1);
#pragma unroll
    for (int r = 0; r < 3; r++) G[((size_t)o * 9 + r * 3 + d) * nn + i] = y[3 * i + r];
  }
}

// Dirichlet dofs: identity row (the probe already left their rows and columns zero)
__global__ void k_stencil_dirichlet(int nx, int ny, int nz, uint32_t dir, double *__restrict__ G)
{
  const size_t nn = (size_t)nx * ny * nz;
  G_LOOP(i, nn)
  {
    const int I = i % nx, J = (i / nx) % ny, K = i / ((size_t)nx * ny);
#pragma unroll
    for (int r = 0; r < 3; r++)
      if (is_dirichlet(dir, I, J, K, 0, 0, 0, nx - 1, ny - 1, nz - 1, r)) G[((size_t)13 * 9 + r * 4) * nn + i] = 1.0;
  }
}

__global__ void k_stencil_diag(int nx, int ny, int nz, const double *__restrict__ G, double *__restrict__ d)
{
  const size_t nn = (size_t)nx * ny * nz;
  G_LOOP(i, nn)
  {
#pragma unroll
    for (int r = 0; r < 3; r++) d[3 * i + r] = G[((size_t)13 * 9 + r * 4) * nn + i];
  }
}

// dense row-major copy (coarsest level, inverted by Gauss-Jordan)
__global__ void k_stencil_dense(int nx, int ny, int nz, const double *__restrict__ G, double *__restrict__ M)
{
  const size_t nn = (size_t)nx * ny * nz, n = 3 * nn;
  G_LOOP(idx, nn * 27)
  {
    const size_t i = idx % nn;
    const int o = idx / nn;
    const int I = i % nx, J = (i / nx) % ny, K = i / ((size_t)nx * ny);
    const int di = o % 3 - 1, dj = (o / 3) % 3 - 1, dk = o / 9 - 1;
    if (I + di < 0 || I + di >= nx || J + dj < 0 || J + dj >= ny || K + dk < 0 || K + dk >= nz) continue;
    const size_t j = (size_t)((long long)i + di + (long long)nx * (dj + (long long)ny * dk));
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) M[(3 * i + r) * n + 3 * j + c] = G[((size_t)o * 9 + r * 3 + c) * nn + i];
  }
}

template <typename T> void g_apply(int nx, int ny, int nz, const T *G, const T *x, T *y, cudaStream_t s)
{
  const size_t nn = (size_t)nx * ny * nz;
  k_stencil_apply<T><<<(unsigned)((nn + STENCIL_NODES - 1) / STENCIL_NODES), 9 * STENCIL_NODES, 0, s>>>(nx, ny, nz, G, x, y);
  count_launch(1);
}
template <typename T> void g_apply_group(const TGroup<T> &P, int K, int nx, int ny, int nz, cudaStream_t s)
{
  const size_t nn = (size_t)nx * ny * nz;
  k_stencil_apply_group<T><<<dim3((unsigned)((nn + STENCIL_NODES - 1) / STENCIL_NODES), K), 9 * STENCIL_NODES, 0, s>>>(P, nx,
                                                                                                                     ny, nz);
  count_launch(1);
}
template void g_apply_group<double>(const TGroup<double> &, int, int, int, int, cudaStream_t);
template void g_apply_group<float>(const TGroup<float> &, int, int, int, int, cudaStream_t);
void g_probe_vec(int nx, int ny, int nz, int ci, int cj, int ck, int d, uint32_t dir, double *x, cudaStream_t s)
{
  k_probe_vec<<<ggrid((size_t)nx * ny * nz), 256, 0, s>>>(nx, ny, nz, ci, cj, ck, d, dir, x);
  count_launch(1);
}
void g_probe_scatter(int nx, int ny, int nz, int ci, int cj, int ck, int d, const double *y, double *G, cudaStream_t s)
{
  k_probe_scatter<<<ggrid((size_t)nx * ny * nz), 256, 0, s>>>(nx, ny, nz, ci, cj, ck, d, y, G);
  count_launch(1);
}
void g_dirichlet(int nx, int ny, int nz, uint32_t dir, double *G, cudaStream_t s)
{
  if (!dir) return;
  k_stencil_dirichlet<<<ggrid((size_t)nx * ny * nz), 256, 0, s>>>(nx, ny, nz, dir, G);
  count_launch(1);
}
void g_diag(int nx, int ny, int nz, const double *G, double *d, cudaStream_t s)
{
  k_stencil_diag<<<ggrid((size_t)nx * ny * nz), 256, 0, s>>>(nx, ny, nz, G, d);
  count_launch(1);
}
void g_dense(int nx, int ny, int nz, const double *G, double *M, cudaStream_t s)
{
  k_stencil_dense<<<ggrid((size_t)nx * ny * nz * 27), 256, 0, s>>>(nx, ny, nz, G, M);
  count_launch(1);
}

template void g_apply<double>(int, int, int, const double *, const double *, double *, cudaStream_t);
template void g_apply<float>(int, int, int, const float *, const float *, float *, cudaStream_t);

} // namespace p3d
