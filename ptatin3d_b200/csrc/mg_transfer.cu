// Geometric-multigrid transfer on the Q2 node lattice.
//
// PETSc's DMCreateInterpolation between two DMDAs whose node counts satisfy
// Nf = 2 Nc - 1 (called at src/ptatin_driver_linear_ts.c:986-990 and handed to
// PCMGSetInterpolation at :850) is the tensor-product linear interpolation on
// the node lattice: a fine node with an even index coincides with a coarse
// node, an odd index sits halfway between two.  Restriction is the transpose.
// Both kernels are gathers (one thread per output node and component), so
// they are deterministic and need no atomics.
#include <cuda_runtime.h>

#include "p3d_b200.h"
#include "p3d_internal.h"
#include "q2_tile.cuh"
#include "solver_internal.h"

namespace p3d {

template <typename T>
__global__ void prolong_kernel(int cnx, int cny, int cnz, int ndof, const T *__restrict__ xc, T *__restrict__ xf)
{
  const int fnx = 2 * cnx - 1, fny = 2 * cny - 1, fnz = 2 * cnz - 1;
  const size_t total = (size_t)fnx * fny * fnz * ndof;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    int d = idx % ndof;
    size_t node = idx / ndof;
    int i = node % fnx, j = (node / fnx) % fny, k = node / ((size_t)fnx * fny);
    int i0 = i >> 1, i1 = (i + 1) >> 1, j0 = j >> 1, j1 = (j + 1) >> 1, k0 = k >> 1, k1 = (k + 1) >> 1;
    auto C = [&](int a, int b, int c) { return xc[((size_t)a + (size_t)cnx * ((size_t)b + (size_t)cny * c)) * ndof + d]; };
    T v;
    // the 2x2x2 average degenerates to copies along even directions
    T s00 = C(i0, j0, k0) + C(i1, j0, k0), s10 = C(i0, j1, k0) + C(i1, j1, k0);
    T s01 = C(i0, j0, k1) + C(i1, j0, k1), s11 = C(i0, j1, k1) + C(i1, j1, k1);
    v = (T)0.125 * ((s00 + s10) + (s01 + s11));
    xf[idx] = v;
  }
}

template <typename T>
__global__ void restrict_kernel(int cnx, int cny, int cnz, int ndof, const T *__restrict__ xf, T *__restrict__ xc)
{
  const int fnx = 2 * cnx - 1, fny = 2 * cny - 1, fnz = 2 * cnz - 1;
  const size_t total = (size_t)cnx * cny * cnz * ndof;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    int d = idx % ndof;
    size_t node = idx / ndof;
    int I = node % cnx, J = (node / cnx) % cny, K = node / ((size_t)cnx * cny);
    T acc = (T)0;
    for (int c = -1; c <= 1; c++) {
      int k = 2 * K + c;
      if (k < 0 || k >= fnz) continue;
      T wk = c == 0 ? (T)1 : (T)0.5;
      for (int b = -1; b <= 1; b++) {
        int j = 2 * J + b;
        if (j < 0 || j >= fny) continue;
        T wj = b == 0 ? (T)1 : (T)0.5;
        for (int a = -1; a <= 1; a++) {
          int i = 2 * I + a;
          if (i < 0 || i >= fnx) continue;
          T wi = a == 0 ? (T)1 : (T)0.5;
          acc += wi * wj * wk * xf[((size_t)i + (size_t)fnx * ((size_t)j + (size_t)fny * k)) * ndof + d];
        }
      }
    }
    xc[idx] = acc;
  }
}

// Velocity V-cycle forms (3 dofs per node, Dirichlet bits dir on the faces of
// both lattices): the residual b - Ax is formed on the fly and its Dirichlet
// dofs count as zero, the coarse Dirichlet dofs are zeroed; one pass instead
// of residual, mask, restriction and mask.
template <typename T>
__device__ __forceinline__ void restrict_residual_body(int cnx, int cny, int cnz, uint32_t dir, const T *__restrict__ b,
                                                       const T *__restrict__ Ax, T *__restrict__ xc)
{
  const int fnx = 2 * cnx - 1, fny = 2 * cny - 1, fnz = 2 * cnz - 1;
  const size_t total = (size_t)cnx * cny * cnz * 3;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int d = idx % 3;
    const size_t node = idx / 3;
    const int I = node % cnx, J = (node / cnx) % cny, K = node / ((size_t)cnx * cny);
    if (is_dirichlet(dir, I, J, K, 0, 0, 0, cnx - 1, cny - 1, cnz - 1, d)) {
      xc[idx] = (T)0;
      continue;
    }
    T acc = (T)0;
    for (int c = -1; c <= 1; c++) {
      const int k = 2 * K + c;
      if (k < 0 || k >= fnz) continue;
      const T wk = c == 0 ? (T)1 : (T)0.5;
      for (int bb = -1; bb <= 1; bb++) {
        const int j = 2 * J + bb;
        if (j < 0 || j >= fny) continue;
        const T wj = bb == 0 ? (T)1 : (T)0.5;
        for (int a = -1; a <= 1; a++) {
          const int i = 2 * I + a;
          if (i < 0 || i >= fnx) continue;
          if (is_dirichlet(dir, i, j, k, 0, 0, 0, fnx - 1, fny - 1, fnz - 1, d)) continue;
          const T wi = a == 0 ? (T)1 : (T)0.5;
          const size_t f = ((size_t)i + (size_t)fnx * ((size_t)j + (size_t)fny * k)) * 3 + d;
          acc += wi * wj * wk * (b[f] - Ax[f]);
        }
      }
    }
    xc[idx] = acc;
  }
}

template <typename T>
__global__ void restrict_residual_kernel(int cnx, int cny, int cnz, uint32_t dir, const T *__restrict__ b,
                                         const T *__restrict__ Ax, T *__restrict__ xc)
{
  restrict_residual_body<T>(cnx, cny, cnz, dir, b, Ax, xc);
}
// over the members of a group (blockIdx.y = member): a = b, b = Ax, out = xc
template <typename T>
__global__ void restrict_residual_group(const __grid_constant__ TGroup<T> G, int cnx, int cny, int cnz, uint32_t dir)
{
  restrict_residual_body<T>(cnx, cny, cnz, dir, G.a[blockIdx.y], G.b[blockIdx.y], G.out[blockIdx.y]);
}

template <typename T>
__device__ __forceinline__ void prolong_add_body(int cnx, int cny, int cnz, uint32_t dir, const T *__restrict__ xc,
                                                 T *__restrict__ xf)
{
  const int fnx = 2 * cnx - 1, fny = 2 * cny - 1, fnz = 2 * cnz - 1;
  const size_t total = (size_t)fnx * fny * fnz * 3;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int d = idx % 3;
    const size_t node = idx / 3;
    const int i = node % fnx, j = (node / fnx) % fny, k = node / ((size_t)fnx * fny);
    if (is_dirichlet(dir, i, j, k, 0, 0, 0, fnx - 1, fny - 1, fnz - 1, d)) continue;
    const int i0 = i >> 1, i1 = (i + 1) >> 1, j0 = j >> 1, j1 = (j + 1) >> 1, k0 = k >> 1, k1 = (k + 1) >> 1;
    auto C = [&](int a, int bb, int c) { return xc[((size_t)a + (size_t)cnx * ((size_t)bb + (size_t)cny * c)) * 3 + d]; };
    const T s00 = C(i0, j0, k0) + C(i1, j0, k0), s10 = C(i0, j1, k0) + C(i1, j1, k0);
    const T s01 = C(i0, j0, k1) + C(i1, j0, k1), s11 = C(i0, j1, k1) + C(i1, j1, k1);
    xf[idx] += (T)0.125 * ((s00 + s10) + (s01 + s11));
  }
}

template <typename T>
__global__ void prolong_add_kernel(int cnx, int cny, int cnz, uint32_t dir, const T *__restrict__ xc, T *__restrict__ xf)
{
  prolong_add_body<T>(cnx, cny, cnz, dir, xc, xf);
}
// over the members of a group: a = xc, out = xf
template <typename T>
__global__ void prolong_add_group(const __grid_constant__ TGroup<T> G, int cnx, int cny, int cnz, uint32_t dir)
{
  prolong_add_body<T>(cnx, cny, cnz, dir, G.a[blockIdx.y], G.out[blockIdx.y]);
}

static int tgrid(size_t n)
{
  size_t g = (n + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  return g < 1 ? 1 : (int)g;
}

template <typename T> int mg_prolong(int cnx, int cny, int cnz, int ndof, const T *xc, T *xf, cudaStream_t st)
{
  size_t n = (size_t)(2 * cnx - 1) * (2 * cny - 1) * (2 * cnz - 1) * ndof;
  prolong_kernel<T><<<tgrid(n), 256, 0, st>>>(cnx, cny, cnz, ndof, xc, xf);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "prolong launch");
}
template <typename T> int mg_restrict(int cnx, int cny, int cnz, int ndof, const T *xf, T *xc, cudaStream_t st)
{
  size_t n = (size_t)cnx * cny * cnz * ndof;
  restrict_kernel<T><<<tgrid(n), 256, 0, st>>>(cnx, cny, cnz, ndof, xf, xc);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "restrict launch");
}
template <typename T>
int mg_restrict_residual(int cnx, int cny, int cnz, uint32_t dir, const T *b, const T *Ax, T *xc, cudaStream_t st)
{
  size_t n = (size_t)cnx * cny * cnz * 3;
  restrict_residual_kernel<T><<<tgrid(n), 256, 0, st>>>(cnx, cny, cnz, dir, b, Ax, xc);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "restrict launch");
}
template <typename T> int mg_prolong_add(int cnx, int cny, int cnz, uint32_t dir, const T *xc, T *xf, cudaStream_t st)
{
  size_t n = (size_t)(2 * cnx - 1) * (2 * cny - 1) * (2 * cnz - 1) * 3;
  prolong_add_kernel<T><<<tgrid(n), 256, 0, st>>>(cnx, cny, cnz, dir, xc, xf);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "prolong launch");
}
template <typename T>
int mg_restrict_residual_group(const TGroup<T> &G, int K, int cnx, int cny, int cnz, uint32_t dir, cudaStream_t st)
{
  size_t n = (size_t)cnx * cny * cnz * 3;
  restrict_residual_group<T><<<dim3(tgrid(n), K), 256, 0, st>>>(G, cnx, cny, cnz, dir);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "grouped restrict launch");
}
template <typename T>
int mg_prolong_add_group(const TGroup<T> &G, int K, int cnx, int cny, int cnz, uint32_t dir, cudaStream_t st)
{
  size_t n = (size_t)(2 * cnx - 1) * (2 * cny - 1) * (2 * cnz - 1) * 3;
  prolong_add_group<T><<<dim3(tgrid(n), K), 256, 0, st>>>(G, cnx, cny, cnz, dir);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "grouped prolong launch");
}
template int mg_restrict_residual_group<double>(const TGroup<double> &, int, int, int, int, uint32_t, cudaStream_t);
template int mg_restrict_residual_group<float>(const TGroup<float> &, int, int, int, int, uint32_t, cudaStream_t);
template int mg_prolong_add_group<double>(const TGroup<double> &, int, int, int, int, uint32_t, cudaStream_t);
template int mg_prolong_add_group<float>(const TGroup<float> &, int, int, int, int, uint32_t, cudaStream_t);
template int mg_restrict_residual<double>(int, int, int, uint32_t, const double *, const double *, double *, cudaStream_t);
template int mg_restrict_residual<float>(int, int, int, uint32_t, const float *, const float *, float *, cudaStream_t);
template int mg_prolong_add<double>(int, int, int, uint32_t, const double *, double *, cudaStream_t);
template int mg_prolong_add<float>(int, int, int, uint32_t, const float *, float *, cudaStream_t);
template int mg_prolong<double>(int, int, int, int, const double *, double *, cudaStream_t);
template int mg_prolong<float>(int, int, int, int, const float *, float *, cudaStream_t);
template int mg_restrict<double>(int, int, int, int, const double *, double *, cudaStream_t);
template int mg_restrict<float>(int, int, int, int, const float *, float *, cudaStream_t);

} // namespace p3d

namespace p3d {

// y += recv on one node plane (3 components per node), then the plane's
// Dirichlet rows reset to x: the second half of DMLocalToGlobal(ADD) on a
// z-slab boundary plane followed by the MatMult row convention
template <typename T>
__global__ void slab_plane_kernel(int nx, int ny, uint32_t dir, const T *__restrict__ recv, const T *__restrict__ x,
                                  T *__restrict__ y)
{
  const int n = 3 * nx * ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % 3, node = i / 3, ix = node % nx, iy = node / nx;
    bool d = (ix == 0 && (dir >> (0 + c) & 1u)) || (ix == nx - 1 && (dir >> (3 + c) & 1u)) ||
             (iy == 0 && (dir >> (6 + c) & 1u)) || (iy == ny - 1 && (dir >> (9 + c) & 1u));
    y[i] = d ? x[i] : y[i] + recv[i];
  }
}

} // namespace p3d

using namespace p3d;

extern "C" {
int p3d_slab_add_plane(int prec, int32_t mx, int32_t my, uint32_t dirichlet, const void *recv, const void *x_plane,
                       void *y_plane, void *stream)
{
  if (mx < 1 || my < 1 || !recv || !x_plane || !y_plane) return set_error(P3D_ERR_ARG, "slab_add_plane: bad args");
  const int nx = 2 * mx + 1, ny = 2 * my + 1, n = 3 * nx * ny;
  const int grid = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == P3D_PREC_F64)
    slab_plane_kernel<double><<<grid, 256, 0, st>>>(nx, ny, dirichlet, (const double *)recv, (const double *)x_plane,
                                                   (double *)y_plane);
  else if (prec == P3D_PREC_F32)
    slab_plane_kernel<float><<<grid, 256, 0, st>>>(nx, ny, dirichlet, (const float *)recv, (const float *)x_plane,
                                                  (float *)y_plane);
  else
    return set_error(P3D_ERR_ARG, "slab_add_plane: precision must be 64 or 32");
  count_launch(1);
  return cuda_check(cudaGetLastError(), "slab_add_plane");
}

int p3d_mg_prolong(int prec, int cnx, int cny, int cnz, int ndof, const void *xc, void *xf, void *stream)
{
  if (cnx < 1 || cny < 1 || cnz < 1 || ndof < 1 || !xc || !xf) return set_error(P3D_ERR_ARG, "mg_prolong: bad args");
  if (prec == P3D_PREC_F64) return mg_prolong<double>(cnx, cny, cnz, ndof, (const double *)xc, (double *)xf, (cudaStream_t)stream);
  if (prec == P3D_PREC_F32) return mg_prolong<float>(cnx, cny, cnz, ndof, (const float *)xc, (float *)xf, (cudaStream_t)stream);
  return set_error(P3D_ERR_ARG, "mg_prolong: precision must be 64 or 32");
}
int p3d_mg_restrict(int prec, int cnx, int cny, int cnz, int ndof, const void *xf, void *xc, void *stream)
{
  if (cnx < 1 || cny < 1 || cnz < 1 || ndof < 1 || !xc || !xf) return set_error(P3D_ERR_ARG, "mg_restrict: bad args");
  if (prec == P3D_PREC_F64) return mg_restrict<double>(cnx, cny, cnz, ndof, (const double *)xf, (double *)xc, (cudaStream_t)stream);
  if (prec == P3D_PREC_F32) return mg_restrict<float>(cnx, cny, cnz, ndof, (const float *)xf, (float *)xc, (cudaStream_t)stream);
  return set_error(P3D_ERR_ARG, "mg_restrict: precision must be 64 or 32");
}
}
