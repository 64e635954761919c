// Vector kernels of the device-resident Stokes solver: grid-stride elementwise
// updates (fused where the Chebyshev and FGMRES recurrences allow), FP64
// reductions (two-phase, deterministic), Dirichlet masking by lattice face
// test, precision conversion, the per-element 4x4 Schur block apply and a
// dense matrix-vector product for the coarse-grid solve.
#include <cuda_runtime.h>

#include "p3d_internal.h"
#include "q2_tile.cuh"
#include "solver_internal.h"

namespace p3d {

static int vgrid(size_t n)
{
  size_t g = (n + 255) / 256;
  size_t cap = 148 * 8;
  if (g > cap) g = cap;
  return g < 1 ? 1 : (int)g;
}
// blocks of a multi-dot launch (per member): about 8 entries per thread, at
// most P3D_MDOT_BLOCKS.  Short vectors take few blocks, so that the last
// block's pass over the partials and the ticket traffic stay small.
static int mdot_blocks(size_t n)
{
  size_t g = (n + 2047) / 2048;
  if (g > P3D_MDOT_BLOCKS) g = P3D_MDOT_BLOCKS;
  return g < 1 ? 1 : (int)g;
}

#define GS_LOOP(i, n) for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

template <typename A, typename B> __global__ void k_convert(size_t n, const A *__restrict__ x, B *__restrict__ y)
{
  GS_LOOP(i, n) y[i] = (B)x[i];
}
template <typename T> __global__ void k_axpby(size_t n, T a, const T *__restrict__ x, T b, T *__restrict__ y)
{
  GS_LOOP(i, n) y[i] = a * x[i] + b * y[i];
}
template <typename T> __global__ void k_scale(size_t n, T a, T *__restrict__ y)
{
  GS_LOOP(i, n) y[i] *= a;
}
// z = dinv .* r   (dinv stored in FP64)
template <typename T> __global__ void k_jacobi(size_t n, const double *__restrict__ dinv, const T *__restrict__ r, T *__restrict__ z)
{
  GS_LOOP(i, n) z[i] = (T)(dinv[i] * (double)r[i]);
}
// Chebyshev start from x = 0: x = 0, r = b, d = dinv .* b / theta (one pass)
template <typename T>
__global__ void k_cheb_init0(size_t n, const double *__restrict__ dinv, const T *__restrict__ b, T inv_theta,
                             T *__restrict__ x, T *__restrict__ r, T *__restrict__ d)
{
  GS_LOOP(i, n)
  {
    const T bi = b[i];
    x[i] = (T)0;
    r[i] = bi;
    d[i] = (T)(dinv[i] * (double)bi) * inv_theta;
  }
}
// Chebyshev start from x: r = b - Ax, d = dinv .* r / theta (one pass)
template <typename T>
__global__ void k_cheb_init_res(size_t n, const double *__restrict__ dinv, const T *__restrict__ b, const T *__restrict__ Ax,
                                T inv_theta, T *__restrict__ r, T *__restrict__ d)
{
  GS_LOOP(i, n)
  {
    const T ri = b[i] - Ax[i];
    r[i] = ri;
    d[i] = (T)(dinv[i] * (double)ri) * inv_theta;
  }
}
// x += d ; r -= Ad ; d = c1 d + c2 dinv .* r   (one pass for the Chebyshev recurrence);
// last: the recurrence ends here, so the new d is added to x as well
template <typename T>
__global__ void k_cheb_step(size_t n, const double *__restrict__ dinv, T *__restrict__ x, T *__restrict__ r,
                            const T *__restrict__ Ad, T *__restrict__ d, T c1, T c2, int last)
{
  GS_LOOP(i, n)
  {
    T di = d[i];
    T ri = r[i] - Ad[i];
    T dn = c1 * di + c2 * (T)(dinv[i] * (double)ri);
    if (last) {
      x[i] += di + dn;
    } else {
      x[i] += di;
      r[i] = ri;
      d[i] = dn;
    }
  }
}
// r = b - Ax
template <typename T> __global__ void k_residual(size_t n, const T *__restrict__ b, const T *__restrict__ Ax, T *__restrict__ r)
{
  GS_LOOP(i, n) r[i] = b[i] - Ax[i];
}

// zero the Dirichlet dofs of a whole-mesh velocity vector (face test on the lattice)
template <typename T>
__global__ void k_mask(int nx, int ny, int nz, uint32_t dir, T *__restrict__ v)
{
  size_t nn = (size_t)nx * ny * nz;
  GS_LOOP(node, nn)
  {
    int i = node % nx, j = (node / nx) % ny, k = node / ((size_t)nx * ny);
    if (!(i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1)) continue;
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (is_dirichlet(dir, i, j, k, 0, 0, 0, nx - 1, ny - 1, nz - 1, c)) v[3 * node + c] = (T)0;
  }
}

// partial dot products  part[blk*KC + j] = sum_i V_j[i] w[i]   (FP64 accumulation),
// KC vectors per launch so that the accumulators stay in registers
template <typename T, int KC>
__global__ void k_mdot_partial(size_t n, const T *const *__restrict__ V, const T *__restrict__ w, double *__restrict__ part,
                               unsigned int *__restrict__ ticket, double *__restrict__ out, double *__restrict__ self_out)
{
  // self_out (optional): also w . w, the (KC+1)-th output
  constexpr int KS = KC + 1; // partials per block
  __shared__ double red[32][KS];
  __shared__ bool last;
  const bool self = self_out != nullptr;
  const int nout = KC + (self ? 1 : 0);
  const T *v[KC];
  double acc[KC], accs = 0.0;
#pragma unroll
  for (int j = 0; j < KC; j++) {
    v[j] = V[j];
    acc[j] = 0.0;
  }
  GS_LOOP(i, n)
  {
    double wi = (double)w[i];
#pragma unroll
    for (int j = 0; j < KC; j++) acc[j] += (double)v[j][i] * wi;
    if (self) accs += wi * wi;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < KS; j++) {
    if (j == KC && !self) break;
    double x = j < KC ? acc[j] : accs;
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp][j] = x;
  }
  __syncthreads();
  if (threadIdx.x < nout) {
    double x = 0.0;
    for (int q = 0; q < nw; q++) x += red[q][threadIdx.x];
    part[(size_t)blockIdx.x * KS + threadIdx.x] = x;
  }
  // the last block to finish sums the partials in block order (deterministic)
  // and re-arms the ticket for the next launch on the stream
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // one warp per output; with KC = 8 and the self product there are nine
  // outputs and only eight warps, so a warp may take a second one
  for (int t = warp; t < nout; t += nw) {
    double x = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) x += __ldcg(part + (size_t)b * KS + t);
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) {
      if (t < KC) out[t] = x;
      else *self_out = x;
    }
  }
  if (threadIdx.x == 0) *ticket = 0u;
}
// w += sign * sum_j h_j V_j   (h on device), KC vectors per launch
template <typename T, int KC>
__global__ void k_maxpy(size_t n, const double *__restrict__ h, const T *const *__restrict__ V, T *__restrict__ w, double sign)
{
  const T *v[KC];
  double c[KC];
#pragma unroll
  for (int j = 0; j < KC; j++) {
    v[j] = V[j];
    c[j] = sign * h[j];
  }
  GS_LOOP(i, n)
  {
    double s = (double)w[i];
#pragma unroll
    for (int j = 0; j < KC; j++) s += c[j] * (double)v[j][i];
    w[i] = (T)s;
  }
}

// Conjugate-gradient updates with the step lengths held on the device (so a
// fixed number of CG iterations can be captured in a CUDA graph):
//   alpha = num/den ; x += alpha p ; r -= alpha q (when update_r)
template <typename T>
__global__ void k_cg_xr(size_t n, const double *__restrict__ num, const double *__restrict__ den, T *__restrict__ x,
                        T *__restrict__ r, const T *__restrict__ p, const T *__restrict__ q, int update_r)
{
  const double d = *den, a0 = *num / d;
  const double a = (d > 0.0 && isfinite(a0)) ? a0 : 0.0; // breakdown: leave x, r unchanged
  GS_LOOP(i, n)
  {
    x[i] = (T)((double)x[i] + a * (double)p[i]);
    if (update_r) r[i] = (T)((double)r[i] - a * (double)q[i]);
  }
}
//   beta = num/den ; p = z + beta p
template <typename T>
__global__ void k_cg_p(size_t n, const double *__restrict__ num, const double *__restrict__ den, const T *__restrict__ z,
                       T *__restrict__ p)
{
  const double d = *den, b0 = *num / d;
  const double b = (d != 0.0 && isfinite(b0)) ? b0 : 0.0;
  GS_LOOP(i, n) p[i] = (T)((double)z[i] + b * (double)p[i]);
}

// dinv = 1/d; counts entries that are not positive and finite
__global__ void k_invert_diag(size_t n, const double *__restrict__ d, double *__restrict__ dinv, unsigned int *__restrict__ bad)
{
  unsigned nb = 0;
  GS_LOOP(i, n)
  {
    const double v = d[i];
    const bool ok = v > 0.0 && isfinite(v);
    dinv[i] = ok ? 1.0 / v : 1.0;
    nb += ok ? 0u : 1u;
  }
  if (nb) atomicAdd(bad, nb);
}

// y = blockdiag(B_e) x  with B_e 4x4 per element (Schur approximation inverse)
__global__ void k_block4(size_t nel, const double *__restrict__ B, const double *__restrict__ x, double *__restrict__ y, double alpha)
{
  GS_LOOP(e, nel)
  {
    const double *b = B + 16 * e;
    double x0 = x[4 * e], x1 = x[4 * e + 1], x2 = x[4 * e + 2], x3 = x[4 * e + 3];
    for (int r = 0; r < 4; r++) y[4 * e + r] = alpha * (b[4 * r] * x0 + b[4 * r + 1] * x1 + b[4 * r + 2] * x2 + b[4 * r + 3] * x3);
  }
}

// y = M x, M dense row-major n x n (coarse-grid inverse); one warp per row
__global__ void k_dense_mv(int n, const double *__restrict__ M, const double *__restrict__ x, double *__restrict__ y)
{
  int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int c = lane; c < n; c += 32) s += M[(size_t)row * n + c] * x[c];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}

// ------------------------------------------------------ grouped kernels ---
// The same recurrences over the K members of a group of same-shape solves in
// one launch (blockIdx.y = member).  Per-member pointers and scalars travel in
// the launch parameters (VGroup), so a captured graph replays them as they are.

template <typename T>
__global__ void kg_cheb_init0(const __grid_constant__ VGroup<T> G, size_t n)
{
  const int m = blockIdx.y;
  const double *dinv = G.dinv[m];
  const T *b = G.v[0][m];
  T *x = G.v[1][m], *r = G.v[2][m], *d = G.v[3][m];
  const T inv_theta = (T)G.s[0][m];
  GS_LOOP(i, n)
  {
    const T bi = b[i];
    x[i] = (T)0;
    r[i] = bi;
    d[i] = (T)(dinv[i] * (double)bi) * inv_theta;
  }
}
template <typename T>
__global__ void kg_cheb_init_res(const __grid_constant__ VGroup<T> G, size_t n)
{
  const int m = blockIdx.y;
  const double *dinv = G.dinv[m];
  const T *b = G.v[0][m], *Ax = G.v[1][m];
  T *r = G.v[2][m], *d = G.v[3][m];
  const T inv_theta = (T)G.s[0][m];
  GS_LOOP(i, n)
  {
    const T ri = b[i] - Ax[i];
    r[i] = ri;
    d[i] = (T)(dinv[i] * (double)ri) * inv_theta;
  }
}
template <typename T>
__global__ void kg_cheb_step(const __grid_constant__ VGroup<T> G, size_t n, int last)
{
  const int m = blockIdx.y;
  const double *dinv = G.dinv[m];
  T *x = G.v[0][m], *r = G.v[1][m], *d = G.v[3][m];
  const T *Ad = G.v[2][m];
  const T c1 = (T)G.s[0][m], c2 = (T)G.s[1][m];
  GS_LOOP(i, n)
  {
    T di = d[i];
    T ri = r[i] - Ad[i];
    T dn = c1 * di + c2 * (T)(dinv[i] * (double)ri);
    if (last) {
      x[i] += di + dn;
    } else {
      x[i] += di;
      r[i] = ri;
      d[i] = dn;
    }
  }
}
// y = a x + b y (y is not read when b == 0, so it may hold anything)
template <typename T>
__global__ void kg_axpby(const __grid_constant__ VGroup<T> G, size_t n)
{
  const int m = blockIdx.y;
  const T *x = G.v[0][m];
  T *y = G.v[1][m];
  const T a = (T)G.s[0][m], b = (T)G.s[1][m];
  if (b == (T)0) {
    GS_LOOP(i, n) y[i] = a * x[i];
  } else {
    GS_LOOP(i, n) y[i] = a * x[i] + b * y[i];
  }
}
// r = b - Ax
template <typename T>
__global__ void kg_residual(const __grid_constant__ VGroup<T> G, size_t n)
{
  const int m = blockIdx.y;
  const T *b = G.v[0][m], *Ax = G.v[1][m];
  T *r = G.v[2][m];
  GS_LOOP(i, n) r[i] = b[i] - Ax[i];
}
// precision conversion: v[1] = (B) v[0] (the roles hold raw pointers)
template <typename A, typename B>
__global__ void kg_convert(const __grid_constant__ VGroup<double> G, size_t n)
{
  const int m = blockIdx.y;
  const A *x = reinterpret_cast<const A *>(G.v[0][m]);
  B *y = reinterpret_cast<B *>(G.v[1][m]);
  GS_LOOP(i, n) y[i] = (B)x[i];
}
// y = blockdiag(B_e) x with 4x4 blocks (v[0] = B, v[1] = x, v[2] = y)
__global__ void kg_block4(const __grid_constant__ VGroup<double> G, size_t nel)
{
  const int m = blockIdx.y;
  const double *B = G.v[0][m], *x = G.v[1][m];
  double *y = G.v[2][m];
  GS_LOOP(e, nel)
  {
    const double *b = B + 16 * e;
    double x0 = x[4 * e], x1 = x[4 * e + 1], x2 = x[4 * e + 2], x3 = x[4 * e + 3];
    for (int r = 0; r < 4; r++) y[4 * e + r] = b[4 * r] * x0 + b[4 * r + 1] * x1 + b[4 * r + 2] * x2 + b[4 * r + 3] * x3;
  }
}
// y = M x, M dense n x n (v[0] = M, v[1] = x, v[2] = y); one warp per row
__global__ void kg_dense_mv(const __grid_constant__ VGroup<double> G, int n)
{
  const int m = blockIdx.y;
  const double *M = G.v[0][m], *x = G.v[1][m];
  double *y = G.v[2][m];
  int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int c = lane; c < n; c += 32) s += M[(size_t)row * n + c] * x[c];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}
// partial dot products of KC basis vectors with w, per member (its own
// partials buffer and ticket); the last block of a member finishes its sums
template <int KC>
__global__ void kg_mdot_partial(const __grid_constant__ MGroup G, size_t n, int j0)
{
  constexpr int KS = KC + 1;
  __shared__ double red[32][KS];
  __shared__ bool last;
  const int mem = blockIdx.y;
  const double *w = G.w[mem];
  double *part = G.part[mem];
  unsigned int *ticket = reinterpret_cast<unsigned int *>(part + (size_t)P3D_MDOT_BLOCKS * (P3D_MDOT_CHUNK + 1));
  double *out = G.out[mem] + j0, *self_out = j0 == 0 ? G.self_out[mem] : nullptr;
  const bool self = self_out != nullptr;
  const int nout = KC + (self ? 1 : 0);
  const double *v[KC];
  double acc[KC], accs = 0.0;
#pragma unroll
  for (int j = 0; j < KC; j++) {
    v[j] = G.V[mem][j0 + j];
    acc[j] = 0.0;
  }
  GS_LOOP(i, n)
  {
    double wi = w[i];
#pragma unroll
    for (int j = 0; j < KC; j++) acc[j] += v[j][i] * wi;
    if (self) accs += wi * wi;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < KS; j++) {
    if (j == KC && !self) break;
    double x = j < KC ? acc[j] : accs;
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp][j] = x;
  }
  __syncthreads();
  if (threadIdx.x < nout) {
    double x = 0.0;
    for (int q = 0; q < nw; q++) x += red[q][threadIdx.x];
    part[(size_t)blockIdx.x * KS + threadIdx.x] = x;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // one warp per output; with KC = 8 and the self product there are nine
  // outputs and only eight warps, so a warp may take a second one
  for (int t = warp; t < nout; t += nw) {
    double x = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) x += __ldcg(part + (size_t)b * KS + t);
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) {
      if (t < KC) out[t] = x;
      else *self_out = x;
    }
  }
  if (threadIdx.x == 0) *ticket = 0u;
}
// w += sign * sum_j h_j V_j per member (h on the device)
template <int KC>
__global__ void kg_maxpy(const __grid_constant__ MGroup G, size_t n, int j0, double sign)
{
  const int mem = blockIdx.y;
  double *w = G.w[mem];
  const double *v[KC];
  double c[KC];
#pragma unroll
  for (int j = 0; j < KC; j++) {
    v[j] = G.V[mem][j0 + j];
    c[j] = sign * G.out[mem][j0 + j];
  }
  GS_LOOP(i, n)
  {
    double s = w[i];
#pragma unroll
    for (int j = 0; j < KC; j++) s += c[j] * v[j][i];
    w[i] = s;
  }
}

template <typename T> void vg_cheb_init0(const VGroup<T> &G, int K, size_t n, cudaStream_t s)
{
  kg_cheb_init0<T><<<dim3(vgrid(n), K), 256, 0, s>>>(G, n);
  count_launch(1);
}
template <typename T> void vg_cheb_init_res(const VGroup<T> &G, int K, size_t n, cudaStream_t s)
{
  kg_cheb_init_res<T><<<dim3(vgrid(n), K), 256, 0, s>>>(G, n);
  count_launch(1);
}
template <typename T> void vg_cheb_step(const VGroup<T> &G, int K, size_t n, bool last, cudaStream_t s)
{
  kg_cheb_step<T><<<dim3(vgrid(n), K), 256, 0, s>>>(G, n, last ? 1 : 0);
  count_launch(1);
}
template <typename T> void vg_axpby(const VGroup<T> &G, int K, size_t n, cudaStream_t s)
{
  kg_axpby<T><<<dim3(vgrid(n), K), 256, 0, s>>>(G, n);
  count_launch(1);
}
template <typename T> void vg_residual(const VGroup<T> &G, int K, size_t n, cudaStream_t s)
{
  kg_residual<T><<<dim3(vgrid(n), K), 256, 0, s>>>(G, n);
  count_launch(1);
}
template <typename A, typename B> void vg_convert(const VGroup<double> &G, int K, size_t n, cudaStream_t s)
{
  kg_convert<A, B><<<dim3(vgrid(n), K), 256, 0, s>>>(G, n);
  count_launch(1);
}
void vg_block4(const VGroup<double> &G, int K, size_t nel, cudaStream_t s)
{
  kg_block4<<<dim3(vgrid(nel), K), 256, 0, s>>>(G, nel);
  count_launch(1);
}
void vg_dense_mv(const VGroup<double> &G, int K, int n, cudaStream_t s)
{
  kg_dense_mv<<<dim3((n + 7) / 8, K), 256, 0, s>>>(G, n);
  count_launch(1);
}
void vg_mdot(const MGroup &G, int K, size_t n, int k, cudaStream_t s)
{
  for (int j0 = 0; j0 < k; j0 += P3D_MDOT_CHUNK) {
    const int kc = k - j0 < P3D_MDOT_CHUNK ? k - j0 : P3D_MDOT_CHUNK;
    const dim3 grid(mdot_blocks(n), K);
    switch (kc) {
    case 1: kg_mdot_partial<1><<<grid, 256, 0, s>>>(G, n, j0); break;
    case 2: kg_mdot_partial<2><<<grid, 256, 0, s>>>(G, n, j0); break;
    case 3: kg_mdot_partial<3><<<grid, 256, 0, s>>>(G, n, j0); break;
    case 4: kg_mdot_partial<4><<<grid, 256, 0, s>>>(G, n, j0); break;
    case 5: kg_mdot_partial<5><<<grid, 256, 0, s>>>(G, n, j0); break;
    case 6: kg_mdot_partial<6><<<grid, 256, 0, s>>>(G, n, j0); break;
    case 7: kg_mdot_partial<7><<<grid, 256, 0, s>>>(G, n, j0); break;
    default: kg_mdot_partial<8><<<grid, 256, 0, s>>>(G, n, j0); break;
    }
    count_launch(1);
  }
}
void vg_maxpy(const MGroup &G, int K, size_t n, int k, double sign, cudaStream_t s)
{
  for (int j0 = 0; j0 < k; j0 += P3D_MDOT_CHUNK) {
    const int kc = k - j0 < P3D_MDOT_CHUNK ? k - j0 : P3D_MDOT_CHUNK;
    const dim3 grid(vgrid(n), K);
    switch (kc) {
    case 1: kg_maxpy<1><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    case 2: kg_maxpy<2><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    case 3: kg_maxpy<3><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    case 4: kg_maxpy<4><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    case 5: kg_maxpy<5><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    case 6: kg_maxpy<6><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    case 7: kg_maxpy<7><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    default: kg_maxpy<8><<<grid, 256, 0, s>>>(G, n, j0, sign); break;
    }
    count_launch(1);
  }
}
template void vg_cheb_init0<double>(const VGroup<double> &, int, size_t, cudaStream_t);
template void vg_cheb_init0<float>(const VGroup<float> &, int, size_t, cudaStream_t);
template void vg_cheb_init_res<double>(const VGroup<double> &, int, size_t, cudaStream_t);
template void vg_cheb_init_res<float>(const VGroup<float> &, int, size_t, cudaStream_t);
template void vg_cheb_step<double>(const VGroup<double> &, int, size_t, bool, cudaStream_t);
template void vg_cheb_step<float>(const VGroup<float> &, int, size_t, bool, cudaStream_t);
template void vg_axpby<double>(const VGroup<double> &, int, size_t, cudaStream_t);
template void vg_axpby<float>(const VGroup<float> &, int, size_t, cudaStream_t);
template void vg_residual<double>(const VGroup<double> &, int, size_t, cudaStream_t);
template void vg_convert<double, float>(const VGroup<double> &, int, size_t, cudaStream_t);
template void vg_convert<float, double>(const VGroup<double> &, int, size_t, cudaStream_t);

// ------------------------------------------------------------ host API ---
template <typename A, typename B> void v_convert(size_t n, const A *x, B *y, cudaStream_t s)
{
  k_convert<<<vgrid(n), 256, 0, s>>>(n, x, y);
  count_launch(1);
}
template <typename T> void v_axpby(size_t n, T a, const T *x, T b, T *y, cudaStream_t s)
{
  k_axpby<<<vgrid(n), 256, 0, s>>>(n, a, x, b, y);
  count_launch(1);
}
template <typename T> void v_scale(size_t n, T a, T *y, cudaStream_t s)
{
  k_scale<<<vgrid(n), 256, 0, s>>>(n, a, y);
  count_launch(1);
}
template <typename T> void v_jacobi(size_t n, const double *dinv, const T *r, T *z, cudaStream_t s)
{
  k_jacobi<<<vgrid(n), 256, 0, s>>>(n, dinv, r, z);
  count_launch(1);
}
template <typename T>
void v_cheb_init0(size_t n, const double *dinv, const T *b, T inv_theta, T *x, T *r, T *d, cudaStream_t s)
{
  k_cheb_init0<<<vgrid(n), 256, 0, s>>>(n, dinv, b, inv_theta, x, r, d);
  count_launch(1);
}
template <typename T>
void v_cheb_init_res(size_t n, const double *dinv, const T *b, const T *Ax, T inv_theta, T *r, T *d, cudaStream_t s)
{
  k_cheb_init_res<<<vgrid(n), 256, 0, s>>>(n, dinv, b, Ax, inv_theta, r, d);
  count_launch(1);
}
template <typename T>
void v_cheb_step(size_t n, const double *dinv, T *x, T *r, const T *Ad, T *d, T c1, T c2, bool last, cudaStream_t s)
{
  k_cheb_step<<<vgrid(n), 256, 0, s>>>(n, dinv, x, r, Ad, d, c1, c2, last ? 1 : 0);
  count_launch(1);
}
template <typename T> void v_residual(size_t n, const T *b, const T *Ax, T *r, cudaStream_t s)
{
  k_residual<<<vgrid(n), 256, 0, s>>>(n, b, Ax, r);
  count_launch(1);
}
template <typename T> void v_mask(int nx, int ny, int nz, uint32_t dir, T *v, cudaStream_t s)
{
  if (!dir) return;
  k_mask<<<vgrid((size_t)nx * ny * nz), 256, 0, s>>>(nx, ny, nz, dir, v);
  count_launch(1);
}
template <typename T, int KC>
static void mdot_chunk(size_t n, const T *const *V_dev, const T *w, double *part, double *out, double *self_out,
                       cudaStream_t s)
{
  // part holds P3D_MDOT_BLOCKS * (P3D_MDOT_CHUNK + 1) partials, then the ticket counter
  unsigned int *ticket = reinterpret_cast<unsigned int *>(part + (size_t)P3D_MDOT_BLOCKS * (P3D_MDOT_CHUNK + 1));
  k_mdot_partial<T, KC><<<mdot_blocks(n), 256, 0, s>>>(n, V_dev, w, part, ticket, out, self_out);
  count_launch(1);
}
template <typename T>
void v_mdot(size_t n, int k, const T *const *V_dev, const T *w, double *part, double *out_dev, cudaStream_t s,
            double *self_out)
{
  for (int j0 = 0; j0 < k; j0 += P3D_MDOT_CHUNK) {
    const int kc = k - j0 < P3D_MDOT_CHUNK ? k - j0 : P3D_MDOT_CHUNK;
    const T *const *V = V_dev + j0;
    double *o = out_dev + j0, *so = j0 == 0 ? self_out : nullptr;
    switch (kc) {
    case 1: mdot_chunk<T, 1>(n, V, w, part, o, so, s); break;
    case 2: mdot_chunk<T, 2>(n, V, w, part, o, so, s); break;
    case 3: mdot_chunk<T, 3>(n, V, w, part, o, so, s); break;
    case 4: mdot_chunk<T, 4>(n, V, w, part, o, so, s); break;
    case 5: mdot_chunk<T, 5>(n, V, w, part, o, so, s); break;
    case 6: mdot_chunk<T, 6>(n, V, w, part, o, so, s); break;
    case 7: mdot_chunk<T, 7>(n, V, w, part, o, so, s); break;
    default: mdot_chunk<T, 8>(n, V, w, part, o, so, s); break;
    }
  }
}
template <typename T> void v_maxpy(size_t n, int k, const double *h, const T *const *V_dev, T *w, double sign, cudaStream_t s)
{
  for (int j0 = 0; j0 < k; j0 += P3D_MDOT_CHUNK) {
    const int kc = k - j0 < P3D_MDOT_CHUNK ? k - j0 : P3D_MDOT_CHUNK;
    const double *hh = h + j0;
    const T *const *V = V_dev + j0;
    const int g = vgrid(n);
    switch (kc) {
    case 1: k_maxpy<T, 1><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    case 2: k_maxpy<T, 2><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    case 3: k_maxpy<T, 3><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    case 4: k_maxpy<T, 4><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    case 5: k_maxpy<T, 5><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    case 6: k_maxpy<T, 6><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    case 7: k_maxpy<T, 7><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    default: k_maxpy<T, 8><<<g, 256, 0, s>>>(n, hh, V, w, sign); break;
    }
    count_launch(1);
  }
}
template <typename T>
void v_cg_xr(size_t n, const double *num, const double *den, T *x, T *r, const T *p, const T *q, bool update_r, cudaStream_t s)
{
  k_cg_xr<<<vgrid(n), 256, 0, s>>>(n, num, den, x, r, p, q, update_r ? 1 : 0);
  count_launch(1);
}
template <typename T> void v_cg_p(size_t n, const double *num, const double *den, const T *z, T *p, cudaStream_t s)
{
  k_cg_p<<<vgrid(n), 256, 0, s>>>(n, num, den, z, p);
  count_launch(1);
}
void v_invert_diag(size_t n, const double *d, double *dinv, unsigned int *bad, cudaStream_t s)
{
  k_invert_diag<<<vgrid(n), 256, 0, s>>>(n, d, dinv, bad);
  count_launch(1);
}
void v_block4(size_t nel, const double *B, const double *x, double *y, double alpha, cudaStream_t s)
{
  k_block4<<<vgrid(nel), 256, 0, s>>>(nel, B, x, y, alpha);
  count_launch(1);
}
void v_dense_mv(int n, const double *M, const double *x, double *y, cudaStream_t s)
{
  k_dense_mv<<<(n + 7) / 8, 256, 0, s>>>(n, M, x, y);
  count_launch(1);
}

template void v_convert<double, float>(size_t, const double *, float *, cudaStream_t);
template void v_convert<float, double>(size_t, const float *, double *, cudaStream_t);
#define P3D_INST(T)                                                                                                    \
  template void v_axpby<T>(size_t, T, const T *, T, T *, cudaStream_t);                                                \
  template void v_scale<T>(size_t, T, T *, cudaStream_t);                                                              \
  template void v_jacobi<T>(size_t, const double *, const T *, T *, cudaStream_t);                                     \
  template void v_cheb_step<T>(size_t, const double *, T *, T *, const T *, T *, T, T, bool, cudaStream_t);            \
  template void v_cheb_init0<T>(size_t, const double *, const T *, T, T *, T *, T *, cudaStream_t);                   \
  template void v_cheb_init_res<T>(size_t, const double *, const T *, const T *, T, T *, T *, cudaStream_t);          \
  template void v_residual<T>(size_t, const T *, const T *, T *, cudaStream_t);                                        \
  template void v_mask<T>(int, int, int, uint32_t, T *, cudaStream_t);                                                 \
  template void v_mdot<T>(size_t, int, const T *const *, const T *, double *, double *, cudaStream_t, double *);       \
  template void v_maxpy<T>(size_t, int, const double *, const T *const *, T *, double, cudaStream_t);              \
  template void v_cg_xr<T>(size_t, const double *, const double *, T *, T *, const T *, const T *, bool, cudaStream_t); \
  template void v_cg_p<T>(size_t, const double *, const double *, const T *, T *, cudaStream_t);
P3D_INST(double)
P3D_INST(float)

} // namespace p3d
