// Operator objects and the C-ABI of libp3d_b200.so (see include/p3d_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "p3d_b200.h"
#include "p3d_internal.h"
#include "solver_internal.h"
#include "stokes_kernels.cuh"

namespace p3d {

// ------------------------------------------------------------- errors ----
static thread_local char g_err[512] = "";
std::atomic<long long> g_launches{0};

int set_error(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}
int cuda_check(cudaError_t e, const char *what)
{
  if (e == cudaSuccess) return P3D_OK;
  return set_error(P3D_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
void count_launch(int n) { g_launches += n; }
int order_after_caller() { return cuda_check(cudaDeviceSynchronize(), "wait for the caller's device work"); }

static std::once_flag g_tables_once;
static int upload_tables()
{
  static int rc = 0;
  std::call_once(g_tables_once, [] {
    double B[3][3], D[3][3];
    const double s = std::sqrt(0.6), xs[3] = {-s, 0.0, s};
    for (int q = 0; q < 3; q++) {
      double x = xs[q];
      B[q][0] = 0.5 * (x * x - x); B[q][1] = 1.0 - x * x; B[q][2] = 0.5 * (x * x + x);
      D[q][0] = x - 0.5; D[q][1] = -2.0 * x; D[q][2] = x + 0.5;
    }
    rc = cuda_check(cudaMemcpyToSymbol(c_B, B, sizeof B), "cudaMemcpyToSymbol(B)");
    if (!rc) rc = cuda_check(cudaMemcpyToSymbol(c_D, D, sizeof D), "cudaMemcpyToSymbol(D)");
  });
  return rc;
}

// brick counts for a layer height
static void bricks(const p3d_mesh_desc &m, int nw, int &ntx, int &nty, int &ntz)
{
  ntx = (m.mx + TX - 1) / TX;
  nty = (m.my + TY - 1) / TY;
  ntz = (m.mz + nw - 1) / nw;
}

template <typename T> static TileArgs<T> tile_args(const p3d_op *op, int nw)
{
  TileArgs<T> a;
  memset(&a, 0, sizeof a);
  a.mx = op->m.mx; a.my = op->m.my; a.mz = op->m.mz;
  a.gx = op->m.gx; a.gy = op->m.gy; a.gz = op->m.gz;
  a.ox = op->m.ox; a.oy = op->m.oy; a.oz = op->m.oz;
  bricks(op->m, nw, a.ntx, a.nty, a.ntz);
  uint32_t dir = 0;
  for (int f = 0; f < 6; f++)
    if (op->m.global_faces & (1u << f)) dir |= op->m.dirichlet & (7u << (3 * f));
  a.dir = dir;
  a.bc = op->bc;
  a.coords = reinterpret_cast<const T *>(op->coords);
  return a;
}

template <typename K> static int prep_kernel(K kernel, size_t smem)
{
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_check(e, "cudaFuncSetAttribute");
  }
  return P3D_OK;
}

template <typename T> static int nbricks_t(const TileArgs<T> &a) { return a.ntx * a.nty * a.ntz; }

// ------------------------------------------------------------- launches ---
// bricks of the layer range [tzb, tze) (tze < 0: all layers); sets a.brick0
template <typename T> static int brick_range(TileArgs<T> &a, int tzb, int tze)
{
  if (tze < 0 || tze > a.ntz) tze = a.ntz;
  if (tzb < 0) tzb = 0;
  a.brick0 = tzb * a.ntx * a.nty;
  return tze > tzb ? (tze - tzb) * a.ntx * a.nty : 0;
}

int a11_brick_height(const p3d_op *op) { return op->geom == P3D_GEOM_AFFINE ? NW_AFF : NW_GEN; }

// per-element constant Jacobian: A11 on affine meshes (or the low-order
// operator), and A12 / A21 / the fused operator where every element was tested affine
template <typename T, bool DA11, bool DA12, bool DA21>
static int launch_affine(p3d_op *op, const T *u, const T *p, T *yu, T *yp, cudaStream_t st, bool overwrite, int tzb,
                         int tze)
{
  TileArgs<T> a = tile_args<T>(op, NW_AFF);
  a.x = u; a.y = yu; a.p = p; a.yp = yp;
  a.kdat = reinterpret_cast<const T *>(op->kaff);
  a.kgq = reinterpret_cast<const T *>(op->kpre);
  a.overwrite = overwrite ? 1 : 0;
  auto kern = stokes_affine_kernel<T, NW_AFF, DA11, DA12, DA21>;
  size_t smem = AffineSmem<T, NW_AFF, DA11, DA12, DA21>::BYTES;
  int rc = prep_kernel(kern, smem);
  if (rc) return rc;
  const int nb = brick_range(a, tzb, tze);
  if (nb == 0) return P3D_OK;
  kern<<<nb, 32 * NW_AFF, smem, st>>>(a);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "affine launch");
}

template <typename T> int launch_a11(p3d_op *op, const T *x, T *y, cudaStream_t st, bool overwrite, int tzb, int tze)
{
  if (op->geom == P3D_GEOM_AFFINE) return launch_affine<T, true, false, false>(op, x, nullptr, y, nullptr, st, overwrite, tzb, tze);
  return launch_general<T, true, false, false>(op, x, nullptr, y, nullptr, st, overwrite, tzb, tze);
}

template <typename T, bool DA11, bool DA12, bool DA21>
int launch_general(p3d_op *op, const T *u, const T *p, T *yu, T *yp, cudaStream_t st, bool overwrite, int tzb, int tze)
{
  if (op->geom == P3D_GEOM_AFFINE && (op->aff_exact || !(DA12 || DA21)))
    return launch_affine<T, DA11, DA12, DA21>(op, u, p, yu, yp, st, overwrite, tzb, tze);
  TileArgs<T> a = tile_args<T>(op, NW_GEN);
  a.x = u; a.y = yu; a.p = p; a.yp = yp; a.kdat = reinterpret_cast<const T *>(op->kgen);
  a.kgq = reinterpret_cast<const T *>(op->kgq);
  a.overwrite = overwrite ? 1 : 0;
  // FP64: Jacobian columns exchanged by warp shuffles; FP32: per-element geometry table
  auto kern = sizeof(T) == 8 ? stokes_general_kernel<T, NW_GEN, DA11, DA12, DA21>
                             : stokes_general_tab_kernel<T, NW_GEN, DA11, DA12, DA21>;
  size_t smem = sizeof(T) == 8 ? GeneralSmem<T, NW_GEN, DA11, DA12, DA21>::BYTES
                               : GeneralTabSmem<T, NW_GEN, DA11, DA12, DA21>::BYTES;
  int rc = prep_kernel(kern, smem);
  if (rc) return rc;
  const int nb = brick_range(a, tzb, tze);
  if (nb == 0) return P3D_OK;
  kern<<<nb, 32 * NW_GEN, smem, st>>>(a);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "stokes launch");
}

// ----------------------------------------------------- grouped launches ---
// The operators of K resident problems of one mesh shape (and precision,
// geometry path and boundary mode) in ONE launch: grid (bricks, K), the
// member's tile arguments passed in the launch parameters (TileGroup).
static bool same_shape_ops(p3d_op *const *ops, int K)
{
  const p3d_mesh_desc &m = ops[0]->m;
  for (int k = 1; k < K; k++) {
    const p3d_op *o = ops[k];
    if (!o || !o->have_coef || o->prec != ops[0]->prec || o->geom != ops[0]->geom || o->bc != ops[0]->bc ||
        o->aff_exact != ops[0]->aff_exact || o->device != ops[0]->device || o->m.mx != m.mx || o->m.my != m.my ||
        o->m.mz != m.mz || o->m.gx != m.gx || o->m.gy != m.gy || o->m.gz != m.gz || o->m.ox != m.ox ||
        o->m.oy != m.oy || o->m.oz != m.oz || o->m.dirichlet != m.dirichlet || o->m.global_faces != m.global_faces)
      return false;
  }
  return true;
}

template <typename T, bool DA11, bool DA12, bool DA21>
int launch_group(p3d_op *const *ops, int K, const T *const *u, const T *const *p, T *const *yu, T *const *yp,
                 cudaStream_t st, bool overwrite)
{
  if (K < 1 || K > P3D_GROUP_MAX) return set_error(P3D_ERR_ARG, "grouped launch: %d members (1..%d)", K, P3D_GROUP_MAX);
  if (!ops[0] || !ops[0]->have_coef) return set_error(P3D_ERR_STATE, "grouped launch: operator not set up");
  if (!same_shape_ops(ops, K)) return set_error(P3D_ERR_ARG, "grouped launch: members differ in shape, path or mode");
  p3d_op *op0 = ops[0];
  const bool affine = op0->geom == P3D_GEOM_AFFINE && (op0->aff_exact || !(DA12 || DA21));
  const int nw = affine ? NW_AFF : NW_GEN;
  TileGroup<T> G;
  memset(&G, 0, sizeof G);
  for (int k = 0; k < K; k++) {
    TileArgs<T> a = tile_args<T>(ops[k], nw);
    a.x = u ? u[k] : nullptr; a.y = yu ? yu[k] : nullptr; a.p = p ? p[k] : nullptr; a.yp = yp ? yp[k] : nullptr;
    a.kdat = reinterpret_cast<const T *>(affine ? ops[k]->kaff : ops[k]->kgen);
    a.kgq = reinterpret_cast<const T *>(affine ? ops[k]->kpre : ops[k]->kgq);
    a.overwrite = overwrite ? 1 : 0;
    a.brick0 = 0;
    G.a[k] = a;
  }
  const int nb = G.a[0].ntx * G.a[0].nty * G.a[0].ntz;
  if (nb == 0) return P3D_OK;
  void (*kern)(const TileGroup<T>) = nullptr;
  size_t smem = 0;
  if (affine) {
    kern = stokes_affine_kernel_group<T, NW_AFF, DA11, DA12, DA21>;
    smem = AffineSmem<T, NW_AFF, DA11, DA12, DA21>::BYTES;
  } else if (sizeof(T) == 8) {
    kern = stokes_general_kernel_group<T, NW_GEN, DA11, DA12, DA21>;
    smem = GeneralSmem<T, NW_GEN, DA11, DA12, DA21>::BYTES;
  } else {
    kern = stokes_general_tab_kernel_group<T, NW_GEN, DA11, DA12, DA21>;
    smem = GeneralTabSmem<T, NW_GEN, DA11, DA12, DA21>::BYTES;
  }
  int rc = prep_kernel(kern, smem);
  if (rc) return rc;
  kern<<<dim3(nb, K), 32 * nw, smem, st>>>(G);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "grouped launch");
}

// zero K vectors of n elements in one launch (blockIdx.y = member)
struct PtrGroup {
  void *p[P3D_GROUP_MAX];
};
__global__ void zero_group_kernel(const __grid_constant__ PtrGroup P, size_t n_words)
{
  uint32_t *v = reinterpret_cast<uint32_t *>(P.p[blockIdx.y]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_words; i += (size_t)gridDim.x * blockDim.x) v[i] = 0u;
}
int zero_group(void *const *v, int K, size_t bytes, cudaStream_t st)
{
  if (K < 1 || K > P3D_GROUP_MAX || bytes % 4) return set_error(P3D_ERR_ARG, "zero_group: bad arguments");
  PtrGroup P;
  memset(&P, 0, sizeof P);
  for (int k = 0; k < K; k++) P.p[k] = v[k];
  const size_t words = bytes / 4;
  size_t g = (words + 255) / 256;
  if (g > 148 * 4) g = 148 * 4;
  if (g < 1) g = 1;
  zero_group_kernel<<<dim3((unsigned)g, K), 256, 0, st>>>(P, words);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "zero_group");
}

template int launch_group<double, true, false, false>(p3d_op *const *, int, const double *const *, const double *const *,
                                                     double *const *, double *const *, cudaStream_t, bool);
template int launch_group<float, true, false, false>(p3d_op *const *, int, const float *const *, const float *const *,
                                                    float *const *, float *const *, cudaStream_t, bool);
template int launch_group<double, true, true, true>(p3d_op *const *, int, const double *const *, const double *const *,
                                                   double *const *, double *const *, cudaStream_t, bool);
template int launch_group<double, false, true, false>(p3d_op *const *, int, const double *const *, const double *const *,
                                                     double *const *, double *const *, cudaStream_t, bool);

template <typename T> int launch_diag(p3d_op *op, T *d, cudaStream_t st)
{
  TileArgs<T> a = tile_args<T>(op, NW_GEN);
  a.y = d; a.kdat = reinterpret_cast<const T *>(op->kgen); a.diag = 1;
  auto kern = diag_general_kernel<T, NW_GEN>;
  size_t smem = DiagSmem<T, NW_GEN>::BYTES;
  int rc = prep_kernel(kern, smem);
  if (rc) return rc;
  if (nbricks_t(a) == 0) return P3D_OK;
  kern<<<nbricks_t(a), 32 * NW_GEN, smem, st>>>(a);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "diag launch");
}

template int launch_a11<double>(p3d_op *, const double *, double *, cudaStream_t, bool, int, int);
template int launch_a11<float>(p3d_op *, const float *, float *, cudaStream_t, bool, int, int);
template int launch_diag<double>(p3d_op *, double *, cudaStream_t);
template int launch_diag<float>(p3d_op *, float *, cudaStream_t);
template int launch_general<double, true, true, true>(p3d_op *, const double *, const double *, double *, double *, cudaStream_t, bool, int, int);
template int launch_general<float, true, true, true>(p3d_op *, const float *, const float *, float *, float *, cudaStream_t, bool, int, int);
template int launch_general<double, false, true, false>(p3d_op *, const double *, const double *, double *, double *, cudaStream_t, bool, int, int);
template int launch_general<double, false, false, true>(p3d_op *, const double *, const double *, double *, double *, cudaStream_t, bool, int, int);
template int launch_general<float, false, true, false>(p3d_op *, const float *, const float *, float *, float *, cudaStream_t, bool, int, int);
template int launch_general<float, false, false, true>(p3d_op *, const float *, const float *, float *, float *, cudaStream_t, bool, int, int);

// --------------------------------------------------------------- setup ---
static void free_dev(void *&p)
{
  if (p) cudaFree(p);
  p = nullptr;
}

// failure injection: allocations left before every device allocation fails (< 0: off)
static std::atomic<long long> g_alloc_budget{-1};
static std::atomic<int> g_alloc_poison{-1}; // fill byte of new allocations, -1: none

int dev_alloc(void **p, size_t bytes, const char *what)
{
  *p = nullptr;
  if (bytes == 0) bytes = 16;
  for (long long b = g_alloc_budget.load(); b >= 0;) {
    if (b == 0) return set_error(P3D_ERR_NOMEM, "cudaMalloc(%zu) for %s: failure injected", bytes, what);
    if (g_alloc_budget.compare_exchange_weak(b, b - 1)) break;
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(P3D_ERR_NOMEM, "cudaMalloc(%zu) for %s: %s", bytes, what, cudaGetErrorString(e));
  }
  const int fill = g_alloc_poison.load();
  if (fill >= 0) {
    e = cudaMemset(*p, fill, bytes);
    if (e != cudaSuccess) {
      cudaFree(*p);
      *p = nullptr;
      return set_error(P3D_ERR_CUDA, "poisoning %s: %s", what, cudaGetErrorString(e));
    }
  }
  return P3D_OK;
}

template <typename T>
__global__ void convert_kernel(size_t n, const double *__restrict__ src, T *__restrict__ dst)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (T)src[i];
}

static int grid_for(size_t n, int block = 256)
{
  size_t g = (n + block - 1) / block;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

// coords/eta are device FP64 arrays
int op_setup_device(p3d_op *op, const double *coords, const double *eta, int geom_mode)
{
  const p3d_mesh_desc &m = op->m;
  size_t nn = (size_t)m.gx * m.gy * m.gz, nel = (size_t)m.mx * m.my * m.mz;
  size_t es = op->prec == P3D_PREC_F64 ? 8 : 4;
  int rc;
  cudaStream_t st = op->stream;
  // coordinates in operator precision
  if (!op->coords && (rc = dev_alloc(&op->coords, 3 * nn * es, "coords"))) return rc;
  if (op->prec == P3D_PREC_F64)
    rc = cuda_check(cudaMemcpyAsync(op->coords, coords, 3 * nn * 8, cudaMemcpyDeviceToDevice, st), "copy coords");
  else {
    convert_kernel<float><<<grid_for(3 * nn), 256, 0, st>>>(3 * nn, coords, (float *)op->coords);
    count_launch(1);
    rc = cuda_check(cudaGetLastError(), "convert coords");
  }
  if (rc) return rc;
  // general-path eta in brick order
  int ntx, nty, ntz;
  bricks(m, NW_GEN, ntx, nty, ntz);
  size_t ng = (size_t)ntx * nty * ntz * Brick<NW_GEN>::NE * 27;
  // buffers keep their size for the mesh: a re-setup (new coefficients) allocates and frees nothing
  if (!op->kgen && (rc = dev_alloc(&op->kgen, ng * es, "eta (brick order)"))) return rc;
  if (op->prec == P3D_PREC_F64)
    pack_eta_kernel<double, NW_GEN><<<grid_for(ng), 256, 0, st>>>(m.mx, m.my, m.mz, ntx, nty, ntz, eta, (double *)op->kgen);
  else
    pack_eta_kernel<float, NW_GEN><<<grid_for(ng), 256, 0, st>>>(m.mx, m.my, m.mz, ntx, nty, ntz, eta, (float *)op->kgen);
  count_launch(1);
  if ((rc = cuda_check(cudaGetLastError(), "pack eta"))) return rc;
  {
    const size_t ngq = (size_t)ntx * nty * ntz * Brick<NW_GEN>::NE;
    if (!op->kgq && (rc = dev_alloc(&op->kgq, ngq * GQC * es, "gauss-point coordinates"))) return rc;
    if (op->prec == P3D_PREC_F64)
      pack_gauss_coords_kernel<double, NW_GEN><<<grid_for(ngq), 128, 0, st>>>(m.mx, m.my, m.mz, m.gx, m.gy, m.ox, m.oy, m.oz,
                                                                             ntx, nty, ntz, coords, (double *)op->kgq);
    else
      pack_gauss_coords_kernel<float, NW_GEN><<<grid_for(ngq), 128, 0, st>>>(m.mx, m.my, m.mz, m.gx, m.gy, m.ox, m.oy, m.oz,
                                                                            ntx, nty, ntz, coords, (float *)op->kgq);
    count_launch(1);
    if ((rc = cuda_check(cudaGetLastError(), "pack gauss coords"))) return rc;
  }
  // affinity
  int mode = geom_mode;
  if (mode == P3D_GEOM_AUTO) {
    unsigned long long hbad = 0;
    if (!op->flag && (rc = dev_alloc((void **)&op->flag, sizeof *op->flag, "affine flag"))) return rc;
    unsigned long long *bad = op->flag;
    cudaMemsetAsync(bad, 0, sizeof *bad, st);
    affine_check_kernel<<<grid_for(nel), 256, 0, st>>>(m.mx, m.my, m.mz, m.gx, m.gy, m.ox, m.oy, m.oz, coords, 1e-13, bad);
    count_launch(1);
    rc = cuda_check(cudaMemcpyAsync(&hbad, bad, sizeof hbad, cudaMemcpyDeviceToHost, st), "affine flag");
    if (!rc) rc = cuda_check(cudaStreamSynchronize(st), "affine sync");
    if (rc) return rc;
    mode = (hbad == 0 && nel > 0) ? P3D_GEOM_AFFINE : P3D_GEOM_GENERAL;
  }
  // the affine A12 / A21 kernels need every element affine (a forced low-order
  // A11 on a deformed mesh keeps the exact general ones)
  op->aff_exact = geom_mode == P3D_GEOM_AUTO && mode == P3D_GEOM_AFFINE;
  if (mode == P3D_GEOM_AFFINE) {
    bricks(m, NW_AFF, ntx, nty, ntz);
    size_t na = (size_t)ntx * nty * ntz * Brick<NW_AFF>::NE;
    if (!op->kaff && (rc = dev_alloc(&op->kaff, na * KAFF * es, "affine geometry"))) return rc;
    if (op->aff_exact && !op->kpre && (rc = dev_alloc(&op->kpre, na * KPRE * es, "affine pressure basis"))) return rc;
    void *pre = op->aff_exact ? op->kpre : nullptr;
    if (op->prec == P3D_PREC_F64)
      pack_affine_kernel<double, NW_AFF><<<grid_for(na), 256, 0, st>>>(m.mx, m.my, m.mz, m.gx, m.gy, m.ox, m.oy, m.oz,
                                                                      ntx, nty, ntz, coords, eta, (double *)op->kaff,
                                                                      (double *)pre);
    else
      pack_affine_kernel<float, NW_AFF><<<grid_for(na), 256, 0, st>>>(m.mx, m.my, m.mz, m.gx, m.gy, m.ox, m.oy, m.oz,
                                                                     ntx, nty, ntz, coords, eta, (float *)op->kaff,
                                                                     (float *)pre);
    count_launch(1);
    if ((rc = cuda_check(cudaGetLastError(), "pack affine"))) return rc;
  }
  op->geom = mode;
  op->have_coef = true;
  return cuda_check(cudaStreamSynchronize(st), "setup sync");
}

// Dirichlet values on the lattice of an operator.  mode 0: out = u with the
// Dirichlet dofs replaced by phi (0 without phi) (BCListInsertLocal,
// src/dmda_bcs.c:409-); mode 1: out_k = u_k - phi_k on the Dirichlet dofs only
// (BCListResidualDirichlet with scale 1).
__global__ void dirichlet_values_kernel(int gx, int gy, int gz, int ox, int oy, int oz, int ex, int ey, int ez, uint32_t dir,
                                        const double *__restrict__ u, const double *__restrict__ phi, double *__restrict__ out,
                                        int mode)
{
  const size_t nn = (size_t)gx * gy * gz;
  for (size_t node = blockIdx.x * (size_t)blockDim.x + threadIdx.x; node < nn; node += (size_t)gridDim.x * blockDim.x) {
    const int i = node % gx, j = (node / gx) % gy, k = node / ((size_t)gx * gy);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const size_t idx = 3 * node + c;
      const bool d = is_dirichlet(dir, i, j, k, ox, oy, oz, ex, ey, ez, c);
      if (mode == 0) out[idx] = d ? (phi ? phi[idx] : 0.0) : u[idx];
      else if (d) out[idx] = u[idx] - (phi ? phi[idx] : 0.0);
    }
  }
}

} // namespace p3d

using namespace p3d;

// ============================================================== C ABI ====
extern "C" {

const char *p3d_last_error(void) { return g_err; }
int64_t p3d_kernel_launch_count(void) { return (int64_t)g_launches.load(); }
const char *p3d_version(void) { return "p3d_b200 0.1 (sm_100a)"; }
int p3d_debug_fail_allocations_after(int64_t after)
{
  g_alloc_budget.store(after < 0 ? -1 : (long long)after);
  return P3D_OK;
}

int p3d_debug_poison_allocations(int32_t fill)
{
  if (fill > 255) return set_error(P3D_ERR_ARG, "poison_allocations: fill byte %d out of range", fill);
  g_alloc_poison.store(fill < 0 ? -1 : fill);
  return P3D_OK;
}

int p3d_mesh_desc_whole(int32_t mx, int32_t my, int32_t mz, uint32_t dirichlet, p3d_mesh_desc *out)
{
  if (!out || mx < 1 || my < 1 || mz < 1) return set_error(P3D_ERR_ARG, "p3d_mesh_desc_whole: bad sizes");
  out->mx = mx; out->my = my; out->mz = mz;
  out->gx = 2 * mx + 1; out->gy = 2 * my + 1; out->gz = 2 * mz + 1;
  out->ox = out->oy = out->oz = 0;
  out->dirichlet = dirichlet;
  out->global_faces = 0x3f;
  return P3D_OK;
}

int p3d_op_create(const p3d_mesh_desc *mesh, int precision, int device, p3d_op **out)
{
  if (!mesh || !out) return set_error(P3D_ERR_ARG, "p3d_op_create: null argument");
  *out = nullptr;
  const p3d_mesh_desc &m = *mesh;
  if (m.mx < 1 || m.my < 1 || m.mz < 1) return set_error(P3D_ERR_ARG, "p3d_op_create: empty mesh");
  if (m.ox < 0 || m.oy < 0 || m.oz < 0 || m.ox + 2 * m.mx + 1 > m.gx || m.oy + 2 * m.my + 1 > m.gy ||
      m.oz + 2 * m.mz + 1 > m.gz)
    return set_error(P3D_ERR_ARG, "p3d_op_create: element block exceeds the ghosted lattice");
  if (precision != P3D_PREC_F64 && precision != P3D_PREC_F32)
    return set_error(P3D_ERR_ARG, "p3d_op_create: precision must be 64 or 32");
  int ndev = 0;
  if (int rc = cuda_check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount")) return rc;
  if (device < 0 || device >= ndev) return set_error(P3D_ERR_ARG, "p3d_op_create: device %d of %d", device, ndev);
  if (int rc = cuda_check(cudaSetDevice(device), "cudaSetDevice")) return rc;
  if (int rc = upload_tables()) return rc;
  p3d_op *op = new p3d_op();
  op->m = m;
  op->prec = precision;
  op->device = device;
  op->bc = P3D_BC_NONE;
  op->geom = P3D_GEOM_GENERAL;
  if (int rc = cuda_check(cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking), "cudaStreamCreate")) {
    delete op;
    return rc;
  }
  *out = op;
  return P3D_OK;
}

int p3d_op_destroy(p3d_op *op)
{
  if (!op) return P3D_OK;
  cudaSetDevice(op->device);
  p3d_op_set_host_register(op, 0);
  free_dev(op->coords);
  free_dev(op->kgen);
  free_dev(op->kgq);
  free_dev(op->kaff);
  free_dev(op->kpre);
  free_dev(op->hx);
  free_dev(op->hy);
  if (op->flag) cudaFree(op->flag);
  free_dev(op->res_u);
  for (auto &e : op->ev)
    if (e) cudaEventDestroy(e);
  if (op->s_h2d) cudaStreamDestroy(op->s_h2d);
  if (op->s_d2h) cudaStreamDestroy(op->s_d2h);
  if (op->stream) cudaStreamDestroy(op->stream);
  delete op;
  return P3D_OK;
}

int p3d_op_set_coefficients_device(p3d_op *op, const double *coords, const double *eta, int geom_mode)
{
  if (!op || !coords || !eta) return set_error(P3D_ERR_ARG, "set_coefficients: null argument");
  if (geom_mode < P3D_GEOM_AUTO || geom_mode > P3D_GEOM_AFFINE) return set_error(P3D_ERR_ARG, "bad geometry mode");
  cudaSetDevice(op->device);
  if (int rc = order_after_caller()) return rc; // coords/eta may still be being written on the caller's stream
  return op_setup_device(op, coords, eta, geom_mode);
}

int p3d_op_set_coefficients(p3d_op *op, const double *coords, const double *eta, int geom_mode)
{
  if (!op || !coords || !eta) return set_error(P3D_ERR_ARG, "set_coefficients: null argument");
  cudaSetDevice(op->device);
  const p3d_mesh_desc &m = op->m;
  size_t nn = (size_t)m.gx * m.gy * m.gz, nel = (size_t)m.mx * m.my * m.mz;
  void *dc = nullptr, *de = nullptr;
  int rc = dev_alloc(&dc, 3 * nn * 8, "coords staging");
  if (!rc) rc = dev_alloc(&de, 27 * nel * 8, "eta staging");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(dc, coords, 3 * nn * 8, cudaMemcpyHostToDevice, op->stream), "H2D coords");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(de, eta, 27 * nel * 8, cudaMemcpyHostToDevice, op->stream), "H2D eta");
  if (!rc && (geom_mode < P3D_GEOM_AUTO || geom_mode > P3D_GEOM_AFFINE)) rc = set_error(P3D_ERR_ARG, "bad geometry mode");
  if (!rc) rc = op_setup_device(op, (const double *)dc, (const double *)de, geom_mode); // same stream as the copies
  cudaStreamSynchronize(op->stream);
  if (dc) cudaFree(dc);
  if (de) cudaFree(de);
  return rc;
}

int p3d_op_set_bc_mode(p3d_op *op, int bc_mode)
{
  if (!op || (bc_mode != P3D_BC_NONE && bc_mode != P3D_BC_MATMULT)) return set_error(P3D_ERR_ARG, "bad bc mode");
  op->bc = bc_mode;
  return P3D_OK;
}

int p3d_op_geometry_mode(const p3d_op *op, int *mode)
{
  if (!op || !mode) return set_error(P3D_ERR_ARG, "null argument");
  *mode = op->geom;
  return P3D_OK;
}

int p3d_op_sizes(const p3d_op *op, int64_t *nv, int64_t *np)
{
  if (!op) return set_error(P3D_ERR_ARG, "null argument");
  if (nv) *nv = 3LL * op->m.gx * op->m.gy * op->m.gz;
  if (np) *np = 4LL * op->m.mx * op->m.my * op->m.mz;
  return P3D_OK;
}

#define P3D_REQUIRE_SETUP(op)                                                                                    \
  do {                                                                                                           \
    if (!(op)) return set_error(P3D_ERR_ARG, "null operator");                                                   \
    if (!(op)->have_coef) return set_error(P3D_ERR_STATE, "operator coefficients not set");                      \
  } while (0)

int p3d_a11_apply(p3d_op *op, const void *x, void *y, void *stream)
{
  P3D_REQUIRE_SETUP(op);
  if (!x || !y) return set_error(P3D_ERR_ARG, "a11_apply: null vector");
  cudaStream_t st = (cudaStream_t)stream;
  if (op->prec == P3D_PREC_F64) return launch_a11<double>(op, (const double *)x, (double *)y, st);
  return launch_a11<float>(op, (const float *)x, (float *)y, st);
}

int p3d_stokes_residual(p3d_op *op, const double *u, const double *p, const double *phi, const double *fu,
                        const double *fp, double *ru, double *rp, void *stream)
{
  P3D_REQUIRE_SETUP(op);
  if (!u || !p || !ru || !rp) return set_error(P3D_ERR_ARG, "stokes_residual: null vector");
  if (op->prec != P3D_PREC_F64) return set_error(P3D_ERR_ARG, "stokes_residual: FP64 operators only");
  cudaStream_t st = (cudaStream_t)stream;
  const p3d_mesh_desc &m = op->m;
  const size_t nn = (size_t)m.gx * m.gy * m.gz, nel = (size_t)m.mx * m.my * m.mz;
  int rc;
  if (!op->res_u && (rc = dev_alloc(&op->res_u, 3 * nn * 8, "residual u"))) return rc;
  const TileArgs<double> a = tile_args<double>(op, NW_GEN);
  const int ex = m.ox + 2 * m.mx, ey = m.oy + 2 * m.my, ez = m.oz + 2 * m.mz;
  double *ub = (double *)op->res_u;
  dirichlet_values_kernel<<<grid_for(nn), 256, 0, st>>>(m.gx, m.gy, m.gz, m.ox, m.oy, m.oz, ex, ey, ez, a.dir, u, phi, ub, 0);
  count_launch(1);
  if ((rc = cuda_check(cudaMemsetAsync(ru, 0, 3 * nn * 8, st), "memset"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(rp, 0, 4 * nel * 8, st), "memset"))) return rc;
  // element terms on u with the Dirichlet values in place: no column zeroing, no row handling
  const int bc = op->bc;
  op->bc = P3D_BC_NONE;
  rc = launch_general<double, true, true, true>(op, ub, p, ru, rp, st, true);
  op->bc = bc;
  if (rc) return rc;
  if (fu) s_force_u(m.mx, m.my, m.mz, m.gx, m.gy, m.ox, m.oy, m.oz, (const double *)op->coords, fu, ru, st);
  if (fp) s_force_p(m.mx, m.my, m.mz, m.gx, m.gy, m.ox, m.oy, m.oz, (const double *)op->coords, fp, rp, st);
  dirichlet_values_kernel<<<grid_for(nn), 256, 0, st>>>(m.gx, m.gy, m.gz, m.ox, m.oy, m.oz, ex, ey, ez, a.dir, u, phi, ru, 1);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "stokes residual");
}

int p3d_a11_mult(p3d_op *op, const void *x, void *y, void *stream)
{
  P3D_REQUIRE_SETUP(op);
  if (!x || !y) return set_error(P3D_ERR_ARG, "a11_mult: null vector");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = 3ull * op->m.gx * op->m.gy * op->m.gz, es = op->prec == P3D_PREC_F64 ? 8 : 4;
  // y is zeroed (brick-face nodes are accumulated atomically) and never read by the kernel
  int rc = cuda_check(cudaMemsetAsync(y, 0, n * es, st), "a11_mult memset");
  if (rc) return rc;
  if (op->prec == P3D_PREC_F64) return launch_a11<double>(op, (const double *)x, (double *)y, st, true);
  return launch_a11<float>(op, (const float *)x, (float *)y, st, true);
}

int p3d_a11_mult_grouped(p3d_op *const ops[], const void *const x[], void *const y[], int32_t k, void *stream)
{
  if (!ops || !x || !y || k < 1 || k > P3D_GROUP_MAX) return set_error(P3D_ERR_ARG, "a11_mult_grouped: bad arguments");
  for (int i = 0; i < k; i++)
    if (!ops[i] || !x[i] || !y[i]) return set_error(P3D_ERR_ARG, "a11_mult_grouped: null member %d", i);
  P3D_REQUIRE_SETUP(ops[0]);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = 3ull * ops[0]->m.gx * ops[0]->m.gy * ops[0]->m.gz, es = ops[0]->prec == P3D_PREC_F64 ? 8 : 4;
  if (!same_shape_ops(ops, k)) return set_error(P3D_ERR_ARG, "a11_mult_grouped: members differ in shape, path or mode");
  // y zeroed (brick-face nodes are accumulated atomically) and never read, as p3d_a11_mult
  int rc = zero_group(y, k, n * es, st);
  if (rc) return rc;
  if (ops[0]->prec == P3D_PREC_F64)
    return launch_group<double, true, false, false>(ops, k, (const double *const *)x, nullptr, (double *const *)y,
                                                    nullptr, st, true);
  return launch_group<float, true, false, false>(ops, k, (const float *const *)x, nullptr, (float *const *)y, nullptr,
                                                 st, true);
}

int p3d_a11_diagonal(p3d_op *op, void *d, void *stream)
{
  P3D_REQUIRE_SETUP(op);
  if (!d) return set_error(P3D_ERR_ARG, "a11_diagonal: null vector");
  cudaStream_t st = (cudaStream_t)stream;
  if (op->prec == P3D_PREC_F64) return launch_diag<double>(op, (double *)d, st);
  return launch_diag<float>(op, (float *)d, st);
}

int p3d_a12_apply(p3d_op *op, const void *p, void *yu, void *stream)
{
  P3D_REQUIRE_SETUP(op);
  if (!p || !yu) return set_error(P3D_ERR_ARG, "a12_apply: null vector");
  cudaStream_t st = (cudaStream_t)stream;
  if (op->prec == P3D_PREC_F64)
    return launch_general<double, false, true, false>(op, nullptr, (const double *)p, (double *)yu, nullptr, st);
  return launch_general<float, false, true, false>(op, nullptr, (const float *)p, (float *)yu, nullptr, st);
}

int p3d_a21_apply(p3d_op *op, const void *u, void *yp, void *stream)
{
  P3D_REQUIRE_SETUP(op);
  if (!u || !yp) return set_error(P3D_ERR_ARG, "a21_apply: null vector");
  cudaStream_t st = (cudaStream_t)stream;
  if (op->prec == P3D_PREC_F64)
    return launch_general<double, false, false, true>(op, (const double *)u, nullptr, nullptr, (double *)yp, st);
  return launch_general<float, false, false, true>(op, (const float *)u, nullptr, nullptr, (float *)yp, st);
}

int p3d_stokes_apply(p3d_op *op, const void *u, const void *p, void *yu, void *yp, void *stream)
{
  P3D_REQUIRE_SETUP(op);
  if (!u || !p || !yu || !yp) return set_error(P3D_ERR_ARG, "stokes_apply: null vector");
  cudaStream_t st = (cudaStream_t)stream;
  if (op->prec == P3D_PREC_F64)
    return launch_general<double, true, true, true>(op, (const double *)u, (const double *)p, (double *)yu,
                                                    (double *)yp, st);
  return launch_general<float, true, true, true>(op, (const float *)u, (const float *)p, (float *)yu, (float *)yp, st);
}

int p3d_op_set_host_chunks(p3d_op *op, int chunks)
{
  if (!op || chunks < 0 || chunks > 16) return set_error(P3D_ERR_ARG, "set_host_chunks: chunks in [0,16]");
  op->host_chunks = chunks;
  return P3D_OK;
}

int p3d_op_set_host_register(p3d_op *op, int enable)
{
  if (!op) return set_error(P3D_ERR_ARG, "set_host_register: null operator");
  if (!enable) {
    cudaSetDevice(op->device);
    for (int i = 0; i < op->n_reg; i++) cudaHostUnregister(op->reg_ptr[i]);
    op->n_reg = 0;
  }
  op->host_register = enable != 0;
  return P3D_OK;
}

} // extern "C"

namespace p3d {
// Page-lock [p, p + bytes) once, so that the copies of later applies run at
// full PCIe speed instead of through the driver's pageable staging.  Memory
// that is already page-locked (by the caller or an earlier call) is left
// alone; a failed registration is not an error (the copy then goes the
// pageable way).
static void host_register_range(p3d_op *op, const void *p, size_t bytes)
{
  const char *c = (const char *)p;
  for (int i = 0; i < op->n_reg; i++) {
    const char *r = (const char *)op->reg_ptr[i];
    if (c >= r && c + bytes <= r + op->reg_bytes[i]) return;
  }
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type != cudaMemoryTypeUnregistered) return;
  cudaGetLastError();
  if (op->n_reg >= 16) return;
  if (cudaHostRegister(const_cast<void *>(p), bytes, cudaHostRegisterDefault) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  op->reg_ptr[op->n_reg] = const_cast<void *>(p);
  op->reg_bytes[op->n_reg++] = bytes;
}
} // namespace p3d

extern "C" {

int p3d_a11_apply_host(p3d_op *op, const double *xh, double *yh)
{
  P3D_REQUIRE_SETUP(op);
  if (!xh || !yh) return set_error(P3D_ERR_ARG, "a11_apply_host: null vector");
  if (op->prec != P3D_PREC_F64) return set_error(P3D_ERR_ARG, "a11_apply_host: FP64 operators only");
  cudaSetDevice(op->device);
  const p3d_mesh_desc &m = op->m;
  const size_t P = 3ull * m.gx * m.gy, n = P * m.gz; // doubles per lattice plane, in total
  int rc;
  if (op->host_register) {
    host_register_range(op, xh, n * 8);
    host_register_range(op, yh, n * 8);
  }
  if (!op->hx && (rc = dev_alloc(&op->hx, n * 8, "host-apply x"))) return rc;
  if (!op->hy && (rc = dev_alloc(&op->hy, n * 8, "host-apply y"))) return rc;
  if (!op->s_h2d) {
    if ((rc = cuda_check(cudaStreamCreateWithFlags(&op->s_h2d, cudaStreamNonBlocking), "h2d stream"))) return rc;
    if ((rc = cuda_check(cudaStreamCreateWithFlags(&op->s_d2h, cudaStreamNonBlocking), "d2h stream"))) return rc;
    for (auto &e : op->ev)
      if ((rc = cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event"))) return rc;
  }
  // Pipeline along z: chunk k's x planes go in on s_h2d while chunk k-1 is
  // applied on the compute stream, and the y planes no later chunk touches go
  // out on s_d2h.  A chunk is a range of whole brick layers; elements of
  // layers [z0, z1) read node planes oz+2z0 .. oz+2z1 and write the same, and
  // plane oz+2z1 also receives the next chunk's (atomic) contributions.
  const int H = a11_brick_height(op), ntz = (m.mz + H - 1) / H;
  int K = op->host_chunks > 0 ? op->host_chunks : (n >= (size_t)4 << 20 ? 16 : 1);
  if (K > ntz) K = ntz < 1 ? 1 : ntz;
  cudaStream_t cs = op->stream;
  double *dx = (double *)op->hx, *dy = (double *)op->hy;
  if ((rc = cuda_check(cudaMemsetAsync(dy, 0, n * 8, cs), "zero y"))) return rc;
  size_t p0 = 0, q0 = 0; // next x plane to send, next y plane to return
  for (int k = 0; k < K; k++) {
    const int tzb = (int)((long long)k * ntz / K), tze = (int)((long long)(k + 1) * ntz / K);
    const int z1 = std::min(tze * H, m.mz);
    const size_t p1 = k == K - 1 ? (size_t)m.gz : (size_t)(m.oz + 2 * z1 + 1); // x planes [p0, p1)
    const size_t q1 = k == K - 1 ? (size_t)m.gz : (size_t)(m.oz + 2 * z1);     // final y planes [q0, q1)
    cudaEvent_t ex = op->ev[2 * k], ec = op->ev[2 * k + 1];
    if (p1 > p0 && (rc = cuda_check(cudaMemcpyAsync(dx + p0 * P, xh + p0 * P, (p1 - p0) * P * 8, cudaMemcpyHostToDevice,
                                                    op->s_h2d), "H2D x")))
      return rc;
    p0 = std::max(p0, p1);
    if ((rc = cuda_check(cudaEventRecord(ex, op->s_h2d), "record"))) return rc;
    if ((rc = cuda_check(cudaStreamWaitEvent(cs, ex, 0), "wait"))) return rc;
    if ((rc = launch_a11<double>(op, dx, dy, cs, true, tzb, tze))) return rc;
    if ((rc = cuda_check(cudaEventRecord(ec, cs), "record"))) return rc;
    if ((rc = cuda_check(cudaStreamWaitEvent(op->s_d2h, ec, 0), "wait"))) return rc;
    if (q1 > q0 && (rc = cuda_check(cudaMemcpyAsync(yh + q0 * P, dy + q0 * P, (q1 - q0) * P * 8, cudaMemcpyDeviceToHost,
                                                    op->s_d2h), "D2H y")))
      return rc;
    q0 = std::max(q0, q1);
  }
  if ((rc = cuda_check(cudaStreamSynchronize(op->s_d2h), "host apply sync"))) return rc;
  return cuda_check(cudaStreamSynchronize(cs), "host apply sync");
}

} // extern "C"
