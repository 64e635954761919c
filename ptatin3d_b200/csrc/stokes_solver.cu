// Device-resident Q2-P1disc Stokes solver (see p3d_solver_* in include/p3d_b200.h).
//
// Host code here only sequences kernels; every vector lives in HBM.  The
// structure follows the solver the reference assembles from PETSc objects
// (src/ptatin_driver_linear_ts.c:558-882 and the options of
// tests/application/linear/sinker_mf_8x8x8/opts): FGMRES outer iteration,
// PCFIELDSPLIT Schur "upper" factorisation, PCMG on the velocity block with
// Chebyshev/Jacobi smoothing, DMDA trilinear transfers and a Galerkin coarse
// operator.  It is not a translation of PETSc: Chebyshev, Lanczos, FGMRES,
// Gauss-Jordan are restated from their textbook definitions (Saad,
// "Iterative Methods for Sparse Linear Systems", Alg. 12.1 (Chebyshev),
// 6.15/9.6 (FGMRES), 6.17 (Lanczos from CG)).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "p3d_b200.h"
#include "p3d_internal.h"
#include "solver_internal.h"

namespace p3d {

struct Level {
  int m[3] = {0, 0, 0}, n[3] = {0, 0, 0};
  size_t nv = 0;                 // velocity dofs
  p3d_op *op64 = nullptr;        // FP64 operator (smoothing in FP64 mode, Galerkin probe, esteig)
  p3d_op *op32 = nullptr;        // FP32 operator (mixed mode smoothing)
  double *coords = nullptr, *eta = nullptr;
  double *dinv = nullptr;        // FP64 inverse diagonal (Dirichlet slots 1)
  double lmax = 0.0;
  bool gal = false;              // Galerkin level: 27-point block stencil instead of a matrix-free operator
  double *G64 = nullptr;         // stencil coefficients (FP64, always kept)
  float *G32 = nullptr;          // FP32 copy (mixed mode smoothing)
  double *vnode = nullptr, *vden = nullptr; // nodal viscosity and its weights (Q1 coefficient hierarchy)
  void *b = nullptr, *x = nullptr, *r = nullptr, *d = nullptr, *t = nullptr; // MG precision work vectors
};

} // namespace p3d

struct p3d_solver {
  p3d_mesh_desc mesh;
  p3d_solver_opts o;
  int device = 0;
  cudaStream_t st = nullptr;
  std::vector<p3d::Level> lv; // lv[0] coarsest ... lv[L-1] finest
  // coarse solve
  int nc = 0;
  double *cinv = nullptr;          // dense inverse of the Galerkin coarse operator
  double *cb64 = nullptr, *cx64 = nullptr;
  double *gj = nullptr;            // scratch of the blocked Gauss-Jordan inverse
  // Stokes system
  size_t nu = 0, np = 0, N = 0;
  double *Binv = nullptr; // Schur block inverses
  double *bvec = nullptr; // rhs [bu; bp]
  // FGMRES
  double *V = nullptr, *Z = nullptr, *w = nullptr;
  double **Vptr = nullptr; // device array of pointers: V_0..V_m, then one scratch slot
  double **Zptr = nullptr; // device array of pointers: Z_0..Z_{m-1} (grouped solves)
  double *part = nullptr, *hdev = nullptr;
  double *hhost = nullptr; // pinned; [0,hs) and [hs,2hs) Gram-Schmidt passes, 2hs norm
  int hs = 0;              // restart + 1
  // inner conjugate gradient on A11 (MG precision vectors, device-held scalars)
  void *cg_r = nullptr, *cg_z = nullptr, *cg_p = nullptr, *cg_q = nullptr;
  void **cg_ptr = nullptr; // device pointers {p, r} for the dot kernels
  double *cg_sc = nullptr; // fixed count: {rz (2 slots, alternating), pq}; tolerance: see CG_* below
  cudaStream_t st_body = nullptr; // side stream on which the inner loop's body is captured
  const std::atomic<int> *cancel = nullptr; // set by another thread: stop after the current outer iteration
  // preconditioner buffers (fixed for graph capture)
  double *pc_in = nullptr, *pc_out = nullptr, *pc_t = nullptr;
  double *xsol = nullptr; // [u; p] iterate of a solve
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool setup_done = false, rhs_set = false;
  double setup_ms = 0.0;
};

namespace p3d {

static double now_ms()
{
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

#define CK(call)                                                                                                       \
  do {                                                                                                                 \
    int rc_ = (call);                                                                                                  \
    if (rc_) return rc_;                                                                                               \
  } while (0)
#define CU(call, what) CK(cuda_check((call), what))

static uint32_t level_dir(const p3d_solver *s) { return s->mesh.dirichlet; }

// y = A11 x on level l in precision T (BC_MATMULT), y overwritten
template <typename T> static int a11(p3d_solver *s, Level &L, const T *x, T *y)
{
  if (L.gal) {
    g_apply<T>(L.n[0], L.n[1], L.n[2], sizeof(T) == 8 ? (const T *)L.G64 : (const T *)L.G32, x, y, s->st);
    return P3D_OK;
  }
  CU(cudaMemsetAsync(y, 0, L.nv * sizeof(T), s->st), "memset");
  p3d_op *op = sizeof(T) == 8 ? L.op64 : L.op32;
  return launch_a11<T>(op, x, y, s->st, true);
}

// Chebyshev smoothing on level l: x <- x + K steps for A x = b (zero_guess: x = 0 on entry)
template <typename T> static int smooth(p3d_solver *s, Level &L, const T *b, T *x, bool zero_guess)
{
  const size_t n = L.nv;
  T *r = (T *)L.r, *d = (T *)L.d, *t = (T *)L.t;
  const double lo = s->o.cheb_lo * L.lmax, hi = s->o.cheb_hi * L.lmax;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  if (zero_guess) {
    v_cheb_init0<T>(n, L.dinv, b, (T)(1.0 / theta), x, r, d, s->st); // x = 0, r = b
  } else {
    CK(a11<T>(s, L, x, t));
    v_cheb_init_res<T>(n, L.dinv, b, t, (T)(1.0 / theta), r, d, s->st); // r = b - A x
  }
  double rho = 1.0 / sigma;
  const int K = std::max(1, s->o.cheb_its);
  if (K == 1) {
    v_axpby<T>(n, (T)1, d, (T)1, x, s->st); // x += d
    return P3D_OK;
  }
  for (int k = 0; k < K - 1; k++) {
    CK(a11<T>(s, L, d, t));
    double rho_new = 1.0 / (2.0 * sigma - rho);
    // the last step also adds the final direction to x
    v_cheb_step<T>(n, L.dinv, x, r, t, d, (T)(rho_new * rho), (T)(2.0 * rho_new / delta), k == K - 2, s->st);
    rho = rho_new;
  }
  return P3D_OK;
}

// coarse solve: x = Ac^{-1} b (FP64 dense inverse); mask: b may hold values on
// Dirichlet dofs (a one-level hierarchy), zero them first
template <typename T> static int coarse_solve(p3d_solver *s, const T *b, T *x, bool mask)
{
  Level &L = s->lv[0];
  if (mask) v_mask<T>(L.n[0], L.n[1], L.n[2], level_dir(s), const_cast<T *>(b), s->st);
  if (sizeof(T) == 8) {
    v_dense_mv(s->nc, s->cinv, (const double *)b, (double *)x, s->st);
  } else {
    v_convert<float, double>(L.nv, (const float *)b, s->cb64, s->st);
    v_dense_mv(s->nc, s->cinv, s->cb64, s->cx64, s->st);
    v_convert<double, float>(L.nv, s->cx64, (float *)x, s->st);
  }
  return P3D_OK;
}

// V-cycle on level l: x = MG(b), x overwritten
template <typename T> static int vcycle(p3d_solver *s, int l, const T *b, T *x)
{
  // the coarse right-hand side comes masked from the restriction
  if (l == 0) return coarse_solve<T>(s, b, x, (int)s->lv.size() == 1);
  Level &L = s->lv[l], &C = s->lv[l - 1];
  const uint32_t dir = level_dir(s);
  CK(smooth<T>(s, L, b, x, true));
  T *t = (T *)L.t;
  CK(a11<T>(s, L, x, t));
  CK(mg_restrict_residual<T>(C.n[0], C.n[1], C.n[2], dir, b, t, (T *)C.b, s->st)); // C.b = mask(P^T mask(b - A x))
  CK(vcycle<T>(s, l - 1, (const T *)C.b, (T *)C.x));
  CK(mg_prolong_add<T>(C.n[0], C.n[1], C.n[2], dir, (const T *)C.x, x, s->st)); // x += mask(P C.x)
  CK(smooth<T>(s, L, b, x, false));
  return P3D_OK;
}

// Velocity block of the preconditioner, x ~ A11^{-1} b on the finest level.
// inner_its = 0: one V-cycle.  inner_its = k: k iterations of conjugate
// gradients preconditioned by the V-cycle (a symmetric positive definite
// operator: Chebyshev pre/post smoothing with the same polynomial and an exact
// coarse solve), x_0 = 0.  The step lengths never leave the device, so the
// whole solve is one captured graph.  b may be overwritten (it is the CG
// residual when it aliases cg_r).
template <typename T> static int velocity_solve_rtol(p3d_solver *s, const T *b, T *x);
template <typename T> static int velocity_solve(p3d_solver *s, const T *b, T *x)
{
  if (s->o.inner_rtol > 0.0) return velocity_solve_rtol<T>(s, b, x);
  const int top = (int)s->lv.size() - 1;
  const int K = s->o.inner_its;
  if (K <= 0) return vcycle<T>(s, top, b, x);
  Level &F = s->lv.back();
  const size_t n = F.nv;
  T *r = (T *)s->cg_r, *z = (T *)s->cg_z, *p = (T *)s->cg_p, *q = (T *)s->cg_q;
  const T *const *pp = (const T *const *)s->cg_ptr;     // {p}
  const T *const *pr = (const T *const *)s->cg_ptr + 1; // {r}
  double *sc = s->cg_sc;
  if ((const void *)b != (const void *)r) CU(cudaMemcpyAsync(r, b, n * sizeof(T), cudaMemcpyDeviceToDevice, s->st), "copy");
  CU(cudaMemsetAsync(x, 0, n * sizeof(T), s->st), "memset");
  CK(vcycle<T>(s, top, r, z));
  CU(cudaMemcpyAsync(p, z, n * sizeof(T), cudaMemcpyDeviceToDevice, s->st), "copy");
  v_mdot<T>(n, 1, pr, z, s->part, sc + 0, s->st); // rz
  for (int k = 0; k < K; k++) {
    double *rz = sc + (k & 1), *rz_new = sc + ((k + 1) & 1), *pq = sc + 2;
    CK(a11<T>(s, F, p, q));
    v_mdot<T>(n, 1, pp, q, s->part, pq, s->st);
    const bool last = k == K - 1;
    v_cg_xr<T>(n, rz, pq, x, r, p, q, !last, s->st);
    if (last) break;
    CK(vcycle<T>(s, top, r, z));
    v_mdot<T>(n, 1, pr, z, s->part, rz_new, s->st);
    v_cg_p<T>(n, rz_new, rz, z, p, s->st);
  }
  return P3D_OK;
}

// Scalars of the tolerance-driven inner CG (device memory, doubles).
enum { CG_RZ_OLD = 0, CG_RZ_NEW, CG_PQ, CG_RR, CG_TOL2, CG_K, CG_TOTAL, CG_CONT, CG_NSC };

// Start of the inner solve: |b|^2 is in sc[CG_RR].  Sets the stopping
// threshold rtol^2 |b|^2, rz_old = 1 (p starts at 0, so the first direction
// is z whatever beta is) and the loop condition.
__global__ void k_cg_begin(double *sc, double rtol2, int kmax, cudaGraphConditionalHandle h, int use_handle)
{
  const double bb = sc[CG_RR];
  sc[CG_TOL2] = rtol2 * bb;
  sc[CG_RZ_OLD] = 1.0;
  sc[CG_K] = 0.0;
  const unsigned cont = (bb > 0.0 && isfinite(bb) && kmax > 0) ? 1u : 0u;
  sc[CG_CONT] = (double)cont;
  if (use_handle) cudaGraphSetConditional(h, cont);
}
// End of one inner iteration: |r|^2 is in sc[CG_RR].  Continue while
// |r| > rtol |b| and fewer than kmax iterations ran (the loop always ends).
__global__ void k_cg_end(double *sc, int kmax, cudaGraphConditionalHandle h, int use_handle)
{
  sc[CG_RZ_OLD] = sc[CG_RZ_NEW];
  const double k = sc[CG_K] + 1.0;
  sc[CG_K] = k;
  sc[CG_TOTAL] += 1.0;
  const double rr = sc[CG_RR];
  const unsigned cont = (rr > sc[CG_TOL2] && isfinite(rr) && k < (double)kmax) ? 1u : 0u;
  sc[CG_CONT] = (double)cont;
  if (use_handle) cudaGraphSetConditional(h, cont);
}

// One iteration of the tolerance-driven inner CG (preconditioned by the V-cycle):
//   z = MG(r); beta = r.z / rz_old; p = z + beta p; q = A p; alpha = r.z / p.q;
//   x += alpha p; r -= alpha q; |r|^2
template <typename T> static int inner_cg_body(p3d_solver *s, T *x, cudaGraphConditionalHandle h, int use_handle)
{
  const int top = (int)s->lv.size() - 1;
  Level &F = s->lv.back();
  const size_t n = F.nv;
  T *r = (T *)s->cg_r, *z = (T *)s->cg_z, *p = (T *)s->cg_p, *q = (T *)s->cg_q;
  const T *const *pp = (const T *const *)s->cg_ptr;     // {p}
  const T *const *pr = (const T *const *)s->cg_ptr + 1; // {r}
  double *sc = s->cg_sc;
  CK(vcycle<T>(s, top, r, z));
  v_mdot<T>(n, 1, pr, z, s->part, sc + CG_RZ_NEW, s->st);
  v_cg_p<T>(n, sc + CG_RZ_NEW, sc + CG_RZ_OLD, z, p, s->st);
  CK(a11<T>(s, F, p, q));
  v_mdot<T>(n, 1, pp, q, s->part, sc + CG_PQ, s->st);
  v_cg_xr<T>(n, sc + CG_RZ_NEW, sc + CG_PQ, x, r, p, q, true, s->st);
  v_mdot<T>(n, 1, pr, r, s->part, sc + CG_RR, s->st);
  k_cg_end<<<1, 1, 0, s->st>>>(sc, s->o.inner_its, h, use_handle);
  count_launch(1);
  return cuda_check(cudaGetLastError(), "inner cg end");
}

// Velocity block solved to a relative tolerance: CG on A11 preconditioned by
// the V-cycle until |b - A x| <= inner_rtol |b| or inner_its iterations (the
// reference's inner -fieldsplit_u_ksp with -fieldsplit_u_ksp_rtol, there an
// FGMRES; with a symmetric positive definite V-cycle CG needs no basis).
// Inside a stream capture the loop becomes a conditional WHILE node whose
// condition a one-thread kernel sets from the device-held residual, so the
// whole preconditioner stays one graph; eagerly the host reads the
// condition after each iteration.
template <typename T> static int velocity_solve_rtol(p3d_solver *s, const T *b, T *x)
{
  Level &F = s->lv.back();
  const size_t n = F.nv;
  T *r = (T *)s->cg_r, *p = (T *)s->cg_p;
  const T *const *pr = (const T *const *)s->cg_ptr + 1; // {r}
  double *sc = s->cg_sc;
  const double rtol2 = s->o.inner_rtol * s->o.inner_rtol;
  const int kmax = s->o.inner_its;
  cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
  CU(cudaStreamIsCapturing(s->st, &cst), "capture status");
  const bool capturing = cst == cudaStreamCaptureStatusActive;
  cudaGraphConditionalHandle h = 0;
  cudaGraph_t g = nullptr;
  if (capturing) {
    CU(cudaStreamGetCaptureInfo(s->st, &cst, nullptr, &g, nullptr, nullptr), "capture info");
    CU(cudaGraphConditionalHandleCreate(&h, g, 0, 0), "conditional handle");
  }
  if ((const void *)b != (const void *)r) CU(cudaMemcpyAsync(r, b, n * sizeof(T), cudaMemcpyDeviceToDevice, s->st), "copy");
  CU(cudaMemsetAsync(x, 0, n * sizeof(T), s->st), "memset");
  CU(cudaMemsetAsync(p, 0, n * sizeof(T), s->st), "memset");
  v_mdot<T>(n, 1, pr, r, s->part, sc + CG_RR, s->st); // |b|^2
  k_cg_begin<<<1, 1, 0, s->st>>>(sc, rtol2, kmax, h, capturing ? 1 : 0);
  count_launch(1);
  CU(cudaGetLastError(), "inner cg begin");
  if (!capturing) {
    for (int k = 0; k < kmax; k++) {
      double cont = 0.0;
      CU(cudaMemcpyAsync(&cont, sc + CG_CONT, 8, cudaMemcpyDeviceToHost, s->st), "d2h");
      CU(cudaStreamSynchronize(s->st), "sync");
      if (cont == 0.0) break;
      CK(inner_cg_body<T>(s, x, h, 0));
    }
    return P3D_OK;
  }
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  CU(cudaStreamGetCaptureInfo(s->st, &cst, nullptr, &g, &deps, &nd), "capture info");
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional}; // the other members zero
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cn = nullptr;
  CU(cudaGraphAddNode(&cn, g, deps, nd, &cp), "conditional node");
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // capture the body into the node's graph on the side stream
  cudaStream_t main = s->st;
  s->st = s->st_body;
  int rc = cuda_check(cudaStreamBeginCaptureToGraph(s->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                      "capture loop body");
  if (!rc) {
    rc = inner_cg_body<T>(s, x, h, 1);
    cudaGraph_t out = nullptr;
    const int rc2 = cuda_check(cudaStreamEndCapture(s->st, &out), "end loop body capture");
    if (!rc) rc = rc2;
  }
  s->st = main;
  if (rc) return rc;
  return cuda_check(cudaStreamUpdateCaptureDependencies(main, &cn, 1, cudaStreamSetCaptureDependencies),
                    "capture dependencies");
}

// block upper-triangular preconditioner: zp = S^{-1} rp ; zu = MG(ru - A12 zp)
static int apply_pc(p3d_solver *s, const double *in, double *out)
{
  const double *ru = in, *rp = in + s->nu;
  double *zu = out, *zp = out + s->nu;
  Level &F = s->lv.back();
  v_block4(s->np / 4, s->Binv, rp, zp, 1.0, s->st);
  double *t = s->pc_t;
  CU(cudaMemsetAsync(t, 0, s->nu * 8, s->st), "memset");
  CK((launch_general<double, false, true, false>(F.op64, nullptr, zp, t, nullptr, s->st)));
  v_axpby<double>(s->nu, 1.0, ru, -1.0, t, s->st); // t = ru - A12 zp
  if (s->o.mg_precision == P3D_PREC_F64) {
    CK(velocity_solve<double>(s, t, zu));
  } else {
    v_convert<double, float>(s->nu, t, (float *)s->cg_r, s->st);
    CK(velocity_solve<float>(s, (const float *)s->cg_r, (float *)F.x));
    v_convert<float, double>(s->nu, (const float *)F.x, zu, s->st);
  }
  return P3D_OK;
}

static int run_pc(p3d_solver *s, const double *in, double *out)
{
  if (s->gexec) {
    CU(cudaMemcpyAsync(s->pc_in, in, s->N * 8, cudaMemcpyDeviceToDevice, s->st), "pc copy in");
    CU(cudaGraphLaunch(s->gexec, s->st), "graph launch");
    count_launch(1);
    CU(cudaMemcpyAsync(out, s->pc_out, s->N * 8, cudaMemcpyDeviceToDevice, s->st), "pc copy out");
    return P3D_OK;
  }
  return apply_pc(s, in, out);
}

// full operator y = [A11 A12; A21 0] x (BC_MATMULT)
static int stokes_op(p3d_solver *s, const double *x, double *y)
{
  CU(cudaMemsetAsync(y, 0, s->N * 8, s->st), "memset");
  Level &F = s->lv.back();
  return launch_general<double, true, true, true>(F.op64, x, x + s->nu, y, y + s->nu, s->st, true);
}

// ||v||_2 (FP64)
static int norm2(p3d_solver *s, const double *v, size_t n, double *out)
{
  const int slot = s->hs, h = 2 * s->hs;
  CU(cudaMemcpyAsync(s->Vptr + slot, &v, sizeof(double *), cudaMemcpyHostToDevice, s->st), "ptr");
  v_mdot<double>(n, 1, (const double *const *)(s->Vptr + slot), v, s->part, s->hdev + h, s->st);
  CU(cudaMemcpyAsync(s->hhost + h, s->hdev + h, 8, cudaMemcpyDeviceToHost, s->st), "d2h");
  CU(cudaStreamSynchronize(s->st), "sync");
  const double ss = s->hhost[h];
  *out = ss > 0.0 ? std::sqrt(ss) : (ss <= 0.0 ? 0.0 : ss); // a NaN stays NaN (std::max(0, NaN) would give 0)
  return P3D_OK;
}

// largest eigenvalue of a symmetric tridiagonal matrix (bisection on Sturm counts)
static double tridiag_lmax(const std::vector<double> &a, const std::vector<double> &b)
{
  int n = (int)a.size();
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < n; i++) {
    double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < n ? std::fabs(b[i]) : 0.0);
    lo = std::min(lo, a[i] - r);
    hi = std::max(hi, a[i] + r);
  }
  auto count_below = [&](double x) {
    int c = 0;
    double q = a[0] - x;
    if (q < 0) c++;
    for (int i = 1; i < n; i++) {
      double qq = (std::fabs(q) < 1e-300) ? 1e-300 : q;
      q = a[i] - x - b[i - 1] * b[i - 1] / qq;
      if (q < 0) c++;
    }
    return c;
  };
  for (int it = 0; it < 200; it++) {
    double mid = 0.5 * (lo + hi);
    if (count_below(mid) >= n) hi = mid;
    else lo = mid;
  }
  return hi;
}

// lmax(D^{-1} A) of level L by CG-Lanczos (FP64)
static int estimate_lmax(p3d_solver *s, Level &L)
{
  const size_t n = L.nv;
  double *x = (double *)L.x, *r = (double *)L.r, *z = (double *)L.d, *p = (double *)L.b, *q = (double *)L.t;
  // deterministic pseudo-random start, Dirichlet entries zero
  std::vector<double> h(n);
  uint64_t st = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < n; i++) {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    h[i] = (double)(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  CU(cudaMemcpyAsync(r, h.data(), n * 8, cudaMemcpyHostToDevice, s->st), "h2d");
  v_mask<double>(L.n[0], L.n[1], L.n[2], level_dir(s), r, s->st);
  (void)x;
  v_jacobi<double>(n, L.dinv, r, z, s->st);
  CU(cudaMemcpyAsync(p, z, n * 8, cudaMemcpyDeviceToDevice, s->st), "copy");
  auto dot = [&](const double *a, const double *b, double *out) -> int {
    const double *ptrs[1] = {a};
    const int slot = s->hs, h = 2 * s->hs;
    CU(cudaMemcpyAsync(s->Vptr + slot, ptrs, sizeof(double *), cudaMemcpyHostToDevice, s->st), "ptr");
    v_mdot<double>(n, 1, (const double *const *)(s->Vptr + slot), b, s->part, s->hdev + h, s->st);
    CU(cudaMemcpyAsync(s->hhost + h, s->hdev + h, 8, cudaMemcpyDeviceToHost, s->st), "d2h");
    CU(cudaStreamSynchronize(s->st), "sync");
    *out = s->hhost[h];
    return P3D_OK;
  };
  double rz;
  CK(dot(r, z, &rz));
  std::vector<double> alpha, beta;
  const int K = std::max(2, s->o.esteig_its);
  for (int k = 0; k < K && rz > 0; k++) {
    CK(a11<double>(s, L, p, q));
    double pq;
    CK(dot(p, q, &pq));
    if (!(pq > 0)) break;
    double a = rz / pq;
    alpha.push_back(a);
    v_axpby<double>(n, -a, q, 1.0, r, s->st);
    v_jacobi<double>(n, L.dinv, r, z, s->st);
    double rz2;
    CK(dot(r, z, &rz2));
    double bt = rz2 / rz;
    beta.push_back(bt);
    v_axpby<double>(n, 1.0, z, bt, p, s->st);
    rz = rz2;
  }
  int m = (int)alpha.size();
  if (m == 0) return set_error(P3D_ERR_BREAKDOWN, "esteig: CG broke down at the first step");
  std::vector<double> ta(m), tb(std::max(1, m - 1));
  for (int j = 0; j < m; j++) {
    ta[j] = 1.0 / alpha[j] + (j > 0 ? beta[j - 1] / alpha[j - 1] : 0.0);
    if (j + 1 < m) tb[j] = std::sqrt(std::max(0.0, beta[j])) / alpha[j];
  }
  L.lmax = tridiag_lmax(ta, tb);
  if (!(L.lmax > 0) || !std::isfinite(L.lmax)) return set_error(P3D_ERR_BREAKDOWN, "esteig: bad lmax %g", L.lmax);
  return P3D_OK;
}

// Galerkin coarse operator Ac = P~^T A1 P~ (+ identity on coarse Dirichlet rows), inverted in place
static int build_coarse(p3d_solver *s)
{
  Level &C = s->lv[0];
  const int nc = (int)C.nv;
  s->nc = nc;
  const uint32_t dir = level_dir(s);
  // kept across setups (a solver re-set up with new coefficients allocates nothing)
  if (!s->cinv) CK(dev_alloc((void **)&s->cinv, (size_t)nc * nc * 8, "coarse operator"));
  if (!s->cb64) CK(dev_alloc((void **)&s->cb64, (size_t)nc * 8, "coarse vec"));
  if (!s->cx64) CK(dev_alloc((void **)&s->cx64, (size_t)nc * 8, "coarse vec"));
  if (!s->gj) CK(dev_alloc((void **)&s->gj, dense_inverse_scratch(nc) * 8, "gauss-jordan"));
  // coarse Dirichlet mask on the host
  std::vector<char> isdir(nc, 0);
  {
    int nx = C.n[0], ny = C.n[1], nz = C.n[2];
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
          for (int c = 0; c < 3; c++) {
            bool d = false;
            d |= (i == 0) && (dir >> (0 + c) & 1u);
            d |= (i == nx - 1) && (dir >> (3 + c) & 1u);
            d |= (j == 0) && (dir >> (6 + c) & 1u);
            d |= (j == ny - 1) && (dir >> (9 + c) & 1u);
            d |= (k == 0) && (dir >> (12 + c) & 1u);
            d |= (k == nz - 1) && (dir >> (15 + c) & 1u);
            isdir[3 * ((size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k)) + c] = d;
          }
  }
  if (C.gal) {
    CU(cudaMemsetAsync(s->cinv, 0, (size_t)nc * nc * 8, s->st), "memset");
    g_dense(C.n[0], C.n[1], C.n[2], C.G64, s->cinv, s->st);
  } else if (s->lv.size() == 1) {
    // single level: probe the operator itself
    for (int j = 0; j < nc; j++) {
      double *e = s->cb64;
      CU(cudaMemsetAsync(e, 0, nc * 8, s->st), "memset");
      double one = 1.0;
      CU(cudaMemcpyAsync(e + j, &one, 8, cudaMemcpyHostToDevice, s->st), "h2d");
      CK(a11<double>(s, C, e, s->cinv + (size_t)j * nc));
    }
  } else {
    Level &F = s->lv[1];
    double *ef = (double *)F.b, *yf = (double *)F.t;
    for (int j = 0; j < nc; j++) {
      double *col = s->cinv + (size_t)j * nc;
      if (isdir[j]) {
        CU(cudaMemsetAsync(col, 0, nc * 8, s->st), "memset");
        double one = 1.0;
        CU(cudaMemcpyAsync(col + j, &one, 8, cudaMemcpyHostToDevice, s->st), "h2d");
        continue;
      }
      CU(cudaMemsetAsync(s->cb64, 0, nc * 8, s->st), "memset");
      double one = 1.0;
      CU(cudaMemcpyAsync(s->cb64 + j, &one, 8, cudaMemcpyHostToDevice, s->st), "h2d");
      CK(mg_prolong<double>(C.n[0], C.n[1], C.n[2], 3, s->cb64, ef, s->st));
      v_mask<double>(F.n[0], F.n[1], F.n[2], dir, ef, s->st);
      CK(a11<double>(s, F, ef, yf));
      v_mask<double>(F.n[0], F.n[1], F.n[2], dir, yf, s->st);
      CK(mg_restrict<double>(C.n[0], C.n[1], C.n[2], 3, yf, col, s->st));
      v_mask<double>(C.n[0], C.n[1], C.n[2], dir, col, s->st);
    }
  }
  // Ac is symmetric: columns stored as rows is the same matrix.  Invert in place.
  CK(dense_inverse_spd(nc, s->cinv, s->gj, s->st));
  return cuda_check(cudaStreamSynchronize(s->st), "coarse inverse");
}

// Galerkin operator of level l from level l+1: Ac = P~^T A P~ (P~ = P with
// Dirichlet rows and columns removed) + identity on the Dirichlet dofs, probed
// with the 81 colour/component vectors.
static int build_galerkin(p3d_solver *s, int l)
{
  Level &C = s->lv[l], &F = s->lv[l + 1];
  const uint32_t dir = level_dir(s);
  const size_t nn = (size_t)C.n[0] * C.n[1] * C.n[2];
  if (!C.G64) CK(dev_alloc((void **)&C.G64, 243 * nn * 8, "galerkin stencil"));
  CU(cudaMemsetAsync(C.G64, 0, 243 * nn * 8, s->st), "memset");
  double *xc = (double *)C.x, *yc = (double *)C.r, *xf = (double *)F.b, *yf = (double *)F.t;
  for (int ck = 0; ck < 3; ck++)
    for (int cj = 0; cj < 3; cj++)
      for (int ci = 0; ci < 3; ci++)
        for (int d = 0; d < 3; d++) {
          g_probe_vec(C.n[0], C.n[1], C.n[2], ci, cj, ck, d, dir, xc, s->st);
          CK(mg_prolong<double>(C.n[0], C.n[1], C.n[2], 3, xc, xf, s->st));
          v_mask<double>(F.n[0], F.n[1], F.n[2], dir, xf, s->st);
          CK(a11<double>(s, F, xf, yf));
          v_mask<double>(F.n[0], F.n[1], F.n[2], dir, yf, s->st);
          CK(mg_restrict<double>(C.n[0], C.n[1], C.n[2], 3, yf, yc, s->st));
          v_mask<double>(C.n[0], C.n[1], C.n[2], dir, yc, s->st);
          g_probe_scatter(C.n[0], C.n[1], C.n[2], ci, cj, ck, d, yc, C.G64, s->st);
        }
  g_dirichlet(C.n[0], C.n[1], C.n[2], dir, C.G64, s->st);
  return cuda_check(cudaStreamSynchronize(s->st), "galerkin");
}

static void free_level(Level &L)
{
  p3d_op_destroy(L.op64);
  p3d_op_destroy(L.op32);
  L.op64 = L.op32 = nullptr;
  for (void *p : {(void *)L.coords, (void *)L.eta, (void *)L.dinv, L.b, L.x, L.r, L.d, L.t, (void *)L.G64, (void *)L.G32,
                  (void *)L.vnode, (void *)L.vden})
    if (p) cudaFree(p);
  L.coords = L.eta = L.dinv = nullptr;
  L.G64 = nullptr;
  L.G32 = nullptr;
  L.vnode = L.vden = nullptr;
  L.b = L.x = L.r = L.d = L.t = nullptr;
}

// eta_nodes: optional finest-level nodal viscosity for the Q1 coefficient
// hierarchy (nullptr: projected from the Gauss-point values)
static int solver_setup(p3d_solver *s, const double *coords, const double *eta, const double *eta_nodes)
{
  double t0 = now_ms();
  const int nlev = (int)s->lv.size();
  const bool mixed = s->o.mg_precision == P3D_PREC_F32;
  // hierarchy: finest first
  for (int l = nlev - 1; l >= 0; l--) {
    Level &L = s->lv[l];
    size_t nn = (size_t)L.n[0] * L.n[1] * L.n[2], nel = (size_t)L.m[0] * L.m[1] * L.m[2];
    L.gal = l < nlev - 1 && s->o.coarse_op == P3D_COARSE_GALERKIN;
    // work vectors: FP64 for esteig/Galerkin probing, reused as MG-precision vectors
    for (void **p : {&L.b, &L.x, &L.r, &L.d, &L.t})
      if (!*p) CK(dev_alloc(p, L.nv * 8, "level vector"));
    if (!L.dinv) CK(dev_alloc((void **)&L.dinv, L.nv * 8, "dinv"));
    if (L.gal) {
      CK(build_galerkin(s, l));
      g_diag(L.n[0], L.n[1], L.n[2], L.G64, (double *)L.t, s->st);
      if (mixed && l > 0) {
        if (!L.G32) CK(dev_alloc((void **)&L.G32, 243 * nn * 4, "galerkin stencil f32"));
        v_convert<double, float>(243 * nn, L.G64, L.G32, s->st);
      }
    } else {
      if (!L.coords) CK(dev_alloc((void **)&L.coords, 3 * nn * 8, "level coords"));
      if (!L.eta) CK(dev_alloc((void **)&L.eta, 27 * nel * 8, "level eta"));
      const bool q1 = s->o.coarse_eta == P3D_COARSE_ETA_Q1 && nlev > 1;
      if (q1 && !L.vnode) {
        CK(dev_alloc((void **)&L.vnode, nn * 8, "nodal viscosity"));
        CK(dev_alloc((void **)&L.vden, nn * 8, "nodal weights"));
      }
      if (l == nlev - 1) {
        CU(cudaMemcpyAsync(L.coords, coords, 3 * nn * 8, cudaMemcpyDeviceToDevice, s->st), "coords");
        CU(cudaMemcpyAsync(L.eta, eta, 27 * nel * 8, cudaMemcpyDeviceToDevice, s->st), "eta");
        if (q1 && eta_nodes)
          CU(cudaMemcpyAsync(L.vnode, eta_nodes, nn * 8, cudaMemcpyDeviceToDevice, s->st), "nodal eta");
        else if (q1)
          s_eta_project(L.m[0], L.m[1], L.m[2], eta, L.vnode, L.vden, s->st);
      } else {
        Level &F = s->lv[l + 1];
        s_inject_coords(L.n[0], L.n[1], L.n[2], F.coords, L.coords, s->st);
        if (q1) {
          // vc = (P^T vf) ./ (P^T 1), then clamped Q1 interpolation to the Gauss points
          const size_t nnf = (size_t)F.n[0] * F.n[1] * F.n[2];
          CK(mg_restrict<double>(L.n[0], L.n[1], L.n[2], 1, F.vnode, L.vnode, s->st));
          s_fill(nnf, 1.0, F.vden, s->st);
          CK(mg_restrict<double>(L.n[0], L.n[1], L.n[2], 1, F.vden, L.vden, s->st));
          s_divide(nn, L.vnode, L.vden, s->st);
          s_eta_to_qp(L.m[0], L.m[1], L.m[2], L.vnode, L.eta, s->st);
        } else {
          s_restrict_eta(L.m[0], L.m[1], L.m[2], F.eta, L.eta, s->st);
        }
      }
      CU(cudaStreamSynchronize(s->st), "hierarchy");
      p3d_mesh_desc d;
      p3d_mesh_desc_whole(L.m[0], L.m[1], L.m[2], s->mesh.dirichlet, &d);
      if (!L.op64) CK(p3d_op_create(&d, P3D_PREC_F64, s->device, &L.op64));
      CK(op_setup_device(L.op64, L.coords, L.eta, P3D_GEOM_AUTO)); // level arrays written on s->st, synchronized above
      CK(p3d_op_set_bc_mode(L.op64, P3D_BC_MATMULT));
      if (mixed && l > 0) {
        if (!L.op32) CK(p3d_op_create(&d, P3D_PREC_F32, s->device, &L.op32));
        CK(op_setup_device(L.op32, L.coords, L.eta, P3D_GEOM_AUTO));
        CK(p3d_op_set_bc_mode(L.op32, P3D_BC_MATMULT));
      }
      CU(cudaMemsetAsync(L.t, 0, L.nv * 8, s->st), "memset");
      CK(launch_diag<double>(L.op64, (double *)L.t, s->st));
    }
    // dinv = 1 / diag on the device; only the count of bad entries comes back
    {
      unsigned int *bad = reinterpret_cast<unsigned int *>(s->hdev + 2 * s->hs + 1);
      CU(cudaMemsetAsync(bad, 0, sizeof(unsigned int), s->st), "memset");
      v_invert_diag(L.nv, (const double *)L.t, L.dinv, bad, s->st);
      unsigned int hbad = 0;
      CU(cudaMemcpyAsync(&hbad, bad, sizeof hbad, cudaMemcpyDeviceToHost, s->st), "d2h");
      CU(cudaStreamSynchronize(s->st), "diag");
      if (hbad) return set_error(P3D_ERR_BREAKDOWN, "A11 diagonal: %u entries not positive on level %d", hbad, l);
    }
    if (l > 0) CK(estimate_lmax(s, L));
  }
  CK(build_coarse(s));
  // Schur blocks on the fine mesh
  Level &F = s->lv.back();
  size_t nel = (size_t)F.m[0] * F.m[1] * F.m[2];
  if (!s->Binv) CK(dev_alloc((void **)&s->Binv, 16 * nel * 8, "schur blocks"));
  s_schur_blocks(F.m[0], F.m[1], F.m[2], F.coords, F.eta, s->o.schur_eta == P3D_SCHUR_ETA_GEOMEAN, s->Binv, s->st);
  CU(cudaStreamSynchronize(s->st), "schur");
  // preconditioner graph
  if (s->o.use_graph) {
    if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
    if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
    CU(cudaMemsetAsync(s->pc_in, 0, s->N * 8, s->st), "memset");
    CK(apply_pc(s, s->pc_in, s->pc_out)); // eager run: sets kernel attributes before capture
    CU(cudaStreamSynchronize(s->st), "pc warm");
    CU(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal), "begin capture");
    int rc = apply_pc(s, s->pc_in, s->pc_out);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->st, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    CU(e, "end capture");
    s->graph = g;
    CU(cudaGraphInstantiate(&s->gexec, g, 0), "graph instantiate");
  }
  s->setup_done = true;
  s->setup_ms = now_ms() - t0;
  return P3D_OK;
}

// FGMRES(m), right preconditioned; x = [u; p]
static int fgmres(p3d_solver *s, double *x, p3d_solve_stats *stats)
{
  const int m = s->o.restart;
  const size_t N = s->N;
  double *V = s->V, *Z = s->Z, *w = s->w;
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
  double r0 = -1.0, rnorm = 0.0;
  int its = 0;
  bool conv = false, cancelled = false;
  while (its < s->o.max_it && !cancelled) {
    // r = b - A x  into V_0
    CK(stokes_op(s, x, w));
    v_residual<double>(N, s->bvec, w, V, s->st);
    double beta;
    CK(norm2(s, V, N, &beta));
    if (r0 < 0) r0 = beta;
    rnorm = beta;
    if (!std::isfinite(beta)) return set_error(P3D_ERR_BREAKDOWN, "FGMRES: non-finite residual");
    const double tol = std::max(s->o.rtol * r0, s->o.atol);
    if (beta <= tol) { conv = true; break; }
    v_scale<double>(N, 1.0 / beta, V, s->st);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < m && its < s->o.max_it; j++, its++) {
      double *vj = V + (size_t)j * N, *zj = Z + (size_t)j * N, *vn = V + (size_t)(j + 1) * N;
      CK(run_pc(s, vj, zj));
      CK(stokes_op(s, zj, w));
      // classical Gram-Schmidt, coefficients on the device.  The first pass
      // also forms |w|^2.  When the projection removed less than half of it
      // (|w - V h|^2 = |w|^2 - |h|^2 > |w|^2 / 2) a second pass is not needed
      // ("twice is enough": Giraud, Langou, Rozloznik 2005) and |w - V h|
      // follows from that difference; otherwise the second pass runs and the
      // norm is formed directly.
      v_mdot<double>(N, j + 1, (const double *const *)s->Vptr, w, s->part, s->hdev, s->st, s->hdev + j + 1);
      v_maxpy<double>(N, j + 1, s->hdev, (const double *const *)s->Vptr, w, -1.0, s->st);
      CU(cudaMemcpyAsync(s->hhost, s->hdev, (j + 2) * 8, cudaMemcpyDeviceToHost, s->st), "d2h");
      CU(cudaStreamSynchronize(s->st), "sync");
      double hh = 0.0;
      for (int i = 0; i <= j; i++) {
        H[(size_t)i * m + j] = s->hhost[i];
        hh += s->hhost[i] * s->hhost[i];
      }
      const double wb2 = s->hhost[j + 1];
      double hn;
      if (wb2 - hh > 0.5 * wb2) {
        hn = std::sqrt(wb2 - hh);
      } else {
        v_mdot<double>(N, j + 1, (const double *const *)s->Vptr, w, s->part, s->hdev, s->st);
        v_maxpy<double>(N, j + 1, s->hdev, (const double *const *)s->Vptr, w, -1.0, s->st);
        CU(cudaMemcpyAsync(s->hhost + s->hs, s->hdev, (j + 1) * 8, cudaMemcpyDeviceToHost, s->st), "d2h");
        CK(norm2(s, w, N, &hn)); // synchronizes
        for (int i = 0; i <= j; i++) H[(size_t)i * m + j] += s->hhost[s->hs + i];
      }
      H[(size_t)(j + 1) * m + j] = hn;
      if (hn > 0) {
        CU(cudaMemcpyAsync(vn, w, N * 8, cudaMemcpyDeviceToDevice, s->st), "copy");
        v_scale<double>(N, 1.0 / hn, vn, s->st);
      }
      // Givens
      for (int i = 0; i < j; i++) {
        double a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
      }
      double a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
      double rr = std::hypot(a, b);
      cs[j] = rr > 0 ? a / rr : 1.0;
      sn[j] = rr > 0 ? b / rr : 0.0;
      H[(size_t)j * m + j] = rr;
      H[(size_t)(j + 1) * m + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      rnorm = std::fabs(g[j + 1]);
      if (s->o.verbose) fprintf(stderr, "  fgmres %3d  |r| %.6e\n", its + 1, rnorm);
      if (!std::isfinite(rnorm)) return set_error(P3D_ERR_BREAKDOWN, "FGMRES: non-finite residual estimate");
      if (rnorm <= tol || hn == 0.0) { j++; its++; conv = rnorm <= tol; break; }
      if (s->cancel && s->cancel->load(std::memory_order_relaxed)) { j++; its++; cancelled = true; break; }
    }
    // y = H^{-1} g ; x += Z y
    for (int i = j - 1; i >= 0; i--) {
      double acc = g[i];
      for (int k = i + 1; k < j; k++) acc -= H[(size_t)i * m + k] * y[k];
      y[i] = acc / H[(size_t)i * m + i];
    }
    for (int i = 0; i < j; i++) v_axpby<double>(N, y[i], Z + (size_t)i * N, 1.0, x, s->st);
    if (conv) break;
  }
  // true residual
  CK(stokes_op(s, x, w));
  v_residual<double>(N, s->bvec, w, w, s->st);
  double rt;
  CK(norm2(s, w, N, &rt));
  stats->iterations = its;
  stats->r0 = r0;
  stats->rfinal = rt;
  stats->converged = conv || rt <= std::max(s->o.rtol * r0, s->o.atol) * 1.0000001;
  return cancelled && !stats->converged ? P3D_ERR_CANCELLED : P3D_OK;
}

void solver_set_cancel_flag(p3d_solver *s, const std::atomic<int> *flag) { s->cancel = flag; }


// ============================================================ grouped solve
// The solves of K solvers of one mesh shape and option set, in lock-step:
// every kernel of an iteration -- operators, smoothers, transfers, stencils,
// coarse solves, Gram-Schmidt -- is one launch over all members (grid
// dimension y = member, per-member pointers and scalars in the launch
// parameters), and the block preconditioner of all members is one captured
// graph.  Each member keeps its own Krylov basis, Hessenberg matrix, step
// lengths and stopping test, so its iterates are those of its own solve; a
// member that converges (or breaks down) leaves the group, and the others go
// on (the graph is captured again for the smaller group).
struct Group {
  int K = 0;
  p3d_solver *m[P3D_GROUP_MAX] = {};
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
};

template <typename T> static T *lvec(void *p) { return reinterpret_cast<T *>(p); }

// y = A_l x on level l for every member (y overwritten)
template <typename T> static int g_a11(Group &g, int l, T *const *x, T *const *y)
{
  Level &L0 = g.m[0]->lv[l];
  if (L0.gal) {
    TGroup<T> P;
    memset(&P, 0, sizeof P);
    for (int k = 0; k < g.K; k++) {
      Level &L = g.m[k]->lv[l];
      P.a[k] = sizeof(T) == 8 ? (const T *)L.G64 : (const T *)L.G32;
      P.b[k] = x[k];
      P.out[k] = y[k];
    }
    g_apply_group<T>(P, g.K, L0.n[0], L0.n[1], L0.n[2], g.st);
    return P3D_OK;
  }
  p3d_op *ops[P3D_GROUP_MAX];
  for (int k = 0; k < g.K; k++) ops[k] = sizeof(T) == 8 ? g.m[k]->lv[l].op64 : g.m[k]->lv[l].op32;
  CK(zero_group((void *const *)y, g.K, L0.nv * sizeof(T), g.st));
  return launch_group<T, true, false, false>(ops, g.K, (const T *const *)x, nullptr, y, nullptr, g.st, true);
}

template <typename T> static int g_smooth(Group &g, int l, T *const *b, T *const *x, bool zero_guess)
{
  const int K = g.K;
  const size_t n = g.m[0]->lv[l].nv;
  double theta[P3D_GROUP_MAX], delta[P3D_GROUP_MAX], sigma[P3D_GROUP_MAX], rho[P3D_GROUP_MAX];
  T *r[P3D_GROUP_MAX], *d[P3D_GROUP_MAX], *t[P3D_GROUP_MAX];
  VGroup<T> V;
  memset(&V, 0, sizeof V);
  for (int k = 0; k < K; k++) {
    Level &L = g.m[k]->lv[l];
    const double lo = g.m[k]->o.cheb_lo * L.lmax, hi = g.m[k]->o.cheb_hi * L.lmax;
    theta[k] = 0.5 * (hi + lo); delta[k] = 0.5 * (hi - lo); sigma[k] = theta[k] / delta[k]; rho[k] = 1.0 / sigma[k];
    r[k] = lvec<T>(L.r); d[k] = lvec<T>(L.d); t[k] = lvec<T>(L.t);
    V.dinv[k] = L.dinv;
    V.s[0][k] = 1.0 / theta[k];
  }
  if (zero_guess) {
    for (int k = 0; k < K; k++) { V.v[0][k] = b[k]; V.v[1][k] = x[k]; V.v[2][k] = r[k]; V.v[3][k] = d[k]; }
    vg_cheb_init0<T>(V, K, n, g.st);
  } else {
    CK(g_a11<T>(g, l, x, t));
    for (int k = 0; k < K; k++) { V.v[0][k] = b[k]; V.v[1][k] = t[k]; V.v[2][k] = r[k]; V.v[3][k] = d[k]; }
    vg_cheb_init_res<T>(V, K, n, g.st);
  }
  const int its = std::max(1, g.m[0]->o.cheb_its);
  if (its == 1) {
    for (int k = 0; k < K; k++) { V.v[0][k] = d[k]; V.v[1][k] = x[k]; V.s[0][k] = 1.0; V.s[1][k] = 1.0; }
    vg_axpby<T>(V, K, n, g.st); // x += d
    return P3D_OK;
  }
  for (int step = 0; step < its - 1; step++) {
    CK(g_a11<T>(g, l, d, t));
    for (int k = 0; k < K; k++) {
      const double rn = 1.0 / (2.0 * sigma[k] - rho[k]);
      V.v[0][k] = x[k]; V.v[1][k] = r[k]; V.v[2][k] = t[k]; V.v[3][k] = d[k];
      V.s[0][k] = rn * rho[k];
      V.s[1][k] = 2.0 * rn / delta[k];
      rho[k] = rn;
    }
    vg_cheb_step<T>(V, K, n, step == its - 2, g.st);
  }
  return P3D_OK;
}

template <typename T> static int g_coarse(Group &g, T *const *b, T *const *x)
{
  const int K = g.K, nc = g.m[0]->nc;
  VGroup<double> V;
  memset(&V, 0, sizeof V);
  if (sizeof(T) == 8) {
    for (int k = 0; k < K; k++) { V.v[0][k] = g.m[k]->cinv; V.v[1][k] = (double *)b[k]; V.v[2][k] = (double *)x[k]; }
    vg_dense_mv(V, K, nc, g.st);
    return P3D_OK;
  }
  for (int k = 0; k < K; k++) { V.v[0][k] = (double *)b[k]; V.v[1][k] = g.m[k]->cb64; }
  vg_convert<float, double>(V, K, nc, g.st);
  for (int k = 0; k < K; k++) { V.v[0][k] = g.m[k]->cinv; V.v[1][k] = g.m[k]->cb64; V.v[2][k] = g.m[k]->cx64; }
  vg_dense_mv(V, K, nc, g.st);
  for (int k = 0; k < K; k++) { V.v[0][k] = g.m[k]->cx64; V.v[1][k] = (double *)x[k]; }
  vg_convert<double, float>(V, K, nc, g.st);
  return P3D_OK;
}

template <typename T> static int g_vcycle(Group &g, int l, T *const *b, T *const *x)
{
  if (l == 0) return g_coarse<T>(g, b, x);
  const int K = g.K;
  Level &C0 = g.m[0]->lv[l - 1];
  const uint32_t dir = level_dir(g.m[0]);
  T *t[P3D_GROUP_MAX], *cb[P3D_GROUP_MAX], *cx[P3D_GROUP_MAX];
  for (int k = 0; k < K; k++) {
    t[k] = lvec<T>(g.m[k]->lv[l].t);
    cb[k] = lvec<T>(g.m[k]->lv[l - 1].b);
    cx[k] = lvec<T>(g.m[k]->lv[l - 1].x);
  }
  CK(g_smooth<T>(g, l, b, x, true));
  CK(g_a11<T>(g, l, x, t));
  TGroup<T> P;
  memset(&P, 0, sizeof P);
  for (int k = 0; k < K; k++) { P.a[k] = b[k]; P.b[k] = t[k]; P.out[k] = cb[k]; }
  CK(mg_restrict_residual_group<T>(P, K, C0.n[0], C0.n[1], C0.n[2], dir, g.st));
  CK(g_vcycle<T>(g, l - 1, cb, cx));
  memset(&P, 0, sizeof P);
  for (int k = 0; k < K; k++) { P.a[k] = cx[k]; P.out[k] = x[k]; }
  CK(mg_prolong_add_group<T>(P, K, C0.n[0], C0.n[1], C0.n[2], dir, g.st));
  return g_smooth<T>(g, l, b, x, false);
}

// the block preconditioner of every member on its pc_in -> pc_out
static int g_apply_pc(Group &g)
{
  const int K = g.K;
  const size_t nu = g.m[0]->nu, np = g.m[0]->np;
  VGroup<double> V;
  memset(&V, 0, sizeof V);
  p3d_op *ops[P3D_GROUP_MAX];
  double *t[P3D_GROUP_MAX], *zp[P3D_GROUP_MAX];
  for (int k = 0; k < K; k++) {
    p3d_solver *s = g.m[k];
    V.v[0][k] = s->Binv; V.v[1][k] = s->pc_in + nu; V.v[2][k] = s->pc_out + nu;
    t[k] = s->pc_t;
    zp[k] = s->pc_out + nu;
    ops[k] = s->lv.back().op64;
  }
  vg_block4(V, K, np / 4, g.st); // zp = S^{-1} rp
  CK(zero_group((void *const *)t, K, nu * 8, g.st));
  CK((launch_group<double, false, true, false>(ops, K, nullptr, (const double *const *)zp, t, nullptr, g.st, false)));
  for (int k = 0; k < K; k++) { V.v[0][k] = g.m[k]->pc_in; V.v[1][k] = t[k]; V.s[0][k] = 1.0; V.s[1][k] = -1.0; }
  vg_axpby<double>(V, K, nu, g.st); // t = ru - A12 zp
  const int top = (int)g.m[0]->lv.size() - 1;
  if (g.m[0]->o.mg_precision == P3D_PREC_F64) {
    double *zu[P3D_GROUP_MAX];
    for (int k = 0; k < K; k++) zu[k] = g.m[k]->pc_out;
    return g_vcycle<double>(g, top, t, zu);
  }
  float *tf[P3D_GROUP_MAX], *xf[P3D_GROUP_MAX];
  for (int k = 0; k < K; k++) {
    tf[k] = lvec<float>(g.m[k]->cg_r);
    xf[k] = lvec<float>(g.m[k]->lv.back().x);
    V.v[0][k] = t[k]; V.v[1][k] = (double *)tf[k];
  }
  vg_convert<double, float>(V, K, nu, g.st);
  CK(g_vcycle<float>(g, top, tf, xf));
  for (int k = 0; k < K; k++) { V.v[0][k] = (double *)xf[k]; V.v[1][k] = g.m[k]->pc_out; }
  vg_convert<float, double>(V, K, nu, g.st);
  return P3D_OK;
}

static void g_release_graph(Group &g)
{
  if (g.gexec) cudaGraphExecDestroy(g.gexec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g.gexec = nullptr;
  g.graph = nullptr;
}

// capture the grouped preconditioner of the current members.  The first
// capture of a group follows one eager run (kernel attributes are set outside
// a capture).  A later capture (the membership changed) has the same
// sequence of kernels, only with other grids and arguments, so it updates the
// executable graph in place; a new one is instantiated only if that fails.
static int g_capture(Group &g)
{
  if (!g.gexec) {
    CK(g_apply_pc(g));
    CU(cudaStreamSynchronize(g.st), "grouped pc warm");
  }
  CU(cudaStreamBeginCapture(g.st, cudaStreamCaptureModeThreadLocal), "begin capture");
  int rc = g_apply_pc(g);
  cudaGraph_t gr = nullptr;
  cudaError_t e = cudaStreamEndCapture(g.st, &gr);
  if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
  CU(e, "end capture");
  if (g.gexec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(g.gexec, gr, &info) == cudaSuccess) {
      if (g.graph) cudaGraphDestroy(g.graph);
      g.graph = gr;
      return P3D_OK;
    }
    cudaGetLastError(); // the update was refused: instantiate anew
    g_release_graph(g);
  }
  g.graph = gr;
  return cuda_check(cudaGraphInstantiate(&g.gexec, gr, 0), "graph instantiate");
}

// y = [A11 A12; A21 0] x for every member
static int g_stokes_op(Group &g, double *const *x, double *const *y)
{
  const int K = g.K;
  const size_t nu = g.m[0]->nu;
  p3d_op *ops[P3D_GROUP_MAX];
  const double *u[P3D_GROUP_MAX], *p[P3D_GROUP_MAX];
  double *yu[P3D_GROUP_MAX], *yp[P3D_GROUP_MAX];
  for (int k = 0; k < K; k++) {
    ops[k] = g.m[k]->lv.back().op64;
    u[k] = x[k]; p[k] = x[k] + nu; yu[k] = y[k]; yp[k] = y[k] + nu;
  }
  CK(zero_group((void *const *)y, K, g.m[0]->N * 8, g.st));
  return launch_group<double, true, true, true>(ops, K, u, p, yu, yp, g.st, true);
}

// |v_k|^2 of every member into hhost[2hs] (one synchronisation); v given by
// the member's Vptr slot `slot`
static int g_norms2(Group &g, int slot, double *const *v, double *out)
{
  MGroup M;
  memset(&M, 0, sizeof M);
  for (int k = 0; k < g.K; k++) {
    p3d_solver *s = g.m[k];
    M.V[k] = s->Vptr + slot;
    M.w[k] = v[k];
    M.out[k] = s->hdev + 2 * s->hs;
    M.part[k] = s->part;
  }
  vg_mdot(M, g.K, g.m[0]->N, 1, g.st);
  for (int k = 0; k < g.K; k++)
    CU(cudaMemcpyAsync(g.m[k]->hhost + 2 * g.m[k]->hs, g.m[k]->hdev + 2 * g.m[k]->hs, 8, cudaMemcpyDeviceToHost, g.st), "d2h");
  CU(cudaStreamSynchronize(g.st), "sync");
  for (int k = 0; k < g.K; k++) {
    const double ss = g.m[k]->hhost[2 * g.m[k]->hs];
    out[k] = ss > 0.0 ? std::sqrt(ss) : (ss <= 0.0 ? 0.0 : ss);
  }
  return P3D_OK;
}

struct MemberState {
  GroupMember m;
  std::vector<double> H, cs, sn, gv, y;
  double r0 = -1.0, tol = 0.0, rnorm = 0.0, t_join = 0.0;
  int its = 0, gmax = 1; // gmax: the largest membership seen
  bool conv = false;
  int status = P3D_OK;
};

// why solver s cannot share a group with ref (nullptr: it can)
static const char *group_mismatch(const p3d_solver *ref, const p3d_solver *s)
{
  if (s->device != ref->device || s->mesh.mx != ref->mesh.mx || s->mesh.my != ref->mesh.my ||
      s->mesh.mz != ref->mesh.mz || s->mesh.dirichlet != ref->mesh.dirichlet)
    return "differs in device or mesh";
  if (s->o.nlevels != ref->o.nlevels || s->o.cheb_its != ref->o.cheb_its || s->o.mg_precision != ref->o.mg_precision ||
      s->o.restart != ref->o.restart || s->o.max_it != ref->o.max_it || s->o.coarse_op != ref->o.coarse_op)
    return "differs in solver options";
  if (s->o.inner_its > 0 || s->o.inner_rtol > 0.0 || s->lv.size() < 2)
    return "needs one V-cycle per outer iteration and >= 2 levels";
  if (!s->setup_done || !s->rhs_set) return "not set up or without right-hand side";
  return nullptr;
}

// x += sum_{i<j} y_i Z_i for the members given (coefficients uploaded to hdev)
static int g_update_x(cudaStream_t st, const std::vector<MemberState *> &mem, int j, int msize)
{
  if (mem.empty() || j == 0) return P3D_OK;
  MGroup M;
  memset(&M, 0, sizeof M);
  int K = 0;
  for (MemberState *q : mem) {
    p3d_solver *s = q->m.solver;
    for (int i = j - 1; i >= 0; i--) {
      double acc = q->gv[i];
      for (int c = i + 1; c < j; c++) acc -= q->H[(size_t)i * msize + c] * q->y[c];
      q->y[i] = acc / q->H[(size_t)i * msize + i];
    }
    CU(cudaMemcpyAsync(s->hdev, q->y.data(), j * 8, cudaMemcpyHostToDevice, st), "h2d y");
    M.V[K] = s->Zptr;
    M.w[K] = s->xsol;
    M.out[K] = s->hdev;
    K++;
  }
  vg_maxpy(M, K, mem[0]->m.solver->N, j, 1.0, st);
  return cuda_check(cudaStreamSynchronize(st), "x update"); // y (host) must outlive the copy
}

// members leaving: true residual |b - A x|, solution to (u, p), stats, hook
static int g_leave(cudaStream_t st, const std::vector<MemberState *> &out, GroupHooks &hooks)
{
  if (out.empty()) return P3D_OK;
  Group gl;
  gl.st = st;
  double *x[P3D_GROUP_MAX], *w[P3D_GROUP_MAX];
  for (MemberState *q : out) {
    gl.m[gl.K] = q->m.solver;
    x[gl.K] = q->m.solver->xsol;
    w[gl.K] = q->m.solver->w;
    gl.K++;
  }
  const size_t N = gl.m[0]->N;
  CK(g_stokes_op(gl, x, w));
  VGroup<double> V;
  memset(&V, 0, sizeof V);
  for (int k = 0; k < gl.K; k++) { V.v[0][k] = gl.m[k]->bvec; V.v[1][k] = w[k]; V.v[2][k] = w[k]; }
  vg_residual<double>(V, gl.K, N, st);
  double rt[P3D_GROUP_MAX];
  CK(g_norms2(gl, gl.m[0]->hs, w, rt));
  for (int k = 0; k < gl.K; k++) {
    p3d_solver *s = gl.m[k];
    CU(cudaMemcpyAsync(out[k]->m.u, s->xsol, s->nu * 8, cudaMemcpyDeviceToDevice, st), "u out");
    CU(cudaMemcpyAsync(out[k]->m.p, s->xsol + s->nu, s->np * 8, cudaMemcpyDeviceToDevice, st), "p out");
  }
  CU(cudaStreamSynchronize(st), "member out");
  const double t = now_ms();
  for (int k = 0; k < gl.K; k++) {
    p3d_solver *s = gl.m[k];
    MemberState &q = *out[k];
    p3d_solve_stats ss;
    memset(&ss, 0, sizeof ss);
    ss.iterations = q.its;
    ss.r0 = q.r0;
    ss.rfinal = rt[k];
    ss.converged = q.status == P3D_OK && (q.conv || rt[k] <= std::max(s->o.rtol * q.r0, s->o.atol) * 1.0000001);
    ss.setup_ms = s->setup_ms;
    ss.solve_ms = t - q.t_join;
    ss.lmax_fine = s->lv.back().lmax;
    ss.coarse_dofs = s->nc;
    ss.group_members = q.gmax;
    const int sk = q.status != P3D_OK ? q.status : (ss.converged ? P3D_OK : P3D_ERR_NOCONV);
    if (hooks.leave) hooks.leave(q.m, sk, ss);
  }
  return P3D_OK;
}

int solver_group_run(const GroupMember *first, int K0, int max_members, GroupHooks &hooks)
{
  if (!first || K0 < 1 || K0 > P3D_GROUP_MAX) return set_error(P3D_ERR_ARG, "group run: bad arguments");
  max_members = std::max(1, std::min(max_members, P3D_GROUP_MAX));
  const p3d_solver *ref = nullptr; // the shape and options every member must share
  for (int k = 0; k < K0 && !ref; k++) ref = first[k].solver;
  if (!ref) {
    p3d_solve_stats z;
    memset(&z, 0, sizeof z);
    const int rc0 = set_error(P3D_ERR_ARG, "group run: no solver given");
    for (int k = 0; k < K0; k++)
      if (hooks.leave) hooks.leave(first[k], rc0, z);
    return rc0;
  }
  const int msize = ref->o.restart, max_it = ref->o.max_it;
  const size_t N = ref->N;
  cudaSetDevice(ref->device);
  p3d_solve_stats none;
  memset(&none, 0, sizeof none);
  // every member handed to the run leaves exactly once, failures included
  auto leave_all = [&](const GroupMember *m, int n, int status) {
    for (int k = 0; k < n; k++)
      if (hooks.leave) hooks.leave(m[k], status, none);
  };
  cudaStream_t st = nullptr;
  if (int rc0 = cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "group stream")) {
    leave_all(first, K0, rc0);
    return rc0;
  }
  std::vector<std::unique_ptr<MemberState>> act; // members in the group's order
  Group g;
  g.st = st;
  bool dirty = true;
  auto rebuild = [&]() -> int {
    g.K = (int)act.size();
    for (int i = 0; i < g.K; i++) {
      g.m[i] = act[i]->m.solver;
      act[i]->gmax = std::max(act[i]->gmax, g.K);
    }
    dirty = false;
    return g.K ? g_capture(g) : P3D_OK;
  };
  auto join = [&](const GroupMember &gm) -> int {
    const char *why = gm.solver && gm.u && gm.p ? group_mismatch(ref, gm.solver) : "null member";
    if (!why)
      for (auto &q : act)
        if (q->m.solver == gm.solver) why = "solver already in the group";
    if (why) {
      set_error(P3D_ERR_ARG, "group member: %s", why);
      if (hooks.leave) hooks.leave(gm, P3D_ERR_ARG, none);
      return P3D_OK;
    }
    p3d_solver *s = gm.solver;
    auto q = std::make_unique<MemberState>();
    q->m = gm;
    q->H.assign((size_t)(msize + 1) * msize, 0.0);
    q->cs.assign(msize, 0.0);
    q->sn.assign(msize, 0.0);
    q->gv.assign(msize + 1, 0.0);
    q->y.assign(msize, 0.0);
    q->t_join = now_ms();
    // its set-up and right-hand side first; the scratch slot of the basis
    // pointers names the member's w (norms)
    double *w = s->w;
    int rc = cuda_check(cudaStreamSynchronize(s->st), "member sync");
    if (!rc) rc = cuda_check(cudaMemcpyAsync(s->Vptr + s->hs, &w, sizeof(double *), cudaMemcpyHostToDevice, st), "ptr");
    if (!rc) rc = cuda_check(cudaMemcpyAsync(s->xsol, gm.u, s->nu * 8, cudaMemcpyDeviceToDevice, st), "x u");
    if (!rc) rc = cuda_check(cudaMemcpyAsync(s->xsol + s->nu, gm.p, s->np * 8, cudaMemcpyDeviceToDevice, st), "x p");
    if (rc) {
      if (hooks.leave) hooks.leave(gm, rc, none);
      return rc;
    }
    act.push_back(std::move(q));
    dirty = true;
    return P3D_OK;
  };
  // members at positions `idx` of act leave (their x final)
  auto leave = [&](const std::vector<int> &idx) -> int {
    std::vector<MemberState *> out;
    for (int i : idx) out.push_back(act[i].get());
    const int rc = g_leave(st, out, hooks);
    if (rc) return rc; // none of them has left: the failure path below lets them go
    std::vector<std::unique_ptr<MemberState>> keep;
    for (int i = 0; i < (int)act.size(); i++)
      if (std::find(idx.begin(), idx.end(), i) == idx.end()) keep.push_back(std::move(act[i]));
    act = std::move(keep);
    dirty = true;
    return rc;
  };
  int rc = P3D_OK;
  bool started = false;
  GroupMember add[P3D_GROUP_MAX];
  for (;;) {
    // admissions at the start of a restart cycle
    if (!started) {
      for (int k = 0; k < K0; k++) {
        if (rc) {
          leave_all(first + k, 1, rc);
        } else if ((int)act.size() >= max_members) {
          set_error(P3D_ERR_ARG, "group member: the group is full");
          leave_all(first + k, 1, P3D_ERR_ARG);
        } else {
          rc = join(first[k]);
        }
      }
      started = true;
    } else if (hooks.admit && (int)act.size() < max_members) {
      const int n = hooks.admit(max_members - (int)act.size(), add);
      for (int k = 0; k < n; k++) {
        if (rc) leave_all(add + k, 1, rc);
        else rc = join(add[k]);
      }
    }
    if (rc || act.empty()) break;
    if (dirty && (rc = rebuild())) break;
    // r = b - A x into V_0 of every member, |r|
    double *x[P3D_GROUP_MAX], *w[P3D_GROUP_MAX], *v0[P3D_GROUP_MAX];
    for (int i = 0; i < g.K; i++) { x[i] = g.m[i]->xsol; w[i] = g.m[i]->w; v0[i] = g.m[i]->V; }
    if ((rc = g_stokes_op(g, x, w))) break;
    VGroup<double> V;
    memset(&V, 0, sizeof V);
    for (int i = 0; i < g.K; i++) { V.v[0][i] = g.m[i]->bvec; V.v[1][i] = w[i]; V.v[2][i] = v0[i]; }
    vg_residual<double>(V, g.K, N, st);
    double beta[P3D_GROUP_MAX];
    if ((rc = g_norms2(g, 0, v0, beta))) break;
    std::vector<int> out;
    for (int i = 0; i < g.K; i++) {
      MemberState &q = *act[i];
      if (q.r0 < 0) q.r0 = beta[i];
      q.rnorm = beta[i];
      q.tol = std::max(g.m[i]->o.rtol * q.r0, g.m[i]->o.atol);
      if (!std::isfinite(beta[i])) {
        q.status = set_error(P3D_ERR_BREAKDOWN, "FGMRES: non-finite residual");
        out.push_back(i);
      } else if (beta[i] <= q.tol) {
        q.conv = true;
        out.push_back(i);
      } else if (q.its >= max_it) {
        out.push_back(i); // iteration limit: not converged
      } else if (g.m[i]->cancel && g.m[i]->cancel->load(std::memory_order_relaxed)) {
        q.status = P3D_ERR_CANCELLED;
        out.push_back(i);
      }
    }
    if (!out.empty()) {
      if ((rc = leave(out))) break;
      continue; // admissions, then the residuals of the new membership
    }
    for (int i = 0; i < g.K; i++) {
      V.v[0][i] = v0[i]; V.v[1][i] = v0[i]; V.s[0][i] = 1.0 / beta[i]; V.s[1][i] = 0.0;
      MemberState &q = *act[i];
      std::fill(q.gv.begin(), q.gv.end(), 0.0);
      q.gv[0] = beta[i];
    }
    vg_axpby<double>(V, g.K, N, st); // V_0 /= beta
    int j = 0;
    for (; j < msize && !act.empty(); j++) {
      // z_j = PC v_j (grouped graph), w = A z_j
      for (int i = 0; i < g.K; i++) {
        V.v[0][i] = g.m[i]->V + (size_t)j * N; V.v[1][i] = g.m[i]->pc_in; V.s[0][i] = 1.0; V.s[1][i] = 0.0;
      }
      vg_axpby<double>(V, g.K, N, st);
      if ((rc = cuda_check(cudaGraphLaunch(g.gexec, st), "grouped pc graph"))) break;
      count_launch(1);
      double *zj[P3D_GROUP_MAX];
      for (int i = 0; i < g.K; i++) {
        zj[i] = g.m[i]->Z + (size_t)j * N;
        V.v[0][i] = g.m[i]->pc_out; V.v[1][i] = zj[i];
      }
      vg_axpby<double>(V, g.K, N, st);
      for (int i = 0; i < g.K; i++) w[i] = g.m[i]->w;
      if ((rc = g_stokes_op(g, zj, w))) break;
      // classical Gram-Schmidt, first pass with |w|^2; second pass where needed
      MGroup M;
      memset(&M, 0, sizeof M);
      for (int i = 0; i < g.K; i++) {
        p3d_solver *s = g.m[i];
        M.V[i] = s->Vptr; M.w[i] = w[i]; M.out[i] = s->hdev; M.self_out[i] = s->hdev + j + 1; M.part[i] = s->part;
      }
      vg_mdot(M, g.K, N, j + 1, st);
      vg_maxpy(M, g.K, N, j + 1, -1.0, st);
      for (int i = 0; i < g.K && !rc; i++)
        rc = cuda_check(cudaMemcpyAsync(g.m[i]->hhost, g.m[i]->hdev, (j + 2) * 8, cudaMemcpyDeviceToHost, st), "d2h");
      if (rc || (rc = cuda_check(cudaStreamSynchronize(st), "sync"))) break;
      double hn[P3D_GROUP_MAX];
      bool second[P3D_GROUP_MAX];
      int nsecond = 0;
      for (int i = 0; i < g.K; i++) {
        MemberState &q = *act[i];
        double hh = 0.0;
        for (int c = 0; c <= j; c++) {
          q.H[(size_t)c * msize + j] = g.m[i]->hhost[c];
          hh += g.m[i]->hhost[c] * g.m[i]->hhost[c];
        }
        const double wb2 = g.m[i]->hhost[j + 1];
        second[i] = !(wb2 - hh > 0.5 * wb2);
        if (!second[i]) hn[i] = std::sqrt(wb2 - hh);
        nsecond += second[i];
      }
      if (nsecond) {
        MGroup M2;
        memset(&M2, 0, sizeof M2);
        int K2 = 0;
        double *w2[P3D_GROUP_MAX];
        Group g2; // the members that need the second pass
        g2.st = st;
        for (int i = 0; i < g.K; i++)
          if (second[i]) {
            p3d_solver *s = g.m[i];
            M2.V[K2] = s->Vptr; M2.w[K2] = w[i]; M2.out[K2] = s->hdev + s->hs; M2.part[K2] = s->part;
            g2.m[K2] = s; w2[K2] = w[i];
            K2++;
          }
        g2.K = K2;
        vg_mdot(M2, K2, N, j + 1, st);
        vg_maxpy(M2, K2, N, j + 1, -1.0, st);
        for (int q = 0; q < K2 && !rc; q++)
          rc = cuda_check(cudaMemcpyAsync(g2.m[q]->hhost + g2.m[q]->hs, g2.m[q]->hdev + g2.m[q]->hs, (j + 1) * 8,
                                          cudaMemcpyDeviceToHost, st), "d2h");
        if (rc) break;
        double n2[P3D_GROUP_MAX];
        if ((rc = g_norms2(g2, g2.m[0]->hs, w2, n2))) break; // synchronizes
        for (int i = 0, q = 0; i < g.K; i++)
          if (second[i]) {
            MemberState &ms = *act[i];
            for (int c = 0; c <= j; c++) ms.H[(size_t)c * msize + j] += g.m[i]->hhost[g.m[i]->hs + c];
            hn[i] = n2[q++];
          }
      }
      // v_{j+1} = w / hn, Givens rotations, residual estimates
      std::vector<int> fin; // members whose solve ends here
      for (int i = 0; i < g.K; i++) {
        MemberState &q = *act[i];
        std::vector<double> &H = q.H;
        H[(size_t)(j + 1) * msize + j] = hn[i];
        V.v[0][i] = w[i]; V.v[1][i] = g.m[i]->V + (size_t)(j + 1) * N; V.s[0][i] = hn[i] > 0 ? 1.0 / hn[i] : 0.0;
        V.s[1][i] = 0.0;
        for (int c = 0; c < j; c++) {
          const double a = H[(size_t)c * msize + j], b = H[(size_t)(c + 1) * msize + j];
          H[(size_t)c * msize + j] = q.cs[c] * a + q.sn[c] * b;
          H[(size_t)(c + 1) * msize + j] = -q.sn[c] * a + q.cs[c] * b;
        }
        const double a = H[(size_t)j * msize + j], b = H[(size_t)(j + 1) * msize + j];
        const double rr = std::hypot(a, b);
        q.cs[j] = rr > 0 ? a / rr : 1.0;
        q.sn[j] = rr > 0 ? b / rr : 0.0;
        H[(size_t)j * msize + j] = rr;
        H[(size_t)(j + 1) * msize + j] = 0.0;
        q.gv[j + 1] = -q.sn[j] * q.gv[j];
        q.gv[j] = q.cs[j] * q.gv[j];
        q.rnorm = std::fabs(q.gv[j + 1]);
        q.its++;
        if (!std::isfinite(q.rnorm)) {
          q.status = set_error(P3D_ERR_BREAKDOWN, "FGMRES: non-finite residual estimate");
          fin.push_back(i);
        } else if (q.rnorm <= q.tol || hn[i] == 0.0) {
          q.conv = q.rnorm <= q.tol;
          fin.push_back(i);
        } else if (q.its >= max_it) {
          fin.push_back(i);
        } else if (g.m[i]->cancel && g.m[i]->cancel->load(std::memory_order_relaxed)) {
          q.status = P3D_ERR_CANCELLED; // keeps the iterate reached
          fin.push_back(i);
        }
      }
      vg_axpby<double>(V, g.K, N, st);
      if (!fin.empty()) {
        // finished members: x += Z y over their j + 1 directions, then they
        // leave (a member that broke down keeps its iterate)
        std::vector<MemberState *> upd;
        for (int i : fin)
          if (act[i]->status == P3D_OK || act[i]->status == P3D_ERR_CANCELLED) upd.push_back(act[i].get());
        if ((rc = g_update_x(st, upd, j + 1, msize))) break;
        if ((rc = leave(fin))) break;
        if (act.empty()) break;
        if ((rc = rebuild())) break;
      }
    }
    if (rc) break;
    if (act.empty()) continue; // every member left during the cycle: admissions
    // end of the cycle (restart): x += Z y for the rest
    std::vector<MemberState *> all;
    for (auto &q : act) all.push_back(q.get());
    if ((rc = g_update_x(st, all, j, msize))) break;
  }
  g_release_graph(g);
  if (rc) {
    // a CUDA failure: the members still in the group leave with it
    for (auto &q : act)
      if (hooks.leave) hooks.leave(q->m, rc, none);
    act.clear();
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return rc;
}

int solver_group_solve(p3d_solver *const *solvers, int K, double *const *u, double *const *p, p3d_solve_stats *stats,
                       int *status)
{
  if (!solvers || !u || !p || !stats || K < 1 || K > P3D_GROUP_MAX)
    return set_error(P3D_ERR_ARG, "group solve: bad arguments");
  for (int k = 0; k < K; k++) {
    p3d_solver *s = solvers[k];
    if (!s || !u[k] || !p[k]) return set_error(P3D_ERR_ARG, "group solve: null member %d", k);
    if (const char *why = group_mismatch(solvers[0], s)) return set_error(P3D_ERR_ARG, "group solve: member %d %s", k, why);
    for (int q = 0; q < k; q++)
      if (solvers[q] == s) return set_error(P3D_ERR_ARG, "group solve: solver %d given twice", k);
  }
  GroupMember mem[P3D_GROUP_MAX];
  int sk[P3D_GROUP_MAX];
  for (int k = 0; k < K; k++) {
    mem[k].solver = solvers[k];
    mem[k].u = u[k];
    mem[k].p = p[k];
    mem[k].tag = reinterpret_cast<void *>((intptr_t)k);
    memset(&stats[k], 0, sizeof stats[k]);
    sk[k] = P3D_ERR_CUDA;
  }
  GroupHooks h;
  h.leave = [&](const GroupMember &m, int s, const p3d_solve_stats &st) {
    const int k = (int)reinterpret_cast<intptr_t>(m.tag);
    stats[k] = st;
    sk[k] = s;
  };
  const int rc = solver_group_run(mem, K, K, h);
  int worst = P3D_OK;
  for (int k = 0; k < K; k++) {
    if (status) status[k] = sk[k];
    if (sk[k] != P3D_OK && (worst == P3D_OK || worst == P3D_ERR_NOCONV)) worst = sk[k];
  }
  return rc ? rc : worst;
}

} // namespace p3d

using namespace p3d;

extern "C" {

int p3d_solver_solve_grouped(p3d_solver *const solvers[], int32_t k, double *const u[], double *const p[],
                             p3d_solve_stats stats[], int32_t status[])
{
  if (!solvers || !u || !p || !stats || k < 1 || k > P3D_GROUP_MAX)
    return set_error(P3D_ERR_ARG, "solve_grouped: bad arguments");
  for (int i = 0; i < k; i++)
    if (!solvers[i]) return set_error(P3D_ERR_ARG, "solve_grouped: null solver %d", i);
  cudaSetDevice(solvers[0]->device);
  CK(order_after_caller());
  return solver_group_solve(solvers, k, u, p, stats, status);
}

} // extern "C"

namespace p3d {
} // namespace p3d

using namespace p3d;

extern "C" {

int p3d_solver_default_opts(p3d_solver_opts *o)
{
  if (!o) return set_error(P3D_ERR_ARG, "null opts");
  o->nlevels = 4;
  o->cheb_its = 3;
  o->cheb_lo = 0.2;
  o->cheb_hi = 1.1;
  o->esteig_its = 10;
  o->mg_precision = P3D_PREC_F64;
  o->restart = 30;
  o->max_it = 200;
  o->rtol = 1e-6;
  o->atol = 0.0;
  o->use_graph = 1;
  o->verbose = 0;
  o->inner_its = 0;
  o->inner_rtol = 0.0;
  o->coarse_op = P3D_COARSE_GALERKIN;
  o->schur_eta = P3D_SCHUR_ETA_QP;
  o->coarse_eta = P3D_COARSE_ETA_GEOMEAN;
  return P3D_OK;
}

int p3d_solver_estimate_bytes(const p3d_mesh_desc *mesh, const p3d_solver_opts *opts, int64_t *bytes)
{
  if (!mesh || !bytes) return set_error(P3D_ERR_ARG, "estimate_bytes: null argument");
  p3d_solver_opts o;
  if (opts) o = *opts;
  else p3d_solver_default_opts(&o);
  if (o.nlevels < 1 || o.nlevels > 12 || o.restart < 1) return set_error(P3D_ERR_ARG, "estimate_bytes: bad options");
  const bool mixed = o.mg_precision == P3D_PREC_F32;
  double total = 0.0;
  const double nnf = (double)(2 * mesh->mx + 1) * (2 * mesh->my + 1) * (2 * mesh->mz + 1);
  const double nu = 3.0 * nnf, np = 4.0 * mesh->mx * mesh->my * mesh->mz, N = nu + np;
  total += 8.0 * ((2.0 * o.restart + 5.0) * N + nu);     // FGMRES basis, rhs, preconditioner buffers, iterate
  total += 8.0 * nu * (o.inner_its > 0 ? 4.0 : 1.0);     // velocity-solve vectors
  for (int l = 0; l < o.nlevels; l++) {
    const int c = 1 << (o.nlevels - 1 - l);
    const double mx = mesh->mx / c, my = mesh->my / c, mz = mesh->mz / c;
    const double nn = (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1), nel = mx * my * mz, nv = 3 * nn;
    total += 8.0 * 6.0 * nv; // work vectors + inverse diagonal
    const bool gal = l < o.nlevels - 1 && o.coarse_op == P3D_COARSE_GALERKIN;
    if (gal) {
      total += 243.0 * nn * (8.0 + (mixed && l > 0 ? 4.0 : 0.0));
    } else {
      total += 8.0 * (3 * nn + 27 * nel);                         // level coordinates + viscosity
      const double op = 3 * nn + 1.2 * (27 + 37 + 13 + 88) * nel; // operator: coords, packed eta, affine data and pressure map, Gauss-point coords
      total += 8.0 * op + (mixed && l > 0 ? 4.0 * op : 0.0);
    }
    if (l == 0) total += 8.0 * (nv * nv + 68 * nv + 1024); // dense coarse inverse and its scratch
    if (l == o.nlevels - 1) total += 8.0 * 16.0 * nel; // Schur blocks
  }
  *bytes = (int64_t)(1.1 * total) + (4 << 20);
  return P3D_OK;
}

int p3d_solver_create(const p3d_mesh_desc *mesh, const p3d_solver_opts *opts, int device, p3d_solver **out)
{
  if (!mesh || !out) return set_error(P3D_ERR_ARG, "solver_create: null argument");
  *out = nullptr;
  p3d_solver_opts o;
  if (opts) o = *opts;
  else p3d_solver_default_opts(&o);
  if (mesh->ox || mesh->oy || mesh->oz || mesh->gx != 2 * mesh->mx + 1 || mesh->gy != 2 * mesh->my + 1 ||
      mesh->gz != 2 * mesh->mz + 1)
    return set_error(P3D_ERR_ARG, "solver_create: the solver takes a whole mesh (no ghost layers)");
  if (o.nlevels < 1 || o.nlevels > 12 || o.restart < 1 || o.restart > P3D_MAX_RESTART || o.max_it < 1 ||
      o.cheb_its < 1 || !(o.cheb_hi > o.cheb_lo) || o.cheb_lo <= 0 || (o.mg_precision != 64 && o.mg_precision != 32) ||
      o.inner_its < 0 || o.inner_its > 1000 || !(o.inner_rtol >= 0.0 && o.inner_rtol < 1.0) ||
      (o.inner_rtol > 0.0 && o.inner_its < 1) || (o.coarse_op != P3D_COARSE_GALERKIN && o.coarse_op != P3D_COARSE_REDISC) ||
      (o.schur_eta != P3D_SCHUR_ETA_QP && o.schur_eta != P3D_SCHUR_ETA_GEOMEAN) ||
      (o.coarse_eta != P3D_COARSE_ETA_GEOMEAN && o.coarse_eta != P3D_COARSE_ETA_Q1))
    return set_error(P3D_ERR_ARG, "solver_create: bad options");
  int f = 1 << (o.nlevels - 1);
  if (mesh->mx % f || mesh->my % f || mesh->mz % f)
    return set_error(P3D_ERR_ARG, "solver_create: %dx%dx%d not divisible by 2^(nlevels-1)=%d", mesh->mx, mesh->my,
                     mesh->mz, f);
  {
    const long long cdofs = 3ll * (2 * (mesh->mx / f) + 1) * (2 * (mesh->my / f) + 1) * (2 * (mesh->mz / f) + 1);
    if (cdofs > P3D_COARSE_MAX_DOFS)
      return set_error(P3D_ERR_ARG, "solver_create: coarse level of %lld dofs exceeds the dense limit %d (add levels)",
                       cdofs, P3D_COARSE_MAX_DOFS);
  }
  CK(cuda_check(cudaSetDevice(device), "cudaSetDevice"));
  p3d_solver *s = new p3d_solver();
  s->mesh = *mesh;
  s->o = o;
  s->device = device;
  int rc = cuda_check(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking), "stream");
  s->lv.resize(o.nlevels);
  for (int l = 0; l < o.nlevels; l++) {
    int c = 1 << (o.nlevels - 1 - l);
    Level &L = s->lv[l];
    L.m[0] = mesh->mx / c; L.m[1] = mesh->my / c; L.m[2] = mesh->mz / c;
    for (int d = 0; d < 3; d++) L.n[d] = 2 * L.m[d] + 1;
    L.nv = 3ull * L.n[0] * L.n[1] * L.n[2];
  }
  Level &F = s->lv.back();
  s->nu = F.nv;
  s->np = 4ull * F.m[0] * F.m[1] * F.m[2];
  s->N = s->nu + s->np;
  const size_t N = s->N;
  const int m = o.restart;
  if (!rc) rc = dev_alloc((void **)&s->V, (size_t)(m + 1) * N * 8, "FGMRES V");
  if (!rc) rc = dev_alloc((void **)&s->Z, (size_t)m * N * 8, "FGMRES Z");
  if (!rc) rc = dev_alloc((void **)&s->w, N * 8, "FGMRES w");
  if (!rc) rc = dev_alloc((void **)&s->bvec, N * 8, "rhs");
  if (!rc) rc = dev_alloc((void **)&s->pc_in, N * 8, "pc in");
  if (!rc) rc = dev_alloc((void **)&s->pc_out, N * 8, "pc out");
  if (!rc) rc = dev_alloc((void **)&s->pc_t, s->nu * 8, "pc t");
  if (!rc) rc = dev_alloc((void **)&s->xsol, N * 8, "solution");
  s->hs = m + 1;
  if (!rc) rc = dev_alloc((void **)&s->Vptr, (size_t)(m + 2) * sizeof(double *), "V ptrs");
  if (!rc) rc = dev_alloc((void **)&s->Zptr, (size_t)m * sizeof(double *), "Z ptrs");
  // partials of the multi-dot kernels, then their ticket counter (zero between launches)
  const size_t npart = (size_t)P3D_MDOT_BLOCKS * (P3D_MDOT_CHUNK + 1) + 2;
  if (!rc) rc = dev_alloc((void **)&s->part, npart * 8, "partials");
  if (!rc) rc = cuda_check(cudaMemset(s->part, 0, npart * 8), "partials");
  if (!rc) rc = dev_alloc((void **)&s->hdev, (size_t)(2 * s->hs + 2) * 8, "h");
  if (!rc) rc = cuda_check(cudaMallocHost((void **)&s->hhost, (size_t)(2 * s->hs + 2) * 8), "pinned h");
  if (!rc) {
    std::vector<double *> ptrs(m + 2, nullptr);
    for (int j = 0; j <= m; j++) ptrs[j] = s->V + (size_t)j * N;
    rc = cuda_check(cudaMemcpy(s->Vptr, ptrs.data(), (m + 2) * sizeof(double *), cudaMemcpyHostToDevice), "ptrs");
    for (int j = 0; j < m; j++) ptrs[j] = s->Z + (size_t)j * N;
    if (!rc) rc = cuda_check(cudaMemcpy(s->Zptr, ptrs.data(), m * sizeof(double *), cudaMemcpyHostToDevice), "ptrs");
  }
  // velocity-solve vectors (sized for FP64; the mixed path uses them as FP32)
  if (!rc) rc = dev_alloc(&s->cg_r, s->nu * 8, "cg r");
  if (!rc && o.inner_its > 0) {
    rc = dev_alloc(&s->cg_z, s->nu * 8, "cg z");
    if (!rc) rc = dev_alloc(&s->cg_p, s->nu * 8, "cg p");
    if (!rc) rc = dev_alloc(&s->cg_q, s->nu * 8, "cg q");
    if (!rc) rc = dev_alloc((void **)&s->cg_ptr, 2 * sizeof(void *), "cg ptrs");
    if (!rc) rc = dev_alloc((void **)&s->cg_sc, CG_NSC * 8, "cg scalars");
    if (!rc) {
      void *ptrs[2] = {s->cg_p, s->cg_r};
      rc = cuda_check(cudaMemcpy(s->cg_ptr, ptrs, sizeof ptrs, cudaMemcpyHostToDevice), "cg ptrs");
    }
    if (!rc) rc = cuda_check(cudaMemset(s->cg_sc, 0, CG_NSC * 8), "cg scalars");
    if (!rc) rc = cuda_check(cudaStreamCreateWithFlags(&s->st_body, cudaStreamNonBlocking), "body stream");
  }
  if (!rc) rc = cuda_check(cudaMemset(s->bvec, 0, N * 8), "rhs zero");
  if (rc) {
    p3d_solver_destroy(s);
    return rc;
  }
  *out = s;
  return P3D_OK;
}

int p3d_solver_setup(p3d_solver *s, const double *coords, const double *eta)
{
  if (!s || !coords || !eta) return set_error(P3D_ERR_ARG, "solver_setup: null argument");
  cudaSetDevice(s->device);
  CK(order_after_caller());
  return solver_setup(s, coords, eta, nullptr);
}

int p3d_solver_setup_nodal(p3d_solver *s, const double *coords, const double *eta, const double *eta_nodes)
{
  if (!s || !coords || !eta || !eta_nodes) return set_error(P3D_ERR_ARG, "solver_setup_nodal: null argument");
  if (s->o.coarse_op != P3D_COARSE_REDISC || s->o.coarse_eta != P3D_COARSE_ETA_Q1 || s->lv.size() < 2)
    return set_error(P3D_ERR_ARG, "solver_setup_nodal: the nodal viscosity feeds only the Q1 coefficient hierarchy "
                                  "(coarse_op P3D_COARSE_REDISC, coarse_eta P3D_COARSE_ETA_Q1, nlevels >= 2)");
  cudaSetDevice(s->device);
  CK(order_after_caller());
  return solver_setup(s, coords, eta, eta_nodes);
}

int p3d_solver_set_rhs_body_force(p3d_solver *s, const double *rho, double gx, double gy, double gz)
{
  if (!s || !rho) return set_error(P3D_ERR_ARG, "set_rhs_body_force: null argument");
  cudaSetDevice(s->device);
  CK(order_after_caller());
  return solver_rhs_body_force_nowait(s, rho, gx, gy, gz);
}

int p3d_solver_set_rhs(p3d_solver *s, const double *bu, const double *bp)
{
  if (!s || !bu || !bp) return set_error(P3D_ERR_ARG, "set_rhs: null argument");
  cudaSetDevice(s->device);
  CK(order_after_caller());
  CU(cudaMemcpyAsync(s->bvec, bu, s->nu * 8, cudaMemcpyDeviceToDevice, s->st), "rhs u");
  CU(cudaMemcpyAsync(s->bvec + s->nu, bp, s->np * 8, cudaMemcpyDeviceToDevice, s->st), "rhs p");
  s->rhs_set = true;
  return cuda_check(cudaStreamSynchronize(s->st), "rhs");
}

int p3d_solver_solve(p3d_solver *s, double *u, double *p, p3d_solve_stats *stats)
{
  if (!s || !u || !p) return set_error(P3D_ERR_ARG, "solve: null argument");
  cudaSetDevice(s->device);
  CK(order_after_caller()); // the initial guess may still be being written on the caller's stream
  return solver_solve_nowait(s, u, p, stats);
}

} // extern "C"

namespace p3d {

int solver_setup_nowait(p3d_solver *s, const double *coords, const double *eta)
{
  if (!s || !coords || !eta) return set_error(P3D_ERR_ARG, "solver_setup: null argument");
  cudaSetDevice(s->device);
  return solver_setup(s, coords, eta, nullptr);
}

int solver_rhs_body_force_nowait(p3d_solver *s, const double *rho, double gx, double gy, double gz)
{
  if (!s || !rho) return set_error(P3D_ERR_ARG, "set_rhs_body_force: null argument");
  if (!s->setup_done) return set_error(P3D_ERR_STATE, "set_rhs_body_force before setup");
  Level &F = s->lv.back();
  CU(cudaMemsetAsync(s->bvec, 0, s->N * 8, s->st), "memset");
  double g[3] = {gx, gy, gz};
  s_body_force(F.m[0], F.m[1], F.m[2], F.coords, rho, g, s->bvec, s->st);
  v_mask<double>(F.n[0], F.n[1], F.n[2], s->mesh.dirichlet, s->bvec, s->st);
  s->rhs_set = true;
  return cuda_check(cudaStreamSynchronize(s->st), "rhs");
}

int solver_solve_nowait(p3d_solver *s, double *u, double *p, p3d_solve_stats *stats)
{
  if (!s || !u || !p) return set_error(P3D_ERR_ARG, "solve: null argument");
  if (!s->setup_done || !s->rhs_set) return set_error(P3D_ERR_STATE, "solve before setup / rhs");
  cudaSetDevice(s->device);
  p3d_solve_stats local;
  memset(&local, 0, sizeof local);
  double t0 = now_ms();
  double *x = s->xsol;
  int rc = cuda_check(cudaMemcpyAsync(x, u, s->nu * 8, cudaMemcpyDeviceToDevice, s->st), "x u");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(x + s->nu, p, s->np * 8, cudaMemcpyDeviceToDevice, s->st), "x p");
  if (!rc && s->cg_sc) rc = cuda_check(cudaMemsetAsync(s->cg_sc + CG_TOTAL, 0, 8, s->st), "inner count");
  bool cancelled = false;
  if (!rc) {
    rc = fgmres(s, x, &local);
    if (rc == P3D_ERR_CANCELLED) { cancelled = true; rc = P3D_OK; }
  }
  if (!rc && s->cg_sc && s->o.inner_rtol > 0.0) {
    double tot = 0.0;
    rc = cuda_check(cudaMemcpyAsync(&tot, s->cg_sc + CG_TOTAL, 8, cudaMemcpyDeviceToHost, s->st), "inner count");
    if (!rc) rc = cuda_check(cudaStreamSynchronize(s->st), "inner count");
    local.inner_iterations = (int32_t)tot;
  }
  if (!rc) rc = cuda_check(cudaMemcpyAsync(u, x, s->nu * 8, cudaMemcpyDeviceToDevice, s->st), "u out");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(p, x + s->nu, s->np * 8, cudaMemcpyDeviceToDevice, s->st), "p out");
  if (!rc) rc = cuda_check(cudaStreamSynchronize(s->st), "solve sync");
  local.solve_ms = now_ms() - t0;
  local.setup_ms = s->setup_ms;
  local.lmax_fine = s->lv.back().lmax;
  local.coarse_dofs = s->nc;
  local.group_members = 1;
  if (stats) *stats = local;
  if (rc) return rc;
  if (cancelled) return set_error(P3D_ERR_CANCELLED, "solve cancelled after %d iterations", local.iterations);
  if (!local.converged) return set_error(P3D_ERR_NOCONV, "FGMRES: %d iterations, |r| %.3e / %.3e", local.iterations,
                                         local.rfinal, local.r0);
  return P3D_OK;
}

} // namespace p3d

extern "C" {

int p3d_solver_apply_pc(p3d_solver *s, const double *ru, const double *rp, double *zu, double *zp)
{
  if (!s || !ru || !rp || !zu || !zp) return set_error(P3D_ERR_ARG, "apply_pc: null argument");
  if (!s->setup_done) return set_error(P3D_ERR_STATE, "apply_pc before setup");
  cudaSetDevice(s->device);
  CK(order_after_caller());
  CU(cudaMemcpyAsync(s->pc_in, ru, s->nu * 8, cudaMemcpyDeviceToDevice, s->st), "copy");
  CU(cudaMemcpyAsync(s->pc_in + s->nu, rp, s->np * 8, cudaMemcpyDeviceToDevice, s->st), "copy");
  CK(run_pc(s, s->pc_in, s->w));
  CU(cudaMemcpyAsync(zu, s->w, s->nu * 8, cudaMemcpyDeviceToDevice, s->st), "copy");
  CU(cudaMemcpyAsync(zp, s->w + s->nu, s->np * 8, cudaMemcpyDeviceToDevice, s->st), "copy");
  return cuda_check(cudaStreamSynchronize(s->st), "apply_pc");
}

int p3d_solver_level_apply(p3d_solver *s, int level, const double *x, double *y)
{
  if (!s || !x || !y) return set_error(P3D_ERR_ARG, "level_apply: null argument");
  if (!s->setup_done) return set_error(P3D_ERR_STATE, "level_apply before setup");
  if (level < 0 || level >= (int)s->lv.size()) return set_error(P3D_ERR_ARG, "level_apply: no level %d", level);
  cudaSetDevice(s->device);
  CK(order_after_caller());
  CK(a11<double>(s, s->lv[level], x, y));
  return cuda_check(cudaStreamSynchronize(s->st), "level_apply");
}

int p3d_solver_destroy(p3d_solver *s)
{
  if (!s) return P3D_OK;
  cudaSetDevice(s->device);
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  if (s->graph) cudaGraphDestroy(s->graph);
  for (auto &L : s->lv) free_level(L);
  for (void *p : {(void *)s->cinv, (void *)s->cb64, (void *)s->cx64, (void *)s->gj, (void *)s->Binv, (void *)s->bvec, (void *)s->V,
                  (void *)s->Z, (void *)s->w, (void *)s->Vptr, (void *)s->Zptr, (void *)s->part, (void *)s->hdev, (void *)s->pc_in,
                  (void *)s->pc_out, (void *)s->pc_t, (void *)s->xsol, s->cg_r, s->cg_z, s->cg_p, s->cg_q, (void *)s->cg_ptr,
                  (void *)s->cg_sc})
    if (p) cudaFree(p);
  if (s->hhost) cudaFreeHost(s->hhost);
  if (s->st_body) cudaStreamDestroy(s->st_body);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
  return P3D_OK;
}

} // extern "C"
