// Internal declarations of the solver translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include <atomic>
#include <functional>
#include <stdint.h>

#ifndef P3D_GROUP_MAX
#define P3D_GROUP_MAX 32
#endif
#define P3D_MDOT_CHUNK 8    // vectors per multi-dot / multi-axpy launch (register accumulators)
#define P3D_MDOT_BLOCKS 592 // 4 x 148 SMs

namespace p3d {

// vec_kernels.cu
template <typename A, typename B> void v_convert(size_t n, const A *x, B *y, cudaStream_t s);
template <typename T> void v_axpby(size_t n, T a, const T *x, T b, T *y, cudaStream_t s);
template <typename T> void v_scale(size_t n, T a, T *y, cudaStream_t s);
template <typename T> void v_jacobi(size_t n, const double *dinv, const T *r, T *z, cudaStream_t s);
template <typename T>
void v_cheb_step(size_t n, const double *dinv, T *x, T *r, const T *Ad, T *d, T c1, T c2, bool last, cudaStream_t s);
template <typename T>
void v_cheb_init0(size_t n, const double *dinv, const T *b, T inv_theta, T *x, T *r, T *d, cudaStream_t s);
template <typename T>
void v_cheb_init_res(size_t n, const double *dinv, const T *b, const T *Ax, T inv_theta, T *r, T *d, cudaStream_t s);
template <typename T> void v_residual(size_t n, const T *b, const T *Ax, T *r, cudaStream_t s);
template <typename T> void v_mask(int nx, int ny, int nz, uint32_t dir, T *v, cudaStream_t s);
template <typename T>
void v_mdot(size_t n, int k, const T *const *V_dev, const T *w, double *part, double *out_dev, cudaStream_t s,
            double *self_out = nullptr); // self_out: also w . w
template <typename T> void v_maxpy(size_t n, int k, const double *h, const T *const *V_dev, T *w, double sign, cudaStream_t s);
template <typename T>
void v_cg_xr(size_t n, const double *num, const double *den, T *x, T *r, const T *p, const T *q, bool update_r, cudaStream_t s);
template <typename T> void v_cg_p(size_t n, const double *num, const double *den, const T *z, T *p, cudaStream_t s);
void v_block4(size_t nel, const double *B, const double *x, double *y, double alpha, cudaStream_t s);
void v_invert_diag(size_t n, const double *d, double *dinv, unsigned int *bad, cudaStream_t s);
void v_dense_mv(int n, const double *M, const double *x, double *y, cudaStream_t s);

// vec_kernels.cu, grouped forms: one launch over the K members of a group of
// same-shape solves (blockIdx.y = member); roles of v[] per kernel:
//   cheb_init0   v0 b, v1 x, v2 r, v3 d; s0 1/theta
//   cheb_init_res v0 b, v1 Ax, v2 r, v3 d; s0 1/theta
//   cheb_step    v0 x, v1 r, v2 Ad, v3 d; s0 c1, s1 c2
//   axpby        v0 x, v1 y; s0 a, s1 b (y = a x + b y; y not read when b = 0)
//   residual     v0 b, v1 Ax, v2 r
//   convert      v0 in, v1 out (raw pointers)
//   block4       v0 B, v1 x, v2 y;  dense_mv v0 M, v1 x, v2 y
template <typename T> struct VGroup {
  T *v[4][P3D_GROUP_MAX];
  const double *dinv[P3D_GROUP_MAX];
  double s[2][P3D_GROUP_MAX];
};
// Gram-Schmidt per member: V[m] its basis (device array of vector pointers),
// w[m] the vector, out[m] the coefficients (device), self_out[m] |w|^2 or
// nullptr, part[m] its partials buffer and ticket
struct MGroup {
  double *const *V[P3D_GROUP_MAX];
  double *w[P3D_GROUP_MAX];
  double *out[P3D_GROUP_MAX];
  double *self_out[P3D_GROUP_MAX];
  double *part[P3D_GROUP_MAX];
};
template <typename T> void vg_cheb_init0(const VGroup<T> &G, int K, size_t n, cudaStream_t s);
template <typename T> void vg_cheb_init_res(const VGroup<T> &G, int K, size_t n, cudaStream_t s);
template <typename T> void vg_cheb_step(const VGroup<T> &G, int K, size_t n, bool last, cudaStream_t s);
template <typename T> void vg_axpby(const VGroup<T> &G, int K, size_t n, cudaStream_t s);
template <typename T> void vg_residual(const VGroup<T> &G, int K, size_t n, cudaStream_t s);
template <typename A, typename B> void vg_convert(const VGroup<double> &G, int K, size_t n, cudaStream_t s);
void vg_block4(const VGroup<double> &G, int K, size_t nel, cudaStream_t s);
void vg_dense_mv(const VGroup<double> &G, int K, int n, cudaStream_t s);
void vg_mdot(const MGroup &G, int K, size_t n, int k, cudaStream_t s);
void vg_maxpy(const MGroup &G, int K, size_t n, int k, double sign, cudaStream_t s);
// per-member operands of the grouped transfers and stencil applies
template <typename T> struct TGroup {
  const T *a[P3D_GROUP_MAX];
  const T *b[P3D_GROUP_MAX];
  T *out[P3D_GROUP_MAX];
};
// mg_transfer.cu: restrict_residual (a = b, b = Ax, out = xc), prolong_add (a = xc, out = xf)
template <typename T>
int mg_restrict_residual_group(const TGroup<T> &G, int K, int cnx, int cny, int cnz, uint32_t dir, cudaStream_t st);
template <typename T>
int mg_prolong_add_group(const TGroup<T> &G, int K, int cnx, int cny, int cnz, uint32_t dir, cudaStream_t st);
// galerkin.cu: y = G x per member (a = G, b = x, out = y)
template <typename T> void g_apply_group(const TGroup<T> &P, int K, int nx, int ny, int nz, cudaStream_t s);

// setup_kernels.cu (whole-mesh lattices, FP64)
void s_schur_blocks(int mx, int my, int mz, const double *coords, const double *eta, int geomean, double *Binv,
                    cudaStream_t s);
void s_body_force(int mx, int my, int mz, const double *coords, const double *rho, double g[3], double *bu, cudaStream_t s);
void s_restrict_eta(int mxc, int myc, int mzc, const double *eta_f, double *eta_c, cudaStream_t s);
void s_eta_project(int mx, int my, int mz, const double *eta, double *A, double *B, cudaStream_t s);
void s_divide(size_t n, double *a, const double *b, cudaStream_t s);
void s_fill(size_t n, double v, double *a, cudaStream_t s);
void s_force_u(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, const double *coords, const double *fu,
               double *ru, cudaStream_t s);
void s_force_p(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, const double *coords, const double *fp,
               double *rp, cudaStream_t s);
void s_eta_to_qp(int mx, int my, int mz, const double *v, double *eta, cudaStream_t s);
void s_inject_coords(int cnx, int cny, int cnz, const double *cf, double *cc, cudaStream_t s);

// galerkin.cu (27-point block-stencil coarse operators)
template <typename T> void g_apply(int nx, int ny, int nz, const T *G, const T *x, T *y, cudaStream_t s);
void g_probe_vec(int nx, int ny, int nz, int ci, int cj, int ck, int d, uint32_t dir, double *x, cudaStream_t s);
void g_probe_scatter(int nx, int ny, int nz, int ci, int cj, int ck, int d, const double *y, double *G, cudaStream_t s);
void g_dirichlet(int nx, int ny, int nz, uint32_t dir, double *G, cudaStream_t s);
void g_diag(int nx, int ny, int nz, const double *G, double *d, cudaStream_t s);
void g_dense(int nx, int ny, int nz, const double *G, double *M, cudaStream_t s);

// stokes_solver.cu: the solver entry points without the wait for the
// caller's device work (the server orders its own copies first)
} // namespace p3d
struct p3d_solver;
namespace p3d {
int solver_setup_nowait(p3d_solver *s, const double *coords, const double *eta);
int solver_rhs_body_force_nowait(p3d_solver *s, const double *rho, double gx, double gy, double gz);
int solver_solve_nowait(p3d_solver *s, double *u, double *p, struct p3d_solve_stats *stats);
// a flag the outer iteration reads between iterations: non-zero ends the
// solve with P3D_ERR_CANCELLED (u, p the iterate reached); nullptr: none
void solver_set_cancel_flag(p3d_solver *s, const std::atomic<int> *flag);
// lock-step solve of K same-shape solvers (set up, right-hand sides set);
// u, p: device initial guesses in, solutions out; stats per member.  Returns
// P3D_OK when all converged, else a failure's status; status[k] (may be
// nullptr) per member: P3D_OK, P3D_ERR_NOCONV, _BREAKDOWN or _CANCELLED.
int solver_group_solve(p3d_solver *const *solvers, int K, double *const *u, double *const *p,
                       struct p3d_solve_stats *stats, int *status);
// A rolling group: members join at the start of a restart cycle and leave as
// soon as they finish, the others going on.  A member is a solver (set up,
// right-hand side set) with device arrays u, p (initial guess in, solution
// out) and a caller's tag.
struct GroupMember {
  p3d_solver *solver = nullptr;
  double *u = nullptr, *p = nullptr;
  void *tag = nullptr;
};
struct GroupHooks {
  // start of every restart cycle: writes up to `room` new members to `add`
  // and returns their count (nullptr: no one joins)
  std::function<int(int room, GroupMember *add)> admit;
  // a member left (its u, p written; stats filled): P3D_OK, P3D_ERR_NOCONV,
  // _BREAKDOWN, _CANCELLED, or P3D_ERR_ARG when it could not join
  std::function<void(const GroupMember &m, int status, const struct p3d_solve_stats &st)> leave;
};
// runs until no member is left and none joins; the members' solvers must
// share the mesh and options (checked; a mismatching joiner leaves with
// P3D_ERR_ARG).  Returns P3D_OK or a CUDA failure (after which every member
// still in the group has left with that status).
int solver_group_run(const GroupMember *first, int K, int max_members, GroupHooks &hooks);

// dense_inverse.cu (coarse-grid operator, in place, blocked Gauss-Jordan)
size_t dense_inverse_scratch(int n);
int dense_inverse_spd(int n, double *A, double *scratch, cudaStream_t s);

// mg_transfer.cu
template <typename T> int mg_prolong(int cnx, int cny, int cnz, int ndof, const T *xc, T *xf, cudaStream_t st);
template <typename T> int mg_restrict(int cnx, int cny, int cnz, int ndof, const T *xf, T *xc, cudaStream_t st);
// velocity V-cycle transfers with the Dirichlet mask dir fused in:
// xc = mask(P^T mask(b - Ax)) and xf += mask(P xc)
template <typename T>
int mg_restrict_residual(int cnx, int cny, int cnz, uint32_t dir, const T *b, const T *Ax, T *xc, cudaStream_t st);
template <typename T> int mg_prolong_add(int cnx, int cny, int cnz, uint32_t dir, const T *xc, T *xf, cudaStream_t st);

} // namespace p3d
