// Internal (non-ABI) declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include "p3d_b200.h"

namespace p3d {
constexpr int NW_AFF = 4; // warp layers per CTA, affine A11 path (40 elements)
constexpr int NW_GEN = 2; // warp layers per CTA, general-geometry paths (20 elements)

int set_error(int code, const char *fmt, ...);
int cuda_check(cudaError_t e, const char *what);
void count_launch(int n);
int dev_alloc(void **p, size_t bytes, const char *what);
// Entry points that read caller device arrays on a library stream first wait
// for all work the caller queued on the device (any stream), so that the
// arrays are complete when the library's copies read them.
int order_after_caller();
} // namespace p3d

struct p3d_op {
  p3d_mesh_desc m;
  int prec = 64;
  int device = 0;
  int bc = 0;
  int geom = 1;
  bool have_coef = false;
  void *coords = nullptr; // [3*gx*gy*gz] in operator precision
  void *kgen = nullptr;   // general path: eta, brick order (NW_GEN)
  void *kgq = nullptr;    // general FP64 path: Gauss-point coordinate table, brick order (NW_GEN)
  void *kaff = nullptr;   // affine path: J^{-1} + eta*w*detJ, brick order (NW_AFF)
  void *kpre = nullptr;   // affine path: pressure-basis map + detJ, brick order (NW_AFF)
  bool aff_exact = false; // every element tested affine: A12/A21 take the affine kernels too
  void *hx = nullptr, *hy = nullptr; // host-apply staging
  unsigned long long *flag = nullptr; // affinity test result (kept: re-setup allocates nothing)
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr; // host-apply copy streams
  cudaEvent_t ev[32] = {};                      // host-apply chunk events (16 chunks x {x in, y done})
  int host_chunks = 0;                           // 0: automatic
  bool host_register = false;                    // page-lock the host arrays p3d_a11_apply_host is given
  int n_reg = 0;                                 // host ranges this operator registered
  void *reg_ptr[16] = {};
  size_t reg_bytes[16] = {};
  void *res_u = nullptr;                         // residual: u with the Dirichlet values inserted
  cudaStream_t stream = nullptr;     // setup / host-apply stream
};

namespace p3d {
// overwrite: y is zero on entry and is not read (y = A x); otherwise y += A x.
// [tzb, tze): range of brick layers along z to apply (tze < 0: all).
template <typename T>
int launch_a11(p3d_op *op, const T *x, T *y, cudaStream_t st, bool overwrite = false, int tzb = 0, int tze = -1);
template <typename T> int launch_diag(p3d_op *op, T *d, cudaStream_t st);
template <typename T, bool DA11, bool DA12, bool DA21>
int launch_general(p3d_op *op, const T *u, const T *p, T *yu, T *yp, cudaStream_t st, bool overwrite = false,
                   int tzb = 0, int tze = -1);
// brick layer height along z of the A11 path the operator uses
int a11_brick_height(const p3d_op *op);
// K operators of one mesh shape, precision, path and mode in one launch
// (u, p, yu, yp: per-member pointers or nullptr); y overwritten when overwrite
template <typename T, bool DA11, bool DA12, bool DA21>
int launch_group(p3d_op *const *ops, int K, const T *const *u, const T *const *p, T *const *yu, T *const *yp,
                 cudaStream_t st, bool overwrite);
// zero K buffers of `bytes` bytes (a multiple of 4) in one launch
int zero_group(void *const *v, int K, size_t bytes, cudaStream_t st);
// coefficient setup from device FP64 arrays on op->stream (no ordering against
// other streams: the caller orders the arrays' producers first)
int op_setup_device(p3d_op *op, const double *coords, const double *eta, int geom_mode);
} // namespace p3d
