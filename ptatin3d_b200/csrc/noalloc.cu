// Host-buffer A11 apply that allocates no device memory.
//
// p3d_a11_apply_host stages x and y through device buffers it allocates on
// first use.  Some callers cannot allow that: a PETSc MatShell callback that
// runs while the application owns the whole device memory pool, or inside
// code that must not call cudaMalloc/cudaFree (they synchronise the device
// and may fail or stall under a capped or externally managed allocator).
// p3d_a11_apply_host_noalloc does the same work with its staging in a fixed
// file-scope __device__ array, sized for meshes up to P3D_NOALLOC_MAX_DOFS
// velocity dofs (the 16^3-element Q2 mesh: 3*33^3 = 107,811 dofs).
//
// The array exists once per device that loads this library and stays
// resident until the process exits.  Its device address is obtained with
// cudaGetSymbolAddress the first time the entry point runs on a device (with
// that device current); that first call should therefore come before any CUDA
// stream capture.  The address is kept for the life of the device's primary
// context: a caller that resets the device (cudaDeviceReset) must not use this
// entry point afterwards in the same process.  All calls on a device share the one array, so calls whose
// work overlaps on the GPU (other host threads, other streams) race; the
// entry point itself is synchronous.
#include <cuda_runtime.h>

#include <mutex>

#include "p3d_b200.h"
#include "p3d_internal.h"

#define P3D_NOALLOC_MAX_DEVICES 64

namespace p3d {

// x staging [0, MAX) and y staging [MAX, 2*MAX)
static __device__ __align__(256) double g_noalloc_scratch[2 * P3D_NOALLOC_MAX_DOFS];

static std::mutex g_noalloc_mu;
static double *g_noalloc_addr[P3D_NOALLOC_MAX_DEVICES] = {nullptr};

// device address of the static scratch on the current device (set up once per device)
static int noalloc_scratch(int device, double **out)
{
  if (device < 0 || device >= P3D_NOALLOC_MAX_DEVICES) return set_error(P3D_ERR_ARG, "noalloc: device %d", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_check(e, "cudaGetSymbolAddress(noalloc scratch)");
    g_noalloc_addr[device] = (double *)p;
  }
  *out = g_noalloc_addr[device];
  return P3D_OK;
}

} // namespace p3d

using namespace p3d;

extern "C" int p3d_a11_apply_host_noalloc(p3d_op *op, const double *x_host, double *y_host)
{
  if (!op) return set_error(P3D_ERR_ARG, "a11_apply_host_noalloc: null operator");
  if (!op->have_coef) return set_error(P3D_ERR_STATE, "operator coefficients not set");
  if (!x_host || !y_host) return set_error(P3D_ERR_ARG, "a11_apply_host_noalloc: null vector");
  if (op->prec != P3D_PREC_F64) return set_error(P3D_ERR_ARG, "a11_apply_host_noalloc: FP64 operators only");
  const size_t n = 3ull * op->m.gx * op->m.gy * op->m.gz;
  if (n > (size_t)P3D_NOALLOC_MAX_DOFS)
    return set_error(P3D_ERR_ARG, "a11_apply_host_noalloc: %zu velocity dofs exceed the static limit %d", n,
                     (int)P3D_NOALLOC_MAX_DOFS);
  int rc = cuda_check(cudaSetDevice(op->device), "cudaSetDevice");
  if (rc) return rc;
  double *scr = nullptr;
  if ((rc = noalloc_scratch(op->device, &scr))) return rc;
  double *dx = scr, *dy = scr + P3D_NOALLOC_MAX_DOFS;
  cudaStream_t st = op->stream;
  if ((rc = cuda_check(cudaMemcpyAsync(dx, x_host, n * 8, cudaMemcpyHostToDevice, st), "H2D x"))) return rc;
  // the array keeps the previous call's contents: y must start at zero (nodes
  // on brick faces are accumulated atomically; the rest are stored, y = A x)
  if ((rc = cuda_check(cudaMemsetAsync(dy, 0, n * 8, st), "zero y"))) return rc;
  if ((rc = launch_a11<double>(op, dx, dy, st, true))) return rc;
  if ((rc = cuda_check(cudaMemcpyAsync(y_host, dy, n * 8, cudaMemcpyDeviceToHost, st), "D2H y"))) return rc;
  return cuda_check(cudaStreamSynchronize(st), "noalloc apply sync");
}
