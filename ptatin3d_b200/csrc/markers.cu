// Material-point coefficients onto the Gauss points: the projection types of
// the reference's rheology update (src/rheology.c:150-185), on the device.
//
//   P0, arithmetic / harmonic / geometric viscosity average, arithmetic density
//       (MPntPStokesProj_P0 -> _LocalP0Projection_MPntPStokes_MapToQuadratePoints,
//        src/material_point_utils.c:2567-2808)
//   Q1  corner-weighted nodal average on the Q2 node lattice, clamped Q1
//       interpolation back to the Gauss points
//       (_SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes, :604-801)
//   one-to-one: marker p is Gauss point p (SwarmUpdateGaussPropertiesOne2OneMap_MPntPStokes, :803-840)
//
// Markers scatter with FP64 atomics: one thread per marker into three sums
// per element for P0; for Q1, warps sum the contributions of each run of
// markers of one element before one atomic per node and field.  A second pass per
// element (P0) or per node then per element (Q1) finishes.  The atomic sums
// differ from the reference's marker-order sums by rounding only.
#include <cuda_runtime.h>
#include <stdint.h>

#include "p3d_internal.h"
#include "solver_internal.h"

namespace p3d {
namespace {

int mgrid(size_t n)
{
  size_t g = (n + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  return g < 1 ? 1 : (int)g;
}

// Q1 corner weight 0.125 (1 -+ xi)(1 -+ eta)(1 -+ zeta); corner bits (x, y, z)
// (pTatinConstructNI_Q1_3D, src/material_point_utils.c:502-519)
__device__ __forceinline__ double q1_corner(int corner, double x0, double x1, double x2)
{
  return 0.125 * ((corner & 1) ? 1.0 + x0 : 1.0 - x0) * ((corner & 2) ? 1.0 + x1 : 1.0 - x1) *
         ((corner & 4) ? 1.0 + x2 : 1.0 - x2);
}

// S[3e] += f(eta_p), S[3e+1] += 1, S[3e+2] += rho_p for every marker in element e
__global__ void k_p0_scatter(int64_t n, int64_t nel, int type, const int32_t *__restrict__ wil,
                             const double *__restrict__ eta_p, const double *__restrict__ rho_p, double *__restrict__ S)
{
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = wil[p];
    if (e < 0 || e >= nel) continue;
    const double v = eta_p[p];
    const double f = type == P3D_PROJ_P0_HARMONIC ? 1.0 / v : (type == P3D_PROJ_P0_GEOMETRIC ? log(v) : v);
    atomicAdd(S + 3 * e, f);
    atomicAdd(S + 3 * e + 1, 1.0);
    atomicAdd(S + 3 * e + 2, rho_p[p]);
  }
}

// the element's average on all 27 of its Gauss points (an element without
// markers gets 0/0, as in the reference)
__global__ void k_p0_finish(int64_t nel, int type, const double *__restrict__ S, double *__restrict__ eta_q,
                            double *__restrict__ rho_q)
{
  const int64_t nq = 27 * nel;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nq; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = i / 27;
    const double s = S[3 * e], c = S[3 * e + 1];
    eta_q[i] = type == P3D_PROJ_P0_HARMONIC ? c / s : (type == P3D_PROJ_P0_GEOMETRIC ? exp(s / c) : s / c);
    rho_q[i] = S[3 * e + 2] / c;
  }
}

// A1 += N eta_p, A2 += N rho_p, B += N over the 27 nodes of the marker's
// element (Q1 weights at the 8 corners, weight 1 at the other 19 Q2 nodes),
// aggregated per warp.  A warp takes 32 consecutive markers;
// consecutive markers of one element (the reference lays new markers out
// element by element) form a segment.  Lane j < 27 owns node j of the
// element: it walks the warp's markers in order, adds each one's weighted
// eta, rho and weight for its node, and at the end of every segment adds the
// three sums to the lattice with one atomic each.  81 atomics per segment
// replace 81 per marker (8x fewer with the reference's 2^3 lattice).  Any
// order of markers is correct: a segment is a run of equal elements, so an
// element split over several runs just flushes once per run.
constexpr int Q1W = 8; // warps per block
__global__ void __launch_bounds__(32 * Q1W) k_q1_scatter_warp(int64_t n, int mx, int my, int mz,
                                                              const int32_t *__restrict__ wil,
                                                              const double *__restrict__ xi,
                                                              const double *__restrict__ eta_p,
                                                              const double *__restrict__ rho_p, double *__restrict__ A1,
                                                              double *__restrict__ A2, double *__restrict__ B)
{
  __shared__ double s_v[Q1W][5][32]; // xi0, xi1, xi2, eta, rho of the warp's markers
  __shared__ int64_t s_e[Q1W][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t nel = (int64_t)mx * my * mz, nx = 2 * (int64_t)mx + 1, ny = 2 * (int64_t)my + 1;
  // node j of the element (lanes 27..31 have none)
  const int a = lane % 3, b = (lane / 3) % 3, c = lane / 9;
  const bool corner = lane < 27 && a != 1 && b != 1 && c != 1;
  const int cbits = (a >> 1) | (b & 2) | ((c >> 1) << 2);
  const int64_t nwarps = (int64_t)gridDim.x * Q1W;
  for (int64_t base = ((int64_t)blockIdx.x * Q1W + w) * 32; base < n; base += nwarps * 32) {
    const int64_t p = base + lane;
    int64_t e = -1;
    if (p < n) {
      e = wil[p];
      if (e < 0 || e >= nel) e = -1;
      s_v[w][0][lane] = xi[3 * p];
      s_v[w][1][lane] = xi[3 * p + 1];
      s_v[w][2][lane] = xi[3 * p + 2];
      s_v[w][3][lane] = eta_p[p];
      s_v[w][4][lane] = rho_p[p];
    }
    s_e[w][lane] = e;
    // bit l: marker l ends a segment (the next one belongs to another element, or l is the last)
    const int64_t e_next = __shfl_down_sync(0xffffffffu, e, 1);
    const unsigned last = __ballot_sync(0xffffffffu, lane == 31 || e_next != e);
    __syncwarp();
    double s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int l = 0; l < 32; l++) {
      const int64_t el = s_e[w][l];
      if (el >= 0) {
        const double x0 = s_v[w][0][l], x1 = s_v[w][1][l], x2 = s_v[w][2][l];
        const double wt = corner ? q1_corner(cbits, x0, x1, x2) : 1.0;
        s1 += wt * s_v[w][3][l];
        s2 += wt * s_v[w][4][l];
        s3 += wt;
      }
      if ((last >> l) & 1u) {
        if (el >= 0 && lane < 27) {
          const int64_t ex = el % mx, ey = (el / mx) % my, ez = el / ((int64_t)mx * my);
          const int64_t g = (2 * ex + a) + nx * ((2 * ey + b) + ny * (2 * ez + c));
          atomicAdd(A1 + g, s1);
          atomicAdd(A2 + g, s2);
          atomicAdd(B + g, s3);
        }
        s1 = s2 = s3 = 0.0;
      }
    }
    __syncwarp(); // the shared slots are rewritten by the next chunk
  }
}

// A1 /= B, A2 /= B, with 0 where B is 0 (the convention of PETSc's
// VecPointwiseDivide, which the reference calls here)
__global__ void k_q1_divide(int64_t nn, double *__restrict__ A1, double *__restrict__ A2, const double *__restrict__ B)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
    const double b = B[i];
    A1[i] = b != 0.0 ? A1[i] / b : 0.0;
    A2[i] = b != 0.0 ? A2[i] / b : 0.0;
  }
}

bool valid_type(int t)
{
  return t == P3D_PROJ_NULL || t == P3D_PROJ_P0_ARITHMETIC || t == P3D_PROJ_P0_HARMONIC ||
         t == P3D_PROJ_P0_GEOMETRIC || t == P3D_PROJ_Q1 || t == P3D_PROJ_ONE2ONE;
}

int64_t workspace_bytes(int32_t mx, int32_t my, int32_t mz, int type)
{
  const int64_t nel = (int64_t)mx * my * mz;
  const int64_t nn = (2 * (int64_t)mx + 1) * (2 * (int64_t)my + 1) * (2 * (int64_t)mz + 1);
  if (type == P3D_PROJ_Q1) return 3 * nn * 8;
  if (type == P3D_PROJ_P0_ARITHMETIC || type == P3D_PROJ_P0_HARMONIC || type == P3D_PROJ_P0_GEOMETRIC)
    return 3 * nel * 8;
  return 0;
}

} // namespace
} // namespace p3d

using namespace p3d;

int p3d_marker_project_workspace(int32_t mx, int32_t my, int32_t mz, int type, int64_t *bytes)
{
  if (mx < 1 || my < 1 || mz < 1 || !bytes) return set_error(P3D_ERR_ARG, "marker_project_workspace: bad sizes");
  if (!valid_type(type)) return set_error(P3D_ERR_ARG, "marker_project_workspace: unknown projection type %d", type);
  *bytes = workspace_bytes(mx, my, mz, type);
  return P3D_OK;
}

int p3d_marker_project(int32_t mx, int32_t my, int32_t mz, int type, int64_t n, const int32_t *wil, const double *xi,
                       const double *eta_p, const double *rho_p, double *eta_q, double *rho_q, void *workspace,
                       void *stream)
{
  if (mx < 1 || my < 1 || mz < 1 || n < 0) return set_error(P3D_ERR_ARG, "marker_project: bad sizes");
  if (!valid_type(type)) return set_error(P3D_ERR_ARG, "marker_project: unknown projection type %d", type);
  if (type == P3D_PROJ_NULL) return P3D_OK; // the values on the Gauss points stay as they are
  if (!eta_q || !rho_q) return set_error(P3D_ERR_ARG, "marker_project: null Gauss-point array");
  if (n > 0 && (!wil || !eta_p || !rho_p || (type == P3D_PROJ_Q1 && !xi)))
    return set_error(P3D_ERR_ARG, "marker_project: null marker array");
  const int64_t nel = (int64_t)mx * my * mz;
  const int64_t nn = (2 * (int64_t)mx + 1) * (2 * (int64_t)my + 1) * (2 * (int64_t)mz + 1);
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (type == P3D_PROJ_ONE2ONE) {
    if (n != 27 * nel)
      return set_error(P3D_ERR_ARG, "marker_project: one-to-one map needs 27 markers per element (%lld != %lld)",
                       (long long)n, (long long)(27 * nel));
    if ((rc = cuda_check(cudaMemcpyAsync(eta_q, eta_p, n * 8, cudaMemcpyDeviceToDevice, st), "one-to-one eta")))
      return rc;
    return cuda_check(cudaMemcpyAsync(rho_q, rho_p, n * 8, cudaMemcpyDeviceToDevice, st), "one-to-one rho");
  }
  const int64_t wb = workspace_bytes(mx, my, mz, type);
  if (!workspace || ((uintptr_t)workspace & 7))
    return set_error(P3D_ERR_ARG, "marker_project: workspace of %lld bytes (8-byte aligned) required", (long long)wb);
  double *W = (double *)workspace;
  if ((rc = cuda_check(cudaMemsetAsync(W, 0, wb, st), "marker_project memset"))) return rc;
  if (type == P3D_PROJ_Q1) {
    double *A1 = W, *A2 = W + nn, *B = W + 2 * nn;
    if (n > 0) {
      k_q1_scatter_warp<<<mgrid(n), 32 * Q1W, 0, st>>>(n, mx, my, mz, wil, xi, eta_p, rho_p, A1, A2, B);
      count_launch(1);
    }
    k_q1_divide<<<mgrid(nn), 256, 0, st>>>(nn, A1, A2, B);
    count_launch(1);
    s_eta_to_qp(mx, my, mz, A1, eta_q, st);
    s_eta_to_qp(mx, my, mz, A2, rho_q, st);
  } else {
    if (n > 0) {
      k_p0_scatter<<<mgrid(n), 256, 0, st>>>(n, nel, type, wil, eta_p, rho_p, W);
      count_launch(1);
    }
    k_p0_finish<<<mgrid(27 * nel), 256, 0, st>>>(nel, type, W, eta_q, rho_q);
    count_launch(1);
  }
  return cuda_check(cudaGetLastError(), "marker_project");
}
