// Element kernels built on the brick decomposition of q2_tile.cuh.
//
//   stokes_affine_kernel   any of {A11, A12, A21}, per-element constant Jacobian
//   stokes_general_kernel  any of {A11, A12, A21} with per-Gauss-point geometry
//   diag_general_kernel    d += diag(A11)
//   setup kernels          brick packing of eta, affinity test, affine packing
#pragma once
#include "q2_tile.cuh"

namespace p3d {

__host__ __device__ constexpr int align16(int n_elems, int elem_bytes)
{
  return ((n_elems * elem_bytes + 15) / 16) * 16 / elem_bytes;
}

// lane -> element slot/component inside the warp's 5x2 layer
struct LaneMap {
  int slot, a, b, c, f, base;
  bool active; // lane < 30
};
__device__ __forceinline__ LaneMap lane_map()
{
  LaneMap m;
  int lane = threadIdx.x & 31;
  int s = lane / 3;
  m.active = lane < 30;
  if (!m.active) s = 9; // idle lanes mirror slot 9 and never write
  m.f = m.active ? lane - 3 * s : lane - 30;
  m.base = 3 * s;
  m.a = s % TX;
  m.b = s / TX;
  m.c = threadIdx.x >> 5;
  m.slot = m.a + TX * (m.b + TY * m.c);
  return m;
}


// reciprocal of a Jacobian determinant: FP64 correctly rounded (CUDA's
// intrinsic); FP32 the hardware approximation rcp.approx (within an ulp, one
// instruction and no slow-path branch; the FP32 operators feed the smoother)
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_rn(float x)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// 3x3 inverse: M[3d+l] = dx_l/dxi_d  ->  Mi[3k+d] = dxi_d/dx_k, returns det
template <typename T> __device__ __forceinline__ T inv3(const T M[9], T Mi[9])
{
  T c00 = M[4] * M[8] - M[5] * M[7];
  T c01 = -(M[3] * M[8] - M[5] * M[6]);
  T c02 = M[3] * M[7] - M[4] * M[6];
  T c10 = -(M[1] * M[8] - M[2] * M[7]);
  T c11 = M[0] * M[8] - M[2] * M[6];
  T c12 = -(M[0] * M[7] - M[1] * M[6]);
  T c20 = M[1] * M[5] - M[2] * M[4];
  T c21 = -(M[0] * M[5] - M[2] * M[3]);
  T c22 = M[0] * M[4] - M[1] * M[3];
  T det = M[0] * c00 + M[1] * c01 + M[2] * c02;
  T r = rcp_rn(det); // = 1 / det
  // Mi[k][d] = cof[d][k] / det
  Mi[0] = c00 * r; Mi[1] = c10 * r; Mi[2] = c20 * r;
  Mi[3] = c01 * r; Mi[4] = c11 * r; Mi[5] = c21 * r;
  Mi[6] = c02 * r; Mi[7] = c12 * r; Mi[8] = c22 * r;
  return det;
}

// Pass 1 of the general path: per-Gauss-point geometry of the lane's element
// into g[q*GQ + ...]: [0..8] J^{-1} (row k = physical direction), [9] eta*w*detJ,
// [10] w*detJ, [11..13] pressure-basis coordinates (xh,yh,zh) when PB.
template <typename T, int NW, int GQ, bool PB>
__device__ __forceinline__ void geometry_pass(const T *s_c, const T *s_eta, T *g, const LaneMap &L, bool valid)
{
  T xq[27];
#pragma unroll
  for (int n = 0; n < 27; n++) xq[n] = s_c[tile_node<NW>(L.a, L.b, L.c, n) + L.f];
  T avg = (T)0, rL = (T)1;
  if (PB) {
#pragma unroll
    for (int n = 0; n < 27; n++) avg += xq[n];
    avg *= cst<T>(1.0 / 27.0);
    T Lf = (L.f == 0) ? xq[14] - xq[12] : ((L.f == 1) ? xq[16] - xq[10] : xq[22] - xq[4]);
    rL = valid ? (T)1 / Lf : (T)0;
  }
  interp27(xq);
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int q = i + 3 * j + 9 * k;
        T d0 = dcol(i, xq[3 * j + 9 * k], xq[1 + 3 * j + 9 * k], xq[2 + 3 * j + 9 * k]);
        T d1 = dcol(j, xq[i + 9 * k], xq[i + 3 + 9 * k], xq[i + 6 + 9 * k]);
        T d2 = dcol(k, xq[i + 3 * j], xq[i + 3 * j + 9], xq[i + 3 * j + 18]);
        if (!valid) { d0 = (T)(L.f == 0); d1 = (T)(L.f == 1); d2 = (T)(L.f == 2); }
        if (L.active) {
          g[q * GQ + 0 + L.f] = d0; // J[0][f]
          g[q * GQ + 3 + L.f] = d1; // J[1][f]
          g[q * GQ + 6 + L.f] = d2; // J[2][f]
          if (PB) g[q * GQ + 11 + L.f] = (xq[q] - avg) * rL;
        }
      }
  __syncwarp();
  for (int t = 0; t < 9; t++) {
    const int q = 3 * t + L.f;
    const int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
    T *G = g + q * GQ;
    T M[9], Mi[9];
#pragma unroll
    for (int r = 0; r < 9; r++) M[r] = G[r];
    T det = inv3(M, Mi);
    T w = (T)(w1d(qi) * w1d(qj) * w1d(qk)) * det;
    T eta = valid ? s_eta[q] : (T)0;
    if (L.active) {
#pragma unroll
      for (int r = 0; r < 9; r++) G[r] = Mi[r];
      G[9] = eta * w;
      if (GQ > 10) G[10] = valid ? w : (T)0;
    }
  }
  __syncwarp();
}

// load the lane's component of the element's 27 nodal values and move to Gauss points
template <typename T, int NW> __device__ __forceinline__ void load_interp(const T *s_x, const LaneMap &L, T uq[27])
{
#pragma unroll
  for (int n = 0; n < 27; n++) uq[n] = s_x[tile_node<NW>(L.a, L.b, L.c, n) + L.f];
  interp27(uq);
}

// strain -> stress -> pulled-back test-side vector for one Gauss point.
// Jr rows rotated so row 0 = physical direction f.  Returns ro[3] (reference dirs).
template <typename T>
__device__ __forceinline__ void qp_action(const T Jr[9], T ce, T g0, T g1, T g2, int src1, int src2, T &D0, T &ro0,
                                          T &ro1, T &ro2)
{
  D0 = Jr[0] * g0 + Jr[1] * g1 + Jr[2] * g2;       // dux[f][f]
  T D1 = Jr[3] * g0 + Jr[4] * g1 + Jr[5] * g2;     // dux[f+1][f]
  T D2 = Jr[6] * g0 + Jr[7] * g1 + Jr[8] * g2;     // dux[f+2][f]
  T rc1 = __shfl_sync(0xffffffffu, D2, src1);      // dux[f][f+1]
  T rc2 = __shfl_sync(0xffffffffu, D1, src2);      // dux[f][f+2]
  T T0 = ce * (D0 + D0), T1 = ce * (D1 + rc1), T2 = ce * (D2 + rc2);
  ro0 = Jr[0] * T0 + Jr[3] * T1 + Jr[6] * T2;
  ro1 = Jr[1] * T0 + Jr[4] * T1 + Jr[7] * T2;
  ro2 = Jr[2] * T0 + Jr[5] * T1 + Jr[8] * T2;
}

// gradient of the Gauss-point field uq at (i,j,k) in reference directions
#define P3D_GRAD(uq, i, j, k, g0, g1, g2)                                                                       \
  T g0 = dcol(i, uq[3 * (j) + 9 * (k)], uq[1 + 3 * (j) + 9 * (k)], uq[2 + 3 * (j) + 9 * (k)]);                  \
  T g1 = dcol(j, uq[(i) + 9 * (k)], uq[(i) + 3 + 9 * (k)], uq[(i) + 6 + 9 * (k)]);                              \
  T g2 = dcol(k, uq[(i) + 3 * (j)], uq[(i) + 3 * (j) + 9], uq[(i) + 3 * (j) + 18]);
#define P3D_SCATTER(r, i, j, k, ro0, ro1, ro2)                                                                  \
  dcolT(i, ro0, r[3 * (j) + 9 * (k)], r[1 + 3 * (j) + 9 * (k)], r[2 + 3 * (j) + 9 * (k)]);                       \
  dcolT(j, ro1, r[(i) + 9 * (k)], r[(i) + 3 + 9 * (k)], r[(i) + 6 + 9 * (k)]);                                   \
  dcolT(k, ro2, r[(i) + 3 * (j)], r[(i) + 3 * (j) + 9], r[(i) + 3 * (j) + 18]);

// A21 epilogue shared by the element kernels: lane f holds the moments
// [t, t*hat_f, t*hat_{f+1}, t*hat_{f+2}] of its own terms t; the element's three
// lanes sum them and lane 0 adds them to the element's 4 pressure rows in the
// basis order [1, xh, yh, zh].
template <typename T>
__device__ __forceinline__ void a21_moments(const LaneMap &L, bool valid, int src1, int src2, T ap0, T ap1, T ap2, T ap3,
                                            T *__restrict__ yp)
{
  const T s0 = ap0 + __shfl_sync(0xffffffffu, ap0, src1) + __shfl_sync(0xffffffffu, ap0, src2);
  // component m of the basis: lane f stores it in slot 1 + (m - f) mod 3
  T mom[3];
#pragma unroll
  for (int m = 0; m < 3; m++) {
    const int sl0 = (m - L.f + 3) % 3;           // this lane's slot for basis m
    const int sl1 = (m - (L.f + 1) % 3 + 3) % 3; // lane src1's slot
    const int sl2 = (m - (L.f + 2) % 3 + 3) % 3; // lane src2's slot
    const T v0 = sl0 == 0 ? ap1 : (sl0 == 1 ? ap2 : ap3);
    const T w1 = __shfl_sync(0xffffffffu, ap1, src1), w2 = __shfl_sync(0xffffffffu, ap2, src1),
            w3 = __shfl_sync(0xffffffffu, ap3, src1);
    const T u1 = __shfl_sync(0xffffffffu, ap1, src2), u2 = __shfl_sync(0xffffffffu, ap2, src2),
            u3 = __shfl_sync(0xffffffffu, ap3, src2);
    mom[m] = v0 + (sl1 == 0 ? w1 : (sl1 == 1 ? w2 : w3)) + (sl2 == 0 ? u1 : (sl2 == 1 ? u2 : u3));
  }
  if (L.active && valid && L.f == 0) {
    yp[0] += s0; yp[1] += mom[0]; yp[2] += mom[1]; yp[3] += mom[2];
  }
}

// ------------------------------------------------------------ affine kernels
// Per-element constant Jacobian.  kdat: [brick][slot][37] = J^{-1} (9),
// eta*w*detJ at the 27 Gauss points, 1 pad; kpre (A12/A21 only):
// [brick][slot][13] = the pressure-basis map C[d][m] = M[d][m] / (2 M[m][m])
// (9, M = dx/dxi), detJ, 3 pad.  The odd strides put the 10 elements of a warp
// on 10 different shared-memory banks (36 and 12 put them on 4).  On an affine
// element the basis coordinate
//   hat_m(x(xi)) = (x_m(xi) - mean of the 27 nodes) / L_m = sum_d C[d][m] xi_d,
// because the node mean is x(0) and the mid-face extent L_m is 2 M[m][m]
// (src/element_utils_q2.c:183-224).
constexpr int KAFF = 37, KPRE = 13;
template <typename T, int NW, bool DA11, bool DA12, bool DA21> struct AffineSmem {
  using BK = Brick<NW>;
  static constexpr bool NEEDX = DA11 || DA21;
  static constexpr bool NEEDY = DA11 || DA12;
  static constexpr bool PB = DA12 || DA21;
  static constexpr int OX = 0;
  static constexpr int OY = OX + (NEEDX ? align16(BK::TILE, sizeof(T)) : 0);
  static constexpr int OK = OY + (NEEDY ? align16(BK::TILE, sizeof(T)) : 0);
  static constexpr int OP = OK + align16(BK::NE * KAFF, sizeof(T));
  static constexpr int OA = OP + (PB ? align16(BK::NE * KPRE, sizeof(T)) : 0); // node-tile accumulator
  static constexpr int TOTAL = OA + (NEEDY ? BK::TILE : 0);
  static constexpr size_t BYTES = (size_t)TOTAL * sizeof(T);
};

template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__device__ __forceinline__ void stokes_affine_kernel_body(const TileArgs<T> &A)
{
  using BK = Brick<NW>;
  using SM = AffineSmem<T, NW, DA11, DA12, DA21>;
  constexpr bool NEEDX = SM::NEEDX, NEEDY = SM::NEEDY, PB = SM::PB;
  extern __shared__ __align__(16) unsigned char p3d_smem[];
  T *sm = reinterpret_cast<T *>(p3d_smem);
  T *s_x = sm + SM::OX, *s_y = sm + SM::OY, *s_k = sm + SM::OK, *s_p = sm + SM::OP, *s_acc = sm + SM::OA;
  const BrickPos b = brick_pos<T, NW>(A);
  const size_t brick = (size_t)blockIdx.x + A.brick0;
  if (NEEDX) stage_nodes<T, NW>(A, b, A.x, s_x, A.bc != 0);
  stage_block(A.kdat + brick * BK::NE * KAFF, s_k, BK::NE * KAFF);
  if (PB) stage_block(A.kgq + brick * BK::NE * KPRE, s_p, BK::NE * KPRE);
  if (NEEDY && !A.overwrite) stage_nodes<T, NW>(A, b, A.y, s_y, false);
  if (NEEDY)
    for (int i = threadIdx.x; i < BK::TILE; i += blockDim.x) s_acc[i] = (T)0;
  cp_async_wait_all();
  __syncthreads();

  const LaneMap L = lane_map();
  const bool valid = L.a < b.ax && L.b < b.ay && L.c < b.az;
  const int src1 = L.base + (L.f + 1) % 3, src2 = L.base + (L.f + 2) % 3;
  const T *K = s_k + L.slot * KAFF;
  T Jr[9];
  {
    const int r0 = 3 * L.f, r1 = 3 * ((L.f + 1) % 3), r2 = 3 * ((L.f + 2) % 3);
#pragma unroll
    for (int d = 0; d < 3; d++) { Jr[d] = K[r0 + d]; Jr[3 + d] = K[r1 + d]; Jr[6 + d] = K[r2 + d]; }
  }
  // pressure basis, rotated to the lane's direction: Cr[3d + t] = C[d][f + t]
  T Cr[9], detJ = 0, pr0 = 0, pr1 = 0, pr2 = 0, pr3 = 0;
  size_t eg = 0;
  if (PB) {
    const T *P = s_p + L.slot * KPRE;
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int t = 0; t < 3; t++) Cr[3 * d + t] = P[3 * d + (L.f + t) % 3];
    detJ = P[9];
    eg = (size_t)(b.e0x + L.a) + (size_t)A.mx * ((size_t)(b.e0y + L.b) + (size_t)A.my * (b.e0z + L.c));
    if (DA12 && valid) {
      const T p0 = A.p[4 * eg], p1 = A.p[4 * eg + 1], p2 = A.p[4 * eg + 2], p3 = A.p[4 * eg + 3];
      pr0 = p0;
      pr1 = L.f == 0 ? p1 : (L.f == 1 ? p2 : p3);
      pr2 = L.f == 0 ? p2 : (L.f == 1 ? p3 : p1);
      pr3 = L.f == 0 ? p3 : (L.f == 1 ? p1 : p2);
    }
  }
  T uq[27], r[27];
  if (NEEDX) load_interp<T, NW>(s_x, L, uq);
#pragma unroll
  for (int n = 0; n < 27; n++) r[n] = (T)0;
  T ap0 = 0, ap1 = 0, ap2 = 0, ap3 = 0;
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        T D0 = 0, ro0 = 0, ro1 = 0, ro2 = 0;
        if (NEEDX) {
          P3D_GRAD(uq, i, j, k, g0, g1, g2)
          if (DA11) {
            qp_action(Jr, K[9 + i + 3 * j + 9 * k], g0, g1, g2, src1, src2, D0, ro0, ro1, ro2);
          } else {
            D0 = Jr[0] * g0 + Jr[1] * g1 + Jr[2] * g2;
          }
        }
        if (PB) {
          // Gauss coordinates -s, 0, s; hats h0 = hat_f, h1 = hat_{f+1}, h2 = hat_{f+2}
          const T xi = cst<T>(i == 0 ? -0.77459666924148337704 : (i == 1 ? 0.0 : 0.77459666924148337704));
          const T xj = cst<T>(j == 0 ? -0.77459666924148337704 : (j == 1 ? 0.0 : 0.77459666924148337704));
          const T xk = cst<T>(k == 0 ? -0.77459666924148337704 : (k == 1 ? 0.0 : 0.77459666924148337704));
          const T h0 = Cr[0] * xi + Cr[3] * xj + Cr[6] * xk;
          const T h1 = Cr[1] * xi + Cr[4] * xj + Cr[7] * xk;
          const T h2 = Cr[2] * xi + Cr[5] * xj + Cr[8] * xk;
          const T wdet = cst<T>(w1d(i) * w1d(j) * w1d(k)) * detJ;
          if (DA12) {
            // -w detJ p_q grad(N) . e_f = -w detJ p_q (row f of J^{-1}) . grad_xi(N)
            const T t = valid ? -wdet * (pr0 + pr1 * h0 + pr2 * h1 + pr3 * h2) : (T)0;
            ro0 += t * Jr[0]; ro1 += t * Jr[1]; ro2 += t * Jr[2];
          }
          if (DA21) {
            const T t = valid ? -wdet * D0 : (T)0; // -w detJ Np du_f/dx_f
            ap0 += t; ap1 += t * h0; ap2 += t * h1; ap3 += t * h2;
          }
        }
        if (NEEDY) { P3D_SCATTER(r, i, j, k, ro0, ro1, ro2) }
      }
  if (DA21) a21_moments(L, valid, src1, src2, ap0, ap1, ap2, ap3, A.yp + 4 * eg);
  if (NEEDY) {
    interp27T(r);
    accumulate_tile<T, NW>(s_acc, r, L.a, L.b, L.c, L.f, L.active && valid);
    write_tile<T, NW>(A, b, s_acc, s_y, DA11 ? 0 : 1);
  }
}
template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__global__ void __launch_bounds__(32 * NW, (DA12 || DA21) ? (DA11 ? 2 : 3) : 4) stokes_affine_kernel(TileArgs<T> A) { stokes_affine_kernel_body<T, NW, DA11, DA12, DA21>(A); }
// the same over the K operators of a group (blockIdx.y = member), one launch
template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__global__ void __launch_bounds__(32 * NW, (DA12 || DA21) ? (DA11 ? 2 : 3) : 4) stokes_affine_kernel_group(const __grid_constant__ TileGroup<T> G)
{
  stokes_affine_kernel_body<T, NW, DA11, DA12, DA21>(G.a[blockIdx.y]);
}

// Gauss-point coordinate table (general path), packed at setup, GQC values per
// element in blocks of one brick.  A brick's block holds
//   [n][slot][f]  the coordinate f of element slot at Gauss point n (27 x NE x 3,
//                 the tensor interpolation of the element's nodes), so that the
//                 30 lanes of a warp read 30 consecutive values (no bank conflicts);
//   [slot][6]     the centroid of the 27 nodes (3 values) and the reciprocal
//                 mid-face extents 1/L (3 values) of the pressure basis;
//   zeros up to NE * GQC values.
constexpr int GQC = 88;
template <int NW> struct GQLayout {
  static constexpr int PT = 3 * Brick<NW>::NE; // values per Gauss point
  static constexpr int EX = 27 * PT;           // start of the per-element extras
  static_assert(EX + 6 * Brick<NW>::NE <= GQC * Brick<NW>::NE, "Gauss-point table block");
};

// ------------------------------------------------------- general geometry
// The Jacobian is recomputed at every Gauss point.  Lane f owns column f of
// M = [dx_l/dxi_d] (d = row); at each point it fetches the element's other two
// columns by warp shuffle and forms the adjugate rows in registers:
//   row_f(M^{-1}) = (col_{f+1} x col_{f+2}) / det,   det = col_f . (col_{f+1} x col_{f+2}),
// rotated so that row 0 belongs to direction f (the rotation makes the strain
// exchange a uniform pair of shuffles).  The 1/det factors of the gradient
// and of the pulled-back stress combine into one scale eta*w/det per point,
// so the action runs on the unscaled adjugate.  The element's Gauss-point
// coordinates come from the setup-time table (one contiguous 16-byte copy per
// brick instead of node rows and an interpolation per apply); each point reads
// the up to 7 coordinate values its column needs from shared memory, which keeps
// the spills of the 168-register cap to 64 bytes.  The cap (6 CTAs of 64
// threads per SM) gives 50 % more resident warps than the uncapped 254
// registers, which this latency-bound kernel converts into speed.
template <typename T, int NW, bool DA11, bool DA12, bool DA21> struct GeneralSmem {
  using BK = Brick<NW>;
  static constexpr bool NEEDX = DA11 || DA21;
  static constexpr bool NEEDY = DA11 || DA12;
  static constexpr int CQ = align16(BK::NE * GQC, sizeof(T)); // Gauss-point coordinate table
  static constexpr int OX = 0;
  static constexpr int OY = OX + (NEEDX ? align16(BK::TILE, sizeof(T)) : 0);
  static constexpr int OC = OY + (NEEDY ? align16(BK::TILE, sizeof(T)) : 0);
  static constexpr int CA = align16(BK::TILE, sizeof(T)); // accumulator (reuses the tile region)
  static constexpr int OK = OC + (CA > CQ ? CA : CQ);
  static constexpr int TOTAL = OK + align16(BK::NE * 27, sizeof(T));
  static constexpr size_t BYTES = (size_t)TOTAL * sizeof(T);
};

template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__device__ __forceinline__ void stokes_general_kernel_body(const TileArgs<T> &A)
{
  using BK = Brick<NW>;
  using SM = GeneralSmem<T, NW, DA11, DA12, DA21>;
  constexpr bool PB = DA12 || DA21;
  constexpr bool NEEDY = SM::NEEDY;
  extern __shared__ __align__(16) unsigned char p3d_smem[];
  T *sm = reinterpret_cast<T *>(p3d_smem);
  T *s_x = sm + SM::OX, *s_y = sm + SM::OY, *s_c = sm + SM::OC, *s_k = sm + SM::OK;
  const BrickPos b = brick_pos<T, NW>(A);
  const size_t brick = (size_t)blockIdx.x + A.brick0;
  if (SM::NEEDX) stage_nodes<T, NW>(A, b, A.x, s_x, A.bc != 0);
  stage_block(A.kgq + brick * BK::NE * GQC, s_c, BK::NE * GQC); // Gauss-point coordinates, centroid, 1/L
  stage_block(A.kdat + brick * BK::NE * 27, s_k, BK::NE * 27);
  if (NEEDY && !A.overwrite) stage_nodes<T, NW>(A, b, A.y, s_y, false);
  cp_async_wait_all();
  __syncthreads();

  const LaneMap L = lane_map();
  const bool valid = L.a < b.ax && L.b < b.ay && L.c < b.az;
  using GL = GQLayout<NW>;
  const T *X = s_c + 3 * L.slot + L.f; // coordinate f at Gauss point n: X[n * GL::PT]
  const T avg = PB ? s_c[GL::EX + 6 * L.slot + L.f] : (T)0, rL = PB ? s_c[GL::EX + 6 * L.slot + 3 + L.f] : (T)1;
  const T *eta_e = s_k + L.slot * 27;

  const int src1 = L.base + (L.f + 1) % 3, src2 = L.base + (L.f + 2) % 3;
  const size_t eg = (size_t)(b.e0x + L.a) + (size_t)A.mx * ((size_t)(b.e0y + L.b) + (size_t)A.my * (b.e0z + L.c));
  T uq[27], r[27];
  if (SM::NEEDX) load_interp<T, NW>(s_x, L, uq);
#pragma unroll
  for (int n = 0; n < 27; n++) r[n] = (T)0;
  // pressure dofs rotated to the lane's direction: pr[0] constant, pr[1+m] multiplies hat_{f+m}
  T pr0 = 0, pr1 = 0, pr2 = 0, pr3 = 0;
  if (DA12 && valid) {
    const T p0 = A.p[4 * eg], p1 = A.p[4 * eg + 1], p2 = A.p[4 * eg + 2], p3 = A.p[4 * eg + 3];
    pr0 = p0;
    pr1 = L.f == 0 ? p1 : (L.f == 1 ? p2 : p3);
    pr2 = L.f == 0 ? p2 : (L.f == 1 ? p3 : p1);
    pr3 = L.f == 0 ? p3 : (L.f == 1 ? p1 : p2);
  }
  T ap0 = 0, ap1 = 0, ap2 = 0, ap3 = 0; // A21: [1, hat_f, hat_{f+1}, hat_{f+2}] moments
#pragma unroll
  for (int k = 0; k < 3; k++) {
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int q9 = i + 3 * j;
        // column f of M at this point, straight from the staged Gauss-point
        // coordinates (conflict-free reads; keeping a plane's columns in
        // registers instead costs spills)
#define P3D_XG(n) X[(n) * GL::PT]
        const T cc0 = dcol(i, P3D_XG(3 * j + 9 * k), P3D_XG(1 + 3 * j + 9 * k), P3D_XG(2 + 3 * j + 9 * k));
        const T cc1 = dcol(j, P3D_XG(i + 9 * k), P3D_XG(i + 3 + 9 * k), P3D_XG(i + 6 + 9 * k));
        const T cc2 = dcol(k, P3D_XG(i + 3 * j), P3D_XG(i + 3 * j + 9), P3D_XG(i + 3 * j + 18));
        const T hq = PB ? (P3D_XG(q9 + 9 * k) - avg) * rL : (T)0;
#undef P3D_XG
        // the element's other two columns: a = col_{f+1}, bb = col_{f+2}
        const T a0 = __shfl_sync(0xffffffffu, cc0, src1), a1 = __shfl_sync(0xffffffffu, cc1, src1),
                a2 = __shfl_sync(0xffffffffu, cc2, src1);
        const T b0 = __shfl_sync(0xffffffffu, cc0, src2), b1 = __shfl_sync(0xffffffffu, cc1, src2),
                b2 = __shfl_sync(0xffffffffu, cc2, src2);
        // unscaled rows of M^{-1}: R0 (direction f) = a x b, R1 = b x c, R2 = c x a
        T Jr[9];
        Jr[0] = a1 * b2 - a2 * b1; Jr[1] = a2 * b0 - a0 * b2; Jr[2] = a0 * b1 - a1 * b0;
        Jr[3] = b1 * cc2 - b2 * cc1; Jr[4] = b2 * cc0 - b0 * cc2; Jr[5] = b0 * cc1 - b1 * cc0;
        Jr[6] = cc1 * a2 - cc2 * a1; Jr[7] = cc2 * a0 - cc0 * a2; Jr[8] = cc0 * a1 - cc1 * a0;
        const T det = cc0 * Jr[0] + cc1 * Jr[1] + cc2 * Jr[2];
        const T wq = cst<T>(w1d(i) * w1d(j) * w1d(k));
        T ro0 = 0, ro1 = 0, ro2 = 0, D0 = 0;
        if (SM::NEEDX) {
          P3D_GRAD(uq, i, j, k, g0, g1, g2)
          if (DA11) {
            // eta*w*det * (D + D^T) pulled back with M^{-T}: with unscaled rows the
            // factors of det leave eta*w/det, formed with the correctly rounded
            // reciprocal (a full division here cost 10 % of the FP64 apply)
            const T sc = (valid ? eta_e[q9 + 9 * k] : (T)0) * wq * rcp_rn(det);
            qp_action(Jr, sc, g0, g1, g2, src1, src2, D0, ro0, ro1, ro2);
          } else {
            D0 = Jr[0] * g0 + Jr[1] * g1 + Jr[2] * g2;
          }
        }
        if (PB) {
          // hats of the element's three lanes, rotated: h0 = hat_f, h1 = hat_{f+1}, h2 = hat_{f+2}
          const T h0 = hq, h1 = __shfl_sync(0xffffffffu, h0, src1), h2 = __shfl_sync(0xffffffffu, h0, src2);
          if (DA12) {
            // -w detJ p_q grad(N) = -w p_q * (adjugate row f) (det cancels)
            const T t = valid ? -wq * (pr0 + pr1 * h0 + pr2 * h1 + pr3 * h2) : (T)0;
            ro0 += t * Jr[0]; ro1 += t * Jr[1]; ro2 += t * Jr[2];
          }
          if (DA21) {
            // -w detJ Np du_f/dx_f = -w Np (adjugate row f . grad)
            const T t = valid ? -wq * D0 : (T)0;
            ap0 += t; ap1 += t * h0; ap2 += t * h1; ap3 += t * h2;
          }
        }
        if (NEEDY) { P3D_SCATTER(r, i, j, k, ro0, ro1, ro2) }
      }
  }
  if (DA21) a21_moments(L, valid, src1, src2, ap0, ap1, ap2, ap3, A.yp + 4 * eg);
  if (NEEDY) {
    interp27T(r);
    __syncthreads(); // every warp is done with the Gauss-point coordinates: reuse as the accumulator
    T *s_acc = s_c;
    for (int i = threadIdx.x; i < BK::TILE; i += blockDim.x) s_acc[i] = (T)0;
    __syncthreads();
    accumulate_tile<T, NW>(s_acc, r, L.a, L.b, L.c, L.f, L.active && valid);
    write_tile<T, NW>(A, b, s_acc, s_y, DA11 ? 0 : 1);
  }
}
template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__global__ void __launch_bounds__(32 * NW, 6) stokes_general_kernel(TileArgs<T> A) { stokes_general_kernel_body<T, NW, DA11, DA12, DA21>(A); }
// the same over the K operators of a group (blockIdx.y = member), one launch
template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__global__ void __launch_bounds__(32 * NW, 6) stokes_general_kernel_group(const __grid_constant__ TileGroup<T> G)
{
  stokes_general_kernel_body<T, NW, DA11, DA12, DA21>(G.a[blockIdx.y]);
}

// ---------------------------------------- general geometry, table variant
// Used for FP32, where the table costs less than the shuffle exchange.
// Geometry is built one Gauss-point plane (9 points, fixed k) at a time from
// the staged Gauss-point coordinate table: every lane inverts 3 of the plane's
// 9 Jacobians into a per-element table read by all three lanes, which holds 9
// points instead of 27 (3x less shared memory, more CTAs per SM).
template <typename T, int NW, bool DA11, bool DA12, bool DA21> struct GeneralTabSmem {
  using BK = Brick<NW>;
  static constexpr bool NEEDX = DA11 || DA21;
  static constexpr bool NEEDY = DA11 || DA12;
  static constexpr int GQ = (DA12 || DA21) ? 14 : 10;
  static constexpr int CQ = align16(BK::NE * GQC, sizeof(T)); // Gauss-point coordinate table
  static constexpr int OX = 0;
  static constexpr int OY = OX + (NEEDX ? align16(BK::TILE, sizeof(T)) : 0);
  static constexpr int OC = OY + (NEEDY ? align16(BK::TILE, sizeof(T)) : 0);
  static constexpr int CA = align16(BK::TILE, sizeof(T)); // accumulator (reuses the tile region)
  static constexpr int OK = OC + (CA > CQ ? CA : CQ);
  static constexpr int OG = OK + align16(BK::NE * 27, sizeof(T));
  // per-element stride of the plane's Jacobian table: 9 points x GQ values,
  // padded so that the 30 lanes of a warp spread over the 4-byte banks
  // (90 -> 105 and 126 -> 133 cut the table's shared wavefronts by a third)
  static constexpr int ES = GQ == 10 ? 105 : (GQ == 14 ? 133 : 9 * GQ);
  static constexpr int TOTAL = OG + BK::NE * ES;
  static constexpr size_t BYTES = (size_t)TOTAL * sizeof(T);
};

template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__device__ __forceinline__ void stokes_general_tab_kernel_body(const TileArgs<T> &A)
{
  using BK = Brick<NW>;
  using SM = GeneralTabSmem<T, NW, DA11, DA12, DA21>;
  constexpr int GQ = SM::GQ;
  constexpr bool PB = DA12 || DA21;
  constexpr bool NEEDY = SM::NEEDY;
  extern __shared__ __align__(16) unsigned char p3d_smem[];
  T *sm = reinterpret_cast<T *>(p3d_smem);
  T *s_x = sm + SM::OX, *s_y = sm + SM::OY, *s_c = sm + SM::OC, *s_k = sm + SM::OK, *s_g = sm + SM::OG;
  const BrickPos b = brick_pos<T, NW>(A);
  const size_t brick = (size_t)blockIdx.x + A.brick0;
  if (SM::NEEDX) stage_nodes<T, NW>(A, b, A.x, s_x, A.bc != 0);
  stage_block(A.kgq + brick * BK::NE * GQC, s_c, BK::NE * GQC); // Gauss-point coordinates, centroid, 1/L
  stage_block(A.kdat + brick * BK::NE * 27, s_k, BK::NE * 27);
  if (NEEDY && !A.overwrite) stage_nodes<T, NW>(A, b, A.y, s_y, false);
  cp_async_wait_all();
  __syncthreads();

  const LaneMap L = lane_map();
  const bool valid = L.a < b.ax && L.b < b.ay && L.c < b.az;
  using GL = GQLayout<NW>;
  const T *X = s_c + 3 * L.slot + L.f; // coordinate f at Gauss point n: X[n * GL::PT]
  const T avg = PB ? s_c[GL::EX + 6 * L.slot + L.f] : (T)0, rL = PB ? s_c[GL::EX + 6 * L.slot + 3 + L.f] : (T)1;
  const T *eta_e = s_k + L.slot * 27;
  T *g = s_g + L.slot * SM::ES;

  const int src1 = L.base + (L.f + 1) % 3, src2 = L.base + (L.f + 2) % 3;
  const int r0 = 3 * L.f, r1 = 3 * ((L.f + 1) % 3), r2 = 3 * ((L.f + 2) % 3);
  const size_t eg = (size_t)(b.e0x + L.a) + (size_t)A.mx * ((size_t)(b.e0y + L.b) + (size_t)A.my * (b.e0z + L.c));
  T uq[27], r[27];
  if (SM::NEEDX) load_interp<T, NW>(s_x, L, uq);
#pragma unroll
  for (int n = 0; n < 27; n++) r[n] = (T)0;
  T pe0 = 0, pe1 = 0, pe2 = 0, pe3 = 0;
  if (DA12 && valid) { pe0 = A.p[4 * eg]; pe1 = A.p[4 * eg + 1]; pe2 = A.p[4 * eg + 2]; pe3 = A.p[4 * eg + 3]; }
  T ap0 = 0, ap1 = 0, ap2 = 0, ap3 = 0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    // ---- plane k: Jacobian columns (lane f owns column f), then 3 inversions per lane
    {
      T xp[27];
#pragma unroll
      for (int n = 0; n < 27; n++) xp[n] = X[n * GL::PT];
#pragma unroll
      for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const int q9 = i + 3 * j;
          T d0 = dcol(i, xp[3 * j + 9 * k], xp[1 + 3 * j + 9 * k], xp[2 + 3 * j + 9 * k]);
          T d1 = dcol(j, xp[i + 9 * k], xp[i + 3 + 9 * k], xp[i + 6 + 9 * k]);
          T d2 = dcol(k, xp[i + 3 * j], xp[i + 3 * j + 9], xp[i + 3 * j + 18]);
          if (!valid) { d0 = (T)(L.f == 0); d1 = (T)(L.f == 1); d2 = (T)(L.f == 2); }
          // lanes 30 and 31 repeat lanes 27 and 28 (slot 9): their stores write
          // the same values to the same places, so no lane guard is needed
          g[q9 * GQ + 0 + L.f] = d0;
          g[q9 * GQ + 3 + L.f] = d1;
          g[q9 * GQ + 6 + L.f] = d2;
          if (PB) g[q9 * GQ + 11 + L.f] = (xp[q9 + 9 * k] - avg) * rL;
        }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 3; t++) {
      const int q9 = 3 * t + L.f; // i = f, j = t
      T *G = g + q9 * GQ;
      T M[9], Mi[9];
#pragma unroll
      for (int rr = 0; rr < 9; rr++) M[rr] = G[rr];
      T det = inv3(M, Mi);
      T w = (T)(w1d(L.f) * w1d(t) * w1d(k)) * det;
      T eta = valid ? eta_e[q9 + 9 * k] : (T)0;
#pragma unroll
      for (int rr = 0; rr < 9; rr++) G[rr] = Mi[rr];
      G[9] = eta * w;
      if (GQ > 10) G[10] = valid ? w : (T)0;
    }
    __syncwarp();
    // ---- the plane's 9 Gauss points
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const T *G = g + (i + 3 * j) * GQ;
        T Jr[9];
#pragma unroll
        for (int d = 0; d < 3; d++) { Jr[d] = G[r0 + d]; Jr[3 + d] = G[r1 + d]; Jr[6 + d] = G[r2 + d]; }
        T ro0 = 0, ro1 = 0, ro2 = 0, D0 = 0;
        if (SM::NEEDX) {
          P3D_GRAD(uq, i, j, k, g0, g1, g2)
          if (DA11) {
            qp_action(Jr, G[9], g0, g1, g2, src1, src2, D0, ro0, ro1, ro2);
          } else {
            D0 = Jr[0] * g0 + Jr[1] * g1 + Jr[2] * g2;
          }
        }
        if (PB) {
          const T c0 = G[10], xh = G[11], yh = G[12], zh = G[13];
          if (DA12) {
            T t = -c0 * (pe0 + pe1 * xh + pe2 * yh + pe3 * zh);
            ro0 += t * Jr[0]; ro1 += t * Jr[1]; ro2 += t * Jr[2];
          }
          if (DA21) {
            T t = -c0 * D0;
            ap0 += t; ap1 += t * xh; ap2 += t * yh; ap3 += t * zh;
          }
        }
        if (NEEDY) { P3D_SCATTER(r, i, j, k, ro0, ro1, ro2) }
      }
    __syncwarp(); // the next plane overwrites this element's table
  }
  if (DA21) {
    // divergence = sum over the element's three lanes
    ap0 += __shfl_sync(0xffffffffu, ap0, src1) + __shfl_sync(0xffffffffu, ap0, src2);
    ap1 += __shfl_sync(0xffffffffu, ap1, src1) + __shfl_sync(0xffffffffu, ap1, src2);
    ap2 += __shfl_sync(0xffffffffu, ap2, src1) + __shfl_sync(0xffffffffu, ap2, src2);
    ap3 += __shfl_sync(0xffffffffu, ap3, src1) + __shfl_sync(0xffffffffu, ap3, src2);
    if (L.active && valid && L.f == 0) {
      A.yp[4 * eg] += ap0; A.yp[4 * eg + 1] += ap1; A.yp[4 * eg + 2] += ap2; A.yp[4 * eg + 3] += ap3;
    }
  }
  if (NEEDY) {
    interp27T(r);
    __syncthreads(); // every warp is done with the Gauss-point coordinates: reuse as the accumulator
    T *s_acc = s_c;
    for (int i = threadIdx.x; i < BK::TILE; i += blockDim.x) s_acc[i] = (T)0;
    __syncthreads();
    accumulate_tile<T, NW>(s_acc, r, L.a, L.b, L.c, L.f, L.active && valid);
    write_tile<T, NW>(A, b, s_acc, s_y, DA11 ? 0 : 1);
  }
}
template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__global__ void __launch_bounds__(32 * NW) stokes_general_tab_kernel(TileArgs<T> A) { stokes_general_tab_kernel_body<T, NW, DA11, DA12, DA21>(A); }
// the same over the K operators of a group (blockIdx.y = member), one launch
template <typename T, int NW, bool DA11, bool DA12, bool DA21>
__global__ void __launch_bounds__(32 * NW) stokes_general_tab_kernel_group(const __grid_constant__ TileGroup<T> G)
{
  stokes_general_tab_kernel_body<T, NW, DA11, DA12, DA21>(G.a[blockIdx.y]);
}

// --------------------------------------------------------------- diagonal
__constant__ double c_B[3][3];
__constant__ double c_D[3][3];

template <typename T, int NW> struct DiagSmem {
  using BK = Brick<NW>;
  static constexpr int GQ = 10;
  static constexpr int OY = 0;
  static constexpr int OC = OY + align16(BK::TILE, sizeof(T));
  static constexpr int OK = OC + align16(BK::TILE, sizeof(T));
  static constexpr int OG = OK + align16(BK::NE * 27, sizeof(T));
  static constexpr int TOTAL = OG + BK::NE * 27 * GQ;
  static constexpr size_t BYTES = (size_t)TOTAL * sizeof(T);
};

template <typename T, int NW>
__global__ void __launch_bounds__(32 * NW) diag_general_kernel(TileArgs<T> A)
{
  using BK = Brick<NW>;
  using SM = DiagSmem<T, NW>;
  constexpr int GQ = SM::GQ;
  extern __shared__ __align__(16) unsigned char p3d_smem[];
  T *sm = reinterpret_cast<T *>(p3d_smem);
  T *s_y = sm + SM::OY, *s_c = sm + SM::OC, *s_k = sm + SM::OK, *s_g = sm + SM::OG;
  const BrickPos b = brick_pos<T, NW>(A);
  stage_nodes<T, NW>(A, b, A.coords, s_c, false);
  stage_block(A.kdat + (size_t)(blockIdx.x + A.brick0) * BK::NE * 27, s_k, BK::NE * 27);
  stage_nodes<T, NW>(A, b, A.y, s_y, false);
  cp_async_wait_all();
  __syncthreads();
  const LaneMap L = lane_map();
  const bool valid = L.a < b.ax && L.b < b.ay && L.c < b.az;
  T *g = s_g + L.slot * 27 * GQ;
  geometry_pass<T, NW, GQ, false>(s_c, s_k + L.slot * 27, g, L, valid);
  T dg[27];
#pragma unroll
  for (int n = 0; n < 27; n++) dg[n] = (T)0;
  for (int q = 0; q < 27; q++) {
    const int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
    const T *G = g + q * GQ;
    T Ji[9];
#pragma unroll
    for (int r = 0; r < 9; r++) Ji[r] = G[r];
    const T ce = G[9];
#pragma unroll
    for (int n = 0; n < 27; n++) {
      const int na = n % 3, nb = (n / 3) % 3, nc = n / 9;
      T r0 = (T)(c_D[qi][na] * c_B[qj][nb] * c_B[qk][nc]);
      T r1 = (T)(c_B[qi][na] * c_D[qj][nb] * c_B[qk][nc]);
      T r2 = (T)(c_B[qi][na] * c_B[qj][nb] * c_D[qk][nc]);
      T d0 = Ji[0] * r0 + Ji[1] * r1 + Ji[2] * r2;
      T d1 = Ji[3] * r0 + Ji[4] * r1 + Ji[5] * r2;
      T d2 = Ji[6] * r0 + Ji[7] * r1 + Ji[8] * r2;
      T df = (L.f == 0) ? d0 : ((L.f == 1) ? d1 : d2);
      dg[n] += ce * (d0 * d0 + d1 * d1 + d2 * d2 + df * df);
    }
  }
  __syncthreads();
  T *s_acc = s_c;
  for (int i = threadIdx.x; i < BK::TILE; i += blockDim.x) s_acc[i] = (T)0;
  __syncthreads();
  accumulate_tile<T, NW>(s_acc, dg, L.a, L.b, L.c, L.f, L.active && valid);
  write_tile<T, NW>(A, b, s_acc, s_y, 2);
}

// ---------------------------------------------------------------- setup ---
// eta (element-lexicographic, FP64) -> brick-ordered [brick][slot][27] in T
template <typename T, int NW>
__global__ void pack_eta_kernel(int mx, int my, int mz, int ntx, int nty, int ntz, const double *__restrict__ eta,
                                T *__restrict__ out)
{
  using BK = Brick<NW>;
  size_t total = (size_t)ntx * nty * ntz * BK::NE * 27;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    int q = idx % 27;
    size_t rest = idx / 27;
    int slot = rest % BK::NE;
    size_t t = rest / BK::NE;
    int tx = t % ntx, ty = (t / ntx) % nty, tz = t / ((size_t)ntx * nty);
    int a = slot % TX, bb = (slot / TX) % TY, c = slot / (TX * TY);
    int ex = tx * TX + a, ey = ty * TY + bb, ez = tz * NW + c;
    T v = (T)0;
    if (ex < mx && ey < my && ez < mz) v = (T)eta[27 * ((size_t)ex + (size_t)mx * ((size_t)ey + (size_t)my * ez)) + q];
    out[idx] = v;
  }
}

// Gauss-point coordinate table (GQLayout, one block per brick).  Slots outside
// the mesh get a unit cube (their results are never written).
template <typename T, int NW>
__global__ void pack_gauss_coords_kernel(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, int ntx, int nty,
                                         int ntz, const double *__restrict__ coords, T *__restrict__ out)
{
  using BK = Brick<NW>;
  const size_t total = (size_t)ntx * nty * ntz * BK::NE;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int slot = idx % BK::NE;
    const size_t t = idx / BK::NE;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / ((size_t)ntx * nty);
    const int a = slot % TX, bb = (slot / TX) % TY, c = slot / (TX * TY);
    const int ex = tx * TX + a, ey = ty * TY + bb, ez = tz * NW + c;
    const bool valid = ex < mx && ey < my && ez < mz;
    using GL = GQLayout<NW>;
    T *o = out + t * (BK::NE * GQC);
    for (int f = 0; f < 3; f++) {
      double xq[27];
      for (int n = 0; n < 27; n++) {
        const int na = n % 3, nb = (n / 3) % 3, nc = n / 9;
        if (valid) {
          const size_t gi = (size_t)(ox + 2 * ex + na) + (size_t)gx * ((size_t)(oy + 2 * ey + nb) + (size_t)gy * (oz + 2 * ez + nc));
          xq[n] = coords[3 * gi + f];
        } else {
          xq[n] = 0.5 * (f == 0 ? na : (f == 1 ? nb : nc));
        }
      }
      double avg = 0.0;
      for (int n = 0; n < 27; n++) avg += xq[n];
      avg *= 1.0 / 27.0;
      const double Lf = (f == 0) ? xq[14] - xq[12] : ((f == 1) ? xq[16] - xq[10] : xq[22] - xq[4]);
      interp27(xq);
      for (int n = 0; n < 27; n++) o[n * GL::PT + 3 * slot + f] = (T)xq[n];
      o[GL::EX + 6 * slot + f] = (T)avg;
      o[GL::EX + 6 * slot + 3 + f] = (T)(1.0 / Lf);
    }
    if (slot == 0)
      for (int i = GL::EX + 6 * BK::NE; i < BK::NE * GQC; i++) o[i] = (T)0;
  }
}

// count elements that are not parallelepipeds (to relative tolerance tol)
__global__ void affine_check_kernel(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz,
                                    const double *__restrict__ coords, double tol, unsigned long long *bad)
{
  size_t nel = (size_t)mx * my * mz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nel; e += (size_t)gridDim.x * blockDim.x) {
    int ex = e % mx, ey = (e / mx) % my, ez = e / ((size_t)mx * my);
    auto X = [&](int a, int b2, int c, int d) {
      size_t gi = (size_t)(ox + 2 * ex + a) + (size_t)gx * ((size_t)(oy + 2 * ey + b2) + (size_t)gy * (oz + 2 * ez + c));
      return coords[3 * gi + d];
    };
    double dev = 0.0, h = 0.0;
    for (int d = 0; d < 3; d++) {
      double x0 = X(0, 0, 0, d);
      double j0 = 0.5 * (X(2, 0, 0, d) - x0), j1 = 0.5 * (X(0, 2, 0, d) - x0), j2 = 0.5 * (X(0, 0, 2, d) - x0);
      h = fmax(h, fmax(fabs(j0), fmax(fabs(j1), fabs(j2))));
      for (int c = 0; c < 3; c++)
        for (int b2 = 0; b2 < 3; b2++)
          for (int a = 0; a < 3; a++) {
            double pred = x0 + j0 * a + j1 * b2 + j2 * c;
            dev = fmax(dev, fabs(X(a, b2, c, d) - pred));
          }
    }
    if (!(dev <= tol * h)) atomicAdd(bad, 1ull);
  }
}

// per element J^{-1} and eta*w*detJ (affine elements), brick-ordered [brick][slot][KAFF];
// pre (optional): the pressure-basis map and detJ, [brick][slot][KPRE]
template <typename T, int NW>
__global__ void pack_affine_kernel(int mx, int my, int mz, int gx, int gy, int ox, int oy, int oz, int ntx, int nty,
                                   int ntz, const double *__restrict__ coords, const double *__restrict__ eta,
                                   T *__restrict__ out, T *__restrict__ pre)
{
  using BK = Brick<NW>;
  size_t total = (size_t)ntx * nty * ntz * BK::NE;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    int slot = idx % BK::NE;
    size_t t = idx / BK::NE;
    int tx = t % ntx, ty = (t / ntx) % nty, tz = t / ((size_t)ntx * nty);
    int a = slot % TX, bb = (slot / TX) % TY, c = slot / (TX * TY);
    int ex = tx * TX + a, ey = ty * TY + bb, ez = tz * NW + c;
    T *o = out + idx * KAFF;
    if (!(ex < mx && ey < my && ez < mz)) {
      for (int r = 0; r < KAFF; r++) o[r] = (T)0;
      if (pre)
        for (int r = 0; r < KPRE; r++) pre[idx * KPRE + r] = (T)0;
      continue;
    }
    auto X = [&](int a2, int b2, int c2, int d) {
      size_t gi = (size_t)(ox + 2 * ex + a2) + (size_t)gx * ((size_t)(oy + 2 * ey + b2) + (size_t)gy * (oz + 2 * ez + c2));
      return coords[3 * gi + d];
    };
    double M[9], Mi[9];
    for (int l = 0; l < 3; l++) {
      M[0 + l] = 0.5 * (X(2, 1, 1, l) - X(0, 1, 1, l)); // dx_l/dxi_0
      M[3 + l] = 0.5 * (X(1, 2, 1, l) - X(1, 0, 1, l)); // dx_l/dxi_1
      M[6 + l] = 0.5 * (X(1, 1, 2, l) - X(1, 1, 0, l)); // dx_l/dxi_2
    }
    double det = inv3<double>(M, Mi);
    for (int r = 0; r < 9; r++) o[r] = (T)Mi[r];
    if (pre) {
      T *pp = pre + idx * KPRE;
      for (int d = 0; d < 3; d++)
        for (int mm = 0; mm < 3; mm++) pp[3 * d + mm] = (T)(M[3 * d + mm] / (2.0 * M[3 * mm + mm]));
      pp[9] = (T)det;
      for (int r = 10; r < KPRE; r++) pp[r] = (T)0;
    }
    for (int r = 36; r < KAFF; r++) o[r] = (T)0;
    size_t e = (size_t)ex + (size_t)mx * ((size_t)ey + (size_t)my * ez);
    for (int q = 0; q < 27; q++) {
      int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
      o[9 + q] = (T)(eta[27 * e + q] * w1d(qi) * w1d(qj) * w1d(qk) * det);
    }
  }
}

} // namespace p3d
