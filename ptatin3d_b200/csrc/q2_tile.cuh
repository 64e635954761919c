// Matrix-free Q2-P1disc Stokes element kernels for sm_100a.
//
// Work decomposition
//   A CTA owns a brick of TX x TY x NW elements (TX=5, TY=2): warp w holds the
//   element layer z=w, lanes 3*s+f (s = 0..9 element slot, f = 0..2 velocity
//   component), lanes 30,31 idle.  The node brick (2TX+1)(2TY+1)(2NW+1) of x
//   is staged in shared memory with coalesced loads, per-element data (eta,
//   packed geometry) with contiguous 16-byte copies; each lane then works on
//   ONE velocity component of ONE element in registers:
//     1. interpolate its 27 nodal values to the 27 Gauss points (three 1-D
//        stages of the Q2 basis at the Gauss points, B(0) row = [0,1,0]),
//     2. per Gauss point take reference derivatives with the collocated
//        derivative matrix Dh = D B^{-1} (Lagrange derivative on the Gauss
//        nodes), map to physical derivatives with J^{-1},
//     3. exchange the two transposed strain entries with the element's other
//        two lanes by warp shuffles, form tau = eta (grad u + grad u^T),
//     4. pull back with J^{-T} and scatter with Dh^T into a Gauss-point
//        accumulator, then apply B^T three times to get nodal contributions.
//   This is mathematically the reference's sum-factorised element action
//   (src/stokes_operators_tensor.c:40-288, src/stokes_operators_cuda.cu:79-159)
//   re-associated through the Gauss-point values; it needs ~1/3 fewer flops
//   and no cross-lane traffic except 2 shuffles per Gauss point.
//   The nodal contributions are added into a shared node tile (shared-memory
//   atomic adds, accumulate_tile), and the tile is written to y:
//   plain stores for nodes no other CTA touches, atomicAdd for nodes on brick
//   faces shared with neighbouring bricks.
//
// Geometry paths
//   AFFINE : setup stores per element J^{-1} of the element centre (9) and
//            eta*w*detJ per Gauss point (27) in brick order; exact for
//            parallelepipeds, the reference's low-order operator otherwise.
//   general: the Jacobian of every Gauss point is recomputed per apply from
//            the element's Gauss-point coordinates (stokes_kernels.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace p3d {

// ---------------------------------------------------------------- tables --
// Q2 Lagrange basis (nodes -1,0,1) at the Gauss points -s,0,s (s = sqrt(3/5)):
// row 0 = [B0, B1, B2], row 1 = [0,1,0], row 2 = [B2, B1, B0].
#define P3D_B0 0.68729833462074168852
#define P3D_B1 0.4
#define P3D_B2 (-0.087298334620741688518)
// Lagrange derivative on the Gauss nodes: row 0 = [H0,H1,H2],
// row 1 = [-H3, 0, H3], row 2 = [-H2, -H1, -H0].
#define P3D_H0 (-1.9364916731037084426)
#define P3D_H1 2.5819888974716112568
#define P3D_H2 (-0.6454972243679028142)
#define P3D_H3 0.6454972243679028142
// 1-D Gauss weights 5/9, 8/9, 5/9
#define P3D_W0 0.55555555555555555556
#define P3D_W1 0.88888888888888888889

constexpr int TX = 5, TY = 2, EPW = TX * TY; // elements per warp layer

template <typename T> __device__ __forceinline__ T cst(double v) { return (T)v; }

// nodes -> Gauss points along one line
template <typename T> __device__ __forceinline__ void interp3(T &a, T &b, T &c)
{
  T o0 = cst<T>(P3D_B0) * a + cst<T>(P3D_B1) * b + cst<T>(P3D_B2) * c;
  T o2 = cst<T>(P3D_B2) * a + cst<T>(P3D_B1) * b + cst<T>(P3D_B0) * c;
  a = o0; c = o2; // b unchanged (centre row is the identity)
}
// Gauss points -> nodes (transpose) along one line
template <typename T> __device__ __forceinline__ void interp3T(T &a, T &b, T &c)
{
  T n0 = cst<T>(P3D_B0) * a + cst<T>(P3D_B2) * c;
  T n1 = cst<T>(P3D_B1) * (a + c) + b;
  T n2 = cst<T>(P3D_B2) * a + cst<T>(P3D_B0) * c;
  a = n0; b = n1; c = n2;
}
// derivative at Gauss point q of the quadratic through (v0,v1,v2) on the Gauss nodes
template <typename T> __device__ __forceinline__ T dcol(int q, T v0, T v1, T v2)
{
  if (q == 0) return cst<T>(P3D_H0) * v0 + cst<T>(P3D_H1) * v1 + cst<T>(P3D_H2) * v2;
  if (q == 1) return cst<T>(P3D_H3) * (v2 - v0);
  return -(cst<T>(P3D_H2) * v0 + cst<T>(P3D_H1) * v1 + cst<T>(P3D_H0) * v2);
}
// transpose of dcol: r_a += Dh[q][a] s
template <typename T> __device__ __forceinline__ void dcolT(int q, T s, T &r0, T &r1, T &r2)
{
  if (q == 0) { r0 += cst<T>(P3D_H0) * s; r1 += cst<T>(P3D_H1) * s; r2 += cst<T>(P3D_H2) * s; }
  else if (q == 1) { r0 -= cst<T>(P3D_H3) * s; r2 += cst<T>(P3D_H3) * s; }
  else { r0 -= cst<T>(P3D_H2) * s; r1 -= cst<T>(P3D_H1) * s; r2 -= cst<T>(P3D_H0) * s; }
}
__host__ __device__ __forceinline__ double w1d(int i) { return i == 1 ? P3D_W1 : P3D_W0; }

// in-place tensor interpolation of a [27] array (x fastest)
template <typename T> __device__ __forceinline__ void interp27(T v[27])
{
#pragma unroll
  for (int l = 0; l < 9; l++) interp3(v[3 * l + 0], v[3 * l + 1], v[3 * l + 2]);
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int a = 0; a < 3; a++) interp3(v[a + 9 * c], v[a + 3 + 9 * c], v[a + 6 + 9 * c]);
#pragma unroll
  for (int l = 0; l < 9; l++) interp3(v[l], v[l + 9], v[l + 18]);
}
template <typename T> __device__ __forceinline__ void interp27T(T v[27])
{
#pragma unroll
  for (int l = 0; l < 9; l++) interp3T(v[l], v[l + 9], v[l + 18]);
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int a = 0; a < 3; a++) interp3T(v[a + 9 * c], v[a + 3 + 9 * c], v[a + 6 + 9 * c]);
#pragma unroll
  for (int l = 0; l < 9; l++) interp3T(v[3 * l + 0], v[3 * l + 1], v[3 * l + 2]);
}

// --------------------------------------------------------------- params ---
template <typename T> struct TileArgs {
  int mx, my, mz;          // local elements
  int gx, gy, gz;          // ghosted lattice extent
  int ox, oy, oz;          // lattice index of element (0,0,0)'s first node
  int ntx, nty, ntz;       // bricks per direction
  uint32_t dir;            // Dirichlet bits restricted to global faces
  int bc;                  // 0 raw element apply, 1 MatMult contract
  const T *__restrict__ x; // velocity in
  T *__restrict__ y;       // velocity out (+=)
  const T *__restrict__ coords;
  const T *__restrict__ kdat; // brick-ordered coefficients
  const T *__restrict__ kgq;  // brick-ordered Gauss-point coordinates (general FP64 path)
  const T *__restrict__ p;    // pressure in  (A12)
  T *__restrict__ yp;         // pressure out (A21)
  int diag;                   // diagonal kernel: 1 -> Dirichlet slots = 1
  int overwrite;              // 1: y is zero on entry and not read (y = A x); 0: y += A x
  int brick0;                 // first brick of the launch (z-chunked launches)
};

// The tile arguments of up to P3D_GROUP_MAX operators of one mesh shape,
// passed by value to a grouped launch (kernel parameters, no device table).
#ifndef P3D_GROUP_MAX
#define P3D_GROUP_MAX 32
#endif
template <typename T> struct TileGroup {
  TileArgs<T> a[P3D_GROUP_MAX];
};

__device__ __forceinline__ bool is_dirichlet(uint32_t m, int ix, int iy, int iz, int ox, int oy, int oz, int ex,
                                             int ey, int ez, int comp)
{
  if (!m) return false;
  bool r = false;
  r |= (ix == ox) && ((m >> (0 + comp)) & 1u);
  r |= (ix == ex) && ((m >> (3 + comp)) & 1u);
  r |= (iy == oy) && ((m >> (6 + comp)) & 1u);
  r |= (iy == ey) && ((m >> (9 + comp)) & 1u);
  r |= (iz == oz) && ((m >> (12 + comp)) & 1u);
  r |= (iz == ez) && ((m >> (15 + comp)) & 1u);
  return r;
}

template <int NW> struct Brick {
  static constexpr int TZ = NW;
  static constexpr int NX = 2 * TX + 1, NY = 2 * TY + 1, NZ = 2 * NW + 1;
  static constexpr int NN = NX * NY * NZ;
  static constexpr int NE = TX * TY * NW;
  // node tiles in shared memory: rows of NX nodes x 3 components (33 values)
  // stored with a stride of 34, so that the 30 lanes of a warp, which read
  // nodes 2 apart in x and rows 2 apart in y, meet in at most 2 of the 16
  // 8-byte banks per half-warp (3 with stride 33)
  static constexpr int RS = 3 * NX + 1;           // row stride
  static constexpr int PL = NY * RS;              // node-plane stride
  static constexpr int TILE = NZ * PL;            // values of one node tile
};
// offset of node n (0..26) of the element at brick slot (a, b, c) in a node tile
template <int NW> __device__ __forceinline__ int tile_node(int a, int b, int c, int n)
{
  using BK = Brick<NW>;
  return 3 * (2 * a + n % 3) + BK::RS * ((2 * b + (n / 3) % 3) + BK::NY * (2 * c + n / 9));
}

// Brick geometry for blockIdx.x
struct BrickPos {
  int e0x, e0y, e0z;  // first element
  int ax, ay, az;     // elements actually present
  int n0x, n0y, n0z;  // lattice index of the brick's first node
  int tx, ty, tz;
  bool on_face; // brick touches a face of the local block
};
template <typename T, int NW> __device__ __forceinline__ BrickPos brick_pos(const TileArgs<T> &A)
{
  BrickPos b;
  int t = blockIdx.x + A.brick0;
  b.tx = t % A.ntx;
  b.ty = (t / A.ntx) % A.nty;
  b.tz = t / (A.ntx * A.nty);
  b.e0x = b.tx * TX; b.e0y = b.ty * TY; b.e0z = b.tz * NW;
  b.ax = min(TX, A.mx - b.e0x); b.ay = min(TY, A.my - b.e0y); b.az = min(NW, A.mz - b.e0z);
  b.n0x = A.ox + 2 * b.e0x; b.n0y = A.oy + 2 * b.e0y; b.n0z = A.oz + 2 * b.e0z;
  b.on_face = b.e0x == 0 || b.e0y == 0 || b.e0z == 0 || b.e0x + b.ax == A.mx || b.e0y + b.ay == A.my ||
              b.e0z + b.az == A.mz;
  return b;
}

// ------------------------------------------------------ async staging ---
// cp.async global -> shared copies: every load of a brick is in flight at once
// (no register round trip); src_bytes = 0 zero-fills the destination.
template <int BYTES> __device__ __forceinline__ void cp_async(void *smem, const void *gmem, int src_bytes)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
  else if (BYTES == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Stage a 3-component node field of the brick, row by row (a row = 2TX+1
// nodes along x = 33 contiguous values in global memory), one warp per row,
// lane l copying columns l and l+32.  mask: zero the Dirichlet entries
// (MatMult column convention); only bricks on a Dirichlet face test entries.
template <typename T, int NW>
__device__ __forceinline__ void stage_nodes(const TileArgs<T> &A, const BrickPos &b, const T *__restrict__ src, T *s,
                                            bool mask)
{
  using BK = Brick<NW>;
  constexpr int NROWS = BK::NY * BK::NZ;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nax = 2 * b.ax + 1, nay = 2 * b.ay + 1, naz = 2 * b.az + 1;
  const int li0 = lane / 3, c0 = lane - 3 * li0; // column `lane`
  const bool ok0 = li0 < nax, ok1 = lane == 0 && 10 < nax; // column 32 = node 10, comp 2
  const bool domask = mask && A.dir && b.on_face;
  const int exn = A.ox + 2 * A.mx, eyn = A.oy + 2 * A.my, ezn = A.oz + 2 * A.mz;
  for (int row = warp; row < NROWS; row += NW) {
    const int lj = row % BK::NY, lk = row / BK::NY;
    if (lj >= nay || lk >= naz) continue;
    const int iy = b.n0y + lj, iz = b.n0z + lk;
    const T *gr = src + 3 * ((size_t)b.n0x + (size_t)A.gx * ((size_t)iy + (size_t)A.gy * (size_t)iz));
    T *sr = s + row * BK::RS;
    bool m0 = ok0, m1 = ok1;
    if (domask) {
      m0 = m0 && !is_dirichlet(A.dir, b.n0x + li0, iy, iz, A.ox, A.oy, A.oz, exn, eyn, ezn, c0);
      m1 = m1 && !is_dirichlet(A.dir, b.n0x + 10, iy, iz, A.ox, A.oy, A.oz, exn, eyn, ezn, 2);
    }
    cp_async<sizeof(T)>(sr + lane, m0 ? (const void *)(gr + lane) : (const void *)src, m0 ? (int)sizeof(T) : 0);
    if (lane == 0) cp_async<sizeof(T)>(sr + 32, m1 ? (const void *)(gr + 32) : (const void *)src, m1 ? (int)sizeof(T) : 0);
  }
}

// contiguous, 16-byte aligned block (brick-ordered coefficients)
template <typename T> __device__ __forceinline__ void stage_block(const T *__restrict__ g, T *s, int n)
{
  const int n16 = (n * (int)sizeof(T)) / 16;
  for (int i = threadIdx.x; i < n16; i += blockDim.x)
    cp_async<16>(reinterpret_cast<char *>(s) + 16 * i, reinterpret_cast<const char *>(g) + 16 * i, 16);
  for (int i = n16 * (16 / (int)sizeof(T)) + threadIdx.x; i < n; i += blockDim.x)
    cp_async<sizeof(T)>(s + i, g + i, (int)sizeof(T));
}

// Add the lane's 27 nodal contributions r[] into the brick's node tile s_acc
// (zeroed by the caller) with shared-memory atomic adds: every lane adds at
// once, and the few nodes that neighbouring elements share are serialised by
// the hardware (measured faster than parity classes taking turns).  Must be
// reached by every thread of the CTA.
template <typename T, int NW>
__device__ __forceinline__ void accumulate_tile(T *s_acc, const T r[27], int a, int bb, int c, int f, bool doit)
{
  using BK = Brick<NW>;
  T *base = s_acc + tile_node<NW>(a, bb, c, 0) + f;
  if (doit) {
#pragma unroll
    for (int n = 0; n < 27; n++) atomicAdd(base + 3 * (n % 3) + BK::RS * ((n / 3) % 3) + (n / 9) * BK::PL, r[n]);
  }
  __syncthreads();
}

// Write the accumulated brick tile into y: y = y_staged + acc for nodes no
// other CTA touches, atomicAdd (fire-and-forget reduction) for nodes on
// brick faces shared with a neighbouring brick, Dirichlet rows by the owner.
// rowmode: 0 -> Dirichlet rows get x (A11 / full operator), 1 -> 0 (A12), 2 -> 1 (diagonal)
template <typename T, int NW>
__device__ __forceinline__ void write_tile(const TileArgs<T> &A, const BrickPos &b, const T *s_acc, const T *s_y,
                                           int rowmode)
{
  using BK = Brick<NW>;
  constexpr int NROWS = BK::NY * BK::NZ;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nax = 2 * b.ax + 1, nay = 2 * b.ay + 1, naz = 2 * b.az + 1;
  const int exn = A.ox + 2 * A.mx, eyn = A.oy + 2 * A.my, ezn = A.oz + 2 * A.mz;
  const bool lo_x = b.tx > 0, lo_y = b.ty > 0, lo_z = b.tz > 0;
  const bool hi_x = b.e0x + b.ax < A.mx, hi_y = b.e0y + b.ay < A.my, hi_z = b.e0z + b.az < A.mz;
  const bool dobc = A.bc && A.dir && b.on_face;
  // the (at most two) columns of this lane
  const int li0 = lane / 3, f0 = lane - 3 * li0;
  const bool ok0 = li0 < nax, ok1 = lane == 0 && 10 < nax;
  const bool xs0 = (li0 == 0 && lo_x) || (li0 == nax - 1 && hi_x), xs1 = (10 == nax - 1 && hi_x);
  const bool own0 = li0 > 0 || !lo_x, own1 = true;
  for (int row = warp; row < NROWS; row += NW) {
    const int lj = row % BK::NY, lk = row / BK::NY;
    if (lj >= nay || lk >= naz) continue;
    const int iy = b.n0y + lj, iz = b.n0z + lk;
    const size_t base = 3 * ((size_t)b.n0x + (size_t)A.gx * ((size_t)iy + (size_t)A.gy * (size_t)iz));
    const bool rs = (lj == 0 && lo_y) || (lj == nay - 1 && hi_y) || (lk == 0 && lo_z) || (lk == naz - 1 && hi_z);
    const bool rown = (lj > 0 || !lo_y) && (lk > 0 || !lo_z);
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const bool ok = k ? ok1 : ok0;
      if (!ok) continue;
      const int col = k ? 32 : lane, li = k ? 10 : li0, f = k ? 2 : f0;
      const size_t g = base + col;
      if (dobc && is_dirichlet(A.dir, b.n0x + li, iy, iz, A.ox, A.oy, A.oz, exn, eyn, ezn, f)) {
        if (rown && (k ? own1 : own0)) A.y[g] = rowmode == 0 ? A.x[g] : (rowmode == 1 ? (T)0 : (T)1);
        continue;
      }
      const T v = s_acc[row * BK::RS + col];
      if (rs || (k ? xs1 : xs0)) atomicAdd(A.y + g, v);
      else A.y[g] = A.overwrite ? v : s_y[row * BK::RS + col] + v;
    }
  }
}

} // namespace p3d
