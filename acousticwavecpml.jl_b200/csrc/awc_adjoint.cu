// Discrete adjoint of the CPML time step, with checkpointing, for the
// gradient of a least-squares trace misfit with respect to c² and for the
// transpose of the source-to-trace map.
//
// The forward step t (0-based, awc_kernels.cuh) maps the state
// (p_{t-1}, p_t, ψ_t, ξ_t) to (p_t, p_{t+1}, ψ_{t+1}, ξ_{t+1}); per axis and
// CPML side, with faces e = 0..h between nodes c_e and c_e + 1 and band nodes
// c with entry q = 1..h (c = q + off, off = 0 on the left, n - h - 2 on the
// right):
//   ψ_{t+1}[e]  = bKh_e ψ_t[e] + ah_e (p_t[c_e + 1] - p_t[c_e]) / d
//   ξ_{t+1}[q-1] = bK_{q-1} ξ_t[q-1] + a_{q-1} (D2 p_t(c) + (ψ_{t+1}[q] - ψ_{t+1}[q-1]) / d)
//   p_{t+1}(c)  = 2 p_t(c) - p_{t-1}(c)
//                 + F(c) (Σ_axes D2 p_t(c) + Σ_bands ((ψ_{t+1}[q] - ψ_{t+1}[q-1]) / d + ξ_{t+1}[q-1]))
//                 + S_t(c),                  traces_t[r] = p_{t+1}(c_r),
// with F = dt² c². For fixed F this is linear in the state. Its exact
// transpose, run backwards in time with adjoint fields λ (of p), μ (of ψ) and
// ν (of ξ), is, for interior nodes c:
//   λ_{t+1}(c) = R_t(c) + 2 λ_{t+2}(c) - λ_{t+3}(c)
//                + Σ_axes D2ᵀ[F λ_{t+2} + a ν_{t+2}](c)
//                + Σ_bands (ah_{e1} μ_{t+2}[e1] - ah_{e2} μ_{t+2}[e2]) / d
//     (e1, e2: the faces left and right of c; R_t: the trace residuals of
//     step t at the receiver nodes),
//   ν_{t+1}[q-1] = bK_{q-1} ν_{t+2}[q-1] + F(c) λ_{t+1}(c),
//   μ_{t+1}[e]   = bKh_e μ_{t+2}[e] + (w_e - w_{e+1}) / d,
//     w_q = a_{q-1} ν_{t+1}[q-1] + F(c_q) λ_{t+1}(c_q) (0 outside q = 1..h),
// and dJ/dF(c) = Σ_t λ_{t+1}(c) B_t(c), where B_t is the bracket multiplying
// F. At a node outside every active CPML band that bracket is the Laplacian
// of p_t, Σ_axes D2 p_t(c), evaluated from the stored p_t in the working
// precision; inside
// a band it also holds the ψ and ξ terms, and B_t = (p_{t+1} - 2 p_t + p_{t-1}
// - S_t)(c) / F(c) there. (The difference form divides a second difference
// in time, about (ω dt)² ≈ 1e-3 of p, by F, and at a source node subtracts
// the injected value from it: in FP32 its rounding error dominates the
// gradient near sources, which the Laplacian form avoids.) Rim nodes carry no
// adjoint: their values never depend on the interior or on c². Sides whose
// recursion is trivial (the free top) feed nothing back and are skipped, as
// in the forward. Bands must not overlap (n >= 2 halo + 2 on every axis with
// an active side).
//
// Checkpointing: the forward run saves the full state every k steps; the
// backward pass, segment by segment from the last, restores a checkpoint,
// recomputes the segment's pressure fields and runs the adjoint steps of the
// segment in reverse.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../../include/awcpml.h"
#include "awc_ctx.h"
#include "awc_kernels.cuh"

namespace awc {

// Parameters of one adjoint step t (the kernels compute λ_{t+1}). The band
// state advances inside the same launch: a band node forms ν_{t+2} and
// μ_{t+2} of its own entries and faces from ν_{t+3}, μ_{t+3} and
// G_{t+2} = F λ_{t+2}, as the update formulas above give them, and, for its
// λ_{t+1}, also those of its axis neighbours (the same pinned arithmetic, so
// the values agree bitwise with what their owners store). G is formed where
// it is used, from F and λ_{t+2}.
template <typename T>
struct AdjStep {
  int32_t nx, ny, nz, halo;
  int64_t px, plane;
  T inv_d[3], inv_d2[3];
  const T* F;
  const T* lam2;   // λ_{t+2}
  T* lam;          // in: λ_{t+3} less the residuals of step t; out: λ_{t+1}
  const T* pm1;    // p_{t-1}, p_t, p_{t+1} (gradient mode)
  const T* p0;
  const T* pp1;
  double* grad;    // dJ/dF accumulator (gradient mode)
  const T* nu_in[3][2];  // ν_{t+3} (layout of ξ)
  T* nu_out[3][2];       // ν_{t+2}
  const T* mu_in[3][2];  // μ_{t+3} (layout of ψ)
  T* mu_out[3][2];       // μ_{t+2}
  // per axis and side: {bK_e, a_e} of the h on-grid entries and {bKh_f,
  // ah_f} of the h + 1 half-grid faces, as pairs
  const typename Vec2<T>::type* nuc[3][2];
  const typename Vec2<T>::type* muc[3][2];
  int32_t active[3][2];
  int32_t off[3][2];     // band node c has entry q = c - off
  // nodes farther than one node from every active band (the core kernel);
  // the TMA-fed core kernel tiles it from x = core_x (a 16-byte-aligned
  // origin at or below core.x0) in z chunks of `zchunk` planes
  Box core;
  int32_t core_x, zchunk;
  int32_t* err;  // set to 1 when a bounded device wait runs out
  // disjoint boxes covering the other interior nodes (the shell kernel); box
  // b owns blocks [box_blk[b], box_blk[b+1]). Box.kind = zx + 3 zy + 9 zz
  // names the band zone of its nodes per axis (0 none, 1 next to or in the
  // left band, 2 the right one); kind ADJ_GENERIC boxes test every node.
  int32_t nbox;
  Box box[27];
  int32_t box_blk[28];
  // ceil(2^32 / d) for the box width and for its column blocks per plane:
  // x / d = (x m) >> 32 exactly when x d < 2^32 for every quotient the
  // kernel forms (fastdiv set; else it divides)
  uint64_t box_mw[27], box_mncb[27];
  int32_t fastdiv;
};
constexpr int ADJ_GENERIC = 27;
// with the five tensor maps of the TMA-fed kernel, within the 4 KB of kernel
// parameters
static_assert(sizeof(AdjStep<double>) + 5 * 128 <= 4096, "AdjStep too large");

// Element index of entry 0 of the band array (`layers` entries along axis a)
// at the node (i, j, k), and the step from one entry to the next: x
// (layers, ny, nz); y (px, layers, nz); z (px, ny, layers).
template <typename I, typename T>
__device__ __forceinline__ I band_base(const AdjStep<T>& A, int a, int layers, int i, int j,
                                       int k) {
  if (a == 0) return (I)layers * ((I)j + (I)A.ny * (I)k);
  if (a == 1) return (I)i + (I)A.px * (I)layers * (I)k;
  return (I)i + (I)A.px * (I)j;
}
template <typename I, typename T>
__device__ __forceinline__ I band_step(const AdjStep<T>& A, int a) {
  return a == 0 ? (I)1 : a == 1 ? (I)A.px : (I)A.plane;
}

// The band part of λ_{t+1} along axis a from side s at a node with entry
// q in [0, h+1] (q = 0 and h+1 are the nodes next to the band), given
// G_{t+2} at the nodes c-1, c, c+1 of the axis (m = 0, 1, 2; entries q-1,
// q, q+1; ν index e = q-2+m):
//   ν_{t+2}[e] = bK_e ν_{t+3}[e] + G,   w = a_e ν_{t+2}[e] + G,
//   μ_{t+2}[f] = bKh_f μ_{t+3}[f] + (w_f - w_{f+1}) / d   (faces f = q-1, q),
// result (a ν(c+1) - 2 a ν(c) + a ν(c-1)) / d² + (ah μ[q-1] - ah μ[q]) / d.
// The node stores ν_{t+2}[q-1] and μ_{t+2}[q] when 1 <= q <= h, and
// μ_{t+2}[0] when q = 1.
template <typename T, typename I>
__device__ __forceinline__ T adj_side(const AdjStep<T>& A, int a, int s, int q, int i, int j,
                                      int k, T gm, T gc, T gp) {
  using V2 = typename Vec2<T>::type;
  const int h = A.halo;
  const I step = band_step<I>(A, a);
  const I nb = band_base<I>(A, a, h, i, j, k), mb = band_base<I>(A, a, h + 1, i, j, k);
  const V2* __restrict__ nuc = A.nuc[a][s];
  const T* __restrict__ nu_in = A.nu_in[a][s];
  const T gv[3] = {gm, gc, gp};
  T w[3], anu[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const int e = q - 2 + m;
    w[m] = T(0);
    anu[m] = T(0);
    if (e >= 0 && e < h) {
      const V2 c = __ldg(nuc + e);  // {bK, a}
      const T nu = fma(c.x, __ldg(nu_in + nb + (I)e * step), gv[m]);
      anu[m] = mul_rn(c.y, nu);
      w[m] = fma(c.y, nu, gv[m]);
      if (m == 1) A.nu_out[a][s][nb + (I)e * step] = nu;
    }
  }
  const T inv_d = A.inv_d[a];
  const V2* __restrict__ muc = A.muc[a][s];
  const T* __restrict__ mu_in = A.mu_in[a][s];
  T* __restrict__ mu_out = A.mu_out[a][s];
  T f = T(0);
  if (q >= 1) {  // face q - 1
    const int e = q - 1;
    const V2 c = __ldg(muc + e);  // {bKh, ah}
    const T mu = fma(c.x, __ldg(mu_in + mb + (I)e * step), mul_rn(inv_d, w[0] - w[1]));
    f = mul_rn(c.y, mu);
    if (q == 1) mu_out[mb] = mu;
  }
  if (q <= h) {  // face q
    const V2 c = __ldg(muc + q);
    const T mu = fma(c.x, __ldg(mu_in + mb + (I)q * step), mul_rn(inv_d, w[1] - w[2]));
    f = f - mul_rn(c.y, mu);
    if (q >= 1) mu_out[mb + (I)q * step] = mu;
  }
  const T acc = (anu[2] - T(2) * anu[1]) + anu[0];
  return fma(A.inv_d2[a], acc, mul_rn(inv_d, f));
}

// G_{t+2} = F λ_{t+2} at node o + d.
template <typename T, typename I>
__device__ __forceinline__ T adj_g(const AdjStep<T>& A, I o) {
  return mul_rn(__ldg(A.F + o), __ldg(A.lam2 + o));
}

// The node update at o: λ_{t+1} = 2 λ_{t+2} - λ_{t+3} + the transposed
// stencil lap of G_{t+2} + band, and the gradient accumulation
// dJ/dF += λ_{t+1} B_t with B_t the Laplacian of p_t (in the working
// precision) at nodes outside every active band, (p_{t+1} - 2 p_t + p_{t-1})
// / F (in double) inside one, where adj_sources removes the source term.
template <typename T, typename I, int ND, bool GRAD>
__device__ __forceinline__ void adj_update(const AdjStep<T>& A, I o, T l2, T f, T lap, T band,
                                           bool in_band) {
  const T lam = (T(2) * l2 - A.lam[o]) + (lap + band);
  if (GRAD) {
    const T* __restrict__ P = A.p0;
    const T c = __ldg(P + o);
    double b;
    if (in_band) {
      // 1/F by Newton's iteration r <- r (2 - F r) from the single-precision
      // reciprocal (two steps: ~1e-14, then below double rounding)
      const double fd = (double)f;
      double r = (double)__frcp_rn((float)fd);
      r = r * fma(-fd, r, 2.0);
      r = r * fma(-fd, r, 2.0);
      b = (((double)__ldg(A.pp1 + o) - 2.0 * (double)c) + (double)__ldg(A.pm1 + o)) * r;
    } else {
      const I px = (I)A.px;
      T bl = second_diff(__ldg(P + o - 1), c, __ldg(P + o + 1), A.inv_d2[0]) +
             second_diff(__ldg(P + o - px), c, __ldg(P + o + px), A.inv_d2[1]);
      if (ND == 3) {
        const I pl = (I)A.plane;
        bl += second_diff(__ldg(P + o - pl), c, __ldg(P + o + pl), A.inv_d2[2]);
      }
      b = (double)bl;
    }
    A.grad[o] += (double)lam * b;
  }
  A.lam[o] = lam;
}

// Nodes of the core box: blocks of 32 x 8 (x, y) nodes of one z plane.
template <typename T, typename I, int ND, bool GRAD>
__global__ void __launch_bounds__(256) adj_core(const __grid_constant__ AdjStep<T> A) {
  const int i = A.core.x0 + blockIdx.x * 32 + threadIdx.x;
  const int j = A.core.y0 + blockIdx.y * 8 + threadIdx.y;
  const int k = ND == 3 ? A.core.z0 + (int)blockIdx.z : 0;
  if (i > A.core.x1 || j > A.core.y1) return;
  const I px = (I)A.px, pl = (I)A.plane;
  const I o = (I)i + px * (I)j + pl * (I)k;
  const T f = __ldg(A.F + o), l2 = __ldg(A.lam2 + o);
  const T gc = mul_rn(f, l2);
  T lap = second_diff(adj_g(A, o - 1), gc, adj_g(A, o + 1), A.inv_d2[0]) +
          second_diff(adj_g(A, o - px), gc, adj_g(A, o + px), A.inv_d2[1]);
  if (ND == 3) lap += second_diff(adj_g(A, o - pl), gc, adj_g(A, o + pl), A.inv_d2[2]);
  adj_update<T, I, ND, GRAD>(A, o, l2, f, lap, T(0), false);
}

// One shell node whose band zone per axis is ZX, ZY, ZZ (0 none, 1 left, 2
// right; 3 unknown: both sides tested at run time).
template <typename T, typename I, int ND, bool GRAD, int ZX, int ZY, int ZZ>
__device__ __forceinline__ void adj_shell_node(const AdjStep<T>& A, int i, int j, int k) {
  const I px = (I)A.px, pl = (I)A.plane;
  const I o = (I)i + px * (I)j + pl * (I)k;
  const T f = __ldg(A.F + o), l2 = __ldg(A.lam2 + o);
  const T gc = mul_rn(f, l2);
  const T g[3][2] = {{adj_g(A, o - 1), adj_g(A, o + 1)},
                     {adj_g(A, o - px), adj_g(A, o + px)},
                     {ND == 3 ? adj_g(A, o - pl) : T(0), ND == 3 ? adj_g(A, o + pl) : T(0)}};
  T lap = second_diff(g[0][0], gc, g[0][1], A.inv_d2[0]) +
          second_diff(g[1][0], gc, g[1][1], A.inv_d2[1]);
  if (ND == 3) lap += second_diff(g[2][0], gc, g[2][1], A.inv_d2[2]);
  const int h = A.halo;
  const int c[3] = {i, j, k}, zone[3] = {ZX, ZY, ZZ};
  T band = T(0);
  bool in_band = false;
#pragma unroll
  for (int a = 0; a < ND; ++a) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      if (zone[a] != 3 && zone[a] != s + 1) continue;
      int q = c[a] - A.off[a][s];
      if (zone[a] == 3 && (!A.active[a][s] || q < 0 || q > h + 1)) continue;
      in_band = in_band || (q >= 1 && q <= h);
      band += adj_side<T, I>(A, a, s, q, i, j, k, g[a][0], gc, g[a][1]);
    }
  }
  adj_update<T, I, ND, GRAD>(A, o, l2, f, lap, band, in_band);
}

// Nodes of the shell boxes: a box's (x, y) columns numbered row by row,
// l = (i - x0) + W (j - y0), in runs of 256 per block, one z plane per block;
// the block's box kind selects the body.
template <typename T, typename I, int ND, bool GRAD>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 4) adj_shell(const __grid_constant__ AdjStep<T> A) {
  // the box of this block: box_blk rises strictly, so a binary search
  const int blk = blockIdx.x;
  int b = 0, hi = A.nbox - 1;
  while (b < hi) {
    const int mid = (b + hi + 1) >> 1;
    if (A.box_blk[mid] <= blk)
      b = mid;
    else
      hi = mid - 1;
  }
  const Box& B = A.box[b];
  const int W = B.x1 - B.x0 + 1, ncol = W * (B.y1 - B.y0 + 1);
  const int ncb = (ncol + 255) / 256;
  const int r = blk - A.box_blk[b];
  const int kz = A.fastdiv ? (int)(((uint64_t)r * A.box_mncb[b]) >> 32) : r / ncb;
  const int l = (r - kz * ncb) * 256 + threadIdx.x;
  if (l >= ncol) return;
  const int jl = A.fastdiv ? (int)(((uint64_t)l * A.box_mw[b]) >> 32) : l / W;
  const int i = B.x0 + (l - jl * W), j = B.y0 + jl, k = ND == 3 ? B.z0 + kz : 0;
#define AWC_SHELL(zx, zy, zz) \
  case (zx) + 3 * (zy) + 9 * (zz): adj_shell_node<T, I, ND, GRAD, zx, zy, zz>(A, i, j, k); break;
  if (ND == 2) {
    switch (B.kind) {
      AWC_SHELL(1, 0, 0) AWC_SHELL(2, 0, 0) AWC_SHELL(0, 1, 0) AWC_SHELL(1, 1, 0)
      AWC_SHELL(2, 1, 0) AWC_SHELL(0, 2, 0) AWC_SHELL(1, 2, 0) AWC_SHELL(2, 2, 0)
      default: adj_shell_node<T, I, ND, GRAD, 3, 3, 0>(A, i, j, k);
    }
  } else {
    switch (B.kind) {
      AWC_SHELL(1, 0, 0) AWC_SHELL(2, 0, 0) AWC_SHELL(0, 1, 0) AWC_SHELL(1, 1, 0)
      AWC_SHELL(2, 1, 0) AWC_SHELL(0, 2, 0) AWC_SHELL(1, 2, 0) AWC_SHELL(2, 2, 0)
      AWC_SHELL(0, 0, 1) AWC_SHELL(1, 0, 1) AWC_SHELL(2, 0, 1) AWC_SHELL(0, 1, 1)
      AWC_SHELL(1, 1, 1) AWC_SHELL(2, 1, 1) AWC_SHELL(0, 2, 1) AWC_SHELL(1, 2, 1)
      AWC_SHELL(2, 2, 1) AWC_SHELL(0, 0, 2) AWC_SHELL(1, 0, 2) AWC_SHELL(2, 0, 2)
      AWC_SHELL(0, 1, 2) AWC_SHELL(1, 1, 2) AWC_SHELL(2, 1, 2) AWC_SHELL(0, 2, 2)
      AWC_SHELL(1, 2, 2) AWC_SHELL(2, 2, 2)
      default: adj_shell_node<T, I, ND, GRAD, 3, 3, 3>(A, i, j, k);
    }
  }
#undef AWC_SHELL
}

// Geometry of the TMA-fed core kernel (32 x TY threads, a 64 x 2TY tile of
// (x, y) nodes, 2 x 2 nodes per thread): one pipeline stage holds, for one z
// plane, the boxes (64 + 2A) x (2TY + 2) around the tile of λ_{t+2}, F and
// p_t (x apron A keeps the box origin 16-byte aligned), then the tile's
// λ_{t+3} (64 x 2TY) and gradient (64 x 2TY doubles).
template <typename T, int TY>
struct AdjTile {
  static constexpr int TX = 64;
  static constexpr int RY = 2 * TY;
  static constexpr int A = 16 / (int)sizeof(T);
  static constexpr int PW = TX + 2 * A;
  static constexpr int BOX = PW * (RY + 2) * (int)sizeof(T);
  static constexpr int BOX_PAD = (BOX + 127) / 128 * 128;
  static constexpr int IN_T = TX * RY * (int)sizeof(T);
  static constexpr int IN_D = TX * RY * 8;
  static constexpr int BYTES = 3 * BOX_PAD + IN_T + IN_D;
};

// The 2 x 2 values a thread reads from one box for its nodes and their x, y
// neighbours: rows r0 (y = j0) and r1, x aprons, rows above and below.
template <typename T>
struct Quad {
  typename Vec2<T>::type r0, r1, ym, yp;
  T xm0, xp0, xm1, xp1;
};
template <typename T>
__device__ __forceinline__ Quad<T> quad_at(const T* b, int c0, int pw) {
  using V2 = typename Vec2<T>::type;
  Quad<T> q;
  q.r0 = *reinterpret_cast<const V2*>(b + c0);
  q.r1 = *reinterpret_cast<const V2*>(b + c0 + pw);
  q.ym = *reinterpret_cast<const V2*>(b + c0 - pw);
  q.yp = *reinterpret_cast<const V2*>(b + c0 + 2 * pw);
  q.xm0 = b[c0 - 1];
  q.xp0 = b[c0 + 2];
  q.xm1 = b[c0 + pw - 1];
  q.xp1 = b[c0 + pw + 2];
  return q;
}
// Element-wise product of two quads (G = F λ at the same points).
template <typename T>
__device__ __forceinline__ Quad<T> quad_mul(const Quad<T>& f, const Quad<T>& l) {
  Quad<T> g;
  g.r0 = {mul_rn(f.r0.x, l.r0.x), mul_rn(f.r0.y, l.r0.y)};
  g.r1 = {mul_rn(f.r1.x, l.r1.x), mul_rn(f.r1.y, l.r1.y)};
  g.ym = {mul_rn(f.ym.x, l.ym.x), mul_rn(f.ym.y, l.ym.y)};
  g.yp = {mul_rn(f.yp.x, l.yp.x), mul_rn(f.yp.y, l.yp.y)};
  g.xm0 = mul_rn(f.xm0, l.xm0);
  g.xp0 = mul_rn(f.xp0, l.xp0);
  g.xm1 = mul_rn(f.xm1, l.xm1);
  g.xp1 = mul_rn(f.xp1, l.xp1);
  return g;
}
// x + y second differences of a quad at its four nodes (00, 01, 10, 11), in
// the order the per-node kernels use (x term + y term).
template <typename T>
__device__ __forceinline__ void quad_d2xy(const Quad<T>& q, T ix2, T iy2, T out[4]) {
  out[0] = second_diff(q.xm0, q.r0.x, q.r0.y, ix2) + second_diff(q.ym.x, q.r0.x, q.r1.x, iy2);
  out[1] = second_diff(q.r0.x, q.r0.y, q.xp0, ix2) + second_diff(q.ym.y, q.r0.y, q.r1.y, iy2);
  out[2] = second_diff(q.xm1, q.r1.x, q.r1.y, ix2) + second_diff(q.r0.x, q.r1.x, q.yp.x, iy2);
  out[3] = second_diff(q.r1.x, q.r1.y, q.xp1, ix2) + second_diff(q.r0.y, q.r1.y, q.yp.y, iy2);
}

// The core box streamed through shared memory: adj_core's arithmetic, node
// for node, in the gradient mode, with λ_{t+2}, F, p_t (boxes with a ring),
// λ_{t+3} and the gradient (the tile) staged by cp.async.bulk.tensor. Grid:
// x tiles of 64 nodes from core_x, y tiles of 2TY rows from core.y0, z
// chunks of `zchunk` planes from core.z0, numbered z chunk fastest. One
// elected thread loads planes k0-1 .. k1 into S stages, each with a "full"
// mbarrier (TMA bytes) and an "empty" one (one arrival per warp); plane k is
// computed from the stages of k-1, k, k+1, and its λ_{t+1} and gradient are
// stored as coalesced pairs. Every wait is bounded: on a timeout the block
// records it in *A.err and drains its loads in flight.
template <typename T, int TY, int S>
__global__ void __launch_bounds__(32 * TY) adj_core_tma(const __grid_constant__ CUtensorMap ml,
                                                        const __grid_constant__ CUtensorMap mf,
                                                        const __grid_constant__ CUtensorMap mp,
                                                        const __grid_constant__ CUtensorMap ml3,
                                                        const __grid_constant__ CUtensorMap mg,
                                                        const __grid_constant__ AdjStep<T> A) {
  using L = AdjTile<T, TY>;
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * L::BYTES);
  uint64_t* empty = full + S;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + S);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  const Box C = A.core;
  const int gz = gridDim.z, gx = gridDim.x;
  const int bz = blk % gz, bx = (blk / gz) % gx, by = blk / (gz * gx);
  const int x0 = A.core_x + bx * L::TX, y0 = C.y0 + by * L::RY;
  const int k0 = C.z0 + bz * A.zchunk;
  int k1 = k0 + A.zchunk;
  if (k1 > C.z1 + 1) k1 = C.z1 + 1;
  if (k0 >= k1) return;  // block-uniform
  const int nplanes = k1 - k0 + 2;  // planes k0-1 .. k1

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TY);
    }
    *abort = 0;
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int u) {  // use u: plane k0 - 1 + u into stage u % S
    const int s = u % S, m = k0 - 1 + u;
    unsigned char* st = smem + s * L::BYTES;
    const bool inner = m >= k0 && m < k1;
    mbar_expect_tx(&full[s], 3 * L::BOX + (inner ? L::IN_T + L::IN_D : 0));
    tma_load_3d(st, &ml, &full[s], x0 - L::A, y0 - 1, m);
    tma_load_3d(st + L::BOX_PAD, &mf, &full[s], x0 - L::A, y0 - 1, m);
    tma_load_3d(st + 2 * L::BOX_PAD, &mp, &full[s], x0 - L::A, y0 - 1, m);
    if (inner) {
      tma_load_3d(st + 3 * L::BOX_PAD, &ml3, &full[s], x0, y0, m);
      tma_load_3d(st + 3 * L::BOX_PAD + L::IN_T, &mg, &full[s], x0, y0, m);
    }
  };
  if (tid == 0)
    for (int u = 0; u < S && u < nplanes; ++u) issue(u);

  const int xa = x0 + 2 * tx, j0 = y0 + 2 * ty;
  const bool vx0 = xa >= C.x0 && xa <= C.x1, vx1 = xa + 1 >= C.x0 && xa + 1 <= C.x1;
  const bool vy0 = j0 <= C.y1, vy1 = j0 + 1 <= C.y1;
  const bool all4 = vx0 && vx1 && vy0 && vy1;
  const bool any = (vx0 || vx1) && vy0;
  const int64_t px = A.px, plane = A.plane;
  int64_t o = (int64_t)xa + px * j0 + plane * k0;
  const int c0 = (2 * ty + 1) * L::PW + 2 * tx + L::A;  // box index of (xa, j0)
  const int i0 = 2 * ty * L::TX + 2 * tx;               // tile index of (xa, j0)
  const T ix2 = A.inv_d2[0], iy2 = A.inv_d2[1], iz2 = A.inv_d2[2];

  bool ok = mbar_wait(&full[0], 0, abort) && mbar_wait(&full[1 % S], (1 / S) & 1, abort);
  int uc = 1;
  for (int k = k0; k < k1; ++k, ++uc, o += plane) {
    ok = ok && mbar_wait(&full[(uc + 1) % S], ((uc + 1) / S) & 1, abort);
    if (!ok) break;
    const T* sm = reinterpret_cast<const T*>(smem + ((uc - 1) % S) * L::BYTES);
    const T* sc = reinterpret_cast<const T*>(smem + (uc % S) * L::BYTES);
    const T* sp = reinterpret_cast<const T*>(smem + ((uc + 1) % S) * L::BYTES);
    constexpr int FO = L::BOX_PAD / (int)sizeof(T), PO = 2 * FO;  // F and p_t box offsets
    // G = F λ on the plane and its two z neighbours
    const Quad<T> lq = quad_at(sc, c0, L::PW);
    const Quad<T> gq = quad_mul(quad_at(sc + FO, c0, L::PW), lq);
    const V2 gm0 = {mul_rn(sm[FO + c0], sm[c0]), mul_rn(sm[FO + c0 + 1], sm[c0 + 1])};
    const V2 gm1 = {mul_rn(sm[FO + c0 + L::PW], sm[c0 + L::PW]),
                    mul_rn(sm[FO + c0 + L::PW + 1], sm[c0 + L::PW + 1])};
    const V2 gp0 = {mul_rn(sp[FO + c0], sp[c0]), mul_rn(sp[FO + c0 + 1], sp[c0 + 1])};
    const V2 gp1 = {mul_rn(sp[FO + c0 + L::PW], sp[c0 + L::PW]),
                    mul_rn(sp[FO + c0 + L::PW + 1], sp[c0 + L::PW + 1])};
    T lap[4];
    quad_d2xy(gq, ix2, iy2, lap);
    lap[0] += second_diff(gm0.x, gq.r0.x, gp0.x, iz2);
    lap[1] += second_diff(gm0.y, gq.r0.y, gp0.y, iz2);
    lap[2] += second_diff(gm1.x, gq.r1.x, gp1.x, iz2);
    lap[3] += second_diff(gm1.y, gq.r1.y, gp1.y, iz2);
    T b[4];
    const Quad<T> pq = quad_at(sc + PO, c0, L::PW);
    quad_d2xy(pq, ix2, iy2, b);
    b[0] += second_diff(sm[PO + c0], pq.r0.x, sp[PO + c0], iz2);
    b[1] += second_diff(sm[PO + c0 + 1], pq.r0.y, sp[PO + c0 + 1], iz2);
    b[2] += second_diff(sm[PO + c0 + L::PW], pq.r1.x, sp[PO + c0 + L::PW], iz2);
    b[3] += second_diff(sm[PO + c0 + L::PW + 1], pq.r1.y, sp[PO + c0 + L::PW + 1], iz2);
    // the tile's λ_{t+3} and gradient of this plane
    const T* l3s = reinterpret_cast<const T*>(smem + (uc % S) * L::BYTES + 3 * L::BOX_PAD);
    const double* gs = reinterpret_cast<const double*>(smem + (uc % S) * L::BYTES +
                                                       3 * L::BOX_PAD + L::IN_T);
    const V2 a0 = *reinterpret_cast<const V2*>(l3s + i0);
    const V2 a1 = *reinterpret_cast<const V2*>(l3s + i0 + L::TX);
    const double2 q0 = *reinterpret_cast<const double2*>(gs + i0);
    const double2 q1 = *reinterpret_cast<const double2*>(gs + i0 + L::TX);
    // this warp is done with stage uc - 1
    __syncwarp();
    if (tx == 0) mbar_arrive(&empty[(uc - 1) % S]);
    const T lam[4] = {(T(2) * lq.r0.x - a0.x) + (lap[0] + T(0)),
                      (T(2) * lq.r0.y - a0.y) + (lap[1] + T(0)),
                      (T(2) * lq.r1.x - a1.x) + (lap[2] + T(0)),
                      (T(2) * lq.r1.y - a1.y) + (lap[3] + T(0))};
    const double gr[4] = {q0.x + (double)lam[0] * (double)b[0], q0.y + (double)lam[1] * (double)b[1],
                          q1.x + (double)lam[2] * (double)b[2], q1.y + (double)lam[3] * (double)b[3]};
    if (all4) {
      *reinterpret_cast<V2*>(A.lam + o) = V2{lam[0], lam[1]};
      *reinterpret_cast<V2*>(A.lam + o + px) = V2{lam[2], lam[3]};
      *reinterpret_cast<double2*>(A.grad + o) = double2{gr[0], gr[1]};
      *reinterpret_cast<double2*>(A.grad + o + px) = double2{gr[2], gr[3]};
    } else if (any) {
      const bool v[4] = {vx0, vx1, vy1 && vx0, vy1 && vx1};
      const int64_t off[4] = {0, 1, px, px + 1};
#pragma unroll
      for (int n = 0; n < 4; ++n) {
        if (!v[n]) continue;
        A.lam[o + off[n]] = lam[n];
        A.grad[o + off[n]] = gr[n];
      }
    }
    if (tid == 0 && uc - 1 + S < nplanes) {
      if (!mbar_wait(&empty[(uc - 1) % S], ((uc - 1) / S) & 1, abort)) {
        ok = false;
        break;
      }
      issue(uc - 1 + S);
    }
  }
  if (!ok) {
    *abort = 1;
    atomicExch(A.err, 1);
    if (tid == 0) {
      const int issued = nplanes < uc - 1 + S ? nplanes : uc - 1 + S;
      for (int u = uc; u < issued; ++u) {
        for (int n = 0; n < 64; ++n)
          if (mbar_try_wait(&full[u % S], (u / S) & 1, 1000000u)) break;
      }
    }
  }
}

// λ_{t+3} -= R_t at the receiver nodes before the step kernels run (the
// residuals of step t enter λ_{t+1} = R_t + 2 λ_{t+2} - λ_{t+3} + ...), one
// thread per node, its receivers in receiver order.
template <typename T>
__global__ void adj_residuals(T* __restrict__ lam3, const int64_t* __restrict__ node,
                              const int32_t* __restrict__ off, const int32_t* __restrict__ ids,
                              int32_t nnode, const T* __restrict__ res_row) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  T v = lam3[node[n]];
  for (int e = off[n]; e < off[n + 1]; ++e) v -= res_row[ids[e]];
  lam3[node[n]] = v;
}

// The residual rows [nt][nrec] in the working precision from a column-major
// (nt x nrec) double array d: rows[t][r] = traces[t][r] - d[t + nt r] when
// traces is given (d = observed data), else d itself (the adjoint traces).
// 32 x 32 tiles through shared memory (coalesced on both sides); with traces,
// each block also writes its sum of res² / 2 to part[block].
template <typename T>
__global__ void __launch_bounds__(256) adj_residual_rows(const T* __restrict__ traces,
                                                         const double* __restrict__ d, int64_t nt,
                                                         int64_t nrec, T* __restrict__ rows,
                                                         double* __restrict__ part) {
  __shared__ double tile[32][33];
  __shared__ double wsum[8];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t r0 = (int64_t)blockIdx.x * 32, t0 = (int64_t)blockIdx.y * 32;
  for (int q = ty; q < 32; q += 8) {
    const int64_t t = t0 + tx, r = r0 + q;
    tile[q][tx] = (t < nt && r < nrec) ? d[t + nt * r] : 0.0;
  }
  __syncthreads();
  double acc = 0.0;
  for (int q = ty; q < 32; q += 8) {
    const int64_t t = t0 + q, r = r0 + tx;
    if (t < nt && r < nrec) {
      double v = tile[tx][q];
      if (traces) v = (double)traces[t * nrec + r] - v;
      rows[t * nrec + r] = (T)v;
      acc += 0.5 * v * v;
    }
  }
  if (!part) return;
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if (tx == 0) wsum[ty] = acc;
  __syncthreads();
  if (tx == 0 && ty == 0) {
    double b = 0.0;
    for (int w = 0; w < 8; ++w) b += wsum[w];
    part[blockIdx.x + (int64_t)gridDim.x * blockIdx.y] = b;
  }
}

// Per source (one thread, serial over sources for a fixed summation order):
// the adjoint of the injected value, λ_{t+1} at the source node, and the
// removal of the source term from the gradient bracket.
template <typename T>
__global__ void adj_sources(const T* __restrict__ lamn, const T* __restrict__ F,
                            const int64_t* __restrict__ node, const int8_t* __restrict__ in_band,
                            int32_t nsrc, const T* __restrict__ stf_row,
                            double* __restrict__ grad, T* __restrict__ out_row) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int s = 0; s < nsrc; ++s) {
    const int64_t o = node[s];
    if (o < 0) continue;  // rim source: no adjoint
    if (out_row) out_row[s] = lamn[o];
    // only band nodes use the difference form of the bracket, which holds S_t
    if (grad && in_band[s]) grad[o] -= (double)lamn[o] * (double)stf_row[s] / (double)F[o];
  }
}

__global__ void scale_unpitch(const double* __restrict__ src, double* __restrict__ dst,
                              int64_t n, int64_t nx, int64_t px, double scale) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c % nx, r = c / nx;
    dst[c] = scale * src[i + px * r];
  }
}

// dst (dense) += scale * src (pitched), each product rounded before the sum:
// the same arithmetic as scale_unpitch followed by a host-side sum.
__global__ void scale_unpitch_add(const double* __restrict__ src, double* __restrict__ dst,
                                  int64_t n, int64_t nx, int64_t px, double scale) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c % nx, r = c / nx;
    dst[c] = __dadd_rn(dst[c], __dmul_rn(scale, src[i + px * r]));
  }
}

template <typename T>
__global__ void to_double(const T* __restrict__ src, double* __restrict__ dst, int64_t n) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    dst[c] = (double)src[c];
}

}  // namespace awc

namespace {

#define ADJ_TRY(C, call)                                                          \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      cudaGetLastError();                                                         \
      return awc::fail((C), AWC_ERR_CUDA, cudaGetErrorString(e_));                \
    }                                                                             \
  } while (0)

// Device working memory of the adjoint, kept by the context between calls:
// a run asks for its blocks in a fixed order, and a later run of the same
// shape gets the same blocks back (no cudaMalloc/cudaFree, whose multi-GB
// checkpoint arena otherwise costs more than the run). A block of another
// size frees it and every later block. Contents are not kept: every run
// initialises what it reads.
struct DevMem {
  std::vector<std::pair<void*, size_t>> blocks;
  size_t next = 0;
  void* sum = nullptr;  // the multi-shot gradient sum, outside the per-call blocks
  size_t sum_bytes = 0;
  void begin() { next = 0; }
  void release() {
    for (auto& b : blocks) cudaFree(b.first);
    blocks.clear();
    next = 0;
    if (sum) cudaFree(sum);
    sum = nullptr;
    sum_bytes = 0;
  }
  cudaError_t get_sum(double** out, size_t bytes) {
    if (sum_bytes != bytes) {
      if (sum) cudaFree(sum);
      sum = nullptr;
      sum_bytes = 0;
      cudaError_t e = cudaMalloc(&sum, bytes);
      if (e != cudaSuccess) return e;
      sum_bytes = bytes;
    }
    *out = (double*)sum;
    return cudaSuccess;
  }
  ~DevMem() { release(); }
  template <typename P>
  cudaError_t get(P** out, size_t bytes) {
    bytes = std::max<size_t>(bytes, 16);
    if (next < blocks.size()) {
      if (blocks[next].second == bytes) {
        *out = (P*)blocks[next++].first;
        return cudaSuccess;
      }
      for (size_t k = next; k < blocks.size(); ++k) cudaFree(blocks[k].first);
      blocks.resize(next);
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      *out = nullptr;
      return e;
    }
    blocks.emplace_back(p, bytes);
    ++next;
    *out = (P*)p;
    return cudaSuccess;
  }
};

// The context's adjoint memory (created on first use).
DevMem& ctx_mem(awc_ctx* C) {
  if (!C->adj_mem) {
    DevMem* m = new DevMem();
    C->adj_mem = m;
    C->adj_release = [C]() {
      delete static_cast<DevMem*>(C->adj_mem);
      C->adj_mem = nullptr;
    };
  }
  DevMem& m = *static_cast<DevMem*>(C->adj_mem);
  m.begin();
  return m;
}

// Interior node groups: each unique interior node of `pos` with its ids.
struct Groups {
  std::vector<int64_t> node;
  std::vector<int32_t> off{0}, ids;
};

Groups group_nodes(const awc_problem* p, int64_t px, const int64_t* pos, int64_t cnt,
                   std::vector<int64_t>* per_item) {
  Groups G;
  std::unordered_map<int64_t, std::vector<int32_t>> m;
  std::vector<int64_t> order;
  const int64_t nz = p->ndim == 3 ? p->nz : 1;
  if (per_item) per_item->assign(cnt, -1);
  for (int64_t r = 0; r < cnt; ++r) {
    const int64_t i = pos[r] - 1, j = pos[r + cnt] - 1, k = p->ndim == 3 ? pos[r + 2 * cnt] - 1 : 0;
    const bool in = i >= 1 && i <= p->nx - 2 && j >= 1 && j <= p->ny - 2 &&
                    (p->ndim == 2 || (k >= 1 && k <= nz - 2));
    if (!in) continue;
    const int64_t node = i + px * (j + p->ny * k);
    if (per_item) (*per_item)[r] = node;
    auto f = m.find(node);
    if (f == m.end()) {
      order.push_back(node);
      m[node] = {(int32_t)r};
    } else {
      f->second.push_back((int32_t)r);
    }
  }
  for (int64_t node : order) {
    G.node.push_back(node);
    for (int32_t r : m[node]) G.ids.push_back(r);
    G.off.push_back((int32_t)G.ids.size());
  }
  return G;
}

// The adjoint's core box (nodes farther than one node from every active
// band) and the shell boxes around it. Per axis the interior splits into the
// left zone [1, h+1] (when the left side is active), the right zone
// [n-h-2, n-2] (when the right one is) and the core range between them; the
// shell is every product of zones but the core's (26 boxes in 3D, 8 in 2D),
// each with its zone code as kind. When the zones of an axis leave no core
// node between them, one generic box holds the whole interior.
template <typename T>
void adj_regions(awc::AdjStep<T>& A, int ndim) {
  const int64_t n[3] = {A.nx, A.ny, A.nz}, h = A.halo;
  int64_t lo[3][3], hi[3][3];  // [axis][zone]: 0 core, 1 left, 2 right
  bool split = true;
  for (int a = 0; a < 3; ++a) {
    for (int z = 1; z < 3; ++z) {
      lo[a][z] = 1;
      hi[a][z] = 0;  // empty
    }
    if (a >= ndim) {
      lo[a][0] = hi[a][0] = 0;
      continue;
    }
    lo[a][0] = 1;
    hi[a][0] = n[a] - 2;
    if (A.active[a][0]) {
      hi[a][1] = h + 1;
      lo[a][0] = h + 2;
    }
    if (A.active[a][1]) {
      lo[a][2] = n[a] - h - 2;
      hi[a][2] = n[a] - 2;
      hi[a][0] = n[a] - h - 3;
    }
    split = split && lo[a][0] <= hi[a][0];
  }
  A.nbox = 0;
  auto add = [&](int zx, int zy, int zz, int32_t kind) {
    if (lo[0][zx] > hi[0][zx] || lo[1][zy] > hi[1][zy] || lo[2][zz] > hi[2][zz]) return;
    A.box[A.nbox++] = awc::Box{(int32_t)lo[0][zx], (int32_t)hi[0][zx], (int32_t)lo[1][zy],
                               (int32_t)hi[1][zy], (int32_t)lo[2][zz], (int32_t)hi[2][zz], kind};
  };
  if (!split) {
    A.core = awc::Box{1, 0, 1, 0, 0, 0, 0};  // none
    for (int a = 0; a < ndim; ++a) {
      lo[a][0] = 1;
      hi[a][0] = n[a] - 2;
    }
    add(0, 0, 0, awc::ADJ_GENERIC);
  } else {
    A.core = awc::Box{(int32_t)lo[0][0], (int32_t)hi[0][0], (int32_t)lo[1][0],
                      (int32_t)hi[1][0], (int32_t)lo[2][0], (int32_t)hi[2][0], 0};
    for (int zz = 0; zz < (ndim == 3 ? 3 : 1); ++zz)
      for (int zy = 0; zy < 3; ++zy)
        for (int zx = 0; zx < 3; ++zx)
          if (zx || zy || zz) add(zx, zy, zz, zx + 3 * zy + 9 * zz);
  }
  A.box_blk[0] = 0;
  A.fastdiv = 1;
  for (int b = 0; b < A.nbox; ++b) {
    const awc::Box& B = A.box[b];
    const int64_t W = B.x1 - B.x0 + 1, ncol = W * (B.y1 - B.y0 + 1);
    const int64_t ncb = (ncol + 255) / 256, nbz = B.z1 - B.z0 + 1;
    A.box_blk[b + 1] = (int32_t)(A.box_blk[b] + ncb * nbz);
    A.box_mw[b] = ((1ull << 32) + (uint64_t)W - 1) / (uint64_t)W;
    A.box_mncb[b] = ((1ull << 32) + (uint64_t)ncb - 1) / (uint64_t)ncb;
    // quotients l / W with l < 256 ncb and r / ncb with r < ncb nbz
    if (256 * ncb * W >= (1ll << 32) || ncb * nbz * ncb >= (1ll << 32)) A.fastdiv = 0;
  }
  for (int b = A.nbox; b < 27; ++b) A.box_blk[b + 1] = A.box_blk[b];
}

// Offsets fit in int32 when every field (and so every band array) does.
template <typename T, int ND, bool GRAD>
void launch_core_i(const awc::AdjStep<T>& A, bool i64, dim3 grid, cudaStream_t st) {
  if (i64)
    awc::adj_core<T, int64_t, ND, GRAD><<<grid, dim3(32, 8), 0, st>>>(A);
  else
    awc::adj_core<T, int32_t, ND, GRAD><<<grid, dim3(32, 8), 0, st>>>(A);
}

template <typename T>
void launch_core(const awc::AdjStep<T>& A, int ndim, bool grad, bool i64, dim3 grid,
                 cudaStream_t st) {
  if (ndim == 3 && grad)
    launch_core_i<T, 3, true>(A, i64, grid, st);
  else if (ndim == 3)
    launch_core_i<T, 3, false>(A, i64, grid, st);
  else if (grad)
    launch_core_i<T, 2, true>(A, i64, grid, st);
  else
    launch_core_i<T, 2, false>(A, i64, grid, st);
}

template <typename T, int ND, bool GRAD>
void launch_shell_i(const awc::AdjStep<T>& A, bool i64, unsigned blocks, cudaStream_t st) {
  if (i64)
    awc::adj_shell<T, int64_t, ND, GRAD><<<blocks, 256, 0, st>>>(A);
  else
    awc::adj_shell<T, int32_t, ND, GRAD><<<blocks, 256, 0, st>>>(A);
}

template <typename T>
void launch_shell(const awc::AdjStep<T>& A, int ndim, bool grad, bool i64, unsigned blocks,
                  cudaStream_t st) {
  if (ndim == 3 && grad)
    launch_shell_i<T, 3, true>(A, i64, blocks, st);
  else if (ndim == 3)
    launch_shell_i<T, 3, false>(A, i64, blocks, st);
  else if (grad)
    launch_shell_i<T, 2, true>(A, i64, blocks, st);
  else
    launch_shell_i<T, 2, false>(A, i64, blocks, st);
}

// TMA-fed core kernel: tile 64 x 8 nodes, 4 stages.
constexpr int ADJ_TY = 4, ADJ_STAGES = 4;
template <typename T>
constexpr int adj_core_smem() {
  return ADJ_STAGES * awc::AdjTile<T, ADJ_TY>::BYTES + 2 * ADJ_STAGES * 8 + 16;
}

// Tensor map of a pitched field (elements of type E) for the TMA core
// kernel: the box with a ring (ring = true) or the tile.
template <typename T, typename E = T>
bool adj_map(CUtensorMap* m, const void* base, const awc::PlanView& V, bool ring) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = awc::tensor_map_encoder();
  if (!enc) return false;
  using L = awc::AdjTile<T, ADJ_TY>;
  const CUtensorMapDataType dt =
      sizeof(E) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[3] = {(cuuint64_t)V.nx, (cuuint64_t)V.ny, (cuuint64_t)V.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)(V.px * sizeof(E)),
                                 (cuuint64_t)(V.px * V.ny * sizeof(E))};
  const cuuint32_t box[3] = {ring ? (cuuint32_t)L::PW : (cuuint32_t)L::TX,
                             (cuuint32_t)L::RY + (ring ? 2 : 0), 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, dt, 3, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The adjoint's two streams and five events of the context (created once).
int adj_streams(awc_ctx* C, cudaStream_t* a, cudaStream_t* b) {
  for (cudaStream_t& s : C->adj_stream)
    if (!s) ADJ_TRY(C, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  for (cudaEvent_t& e : C->adj_ev)
    if (!e) ADJ_TRY(C, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  *a = C->adj_stream[0];
  *b = C->adj_stream[1];
  return AWC_OK;
}

template <typename T>
// Gradient mode (grad_out or grad_sum set): the checkpointed forward run
// gives the traces, the misfit against `observed` and the residuals; the
// gradient goes to the host (grad_out) or is added to a dense device sum
// (grad_sum). Transpose mode (src_out set): `residual` are the adjoint traces.
int adjoint_impl(awc_ctx* C, awc_plan* plan, const awc_problem* p, const double* coeffs,
                 const int64_t* possrcs, const double* dt2srctf, const int64_t* posrecs,
                 const double* residual, const double* observed, double* misfit,
                 double* traces_out, int64_t kchk, double* grad_out, double* src_out,
                 double* grad_sum = nullptr) {
  const awc::PlanView V = awc::plan_view(plan);
  cudaStream_t st = V.stream;
  const int64_t nt = p->nt, nsrc = p->nsrc, nrec = p->nrec, h = p->halo;
  const int64_t NP = V.NP, fb = NP * (int64_t)sizeof(T);
  const bool want_grad = grad_out != nullptr || grad_sum != nullptr;
  DevMem& mem = ctx_mem(C);
  // adjoint fields
  T *lam[2], *mu[3][2][2] = {}, *nu[3][2][2] = {};
  for (int b = 0; b < 2; ++b) ADJ_TRY(C, mem.get(&lam[b], fb));
  for (int a = 0; a < p->ndim; ++a)
    for (int s = 0; s < 2; ++s) {
      for (int b = 0; b < 2; ++b) {
        ADJ_TRY(C, mem.get(&mu[a][s][b], V.psi_len[a] * sizeof(T)));
        ADJ_TRY(C, cudaMemsetAsync(mu[a][s][b], 0, std::max<int64_t>(V.psi_len[a], 1) * sizeof(T), st));
        ADJ_TRY(C, mem.get(&nu[a][s][b], V.xi_len[a] * sizeof(T)));
        ADJ_TRY(C, cudaMemsetAsync(nu[a][s][b], 0, std::max<int64_t>(V.xi_len[a], 1) * sizeof(T), st));
      }
    }
  for (int b = 0; b < 2; ++b) ADJ_TRY(C, cudaMemsetAsync(lam[b], 0, fb, st));
  double* grad = nullptr;
  if (want_grad) {
    ADJ_TRY(C, mem.get(&grad, NP * sizeof(double)));
    ADJ_TRY(C, cudaMemsetAsync(grad, 0, NP * sizeof(double), st));
  }
  // source rows [nt][nsrc] in T (the residual rows follow the forward run)
  // residual rows [nt][nrec] (device) from column-major doubles uploaded to colm_d
  T* res_d;
  ADJ_TRY(C, mem.get(&res_d, std::max<int64_t>(nt * nrec, 1) * sizeof(T)));
  double* colm_d;
  ADJ_TRY(C, mem.get(&colm_d, std::max<int64_t>(nt * nrec, 1) * sizeof(double)));
  const dim3 rgrid((unsigned)std::max<int64_t>(1, (nrec + 31) / 32),
                   (unsigned)std::max<int64_t>(1, (nt + 31) / 32));
  double* part_d;
  ADJ_TRY(C, mem.get(&part_d, (size_t)rgrid.x * rgrid.y * sizeof(double)));
  std::vector<T> srows(std::max<int64_t>(nt * nsrc, 1), T(0));
  if (dt2srctf)
    for (int64_t s = 0; s < nsrc; ++s)
      for (int64_t t = 0; t < nt; ++t) srows[t * nsrc + s] = (T)dt2srctf[t + nt * s];
  T* stf_d;
  ADJ_TRY(C, mem.get(&stf_d, srows.size() * sizeof(T)));
  ADJ_TRY(C, cudaMemcpyAsync(stf_d, srows.data(), srows.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  T* sout_d = nullptr;
  if (src_out) ADJ_TRY(C, mem.get(&sout_d, std::max<int64_t>(nt * nsrc, 1) * sizeof(T)));
  // receiver groups and source nodes (interior only)
  const Groups RG = group_nodes(p, V.px, posrecs, nrec, nullptr);
  std::vector<int64_t> snode;
  group_nodes(p, V.px, possrcs, nsrc, &snode);
  int64_t* rnode_d;
  int32_t *roff_d, *rids_d;
  int64_t* snode_d;
  ADJ_TRY(C, mem.get(&rnode_d, RG.node.size() * 8));
  ADJ_TRY(C, mem.get(&roff_d, RG.off.size() * 4));
  ADJ_TRY(C, mem.get(&rids_d, RG.ids.size() * 4));
  ADJ_TRY(C, mem.get(&snode_d, snode.size() * 8));
  if (!RG.node.empty()) {
    ADJ_TRY(C, cudaMemcpyAsync(rnode_d, RG.node.data(), RG.node.size() * 8, cudaMemcpyHostToDevice, st));
    ADJ_TRY(C, cudaMemcpyAsync(rids_d, RG.ids.data(), RG.ids.size() * 4, cudaMemcpyHostToDevice, st));
  }
  ADJ_TRY(C, cudaMemcpyAsync(roff_d, RG.off.data(), RG.off.size() * 4, cudaMemcpyHostToDevice, st));
  if (!snode.empty())
    ADJ_TRY(C, cudaMemcpyAsync(snode_d, snode.data(), snode.size() * 8, cudaMemcpyHostToDevice, st));
  // which sources sit in an active CPML band (their bracket uses S_t)
  std::vector<int8_t> sband(std::max<int64_t>(nsrc, 1), 0);
  {
    const int64_t nn[3] = {p->nx, p->ny, V.nz};
    for (int64_t s2 = 0; s2 < nsrc; ++s2) {
      const int64_t c[3] = {possrcs[s2] - 1, possrcs[s2 + nsrc] - 1,
                            p->ndim == 3 ? possrcs[s2 + 2 * nsrc] - 1 : 0};
      for (int a = 0; a < p->ndim && h > 0; ++a)
        if ((V.active[a][0] && c[a] <= h) || (V.active[a][1] && c[a] >= nn[a] - h - 1))
          sband[s2] = 1;
    }
  }
  int8_t* sband_d;
  ADJ_TRY(C, mem.get(&sband_d, sband.size()));
  ADJ_TRY(C, cudaMemcpyAsync(sband_d, sband.data(), sband.size(), cudaMemcpyHostToDevice, st));
  // kernel parameters
  awc::AdjStep<T> A{};
  A.nx = (int32_t)p->nx;
  A.ny = (int32_t)p->ny;
  A.nz = (int32_t)V.nz;
  A.halo = (int32_t)h;
  A.px = V.px;
  A.plane = V.px * p->ny;
  const double d[3] = {p->dx, p->dy, p->ndim == 3 ? p->dz : 1.0};
  for (int a = 0; a < 3; ++a) {
    A.inv_d[a] = (T)(1.0 / d[a]);
    A.inv_d2[a] = (T)(1.0 / (d[a] * d[a]));
  }
  A.F = (const T*)V.fact;
  const int64_t n3[3] = {p->nx, p->ny, V.nz};
  // coefficient pairs per axis and side: h {bK, a} then h + 1 {bKh, ah}, from
  // the problem's coefficient vector (a_l a_r bK_l bK_r ah_l ah_r bKh_l bKh_r)
  using V2 = typename awc::Vec2<T>::type;
  const int64_t npair = 2 * h + 1;
  std::vector<V2> pairs(std::max<int64_t>(p->ndim * 2 * npair, 1));
  for (int a = 0; a < p->ndim; ++a) {
    const double* blk = coeffs + a * (8 * h + 4);
    for (int s = 0; s < 2; ++s) {
      V2* pr = pairs.data() + (a * 2 + s) * npair;
      for (int64_t e = 0; e < h; ++e)
        pr[e] = V2{(T)blk[2 * h + s * h + e], (T)blk[s * h + e]};
      for (int64_t f = 0; f <= h; ++f)
        pr[h + f] = V2{(T)blk[4 * h + 2 * (h + 1) + s * (h + 1) + f], (T)blk[4 * h + s * (h + 1) + f]};
    }
  }
  V2* pairs_d;
  ADJ_TRY(C, mem.get(&pairs_d, pairs.size() * sizeof(V2)));
  ADJ_TRY(C, cudaMemcpyAsync(pairs_d, pairs.data(), pairs.size() * sizeof(V2),
                             cudaMemcpyHostToDevice, st));
  for (int a = 0; a < p->ndim; ++a) {
    for (int s = 0; s < 2; ++s) {
      A.nuc[a][s] = pairs_d + (a * 2 + s) * npair;
      A.muc[a][s] = pairs_d + (a * 2 + s) * npair + h;
      A.active[a][s] = h > 0 ? V.active[a][s] : 0;
      A.off[a][s] = s == 0 ? 0 : (int32_t)(n3[a] - h - 2);
    }
  }
  adj_regions(A, p->ndim);
  const bool has_core = A.core.x0 <= A.core.x1;
  const dim3 core_grid((unsigned)((A.core.x1 - A.core.x0 + 32) / 32),
                       (unsigned)((A.core.y1 - A.core.y0 + 8) / 8),
                       (unsigned)(A.core.z1 - A.core.z0 + 1));
  const unsigned shell_blocks = (unsigned)A.box_blk[A.nbox];
  const bool i64 = NP > (int64_t)INT32_MAX;
  // 3D gradient runs stream the core box through the TMA-fed kernel, in z
  // chunks sized for about four waves of resident blocks
  using Tile = awc::AdjTile<T, ADJ_TY>;
  A.err = V.err_flag;
  A.core_x = (int32_t)(A.core.x0 / Tile::A * Tile::A);
  bool use_tma = p->ndim == 3 && want_grad && has_core && awc::tensor_map_encoder() != nullptr;
  dim3 tma_grid;
  if (use_tma) {
    const int64_t gx = (A.core.x1 + 1 - A.core_x + Tile::TX - 1) / Tile::TX;
    const int64_t gy = (A.core.y1 - A.core.y0 + Tile::RY) / Tile::RY;
    const int64_t nzc = A.core.z1 - A.core.z0 + 1;
    int per_sm = 0;
    ADJ_TRY(C, cudaFuncSetAttribute(awc::adj_core_tma<T, ADJ_TY, ADJ_STAGES>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    adj_core_smem<T>()));
    ADJ_TRY(C, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                   &per_sm, awc::adj_core_tma<T, ADJ_TY, ADJ_STAGES>, 32 * ADJ_TY,
                   adj_core_smem<T>()));
    const int64_t target = 4 * (int64_t)C->num_sms * std::max(per_sm, 1);
    const int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(nzc, target / (gx * gy)));
    A.zchunk = (int32_t)std::max<int64_t>(4, (nzc + chunks - 1) / chunks);
    tma_grid = dim3((unsigned)gx, (unsigned)gy, (unsigned)((nzc + A.zchunk - 1) / A.zchunk));
  }
  // checkpoints and segment fields (gradient only)
  const int64_t nseg = want_grad ? (nt + kchk - 1) / kchk : 0;
  int64_t band_elems = 0;
  for (int a = 0; a < p->ndim; ++a) band_elems += 2 * (V.psi_len[a] + V.xi_len[a]);
  std::vector<T*> chk(nseg, nullptr);
  // segment fields: two sets, so that segment c - 1 is recomputed into one
  // while the backward steps of segment c read the other
  const int nset = nseg > 1 ? 2 : 1;
  std::vector<T*> seg[2];
  if (want_grad) {
    // one allocation for the saved states and the segments' fields
    const int64_t chk_elems = (3 * NP + band_elems + 63) / 64 * 64;
    const int64_t nfield = std::min<int64_t>(kchk, nt) + 2;
    T* arena;
    ADJ_TRY(C, mem.get(&arena, (nseg * chk_elems + nset * nfield * NP) * sizeof(T)));
    for (int64_t c = 0; c < nseg; ++c) chk[c] = arena + c * chk_elems;
    for (int b = 0; b < nset; ++b) {
      seg[b].resize(nfield);
      for (int64_t m = 0; m < nfield; ++m)
        seg[b][m] = arena + nseg * chk_elems + (b * nfield + m) * NP;
    }
    // the steps write the segment fields in place, interior nodes only: the
    // rims stay zero
    ADJ_TRY(C, cudaMemsetAsync(seg[0][0], 0, nset * nfield * NP * sizeof(T), st));
  }
  // tensor maps of the TMA-fed core kernel: both λ buffers, F, every segment field
  CUtensorMap map_lam[2], map_lam3[2], map_f, map_grad;
  std::vector<CUtensorMap> map_seg[2];
  if (use_tma) {
    use_tma = adj_map<T>(&map_lam[0], lam[0], V, true) && adj_map<T>(&map_lam[1], lam[1], V, true) &&
              adj_map<T>(&map_lam3[0], lam[0], V, false) &&
              adj_map<T>(&map_lam3[1], lam[1], V, false) && adj_map<T>(&map_f, V.fact, V, true) &&
              adj_map<T, double>(&map_grad, grad, V, false);
    for (int b = 0; b < nset; ++b) {
      map_seg[b].resize(seg[b].size());
      for (size_t m = 0; use_tma && m < seg[b].size(); ++m)
        use_tma = adj_map<T>(&map_seg[b][m], seg[b][m], V, true);
    }
  }
  auto save_or_restore = [&](T* base, int64_t s, bool save) -> int {
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st);
    };
    T* q = base;
    for (int b = 0; b < 3; ++b, q += NP)
      ADJ_TRY(C, save ? cp(q, V.buf[b], fb) : cp(V.buf[b], q, fb));
    for (int a = 0; a < p->ndim; ++a)
      for (int sd = 0; sd < 2; ++sd) {
        void* ps = V.psi[a][sd][s & 1];
        ADJ_TRY(C, save ? cp(q, ps, V.psi_len[a] * sizeof(T)) : cp(ps, q, V.psi_len[a] * sizeof(T)));
        q += V.psi_len[a];
        ADJ_TRY(C, save ? cp(q, V.xi[a][sd], V.xi_len[a] * sizeof(T))
                        : cp(V.xi[a][sd], q, V.xi_len[a] * sizeof(T)));
        q += V.xi_len[a];
      }
    return AWC_OK;
  };
  int rc;
  if (want_grad) {
    // forward run with checkpoints, then the traces, misfit and residuals
    if ((rc = awc_plan_reset(plan))) return rc;
    for (int64_t c = 0; c < nseg; ++c) {
      const int64_t s = c * kchk, e = std::min(s + kchk, nt);
      if ((rc = save_or_restore(chk[c], s, true))) return rc;
      if (c == nseg - 1) {
        // the last segment's fields are kept as they are computed, so the
        // backward pass starts without a recompute
        std::vector<T*>& f = seg[c % nset];
        ADJ_TRY(C, cudaMemcpyAsync(f[0], V.buf[s % 3], fb, cudaMemcpyDeviceToDevice, st));
        ADJ_TRY(C, cudaMemcpyAsync(f[1], V.buf[(s + 1) % 3], fb, cudaMemcpyDeviceToDevice, st));
        awc::plan_keep_fields(plan, (void* const*)(f.data() + 2), s, e - s, true);
      }
      rc = awc_plan_run(plan, e - s, 1, nullptr);
      awc::plan_keep_fields(plan, nullptr, 0, 0);
      if (rc) return rc;
    }
    if (traces_out && nt * nrec > 0 && (rc = awc_plan_traces(plan, traces_out))) return rc;
  }
  if (want_grad) *misfit = 0.0;
  if (nt * nrec > 0) {
    // residuals (and the misfit's block sums) on the device
    ADJ_TRY(C, awc::copy_to_device(C, colm_d, want_grad ? observed : residual,
                                   nt * nrec * sizeof(double), st));
    awc::adj_residual_rows<T><<<rgrid, dim3(32, 8), 0, st>>>(
        want_grad ? (const T*)V.traces : nullptr, colm_d, nt, nrec, res_d,
        want_grad ? part_d : nullptr);
    ADJ_TRY(C, cudaGetLastError());
    if (want_grad) {
      std::vector<double> part((size_t)rgrid.x * rgrid.y);
      ADJ_TRY(C, cudaMemcpyAsync(part.data(), part_d, part.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
      ADJ_TRY(C, cudaStreamSynchronize(st));
      double J = 0.0;
      for (double v : part) J += v;  // fixed order
      *misfit = J;
    }
  }
  // backward: the steps run on the adjoint's two streams (core kernel on the
  // first, shell kernel on the second); segment c - 1 is recomputed on the
  // plan's stream into the other field set meanwhile
  cudaStream_t bs = nullptr, bs2 = nullptr;
  if ((rc = adj_streams(C, &bs, &bs2))) return rc;
  cudaEvent_t ev_fork = C->adj_ev[0], ev_join = C->adj_ev[1], ev_rec = C->adj_ev[2];
  cudaEvent_t* ev_free = C->adj_ev + 3;  // set b's backward steps are done
  ADJ_TRY(C, cudaEventRecord(ev_rec, st));  // the set-up above
  ADJ_TRY(C, cudaStreamWaitEvent(bs, ev_rec, 0));
  auto recompute = [&](int64_t c) -> int {
    // p_{s-1} .. p_e of segment c into field set c % 2
    const int64_t s = c * kchk, e = std::min(s + kchk, nt);
    const int b = (int)(c % nset);
    if (c + nset <= nseg - 1) ADJ_TRY(C, cudaStreamWaitEvent(st, ev_free[b], 0));
    int r;
    if ((r = save_or_restore(chk[c], s, false))) return r;
    awc::plan_set_step(plan, s);
    ADJ_TRY(C, cudaMemcpyAsync(seg[b][0], V.buf[s % 3], fb, cudaMemcpyDeviceToDevice, st));
    ADJ_TRY(C, cudaMemcpyAsync(seg[b][1], V.buf[(s + 1) % 3], fb, cudaMemcpyDeviceToDevice, st));
    awc::plan_keep_fields(plan, (void* const*)(seg[b].data() + 2), s, e - s, true);
    r = awc_plan_run(plan, e - s, 1, nullptr);
    awc::plan_keep_fields(plan, nullptr, 0, 0);
    if (r) return r;
    ADJ_TRY(C, cudaEventRecord(ev_rec, st));
    return AWC_OK;
  };
  int i2 = 0, i3 = 1;  // lam[i2] = λ_{t+2}, lam[i3] = λ_{t+3}
  int par = 0;         // nu[..][par] holds ν_{t+2}
  for (int64_t c = (want_grad ? nseg : 1) - 1; c >= 0; --c) {
    const int64_t s = want_grad ? c * kchk : 0, e = want_grad ? std::min(s + kchk, nt) : nt;
    const int b = want_grad ? (int)(c % nset) : 0;
    if (want_grad) ADJ_TRY(C, cudaStreamWaitEvent(bs, ev_rec, 0));
    for (int64_t t = e - 1; t >= s; --t) {
      // λ_{t+1} overwrites λ_{t+3}, which the step kernels read only at the
      // node they write
      A.lam2 = lam[i2];
      A.lam = lam[i3];
      for (int a = 0; a < p->ndim; ++a)
        for (int sd = 0; sd < 2; ++sd) {
          A.nu_in[a][sd] = nu[a][sd][par];
          A.nu_out[a][sd] = nu[a][sd][par ^ 1];
          A.mu_in[a][sd] = mu[a][sd][par];
          A.mu_out[a][sd] = mu[a][sd][par ^ 1];
        }
      if (!RG.node.empty())
        awc::adj_residuals<T><<<(unsigned)((RG.node.size() + 127) / 128), 128, 0, bs>>>(
            A.lam, rnode_d, roff_d, rids_d, (int32_t)RG.node.size(), res_d + t * nrec);
      A.pm1 = want_grad ? seg[b][t - s] : nullptr;
      A.p0 = want_grad ? seg[b][t - s + 1] : nullptr;
      A.pp1 = want_grad ? seg[b][t - s + 2] : nullptr;
      A.grad = grad;
      const bool fork = has_core && shell_blocks > 0;
      if (fork) {
        ADJ_TRY(C, cudaEventRecord(ev_fork, bs));
        ADJ_TRY(C, cudaStreamWaitEvent(bs2, ev_fork, 0));
      }
      if (shell_blocks > 0)
        launch_shell(A, p->ndim, want_grad, i64, shell_blocks, fork ? bs2 : bs);
      if (has_core && use_tma) {
        awc::adj_core_tma<T, ADJ_TY, ADJ_STAGES>
            <<<tma_grid, dim3(32, ADJ_TY), adj_core_smem<T>(), bs>>>(
                map_lam[i2], map_f, map_seg[b][t - s + 1], map_lam3[i3], map_grad, A);
      } else if (has_core) {
        launch_core(A, p->ndim, want_grad, i64, core_grid, bs);
      }
      if (fork) {
        ADJ_TRY(C, cudaEventRecord(ev_join, bs2));
        ADJ_TRY(C, cudaStreamWaitEvent(bs, ev_join, 0));
      }
      if (nsrc > 0)
        awc::adj_sources<T><<<1, 32, 0, bs>>>(A.lam, A.F, snode_d, sband_d, (int32_t)nsrc,
                                              stf_d + t * nsrc, grad,
                                              sout_d ? sout_d + t * nsrc : nullptr);
      ADJ_TRY(C, cudaGetLastError());
      std::swap(i2, i3);  // λ_{t+1} is the next step's λ_{t+2}
      par ^= 1;
    }
    ADJ_TRY(C, cudaEventRecord(ev_free[b], bs));
    if (want_grad && c > 0 && (rc = recompute(c - 1))) return rc;
  }
  // the outputs follow the backward steps
  ADJ_TRY(C, cudaEventRecord(ev_join, bs));
  ADJ_TRY(C, cudaStreamWaitEvent(st, ev_join, 0));
  // outputs
  if (want_grad) {
    const int64_t N = p->nx * p->ny * V.nz;
    const int blocks = (int)std::min<int64_t>((N + 255) / 256, (int64_t)C->num_sms * 16);
    if (grad_sum) {
      awc::scale_unpitch_add<<<blocks, 256, 0, st>>>(grad, grad_sum, N, p->nx, V.px,
                                                     p->dt * p->dt);
      ADJ_TRY(C, cudaGetLastError());
    } else {
      double* dense;
      ADJ_TRY(C, mem.get(&dense, N * sizeof(double)));
      awc::scale_unpitch<<<blocks, 256, 0, st>>>(grad, dense, N, p->nx, V.px, p->dt * p->dt);
      ADJ_TRY(C, cudaGetLastError());
      ADJ_TRY(C, awc::copy_to_host(C, grad_out, dense, N * sizeof(double), st));
    }
  }
  if (src_out && nsrc > 0) {
    double* sd;
    ADJ_TRY(C, mem.get(&sd, nt * nsrc * sizeof(double)));
    awc::to_double<T><<<(unsigned)std::min<int64_t>((nt * nsrc + 255) / 256, 4096), 256, 0, st>>>(
        sout_d, sd, nt * nsrc);
    ADJ_TRY(C, cudaGetLastError());
    std::vector<double> tmp(nt * nsrc);
    ADJ_TRY(C, cudaMemcpyAsync(tmp.data(), sd, tmp.size() * 8, cudaMemcpyDeviceToHost, st));
    ADJ_TRY(C, cudaStreamSynchronize(st));
    for (int64_t s2 = 0; s2 < nsrc; ++s2)
      for (int64_t t = 0; t < nt; ++t) src_out[t + nt * s2] = tmp[t * nsrc + s2];
  }
  int32_t flag = 0;
  ADJ_TRY(C, cudaMemcpyAsync(&flag, V.err_flag, 4, cudaMemcpyDeviceToHost, st));
  ADJ_TRY(C, cudaStreamSynchronize(st));
  if (flag) {
    ADJ_TRY(C, cudaMemsetAsync(V.err_flag, 0, 4, st));
    return awc::fail(C, AWC_ERR_TIMEOUT, "a bounded wait on a pipeline barrier ran out");
  }
  return AWC_OK;
}

int check_adjoint_problem(awc_ctx* C, const awc_problem* p) {
  if (!p) return awc::fail(C, AWC_ERR_INVALID, "problem is NULL");
  if (p->ndim != 2 && p->ndim != 3)
    return awc::fail(C, AWC_ERR_INVALID, "the adjoint solves 2D and 3D problems");
  const int64_t n[3] = {p->nx, p->ny, p->ndim == 3 ? p->nz : 1};
  for (int a = 0; a < p->ndim; ++a)
    if (p->halo > 0 && n[a] < 2 * (int64_t)p->halo + 2)
      return awc::fail(C, AWC_ERR_INVALID,
                       "the adjoint needs non-overlapping CPML bands (n >= 2 halo + 2 per axis)");
  return AWC_OK;
}

}  // namespace

extern "C" {

int awc_misfit_gradient(awc_ctx* ctx, const awc_problem* p, const double* vel,
                        const double* coeffs, const int64_t* possrcs, const double* dt2srctf,
                        const int64_t* posrecs, const double* observed, int32_t checkpoint_every,
                        double* misfit, double* grad_c2, double* traces) {
  if (!ctx) return awc::fail(nullptr, AWC_ERR_INVALID, "ctx is NULL");
  int rc;
  if ((rc = check_adjoint_problem(ctx, p))) return rc;
  if (!observed || !grad_c2 || !misfit)
    return awc::fail(ctx, AWC_ERR_INVALID, "observed/grad_c2/misfit is NULL");
  if (checkpoint_every < 1) return awc::fail(ctx, AWC_ERR_INVALID, "checkpoint_every must be >= 1");
  if ((rc = awc::plan_for(ctx, &ctx->adj_plan, p, vel, coeffs, possrcs, dt2srctf, posrecs,
                          true)))
    return rc;
  awc_plan* plan = ctx->adj_plan;
  rc = p->precision == AWC_F64
           ? adjoint_impl<double>(ctx, plan, p, coeffs, possrcs, dt2srctf, posrecs, nullptr,
                                  observed, misfit, traces, checkpoint_every, grad_c2, nullptr)
           : adjoint_impl<float>(ctx, plan, p, coeffs, possrcs, dt2srctf, posrecs, nullptr,
                                 observed, misfit, traces, checkpoint_every, grad_c2, nullptr);
  return rc;
}

int awc_misfit_gradient_shots(awc_ctx* ctx, const awc_problem* p, int32_t nshot,
                              const double* vel, const double* coeffs, const int64_t* possrcs,
                              const double* dt2srctf, const int64_t* posrecs,
                              const double* observed, int32_t checkpoint_every, double* misfit,
                              double* grad_c2) {
  if (!ctx) return awc::fail(nullptr, AWC_ERR_INVALID, "ctx is NULL");
  int rc;
  if ((rc = check_adjoint_problem(ctx, p))) return rc;
  if (nshot < 1) return awc::fail(ctx, AWC_ERR_INVALID, "nshot must be >= 1");
  if (!observed || !grad_c2 || !misfit)
    return awc::fail(ctx, AWC_ERR_INVALID, "observed/grad_c2/misfit is NULL");
  if (p->nsrc > 0 && (!possrcs || (p->nt > 0 && !dt2srctf)))
    return awc::fail(ctx, AWC_ERR_INVALID, "possrcs/dt2srctf is NULL");
  if (checkpoint_every < 1) return awc::fail(ctx, AWC_ERR_INVALID, "checkpoint_every must be >= 1");
  // per-shot strides of the stacked inputs
  const int64_t s_pos = p->nsrc * p->ndim, s_stf = p->nt * p->nsrc, s_obs = p->nt * p->nrec;
  auto pos_of = [&](int32_t s) { return p->nsrc > 0 ? possrcs + s * s_pos : possrcs; };
  auto stf_of = [&](int32_t s) { return dt2srctf ? dt2srctf + s * s_stf : dt2srctf; };
  // the first shot uploads the model; the others replace only the sources
  if ((rc = awc::plan_for(ctx, &ctx->adj_plan, p, vel, coeffs, pos_of(0), stf_of(0), posrecs,
                          true)))
    return rc;
  awc_plan* plan = ctx->adj_plan;
  const cudaStream_t st = awc::plan_view(plan).stream;
  const int64_t N = p->nx * p->ny * (p->ndim == 3 ? p->nz : 1);
  double* sum;
  ADJ_TRY(ctx, ctx_mem(ctx).get_sum(&sum, N * sizeof(double)));
  ADJ_TRY(ctx, cudaMemsetAsync(sum, 0, N * sizeof(double), st));
  double J = 0.0;
  for (int32_t s = 0; s < nshot; ++s) {
    if (s > 0 && (rc = awc::plan_shot(ctx, plan, pos_of(s), stf_of(s), posrecs))) return rc;
    double Js = 0.0;
    rc = p->precision == AWC_F64
             ? adjoint_impl<double>(ctx, plan, p, coeffs, pos_of(s), stf_of(s), posrecs, nullptr,
                                    observed + s * s_obs, &Js, nullptr, checkpoint_every,
                                    nullptr, nullptr, sum)
             : adjoint_impl<float>(ctx, plan, p, coeffs, pos_of(s), stf_of(s), posrecs, nullptr,
                                   observed + s * s_obs, &Js, nullptr, checkpoint_every,
                                   nullptr, nullptr, sum);
    if (rc) return rc;
    J += Js;  // shot order
  }
  ADJ_TRY(ctx, awc::copy_to_host(ctx, grad_c2, sum, N * sizeof(double), st));
  *misfit = J;
  return AWC_OK;
}

int awc_adjoint_sources(awc_ctx* ctx, const awc_problem* p, const double* vel,
                        const double* coeffs, const int64_t* possrcs, const int64_t* posrecs,
                        const double* adjoint_traces, double* src_out) {
  if (!ctx) return awc::fail(nullptr, AWC_ERR_INVALID, "ctx is NULL");
  int rc;
  if ((rc = check_adjoint_problem(ctx, p))) return rc;
  if (!adjoint_traces || !src_out)
    return awc::fail(ctx, AWC_ERR_INVALID, "adjoint_traces/src_out is NULL");
  // the plan only provides fact and the coefficients; the injected values
  // play no part in the transpose
  std::vector<double> zero(std::max<int64_t>(p->nt * p->nsrc, 1), 0.0);
  if ((rc = awc::plan_for(ctx, &ctx->adj_plan, p, vel, coeffs, possrcs, zero.data(), posrecs)))
    return rc;
  awc_plan* plan = ctx->adj_plan;
  rc = p->precision == AWC_F64
           ? adjoint_impl<double>(ctx, plan, p, coeffs, possrcs, nullptr, posrecs,
                                  adjoint_traces, nullptr, nullptr, nullptr, 1, nullptr, src_out)
           : adjoint_impl<float>(ctx, plan, p, coeffs, possrcs, nullptr, posrecs,
                                 adjoint_traces, nullptr, nullptr, nullptr, 1, nullptr, src_out);
  return rc;
}

}  // extern "C"
