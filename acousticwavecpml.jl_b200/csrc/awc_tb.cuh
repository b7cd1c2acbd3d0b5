// awc_tb.cuh — the 3D CPML step advanced two time steps per pass (temporal
// blocking).
//
// A pass computes, for every interior node, the pressure of steps s+1 and
// s+2 from those of steps s-1 and s, and the CPML state (ψ, ξ) of step s+2
// from that of step s: two applications of the reference's forward!
// (src/shared/acoustic_3D_xPU.jl:124-167) with the same arithmetic, operation
// for operation, as the one-step kernels of awc_kernels.cuh (so a run gives
// bitwise the results of one-step launches). Per node and pass the fields
// cost 5 words of HBM traffic (read pold, pcur, fact; write the two new
// fields) instead of 8 for two one-step launches, and each live CPML entry is
// read and written once instead of twice.
//
// Geometry. A block of 32 x W threads owns a column tile of 62 x (W-2)
// interior nodes (the level-2 tile) and streams a chunk of z planes. Lane l
// of warp w owns the x pair of columns X0 - 1 + 2l, X0 + 2l at row
// Y0 - 1 + w of the 64 x W level-1 region, which is the tile plus a ring of
// one node: the ring's step-s+1 values are the neighbours of the tile's
// step-s+2 update, so every thread computes step s+1 on its pair (from the
// staged p_s, p_{s-1} and fact) and then step s+2 on the nodes of its pair
// that lie in the tile. The step-s+1 values of one plane are exchanged
// through a two-slot shared-memory ring; each thread keeps its own columns'
// z neighbours (p_s and p_{s+1} of three planes) in registers.
//
// Staging. One elected thread streams, per z plane, three TMA boxes into a
// ring of S stages: p_s on the region plus one node (72 x (W+2), x origin
// rounded down to 16 bytes), p_{s-1} and fact on the region (72 x W). One
// block-wide barrier per plane orders the slot ring and frees the stage of
// the plane just finished for the next load.
//
// CPML state. The level-1 update of a band node reads ψ_s on both of its
// faces and ξ_s from the "in" arrays; its new values stay in the thread's
// registers for the level-2 update of the same node one iteration later,
// which writes ψ_{s+2} and ξ_{s+2} to the "out" arrays. Ring nodes read the
// "in" arrays of nodes other blocks own, so ψ and ξ both alternate between
// two arrays across passes, and the four pressure fields of a pass
// (p_{s-1}, p_s in; p_{s+1}, p_{s+2} out) are four distinct buffers.
//
// Scope. Sources and receivers must be interior nodes (no Dirichlet-rim
// I/O): the rim of every field is then zero for ever and no pass writes it.
#pragma once
#include <type_traits>

#include "awc_kernels.cuh"

namespace awc {

// ψ/ξ arrays and coefficients of one axis for a two-step pass. Pointers are
// the left side's; the right side's ψ/ξ follow at psi_side/xi_side elements
// and its coefficients at halo (on-grid) or halo + 1 (half-grid) elements.
template <typename T>
struct TbAxis {
  const T* psi_in;
  T* psi_out;
  const T* xi_in;
  T* xi_out;
  const T* a;    // on-grid a
  const T* bK;   // on-grid b/K
  const T* ah;   // half-grid a
  const T* bKh;  // half-grid b/K
  int64_t psi_side, xi_side;
};

template <typename T>
struct TbParams {
  const T* pold;  // p_{s-1}
  const T* pcur;  // p_s
  T* p1;          // p_{s+1} (written)
  T* p2;          // p_{s+2} (written)
  const T* fact;
  int32_t nx, ny, nz, halo;
  int64_t px, plane;
  T inv_d[3], inv_d2[3];
  TbAxis<T> ax[3];
  int32_t active[3][2];
  int32_t first_r[3];
  int32_t damp_all;  // add the damping term at every node (grids with no band-free core)
  int32_t it;        // 0-based index of step s+1 (row of stf/traces)
  int32_t* err;
  // sources/receivers of this launch: per block [blk_off[b], blk_off[b+1])
  // entries {2 x thread + node of its pair, plane, source group, receiver
  // group or -1}, sorted by (plane, thread); a node appears in the list of
  // every block whose level-1 region and plane range hold it, with its
  // receiver group only in its owner's
  Io<T> io;
  const int2* tiles;  // level-2 tile origins (x0, y0) of this launch
  int32_t nch, zc;    // z chunks per tile, planes per chunk
  int32_t wait_rounds, wait_ns;  // bounded waits: rounds x suspend hint (ns)
  int32_t withhold;              // test only: load index the producer skips (-1: none)
};

template <typename T, int W>
struct TbTile {
  static constexpr int NT = 32 * W;
  static constexpr int RX = 64;  // level-1 region width (x pairs of 32 lanes)
  static constexpr int TX = RX - 2;
  static constexpr int BX = 72;  // box width: 66 columns + x alignment slack
  static constexpr int A = 16 / (int)sizeof(T);
  static constexpr int PT_BYTES = BX * (W + 2) * (int)sizeof(T);
  static constexpr int IN_BYTES = BX * W * (int)sizeof(T);
  static constexpr int PT_PAD = (PT_BYTES + 127) / 128 * 128;
  static constexpr int IN_PAD = (IN_BYTES + 127) / 128 * 128;
  static constexpr int STAGE = PT_PAD + 2 * IN_PAD;
  static constexpr int SLOT = RX * W;  // elements of one slot of step-s+1 values
};

template <typename T, int W, int S>
constexpr int tb_smem() {
  return S * TbTile<T, W>::STAGE + 2 * TbTile<T, W>::SLOT * (int)sizeof(T) + 8 * S + 16;
}

// Bounded wait on a phase: at most `rounds` try_waits with a suspend hint of
// `ns` nanoseconds each. False when it gives up.
__device__ __forceinline__ bool tb_wait(uint64_t* bar, uint32_t parity, int rounds, int ns) {
  for (int n = 0; n < rounds; ++n)
    if (mbar_try_wait(bar, parity, (uint32_t)ns)) return true;
  return false;
}

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Level-1 results of one band axis at one node: new ψ on the node's upper
// (q) and lower (q-1) faces and new ξ.
template <typename T>
struct Lv1 {
  T sq, sm, xn;
};

// Band position of a node along x or y: side (0 none), entry q and the
// offsets of ψ[q] and ξ[q-1] at the current plane.
template <typename I>
struct TbBand {
  int s = 0, q = 0;
  I pq = 0, xq = 0;
};

template <typename T>
__device__ __forceinline__ BandCoef<T> tb_coef(const TbAxis<T>& X, int h, int g) {
  return BandCoef<T>{__ldg(X.bKh + h), __ldg(X.ah + h), __ldg(X.bKh + h - 1), __ldg(X.ah + h - 1),
                     __ldg(X.bK + g), __ldg(X.a + g)};
}

template <typename T, typename I, int W, int S, bool XY>
__global__ void __launch_bounds__(32 * W, W <= 8 ? 2 : 1)
    step3d_tb(const __grid_constant__ CUtensorMap mpt, const __grid_constant__ CUtensorMap mpo,
              const __grid_constant__ CUtensorMap mf, TbParams<T> P) {
  using L = TbTile<T, W>;
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem[];
  T* slot = reinterpret_cast<T*>(smem + S * L::STAGE);  // [2][SLOT] step-s+1 values
  uint64_t* full = reinterpret_cast<uint64_t*>(slot + 2 * L::SLOT);
  // abort flags: [0], [1] by iteration parity (a flag is only written before
  // the barrier of its iteration and read after it), [2] for the prologue
  volatile int* abort = reinterpret_cast<volatile int*>(full + S);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int blk = blockIdx.x;
  const int2 org = P.tiles[blk / P.nch];
  const int k0 = 1 + (blk % P.nch) * P.zc;
  const int k1 = min(k0 + P.zc, P.nz - 1);
  if (k0 >= k1) return;  // block-uniform
  const int xr = org.x - 1, yr = org.y - 1;       // region origin (xr even)
  const int xa = floor_div(xr - 1, L::A) * L::A;  // 16-byte-aligned box origin
  const int ox = xr - xa;                         // even, 2..A
  const int nplanes = k1 - k0 + 4;                // p_s planes k0-2 .. k1+1

  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
    abort[0] = 0;
    abort[1] = 0;
    abort[2] = 0;
    fence_mbar_init();
  }
  __syncthreads();
  // load u: plane k0-2+u into stage u % S; p_{s-1} and fact only for the
  // planes that get a level-1 update (k0-1 .. k1)
  int next_u = 0;
  auto issue = [&](int u) {
    const int s = u % S, m = k0 - 2 + u;
    if (u == P.withhold) return;
    unsigned char* st = smem + s * L::STAGE;
    const bool lv1 = m >= k0 - 1 && m <= k1;
    mbar_expect_tx(&full[s], L::PT_BYTES + (lv1 ? 2 * L::IN_BYTES : 0));
    tma_load_3d(st, &mpt, &full[s], xa, yr - 1, m);
    if (lv1) {
      tma_load_3d(st + L::PT_PAD, &mpo, &full[s], xa, yr, m);
      tma_load_3d(st + L::PT_PAD + L::IN_PAD, &mf, &full[s], xa, yr, m);
    }
  };
  if (tid == 0)
    for (; next_u < S && next_u < nplanes; ++next_u) issue(next_u);

  const int x0 = xr + 2 * lane, y = yr + w;
  const bool rowv = y >= 1 && y <= P.ny - 2;
  bool colv[2], own[2];
  colv[0] = rowv && x0 >= 1 && x0 <= P.nx - 2;
  colv[1] = rowv && x0 + 1 >= 1 && x0 + 1 <= P.nx - 2;
  const bool inner_y = w >= 1 && w <= W - 2;
  own[0] = colv[0] && inner_y && lane >= 1;
  own[1] = colv[1] && inner_y && lane <= 30;
  const bool lv2 = own[0] || own[1];
  const bool anyv = colv[0] || colv[1];
  const int ip = (w + 1) * L::BX + 2 * lane + ox;  // node 0 in the p_s box (even)
  const int ii = w * L::BX + 2 * lane + ox;        // in the p_{s-1} / fact boxes
  const int si = w * L::RX + 2 * lane;             // in a slot
  const int halo = P.halo;
  const I px = (I)P.px, plane = (I)P.plane;
  const I col = (I)x0 + px * (I)y;  // node 0's column offset
  int e1 = P.io.blk_off[blk];
  const int e_end = P.io.blk_off[blk + 1];
  int e2 = e1;
  const TbAxis<T>&AX = P.ax[0], &AY = P.ax[1], &AZ = P.ax[2];

  // band state of the pair's columns along x (per node) and y (shared by
  // the pair: same row) — XY launches only
  TbBand<I> bx[2], by;
  // q of the first right-band node of x and y (its lower face is written too)
  const int qfx = P.first_r[0] - (P.nx - halo - 2), qfy = P.first_r[1] - (P.ny - halo - 2);
  if (XY) {
#pragma unroll
    for (int n = 0; n < 2; ++n) {
      if (!colv[n]) continue;
      int q;
      bool f;
      int s = band_of(x0 + n, P.nx, halo, P.first_r[0], q, f);
      if (s && !P.active[0][s - 1]) s = 0;
      if (s) {
        const I jk = (I)y + (I)P.ny * (I)(k0 - 1);
        bx[n].s = s;
        bx[n].q = q;
        bx[n].pq = (I)(halo + 1) * jk + (I)q + (s == 2 ? (I)AX.psi_side : (I)0);
        bx[n].xq = (I)halo * jk + (I)(q - 1) + (s == 2 ? (I)AX.xi_side : (I)0);
      }
    }
    if (rowv) {
      int q;
      bool f;
      int s = band_of(y, P.ny, halo, P.first_r[1], q, f);
      if (s && !P.active[1][s - 1]) s = 0;
      if (s) {
        by.s = s;
        by.q = q;
        by.pq = (I)x0 + px * ((I)q + (I)(halo + 1) * (I)(k0 - 1)) +
                (s == 2 ? (I)AY.psi_side : (I)0);
        by.xq = (I)x0 + px * ((I)(q - 1) + (I)halo * (I)(k0 - 1)) +
                (s == 2 ? (I)AY.xi_side : (I)0);
      }
    }
  }
  const I xq_dz = (I)(halo + 1) * (I)P.ny, xxq_dz = (I)halo * (I)P.ny;
  const I yq_dz = px * (I)(halo + 1), yxq_dz = px * (I)halo;
  const T ix2 = P.inv_d2[0], iy2 = P.inv_d2[1], iz2 = P.inv_d2[2];

  // register queues of the own columns: p_s at m-1, m (m+1 loaded each
  // plane); p_{s+1} at m-2, m-1; fact at m-1; level-1 band results of m-1
  V2 ptm{}, ptc{}, p1m{}, p1c{}, fprev{};
  Lv1<T> lx[2] = {}, ly[2] = {}, lz[2] = {};  // level-1 band results of the previous plane
  T z1carry[2] = {}, z2carry[2] = {};  // new ψ_z on the upper face of the previous plane
  int szp = 0, qzp = 0;                // z band of the previous plane
  bool fzp = false;

  const int wr = P.wait_rounds, wns = P.wait_ns;
  int ucons = -1;  // last load index whose phase this thread has seen complete
  if (tb_wait(&full[0], 0, wr, wns)) ucons = 0;
  if (ucons == 0 && tb_wait(&full[1 % S], (1 / S) & 1, wr, wns)) ucons = 1;
  if (ucons != 1) abort[2] = 1;
  __syncthreads();
  const bool go = !abort[2];  // uniform: written before the barrier only
  if (go) {
    ptm = *reinterpret_cast<const V2*>(reinterpret_cast<const T*>(smem) + ip);
    ptc = *reinterpret_cast<const V2*>(reinterpret_cast<const T*>(smem + (1 % S) * L::STAGE) + ip);
  }
  I o = col + plane * (I)(k0 - 1);  // node 0's offset at plane m
  int sm_ = 1 % S, sp_ = 2 % S;      // stages of planes m and m+1
  int u1 = 2;                        // load index of plane m+1
  // One plane iteration, compiled for each combination of "plane m lies in
  // an active z band" (ZB1, level 1) and "plane m-1 does" (ZB2, level 2), so
  // that the z-band code runs only on those planes instead of being
  // predicated over all of them. Returns true when the block must stop.
  //
  // Order within an iteration: (A) the x/y band part of level 2 at plane
  // m-1, which needs only the step-s+1 values of plane m-1 and the level-1
  // x/y band results of plane m-1; (B) level 1 at plane m, whose x/y band
  // results then replace those; (C) the rest of level 2 at plane m-1, which
  // needs step s+1 at plane m. The damping terms still add up x, y, z.
  int m = k0 - 1;
  int sz = 0, qz = 0;  // z band of plane m
  bool fz = false;
  auto iteration = [&](auto zb1, auto zb2) -> bool {
    constexpr bool ZB1 = decltype(zb1)::value, ZB2 = decltype(zb2)::value;
    const int par = m & 1;
    const bool ok = tb_wait(&full[sp_], (u1 / S) & 1, wr, wns);
    if (ok)
      ucons = u1;
    else
      abort[par] = 1;
    V2 v1{}, f{}, ptp{};
    Lv1<T> cz[2] = {};
    if (ok) {
      const T* pt = reinterpret_cast<const T*>(smem + sm_ * L::STAGE);
      const T* sto = reinterpret_cast<const T*>(smem + sm_ * L::STAGE + L::PT_PAD);
      const T* stf = reinterpret_cast<const T*>(smem + sm_ * L::STAGE + L::PT_PAD + L::IN_PAD);
      ptp = *reinterpret_cast<const V2*>(reinterpret_cast<const T*>(smem + sp_ * L::STAGE) + ip);
      const int m2 = m - 1;
      const bool do2 = lv2 && m2 >= k0 && m2 < k1;
      const T* sl = slot + (par ^ 1) * L::SLOT;  // step s+1 at plane m-1
      // ---- (A) level 2, x/y part: second differences and x/y band --------
      T d2x2[2] = {}, d2y2[2] = {}, damp2[2] = {};
      bool band2[2] = {false, false};
      if (do2) {
        const T xl = sl[si - 1], xh = sl[si + 2];
        const V2 ym = *reinterpret_cast<const V2*>(sl + si - L::RX);
        const V2 yp = *reinterpret_cast<const V2*>(sl + si + L::RX);
        const T pcs[2] = {p1c.x, p1c.y}, xms[2] = {xl, p1c.x}, xps[2] = {p1c.y, xh};
        const T yms[2] = {ym.x, ym.y}, yps[2] = {yp.x, yp.y}, fs[2] = {fprev.x, fprev.y};
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          const T c = pcs[n];
          d2x2[n] = second_diff(xms[n], c, xps[n], ix2);
          d2y2[n] = second_diff(yms[n], c, yps[n], iy2);
          if (XY && bx[n].s && own[n]) {
            const int q = bx[n].q, R = bx[n].s == 2;
            T sq, sm, xn;
            cpml_axis(tb_coef(AX, q + (R ? halo + 1 : 0), q - 1 + (R ? halo : 0)), lx[n].sq,
                      lx[n].sm, lx[n].xn, xms[n], c, xps[n], d2x2[n], fs[n], P.inv_d[0], sq, sm,
                      xn, damp2[n]);
            const I q2 = bx[n].pq - xq_dz;
            AX.psi_out[q2] = sq;
            if (q == (R ? qfx : 1)) AX.psi_out[q2 - 1] = sm;
            AX.xi_out[bx[n].xq - xxq_dz] = xn;
            band2[n] = true;
          }
          if (XY && by.s && own[n]) {
            const int q = by.q, R = by.s == 2;
            T sq, sm, xn;
            cpml_axis(tb_coef(AY, q + (R ? halo + 1 : 0), q - 1 + (R ? halo : 0)), ly[n].sq,
                      ly[n].sm, ly[n].xn, yms[n], c, yps[n], d2y2[n], fs[n], P.inv_d[1], sq, sm,
                      xn, damp2[n]);
            const I q2 = by.pq + (I)n - yq_dz;
            AY.psi_out[q2] = sq;
            if (q == (R ? qfy : 1)) AY.psi_out[q2 - px] = sm;
            AY.xi_out[by.xq + (I)n - yxq_dz] = xn;
            band2[n] = true;
          }
        }
      }
      // ---- (B) level 1: step s+1 on the pair at plane m --------------------
      if (anyv && m >= 1 && m <= P.nz - 2) {
        const V2 c = *reinterpret_cast<const V2*>(pt + ip);
        const T xl = pt[ip - 1], xh = pt[ip + 2];
        const V2 ym = *reinterpret_cast<const V2*>(pt + ip - L::BX);
        const V2 yp = *reinterpret_cast<const V2*>(pt + ip + L::BX);
        const V2 po = *reinterpret_cast<const V2*>(sto + ii);
        f = *reinterpret_cast<const V2*>(stf + ii);
        const T pcs[2] = {c.x, c.y}, xms[2] = {xl, c.x}, xps[2] = {c.y, xh};
        const T yms[2] = {ym.x, ym.y}, yps[2] = {yp.x, yp.y}, pos[2] = {po.x, po.y};
        const T fs[2] = {f.x, f.y}, zms[2] = {ptm.x, ptm.y}, zps[2] = {ptp.x, ptp.y};
        T vs[2];
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          const T pc = pcs[n];
          const T d2x = second_diff(xms[n], pc, xps[n], ix2);
          const T d2y = second_diff(yms[n], pc, yps[n], iy2);
          const T d2z = second_diff(zms[n], pc, zps[n], iz2);
          T v = leapfrog3d(pc, pos[n], fs[n], d2x, d2y, d2z);
          T damp = 0;
          bool band = false;
          if (XY && bx[n].s) {
            const int q = bx[n].q, R = bx[n].s == 2;
            cpml_axis(tb_coef(AX, q + (R ? halo + 1 : 0), q - 1 + (R ? halo : 0)),
                      AX.psi_in[bx[n].pq], AX.psi_in[bx[n].pq - 1], AX.xi_in[bx[n].xq], xms[n], pc,
                      xps[n], d2x, fs[n], P.inv_d[0], lx[n].sq, lx[n].sm, lx[n].xn, damp);
            band = true;
          }
          if (XY && by.s && colv[n]) {
            const int q = by.q, R = by.s == 2;
            const I yq = by.pq + (I)n;
            cpml_axis(tb_coef(AY, q + (R ? halo + 1 : 0), q - 1 + (R ? halo : 0)), AY.psi_in[yq],
                      AY.psi_in[yq - px], AY.xi_in[by.xq + (I)n], yms[n], pc, yps[n], d2y, fs[n],
                      P.inv_d[1], ly[n].sq, ly[n].sm, ly[n].xn, damp);
            band = true;
          }
          if (ZB1 && colv[n]) {
            const bool zR = sz == 2;
            const int hq = qz + (zR ? halo + 1 : 0), g = qz - 1 + (zR ? halo : 0);
            const I zp = col + (I)n + plane * (I)qz + (zR ? (I)AZ.psi_side : (I)0);
            const I zx = col + (I)n + plane * (I)(qz - 1) + (zR ? (I)AZ.xi_side : (I)0);
            const T inv = P.inv_d[2];
            cz[n].sq = psi_face(__ldg(AZ.bKh + hq), __ldg(AZ.ah + hq), AZ.psi_in[zp],
                                zps[n] - pc, inv);
            // the lower face's new ψ is the previous plane's upper-face value
            // (same operands) unless this plane starts the band or the chunk
            cz[n].sm = (m > k0 - 1 && !fz)
                           ? z1carry[n]
                           : psi_face(__ldg(AZ.bKh + hq - 1), __ldg(AZ.ah + hq - 1),
                                      AZ.psi_in[zp - plane], pc - zms[n], inv);
            cpml_tail(__ldg(AZ.bK + g), __ldg(AZ.a + g), cz[n].sq, cz[n].sm, AZ.xi_in[zx], d2z,
                      fs[n], inv, cz[n].xn, damp);
            z1carry[n] = cz[n].sq;
            band = true;
          }
          if (band || P.damp_all) v += damp;
          vs[n] = colv[n] ? v : T(0);
        }
        v1 = V2{vs[0], vs[1]};
      }
      // sources (and the owner's receivers) of step s+1 on this plane
      if (e1 < e_end) {
        while (e1 < e_end && P.io.ent[e1].y < m) ++e1;
        for (; e1 < e_end; ++e1) {
          const int4 en = P.io.ent[e1];
          if (en.y != m) break;
          if ((en.x >> 1) == tid) {
            if (en.x & 1)
              v1.y = node_io(P.io, P.it, en.z, en.w, v1.y);
            else
              v1.x = node_io(P.io, P.it, en.z, en.w, v1.x);
          }
        }
      }
      if (m >= k0 && m < k1) {
        if (own[0] && own[1])
          *reinterpret_cast<V2*>(P.p1 + o) = v1;
        else if (own[0])
          P.p1[o] = v1.x;
        else if (own[1])
          P.p1[o + 1] = v1.y;
      }
      *reinterpret_cast<V2*>(slot + par * L::SLOT + si) = v1;
      // ---- (C) level 2, the rest: step s+2 on the pair's tile nodes at m-1
      if (do2) {
        const T pcs[2] = {p1c.x, p1c.y}, pos[2] = {ptm.x, ptm.y};
        const T fs[2] = {fprev.x, fprev.y}, zms[2] = {p1m.x, p1m.y}, zps[2] = {v1.x, v1.y};
        const I o2 = o - plane;
        T vs[2];
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          const T c = pcs[n];
          const T d2z = second_diff(zms[n], c, zps[n], iz2);
          T v = leapfrog3d(c, pos[n], fs[n], d2x2[n], d2y2[n], d2z);
          T damp = damp2[n];
          bool band = band2[n];
          if (ZB2 && own[n]) {
            const bool zR = szp == 2;
            const int hq = qzp + (zR ? halo + 1 : 0), g = qzp - 1 + (zR ? halo : 0);
            const T inv = P.inv_d[2];
            const T sq = psi_face(__ldg(AZ.bKh + hq), __ldg(AZ.ah + hq), lz[n].sq, zps[n] - c, inv);
            const T sm = (m2 > k0 && !fzp) ? z2carry[n]
                                           : psi_face(__ldg(AZ.bKh + hq - 1), __ldg(AZ.ah + hq - 1),
                                                      lz[n].sm, c - zms[n], inv);
            T xn;
            cpml_tail(__ldg(AZ.bK + g), __ldg(AZ.a + g), sq, sm, lz[n].xn, d2z, fs[n], inv, xn,
                      damp);
            const I zp = col + (I)n + plane * (I)qzp + (zR ? (I)AZ.psi_side : (I)0);
            AZ.psi_out[zp] = sq;
            if (fzp) AZ.psi_out[zp - plane] = sm;
            AZ.xi_out[col + (I)n + plane * (I)(qzp - 1) + (zR ? (I)AZ.xi_side : (I)0)] = xn;
            z2carry[n] = sq;
            band = true;
          }
          if (band || P.damp_all) v += damp;
          vs[n] = v;
        }
        if (e2 < e_end) {
          while (e2 < e_end && P.io.ent[e2].y < m2) ++e2;
          for (; e2 < e_end; ++e2) {
            const int4 en = P.io.ent[e2];
            if (en.y != m2) break;
            if ((en.x >> 1) == tid) {
              if (en.x & 1)
                vs[1] = node_io(P.io, P.it + 1, en.z, en.w, vs[1]);
              else
                vs[0] = node_io(P.io, P.it + 1, en.z, en.w, vs[0]);
            }
          }
        }
        if (own[0] && own[1])
          *reinterpret_cast<V2*>(P.p2 + o2) = V2{vs[0], vs[1]};
        else if (own[0])
          P.p2[o2] = vs[0];
        else if (own[1])
          P.p2[o2 + 1] = vs[1];
      }
    }
    __syncthreads();
    if (abort[par]) return true;
    // the stage of plane m is free: refill it (and, on the first plane, the
    // stage of plane k0-2) with the next planes
    if (tid == 0)
      for (; next_u < nplanes && next_u <= u1 + S - 1; ++next_u) issue(next_u);
    // rotate the columns' queues
    p1m = p1c;
    p1c = v1;
    ptm = ptc;
    ptc = ptp;
    fprev = f;
#pragma unroll
    for (int n = 0; n < 2; ++n) {
      lz[n] = cz[n];
      if (XY) {
        bx[n].pq += xq_dz;
        bx[n].xq += xxq_dz;
      }
    }
    if (XY) {
      by.pq += yq_dz;
      by.xq += yxq_dz;
    }
    szp = sz;
    qzp = qz;
    fzp = fz;
    sm_ = sp_;
    sp_ = sp_ + 1 == S ? 0 : sp_ + 1;
    return false;
  };
  for (; go && m <= k1; ++m, o += plane, ++u1) {
    // z band of this plane (uniform over the block)
    sz = 0;
    qz = 0;
    fz = false;
    if (m >= 1 && m <= P.nz - 2) {
      sz = band_of(m, P.nz, halo, P.first_r[2], qz, fz);
      if (sz && !P.active[2][sz - 1]) sz = 0;
    }
    using Y = std::true_type;
    using N = std::false_type;
    const bool stop = sz ? (szp ? iteration(Y{}, Y{}) : iteration(Y{}, N{}))
                         : (szp ? iteration(N{}, Y{}) : iteration(N{}, N{}));
    if (stop) break;
  }
  if (abort[0] || abort[1] || abort[2]) {
    // a wait ran out: record it and let the producer drain the loads still in
    // flight before the block's shared memory goes away
    if (tid == 0) {
      atomicExch(P.err, 1);
      for (int u = ucons + 1; u < next_u; ++u)
        if (u != P.withhold) tb_wait(&full[u % S], (u / S) & 1, 64, 1000000);
    }
  }
}

// Pipeline stages of the two-step kernel; its level-1 region has 8 or 16
// rows (blocks of 256 or 512 threads).
constexpr int TB_STAGES = 4;

// Host side, defined in awc_tb.cu (the kernel instantiations live there).
// Launches one two-step pass over `nblocks` blocks (tiles x z chunks) of the
// XY (tiles meeting an x or y band) or Z variant with `rows` region rows,
// with int64 offsets when i64.
template <typename T>
cudaError_t tb_launch(const TbParams<T>& P, bool xy, bool i64, int rows, const CUtensorMap& mpt,
                      const CUtensorMap& mpo, const CUtensorMap& mf, unsigned nblocks,
                      cudaStream_t st);
// Opts every instantiation into its dynamic shared memory on the current device.
cudaError_t tb_init_attrs();
// Resident blocks per SM of the kernel variant.
int tb_occupancy(bool f64, bool xy, int rows);

}  // namespace awc
