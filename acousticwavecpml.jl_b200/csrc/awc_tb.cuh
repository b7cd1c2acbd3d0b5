// awc_tb.cuh — the 3D CPML step advanced two time steps per pass (temporal
// blocking).
//
// A pass computes, for every interior node, the pressure of steps s+1 and
// s+2 from those of steps s-1 and s, and the CPML state (ψ, ξ) of step s+2
// from that of step s: two applications of the reference's forward!
// (src/shared/acoustic_3D_xPU.jl:124-167) with the same arithmetic, operation
// for operation, as the one-step kernels of awc_kernels.cuh (so a run gives
// bitwise the results of one-step passes). Per node and pass the fields cost
// 5 words of HBM traffic (read pold, pcur, fact; write the two new fields)
// instead of 8 for two one-step passes, and each live CPML entry is read and
// written once instead of twice.
//
// Geometry. A block of 32 x W threads owns a column tile of 30 x (W-2)
// interior nodes (the level-2 tile) and streams a chunk of z planes. Thread
// (lane, w) owns the column x = X0 - 1 + lane, y = Y0 - 1 + w of the
// 32 x W level-1 region, which is the tile plus a ring of one node: the
// ring's step-s+1 values are the neighbours of the tile's step-s+2 update,
// so every thread computes step s+1 on its column (from the staged p_s,
// p_{s-1} and fact) and the inner 30 x (W-2) threads then compute step s+2
// on theirs. The step-s+1 values of one plane are exchanged through a
// two-slot shared-memory ring; each thread keeps its own column's z
// neighbours (p_s and p_{s+1} of three planes) in registers.
//
// Staging. One elected thread streams, per z plane, three TMA boxes into a
// ring of S stages: p_s on the region plus one node ((40) x (W+2), x origin
// rounded down to 16 bytes), p_{s-1} and fact on the region (40 x W). One
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
  // entries {thread, plane, source group, receiver group or -1}, sorted by
  // (plane, thread); a node appears in the list of every block whose level-1
  // region and plane range hold it, with its receiver group only in its owner's
  Io<T> io;
  const int2* tiles;  // level-2 tile origins (x0, y0) of this launch
  int32_t nch, zc;    // z chunks per tile, planes per chunk
  int32_t wait_rounds, wait_ns;  // bounded waits: rounds x suspend hint (ns)
  int32_t withhold;              // test only: load index the producer skips (-1: none)
};

template <typename T, int W>
struct TbTile {
  static constexpr int NT = 32 * W;
  static constexpr int BX = 40;  // box width: 34 columns + x alignment slack
  static constexpr int A = 16 / (int)sizeof(T);
  static constexpr int PT_BYTES = BX * (W + 2) * (int)sizeof(T);
  static constexpr int IN_BYTES = BX * W * (int)sizeof(T);
  static constexpr int PT_PAD = (PT_BYTES + 127) / 128 * 128;
  static constexpr int IN_PAD = (IN_BYTES + 127) / 128 * 128;
  static constexpr int STAGE = PT_PAD + 2 * IN_PAD;
};

template <typename T, int W, int S>
constexpr int tb_smem() {
  return S * TbTile<T, W>::STAGE + 2 * TbTile<T, W>::NT * (int)sizeof(T) + 8 * S + 16;
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

template <typename T, typename I, int W, int S, bool XY>
__global__ void __launch_bounds__(32 * W) step3d_tb(const __grid_constant__ CUtensorMap mpt,
                                                    const __grid_constant__ CUtensorMap mpo,
                                                    const __grid_constant__ CUtensorMap mf,
                                                    TbParams<T> P) {
  using L = TbTile<T, W>;
  extern __shared__ __align__(128) unsigned char smem[];
  T* slot = reinterpret_cast<T*>(smem + S * L::STAGE);  // [2][NT] step-s+1 values
  uint64_t* full = reinterpret_cast<uint64_t*>(slot + 2 * L::NT);
  // abort flags: [0], [1] by iteration parity (a flag is only written before
  // the barrier of its iteration and read after it), [2] for the prologue
  volatile int* abort = reinterpret_cast<volatile int*>(full + S);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int blk = blockIdx.x;
  const int2 org = P.tiles[blk / P.nch];
  const int k0 = 1 + (blk % P.nch) * P.zc;
  const int k1 = min(k0 + P.zc, P.nz - 1);
  if (k0 >= k1) return;  // block-uniform
  const int xr = org.x - 1, yr = org.y - 1;
  const int xa = floor_div(xr - 1, L::A) * L::A;  // 16-byte-aligned box origin
  const int ox = xr - xa;                         // 1..A
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

  const int x = xr + lane, y = yr + w;
  const bool colv = x >= 1 && x <= P.nx - 2 && y >= 1 && y <= P.ny - 2;
  const bool inner = lane >= 1 && lane <= 30 && w >= 1 && w <= W - 2;
  const bool own = inner && colv;
  const int ip = (w + 1) * L::BX + lane + ox;  // this column in the p_s box
  const int ii = w * L::BX + lane + ox;        // in the p_{s-1} / fact boxes
  const int halo = P.halo;
  const I px = (I)P.px, plane = (I)P.plane;
  const I col = (I)x + px * (I)y;
  int e1 = P.io.blk_off[blk], e2 = e1;
  const int e_end = P.io.blk_off[blk + 1];

  // band state of the column along x and y (XY launches only)
  int sx = 0, qx = 0, sy = 0, qy = 0;
  bool fx = false, fy = false;
  I xq = 0, xxq = 0, yq = 0, yxq = 0;  // ψ[q] / ξ[q-1] offsets at the current plane
  if (XY && colv) {
    sx = band_of(x, P.nx, halo, P.first_r[0], qx, fx);
    if (sx && !P.active[0][sx - 1]) sx = 0;
    sy = band_of(y, P.ny, halo, P.first_r[1], qy, fy);
    if (sy && !P.active[1][sy - 1]) sy = 0;
  }
  const TbAxis<T>&AX = P.ax[0], &AY = P.ax[1], &AZ = P.ax[2];
  if (XY && sx) {
    const I jk = (I)y + (I)P.ny * (I)(k0 - 1);
    xq = (I)(halo + 1) * jk + (I)qx + (sx == 2 ? (I)AX.psi_side : (I)0);
    xxq = (I)halo * jk + (I)(qx - 1) + (sx == 2 ? (I)AX.xi_side : (I)0);
  }
  if (XY && sy) {
    yq = (I)x + px * ((I)qy + (I)(halo + 1) * (I)(k0 - 1)) + (sy == 2 ? (I)AY.psi_side : (I)0);
    yxq = (I)x + px * ((I)(qy - 1) + (I)halo * (I)(k0 - 1)) + (sy == 2 ? (I)AY.xi_side : (I)0);
  }
  const I xq_dz = (I)(halo + 1) * (I)P.ny, xxq_dz = (I)halo * (I)P.ny;
  const I yq_dz = px * (I)(halo + 1), yxq_dz = px * (I)halo;
  const int hx = qx + (sx == 2 ? halo + 1 : 0), gx = qx - 1 + (sx == 2 ? halo : 0);
  const int hy = qy + (sy == 2 ? halo + 1 : 0), gy = qy - 1 + (sy == 2 ? halo : 0);

  // register queues of the own column: p_s at m-1, m (and m+1 loaded each
  // plane); p_{s+1} at m-2, m-1; fact at m-1; level-1 band results of m-1
  T ptm = 0, ptc = 0, p1m = 0, p1c = 0, fprev = 0;
  Lv1<T> bx{}, by{}, bz{};     // level-1 band results of the previous plane
  T z1carry = 0, z2carry = 0;  // new ψ_z on the upper face of the previous plane (levels 1, 2)
  int szp = 0, qzp = 0;        // z band of the previous plane
  bool fzp = false;

  const int wr = P.wait_rounds, wns = P.wait_ns;
  int ucons = -1;  // last load index whose phase this thread has seen complete
  if (tb_wait(&full[0], 0, wr, wns)) ucons = 0;
  if (ucons == 0 && tb_wait(&full[1 % S], (1 / S) & 1, wr, wns)) ucons = 1;
  if (ucons != 1) abort[2] = 1;
  __syncthreads();
  const bool go = !abort[2];  // uniform: written before the barrier only
  if (go) {
    ptm = reinterpret_cast<const T*>(smem)[ip];
    ptc = reinterpret_cast<const T*>(smem + (1 % S) * L::STAGE)[ip];
  }
  I o = col + plane * (I)(k0 - 1);  // this column's offset at plane m
  for (int m = k0 - 1; go && m <= k1; ++m, o += plane) {
    const int par = m & 1;
    const int u1 = m - k0 + 3;  // load index of plane m+1
    if (tb_wait(&full[u1 % S], (u1 / S) & 1, wr, wns))
      ucons = u1;
    else
      abort[par] = 1;
    // z band of this plane (uniform over the block)
    int sz = 0, qz = 0;
    bool fz = false;
    if (m >= 1 && m <= P.nz - 2) {
      sz = band_of(m, P.nz, halo, P.first_r[2], qz, fz);
      if (sz && !P.active[2][sz - 1]) sz = 0;
    }
    T v1 = 0, f = 0, ptp = 0;
    Lv1<T> cx{}, cy{}, cz{};
    if (!abort[par]) {
      const T* stm = reinterpret_cast<const T*>(smem + ((m - k0 + 2) % S) * L::STAGE);
      ptp = reinterpret_cast<const T*>(smem + (u1 % S) * L::STAGE)[ip];
      // ---- level 1: step s+1 at (x, y, m) --------------------------------
      if (colv && m >= 1 && m <= P.nz - 2) {
        const T pc = ptc;
        const T xm = stm[ip - 1], xp = stm[ip + 1], ym = stm[ip - L::BX], yp = stm[ip + L::BX];
        const T* sto = reinterpret_cast<const T*>(reinterpret_cast<const unsigned char*>(stm) + L::PT_PAD);
        const T* stf = reinterpret_cast<const T*>(reinterpret_cast<const unsigned char*>(stm) + L::PT_PAD + L::IN_PAD);
        const T po = sto[ii];
        f = stf[ii];
        const T d2x = second_diff(xm, pc, xp, P.inv_d2[0]);
        const T d2y = second_diff(ym, pc, yp, P.inv_d2[1]);
        const T d2z = second_diff(ptm, pc, ptp, P.inv_d2[2]);
        v1 = leapfrog3d(pc, po, f, d2x, d2y, d2z);
        T damp = 0;
        if (XY && sx) {
          const BandCoef<T> c{__ldg(AX.bKh + hx), __ldg(AX.ah + hx), __ldg(AX.bKh + hx - 1),
                              __ldg(AX.ah + hx - 1), __ldg(AX.bK + gx), __ldg(AX.a + gx)};
          cpml_axis(c, AX.psi_in[xq], AX.psi_in[xq - 1], AX.xi_in[xxq], xm, pc, xp, d2x, f,
                    P.inv_d[0], cx.sq, cx.sm, cx.xn, damp);
        }
        if (XY && sy) {
          const BandCoef<T> c{__ldg(AY.bKh + hy), __ldg(AY.ah + hy), __ldg(AY.bKh + hy - 1),
                              __ldg(AY.ah + hy - 1), __ldg(AY.bK + gy), __ldg(AY.a + gy)};
          cpml_axis(c, AY.psi_in[yq], AY.psi_in[yq - px], AY.xi_in[yxq], ym, pc, yp, d2y, f,
                    P.inv_d[1], cy.sq, cy.sm, cy.xn, damp);
        }
        if (sz) {
          const bool zR = sz == 2;
          const int hq = qz + (zR ? halo + 1 : 0), g = qz - 1 + (zR ? halo : 0);
          const I zp = col + plane * (I)qz + (zR ? (I)AZ.psi_side : (I)0);
          const I zx = col + plane * (I)(qz - 1) + (zR ? (I)AZ.xi_side : (I)0);
          const T inv = P.inv_d[2];
          cz.sq = psi_face(__ldg(AZ.bKh + hq), __ldg(AZ.ah + hq), AZ.psi_in[zp], ptp - pc, inv);
          // the lower face's new ψ is the previous plane's upper-face value
          // (same operands) unless this plane starts the band or the chunk
          cz.sm = (m > k0 - 1 && !fz) ? z1carry
                                      : psi_face(__ldg(AZ.bKh + hq - 1), __ldg(AZ.ah + hq - 1),
                                                 AZ.psi_in[zp - plane], pc - ptm, inv);
          cpml_tail(__ldg(AZ.bK + g), __ldg(AZ.a + g), cz.sq, cz.sm, AZ.xi_in[zx], d2z, f, inv,
                    cz.xn, damp);
          z1carry = cz.sq;
        }
        if ((XY && (sx || sy)) || sz || P.damp_all) v1 += damp;
      }
      // sources (and the owner's receivers) of step s+1 on this plane
      while (e1 < e_end && P.io.ent[e1].y < m) ++e1;
      for (; e1 < e_end; ++e1) {
        const int4 en = P.io.ent[e1];
        if (en.y != m) break;
        if (en.x == tid) v1 = node_io(P.io, P.it, en.z, en.w, v1);
      }
      const bool in_chunk = m >= k0 && m < k1;
      if (own && in_chunk) P.p1[o] = v1;
      slot[par * L::NT + tid] = v1;
      // ---- level 2: step s+2 at (x, y, m-1) ------------------------------
      const int m2 = m - 1;
      if (own && m2 >= k0 && m2 < k1) {
        const T* sl = slot + (par ^ 1) * L::NT;
        const T c = p1c;
        const T xm = sl[tid - 1], xp = sl[tid + 1], ym = sl[tid - 32], yp = sl[tid + 32];
        const T d2x = second_diff(xm, c, xp, P.inv_d2[0]);
        const T d2y = second_diff(ym, c, yp, P.inv_d2[1]);
        const T d2z = second_diff(p1m, c, v1, P.inv_d2[2]);
        T v2 = leapfrog3d(c, ptm, fprev, d2x, d2y, d2z);
        T damp = 0;
        const I o2 = o - plane;
        if (XY && sx) {
          const BandCoef<T> cf{__ldg(AX.bKh + hx), __ldg(AX.ah + hx), __ldg(AX.bKh + hx - 1),
                               __ldg(AX.ah + hx - 1), __ldg(AX.bK + gx), __ldg(AX.a + gx)};
          T sq, sm, xn;
          cpml_axis(cf, bx.sq, bx.sm, bx.xn, xm, c, xp, d2x, fprev, P.inv_d[0], sq, sm, xn, damp);
          const I q2 = xq - xq_dz, x2 = xxq - xxq_dz;
          AX.psi_out[q2] = sq;
          if (fx) AX.psi_out[q2 - 1] = sm;
          AX.xi_out[x2] = xn;
        }
        if (XY && sy) {
          const BandCoef<T> cf{__ldg(AY.bKh + hy), __ldg(AY.ah + hy), __ldg(AY.bKh + hy - 1),
                               __ldg(AY.ah + hy - 1), __ldg(AY.bK + gy), __ldg(AY.a + gy)};
          T sq, sm, xn;
          cpml_axis(cf, by.sq, by.sm, by.xn, ym, c, yp, d2y, fprev, P.inv_d[1], sq, sm, xn, damp);
          const I q2 = yq - yq_dz, x2 = yxq - yxq_dz;
          AY.psi_out[q2] = sq;
          if (fy) AY.psi_out[q2 - px] = sm;
          AY.xi_out[x2] = xn;
        }
        if (szp) {
          const bool zR = szp == 2;
          const int hq = qzp + (zR ? halo + 1 : 0), g = qzp - 1 + (zR ? halo : 0);
          const T inv = P.inv_d[2];
          const T sq = psi_face(__ldg(AZ.bKh + hq), __ldg(AZ.ah + hq), bz.sq, v1 - c, inv);
          const T sm = (m2 > k0 && !fzp) ? z2carry
                                         : psi_face(__ldg(AZ.bKh + hq - 1), __ldg(AZ.ah + hq - 1),
                                                    bz.sm, c - p1m, inv);
          T xn;
          cpml_tail(__ldg(AZ.bK + g), __ldg(AZ.a + g), sq, sm, bz.xn, d2z, fprev, inv, xn, damp);
          const I zp = col + plane * (I)qzp + (zR ? (I)AZ.psi_side : (I)0);
          AZ.psi_out[zp] = sq;
          if (fzp) AZ.psi_out[zp - plane] = sm;
          AZ.xi_out[col + plane * (I)(qzp - 1) + (zR ? (I)AZ.xi_side : (I)0)] = xn;
          z2carry = sq;
        }
        if ((XY && (sx || sy)) || szp || P.damp_all) v2 += damp;
        while (e2 < e_end && P.io.ent[e2].y < m2) ++e2;
        for (; e2 < e_end; ++e2) {
          const int4 en = P.io.ent[e2];
          if (en.y != m2) break;
          if (en.x == tid) v2 = node_io(P.io, P.it + 1, en.z, en.w, v2);
        }
        P.p2[o2] = v2;
      }
    }
    __syncthreads();
    if (abort[par]) break;
    // the stage of plane m is free: refill it (and, on the first plane, the
    // stage of plane k0-2) with the next planes
    if (tid == 0)
      for (; next_u < nplanes && next_u <= m - k0 + 2 + S; ++next_u) issue(next_u);
    // rotate the column's queues
    p1m = p1c;
    p1c = v1;
    ptm = ptc;
    ptc = ptp;
    fprev = f;
    bx = cx;
    by = cy;
    bz = cz;
    szp = sz;
    qzp = qz;
    fzp = fz;
    if (XY && sx) {
      xq += xq_dz;
      xxq += xxq_dz;
    }
    if (XY && sy) {
      yq += yq_dz;
      yxq += yxq_dz;
    }
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

}  // namespace awc

namespace awc {
// Pipeline stages and level-1 region rows of the two-step kernel.
constexpr int TB_STAGES = 4;
constexpr int TB_ROWS = 16;

// Host side, defined in awc_tb.cu (the kernel instantiations live there).
// Launches one two-step pass over `nblocks` blocks (tiles x z chunks) of the
// XY (tiles meeting an x or y band) or Z variant, with int64 offsets when i64.
template <typename T>
cudaError_t tb_launch(const TbParams<T>& P, bool xy, bool i64, const CUtensorMap& mpt,
                      const CUtensorMap& mpo, const CUtensorMap& mf, unsigned nblocks,
                      cudaStream_t st);
// Opts every instantiation into its dynamic shared memory on the current device.
cudaError_t tb_init_attrs();
// Resident blocks per SM of the kernel variant.
int tb_occupancy(bool f64, bool xy);
}  // namespace awc
