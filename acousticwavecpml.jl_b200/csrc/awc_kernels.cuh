// awc_kernels.cuh — sm_100a kernels of one CPML acoustic time step.
//
// One launch of a step kernel is one whole time step of the reference's
// forward! (src/shared/acoustic_3D_xPU.jl:124-167; 2D
// src/shared/acoustic_2D_xPU.jl:93-131):
//   - update_ψ_{x,y,z}! + update_p! (:8-104): for every interior node the
//     2nd-order Laplacian of pcur, inside the CPML bands the staggered ψ
//     recursion, the ξ recursion and the damping term, then the leapfrog
//     update pnew = 2 pcur - pold + fact*lap + damp;
//   - inject_sources! + record_receivers! (:106-122): the thread that owns a
//     node adds that node's sources to its new value and samples it for the
//     node's receivers; nodes on the Dirichlet rim, which no thread updates,
//     are served by block 0 (nothing else writes the rim of pnew during a
//     step, so this needs no ordering against the other blocks).
//
// Memory layout in HBM (x fastest, like the reference's column-major arrays;
// px = nx rounded up to 32 elements, so rows are 128/256-byte aligned and
// every TMA stride and tile origin is 16-byte aligned):
//   p fields, fact   node (i, j, k) at i + px*(j + ny*k)
//   ψ axis x  (halo+1, ny, nz)   q + (halo+1)*(j + ny*k)
//   ψ axis y  (px, halo+1, nz)   i + px*(q + (halo+1)*k)
//   ψ axis z  (px, ny, halo+1)   i + px*(j + ny*q)
//   ξ         the same with halo entries and q-1 in place of q.
// ψ is double-buffered (old/new): node c needs the new ψ on both of its
// faces, ψ[q] (between c and c+1) and ψ[q-1] (between c-1 and c). Both depend
// only on pcur and the old ψ, so each node recomputes the two values it needs
// and writes only ψ[q] (plus ψ[q-1] for the first node of a band); reading
// the old buffer while writing the new one removes the cross-block race a
// single buffer would have. ξ has one reader/writer per entry and stays in
// place. ψ on the Dirichlet rim (j or k on the outer rows) is never read by
// the pressure update in the reference and is not stored as live state here.
//
// Index conventions below are 0-based: reference node I (1-based) is c = I-1.
// Left band: c <= halo, ψ index q = c. Right band: c >= n-halo-1 (and not in
// the left band), q = c - (n-halo-2). ξ and on-grid coefficients use q-1,
// half-grid coefficients use q and q-1.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace awc {

template <typename T>
struct BandSide {
  const T* psi_old;
  T* psi_new;
  T* xi;
  const T* a;    // on-grid a (halo)
  const T* bK;   // on-grid b/K (halo)
  const T* ah;   // half-grid a (halo+1)
  const T* bKh;  // half-grid b/K (halo+1)
};

// A node that carries sources and/or receivers. Interior entries are
// bucketed by the block that owns the node: {node index inside the block's
// tile, z plane (3D), source group, receiver group}; a group is an index
// into a CSR (off/ids) list, -1 when the node has none of that kind.
struct IoRim {
  int64_t node;  // pitched linear index of a Dirichlet-rim node
  int32_t sgrp, rgrp;
};

template <typename T>
struct Io {
  const int32_t* blk_off;  // per block: [blk_off[b], blk_off[b+1]) into ent
  const int4* ent;         // interior entries sorted by (block, k, local)
  const IoRim* rim;        // rim entries
  int32_t nrim;
  const int32_t* src_off;  // source groups: ids[src_off[g] .. src_off[g+1])
  const int32_t* src_ids;  // source index, in source order within a group
  const int32_t* rec_off;  // receiver groups
  const int32_t* rec_ids;
  const T* stf;            // [nt][nsrc] scaled source time functions
  int32_t nsrc, nrec;
  T* traces;               // [nt][nrec]
};

// Inclusive 0-based node ranges of an axis-aligned box.
struct Box {
  int32_t x0, x1, y0, y1, z0, z1;
  int32_t kind;  // band kernel: which bands the box's nodes lie in (1, 3, 7 or 15)
};

template <typename T>
struct StepParams {
  const T* pold;
  const T* pcur;
  T* pnew;
  const T* fact;
  int32_t nx, ny, nz, halo;
  int64_t px;              // row pitch of fields and y/z band arrays (elements)
  T inv_d[3];
  T inv_d2[3];
  BandSide<T> band[3][2];  // [axis][left/right]
  int32_t active[3][2];    // side carries a non-trivial CPML recursion
  int32_t first_r[3];      // first node (0-based) of the right band per axis
  int32_t zchunk;          // planes per block along z (3D core kernel)
  int32_t it;              // 0-based time step index (row of stf/traces)
  int32_t* err;            // set to 1 when a bounded device wait runs out
  Io<T> io;                // this kernel's sources/receivers
  int32_t do_rim;          // this kernel's block 0 serves the rim nodes
  // 3D core kernel: the box of nodes outside every active CPML band, tiled
  // from x = core_x (a 16-byte-aligned origin at or below core.x0)
  Box core;
  int32_t core_x;
  // 3D shell kernel: disjoint boxes covering the interior nodes outside the
  // core box; box b owns blocks [box_blk[b], box_blk[b+1])
  int32_t nbox;
  Box box[6];
  int32_t box_blk[7];
  int32_t shell_zchunk;  // planes per block of the band kernel
  int64_t plane;             // px * ny
  int64_t psi_dz[2], xi_dz[2];  // x and y: ψ / ξ element step from one z plane to the next
  int64_t psi_side[3], xi_side[3];  // element offset of the right side's ψ / ξ from the left's
};

// Node arithmetic with its rounding pinned. Every kernel forms a second
// difference with a multiply the compiler may not fuse into the following
// add, the leapfrog as one fused multiply-add 2 pc - po + f (Σ d2), and the
// CPML recursions with explicit fused multiply-adds. So the result of a node
// does not depend on which copy of the code computes it: batched and
// single-shot 2D kernels agree bitwise, and so do all launch shapes.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
template <typename T>
__device__ __forceinline__ T second_diff(T m, T c, T p, T inv_d2) {
  return mul_rn(p - T(2) * c + m, inv_d2);
}
template <typename T>
__device__ __forceinline__ T leapfrog2d(T pc, T po, T f, T d2x, T d2y) {
  return fma(f, d2x + d2y, T(2) * pc - po);
}
template <typename T>
__device__ __forceinline__ T leapfrog3d(T pc, T po, T f, T d2x, T d2y, T d2z) {
  return fma(f, d2x + d2y + d2z, T(2) * pc - po);
}

// The CPML coefficients of one band entry q: half-grid b/K and a at q and
// q-1, on-grid b/K and a at q-1.
template <typename T>
struct BandCoef {
  T bh, ah, bhm, ahm, bk, a;
};
template <typename T>
__device__ __forceinline__ BandCoef<T> band_coef(const BandSide<T>& B, int q) {
  return BandCoef<T>{__ldg(B.bKh + q), __ldg(B.ah + q), __ldg(B.bKh + q - 1),
                     __ldg(B.ah + q - 1), __ldg(B.bK + q - 1), __ldg(B.a + q - 1)};
}
// One axis of the CPML band update at one node (update_ψ! on both faces of
// the node, then the ξ recursion and the damping term of update_p!):
// ψ[q] = b/K_half[q] ψ[q] + a_half[q] (pp - pc) / d, ψ[q-1] likewise with
// (pc - pm); dψ = (ψ[q] - ψ[q-1]) / d; ξ = b/K[q-1] ξ + a[q-1] (d2 + dψ);
// damp += f (dψ + ξ).
// psi_face: the new ψ on one face from its old value and the pressure jump
// dp across it; cpml_tail: dψ, ξ and the damping term from both faces' ψ.
template <typename T>
__device__ __forceinline__ T psi_face(T bh, T ah, T ps, T dp, T inv) {
  return fma(bh, ps, mul_rn(mul_rn(ah, dp), inv));
}
template <typename T>
__device__ __forceinline__ void cpml_tail(T bk, T a, T sq, T sm, T xo, T d2, T f, T inv, T& xn,
                                          T& damp) {
  const T dps = mul_rn(sq - sm, inv);
  xn = fma(bk, xo, mul_rn(a, d2 + dps));
  damp = fma(f, dps + xn, damp);
}
template <typename T>
__device__ __forceinline__ void cpml_axis(const BandCoef<T>& c, T psq, T psm, T xo, T pm, T pc,
                                          T pp, T d2, T f, T inv, T& sq, T& sm, T& xn,
                                          T& damp) {
  sq = psi_face(c.bh, c.ah, psq, pp - pc, inv);
  sm = psi_face(c.bhm, c.ahm, psm, pc - pm, inv);
  cpml_tail(c.bk, c.a, sq, sm, xo, d2, f, inv, xn, damp);
}

// Which band (if any) coordinate c of an axis of length n lies in.
// Returns 0 none, 1 left, 2 right; sets q and `first`.
__device__ __forceinline__ int band_of(int c, int n, int halo, int first_r, int& q, bool& first) {
  if (c <= halo) {
    q = c;
    first = (c == 1);
    return 1;
  }
  if (c >= n - halo - 1) {
    q = c - (n - halo - 2);
    first = (c == first_r);
    return 2;
  }
  return 0;
}

// One axis of the CPML band update at one node: ψ on both faces (update_ψ!),
// dψ, the ξ recursion and the damping term (update_p! band branch).
// ψ entry q sits at psi_base + q*stride, ξ entry q-1 at xi_base + (q-1)*stride.
// pm, pc, pp: pressure at c-1, c, c+1 along the axis; d2: that axis's second
// difference; f: fact at the node.
template <typename T>
__device__ __forceinline__ void band_axis(const BandSide<T>& B, int q, bool first, T pm, T pc,
                                          T pp, T d2, T f, T inv_d, int64_t psi_base,
                                          int64_t xi_base, int64_t stride, T& damp) {
  const T ps_q_old = B.psi_old[psi_base + (int64_t)q * stride];
  const T ps_m_old = B.psi_old[psi_base + (int64_t)(q - 1) * stride];
  T* xp = B.xi + xi_base + (int64_t)(q - 1) * stride;
  T sq, sm, xn;
  cpml_axis(band_coef(B, q), ps_q_old, ps_m_old, *xp, pm, pc, pp, d2, f, inv_d, sq, sm, xn, damp);
  B.psi_new[psi_base + (int64_t)q * stride] = sq;
  if (first) B.psi_new[psi_base + (int64_t)(q - 1) * stride] = sm;
  *xp = xn;
}

// Sources then receivers of one node, for the thread that owns its value v.
template <typename T>
__device__ __forceinline__ T node_io(const Io<T>& io, int it, int sgrp, int rgrp, T v) {
  if (sgrp >= 0) {
    const T* row = io.stf + (int64_t)it * io.nsrc;
    for (int e = io.src_off[sgrp]; e < io.src_off[sgrp + 1]; ++e) v += row[io.src_ids[e]];
  }
  if (rgrp >= 0) {
    T* row = io.traces + (int64_t)it * io.nrec;
    for (int e = io.rec_off[rgrp]; e < io.rec_off[rgrp + 1]; ++e) row[io.rec_ids[e]] = v;
  }
  return v;
}

// Rim nodes of the step (block 0 only): pnew[rim] += sources, then sample.
template <typename T>
__device__ __forceinline__ void rim_io(const Io<T>& io, T* pnew, int it, int t, int nt) {
  for (int e = t; e < io.nrim; e += nt) {
    const IoRim r = io.rim[e];
    pnew[r.node] = node_io(io, it, r.sgrp, r.rgrp, pnew[r.node]);
  }
}
template <typename T>
__device__ __forceinline__ void rim_io(const Io<T>& io, T* pnew, int it) {
  rim_io(io, pnew, it, (int)(threadIdx.x + blockDim.x * threadIdx.y),
         (int)(blockDim.x * blockDim.y));
}

// ---------------------------------------------------------------------------
// TMA / mbarrier primitives (sm_90+ PTX, used here on sm_100a).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// One try_wait with a suspend-time hint: the warp sleeps in hardware until the
// phase completes or about `ns` nanoseconds pass, instead of spinning.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
// Bounded wait on a phase: at most ~4 s (4096 x 1 ms), or until another thread
// of the block has raised `abort`. False when it gives up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  for (int n = 0; n < 4096; ++n) {
    if (mbar_try_wait(bar, parity, 1000000u)) return true;
    if (*abort) return false;
  }
  return false;
}
// 3D tiled TMA load of one box into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// 2D tiled TMA load of one box into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

// Geometry of the 3D step kernel for element type T and TY thread rows:
// a block of 32 x TY threads owns a 64 x 2TY tile of (x, y) nodes; thread
// (tx, ty) owns the 2 x 2 nodes x0 + 2tx + {0,1}, y0 + 2ty + {0,1}. One
// pipeline stage holds, for one z plane, the pcur box (64 + 2A) x (2TY + 2)
// around the tile (x apron A keeps the box origin 16-byte aligned; the y ring
// is one row) and the pold and fact boxes 64 x 2TY.
template <typename T, int TY>
struct Tile3 {
  static constexpr int TX = 64;
  static constexpr int RY = 2 * TY;
  static constexpr int A = 16 / (int)sizeof(T);
  static constexpr int PW = TX + 2 * A;
  static constexpr int PC_BYTES = PW * (RY + 2) * (int)sizeof(T);
  static constexpr int PC_PAD = (PC_BYTES + 127) / 128 * 128;
  static constexpr int IN_BYTES = TX * RY * (int)sizeof(T);
  static constexpr int BYTES = PC_PAD + 2 * IN_BYTES;
};

// ---------------------------------------------------------------------------
// 3D core step: the nodes of P.core, which lie outside every active CPML
// band, so no band state is touched. Grid: x tiles of 64 nodes from P.core_x,
// y tiles of 2TY rows from core.y0, z chunks of `zchunk` planes from core.z0.
// One elected thread streams the planes of the block's chunk through S
// shared-memory stages with cp.async.bulk.tensor, each stage with a "full"
// mbarrier (TMA bytes) and an "empty" mbarrier (one arrival per warp once the
// warp is done with the stage). Plane k is computed from the stages of planes
// k-1, k, k+1; loads run up to S-3 planes ahead and warps may drift apart by
// as much, with no block-wide barrier in the loop. Each thread owns 2 x 2
// nodes: an x pair read and written as one vector, in two rows.
template <typename T, int TY, int S>
__global__ void __launch_bounds__(32 * TY) step3d_core(const __grid_constant__ CUtensorMap mc,
                                                       const __grid_constant__ CUtensorMap mo,
                                                       const __grid_constant__ CUtensorMap mf,
                                                       StepParams<T> P) {
  using L = Tile3<T, TY>;
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * L::BYTES);
  uint64_t* empty = full + S;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + S);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  // blocks are numbered z chunk fastest, so the chunks of one column tile run
  // together and the planes they share come from L2
  const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (blk == 0 && P.do_rim && P.io.nrim > 0) rim_io(P.io, P.pnew, P.it);
  const Box C = P.core;
  const int gz = gridDim.z, gx = gridDim.x;
  const int bz = blk % gz, bx = (blk / gz) % gx, by = blk / (gz * gx);
  const int x0 = P.core_x + bx * L::TX, y0 = C.y0 + by * L::RY;
  const int k0 = C.z0 + bz * P.zchunk;
  int k1 = k0 + P.zchunk;
  if (k1 > C.z1 + 1) k1 = C.z1 + 1;
  if (k0 >= k1) return;  // block-uniform
  const int nplanes = k1 - k0 + 2;  // pcur planes k0-1 .. k1

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TY);
    }
    *abort = 0;
    fence_mbar_init();
  }
  __syncthreads();
  // use u loads plane m = k0-1+u into stage u % S; pold/fact only for m in [k0, k1)
  auto issue = [&](int u) {
    const int s = u % S, m = k0 - 1 + u;
    unsigned char* st = smem + s * L::BYTES;
    const bool inner = m >= k0 && m < k1;
    mbar_expect_tx(&full[s], L::PC_BYTES + (inner ? 2 * L::IN_BYTES : 0));
    tma_load_3d(st, &mc, &full[s], x0 - L::A, y0 - 1, m);
    if (inner) {
      tma_load_3d(st + L::PC_PAD, &mo, &full[s], x0, y0, m);
      tma_load_3d(st + L::PC_PAD + L::IN_BYTES, &mf, &full[s], x0, y0, m);
    }
  };
  if (tid == 0)
    for (int u = 0; u < S && u < nplanes; ++u) issue(u);

  // the thread's 2 x 2 nodes
  const int xa = x0 + 2 * tx, j0 = y0 + 2 * ty;
  const bool vx0 = xa >= C.x0 && xa <= C.x1, vx1 = xa + 1 >= C.x0 && xa + 1 <= C.x1;
  const bool vy0 = j0 <= C.y1, vy1 = j0 + 1 <= C.y1;
  const bool any = (vx0 || vx1) && vy0;
  const bool all4 = vx0 && vx1 && vy0 && vy1;
  const int64_t px = P.px, plane = px * P.ny;
  int64_t o = (int64_t)xa + px * j0 + plane * k0;  // pitched offset of node (xa, j0, k)
  int ioe = P.io.blk_off[blk];
  const int ioe1 = P.io.blk_off[blk + 1];
  const int c0 = (2 * ty + 1) * L::PW + 2 * tx + L::A;  // pcur stage index of (xa, j0)
  const int i0 = 2 * ty * L::TX + 2 * tx;               // pold/fact stage index of (xa, j0)
  const T ix2 = P.inv_d2[0], iy2 = P.inv_d2[1], iz2 = P.inv_d2[2];

  bool ok = mbar_wait(&full[0], 0, abort) && mbar_wait(&full[1 % S], (1 / S) & 1, abort);
  int uc = 1;  // use index of the current plane
  for (int k = k0; k < k1; ++k, ++uc, o += plane) {
    ok = ok && mbar_wait(&full[(uc + 1) % S], ((uc + 1) / S) & 1, abort);
    if (!ok) break;
    const T* cm = reinterpret_cast<const T*>(smem + ((uc - 1) % S) * L::BYTES);
    const T* cc = reinterpret_cast<const T*>(smem + (uc % S) * L::BYTES);
    const T* cp = reinterpret_cast<const T*>(smem + ((uc + 1) % S) * L::BYTES);
    const T* oo = reinterpret_cast<const T*>(smem + (uc % S) * L::BYTES + L::PC_PAD);
    const T* ff = oo + L::TX * L::RY;
    // rows j0 and j0+1: centre pairs, x apron scalars, y and z neighbours,
    // pold and fact
    const V2 c_0 = *reinterpret_cast<const V2*>(cc + c0);
    const V2 c_1 = *reinterpret_cast<const V2*>(cc + c0 + L::PW);
    const T xm0 = cc[c0 - 1], xp0 = cc[c0 + 2], xm1 = cc[c0 + L::PW - 1], xp1 = cc[c0 + L::PW + 2];
    const V2 ym = *reinterpret_cast<const V2*>(cc + c0 - L::PW);
    const V2 yp = *reinterpret_cast<const V2*>(cc + c0 + 2 * L::PW);
    const V2 zm0 = *reinterpret_cast<const V2*>(cm + c0);
    const V2 zm1 = *reinterpret_cast<const V2*>(cm + c0 + L::PW);
    const V2 zp0 = *reinterpret_cast<const V2*>(cp + c0);
    const V2 zp1 = *reinterpret_cast<const V2*>(cp + c0 + L::PW);
    const V2 po0 = *reinterpret_cast<const V2*>(oo + i0);
    const V2 po1 = *reinterpret_cast<const V2*>(oo + i0 + L::TX);
    const V2 f_0 = *reinterpret_cast<const V2*>(ff + i0);
    const V2 f_1 = *reinterpret_cast<const V2*>(ff + i0 + L::TX);
    // node (row, x): 2 pcur - pold + fact * (d2x + d2y + d2z)
    T v00 = leapfrog3d(c_0.x, po0.x, f_0.x, second_diff(xm0, c_0.x, c_0.y, ix2),
                       second_diff(ym.x, c_0.x, c_1.x, iy2), second_diff(zm0.x, c_0.x, zp0.x, iz2));
    T v01 = leapfrog3d(c_0.y, po0.y, f_0.y, second_diff(c_0.x, c_0.y, xp0, ix2),
                       second_diff(ym.y, c_0.y, c_1.y, iy2), second_diff(zm0.y, c_0.y, zp0.y, iz2));
    T v10 = leapfrog3d(c_1.x, po1.x, f_1.x, second_diff(xm1, c_1.x, c_1.y, ix2),
                       second_diff(c_0.x, c_1.x, yp.x, iy2), second_diff(zm1.x, c_1.x, zp1.x, iz2));
    T v11 = leapfrog3d(c_1.y, po1.y, f_1.y, second_diff(c_1.x, c_1.y, xp1, ix2),
                       second_diff(c_0.y, c_1.y, yp.y, iy2), second_diff(zm1.y, c_1.y, zp1.y, iz2));
    // sources and receivers of this plane (block-uniform walk, rarely taken)
    for (; ioe < ioe1; ++ioe) {
      const int4 en = P.io.ent[ioe];
      if (en.y != k) break;
      const int lx = en.x & (L::TX - 1), ly = en.x / L::TX;
      if ((lx >> 1) == tx && (ly >> 1) == ty) {
        const int sub = ((ly & 1) << 1) | (lx & 1);
        if (sub == 0) v00 = node_io(P.io, P.it, en.z, en.w, v00);
        if (sub == 1) v01 = node_io(P.io, P.it, en.z, en.w, v01);
        if (sub == 2) v10 = node_io(P.io, P.it, en.z, en.w, v10);
        if (sub == 3) v11 = node_io(P.io, P.it, en.z, en.w, v11);
      }
    }
    // this warp is done with stage uc-1; the producer may refill it
    __syncwarp();
    if (tx == 0) mbar_arrive(&empty[(uc - 1) % S]);
    if (all4) {
      *reinterpret_cast<V2*>(P.pnew + o) = V2{v00, v01};
      *reinterpret_cast<V2*>(P.pnew + o + px) = V2{v10, v11};
    } else if (any) {
      if (vx0) P.pnew[o] = v00;
      if (vx1) P.pnew[o + 1] = v01;
      if (vy1 && vx0) P.pnew[o + px] = v10;
      if (vy1 && vx1) P.pnew[o + px + 1] = v11;
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
    // a wait ran out: record it, stop the block, and let the producer drain
    // the loads it still has in flight before the block's memory goes away
    *abort = 1;
    atomicExch(P.err, 1);
    if (tid == 0) {
      const int issued = nplanes < uc - 1 + S ? nplanes : uc - 1 + S;
      for (int u = uc; u < issued; ++u) {
        for (int n = 0; n < 64; ++n)
          if (mbar_try_wait(&full[u % S], (u / S) & 1, 1000000u)) break;
      }
    }
  }
}

// CPML update of one band axis at one node whose ψ entry q sits at element
// `pq` of the side's arrays (ψ[q-1] at pq - dq) and ξ entry q-1 at `xq`;
// c holds the entry's coefficients.
template <typename T, typename I>
__device__ __forceinline__ void band_apply(const BandSide<T>& B, const BandCoef<T>& c, bool first,
                                           I pq, I dq, I xq, T psq, T psm, T xo, T pm, T pc,
                                           T pp, T d2, T f, T inv, T& damp) {
  T sq, sm, xn;
  cpml_axis(c, psq, psm, xo, pm, pc, pp, d2, f, inv, sq, sm, xn, damp);
  B.psi_new[pq] = sq;
  if (first) B.psi_new[pq - dq] = sm;
  B.xi[xq] = xn;
}

// ---------------------------------------------------------------------------
// 3D band step: the interior nodes outside P.core (the CPML bands), in the
// boxes P.box[0..nbox). The (x, y) columns of a box are numbered row by row,
// l = (i - x0) + W (j - y0) with W the box width, so the 20-node-wide x slabs
// waste no thread slots; a block of BAND_NT threads owns BAND_NT consecutive
// columns and streams a chunk of P.shell_zchunk planes of them, keeping each
// column's z neighbours in registers.
//
// Box.kind says which bands the nodes of a box lie in, and the block body is
// compiled per kind:
//   1  an x slab: every node lies in the x band of the slab's side;
//   3  a y slab: every node lies in the y band of the slab's side, the
//      columns at its x ends in an x band too;
//   7  a z slab: every node lies in the z band of the slab's side, the
//      columns at its x and y edges in x and y bands too;
//   15 a grid without a core: any band anywhere.
// The right side's ψ, ξ and coefficient arrays of an axis follow the left
// side's at fixed offsets (P.psi_side, P.xi_side; halo + 1 and halo
// coefficients), so every band access is the left side's base pointer plus
// an offset with the side folded in, and no pointer is selected per thread.
// x and y entries are fixed along a column (offsets and, in their own slab,
// coefficients held in registers); in a z slab ψ[q] of node (i, j, k) sits at
// the node's own field offset less a constant. Integer offsets are of type
// I: int32 when every field fits, else int64. Along z the new ψ on a node's
// lower face is the value the column computed on the previous plane's upper
// face (the same operations on the same operands), so it is carried instead
// of recomputed.
constexpr int BAND_NT = 128;

// Blocks of BAND_NT threads per SM the band kernel is compiled for (its
// register budget: 65536 / (BAND_NT * blocks) per thread).
template <typename T>
struct BandOcc {
  static constexpr int blocks = (sizeof(T) == 4 ? 1024 : 512) / BAND_NT;
};

// Coefficients of entry q from the left side's arrays L: hq = half-grid index
// of ψ[q] (q, or q + halo + 1 on the right), g = on-grid index of q - 1
// (q - 1, or q - 1 + halo on the right).
template <typename T>
__device__ __forceinline__ BandCoef<T> coef_at(const BandSide<T>& L, int hq, int g) {
  return BandCoef<T>{__ldg(L.bKh + hq), __ldg(L.ah + hq), __ldg(L.bKh + hq - 1),
                     __ldg(L.ah + hq - 1), __ldg(L.bK + g), __ldg(L.a + g)};
}

// Band state of one column along x or y: side (0 none), entry q, first
// flag; for the slab's own axis also the offsets of ψ[q] and ξ[q-1] at the
// current plane (side folded in) and the coefficients, held along the column.
// Columns that lie in an x or y band only at the edge of another slab
// recompute their offsets per plane, so the state they keep is small.
template <typename I>
struct ColBand {
  int s = 0, q = 0;
  bool first = false;
  I pq = 0, xq = 0;
};

template <typename T, typename I, int KIND>
__device__ __forceinline__ void band_body(const StepParams<T>& P, int blk, const Box& B, int r) {
  constexpr bool GEN = KIND == 15;
  constexpr bool XPRIM = KIND == 1, YPRIM = KIND == 3;  // the slab's own axis
  const int W = B.x1 - B.x0 + 1;
  const int ncol = W * (B.y1 - B.y0 + 1);
  const int ncb = (ncol + BAND_NT - 1) / BAND_NT;
  const int l = (r % ncb) * BAND_NT + (int)threadIdx.x;
  const int k0 = B.z0 + (r / ncb) * P.shell_zchunk;
  const int k1 = min(k0 + P.shell_zchunk, B.z1 + 1);
  const bool valid = l < ncol;
  const int i = B.x0 + (valid ? l % W : 0), j = B.y0 + (valid ? l / W : 0);
  const int halo = P.halo;
  const I px = (I)P.px, plane = (I)P.plane;
  const I col = (I)i + px * (I)j;
  I o = col + plane * (I)k0;
  int ioe = P.io.blk_off[blk];
  const int ioe1 = P.io.blk_off[blk + 1];
  const BandSide<T>&LX = P.band[0][0], &LY = P.band[1][0], &LZ = P.band[2][0];
  ColBand<I> X, Y;
  BandCoef<T> cx{}, cy{};
  if ((KIND & 1) && valid) {
    X.s = band_of(i, P.nx, halo, P.first_r[0], X.q, X.first);
    if (!XPRIM && X.s != 0 && !(X.s == 1 ? P.active[0][0] : P.active[0][1])) X.s = 0;
    if (XPRIM) {
      const bool R = X.s == 2;
      const I jk = (I)j + (I)P.ny * (I)k0;
      X.pq = (I)(halo + 1) * jk + (I)X.q + (R ? (I)P.psi_side[0] : (I)0);
      X.xq = (I)halo * jk + (I)(X.q - 1) + (R ? (I)P.xi_side[0] : (I)0);
      cx = coef_at(LX, X.q + (R ? halo + 1 : 0), X.q - 1 + (R ? halo : 0));
    }
  }
  if ((KIND & 2) && valid) {
    Y.s = band_of(j, P.ny, halo, P.first_r[1], Y.q, Y.first);
    if (!YPRIM && Y.s != 0 && !(Y.s == 1 ? P.active[1][0] : P.active[1][1])) Y.s = 0;
    if (YPRIM) {
      const bool R = Y.s == 2;
      Y.pq = (I)i + px * ((I)Y.q + (I)(halo + 1) * (I)k0) + (R ? (I)P.psi_side[1] : (I)0);
      Y.xq = (I)i + px * ((I)(Y.q - 1) + (I)halo * (I)k0) + (R ? (I)P.xi_side[1] : (I)0);
      cy = coef_at(LY, Y.q + (R ? halo + 1 : 0), Y.q - 1 + (R ? halo : 0));
    }
  }
  // z slab: ψ[q] of node (i, j, k) at o - zsp and ξ[q-1] at o - plane - zsx
  // (zs = plane * (k - q) less the side offset)
  I zsp = 0, zsx = 0;
  if (KIND == 7 && B.z0 != 1) {
    const I zs = plane * (I)(P.nz - halo - 2);
    zsp = zs - (I)P.psi_side[2];
    zsx = zs - (I)P.xi_side[2];
  }
  const T* __restrict__ pcur = P.pcur;
  T pm = 0, pc = 0, pp = 0;
  if (valid) {
    pm = __ldg(pcur + (o - plane));
    pc = __ldg(pcur + o);
  }
  T zsq = 0;  // new ψ on the upper z face of the previous plane's node
  for (int k = k0; k < k1; ++k, o += plane) {
    // z band of the plane (uniform over the block)
    int sz = 0, qz = 0;
    bool fz = false;
    if (KIND & 4) {
      sz = band_of(k, P.nz, halo, P.first_r[2], qz, fz);
      if (GEN && sz != 0 && !(sz == 1 ? P.active[2][0] : P.active[2][1])) sz = 0;
    }
    const bool zR = sz == 2;
    const bool zcarry = k > k0 && !fz;
    T v = 0;
    if (valid) {
      pp = __ldg(pcur + (o + plane));
      const T po = __ldg(P.pold + o), f = __ldg(P.fact + o);
      // offsets of this plane's x and y entries
      I xpq = X.pq, xxq = X.xq, ypq = Y.pq, yxq = Y.xq;
      if ((KIND & 1) && !XPRIM && X.s) {
        const bool R = X.s == 2;
        const I jk = (I)j + (I)P.ny * (I)k;
        xpq = (I)(halo + 1) * jk + (I)X.q + (R ? (I)P.psi_side[0] : (I)0);
        xxq = (I)halo * jk + (I)(X.q - 1) + (R ? (I)P.xi_side[0] : (I)0);
      }
      if ((KIND & 2) && !YPRIM && Y.s) {
        const bool R = Y.s == 2;
        ypq = (I)i + px * ((I)Y.q + (I)(halo + 1) * (I)k) + (R ? (I)P.psi_side[1] : (I)0);
        yxq = (I)i + px * ((I)(Y.q - 1) + (I)halo * (I)k) + (R ? (I)P.xi_side[1] : (I)0);
      }
      // band values of this plane, issued before the arithmetic
      T xq = 0, xmq = 0, xx = 0, yq = 0, ymq = 0, yx = 0, zq = 0, zmq = 0, zx = 0;
      if ((KIND & 1) && X.s) {
        xq = LX.psi_old[xpq];
        xmq = LX.psi_old[xpq - 1];
        xx = LX.xi[xxq];
      }
      if ((KIND & 2) && Y.s) {
        yq = LY.psi_old[ypq];
        ymq = LY.psi_old[ypq - px];
        yx = LY.xi[yxq];
      }
      I zp = o - zsp, zxo = o - plane - zsx;
      if (GEN) {
        zp = col + plane * (I)qz + (zR ? (I)P.psi_side[2] : (I)0);
        zxo = col + plane * (I)(qz - 1) + (zR ? (I)P.xi_side[2] : (I)0);
      }
      if ((KIND & 4) && sz) {
        zq = LZ.psi_old[zp];
        if (!zcarry) zmq = LZ.psi_old[zp - plane];
        zx = LZ.xi[zxo];
      }
      const T xm = __ldg(pcur + (o - 1)), xp = __ldg(pcur + (o + 1));
      const T ym = __ldg(pcur + (o - px)), yp = __ldg(pcur + (o + px));
      const T d2x = second_diff(xm, pc, xp, P.inv_d2[0]);
      const T d2y = second_diff(ym, pc, yp, P.inv_d2[1]);
      const T d2z = second_diff(pm, pc, pp, P.inv_d2[2]);
      v = leapfrog3d(pc, po, f, d2x, d2y, d2z);
      T damp = 0;
      if ((KIND & 1) && X.s) {
        const bool R = X.s == 2;
        band_apply(LX, XPRIM ? cx : coef_at(LX, X.q + (R ? halo + 1 : 0), X.q - 1 + (R ? halo : 0)),
                   X.first, xpq, (I)1, xxq, xq, xmq, xx, xm, pc, xp, d2x, f, P.inv_d[0], damp);
      }
      if ((KIND & 2) && Y.s) {
        const bool R = Y.s == 2;
        band_apply(LY, YPRIM ? cy : coef_at(LY, Y.q + (R ? halo + 1 : 0), Y.q - 1 + (R ? halo : 0)),
                   Y.first, ypq, px, yxq, yq, ymq, yx, ym, pc, yp, d2y, f, P.inv_d[1], damp);
      }
      if ((KIND & 4) && sz) {
        const T inv = P.inv_d[2];
        const int hq = qz + (zR ? halo + 1 : 0), g = qz - 1 + (zR ? halo : 0);
        const T sq = psi_face(__ldg(LZ.bKh + hq), __ldg(LZ.ah + hq), zq, pp - pc, inv);
        const T sm = zcarry ? zsq
                            : psi_face(__ldg(LZ.bKh + hq - 1), __ldg(LZ.ah + hq - 1), zmq,
                                       pc - pm, inv);
        T xn;
        cpml_tail(__ldg(LZ.bK + g), __ldg(LZ.a + g), sq, sm, zx, d2z, f, inv, xn, damp);
        LZ.psi_new[zp] = sq;
        if (fz) LZ.psi_new[zp - plane] = sm;
        LZ.xi[zxo] = xn;
        zsq = sq;
      }
      v += damp;
    }
    // sources and receivers of this plane (block-uniform walk)
    for (; ioe < ioe1; ++ioe) {
      const int4 en = P.io.ent[ioe];
      if (en.y != k) break;
      if (valid && en.x == (int)threadIdx.x) v = node_io(P.io, P.it, en.z, en.w, v);
    }
    if (valid) P.pnew[o] = v;
    pm = pc;
    pc = pp;
    if (XPRIM) {
      X.pq += (I)P.psi_dz[0];
      X.xq += (I)P.xi_dz[0];
    }
    if (YPRIM) {
      Y.pq += (I)P.psi_dz[1];
      Y.xq += (I)P.xi_dz[1];
    }
  }
}

template <typename T, typename I>
__global__ void __launch_bounds__(BAND_NT, BandOcc<T>::blocks) step3d_band(StepParams<T> P) {
  const int blk = (int)blockIdx.x;
  if (blk == 0 && P.do_rim && P.io.nrim > 0) rim_io(P.io, P.pnew, P.it);
  int b = 0;
  while (b + 1 < P.nbox && blk >= P.box_blk[b + 1]) ++b;
  const Box B = P.box[b];
  const int r = blk - P.box_blk[b];
  if (B.kind == 1)
    band_body<T, I, 1>(P, blk, B, r);
  else if (B.kind == 3)
    band_body<T, I, 3>(P, blk, B, r);
  else if (B.kind == 7)
    band_body<T, I, 7>(P, blk, B, r);
  else
    band_body<T, I, 15>(P, blk, B, r);
}

// ---------------------------------------------------------------------------
// 2D step: one thread per interior node (x tiles of 32 from x = 0, y tiles of
// 8 rows from y = 1); neighbours through L1.
template <typename T>
__global__ void __launch_bounds__(256) step2d(StepParams<T> P) {
  const int nx = P.nx, ny = P.ny, halo = P.halo;
  const int blk = blockIdx.x + gridDim.x * blockIdx.y;
  if (blk == 0 && P.do_rim && P.io.nrim > 0) rim_io(P.io, P.pnew, P.it);
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i < 1 || i > nx - 2 || j > ny - 2) return;
  const int64_t px = P.px;
  const int64_t o = (int64_t)i + px * j;
  const T* __restrict__ pcur = P.pcur;
  const T pc = __ldg(pcur + o);
  const T xm = __ldg(pcur + o - 1), xp = __ldg(pcur + o + 1);
  const T ym = __ldg(pcur + o - px), yp = __ldg(pcur + o + px);
  const T po = __ldg(P.pold + o), f = __ldg(P.fact + o);
  const T d2x = second_diff(xm, pc, xp, P.inv_d2[0]);
  const T d2y = second_diff(ym, pc, yp, P.inv_d2[1]);
  T damp = 0;
  int q;
  bool first;
  const int bx = band_of(i, nx, halo, P.first_r[0], q, first);
  if (bx != 0 && P.active[0][bx - 1])
    band_axis(P.band[0][bx - 1], q, first, xm, pc, xp, d2x, f, P.inv_d[0],
              (int64_t)(halo + 1) * j, (int64_t)halo * j, (int64_t)1, damp);
  const int by = band_of(j, ny, halo, P.first_r[1], q, first);
  if (by != 0 && P.active[1][by - 1])
    band_axis(P.band[1][by - 1], q, first, ym, pc, yp, d2y, f, P.inv_d[1], (int64_t)i,
              (int64_t)i, px, damp);
  T v = leapfrog2d(pc, po, f, d2x, d2y) + damp;
  const int local = threadIdx.x + 32 * threadIdx.y;
  for (int e = P.io.blk_off[blk]; e < P.io.blk_off[blk + 1]; ++e) {
    const int4 en = P.io.ent[e];
    if (en.x == local) v = node_io(P.io, P.it, en.z, en.w, v);
  }
  P.pnew[o] = v;
}

// ---------------------------------------------------------------------------
// Batched 2D shots. Every shot owns its fields, CPML state, traces and
// source/receiver lists; shots of one velocity model share fact. One launch
// advances every shot of the batch by one time step: a persistent grid walks
// the global list of 32 x (TY*R) tiles of all shots (tile t belongs to shot s
// when tile_start[s] <= t < tile_start[s+1]). Warp ty of a block owns a
// strip of R consecutive rows of the tile: each pressure row of the strip is
// read once (y neighbours are registers, x neighbours adjacent lanes), and
// the per-tile work (shot lookup, descriptor, source/receiver list bounds) is
// shared by R nodes per thread.
template <typename T>
struct ShotDesc {
  T* buf[3];               // rotated like the single-shot fields
  const T* fact;           // the model's fact (pitched)
  int64_t px;
  int32_t nx, ny, halo, gx;  // gx: x tiles of the shot
  T inv_d[2], inv_d2[2];
  T* psi[2][2][2];         // [axis][side][parity]
  BandSide<T> band[2][2];  // coefficients and ξ (ψ pointers filled per step)
  int32_t active[2][2];
  int32_t first_r[2];
  Io<T> io;                // per-tile lists of this shot; rim served by tile 0
};

template <typename T, int TY, int R>
__global__ void __launch_bounds__(32 * TY) step2d_batch(const ShotDesc<T>* __restrict__ shots,
                                                        const int32_t* __restrict__ tile_start,
                                                        int32_t nshots, int32_t ntiles,
                                                        int32_t it) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  int s = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    // tiles of a block increase, so the shot index only moves forward
    while (s + 1 < nshots && __ldg(tile_start + s + 1) <= t) ++s;
    const ShotDesc<T>& D = shots[s];
    const int local = t - __ldg(tile_start + s);
    const int nx = D.nx, ny = D.ny, halo = D.halo;
    T* pnew = D.buf[(it + 2) % 3];
    if (local == 0 && D.io.nrim > 0) {
      Io<T> io = D.io;
      rim_io(io, pnew, it);
    }
    const int x0 = (local % D.gx) * 32;
    const int i = x0 + tx;
    const int j0 = 1 + (local / D.gx) * (TY * R) + ty * R;
    if (j0 > ny - 2) continue;  // whole warp
    const int64_t px = D.px;
    const T* __restrict__ pcur = D.buf[(it + 1) % 3];
    const T* __restrict__ pold = D.buf[it % 3];
    const int e0 = D.io.blk_off[local], e1 = D.io.blk_off[local + 1];
    // Load phase, free of branches so that all loads of the strip are in
    // flight together: R + 2 pressure rows, R rows of the old field and of
    // fact. Rows past the grid are clamped to the last rows (their values are
    // never stored); x neighbours come from the adjacent lanes, and lanes 0
    // and 31 also load the node just outside the 32-node strip (clamped into
    // [0, nx-1]; a clamped value is never used).
    T pcv[R + 2], pov[R], fv[R], xe[R];
    const int ie = tx == 0 ? max(x0 - 1, 0) : min(x0 + 32, nx - 1);
    const bool edge = tx == 0 || tx == 31;
#pragma unroll
    for (int r = 0; r < R + 2; ++r) pcv[r] = __ldg(pcur + i + px * min(j0 - 1 + r, ny - 1));
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t row = px * min(j0 + r, ny - 2);
      pov[r] = __ldg(pold + i + row);
      fv[r] = __ldg(D.fact + i + row);
      xe[r] = edge ? __ldg(pcur + ie + row) : T(0);
    }
    const bool live = i >= 1 && i <= nx - 2;
    // Fast path: the warp's 32 x R strip meets no active CPML band and holds
    // no source or receiver.
    const bool xband = (D.active[0][0] && x0 <= halo) ||
                       (D.active[0][1] && x0 + 31 >= nx - halo - 1);
    const bool yband = (D.active[1][0] && j0 <= halo) ||
                       (D.active[1][1] && j0 + R - 1 >= ny - halo - 1);
    if (!xband && !yband && e0 == e1) {
      const T cx = D.inv_d2[0], cy = D.inv_d2[1];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const T pc = pcv[r + 1];
        T xm = __shfl_up_sync(0xffffffffu, pc, 1), xp = __shfl_down_sync(0xffffffffu, pc, 1);
        if (tx == 0) xm = xe[r];
        if (tx == 31) xp = xe[r];
        const T d2x = second_diff(xm, pc, xp, cx);
        const T d2y = second_diff(pcv[r], pc, pcv[r + 2], cy);
        if (live && j0 + r <= ny - 2) pnew[i + px * (j0 + r)] = leapfrog2d(pc, pov[r], fv[r], d2x, d2y);
      }
      continue;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      const T ym = pcv[r], pc = pcv[r + 1], yp = pcv[r + 2];
      T xm = __shfl_up_sync(0xffffffffu, pc, 1), xp = __shfl_down_sync(0xffffffffu, pc, 1);
      if (tx == 0) xm = xe[r];
      if (tx == 31) xp = xe[r];
      if (!live || j > ny - 2) continue;
      const int64_t o = (int64_t)i + px * j;
      const T po = pov[r], f = fv[r];
      const T d2x = second_diff(xm, pc, xp, D.inv_d2[0]);
      const T d2y = second_diff(ym, pc, yp, D.inv_d2[1]);
      T v = leapfrog2d(pc, po, f, d2x, d2y);
      int q;
      bool first;
      const int bx = band_of(i, nx, halo, D.first_r[0], q, first);
      const int by = band_of(j, ny, halo, D.first_r[1], q, first);
      if ((bx != 0 && D.active[0][bx - 1]) || (by != 0 && D.active[1][by - 1])) {
        T damp = 0;
        if (bx != 0 && D.active[0][bx - 1]) {
          BandSide<T> B = D.band[0][bx - 1];
          B.psi_old = D.psi[0][bx - 1][it & 1];
          B.psi_new = D.psi[0][bx - 1][(it + 1) & 1];
          band_of(i, nx, halo, D.first_r[0], q, first);
          band_axis(B, q, first, xm, pc, xp, d2x, f, D.inv_d[0], (int64_t)(halo + 1) * j,
                    (int64_t)halo * j, (int64_t)1, damp);
        }
        if (by != 0 && D.active[1][by - 1]) {
          BandSide<T> B = D.band[1][by - 1];
          B.psi_old = D.psi[1][by - 1][it & 1];
          B.psi_new = D.psi[1][by - 1][(it + 1) & 1];
          band_of(j, ny, halo, D.first_r[1], q, first);
          band_axis(B, q, first, ym, pc, yp, d2y, f, D.inv_d[1], (int64_t)i, (int64_t)i, px,
                    damp);
        }
        v += damp;
      }
      const int lidx = tx + 32 * (ty * R + r);
      for (int e = e0; e < e1; ++e) {
        const int4 en = D.io.ent[e];
        if (en.x == lidx) v = node_io(D.io, it, en.z, en.w, v);
      }
      pnew[o] = v;
    }
  }
}

// Tensor maps of one batched shot (in global memory, 64-byte aligned): for
// each rotating field buffer a map with the pcur box ((64 + 2A) x (RY + 2))
// and one with the inner box (64 x RY), and the map of its model's fact.
struct ShotMaps {
  CUtensorMap c[3];
  CUtensorMap o[3];
  CUtensorMap f;
};

// Batched 2D shots, TMA-fed: the same persistent walk of the global tile list
// as step2d_batch, with tiles of 64 x (4 RR) nodes. A block has CW = 4
// consumer warps and one producer warp. The producer's lane 0 streams the
// block's tiles through S shared-memory stages, up to S tiles ahead: for each
// tile it writes a header (shot, tile origin, the shot's sizes, its output
// field, whether the tile meets a CPML band, the tile's source/receiver list
// bounds) and issues cp.async.bulk.tensor loads of the pcur box with a
// one-node ring and of the pold and fact boxes from the shot's tensor maps.
// Each stage has a "full" mbarrier (the header arrival and the TMA bytes) and
// an "empty" one (one arrival per consumer warp once its values are in
// registers). Consumer lane l of warp w owns nodes x0 + 2l, x0 + 2l + 1 of
// rows y0 + w RR .. y0 + w RR + RR - 1. Band nodes and sources/receivers take
// the same per-node code as step2d_batch, so every shot computes bitwise
// what its single-shot run computes. Waits are bounded: a wait that runs out
// sets *err and ends the block.
constexpr int BATCH_CW = 4;  // consumer warps of the TMA batched kernel

template <typename T>
struct TileHdr {
  int32_t shot, local, x0, y0;
  int32_t nx, ny, band, e0;
  int32_t e1, rim;
  int64_t px;
  T* pnew;
  T ix2, iy2;
};

template <typename T, int RR>
struct BatchTile {
  static constexpr int TX = 64, RY = BATCH_CW * RR;
  static constexpr int A = 16 / (int)sizeof(T);
  static constexpr int PW = TX + 2 * A;
  static constexpr int PC_BYTES = PW * (RY + 2) * (int)sizeof(T);
  static constexpr int PC_PAD = (PC_BYTES + 127) / 128 * 128;
  static constexpr int IN_BYTES = TX * RY * (int)sizeof(T);
  static constexpr int HDR = 128;  // header slot (TileHdr, padded)
  static constexpr int BYTES = PC_PAD + 2 * IN_BYTES + HDR;
};

template <typename T, int RR, int S>
__global__ void __launch_bounds__(32 * (BATCH_CW + 1))
    step2d_batch_tma(const ShotDesc<T>* __restrict__ shots, const ShotMaps* __restrict__ maps,
                     const int32_t* __restrict__ tile_start, int32_t nshots, int32_t ntiles,
                     int32_t it, int32_t* err) {
  using L = BatchTile<T, RR>;
  using V2 = typename Vec2<T>::type;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * L::BYTES);
  uint64_t* empty = full + S;
  volatile int* abort = reinterpret_cast<volatile int*>(empty + S);
  const int lane = threadIdx.x, w = threadIdx.y;
  const int nb = (int)gridDim.x, b0 = (int)blockIdx.x;
  const int nu = b0 < ntiles ? (ntiles - 1 - b0) / nb + 1 : 0;  // tiles of this block
  if (nu == 0) return;  // block-uniform
  if (w == 0 && lane == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], BATCH_CW);
    }
    *abort = 0;
    fence_mbar_init();
  }
  __syncthreads();
  const int pb = (it + 1) % 3, ob = it % 3, wb = (it + 2) % 3;

  if (w == BATCH_CW) {
    // ---- producer ----------------------------------------------------------
    if (lane != 0) return;
    int ps = 0;  // shot cursor (tiles of a block increase)
    int u = 0;
    bool ok = true;
    for (; u < nu; ++u) {
      const int s = u % S;
      if (u >= S && !mbar_wait(&empty[s], ((u / S) + 1) & 1, abort)) {
        ok = false;
        break;
      }
      const int t = b0 + u * nb;
      while (ps + 1 < nshots && __ldg(tile_start + ps + 1) <= t) ++ps;
      const ShotDesc<T>& D = shots[ps];
      const int local = t - __ldg(tile_start + ps);
      const int x0 = (local % D.gx) * L::TX, y0 = 1 + (local / D.gx) * L::RY;
      const int nx = D.nx, ny = D.ny, halo = D.halo;
      unsigned char* st = smem + s * L::BYTES;
      TileHdr<T>* h = reinterpret_cast<TileHdr<T>*>(st + L::PC_PAD + 2 * L::IN_BYTES);
      h->shot = ps;
      h->local = local;
      h->x0 = x0;
      h->y0 = y0;
      h->nx = nx;
      h->ny = ny;
      h->band = ((D.active[0][0] && x0 <= halo) || (D.active[0][1] && x0 + L::TX - 1 >= nx - halo - 1) ||
                 (D.active[1][0] && y0 <= halo) || (D.active[1][1] && y0 + L::RY - 1 >= ny - halo - 1))
                    ? 1 : 0;
      h->e0 = D.io.blk_off[local];
      h->e1 = D.io.blk_off[local + 1];
      h->rim = (local == 0 && D.io.nrim > 0) ? 1 : 0;
      h->px = D.px;
      h->pnew = D.buf[wb];
      h->ix2 = D.inv_d2[0];
      h->iy2 = D.inv_d2[1];
      const ShotMaps* M = maps + ps;
      // the arrive that follows releases the header writes with the stage
      mbar_expect_tx(&full[s], L::PC_BYTES + 2 * L::IN_BYTES);
      tma_load_2d(st, &M->c[pb], &full[s], x0 - L::A, y0 - 1);
      tma_load_2d(st + L::PC_PAD, &M->o[ob], &full[s], x0, y0);
      tma_load_2d(st + L::PC_PAD + L::IN_BYTES, &M->f, &full[s], x0, y0);
    }
    if (!ok) {
      // a wait ran out: record it and let the loads in flight land first
      *abort = 1;
      atomicExch(err, 1);
      for (int v = u - S > 0 ? u - S : 0; v < u; ++v)
        for (int n = 0; n < 64; ++n)
          if (mbar_try_wait(&full[v % S], (v / S) & 1, 1000000u)) break;
    }
    return;
  }

  // ---- consumers -----------------------------------------------------------
  const int ct = lane + 32 * w;  // consumer thread index
  const int cbase = (w * RR + 1) * L::PW + 2 * lane + L::A;  // pcur stage index of row 0
  const int ibase = w * RR * L::TX + 2 * lane;               // pold/fact stage index of row 0
  for (int u = 0; u < nu; ++u) {
    const int s = u % S;
    if (!mbar_wait(&full[s], (u / S) & 1, abort)) {
      // a wait ran out: record it, stop, and let the loads that may still be
      // in flight (at most S uses from here) land before the block ends
      *abort = 1;
      atomicExch(err, 1);
      if (ct == 0)
        for (int v = u; v < nu && v < u + S; ++v)
          for (int n = 0; n < 64; ++n)
            if (mbar_try_wait(&full[v % S], (v / S) & 1, 1000000u)) break;
      return;
    }
    const unsigned char* st = smem + s * L::BYTES;
    const TileHdr<T> h = *reinterpret_cast<const TileHdr<T>*>(st + L::PC_PAD + 2 * L::IN_BYTES);
    const T* cc = reinterpret_cast<const T*>(st);
    const T* oo = reinterpret_cast<const T*>(st + L::PC_PAD);
    const T* ff = oo + L::TX * L::RY;
    // rows -1 .. RR of the thread's column pair, its x aprons, pold and fact
    V2 pcv[RR + 2];
    T xmv[RR], xpv[RR];
    V2 pov[RR], fv[RR];
#pragma unroll
    for (int r = 0; r < RR + 2; ++r)
      pcv[r] = *reinterpret_cast<const V2*>(cc + cbase + (r - 1) * L::PW);
#pragma unroll
    for (int r = 0; r < RR; ++r) {
      xmv[r] = cc[cbase + r * L::PW - 1];
      xpv[r] = cc[cbase + r * L::PW + 2];
      pov[r] = *reinterpret_cast<const V2*>(oo + ibase + r * L::TX);
      fv[r] = *reinterpret_cast<const V2*>(ff + ibase + r * L::TX);
    }
    // this warp's values are in registers: the producer may refill the stage
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (h.rim) {
      const Io<T> io = shots[h.shot].io;
      rim_io(io, h.pnew, it, ct, 32 * BATCH_CW);
    }
    const int xa = h.x0 + 2 * lane, ja = h.y0 + w * RR;
    T v[RR][2], d2x[RR][2], d2y[RR][2];
#pragma unroll
    for (int r = 0; r < RR; ++r) {
      const T pc0 = pcv[r + 1].x, pc1 = pcv[r + 1].y;
      d2x[r][0] = second_diff(xmv[r], pc0, pc1, h.ix2);
      d2x[r][1] = second_diff(pc0, pc1, xpv[r], h.ix2);
      d2y[r][0] = second_diff(pcv[r].x, pc0, pcv[r + 2].x, h.iy2);
      d2y[r][1] = second_diff(pcv[r].y, pc1, pcv[r + 2].y, h.iy2);
      v[r][0] = leapfrog2d(pc0, pov[r].x, fv[r].x, d2x[r][0], d2y[r][0]);
      v[r][1] = leapfrog2d(pc1, pov[r].y, fv[r].y, d2x[r][1], d2y[r][1]);
    }
    if (h.band) {
      const ShotDesc<T>& D = shots[h.shot];
      const int nx = h.nx, ny = h.ny, halo = D.halo;
#pragma unroll
      for (int r = 0; r < RR; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int i = xa + c, j = ja + r;
          if (i < 1 || i > nx - 2 || j > ny - 2) continue;
          int q;
          bool first;
          const int bx = band_of(i, nx, halo, D.first_r[0], q, first);
          const int by = band_of(j, ny, halo, D.first_r[1], q, first);
          const bool ax = bx != 0 && D.active[0][bx - 1], ay = by != 0 && D.active[1][by - 1];
          if (!ax && !ay) continue;
          const T pc = c ? pcv[r + 1].y : pcv[r + 1].x;
          const T xm = c ? pcv[r + 1].x : xmv[r], xp = c ? xpv[r] : pcv[r + 1].y;
          const T ym = c ? pcv[r].y : pcv[r].x, yp = c ? pcv[r + 2].y : pcv[r + 2].x;
          const T f = c ? fv[r].y : fv[r].x;
          T damp = 0;
          if (ax) {
            BandSide<T> B = D.band[0][bx - 1];
            B.psi_old = D.psi[0][bx - 1][it & 1];
            B.psi_new = D.psi[0][bx - 1][(it + 1) & 1];
            band_of(i, nx, halo, D.first_r[0], q, first);
            band_axis(B, q, first, xm, pc, xp, d2x[r][c], f, D.inv_d[0], (int64_t)(halo + 1) * j,
                      (int64_t)halo * j, (int64_t)1, damp);
          }
          if (ay) {
            BandSide<T> B = D.band[1][by - 1];
            B.psi_old = D.psi[1][by - 1][it & 1];
            B.psi_new = D.psi[1][by - 1][(it + 1) & 1];
            band_of(j, ny, halo, D.first_r[1], q, first);
            band_axis(B, q, first, ym, pc, yp, d2y[r][c], f, D.inv_d[1], (int64_t)i, (int64_t)i,
                      h.px, damp);
          }
          v[r][c] += damp;
        }
    }
    // sources and receivers of the tile (lists are per tile, rarely non-empty)
    if (h.e0 < h.e1) {
      const Io<T>& io = shots[h.shot].io;
      for (int e = h.e0; e < h.e1; ++e) {
        const int4 en = io.ent[e];
        const int lx = en.x % L::TX - 2 * lane, ly = en.x / L::TX - w * RR;
        if (lx >= 0 && lx < 2 && ly >= 0 && ly < RR) {
#pragma unroll
          for (int r = 0; r < RR; ++r)
            if (ly == r) {
              if (lx == 0) v[r][0] = node_io(io, it, en.z, en.w, v[r][0]);
              else v[r][1] = node_io(io, it, en.z, en.w, v[r][1]);
            }
        }
      }
    }
    const bool vx0 = xa >= 1 && xa <= h.nx - 2, vx1 = xa + 1 <= h.nx - 2;
#pragma unroll
    for (int r = 0; r < RR; ++r) {
      const int j = ja + r;
      if (j > h.ny - 2) break;
      T* row = h.pnew + h.px * j + xa;
      if (vx0 && vx1)
        *reinterpret_cast<V2*>(row) = V2{v[r][0], v[r][1]};
      else {
        if (vx0) row[0] = v[r][0];
        if (vx1) row[1] = v[r][1];
      }
    }
  }
}

// fact = (dt^2) * (vel^2) in FP64, rounded once to T (acoustic_3D_xPU.jl:242);
// dense column-major vel in, pitched fact out.
template <typename T>
__global__ void make_fact(const double* __restrict__ vel, T* __restrict__ fact, double dt2,
                          int64_t n, int64_t nx, int64_t px) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const double v = vel[c];
    fact[c % nx + px * (c / nx)] = (T)(dt2 * (v * v));
  }
}

// pitched T field -> dense column-major double.
template <typename T>
__global__ void unpitch(const T* __restrict__ src, double* __restrict__ dst, int64_t n,
                        int64_t nx, int64_t px) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    dst[c] = (double)src[c % nx + px * (c / nx)];
}

// traces [nt][nrec] (T) -> (nt x nrec) column-major double.
template <typename T>
__global__ void traces_out(const T* __restrict__ src, double* __restrict__ dst, int64_t nt,
                           int64_t nrec) {
  __shared__ T tile[32][33];
  const int64_t t0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
  for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
    const int64_t t = t0 + yy, r = r0 + threadIdx.x;
    if (t < nt && r < nrec) tile[yy][threadIdx.x] = src[t * nrec + r];
  }
  __syncthreads();
  for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
    const int64_t r = r0 + yy, t = t0 + threadIdx.x;
    if (t < nt && r < nrec) dst[r * nt + t] = (double)tile[threadIdx.x][yy];
  }
}

}  // namespace awc
