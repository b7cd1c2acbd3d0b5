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
// Memory layout in HBM (x fastest, like the reference's column-major arrays):
//   p fields, fact   pitched: node (i, j, k) at i + px*(j + ny*k), px = nx
//                    rounded up to 32 elements (128/256-byte rows, so every
//                    TMA stride and tile origin is 16-byte aligned)
//   ψ axis x  (halo+1, ny, nz)   ψ axis y (nx, halo+1, nz)   ψ axis z (nx, ny, halo+1)
//   ξ axis x  (halo,   ny, nz)   ξ axis y (nx, halo,   nz)   ξ axis z (nx, ny, halo)
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
//
// Tiles: a block owns x range [32 bx, 32 bx + 32) (nodes 0 and nx-1 are rim
// and not computed), y range [1 + BY by, 1 + BY (by+1)) and, in 3D, z planes
// [1 + zchunk bz, ...). Thread (tx, ty) owns node (32 bx + tx, 1 + BY by + ty).
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
// bucketed by the block that owns the node: {local thread index in the
// block, z plane (3D), source group, receiver group}; a group is an index
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

template <typename T>
struct StepParams {
  const T* pold;
  const T* pcur;
  T* pnew;
  const T* fact;
  int32_t nx, ny, nz, halo;
  int64_t px;              // row pitch of the fields (elements)
  T inv_d[3];
  T inv_d2[3];
  BandSide<T> band[3][2];  // [axis][left/right]
  int32_t active[3][2];    // side carries a non-trivial CPML recursion
  int32_t first_r[3];      // first node (0-based) of the right band per axis
  int32_t zchunk;          // planes per block along z (3D)
  int32_t it;              // 0-based time step index (row of stf/traces)
  int32_t* err;            // set to 1 when a bounded device wait runs out
  Io<T> io;
};

// ---------------------------------------------------------------------------
// CPML band arithmetic, split into the loads (issued early) and the update.
template <typename T>
struct BandVals {
  T pq, pm, xi;  // old ψ[q], old ψ[q-1], ξ[q-1]
};

template <typename T>
__device__ __forceinline__ BandVals<T> band_load(const BandSide<T>& B, int q, int64_t psi_base,
                                                 int64_t xi_base, int64_t stride) {
  BandVals<T> v;
  v.pq = B.psi_old[psi_base + (int64_t)q * stride];
  v.pm = B.psi_old[psi_base + (int64_t)(q - 1) * stride];
  v.xi = B.xi[xi_base + (int64_t)(q - 1) * stride];
  return v;
}

// pm, pc, pp: pressure at c-1, c, c+1 along the axis; d2: that axis's second
// difference; f: fact at the node.
template <typename T>
__device__ __forceinline__ void band_apply(const BandSide<T>& B, const BandVals<T>& L, int q,
                                           bool first, T pm, T pc, T pp, T d2, T f, T inv_d,
                                           int64_t psi_base, int64_t xi_base, int64_t stride,
                                           T& damp) {
  // update_ψ!: ψ = b_K_h ψ + a_h (p[c+1] - p[c]) / d, on both faces of the node
  const T ps_q = B.bKh[q] * L.pq + B.ah[q] * (pp - pc) * inv_d;
  const T ps_m = B.bKh[q - 1] * L.pm + B.ah[q - 1] * (pc - pm) * inv_d;
  B.psi_new[psi_base + (int64_t)q * stride] = ps_q;
  if (first) B.psi_new[psi_base + (int64_t)(q - 1) * stride] = ps_m;
  // update_p! band branch: dψ, ξ recursion, damping term
  const T dpsi = (ps_q - ps_m) * inv_d;
  const T xn = B.bK[q - 1] * L.xi + B.a[q - 1] * (d2 + dpsi);
  B.xi[xi_base + (int64_t)(q - 1) * stride] = xn;
  damp += f * (dpsi + xn);
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

// Element offsets of a node's band entries: ψ at psi_base + q*stride, ξ at
// xi_base + (q-1)*stride, for the three axes.
struct BandAddr {
  int64_t psi_base, xi_base, stride;
};
__device__ __forceinline__ BandAddr addr_x(int halo, int ny, int j, int k) {
  const int64_t jk = (int64_t)j + (int64_t)ny * k;
  return {(int64_t)(halo + 1) * jk, (int64_t)halo * jk, 1};
}
__device__ __forceinline__ BandAddr addr_y(int halo, int nx, int i, int k) {
  return {(int64_t)i + (int64_t)nx * (halo + 1) * k, (int64_t)i + (int64_t)nx * halo * k,
          (int64_t)nx};
}
__device__ __forceinline__ BandAddr addr_z(int nx, int ny, int i, int j) {
  const int64_t c = (int64_t)i + (int64_t)nx * j;
  return {c, c, (int64_t)nx * ny};
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
__device__ __forceinline__ void rim_io(const Io<T>& io, T* pnew, int it) {
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  const int nt = blockDim.x * blockDim.y;
  for (int e = t; e < io.nrim; e += nt) {
    const IoRim r = io.rim[e];
    pnew[r.node] = node_io(io, it, r.sgrp, r.rgrp, pnew[r.node]);
  }
}

// Walks this block's source/receiver entries of plane k (sorted by plane).
template <typename T>
__device__ __forceinline__ T plane_io(const Io<T>& io, int it, int& e, int e1, int k, int local,
                                      bool valid, T v) {
  for (; e < e1; ++e) {
    const int4 en = io.ent[e];
    if (en.y != k) break;
    if (valid && en.x == local) v = node_io(io, it, en.z, en.w, v);
  }
  return v;
}

// ---------------------------------------------------------------------------
// 3D step, register-queue variant: 2.5D blocking with the current plane of
// pcur (and a one-node ring) in shared memory for the x/y neighbours and the
// z neighbours in registers; the next plane's loads are issued one iteration
// ahead.
template <typename T, int BY>
__global__ void __launch_bounds__(32 * BY) step3d(StepParams<T> P) {
  __shared__ T tile[BY + 2][32 + 2];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = P.nx, ny = P.ny, nz = P.nz, halo = P.halo;
  const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (blk == 0 && P.io.nrim > 0) rim_io(P.io, P.pnew, P.it);
  const int i = blockIdx.x * 32 + tx;
  const int j = 1 + blockIdx.y * BY + ty;
  const bool valid = i >= 1 && i <= nx - 2 && j <= ny - 2;
  const int k0 = 1 + blockIdx.z * P.zchunk;
  int k1 = k0 + P.zchunk;
  if (k1 > nz - 1) k1 = nz - 1;
  if (k0 >= k1) return;  // block-uniform

  const int64_t px = P.px;
  const int64_t plane = px * ny;
  const int64_t col = (int64_t)i + px * j;
  const bool ldxl = valid && (tx == 0 || i == 1);
  const bool ldxr = valid && (tx == 31 || i == nx - 2);
  const bool ldyl = valid && ty == 0;
  const bool ldyh = valid && (ty == BY - 1 || j == ny - 2);

  const T* __restrict__ pcur = P.pcur;
  T pm = 0, pc = 0, pp = 0, po = 0, f = 0;
  T rxl = 0, rxr = 0, ryl = 0, ryh = 0;
  if (valid) {
    const int64_t o0 = col + (int64_t)k0 * plane;
    pm = __ldg(pcur + o0 - plane);
    pc = __ldg(pcur + o0);
    pp = __ldg(pcur + o0 + plane);
    po = __ldg(P.pold + o0);
    f = __ldg(P.fact + o0);
    if (ldxl) rxl = __ldg(pcur + o0 - 1);
    if (ldxr) rxr = __ldg(pcur + o0 + 1);
    if (ldyl) ryl = __ldg(pcur + o0 - px);
    if (ldyh) ryh = __ldg(pcur + o0 + px);
  }
  int qx = 0, qy = 0;
  bool fx = false, fy = false;
  const int bx = valid ? band_of(i, nx, halo, P.first_r[0], qx, fx) : 0;
  const int by = valid ? band_of(j, ny, halo, P.first_r[1], qy, fy) : 0;
  const bool doxb = bx != 0 && P.active[0][bx - 1];
  const bool doyb = by != 0 && P.active[1][by - 1];
  int ioe = P.io.blk_off[blk];
  const int ioe1 = P.io.blk_off[blk + 1];
  const int local = tx + 32 * ty;

  for (int k = k0; k < k1; ++k) {
    const int64_t o = col + (int64_t)k * plane;
    T npp = 0, npo = 0, nf = 0, nxl = 0, nxr = 0, nyl = 0, nyh = 0;
    if (valid && k + 1 < k1) {
      const int64_t on = o + plane;
      npp = __ldg(pcur + on + plane);
      npo = __ldg(P.pold + on);
      nf = __ldg(P.fact + on);
      if (ldxl) nxl = __ldg(pcur + on - 1);
      if (ldxr) nxr = __ldg(pcur + on + 1);
      if (ldyl) nyl = __ldg(pcur + on - px);
      if (ldyh) nyh = __ldg(pcur + on + px);
    }
    __syncthreads();  // the previous plane's readers are done with the tile
    if (valid) {
      tile[ty + 1][tx + 1] = pc;
      if (ldxl) tile[ty + 1][tx] = rxl;
      if (ldxr) tile[ty + 1][tx + 2] = rxr;
      if (ldyl) tile[ty][tx + 1] = ryl;
      if (ldyh) tile[ty + 2][tx + 1] = ryh;
    }
    __syncthreads();
    T v = 0;
    if (valid) {
      const T xm = tile[ty + 1][tx], xp = tile[ty + 1][tx + 2];
      const T ym = tile[ty][tx + 1], yp = tile[ty + 2][tx + 1];
      const T d2x = (xp - T(2) * pc + xm) * P.inv_d2[0];
      const T d2y = (yp - T(2) * pc + ym) * P.inv_d2[1];
      const T d2z = (pp - T(2) * pc + pm) * P.inv_d2[2];
      T damp = 0;
      if (doxb) {
        const BandAddr a = addr_x(halo, ny, j, k);
        const BandSide<T>& B = P.band[0][bx - 1];
        band_apply(B, band_load(B, qx, a.psi_base, a.xi_base, a.stride), qx, fx, xm, pc, xp, d2x,
                   f, P.inv_d[0], a.psi_base, a.xi_base, a.stride, damp);
      }
      if (doyb) {
        const BandAddr a = addr_y(halo, nx, i, k);
        const BandSide<T>& B = P.band[1][by - 1];
        band_apply(B, band_load(B, qy, a.psi_base, a.xi_base, a.stride), qy, fy, ym, pc, yp, d2y,
                   f, P.inv_d[1], a.psi_base, a.xi_base, a.stride, damp);
      }
      {
        int qz;
        bool fz;
        const int bz = band_of(k, nz, halo, P.first_r[2], qz, fz);
        if (bz != 0 && P.active[2][bz - 1]) {
          const BandAddr a = addr_z(nx, ny, i, j);
          const BandSide<T>& B = P.band[2][bz - 1];
          band_apply(B, band_load(B, qz, a.psi_base, a.xi_base, a.stride), qz, fz, pm, pc, pp,
                     d2z, f, P.inv_d[2], a.psi_base, a.xi_base, a.stride, damp);
        }
      }
      v = T(2) * pc - po + f * (d2x + d2y + d2z) + damp;
    }
    v = plane_io(P.io, P.it, ioe, ioe1, k, local, valid, v);
    if (valid) P.pnew[o] = v;
    pm = pc;
    pc = pp;
    pp = npp;
    po = npo;
    f = nf;
    rxl = nxl;
    rxr = nxr;
    ryl = nyl;
    ryh = nyh;
  }
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
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on a phase of an mbarrier: false when the limit runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int n = 0; n < (1 << 22); ++n)
    if (mbar_try_wait(bar, parity)) return true;
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

// Shared-memory layout of one pipeline stage (plane m) of step3d_tma.
template <typename T, int BY>
struct TmaStage {
  static constexpr int A = 16 / (int)sizeof(T);  // x apron keeping the box origin 16-B aligned
  static constexpr int PW = 32 + 2 * A;          // pcur box width
  static constexpr int PC_BYTES = PW * (BY + 2) * (int)sizeof(T);
  static constexpr int PC_PAD = (PC_BYTES + 127) / 128 * 128;
  static constexpr int IN_BYTES = 32 * BY * (int)sizeof(T);
  static constexpr int BYTES = PC_PAD + 2 * IN_BYTES;
};

// ---------------------------------------------------------------------------
// 3D step, TMA-pipelined variant. Same tile/chunk decomposition as step3d;
// one elected thread streams, per z plane m, three boxes into a ring of S
// shared-memory stages with cp.async.bulk.tensor:
//   pcur (32 + 2A) x (BY + 2) around the tile (the x/y ring included;
//        outside the grid TMA fills zeros), pold 32 x BY, fact 32 x BY,
// each stage completing on its own mbarrier. Plane k is computed from the
// stages of planes k-1, k, k+1 while the loads of planes up to k+S-2 are in
// flight, so the memory pipeline runs S-3 planes ahead with no register cost.
// The CPML band values of the plane are loaded by the owning threads before
// they wait on the plane's barrier.
template <typename T, int BY, int S>
__global__ void __launch_bounds__(32 * BY) step3d_tma(const __grid_constant__ CUtensorMap mc,
                                                      const __grid_constant__ CUtensorMap mo,
                                                      const __grid_constant__ CUtensorMap mf,
                                                      StepParams<T> P) {
  using L = TmaStage<T, BY>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + S * L::BYTES);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  const int nx = P.nx, ny = P.ny, nz = P.nz, halo = P.halo;
  const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (blk == 0 && P.io.nrim > 0) rim_io(P.io, P.pnew, P.it);
  const int x0 = blockIdx.x * 32, y0 = 1 + blockIdx.y * BY;
  const int i = x0 + tx, j = y0 + ty;
  const bool valid = i >= 1 && i <= nx - 2 && j <= ny - 2;
  const int k0 = 1 + blockIdx.z * P.zchunk;
  int k1 = k0 + P.zchunk;
  if (k1 > nz - 1) k1 = nz - 1;
  if (k0 >= k1) return;  // block-uniform
  const int nplanes = k1 - k0 + 2;  // pcur planes k0-1 .. k1

  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // use u loads plane m = k0-1+u into stage u % S; pold/fact only for m in [k0, k1)
  auto issue = [&](int u) {
    const int s = u % S, m = k0 - 1 + u;
    unsigned char* st = smem + s * L::BYTES;
    const bool full = m >= k0 && m < k1;
    mbar_expect_tx(&bar[s], L::PC_BYTES + (full ? 2 * L::IN_BYTES : 0));
    tma_load_3d(st, &mc, &bar[s], x0 - L::A, y0 - 1, m);
    if (full) {
      tma_load_3d(st + L::PC_PAD, &mo, &bar[s], x0, y0, m);
      tma_load_3d(st + L::PC_PAD + L::IN_BYTES, &mf, &bar[s], x0, y0, m);
    }
  };
  if (tid == 0)
    for (int u = 0; u < S && u < nplanes; ++u) issue(u);

  int qx = 0, qy = 0;
  bool fx = false, fy = false;
  const int bx = valid ? band_of(i, nx, halo, P.first_r[0], qx, fx) : 0;
  const int by = valid ? band_of(j, ny, halo, P.first_r[1], qy, fy) : 0;
  const bool doxb = bx != 0 && P.active[0][bx - 1];
  const bool doyb = by != 0 && P.active[1][by - 1];
  int ioe = P.io.blk_off[blk];
  const int ioe1 = P.io.blk_off[blk + 1];
  const int64_t px = P.px, plane = px * ny;
  const int64_t col = (int64_t)i + px * j;
  constexpr int A = L::A, PW = L::PW;

  bool ok = mbar_wait(&bar[0], 0) && mbar_wait(&bar[1 % S], (1 / S) & 1);
  int uc = 1;  // use index of the current plane
  for (int k = k0; k < k1; ++k, ++uc) {
    // CPML band values of this plane, issued before the barrier wait
    BandVals<T> lx{}, ly{}, lz{};
    int qz = 0;
    bool fz = false;
    const int bz = band_of(k, nz, halo, P.first_r[2], qz, fz);
    const bool dozb = valid && bz != 0 && P.active[2][bz - 1];
    const BandAddr axx = addr_x(halo, ny, j, k), ayy = addr_y(halo, nx, i, k),
                   azz = addr_z(nx, ny, i, j);
    if (doxb) lx = band_load(P.band[0][bx - 1], qx, axx.psi_base, axx.xi_base, axx.stride);
    if (doyb) ly = band_load(P.band[1][by - 1], qy, ayy.psi_base, ayy.xi_base, ayy.stride);
    if (dozb) lz = band_load(P.band[2][bz - 1], qz, azz.psi_base, azz.xi_base, azz.stride);

    ok = ok && mbar_wait(&bar[(uc + 1) % S], ((uc + 1) / S) & 1);
    const T* cm = reinterpret_cast<const T*>(smem + ((uc - 1) % S) * L::BYTES);
    const T* cc = reinterpret_cast<const T*>(smem + (uc % S) * L::BYTES);
    const T* cp = reinterpret_cast<const T*>(smem + ((uc + 1) % S) * L::BYTES);
    const T* oo = reinterpret_cast<const T*>(smem + (uc % S) * L::BYTES + L::PC_PAD);
    const T* ff = oo + 32 * BY;
    T v = 0;
    if (valid && ok) {
      const int c = (ty + 1) * PW + tx + A;
      const T pc = cc[c], xm = cc[c - 1], xp = cc[c + 1], ym = cc[c - PW], yp = cc[c + PW];
      const T pm = cm[c], pp = cp[c];
      const T po = oo[ty * 32 + tx], f = ff[ty * 32 + tx];
      const T d2x = (xp - T(2) * pc + xm) * P.inv_d2[0];
      const T d2y = (yp - T(2) * pc + ym) * P.inv_d2[1];
      const T d2z = (pp - T(2) * pc + pm) * P.inv_d2[2];
      T damp = 0;
      if (doxb)
        band_apply(P.band[0][bx - 1], lx, qx, fx, xm, pc, xp, d2x, f, P.inv_d[0], axx.psi_base,
                   axx.xi_base, axx.stride, damp);
      if (doyb)
        band_apply(P.band[1][by - 1], ly, qy, fy, ym, pc, yp, d2y, f, P.inv_d[1], ayy.psi_base,
                   ayy.xi_base, ayy.stride, damp);
      if (dozb)
        band_apply(P.band[2][bz - 1], lz, qz, fz, pm, pc, pp, d2z, f, P.inv_d[2], azz.psi_base,
                   azz.xi_base, azz.stride, damp);
      v = T(2) * pc - po + f * (d2x + d2y + d2z) + damp;
    }
    v = plane_io(P.io, P.it, ioe, ioe1, k, tid, valid && ok, v);
    if (valid && ok) P.pnew[col + (int64_t)k * plane] = v;
    // every thread is done with stage (uc-1): refill it with plane use uc-1+S
    if (__syncthreads_or(!ok)) {
      // a wait ran out: record it and drain what this block still has in flight
      if (tid == 0) {
        atomicExch(P.err, 1);
        for (int u = uc + 1; u < nplanes && u < uc - 1 + S; ++u) mbar_wait(&bar[u % S], (u / S) & 1);
      }
      return;
    }
    if (tid == 0 && uc - 1 + S < nplanes) issue(uc - 1 + S);
  }
}

// ---------------------------------------------------------------------------
// 2D step: one thread per interior node; neighbours through L1.
template <typename T>
__global__ void __launch_bounds__(256) step2d(StepParams<T> P) {
  const int nx = P.nx, ny = P.ny, halo = P.halo;
  const int blk = blockIdx.x + gridDim.x * blockIdx.y;
  if (blk == 0 && P.io.nrim > 0) rim_io(P.io, P.pnew, P.it);
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
  const T d2x = (xp - T(2) * pc + xm) * P.inv_d2[0];
  const T d2y = (yp - T(2) * pc + ym) * P.inv_d2[1];
  T damp = 0;
  int q;
  bool first;
  const int bx = band_of(i, nx, halo, P.first_r[0], q, first);
  if (bx != 0 && P.active[0][bx - 1]) {
    const BandSide<T>& B = P.band[0][bx - 1];
    const int64_t pb = (int64_t)(halo + 1) * j, xb = (int64_t)halo * j;
    band_apply(B, band_load(B, q, pb, xb, (int64_t)1), q, first, xm, pc, xp, d2x, f, P.inv_d[0],
               pb, xb, (int64_t)1, damp);
  }
  const int by = band_of(j, ny, halo, P.first_r[1], q, first);
  if (by != 0 && P.active[1][by - 1]) {
    const BandSide<T>& B = P.band[1][by - 1];
    band_apply(B, band_load(B, q, (int64_t)i, (int64_t)i, (int64_t)nx), q, first, ym, pc, yp, d2y,
               f, P.inv_d[1], (int64_t)i, (int64_t)i, (int64_t)nx, damp);
  }
  T v = T(2) * pc - po + f * (d2x + d2y) + damp;
  const int local = threadIdx.x + 32 * threadIdx.y;
  for (int e = P.io.blk_off[blk]; e < P.io.blk_off[blk + 1]; ++e) {
    const int4 en = P.io.ent[e];
    if (en.x == local) v = node_io(P.io, P.it, en.z, en.w, v);
  }
  P.pnew[o] = v;
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
