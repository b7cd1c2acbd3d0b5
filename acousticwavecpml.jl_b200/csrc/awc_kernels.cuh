// awc_kernels.cuh — sm_100a kernels of one CPML acoustic time step.
//
// One launch of step3d/step2d performs, for every interior node, the work of
// the reference's update_ψ_{x,y,z}! + update_p! pair
// (src/shared/acoustic_3D_xPU.jl:8-104; 2D src/shared/acoustic_2D_xPU.jl:7-75):
//   - the 2nd-order Laplacian of pcur,
//   - inside the CPML bands, the staggered ψ recursion, ξ recursion and the
//     damping term,
//   - the leapfrog update pnew = 2 pcur - pold + fact*lap + damp,
// inject_record then adds the sources and samples the receivers (:106-122).
//
// Memory layout in HBM (column-major like the reference, x fastest):
//   p fields, fact        nx*ny*nz
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
#pragma once
#include <cstdint>
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

// Sources and receivers of the step handled inside the step kernel.
// Interior sources are grouped by node (CSR: node, [off, off+1) into ids).
template <typename T>
struct Io {
  const int64_t* src_node;  // unique source nodes (linear index)
  const int32_t* src_off;   // nsrc_nodes+1 offsets into src_ids
  const int32_t* src_ids;   // source indices in source order
  int32_t nsrc_nodes;
  const T* stf;             // [nt][nsrc] scaled source time functions, row `it` used
  int32_t nsrc;
  const int64_t* rec_node;  // receiver node per receiver
  int32_t nrec;
  T* traces;                // [nt][nrec]
};

template <typename T>
struct StepParams {
  const T* pold;
  const T* pcur;
  T* pnew;
  const T* fact;
  int32_t nx, ny, nz, halo;
  T inv_d[3];
  T inv_d2[3];
  BandSide<T> band[3][2];  // [axis][left/right]
  int32_t active[3][2];    // side carries a non-trivial CPML recursion
  int32_t first_r[3];      // first node (0-based) of the right band per axis
  int32_t zchunk;          // planes per block along z (3D)
  int32_t it;              // 0-based time step index (row of stf/traces)
};

// The CPML contribution of one axis at one node; see the header comment.
// pm, pc, pp: pressure at c-1, c, c+1 along the axis; d2: that axis's second
// difference; f: fact at the node; psi/xi element offsets of the node's
// cross-section: psi_base + q*stride, xi_base + (q-1)*stride.
template <typename T>
__device__ __forceinline__ void band_axis(const BandSide<T>& B, int q, bool first, T pm, T pc,
                                          T pp, T d2, T f, T inv_d, int64_t psi_base,
                                          int64_t xi_base, int64_t stride, T& damp) {
  const T ps_q_old = B.psi_old[psi_base + (int64_t)q * stride];
  const T ps_m_old = B.psi_old[psi_base + (int64_t)(q - 1) * stride];
  // update_ψ!: ψ = b_K_h ψ + a_h (p[c+1] - p[c]) / d, on both faces of the node
  const T ps_q = B.bKh[q] * ps_q_old + B.ah[q] * (pp - pc) * inv_d;
  const T ps_m = B.bKh[q - 1] * ps_m_old + B.ah[q - 1] * (pc - pm) * inv_d;
  B.psi_new[psi_base + (int64_t)q * stride] = ps_q;
  if (first) B.psi_new[psi_base + (int64_t)(q - 1) * stride] = ps_m;
  // update_p! band branch: dψ, ξ recursion, damping term
  const T dpsi = (ps_q - ps_m) * inv_d;
  T* xp = B.xi + xi_base + (int64_t)(q - 1) * stride;
  const T xn = B.bK[q - 1] * (*xp) + B.a[q - 1] * (d2 + dpsi);
  *xp = xn;
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

// ---------------------------------------------------------------------------
// 3D step: 2.5D blocking. A block of 32 x BY threads owns a 32 x BY column
// tile of interior (i, j) and streams `zchunk` consecutive z planes. The
// current plane of pcur (with a one-node ring) sits in shared memory for the
// x/y neighbours; the z neighbours ride in registers. Every global load of
// the next plane (pcur centre and ring, pold, fact) is issued one iteration
// ahead so that its latency overlaps the current plane's arithmetic.
template <typename T, int BY>
__global__ void __launch_bounds__(32 * BY) step3d(StepParams<T> P) {
  __shared__ T tile[BY + 2][32 + 2];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nx = P.nx, ny = P.ny, nz = P.nz, halo = P.halo;
  const int i = 1 + blockIdx.x * 32 + tx;
  const int j = 1 + blockIdx.y * BY + ty;
  const bool valid = (i <= nx - 2) && (j <= ny - 2);
  const int k0 = 1 + blockIdx.z * P.zchunk;
  int k1 = k0 + P.zchunk;
  if (k1 > nz - 1) k1 = nz - 1;
  if (k0 >= k1) return;  // block-uniform

  const int64_t plane = (int64_t)nx * ny;
  const int64_t col = (int64_t)i + (int64_t)nx * j;
  // ring loaders: x-left (tx==0), x-right (last valid x of the tile row),
  // y-low (ty==0), y-high (last valid y of the tile column)
  const bool ldxl = valid && tx == 0;
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
    if (ldyl) ryl = __ldg(pcur + o0 - nx);
    if (ldyh) ryh = __ldg(pcur + o0 + nx);
  }
  // band membership along x and y is fixed for the thread
  int qx = 0, qy = 0;
  bool fx = false, fy = false;
  const int bx = valid ? band_of(i, nx, halo, P.first_r[0], qx, fx) : 0;
  const int by = valid ? band_of(j, ny, halo, P.first_r[1], qy, fy) : 0;
  const bool doxb = bx != 0 && P.active[0][bx - 1];
  const bool doyb = by != 0 && P.active[1][by - 1];

  for (int k = k0; k < k1; ++k) {
    const int64_t o = col + (int64_t)k * plane;
    // prefetch plane k+1 (its z+1 neighbour is plane k+2)
    T npp = 0, npo = 0, nf = 0, nxl = 0, nxr = 0, nyl = 0, nyh = 0;
    const bool more = valid && (k + 1 < k1);
    if (more) {
      const int64_t on = o + plane;
      npp = __ldg(pcur + on + plane);
      npo = __ldg(P.pold + on);
      nf = __ldg(P.fact + on);
      if (ldxl) nxl = __ldg(pcur + on - 1);
      if (ldxr) nxr = __ldg(pcur + on + 1);
      if (ldyl) nyl = __ldg(pcur + on - nx);
      if (ldyh) nyh = __ldg(pcur + on + nx);
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
    if (valid) {
      const T xm = tile[ty + 1][tx], xp = tile[ty + 1][tx + 2];
      const T ym = tile[ty][tx + 1], yp = tile[ty + 2][tx + 1];
      const T d2x = (xp - T(2) * pc + xm) * P.inv_d2[0];
      const T d2y = (yp - T(2) * pc + ym) * P.inv_d2[1];
      const T d2z = (pp - T(2) * pc + pm) * P.inv_d2[2];
      T damp = 0;
      if (doxb) {
        const int64_t hq = halo + 1;
        band_axis(P.band[0][bx - 1], qx, fx, xm, pc, xp, d2x, f, P.inv_d[0],
                  hq * ((int64_t)j + (int64_t)ny * k), (int64_t)halo * ((int64_t)j + (int64_t)ny * k),
                  (int64_t)1, damp);
      }
      if (doyb) {
        band_axis(P.band[1][by - 1], qy, fy, ym, pc, yp, d2y, f, P.inv_d[1],
                  (int64_t)i + (int64_t)nx * (halo + 1) * k, (int64_t)i + (int64_t)nx * halo * k,
                  (int64_t)nx, damp);
      }
      {
        int qz;
        bool fz;
        const int bz = band_of(k, nz, halo, P.first_r[2], qz, fz);
        if (bz != 0 && P.active[2][bz - 1]) {
          band_axis(P.band[2][bz - 1], qz, fz, pm, pc, pp, d2z, f, P.inv_d[2], col, col, plane,
                    damp);
        }
      }
      P.pnew[o] = T(2) * pc - po + f * (d2x + d2y + d2z) + damp;
    }
    // rotate the register queue
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
// 2D step: one thread per interior node; neighbours through L1.
template <typename T>
__global__ void __launch_bounds__(256) step2d(StepParams<T> P) {
  const int nx = P.nx, ny = P.ny, halo = P.halo;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx - 2 || j > ny - 2) return;
  const int64_t o = (int64_t)i + (int64_t)nx * j;
  const T* __restrict__ pcur = P.pcur;
  const T pc = __ldg(pcur + o);
  const T xm = __ldg(pcur + o - 1), xp = __ldg(pcur + o + 1);
  const T ym = __ldg(pcur + o - nx), yp = __ldg(pcur + o + nx);
  const T po = __ldg(P.pold + o), f = __ldg(P.fact + o);
  const T d2x = (xp - T(2) * pc + xm) * P.inv_d2[0];
  const T d2y = (yp - T(2) * pc + ym) * P.inv_d2[1];
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
              (int64_t)i, (int64_t)nx, damp);
  P.pnew[o] = T(2) * pc - po + f * (d2x + d2y) + damp;
}

// ---------------------------------------------------------------------------
// inject_sources! then record_receivers! for one step, one block: sources
// grouped by node are summed in source order, then every receiver samples
// the new field (acoustic_3D_xPU.jl:106-122).
template <typename T>
__global__ void __launch_bounds__(1024) inject_record(T* __restrict__ pnew, Io<T> io, int it) {
  for (int u = threadIdx.x; u < io.nsrc_nodes; u += blockDim.x) {
    const int64_t node = io.src_node[u];
    T v = pnew[node];
    for (int e = io.src_off[u]; e < io.src_off[u + 1]; ++e)
      v += io.stf[(int64_t)it * io.nsrc + io.src_ids[e]];
    pnew[node] = v;
  }
  __syncthreads();  // injected values are visible to the whole block
  for (int r = threadIdx.x; r < io.nrec; r += blockDim.x)
    io.traces[(int64_t)it * io.nrec + r] = pnew[io.rec_node[r]];
}

// fact = (dt^2) * (vel^2) in FP64, rounded once to T (acoustic_3D_xPU.jl:242).
template <typename T>
__global__ void make_fact(const double* __restrict__ vel, T* __restrict__ fact, double dt2,
                          int64_t n) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const double v = vel[c];
    fact[c] = (T)(dt2 * (v * v));
  }
}

// T -> double copy (field read-out).
template <typename T>
__global__ void widen(const T* __restrict__ src, double* __restrict__ dst, int64_t n) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    dst[c] = (double)src[c];
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
