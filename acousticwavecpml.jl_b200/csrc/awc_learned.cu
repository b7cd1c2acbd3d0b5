// Forward solve with a learned thin absorbing layer in place of the CPML.
//
// The outermost W interior nodes of every absorbing side (all sides but a
// free top) form the layer. Interior nodes farther in take the plain
// leapfrog step p_{t+1} = 2 p_t - p_{t-1} + F lap(p_t) (no CPML state).
// A layer node n takes p_{t+1}(n) = s MLP(x / s) with
//   x = (p_{t-2}, p_{t-1}, p_t) on the 3^d block around n (nodes outside the
//       grid read 0; the Dirichlet rim is 0), ordered by time level, then
//       along the outward normal u = -1, 0, +1 of the nearest absorbing side,
//       then along the remaining axes in increasing axis order;
//   s = max |x| (or 1 when x = 0), so that the layer is linear in amplitude;
//   MLP: K -> 32 -> 32 -> 1 with ReLU over x / s and the local Courant number
//       r = c dt / d along the normal (K = 3 * 3^d + 1: 28 in 2D, 82 in 3D;
//       without r a local operator cannot tell how fast the wave leaves),
//       weights in BF16, products accumulated in FP32.
// The two hidden layers run on the tensor cores (mma.sync m16n8k16, BF16
// operands, FP32 accumulation): a warp takes 16 layer nodes at a time, the
// weights are B operands as they are, and each FP32 activation enters as
// the sum of three BF16 terms (hi + mid + lo, three MMAs), which carries its
// 24 bits: the products are those of the FP32 activations with the BF16
// weights, accumulated in FP32 (a BF16-rounded activation would change the
// solution by up to 5e-2 relative over a few hundred steps of an unstable
// layer).
// A node within W of two sides uses the nearer one (x before y before z on
// ties). Sources are added after the update, then receivers sample p_{t+1}.
// FP32 only; rim sources and receivers are rejected.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/awcpml.h"
#include "awc_ctx.h"

namespace {

constexpr int kHid = 32;
constexpr int kMaxKP = 96;          // K (at most 82) padded to the MMA's k of 16
constexpr int kWS1 = kMaxKP + 8;    // smem row strides (bf16): conflict-free B loads
constexpr int kWS2 = kHid + 8;
constexpr int kXS = kMaxKP + 8;     // smem row stride (floats) of a warp's input tile
constexpr int kWarps = 4;

struct LearnedParams {
  int32_t ndim, nx, ny, nz, width, freetop;
  int64_t px, plane;
  float inv_d2[3];
  float inv_d[3];
  const float* F;
  const float* p0;  // p_{t-2}
  const float* p1;  // p_{t-1}
  const float* p2;  // p_t
  float* p3;        // p_{t+1}
  const __nv_bfloat16* w;  // W1 (32 x K), b1 (32), W2 (32 x 32), b2 (32), W3 (32), b3 (1)
  int32_t nin;
  const int4* layer;  // layer nodes (i, j, k, 2 axis + (sign > 0)), memory order
  int32_t nlayer;
};

// The leapfrog step at every interior node; the layer kernel, which runs
// after it, overwrites the layer nodes.
__global__ void __launch_bounds__(256) learned_interior(LearnedParams L) {
  const int i = 1 + blockIdx.x * 32 + threadIdx.x;
  const int j = 1 + blockIdx.y * 8 + threadIdx.y;
  const int k = L.ndim == 3 ? 1 + blockIdx.z : 0;
  if (i > L.nx - 2 || j > L.ny - 2) return;
  const int64_t o = i + L.px * j + L.plane * k;
  const float pc = L.p2[o];
  float lap = (L.p2[o + 1] - 2.f * pc + L.p2[o - 1]) * L.inv_d2[0] +
              (L.p2[o + L.px] - 2.f * pc + L.p2[o - L.px]) * L.inv_d2[1];
  if (L.ndim == 3) lap += (L.p2[o + L.plane] - 2.f * pc + L.p2[o - L.plane]) * L.inv_d2[2];
  L.p3[o] = fmaf(L.F[o], lap, 2.f * pc - L.p1[o]);
}

// D += A B on the tensor cores: m16n8k16, A and B BF16, D and C FP32.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Two FP32 values as three pairs of BF16 terms (hi, mid, lo), each pair
// packed low element first: x = hi + mid + lo to within 2^-27 |x|.
__device__ __forceinline__ void split3(float x0, float x1, uint32_t& hi, uint32_t& mid,
                                       uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float r0 = x0 - __low2float(h), r1 = x1 - __high2float(h);
  const __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
  const __nv_bfloat162 l = __floats2bfloat162_rn(r0 - __low2float(m), r1 - __high2float(m));
  hi = *reinterpret_cast<const uint32_t*>(&h);
  mid = *reinterpret_cast<const uint32_t*>(&m);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// acc (16 x 8 tile nt) += A B for the A fragment given as values: row g
// (x[0..1] at k 2t, 2t+1; x[4..5] at k 2t+8, 2t+9) and row g+8 (x[2..3],
// x[6..7]); B from the bf16 rows of w (row stride ws) at k0.
__device__ __forceinline__ void mma_split(float (&acc)[4][4], const float (&x)[8],
                                          const __nv_bfloat16* w, int ws, int k0, int g, int t) {
  uint32_t ah[4], am[4], al[4];
  split3(x[0], x[1], ah[0], am[0], al[0]);
  split3(x[2], x[3], ah[1], am[1], al[1]);
  split3(x[4], x[5], ah[2], am[2], al[2]);
  split3(x[6], x[7], ah[3], am[3], al[3]);
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) {
    const __nv_bfloat16* row = w + (nt * 8 + g) * ws + k0 + 2 * t;
    const uint32_t b0 = *reinterpret_cast<const uint32_t*>(row);
    const uint32_t b1 = *reinterpret_cast<const uint32_t*>(row + 8);
    mma_bf16(acc[nt], al, b0, b1);  // small terms first
    mma_bf16(acc[nt], am, b0, b1);
    mma_bf16(acc[nt], ah, b0, b1);
  }
}

// The layer nodes, 16 per warp and step of its loop: the inputs of the 16
// nodes are gathered into a shared tile (two lanes per node), scaled by
// 1/s, and the two hidden layers run as MMAs whose accumulators stay in
// registers (layer 1's output fragments are layer 2's A operand); the
// output layer is a dot product reduced over the four lanes of a row.
__global__ void __launch_bounds__(32 * kWarps) learned_layer(LearnedParams L) {
  __shared__ __align__(16) __nv_bfloat16 w1s[kHid * kWS1];
  __shared__ __align__(16) __nv_bfloat16 w2s[kHid * kWS2];
  __shared__ float b1s[kHid], b2s[kHid], w3s[kHid];
  __shared__ __align__(16) float xs[kWarps][16 * kXS];
  __shared__ float ss[kWarps][16];
  const int K = L.nin, KP = (K + 15) / 16 * 16;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const __nv_bfloat16* W1 = L.w;
  const __nv_bfloat16* W2 = W1 + kHid * K + kHid;
  for (int e = tid; e < kHid * kWS1; e += 32 * kWarps) {
    const int n = e / kWS1, c = e % kWS1;
    w1s[e] = c < K ? W1[n * K + c] : __float2bfloat16(0.f);
  }
  for (int e = tid; e < kHid * kWS2; e += 32 * kWarps) {
    const int n = e / kWS2, c = e % kWS2;
    w2s[e] = c < kHid ? W2[n * kHid + c] : __float2bfloat16(0.f);
  }
  for (int e = tid; e < kHid; e += 32 * kWarps) {
    b1s[e] = __bfloat162float(W1[kHid * K + e]);
    b2s[e] = __bfloat162float(W2[kHid * kHid + e]);
    w3s[e] = __bfloat162float(W2[kHid * kHid + kHid + e]);
  }
  float* X = xs[warp];
  for (int e = lane; e < 16 * kXS; e += 32) X[e] = 0.f;  // the padding columns stay 0
  __syncthreads();
  const float b3 = __bfloat162float(W2[kHid * kHid + 2 * kHid]);
  const bool d3 = L.ndim == 3;
  const int npos = d3 ? 27 : 9;    // block positions per time level
  const int nfield = 3 * npos;     // inputs from the field; input nfield is r
  const int g = lane >> 2, t = lane & 3;
  const int n = lane & 15, h = lane >> 4;  // gather: node n of the group, half h
  for (int grp = blockIdx.x * kWarps + warp; grp * 16 < L.nlayer; grp += gridDim.x * kWarps) {
    // gather the raw inputs of node n: this lane takes every other block
    // position and its three time levels
    const int m = grp * 16 + n;
    const bool valid = m < L.nlayer;
    const int4 nd = valid ? L.layer[m] : make_int4(1, 1, 1, 1);
    const int ax = nd.w >> 1;
    const bool pos = nd.w & 1;
    // steps along the outward normal (u), the first transverse axis (v) and
    // the second (w, 3D), and which of the offsets -1, 0, +1 stay inside
    // the interior (bit e for offset e - 1)
    const int64_t sx = 1, sy = L.px, sz = L.plane;
    const int64_t su0 = ax == 0 ? sx : ax == 1 ? sy : sz;
    const int64_t su = pos ? su0 : -su0;
    const int64_t sv = ax == 0 ? sy : sx;
    const int64_t sw = ax == 2 ? sy : sz;
    auto ok3 = [](int c, int nmax) {  // offsets -1, 0, +1 of c within [1, nmax]
      return (c - 1 >= 1 ? 1 : 0) | 2 | (c + 1 <= nmax ? 4 : 0);
    };
    const int cu = ax == 0 ? nd.x : ax == 1 ? nd.y : nd.z;
    const int nu = ax == 0 ? L.nx : ax == 1 ? L.ny : L.nz;
    int mu = ok3(cu, nu - 2);
    if (!pos) mu = ((mu & 1) << 2) | (mu & 2) | ((mu >> 2) & 1);  // u runs against the axis
    const int mv = ax == 0 ? ok3(nd.y, L.ny - 2) : ok3(nd.x, L.nx - 2);
    const int mw = d3 ? (ax == 2 ? ok3(nd.y, L.ny - 2) : ok3(nd.z, L.nz - 2)) : 2;
    const int64_t o = nd.x + L.px * nd.y + L.plane * nd.z;
    float smax = 0.f;
    for (int q = h; q < npos; q += 2) {
      const int u1 = d3 ? q / 9 : q / 3;
      const int r1 = d3 ? q - 9 * u1 : q - 3 * u1;
      const int v1 = d3 ? r1 / 3 : r1;
      const int w1 = d3 ? r1 - 3 * v1 : 1;
      const bool in = valid && ((mu >> u1) & (mv >> v1) & (mw >> w1) & 1);
      const int64_t off = o + (u1 - 1) * su + (v1 - 1) * sv + (d3 ? (w1 - 1) * sw : 0);
      const float a = in ? L.p0[off] : 0.f;
      const float b = in ? L.p1[off] : 0.f;
      const float c = in ? L.p2[off] : 0.f;
      X[n * kXS + q] = a;
      X[n * kXS + npos + q] = b;
      X[n * kXS + 2 * npos + q] = c;
      smax = fmaxf(smax, fmaxf(fabsf(a), fmaxf(fabsf(b), fabsf(c))));
    }
    smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, 16));
    if (h == 0) {
      X[n * kXS + nfield] = valid ? sqrtf(L.F[o]) * L.inv_d[ax] : 0.f;  // Courant number
      ss[warp][n] = smax;
    }
    __syncwarp();
    // the field inputs enter scaled by 1/s of their row (r as it is)
    const float sg0 = ss[warp][g], sg1 = ss[warp][g + 8];
    const float inv0 = sg0 > 0.f ? 1.f / sg0 : 1.f, inv1 = sg1 > 0.f ? 1.f / sg1 : 1.f;
    // layer 1: 16 x KP by KP x 32
    float acc[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      acc[nt][0] = acc[nt][2] = b1s[nt * 8 + 2 * t];
      acc[nt][1] = acc[nt][3] = b1s[nt * 8 + 2 * t + 1];
    }
    for (int k0 = 0; k0 < KP; k0 += 16) {
      const int ca = k0 + 2 * t, cb = ca + 8;  // this lane's columns ca, ca + 1, cb, cb + 1
      const float2 r0 = *reinterpret_cast<const float2*>(X + g * kXS + ca);
      const float2 r1 = *reinterpret_cast<const float2*>(X + (g + 8) * kXS + ca);
      const float2 r2 = *reinterpret_cast<const float2*>(X + g * kXS + cb);
      const float2 r3 = *reinterpret_cast<const float2*>(X + (g + 8) * kXS + cb);
      auto sc = [&](float v, int col, float inv) { return col < nfield ? v * inv : v; };
      const float xa[8] = {sc(r0.x, ca, inv0), sc(r0.y, ca + 1, inv0), sc(r1.x, ca, inv1),
                           sc(r1.y, ca + 1, inv1), sc(r2.x, cb, inv0), sc(r2.y, cb + 1, inv0),
                           sc(r3.x, cb, inv1), sc(r3.y, cb + 1, inv1)};
      mma_split(acc, xa, w1s, kWS1, k0, g, t);
    }
    // layer 2: the ReLU'd accumulators are the A operand (k block kb = the
    // n tiles 2kb, 2kb + 1)
    float acc2[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      acc2[nt][0] = acc2[nt][2] = b2s[nt * 8 + 2 * t];
      acc2[nt][1] = acc2[nt][3] = b2s[nt * 8 + 2 * t + 1];
    }
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) {
      const float* lo = acc[2 * kb];
      const float* hi = acc[2 * kb + 1];
      const float xa[8] = {fmaxf(lo[0], 0.f), fmaxf(lo[1], 0.f), fmaxf(lo[2], 0.f),
                           fmaxf(lo[3], 0.f), fmaxf(hi[0], 0.f), fmaxf(hi[1], 0.f),
                           fmaxf(hi[2], 0.f), fmaxf(hi[3], 0.f)};
      mma_split(acc2, xa, w2s, kWS2, kb * 16, g, t);
    }
    // output layer: rows g and g + 8, reduced over the row's four lanes
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const float wa = w3s[nt * 8 + 2 * t], wb = w3s[nt * 8 + 2 * t + 1];
      y0 = fmaf(wa, fmaxf(acc2[nt][0], 0.f), fmaf(wb, fmaxf(acc2[nt][1], 0.f), y0));
      y1 = fmaf(wa, fmaxf(acc2[nt][2], 0.f), fmaf(wb, fmaxf(acc2[nt][3], 0.f), y1));
    }
    y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
    y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
    if (t == 0) {
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        const int row = g + 8 * rr, mr = grp * 16 + row;
        if (mr < L.nlayer) {
          const int4 q = L.layer[mr];
          const float sc = ss[warp][row];
          L.p3[q.x + L.px * q.y + L.plane * q.z] = ((rr ? y1 : y0) + b3) * (sc > 0.f ? sc : 1.f);
        }
      }
    }
    __syncwarp();  // the tile and ss are rewritten by the next group
  }
}

__global__ void learned_io(float* __restrict__ p3, const int64_t* __restrict__ snode, int32_t nsrc,
                           const float* __restrict__ stf_row, const int64_t* __restrict__ rnode,
                           int32_t nrec, float* __restrict__ tr_row) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int s = 0; s < nsrc; ++s) p3[snode[s]] += stf_row[s];
  for (int r = 0; r < nrec; ++r) tr_row[r] = p3[rnode[r]];
}

__global__ void learned_fact(const double* __restrict__ vel, float* __restrict__ F, double dt2,
                             int64_t n, int64_t nx, int64_t px) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = c % nx, r = c / nx;
    F[i + px * r] = (float)(dt2 * vel[c] * vel[c]);
  }
}

__global__ void learned_unpitch(const float* __restrict__ src, double* __restrict__ dst, int64_t n,
                                int64_t nx, int64_t px) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    dst[c] = (double)src[(c % nx) + px * (c / nx)];
}

#define LTRY(C, call)                                                         \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      cudaGetLastError();                                                     \
      return awc::fail((C), AWC_ERR_CUDA, cudaGetErrorString(e_));            \
    }                                                                         \
  } while (0)

struct Mem {
  std::vector<void*> p;
  ~Mem() {
    for (void* q : p) cudaFree(q);
  }
  template <typename P>
  cudaError_t get(P** out, size_t bytes) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) p.push_back(q);
    *out = (P*)q;
    return e;
  }
};

}  // namespace

extern "C" {

int awc_learned_weights_len(int32_t ndim) {
  if (ndim != 2 && ndim != 3) return 0;
  const int K = ndim == 3 ? 82 : 28;
  return kHid * K + kHid + kHid * kHid + kHid + kHid + 1;
}

int awc_forward_learned(awc_ctx* ctx, const awc_problem* p, const double* vel,
                        const uint16_t* weights_bf16, const int64_t* possrcs,
                        const double* dt2srctf, const int64_t* posrecs, double* traces,
                        double* pfinal) {
  if (!ctx) return awc::fail(nullptr, AWC_ERR_INVALID, "ctx is NULL");
  if (!p || !vel || !weights_bf16) return awc::fail(ctx, AWC_ERR_INVALID, "p/vel/weights is NULL");
  if (p->ndim != 2 && p->ndim != 3) return awc::fail(ctx, AWC_ERR_INVALID, "ndim must be 2 or 3");
  if (p->precision != AWC_F32)
    return awc::fail(ctx, AWC_ERR_INVALID, "the learned layer runs in FP32 (precision AWC_F32)");
  const int64_t nz = p->ndim == 3 ? p->nz : 1;
  const int64_t n3[3] = {p->nx, p->ny, nz};
  if (p->halo < 1 || p->halo > 8)
    return awc::fail(ctx, AWC_ERR_INVALID, "halo (the layer width) must be in [1, 8]");
  for (int a = 0; a < p->ndim; ++a)
    if (n3[a] < 2 * p->halo + 3) return awc::fail(ctx, AWC_ERR_INVALID, "grid too small for the layer");
  if (p->nt < 0 || p->nsrc < 0 || p->nrec < 0 || (p->nsrc > 0 && p->nt > 0 && !dt2srctf) ||
      (p->nsrc > 0 && !possrcs) || (p->nrec > 0 && (!posrecs || (p->nt > 0 && !traces))))
    return awc::fail(ctx, AWC_ERR_INVALID, "inconsistent sources/receivers");
  const int64_t px = (p->nx + 31) / 32 * 32, plane = px * p->ny, NP = plane * nz;
  auto node = [&](const int64_t* pos, int64_t cnt, int64_t r, int64_t* out) {
    int64_t c[3] = {pos[r] - 1, pos[r + cnt] - 1, p->ndim == 3 ? pos[r + 2 * cnt] - 1 : 0};
    for (int a = 0; a < p->ndim; ++a)
      if (c[a] < 1 || c[a] > n3[a] - 2) return false;
    *out = c[0] + px * c[1] + plane * c[2];
    return true;
  };
  std::vector<int64_t> sn(std::max<int64_t>(p->nsrc, 1)), rn(std::max<int64_t>(p->nrec, 1));
  for (int64_t s = 0; s < p->nsrc; ++s)
    if (!node(possrcs, p->nsrc, s, &sn[s]))
      return awc::fail(ctx, AWC_ERR_INVALID, "sources must be interior nodes");
  for (int64_t r = 0; r < p->nrec; ++r)
    if (!node(posrecs, p->nrec, r, &rn[r]))
      return awc::fail(ctx, AWC_ERR_INVALID, "receivers must be interior nodes");
  // the layer nodes: within `width` of the nearest absorbing side (x before
  // y before z, left before right on ties), in memory order
  std::vector<int4> lay;
  {
    const int64_t W = p->halo;
    const bool ytop = !p->freetop;
    for (int64_t k = p->ndim == 3 ? 1 : 0; k <= (p->ndim == 3 ? nz - 2 : 0); ++k)
      for (int64_t j = 1; j <= p->ny - 2; ++j) {
        const bool near = (ytop && j <= W) || j >= p->ny - 1 - W ||
                          (p->ndim == 3 && (k <= W || k >= nz - 1 - W));
        for (int64_t i = 1; i <= p->nx - 2; ++i) {
          if (!near && i > W && i < p->nx - 1 - W) i = p->nx - 1 - W;  // skip the middle
          const int64_t c[3] = {i, j, k};
          int64_t best = W + 1;
          int ax = 0, sg = 1;
          for (int a = 0; a < p->ndim; ++a) {
            const int64_t dl = c[a], dr = n3[a] - 1 - c[a];
            if (!(a == 1 && p->freetop) && dl < best) {
              best = dl;
              ax = a;
              sg = -1;
            }
            if (dr < best) {
              best = dr;
              ax = a;
              sg = 1;
            }
          }
          if (best <= W) lay.push_back(make_int4((int)i, (int)j, (int)k, 2 * ax + (sg > 0)));
        }
      }
  }
  LTRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  Mem m;
  float *buf[4], *F, *stf, *tr;
  double* stage;
  int64_t *sn_d, *rn_d;
  __nv_bfloat16* w_d;
  int4* lay_d;
  LTRY(ctx, m.get(&lay_d, std::max<size_t>(lay.size(), 1) * sizeof(int4)));
  if (!lay.empty())
    LTRY(ctx, cudaMemcpyAsync(lay_d, lay.data(), lay.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
  const int nw = awc_learned_weights_len(p->ndim);
  for (auto& b : buf) {
    LTRY(ctx, m.get(&b, NP * 4));
    LTRY(ctx, cudaMemsetAsync(b, 0, NP * 4, st));
  }
  LTRY(ctx, m.get(&F, NP * 4));
  LTRY(ctx, cudaMemsetAsync(F, 0, NP * 4, st));
  const int64_t N = p->nx * p->ny * nz;
  LTRY(ctx, m.get(&stage, std::max<int64_t>(N, p->nt * p->nrec) * 8));
  LTRY(ctx, m.get(&stf, std::max<int64_t>(p->nt * p->nsrc, 1) * 4));
  LTRY(ctx, m.get(&tr, std::max<int64_t>(p->nt * p->nrec, 1) * 4));
  LTRY(ctx, m.get(&sn_d, sn.size() * 8));
  LTRY(ctx, m.get(&rn_d, rn.size() * 8));
  LTRY(ctx, m.get(&w_d, nw * 2));
  LTRY(ctx, cudaMemcpyAsync(stage, vel, N * 8, cudaMemcpyHostToDevice, st));
  learned_fact<<<(unsigned)std::min<int64_t>((N + 255) / 256, 4096), 256, 0, st>>>(
      stage, F, p->dt * p->dt, N, p->nx, px);
  std::vector<float> rows(std::max<int64_t>(p->nt * p->nsrc, 1));
  for (int64_t s = 0; s < p->nsrc; ++s)
    for (int64_t t = 0; t < p->nt; ++t) rows[t * p->nsrc + s] = (float)dt2srctf[t + p->nt * s];
  LTRY(ctx, cudaMemcpyAsync(stf, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, st));
  LTRY(ctx, cudaMemcpyAsync(sn_d, sn.data(), sn.size() * 8, cudaMemcpyHostToDevice, st));
  LTRY(ctx, cudaMemcpyAsync(rn_d, rn.data(), rn.size() * 8, cudaMemcpyHostToDevice, st));
  LTRY(ctx, cudaMemcpyAsync(w_d, weights_bf16, nw * 2, cudaMemcpyHostToDevice, st));
  LearnedParams L{};
  L.ndim = p->ndim;
  L.nx = (int32_t)p->nx;
  L.ny = (int32_t)p->ny;
  L.nz = (int32_t)nz;
  L.width = p->halo;
  L.freetop = p->freetop;
  L.px = px;
  L.plane = plane;
  const double d[3] = {p->dx, p->dy, p->ndim == 3 ? p->dz : 1.0};
  for (int a = 0; a < 3; ++a) {
    L.inv_d2[a] = (float)(1.0 / (d[a] * d[a]));
    L.inv_d[a] = (float)(1.0 / d[a]);
  }
  L.F = F;
  L.w = w_d;
  L.nin = p->ndim == 3 ? 82 : 28;
  L.layer = lay_d;
  L.nlayer = (int32_t)lay.size();
  const unsigned lgrid = (unsigned)std::max<int64_t>(
      1, std::min<int64_t>(((int64_t)lay.size() + 16 * kWarps - 1) / (16 * kWarps),
                           (int64_t)ctx->num_sms * 6));
  const dim3 blk(32, 8);
  const dim3 grid((unsigned)((p->nx - 2 + 31) / 32), (unsigned)((p->ny - 2 + 7) / 8),
                  (unsigned)(p->ndim == 3 ? nz - 2 : 1));
  LTRY(ctx, cudaEventRecord(ctx->ev0, st));
  for (int64_t it = 0; it < p->nt; ++it) {
    L.p0 = buf[it % 4];
    L.p1 = buf[(it + 1) % 4];
    L.p2 = buf[(it + 2) % 4];
    L.p3 = buf[(it + 3) % 4];
    learned_interior<<<grid, blk, 0, st>>>(L);
    if (!lay.empty()) learned_layer<<<lgrid, 32 * kWarps, 0, st>>>(L);
    learned_io<<<1, 32, 0, st>>>(L.p3, sn_d, (int32_t)p->nsrc, stf + it * p->nsrc, rn_d,
                                 (int32_t)p->nrec, tr + it * p->nrec);
  }
  LTRY(ctx, cudaGetLastError());
  LTRY(ctx, cudaEventRecord(ctx->ev1, st));
  LTRY(ctx, cudaEventSynchronize(ctx->ev1));
  cudaEventElapsedTime(&ctx->last_run_ms, ctx->ev0, ctx->ev1);
  if (p->nt * p->nrec > 0) {
    std::vector<float> t(p->nt * p->nrec);
    LTRY(ctx, cudaMemcpyAsync(t.data(), tr, t.size() * 4, cudaMemcpyDeviceToHost, st));
    LTRY(ctx, cudaStreamSynchronize(st));
    for (int64_t r = 0; r < p->nrec; ++r)
      for (int64_t q = 0; q < p->nt; ++q) traces[q + p->nt * r] = t[q * p->nrec + r];
  }
  if (pfinal) {
    learned_unpitch<<<(unsigned)std::min<int64_t>((N + 255) / 256, 4096), 256, 0, st>>>(
        buf[(p->nt + 2) % 4], stage, N, p->nx, px);
    LTRY(ctx, cudaGetLastError());
    LTRY(ctx, cudaMemcpyAsync(pfinal, stage, N * 8, cudaMemcpyDeviceToHost, st));
  }
  LTRY(ctx, cudaStreamSynchronize(st));
  return AWC_OK;
}

}  // extern "C"
