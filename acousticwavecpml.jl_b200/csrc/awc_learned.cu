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
constexpr int kMaxIn = 82;

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
};

__device__ __forceinline__ bool interior_node(const LearnedParams& L, int i, int j, int k) {
  return i >= 1 && i <= L.nx - 2 && j >= 1 && j <= L.ny - 2 &&
         (L.ndim == 2 || (k >= 1 && k <= L.nz - 2));
}

// Depth (1 = next to the rim) of the nearest absorbing side and its axis and
// outward sign, or 0 when the node is not in the layer.
__device__ __forceinline__ int layer_side(const LearnedParams& L, int i, int j, int k, int& axis,
                                          int& sign) {
  const int c[3] = {i, j, k};
  const int n[3] = {L.nx, L.ny, L.nz};
  int best = L.width + 1;
  for (int a = 0; a < L.ndim; ++a) {
    const int dl = c[a], dr = n[a] - 1 - c[a];
    const bool left_abs = !(a == 1 && L.freetop);
    if (left_abs && dl < best) {
      best = dl;
      axis = a;
      sign = -1;
    }
    if (dr < best) {
      best = dr;
      axis = a;
      sign = 1;
    }
  }
  return best <= L.width ? best : 0;
}

__global__ void __launch_bounds__(256) learned_interior(LearnedParams L) {
  const int i = 1 + blockIdx.x * 32 + threadIdx.x;
  const int j = 1 + blockIdx.y * 8 + threadIdx.y;
  const int k = L.ndim == 3 ? 1 + blockIdx.z : 0;
  if (i > L.nx - 2 || j > L.ny - 2) return;
  int ax, sg;
  if (layer_side(L, i, j, k, ax, sg)) return;
  const int64_t o = i + L.px * j + L.plane * k;
  const float pc = L.p2[o];
  float lap = (L.p2[o + 1] - 2.f * pc + L.p2[o - 1]) * L.inv_d2[0] +
              (L.p2[o + L.px] - 2.f * pc + L.p2[o - L.px]) * L.inv_d2[1];
  if (L.ndim == 3) lap += (L.p2[o + L.plane] - 2.f * pc + L.p2[o - L.plane]) * L.inv_d2[2];
  L.p3[o] = fmaf(L.F[o], lap, 2.f * pc - L.p1[o]);
}

// One thread per interior node; layer nodes run the MLP. The weights are
// staged in shared memory as floats.
__global__ void __launch_bounds__(256) learned_layer(LearnedParams L) {
  __shared__ float w[kHid * kMaxIn + kHid + kHid * kHid + kHid + kHid + 1];
  const int K = L.nin;
  const int nw = kHid * K + kHid + kHid * kHid + kHid + kHid + 1;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  for (int e = tid; e < nw; e += blockDim.x * blockDim.y) w[e] = __bfloat162float(L.w[e]);
  __syncthreads();
  const float* W1 = w;
  const float* b1 = W1 + kHid * K;
  const float* W2 = b1 + kHid;
  const float* b2 = W2 + kHid * kHid;
  const float* W3 = b2 + kHid;
  const float b3 = W3[kHid];
  const int i = 1 + blockIdx.x * 32 + threadIdx.x;
  const int j = 1 + blockIdx.y * 8 + threadIdx.y;
  const int k = L.ndim == 3 ? 1 + blockIdx.z : 0;
  if (i > L.nx - 2 || j > L.ny - 2) return;
  int ax = 0, sg = 1;
  if (!layer_side(L, i, j, k, ax, sg)) return;
  // the two transverse axes in increasing order
  int t1 = -1, t2 = -1;
  for (int a = 0; a < L.ndim; ++a)
    if (a != ax) (t1 < 0 ? t1 : t2) = a;
  float x[kMaxIn];
  float s = 0.f;
  const float* lv[3] = {L.p0, L.p1, L.p2};
  const int nv = L.ndim == 3 ? 3 : 1;
  int f = 0;
  for (int l = 0; l < 3; ++l)
    for (int u = -1; u <= 1; ++u)
      for (int v = -1; v <= 1; ++v)
        for (int q = 0; q < nv; ++q) {
          const int wq = L.ndim == 3 ? q - 1 : 0;
          int d[3] = {0, 0, 0};
          d[ax] = sg * u;
          d[t1] = v;
          if (t2 >= 0) d[t2] = wq;
          const int ii = i + d[0], jj = j + d[1], kk = k + d[2];
          float val = 0.f;
          if (interior_node(L, ii, jj, kk)) val = lv[l][ii + L.px * jj + L.plane * kk];
          x[f++] = val;
          s = fmaxf(s, fabsf(val));
        }
  const float inv = s > 0.f ? 1.f / s : 1.f;
  for (int c = 0; c < f; ++c) x[c] *= inv;
  x[f] = sqrtf(L.F[i + L.px * j + L.plane * k]) * L.inv_d[ax];  // Courant number
  float h1[kHid];
#pragma unroll 4
  for (int r = 0; r < kHid; ++r) {
    float acc = b1[r];
    for (int c = 0; c < K; ++c) acc = fmaf(W1[r * K + c], x[c], acc);
    h1[r] = fmaxf(acc, 0.f);
  }
  float out = b3;
#pragma unroll 4
  for (int r = 0; r < kHid; ++r) {
    float acc = b2[r];
#pragma unroll
    for (int c = 0; c < kHid; ++c) acc = fmaf(W2[r * kHid + c], h1[c], acc);
    out = fmaf(W3[r], fmaxf(acc, 0.f), out);
  }
  L.p3[i + L.px * j + L.plane * k] = out * (s > 0.f ? s : 1.f);
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
  LTRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  Mem m;
  float *buf[4], *F, *stf, *tr;
  double* stage;
  int64_t *sn_d, *rn_d;
  __nv_bfloat16* w_d;
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
    learned_layer<<<grid, blk, 0, st>>>(L);
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
