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
// of p_t, Σ_axes D2 p_t(c), evaluated from the stored p_t in double; inside
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

template <typename T>
struct AdjParams {
  int32_t ndim, nx, ny, nz, halo;
  int64_t px, plane;
  T inv_d[3], inv_d2[3];
  const T* F;
  const T* G;     // F λ_{t+2} on the interior, 0 on the rim
  const T* lam2;  // λ_{t+2}
  const T* lam3;  // λ_{t+3}
  T* lamn;        // λ_{t+1} (may alias lam3: read and written at the same node)
  T* mu[3][2];    // μ, updated in place (layout of ψ)
  const T* nu_old[3][2];  // ν_{t+2} (layout of ξ)
  T* nu_new[3][2];        // ν_{t+1}
  const T* a[3][2];
  const T* bK[3][2];
  const T* ah[3][2];
  const T* bKh[3][2];
  int32_t active[3][2];
  int32_t off[3][2];  // band node c has entry q = c - off
};

// Element index of entry e of a band array (ψ: h+1 layers, ξ: h layers) of
// axis a at the node (i, j, k) (the node's own axis coordinate is replaced
// by e): x (layers, ny, nz); y (px, layers, nz); z (px, ny, layers).
template <typename T>
__device__ __forceinline__ int64_t band_index(const AdjParams<T>& A, int a, int layers, int e,
                                              int i, int j, int k) {
  if (a == 0) return e + (int64_t)layers * (j + (int64_t)A.ny * k);
  if (a == 1) return i + A.px * (e + (int64_t)layers * k);
  return i + A.px * (j + (int64_t)A.ny * e);
}

// a ν_{t+2} of axis a at the node whose axis coordinate is c (other
// coordinates i, j, k), when it is a band node of that axis.
template <typename T>
__device__ __forceinline__ T adj_anu(const AdjParams<T>& A, int a, int c, int i, int j, int k) {
  T g = 0;
  for (int s = 0; s < 2; ++s) {
    if (!A.active[a][s]) continue;
    const int q = c - A.off[a][s];
    if (q >= 1 && q <= A.halo)
      g += A.a[a][s][q - 1] * A.nu_old[a][s][band_index(A, a, A.halo, q - 1, i, j, k)];
  }
  return g;
}

// Whether axis coordinate c lies within one node of a band (of any side).
template <typename T>
__device__ __forceinline__ bool adj_band_near(const AdjParams<T>& A, int c, int n) {
  return A.halo > 0 && (c <= A.halo + 1 || c >= n - A.halo - 2);
}

// The band part of λ_{t+1} along axis a at node (i, j, k) whose axis
// coordinate is c: the transposed stencil of a ν_{t+2} and the ψ-face terms,
// non-zero only within one node of a band.
template <typename T>
__device__ __forceinline__ T adj_band_terms(const AdjParams<T>& A, int a, int c, int n, int i,
                                            int j, int k) {
  if (A.halo == 0 || (c > A.halo + 1 && c < n - A.halo - 2)) return T(0);
  const int di = a == 0, dj = a == 1, dk = a == 2;
  T acc = T(-2) * adj_anu(A, a, c, i, j, k);
  if (c + 1 <= n - 2) acc += adj_anu(A, a, c + 1, i + di, j + dj, k + dk);
  if (c - 1 >= 1) acc += adj_anu(A, a, c - 1, i - di, j - dj, k - dk);
  T r = A.inv_d2[a] * acc;
  for (int s = 0; s < 2; ++s) {
    if (!A.active[a][s]) continue;
    const int e1 = c - 1 - A.off[a][s], e2 = c - A.off[a][s];
    T f = 0;
    if (e1 >= 0 && e1 <= A.halo)
      f += A.ah[a][s][e1] * A.mu[a][s][band_index(A, a, A.halo + 1, e1, i, j, k)];
    if (e2 >= 0 && e2 <= A.halo)
      f -= A.ah[a][s][e2] * A.mu[a][s][band_index(A, a, A.halo + 1, e2, i, j, k)];
    r += A.inv_d[a] * f;
  }
  return r;
}

// The residuals of step t enter λ_{t+1} = R_t + 2 λ_{t+2} - λ_{t+3} + ...
// through λ_{t+3}: before adj_lambda_grad runs, λ_{t+3} -= R_t at the receiver
// nodes (one thread per node, its receivers in receiver order), so that the
// fused kernel needs no receiver lookup.
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

// Whether node (i, j, k) lies in an active CPML band of any axis (where the
// forward bracket holds ψ/ξ terms besides the Laplacian).
template <typename T>
__device__ __forceinline__ bool adj_in_band(const AdjParams<T>& A, int i, int j, int k) {
  if (A.halo == 0) return false;
  const int c[3] = {i, j, k}, n[3] = {A.nx, A.ny, A.nz};
  for (int a = 0; a < A.ndim; ++a)
    if ((A.active[a][0] && c[a] <= A.halo) || (A.active[a][1] && c[a] >= n[a] - A.halo - 1))
      return true;
  return false;
}

// λ_{t+1} = 2 λ_{t+2} - λ_{t+3} (residuals included, see adj_residuals) plus
// the transposed stencil of G = F λ_{t+2} and the band terms, one thread per
// node; then at the same node G = F λ_{t+1} for the next step and the
// gradient accumulation dJ/dF += λ_{t+1} B_t: the Laplacian of p_t outside
// the bands, (p_{t+1} - 2 p_t + p_{t-1}) / F inside them (where adj_sources
// removes the source term).
template <typename T>
__global__ void __launch_bounds__(256) adj_lambda_grad(AdjParams<T> A, T* __restrict__ Gn,
                                                       const T* __restrict__ pm1,
                                                       const T* __restrict__ p0,
                                                       const T* __restrict__ pp1,
                                                       double* __restrict__ grad) {
  const int i = 1 + blockIdx.x * 32 + threadIdx.x;
  const int j = 1 + blockIdx.y * 8 + threadIdx.y;
  const int k = A.ndim == 3 ? 1 + blockIdx.z : 0;
  if (i > A.nx - 2 || j > A.ny - 2) return;
  const int64_t px = A.px, plane = A.plane;
  const int64_t o = i + px * j + plane * k;
  const T gc = __ldg(A.G + o);
  T lam = T(2) * __ldg(A.lam2 + o) - A.lam3[o];
  lam += A.inv_d2[0] * (__ldg(A.G + o + 1) - T(2) * gc + __ldg(A.G + o - 1)) +
         A.inv_d2[1] * (__ldg(A.G + o + px) - T(2) * gc + __ldg(A.G + o - px));
  if (adj_band_near(A, i, A.nx)) lam += adj_band_terms(A, 0, i, A.nx, i, j, k);
  if (adj_band_near(A, j, A.ny)) lam += adj_band_terms(A, 1, j, A.ny, i, j, k);
  if (A.ndim == 3) {
    lam += A.inv_d2[2] * (__ldg(A.G + o + plane) - T(2) * gc + __ldg(A.G + o - plane));
    if (adj_band_near(A, k, A.nz)) lam += adj_band_terms(A, 2, k, A.nz, i, j, k);
  }
  A.lamn[o] = lam;
  const T f = __ldg(A.F + o);
  Gn[o] = f * lam;
  if (grad) {
    double b;
    if (adj_in_band(A, i, j, k)) {
      b = ((double)__ldg(pp1 + o) - 2.0 * (double)__ldg(p0 + o) + (double)__ldg(pm1 + o)) /
          (double)f;
    } else {
      const double c = __ldg(p0 + o);
      b = (double)A.inv_d2[0] * (((double)__ldg(p0 + o + 1) - 2.0 * c) + (double)__ldg(p0 + o - 1)) +
          (double)A.inv_d2[1] * (((double)__ldg(p0 + o + px) - 2.0 * c) + (double)__ldg(p0 + o - px));
      if (A.ndim == 3)
        b += (double)A.inv_d2[2] *
             (((double)__ldg(p0 + o + plane) - 2.0 * c) + (double)__ldg(p0 + o - plane));
    }
    grad[o] += (double)lam * b;
  }
}

// The active band sides of one adjoint step, for one launch over all of
// them: side n is axis ax[n], side sd[n], band nodes [start[n], start[n+1]).
struct AdjSides {
  int32_t n;
  int32_t ax[6], sd[6];
  int64_t start[7];
};

// ν_{t+1} and μ_{t+1} of every active side, one thread per band node (side,
// entry q, other coordinates): ν_{t+1}[q-1] = bK ν_{t+2}[q-1] + F λ_{t+1};
// face q (and face 0 for q = 1) of μ in place, with w of node q+1 formed from
// ν_{t+2} so that no thread reads another's new ν. Sides touch disjoint
// arrays.
template <typename T>
__global__ void __launch_bounds__(256) adj_band(AdjParams<T> A, AdjSides L) {
  const int h = A.halo;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < L.start[L.n];
       g += (int64_t)gridDim.x * blockDim.x) {
    int side = 0;
    while (side + 1 < L.n && g >= L.start[side + 1]) ++side;
    const int a = L.ax[side], s = L.sd[side];
    const int64_t t = g - L.start[side];
    const int n1 = a == 0 ? A.ny - 2 : A.nx - 2;  // fastest other coordinate count
    int q, u, v;
    if (a == 0) {  // q fastest: ψ_x is contiguous in q
      q = 1 + (int)(t % h);
      u = (int)((t / h) % n1);
      v = (int)(t / ((int64_t)h * n1));
    } else {       // x fastest
      u = (int)(t % n1);
      q = 1 + (int)((t / n1) % h);
      v = (int)(t / ((int64_t)n1 * h));
    }
    const int c = q + A.off[a][s];
    int i, j, k;
    if (a == 0) { i = c; j = 1 + u; k = A.ndim == 3 ? 1 + v : 0; }
    else if (a == 1) { i = 1 + u; j = c; k = A.ndim == 3 ? 1 + v : 0; }
    else { i = 1 + u; j = 1 + v; k = c; }
    const int64_t step = a == 0 ? 1 : a == 1 ? A.px : A.plane;
    const int64_t o = i + A.px * j + A.plane * k;
    const T flam = A.F[o] * A.lamn[o];
    const int64_t x = band_index(A, a, h, q - 1, i, j, k);
    const T nu_n = A.bK[a][s][q - 1] * A.nu_old[a][s][x] + flam;
    A.nu_new[a][s][x] = nu_n;
    const T wq = A.a[a][s][q - 1] * nu_n + flam;
    T wn = 0;
    if (q + 1 <= h) {
      const int di = a == 0, dj = a == 1, dk = a == 2;
      const T flam1 = A.F[o + step] * A.lamn[o + step];
      const T nu1 = A.bK[a][s][q] * A.nu_old[a][s][band_index(A, a, h, q, i + di, j + dj, k + dk)] +
                    flam1;
      wn = A.a[a][s][q] * nu1 + flam1;
    }
    const int64_t m = band_index(A, a, h + 1, q, i, j, k);
    A.mu[a][s][m] = A.bKh[a][s][q] * A.mu[a][s][m] + A.inv_d[a] * (wq - wn);
    if (q == 1) {
      const int64_t m0 = band_index(A, a, h + 1, 0, i, j, k);
      A.mu[a][s][m0] = A.bKh[a][s][0] * A.mu[a][s][m0] - A.inv_d[a] * wq;
    }
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
  void begin() { next = 0; }
  void release() {
    for (auto& b : blocks) cudaFree(b.first);
    blocks.clear();
    next = 0;
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

template <typename T>
// Gradient mode (grad_out set): the checkpointed forward run gives the
// traces, the misfit against `observed` and the residuals. Transpose mode
// (src_out set): `residual` are the adjoint traces.
int adjoint_impl(awc_ctx* C, awc_plan* plan, const awc_problem* p, const int64_t* possrcs,
                 const double* dt2srctf, const int64_t* posrecs, const double* residual,
                 const double* observed, double* misfit, double* traces_out, int64_t kchk,
                 double* grad_out, double* src_out) {
  const awc::PlanView V = awc::plan_view(plan);
  cudaStream_t st = V.stream;
  const int64_t nt = p->nt, nsrc = p->nsrc, nrec = p->nrec, h = p->halo;
  const int64_t NP = V.NP, fb = NP * (int64_t)sizeof(T);
  const bool want_grad = grad_out != nullptr;
  DevMem& mem = ctx_mem(C);
  // adjoint fields
  T *lam[2], *G[2], *mu[3][2] = {}, *nu[3][2][2] = {};
  for (int b = 0; b < 2; ++b) {
    ADJ_TRY(C, mem.get(&lam[b], fb));
    ADJ_TRY(C, mem.get(&G[b], fb));
    ADJ_TRY(C, cudaMemsetAsync(G[b], 0, fb, st));
  }
  for (int a = 0; a < p->ndim; ++a)
    for (int s = 0; s < 2; ++s) {
      ADJ_TRY(C, mem.get(&mu[a][s], V.psi_len[a] * sizeof(T)));
      ADJ_TRY(C, cudaMemsetAsync(mu[a][s], 0, std::max<int64_t>(V.psi_len[a], 1) * sizeof(T), st));
      for (int b = 0; b < 2; ++b) {
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
  std::vector<T> rows(std::max<int64_t>(nt * nrec, 1));
  T* res_d;
  ADJ_TRY(C, mem.get(&res_d, rows.size() * sizeof(T)));
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
  awc::AdjParams<T> A{};
  A.ndim = p->ndim;
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
  const T* cf = (const T*)V.coef;
  const int64_t n3[3] = {p->nx, p->ny, V.nz};
  for (int a = 0; a < p->ndim; ++a) {
    const T* blk = cf + a * (8 * h + 4);
    for (int s = 0; s < 2; ++s) {
      A.a[a][s] = blk + s * h;
      A.bK[a][s] = blk + 2 * h + s * h;
      A.ah[a][s] = blk + 4 * h + s * (h + 1);
      A.bKh[a][s] = blk + 4 * h + 2 * (h + 1) + s * (h + 1);
      A.active[a][s] = V.active[a][s];
      A.off[a][s] = s == 0 ? 0 : (int32_t)(n3[a] - h - 2);
      A.mu[a][s] = mu[a][s];
    }
  }
  // the active band sides, one launch per step over all of them
  awc::AdjSides sides{};
  sides.start[0] = 0;
  for (int a = 0; a < p->ndim && h > 0; ++a)
    for (int sd = 0; sd < 2; ++sd) {
      if (!A.active[a][sd]) continue;
      const int64_t n1 = a == 0 ? p->ny - 2 : p->nx - 2;
      const int64_t n2 = p->ndim == 3 ? (a == 2 ? p->ny - 2 : V.nz - 2) : 1;
      sides.ax[sides.n] = a;
      sides.sd[sides.n] = sd;
      sides.start[sides.n + 1] = sides.start[sides.n] + h * n1 * n2;
      ++sides.n;
    }
  const unsigned band_blocks =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>((sides.start[sides.n] + 255) / 256,
                                                       (int64_t)C->num_sms * 8));
  const dim3 blk(32, 8);
  const dim3 grid((unsigned)((p->nx - 2 + 31) / 32), (unsigned)((p->ny - 2 + 7) / 8),
                  (unsigned)(p->ndim == 3 ? V.nz - 2 : 1));
  // checkpoints and segment fields (gradient only)
  const int64_t nseg = want_grad ? (nt + kchk - 1) / kchk : 0;
  int64_t band_elems = 0;
  for (int a = 0; a < p->ndim; ++a) band_elems += 2 * (V.psi_len[a] + V.xi_len[a]);
  std::vector<T*> chk(nseg, nullptr);
  std::vector<T*> seg;
  if (want_grad) {
    // one allocation for the saved states and the segment's fields
    const int64_t chk_elems = (3 * NP + band_elems + 63) / 64 * 64;
    seg.resize(std::min<int64_t>(kchk, nt) + 2);
    T* arena;
    ADJ_TRY(C, mem.get(&arena, (nseg * chk_elems + (int64_t)seg.size() * NP) * sizeof(T)));
    for (int64_t c = 0; c < nseg; ++c) chk[c] = arena + c * chk_elems;
    for (size_t m = 0; m < seg.size(); ++m) seg[m] = arena + nseg * chk_elems + (int64_t)m * NP;
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
  std::vector<double> res_h;
  if (want_grad) {
    // forward run with checkpoints, then the traces, misfit and residuals
    if ((rc = awc_plan_reset(plan))) return rc;
    for (int64_t c = 0; c < nseg; ++c) {
      const int64_t s = c * kchk;
      if ((rc = save_or_restore(chk[c], s, true))) return rc;
      if ((rc = awc_plan_run(plan, std::min(kchk, nt - s), 0, nullptr))) return rc;
    }
    res_h.assign(std::max<int64_t>(nt * nrec, 1), 0.0);
    if (nt * nrec > 0 && (rc = awc_plan_traces(plan, res_h.data()))) return rc;
    if (traces_out && nt * nrec > 0) std::memcpy(traces_out, res_h.data(), nt * nrec * sizeof(double));
    double J = 0.0;
    for (int64_t c = 0; c < nt * nrec; ++c) {
      res_h[c] -= observed[c];
      J += 0.5 * res_h[c] * res_h[c];
    }
    *misfit = J;
    residual = res_h.data();
  }
  for (int64_t r = 0; r < nrec; ++r)
    for (int64_t t = 0; t < nt; ++t) rows[t * nrec + r] = (T)residual[t + nt * r];
  ADJ_TRY(C, cudaMemcpyAsync(res_d, rows.data(), rows.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  // backward
  int i2 = 0, i3 = 1;  // lam[i2] = λ_{t+2}, lam[i3] = λ_{t+3}
  int gi = 0;          // G[gi] = F λ_{t+2}
  int par = 0;         // nu[..][par] holds ν_{t+2}
  for (int64_t c = (want_grad ? nseg : 1) - 1; c >= 0; --c) {
    const int64_t s = want_grad ? c * kchk : 0, e = want_grad ? std::min(s + kchk, nt) : nt;
    if (want_grad) {
      // recompute p_{s-1} .. p_e of the segment
      if ((rc = save_or_restore(chk[c], s, false))) return rc;
      awc::plan_set_step(plan, s);
      ADJ_TRY(C, cudaMemcpyAsync(seg[0], V.buf[s % 3], fb, cudaMemcpyDeviceToDevice, st));
      ADJ_TRY(C, cudaMemcpyAsync(seg[1], V.buf[(s + 1) % 3], fb, cudaMemcpyDeviceToDevice, st));
      awc::plan_keep_fields(plan, (void* const*)(seg.data() + 2), s, e - s);
      rc = awc_plan_run(plan, e - s, 0, nullptr);
      awc::plan_keep_fields(plan, nullptr, 0, 0);
      if (rc) return rc;
    }
    for (int64_t t = e - 1; t >= s; --t) {
      // λ_{t+1} overwrites λ_{t+3}: adj_lambda_grad reads λ_{t+3} only at the
      // node it writes
      T* ln = lam[i3];
      A.lam2 = lam[i2];
      A.lam3 = lam[i3];
      A.lamn = ln;
      A.G = G[gi];
      for (int a = 0; a < p->ndim; ++a)
        for (int sd = 0; sd < 2; ++sd) {
          A.nu_old[a][sd] = nu[a][sd][par];
          A.nu_new[a][sd] = nu[a][sd][par ^ 1];
        }
      if (!RG.node.empty())
        awc::adj_residuals<T><<<(unsigned)((RG.node.size() + 127) / 128), 128, 0, st>>>(
            ln, rnode_d, roff_d, rids_d, (int32_t)RG.node.size(), res_d + t * nrec);
      const T* pm1 = want_grad ? seg[t - s] : nullptr;
      const T* p0 = want_grad ? seg[t - s + 1] : nullptr;
      const T* pp1 = want_grad ? seg[t - s + 2] : nullptr;
      awc::adj_lambda_grad<T><<<grid, blk, 0, st>>>(A, G[gi ^ 1], pm1, p0, pp1, grad);
      if (nsrc > 0)
        awc::adj_sources<T><<<1, 32, 0, st>>>(ln, A.F, snode_d, sband_d, (int32_t)nsrc,
                                              stf_d + t * nsrc, grad,
                                              sout_d ? sout_d + t * nsrc : nullptr);
      if (sides.n > 0) awc::adj_band<T><<<band_blocks, 256, 0, st>>>(A, sides);
      ADJ_TRY(C, cudaGetLastError());
      std::swap(i2, i3);  // λ_{t+1} is the next step's λ_{t+2}
      par ^= 1;
      gi ^= 1;
    }
  }
  // outputs
  if (want_grad) {
    double* dense;
    const int64_t N = p->nx * p->ny * V.nz;
    ADJ_TRY(C, mem.get(&dense, N * sizeof(double)));
    const int blocks = (int)std::min<int64_t>((N + 255) / 256, (int64_t)C->num_sms * 16);
    awc::scale_unpitch<<<blocks, 256, 0, st>>>(grad, dense, N, p->nx, V.px, p->dt * p->dt);
    ADJ_TRY(C, cudaGetLastError());
    ADJ_TRY(C, cudaMemcpyAsync(grad_out, dense, N * sizeof(double), cudaMemcpyDeviceToHost, st));
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
  ADJ_TRY(C, cudaStreamSynchronize(st));
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
  if ((rc = awc::plan_for(ctx, &ctx->adj_plan, p, vel, coeffs, possrcs, dt2srctf, posrecs)))
    return rc;
  awc_plan* plan = ctx->adj_plan;
  rc = p->precision == AWC_F64
           ? adjoint_impl<double>(ctx, plan, p, possrcs, dt2srctf, posrecs, nullptr, observed,
                                  misfit, traces, checkpoint_every, grad_c2, nullptr)
           : adjoint_impl<float>(ctx, plan, p, possrcs, dt2srctf, posrecs, nullptr, observed,
                                 misfit, traces, checkpoint_every, grad_c2, nullptr);
  return rc;
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
           ? adjoint_impl<double>(ctx, plan, p, possrcs, nullptr, posrecs, adjoint_traces,
                                  nullptr, nullptr, nullptr, 1, nullptr, src_out)
           : adjoint_impl<float>(ctx, plan, p, possrcs, nullptr, posrecs, adjoint_traces,
                                 nullptr, nullptr, nullptr, 1, nullptr, src_out);
  return rc;
}

}  // extern "C"
