// awc_api.cu — host side of the C ABI declared in include/awcpml.h.
//
// Responsibilities: argument validation with the reference's error cases
// (positions inside the model, src/shared/acoustic_3D_xPU.jl:281,289; halo
// small enough for the band index arithmetic of :12,:68), the FP64 CPML
// coefficient setup (src/utils.jl:19-57), device buffers, the per-step launch
// sequence of forward! (:124-167), its capture into CUDA graphs, and the
// launch-shape autotuner.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/awcpml.h"
#include "awc_ctx.h"
#include "awc_kernels.cuh"
#include "awc_tb.cuh"

namespace {

thread_local std::string g_thread_err;

int set_err(std::string* dst, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_thread_err = buf;
  if (dst) *dst = buf;
  return code;
}

#define CUDA_TRY(dst, call)                                                              \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      return set_err(dst, e_ == cudaErrorMemoryAllocation ? AWC_ERR_OOM : AWC_ERR_CUDA,  \
                     "%s failed: %s", #call, cudaGetErrorString(e_));                    \
    }                                                                                    \
  } while (0)

// CPML profile restated from calc_Kab_CPML (src/utils.jl:19-57), FP64.
void kab(int32_t halo, double dt, double npower, double d0, double alpha_max, double K_max,
         bool halfgrid, double* a_l, double* a_r, double* bK_l, double* bK_r) {
  const int64_t n = halo + (halfgrid ? 1 : 0);
  if (n == 0) return;
  const double shift = halfgrid ? 0.5 : 0.0;
  std::vector<double> dist(n);
  // LinRange(0-shift, n-shift-1, n): element j = (1-t)*start + t*stop, t = j/(n-1)
  const double lo = 0.0 - shift, hi = (double)n - shift - 1.0;
  for (int64_t j = 0; j < n; ++j) {
    if (n == 1) {
      dist[j] = lo;
    } else {
      const double t = (double)j / (double)(n - 1);
      dist[j] = (1.0 - t) * lo + t * hi;
    }
  }
  if (halfgrid) dist[0] = 0.0;  // the staggered profile starts on the edge node
  auto powN = [npower](double x) { return npower == 2.0 ? x * x : std::pow(x, npower); };
  for (int64_t m = 0; m < n; ++m) {
    for (int side = 0; side < 2; ++side) {
      // left side reads the distance profile reversed
      const double r = (side == 0 ? dist[n - 1 - m] : dist[m]) / (double)halo;
      const double rN = powN(r);
      const double d = d0 * rN;
      const double alpha = alpha_max * (1.0 - r);
      const double K = 1.0 + (K_max - 1.0) * rN;
      const double b = std::exp(-(d / K + alpha) * dt);
      const double a = d * (b - 1.0) / (K * (d + K * alpha));
      (side == 0 ? a_l : a_r)[m] = a;
      (side == 0 ? bK_l : bK_r)[m] = b / K;
    }
  }
}

// lifted1d: p is the three-row form of a 1D problem, whose y axis carries no
// CPML (its halo is not bounded by ny).
int validate(const awc_problem* p, std::string* err, bool lifted1d = false) {
  if (!p) return set_err(err, AWC_ERR_INVALID, "problem is NULL");
  if (p->ndim != 2 && p->ndim != 3)
    return set_err(err, AWC_ERR_INVALID, "ndim must be 2 or 3 (got %d)", p->ndim);
  if (p->precision != AWC_F32 && p->precision != AWC_F64)
    return set_err(err, AWC_ERR_INVALID, "precision must be AWC_F32 or AWC_F64");
  const int64_t n[3] = {p->nx, p->ny, p->ndim == 3 ? p->nz : 3};
  for (int a = 0; a < p->ndim; ++a) {
    if (n[a] < 3 || n[a] > (int64_t)1 << 30)
      return set_err(err, AWC_ERR_INVALID, "grid size along axis %d must be in [3, 2^30]", a);
  }
  if (p->ndim == 2 && p->nz != 1) return set_err(err, AWC_ERR_INVALID, "2D problems need nz = 1");
  if (p->halo < 0) return set_err(err, AWC_ERR_INVALID, "halo must be >= 0");
  for (int a = 0; a < p->ndim; ++a) {
    if (lifted1d && a == 1) continue;
    // right-band ψ reads pcur[i + n - halo - 2] for i = 1 (acoustic_3D_xPU.jl:12)
    if (p->halo > n[a] - 2)
      return set_err(err, AWC_ERR_INVALID, "halo %d too large for %lld nodes on axis %d",
                     p->halo, (long long)n[a], a);
  }
  const double d[3] = {p->dx, p->dy, p->ndim == 3 ? p->dz : 1.0};
  for (int a = 0; a < p->ndim; ++a)
    if (!(d[a] > 0.0) || !std::isfinite(d[a]))
      return set_err(err, AWC_ERR_INVALID, "grid spacing must be positive and finite");
  if (!(p->dt > 0.0) || !std::isfinite(p->dt))
    return set_err(err, AWC_ERR_INVALID, "dt must be positive and finite");
  if (p->nt < 0 || p->nt > ((int64_t)1 << 31))
    return set_err(err, AWC_ERR_INVALID, "nt out of range");
  if (p->nsrc < 0 || p->nrec < 0 || p->nsrc > (1 << 30) || p->nrec > (1 << 30))
    return set_err(err, AWC_ERR_INVALID, "nsrc/nrec out of range");
  return AWC_OK;
}

int check_positions(const awc_problem* p, const int64_t* pos, int64_t cnt, const char* what,
                    std::string* err) {
  if (cnt > 0 && !pos) return set_err(err, AWC_ERR_INVALID, "%s positions are NULL", what);
  const int64_t n[3] = {p->nx, p->ny, p->nz};
  for (int64_t s = 0; s < cnt; ++s)
    for (int a = 0; a < p->ndim; ++a) {
      const int64_t v = pos[s + cnt * a];
      if (v < 1 || v > n[a])
        return set_err(err, AWC_ERR_INVALID, "At least one %s is not inside the model!", what);
    }
  return AWC_OK;
}

// A 1D problem (the reference's solve1D, src/shared/acoustic_1D.jl:7-89)
// runs as the 2D problem of three rows whose middle row is the line: the
// outer rows are Dirichlet rim (never updated, zero), the y spacing enters
// with zero inverse (plan flag is1d), and the y CPML block is the trivial
// one (a = 0, b/K = 1), so every node of the line takes exactly the 1D
// update: pnew = 2 pcur - pold + fact (d2x + 0) + damp_x.
struct Lifted {
  awc_problem p{};
  std::vector<double> vel, coeffs;
  std::vector<int64_t> possrcs, posrecs;
};

int validate_1d(const awc_problem* p, std::string* err) {
  if (p->ny != 1 || p->nz != 1) return set_err(err, AWC_ERR_INVALID, "1D problems need ny = nz = 1");
  awc_problem q = *p;
  q.ndim = 2;
  q.ny = 3;
  q.dy = p->dx;
  return validate(&q, err, true);
}

void lift_1d(const awc_problem* p, const double* vel, const double* coeffs, const int64_t* possrcs,
             const int64_t* posrecs, Lifted* L) {
  const int64_t nx = p->nx, h = p->halo;
  L->p = *p;
  L->p.ndim = 2;
  L->p.ny = 3;
  L->p.nz = 1;
  L->p.dy = p->dx;  // its inverse is replaced by 0 (awc_plan.is1d)
  L->p.freetop = 0;
  L->vel.assign(3 * nx, 0.0);
  for (int r = 0; r < 3; ++r)
    for (int64_t i = 0; i < nx; ++i) L->vel[i + nx * r] = vel ? vel[i] : 0.0;
  L->coeffs.assign(2 * (8 * h + 4), 0.0);
  if (coeffs) std::copy(coeffs, coeffs + 8 * h + 4, L->coeffs.begin());
  double* yb = L->coeffs.data() + 8 * h + 4;  // y block: a = 0, b/K = 1
  for (int64_t m = 0; m < 2 * h; ++m) yb[2 * h + m] = 1.0;
  for (int64_t m = 0; m < 2 * (h + 1); ++m) yb[4 * h + 2 * (h + 1) + m] = 1.0;
  auto lift_pos = [](const int64_t* pos, int64_t n, std::vector<int64_t>& out) {
    out.assign(2 * std::max<int64_t>(n, 1), 2);
    for (int64_t s = 0; s < n; ++s) out[s] = pos ? pos[s] : 0;
  };
  lift_pos(possrcs, p->nsrc, L->possrcs);
  lift_pos(posrecs, p->nrec, L->posrecs);
}

// Row pitch of the field arrays: nx rounded up to 32 elements.
int64_t pitch_of(int64_t nx) { return (nx + 31) / 32 * 32; }

// Pitched linear index of item s of a 1-based (cnt x ndim) position array.
int64_t node_of(const awc_problem* p, int64_t px, const int64_t* pos, int64_t cnt, int64_t s) {
  const int64_t i = pos[s] - 1, j = pos[s + cnt] - 1, k = p->ndim == 3 ? pos[s + 2 * cnt] - 1 : 0;
  return i + px * (j + p->ny * k);
}

// Pipeline depth of the 3D core kernel: S stages let the TMA loads run S-3
// planes ahead of the plane being computed. Five stages (two planes ahead)
// measured best with the 64 x 4 tiles the autotuner picks on large grids:
// 131.6 us per step at 296 x 276 x 296 against 132.4 us with four stages and
// 131.6 us with six (more stages mean larger blocks, fewer per SM).
template <typename T>
constexpr int stages() { return 5; }

// Where the fields and the CPML state of the current step live. ord[0] is
// the buffer of the newest pressure field p_s, ord[1] of p_{s-1}, ord[2] of
// p_{s-2}, ord[3] the fourth buffer (3D plans). A one-step launch reads
// ord[1], ord[0] and writes ord[2] (the reference's three-buffer rotation,
// forward! at acoustic_3D_xPU.jl:166, which sources on the Dirichlet rim rely
// on); a two-step pass reads ord[1], ord[0] and writes ord[2], ord[3]. ψ_s is
// psi[..][psi_par]; ξ_s is xi (xi_par 0) or xi_alt (1).
struct StepState {
  int8_t ord[4] = {1, 0, 2, 3};
  int8_t psi_par = 0, xi_par = 0;
  void step1() {
    const int8_t o[4] = {ord[2], ord[0], ord[1], ord[3]};
    std::memcpy(ord, o, 4);
    psi_par ^= 1;
  }
  void pass2() {
    const int8_t o[4] = {ord[3], ord[2], ord[0], ord[1]};
    std::memcpy(ord, o, 4);
    psi_par ^= 1;
    xi_par ^= 1;
  }
  // the state after `it` one-step launches from the initial one
  static StepState after_steps(int64_t it) {
    StepState s;
    s.ord[0] = (int8_t)((it + 1) % 3);
    s.ord[1] = (int8_t)(it % 3);
    s.ord[2] = (int8_t)((it + 2) % 3);
    s.psi_par = (int8_t)(it & 1);
    return s;
  }
  int code() const {
    return ord[0] | ord[1] << 2 | ord[2] << 4 | ord[3] << 6 | psi_par << 8 | xi_par << 9;
  }
};

}  // namespace

struct awc_plan {
  awc_ctx* ctx = nullptr;
  awc_problem p{};
  size_t esz = 0;  // bytes per element of T
  int64_t N = 0;   // nodes (dense count)
  int64_t px = 0;  // field row pitch (elements)
  int64_t NP = 0;  // pitched field length
  int64_t psi_side[3] = {}, xi_side[3] = {};  // right side's ψ / ξ offset from the left's (elements)
  // device buffers
  void* buf[4] = {nullptr, nullptr, nullptr, nullptr};  // 4th: 3D plans only
  int32_t nbuf = 3;
  void* fact = nullptr;
  void* psi[3][2][2] = {};  // [axis][side][old/new parity]
  void* xi[3][2] = {};
  void* xi_alt[3][2] = {};  // 3D: the second ξ array of two-step passes
  void* coef = nullptr;  // packed coefficients in T
  int32_t* err_flag = nullptr;
  // sources and receivers: groups per node (CSR), the nodes themselves, and
  // their layout for the current launch shape (see awc::Io)
  int32_t* src_off = nullptr;
  int32_t* src_ids = nullptr;
  int32_t* rec_off = nullptr;
  int32_t* rec_ids = nullptr;
  std::vector<awc::IoRim> io_nodes;  // host copy: node, source group, receiver group
  struct IoSet {                     // one kernel's per-block source/receiver lists
    int32_t* blk_off = nullptr;
    int64_t cap = 0;
    int4* ent = nullptr;
    int64_t ecap = 0;
    int32_t do_rim = 0;
  } io_k[2];                         // [0] 3D core or 2D kernel, [1] 3D shell kernel
  awc::IoRim* io_rim = nullptr;
  int32_t io_nrim = 0;
  uint64_t io_shape = ~0ull;  // launch shape io_* were built for
  // 3D regions: the band-free core box and the shell boxes around it
  bool has_core = false;
  awc::Box core{};
  int32_t core_x = 0;
  int32_t nbox = 0;
  awc::Box box[6] = {};
  int32_t box_blk[7] = {};
  int32_t szc = 10;  // z planes per block of the band kernel
  void* stf = nullptr;     // [nt][nsrc]
  void* traces = nullptr;  // [nt][nrec]
  double* staging = nullptr;
  int64_t staging_len = 0;
  double* snap_staging = nullptr;  // two unpitched fields for snapshot runs (lazily allocated)
  std::vector<void*> allocs;
  // launch shape of the 3D core kernel: tile rows (4, 8, 16; the tile is
  // 64 x by nodes, 32 x by/2 threads) and z planes per block
  int32_t by = 8, zchunk = 1;
  CUtensorMap map_c[4], map_o[4], map_f;
  int32_t maps_by = 0;  // tile height the tensor maps were encoded for
  // two-step passes (awc_tb.cuh): depth 2 advances two steps per pass
  int32_t depth = 1;
  int32_t tb_nch = 1;        // z chunks per column tile
  int32_t tb_zc = 1;         // planes per chunk
  int32_t tb_ntiles[2] = {};  // [0] Z tiles, [1] XY tiles
  int2* tb_tiles[2] = {};
  int64_t tb_tiles_cap[2] = {};
  IoSet tb_io[2];
  uint64_t tb_io_shape = ~0ull;
  int32_t tb_rows = 16;      // rows of the level-1 region (8 or 16)
  CUtensorMap tb_map_pt[4], tb_map_in[4], tb_map_f;
  int32_t tb_maps_rows = 0;  // rows the tensor maps were encoded for
  int32_t wait_rounds = 4096, wait_ns = 1000000, withhold = -1;
  bool is1d = false;  // a 1D problem lifted to three rows (see Lifted)
  // run state
  int64_t step = 0;
  StepState state;
  int32_t active[3][2] = {};
  // captured runs, by (first step, steps, state code at the first step,
  // first kept step, hash of the kept-field destinations; 0 without)
  std::map<std::array<int64_t, 5>, cudaGraphExec_t> graphs;
  // Everything the captured kernel parameters hold by value besides the grid
  // shape and the fixed device buffers: the graphs are reused while it is
  // unchanged (a new shot of the same shape re-uploads data only).
  struct GraphKey {
    uint64_t launch = ~0ull;
    int32_t active[3][2] = {};
    double d[3] = {};
    int32_t nrim = -1, do_rim[2] = {};
    const void* blk_off[4] = {};  // one-step core/shell, two-step Z/XY
    const void* tiles[2] = {};
    int32_t wait[3] = {};
    bool operator==(const GraphKey& o) const {
      if (launch != o.launch || nrim != o.nrim || do_rim[0] != o.do_rim[0] ||
          do_rim[1] != o.do_rim[1])
        return false;
      for (int w = 0; w < 4; ++w)
        if (blk_off[w] != o.blk_off[w]) return false;
      for (int w = 0; w < 2; ++w)
        if (tiles[w] != o.tiles[w]) return false;
      for (int w = 0; w < 3; ++w)
        if (wait[w] != o.wait[w]) return false;
      for (int a = 0; a < 3; ++a) {
        if (d[a] != o.d[a]) return false;
        for (int s = 0; s < 2; ++s)
          if (active[a][s] != o.active[a][s]) return false;
      }
      return true;
    }
  } graph_key;
  // fields to keep: the new field of step it in [keep_first, keep_first +
  // keep_count) goes to keep[it - keep_first] (set by the adjoint's forward
  // run and segment recompute). Copied after the step, or, with keep_in_place,
  // written there by the step itself, which then reads p_{it-1} and p_it from
  // keep[m - 2] and keep[m - 1] (m = it - keep_first; keep[-2] and keep[-1]
  // hold the fields before the range), the plan's buffers refreshed after
  // the range's last step.
  void* const* keep = nullptr;
  int64_t keep_first = 0, keep_count = 0;
  bool keep_in_place = false;

  int alloc(void** out, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(out, bytes);
    if (e != cudaSuccess) {
      *out = nullptr;
      cudaGetLastError();
      return set_err(&ctx->err, e == cudaErrorMemoryAllocation ? AWC_ERR_OOM : AWC_ERR_CUDA,
                     "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    allocs.push_back(*out);
    return AWC_OK;
  }
  void release(void* ptr) {
    if (!ptr) return;
    auto f = std::find(allocs.begin(), allocs.end(), ptr);
    if (f != allocs.end()) allocs.erase(f);
    cudaFree(ptr);
  }
  void drop_graphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
  }
  ~awc_plan() {
    drop_graphs();
    for (void* a : allocs) cudaFree(a);
  }
};

namespace awc {
namespace {
// A host buffer is pinned when the runtime knows it as host memory.
bool is_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}
// memcpy split over up to 8 threads (one 8 MB slice per thread at least).
void host_copy(void* dst, const void* src, size_t bytes) {
  const size_t nth = std::max<size_t>(
      1, std::min<size_t>({8, (size_t)std::max(1u, std::thread::hardware_concurrency()),
                           bytes / (8u << 20)}));
  if (nth == 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  std::vector<std::thread> th;
  const size_t chunk = (bytes + nth - 1) / nth;
  for (size_t t = 0; t < nth; ++t) {
    const size_t a = t * chunk, b = std::min(bytes, a + chunk);
    if (a >= b) break;
    th.emplace_back([=]() { std::memcpy((char*)dst + a, (const char*)src + a, b - a); });
  }
  for (auto& x : th) x.join();
}
cudaError_t stage(awc_ctx* C, size_t bytes) {
  if (C->host_stage_bytes >= bytes) return cudaSuccess;
  if (C->host_stage) cudaFreeHost(C->host_stage);
  C->host_stage = nullptr;
  C->host_stage_bytes = 0;
  cudaError_t e = cudaMallocHost(&C->host_stage, bytes);
  if (e == cudaSuccess) C->host_stage_bytes = bytes;
  return e;
}
constexpr size_t kStageMin = 16u << 20;  // smaller copies go directly
}  // namespace

cudaError_t copy_to_device(awc_ctx* C, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  cudaError_t e;
  if (bytes < kStageMin || is_pinned(src) || stage(C, bytes) != cudaSuccess) {
    cudaGetLastError();
    e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  } else {
    host_copy(C->host_stage, src, bytes);
    e = cudaMemcpyAsync(dst, C->host_stage, bytes, cudaMemcpyHostToDevice, st);
  }
  return e != cudaSuccess ? e : cudaStreamSynchronize(st);
}

cudaError_t copy_to_host(awc_ctx* C, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes < kStageMin || is_pinned(dst) || stage(C, bytes) != cudaSuccess) {
    cudaGetLastError();
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
    return e != cudaSuccess ? e : cudaStreamSynchronize(st);
  }
  cudaError_t e = cudaMemcpyAsync(C->host_stage, src, bytes, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) host_copy(dst, C->host_stage, bytes);
  return e;
}
}  // namespace awc

namespace {

// Elements of one band layer of axis `axis`: ψ/ξ of axis x are
// (halo[+1], ny, nz); those of axes y and z are pitched like the fields,
// (px, halo[+1], nz) and (px, ny, halo[+1]).
int64_t cross_section(const awc_problem* p, int axis) {
  const int64_t nz = p->ndim == 3 ? p->nz : 1, px = pitch_of(p->nx);
  return axis == 0 ? p->ny * nz : axis == 1 ? px * nz : px * p->ny;
}

// Elements from the left side's ψ or ξ array of an axis to the right side's:
// the left array's length rounded up to 64 elements (256-byte aligned starts).
int64_t side_stride(int64_t len) { return (len + 63) / 64 * 64; }

// Allocates every device buffer of a plan (shape only, contents undefined).
int plan_alloc(awc_plan* P) {
  const awc_problem* p = &P->p;
  const int64_t h = p->halo;
  P->esz = p->precision == AWC_F64 ? 8 : 4;
  const int64_t nz = p->ndim == 3 ? p->nz : 1;
  P->N = p->nx * p->ny * nz;
  P->px = pitch_of(p->nx);
  P->NP = P->px * p->ny * nz;
  int rc;
  P->nbuf = p->ndim == 3 ? 4 : 3;
  for (int b = 0; b < P->nbuf; ++b)
    if ((rc = P->alloc(&P->buf[b], P->NP * P->esz))) return rc;
  if ((rc = P->alloc(&P->fact, P->NP * P->esz))) return rc;
  // ψ (each parity) and ξ of an axis: one allocation per array kind, the
  // right side's array at a fixed offset after the left side's (the 3D band
  // kernel addresses both sides from the left base)
  for (int a = 0; a < p->ndim; ++a) {
    const int64_t cs = cross_section(p, a);
    P->psi_side[a] = side_stride((h + 1) * cs);
    P->xi_side[a] = side_stride(h * cs);
    for (int par = 0; par < 2; ++par) {
      void* base = nullptr;
      if ((rc = P->alloc(&base, 2 * P->psi_side[a] * P->esz))) return rc;
      P->psi[a][0][par] = base;
      P->psi[a][1][par] = (char*)base + P->psi_side[a] * P->esz;
    }
    void* base = nullptr;
    if ((rc = P->alloc(&base, 2 * P->xi_side[a] * P->esz))) return rc;
    P->xi[a][0] = base;
    P->xi[a][1] = (char*)base + P->xi_side[a] * P->esz;
    if (p->ndim == 3) {
      if ((rc = P->alloc(&base, 2 * P->xi_side[a] * P->esz))) return rc;
      P->xi_alt[a][0] = base;
      P->xi_alt[a][1] = (char*)base + P->xi_side[a] * P->esz;
    }
  }
  if ((rc = P->alloc(&P->coef, awc_coeffs_len(p) * P->esz))) return rc;
  if ((rc = P->alloc((void**)&P->err_flag, 4))) return rc;
  const int64_t ns = std::max<int64_t>(p->nsrc, 1), nr = std::max<int64_t>(p->nrec, 1);
  if ((rc = P->alloc((void**)&P->src_off, (ns + 1) * 4))) return rc;
  if ((rc = P->alloc((void**)&P->src_ids, ns * 4))) return rc;
  if ((rc = P->alloc((void**)&P->rec_off, (nr + 1) * 4))) return rc;
  if ((rc = P->alloc((void**)&P->rec_ids, nr * 4))) return rc;
  for (int kk = 0; kk < 2; ++kk)
    if ((rc = P->alloc((void**)&P->io_k[kk].ent, (ns + nr) * sizeof(int4)))) return rc;
  if ((rc = P->alloc((void**)&P->io_rim, (ns + nr) * sizeof(awc::IoRim)))) return rc;
  if ((rc = P->alloc(&P->stf, std::max<int64_t>(p->nt * p->nsrc, 1) * P->esz))) return rc;
  if ((rc = P->alloc(&P->traces, std::max<int64_t>(p->nt * p->nrec, 1) * P->esz))) return rc;
  P->staging_len = std::max<int64_t>(P->N, p->nt * p->nrec);
  if ((rc = P->alloc((void**)&P->staging, P->staging_len * 8))) return rc;
  CUDA_TRY(&P->ctx->err, cudaMemsetAsync(P->err_flag, 0, 4, P->ctx->stream));
  return AWC_OK;
}

template <typename T>
void to_T(const double* src, std::vector<unsigned char>& out, int64_t n) {
  out.resize(n * sizeof(T));
  T* d = reinterpret_cast<T*>(out.data());
  for (int64_t c = 0; c < n; ++c) d[c] = (T)src[c];
}

int grid_for(const awc_ctx* C, int64_t n, int threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads,
                                                     (int64_t)C->num_sms * 16));
}


void make_regions(awc_plan* P);
void box_blocks(awc_plan* P);
bool tb_eligible(const awc_plan* P);

// Uploads the inputs of one shot into an allocated plan. The copies are
// stream-ordered on the context stream.
int plan_upload(awc_plan* P, const double* vel, const double* coeffs, const int64_t* possrcs,
                const double* dt2srctf, const int64_t* posrecs) {
  awc_ctx* C = P->ctx;
  const awc_problem* p = &P->p;
  std::string* err = &C->err;
  cudaStream_t st = C->stream;
  const int64_t h = p->halo, nt = p->nt, nsrc = p->nsrc, nrec = p->nrec;
  const bool f64 = p->precision == AWC_F64;
  std::vector<unsigned char> tmp;
  if (vel) {  // NULL: a new shot over the model already uploaded
    // fact = dt^2 vel^2 on the device in FP64, written pitched
    CUDA_TRY(err, awc::copy_to_device(C, P->staging, vel, P->N * 8, st));
    {
      const double dt2 = p->dt * p->dt;
      const int blocks = grid_for(C, P->N, 256);
      if (f64)
        awc::make_fact<double><<<blocks, 256, 0, st>>>(P->staging, (double*)P->fact, dt2, P->N,
                                                       p->nx, P->px);
      else
        awc::make_fact<float><<<blocks, 256, 0, st>>>(P->staging, (float*)P->fact, dt2, P->N,
                                                      p->nx, P->px);
      CUDA_TRY(err, cudaGetLastError());
    }
    // coefficients (and which band sides are live)
    const int64_t clen = awc_coeffs_len(p);
    if (f64) to_T<double>(coeffs, tmp, clen); else to_T<float>(coeffs, tmp, clen);
    CUDA_TRY(err, cudaMemcpyAsync(P->coef, tmp.data(), tmp.size(), cudaMemcpyHostToDevice, st));
    CUDA_TRY(err, cudaStreamSynchronize(st));  // tmp is reused below
    for (int a = 0; a < p->ndim; ++a) {
      const double* blk = coeffs + a * (8 * h + 4);
      for (int s = 0; s < 2; ++s) {
        // a side whose every a is 0 and every b/K is 1 keeps ψ = ξ = 0 for ever
        // (the free top, acoustic_3D_xPU.jl:225-230); its updates are skipped.
        bool trivial = true;
        for (int64_t m = 0; m < h; ++m)
          trivial = trivial && blk[s * h + m] == 0.0 && blk[2 * h + s * h + m] == 1.0;
        const double* hb = blk + 4 * h;
        for (int64_t m = 0; m < h + 1; ++m)
          trivial = trivial && hb[s * (h + 1) + m] == 0.0 && hb[2 * (h + 1) + s * (h + 1) + m] == 1.0;
        P->active[a][s] = (h > 0 && !trivial) ? 1 : 0;
      }
    }
    if (p->ndim == 3) make_regions(P);
  }
  P->tb_io_shape = ~0ull;
  // every node carrying sources and/or receivers, in first-appearance order
  // (sources first); its sources are summed in source order
  {
    std::unordered_map<int64_t, int32_t> where;
    std::vector<std::vector<int32_t>> sg, rg;  // groups
    P->io_nodes.clear();
    auto node_slot = [&](int64_t nd) -> awc::IoRim& {
      auto f = where.find(nd);
      if (f == where.end()) {
        where.emplace(nd, (int32_t)P->io_nodes.size());
        P->io_nodes.push_back(awc::IoRim{nd, -1, -1});
        return P->io_nodes.back();
      }
      return P->io_nodes[f->second];
    };
    for (int64_t s = 0; s < nsrc; ++s) {
      awc::IoRim& e = node_slot(node_of(p, P->px, possrcs, nsrc, s));
      if (e.sgrp < 0) {
        e.sgrp = (int32_t)sg.size();
        sg.emplace_back();
      }
      sg[e.sgrp].push_back((int32_t)s);
    }
    for (int64_t r = 0; r < nrec; ++r) {
      awc::IoRim& e = node_slot(node_of(p, P->px, posrecs, nrec, r));
      if (e.rgrp < 0) {
        e.rgrp = (int32_t)rg.size();
        rg.emplace_back();
      }
      rg[e.rgrp].push_back((int32_t)r);
    }
    auto csr = [](const std::vector<std::vector<int32_t>>& g, std::vector<int32_t>& off,
                  std::vector<int32_t>& ids) {
      off.assign(1, 0);
      ids.clear();
      for (auto& v : g) {
        ids.insert(ids.end(), v.begin(), v.end());
        off.push_back((int32_t)ids.size());
      }
    };
    std::vector<int32_t> soff, sids, roff, rids;
    csr(sg, soff, sids);
    csr(rg, roff, rids);
    CUDA_TRY(err, cudaMemcpyAsync(P->src_off, soff.data(), soff.size() * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(err, cudaMemcpyAsync(P->rec_off, roff.data(), roff.size() * 4, cudaMemcpyHostToDevice, st));
    if (!sids.empty())
      CUDA_TRY(err, cudaMemcpyAsync(P->src_ids, sids.data(), sids.size() * 4, cudaMemcpyHostToDevice, st));
    if (!rids.empty())
      CUDA_TRY(err, cudaMemcpyAsync(P->rec_ids, rids.data(), rids.size() * 4, cudaMemcpyHostToDevice, st));
    P->io_shape = ~0ull;  // rebuild the block lists before the next launch
    P->tb_io_shape = ~0ull;
    // stf rows: [it][s] from the column-major (nt x nsrc) input
    std::vector<double> rows((size_t)std::max<int64_t>(nt * nsrc, 1), 0.0);
    for (int64_t s = 0; s < nsrc; ++s)
      for (int64_t t = 0; t < nt; ++t) rows[t * nsrc + s] = dt2srctf[t + nt * s];
    if (f64) to_T<double>(rows.data(), tmp, nt * nsrc); else to_T<float>(rows.data(), tmp, nt * nsrc);
    if (nt * nsrc > 0)
      CUDA_TRY(err, cudaMemcpyAsync(P->stf, tmp.data(), tmp.size(), cudaMemcpyHostToDevice, st));
    CUDA_TRY(err, cudaStreamSynchronize(st));  // host vectors go out of scope
  }
  if (P->depth == 2 && !tb_eligible(P)) P->depth = 1;  // this shot has rim sources/receivers
  return AWC_OK;
}

// Parameters of step `it` shared by every kernel of the step; the per-kernel
// source/receiver lists are filled by kernel_params.
template <typename T>
awc::StepParams<T> step_params(const awc_plan* P, int64_t it, const StepState& stt) {
  const awc_problem* p = &P->p;
  awc::StepParams<T> S{};
  // step it (0-based) reads pold = p_{it-1}, pcur = p_it and writes pnew into
  // the buffer of p_{it-2}: the (pold, pcur, pnew) <- (pcur, pnew, pold)
  // rotation of forward! (acoustic_3D_xPU.jl:166)
  S.pold = (const T*)P->buf[stt.ord[1]];
  S.pcur = (const T*)P->buf[stt.ord[0]];
  S.pnew = (T*)P->buf[stt.ord[2]];
  S.fact = (const T*)P->fact;
  S.nx = (int32_t)p->nx;
  S.ny = (int32_t)p->ny;
  S.nz = (int32_t)(p->ndim == 3 ? p->nz : 1);
  S.halo = p->halo;
  S.px = P->px;
  const double d[3] = {p->dx, p->dy, p->ndim == 3 ? p->dz : 1.0};
  for (int a = 0; a < 3; ++a) {
    S.inv_d[a] = (T)(1.0 / d[a]);
    S.inv_d2[a] = (T)(1.0 / (d[a] * d[a]));
  }
  if (P->is1d) S.inv_d[1] = S.inv_d2[1] = T(0);  // no y derivative on the line
  const int64_t h = p->halo;
  const T* cf = (const T*)P->coef;
  for (int a = 0; a < p->ndim; ++a) {
    const T* blk = cf + a * (8 * h + 4);
    for (int s = 0; s < 2; ++s) {
      awc::BandSide<T>& B = S.band[a][s];
      B.psi_old = (const T*)P->psi[a][s][stt.psi_par];
      B.psi_new = (T*)P->psi[a][s][stt.psi_par ^ 1];
      B.xi = (T*)(stt.xi_par ? P->xi_alt[a][s] : P->xi[a][s]);
      B.a = blk + s * h;
      B.bK = blk + 2 * h + s * h;
      B.ah = blk + 4 * h + s * (h + 1);
      B.bKh = blk + 4 * h + 2 * (h + 1) + s * (h + 1);
      S.active[a][s] = P->active[a][s];
    }
    const int64_t n = a == 0 ? p->nx : a == 1 ? p->ny : p->nz;
    S.first_r[a] = (int32_t)std::max<int64_t>(n - h - 1, h + 1);
  }
  S.zchunk = P->zchunk;
  S.it = (int32_t)it;
  S.err = P->err_flag;
  S.io.rim = P->io_rim;
  S.io.nrim = P->io_nrim;
  S.io.src_off = P->src_off;
  S.io.src_ids = P->src_ids;
  S.io.rec_off = P->rec_off;
  S.io.rec_ids = P->rec_ids;
  S.io.stf = (const T*)P->stf;
  S.io.nsrc = (int32_t)p->nsrc;
  S.io.nrec = (int32_t)p->nrec;
  S.io.traces = (T*)P->traces;
  S.core = P->core;
  S.core_x = P->core_x;
  S.nbox = P->nbox;
  for (int b2 = 0; b2 < 6; ++b2) S.box[b2] = P->box[b2];
  for (int b2 = 0; b2 < 7; ++b2) S.box_blk[b2] = P->box_blk[b2];
  S.shell_zchunk = P->szc;
  S.plane = P->px * p->ny;
  S.psi_dz[0] = (h + 1) * p->ny;
  S.xi_dz[0] = h * p->ny;
  S.psi_dz[1] = P->px * (h + 1);
  S.xi_dz[1] = P->px * h;
  for (int a = 0; a < 3; ++a) {
    S.psi_side[a] = P->psi_side[a];
    S.xi_side[a] = P->xi_side[a];
  }
  return S;
}

template <typename T>
void kernel_params(const awc_plan* P, int which, awc::StepParams<T>& S) {
  S.io.blk_off = P->io_k[which].blk_off;
  S.io.ent = P->io_k[which].ent;
  S.do_rim = P->io_k[which].do_rim;
}

// Splits the interior of a 3D grid into the core box (nodes outside every
// active CPML band: x in [halo+1, nx-halo-2] when both x sides are active,
// and so on) and up to six disjoint shell boxes covering the rest: the two
// z slabs over the whole x-y interior, the two y slabs over the core z range,
// the two x slabs over the core y and z ranges.
void make_regions(awc_plan* P) {
  const awc_problem* p = &P->p;
  const int64_t n[3] = {p->nx, p->ny, p->nz};
  int64_t lo[3], hi[3];
  bool empty = false;
  for (int a = 0; a < 3; ++a) {
    lo[a] = 1;
    hi[a] = n[a] - 2;
    if (P->active[a][0]) lo[a] = std::max<int64_t>(lo[a], p->halo + 1);
    if (P->active[a][1]) hi[a] = std::min<int64_t>(hi[a], n[a] - p->halo - 2);
    empty = empty || lo[a] > hi[a];
  }
  P->nbox = 0;
  // kind: 7 z slab, 3 y slab, 1 x slab, 15 no core (the band kernel's body)
  auto add = [&](int64_t x0, int64_t x1, int64_t y0, int64_t y1, int64_t z0, int64_t z1,
                 int32_t kind) {
    if (x0 > x1 || y0 > y1 || z0 > z1) return;
    P->box[P->nbox++] = awc::Box{(int32_t)x0, (int32_t)x1, (int32_t)y0, (int32_t)y1,
                                 (int32_t)z0, (int32_t)z1, kind};
  };
  if (empty) {
    P->has_core = false;
    add(1, n[0] - 2, 1, n[1] - 2, 1, n[2] - 2, 15);
  } else {
    P->has_core = true;
    P->core = awc::Box{(int32_t)lo[0], (int32_t)hi[0], (int32_t)lo[1], (int32_t)hi[1],
                       (int32_t)lo[2], (int32_t)hi[2], 0};
    const int64_t align = 16 / (int64_t)P->esz;  // TMA x origin alignment
    P->core_x = (int32_t)(lo[0] / align * align);
    add(1, n[0] - 2, 1, n[1] - 2, 1, lo[2] - 1, 7);
    add(1, n[0] - 2, 1, n[1] - 2, hi[2] + 1, n[2] - 2, 7);
    add(1, n[0] - 2, 1, lo[1] - 1, lo[2], hi[2], 3);
    add(1, n[0] - 2, hi[1] + 1, n[1] - 2, lo[2], hi[2], 3);
    add(1, lo[0] - 1, lo[1], hi[1], lo[2], hi[2], 1);
    add(hi[0] + 1, n[0] - 2, lo[1], hi[1], lo[2], hi[2], 1);
  }
  box_blocks(P);
}

// Block ranges of the band kernel: box b has its W x H columns in runs of
// BAND_NT times chunks of szc planes.
int64_t band_col_blocks(const awc::Box& B) {
  const int64_t ncol = (int64_t)(B.x1 - B.x0 + 1) * (B.y1 - B.y0 + 1);
  return (ncol + awc::BAND_NT - 1) / awc::BAND_NT;
}

void box_blocks(awc_plan* P) {
  P->box_blk[0] = 0;
  for (int b = 0; b < P->nbox; ++b) {
    const awc::Box& B = P->box[b];
    const int64_t blocks = band_col_blocks(B) * ((B.z1 - B.z0 + P->szc) / P->szc);
    P->box_blk[b + 1] = (int32_t)(P->box_blk[b] + blocks);
  }
  for (int b = P->nbox; b < 6; ++b) P->box_blk[b + 1] = P->box_blk[b];
}

// Launch grid of the 2D kernel (x tiles of 32 from x = 0, y tiles of 8 rows
// from y = 1) or of the 3D core kernel (x tiles of 64 from core_x, y tiles of
// `by` rows from core.y0, z chunks of `zchunk` planes from core.z0).
dim3 step_grid(const awc_plan* P) {
  const awc_problem* p = &P->p;
  if (p->ndim == 2)
    return dim3((unsigned)((p->nx - 2) / 32 + 1), (unsigned)((p->ny - 2 + 7) / 8), 1);
  if (!P->has_core) return dim3(0, 0, 0);
  const awc::Box& C = P->core;
  return dim3((unsigned)((C.x1 - P->core_x) / 64 + 1), (unsigned)((C.y1 - C.y0 + P->by) / P->by),
              (unsigned)((C.z1 - C.z0 + P->zchunk) / P->zchunk));
}

uint64_t launch_shape(const awc_plan* P) {
  return (uint64_t)P->by | ((uint64_t)P->zchunk << 8) | ((uint64_t)(P->szc & 0xff) << 40) |
         ((uint64_t)(P->depth & 3) << 48) | ((uint64_t)(P->tb_nch & 0xfff) << 50) |
         ((uint64_t)(P->tb_rows == 8 ? 1 : 0) << 62);
}

// Buckets the source/receiver nodes by the kernel and block that own them for
// the current launch shape: rim nodes to the rim list; 3D nodes inside the
// core box to the core kernel, in (block, plane, local) order; other interior
// nodes to the shell kernel's block of their box tile; 2D nodes to the 2D
// kernel.
int ensure_io(awc_plan* P) {
  if (P->io_shape == launch_shape(P)) return AWC_OK;
  awc_ctx* C = P->ctx;
  const awc_problem* p = &P->p;
  const bool d3 = p->ndim == 3;
  const dim3 g = step_grid(P);
  const int64_t nblk[2] = {(int64_t)g.x * g.y * g.z, d3 ? (int64_t)P->box_blk[P->nbox] : 0};
  std::vector<awc::IoRim> rim;
  std::vector<std::pair<std::pair<int64_t, int64_t>, int4>> ent[2];  // ((blk, k*2^32+local), entry)
  for (const awc::IoRim& e : P->io_nodes) {
    const int64_t i = e.node % P->px, j = (e.node / P->px) % p->ny, k = e.node / (P->px * p->ny);
    const bool interior = i >= 1 && i <= p->nx - 2 && j >= 1 && j <= p->ny - 2 &&
                          (!d3 || (k >= 1 && k <= p->nz - 2));
    if (!interior) {
      rim.push_back(e);
      continue;
    }
    if (!d3) {
      const int64_t blk = i / 32 + g.x * ((j - 1) / 8);
      const int local = (int)(i % 32 + 32 * ((j - 1) % 8));
      ent[0].push_back({{blk, local}, make_int4(local, 0, e.sgrp, e.rgrp)});
      continue;
    }
    const awc::Box& Cb = P->core;
    if (P->has_core && i >= Cb.x0 && i <= Cb.x1 && j >= Cb.y0 && j <= Cb.y1 && k >= Cb.z0 &&
        k <= Cb.z1) {
      const int64_t lx = (i - P->core_x) % 64, ly = (j - Cb.y0) % P->by;
      const int64_t blk = (k - Cb.z0) / P->zchunk +
                          g.z * ((i - P->core_x) / 64 + (int64_t)g.x * ((j - Cb.y0) / P->by));
      const int local = (int)(lx + 64 * ly);
      ent[0].push_back({{blk, (k << 32) | local}, make_int4(local, (int)k, e.sgrp, e.rgrp)});
      continue;
    }
    for (int b = 0; b < P->nbox; ++b) {
      const awc::Box& B = P->box[b];
      if (i < B.x0 || i > B.x1 || j < B.y0 || j > B.y1 || k < B.z0 || k > B.z1) continue;
      const int64_t l = (i - B.x0) + (int64_t)(B.x1 - B.x0 + 1) * (j - B.y0);
      const int64_t blk = P->box_blk[b] + l / awc::BAND_NT +
                          band_col_blocks(B) * ((k - B.z0) / P->szc);
      const int local = (int)(l % awc::BAND_NT);
      ent[1].push_back({{blk, (k << 32) | local}, make_int4(local, (int)k, e.sgrp, e.rgrp)});
      break;
    }
  }
  cudaStream_t st = C->stream;
  std::vector<int32_t> off[2];
  std::vector<int4> flat[2];
  for (int kk = 0; kk < 2; ++kk) {
    auto& E = ent[kk];
    std::sort(E.begin(), E.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    off[kk].assign(nblk[kk] + 1, 0);
    flat[kk].resize(E.size());
    for (size_t n = 0; n < E.size(); ++n) {
      off[kk][E[n].first.first + 1]++;
      flat[kk][n] = E[n].second;
    }
    for (int64_t b = 0; b < nblk[kk]; ++b) off[kk][b + 1] += off[kk][b];
    auto& S = P->io_k[kk];
    if (S.cap < nblk[kk] + 1) {
      P->release(S.blk_off);
      S.blk_off = nullptr;
      S.cap = 0;
      int rc = P->alloc((void**)&S.blk_off, (nblk[kk] + 1) * 4);
      if (rc) return rc;
      S.cap = nblk[kk] + 1;
    }
    CUDA_TRY(&C->err, cudaMemcpyAsync(S.blk_off, off[kk].data(), off[kk].size() * 4,
                                      cudaMemcpyHostToDevice, st));
    if (!flat[kk].empty())
      CUDA_TRY(&C->err, cudaMemcpyAsync(S.ent, flat[kk].data(), flat[kk].size() * sizeof(int4),
                                        cudaMemcpyHostToDevice, st));
  }
  // the rim is served by the shell kernel when there is one, else by the other
  P->io_k[1].do_rim = d3 && P->nbox > 0 ? 1 : 0;
  P->io_k[0].do_rim = P->io_k[1].do_rim ? 0 : 1;
  if (!rim.empty())
    CUDA_TRY(&C->err, cudaMemcpyAsync(P->io_rim, rim.data(), rim.size() * sizeof(awc::IoRim),
                                      cudaMemcpyHostToDevice, st));
  CUDA_TRY(&C->err, cudaStreamSynchronize(st));
  P->io_nrim = (int32_t)rim.size();
  P->io_shape = launch_shape(P);
  return AWC_OK;
}

// Tensor map of a pitched field of the plan for the core kernel at the
// current tile height: the pcur box with its ring ((64 + 2A) x (by + 2) x 1,
// ring = true) or the pold / fact tile (64 x by x 1). Dims (nx, ny, nz),
// pitched strides.
bool field_map(const awc_plan* P, CUtensorMap* m, const void* base, bool ring) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = awc::tensor_map_encoder();
  if (!enc) return false;
  const awc_problem* p = &P->p;
  const bool f64 = p->precision == AWC_F64;
  const CUtensorMapDataType dt = f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint32_t A = 16 / (cuuint32_t)P->esz;
  const cuuint64_t dims[3] = {(cuuint64_t)p->nx, (cuuint64_t)p->ny, (cuuint64_t)p->nz};
  const cuuint64_t strides[2] = {(cuuint64_t)(P->px * P->esz), (cuuint64_t)(P->px * p->ny * P->esz)};
  const cuuint32_t box_c[3] = {64 + 2 * A, (cuuint32_t)P->by + 2, 1};
  const cuuint32_t box_i[3] = {64, (cuuint32_t)P->by, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, dt, 3, const_cast<void*>(base), dims, strides, ring ? box_c : box_i, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of the 3D core kernel: both boxes for each rotating field
// buffer, and the tile of fact.
int ensure_maps(awc_plan* P) {
  if (P->maps_by == P->by) return AWC_OK;
  awc_ctx* C = P->ctx;
  if (!awc::tensor_map_encoder())
    return set_err(&C->err, AWC_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  for (int b = 0; b < P->nbuf; ++b)
    if (!field_map(P, &P->map_c[b], P->buf[b], true) || !field_map(P, &P->map_o[b], P->buf[b], false))
      return set_err(&C->err, AWC_ERR_CUDA, "tensor map encoding failed");
  if (!field_map(P, &P->map_f, P->fact, false))
    return set_err(&C->err, AWC_ERR_CUDA, "tensor map encoding failed");
  P->maps_by = P->by;
  return AWC_OK;
}

// ---- two-step passes (awc_tb.cuh) ------------------------------------------

// Level-2 tile of the two-step kernel: 62 x (rows - 2) nodes; its level-1
// region adds a ring of one node (64 x rows).
constexpr int TB_TX = awc::TbTile<float, 16>::TX;
constexpr int TB_RX = awc::TbTile<float, 16>::RX;

// The number of z chunks the two-step kernel really has when asked for c:
// chunks of ceil(iz / c) planes cover the iz interior planes in
// ceil(iz / ceil(iz / c)) chunks.
int32_t tb_chunks(const awc_plan* P, int64_t c) {
  const int64_t iz = P->p.nz - 2;
  c = std::max<int64_t>(1, std::min<int64_t>(c, iz));
  const int64_t zc = (iz + c - 1) / c;
  return (int32_t)((iz + zc - 1) / zc);
}

// Whether the problem can run two-step passes: 3D with every source and
// receiver on an interior node (the rim of every field then stays zero).
bool tb_eligible(const awc_plan* P) {
  if (P->p.ndim != 3) return false;
  for (const awc::IoRim& e : P->io_nodes) {
    const int64_t i = e.node % P->px, j = (e.node / P->px) % P->p.ny,
                  k = e.node / (P->px * P->p.ny);
    if (i < 1 || i > P->p.nx - 2 || j < 1 || j > P->p.ny - 2 || k < 1 || k > P->p.nz - 2)
      return false;
  }
  return true;
}

// Whether interior coordinate c of an axis of n nodes lies in an active band.
bool in_active_band(const awc_plan* P, int a, int64_t c) {
  const int64_t n = a == 0 ? P->p.nx : a == 1 ? P->p.ny : P->p.nz, h = P->p.halo;
  if (c < 1 || c > n - 2) return false;
  if (c <= h) return P->active[a][0] != 0;
  if (c >= n - h - 1) return P->active[a][1] != 0;
  return false;
}

// Tile lists and per-block source/receiver lists of the two-step kernel for
// the current chunking. Tile (tx, ty) has level-2 origin (1 + 30 tx,
// 1 + TY ty); it goes to the XY list when its level-1 region (the tile and a
// ring of one node) meets an active x or y band, else to the Z list.
int ensure_tb(awc_plan* P) {
  const uint64_t shape = (uint64_t)P->tb_nch | ((uint64_t)P->tb_rows << 32);
  if (P->tb_io_shape == shape) return AWC_OK;
  const int64_t TB_TY = P->tb_rows - 2;
  awc_ctx* C = P->ctx;
  const awc_problem* p = &P->p;
  const int64_t ntx = (p->nx - 2 + TB_TX - 1) / TB_TX, nty = (p->ny - 2 + TB_TY - 1) / TB_TY;
  std::vector<int2> tiles[2];
  std::vector<std::pair<int, int32_t>> where((size_t)(ntx * nty));  // (list, index)
  for (int64_t ty = 0; ty < nty; ++ty)
    for (int64_t tx = 0; tx < ntx; ++tx) {
      const int64_t X0 = 1 + TB_TX * tx, Y0 = 1 + TB_TY * ty;
      bool xy = false;
      for (int64_t x = X0 - 1; x <= X0 + TB_TX && !xy; ++x) xy = in_active_band(P, 0, x);
      for (int64_t y = Y0 - 1; y <= Y0 + TB_TY && !xy; ++y) xy = in_active_band(P, 1, y);
      where[ty * ntx + tx] = {xy ? 1 : 0, (int32_t)tiles[xy ? 1 : 0].size()};
      tiles[xy ? 1 : 0].push_back(make_int2((int)X0, (int)Y0));
    }
  const int64_t iz = p->nz - 2;
  P->tb_zc = (int32_t)((iz + P->tb_nch - 1) / P->tb_nch);
  const int32_t nch = P->tb_nch;  // normalised by tb_chunks: exactly covers iz
  if ((int64_t)nch * P->tb_zc < iz || (int64_t)(nch - 1) * P->tb_zc >= iz)
    return set_err(&C->err, AWC_ERR_INVALID, "internal: z chunking does not cover the grid");
  // entries ((block, plane << 32 | thread), {thread, plane, sgrp, rgrp or -1})
  std::vector<std::pair<std::pair<int64_t, int64_t>, int4>> ent[2];
  for (const awc::IoRim& e : P->io_nodes) {
    const int64_t i = e.node % P->px, j = (e.node / P->px) % p->ny, k = e.node / (P->px * p->ny);
    const int64_t tx0 = (i - 1) / TB_TX, ty0 = (j - 1) / TB_TY;
    for (int64_t ty = std::max<int64_t>(ty0 - 1, 0); ty <= std::min(ty0 + 1, nty - 1); ++ty)
      for (int64_t tx = std::max<int64_t>(tx0 - 1, 0); tx <= std::min(tx0 + 1, ntx - 1); ++tx) {
        const int64_t X0 = 1 + TB_TX * tx, Y0 = 1 + TB_TY * ty;
        if (i < X0 - 1 || i > X0 + TB_TX || j < Y0 - 1 || j > Y0 + TB_TY) continue;
        const bool own_col = i >= X0 && i < X0 + TB_TX && j >= Y0 && j < Y0 + TB_TY;
        // the node's index in the level-1 region: 2 x (thread) + (node of its pair)
        const int thread = (int)((i - (X0 - 1)) + TB_RX * (j - (Y0 - 1)));
        const auto& wh = where[ty * ntx + tx];
        for (int32_t c = 0; c < nch; ++c) {
          const int64_t k0 = 1 + (int64_t)c * P->tb_zc, k1 = std::min<int64_t>(k0 + P->tb_zc, p->nz - 1);
          if (k < k0 - 1 || k > k1) continue;
          const bool own = own_col && k >= k0 && k < k1;
          const int64_t blk = (int64_t)wh.second * nch + c;
          ent[wh.first].push_back(
              {{blk, (k << 32) | thread}, make_int4(thread, (int)k, e.sgrp, own ? e.rgrp : -1)});
        }
      }
  }
  cudaStream_t st = C->stream;
  for (int v = 0; v < 2; ++v) {
    const int64_t nt_ = (int64_t)tiles[v].size();
    P->tb_ntiles[v] = (int32_t)nt_;
    if (P->tb_tiles_cap[v] < std::max<int64_t>(nt_, 1)) {
      P->release(P->tb_tiles[v]);
      P->tb_tiles[v] = nullptr;
      P->tb_tiles_cap[v] = 0;
      if (int rc = P->alloc((void**)&P->tb_tiles[v], std::max<int64_t>(nt_, 1) * sizeof(int2)))
        return rc;
      P->tb_tiles_cap[v] = std::max<int64_t>(nt_, 1);
    }
    if (nt_ > 0)
      CUDA_TRY(&C->err, cudaMemcpyAsync(P->tb_tiles[v], tiles[v].data(), nt_ * sizeof(int2),
                                        cudaMemcpyHostToDevice, st));
    const int64_t nblk = nt_ * nch;
    auto& E = ent[v];
    std::sort(E.begin(), E.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<int32_t> off((size_t)nblk + 1, 0);
    std::vector<int4> flat(E.size());
    for (size_t n = 0; n < E.size(); ++n) {
      off[E[n].first.first + 1]++;
      flat[n] = E[n].second;
    }
    for (int64_t b = 0; b < nblk; ++b) off[b + 1] += off[b];
    auto& S = P->tb_io[v];
    if (S.cap < nblk + 1) {
      P->release(S.blk_off);
      S.blk_off = nullptr;
      S.cap = 0;
      if (int rc = P->alloc((void**)&S.blk_off, (nblk + 1) * 4)) return rc;
      S.cap = nblk + 1;
    }
    // every node appears in at most 4 tiles x 2 chunks
    const int64_t ecap = std::max<int64_t>((int64_t)flat.size(), 1);
    if (S.ecap < ecap) {
      P->release(S.ent);
      S.ent = nullptr;
      S.ecap = 0;
      if (int rc = P->alloc((void**)&S.ent, ecap * sizeof(int4))) return rc;
      S.ecap = ecap;
    }
    CUDA_TRY(&C->err, cudaMemcpyAsync(S.blk_off, off.data(), off.size() * 4,
                                      cudaMemcpyHostToDevice, st));
    if (!flat.empty())
      CUDA_TRY(&C->err, cudaMemcpyAsync(S.ent, flat.data(), flat.size() * sizeof(int4),
                                        cudaMemcpyHostToDevice, st));
  }
  CUDA_TRY(&C->err, cudaStreamSynchronize(st));
  P->tb_io_shape = shape;
  return AWC_OK;
}

// Tensor maps of the two-step kernel for every field buffer: the p_s box
// (40 x (TB_ROWS + 2)) and the p_{s-1} box (40 x TB_ROWS), and fact's.
int ensure_tb_maps(awc_plan* P) {
  if (P->tb_maps_rows == P->tb_rows) return AWC_OK;
  awc_ctx* C = P->ctx;
  const awc_problem* p = &P->p;
  PFN_cuTensorMapEncodeTiled_v12000 enc = awc::tensor_map_encoder();
  if (!enc) return set_err(&C->err, AWC_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const CUtensorMapDataType dt =
      p->precision == AWC_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[3] = {(cuuint64_t)p->nx, (cuuint64_t)p->ny, (cuuint64_t)p->nz};
  const cuuint64_t strides[2] = {(cuuint64_t)(P->px * P->esz), (cuuint64_t)(P->px * p->ny * P->esz)};
  constexpr int BX = awc::TbTile<float, 16>::BX;
  const cuuint32_t box_pt[3] = {BX, (cuuint32_t)P->tb_rows + 2, 1};
  const cuuint32_t box_in[3] = {BX, (cuuint32_t)P->tb_rows, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  auto make = [&](CUtensorMap* m, void* base, const cuuint32_t* box) -> bool {
    return enc(m, dt, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  for (int b = 0; b < P->nbuf; ++b)
    if (!make(&P->tb_map_pt[b], P->buf[b], box_pt) || !make(&P->tb_map_in[b], P->buf[b], box_in))
      return set_err(&C->err, AWC_ERR_CUDA, "tensor map encoding failed");
  if (!make(&P->tb_map_f, P->fact, box_in))
    return set_err(&C->err, AWC_ERR_CUDA, "tensor map encoding failed");
  P->tb_maps_rows = P->tb_rows;
  return AWC_OK;
}

template <typename T, int TY>
constexpr int core_smem() {
  return stages<T>() * awc::Tile3<T, TY>::BYTES + 2 * stages<T>() * 8 + 16;
}

// Opts every core-kernel instantiation into its dynamic shared memory size on
// the current device (done at context creation, outside any capture).
int init_kernel_attrs(std::string* err) {
#define AWC_ATTR(T, TY)                                                                    \
  CUDA_TRY(err, cudaFuncSetAttribute(awc::step3d_core<T, TY, stages<T>()>,                 \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                                     core_smem<T, TY>()))
  AWC_ATTR(float, 2);
  AWC_ATTR(float, 4);
  AWC_ATTR(float, 8);
  AWC_ATTR(double, 2);
  AWC_ATTR(double, 4);
  AWC_ATTR(double, 8);
#undef AWC_ATTR
  CUDA_TRY(err, awc::tb_init_attrs());
  return AWC_OK;
}

template <typename T, int TY>
void launch_core(awc_plan* P, const CUtensorMap& mc, const CUtensorMap& mo,
                 const awc::StepParams<T>& S, dim3 grid, cudaStream_t st) {
  awc::step3d_core<T, TY, stages<T>()><<<grid, dim3(32, TY), core_smem<T, TY>(), st>>>(
      mc, mo, P->map_f, S);
}

// Whether step it writes its field into the keep list itself: only when no
// source or receiver sits on the rim, whose values (p_{t+1} = p_{t-1} + S_t
// there) the step reads from the buffer it overwrites; the keep list's rims
// are zero, as the plan's are without rim sources.
bool kept_in_place(const awc_plan* P, int64_t it) {
  return P->keep && P->keep_in_place && P->io_nrim == 0 && it >= P->keep_first &&
         it < P->keep_first + P->keep_count;
}

// One time step. 3D: the shell kernel on the context's second stream and the
// core kernel on its main stream, forked from and joined back into the main
// stream (parallel branches once captured in a graph). 2D: one kernel.
template <typename T>
int launch_step(awc_plan* P, int64_t it, const StepState& stt, cudaStream_t st) {
  awc_ctx* C = P->ctx;
  const awc_problem* p = &P->p;
  awc::StepParams<T> S = step_params<T>(P, it, stt);
  const CUtensorMap* mc = &P->map_c[stt.ord[0]];
  const CUtensorMap* mo = &P->map_o[stt.ord[1]];
  CUtensorMap kc, ko;
  if (kept_in_place(P, it)) {
    void* const* f = P->keep + (it - P->keep_first);
    S.pold = (const T*)f[-2];
    S.pcur = (const T*)f[-1];
    S.pnew = (T*)f[0];
    if (p->ndim == 3 && P->has_core) {
      if (!field_map(P, &kc, f[-1], true) || !field_map(P, &ko, f[-2], false))
        return set_err(&C->err, AWC_ERR_CUDA, "tensor map encoding failed");
      mc = &kc;
      mo = &ko;
    }
  }
  if (p->ndim == 2) {
    kernel_params(P, 0, S);
    awc::step2d<T><<<step_grid(P), dim3(32, 8), 0, st>>>(S);
  } else {
    const bool shell = P->nbox > 0, core = P->has_core;
    if (shell && core) {
      CUDA_TRY(&C->err, cudaEventRecord(C->ev_fork, st));
      CUDA_TRY(&C->err, cudaStreamWaitEvent(C->stream2, C->ev_fork, 0));
    }
    if (shell) {
      awc::StepParams<T> Sh = S;
      kernel_params(P, 1, Sh);
      cudaStream_t sb = core ? C->stream2 : st;
      // offsets fit in int32 when every field (and so every ψ/ξ array) does
      const unsigned nb = (unsigned)P->box_blk[P->nbox];
      if (P->NP <= (int64_t)INT32_MAX)
        awc::step3d_band<T, int32_t><<<nb, awc::BAND_NT, 0, sb>>>(Sh);
      else
        awc::step3d_band<T, int64_t><<<nb, awc::BAND_NT, 0, sb>>>(Sh);
    }
    if (core) {
      kernel_params(P, 0, S);
      const dim3 grid = step_grid(P);
      switch (P->by) {
        case 4: launch_core<T, 2>(P, *mc, *mo, S, grid, st); break;
        case 8: launch_core<T, 4>(P, *mc, *mo, S, grid, st); break;
        case 16: launch_core<T, 8>(P, *mc, *mo, S, grid, st); break;
        default: return set_err(&C->err, AWC_ERR_INVALID, "unsupported tile height %d", P->by);
      }
    }
    if (shell && core) {
      CUDA_TRY(&C->err, cudaEventRecord(C->ev_join, C->stream2));
      CUDA_TRY(&C->err, cudaStreamWaitEvent(st, C->ev_join, 0));
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(&C->err, AWC_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  return AWC_OK;
}

// Parameters of the two-step pass that starts after step `it` - 1 (it is the
// 0-based index of its first step) in state `stt`.
template <typename T>
awc::TbParams<T> tb_params(const awc_plan* P, int64_t it, const StepState& stt) {
  const awc_problem* p = &P->p;
  awc::TbParams<T> Q{};
  Q.pold = (const T*)P->buf[stt.ord[1]];
  Q.pcur = (const T*)P->buf[stt.ord[0]];
  Q.p1 = (T*)P->buf[stt.ord[2]];
  Q.p2 = (T*)P->buf[stt.ord[3]];
  Q.fact = (const T*)P->fact;
  Q.nx = (int32_t)p->nx;
  Q.ny = (int32_t)p->ny;
  Q.nz = (int32_t)p->nz;
  Q.halo = p->halo;
  Q.px = P->px;
  Q.plane = P->px * p->ny;
  const double d[3] = {p->dx, p->dy, p->dz};
  for (int a = 0; a < 3; ++a) {
    Q.inv_d[a] = (T)(1.0 / d[a]);
    Q.inv_d2[a] = (T)(1.0 / (d[a] * d[a]));
  }
  const int64_t h = p->halo;
  const T* cf = (const T*)P->coef;
  for (int a = 0; a < 3; ++a) {
    const T* blk = cf + a * (8 * h + 4);
    awc::TbAxis<T>& X = Q.ax[a];
    X.psi_in = (const T*)P->psi[a][0][stt.psi_par];
    X.psi_out = (T*)P->psi[a][0][stt.psi_par ^ 1];
    X.xi_in = (const T*)(stt.xi_par ? P->xi_alt[a][0] : P->xi[a][0]);
    X.xi_out = (T*)(stt.xi_par ? P->xi[a][0] : P->xi_alt[a][0]);
    X.a = blk;
    X.bK = blk + 2 * h;
    X.ah = blk + 4 * h;
    X.bKh = blk + 4 * h + 2 * (h + 1);
    X.psi_side = P->psi_side[a];
    X.xi_side = P->xi_side[a];
    for (int sd = 0; sd < 2; ++sd) Q.active[a][sd] = P->active[a][sd];
    const int64_t n = a == 0 ? p->nx : a == 1 ? p->ny : p->nz;
    Q.first_r[a] = (int32_t)std::max<int64_t>(n - h - 1, h + 1);
  }
  Q.damp_all = P->has_core ? 0 : 1;
  Q.it = (int32_t)it;
  Q.err = P->err_flag;
  Q.io.src_off = P->src_off;
  Q.io.src_ids = P->src_ids;
  Q.io.rec_off = P->rec_off;
  Q.io.rec_ids = P->rec_ids;
  Q.io.stf = (const T*)P->stf;
  Q.io.nsrc = (int32_t)p->nsrc;
  Q.io.nrec = (int32_t)p->nrec;
  Q.io.traces = (T*)P->traces;
  Q.nch = P->tb_nch;
  Q.zc = P->tb_zc;
  Q.wait_rounds = P->wait_rounds;
  Q.wait_ns = P->wait_ns;
  Q.withhold = P->withhold;
  return Q;
}

// One two-step pass (steps it and it + 1): the XY tiles on the second stream
// and the Z tiles on the main one, as parallel branches like a 3D step.
template <typename T>
int launch_pass2(awc_plan* P, int64_t it, const StepState& stt, cudaStream_t st) {
  awc_ctx* C = P->ctx;
  awc::TbParams<T> Q = tb_params<T>(P, it, stt);
  const bool i64 = P->NP > (int64_t)INT32_MAX;
  const bool both = P->tb_ntiles[0] > 0 && P->tb_ntiles[1] > 0;
  if (both) {
    CUDA_TRY(&C->err, cudaEventRecord(C->ev_fork, st));
    CUDA_TRY(&C->err, cudaStreamWaitEvent(C->stream2, C->ev_fork, 0));
  }
  for (int v = 1; v >= 0; --v) {
    if (P->tb_ntiles[v] == 0) continue;
    Q.tiles = P->tb_tiles[v];
    Q.io.blk_off = P->tb_io[v].blk_off;
    Q.io.ent = P->tb_io[v].ent;
    const unsigned nb = (unsigned)((int64_t)P->tb_ntiles[v] * P->tb_nch);
    const cudaError_t e =
        awc::tb_launch<T>(Q, v == 1, i64, P->tb_rows, P->tb_map_pt[stt.ord[0]],
                          P->tb_map_in[stt.ord[1]], P->tb_map_f, nb,
                          (v == 1 && both) ? C->stream2 : st);
    if (e != cudaSuccess)
      return set_err(&C->err, AWC_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  }
  if (both) {
    CUDA_TRY(&C->err, cudaEventRecord(C->ev_join, C->stream2));
    CUDA_TRY(&C->err, cudaStreamWaitEvent(st, C->ev_join, 0));
  }
  return AWC_OK;
}

// Whether the launch sequence of this plan advances two steps per pass.
bool two_step(const awc_plan* P) { return P->depth == 2 && !P->keep; }

// Launches steps [start, start + n) from state `stt` (updated to the state
// after them): two-step passes while two steps remain at depth 2, else
// one-step launches.
int launch_range(awc_plan* P, int64_t start, int64_t n, StepState& stt, cudaStream_t st) {
  const bool f64 = P->p.precision == AWC_F64;
  for (int64_t it = start; it < start + n;) {
    int rc;
    if (two_step(P) && it + 1 < start + n) {
      rc = f64 ? launch_pass2<double>(P, it, stt, st) : launch_pass2<float>(P, it, stt, st);
      if (rc) return rc;
      stt.pass2();
      it += 2;
      continue;
    }
    rc = f64 ? launch_step<double>(P, it, stt, st) : launch_step<float>(P, it, stt, st);
    if (rc) return rc;
    const bool in_place = kept_in_place(P, it);
    if (P->keep && !in_place && it >= P->keep_first && it < P->keep_first + P->keep_count)
      CUDA_TRY(&P->ctx->err, cudaMemcpyAsync(P->keep[it - P->keep_first], P->buf[stt.ord[2]],
                                             P->NP * P->esz, cudaMemcpyDeviceToDevice, st));
    stt.step1();
    if (in_place && it == P->keep_first + P->keep_count - 1) {
      // the plan's buffers take p_it and p_{it+1} back from the keep list
      void* const* f = P->keep + (it - P->keep_first);
      const size_t fb = P->NP * P->esz;
      CUDA_TRY(&P->ctx->err, cudaMemcpyAsync(P->buf[stt.ord[0]], f[0], fb, cudaMemcpyDeviceToDevice, st));
      CUDA_TRY(&P->ctx->err, cudaMemcpyAsync(P->buf[stt.ord[1]], f[-1], fb, cudaMemcpyDeviceToDevice, st));
    }
    ++it;
  }
  return AWC_OK;
}

// Kernel launches of n steps from the current state.
int64_t launch_count(const awc_plan* P, int64_t n) {
  const int64_t one = (P->p.ndim == 3 && P->has_core && P->nbox > 0) ? 2 : 1;
  if (!two_step(P)) return one * n;
  const int64_t per_pass = (P->tb_ntiles[0] > 0 ? 1 : 0) + (P->tb_ntiles[1] > 0 ? 1 : 0);
  return per_pass * (n / 2) + one * (n % 2);
}

// Everything a launch sequence depends on besides the step index.
int prepare_launch(awc_plan* P) {
  int rc;
  if ((rc = ensure_io(P))) return rc;
  if (P->p.ndim == 3 && P->has_core && (rc = ensure_maps(P))) return rc;
  if (two_step(P) && ((rc = ensure_tb(P)) || (rc = ensure_tb_maps(P)))) return rc;
  return AWC_OK;
}

awc_plan::GraphKey config_key(const awc_plan* P) {
  awc_plan::GraphKey k;
  k.launch = launch_shape(P);
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s) k.active[a][s] = P->active[a][s];
  k.d[0] = P->p.dx;
  k.d[1] = P->p.dy;
  k.d[2] = P->p.ndim == 3 ? P->p.dz : 1.0;
  k.nrim = P->io_nrim;
  for (int w = 0; w < 2; ++w) {
    k.do_rim[w] = P->io_k[w].do_rim;
    k.blk_off[w] = P->io_k[w].blk_off;
    k.blk_off[2 + w] = P->tb_io[w].blk_off;
    k.tiles[w] = P->tb_tiles[w];
  }
  k.wait[0] = P->wait_rounds;
  k.wait[1] = P->wait_ns;
  k.wait[2] = P->withhold;
  return k;
}

int get_graph(awc_plan* P, int64_t start, int64_t n, cudaGraphExec_t* out) {
  awc_ctx* C = P->ctx;
  const awc_plan::GraphKey key = config_key(P);
  if (!(key == P->graph_key)) {
    P->drop_graphs();
    P->graph_key = key;
  }
  // the field copies of a keep-fields run are part of the capture
  int64_t kh = 0, kfirst = 0;
  if (P->keep) {
    kfirst = P->keep_first;
    uint64_t hsh = 1469598103934665603ull;  // FNV-1a over the destinations in range
    for (int64_t it = std::max(start, P->keep_first);
         it < std::min(start + n, P->keep_first + P->keep_count); ++it) {
      for (int64_t d = P->keep_in_place ? -2 : 0; d <= 0; ++d) {  // in place: the fields read too
        hsh ^= (uint64_t)(uintptr_t)P->keep[it - P->keep_first + d];
        hsh *= 1099511628211ull;
      }
    }
    hsh ^= P->keep_in_place ? 0x9e3779b97f4a7c15ull : 0ull;
    kh = (int64_t)(hsh | 1);
  }
  const std::array<int64_t, 5> gk{start, n, P->state.code(), kfirst, kh};
  auto f = P->graphs.find(gk);
  if (f != P->graphs.end()) {
    *out = f->second;
    return AWC_OK;
  }
  cudaGraph_t g = nullptr;
  CUDA_TRY(&C->err, cudaStreamBeginCapture(C->stream, cudaStreamCaptureModeThreadLocal));
  StepState stt = P->state;
  int rc = launch_range(P, start, n, stt, C->stream);
  cudaError_t e = cudaStreamEndCapture(C->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess)
    return set_err(&C->err, AWC_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess)
    return set_err(&C->err, AWC_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
  P->graphs[gk] = ex;
  *out = ex;
  return AWC_OK;
}

int occupancy(const awc_plan* P, int by) {
  int occ = 0;
  const bool f64 = P->p.precision == AWC_F64;
#define AWC_OCC(T, TY)                                                                     \
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, awc::step3d_core<T, TY, stages<T>()>, \
                                                32 * TY, core_smem<T, TY>())
  if (f64) {
    if (by == 4) AWC_OCC(double, 2);
    if (by == 8) AWC_OCC(double, 4);
    if (by == 16) AWC_OCC(double, 8);
  } else {
    if (by == 4) AWC_OCC(float, 2);
    if (by == 8) AWC_OCC(float, 4);
    if (by == 16) AWC_OCC(float, 8);
  }
#undef AWC_OCC
  cudaGetLastError();
  return occ > 0 ? occ : 1;
}

// z chunk that spreads the core tiles of one tile height over about `waves`
// rounds of resident blocks.
int32_t chunk_for(const awc_plan* P, int by, double waves) {
  if (!P->has_core) return 1;
  const awc::Box& C = P->core;
  const int64_t iz = C.z1 - C.z0 + 1;
  const int64_t tiles = ((C.x1 - P->core_x) / 64 + 1) * ((C.y1 - C.y0 + by) / by);
  const int64_t resident = (int64_t)P->ctx->num_sms * occupancy(P, by);
  int64_t nch = (int64_t)std::llround(waves * (double)resident / (double)std::max<int64_t>(tiles, 1));
  nch = std::max<int64_t>(1, std::min<int64_t>(nch, iz));
  return (int32_t)((iz + nch - 1) / nch);
}

// Default launch shape: 64 x 8 core tiles and one wave of resident blocks;
// the autotuner refines it.
void default_tuning(awc_plan* P) {
  P->by = 8;
  P->zchunk = P->p.ndim == 3 ? chunk_for(P, P->by, 1.0) : 1;
}

int forward_impl(awc_ctx* C, const awc_problem* p, const double* vel, const double* coeffs,
                 const int64_t* possrcs, const double* dt2srctf, const int64_t* posrecs,
                 awc_plan** out, bool lifted1d = false) {
  std::string* err = &C->err;
  int rc;
  if ((rc = validate(p, err, lifted1d))) return rc;
  if (!vel || !coeffs) return set_err(err, AWC_ERR_INVALID, "vel/coeffs are NULL");
  if (p->nsrc > 0 && p->nt > 0 && !dt2srctf)
    return set_err(err, AWC_ERR_INVALID, "dt2srctf is NULL");
  if ((rc = check_positions(p, possrcs, p->nsrc, "source", err))) return rc;
  if ((rc = check_positions(p, posrecs, p->nrec, "receiver", err))) return rc;
  CUDA_TRY(err, cudaSetDevice(C->device));
  awc_plan* P = new awc_plan();
  P->ctx = C;
  P->p = *p;
  if (p->ndim == 2) P->p.nz = 1;
  if ((rc = plan_alloc(P)) || (rc = plan_upload(P, vel, coeffs, possrcs, dt2srctf, posrecs))) {
    delete P;
    return rc;
  }
  default_tuning(P);
  *out = P;
  return awc_plan_reset(P);
}

bool same_shape(const awc_problem& a, const awc_problem& b) {
  return a.ndim == b.ndim && a.precision == b.precision && a.nx == b.nx && a.ny == b.ny &&
         (a.ndim == 2 || a.nz == b.nz) && a.halo == b.halo && a.nt == b.nt && a.nsrc == b.nsrc &&
         a.nrec == b.nrec;
}

// Reads and clears the device error flag after the stream has drained.
int check_device_flag(awc_plan* P) {
  awc_ctx* C = P->ctx;
  int32_t flag = 0;
  CUDA_TRY(&C->err, cudaMemcpyAsync(&flag, P->err_flag, 4, cudaMemcpyDeviceToHost, C->stream));
  CUDA_TRY(&C->err, cudaStreamSynchronize(C->stream));
  if (flag) {
    CUDA_TRY(&C->err, cudaMemsetAsync(P->err_flag, 0, 4, C->stream));
    return set_err(&C->err, AWC_ERR_TIMEOUT, "a bounded wait on a pipeline barrier ran out");
  }
  return AWC_OK;
}

}  // namespace

namespace awc {
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  return fn;
}

// Sets the calling thread's last error (awc_last_error(NULL)) for entry
// points defined in other translation units.
void record_error(const char* msg) { g_thread_err = msg; }

int fail(awc_ctx* ctx, int code, const char* msg) {
  return set_err(ctx ? &ctx->err : nullptr, code, "%s", msg);
}

PlanView plan_view(awc_plan* P) {
  PlanView V;
  const awc_problem* p = &P->p;
  V.ndim = p->ndim;
  V.precision = p->precision;
  V.halo = p->halo;
  V.nx = p->nx;
  V.ny = p->ny;
  V.nz = p->ndim == 3 ? p->nz : 1;
  V.px = P->px;
  V.NP = P->NP;
  V.nt = p->nt;
  V.esz = P->esz;
  for (int b = 0; b < 3; ++b) V.buf[b] = P->buf[b];
  V.fact = P->fact;
  for (int a = 0; a < p->ndim; ++a) {
    V.psi_len[a] = (p->halo + 1) * cross_section(p, a);
    V.xi_len[a] = p->halo * cross_section(p, a);
    for (int sd = 0; sd < 2; ++sd) {
      V.psi[a][sd][0] = P->psi[a][sd][0];
      V.psi[a][sd][1] = P->psi[a][sd][1];
      V.xi[a][sd] = P->xi[a][sd];
      V.active[a][sd] = P->active[a][sd];
    }
  }
  V.coef = P->coef;
  V.traces = P->traces;
  V.err_flag = P->err_flag;
  V.stream = P->ctx->stream;
  return V;
}

int plan_for(awc_ctx* C, awc_plan** slot, const awc_problem* p, const double* vel,
             const double* coeffs, const int64_t* possrcs, const double* dt2srctf,
             const int64_t* posrecs, bool tune) {
  awc_plan* P = *slot;
  if (P && p && p->ndim != 1 && !P->is1d && same_shape(P->p, *p)) {
    int rc;
    if ((rc = validate(p, &C->err)) ||
        (rc = check_positions(p, possrcs, p->nsrc, "source", &C->err)) ||
        (rc = check_positions(p, posrecs, p->nrec, "receiver", &C->err)))
      return rc;
    if (!vel || !coeffs || (p->nsrc > 0 && p->nt > 0 && !dt2srctf))
      return set_err(&C->err, AWC_ERR_INVALID, "vel/coeffs/dt2srctf is NULL");
    CUDA_TRY(&C->err, cudaSetDevice(C->device));
    P->p = *p;
    if (p->ndim == 2) P->p.nz = 1;
    P->depth = 1;
    if ((rc = plan_upload(P, vel, coeffs, possrcs, dt2srctf, posrecs))) return rc;
    return awc_plan_reset(P);
  }
  if (P) {
    awc_plan_destroy(P);
    *slot = nullptr;
  }
  int rc = awc_plan_create(C, p, vel, coeffs, possrcs, dt2srctf, posrecs, slot);
  if (rc || !tune || p->ndim != 3 || C->autotune_steps <= 0 || p->nt < 100) return rc;
  P = *slot;
  if ((rc = awc_plan_autotune(P, C->autotune_steps, nullptr))) return rc;
  P->depth = 1;
  return awc_plan_reset(P);
}

int plan_shot(awc_ctx* C, awc_plan* P, const int64_t* possrcs, const double* dt2srctf,
              const int64_t* posrecs) {
  const awc_problem* p = &P->p;
  int rc;
  if ((rc = check_positions(p, possrcs, p->nsrc, "source", &C->err)) ||
      (rc = check_positions(p, posrecs, p->nrec, "receiver", &C->err)))
    return rc;
  if (p->nsrc > 0 && p->nt > 0 && !dt2srctf)
    return set_err(&C->err, AWC_ERR_INVALID, "dt2srctf is NULL");
  CUDA_TRY(&C->err, cudaSetDevice(C->device));
  P->depth = 1;
  if ((rc = plan_upload(P, nullptr, nullptr, possrcs, dt2srctf, posrecs))) return rc;
  return awc_plan_reset(P);
}

void plan_set_step(awc_plan* P, int64_t step) {
  P->step = step;
  P->state = StepState::after_steps(step);
}

void plan_keep_fields(awc_plan* P, void* const* dst, int64_t first, int64_t count,
                      bool in_place) {
  P->keep = dst;
  P->keep_first = first;
  P->keep_count = dst ? count : 0;
  P->keep_in_place = dst && in_place;
}
}  // namespace awc

// ---------------------------------------------------------------------------
extern "C" {

int64_t awc_coeffs_len(const awc_problem* p) {
  if (!p || p->ndim < 1 || p->ndim > 3 || p->halo < 0) return 0;
  return (int64_t)p->ndim * (8 * (int64_t)p->halo + 4);
}

int awc_cpml_coeffs(int32_t halo, double dt, double npower, double d0, double alpha_max,
                    double K_max, int32_t halfgrid, double* a_l, double* a_r, double* bK_l,
                    double* bK_r) {
  if (halo < 0) return set_err(nullptr, AWC_ERR_INVALID, "halo must be >= 0");
  if ((halo > 0 || halfgrid) && (!a_l || !a_r || !bK_l || !bK_r))
    return set_err(nullptr, AWC_ERR_INVALID, "output vectors are NULL");
  kab(halo, dt, npower, d0, alpha_max, K_max, halfgrid != 0, a_l, a_r, bK_l, bK_r);
  return AWC_OK;
}

int awc_problem_coeffs(const awc_problem* p, double rcoef, double f0, double vel_max,
                       double* coeffs) {
  int rc = p && p->ndim == 1 ? validate_1d(p, nullptr) : validate(p, nullptr);
  if (rc) return rc;
  if (!coeffs) return set_err(nullptr, AWC_ERR_INVALID, "coeffs is NULL");
  const int64_t h = p->halo;
  const double alpha_max = M_PI * f0, npower = 2.0, K_max = 1.0;
  const double d[3] = {p->dx, p->dy, p->dz};
  for (int a = 0; a < p->ndim; ++a) {
    double* blk = coeffs + a * (8 * h + 4);
    const double thickness = (double)h * d[a];
    const double d0 = -(npower + 1.0) * vel_max * std::log(rcoef) / (2.0 * thickness);
    kab(p->halo, p->dt, npower, d0, alpha_max, K_max, false, blk, blk + h, blk + 2 * h, blk + 3 * h);
    double* hb = blk + 4 * h;
    kab(p->halo, p->dt, npower, d0, alpha_max, K_max, true, hb, hb + (h + 1), hb + 2 * (h + 1),
        hb + 3 * (h + 1));
    if (a == 1 && p->freetop) {
      for (int64_t m = 0; m < h; ++m) {
        blk[m] = 0.0;
        blk[2 * h + m] = 1.0;
      }
      for (int64_t m = 0; m < h + 1; ++m) {
        hb[m] = 0.0;
        hb[2 * (h + 1) + m] = 1.0;
      }
    }
  }
  return AWC_OK;
}

int awc_ricker(int64_t n, const double* t, double t0, double f0, double* out) {
  if (n < 0 || (n > 0 && (!t || !out))) return set_err(nullptr, AWC_ERR_INVALID, "bad arguments");
  for (int64_t m = 0; m < n; ++m) {
    const double x = M_PI * f0 * (t[m] - t0);
    out[m] = (1.0 - 2.0 * (x * x)) * std::exp(-(x * x));
  }
  return AWC_OK;
}

int awc_create(awc_ctx** out, int32_t device) {
  if (!out) return set_err(nullptr, AWC_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return set_err(nullptr, AWC_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
  }
  if (device < 0 || device >= count)
    return set_err(nullptr, AWC_ERR_INVALID, "device %d out of range (%d devices)", device, count);
  cudaDeviceProp prop;
  CUDA_TRY(nullptr, cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return set_err(nullptr, AWC_ERR_NODEVICE, "device %d is sm_%d%d; this build targets sm_100a",
                   device, prop.major, prop.minor);
  CUDA_TRY(nullptr, cudaSetDevice(device));
  if (int rc = init_kernel_attrs(nullptr)) return rc;
  awc_ctx* C = new awc_ctx();
  C->device = device;
  C->num_sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&C->stream2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&C->ev0) != cudaSuccess || cudaEventCreate(&C->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&C->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&C->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    awc_destroy(C);
    return set_err(nullptr, AWC_ERR_CUDA, "stream/event creation failed");
  }
  *out = C;
  return AWC_OK;
}

void awc_destroy(awc_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  for (awc_plan* P : ctx->cache) delete P;
  ctx->cache.clear();
  if (ctx->adj_release) ctx->adj_release();
  ctx->adj_release = nullptr;
  if (ctx->adj_plan) delete ctx->adj_plan;
  ctx->adj_plan = nullptr;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  for (cudaStream_t& a : ctx->adj_stream)
    if (a) {
      cudaStreamSynchronize(a);
      cudaStreamDestroy(a);
    }
  for (cudaEvent_t& e : ctx->adj_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->host_stage) cudaFreeHost(ctx->host_stage);
  delete ctx;
}

const char* awc_last_error(const awc_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_thread_err.c_str();
}

float awc_last_run_ms(const awc_ctx* ctx) { return ctx ? ctx->last_run_ms : 0.f; }

void* awc_ctx_stream(const awc_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int awc_ctx_set_autotune(awc_ctx* ctx, int64_t steps) {
  if (!ctx) return set_err(nullptr, AWC_ERR_INVALID, "ctx is NULL");
  if (steps < 0) return set_err(&ctx->err, AWC_ERR_INVALID, "steps must be >= 0");
  ctx->autotune_steps = steps;
  return AWC_OK;
}

int awc_plan_create(awc_ctx* ctx, const awc_problem* p, const double* vel, const double* coeffs,
                    const int64_t* possrcs, const double* dt2srctf, const int64_t* posrecs,
                    awc_plan** out) {
  if (!ctx || !out) return set_err(nullptr, AWC_ERR_INVALID, "ctx/out is NULL");
  *out = nullptr;
  if (p && p->ndim == 1) {
    int rc;
    if ((rc = validate_1d(p, &ctx->err)) ||
        (rc = check_positions(p, possrcs, p->nsrc, "source", &ctx->err)) ||
        (rc = check_positions(p, posrecs, p->nrec, "receiver", &ctx->err)))
      return rc;
    if (!vel || !coeffs) return set_err(&ctx->err, AWC_ERR_INVALID, "vel/coeffs are NULL");
    Lifted L;
    lift_1d(p, vel, coeffs, possrcs, posrecs, &L);
    if ((rc = forward_impl(ctx, &L.p, L.vel.data(), L.coeffs.data(), L.possrcs.data(), dt2srctf,
                           L.posrecs.data(), out, true)))
      return rc;
    (*out)->is1d = true;
    return AWC_OK;
  }
  return forward_impl(ctx, p, vel, coeffs, possrcs, dt2srctf, posrecs, out);
}

void awc_plan_destroy(awc_plan* plan) {
  if (!plan) return;
  cudaSetDevice(plan->ctx->device);
  cudaStreamSynchronize(plan->ctx->stream);
  delete plan;
}

int awc_plan_reset(awc_plan* P) {
  if (!P) return set_err(nullptr, AWC_ERR_INVALID, "plan is NULL");
  awc_ctx* C = P->ctx;
  const awc_problem* p = &P->p;
  cudaStream_t st = C->stream;
  CUDA_TRY(&C->err, cudaSetDevice(C->device));
  for (int b = 0; b < P->nbuf; ++b)
    CUDA_TRY(&C->err, cudaMemsetAsync(P->buf[b], 0, P->NP * P->esz, st));
  for (int a = 0; a < p->ndim; ++a)
    for (int s = 0; s < 2; ++s) {
      const int64_t cs = cross_section(p, a);
      for (int par = 0; par < 2; ++par)
        CUDA_TRY(&C->err, cudaMemsetAsync(P->psi[a][s][par], 0, (p->halo + 1) * cs * P->esz, st));
      if (p->halo > 0) {
        CUDA_TRY(&C->err, cudaMemsetAsync(P->xi[a][s], 0, p->halo * cs * P->esz, st));
        if (P->xi_alt[a][s])
          CUDA_TRY(&C->err, cudaMemsetAsync(P->xi_alt[a][s], 0, p->halo * cs * P->esz, st));
      }
    }
  if (p->nt * p->nrec > 0)
    CUDA_TRY(&C->err, cudaMemsetAsync(P->traces, 0, p->nt * p->nrec * P->esz, st));
  P->step = 0;
  P->state = StepState();
  return AWC_OK;
}

int awc_plan_run(awc_plan* P, int64_t nsteps, int32_t use_graph, float* ms) {
  if (!P) return set_err(nullptr, AWC_ERR_INVALID, "plan is NULL");
  awc_ctx* C = P->ctx;
  if (nsteps < 0) return set_err(&C->err, AWC_ERR_INVALID, "nsteps < 0");
  CUDA_TRY(&C->err, cudaSetDevice(C->device));
  const int64_t n = std::min<int64_t>(nsteps, P->p.nt - P->step);
  if (ms) *ms = 0.f;
  if (n <= 0) return AWC_OK;
  int rc;
  if ((rc = prepare_launch(P))) return rc;
  cudaGraphExec_t ex = nullptr;
  if (use_graph && (rc = get_graph(P, P->step, n, &ex))) return rc;
  CUDA_TRY(&C->err, cudaEventRecord(C->ev0, C->stream));
  if (use_graph) {
    CUDA_TRY(&C->err, cudaGraphLaunch(ex, C->stream));
  }
  StepState end = P->state;
  if (!use_graph) {
    if ((rc = launch_range(P, P->step, n, end, C->stream))) return rc;
  } else {
    for (int64_t it = P->step; it < P->step + n;) {  // the state the graph leaves
      if (two_step(P) && it + 1 < P->step + n) {
        end.pass2();
        it += 2;
      } else {
        end.step1();
        ++it;
      }
    }
  }
  CUDA_TRY(&C->err, cudaEventRecord(C->ev1, C->stream));
  CUDA_TRY(&C->err, cudaEventSynchronize(C->ev1));
  if (ms) CUDA_TRY(&C->err, cudaEventElapsedTime(ms, C->ev0, C->ev1));
  P->step += n;
  P->state = end;
  return check_device_flag(P);
}

int64_t awc_plan_step(const awc_plan* P) { return P ? P->step : -1; }

int awc_plan_run_snapshots(awc_plan* P, int64_t nsteps, int64_t nsave, double* out,
                           int64_t max_snaps, int64_t* nsnaps) {
  if (!P) return set_err(nullptr, AWC_ERR_INVALID, "plan is NULL");
  awc_ctx* C = P->ctx;
  if (nsnaps) *nsnaps = 0;
  if (nsteps < 0 || nsave < 1 || max_snaps < 0)
    return set_err(&C->err, AWC_ERR_INVALID, "nsteps >= 0, nsave >= 1 and max_snaps >= 0 needed");
  const int64_t n = std::min<int64_t>(nsteps, P->p.nt - P->step);
  if (n <= 0) return AWC_OK;
  const int64_t first = P->step, last = P->step + n;  // steps first+1 .. last complete
  const int64_t count = last / nsave - first / nsave;
  if (count > max_snaps)
    return set_err(&C->err, AWC_ERR_INVALID,
                   "%lld snapshots fall in this run but out holds %lld",
                   (long long)count, (long long)max_snaps);
  if (count > 0 && !out) return set_err(&C->err, AWC_ERR_INVALID, "out is NULL");
  CUDA_TRY(&C->err, cudaSetDevice(C->device));
  int rc;
  if ((rc = prepare_launch(P))) return rc;
  // two device staging slots of N doubles: the unpitched copy of snapshot k
  // goes to slot k % 2, then to the host on the second stream while the next
  // steps run
  if (count > 0 && !P->snap_staging && (rc = P->alloc((void**)&P->snap_staging, 2 * P->N * 8)))
    return rc;
  cudaEvent_t ready = nullptr, copied[2] = {nullptr, nullptr};
  auto cleanup = [&]() {
    if (ready) cudaEventDestroy(ready);
    for (cudaEvent_t e : copied)
      if (e) cudaEventDestroy(e);
  };
  if (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&copied[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&copied[1], cudaEventDisableTiming) != cudaSuccess) {
    cleanup();
    return set_err(&C->err, AWC_ERR_CUDA, "event creation failed");
  }
  StepState stt = P->state;
  int64_t it = first, k = 0;
  bool used[2] = {false, false};
  const int blocks = grid_for(C, P->N, 256);
  while (it < last) {
    const int64_t next = std::min<int64_t>(last, (it / nsave + 1) * nsave);
    if ((rc = launch_range(P, it, next - it, stt, C->stream))) {
      cleanup();
      return rc;
    }
    it = next;
    if (it % nsave != 0) continue;
    const int slot = (int)(k & 1);
    const int64_t nf = P->is1d ? P->p.nx : P->N;  // values per snapshot
    double* dst = P->snap_staging + slot * P->N;
    const size_t row = P->is1d ? (size_t)P->px * P->esz : 0;  // a 1D plan's line is row 1
    cudaError_t e = cudaSuccess;
    if (used[slot]) e = cudaStreamWaitEvent(C->stream, copied[slot], 0);
    if (e == cudaSuccess) {
      const char* src = (const char*)P->buf[stt.ord[0]] + row;
      if (P->p.precision == AWC_F64)
        awc::unpitch<double><<<blocks, 256, 0, C->stream>>>((const double*)src, dst, nf,
                                                            P->p.nx, P->px);
      else
        awc::unpitch<float><<<blocks, 256, 0, C->stream>>>((const float*)src, dst, nf, P->p.nx,
                                                           P->px);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(ready, C->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(C->stream2, ready, 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out + k * nf, dst, nf * 8, cudaMemcpyDeviceToHost, C->stream2);
    if (e == cudaSuccess) e = cudaEventRecord(copied[slot], C->stream2);
    if (e != cudaSuccess) {
      cudaStreamSynchronize(C->stream2);
      cudaStreamSynchronize(C->stream);
      cleanup();
      return set_err(&C->err, AWC_ERR_CUDA, "snapshot copy failed: %s", cudaGetErrorString(e));
    }
    used[slot] = true;
    ++k;
  }
  const cudaError_t e1 = cudaStreamSynchronize(C->stream2), e2 = cudaStreamSynchronize(C->stream);
  cleanup();
  if (e1 != cudaSuccess || e2 != cudaSuccess)
    return set_err(&C->err, AWC_ERR_CUDA, "snapshot run failed: %s",
                   cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
  P->step = last;
  P->state = stt;
  if (nsnaps) *nsnaps = k;
  return check_device_flag(P);
}

int awc_plan_traces(awc_plan* P, double* traces) {
  if (!P || !traces) return set_err(nullptr, AWC_ERR_INVALID, "plan/traces is NULL");
  awc_ctx* C = P->ctx;
  const int64_t nt = P->p.nt, nrec = P->p.nrec;
  if (nt * nrec == 0) return AWC_OK;
  CUDA_TRY(&C->err, cudaSetDevice(C->device));
  dim3 grid((unsigned)((nt + 31) / 32), (unsigned)((nrec + 31) / 32));
  if (P->p.precision == AWC_F64)
    awc::traces_out<double><<<grid, dim3(32, 8), 0, C->stream>>>((const double*)P->traces, P->staging, nt, nrec);
  else
    awc::traces_out<float><<<grid, dim3(32, 8), 0, C->stream>>>((const float*)P->traces, P->staging, nt, nrec);
  CUDA_TRY(&C->err, cudaGetLastError());
  CUDA_TRY(&C->err, awc::copy_to_host(C, traces, P->staging, nt * nrec * 8, C->stream));
  return AWC_OK;
}

int awc_plan_field(awc_plan* P, double* out) {
  if (!P || !out) return set_err(nullptr, AWC_ERR_INVALID, "plan/out is NULL");
  awc_ctx* C = P->ctx;
  CUDA_TRY(&C->err, cudaSetDevice(C->device));
  // the latest new field (the reference's pcur); a 1D plan's line is row 1
  const int64_t n = P->is1d ? P->p.nx : P->N;
  const char* cur = (const char*)P->buf[P->state.ord[0]] + (P->is1d ? P->px * P->esz : 0);
  const int blocks = grid_for(C, n, 256);
  if (P->p.precision == AWC_F64)
    awc::unpitch<double><<<blocks, 256, 0, C->stream>>>((const double*)cur, P->staging, n, P->p.nx, P->px);
  else
    awc::unpitch<float><<<blocks, 256, 0, C->stream>>>((const float*)cur, P->staging, n, P->p.nx, P->px);
  CUDA_TRY(&C->err, cudaGetLastError());
  CUDA_TRY(&C->err, awc::copy_to_host(C, out, P->staging, n * 8, C->stream));
  return AWC_OK;
}

int32_t awc_plan_launches_per_step(const awc_plan* P) {
  if (!P) return 0;
  return (P->p.ndim == 3 && P->has_core && P->nbox > 0) ? 2 : 1;
}

int awc_plan_set_launch(awc_plan* P, int32_t tile_y, int32_t zchunk, int32_t band_zchunk) {
  if (!P) return set_err(nullptr, AWC_ERR_INVALID, "plan is NULL");
  if (tile_y != 4 && tile_y != 8 && tile_y != 16)
    return set_err(&P->ctx->err, AWC_ERR_INVALID, "tile_y must be 4, 8 or 16");
  if (zchunk < 1 || band_zchunk < 1 || band_zchunk > 255)
    return set_err(&P->ctx->err, AWC_ERR_INVALID, "zchunk must be >= 1, band_zchunk in [1, 255]");
  if (P->p.ndim == 3) {
    P->by = tile_y;
    P->zchunk = (int32_t)std::min<int64_t>(zchunk, P->p.nz - 2);
    P->szc = band_zchunk;
    box_blocks(P);
  }
  return AWC_OK;
}

int awc_plan_get_launch(const awc_plan* P, int32_t* tile_y, int32_t* zchunk, int32_t* band_zchunk) {
  if (!P || !tile_y || !zchunk || !band_zchunk)
    return set_err(nullptr, AWC_ERR_INVALID, "NULL argument");
  *tile_y = P->by;
  *zchunk = P->zchunk;
  *band_zchunk = P->szc;
  return AWC_OK;
}

int awc_plan_set_blocking(awc_plan* P, int32_t depth, int32_t rows, int32_t zchunks) {
  if (!P) return set_err(nullptr, AWC_ERR_INVALID, "plan is NULL");
  if (depth != 1 && depth != 2)
    return set_err(&P->ctx->err, AWC_ERR_INVALID, "depth must be 1 or 2");
  if (rows != 8 && rows != 16) return set_err(&P->ctx->err, AWC_ERR_INVALID, "rows must be 8 or 16");
  if (zchunks < 1) return set_err(&P->ctx->err, AWC_ERR_INVALID, "zchunks must be >= 1");
  if (depth == 2 && !tb_eligible(P))
    return set_err(&P->ctx->err, AWC_ERR_INVALID,
                   "two-step passes need a 3D problem whose sources and receivers are all "
                   "interior nodes");
  P->depth = depth;
  P->tb_rows = rows;
  if (P->p.ndim == 3) P->tb_nch = tb_chunks(P, zchunks);
  return AWC_OK;
}

int awc_plan_get_blocking(const awc_plan* P, int32_t* depth, int32_t* rows, int32_t* zchunks) {
  if (!P || !depth || !rows || !zchunks) return set_err(nullptr, AWC_ERR_INVALID, "NULL argument");
  *depth = P->depth;
  *rows = P->tb_rows;
  *zchunks = P->tb_nch;
  return AWC_OK;
}

int awc_plan_set_wait(awc_plan* P, int32_t rounds, int32_t round_ns, int32_t withhold) {
  if (!P) return set_err(nullptr, AWC_ERR_INVALID, "plan is NULL");
  if (rounds < 1 || round_ns < 1 || round_ns > 10000000 || withhold < -1)
    return set_err(&P->ctx->err, AWC_ERR_INVALID,
                   "rounds >= 1, round_ns in [1, 1e7] and withhold >= -1 are required");
  P->wait_rounds = rounds;
  P->wait_ns = round_ns;
  P->withhold = withhold;
  return AWC_OK;
}

int64_t awc_plan_launch_count(const awc_plan* P, int64_t nsteps) {
  if (!P || nsteps < 0) return -1;
  // the tile lists (how many launches a pass has) follow the blocking
  if (two_step(P) && ensure_tb(const_cast<awc_plan*>(P)) != AWC_OK) return -1;
  return launch_count(P, std::min<int64_t>(nsteps, P->p.nt - P->step));
}

namespace {
// Device time per step [ms] of the current launch shape: the faster of two
// runs of n steps (the state is reset before and is garbage after).
int time_shape(awc_plan* P, int64_t n, float* per) {
  int rc;
  *per = 1e30f;
  // replays of a captured run, as the solves run (the capture is not timed)
  for (int rep = 0; rep < 2; ++rep) {
    if ((rc = awc_plan_reset(P)) || (rc = awc_plan_run(P, 2, 0, nullptr))) return rc;  // warm-up
    float ms = 0.f;
    if ((rc = awc_plan_run(P, n, 1, &ms))) return rc;
    *per = std::min(*per, ms / (float)n);
  }
  return AWC_OK;
}
}  // namespace

int awc_plan_autotune(awc_plan* P, int64_t steps, float* best_ms_per_step) {
  if (!P) return set_err(nullptr, AWC_ERR_INVALID, "plan is NULL");
  awc_ctx* C = P->ctx;
  if (steps < 1) return set_err(&C->err, AWC_ERR_INVALID, "steps must be >= 1");
  if (P->p.ndim != 3 || P->p.nt < 2) {
    if (best_ms_per_step) *best_ms_per_step = 0.f;
    return AWC_OK;
  }
  // an even number of timed steps (two-step passes), after 2 warm-up steps
  const int64_t n = std::max<int64_t>(2, std::min<int64_t>(steps, P->p.nt - 2) / 2 * 2);
  if (P->p.nt < n + 2) {
    if (best_ms_per_step) *best_ms_per_step = 0.f;
    return AWC_OK;
  }
  int rc;
  P->depth = 1;
  // phase 1: core tile height and z chunk
  std::vector<std::pair<int32_t, int32_t>> cands;
  for (int by : {4, 8, 16})
    for (double waves : {0.5, 1.0, 2.0, 4.0, 8.0}) {
      const std::pair<int32_t, int32_t> c{by, chunk_for(P, by, waves)};
      if (std::find(cands.begin(), cands.end(), c) == cands.end()) cands.push_back(c);
    }
  float best = 1e30f;
  std::pair<int32_t, int32_t> win{P->by, P->zchunk};
  for (const auto& c : cands) {
    P->by = c.first;
    P->zchunk = c.second;
    float per = 0.f;
    if ((rc = time_shape(P, n, &per))) return rc;
    if (per < best) {
      best = per;
      win = c;
    }
  }
  P->by = win.first;
  P->zchunk = win.second;
  // phase 2: z planes per block of the band kernel
  if (P->nbox > 0) {
    int32_t wz = P->szc;
    for (int32_t zc : {4, 6, 8, 10, 12, 16, 20, 24, 28, 30, 32, 36, 40}) {
      P->szc = zc;
      box_blocks(P);
      float per = 0.f;
      if ((rc = time_shape(P, n, &per))) return rc;
      if (per < best) {
        best = per;
        wz = zc;
      }
    }
    P->szc = wz;
    box_blocks(P);
    // the core z chunk again, next to its winner, with the band's chunk set
    const int32_t zc0 = P->zchunk;
    int32_t wc = zc0;
    for (int32_t d : {-2, -1, 1, 2}) {
      if (zc0 + d < 1) continue;
      P->zchunk = zc0 + d;
      float per = 0.f;
      if ((rc = time_shape(P, n, &per))) return rc;
      if (per < best) {
        best = per;
        wc = zc0 + d;
      }
    }
    P->zchunk = wc;
  }
  // phase 3: two-step passes, z chunks per column tile
  if (tb_eligible(P)) {
    int32_t wdepth = 1, wrows = P->tb_rows, wch = P->tb_nch;
    for (int32_t rows : {16, 8}) {
      const int64_t ty = rows - 2;
      const int64_t ntiles = ((P->p.nx - 2 + TB_TX - 1) / TB_TX) * ((P->p.ny - 2 + ty - 1) / ty);
      const int64_t resident =
          (int64_t)C->num_sms * awc::tb_occupancy(P->p.precision == AWC_F64, false, rows);
      std::vector<int32_t> chs;
      for (double waves : {1.0, 2.0, 3.0, 4.0, 6.0}) {
        const int32_t c = tb_chunks(P, std::llround(waves * (double)resident / (double)ntiles));
        if (std::find(chs.begin(), chs.end(), c) == chs.end()) chs.push_back(c);
      }
      for (int32_t c : chs) {
        P->depth = 2;
        P->tb_rows = rows;
        P->tb_nch = c;
        float per = 0.f;
        if ((rc = time_shape(P, n, &per))) return rc;
        if (per < best) {
          best = per;
          wdepth = 2;
          wrows = rows;
          wch = c;
        }
      }
    }
    P->depth = wdepth;
    P->tb_rows = wrows;
    P->tb_nch = wch;
  }
  if (best_ms_per_step) *best_ms_per_step = best;
  return awc_plan_reset(P);
}

int awc_forward(awc_ctx* ctx, const awc_problem* p, const double* vel, const double* coeffs,
                const int64_t* possrcs, const double* dt2srctf, const int64_t* posrecs,
                double* traces, double* pfinal) {
  if (!ctx) return set_err(nullptr, AWC_ERR_INVALID, "ctx is NULL");
  if (p && p->ndim == 1) {
    int rc;
    if ((rc = validate_1d(p, &ctx->err)) ||
        (rc = check_positions(p, possrcs, p->nsrc, "source", &ctx->err)) ||
        (rc = check_positions(p, posrecs, p->nrec, "receiver", &ctx->err)))
      return rc;
    if (!vel || !coeffs) return set_err(&ctx->err, AWC_ERR_INVALID, "vel/coeffs are NULL");
    awc_plan* P = nullptr;
    if ((rc = awc_plan_create(ctx, p, vel, coeffs, possrcs, dt2srctf, posrecs, &P))) return rc;
    rc = awc_plan_run(P, p->nt, 1, &ctx->last_run_ms);
    if (!rc && traces) rc = awc_plan_traces(P, traces);
    if (!rc && pfinal) rc = awc_plan_field(P, pfinal);
    awc_plan_destroy(P);
    return rc;
  }
  int rc = validate(p, &ctx->err);
  if (rc) return rc;
  if (p->nt * p->nrec > 0 && !traces) return set_err(&ctx->err, AWC_ERR_INVALID, "traces is NULL");
  // reuse a cached plan of the same shape: same buffers, same graphs
  awc_plan* P = nullptr;
  for (size_t c = 0; c < ctx->cache.size(); ++c)
    if (same_shape(ctx->cache[c]->p, *p)) {
      P = ctx->cache[c];
      ctx->cache.erase(ctx->cache.begin() + c);
      break;
    }
  if (P) {
    if ((rc = check_positions(p, possrcs, p->nsrc, "source", &ctx->err)) ||
        (rc = check_positions(p, posrecs, p->nrec, "receiver", &ctx->err))) {
      ctx->cache.push_back(P);
      return rc;
    }
    if (!vel || !coeffs || (p->nsrc > 0 && p->nt > 0 && !dt2srctf)) {
      ctx->cache.push_back(P);
      return set_err(&ctx->err, AWC_ERR_INVALID, "vel/coeffs/dt2srctf is NULL");
    }
    P->p = *p;
    if (p->ndim == 2) P->p.nz = 1;
    if ((rc = plan_upload(P, vel, coeffs, possrcs, dt2srctf, posrecs)) || (rc = awc_plan_reset(P))) {
      delete P;
      return rc;
    }
  } else {
    if ((rc = forward_impl(ctx, p, vel, coeffs, possrcs, dt2srctf, posrecs, &P))) return rc;
    // a new 3D shape: pick its launch shape once, on its own data
    if (p->ndim == 3 && ctx->autotune_steps > 0 && p->nt >= 100 &&
        (rc = awc_plan_autotune(P, ctx->autotune_steps, nullptr))) {
      delete P;
      return rc;
    }
  }
  ctx->cache.push_back(P);
  while (ctx->cache.size() > 2) {
    delete ctx->cache.front();
    ctx->cache.erase(ctx->cache.begin());
  }
  if ((rc = awc_plan_run(P, p->nt, 1, &ctx->last_run_ms))) return rc;
  if (traces && (rc = awc_plan_traces(P, traces))) return rc;
  if (pfinal && (rc = awc_plan_field(P, pfinal))) return rc;
  return AWC_OK;
}

int awc_forward_decomposed(awc_ctx* const* ctxs, int32_t nsub, const awc_problem* p,
                           const double* vel, const double* coeffs, const int64_t* possrcs,
                           const double* dt2srctf, const int64_t* posrecs, double* traces,
                           double* pfinal) {
  std::string terr;
  if (!ctxs || nsub < 1) return set_err(nullptr, AWC_ERR_INVALID, "ctxs is NULL or nsub < 1");
  for (int32_t s = 0; s < nsub; ++s)
    if (!ctxs[s]) return set_err(nullptr, AWC_ERR_INVALID, "ctxs[%d] is NULL", s);
  awc_ctx* C0 = ctxs[0];
  int rc;
  if ((rc = validate(p, &C0->err))) return rc;
  if (!vel || !coeffs) return set_err(&C0->err, AWC_ERR_INVALID, "vel/coeffs are NULL");
  if (p->nsrc > 0 && p->nt > 0 && !dt2srctf)
    return set_err(&C0->err, AWC_ERR_INVALID, "dt2srctf is NULL");
  if ((rc = check_positions(p, possrcs, p->nsrc, "source", &C0->err)) ||
      (rc = check_positions(p, posrecs, p->nrec, "receiver", &C0->err)))
    return rc;
  if (p->nt * p->nrec > 0 && !traces) return set_err(&C0->err, AWC_ERR_INVALID, "traces is NULL");
  const int ax = p->ndim - 1;  // the split axis: y in 2D, z in 3D
  const int64_t nx = p->nx, ny = p->ny, nz = p->ndim == 3 ? p->nz : 1;
  const int64_t n = ax == 2 ? nz : ny, ni = n - 2, h = p->halo;
  // contiguous interior ranges [a_s, b_s] (global, 0-based) of nearly equal size
  std::vector<int64_t> a(nsub), b(nsub);
  for (int32_t s = 0; s < nsub; ++s) {
    a[s] = 1 + ni * s / nsub;
    b[s] = ni * (s + 1) / nsub;
    if (b[s] < a[s])
      return set_err(&C0->err, AWC_ERR_INVALID, "%d subdomains for %lld interior planes",
                     nsub, (long long)ni);
  }
  // the outer subdomains hold the whole CPML band of the split axis
  if (nsub > 1 && h > 0 && (b[0] - a[0] + 3 < 2 * h + 2 || b[nsub - 1] - a[nsub - 1] + 3 < 2 * h + 2))
    return set_err(&C0->err, AWC_ERR_INVALID,
                   "the first and last subdomains need at least 2 halo + 2 planes along the "
                   "split axis (use fewer subdomains)");
  const int64_t clen = awc_coeffs_len(p), blk = 8 * h + 4;
  auto plane_of = [&](const int64_t* pos, int64_t cnt, int64_t r) { return pos[r + cnt * ax] - 1; };
  auto owner = [&](int64_t g) -> int32_t {  // subdomain holding global plane g
    if (g <= a[0]) return 0;
    for (int32_t s = 0; s < nsub; ++s)
      if (g >= a[s] && g <= b[s]) return s;
    return nsub - 1;  // the far rim plane
  };
  struct Sub {
    awc_problem p{};
    std::vector<double> vel, coeffs, stf;
    std::vector<int64_t> ps, pr, sid, rid;
    awc_plan* plan = nullptr;
    cudaEvent_t stepped = nullptr, filled = nullptr;
  };
  std::vector<Sub> sub(nsub);
  auto cleanup = [&]() {
    for (Sub& u : sub) {
      if (u.plan) awc_plan_destroy(u.plan);
      if (u.stepped) cudaEventDestroy(u.stepped);
      if (u.filled) cudaEventDestroy(u.filled);
    }
  };
  for (int32_t s = 0; s < nsub; ++s) {
    Sub& u = sub[s];
    const int64_t g0 = a[s] - 1, nl = b[s] - a[s] + 3;  // local plane l = global g0 + l
    u.p = *p;
    (ax == 2 ? u.p.nz : u.p.ny) = nl;
    u.p.freetop = ax == 1 && s > 0 ? 0 : p->freetop;
    // velocity slab
    const int64_t per = ax == 2 ? nx * ny : nx;          // values per plane
    const int64_t rows = ax == 2 ? 1 : 1, outer = ax == 2 ? 1 : nz;  // 2D: one "outer" block
    (void)rows;
    u.vel.resize((size_t)(per * nl * outer));
    for (int64_t o = 0; o < outer; ++o)
      for (int64_t l = 0; l < nl; ++l)
        std::memcpy(&u.vel[(size_t)((o * nl + l) * per)], vel + (o * n + g0 + l) * per,
                    per * sizeof(double));
    // CPML coefficients: the split axis keeps only the outer sides' bands
    u.coeffs.assign(coeffs, coeffs + clen);
    double* zb = u.coeffs.data() + ax * blk;
    for (int side = 0; side < 2; ++side) {
      const bool inner = side == 0 ? s > 0 : s < nsub - 1;
      if (!inner) continue;
      for (int64_t m = 0; m < h; ++m) {
        zb[side * h + m] = 0.0;
        zb[2 * h + side * h + m] = 1.0;
      }
      for (int64_t m = 0; m < h + 1; ++m) {
        zb[4 * h + side * (h + 1) + m] = 0.0;
        zb[4 * h + 2 * (h + 1) + side * (h + 1) + m] = 1.0;
      }
    }
    // the sources and receivers this subdomain owns, in local coordinates
    auto take = [&](const int64_t* pos, int64_t cnt, std::vector<int64_t>& out,
                    std::vector<int64_t>& ids) {
      ids.clear();
      for (int64_t r = 0; r < cnt; ++r)
        if (owner(plane_of(pos, cnt, r)) == s) ids.push_back(r);
      const int64_t m = (int64_t)ids.size();
      out.assign((size_t)std::max<int64_t>(m * p->ndim, 1), 1);
      for (int64_t e = 0; e < m; ++e)
        for (int d = 0; d < p->ndim; ++d)
          out[e + m * d] = pos[ids[e] + cnt * d] - (d == ax ? g0 : 0);
    };
    take(possrcs, p->nsrc, u.ps, u.sid);
    take(posrecs, p->nrec, u.pr, u.rid);
    u.p.nsrc = (int64_t)u.sid.size();
    u.p.nrec = (int64_t)u.rid.size();
    u.stf.assign((size_t)std::max<int64_t>(p->nt * u.p.nsrc, 1), 0.0);
    for (size_t e = 0; e < u.sid.size(); ++e)
      std::memcpy(&u.stf[e * p->nt], dt2srctf + u.sid[e] * p->nt, p->nt * sizeof(double));
    if ((rc = awc_plan_create(ctxs[s], &u.p, u.vel.data(), u.coeffs.data(), u.ps.data(),
                              u.stf.data(), u.pr.data(), &u.plan))) {
      cleanup();
      return rc;
    }
    awc_ctx* C = ctxs[s];
    if (cudaSetDevice(C->device) != cudaSuccess ||
        cudaEventCreateWithFlags(&u.stepped, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&u.filled, cudaEventDisableTiming) != cudaSuccess ||
        (rc = prepare_launch(u.plan))) {
      cleanup();
      return rc ? rc : set_err(&C->err, AWC_ERR_CUDA, "event creation failed");
    }
  }
  // time loop: every subdomain advances one step, then the planes next to
  // each interface cross it (one-plane halo exchange, update_halo! of
  // acoustic_3D_multixPU.jl:221): subdomain s's last interior plane becomes
  // s+1's plane 0, s+1's first interior plane becomes s's last plane
  auto plane_ptr = [&](Sub& u, int64_t l) {
    awc_plan* P = u.plan;
    const int64_t stride = ax == 2 ? P->px * ny : P->px;  // elements per plane
    return (char*)P->buf[P->state.ord[0]] + l * stride * P->esz;
  };
  const size_t plane_bytes = (size_t)((ax == 2 ? sub[0].plan->px * ny : sub[0].plan->px) *
                                      sub[0].plan->esz);
  for (int64_t it = 0; it < p->nt; ++it) {
    for (int32_t s = 0; s < nsub; ++s) {
      Sub& u = sub[s];
      awc_ctx* C = ctxs[s];
      cudaSetDevice(C->device);
      if (it > 0)  // the copies into and out of this subdomain's planes are done
        for (int32_t t : {s - 1, s + 1})
          if (t >= 0 && t < nsub && cudaStreamWaitEvent(C->stream, sub[t].filled, 0) != cudaSuccess) {
            cleanup();
            return set_err(&C->err, AWC_ERR_CUDA, "stream wait failed");
          }
      StepState stt = u.plan->state;
      if ((rc = launch_range(u.plan, it, 1, stt, C->stream))) {
        cleanup();
        return rc;
      }
      u.plan->state = stt;
      u.plan->step = it + 1;
      cudaEventRecord(u.stepped, C->stream);
    }
    for (int32_t s = 0; s < nsub; ++s) {
      Sub& u = sub[s];
      awc_ctx* C = ctxs[s];
      cudaSetDevice(C->device);
      const int64_t nl = ax == 2 ? u.p.nz : u.p.ny;
      cudaError_t e = cudaSuccess;
      if (s > 0) {  // plane 0 <- the left neighbour's last interior plane
        Sub& v = sub[s - 1];
        const int64_t nv = ax == 2 ? v.p.nz : v.p.ny;
        e = cudaStreamWaitEvent(C->stream, v.stepped, 0);
        if (e == cudaSuccess)
          e = cudaMemcpyPeerAsync(plane_ptr(u, 0), C->device, plane_ptr(v, nv - 2),
                                  ctxs[s - 1]->device, plane_bytes, C->stream);
      }
      if (e == cudaSuccess && s + 1 < nsub) {  // last plane <- the right neighbour's plane 1
        Sub& v = sub[s + 1];
        e = cudaStreamWaitEvent(C->stream, v.stepped, 0);
        if (e == cudaSuccess)
          e = cudaMemcpyPeerAsync(plane_ptr(u, nl - 1), C->device, plane_ptr(v, 1),
                                  ctxs[s + 1]->device, plane_bytes, C->stream);
      }
      if (e == cudaSuccess) e = cudaEventRecord(u.filled, C->stream);
      if (e != cudaSuccess) {
        cleanup();
        return set_err(&C->err, AWC_ERR_CUDA, "halo exchange failed: %s", cudaGetErrorString(e));
      }
    }
  }
  for (int32_t s = 0; s < nsub; ++s) {
    cudaSetDevice(ctxs[s]->device);
    if (cudaStreamSynchronize(ctxs[s]->stream) != cudaSuccess ||
        (rc = check_device_flag(sub[s].plan))) {
      cleanup();
      return rc ? rc : set_err(&ctxs[s]->err, AWC_ERR_CUDA, "decomposed run failed");
    }
  }
  // outputs: each subdomain's receivers, and its interior planes of the field
  for (int32_t s = 0; s < nsub && p->nt * p->nrec > 0; ++s) {
    Sub& u = sub[s];
    if (u.p.nrec == 0) continue;
    std::vector<double> tr((size_t)(p->nt * u.p.nrec));
    if ((rc = awc_plan_traces(u.plan, tr.data()))) {
      cleanup();
      return rc;
    }
    for (size_t e = 0; e < u.rid.size(); ++e)
      std::memcpy(traces + u.rid[e] * p->nt, &tr[e * p->nt], p->nt * sizeof(double));
  }
  if (pfinal) {
    const int64_t per = ax == 2 ? nx * ny : nx, outer = ax == 2 ? 1 : nz;
    for (int32_t s = 0; s < nsub; ++s) {
      Sub& u = sub[s];
      const int64_t nl = ax == 2 ? u.p.nz : u.p.ny, g0 = a[s] - 1;
      std::vector<double> f((size_t)(per * nl * outer));
      if ((rc = awc_plan_field(u.plan, f.data()))) {
        cleanup();
        return rc;
      }
      const int64_t l0 = s == 0 ? 0 : 1, l1 = s == nsub - 1 ? nl - 1 : nl - 2;
      for (int64_t o = 0; o < outer; ++o)
        for (int64_t l = l0; l <= l1; ++l)
          std::memcpy(pfinal + (o * n + g0 + l) * per, &f[(size_t)((o * nl + l) * per)],
                      per * sizeof(double));
    }
  }
  cleanup();
  return AWC_OK;
}

}  // extern "C"
