// awc_batch.cu — batched 2D shots over several velocity models.
//
// Many shots (sources) over velocity models of uneven size advance together:
// one kernel launch per time step covers every shot (a persistent grid over
// the global tile list, awc::step2d_batch), and the nt-step loop is captured
// once into a CUDA graph. Each shot computes exactly what a single-shot
// awc_forward of the same problem computes (the same per-node arithmetic).
// The reference has no batched API: its solve2D runs one shot per call
// (src/shared/acoustic_2D_xPU.jl:133-445).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/awcpml.h"
#include "awc_ctx.h"
#include "awc_kernels.cuh"

namespace {

int64_t pitch32(int64_t n) { return (n + 31) / 32 * 32; }
size_t up256(size_t b) { return (b + 255) / 256 * 256; }

#define BATCH_TRY(ctx, call)                                                              \
  do {                                                                                    \
    const cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                              \
      cudaGetLastError();                                                                 \
      return awc::fail(ctx, e_ == cudaErrorMemoryAllocation ? AWC_ERR_OOM : AWC_ERR_CUDA, \
                       cudaGetErrorString(e_));                                           \
    }                                                                                     \
  } while (0)

}  // namespace

struct awc_batch {
  awc_ctx* ctx = nullptr;
  int32_t nmodels = 0, nshots = 0;
  int32_t prec = AWC_F32;
  size_t esz = 4;
  int64_t nt = 0;
  std::vector<awc_problem> models;
  std::vector<awc_shot> shots;          // host copy (input pointers not kept)
  std::vector<int32_t> shot_nsrc, shot_nrec;
  std::vector<int32_t> active;          // [shot][axis][side]
  // device arena and the offsets of every region in it
  unsigned char* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<size_t> m_fact;           // per model
  struct ShotMem {
    size_t buf[3], psi[2][2][2], xi[2][2], stf, traces, src_off, src_ids, rec_off, rec_ids,
        rim, blk_off, ent, coef;
    int64_t max_tiles;
  };
  std::vector<ShotMem> sm;
  size_t descs = 0, tile_start = 0, maps = 0, err = 0;
  // per-shot source/receiver nodes (pitched index, groups)
  std::vector<std::vector<awc::IoRim>> io_nodes;
  // launch shape
  int32_t ty = 32, bps = 8, ntiles = 0;
  int32_t io_ty = 0;  // tile height the device lists were built for
  std::map<int32_t, int> occ;  // tile height -> resident blocks per SM
  int64_t step = 0;
  std::map<std::pair<int64_t, int64_t>, cudaGraphExec_t> graphs;
  uint64_t graph_key = 0;
  double* staging = nullptr;  // inside the arena (read-out)
  int64_t staging_len = 0;

  ~awc_batch() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    if (arena) cudaFree(arena);
  }
};

namespace {

int check_batch(awc_ctx* C, int32_t nmodels, const awc_problem* models, const double* const* vel,
                int32_t nshots, const awc_shot* shots) {
  if (nmodels < 1 || nshots < 1 || !models || !vel || !shots)
    return awc::fail(C, AWC_ERR_INVALID, "a batch needs at least one model and one shot");
  const awc_problem& m0 = models[0];
  for (int32_t m = 0; m < nmodels; ++m) {
    const awc_problem& p = models[m];
    if (p.ndim != 2 || p.nz != 1)
      return awc::fail(C, AWC_ERR_INVALID, "batched shots are 2D (ndim = 2, nz = 1)");
    if (p.precision != m0.precision || p.nt != m0.nt)
      return awc::fail(C, AWC_ERR_INVALID, "all models of a batch share precision and nt");
    if (p.precision != AWC_F32 && p.precision != AWC_F64)
      return awc::fail(C, AWC_ERR_INVALID, "precision must be AWC_F32 or AWC_F64");
    if (p.nx < 3 || p.ny < 3 || p.nx > (1 << 24) || p.ny > (1 << 24))
      return awc::fail(C, AWC_ERR_INVALID, "grid size must be in [3, 2^24] per axis");
    if (p.halo < 0 || p.halo > p.nx - 2 || p.halo > p.ny - 2)
      return awc::fail(C, AWC_ERR_INVALID, "halo out of range for a model");
    if (!(p.dx > 0.0) || !(p.dy > 0.0) || !(p.dt > 0.0) || p.nt < 0)
      return awc::fail(C, AWC_ERR_INVALID, "spacing and dt must be positive, nt >= 0");
    if (!vel[m]) return awc::fail(C, AWC_ERR_INVALID, "vel of a model is NULL");
  }
  for (int32_t s = 0; s < nshots; ++s) {
    const awc_shot& sh = shots[s];
    if (sh.model < 0 || sh.model >= nmodels)
      return awc::fail(C, AWC_ERR_INVALID, "a shot names a model that does not exist");
    if (!sh.coeffs) return awc::fail(C, AWC_ERR_INVALID, "a shot's coeffs is NULL");
    if (sh.nsrc < 0 || sh.nrec < 0 || (sh.nsrc > 0 && (!sh.possrcs || (m0.nt > 0 && !sh.dt2srctf))) ||
        (sh.nrec > 0 && !sh.posrecs))
      return awc::fail(C, AWC_ERR_INVALID, "a shot's sources/receivers are inconsistent");
    const awc_problem& p = models[sh.model];
    for (int32_t k = 0; k < sh.nsrc; ++k)
      if (sh.possrcs[k] < 1 || sh.possrcs[k] > p.nx || sh.possrcs[k + sh.nsrc] < 1 ||
          sh.possrcs[k + sh.nsrc] > p.ny)
        return awc::fail(C, AWC_ERR_INVALID, "At least one source is not inside the model!");
    for (int32_t k = 0; k < sh.nrec; ++k)
      if (sh.posrecs[k] < 1 || sh.posrecs[k] > p.nx || sh.posrecs[k + sh.nrec] < 1 ||
          sh.posrecs[k + sh.nrec] > p.ny)
        return awc::fail(C, AWC_ERR_INVALID, "At least one receiver is not inside the model!");
  }
  return AWC_OK;
}

template <typename T>
void to_T(const double* src, std::vector<unsigned char>& out, int64_t n) {
  out.resize(std::max<int64_t>(n, 1) * sizeof(T));
  T* d = reinterpret_cast<T*>(out.data());
  for (int64_t c = 0; c < n; ++c) d[c] = (T)src[c];
}

// Tile heights 4, 8 and 16 run the TMA-fed kernel on tiles 64 nodes wide;
// 32 and 64 the register-strip kernel on tiles 32 nodes wide.
bool tma_tiles(int ty) { return ty <= 16; }
int64_t tile_w(int ty) { return tma_tiles(ty) ? 64 : 32; }
int64_t tiles_x(const awc_problem& p, int ty) { return (p.nx - 2) / tile_w(ty) + 1; }
int64_t tiles_of(const awc_problem& p, int ty) {
  return tiles_x(p, ty) * ((p.ny - 2 + ty - 1) / ty);
}

constexpr int kBatchStages = 6;  // TMA stages: tiles loaded up to 6 ahead (measured best of 3, 4, 6)

template <typename T, int RR>
constexpr int batch_smem() {
  return kBatchStages * awc::BatchTile<T, RR>::BYTES + 2 * kBatchStages * 8 + 16;
}

// Tensor maps of every shot for tile height ty (TMA kernel): dims (nx, ny),
// pitched rows; pcur box (64 + 2A) x (ty + 2), pold and fact boxes 64 x ty.
template <typename T>
int build_maps(awc_batch* B, int ty) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = awc::tensor_map_encoder();
  if (!enc) return awc::fail(B->ctx, AWC_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const CUtensorMapDataType dt =
      sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint32_t A = 16 / (cuuint32_t)sizeof(T);
  const cuuint32_t box_c[2] = {64 + 2 * A, (cuuint32_t)ty + 2}, box_i[2] = {64, (cuuint32_t)ty};
  const cuuint32_t es[2] = {1, 1};
  std::vector<awc::ShotMaps> maps(B->nshots);
  for (int32_t s = 0; s < B->nshots; ++s) {
    const awc_problem& p = B->models[B->shots[s].model];
    const cuuint64_t dims[2] = {(cuuint64_t)p.nx, (cuuint64_t)p.ny};
    const cuuint64_t strides[1] = {(cuuint64_t)(pitch32(p.nx) * sizeof(T))};
    auto make = [&](CUtensorMap* m, void* base, const cuuint32_t* box) {
      return enc(m, dt, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    const auto& M = B->sm[s];
    for (int b = 0; b < 3; ++b)
      if (!make(&maps[s].c[b], B->arena + M.buf[b], box_c) ||
          !make(&maps[s].o[b], B->arena + M.buf[b], box_i))
        return awc::fail(B->ctx, AWC_ERR_CUDA, "tensor map encoding failed");
    if (!make(&maps[s].f, B->arena + B->m_fact[B->shots[s].model], box_i))
      return awc::fail(B->ctx, AWC_ERR_CUDA, "tensor map encoding failed");
  }
  BATCH_TRY(B->ctx, cudaMemcpyAsync(B->arena + B->maps, maps.data(), maps.size() * sizeof(maps[0]),
                                    cudaMemcpyHostToDevice, B->ctx->stream));
  BATCH_TRY(B->ctx, cudaStreamSynchronize(B->ctx->stream));
  return AWC_OK;
}

// Opts the TMA kernels into their dynamic shared memory (once per process).
int init_batch_attrs(awc_ctx* C) {
#define AWC_BATTR(T, RR)                                                                   \
  BATCH_TRY(C, cudaFuncSetAttribute(awc::step2d_batch_tma<T, RR, kBatchStages>,             \
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                                    batch_smem<T, RR>()))
  AWC_BATTR(float, 1);
  AWC_BATTR(float, 2);
  AWC_BATTR(float, 4);
  AWC_BATTR(double, 1);
  AWC_BATTR(double, 2);
  AWC_BATTR(double, 4);
#undef AWC_BATTR
  return AWC_OK;
}

// Device descriptors and per-tile source/receiver lists for tile height ty.
template <typename T>
int build_layout(awc_batch* B) {
  awc_ctx* C = B->ctx;
  const int ty = B->ty;
  std::vector<awc::ShotDesc<T>> descs(B->nshots);
  std::vector<int32_t> tile_start(B->nshots + 1, 0);
  for (int32_t s = 0; s < B->nshots; ++s) {
    const awc_problem& p = B->models[B->shots[s].model];
    const int32_t m = B->shots[s].model;
    const auto& M = B->sm[s];
    awc::ShotDesc<T>& D = descs[s];
    for (int b = 0; b < 3; ++b) D.buf[b] = (T*)(B->arena + M.buf[b]);
    D.fact = (const T*)(B->arena + B->m_fact[m]);
    D.px = pitch32(p.nx);
    D.nx = (int32_t)p.nx;
    D.ny = (int32_t)p.ny;
    D.halo = p.halo;
    D.gx = (int32_t)tiles_x(p, ty);
    const double d[2] = {p.dx, p.dy};
    for (int a = 0; a < 2; ++a) {
      D.inv_d[a] = (T)(1.0 / d[a]);
      D.inv_d2[a] = (T)(1.0 / (d[a] * d[a]));
    }
    const int64_t h = p.halo;
    const T* cf = (const T*)(B->arena + M.coef);
    for (int a = 0; a < 2; ++a) {
      const T* blk = cf + a * (8 * h + 4);
      for (int sd = 0; sd < 2; ++sd) {
        for (int par = 0; par < 2; ++par) D.psi[a][sd][par] = (T*)(B->arena + M.psi[a][sd][par]);
        awc::BandSide<T>& Bs = D.band[a][sd];
        Bs.psi_old = nullptr;
        Bs.psi_new = nullptr;
        Bs.xi = (T*)(B->arena + M.xi[a][sd]);
        Bs.a = blk + sd * h;
        Bs.bK = blk + 2 * h + sd * h;
        Bs.ah = blk + 4 * h + sd * (h + 1);
        Bs.bKh = blk + 4 * h + 2 * (h + 1) + sd * (h + 1);
        D.active[a][sd] = B->active[(s * 2 + a) * 2 + sd];
      }
      const int64_t n = a == 0 ? p.nx : p.ny;
      D.first_r[a] = (int32_t)std::max<int64_t>(n - h - 1, h + 1);
    }
    // sources and receivers: rim nodes to the shot's rim list (tile 0),
    // interior nodes to their tile, (tile, local) order
    const int64_t px = pitch32(p.nx), gx = tiles_x(p, ty), W = tile_w(ty);
    const int64_t nt_tiles = tiles_of(p, ty);
    std::vector<awc::IoRim> rim;
    std::vector<std::pair<int64_t, int4>> ent;
    for (const awc::IoRim& e : B->io_nodes[s]) {
      const int64_t i = e.node % px, j = e.node / px;
      if (i < 1 || i > p.nx - 2 || j < 1 || j > p.ny - 2) {
        rim.push_back(e);
        continue;
      }
      const int64_t tile = i / W + gx * ((j - 1) / ty);
      const int local = (int)(i % W + W * ((j - 1) % ty));
      ent.push_back({tile * 4096 + local, make_int4(local, 0, e.sgrp, e.rgrp)});
    }
    std::sort(ent.begin(), ent.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<int32_t> off(nt_tiles + 1, 0);
    std::vector<int4> flat(ent.size());
    for (size_t n = 0; n < ent.size(); ++n) {
      off[ent[n].first / 4096 + 1]++;
      flat[n] = ent[n].second;
    }
    for (int64_t b = 0; b < nt_tiles; ++b) off[b + 1] += off[b];
    cudaStream_t st = C->stream;
    BATCH_TRY(C, cudaMemcpyAsync(B->arena + M.blk_off, off.data(), off.size() * 4,
                                 cudaMemcpyHostToDevice, st));
    if (!flat.empty())
      BATCH_TRY(C, cudaMemcpyAsync(B->arena + M.ent, flat.data(), flat.size() * sizeof(int4),
                                   cudaMemcpyHostToDevice, st));
    if (!rim.empty())
      BATCH_TRY(C, cudaMemcpyAsync(B->arena + M.rim, rim.data(), rim.size() * sizeof(awc::IoRim),
                                   cudaMemcpyHostToDevice, st));
    BATCH_TRY(C, cudaStreamSynchronize(st));  // host vectors go out of scope
    awc::Io<T>& io = D.io;
    io.blk_off = (const int32_t*)(B->arena + M.blk_off);
    io.ent = (const int4*)(B->arena + M.ent);
    io.rim = (const awc::IoRim*)(B->arena + M.rim);
    io.nrim = (int32_t)rim.size();
    io.src_off = (const int32_t*)(B->arena + M.src_off);
    io.src_ids = (const int32_t*)(B->arena + M.src_ids);
    io.rec_off = (const int32_t*)(B->arena + M.rec_off);
    io.rec_ids = (const int32_t*)(B->arena + M.rec_ids);
    io.stf = (const T*)(B->arena + M.stf);
    io.nsrc = B->shot_nsrc[s];
    io.nrec = B->shot_nrec[s];
    io.traces = (T*)(B->arena + M.traces);
    tile_start[s + 1] = (int32_t)(tile_start[s] + nt_tiles);
  }
  BATCH_TRY(C, cudaMemcpyAsync(B->arena + B->descs, descs.data(), descs.size() * sizeof(descs[0]),
                               cudaMemcpyHostToDevice, C->stream));
  BATCH_TRY(C, cudaMemcpyAsync(B->arena + B->tile_start, tile_start.data(), tile_start.size() * 4,
                               cudaMemcpyHostToDevice, C->stream));
  BATCH_TRY(C, cudaStreamSynchronize(C->stream));
  if (tma_tiles(ty)) {
    const int rc = build_maps<T>(B, ty);
    if (rc) return rc;
  }
  B->ntiles = tile_start[B->nshots];
  B->io_ty = ty;
  return AWC_OK;
}

template <typename T>
using BatchKernel = void (*)(const awc::ShotDesc<T>*, const int32_t*, int32_t, int32_t, int32_t);

// Tile height 32 or 64 -> register-strip kernel: 4 warps per block, each
// streaming tile_y / 4 rows.
template <typename T>
BatchKernel<T> batch_kernel(int tile_y) {
  switch (tile_y) {
    case 32: return awc::step2d_batch<T, 4, 8>;
    case 64: return awc::step2d_batch<T, 4, 16>;
    default: return nullptr;
  }
}

template <typename T>
using BatchTmaKernel = void (*)(const awc::ShotDesc<T>*, const awc::ShotMaps*, const int32_t*,
                                int32_t, int32_t, int32_t, int32_t*);

template <typename T>
int launch_batch_step(awc_batch* B, int64_t it, cudaStream_t st) {
  const auto* D = (const awc::ShotDesc<T>*)(B->arena + B->descs);
  const auto* ts = (const int32_t*)(B->arena + B->tile_start);
  int& occ = B->occ[B->ty];
  if (tma_tiles(B->ty)) {
    // tile_y rows = BATCH_CW consumer warps x RR rows each, plus a producer warp
    BatchTmaKernel<T> k = nullptr;
    int smem = 0;
    const int warps = awc::BATCH_CW + 1;
    switch (B->ty) {
      case 4: k = awc::step2d_batch_tma<T, 1, kBatchStages>; smem = batch_smem<T, 1>(); break;
      case 8: k = awc::step2d_batch_tma<T, 2, kBatchStages>; smem = batch_smem<T, 2>(); break;
      default: k = awc::step2d_batch_tma<T, 4, kBatchStages>; smem = batch_smem<T, 4>(); break;
    }
    if (occ == 0) {
      BATCH_TRY(B->ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 32 * warps, smem));
      occ = std::max(occ, 1);
    }
    const int per_sm = std::min<int>(B->bps, occ);
    const int grid = std::max(1, std::min(B->ntiles, B->ctx->num_sms * per_sm));
    k<<<grid, dim3(32, warps), smem, st>>>(D, (const awc::ShotMaps*)(B->arena + B->maps), ts,
                                          B->nshots, B->ntiles, (int)it,
                                          (int32_t*)(B->arena + B->err));
    BATCH_TRY(B->ctx, cudaGetLastError());
    return AWC_OK;
  }
  const BatchKernel<T> k = batch_kernel<T>(B->ty);
  if (!k) return awc::fail(B->ctx, AWC_ERR_INVALID, "unsupported tile height");
  if (occ == 0) {
    BATCH_TRY(B->ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 128, 0));
    occ = std::max(occ, 1);
  }
  // a persistent grid: never more blocks than can be resident at once
  const int per_sm = std::min<int>(B->bps, occ);
  const int grid = std::max(1, std::min(B->ntiles, B->ctx->num_sms * per_sm));
  k<<<grid, dim3(32, 4), 0, st>>>(D, ts, B->nshots, B->ntiles, (int)it);
  BATCH_TRY(B->ctx, cudaGetLastError());
  return AWC_OK;
}

int launch_batch_range(awc_batch* B, int64_t start, int64_t n, cudaStream_t st) {
  for (int64_t it = start; it < start + n; ++it) {
    const int rc = B->prec == AWC_F64 ? launch_batch_step<double>(B, it, st)
                                      : launch_batch_step<float>(B, it, st);
    if (rc) return rc;
  }
  return AWC_OK;
}

int ensure_layout(awc_batch* B) {
  if (B->io_ty == B->ty) return AWC_OK;
  return B->prec == AWC_F64 ? build_layout<double>(B) : build_layout<float>(B);
}

}  // namespace

extern "C" {

int awc_batch_create(awc_ctx* C, int32_t nmodels, const awc_problem* models,
                     const double* const* vel, int32_t nshots, const awc_shot* shots,
                     awc_batch** out) {
  if (!C || !out) return awc::fail(nullptr, AWC_ERR_INVALID, "ctx/out is NULL");
  *out = nullptr;
  int rc = check_batch(C, nmodels, models, vel, nshots, shots);
  if (rc) return rc;
  BATCH_TRY(C, cudaSetDevice(C->device));
  awc_batch* B = new awc_batch();
  B->ctx = C;
  B->nmodels = nmodels;
  B->nshots = nshots;
  B->models.assign(models, models + nmodels);
  B->shots.assign(shots, shots + nshots);
  for (awc_shot& sh : B->shots)  // the host arrays are read during create only
    sh.coeffs = nullptr, sh.possrcs = nullptr, sh.dt2srctf = nullptr, sh.posrecs = nullptr;
  B->prec = models[0].precision;
  B->esz = B->prec == AWC_F64 ? 8 : 4;
  B->nt = models[0].nt;
  const size_t esz = B->esz;
  const int64_t nt = B->nt;
  // ---- arena layout ---------------------------------------------------------
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += up256(std::max<size_t>(bytes, 16));
    return at;
  };
  int64_t staging = 0;
  B->m_fact.resize(nmodels);
  for (int32_t m = 0; m < nmodels; ++m) {
    const awc_problem& p = models[m];
    B->m_fact[m] = take(pitch32(p.nx) * p.ny * esz);
    staging = std::max<int64_t>(staging, p.nx * p.ny);
  }
  B->sm.resize(nshots);
  B->shot_nsrc.resize(nshots);
  B->shot_nrec.resize(nshots);
  for (int32_t s = 0; s < nshots; ++s) {
    const awc_problem& p = models[shots[s].model];
    auto& M = B->sm[s];
    const int64_t px = pitch32(p.nx), h = p.halo, ns = shots[s].nsrc, nr = shots[s].nrec;
    for (int b = 0; b < 3; ++b) M.buf[b] = take(px * p.ny * esz);
    const int64_t cs[2] = {p.ny, px};  // band cross-sections: ψ_x (h+1, ny), ψ_y (px, h+1)
    for (int a = 0; a < 2; ++a)
      for (int sd = 0; sd < 2; ++sd) {
        for (int par = 0; par < 2; ++par) M.psi[a][sd][par] = take((h + 1) * cs[a] * esz);
        M.xi[a][sd] = take(h * cs[a] * esz);
      }
    M.stf = take(nt * ns * esz);
    M.traces = take(nt * nr * esz);
    M.src_off = take((ns + 1) * 4);
    M.src_ids = take(ns * 4);
    M.rec_off = take((nr + 1) * 4);
    M.rec_ids = take(nr * 4);
    M.rim = take((ns + nr) * sizeof(awc::IoRim));
    M.max_tiles = 0;  // per-tile list bounds for the most numerous tiles of any height
    for (int t : {4, 8, 16, 32, 64}) M.max_tiles = std::max(M.max_tiles, tiles_of(p, t));
    M.blk_off = take((M.max_tiles + 1) * 4);
    M.ent = take((ns + nr) * sizeof(int4));
    M.coef = take(2 * (8 * h + 4) * esz);
    B->shot_nsrc[s] = (int32_t)ns;
    B->shot_nrec[s] = (int32_t)nr;
    staging = std::max<int64_t>(staging, nt * nr);
  }
  B->descs = take(nshots * std::max(sizeof(awc::ShotDesc<float>), sizeof(awc::ShotDesc<double>)));
  B->maps = take(nshots * sizeof(awc::ShotMaps));
  B->err = take(16);
  B->tile_start = take((nshots + 1) * 4);
  const size_t o_staging = take(staging * 8);
  B->staging_len = staging;
  B->arena_bytes = off;
  cudaError_t e = cudaMalloc((void**)&B->arena, off);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete B;
    return awc::fail(C, e == cudaErrorMemoryAllocation ? AWC_ERR_OOM : AWC_ERR_CUDA,
                     "batch arena allocation failed");
  }
  B->staging = (double*)(B->arena + o_staging);
  cudaStream_t st = C->stream;
  if (cudaMemsetAsync(B->arena + B->err, 0, 4, st) != cudaSuccess || init_batch_attrs(C)) {
    delete B;
    return awc::fail(C, AWC_ERR_CUDA, "batch setup failed");
  }
  std::vector<unsigned char> tmp;
  auto up = [&](size_t at, const void* src, size_t bytes) {
    return cudaMemcpyAsync(B->arena + at, src, bytes, cudaMemcpyHostToDevice, st);
  };
  // ---- models: fact = dt^2 vel^2, in FP64 on the device, pitched ---------
  for (int32_t m = 0; m < nmodels && !rc; ++m) {
    const awc_problem& p = models[m];
    const int64_t N = p.nx * p.ny;
    if (up(o_staging, vel[m], N * 8) != cudaSuccess) rc = AWC_ERR_CUDA;
    const int blocks = (int)std::min<int64_t>((N + 255) / 256, (int64_t)C->num_sms * 16);
    if (B->prec == AWC_F64)
      awc::make_fact<double><<<blocks, 256, 0, st>>>(B->staging, (double*)(B->arena + B->m_fact[m]),
                                                     p.dt * p.dt, N, p.nx, pitch32(p.nx));
    else
      awc::make_fact<float><<<blocks, 256, 0, st>>>(B->staging, (float*)(B->arena + B->m_fact[m]),
                                                    p.dt * p.dt, N, p.nx, pitch32(p.nx));
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = AWC_ERR_CUDA;  // staging is reused
  }
  // ---- shots: source functions, source/receiver groups --------------------
  B->io_nodes.resize(nshots);
  B->active.assign(nshots * 4, 0);
  for (int32_t s = 0; s < nshots && !rc; ++s) {
    const awc_shot& sh = shots[s];
    const awc_problem& p = models[sh.model];
    const auto& M = B->sm[s];
    const int64_t px = pitch32(p.nx), ns = sh.nsrc, nr = sh.nrec, h = p.halo;
    // the shot's CPML coefficients (they depend on its f0) and live sides
    const int64_t clen = 2 * (8 * h + 4);
    if (B->prec == AWC_F64) to_T<double>(sh.coeffs, tmp, clen); else to_T<float>(sh.coeffs, tmp, clen);
    if (up(M.coef, tmp.data(), clen * esz) != cudaSuccess) rc = AWC_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = AWC_ERR_CUDA;  // tmp is reused
    for (int a = 0; a < 2; ++a) {
      const double* blk = sh.coeffs + a * (8 * h + 4);
      for (int sd = 0; sd < 2; ++sd) {
        bool trivial = true;  // a free-top side: ψ = ξ = 0 for ever
        for (int64_t k = 0; k < h; ++k)
          trivial = trivial && blk[sd * h + k] == 0.0 && blk[2 * h + sd * h + k] == 1.0;
        for (int64_t k = 0; k < h + 1; ++k)
          trivial = trivial && blk[4 * h + sd * (h + 1) + k] == 0.0 &&
                    blk[4 * h + 2 * (h + 1) + sd * (h + 1) + k] == 1.0;
        B->active[(s * 2 + a) * 2 + sd] = (h > 0 && !trivial) ? 1 : 0;
      }
    }
    std::vector<double> rows(std::max<int64_t>(nt * ns, 1), 0.0);
    for (int64_t k = 0; k < ns; ++k)
      for (int64_t t = 0; t < nt; ++t) rows[t * ns + k] = sh.dt2srctf[t + nt * k];
    if (B->prec == AWC_F64) to_T<double>(rows.data(), tmp, nt * ns); else to_T<float>(rows.data(), tmp, nt * ns);
    if (nt * ns > 0 && up(M.stf, tmp.data(), nt * ns * esz) != cudaSuccess) rc = AWC_ERR_CUDA;
    std::unordered_map<int64_t, int32_t> where;
    std::vector<std::vector<int32_t>> sg, rg;
    auto& nodes = B->io_nodes[s];
    auto slot = [&](int64_t nd) -> awc::IoRim& {
      auto f = where.find(nd);
      if (f == where.end()) {
        where.emplace(nd, (int32_t)nodes.size());
        nodes.push_back(awc::IoRim{nd, -1, -1});
        return nodes.back();
      }
      return nodes[f->second];
    };
    for (int64_t k = 0; k < ns; ++k) {
      awc::IoRim& e2 = slot((sh.possrcs[k] - 1) + px * (sh.possrcs[k + ns] - 1));
      if (e2.sgrp < 0) {
        e2.sgrp = (int32_t)sg.size();
        sg.emplace_back();
      }
      sg[e2.sgrp].push_back((int32_t)k);
    }
    for (int64_t k = 0; k < nr; ++k) {
      awc::IoRim& e2 = slot((sh.posrecs[k] - 1) + px * (sh.posrecs[k + nr] - 1));
      if (e2.rgrp < 0) {
        e2.rgrp = (int32_t)rg.size();
        rg.emplace_back();
      }
      rg[e2.rgrp].push_back((int32_t)k);
    }
    auto csr = [](const std::vector<std::vector<int32_t>>& g, std::vector<int32_t>& o,
                  std::vector<int32_t>& ids) {
      o.assign(1, 0);
      ids.clear();
      for (auto& v : g) {
        ids.insert(ids.end(), v.begin(), v.end());
        o.push_back((int32_t)ids.size());
      }
    };
    std::vector<int32_t> soff, sids, roff, rids;
    csr(sg, soff, sids);
    csr(rg, roff, rids);
    if (up(M.src_off, soff.data(), soff.size() * 4) != cudaSuccess ||
        up(M.rec_off, roff.data(), roff.size() * 4) != cudaSuccess ||
        (!sids.empty() && up(M.src_ids, sids.data(), sids.size() * 4) != cudaSuccess) ||
        (!rids.empty() && up(M.rec_ids, rids.data(), rids.size() * 4) != cudaSuccess))
      rc = AWC_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = AWC_ERR_CUDA;
  }
  if (rc || (rc = ensure_layout(B)) || (rc = awc_batch_reset(B))) {
    if (rc == AWC_ERR_CUDA) awc::fail(C, rc, "batch upload failed");
    delete B;
    return rc;
  }
  *out = B;
  return AWC_OK;
}

void awc_batch_destroy(awc_batch* B) {
  if (!B) return;
  cudaSetDevice(B->ctx->device);
  cudaStreamSynchronize(B->ctx->stream);
  delete B;
}

int awc_batch_reset(awc_batch* B) {
  if (!B) return awc::fail(nullptr, AWC_ERR_INVALID, "batch is NULL");
  awc_ctx* C = B->ctx;
  BATCH_TRY(C, cudaSetDevice(C->device));
  for (int32_t s = 0; s < B->nshots; ++s) {
    const auto& M = B->sm[s];
    // fields, ψ, ξ, source functions' neighbours and traces are contiguous
    // from buf[0] up to stf, then traces after it
    BATCH_TRY(C, cudaMemsetAsync(B->arena + M.buf[0], 0, M.stf - M.buf[0], C->stream));
    BATCH_TRY(C, cudaMemsetAsync(B->arena + M.traces, 0, M.src_off - M.traces, C->stream));
  }
  B->step = 0;
  return AWC_OK;
}

int awc_batch_set_launch(awc_batch* B, int32_t tile_y, int32_t blocks_per_sm) {
  if (!B) return awc::fail(nullptr, AWC_ERR_INVALID, "batch is NULL");
  if ((tile_y != 4 && tile_y != 8 && tile_y != 16 && tile_y != 32 && tile_y != 64) ||
      blocks_per_sm < 1 || blocks_per_sm > 32)
    return awc::fail(B->ctx, AWC_ERR_INVALID,
                     "tile_y must be 4, 8, 16, 32 or 64; blocks_per_sm in [1, 32]");
  B->ty = tile_y;
  B->bps = blocks_per_sm;
  return AWC_OK;
}

int awc_batch_get_launch(const awc_batch* B, int32_t* tile_y, int32_t* blocks_per_sm) {
  if (!B || !tile_y || !blocks_per_sm) return awc::fail(nullptr, AWC_ERR_INVALID, "NULL argument");
  *tile_y = B->ty;
  *blocks_per_sm = B->bps;
  return AWC_OK;
}

int awc_batch_run(awc_batch* B, int64_t nsteps, int32_t use_graph, float* ms) {
  if (!B) return awc::fail(nullptr, AWC_ERR_INVALID, "batch is NULL");
  awc_ctx* C = B->ctx;
  if (nsteps < 0) return awc::fail(C, AWC_ERR_INVALID, "nsteps < 0");
  BATCH_TRY(C, cudaSetDevice(C->device));
  const int64_t n = std::min<int64_t>(nsteps, B->nt - B->step);
  if (ms) *ms = 0.f;
  if (n <= 0) return AWC_OK;
  int rc;
  if ((rc = ensure_layout(B))) return rc;
  cudaGraphExec_t ex = nullptr;
  if (use_graph) {
    const uint64_t key = (uint64_t)B->ty | ((uint64_t)B->bps << 8);
    if (key != B->graph_key) {
      for (auto& kv : B->graphs) cudaGraphExecDestroy(kv.second);
      B->graphs.clear();
      B->graph_key = key;
    }
    auto f = B->graphs.find({B->step, n});
    if (f != B->graphs.end()) {
      ex = f->second;
    } else {
      cudaGraph_t g = nullptr;
      BATCH_TRY(C, cudaStreamBeginCapture(C->stream, cudaStreamCaptureModeThreadLocal));
      rc = launch_batch_range(B, B->step, n, C->stream);
      const cudaError_t e = cudaStreamEndCapture(C->stream, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      BATCH_TRY(C, e);
      const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      BATCH_TRY(C, e2);
      B->graphs[{B->step, n}] = ex;
    }
  }
  BATCH_TRY(C, cudaEventRecord(C->ev0, C->stream));
  if (use_graph) {
    BATCH_TRY(C, cudaGraphLaunch(ex, C->stream));
  } else if ((rc = launch_batch_range(B, B->step, n, C->stream))) {
    return rc;
  }
  BATCH_TRY(C, cudaEventRecord(C->ev1, C->stream));
  BATCH_TRY(C, cudaEventSynchronize(C->ev1));
  if (ms) BATCH_TRY(C, cudaEventElapsedTime(ms, C->ev0, C->ev1));
  B->step += n;
  // a bounded wait of the TMA kernel that ran out
  int32_t flag = 0;
  BATCH_TRY(C, cudaMemcpy(&flag, B->arena + B->err, 4, cudaMemcpyDeviceToHost));
  if (flag) {
    BATCH_TRY(C, cudaMemset(B->arena + B->err, 0, 4));
    return awc::fail(C, AWC_ERR_TIMEOUT, "a bounded wait on a pipeline barrier ran out");
  }
  return AWC_OK;
}

int64_t awc_batch_step(const awc_batch* B) { return B ? B->step : -1; }

int awc_batch_traces(awc_batch* B, int32_t shot, double* traces) {
  if (!B || !traces || shot < 0 || shot >= B->nshots)
    return awc::fail(B ? B->ctx : nullptr, AWC_ERR_INVALID, "bad batch/shot/traces");
  awc_ctx* C = B->ctx;
  const int64_t nt = B->nt, nr = B->shot_nrec[shot];
  if (nt * nr == 0) return AWC_OK;
  BATCH_TRY(C, cudaSetDevice(C->device));
  dim3 grid((unsigned)((nt + 31) / 32), (unsigned)((nr + 31) / 32));
  const unsigned char* src = B->arena + B->sm[shot].traces;
  if (B->prec == AWC_F64)
    awc::traces_out<double><<<grid, dim3(32, 8), 0, C->stream>>>((const double*)src, B->staging, nt, nr);
  else
    awc::traces_out<float><<<grid, dim3(32, 8), 0, C->stream>>>((const float*)src, B->staging, nt, nr);
  BATCH_TRY(C, cudaGetLastError());
  BATCH_TRY(C, cudaMemcpyAsync(traces, B->staging, nt * nr * 8, cudaMemcpyDeviceToHost, C->stream));
  BATCH_TRY(C, cudaStreamSynchronize(C->stream));
  return AWC_OK;
}

int awc_batch_field(awc_batch* B, int32_t shot, double* out) {
  if (!B || !out || shot < 0 || shot >= B->nshots)
    return awc::fail(B ? B->ctx : nullptr, AWC_ERR_INVALID, "bad batch/shot/out");
  awc_ctx* C = B->ctx;
  const awc_problem& p = B->models[B->shots[shot].model];
  const int64_t N = p.nx * p.ny;
  BATCH_TRY(C, cudaSetDevice(C->device));
  const unsigned char* cur = B->arena + B->sm[shot].buf[(B->step + 1) % 3];
  const int blocks = (int)std::min<int64_t>((N + 255) / 256, (int64_t)C->num_sms * 16);
  if (B->prec == AWC_F64)
    awc::unpitch<double><<<blocks, 256, 0, C->stream>>>((const double*)cur, B->staging, N, p.nx, pitch32(p.nx));
  else
    awc::unpitch<float><<<blocks, 256, 0, C->stream>>>((const float*)cur, B->staging, N, p.nx, pitch32(p.nx));
  BATCH_TRY(C, cudaGetLastError());
  BATCH_TRY(C, cudaMemcpyAsync(out, B->staging, N * 8, cudaMemcpyDeviceToHost, C->stream));
  BATCH_TRY(C, cudaStreamSynchronize(C->stream));
  return AWC_OK;
}

int awc_batch_autotune(awc_batch* B, int64_t steps, float* best_ms_per_step) {
  if (!B) return awc::fail(nullptr, AWC_ERR_INVALID, "batch is NULL");
  if (steps < 1) return awc::fail(B->ctx, AWC_ERR_INVALID, "steps must be >= 1");
  const int64_t n = std::min<int64_t>(steps, B->nt);
  float best = 1e30f;
  int32_t wty = B->ty, wbps = B->bps;
  int rc;
  for (int32_t ty : {4, 8, 16, 32, 64})
    for (int32_t bps : {4, 8, 16}) {
      B->ty = ty;
      B->bps = bps;
      float per = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        float ms = 0.f;
        if ((rc = awc_batch_reset(B)) || (rc = awc_batch_run(B, n, 0, &ms))) return rc;
        per = std::min(per, ms / (float)n);
      }
      if (per < best) {
        best = per;
        wty = ty;
        wbps = bps;
      }
    }
  B->ty = wty;
  B->bps = wbps;
  if (best_ms_per_step) *best_ms_per_step = best;
  return awc_batch_reset(B);
}

int awc_forward_batch(awc_ctx* C, int32_t nmodels, const awc_problem* models,
                      const double* const* vel, int32_t nshots, const awc_shot* shots,
                      double* const* traces) {
  if (!traces) return awc::fail(C, AWC_ERR_INVALID, "traces is NULL");
  awc_batch* B = nullptr;
  int rc = awc_batch_create(C, nmodels, models, vel, nshots, shots, &B);
  if (rc) return rc;
  if (models[0].nt >= 100) rc = awc_batch_autotune(B, 10, nullptr);
  if (!rc) rc = awc_batch_run(B, B->nt, 1, &C->last_run_ms);
  for (int32_t s = 0; s < nshots && !rc; ++s)
    if (shots[s].nrec > 0) {
      if (!traces[s]) rc = awc::fail(C, AWC_ERR_INVALID, "a shot's traces buffer is NULL");
      else rc = awc_batch_traces(B, s, traces[s]);
    }
  awc_batch_destroy(B);
  return rc;
}

}  // extern "C"
