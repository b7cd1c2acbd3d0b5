// awc_static.cu — awc_forward2d_f32_static: a 2D FP32 forward solve that
// performs no device memory allocation.
//
// Some callers cannot let a library call cudaMalloc. A solver loop that must
// not stall the device (cudaMalloc and cudaFree synchronise it) is one. A
// host framework whose own allocator owns every device byte is another: Julia
// CUDA.jl's memory pool or a caching allocator can be starved or fragmented
// by allocations it does not see. For them this entry point keeps every
// device buffer of the solve in one file-scope __device__ array of fixed size
// (kScratchBytes below). The array exists on every GPU that loads this
// library, from module load until process exit. The caller passes host
// inputs and outputs exactly as for awc_forward.
//
// The solve is the same as awc_forward's FP32 2D path: the same step2d
// kernel over a dense (unpitched) layout, with sources and receivers applied
// by a one-block kernel after each step.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/awcpml.h"
#include "awc_kernels.cuh"

namespace awc {
void record_error(const char* msg);  // awc_api.cu
}

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;  // 32 MiB

// The scratch array. In host code this name is only a stand-in for the
// device symbol: its device address comes from cudaGetSymbolAddress.
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

int fail(int code, const char* msg) {
  awc::record_error(msg);  // what awc_last_error(NULL) returns on this thread
  return code;
}

// Device address of g_scratch on the current device. It is looked up on
// every call rather than cached: a cached address would dangle after a device
// reset (cudaDeviceReset, CUDA.jl's device_reset!), which reloads the module.
// The first lookup on a device loads the module there.
int scratch_address(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorNoDevice || e == cudaErrorInvalidDevice ? AWC_ERR_NODEVICE
                                                                       : AWC_ERR_CUDA,
                cudaGetErrorString(e));
  }
  *out = static_cast<unsigned char*>(p);
  return AWC_OK;
}

size_t up256(size_t b) { return (b + 255) / 256 * 256; }

// Sources then receivers of step `it`, in one block (reference
// inject_sources!/record_receivers!). Sources are grouped by node on the
// host; one thread owns a group and adds its sources in source order, so
// several sources on one node are summed in the order awc_forward sums them.
// Then each receiver samples the new field.
__global__ void static_io(float* pnew, const double* stf, const int64_t* grp_node,
                          const int32_t* grp_off, const int32_t* grp_src, int ngrp,
                          const int64_t* rec_node, int nrec, int64_t nt, int64_t it,
                          double* traces) {
  for (int g = threadIdx.x; g < ngrp; g += blockDim.x) {
    float v = pnew[grp_node[g]];
    for (int e = grp_off[g]; e < grp_off[g + 1]; ++e) v += (float)stf[it + nt * grp_src[e]];
    pnew[grp_node[g]] = v;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < nrec; r += blockDim.x)
    traces[it + nt * r] = (double)pnew[rec_node[r]];
}

// a * b, or false when the product of two non-negative sizes overflows.
bool mul_ok(size_t a, size_t b, size_t* out) {
  if (a != 0 && b > SIZE_MAX / a) return false;
  *out = a * b;
  return true;
}

__global__ void static_narrow(const double* src, float* dst, int64_t n) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    dst[c] = (float)src[c];
}

#define STATIC_TRY(call)                                             \
  do {                                                               \
    const cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) {                                         \
      cudaGetLastError();                                            \
      return fail(AWC_ERR_CUDA, cudaGetErrorString(e_));             \
    }                                                                \
  } while (0)

}  // namespace

extern "C" int awc_forward2d_f32_static(const awc_problem* p, const double* vel,
                                        const double* coeffs, const int64_t* possrcs,
                                        const double* dt2srctf, const int64_t* posrecs,
                                        double* traces, double* pfinal) {
  // ---- arguments (the same checks as awc_forward, for this variant) ------
  if (!p) return fail(AWC_ERR_INVALID, "problem is NULL");
  if (p->ndim != 2 || p->nz != 1) return fail(AWC_ERR_INVALID, "this entry point solves 2D problems only");
  if (p->precision != AWC_F32) return fail(AWC_ERR_INVALID, "this entry point computes in FP32 only");
  if (p->nx < 3 || p->ny < 3 || p->nx > (1 << 20) || p->ny > (1 << 20))
    return fail(AWC_ERR_INVALID, "grid size must be in [3, 2^20] per axis");
  if (p->halo < 0 || p->halo > p->nx - 2 || p->halo > p->ny - 2)
    return fail(AWC_ERR_INVALID, "halo out of range for the grid");
  if (!(p->dx > 0.0) || !(p->dy > 0.0) || !(p->dt > 0.0) || !std::isfinite(p->dx) ||
      !std::isfinite(p->dy) || !std::isfinite(p->dt))
    return fail(AWC_ERR_INVALID, "grid spacing and dt must be positive and finite");
  // the same limits as awc_forward: nt <= 2^31, so step indices fit in int32
  // and every size below fits in size_t without overflow
  if (p->nt < 0 || p->nt > ((int64_t)1 << 31))
    return fail(AWC_ERR_INVALID, "nt out of range");
  if (p->nsrc < 0 || p->nrec < 0 || p->nsrc > (1 << 20) || p->nrec > (1 << 20))
    return fail(AWC_ERR_INVALID, "nsrc/nrec out of range");
  if (!vel || !coeffs || (p->nsrc > 0 && (!possrcs || (p->nt > 0 && !dt2srctf))) ||
      (p->nrec > 0 && !posrecs) || (p->nt * p->nrec > 0 && !traces))
    return fail(AWC_ERR_INVALID, "a required array is NULL");
  const int64_t nx = p->nx, ny = p->ny, h = p->halo, nt = p->nt, ns = p->nsrc, nr = p->nrec;
  for (int64_t s = 0; s < ns; ++s)
    if (possrcs[s] < 1 || possrcs[s] > nx || possrcs[s + ns] < 1 || possrcs[s + ns] > ny)
      return fail(AWC_ERR_INVALID, "At least one source is not inside the model!");
  for (int64_t r = 0; r < nr; ++r)
    if (posrecs[r] < 1 || posrecs[r] > nx || posrecs[r + nr] < 1 || posrecs[r + nr] > ny)
      return fail(AWC_ERR_INVALID, "At least one receiver is not inside the model!");

  // sources grouped by node, in source order within a group
  std::vector<int32_t> order((size_t)ns);
  for (int64_t s = 0; s < ns; ++s) order[s] = (int32_t)s;
  auto src_node = [&](int64_t s) { return (possrcs[s] - 1) + nx * (possrcs[s + ns] - 1); };
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t a, int32_t b) { return src_node(a) < src_node(b); });
  std::vector<int64_t> grp_node, rec_node((size_t)nr);
  std::vector<int32_t> grp_off;
  for (int64_t e = 0; e < ns; ++e) {
    if (e == 0 || src_node(order[e]) != src_node(order[e - 1])) {
      grp_node.push_back(src_node(order[e]));
      grp_off.push_back((int32_t)e);
    }
  }
  grp_off.push_back((int32_t)ns);
  for (int64_t r = 0; r < nr; ++r) rec_node[r] = (posrecs[r] - 1) + nx * (posrecs[r + nr] - 1);
  const int64_t ngrp = (int64_t)grp_node.size();

  // ---- scratch layout (every region 256-byte aligned) --------------------
  // With the limits above every product fits in size_t; the sizes are still
  // formed with checked multiplies so that no wrapped size can pass the
  // capacity test.
  const int64_t N = nx * ny;
  const int gx = (int)((nx - 2) / 32 + 1), gy = (int)((ny - 2 + 7) / 8);
  const int64_t clen = 2 * (8 * h + 4);
  size_t off = 0;
  bool fits = true;
  auto take = [&](size_t count, size_t elem) {
    size_t bytes = 0;
    const size_t at = off;
    if (!mul_ok(count, elem, &bytes) || bytes > kScratchBytes) {
      fits = false;
      return at;
    }
    off += up256(bytes);
    return at;
  };
  size_t nt_ns = 0, nt_nr = 0;
  fits = mul_ok((size_t)nt, (size_t)ns, &nt_ns) && mul_ok((size_t)nt, (size_t)nr, &nt_nr);
  const size_t o_buf = take(3 * (size_t)N, sizeof(float));
  const size_t o_fact = take((size_t)N, sizeof(float));
  const size_t o_vel = take((size_t)N, sizeof(double));  // vel in, then pfinal out
  const size_t o_psx = take(2 * 2 * (size_t)(h + 1) * ny, sizeof(float));
  const size_t o_xix = take(2 * (size_t)h * ny, sizeof(float));
  const size_t o_psy = take(2 * 2 * (size_t)(h + 1) * nx, sizeof(float));
  const size_t o_xiy = take(2 * (size_t)h * nx, sizeof(float));
  const size_t o_cd = take((size_t)clen, sizeof(double));
  const size_t o_cf = take((size_t)clen, sizeof(float));
  const size_t o_stf = take(nt_ns, sizeof(double));
  const size_t o_gn = take((size_t)ngrp, sizeof(int64_t));
  const size_t o_go = take((size_t)ngrp + 1, sizeof(int32_t));
  const size_t o_gs = take((size_t)ns, sizeof(int32_t));
  const size_t o_pr = take((size_t)nr, sizeof(int64_t));
  const size_t o_tr = take(nt_nr, sizeof(double));
  const size_t o_blk = take((size_t)gx * gy + 1, sizeof(int32_t));
  if (!fits || off > kScratchBytes) {
    char msg[200];
    if (fits)
      std::snprintf(msg, sizeof msg,
                    "problem needs %zu bytes of device scratch; this entry point has %zu "
                    "(use awc_forward for larger problems)",
                    off, kScratchBytes);
    else
      std::snprintf(msg, sizeof msg,
                    "problem needs more than the %zu bytes of device scratch this entry point "
                    "has (use awc_forward for larger problems)",
                    kScratchBytes);
    return fail(AWC_ERR_INVALID, msg);
  }

  unsigned char* S = nullptr;
  if (int rc = scratch_address(&S)) return rc;
  float* buf[3] = {(float*)(S + o_buf), (float*)(S + o_buf) + N, (float*)(S + o_buf) + 2 * N};
  float* fact = (float*)(S + o_fact);
  double* veld = (double*)(S + o_vel);
  float* cf = (float*)(S + o_cf);

  // ---- inputs in, state cleared (the array keeps the last call's data) ---
  STATIC_TRY(cudaMemset(S + o_buf, 0, 3 * N * sizeof(float)));
  STATIC_TRY(cudaMemset(S + o_psx, 0, o_cd - o_psx));  // ψ and ξ of both axes
  STATIC_TRY(cudaMemset(S + o_tr, 0, nt * nr * sizeof(double)));
  STATIC_TRY(cudaMemset(S + o_blk, 0, ((int64_t)gx * gy + 1) * sizeof(int32_t)));
  STATIC_TRY(cudaMemcpy(veld, vel, N * sizeof(double), cudaMemcpyHostToDevice));
  STATIC_TRY(cudaMemcpy(S + o_cd, coeffs, clen * sizeof(double), cudaMemcpyHostToDevice));
  if (nt * ns > 0)
    STATIC_TRY(cudaMemcpy(S + o_stf, dt2srctf, nt * ns * sizeof(double), cudaMemcpyHostToDevice));
  if (ns > 0) {
    STATIC_TRY(cudaMemcpy(S + o_gn, grp_node.data(), ngrp * sizeof(int64_t), cudaMemcpyHostToDevice));
    STATIC_TRY(cudaMemcpy(S + o_go, grp_off.data(), (ngrp + 1) * sizeof(int32_t), cudaMemcpyHostToDevice));
    STATIC_TRY(cudaMemcpy(S + o_gs, order.data(), ns * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  if (nr > 0) STATIC_TRY(cudaMemcpy(S + o_pr, rec_node.data(), nr * sizeof(int64_t), cudaMemcpyHostToDevice));
  awc::make_fact<float><<<256, 256>>>(veld, fact, p->dt * p->dt, N, nx, nx);
  static_narrow<<<1, 256>>>((const double*)(S + o_cd), cf, clen);
  STATIC_TRY(cudaGetLastError());

  // ---- step parameters (the step2d kernel of awc_forward) ----------------
  awc::StepParams<float> P{};
  P.fact = fact;
  P.nx = (int32_t)nx;
  P.ny = (int32_t)ny;
  P.nz = 1;
  P.halo = (int32_t)h;
  P.px = nx;
  const double d[2] = {p->dx, p->dy};
  for (int a = 0; a < 2; ++a) {
    P.inv_d[a] = (float)(1.0 / d[a]);
    P.inv_d2[a] = (float)(1.0 / (d[a] * d[a]));
  }
  float* psx = (float*)(S + o_psx);
  float* xix = (float*)(S + o_xix);
  float* psy = (float*)(S + o_psy);
  float* xiy = (float*)(S + o_xiy);
  const int64_t cs[2] = {ny, nx};  // band cross-sections of axes x and y
  float* ps_base[2] = {psx, psy};
  float* xi_base[2] = {xix, xiy};
  for (int a = 0; a < 2; ++a) {
    const double* blk = coeffs + a * (8 * h + 4);
    for (int s = 0; s < 2; ++s) {
      // a side whose a are all 0 and b/K all 1 keeps ψ = ξ = 0 (the free top)
      bool trivial = true;
      for (int64_t m = 0; m < h; ++m)
        trivial = trivial && blk[s * h + m] == 0.0 && blk[2 * h + s * h + m] == 1.0;
      for (int64_t m = 0; m < h + 1; ++m)
        trivial = trivial && blk[4 * h + s * (h + 1) + m] == 0.0 &&
                  blk[4 * h + 2 * (h + 1) + s * (h + 1) + m] == 1.0;
      P.active[a][s] = (h > 0 && !trivial) ? 1 : 0;
      const float* cb = cf + a * (8 * h + 4);
      awc::BandSide<float>& B = P.band[a][s];
      B.xi = xi_base[a] + s * h * cs[a];
      B.a = cb + s * h;
      B.bK = cb + 2 * h + s * h;
      B.ah = cb + 4 * h + s * (h + 1);
      B.bKh = cb + 4 * h + 2 * (h + 1) + s * (h + 1);
    }
    const int64_t n = a == 0 ? nx : ny;
    P.first_r[a] = (int32_t)(n - h - 1 > h + 1 ? n - h - 1 : h + 1);
  }
  P.zchunk = 1;
  P.io.blk_off = (const int32_t*)(S + o_blk);  // all zero: I/O is done by static_io
  P.io.nrim = 0;
  P.do_rim = 0;
  P.err = nullptr;

  // ---- time loop ----------------------------------------------------------
  const double* stf = (const double*)(S + o_stf);
  const int64_t* gnode = (const int64_t*)(S + o_gn);
  const int32_t* goff = (const int32_t*)(S + o_go);
  const int32_t* gsrc = (const int32_t*)(S + o_gs);
  const int64_t* rnode = (const int64_t*)(S + o_pr);
  double* dtr = (double*)(S + o_tr);
  const int io_threads = (int)((ngrp > nr ? ngrp : nr) > 255 ? 256 : 32);
  for (int64_t it = 0; it < nt; ++it) {
    P.pold = buf[it % 3];
    P.pcur = buf[(it + 1) % 3];
    P.pnew = buf[(it + 2) % 3];
    for (int a = 0; a < 2; ++a)
      for (int s = 0; s < 2; ++s) {
        float* base = ps_base[a] + (int64_t)s * 2 * (h + 1) * cs[a];
        P.band[a][s].psi_old = base + (it & 1) * (h + 1) * cs[a];
        P.band[a][s].psi_new = base + ((it + 1) & 1) * (h + 1) * cs[a];
      }
    P.it = (int32_t)it;
    awc::step2d<float><<<dim3(gx, gy), dim3(32, 8)>>>(P);
    if (ns > 0 || nr > 0)
      static_io<<<1, io_threads>>>(P.pnew, stf, gnode, goff, gsrc, (int)ngrp, rnode, (int)nr, nt,
                                   it, dtr);
  }
  STATIC_TRY(cudaGetLastError());

  // ---- outputs -------------------------------------------------------------
  if (nt * nr > 0) STATIC_TRY(cudaMemcpy(traces, dtr, nt * nr * sizeof(double), cudaMemcpyDeviceToHost));
  if (pfinal) {
    awc::unpitch<float><<<256, 256>>>(buf[(nt + 1) % 3], veld, N, nx, nx);
    STATIC_TRY(cudaGetLastError());
    STATIC_TRY(cudaMemcpy(pfinal, veld, N * sizeof(double), cudaMemcpyDeviceToHost));
  }
  STATIC_TRY(cudaStreamSynchronize(0));
  return AWC_OK;
}
