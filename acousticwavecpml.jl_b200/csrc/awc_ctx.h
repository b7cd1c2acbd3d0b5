// awc_ctx.h — the context object shared by the translation units of
// libawcpml (internal; the public API sees it as an opaque handle).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/awcpml.h"

struct awc_plan;

struct awc_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;  // second branch of a 3D step (the band kernel)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string err;
  float last_run_ms = 0.f;
  int64_t autotune_steps = 40;   // per candidate, for new 3D plans of awc_forward
  std::vector<awc_plan*> cache;  // plans reused by awc_forward, most recent last
  // the adjoint entry points keep their plan and working memory between
  // calls of one shape (released by awc_destroy or a call of another shape)
  awc_plan* adj_plan = nullptr;
  void* adj_mem = nullptr;
  std::function<void()> adj_release;
  // the adjoint's backward steps run on their own two streams, so that a
  // segment's recompute (on `stream`) overlaps the previous segment's
  // backward steps; events: fork, join, recomputed, segment set 0/1 free
  cudaStream_t adj_stream[2] = {nullptr, nullptr};
  cudaEvent_t adj_ev[5] = {};
  // pinned host staging buffer for large pageable copies (grown on demand)
  void* host_stage = nullptr;
  size_t host_stage_bytes = 0;
};

namespace awc {
// The device state of a plan, for code outside the forward stepper (the
// adjoint): step it reads pold = buf[it % 3], pcur = buf[(it + 1) % 3] and
// writes pnew = buf[(it + 2) % 3]; ψ_old of step it is psi[axis][side][it & 1].
struct PlanView {
  int32_t ndim = 0, precision = 0, halo = 0;
  int64_t nx = 0, ny = 0, nz = 1, px = 0, NP = 0, nt = 0;
  size_t esz = 0;
  void* buf[3] = {};
  const void* fact = nullptr;
  void* psi[3][2][2] = {};
  void* xi[3][2] = {};
  int64_t psi_len[3] = {}, xi_len[3] = {};  // elements of one side's array
  const void* coef = nullptr;               // packed coefficients in the working precision
  int32_t active[3][2] = {};
  const void* traces = nullptr;             // device [nt][nrec]
  int32_t* err_flag = nullptr;              // device flag of timed-out bounded waits
  cudaStream_t stream = nullptr;
};
PlanView plan_view(awc_plan* P);
// Sets the step counter of a plan whose state was restored from a copy.
void plan_set_step(awc_plan* P, int64_t step);
// Keeps the new field of each step it in [first, first + count) in
// dst[it - first]: a stream-ordered copy after the step, or, in place (when
// the shot has no source or receiver on the rim; else copied), the step
// writes it there and reads p_{it-1}, p_it from dst[it - first - 2],
// dst[it - first - 1] (dst[-2] and dst[-1] must hold p_{first-1} and
// p_first, and every dst field a zero rim); the plan's own buffers are
// refreshed after the last step. NULL stops it.
void plan_keep_fields(awc_plan* P, void* const* dst, int64_t first, int64_t count,
                      bool in_place = false);

// Re-uploads a new shot into *slot when it holds a plan of the same shape
// (same buffers), else replaces it by a new plan, whose 3D launch shape is
// autotuned when `tune` is set (one-step passes either way). The plan is
// reset.
int plan_for(awc_ctx* C, awc_plan** slot, const awc_problem* p, const double* vel,
             const double* coeffs, const int64_t* possrcs, const double* dt2srctf,
             const int64_t* posrecs, bool tune = false);
// Replaces the sources and receivers of plan P (its model, fact and CPML
// coefficients kept) and resets it: the next shot over the same model.
int plan_shot(awc_ctx* C, awc_plan* P, const int64_t* possrcs, const double* dt2srctf,
              const int64_t* posrecs);

// Host <-> device copies that return once complete. Large pageable host
// buffers go through the context's pinned staging buffer, the host side of
// the copy split over several threads; pinned buffers and small copies go
// directly.
cudaError_t copy_to_device(awc_ctx* C, void* dst, const void* src, size_t bytes, cudaStream_t st);
cudaError_t copy_to_host(awc_ctx* C, void* dst, const void* src, size_t bytes, cudaStream_t st);

// Sets the calling thread's last error (awc_last_error(NULL)) and, when ctx
// is not NULL, the context's; returns code.
int fail(awc_ctx* ctx, int code, const char* msg);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda); NULL when the driver does not offer it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();
}  // namespace awc
