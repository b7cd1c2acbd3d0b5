// awc_ctx.h — the context object shared by the translation units of
// libawcpml (internal; the public API sees it as an opaque handle).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

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
  int64_t autotune_steps = 10;   // per candidate, for new 3D plans of awc_forward
  std::vector<awc_plan*> cache;  // plans reused by awc_forward, most recent last
};

namespace awc {
// Sets the calling thread's last error (awc_last_error(NULL)) and, when ctx
// is not NULL, the context's; returns code.
int fail(awc_ctx* ctx, int code, const char* msg);
}  // namespace awc
