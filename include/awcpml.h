/*
 * awcpml.h — C ABI of the B200 (sm_100a) CPML acoustic time-stepping library.
 *
 * This library replaces the device time loop behind the Julia entry points
 * Acoustic2D_CUDA.solve2D / Acoustic3D_CUDA.solve3D of AcousticWaveCPML.jl
 * (src/Acoustic2D_CUDA.jl:52-56, src/Acoustic3D_CUDA.jl:60-64, whose bodies are
 * src/shared/acoustic_2D_xPU.jl:133-445 and src/shared/acoustic_3D_xPU.jl:169-545).
 * The Julia side keeps the reference's host setup (dt, nt, CPML coefficients,
 * source time functions, position snapping) and hands the arrays to
 * awc_forward(); everything the reference runs through ParallelStencil kernels
 * (update_ψ_*!, update_p!, inject_sources!, record_receivers!, forward!) runs
 * here as one fused CUDA kernel per time step, replayed from a CUDA graph.
 *
 * Conventions shared by every entry point:
 *  - Arrays are host memory, column-major (Julia layout), unless stated.
 *  - Grid sizes nx, ny, nz count every node, CPML band and the Dirichlet rim
 *    included (the size of `vel` in the reference). 2D problems use nz = 1.
 *  - Positions are 1-based Int64 grid indices, (n × ndim) column-major, i.e.
 *    pos[s + n*d] is coordinate d of item s, exactly as the reference stores
 *    possrcs/posrecs (acoustic_3D_xPU.jl:277-289).
 *  - Return value: AWC_OK (0) or a negative AWC_ERR_* code; the message is
 *    available from awc_last_error(). The library never aborts the process.
 *  - Depth is the second array axis (j, "y"), as in the reference: the free
 *    top surface is j = 1 (acoustic_3D_xPU.jl:225-230).
 */
#ifndef AWCPML_H
#define AWCPML_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AWC_OK 0
#define AWC_ERR_INVALID (-1)  /* bad argument (shape, position, size, pointer) */
#define AWC_ERR_OOM (-2)      /* device memory allocation failed */
#define AWC_ERR_CUDA (-3)     /* a CUDA runtime call failed */
#define AWC_ERR_TIMEOUT (-4)  /* a bounded device wait ran out */
#define AWC_ERR_NODEVICE (-5) /* no usable sm_100 device */

#define AWC_F32 1 /* fields, ψ, ξ and coefficients stored and updated in float */
#define AWC_F64 2 /* everything in double (parity build) */

/* One forward problem: a single shot on one velocity model.
 * Mirrors the scalars solve2D/solve3D derive (acoustic_3D_xPU.jl:195-206),
 * and solve1D's (src/shared/acoustic_1D.jl:104-128) with ndim = 1:
 * ny = nz = 1, dy/dz/freetop unused, positions (n x 1); a 1D problem runs as
 * the middle line of a three-row 2D problem with no y derivative and no y
 * CPML (awc_forward, the plan API and snapshots; not the batch, adjoint or
 * learned-layer entry points). */
typedef struct awc_problem {
  int32_t ndim;      /* 1, 2 or 3 */
  int32_t precision; /* AWC_F32 or AWC_F64 */
  int64_t nx, ny, nz;
  int32_t halo;    /* CPML layers per side (reference keyword `halo`) */
  int32_t freetop; /* 1: no CPML on the j = 1 side (coefficients say so too) */
  double dx, dy, dz; /* grid spacing [m]; dz ignored in 2D */
  double dt;         /* time step [s] */
  int64_t nt;        /* number of time steps */
  int64_t nsrc, nrec;
} awc_problem;

/* Number of doubles in the packed CPML coefficient array for `p`:
 * ndim blocks of (8*halo + 4), each block laid out as
 *   a_l[halo] a_r[halo] bK_l[halo] bK_r[halo]
 *   a_hl[halo+1] a_hr[halo+1] bK_hl[halo+1] bK_hr[halo+1]
 * for axis x, then y, then z (the 24 vectors of acoustic_3D_xPU.jl:218-223). */
int64_t awc_coeffs_len(const awc_problem* p);

/* calc_Kab_CPML (src/utils.jl:19-57): K, a, b CPML profile of `halo` layers.
 * halfgrid = 0 gives the on-grid set (length halo), 1 the staggered set
 * (length halo+1). Outputs a_l, a_r, bK_l = b/K left, bK_r = b/K right. FP64. */
int awc_cpml_coeffs(int32_t halo, double dt, double npower, double d0, double alpha_max,
                    double K_max, int32_t halfgrid, double* a_l, double* a_r, double* bK_l,
                    double* bK_r);

/* The CPML block of solve2D/solve3D (acoustic_3D_xPU.jl:207-230,
 * acoustic_2D_xPU.jl:166-185): alpha_max = π f0, npower = 2, K_max = 1,
 * d0 = -(npower+1) vel_max log(rcoef) / (2 halo d) per axis, both grids, then
 * the free-top override when p->freetop. Fills awc_coeffs_len(p) doubles. */
int awc_problem_coeffs(const awc_problem* p, double rcoef, double f0, double vel_max,
                       double* coeffs);

/* rickersource1D (src/utils.jl:64-66) evaluated at n times. */
int awc_ricker(int64_t n, const double* t, double t0, double f0, double* out);

/* Opaque per-thread context: owns the CUDA stream, device buffers and the
 * captured time-loop graphs (cached by problem shape). Not thread-safe; use
 * one context per host thread. */
typedef struct awc_ctx awc_ctx;

/* Creates a context on CUDA device `device` (must be sm_100). */
int awc_create(awc_ctx** out, int32_t device);
void awc_destroy(awc_ctx* ctx);
/* Last error message of `ctx`, or of the calling thread when ctx is NULL. */
const char* awc_last_error(const awc_ctx* ctx);
/* Device time [ms] of the time loop of the last awc_forward on `ctx`
 * (CUDA events around the graph replay; host copies excluded). */
float awc_last_run_ms(const awc_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), on which every copy and kernel
 * of the context is ordered; callers may record their own events on it. */
void* awc_ctx_stream(const awc_ctx* ctx);
/* Steps per candidate with which awc_forward autotunes the launch shape of
 * each new 3D problem shape (nt >= 100) before its first solve; 0 disables
 * it. Default 40. The choice is cached with the plan. */
int awc_ctx_set_autotune(awc_ctx* ctx, int64_t steps);

/* The forward solve (the time loop of acoustic_3D_xPU.jl:392-409 and the
 * returns at :541-544; 2D acoustic_2D_xPU.jl:327-343, :441-444).
 *   vel      [nx*ny*nz]       velocity [m/s]; fact = dt^2 vel^2 is formed on
 *                             the device in FP64 (acoustic_3D_xPU.jl:242)
 *   coeffs   [awc_coeffs_len] packed CPML vectors (awc_problem_coeffs)
 *   possrcs  [nsrc*ndim]      1-based source nodes
 *   dt2srctf [nt*nsrc]        scaled source time functions, column-major
 *                             (acoustic_3D_xPU.jl:272-275)
 *   posrecs  [nrec*ndim]      1-based receiver nodes
 *   traces   [nt*nrec] out    recorded pressure, traces[it + nt*r]
 *   pfinal   [nx*ny*nz] out   final field (the reference's Array(pcur));
 *                             may be NULL
 * Step it (1-based) updates ψ, ξ and p, adds dt2srctf[it, s] into the new
 * field at each source, then records the new field at each receiver. Several
 * sources on one node are summed in source order. */
int awc_forward(awc_ctx* ctx, const awc_problem* p, const double* vel, const double* coeffs,
                const int64_t* possrcs, const double* dt2srctf, const int64_t* posrecs,
                double* traces, double* pfinal);

/* Domain decomposition, the reference's multi-process strategy
 * (solve2D_multi/solve3D_multi, src/shared/acoustic_3D_multixPU.jl:157-230:
 * each rank updates its subdomain, then update_halo! exchanges one plane per
 * interface): the problem of awc_forward split along its last axis (y in
 * 2D, z in 3D) into nsub contiguous subdomains of nearly equal size, each a
 * plan on ctxs[s] with a halo plane on each inner side. Every time step all
 * subdomains advance, then each interface's two planes cross it (peer copies
 * when the contexts sit on different devices; a context may appear several
 * times, its subdomains then take turns on its stream). The CPML of the
 * split axis stays on the outer subdomains, which need at least 2 halo + 2
 * planes along it. Sources and receivers belong to the subdomain that
 * updates their node. Results (traces, final field) are bitwise those of
 * awc_forward. No sources or receivers are exchanged: only field planes. */
int awc_forward_decomposed(awc_ctx* const* ctxs, int32_t nsub, const awc_problem* p,
                           const double* vel, const double* coeffs, const int64_t* possrcs,
                           const double* dt2srctf, const int64_t* posrecs, double* traces,
                           double* pfinal);

/* Device-resident plan: the inputs of awc_forward uploaded once, the state
 * kept in HBM between calls. awc_forward is plan create + run(nt) + read-out.
 * The plan belongs to its context and must be destroyed before it. */
typedef struct awc_plan awc_plan;

int awc_plan_create(awc_ctx* ctx, const awc_problem* p, const double* vel, const double* coeffs,
                    const int64_t* possrcs, const double* dt2srctf, const int64_t* posrecs,
                    awc_plan** out);
void awc_plan_destroy(awc_plan* plan);
/* Zeroes pressure, ψ, ξ and traces; the next run starts at it = 1. */
int awc_plan_reset(awc_plan* plan);
/* Advances `nsteps` time steps (clamped to nt). use_graph = 1 replays a
 * captured CUDA graph, 0 launches the kernels one by one. When ms != NULL the
 * device time of the run, measured with CUDA events on the plan's stream, is
 * written there. Returns after the run completes. */
int awc_plan_run(awc_plan* plan, int64_t nsteps, int32_t use_graph, float* ms);
/* Steps completed since the last reset. */
int64_t awc_plan_step(const awc_plan* plan);
/* Snapshot output, the do_save branch of solve3D (acoustic_3D_xPU.jl:375-379,
 * 479-498, which writes pcur to an HDF5 file after every step it with
 * it % nsave == 0): advances `nsteps` steps (clamped to nt) like
 * awc_plan_run and copies the current field after each step whose 1-based
 * count since the reset is a multiple of nsave into `out` (host memory,
 * column-major doubles), snapshot j at out + j*nx*ny*nz, in order. The copy
 * of a snapshot overlaps the steps that follow it (second stream, two device
 * staging fields); use pinned host memory for the overlap. Returns
 * AWC_ERR_INVALID, before running, when more than max_snaps snapshots fall in
 * the run; *nsnaps (may be NULL) receives the number written. Kernels launch
 * one by one (no graph). Callers split a long run into pieces whose
 * snapshots fit their buffer and write each piece out as it returns. */
int awc_plan_run_snapshots(awc_plan* plan, int64_t nsteps, int64_t nsave, double* out,
                           int64_t max_snaps, int64_t* nsnaps);
/* Copies the traces (nt*nrec, column-major; rows not yet reached are zero)
 * and the current field (the latest new pressure, nx*ny*nz) to the host. */
int awc_plan_traces(awc_plan* plan, double* traces);
int awc_plan_field(awc_plan* plan, double* p);
/* Number of kernel launches one time step issues (for launch accounting):
 * 2 for a 3D problem with both a core and a CPML band region, else 1. */
int32_t awc_plan_launches_per_step(const awc_plan* plan);
/* Launch shape of a 3D time step, which runs as two kernels over disjoint
 * nodes: the core kernel (nodes outside every CPML band; blocks of 64 x
 * `tile_y` nodes, tile_y = 4, 8 or 16, streaming `zchunk` z planes through a
 * TMA pipeline) and the band kernel (the CPML band nodes; 32 x 8 columns
 * streaming `band_zchunk` planes, 1..255). Every shape gives the same
 * results; only the speed differs. The state is kept. 2D plans ignore it. */
int awc_plan_set_launch(awc_plan* plan, int32_t tile_y, int32_t zchunk, int32_t band_zchunk);
int awc_plan_get_launch(const awc_plan* plan, int32_t* tile_y, int32_t* zchunk,
                        int32_t* band_zchunk);
/* Times `steps` time steps of every candidate launch shape on this plan's own
 * data, keeps the fastest, and resets the state. Writes the best time per
 * step [ms] to best_ms_per_step when not NULL. */
int awc_plan_autotune(awc_plan* plan, int64_t steps, float* best_ms_per_step);
/* Time blocking of a 3D plan: `depth` time steps per kernel pass, 1 or 2.
 * At depth 2 one pass of one kernel advances two steps (two launches per
 * pass, run as parallel graph branches: the column tiles that meet an x or y
 * CPML band, and the others). A block of 32 x `rows` threads (rows 8 or 16)
 * stages p_s, p_{s-1} and fact of a 62 x (rows - 2) column tile plus a
 * one-node ring through TMA, computes step s+1 on the tile and its ring and
 * step s+2 on the tile (each thread an x pair of nodes), streaming one of
 * `zchunks` chunks of z planes; per node and two steps the fields cost 5 words of HBM
 * traffic instead of 8, and the CPML state one read and one write instead of
 * two. Results are bitwise those of depth 1; an odd step count ends with a
 * one-step launch. Depth 2 needs a 3D problem whose sources and receivers are
 * all interior nodes (AWC_ERR_INVALID otherwise). The state is kept.
 * awc_plan_autotune times depth 2 as well and keeps the faster. No
 * counterpart in the reference, whose forward! advances one step per
 * launch sequence (src/shared/acoustic_3D_xPU.jl:124-167). */
int awc_plan_set_blocking(awc_plan* plan, int32_t depth, int32_t rows, int32_t zchunks);
int awc_plan_get_blocking(const awc_plan* plan, int32_t* depth, int32_t* rows, int32_t* zchunks);
/* Kernel launches that a run of nsteps steps from the plan's current step
 * issues (for launch accounting at either depth); -1 on a bad argument. */
int64_t awc_plan_launch_count(const awc_plan* plan, int64_t nsteps);
/* Bounded waits of the two-step kernel's TMA pipeline: a wait gives up after
 * `rounds` try-waits of at most round_ns nanoseconds each (default 4096 x
 * 1 ms), and the run returns AWC_ERR_TIMEOUT with the context still usable.
 * withhold >= 0 exists to test that path: the producer of every block skips
 * the plane load with that index, so that its consumers' wait runs out;
 * -1 (the default) loads every plane. */
int awc_plan_set_wait(awc_plan* plan, int32_t rounds, int32_t round_ns, int32_t withhold);

/* ---- Batched 2D shots ----------------------------------------------------
 * Many shots over several 2D velocity models of uneven size advance together:
 * one kernel launch per time step covers every shot, and the nt-step loop is
 * one CUDA graph. Each shot computes what awc_forward computes for the same
 * problem. No counterpart in the reference, whose solve2D runs one shot per
 * call (src/shared/acoustic_2D_xPU.jl:133-445). */
typedef struct awc_shot {
  int32_t model;          /* index of the shot's velocity model */
  int32_t nsrc, nrec;
  const double* coeffs;   /* packed CPML coefficients of the shot (they depend
                             on its f0 through alpha_max = pi f0) */
  const int64_t* possrcs; /* (nsrc x 2) 1-based nodes */
  const double* dt2srctf; /* (nt x nsrc) scaled source time functions */
  const int64_t* posrecs; /* (nrec x 2) 1-based nodes */
} awc_shot;

typedef struct awc_batch awc_batch;

/* models[m]: model m (ndim = 2; every model has the same precision and nt;
 * its own nx, ny, dx, dy, dt, halo; nsrc/nrec ignored); vel[m]: its velocity
 * (nx*ny, column-major). */
int awc_batch_create(awc_ctx* ctx, int32_t nmodels, const awc_problem* models,
                     const double* const* vel, int32_t nshots, const awc_shot* shots,
                     awc_batch** out);
void awc_batch_destroy(awc_batch* batch);
int awc_batch_reset(awc_batch* batch);
/* Same contract as awc_plan_run, for every shot of the batch. */
int awc_batch_run(awc_batch* batch, int64_t nsteps, int32_t use_graph, float* ms);
int64_t awc_batch_step(const awc_batch* batch);
/* One shot's traces (nt x nrec) and current field (nx*ny), as doubles. */
int awc_batch_traces(awc_batch* batch, int32_t shot, double* traces);
int awc_batch_field(awc_batch* batch, int32_t shot, double* p);
/* Tile height and resident blocks per SM (1..32) of the persistent step
 * kernel; results do not depend on them. tile_y 4, 8 or 16: tiles 64 nodes
 * wide staged through shared memory by TMA (4 consumer warps of tile_y/4 rows
 * and a producer warp per block); 32 or 64: tiles 32 nodes wide read into
 * registers (4 warps per block, each streaming tile_y/4 rows). */
int awc_batch_set_launch(awc_batch* batch, int32_t tile_y, int32_t blocks_per_sm);
int awc_batch_get_launch(const awc_batch* batch, int32_t* tile_y, int32_t* blocks_per_sm);
/* Times every launch shape on the batch's data, keeps the fastest, resets. */
int awc_batch_autotune(awc_batch* batch, int64_t steps, float* best_ms_per_step);
/* create + autotune (nt >= 100) + run(nt) + every shot's traces + destroy;
 * traces[s] is shot s's (nt x nrec) output. */
int awc_forward_batch(awc_ctx* ctx, int32_t nmodels, const awc_problem* models,
                      const double* const* vel, int32_t nshots, const awc_shot* shots,
                      double* const* traces);

/* ---- Adjoint ---------------------------------------------------------------
 * No counterpart in the reference, which has no gradient. Both entry points
 * run the exact discrete transpose of the time step above (awc_forward's
 * arithmetic for fixed c), backwards in time, on the interior nodes. They
 * need CPML bands that do not overlap (n >= 2 halo + 2 on each axis). Their
 * plan and working memory (nt / checkpoint_every saved states, the
 * checkpoint_every + 2 pressure fields of a segment and the adjoint fields)
 * stay allocated in the context between calls of one shape, so that a
 * sequence of gradients of one survey allocates once; a call of another
 * shape replaces them and awc_destroy frees them.
 *
 * awc_misfit_gradient: J = 1/2 Σ_t Σ_r (traces[t,r] - observed[t,r])² of the
 * shot described like awc_forward, and dJ/d(c²) per node (nx*ny[*nz],
 * column-major, 0 on the rim). The forward state is saved every
 * `checkpoint_every` steps and each segment is recomputed once during the
 * backward pass, the next one beside the current one's adjoint steps
 * (memory: nt / checkpoint_every saved states plus two sets of
 * checkpoint_every + 2 pressure fields, one set when a single segment covers
 * nt). `traces` (nt x nrec) may be NULL. */
int awc_misfit_gradient(awc_ctx* ctx, const awc_problem* p, const double* vel,
                        const double* coeffs, const int64_t* possrcs, const double* dt2srctf,
                        const int64_t* posrecs, const double* observed, int32_t checkpoint_every,
                        double* misfit, double* grad_c2, double* traces);

/* awc_misfit_gradient summed over `nshot` shots of one model (the sum of
 * the shots' J and of their dJ/d(c²), each shot's as awc_misfit_gradient
 * returns it, added in shot order): vel is uploaded once, the gradients
 * are summed on the device and read back once. The shots share p (so the
 * same nsrc, nrec and nt), vel, coeffs and posrecs; shot s reads
 * possrcs + s*nsrc*ndim (nsrc x ndim), dt2srctf + s*nt*nsrc (nt x nsrc) and
 * observed + s*nt*nrec (nt x nrec). Replaces a caller-side loop of
 * awc_misfit_gradient calls over the shots of one source survey. */
int awc_misfit_gradient_shots(awc_ctx* ctx, const awc_problem* p, int32_t nshot,
                              const double* vel, const double* coeffs, const int64_t* possrcs,
                              const double* dt2srctf, const int64_t* posrecs,
                              const double* observed, int32_t checkpoint_every, double* misfit,
                              double* grad_c2);

/* The transpose of the linear map from injected source values (dt2srctf,
 * nt x nsrc) to traces (nt x nrec) for fixed c: src_out (nt x nsrc) =
 * Aᵀ adjoint_traces. Sources and receivers on the Dirichlet rim have no
 * adjoint (their entries are 0). */
int awc_adjoint_sources(awc_ctx* ctx, const awc_problem* p, const double* vel,
                        const double* coeffs, const int64_t* possrcs, const int64_t* posrecs,
                        const double* adjoint_traces, double* src_out);

/* ---- Learned thin absorbing layer --------------------------------------------
 * No counterpart in the reference. awc_forward with the CPML replaced by a
 * layer of p->halo (1..8) nodes on every absorbing side whose new values come
 * from a small MLP: the block of 3^d nodes around a layer node at the three
 * latest time levels (oriented along the nearest side's outward normal and
 * scaled by their largest magnitude) and the local Courant number, K = 28
 * inputs in 2D, 82 in 3D, then K -> 32 -> 32 -> 1 with ReLU. Interior nodes take the plain leapfrog step.
 * FP32 only (p->precision == AWC_F32); `coeffs` are not used; sources and
 * receivers must be interior nodes. weights_bf16: awc_learned_weights_len(ndim)
 * BF16 values, W1 (32 x K, row-major), b1 (32), W2 (32 x 32), b2 (32),
 * W3 (32), b3 (1). */
int awc_learned_weights_len(int32_t ndim);
int awc_forward_learned(awc_ctx* ctx, const awc_problem* p, const double* vel,
                        const uint16_t* weights_bf16, const int64_t* possrcs,
                        const double* dt2srctf, const int64_t* posrecs, double* traces,
                        double* pfinal);

/* awc_forward for 2D FP32 problems without any device memory allocation.
 * No counterpart in the reference (its solvers always allocate).
 *
 * For callers that cannot let a library call cudaMalloc: a solver loop that
 * must not stall the device (cudaMalloc/cudaFree synchronise it), or a host
 * framework whose own allocator owns all device memory (Julia CUDA.jl's pool,
 * a caching allocator), where allocations it does not see starve it.
 * Arguments, layouts and results are those of awc_forward with p->ndim == 2
 * and p->precision == AWC_F32; no context is needed. Every device buffer of
 * the solve lives in one fixed 32 MiB array of device memory, which exists on
 * every GPU that loads this library until the process exits. A problem needs
 * about 24 nx ny + 8 nt nrec + 8 nt nsrc bytes plus the CPML band arrays;
 * larger problems are rejected with AWC_ERR_INVALID and a message giving the
 * size needed (use awc_forward for them).
 * Every call looks up the array's device address with cudaGetSymbolAddress
 * (so a device reset between calls is harmless); the first call on a device
 * also loads the module there, so make that first call before any stream
 * capture. Several sources on one node are summed in source order, as in
 * awc_forward, and the scalar limits are awc_forward's (nt <= 2^31, finite
 * positive spacing and dt). Every call clears the state it
 * needs, but all calls share the one array: calls that overlap on the GPU
 * (from several host threads on one device) race and must be serialised by
 * the caller. Runs on the current device and the legacy default stream and
 * returns when the results are on the host. */
int awc_forward2d_f32_static(const awc_problem* p, const double* vel, const double* coeffs,
                             const int64_t* possrcs, const double* dt2srctf,
                             const int64_t* posrecs, double* traces, double* pfinal);

#ifdef __cplusplus
}
#endif

#endif /* AWCPML_H */
