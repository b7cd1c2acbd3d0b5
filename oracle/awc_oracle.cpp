// awc_oracle.cpp — CPU FP64 restatement of AcousticWaveCPML.jl's CPML
// time-stepping path. TEST INFRASTRUCTURE ONLY: the parity tests, the smoke
// check and the CPU-baseline leg of the benchmark load it as the checker.
// Nothing in the product (the CUDA library or its host wrappers) calls it.
//
// Parity is pinned against the reference's own golden fields
// (test/references/acoustic2D_{center_halo20,center_freetop_halo20,
// gradient_freetop_halo20}.bson) and its ψ known-answer tests
// (test/test2D.jl:13-43, test/test3D.jl:13-71). The 3D path has no golden
// field in the reference tree (.MISSING_LARGE_BLOBS lists the 3D BSONs), so in
// 3D it is pinned by the analytic Green's-function tests and by sharing every
// line of arithmetic with the pinned 2D path.
//
// Each function names the reference lines it restates. The op order of every
// floating-point expression follows the reference (no contraction: build with
// -ffp-contract=off), so that the FP64 result matches the Julia Float64 run to
// rounding. The step structure is the xPU one: all ψ updates for the step
// first (update_ψ_{x,y,z}!), then update_p!, inject_sources!,
// record_receivers!, then the (pold, pcur, pnew) <- (pcur, pnew, pold)
// rotation (src/shared/acoustic_3D_xPU.jl:124-167).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/awcpml.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

double g_loop_seconds = 0.0;

double wall_seconds() {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return 0.0;
#endif
}

// Column-major index helpers (1-based, like the reference).
struct Dims {
  int64_t nx, ny, nz;
  inline int64_t at(int64_t i, int64_t j, int64_t k) const {
    return (i - 1) + nx * ((j - 1) + ny * (k - 1));
  }
};

// LinRange element (Base.lerpi): t = j/d; (1-t)*a + t*b.
inline double lerpi(int64_t j, int64_t d, double a, double b) {
  double t = (double)j / (double)d;
  return (1.0 - t) * a + t * b;
}

}  // namespace

extern "C" {

// calc_Kab_CPML, src/utils.jl:19-57.
int oracle_calc_Kab_CPML(int32_t halo, double dt, double npower, double d0, double alpha_max_pml,
                         double K_max_pml, int32_t halfgrd, double* a_left, double* a_right,
                         double* b_K_left, double* b_K_right) {
  int64_t Kab_size = halo;
  double shift = 0.0;
  if (halfgrd) {  // utils.jl:25-27
    Kab_size += 1;
    shift = 0.5;
  }
  if (Kab_size == 0) return 0;
  // dist = collect(LinRange(0-shift, Kab_size-shift-1, Kab_size)) (utils.jl:35)
  std::vector<double> dist(Kab_size);
  double start = 0.0 - shift, stop = (double)Kab_size - shift - 1.0;
  if (Kab_size == 1) {
    dist[0] = start;
  } else {
    for (int64_t j = 0; j < Kab_size; ++j) dist[j] = lerpi(j, Kab_size - 1, start, stop);
  }
  if (halfgrd) dist[0] = 0.0;  // utils.jl:36-38
  for (int64_t n = 0; n < Kab_size; ++n) {
    // normdist_left = reverse(dist) ./ halo ; normdist_right = dist ./ halo (utils.jl:39-40)
    double nl = dist[Kab_size - 1 - n] / (double)halo;
    double nr = dist[n] / (double)halo;
    // x^npower with a Float64 exponent; Julia evaluates an integral exponent 2
    // as the correctly rounded x*x, and npower = 2.0 in every caller.
    double nlp = npower == 2.0 ? nl * nl : std::pow(nl, npower);
    double nrp = npower == 2.0 ? nr * nr : std::pow(nr, npower);
    double d_l = d0 * nlp;                             // utils.jl:42
    double al_l = alpha_max_pml * (1.0 - nl);          // :43
    double K_l = 1.0 + (K_max_pml - 1.0) * nlp;        // :44
    double b_l = std::exp(-(d_l / K_l + al_l) * dt);   // :45
    a_left[n] = d_l * (b_l - 1.0) / (K_l * (d_l + K_l * al_l));  // :46
    b_K_left[n] = b_l / K_l;                           // :47
    double d_r = d0 * nrp;                             // :49
    double al_r = alpha_max_pml * (1.0 - nr);          // :50
    double K_r = 1.0 + (K_max_pml - 1.0) * nrp;        // :51
    double b_r = std::exp(-(d_r / K_r + al_r) * dt);   // :52
    a_right[n] = d_r * (b_r - 1.0) / (K_r * (d_r + K_r * al_r));  // :53
    b_K_right[n] = b_r / K_r;                          // :54
  }
  return 0;
}

// rickersource1D, src/utils.jl:64-66.
double oracle_ricker(double t, double t0, double f0) {
  double x = M_PI * f0 * (t - t0);
  return (1.0 - 2.0 * (x * x)) * std::exp(-(x * x));
}

// CPML block of solve3D (acoustic_3D_xPU.jl:207-230) / solve2D
// (acoustic_2D_xPU.jl:166-185), packed per axis like awc_problem_coeffs.
int oracle_problem_coeffs(const awc_problem* p, double rcoef, double f0, double vel_max,
                          double* coeffs) {
  const int64_t h = p->halo;
  const double alpha_max = M_PI * f0, npower = 2.0, K_max = 1.0;
  const double d[3] = {p->dx, p->dy, p->dz};
  for (int ax = 0; ax < p->ndim; ++ax) {
    double* blk = coeffs + ax * (8 * h + 4);
    double thickness = (double)h * d[ax];
    double d0 = -(npower + 1.0) * vel_max * std::log(rcoef) / (2.0 * thickness);
    oracle_calc_Kab_CPML(p->halo, p->dt, npower, d0, alpha_max, K_max, 0, blk, blk + h,
                         blk + 2 * h, blk + 3 * h);
    double* hb = blk + 4 * h;
    oracle_calc_Kab_CPML(p->halo, p->dt, npower, d0, alpha_max, K_max, 1, hb, hb + (h + 1),
                         hb + 2 * (h + 1), hb + 3 * (h + 1));
    if (ax == 1 && p->freetop) {  // free top: a_y_l = a_y_hl = 0, b_K_y_l = b_K_y_hl = 1
      for (int64_t n = 0; n < h; ++n) { blk[n] = 0.0; blk[2 * h + n] = 1.0; }
      for (int64_t n = 0; n < h + 1; ++n) { hb[n] = 0.0; hb[2 * (h + 1) + n] = 1.0; }
    }
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Per-axis CPML arrays of the reference (acoustic_3D_xPU.jl:259-264): for axis
// x, ψ_x_{l,r} is (halo+1, ny, nz) and ξ_x_{l,r} is (halo, ny, nz); for y the
// band extent replaces ny, for z it replaces nz.
struct AxisBand {
  std::vector<double> psi_l, psi_r, xi_l, xi_r;
  const double *a_l, *a_r, *bK_l, *bK_r, *a_hl, *a_hr, *bK_hl, *bK_hr;
};

static void bind_coeffs(AxisBand& b, const double* blk, int64_t h) {
  b.a_l = blk; b.a_r = blk + h; b.bK_l = blk + 2 * h; b.bK_r = blk + 3 * h;
  const double* hb = blk + 4 * h;
  b.a_hl = hb; b.a_hr = hb + (h + 1); b.bK_hl = hb + 2 * (h + 1); b.bK_hr = hb + 3 * (h + 1);
}

// update_ψ_x! (acoustic_3D_xPU.jl:8-19), over (1:halo+1, 1:ny, 1:nz).
static void update_psi_x(AxisBand& b, const double* pcur, const Dims& D, int64_t halo, double _dx) {
  const int64_t H = halo + 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t k = 1; k <= D.nz; ++k)
    for (int64_t j = 1; j <= D.ny; ++j)
      for (int64_t i = 1; i <= H; ++i) {
        int64_t ii = i + D.nx - halo - 2;
        int64_t q = (i - 1) + H * ((j - 1) + D.ny * (k - 1));
        b.psi_l[q] = b.bK_hl[i - 1] * b.psi_l[q] +
                     b.a_hl[i - 1] * (pcur[D.at(i + 1, j, k)] - pcur[D.at(i, j, k)]) * _dx;
        b.psi_r[q] = b.bK_hr[i - 1] * b.psi_r[q] +
                     b.a_hr[i - 1] * (pcur[D.at(ii + 1, j, k)] - pcur[D.at(ii, j, k)]) * _dx;
      }
}

// update_ψ_y! (acoustic_3D_xPU.jl:21-32), over (1:nx, 1:halo+1, 1:nz).
static void update_psi_y(AxisBand& b, const double* pcur, const Dims& D, int64_t halo, double _dy) {
  const int64_t H = halo + 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t k = 1; k <= D.nz; ++k)
    for (int64_t j = 1; j <= H; ++j)
      for (int64_t i = 1; i <= D.nx; ++i) {
        int64_t jj = j + D.ny - halo - 2;
        int64_t q = (i - 1) + D.nx * ((j - 1) + H * (k - 1));
        b.psi_l[q] = b.bK_hl[j - 1] * b.psi_l[q] +
                     b.a_hl[j - 1] * (pcur[D.at(i, j + 1, k)] - pcur[D.at(i, j, k)]) * _dy;
        b.psi_r[q] = b.bK_hr[j - 1] * b.psi_r[q] +
                     b.a_hr[j - 1] * (pcur[D.at(i, jj + 1, k)] - pcur[D.at(i, jj, k)]) * _dy;
      }
}

// update_ψ_z! (acoustic_3D_xPU.jl:34-45), over (1:nx, 1:ny, 1:halo+1).
static void update_psi_z(AxisBand& b, const double* pcur, const Dims& D, int64_t halo, double _dz) {
  const int64_t H = halo + 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t k = 1; k <= H; ++k)
    for (int64_t j = 1; j <= D.ny; ++j)
      for (int64_t i = 1; i <= D.nx; ++i) {
        int64_t kk = k + D.nz - halo - 2;
        int64_t q = (i - 1) + D.nx * ((j - 1) + D.ny * (k - 1));
        b.psi_l[q] = b.bK_hl[k - 1] * b.psi_l[q] +
                     b.a_hl[k - 1] * (pcur[D.at(i, j, k + 1)] - pcur[D.at(i, j, k)]) * _dz;
        b.psi_r[q] = b.bK_hr[k - 1] * b.psi_r[q] +
                     b.a_hr[k - 1] * (pcur[D.at(i, j, kk + 1)] - pcur[D.at(i, j, kk)]) * _dz;
      }
}

// update_p! (acoustic_3D_xPU.jl:47-104; 2D acoustic_2D_xPU.jl:33-75 is the
// same with the z terms absent), over (2:nx-1, 2:ny-1, 2:nz-1).
static void update_p(const double* pold, const double* pcur, double* pnew, const double* fact,
                     AxisBand* B, const Dims& D, int ndim, int64_t halo, const double* _d,
                     const double* _d2) {
  const int64_t H = halo + 1;
  const int64_t klo = ndim == 3 ? 2 : 1, khi = ndim == 3 ? D.nz - 1 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t k = klo; k <= khi; ++k)
    for (int64_t j = 2; j <= D.ny - 1; ++j)
      for (int64_t i = 2; i <= D.nx - 1; ++i) {
        const int64_t c = D.at(i, j, k);
        const double pc = pcur[c];
        double d2p_dx2 = (pcur[D.at(i + 1, j, k)] - 2.0 * pc + pcur[D.at(i - 1, j, k)]) * _d2[0];
        double d2p_dy2 = (pcur[D.at(i, j + 1, k)] - 2.0 * pc + pcur[D.at(i, j - 1, k)]) * _d2[1];
        double d2p_dz2 = 0.0;
        if (ndim == 3)
          d2p_dz2 = (pcur[D.at(i, j, k + 1)] - 2.0 * pc + pcur[D.at(i, j, k - 1)]) * _d2[2];
        double damp = 0.0;
        const double f = fact[c];
        // x boundaries (:60-72)
        {
          AxisBand& b = B[0];
          if (i <= halo + 1) {
            int64_t q = (i - 1) + H * ((j - 1) + D.ny * (k - 1));
            int64_t x = (i - 2) + halo * ((j - 1) + D.ny * (k - 1));
            double dpsi = (b.psi_l[q] - b.psi_l[q - 1]) * _d[0];
            b.xi_l[x] = b.bK_l[i - 2] * b.xi_l[x] + b.a_l[i - 2] * (d2p_dx2 + dpsi);
            damp += f * (dpsi + b.xi_l[x]);
          } else if (i >= D.nx - halo) {
            int64_t ii = i - (D.nx - halo) + 2;
            int64_t q = (ii - 1) + H * ((j - 1) + D.ny * (k - 1));
            int64_t x = (ii - 2) + halo * ((j - 1) + D.ny * (k - 1));
            double dpsi = (b.psi_r[q] - b.psi_r[q - 1]) * _d[0];
            b.xi_r[x] = b.bK_r[ii - 2] * b.xi_r[x] + b.a_r[ii - 2] * (d2p_dx2 + dpsi);
            damp += f * (dpsi + b.xi_r[x]);
          }
        }
        // y boundaries (:73-85)
        {
          AxisBand& b = B[1];
          if (j <= halo + 1) {
            int64_t q = (i - 1) + D.nx * ((j - 1) + H * (k - 1));
            int64_t x = (i - 1) + D.nx * ((j - 2) + halo * (k - 1));
            double dpsi = (b.psi_l[q] - b.psi_l[q - D.nx]) * _d[1];
            b.xi_l[x] = b.bK_l[j - 2] * b.xi_l[x] + b.a_l[j - 2] * (d2p_dy2 + dpsi);
            damp += f * (dpsi + b.xi_l[x]);
          } else if (j >= D.ny - halo) {
            int64_t jj = j - (D.ny - halo) + 2;
            int64_t q = (i - 1) + D.nx * ((jj - 1) + H * (k - 1));
            int64_t x = (i - 1) + D.nx * ((jj - 2) + halo * (k - 1));
            double dpsi = (b.psi_r[q] - b.psi_r[q - D.nx]) * _d[1];
            b.xi_r[x] = b.bK_r[jj - 2] * b.xi_r[x] + b.a_r[jj - 2] * (d2p_dy2 + dpsi);
            damp += f * (dpsi + b.xi_r[x]);
          }
        }
        // z boundaries (:86-98)
        if (ndim == 3) {
          AxisBand& b = B[2];
          const int64_t pl = D.nx * D.ny;
          if (k <= halo + 1) {
            int64_t q = (i - 1) + D.nx * ((j - 1) + D.ny * (k - 1));
            int64_t x = (i - 1) + D.nx * ((j - 1) + D.ny * (k - 2));
            double dpsi = (b.psi_l[q] - b.psi_l[q - pl]) * _d[2];
            b.xi_l[x] = b.bK_l[k - 2] * b.xi_l[x] + b.a_l[k - 2] * (d2p_dz2 + dpsi);
            damp += f * (dpsi + b.xi_l[x]);
          } else if (k >= D.nz - halo) {
            int64_t kk = k - (D.nz - halo) + 2;
            int64_t q = (i - 1) + D.nx * ((j - 1) + D.ny * (kk - 1));
            int64_t x = (i - 1) + D.nx * ((j - 1) + D.ny * (kk - 2));
            double dpsi = (b.psi_r[q] - b.psi_r[q - pl]) * _d[2];
            b.xi_r[x] = b.bK_r[kk - 2] * b.xi_r[x] + b.a_r[kk - 2] * (d2p_dz2 + dpsi);
            damp += f * (dpsi + b.xi_r[x]);
          }
        }
        // update pressure (:101)
        double lap = ndim == 3 ? (d2p_dx2 + d2p_dy2 + d2p_dz2) : (d2p_dx2 + d2p_dy2);
        pnew[c] = 2.0 * pc - pold[c] + f * lap + damp;
      }
}

// update_ψ! of the serial solvers (src/shared/acoustic_2D.jl:7-34 and the 3D
// twin) on caller-owned arrays, for the known-answer tests. Arrays use the
// reference shapes; pass nz = 1 and NULL z arrays in 2D.
int oracle_update_psi(int32_t ndim, int64_t nx, int64_t ny, int64_t nz, int32_t halo,
                      const double* pcur, const double* _d, double* const* psi,
                      const double* const* coef) {
  // psi = {ψx_l, ψx_r, ψy_l, ψy_r, ψz_l, ψz_r};
  // coef = {a_xhl, a_xhr, bK_xhl, bK_xhr, a_yhl, ..., bK_zhr} (4 per axis).
  Dims D{nx, ny, ndim == 3 ? nz : 1};
  for (int ax = 0; ax < ndim; ++ax) {
    AxisBand b;
    int64_t n = (int64_t)(halo + 1) * (ax == 0 ? D.ny * D.nz : ax == 1 ? D.nx * D.nz : D.nx * D.ny);
    b.psi_l.assign(psi[2 * ax], psi[2 * ax] + n);
    b.psi_r.assign(psi[2 * ax + 1], psi[2 * ax + 1] + n);
    b.a_hl = coef[4 * ax]; b.a_hr = coef[4 * ax + 1];
    b.bK_hl = coef[4 * ax + 2]; b.bK_hr = coef[4 * ax + 3];
    if (ax == 0) update_psi_x(b, pcur, D, halo, _d[0]);
    if (ax == 1) update_psi_y(b, pcur, D, halo, _d[1]);
    if (ax == 2) update_psi_z(b, pcur, D, halo, _d[2]);
    std::memcpy(psi[2 * ax], b.psi_l.data(), n * sizeof(double));
    std::memcpy(psi[2 * ax + 1], b.psi_r.data(), n * sizeof(double));
  }
  return 0;
}

// The forward solve: arrays of forward! / the time loop
// (acoustic_3D_xPU.jl:124-167, 255-264, 392-409, 541-544). Same argument
// meaning as awc_forward. nthreads <= 0 uses the OpenMP default.
// `steps` < 0 runs p->nt steps; otherwise only the first `steps` (for timing
// a bounded sample); traces rows beyond are left zero.
int oracle_forward(const awc_problem* p, const double* vel, const double* coeffs,
                   const int64_t* possrcs, const double* dt2srctf, const int64_t* posrecs,
                   double* traces, double* pfinal, int32_t nthreads, int64_t steps) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  const int ndim = p->ndim;
  Dims D{p->nx, p->ny, ndim == 3 ? p->nz : 1};
  const int64_t h = p->halo, H = h + 1;
  const int64_t N = D.nx * D.ny * D.nz;
  const double dt = p->dt;
  const double dd[3] = {p->dx, p->dy, p->dz};
  double _d[3], _d2[3];
  for (int a = 0; a < 3; ++a) { _d[a] = 1.0 / dd[a]; _d2[a] = 1.0 / (dd[a] * dd[a]); }

  // fact = (dt^2) .* (vel .^ 2) (acoustic_3D_xPU.jl:242)
  std::vector<double> fact(N);
  const double dt2 = dt * dt;
  for (int64_t c = 0; c < N; ++c) fact[c] = dt2 * (vel[c] * vel[c]);

  std::vector<double> b0(N, 0.0), b1(N, 0.0), b2(N, 0.0);
  double *pold = b0.data(), *pcur = b1.data(), *pnew = b2.data();

  AxisBand B[3];
  const int64_t cross[3] = {D.ny * D.nz, D.nx * D.nz, D.nx * D.ny};
  for (int a = 0; a < ndim; ++a) {
    B[a].psi_l.assign(H * cross[a], 0.0);
    B[a].psi_r.assign(H * cross[a], 0.0);
    B[a].xi_l.assign(h * cross[a], 0.0);
    B[a].xi_r.assign(h * cross[a], 0.0);
    bind_coeffs(B[a], coeffs + a * (8 * h + 4), h);
  }
  // Unused y/z slots in 2D keep empty arrays; update_p never touches them.
  const int64_t nsrc = p->nsrc, nrec = p->nrec, nt = p->nt;
  std::memset(traces, 0, sizeof(double) * nt * nrec);
  const int64_t nrun = steps < 0 || steps > nt ? nt : steps;

  const double t_loop0 = wall_seconds();
  for (int64_t it = 1; it <= nrun; ++it) {
    update_psi_x(B[0], pcur, D, h, _d[0]);
    update_psi_y(B[1], pcur, D, h, _d[1]);
    if (ndim == 3) update_psi_z(B[2], pcur, D, h, _d[2]);
    update_p(pold, pcur, pnew, fact.data(), B, D, ndim, h, _d, _d2);
    // inject_sources! (:106-113): pnew[src] += dt2srctf[it, s]
    for (int64_t s = 0; s < nsrc; ++s) {
      int64_t i = possrcs[s], j = possrcs[s + nsrc], k = ndim == 3 ? possrcs[s + 2 * nsrc] : 1;
      pnew[D.at(i, j, k)] += dt2srctf[(it - 1) + nt * s];
    }
    // record_receivers! (:115-122): traces[it, r] = pnew[rec]
    for (int64_t r = 0; r < nrec; ++r) {
      int64_t i = posrecs[r], j = posrecs[r + nrec], k = ndim == 3 ? posrecs[r + 2 * nrec] : 1;
      traces[(it - 1) + nt * r] = pnew[D.at(i, j, k)];
    }
    // return pcur, pnew, pold  ->  (pold, pcur, pnew) = (pcur, pnew, pold)  (:166, :397)
    double* t = pold;
    pold = pcur;
    pcur = pnew;
    pnew = t;
  }
  g_loop_seconds = wall_seconds() - t_loop0;
  if (pfinal) std::memcpy(pfinal, pcur, sizeof(double) * N);  // Array(pcur) (:544)
  return 0;
}

// Wall time of the time loop of the last oracle_forward (setup excluded).
double oracle_last_loop_seconds(void) { return g_loop_seconds; }

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
