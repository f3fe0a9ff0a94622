// kg_capi.cu -- the C ABI (include/kg_capi.h): solver handle, device memory,
// geometry set-up, the time-stepper drivers and the diagnostics front end.
//
// Host code here does only set-up that the reference also does once at
// start-up (grid, metric tables, detector and Y_lm tables; MoL/geometry.f90,
// MoL/diagnostic_lib.f90:40-151, tools/FFT_sph.f90:282-336) and the
// orchestration of device launches.  Every time step, RHS evaluation, boundary
// fill, reduction and projection runs in the kernels of kg_stencil.cu,
// kg_boundary.cu and kg_diag.cu.  There is no host fallback: without a usable
// device kg_create fails with KG_ENODEV.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/kg_capi.h"
#include "kg_device.cuh"
#include "kg_internal.h"
#include "kg_diag.h"

using kg::Grid;
using kg::Metric;

const char* kg_noalloc_last_error();  // kg_noalloc.cu

namespace {

enum { T_ALPHA = 0, T_BETA, T_DXBETA, T_SQRTG, T_ASG, T_GRR, T_GRP, T_GPP, T_ASG_GTT, T_ASG_GRR, T_A_GPP, T_AM2,
       T_GTT, T_RSG, T_DXBETA4, T_COUNT };

}  // namespace

struct kg_solver {
  kg_params p;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  Grid g;
  int Nx, Ny, Nz, NI, NJ, NK, PI;
  double dx, dy, dz, dt, t, xmin, xmax, r_max;
  int Nt = 0, save = 1;
  int L = 10;
  size_t bytes = 0;
  // host geometry (2-D, index i + NI*j)
  std::vector<double> x1d, y1d, tables;  // tables: T_COUNT x NJ x NI (unpadded)
  std::vector<double> gdn, gup, gam;     // 16, 16, 9 tables of NI*NJ
  // device memory
  double* dmet = nullptr;                // T_COUNT x NJ x PI
  double2* U = nullptr;                  // u (5 variables)
  double2* S = nullptr;                  // u_stage (6 slots; slot 4/5 alternate for Pi)
  double2* T = nullptr;                  // u_stage_2 (6 slots)
  double2* RK = nullptr;                 // RK stage buffers R1, R2 and accumulator (15 slots)
  double2* UP = nullptr;                 // u_p for the boundary hook
  double2* HV = nullptr;                 // rhs hook input / output (10 slots)
  double2* stage_buf = nullptr;          // Fortran-layout staging buffer
  size_t stage_bytes = 0;
  int stage_planes = 0;
  double* rho = nullptr;
  double* partials = nullptr;            // mass partial sums + result
  int s_cur = 4, t_cur = 4;              // slot holding the current Pi stage value
  int variant = 3;                       // 0: per-point, 1: 2.5-D marching, 2, 3: TMA-pipelined marching
                                         // (3: PIRK stage 1 fused in one kernel; 2: two launches)
  int tile_rows = 8;                     // theta rows of the TMA tiles of the RK4 stages (8 or 4)
  int* derr = nullptr;                   // device flag: a bounded wait in a kernel ran out
  // CUDA graphs of two consecutive steps per stepper and Pi-slot state
  int use_graphs = 1;
  struct GraphEntry { cudaGraphExec_t exec = nullptr; int gen = -1; long long launches = 0; };
  GraphEntry graphs[6][4];               // [stepper (pirk2, pirk3, rk3, rk4, mixed rk4, configured rk4)][slot]
  // method: 0 = the reference's second-order scheme, 1 = configured fourth-order (kg_config.cu)
  int scheme = 0;
  double ko_eps = 0.02;
  // mixed precision (RK4): FP32 stage states R1, R2 and increment sum, 5 slots each
  int precision = 0;                     // 0: FP64, 1: FP32 RHS with FP64 state update
  float2* MX = nullptr;
  unsigned char* mx_gdesc = nullptr;     // FP32 ghost-fill descriptors of R1, R2 (device)
  int graph_gen = 0;
  // detectors and projection
  int n_det = 5;
  std::vector<double> r_det;
  std::vector<int> index_det;
  int* d_int = nullptr;                  // active[n_det], i_r[n_det], i_th[Ny], th_flag[Ny], i_ph[Nz]
  double* d_dbl = nullptr;               // w_r, w_th, w_ph, sint, normP, cosm, sinm
  double2* shells = nullptr;             // n_det x 4 x Ny x Nz
  double2* alm = nullptr;                // (L+1) x (2L+1) x n_det
  double* flux = nullptr;                // 3 x n_det
  kg::ShellInterp si;
  const double *normP = nullptr, *cosm = nullptr, *sinm = nullptr, *sint = nullptr;
  std::vector<int> active;
  // all-shell Y_lm projection (allocated on first use, per L)
  int ylmL = -1;
  double* ylm_tab = nullptr;            // normP, cosm, sinm for ylmL
  unsigned char* ylm_buf = nullptr;     // Ahi, Alo, Bhi, Blo, C, F, alm
  size_t ylm_bytes = 0;
  int ylm_b_ready = 0;
  // spherical-Bessel radial basis (per L, Nk) and transform output
  int radL = -1, radNk = -1;
  std::vector<double> rad_k, rad_basis;  // k[l*Nk+n], basis[(l*Nk+n)*Nx+i]
  double* rad_jr = nullptr;              // device: j_basis * r^2, [(l*Nx+i)*Nk+n]
  double2* rad_ft = nullptr;             // device: ft(Nk, 0:L, -L:L)
  // instrumentation
  long long launches = 0;
  int prof_on = 0;
  struct Rec { int kind; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
};

#define KG_CK(call)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
      return KG_ECUDA;                                                                \
    }                                                                                 \
  } while (0)

namespace {

int set_err(kg_solver* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

// Solver buffers come from one stream-ordered memory pool per device: a
// serving loop creates and destroys solves continuously, and cudaMalloc /
// cudaFree would synchronise the whole device at every creation and
// retirement; pool allocations and frees are ordered on the solver's stream
// and freed blocks are reused.  Up to POOL_KEEP bytes of freed blocks stay
// reserved for reuse; an allocation that finds the device full gives every
// cached block back and retries once.
constexpr uint64_t POOL_KEEP = 32ull << 30;
constexpr int POOL_DEVICES = 64;

cudaMemPool_t solver_pool(int dev) {
  static std::mutex mu;
  static cudaMemPool_t pools[POOL_DEVICES] = {};
  if (dev < 0 || dev >= POOL_DEVICES) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps pr;
    memset(&pr, 0, sizeof(pr));
    pr.allocType = cudaMemAllocationTypePinned;
    pr.handleTypes = cudaMemHandleTypeNone;
    pr.location.type = cudaMemLocationTypeDevice;
    pr.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &pr) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = POOL_KEEP;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = pool;
  }
  return pools[dev];
}

int dalloc(kg_solver* h, void** p, size_t n) {
  *p = nullptr;
  cudaMemPool_t pool = solver_pool(h->device);
  if (!pool) {
    h->err = "no device memory pool";
    return KG_ECUDA;
  }
  cudaError_t e = cudaMallocFromPoolAsync(p, n, pool, h->stream);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    cudaDeviceSynchronize();  // pending frees complete, then the cache is released
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(p, n, pool, h->stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    h->err = std::string("device allocation of ") + std::to_string(n) + " bytes: " + cudaGetErrorString(e);
    *p = nullptr;
    return KG_ENOMEM;
  }
  if (reinterpret_cast<uintptr_t>(*p) & 255u) {  // rows and TMA boxes assume 256-byte aligned bases
    cudaFreeAsync(*p, h->stream);
    *p = nullptr;
    h->err = "device allocation not 256-byte aligned";
    return KG_ECUDA;
  }
  h->bytes += n;
  cudaMemsetAsync(*p, 0, n, h->stream);
  return KG_OK;
}

// returns a dalloc block to the pool, ordered after the solver's queued work
void dfree(kg_solver* h, void* p) {
  if (p) cudaFreeAsync(p, h->stream);
}

size_t field_bytes(const kg_solver* h) { return (size_t)h->g.fs * sizeof(double2); }

double2* fld(double2* base, const Grid& g, int v) { return base + (long long)v * g.fs; }

// kernel kinds reported by kg_profile_read: the 13 stage kinds, then these
enum { PK_GHOST = 13, PK_FACE, PK_RHS, PK_CONVERT, PK_DENSITY, PK_MASS, PK_SHELL, PK_FLUX, PK_PROJECT,
       PK_YLM_PREP, PK_YLM_GEMM, PK_YLM_FP64, PK_RADIAL, PK_MX1, PK_MX2, PK_MX3, PK_MX4, PK_GHOST_F32, PK_PROLONG,
       PK_RESTRICT, PK_S1_FUSED, PK_COUNT };
const char* const kPkNames[PK_COUNT] = {
    "stage_pirk_s1_psi", "stage_pirk_s1_pi", "stage_pirk2_s2", "stage_pirk3_s2_psi", "stage_pirk3_s2_pi",
    "stage_pirk3_s3", "stage_rk3_1", "stage_rk3_2", "stage_rk3_3", "stage_rk4_1", "stage_rk4_2", "stage_rk4_3",
    "stage_rk4_4", "ghost_fill", "boundary_face", "rhs", "layout_convert", "density", "mass_reduce",
    "shell_interp", "flux_reduce", "ylm_project", "ylm_all_prepare", "ylm_all_gemm_bf16x3", "ylm_all_fp64", "radial_ft", "mixed_rk4_1",
    "mixed_rk4_2", "mixed_rk4_3", "mixed_rk4_4", "ghost_fill_f32", "bo_prolong", "bo_restrict", "stage_pirk_s1_fused"};

cudaEvent_t take_event(kg_solver* h) {
  if (!h->pool.empty()) {
    cudaEvent_t e = h->pool.back();
    h->pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

struct Prof {
  kg_solver* h;
  int kind, n;
  cudaEvent_t a = nullptr;
  Prof(kg_solver* h_, int kind_, int n_) : h(h_), kind(kind_), n(n_) {
    if (h->prof_on) {
      a = take_event(h);
      cudaEventRecord(a, h->stream);
    }
  }
  ~Prof() {
    h->launches += n;
    if (a) {
      cudaEvent_t b = take_event(h);
      cudaEventRecord(b, h->stream);
      h->recs.push_back({kind, a, b});
    }
  }
};

// ---- geometry (MoL/mesh_refinement_lib.f90:100-147, MoL/geometry.f90:92-406) ----
void build_geometry(kg_solver* h) {
  const int NI = h->NI, NJ = h->NJ, g = h->p.g_pts;
  const double pi = std::acos(-1.0);
  const double dxr = (h->p.xmax - h->p.xmin) / 1.0;
  h->xmin = h->p.xmin + 0.0 * dxr;
  h->xmax = h->p.xmin + 1.0 * dxr;
  h->dx = (h->xmax - h->xmin) / (double)h->Nx;
  h->dy = pi / (double)(h->Ny - 1);
  h->dz = 2.0 * pi / (double)(h->Nz - 1);
  h->x1d.resize(NI);
  h->y1d.resize(NJ);
  for (int i = -g; i <= h->Nx + g; ++i) h->x1d[i + g] = h->xmin + (double)(i + g) * h->dx;
  for (int j = -g; j <= h->Ny + g; ++j) h->y1d[j + g] = -h->dy / 2.0 + (double)j * h->dy;
  h->r_max = h->x1d[NI - 1];
  const double dxx = h->x1d[1] - h->x1d[0];
  double c1 = dxx, c2 = std::exp(h->p.xmin) * h->dy, c3 = std::exp(h->p.xmin) * std::sin(h->dy / 2.0) * h->dz;
  double mn = c1 < c2 ? c1 : c2;
  mn = mn < c3 ? mn : c3;
  h->dt = h->p.CFL * mn;
  if (h->p.dt_override > 0.0) h->dt = h->p.dt_override;
  h->Nt = (int)((h->p.tmax - h->p.tmin) / h->dt);
  if (h->Nt % 2 != 0) h->Nt += 1;
  h->t = h->p.tmin;
  h->save = (int)(h->p.tmin + std::ceil((h->p.save_ > 0 ? h->p.save_ : h->dt) / h->dt));
  if (h->save < 1) h->save = 1;

  const size_t n2 = (size_t)NI * NJ;
  h->gdn.assign(16 * n2, 0.0);
  h->gup.assign(16 * n2, 0.0);
  h->gam.assign(9 * n2, 0.0);
  auto GD = [&](int a, int b, size_t q) -> double& { return h->gdn[(a * 4 + b) * n2 + q]; };
  auto GU = [&](int a, int b, size_t q) -> double& { return h->gup[(a * 4 + b) * n2 + q]; };
  const double M = h->p.M_bh, A = h->p.a;
  for (int jj = 0; jj < NJ; ++jj)
    for (int ii = 0; ii < NI; ++ii) {
      const size_t q = ii + (size_t)NI * jj;
      const double x = h->x1d[ii], y = h->y1d[jj];
      if (h->p.metric == KG_KERR_SCHILD) {
        const double cy = std::cos(y), sy = std::sin(y);
        const double c2v = cy * cy, s2 = sy * sy;
        const double rho2 = x * x + (A * A) * c2v;
        GD(0, 0, q) = -1.0 + 2.0 * M * x / rho2;
        GD(0, 1, q) = (2.0 * M * x / rho2);
        GD(0, 2, q) = 0.0;
        GD(0, 3, q) = -(2.0 * A * M * x * s2 / rho2);
        GD(1, 0, q) = GD(0, 1, q);
        GD(1, 1, q) = (1.0 + 2.0 * M * x / rho2);
        GD(1, 2, q) = 0.0;
        GD(1, 3, q) = (-(A * (1.0 + 2.0 * M * x / rho2) * s2));
        GD(2, 2, q) = (x * x + (A * A) * c2v);
        GD(3, 0, q) = GD(0, 3, q);
        GD(3, 1, q) = GD(1, 3, q);
        const double ax = (A * A + x * x);
        GD(3, 3, q) = ((ax * ax) - (A * A) * (-(2.0 * M * x) + A * A + x * x) * s2) * s2 / rho2;
      } else {
        const double sy = std::sin(y);
        GD(0, 0, q) = -(1.0 - 2.0 * M / x);
        GD(0, 1, q) = 2.0 * M / x;
        GD(1, 0, q) = GD(0, 1, q);
        GD(1, 1, q) = 1.0 + 2.0 * M / x;
        GD(2, 2, q) = x * x;
        GD(3, 3, q) = x * x * (sy * sy);
      }
    }
  // boundary_theta_dn: last theta row <- the row before (metric is phi-independent)
  for (int ii = 0; ii < NI; ++ii) {
    const size_t qt = ii + (size_t)NI * (NJ - 1), qs = ii + (size_t)NI * (NJ - 2);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) GD(a, b, qt) = GD(a, b, qs);
    GD(0, 2, qt) = -GD(0, 2, qs);
    GD(1, 2, qt) = -GD(1, 2, qs);
  }
  std::vector<double> sqrtg(n2), alpha(n2), beta(3 * n2), dxbeta(n2);
  for (size_t q = 0; q < n2; ++q) {
    GD(1, 0, q) = GD(0, 1, q); GD(2, 0, q) = GD(0, 2, q); GD(3, 0, q) = GD(0, 3, q);
    GD(2, 1, q) = GD(1, 2, q); GD(3, 1, q) = GD(1, 3, q); GD(3, 2, q) = GD(2, 3, q);
    sqrtg[q] = std::sqrt(GD(2, 2, q) * (GD(1, 1, q) * GD(3, 3, q) - GD(1, 3, q) * GD(1, 3, q)));
  }
  for (size_t q = 0; q < n2; ++q) {
    const double g00 = GD(0, 0, q), g01 = GD(0, 1, q), g03 = GD(0, 3, q), g11 = GD(1, 1, q), g13 = GD(1, 3, q),
                 g22 = GD(2, 2, q), g33 = GD(3, 3, q);
    const double det =
        ((g33 * g11 - g13 * g13) * g00 - g33 * (g01 * g01) + 2.0 * g13 * g03 * g01 - g11 * (g03 * g03)) * g22;
    const double idetg = 1.0 / det;
    GU(0, 0, q) = g22 * (g11 * g33 - g13 * g13) * idetg;
    GU(0, 1, q) = g22 * (g13 * g03 - g01 * g33) * idetg;
    GU(0, 2, q) = 0.0;
    GU(0, 3, q) = g22 * (g13 * g01 - g11 * g03) * idetg;
    GU(1, 1, q) = g22 * (g33 * g00 - g03 * g03) * idetg;
    GU(1, 2, q) = 0.0;
    GU(1, 3, q) = g22 * (-(g13 * g00) + g03 * g01) * idetg;
    GU(2, 2, q) =
        ((g33 * g11 - g13 * g13) * g00 - g33 * (g01 * g01) + 2.0 * g13 * g03 * g01 - g11 * (g03 * g03)) * idetg;
    GU(2, 3, q) = 0.0;
    GU(3, 3, q) = g22 * (g11 * g00 - g01 * g01) * idetg;
  }
  for (int ii = 0; ii < NI; ++ii) {  // boundary_theta_up
    const size_t qt = ii + (size_t)NI * (NJ - 1), qs = ii + (size_t)NI * (NJ - 2);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) GU(a, b, qt) = GU(a, b, qs);
    GU(0, 2, qt) = -GU(0, 2, qs);
    GU(1, 2, qt) = -GU(1, 2, qs);
  }
  for (size_t q = 0; q < n2; ++q) {
    GU(1, 0, q) = GU(0, 1, q); GU(2, 0, q) = GU(0, 2, q); GU(3, 0, q) = GU(0, 3, q);
    GU(2, 1, q) = GU(1, 2, q); GU(3, 1, q) = GU(1, 3, q); GU(3, 2, q) = GU(2, 3, q);
    const double al = std::sqrt(-1.0 / GU(0, 0, q));
    alpha[q] = al;
    const double a2 = al * al;
    beta[q] = a2 * GU(0, 1, q);
    beta[n2 + q] = a2 * GU(0, 2, q);
    beta[2 * n2 + q] = a2 * GU(0, 3, q);
  }
  for (size_t q = 0; q < n2; ++q) {
    const double a2 = alpha[q] * alpha[q];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        h->gam[(a * 3 + b) * n2 + q] = GU(a + 1, b + 1, q) + beta[a * n2 + q] * beta[b * n2 + q] / a2;
  }
  {  // dx_beta = real(dx1(dcmplx(beta(1)))), MoL/geometry.f90:344
    const double res = 0.50 / h->dx;
    for (int jj = 0; jj < NJ; ++jj) {
      const double* F = beta.data() + (size_t)NI * jj;
      double* D = dxbeta.data() + (size_t)NI * jj;
      const int n = NI - 1;
      D[0] = (-(3.0 * F[0]) + 4.0 * F[1] - F[2]) * res;
      for (int o = 1; o <= n - 1; ++o) D[o] = (-F[o - 1] + F[o + 1]) * res;
      D[n] = (3.0 * F[n] - 4.0 * F[n - 1] + F[n - 2]) * res;
    }
  }
  h->tables.assign((size_t)T_COUNT * n2, 0.0);
  auto TB = [&](int t, size_t q) -> double& { return h->tables[(size_t)t * n2 + q]; };
  const double m2 = h->p.m * h->p.m;
  for (size_t q = 0; q < n2; ++q) {
    TB(T_ALPHA, q) = alpha[q];
    TB(T_BETA, q) = beta[q];
    TB(T_DXBETA, q) = dxbeta[q];
    TB(T_SQRTG, q) = sqrtg[q];
    TB(T_GRR, q) = h->gam[0 * n2 + q];
    TB(T_GRP, q) = h->gam[2 * n2 + q];
    TB(T_GTT, q) = h->gam[4 * n2 + q];
    TB(T_GPP, q) = h->gam[8 * n2 + q];
  }
  (void)m2;
}

// derived products kept exactly as the reference groups them
void derive_tables(kg_solver* h) {
  const size_t n2 = (size_t)h->NI * h->NJ;
  auto TB = [&](int t, size_t q) -> double& { return h->tables[(size_t)t * n2 + q]; };
  const double m2 = h->p.m * h->p.m;
  for (size_t q = 0; q < n2; ++q) {
    const double asg = TB(T_ALPHA, q) * TB(T_SQRTG, q);
    TB(T_ASG, q) = asg;
    TB(T_ASG_GTT, q) = asg * TB(T_GTT, q);
    TB(T_ASG_GRR, q) = asg * TB(T_GRR, q);
    TB(T_A_GPP, q) = TB(T_ALPHA, q) * TB(T_GPP, q);
    TB(T_AM2, q) = TB(T_ALPHA, q) * m2;
    TB(T_RSG, q) = 1.0 / TB(T_SQRTG, q);  // correctly rounded reciprocal for the Markstein quotient
  }
  // d_r beta^r by first_derivative_x_4 (tools/finite_differences.f90:124-154), for the configured method
  const int NI = h->NI, NJ = h->NJ, n = NI - 1;
  const double res = 1.0 / (12.0 * h->dx);
  for (int jj = 0; jj < NJ; ++jj) {
    const double* F = h->tables.data() + (size_t)T_BETA * n2 + (size_t)NI * jj;
    double* D = h->tables.data() + (size_t)T_DXBETA4 * n2 + (size_t)NI * jj;
    D[0] = (-25.0 * F[0] + 48.0 * F[1] - 36.0 * F[2] + 16.0 * F[3] - 3.0 * F[4]) * res;
    D[1] = (-3.0 * F[0] - 10.0 * F[1] + 18.0 * F[2] - 6.0 * F[3] + 1.0 * F[4]) * res;
    for (int o = 2; o <= n - 2; ++o) D[o] = (F[o - 2] - 8.0 * F[o - 1] + 8.0 * F[o + 1] - F[o + 2]) * res;
    D[n - 1] = (3.0 * F[n] + 10.0 * F[n - 1] - 18.0 * F[n - 2] + 6.0 * F[n - 3] - 1.0 * F[n - 4]) * res;
    D[n] = (25.0 * F[n] - 48.0 * F[n - 1] + 36.0 * F[n - 2] - 16.0 * F[n - 3] + 3.0 * F[n - 4]) * res;
  }
}

int upload_tables(kg_solver* h) {
  const size_t n2 = (size_t)h->NI * h->NJ;
  derive_tables(h);
  KG_CK(cudaMemcpy2DAsync(h->dmet, sizeof(double) * h->PI, h->tables.data(), sizeof(double) * h->NI,
                          sizeof(double) * h->NI, (size_t)T_COUNT * h->NJ, cudaMemcpyHostToDevice, h->stream));
  (void)n2;
  return KG_OK;
}

Metric metric_of(const kg_solver* h) {
  Metric m;
  const size_t tp = (size_t)h->NJ * h->PI;
  const double* b = h->dmet;
  m.alpha = b + T_ALPHA * tp;
  m.beta = b + T_BETA * tp;
  m.dxbeta = b + T_DXBETA * tp;
  m.sqrtg = b + T_SQRTG * tp;
  m.asg = b + T_ASG * tp;
  m.grr = b + T_GRR * tp;
  m.grp = b + T_GRP * tp;
  m.gpp = b + T_GPP * tp;
  m.asg_gtt = b + T_ASG_GTT * tp;
  m.asg_grr = b + T_ASG_GRR * tp;
  m.a_gpp = b + T_A_GPP * tp;
  m.am2 = b + T_AM2 * tp;
  m.gtt = b + T_GTT * tp;
  return m;
}

// associated Legendre P_l^m with the Condon-Shortley phase (the convention of
// GSL's gsl_sf_legendre_Plm used by tools/FFT_sph.f90:323): upward recurrence
double plm(int l, int m, double x) {
  double pmm = 1.0;
  if (m > 0) {
    const double somx2 = std::sqrt((1.0 - x) * (1.0 + x));
    double fact = 1.0;
    for (int i = 1; i <= m; ++i) {
      pmm *= -fact * somx2;
      fact += 2.0;
    }
  }
  if (l == m) return pmm;
  double pmmp1 = x * (2.0 * m + 1.0) * pmm;
  if (l == m + 1) return pmmp1;
  double pll = 0.0;
  for (int ll = m + 2; ll <= l; ++ll) {
    pll = (x * (2.0 * ll - 1.0) * pmmp1 - (ll + m - 1.0) * pmm) / (double)(ll - m);
    pmm = pmmp1;
    pmmp1 = pll;
  }
  return pll;
}

// norm * Plm of sph_harmonics (tools/FFT_sph.f90:306-324), incl. the pole rule
double norm_plm(int l, int m, double theta) {
  const double pi = std::acos(-1.0);
  const double fact = std::sqrt((2.0 * l + 1.0) / (4.0 * pi));
  double norm = fact;
  if (m > 0)
    for (int i = 1; i <= 2 * m; ++i) norm = norm / std::sqrt((double)(l - m + i));
  const double x = std::cos(theta);
  const double P = (std::fabs(x) > 0.9999) ? (m == 0 ? fact : 0.0) : plm(l, m, x);
  return norm * P;
}

// detectors (MoL/diagnostic_lib.f90:124-134, main/global_numbers.f90:152-164)
// and the domain_to_sph index search (tools/FFT_sph.f90:553-613)
// radii = nullptr: the reference's detector placement
int build_detectors(kg_solver* h, const double* radii = nullptr) {
  const int n = h->n_det, Ny = h->Ny, Nz = h->Nz, L = h->L;
  h->r_det.assign(n, 0.0);
  h->index_det.assign(n, 0);
  h->active.assign(n, 0);
  if (radii) {
    for (int d = 0; d < n; ++d) h->r_det[d] = radii[d];
  } else {
    h->r_det[0] = (1.0 + std::sqrt(1.0 - h->p.a * h->p.a));
    h->r_det[n - 1] = h->p.xmax * 0.99;
    for (int d = 2; d <= n - 1; ++d)
      h->r_det[d - 1] = h->r_det[0] + (h->r_det[n - 1] - h->r_det[0]) / (double)n * (double)(d - 1);
  }
  for (void** p : {(void**)&h->d_int, (void**)&h->d_dbl, (void**)&h->shells, (void**)&h->alm, (void**)&h->flux})
    if (*p) {
      dfree(h, *p);
      *p = nullptr;
    }
  auto rv = [&](int iv) { return h->xmin + (double)(iv - 1) * h->dx; };
  for (int d = 0; d < n; ++d) {
    for (int i = 1; i <= h->Nx - 1; ++i)
      if (rv(i) <= h->r_det[d] && h->r_det[d] <= rv(i + 1)) {
        h->index_det[d] = i;
        break;
      }
    h->active[d] = (rv(1) <= h->r_det[d] && rv(h->Nx) > h->r_det[d] && h->index_det[d] > 0) ? 1 : 0;
  }
  // index search with the reference's arithmetic, per direction
  const int b1l = -2, b1r = h->Nx + 2, b2l = -2, b2r = h->Ny + 2, b3l = 0, b3r = h->Nz;
  auto RD = [&](int i) { return h->x1d[i - b1l]; };
  auto TD = [&](int j) { return h->y1d[j - b2l]; };
  auto PD = [&](int k) { return (double)k * h->dz; };
  const double rmin = RD(b1l), dr = RD(b1l + 1) - RD(b1l);
  const double thetamin = TD(b2l), dth = std::fabs(TD(b2l + 1) - TD(b2l));
  const double phimin = PD(b3l), dph = std::fabs(PD(b3l + 1) - PD(b3l));
  std::vector<int> i_r(n), i_th(Ny), th_flag(Ny), i_ph(Nz);
  std::vector<double> w_r(n), w_th(Ny), w_ph(Nz), sint(Ny);
  for (int d = 0; d < n; ++d) {
    const double rr = rv(h->index_det[d] > 0 ? h->index_det[d] : 1);
    int ir = (int)((rr - rmin) / dr) + b1l;
    if (ir < b1l) ir = b1l;
    if (ir > b1r - 1) ir = b1r - 1;
    while (ir < b1r - 1 && rr >= RD(ir + 1)) ir++;
    while (ir > b1l && rr < RD(ir)) ir--;
    i_r[d] = ir - b1l;
    w_r[d] = (rr - RD(ir)) / dr;
  }
  for (int jv = 1; jv <= Ny; ++jv) {
    const double tt = (double)(jv - 1) * h->dy;
    int it = (int)((tt - thetamin) / dth) + b2l;
    if (it < b2l) it = b2l;
    if (it > b2r - 1) it = b2r - 1;
    while (it < b2r - 1 && tt >= TD(it + 1)) it++;
    while (it > b2l && tt < TD(it)) it--;
    i_th[jv - 1] = it - b2l;
    w_th[jv - 1] = (tt - TD(it)) / dth;
    th_flag[jv - 1] = (tt <= thetamin) ? 1 : (tt >= thetamin + dth * (double)(b2r - b2l)) ? 2 : 0;
    sint[jv - 1] = std::sin(tt);
  }
  for (int kv = 1; kv <= Nz; ++kv) {
    const double pp = (double)(kv - 1) * h->dz;
    int ip = (int)((pp - phimin) / dph) + b3l;
    if (ip < b3l) ip = b3l;
    if (ip > b3r - 1) ip = b3r - 1;
    while (ip < b3r - 1 && pp >= PD(ip + 1)) ip++;
    while (ip > b3l && pp < PD(ip)) ip--;
    i_ph[kv - 1] = ip;
    w_ph[kv - 1] = (pp - PD(ip)) / dph;
  }
  // Y_lm factors: normP[l][m][jv], cos/sin(m phi_kv)
  std::vector<double> normP((size_t)(L + 1) * (L + 1) * Ny, 0.0), cosm((size_t)(L + 1) * Nz), sinm((size_t)(L + 1) * Nz);
  for (int l = 0; l <= L; ++l)
    for (int m = 0; m <= l; ++m)
      for (int jv = 1; jv <= Ny; ++jv) normP[((size_t)l * (L + 1) + m) * Ny + jv - 1] = norm_plm(l, m, (double)(jv - 1) * h->dy);
  for (int m = 0; m <= L; ++m)
    for (int kv = 1; kv <= Nz; ++kv) {
      const double ph = (double)(kv - 1) * h->dz;
      cosm[(size_t)m * Nz + kv - 1] = std::cos(m * ph);
      sinm[(size_t)m * Nz + kv - 1] = std::sin(m * ph);
    }
  // device copies
  const size_t nint = 2 * (size_t)n + 2 * (size_t)Ny + Nz;
  const size_t ndbl = (size_t)n + 2 * (size_t)Ny + Nz + normP.size() + cosm.size() + sinm.size();
  int rc;
  if ((rc = dalloc(h, (void**)&h->d_int, nint * sizeof(int)))) return rc;
  if ((rc = dalloc(h, (void**)&h->d_dbl, ndbl * sizeof(double)))) return rc;
  std::vector<int> hi;
  hi.insert(hi.end(), h->active.begin(), h->active.end());
  hi.insert(hi.end(), i_r.begin(), i_r.end());
  hi.insert(hi.end(), i_th.begin(), i_th.end());
  hi.insert(hi.end(), th_flag.begin(), th_flag.end());
  hi.insert(hi.end(), i_ph.begin(), i_ph.end());
  std::vector<double> hd;
  hd.insert(hd.end(), w_r.begin(), w_r.end());
  hd.insert(hd.end(), w_th.begin(), w_th.end());
  hd.insert(hd.end(), w_ph.begin(), w_ph.end());
  hd.insert(hd.end(), sint.begin(), sint.end());
  hd.insert(hd.end(), normP.begin(), normP.end());
  hd.insert(hd.end(), cosm.begin(), cosm.end());
  hd.insert(hd.end(), sinm.begin(), sinm.end());
  // on the solver's stream, behind dalloc's zero fill of the same buffers (the
  // stream is non-blocking, so a legacy-stream copy could land before that fill)
  KG_CK(cudaMemcpyAsync(h->d_int, hi.data(), hi.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  KG_CK(cudaMemcpyAsync(h->d_dbl, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  const int* ip = h->d_int;
  h->si.active = ip;
  h->si.i_r = ip + n;
  h->si.i_th = ip + 2 * n;
  h->si.th_flag = ip + 2 * n + Ny;
  h->si.i_ph = ip + 2 * n + 2 * Ny;
  const double* dp = h->d_dbl;
  h->si.w_r = dp;
  h->si.w_th = dp + n;
  h->si.w_ph = dp + n + Ny;
  h->sint = dp + n + Ny + Nz;
  h->normP = h->sint + Ny;
  h->cosm = h->normP + normP.size();
  h->sinm = h->cosm + cosm.size();
  if ((rc = dalloc(h, (void**)&h->shells, (size_t)n * 4 * Ny * Nz * sizeof(double2)))) return rc;
  if ((rc = dalloc(h, (void**)&h->alm, (size_t)(L + 1) * (2 * L + 1) * n * sizeof(double2)))) return rc;
  if ((rc = dalloc(h, (void**)&h->flux, (size_t)3 * n * sizeof(double)))) return rc;
  return KG_OK;
}

int ensure(kg_solver* h, double2** buf, int nslots) {
  if (*buf) return KG_OK;
  return dalloc(h, (void**)buf, (size_t)nslots * field_bytes(h));
}

int ensure_staging(kg_solver* h) {
  if (h->stage_buf) return KG_OK;
  const size_t plane_bytes = (size_t)5 * h->NI * h->NJ * sizeof(double2);
  size_t want = (size_t)256 << 20;
  int planes = (int)(want / plane_bytes);
  if (planes < 1) planes = 1;
  if (planes > h->NK) planes = h->NK;
  h->stage_planes = planes;
  h->stage_bytes = (size_t)planes * plane_bytes;
  return dalloc(h, (void**)&h->stage_buf, h->stage_bytes);
}

// pointer to the 5-variable view of state `which`, or the Pi slot adjustments
struct View {
  double2* v[5];
};

int state_view(kg_solver* h, int which, View* out) {
  int rc;
  const Grid& g = h->g;
  switch (which) {
    case 0:
      for (int v = 0; v < 5; ++v) out->v[v] = fld(h->U, g, v);
      return KG_OK;
    case 1:
      if ((rc = ensure(h, &h->S, 6))) return rc;
      for (int v = 0; v < 4; ++v) out->v[v] = fld(h->S, g, v);
      out->v[4] = fld(h->S, g, h->s_cur);
      return KG_OK;
    case 2:
      if ((rc = ensure(h, &h->T, 6))) return rc;
      for (int v = 0; v < 4; ++v) out->v[v] = fld(h->T, g, v);
      out->v[4] = fld(h->T, g, h->t_cur);
      return KG_OK;
    case 3:
      if ((rc = ensure(h, &h->UP, 5))) return rc;
      for (int v = 0; v < 5; ++v) out->v[v] = fld(h->UP, g, v);
      return KG_OK;
    default:
      return set_err(h, KG_EINVAL, "state index must be 0..3");
  }
}

// copy a Fortran-layout state (host or device memory) into 5 device planes
int load_view(kg_solver* h, const View& V, const double* src, cudaMemcpyKind kind) {
  int rc;
  if ((rc = ensure_staging(h))) return rc;
  const Grid& g = h->g;
  const size_t plane_elems = (size_t)5 * h->NI * h->NJ;
  // contiguous 5-variable device view? (slots 0..4 of one buffer)
  for (int k0 = 0; k0 < h->NK; k0 += h->stage_planes) {
    const int k1 = (k0 + h->stage_planes < h->NK) ? k0 + h->stage_planes : h->NK;
    const size_t n = (size_t)(k1 - k0) * plane_elems;
    KG_CK(cudaMemcpyAsync(h->stage_buf, (const double2*)src + (size_t)k0 * plane_elems, n * sizeof(double2), kind,
                          h->stream));
    // convert into a temporary contiguous 5-slot view if the slots are not contiguous
    bool contiguous = true;
    for (int v = 1; v < 5; ++v) contiguous = contiguous && (V.v[v] == V.v[0] + (long long)v * g.fs);
    if (contiguous) {
      { Prof pf(h, PK_CONVERT, 1); kg::launch_aos_to_soa(g, h->stage_buf, V.v[0], k0, k1, h->stream); }
    } else {
      // slot 4 lives elsewhere: convert variables 0..3 in place and variable 4 via its own base
      // (aos_to_soa writes v*fs offsets from the base, so run it on a base that puts
      // variable 4 at V.v[4]: write 0..4 at V.v[0], then move slot 4)
      { Prof pf(h, PK_CONVERT, 1); kg::launch_aos_to_soa(g, h->stage_buf, V.v[0], k0, k1, h->stream); }
      KG_CK(cudaMemcpyAsync(V.v[4] + (long long)k0 * g.plane, V.v[0] + 4 * g.fs + (long long)k0 * g.plane,
                            (size_t)(k1 - k0) * g.plane * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    }
    KG_CK(cudaGetLastError());
  }
  return KG_OK;
}

int store_view(kg_solver* h, const View& V, double* dst, cudaMemcpyKind kind) {
  int rc;
  if ((rc = ensure_staging(h))) return rc;
  const Grid& g = h->g;
  const size_t plane_elems = (size_t)5 * h->NI * h->NJ;
  bool contiguous = true;
  for (int v = 1; v < 5; ++v) contiguous = contiguous && (V.v[v] == V.v[0] + (long long)v * g.fs);
  for (int k0 = 0; k0 < h->NK; k0 += h->stage_planes) {
    const int k1 = (k0 + h->stage_planes < h->NK) ? k0 + h->stage_planes : h->NK;
    const size_t n = (size_t)(k1 - k0) * plane_elems;
    if (!contiguous) {
      // gather slot 4 next to 0..3 (slot 4 of the same buffer is free scratch for S/T)
      KG_CK(cudaMemcpyAsync(V.v[0] + 4 * g.fs + (long long)k0 * g.plane, V.v[4] + (long long)k0 * g.plane,
                            (size_t)(k1 - k0) * g.plane * sizeof(double2), cudaMemcpyDeviceToDevice, h->stream));
    }
    { Prof pf(h, PK_CONVERT, 1); kg::launch_soa_to_aos(g, V.v[0], h->stage_buf, k0, k1, h->stream); }
    KG_CK(cudaGetLastError());
    KG_CK(cudaMemcpyAsync((double2*)dst + (size_t)k0 * plane_elems, h->stage_buf, n * sizeof(double2), kind,
                          h->stream));
  }
  return KG_OK;
}

void run_stage(kg_solver* h, int kind, const kg::StageLaunch& L) {
  Prof pf(h, kind, 1);
  const double* rsg = h->dmet + (size_t)T_RSG * h->NJ * h->PI;
  if (h->variant >= 2 && kg::launch_stage_tma(kind, L, rsg, h->derr, h->stream, h->tile_rows) == 0) return;
  if (h->variant >= 1)
    kg::launch_stage_march(kind, L, rsg, h->stream);
  else
    kg::launch_stage(kind, L, h->stream);
}

// KG_ETIMEOUT if a kernel reported a bounded wait that ran out (flag is sticky)
int check_device_flag(kg_solver* h) {
  int f = 0;
  KG_CK(cudaMemcpyAsync(&f, h->derr, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  if (f) {
    h->err = "a device wait ran out (TMA stage kernel); results of the affected launch are invalid";
    return KG_ETIMEOUT;
  }
  return KG_OK;
}
void run_ghost(kg_solver* h, double2* u, const double2* up, int inflow) {
  Prof pf(h, PK_GHOST, 2);
  kg::launch_ghost_fill(h->g, u, up, inflow, h->stream);
}

kg::StageLaunch base_launch(kg_solver* h) {
  kg::StageLaunch L;
  memset(&L, 0, sizeof(L));
  L.g = h->g;
  L.m = metric_of(h);
  L.metric_kind = h->p.metric == KG_SCHW_EF ? kg::MK_SCHW : kg::MK_KS;
  return L;
}

void set_in(kg::StageLaunch& L, const Grid& g, double2* b0, double2* b4) {
  for (int v = 0; v < 4; ++v) L.in[v] = fld(b0, g, v);
  L.in[4] = b4;
}

// PIRK stage 1 (pirk2 :278-289, pirk3 :341-352): u_stage(1:4) from u, then
// u_stage(5) from u_stage(1:4) and the previous step's Pi in Sold; one fused
// kernel in form 3, two launches otherwise
void run_pirk_s1(kg_solver* h, double2* Sold, double2* Snew) {
  const Grid& g = h->g;
  if (h->variant == 3) {
    Prof pf(h, PK_S1_FUSED, 1);
    const double* rsg = h->dmet + (size_t)T_RSG * h->NJ * h->PI;
    const int mk = h->p.metric == KG_SCHW_EF ? kg::MK_SCHW : kg::MK_KS;
    if (kg::launch_pirk_s1_fused(g, metric_of(h), mk, h->U, Sold, h->S, Snew, rsg, h->derr, h->stream) == 0)
      return;
    pf.n = 0;
  }
  kg::StageLaunch L = base_launch(h);
  set_in(L, g, h->U, fld(h->U, g, 4));
  L.base = h->U;
  L.out = h->S;
  run_stage(h, kg::ST_P2_S1A, L);
  set_in(L, g, h->S, Sold);
  L.out4 = Snew;
  run_stage(h, kg::ST_P2_S1B, L);
}

}  // namespace

// =============================================================================
extern "C" {

int kg_create(const kg_params* p, int device, kg_solver** out) {
  if (!p || !out) return KG_EINVAL;
  *out = nullptr;
  if (p->g_pts != 2 || p->Nx < 4 || p->Ny < 5 || p->Nz < 5 || !(p->xmax > p->xmin) || !(p->CFL > 0.0) ||
      (p->metric != KG_KERR_SCHILD && p->metric != KG_SCHW_EF) ||
      (p->bc_rmax != KG_OUTFLOW && p->bc_rmax != KG_INFLOW) || p->l_max < 0 || p->l_max > 128)
    return KG_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return KG_ENODEV;
  }
  if (device >= 0) {
    if (device >= ndev || cudaSetDevice(device) != cudaSuccess) return KG_ENODEV;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major < 10)
    return KG_ENODEV;
  kg_solver* h = new kg_solver();
  h->p = *p;
  h->device = dev;
  h->Nx = p->Nx; h->Ny = p->Ny; h->Nz = p->Nz;
  h->NI = p->Nx + 5; h->NJ = p->Ny + 5; h->NK = p->Nz + 1;
  h->PI = (h->NI + 7) / 8 * 8;
  h->n_det = p->n_det < 2 ? 2 : p->n_det;
  h->L = p->l_max;
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return KG_ECUDA;
  }
  build_geometry(h);
  Grid& g = h->g;
  g.NI = h->NI; g.NJ = h->NJ; g.NK = h->NK; g.PI = h->PI;
  g.plane = (long long)h->NJ * h->PI;
  g.fs = (long long)h->NK * g.plane;
  g.Nz = h->Nz; g.dis = h->Nz / 2; g.Nzm1 = h->Nz - 1;
  g.rdx = 0.50 / h->dx; g.rdy = 0.50 / h->dy; g.rdz = 0.50 / h->dz;
  g.dt = h->dt;
  int rc = KG_OK;
  if ((rc = dalloc(h, (void**)&h->dmet, (size_t)T_COUNT * h->NJ * h->PI * sizeof(double))) ||
      (rc = upload_tables(h)) || (rc = dalloc(h, (void**)&h->U, 5 * field_bytes(h))) ||
      (rc = dalloc(h, (void**)&h->partials, (size_t)(kg::mass_blocks(g) + 1) * sizeof(double))) ||
      (rc = dalloc(h, (void**)&h->derr, 16)) ||
      (rc = build_detectors(h))) {
    kg_destroy(h);
    return rc;
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    kg_destroy(h);
    return KG_ECUDA;
  }
  if (!kg::tma_available(h->g, h->U)) h->variant = 1;  // tensor maps unavailable: register-prefetch form
  *out = h;
  return KG_OK;
}

int kg_destroy(kg_solver* h) {
  if (!h) return KG_EINVAL;
  if (h->stream) cudaStreamSynchronize(h->stream);
  void* bufs[] = {h->dmet, h->U, h->S, h->T, h->RK, h->UP, h->HV, h->stage_buf, h->rho, h->partials,
                  h->d_int, h->d_dbl, h->shells, h->alm, h->flux, h->derr, h->ylm_tab, h->ylm_buf,
                  h->rad_jr, h->rad_ft, h->MX, h->mx_gdesc};
  for (void* b : bufs) dfree(h, b);
  for (auto& row : h->graphs)
    for (auto& e : row)
      if (e.exec) cudaGraphExecDestroy(e.exec);
  for (auto& r : h->recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : h->pool) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return KG_OK;
}

const char* kg_last_error(const kg_solver* h) { return h ? h->err.c_str() : kg_noalloc_last_error(); }

int kg_get_scalars(const kg_solver* h, double* o) {
  if (!h || !o) return KG_EINVAL;
  o[0] = h->dx; o[1] = h->dy; o[2] = h->dz; o[3] = h->dt; o[4] = h->t;
  o[5] = h->xmin; o[6] = h->xmax; o[7] = (double)h->Nt; o[8] = h->r_max;
  return KG_OK;
}

int kg_set_time(kg_solver* h, double t) {
  if (!h) return KG_EINVAL;
  h->t = t;
  return KG_OK;
}

int kg_set_dt(kg_solver* h, double dt) {
  if (!h || !(dt > 0.0)) return KG_EINVAL;
  h->dt = dt;
  h->g.dt = dt;
  h->graph_gen++;
  return KG_OK;
}

void* kg_get_stream(const kg_solver* h) { return h ? (void*)h->stream : nullptr; }
size_t kg_device_bytes(const kg_solver* h) { return h ? h->bytes : 0; }

int kg_synchronize(kg_solver* h) {
  if (!h) return KG_EINVAL;
  KG_CK(cudaStreamSynchronize(h->stream));
  return check_device_flag(h);
}

int kg_set_state(kg_solver* h, int which, const double* host_u) {
  if (!h || !host_u) return KG_EINVAL;
  View V;
  int rc;
  if ((rc = state_view(h, which, &V))) return rc;
  if ((rc = load_view(h, V, host_u, cudaMemcpyHostToDevice))) return rc;
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

int kg_get_state(kg_solver* h, int which, double* host_u) {
  if (!h || !host_u) return KG_EINVAL;
  View V;
  int rc;
  if ((rc = state_view(h, which, &V))) return rc;
  if ((rc = store_view(h, V, host_u, cudaMemcpyDeviceToHost))) return rc;
  KG_CK(cudaStreamSynchronize(h->stream));
  return check_device_flag(h);
}

int kg_set_state_device(kg_solver* h, int which, const double* dev_u) {
  if (!h || !dev_u) return KG_EINVAL;
  View V;
  int rc;
  if ((rc = state_view(h, which, &V))) return rc;
  return load_view(h, V, dev_u, cudaMemcpyDeviceToDevice);
}

int kg_get_state_device(kg_solver* h, int which, double* dev_u) {
  if (!h || !dev_u) return KG_EINVAL;
  View V;
  int rc;
  if ((rc = state_view(h, which, &V))) return rc;
  return store_view(h, V, dev_u, cudaMemcpyDeviceToDevice);
}

namespace {
int step_pirk2(kg_solver* h, int nsteps) {
  int rc;
  if ((rc = ensure(h, &h->S, 6))) return rc;
  const Grid& g = h->g;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  for (int s = 0; s < nsteps; ++s) {
    double2* Sold = fld(h->S, g, h->s_cur);
    double2* Snew = fld(h->S, g, 9 - h->s_cur);
    run_pirk_s1(h, Sold, Snew);
    kg::StageLaunch L = base_launch(h);
    L.base = h->U;
    set_in(L, g, h->S, Snew);
    L.out = h->U;
    L.skip_last_i = inflow;
    run_stage(h, kg::ST_P2_S2, L);
    run_ghost(h, h->U, h->U, inflow);
    h->s_cur = 9 - h->s_cur;
    h->t = h->t + h->dt;
  }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

int step_pirk3(kg_solver* h, int nsteps) {
  int rc;
  if ((rc = ensure(h, &h->S, 6)) || (rc = ensure(h, &h->T, 6))) return rc;
  const Grid& g = h->g;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  for (int s = 0; s < nsteps; ++s) {
    double2* Sold = fld(h->S, g, h->s_cur);
    double2* Snew = fld(h->S, g, 9 - h->s_cur);
    double2* Told = fld(h->T, g, h->t_cur);
    double2* Tnew = fld(h->T, g, 9 - h->t_cur);
    run_pirk_s1(h, Sold, Snew);
    kg::StageLaunch L = base_launch(h);
    L.base = h->U;
    set_in(L, g, h->S, Snew);
    L.out = h->T;
    run_stage(h, kg::ST_P3_S2A, L);
    set_in(L, g, h->T, Told);
    L.aux4 = Snew;
    L.out4 = Tnew;
    run_stage(h, kg::ST_P3_S2B, L);
    set_in(L, g, h->T, Tnew);
    L.out = h->U;
    L.skip_last_i = inflow;
    run_stage(h, kg::ST_P3_S3, L);
    run_ghost(h, h->U, h->U, inflow);
    h->s_cur = 9 - h->s_cur;
    h->t_cur = 9 - h->t_cur;
    h->t = h->t + h->dt;
  }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

int step_rk3(kg_solver* h, int nsteps) {
  int rc;
  if ((rc = ensure(h, &h->RK, 15))) return rc;
  const Grid& g = h->g;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  double2* R1 = h->RK;
  double2* R2 = fld(h->RK, g, 5);
  for (int s = 0; s < nsteps; ++s) {
    kg::StageLaunch L = base_launch(h);
    L.base = h->U;
    set_in(L, g, h->U, fld(h->U, g, 4));
    L.out = R1;
    run_stage(h, kg::ST_RK3_1, L);
    run_ghost(h, R1, h->U, inflow);
    set_in(L, g, R1, fld(R1, g, 4));
    L.out = R2;
    run_stage(h, kg::ST_RK3_2, L);
    run_ghost(h, R2, h->U, inflow);
    set_in(L, g, R2, fld(R2, g, 4));
    L.out = h->U;
    L.skip_last_i = inflow;
    run_stage(h, kg::ST_RK3_3, L);
    run_ghost(h, h->U, h->U, inflow);
    h->t = h->t + h->dt;
  }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

int step_rk4(kg_solver* h, int nsteps) {
  int rc;
  if ((rc = ensure(h, &h->RK, 15))) return rc;
  const Grid& g = h->g;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  double2* R1 = h->RK;
  double2* R2 = fld(h->RK, g, 5);
  double2* A = fld(h->RK, g, 10);
  for (int s = 0; s < nsteps; ++s) {
    kg::StageLaunch L = base_launch(h);
    L.base = h->U;
    L.acc = A;
    set_in(L, g, h->U, fld(h->U, g, 4));
    L.out = R1;
    run_stage(h, kg::ST_RK4_1, L);
    run_ghost(h, R1, h->U, inflow);
    set_in(L, g, R1, fld(R1, g, 4));
    L.out = R2;
    run_stage(h, kg::ST_RK4_2, L);
    run_ghost(h, R2, h->U, inflow);
    set_in(L, g, R2, fld(R2, g, 4));
    L.out = R1;
    run_stage(h, kg::ST_RK4_3, L);
    run_ghost(h, R1, h->U, inflow);
    set_in(L, g, R1, fld(R1, g, 4));
    L.out = h->U;
    L.skip_last_i = inflow;
    run_stage(h, kg::ST_RK4_4, L);
    run_ghost(h, h->U, h->U, inflow);
    h->t = h->t + h->dt;
  }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

// FP32 stage buffers and their ghost-fill descriptors
int ensure_mixed(kg_solver* h) {
  if (h->MX) return KG_OK;
  int rc;
  if ((rc = dalloc(h, (void**)&h->MX, (size_t)15 * h->g.fs * sizeof(float2)))) return rc;
  const size_t dsz = kg::ghost_f32_desc_bytes();
  if ((rc = dalloc(h, (void**)&h->mx_gdesc, 2 * dsz))) return rc;
  std::vector<unsigned char> d(2 * dsz);
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  kg::fill_ghost_f32_desc(d.data(), h->g, h->MX, h->U, inflow);
  kg::fill_ghost_f32_desc(d.data() + dsz, h->g, h->MX + 5 * h->g.fs, h->U, inflow);
  KG_CK(cudaMemcpyAsync(h->mx_gdesc, d.data(), d.size(), cudaMemcpyHostToDevice, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

kg::MixedLaunch mixed_launch(kg_solver* h) {
  kg::MixedLaunch L;
  memset(&L, 0, sizeof(L));
  L.g = h->g;
  L.m = metric_of(h);
  L.metric_kind = h->p.metric == KG_SCHW_EF ? kg::MK_SCHW : kg::MK_KS;
  L.base = h->U;
  L.acc = h->MX + 10 * h->g.fs;
  return L;
}

int run_mixed_stage(kg_solver* h, int st, const kg::MixedLaunch& L) {
  static const int kinds[4] = {kg::ST_RK4_1, kg::ST_RK4_2, kg::ST_RK4_3, kg::ST_RK4_4};
  Prof pf(h, PK_MX1 + st, 1);
  const double* rsg = h->dmet + (size_t)T_RSG * h->NJ * h->PI;
  if (kg::launch_stage_mixed(kinds[st], L, rsg, h->derr, h->stream, h->tile_rows))
    return set_err(h, KG_ECUDA, "mixed-precision stage could not be configured (tensor maps)");
  return KG_OK;
}

void run_ghost_f32(kg_solver* h, int which) {
  Prof pf(h, PK_GHOST_F32, 2);
  const Grid& g = h->g;
  kg::launch_ghost_fill_f32(h->mx_gdesc + which * kg::ghost_f32_desc_bytes(), 1, 6LL * g.NK * g.NI,
                            2LL * (g.NJ - 6) * g.NK, 2LL * g.NI * g.NJ, h->stream);
}

// RK4 with the stencil RHS in FP32 and the state update in FP64 (kg_mixed.cu)
int step_rk4_mixed(kg_solver* h, int nsteps) {
  int rc;
  if ((rc = ensure_mixed(h))) return rc;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  float2* R1 = h->MX;
  float2* R2 = h->MX + 5 * h->g.fs;
  for (int s = 0; s < nsteps; ++s) {
    kg::MixedLaunch L = mixed_launch(h);
    L.out_f = R1;
    if ((rc = run_mixed_stage(h, 0, L))) return rc;
    run_ghost_f32(h, 0);
    L.in_f = R1;
    L.out_f = R2;
    if ((rc = run_mixed_stage(h, 1, L))) return rc;
    run_ghost_f32(h, 1);
    L.in_f = R2;
    L.out_f = R1;
    if ((rc = run_mixed_stage(h, 2, L))) return rc;
    run_ghost_f32(h, 0);
    L.in_f = R1;
    L.out_f = nullptr;
    L.out_d = h->U;
    L.skip_last_i = inflow;
    if ((rc = run_mixed_stage(h, 3, L))) return rc;
    run_ghost(h, h->U, h->U, inflow);
    h->t = h->t + h->dt;
  }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

// RK4 of the configured method (fourth-order differences, Kreiss-Oliger
// dissipation, Sommerfeld outer plane; kg_config.cu)
int step_rk4_cfg(kg_solver* h, int nsteps) {
  int rc;
  if ((rc = ensure(h, &h->RK, 15))) return rc;
  const Grid& g = h->g;
  double2* R1 = h->RK;
  double2* R2 = fld(h->RK, g, 5);
  double2* A = fld(h->RK, g, 10);
  const double* dxb4 = h->dmet + (size_t)T_DXBETA4 * h->NJ * h->PI;
  const double coef[6] = {1.0 / (12.0 * h->dx), 1.0 / (12.0 * h->dy), 1.0 / (12.0 * h->dz),
                          h->ko_eps / (64.0 * h->dx), h->ko_eps / (64.0 * h->dy), h->ko_eps / (64.0 * h->dz)};
  const double rN = h->x1d[h->NI - 1];
  static const int kinds[4] = {kg::ST_RK4_1, kg::ST_RK4_2, kg::ST_RK4_3, kg::ST_RK4_4};
  for (int s = 0; s < nsteps; ++s) {
    kg::StageLaunch L = base_launch(h);
    L.base = h->U;
    L.acc = A;
    double2* ins[4] = {h->U, R1, R2, R1};
    double2* outs[4] = {R1, R2, R1, h->U};
    for (int st = 0; st < 4; ++st) {
      set_in(L, g, ins[st], fld(ins[st], g, 4));
      L.out = outs[st];
      {
        Prof pf(h, kg::ST_RK4_1 + st, 1);
        if (kg::launch_stage_cfg(kinds[st], L, dxb4, h->dmet + (size_t)T_RSG * h->NJ * h->PI, coef, rN,
                                 h->variant != 0, h->stream))
          return set_err(h, KG_ECUDA, "configured stage could not be launched");
      }
      Prof pg(h, PK_GHOST, 2);
      kg::launch_ghost_fill_cfg(g, outs[st], h->stream);
    }
    h->t = h->t + h->dt;
  }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

// RK4 step of a refined level whose outermost planes follow the coarser level:
// after every stage the stage output's buffer planes take the coarse values
// interpolated to the time of the stage that reads them (alpha = position in
// [t_coarse, t_coarse + dt_coarse]; a0 at this step's start, da its length).
int step_rk4_bo(kg_solver* h, kg_solver* c, const double2* c_old, double a0, double da, int nbuf) {
  int rc;
  if ((rc = ensure(h, &h->RK, 15))) return rc;
  const Grid& g = h->g;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  double2* R1 = h->RK;
  double2* R2 = fld(h->RK, g, 5);
  double2* A = fld(h->RK, g, 10);
  auto prolong = [&](double2* u, double alpha) -> int {
    Prof pf(h, PK_PROLONG, 1);
    if (kg::launch_prolong(g, u, c->g, c_old, c->U, alpha, nbuf, h->stream))
      return set_err(h, KG_EINVAL, "refined level does not fit inside its coarser level");
    return KG_OK;
  };
  if ((rc = prolong(h->U, a0))) return rc;
  kg::StageLaunch L = base_launch(h);
  L.base = h->U;
  L.acc = A;
  double2* ins[4] = {h->U, R1, R2, R1};
  double2* outs[4] = {R1, R2, R1, h->U};
  const int kinds[4] = {kg::ST_RK4_1, kg::ST_RK4_2, kg::ST_RK4_3, kg::ST_RK4_4};
  const double at[4] = {a0 + 0.5 * da, a0 + 0.5 * da, a0 + da, a0 + da};
  for (int st = 0; st < 4; ++st) {
    set_in(L, g, ins[st], fld(ins[st], g, 4));
    L.out = outs[st];
    L.skip_last_i = (st == 3) ? inflow : 0;
    run_stage(h, kinds[st], L);
    run_ghost(h, outs[st], h->U, inflow);
    if ((rc = prolong(outs[st], at[st]))) return rc;
  }
  h->t = h->t + h->dt;
  KG_CK(cudaGetLastError());
  return KG_OK;
}

// SSP-RK3 step of a refined level (rk3, MoL/lines_method_lib.f90:211-269): the
// stage inputs u, u1 = u + dt L(u) and u2 = 3/4 u + 1/4 (u1 + dt L(u1)) stand
// at t, t + dt and t + dt/2, so each stage output's buffer planes take the
// coarse values interpolated to those times.
int step_rk3_bo(kg_solver* h, kg_solver* c, const double2* c_old, double a0, double da, int nbuf) {
  int rc;
  if ((rc = ensure(h, &h->RK, 15))) return rc;
  const Grid& g = h->g;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  double2* R1 = h->RK;
  double2* R2 = fld(h->RK, g, 5);
  auto prolong = [&](double2* u, double alpha) -> int {
    Prof pf(h, PK_PROLONG, 1);
    if (kg::launch_prolong(g, u, c->g, c_old, c->U, alpha, nbuf, h->stream))
      return set_err(h, KG_EINVAL, "refined level does not fit inside its coarser level");
    return KG_OK;
  };
  if ((rc = prolong(h->U, a0))) return rc;
  kg::StageLaunch L = base_launch(h);
  L.base = h->U;
  double2* ins[3] = {h->U, R1, R2};
  double2* outs[3] = {R1, R2, h->U};
  const int kinds[3] = {kg::ST_RK3_1, kg::ST_RK3_2, kg::ST_RK3_3};
  const double at[3] = {a0 + da, a0 + 0.5 * da, a0 + da};
  for (int st = 0; st < 3; ++st) {
    set_in(L, g, ins[st], fld(ins[st], g, 4));
    L.out = outs[st];
    L.skip_last_i = (st == 2) ? inflow : 0;
    run_stage(h, kinds[st], L);
    run_ghost(h, outs[st], h->U, inflow);
    if ((rc = prolong(outs[st], at[st]))) return rc;
  }
  h->t = h->t + h->dt;
  KG_CK(cudaGetLastError());
  return KG_OK;
}

// PIRK2 / PIRK3 step of a refined level (pirk2, MoL/lines_method_lib.f90:271-332;
// pirk3, :334-408).  The stage arrays stand at t + dt (u_stage) and t + dt/2
// (u_stage_2, PIRK3), and their buffer planes take the coarse state
// interpolated to those times, Pi included.  So the stale-Pi slot that the
// next step's stage 1 reads holds, on the buffer planes, the coarse Pi at the
// start of that step: the same role the slot plays on the interior, where it
// holds this level's own prediction of Pi there.
int step_pirk_bo(kg_solver* h, kg_solver* c, const double2* c_old, double a0, double da, int nbuf, int order) {
  int rc;
  if ((rc = ensure(h, &h->S, 6))) return rc;
  if (order == 3 && (rc = ensure(h, &h->T, 6))) return rc;
  const Grid& g = h->g;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  auto prolong = [&](double2* u, double2* upi, double alpha) -> int {
    Prof pf(h, PK_PROLONG, 1);
    if (kg::launch_prolong(g, u, c->g, c_old, c->U, alpha, nbuf, h->stream, upi))
      return set_err(h, KG_EINVAL, "refined level does not fit inside its coarser level");
    return KG_OK;
  };
  if ((rc = prolong(h->U, nullptr, a0))) return rc;
  double2* Sold = fld(h->S, g, h->s_cur);
  double2* Snew = fld(h->S, g, 9 - h->s_cur);
  run_pirk_s1(h, Sold, Snew);
  if ((rc = prolong(h->S, Snew, a0 + da))) return rc;
  kg::StageLaunch L = base_launch(h);
  L.base = h->U;
  set_in(L, g, h->S, Snew);
  if (order == 3) {
    double2* Told = fld(h->T, g, h->t_cur);
    double2* Tnew = fld(h->T, g, 9 - h->t_cur);
    L.out = h->T;
    run_stage(h, kg::ST_P3_S2A, L);
    set_in(L, g, h->T, Told);
    L.aux4 = Snew;
    L.out4 = Tnew;
    run_stage(h, kg::ST_P3_S2B, L);
    if ((rc = prolong(h->T, Tnew, a0 + 0.5 * da))) return rc;
    set_in(L, g, h->T, Tnew);
    L.out = h->U;
    L.skip_last_i = inflow;
    run_stage(h, kg::ST_P3_S3, L);
    h->t_cur = 9 - h->t_cur;
  } else {
    L.out = h->U;
    L.skip_last_i = inflow;
    run_stage(h, kg::ST_P2_S2, L);
  }
  run_ghost(h, h->U, h->U, inflow);
  if ((rc = prolong(h->U, nullptr, a0 + da))) return rc;
  h->s_cur = 9 - h->s_cur;
  h->t = h->t + h->dt;
  KG_CK(cudaGetLastError());
  return KG_OK;
}

// Runs nsteps steps.  Pairs of steps are replayed from a CUDA graph captured
// once per stepper and Pi-slot state (two steps return the PIRK slots to the
// state they started in); an odd last step, or runs with profiling on, launch
// directly.  The host-side clock advances exactly as for direct launches.
int run_steps(kg_solver* h, int which, int nsteps, int (*step)(kg_solver*, int)) {
  if (!h || nsteps < 0) return KG_EINVAL;
  int rc;
  if (nsteps < 2 || !h->use_graphs || h->prof_on) return step(h, nsteps);
  int key = ((h->s_cur == 5) ? 1 : 0) + ((h->t_cur == 5) ? 2 : 0);
  if (!h->graphs[which][key].exec || h->graphs[which][key].gen != h->graph_gen) {
    // one direct step first: buffers, kernel attributes and tensor-map encoders
    // are set up outside of any capture
    if ((rc = step(h, 1))) return rc;
    nsteps -= 1;
    if (nsteps < 2) return nsteps ? step(h, nsteps) : KG_OK;
    key = ((h->s_cur == 5) ? 1 : 0) + ((h->t_cur == 5) ? 2 : 0);
  }
  kg_solver::GraphEntry& ge = h->graphs[which][key];
  if (!ge.exec || ge.gen != h->graph_gen) {
    if (ge.exec) {
      cudaGraphExecDestroy(ge.exec);
      ge.exec = nullptr;
    }
    const int s0 = h->s_cur, t0 = h->t_cur;
    const double tt = h->t;
    const long long l0 = h->launches;
    cudaGraph_t graph;
    KG_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    rc = step(h, 2);
    cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
    h->s_cur = s0;
    h->t_cur = t0;
    h->t = tt;
    ge.launches = h->launches - l0;
    h->launches = l0;
    if (rc) return rc;
    if (ec != cudaSuccess) {
      h->err = std::string("graph capture: ") + cudaGetErrorString(ec);
      return KG_ECUDA;
    }
    ec = cudaGraphInstantiate(&ge.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ec != cudaSuccess) {
      ge.exec = nullptr;
      h->err = std::string("graph instantiate: ") + cudaGetErrorString(ec);
      return KG_ECUDA;
    }
    ge.gen = h->graph_gen;
  }
  for (int i = 0; i + 1 < nsteps; i += 2) {
    KG_CK(cudaGraphLaunch(ge.exec, h->stream));
    h->launches += ge.launches;
    h->t = h->t + h->dt;
    h->t = h->t + h->dt;
  }
  if (nsteps & 1) return step(h, 1);
  return KG_OK;
}

}  // namespace

static int only_rk4(kg_solver* h) {
  return set_err(h, KG_EINVAL, "the configured method (kg_set_scheme 1) runs with kg_rk4 only");
}
int kg_pirk2(kg_solver* h, int nsteps) { return h && h->scheme ? only_rk4(h) : run_steps(h, 0, nsteps, step_pirk2); }
int kg_pirk3(kg_solver* h, int nsteps) { return h && h->scheme ? only_rk4(h) : run_steps(h, 1, nsteps, step_pirk3); }
int kg_rk3(kg_solver* h, int nsteps) { return h && h->scheme ? only_rk4(h) : run_steps(h, 2, nsteps, step_rk3); }
int kg_rk4(kg_solver* h, int nsteps) {
  if (h && h->scheme == 1) return run_steps(h, 5, nsteps, step_rk4_cfg);
  if (h && h->precision == 1) return run_steps(h, 4, nsteps, step_rk4_mixed);
  return run_steps(h, 3, nsteps, step_rk4);
}

int kg_set_scheme(kg_solver* h, int scheme, double ko_eps) {
  if (!h || scheme < 0 || scheme > 1 || !(ko_eps >= 0.0)) return KG_EINVAL;
  if (scheme == 1 && h->p.metric != KG_KERR_SCHILD)
    return set_err(h, KG_EINVAL, "the configured method is written for the Kerr_Schild metric form");
  if (scheme == 1 && h->precision == 1)
    return set_err(h, KG_EINVAL, "the configured method runs in FP64 (set precision 0 first)");
  h->scheme = scheme;
  h->ko_eps = ko_eps;
  h->graph_gen++;
  return KG_OK;
}

int kg_get_scheme(const kg_solver* h) { return h ? h->scheme : -1; }

int kg_fill_ghosts_cfg(kg_solver* h) {
  if (!h) return KG_EINVAL;
  kg::launch_ghost_fill_cfg(h->g, h->U, h->stream);
  KG_CK(cudaGetLastError());
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

int kg_set_precision(kg_solver* h, int mode) {
  if (!h || mode < 0 || mode > 1) return KG_EINVAL;
  if (mode == 1 && h->scheme == 1) return set_err(h, KG_EINVAL, "the configured method runs in FP64");
  if (mode == 1 && !kg::tma_available(h->g, h->U)) return set_err(h, KG_EINVAL, "tensor maps unavailable");
  h->precision = mode;
  return KG_OK;
}

int kg_get_precision(const kg_solver* h) { return h ? h->precision : -1; }

int kg_set_graphs(kg_solver* h, int on) {
  if (!h) return KG_EINVAL;
  h->use_graphs = on ? 1 : 0;
  return KG_OK;
}

int kg_rhs(kg_solver* h, const double* host_vars, double* host_rhs, unsigned mask) {
  if (!h || !host_vars || !host_rhs) return KG_EINVAL;
  int rc;
  if ((rc = ensure(h, &h->HV, 10))) return rc;
  const Grid& g = h->g;
  View Vin, Vout;
  for (int v = 0; v < 5; ++v) {
    Vin.v[v] = fld(h->HV, g, v);
    Vout.v[v] = fld(h->HV, g, 5 + v);
  }
  if ((rc = load_view(h, Vin, host_vars, cudaMemcpyHostToDevice))) return rc;
  if ((rc = load_view(h, Vout, host_rhs, cudaMemcpyHostToDevice))) return rc;
  const double2* in[5];
  for (int v = 0; v < 5; ++v) in[v] = Vin.v[v];
  Prof pf(h, PK_RHS, 1);
  kg::launch_rhs(g, metric_of(h), h->p.metric == KG_SCHW_EF ? kg::MK_SCHW : kg::MK_KS, in, Vout.v[0], mask,
                 h->stream);
  KG_CK(cudaGetLastError());
  if ((rc = store_view(h, Vout, host_rhs, cudaMemcpyDeviceToHost))) return rc;
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

int kg_boundary(kg_solver* h, unsigned mask) {
  if (!h) return KG_EINVAL;
  const int inflow = h->p.bc_rmax == KG_INFLOW;
  const double2* up = h->UP ? h->UP : h->U;
  for (int f = 0; f < 6; ++f)
    if (mask & (1u << f)) {
      Prof pf(h, PK_FACE, 1);
      kg::launch_face(h->g, h->U, up, inflow, f, h->stream);
    }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

int kg_send_recv(kg_solver* h) { return h ? KG_OK : KG_EINVAL; }

int kg_get_metric(kg_solver* h, double* out8) {
  if (!h || !out8) return KG_EINVAL;
  const size_t n2 = (size_t)h->NI * h->NJ;
  const int order[8] = {T_ALPHA, T_BETA, T_DXBETA, T_SQRTG, T_GRR, T_GRP, T_GTT, T_GPP};
  for (int t = 0; t < 8; ++t)
    KG_CK(cudaMemcpy2DAsync(out8 + t * n2, sizeof(double) * h->NI, h->dmet + (size_t)order[t] * h->NJ * h->PI,
                            sizeof(double) * h->PI, sizeof(double) * h->NI, h->NJ, cudaMemcpyDeviceToHost,
                            h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

int kg_set_metric(kg_solver* h, const double* in8) {
  if (!h || !in8) return KG_EINVAL;
  const size_t n2 = (size_t)h->NI * h->NJ;
  const int order[8] = {T_ALPHA, T_BETA, T_DXBETA, T_SQRTG, T_GRR, T_GRP, T_GTT, T_GPP};
  for (int t = 0; t < 8; ++t) memcpy(h->tables.data() + (size_t)order[t] * n2, in8 + t * n2, n2 * sizeof(double));
  int rc;
  if ((rc = upload_tables(h))) return rc;
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

int kg_validate_inverse_metric(kg_solver* h, int* e4, int* e3) {
  if (!h) return KG_EINVAL;
  const size_t n2 = (size_t)h->NI * h->NJ;
  const double tol = 1.0e-10;
  long a4 = 0, a3 = 0;
  for (size_t q = 0; q < n2; ++q) {
    for (int mu = 0; mu < 4; ++mu)
      for (int la = 0; la < 4; ++la) {
        double d = 0.0;
        for (int nu = 0; nu < 4; ++nu) d = d + h->gdn[(mu * 4 + nu) * n2 + q] * h->gup[(nu * 4 + la) * n2 + q];
        if (mu == la ? std::fabs(d - 1.0) > tol : std::fabs(d) > tol) a4++;
      }
    for (int mu = 1; mu < 4; ++mu)
      for (int la = 1; la < 4; ++la) {
        double d = 0.0;
        for (int nu = 1; nu < 4; ++nu) d = d + h->gdn[(mu * 4 + nu) * n2 + q] * h->gam[((nu - 1) * 3 + la - 1) * n2 + q];
        if (mu == la ? std::fabs(d - 1.0) > tol : std::fabs(d) > tol) a3++;
      }
  }
  if (e4) *e4 = (int)(a4 * h->NK);
  if (e3) *e3 = (int)(a3 * h->NK);
  return KG_OK;
}

int kg_density(kg_solver* h) {
  if (!h) return KG_EINVAL;
  if (!h->rho) {
    int rc = dalloc(h, (void**)&h->rho, (size_t)h->g.fs * sizeof(double));
    if (rc) return rc;
  }
  {
    Prof pf(h, PK_DENSITY, 1);
    kg::launch_density(h->g, metric_of(h), h->U, h->p.m * h->p.m, h->rho, h->stream);
  }
  KG_CK(cudaGetLastError());
  return KG_OK;
}

int kg_get_density(kg_solver* h, double* host_rho) {
  if (!h || !host_rho) return KG_EINVAL;
  if (!h->rho) return set_err(h, KG_ESTATE, "density has not been computed");
  KG_CK(cudaMemcpy2DAsync(host_rho, sizeof(double) * h->NI, h->rho, sizeof(double) * h->PI, sizeof(double) * h->NI,
                          (size_t)h->NJ * h->NK, cudaMemcpyDeviceToHost, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

int kg_mass_scalar(kg_solver* h, double* out) {
  if (!h || !out) return KG_EINVAL;
  if (!h->rho) {
    int rc = dalloc(h, (void**)&h->rho, (size_t)h->g.fs * sizeof(double));
    if (rc) return rc;
  }
  double* res = h->partials + kg::mass_blocks(h->g);
  {
    Prof pf(h, PK_MASS, 2);
    kg::launch_mass(h->g, metric_of(h), h->rho, h->dx * h->dy * h->dz, h->partials, res, h->stream);
  }
  KG_CK(cudaGetLastError());
  KG_CK(cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

int kg_currents_detectors(kg_solver* h, double* mom) {
  if (!h || !mom) return KG_EINVAL;
  {
    Prof pf(h, PK_SHELL, __builtin_popcount(2 | 4 | 8));
    kg::launch_shell_interp(h->g, metric_of(h), h->U, h->si, h->n_det, h->Ny, h->Nz, 2 | 4 | 8, h->shells, h->stream);
  }
  {
    Prof pf(h, PK_FLUX, 1);
    kg::launch_flux(h->shells, h->si.active, h->n_det, h->Ny, h->Nz, h->dy * h->dz, h->flux, h->stream);
  }
  KG_CK(cudaGetLastError());
  std::vector<double> f(3 * (size_t)h->n_det);
  KG_CK(cudaMemcpyAsync(f.data(), h->flux, f.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  for (int d = 0; d < h->n_det; ++d)
    if (h->active[d])
      for (int c = 0; c < 3; ++c) mom[c + 3 * d] = f[c + 3 * d];
  return KG_OK;
}

int kg_proyector_detectors(kg_solver* h, double* host_alm) {
  if (!h || !host_alm) return KG_EINVAL;
  {
    Prof pf(h, PK_SHELL, __builtin_popcount(1));
    kg::launch_shell_interp(h->g, metric_of(h), h->U, h->si, h->n_det, h->Ny, h->Nz, 1, h->shells, h->stream);
  }
  {
    Prof pf(h, PK_PROJECT, 1);
    kg::launch_project(h->shells, h->si.active, h->n_det, h->L, h->Ny, h->Nz, h->normP, h->cosm, h->sinm, h->sint,
                     h->dy * h->dz, h->alm, h->stream);
  }
  KG_CK(cudaGetLastError());
  const size_t per = (size_t)(h->L + 1) * (2 * h->L + 1);
  std::vector<double2> a(per * h->n_det);
  KG_CK(cudaMemcpyAsync(a.data(), h->alm, a.size() * sizeof(double2), cudaMemcpyDeviceToHost, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  for (int d = 0; d < h->n_det; ++d)
    if (h->active[d]) memcpy(host_alm + 2 * per * d, a.data() + per * d, per * sizeof(double2));
  return KG_OK;
}

int kg_diagnostic(kg_solver* h, int index, double* mass_out) {
  if (!h) return KG_EINVAL;
  if (index % h->save == 0) {
    {
      Prof pf(h, PK_SHELL, __builtin_popcount(15));
      kg::launch_shell_interp(h->g, metric_of(h), h->U, h->si, h->n_det, h->Ny, h->Nz, 15, h->shells, h->stream);
    }
    {
      Prof pf(h, PK_FLUX, 1);
      kg::launch_flux(h->shells, h->si.active, h->n_det, h->Ny, h->Nz, h->dy * h->dz, h->flux, h->stream);
    }
    {
      Prof pf(h, PK_PROJECT, 1);
      kg::launch_project(h->shells, h->si.active, h->n_det, h->L, h->Ny, h->Nz, h->normP, h->cosm, h->sinm, h->sint,
                       h->dy * h->dz, h->alm, h->stream);
    }
    KG_CK(cudaGetLastError());
  }
  if (mass_out) return kg_mass_scalar(h, mass_out);
  return KG_OK;
}

int kg_set_detectors(kg_solver* h, int n, const double* radii) {
  if (!h || n < 1 || !radii) return KG_EINVAL;
  KG_CK(cudaStreamSynchronize(h->stream));
  h->n_det = n;
  int rc = build_detectors(h, radii);
  if (rc) return rc;
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_OK;
}

}  // extern "C"

namespace {
// the all-shell projection into device memory; *out_alm = (L+1) x (2L+1) x Nx complex
int project_all(kg_solver* h, int L, int precision, double2** out_alm) {
  const int Ny = h->Ny, Nz = h->Nz, Nx = h->Nx;
  const int Nm = (L + 1) * (L + 2) / 2;
  const int K = Ny * Nz;
  const int Kp = kg::ylm_gemm_pad_k(K), Mp = kg::ylm_gemm_pad_m(2 * Nx), Np = kg::ylm_gemm_pad_n(2 * Nm);
  const size_t nalm = (size_t)(L + 1) * (2 * L + 1) * Nx;
  // buffer plan: Ahi, Alo (Mp x Kp bf16), Bhi, Blo (Np x Kp), C (nsplit x Mp x Np f32), F (Nx K c128), alm
  const int nsplit = kg::ylm_gemm_splits(Kp);
  const size_t szA = (size_t)Mp * Kp * 2, szB = (size_t)Np * Kp * 2, szC = (size_t)nsplit * Mp * Np * 4;
  const size_t szF = (size_t)Nx * K * 16, szAlm = nalm * 16;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t need = 2 * al(szA) + 2 * al(szB) + al(szC) + al(szF) + al(szAlm);
  if (h->ylmL != L) {
    dfree(h, h->ylm_tab);
    h->ylm_tab = nullptr;
    std::vector<double> tab((size_t)(L + 1) * (L + 1) * Ny + 2 * (size_t)(L + 1) * Nz, 0.0);
    double* normP = tab.data();
    double* cosm = normP + (size_t)(L + 1) * (L + 1) * Ny;
    double* sinm = cosm + (size_t)(L + 1) * Nz;
    for (int l = 0; l <= L; ++l)
      for (int m = 0; m <= l; ++m)
        for (int jv = 1; jv <= Ny; ++jv)
          normP[((size_t)l * (L + 1) + m) * Ny + jv - 1] = norm_plm(l, m, (double)(jv - 1) * h->dy);
    for (int m = 0; m <= L; ++m)
      for (int kv = 1; kv <= Nz; ++kv) {
        const double ph = (double)(kv - 1) * h->dz;
        cosm[(size_t)m * Nz + kv - 1] = std::cos(m * ph);
        sinm[(size_t)m * Nz + kv - 1] = std::sin(m * ph);
      }
    int rc = dalloc(h, (void**)&h->ylm_tab, tab.size() * sizeof(double));
    if (rc) return rc;
    KG_CK(cudaMemcpyAsync(h->ylm_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->ylmL = L;
    h->ylm_b_ready = 0;
  }
  if (h->ylm_bytes < need) {
    dfree(h, h->ylm_buf);
    h->ylm_buf = nullptr;
    int rc = dalloc(h, (void**)&h->ylm_buf, need);
    if (rc) return rc;
    h->ylm_bytes = need;
    h->ylm_b_ready = 0;
  }
  unsigned char* q = h->ylm_buf;
  __nv_bfloat16* Ahi = (__nv_bfloat16*)q; q += al(szA);
  __nv_bfloat16* Alo = (__nv_bfloat16*)q; q += al(szA);
  __nv_bfloat16* Bhi = (__nv_bfloat16*)q; q += al(szB);
  __nv_bfloat16* Blo = (__nv_bfloat16*)q; q += al(szB);
  float* Cm = (float*)q; q += al(szC);
  double2* F = (double2*)q; q += al(szF);
  double2* dalm = (double2*)q;
  const double* normP = h->ylm_tab;
  const double* cosm = normP + (size_t)(L + 1) * (L + 1) * Ny;
  const double* sinm = cosm + (size_t)(L + 1) * Nz;
  const double dydz = h->dy * h->dz;
  if (precision == 1) {
    if (!h->ylm_b_ready) {
      KG_CK(cudaMemsetAsync(Bhi, 0, 2 * al(szB), h->stream));
      KG_CK(cudaMemsetAsync(Ahi, 0, 2 * al(szA), h->stream));
      // the a_lm entries with |m| > l, which the assembly never writes (the FP64
      // path writes them as zeros); the layout changes only with L or the buffer
      KG_CK(cudaMemsetAsync(dalm, 0, al(szAlm), h->stream));
      {
        Prof pf(h, PK_YLM_PREP, 1);
        kg::launch_ylm_b(L, Ny, Nz, Kp, normP, cosm, sinm, h->sint, Bhi, Blo, h->stream);
      }
      h->ylm_b_ready = 1;
    }
    {
      Prof pf(h, PK_YLM_PREP, 1);
      kg::launch_shells_to_a(h->g, h->U, h->si, Nx, Ny, Nz, Kp, Ahi, Alo, nullptr, h->stream);
    }
    {
      Prof pf(h, PK_YLM_GEMM, 1);
      if (kg::launch_ylm_gemm(Ahi, Alo, Bhi, Blo, Cm, Mp, Np, Kp, h->derr, h->stream))
        return set_err(h, KG_ECUDA, "tensor-core projection could not be configured");
    }
    {
      Prof pf(h, PK_YLM_PREP, 1);
      kg::launch_ylm_assemble(Cm, Np, (long long)Mp * Np, nsplit, Nx, L, dydz, dalm, h->stream);
    }
  } else {
    {
      Prof pf(h, PK_YLM_PREP, 1);
      kg::launch_shells_to_a(h->g, h->U, h->si, Nx, Ny, Nz, Kp, nullptr, nullptr, F, h->stream);
    }
    Prof pf(h, PK_YLM_FP64, 1);
    kg::launch_ylm_fp64(F, Nx, L, Ny, Nz, normP, cosm, sinm, h->sint, dydz, dalm, h->stream);
  }
  KG_CK(cudaGetLastError());
  *out_alm = dalm;
  return KG_OK;
}

int ensure_radial_basis(kg_solver* h, int L, int Nk) {
  if (h->radL == L && h->radNk == Nk) return KG_OK;
  const int Nx = h->Nx;
  kg::bessel_basis(L, Nk, Nx, h->xmin, h->dx, h->r_max, h->rad_k, h->rad_basis);
  std::vector<double> jr((size_t)(L + 1) * Nx * Nk);
  for (int l = 0; l <= L; ++l)
    for (int n = 0; n < Nk; ++n)
      for (int i = 0; i < Nx; ++i) {
        const double r = h->xmin + (double)i * h->dx;
        jr[((size_t)l * Nx + i) * Nk + n] = h->rad_basis[((size_t)l * Nk + n) * Nx + i] * (r * r);
      }
  for (void** p : {(void**)&h->rad_jr, (void**)&h->rad_ft})
    if (*p) {
      dfree(h, *p);
      *p = nullptr;
    }
  int rc;
  if ((rc = dalloc(h, (void**)&h->rad_jr, jr.size() * sizeof(double)))) return rc;
  if ((rc = dalloc(h, (void**)&h->rad_ft, (size_t)Nk * (L + 1) * (2 * L + 1) * sizeof(double2)))) return rc;
  KG_CK(cudaMemcpyAsync(h->rad_jr, jr.data(), jr.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  h->radL = L;
  h->radNk = Nk;
  return KG_OK;
}
}  // namespace

extern "C" {

int kg_project_all_shells(kg_solver* h, int L, int precision, double* host_alm) {
  if (!h || !host_alm || L < 0 || L > 128 || precision < 0 || precision > 1) return KG_EINVAL;
  double2* dalm = nullptr;
  int rc = project_all(h, L, precision, &dalm);
  if (rc) return rc;
  const size_t szAlm = (size_t)(L + 1) * (2 * L + 1) * h->Nx * sizeof(double2);
  KG_CK(cudaMemcpyAsync(host_alm, dalm, szAlm, cudaMemcpyDeviceToHost, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  return check_device_flag(h);
}

int kg_bessel_basis(kg_solver* h, int L, int Nk, double* k_values, double* j_basis) {
  if (!h || L < 0 || L > 128 || Nk < 1 || Nk > 4096) return KG_EINVAL;
  int rc = ensure_radial_basis(h, L, Nk);
  if (rc) return rc;
  const int NL = L + 1, Nx = h->Nx;
  for (int l = 0; l <= L; ++l)
    for (int n = 0; n < Nk; ++n) {
      if (k_values) k_values[l + (size_t)NL * n] = h->rad_k[(size_t)l * Nk + n];
      if (j_basis)
        for (int i = 0; i < Nx; ++i)
          j_basis[l + (size_t)NL * (n + (size_t)Nk * i)] = h->rad_basis[((size_t)l * Nk + n) * Nx + i];
    }
  return KG_OK;
}

int kg_sph_ft_radial(kg_solver* h, int L, int Nk, int precision, double* host_ft) {
  if (!h || !host_ft || L < 0 || L > 128 || Nk < 1 || Nk > 4096 || precision < 0 || precision > 1)
    return KG_EINVAL;
  int rc = ensure_radial_basis(h, L, Nk);
  if (rc) return rc;
  double2* dalm = nullptr;
  if ((rc = project_all(h, L, precision, &dalm))) return rc;
  const double dr = std::fabs((h->xmin + h->dx) - h->xmin);
  {
    Prof pf(h, PK_RADIAL, 1);
    kg::launch_radial_ft(dalm, h->rad_jr, L, Nk, h->Nx, dr, h->rad_ft, h->stream);
  }
  KG_CK(cudaGetLastError());
  KG_CK(cudaMemcpyAsync(host_ft, h->rad_ft, (size_t)Nk * (L + 1) * (2 * L + 1) * sizeof(double2),
                        cudaMemcpyDeviceToHost, h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  return check_device_flag(h);
}

// ---- checkpoint / resume ----------------------------------------------------
// check_point / read_from_check_point (MoL/lines_method_lib.f90:599-667) write
// nvars, Nx, Ny, Nz, g_pts, t and, per stored point, x, y, z, u(:) as list-
// directed text; the reader deletes the file before opening it, and neither
// keeps the PIRK stage state that the next step reads (the previous step's Pi
// in u_stage), so a resumed PIRK run differs from an uninterrupted one.  This
// format is binary and complete: a 128-byte header, then u and, when they
// exist, u_stage and u_stage_2, each as complex(8) u(1:5, -g:Nx+g, -g:Ny+g,
// 0:Nz) (the reference's array layout, variable fastest).  Loading into a handle
// of the same grid continues bit for bit.
namespace {
struct CkptHeader {
  char magic[8];        // "KGB2CKPT"
  int version;          // 1
  int Nx, Ny, Nz, g_pts, metric, bc_rmax, scheme, precision;
  int has_stage, has_stage2, reserved;
  double t, dt, ko_eps, m, xmin, xmax;
  char pad[128 - 8 - 12 * 4 - 6 * 8];
};
static_assert(sizeof(CkptHeader) == 128, "checkpoint header is 128 bytes");
}  // namespace

int kg_save_checkpoint(kg_solver* h, const char* path) {
  if (!h || !path) return KG_EINVAL;
  CkptHeader hd;
  memset(&hd, 0, sizeof(hd));
  memcpy(hd.magic, "KGB2CKPT", 8);
  hd.version = 1;
  hd.Nx = h->Nx; hd.Ny = h->Ny; hd.Nz = h->Nz; hd.g_pts = h->p.g_pts;
  hd.metric = h->p.metric; hd.bc_rmax = h->p.bc_rmax; hd.scheme = h->scheme; hd.precision = h->precision;
  hd.has_stage = h->S ? 1 : 0;
  hd.has_stage2 = h->T ? 1 : 0;
  hd.t = h->t; hd.dt = h->dt; hd.ko_eps = h->ko_eps; hd.m = h->p.m; hd.xmin = h->p.xmin; hd.xmax = h->p.xmax;
  const size_t n = (size_t)5 * h->NI * h->NJ * h->NK * 2;  // doubles per state
  std::vector<double> buf;
  try {
    buf.resize(n);
  } catch (...) {
    return set_err(h, KG_ENOMEM, "host buffer for the checkpoint");
  }
  FILE* f = fopen(path, "wb");
  if (!f) return set_err(h, KG_EINVAL, std::string("cannot open for writing: ") + path);
  int rc = KG_OK;
  if (fwrite(&hd, sizeof(hd), 1, f) != 1) rc = set_err(h, KG_EINVAL, "checkpoint write failed");
  const int whichs[3] = {0, 1, 2};
  const int have[3] = {1, hd.has_stage, hd.has_stage2};
  for (int w = 0; w < 3 && rc == KG_OK; ++w) {
    if (!have[w]) continue;
    if ((rc = kg_get_state(h, whichs[w], buf.data()))) break;
    if (fwrite(buf.data(), sizeof(double), n, f) != n) rc = set_err(h, KG_EINVAL, "checkpoint write failed");
  }
  if (fclose(f) != 0 && rc == KG_OK) rc = set_err(h, KG_EINVAL, "checkpoint close failed");
  return rc;
}

int kg_load_checkpoint(kg_solver* h, const char* path) {
  if (!h || !path) return KG_EINVAL;
  FILE* f = fopen(path, "rb");
  if (!f) return set_err(h, KG_EINVAL, std::string("cannot open for reading: ") + path);
  CkptHeader hd;
  if (fread(&hd, sizeof(hd), 1, f) != 1 || memcmp(hd.magic, "KGB2CKPT", 8) != 0 || hd.version != 1) {
    fclose(f);
    return set_err(h, KG_EINVAL, "not a checkpoint of this library");
  }
  // the state only means the same thing on the same grid, metric, outer
  // boundary, field mass, radial extent and method
  std::string why;
  if (hd.Nx != h->Nx || hd.Ny != h->Ny || hd.Nz != h->Nz || hd.g_pts != h->p.g_pts)
    why = "checkpoint grid differs from the handle's grid";
  else if (hd.metric != h->p.metric)
    why = "checkpoint metric differs from the handle's metric";
  else if (hd.bc_rmax != h->p.bc_rmax)
    why = "checkpoint outer boundary condition differs from the handle's";
  else if (hd.m != h->p.m)
    why = "checkpoint field mass differs from the handle's";
  else if (hd.xmin != h->p.xmin || hd.xmax != h->p.xmax)
    why = "checkpoint radial extent (xmin, xmax) differs from the handle's";
  else if (hd.scheme != h->scheme || (hd.scheme == 1 && hd.ko_eps != h->ko_eps))
    why = "checkpoint method (scheme, Kreiss-Oliger eps) differs from the handle's; call kg_set_scheme first";
  else if (hd.precision != h->precision)
    why = "checkpoint precision mode differs from the handle's; call kg_set_precision first";
  else if (hd.has_stage < 0 || hd.has_stage > 1 || hd.has_stage2 < 0 || hd.has_stage2 > 1)
    why = "checkpoint header is corrupt";
  if (!why.empty()) {
    fclose(f);
    return set_err(h, KG_EINVAL, why);
  }
  // read the whole file before touching the handle, so a truncated or
  // unreadable file leaves it as it was
  const size_t n = (size_t)5 * h->NI * h->NJ * h->NK * 2;
  const int have[3] = {1, hd.has_stage, hd.has_stage2};
  const int nstates = have[0] + have[1] + have[2];
  std::vector<double> buf;
  try {
    buf.resize(n * nstates);
  } catch (...) {
    fclose(f);
    return set_err(h, KG_ENOMEM, "host buffer for the checkpoint");
  }
  const bool complete = fread(buf.data(), sizeof(double), n * nstates, f) == n * nstates;
  fclose(f);
  if (!complete) return set_err(h, KG_EINVAL, "checkpoint truncated");
  int rc;
  size_t at = 0;
  for (int w = 0; w < 3; ++w) {
    if (!have[w]) continue;
    if ((rc = kg_set_state(h, w, buf.data() + at))) return rc;
    at += n;
  }
  // stage arrays the file does not hold return to the state of a fresh
  // handle: zero, with the current Pi value in slot 4 (PIRK stage 1 reads it
  // as the previous step's Pi)
  if (!hd.has_stage) {
    h->s_cur = 4;
    if (h->S) KG_CK(cudaMemsetAsync(h->S, 0, 6 * field_bytes(h), h->stream));
  }
  if (!hd.has_stage2) {
    h->t_cur = 4;
    if (h->T) KG_CK(cudaMemsetAsync(h->T, 0, 6 * field_bytes(h), h->stream));
  }
  KG_CK(cudaStreamSynchronize(h->stream));
  h->t = hd.t;
  h->dt = hd.dt;
  return KG_OK;
}

int kg_get_detectors(kg_solver* h, double* r_det, int* index_det) {
  if (!h) return KG_EINVAL;
  for (int d = 0; d < h->n_det; ++d) {
    if (r_det) r_det[d] = h->r_det[d];
    if (index_det) index_det[d] = h->index_det[d];
  }
  return KG_OK;
}

int kg_sph_harmonics(kg_solver* h, int L, double* out) {
  if (!h || !out || L < 0) return KG_EINVAL;
  const int NL = L + 1, NM = 2 * L + 1;
  double2* Y = (double2*)out;
  memset(Y, 0, sizeof(double2) * (size_t)NL * NM * h->Ny * h->Nz);
  for (int l = 0; l <= L; ++l)
    for (int m = 0; m <= l; ++m)
      for (int jv = 1; jv <= h->Ny; ++jv) {
        const double np = norm_plm(l, m, (double)(jv - 1) * h->dy);
        for (int kv = 1; kv <= h->Nz; ++kv) {
          const double ph = (double)(kv - 1) * h->dz;
          const double2 y = make_double2(np * std::cos(m * ph), np * std::sin(m * ph));
          const size_t base = (size_t)(jv - 1) + (size_t)h->Ny * (kv - 1);
          Y[l + NL * ((m + L) + NM * base)] = y;
          if (m > 0) {
            const double sg = (m % 2) ? -1.0 : 1.0;
            Y[l + NL * ((-m + L) + NM * base)] = make_double2(sg * y.x, sg * -y.y);
          }
        }
      }
  return KG_OK;
}

int kg_set_kernel_variant(kg_solver* h, int variant) {
  if (!h || variant < 0 || variant > 3) return KG_EINVAL;
  if (variant >= 2 && !kg::tma_available(h->g, h->U))
    return set_err(h, KG_EINVAL, "tensor maps unavailable for this grid: forms 2 and 3 need them");
  h->variant = variant;
  h->graph_gen++;
  return KG_OK;
}

int kg_check_wait_timeout(kg_solver* h, long long polls) {
  if (!h || polls < 1 || polls > (1LL << 20)) return KG_EINVAL;
  KG_CK(cudaStreamSynchronize(h->stream));
  int rc = check_device_flag(h);
  if (rc) return rc;  // an earlier wait ran out: report that one
  if (kg::launch_wait_check(h->derr, polls, h->stream)) return set_err(h, KG_ECUDA, "wait check launch failed");
  rc = check_device_flag(h);  // KG_ETIMEOUT, with the message of a stage launch whose copies never landed
  if (rc != KG_ETIMEOUT) return rc ? rc : set_err(h, KG_ECUDA, "the bounded wait did not run out");
  // clear the flag: the CTA left nothing in flight, so the handle stays usable
  KG_CK(cudaMemsetAsync(h->derr, 0, sizeof(int), h->stream));
  KG_CK(cudaStreamSynchronize(h->stream));
  return KG_ETIMEOUT;
}

int kg_set_tile_rows(kg_solver* h, int rows) {
  if (!h || (rows != 4 && rows != 8)) return KG_EINVAL;
  if (rows != h->tile_rows) {
    h->tile_rows = rows;
    h->graph_gen++;
  }
  return KG_OK;
}

int kg_get_tile_rows(const kg_solver* h) { return h ? h->tile_rows : KG_EINVAL; }

int kg_profile_enable(kg_solver* h, int on) {
  if (!h) return KG_EINVAL;
  h->prof_on = on ? 1 : 0;
  return KG_OK;
}

int kg_profile_kinds(void) { return PK_COUNT; }

const char* kg_profile_kind_name(int kind) { return (kind >= 0 && kind < PK_COUNT) ? kPkNames[kind] : ""; }

int kg_profile_read(kg_solver* h, double* ms, long long* launches) {
  if (!h) return KG_EINVAL;
  KG_CK(cudaStreamSynchronize(h->stream));
  if (ms)
    for (int k = 0; k < PK_COUNT; ++k) ms[k] = 0.0;
  if (launches)
    for (int k = 0; k < PK_COUNT; ++k) launches[k] = 0;
  for (auto& r : h->recs) {
    float t = 0.f;
    cudaEventElapsedTime(&t, r.a, r.b);
    if (ms) ms[r.kind] += t;
    if (launches) launches[r.kind] += 1;
    h->pool.push_back(r.a);
    h->pool.push_back(r.b);
  }
  h->recs.clear();
  return KG_OK;
}

long long kg_launch_count(const kg_solver* h) { return h ? h->launches : 0; }

}  // extern "C"

// =============================================================================
// Batched engine: many solves advanced together by RK4 with one persistent
// launch per stage over the ragged work list of all their tiles, plus one
// batched ghost fill, the whole step replayed from a CUDA graph.
struct kg_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  int metric_kind = -1;
  std::vector<kg_solver*> members;
  bool dirty = true;
  int kchunk = 32;
  int blocks = 0;
  // per RK4 stage: item records and ghost descriptors (device)
  unsigned char* ditems[4] = {nullptr, nullptr, nullptr, nullptr};
  kg::GhostDesc* dghost[4] = {nullptr, nullptr, nullptr, nullptr};
  unsigned char* dghost_f[3] = {nullptr, nullptr, nullptr};  // FP32 stage fills (mixed precision)
  int precision = 0;                                         // 0: FP64 RK4, 1: mixed (kg_mixed.cu)
  size_t items_cap = 0, ghost_cap = 0;
  int n_items[4] = {0, 0, 0, 0};
  long long max_rows = 0, max_faces = 0, max_z = 0;
  int* derr = nullptr;
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0;
  long long launches = 0;
  cudaEvent_t ev = nullptr;
  double2* pin = nullptr;  // pinned staging of the members' detector a_lm
  size_t pin_cap = 0;
  // 0: one persistent launch per stage over every member; 1: every member's
  // own single-solve kernels on its own stream, concurrently (forked from and
  // joined back into the batch stream); variant: the members' stage-kernel form
  // in dispatch 1 (-1 keeps each member's own)
  int dispatch = 0;
  int variant = -1;
  // theta rows of the TMA tiles (8 or 4): the persistent launch's work items,
  // and in dispatch 1 every member's RK4 stage kernels
  int tile_rows = 8;
};

#define KG_BCK(call)                                                        \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) {                                                \
      b->err = std::string(#call) + ": " + cudaGetErrorString(e_);         \
      return KG_ECUDA;                                                      \
    }                                                                       \
  } while (0)

namespace {

int batch_rebuild(kg_batch* b) {
  const int n = (int)b->members.size();
  const bool mixed = b->precision == 1;
  const size_t isz = mixed ? kg::mixed_item_bytes() : kg::batch_item_bytes();
  const size_t isz_max = std::max(kg::mixed_item_bytes(), kg::batch_item_bytes());
  const size_t gfsz = kg::ghost_f32_desc_bytes();
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  if ((size_t)n > b->items_cap) {
    for (int st = 0; st < 4; ++st) {
      if (b->ditems[st]) cudaFree(b->ditems[st]);
      if (b->dghost[st]) cudaFree(b->dghost[st]);
      b->ditems[st] = nullptr;
      b->dghost[st] = nullptr;
    }
    for (int st = 0; st < 3; ++st) {
      if (b->dghost_f[st]) cudaFree(b->dghost_f[st]);
      b->dghost_f[st] = nullptr;
    }
    size_t cap = n < 16 ? 16 : (size_t)n * 2;
    for (int st = 0; st < 4; ++st) {
      KG_BCK(cudaMalloc((void**)&b->ditems[st], cap * isz_max));
      KG_BCK(cudaMalloc((void**)&b->dghost[st], cap * sizeof(kg::GhostDesc)));
    }
    for (int st = 0; st < 3; ++st) KG_BCK(cudaMalloc((void**)&b->dghost_f[st], cap * gfsz));
    b->items_cap = cap;
  }
  std::vector<unsigned char> hitems((size_t)n * isz);
  std::vector<kg::GhostDesc> hg(n);
  std::vector<unsigned char> hgf((size_t)n * gfsz);
  const int kinds[4] = {kg::ST_RK4_1, kg::ST_RK4_2, kg::ST_RK4_3, kg::ST_RK4_4};
  b->max_rows = b->max_faces = b->max_z = 0;
  for (int st = 0; st < 4; ++st) {
    int item0 = 0;
    for (int i = 0; i < n; ++i) {
      kg_solver* h = b->members[i];
      const Grid& g = h->g;
      if (mixed) {
        const int inflow = h->p.bc_rmax == KG_INFLOW;
        float2* F1 = h->MX;
        float2* F2 = h->MX + 5 * g.fs;
        kg::MixedLaunch M = mixed_launch(h);
        M.in_f = st == 1 ? F1 : (st == 2 ? F2 : (st == 3 ? F1 : nullptr));
        M.out_f = st == 0 ? F1 : (st == 1 ? F2 : (st == 2 ? F1 : nullptr));
        M.out_d = st == 3 ? h->U : nullptr;
        M.skip_last_i = st == 3 ? inflow : 0;
        const double* rsg = h->dmet + (size_t)T_RSG * h->NJ * h->PI;
        const int ni = kg::build_mixed_item(hitems.data() + (size_t)i * isz, kinds[st], M, rsg, b->derr, b->kchunk,
                                            item0, b->tile_rows);
        if (ni < 0) {
          b->err = "tensor-map encoding failed for a batch member";
          return KG_ECUDA;
        }
        item0 += ni;
        if (st < 3) kg::fill_ghost_f32_desc(hgf.data() + (size_t)i * gfsz, g, M.out_f, h->U, inflow);
        hg[i].g = g;
        hg[i].u = h->U;
        hg[i].up = h->U;
        hg[i].inflow = inflow;
        if (st == 0) {
          b->max_rows = std::max(b->max_rows, 6LL * g.NK * g.NI);
          b->max_faces = std::max(b->max_faces, 2LL * (g.NJ - 6) * g.NK);
          b->max_z = std::max(b->max_z, 2LL * g.NI * g.NJ);
        }
        continue;
      }
      double2* R1 = h->RK;
      double2* R2 = fld(h->RK, g, 5);
      double2* A = fld(h->RK, g, 10);
      kg::StageLaunch L = base_launch(h);
      L.base = h->U;
      L.acc = A;
      double2* in = st == 0 ? h->U : (st == 1 ? R1 : (st == 2 ? R2 : R1));
      double2* out = st == 0 ? R1 : (st == 1 ? R2 : (st == 2 ? R1 : h->U));
      set_in(L, g, in, fld(in, g, 4));
      L.out = out;
      L.skip_last_i = (st == 3) ? (h->p.bc_rmax == KG_INFLOW) : 0;
      const double* rsg = h->dmet + (size_t)T_RSG * h->NJ * h->PI;
      const int ni = kg::build_batch_item(hitems.data() + (size_t)i * isz, kinds[st], L, rsg, b->derr, b->kchunk,
                                          item0, b->tile_rows);
      if (ni < 0) {
        b->err = "tensor-map encoding failed for a batch member";
        return KG_ECUDA;
      }
      item0 += ni;
      hg[i].g = g;
      hg[i].u = out;
      hg[i].up = h->U;
      hg[i].inflow = h->p.bc_rmax == KG_INFLOW;
      if (st == 0) {
        b->max_rows = std::max(b->max_rows, 6LL * g.NK * g.NI);
        b->max_faces = std::max(b->max_faces, 2LL * (g.NJ - 6) * g.NK);
        b->max_z = std::max(b->max_z, 2LL * g.NI * g.NJ);
      }
    }
    b->n_items[st] = item0;
    KG_BCK(cudaMemcpyAsync(b->ditems[st], hitems.data(), (size_t)n * isz, cudaMemcpyHostToDevice, b->stream));
    KG_BCK(cudaMemcpyAsync(b->dghost[st], hg.data(), (size_t)n * sizeof(kg::GhostDesc), cudaMemcpyHostToDevice,
                           b->stream));
    if (mixed && st < 3)
      KG_BCK(cudaMemcpyAsync(b->dghost_f[st], hgf.data(), (size_t)n * gfsz, cudaMemcpyHostToDevice, b->stream));
  }
  KG_BCK(cudaStreamSynchronize(b->stream));
  b->dirty = false;
  return KG_OK;
}

int batch_enqueue_step(kg_batch* b) {
  const int n = (int)b->members.size();
  const int kinds[4] = {kg::ST_RK4_1, kg::ST_RK4_2, kg::ST_RK4_3, kg::ST_RK4_4};
  for (int st = 0; st < 4; ++st) {
    const int bad = b->precision == 1
                        ? kg::launch_batch_mixed(kinds[st], b->metric_kind, b->ditems[st], n, b->n_items[st],
                                                 b->blocks, b->tile_rows, b->stream)
                        : kg::launch_batch_tma(kinds[st], b->metric_kind, b->ditems[st], n, b->n_items[st],
                                               b->blocks, b->tile_rows, b->stream);
    if (bad) {
      b->err = "batched stage launch could not be configured";
      return KG_ECUDA;
    }
    if (b->precision == 1 && st < 3)
      kg::launch_ghost_fill_f32(b->dghost_f[st], n, b->max_rows, b->max_faces, b->max_z, b->stream);
    else
      kg::launch_ghost_fill_batch(b->dghost[st], n, b->max_rows, b->max_faces, b->max_z, b->stream);
    b->launches += 3;
  }
  KG_BCK(cudaGetLastError());
  return KG_OK;
}

}  // namespace

extern "C" {

int kg_batch_create(int device, kg_batch** out) {
  if (!out) return KG_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return KG_ENODEV;
  }
  if (device >= 0 && (device >= ndev || cudaSetDevice(device) != cudaSuccess)) return KG_ENODEV;
  kg_batch* b = new kg_batch();
  cudaGetDevice(&b->device);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  b->blocks = 2 * sms;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc((void**)&b->derr, 16) != cudaSuccess || cudaMemsetAsync(b->derr, 0, 16, b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess) {
    kg_batch_destroy(b);
    return KG_ECUDA;
  }
  *out = b;
  return KG_OK;
}

int kg_batch_destroy(kg_batch* b) {
  if (!b) return KG_EINVAL;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (int st = 0; st < 4; ++st) {
    if (b->ditems[st]) cudaFree(b->ditems[st]);
    if (b->dghost[st]) cudaFree(b->dghost[st]);
  }
  for (int st = 0; st < 3; ++st)
    if (b->dghost_f[st]) cudaFree(b->dghost_f[st]);
  if (b->pin) cudaFreeHost(b->pin);
  if (b->derr) cudaFree(b->derr);
  if (b->ev) cudaEventDestroy(b->ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return KG_OK;
}

const char* kg_batch_last_error(const kg_batch* b) { return b ? b->err.c_str() : "null batch"; }

int kg_batch_add(kg_batch* b, kg_solver* h) {
  if (!b || !h) return KG_EINVAL;
  if (h->device != b->device) return set_err(h, KG_EINVAL, "batch member on another device");
  const int mk = h->p.metric == KG_SCHW_EF ? kg::MK_SCHW : kg::MK_KS;
  if (b->metric_kind >= 0 && mk != b->metric_kind) {
    b->err = "all members of a batch use the same metric";
    return KG_EINVAL;
  }
  for (kg_solver* m : b->members)
    if (m == h) return KG_OK;
  int rc;
  if ((rc = b->precision == 1 ? ensure_mixed(h) : ensure(h, &h->RK, 15))) return rc;
  if (!kg::tma_available(h->g, h->U)) {
    b->err = "tensor maps unavailable for this grid";
    return KG_EINVAL;
  }
  b->metric_kind = mk;
  b->members.push_back(h);
  b->dirty = true;
  return KG_OK;
}

int kg_batch_remove(kg_batch* b, kg_solver* h) {
  if (!b || !h) return KG_EINVAL;
  for (size_t i = 0; i < b->members.size(); ++i)
    if (b->members[i] == h) {
      // a member leaving must not have batch work in flight on its buffers
      KG_BCK(cudaStreamSynchronize(b->stream));
      b->members.erase(b->members.begin() + (long)i);
      b->dirty = true;
      if (b->members.empty()) b->metric_kind = -1;
      return KG_OK;
    }
  return KG_EINVAL;
}

int kg_batch_size(const kg_batch* b) { return b ? (int)b->members.size() : 0; }

// RK4 (MoL/lines_method_lib.f90:411-474) for every member, nsteps times.
int kg_batch_rk4(kg_batch* b, int nsteps) {
  if (!b || nsteps < 0) return KG_EINVAL;
  if (b->members.empty() || nsteps == 0) return KG_OK;
  int rc;
  if (b->dispatch == 1) {
    // fork: each member's stream waits for the batch stream's pending work
    KG_BCK(cudaEventRecord(b->ev, b->stream));
    for (kg_solver* h : b->members) KG_BCK(cudaStreamWaitEvent(h->stream, b->ev, 0));
    for (kg_solver* h : b->members) {
      if (b->variant >= 0 && h->variant != b->variant) {
        h->variant = b->variant;
        h->graph_gen++;
      }
      if (h->tile_rows != b->tile_rows) {
        h->tile_rows = b->tile_rows;
        h->graph_gen++;
      }
      rc = b->precision ? run_steps(h, 4, nsteps, step_rk4_mixed) : run_steps(h, 3, nsteps, step_rk4);
      if (rc) {
        b->err = h->err;
        return rc;
      }
    }
    // join: the batch stream (detector sampling, admissions) waits for every member
    for (kg_solver* h : b->members) {
      KG_BCK(cudaEventRecord(b->ev, h->stream));
      KG_BCK(cudaStreamWaitEvent(b->stream, b->ev, 0));
    }
    return KG_OK;
  }
  if (b->dirty && (rc = batch_rebuild(b))) return rc;
  // order after each member's own pending work
  for (kg_solver* h : b->members) {
    KG_BCK(cudaEventRecord(b->ev, h->stream));
    KG_BCK(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  if (!b->graph) {
    // first step direct (kernel attributes), then capture one step
    const long long l0 = b->launches;
    if ((rc = batch_enqueue_step(b))) return rc;
    for (kg_solver* h : b->members) h->t = h->t + h->dt;
    nsteps -= 1;
    cudaGraph_t graph;
    KG_BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const long long l1 = b->launches;
    rc = batch_enqueue_step(b);
    cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
    b->graph_launches = b->launches - l1;
    b->launches = l1;
    if (rc) return rc;
    if (ec != cudaSuccess) {
      b->err = std::string("batch graph capture: ") + cudaGetErrorString(ec);
      return KG_ECUDA;
    }
    ec = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ec != cudaSuccess) {
      b->graph = nullptr;
      b->err = std::string("batch graph instantiate: ") + cudaGetErrorString(ec);
      return KG_ECUDA;
    }
    (void)l0;
  }
  for (int s = 0; s < nsteps; ++s) {
    KG_BCK(cudaGraphLaunch(b->graph, b->stream));
    b->launches += b->graph_launches;
    for (kg_solver* h : b->members) h->t = h->t + h->dt;
  }
  // members' later work waits for the batch
  KG_BCK(cudaEventRecord(b->ev, b->stream));
  for (kg_solver* h : b->members) KG_BCK(cudaStreamWaitEvent(h->stream, b->ev, 0));
  return KG_OK;
}

// proyector_detectors (MoL/diagnostic_lib.f90:231-250) of every member, enqueued
// on the batch stream behind its steps, with one synchronisation for all of
// them: host_alm receives the members' a_lm(n_det, -L:L, 0:L) blocks in member
// order (zeros for detectors outside the grid).
long long kg_batch_alm_count(const kg_batch* b) {
  if (!b) return -1;
  long long total = 0;
  for (kg_solver* h : b->members) total += (long long)(h->L + 1) * (2 * h->L + 1) * h->n_det;
  return total;
}

int kg_batch_proyector_detectors(kg_batch* b, double* host_alm) {
  if (!b || !host_alm) return KG_EINVAL;
  size_t total = 0;
  for (kg_solver* h : b->members) total += (size_t)(h->L + 1) * (2 * h->L + 1) * h->n_det;
  if (total == 0) return KG_OK;
  if (total > b->pin_cap) {
    if (b->pin) cudaFreeHost(b->pin);
    b->pin = nullptr;
    b->pin_cap = 0;
    KG_BCK(cudaMallocHost((void**)&b->pin, 2 * total * sizeof(double2)));
    b->pin_cap = 2 * total;
  }
  for (kg_solver* h : b->members) {
    KG_BCK(cudaEventRecord(b->ev, h->stream));
    KG_BCK(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  size_t off = 0;
  for (kg_solver* h : b->members) {
    const size_t n = (size_t)(h->L + 1) * (2 * h->L + 1) * h->n_det;
    kg::launch_shell_interp(h->g, metric_of(h), h->U, h->si, h->n_det, h->Ny, h->Nz, 1, h->shells, b->stream);
    kg::launch_project(h->shells, h->si.active, h->n_det, h->L, h->Ny, h->Nz, h->normP, h->cosm, h->sinm, h->sint,
                       h->dy * h->dz, h->alm, b->stream);
    KG_BCK(cudaMemcpyAsync(b->pin + off, h->alm, n * sizeof(double2), cudaMemcpyDeviceToHost, b->stream));
    off += n;
  }
  b->launches += 2 * (long long)b->members.size();
  KG_BCK(cudaGetLastError());
  KG_BCK(cudaStreamSynchronize(b->stream));
  off = 0;
  for (kg_solver* h : b->members) {
    const size_t per = (size_t)(h->L + 1) * (2 * h->L + 1);
    for (int d = 0; d < h->n_det; ++d) {
      double2* dst = reinterpret_cast<double2*>(host_alm) + off + per * d;
      if (h->active[d]) memcpy(dst, b->pin + off + per * d, per * sizeof(double2));
      else memset(dst, 0, per * sizeof(double2));
    }
    off += per * h->n_det;
  }
  return KG_OK;
}

int kg_batch_synchronize(kg_batch* b) {
  if (!b) return KG_EINVAL;
  KG_BCK(cudaStreamSynchronize(b->stream));
  int f = 0;
  KG_BCK(cudaMemcpyAsync(&f, b->derr, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  KG_BCK(cudaStreamSynchronize(b->stream));
  if (f) {
    b->err = "a device wait ran out in a batched launch";
    return KG_ETIMEOUT;
  }
  return KG_OK;
}

int kg_batch_set_tuning(kg_batch* b, int kchunk, int blocks) {
  if (!b || kchunk < 1 || blocks < 1) return KG_EINVAL;
  if (kchunk != b->kchunk || blocks != b->blocks) {
    b->kchunk = kchunk;
    b->blocks = blocks;
    b->dirty = true;
  }
  return KG_OK;
}

int kg_batch_set_precision(kg_batch* b, int mode) {
  if (!b || mode < 0 || mode > 1) return KG_EINVAL;
  if (mode == b->precision) return KG_OK;
  KG_BCK(cudaStreamSynchronize(b->stream));
  for (kg_solver* h : b->members) {
    const int rc = mode == 1 ? ensure_mixed(h) : ensure(h, &h->RK, 15);
    if (rc) {
      b->err = "could not allocate stage buffers of a member: " + h->err;
      return rc;
    }
  }
  b->precision = mode;
  b->dirty = true;
  return KG_OK;
}

int kg_batch_set_dispatch(kg_batch* b, int dispatch, int variant) {
  if (!b || dispatch < 0 || dispatch > 1 || variant < -1 || variant > 3) return KG_EINVAL;
  if (dispatch == 1 && b->precision == 1 && variant >= 0 && variant < 2) {
    b->err = "the mixed-precision stages have the TMA form only (variant 2, 3 or -1)";
    return KG_EINVAL;
  }
  b->dispatch = dispatch;
  b->variant = variant;
  return KG_OK;
}

int kg_batch_set_tile_rows(kg_batch* b, int rows) {
  if (!b || (rows != 4 && rows != 8)) return KG_EINVAL;
  if (rows != b->tile_rows) {
    b->tile_rows = rows;
    b->dirty = true;  // the work items and their tensor maps depend on the tile
  }
  return KG_OK;
}

int kg_batch_get_tile_rows(const kg_batch* b, int* rows) {
  if (!b || !rows) return KG_EINVAL;
  *rows = b->tile_rows;
  return KG_OK;
}

int kg_batch_get_dispatch(const kg_batch* b, int* dispatch, int* variant) {
  if (!b) return KG_EINVAL;
  if (dispatch) *dispatch = b->dispatch;
  if (variant) *variant = b->variant;
  return KG_OK;
}

int kg_batch_get_tuning(const kg_batch* b, int* kchunk, int* blocks) {
  if (!b) return KG_EINVAL;
  if (kchunk) *kchunk = b->kchunk;
  if (blocks) *blocks = b->blocks;
  return KG_OK;
}

long long kg_batch_launch_count(const kg_batch* b) { return b ? b->launches : 0; }

void* kg_batch_get_stream(const kg_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"

// =============================================================================
// Berger-Oliger hierarchy: radially nested 2:1 levels (kg_refine.cu), each a
// full solver handle on [xmin, r_l] with dx_l = dx_0 / 2^l and dt_l = dt_0 / 2^l.
// One coarse step: level 0 takes an RK4 step; every finer level takes two
// steps per step of its parent, its outermost planes following the parent in
// space and time; then it is restricted onto the parent.
struct kg_hier {
  std::vector<kg_solver*> lv;
  std::vector<double2*> uold;  // state of each non-finest level at the start of its current step
  std::vector<cudaEvent_t> ev;
  int nbuf = 4, keep_out = 8;
  long long coarse_steps = 0;
  std::string err;
};

namespace {
int hier_order(kg_hier* H, kg_solver* from, kg_solver* to, int l) {
  if (cudaEventRecord(H->ev[l], from->stream) != cudaSuccess ||
      cudaStreamWaitEvent(to->stream, H->ev[l], 0) != cudaSuccess) {
    H->err = "stream ordering between levels failed";
    return KG_ECUDA;
  }
  return KG_OK;
}

// method: 3 = SSP-RK3, 4 = RK4, 12 = PIRK2, 13 = PIRK3 on every level
int hier_step(kg_hier* H, int l, double a0, double da, int method) {
  kg_solver* h = H->lv[l];
  const int n = (int)H->lv.size();
  int rc;
  if (l + 1 < n) {
    if (cudaMemcpyAsync(H->uold[l], h->U, 5 * field_bytes(h), cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess) {
      H->err = "level state copy failed";
      return KG_ECUDA;
    }
  }
  if (l == 0)
    rc = method == 3 ? step_rk3(h, 1) : method == 4 ? step_rk4(h, 1) : method == 12 ? step_pirk2(h, 1)
                                                                              : step_pirk3(h, 1);
  else if (method == 3) rc = step_rk3_bo(h, H->lv[l - 1], H->uold[l - 1], a0, da, H->nbuf);
  else if (method == 4) rc = step_rk4_bo(h, H->lv[l - 1], H->uold[l - 1], a0, da, H->nbuf);
  else rc = step_pirk_bo(h, H->lv[l - 1], H->uold[l - 1], a0, da, H->nbuf, method == 12 ? 2 : 3);
  if (rc) {
    H->err = h->err;
    return rc;
  }
  if (l + 1 < n) {
    kg_solver* f = H->lv[l + 1];
    if ((rc = hier_order(H, h, f, l))) return rc;
    for (int sub = 0; sub < 2; ++sub)
      if ((rc = hier_step(H, l + 1, 0.5 * sub, 0.5, method))) return rc;
    if ((rc = hier_order(H, f, h, l))) return rc;
    Prof pf(h, PK_RESTRICT, 1);
    if (kg::launch_restrict(h->g, h->U, f->g, f->U, H->keep_out, h->stream)) {
      H->err = "restriction does not fit";
      return KG_EINVAL;
    }
  }
  return KG_OK;
}
}  // namespace

extern "C" {

int kg_hier_create(const kg_params* base, int nlevels, const double* r_fine, int device, kg_hier** out) {
  if (!base || !out || nlevels < 1 || nlevels > 8 || (nlevels > 1 && !r_fine)) return KG_EINVAL;
  *out = nullptr;
  kg_hier* H = new kg_hier();
  kg_solver* h0 = nullptr;
  int rc = kg_create(base, device, &h0);
  if (rc) {
    delete H;
    return rc;
  }
  H->lv.push_back(h0);
  const double dt0 = h0->dt, dx0 = h0->dx;
  for (int l = 1; l < nlevels; ++l) {
    kg_params p = *base;
    const double dxl = dx0 / (double)(1 << l);
    const int nx = (int)((r_fine[l - 1] - base->xmin) / dxl);
    kg_solver* parent = H->lv[l - 1];
    if (nx < 8 || (nx + 2 * p.g_pts + 1 - 1) / 2 + 2 > parent->NI - 1) {
      H->err = "refined level " + std::to_string(l) + " must lie inside its parent and hold at least 8 cells";
      kg_hier_destroy(H);
      return KG_EINVAL;
    }
    p.Nx = nx;
    p.xmax = base->xmin + (double)nx * dxl;
    p.dt_override = dt0 / (double)(1 << l);
    p.bc_rmax = KG_OUTFLOW;
    kg_solver* hl = nullptr;
    if ((rc = kg_create(&p, device, &hl))) {
      H->err = "creating refined level failed";
      kg_hier_destroy(H);
      return rc;
    }
    H->lv.push_back(hl);
  }
  for (int l = 0; l + 1 < nlevels; ++l) {
    double2* b = nullptr;
    if ((rc = dalloc(H->lv[l], (void**)&b, 5 * field_bytes(H->lv[l])))) {
      H->err = "allocating level copies failed";
      kg_hier_destroy(H);
      return rc;
    }
    H->uold.push_back(b);
  }
  for (kg_solver* h : H->lv)  // the level copies exist before any level's stream uses them
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
      H->err = "allocating level copies failed";
      kg_hier_destroy(H);
      return KG_ECUDA;
    }
  H->ev.resize(nlevels);
  for (auto& e : H->ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  *out = H;
  return KG_OK;
}

int kg_hier_destroy(kg_hier* H) {
  if (!H) return KG_EINVAL;
  for (kg_solver* h : H->lv)
    if (h) cudaStreamSynchronize(h->stream);
  for (size_t l = 0; l < H->uold.size(); ++l) dfree(H->lv[l], H->uold[l]);
  for (auto e : H->ev)
    if (e) cudaEventDestroy(e);
  for (kg_solver* h : H->lv)
    if (h) kg_destroy(h);
  delete H;
  return KG_OK;
}

const char* kg_hier_last_error(const kg_hier* H) { return H ? H->err.c_str() : "null hierarchy"; }

int kg_hier_levels(const kg_hier* H) { return H ? (int)H->lv.size() : 0; }

kg_solver* kg_hier_level(kg_hier* H, int l) {
  return (H && l >= 0 && l < (int)H->lv.size()) ? H->lv[l] : nullptr;
}

// nsteps coarse steps of RK4 (MoL/lines_method_lib.f90:411-474) on every level
namespace {
int hier_run(kg_hier* H, int nsteps, int method) {
  if (!H || nsteps < 0) return KG_EINVAL;
  for (kg_solver* h : H->lv)
    if (h->scheme != 0 || h->precision != 0) {
      H->err = "the hierarchy steps the reference FP64 scheme";
      return KG_EINVAL;
    }
  for (int s = 0; s < nsteps; ++s) {
    const int rc = hier_step(H, 0, 0.0, 1.0, method);
    if (rc) return rc;
    H->coarse_steps++;
  }
  return KG_OK;
}
}  // namespace

int kg_hier_rk4(kg_hier* H, int nsteps) { return hier_run(H, nsteps, 4); }
int kg_hier_rk3(kg_hier* H, int nsteps) { return hier_run(H, nsteps, 3); }
int kg_hier_pirk2(kg_hier* H, int nsteps) { return hier_run(H, nsteps, 12); }
int kg_hier_pirk3(kg_hier* H, int nsteps) { return hier_run(H, nsteps, 13); }

int kg_hier_synchronize(kg_hier* H) {
  if (!H) return KG_EINVAL;
  for (kg_solver* h : H->lv) {
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
      H->err = "synchronize failed";
      return KG_ECUDA;
    }
    const int rc = check_device_flag(h);
    if (rc) {
      H->err = h->err;
      return rc;
    }
  }
  return KG_OK;
}

}  // extern "C"

