// kg_internal.h -- declarations shared by the translation units of
// libkg_b200.so (not part of the public C ABI).
#pragma once
#include <cuda_runtime.h>
#include "kg_device.cuh"

namespace kg {

// stage kinds of the fused RHS + combination kernel
enum StageKind {
  ST_P2_S1A = 0,  // PIRK stage 1, phi/psi part:   S(1:4) = u + dt*rhs(u)
  ST_P2_S1B,      // PIRK stage 1, Pi part:        S(5)   = u(5) + dt*rhs_pi(S)
  ST_P2_S2,       // PIRK2 stage 2:                u = 0.5*(u_p + S + dt*rhs(S))
  ST_P3_S2A,      // PIRK3 stage 2, phi/psi part:  T(1:4) = 0.75 u_p + 0.25 (S + dt rhs(S))
  ST_P3_S2B,      // PIRK3 stage 2, Pi part:       T(5)   = 0.75 u_p + 0.25 (S(5) + dt rhs_pi(T))
  ST_P3_S3,       // PIRK3 stage 3:                u = 1/3 u_p + 2/3 (T + dt rhs(T))
  ST_RK3_1,       // RK3 stage 1:                  S = u_p + rhs*dt
  ST_RK3_2,       // RK3 stage 2:                  S' = 0.75 u_p + 0.25 (S + rhs*dt)
  ST_RK3_3,       // RK3 stage 3:                  u = u_p/3 + 2 (S' + rhs*dt)/3
  ST_RK4_1,       // RK4 stages: k = rhs*dt, accumulator k1 + 2k2 + 2k3
  ST_RK4_2,
  ST_RK4_3,
  ST_RK4_4
};

struct StageLaunch {
  Grid g;
  Metric m;
  int metric_kind;
  const double2* in[5];
  const double2* base;
  const double2* aux4;
  double2* out;
  double2* out4;
  double2* acc;
  int skip_last_i;
};

void launch_stage(int kind, const StageLaunch& L, cudaStream_t st);
// 2.5-D marching form of the same kernels (kg_march.cu); rsg = 1/sqrt(gamma) table
void launch_stage_march(int kind, const StageLaunch& L, const double* rsg, cudaStream_t st);
// TMA-pipelined form (kg_tma.cu); err: device flag set to 1 when a bounded wait runs out;
// tj: theta rows of a tile, 8, or 4 for the RK4 stages (other kinds run 8).
// Returns 0, or -1 if the tensor maps cannot be encoded / the kernel cannot be configured.
int launch_stage_tma(int kind, const StageLaunch& L, const double* rsg, int* err, cudaStream_t st, int tj = 8);
// PIRK stage 1 in one kernel (kg_fused.cu): S(1:4) = u + dt rhs(u), Snew = u(5) +
// dt rhs_pi(S(1:4), Sold).  Returns -1 if the tensor maps cannot be encoded.
int launch_pirk_s1_fused(const Grid& g, const Metric& m, int mk, const double2* U, const double2* Sold, double2* S,
                         double2* Snew, const double* rsg, int* err, cudaStream_t st);
// one warp waits at most `polls` polls on an mbarrier phase that never completes,
// then sets *err (the failure path of every bounded wait); returns -1 if the launch fails
int launch_wait_check(int* err, long long polls, cudaStream_t st);
// true when the driver can encode the tensor maps the TMA form needs for this grid
bool tma_available(const Grid& g, const double2* some_state);
// batched (multi-solve) persistent launches of the TMA stage kernel
size_t batch_item_bytes();
int build_batch_item(void* dst, int kind, const StageLaunch& L, const double* rsg, int* err, int kchunk, int item0,
                     int tj);
int launch_batch_tma(int kind, int mk, const void* d_items, int n_solves, int n_items, int blocks, int tj,
                     cudaStream_t st);
// Y_lm projection over all shells (kg_ylm_gemm.cu)
int ylm_gemm_pad_m(int rows);
int ylm_gemm_pad_n(int cols);
int ylm_gemm_pad_k(int k);
int ylm_gemm_splits(int Kp);  // K ranges of the split-K GEMM (FP32 partial tiles added in FP64)
// batched ghost fill: one launch pair for many solves
struct GhostDesc {
  Grid g;
  double2* u;
  const double2* up;
  int inflow;
};
void launch_ghost_fill_batch(const GhostDesc* d_desc, int n, long long max_rows, long long max_faces,
                             long long max_zplanes, cudaStream_t st);
// mixed-precision RK4 (kg_mixed.cu): FP32 stage states and increment sum, FP64 u
struct MixedLaunch {
  Grid g;
  Metric m;
  int metric_kind;
  const float2* in_f;    // stage input of stages 2-4 (5 variables, stride g.fs)
  const double2* base;   // u^n; the stencil input of stage 1
  float2* acc;           // k1 + 2 k2 + 2 k3
  float2* out_f;         // stage output of stages 1-3
  double2* out_d;        // u^{n+1} (stage 4)
  int skip_last_i;
};
// tj: theta rows of a tile, 8 or 4 (other values: 8 for a single solve, an error for a batch)
int launch_stage_mixed(int kind, const MixedLaunch& L, const double* rsg, int* err, cudaStream_t st, int tj = 8);
size_t mixed_item_bytes();
int build_mixed_item(void* dst, int kind, const MixedLaunch& L, const double* rsg, int* err, int kchunk, int item0,
                     int tj);
int launch_batch_mixed(int kind, int mk, const void* d_items, int n_solves, int n_items, int blocks, int tj,
                       cudaStream_t st);
size_t ghost_f32_desc_bytes();
void fill_ghost_f32_desc(void* dst, const Grid& g, float2* u, const double2* up, int inflow);
void launch_ghost_fill_f32(const void* d_desc, int n, long long max_rows, long long max_faces, long long max_z,
                           cudaStream_t st);
// configured method (kg_config.cu): RK4 stage with fourth-order differences,
// Kreiss-Oliger dissipation and a Sommerfeld outer plane; coef = 1/(12 h) for
// r, theta, phi then eps/(64 h) for r, theta, phi; rN = outermost r; rsg = the
// 1/sqrt(gamma) table; tiled = 1 for the shared-memory tiled marching form, 0 for
// one thread per point (same bits)
int launch_stage_cfg(int kind, const StageLaunch& L, const double* dxbeta4, const double* rsg, const double coef[6],
                     double rN, int tiled, cudaStream_t st);
void launch_ghost_fill_cfg(const Grid& g, double2* u, cudaStream_t st);
// Berger-Oliger transfers between radially nested 2:1 levels (kg_refine.cu)
// uf_pi: where the fine Pi variable lives (nullptr: uf + 4 fs, the 5-variable layout)
int launch_prolong(const Grid& gf, double2* uf, const Grid& gc, const double2* c_old, const double2* c_new,
                   double alpha, int nbuf, cudaStream_t st, double2* uf_pi = nullptr);
int launch_restrict(const Grid& gc, double2* uc, const Grid& gf, const double2* uf, int keep_out, cudaStream_t st);
void launch_rhs(const Grid& g, const Metric& m, int metric_kind, const double2* const in[5], double2* out,
                unsigned mask, cudaStream_t st);

// boundary fills on a 5-variable state u; up = u_p (inflow source)
void launch_ghost_fill(const Grid& g, double2* u, const double2* up, int inflow, cudaStream_t st);
void launch_face(const Grid& g, double2* u, const double2* up, int inflow, int face, cudaStream_t st);

// layout conversion between the Fortran AoS layout and the device planes,
// for planes [k0, k1) of all 5 variables; aos points at plane k0
void launch_aos_to_soa(const Grid& g, const double2* aos, double2* soa, int k0, int k1, cudaStream_t st);
void launch_soa_to_aos(const Grid& g, const double2* soa, double2* aos, int k0, int k1, cudaStream_t st);

// diagnostics
struct ShellInterp;  // per-detector interpolation tables (kg_diag.cu)
void launch_density(const Grid& g, const Metric& m, const double2* u, double mass2, double* rho, cudaStream_t st);
// trapezium integral of rho*sqrtg over i in [0,Nx], j in [0,Ny], k in [0,Nz];
// partial sums in `partials` (>= nblocks doubles), result in *out (device)
int mass_blocks(const Grid& g);
void launch_mass(const Grid& g, const Metric& m, const double* rho, double dxdydz, double* partials,
                 double* out, cudaStream_t st);

}  // namespace kg
