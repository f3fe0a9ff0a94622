// kg_diag.h -- detector-shell tables and launchers of kg_diag.cu
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "kg_device.cuh"

namespace kg {

// Interpolation tables of domain_to_sph (tools/FFT_sph.f90:525-651) for the
// detector shells, all device pointers.  Per detector: evolution-grid r index
// (0-based ii) and weight; per vertex theta index jv: jj index, weight and a
// pole flag (1: copy row 0, 2: copy row NJ-1); per vertex phi index kv: k
// index and weight.
struct ShellInterp {
  const int* active;   // [n_det] detector inside the grid
  const int* i_r;      // [n_det]
  const double* w_r;   // [n_det]
  const int* i_th;     // [Ny]
  const double* w_th;  // [Ny]
  const int* th_flag;  // [Ny]
  const int* i_ph;     // [Nz]
  const double* w_ph;  // [Nz]
};

void launch_shell_interp(const Grid& g, const Metric& m, const double2* u, const ShellInterp& si, int n_det, int Ny,
                         int Nz, int which_mask, double2* out, cudaStream_t st);
void launch_flux(const double2* shells, const int* active, int n_det, int Ny, int Nz, double dydz, double* out,
                 cudaStream_t st);
void launch_project(const double2* shells, const int* active, int n_det, int L, int Ny, int Nz, const double* normP,
                    const double* cosm, const double* sinm, const double* sint, double dydz, double2* alm,
                    cudaStream_t st);

// all-shell Y_lm projection (kg_ylm_gemm.cu)
}  // namespace kg
#include <cuda_bf16.h>
namespace kg {
int launch_ylm_gemm(const __nv_bfloat16* Ahi, const __nv_bfloat16* Alo, const __nv_bfloat16* Bhi,
                    const __nv_bfloat16* Blo, float* C, int Mp, int Np, int Kp, int* err, cudaStream_t st);
void launch_shells_to_a(const Grid& g, const double2* u, const ShellInterp& si, int Nx, int Ny, int Nz, int Kp,
                        __nv_bfloat16* Ahi, __nv_bfloat16* Alo, double2* F, cudaStream_t st);
void launch_ylm_b(int L, int Ny, int Nz, int Kp, const double* normP, const double* cosm, const double* sinm,
                  const double* sint, __nv_bfloat16* Bhi, __nv_bfloat16* Blo, cudaStream_t st);
void launch_ylm_assemble(const float* C, int ldc, long long csplit, int nsplit, int Nx, int L, double dydz,
                         double2* alm, cudaStream_t st);
void launch_ylm_fp64(const double2* F, int Nx, int L, int Ny, int Nz, const double* normP, const double* cosm,
                     const double* sinm, const double* sint, double dydz, double2* alm, cudaStream_t st);

// spherical-Bessel radial basis and transform (kg_radial.cu)
double sph_jl(int l, double x);
void sph_jl_zeros(int L, int Nk, std::vector<double>& z);
void bessel_basis(int L, int Nk, int Nx, double xmin, double dx, double r_max, std::vector<double>& k_values,
                  std::vector<double>& basis);
void launch_radial_ft(const double2* flm, const double* jr, int L, int Nk, int Nx, double dr, double2* ft,
                      cudaStream_t st);
}  // namespace kg
