// kg_noalloc.cu -- the mass integral for callers that cannot allocate device
// memory.
//
// kg_mass_scalar() reduces into partial sums that live in device memory owned
// by a solver handle, and the handle itself is created with cudaMalloc.  Some
// callers cannot do that: a host whose device memory is all owned by its own
// pool allocator or already committed to live solves under a fixed budget, or
// one that must not take the device-wide synchronisation cudaMalloc and
// cudaFree imply in the middle of its time loop.  kg_integrate_mass_noalloc()
// gives them the same diagnostic with no allocation at all: the caller passes
// the density, the sqrt(gamma) table and an output slot, all in its own device
// memory, and the intermediate sums go to one file-scope __device__ array.
//
// The reduction follows the reference's nested trapezium exactly
// (tools/integral.f90:220-255 via integrate, :646-674): first along phi for
// every (r, theta) column, then along theta, then along r, each as the
// reference's sequential (acc + f(i)) + f(i+1) sum scaled by 0.5*h, so its
// result is the reference's Mass_scalar bit for bit for the same rho.
//
// Limits and sharing:
//   * the scratch holds KG_NOALLOC_MAX_DOUBLES doubles (4 MiB); a call needs
//     (Nx+1)*(Ny+1) + (Nx+1) of them and is rejected with KG_EINVAL and a
//     message from kg_last_error(NULL) when that is more;
//   * every GPU that loads the library keeps this array until the process
//     exits;
//   * all calls share the array and it keeps the last call's contents; each
//     call overwrites every entry it reads before reading it, so nothing has
//     to start at zero, but two calls whose work overlaps on the GPU (for
//     example on two streams without ordering between them) race on it;
//   * the device address of the array is looked up with cudaGetSymbolAddress
//     the first time the entry point runs on a device (with that device
//     current); make that first call before any stream capture begins.
#include <cuda_runtime.h>
#include <mutex>
#include <string>

#include "../../include/kg_capi.h"

namespace {

constexpr size_t KG_NOALLOC_MAX_DOUBLES = (size_t)1 << 19;

__device__ __align__(256) double g_noalloc_scratch[KG_NOALLOC_MAX_DOUBLES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// f2d(a, b) = 0.5 dz sum_k (f(k) + f(k+1)),  f = rho * sqrtg at i = a, j = b;
// one thread per (a, b) column on a 1-D grid (a fastest, so loads coalesce along r)
__global__ void noalloc_phi_sum(const double* __restrict__ rho, const double* __restrict__ sqrtg, int Nx, int Ny,
                                int Nz, double dz, double* __restrict__ f2d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)(Nx + 1) * (Ny + 1)) return;
  const int a = (int)(t % (Nx + 1));
  const int b = (int)(t / (Nx + 1));
  const int NI = Nx + 5, NJ = Ny + 5;
  const int ii = a + 2, jj = b + 2;
  const double sg = sqrtg[(size_t)jj * NI + ii];
  const size_t plane = (size_t)NI * NJ;
  const double* col = rho + (size_t)jj * NI + ii;
  double prev = col[0] * sg;
  double acc = 0.0;
  for (int k = 0; k < Nz; ++k) {
    const double cur = col[(size_t)(k + 1) * plane] * sg;
    acc = acc + prev;
    acc = acc + cur;
    prev = cur;
  }
  f2d[a + (size_t)(Nx + 1) * b] = 0.50 * acc * dz;
}

// f1d(a) = 0.5 dy sum_b (f2d(a, b) + f2d(a, b+1))
__global__ void noalloc_theta_sum(const double* __restrict__ f2d, int Nx, int Ny, double dy, double* __restrict__ f1d) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a > Nx) return;
  double acc = 0.0;
  for (int b = 0; b < Ny; ++b) {
    acc = acc + f2d[a + (size_t)(Nx + 1) * b];
    acc = acc + f2d[a + (size_t)(Nx + 1) * (b + 1)];
  }
  f1d[a] = 0.50 * acc * dy;
}

// out = 0.5 dx sum_a (f1d(a) + f1d(a+1))
__global__ void noalloc_r_sum(const double* __restrict__ f1d, int Nx, double dx, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double acc = 0.0;
  for (int a = 0; a < Nx; ++a) {
    acc = acc + f1d[a];
    acc = acc + f1d[a + 1];
  }
  *out = 0.50 * acc * dx;
}

thread_local std::string t_err;

}  // namespace

// message of the last handle-less call (kg_last_error(NULL))
const char* kg_noalloc_last_error() { return t_err.c_str(); }

extern "C" int kg_integrate_mass_noalloc(const double* rho_dev, const double* sqrtg_dev, int Nx, int Ny, int Nz,
                                         double dx, double dy, double dz, double* out_dev, void* stream) {
  t_err.clear();  // kg_last_error(NULL) reports this call only
  if (!rho_dev || !sqrtg_dev || !out_dev || Nx < 1 || Ny < 1 || Nz < 1) {
    t_err = "kg_integrate_mass_noalloc: null pointer or non-positive grid size";
    return KG_EINVAL;
  }
  const size_t need = (size_t)(Nx + 1) * (size_t)(Ny + 1) + (size_t)(Nx + 1);
  if (need > KG_NOALLOC_MAX_DOUBLES) {
    t_err = "kg_integrate_mass_noalloc: grid needs " + std::to_string(need) +
            " doubles of scratch ((Nx+1)*(Ny+1) + Nx+1); the static scratch holds " +
            std::to_string(KG_NOALLOC_MAX_DOUBLES);
    return KG_EINVAL;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    t_err = std::string("kg_integrate_mass_noalloc: no current device: ") + cudaGetErrorString(e);
    return KG_ENODEV;
  }
  double* scratch;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        t_err = std::string("kg_integrate_mass_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
        return KG_ECUDA;
      }
      g_scratch_ptr[dev] = (double*)p;
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  double* f2d = scratch;
  double* f1d = scratch + (size_t)(Nx + 1) * (Ny + 1);
  const unsigned cols_blocks = (unsigned)(((size_t)(Nx + 1) * (size_t)(Ny + 1) + 127) / 128);  // <= 4096
  noalloc_phi_sum<<<cols_blocks, 128, 0, st>>>(rho_dev, sqrtg_dev, Nx, Ny, Nz, dz, f2d);
  noalloc_theta_sum<<<(Nx + 1 + 127) / 128, 128, 0, st>>>(f2d, Nx, Ny, dy, f1d);
  noalloc_r_sum<<<1, 32, 0, st>>>(f1d, Nx, dx, out_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    t_err = std::string("kg_integrate_mass_noalloc: launch failed: ") + cudaGetErrorString(e);
    return KG_ECUDA;
  }
  return KG_OK;
}
