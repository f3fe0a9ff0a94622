// kg_refine.cu -- Berger-Oliger transfer operators between radially nested
// levels (2:1 in r and t; the reference's mesh_refinement_lib.f90 builds a
// single uniform level, MoL/mesh_refinement_lib.f90:100-147, so refinement is
// new here).  A fine level covers [xmin, r_l] with dx_l = dx_{l-1} / 2; fine
// point ii_f sits on coarse point ii_f / 2 when ii_f is even (both grids start
// at xmin).
//   prolongation: the outermost `nbuf` fine planes take coarse values at the
//     stage time, cubic Lagrange in r, (-c(a-1) + 9 c(a) + 9 c(a+1) - c(a+2)) / 16
//     at the odd (midpoint) planes, injection at the even ones, and linear in
//     time between the coarse level's states at t and t + dt_coarse (the Pi
//     variable may live in a separate slot, as the PIRK stage arrays keep it);
//   restriction: every coarse point under the fine level's interior (all but
//     the last `keep_out` fine planes) takes the coincident fine value.
#include <cuda_runtime.h>
#include "kg_device.cuh"
#include "kg_internal.h"

namespace kg {
namespace {

__device__ __forceinline__ double2 prolong_r(const Grid& gc, const double2* c, int iif, int jj, int k) {
  if ((iif & 1) == 0) return c[off3(gc, iif >> 1, jj, k)];
  const int a = iif >> 1;
  const double2 cm = c[off3(gc, a - 1, jj, k)], c0 = c[off3(gc, a, jj, k)], c1 = c[off3(gc, a + 1, jj, k)],
                c2v = c[off3(gc, a + 2, jj, k)];
  return rmul(1.0 / 16.0, csub(cadd(cadd(cneg(cm), rmul(9.0, c0)), rmul(9.0, c1)), c2v));
}

__global__ void prolong_kernel(Grid gf, double2* uf, double2* uf_pi, Grid gc, const double2* c_old,
                               const double2* c_new, double alpha, int nbuf) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)nbuf * gf.NJ * gf.NK;
  if (t >= n) return;
  const int b = (int)(t % nbuf);
  const long long r = t / nbuf;
  const int jj = (int)(r % gf.NJ), k = (int)(r / gf.NJ);
  const int iif = gf.NI - nbuf + b;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const double2 po = prolong_r(gc, c_old + (long long)v * gc.fs, iif, jj, k);
    const double2 pn = prolong_r(gc, c_new + (long long)v * gc.fs, iif, jj, k);
    double2* dst = (v == 4) ? uf_pi : uf + (long long)v * gf.fs;
    dst[off3(gf, iif, jj, k)] = cadd(rmul(1.0 - alpha, po), rmul(alpha, pn));
  }
}

__global__ void restrict_kernel(Grid gc, double2* uc, Grid gf, const double2* uf, int nc) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)nc * gc.NJ * gc.NK;
  if (t >= n) return;
  const int ic = (int)(t % nc);
  const long long r = t / nc;
  const int jj = (int)(r % gc.NJ), k = (int)(r / gc.NJ);
#pragma unroll
  for (int v = 0; v < 5; ++v)
    uc[(long long)v * gc.fs + off3(gc, ic, jj, k)] = uf[(long long)v * gf.fs + off3(gf, 2 * ic, jj, k)];
}

}  // namespace

int launch_prolong(const Grid& gf, double2* uf, const Grid& gc, const double2* c_old, const double2* c_new,
                   double alpha, int nbuf, cudaStream_t st, double2* uf_pi) {
  // the stencil reaches coarse plane (NI_f - 1) / 2 + 2, which must lie inside the coarse grid
  if (nbuf < 1 || nbuf > gf.NI || gf.NJ != gc.NJ || gf.NK != gc.NK || (gf.NI - 1) / 2 + 2 > gc.NI - 1 ||
      (gf.NI - nbuf) / 2 - 1 < 0)
    return -1;
  const long long n = (long long)nbuf * gf.NJ * gf.NK;
  if (!uf_pi) uf_pi = uf + 4 * gf.fs;
  prolong_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(gf, uf, uf_pi, gc, c_old, c_new, alpha, nbuf);
  return 0;
}

int launch_restrict(const Grid& gc, double2* uc, const Grid& gf, const double2* uf, int keep_out, cudaStream_t st) {
  const int last_f = gf.NI - 1 - keep_out;  // last fine plane taken
  const int nc = last_f / 2 + 1;            // coarse planes 0..nc-1
  if (nc < 1 || nc > gc.NI || gf.NJ != gc.NJ || gf.NK != gc.NK) return -1;
  const long long n = (long long)nc * gc.NJ * gc.NK;
  restrict_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(gc, uc, gf, uf, nc);
  return 0;
}

}  // namespace kg
