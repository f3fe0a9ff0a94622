// kg_device.cuh -- device-side layout, complex helpers and the second-order
// stencils of the reference (tools/finite_differences.f90), shared by the
// stage, boundary and diagnostic kernels.
//
// Device layout (HBM): each variable is a 3-D array of double2 (re, im),
// indexed [k][jj][ii] with ii = i + g (r, fastest, rows padded to `PI`
// elements so every row starts on a 128-byte boundary), jj = j + g (theta)
// and k = 0..Nz (phi).  A state is 5 such arrays; `fs` is the distance
// between variables.  The metric is phi-independent, so every metric
// quantity is a 2-D [jj][ii] table of doubles with the same row pitch.
//
// All arithmetic keeps the reference's order of operations, complex-by-real
// products and quotients component-wise, and the translation unit is built
// with --fmad=false, so each FP64 result is rounded exactly as the reference's
// x86-64 build rounds it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace kg {

struct Grid {
  int NI, NJ, NK;      // stored extents: Nx+2g+1, Ny+2g+1, Nz+1
  int PI;              // row pitch in elements
  long long plane;     // NJ * PI
  long long fs;        // NK * plane (distance between variables)
  int Nz, dis, Nzm1;   // reference Nz, Nz/2, Nz-1
  double rdx, rdy, rdz;  // 0.5/dx, 0.5/dy, 0.5/dz
  double dt;
};

// 2-D metric tables, [jj][ii] with pitch PI
struct Metric {
  const double* alpha;    // alpha
  const double* beta;     // beta^r
  const double* dxbeta;   // d_r beta^r
  const double* sqrtg;    // sqrt(gamma)
  const double* asg;      // alpha*sqrtg
  const double* grr;      // gamma^rr
  const double* grp;      // gamma^rphi
  const double* gpp;      // gamma^phph
  const double* asg_gtt;  // (alpha*sqrtg)*gamma^thth
  const double* asg_grr;  // (alpha*sqrtg)*gamma^rr   (Schw_EF form)
  const double* a_gpp;    // alpha*gamma^phph        (Schw_EF form)
  const double* am2;      // alpha*m**2
  const double* gtt;      // gamma^thth
};

enum MetricKind { MK_KS = 0, MK_SCHW = 1 };

// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 c2(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return c2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return c2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cneg(double2 a) { return c2(-a.x, -a.y); }
__device__ __forceinline__ double2 rmul(double s, double2 a) { return c2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 cdivr(double2 a, double s) { return c2(a.x / s, a.y / s); }

__device__ __forceinline__ long long off3(const Grid& g, int ii, int jj, int k) {
  return (long long)k * g.plane + (long long)jj * g.PI + ii;
}
__device__ __forceinline__ int off2(const Grid& g, int ii, int jj) { return jj * g.PI + ii; }

__device__ __forceinline__ double2 ldf(const double2* __restrict__ f, long long o) { return __ldg(f + o); }
__device__ __forceinline__ double ldm(const double* __restrict__ t, int o) { return __ldg(t + o); }

// one-sided and centred building blocks, written exactly as the Fortran
// statements group them: (-3f0 + 4f1 - f2), (3f0 - 4f1 + f2), (-fm + fp)
__device__ __forceinline__ double2 fwd3(double2 f0, double2 f1, double2 f2) {
  return csub(cadd(cneg(rmul(3.0, f0)), rmul(4.0, f1)), f2);
}
__device__ __forceinline__ double2 bwd3(double2 f0, double2 fm1, double2 fm2) {
  return cadd(csub(rmul(3.0, f0), rmul(4.0, fm1)), fm2);
}
__device__ __forceinline__ double2 ctr(double2 fm, double2 fp) { return cadd(cneg(fm), fp); }

// phi partner of the pole fill and of the theta pole stencil
__device__ __forceinline__ int ktarget(const Grid& g, int k) { return (k + g.dis) % g.Nzm1; }

// ---------------------------------------------------------------------------
// Generic second-order operators on a "point function" F(ii, jj, k) -> double2.
// first_derivative_x_2_uniform (finite_differences.f90:17-44)
template <class F>
__device__ __forceinline__ double2 op_dr(const Grid& g, const F& f, int ii, int jj, int k) {
  double2 v;
  if (ii == 0) v = fwd3(f(0, jj, k), f(1, jj, k), f(2, jj, k));
  else if (ii == g.NI - 1) v = bwd3(f(ii, jj, k), f(ii - 1, jj, k), f(ii - 2, jj, k));
  else v = ctr(f(ii - 1, jj, k), f(ii + 1, jj, k));
  return rmul(g.rdx, v);  // (..) * res
}
// advec_x_uniform (finite_differences.f90:767-801); beta at (ii, jj)
template <class F>
__device__ __forceinline__ double2 op_ar(const Grid& g, const F& f, double beta, int ii, int jj, int k) {
  double2 v;
  const int n = g.NI - 1;
  if (ii <= 1) v = fwd3(f(ii, jj, k), f(ii + 1, jj, k), f(ii + 2, jj, k));
  else if (ii == n - 1) v = csub(f(n, jj, k), f(n - 2, jj, k));
  else if (ii == n) v = bwd3(f(n, jj, k), f(n - 1, jj, k), f(n - 2, jj, k));
  else if (beta > 0.0) v = fwd3(f(ii, jj, k), f(ii + 1, jj, k), f(ii + 2, jj, k));
  else if (beta < 0.0) v = bwd3(f(ii, jj, k), f(ii - 1, jj, k), f(ii - 2, jj, k));
  else v = csub(f(ii + 1, jj, k), f(ii - 1, jj, k));
  return rmul(g.rdx, v);
}
// first_derivative_y_2 with inpar = .false. (finite_differences.f90:193-239)
template <class F>
__device__ __forceinline__ double2 op_dth(const Grid& g, const F& f, int ii, int jj, int k) {
  double2 v;
  if (jj == 0) v = cadd(cneg(f(ii, 1, k)), f(ii, 2, ktarget(g, k)));
  else if (jj == g.NJ - 1) v = bwd3(f(ii, jj, k), f(ii, jj - 1, k), f(ii, jj - 2, k));
  else v = ctr(f(ii, jj - 1, k), f(ii, jj + 1, k));
  return rmul(g.rdy, v);
}
// first_derivative_z_2 (finite_differences.f90:310-338)
template <class F>
__device__ __forceinline__ double2 op_dph(const Grid& g, const F& f, int ii, int jj, int k) {
  double2 v;
  if (k == 0) v = cadd(cneg(f(ii, jj, g.Nz - 2)), f(ii, jj, 1));
  else if (k == g.Nz) v = cadd(cneg(f(ii, jj, 2)), f(ii, jj, g.Nz - 1));
  else v = ctr(f(ii, jj, k - 1), f(ii, jj, k + 1));
  return rmul(g.rdz, v);
}

}  // namespace kg
