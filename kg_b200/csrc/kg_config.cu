// kg_config.cu -- the configured method (scheme 1): fourth-order centred
// differences, sixth-order Kreiss-Oliger dissipation and a Sommerfeld outer
// boundary, with RK4.  The reference wires only second-order operators (its
// fourth-order x stencil, first_derivative_x_4 in
// tools/finite_differences.f90:124-154, is real-only and never called), so this
// method is defined here and by the oracle's restatement of it, which this
// code matches bit for bit:
//   * D4 f = (f(-2) - 8 f(-1) + 8 f(+1) - f(+2)) / (12 h) in r, theta and phi;
//     in r the one-sided closures of first_derivative_x_4 on the first and last
//     two stored planes; theta on the interior rows (the +-2 rows of the first
//     and last interior rows are ghost rows); phi periodic over the Nz-1
//     distinct planes.  The shift advection term uses D4 as well, and d_r beta
//     is the D4 derivative of beta^r.
//   * + eps / (64 h) (f(-3) - 6 f(-2) + 15 f(-1) - 20 f + 15 f(+1) - 6 f(+2) + f(+3))
//     per direction on all five variables (r planes 3..N-3 only).
//   * the outermost r plane obeys d_t u = -(d_r u + u / r) (Sommerfeld); the
//     innermost planes (inside the horizon) evolve with the one-sided closures.
//   * the theta ghost rows and the duplicated phi planes get a zero RHS and are
//     refilled after every stage: the phi planes first, then the theta ghost
//     rows from the interior rows at phi + pi with psi_2 negated (the parity of
//     d_theta of a smooth function on the sphere); the theta flux
//     alpha sqrt(gamma) gamma^thth psi_2 takes the sign of sin(theta), negative
//     on the ghost rows where the table holds |sqrt(gamma)|.
// One thread per stored point; neighbours come through the read-only cache.
#include <cuda_runtime.h>
#include "kg_device.cuh"
#include "kg_internal.h"

namespace kg {
namespace {

struct CfgArgs {
  Grid g;
  Metric m;
  const double* dxb4;  // D4 d_r beta^r, [jj][ii] with pitch PI
  const double2* in;   // stage input (5 variables, stride g.fs)
  const double2* base; // u^n
  double2* acc;
  double2* out;
  double rr, rt, rp;   // 1 / (12 h) per direction
  double kr, kt, kp;   // eps / (64 h) per direction
  double rN;           // r of the outermost stored plane
};

__device__ __forceinline__ int kper(const Grid& g, int k, int d) {
  const int M = g.Nzm1;
  int kk = (k - 1 + d) % M;
  if (kk < 0) kk += M;
  return kk + 1;
}

// first_derivative_x_4 closures and centred stencil along r of a point function
template <class F>
__device__ __forceinline__ double2 d4r(const Grid& g, const F& f, int ii, double res) {
  const int n = g.NI - 1;
  double2 r;
  if (ii == 0)
    r = csub(cadd(csub(cadd(rmul(-25.0, f(0)), rmul(48.0, f(1))), rmul(36.0, f(2))), rmul(16.0, f(3))),
             rmul(3.0, f(4)));
  else if (ii == 1)
    r = cadd(csub(cadd(csub(rmul(-3.0, f(0)), rmul(10.0, f(1))), rmul(18.0, f(2))), rmul(6.0, f(3))),
             rmul(1.0, f(4)));
  else if (ii == n - 1)
    r = csub(cadd(csub(cadd(rmul(3.0, f(n)), rmul(10.0, f(n - 1))), rmul(18.0, f(n - 2))), rmul(6.0, f(n - 3))),
             rmul(1.0, f(n - 4)));
  else if (ii == n)
    r = cadd(csub(cadd(csub(rmul(25.0, f(n)), rmul(48.0, f(n - 1))), rmul(36.0, f(n - 2))), rmul(16.0, f(n - 3))),
             rmul(3.0, f(n - 4)));
  else
    r = csub(cadd(csub(f(ii - 2), rmul(8.0, f(ii - 1))), rmul(8.0, f(ii + 1))), f(ii + 2));
  return c2(r.x * res, r.y * res);
}
__device__ __forceinline__ double2 d4c(double2 m2, double2 m1, double2 p1, double2 p2, double res) {
  const double2 r = csub(cadd(csub(m2, rmul(8.0, m1)), rmul(8.0, p1)), p2);
  return c2(r.x * res, r.y * res);
}
__device__ __forceinline__ double2 ko6(double2 m3, double2 m2, double2 m1, double2 c0, double2 p1, double2 p2,
                                       double2 p3) {
  return cadd(csub(cadd(csub(cadd(csub(m3, rmul(6.0, m2)), rmul(15.0, m1)), rmul(20.0, c0)), rmul(15.0, p1)),
                   rmul(6.0, p2)),
              p3);
}
__device__ __forceinline__ double2 cdiv(double2 a, double s) { return c2(a.x / s, a.y / s); }

template <int KIND>
__global__ void __launch_bounds__(128) cfg_stage_kernel(CfgArgs a) {
  const Grid& g = a.g;
  const Metric& M = a.m;
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y;
  const int k = blockIdx.z;
  if (ii >= g.NI) return;
  const long long p = off3(g, ii, jj, k);
  const int q = off2(g, ii, jj);
  const double2* U = a.in;
  auto V = [&](int v, int i2, int j2, int k2) { return ldf(U + (long long)v * g.fs, off3(g, i2, j2, k2)); };
  double2 r[5];
  const int n = g.NI - 1;
  if (jj <= 2 || jj >= g.NJ - 3 || k == 0 || k == g.Nz) {
#pragma unroll
    for (int v = 0; v < 5; ++v) r[v] = c2(0.0, 0.0);
  } else if (ii == n) {
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      auto f = [&](int i2) { return V(v, i2, jj, k); };
      r[v] = cneg(cadd(d4r(g, f, ii, a.rr), cdiv(V(v, ii, jj, k), a.rN)));
    }
  } else {
    const double al = ldm(M.alpha, q), b1 = ldm(M.beta, q), sg = ldm(M.sqrtg, q), dxb = ldm(a.dxb4, q);
    const int km2 = kper(g, k, -2), km1 = kper(g, k, -1), kp1 = kper(g, k, 1), kp2 = kper(g, k, 2);
    auto E = [&](int i2, int j2, int k2) {
      const int q2 = off2(g, i2, j2);
      return cadd(rmul(ldm(M.alpha, q2), V(4, i2, j2, k2)), rmul(ldm(M.beta, q2), V(1, i2, j2, k2)));
    };
    auto Fp = [&](int j2, int k2) {
      const int q2 = off2(g, ii, j2);
      return rmul(ldm(M.asg, q2), cadd(rmul(ldm(M.grp, q2), V(1, ii, j2, k2)), rmul(ldm(M.gpp, q2), V(3, ii, j2, k2))));
    };
    // sqrt(gamma) carries the sign of sin(theta) through the pole: negative on the ghost rows
    auto H = [&](int j2, int k2) {
      const double2 h = rmul(ldm(M.asg_gtt, off2(g, ii, j2)), V(2, ii, j2, k2));
      return (j2 <= 2 || j2 >= g.NJ - 3) ? cneg(h) : h;
    };
    const double2 pi = V(4, ii, jj, k), ps1 = V(1, ii, jj, k);
    r[0] = cadd(rmul(al, pi), rmul(b1, ps1));
    {
      auto fA = [&](int i2) { return rmul(ldm(M.alpha, off2(g, i2, jj)), V(4, i2, jj, k)); };
      auto fP = [&](int i2) { return V(1, i2, jj, k); };
      r[1] = cadd(cadd(d4r(g, fA, ii, a.rr), rmul(b1, d4r(g, fP, ii, a.rr))), rmul(dxb, ps1));
    }
    r[2] = d4c(E(ii, jj - 2, k), E(ii, jj - 1, k), E(ii, jj + 1, k), E(ii, jj + 2, k), a.rt);
    r[3] = d4c(E(ii, jj, km2), E(ii, jj, km1), E(ii, jj, kp1), E(ii, jj, kp2), a.rp);
    {
      auto fG = [&](int i2) {
        const int q2 = off2(g, i2, jj);
        return rmul(ldm(M.asg, q2), cadd(rmul(ldm(M.grr, q2), V(1, i2, jj, k)), rmul(ldm(M.grp, q2), V(3, i2, jj, k))));
      };
      auto fQ = [&](int i2) {
        const double2 w = V(4, i2, jj, k);
        const double s2 = ldm(M.sqrtg, off2(g, i2, jj));
        return c2(w.x * s2, w.y * s2);
      };
      const double2 t1 = cdiv(d4r(g, fG, ii, a.rr), sg);
      const double2 t2 = cdiv(d4c(H(jj - 2, k), H(jj - 1, k), H(jj + 1, k), H(jj + 2, k), a.rt), sg);
      const double2 t3 = cdiv(d4c(Fp(jj, km2), Fp(jj, km1), Fp(jj, kp1), Fp(jj, kp2), a.rp), sg);
      const double2 t4 = c2(pi.x * dxb, pi.y * dxb);
      const double2 t5 = cdiv(rmul(b1, d4r(g, fQ, ii, a.rr)), sg);
      const double2 t6 = rmul(ldm(M.am2, q), V(0, ii, jj, k));
      r[4] = csub(cadd(cadd(cadd(cadd(t1, t2), t3), t4), t5), t6);
    }
    const int km3 = kper(g, k, -3), kp3 = kper(g, k, 3);
    const bool kor = ii >= 3 && ii <= n - 3;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      double2 s = r[v];
      if (kor)
        s = cadd(s, rmul(a.kr, ko6(V(v, ii - 3, jj, k), V(v, ii - 2, jj, k), V(v, ii - 1, jj, k), V(v, ii, jj, k),
                                   V(v, ii + 1, jj, k), V(v, ii + 2, jj, k), V(v, ii + 3, jj, k))));
      s = cadd(s, rmul(a.kt, ko6(V(v, ii, jj - 3, k), V(v, ii, jj - 2, k), V(v, ii, jj - 1, k), V(v, ii, jj, k),
                                 V(v, ii, jj + 1, k), V(v, ii, jj + 2, k), V(v, ii, jj + 3, k))));
      s = cadd(s, rmul(a.kp, ko6(V(v, ii, jj, km3), V(v, ii, jj, km2), V(v, ii, jj, km1), V(v, ii, jj, k),
                                 V(v, ii, jj, kp1), V(v, ii, jj, kp2), V(v, ii, jj, kp3))));
      r[v] = s;
    }
  }
  // RK4 combination, as the reference's k1..k4 form (MoL/lines_method_lib.f90:411-474)
  const double dt = g.dt;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const long long o = (long long)v * g.fs + p;
    const double2 b = ldf(a.base, o);
    const double2 kk = c2(r[v].x * dt, r[v].y * dt);
    double2 res;
    if (KIND == ST_RK4_1) {
      a.acc[o] = kk;
      res = cadd(b, rmul(0.50, kk));
    } else if (KIND == ST_RK4_2) {
      a.acc[o] = cadd(a.acc[o], rmul(2.0, kk));
      res = cadd(b, rmul(0.50, kk));
    } else if (KIND == ST_RK4_3) {
      a.acc[o] = cadd(a.acc[o], rmul(2.0, kk));
      res = cadd(b, kk);
    } else {
      res = cadd(b, cdivr(cadd(a.acc[o], kk), 6.0));
    }
    a.out[o] = res;
  }
}

// duplicated phi planes: k = 0 <- Nz-1, k = Nz <- 1
__global__ void cfg_ghost_z(Grid g, double2* u) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)g.NI * g.NJ;
  if (t >= n) return;
  const int ii = (int)(t % g.NI), jj = (int)(t / g.NI);
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    double2* w = u + (long long)v * g.fs;
    w[off3(g, ii, jj, 0)] = w[off3(g, ii, jj, g.Nz - 1)];
    w[off3(g, ii, jj, g.Nz)] = w[off3(g, ii, jj, 1)];
  }
}

// theta ghost rows from the interior rows at phi + pi, psi_2 negated
__global__ void cfg_ghost_rows(Grid g, double2* u) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = 6LL * g.NI * g.NK;
  if (t >= n) return;
  const int ii = (int)(t % g.NI);
  const long long rk = t / g.NI;
  const int r = (int)(rk % 6);
  const int k = (int)(rk / 6);
  const int jj = (r < 3) ? r : (g.NJ - 6 + r);
  const int js = (jj <= 2) ? (5 - jj) : (2 * g.NJ - 7 - jj);
  const int kt = ktarget(g, k);
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    double2* w = u + (long long)v * g.fs;
    const double2 s = w[off3(g, ii, js, kt)];
    w[off3(g, ii, jj, k)] = (v == 2) ? rmul(-1.0, s) : s;
  }
}

}  // namespace

int launch_stage_cfg(int kind, const StageLaunch& L, const double* dxbeta4, const double coef[6], double rN,
                       cudaStream_t st) {
  CfgArgs a;
  a.g = L.g;
  a.m = L.m;
  a.dxb4 = dxbeta4;
  a.in = L.in[0];
  a.base = L.base;
  a.acc = L.acc;
  a.out = L.out;
  a.rr = coef[0];
  a.rt = coef[1];
  a.rp = coef[2];
  a.kr = coef[3];
  a.kt = coef[4];
  a.kp = coef[5];
  a.rN = rN;
  dim3 grid((L.g.NI + 127) / 128, L.g.NJ, L.g.NK);
  switch (kind) {
    case ST_RK4_1: cfg_stage_kernel<ST_RK4_1><<<grid, 128, 0, st>>>(a); return 0;
    case ST_RK4_2: cfg_stage_kernel<ST_RK4_2><<<grid, 128, 0, st>>>(a); return 0;
    case ST_RK4_3: cfg_stage_kernel<ST_RK4_3><<<grid, 128, 0, st>>>(a); return 0;
    case ST_RK4_4: cfg_stage_kernel<ST_RK4_4><<<grid, 128, 0, st>>>(a); return 0;
    default: return -1;
  }
}

void launch_ghost_fill_cfg(const Grid& g, double2* u, cudaStream_t st) {
  const long long nz = (long long)g.NI * g.NJ;
  cfg_ghost_z<<<(unsigned)((nz + 255) / 256), 256, 0, st>>>(g, u);
  const long long nr = 6LL * g.NI * g.NK;
  cfg_ghost_rows<<<(unsigned)((nr + 255) / 256), 256, 0, st>>>(g, u);
}

}  // namespace kg
