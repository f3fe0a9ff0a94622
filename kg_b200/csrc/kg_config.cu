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
// Divisions by sqrt(gamma) and RK4's 1/6 use the correctly rounded reciprocal
// with one Markstein correction (the IEEE quotient for dividends above about
// 2^-1000 in magnitude).
#include <cuda_runtime.h>
#include "kg_device.cuh"
#include "kg_internal.h"
#include "kg_tma_ops.cuh"

namespace kg {
using namespace tmaops;
namespace {

struct CfgArgs {
  Grid g;
  Metric m;
  const double* dxb4;  // D4 d_r beta^r, [jj][ii] with pitch PI
  const double* rsg;   // 1 / sqrt(gamma), host-rounded, same layout
  const double2* in;   // stage input (5 variables, stride g.fs)
  const double2* base; // u^n
  double2* acc;
  double2* out;
  double rr, rt, rp;   // 1 / (12 h) per direction
  double kr, kt, kp;   // eps / (64 h) per direction
  double rN;           // r of the outermost stored plane
};

// plane d steps from plane k (1 <= k <= Nz-1) over the Nz-1 distinct planes 1..Nz-1;
// |d| <= 4 <= Nz-1, so one wrap at most
__device__ __forceinline__ int kper(const Grid& g, int k, int d) {
  const int M = g.Nzm1;
  int kk = k - 1 + d;
  if (kk < 0) kk += M;
  if (kk >= M) kk -= M;
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
// a / b from the correctly rounded reciprocal rb and one Markstein correction
// (q = a rb, r = a - q b, q + r rb): the IEEE quotient for dividends above about
// 2^-1000 in magnitude, at three operations instead of a division sequence
__device__ __forceinline__ double qdiv(double a, double b, double rb) {
  const double q = a * rb;
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, rb, q);
}
__device__ __forceinline__ double2 cqdiv(double2 a, double b, double rb) { return c2(qdiv(a.x, b, rb), qdiv(a.y, b, rb)); }
constexpr double kSixth = 1.0 / 6.0;

// RHS and RK4 combination at one stored point (ii, jj, k).  S(v, i, j) returns
// variable v of the stage input at (i, j) on plane k, P(v, d) at the point's
// own (ii, jj) on the plane d steps away in phi (d = -3..3, d != 0; only asked
// for 1 <= k <= Nz-1); the two kernels below differ only in where S and P read
// from, so they produce the same bits.
template <int KIND, class SF, class PF>
__device__ __forceinline__ void cfg_point(const CfgArgs& a, int ii, int jj, int k, const SF& S, const PF& P) {
  const Grid& g = a.g;
  const Metric& M = a.m;
  const long long p = off3(g, ii, jj, k);
  const int q = off2(g, ii, jj);
  double2 r[5];
  const int n = g.NI - 1;
  if (jj <= 2 || jj >= g.NJ - 3 || k == 0 || k == g.Nz) {
#pragma unroll
    for (int v = 0; v < 5; ++v) r[v] = c2(0.0, 0.0);
  } else if (ii == n) {
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      auto f = [&](int i2) { return S(v, i2, jj); };
      r[v] = cneg(cadd(d4r(g, f, ii, a.rr), cdiv(S(v, ii, jj), a.rN)));
    }
  } else {
    const double al = ldm(M.alpha, q), b1 = ldm(M.beta, q), sg = ldm(M.sqrtg, q), dxb = ldm(a.dxb4, q);
    // alpha Pi + beta psi_1 on this plane (ES) and in the own column (EP)
    auto ES = [&](int i2, int j2) {
      const int q2 = off2(g, i2, j2);
      return cadd(rmul(ldm(M.alpha, q2), S(4, i2, j2)), rmul(ldm(M.beta, q2), S(1, i2, j2)));
    };
    auto EP = [&](int d) { return cadd(rmul(ldm(M.alpha, q), P(4, d)), rmul(ldm(M.beta, q), P(1, d))); };
    auto Fp = [&](int d) {
      return rmul(ldm(M.asg, q), cadd(rmul(ldm(M.grp, q), P(1, d)), rmul(ldm(M.gpp, q), P(3, d))));
    };
    // sqrt(gamma) carries the sign of sin(theta) through the pole: negative on the ghost rows
    auto H = [&](int j2) {
      const double2 h = rmul(ldm(M.asg_gtt, off2(g, ii, j2)), S(2, ii, j2));
      return (j2 <= 2 || j2 >= g.NJ - 3) ? cneg(h) : h;
    };
    const double2 pi = S(4, ii, jj), ps1 = S(1, ii, jj);
    r[0] = cadd(rmul(al, pi), rmul(b1, ps1));
    {
      auto fA = [&](int i2) { return rmul(ldm(M.alpha, off2(g, i2, jj)), S(4, i2, jj)); };
      auto fP = [&](int i2) { return S(1, i2, jj); };
      r[1] = cadd(cadd(d4r(g, fA, ii, a.rr), rmul(b1, d4r(g, fP, ii, a.rr))), rmul(dxb, ps1));
    }
    r[2] = d4c(ES(ii, jj - 2), ES(ii, jj - 1), ES(ii, jj + 1), ES(ii, jj + 2), a.rt);
    r[3] = d4c(EP(-2), EP(-1), EP(1), EP(2), a.rp);
    {
      auto fG = [&](int i2) {
        const int q2 = off2(g, i2, jj);
        return rmul(ldm(M.asg, q2), cadd(rmul(ldm(M.grr, q2), S(1, i2, jj)), rmul(ldm(M.grp, q2), S(3, i2, jj))));
      };
      auto fQ = [&](int i2) {
        const double2 w = S(4, i2, jj);
        const double s2 = ldm(M.sqrtg, off2(g, i2, jj));
        return c2(w.x * s2, w.y * s2);
      };
      const double rs = ldm(a.rsg, q);
      const double2 t1 = cqdiv(d4r(g, fG, ii, a.rr), sg, rs);
      const double2 t2 = cqdiv(d4c(H(jj - 2), H(jj - 1), H(jj + 1), H(jj + 2), a.rt), sg, rs);
      const double2 t3 = cqdiv(d4c(Fp(-2), Fp(-1), Fp(1), Fp(2), a.rp), sg, rs);
      const double2 t4 = c2(pi.x * dxb, pi.y * dxb);
      const double2 t5 = cqdiv(rmul(b1, d4r(g, fQ, ii, a.rr)), sg, rs);
      const double2 t6 = rmul(ldm(M.am2, q), S(0, ii, jj));
      r[4] = csub(cadd(cadd(cadd(cadd(t1, t2), t3), t4), t5), t6);
    }
    const bool kor = ii >= 3 && ii <= n - 3;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      double2 s = r[v];
      if (kor)
        s = cadd(s, rmul(a.kr, ko6(S(v, ii - 3, jj), S(v, ii - 2, jj), S(v, ii - 1, jj), S(v, ii, jj),
                                   S(v, ii + 1, jj), S(v, ii + 2, jj), S(v, ii + 3, jj))));
      s = cadd(s, rmul(a.kt, ko6(S(v, ii, jj - 3), S(v, ii, jj - 2), S(v, ii, jj - 1), S(v, ii, jj),
                                 S(v, ii, jj + 1), S(v, ii, jj + 2), S(v, ii, jj + 3))));
      s = cadd(s, rmul(a.kp, ko6(P(v, -3), P(v, -2), P(v, -1), S(v, ii, jj), P(v, 1), P(v, 2), P(v, 3))));
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
      res = cadd(b, cqdiv(cadd(a.acc[o], kk), 6.0, kSixth));
    }
    a.out[o] = res;
  }
}

// One thread per stored point; every neighbour through the read-only cache.
template <int KIND>
__global__ void __launch_bounds__(128) cfg_stage_kernel(CfgArgs a) {
  const Grid& g = a.g;
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y;
  const int k = blockIdx.z;
  if (ii >= g.NI) return;
  const double2* U = a.in;
  auto S = [&](int v, int i2, int j2) { return ldf(U + (long long)v * g.fs, off3(g, i2, j2, k)); };
  auto P = [&](int v, int d) { return ldf(U + (long long)v * g.fs, off3(g, ii, jj, kper(g, k, d))); };
  cfg_point<KIND>(a, ii, jj, k, S, P);
}

// Tiled form: a CTA owns a 32 x 8 tile of (r, theta) columns and marches through
// a chunk of phi planes.  The plane being updated arrives in shared memory with
// a +-4 r and +-3 theta halo (every same-plane neighbour the fourth-order
// differences, the r closures and the sixth-order dissipation touch), double
// buffered: the next plane's tile is copied by cp.async while this plane is
// computed.  The phi neighbours of the thread's own column (planes k+-1..3)
// are read through the read-only cache; the same values serve seven
// consecutive planes of the march.  (Holding them in a rolling register window
// instead needs 255 registers per thread and one CTA per SM, and ran the C0
// grid at half the speed.)
constexpr int CTI = 32, CTJ = 8, CRH = 4, CTH = 3;
constexpr int CW = CTI + 2 * CRH, CH = CTJ + 2 * CTH, CT_N = CW * CH;
constexpr size_t CFG_TILE_BYTES = (size_t)5 * CT_N * sizeof(double2);

template <int KIND>
__global__ void __launch_bounds__(CTI * CTJ, 2) cfg_march_kernel(CfgArgs a, int kchunk) {
  extern __shared__ __align__(16) unsigned char cfg_smem[];
  double2* tiles = reinterpret_cast<double2*>(cfg_smem);
  const Grid& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * CTI + tx;
  const int ii0 = blockIdx.x * CTI, jj0 = blockIdx.y * CTJ;
  const int ii = ii0 + tx, jj = jj0 + ty;
  const bool act = ii < g.NI && jj < g.NJ;
  const int k0 = blockIdx.z * kchunk;
  if (k0 >= g.NK) return;  // uniform over the block
  const int k1 = min(k0 + kchunk, g.NK);
  const double2* col = a.in + (act ? off3(g, ii, jj, 0) : 0);
  // points of the halo tile outside the array are not copied; no stencil reads them
  auto load = [&](int k, int buf) {
    double2* dst = tiles + (size_t)buf * 5 * CT_N;
    for (int t = tid; t < 5 * CT_N; t += CTI * CTJ) {
      const int v = t / CT_N, r = t - v * CT_N, ly = r / CW, lx = r - ly * CW;
      const int gi = ii0 - CRH + lx, gj = jj0 - CTH + ly;
      if (gi >= 0 && gi < g.NI && gj >= 0 && gj < g.NJ)
        cp_async16(dst + t, a.in + (long long)v * g.fs + off3(g, gi, gj, k));
    }
    cp_async_commit();
  };
  load(k0, 0);
  for (int k = k0; k < k1; ++k) {
    const int buf = (k - k0) & 1;
    if (k + 1 < k1) {
      load(k + 1, buf ^ 1);  // that buffer was last read before the previous block barrier
      cp_async_wait_prior();
    } else {
      cp_async_wait_all();
    }
    __syncthreads();
    if (act) {
      // every same-plane neighbour lies inside the halo tile
      const double2* T = tiles + (size_t)buf * 5 * CT_N + (ty + CTH) * CW + (tx + CRH);
      auto S = [&](int v, int i2, int j2) { return T[v * CT_N + (j2 - jj) * CW + (i2 - ii)]; };
      auto P = [&](int v, int d) { return ldf(col + (long long)v * g.fs, (long long)kper(g, k, d) * g.plane); };
      cfg_point<KIND>(a, ii, jj, k, S, P);
    }
    __syncthreads();
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

template <int KIND>
int cfg_march_launch(const CfgArgs& a, cudaStream_t st) {
  static bool attr = false;  // dynamic shared memory above 48 KB, set once per stage kind
  if (!attr) {
    if (cudaFuncSetAttribute(cfg_march_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * CFG_TILE_BYTES)) != cudaSuccess)
      return -1;
    attr = true;
  }
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  }
  const Grid& g = a.g;
  const int tx = (g.NI + CTI - 1) / CTI, ty = (g.NJ + CTJ - 1) / CTJ;
  // about two waves of two CTAs per SM: small grids are cut into phi chunks
  int nch = (4 * sms + tx * ty - 1) / (tx * ty);
  nch = nch < 1 ? 1 : (nch > g.NK ? g.NK : nch);
  const int kchunk = (g.NK + nch - 1) / nch;
  nch = (g.NK + kchunk - 1) / kchunk;
  cfg_march_kernel<KIND><<<dim3(tx, ty, nch), dim3(CTI, CTJ, 1), 2 * CFG_TILE_BYTES, st>>>(a, kchunk);
  return 0;
}

}  // namespace

int launch_stage_cfg(int kind, const StageLaunch& L, const double* dxbeta4, const double* rsg, const double coef[6],
                     double rN, int tiled, cudaStream_t st) {
  CfgArgs a;
  a.g = L.g;
  a.m = L.m;
  a.dxb4 = dxbeta4;
  a.rsg = rsg;
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
  if (tiled) {
    switch (kind) {
      case ST_RK4_1: return cfg_march_launch<ST_RK4_1>(a, st);
      case ST_RK4_2: return cfg_march_launch<ST_RK4_2>(a, st);
      case ST_RK4_3: return cfg_march_launch<ST_RK4_3>(a, st);
      case ST_RK4_4: return cfg_march_launch<ST_RK4_4>(a, st);
      default: return -1;
    }
  }
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
