// kg_stencil.cu -- RHS + stage-combination kernels of the time steppers.
//
// One kernel launch evaluates the reference's right-hand side at every stored
// point (ghosts included, with the one-sided / pole / seam stencils at the
// array ends, MoL/lines_method_lib.f90:671-753) and immediately applies the
// stage combination of the stepper being run (MoL/lines_method_lib.f90:211-474),
// so the RHS never round-trips through HBM.  The PIRK stage 1 needs the new
// psi stage values at neighbouring points before rhs_pi can be evaluated, so it
// is split into two launches (psi/phi part, then Pi part).
//
// Thread mapping: x -> r (ii, coalesced 16-byte loads/stores of double2),
// y -> theta (jj), z -> phi (k).  Grid sizes are ceil-divided and every thread
// checks ii < NI, jj < NJ, k < NK before touching memory.
#include "kg_device.cuh"
#include "kg_internal.h"

namespace kg {

struct Vars {
  const double2* v[5];  // stencil input, one pointer per variable
};

// rhs_phi, rhs_psi1, rhs_psi2, rhs_psi3 at one point (lines_method_lib.f90:671-713)
__device__ __forceinline__ void rhs_psi(const Grid& g, const Metric& M, const Vars& V,
                                        int ii, int jj, int k, double2 r[4]) {
  const int q = off2(g, ii, jj);
  const long long p = off3(g, ii, jj, k);
  const double al = ldm(M.alpha, q), be = ldm(M.beta, q), dxb = ldm(M.dxbeta, q);
  const double2 pi_ = ldf(V.v[4], p), ps1 = ldf(V.v[1], p);
  // rhs_phi = alpha*Pi + beta*psi1
  r[0] = cadd(rmul(al, pi_), rmul(be, ps1));
  // rhs_psi1 = dx1(alpha*Pi) + beta*ad_1(psi1) + dx_beta*psi1
  auto aPi = [&](int i2, int j2, int k2) {
    return rmul(ldm(M.alpha, off2(g, i2, j2)), ldf(V.v[4], off3(g, i2, j2, k2)));
  };
  auto fps1 = [&](int i2, int j2, int k2) { return ldf(V.v[1], off3(g, i2, j2, k2)); };
  const double2 d = op_dr(g, aPi, ii, jj, k);
  const double2 a = op_ar(g, fps1, be, ii, jj, k);
  r[1] = cadd(cadd(d, rmul(be, a)), rmul(dxb, ps1));
  // rhs_psi2/3 = dx2/dx3(alpha*Pi + beta*psi1)
  auto E = [&](int i2, int j2, int k2) {
    const int q2 = off2(g, i2, j2);
    const long long p2 = off3(g, i2, j2, k2);
    return cadd(rmul(ldm(M.alpha, q2), ldf(V.v[4], p2)), rmul(ldm(M.beta, q2), ldf(V.v[1], p2)));
  };
  r[2] = op_dth(g, E, ii, jj, k);
  r[3] = op_dph(g, E, ii, jj, k);
}

// rhs_pi at one point (lines_method_lib.f90:716-753)
template <int MK>
__device__ __forceinline__ double2 rhs_pi(const Grid& g, const Metric& M, const Vars& V,
                                          int ii, int jj, int k) {
  const int q = off2(g, ii, jj);
  const long long p = off3(g, ii, jj, k);
  const double sg = ldm(M.sqrtg, q), be = ldm(M.beta, q), dxb = ldm(M.dxbeta, q), am2 = ldm(M.am2, q);
  auto G1 = [&](int i2, int j2, int k2) {
    const int q2 = off2(g, i2, j2);
    const long long p2 = off3(g, i2, j2, k2);
    if (MK == MK_KS)
      return rmul(ldm(M.asg, q2), cadd(rmul(ldm(M.grr, q2), ldf(V.v[1], p2)), rmul(ldm(M.grp, q2), ldf(V.v[3], p2))));
    else
      return rmul(ldm(M.asg_grr, q2), ldf(V.v[1], p2));
  };
  auto H = [&](int i2, int j2, int k2) {
    return rmul(ldm(M.asg_gtt, off2(g, i2, j2)), ldf(V.v[2], off3(g, i2, j2, k2)));
  };
  auto Fp = [&](int i2, int j2, int k2) {
    const int q2 = off2(g, i2, j2);
    const long long p2 = off3(g, i2, j2, k2);
    if (MK == MK_KS)
      return rmul(ldm(M.asg, q2), cadd(rmul(ldm(M.grp, q2), ldf(V.v[1], p2)), rmul(ldm(M.gpp, q2), ldf(V.v[3], p2))));
    else
      return rmul(ldm(M.a_gpp, q2), ldf(V.v[3], p2));
  };
  auto Q = [&](int i2, int j2, int k2) {
    return rmul(ldm(M.sqrtg, off2(g, i2, j2)), ldf(V.v[4], off3(g, i2, j2, k2)));
  };
  const double2 r1 = cdivr(op_dr(g, G1, ii, jj, k), sg);
  const double2 r2 = cdivr(op_dth(g, H, ii, jj, k), sg);
  const double2 d3 = op_dph(g, Fp, ii, jj, k);
  const double2 r3 = (MK == MK_KS) ? cdivr(d3, sg) : d3;
  const double2 r4 = rmul(dxb, ldf(V.v[4], p));
  const double2 r5 = cdivr(rmul(be, op_ar(g, Q, be, ii, jj, k)), sg);
  const double2 r6 = rmul(am2, ldf(V.v[0], p));
  return csub(cadd(cadd(cadd(cadd(r1, r2), r3), r4), r5), r6);
}

struct StageArgs {
  Grid g;
  Metric m;
  Vars in;               // stencil input
  const double2* base;   // u_p / u^n (5 variables, stride g.fs)
  const double2* aux4;   // PIRK3 stage 2b: u_stage(5)
  double2* out;          // output state (5 variables)
  double2* out4;         // output of a Pi-only stage
  double2* acc;          // RK4 accumulator k1 + 2k2 + 2k3
  int skip_last_i;       // inflow: keep u_p at ii = NI-1 in an in-place final stage
};

template <int KIND>
__device__ __forceinline__ void combine(const StageArgs& a, long long p, int ii, const double2 r[5]) {
  const Grid& g = a.g;
  const double dt = g.dt;
  if (KIND == ST_P2_S1A) {
#pragma unroll
    for (int v = 0; v < 4; ++v) a.out[v * g.fs + p] = cadd(ldf(a.base + v * g.fs, p), rmul(dt, r[v]));
    return;
  }
  if (KIND == ST_P3_S2A) {
#pragma unroll
    for (int v = 0; v < 4; ++v)
      a.out[v * g.fs + p] = cadd(rmul(0.75, ldf(a.base + v * g.fs, p)), rmul(0.25, cadd(ldf(a.in.v[v], p), rmul(dt, r[v]))));
    return;
  }
  if (a.skip_last_i && ii == g.NI - 1) return;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const long long o = v * g.fs + p;
    const double2 b = ldf(a.base + v * g.fs, p);
    double2 res;
    if (KIND == ST_P2_S2) {
      res = rmul(0.5, cadd(cadd(b, ldf(a.in.v[v], p)), rmul(dt, r[v])));
    } else if (KIND == ST_P3_S3) {
      res = cadd(rmul(1.0 / 3.0, b), rmul(2.0 / 3.0, cadd(ldf(a.in.v[v], p), rmul(dt, r[v]))));
    } else if (KIND == ST_RK3_1) {
      res = cadd(b, rmul(dt, r[v]));
    } else if (KIND == ST_RK3_2) {
      res = cadd(rmul(0.750, b), rmul(0.250, cadd(ldf(a.in.v[v], p), rmul(dt, r[v]))));
    } else if (KIND == ST_RK3_3) {
      res = cadd(cdivr(b, 3.0), cdivr(rmul(2.0, cadd(ldf(a.in.v[v], p), rmul(dt, r[v]))), 3.0));
    } else if (KIND == ST_RK4_1) {
      const double2 kk = rmul(dt, r[v]);
      a.acc[o] = kk;
      res = cadd(b, rmul(0.50, kk));
    } else if (KIND == ST_RK4_2) {
      const double2 kk = rmul(dt, r[v]);
      a.acc[o] = cadd(a.acc[o], rmul(2.0, kk));
      res = cadd(b, rmul(0.50, kk));
    } else if (KIND == ST_RK4_3) {
      const double2 kk = rmul(dt, r[v]);
      a.acc[o] = cadd(a.acc[o], rmul(2.0, kk));
      res = cadd(b, kk);
    } else {  // ST_RK4_4
      const double2 kk = rmul(dt, r[v]);
      res = cadd(b, cdivr(cadd(a.acc[o], kk), 6.0));
    }
    a.out[o] = res;
  }
}

template <int KIND, int MK>
__global__ void __launch_bounds__(256) stage_kernel(StageArgs a) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const Grid& g = a.g;
  if (ii >= g.NI || jj >= g.NJ || k >= g.NK) return;
  const long long p = off3(g, ii, jj, k);
  if (KIND == ST_P2_S1B || KIND == ST_P3_S2B) {
    const double2 r4 = rhs_pi<MK>(g, a.m, a.in, ii, jj, k);
    const double dt = g.dt;
    if (KIND == ST_P2_S1B)
      a.out4[p] = cadd(ldf(a.base + 4 * g.fs, p), rmul(dt, r4));
    else
      a.out4[p] = cadd(rmul(0.75, ldf(a.base + 4 * g.fs, p)), rmul(0.25, cadd(ldf(a.aux4, p), rmul(dt, r4))));
    return;
  }
  double2 r[5];
  rhs_psi(g, a.m, a.in, ii, jj, k, r);
  if (KIND != ST_P2_S1A && KIND != ST_P3_S2A) r[4] = rhs_pi<MK>(g, a.m, a.in, ii, jj, k);
  combine<KIND>(a, p, ii, r);
}

// rhs hook: selected rhs_* of arbitrary vars into out (5 variables)
template <int MK>
__global__ void __launch_bounds__(256) rhs_kernel(Grid g, Metric m, Vars in, double2* out, unsigned mask) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (ii >= g.NI || jj >= g.NJ || k >= g.NK) return;
  const long long p = off3(g, ii, jj, k);
  double2 r[4];
  rhs_psi(g, m, in, ii, jj, k, r);
  for (int v = 0; v < 4; ++v)
    if (mask & (1u << v)) out[v * g.fs + p] = r[v];
  if (mask & 16u) out[4 * g.fs + p] = rhs_pi<MK>(g, m, in, ii, jj, k);
}

static dim3 stage_block() { return dim3(64, 4, 1); }
static dim3 stage_grid(const Grid& g) {
  dim3 b = stage_block();
  return dim3((g.NI + b.x - 1) / b.x, (g.NJ + b.y - 1) / b.y, g.NK);
}

template <int KIND>
static void launch_kind(const StageLaunch& L, cudaStream_t st) {
  StageArgs a;
  a.g = L.g;
  a.m = L.m;
  for (int v = 0; v < 5; ++v) a.in.v[v] = L.in[v];
  a.base = L.base;
  a.aux4 = L.aux4;
  a.out = L.out;
  a.out4 = L.out4;
  a.acc = L.acc;
  a.skip_last_i = L.skip_last_i;
  if (L.metric_kind == MK_KS)
    stage_kernel<KIND, MK_KS><<<stage_grid(L.g), stage_block(), 0, st>>>(a);
  else
    stage_kernel<KIND, MK_SCHW><<<stage_grid(L.g), stage_block(), 0, st>>>(a);
}

void launch_stage(int kind, const StageLaunch& L, cudaStream_t st) {
  switch (kind) {
    case ST_P2_S1A: launch_kind<ST_P2_S1A>(L, st); break;
    case ST_P2_S1B: launch_kind<ST_P2_S1B>(L, st); break;
    case ST_P2_S2: launch_kind<ST_P2_S2>(L, st); break;
    case ST_P3_S2A: launch_kind<ST_P3_S2A>(L, st); break;
    case ST_P3_S2B: launch_kind<ST_P3_S2B>(L, st); break;
    case ST_P3_S3: launch_kind<ST_P3_S3>(L, st); break;
    case ST_RK3_1: launch_kind<ST_RK3_1>(L, st); break;
    case ST_RK3_2: launch_kind<ST_RK3_2>(L, st); break;
    case ST_RK3_3: launch_kind<ST_RK3_3>(L, st); break;
    case ST_RK4_1: launch_kind<ST_RK4_1>(L, st); break;
    case ST_RK4_2: launch_kind<ST_RK4_2>(L, st); break;
    case ST_RK4_3: launch_kind<ST_RK4_3>(L, st); break;
    case ST_RK4_4: launch_kind<ST_RK4_4>(L, st); break;
    default: break;
  }
}

void launch_rhs(const Grid& g, const Metric& m, int metric_kind, const double2* const in[5], double2* out,
                unsigned mask, cudaStream_t st) {
  Vars V;
  for (int v = 0; v < 5; ++v) V.v[v] = in[v];
  if (metric_kind == MK_KS)
    rhs_kernel<MK_KS><<<stage_grid(g), stage_block(), 0, st>>>(g, m, V, out, mask);
  else
    rhs_kernel<MK_SCHW><<<stage_grid(g), stage_block(), 0, st>>>(g, m, V, out, mask);
}

}  // namespace kg
