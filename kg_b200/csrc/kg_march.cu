// kg_march.cu -- 2.5-D marching form of the fused RHS + stage kernels.
//
// Same arithmetic as kg_stencil.cu (bit for bit), organised for HBM:
//   * a CTA owns a TI x TJ tile of (r, theta) columns and marches through a
//     chunk of phi planes;
//   * each thread keeps its own column's phi window (the combinations that the
//     phi derivative needs at k-1, k, k+1) in registers, so phi neighbours are
//     never re-read from memory;
//   * the in-plane neighbours come from shared memory: per plane the CTA stores
//     the r-direction combinations with a +-2 halo and the theta-direction
//     combinations with a +-1 halo, each computed once by the thread that
//     loaded the point;
//   * the next plane of the thread's own point is loaded one plane ahead
//     (16-byte loads, coalesced along r) to keep memory requests in flight;
//   * divisions by sqrt(gamma) use the host-computed reciprocal with one
//     Markstein correction step, q' = q + (a - b q) y, which returns the
//     correctly rounded quotient a/b when y = RN(1/b) and q = RN(a y)
//     (P. Markstein, IBM J. Res. Dev. 34 (1990); Muller et al., Handbook of
//     Floating-Point Arithmetic, the theorem on division by a correctly rounded
//     reciprocal), so results equal IEEE division while the residual a - b q
//     stays normal: for dividends below about 2^-1000 in magnitude (a field
//     tail on its way to underflow) the quotient can be one unit off.  A guard
//     that divides outright there cost the PIRK2 step 9 %; the per-point form
//     (kg_stencil.cu) divides outright everywhere.
// Stencils at the array ends, the theta pole row (partner plane k + Nz/2) and
// the phi seam planes follow the reference exactly; values that fall outside
// the tile are computed directly from global memory.
#include "kg_device.cuh"
#include "kg_internal.h"

namespace kg {

constexpr int TI = 32;  // r extent of a tile (one warp = one row of 512 B)
constexpr int TJ = 8;   // theta extent
constexpr int RH = 2;   // r halo

__device__ __forceinline__ double ddiv(double a, double b, double rb) {
  const double q = a * rb;
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, rb, q);
}
__device__ __forceinline__ double2 cdivm(double2 a, double b, double rb) {
  return c2(ddiv(a.x, b, rb), ddiv(a.y, b, rb));
}
// the stage combinations' divisions by 3 (SSP-RK3) and 6 (RK4) take the same
// route, from the correctly rounded reciprocals
constexpr double kThird = 1.0 / 3.0, kSixth = 1.0 / 6.0;

struct MarchArgs {
  Grid g;
  Metric m;
  const double* rsg;      // 1/sqrt(gamma) table (correctly rounded on the host)
  const double2* in[5];   // stencil input
  const double2* base;    // u_p / u^n
  const double2* aux4;    // PIRK3 stage 2b: u_stage(5)
  double2* out;
  double2* out4;
  double2* acc;
  int skip_last_i;
  int kchunk;             // planes per CTA
};

// combinations of one point (the quantities whose derivatives the RHS takes)
struct Combo {
  double2 aPi, ps1, E, G1, Q, H, F;
};

// the two combinations whose phi derivative the RHS takes
struct PhiPair {
  double2 E, F;
};

template <int MK, bool PSI, bool PI_>
__device__ __forceinline__ void make_phi(const Metric& M, int q, const double2 f[5], PhiPair& c) {
  if (PSI) c.E = cadd(rmul(ldm(M.alpha, q), f[4]), rmul(ldm(M.beta, q), f[1]));
  if (PI_) {
    if (MK == MK_KS)
      c.F = rmul(ldm(M.asg, q), cadd(rmul(ldm(M.grp, q), f[1]), rmul(ldm(M.gpp, q), f[3])));
    else
      c.F = rmul(ldm(M.a_gpp, q), f[3]);
  }
}

template <int MK, bool PSI, bool PI_>
__device__ __forceinline__ void make_combo(const Metric& M, int q, const double2 f[5], Combo& c) {
  const double al = ldm(M.alpha, q);
  if (PSI) {
    c.aPi = rmul(al, f[4]);
    c.ps1 = f[1];
    c.E = cadd(rmul(al, f[4]), rmul(ldm(M.beta, q), f[1]));
  }
  if (PI_) {
    if (MK == MK_KS) {
      const double asg = ldm(M.asg, q), grp = ldm(M.grp, q);
      c.G1 = rmul(asg, cadd(rmul(ldm(M.grr, q), f[1]), rmul(grp, f[3])));
      c.F = rmul(asg, cadd(rmul(grp, f[1]), rmul(ldm(M.gpp, q), f[3])));
    } else {
      c.G1 = rmul(ldm(M.asg_grr, q), f[1]);
      c.F = rmul(ldm(M.a_gpp, q), f[3]);
    }
    c.Q = rmul(ldm(M.sqrtg, q), f[4]);
    c.H = rmul(ldm(M.asg_gtt, q), f[2]);
  }
}

__device__ __forceinline__ void load5(const double2* const in[5], long long p, double2 f[5]) {
#pragma unroll
  for (int v = 0; v < 5; ++v) f[v] = ldf(in[v], p);
}

// E and H (theta-derivative arguments) or E/F at an arbitrary point, from global memory
template <int MK, bool PSI, bool PI_>
__device__ __forceinline__ void direct_combo(const Grid& g, const Metric& M, const double2* const in[5], int ii,
                                             int jj, int k, Combo& c) {
  double2 f[5];
  load5(in, off3(g, ii, jj, k), f);
  make_combo<MK, PSI, PI_>(M, off2(g, ii, jj), f, c);
}

template <int KIND, int MK>
__global__ void __launch_bounds__(TI * TJ, 2) march_kernel(MarchArgs a) {
  constexpr bool PSI = (KIND != ST_P2_S1B && KIND != ST_P3_S2B);
  constexpr bool PI_ = (KIND != ST_P2_S1A && KIND != ST_P3_S2A);
  // r-direction combinations: aPi, ps1 (PSI); G1, Q (PI); theta: E (PSI), H (PI)
  __shared__ double2 sAPi[PSI ? TJ : 1][TI + 2 * RH];
  __shared__ double2 sPs1[PSI ? TJ : 1][TI + 2 * RH];
  __shared__ double2 sG1[PI_ ? TJ : 1][TI + 2 * RH];
  __shared__ double2 sQ[PI_ ? TJ : 1][TI + 2 * RH];
  __shared__ double2 sE[PSI ? TJ + 2 : 1][TI];
  __shared__ double2 sH[PI_ ? TJ + 2 : 1][TI];

  const Grid& g = a.g;
  const Metric& M = a.m;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TI + tx;
  const int ii = blockIdx.x * TI + tx, jj = blockIdx.y * TJ + ty;
  const bool act = (ii < g.NI) && (jj < g.NJ);
  const int k0 = blockIdx.z * a.kchunk;
  const int k1 = min(k0 + a.kchunk, g.NK);
  if (k0 >= g.NK) return;

  // halo role: tid 0..4TJ-1 -> r halo (row tid/4, column -2,-1,TI,TI+1);
  //            tid 4TJ..4TJ+2TI-1 -> theta halo (row -1 or TJ, column tid%TI)
  int hrole = 0, hi = -1, hj = -1, hsx = 0, hsy = 0;
  if (tid < 4 * TJ) {
    const int row = tid >> 2, c = tid & 3;
    hsx = (c < 2) ? c : TI + c;  // smem column (with +RH offset already applied)
    hsy = row;
    hi = blockIdx.x * TI + ((c < 2) ? c - 2 : TI + c - 2);
    hj = blockIdx.y * TJ + row;
    hrole = (hi >= 0 && hi < g.NI && hj < g.NJ) ? 1 : 0;
  } else if (tid < 4 * TJ + 2 * TI) {
    const int t = tid - 4 * TJ;
    const int side = t / TI;
    hsx = t % TI;
    hsy = side ? TJ + 1 : 0;
    hi = blockIdx.x * TI + hsx;
    hj = blockIdx.y * TJ + (side ? TJ : -1);
    hrole = (hi < g.NI && hj >= 0 && hj < g.NJ) ? 2 : 0;
  }
  const int hq = hrole ? off2(g, hi, hj) : 0;

  const int q = act ? off2(g, ii, jj) : 0;
  double be = 0.0, dxb = 0.0, sg = 1.0, rs = 1.0, am2 = 0.0;
  if (act) {
    be = ldm(M.beta, q);
    dxb = ldm(M.dxbeta, q);
    if (PI_) {
      sg = ldm(M.sqrtg, q);
      rs = ldm(a.rsg, q);
      am2 = ldm(M.am2, q);
    }
  }
  const long long pcol = act ? off3(g, ii, jj, 0) : 0;  // offset of (ii, jj, 0)

  // phi window: the E / F combinations at k-1 (pv), k (cu), k+1 (nx)
  PhiPair cpv, ccu, cnx;
  double2 fcu[5], fnx[5];
  if (act) {
    const int kp = (k0 == 0) ? g.Nz - 2 : k0 - 1;
    double2 f[5];
    load5(a.in, pcol + (long long)kp * g.plane, f);
    make_phi<MK, PSI, PI_>(M, q, f, cpv);
    load5(a.in, pcol + (long long)k0 * g.plane, fcu);
    make_phi<MK, PSI, PI_>(M, q, fcu, ccu);
  }

  for (int k = k0; k < k1; ++k) {
    const int kn = (k == g.Nz) ? 2 : k + 1;
    if (act) load5(a.in, pcol + (long long)kn * g.plane, fnx);
    // halo point of this plane
    if (hrole) {
      double2 f[5];
      load5(a.in, off3(g, hi, hj, k), f);
      Combo c;
      make_combo<MK, PSI, PI_>(M, hq, f, c);
      if (hrole == 1) {
        if (PSI) { sAPi[hsy][hsx] = c.aPi; sPs1[hsy][hsx] = c.ps1; }
        if (PI_) { sG1[hsy][hsx] = c.G1; sQ[hsy][hsx] = c.Q; }
      } else {
        if (PSI) sE[hsy][hsx] = c.E;
        if (PI_) sH[hsy][hsx] = c.H;
      }
    }
    if (act) {
      Combo c;
      make_combo<MK, PSI, PI_>(M, q, fcu, c);
      if (PSI) { sAPi[ty][tx + RH] = c.aPi; sPs1[ty][tx + RH] = c.ps1; sE[ty + 1][tx] = c.E; }
      if (PI_) { sG1[ty][tx + RH] = c.G1; sQ[ty][tx + RH] = c.Q; sH[ty + 1][tx] = c.H; }
    }
    __syncthreads();
    if (act) {
      make_phi<MK, PSI, PI_>(M, q, fnx, cnx);
      const long long p = pcol + (long long)k * g.plane;
      const int n = g.NI - 1;
      const int sx = tx + RH;
      double2 r[5];
      // ---------------- rhs_phi .. rhs_psi3
      if (PSI) {
        r[0] = cadd(rmul(ldm(M.alpha, q), fcu[4]), rmul(be, fcu[1]));
        double2 d;
        if (ii == 0) d = fwd3(sAPi[ty][sx], sAPi[ty][sx + 1], sAPi[ty][sx + 2]);
        else if (ii == n) d = bwd3(sAPi[ty][sx], sAPi[ty][sx - 1], sAPi[ty][sx - 2]);
        else d = ctr(sAPi[ty][sx - 1], sAPi[ty][sx + 1]);
        d = rmul(g.rdx, d);
        double2 av;
        if (ii <= 1) av = fwd3(sPs1[ty][sx], sPs1[ty][sx + 1], sPs1[ty][sx + 2]);
        else if (ii == n - 1) av = csub(sPs1[ty][sx + 1], sPs1[ty][sx - 1]);
        else if (ii == n) av = bwd3(sPs1[ty][sx], sPs1[ty][sx - 1], sPs1[ty][sx - 2]);
        else if (be > 0.0) av = fwd3(sPs1[ty][sx], sPs1[ty][sx + 1], sPs1[ty][sx + 2]);
        else if (be < 0.0) av = bwd3(sPs1[ty][sx], sPs1[ty][sx - 1], sPs1[ty][sx - 2]);
        else av = csub(sPs1[ty][sx + 1], sPs1[ty][sx - 1]);
        av = rmul(g.rdx, av);
        r[1] = cadd(cadd(d, rmul(be, av)), rmul(dxb, fcu[1]));
        double2 t;
        if (jj == 0) {
          Combo c2v;
          direct_combo<MK, true, false>(g, M, a.in, ii, 2, ktarget(g, k), c2v);
          t = cadd(cneg(sE[ty + 2][tx]), c2v.E);
        } else if (jj == g.NJ - 1) {
          double2 em2;
          if (ty >= 1) em2 = sE[ty - 1][tx];
          else { Combo c2v; direct_combo<MK, true, false>(g, M, a.in, ii, jj - 2, k, c2v); em2 = c2v.E; }
          t = bwd3(sE[ty + 1][tx], sE[ty][tx], em2);
        } else {
          t = ctr(sE[ty][tx], sE[ty + 2][tx]);
        }
        r[2] = rmul(g.rdy, t);
        double2 z;
        if (k == 0) z = cadd(cneg(cpv.E), cnx.E);
        else if (k == g.Nz) z = cadd(cneg(cnx.E), cpv.E);
        else z = ctr(cpv.E, cnx.E);
        r[3] = rmul(g.rdz, z);
      }
      // ---------------- rhs_pi
      if (PI_) {
        double2 d;
        if (ii == 0) d = fwd3(sG1[ty][sx], sG1[ty][sx + 1], sG1[ty][sx + 2]);
        else if (ii == n) d = bwd3(sG1[ty][sx], sG1[ty][sx - 1], sG1[ty][sx - 2]);
        else d = ctr(sG1[ty][sx - 1], sG1[ty][sx + 1]);
        const double2 r1 = cdivm(rmul(g.rdx, d), sg, rs);
        double2 t;
        if (jj == 0) {
          Combo c2v;
          direct_combo<MK, false, true>(g, M, a.in, ii, 2, ktarget(g, k), c2v);
          t = cadd(cneg(sH[ty + 2][tx]), c2v.H);
        } else if (jj == g.NJ - 1) {
          double2 hm2;
          if (ty >= 1) hm2 = sH[ty - 1][tx];
          else { Combo c2v; direct_combo<MK, false, true>(g, M, a.in, ii, jj - 2, k, c2v); hm2 = c2v.H; }
          t = bwd3(sH[ty + 1][tx], sH[ty][tx], hm2);
        } else {
          t = ctr(sH[ty][tx], sH[ty + 2][tx]);
        }
        const double2 r2 = cdivm(rmul(g.rdy, t), sg, rs);
        double2 z;
        if (k == 0) z = cadd(cneg(cpv.F), cnx.F);
        else if (k == g.Nz) z = cadd(cneg(cnx.F), cpv.F);
        else z = ctr(cpv.F, cnx.F);
        z = rmul(g.rdz, z);
        const double2 r3 = (MK == MK_KS) ? cdivm(z, sg, rs) : z;
        const double2 r4 = rmul(dxb, fcu[4]);
        double2 av;
        if (ii <= 1) av = fwd3(sQ[ty][sx], sQ[ty][sx + 1], sQ[ty][sx + 2]);
        else if (ii == n - 1) av = csub(sQ[ty][sx + 1], sQ[ty][sx - 1]);
        else if (ii == n) av = bwd3(sQ[ty][sx], sQ[ty][sx - 1], sQ[ty][sx - 2]);
        else if (be > 0.0) av = fwd3(sQ[ty][sx], sQ[ty][sx + 1], sQ[ty][sx + 2]);
        else if (be < 0.0) av = bwd3(sQ[ty][sx], sQ[ty][sx - 1], sQ[ty][sx - 2]);
        else av = csub(sQ[ty][sx + 1], sQ[ty][sx - 1]);
        av = rmul(g.rdx, av);
        const double2 r5 = cdivm(rmul(be, av), sg, rs);
        const double2 r6 = rmul(am2, fcu[0]);
        r[4] = csub(cadd(cadd(cadd(cadd(r1, r2), r3), r4), r5), r6);
      }
      // ---------------- stage combination
      const double dt = g.dt;
      if (KIND == ST_P2_S1A) {
#pragma unroll
        for (int v = 0; v < 4; ++v) a.out[v * g.fs + p] = cadd(ldf(a.base + v * g.fs, p), rmul(dt, r[v]));
      } else if (KIND == ST_P3_S2A) {
#pragma unroll
        for (int v = 0; v < 4; ++v)
          a.out[v * g.fs + p] = cadd(rmul(0.75, ldf(a.base + v * g.fs, p)), rmul(0.25, cadd(fcu[v], rmul(dt, r[v]))));
      } else if (KIND == ST_P2_S1B) {
        a.out4[p] = cadd(ldf(a.base + 4 * g.fs, p), rmul(dt, r[4]));
      } else if (KIND == ST_P3_S2B) {
        a.out4[p] = cadd(rmul(0.75, ldf(a.base + 4 * g.fs, p)), rmul(0.25, cadd(ldf(a.aux4, p), rmul(dt, r[4]))));
      } else if (!(a.skip_last_i && ii == n)) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const long long o = v * g.fs + p;
          const double2 b = ldf(a.base + v * g.fs, p);
          double2 res;
          if (KIND == ST_P2_S2) {
            res = rmul(0.5, cadd(cadd(b, fcu[v]), rmul(dt, r[v])));
          } else if (KIND == ST_P3_S3) {
            res = cadd(rmul(1.0 / 3.0, b), rmul(2.0 / 3.0, cadd(fcu[v], rmul(dt, r[v]))));
          } else if (KIND == ST_RK3_1) {
            res = cadd(b, rmul(dt, r[v]));
          } else if (KIND == ST_RK3_2) {
            res = cadd(rmul(0.750, b), rmul(0.250, cadd(fcu[v], rmul(dt, r[v]))));
          } else if (KIND == ST_RK3_3) {
            res = cadd(cdivm(b, 3.0, kThird), cdivm(rmul(2.0, cadd(fcu[v], rmul(dt, r[v]))), 3.0, kThird));
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
            res = cadd(b, cdivm(cadd(a.acc[o], kk), 6.0, kSixth));
          }
          a.out[o] = res;
        }
      }
      // roll the phi window
      cpv = ccu;
      ccu = cnx;
#pragma unroll
      for (int v = 0; v < 5; ++v) fcu[v] = fnx[v];
    }
    __syncthreads();
  }
}

static int march_chunk(const Grid& g) {
  // about 32 planes per CTA, spread evenly
  const int nchunks = (g.NK + 31) / 32;
  return (g.NK + nchunks - 1) / nchunks;
}

template <int KIND>
static void march_launch_kind(const MarchArgs& a, int mk, cudaStream_t st) {
  const Grid& g = a.g;
  dim3 block(TI, TJ, 1);
  dim3 grid((g.NI + TI - 1) / TI, (g.NJ + TJ - 1) / TJ, (g.NK + a.kchunk - 1) / a.kchunk);
  if (mk == MK_KS)
    march_kernel<KIND, MK_KS><<<grid, block, 0, st>>>(a);
  else
    march_kernel<KIND, MK_SCHW><<<grid, block, 0, st>>>(a);
}

void launch_stage_march(int kind, const StageLaunch& L, const double* rsg, cudaStream_t st) {
  MarchArgs a;
  a.g = L.g;
  a.m = L.m;
  a.rsg = rsg;
  for (int v = 0; v < 5; ++v) a.in[v] = L.in[v];
  a.base = L.base;
  a.aux4 = L.aux4;
  a.out = L.out;
  a.out4 = L.out4;
  a.acc = L.acc;
  a.skip_last_i = L.skip_last_i;
  a.kchunk = march_chunk(L.g);
  switch (kind) {
    case ST_P2_S1A: march_launch_kind<ST_P2_S1A>(a, L.metric_kind, st); break;
    case ST_P2_S1B: march_launch_kind<ST_P2_S1B>(a, L.metric_kind, st); break;
    case ST_P2_S2: march_launch_kind<ST_P2_S2>(a, L.metric_kind, st); break;
    case ST_P3_S2A: march_launch_kind<ST_P3_S2A>(a, L.metric_kind, st); break;
    case ST_P3_S2B: march_launch_kind<ST_P3_S2B>(a, L.metric_kind, st); break;
    case ST_P3_S3: march_launch_kind<ST_P3_S3>(a, L.metric_kind, st); break;
    case ST_RK3_1: march_launch_kind<ST_RK3_1>(a, L.metric_kind, st); break;
    case ST_RK3_2: march_launch_kind<ST_RK3_2>(a, L.metric_kind, st); break;
    case ST_RK3_3: march_launch_kind<ST_RK3_3>(a, L.metric_kind, st); break;
    case ST_RK4_1: march_launch_kind<ST_RK4_1>(a, L.metric_kind, st); break;
    case ST_RK4_2: march_launch_kind<ST_RK4_2>(a, L.metric_kind, st); break;
    case ST_RK4_3: march_launch_kind<ST_RK4_3>(a, L.metric_kind, st); break;
    case ST_RK4_4: march_launch_kind<ST_RK4_4>(a, L.metric_kind, st); break;
    default: break;
  }
}

}  // namespace kg
