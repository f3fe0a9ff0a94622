// kg_mixed.cu -- mixed-precision RK4 (MoL/lines_method_lib.f90:411-474).
//
// The stencil RHS (rhs_phi .. rhs_pi, MoL/lines_method_lib.f90:671-743) runs in
// FP32 on FP32 stage states; the RK state stays FP64: u^n is read in FP64, the
// stage inputs u^n + c k are formed in FP64 and stored in FP32, the increments
// k = dt rhs are kept as an FP32 sum k1 + 2 k2 + 2 k3, and the update
// u^{n+1} = u^n + (k1 + 2 k2 + 2 k3 + k4) / 6 is computed in FP64.  Points of
// the excision side (r index 0, 1) and of the two interior theta rows next to
// each pole (j = 1, 2 and Ny-2, Ny-1, where the 1/sqrt(gamma) ~ 1/sin(theta)
// factors are largest) evaluate their RHS in FP64 from the same stored values.
//
// Bytes per stored point and step (5 complex variables, 8 B per FP32 value
// pair, 16 B per FP64 pair): stage 1 reads u (80) and writes the stage (40)
// and the sum (40); stages 2 and 3 read the stage (40), u (80) and the sum (40)
// and write the stage (40) and the sum (40); stage 4 reads the stage (40), u
// (80) and the sum (40) and writes u (80): 880 B against 1360 B in FP64.
//
// Kernel organisation is that of the FP64 TMA form: a CTA owns a 32 x 8 (or
// 32 x 4) tile of (r, theta) columns and marches through a chunk of phi planes; each plane
// of the five stencil inputs with its r (+-2) and theta (+-1) halo arrives by
// one cp.async.bulk.tensor box into a 3-deep shared-memory ring tracked by
// mbarriers with bounded waits; the point-wise operands are prefetched into L2
// two planes ahead.  x coordinates of every box are multiples of 16 bytes.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstring>
#include "kg_device.cuh"
#include "kg_internal.h"
#include "kg_tma_ops.cuh"

namespace kg {
using namespace tmaops;
namespace {

constexpr int TI = 32, RH = 2;
constexpr int RW = 2 * (TI + 2 * RH);  // ring row width in elements (two per complex value)
constexpr int NST = 3;
constexpr int MW = TI + 2 * RH;
enum { MT_AL = 0, MT_BE, MT_A, MT_GRR, MT_GRP, MT_SG, MT_HT, MT_COUNT };
// tile geometry for TJ theta rows (one warp per row): 8 (256 threads, 2 CTAs
// per SM) or 4 (128 threads, 3 CTAs per SM)
template <int TJ>
struct MGeom {
  static constexpr int RROWS = TJ + 2;
  static constexpr int FIELD_E = RROWS * RW;
  static constexpr int STAGE_E = 5 * FIELD_E;
  static constexpr int MH = TJ + 2, MT_N = MW * MH;
  // stages 2-4 (FP32 ring) stage their point-wise operands -- u^n (FP64) and the
  // increment sum (FP32), five variables of the thread's own point -- in shared
  // memory with cp.async issued at the start of each plane, so the loads run
  // under the RHS arithmetic instead of after it
  static constexpr int STG_BYTES = TI * TJ * 5 * (16 + 8);
  static constexpr int MIN_BLOCKS = TJ == 4 ? 3 : 2;
  // ring slot stride in elements: TMA destinations start on 128-byte boundaries
  template <class T>
  static __host__ __device__ constexpr int slot_e() {
    return (int)(((STAGE_E * sizeof(T) + 127) / 128) * 128 / sizeof(T));
  }
  template <class T>
  static __host__ __device__ constexpr size_t smem() {
    return (size_t)NST * slot_e<T>() * sizeof(T) + (size_t)MT_COUNT * MT_N * 8 + 64 + 128 +
           (sizeof(T) == 4 ? (size_t)STG_BYTES + (size_t)MT_COUNT * MT_N * 4 : 0);
  }
};

// ---- a complex value in arithmetic type R -----------------------------------
template <class R>
struct cx {
  R x, y;
};
template <class R>
__device__ __forceinline__ cx<R> CX(R a, R b) {
  cx<R> z;
  z.x = a;
  z.y = b;
  return z;
}
template <class R>
__device__ __forceinline__ cx<R> add(cx<R> a, cx<R> b) { return CX<R>(a.x + b.x, a.y + b.y); }
template <class R>
__device__ __forceinline__ cx<R> sub(cx<R> a, cx<R> b) { return CX<R>(a.x - b.x, a.y - b.y); }
template <class R>
__device__ __forceinline__ cx<R> neg(cx<R> a) { return CX<R>(-a.x, -a.y); }
template <class R>
__device__ __forceinline__ cx<R> sm(R s, cx<R> a) { return CX<R>(s * a.x, s * a.y); }
template <class R>
__device__ __forceinline__ cx<R> f3(cx<R> f0, cx<R> f1, cx<R> f2) {
  return sub(add(neg(sm((R)3, f0)), sm((R)4, f1)), f2);
}
template <class R>
__device__ __forceinline__ cx<R> b3(cx<R> f0, cx<R> fm1, cx<R> fm2) {
  return add(sub(sm((R)3, f0), sm((R)4, fm1)), fm2);
}
template <class R>
__device__ __forceinline__ cx<R> cc(cx<R> fm, cx<R> fp) { return add(neg(fm), fp); }
// division by sqrt(gamma): FP64 as the reference form (host reciprocal and one
// Markstein step), FP32 by the FP32 reciprocal
__device__ __forceinline__ cx<double> dsg(cx<double> a, double b, double rb) {
  auto q = [&](double v) {
    const double t = v * rb;
    return __fma_rn(__fma_rn(-t, b, v), rb, t);
  };
  return CX<double>(q(a.x), q(a.y));
}
__device__ __forceinline__ cx<float> dsg(cx<float> a, float, float rb) { return CX<float>(a.x * rb, a.y * rb); }

template <class R, class T>
__device__ __forceinline__ cx<R> ld2(const T* p) {
  return CX<R>((R)p[0], (R)p[1]);
}

struct MxArgs {
  Grid g;
  Metric m;
  const double* rsg;
  const void* in;       // stencil input, 5 variables (stride g.fs complex): double2 in stage 1, float2 after
  const double2* base;  // u^n
  float2* acc;          // k1 + 2 k2 + 2 k3
  float2* outf;         // next stage input (stages 1-3)
  double2* outd;        // u^{n+1} (stage 4)
  int skip_last_i;
  int kchunk;
  int npf;
  int* err;
};

}  // namespace

struct alignas(64) MxItem {
  CUtensorMap tin, tp0, tp1;
  MxArgs a;
  int tiles_x, tiles_y, item0, n_items;
};

namespace {

// RHS of all five variables at the thread's own point, arithmetic in R.
// cu: ring slot of plane k; E/F: phi-derivative arguments at k-1 and k+1.
// FAST: every lane of the warp lies two points inside the array in r with
// beta^r > 0 (in R), so every lane takes the centred derivative and the forward
// upwind difference -- the branches the general form takes there
template <class R, int MK, class TIN, int TJ, bool FAST = false>
__device__ __forceinline__ void mx_rhs(const MxArgs& a, const TIN* cu, const double* mt, const float* mtf, int tx,
                                       int ty, int ii, int jj, int k, const double* own, double2 Epv, double2 Enx,
                                       double2 Fpv, double2 Fnx, cx<R> r[5]) {
  constexpr int FIELD_E = MGeom<TJ>::FIELD_E, MT_N = MGeom<TJ>::MT_N;
  const Grid& g = a.g;
  const Metric& M = a.m;
  const TIN* gin = reinterpret_cast<const TIN*>(a.in);
  const R al = (R)own[0], be = (R)own[1], dxb = (R)own[2], sg = (R)own[3], rs = (R)own[4], am2 = (R)own[5];
  const R rdx = (R)g.rdx, rdy = (R)g.rdy, rdz = (R)g.rdz;
  const int n = g.NI - 1;
  auto RF = [&](int f, int dx, int dy) -> cx<R> {
    return ld2<R>(cu + (size_t)f * FIELD_E + (dy + 1) * RW + 2 * (dx + RH));
  };
  // metric at tile point (dx, dy); the FP32 arithmetic reads the FP32 copy of the
  // tile where there is one (stages with an FP32 ring), without a conversion per use
  auto MTV = [&](int which, int dx, int dy) -> R {
    const int o = which * MT_N + (dy + 1) * MW + dx + RH;
    if (sizeof(R) == 4 && sizeof(TIN) == 4) return (R)mtf[o];
    return (R)mt[o];
  };
  auto G = [&](int v, long long p) -> cx<R> { return ld2<R>(gin + 2 * ((long long)v * g.fs + p)); };
  cx<R> fcu[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) fcu[v] = RF(v, tx, ty);
  // rhs_phi, rhs_psi1 (MoL/lines_method_lib.f90:671-690)
  r[0] = add(sm(al, fcu[4]), sm(be, fcu[1]));
  {
    auto aPi = [&](int dx) { return sm(MTV(MT_AL, tx + dx, ty), RF(4, tx + dx, ty)); };
    auto ps1 = [&](int dx) { return RF(1, tx + dx, ty); };
    cx<R> d;
    if (FAST) d = cc(aPi(-1), aPi(1));
    else if (ii == 0) d = f3(aPi(0), aPi(1), aPi(2));
    else if (ii == n) d = b3(aPi(0), aPi(-1), aPi(-2));
    else d = cc(aPi(-1), aPi(1));
    d = sm(rdx, d);
    cx<R> av;
    if (FAST) av = f3(fcu[1], ps1(1), ps1(2));
    else if (ii <= 1) av = f3(fcu[1], ps1(1), ps1(2));
    else if (ii == n - 1) av = sub(ps1(1), ps1(-1));
    else if (ii == n) av = b3(fcu[1], ps1(-1), ps1(-2));
    else if (be > (R)0) av = f3(fcu[1], ps1(1), ps1(2));
    else if (be < (R)0) av = b3(fcu[1], ps1(-1), ps1(-2));
    else av = sub(ps1(1), ps1(-1));
    av = sm(rdx, av);
    r[1] = add(add(d, sm(be, av)), sm(dxb, fcu[1]));
  }
  // rhs_psi2 (:693-701), theta derivative of alpha Pi + beta psi1
  {
    auto E = [&](int dy) {
      return add(sm(MTV(MT_AL, tx, ty + dy), RF(4, tx, ty + dy)), sm(MTV(MT_BE, tx, ty + dy), RF(1, tx, ty + dy)));
    };
    auto Eg = [&](int j2, int k2) {
      const int q2 = off2(g, ii, j2);
      const long long p2 = off3(g, ii, j2, k2);
      return add(sm((R)ldm(M.alpha, q2), G(4, p2)), sm((R)ldm(M.beta, q2), G(1, p2)));
    };
    cx<R> t;
    if (jj == 0) t = add(neg(E(1)), Eg(2, ktarget(g, k)));
    else if (jj == g.NJ - 1) t = b3(E(0), E(-1), (ty >= 1) ? E(-2) : Eg(jj - 2, k));
    else t = cc(E(-1), E(1));
    r[2] = sm(rdy, t);
  }
  // rhs_psi3 (:704-713)
  {
    const cx<R> ep = CX<R>((R)Epv.x, (R)Epv.y), en = CX<R>((R)Enx.x, (R)Enx.y);
    cx<R> z;
    if (k == 0) z = add(neg(ep), en);
    else if (k == g.Nz) z = add(neg(en), ep);
    else z = cc(ep, en);
    r[3] = sm(rdz, z);
  }
  // rhs_pi (:727-743)
  {
    auto G1 = [&](int dx) {
      if (MK == MK_KS)
        return sm(MTV(MT_A, tx + dx, ty),
                  add(sm(MTV(MT_GRR, tx + dx, ty), RF(1, tx + dx, ty)), sm(MTV(MT_GRP, tx + dx, ty), RF(3, tx + dx, ty))));
      return sm(MTV(MT_A, tx + dx, ty), RF(1, tx + dx, ty));
    };
    cx<R> d;
    if (FAST) d = cc(G1(-1), G1(1));
    else if (ii == 0) d = f3(G1(0), G1(1), G1(2));
    else if (ii == n) d = b3(G1(0), G1(-1), G1(-2));
    else d = cc(G1(-1), G1(1));
    const cx<R> r1 = dsg(sm(rdx, d), sg, rs);
    auto H = [&](int dy) { return sm(MTV(MT_HT, tx, ty + dy), RF(2, tx, ty + dy)); };
    auto Hg = [&](int j2, int k2) { return sm((R)ldm(M.asg_gtt, off2(g, ii, j2)), G(2, off3(g, ii, j2, k2))); };
    cx<R> t;
    if (jj == 0) t = add(neg(H(1)), Hg(2, ktarget(g, k)));
    else if (jj == g.NJ - 1) t = b3(H(0), H(-1), (ty >= 1) ? H(-2) : Hg(jj - 2, k));
    else t = cc(H(-1), H(1));
    const cx<R> r2 = dsg(sm(rdy, t), sg, rs);
    const cx<R> fp = CX<R>((R)Fpv.x, (R)Fpv.y), fn = CX<R>((R)Fnx.x, (R)Fnx.y);
    cx<R> z;
    if (k == 0) z = add(neg(fp), fn);
    else if (k == g.Nz) z = add(neg(fn), fp);
    else z = cc(fp, fn);
    z = sm(rdz, z);
    const cx<R> r3 = (MK == MK_KS) ? dsg(z, sg, rs) : z;
    const cx<R> r4 = sm(dxb, fcu[4]);
    auto Q = [&](int dx) { return sm(MTV(MT_SG, tx + dx, ty), RF(4, tx + dx, ty)); };
    cx<R> av;
    if (FAST) av = f3(Q(0), Q(1), Q(2));
    else if (ii <= 1) av = f3(Q(0), Q(1), Q(2));
    else if (ii == n - 1) av = sub(Q(1), Q(-1));
    else if (ii == n) av = b3(Q(0), Q(-1), Q(-2));
    else if (be > (R)0) av = f3(Q(0), Q(1), Q(2));
    else if (be < (R)0) av = b3(Q(0), Q(-1), Q(-2));
    else av = sub(Q(1), Q(-1));
    av = sm(rdx, av);
    const cx<R> r5 = dsg(sm(be, av), sg, rs);
    const cx<R> r6 = sm(am2, fcu[0]);
    r[4] = sub(add(add(add(add(r1, r2), r3), r4), r5), r6);
  }
}

// phi-derivative arguments at the own point of a ring slot, in R, widened
template <class R, int MK, class TIN, int TJ>
__device__ __forceinline__ void mx_EF(const TIN* st, int tx, int ty, const double* own, double2& E, double2& F) {
  constexpr int FIELD_E = MGeom<TJ>::FIELD_E;
  auto RF = [&](int f) -> cx<R> { return ld2<R>(st + (size_t)f * FIELD_E + (ty + 1) * RW + 2 * (tx + RH)); };
  const R al = (R)own[0], be = (R)own[1], fa = (R)own[6], fgrp = (R)own[7], fgpp = (R)own[8];
  const cx<R> e = add(sm(al, RF(4)), sm(be, RF(1)));
  cx<R> f;
  if (MK == MK_KS) f = sm(fa, add(sm(fgrp, RF(1)), sm(fgpp, RF(3))));
  else f = sm(fa, RF(3));
  E = make_double2((double)e.x, (double)e.y);
  F = make_double2((double)f.x, (double)f.y);
}

template <int KIND, int MK, class TIN, int TJ>
__device__ __forceinline__ int mx_item(const CUtensorMap* tinp, const CUtensorMap* tp0p, const CUtensorMap* tp1p,
                                       const MxArgs& a, int bx, int by, int bz, TIN* ring, double* mt,
                                       uint64_t* bars, uint32_t tb, unsigned char* stg) {
  using GT = MGeom<TJ>;
  constexpr int FIELD_E = GT::FIELD_E, STAGE_E = GT::STAGE_E, MT_N = GT::MT_N;
  constexpr bool STG = sizeof(TIN) == 4;
  double2* base_s = reinterpret_cast<double2*>(stg);
  float2* acc_s = reinterpret_cast<float2*>(stg + (size_t)TI * TJ * 5 * 16);
  // FP32 copy of the metric tile (stages with an FP32 ring; it sits after the FP64 tile)
  float* mtf = reinterpret_cast<float*>(mt + (size_t)MT_COUNT * MT_N);
  const Grid& g = a.g;
  const Metric& M = a.m;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TI + tx;
  const int ii0 = bx * TI, jj0 = by * TJ;
  const int ii = ii0 + tx, jj = jj0 + ty;
  const bool act = (ii < g.NI) && (jj < g.NJ);
  // ring slot protocol: full[s] completes when a plane's box has landed (one
  // expect_tx arrival + the bytes); empty[s] when every warp has read the plane
  // for the last time (one arrival per warp), after which thread 0 may load the
  // next plane into the slot -- warps are not held at a block barrier per plane
  uint64_t* empty = bars + NST;
  const int lane = tid & 31;
  auto release = [&](int t) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[(tb + (uint32_t)t) % NST]);
  };
  const int k0 = bz * a.kchunk;
  if (k0 >= g.NK) return 0;
  const int k1 = min(k0 + a.kchunk, g.NK);
  const int nplanes = (k1 - k0) + 2;
  auto plane_of = [&](int t) -> int {
    if (t == 0) return (k0 == 0) ? g.Nz - 2 : k0 - 1;
    if (t <= k1 - k0) return k0 + t - 1;
    return (k1 - 1 == g.Nz) ? 2 : k1;
  };
  auto slot = [&](int t) -> int { return (int)((tb + (uint32_t)t) % NST); };
  auto parity = [&](int t) -> uint32_t { return ((tb + (uint32_t)t) / NST) & 1u; };
  auto issue = [&](int t) {
    const int s = slot(t);
    mbar_expect_tx(&bars[s], (uint32_t)(STAGE_E * sizeof(TIN)));
    tma_load_4d(ring + (size_t)s * GT::template slot_e<TIN>(), tinp, 2 * (ii0 - RH), jj0 - 1, plane_of(t), 0,
                &bars[s]);
  };
  // the first planes are requested before the metric tile is loaded, so the
  // copies are in flight while the tile loads (the ring is free: every warp
  // finished the previous item before this one started)
  auto prefetch = [&](int k) {
    if (k >= k1) return;
    if (a.npf > 0) tma_prefetch_4d(tp0p, 2 * ii0, jj0, k, 0);
    if (a.npf > 1) tma_prefetch_4d(tp1p, 2 * ii0, jj0, k, 0);
  };
  int nissued = 0;
  if (tid == 0) {
    for (int t = 0; t < NST && t < nplanes; ++t) {
      issue(t);
      nissued = t + 1;
    }
    prefetch(k0);
    prefetch(k0 + 1);
  }
  for (int t = tid; t < MT_N; t += TI * TJ) {
    const int mx = t % MW, my = t / MW;
    const int gi = ii0 - RH + mx, gj = jj0 - 1 + my;
    const bool in = gi >= 0 && gi < g.NI && gj >= 0 && gj < g.NJ;
    const int q = in ? off2(g, gi, gj) : 0;
    mt[MT_AL * MT_N + t] = in ? ldm(M.alpha, q) : 0.0;
    mt[MT_BE * MT_N + t] = in ? ldm(M.beta, q) : 0.0;
    mt[MT_A * MT_N + t] = in ? ldm(MK == MK_KS ? M.asg : M.asg_grr, q) : 0.0;
    mt[MT_GRR * MT_N + t] = in ? ldm(M.grr, q) : 0.0;
    mt[MT_GRP * MT_N + t] = in ? ldm(M.grp, q) : 0.0;
    mt[MT_SG * MT_N + t] = in ? ldm(M.sqrtg, q) : 0.0;
    mt[MT_HT * MT_N + t] = in ? ldm(M.asg_gtt, q) : 0.0;
    if (STG)
      for (int w = 0; w < MT_COUNT; ++w) mtf[w * MT_N + t] = (float)mt[w * MT_N + t];
  }
  __syncthreads();
  // own-point metric: alpha, beta, d_r beta, sqrt(gamma), 1/sqrt(gamma), alpha m^2, phi-flux factors
  double own[9] = {0, 0, 0, 1, 1, 0, 0, 0, 0};
  if (act) {
    const int q = off2(g, ii, jj);
    own[0] = ldm(M.alpha, q);
    own[1] = ldm(M.beta, q);
    own[2] = ldm(M.dxbeta, q);
    own[3] = ldm(M.sqrtg, q);
    own[4] = ldm(a.rsg, q);
    own[5] = ldm(M.am2, q);
    if (MK == MK_KS) {
      own[6] = ldm(M.asg, q);
      own[7] = ldm(M.grp, q);
      own[8] = ldm(M.gpp, q);
    } else {
      own[6] = ldm(M.a_gpp, q);
    }
  }
  // FP64 RHS at the excision side (r index 0, 1) and on the two interior theta
  // rows next to each pole (stored rows 3, 4 and NJ-5, NJ-4: j = 1, 2 and Ny-2,
  // Ny-1, where 1/sqrt(gamma) ~ 1/sin(theta) is largest).  The three stored rows
  // beyond each pole are ghost rows, which the pole fill overwrites from interior
  // rows after every stage, so their RHS stays in FP32.
  const bool hp = (ii <= 1) || (jj == 3) || (jj == 4) || (jj == g.NJ - 5) || (jj == g.NJ - 4);
  const bool fast =
      __all_sync(0xffffffffu, act && !hp && ii <= g.NI - 3 && (float)own[1] > 0.0f);  // warp-uniform
  auto EF = [&](const TIN* st, double2& E, double2& F) {
    if (hp) mx_EF<double, MK, TIN, TJ>(st, tx, ty, own, E, F);
    else mx_EF<float, MK, TIN, TJ>(st, tx, ty, own, E, F);
  };
  const long long pcol = act ? off3(g, ii, jj, 0) : 0;
  int timed_out = 0;
  double2 Epv = make_double2(0, 0), Fpv = Epv, Ecu = Epv, Fcu = Epv;
  if (!mbar_wait_bounded(&bars[slot(0)], parity(0))) timed_out = 1;
  if (act && !timed_out) EF(ring + (size_t)slot(0) * GT::template slot_e<TIN>(), Epv, Fpv);
  release(0);
  bool failed = __syncthreads_or(timed_out) != 0;
  const int last = k1 - k0 - 1;

  for (int i = 0; i <= last && !failed; ++i) {
    const int k = k0 + i;
    if (tid == 0 && !timed_out) {
      if (i + NST < nplanes) {
        // plane i shares the slot; every warp released it after its last use
        if (mbar_wait_bounded(&empty[slot(i)], parity(i))) {
          issue(i + NST);
          nissued = i + NST + 1;
        } else {
          timed_out = 1;
        }
      }
      prefetch(k + 2);
    }
    if (STG && act) {
      const long long p0 = pcol + (long long)k * g.plane;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        cp_async16(&base_s[v * TI * TJ + tid], a.base + (long long)v * g.fs + p0);
        cp_async8(&acc_s[v * TI * TJ + tid], a.acc + (long long)v * g.fs + p0);
      }
      cp_async_commit();
    }
    const int tc = i + 1, tn = i + 2;
    if (!timed_out) {
      const bool okc = mbar_wait_bounded(&bars[slot(tc)], parity(tc));
      const bool okn = okc && mbar_wait_bounded(&bars[slot(tn)], parity(tn));
      if (!okn) timed_out = 1;
    }
    if (act && !timed_out) {
      const TIN* cu = ring + (size_t)slot(tc) * GT::template slot_e<TIN>();
      const TIN* nx = ring + (size_t)slot(tn) * GT::template slot_e<TIN>();
      if (i == 0) EF(cu, Ecu, Fcu);
      double2 Enx, Fnx;
      EF(nx, Enx, Fnx);
      double2 rr[5];
      if (hp) {
        cx<double> r[5];
        mx_rhs<double, MK, TIN, TJ>(a, cu, mt, mtf, tx, ty, ii, jj, k, own, Epv, Enx, Fpv, Fnx, r);
#pragma unroll
        for (int v = 0; v < 5; ++v) rr[v] = make_double2(r[v].x, r[v].y);
      } else {
        cx<float> r[5];
        if (fast) mx_rhs<float, MK, TIN, TJ, true>(a, cu, mt, mtf, tx, ty, ii, jj, k, own, Epv, Enx, Fpv, Fnx, r);
        else mx_rhs<float, MK, TIN, TJ, false>(a, cu, mt, mtf, tx, ty, ii, jj, k, own, Epv, Enx, Fpv, Fnx, r);
#pragma unroll
        for (int v = 0; v < 5; ++v) rr[v] = make_double2((double)r[v].x, (double)r[v].y);
      }
      const long long p = pcol + (long long)k * g.plane;
      const int n = g.NI - 1;
      const double dt = g.dt;
      if (STG) cp_async_wait_all();
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const long long o = (long long)v * g.fs + p;
        const double2 kk = rmul(dt, rr[v]);
        double2 b;
        if (KIND == ST_RK4_1) {
          const TIN* e = cu + (size_t)v * FIELD_E + (ty + 1) * RW + 2 * (tx + RH);
          b = make_double2((double)e[0], (double)e[1]);  // the stencil input is u^n itself
        } else if (STG) {
          b = base_s[v * TI * TJ + tid];
        } else {
          b = ldf(a.base, o);
        }
        if (KIND == ST_RK4_1) {
          a.acc[o] = make_float2((float)kk.x, (float)kk.y);
          const double2 s = cadd(b, rmul(0.50, kk));
          a.outf[o] = make_float2((float)s.x, (float)s.y);
        } else if (KIND == ST_RK4_2 || KIND == ST_RK4_3) {
          const float2 av = STG ? acc_s[v * TI * TJ + tid] : a.acc[o];
          const double2 acc = cadd(make_double2((double)av.x, (double)av.y), rmul(2.0, kk));
          a.acc[o] = make_float2((float)acc.x, (float)acc.y);
          const double2 s = (KIND == ST_RK4_2) ? cadd(b, rmul(0.50, kk)) : cadd(b, kk);
          a.outf[o] = make_float2((float)s.x, (float)s.y);
        } else if (!(a.skip_last_i && ii == n)) {
          const float2 av = STG ? acc_s[v * TI * TJ + tid] : a.acc[o];
          // u^n + (k1 + 2 k2 + 2 k3 + k4) / 6 in FP64, the 1/6 as a product: this form is not
          // bit-matched to the reference, and a division per component costs the stage ~30 %
          a.outd[o] = cadd(b, rmul(1.0 / 6.0, cadd(make_double2((double)av.x, (double)av.y), kk)));
        }
      }
      Epv = Ecu;
      Fpv = Fcu;
      Ecu = Enx;
      Fcu = Fnx;
    }
    release(i + 1);
    if (i == last) release(i + 2);
  }
  failed = __syncthreads_or(timed_out) != 0;
  if (STG) cp_async_wait_all();  // no staged copy outlives the item
  if (failed) {
    if (tid == 0) {
      atomicExch(a.err, 1);
      for (int s = 0; s < NST; ++s) {
        int tl = -1;
        for (int t = 0; t < nissued; ++t)
          if (slot(t) == s) tl = t;
        if (tl >= 0) (void)mbar_wait_bounded(&bars[s], parity(tl));
      }
    }
    __syncthreads();
    return -1;
  }
  return nplanes;
}

__device__ __forceinline__ unsigned char* align128(unsigned char* p) {
  const uint32_t a = saddr(p);
  return p + ((128u - (a & 127u)) & 127u);
}

template <int TJ>
__device__ __forceinline__ void init_bars(uint64_t* bars) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bars[s], 1);
    for (int s = 0; s < NST; ++s) mbar_init(&bars[NST + s], TJ);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

}  // namespace

template <int KIND, int MK, class TIN, int TJ>
__global__ void __launch_bounds__(TI * TJ, MGeom<TJ>::MIN_BLOCKS)
    mx_stage_kernel(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tp0,
                    const __grid_constant__ CUtensorMap tp1, MxArgs a) {
  using GT = MGeom<TJ>;
  constexpr int MT_N = GT::MT_N;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TIN* ring = reinterpret_cast<TIN*>(align128(smem_raw));
  double* mt = reinterpret_cast<double*>(ring + (size_t)NST * GT::template slot_e<TIN>());
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(mt + (size_t)MT_COUNT * MT_N) +
                                               (sizeof(TIN) == 4 ? (size_t)MT_COUNT * MT_N * 4 : 0));
  unsigned char* stg = reinterpret_cast<unsigned char*>(bars + 8);
  if ((int)blockIdx.z * a.kchunk >= a.g.NK) return;
  init_bars<TJ>(bars);
  (void)mx_item<KIND, MK, TIN, TJ>(&tin, &tp0, &tp1, a, blockIdx.x, blockIdx.y, blockIdx.z, ring, mt, bars, 0u, stg);
}

template <int KIND, int MK, class TIN, int TJ>
__global__ void __launch_bounds__(TI * TJ, MGeom<TJ>::MIN_BLOCKS)
    mx_batch_kernel(const MxItem* __restrict__ solves, int n_solves, int n_items) {
  using GT = MGeom<TJ>;
  constexpr int MT_N = GT::MT_N;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TIN* ring = reinterpret_cast<TIN*>(align128(smem_raw));
  double* mt = reinterpret_cast<double*>(ring + (size_t)NST * GT::template slot_e<TIN>());
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(mt + (size_t)MT_COUNT * MT_N) +
                                               (sizeof(TIN) == 4 ? (size_t)MT_COUNT * MT_N * 4 : 0));
  unsigned char* stg = reinterpret_cast<unsigned char*>(bars + 8);
  __shared__ MxArgs sa;
  __shared__ int s_bx, s_by, s_bz, s_solve;
  init_bars<TJ>(bars);
  uint32_t tb = 0;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      int lo = 0, hi = n_solves - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (solves[mid].item0 <= item) lo = mid;
        else hi = mid - 1;
      }
      const MxItem& B = solves[lo];
      const int local = item - B.item0;
      s_solve = lo;
      s_bx = local % B.tiles_x;
      s_by = (local / B.tiles_x) % B.tiles_y;
      s_bz = local / (B.tiles_x * B.tiles_y);
      sa = B.a;
    }
    __syncthreads();
    const MxItem& B = solves[s_solve];
    const int used = mx_item<KIND, MK, TIN, TJ>(&B.tin, &B.tp0, &B.tp1, sa, s_bx, s_by, s_bz, ring, mt, bars, tb, stg);
    if (used < 0) break;
    tb += (uint32_t)used;
    __syncthreads();
  }
}

// ---- FP32 stage states: ghost-zone, pole and outer-boundary fills ----------
// Same points and order as the FP64 fill (boundary_xL .. boundary_zR,
// MoL/lines_method_lib.f90:507-597); the excision extrapolation
// 3 u1 - 3 u2 + u3 is formed in FP64, the inflow hold reads u^n (FP64).
__device__ __forceinline__ float2 xval_f(const Grid& g, const float2* u, const double2* up, int inflow, int ii,
                                         int jj, int k) {
  if (ii == 0) {
    const float2 a = u[off3(g, 1, jj, k)], b = u[off3(g, 2, jj, k)], c = u[off3(g, 3, jj, k)];
    const double rx = (3.0 * (double)a.x - 3.0 * (double)b.x) + (double)c.x;
    const double ry = (3.0 * (double)a.y - 3.0 * (double)b.y) + (double)c.y;
    return make_float2((float)rx, (float)ry);
  }
  if (ii == g.NI - 1) {
    if (inflow) {
      const double2 v = up[off3(g, ii, jj, k)];
      return make_float2((float)v.x, (float)v.y);
    }
    return u[off3(g, ii - 1, jj, k)];
  }
  return u[off3(g, ii, jj, k)];
}

__device__ __forceinline__ int src_row(const Grid& g, int jj) { return (jj <= 2) ? (5 - jj) : (2 * g.NJ - 7 - jj); }

struct GhostF {
  Grid g;
  float2* u;
  const double2* up;
  int inflow;
};

__global__ void ghost_xy_f32(const GhostF* __restrict__ d) {
  const GhostF& D = d[blockIdx.y];
  const Grid& g = D.g;
  const long long n_rows = 6LL * g.NK * g.NI;
  const long long n_faces = 2LL * (g.NJ - 6) * g.NK;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n_rows + n_faces;
       t += (long long)gridDim.x * blockDim.x) {
    int ii, jj, k, si, sj, sk;
    if (t < n_rows) {
      ii = (int)(t % g.NI);
      const long long rk = t / g.NI;
      const int r = (int)(rk % 6);
      k = (int)(rk / 6);
      jj = (r < 3) ? r : (g.NJ - 6 + r);
      si = ii;
      sj = src_row(g, jj);
      sk = ktarget(g, k);
    } else {
      const long long f = t - n_rows;
      const int nin = g.NJ - 6;
      jj = 3 + (int)(f % nin);
      const long long s2 = f / nin;
      const int side = (int)(s2 % 2);
      k = (int)(s2 / 2);
      ii = side ? g.NI - 1 : 0;
      si = ii;
      sj = jj;
      sk = k;
    }
#pragma unroll
    for (int v = 0; v < 5; ++v)
      D.u[v * g.fs + off3(g, ii, jj, k)] = xval_f(g, D.u + v * g.fs, D.up + v * g.fs, D.inflow, si, sj, sk);
  }
}

__global__ void ghost_z_f32(const GhostF* __restrict__ d) {
  const GhostF& D = d[blockIdx.y];
  const Grid& g = D.g;
  const long long n = (long long)g.NI * g.NJ;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int side = (int)(t / n);
    const long long q = t % n;
    const int ii = (int)(q % g.NI), jj = (int)(q / g.NI);
    const int kd = side ? g.Nz : 0;
    const int ks = side ? 1 : g.Nz - 1;
#pragma unroll
    for (int v = 0; v < 5; ++v) D.u[v * g.fs + off3(g, ii, jj, kd)] = D.u[v * g.fs + off3(g, ii, jj, ks)];
  }
}

// ---------------------------------------------------------------------------
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn enc_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 4-D view of a 5-variable state in element type of `esize` bytes (8 or 4):
// x = elements along r (two per complex value), theta rows, phi planes, variables
bool enc(CUtensorMap* tm, const Grid& g, const void* base, int esize, bool halo, int tj) {
  EncodeTiledFn fn = enc_fn();
  if (!fn) return false;
  const cuuint64_t cb = 2 * (cuuint64_t)esize;  // bytes per complex value
  cuuint64_t dims[4] = {(cuuint64_t)(2 * g.PI), (cuuint64_t)g.NJ, (cuuint64_t)g.NK, 5};
  cuuint64_t strides[3] = {(cuuint64_t)g.PI * cb, (cuuint64_t)g.plane * cb, (cuuint64_t)g.fs * cb};
  cuuint32_t box[4] = {halo ? (cuuint32_t)RW : (cuuint32_t)(2 * TI), (cuuint32_t)(halo ? tj + 2 : tj), 1, 5u};
  cuuint32_t es[4] = {1, 1, 1, 1};
  return fn(tm, esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void*)base, dims,
            strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int mx_chunk(const Grid& g) {
  const int nchunks = (g.NK + 31) / 32;
  return (g.NK + nchunks - 1) / nchunks;
}

// maps and arguments of one solve's stage
int mx_prepare(int kind, const MixedLaunch& L, const double* rsg, int* err, int kchunk, int tj, CUtensorMap* tin,
               CUtensorMap* tp0, CUtensorMap* tp1, MxArgs* a) {
  const bool first = kind == ST_RK4_1;
  if (!enc(tin, L.g, first ? (const void*)L.base : (const void*)L.in_f, first ? 8 : 4, true, tj)) return -1;
  int npf = 0;
  if (!first) {
    if (enc(tp0, L.g, L.base, 8, false, tj)) ++npf;
    if (npf == 1 && enc(tp1, L.g, L.acc, 4, false, tj)) ++npf;
  }
  if (npf < 2) *tp1 = *tin;
  if (npf < 1) *tp0 = *tin;
  a->g = L.g;
  a->m = L.m;
  a->rsg = rsg;
  a->in = first ? (const void*)L.base : (const void*)L.in_f;
  a->base = L.base;
  a->acc = L.acc;
  a->outf = L.out_f;
  a->outd = L.out_d;
  a->skip_last_i = L.skip_last_i;
  a->kchunk = kchunk;
  a->npf = npf;
  a->err = err;
  return 0;
}

template <int KIND, int MK, class TIN, int TJ>
int mx_launch_one(const CUtensorMap& tin, const CUtensorMap& tp0, const CUtensorMap& tp1, const MxArgs& a,
                  cudaStream_t st) {
  constexpr size_t SMEM = MGeom<TJ>::template smem<TIN>();
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(mx_stage_kernel<KIND, MK, TIN, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)SMEM) != cudaSuccess)
      return -1;
    attr = true;
  }
  const Grid& g = a.g;
  dim3 grid((g.NI + TI - 1) / TI, (g.NJ + TJ - 1) / TJ, (g.NK + a.kchunk - 1) / a.kchunk);
  mx_stage_kernel<KIND, MK, TIN, TJ><<<grid, dim3(TI, TJ, 1), SMEM, st>>>(tin, tp0, tp1, a);
  return 0;
}

template <int MK, int TJ>
int mx_launch_mk(int kind, const CUtensorMap& tin, const CUtensorMap& tp0, const CUtensorMap& tp1, const MxArgs& a,
                 cudaStream_t st) {
  switch (kind) {
    case ST_RK4_1: return mx_launch_one<ST_RK4_1, MK, double, TJ>(tin, tp0, tp1, a, st);
    case ST_RK4_2: return mx_launch_one<ST_RK4_2, MK, float, TJ>(tin, tp0, tp1, a, st);
    case ST_RK4_3: return mx_launch_one<ST_RK4_3, MK, float, TJ>(tin, tp0, tp1, a, st);
    case ST_RK4_4: return mx_launch_one<ST_RK4_4, MK, float, TJ>(tin, tp0, tp1, a, st);
    default: return -1;
  }
}

template <int KIND, int MK, class TIN, int TJ>
int mx_batch_one(const void* items, int n_solves, int n_items, int blocks, cudaStream_t st) {
  constexpr size_t SMEM = MGeom<TJ>::template smem<TIN>();
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(mx_batch_kernel<KIND, MK, TIN, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)SMEM) != cudaSuccess)
      return -1;
    attr = true;
  }
  if (n_items <= 0) return 0;
  mx_batch_kernel<KIND, MK, TIN, TJ><<<blocks, dim3(TI, TJ, 1), SMEM, st>>>(reinterpret_cast<const MxItem*>(items),
                                                                           n_solves, n_items);
  return 0;
}

template <int MK, int TJ>
int mx_batch_mk(int kind, const void* items, int n_solves, int n_items, int blocks, cudaStream_t st) {
  switch (kind) {
    case ST_RK4_1: return mx_batch_one<ST_RK4_1, MK, double, TJ>(items, n_solves, n_items, blocks, st);
    case ST_RK4_2: return mx_batch_one<ST_RK4_2, MK, float, TJ>(items, n_solves, n_items, blocks, st);
    case ST_RK4_3: return mx_batch_one<ST_RK4_3, MK, float, TJ>(items, n_solves, n_items, blocks, st);
    case ST_RK4_4: return mx_batch_one<ST_RK4_4, MK, float, TJ>(items, n_solves, n_items, blocks, st);
    default: return -1;
  }
}

}  // namespace

int launch_stage_mixed(int kind, const MixedLaunch& L, const double* rsg, int* err, cudaStream_t st, int tj) {
  if (tj != 4) tj = 8;
  CUtensorMap tin, tp0, tp1;
  MxArgs a;
  if (mx_prepare(kind, L, rsg, err, mx_chunk(L.g), tj, &tin, &tp0, &tp1, &a)) return -1;
  if (tj == 4)
    return L.metric_kind == MK_KS ? mx_launch_mk<MK_KS, 4>(kind, tin, tp0, tp1, a, st)
                                  : mx_launch_mk<MK_SCHW, 4>(kind, tin, tp0, tp1, a, st);
  return L.metric_kind == MK_KS ? mx_launch_mk<MK_KS, 8>(kind, tin, tp0, tp1, a, st)
                                : mx_launch_mk<MK_SCHW, 8>(kind, tin, tp0, tp1, a, st);
}

size_t mixed_item_bytes() { return sizeof(MxItem); }

int build_mixed_item(void* dst, int kind, const MixedLaunch& L, const double* rsg, int* err, int kchunk, int item0,
                     int tj) {
  {  // equal chunks of at most the requested length (as in the FP64 batch)
    const int nch = (L.g.NK + kchunk - 1) / kchunk;
    kchunk = (L.g.NK + nch - 1) / nch;
  }
  MxItem* B = reinterpret_cast<MxItem*>(dst);
  memset(B, 0, sizeof(MxItem));
  if (mx_prepare(kind, L, rsg, err, kchunk, tj, &B->tin, &B->tp0, &B->tp1, &B->a)) return -1;
  B->tiles_x = (L.g.NI + TI - 1) / TI;
  B->tiles_y = (L.g.NJ + tj - 1) / tj;
  B->item0 = item0;
  B->n_items = B->tiles_x * B->tiles_y * ((L.g.NK + kchunk - 1) / kchunk);
  return B->n_items;
}

int launch_batch_mixed(int kind, int mk, const void* d_items, int n_solves, int n_items, int blocks, int tj,
                       cudaStream_t st) {
  if (tj == 4)
    return mk == MK_KS ? mx_batch_mk<MK_KS, 4>(kind, d_items, n_solves, n_items, blocks, st)
                       : mx_batch_mk<MK_SCHW, 4>(kind, d_items, n_solves, n_items, blocks, st);
  if (tj != 8) return -1;
  return mk == MK_KS ? mx_batch_mk<MK_KS, 8>(kind, d_items, n_solves, n_items, blocks, st)
                     : mx_batch_mk<MK_SCHW, 8>(kind, d_items, n_solves, n_items, blocks, st);
}

size_t ghost_f32_desc_bytes() { return sizeof(GhostF); }

void fill_ghost_f32_desc(void* dst, const Grid& g, float2* u, const double2* up, int inflow) {
  GhostF* d = reinterpret_cast<GhostF*>(dst);
  d->g = g;
  d->u = u;
  d->up = up;
  d->inflow = inflow;
}

void launch_ghost_fill_f32(const void* d_desc, int n, long long max_rows, long long max_faces, long long max_z,
                           cudaStream_t st) {
  if (n <= 0) return;
  long long bx = (max_rows + max_faces + 255) / 256;
  bx = bx > 1024 ? 1024 : (bx < 1 ? 1 : bx);
  ghost_xy_f32<<<dim3((unsigned)bx, n), 256, 0, st>>>(reinterpret_cast<const GhostF*>(d_desc));
  long long bz = (max_z + 255) / 256;
  bz = bz > 1024 ? 1024 : (bz < 1 ? 1 : bz);
  ghost_z_f32<<<dim3((unsigned)bz, n), 256, 0, st>>>(reinterpret_cast<const GhostF*>(d_desc));
}

}  // namespace kg
