// kg_tma.cu -- TMA-pipelined form of the fused RHS + stage kernels.
//
// Same arithmetic as kg_stencil.cu and kg_march.cu, bit for bit; the memory
// side is organised for Blackwell:
//   * a CTA owns a 32 x 8 tile of (r, theta) columns (32 x 4 for the RK4
//     stages when asked: twice the tiles of a small grid) and marches through
//     a chunk of phi planes; a warp whose lanes all lie two points inside the
//     array in r with beta^r > 0 takes the centred and forward-upwind
//     differences without per-lane branches;
//   * every plane the CTA needs -- the tile with a +-2 r halo and a +-1 theta
//     halo, all five stencil inputs -- is brought into a 3-deep shared-memory
//     ring by the tensor-memory accelerator (cp.async.bulk.tensor, two boxes
//     per plane: variables 1-4 and the Pi variable, which the PIRK stages keep
//     in a separate slot), completion tracked by one mbarrier per ring slot;
//     while the CTA computes plane k, the loads of planes k+1 and k+2 are in
//     flight, so HBM latency is hidden without holding prefetched values in
//     registers;
//   * the phi-derivative arguments of the thread's own column roll in
//     registers; r and theta neighbours are read from the ring and combined
//     with a per-CTA metric tile that is loaded once (the metric is
//     phi-independent);
//   * divisions by sqrt(gamma) use the correctly rounded host reciprocal and
//     one Markstein step (see kg_march.cu), equal to IEEE division for
//     dividends above about 2^-1000 in magnitude.
// All TMA coordinates are multiples of 16 bytes in x (the r axis is addressed
// in doubles, two per complex value) and the boxes start at most 2 points
// before the array or one row above it, where the loads read zeros.  Waits on
// the mbarriers are bounded: a CTA that runs out sets the error flag, waits
// (bounded) for its own copies and returns; the host reports KG_ETIMEOUT.
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
template <bool B>
struct TBool {
  static constexpr bool value = B;
};
constexpr int RW = 2 * (TI + 2 * RH);  // ring row width in doubles (72 = 576 B)
constexpr int NST = 3;                 // ring depth
constexpr int MW = TI + 2 * RH;        // metric tile width
enum { MT_AL = 0, MT_BE, MT_A, MT_GRR, MT_GRP, MT_SG, MT_HT, MT_COUNT };
// tile geometry for TJ theta rows (one warp per row): 8 (256 threads, 2 CTAs
// per SM) or 4 (128 threads, 3 CTAs per SM, twice the tiles of a grid)
template <int TJ>
struct Geom {
  static constexpr int RROWS = TJ + 2;             // theta rows with halo
  static constexpr int FIELD_D = RROWS * RW;       // doubles per variable per plane
  static constexpr int STAGE_D = 5 * FIELD_D;      // doubles per ring slot
  static constexpr int STAGE_B = STAGE_D * 8;      // 28800 bytes at TJ = 8
  static constexpr int MH = TJ + 2, MT_N = MW * MH;  // metric tile
  static constexpr size_t SMEM_BYTES = (size_t)NST * STAGE_B + (size_t)MT_COUNT * MT_N * 8 + 64 + 128;
  static constexpr int MIN_BLOCKS = TJ == 4 ? 3 : 2;
};
__device__ __forceinline__ double ddiv(double a, double b, double rb) {
  const double q = a * rb;
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, rb, q);
}
__device__ __forceinline__ double2 cdivm(double2 a, double b, double rb) {
  return c2(ddiv(a.x, b, rb), ddiv(a.y, b, rb));
}
// the stage combinations' divisions by 3 (SSP-RK3) and 6 (RK4) take the same
// route, from the correctly rounded reciprocals: equal to IEEE division for every
// finite dividend in the case of 3, for dividends above 2^-1000 in that of 6
// (2e8 random operands over all exponents)
constexpr double kThird = 1.0 / 3.0, kSixth = 1.0 / 6.0;

struct TmaArgs {
  Grid g;
  Metric m;
  const double* rsg;
  const double2* in[5];  // for direct (out-of-tile) reads
  const double2* base;
  const double2* aux4;
  double2* out;
  double2* out4;
  double2* acc;
  int skip_last_i;
  int kchunk;
  int* err;
  int npf;      // number of prefetch maps in use (0..2)
  int base_in;  // the point-wise base is the stencil input itself (values already in the ring)
};

}  // namespace

// one solve of a batched launch (kept in device memory; tensor maps 64-byte aligned)
struct alignas(64) BatchItem {
  CUtensorMap tm4, tm1, tp0, tp1;
  TmaArgs a;
  int tiles_x, tiles_y, item0, n_items;
};

// One work item: a tile of (r, theta) columns through one chunk of phi planes.
// `tb` counts the planes this CTA has already pulled through its ring (ring
// slot and mbarrier parity continue across items in the persistent kernel).
// Returns the number of planes consumed, or -1 when a bounded wait ran out.
template <int KIND, int MK, int TJ>
__device__ __forceinline__ int stage_item(const CUtensorMap* tm4p, const CUtensorMap* tm1p, const CUtensorMap* tp0p,
                                          const CUtensorMap* tp1p, const TmaArgs& a, int bx, int by, int bz,
                                          double* ring, double* mt, uint64_t* bars, uint32_t tb) {
  using GT = Geom<TJ>;
  constexpr int FIELD_D = GT::FIELD_D, STAGE_D = GT::STAGE_D, STAGE_B = GT::STAGE_B, MT_N = GT::MT_N;
  constexpr bool PSI = (KIND != ST_P2_S1B && KIND != ST_P3_S2B);
  constexpr bool PI_ = (KIND != ST_P2_S1A && KIND != ST_P3_S2A);
  const Grid& g = a.g;
  const Metric& M = a.m;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TI + tx;
  const int ii0 = bx * TI, jj0 = by * TJ;
  const int ii = ii0 + tx, jj = jj0 + ty;
  const bool act = (ii < g.NI) && (jj < g.NJ);
  // ring slot protocol: full[s] (bars[s]) completes when a plane's boxes have
  // landed; empty[s] when all eight warps have read the plane for the last
  // time, after which thread 0 may load the next plane into the slot, so the
  // warps are not held at a block barrier per plane
  uint64_t* empty = bars + NST;
  const int lane = tid & 31;
  const int k0 = bz * a.kchunk;
  if (k0 >= g.NK) return 0;
  const int k1 = min(k0 + a.kchunk, g.NK);
  const int nplanes = (k1 - k0) + 2;  // previous, the chunk, next
  auto plane_of = [&](int t) -> int {
    if (t == 0) return (k0 == 0) ? g.Nz - 2 : k0 - 1;
    if (t <= k1 - k0) return k0 + t - 1;
    return (k1 - 1 == g.Nz) ? 2 : k1;
  };
  auto slot = [&](int t) -> int { return (int)((tb + (uint32_t)t) % NST); };
  auto parity = [&](int t) -> uint32_t { return ((tb + (uint32_t)t) / NST) & 1u; };
  auto release = [&](int t) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[slot(t)]);
  };
  auto issue = [&](int t) {
    const int s = slot(t);
    uint64_t* b = &bars[s];
    double* dst = ring + (size_t)s * STAGE_D;
    mbar_expect_tx(b, STAGE_B);
    const int z = plane_of(t);
    tma_load_4d(dst, tm4p, 2 * (ii0 - RH), jj0 - 1, z, 0, b);
    tma_load_4d(dst + 4 * FIELD_D, tm1p, 2 * (ii0 - RH), jj0 - 1, z, 0, b);
  };

  // the first planes are requested before the metric tile is loaded, so the
  // copies are in flight while the tile loads (the ring is free: every warp
  // finished the previous item before this one started)
  // the point-wise operands (u_p, accumulator, ...) of plane k are pulled into
  // L2 one plane ahead, so their loads in the combination hit L2 (two or more
  // planes ahead measured slower: 5-20 % on the stages with point-wise operands)
  auto prefetch = [&](int k) {
    if (k >= k1) return;
    if (a.npf > 0) tma_prefetch_4d(tp0p, 2 * ii0, jj0, k, 0);
    if (a.npf > 1) tma_prefetch_4d(tp1p, 2 * ii0, jj0, k, 0);
  };
  int nissued = 0;  // meaningful in thread 0 only
  if (tid == 0) {
    for (int t = 0; t < NST && t < nplanes; ++t) {
      issue(t);
      nissued = t + 1;
    }
    prefetch(k0);
  }

  // metric tile (phi-independent), zero outside the array
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
  }
  __syncthreads();
  // own-point metric
  const int q = act ? off2(g, ii, jj) : 0;
  double al = 0, be = 0, dxb = 0, sg = 1, rs = 1, am2 = 0, fa = 0, fgrp = 0, fgpp = 0;
  if (act) {
    al = ldm(M.alpha, q);
    be = ldm(M.beta, q);
    dxb = ldm(M.dxbeta, q);
    sg = ldm(M.sqrtg, q);
    rs = ldm(a.rsg, q);
    am2 = ldm(M.am2, q);
    if (MK == MK_KS) {
      fa = ldm(M.asg, q);
      fgrp = ldm(M.grp, q);
      fgpp = ldm(M.gpp, q);
    } else {
      fa = ldm(M.a_gpp, q);
    }
  }
  const long long pcol = act ? off3(g, ii, jj, 0) : 0;
  auto RF = [&](const double* st, int f, int dx, int dy) -> double2 {
    return *reinterpret_cast<const double2*>(st + (size_t)f * FIELD_D + (dy + 1) * RW + 2 * (dx + RH));
  };
  auto MTV = [&](int which, int dx, int dy) -> double { return mt[which * MT_N + (dy + 1) * MW + dx + RH]; };
  auto phiE = [&](const double* st) { return cadd(rmul(al, RF(st, 4, tx, ty)), rmul(be, RF(st, 1, tx, ty))); };
  auto phiF = [&](const double* st) {
    if (MK == MK_KS) return rmul(fa, cadd(rmul(fgrp, RF(st, 1, tx, ty)), rmul(fgpp, RF(st, 3, tx, ty))));
    return rmul(fa, RF(st, 3, tx, ty));
  };

  int timed_out = 0;
  double2 Epv = c2(0, 0), Fpv = c2(0, 0), Ecu = c2(0, 0), Fcu = c2(0, 0);
  if (!mbar_wait_bounded(&bars[slot(0)], parity(0))) timed_out = 1;
  if (act && !timed_out) {
    const double* st = ring + (size_t)slot(0) * STAGE_D;
    if (PSI) Epv = phiE(st);
    if (PI_) Fpv = phiF(st);
  }
  release(0);
  bool failed = __syncthreads_or(timed_out) != 0;
  const int last = k1 - k0 - 1;

  // FAST: every lane of the warp is two points inside the array in r and beta^r > 0
  // there, so every lane takes the centred derivative and the forward upwind
  // difference (the branches the general form would take); warp-uniform
  const bool fast = __all_sync(0xffffffffu, act && ii >= 2 && ii <= g.NI - 3 && be > 0.0);
  auto march = [&](auto fastc) {
  constexpr bool FAST = decltype(fastc)::value;
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
      prefetch(k + 1);
    }
    {
      const int tc = i + 1, tn = i + 2;
      if (!timed_out) {
        const bool okc = mbar_wait_bounded(&bars[slot(tc)], parity(tc));
        const bool okn = okc && mbar_wait_bounded(&bars[slot(tn)], parity(tn));
        if (!okn) timed_out = 1;
      }
      if (act && !timed_out) {
        const double* cu = ring + (size_t)slot(tc) * STAGE_D;
        const double* nx = ring + (size_t)slot(tn) * STAGE_D;
        if (i == 0) {
          if (PSI) Ecu = phiE(cu);
          if (PI_) Fcu = phiF(cu);
        }
        double2 Enx = c2(0, 0), Fnx = c2(0, 0);
        if (PSI) Enx = phiE(nx);
        if (PI_) Fnx = phiF(nx);
        double2 fcu[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) fcu[v] = RF(cu, v, tx, ty);
        const long long p = pcol + (long long)k * g.plane;
        const int n = g.NI - 1;
        double2 r[5];
        if (PSI) {
          r[0] = cadd(rmul(al, fcu[4]), rmul(be, fcu[1]));
          auto aPi = [&](int dx) { return rmul(MTV(MT_AL, tx + dx, ty), RF(cu, 4, tx + dx, ty)); };
          auto ps1 = [&](int dx) { return RF(cu, 1, tx + dx, ty); };
          double2 d;
          if (FAST) d = ctr(aPi(-1), aPi(1));
          else if (ii == 0) d = fwd3(aPi(0), aPi(1), aPi(2));
          else if (ii == n) d = bwd3(aPi(0), aPi(-1), aPi(-2));
          else d = ctr(aPi(-1), aPi(1));
          d = rmul(g.rdx, d);
          double2 av;
          if (FAST) av = fwd3(fcu[1], ps1(1), ps1(2));
          else if (ii <= 1) av = fwd3(fcu[1], ps1(1), ps1(2));
          else if (ii == n - 1) av = csub(ps1(1), ps1(-1));
          else if (ii == n) av = bwd3(fcu[1], ps1(-1), ps1(-2));
          else if (be > 0.0) av = fwd3(fcu[1], ps1(1), ps1(2));
          else if (be < 0.0) av = bwd3(fcu[1], ps1(-1), ps1(-2));
          else av = csub(ps1(1), ps1(-1));
          av = rmul(g.rdx, av);
          r[1] = cadd(cadd(d, rmul(be, av)), rmul(dxb, fcu[1]));
          auto E = [&](int dy) {
            return cadd(rmul(MTV(MT_AL, tx, ty + dy), RF(cu, 4, tx, ty + dy)),
                        rmul(MTV(MT_BE, tx, ty + dy), RF(cu, 1, tx, ty + dy)));
          };
          auto Eg = [&](int j2, int k2) {
            const int q2 = off2(g, ii, j2);
            const long long p2 = off3(g, ii, j2, k2);
            return cadd(rmul(ldm(M.alpha, q2), ldf(a.in[4], p2)), rmul(ldm(M.beta, q2), ldf(a.in[1], p2)));
          };
          double2 t;
          if (jj == 0) t = cadd(cneg(E(1)), Eg(2, ktarget(g, k)));
          else if (jj == g.NJ - 1) t = bwd3(E(0), E(-1), (ty >= 1) ? E(-2) : Eg(jj - 2, k));
          else t = ctr(E(-1), E(1));
          r[2] = rmul(g.rdy, t);
          double2 z;
          if (k == 0) z = cadd(cneg(Epv), Enx);
          else if (k == g.Nz) z = cadd(cneg(Enx), Epv);
          else z = ctr(Epv, Enx);
          r[3] = rmul(g.rdz, z);
        }
        if (PI_) {
          auto G1 = [&](int dx) {
            if (MK == MK_KS)
              return rmul(MTV(MT_A, tx + dx, ty), cadd(rmul(MTV(MT_GRR, tx + dx, ty), RF(cu, 1, tx + dx, ty)),
                                                       rmul(MTV(MT_GRP, tx + dx, ty), RF(cu, 3, tx + dx, ty))));
            return rmul(MTV(MT_A, tx + dx, ty), RF(cu, 1, tx + dx, ty));
          };
          double2 d;
          if (FAST) d = ctr(G1(-1), G1(1));
          else if (ii == 0) d = fwd3(G1(0), G1(1), G1(2));
          else if (ii == n) d = bwd3(G1(0), G1(-1), G1(-2));
          else d = ctr(G1(-1), G1(1));
          const double2 r1 = cdivm(rmul(g.rdx, d), sg, rs);
          auto H = [&](int dy) { return rmul(MTV(MT_HT, tx, ty + dy), RF(cu, 2, tx, ty + dy)); };
          auto Hg = [&](int j2, int k2) {
            return rmul(ldm(M.asg_gtt, off2(g, ii, j2)), ldf(a.in[2], off3(g, ii, j2, k2)));
          };
          double2 t;
          if (jj == 0) t = cadd(cneg(H(1)), Hg(2, ktarget(g, k)));
          else if (jj == g.NJ - 1) t = bwd3(H(0), H(-1), (ty >= 1) ? H(-2) : Hg(jj - 2, k));
          else t = ctr(H(-1), H(1));
          const double2 r2 = cdivm(rmul(g.rdy, t), sg, rs);
          double2 z;
          if (k == 0) z = cadd(cneg(Fpv), Fnx);
          else if (k == g.Nz) z = cadd(cneg(Fnx), Fpv);
          else z = ctr(Fpv, Fnx);
          z = rmul(g.rdz, z);
          const double2 r3 = (MK == MK_KS) ? cdivm(z, sg, rs) : z;
          const double2 r4 = rmul(dxb, fcu[4]);
          auto Q = [&](int dx) { return rmul(MTV(MT_SG, tx + dx, ty), RF(cu, 4, tx + dx, ty)); };
          double2 av;
          if (FAST) av = fwd3(Q(0), Q(1), Q(2));
          else if (ii <= 1) av = fwd3(Q(0), Q(1), Q(2));
          else if (ii == n - 1) av = csub(Q(1), Q(-1));
          else if (ii == n) av = bwd3(Q(0), Q(-1), Q(-2));
          else if (be > 0.0) av = fwd3(Q(0), Q(1), Q(2));
          else if (be < 0.0) av = bwd3(Q(0), Q(-1), Q(-2));
          else av = csub(Q(1), Q(-1));
          av = rmul(g.rdx, av);
          const double2 r5 = cdivm(rmul(be, av), sg, rs);
          const double2 r6 = rmul(am2, fcu[0]);
          r[4] = csub(cadd(cadd(cadd(cadd(r1, r2), r3), r4), r5), r6);
        }
        const double dt = g.dt;
        auto B = [&](int v) { return a.base_in ? fcu[v] : ldf(a.base + v * g.fs, p); };
        if (KIND == ST_P2_S1A) {
#pragma unroll
          for (int v = 0; v < 4; ++v) a.out[v * g.fs + p] = cadd(B(v), rmul(dt, r[v]));
        } else if (KIND == ST_P3_S2A) {
#pragma unroll
          for (int v = 0; v < 4; ++v)
            a.out[v * g.fs + p] =
                cadd(rmul(0.75, ldf(a.base + v * g.fs, p)), rmul(0.25, cadd(fcu[v], rmul(dt, r[v]))));
        } else if (KIND == ST_P2_S1B) {
          a.out4[p] = cadd(ldf(a.base + 4 * g.fs, p), rmul(dt, r[4]));
        } else if (KIND == ST_P3_S2B) {
          a.out4[p] = cadd(rmul(0.75, ldf(a.base + 4 * g.fs, p)), rmul(0.25, cadd(ldf(a.aux4, p), rmul(dt, r[4]))));
        } else if (!(a.skip_last_i && ii == n)) {
#pragma unroll
          for (int v = 0; v < 5; ++v) {
            const long long o = v * g.fs + p;
            const double2 b = B(v);
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
            } else {
              const double2 kk = rmul(dt, r[v]);
              res = cadd(b, cdivm(cadd(a.acc[o], kk), 6.0, kSixth));
            }
            a.out[o] = res;
          }
        }
        Epv = Ecu;
        Fpv = Fcu;
        Ecu = Enx;
        Fcu = Fnx;
      }
    }
    release(i + 1);
    if (i == last) release(i + 2);
  }
  };
  if (fast) march(TBool<true>());
  else march(TBool<false>());
  failed = __syncthreads_or(timed_out) != 0;
  if (failed) {
    if (tid == 0) {
      atomicExch(a.err, 1);
      // let the last copy issued into each ring slot land before the CTA's
      // shared memory is released (bounded as well)
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

// the TMA destinations must start on 128-byte boundaries of the shared window
__device__ __forceinline__ unsigned char* align128(unsigned char* p) {
  const uint32_t a = saddr(p);
  return p + ((128u - (a & 127u)) & 127u);
}

template <int TJ>
__device__ __forceinline__ void init_ring_barriers(uint64_t* bars) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bars[s], 1);
    for (int s = 0; s < NST; ++s) mbar_init(&bars[NST + s], TJ);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

template <int KIND, int MK, int TJ>
__global__ void __launch_bounds__(TI * TJ, Geom<TJ>::MIN_BLOCKS)
    tma_stage_kernel(const __grid_constant__ CUtensorMap tm4, const __grid_constant__ CUtensorMap tm1,
                     const __grid_constant__ CUtensorMap tp0, const __grid_constant__ CUtensorMap tp1, TmaArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* ring = reinterpret_cast<double*>(align128(smem_raw));
  double* mt = ring + (size_t)NST * Geom<TJ>::STAGE_D;
  uint64_t* bars = reinterpret_cast<uint64_t*>(mt + (size_t)MT_COUNT * Geom<TJ>::MT_N);
  if ((int)blockIdx.z * a.kchunk >= a.g.NK) return;
  init_ring_barriers<TJ>(bars);
  (void)stage_item<KIND, MK, TJ>(&tm4, &tm1, &tp0, &tp1, a, blockIdx.x, blockIdx.y, blockIdx.z, ring, mt, bars, 0u);
}

// ---- persistent kernel over many solves -------------------------------------
// Every solve of a batch contributes tiles_x * tiles_y * chunks work items; a
// CTA walks the ragged list item = blockIdx.x, blockIdx.x + gridDim.x, ...
// and runs each with the solve's own grid, metric, buffers and tensor maps.
template <int KIND, int MK, int TJ>
__global__ void __launch_bounds__(TI * TJ, Geom<TJ>::MIN_BLOCKS)
    tma_batch_kernel(const BatchItem* __restrict__ solves, int n_solves, int n_items) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* ring = reinterpret_cast<double*>(align128(smem_raw));
  double* mt = ring + (size_t)NST * Geom<TJ>::STAGE_D;
  uint64_t* bars = reinterpret_cast<uint64_t*>(mt + (size_t)MT_COUNT * Geom<TJ>::MT_N);
  __shared__ TmaArgs sa;
  __shared__ int s_bx, s_by, s_bz, s_solve;
  init_ring_barriers<TJ>(bars);
  uint32_t tb = 0;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      int lo = 0, hi = n_solves - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (solves[mid].item0 <= item) lo = mid;
        else hi = mid - 1;
      }
      const BatchItem& B = solves[lo];
      const int local = item - B.item0;
      s_solve = lo;
      s_bx = local % B.tiles_x;
      s_by = (local / B.tiles_x) % B.tiles_y;
      s_bz = local / (B.tiles_x * B.tiles_y);
      sa = B.a;
    }
    __syncthreads();
    const BatchItem& B = solves[s_solve];
    const int used = stage_item<KIND, MK, TJ>(&B.tm4, &B.tm1, &B.tp0, &B.tp1, sa, s_bx, s_by, s_bz, ring, mt, bars, tb);
    if (used < 0) break;
    tb += (uint32_t)used;
    __syncthreads();  // sa and the item indices are rewritten for the next item
  }
}

// ---------------------------------------------------------------------------
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
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

// 4-D view (x = doubles along r incl. row padding, theta rows, phi planes, variables);
// halo = true: the stencil box (tile + r halo 2 + theta halo 1), false: the tile;
// tj: theta rows of the tile
bool encode(CUtensorMap* tm, const Grid& g, const double2* base, int nvars, bool halo = true, int tj = 8) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)(2 * g.PI), (cuuint64_t)g.NJ, (cuuint64_t)g.NK, (cuuint64_t)nvars};
  cuuint64_t strides[3] = {(cuuint64_t)g.PI * 16, (cuuint64_t)g.plane * 16, (cuuint64_t)g.fs * 16};
  cuuint32_t box[4] = {halo ? (cuuint32_t)RW : (cuuint32_t)(2 * TI), (cuuint32_t)(halo ? tj + 2 : tj), 1,
                       (cuuint32_t)nvars};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int tma_chunk(const Grid& g) {
  const int nchunks = (g.NK + 31) / 32;
  return (g.NK + nchunks - 1) / nchunks;
}

struct Maps {
  CUtensorMap tm4, tm1, tp0, tp1;
};

template <int KIND, int MK, int TJ>
int launch_one(const Maps& m, const TmaArgs& a, cudaStream_t st) {
  constexpr size_t SMEM = Geom<TJ>::SMEM_BYTES;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(tma_stage_kernel<KIND, MK, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)SMEM) != cudaSuccess)
      return -1;
    attr_set = true;
  }
  const Grid& g = a.g;
  dim3 block(TI, TJ, 1);
  dim3 grid((g.NI + TI - 1) / TI, (g.NJ + TJ - 1) / TJ, (g.NK + a.kchunk - 1) / a.kchunk);
  tma_stage_kernel<KIND, MK, TJ><<<grid, block, SMEM, st>>>(m.tm4, m.tm1, m.tp0, m.tp1, a);
  return 0;
}

// the 4-row tiles are built for the RK4 stages (the batched forms' stepper) only
template <int KIND>
constexpr bool has_tj4() {
  return KIND == ST_RK4_1 || KIND == ST_RK4_2 || KIND == ST_RK4_3 || KIND == ST_RK4_4;
}
template <int KIND>
int launch_kind(const Maps& m, const TmaArgs& a, int mk, int tj, cudaStream_t st) {
  if constexpr (has_tj4<KIND>()) {
    if (tj == 4) return mk == MK_KS ? launch_one<KIND, MK_KS, 4>(m, a, st) : launch_one<KIND, MK_SCHW, 4>(m, a, st);
  }
  return mk == MK_KS ? launch_one<KIND, MK_KS, 8>(m, a, st) : launch_one<KIND, MK_SCHW, 8>(m, a, st);
}

}  // namespace

size_t batch_item_bytes() { return sizeof(BatchItem); }

// fill one solve's item record for a batched launch of stage `kind`
int build_batch_item(void* dst, int kind, const StageLaunch& L, const double* rsg, int* err, int kchunk, int item0,
                     int tj) {
  // the requested chunk length is an upper bound: the solve's planes are split
  // into equal chunks, so no chunk is a short remainder that pays a whole
  // pipeline prologue for a few planes
  {
    const int nch = (L.g.NK + kchunk - 1) / kchunk;
    kchunk = (L.g.NK + nch - 1) / nch;
  }
  BatchItem* B = reinterpret_cast<BatchItem*>(dst);
  memset(B, 0, sizeof(BatchItem));
  if (!encode(&B->tm4, L.g, L.in[0], 4, true, tj) || !encode(&B->tm1, L.g, L.in[4], 1, true, tj)) return -1;
  const long long fsl = L.g.fs;
  int base_in = 1;
  for (int v = 0; v < 5; ++v) base_in = base_in && (L.in[v] == L.base + v * fsl);
  base_in = base_in && (kind == ST_P2_S1A || kind == ST_RK3_1 || kind == ST_RK4_1);
  int npf = 0;
  auto add = [&](const double2* p, int nv) {
    CUtensorMap* t = npf == 0 ? &B->tp0 : &B->tp1;
    if (npf < 2 && p && encode(t, L.g, p, nv, false, tj)) ++npf;
  };
  if (!base_in) {
    switch (kind) {
      case ST_P2_S1A: case ST_P3_S2A: add(L.base, 4); break;
      case ST_P2_S1B: add(L.base + 4 * fsl, 1); break;
      case ST_P3_S2B: add(L.base + 4 * fsl, 1); add(L.aux4, 1); break;
      case ST_RK4_2: case ST_RK4_3: case ST_RK4_4: add(L.base, 5); add(L.acc, 5); break;
      default: add(L.base, 5); break;
    }
  }
  if (npf < 2) B->tp1 = B->tm1;
  if (npf < 1) B->tp0 = B->tm1;
  TmaArgs& a = B->a;
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
  a.kchunk = kchunk;
  a.err = err;
  a.npf = npf;
  a.base_in = base_in;
  B->tiles_x = (L.g.NI + TI - 1) / TI;
  B->tiles_y = (L.g.NJ + tj - 1) / tj;
  const int chunks = (L.g.NK + kchunk - 1) / kchunk;
  B->item0 = item0;
  B->n_items = B->tiles_x * B->tiles_y * chunks;
  return B->n_items;
}

namespace {
template <int KIND, int MK, int TJ>
int batch_one(const void* items, int n_solves, int n_items, int blocks, cudaStream_t st) {
  constexpr size_t SMEM = Geom<TJ>::SMEM_BYTES;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(tma_batch_kernel<KIND, MK, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)SMEM) != cudaSuccess)
      return -1;
    attr_set = true;
  }
  if (n_items <= 0) return 0;
  tma_batch_kernel<KIND, MK, TJ><<<blocks, dim3(TI, TJ, 1), SMEM, st>>>(reinterpret_cast<const BatchItem*>(items),
                                                                       n_solves, n_items);
  return 0;
}
template <int KIND>
int batch_kind(const void* items, int n_solves, int n_items, int blocks, int mk, int tj, cudaStream_t st) {
  if constexpr (has_tj4<KIND>()) {
    if (tj == 4)
      return mk == MK_KS ? batch_one<KIND, MK_KS, 4>(items, n_solves, n_items, blocks, st)
                         : batch_one<KIND, MK_SCHW, 4>(items, n_solves, n_items, blocks, st);
  }
  if (tj != 8) return -1;
  return mk == MK_KS ? batch_one<KIND, MK_KS, 8>(items, n_solves, n_items, blocks, st)
                     : batch_one<KIND, MK_SCHW, 8>(items, n_solves, n_items, blocks, st);
}
}  // namespace

int launch_batch_tma(int kind, int mk, const void* d_items, int n_solves, int n_items, int blocks, int tj,
                     cudaStream_t st) {
  switch (kind) {
    case ST_P2_S1A: return batch_kind<ST_P2_S1A>(d_items, n_solves, n_items, blocks, mk, tj, st);
    case ST_P2_S1B: return batch_kind<ST_P2_S1B>(d_items, n_solves, n_items, blocks, mk, tj, st);
    case ST_P2_S2: return batch_kind<ST_P2_S2>(d_items, n_solves, n_items, blocks, mk, tj, st);
    case ST_RK4_1: return batch_kind<ST_RK4_1>(d_items, n_solves, n_items, blocks, mk, tj, st);
    case ST_RK4_2: return batch_kind<ST_RK4_2>(d_items, n_solves, n_items, blocks, mk, tj, st);
    case ST_RK4_3: return batch_kind<ST_RK4_3>(d_items, n_solves, n_items, blocks, mk, tj, st);
    case ST_RK4_4: return batch_kind<ST_RK4_4>(d_items, n_solves, n_items, blocks, mk, tj, st);
    default: return -1;
  }
}

// The failure path of a bounded wait, on its own: one warp waits, at most
// `polls` polls, on the first phase of an mbarrier that nothing arrives on and
// no copy completes, then sets the error flag and returns -- what a stage
// kernel does when its copies never land.  Nothing is left in flight.
__global__ void wait_check_kernel(int* err, long long polls) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  const bool ok = mbar_wait_bounded_n(&bar, 0u, polls);
  if (__any_sync(0xffffffffu, !ok) && threadIdx.x == 0) atomicExch(err, 1);
}

int launch_wait_check(int* err, long long polls, cudaStream_t st) {
  wait_check_kernel<<<1, 32, 0, st>>>(err, polls);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

bool tma_available(const Grid& g, const double2* some_state) {
  CUtensorMap tm;
  return encode(&tm, g, some_state, 4) && encode(&tm, g, some_state, 1);
}

int launch_stage_tma(int kind, const StageLaunch& L, const double* rsg, int* err, cudaStream_t st, int tj) {
  const bool rk4 = kind == ST_RK4_1 || kind == ST_RK4_2 || kind == ST_RK4_3 || kind == ST_RK4_4;
  if (!rk4 || tj != 4) tj = 8;  // the 4-row tiles exist for the RK4 stages
  Maps mp;
  if (!encode(&mp.tm4, L.g, L.in[0], 4, true, tj) || !encode(&mp.tm1, L.g, L.in[4], 1, true, tj)) return -1;
  // point-wise operands read in the combination, prefetched into L2
  int npf = 0;
  const long long fs = L.g.fs;
  auto add = [&](const double2* p, int nv) {
    CUtensorMap* t = npf == 0 ? &mp.tp0 : &mp.tp1;
    if (npf < 2 && p && encode(t, L.g, p, nv, false, tj)) ++npf;
  };
  const long long fsl = L.g.fs;
  int base_in = 1;
  for (int v = 0; v < 5; ++v) base_in = base_in && (L.in[v] == L.base + v * fsl);
  if (base_in && (kind == ST_P2_S1A || kind == ST_RK3_1 || kind == ST_RK4_1)) {
    // nothing point-wise to prefetch except the accumulator (written, not read, in RK4 stage 1)
  } else switch (kind) {
    case ST_P2_S1A: case ST_P3_S2A: add(L.base, 4); break;
    case ST_P2_S1B: add(L.base + 4 * fs, 1); break;
    case ST_P3_S2B: add(L.base + 4 * fs, 1); add(L.aux4, 1); break;
    case ST_RK4_2: case ST_RK4_3: case ST_RK4_4: add(L.base, 5); add(L.acc, 5); break;
    default: add(L.base, 5); break;
  }
  TmaArgs a;
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
  a.kchunk = tma_chunk(L.g);
  a.err = err;
  a.npf = npf;
  a.base_in = base_in && (kind == ST_P2_S1A || kind == ST_RK3_1 || kind == ST_RK4_1);
  if (npf < 2) mp.tp1 = mp.tm1;  // unused parameter slot, never issued
  if (npf < 1) mp.tp0 = mp.tm1;
  const int mk = L.metric_kind;
  switch (kind) {
    case ST_P2_S1A: return launch_kind<ST_P2_S1A>(mp, a, mk, tj, st);
    case ST_P2_S1B: return launch_kind<ST_P2_S1B>(mp, a, mk, tj, st);
    case ST_P2_S2: return launch_kind<ST_P2_S2>(mp, a, mk, tj, st);
    case ST_P3_S2A: return launch_kind<ST_P3_S2A>(mp, a, mk, tj, st);
    case ST_P3_S2B: return launch_kind<ST_P3_S2B>(mp, a, mk, tj, st);
    case ST_P3_S3: return launch_kind<ST_P3_S3>(mp, a, mk, tj, st);
    case ST_RK3_1: return launch_kind<ST_RK3_1>(mp, a, mk, tj, st);
    case ST_RK3_2: return launch_kind<ST_RK3_2>(mp, a, mk, tj, st);
    case ST_RK3_3: return launch_kind<ST_RK3_3>(mp, a, mk, tj, st);
    case ST_RK4_1: return launch_kind<ST_RK4_1>(mp, a, mk, tj, st);
    case ST_RK4_2: return launch_kind<ST_RK4_2>(mp, a, mk, tj, st);
    case ST_RK4_3: return launch_kind<ST_RK4_3>(mp, a, mk, tj, st);
    case ST_RK4_4: return launch_kind<ST_RK4_4>(mp, a, mk, tj, st);
    default: return -1;
  }
}

}  // namespace kg
