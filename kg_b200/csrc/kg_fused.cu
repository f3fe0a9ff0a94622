// kg_fused.cu -- PIRK stage 1 as one TMA-pipelined kernel.
//
// The reference's PIRK stage 1 (MoL/lines_method_lib.f90:278-289, pirk2; the
// same statements open pirk3 at :341-352) is
//     u_stage(1:4) = u(1:4) + dt * rhs_{phi,psi1,psi2,psi3}(u)
//     u_stage(5)   = u(5)   + dt * rhs_pi(u_stage)
// where rhs_pi reads the fresh u_stage(1:4) with their r, theta and phi
// neighbours, and the u_stage(5) slot still holding the previous step's Pi.
// Done as two launches, the psi part writes u_stage(1:4) (144 B/point) and
// the Pi part reads it back (112 B/point).  This kernel does both in one pass
// over u (176 B/point: u, the stale Pi slot, u_stage(1:5)).
//
// Work layout.  A CTA of 8 warps owns 30 r columns x 8 theta rows and marches
// through a chunk of phi planes.  Lane L of warp w stands at column i0-1+L and
// row j0+w: lanes 1..30 are the tile's own columns, lanes 0 and 31 the columns
// on either side, whose psi stage the r-flux of the Pi rhs needs.  Every lane
// forms the psi1/psi3 stage and the two Pi fluxes that depend on them at its
// column, so the r neighbours of the Pi rhs come from warp shuffles and no lane
// idles while another forms a halo value.  The last tile in r (and in theta) is
// moved back to end at the array's last column (row), so the one-sided closures
// at the array ends always find their neighbours inside the tile; the overlap
// with the previous tile is written twice with the same bits.
//
// Per phi plane P[t] of the marched sequence (the chunk with one plane on
// either side):
//   * E = alpha Pi + beta psi1 (the phi rhs and the psi fluxes) of plane P[t+1]
//     is formed on the lane's own column and rolls in registers, so the psi3
//     stage of P[t] takes its phi derivative from registers;
//   * the psi1, psi3 stages and the Pi phi-flux F of P[t] are formed on every
//     plane (the Pi rhs of P[t-1] needs F at P[t]); on the chunk's own planes
//     also the phi and psi2 stages, the output u_stage(1:4), the r-flux G of the
//     Pi rhs (kept in registers for the next step) and the theta flux H, which
//     goes to shared memory for the rows on either side (warps 0 and 7 also form
//     it on the rows just outside the tile);
//   * the Pi stage of P[t-1] follows from G (shuffles), H (shared memory), F at
//     P[t-2] and P[t] (registers) and the stale Pi slot, and is written to the
//     new Pi slot.
// The planes arrive by TMA in a 3-deep shared-memory ring (psi1 and Pi with a
// -3/+2 column and +-2 row halo, psi2 with a +-1 row halo, psi3 on the lanes'
// columns, the stale Pi of the previous plane with a +-2 column halo), one
// "full" mbarrier per slot with bounded waits.  One block barrier per plane
// orders the H exchange and frees the ring slot of the plane just finished for
// the next copy.
//
// Every value is formed with the same operations in the same order as the
// two-launch form (kg_tma.cu, kinds ST_P2_S1A and ST_P2_S1B), so results are
// the same bits.  Values outside the boxes (the pole partner plane, and E on the
// phi planes just outside the sequence) are read from global memory.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstring>
#include "kg_device.cuh"
#include "kg_internal.h"
#include "kg_tma_ops.cuh"

namespace kg {
using namespace tmaops;
namespace {

constexpr int FL = 32;            // lanes: the tile's r columns plus one on either side
constexpr int FO = FL - 2;        // own r columns per tile
constexpr int FJ = 8;             // own theta rows per tile (one warp each)
constexpr int NSTF = 3;           // ring depth
constexpr int NTH = FL * FJ;
// boxes, relative to the tile origin (i0, j0), in complex columns and rows
constexpr int A_C0 = -3, A_NC = 36, A_R0 = -2, A_NR = FJ + 4;  // psi1, Pi
constexpr int B_C0 = -1, B_NC = 32, B_R0 = -1, B_NR = FJ + 2;  // psi2
constexpr int C_C0 = -1, C_NC = 32, C_NR = FJ;                 // psi3
constexpr int D_C0 = -2, D_NC = 34, D_NR = FJ;                 // stale Pi (previous plane)
// metric tables in shared memory: columns i0-2 .. i0+31
constexpr int M_C0 = -2, M_NC = 34;
constexpr int MAB_R0 = -2, MAB_NR = FJ + 4;  // alpha, beta
constexpr int MHT_R0 = -1, MHT_NR = FJ + 2;  // (alpha sqrtg) gamma^thth
constexpr int MSG_NR = FJ;                   // sqrtg
constexpr int H_NR = FJ + 2;                 // theta flux rows j0-1 .. j0+FJ

__host__ __device__ constexpr int rnd128(int b) { return (b + 127) / 128 * 128; }

constexpr int A_BYTES = A_NC * A_NR * 16;
constexpr int B_BYTES = B_NC * B_NR * 16;
constexpr int C_BYTES = C_NC * C_NR * 16;
constexpr int D_BYTES = D_NC * D_NR * 16;
constexpr int OFF_A1 = 0;
constexpr int OFF_A4 = rnd128(A_BYTES);
constexpr int OFF_B = OFF_A4 + rnd128(A_BYTES);
constexpr int OFF_C = OFF_B + rnd128(B_BYTES);
constexpr int OFF_D = OFF_C + rnd128(C_BYTES);
constexpr int SLOT = OFF_D + rnd128(D_BYTES);
constexpr int H_BYTES = H_NR * FL * 16;
// (two doubles of padding after the sqrtg table: the Pi stage's discarded lanes
// read one value past it)
constexpr int MT_DOUBLES = 2 * M_NC * MAB_NR + M_NC * MHT_NR + M_NC * MSG_NR + 2;
constexpr size_t SMEM = (size_t)NSTF * SLOT + 2 * (size_t)H_BYTES + (size_t)MT_DOUBLES * 8 + NSTF * 8 + 128;
static_assert(SMEM <= 113 * 1024, "two CTAs per SM");

struct FusedArgs {
  Grid g;
  Metric m;
  const double* rsg;
  const double2* U;     // u, 5 variables
  const double2* Sold;  // u_stage(5) of the previous step
  double2* S;           // u_stage(1:4) (variables 0..3 of this base)
  double2* Snew;        // u_stage(5) of this step
  int kchunk;
  int* err;
};

__device__ __forceinline__ double fddiv(double a, double b, double rb) {
  const double q = a * rb;
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, rb, q);
}
__device__ __forceinline__ double2 fcdivm(double2 a, double b, double rb) {
  return c2(fddiv(a.x, b, rb), fddiv(a.y, b, rb));
}
__device__ __forceinline__ double2 shfl2_up(double2 v, int d) {
  return c2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ double2 shfl2_down(double2 v, int d) {
  return c2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}
template <bool B>
struct BoolC {
  static constexpr bool value = B;
};
__device__ __forceinline__ unsigned char* falign128(unsigned char* p) {
  const uint32_t a = saddr(p);
  return p + ((128u - (a & 127u)) & 127u);
}
// tile origins: the last tile ends at the array's last column / row
__host__ __device__ __forceinline__ int tile_i0(int bx, int NI) {
  const int i0 = bx * FO;
  return (NI > FO && i0 > NI - FO) ? NI - FO : i0;
}
__host__ __device__ __forceinline__ int tile_j0(int by, int NJ) {
  const int j0 = by * FJ;
  return (j0 > NJ - FJ) ? NJ - FJ : j0;
}

}  // namespace

template <int MK>
__global__ void __launch_bounds__(NTH, 2)
    pirk_s1_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                         const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD,
                         FusedArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* ring = falign128(smem_raw);
  double2* hbuf = reinterpret_cast<double2*>(ring + (size_t)NSTF * SLOT);  // 2 x H_NR x FL
  double* mAL = reinterpret_cast<double*>(ring + (size_t)NSTF * SLOT + 2 * (size_t)H_BYTES);
  double* mBE = mAL + M_NC * MAB_NR;
  double* mHT = mBE + M_NC * MAB_NR;
  double* mSG = mHT + M_NC * MHT_NR;
  uint64_t* bars = reinterpret_cast<uint64_t*>(mSG + M_NC * MSG_NR + 2);
  const Grid& g = a.g;
  const Metric& M = a.m;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * FL + tx;
  const int i0 = tile_i0(blockIdx.x, g.NI), j0 = tile_j0(blockIdx.y, g.NJ);
  const int c = i0 - 1 + tx, jj = j0 + ty;  // this lane's column and row
  const int n = g.NI - 1;
  const bool vcol = c >= 0 && c <= n;
  const bool own = vcol && tx >= 1 && tx <= FO;
  const int k0 = blockIdx.z * a.kchunk;
  if (k0 >= g.NK) return;
  const int k1 = min(k0 + a.kchunk, g.NK);
  const int NP = (k1 - k0) + 2;
  const long long fs = g.fs;
  const double2* __restrict__ U = a.U;

  if (tid == 0) {
    for (int s = 0; s < NSTF; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // plane sequence: P[0] = prev(k0), P[1..NP-2] = k0..k1-1, P[NP-1] = next(k1-1)
  auto plane_of = [&](int t) -> int {
    if (t == 0) return (k0 == 0) ? g.Nz - 2 : k0 - 1;
    if (t <= k1 - k0) return k0 + t - 1;
    return (k1 - 1 == g.Nz) ? 2 : k1;
  };
  auto slot = [&](int t) -> int { return t % NSTF; };
  auto parity = [&](int t) -> uint32_t { return (uint32_t)((t / NSTF) & 1); };
  auto issue = [&](int t) {
    unsigned char* dst = ring + (size_t)slot(t) * SLOT;
    uint64_t* b = &bars[slot(t)];
    mbar_expect_tx(b, (uint32_t)(2 * A_BYTES + B_BYTES + C_BYTES + (t >= 2 ? D_BYTES : 0)));
    const int z = plane_of(t);
    tma_load_4d(dst + OFF_A1, &tmA, 2 * (i0 + A_C0), j0 + A_R0, z, 1, b);
    tma_load_4d(dst + OFF_A4, &tmA, 2 * (i0 + A_C0), j0 + A_R0, z, 4, b);
    tma_load_4d(dst + OFF_B, &tmB, 2 * (i0 + B_C0), j0 + B_R0, z, 2, b);
    tma_load_4d(dst + OFF_C, &tmC, 2 * (i0 + C_C0), j0, z, 3, b);
    // the stale Pi of the previous plane rides with this one: it is read in
    // the step that forms the Pi stage of plane P[t-1]
    if (t >= 2) tma_load_4d(dst + OFF_D, &tmD, 2 * (i0 + D_C0), j0, plane_of(t - 1), 0, b);
  };
  int nissued = 0;
  if (tid == 0) {
    for (int t = 0; t < NSTF && t < NP; ++t) {
      issue(t);
      nissued = t + 1;
    }
  }

  // metric tables (phi-independent), zero outside the array
  for (int q = tid; q < M_NC * MAB_NR; q += NTH) {
    const int gi = i0 + M_C0 + q % M_NC, gj = j0 + MAB_R0 + q / M_NC;
    const bool in = gi >= 0 && gi <= n && gj >= 0 && gj < g.NJ;
    const int o = in ? off2(g, gi, gj) : 0;
    mAL[q] = in ? ldm(M.alpha, o) : 0.0;
    mBE[q] = in ? ldm(M.beta, o) : 0.0;
  }
  for (int q = tid; q < M_NC * MHT_NR; q += NTH) {
    const int gi = i0 + M_C0 + q % M_NC, gj = j0 + MHT_R0 + q / M_NC;
    const bool in = gi >= 0 && gi <= n && gj >= 0 && gj < g.NJ;
    mHT[q] = in ? ldm(M.asg_gtt, off2(g, gi, gj)) : 0.0;
  }
  for (int q = tid; q < M_NC * MSG_NR; q += NTH) {
    const int gi = i0 + M_C0 + q % M_NC, gj = j0 + q / M_NC;
    const bool in = gi >= 0 && gi <= n && gj >= 0 && gj < g.NJ;
    mSG[q] = in ? ldm(M.sqrtg, off2(g, gi, gj)) : 0.0;
  }
  // own-column metric in registers
  double dxb = 0, fA = 0, fgrr = 0, fgrp = 0, fgpp = 0, rs = 1, am2 = 0;
  if (vcol) {
    const int q = off2(g, c, jj);
    dxb = ldm(M.dxbeta, q);
    fA = ldm(MK == MK_KS ? M.asg : M.asg_grr, q);
    fgrr = ldm(M.grr, q);
    fgrp = ldm(M.grp, q);
    fgpp = ldm(MK == MK_KS ? M.gpp : M.a_gpp, q);
    rs = ldm(a.rsg, q);
    am2 = ldm(M.am2, q);
  }
  const long long pcol = vcol ? off3(g, c, jj, 0) : 0;

  // ---- accessors (dc, dr: offsets from this lane's column and row) ---------
  auto RA = [&](const unsigned char* st, int off, int dc, int dr) -> double2 {
    return *reinterpret_cast<const double2*>(st + off + ((ty - A_R0 + dr) * A_NC + (tx - 1 - A_C0 + dc)) * 16);
  };
  auto MAB = [&](const double* t, int dc, int dr) { return t[(ty - MAB_R0 + dr) * M_NC + (tx - 1 - M_C0 + dc)]; };
  // E = alpha Pi + beta psi1 at this lane's column, row jj + dr, from the ring
  auto Ebox = [&](const unsigned char* st, int dr) {
    return cadd(rmul(MAB(mAL, 0, dr), RA(st, OFF_A4, 0, dr)), rmul(MAB(mBE, 0, dr), RA(st, OFF_A1, 0, dr)));
  };
  // the same from global memory, at row r of plane p
  auto Eglob = [&](int r, int p) {
    const int q = off2(g, c, r);
    const long long o = off3(g, c, r, p);
    return cadd(rmul(ldm(M.alpha, q), ldf(U + 4 * fs, o)), rmul(ldm(M.beta, q), ldf(U + fs, o)));
  };
  // phi-direction difference at plane k from the values at prev(k), next(k)
  // (the seam planes as the reference writes them)
  auto dphi = [&](int k, double2 vp, double2 vn) {
    double2 z;
    if (k == 0) z = cadd(cneg(vp), vn);
    else if (k == g.Nz) z = cadd(cneg(vn), vp);
    else z = ctr(vp, vn);
    return rmul(g.rdz, z);
  };
  // rhs_psi1 at this lane's column (all r neighbours lie in the box); FAST:
  // the warp's columns are all at least two points from an array end and
  // beta^r > 0 on all of them, so every lane takes the centred derivative and
  // the forward upwind difference (the branches the general form would take)
  auto psi1_rhs = [&](const unsigned char* st, auto fastc) {
    constexpr bool FAST = decltype(fastc)::value;
    const double be = MAB(mBE, 0, 0);
    auto aPi = [&](int dc) { return rmul(MAB(mAL, dc, 0), RA(st, OFF_A4, dc, 0)); };
    auto ps1 = [&](int dc) { return RA(st, OFF_A1, dc, 0); };
    double2 d;
    if (FAST) d = ctr(aPi(-1), aPi(1));
    else if (c == 0) d = fwd3(aPi(0), aPi(1), aPi(2));
    else if (c == n) d = bwd3(aPi(0), aPi(-1), aPi(-2));
    else d = ctr(aPi(-1), aPi(1));
    d = rmul(g.rdx, d);
    const double2 f0 = ps1(0);
    double2 av;
    if (FAST) av = fwd3(f0, ps1(1), ps1(2));
    else if (c <= 1) av = fwd3(f0, ps1(1), ps1(2));
    else if (c == n - 1) av = csub(ps1(1), ps1(-1));
    else if (c == n) av = bwd3(f0, ps1(-1), ps1(-2));
    else if (be > 0.0) av = fwd3(f0, ps1(1), ps1(2));
    else if (be < 0.0) av = bwd3(f0, ps1(-1), ps1(-2));
    else av = csub(ps1(1), ps1(-1));
    av = rmul(g.rdx, av);
    return cadd(cadd(d, rmul(be, av)), rmul(dxb, f0));
  };
  // psi2 stage at this lane's column, row jj + dr of plane p (slot st)
  auto psi2_stage = [&](const unsigned char* st, int p, int dr) {
    const int r = jj + dr;
    double2 t;
    if (r == 0) t = cadd(cneg(Ebox(st, dr + 1)), Eglob(2, ktarget(g, p)));
    else if (r == g.NJ - 1) t = bwd3(Ebox(st, dr), Ebox(st, dr - 1), Ebox(st, dr - 2));
    else t = ctr(Ebox(st, dr - 1), Ebox(st, dr + 1));
    const double2 u2 = *reinterpret_cast<const double2*>(st + OFF_B + ((ty - B_R0 + dr) * B_NC + tx) * 16);
    return cadd(u2, rmul(g.dt, rmul(g.rdy, t)));
  };
  auto Hst = [&](double2* hb, int dr, double2 s2) {
    hb[(ty + 1 + dr) * FL + tx] = rmul(mHT[(ty - MHT_R0 + dr) * M_NC + tx + 1], s2);
  };

  // planes just outside the sequence whose E the psi3 stage at P[0] / P[NP-1] needs
  const int X1 = (plane_of(0) == 0) ? g.Nz - 2 : plane_of(0) - 1;        // prev(P[0])
  const int X4 = (plane_of(NP - 1) == g.Nz) ? 2 : plane_of(NP - 1) + 1;  // next(P[NP-1])
  double2 phinx = c2(0, 0);  // phi of the own point at the next inner plane, loaded a step ahead
  if (own) phinx = ldf(U, pcol + (long long)plane_of(1) * g.plane);
  __syncthreads();  // metric tables
  const bool ends = (i0 == 0) || (n < i0 + FO);  // the tile holds an array end (block-uniform)
  const bool fast = __all_sync(0xffffffffu, c >= 2 && c <= n - 2 && MAB(mBE, 0, 0) > 0.0);

  // rolling state
  double2 Ep = c2(0, 0), Ec = c2(0, 0);   // E at P[t-1], P[t]
  double2 Fm2 = c2(0, 0), Fm1 = c2(0, 0);  // phi flux of the Pi rhs at P[t-2], P[t-1]
  double2 Gc = c2(0, 0);                   // r flux of the Pi rhs at P[t-1]
  double2 S0p = c2(0, 0), U4p = c2(0, 0);  // phi stage and u(5) at P[t-1]
  double2 Hpc = c2(0, 0);                  // pole row: theta flux at row 2 of the partner of P[t-1]
  int timed_out = mbar_wait_bounded(&bars[slot(0)], parity(0)) ? 0 : 1;
  timed_out = __any_sync(0xffffffffu, timed_out) ? 1 : 0;
  if (!timed_out) Ec = Ebox(ring + (size_t)slot(0) * SLOT, 0);
  bool failed = __syncthreads_or(timed_out) != 0;

  // One step of the march at ring step t.  EDGE: t is 0 or NP-1 (E from global
  // memory outside the sequence); INNER: P[t] is one of the chunk's planes
  // (outputs, G and H); PI: the Pi stage of P[t-1] follows.  The steady state
  // (INNER and PI, not EDGE) has no branch around its blocks.
  auto step = [&](int t, auto fastc, auto edgec, auto innerc, auto pic) {
    constexpr bool FAST = decltype(fastc)::value, EDGE = decltype(edgec)::value;
    constexpr bool INNER = decltype(innerc)::value, PI_ = decltype(pic)::value;
    // slot t-1 was released by the barrier that ended the previous step
    if (tid == 0 && t >= 1 && t + 2 < NP) {
      issue(t + 2);
      nissued = t + 3;
    }
    if (t + 1 < NP && !mbar_wait_bounded(&bars[slot(t + 1)], parity(t + 1))) timed_out = 1;
    timed_out = __any_sync(0xffffffffu, timed_out) ? 1 : 0;
    if (!timed_out) {
      const int p = plane_of(t);
      const unsigned char* cu = ring + (size_t)slot(t) * SLOT;
      const double2 En = (t + 1 < NP) ? Ebox(ring + (size_t)slot(t + 1) * SLOT, 0) : c2(0, 0);
      // ---- psi1, psi3 stages and the phi flux F at P[t]
      double2 vp = Ep, vn = En;
      if (EDGE && vcol) {
        if (t == 0) {
          vp = Eglob(jj, X1);
          if (k0 == 0) vn = Eglob(jj, g.Nz - 1);  // next(Nz-2) is Nz-1, not plane 0
        } else {
          if (k1 - 1 == g.Nz) vp = Eglob(jj, 1);  // prev(2) is plane 1, not Nz
          vn = Eglob(jj, X4);
        }
      }
      const double2 S1 = cadd(RA(cu, OFF_A1, 0, 0), rmul(g.dt, psi1_rhs(cu, fastc)));
      const double2 u3 = *reinterpret_cast<const double2*>(cu + OFF_C + (ty * C_NC + tx) * 16);
      const double2 S3 = cadd(u3, rmul(g.dt, dphi(p, vp, vn)));
      const double2 F0 = (MK == MK_KS) ? rmul(fA, cadd(rmul(fgrp, S1), rmul(fgpp, S3))) : rmul(fgpp, S3);
      double2 Gn = c2(0, 0), S0 = c2(0, 0), U4n = c2(0, 0), Hpn = c2(0, 0);
      if (INNER) {
        Gn = (MK == MK_KS) ? rmul(fA, cadd(rmul(fgrr, S1), rmul(fgrp, S3))) : rmul(fA, S1);
        S0 = cadd(phinx, rmul(g.dt, Ec));
        // psi2 stage and the theta flux H on the lane's column (columns outside
        // the array: never read, and the pole row would read global memory there)
        const double2 S2 = (FAST || vcol) ? psi2_stage(cu, p, 0) : c2(0, 0);
        double2* hb = hbuf + (size_t)(t & 1) * H_NR * FL;
        Hst(hb, 0, S2);
        if ((FAST || vcol) && ty == 0 && j0 >= 1) Hst(hb, -1, psi2_stage(cu, p, -1));
        if ((FAST || vcol) && ty == FJ - 1 && j0 + FJ < g.NJ) Hst(hb, 1, psi2_stage(cu, p, 1));
        U4n = RA(cu, OFF_A4, 0, 0);
        if (own) {
          const long long o = pcol + (long long)p * g.plane;
          a.S[o] = S0;
          a.S[fs + o] = S1;
          a.S[2 * fs + o] = S2;
          a.S[3 * fs + o] = S3;
          if (jj == 0) {
            // theta flux at row 2 of the pole partner plane, from global memory
            // (row 2 is an interior row: a centred difference of E)
            const int pk = ktarget(g, p);
            const double2 tt = ctr(Eglob(1, pk), Eglob(3, pk));
            const double2 s2 = cadd(ldf(U + 2 * fs, off3(g, c, 2, pk)), rmul(g.dt, rmul(g.rdy, tt)));
            Hpn = rmul(ldm(M.asg_gtt, off2(g, c, 2)), s2);
          }
          if (t + 1 <= NP - 2) phinx = ldf(U, pcol + (long long)plane_of(t + 1) * g.plane);
        }
      }
      // ---- Pi stage of P[t-1]
      if (PI_) {
        const int pm = plane_of(t - 1);
        const double2 gm1 = shfl2_up(Gc, 1), gp1 = shfl2_down(Gc, 1);
        double2 gm2 = c2(0, 0), gp2 = c2(0, 0);
        if (!FAST && ends) {
          gm2 = shfl2_up(Gc, 2);
          gp2 = shfl2_down(Gc, 2);
        }
        // the shared-memory reads below stay inside the CTA's window on every lane
        // (lanes 0 and 31 read one value past the boxes' own columns, never used)
        const double sg = mSG[ty * M_NC + tx + 1], be = MAB(mBE, 0, 0);
        double2 d;
        if (FAST) d = ctr(gm1, gp1);
        else if (c == 0) d = fwd3(Gc, gp1, gp2);
        else if (c == n) d = bwd3(Gc, gm1, gm2);
        else d = ctr(gm1, gp1);
        const double2 r1 = fcdivm(rmul(g.rdx, d), sg, rs);
        const double2* hp = hbuf + (size_t)((t - 1) & 1) * H_NR * FL;
        auto Hr = [&](int dr) { return hp[(ty + 1 + dr) * FL + tx]; };
        double2 tt;
        if (jj == 0) tt = cadd(cneg(Hr(1)), Hpc);
        else if (jj == g.NJ - 1) tt = bwd3(Hr(0), Hr(-1), Hr(-2));
        else tt = ctr(Hr(-1), Hr(1));
        const double2 r2 = fcdivm(rmul(g.rdy, tt), sg, rs);
        const double2 z = dphi(pm, Fm2, F0);
        const double2 r3 = (MK == MK_KS) ? fcdivm(z, sg, rs) : z;
        auto PD = [&](int dc) {
          return *reinterpret_cast<const double2*>(cu + OFF_D + (ty * D_NC + (tx - 1 - D_C0 + dc)) * 16);
        };
        const double2 r4 = rmul(dxb, PD(0));
        auto Q = [&](int dc) { return rmul(mSG[ty * M_NC + tx + 1 + dc], PD(dc)); };
        double2 av;
        if (FAST) av = fwd3(Q(0), Q(1), Q(2));
        else if (c <= 1) av = fwd3(Q(0), Q(1), Q(2));
        else if (c == n - 1) av = csub(Q(1), Q(-1));
        else if (c == n) av = bwd3(Q(0), Q(-1), Q(-2));
        else if (be > 0.0) av = fwd3(Q(0), Q(1), Q(2));
        else if (be < 0.0) av = bwd3(Q(0), Q(-1), Q(-2));
        else av = csub(Q(1), Q(-1));
        av = rmul(g.rdx, av);
        const double2 r5 = fcdivm(rmul(be, av), sg, rs);
        const double2 r6 = rmul(am2, S0p);
        const double2 rr = csub(cadd(cadd(cadd(cadd(r1, r2), r3), r4), r5), r6);
        if (own) a.Snew[pcol + (long long)pm * g.plane] = cadd(U4p, rmul(g.dt, rr));
      }
      // roll
      Ep = Ec;
      Ec = En;
      Fm2 = Fm1;
      Fm1 = F0;
      Gc = Gn;
      S0p = S0;
      U4p = U4n;
      Hpc = Hpn;
    }
    // the H rows of P[t] are visible to every warp, and every warp is done
    // with ring slot t, which the next step refills
    failed = __syncthreads_or(timed_out) != 0;
  };
  // P[0]: psi stage only; P[1]: the first own plane; P[2 .. NP-2]: steady
  // state; P[NP-1]: psi stage and the Pi stage of the last own plane
  auto march = [&](auto fastc) {
    const BoolC<false> no;
    const BoolC<true> yes;
    // NP >= 3: a chunk holds at least one plane
    if (!failed) step(0, fastc, yes, no, no);
    if (!failed) step(1, fastc, no, yes, no);
    for (int t = 2; t <= NP - 2 && !failed; ++t) step(t, fastc, no, yes, yes);
    if (!failed) step(NP - 1, fastc, yes, no, yes);
  };
  if (fast) march(BoolC<true>());
  else march(BoolC<false>());
  if (failed) {
    if (tid == 0) {
      atomicExch(a.err, 1);
      // let the last copy issued into each ring slot land before the CTA's
      // shared memory is released (bounded as well)
      for (int s = 0; s < NSTF; ++s) {
        int tl = -1;
        for (int t = 0; t < nissued; ++t)
          if (slot(t) == s) tl = t;
        if (tl >= 0) (void)mbar_wait_bounded(&bars[s], parity(tl));
      }
    }
    __syncthreads();
  }
}

}  // namespace kg

// ---------------------------------------------------------------------------
namespace kg {
namespace {

typedef CUresult (*EncodeTiledFnF)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFnF encode_fn_f() {
  static EncodeTiledFnF fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFnF)p;
  }
  return fn;
}

// 4-D view of a state (doubles along r incl. row padding, theta rows, phi
// planes, variables) with a box of `cols` complex columns x `rows` rows of one
// variable of one plane
bool encode_box(CUtensorMap* tm, const Grid& g, const double2* base, int nvars, int cols, int rows) {
  EncodeTiledFnF fn = encode_fn_f();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)(2 * g.PI), (cuuint64_t)g.NJ, (cuuint64_t)g.NK, (cuuint64_t)nvars};
  cuuint64_t strides[3] = {(cuuint64_t)g.PI * 16, (cuuint64_t)g.plane * 16, (cuuint64_t)g.fs * 16};
  cuuint32_t box[4] = {(cuuint32_t)(2 * cols), (cuuint32_t)rows, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void*)base, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MK>
int fused_launch(const CUtensorMap* tms, const FusedArgs& a, cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(pirk_s1_fused_kernel<MK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM) !=
        cudaSuccess)
      return -1;
    attr_set = true;
  }
  const Grid& g = a.g;
  const int tiles_x = (g.NI <= FO) ? 1 : (g.NI + FO - 1) / FO;
  dim3 grid(tiles_x, (g.NJ + FJ - 1) / FJ, (g.NK + a.kchunk - 1) / a.kchunk);
  pirk_s1_fused_kernel<MK><<<grid, dim3(FL, FJ, 1), SMEM, st>>>(tms[0], tms[1], tms[2], tms[3], a);
  return 0;
}

}  // namespace

int launch_pirk_s1_fused(const Grid& g, const Metric& m, int mk, const double2* U, const double2* Sold, double2* S,
                         double2* Snew, const double* rsg, int* err, cudaStream_t st) {
  // the theta tiles hold FJ rows and the pole partner's row 2 is an interior row
  if (g.NJ < FJ || g.NJ < 5) return -1;
  CUtensorMap tms[4];
  if (!encode_box(&tms[0], g, U, 5, A_NC, A_NR) || !encode_box(&tms[1], g, U, 5, B_NC, B_NR) ||
      !encode_box(&tms[2], g, U, 5, C_NC, C_NR) || !encode_box(&tms[3], g, Sold, 1, D_NC, D_NR))
    return -1;
  FusedArgs a;
  a.g = g;
  a.m = m;
  a.rsg = rsg;
  a.U = U;
  a.Sold = Sold;
  a.S = S;
  a.Snew = Snew;
  a.err = err;
  // long chunks: each chunk reads two planes beyond its own
  const int nch = (g.NK + 63) / 64;
  a.kchunk = (g.NK + nch - 1) / nch;
  return mk == MK_KS ? fused_launch<MK_KS>(tms, a, st) : fused_launch<MK_SCHW>(tms, a, st);
}

}  // namespace kg
