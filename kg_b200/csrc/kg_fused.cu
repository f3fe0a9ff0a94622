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
// over u (176 B/point: u, the stale Pi slot, u_stage(1:5)):
//   * a CTA owns a 32 x TJ tile of (r, theta) columns (one warp per theta row)
//     and marches through a chunk of phi planes; the u planes arrive by TMA in
//     a 3-deep shared-memory ring (boxes: psi1 and Pi with a -2/+3 r and +-2
//     theta halo, psi2 with a +-1 theta halo, psi3 with a +-1 r halo, and the
//     stale Pi of the previous plane with a +-2 r halo), with the full/empty
//     mbarrier protocol of kg_tma.cu and bounded waits;
//   * at ring step t the CTA forms the psi stage of plane P[t] for its tile and
//     writes u_stage(1:4) there; the same warp also forms, from the same plane,
//     the psi2 stage on its theta neighbour rows (the Pi flux of the theta
//     derivative), and lanes 0 and 31 form psi1/psi3 stage values on the
//     columns just outside the tile (the Pi flux of the r derivative), so no
//     value has to cross warps or CTAs;
//   * the Pi stage of plane P[t-1] follows in the same step, from the fluxes of
//     the previous step kept in registers (r neighbours by warp shuffles), the
//     phi-flux of the own column at P[t-2] and P[t] (rolling registers) and the
//     stale Pi box; it is written to the new Pi slot.
// Every value is formed with the same operations in the same order as the
// two-launch form (kg_tma.cu, kinds ST_P2_S1A and ST_P2_S1B), so results are
// the same bits.  Values outside the boxes (the pole partner plane, the rows
// and columns the one-sided closures reach at a tile edge, the phi planes just
// outside the chunk) are read from global memory.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstring>
#include "kg_device.cuh"
#include "kg_internal.h"
#include "kg_tma_ops.cuh"

namespace kg {
using namespace tmaops;
namespace {

constexpr int FI = 32;           // r extent of a tile
constexpr int NSTF = 3;          // ring depth
// box extents in complex columns / rows relative to the tile origin (i0, j0)
constexpr int A_C0 = -2, A_NC = 37;   // psi1, Pi: columns i0-2 .. i0+34
constexpr int B_NC = 32;              // psi2: columns i0 .. i0+31, rows j0-1 .. j0+TJ
constexpr int C_C0 = -1, C_NC = 34;   // psi3: columns i0-1 .. i0+32, rows j0 .. j0+TJ-1
constexpr int D_C0 = -2, D_NC = 36;   // stale Pi: columns i0-2 .. i0+33, rows j0 .. j0+TJ-1
constexpr int MW = 36, M_C0 = -2;     // metric tile columns i0-2 .. i0+33

__host__ __device__ constexpr int rnd128(int b) { return (b + 127) / 128 * 128; }

template <int TJ>
struct Geo {
  static constexpr int A_ROWS = TJ + 4, B_ROWS = TJ + 2, C_ROWS = TJ, D_ROWS = TJ;
  static constexpr int A_BYTES = A_NC * 16 * A_ROWS;
  static constexpr int B_BYTES = B_NC * 16 * B_ROWS;
  static constexpr int C_BYTES = C_NC * 16 * C_ROWS;
  static constexpr int D_BYTES = D_NC * 16 * D_ROWS;
  static constexpr int OFF_A1 = 0;
  static constexpr int OFF_A4 = rnd128(A_BYTES);
  static constexpr int OFF_B = OFF_A4 + rnd128(A_BYTES);
  static constexpr int OFF_C = OFF_B + rnd128(B_BYTES);
  static constexpr int OFF_D = OFF_C + rnd128(C_BYTES);
  static constexpr int SLOT = OFF_D + rnd128(D_BYTES);
  // metric tile: alpha, beta, (alpha sqrtg) gamma^thth over TJ+4 rows from j0-2;
  // sqrtg, A, gamma^rr, gamma^rphi, d_r beta over the TJ tile rows
  static constexpr int MT_WIDE = MW * (TJ + 4), MT_TILE = MW * TJ;
  static constexpr int MT_DOUBLES = 3 * MT_WIDE + 5 * MT_TILE;
  static constexpr size_t SMEM = (size_t)NSTF * SLOT + (size_t)MT_DOUBLES * 8 + 2 * NSTF * 8 + 128;
};

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

__device__ __forceinline__ double2 shfl2(double2 v, int src) {
  return c2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ double2 shfl2_up(double2 v, int d) {
  return c2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ double2 shfl2_down(double2 v, int d) {
  return c2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}

__device__ __forceinline__ unsigned char* falign128(unsigned char* p) {
  const uint32_t a = saddr(p);
  return p + ((128u - (a & 127u)) & 127u);
}

}  // namespace

template <int MK, int TJ, int MINB>
__global__ void __launch_bounds__(FI * TJ, MINB)
    pirk_s1_fused_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                         const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD,
                         FusedArgs a) {
  using G = Geo<TJ>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* ring = falign128(smem_raw);
  double* mt = reinterpret_cast<double*>(ring + (size_t)NSTF * G::SLOT);
  uint64_t* bars = reinterpret_cast<uint64_t*>(mt + G::MT_DOUBLES);
  uint64_t* empty = bars + NSTF;
  const Grid& g = a.g;
  const Metric& M = a.m;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * FI + tx;
  const int i0 = blockIdx.x * FI, j0 = blockIdx.y * TJ;
  const int ii = i0 + tx, jj = j0 + ty;
  const int n = g.NI - 1;
  const bool row_act = jj < g.NJ;
  const bool act = row_act && ii < g.NI;
  const int k0 = blockIdx.z * a.kchunk;
  if (k0 >= g.NK) return;
  const int k1 = min(k0 + a.kchunk, g.NK);
  const int NP = (k1 - k0) + 2;
  const long long fs = g.fs;
  const double2* __restrict__ U = a.U;

  if (tid == 0) {
    for (int s = 0; s < NSTF; ++s) mbar_init(&bars[s], 1);
    for (int s = 0; s < NSTF; ++s) mbar_init(&empty[s], TJ);
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
  auto slot_tx = [&](int t) -> uint32_t {
    return (uint32_t)(2 * G::A_BYTES + G::B_BYTES + G::C_BYTES + (t >= 2 ? G::D_BYTES : 0));
  };
  auto issue = [&](int t) {
    unsigned char* dst = ring + (size_t)slot(t) * G::SLOT;
    uint64_t* b = &bars[slot(t)];
    mbar_expect_tx(b, slot_tx(t));
    const int z = plane_of(t);
    tma_load_4d(dst + G::OFF_A1, &tmA, 2 * (i0 + A_C0), j0 - 2, z, 1, b);
    tma_load_4d(dst + G::OFF_A4, &tmA, 2 * (i0 + A_C0), j0 - 2, z, 4, b);
    tma_load_4d(dst + G::OFF_B, &tmB, 2 * i0, j0 - 1, z, 2, b);
    tma_load_4d(dst + G::OFF_C, &tmC, 2 * (i0 + C_C0), j0, z, 3, b);
    // the stale Pi of the previous plane rides with this one: it is read in
    // the step that forms the Pi stage of plane P[t-1]
    if (t >= 2) tma_load_4d(dst + G::OFF_D, &tmD, 2 * (i0 + D_C0), j0, plane_of(t - 1), 0, b);
  };
  int nissued = 0;
  if (tid == 0) {
    for (int t = 0; t < NSTF && t < NP; ++t) {
      issue(t);
      nissued = t + 1;
    }
  }

  // metric tile (phi-independent), zero outside the array
  double* mAL = mt;
  double* mBE = mAL + G::MT_WIDE;
  double* mHT = mBE + G::MT_WIDE;
  double* mSG = mHT + G::MT_WIDE;
  double* mA = mSG + G::MT_TILE;
  double* mGRR = mA + G::MT_TILE;
  double* mGRP = mGRR + G::MT_TILE;
  double* mDXB = mGRP + G::MT_TILE;
  for (int t = tid; t < G::MT_WIDE; t += FI * TJ) {
    const int mx = t % MW, my = t / MW;
    const int gi = i0 + M_C0 + mx, gj = j0 - 2 + my;
    const bool in = gi >= 0 && gi < g.NI && gj >= 0 && gj < g.NJ;
    const int q = in ? off2(g, gi, gj) : 0;
    mAL[t] = in ? ldm(M.alpha, q) : 0.0;
    mBE[t] = in ? ldm(M.beta, q) : 0.0;
    mHT[t] = in ? ldm(M.asg_gtt, q) : 0.0;
  }
  for (int t = tid; t < G::MT_TILE; t += FI * TJ) {
    const int mx = t % MW, my = t / MW;
    const int gi = i0 + M_C0 + mx, gj = j0 + my;
    const bool in = gi >= 0 && gi < g.NI && gj >= 0 && gj < g.NJ;
    const int q = in ? off2(g, gi, gj) : 0;
    mSG[t] = in ? ldm(M.sqrtg, q) : 0.0;
    mA[t] = in ? ldm(MK == MK_KS ? M.asg : M.asg_grr, q) : 0.0;
    mGRR[t] = in ? ldm(M.grr, q) : 0.0;
    mGRP[t] = in ? ldm(M.grp, q) : 0.0;
    mDXB[t] = in ? ldm(M.dxbeta, q) : 0.0;
  }

  // ---- accessors -----------------------------------------------------------
  // ring values of plane slot `st` at absolute column c and row r
  auto RA = [&](const unsigned char* st, int off, int c, int r) -> double2 {  // psi1 / Pi box
    return *reinterpret_cast<const double2*>(st + off + ((size_t)(r - (j0 - 2)) * A_NC + (c - (i0 + A_C0))) * 16);
  };
  auto in_A = [&](int c, int r) { return c >= i0 + A_C0 && c < i0 + A_C0 + A_NC && r >= j0 - 2 && r < j0 + TJ + 2; };
  auto RB = [&](const unsigned char* st, int c, int r) -> double2 {
    return *reinterpret_cast<const double2*>(st + G::OFF_B + ((size_t)(r - (j0 - 1)) * B_NC + (c - i0)) * 16);
  };
  auto in_B = [&](int c, int r) { return c >= i0 && c < i0 + B_NC && r >= j0 - 1 && r < j0 + TJ + 1; };
  auto RC = [&](const unsigned char* st, int c, int r) -> double2 {
    return *reinterpret_cast<const double2*>(st + G::OFF_C + ((size_t)(r - j0) * C_NC + (c - (i0 + C_C0))) * 16);
  };
  auto RD = [&](const unsigned char* st, int c, int r) -> double2 {
    return *reinterpret_cast<const double2*>(st + G::OFF_D + ((size_t)(r - j0) * D_NC + (c - (i0 + D_C0))) * 16);
  };
  // metric: the wide tables (rows j0-2 ..) and the tile tables (rows j0 ..)
  auto MWd = [&](const double* t, int c, int r) { return t[(r - (j0 - 2)) * MW + (c - (i0 + M_C0))]; };
  auto MTl = [&](const double* t, int c, int r) { return t[(r - j0) * MW + (c - (i0 + M_C0))]; };
  auto in_MW = [&](int c, int r) { return c >= i0 + M_C0 && c < i0 + M_C0 + MW && r >= j0 - 2 && r < j0 + TJ + 2; };
  // checked forms: box or tile when inside, global memory otherwise
  auto u1c = [&](const unsigned char* st, int p, int c, int r) -> double2 {
    return in_A(c, r) ? RA(st, G::OFF_A1, c, r) : ldf(U + fs, off3(g, c, r, p));
  };
  auto u4c = [&](const unsigned char* st, int p, int c, int r) -> double2 {
    return in_A(c, r) ? RA(st, G::OFF_A4, c, r) : ldf(U + 4 * fs, off3(g, c, r, p));
  };
  auto u2c = [&](const unsigned char* st, int p, int c, int r) -> double2 {
    return in_B(c, r) ? RB(st, c, r) : ldf(U + 2 * fs, off3(g, c, r, p));
  };
  auto alc = [&](int c, int r) { return in_MW(c, r) ? MWd(mAL, c, r) : ldm(M.alpha, off2(g, c, r)); };
  auto bec = [&](int c, int r) { return in_MW(c, r) ? MWd(mBE, c, r) : ldm(M.beta, off2(g, c, r)); };
  // E = alpha Pi + beta^r psi1 (the psi fluxes; also the phi rhs)
  auto Eglob = [&](int c, int r, int p) {
    const int q = off2(g, c, r);
    const long long o = off3(g, c, r, p);
    return cadd(rmul(ldm(M.alpha, q), ldf(U + 4 * fs, o)), rmul(ldm(M.beta, q), ldf(U + fs, o)));
  };
  auto Ec = [&](const unsigned char* st, int p, int c, int r) {
    if (in_A(c, r) && in_MW(c, r))
      return cadd(rmul(MWd(mAL, c, r), RA(st, G::OFF_A4, c, r)), rmul(MWd(mBE, c, r), RA(st, G::OFF_A1, c, r)));
    return Eglob(c, r, p);
  };
  // rhs_psi1 at column c, row r of plane p (slot st); be_c, dxb_c at (c, r)
  auto psi1_rhs = [&](const unsigned char* st, int p, int c, int r, double be_c, double dxb_c) {
    auto aPi = [&](int cc) { return rmul(alc(cc, r), u4c(st, p, cc, r)); };
    auto ps1 = [&](int cc) { return u1c(st, p, cc, r); };
    double2 d;
    if (c == 0) d = fwd3(aPi(0), aPi(1), aPi(2));
    else if (c == n) d = bwd3(aPi(c), aPi(c - 1), aPi(c - 2));
    else d = ctr(aPi(c - 1), aPi(c + 1));
    d = rmul(g.rdx, d);
    const double2 f0 = ps1(c);
    double2 av;
    if (c <= 1) av = fwd3(f0, ps1(c + 1), ps1(c + 2));
    else if (c == n - 1) av = csub(ps1(c + 1), ps1(c - 1));
    else if (c == n) av = bwd3(f0, ps1(c - 1), ps1(c - 2));
    else if (be_c > 0.0) av = fwd3(f0, ps1(c + 1), ps1(c + 2));
    else if (be_c < 0.0) av = bwd3(f0, ps1(c - 1), ps1(c - 2));
    else av = csub(ps1(c + 1), ps1(c - 1));
    av = rmul(g.rdx, av);
    return cadd(cadd(d, rmul(be_c, av)), rmul(dxb_c, f0));
  };
  // the same for the tile's own columns, whose r neighbours (two on each side)
  // and alpha at +-1 all lie in the box and the tile: no bounds checks
  auto psi1_rhs_own = [&](const unsigned char* st, int c, int r, double be_c, double dxb_c) {
    auto aPi = [&](int cc) { return rmul(MWd(mAL, cc, r), RA(st, G::OFF_A4, cc, r)); };
    auto ps1 = [&](int cc) { return RA(st, G::OFF_A1, cc, r); };
    double2 d;
    if (c == 0) d = fwd3(aPi(0), aPi(1), aPi(2));
    else if (c == n) d = bwd3(aPi(c), aPi(c - 1), aPi(c - 2));
    else d = ctr(aPi(c - 1), aPi(c + 1));
    d = rmul(g.rdx, d);
    const double2 f0 = ps1(c);
    double2 av;
    if (c <= 1) av = fwd3(f0, ps1(c + 1), ps1(c + 2));
    else if (c == n - 1) av = csub(ps1(c + 1), ps1(c - 1));
    else if (c == n) av = bwd3(f0, ps1(c - 1), ps1(c - 2));
    else if (be_c > 0.0) av = fwd3(f0, ps1(c + 1), ps1(c + 2));
    else if (be_c < 0.0) av = bwd3(f0, ps1(c - 1), ps1(c - 2));
    else av = csub(ps1(c + 1), ps1(c - 1));
    av = rmul(g.rdx, av);
    return cadd(cadd(d, rmul(be_c, av)), rmul(dxb_c, f0));
  };
  // phi-direction difference of a quantity at plane k from its values at
  // prev(k) and next(k) (the seam planes as the reference writes them)
  auto dphi = [&](int k, double2 vp, double2 vn) {
    double2 z;
    if (k == 0) z = cadd(cneg(vp), vn);
    else if (k == g.Nz) z = cadd(cneg(vn), vp);
    else z = ctr(vp, vn);
    return rmul(g.rdz, z);
  };
  // psi2 stage at column c (own), row r of plane p: u2 + dt rhs_psi2
  auto psi2_stage = [&](const unsigned char* st, int p, int c, int r) {
    double2 t;
    if (r == 0) t = cadd(cneg(Ec(st, p, c, 1)), Eglob(c, 2, ktarget(g, p)));
    else if (r == g.NJ - 1) t = bwd3(Ec(st, p, c, r), Ec(st, p, c, r - 1), Ec(st, p, c, r - 2));
    else t = ctr(Ec(st, p, c, r - 1), Ec(st, p, c, r + 1));
    return cadd(u2c(st, p, c, r), rmul(g.dt, rmul(g.rdy, t)));
  };
  // the same at the pole partner plane, row 2, from global memory only
  auto psi2_stage_glob = [&](int c, int p) {
    const double2 t = ctr(Eglob(c, 1, p), Eglob(c, 3, p));
    return cadd(ldf(U + 2 * fs, off3(g, c, 2, p)), rmul(g.dt, rmul(g.rdy, t)));
  };
  auto G1of = [&](double A_, double grr_, double grp_, double2 s1, double2 s3) {
    if (MK == MK_KS) return rmul(A_, cadd(rmul(grr_, s1), rmul(grp_, s3)));
    return rmul(A_, s1);
  };

  // own-point metric: the tile holds alpha, beta, d_r beta, sqrtg, the r-flux
  // coefficients and the theta-flux coefficient; the rest stays in registers
  double rs = 1, am2 = 0, fgpp = 0;
  if (act) {
    const int q = off2(g, ii, jj);
    rs = ldm(a.rsg, q);
    am2 = ldm(M.am2, q);
    fgpp = ldm(MK == MK_KS ? M.gpp : M.a_gpp, q);
  }
  // halo column of this lane: lanes 0 and 31 the columns on either side of the
  // tile; lane 1 the second column to the left when the last column of the
  // array is the tile's first (its backward closure reaches two columns back)
  int hc = -1;
  if (tx == 0) hc = i0 - 1;
  else if (tx == FI - 1) hc = i0 + FI;
  else if (tx == 1 && i0 == n) hc = i0 - 2;
  const bool halo = row_act && hc >= 0 && hc < g.NI;
  const bool ends = (i0 == 0) || (n >= i0 && n < i0 + FI);  // the tile holds an array end (warp-uniform)
  const long long pcol = act ? off3(g, ii, jj, 0) : 0;

  // planes just outside the sequence whose E the own column needs
  const int X1 = (plane_of(0) == 0) ? g.Nz - 2 : plane_of(0) - 1;        // prev(P[0])
  const int X4 = (plane_of(NP - 1) == g.Nz) ? 2 : plane_of(NP - 1) + 1;  // next(P[NP-1])
  double2 phinx = c2(0, 0);  // phi of the own point at the next inner plane, loaded a step ahead
  if (act) phinx = ldf(U, pcol + (long long)plane_of(1) * g.plane);
  __syncthreads();  // metric tile

  // own-column E at a ring slot (alpha, beta from the tile)
  auto Eown = [&](const unsigned char* st) {
    return cadd(rmul(MTl(mAL + 2 * MW, ii, jj), RA(st, G::OFF_A4, ii, jj)),
                rmul(MTl(mBE + 2 * MW, ii, jj), RA(st, G::OFF_A1, ii, jj)));
  };
  // rolling state
  double2 EoP = c2(0, 0);                               // E own at P[t-1]
  double2 EhP = c2(0, 0), EhC = c2(0, 0);               // E at the halo column, P[t-1] and P[t]
  double2 Fm2 = c2(0, 0), Fm1 = c2(0, 0);               // phi-flux of the Pi rhs at P[t-2], P[t-1]
  double2 G1c = c2(0, 0), G1h = c2(0, 0);               // r-flux at P[t-1], own and halo column
  double2 Ha = c2(0, 0), Hb = c2(0, 0), Hc = c2(0, 0);  // theta fluxes at P[t-1]: neighbours, own
  double2 S0p = c2(0, 0), U4p = c2(0, 0);               // phi stage and u(5) at P[t-1]
  int timed_out = 0;

  for (int t = 0; t < NP; ++t) {
    if (tid == 0 && !timed_out && t >= 1 && t + 2 < NP) {
      if (mbar_wait_bounded(&empty[slot(t - 1)], parity(t - 1))) {
        issue(t + 2);
        nissued = t + 3;
      } else {
        timed_out = 1;
      }
    }
    if (!timed_out) {
      bool ok = mbar_wait_bounded(&bars[slot(t)], parity(t));
      if (ok && t + 1 < NP) ok = mbar_wait_bounded(&bars[slot(t + 1)], parity(t + 1));
      if (!ok) timed_out = 1;
    }
    // the step's shuffles need every lane: a wait that ran out stops the whole warp
    timed_out = __any_sync(0xffffffffu, timed_out) ? 1 : 0;
    if (row_act && !timed_out) {
      const int p = plane_of(t);
      const bool inner = (t >= 1 && t <= NP - 2);
      const unsigned char* cu = ring + (size_t)slot(t) * G::SLOT;
      const unsigned char* nx = ring + (size_t)slot(t + 1 < NP ? t + 1 : t) * G::SLOT;
      // ---- psi stage of the own point at P[t]: psi1 always (the phi-flux of
      // the Pi rhs), all four on the inner planes
      double2 EoC = c2(0, 0), S1 = c2(0, 0), S3 = c2(0, 0), F0 = c2(0, 0);
      if (act) {
        double2 EoN, EoPv = EoP;
        EoC = Eown(cu);
        if (t == 0) {
          EoPv = Eglob(ii, jj, X1);
          EoN = (k0 == 0) ? Eglob(ii, jj, g.Nz - 1) : Eown(nx);  // next(Nz-2) is Nz-1, not plane 0
        } else if (t == NP - 1) {
          if (k1 - 1 == g.Nz) EoPv = Eglob(ii, jj, 1);  // prev(2) is plane 1, not Nz
          EoN = Eglob(ii, jj, X4);
        } else {
          EoN = Eown(nx);
        }
        S1 = cadd(RA(cu, G::OFF_A1, ii, jj),
                  rmul(g.dt, psi1_rhs_own(cu, ii, jj, MWd(mBE, ii, jj), MTl(mDXB, ii, jj))));
        S3 = cadd(RC(cu, ii, jj), rmul(g.dt, dphi(p, EoPv, EoN)));
        const double fa = MTl(mA, ii, jj);  // alpha sqrtg (KS) / alpha gamma^phph (Schw, below)
        F0 = (MK == MK_KS) ? rmul(fa, cadd(rmul(MTl(mGRP, ii, jj), S1), rmul(fgpp, S3))) : rmul(fgpp, S3);
      }
      // halo columns: E rolls at every step; psi stage only on the inner planes
      double2 G1hn = c2(0, 0);
      if (halo) {
        if (t == 0) EhC = Ec(cu, p, hc, jj);
        const double2 EhN = (t + 1 < NP) ? Ec(nx, plane_of(t + 1), hc, jj) : c2(0, 0);
        if (inner) {
          const double2 s1 = cadd(u1c(cu, p, hc, jj),
                                  rmul(g.dt, psi1_rhs(cu, p, hc, jj, MWd(mBE, hc, jj), MTl(mDXB, hc, jj))));
          const double2 u3h = (hc >= i0 + C_C0) ? RC(cu, hc, jj) : ldf(U + 3 * fs, off3(g, hc, jj, p));
          const double2 s3 = cadd(u3h, rmul(g.dt, dphi(p, EhP, EhN)));
          G1hn = G1of(MTl(mA, hc, jj), MTl(mGRR, hc, jj), MTl(mGRP, hc, jj), s1, s3);
        }
        EhP = EhC;
        EhC = EhN;
      }
      double2 G1n = c2(0, 0), Han = c2(0, 0), Hbn = c2(0, 0), Hcn = c2(0, 0), S0n = c2(0, 0), U4n = c2(0, 0);
      if (inner && act) {
        // outputs u_stage(1:4) at P[t]
        const long long o = pcol + (long long)p * g.plane;
        S0n = cadd(phinx, rmul(g.dt, EoC));
        const double2 S2 = psi2_stage(cu, p, ii, jj);
        a.S[o] = S0n;
        a.S[fs + o] = S1;
        a.S[2 * fs + o] = S2;
        a.S[3 * fs + o] = S3;
        U4n = RA(cu, G::OFF_A4, ii, jj);
        G1n = G1of(MTl(mA, ii, jj), MTl(mGRR, ii, jj), MTl(mGRP, ii, jj), S1, S3);
        // theta-flux neighbours of the Pi rhs: rows jj-1, jj+1 (pole row: row 1
        // and row 2 of the partner plane; last row: jj-1, jj-2 and its own)
        auto Hrow = [&](int r) {
          const double htr = (r >= j0 - 2 && r < j0 + TJ + 2) ? MWd(mHT, ii, r) : ldm(M.asg_gtt, off2(g, ii, r));
          return rmul(htr, psi2_stage(cu, p, ii, r));
        };
        if (jj == 0) {
          Han = Hrow(1);
          Hbn = rmul(ldm(M.asg_gtt, off2(g, ii, 2)), psi2_stage_glob(ii, ktarget(g, p)));
        } else if (jj == g.NJ - 1) {
          Han = Hrow(jj - 1);
          Hbn = Hrow(jj - 2);
          Hcn = rmul(MWd(mHT, ii, jj), S2);
        } else {
          Han = Hrow(jj - 1);
          Hbn = Hrow(jj + 1);
        }
        if (t + 1 <= NP - 2) phinx = ldf(U, pcol + (long long)plane_of(t + 1) * g.plane);
      }
      // ---- Pi stage of P[t-1]
      if (t >= 2) {
        const int pm = plane_of(t - 1);
        // r-flux neighbours from the previous step (lanes 0 / 31: the halo columns)
        double2 gm1 = shfl2_up(G1c, 1), gp1 = shfl2_down(G1c, 1);
        const double2 hl = shfl2(G1h, 0), hr = shfl2(G1h, FI - 1);
        if (tx == 0) gm1 = hl;
        if (tx == FI - 1) gp1 = hr;
        double2 gm2 = c2(0, 0), gp2 = c2(0, 0);
        if (ends) {
          gm2 = shfl2_up(G1c, 2);
          gp2 = shfl2_down(G1c, 2);
          const double2 hl2 = shfl2(G1h, 1);
          if (tx == 1) gm2 = hl;
          if (tx == 0) gm2 = hl2;
        }
        if (act) {
          const double sg = MTl(mSG, ii, jj), be = MTl(mBE + 2 * MW, ii, jj);
          double2 d;
          if (ii == 0) d = fwd3(G1c, gp1, gp2);
          else if (ii == n) d = bwd3(G1c, gm1, gm2);
          else d = ctr(gm1, gp1);
          const double2 r1 = fcdivm(rmul(g.rdx, d), sg, rs);
          double2 tt;
          if (jj == 0) tt = cadd(cneg(Ha), Hb);
          else if (jj == g.NJ - 1) tt = bwd3(Hc, Ha, Hb);
          else tt = ctr(Ha, Hb);
          const double2 r2 = fcdivm(rmul(g.rdy, tt), sg, rs);
          const double2 z = dphi(pm, Fm2, F0);
          const double2 r3 = (MK == MK_KS) ? fcdivm(z, sg, rs) : z;
          const double2 r4 = rmul(MTl(mDXB, ii, jj), RD(cu, ii, jj));
          auto Q = [&](int dx) { return rmul(MTl(mSG, ii + dx, jj), RD(cu, ii + dx, jj)); };
          double2 av;
          if (ii <= 1) av = fwd3(Q(0), Q(1), Q(2));
          else if (ii == n - 1) av = csub(Q(1), Q(-1));
          else if (ii == n) av = bwd3(Q(0), Q(-1), Q(-2));
          else if (be > 0.0) av = fwd3(Q(0), Q(1), Q(2));
          else if (be < 0.0) av = bwd3(Q(0), Q(-1), Q(-2));
          else av = csub(Q(1), Q(-1));
          av = rmul(g.rdx, av);
          const double2 r5 = fcdivm(rmul(be, av), sg, rs);
          const double2 r6 = rmul(am2, S0p);
          const double2 rr = csub(cadd(cadd(cadd(cadd(r1, r2), r3), r4), r5), r6);
          a.Snew[pcol + (long long)pm * g.plane] = cadd(U4p, rmul(g.dt, rr));
        }
      }
      // roll
      EoP = EoC;
      Fm2 = Fm1;
      Fm1 = F0;
      G1c = G1n;
      G1h = G1hn;
      Ha = Han;
      Hb = Hbn;
      Hc = Hcn;
      S0p = S0n;
      U4p = U4n;
    }
    __syncwarp();
    if (tx == 0) mbar_arrive(&empty[slot(t)]);
  }
  const bool failed = __syncthreads_or(timed_out) != 0;
  if (failed) {
    if (tid == 0) {
      atomicExch(a.err, 1);
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

template <int MK, int TJ, int MINB>
int fused_launch(const CUtensorMap* tms, const FusedArgs& a, cudaStream_t st) {
  using G = Geo<TJ>;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(pirk_s1_fused_kernel<MK, TJ, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)G::SMEM) != cudaSuccess)
      return -1;
    attr_set = true;
  }
  const Grid& g = a.g;
  dim3 grid((g.NI + FI - 1) / FI, (g.NJ + TJ - 1) / TJ, (g.NK + a.kchunk - 1) / a.kchunk);
  pirk_s1_fused_kernel<MK, TJ, MINB><<<grid, dim3(FI, TJ, 1), G::SMEM, st>>>(tms[0], tms[1], tms[2], tms[3], a);
  return 0;
}

template <int TJ, int MINB>
int fused_cfg(const Grid& g, const CUtensorMap* tms, const FusedArgs& a, int mk, cudaStream_t st) {
  return mk == MK_KS ? fused_launch<MK_KS, TJ, MINB>(tms, a, st) : fused_launch<MK_SCHW, TJ, MINB>(tms, a, st);
}

}  // namespace

int launch_pirk_s1_fused(int cfg, const Grid& g, const Metric& m, int mk, const double2* U, const double2* Sold,
                         double2* S, double2* Snew, const double* rsg, int* err, cudaStream_t st) {
  const int TJ = (cfg == 2) ? 12 : 8;
  CUtensorMap tms[4];
  if (!encode_box(&tms[0], g, U, 5, A_NC, TJ + 4) || !encode_box(&tms[1], g, U, 5, B_NC, TJ + 2) ||
      !encode_box(&tms[2], g, U, 5, C_NC, TJ) || !encode_box(&tms[3], g, Sold, 1, D_NC, TJ))
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
  switch (cfg) {
    case 1: return fused_cfg<8, 1>(g, tms, a, mk, st);
    case 2: return fused_cfg<12, 1>(g, tms, a, mk, st);
    default: return fused_cfg<8, 2>(g, tms, a, mk, st);
  }
}

}  // namespace kg
