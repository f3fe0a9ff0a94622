// kg_ylm_gemm.cu -- the Y_lm projection of phi over every radial shell as a
// tensor-core GEMM (tcgen05, BF16 inputs, FP32 accumulation in TMEM).
//
// The reference projects phi onto Y_lm at a detector radius
// (tools/FFT_sph.f90:247-279, proyector_detectors in MoL/diagnostic_lib.f90):
//   a_lm = dtheta dphi sum_jk w_jk f(j,k) conj(Y_lm(j,k)) sin(theta_j)
// on the vertex sphere, with trapezium weights w_jk.  Over all Nx shells this
// is one dense contraction.  With f = a + i b, Y_lm = C + i S (m >= 0) and
// P = a.C', Q = a.S', R = b.C', T = b.S' (C' = w sin C, S' = w sin S):
//   a_lm = (P + T) + i (R - Q),   a_l,-m = (-1)^m [(P - T) + i (R + Q)].
// So the projection is the real GEMM  [a; b] (2 Nx x K)  times  [C' S'] (K x 2 Nm)
// with K = Ny Nz sphere points and Nm = (L+1)(L+2)/2 modes with m >= 0.
//
// Precision: each operand is split into a BF16 head and a BF16 tail
// (x = hi + lo, |lo| <= 2^-8 |x|); the product is formed as the three-term sum
// hi.hi + hi.lo + lo.hi, all accumulated in FP32 -- three passes of the same
// BF16 GEMM over K, the dropped lo.lo term being of order 2^-16.
//
// Split K: each CTA sums the three passes over one range of at most KB_SPLIT
// K-slices of 64 (3072 sphere points) into its own FP32 partial tile, and the
// assembly adds the partials in FP64.  A single FP32 accumulator over the whole
// K = 33153 of the 129 x 257 sphere took some 6000 accumulation steps and
// carried an error near 1e-4 of the shell norm; per split it is ~20x shorter.
//
// GEMM kernel: one CTA per 128 x 256 output tile and K range, 4 warps.  Warp 0 lane 0
// feeds a 4-deep shared-memory ring with TMA (cp.async.bulk.tensor 2-D,
// 128-byte swizzle, K-major 64-element slices); warp 1 lane 0 issues
// tcgen05.mma (kind::f16, M=128, N=256, K=16 per instruction) into a TMEM
// accumulator of 256 columns and releases ring slots with tcgen05.commit; all
// four warps then read the accumulator with tcgen05.ld (32 lanes each) and
// store FP32 rows.  Every mbarrier wait is bounded; a CTA that runs out sets
// the error flag and still frees its TMEM.  No multicast is used.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "kg_device.cuh"
#include "kg_internal.h"
#include "kg_diag.h"

namespace kg {
namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int KB_SPLIT = 48;  // K-slices per CTA
constexpr int A_TILE_B = BM * BK * 2;  // 16 KB
constexpr int B_TILE_B = BN * BK * 2;  // 32 KB
constexpr int STAGE_B = A_TILE_B + B_TILE_B;
constexpr size_t GEMM_SMEM = (size_t)STAGES * STAGE_B + 1024 /*align*/ + 256 /*barriers, tmem slot*/;
constexpr long long WAIT_LIMIT = 1LL << 24;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t c) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(c) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i)
    if (mbar_try(b, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* tm, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(saddr(bar))
      : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t sw128_desc(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr & 0x3FFFFu) >> 4);  // start address (16-byte units), bits 0-13
  d |= (uint64_t)1 << 16;                        // leading-byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;              // stride-byte offset between 8-row groups
  d |= (uint64_t)1 << 46;                        // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                        // layout: 128-byte swizzle
  return d;
}

// instruction descriptor: kind::f16 with BF16 A and B, FP32 accumulator, both K-major
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(IDESC), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}

}  // namespace

// C_z (M' x ldc, FP32, row-major) = sum over three passes of A_p B_p^T over
// the K-slices [z KB_SPLIT, (z+1) KB_SPLIT) of split z = blockIdx.z, pass 0:
// (Ahi, Bhi), 1: (Ahi, Blo), 2: (Alo, Bhi); A and B K-major BF16; the split
// partials C_z lie csplit floats apart.
__global__ void __launch_bounds__(128, 1)
    ylm_gemm_kernel(const __grid_constant__ CUtensorMap tAhi, const __grid_constant__ CUtensorMap tAlo,
                    const __grid_constant__ CUtensorMap tBhi, const __grid_constant__ CUtensorMap tBlo, float* C,
                    int ldc, int Mrows, int Ncols, int K, long long csplit, int* err) {
  extern __shared__ __align__(1024) unsigned char gsm[];
  unsigned char* base = gsm + ((1024u - (saddr(gsm) & 1023u)) & 1023u);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + (size_t)STAGES * STAGE_B);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kb0 = blockIdx.z * KB_SPLIT;
  const int nk = min(K / BK - kb0, KB_SPLIT);  // K-slices of this split (>= 1 by the launch)
  const int total = 3 * nk;
  C += (long long)blockIdx.z * csplit;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)),
                 "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  int bad = 0;

  if (warp == 0 && lane == 0) {
    // producer
    for (int it = 0; it < total && !bad; ++it) {
      const int s = it % STAGES;
      if (it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1)) {
        bad = 1;
        break;
      }
      const int pass = it / nk, kb = kb0 + it % nk;
      unsigned char* sa = base + (size_t)s * STAGE_B;
      unsigned char* sb = sa + A_TILE_B;
      mbar_expect_tx(&full[s], STAGE_B);
      tma_2d(sa, pass == 2 ? &tAlo : &tAhi, kb * BK, m0, &full[s]);
      tma_2d(sb, pass == 1 ? &tBlo : &tBhi, kb * BK, n0, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    for (int it = 0; it < total && !bad; ++it) {
      const int s = it % STAGES;
      if (!mbar_wait(&full[s], (it / STAGES) & 1)) {
        bad = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = saddr(base + (size_t)s * STAGE_B);
      const uint32_t sb = sa + A_TILE_B;
#pragma unroll
      for (int k = 0; k < BK / 16; ++k)
        umma(tmem, sw128_desc(sa + k * 32), sw128_desc(sb + k * 32), (it > 0 || k > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  __syncwarp();
  // epilogue: every warp reads its 32 accumulator lanes (tcgen05.ld is warp-collective,
  // so the error decision is made block-uniform first)
  if (!mbar_wait(done, 0)) bad = 1;
  bad = __syncthreads_or(bad);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int row = m0 + warp * 32 + lane;
  if (!bad) {
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
            "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < Mrows && n0 + c0 < Ncols) {
        float4* dst = reinterpret_cast<float4*>(C + (size_t)row * ldc + n0 + c0);
#pragma unroll
        for (int q = 0; q < 8; ++q)
          dst[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                               __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
      }
    }
  }
  if (bad && threadIdx.x == 0) atomicExch(err, 2);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
  }
}

// ---------------------------------------------------------------------------
// operand preparation

// phi on every vertex shell (domain_to_sph at all r), split into BF16 head/tail:
// A rows 0..Nx-1 = Re, Nx..2Nx-1 = Im, columns (jv, kv) -> jv + Ny kv, row pitch Kp.
// A block transposes a tile of 32 shells x 64 sphere columns through shared
// memory: each warp reads the interpolation points of one sphere column on 32
// consecutive shells (consecutive r, so the loads are coalesced), and each warp
// then writes 64 consecutive columns of one shell's A rows.  The value of each
// point is the same expression as the one-point-per-thread form gave.
constexpr int SA_R = 32, SA_C = 64;
__global__ void __launch_bounds__(256) shells_to_a_kernel(Grid g, const double2* __restrict__ u, ShellInterp si,
                                                          int Nx, int Ny, int Nz, int Kp, __nv_bfloat16* Ahi,
                                                          __nv_bfloat16* Alo, double2* Fout) {
  __shared__ double2 T[SA_C][SA_R + 1];  // odd pitch in 16-byte units: conflict-free column reads
  __shared__ int s_ith[SA_C], s_iph[SA_C], s_fl[SA_C];
  __shared__ double s_wt[SA_C], s_wp[SA_C];
  const int K = Ny * Nz;
  const int iv0 = blockIdx.x * SA_R, col0 = blockIdx.y * SA_C;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // the interpolation data of the block's sphere columns, once
  if (threadIdx.x < SA_C) {
    const int col = col0 + threadIdx.x;
    if (col < K) {
      const int jv = col % Ny, kv = col / Ny;
      s_ith[threadIdx.x] = si.i_th[jv];
      s_iph[threadIdx.x] = si.i_ph[kv];
      s_fl[threadIdx.x] = si.th_flag[jv];
      s_wt[threadIdx.x] = si.w_th[jv];
      s_wp[threadIdx.x] = si.w_ph[kv];
    }
  }
  __syncthreads();
#pragma unroll 4
  for (int cc = warp; cc < SA_C; cc += 8) {
    const int col = col0 + cc, iv = iv0 + lane;  // 0-based shell: vertex r index iv+1 -> evolution ii = iv
    double2 f = c2(0.0, 0.0);
    if (col < K && iv < Nx) {
      const int ir = iv, ith = s_ith[cc], iph = s_iph[cc];
      const int fl = s_fl[cc];
      if (fl == 1) f = u[off3(g, ir, 0, iph)];
      else if (fl == 2) f = u[off3(g, ir, g.NJ - 1, iph)];
      else {
        const double wt = s_wt[cc], wp = s_wp[cc];
        const int ip1 = iph + 1;
        const double2 f00 = cadd(rmul(1.0 - wp, u[off3(g, ir, ith, iph)]), rmul(wp, u[off3(g, ir, ith, ip1)]));
        const double2 f01 =
            cadd(rmul(1.0 - wp, u[off3(g, ir, ith + 1, iph)]), rmul(wp, u[off3(g, ir, ith + 1, ip1)]));
        f = cadd(rmul(1.0 - wt, f00), rmul(wt, f01));
      }
    }
    T[cc][lane] = f;
  }
  __syncthreads();
  for (int rr = warp; rr < SA_R; rr += 8) {
    const int iv = iv0 + rr;
    if (iv >= Nx) break;
    if (Fout) {
      for (int c = lane; c < SA_C; c += 32) {
        const int col = col0 + c;
        if (col < K) Fout[(long long)iv * K + col] = T[c][rr];
      }
    }
    if (Ahi) {
      // two adjacent columns per lane, stored as BF16 pairs (col0 and Kp are even)
      const int c = 2 * lane, col = col0 + c;
      if (col < K) {
        const double2 f0 = T[c][rr];
        const double2 f1 = (col + 1 < K) ? T[c + 1][rr] : c2(0.0, 0.0);  // K <= column < Kp: the zero pad
        const float re0 = (float)f0.x, im0 = (float)f0.y, re1 = (float)f1.x, im1 = (float)f1.y;
        const __nv_bfloat16 rh0 = __float2bfloat16_rn(re0), ih0 = __float2bfloat16_rn(im0);
        const __nv_bfloat16 rh1 = __float2bfloat16_rn(re1), ih1 = __float2bfloat16_rn(im1);
        const __nv_bfloat162 rh = __halves2bfloat162(rh0, rh1), ih = __halves2bfloat162(ih0, ih1);
        const __nv_bfloat162 rl = __halves2bfloat162(__float2bfloat16_rn(re0 - __bfloat162float(rh0)),
                                                     __float2bfloat16_rn(re1 - __bfloat162float(rh1)));
        const __nv_bfloat162 il = __halves2bfloat162(__float2bfloat16_rn(im0 - __bfloat162float(ih0)),
                                                     __float2bfloat16_rn(im1 - __bfloat162float(ih1)));
        *reinterpret_cast<__nv_bfloat162*>(Ahi + (long long)iv * Kp + col) = rh;
        *reinterpret_cast<__nv_bfloat162*>(Alo + (long long)iv * Kp + col) = rl;
        *reinterpret_cast<__nv_bfloat162*>(Ahi + (long long)(Nx + iv) * Kp + col) = ih;
        *reinterpret_cast<__nv_bfloat162*>(Alo + (long long)(Nx + iv) * Kp + col) = il;
      }
    }
  }
}

// B^T rows: n < Nm: w sin C_lm, Nm <= n < 2Nm: w sin S_lm (mode index n of (l, m>=0) as l(l+1)/2 + m)
__global__ void ylm_b_kernel(int L, int Ny, int Nz, int Kp, const double* __restrict__ normP,
                             const double* __restrict__ cosm, const double* __restrict__ sinm,
                             const double* __restrict__ sint, __nv_bfloat16* Bhi, __nv_bfloat16* Blo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Nm = (L + 1) * (L + 2) / 2;
  const long long n = (long long)2 * Nm * Ny * Nz;
  if (t >= n) return;
  const int jv = (int)(t % Ny);
  const long long r2 = t / Ny;
  const int kv = (int)(r2 % Nz);
  const int row = (int)(r2 / Nz);
  const int mode = row % Nm, part = row / Nm;
  int l = 0;
  while ((l + 1) * (l + 2) / 2 <= mode) ++l;
  const int m = mode - l * (l + 1) / 2;
  const int sel = ((jv == 0 || jv == Ny - 1) ? 1 : 0) + 2 * ((kv == 0 || kv == Nz - 1) ? 1 : 0);
  const double w = sel == 0 ? 1.0 : (sel == 3 ? 0.25 : 0.5);
  const double np = normP[((long long)l * (L + 1) + m) * Ny + jv];
  const double trig = part == 0 ? cosm[(long long)m * Nz + kv] : sinm[(long long)m * Nz + kv];
  const float v = (float)(w * sint[jv] * (np * trig));
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  const long long o = (long long)row * Kp + jv + (long long)Ny * kv;
  Bhi[o] = h;
  Blo[o] = __float2bfloat16_rn(v - __bfloat162float(h));
}

// a_lm(l, m, shell) from the GEMM blocks P Q / R T.  One thread per (mode with
// m >= 0, shell), modes fastest, so the reads of each split's partial rows are
// coalesced; the thread writes a_l,m and a_l,-m.  The entries with |m| > l are
// never written: the caller zeroes them once per buffer layout.
__global__ void ylm_assemble_kernel(const float* __restrict__ C, int ldc, long long csplit, int nsplit, int Nx,
                                    int L, double dydz, double2* __restrict__ alm) {
  const int Nm = (L + 1) * (L + 2) / 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)Nm * Nx) return;
  const int mode = (int)(t % Nm);
  const int iv = (int)(t / Nm);
  int l = (int)((sqrt(8.0 * mode + 1.0) - 1.0) * 0.5);  // mode = l (l + 1) / 2 + m
  while (l * (l + 1) / 2 > mode) --l;
  while ((l + 1) * (l + 2) / 2 <= mode) ++l;
  const int am = mode - l * (l + 1) / 2;
  // the split partials added in FP64, in split order; four splits' loads are
  // issued before their sums, so a thread has sixteen loads in flight
  double P = 0.0, Q = 0.0, R = 0.0, T = 0.0;
  const float* c0 = C + (size_t)iv * ldc + mode;
  const float* c1 = C + (size_t)(Nx + iv) * ldc + mode;
  int z = 0;
  for (; z + 4 <= nsplit; z += 4) {
    float p[4], q[4], r[4], t4[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      const long long o = (long long)(z + w) * csplit;
      p[w] = __ldg(c0 + o);
      q[w] = __ldg(c0 + o + Nm);
      r[w] = __ldg(c1 + o);
      t4[w] = __ldg(c1 + o + Nm);
    }
#pragma unroll
    for (int w = 0; w < 4; ++w) {
      P += (double)p[w];
      Q += (double)q[w];
      R += (double)r[w];
      T += (double)t4[w];
    }
  }
  for (; z < nsplit; ++z) {
    const long long o = (long long)z * csplit;
    P += (double)__ldg(c0 + o);
    Q += (double)__ldg(c0 + o + Nm);
    R += (double)__ldg(c1 + o);
    T += (double)__ldg(c1 + o + Nm);
  }
  const int NL = L + 1, NM = 2 * L + 1;
  alm[((long long)iv * NM + (L + am)) * NL + l] = rmul(dydz, c2(P + T, R - Q));
  if (am > 0) {
    const double sg = (am & 1) ? -1.0 : 1.0;
    alm[((long long)iv * NM + (L - am)) * NL + l] = rmul(dydz, c2(sg * (P - T), sg * (R + Q)));
  }
}

// FP64 projection over all shells.  One block per (l-chunk, m >= 0, shell): the
// shell is read once for LC degrees and both signs of m, from four real sums per
// degree (f = a + ib, Y_lm = C + iS, m >= 0):
//   a_lm   = dtdp sum w sin [(aC + bS) + i (bC - aS)]
//   a_l,-m = (-1)^m dtdp sum w sin [(aC - bS) + i (bC + aS)]
constexpr int LC = 8;
__global__ void __launch_bounds__(256) ylm_fp64_kernel(const double2* __restrict__ F, int Nx, int L, int Ny, int Nz,
                                                       const double* __restrict__ normP,
                                                       const double* __restrict__ cosm,
                                                       const double* __restrict__ sinm,
                                                       const double* __restrict__ sint, double dydz,
                                                       double2* __restrict__ alm) {
  const int l0 = blockIdx.x * LC, m = blockIdx.y, iv = blockIdx.z;
  const int NL = L + 1, NM = 2 * L + 1;
  double acc[LC][4];
#pragma unroll
  for (int q = 0; q < LC; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.0;
  const double2* f = F + (long long)iv * Ny * Nz;
  const double* cm = cosm + (long long)m * Nz;
  const double* sm = sinm + (long long)m * Nz;
  for (int t = threadIdx.x; t < Ny * Nz; t += blockDim.x) {
    const int jv = t % Ny, kv = t / Ny;
    const int sel = ((jv == 0 || jv == Ny - 1) ? 1 : 0) + 2 * ((kv == 0 || kv == Nz - 1) ? 1 : 0);
    const double w = (sel == 0 ? 1.0 : (sel == 3 ? 0.25 : 0.5)) * sint[jv];
    const double2 a = f[t];
    const double c = cm[kv], s = sm[kv];
    const double ac = w * (a.x * c), bs = w * (a.y * s), bc = w * (a.y * c), as = w * (a.x * s);
#pragma unroll
    for (int q = 0; q < LC; ++q) {
      const int l = l0 + q;
      if (l <= L && l >= m) {
        const double np = normP[((long long)l * NL + m) * Ny + jv];
        acc[q][0] += np * ac;
        acc[q][1] += np * bs;
        acc[q][2] += np * bc;
        acc[q][3] += np * as;
      }
    }
  }
  __shared__ double red[8][LC * 4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < LC; ++q)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      double v = acc[q][e];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) red[warp][q * 4 + e] = v;
    }
  __syncthreads();
  if (threadIdx.x < LC) {
    const int q = threadIdx.x, l = l0 + q;
    if (l > L) return;
    double ac = 0.0, bs = 0.0, bc = 0.0, as = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      ac += red[w][q * 4 + 0];
      bs += red[w][q * 4 + 1];
      bc += red[w][q * 4 + 2];
      as += red[w][q * 4 + 3];
    }
    double2* o = alm + (long long)NL * NM * iv;
    if (l < m) {  // outside |m| <= l: zero both entries
      o[l + NL * (m + L)] = c2(0.0, 0.0);
      o[l + NL * (-m + L)] = c2(0.0, 0.0);
      return;
    }
    o[l + NL * (m + L)] = c2(dydz * (ac + bs), dydz * (bc - as));
    if (m > 0) {
      const double sg = (m & 1) ? -1.0 : 1.0;
      o[l + NL * (-m + L)] = c2(dydz * (sg * (ac - bs)), dydz * (sg * (bc + as)));
    }
  }
}

// ---------------------------------------------------------------------------
namespace {
typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeFn enc() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeFn)p;
  }
  return fn;
}
bool map_kmajor(CUtensorMap* tm, const __nv_bfloat16* p, int Kp, int rows, int box_rows) {
  EncodeFn fn = enc();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)Kp * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)p, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}
}  // namespace

int ylm_gemm_pad_m(int rows) { return (rows + BM - 1) / BM * BM; }
int ylm_gemm_pad_n(int cols) { return (cols + BN - 1) / BN * BN; }
int ylm_gemm_pad_k(int k) { return (k + BK - 1) / BK * BK; }
int ylm_gemm_splits(int Kp) { return (Kp / BK + KB_SPLIT - 1) / KB_SPLIT; }

// C_z (Mp x Np each, ylm_gemm_splits(Kp) of them, back to back) = three-pass
// split-BF16 product over split z's K range; all dimensions already padded
int launch_ylm_gemm(const __nv_bfloat16* Ahi, const __nv_bfloat16* Alo, const __nv_bfloat16* Bhi,
                    const __nv_bfloat16* Blo, float* C, int Mp, int Np, int Kp, int* err, cudaStream_t st) {
  CUtensorMap a0, a1, b0, b1;
  if (!map_kmajor(&a0, Ahi, Kp, Mp, BM) || !map_kmajor(&a1, Alo, Kp, Mp, BM) || !map_kmajor(&b0, Bhi, Kp, Np, BN) ||
      !map_kmajor(&b1, Blo, Kp, Np, BN))
    return -1;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(ylm_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM) !=
        cudaSuccess)
      return -1;
    attr = true;
  }
  ylm_gemm_kernel<<<dim3(Np / BN, Mp / BM, ylm_gemm_splits(Kp)), 128, GEMM_SMEM, st>>>(
      a0, a1, b0, b1, C, Np, Mp, Np, Kp, (long long)Mp * Np, err);
  return 0;
}

void launch_shells_to_a(const Grid& g, const double2* u, const ShellInterp& si, int Nx, int Ny, int Nz, int Kp,
                        __nv_bfloat16* Ahi, __nv_bfloat16* Alo, double2* F, cudaStream_t st) {
  const dim3 grid((Nx + SA_R - 1) / SA_R, (Ny * Nz + SA_C - 1) / SA_C);
  shells_to_a_kernel<<<grid, 256, 0, st>>>(g, u, si, Nx, Ny, Nz, Kp, Ahi, Alo, F);
}

void launch_ylm_b(int L, int Ny, int Nz, int Kp, const double* normP, const double* cosm, const double* sinm,
                  const double* sint, __nv_bfloat16* Bhi, __nv_bfloat16* Blo, cudaStream_t st) {
  const int Nm = (L + 1) * (L + 2) / 2;
  const long long n = (long long)2 * Nm * Ny * Nz;
  ylm_b_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(L, Ny, Nz, Kp, normP, cosm, sinm, sint, Bhi, Blo);
}

void launch_ylm_assemble(const float* C, int ldc, long long csplit, int nsplit, int Nx, int L, double dydz,
                         double2* alm, cudaStream_t st) {
  const long long n = (long long)(L + 1) * (L + 2) / 2 * Nx;
  ylm_assemble_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(C, ldc, csplit, nsplit, Nx, L, dydz, alm);
}

void launch_ylm_fp64(const double2* F, int Nx, int L, int Ny, int Nz, const double* normP, const double* cosm,
                     const double* sinm, const double* sint, double dydz, double2* alm, cudaStream_t st) {
  ylm_fp64_kernel<<<dim3((L + LC) / LC, L + 1, Nx), 256, 0, st>>>(F, Nx, L, Ny, Nz, normP, cosm, sinm, sint, dydz,
                                                                   alm);
}

}  // namespace kg
