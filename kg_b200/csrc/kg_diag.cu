// kg_diag.cu -- diagnostics of MoL/diagnostic_lib.f90 on the device:
// energy density, the trapezium-weighted mass integral, the ADM currents and
// detector fluxes, and the Y_lm projection at the detector radii.
//
// All reductions are deterministic: each block reduces its slice with warp
// shuffles (FP64) into one partial, and a single block adds the partials in
// a fixed order.  No atomics, so a result does not depend on scheduling.
#include "kg_device.cuh"
#include "kg_internal.h"
#include "kg_diag.h"

namespace kg {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return v;
}
// block-wide sum (blockDim.x multiple of 32, <= 1024); result valid in thread 0
__device__ double block_sum(double v) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  __syncthreads();
  return v;
}
__device__ double2 block_sum2(double2 v) {
  __shared__ double2 sh2[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum2(v);
  if (lane == 0) sh2[w] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  v = (threadIdx.x < nw) ? sh2[threadIdx.x] : make_double2(0.0, 0.0);
  if (w == 0) v = warp_sum2(v);
  __syncthreads();
  return v;
}

// density (diagnostic_lib.f90:277-289); the complex term 2 g^rphi |psi1| psi3
// makes the sum complex and rho keeps its real part.
__global__ void density_kernel(Grid g, Metric m, const double2* __restrict__ u, double mass2,
                               double* __restrict__ rho) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (ii >= g.NI || jj >= g.NJ || k >= g.NK) return;
  const long long p = off3(g, ii, jj, k);
  const int q = off2(g, ii, jj);
  const double2 u1 = u[p], u2 = u[g.fs + p], u3 = u[2 * g.fs + p], u4 = u[3 * g.fs + p], u5 = u[4 * g.fs + p];
  const double a5 = hypot(u5.x, u5.y), a2 = hypot(u2.x, u2.y), a3 = hypot(u3.x, u3.y);
  const double a4 = hypot(u4.x, u4.y), a1 = hypot(u1.x, u1.y);
  const double t1 = m.grr[q] * (a2 * a2);
  const double t2re = (2.0 * m.grp[q] * a2) * u4.x;
  const double t3 = m.gtt[q] * (a3 * a3);
  const double t4 = m.gpp[q] * (a4 * a4);
  const double t5 = mass2 * a1;
  double re = a5 + t1;
  re = re + t2re;
  re = re + t3;
  re = re + t4;
  re = re + t5;
  rho[p] = 0.5 * re;
}

void launch_density(const Grid& g, const Metric& m, const double2* u, double mass2, double* rho, cudaStream_t st) {
  dim3 b(64, 4, 1), gr((g.NI + 63) / 64, (g.NJ + 3) / 4, g.NK);
  density_kernel<<<gr, b, 0, st>>>(g, m, u, mass2, rho);
}

// trapezium over i in [0,Nx] (ii in [2, NI-3]), j in [0,Ny], k in [0,Nz] of
// rho*sqrtg, weights 1/2 on the first and last index of each direction
static const int MASS_THREADS = 256;
int mass_blocks(const Grid& g) { return 148 * 4; }  // one wave at 4 CTAs (64 registers) per SM

// Each warp takes whole (theta, phi) rows in turn and its lanes stride along r
// with eight independent loads of rho (and of sqrt(gamma)) in flight, so the
// loads are coalesced and no per-point index division is needed; the block
// count is fixed, so the partial sums (and the result) do not depend on the
// device.
__global__ void mass_partial_kernel(Grid g, const double* __restrict__ sqrtg, const double* __restrict__ rho,
                                    double* partials) {
  const int ni = g.NI - 4, nj = g.NJ - 4, nk = g.NK;
  const int rows = nj * nk;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double acc = 0.0;
  for (int row = blockIdx.x * nw + (threadIdx.x >> 5); row < rows; row += gridDim.x * nw) {
    const int b = row % nj, k = row / nj;
    const int jj = b + 2;
    double wjk = 1.0;
    if (b == 0 || b == nj - 1) wjk *= 0.5;
    if (k == 0 || k == nk - 1) wjk *= 0.5;
    const double* rr = rho + off3(g, 2, jj, k);
    const double* sr = sqrtg + off2(g, 2, jj);
    for (int a0 = lane; a0 < ni; a0 += 256) {
      double rv[8], sv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int a = a0 + 32 * u;
        rv[u] = a < ni ? __ldg(rr + a) : 0.0;
        sv[u] = a < ni ? __ldg(sr + a) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int a = a0 + 32 * u;
        const double w = (a == 0 || a == ni - 1) ? 0.5 * wjk : wjk;
        acc += w * (rv[u] * sv[u]);
      }
    }
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void sum_partials_kernel(const double* partials, int n, double scale, double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) *out = acc * scale;
}

void launch_mass(const Grid& g, const Metric& m, const double* rho, double dxdydz, double* partials, double* out,
                 cudaStream_t st) {
  const int nb = mass_blocks(g);
  mass_partial_kernel<<<nb, MASS_THREADS, 0, st>>>(g, m.sqrtg, rho, partials);
  sum_partials_kernel<<<1, 1024, 0, st>>>(partials, nb, dxdydz, out);
}

// ---- detector shells ---------------------------------------------------------
// Vertex values of one field on the detector shells by the reference's
// trilinear interpolation (tools/FFT_sph.f90:525-651).  The index search and
// the weights depend only on the vertex index in each direction; they are
// computed once on the host with the reference's arithmetic and passed in.
//   src: 0 = phi, 1..3 = j_i * sqrtg (currents_ADM, diagnostic_lib.f90:219-229)
template <int SRC>
__device__ __forceinline__ double2 shell_src(const Grid& g, const Metric& m, const double2* u, int ii, int jj,
                                             int k) {
  const long long p = off3(g, ii, jj, k);
  if (SRC == 0) return u[p];
  const int q = off2(g, ii, jj);
  const double2 u2 = u[g.fs + p], u3 = u[2 * g.fs + p], u4 = u[3 * g.fs + p], u5 = u[4 * g.fs + p];
  const double2 n5 = cneg(u5);
  double2 a;
  if (SRC == 1) a = cadd(rmul(m.grr[q], u2), rmul(m.grp[q], u4));
  else if (SRC == 2) a = rmul(m.gtt[q], u3);
  else a = cadd(rmul(m.grp[q], u2), rmul(m.gpp[q], u4));
  const double2 j = c2(n5.x * a.x - n5.y * a.y, n5.x * a.y + n5.y * a.x);
  const double sg = m.sqrtg[q];
  return c2(j.x * sg, j.y * sg);
}

template <int SRC>
__global__ void shell_interp_kernel(Grid g, Metric m, const double2* __restrict__ u, ShellInterp si, int Ny, int Nz,
                                    double2* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int d = blockIdx.y;
  if (t >= Ny * Nz || !si.active[d]) return;
  const int jv = t % Ny, kv = t / Ny;
  const int ir = si.i_r[d], ith = si.i_th[jv], iph = si.i_ph[kv];
  double2* o = out + ((long long)d * 4 + SRC) * Ny * Nz + t;
  const int fl = si.th_flag[jv];
  if (fl == 1) { *o = shell_src<SRC>(g, m, u, ir, 0, iph); return; }
  if (fl == 2) { *o = shell_src<SRC>(g, m, u, ir, g.NJ - 1, iph); return; }
  const int ip1 = iph + 1;
  const double wr = si.w_r[d], wt = si.w_th[jv], wp = si.w_ph[kv];
  const double2 f000 = shell_src<SRC>(g, m, u, ir, ith, iph), f001 = shell_src<SRC>(g, m, u, ir, ith, ip1);
  const double2 f010 = shell_src<SRC>(g, m, u, ir, ith + 1, iph), f011 = shell_src<SRC>(g, m, u, ir, ith + 1, ip1);
  const double2 f100 = shell_src<SRC>(g, m, u, ir + 1, ith, iph), f101 = shell_src<SRC>(g, m, u, ir + 1, ith, ip1);
  const double2 f110 = shell_src<SRC>(g, m, u, ir + 1, ith + 1, iph),
                f111 = shell_src<SRC>(g, m, u, ir + 1, ith + 1, ip1);
  const double2 f00 = cadd(rmul(1.0 - wp, f000), rmul(wp, f001));
  const double2 f01 = cadd(rmul(1.0 - wp, f010), rmul(wp, f011));
  const double2 f10 = cadd(rmul(1.0 - wp, f100), rmul(wp, f101));
  const double2 f11 = cadd(rmul(1.0 - wp, f110), rmul(wp, f111));
  const double2 f0 = cadd(rmul(1.0 - wt, f00), rmul(wt, f01));
  const double2 f1 = cadd(rmul(1.0 - wt, f10), rmul(wt, f11));
  *o = cadd(rmul(1.0 - wr, f0), rmul(wr, f1));
}

void launch_shell_interp(const Grid& g, const Metric& m, const double2* u, const ShellInterp& si, int n_det, int Ny,
                         int Nz, int which_mask, double2* out, cudaStream_t st) {
  dim3 gr((Ny * Nz + 255) / 256, n_det);
  if (which_mask & 1) shell_interp_kernel<0><<<gr, 256, 0, st>>>(g, m, u, si, Ny, Nz, out);
  if (which_mask & 2) shell_interp_kernel<1><<<gr, 256, 0, st>>>(g, m, u, si, Ny, Nz, out);
  if (which_mask & 4) shell_interp_kernel<2><<<gr, 256, 0, st>>>(g, m, u, si, Ny, Nz, out);
  if (which_mask & 8) shell_interp_kernel<3><<<gr, 256, 0, st>>>(g, m, u, si, Ny, Nz, out);
}

// trapezium_2D_complex selector weight (tools/integral.f90:330-362)
__device__ __forceinline__ double trap_w(int jv, int kv, int Ny, int Nz) {
  const int sel = ((jv == 0 || jv == Ny - 1) ? 1 : 0) + 2 * ((kv == 0 || kv == Nz - 1) ? 1 : 0);
  return sel == 0 ? 1.0 : (sel == 3 ? 0.25 : 0.5);
}

// momentum(c, d) = Re trapezium_2D(shell of j_c sqrtg): one block per (c, d)
__global__ void flux_kernel(const double2* __restrict__ shells, const int* active, int Ny, int Nz, double dydz,
                            double* out) {
  const int c = blockIdx.x, d = blockIdx.y;
  if (!active[d]) return;
  const double2* f = shells + ((long long)d * 4 + 1 + c) * Ny * Nz;
  double2 acc = c2(0.0, 0.0);
  for (int t = threadIdx.x; t < Ny * Nz; t += blockDim.x) {
    const int jv = t % Ny, kv = t / Ny;
    acc = cadd(acc, rmul(trap_w(jv, kv, Ny, Nz), f[t]));
  }
  acc = block_sum2(acc);
  if (threadIdx.x == 0) out[c + 3 * d] = dydz * acc.x;
}

void launch_flux(const double2* shells, const int* active, int n_det, int Ny, int Nz, double dydz, double* out,
                 cudaStream_t st) {
  flux_kernel<<<dim3(3, n_det), 256, 0, st>>>(shells, active, Ny, Nz, dydz, out);
}

// project_sh (tools/FFT_sph.f90:247-279): a_lm = dy dz sum_jk w_jk f conj(Y_lm) sin(theta_j).
// Y_lm = (norm P_lm)(theta_j) (cos m phi_k, sin m phi_k); Y_l,-m = (-1)^m conj(Y_lm).
// One block per (l, m, detector).
__global__ void project_kernel(const double2* __restrict__ shells, const int* active, int L, int Ny, int Nz,
                               const double* __restrict__ normP, const double* __restrict__ cosm,
                               const double* __restrict__ sinm, const double* __restrict__ sint, double dydz,
                               double2* alm) {
  const int l = blockIdx.x, mi = blockIdx.y, d = blockIdx.z;
  const int m = mi - L;
  if (!active[d] || (m < -l) || (m > l)) return;
  const int am = m < 0 ? -m : m;
  const double sgn = (am & 1) ? -1.0 : 1.0;
  const double* P = normP + ((long long)l * (L + 1) + am) * Ny;
  const double* cm = cosm + (long long)am * Nz;
  const double* sm = sinm + (long long)am * Nz;
  const double2* f = shells + ((long long)d * 4) * Ny * Nz;
  double2 acc = c2(0.0, 0.0);
  for (int t = threadIdx.x; t < Ny * Nz; t += blockDim.x) {
    const int jv = t % Ny, kv = t / Ny;
    const double np = P[jv];
    double2 y = c2(np * cm[kv], np * sm[kv]);
    if (m < 0) y = c2(sgn * y.x, sgn * -y.y);
    const double2 a = f[t];
    const double2 cy = c2(y.x, -y.y);
    const double2 fy = c2(a.x * cy.x - a.y * cy.y, a.x * cy.y + a.y * cy.x);
    const double s = sint[jv];
    const double2 fun = c2(fy.x * s, fy.y * s);
    acc = cadd(acc, rmul(trap_w(jv, kv, Ny, Nz), fun));
  }
  acc = block_sum2(acc);
  if (threadIdx.x == 0) alm[(long long)l + (L + 1) * ((long long)mi + (2 * L + 1) * d)] = rmul(dydz, acc);
}

void launch_project(const double2* shells, const int* active, int n_det, int L, int Ny, int Nz, const double* normP,
                    const double* cosm, const double* sinm, const double* sint, double dydz, double2* alm,
                    cudaStream_t st) {
  project_kernel<<<dim3(L + 1, 2 * L + 1, n_det), 256, 0, st>>>(shells, active, L, Ny, Nz, normP, cosm, sinm, sint,
                                                                 dydz, alm);
}

}  // namespace kg
