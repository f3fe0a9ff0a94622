// kg_boundary.cu -- ghost-zone, pole-parity and outer-boundary fills on the
// device (MoL/lines_method_lib.f90:507-597) and the Fortran <-> device layout
// conversion.
//
// The reference applies, in order: boundary_xL (third-order extrapolation into
// the excision plane), boundary_xR (outflow copy or inflow hold), boundary_yL
// and boundary_yR (theta ghost rows copied from the interior rows at phi + pi,
// no sign change), boundary_zL and boundary_zR (duplicated phi planes).
//
// The stepper path runs this as two launches:
//   ghost_xy: every x-face point of the interior theta rows and every point of
//             the six theta ghost rows.  A theta ghost row takes the post-x
//             value of its source, which is computed on the fly from the
//             pre-boundary state, so no point read is written by the launch.
//   ghost_z:  the two duplicated phi planes, from planes Nz-1 and 1 after
//             ghost_xy (the reference's zL/zR run after the theta fill).
// `face` launches run one reference routine at a time (parity hook).
#include "kg_device.cuh"
#include "kg_internal.h"

namespace kg {

// value of u after boundary_xL / boundary_xR at (ii, jj, k)
__device__ __forceinline__ double2 xval(const Grid& g, const double2* u, const double2* up, int inflow,
                                        int ii, int jj, int k) {
  if (ii == 0)
    return cadd(csub(rmul(3.0, u[off3(g, 1, jj, k)]), rmul(3.0, u[off3(g, 2, jj, k)])), u[off3(g, 3, jj, k)]);
  if (ii == g.NI - 1) return inflow ? up[off3(g, ii, jj, k)] : u[off3(g, ii - 1, jj, k)];
  return u[off3(g, ii, jj, k)];
}

// source theta row of ghost row jj (0-based rows; rows 0..2 and NJ-3..NJ-1)
__device__ __forceinline__ int ghost_src_row(const Grid& g, int jj) {
  return (jj <= 2) ? (5 - jj) : (2 * g.NJ - 7 - jj);
}

__global__ void ghost_xy_kernel(Grid g, double2* u, const double2* up, int inflow, long long n_rows,
                                long long n_faces) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = n_rows + n_faces;
  if (t >= total) return;
  if (t < n_rows) {
    // ghost-row points: t = ii + NI*(r + 6*k), r in 0..5
    const int ii = (int)(t % g.NI);
    const long long rk = t / g.NI;
    const int r = (int)(rk % 6);
    const int k = (int)(rk / 6);
    const int jj = (r < 3) ? r : (g.NJ - 6 + r);
    const int js = ghost_src_row(g, jj);
    const int kt = ktarget(g, k);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double2* uv = u + v * g.fs;
      const double2* upv = up + v * g.fs;
      u[v * g.fs + off3(g, ii, jj, k)] = xval(g, uv, upv, inflow, ii, js, kt);
    }
  } else {
    // x-face points of interior rows: f = jr + (NJ-6)*(side + 2*k)
    const long long f = t - n_rows;
    const int nin = g.NJ - 6;
    const int jj = 3 + (int)(f % nin);
    const long long sk = f / nin;
    const int side = (int)(sk % 2);
    const int k = (int)(sk / 2);
    const int ii = side ? g.NI - 1 : 0;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double2* uv = u + v * g.fs;
      const double2* upv = up + v * g.fs;
      u[v * g.fs + off3(g, ii, jj, k)] = xval(g, uv, upv, inflow, ii, jj, k);
    }
  }
}

__global__ void ghost_z_kernel(Grid g, double2* u) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)g.NI * g.NJ;
  if (t >= 2 * n) return;
  const int side = (int)(t / n);
  const long long q = t % n;
  const int ii = (int)(q % g.NI), jj = (int)(q / g.NI);
  const int kd = side ? g.Nz : 0;
  const int ks = side ? 1 : g.Nz - 1;
#pragma unroll
  for (int v = 0; v < 5; ++v) u[v * g.fs + off3(g, ii, jj, kd)] = u[v * g.fs + off3(g, ii, jj, ks)];
}

void launch_ghost_fill(const Grid& g, double2* u, const double2* up, int inflow, cudaStream_t st) {
  const long long n_rows = 6LL * g.NK * g.NI;
  const long long n_faces = 2LL * (g.NJ - 6) * g.NK;
  const long long total = n_rows + n_faces;
  ghost_xy_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(g, u, up, inflow, n_rows, n_faces);
  const long long nz = 2LL * g.NI * g.NJ;
  ghost_z_kernel<<<(unsigned)((nz + 255) / 256), 256, 0, st>>>(g, u);
}

// ---- many solves at once (batched engine) -----------------------------------
__global__ void ghost_xy_batch_kernel(const GhostDesc* __restrict__ d) {
  const GhostDesc& D = d[blockIdx.y];
  const Grid& g = D.g;
  const long long n_rows = 6LL * g.NK * g.NI;
  const long long n_faces = 2LL * (g.NJ - 6) * g.NK;
  const long long total = n_rows + n_faces;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int ii, jj, k, si, sj, sk;
    if (t < n_rows) {
      ii = (int)(t % g.NI);
      const long long rk = t / g.NI;
      const int r = (int)(rk % 6);
      k = (int)(rk / 6);
      jj = (r < 3) ? r : (g.NJ - 6 + r);
      si = ii;
      sj = ghost_src_row(g, jj);
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
      D.u[v * g.fs + off3(g, ii, jj, k)] = xval(g, D.u + v * g.fs, D.up + v * g.fs, D.inflow, si, sj, sk);
  }
}

__global__ void ghost_z_batch_kernel(const GhostDesc* __restrict__ d) {
  const GhostDesc& D = d[blockIdx.y];
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

void launch_ghost_fill_batch(const GhostDesc* d_desc, int n, long long max_rows, long long max_faces,
                             long long max_zplanes, cudaStream_t st) {
  if (n <= 0) return;
  long long bx = (max_rows + max_faces + 255) / 256;
  if (bx > 1024) bx = 1024;
  if (bx < 1) bx = 1;
  ghost_xy_batch_kernel<<<dim3((unsigned)bx, n), 256, 0, st>>>(d_desc);
  long long bz = (max_zplanes + 255) / 256;
  if (bz > 1024) bz = 1024;
  if (bz < 1) bz = 1;
  ghost_z_batch_kernel<<<dim3((unsigned)bz, n), 256, 0, st>>>(d_desc);
}

// ---- one reference routine at a time ---------------------------------------
// face 0 = xL, 1 = xR, 2 = yL, 3 = yR, 4 = zL, 5 = zR
__global__ void face_kernel(Grid g, double2* u, const double2* up, int inflow, int face) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (face <= 1) {  // all (jj, k) of one x-face
    const long long n = (long long)g.NJ * g.NK;
    if (t >= n) return;
    const int jj = (int)(t % g.NJ), k = (int)(t / g.NJ);
    const int ii = face == 0 ? 0 : g.NI - 1;
    for (int v = 0; v < 5; ++v)
      u[v * g.fs + off3(g, ii, jj, k)] = xval(g, u + v * g.fs, up + v * g.fs, inflow, ii, jj, k);
  } else if (face <= 3) {  // three ghost rows of one pole, all (ii, k)
    const long long n = 3LL * g.NI * g.NK;
    if (t >= n) return;
    const int ii = (int)(t % g.NI);
    const long long rk = t / g.NI;
    const int r = (int)(rk % 3), k = (int)(rk / 3);
    const int jj = face == 2 ? r : g.NJ - 3 + r;
    const int js = ghost_src_row(g, jj), kt = ktarget(g, k);
    for (int v = 0; v < 5; ++v) u[v * g.fs + off3(g, ii, jj, k)] = u[v * g.fs + off3(g, ii, js, kt)];
  } else {  // one duplicated phi plane
    const long long n = (long long)g.NI * g.NJ;
    if (t >= n) return;
    const int ii = (int)(t % g.NI), jj = (int)(t / g.NI);
    const int kd = face == 4 ? 0 : g.Nz;
    const int ks = face == 4 ? g.Nz - 1 : 1;
    for (int v = 0; v < 5; ++v) u[v * g.fs + off3(g, ii, jj, kd)] = u[v * g.fs + off3(g, ii, jj, ks)];
  }
}

void launch_face(const Grid& g, double2* u, const double2* up, int inflow, int face, cudaStream_t st) {
  long long n = face <= 1 ? (long long)g.NJ * g.NK : face <= 3 ? 3LL * g.NI * g.NK : (long long)g.NI * g.NJ;
  face_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, u, up, inflow, face);
}

// ---- layout conversion -------------------------------------------------------
// aos: complex u(5, NI, NJ, planes k0..k1-1) (Fortran order, variable fastest)
__global__ void aos_to_soa_kernel(Grid g, const double2* __restrict__ aos, double2* __restrict__ soa, int k0,
                                  int k1) {
  const long long n = (long long)g.NI * g.NJ * (k1 - k0);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int ii = (int)(t % g.NI);
  const long long r = t / g.NI;
  const int jj = (int)(r % g.NJ), k = k0 + (int)(r / g.NJ);
  const long long o = off3(g, ii, jj, k);
#pragma unroll
  for (int v = 0; v < 5; ++v) soa[v * g.fs + o] = aos[5 * t + v];
}

__global__ void soa_to_aos_kernel(Grid g, const double2* __restrict__ soa, double2* __restrict__ aos, int k0,
                                  int k1) {
  const long long n = (long long)g.NI * g.NJ * (k1 - k0);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int ii = (int)(t % g.NI);
  const long long r = t / g.NI;
  const int jj = (int)(r % g.NJ), k = k0 + (int)(r / g.NJ);
  const long long o = off3(g, ii, jj, k);
#pragma unroll
  for (int v = 0; v < 5; ++v) aos[5 * t + v] = soa[v * g.fs + o];
}

void launch_aos_to_soa(const Grid& g, const double2* aos, double2* soa, int k0, int k1, cudaStream_t st) {
  const long long n = (long long)g.NI * g.NJ * (k1 - k0);
  if (n <= 0) return;
  aos_to_soa_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, aos, soa, k0, k1);
}

void launch_soa_to_aos(const Grid& g, const double2* soa, double2* aos, int k0, int k1, cudaStream_t st) {
  const long long n = (long long)g.NI * g.NJ * (k1 - k0);
  if (n <= 0) return;
  soa_to_aos_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, soa, aos, k0, k1);
}

}  // namespace kg
