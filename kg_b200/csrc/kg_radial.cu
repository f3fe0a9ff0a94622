// kg_radial.cu -- spherical-Bessel radial basis and the discrete radial
// transform of the all-shell Y_lm coefficients.
//
// generate_full_bessel_basis (tools/FFT_sph.f90:13-95): for l <= L and
// n = 1..Nk, k_ln = z_n(J_{l+1/2}) / r_max (the n-th positive zero of the
// spherical Bessel function j_l, over the outermost r of the evolution grid),
// and j_basis(l,n,i) = j_l(k_ln r_i) / sqrt(trapezium_1D(j_l(k_ln r)^2 r^2, dr))
// on the vertex radii r_i = xmin + (i-1) dx, i = 1..Nx.  The reference takes
// j_l and the zeros from GSL (gsl_sf_bessel_jl, gsl_sf_bessel_zero_Jnu); here
// they are computed on the host by published methods:
//   * j_l(x): for x > l the upward three-term recurrence
//     j_{k+1} = (2k+1)/x j_k - j_{k-1} from j_0 = sin x / x, j_1 = sin x / x^2 - cos x / x
//     (stable in that range); otherwise Miller's downward recurrence from an
//     order well above l and x, normalised by j_0 or j_1 (whichever is larger);
//   * zeros: those of j_0 are n pi; the zeros of J_nu and J_{nu+1} interlace,
//     so the n-th zero of j_{l+1} lies between the n-th and (n+1)-th zeros of
//     j_l, where bisection runs until the bracket stops shrinking.
//
// SphFT_discrete_radial (tools/FFT_sph.f90:213-244): a_nlm = trapezium_1D over
// the shells of flm(r_i, l, m) j_basis(l, n, i) r_i^2 (end weights 1/2, times dr),
// with flm the Y_lm projection on every shell.  The reference declares its
// j_basis dummy as (0:l_max, 0:Nk, r) while the basis is built as
// (0:l_max, Nk, r), so its loop over n = 0..Nk reads the array with the wrong
// shape; the contraction here is the intended one, n = 1..Nk of the built basis.
#include <cuda_runtime.h>
#include <cmath>
#include <vector>
#include "kg_device.cuh"
#include "kg_diag.h"

namespace kg {

double sph_jl(int l, double x) {
  if (x == 0.0) return l == 0 ? 1.0 : 0.0;
  const double ax = std::fabs(x);
  const double s = std::sin(ax), c = std::cos(ax);
  const double j0 = s / ax;
  const double j1 = s / (ax * ax) - c / ax;
  const double sg = (x < 0.0 && (l & 1)) ? -1.0 : 1.0;
  if (l == 0) return j0;
  if (l == 1 && ax > 1.0) return sg * j1;  // the closed form cancels for small x
  if (ax > (double)l) {
    double jm = j0, jc = j1;
    for (int k = 1; k < l; ++k) {
      const double jn = (2.0 * k + 1.0) / ax * jc - jm;
      jm = jc;
      jc = jn;
    }
    return sg * jc;
  }
  // Miller: start well above both l and x, recur down to order 0
  const int top = l + 20 + (int)std::sqrt(40.0 * (double)(l > (int)ax ? l : (int)ax + 1));
  double jp = 0.0, jc = 1.0e-30, keep = 0.0;
  for (int k = top; k >= 1; --k) {
    const double jm = (2.0 * k + 1.0) / ax * jc - jp;  // order k-1
    jp = jc;
    jc = jm;
    if (k - 1 == l) keep = jc;
    if (std::fabs(jc) > 1.0e250) {
      jc *= 1.0e-250;
      jp *= 1.0e-250;
      keep *= 1.0e-250;
    }
  }
  // jc = order 0, jp = order 1 (unnormalised)
  const double scale = (std::fabs(j0) >= std::fabs(j1)) ? j0 / jc : j1 / jp;
  return sg * keep * scale;
}

// z[l * Nk + (n - 1)] = n-th positive zero of j_l, l = 0..L, n = 1..Nk
void sph_jl_zeros(int L, int Nk, std::vector<double>& z) {
  const double pi = std::acos(-1.0);
  z.assign((size_t)(L + 1) * Nk, 0.0);
  std::vector<double> prev(Nk + L + 1), cur;
  for (int n = 1; n <= Nk + L; ++n) prev[n - 1] = n * pi;
  for (int n = 0; n < Nk; ++n) z[n] = prev[n];
  for (int l = 1; l <= L; ++l) {
    const int cnt = Nk + L - l;
    cur.assign(cnt, 0.0);
    for (int n = 0; n < cnt; ++n) {
      double lo = prev[n], hi = prev[n + 1];
      double flo = sph_jl(l, lo);
      for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        const double fm = sph_jl(l, mid);
        if (fm == 0.0) {
          lo = hi = mid;
          break;
        }
        if ((fm > 0.0) == (flo > 0.0)) {
          lo = mid;
          flo = fm;
        } else {
          hi = mid;
        }
      }
      cur[n] = 0.5 * (lo + hi);
    }
    for (int n = 0; n < Nk; ++n) z[(size_t)l * Nk + n] = cur[n];
    prev.swap(cur);
  }
}

// k_values[l * Nk + n-1], basis[(l * Nk + n-1) * Nx + i-1] (normalised j_basis)
void bessel_basis(int L, int Nk, int Nx, double xmin, double dx, double r_max, std::vector<double>& k_values,
                  std::vector<double>& basis) {
  std::vector<double> z;
  sph_jl_zeros(L, Nk, z);
  k_values.assign((size_t)(L + 1) * Nk, 0.0);
  basis.assign((size_t)(L + 1) * Nk * Nx, 0.0);
  std::vector<double> r(Nx), f(Nx);
  for (int i = 1; i <= Nx; ++i) r[i - 1] = xmin + (double)(i - 1) * dx;
  const double dr = std::fabs(r[1] - r[0]);
  for (int l = 0; l <= L; ++l)
    for (int n = 1; n <= Nk; ++n) {
      const double kv = z[(size_t)l * Nk + n - 1] / r_max;
      k_values[(size_t)l * Nk + n - 1] = kv;
      double* jb = basis.data() + ((size_t)l * Nk + n - 1) * Nx;
      for (int i = 0; i < Nx; ++i) jb[i] = sph_jl(l, kv * r[i]);
      for (int i = 0; i < Nx; ++i) f[i] = (jb[i] * jb[i]) * (r[i] * r[i]);
      // trapezium_1D_real (tools/integral.f90:176-195)
      double sum = 0.0;
      for (int i = 1; i < Nx - 1; ++i) sum += f[i];
      const double nrm = std::sqrt(dr * (0.5 * f[0] + sum + 0.5 * f[Nx - 1]));
      if (nrm > 0.0)
        for (int i = 0; i < Nx; ++i) jb[i] = jb[i] / nrm;
    }
}

// ft(n, l, m) for one (l, m) per block; threads over n.  jr[(l * Nx + i) * Nk + n]
// holds j_basis(l, n, i) r_i^2; flm[l + NL (mi + NM i)] the all-shell projection.
__global__ void radial_ft_kernel(const double2* __restrict__ flm, const double* __restrict__ jr, int L, int Nk,
                                 int Nx, double dr, double2* __restrict__ ft) {
  const int l = blockIdx.x, mi = blockIdx.y, m = mi - L;
  const int NL = L + 1, NM = 2 * L + 1;
  for (int n = threadIdx.x; n < Nk; n += blockDim.x) {
    double2 acc = c2(0.0, 0.0);
    if (m >= -l && m <= l) {
      const double* j = jr + (long long)l * Nx * Nk + n;
      auto term = [&](int i) {
        const double2 f = flm[l + (long long)NL * (mi + (long long)NM * i)];
        return rmul(j[(long long)i * Nk], f);
      };
      // trapezium_1D_complex (tools/integral.f90:197-217)
      acc = rmul(0.5, cadd(term(0), term(Nx - 1)));
      for (int i = 1; i < Nx - 1; ++i) acc = cadd(acc, term(i));
      acc = rmul(dr, acc);
    }
    ft[n + (long long)Nk * (l + (long long)NL * mi)] = acc;
  }
}

void launch_radial_ft(const double2* flm, const double* jr, int L, int Nk, int Nx, double dr, double2* ft,
                      cudaStream_t st) {
  radial_ft_kernel<<<dim3(L + 1, 2 * L + 1), 128, 0, st>>>(flm, jr, L, Nk, Nx, dr, ft);
}

}  // namespace kg
