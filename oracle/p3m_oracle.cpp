/*
 * TEST INFRASTRUCTURE ONLY -- the checker, never the product.
 *
 * FP64 CPU restatement of the reference (ESPResSo 4.3-dev) CPU P3M and
 * short-range force path, written from the reference's algorithm, plus an
 * independent direct Ewald sum.  Each function cites the reference
 * file:line it follows (paths relative to the ESPResSo source tree).
 * Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg (ctypes).  OpenMP is used only to make the CPU baseline use
 * all host cores; results do not depend on the thread count except for
 * FP64 summation order in reductions.
 */
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numbers>
#include <set>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

using cd = std::complex<double>;

namespace {

constexpr double PI = std::numbers::pi;

/* ---------------------------------------------------------------------- */
/* Math.                                                                   */
/* ---------------------------------------------------------------------- */

/* Cardinal B-spline weights of order P at the P mesh points around a
 * particle, for x = distance to the nearest mesh point in [-0.5, 0.5].
 * Computed with the Cox-de Boor recursion M_{n+1}(u+k) = ((u+k) M_n(u+k)
 * + (n+1-u-k) M_n(u+k-1)) / n, u = x + 1/2; weight i is M_P(u + P-1-i).
 * Same values as the tabulated polynomials of utils/math/bspline.hpp:30-177
 * (Hockney & Eastwood 5-189), up to FP64 rounding. */
void bspline_weights(int P, double x, double *w) {
  double c[8];
  double const u = x + 0.5;
  c[0] = 1.0;
  for (int n = 1; n < P; ++n) {
    double const inv_n = 1.0 / n;
    c[n] = 0.0;
    for (int k = n; k >= 0; --k) {
      double const left = (k > 0) ? c[k - 1] : 0.0;
      c[k] = ((u + k) * c[k] + (n + 1 - u - k) * left) * inv_n;
    }
  }
  for (int i = 0; i < P; ++i)
    w[i] = c[P - 1 - i];
}

/* exp(d^2) erfc(d) by Abramowitz & Stegun 7.1.26 (five-term rational
 * approximation, |error| <= 1.5e-7), as used by the reference real-space
 * kernel (utils/math/AS_erfc_part.hpp:29-40, config.hpp:60-61). */
double as_erfc_part(double d) {
  double const a1 = 0.254829592, a2 = -0.284496736, a3 = 1.421413741,
               a4 = -1.453152027, a5 = 1.061405429, p = 0.3275911;
  double const t = 1.0 / (1.0 + p * d);
  return t * (a1 + t * (a2 + t * (a3 + t * (a4 + t * a5))));
}

/* sin(pi x)/(pi x), with the 8th-order Taylor series for |x| <= 0.1
 * (p3m/math.hpp:53-81). */
double sinc(double x) {
  double const pix = PI * x;
  if (std::fabs(x) > 0.1)
    return std::sin(pix) / pix;
  double const p2 = pix * pix;
  double const c2 = -1.0 / 6.0, c4 = 1.0 / 120.0, c6 = -1.0 / 5040.0,
               c8 = 1.0 / 362880.0;
  return 1.0 + p2 * (c2 + p2 * (c4 + p2 * (c6 + p2 * c8)));
}

/* Closed form of sum_m sinc^(2P)(n/M + m) as an even trigonometric
 * polynomial in c = cos^2(pi n / M) (Hockney & Eastwood eq. 7-66;
 * p3m/math.hpp:92-149). */
double cotangent_sum(int cao, int n, double mesh_i) {
  double const th = static_cast<double>(n) * mesh_i * PI;
  double const c = std::cos(th) * std::cos(th);
  switch (cao) {
  case 1:
    return 1.0;
  case 2:
    return (1. + c * 2.) / 3.;
  case 3:
    return (2. + c * (11. + c * 2.)) / 15.;
  case 4:
    return (17. + c * (180. + c * (114. + c * 4.))) / 315.;
  case 5:
    return (62. + c * (1072. + c * (1452. + c * (247. + c * 2.)))) / 2835.;
  case 6:
    return (1382. +
            c * (35396. + c * (83021. + c * (34096. + c * (2026. + c * 4.))))) /
           155925.;
  default:
    return (21844. +
            c * (776661. +
                 c * (2801040. +
                      c * (2123860. + c * (349500. + c * (8166. + c * 4.)))))) /
           6081075.;
  }
}

/* ---------------------------------------------------------------------- */
/* FP64 mixed-radix complex FFT (Cooley-Tukey, recursive decimation in     */
/* time; radix 4, 2 and a generic O(p^2) butterfly for other primes).      */
/* Unnormalised; sign -1 = forward (exp(-i k x)), +1 = backward, the       */
/* FFTW_FORWARD / FFTW_BACKWARD conventions of fft/fft.cpp:682-696.        */
/* ---------------------------------------------------------------------- */
struct FFTPlan {
  int n = 0, sign = -1;
  std::vector<int> factors; // pairs (p, m)
  std::vector<cd> tw;
  void init(int n_, int sign_) {
    n = n_;
    sign = sign_;
    tw.resize(n);
    for (int i = 0; i < n; ++i)
      tw[i] = std::polar(1.0, sign * 2.0 * PI * i / n);
    factors.clear();
    int m = n, p = 4;
    double const floor_sqrt = std::floor(std::sqrt(static_cast<double>(n)));
    do {
      while (m % p) {
        switch (p) {
        case 4:
          p = 2;
          break;
        case 2:
          p = 3;
          break;
        default:
          p += 2;
          break;
        }
        if (p > floor_sqrt)
          p = m;
      }
      m /= p;
      factors.push_back(p);
      factors.push_back(m);
    } while (m > 1);
  }

  void work(cd *out, const cd *in, std::size_t fstride, const int *fac,
            std::vector<cd> &scratch) const {
    int const p = fac[0], m = fac[1];
    cd *const out_beg = out;
    cd *const out_end = out + p * m;
    if (m == 1) {
      do {
        *out = *in;
        in += fstride;
      } while (++out != out_end);
    } else {
      do {
        work(out, in, fstride * p, fac + 2, scratch);
        in += fstride;
        out += m;
      } while (out != out_end);
    }
    out = out_beg;
    if (p == 2) {
      for (int u = 0; u < m; ++u) {
        cd const t = out[u + m] * tw[u * fstride];
        out[u + m] = out[u] - t;
        out[u] += t;
      }
    } else if (p == 4) {
      for (int u = 0; u < m; ++u) {
        cd const a0 = out[u];
        cd const a1 = out[u + m] * tw[u * fstride];
        cd const a2 = out[u + 2 * m] * tw[2 * u * fstride];
        cd const a3 = out[u + 3 * m] * tw[3 * u * fstride];
        cd const s0 = a0 + a2, s1 = a0 - a2, s2 = a1 + a3, s3 = a1 - a3;
        // multiply s3 by sign*i
        cd const s3i = (sign < 0) ? cd(s3.imag(), -s3.real())
                                  : cd(-s3.imag(), s3.real());
        out[u] = s0 + s2;
        out[u + 2 * m] = s0 - s2;
        out[u + m] = s1 + s3i;
        out[u + 3 * m] = s1 - s3i;
      }
    } else {
      scratch.resize(p);
      for (int u = 0; u < m; ++u) {
        for (int q1 = 0; q1 < p; ++q1)
          scratch[q1] = out[u + q1 * m];
        for (int q1 = 0; q1 < p; ++q1) {
          std::size_t const k = u + q1 * m;
          cd acc = scratch[0];
          std::size_t twidx = 0;
          for (int q = 1; q < p; ++q) {
            twidx += fstride * k;
            twidx %= n;
            acc += scratch[q] * tw[twidx];
          }
          out[k] = acc;
        }
      }
    }
  }
  void exec(cd *out, const cd *in) const {
    std::vector<cd> scratch;
    work(out, in, 1, factors.data(), scratch);
  }
};

/* In-place 3D c2c transform of a row-major [M0][M1][M2] mesh. */
void fft3d(std::vector<cd> &a, const int *M, int sign) {
  for (int axis = 2; axis >= 0; --axis) {
    int const n = M[axis];
    FFTPlan plan;
    plan.init(n, sign);
    std::size_t const stride =
        (axis == 2) ? 1 : (axis == 1 ? M[2] : std::size_t(M[1]) * M[2]);
    long const nlines = static_cast<long>(a.size() / n);
#pragma omp parallel
    {
      std::vector<cd> in(n), out(n);
#pragma omp for schedule(static)
      for (long l = 0; l < nlines; ++l) {
        // line l: decompose into base offset
        std::size_t base;
        if (axis == 2) {
          base = std::size_t(l) * n;
        } else if (axis == 1) {
          std::size_t const x = l / M[2], z = l % M[2];
          base = x * std::size_t(M[1]) * M[2] + z;
        } else {
          base = std::size_t(l);
        }
        for (int i = 0; i < n; ++i)
          in[i] = a[base + i * stride];
        plan.exec(out.data(), in.data());
        for (int i = 0; i < n; ++i)
          a[base + i * stride] = out[i];
      }
    }
  }
}

/* Mesh shift for k-vectors: (0..M/2, -M/2+1..-1) with entry M/2 equal to
 * -M/2 (or 0 when zero_mid), p3m/common.hpp:248-264. */
std::vector<int> meshift(int M, bool zero_mid) {
  std::vector<int> r(M, 0);
  for (int j = 1; j <= M / 2; ++j) {
    r[j] = j;
    r[M - j] = -j;
  }
  if (zero_mid)
    r[M / 2] = 0;
  return r;
}

/* Fold into [0, L) by repeated shifts (algorithm/periodic_fold.hpp:72-89). */
double fold(double x, double L) {
  while (x < 0)
    x += L;
  while (x >= L)
    x -= L;
  return x;
}

struct Geometry {
  double a[3], ai[3], cao_cut[3], ld_pos[3], V;
  int ld_ind[3];
  double pos_shift;
  Geometry(const oracle_p3m_params &p) {
    V = p.box[0] * p.box[1] * p.box[2];
    for (int d = 0; d < 3; ++d) {
      // recalc_a_ai_cao_cut, p3m/common.hpp:156-160
      ai[d] = p.mesh[d] / p.box[d];
      a[d] = 1.0 / ai[d];
      cao_cut[d] = (static_cast<double>(p.cao) / 2.0) * a[d];
      // calc_local_ca_mesh on a single rank, p3m/common.cpp:34-106
      double const outer_ld = 0.0 - (cao_cut[d] + p.skin);
      double const outer_ld_grid = outer_ld * ai[d] - p.mesh_off[d];
      ld_ind[d] = static_cast<int>(std::ceil(outer_ld_grid));
      // recalc_ld_pos, common.hpp:204-209
      ld_pos[d] = (ld_ind[d] + p.mesh_off[d]) * a[d];
    }
    // interpolation.hpp:142
    pos_shift = std::floor((p.cao - 1) / 2.0) - (p.cao % 2) / 2.0;
  }
  /* interpolation.hpp:138-178: returns the global corner index and the
   * three weight vectors. */
  void weights(const oracle_p3m_params &p, const double *x, int *corner,
               double *wx, double *wy, double *wz) const {
    double *w[3] = {wx, wy, wz};
    for (int d = 0; d < 3; ++d) {
      double const xf = fold(x[d], p.box[d]);
      double const pos = ((xf - ld_pos[d]) * ai[d]) - pos_shift;
      int const nmp = static_cast<int>(pos);
      double const dist = (pos - nmp) - 0.5;
      int g = (ld_ind[d] + nmp) % p.mesh[d];
      if (g < 0)
        g += p.mesh[d];
      corner[d] = g;
      bspline_weights(p.cao, dist, w[d]);
    }
  }
};

/* Optimal influence function for m = 0 aliasing (P3M_BRILLOUIN = 0):
 * G_opt<S,0> of p3m/influence_function.hpp:53-94 and the grid map of
 * :121-150 (zero where every index is a multiple of M/2).  With only the
 * m = 0 term the S = 0 (energy) and S = 1 (force) functions coincide. */
double g_opt_m0(const oracle_p3m_params &p, int nx, int ny, int nz,
                const std::vector<int> *sh) {
  int const idx[3] = {nx, ny, nz};
  bool all_half = true;
  for (int d = 0; d < 3; ++d)
    if (idx[d] % (p.mesh[d] / 2) != 0)
      all_half = false;
  if (all_half)
    return 0.0;
  double k[3], fnm[3];
  double const wavevector_i[3] = {
      1.0 / ((2.0 * PI) / (p.box[0] / p.mesh[0])),
      1.0 / ((2.0 * PI) / (p.box[1] / p.mesh[1])),
      1.0 / ((2.0 * PI) / (p.box[2] / p.mesh[2]))};
  for (int d = 0; d < 3; ++d) {
    k[d] = sh[d][idx[d]] * ((2.0 * PI) / p.box[d]);
    fnm[d] = sinc(k[d] * wavevector_i[d]);
  }
  double const k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  if (k2 == 0.0)
    return 0.0;
  double const U2 = std::pow(fnm[0] * fnm[1] * fnm[2], 2 * p.cao);
  double const exponent = (1.0 / (2.0 * p.alpha)) * (1.0 / (2.0 * p.alpha)) * k2;
  double numerator = 0.0;
  if (exponent < 30.0)
    numerator = U2 * (std::exp(-exponent) * (4.0 * PI / k2));
  return numerator / (U2 * U2);
}

} // namespace

extern "C" {

double oracle_bspline(int order, int i, double x) {
  double w[8];
  bspline_weights(order, x, w);
  return w[i];
}
double oracle_as_erfc_part(double d) { return as_erfc_part(d); }
double oracle_sinc(double x) { return sinc(x); }
double oracle_cotangent_sum(int cao, int n, double mesh_i) {
  return cotangent_sum(cao, n, mesh_i);
}

int oracle_influence_function(const oracle_p3m_params *pp, double *g_out) {
  auto const &p = *pp;
  std::vector<int> sh[3] = {meshift(p.mesh[0], false),
                            meshift(p.mesh[1], false),
                            meshift(p.mesh[2], false)};
  for (int x = 0; x < p.mesh[0]; ++x)
    for (int y = 0; y < p.mesh[1]; ++y)
      for (int z = 0; z < p.mesh[2]; ++z)
        g_out[(std::size_t(x) * p.mesh[1] + y) * p.mesh[2] + z] =
            g_opt_m0(p, x, y, z, sh);
  return 0;
}

/* k-space forces, energy and pressure tensor: p3m.cpp:283-373 (assignment
 * and force interpolation), 394-449 (pressure), 452-592 (long_range_kernel:
 * ik-differentiation, backward FFTs, dipole correction, energy with self,
 * net-charge and dipole terms). */
int oracle_p3m_kspace(const oracle_p3m_params *pp, long n, const double *pos,
                      const double *q, double *f, double *energy,
                      double *virial9, double *rho_out) {
  auto const &p = *pp;
  if (p.cao < 1 || p.cao > 7)
    return 1;
  Geometry const geo(p);
  int const M0 = p.mesh[0], M1 = p.mesh[1], M2 = p.mesh[2];
  std::size_t const msize = std::size_t(M0) * M1 * M2;
  int const cao = p.cao;

  // charge counts, p3m.cpp:98-115
  double sum_q2 = 0.0, sum_q = 0.0;
  for (long i = 0; i < n; ++i) {
    if (q[i] != 0.0) {
      sum_q2 += q[i] * q[i];
      sum_q += q[i];
    }
  }
  double const square_sum_q = sum_q * sum_q;

  // charge assignment: p3m_interpolate order x, y, z with value w*q,
  // w = (wx*wy)*wz (interpolation.hpp:191-208, p3m.cpp:283-291)
  std::vector<double> rho(msize, 0.0);
  std::vector<int> corners(3 * n);
  std::vector<double> wts(3 * 7 * n);
  for (long i = 0; i < n; ++i) {
    double *wx = &wts[21 * i], *wy = wx + 7, *wz = wx + 14;
    geo.weights(p, &pos[3 * i], &corners[3 * i], wx, wy, wz);
    if (q[i] == 0.0)
      continue;
    int const *c = &corners[3 * i];
    for (int i0 = 0; i0 < cao; ++i0) {
      int const gx = (c[0] + i0) % M0;
      double const t0 = wx[i0];
      for (int i1 = 0; i1 < cao; ++i1) {
        int const gy = (c[1] + i1) % M1;
        double const t1 = t0 * wy[i1];
        std::size_t const row = (std::size_t(gx) * M1 + gy) * M2;
        for (int i2 = 0; i2 < cao; ++i2) {
          int const gz = (c[2] + i2) % M2;
          rho[row + gz] += (t1 * wz[i2]) * q[i];
        }
      }
    }
  }
  if (rho_out)
    std::memcpy(rho_out, rho.data(), msize * sizeof(double));

  std::vector<cd> rhat(msize);
  for (std::size_t i = 0; i < msize; ++i)
    rhat[i] = cd(rho[i], 0.0);
  fft3d(rhat, p.mesh, -1);

  std::vector<int> sh[3] = {meshift(M0, false), meshift(M1, false),
                            meshift(M2, false)};
  std::vector<int> dop[3] = {meshift(M0, true), meshift(M1, true),
                             meshift(M2, true)};
  std::vector<double> g(msize);
#pragma omp parallel for schedule(static)
  for (int x = 0; x < M0; ++x)
    for (int y = 0; y < M1; ++y)
      for (int z = 0; z < M2; ++z)
        g[(std::size_t(x) * M1 + y) * M2 + z] = g_opt_m0(p, x, y, z, sh);

  // dipole moment of the unfolded positions (p3m.cpp:376-386)
  double dip[3] = {0, 0, 0};
  bool const metallic = (p.epsilon == 0.0);
  if (!metallic) {
    for (long i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d)
        dip[d] += q[i] * pos[3 * i + d];
  }
  double const V = geo.V;
  double const pref_dip = 4.0 * PI / V / (2.0 * p.epsilon + 1.0);

  if (energy) {
    double node_energy = 0.0;
    for (std::size_t i = 0; i < msize; ++i)
      node_energy += g[i] * (rhat[i].real() * rhat[i].real() +
                             rhat[i].imag() * rhat[i].imag());
    node_energy /= 2.0 * V;
    double e = node_energy;
    e -= sum_q2 * p.alpha * (1.0 / std::sqrt(PI));
    e -= square_sum_q * PI / (2.0 * V * p.alpha * p.alpha);
    if (!metallic)
      e += pref_dip * (dip[0] * dip[0] + dip[1] * dip[1] + dip[2] * dip[2]);
    *energy = e * p.prefactor;
  }

  if (virial9) {
    double t[9] = {0};
    double diagonal = 0.0;
    double const hai2 = (1.0 / 2.0 / p.alpha) * (1.0 / 2.0 / p.alpha);
    double const wv[3] = {2.0 * PI / p.box[0], 2.0 * PI / p.box[1],
                          2.0 * PI / p.box[2]};
    for (int x = 0; x < M0; ++x)
      for (int y = 0; y < M1; ++y)
        for (int z = 0; z < M2; ++z) {
          std::size_t const i = (std::size_t(x) * M1 + y) * M2 + z;
          double const kx = dop[0][x] * wv[0];
          double const ky = dop[1][y] * wv[1];
          double const kz = dop[2][z] * wv[2];
          double const nsq = kx * kx + ky * ky + kz * kz;
          if (nsq != 0.0) {
            double const ek = g[i] * (rhat[i].real() * rhat[i].real() +
                                      rhat[i].imag() * rhat[i].imag());
            double const vterm = -2.0 * (1.0 / nsq + hai2);
            double const pr = ek * vterm;
            t[0] += pr * kx * kx;
            t[1] += pr * kx * ky;
            t[2] += pr * kx * kz;
            t[4] += pr * ky * ky;
            t[5] += pr * ky * kz;
            t[8] += pr * kz * kz;
            diagonal += ek;
          }
        }
    t[0] += diagonal;
    t[4] += diagonal;
    t[8] += diagonal;
    t[3] = t[1];
    t[6] = t[2];
    t[7] = t[5];
    for (int k = 0; k < 9; ++k)
      virial9[k] = t[k] * p.prefactor / (2.0 * V);
  }

  if (f) {
    double const wv[3] = {2.0 * PI / p.box[0], 2.0 * PI / p.box[1],
                          2.0 * PI / p.box[2]};
    std::vector<double> field[3];
    for (int d = 0; d < 3; ++d) {
      std::vector<cd> e(msize);
#pragma omp parallel for schedule(static)
      for (int x = 0; x < M0; ++x)
        for (int y = 0; y < M1; ++y)
          for (int z = 0; z < M2; ++z) {
            std::size_t const i = (std::size_t(x) * M1 + y) * M2 + z;
            int const nd = (d == 0) ? dop[0][x] : (d == 1 ? dop[1][y] : dop[2][z]);
            double const k = static_cast<double>(nd) * wv[d];
            cd const phi = g[i] * rhat[i];
            e[i] = cd(-k * phi.imag(), k * phi.real());
          }
      fft3d(e, p.mesh, +1);
      field[d].resize(msize);
      for (std::size_t i = 0; i < msize; ++i)
        field[d][i] = e[i].real();
    }
    double const force_prefac = p.prefactor / V;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
      if (q[i] == 0.0)
        continue;
      double const *wx = &wts[21 * i], *wy = wx + 7, *wz = wx + 14;
      int const *c = &corners[3 * i];
      double fr[3] = {0, 0, 0};
      for (int i0 = 0; i0 < cao; ++i0) {
        int const gx = (c[0] + i0) % M0;
        double const t0 = wx[i0];
        for (int i1 = 0; i1 < cao; ++i1) {
          int const gy = (c[1] + i1) % M1;
          double const t1 = t0 * wy[i1];
          std::size_t const row = (std::size_t(gx) * M1 + gy) * M2;
          for (int i2 = 0; i2 < cao; ++i2) {
            std::size_t const ind = row + (c[2] + i2) % M2;
            double const w = t1 * wz[i2];
            fr[0] += w * field[0][ind];
            fr[1] += w * field[1][ind];
            fr[2] += w * field[2][ind];
          }
        }
      }
      double const pr = q[i] * force_prefac;
      for (int d = 0; d < 3; ++d)
        f[3 * i + d] -= pr * fr[d];
      if (!metallic) {
        for (int d = 0; d < 3; ++d)
          f[3 * i + d] -= q[i] * (p.prefactor * pref_dip * dip[d]);
      }
    }
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Cell system restatement.                                               */
/* ---------------------------------------------------------------------- */

/* RegularDecomposition::create_cell_grid on one rank (node grid 1x1x1):
 * RegularDecomposition.cpp:289-385 with max_num_cells = 32768
 * (RegularDecomposition.hpp:238). */
int oracle_cell_grid(const double *box, double range, int *cell_grid,
                     double *cell_size) {
  int const max_num_cells = 32768;
  int const min_num_cells = 8; // 2 per direction on one rank, :277-287
  double cell_range[3] = {range, range, range};
  if (range <= 0.0) {
    int const cpd = static_cast<int>(std::ceil(std::cbrt(double(min_num_cells))));
    for (int i = 0; i < 3; ++i)
      cell_grid[i] = cpd;
  } else {
    double const volume = box[0] * box[1] * box[2];
    double const scale = std::cbrt(max_num_cells / volume);
    for (int i = 0; i < 3; ++i) {
      cell_grid[i] = static_cast<int>(std::ceil(box[i] * scale));
      cell_range[i] = box[i] / static_cast<double>(cell_grid[i]);
      if (cell_range[i] < range) {
        cell_grid[i] = static_cast<int>(std::floor(box[i] / range));
        if (cell_grid[i] < 1)
          return 2; // interaction range larger than the box
        cell_range[i] = box[i] / static_cast<double>(cell_grid[i]);
      }
    }
    for (;;) {
      long const nc = long(cell_grid[0]) * cell_grid[1] * cell_grid[2];
      if (nc <= max_num_cells)
        break;
      int min_ind = 0;
      double min_size = cell_range[0];
      for (int i = 1; i < 3; ++i) {
        if (cell_grid[i] > 1 && cell_range[i] < min_size) {
          min_ind = i;
          min_size = cell_range[i];
        }
      }
      cell_grid[min_ind]--;
      cell_range[min_ind] = box[min_ind] / cell_grid[min_ind];
    }
    if (long(cell_grid[0]) * cell_grid[1] * cell_grid[2] < min_num_cells)
      return 3; // number of cells smaller than the minimum
  }
  for (int i = 0; i < 3; ++i)
    cell_size[i] = box[i] / static_cast<double>(cell_grid[i]);
  return 0;
}

/* position_to_cell_index (RegularDecomposition.cpp:51-80) for a periodic
 * box on one rank, linear index over the ghost grid in column-major order
 * (utils/index.hpp:43-53). */
int oracle_cell_index(const double *box, double range, long n,
                      const double *pos, int *cell_out) {
  int cg[3];
  double cs[3];
  int const rc = oracle_cell_grid(box, range, cg, cs);
  if (rc)
    return rc;
  double inv_cs[3];
  for (int i = 0; i < 3; ++i)
    inv_cs[i] = 1.0 / cs[i];
  int const gg[3] = {cg[0] + 2, cg[1] + 2, cg[2] + 2};
  for (long p = 0; p < n; ++p) {
    int cpos[3];
    bool out = false;
    for (int i = 0; i < 3; ++i) {
      double const x = pos[3 * p + i];
      cpos[i] = static_cast<int>(std::floor(x * inv_cs[i])) + 1;
      if (cpos[i] < 1) {
        if (x >= box[i])
          cpos[i] = 1;
        else
          out = true;
      } else if (cpos[i] > cg[i]) {
        if (x < box[i])
          cpos[i] = cg[i];
        else
          out = true;
      }
    }
    cell_out[p] = out ? -1 : cpos[0] + gg[0] * (cpos[1] + gg[1] * cpos[2]);
  }
  return 0;
}

} // extern "C"

namespace {
struct CellList {
  int cg[3];
  double cs[3], inv_cs[3];
  std::vector<long> start, order;
  std::vector<std::vector<int>> neigh; // unique neighbour cells (27 or fewer)
  int build(const double *box, double range, long n, const double *posf) {
    int const rc = oracle_cell_grid(box, range, cg, cs);
    if (rc)
      return rc;
    for (int i = 0; i < 3; ++i)
      inv_cs[i] = 1.0 / cs[i];
    long const nc = long(cg[0]) * cg[1] * cg[2];
    std::vector<int> cell(n);
    std::vector<long> cnt(nc + 1, 0);
    for (long p = 0; p < n; ++p) {
      int c3[3];
      for (int i = 0; i < 3; ++i) {
        int c = static_cast<int>(std::floor(posf[3 * p + i] * inv_cs[i]));
        c = std::min(std::max(c, 0), cg[i] - 1);
        c3[i] = c;
      }
      cell[p] = c3[0] + cg[0] * (c3[1] + cg[1] * c3[2]);
      cnt[cell[p] + 1]++;
    }
    for (long c = 0; c < nc; ++c)
      cnt[c + 1] += cnt[c];
    start = cnt;
    order.assign(n, 0);
    std::vector<long> fill(cnt.begin(), cnt.end() - 1);
    for (long p = 0; p < n; ++p)
      order[fill[cell[p]]++] = p;
    neigh.assign(nc, {});
    for (int z = 0; z < cg[2]; ++z)
      for (int y = 0; y < cg[1]; ++y)
        for (int x = 0; x < cg[0]; ++x) {
          std::set<int> s;
          for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
              for (int dx = -1; dx <= 1; ++dx) {
                int const xx = (x + dx + cg[0]) % cg[0];
                int const yy = (y + dy + cg[1]) % cg[1];
                int const zz = (z + dz + cg[2]) % cg[2];
                s.insert(xx + cg[0] * (yy + cg[1] * zz));
              }
          neigh[x + cg[0] * (y + cg[1] * z)].assign(s.begin(), s.end());
        }
    return 0;
  }
};

/* get_mi_vector, BoxGeometry.hpp:47-60 and 210-225 */
inline double mi(double dx, double L) {
  if (std::fabs(dx) > 0.5 * L)
    return dx - std::round(dx * (1.0 / L)) * L;
  return dx;
}
} // namespace

extern "C" {

long oracle_verlet_pairs(const double *box, double skin, double coulomb_cut,
                         long n, const double *pos, const double *q,
                         const int *type, int ntypes, const double *ia_cut,
                         long cap, long *pairs_out) {
  double max_cut = coulomb_cut;
  for (int i = 0; i < ntypes * ntypes; ++i)
    max_cut = std::max(max_cut, ia_cut[i]);
  double const range = max_cut + skin;
  std::vector<double> pf(3 * n);
  for (long i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d)
      pf[3 * i + d] = fold(pos[3 * i + d], box[d]);
  CellList cl;
  if (cl.build(box, range, n, pf.data()))
    return -2;
  double const eff_max2 = (max_cut + skin) * (max_cut + skin);
  double const eff_coul2 = coulomb_cut > 0 ? (coulomb_cut + skin) * (coulomb_cut + skin) : -1.0;
  long count = 0;
  long const nc = long(cl.cg[0]) * cl.cg[1] * cl.cg[2];
  for (long c = 0; c < nc; ++c) {
    for (long a = cl.start[c]; a < cl.start[c + 1]; ++a) {
      long const i = cl.order[a];
      for (int c2 : cl.neigh[c]) {
        for (long b = cl.start[c2]; b < cl.start[c2 + 1]; ++b) {
          long const j = cl.order[b];
          if (j <= i)
            continue;
          double d2 = 0.0;
          for (int d = 0; d < 3; ++d) {
            double const dx = mi(pf[3 * i + d] - pf[3 * j + d], box[d]);
            d2 += dx * dx;
          }
          if (d2 > eff_max2)
            continue;
          bool take = false;
          if (eff_coul2 >= 0 && d2 <= eff_coul2 && q[i] != 0.0 && q[j] != 0.0)
            take = true;
          if (!take) {
            int const ti = type ? type[i] : 0, tj = type ? type[j] : 0;
            double const ic = ia_cut[ti * ntypes + tj];
            if (ic != -1.0 && d2 <= (ic + skin) * (ic + skin))
              take = true;
          }
          if (take) {
            if (count < cap) {
              pairs_out[2 * count] = i;
              pairs_out[2 * count + 1] = j;
            }
            ++count;
          }
        }
      }
    }
  }
  return count <= cap ? count : -1;
}

/* Real-space Coulomb (p3m.hpp:146-180) + LJ/WCA (lj.hpp:41-60,
 * wca.hpp:39-55) over the link-cell pair loop (short_range_loop.hpp:44-61,
 * forces_inline.hpp:188-273, energy_inline.hpp, pressure_inline.hpp:59-92).
 * Each unordered pair within the cutoffs is evaluated once, d = p_i - p_j. */
int oracle_short_range(const oracle_p3m_params *pp, long n, const double *pos,
                       const double *q, const int *type, int ntypes,
                       const oracle_pair_params *tab, double *f,
                       double *energy_out, double *virial_out) {
  auto const &p = *pp;
  double max_cut = (p.prefactor != 0.0) ? p.r_cut : 0.0;
  std::vector<double> lj_cut(ntypes * ntypes), wca_cut(ntypes * ntypes);
  for (int i = 0; i < ntypes * ntypes; ++i) {
    lj_cut[i] = tab ? tab[i].lj_cut : 0.0;
    wca_cut[i] = (tab && tab[i].wca_sig != 0.0) ? tab[i].wca_sig * std::pow(2.0, 1.0 / 6.0) : 0.0;
    max_cut = std::max(max_cut, std::max(lj_cut[i], wca_cut[i]));
  }
  std::vector<double> pf(3 * n);
  for (long i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d)
      pf[3 * i + d] = fold(pos[3 * i + d], p.box[d]);
  CellList cl;
  if (cl.build(p.box, max_cut + p.skin, n, pf.data()))
    return 2;
  double const alpha = p.alpha;
  double const max_cut2 = max_cut * max_cut;
  double const two_a_sqrt_pi_i = 2.0 * alpha * (1.0 / std::sqrt(PI));
  long const nc = long(cl.cg[0]) * cl.cg[1] * cl.cg[2];
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  std::vector<double> e_c(nthreads, 0.0), e_n(nthreads, 0.0);
  std::vector<double> v_c(9 * nthreads, 0.0), v_n(9 * nthreads, 0.0);
  // each particle accumulates its own force over all neighbours (full
  // list), energies/virials count each pair once (j > i)
#pragma omp parallel for schedule(dynamic, 16)
  for (long c = 0; c < nc; ++c) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    for (long a = cl.start[c]; a < cl.start[c + 1]; ++a) {
      long const i = cl.order[a];
      double fi[3] = {0, 0, 0};
      for (int c2 : cl.neigh[c]) {
        for (long b = cl.start[c2]; b < cl.start[c2 + 1]; ++b) {
          long const j = cl.order[b];
          if (j == i)
            continue;
          double d[3];
          double d2 = 0.0;
          for (int k = 0; k < 3; ++k) {
            d[k] = mi(pf[3 * i + k] - pf[3 * j + k], p.box[k]);
            d2 += d[k] * d[k];
          }
          if (d2 >= max_cut2)
            continue; // beyond every cutoff: all kernels return zero
          double const dist = std::sqrt(d2);
          double fc[3] = {0, 0, 0}, fnb[3] = {0, 0, 0};
          double ec = 0.0, en = 0.0;
          double const q1q2 = q[i] * q[j];
          if (p.prefactor != 0.0 && q1q2 != 0.0 && dist < p.r_cut && dist > 0.0) {
            double const adist = alpha * dist;
            double const exp_adist_sq = std::exp(-adist * adist);
            double const dist_sq = dist * dist;
            double const erfc_part_ri = as_erfc_part(adist) / dist;
            double const fac = exp_adist_sq * (erfc_part_ri + two_a_sqrt_pi_i) / dist_sq;
            for (int k = 0; k < 3; ++k)
              fc[k] = (fac * p.prefactor * q1q2) * d[k];
            ec = p.prefactor * q1q2 * erfc_part_ri * exp_adist_sq;
          }
          if (tab) {
            int const ti = type ? type[i] : 0, tj = type ? type[j] : 0;
            auto const &ia = tab[ti * ntypes + tj];
            double ff = 0.0;
            if (dist < ia.lj_cut + ia.lj_offset && dist > ia.lj_min + ia.lj_offset) {
              double const r_off = dist - ia.lj_offset;
              double const s = ia.lj_sig / r_off;
              double const s2 = s * s;
              double const frac6 = s2 * s2 * s2;
              ff += 48.0 * ia.lj_eps * frac6 * (frac6 - 0.5) / (r_off * dist);
              en += 4.0 * ia.lj_eps * (frac6 * frac6 - frac6 + ia.lj_shift);
            }
            double const wc = wca_cut[ti * ntypes + tj];
            if (dist < wc) {
              double const s = ia.wca_sig / dist;
              double const s2 = s * s;
              double const frac6 = s2 * s2 * s2;
              ff += 48.0 * ia.wca_eps * frac6 * (frac6 - 0.5) / (dist * dist);
              en += 4.0 * ia.wca_eps * (frac6 * frac6 - frac6 + 0.25);
            }
            for (int k = 0; k < 3; ++k)
              fnb[k] = ff * d[k];
          }
          for (int k = 0; k < 3; ++k)
            fi[k] += fc[k] + fnb[k];
          if (j > i) {
            e_c[tid] += ec;
            e_n[tid] += en;
            for (int r = 0; r < 3; ++r)
              for (int s = 0; s < 3; ++s) {
                v_c[9 * tid + 3 * r + s] += fc[r] * d[s];
                v_n[9 * tid + 3 * r + s] += d[r] * fnb[s];
              }
          }
        }
      }
      for (int k = 0; k < 3; ++k)
        f[3 * i + k] += fi[k];
    }
  }
  if (energy_out) {
    energy_out[0] = energy_out[1] = 0.0;
    for (int t = 0; t < nthreads; ++t) {
      energy_out[0] += e_c[t];
      energy_out[1] += e_n[t];
    }
  }
  if (virial_out) {
    for (int k = 0; k < 18; ++k)
      virial_out[k] = 0.0;
    for (int t = 0; t < nthreads; ++t)
      for (int k = 0; k < 9; ++k) {
        virial_out[k] += v_c[9 * t + k];
        virial_out[9 + k] += v_n[9 * t + k];
      }
  }
  return 0;
}

/* p3m_real_space_error, p3m.cpp:187-193 */
double oracle_rs_error(double pref, double r_cut_iL, int n_c_part,
                       double sum_q2, double alpha_L, const double *box) {
  double const volume = box[0] * box[1] * box[2];
  return (2. * pref * sum_q2 * std::exp(-(r_cut_iL * alpha_L) * (r_cut_iL * alpha_L))) /
         std::sqrt(static_cast<double>(n_c_part) * r_cut_iL * box[0] * volume);
}

/* p3m_k_space_error + p3m_tune_aliasing_sums, p3m.cpp:146-175, 208-243 */
double oracle_ks_error(double pref, const int *mesh, int cao, int n_c_part,
                       double sum_q2, double alpha_L, const double *box) {
  double const mesh_i[3] = {1.0 / mesh[0], 1.0 / mesh[1], 1.0 / mesh[2]};
  double const alpha_L_i = 1.0 / alpha_L;
  double const factor1 = (PI * alpha_L_i) * (PI * alpha_L_i);
  double he_q = 0.0;
#pragma omp parallel for reduction(+ : he_q) schedule(static)
  for (int nx = -mesh[0] / 2; nx < mesh[0] / 2; ++nx) {
    double const csx = cotangent_sum(cao, nx, mesh_i[0]);
    double const fx = sinc(nx * mesh_i[0]);
    for (int ny = -mesh[1] / 2; ny < mesh[1] / 2; ++ny) {
      double const csy = cotangent_sum(cao, ny, mesh_i[1]);
      double const fy = sinc(ny * mesh_i[1]);
      for (int nz = -mesh[2] / 2; nz < mesh[2] / 2; ++nz) {
        if (nx == 0 && ny == 0 && nz == 0)
          continue;
        double const csz = cotangent_sum(cao, nz, mesh_i[2]);
        double const fz = sinc(nz * mesh_i[2]);
        double const n2 = double(nx) * nx + double(ny) * ny + double(nz) * nz;
        double const cs = csx * csy * csz;
        double const ex = std::exp(-factor1 * n2);
        double const energy = std::pow(fx * fy * fz, 2 * cao);
        double const alias1 = ex * ex / n2;
        double const alias2 = energy * ex * n2 / n2;
        double const d = alias1 - (alias2 / cs) * (alias2 / cs) / n2;
        if (d > 0. && std::fabs(d / alias1) > 1e-14)
          he_q += d;
      }
    }
  }
  return 2. * pref * sum_q2 * std::sqrt(he_q / static_cast<double>(n_c_part)) /
         (box[1] * box[2]);
}

/* Independent FP64 Ewald sum: real space with exact erfc over the minimum
 * image (r_cut <= L/2), reciprocal sum over |n| <= kmax, self term, the
 * neutralising-background term and (epsilon > 0) the textbook surface term
 * 2 pi |M|^2 / ((2 eps + 1) V). */
int oracle_ewald(const double *box, long n, const double *pos, const double *q,
                 double prefactor, double alpha, double r_cut, int kmax,
                 double epsilon, double *f, double *energy) {
  double const V = box[0] * box[1] * box[2];
  double e_real = 0.0;
  double const two_a_sqrt_pi_i = 2.0 * alpha / std::sqrt(PI);
#pragma omp parallel for reduction(+ : e_real) schedule(dynamic, 8)
  for (long i = 0; i < n; ++i) {
    double fi[3] = {0, 0, 0};
    for (long j = 0; j < n; ++j) {
      if (j == i)
        continue;
      double d[3], d2 = 0.0;
      for (int k = 0; k < 3; ++k) {
        double dx = pos[3 * i + k] - pos[3 * j + k];
        dx -= std::round(dx / box[k]) * box[k];
        d[k] = dx;
        d2 += dx * dx;
      }
      if (d2 >= r_cut * r_cut)
        continue;
      double const r = std::sqrt(d2);
      double const qq = q[i] * q[j];
      double const erfc_r = std::erfc(alpha * r) / r;
      double const fac = (erfc_r + two_a_sqrt_pi_i * std::exp(-alpha * alpha * d2)) / d2;
      for (int k = 0; k < 3; ++k)
        fi[k] += prefactor * qq * fac * d[k];
      e_real += 0.5 * qq * erfc_r;
    }
    for (int k = 0; k < 3; ++k)
      f[3 * i + k] += fi[k];
  }
  // reciprocal space over the half space n > 0 (lexicographic), doubled
  std::vector<int> nvec;
  for (int nx = 0; nx <= kmax; ++nx)
    for (int ny = -kmax; ny <= kmax; ++ny)
      for (int nz = -kmax; nz <= kmax; ++nz) {
        if (nx == 0 && (ny < 0 || (ny == 0 && nz <= 0)))
          continue;
        if (nx * nx + ny * ny + nz * nz > kmax * kmax)
          continue;
        nvec.push_back(nx);
        nvec.push_back(ny);
        nvec.push_back(nz);
      }
  long const nk = static_cast<long>(nvec.size() / 3);
  std::vector<double> Sr(nk, 0.0), Si(nk, 0.0), A(nk), kv(3 * nk);
  for (long k = 0; k < nk; ++k) {
    double k2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      kv[3 * k + d] = 2.0 * PI * nvec[3 * k + d] / box[d];
      k2 += kv[3 * k + d] * kv[3 * k + d];
    }
    A[k] = std::exp(-k2 / (4.0 * alpha * alpha)) / k2;
  }
#pragma omp parallel for schedule(static)
  for (long k = 0; k < nk; ++k) {
    double sr = 0.0, si = 0.0;
    for (long j = 0; j < n; ++j) {
      double const th = kv[3 * k] * pos[3 * j] + kv[3 * k + 1] * pos[3 * j + 1] +
                        kv[3 * k + 2] * pos[3 * j + 2];
      sr += q[j] * std::cos(th);
      si += q[j] * std::sin(th);
    }
    Sr[k] = sr;
    Si[k] = si;
  }
  double e_rec = 0.0;
  for (long k = 0; k < nk; ++k)
    e_rec += 2.0 * A[k] * (Sr[k] * Sr[k] + Si[k] * Si[k]);
  e_rec *= 2.0 * PI / V;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    double fi[3] = {0, 0, 0};
    for (long k = 0; k < nk; ++k) {
      double const th = kv[3 * k] * pos[3 * i] + kv[3 * k + 1] * pos[3 * i + 1] +
                        kv[3 * k + 2] * pos[3 * i + 2];
      double const s = std::sin(th), c = std::cos(th);
      double const w = 2.0 * A[k] * (s * Sr[k] - c * Si[k]);
      for (int d = 0; d < 3; ++d)
        fi[d] += w * kv[3 * k + d];
    }
    for (int d = 0; d < 3; ++d)
      f[3 * i + d] += prefactor * (4.0 * PI * q[i] / V) * fi[d];
  }
  double sum_q2 = 0.0, sum_q = 0.0, M[3] = {0, 0, 0};
  for (long i = 0; i < n; ++i) {
    sum_q2 += q[i] * q[i];
    sum_q += q[i];
    for (int d = 0; d < 3; ++d)
      M[d] += q[i] * pos[3 * i + d];
  }
  double e = e_real + e_rec - alpha / std::sqrt(PI) * sum_q2 -
             PI * sum_q * sum_q / (2.0 * V * alpha * alpha);
  if (epsilon > 0.0) {
    double const c = 2.0 * PI / ((2.0 * epsilon + 1.0) * V);
    e += c * (M[0] * M[0] + M[1] * M[1] + M[2] * M[2]);
    for (long i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d)
        f[3 * i + d] -= prefactor * 2.0 * c * q[i] * M[d];
  }
  *energy = prefactor * e;
  return 0;
}


/* Direct FP64 Ewald forces on a subsample of targets from ALL n sources
 * (metallic boundary), for error measurements on systems too large for the
 * all-pairs sum.  Real space: exact erfc over a cell list of the sources
 * (minimum image, r_cut <= min(L)/2).  Reciprocal space: structure factor
 * S(k) = sum_j q_j exp(i k.r_j) over |n| <= kmax (half space, doubled), the
 * phases built per source from the three axis phases exp(i 2 pi n x / L) by
 * repeated multiplication (one complex product per k vector and source),
 * summed per thread and then added over threads in thread order.  Forces
 * are written (not added) to f (3 nt). */
int oracle_ewald_targets(const double *box, long n, const double *pos, const double *q,
                         long nt, const long *tidx, double prefactor, double alpha,
                         double r_cut, int kmax, double *f) {
  double const V = box[0] * box[1] * box[2];
  for (int d = 0; d < 3; ++d)
    if (!(r_cut <= 0.5 * box[d]))
      return 1;
  for (long t = 0; t < nt; ++t)
    if (tidx[t] < 0 || tidx[t] >= n)
      return 2;
  // cell list of the sources: cells of edge >= r_cut / 4
  int nc[3];
  double cs[3];
  for (int d = 0; d < 3; ++d) {
    nc[d] = std::max(1, static_cast<int>(std::floor(box[d] / (0.25 * r_cut))));
    nc[d] = std::min(nc[d], 256);
    cs[d] = box[d] / nc[d];
  }
  long const ncell = static_cast<long>(nc[0]) * nc[1] * nc[2];
  auto fold = [&](double x, int d) {
    double y = x - std::floor(x / box[d]) * box[d];
    return (y >= box[d]) ? 0.0 : y;
  };
  std::vector<long> cstart(ncell + 1, 0), order(n);
  std::vector<int> cell_of(n);
  for (long j = 0; j < n; ++j) {
    int c[3];
    for (int d = 0; d < 3; ++d)
      c[d] = std::min(nc[d] - 1, static_cast<int>(fold(pos[3 * j + d], d) / cs[d]));
    cell_of[j] = (c[0] * nc[1] + c[1]) * nc[2] + c[2];
    ++cstart[cell_of[j] + 1];
  }
  for (long c = 0; c < ncell; ++c)
    cstart[c + 1] += cstart[c];
  {
    std::vector<long> fill(cstart.begin(), cstart.end() - 1);
    for (long j = 0; j < n; ++j)
      order[fill[cell_of[j]]++] = j;
  }
  int reach[3];
  for (int d = 0; d < 3; ++d)
    reach[d] = std::min(static_cast<int>(std::ceil(r_cut / cs[d])), (nc[d] - 1) / 2);
  double const two_a_sqrt_pi_i = 2.0 * alpha / std::sqrt(PI);
  double const rc2 = r_cut * r_cut;
#pragma omp parallel for schedule(dynamic, 4)
  for (long t = 0; t < nt; ++t) {
    long const i = tidx[t];
    double xi[3];
    int ci[3];
    for (int d = 0; d < 3; ++d) {
      xi[d] = pos[3 * i + d];
      ci[d] = std::min(nc[d] - 1, static_cast<int>(fold(xi[d], d) / cs[d]));
    }
    double fi[3] = {0, 0, 0};
    // every cell within reach, each visited once even when the reach
    // covers the whole axis
    for (int ox = -reach[0]; ox <= reach[0]; ++ox)
      for (int oy = -reach[1]; oy <= reach[1]; ++oy)
        for (int oz = -reach[2]; oz <= reach[2]; ++oz) {
          int const cx = ((ci[0] + ox) % nc[0] + nc[0]) % nc[0];
          int const cy = ((ci[1] + oy) % nc[1] + nc[1]) % nc[1];
          int const cz = ((ci[2] + oz) % nc[2] + nc[2]) % nc[2];
          long const c = (static_cast<long>(cx) * nc[1] + cy) * nc[2] + cz;
          for (long s = cstart[c]; s < cstart[c + 1]; ++s) {
            long const j = order[s];
            if (j == i)
              continue;
            double dv[3], d2 = 0.0;
            for (int d = 0; d < 3; ++d) {
              double dx = xi[d] - pos[3 * j + d];
              dx -= std::round(dx / box[d]) * box[d];
              dv[d] = dx;
              d2 += dx * dx;
            }
            if (d2 >= rc2)
              continue;
            double const r = std::sqrt(d2);
            double const fac =
                q[j] * (std::erfc(alpha * r) / r + two_a_sqrt_pi_i * std::exp(-alpha * alpha * d2)) / d2;
            for (int d = 0; d < 3; ++d)
              fi[d] += fac * dv[d];
          }
        }
    for (int d = 0; d < 3; ++d)
      f[3 * t + d] = prefactor * q[i] * fi[d];
  }
  // reciprocal space: k vectors of the half space nx > 0, or nx = 0 and
  // (ny > 0 or ny = 0 and nz > 0), |n| <= kmax; for each (nx, ny) the nz run
  // [nz0, nz1] is contiguous
  struct Run {
    int nx, ny, nz0, nz1;
    long k0;
  };
  std::vector<Run> runs;
  long nk = 0;
  for (int nx = 0; nx <= kmax; ++nx)
    for (int ny = -kmax; ny <= kmax; ++ny) {
      int const rem = kmax * kmax - nx * nx - ny * ny;
      if (rem < 0 || (nx == 0 && ny < 0))
        continue;
      int const zm = static_cast<int>(std::floor(std::sqrt(static_cast<double>(rem)) + 1e-12));
      int const z0 = (nx == 0 && ny == 0) ? 1 : -zm;
      if (z0 > zm)
        continue;
      runs.push_back(Run{nx, ny, z0, zm, nk});
      nk += zm - z0 + 1;
    }
  std::vector<double> A(nk);
  for (auto const &rn : runs)
    for (int nz = rn.nz0; nz <= rn.nz1; ++nz) {
      double const kx = 2.0 * PI * rn.nx / box[0], ky = 2.0 * PI * rn.ny / box[1],
                   kz = 2.0 * PI * nz / box[2];
      double const k2 = kx * kx + ky * ky + kz * kz;
      A[rn.k0 + nz - rn.nz0] = std::exp(-k2 / (4.0 * alpha * alpha)) / k2;
    }
  int nthr = 1;
#ifdef _OPENMP
  nthr = omp_get_max_threads();
#endif
  std::vector<double> Sr_t(static_cast<size_t>(nthr) * nk, 0.0), Si_t(static_cast<size_t>(nthr) * nk, 0.0);
  int const W = 2 * kmax + 1;
  // axis phases of one particle: px[n] (n = 0..kmax), py/pz[n + kmax] (n = -kmax..kmax)
  auto axis_phases = [&](const double *x, std::vector<cd> &px, std::vector<cd> &py,
                         std::vector<cd> &pz) {
    cd const ux = std::polar(1.0, 2.0 * PI * x[0] / box[0]);
    cd const uy = std::polar(1.0, 2.0 * PI * x[1] / box[1]);
    cd const uz = std::polar(1.0, 2.0 * PI * x[2] / box[2]);
    px[0] = 1.0;
    py[kmax] = 1.0;
    pz[kmax] = 1.0;
    for (int m = 1; m <= kmax; ++m) {
      px[m] = px[m - 1] * ux;
      py[kmax + m] = py[kmax + m - 1] * uy;
      pz[kmax + m] = pz[kmax + m - 1] * uz;
      py[kmax - m] = std::conj(py[kmax + m]);
      pz[kmax - m] = std::conj(pz[kmax + m]);
    }
  };
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double *sr = Sr_t.data() + static_cast<size_t>(tid) * nk;
    double *si = Si_t.data() + static_cast<size_t>(tid) * nk;
    std::vector<cd> px(kmax + 1), py(W), pz(W);
    std::vector<double> zr(W), zi(W);
#pragma omp for schedule(static)
    for (long j = 0; j < n; ++j) {
      axis_phases(pos + 3 * j, px, py, pz);
      for (int m = 0; m < W; ++m) {
        zr[m] = pz[m].real();
        zi[m] = pz[m].imag();
      }
      double const qj = q[j];
      for (auto const &rn : runs) {
        cd const exy = qj * px[rn.nx] * py[kmax + rn.ny];
        double const ar = exy.real(), ai = exy.imag();
        double *srk = sr + rn.k0 - rn.nz0;
        double *sik = si + rn.k0 - rn.nz0;
        for (int nz = rn.nz0; nz <= rn.nz1; ++nz) {
          double const br = zr[kmax + nz], bi = zi[kmax + nz];
          srk[nz] += ar * br - ai * bi;
          sik[nz] += ar * bi + ai * br;
        }
      }
    }
  }
  std::vector<double> Sr(nk, 0.0), Si(nk, 0.0);
  for (int t = 0; t < nthr; ++t)
    for (long k = 0; k < nk; ++k) {
      Sr[k] += Sr_t[static_cast<size_t>(t) * nk + k];
      Si[k] += Si_t[static_cast<size_t>(t) * nk + k];
    }
#pragma omp parallel
  {
    std::vector<cd> px(kmax + 1), py(W), pz(W);
#pragma omp for schedule(dynamic, 8)
    for (long t = 0; t < nt; ++t) {
      long const i = tidx[t];
      axis_phases(pos + 3 * i, px, py, pz);
      double fi[3] = {0, 0, 0};
      for (auto const &rn : runs) {
        cd const exy = px[rn.nx] * py[kmax + rn.ny];
        double const kx = 2.0 * PI * rn.nx / box[0], ky = 2.0 * PI * rn.ny / box[1];
        for (int nz = rn.nz0; nz <= rn.nz1; ++nz) {
          cd const e = exy * pz[kmax + nz];
          long const k = rn.k0 + nz - rn.nz0;
          // sin(k.r) Sr - cos(k.r) Si
          double const w = 2.0 * A[k] * (e.imag() * Sr[k] - e.real() * Si[k]);
          fi[0] += w * kx;
          fi[1] += w * ky;
          fi[2] += w * (2.0 * PI * nz / box[2]);
        }
      }
      for (int d = 0; d < 3; ++d)
        f[3 * t + d] += prefactor * (4.0 * PI * q[i] / V) * fi[d];
    }
  }
  return 0;
}

} // extern "C"
