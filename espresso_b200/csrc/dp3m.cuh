// Dipolar P3M kernels (magnetostatics/dp3m.cpp, p3m/influence_function_dipolar.hpp).
//
// The three dipole-moment components are assigned to three meshes with the
// charge-assignment kernels (a component of mu in the charge slot of the
// weight record) and transformed forward with the z and y passes of the
// charge path.  This file adds what is specific to point dipoles:
//  * the dipolar influence functions G_energy (S = 2) and G_force (S = 3)
//    on the r2c half mesh, and the aliasing sum of the energy correction;
//  * an x pass that transforms the three components, forms
//    mu(k) . d_op(k) once per point, accumulates the k-space energy, and
//    emits three backward-x-transformed field spectra per launch (torque
//    fields, or one half of the symmetric force-field tensor);
//  * the per-particle combination of the interpolated fields into forces
//    and torques, and the real-space pair kernel over the Verlet lists.
#pragma once

#include "fft.cuh"
#include "p3m_kernels.cuh"
#include "pair.cuh"

namespace p3mx {

// calc_meshift (p3m/common.hpp:248-264): index shift of the influence
// function (M/2 -> -M/2) and of the differential operator (M/2 -> 0).
__host__ __device__ inline int dp_shift(int i, int m) { return (i < m / 2) ? i : i - m; }
__host__ __device__ inline int dp_dop(int i, int m) { return (i == m / 2) ? 0 : dp_shift(i, m); }

// G_opt_dipolar<S> for m = 0 aliasing at mesh index (x, y, z) of a cubic
// mesh M, box L (influence_function_dipolar.hpp:62-130): numerator
// U^2 exp(-pi^2 |n|^2 / alpha_L^2) / |n|^2 (d_op . n)^S, denominator
// |d_op|^(2S) (U^2)^2, zero at the points whose indices are all multiples
// of M/2, scaled by 2 M^3 / L^2.  Both S = 2 (energy) and S = 3 (force).
__device__ inline void dp3m_g(int x, int y, int z, int M, double L, double alpha, int cao,
                              double &g2, double &g3) {
  g2 = g3 = 0.0;
  int const h = M / 2;
  if (x % h == 0 && y % h == 0 && z % h == 0)
    return;
  int const sx = dp_shift(x, M), sy = dp_shift(y, M), sz = dp_shift(z, M);
  int const dx = dp_dop(x, M), dy = dp_dop(y, M), dz = dp_dop(z, M);
  double const mi = 1.0 / M;
  double const u = sinc_d(sx * mi) * sinc_d(sy * mi) * sinc_d(sz * mi);
  double const u2 = pow(u, 2.0 * cao);
  double const n2 = static_cast<double>(sx * sx + sy * sy + sz * sz);
  double const pa = kPi / (alpha * L);
  double const ex = pa * pa * n2;
  if (!(ex < 30.0))
    return;
  double const dn = static_cast<double>(dx * sx + dy * sy + dz * sz);
  double const dd = static_cast<double>(dx * dx + dy * dy + dz * dz);
  double const base = u2 * exp(-ex) / n2;
  double const fac = 2.0 * static_cast<double>(M) * M * M / (L * L);
  g2 = fac * (base * dn * dn) / (dd * dd * u2 * u2);
  g3 = fac * (base * dn * dn * dn) / (dd * dd * dd * u2 * u2);
}

// Both influence functions on the r2c half mesh (same point layout and
// block table as k_influence); computed in FP64, stored in Real.
template <typename Real>
__global__ void k_dp3m_influence(const RepGeom *__restrict__ reps, const int2 *__restrict__ blk,
                                 Real *__restrict__ g_e, Real *__restrict__ g_f) {
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  int const M = G.mesh[0];
  long long const local = static_cast<long long>(bk.y) * blockDim.x + threadIdx.x;
  long long const csize = static_cast<long long>(M) * M * G.hp;
  if (local >= csize)
    return;
  int const kz = static_cast<int>(local % G.hp);
  int const y = static_cast<int>((local / G.hp) % M);
  int const x = static_cast<int>(local / (static_cast<long long>(M) * G.hp));
  double g2 = 0.0, g3 = 0.0;
  if (kz <= M / 2)
    dp3m_g(x, y, kz, M, G.box[0], G.alpha, G.cao, g2, g3);
  g_e[G.km_off + local] = static_cast<Real>(g2);
  g_f[G.km_off + local] = static_cast<Real>(g3);
}

// Per-block partials of sum G_energy U2s |d_op|^2 over the full mesh, the
// mesh sum of calc_average_self_energy_k_space (dp3m.cpp:320-360): U2s the
// product of sinc(shift/M + m M)^(2 cao) summed over m in [-1, 1]^3 (the
// reference's aliasing loop steps the sinc argument by whole meshes).  A
// fixed grid-stride assignment of points to threads and fixed reductions:
// deterministic.
__global__ void k_dp3m_self_sum(int M, double L, double alpha, int cao,
                                double *__restrict__ partials) {
  long long const total = static_cast<long long>(M) * M * M;
  double acc = 0.0;
  for (long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; p < total;
       p += static_cast<long long>(gridDim.x) * blockDim.x) {
    int const z = static_cast<int>(p % M), y = static_cast<int>((p / M) % M),
              x = static_cast<int>(p / (static_cast<long long>(M) * M));
    double g2, g3;
    dp3m_g(x, y, z, M, L, alpha, cao, g2, g3);
    if (g2 == 0.0)
      continue;
    double const mi = 1.0 / M;
    int const s[3] = {dp_shift(x, M), dp_shift(y, M), dp_shift(z, M)};
    double sn[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int m = -1; m <= 1; ++m)
        sn[d][m + 1] = sinc_d(s[d] * mi + m * M);
    double u2s = 0.0;
    for (int m0 = 0; m0 < 3; ++m0)
      for (int m1 = 0; m1 < 3; ++m1)
        for (int m2 = 0; m2 < 3; ++m2)
          u2s += pow(sn[0][m0] * sn[1][m1] * sn[2][m2], 2.0 * cao);
    int const dx = dp_dop(x, M), dy = dp_dop(y, M), dz = dp_dop(z, M);
    acc += g2 * u2s * static_cast<double>(dx * dx + dy * dy + dz * dz);
  }
  __shared__ double red[32];
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1)
    acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0)
    red[wid] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w)
      s += red[w];
    partials[blockIdx.x] = s;
  }
}

// Per-block partials of the dipolar k-space error sum of the tuner
// (dp3m_k_space_error and dp3m_tune_aliasing_sums, dp3m.cpp:680-740, with
// the m = 0 aliasing term): over n in [-M/2, M/2)^3 without n = 0,
//   d = ex^2 |n|^2 - (U2 ex |n|^4 / cs)^2 / |n|^6,  ex = exp(-(pi/alpha_L)^2 |n|^2),
// cs the product of the analytic cotangent sums, added where d > 0 and
// |d / (ex^2 |n|^2)| > 1e-14.  Fixed grid-stride assignment and reductions.
__global__ void k_dp3m_ks_error(int M, int cao, double alpha_L, double *__restrict__ partials) {
  long long const total = static_cast<long long>(M) * M * M;
  double const mi = 1.0 / M;
  double const f1 = (kPi / alpha_L) * (kPi / alpha_L);
  double acc = 0.0;
  for (long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    int const nz = static_cast<int>(t % M) - M / 2;
    int const ny = static_cast<int>((t / M) % M) - M / 2;
    int const nx = static_cast<int>(t / (static_cast<long long>(M) * M)) - M / 2;
    if (nx == 0 && ny == 0 && nz == 0)
      continue;
    double const n2 = double(nx) * nx + double(ny) * ny + double(nz) * nz;
    double const cs = cot_sum(cao, nx, mi) * cot_sum(cao, ny, mi) * cot_sum(cao, nz, mi);
    double const ex = exp(-f1 * n2);
    double const u2 = pow(sinc_d(nx * mi) * sinc_d(ny * mi) * sinc_d(nz * mi), 2.0 * cao);
    double const a1 = ex * ex * n2;
    double const a2 = u2 * ex * (n2 * n2 * n2) / n2;
    double const d = a1 - (a2 / cs) * (a2 / cs) / (n2 * n2 * n2);
    if (d > 0.0 && fabs(d / a1) > 1e-14)
      acc += d;
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1)
    acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0)
    red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w)
      s += red[w];
    partials[blockIdx.x] = s;
  }
}

// Dipole moments (AoS, 3 per particle) -> the three components as separate
// arrays (the charge slot of the assignment weights), the list selector
// sel = 1 for a particle with a non-zero moment (0 otherwise: it has no
// real-space partners), a flag set when a selector changed since the last
// call, and per-block partials {n_dipoles, sum mu^2, M_x, M_y, M_z}.
__global__ void k_dp3m_prepare(long long n, const double *__restrict__ mu,
                               double *__restrict__ comp, double *__restrict__ sel,
                               int *__restrict__ sel_changed, double *__restrict__ partials) {
  double acc[5] = {0, 0, 0, 0, 0};
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) {
    double const m0 = mu[3 * i], m1 = mu[3 * i + 1], m2 = mu[3 * i + 2];
    comp[i] = m0;
    comp[n + i] = m1;
    comp[2 * n + i] = m2;
    double const m2s = m0 * m0 + m1 * m1 + m2 * m2;
    double const s = (m2s != 0.0) ? 1.0 : 0.0;
    if (sel[i] != s) {
      sel[i] = s;
      atomicOr(sel_changed, 1);
    }
    if (m2s != 0.0) {
      acc[0] = 1.0;
      acc[1] = m2s;
      acc[2] = m0;
      acc[3] = m1;
      acc[4] = m2;
    }
  }
  __shared__ double red[5][8];
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0)
      red[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w)
      s += red[threadIdx.x][w];
    partials[static_cast<long long>(blockIdx.x) * 5 + threadIdx.x] = s;
  }
}

// Fixed-order sum of nblk rows of `width` partials: one warp per column
// (launched with 32 * width threads), lane l summing rows l, l + 32, ...,
// then a fixed shuffle tree (deterministic; the loads of a lane are
// independent, not one serial chain per column).
__global__ void k_dp3m_sum_rows(const double *__restrict__ partials, int nblk, int width,
                                double *__restrict__ out) {
  int const k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= width)
    return;
  double s = 0.0;
  for (int b = lane; b < nblk; b += 32)
    s += partials[static_cast<long long>(b) * width + k];
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0)
    out[k] = s;
}

// ---- x pass of the dipolar k-space operator ------------------------------
// Per block: one ky, a tile of kz (the block table of the charge x pass).
// In mode 0 the three forward-transformed components F_d are staged and
// transformed along x one after another, accumulating mk = sum_d d_op_d F_d,
// which then replaces component x in place (each block rewrites only the
// lines it read); modes 1 and 2 load that mk.  Three output spectra are
// formed from mk and transformed backward along x:
//   mode 0 (torques, AssignTorques, dp3m.cpp:372-395):
//     d_op_j G_energy mk,                                   j = x, y, z
//   mode 1 / 2 (forces, AssignForces, dp3m.cpp:396-430):
//     -i d_op_c d_op_d G_force mk,  (c, d) = (x,x) (x,y) (x,z) / (y,y) (y,z) (z,z)
// EV: per-block partial of the k-space energy sum G_energy |mk|^2 with the
// Hermitian weights of the half mesh (1 at kz = 0 and M/2, else 2).
// Shared memory: 3 x tile staged lines of line_ld(M) (two FFT buffers and
// mk), twiddles (M): the charge x pass's layout.
template <typename Real, bool EV>
__global__ void __launch_bounds__(256, 1)
k_fft_x_dp3m(const RepGeom *__restrict__ reps, const Blk *__restrict__ blks,
             typename CplxOf<Real>::type *__restrict__ comp_hat, long long fstride,
             const Real *__restrict__ g_e, const Real *__restrict__ g_f, int mode,
             typename CplxOf<Real>::type *__restrict__ field0, int tile,
             double *__restrict__ partials, const typename CplxOf<Real>::type *__restrict__ twtab) {
  using C = typename CplxOf<Real>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Blk const bk = blks[blockIdx.x];
  RepGeom const &G = reps[bk.rep];
  int const M0 = G.mesh[0], M1 = G.mesh[1], M2 = G.mesh[2];
  int const H = M2 / 2 + 1;
  int const y = bk.a, kz0 = bk.b;
  int const T = min(tile, H - kz0);
  int const ld = line_ld(M0);
  int const L = tile * ld;
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + L;
  C *mk = b + L;
  C *tw = mk + L;
  load_twiddles(tw, twtab, G.plan[0]);
  long long const stride_x = static_cast<long long>(M1) * G.hp;
  long long const base = G.km_off + static_cast<long long>(y) * G.hp + kz0;
  int const tq = threadIdx.x & 15, xq = threadIdx.x >> 4;
  bool const col = tq < T;
  int const kz = kz0 + tq;
  int const dop_y = dp_dop(y, M1), dop_z = dp_dop(kz, M2);
  // stage T lines of src (column tq, rows x) into dst
  auto stage = [&](const C *src, C *dst) {
    for (int x0 = xq; x0 < M0; x0 += 64) {
      C v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int const x = x0 + 16 * u;
        if (col && x < M0)
          v[u] = src[base + x * stride_x + tq];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int const x = x0 + 16 * u;
        if (col && x < M0)
          dst[tq * ld + pix(x)] = v[u];
      }
    }
  };
  if (mode == 0) {
    for (int d = 0; d < 3; ++d) {
      stage(comp_hat + fstride * d, a);
      __syncthreads();
      C const *res = fft_lines<C>(a, b, T, ld, G.plan[0], tw, false);
      for (int x = xq; col && x < M0; x += 16) {
        Real const op = static_cast<Real>(d == 0 ? dp_dop(x, M0) : (d == 1 ? dop_y : dop_z));
        C const v = res[tq * ld + pix(x)];
        C const m = (d == 0) ? C{Real(0), Real(0)} : mk[tq * ld + pix(x)];
        mk[tq * ld + pix(x)] = C{m.x + op * v.x, m.y + op * v.y};
      }
      __syncthreads();
    }
    // mk for the force modes, in place of component x (same thread, same
    // point as the staging: the block's own lines only)
    if (col)
      for (int x = xq; x < M0; x += 16)
        comp_hat[base + x * stride_x + tq] = mk[tq * ld + pix(x)];
  } else {
    stage(comp_hat, mk);
    __syncthreads();
  }
  if constexpr (EV) {
    double acc = 0.0;
    double const wgt = (kz == 0 || kz == M2 / 2) ? 1.0 : 2.0;
    for (int x = xq; col && x < M0; x += 16) {
      C const m = mk[tq * ld + pix(x)];
      double const g = static_cast<double>(g_e[base + x * stride_x + tq]);
      acc += wgt * g * (static_cast<double>(m.x) * m.x + static_cast<double>(m.y) * m.y);
    }
    __shared__ double red[8];
    int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1)
      acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0)
      red[wid] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (blockDim.x >> 5); ++w)
        s += red[w];
      partials[blockIdx.x] = s;
    }
  }
  for (int j = 0; j < 3; ++j) {
    __syncthreads(); // the previous field's transform has been stored
    for (int x = xq; col && x < M0; x += 16) {
      int const op[3] = {dp_dop(x, M0), dop_y, dop_z};
      C const m = mk[tq * ld + pix(x)];
      C v;
      if (mode == 0) {
        Real const c = static_cast<Real>(op[j]) * g_e[base + x * stride_x + tq];
        v = C{c * m.x, c * m.y};
      } else {
        int const c0 = (mode == 1) ? 0 : (j == 2 ? 2 : 1);
        int const c1 = (mode == 1) ? j : (j == 0 ? 1 : 2);
        Real const c = static_cast<Real>(op[c0] * op[c1]) * g_f[base + x * stride_x + tq];
        v = C{c * m.y, -c * m.x}; // -i c mk
      }
      a[tq * ld + pix(x)] = v;
    }
    __syncthreads();
    C const *fres = fft_lines<C>(a, b, T, ld, G.plan[0], tw, true);
    if (col)
      for (int x = xq; x < M0; x += 16)
        field0[fstride * j + base + x * stride_x + tq] = fres[tq * ld + pix(x)];
  }
}

// Forces and torques from the interpolated fields (AoS, 3 per particle):
//   tau = -pt mu x E_t                        (dp3m.cpp:380-395)
//   F_d = pf sum_c mu_c E_f(d, c)             (dp3m.cpp:410-430)
// with et = E_t, efa = (E_xx, E_xy, E_xz), efb = (E_yy, E_yz, E_zz); for a
// non-metallic boundary (ps != 0) the surface-term torque
// tau -= ps mu x M, M = the total moment at sums[2..4] (calc_surface_term,
// dp3m.cpp:452-510).
__global__ void k_dp3m_combine(long long n, const double *__restrict__ mu,
                               const double *__restrict__ et, const double *__restrict__ efa,
                               const double *__restrict__ efb, double pt, double pf, double ps,
                               const double *__restrict__ sums, double *__restrict__ f,
                               double *__restrict__ tq, int overwrite) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double const m0 = mu[3 * i], m1 = mu[3 * i + 1], m2 = mu[3 * i + 2];
  double e0 = pt * et[3 * i], e1 = pt * et[3 * i + 1], e2 = pt * et[3 * i + 2];
  if (ps != 0.0) {
    e0 += ps * sums[2];
    e1 += ps * sums[3];
    e2 += ps * sums[4];
  }
  double const t0 = -(m1 * e2 - m2 * e1);
  double const t1 = -(m2 * e0 - m0 * e2);
  double const t2 = -(m0 * e1 - m1 * e0);
  double const xx = efa[3 * i], xy = efa[3 * i + 1], xz = efa[3 * i + 2];
  double const yy = efb[3 * i], yz = efb[3 * i + 1], zz = efb[3 * i + 2];
  double const f0 = pf * (m0 * xx + m1 * xy + m2 * xz);
  double const f1 = pf * (m0 * xy + m1 * yy + m2 * yz);
  double const f2 = pf * (m0 * xz + m1 * yz + m2 * zz);
  if (overwrite) {
    f[3 * i] = f0;
    f[3 * i + 1] = f1;
    f[3 * i + 2] = f2;
    tq[3 * i] = t0;
    tq[3 * i + 1] = t1;
    tq[3 * i + 2] = t2;
  } else {
    f[3 * i] += f0;
    f[3 * i + 1] += f1;
    f[3 * i + 2] += f2;
    tq[3 * i] += t0;
    tq[3 * i + 1] += t1;
    tq[3 * i + 2] += t2;
  }
}

// Dipole moments in cell-sorted order (the pair kernel's partner reads):
// FP64 records, or FP32 records in the same buffer for k_dp3m_pairs_rel.
__global__ void k_dp3m_sort_mu(long long n, const int *__restrict__ perm,
                               const double *__restrict__ mu, double4 *__restrict__ smu,
                               int fp32) {
  long long const s = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n)
    return;
  int const i = perm[s];
  if (fp32)
    reinterpret_cast<float4 *>(smu)[s] =
        make_float4(static_cast<float>(mu[3 * i]), static_cast<float>(mu[3 * i + 1]),
                    static_cast<float>(mu[3 * i + 2]), 0.f);
  else
    smu[s] = make_double4(mu[3 * i], mu[3 * i + 1], mu[3 * i + 2], 0.0);
}

// Real-space dipole-dipole energy, force and torque over the Verlet lists
// (dp3m.hpp:142-232, pair_force / pair_energy): with d = x_i - x_j and
//   B = (erfc(a r) / r + 2a/sqrt(pi) exp(-a^2 r^2)) / r^2
//   C = (3 B + 2 a^2 (2a/sqrt(pi)) exp(-a^2 r^2)) / r^2
//   D = (5 C + 4 a^4 (2a/sqrt(pi)) exp(-a^2 r^2)) / r^2
//   E   = mu_i.mu_j B - (mu_i.d)(mu_j.d) C
//   F_i = (mu_i.mu_j) C d + (mu_j.d) C mu_i + (mu_i.d) C mu_j - (mu_i.d)(mu_j.d) D d
//   T_i = -mu_i x mu_j B + (mu_i x d)(mu_j.d) C
// for r < r_cut; erfc(a r) exp(a^2 r^2) by Abramowitz & Stegun 7.1.26 when
// the target accuracy is above 5e-6, else erfc itself.  The lists hold both
// directions of every pair, so each particle sums its own force and torque
// (no atomics, a fixed order: deterministic); the energy takes half of
// every ordered pair.  One thread per cell-sorted particle.
template <bool EV>
__global__ void __launch_bounds__(256)
k_dp3m_pairs(const RepGeom *__restrict__ reps, const int2 *__restrict__ blk,
             const double4 *__restrict__ spq, const double4 *__restrict__ smu,
             const int *__restrict__ perm, const int *__restrict__ nb,
             const int *__restrict__ nb_cnt, double pref, int exact_erfc,
             double *__restrict__ f, double *__restrict__ tq, int overwrite,
             double *__restrict__ partials) {
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  long long const a = G.p0 + static_cast<long long>(bk.y) * blockDim.x + threadIdx.x;
  double energy = 0.0;
  if (a < G.p0 + G.np) {
    double4 const pa = spq[a];
    double4 const ma = smu[a];
    double const alpha = G.alpha, rc = G.r_cut;
    double const coeff = 2.0 * alpha / sqrt(kPi);
    double const a2 = alpha * alpha;
    double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
    int const cw = nb_cnt[a];
    int const cnt = nb_count(cw), cna = nb_count_a(cw);
    const int *nbp = nb + nb_base(G.nb_off, G.max_nb, a - G.p0);
    int const base0 = static_cast<int>(G.p0);
    // the next partner's records are loaded while the current pair is
    // evaluated (two dependent gathers per entry otherwise serialise)
    auto partner = [&](int k) {
      return base0 + static_cast<int>(static_cast<unsigned>(nbp[nb_logical(0, G.max_nb, cna, k)]) &
                                      kNbIndexMask);
    };
    int b_next = (cnt > 0) ? partner(0) : 0;
    double4 p_next = (cnt > 0) ? spq[b_next] : pa;
    double4 m_next = (cnt > 0) ? smu[b_next] : ma;
    for (int k = 0; k < cnt; ++k) {
      double4 const pb = p_next;
      double4 const mb = m_next;
      if (k + 1 < cnt) {
        b_next = partner(k + 1);
        p_next = spq[b_next];
        m_next = smu[b_next];
      }
      double const d0 = mi_d(pa.x - pb.x, G.box[0], G.box_i[0]);
      double const d1 = mi_d(pa.y - pb.y, G.box[1], G.box_i[1]);
      double const d2 = mi_d(pa.z - pb.z, G.box[2], G.box_i[2]);
      double const r2 = d0 * d0 + d1 * d1 + d2 * d2;
      double const r = sqrt(r2);
      if (!(r < rc) || !(r > 0.0))
        continue;
      // one division for 1/r^2 (1/r = r / r^2) and one for the A&S t
      double const inv_r2 = 1.0 / r2;
      double const inv_r = r * inv_r2;
      double const ad = alpha * r;
      double const exa = exp(-ad * ad);
      double B;
      if (exact_erfc) {
        B = (erfc(ad) * inv_r + coeff * exa) * inv_r2;
      } else {
        double const t = 1.0 / (1.0 + 0.3275911 * ad);
        double const asp =
            t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 +
                                                                         t * 1.061405429))));
        B = (asp * inv_r + coeff) * exa * inv_r2;
      }
      double const common = a2 * coeff * exa;
      double const Cc = (3.0 * B + 2.0 * common) * inv_r2;
      double const Dd = (5.0 * Cc + 4.0 * common * a2) * inv_r2;
      double const mimj = ma.x * mb.x + ma.y * mb.y + ma.z * mb.z;
      double const mir = ma.x * d0 + ma.y * d1 + ma.z * d2;
      double const mjr = mb.x * d0 + mb.y * d1 + mb.z * d2;
      if constexpr (EV)
        energy += mimj * B - mir * mjr * Cc;
      double const cd = mimj * Cc - mir * mjr * Dd;
      fx += cd * d0 + mjr * Cc * ma.x + mir * Cc * mb.x;
      fy += cd * d1 + mjr * Cc * ma.y + mir * Cc * mb.y;
      fz += cd * d2 + mjr * Cc * ma.z + mir * Cc * mb.z;
      double const s = mjr * Cc;
      tx += -(ma.y * mb.z - ma.z * mb.y) * B + (ma.y * d2 - ma.z * d1) * s;
      ty += -(ma.z * mb.x - ma.x * mb.z) * B + (ma.z * d0 - ma.x * d2) * s;
      tz += -(ma.x * mb.y - ma.y * mb.x) * B + (ma.x * d1 - ma.y * d0) * s;
    }
    if (f) {
      int const i = perm[a];
      if (overwrite) {
        f[3 * i] = pref * fx;
        f[3 * i + 1] = pref * fy;
        f[3 * i + 2] = pref * fz;
        tq[3 * i] = pref * tx;
        tq[3 * i + 1] = pref * ty;
        tq[3 * i + 2] = pref * tz;
      } else {
        f[3 * i] += pref * fx;
        f[3 * i + 1] += pref * fy;
        f[3 * i + 2] += pref * fz;
        tq[3 * i] += pref * tx;
        tq[3 * i + 1] += pref * ty;
        tq[3 * i + 2] += pref * tz;
      }
    }
  }
  if constexpr (EV) {
    __shared__ double red[8];
    int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double v = 0.5 * pref * energy;
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0)
      red[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (blockDim.x >> 5); ++w)
        s += red[w];
      partials[blockIdx.x] = s;
    }
  }
}

// The same pair terms for the FP32-mesh mode, in FP32 from the cell-relative
// offsets (as k_pair_forces_rel: d = (off_a - off_b) - dc cs with dc from
// the entry's offset code, no minimum-image arithmetic): hardware reciprocal
// square root, reciprocal and 2^x, A&S 7.1.26 or erfcf; each pair's force, torque and
// energy terms summed in FP64.
template <bool EV>
__global__ void __launch_bounds__(256)
k_dp3m_pairs_rel(const RepGeom *__restrict__ reps, const int2 *__restrict__ blk,
                 const float4 *__restrict__ spf, const float4 *__restrict__ smu,
                 const int *__restrict__ perm, const int *__restrict__ nb,
                 const int *__restrict__ nb_cnt, double pref, int exact_erfc,
                 double *__restrict__ f, double *__restrict__ tq, int overwrite,
                 double *__restrict__ partials) {
  int2 const bk = blk[blockIdx.x];
  RepGeom const &G = reps[bk.x];
  long long const a = G.p0 + static_cast<long long>(bk.y) * blockDim.x + threadIdx.x;
  double energy = 0.0;
  if (a < G.p0 + G.np) {
    float4 const pa = spf[a];
    float4 const ma = smu[a];
    float const alpha = static_cast<float>(G.alpha);
    float const rc2 = static_cast<float>(G.r_cut * G.r_cut);
    float const coeff = static_cast<float>(2.0 * G.alpha / sqrt(kPi));
    float const a2 = static_cast<float>(G.alpha * G.alpha);
    // exp(-(alpha r)^2) = 2^(c_exp r^2)
    float const c_exp = static_cast<float>(-G.alpha * G.alpha * 1.4426950408889634);
    float const cs_x = static_cast<float>(G.box[0] / G.cg[0]);
    float const cs_y = static_cast<float>(G.box[1] / G.cg[1]);
    float const cs_z = static_cast<float>(G.box[2] / G.cg[2]);
    double fx = 0, fy = 0, fz = 0, tx = 0, ty = 0, tz = 0;
    int const cw = nb_cnt[a];
    int const cnt = nb_count(cw), cna = nb_count_a(cw);
    const int *nbp = nb + nb_base(G.nb_off, G.max_nb, a - G.p0);
    long long const base0 = G.p0;
    auto entry = [&](int k) {
      return static_cast<unsigned>(nbp[nb_logical(0, G.max_nb, cna, k)]);
    };
    // the next partner's records are loaded while the current pair is
    // evaluated
    unsigned e_next = (cnt > 0) ? entry(0) : 0u;
    float4 p_next = (cnt > 0) ? spf[base0 + (e_next & kNbIndexMask)] : pa;
    float4 m_next = (cnt > 0) ? smu[base0 + (e_next & kNbIndexMask)] : ma;
    for (int k = 0; k < cnt; ++k) {
      unsigned const e = e_next;
      float4 const pb = p_next;
      float4 const mb = m_next;
      if (k + 1 < cnt) {
        e_next = entry(k + 1);
        p_next = spf[base0 + (e_next & kNbIndexMask)];
        m_next = smu[base0 + (e_next & kNbIndexMask)];
      }
      unsigned const code = e >> kNbIndexBits;
      float const d0 = fmaf(code_axis(code, 0), -cs_x, pa.x - pb.x);
      float const d1 = fmaf(code_axis(code, 1), -cs_y, pa.y - pb.y);
      float const d2 = fmaf(code_axis(code, 2), -cs_z, pa.z - pb.z);
      float const r2 = d0 * d0 + d1 * d1 + d2 * d2;
      if (!(r2 < rc2) || !(r2 > 0.f))
        continue;
      float const inv_r = rsqrt_approx(r2);
      float const inv_r2 = inv_r * inv_r;
      float const ad = alpha * (r2 * inv_r);
      float const exa = ex2_approx(c_exp * r2);
      float B;
      if (exact_erfc) {
        B = (erfcf(ad) * inv_r + coeff * exa) * inv_r2;
      } else {
        float const t = rcp_r(1.f + 0.3275911f * ad);
        float const asp =
            t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f +
                                                                           t * 1.061405429f))));
        B = (asp * inv_r + coeff) * exa * inv_r2;
      }
      float const common = a2 * coeff * exa;
      float const Cc = (3.f * B + 2.f * common) * inv_r2;
      float const Dd = (5.f * Cc + 4.f * common * a2) * inv_r2;
      float const mimj = ma.x * mb.x + ma.y * mb.y + ma.z * mb.z;
      float const mir = ma.x * d0 + ma.y * d1 + ma.z * d2;
      float const mjr = mb.x * d0 + mb.y * d1 + mb.z * d2;
      if constexpr (EV)
        energy += static_cast<double>(mimj * B - mir * mjr * Cc);
      float const cd = mimj * Cc - mir * mjr * Dd;
      fx += static_cast<double>(cd * d0 + mjr * Cc * ma.x + mir * Cc * mb.x);
      fy += static_cast<double>(cd * d1 + mjr * Cc * ma.y + mir * Cc * mb.y);
      fz += static_cast<double>(cd * d2 + mjr * Cc * ma.z + mir * Cc * mb.z);
      float const s = mjr * Cc;
      tx += static_cast<double>(-(ma.y * mb.z - ma.z * mb.y) * B + (ma.y * d2 - ma.z * d1) * s);
      ty += static_cast<double>(-(ma.z * mb.x - ma.x * mb.z) * B + (ma.z * d0 - ma.x * d2) * s);
      tz += static_cast<double>(-(ma.x * mb.y - ma.y * mb.x) * B + (ma.x * d1 - ma.y * d0) * s);
    }
    if (f) {
      int const i = perm[a];
      if (overwrite) {
        f[3 * i] = pref * fx;
        f[3 * i + 1] = pref * fy;
        f[3 * i + 2] = pref * fz;
        tq[3 * i] = pref * tx;
        tq[3 * i + 1] = pref * ty;
        tq[3 * i + 2] = pref * tz;
      } else {
        f[3 * i] += pref * fx;
        f[3 * i + 1] += pref * fy;
        f[3 * i + 2] += pref * fz;
        tq[3 * i] += pref * tx;
        tq[3 * i + 1] += pref * ty;
        tq[3 * i + 2] += pref * tz;
      }
    }
  }
  if constexpr (EV) {
    __shared__ double red[8];
    int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double v = 0.5 * pref * energy;
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0)
      red[wid] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (blockDim.x >> 5); ++w)
        s += red[w];
      partials[blockIdx.x] = s;
    }
  }
}

} // namespace p3mx
