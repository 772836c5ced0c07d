// Electrostatic layer correction (ELC) for slab systems: the far-formula
// correction that removes the interactions with the periodic images along z
// from a 3D-periodic P3M solution (electrostatics/elc.cpp), here without
// dielectric contrasts (delta_mid_top = delta_mid_bot = 0, no const_pot).
//
// The correction is a sum over Fourier modes (p, q) of the x-y plane; per
// mode it is a product decomposition: each particle contributes 4 (modes with
// p = 0 or q = 0) or 8 (p, q > 0) products of charge, sin/cos of its x and y
// phases and exp(+-omega z) (setup_PoQ :501-598, setup_PQ :641-769); the
// per-mode sums over all particles, times the mode prefactor, give each
// particle's force (add_PoQ_force :601-618, add_PQ_force :771-810) and the
// energy (PoQ_energy :620-634, PQ_energy :812-828).  The dipole term
// (add_dipole_force :201-264, dipole_energy :267-343) is three more sums.
//
// Device layout (all FP64):
//   sc   : per frequency f and particle i, (sin, cos) of 2 pi f x_i / L_x
//          (f = 1..nfx) then of 2 pi f y_i / L_y (f = 1..nfy), [f][i]
//          (calc_sc_cache :107-125);
//   part : per particle tile b and mode m, the 8 product sums
//          [b][m][8], then per tile the 3 dipole sums [b][3];
//   G    : per mode the 8 sums over all tiles times the mode prefactor, then
//          the 3 dipole sums;
//   epart: per block of the force kernel, its energy sum (EV only).
// Every sum is taken in a fixed order (no atomics): results are
// deterministic run to run.
#pragma once

#include "common.cuh"

namespace p3mx {

struct ElcMode {
  double omega; // 2 pi |(p / L_x, q / L_y)|
  double pref;  // -prefactor * {4, 8} pi / (L_x L_y) / expm1(omega L_z)
  double px, py; // 2 pi p / (L_x omega), 2 pi q / (L_y omega) (pq modes)
  int kind;      // 0: p-mode (q = 0), 1: q-mode (p = 0), 2: pq-mode
  int p, q, pad;
};

struct ElcGeom {
  double box[3];
  double box_h;        // L_z - gap
  double shift;        // L_z / 2
  double pref_dip;     // prefactor 4 pi / V (add_dipole_force)
  long long n;
  int nmodes, nfx, nfy, neutralize;
};

constexpr int kElcThreads = 256;
constexpr int kElcPPT = 4;            // particles per thread in the sums kernel
constexpr int kElcModesPerBlock = 16; // modes per block of the sums kernel

__device__ __forceinline__ double elc_fold(double x, double l) { return x - floor(x / l) * l; }

// sin / cos of the x and y phases of every particle at every frequency.
__global__ void __launch_bounds__(kElcThreads)
k_elc_sc(ElcGeom g, const double *__restrict__ pos, double2 *__restrict__ sc) {
  long long const t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  long long const nf = static_cast<long long>(g.nfx) + g.nfy;
  if (t >= nf * g.n)
    return;
  long long const f = t / g.n, i = t - f * g.n;
  int const dir = f < g.nfx ? 0 : 1;
  int const freq = static_cast<int>(dir == 0 ? f + 1 : f - g.nfx + 1);
  double const c = elc_fold(pos[3 * i + dir], g.box[dir]);
  double const pref = 2.0 * kPi * (1.0 / g.box[dir]) * static_cast<double>(freq);
  double s, co;
  sincos(pref * c, &s, &co);
  sc[t] = make_double2(s, co);
}

// the 4 / 8 products of particle i for mode md (z folded, e = exp(omega z))
__device__ __forceinline__ int elc_products(ElcMode const &md, ElcGeom const &g,
                                            const double2 *__restrict__ sc, long long i,
                                            double q, double z, double v[8]) {
  double const e = exp(md.omega * z);
  if (md.kind < 2) {
    long long const f = (md.kind == 0) ? (md.p - 1) : (g.nfx + md.q - 1);
    double2 const a = sc[f * g.n + i];
    // POQESP, POQECP, POQESM, POQECM
    v[0] = q * a.x * e;
    v[1] = q * a.y * e;
    v[2] = q * a.x / e;
    v[3] = q * a.y / e;
    return 4;
  }
  double2 const ax = sc[static_cast<long long>(md.p - 1) * g.n + i];
  double2 const ay = sc[static_cast<long long>(g.nfx + md.q - 1) * g.n + i];
  // PQESSP, PQESCP, PQECSP, PQECCP, PQESSM, PQESCM, PQECSM, PQECCM
  v[0] = ax.x * ay.x * q * e;
  v[1] = ax.x * ay.y * q * e;
  v[2] = ax.y * ay.x * q * e;
  v[3] = ax.y * ay.y * q * e;
  v[4] = ax.x * ay.x * q / e;
  v[5] = ax.x * ay.y * q / e;
  v[6] = ax.y * ay.x * q / e;
  v[7] = ax.y * ay.y * q / e;
  return 8;
}

// sum of v over the block (256 threads) in a fixed order, written by threads
// 0..W-1 to out[0..W); red: scratch of [8 warps][W] doubles.
template <int W>
__device__ __forceinline__ void elc_block_sum(double (&v)[W], double *red, double *out) {
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < W; ++c) {
    double s = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0)
      red[wid * W + c] = s;
  }
  __syncthreads();
  if (threadIdx.x < W) {
    double s = 0.0;
    for (int w = 0; w < kElcThreads / 32; ++w)
      s += red[w * W + threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Per particle tile (blockIdx.x) and mode chunk (blockIdx.y): the product sums
// of each mode; chunk 0 also takes the dipole sums and the gap check
// (check_gap :184-194: a charged particle below 0 or above L_z - gap).
__global__ void __launch_bounds__(kElcThreads)
k_elc_sums(ElcGeom g, const ElcMode *__restrict__ modes, const double *__restrict__ pos,
           const double *__restrict__ qv, const double2 *__restrict__ sc,
           double *__restrict__ part, int *__restrict__ gap_err) {
  __shared__ double red[(kElcThreads / 32) * 8];
  long long const tile0 = static_cast<long long>(blockIdx.x) * kElcThreads * kElcPPT;
  double zz[kElcPPT], qq[kElcPPT];
#pragma unroll
  for (int k = 0; k < kElcPPT; ++k) {
    long long const i = tile0 + k * kElcThreads + threadIdx.x;
    bool const ok = i < g.n;
    qq[k] = ok ? qv[i] : 0.0;
    zz[k] = ok ? elc_fold(pos[3 * i + 2], g.box[2]) : 0.0;
  }
  int const m0 = blockIdx.y * kElcModesPerBlock;
  int const m1 = min(g.nmodes, m0 + kElcModesPerBlock);
  for (int m = m0; m < m1; ++m) {
    ElcMode const md = modes[m];
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < kElcPPT; ++k) {
      long long const i = tile0 + k * kElcThreads + threadIdx.x;
      if (i < g.n && qq[k] != 0.0) {
        double v[8];
        int const w = elc_products(md, g, sc, i, qq[k], zz[k], v);
        for (int c = 0; c < w; ++c)
          acc[c] += v[c];
      }
    }
    elc_block_sum<8>(acc, red, part + (static_cast<long long>(blockIdx.x) * g.nmodes + m) * 8);
  }
  if (blockIdx.y == 0) {
    double d[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < kElcPPT; ++k) {
      long long const i = tile0 + k * kElcThreads + threadIdx.x;
      if (i < g.n && qq[k] != 0.0) {
        double const dz = zz[k] - g.shift;
        d[0] += qq[k] * dz;
        d[1] += qq[k];
        d[2] += qq[k] * dz * dz;
        if (zz[k] < 0.0 || zz[k] > g.box_h)
          atomicMin(gap_err, static_cast<int>(i));
      }
    }
    long long const nbp = gridDim.x;
    elc_block_sum<3>(d, red, part + nbp * g.nmodes * 8 + static_cast<long long>(blockIdx.x) * 3);
  }
}

// G[m][c] = pref_m * sum over tiles (fixed order); the dipole sums after them.
__global__ void k_elc_reduce(ElcGeom g, const ElcMode *__restrict__ modes,
                             const double *__restrict__ part, int nbp, double *__restrict__ G) {
  int const t = blockIdx.x * blockDim.x + threadIdx.x;
  int const nm8 = g.nmodes * 8;
  if (t < nm8) {
    double s = 0.0;
    for (int b = 0; b < nbp; ++b)
      s += part[static_cast<long long>(b) * nm8 + t];
    G[t] = modes[t >> 3].pref * s;
  } else if (t < nm8 + 3) {
    int const c = t - nm8;
    double s = 0.0;
    for (int b = 0; b < nbp; ++b)
      s += part[static_cast<long long>(nbp) * nm8 + static_cast<long long>(b) * 3 + c];
    G[t] = s;
  }
}

// Per particle: the mode forces from the global sums (add_PoQ_force,
// add_PQ_force), the dipole force, and with EV its energy terms
// (PoQ_energy, PQ_energy before the 1 / omega and the final halving).
template <bool EV>
__global__ void __launch_bounds__(kElcThreads)
k_elc_forces(ElcGeom g, const ElcMode *__restrict__ modes, const double *__restrict__ pos,
             const double *__restrict__ qv, const double2 *__restrict__ sc,
             const double *__restrict__ G, double *__restrict__ f, double *__restrict__ epart) {
  __shared__ double red[(kElcThreads / 32) * 8];
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  double en[1] = {0.0};
  if (i < g.n && qv[i] != 0.0) {
    double const q = qv[i];
    double const z = elc_fold(pos[3 * i + 2], g.box[2]);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int m = 0; m < g.nmodes; ++m) {
      ElcMode const md = modes[m];
      double v[8];
      elc_products(md, g, sc, i, q, z, v);
      const double *Gm = G + static_cast<long long>(m) * 8;
      if (md.kind < 2) {
        double const ft = v[2] * Gm[1] - v[3] * Gm[0] + v[0] * Gm[3] - v[1] * Gm[2];
        if (md.kind == 0)
          fx += ft;
        else
          fy += ft;
        fz += v[3] * Gm[1] + v[2] * Gm[0] - v[1] * Gm[3] - v[0] * Gm[2];
        if constexpr (EV)
          en[0] += (v[3] * Gm[1] + v[2] * Gm[0] + v[1] * Gm[3] + v[0] * Gm[2]) / md.omega;
      } else {
        fx += md.px * (v[5] * Gm[3] + v[4] * Gm[2] - v[7] * Gm[1] - v[6] * Gm[0] +
                       v[1] * Gm[7] + v[0] * Gm[6] - v[3] * Gm[5] - v[2] * Gm[4]);
        fy += md.py * (v[6] * Gm[3] + v[4] * Gm[1] - v[7] * Gm[2] - v[5] * Gm[0] +
                       v[2] * Gm[7] + v[0] * Gm[5] - v[3] * Gm[6] - v[1] * Gm[4]);
        fz += v[7] * Gm[3] + v[6] * Gm[2] + v[5] * Gm[1] + v[4] * Gm[0] - v[3] * Gm[7] -
              v[2] * Gm[6] - v[1] * Gm[5] - v[0] * Gm[4];
        if constexpr (EV)
          en[0] += (v[7] * Gm[3] + v[6] * Gm[2] + v[5] * Gm[1] + v[4] * Gm[0] + v[3] * Gm[7] +
                    v[2] * Gm[6] + v[1] * Gm[5] + v[0] * Gm[4]) /
                   md.omega;
      }
    }
    // dipole force (add_dipole_force :201-264 without contrasts / const_pot)
    const double *D = G + static_cast<long long>(g.nmodes) * 8;
    fz -= g.pref_dip * D[0] * q;
    if (!g.neutralize)
      fz += g.pref_dip * D[1] * q * (z - g.shift);
    f[3 * i + 0] += fx;
    f[3 * i + 1] += fy;
    f[3 * i + 2] += fz;
  }
  if constexpr (EV) {
    __shared__ double eb[1];
    elc_block_sum<1>(en, red, eb);
    if (threadIdx.x == 0)
      epart[blockIdx.x] = eb[0];
  }
}

} // namespace p3mx
