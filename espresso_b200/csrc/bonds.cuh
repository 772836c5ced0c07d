// Pair bonds: FENE (bonded_interactions/fene.hpp:37-105) and harmonic
// (harmonic.hpp:35-93) over the minimum-image vector d = x_i - x_j of the
// two partners (add_bonded_two_body_force, forces_inline.hpp:320-350: p1
// gets F(d), p2 gets -F(d) = F(-d)).
//
// Layout: every bond is listed at both of its ends (CSR over particles,
// entry = {partner, bond type}, entries of a particle in bond order), so one
// thread per particle sums its own bond forces in a fixed order: no atomics,
// bitwise reproducible, like the full Verlet lists of the pair kernel.
#pragma once

#include "common.cuh"

namespace p3mx {

constexpr int kBondFene = 1;
constexpr int kBondHarmonic = 2;

// One bond type (FP64, as the reference).  r_max: FENE d_r_max (largest
// r - r0), harmonic r_cut (0: no cutoff).
struct BondParam {
  int kind;
  double k, r0, r_max;
};

// Force factor and energy of a bond of length len: F = fac * d.  Status 0,
// 1 when the bond is stretched past its range (FeneBond::force returns no
// value for r - r0 >= d_r_max, HarmonicBond::force for r > r_cut: the
// reference reports "bond broken"), 2 for a zero-length bond with r0 > 0
// (the reference's "Particles have zero distance" runtime error).  The
// length guard ROUND_ERROR_PREC is 1e-14 (config.hpp:66).
__host__ __device__ inline int bond_eval(BondParam const &b, double len, double &fac,
                                         double &energy) {
  double const dr = len - b.r0;
  if (b.kind == kBondFene) {
    double const drmax2 = b.r_max * b.r_max;
    double const drmax2i = 1.0 / drmax2;
    if (dr >= b.r_max)
      return 1;
    fac = -b.k * dr / (1.0 - dr * dr * drmax2i);
    energy = -0.5 * b.k * drmax2 * log(1.0 - dr * dr * drmax2i);
  } else {
    if (b.r_max > 0.0 && len > b.r_max)
      return 1;
    fac = -b.k * dr;
    energy = 0.5 * b.k * dr * dr;
  }
  if (len > 1.0e-14)
    fac /= len;
  else if (b.r0 > 0.0)
    return 2;
  return 0;
}

// First failing bond: err[1] = status (1 broken, 2 zero length), err[2..3]
// = the two particles (the first thread to fail writes them).
__device__ inline void bond_report(int *err, int status, int i, int j) {
  if (atomicCAS(&err[1], 0, status) == 0) {
    err[2] = i;
    err[3] = j;
  }
}

// Minimum-image bond vector x_i - x_j of one entry.
__device__ inline void bond_vector(RepGeom const &G, const double *__restrict__ pos, long long i,
                                   int j, double d[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double const dx = pos[3 * i + k] - pos[3 * static_cast<long long>(j) + k];
    // get_mi_coord (BoxGeometry.hpp:47-60)
    d[k] = (fabs(dx) > 0.5 * G.box[k]) ? dx - rint(dx * G.box_i[k]) * G.box[k] : dx;
  }
}

// Adds each particle's bond forces to f (FP64 sums in entry order).
__global__ void k_bond_forces(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                              const double *__restrict__ pos, const int *__restrict__ bstart,
                              const int2 *__restrict__ bent, const BondParam *__restrict__ bp,
                              long long n, double *__restrict__ f, int *__restrict__ err) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  int const s0 = bstart[i], s1 = bstart[i + 1];
  if (s0 == s1)
    return;
  RepGeom const &G = reps[rep_of[i]];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int e = s0; e < s1; ++e) {
    int2 const en = bent[e];
    double d[3];
    bond_vector(G, pos, i, en.x, d);
    double const len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double fac = 0.0, energy = 0.0;
    int const st = bond_eval(bp[en.y], len, fac, energy);
    if (st != 0) {
      bond_report(err, st, static_cast<int>(i), en.x);
      continue;
    }
    fx += fac * d[0];
    fy += fac * d[1];
    fz += fac * d[2];
  }
  f[3 * i + 0] += fx;
  f[3 * i + 1] += fy;
  f[3 * i + 2] += fz;
}

// Bond energy of every particle (half of each of its bonds; a bond is seen
// from both ends), for per-replica sums on the host.
__global__ void k_bond_energy_pp(const RepGeom *__restrict__ reps, const int *__restrict__ rep_of,
                                 const double *__restrict__ pos, const int *__restrict__ bstart,
                                 const int2 *__restrict__ bent, const BondParam *__restrict__ bp,
                                 long long n, double *__restrict__ e_pp, int *__restrict__ err) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  RepGeom const &G = reps[rep_of[i]];
  double acc = 0.0;
  for (int e = bstart[i]; e < bstart[i + 1]; ++e) {
    int2 const en = bent[e];
    double d[3];
    bond_vector(G, pos, i, en.x, d);
    double const len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double fac = 0.0, energy = 0.0;
    int const st = bond_eval(bp[en.y], len, fac, energy);
    if (st != 0) {
      bond_report(err, st, static_cast<int>(i), en.x);
      continue;
    }
    acc += 0.5 * energy;
  }
  e_pp[i] = acc;
}

// Bonded energy and virial (sum over bonds of F (x) d): each bond is seen
// from both ends with the same F (x) d, so every end adds half.  Per-block
// partials[block * 10 + {E, V00..V22}], reduced in a fixed order.
__global__ void k_bond_observables(const RepGeom *__restrict__ reps,
                                   const int *__restrict__ rep_of, const double *__restrict__ pos,
                                   const int *__restrict__ bstart, const int2 *__restrict__ bent,
                                   const BondParam *__restrict__ bp, long long n,
                                   double *__restrict__ partials, int *__restrict__ err) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (i < n) {
    RepGeom const &G = reps[rep_of[i]];
    for (int e = bstart[i]; e < bstart[i + 1]; ++e) {
      int2 const en = bent[e];
      double d[3];
      bond_vector(G, pos, i, en.x, d);
      double const len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      double fac = 0.0, energy = 0.0;
      int const st = bond_eval(bp[en.y], len, fac, energy);
      if (st != 0) {
        bond_report(err, st, static_cast<int>(i), en.x);
        continue;
      }
      acc[0] += 0.5 * energy;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          acc[1 + 3 * r + c] += 0.5 * fac * d[r] * d[c];
    }
  }
  __shared__ double red[10][8];
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0)
      red[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 10) {
    double s = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
      s += red[threadIdx.x][w];
    partials[static_cast<long long>(blockIdx.x) * 10 + threadIdx.x] = s;
  }
}

} // namespace p3mx
