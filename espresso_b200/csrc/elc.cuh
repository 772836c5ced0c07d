// Electrostatic layer correction (ELC) for slab systems: the far-formula
// correction that removes the interactions with the periodic images along z
// from a 3D-periodic P3M solution (electrostatics/elc.cpp), with dielectric
// contrasts at the slab walls and a constant potential difference (their
// image-charge mesh and short-range terms are driven from elc_host.cuh and
// the engine's k_elc_image_pairs).
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
// The sin / cos of a particle's x and y phases at frequency k (the
// reference caches them per particle, calc_sc_cache :107-125) are carried in
// registers from mode to mode: the next frequency is one rotation by the
// unit phase (4 FMA), a new p or a chunk start takes one sincos.  Modes run
// p-major, so a pq-mode block needs one x sincos per p and rotations in q.
//
// Device layout (all FP64):
//   part : per mode m and row c, the sums of every particle tile b,
//          [m * R + c][b] with R = 8 (own products plus image-layer terms)
//          or 16 with contrasts (then 8 more lclimge rows); then the
//          kElcScalars dipole / z sums [nmodes * R + c][b];
//   G    : per mode the 8 sums over all tiles times the mode prefactors,
//          then the kElcScalars scalar sums;
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
  // dielectric contrasts (setup_PoQ :511-518, setup_PQ :651-658)
  double pref_di;       // prefactor * {4, 8} pi / (L_x L_y)
  double fdb, fdt, fd;  // delta_bot fac_elc, delta_top fac_elc, fdb delta_top
  double em2h;          // exp(-2 omega box_h)
};

struct ElcGeom {
  double box[3];
  double box_h;        // L_z - gap
  double shift;        // L_z / 2
  double pref_dip;     // prefactor 4 pi / V (add_dipole_force)
  long long n;
  int nmodes, nfx, nfy, neutralize;
  // dielectric contrasts / constant potential (effective flags of elc_data)
  int contrast, const_pot;
  double sl;            // space_layer
  double db, dt;        // delta_mid_bot, delta_mid_top
  double pot_diff;
  double pref_z;        // prefactor 2 pi / (L_x L_y) (add_z_force)
  double zf[3];         // z-force factors fdb, fdt, fd of add_z_force :446-449
};

// the scalar sums of one evaluation (dipole, z terms), after the mode sums
constexpr int kElcScalars = 12;

constexpr int kElcThreads = 256;
constexpr int kElcPPT = 2;            // particles per thread in the sums kernel
constexpr int kElcModesPerBlock = 16; // modes per block of the sums kernel

__device__ __forceinline__ double elc_fold(double x, double l) { return x - floor(x / l) * l; }

// sin / cos of the phase 2 pi k u x at frequency k, from the state of the
// previous mode: kept (same k), rotated by the unit phase (k - 1), the unit
// phase itself (k = 1) or computed (c2pu = 2 pi u, as the reference forms
// its argument (2 pi u k) x).
struct ElcPhase {
  int k;
  double s, c;
};

__device__ __forceinline__ void elc_phase(ElcPhase &ph, int k, double s1, double c1, double c2pu,
                                          double x) {
  if (ph.k == k)
    return;
  if (ph.k == k - 1) {
    double const sn = ph.s * c1 + ph.c * s1;
    double const cn = ph.c * c1 - ph.s * s1;
    ph.s = sn;
    ph.c = cn;
  } else if (k == 1) {
    ph.s = s1;
    ph.c = c1;
  } else {
    sincos((c2pu * static_cast<double>(k)) * x, &ph.s, &ph.c);
  }
  ph.k = k;
}

// One particle's state: folded position, charge, unit phases and the
// current x / y phases.
struct ElcPart {
  double x, y, z, q;
  double s1x, c1x, s1y, c1y;
  ElcPhase px, py;
};

__device__ __forceinline__ void elc_part_init(ElcPart &P, ElcGeom const &g,
                                              const double *__restrict__ pos, double q) {
  P.x = elc_fold(pos[0], g.box[0]);
  P.y = elc_fold(pos[1], g.box[1]);
  P.z = elc_fold(pos[2], g.box[2]);
  P.q = q;
  sincos((2.0 * kPi * (1.0 / g.box[0])) * P.x, &P.s1x, &P.c1x);
  sincos((2.0 * kPi * (1.0 / g.box[1])) * P.y, &P.s1y, &P.c1y);
  P.px.k = P.py.k = -1;
  P.px.s = P.px.c = P.py.s = P.py.c = 0.0;
}

// the 4 / 8 products of the particle for mode md (e = exp(omega z); the
// reference divides by e, here one reciprocal is multiplied in)
__device__ __forceinline__ int elc_products(ElcMode const &md, ElcGeom const &g, ElcPart &P,
                                            double v[8]) {
  double const e = exp(md.omega * P.z);
  double const ie = 1.0 / e;
  double const q = P.q;
  if (md.kind < 2) {
    double sn, cs;
    if (md.kind == 0) {
      elc_phase(P.px, md.p, P.s1x, P.c1x, 2.0 * kPi * (1.0 / g.box[0]), P.x);
      sn = P.px.s;
      cs = P.px.c;
    } else {
      elc_phase(P.py, md.q, P.s1y, P.c1y, 2.0 * kPi * (1.0 / g.box[1]), P.y);
      sn = P.py.s;
      cs = P.py.c;
    }
    // POQESP, POQECP, POQESM, POQECM
    v[0] = q * sn * e;
    v[1] = q * cs * e;
    v[2] = q * sn * ie;
    v[3] = q * cs * ie;
    return 4;
  }
  elc_phase(P.px, md.p, P.s1x, P.c1x, 2.0 * kPi * (1.0 / g.box[0]), P.x);
  elc_phase(P.py, md.q, P.s1y, P.c1y, 2.0 * kPi * (1.0 / g.box[1]), P.y);
  double const sx = P.px.s, cx = P.px.c, sy = P.py.s, cy = P.py.c;
  // PQESSP, PQESCP, PQECSP, PQECCP, PQESSM, PQESCM, PQECSM, PQECCM
  v[0] = sx * sy * q * e;
  v[1] = sx * cy * q * e;
  v[2] = cx * sy * q * e;
  v[3] = cx * cy * q * e;
  v[4] = sx * sy * q * ie;
  v[5] = sx * cy * q * ie;
  v[6] = cx * sy * q * ie;
  v[7] = cx * cy * q * ie;
  return 8;
}

// sum of v over the block (256 threads) in a fixed order, written by threads
// 0..W-1 to out[c * stride] for c < W; red: scratch of [8 warps][W] doubles.
template <int W>
__device__ __forceinline__ void elc_block_sum(double (&v)[W], double *red, double *out,
                                              long long stride = 1) {
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
    out[threadIdx.x * stride] = s;
  }
  __syncthreads();
}

// Warp sum of 8 values with 9 shuffles: three halving exchanges (lanes
// l and l ^ 16 / 8 / 4 each keep one half of the values and add the half the
// partner sends), then two butterfly steps over l ^ 2, l ^ 1.  Lane l with
// (l & 3) == 0 ends with the warp total of value ((l >> 2) & 7) (bit 4 of l
// selects values 4-7, bit 3 values +2, bit 2 value +1); fixed order.
__device__ __forceinline__ double elc_warp_sum8(double const (&v)[8]) {
  int const lane = threadIdx.x & 31;
  bool const b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  double w[4], x[2];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double const send = b4 ? v[j] : v[j + 4];
    double const keep = b4 ? v[j + 4] : v[j];
    w[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    double const send = b3 ? w[j] : w[j + 2];
    double const keep = b3 ? w[j + 2] : w[j];
    x[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  double y;
  {
    double const send = b2 ? x[0] : x[1];
    double const keep = b2 ? x[1] : x[0];
    y = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  y += __shfl_xor_sync(0xffffffffu, y, 2);
  y += __shfl_xor_sync(0xffffffffu, y, 1);
  return y;
}

// Per particle tile (blockIdx.x) and mode chunk (blockIdx.y): the product sums
// of each mode; chunk 0 also takes the dipole sums and the gap check
// (check_gap :184-194: a charged particle below 0 or above L_z - gap).
template <bool C>
__global__ void __launch_bounds__(kElcThreads)
k_elc_sums(ElcGeom g, const ElcMode *__restrict__ modes, const double *__restrict__ pos,
           const double *__restrict__ qv, double *__restrict__ part, int *__restrict__ gap_err) {
  constexpr int R = C ? 16 : 8; // sums per mode: own (+ image layers), then lclimge
  __shared__ double red[(kElcThreads / 32) * 16];
  // per mode of the chunk, per warp, the R warp sums (one barrier per chunk)
  __shared__ double wsum[kElcModesPerBlock][kElcThreads / 32][R];
  long long const tile0 = static_cast<long long>(blockIdx.x) * kElcThreads * kElcPPT;
  int const lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  ElcPart P[kElcPPT];
#pragma unroll
  for (int k = 0; k < kElcPPT; ++k) {
    long long const i = tile0 + k * kElcThreads + threadIdx.x;
    long long const ic = i < g.n ? i : 0;
    elc_part_init(P[k], g, pos + 3 * ic, i < g.n ? qv[i] : 0.0);
  }
  int const m0 = blockIdx.y * kElcModesPerBlock;
  int const m1 = min(g.nmodes, m0 + kElcModesPerBlock);
  double const h = g.box_h;
  for (int m = m0; m < m1; ++m) {
    ElcMode const md = modes[m];
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double lcl[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < kElcPPT; ++k) {
      // uncharged particles and the tile's tail add zeros (q = 0)
      double v[8];
      int const w = elc_products(md, g, P[k], v);
      for (int c = 0; c < w; ++c)
        acc[c] += v[c];
      if constexpr (C) {
        // image-layer terms (setup_PoQ :542-593, setup_PQ :699-763): the
        // phase products pp (2 or 4) times exp(-+omega z') of the images
        int const np = w >> 1;
        double const q = P[k].q, z = P[k].z;
        double const e = exp(md.omega * z), ie = 1.0 / e;
        double pp[4];
        for (int c = 0; c < np; ++c)
          pp[c] = (q != 0.0) ? v[c] / (q * e) : 0.0;
        bool const mb = z < g.sl, mt = z > h - g.sl;
        double const e2 = mb ? (ie * md.em2h * g.db + e * md.em2h) * md.fd
                             : (ie + e * md.em2h * g.dt) * md.fdb;
        double const e3 = mt ? (e * md.em2h * md.em2h * g.dt + ie * md.em2h) * md.fd
                             : (e * md.em2h + ie * md.em2h * g.db) * md.fdt;
        double const et = mt ? exp(md.omega * (2.0 * h - z)) : 1.0;
        for (int c = 0; c < np; ++c) {
          if (mb) {
            acc[c] += q * g.db * pp[c] * ie;
            acc[np + c] += q * g.db * pp[c] * e;
          }
          if (mt) {
            acc[c] += q * g.dt * pp[c] * et;
            acc[np + c] += q * g.dt * pp[c] / et;
          }
          lcl[c] += pp[c] * q * e2;
          lcl[np + c] += pp[c] * q * e3;
        }
      }
    }
    double const ws = elc_warp_sum8(acc);
    if ((lane & 3) == 0)
      wsum[m - m0][wid][lane >> 2] = ws;
    if constexpr (C) {
      double const wl = elc_warp_sum8(lcl);
      if ((lane & 3) == 0)
        wsum[m - m0][wid][8 + (lane >> 2)] = wl;
    }
  }
  __syncthreads();
  for (int o = threadIdx.x; o < (m1 - m0) * R; o += kElcThreads) {
    int const mm = o / R, c = o % R;
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kElcThreads / 32; ++w)
      t += wsum[mm][w][c];
    part[static_cast<long long>((m0 + mm) * R + c) * gridDim.x + blockIdx.x] = t;
  }
  if (blockIdx.y == 0) {
    // scalar sums (add_dipole_force, dipole_energy, add_z_force, z_energy):
    // 0 q (z - s) + image terms, 1 q z, 2 q + image q, 3 q, 4 image q,
    // 5 q (z - s), 6 image q (z' - s), 7 q (z - s)^2, 8 image q (z' - s)^2,
    // 9 z-force charge sum, 10 z-energy image sum
    double d[kElcScalars] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < kElcPPT; ++k) {
      long long const i = tile0 + k * kElcThreads + threadIdx.x;
      double const q = P[k].q, z = P[k].z;
      if (i < g.n && q != 0.0) {
        double const dz = z - g.shift;
        d[0] += q * dz;
        d[1] += q * z;
        d[2] += q;
        d[3] += q;
        d[5] += q * dz;
        d[7] += q * dz * dz;
        if (z < 0.0 || z > g.box_h)
          atomicMin(gap_err, static_cast<int>(i));
        if constexpr (C) {
          bool const mb = z < g.sl, mt = z > h - g.sl;
          double const zb = -z - g.shift, zt = 2.0 * h - z - g.shift;
          if (mb) {
            d[0] += g.db * q * zb;
            d[2] += g.db * q;
            d[4] += g.db * q;
            d[6] += g.db * q * zb;
            d[8] += g.db * q * zb * zb;
          }
          if (mt) {
            d[0] += g.dt * q * zt;
            d[2] += g.dt * q;
            d[4] += g.dt * q;
            d[6] += g.dt * q * zt;
            d[8] += g.dt * q * zt * zt;
          }
          double const delta = g.dt * g.db;
          if (g.const_pot) {
            double zs = 0.0, z3 = 0.0;
            if (mb) {
              zs -= g.db * q;
              z3 -= g.db * q * zb;
            }
            if (mt) {
              zs += g.dt * q;
              z3 += g.dt * q * zt;
            }
            d[9] += zs;
            d[10] += z3;
          } else {
            double const fdb = g.zf[0], fdt = g.zf[1], fd = g.zf[2];
            double const dci = 1.0 / (1.0 - delta), lz = g.box[2];
            auto ib = [&](double a, double zz) {
              return a * dci * (zz - 2.0 * delta * lz * dci) - a * dci * g.shift;
            };
            auto it = [&](double a, double zz) {
              return a * dci * (zz + 2.0 * delta * lz * dci) - a * dci * g.shift;
            };
            d[9] += mb ? fd * (g.db + 1.0) * q : fdb * (g.dt + 1.0) * q;
            d[9] -= mt ? fd * (g.dt + 1.0) * q : fdt * (g.db + 1.0) * q;
            d[10] += q * (mb ? ib(g.db * delta, -(2.0 * h + z)) + ib(delta, -(2.0 * h - z))
                             : ib(g.db, -z) + ib(delta, -(2.0 * h - z)));
            d[10] -= q * (mt ? it(g.dt * delta, 4.0 * h - z) + it(delta, 2.0 * h + z)
                             : it(g.dt, 2.0 * h - z) + it(delta, 2.0 * h + z));
          }
        }
      }
    }
    long long const nbp = gridDim.x;
    elc_block_sum<kElcScalars>(d, red, part + nbp * g.nmodes * R + blockIdx.x, nbp);
  }
}

// G[m * 8 + c] = pref_m * (sum over tiles) [+ pref_di * (lclimge sum) with
// contrasts], one block per sum, tiles read contiguously and added in a
// fixed order; the kElcScalars scalar sums after them.
template <bool C>
__global__ void __launch_bounds__(kElcThreads)
k_elc_reduce(ElcGeom g, const ElcMode *__restrict__ modes, const double *__restrict__ part,
             int nbp, double *__restrict__ G) {
  constexpr int R = C ? 16 : 8;
  __shared__ double red[kElcThreads / 32];
  __shared__ double out[1];
  int const t = blockIdx.x;
  int const nm8 = g.nmodes * 8;
  long long const r0 = (t < nm8) ? static_cast<long long>(t >> 3) * R + (t & 7)
                                 : static_cast<long long>(g.nmodes) * R + (t - nm8);
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nbp; b += kElcThreads)
    v[0] += part[r0 * nbp + b];
  elc_block_sum<1>(v, red, out);
  if (t >= nm8) {
    if (threadIdx.x == 0)
      G[t] = out[0];
    return;
  }
  double const own = out[0];
  double other = 0.0;
  if constexpr (C) {
    double w[1] = {0.0};
    for (int b = threadIdx.x; b < nbp; b += kElcThreads)
      w[0] += part[(r0 + 8) * nbp + b];
    elc_block_sum<1>(w, red, out);
    other = out[0];
  }
  if (threadIdx.x == 0) {
    ElcMode const md = modes[t >> 3];
    G[t] = C ? md.pref * own + md.pref_di * other : md.pref * own;
  }
}

// Three blocks per SM (80 registers, a few spilled): 0.401 -> 0.367 ms at
// 2^20 ions and 57 modes.  Per particle: the mode forces from the global sums (add_PoQ_force,
// add_PQ_force), the dipole force, and with EV its energy terms
// (PoQ_energy, PQ_energy before the 1 / omega and the final halving).
template <bool EV>
__global__ void __launch_bounds__(kElcThreads, 3)
k_elc_forces(ElcGeom g, const ElcMode *__restrict__ modes, const double *__restrict__ pos,
             const double *__restrict__ qv, const double *__restrict__ G, double *__restrict__ f,
             double *__restrict__ epart) {
  __shared__ double red[(kElcThreads / 32) * 8];
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  double en[1] = {0.0};
  if (i < g.n && qv[i] != 0.0) {
    ElcPart P;
    elc_part_init(P, g, pos + 3 * i, qv[i]);
    double const q = P.q, z = P.z;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    // the mode terms factored as q (1/e A +- e B), A and B the phase
    // products dotted with the mode's sums (the reference's 8-product sums
    // regrouped; q is multiplied in once at the end)
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int m = 0; m < g.nmodes; ++m) {
      ElcMode const md = modes[m];
      double const e = exp(md.omega * z);
      double const ie = 1.0 / e;
      const double *Gm = G + static_cast<long long>(m) * 8;
      if (md.kind < 2) {
        double sn, cs;
        if (md.kind == 0) {
          elc_phase(P.px, md.p, P.s1x, P.c1x, 2.0 * kPi * (1.0 / g.box[0]), P.x);
          sn = P.px.s;
          cs = P.px.c;
        } else {
          elc_phase(P.py, md.q, P.s1y, P.c1y, 2.0 * kPi * (1.0 / g.box[1]), P.y);
          sn = P.py.s;
          cs = P.py.c;
        }
        // G: POQESP, POQECP, POQESM, POQECM
        double const ft = ie * (sn * Gm[1] - cs * Gm[0]) + e * (sn * Gm[3] - cs * Gm[2]);
        if (md.kind == 0)
          ax += ft;
        else
          ay += ft;
        double const a1 = cs * Gm[1] + sn * Gm[0], b1 = cs * Gm[3] + sn * Gm[2];
        az += ie * a1 - e * b1;
        if constexpr (EV)
          en[0] += q * (ie * a1 + e * b1) / md.omega;
      } else {
        elc_phase(P.px, md.p, P.s1x, P.c1x, 2.0 * kPi * (1.0 / g.box[0]), P.x);
        elc_phase(P.py, md.q, P.s1y, P.c1y, 2.0 * kPi * (1.0 / g.box[1]), P.y);
        double const ss = P.px.s * P.py.s, sc = P.px.s * P.py.c;
        double const cs = P.px.c * P.py.s, cc = P.px.c * P.py.c;
        // G: PQESSP, PQESCP, PQECSP, PQECCP, PQESSM, PQESCM, PQECSM, PQECCM
        double const A = cc * Gm[3] + cs * Gm[2] + sc * Gm[1] + ss * Gm[0];
        double const B = cc * Gm[7] + cs * Gm[6] + sc * Gm[5] + ss * Gm[4];
        double const Cx = sc * Gm[3] + ss * Gm[2] - cc * Gm[1] - cs * Gm[0];
        double const Dx = sc * Gm[7] + ss * Gm[6] - cc * Gm[5] - cs * Gm[4];
        double const Cy = cs * Gm[3] + ss * Gm[1] - cc * Gm[2] - sc * Gm[0];
        double const Dy = cs * Gm[7] + ss * Gm[5] - cc * Gm[6] - sc * Gm[4];
        ax += md.px * (ie * Cx + e * Dx);
        ay += md.py * (ie * Cy + e * Dy);
        az += ie * A - e * B;
        if constexpr (EV)
          en[0] += q * (ie * A + e * B) / md.omega;
      }
    }
    fx = q * ax;
    fy = q * ay;
    fz = q * az;
    // dipole force (add_dipole_force :201-264) and the z force of
    // contrasts (add_z_force :441-494) from the scalar sums
    const double *D = G + static_cast<long long>(g.nmodes) * 8;
    double field = g.pref_dip * D[0];
    if (g.const_pot)
      field -= g.pot_diff / g.box_h + g.pref_dip / g.box_h * g.box[2] * D[1];
    fz -= field * q;
    if (!g.neutralize)
      fz += g.pref_dip * D[2] * q * (z - g.shift);
    if (g.contrast)
      fz += g.pref_z * D[9] * q;
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

// Image charges for the mesh (charge_assign :1111-1142): slot i the
// particle (charge kept when bit 0 of which), slot n + i its bottom image
// (x, y, -z) with q delta_bot, slot 2n + i its top image (x, y, 2h - z) with
// q delta_top (bit 1; zero charge outside the space layer); positions folded.
__global__ void k_elc_augment(const double *__restrict__ pos, const double *__restrict__ q,
                              long long n, ElcGeom g, int which, double *__restrict__ apos,
                              double *__restrict__ aq) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double x[3];
  for (int d = 0; d < 3; ++d)
    x[d] = elc_fold(pos[3 * i + d], g.box[d]);
  double const qi = q[i];
  double const h = g.box_h;
  bool const img = (which & 2) && qi != 0.0;
  double const zb = elc_fold(-x[2], g.box[2]), zt = elc_fold(2.0 * h - x[2], g.box[2]);
  for (int d = 0; d < 2; ++d) {
    apos[3 * i + d] = x[d];
    apos[3 * (n + i) + d] = x[d];
    apos[3 * (2 * n + i) + d] = x[d];
  }
  apos[3 * i + 2] = x[2];
  apos[3 * (n + i) + 2] = zb;
  apos[3 * (2 * n + i) + 2] = zt;
  aq[i] = (which & 1) ? qi : 0.0;
  aq[n + i] = (img && x[2] < g.sl) ? g.db * qi : 0.0;
  aq[2 * n + i] = (img && x[2] > h - g.sl) ? g.dt * qi : 0.0;
}

// f[k] += a[k], k < m
__global__ void k_elc_add(double *__restrict__ f, const double *__restrict__ a, long long m) {
  long long const k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k < m)
    f[k] += a[k];
}

} // namespace p3mx
