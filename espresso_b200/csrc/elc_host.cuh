// Host side of the electrostatic layer correction: parameter checks
// (elc_data::elc_data, core/electrostatics/elc.cpp:1056-1102), slab height
// and far-formula cutoff (recalc_box_h :1020-1030, tune_far_cut :942-973),
// the mode table in the reference's loop order (add_force :830-883) and the
// kernel chain of elc.cuh on a caller's stream.
#pragma once

#include "../../include/p3mx.h"
#include "elc.cuh"
#include "engine.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace p3mx {

struct ElcState {
  p3mx_elc_params prm{};
  bool far_calculated = false;
  double far_cut = 0.0, box_h = 0.0, space_layer = 0.0;
  double built_r_cut = -1.0;
  double built_box[3] = {0, 0, 0};
  double built_prefactor = 0.0;
  std::vector<ElcMode> modes;
  int nfx = 0, nfy = 0;
  DevBuf d_modes, d_part, d_G, d_epart, d_err;
  std::vector<double> h_epart;
  // dielectric contrasts: image charges on the mesh through a second FP64
  // engine over 3N slots (particles, bottom images, top images)
  std::unique_ptr<Engine> img;
  const Engine *img_for = nullptr;
  long long img_n = -1;
  DevBuf d_aug_pos, d_aug_q, d_faug;
  bool contrast() const { return prm.delta_mid_top != 0.0 || prm.delta_mid_bot != 0.0; }
  bool const_pot() const { return prm.const_pot && contrast(); }
  bool neutralize() const { return prm.neutralize && !contrast(); }
};

// elc_data::elc_data (elc.cpp:1056-1102): the parameter domains and the
// rule that two metallic walls need const_pot.
inline void elc_validate(p3mx_elc_params const &p) {
  double const delta_range = 1.0 + std::sqrt(1e-14);
  bool const far_calc = (p.far_cut == -1.0);
  if (p.far_cut <= 0.0 && !far_calc)
    throw Error(P3MX_EDOMAIN, "Parameter 'far_cut' must be > 0");
  if (p.maxPWerror <= 0.0)
    throw Error(P3MX_EDOMAIN, "Parameter 'maxPWerror' must be > 0");
  if (p.gap_size <= 0.0)
    throw Error(P3MX_EDOMAIN, "Parameter 'gap_size' must be > 0");
  if (p.pot_diff != 0.0 && !p.const_pot)
    throw Error(P3MX_EDOMAIN, "Parameter 'const_pot' must be True when 'pot_diff' is non-zero");
  if (p.delta_mid_top < -delta_range || p.delta_mid_top > delta_range)
    throw Error(P3MX_EDOMAIN, "Parameter 'delta_mid_top' must be >= -1 and <= +1");
  if (p.delta_mid_bot < -delta_range || p.delta_mid_bot > delta_range)
    throw Error(P3MX_EDOMAIN, "Parameter 'delta_mid_bot' must be >= -1 and <= +1");
  bool const contrast = p.delta_mid_top != 0.0 || p.delta_mid_bot != 0.0;
  double const dt = std::clamp(p.delta_mid_top, -1.0, 1.0);
  double const db = std::clamp(p.delta_mid_bot, -1.0, 1.0);
  if (contrast && !p.const_pot && std::fabs(1.0 - dt * db) < 1e-14)
    throw Error(P3MX_EDOMAIN, "ELC with two parallel metallic boundaries requires the "
                              "const_pot option");
}

// tune_far_cut (elc.cpp:942-973): lz = L_z, or box_h + space_layer with
// dielectric contrasts.
inline double elc_tune_far_cut(double const box[3], double box_h, double max_pw_error,
                               double lz) {
  double const maximal_far_cut = 50.0;
  double const ux = 1.0 / box[0], uy = 1.0 / box[1];
  double const umin = std::min(ux, uy);
  double fc = umin, err;
  do {
    double const pref = 2.0 * kPi * fc;
    double const sum = pref + 2.0 * (ux + uy);
    double const den = -std::expm1(-pref * lz);
    double const num1 = std::exp(pref * (box_h - lz));
    double const num2 = std::exp(-pref * (box_h + lz));
    err = 0.5 / den *
          (num1 * (sum + 1.0 / (lz - box_h)) / (lz - box_h) +
           num2 * (sum + 1.0 / (lz + box_h)) / (lz + box_h));
    fc += umin;
  } while (err > max_pw_error && fc < maximal_far_cut);
  if (fc >= maximal_far_cut)
    throw Error(P3MX_ERUNTIME, "ELC tuning failed: maxPWerror too small");
  return fc - umin;
}

// box_h, far_cut and the mode table for the box and prefactor (again only
// when either changed: on_boxl_change -> recalc_box_h, recalc_far_cut).
inline void elc_prepare(ElcState &s, double const box[3], double prefactor, double r_cut,
                        cudaStream_t st) {
  if (box[0] == s.built_box[0] && box[1] == s.built_box[1] && box[2] == s.built_box[2] &&
      prefactor == s.built_prefactor && r_cut == s.built_r_cut && !s.modes.empty())
    return;
  double const bh = box[2] - s.prm.gap_size;
  if (bh < 0.0) {
    char m[160];
    std::snprintf(m, sizeof m, "ELC gap size (%f) larger than box length in z-direction (%f)",
                  s.prm.gap_size, box[2]);
    throw Error(P3MX_ERUNTIME, m);
  }
  s.box_h = bh;
  s.space_layer = 0.0;
  if (s.contrast()) {
    // recalc_space_layer (elc.cpp:1032-1054)
    double sl = s.prm.gap_size / 3.0;
    double const mx = std::min(s.prm.gap_size - r_cut, bh / 2.0);
    if (sl > mx) {
      if (mx <= 0.0)
        throw Error(P3MX_ERUNTIME, "P3M real-space cutoff too large for ELC w/ dielectric "
                                   "contrast");
      sl = mx;
    }
    s.space_layer = sl;
  }
  double const lz_tune = s.contrast() ? bh + s.space_layer : box[2];
  s.far_cut = s.far_calculated ? elc_tune_far_cut(box, bh, s.prm.maxPWerror, lz_tune)
                               : s.prm.far_cut;
  double const fc = s.far_cut, fc2 = fc * fc;
  double const ux = 1.0 / box[0], uy = 1.0 / box[1];
  s.nfx = static_cast<int>(std::ceil(fc * box[0]) + 1.0);
  s.nfy = static_cast<int>(std::ceil(fc * box[1]) + 1.0);
  double const area_inv = ux * uy;
  s.modes.clear();
  auto add = [&](int kind, int p, int q, double omega) {
    ElcMode m{};
    m.kind = kind;
    m.p = p;
    m.q = q;
    m.omega = omega;
    double const pref_di = prefactor * (kind < 2 ? 4.0 : 8.0) * kPi * area_inv;
    m.pref = -pref_di / std::expm1(omega * box[2]);
    m.pref_di = pref_di;
    double const dt = s.prm.delta_mid_top, db = s.prm.delta_mid_bot;
    double const fac_elc = 1.0 / (1.0 - dt * db * std::exp(-omega * 2.0 * bh));
    m.fdb = db * fac_elc;
    m.fdt = dt * fac_elc;
    m.fd = m.fdb * dt;
    m.em2h = std::exp(-2.0 * omega * bh);
    m.px = 2.0 * kPi * ux * static_cast<double>(p) / omega;
    m.py = 2.0 * kPi * uy * static_cast<double>(q) / omega;
    s.modes.push_back(m);
  };
  for (int p = 1; ux * static_cast<double>(p - 1) < fc && p <= s.nfx; ++p)
    add(0, p, 0, 2.0 * kPi * ux * static_cast<double>(p));
  for (int q = 1; uy * static_cast<double>(q - 1) < fc && q <= s.nfy; ++q)
    add(1, 0, q, 2.0 * kPi * uy * static_cast<double>(q));
  for (int p = 1; ux * static_cast<double>(p - 1) < fc && p <= s.nfx; ++p)
    for (int q = 1; (ux * static_cast<double>(p - 1)) * (ux * static_cast<double>(p - 1)) +
                            (uy * static_cast<double>(q - 1)) * (uy * static_cast<double>(q - 1)) <
                        fc2 &&
                    q <= s.nfy;
         ++q)
      add(2, p, q,
          2.0 * kPi * std::sqrt((ux * p) * (ux * p) + (uy * q) * (uy * q)));
  s.d_modes.ensure(s.modes.size() * sizeof(ElcMode));
  P3MX_CUDA(cudaMemcpyAsync(s.d_modes.p, s.modes.data(), s.modes.size() * sizeof(ElcMode),
                            cudaMemcpyHostToDevice, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  for (int d = 0; d < 3; ++d)
    s.built_box[d] = box[d];
  s.built_prefactor = prefactor;
  s.built_r_cut = r_cut;
}

// Kernel geometry of one ELC evaluation of n particles.
inline ElcGeom elc_geom(ElcState const &s, double const box[3], double prefactor, long long n) {
  ElcGeom g{};
  for (int d = 0; d < 3; ++d)
    g.box[d] = box[d];
  g.box_h = s.box_h;
  g.shift = 0.5 * box[2];
  g.pref_dip = prefactor * 4.0 * kPi / (box[0] * box[1] * box[2]);
  g.n = n;
  g.nmodes = static_cast<int>(s.modes.size());
  g.nfx = s.nfx;
  g.nfy = s.nfy;
  g.neutralize = s.neutralize() ? 1 : 0;
  g.contrast = s.contrast() ? 1 : 0;
  g.const_pot = s.const_pot() ? 1 : 0;
  g.sl = s.space_layer;
  g.db = s.prm.delta_mid_bot;
  g.dt = s.prm.delta_mid_top;
  g.pot_diff = s.prm.const_pot ? s.prm.pot_diff : 0.0;
  g.pref_z = prefactor * 2.0 * kPi / (box[0] * box[1]);
  double const delta = g.dt * g.db;
  if (g.contrast && !g.const_pot) {
    g.zf[0] = g.db / (1.0 - delta);
    g.zf[1] = g.dt / (1.0 - delta);
    g.zf[2] = delta / (1.0 - delta);
  }
  return g;
}

// The three kernels of one evaluation on st; ev (4 events or nullptr) is
// recorded before, between and after them for the stage profile.
inline void elc_launch(ElcState &s, ElcGeom const &g, const double *pos, const double *q,
                       double *f, bool want_e, cudaStream_t st, cudaEvent_t *ev) {
  long long const n = g.n;
  int const nbp = static_cast<int>((n + kElcThreads * kElcPPT - 1) / (kElcThreads * kElcPPT));
  int const nbf = static_cast<int>((n + kElcThreads - 1) / kElcThreads);
  int const R = g.contrast ? 16 : 8;
  s.d_part.ensure(static_cast<size_t>(nbp) * (g.nmodes * R + kElcScalars) * sizeof(double));
  s.d_G.ensure(static_cast<size_t>(g.nmodes * 8 + kElcScalars) * sizeof(double));
  s.d_epart.ensure(static_cast<size_t>(nbf) * sizeof(double));
  s.d_err.ensure(sizeof(int));
  P3MX_CUDA(cudaMemsetAsync(s.d_err.p, 0x7f, sizeof(int), st));
  if (ev)
    P3MX_CUDA(cudaEventRecord(ev[0], st));
  dim3 const gs(nbp, std::max(1, (g.nmodes + kElcModesPerBlock - 1) / kElcModesPerBlock));
  if (g.contrast)
    k_elc_sums<true><<<gs, kElcThreads, 0, st>>>(g, s.d_modes.as<ElcMode>(), pos, q,
                                                 s.d_part.as<double>(), s.d_err.as<int>());
  else
    k_elc_sums<false><<<gs, kElcThreads, 0, st>>>(g, s.d_modes.as<ElcMode>(), pos, q,
                                                  s.d_part.as<double>(), s.d_err.as<int>());
  if (ev)
    P3MX_CUDA(cudaEventRecord(ev[1], st));
  int const nred = g.nmodes * 8 + kElcScalars;
  if (g.contrast)
    k_elc_reduce<true><<<nred, kElcThreads, 0, st>>>(g, s.d_modes.as<ElcMode>(),
                                                     s.d_part.as<double>(), nbp,
                                                     s.d_G.as<double>());
  else
    k_elc_reduce<false><<<nred, kElcThreads, 0, st>>>(g, s.d_modes.as<ElcMode>(),
                                                      s.d_part.as<double>(), nbp,
                                                      s.d_G.as<double>());
  if (ev)
    P3MX_CUDA(cudaEventRecord(ev[2], st));
  if (want_e)
    k_elc_forces<true><<<nbf, kElcThreads, 0, st>>>(g, s.d_modes.as<ElcMode>(), pos, q,
                                                    s.d_G.as<double>(), f, s.d_epart.as<double>());
  else
    k_elc_forces<false><<<nbf, kElcThreads, 0, st>>>(g, s.d_modes.as<ElcMode>(), pos, q,
                                                     s.d_G.as<double>(), f, nullptr);
  if (ev)
    P3MX_CUDA(cudaEventRecord(ev[3], st));
  P3MX_CUDA(cudaGetLastError());
}

// Mean device time (ms) of each ELC kernel over reps evaluations of the
// forces (no energy) into f; names elc_sums, elc_reduce, elc_forces.
inline std::vector<std::pair<std::string, double>>
elc_profile(ElcState &s, double const box[3], double prefactor, double r_cut, long long n,
            const double *pos, const double *q, double *f, int reps, cudaStream_t st) {
  elc_prepare(s, box, prefactor, r_cut, st);
  std::vector<std::pair<std::string, double>> out = {
      {"elc_sums", 0.0}, {"elc_reduce", 0.0}, {"elc_forces", 0.0}};
  if (n == 0)
    return out;
  ElcGeom const g = elc_geom(s, box, prefactor, n);
  cudaEvent_t ev[4];
  for (auto &e : ev)
    P3MX_CUDA(cudaEventCreate(&e));
  for (int r = 0; r < reps; ++r) {
    elc_launch(s, g, pos, q, f, false, st, ev);
    P3MX_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < 3; ++k) {
      float ms = 0.f;
      P3MX_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      out[k].second += ms / reps;
    }
  }
  for (auto &e : ev)
    cudaEventDestroy(e);
  return out;
}

// Adds the ELC forces to f (device, 3n FP64, original particle order) for
// the positions and charges on the device; with energy != nullptr also the
// ELC energy (calc_energy :885-940: dipole + z + mode terms, halved).  Ends
// with a stream synchronisation: a charged particle in the gap raises the
// reference's runtime error (check_gap :184-194), a net charge with
// contrasts the errors of sanity_checks_dielectric_contrasts (:990-1008).
inline void elc_apply(ElcState &s, double const box[3], double prefactor, double r_cut,
                      long long n, const double *pos, const double *q, double *f,
                      double *energy, long long *launches, cudaStream_t st) {
  elc_prepare(s, box, prefactor, r_cut, st);
  if (energy)
    *energy = 0.0;
  if (n == 0)
    return;
  ElcGeom const g = elc_geom(s, box, prefactor, n);
  int const nbf = static_cast<int>((n + kElcThreads - 1) / kElcThreads);
  elc_launch(s, g, pos, q, f, energy != nullptr, st, nullptr);
  if (launches)
    *launches += 3;
  int bad = INT_MAX;
  double D[kElcScalars] = {};
  P3MX_CUDA(cudaMemcpyAsync(&bad, s.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaMemcpyAsync(D, s.d_G.as<double>() + g.nmodes * 8, sizeof D,
                            cudaMemcpyDeviceToHost, st));
  if (energy) {
    s.h_epart.assign(nbf, 0.0);
    P3MX_CUDA(cudaMemcpyAsync(s.h_epart.data(), s.d_epart.p, nbf * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
  }
  P3MX_CUDA(cudaStreamSynchronize(st));
  if (bad >= 0 && bad < n) {
    double zb[3];
    P3MX_CUDA(cudaMemcpy(zb, pos + 3 * static_cast<long long>(bad), sizeof zb,
                         cudaMemcpyDeviceToHost));
    double const z = zb[2] - std::floor(zb[2] / box[2]) * box[2];
    char m[160];
    std::snprintf(m, sizeof m, "Particle %d entered ELC gap region by %g", bad,
                  z < 0.0 ? z : z - s.box_h);
    throw Error(P3MX_ERUNTIME, m);
  }
  if (g.contrast && std::fabs(D[3]) >= std::sqrt(1e-14))
    throw Error(P3MX_ERUNTIME, g.const_pot
                                   ? "ELC does not currently support non-neutral systems with "
                                     "a dielectric contrast."
                                   : "ELC does not work for non-neutral systems and "
                                     "non-metallic dielectric contrast.");
  if (energy) {
    // dipole_energy (elc.cpp:267-343) and z_energy (:366-439) from the
    // scalar sums: s0 q, s1 image q, s2 q (z - s), s3 image q (z' - s),
    // s4 q (z - s)^2, s5 image q (z' - s)^2, s6 q z
    double const lz = box[2], h = s.box_h;
    double const pref = prefactor * 2.0 * kPi / (box[0] * box[1] * box[2]);
    double const s0 = D[3], s1 = D[4], s2 = D[5], s3 = D[6], s4 = D[7], s5 = D[8], s6 = D[1];
    double e = 2.0 * pref * (s2 * s2 + s2 * s3);
    if (!g.neutralize)
      e += 2.0 * pref * (-s0 * s4 - (0.25 - 0.5 / 3.0) * (s0 * lz) * (s0 * lz));
    if (g.contrast) {
      if (g.const_pot) {
        e += pref / h * lz * s6 * s6;
        e -= 2.0 * g.pot_diff / h * s6;
      }
      e += pref * (-(s1 * s4 + s0 * s5) - (1.0 - 2.0 / 3.0) * s0 * s1 * lz * lz);
      e += -g.pref_z * (s2 * D[9] - s0 * D[10]);
    }
    for (double v : s.h_epart)
      e += v;
    *energy = 0.5 * e;
  }
}

} // namespace p3mx
