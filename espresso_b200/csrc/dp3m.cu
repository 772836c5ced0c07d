// Dipolar P3M (magnetostatics/dp3m.cpp, dp3m.hpp, dp3m.impl.hpp) on the
// B200: the actor's C ABI (p3mx_dp3m_*, include/p3mx.h), its tuner
// (DipolarTuningAlgorithm, dp3m.cpp:535-660) and the device pipeline.
//
// Pipeline of one force/torque/energy evaluation (one cubic system):
//  1. k_dp3m_prepare: moment components, list selector, census partials;
//  2. brick binning and sort of the particles (once), weight records with
//     q = mu_d for each component d = x, y, z, the coloured super-brick
//     assignment of all three per colour launch, the r2c z pass of each;
//     one y pass over the three spectra;
//  3. k_fft_x_dp3m in three modes (torque fields with the energy sum, the
//     two halves of the force-field tensor), each followed by the backward
//     y and z passes and the back-interpolation with unit-charge weights;
//  4. k_dp3m_combine: forces and torques from the nine interpolated values;
//  5. the real-space pair kernel over the Verlet lists of the dipoles.
// The charge engine provides steps 2-3's kernels, buffers, block tables,
// FFT plans and the Verlet lists; Dp3mEngine drives them (a friend).
#include "../../include/p3mx.h"
#include "dp3m.cuh"
#include "engine.cuh"

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <limits>
#include <memory>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

namespace p3mx {

class Dp3mEngine {
public:
  explicit Dp3mEngine(bool fp32) : m_eng(fp32) {}

  Engine &engine() { return m_eng; }
  long long n() const { return m_eng.n_part(); }

  // One cubic replica of edge L with mesh M^3.
  void configure(double L, int M, int cao, double alpha, double r_cut, double skin,
                 const double *mesh_off, long long n) {
    ReplicaConf c;
    for (int d = 0; d < 3; ++d) {
      c.box[d] = L;
      c.mesh[d] = M;
      c.mesh_off[d] = mesh_off[d];
    }
    c.prefactor = 1.0; // selects the list range r_cut (the value is unused)
    c.epsilon = 0.0;
    c.cao = cao;
    c.alpha = alpha;
    c.r_cut = r_cut;
    c.skin = skin;
    c.p0 = 0;
    c.np = n;
    if (!m_table_set) {
      // no LJ/WCA: the lists hold the dipole pairs within r_cut + skin
      m_eng.set_pair_table(1, {PairIA{0, 0, 0, 0, 0, 0, 0, 0, 0, -1.0}});
      m_table_set = true;
    }
    m_eng.configure({c}, n);
    cudaStream_t const st = m_eng.stream();
    Engine &E = m_eng;
    size_t const rsz = E.fp32() ? sizeof(float) : sizeof(double);
    size_t const csz = 2 * rsz;
    long long const nn = std::max<long long>(1, n);
    m_mu.ensure(3 * nn * sizeof(double));
    m_comp.ensure(3 * nn * sizeof(double));
    m_out.ensure(9 * nn * sizeof(double));
    m_smu.ensure(nn * sizeof(double4));
    m_ck3.ensure(3 * E.m_cplx * csz);
    m_ge.ensure(E.m_cplx * rsz);
    // three weight-record sets and meshes for the one-launch assignment
    // (+ slack: the z pass stages 16-byte aligned supersets of mesh rows)
    m_W3.ensure(3 * static_cast<size_t>(kRecStride) * nn * rsz);
    m_rho3.ensure(3 * E.m_bins * rsz + 64);
    m_qmax3.ensure(4 * sizeof(unsigned));
    m_gf.ensure(E.m_cplx * rsz);
    long long const nprep = ceil_div(nn, 256);
    size_t const np = std::max<size_t>({static_cast<size_t>(E.m_n_blk_x), 5 * static_cast<size_t>(nprep),
                                        static_cast<size_t>(E.m_n_blk_pair), size_t(kSumBlocks)});
    m_part.ensure(np * sizeof(double));
    m_sums.ensure(8 * sizeof(double));
    m_flag.ensure(sizeof(int));
    // selector and types: all zero until the first upload
    P3MX_CUDA(cudaMemsetAsync(E.m_q.p, 0, nn * sizeof(double), st));
    P3MX_CUDA(cudaMemsetAsync(E.m_type.p, 0, nn * sizeof(int), st));
    // the back-interpolation's geometry: prefactor -V turns its output
    // -prefactor/V sum(w E) into the plain interpolated field
    std::vector<RepGeom> g = E.m_geom;
    for (auto &G : g) {
      G.prefactor = -G.V;
      G.epsilon = 0.0;
    }
    m_geom_interp.ensure(g.size() * sizeof(RepGeom));
    P3MX_CUDA(cudaMemcpyAsync(m_geom_interp.p, g.data(), g.size() * sizeof(RepGeom),
                              cudaMemcpyHostToDevice, st));
    size_t const limit = 220 * 1024;
    auto attr = [limit](auto kern) {
      P3MX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(limit)));
    };
    if (E.fp32()) {
      attr(k_fft_x_dp3m<float, true>);
      attr(k_fft_x_dp3m<float, false>);
    } else {
      attr(k_fft_x_dp3m<double, true>);
      attr(k_fft_x_dp3m<double, false>);
    }
    m_g_valid = false;
    m_phi_valid = false;
    m_M = M;
    m_L = L;
    m_alpha = alpha;
    m_cao = cao;
    P3MX_CUDA(cudaStreamSynchronize(st));
  }

  // Stages positions and moments; returns {n_dipoles, sum mu^2, Mx, My, Mz}
  // (synchronises the stream).  A particle whose moment became zero or
  // non-zero invalidates the Verlet lists.
  std::vector<double> upload(const double *pos, const double *dip, bool dev, cudaStream_t st) {
    Engine &E = m_eng;
    long long const n = E.n_part();
    std::vector<double> census(5, 0.0);
    if (n == 0)
      return census;
    cudaMemcpyKind const k = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    P3MX_CUDA(cudaMemcpyAsync(E.m_pos.p, pos, 3 * n * sizeof(double), k, st));
    P3MX_CUDA(cudaMemcpyAsync(m_mu.p, dip, 3 * n * sizeof(double), k, st));
    P3MX_CUDA(cudaMemsetAsync(m_flag.p, 0, sizeof(int), st));
    int const nb = static_cast<int>(ceil_div(n, 256));
    k_dp3m_prepare<<<nb, 256, 0, st>>>(n, m_mu.as<double>(), m_comp.as<double>(), E.d_q(),
                                       m_flag.as<int>(), m_part.as<double>());
    ++E.m_launches;
    k_dp3m_sum_rows<<<1, 32 * 5, 0, st>>>(m_part.as<double>(), nb, 5, m_sums.as<double>());
    ++E.m_launches;
    int flag = 0;
    P3MX_CUDA(cudaMemcpyAsync(census.data(), m_sums.p, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaMemcpyAsync(&flag, m_flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
    if (flag)
      E.invalidate_lists();
    return census;
  }

  // The k-space part (forces and torques into the scratch fields when
  // want_ft, the mesh energy sum when want_e) for the staged particles.
  template <typename Real> void kspace(bool want_ft, bool want_e, cudaStream_t st) {
    using C = typename CplxOf<Real>::type;
    Engine &E = m_eng;
    long long const n = E.n_part();
    RepGeom const *geom = E.m_geom_d.as<RepGeom>();
    if (!m_g_valid) {
      k_dp3m_influence<Real><<<E.m_n_blk_cplx, 256, 0, st>>>(geom, E.m_blk_cplx.as<int2>(),
                                                             m_ge.as<Real>(), m_gf.as<Real>());
      ++E.m_launches;
      m_g_valid = true;
    }
    // 1. brick binning and sort (shared by the three components)
    P3MX_CUDA(cudaMemsetAsync(E.m_cnt.p, 0, (E.m_nkeys + 2) * sizeof(int), st));
    unsigned *qmax_bits = reinterpret_cast<unsigned *>(E.m_cnt.as<int>() + E.m_nkeys + 1);
    int const nb = static_cast<int>(ceil_div(n, 256));
    k_p3m_bin<Real><<<nb, 256, 0, st>>>(geom, E.m_rep_of.as<int>(), E.d_pos(), n, E.m_key.as<int>(),
                                        E.m_bkey.as<int>(), E.m_slot.as<int>(), E.m_cnt.as<int>(),
                                        E.m_dist.as<Real>());
    ++E.m_launches;
    E.sort_keys(E.m_bkey.as<int>(), E.m_slot.as<int>(), E.m_cnt.as<int>(), E.m_start.as<int>(),
                E.m_perm.as<int>(), E.m_nkeys, st, nullptr, false);
    E.mark("dp_sort", st);
    // 2. the three component meshes: weight records per component, then
    // every colour launch assigns all three (blockIdx.y = component), then
    // the z pass of each
    C const *tw = E.m_tw.as<C>();
    C *ck3 = m_ck3.as<C>();
    long long const wst = static_cast<long long>(kRecStride) * n;
    unsigned *qmax3 = m_qmax3.as<unsigned>();
    P3MX_CUDA(cudaMemsetAsync(qmax3, 0, 3 * sizeof(unsigned), st));
    for (int d = 0; d < 3; ++d) {
      k_p3m_weights<Real><<<nb, 256, 0, st>>>(geom, E.m_perm.as<int>(), E.m_key.as<int>(),
                                              E.m_dist.as<Real>(), m_comp.as<double>() + d * n,
                                              E.m_rep_of.as<int>(), n, m_W3.as<Real>() + d * wst,
                                              E.m_skey.as<int>(), qmax3 + d);
      ++E.m_launches;
    }
    P3MX_CUDA(cudaMemsetAsync(m_rho3.p, 0, 3 * E.m_bins * sizeof(Real), st));
    {
      bool chained = false;
      for (size_t p = 0; p + 1 < E.m_phase_off.size(); ++p) {
        int const cnt = E.m_phase_off[p + 1] - E.m_phase_off[p];
        if (cnt == 0)
          continue;
        int2 const *tab = E.m_blk_mesh.as<int2>() + E.m_phase_off[p];
        P3MX_CAO_DISPATCH_R(E.m_phase_cao[p],
                            (launch_assign<Real, P>(E.m_sb_edge, chained, cnt, st, geom, tab,
                                                    E.m_start.as<int>(), m_W3.as<Real>(),
                                                    E.m_skey.as<int>(), qmax3, m_rho3.as<Real>(),
                                                    E.m_kerr.as<int>(), 3, wst, E.m_bins, 1)));
        chained = true;
        ++E.m_launches;
      }
    }
    for (int d = 0; d < 3; ++d) {
      k_fft_z_fwd<Real><<<E.m_n_blk_zf, 256, E.m_smem_zf, st>>>(
          geom, E.m_blk_zf.as<Blk>(), m_rho3.as<Real>() + d * E.m_bins, ck3 + d * E.m_cplx, tw,
          E.m_kerr.as<int>());
      ++E.m_launches;
    }
    E.mark("dp_assign_fft_z", st);
    E.launch_fft_y<Real>(ck3, E.m_cplx, 3, false, st);
    // unit-charge weights of the magnetic particles (selector) for the
    // back-interpolation
    if (want_ft) {
      k_p3m_weights<Real><<<nb, 256, 0, st>>>(geom, E.m_perm.as<int>(), E.m_key.as<int>(),
                                              E.m_dist.as<Real>(), E.d_q(), E.m_rep_of.as<int>(), n,
                                              E.m_W.as<Real>(), E.m_skey.as<int>(), qmax_bits);
      ++E.m_launches;
    }
    E.mark("dp_fft_y_weights", st);
    // 3. x pass per mode, backward y and z, interpolation
    for (int mode = 0; mode < 3; ++mode) {
      bool const ev = want_e && mode == 0;
      if (!want_ft && !ev)
        break;
      if (ev) {
        k_fft_x_dp3m<Real, true><<<E.m_n_blk_x, 256, E.m_smem_x, st>>>(
            geom, E.m_blk_x.as<Blk>(), ck3, E.m_cplx, m_ge.as<Real>(), m_gf.as<Real>(), mode,
            E.m_field.as<C>(), E.m_tile_x, m_part.as<double>(), tw);
        ++E.m_launches;
        k_dp3m_sum_rows<<<1, 32 * 1, 0, st>>>(m_part.as<double>(), E.m_n_blk_x, 1,
                                          m_sums.as<double>() + 5);
        ++E.m_launches;
      } else {
        k_fft_x_dp3m<Real, false><<<E.m_n_blk_x, 256, E.m_smem_x, st>>>(
            geom, E.m_blk_x.as<Blk>(), ck3, E.m_cplx, m_ge.as<Real>(), m_gf.as<Real>(), mode,
            E.m_field.as<C>(), E.m_tile_x, nullptr, tw);
        ++E.m_launches;
      }
      E.mark("dp_x_pass", st);
      if (!want_ft)
        break;
      E.launch_fft_y<Real>(E.m_field.p, E.m_cplx, 3, true, st);
      k_fft_z_inv3<Real><<<E.m_n_blk_zi, 256, E.m_smem_zi, st>>>(
          geom, E.m_blk_zi.as<Blk>(), E.m_field.as<C>(), E.m_cplx, E.m_E.as<Real>(), tw,
          E.m_kerr.as<int>());
      ++E.m_launches;
      E.mark("dp_inv_yz", st);
      double *out = m_out.as<double>() + 3 * n * mode;
      RepGeom const *gi = m_geom_interp.as<RepGeom>();
      for (int c = 1; n > 0 && c <= 7; ++c) {
        int const nbr = E.m_brick_off[c + 1] - E.m_brick_off[c];
        if (nbr == 0)
          continue;
        int2 const *tab = E.m_blk_brick.as<int2>() + E.m_brick_off[c];
        P3MX_CAO_DISPATCH_R(c, (k_p3m_interp<Real, P><<<interp_grid<Real, P>(nbr),
                                   32 * (1 + kInterpWarps), interp_smem<Real, P>(), st>>>(
                                   gi, tab, nbr, E.m_start.as<int>(), E.m_perm.as<int>(),
                                   E.m_skey.as<int>(), E.m_W.as<Real>(), E.m_E.as<Real>(),
                                   E.m_tmap.as<CUtensorMap>(), E.d_q(), E.m_dipole.as<double>(),
                                   out, 1, E.m_kerr.as<int>())));
        ++E.m_launches;
      }
      E.mark("dp_interp", st);
    }
  }

  // Full evaluation.  f, t: device arrays (3N) or nullptr when not wanted;
  // energies (host): {k-space with its corrections, real space}.
  void compute(double prefactor, double accuracy, double epsilon, double *f, double *t,
               bool overwrite, bool want_e, std::vector<double> const &census, cudaStream_t st,
               double *energies) {
    Engine &E = m_eng;
    long long const n = E.n_part();
    bool const want_ft = (f != nullptr);
    double const sum_mu2 = census[1];
    double const L = m_L, V = L * L * L;
    double const M3 = static_cast<double>(m_M) * m_M * m_M;
    double e_k = 0.0, e_r = 0.0;
    bool const kspace_on = sum_mu2 > 0.0;
    // the Verlet-list check goes ahead of the k-space chain (outside stage
    // profiles), so the host waits for its flag while the GPU is busy
    if (n > 0 && (want_ft || want_e) && !E.m_profiling)
      E.check_lists(st, true);
    try {
      if (kspace_on && (want_ft || want_e)) {
        if (E.fp32())
          kspace<float>(want_ft, want_e, st);
        else
          kspace<double>(want_ft, want_e, st);
      }
    } catch (...) {
      E.m_check_pending = false;
      throw;
    }
    double const ps = (epsilon != 0.0) ? prefactor * 4.0 * kPi / V / (2.0 * epsilon + 1.0) : 0.0;
    if (want_ft && n > 0) {
      if (kspace_on) {
        double const wn = 2.0 * kPi / L;
        double const pt = prefactor / M3 * wn, pf = prefactor / M3 * wn * wn;
        double const *o = m_out.as<double>();
        k_dp3m_combine<<<static_cast<int>(ceil_div(n, 256)), 256, 0, st>>>(
            n, m_mu.as<double>(), o, o + 3 * n, o + 6 * n, pt, pf, ps, m_sums.as<double>(), f, t,
            overwrite ? 1 : 0);
        ++E.m_launches;
        E.mark("dp_combine", st);
      } else if (overwrite) {
        P3MX_CUDA(cudaMemsetAsync(f, 0, 3 * n * sizeof(double), st));
        P3MX_CUDA(cudaMemsetAsync(t, 0, 3 * n * sizeof(double), st));
      }
    }
    // real space over the Verlet lists (the selector keeps the non-magnetic
    // particles out of them)
    if (n > 0 && (want_ft || want_e)) {
      E.prepare_short_range(st, true);
      bool const rel = E.fp32();
      k_dp3m_sort_mu<<<static_cast<int>(ceil_div(n, 256)), 256, 0, st>>>(
          n, E.m_cperm.as<int>(), m_mu.as<double>(), m_smu.as<double4>(), rel ? 1 : 0);
      ++E.m_launches;
      E.mark("dp_sort_mu", st);
      int const exact = accuracy > 5e-6 ? 0 : 1;
      RepGeom const *geom = E.m_geom_d.as<RepGeom>();
      // FP32-mesh mode: the pair terms in FP32 on the cell-relative offsets
      auto pairs = [&](auto ev, double *fo, double *part) {
        constexpr bool EV = decltype(ev)::value;
        if (rel)
          k_dp3m_pairs_rel<EV><<<E.m_n_blk_pair, 256, 0, st>>>(
              geom, E.m_blk_pair.as<int2>(), E.m_spf.as<float4>(), m_smu.as<float4>(),
              E.m_cperm.as<int>(), E.m_nb.as<int>(), E.m_nb_cnt.as<int>(), prefactor, exact, fo,
              t, 0, part);
        else
          k_dp3m_pairs<EV><<<E.m_n_blk_pair, 256, 0, st>>>(
              geom, E.m_blk_pair.as<int2>(), E.m_spq.as<double4>(), m_smu.as<double4>(),
              E.m_cperm.as<int>(), E.m_nb.as<int>(), E.m_nb_cnt.as<int>(), prefactor, exact, fo,
              t, 0, part);
        ++E.m_launches;
      };
      if (want_e) {
        pairs(std::true_type{}, want_ft ? f : nullptr, m_part.as<double>());
        k_dp3m_sum_rows<<<1, 32 * 1, 0, st>>>(m_part.as<double>(), E.m_n_blk_pair, 1,
                                          m_sums.as<double>() + 6);
        ++E.m_launches;
      } else {
        pairs(std::false_type{}, f, nullptr);
      }
      E.mark("dp_pairs", st);
    }
    P3MX_CUDA(cudaGetLastError());
    if (want_e) {
      double s[2] = {0.0, 0.0};
      P3MX_CUDA(cudaMemcpyAsync(s, m_sums.as<double>() + 5, 2 * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
      P3MX_CUDA(cudaStreamSynchronize(st));
      if (kspace_on) {
        // long_range_kernel (dp3m.cpp:268-310): mesh sum, self energy,
        // Madelung-self correction (calc_energy_correction, :800-810)
        e_k = s[0] * prefactor / M3 * kPi / L;
        e_k -= prefactor * sum_mu2 / std::sqrt(kPi) * (2.0 / 3.0) * std::pow(m_alpha, 3);
        double const phi = self_sum(st);
        double const uk = phi / (3.0 * L * M3) * kPi * V;
        double const aL = m_alpha * L;
        double const e_self = -2.0 * aL * aL * aL / std::sqrt(kPi) / 3.0;
        e_k += prefactor * (-sum_mu2 * (uk + e_self + 2.0 * kPi / 3.0)) / V;
      }
      if (ps != 0.0) {
        double const Mx = census[2], My = census[3], Mz = census[4];
        e_k += 0.5 * ps * (Mx * Mx + My * My + Mz * Mz);
      }
      e_r = (n > 0) ? s[1] : 0.0;
    }
    E.check_kernel_error(st);
    if (energies) {
      energies[0] = e_k;
      energies[1] = e_r;
    }
  }

  // Per-stage device times (ms, mean of reps) of one force and torque
  // evaluation of the staged particles, from CUDA events between stages.
  std::vector<std::pair<std::string, double>> profile(double prefactor, double accuracy,
                                                      double epsilon,
                                                      std::vector<double> const &census,
                                                      double *f, double *t, int reps,
                                                      cudaStream_t st) {
    Engine &E = m_eng;
    std::vector<std::pair<std::string, double>> acc;
    for (int r = 0; r < reps; ++r) {
      E.m_marks.clear();
      E.m_profiling = true;
      E.mark("start", st);
      compute(prefactor, accuracy, epsilon, f, t, true, false, census, st, nullptr);
      E.m_profiling = false;
      P3MX_CUDA(cudaStreamSynchronize(st));
      for (size_t k = 1; k < E.m_marks.size(); ++k) {
        float ms = 0.f;
        P3MX_CUDA(cudaEventElapsedTime(&ms, E.m_marks[k - 1].second, E.m_marks[k].second));
        std::string const &name = E.m_marks[k].first;
        auto it = std::find_if(acc.begin(), acc.end(), [&](auto const &p) { return p.first == name; });
        if (it == acc.end())
          acc.emplace_back(name, ms / reps);
        else
          it->second += ms / reps;
      }
      for (auto &m : E.m_marks)
        cudaEventDestroy(m.second);
      E.m_marks.clear();
    }
    return acc;
  }

  // sum over the full mesh of G_energy U2s |d_op|^2 (cached per geometry).
  double self_sum(cudaStream_t st) {
    if (!m_phi_valid) {
      k_dp3m_self_sum<<<kSumBlocks, 256, 0, st>>>(m_M, m_L, m_alpha, m_cao, m_part.as<double>());
      ++m_eng.m_launches;
      k_dp3m_sum_rows<<<1, 32 * 1, 0, st>>>(m_part.as<double>(), kSumBlocks, 1, m_sums.as<double>() + 7);
      ++m_eng.m_launches;
      P3MX_CUDA(cudaMemcpyAsync(&m_phi, m_sums.as<double>() + 7, sizeof(double),
                                cudaMemcpyDeviceToHost, st));
      P3MX_CUDA(cudaStreamSynchronize(st));
      m_phi_valid = true;
    }
    return m_phi;
  }

  static constexpr int kSumBlocks = 296;

private:
  Engine m_eng;
  DevBuf m_mu, m_comp, m_out, m_smu, m_ck3, m_ge, m_gf, m_part, m_sums, m_flag, m_geom_interp;
  DevBuf m_W3, m_rho3, m_qmax3;
  bool m_g_valid = false, m_phi_valid = false, m_table_set = false;
  double m_phi = 0.0;
  int m_M = 0, m_cao = 0;
  double m_L = 0.0, m_alpha = 0.0;
};

namespace {

// dp3m_real_space_error (dp3m.cpp:745-775): eq. (33) of Wang & Holm 2001.
double dp3m_rs_error(double L, double r_cut_iL, int n_c, double sum_mu2, double alpha_L) {
  double const rc = r_cut_iL * L, rc2 = rc * rc, rc4 = rc2 * rc2;
  double const a2 = alpha_L * alpha_L / (L * L);
  double const c = sum_mu2 * std::exp(-a2 * rc2);
  double const cc = 4.0 * a2 * a2 * rc2 * rc2 + 6.0 * a2 * rc2 + 3.0;
  double const dc = 8.0 * a2 * a2 * a2 * rc2 * rc2 * rc2 + 20.0 * a2 * a2 * rc4 + 30.0 * a2 * rc2 + 15.0;
  double const con = 1.0 / std::sqrt(L * L * L * a2 * a2 * rc * rc4 * rc4 * static_cast<double>(n_c));
  return c * con * std::sqrt((13.0 / 6.0) * cc * cc + (2.0 / 15.0) * dc * dc - (13.0 / 15.0) * cc * dc);
}

// dp3m_rtbisection (dp3m.cpp:780-820): alpha_L where the real-space error
// equals accuracy / sqrt(2), bracketed by [x1, x2], to +-xacc.
double dp3m_rtbisection(double L, double r_cut_iL, int n_c, double sum_mu2, double x1, double x2,
                        double xacc, double accuracy) {
  double const target = accuracy / std::sqrt(2.0);
  double const f1 = dp3m_rs_error(L, r_cut_iL, n_c, sum_mu2, x1) - target;
  double const f2 = dp3m_rs_error(L, r_cut_iL, n_c, sum_mu2, x2) - target;
  if (f1 * f2 >= 0.0)
    throw Error(P3MX_ERUNTIME, "Root must be bracketed for bisection in dp3m_rtbisection");
  double dx, rtb;
  if (f1 < 0.0) {
    dx = x2 - x1;
    rtb = x1;
  } else {
    dx = x1 - x2;
    rtb = x2;
  }
  for (int j = 1; j <= 40; ++j) {
    dx *= 0.5;
    double const xmid = rtb + dx;
    double const fmid = dp3m_rs_error(L, r_cut_iL, n_c, sum_mu2, xmid) - target;
    if (fmid <= 0.0)
      rtb = xmid;
    if (std::fabs(dx) < xacc || fmid == 0.0)
      return rtb;
  }
  throw Error(P3MX_ERUNTIME, "Too many bisections in dp3m_rtbisection");
}

} // namespace
} // namespace p3mx

using namespace p3mx;

struct p3mx_dp3m {
  p3mx_dp3m_params prm{};
  p3mx_system sys{};
  bool sys_set = false;
  int mesh = -1, cao = -1;
  double r_cut = 0, alpha = 0, accuracy = 0, mesh_off[3] = {0.5, 0.5, 0.5};
  double r_cut_iL = 0, alpha_L = 0;
  bool is_tuned = false, activated = false;
  double rs_err = 0, ks_err = 0;
  size_t n = 0;
  int n_dip = 0;
  double sum_mu2 = 0;
  std::vector<double> census;
  std::unique_ptr<Dp3mEngine> de;
  DevBuf ks_part; // k-space error partials of the tuner
  DevBuf scratch; // device copies of host inputs / outputs
  std::string err;
};

namespace {

template <typename F> int dp_guarded(p3mx_dp3m *h, F &&fn) {
  if (!h)
    return P3MX_EHANDLE;
  try {
    fn();
    h->err.clear();
    return P3MX_OK;
  } catch (Error const &e) {
    h->err = e.what();
    return e.code;
  } catch (std::exception const &e) {
    h->err = e.what();
    return P3MX_ERUNTIME;
  }
}

// In the reference's order: the P3MParameters checks
// (p3m/common.hpp:95-150), the DipolarP3MImpl constructor's
// (dp3m.impl.hpp:85-92), then Actor::set_prefactor's.
void dp_validate(p3mx_dp3m_params const &p) {
  bool const tuning = p.tune != 0;
  if (p.epsilon < 0.)
    throw Error(P3MX_EDOMAIN, "Parameter 'epsilon' must be >= 0");
  if (p.accuracy <= 0.)
    throw Error(P3MX_EDOMAIN, "Parameter 'accuracy' must be > 0");
  if (p.r_cut <= 0. && !(tuning && p.r_cut == -1.))
    throw Error(P3MX_EDOMAIN, "Parameter 'r_cut' must be > 0");
  if (p.alpha <= 0. && !(tuning && p.alpha == -1.))
    throw Error(P3MX_EDOMAIN, "Parameter 'alpha' must be > 0");
  bool const all_pos = p.mesh[0] >= 1 && p.mesh[1] >= 1 && p.mesh[2] >= 1;
  bool const first_only = p.mesh[0] >= 1 && p.mesh[1] == -1 && p.mesh[2] == -1;
  bool const all_tune = tuning && p.mesh[0] == -1 && p.mesh[1] == -1 && p.mesh[2] == -1;
  if (!(all_pos || first_only || all_tune))
    throw Error(P3MX_EDOMAIN, "Parameter 'mesh' must be > 0");
  bool const off_ok = p.mesh_off[0] >= 0. && p.mesh_off[0] <= 1. && p.mesh_off[1] >= 0. &&
                      p.mesh_off[1] <= 1. && p.mesh_off[2] >= 0. && p.mesh_off[2] <= 1.;
  bool const off_default = p.mesh_off[0] == -1. && p.mesh_off[1] == -1. && p.mesh_off[2] == -1.;
  if (!off_ok && !off_default)
    throw Error(P3MX_EDOMAIN, "Parameter 'mesh_off' must be >= 0 and <= 1");
  if ((p.cao < 1 || p.cao > 7) && (!tuning || p.cao != -1))
    throw Error(P3MX_EDOMAIN, "Parameter 'cao' must be >= 1 and <= 7");
  if (!tuning && (p.cao > p.mesh[0] || p.cao > p.mesh[1] || p.cao > p.mesh[2]))
    throw Error(P3MX_EDOMAIN, "Parameter 'cao' cannot be larger than 'mesh'");
  if (p.timings <= 0)
    throw Error(P3MX_EDOMAIN, "Parameter 'timings' must be > 0");
  if (!(p.mesh[0] == p.mesh[1] && p.mesh[1] == p.mesh[2]))
    throw Error(P3MX_EDOMAIN, "DipolarP3M requires a cubic mesh");
  if (p.prefactor <= 0.)
    throw Error(P3MX_EDOMAIN, "Parameter 'prefactor' must be > 0");
}

bool dp_mesh_ok(int m) {
  if (m < 2 || (m % 2))
    return false;
  int x = m;
  for (int p = 2; p <= 31; ++p)
    while (x % p == 0)
      x /= p;
  return x == 1;
}

// sanity_checks_boxl (dp3m.cpp:822-846) and the FFT's supported sizes.
void dp_sanity_checks(p3mx_dp3m *h) {
  double const *box = h->sys.box;
  for (int i = 0; i < 3; ++i) {
    double const cao_cut = (static_cast<double>(h->cao) / 2.0) * (box[i] / h->mesh);
    if (cao_cut >= 0.5 * box[i]) {
      std::ostringstream m;
      m << "dipolar P3M_init: k-space cutoff " << cao_cut
        << " is larger than half of box dimension " << box[i];
      throw Error(P3MX_ERUNTIME, m.str());
    }
  }
  if (box[0] != box[1] || box[1] != box[2])
    throw Error(P3MX_ERUNTIME, "DipolarP3M: requires a cubic box");
  if (!dp_mesh_ok(h->mesh))
    throw Error(P3MX_EDOMAIN, "mesh " + std::to_string(h->mesh) +
                                  " is not supported by the FFT (even sizes with prime factors <= 31)");
}

void dp_configure(p3mx_dp3m *h) {
  bool const fp32 = h->prm.single_precision != 0;
  if (!h->de || h->de->engine().fp32() != fp32)
    h->de = std::make_unique<Dp3mEngine>(fp32);
  h->de->configure(h->sys.box[0], h->mesh, h->cao, h->alpha, h->r_cut, h->sys.skin, h->mesh_off,
                   static_cast<long long>(h->n));
}

// dp3m_k_space_error (dp3m.cpp:700-740): the mesh sum on the device, the
// prefactor 8 pi^2 / 3 sum mu^2 sqrt(sum / N_dip) / L^4 on the host.
double dp_ks_error(p3mx_dp3m *h, int M, int cao, double alpha_L) {
  cudaStream_t const st = nullptr;
  int const nblk = Dp3mEngine::kSumBlocks;
  h->ks_part.ensure((nblk + 1) * sizeof(double));
  k_dp3m_ks_error<<<nblk, 256, 0, st>>>(M, cao, alpha_L, h->ks_part.as<double>());
  k_dp3m_sum_rows<<<1, 32 * 1, 0, st>>>(h->ks_part.as<double>(), nblk, 1, h->ks_part.as<double>() + nblk);
  double he_q = 0.0;
  P3MX_CUDA(cudaGetLastError());
  P3MX_CUDA(cudaMemcpyAsync(&he_q, h->ks_part.as<double>() + nblk, sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  double const L = h->sys.box[0];
  return 8.0 * kPi * kPi / 3.0 * h->sum_mu2 * std::sqrt(he_q / std::max(1, h->n_dip)) /
         (L * L * L * L);
}

constexpr double kDpCaoTooLarge = 1.0;  // TuningAlgorithm.cpp:47-51
constexpr double kDpAccTooLarge = 3.0;
constexpr double kDpRcutPrec = 1e-3;    // P3M_RCUT_PREC
constexpr double kDpTimeGranularity = 2.0;
constexpr int kDpMaxTrials = 20;

// DipolarTuningAlgorithm (dp3m.cpp:535-660) on the generic search of
// TuningAlgorithm (p3m/TuningAlgorithm.cpp): mesh from the heuristic
// minimum to 128 in steps of 2, cao from 3, r_cut by bisection on the error
// estimate, each candidate timed with CUDA events on full evaluations
// (forces, torques; k-space and real space).
struct DpTuner {
  p3mx_dp3m *h;
  const double *pos, *dip;
  bool dev;
  double rc_min = 0, rc_max = 0;
  int cao_min = 1, cao_max = 7, cao_best = 3;
  int mesh_min = 0, mesh_max = 0;
  size_t n_trials = 0;

  std::tuple<double, double, double, double> accuracy(int mesh, int cao, double r_cut_iL) {
    double const L = h->sys.box[0];
    double rs = dp3m_rs_error(L, r_cut_iL, h->n_dip, h->sum_mu2, 0.001);
    double alpha_L;
    if (std::sqrt(2.0) * rs > h->prm.accuracy)
      alpha_L = dp3m_rtbisection(L, r_cut_iL, h->n_dip, h->sum_mu2, 0.0001 * L, 5.0 * L, 0.0001,
                                 h->prm.accuracy);
    else
      alpha_L = 0.1;
    rs = dp3m_rs_error(L, r_cut_iL, h->n_dip, h->sum_mu2, alpha_L);
    double const ks = dp_ks_error(h, mesh, cao, alpha_L);
    return {std::hypot(rs, ks), rs, ks, alpha_L};
  }

  void commit(int mesh, int cao, double r_cut_iL, double alpha_L) {
    double const L = h->sys.box[0];
    h->r_cut = r_cut_iL * L;
    h->r_cut_iL = r_cut_iL;
    h->cao = cao;
    h->alpha_L = alpha_L;
    h->alpha = alpha_L / L;
    h->mesh = mesh;
  }

  double benchmark() {
    dp_configure(h);
    Dp3mEngine &de = *h->de;
    Engine &e = de.engine();
    cudaStream_t const st = e.stream();
    auto const census = de.upload(pos, dip, dev, st);
    long long const n = de.n();
    h->scratch.ensure(6 * std::max<long long>(1, n) * sizeof(double));
    double *f = h->scratch.as<double>(), *t = f + 3 * n;
    de.compute(h->prm.prefactor, h->accuracy, h->prm.epsilon, f, t, true, false, census, st,
               nullptr);
    cudaEvent_t t0, t1;
    P3MX_CUDA(cudaEventCreate(&t0));
    P3MX_CUDA(cudaEventCreate(&t1));
    int const timings = std::max(1, h->prm.timings);
    P3MX_CUDA(cudaEventRecord(t0, st));
    for (int k = 0; k < timings; ++k)
      de.compute(h->prm.prefactor, h->accuracy, h->prm.epsilon, f, t, true, false, census, st,
                 nullptr);
    P3MX_CUDA(cudaEventRecord(t1, st));
    P3MX_CUDA(cudaEventSynchronize(t1));
    float ms = 0.f;
    P3MX_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return static_cast<double>(ms) / timings;
  }

  double get_mc_time(int mesh, int cao, double &t_rc, double &t_al, double &t_acc) {
    double const L = h->sys.box[0];
    double const skin = h->sys.skin;
    double const k_cut = (static_cast<double>(cao) / 2.) * L / mesh;
    if (cao >= mesh || k_cut >= L - skin || !dp_mesh_ok(mesh))
      return -kDpCaoTooLarge;
    double rs, ks;
    std::tie(t_acc, rs, ks, t_al) = accuracy(mesh, cao, rc_max);
    if (t_acc > h->prm.accuracy)
      return -kDpAccTooLarge;
    double lo = rc_min, hi = rc_max;
    for (;;) {
      double const rc = 0.5 * (lo + hi);
      if (hi - lo < kDpRcutPrec)
        break;
      double acc;
      std::tie(acc, rs, ks, t_al) = accuracy(mesh, cao, rc);
      if (acc > h->prm.accuracy)
        lo = rc;
      else
        hi = rc;
    }
    t_rc = hi;
    // the real-space cutoff plus skin must fit the cell system
    if (t_rc * L + skin > 0.5 * L)
      return -kDpAccTooLarge;
    std::tie(t_acc, rs, ks, t_al) = accuracy(mesh, cao, t_rc);
    commit(mesh, cao, t_rc, t_al);
    double const t = benchmark();
    if (h->prm.verbose)
      std::printf("%-4d %-3d %.5e %.5e %.3e %.3e %.3e %-8.4f\n", mesh, cao, t_rc, t_al, t_acc, rs,
                  ks, t);
    ++n_trials;
    return t;
  }

  double get_m_time(int mesh, int &t_cao, double &t_rc, double &t_al, double &t_acc) {
    double best = -1., rc = 0., al = 0., acc = 0.;
    int final_dir = 0;
    int cao = t_cao;
    double tmp;
    do {
      tmp = get_mc_time(mesh, cao, rc, al, acc);
      if (tmp == -kDpCaoTooLarge)
        return tmp;
      if (tmp >= 0.) {
        best = tmp;
        t_rc = rc;
        t_al = al;
        t_acc = acc;
        t_cao = cao;
        break;
      }
      cao++;
      final_dir = 1;
    } while (cao <= cao_max);
    if (cao > cao_max)
      return -kDpCaoTooLarge;
    if (cao == cao_min)
      final_dir = 1;
    else if (cao == cao_max)
      final_dir = -1;
    if (final_dir == 0) {
      double dir_times[3] = {0, 0, 0};
      for (final_dir = -1; final_dir <= 1; final_dir += 2) {
        dir_times[final_dir + 1] = tmp = get_mc_time(mesh, cao + final_dir, rc, al, acc);
        if (tmp < 0.)
          continue;
        if (tmp < best) {
          best = tmp;
          t_rc = rc;
          t_al = al;
          t_acc = acc;
          t_cao = cao + final_dir;
        }
      }
      if (dir_times[0] == best) {
        final_dir = -1;
      } else if (dir_times[2] == best) {
        final_dir = 1;
      } else {
        if ((dir_times[0] >= 0 && dir_times[0] < best + kDpTimeGranularity) &&
            (dir_times[2] < 0 || dir_times[2] > dir_times[0]))
          final_dir = -1;
        else if ((dir_times[2] >= 0 && dir_times[2] < best + kDpTimeGranularity) &&
                 (dir_times[0] < 0 || dir_times[0] > dir_times[2]))
          final_dir = 1;
        else
          return best;
      }
      cao += 2 * final_dir;
    } else {
      cao += final_dir;
    }
    for (; cao >= cao_min && cao <= cao_max; cao += final_dir) {
      tmp = get_mc_time(mesh, cao, rc, al, acc);
      if (tmp < 0.)
        break;
      if (tmp < best) {
        best = tmp;
        t_rc = rc;
        t_al = al;
        t_acc = acc;
        t_cao = cao;
      } else if (tmp > best + kDpTimeGranularity) {
        break;
      }
    }
    return best;
  }

  void run() {
    double const L = h->sys.box[0];
    // determine_r_cut_limits (TuningAlgorithm.cpp:57-74)
    if (h->r_cut_iL == 0.) {
      rc_min = 0.;
      rc_max = (L / 2. - h->sys.skin) / L;
    } else {
      rc_min = rc_max = h->r_cut_iL;
    }
    // determine_cao_limits(3)
    if (h->cao == -1) {
      cao_min = 1;
      cao_max = 7;
      cao_best = 3;
    } else {
      cao_min = cao_max = cao_best = h->cao;
    }
    // determine_mesh_limits (dp3m.cpp:600-615)
    if (h->mesh == -1) {
      double const expo = std::log(std::cbrt(static_cast<double>(h->n_dip))) / std::log(2.);
      mesh_min = static_cast<int>(std::round(std::pow(2., std::floor(expo))));
      mesh_max = 128;
    } else {
      mesh_min = mesh_max = h->mesh;
    }
    if (h->prm.verbose) {
      std::printf("DipolarP3M tune parameters: Accuracy goal = %.5e prefactor = %.5e\n",
                  h->prm.accuracy, h->prm.prefactor);
      std::printf("System: box_l = %.5e # dipolar part = %d Sum[mu_i^2] = %.5e\n", L, h->n_dip,
                  h->sum_mu2);
      std::printf("mesh cao r_cut_iL    alpha_L     err       rs_err    ks_err    time [ms]\n");
    }
    // get_time (dp3m.cpp:617-645)
    struct {
      int mesh = -1, cao = -1;
      double alpha_L = -1, r_cut_iL = -1, accuracy = -1;
      double time = std::numeric_limits<double>::max();
    } best;
    for (int m = mesh_min; m <= mesh_max; m += 2) {
      int tcao = cao_best;
      double trc = 0, tal = 0, tacc = 0;
      double const t = get_m_time(m, tcao, trc, tal, tacc);
      if (t < 0.)
        continue;
      rc_max = trc;
      if (t < best.time) {
        n_trials = 0;
        best.mesh = m;
        best.cao = tcao;
        best.r_cut_iL = trc;
        best.alpha_L = tal;
        best.accuracy = tacc;
        best.time = t;
      } else if (t > best.time + kDpTimeGranularity || n_trials > static_cast<size_t>(kDpMaxTrials)) {
        break;
      }
    }
    if (best.time == std::numeric_limits<double>::max())
      throw Error(P3MX_ERUNTIME, "DipolarP3M: failed to reach requested accuracy");
    h->accuracy = best.accuracy;
    commit(best.mesh, best.cao, best.r_cut_iL, best.alpha_L);
    if (h->prm.verbose)
      std::printf("\nresulting parameters: mesh: (%d, %d, %d), cao: %d, r_cut_iL: %.4e,\n"
                  "                      alpha_L: %.4e, accuracy: %.4e, time: %.2f\n",
                  best.mesh, best.mesh, best.mesh, best.cao, best.r_cut_iL, best.alpha_L,
                  best.accuracy, best.time);
  }
};

// count_magnetic_particles (dp3m.cpp:160-175) on the host copy of the moments.
void dp_census(p3mx_dp3m *h, size_t n, const double *dip, bool dev) {
  std::vector<double> m(3 * n);
  if (n) {
    if (dev)
      P3MX_CUDA(cudaMemcpy(m.data(), dip, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
    else
      std::copy(dip, dip + 3 * n, m.begin());
  }
  h->n_dip = 0;
  h->sum_mu2 = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double const s = m[3 * i] * m[3 * i] + m[3 * i + 1] * m[3 * i + 1] + m[3 * i + 2] * m[3 * i + 2];
    if (s != 0.0) {
      h->n_dip++;
      h->sum_mu2 += s;
    }
  }
}

} // namespace

extern "C" {

int p3mx_dp3m_create(const p3mx_dp3m_params *params, p3mx_dp3m **out) {
  if (!params || !out)
    return P3MX_EHANDLE;
  *out = nullptr;
  auto h = std::make_unique<p3mx_dp3m>();
  h->prm = *params;
  try {
    dp_validate(h->prm);
  } catch (Error const &e) {
    h->err = e.what();
    *out = h.release();
    return e.code;
  }
  h->mesh = params->mesh[0];
  for (int d = 0; d < 3; ++d)
    h->mesh_off[d] = (params->mesh_off[d] == -1.) ? 0.5 : params->mesh_off[d];
  h->cao = params->cao;
  h->r_cut = params->r_cut == -1. ? 0. : params->r_cut;
  h->alpha = params->alpha == -1. ? 0. : params->alpha;
  h->accuracy = params->accuracy;
  h->is_tuned = !params->tune;
  *out = h.release();
  return P3MX_OK;
}

void p3mx_dp3m_destroy(p3mx_dp3m *h) { delete h; }

const char *p3mx_dp3m_last_error(const p3mx_dp3m *h) { return h ? h->err.c_str() : "NULL handle"; }

int p3mx_dp3m_set_system(p3mx_dp3m *h, const p3mx_system *sys) {
  return dp_guarded(h, [&] {
    if (!sys)
      throw Error(P3MX_EDOMAIN, "system descriptor is NULL");
    for (int d = 0; d < 3; ++d)
      if (!(sys->box[d] > 0.))
        throw Error(P3MX_EDOMAIN, "box_l must be > 0");
    if (sys->skin < 0.)
      throw Error(P3MX_EDOMAIN, "Parameter 'skin' must be >= 0");
    h->sys = *sys;
    h->sys_set = true;
    if (h->activated) {
      // scaleby_box_l (dp3m.cpp:880-893): r_cut and alpha follow the box
      h->r_cut = h->r_cut_iL * h->sys.box[0];
      h->alpha = h->alpha_L / h->sys.box[0];
      dp_sanity_checks(h);
      dp_configure(h);
    }
  });
}

int p3mx_dp3m_activate(p3mx_dp3m *h, size_t n, const double *pos, const double *dip,
                       unsigned flags) {
  return dp_guarded(h, [&] {
    if (!h->sys_set)
      throw Error(P3MX_ERUNTIME, "box not set: call p3mx_dp3m_set_system first");
    if (!(h->sys.periodic[0] && h->sys.periodic[1] && h->sys.periodic[2]))
      throw Error(P3MX_ERUNTIME, "DipolarP3M: requires periodicity (True, True, True)");
    if (h->sys.box[0] != h->sys.box[1] || h->sys.box[1] != h->sys.box[2])
      throw Error(P3MX_ERUNTIME, "DipolarP3M: requires a cubic box");
    bool const dev = (flags & P3MX_DEVICE_PTRS) != 0;
    h->activated = false;
    double const L = h->sys.box[0];
    // tune() (dp3m.cpp:647-680)
    if (h->alpha_L == 0. && h->alpha != 0.)
      h->alpha_L = h->alpha * L;
    if (h->r_cut_iL == 0. && h->r_cut != 0.)
      h->r_cut_iL = h->r_cut / L;
    dp_census(h, n, dip, dev);
    h->n = n;
    if (!h->is_tuned) {
      if (h->n_dip == 0)
        throw Error(P3MX_ERUNTIME, "DipolarP3M: no dipolar particles in the system");
      DpTuner t{h, pos, dip, dev};
      t.run();
      h->is_tuned = true;
    } else {
      h->r_cut_iL = h->r_cut / L;
      h->alpha_L = h->alpha * L;
    }
    if (h->mesh == -1)
      throw Error(P3MX_EDOMAIN, "Parameter 'mesh' must be > 0");
    dp_sanity_checks(h);
    dp_configure(h);
    if (h->n_dip > 0) {
      h->rs_err = dp3m_rs_error(L, h->r_cut_iL, h->n_dip, h->sum_mu2, h->alpha_L);
      h->ks_err = dp_ks_error(h, h->mesh, h->cao, h->alpha_L);
    }
    h->activated = true;
  });
}

int p3mx_dp3m_get_tuned(const p3mx_dp3m *h, p3mx_tuned *out) {
  if (!h || !out)
    return P3MX_EHANDLE;
  for (int d = 0; d < 3; ++d) {
    out->mesh[d] = h->mesh;
    out->mesh_off[d] = h->mesh_off[d];
    out->a[d] = (h->sys_set && h->mesh > 0) ? h->sys.box[d] / h->mesh : 0.;
  }
  out->cao = h->cao;
  out->r_cut = h->r_cut;
  out->alpha = h->alpha;
  out->r_cut_iL = h->r_cut_iL;
  out->alpha_L = h->alpha_L;
  out->accuracy = h->accuracy;
  out->epsilon = h->prm.epsilon;
  out->is_tuned = h->is_tuned ? 1 : 0;
  out->single_precision = h->prm.single_precision;
  out->rs_error = h->rs_err;
  out->ks_error = h->ks_err;
  return P3MX_OK;
}

int p3mx_dp3m_compute(p3mx_dp3m *h, size_t n, const double *pos, const double *dip, double *f,
                      double *torque, double *energy, unsigned flags, void *stream) {
  return dp_guarded(h, [&] {
    if (!h->activated)
      throw Error(P3MX_ERUNTIME, "DipolarP3M: actor not activated");
    bool const dev = (flags & P3MX_DEVICE_PTRS) != 0;
    bool const want_ft = (flags & P3MX_FORCES) != 0;
    bool const want_e = (flags & P3MX_ENERGY) != 0 && energy != nullptr;
    bool const overwrite = (flags & P3MX_OVERWRITE) != 0;
    if (want_ft && (!f || !torque))
      throw Error(P3MX_EDOMAIN, "forces requested with a NULL force or torque array");
    if (n && (!pos || !dip))
      throw Error(P3MX_EDOMAIN, "NULL position or dipole array");
    if (n != h->n || !h->de) {
      h->n = n;
      dp_configure(h);
    }
    Dp3mEngine &de = *h->de;
    cudaStream_t const st = stream ? static_cast<cudaStream_t>(stream) : de.engine().stream();
    auto const census = de.upload(pos, dip, dev, st);
    h->n_dip = static_cast<int>(census[0]);
    h->sum_mu2 = census[1];
    double *df = nullptr, *dt = nullptr;
    if (want_ft) {
      if (dev) {
        df = f;
        dt = torque;
      } else {
        h->scratch.ensure(6 * std::max<size_t>(1, n) * sizeof(double));
        df = h->scratch.as<double>();
        dt = df + 3 * n;
        if (!overwrite && n) {
          P3MX_CUDA(cudaMemcpyAsync(df, f, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
          P3MX_CUDA(cudaMemcpyAsync(dt, torque, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
        }
      }
    }
    double e2[2] = {0.0, 0.0};
    de.compute(h->prm.prefactor, h->accuracy, h->prm.epsilon, df, dt, overwrite, want_e, census,
               st, e2);
    if (want_ft && !dev && n) {
      P3MX_CUDA(cudaMemcpyAsync(f, df, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
      P3MX_CUDA(cudaMemcpyAsync(torque, dt, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    P3MX_CUDA(cudaStreamSynchronize(st));
    if (want_e) {
      energy[0] = e2[0];
      energy[1] = e2[1];
    }
  });
}

int p3mx_dp3m_profile(p3mx_dp3m *h, size_t n, const double *pos, const double *dip, int reps,
                      double *ms, const char **names, int cap, int *nstages) {
  return dp_guarded(h, [&] {
    if (!h->activated)
      throw Error(P3MX_ERUNTIME, "DipolarP3M: actor not activated");
    if (n != h->n || !h->de) {
      h->n = n;
      dp_configure(h);
    }
    Dp3mEngine &de = *h->de;
    cudaStream_t const st = de.engine().stream();
    auto const census = de.upload(pos, dip, false, st);
    h->scratch.ensure(6 * std::max<size_t>(1, n) * sizeof(double));
    double *f = h->scratch.as<double>(), *t = f + 3 * n;
    // one unprofiled evaluation first (list build, influence functions)
    de.compute(h->prm.prefactor, h->accuracy, h->prm.epsilon, f, t, true, false, census, st,
               nullptr);
    static std::vector<std::string> keep;
    auto prof = de.profile(h->prm.prefactor, h->accuracy, h->prm.epsilon, census, f, t,
                           std::max(1, reps), st);
    keep.clear();
    for (auto const &p : prof)
      keep.push_back(p.first);
    int const ns = static_cast<int>(prof.size());
    if (nstages)
      *nstages = ns;
    for (int k = 0; k < std::min(ns, cap); ++k) {
      if (ms)
        ms[k] = prof[k].second;
      if (names)
        names[k] = keep[k].c_str();
    }
  });
}

int p3mx_dp3m_launch_count(const p3mx_dp3m *h, long long *count) {
  if (!h || !count)
    return P3MX_EHANDLE;
  *count = h->de ? h->de->engine().launches() : 0;
  return P3MX_OK;
}

} // extern "C"
