// C ABI of the drop-in boundary (include/p3mx.h): actor life cycle,
// parameter validation with the reference's messages, the P3M tuner, and
// host<->device staging.  No exception crosses the ABI.
#include "../../include/p3mx.h"
#include "bond_abi.cuh"
#include "elc_host.cuh"
#include "engine.cuh"
#include "host_pool.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

using namespace p3mx;

namespace {

constexpr double kMeshOff = 0.5;            // P3M_MESHOFF, config.hpp:45-46
constexpr double kTuneCaoTooLarge = 1.0;    // TuningAlgorithm.cpp:47-51
constexpr double kTuneAccTooLarge = 3.0;
constexpr double kRcutPrec = 1e-3;          // P3M_RCUT_PREC
constexpr double kTimeGranularity = 2.0;    // TuningAlgorithm.hpp:82
constexpr int kMaxConsecutiveTrials = 20;   // TuningAlgorithm.hpp:86

// pinned host staging for host-pointer calls
struct Pinned {
  void *p = nullptr;
  size_t bytes = 0;
  ~Pinned() {
    if (p)
      cudaFreeHost(p);
  }
  void ensure(size_t n) {
    if (n <= bytes && p)
      return;
    if (p)
      cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    if (cudaMallocHost(&p, n ? n : 16) != cudaSuccess) {
      cudaGetLastError();
      throw Error(P3MX_ENOMEM, "pinned host allocation failed");
    }
    bytes = n ? n : 16;
  }
  template <typename T> T *as() { return static_cast<T *>(p); }
};

// Events marking the chunks of a pipelined device->host copy.
struct ChunkEvents {
  std::vector<cudaEvent_t> ev;
  ~ChunkEvents() {
    for (auto e : ev)
      cudaEventDestroy(e);
  }
  cudaEvent_t get(size_t i) {
    while (ev.size() <= i) {
      cudaEvent_t e;
      P3MX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ev.push_back(e);
    }
    return ev[i];
  }
};

// Chunks of the host<->device staging pipeline (bytes): sizes double from
// kStageFirst up to kStageChunk, so that the host copy of the first chunk
// (before any DMA can start) and of the last one (after the last DMA) are
// short.
constexpr size_t kStageChunk = size_t(4) << 20;
constexpr size_t kStageFirst = size_t(512) << 10;

// Chunk sizes of a transfer of `bytes`: ramping up from kStageFirst
// (host -> device) or, reversed, ramping down to it (device -> host).
std::vector<size_t> stage_chunks(size_t bytes, bool ramp_up) {
  std::vector<size_t> sizes;
  size_t c = kStageFirst;
  for (size_t left = bytes; left > 0;) {
    size_t const nb = std::min(c, left);
    sizes.push_back(nb);
    left -= nb;
    c = std::min(2 * c, kStageChunk);
  }
  if (!ramp_up)
    std::reverse(sizes.begin(), sizes.end());
  return sizes;
}

// Process-wide host worker pool; calls from different handles take turns.
HostPool &host_pool(std::unique_lock<std::mutex> &lk) {
  static HostPool pool;
  static std::mutex mu;
  lk = std::unique_lock<std::mutex>(mu);
  return pool;
}

bool mesh_fft_ok(int m) {
  if (m < 2 || (m % 2))
    return false;
  int x = m;
  for (int p = 2; p <= 31; ++p)
    while (x % p == 0)
      x /= p;
  return x == 1;
}

} // namespace

struct p3mx_handle {
  p3mx_params prm{};
  p3mx_system sys{};
  bool sys_set = false;
  // current P3M parameters (given or tuned)
  int mesh[3] = {-1, -1, -1};
  int cao = -1;
  double r_cut = -1, alpha = -1, accuracy = 0, mesh_off[3] = {kMeshOff, kMeshOff, kMeshOff};
  double r_cut_iL = 0, alpha_L = 0;
  bool is_tuned = false, activated = false;
  double rs_err = 0, ks_err = 0;
  std::unique_ptr<Engine> eng;
  // FP64 engine for the observables of the FP32-mixed actor: energies and
  // pressures are evaluated in FP64, as the reference GPU actor evaluates
  // them with its double-precision CPU kernels (p3m.impl.hpp:328-343)
  std::unique_ptr<Engine> eng64;
  size_t n = 0;
  int ntypes = 1;
  std::vector<PairIA> table{PairIA{0, 0, 0, 0, 0, 0, 0, 0, 0, -1.0}};
  std::string err;
  Pinned h_in, h_out;
  ChunkEvents out_events;
  // charges and types of the last host-pointer call, still in h_in and on
  // the device (unchanged chunks are not uploaded again)
  size_t staged_n = 0;
  bool staged_q = false, staged_type = false;
  // pair bonds (p3mx_set_bonds): built into the engine's lists on the next
  // call after a change (or after the engine was configured anew)
  std::vector<BondParam> bond_types;
  std::vector<int> bonds;
  bool bonds_dirty = false;
  // charge census
  int n_charged = 0;
  double sum_q2 = 0, sum_q = 0;
  // electrostatic layer correction attached to the actor (p3mx_set_elc)
  std::unique_ptr<ElcState> elc;
};

namespace {

int fail(p3mx_handle *h, Error const &e) {
  if (h)
    h->err = e.what();
  return e.code;
}

template <typename F> int guarded(p3mx_handle *h, F &&fn) {
  if (!h)
    return P3MX_EHANDLE;
  try {
    fn();
    h->err.clear();
    return P3MX_OK;
  } catch (Error const &e) {
    return fail(h, e);
  } catch (std::exception const &e) {
    h->err = e.what();
    return P3MX_ERUNTIME;
  }
}

// P3MParameters constructor checks (p3m/common.hpp:95-150) and the
// prefactor check of Actor::set_prefactor (actor.hpp:49-54).
void validate(p3mx_params const &p) {
  bool const tuning = p.tune != 0;
  if (p.prefactor <= 0.)
    throw Error(P3MX_EDOMAIN, "Parameter 'prefactor' must be > 0");
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
  for (int d = 0; d < 3; ++d)
    if (p.mesh[d] != -1 && p.mesh[d] % 2)
      throw Error(P3MX_EDOMAIN, "P3M requires an even number of mesh points in all directions");
  bool const off_ok = p.mesh_off[0] >= 0. && p.mesh_off[0] <= 1. && p.mesh_off[1] >= 0. &&
                      p.mesh_off[1] <= 1. && p.mesh_off[2] >= 0. && p.mesh_off[2] <= 1.;
  bool const off_default = p.mesh_off[0] == -1. && p.mesh_off[1] == -1. && p.mesh_off[2] == -1.;
  if (!off_ok && !off_default)
    throw Error(P3MX_EDOMAIN, "Parameter 'mesh_off' must be >= 0 and <= 1");
  if ((p.cao < 1 || p.cao > 7) && (!tuning || p.cao != -1))
    throw Error(P3MX_EDOMAIN, "Parameter 'cao' must be >= 1 and <= 7");
  if (!tuning && (p.cao > p.mesh[0] || p.cao > p.mesh[1] || p.cao > p.mesh[2]))
    throw Error(P3MX_EDOMAIN, "Parameter 'cao' cannot be larger than 'mesh'");
  if (p.charge_neutrality_tolerance < 0. && p.charge_neutrality_tolerance != -1.)
    throw Error(P3MX_EDOMAIN, "Parameter 'charge_neutrality_tolerance' must be >= 0");
}

std::string actor_name(p3mx_handle const *h) {
  return h->prm.single_precision ? "CoulombP3MGPU" : "CoulombP3M";
}

// Engine configuration for the handle's current parameters.
void configure_engine(p3mx_handle *h) {
  if (!h->eng || h->eng->fp32() != (h->prm.single_precision != 0))
    h->eng = std::make_unique<Engine>(h->prm.single_precision != 0);
  // (re)configuration may reallocate the device arrays: stage them again
  h->staged_q = h->staged_type = false;
  ReplicaConf c;
  for (int d = 0; d < 3; ++d) {
    c.box[d] = h->sys.box[d];
    c.mesh[d] = h->mesh[d];
    c.mesh_off[d] = h->mesh_off[d];
  }
  c.prefactor = h->prm.prefactor;
  c.epsilon = h->prm.epsilon;
  c.cao = h->cao;
  c.alpha = h->alpha;
  c.r_cut = h->r_cut;
  c.skin = h->sys.skin;
  c.p0 = 0;
  c.np = static_cast<long long>(h->n);
  h->eng->set_pair_table(h->ntypes, h->table);
  h->eng->configure({c}, static_cast<long long>(h->n));
  h->eng64.reset();
  if (h->elc)
    h->elc->img.reset();
}

Engine &observables_engine(p3mx_handle *h) {
  if (!h->eng64) {
    h->eng64 = std::make_unique<Engine>(false);
    ReplicaConf c = h->eng->conf(0);
    h->eng64->set_pair_table(h->ntypes, h->table);
    h->eng64->configure({c}, static_cast<long long>(h->n));
  }
  return *h->eng64;
}

// k-space energy / virial of the FP32-mixed actor in FP64 (see eng64).
void fp64_kspace_observables(p3mx_handle *h, cudaStream_t st, bool want_e, bool want_v,
                             std::vector<double> &en, std::vector<double> &vir) {
  Engine &e = *h->eng;
  Engine &e64 = observables_engine(h);
  e64.upload(e.d_pos(), e.d_q(), e.d_type(), true, st);
  e64.census(st);
  e64.long_range(nullptr, true, want_e, want_v, st, &en, &vir);
}

// sanity_checks_boxl (p3m.cpp:793-818) and the non-metallic cubic-box rule.
void sanity_checks(p3mx_handle *h) {
  for (int i = 0; i < 3; ++i) {
    double const cao_cut = (static_cast<double>(h->cao) / 2.0) * (h->sys.box[i] / h->mesh[i]);
    if (cao_cut >= 0.5 * h->sys.box[i]) {
      std::ostringstream m;
      m << "P3M_init: k-space cutoff " << cao_cut << " is larger than half of box dimension "
        << h->sys.box[i];
      throw Error(P3MX_ERUNTIME, m.str());
    }
  }
  if (h->prm.epsilon != 0.0) {
    if (h->sys.box[0] != h->sys.box[1] || h->sys.box[1] != h->sys.box[2] ||
        h->mesh[0] != h->mesh[1] || h->mesh[1] != h->mesh[2])
      throw Error(P3MX_ERUNTIME, actor_name(h) + ": non-metallic epsilon requires cubic box");
  }
  for (int d = 0; d < 3; ++d)
    if (!mesh_fft_ok(h->mesh[d]))
      throw Error(P3MX_EDOMAIN, "mesh " + std::to_string(h->mesh[d]) +
                                    " is not supported by the FFT (even sizes with prime factors <= 31)");
}

double rs_error(double pref, double r_cut_iL, int n_c, double sum_q2, double alpha_L,
                const double *box) {
  double const V = box[0] * box[1] * box[2];
  return (2. * pref * sum_q2 * std::exp(-(r_cut_iL * alpha_L) * (r_cut_iL * alpha_L))) /
         std::sqrt(static_cast<double>(n_c) * r_cut_iL * box[0] * V);
}

// ---------------------------------------------------------------------
// Tuner: restatement of TuningAlgorithm / CoulombTuningAlgorithm
// (p3m/TuningAlgorithm.cpp:57-328, electrostatics/p3m.cpp:595-791) with the
// k-space error summed on the device and trials timed with CUDA events on
// full force evaluations (long + short range).
struct Tuner {
  p3mx_handle *h;
  const double *pos;
  const double *q;
  const int *type;
  bool dev;
  double r_cut_iL_min = 0, r_cut_iL_max = 0;
  int cao_min = 1, cao_max = 7, cao_best = 7;
  double dens_min = 0, dens_max = 0;
  bool tune_mesh = false;
  size_t n_trials = 0;
  Engine *err_eng = nullptr;

  void log(const char *fmt, double a = 0, double b = 0) {
    (void)fmt;
    (void)a;
    (void)b;
  }

  std::tuple<double, double, double, double> accuracy(const int *mesh, int cao, double r_cut_iL) {
    double const *box = h->sys.box;
    double const pref = h->prm.prefactor;
    double rs = rs_error(pref, r_cut_iL, h->n_charged, h->sum_q2, 0., box);
    double alpha_L;
    if (std::sqrt(2.0) * rs > h->prm.accuracy)
      alpha_L = std::sqrt(std::log(std::sqrt(2.0) * rs / h->prm.accuracy)) / r_cut_iL;
    else
      alpha_L = 0.1;
    rs = rs_error(pref, r_cut_iL, h->n_charged, h->sum_q2, alpha_L, box);
    double const ks = err_eng->ks_error(mesh, cao, h->n_charged, h->sum_q2, alpha_L, box, pref);
    return {std::hypot(rs, ks), rs, ks, alpha_L};
  }

  double benchmark() {
    configure_engine(h);
    Engine &e = *h->eng;
    e.upload(pos, q, type, dev, e.stream());
    h->staged_q = h->staged_type = false;
    e.census(e.stream());
    cudaEvent_t t0, t1;
    P3MX_CUDA(cudaEventCreate(&t0));
    P3MX_CUDA(cudaEventCreate(&t1));
    int const timings = std::max(1, h->prm.timings);
    e.long_range(e.d_force(), true, false, false, e.stream(), nullptr, nullptr);
    e.short_range(e.d_force(), false, false, e.stream(), nullptr, nullptr);
    P3MX_CUDA(cudaEventRecord(t0, e.stream()));
    for (int k = 0; k < timings; ++k) {
      e.long_range(e.d_force(), true, false, false, e.stream(), nullptr, nullptr);
      e.short_range(e.d_force(), false, false, e.stream(), nullptr, nullptr);
    }
    P3MX_CUDA(cudaEventRecord(t1, e.stream()));
    P3MX_CUDA(cudaEventSynchronize(t1));
    float ms = 0.f;
    P3MX_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return static_cast<double>(ms) / timings;
  }

  void commit(const int *mesh, int cao, double r_cut_iL, double alpha_L) {
    double const L0 = h->sys.box[0];
    h->r_cut = r_cut_iL * L0;
    h->r_cut_iL = r_cut_iL;
    h->cao = cao;
    h->alpha_L = alpha_L;
    h->alpha = alpha_L / L0;
    for (int d = 0; d < 3; ++d)
      h->mesh[d] = mesh[d];
  }

  double get_mc_time(const int *mesh, int cao, double &t_rc, double &t_al, double &t_acc) {
    double const *box = h->sys.box;
    double const skin = h->sys.skin;
    double k_cut = std::numeric_limits<double>::max();
    int min_mesh = std::min({mesh[0], mesh[1], mesh[2]});
    for (int d = 0; d < 3; ++d)
      k_cut = std::min(k_cut, (static_cast<double>(cao) / 2.) * box[d] / mesh[d]);
    double const min_box = std::min({box[0], box[1], box[2]});
    double const k_cut_max = min_box - skin;
    if (cao >= min_mesh || k_cut >= k_cut_max)
      return -kTuneCaoTooLarge;
    for (int d = 0; d < 3; ++d)
      if (!mesh_fft_ok(mesh[d]))
        return -kTuneCaoTooLarge;
    double rs, ks;
    std::tie(t_acc, rs, ks, t_al) = accuracy(mesh, cao, r_cut_iL_max);
    if (t_acc > h->prm.accuracy)
      return -kTuneAccTooLarge;
    double lo = r_cut_iL_min, hi = r_cut_iL_max, rc;
    for (;;) {
      rc = 0.5 * (lo + hi);
      if (hi - lo < kRcutPrec)
        break;
      double acc;
      std::tie(acc, rs, ks, t_al) = accuracy(mesh, cao, rc);
      if (acc > h->prm.accuracy)
        lo = rc;
      else
        hi = rc;
    }
    t_rc = rc = hi;
    // the real-space cutoff plus skin must fit the cell system
    if (t_rc * box[0] + skin > 0.5 * min_box)
      return -kTuneAccTooLarge;
    commit(mesh, cao, rc, t_al);
    double const t = benchmark();
    std::tie(t_acc, rs, ks, t_al) = accuracy(mesh, cao, rc);
    if (h->prm.verbose)
      std::printf("%-4d %-3d %.5e %.5e %.3e %.3e %.3e %-8.4f\n", mesh[0], cao, rc, t_al, t_acc, rs,
                  ks, t);
    ++n_trials;
    return t;
  }

  double get_m_time(const int *mesh, int &t_cao, double &t_rc, double &t_al, double &t_acc) {
    double best = -1., rc = 0., al = 0., acc = 0.;
    int final_dir = 0;
    int cao = t_cao;
    double tmp;
    do {
      tmp = get_mc_time(mesh, cao, rc, al, acc);
      if (tmp == -kTuneCaoTooLarge)
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
      return -kTuneCaoTooLarge;
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
        if ((dir_times[0] >= 0 && dir_times[0] < best + kTimeGranularity) &&
            (dir_times[2] < 0 || dir_times[2] > dir_times[0]))
          final_dir = -1;
        else if ((dir_times[2] >= 0 && dir_times[2] < best + kTimeGranularity) &&
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
      } else if (tmp > best + kTimeGranularity) {
        break;
      }
    }
    return best;
  }

  void run() {
    double const *box = h->sys.box;
    double const L0 = box[0];
    // determine_r_cut_limits (TuningAlgorithm.cpp:57-74)
    if (h->r_cut_iL == 0.) {
      double const min_box = std::min({box[0], box[1], box[2]});
      r_cut_iL_min = 0.;
      r_cut_iL_max = (std::min(min_box, min_box / 2.) - h->sys.skin) / L0;
    } else {
      r_cut_iL_min = r_cut_iL_max = h->r_cut_iL;
    }
    // determine_cao_limits(7)
    if (h->cao == -1) {
      cao_min = 1;
      cao_max = 7;
      cao_best = 7;
    } else {
      cao_min = cao_max = cao_best = h->cao;
    }
    // determine_mesh_limits (p3m.cpp:676-707)
    int fixed_mesh[3] = {h->mesh[0], h->mesh[1], h->mesh[2]};
    if (h->mesh[0] == -1 && h->mesh[1] == -1 && h->mesh[2] == -1) {
      double const norm = std::cbrt(box[0] * box[1] * box[2]);
      double const maxn = 512., minn = std::min(maxn, std::cbrt(static_cast<double>(h->n_charged)));
      dens_min = minn / norm;
      dens_max = maxn / norm;
      tune_mesh = true;
    } else {
      double const dens = static_cast<double>(h->mesh[0]) / box[0];
      dens_min = dens_max = dens;
      if (h->mesh[1] == -1 && h->mesh[2] == -1) {
        for (int i : {1, 2}) {
          fixed_mesh[i] = static_cast<int>(std::round(dens * box[i]));
          fixed_mesh[i] += fixed_mesh[i] % 2;
        }
      }
    }
    if (h->prm.verbose) {
      std::printf("%s tune parameters: Accuracy goal = %.5e prefactor = %.5e\n",
                  actor_name(h).c_str(), h->prm.accuracy, h->prm.prefactor);
      std::printf("System: box_l = %.5e # charged part = %d Sum[q_i^2] = %.5e\n", box[0],
                  h->n_charged, h->sum_q2);
      std::printf("mesh cao r_cut_iL    alpha_L     err       rs_err    ks_err    time [ms]\n");
    }
    // get_time (p3m.cpp:709-754)
    struct {
      int mesh[3];
      int cao = -1;
      double alpha_L = -1, r_cut_iL = -1, accuracy = -1;
      double time = std::numeric_limits<double>::max();
    } best;
    double dens = dens_min;
    while (dens <= dens_max) {
      int tm[3];
      if (tune_mesh) {
        for (int i = 0; i < 3; ++i) {
          tm[i] = static_cast<int>(std::round(box[i] * dens));
          tm[i] += tm[i] % 2;
        }
      } else {
        for (int i = 0; i < 3; ++i)
          tm[i] = fixed_mesh[i];
      }
      int tcao = cao_best;
      double trc = 0, tal = 0, tacc = 0;
      double const t = get_m_time(tm, tcao, trc, tal, tacc);
      if (t >= 0.) {
        r_cut_iL_max = trc;
        if (t < best.time) {
          n_trials = 0;
          for (int i = 0; i < 3; ++i)
            best.mesh[i] = tm[i];
          best.cao = tcao;
          best.r_cut_iL = trc;
          best.alpha_L = tal;
          best.accuracy = tacc;
          best.time = t;
        } else if (t > best.time + kTimeGranularity ||
                   n_trials > static_cast<size_t>(kMaxConsecutiveTrials)) {
          break;
        }
      }
      if (!tune_mesh)
        break;
      dens += 0.1;
    }
    if (best.time == std::numeric_limits<double>::max())
      throw Error(P3MX_ERUNTIME, actor_name(h) + ": failed to reach requested accuracy");
    h->accuracy = best.accuracy;
    commit(best.mesh, best.cao, best.r_cut_iL, best.alpha_L);
    if (h->prm.verbose)
      std::printf("\nresulting parameters: mesh: (%d, %d, %d), cao: %d, r_cut_iL: %.4e,\n"
                  "                      alpha_L: %.4e, accuracy: %.4e, time: %.2f\n",
                  best.mesh[0], best.mesh[1], best.mesh[2], best.cao, best.r_cut_iL, best.alpha_L,
                  best.accuracy, best.time);
  }
};

void host_census(p3mx_handle *h, size_t n, const double *q, bool dev) {
  std::vector<double> qq(n);
  if (n) {
    if (dev)
      P3MX_CUDA(cudaMemcpy(qq.data(), q, n * sizeof(double), cudaMemcpyDeviceToHost));
    else
      std::memcpy(qq.data(), q, n * sizeof(double));
  }
  h->n_charged = 0;
  h->sum_q2 = h->sum_q = 0.;
  // Kahan sum for the neutrality ratio (coulomb.cpp:269-285)
  double ks = 0., kc = 0., qmin = std::numeric_limits<double>::infinity();
  for (double v : qq) {
    if (v != 0.) {
      h->n_charged++;
      h->sum_q2 += v * v;
      h->sum_q += v;
      double const y = v - kc;
      double const t = ks + y;
      kc = (t - ks) - y;
      ks = t;
      qmin = std::min(qmin, std::abs(v));
    }
  }
  if (h->prm.check_neutrality && h->prm.charge_neutrality_tolerance != -1. && h->n_charged > 0) {
    double const ratio = std::abs(ks) / qmin;
    if (ratio >= h->prm.charge_neutrality_tolerance) {
      std::ostringstream m;
      m.setf(std::ios::scientific);
      m.precision(4);
      m << ratio;
      throw Error(P3MX_ERUNTIME,
                  "The system is not charge neutral. Please neutralize the system before adding a "
                  "new actor by adding the corresponding counterions to the system. Alternatively "
                  "you can turn off the electroneutrality check by supplying "
                  "check_neutrality=False when creating the actor. In this case you may be "
                  "simulating a non-neutral system which will affect physical observables like "
                  "e.g. the pressure, the chemical potentials of charged species or potential "
                  "energies of the system. Since simulations of non charge neutral systems are "
                  "special please make sure you know what you are doing. The relative charge "
                  "excess was " +
                      m.str());
    }
  }
}

void ensure_ready(p3mx_handle *h, size_t n) {
  if (!h->activated)
    throw Error(P3MX_ERUNTIME, "actor not activated: call p3mx_activate first");
  if (n != h->n || !h->eng) {
    h->n = n;
    configure_engine(h);
    h->bonds_dirty = !h->bonds.empty();
  }
  if (h->bonds_dirty) {
    h->eng->set_bonds(h->bond_types, h->bonds, h->eng->stream());
    h->bonds_dirty = false;
  }
}

} // namespace

extern "C" {

const char *p3mx_version(void) { return "p3mx 0.1 sm_100a (FP64 + FP32-mixed P3M, LJ/WCA)"; }

int p3mx_create(const p3mx_params *params, p3mx_handle **out) {
  if (!params || !out)
    return P3MX_EHANDLE;
  *out = nullptr;
  auto h = std::make_unique<p3mx_handle>();
  h->prm = *params;
  try {
    validate(h->prm);
  } catch (Error const &e) {
    // no handle exists yet; report via a detached handle carrying the message
    h->err = e.what();
    *out = h.release();
    return e.code;
  }
  for (int d = 0; d < 3; ++d) {
    h->mesh[d] = params->mesh[d];
    h->mesh_off[d] = (params->mesh_off[d] == -1.) ? kMeshOff : params->mesh_off[d];
  }
  h->cao = params->cao;
  h->r_cut = params->r_cut == -1. ? 0. : params->r_cut;
  h->alpha = params->alpha == -1. ? 0. : params->alpha;
  h->accuracy = params->accuracy;
  h->is_tuned = !params->tune;
  *out = h.release();
  return P3MX_OK;
}

void p3mx_destroy(p3mx_handle *h) { delete h; }

const char *p3mx_last_error(const p3mx_handle *h) { return h ? h->err.c_str() : "NULL handle"; }

int p3mx_set_system(p3mx_handle *h, const p3mx_system *sys) {
  return guarded(h, [&] {
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
      // on_boxl_change -> scaleby_box_l: r_cut and alpha follow the box
      h->r_cut = h->r_cut_iL * h->sys.box[0];
      h->alpha = h->alpha_L / h->sys.box[0];
      sanity_checks(h);
      configure_engine(h);
    }
  });
}

int p3mx_activate(p3mx_handle *h, size_t n, const double *pos, const double *q, unsigned flags) {
  return guarded(h, [&] {
    if (!h->sys_set)
      throw Error(P3MX_ERUNTIME, "box not set: call p3mx_set_system first");
    if (!(h->sys.periodic[0] && h->sys.periodic[1] && h->sys.periodic[2]))
      throw Error(P3MX_ERUNTIME, actor_name(h) + ": requires periodicity (True, True, True)");
    bool const dev = (flags & P3MX_DEVICE_PTRS) != 0;
    h->activated = false;
    // scaled parameters, tune() p3m.cpp:758-765
    double const L0 = h->sys.box[0];
    if (h->alpha_L == 0. && h->alpha != 0.)
      h->alpha_L = h->alpha * L0;
    if (h->r_cut_iL == 0. && h->r_cut != 0.)
      h->r_cut_iL = h->r_cut / L0;
    host_census(h, n, q, dev);
    h->n = n;
    if (!h->is_tuned) {
      if (h->n_charged == 0)
        throw Error(P3MX_ERUNTIME, actor_name(h) + ": no charged particles in the system");
      Engine err_eng(false);
      Tuner t{h, pos, q, nullptr, dev};
      t.err_eng = &err_eng;
      t.run();
      h->is_tuned = true;
    } else {
      h->r_cut_iL = h->r_cut / L0;
      h->alpha_L = h->alpha * L0;
    }
    for (int d = 0; d < 3; ++d)
      if (h->mesh[d] == -1)
        throw Error(P3MX_EDOMAIN, "Parameter 'mesh' must be > 0");
    sanity_checks(h);
    configure_engine(h);
    // final error estimate of the committed parameters
    h->rs_err = rs_error(h->prm.prefactor, h->r_cut_iL, std::max(1, h->n_charged), h->sum_q2,
                         h->alpha_L, h->sys.box);
    h->ks_err = h->eng->ks_error(h->mesh, h->cao, std::max(1, h->n_charged), h->sum_q2,
                                 h->alpha_L, h->sys.box, h->prm.prefactor);
    h->activated = true;
  });
}

int p3mx_get_tuned(const p3mx_handle *h, p3mx_tuned *out) {
  if (!h || !out)
    return P3MX_EHANDLE;
  for (int d = 0; d < 3; ++d) {
    out->mesh[d] = h->mesh[d];
    out->mesh_off[d] = h->mesh_off[d];
    out->a[d] = (h->sys_set && h->mesh[d] > 0) ? h->sys.box[d] / h->mesh[d] : 0.;
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

int p3mx_set_bonds(p3mx_handle *h, int n_types, const p3mx_bond_params *types, size_t n_bonds,
                   const int *bonds) {
  return guarded(h, [&] {
    h->bond_types = bond_types_from_abi(n_types, types, n_bonds, bonds);
    h->bonds.assign(bonds, bonds + 3 * n_bonds);
    h->bonds_dirty = true;
    if (h->eng && h->activated) {
      h->eng->set_bonds(h->bond_types, h->bonds, h->eng->stream());
      h->bonds_dirty = false;
    }
  });
}

int p3mx_bond_observables(p3mx_handle *h, size_t n, const double *pos, double *energy,
                          double *virial9, unsigned flags, void *stream) {
  return guarded(h, [&] {
    ensure_ready(h, n);
    Engine &e = *h->eng;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : e.stream();
    double en = 0.0, vir[9];
    if (n > 0)
      e.upload_positions(pos, flags & P3MX_DEVICE_PTRS, st);
    e.bond_observables(st, &en, vir);
    if (energy)
      *energy = en;
    if (virial9)
      for (int k = 0; k < 9; ++k)
        virial9[k] = vir[k];
  });
}

int p3mx_set_pair_params(p3mx_handle *h, int ntypes, const p3mx_pair_params *table) {
  return guarded(h, [&] {
    if (ntypes < 1 || !table)
      throw Error(P3MX_EDOMAIN, "pair table needs ntypes >= 1");
    std::vector<PairIA> t(static_cast<size_t>(ntypes) * ntypes);
    for (int k = 0; k < ntypes * ntypes; ++k) {
      auto const &s = table[k];
      if (s.lj_eps < 0.)
        throw Error(P3MX_EDOMAIN, "LJ parameter 'epsilon' has to be >= 0");
      if (s.lj_sig < 0.)
        throw Error(P3MX_EDOMAIN, "LJ parameter 'sigma' has to be >= 0");
      if (s.lj_cut < 0.)
        throw Error(P3MX_EDOMAIN, "LJ parameter 'cutoff' has to be >= 0");
      if (s.wca_eps < 0.)
        throw Error(P3MX_EDOMAIN, "WCA parameter 'epsilon' has to be >= 0");
      if (s.wca_sig < 0.)
        throw Error(P3MX_EDOMAIN, "WCA parameter 'sigma' has to be >= 0");
      PairIA &d = t[k];
      d.lj_eps = s.lj_eps;
      d.lj_sig = s.lj_sig;
      d.lj_cut = s.lj_cut;
      d.lj_shift = s.lj_shift;
      d.lj_offset = s.lj_offset;
      d.lj_min = std::max(s.lj_min, 0.);
      d.wca_eps = s.wca_eps;
      d.wca_sig = s.wca_sig;
      d.wca_cut = (s.wca_sig != 0.) ? s.wca_sig * std::pow(2., 1. / 6.) : 0.;
      // max_cutoff of the pair (nonbonded_interaction_data.cpp): inactive
      // when no potential is switched on
      double ic = -1.0;
      if (s.lj_cut > 0. && s.lj_eps != 0.)
        ic = std::max(ic, s.lj_cut + s.lj_offset);
      if (d.wca_cut > 0. && s.wca_eps != 0.)
        ic = std::max(ic, d.wca_cut);
      d.ia_cut = ic;
    }
    h->ntypes = ntypes;
    h->table = t;
    if (h->eng) {
      h->eng->set_pair_table(ntypes, t);
    }
  });
}

// want_pos / want_qt select the positions and/or the charges and types (a
// split used by the speculative path of p3mx_forces).
static void stage_in(p3mx_handle *h, size_t n, const double *pos, const double *q, const int *type,
                     bool dev, cudaStream_t st, bool want_pos = true, bool want_qt = true) {
  Engine &e = *h->eng;
  if (dev || n == 0) {
    e.upload(pos, q, type, true, st);
    h->staged_q = h->staged_type = false;
    return;
  }
  // host arrays -> pinned staging (parallel host copies) -> device, chunk by
  // chunk: the DMA of one chunk overlaps the host copy of the next.  Charges
  // and types rarely change between calls: a chunk equal to the staged copy
  // of the last call (which is also on the device) is not sent again.
  size_t const bytes = n * (4 * sizeof(double) + sizeof(int));
  bool const kept = h->h_in.p != nullptr && h->h_in.bytes >= bytes && h->staged_n == n;
  h->h_in.ensure(bytes);
  if (!kept)
    h->staged_q = h->staged_type = false;
  char *pinned = h->h_in.as<char>();
  std::unique_lock<std::mutex> lk;
  HostPool &pool = host_pool(lk);
  auto push = [&](const void *src, void *dst, size_t nbytes, bool cached) {
    size_t b0 = 0;
    for (size_t const nb : stage_chunks(nbytes, true)) {
      const char *s = static_cast<const char *>(src) + b0;
      if (!(cached && pool.equal(pinned + b0, s, nb))) {
        pool.copy(pinned + b0, s, nb);
        P3MX_CUDA(cudaMemcpyAsync(static_cast<char *>(dst) + b0, pinned + b0, nb,
                                  cudaMemcpyHostToDevice, st));
      }
      b0 += nb;
    }
    pinned += nbytes;
  };
  if (want_pos)
    push(pos, e.d_pos(), 3 * n * sizeof(double), false);
  else
    pinned += 3 * n * sizeof(double);
  if (!want_qt)
    return;
  push(q, e.d_q(), n * sizeof(double), h->staged_q);
  if (type) {
    push(type, e.d_type(), n * sizeof(int), h->staged_type);
  } else {
    P3MX_CUDA(cudaMemsetAsync(e.d_type(), 0, n * sizeof(int), st));
  }
  h->staged_n = n;
  h->staged_q = true;
  h->staged_type = (type != nullptr);
}

// True when the host arrays q and type (nullptr: all zero) equal the
// staged copies of the last call, which are also on the device.
static bool staged_match(p3mx_handle *h, size_t n, const double *q, const int *type) {
  if (h->h_in.p == nullptr || h->staged_n != n || !h->staged_q ||
      (type != nullptr) != h->staged_type)
    return false;
  const char *pinned = h->h_in.as<char>() + 3 * n * sizeof(double);
  std::unique_lock<std::mutex> lk;
  HostPool &pool = host_pool(lk);
  if (!pool.equal(pinned, q, n * sizeof(double)))
    return false;
  return type == nullptr || pool.equal(pinned + n * sizeof(double), type, n * sizeof(int));
}

// Raise the error of a kernel whose bounded wait ran out (both engines).
static void check_kernels(p3mx_handle *h, cudaStream_t st) {
  h->eng->check_kernel_error(st);
  if (h->eng64)
    h->eng64->check_kernel_error(st);
}

static void stage_out(p3mx_handle *h, size_t n, double *f, bool dev, bool overwrite,
                      cudaStream_t st) {
  Engine &e = *h->eng;
  if (!f || n == 0)
    return;
  if (dev) {
    // device destination: forces were computed straight into f
    return;
  }
  // device -> pinned staging in chunks, each chunk copied (or added) to the
  // user's array by the host pool while the next chunk is in flight
  size_t const bytes = 3 * n * sizeof(double);
  h->h_out.ensure(bytes);
  double *o = h->h_out.as<double>();
  std::vector<size_t> const sizes = stage_chunks(bytes, false);
  size_t const nch = sizes.size();
  std::vector<size_t> off(nch + 1, 0);
  for (size_t c = 0; c < nch; ++c)
    off[c + 1] = off[c] + sizes[c];
  for (size_t c = 0; c < nch; ++c) {
    P3MX_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(o) + off[c],
                              reinterpret_cast<const char *>(e.d_force()) + off[c], sizes[c],
                              cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaEventRecord(h->out_events.get(c), st));
  }
  std::unique_lock<std::mutex> lk;
  HostPool &pool = host_pool(lk);
  for (size_t c = 0; c < nch; ++c) {
    size_t const b0 = off[c], nb = sizes[c];
    P3MX_CUDA(cudaEventSynchronize(h->out_events.get(c)));
    if (overwrite) {
      pool.copy(reinterpret_cast<char *>(f) + b0, reinterpret_cast<const char *>(o) + b0, nb);
    } else {
      size_t const k0 = b0 / sizeof(double), nk = nb / sizeof(double);
      size_t const piece = std::max<size_t>(32768, (nk + pool.size() - 1) / pool.size());
      pool.run(static_cast<int>((nk + piece - 1) / piece), [&](int i) {
        size_t const a0 = k0 + i * piece, a1 = std::min(k0 + nk, a0 + piece);
        for (size_t k = a0; k < a1; ++k)
          f[k] += o[k];
      });
    }
  }
}

// ELC correction of the staged particles into the device forces fd
// (ElectrostaticLayerCorrection::add_long_range_forces :1231-1254 after the
// P3M forces; long_range_energy :1189-1229 adds calc_energy).
static void elc_add(p3mx_handle *h, double *fd, double *energy, cudaStream_t st) {
  Engine &e = *h->eng;
  // sanity_checks_periodicity (elc.cpp:983-988), also after a later
  // p3mx_set_system
  if (!(h->sys.periodic[0] && h->sys.periodic[1] && h->sys.periodic[2]))
    throw Error(P3MX_ERUNTIME, "ELC: requires periodicity (True, True, True)");
  elc_apply(*h->elc, h->sys.box, h->prm.prefactor, h->r_cut, static_cast<long long>(h->n),
            e.d_pos(), e.d_q(), fd, energy, nullptr, st);
}

// ELC with dielectric contrasts, the whole Coulomb + non-bonded force
// evaluation (add_long_range_forces :1231-1254, long_range_energy
// :1189-1229, the short-range corrections of elc.hpp): short range and
// bonds on the engine, the image-layer pair and self terms over its Verlet
// lists, the mesh part from an FP64 engine over 3N slots holding the
// particles and their images (forces of the first N slots; the energy
// 0.5 E(real) + 0.5 E(both) - 0.5 E(images) from three runs whose censuses
// give the P3M sums of each charge set, as modify_p3m_sums does), then the
// ELC mode, dipole and z terms.  fd is overwritten.  energy3 / virial27 as
// p3mx_forces (k-space virial zero).
static void elc_contrast_forces(p3mx_handle *h, double *fd, double *energy3, double *virial27,
                                cudaStream_t st) {
  Engine &e = *h->eng;
  ElcState &s = *h->elc;
  elc_prepare(s, h->sys.box, h->prm.prefactor, h->r_cut, st);
  if (!(h->sys.periodic[0] && h->sys.periodic[1] && h->sys.periodic[2]))
    throw Error(P3MX_ERUNTIME, "ELC: requires periodicity (True, True, True)");
  bool const want = energy3 || virial27;
  e.short_range(fd, true, false, st, nullptr, nullptr);
  e.bond_forces(fd, st);
  std::vector<double> ens, virs;
  if (want)
    e.short_range(observables_engine(h).d_force(), true, true, st, &ens, &virs, true);
  double e_img_pairs = 0.0;
  e.elc_image_pairs(s.space_layer, s.box_h, s.prm.delta_mid_bot, s.prm.delta_mid_top, fd,
                    energy3 ? &e_img_pairs : nullptr, st);
  long long const n = static_cast<long long>(h->n);
  long long const n3 = 3 * n;
  if (!s.img) {
    s.img = std::make_unique<Engine>(false);
    ReplicaConf c = e.conf(0);
    c.np = n3;
    s.img->set_pair_table(h->ntypes, h->table);
    s.img->configure({c}, n3);
  }
  Engine &im = *s.img;
  s.d_aug_pos.ensure(static_cast<size_t>(3 * n3) * sizeof(double));
  s.d_aug_q.ensure(static_cast<size_t>(n3) * sizeof(double));
  s.d_faug.ensure(static_cast<size_t>(3 * n3) * sizeof(double));
  ElcGeom const g = elc_geom(s, h->sys.box, h->prm.prefactor, n);
  auto run = [&](int which, double *faug, double *energy) {
    if (n == 0)
      return;
    k_elc_augment<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(
        e.d_pos(), e.d_q(), n, g, which, s.d_aug_pos.as<double>(), s.d_aug_q.as<double>());
    P3MX_CUDA(cudaGetLastError());
    im.upload(s.d_aug_pos.as<double>(), s.d_aug_q.as<double>(), nullptr, true, st);
    im.census(st);
    std::vector<double> en, vir;
    im.long_range(faug, true, energy != nullptr, false, st, &en, &vir);
    if (energy)
      *energy = en.empty() ? 0.0 : en[0];
  };
  double e_both = 0.0, e_real = 0.0, e_imgs = 0.0;
  run(3, s.d_faug.as<double>(), energy3 ? &e_both : nullptr);
  if (n > 0) {
    k_elc_add<<<static_cast<unsigned>((3 * n + 255) / 256), 256, 0, st>>>(
        fd, s.d_faug.as<double>(), 3 * n);
    P3MX_CUDA(cudaGetLastError());
  }
  if (energy3) {
    run(1, nullptr, &e_real);
    run(2, nullptr, &e_imgs);
  }
  double e_elc = 0.0;
  elc_add(h, fd, energy3 ? &e_elc : nullptr, st);
  if (energy3) {
    energy3[0] = ens[0] + e_img_pairs;
    energy3[1] = 0.5 * e_real + 0.5 * e_both - 0.5 * e_imgs + e_elc;
    energy3[2] = ens[1];
  }
  if (virial27)
    for (int k = 0; k < 9; ++k) {
      virial27[k] = virs[k];
      virial27[9 + k] = 0.0;
      virial27[18 + k] = virs[9 + k];
    }
}

int p3mx_set_elc(p3mx_handle *h, const p3mx_elc_params *p) {
  return guarded(h, [&] {
    if (!p) {
      h->elc.reset();
      return;
    }
    elc_validate(*p);
    if (h->sys_set && !(h->sys.periodic[0] && h->sys.periodic[1] && h->sys.periodic[2]))
      throw Error(P3MX_ERUNTIME, "ELC: requires periodicity (True, True, True)");
    auto s = std::make_unique<ElcState>();
    s->prm = *p;
    s->far_calculated = (p->far_cut == -1.0);
    // adapt_epsilon_elc (p3m.impl.hpp:112-114): the base P3M is metallic
    h->prm.epsilon = 0.0;
    if (h->sys_set) {
      Engine *e = h->eng.get();
      elc_prepare(*s, h->sys.box, h->prm.prefactor, h->r_cut, e ? e->stream() : nullptr);
    }
    h->elc = std::move(s);
  });
}

int p3mx_get_elc(const p3mx_handle *h, double *far_cut, double *box_h, int *n_modes) {
  if (!h)
    return P3MX_EHANDLE;
  if (!h->elc)
    return P3MX_ERUNTIME;
  if (far_cut)
    *far_cut = h->elc->far_cut;
  if (box_h)
    *box_h = h->elc->box_h;
  if (n_modes)
    *n_modes = static_cast<int>(h->elc->modes.size());
  return 0;
}

int p3mx_long_range(p3mx_handle *h, size_t n, const double *pos, const double *q, double *f,
                    double *energy, double *virial9, unsigned flags, void *stream) {
  return guarded(h, [&] {
    ensure_ready(h, n);
    if (h->elc && h->elc->contrast())
      throw Error(P3MX_ERUNTIME, "ELC with dielectric contrasts: the image terms span the "
                                 "short and long range; use p3mx_forces");
    Engine &e = *h->eng;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : e.stream();
    bool const dev = flags & P3MX_DEVICE_PTRS;
    bool const ow = flags & P3MX_OVERWRITE;
    stage_in(h, n, pos, q, nullptr, dev, st);
    e.census(st);
    double *fd = nullptr;
    if ((flags & P3MX_FORCES) && f)
      fd = dev ? f : e.d_force();
    std::vector<double> en, vir;
    bool const want_e = energy && (flags & P3MX_ENERGY);
    bool const want_v = virial9 && (flags & P3MX_VIRIAL);
    bool const obs64 = h->prm.single_precision && !(flags & P3MX_MIXED_OBSERVABLES);
    e.long_range(fd, dev ? ow : true, want_e && !obs64, want_v && !obs64, st, &en, &vir);
    if (obs64 && (want_e || want_v))
      fp64_kspace_observables(h, st, want_e, want_v, en, vir);
    double e_elc = 0.0;
    if (h->elc) {
      elc_add(h, fd ? fd : e.d_force(), want_e ? &e_elc : nullptr, st);
      vir.assign(9, 0.0);
    }
    if (energy && (flags & P3MX_ENERGY))
      *energy = (en.empty() ? 0. : en[0]) + e_elc;
    if (virial9 && (flags & P3MX_VIRIAL))
      for (int k = 0; k < 9; ++k)
        virial9[k] = vir.empty() ? 0. : vir[k];
    if (fd)
      stage_out(h, n, f, dev, ow, st);
    P3MX_CUDA(cudaStreamSynchronize(st));
    check_kernels(h, st);
  });
}

int p3mx_short_range(p3mx_handle *h, size_t n, const double *pos, const double *q, const int *type,
                     double *f, double *energy2, double *virial18, unsigned flags, void *stream) {
  return guarded(h, [&] {
    ensure_ready(h, n);
    Engine &e = *h->eng;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : e.stream();
    bool const dev = flags & P3MX_DEVICE_PTRS;
    bool const ow = flags & P3MX_OVERWRITE;
    stage_in(h, n, pos, q, type, dev, st);
    double *fd = nullptr;
    if ((flags & P3MX_FORCES) && f)
      fd = dev ? f : e.d_force();
    bool const want = (energy2 && (flags & P3MX_ENERGY)) || (virial18 && (flags & P3MX_VIRIAL));
    std::vector<double> en, vir;
    bool const obs64 = h->prm.single_precision && !(flags & P3MX_MIXED_OBSERVABLES);
    if (fd) {
      e.short_range(fd, dev ? ow : true, want && !obs64, st, &en, &vir);
      e.bond_forces(fd, st);
    } else if (!(want && obs64)) {
      // energies only: compute into the scratch force buffer
      e.short_range(e.d_force(), true, want, st, &en, &vir);
    }
    if (want && obs64)
      e.short_range(observables_engine(h).d_force(), true, true, st, &en, &vir, true);
    if (energy2 && (flags & P3MX_ENERGY))
      for (int k = 0; k < 2; ++k)
        energy2[k] = en.empty() ? 0. : en[k];
    if (virial18 && (flags & P3MX_VIRIAL))
      for (int k = 0; k < 18; ++k)
        virial18[k] = vir.empty() ? 0. : vir[k];
    if (fd)
      stage_out(h, n, f, dev, ow, st);
    P3MX_CUDA(cudaStreamSynchronize(st));
    check_kernels(h, st);
  });
}

int p3mx_forces(p3mx_handle *h, size_t n, const double *pos, const double *q, const int *type,
                double *f, double *energy3, double *virial27, unsigned flags, void *stream) {
  return guarded(h, [&] {
    ensure_ready(h, n);
    Engine &e = *h->eng;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : e.stream();
    bool const dev = flags & P3MX_DEVICE_PTRS;
    bool const ow = flags & P3MX_OVERWRITE;
    bool const want_e = energy3 && (flags & P3MX_ENERGY);
    bool const want_v = virial27 && (flags & P3MX_VIRIAL);
    double *fd = (dev && f) ? f : e.d_force();
    if (h->elc && h->elc->contrast()) {
      stage_in(h, n, pos, q, type, dev, st);
      bool const add_dev = dev && f && !ow;
      double *fo = add_dev ? e.d_force() : fd;
      elc_contrast_forces(h, fo, want_e ? energy3 : nullptr, want_v ? virial27 : nullptr, st);
      if (add_dev && n > 0)
        k_elc_add<<<static_cast<unsigned>((3 * n + 255) / 256), 256, 0, st>>>(f, fo, 3 * n);
      if (f)
        stage_out(h, n, f, dev, ow, st);
      P3MX_CUDA(cudaStreamSynchronize(st));
      check_kernels(h, st);
      return;
    }
    // Forces only from host arrays, with charges and types staged by an
    // earlier call: the device computes with the staged copies while the
    // host compares them with q and type; on a difference the changed
    // chunks are uploaded and the forces computed again.  The comparison
    // is thereby off the critical path of the common case (unchanged
    // charges and types).
    bool const spec = !dev && f && !want_e && !want_v && n > 0 && h->h_in.p &&
                      h->staged_n == n && h->staged_q && (type != nullptr) == h->staged_type;
    stage_in(h, n, pos, q, type, dev, st, true, !spec);
    if (spec) {
      auto forces = [&] {
        if (h->prm.epsilon != 0.)
          e.census(st);
        e.forces_all(fd, true, st);
        if (h->elc)
          elc_add(h, fd, nullptr, st);
      };
      forces();
      if (!staged_match(h, n, q, type)) {
        P3MX_CUDA(cudaStreamSynchronize(st));
        stage_in(h, n, pos, q, type, dev, st, false, true);
        forces();
      }
      stage_out(h, n, f, dev, ow, st);
      P3MX_CUDA(cudaStreamSynchronize(st));
      check_kernels(h, st);
      return;
    }
    if (want_e || h->prm.epsilon != 0.)
      e.census(st);
    std::vector<double> enk, virk, ens, virs;
    bool const obs64 = h->prm.single_precision && !(flags & P3MX_MIXED_OBSERVABLES);
    if (!want_e && !want_v) {
      // forces only: real-space pairs concurrent with the k-space chain
      e.forces_all(fd, dev ? ow : true, st);
    } else {
      e.long_range(fd, dev ? ow : true, want_e && !obs64, want_v && !obs64, st, &enk, &virk);
      e.short_range(fd, false, (want_e || want_v) && !obs64, st, &ens, &virs);
      e.bond_forces(fd, st);
    }
    if (obs64 && (want_e || want_v)) {
      fp64_kspace_observables(h, st, want_e, want_v, enk, virk);
      e.short_range(observables_engine(h).d_force(), true, true, st, &ens, &virs, true);
    }
    double e_elc = 0.0;
    if (h->elc) {
      // ELC: correction forces and energy; no k-space pressure (the
      // reference warns and reports zero, coulomb.cpp:124-131)
      elc_add(h, fd, want_e ? &e_elc : nullptr, st);
      for (auto &v : virk)
        v = 0.0;
    }
    if (want_e) {
      energy3[0] = ens[0];
      energy3[1] = enk[0] + e_elc;
      energy3[2] = ens[1];
    }
    if (want_v)
      for (int k = 0; k < 9; ++k) {
        virial27[k] = virs[k];
        virial27[9 + k] = virk[k];
        virial27[18 + k] = virs[9 + k];
      }
    if (f)
      stage_out(h, n, f, dev, ow, st);
    P3MX_CUDA(cudaStreamSynchronize(st));
    check_kernels(h, st);
  });
}

int p3mx_cell_grid(p3mx_handle *h, int *cell_grid, double *cell_size) {
  return guarded(h, [&] {
    if (!h->eng)
      throw Error(P3MX_ERUNTIME, "actor not activated");
    h->eng->cell_grid(0, cell_grid, cell_size);
  });
}

int p3mx_cell_index(p3mx_handle *h, size_t n, const double *pos, int *cell) {
  return guarded(h, [&] {
    ensure_ready(h, n);
    Engine &e = *h->eng;
    e.upload_positions(pos, false, e.stream());
    auto v = e.cell_index_ghost(e.stream());
    std::memcpy(cell, v.data(), n * sizeof(int));
  });
}

int p3mx_verlet_pairs(p3mx_handle *h, size_t n, const double *pos, const double *q, const int *type,
                      int *pairs, size_t cap, size_t *count) {
  return guarded(h, [&] {
    ensure_ready(h, n);
    Engine &e = *h->eng;
    e.upload(pos, q, type, false, e.stream());
    h->staged_q = h->staged_type = false;
    auto v = e.verlet_pairs(e.stream());
    size_t const np = v.size() / 2;
    if (count)
      *count = np;
    std::memcpy(pairs, v.data(), std::min(np, cap) * 2 * sizeof(int));
  });
}

int p3mx_copy_mesh(p3mx_handle *h, double *out, size_t cap) {
  return guarded(h, [&] {
    if (!h->eng)
      throw Error(P3MX_ERUNTIME, "actor not activated");
    auto v = h->eng->mesh_copy(0, h->eng->stream());
    if (cap < v.size())
      throw Error(P3MX_EDOMAIN, "output buffer too small for the mesh");
    std::memcpy(out, v.data(), v.size() * sizeof(double));
  });
}

int p3mx_profile(p3mx_handle *h, int reps, double *ms, const char **names, int cap,
                 int *nstages) {
  return guarded(h, [&] {
    if (!h->eng || !h->activated)
      throw Error(P3MX_ERUNTIME, "actor not activated");
    static std::vector<std::string> keep;
    auto prof = h->eng->profile(std::max(1, reps), h->eng->stream());
    if (h->elc) {
      Engine &e = *h->eng;
      auto pe = elc_profile(*h->elc, h->sys.box, h->prm.prefactor, h->r_cut,
                            static_cast<long long>(h->n),
                            e.d_pos(), e.d_q(), e.d_force(), std::max(1, reps), e.stream());
      prof.insert(prof.end(), pe.begin(), pe.end());
    }
    keep.clear();
    for (auto const &p : prof)
      keep.push_back(p.first);
    int const n = static_cast<int>(prof.size());
    if (nstages)
      *nstages = n;
    for (int k = 0; k < std::min(n, cap); ++k) {
      if (ms)
        ms[k] = prof[k].second;
      if (names)
        names[k] = keep[k].c_str();
    }
  });
}

int p3mx_resort(p3mx_handle *h) {
  return guarded(h, [&] {
    if (h->eng)
      h->eng->invalidate_lists();
    if (h->eng64)
      h->eng64->invalidate_lists();
  });
}

int p3mx_launch_count(const p3mx_handle *h, long long *count) {
  if (!h || !count)
    return P3MX_EHANDLE;
  *count = (h->eng ? h->eng->launches() : 0) + (h->eng64 ? h->eng64->launches() : 0);
  return P3MX_OK;
}

int p3mx_exp_check(size_t n, const float *x, float *out, void *stream) {
  if (n && (!x || !out))
    return P3MX_EDOMAIN;
  if (n == 0)
    return P3MX_OK;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  long long const nn = static_cast<long long>(n);
  k_exp_check<<<static_cast<unsigned>((nn + 255) / 256), 256, 0, st>>>(nn, x, out);
  return cudaGetLastError() == cudaSuccess ? P3MX_OK : P3MX_ECUDA;
}

int p3mx_error_estimate(const int *mesh, int cao, int n_c_part, double sum_q2, double alpha_L,
                        double r_cut_iL, const double *box, double prefactor, double *rs_err,
                        double *ks_err) {
  try {
    Engine e(false);
    if (rs_err)
      *rs_err = rs_error(prefactor, r_cut_iL, n_c_part, sum_q2, alpha_L, box);
    if (ks_err)
      *ks_err = e.ks_error(mesh, cao, n_c_part, sum_q2, alpha_L, box, prefactor);
    return P3MX_OK;
  } catch (Error const &e) {
    return e.code;
  }
}

} // extern "C"
