// Batched replicas: many independent periodic systems of uneven size and
// box advanced by one launch per kernel, tuned by a batch autotuner, and
// integrated with velocity Verlet + Langevin inside a captured CUDA graph.
// (The reference has no batched path: every replica would be one ESPResSo
// System running its own MPI job.)
#include "../../include/p3mx.h"
#include "bond_abi.cuh"
#include "engine.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

using namespace p3mx;

namespace p3mx {

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// SC'11), the generator family the reference thermostat uses
// (random.hpp:74-125 over libs/Random123).
__device__ inline uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    unsigned const hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    unsigned const hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

__device__ inline double u01(unsigned v) { return (v + 0.5) * (1.0 / 4294967296.0); }

// velocity Verlet step 1 (integrators/velocity_verlet_inline.hpp:38-54),
// unit masses: v += dt/2 f; x += dt v
__global__ void k_vv_step1(double *__restrict__ x, double *__restrict__ v,
                           const double *__restrict__ f, long long n3, double dt) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n3)
    return;
  double const vi = v[i] + 0.5 * dt * f[i];
  v[i] = vi;
  x[i] += dt * vi;
}

// velocity Verlet step 2: v += dt/2 f
__global__ void k_vv_step2(double *__restrict__ v, const double *__restrict__ f, long long n3,
                           double dt) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n3)
    return;
  v[i] += 0.5 * dt * f[i];
}

// Langevin friction and uniform noise of variance 2 kT gamma / dt per
// component (thermostats/langevin_inline.hpp:40-59: prefactor
// sqrt(24 kT gamma / dt) times U(-1/2, 1/2)).
__global__ void k_langevin(double *__restrict__ f, const double *__restrict__ v, long long n,
                           double gamma, double noise, unsigned long long seed,
                           const unsigned long long *__restrict__ step) {
  long long const i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  unsigned long long const s = *step;
  uint4 const r = philox4x32_10(
      make_uint4(static_cast<unsigned>(i), static_cast<unsigned>(i >> 32),
                 static_cast<unsigned>(s), static_cast<unsigned>(s >> 32)),
      make_uint2(static_cast<unsigned>(seed), static_cast<unsigned>(seed >> 32)));
  f[3 * i + 0] += -gamma * v[3 * i + 0] + noise * (u01(r.x) - 0.5);
  f[3 * i + 1] += -gamma * v[3 * i + 1] + noise * (u01(r.y) - 0.5);
  f[3 * i + 2] += -gamma * v[3 * i + 2] + noise * (u01(r.z) - 0.5);
}

__global__ void k_step_inc(unsigned long long *step) { *step += 1; }

// Batched Hockney-Eastwood k-space error sums: query q = (mesh, cao,
// alpha_L) for cubic meshes, blockIdx.y = query, per-block partials.
__global__ void k_ks_error_batch(const int2 *__restrict__ mc, const double *__restrict__ aL,
                                 double *__restrict__ partials) {
  int const qi = blockIdx.y;
  int const M = mc[qi].x, cao = mc[qi].y;
  double const alpha_L = aL[qi];
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
    double const en = pow(sinc_d(nx * mi) * sinc_d(ny * mi) * sinc_d(nz * mi), 2.0 * cao);
    double const a1 = ex * ex / n2;
    double const a2 = en * ex * n2 / n2;
    double const d = a1 - (a2 / cs) * (a2 / cs) / n2;
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
    partials[static_cast<long long>(qi) * gridDim.x + blockIdx.x] = s;
  }
}

// Tuned parameters of one replica for one cao (batch autotuner).
struct BatchChoice {
  int mesh = 0;
  double r_cut_iL = 0, alpha_L = 0, acc = 0, rs = 0, ks = 0, cost = 0;
};

} // namespace p3mx

struct p3mx_batch {
  p3mx_batch_desc d{};
  long long graph_nodes = 0, graph_launches = 0;
  std::vector<double> box, pref;
  std::vector<long long> off;
  std::vector<int> n_charged;
  std::vector<double> sum_q2, accuracy, rs_err, ks_err;
  std::unique_ptr<Engine> eng;
  // per cao (index 1..7) the tuned choice of every replica (mesh 0: the
  // accuracy is out of reach at that cao)
  std::vector<std::vector<BatchChoice>> by_cao;
  std::vector<int> caos; // the cao of every replica
  DevBuf vel, step;
  bool forces_valid = false;
  cudaGraphExec_t graph = nullptr;
  double g_dt = 0, g_kT = -1, g_gamma = -1;
  unsigned long long g_seed = 0;
  std::string err;
  ~p3mx_batch() {
    if (graph)
      cudaGraphExecDestroy(graph);
  }
};

namespace {

bool fft_friendly(int m) {
  if (m % 2)
    return false;
  for (int p : {2, 3, 5, 7})
    while (m % p == 0)
      m /= p;
  return m == 1;
}

template <typename F> int bguard(p3mx_batch *b, F &&fn) {
  if (!b)
    return P3MX_EHANDLE;
  try {
    fn();
    b->err.clear();
    return P3MX_OK;
  } catch (Error const &e) {
    b->err = e.what();
    return e.code;
  } catch (std::exception const &e) {
    b->err = e.what();
    return P3MX_ERUNTIME;
  }
}

double rs_err_f(double pref, double r_cut_iL, int n_c, double sum_q2, double alpha_L, double L) {
  double const V = L * L * L;
  return (2. * pref * sum_q2 * std::exp(-(r_cut_iL * alpha_L) * (r_cut_iL * alpha_L))) /
         std::sqrt(static_cast<double>(n_c) * r_cut_iL * L * V);
}

// Evaluate he_q for all queries on the device.
std::vector<double> ks_heq_batch(std::vector<int2> const &mc, std::vector<double> const &aL,
                                 cudaStream_t st) {
  int const Q = static_cast<int>(mc.size());
  std::vector<double> out(Q, 0.0);
  if (Q == 0)
    return out;
  int const gx = 16;
  DevBuf dmc, dal, dpart;
  dmc.ensure(Q * sizeof(int2));
  dal.ensure(Q * sizeof(double));
  dpart.ensure(static_cast<size_t>(Q) * gx * sizeof(double));
  P3MX_CUDA(cudaMemcpyAsync(dmc.p, mc.data(), Q * sizeof(int2), cudaMemcpyHostToDevice, st));
  P3MX_CUDA(cudaMemcpyAsync(dal.p, aL.data(), Q * sizeof(double), cudaMemcpyHostToDevice, st));
  for (int q0 = 0; q0 < Q; q0 += 65535) {
    int const nq = std::min(65535, Q - q0);
    k_ks_error_batch<<<dim3(gx, nq), 256, 0, st>>>(dmc.as<int2>() + q0, dal.as<double>() + q0,
                                                   dpart.as<double>() + static_cast<size_t>(q0) * gx);
  }
  std::vector<double> part(static_cast<size_t>(Q) * gx);
  P3MX_CUDA(cudaMemcpyAsync(part.data(), dpart.p, part.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  P3MX_CUDA(cudaStreamSynchronize(st));
  for (int q = 0; q < Q; ++q)
    for (int k = 0; k < gx; ++k)
      out[q] += part[static_cast<size_t>(q) * gx + k];
  return out;
}

using Choice = BatchChoice;

// Per-replica choice of (mesh, r_cut, alpha) for one cao: lock-step
// bisection of r_cut (P3M_RCUT_PREC) over every feasible (replica, mesh)
// pair with the batched device error sum, then the mesh minimising a cost
// model of the B200 kernels (pairs, stencil points, mesh points).
std::vector<Choice> choose_for_cao(p3mx_batch *b, int cao, std::vector<int> const &meshes,
                                   cudaStream_t st) {
  int const R = b->d.n_rep;
  double const skin = b->d.skin, target = b->d.accuracy;
  struct Cand {
    int r, M;
    double lo, hi, aL;
  };
  std::vector<Cand> c;
  for (int r = 0; r < R; ++r) {
    double const L = b->box[3 * r];
    double const rmax = (0.5 * L - skin) / L;
    if (rmax <= 0 || b->n_charged[r] == 0)
      continue;
    for (int M : meshes) {
      if (cao >= M)
        continue;
      double const k_cut = (cao / 2.0) * L / M;
      if (k_cut >= L - skin || k_cut >= 0.5 * L)
        continue;
      c.push_back(Cand{r, M, 0.0, rmax, 0.1});
    }
  }
  auto alpha_for = [&](Cand const &k, double rc) {
    int const r = k.r;
    double const L = b->box[3 * r];
    double rs = rs_err_f(b->pref[r], rc, b->n_charged[r], b->sum_q2[r], 0., L);
    if (std::sqrt(2.0) * rs > target)
      return std::sqrt(std::log(std::sqrt(2.0) * rs / target)) / rc;
    return 0.1;
  };
  auto acc_all = [&](std::vector<double> const &rc, std::vector<double> &aL,
                     std::vector<double> &rs, std::vector<double> &ks) {
    std::vector<int2> mc(c.size());
    aL.resize(c.size());
    rs.resize(c.size());
    ks.resize(c.size());
    for (size_t k = 0; k < c.size(); ++k) {
      mc[k] = int2{c[k].M, cao};
      aL[k] = alpha_for(c[k], rc[k]);
    }
    auto heq = ks_heq_batch(mc, aL, st);
    std::vector<double> acc(c.size());
    for (size_t k = 0; k < c.size(); ++k) {
      int const r = c[k].r;
      double const L = b->box[3 * r];
      rs[k] = rs_err_f(b->pref[r], rc[k], b->n_charged[r], b->sum_q2[r], aL[k], L);
      ks[k] = 2. * b->pref[r] * b->sum_q2[r] * std::sqrt(heq[k] / b->n_charged[r]) / (L * L);
      acc[k] = std::hypot(rs[k], ks[k]);
    }
    return acc;
  };
  std::vector<double> rc(c.size()), aL, rs, ks;
  for (size_t k = 0; k < c.size(); ++k)
    rc[k] = c[k].hi;
  auto acc = acc_all(rc, aL, rs, ks);
  std::vector<char> ok(c.size());
  for (size_t k = 0; k < c.size(); ++k)
    ok[k] = acc[k] <= target;
  for (int it = 0; it < 40; ++it) {
    bool any = false;
    for (size_t k = 0; k < c.size(); ++k) {
      rc[k] = 0.5 * (c[k].lo + c[k].hi);
      if (ok[k] && c[k].hi - c[k].lo >= 1e-3)
        any = true;
    }
    if (!any)
      break;
    acc = acc_all(rc, aL, rs, ks);
    for (size_t k = 0; k < c.size(); ++k) {
      if (!ok[k] || c[k].hi - c[k].lo < 1e-3)
        continue;
      if (acc[k] > target)
        c[k].lo = rc[k];
      else
        c[k].hi = rc[k];
    }
  }
  for (size_t k = 0; k < c.size(); ++k)
    rc[k] = c[k].hi;
  acc = acc_all(rc, aL, rs, ks);
  std::vector<Choice> best(R);
  for (auto &x : best)
    x.cost = std::numeric_limits<double>::max();
  for (size_t k = 0; k < c.size(); ++k) {
    if (!ok[k])
      continue;
    int const r = c[k].r;
    double const L = b->box[3 * r];
    double const N = static_cast<double>(b->off[r + 1] - b->off[r]);
    double const rcut = rc[k] * L + skin;
    double const pairs = N * 4.18879 * rcut * rcut * rcut * N / (L * L * L);
    double const M3 = double(c[k].M) * c[k].M * c[k].M;
    double const cost = 0.02 * pairs + 0.006 * N * cao * cao * cao + 0.06 * M3;
    if (cost < best[r].cost) {
      best[r].cost = cost;
      best[r].mesh = c[k].M;
      best[r].r_cut_iL = rc[k];
      best[r].alpha_L = aL[k];
      best[r].acc = acc[k];
      best[r].rs = rs[k];
      best[r].ks = ks[k];
    }
  }
  return best;
}

void configure_batch(p3mx_batch *b, std::vector<int> const &caos, std::vector<Choice> const &ch) {
  std::vector<ReplicaConf> conf(b->d.n_rep);
  for (int r = 0; r < b->d.n_rep; ++r) {
    auto &c = conf[r];
    double const L = b->box[3 * r];
    for (int d = 0; d < 3; ++d) {
      c.box[d] = b->box[3 * r + d];
      c.mesh[d] = ch[r].mesh;
    }
    c.prefactor = b->pref[r];
    c.cao = caos[r];
    c.r_cut = ch[r].r_cut_iL * L;
    c.alpha = ch[r].alpha_L / L;
    c.skin = b->d.skin;
    c.p0 = b->off[r];
    c.np = b->off[r + 1] - b->off[r];
  }
  b->eng->configure(conf, b->off.back());
}

double time_batch(p3mx_batch *b, int reps) {
  Engine &e = *b->eng;
  cudaStream_t st = e.stream();
  e.invalidate_lists();
  e.long_range(e.d_force(), true, false, false, st, nullptr, nullptr);
  e.short_range(e.d_force(), false, false, st, nullptr, nullptr);
  cudaEvent_t t0, t1;
  P3MX_CUDA(cudaEventCreate(&t0));
  P3MX_CUDA(cudaEventCreate(&t1));
  P3MX_CUDA(cudaEventRecord(t0, st));
  for (int k = 0; k < reps; ++k) {
    e.long_range(e.d_force(), true, false, false, st, nullptr, nullptr);
    e.short_range(e.d_force(), false, false, st, nullptr, nullptr);
  }
  P3MX_CUDA(cudaEventRecord(t1, st));
  P3MX_CUDA(cudaEventSynchronize(t1));
  float ms = 0;
  P3MX_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  return ms / reps;
}

void batch_forces(p3mx_batch *b, cudaStream_t st, bool graph_mode) {
  Engine &e = *b->eng;
  e.long_range(e.d_force(), true, false, false, st, nullptr, nullptr);
  if (graph_mode)
    e.short_range_graph(e.d_force(), false, st);
  else
    e.short_range(e.d_force(), false, false, st, nullptr, nullptr);
  e.bond_forces(e.d_force(), st);
}

} // namespace

extern "C" {

int p3mx_batch_create(const p3mx_batch_desc *d, const double *pos, const double *q,
                      const int *type, int ntypes, const p3mx_pair_params *table,
                      p3mx_batch **out) {
  if (!d || !out || !pos || !q)
    return P3MX_EHANDLE;
  auto b = std::make_unique<p3mx_batch>();
  b->d = *d;
  int const rc = bguard(b.get(), [&] {
    int const R = d->n_rep;
    if (R < 1 || !d->box || !d->prefactor || !d->offset)
      throw Error(P3MX_EDOMAIN, "batch needs n_rep >= 1, box, prefactor and offset arrays");
    if (d->accuracy <= 0.)
      throw Error(P3MX_EDOMAIN, "Parameter 'accuracy' must be > 0");
    if (d->cao_min < 1 || d->cao_max > 7 || d->cao_min > d->cao_max)
      throw Error(P3MX_EDOMAIN, "Parameter 'cao' must be >= 1 and <= 7");
    if (d->mesh_min < 2 || d->mesh_max < d->mesh_min)
      throw Error(P3MX_EDOMAIN, "Parameter 'mesh' must be > 0");
    b->box.assign(d->box, d->box + 3 * R);
    b->pref.assign(d->prefactor, d->prefactor + R);
    b->off.assign(d->offset, d->offset + R + 1);
    for (int r = 0; r < R; ++r) {
      if (b->pref[r] <= 0.)
        throw Error(P3MX_EDOMAIN, "Parameter 'prefactor' must be > 0");
      if (b->box[3 * r] != b->box[3 * r + 1] || b->box[3 * r] != b->box[3 * r + 2])
        throw Error(P3MX_EDOMAIN, "batched replicas must be cubic boxes");
      if (b->off[r + 1] < b->off[r])
        throw Error(P3MX_EDOMAIN, "replica offsets must be non-decreasing");
    }
    long long const N = b->off[R];
    // charge census per replica
    b->n_charged.assign(R, 0);
    b->sum_q2.assign(R, 0.);
    for (int r = 0; r < R; ++r)
      for (long long i = b->off[r]; i < b->off[r + 1]; ++i)
        if (q[i] != 0.) {
          b->n_charged[r]++;
          b->sum_q2[r] += q[i] * q[i];
        }
    b->eng = std::make_unique<Engine>(d->single_precision != 0);
    Engine &e = *b->eng;
    // pair table
    std::vector<PairIA> tab(static_cast<size_t>(std::max(1, ntypes)) * std::max(1, ntypes),
                            PairIA{0, 0, 0, 0, 0, 0, 0, 0, 0, -1.0});
    if (table && ntypes >= 1) {
      for (int k = 0; k < ntypes * ntypes; ++k) {
        auto const &s = table[k];
        PairIA &t = tab[k];
        t.lj_eps = s.lj_eps;
        t.lj_sig = s.lj_sig;
        t.lj_cut = s.lj_cut;
        t.lj_shift = s.lj_shift;
        t.lj_offset = s.lj_offset;
        t.lj_min = std::max(0., s.lj_min);
        t.wca_eps = s.wca_eps;
        t.wca_sig = s.wca_sig;
        t.wca_cut = s.wca_sig != 0. ? s.wca_sig * std::pow(2., 1. / 6.) : 0.;
        double ic = -1.0;
        if (s.lj_cut > 0. && s.lj_eps != 0.)
          ic = std::max(ic, s.lj_cut + s.lj_offset);
        if (t.wca_cut > 0. && s.wca_eps != 0.)
          ic = std::max(ic, t.wca_cut);
        t.ia_cut = ic;
      }
    }
    e.set_pair_table(std::max(1, ntypes), tab);
    // autotuner: per cao, per-replica mesh/r_cut/alpha, then timed trials
    std::vector<int> meshes;
    for (int m = d->mesh_min + (d->mesh_min % 2); m <= d->mesh_max; m += 2)
      if (fft_friendly(m))
        meshes.push_back(m);
    if (meshes.empty())
      throw Error(P3MX_EDOMAIN, "no FFT-friendly even mesh in [mesh_min, mesh_max]");
    // per cao: every replica's best (mesh, r_cut, alpha) by the error
    // estimate and the cost model; uncharged replicas get the smallest mesh
    std::vector<std::vector<Choice>> by_cao(8);
    std::vector<char> cao_ok(8, 0);
    for (int cao = d->cao_min; cao <= d->cao_max; ++cao) {
      auto ch = choose_for_cao(b.get(), cao, meshes, e.stream());
      bool feasible = true;
      for (int r = 0; r < R; ++r)
        if (b->n_charged[r] > 0 && ch[r].mesh == 0)
          feasible = false;
      for (int r = 0; r < R; ++r)
        if (ch[r].mesh == 0 && b->n_charged[r] == 0) {
          ch[r].mesh = std::max(meshes[0], cao + 2);
          ch[r].r_cut_iL = 1e-6;
          ch[r].alpha_L = 1.0;
          ch[r].cost = 0.0;
        }
      by_cao[cao] = ch;
      cao_ok[cao] = feasible;
    }
    // candidate assignments: one cao for every replica (each feasible cao),
    // and per replica the cao of lowest model cost among those that reach the
    // accuracy for it; the timed trials pick the fastest
    std::vector<std::vector<int>> cands;
    for (int cao = d->cao_min; cao <= d->cao_max; ++cao)
      if (cao_ok[cao])
        cands.push_back(std::vector<int>(R, cao));
    {
      std::vector<int> mix(R, -1);
      bool ok = true;
      for (int r = 0; r < R; ++r) {
        double best = std::numeric_limits<double>::max();
        for (int cao = d->cao_min; cao <= d->cao_max; ++cao) {
          auto const &ch = by_cao[cao];
          if (ch.empty() || ch[r].mesh == 0)
            continue;
          if (ch[r].cost < best) {
            best = ch[r].cost;
            mix[r] = cao;
          }
        }
        ok = ok && mix[r] > 0;
      }
      if (ok && std::find(cands.begin(), cands.end(), mix) == cands.end())
        cands.push_back(mix);
    }
    if (cands.empty())
      throw Error(P3MX_ERUNTIME, "CoulombP3MGPU: failed to reach requested accuracy");
    auto choices_of = [&](std::vector<int> const &caos) {
      std::vector<Choice> ch(R);
      for (int r = 0; r < R; ++r)
        ch[r] = by_cao[caos[r]][r];
      return ch;
    };
    double best_t = std::numeric_limits<double>::max();
    std::vector<int> best_caos;
    for (auto const &caos : cands) {
      configure_batch(b.get(), caos, choices_of(caos));
      e.upload(pos, q, type, false, e.stream());
      e.census(e.stream());
      double const t = time_batch(b.get(), 3);
      if (t < best_t) {
        best_t = t;
        best_caos = caos;
      }
    }
    std::vector<Choice> const best_ch = choices_of(best_caos);
    configure_batch(b.get(), best_caos, best_ch);
    e.upload(pos, q, type, false, e.stream());
    e.census(e.stream());
    b->by_cao = by_cao;
    b->caos = best_caos;
    b->accuracy.resize(R);
    b->rs_err.resize(R);
    b->ks_err.resize(R);
    for (int r = 0; r < R; ++r) {
      b->accuracy[r] = best_ch[r].acc;
      b->rs_err[r] = best_ch[r].rs;
      b->ks_err[r] = best_ch[r].ks;
    }
    b->vel.ensure(3 * std::max<long long>(1, N) * sizeof(double));
    P3MX_CUDA(cudaMemsetAsync(b->vel.p, 0, 3 * std::max<long long>(1, N) * sizeof(double), e.stream()));
    b->step.ensure(sizeof(unsigned long long));
    P3MX_CUDA(cudaMemsetAsync(b->step.p, 0, sizeof(unsigned long long), e.stream()));
    P3MX_CUDA(cudaStreamSynchronize(e.stream()));
  });
  *out = b.release();
  return rc;
}

void p3mx_batch_destroy(p3mx_batch *b) { delete b; }

const char *p3mx_batch_last_error(const p3mx_batch *b) { return b ? b->err.c_str() : "NULL batch"; }

int p3mx_batch_get_tuned(const p3mx_batch *b, int r, p3mx_tuned *out) {
  if (!b || !out || !b->eng)
    return P3MX_EHANDLE;
  if (r < 0 || r >= b->d.n_rep)
    return P3MX_EDOMAIN;
  auto const &c = b->eng->conf(r);
  for (int d = 0; d < 3; ++d) {
    out->mesh[d] = c.mesh[d];
    out->mesh_off[d] = c.mesh_off[d];
    out->a[d] = c.box[d] / c.mesh[d];
  }
  out->cao = c.cao;
  out->r_cut = c.r_cut;
  out->alpha = c.alpha;
  out->r_cut_iL = c.r_cut / c.box[0];
  out->alpha_L = c.alpha * c.box[0];
  out->accuracy = b->accuracy[r];
  out->epsilon = 0.;
  out->is_tuned = 1;
  out->single_precision = b->d.single_precision;
  out->rs_error = b->rs_err[r];
  out->ks_error = b->ks_err[r];
  return P3MX_OK;
}

int p3mx_batch_forces(p3mx_batch *b, double *energy_out) {
  return bguard(b, [&] {
    Engine &e = *b->eng;
    cudaStream_t st = e.stream();
    int const R = b->d.n_rep;
    std::vector<double> ek, es;
    e.long_range(e.d_force(), true, energy_out != nullptr, false, st, &ek, nullptr);
    e.short_range(e.d_force(), false, energy_out != nullptr, st, &es, nullptr);
    e.bond_forces(e.d_force(), st);
    if (energy_out) {
      std::vector<double> const eb = e.bond_energies(st);
      for (int r = 0; r < R; ++r)
        energy_out[r] = ek[r] + es[2 * r] + es[2 * r + 1] + eb[r];
    }
    P3MX_CUDA(cudaStreamSynchronize(st));
    e.check_kernel_error(st);
    b->forces_valid = true;
  });
}

int p3mx_batch_run(p3mx_batch *b, int steps, double dt, double kT, double gamma,
                   unsigned long long seed) {
  return bguard(b, [&] {
    if (steps < 0 || dt <= 0.)
      throw Error(P3MX_EDOMAIN, "steps must be >= 0 and dt > 0");
    Engine &e = *b->eng;
    cudaStream_t st = e.stream();
    long long const N = e.n_part();
    long long const n3 = 3 * N;
    double const noise = (kT > 0. && gamma > 0.) ? std::sqrt(24.0 * kT * gamma / dt) : 0.0;
    double const g = (gamma > 0.) ? gamma : 0.0;
    auto *stp = b->step.as<unsigned long long>();
    auto enqueue_forces = [&](bool graph_mode) {
      batch_forces(b, st, graph_mode);
      if (noise > 0. || g > 0.)
        k_langevin<<<ceil_div(N, 256), 256, 0, st>>>(e.d_force(), b->vel.as<double>(), N, g, noise,
                                                     seed, stp);
    };
    if (!b->forces_valid) {
      e.ensure_lists(st, 2.0);
      enqueue_forces(false);
      b->forces_valid = true;
    }
    e.ensure_lists(st, 2.0);
    bool const reuse = b->graph && b->g_dt == dt && b->g_kT == kT && b->g_gamma == gamma &&
                       b->g_seed == seed;
    if (!reuse) {
      if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
      }
      cudaGraph_t gr;
      P3MX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      k_vv_step1<<<ceil_div(n3, 256), 256, 0, st>>>(e.d_pos(), b->vel.as<double>(), e.d_force(), n3, dt);
      enqueue_forces(true);
      k_vv_step2<<<ceil_div(n3, 256), 256, 0, st>>>(b->vel.as<double>(), e.d_force(), n3, dt);
      k_step_inc<<<1, 1, 0, st>>>(stp);
      P3MX_CUDA(cudaStreamEndCapture(st, &gr));
      size_t nodes = 0;
      P3MX_CUDA(cudaGraphGetNodes(gr, nullptr, &nodes));
      b->graph_nodes = static_cast<long long>(nodes);
      P3MX_CUDA(cudaGraphInstantiate(&b->graph, gr, 0));
      cudaGraphDestroy(gr);
      b->g_dt = dt;
      b->g_kT = kT;
      b->g_gamma = gamma;
      b->g_seed = seed;
    }
    for (int s = 0; s < steps; ++s)
      P3MX_CUDA(cudaGraphLaunch(b->graph, st));
    b->graph_launches += steps;
    P3MX_CUDA(cudaStreamSynchronize(st));
    e.check_kernel_error(st);
    if (e.list_overflow(st))
      throw Error(P3MX_ERUNTIME, "Verlet list capacity exceeded during the graph run");
  });
}

int p3mx_batch_set_cao(p3mx_batch *b, const int *cao) {
  return bguard(b, [&] {
    if (!cao)
      throw Error(P3MX_EHANDLE, "cao array must not be NULL");
    int const R = b->d.n_rep;
    std::vector<int> caos(cao, cao + R);
    std::vector<BatchChoice> ch(R);
    for (int r = 0; r < R; ++r) {
      if (caos[r] < b->d.cao_min || caos[r] > b->d.cao_max)
        throw Error(P3MX_EDOMAIN, "cao of replica " + std::to_string(r) +
                                      " outside the batch's [cao_min, cao_max]");
      auto const &bc = b->by_cao[caos[r]];
      if (bc.empty() || bc[r].mesh == 0)
        throw Error(P3MX_EDOMAIN, "replica " + std::to_string(r) +
                                      " cannot reach the accuracy with cao " +
                                      std::to_string(caos[r]));
      ch[r] = bc[r];
    }
    Engine &e = *b->eng;
    cudaStream_t st = e.stream();
    long long const N = e.n_part();
    // keep the current particles across the reconfiguration
    DevBuf xp, qp, tp;
    xp.ensure(3 * std::max<long long>(1, N) * sizeof(double));
    qp.ensure(std::max<long long>(1, N) * sizeof(double));
    tp.ensure(std::max<long long>(1, N) * sizeof(int));
    if (N > 0) {
      P3MX_CUDA(cudaMemcpyAsync(xp.p, e.d_pos(), 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, st));
      P3MX_CUDA(cudaMemcpyAsync(qp.p, e.d_q(), N * sizeof(double), cudaMemcpyDeviceToDevice, st));
      P3MX_CUDA(cudaMemcpyAsync(tp.p, e.d_type(), N * sizeof(int), cudaMemcpyDeviceToDevice, st));
    }
    configure_batch(b, caos, ch);
    e.upload(xp.as<double>(), qp.as<double>(), tp.as<int>(), true, st);
    e.census(st);
    P3MX_CUDA(cudaStreamSynchronize(st));
    b->caos = caos;
    for (int r = 0; r < R; ++r) {
      b->accuracy[r] = ch[r].acc;
      b->rs_err[r] = ch[r].rs;
      b->ks_err[r] = ch[r].ks;
    }
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    b->forces_valid = false;
  });
}

int p3mx_batch_set_bonds(p3mx_batch *b, int n_types, const p3mx_bond_params *types,
                         size_t n_bonds, const int *bonds) {
  return bguard(b, [&] {
    std::vector<BondParam> const t = bond_types_from_abi(n_types, types, n_bonds, bonds);
    // both partners of a bond in one replica (offsets are replica starts)
    auto rep = [&](int i) {
      return static_cast<int>(std::upper_bound(b->off.begin(), b->off.end(),
                                               static_cast<long long>(i)) -
                              b->off.begin()) - 1;
    };
    for (size_t k = 0; k < n_bonds; ++k)
      if (rep(bonds[3 * k + 1]) != rep(bonds[3 * k + 2]))
        throw Error(P3MX_EDOMAIN, "bond between particles " + std::to_string(bonds[3 * k + 1]) +
                                      " and " + std::to_string(bonds[3 * k + 2]) +
                                      " of different replicas");
    Engine &e = *b->eng;
    e.set_bonds(t, std::vector<int>(bonds, bonds + 3 * n_bonds), e.stream());
    // the captured step holds the old bond tables (or none): capture anew
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    b->forces_valid = false;
  });
}

int p3mx_batch_profile(p3mx_batch *b, int reps, double *ms, const char **names, int cap,
                       int *nstages) {
  return bguard(b, [&] {
    static std::vector<std::string> keep;
    Engine &e = *b->eng;
    e.ensure_lists(e.stream(), 2.0);
    auto prof = e.profile(std::max(1, reps), e.stream());
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
    b->forces_valid = false;
  });
}

void *p3mx_batch_stream(const p3mx_batch *b) {
  return (b && b->eng) ? static_cast<void *>(b->eng->stream()) : nullptr;
}

int p3mx_batch_launch_count(const p3mx_batch *b, long long *count) {
  if (!b || !count || !b->eng)
    return P3MX_EHANDLE;
  // kernel nodes of the captured step (memset nodes included) times launches,
  // plus the kernels launched outside graphs
  *count = b->eng->launches() + b->graph_nodes * b->graph_launches;
  return P3MX_OK;
}

int p3mx_batch_get(p3mx_batch *b, double *pos, double *f, double *vel) {
  return bguard(b, [&] {
    Engine &e = *b->eng;
    cudaStream_t st = e.stream();
    size_t const bytes = 3 * static_cast<size_t>(e.n_part()) * sizeof(double);
    if (pos)
      P3MX_CUDA(cudaMemcpyAsync(pos, e.d_pos(), bytes, cudaMemcpyDeviceToHost, st));
    if (f)
      P3MX_CUDA(cudaMemcpyAsync(f, e.d_force(), bytes, cudaMemcpyDeviceToHost, st));
    if (vel)
      P3MX_CUDA(cudaMemcpyAsync(vel, b->vel.p, bytes, cudaMemcpyDeviceToHost, st));
    P3MX_CUDA(cudaStreamSynchronize(st));
  });
}

} // extern "C"
