// Host-side engine: owns device buffers, FFT plans and block tables for a
// batch of one or more independent periodic systems (replicas), and runs
// the long-range (P3M) and short-range (pair) pipelines on one stream.
#pragma once

#include "common.cuh"
#include "fft.cuh"
#include "pair.cuh"
#include "bonds.cuh"

#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace p3mx {

// Raw device buffer with grow-only reallocation.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(DevBuf const &) = delete;
  DevBuf &operator=(DevBuf const &) = delete;
  ~DevBuf() {
    if (p)
      cudaFree(p);
  }
  void ensure(size_t nbytes) {
    if (nbytes <= bytes && p)
      return;
    if (p)
      cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t const want = nbytes ? nbytes : 16;
    if (cudaMalloc(&p, want) != cudaSuccess) {
      cudaGetLastError();
      throw Error(4, "device allocation of " + std::to_string(want) + " bytes failed");
    }
    bytes = want;
  }
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Host-side configuration of one replica.
struct ReplicaConf {
  double box[3] = {0, 0, 0};
  double prefactor = 0.0;
  double epsilon = 0.0;
  double mesh_off[3] = {0.5, 0.5, 0.5};
  int mesh[3] = {0, 0, 0};
  int cao = 0;
  double alpha = 0.0;
  double r_cut = 0.0;
  double skin = 0.4;
  long long p0 = 0, np = 0;
};

struct Timing {
  float ms_long = 0.f, ms_short = 0.f;
};

class Dp3mEngine;

class Engine {
  friend class Dp3mEngine; // the dipolar P3M pipeline drives the mesh stages
public:
  explicit Engine(bool fp32);
  ~Engine();

  bool fp32() const { return m_fp32; }
  int n_rep() const { return static_cast<int>(m_conf.size()); }
  long long n_part() const { return m_n; }
  ReplicaConf const &conf(int r) const { return m_conf[r]; }
  cudaStream_t stream() const { return m_stream; }

  // (Re)builds geometry, plans, block tables; allocates the buffers.
  void configure(std::vector<ReplicaConf> const &conf, long long n_total);
  // LJ/WCA table (ntypes^2 entries, symmetric).
  void set_pair_table(int ntypes, std::vector<PairIA> const &tab);

  // Device-resident particle arrays in user order (AoS positions/forces).
  double *d_pos() const { return m_pos.as<double>(); }
  double *d_q() const { return m_q.as<double>(); }
  int *d_type() const { return m_type.as<int>(); }
  double *d_force() const { return m_force.as<double>(); }
  void upload(const double *pos, const double *q, const int *type, bool device_ptrs,
              cudaStream_t st);
  void upload_positions(const double *pos, bool device_ptrs, cudaStream_t st);

  // Charge census (n_charged, sum q, sum q^2, dipole) per replica -> host.
  void census(cudaStream_t st);
  std::vector<double> const &census_host() const { return m_census_h; }

  // k-space pipeline for all replicas.  f: device force array (3N) or
  // nullptr; energies[r], virial[r*9] written on the host if requested.
  void long_range(double *f, bool overwrite, bool want_energy, bool want_virial,
                  cudaStream_t st, std::vector<double> *energies,
                  std::vector<double> *virials);
  // Real-space + LJ/WCA over Verlet lists.  energies[r*2], virials[r*18].
  // fp64_math runs the pair arithmetic in FP64 even on an FP32-mixed engine
  // (observables of the FP32-mixed actor are evaluated in FP64).
  void short_range(double *f, bool overwrite, bool want_ev, cudaStream_t st,
                   std::vector<double> *energies, std::vector<double> *virials,
                   bool fp64_math = false);
  // Forces of the whole path (k-space + real-space + LJ/WCA), no energies:
  // the k-space chain, the list check, then the pair kernel, on one stream.
  void forces_all(double *f, bool overwrite, cudaStream_t st);
  // Graph-capturable short-range evaluation (device-side rebuild decision).
  void short_range_graph(double *f, bool overwrite, cudaStream_t st);
  // Build lists now if invalid (capacity margin factor for graph use).
  void ensure_lists(cudaStream_t st, double nb_margin = 1.5);
  // Largest neighbour count that did not fit (0 if none) since last reset.
  int list_overflow(cudaStream_t st);
  // Force the next short_range call to rebuild cells and lists.
  void invalidate_lists() { m_lists_valid = false; }

  // Introspection for parity tests.
  std::vector<int> cell_index_ghost(cudaStream_t st);
  std::vector<int> verlet_pairs(cudaStream_t st);
  std::vector<double> mesh_copy(int r, cudaStream_t st);
  void cell_grid(int r, int *cg, double *cs) const;

  // Per-stage device times (ms, mean of reps) of one full force evaluation,
  // measured with CUDA events between the stages on the stream.
  std::vector<std::pair<std::string, double>> profile(int reps, cudaStream_t st);
  // Throws if a kernel reported that a bounded wait ran out (synchronises st).
  void check_kernel_error(cudaStream_t st);
  // Pair bonds (bonds.cuh): `bonds` holds (type, i, j) triples of particle
  // indices; forces are added by the force paths, observables on request.
  void set_bonds(std::vector<BondParam> const &types, std::vector<int> const &bonds,
                 cudaStream_t st);
  void bond_forces(double *f, cudaStream_t st);
  // ELC with dielectric contrasts: every charged particle within sl of a
  // wall feels its own image and, over its Verlet partners, the partners'
  // interaction with its image (added to f; energy sum with energy != null)
  void elc_image_pairs(double sl, double h, double db, double dt, double *f, double *energy,
                       cudaStream_t st);
  void bond_observables(cudaStream_t st, double *energy, double *virial9);
  // bonded energy of every replica (zeros without bonds); synchronises
  std::vector<double> bond_energies(cudaStream_t st);
  bool has_bonds() const { return m_nbonds > 0; }
  // Number of kernels launched by this engine so far.
  long long launches() const { return m_launches; }

  // k-space error sum (device, FP64) for tuning.
  double ks_error(const int *mesh, int cao, int n_c_part, double sum_q2, double alpha_L,
                  const double *box, double prefactor);

private:
  template <typename Real> void long_range_t(double *f, bool overwrite, bool want_e, bool want_v,
                                             cudaStream_t st);
  template <typename Real> void short_range_t(double *f, bool overwrite, bool want_ev,
                                              cudaStream_t st);
  template <typename Real>
  void launch_fft_y(void *c0, long long field_stride, int nf, bool inv, cudaStream_t st);
  template <typename Real> void launch_pair(double *f, bool overwrite, bool want_ev,
                                            cudaStream_t st);
  void prepare_short_range(cudaStream_t st, bool need_spq);
  // the list check of prepare_short_range issued early: its flag lands in
  // pinned host memory behind m_check_ev, so the host can wait for it while
  // later work keeps the GPU busy; prepare_short_range consumes it
  void check_lists(cudaStream_t st, bool need_spq);
  void build_lists(cudaStream_t st);
  void set_list_capacity(double margin);
  void layout_lists(cudaStream_t st);
  void encode_field_maps(cudaStream_t st);
  // want_spq: also the FP64 double4 positions (FP64 pair kernel)
  void refresh_sorted_positions(cudaStream_t st, bool want_spq = true);
  // Counting sort by key (perm: sorted position -> particle); index_order
  // orders each bucket by particle index (deterministic), else the order
  // inside a bucket is that of the atomic slots.
  void sort_keys(int *key, int *slot, int *cnt, int *start, int *perm, long long nkeys,
                 cudaStream_t st, const int *cond = nullptr, bool index_order = true);

  void mark(const char *name, cudaStream_t st);

  bool m_fp32;
  cudaStream_t m_stream = nullptr;
  long long m_launches = 0;
  bool m_profiling = false;
  std::vector<std::pair<std::string, cudaEvent_t>> m_marks;
  std::vector<ReplicaConf> m_conf;
  std::vector<RepGeom> m_geom;
  long long m_n = 0;
  long long m_bins = 0, m_cplx = 0, m_cells = 0, m_nkeys = 0; // m_nkeys: bricks (sort keys)
  long long m_ebins = 0; // field mesh records (ghost layers included)
  long long m_ncorner = 0; // corner keys (bricks x brick^3)
  int m_n_bricks = 0; // sort bricks of all replicas (interpolation blocks)
  int m_sb_edge = 16; // super-brick edge of the charge assignment (16, or 8 for small meshes)
  std::vector<int> m_phase_off; // assignment super-brick table offsets per (cao, colour) phase
  std::vector<int> m_phase_cao; // the cao of each phase
  std::vector<int> m_brick_off; // interpolation brick table offsets per cao (index cao .. cao+1)
  int m_ntypes = 1;
  std::vector<PairIA> m_ia;

  // tables
  DevBuf m_geom_d, m_rep_of, m_tw, m_ia_d;
  DevBuf m_blk_mesh; // super-bricks of the charge assignment, grouped by colour
  DevBuf m_blk_cplx, m_blk_census, m_blk_pair;
  DevBuf m_blk_brick; // all bricks in spatial order (interpolation)
  DevBuf m_blk_zf, m_blk_y, m_blk_x, m_blk_zi;
  std::vector<int> m_blk_x_start, m_blk_census_start, m_blk_pair_start;
  DevBuf m_blk_x_start_d, m_blk_census_start_d, m_blk_pair_start_d;
  int m_n_blk_mesh = 0, m_n_blk_cplx = 0, m_n_blk_census = 0, m_n_blk_pair = 0;
  int m_n_blk_zf = 0, m_n_blk_y = 0, m_n_blk_x = 0, m_n_blk_zi = 0;
  int m_tile_y = 16, m_tile_x = 16;
  bool m_yin = true;  // every replica's y lines transform in place
  size_t m_smem_zf = 0, m_smem_y = 0, m_smem_x = 0, m_smem_zi = 0;

  // particles
  DevBuf m_pos, m_q, m_type, m_force;
  // p3m
  DevBuf m_key, m_bkey, m_slot, m_cnt, m_start, m_perm, m_scan_tiles;
  DevBuf m_dist, m_W, m_skey;
  DevBuf m_rho, m_ck, m_field, m_E, m_ginf;
  DevBuf m_tmap; // per replica: tensor map of its field mesh (interpolation tiles)
  DevBuf m_part_x, m_part_census, m_sums_x, m_sums_census, m_dipole;
  bool m_ginf_valid = false;
  std::vector<double> m_census_h;
  // short range
  DevBuf m_ckey, m_cslot, m_ccnt, m_cstart, m_cperm, m_pq, m_spq, m_spf, m_stype, m_scell;
  DevBuf m_cinv; // sorted slot of each particle (inverse of m_cperm)
  DevBuf m_cbkey; // cell-octant key of each particle (sort key of the cell sort)
  long long m_oct_mult = 1; // cell-sort keys per cell (8 with octant-sorted replicas)
  DevBuf m_elc_epart;
  DevBuf m_nb, m_nb_cnt, m_overflow, m_pos_ref, m_flag, m_rflag, m_part_pair, m_sums_pair;
  DevBuf m_type_ref; // types at the last list build (a change triggers a rebuild)
  // kernel error word: [0] a bounded wait ran out; [1] bond status (1 broken,
  // 2 zero length), [2], [3] the two particles of the first failing bond
  DevBuf m_kerr;
  long long m_nbonds = 0, m_bond_n = 0; // bonds, particle count they were set for
  DevBuf m_bstart, m_bent, m_bparam, m_bpart;
  std::vector<int> m_cap; // neighbour capacity per replica
  bool m_lists_valid = false;
  // pending early list check (check_lists): rebuild regardless, or read the
  // flag copied to m_flag_host once m_check_ev has completed
  bool m_check_pending = false, m_check_rebuild = false;
  int *m_flag_host = nullptr;
  cudaEvent_t m_check_ev = nullptr;
  DevBuf m_chk;       // the check's two flag words (slot m_chk_slot is next)
  int m_chk_slot = 0;
  // misc host staging
  DevBuf m_ks_part;
};

} // namespace p3mx
