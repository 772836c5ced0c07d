/*
 * p3mx -- B200-native P3M electrostatics + short-range pair engine.
 *
 * C ABI of the drop-in boundary.  Every entry point returns 0 on success or
 * a non-zero P3MX_E* status; the message of the last failure is available
 * from p3mx_last_error().  Nothing here throws or calls exit() (the
 * reference exits the process on CUDA errors, src/core/cuda/utils.cuh:64-80).
 *
 * Pointers: positions/charges/forces are plain FP64 arrays in AoS layout
 * (x0 y0 z0 x1 ...), as ESPResSo's Particle::pos()/force() hold them.  With
 * P3MX_DEVICE_PTRS in `flags` they are device pointers already resident in
 * HBM; otherwise they are host pointers and the call copies them in and out
 * (the GpuParticleData gather/scatter of system/GpuParticleData.cpp:85-184).
 * `stream` is a cudaStream_t (NULL = the handle's own stream).
 */
#ifndef P3MX_H
#define P3MX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P3MX_OK 0
#define P3MX_EDOMAIN 1    /* parameter outside its domain (std::domain_error) */
#define P3MX_ERUNTIME 2   /* state error (std::runtime_error in the reference) */
#define P3MX_ECUDA 3      /* CUDA runtime error */
#define P3MX_ENOMEM 4     /* device allocation failed */
#define P3MX_EHANDLE 5    /* NULL or destroyed handle */

#define P3MX_DEVICE_PTRS 1u   /* pos/q/f/type are device pointers */
#define P3MX_FORCES 2u        /* compute forces (added to f) */
#define P3MX_ENERGY 4u        /* compute energy */
#define P3MX_VIRIAL 8u        /* compute the 3x3 virial / pressure tensor */
#define P3MX_OVERWRITE 16u    /* f is overwritten instead of accumulated */
/* FP32-mixed actor only: evaluate energy/virial with the FP32 pipeline too.
 * By default the FP32-mixed actor evaluates these observables in FP64, as
 * the reference GPU actor does with its double-precision CPU kernels. */
#define P3MX_MIXED_OBSERVABLES 32u

typedef struct p3mx_handle p3mx_handle;

/* Actor parameters: the kwargs of espressomd.electrostatics.P3M / P3MGPU
 * (src/python/espressomd/electrostatics.py:129-284) and the
 * P3MParameters constructor (src/core/p3m/common.hpp:59-150).  -1 marks a
 * value left to the tuner. */
typedef struct {
  double prefactor;
  double accuracy;
  int mesh[3];
  int cao;
  double r_cut;
  double alpha;
  double epsilon;       /* 0 = metallic */
  double mesh_off[3];   /* -1 = P3M_MESHOFF (0.5) */
  int tune;             /* bool */
  int timings;          /* force evaluations timed per tuning trial */
  int verbose;          /* print the tuning log */
  int single_precision; /* 1 = FP32-mixed mesh/FFT path, 0 = plain FP64 */
  int check_neutrality;
  double charge_neutrality_tolerance; /* reference default 2e-12 */
} p3mx_params;

/* Geometry and cell-system settings (BoxGeometry + CellStructure skin). */
typedef struct {
  double box[3];
  double skin;
  int periodic[3];
} p3mx_system;

/* Read-only parameter view: the getters of CoulombP3M<Arch>
 * (src/script_interface/electrostatics/CoulombP3M.hpp:67-99). */
typedef struct {
  int mesh[3];
  int cao;
  double r_cut, alpha, r_cut_iL, alpha_L, accuracy, epsilon;
  double mesh_off[3];
  double a[3];
  int is_tuned;
  int single_precision;
  double rs_error, ks_error;
} p3mx_tuned;

/* LJ and WCA parameters of one type pair
 * (src/core/nonbonded_interactions/lj.cpp:33-46, wca.cpp:31-42). */
typedef struct {
  double lj_eps, lj_sig, lj_cut, lj_shift, lj_offset, lj_min;
  double wca_eps, wca_sig;
} p3mx_pair_params;

/* --- actor life cycle ------------------------------------------------- */

/* Validates and stores the parameters; replaces the constructor path
 * CoulombP3M<Arch>::do_construct + new_p3m_handle
 * (script_interface/electrostatics/CoulombP3M.hpp:102-142,
 *  core/electrostatics/p3m.impl.hpp:390-401). */
int p3mx_create(const p3mx_params *params, p3mx_handle **out);
void p3mx_destroy(p3mx_handle *h);
const char *p3mx_last_error(const p3mx_handle *h);
/* Version and build string ("p3mx <ver> sm_100a ..."). */
const char *p3mx_version(void);

/* Box / skin change: CoulombP3M::on_boxl_change -> scaleby_box_l
 * (electrostatics/p3m.cpp:856-865) and the cell-system rebuild. */
int p3mx_set_system(p3mx_handle *h, const p3mx_system *sys);

/* Activation: sanity checks + charge counting + (optional) tuning + init,
 * CoulombP3MImpl::on_activation / tune / init
 * (p3m.impl.hpp:328-343, p3m.cpp:758-791, p3m.cpp:246-280 and
 *  p3m_gpu_init, p3m_gpu_cuda.cu:549-667).  Positions/charges are needed
 * for the charge count and the timed tuning trials. */
int p3mx_activate(p3mx_handle *h, size_t n, const double *pos,
                  const double *q, unsigned flags);
int p3mx_get_tuned(const p3mx_handle *h, p3mx_tuned *out);

/* --- force / energy / pressure ---------------------------------------- */

/* k-space part: replaces CoulombP3MImpl::add_long_range_forces,
 * long_range_energy and long_range_pressure (p3m.impl.hpp:345-358,
 * p3m.cpp:394-592) and the GPU entry p3m_gpu_add_farfield_force
 * (p3m_gpu_cuda.cuh:31-35).  energy: 1 double; virial9: 3x3 k-space
 * pressure tensor times volume (as long_range_pressure returns it). */
int p3mx_long_range(p3mx_handle *h, size_t n, const double *pos,
                    const double *q, double *f, double *energy,
                    double *virial9, unsigned flags, void *stream);

/* Short-range part over the cell system: real-space Coulomb
 * (CoulombP3M::pair_force / pair_energy, electrostatics/p3m.hpp:146-180)
 * plus LJ/WCA (lj.hpp:41-60, wca.hpp:39-55) through the Verlet list
 * (CellStructure::verlet_list_loop, CellStructure.hpp:612-646).
 * energy2 = {coulomb real space, non-bonded}; virial18 = two 3x3 tensors
 * (coulomb, non-bonded), each sum over pairs of F (x) d. */
int p3mx_set_pair_params(p3mx_handle *h, int ntypes,
                         const p3mx_pair_params *table);
int p3mx_short_range(p3mx_handle *h, size_t n, const double *pos,
                     const double *q, const int *type, double *f,
                     double *energy2, double *virial18, unsigned flags,
                     void *stream);

/* Pair bonds: FENE (bonded_interactions/fene.hpp:37-105) and harmonic
 * (harmonic.hpp:35-93) over the minimum-image vector d = x_i - x_j, i
 * getting F(d) and j -F(d) (add_bonded_two_body_force,
 * forces_inline.hpp:320-350).  types[t] describes bond type t; bonds[3b] =
 * type, bonds[3b+1] = i, bonds[3b+2] = j (particle indices).  The call
 * replaces the bonds set before (n_bonds 0 clears them).  p3mx_forces and
 * p3mx_short_range add the bond forces; a bond stretched past its range
 * fails the call with P3MX_ERUNTIME and "bond broken between particles i,
 * j" (bond_error.cpp:28-35), a zero-length bond with r0 > 0 likewise (the
 * reference's zero-distance runtime error).  No counterpart in the
 * reference's GPU path, which has no bonded kernels. */
#define P3MX_BOND_FENE 1
#define P3MX_BOND_HARMONIC 2
typedef struct {
  int kind;     /* P3MX_BOND_FENE or P3MX_BOND_HARMONIC */
  double k;     /* spring constant */
  double r0;    /* equilibrium length */
  double r_max; /* FENE: d_r_max (largest r - r0); harmonic: r_cut (0: none) */
} p3mx_bond_params;
int p3mx_set_bonds(p3mx_handle *h, int n_types, const p3mx_bond_params *types,
                   size_t n_bonds, const int *bonds);
/* Bonded energy and virial (sum over bonds of F (x) d, 3x3) of the
 * configuration pos (device pointer with P3MX_DEVICE_PTRS in flags). */
int p3mx_bond_observables(p3mx_handle *h, size_t n, const double *pos,
                          double *energy, double *virial9, unsigned flags,
                          void *stream);

/* Full force evaluation in one call: one upload of pos/q/type, the
 * k-space and short-range pipelines, one download of the forces --
 * System::calculate_forces for the non-bonded + electrostatic part
 * (forces.cpp:121-249 with gpu.update / copy_forces_to_host at :129, :225).
 * energy3 = {coulomb real, coulomb k-space, non-bonded};
 * virial27 = {coulomb real, coulomb k-space, non-bonded} 3x3 each. */
int p3mx_forces(p3mx_handle *h, size_t n, const double *pos, const double *q,
                const int *type, double *f, double *energy3, double *virial27,
                unsigned flags, void *stream);

/* --- electrostatic layer correction (slab geometry) -------------------- */

/* Parameters of espressomd.electrostatics.ELC (src/python/espressomd/
 * electrostatics.py:288-365) as the elc_data constructor takes them
 * (src/core/electrostatics/elc.cpp:1056-1102); const_pot has an effect only
 * with a dielectric contrast, as in the reference. */
typedef struct {
  double maxPWerror;
  double gap_size;
  double far_cut;       /* -1: tuned from maxPWerror (tune_far_cut) */
  int neutralize;       /* bool; reference default 1 (off with contrasts) */
  double delta_mid_top; /* dielectric contrast above the slab, [-1, 1] */
  double delta_mid_bot; /* dielectric contrast below the slab, [-1, 1] */
  int const_pot;        /* bool */
  double pot_diff;
} p3mx_elc_params;

/* Attaches ELC to the actor, replacing the ElectrostaticLayerCorrection
 * constructor and activation (elc.hpp ElectrostaticLayerCorrection,
 * elc.cpp:1104-1109, on_activation): parameter checks, the base P3M set to
 * metallic (adapt_epsilon_elc, p3m.impl.hpp:112-114), slab height and
 * far cutoff (recalc_box_h elc.cpp:1020-1030, tune_far_cut :942-973).  NULL
 * detaches.  While attached, p3mx_forces and p3mx_long_range add the ELC
 * forces and energy (add_long_range_forces :1231-1254, long_range_energy
 * :1189-1229) and report a zero k-space virial (the reference computes no
 * ELC pressure, electrostatics/coulomb.cpp:124-131).  A charged particle in
 * the gap fails the call with "Particle <i> entered ELC gap region by <dz>"
 * (check_gap :184-194).  With dielectric contrasts only p3mx_forces
 * evaluates (the image terms span short and long range): the mesh carries
 * the image charges, the short-range loop the image-layer corrections
 * (elc.hpp), and p3mx_long_range fails with a message. */
int p3mx_set_elc(p3mx_handle *h, const p3mx_elc_params *p);
/* The far-formula cutoff in use, the slab height L_z - gap_size and the
 * number of Fourier modes summed (each may be NULL). */
int p3mx_get_elc(const p3mx_handle *h, double *far_cut, double *box_h, int *n_modes);

/* Cell-system introspection for parity tests: the cell grid and the cell
 * index of each particle as RegularDecomposition::position_to_cell_index
 * returns it (RegularDecomposition.cpp:51-80, 289-385), and the Verlet pair
 * set as non_bonded_loop_trace reports it (core/cells.cpp:178-188). */
int p3mx_cell_grid(p3mx_handle *h, int *cell_grid, double *cell_size);
int p3mx_cell_index(p3mx_handle *h, size_t n, const double *pos, int *cell);
/* Writes up to `cap` pairs (i<j) into pairs (2*cap ints); *count gets the
 * total pair count (may exceed cap). */
int p3mx_verlet_pairs(p3mx_handle *h, size_t n, const double *pos,
                      const double *q, const int *type, int *pairs,
                      size_t cap, size_t *count);

/* Charge-assignment mesh of the last long-range call (M0*M1*M2, FP64 copy
 * of the device mesh) for element-wise parity checks. */
int p3mx_copy_mesh(p3mx_handle *h, double *out, size_t cap);

/* Stage profile of one force evaluation with the current particles (no
 * counterpart in the reference, which has no GPU timers): per-stage mean
 * device time in ms over `reps` evaluations, stage names in
 * names[k] (static strings).  *nstages receives the stage count.  With ELC
 * attached (p3mx_set_elc) its three kernels follow: elc_sums, elc_reduce,
 * elc_forces. */
int p3mx_profile(p3mx_handle *h, int reps, double *ms, const char **names,
                 int cap, int *nstages);
/* Forces a rebuild of the cell lists and Verlet lists at the next force
 * evaluation, as CellSystem.resort() does in the reference
 * (CellStructure::set_resort_particles(Cells::RESORT_GLOBAL),
 * CellStructure.hpp:393-401 makes the next step rebuild). */
int p3mx_resort(p3mx_handle *h);
/* Total number of kernels launched by the handle's engines so far. */
int p3mx_launch_count(const p3mx_handle *h, long long *count);
/* Accuracy check of the FP32 exponentials of the FP32-mixed real-space
 * kernels (no counterpart in the reference): for n device values x, writes
 * to the device array out (3n floats) exp_fast(x), the single hardware
 * ex2 of x log2(e) the force-only kernel uses, and CUDA's expf(x). */
int p3mx_exp_check(size_t n, const float *x, float *out, void *stream);

/* Tuning error estimates (p3m.cpp:187-243; GPU k-space sum of
 * p3m_gpu_error_cuda.cu:87-143). */
int p3mx_error_estimate(const int *mesh, int cao, int n_c_part,
                        double sum_q2, double alpha_L, double r_cut_iL,
                        const double *box, double prefactor, double *rs_err,
                        double *ks_err);

/* Allocation-free k-space / real-space error estimate (no counterpart in
 * the reference).  For callers that must not allocate device memory while
 * they run -- engines that hand all GPU memory to their own pool at start-up,
 * or loops that cannot take the device synchronisation cudaMalloc/cudaFree
 * may imply.  Same results as p3mx_error_estimate, but the scratch is a
 * fixed 32 KiB device array inside the library (held on every GPU that loads
 * it until exit): meshes above 4096*16384 points are rejected with
 * P3MX_EDOMAIN and a message in errbuf.  Every call looks up the array's
 * address on the current device (no allocation), so a cudaDeviceReset leaves
 * no stale address behind; the first call on a device may load the
 * library's device code: make it before any stream capture.  All calls share the array, so calls
 * that overlap on the GPU race.  Each call returns only when its result is
 * on the host (it synchronises the stream).  stream: cudaStream_t or NULL;
 * errbuf/errbuf_len may be NULL/0. */
int p3mx_error_estimate_noalloc(const int *mesh, int cao, int n_c_part,
                                double sum_q2, double alpha_L, double r_cut_iL,
                                const double *box, double prefactor,
                                double *rs_err, double *ks_err, void *stream,
                                char *errbuf, size_t errbuf_len);

/* --- batched replicas -------------------------------------------------- */

/* Many independent cubic or orthorhombic systems advanced by one launch
 * per kernel (the reference has no batched path; each replica otherwise is
 * one ESPResSo System).  Per-replica arrays have n_rep entries; particles
 * of replica r occupy [offset[r], offset[r+1]) of the global arrays. */
typedef struct {
  int n_rep;
  const double *box;       /* 3*n_rep */
  const double *prefactor; /* n_rep (Bjerrum length * kT) */
  const long long *offset; /* n_rep+1 */
  double accuracy;         /* common target accuracy */
  double skin;
  int single_precision;
  int mesh_min, mesh_max;  /* autotuner mesh range (per dimension) */
  int cao_min, cao_max;
} p3mx_batch_desc;

typedef struct p3mx_batch p3mx_batch;

/* Creates the batch, uploads positions/charges/types, tunes every replica
 * (mesh, cao, r_cut, alpha by the error estimate plus timed trials). */
int p3mx_batch_create(const p3mx_batch_desc *d, const double *pos,
                      const double *q, const int *type, int ntypes,
                      const p3mx_pair_params *table, p3mx_batch **out);
void p3mx_batch_destroy(p3mx_batch *b);
const char *p3mx_batch_last_error(const p3mx_batch *b);
/* Tuned parameters of replica r. */
int p3mx_batch_get_tuned(const p3mx_batch *b, int r, p3mx_tuned *out);
/* Fix the charge-assignment order of every replica (n_rep values in the
 * batch's [cao_min, cao_max]), as P3M(cao=...) fixes it for one system
 * (p3m/common.hpp:59-172; no batched counterpart in the reference): each
 * replica takes the mesh, r_cut and alpha the autotuner found for that
 * order.  P3MX_EDOMAIN when an order cannot reach the accuracy for a
 * replica.  Positions, charges and velocities are kept. */
int p3mx_batch_set_cao(p3mx_batch *b, const int *cao);
/* One force evaluation for all replicas (forces overwritten, device
 * resident); optional per-replica energies (n_rep doubles, host). */
int p3mx_batch_forces(p3mx_batch *b, double *energy_out);
/* Stage profile of one force evaluation of the whole batch, as
 * p3mx_profile (no counterpart in the reference). */
int p3mx_batch_profile(p3mx_batch *b, int reps, double *ms, const char **names,
                       int cap, int *nstages);
/* Pair bonds of the batch, as p3mx_set_bonds with particle indices over the
 * whole batch (both partners in one replica); forces enter
 * p3mx_batch_forces and the graph step of p3mx_batch_run (captured anew
 * after this call), bonded energies the per-replica energy_out. */
int p3mx_batch_set_bonds(p3mx_batch *b, int n_types,
                         const p3mx_bond_params *types, size_t n_bonds,
                         const int *bonds);
/* Velocity-Verlet + Langevin (kT, gamma, dt) for `steps` steps, captured
 * in a CUDA graph after the first step.  Positions stay FP64 on device. */
int p3mx_batch_run(p3mx_batch *b, int steps, double dt, double kT,
                   double gamma, unsigned long long seed);
/* The CUDA stream (cudaStream_t) the batch launches its work and graphs on,
 * for callers that time or order work around p3mx_batch_run. */
void *p3mx_batch_stream(const p3mx_batch *b);
/* Kernels launched by the batch so far (graph launches count their nodes). */
int p3mx_batch_launch_count(const p3mx_batch *b, long long *count);
/* Copy positions / forces (3*N doubles, host) of all replicas. */
int p3mx_batch_get(p3mx_batch *b, double *pos, double *f, double *vel);

/* --- dipolar P3M --------------------------------------------------------- */

/* Actor parameters: the kwargs of espressomd.magnetostatics.DipolarP3M
 * (src/python/espressomd/magnetostatics.py:82-160) and the P3MParameters of
 * DipolarP3M (script_interface/magnetostatics/DipolarP3M.hpp:95-112).
 * -1 marks a value left to the tuner; the mesh must be cubic. */
typedef struct {
  double prefactor;
  double accuracy;
  int mesh[3];
  int cao;
  double r_cut;
  double alpha;
  double epsilon;       /* 0 = metallic */
  double mesh_off[3];   /* -1 = P3M_MESHOFF (0.5) */
  int tune;             /* bool */
  int timings;          /* force evaluations timed per tuning trial */
  int verbose;          /* print the tuning log */
  int single_precision; /* 1 = FP32 mesh/FFT path, 0 = FP64 */
} p3mx_dp3m_params;

typedef struct p3mx_dp3m p3mx_dp3m;

/* Validates and stores the parameters, as DipolarP3M::do_construct +
 * new_dp3m_handle (script_interface/magnetostatics/DipolarP3M.hpp:95-130,
 * core/magnetostatics/dp3m.impl.hpp:80-92).  On a validation failure *out
 * still receives a handle that carries the message. */
int p3mx_dp3m_create(const p3mx_dp3m_params *params, p3mx_dp3m **out);
void p3mx_dp3m_destroy(p3mx_dp3m *h);
const char *p3mx_dp3m_last_error(const p3mx_dp3m *h);
/* Box and skin (on_boxl_change -> scaleby_box_l once activated). */
int p3mx_dp3m_set_system(p3mx_dp3m *h, const p3mx_system *sys);
/* on_activation: sanity checks and tune() (dp3m.cpp:647-680, 880-893).
 * dip: 3*n moments (AoS, Particle::calc_dip()). */
int p3mx_dp3m_activate(p3mx_dp3m *h, size_t n, const double *pos,
                       const double *dip, unsigned flags);
int p3mx_dp3m_get_tuned(const p3mx_dp3m *h, p3mx_tuned *out);
/* k-space (DipolarP3MImpl::long_range_kernel, dp3m.cpp:247-445) plus the
 * real-space pair part (dp3m.hpp:142-232) for all n particles.  With
 * P3MX_FORCES, forces and torques (3*n each) are added to f / torque (or
 * overwrite them with P3MX_OVERWRITE); with P3MX_ENERGY, energy[0] gets
 * the k-space energy with its self and Madelung corrections (and the
 * surface term for epsilon != 0) and energy[1] the real-space energy. */
int p3mx_dp3m_compute(p3mx_dp3m *h, size_t n, const double *pos,
                      const double *dip, double *f, double *torque,
                      double *energy, unsigned flags, void *stream);
/* Stage profile (no counterpart in the reference): the host arrays pos and
 * dip (3*n each) are staged, one evaluation of forces and torques runs
 * unprofiled, then reps profiled ones; ms[k] is the mean device time of
 * stage names[k] (static strings), *nstages the stage count. */
int p3mx_dp3m_profile(p3mx_dp3m *h, size_t n, const double *pos,
                      const double *dip, int reps, double *ms, const char **names,
                      int cap, int *nstages);
/* Kernels launched by the handle so far. */
int p3mx_dp3m_launch_count(const p3mx_dp3m *h, long long *count);

#ifdef __cplusplus
}
#endif
#endif
