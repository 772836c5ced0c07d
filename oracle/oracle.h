/*
 * TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * FP64 CPU restatement of ESPResSo's CPU P3M + short-range force path
 * (src/core/electrostatics/p3m.cpp, src/core/p3m/*, p3m.hpp:146-180,
 * nonbonded_interactions/{lj,wca}.hpp, cell_system/RegularDecomposition.cpp)
 * plus an independent FP64 direct Ewald sum.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load this library.
 */
#ifndef P3MX_ORACLE_H
#define P3MX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Parameters of one periodic system (mirrors P3MParameters, p3m/common.hpp:59-172). */
typedef struct {
  double box[3];
  int mesh[3];
  int cao;
  double alpha;
  double r_cut;
  double prefactor;
  double epsilon;     /* 0 = metallic */
  double mesh_off[3]; /* reference default 0.5 */
  double skin;        /* Verlet skin; only shapes the local CA mesh margin */
} oracle_p3m_params;

/* Lennard-Jones / WCA parameters for one type pair (lj.hpp:41-60, wca.hpp:39-55). */
typedef struct {
  double lj_eps, lj_sig, lj_cut, lj_shift, lj_offset, lj_min;
  double wca_eps, wca_sig; /* wca cut = sig * 2^(1/6) (wca.cpp:31-42) */
} oracle_pair_params;

/* k-space part: forces are ADDED to f (3n, AoS), energy/virial overwritten.
 * rho_out (optional, M0*M1*M2 row-major z fastest) receives the assigned mesh. */
int oracle_p3m_kspace(const oracle_p3m_params *p, long n, const double *pos,
                      const double *q, double *f, double *energy,
                      double *virial9, double *rho_out);

/* Influence function on the full mesh (M0*M1*M2, row-major). */
int oracle_influence_function(const oracle_p3m_params *p, double *g_out);

/* Short-range part: real-space Coulomb (if prefactor != 0 and r_cut > 0) plus
 * LJ/WCA for the type-pair table tab[ntypes*ntypes].  Forces are ADDED.
 * energy_out[2] = {coulomb real-space, non-bonded}; virial_out[18] = two
 * 3x3 tensors in the same order.  Pairs are found with a restatement of the
 * regular-decomposition link-cell loop. */
int oracle_short_range(const oracle_p3m_params *p, long n, const double *pos,
                       const double *q, const int *type, int ntypes,
                       const oracle_pair_params *tab, double *f,
                       double *energy_out, double *virial_out);

/* Cell system restatement (RegularDecomposition.cpp:289-385, 51-80).
 * Writes cell_grid[3] and cell_size[3] for interaction range `range`. */
int oracle_cell_grid(const double *box, double range, int *cell_grid,
                     double *cell_size);
/* Cell index of each (already folded) position, column-major over the ghost
 * grid (cell_grid + 2), as position_to_cell_index returns it. */
int oracle_cell_index(const double *box, double range, long n,
                      const double *pos, int *cell_out);
/* Verlet pair set: pairs (i<j) whose minimum-image distance satisfies the
 * VerletCriterion (VerletCriterion.hpp:68-97).  Returns the pair count, or
 * -1 if cap is too small (pairs_out must then be re-sized). */
long oracle_verlet_pairs(const double *box, double skin, double coulomb_cut,
                         long n, const double *pos, const double *q,
                         const int *type, int ntypes, const double *ia_cut,
                         long cap, long *pairs_out);

/* Tuning error estimates (p3m.cpp:146-243, 187-193). */
double oracle_rs_error(double pref, double r_cut_iL, int n_c_part,
                       double sum_q2, double alpha_L, const double *box);
double oracle_ks_error(double pref, const int *mesh, int cao, int n_c_part,
                       double sum_q2, double alpha_L, const double *box);

/* Direct FP64 Ewald sum (independent of the reference), metallic or with
 * the dipole term for epsilon > 0.  Forces ADDED to f (3n); returns energy
 * in *energy.  r_cut < box/2; kmax in units of 2*pi/L per axis. */
int oracle_ewald(const double *box, long n, const double *pos, const double *q,
                 double prefactor, double alpha, double r_cut, int kmax,
                 double epsilon, double *f, double *energy);

/* Direct FP64 Ewald forces (metallic) on the nt particles tidx[] from all n
 * sources: cell-list real space, structure-factor reciprocal space.  Forces
 * written to f (3 nt).  Returns 0, or nonzero for r_cut > L/2 or a bad index. */
int oracle_ewald_targets(const double *box, long n, const double *pos, const double *q,
                         long nt, const long *tidx, double prefactor, double alpha,
                         double r_cut, int kmax, double *f);

/* Math restatements, exported for comparison with the reference headers. */
double oracle_bspline(int order, int i, double x);
double oracle_as_erfc_part(double d);
double oracle_sinc(double x);
double oracle_cotangent_sum(int cao, int n, double mesh_i);

#ifdef __cplusplus
}
#endif
#endif
