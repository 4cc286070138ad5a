/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in plain C, of simcore's Brownian-dynamics step for
 * semiflexible filaments (cell list, segment-segment WCA pair forces with
 * the reference's stale-force and stale-list behaviour, bond-to-site force
 * conversion, bending and metric forces, the two Thomas solves, the
 * midpoint position update and bond renormalisation).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker.  It is pinned bit for bit against the reference's own
 * code (oracle/_ref, built by oracle/ref/Makefile) through the fixtures in
 * tests/golden/.
 *
 * Every array is site-, bond- or pair-major with 3 doubles per vector (z = 0
 * in 2D), filaments stored back to back in the order they were given. */
#ifndef SC_ORACLE_H
#define SC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n_dim;              /* 2 or 3, every dimension periodic */
  double system_radius;   /* R: cube (square) of side 2R */
  double delta;
  double wca_eps;
  double wca_sig;
  double f_cutoff;
  int stoch_flag;
  int interaction_flag;
  int like_like_interactions;
  unsigned int seed;      /* Philox key word 0 */
  int n_threads;          /* unused: the oracle is single threaded */
} sco_system;

typedef struct {
  double length;
  double persistence_length;
  double diameter;
  double min_bond_length;
  double friction_ratio;
} sco_filament;

typedef struct sco_sim sco_sim;

/* Number of bonds the reference gives a filament (src/filament.cpp:142-147). */
int sco_filament_n_bonds(const sco_filament *f);

sco_sim *sco_create(const sco_system *sys, int n_fil, const sco_filament *fils,
                    const double *site_xyz, int n_sites);
void sco_destroy(sco_sim *s);
int sco_n_sites(const sco_sim *s);
int sco_n_bonds(const sco_sim *s);
int sco_n_cells_1d(const sco_sim *s);
double sco_cell_length(const sco_sim *s);
double sco_dr_update(const sco_sim *s);
long sco_n_rebuilds(const sco_sim *s);
int sco_i_step(const sco_sim *s);

/* Runs n steps (i_steps).  Returns 0, or -1 when the reference would throw
 * "Unphysical result" (accumulated displacement above 10000). */
int sco_step(sco_sim *s, int n);

void sco_get_sites(const sco_sim *s, double *xyz);
void sco_get_prev_sites(const sco_sim *s, double *xyz);
void sco_get_site_forces(const sco_sim *s, double *f);
void sco_get_random_forces(const sco_sim *s, double *f);
void sco_get_bond_ft(const sco_sim *s, double *f, double *t);
void sco_get_tensions(const sco_sim *s, double *t);
void sco_get_bond_geom(const sco_sim *s, double *pos, double *spos, double *u,
                       double *len);
void sco_get_filament_state(const sco_sim *s, int *normalize_switch,
                            int *n_normalize);
void sco_get_frictions(const sco_sim *s, double *gpar, double *gperp,
                       double *spar, double *sperp);
long sco_get_pairs(const sco_sim *s, int *out, long cap);
void sco_get_bond_cells(const sco_sim *s, int *xyz);
void sco_get_dr_tot(const sco_sim *s, double *dr);

/* Overwrite all site positions (and previous positions) with xyz, rebuild
 * bond geometry, as when a configuration is loaded. */
void sco_set_sites(sco_sim *s, const double *xyz);

/* Static doubly-bound crosslinks (harmonic tethers) between site_a[k] and
 * site_b[k] (global site indices): an anchor on site j < last sits at the
 * tail of bond j, an anchor on a filament's last site at the head of its last
 * bond.  Once per simulation, before the first step.  Returns 0 or -1. */
int sco_add_crosslinks(sco_sim *s, int n, const int *site_a, const int *site_b,
                       double k_spring, double k_spring_compress, double rest_length);
/* Tether force of each link from its last recomputation (anchor 0 gets +F). */
void sco_get_crosslink_forces(const sco_sim *s, double *f);

/* Pair forces alone, evaluated from the current bond geometry on the
 * current pair list with the pair forces stored so far, without changing
 * any state: bond forces/torques are written to f and t. */
void sco_pair_forces(sco_sim *s, double *f, double *t);

/* Thermo: the pair virial accumulated every step and, every n_thermo steps
 * (i_step % n_thermo == 0), the pressure tensor and pressure of
 * InteractionManager::CalculatePressure; 0 stops the records.  Per-filament
 * potential energy of the last step. */
void sco_set_thermo(sco_sim *s, int n_thermo);
long sco_thermo_records(sco_sim *s, long max, long *i_step, double *tensor, double *pressure,
                        double *volume);
void sco_get_stress(const sco_sim *s, double *stress);
void sco_get_potential_energy(const sco_sim *s, double *pote);

/* Seeded random insertion with overlap rejection (sc_oracle_insert.c):
 * n_fil filaments of n_bonds[i] bonds, lengths and persistence lengths given,
 * in a periodic box of radius system_radius; insertion_type 0 random, 1
 * random_nematic, 2 random_polar.  Writes sum(n_bonds[i] + 1) x 3 doubles.
 * Returns 0, 1 (invalid arguments) or 8 (a filament found no place within
 * max_attempts). */
int sco_insert_filaments(int n_dim, double system_radius, uint64_t seed, int n_fil,
                         const int *n_bonds, const double *length,
                         const double *persistence_length, double diameter,
                         int insertion_type, int max_attempts, double *site_xyz);

/* Philox4x32-10 block (for the known-answer test of the shared stream). */
void sco_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Pair force of two bonds given by end points (a1, a2) and (b1, b2) in an
 * otherwise empty box: force on bond a, following Sphero + WCA.  Returns 1
 * when the pair is within the cutoff. */
int sco_segment_force(const sco_system *sys, const double *a1, const double *a2,
                      const double *b1, const double *b2, double *force);

#ifdef __cplusplus
}
#endif
#endif
