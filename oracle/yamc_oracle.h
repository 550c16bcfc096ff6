/*
 * yamc_oracle.h -- CPU oracle for the YAMC per-trial-move energy path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference Fortran (voovrat/YAMC) that the parity tests, smoke() and the
 * cpu_baseline leg of bench.py use as the checker.  The product library
 * (yamc_b200/) never links, imports or calls anything in this directory.
 *
 * Every function cites the reference file:line it restates; the operation
 * order of the reference is kept (sequential sums, 8 sign-combination
 * arrays per structure factor, the incremental uu/F bookkeeping), so the
 * oracle reproduces the reference's arithmetic up to the compiler's
 * floating-point contraction (built with -ffp-contract=off).
 *
 * Pinning: Parameters_recalc is pinned against the reference's own
 * parameters.out (tests/golden); the random stream is the reference's own
 * gfortran random_number, produced by calling libgfortran.  The movemc
 * arithmetic itself has no reference-produced golden vector (the reference
 * ships none and no Fortran compiler is available), so its parity against
 * the reference binary is unpinned; it is checked by the reference's own
 * debug invariants (incremental vs full recompute, MC.f90:1886-1951) and by
 * physics known answers (Madelung constant, direct LJ lattice sums).
 */
#ifndef YAMC_ORACLE_H
#define YAMC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* parameters.f90:11-86 (primary and derived module variables) */
typedef struct {
    /* primary: read from parameters.prm (parameters.f90:102-148) */
    double sr, sk, alphaL, temp, external_permutivity, BoxLength, density;
    double dr_a, d_angle_degree, xlambda_c, xlambda_f, pressure;
    double pressure_step_multiplier, max_volume_scaling;
    double n_store_traj_interval, n_store_energy_interval;
    int32_t max_cycle, rnd_seed;
    int32_t input_nbytes_xyz, input_nbytes_ang, output_nbytes_xyz, output_nbytes_ang;
    /* derived: Parameters_recalc (parameters.f90:355-413) */
    double alpha; /* = alphaL after the 2*sr default */
    double rmax, rmax2, kT_kcal_mol, dbjr_a, dbjr, xclb;
    double alpha_over_sqrt_pi, two_alpha_over_sqrt_pi, kext, minus_two_kext;
    double dr, d_angle, log_max_volume_scaling, pressure_angstr_kT;
    int32_t kmax;
    int32_t are_read;
    char freq_file[256];
} orc_params;

typedef struct orc_state orc_state;

/* per-move record written by orc_run_mc */
typedef struct {
    int32_t imol;       /* 1-based molecule index chosen */
    int32_t flags;      /* bit0 accepted, bit1 overlap */
    int64_t cursor;     /* RNG cursor after the move */
    double du_real, du_k_coul, du_k_lj, du_ext; /* movemc Steps 7, 10, 11, 11A */
    double f_old[3], t_old[3], f_new[3], t_new[3];
} orc_move_rec;

/* one mcvol step (MC.f90:701-825) written by orc_run_cycles / orc_mcvol */
typedef struct {
    int64_t cycle;      /* run_mc cycle number */
    int32_t flags;      /* bit0 accepted, bit1 hard-core overlap at the new volume */
    int32_t pad;
    int64_t cursor;     /* RNG cursor after the step */
    double box_old, box_new;  /* BoxLength before and tried (Angstrom) */
    double du, arg;     /* U_new - U_old (kT) and the acceptance exponent */
} orc_vol_rec;

/* ---- parameters ---- */
void orc_params_defaults(orc_params *p);
int orc_params_read(orc_params *p, const char *path);
int orc_params_read_string(orc_params *p, const char *str);
int orc_params_init(orc_params *p, int32_t nmol);   /* BoxLength from density + recalc */
int orc_params_recalc(orc_params *p, double box_length);

/* ---- special functions (Functions.f90) ---- */
double orc_erfc_luc(double x);
double orc_erf_luc(double x);
void orc_erfc_bet6_bet12(double x, double x2, double e2, double *erfk, double *bet6, double *bet12);
double orc_shi_sans_exp(double x);
int32_t orc_grid_count(int32_t kmax);

/* ---- system ---- */
int32_t orc_set_move_weights(orc_state *s, const double *w, int32_t n);
orc_state *orc_create(const orc_params *p, const char *composition_path, const char *moltab_path,
                      int32_t *status);
void orc_destroy(orc_state *s);
int32_t orc_natom(const orc_state *s);
int32_t orc_nmol(const orc_state *s);
int32_t orc_nk(const orc_state *s);
int32_t orc_ntype(const orc_state *s);
void orc_get_params(const orc_state *s, orc_params *p);
void orc_get_atoms(const orc_state *s, double *x, double *y, double *z, double *q,
                   int32_t *type_by_index, int32_t *molnum);
void orc_get_mols(const orc_state *s, int32_t *first_atom, int32_t *last_atom);
/* energy.dat columns 2..9 (runmc.f90:349-351): U_total, U_total_ew, U_total_lj,
   uu_ew, uu_lj6, uu_lj12, E_k_coulomb, E_k_lj  */
void orc_energies(orc_state *s, double e[8]);
/* mc_calc_total_sums (MC.f90:477-585): recompute everything from the positions */
int32_t orc_full_sums(orc_state *s, double e[8]);
/* snapshot of the incremental per-atom state (uu, F) and rho(k) for invariant tests */
void orc_get_uuF(const orc_state *s, double *uu, double *fx, double *fy, double *fz);
void orc_intra_sums(const orc_state *s, double out[3]);
void orc_get_rho(const orc_state *s, double *out); /* (1+ntype) x 8 x nk */
double orc_mu(const orc_state *s, int32_t c);

/* run_mc NVT loop (runmc.f90:178-334) consuming a float32 buffer of gfortran
   random_number values from *cursor.  n_moves counts movemc calls.  Returns 0,
   or -6 when the buffer ran out (the partially done move is not committed).
   energy rows (9 doubles: frame + energy.dat columns) are appended to rows. */
int32_t orc_run_mc(orc_state *s, const float *rng, int64_t n_rng, int64_t *cursor,
                   int64_t n_moves, orc_move_rec *log, double *rows, int32_t max_rows,
                   int32_t *n_rows);
/* run_mc by cycles with NPT volume steps (pressure_step_multiplier > 0); move records
   go to log (when max_log leaves room for the whole cycle), volume steps to vlog.
   Returns 0 or -6 (buffer exhausted; an interrupted volume step is undone and its
   cycle draw given back, an interrupted move cycle resumes mid-cycle). */
int32_t orc_run_cycles(orc_state *s, const float *rng, int64_t n_rng, int64_t *cursor, int64_t n_cycles,
                       int64_t *cycles_done, orc_move_rec *log, int64_t max_log, int64_t *n_log,
                       orc_vol_rec *vlog, int64_t max_vlog, int64_t *n_vlog, double *rows, int32_t max_rows,
                       int32_t *n_rows);
/* a single mcvol with its draws from the RNG buffer */
int32_t orc_mcvol(orc_state *s, const float *rng, int64_t n_rng, int64_t *cursor, orc_vol_rec *rec);
/* current BoxLength (Angstrom) and the molecule-atom distances in Angstrom follow from it */
double orc_box_length(const orc_state *s);
/* init_freq with exchange weights: xchange_freq and xchange_probability = Sxch/(Smv+Sxch);
   run_mc then takes an exchange step when the move's first draw is below it */
int32_t orc_set_xchange_weights(orc_state *s, const double *w, int32_t n);
/* one mc_xchange (MC.f90:1325-1954) of molecules imol1 != imol2 (1-based); the record has
   imol = imol1, flags bit0 accepted, bit1 overlap, bit2 exchange, bits 8.. imol2 */
int32_t orc_xchange(orc_state *s, int32_t imol1, int32_t imol2, const float *rng, int64_t n_rng,
                    int64_t *cursor, orc_move_rec *rec);
/* a single movemc(imol) with the proposal drawn from the RNG buffer */
int32_t orc_movemc(orc_state *s, int32_t imol, const float *rng, int64_t n_rng,
                   int64_t *cursor, orc_move_rec *rec);

/* host-driven movemc stages: Steps 0-4, Steps 6-12 for given new positions, Step 14 */
int32_t orc_move_old(orc_state *s, int32_t imol, double f[3], double t[3]);
int32_t orc_move_eval(orc_state *s, const double *xn, const double *yn, const double *zn, double du[4],
                      int32_t *overlap, double f[3], double t[3]);
int32_t orc_move_commit(orc_state *s);

/* radial distribution functions of molecule centres (mcrdf2.f90:110-440): counts of one frame
   added to cnt4[(t1*ntypes+t2)*nbin + b] and n_total[t1*ntypes+t2] (t1 <= t2, 0-based species,
   nbin = aint((Rmax-1e-10)/dr) + 2), and the written g(r) from the accumulated counts */
void orc_rdf_count(int32_t M, const double *x, const double *y, const double *z, const int32_t *type, int32_t ntypes,
                   double L, double dr, double rmax, double *cnt4, double *n_total);
void orc_rdf_normalize(int32_t ntypes, const int32_t *mol_numbers, double dr, double rmax, const double *cnt4,
                       const double *n_total, int32_t n_frame, double avg_inv_vol, double *g);

/* k-space forces on one atom at (x,y,z) with the current total rho (ForceKSpace.f90) */
void orc_force_kspace_atom(orc_state *s, int32_t atom1, double x, double y, double z,
                           double f[3]);

#ifdef __cplusplus
}
#endif
#endif
