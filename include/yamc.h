/*
 * yamc.h -- C ABI of the B200 engine for YAMC's per-trial-move energy path.
 *
 * The engine replaces the body of the reference's MC module (MC.f90): initmc,
 * movemc and mc_total_energy, and the run_mc loop that calls movemc
 * (runmc.f90:178-334).  A Fortran host binds these entry points through
 * ISO_C_BINDING (an interface module of BIND(C) declarations, one per entry
 * point, with the structs below as BIND(C) derived types); the Python package
 * yamc_b200 binds them through ctypes.
 *
 * Conventions (as in the reference): coordinates in box units (-0.5..0.5),
 * energies in kT, molecule numbers 1-based, atoms stored molecule by molecule.
 * Every function returns an int status: 0 = OK, negative = error (below).
 * A hard-core overlap is not an error; it is reported through *overlap or the
 * per-move flags, exactly like EwaldSumRealSpace_calc's logical overlap.
 * No function aborts the process or throws across the ABI.
 */
#ifndef YAMC_H
#define YAMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; -1..-5 mirror ERROR_IO, ERROR_LIMITS, ERROR_PARAMETER,
   ERROR_INITIALIZATION, ERROR_WRONG_FUNCTION of error.f90:47-51 */
#define YAMC_OK 0
#define YAMC_EIO (-1)
#define YAMC_ELIMITS (-2)
#define YAMC_EPARAMETER (-3)
#define YAMC_EINIT (-4)
#define YAMC_EWRONG_FUNCTION (-5)
#define YAMC_ECUDA (-10)
#define YAMC_ETIMEOUT (-11)
#define YAMC_ERNG_EXHAUSTED (-12)
/* YAMC_ENAN: a non-finite value where the arithmetic cannot go on.  Refused inputs (a
   non-finite coordinate, charge or LJ parameter at yamc_create or yamc_set_positions) leave the
   context unchanged.  A chain (yamc_run_chain, yamc_run_mc, a batch replica) whose move gives a
   non-finite energy change or bias force stops before deciding that move, with the state, the
   records and *cursor as they were after the last completed move.  yamc_move_old/_eval return
   it for a non-finite energy or force (the move cannot be committed), yamc_forces when a force
   is non-finite (the outputs hold the values), and a full sum (yamc_full_sums, a volume step)
   when an energy is non-finite (the context then holds those sums: load finite positions). */
#define YAMC_ENAN (-13)
#define YAMC_EOVERLAP_INIT (-14)
/* YAMC_EBOUNDS: bounds-checked builds only (libyamc_b200_checked.so, compiled with
   -DYAMC_CHECKED): an index the chain kernel computed fell outside its array.  The kernel
   replaced it by 0 (no fault) and the call returns this code; yamc_last_error_detail names the
   source line.  The state of the context is then unreliable. */
#define YAMC_EBOUNDS (-15)

/* precision of the device arithmetic */
#define YAMC_FP64 0   /* plain method: every operation in FP64 */
#define YAMC_MIXED 1  /* FP32 pair/erfc/phase arithmetic, FP64 rho(k), sums and Metropolis */

/* Simulation parameters: the module variables of parameters.f90:11-86.
   The primary block is what parameters.prm sets; yamc_params_recalc fills
   the derived block exactly as Parameters_recalc (parameters.f90:355-413). */
typedef struct {
    /* primary */
    double sr, sk, alphaL, temp, external_permutivity, BoxLength, density;
    double dr_a, d_angle_degree, xlambda_c, xlambda_f, pressure;
    double pressure_step_multiplier, max_volume_scaling;
    double n_store_traj_interval, n_store_energy_interval;
    int32_t max_cycle, random_seed;
    int32_t input_nbytes_xyz, input_nbytes_ang, output_nbytes_xyz, output_nbytes_ang;
    /* derived (Parameters_recalc) */
    double alpha; /* alpha*L in box units (alphaL, defaulted to 2*sr) */
    double rmax, rmax2, kT_kcal_mol, dbjr_a, dbjr, xclb;
    double alpha_over_sqrt_pi, two_alpha_over_sqrt_pi, kext, minus_two_kext;
    double dr, d_angle, log_max_volume_scaling, pressure_angstr_kT;
    int32_t kmax;
    int32_t precision; /* YAMC_FP64 or YAMC_MIXED (not a reference parameter) */
} yamc_params;

/* The system as the reference host holds it after MoleculeTable_fillAtomicData
   (MoleculeTable.f90:584-705): per-atom arrays of length natom in molecule order. */
typedef struct {
    int32_t natom, nmol;
    const double *x, *y, *z;        /* box units */
    const double *charge;           /* e */
    const double *sigma;            /* sigma / BoxLength */
    const double *epsilon;          /* epsilon / kT */
    const double *hard_core_angstr; /* hard-core diameter, Angstrom */
    const double *mass;             /* atomic masses (centre of mass of a molecule) */
    const int32_t *first_atom;      /* per molecule, 1-based, inclusive */
    const int32_t *last_atom;       /* per molecule, 1-based, inclusive */
    /* composition: molecule counts per species in composition order; the LJ
       tails read them by LJ type (EwaldSumTails.f90:88) */
    int32_t n_species;
    const int32_t *mol_numbers;
    /* molecule-choice weights of run_mc (init_freq, runmc.f90:25-67);
       NULL = flat weights (no frequencies file) */
    const double *move_weights;
} yamc_system;

typedef struct yamc_ctx yamc_ctx;

/* One movemc record (optional output of yamc_run_chain). */
typedef struct {
    int32_t imol;    /* 1-based molecule tried */
    int32_t flags;   /* bit0 accepted, bit1 hard-core overlap (rejected, no acceptance draw) */
    int64_t cursor;  /* RNG cursor after the move */
    double du_real, du_k_coul, du_k_lj, du_ext; /* movemc Steps 7, 10, 11, 11A */
} yamc_move_record;

/* One NPT volume step (mcvol, MC.f90:701-825), an optional output of yamc_run_mc. */
typedef struct {
    int64_t cycle;   /* run_mc cycle number of the step */
    int32_t flags;   /* bit0 accepted, bit1 hard-core overlap at the new volume (rejected) */
    int32_t pad;
    int64_t cursor;  /* RNG cursor after the step */
    double box_old, box_new; /* BoxLength before the step and the one tried (Angstrom) */
    double du, arg;  /* U_new - U_old (kT; 0 on overlap) and the acceptance exponent
                        -dU - P dV + (nmol+1) ln(V_new/V_old) */
} yamc_volume_record;

/* ---- parameters (parameters.f90) ---- */
/* Parameters_read (parameters.f90:266-305) on top of the defaults (:18-72). */
int yamc_params_read(const char *path, const char *extra, yamc_params *p);
/* Parameters_init (:323-352): BoxLength from density when zero, then recalc. */
int yamc_params_init(yamc_params *p, int32_t nmol);
/* Parameters_recalc (:355-413). */
int yamc_params_recalc(yamc_params *p, double box_length);

/* ---- host-side inputs: the reference readers, for hosts without their own ----
   Composition_read_from_file + Molecule_read_from_file/centrate (composition.f90:84-142,
   Molecule.f90:142-209), MoleculeTable_load_binary (MoleculeTable.f90:240-319) and
   MoleculeTable_fillAtomicData (:584-705).  The returned yamc_system's arrays are
   owned by the handle and freed by yamc_inputs_free. */
typedef struct yamc_inputs yamc_inputs;
int yamc_inputs_load(const char *parameters_path, const char *composition_path,
                     const char *moltab_path, const char *extra, yamc_inputs **out);
int yamc_inputs_get(const yamc_inputs *in, yamc_system *sys, yamc_params *p);
int yamc_inputs_free(yamc_inputs *in);

/* ---- engine lifecycle: initmc (MC.f90:587-602) ---- */
/* Copies the system to the device, builds LJ types (LJTypes_fill), the k-grid
   (FourierGrid_init), beta/beta6/beta12/beta_LJ (EwaldSumKSpace_initBeta[LJ]),
   the tails (EwaldSumTails) and runs the full sums (mc_calc_total_sums). */
int yamc_create(const yamc_system *sys, const yamc_params *p, int32_t device, yamc_ctx **out);
int yamc_destroy(yamc_ctx *ctx);

/* energy.dat columns 2..9 (runmc.f90:349-351): U_total, U_total_ew, U_total_lj,
   uu_ew, uu_lj6, uu_lj12, E_k_coulomb, E_k_lj -- the incremental values
   (mc_total_energy, MC.f90:681-698). */
int yamc_energies(yamc_ctx *ctx, double e[8]);
/* mc_calc_total_sums (MC.f90:477-585): recompute rho(k), the real-space sums and
   mu from the current positions and return the same 8 numbers. */
int yamc_full_sums(yamc_ctx *ctx, double e[8]);
int yamc_get_positions(yamc_ctx *ctx, double *x, double *y, double *z);
/* sizes: natom, nmol, nk (half-space k), nsigned (signed k entries), ntype */
int yamc_sizes(yamc_ctx *ctx, int32_t out[5]);

/* Replace the configuration (atom positions in box units, the molecule layout
   unchanged) and recompute the sums as mc_calc_total_sums does (MC.f90:477-585);
   e (optional) receives the 8 energy.dat numbers.  The counterpart of loading a
   new frame into atomic_data before a full recompute. */
int yamc_set_positions(yamc_ctx *ctx, const double *x, const double *y, const double *z, double e[8]);

/* ---- exact checkpoint ----
   The reference restarts a run from the last trajectory frame and a new seed (mccont.f90:121-171),
   which continues the ensemble but not the chain.  These calls save and restore a context's whole
   state bit for bit -- positions, rho(k), the engine scalars (energies, dipole, tails, step
   counts), the run_mc counters, the parameters and box-dependent tables as they stand after NPT
   steps -- together with the caller's random-stream cursor, so a chain continued from a loaded
   state in a fresh context is identical, move for move and bit for bit, to the uninterrupted one.
   yamc_state_size gives the blob's size for this context; yamc_save_state writes it (host
   buffer, host byte order); yamc_load_state reads it into a context created from the same system
   (same atom, molecule, LJ type and k counts, else YAMC_EPARAMETER), keeping that context's
   precision, and returns the saved cursor.  Neither may come between an eval and its commit
   (YAMC_EWRONG_FUNCTION); a batch replica can be saved but not loaded into. */
int yamc_state_size(yamc_ctx *ctx, int64_t *bytes);
int yamc_save_state(yamc_ctx *ctx, int64_t cursor, void *buf, int64_t bytes);
int yamc_load_state(yamc_ctx *ctx, const void *buf, int64_t bytes, int64_t *cursor);

/* ---- adjoint forces ----
   Forces = -gradient of the total energy as implemented, for every atom (kT per
   box length): real space differentiating the piecewise erfc_Luc that the energy
   uses (the reference's own real-space forces use the exact erfc derivative,
   RealSumLocal.f90:104, so they differ at the level of erfc_Luc's error), k-space
   Coulomb + dispersion as ForceKSpace_coulomb/_LJ (ForceKSpace.f90:59-302) with
   sin/cos(k r) recomputed per atom, and the external term -2 kext q mu
   (EwaldSumExternal.f90:84-102).  fx/fy/fz: natom each; mol_f, mol_tau: nmol x 3,
   the molecular force and the torque about the centre of mass (MC.f90:988-1025,
   geometry.f90:65-201).  Any output may be NULL. */
int yamc_forces(yamc_ctx *ctx, double *fx, double *fy, double *fz, double *mol_f, double *mol_tau);

/* ---- per-move drop-in for the body of movemc (MC.f90:831-1322) ---- */
/* Steps 0-4: old molecular force and torque of molecule imol (1-based). */
int yamc_move_old(yamc_ctx *ctx, int32_t imol, double f[3], double tau[3]);
/* Steps 6-12 for the proposed atom positions (box units, natom of the molecule):
   du = {dU_real, dU_k_coulomb, dU_k_LJ, dU_ext}; *overlap as Step 6; new
   molecular force and torque.  Must follow yamc_move_old for the same imol. */
int yamc_move_eval(yamc_ctx *ctx, int32_t imol, const double *xn, const double *yn,
                   const double *zn, double du[4], int32_t *overlap, double f[3], double tau[3]);
/* Step 14: commit (accepted != 0) or drop the evaluated move. */
int yamc_move_commit(yamc_ctx *ctx, int32_t accepted);

/* ---- device-resident run_mc (runmc.f90:178-334, NVT single-molecule moves) ----
   Runs n_moves movemc calls with the proposal, Metropolis test and commit on
   the device, consuming the raw gfortran random_number stream rng[0..n_rng)
   from *cursor (rand() redraw rule of random.f90:65-93 applied on the device).
   Cycle structure, the per-cycle pressure draw and the energy.dat rows
   (frame + 8 columns, at cycles where mod(n_mv_steps/nmol + n_vol_steps,
   n_store_energy_interval) < 1e-10) follow run_mc.  rng is a HOST pointer; it
   is copied to the device inside the call.  log (n_moves records) and rows
   (9 doubles each, max_rows) are optional host outputs.  Returns
   YAMC_ERNG_EXHAUSTED with *moves_done < n_moves when the buffer runs out; the
   interrupted move is not committed and resumes exactly from *cursor. */
int yamc_run_chain(yamc_ctx *ctx, const float *rng, int64_t n_rng, int64_t *cursor,
                   int64_t n_moves, int64_t *moves_done, yamc_move_record *log,
                   double *rows, int32_t max_rows, int32_t *n_rows);
/* Same loop with the random stream and outputs already on the device (device
   pointers); used by the benchmark to time the device-resident path. */
int yamc_run_chain_device(yamc_ctx *ctx, const float *d_rng, int64_t n_rng, int64_t *cursor,
                          int64_t n_moves, int64_t *moves_done, yamc_move_record *d_log,
                          double *d_rows, int32_t max_rows, int32_t *n_rows);

/* ---- NPT: volume moves (mcvol, MC.f90:701-825) ----
   yamc_run_mc is run_mc (runmc.f90:178-334) by cycles, with the volume cycles of an NPT run
   (pressure_step_multiplier > 0): each cycle draws rnd = rand()*(psm+1); when psm > 0 and
   rnd > psm the cycle is one volume step, otherwise nmol movemc calls on the device (the chain
   kernel runs the move steps and stops before a volume cycle or an exchange step, which the
   host runs).  A volume
   step draws lambda, scales the box (scale_box, scale_box.f90:6-62), recomputes the parameters,
   the LJ tables and beta_LJ for the new length, scales beta by xclb_new/xclb_old, redoes the
   full sums on the device and takes the Metropolis test
   exp(-dU - P dV + (nmol+1) ln(V_new/V_old)), drawing only when that is not above 1; a
   rejected step restores the state as mc_restore_state does.  rng is a HOST pointer (copied to
   the device inside the call).  log: up to max_log movemc records (whole cycles only); vlog: up
   to max_vlog volume records; rows: energy.dat rows (frame + 8 columns, as yamc_run_chain).
   Returns YAMC_ERNG_EXHAUSTED when the stream runs out (an interrupted volume step is undone and
   its cycle draw given back; an interrupted move cycle resumes where it stopped).  With
   pressure_step_multiplier 0 it is the NVT loop of yamc_run_chain counted in cycles, and
   yamc_run_chain refuses NPT parameters. */
int yamc_run_mc(yamc_ctx *ctx, const float *rng, int64_t n_rng, int64_t *cursor, int64_t n_cycles,
                int64_t *cycles_done, yamc_move_record *log, int64_t max_log, int64_t *n_log,
                yamc_volume_record *vlog, int64_t max_vlog, int64_t *n_vlog, double *rows,
                int32_t max_rows, int32_t *n_rows);
/* The volume step as a drop-in for the body of mcvol, for a host that draws its own random
   numbers: yamc_volume_eval takes the new box length (Angstrom; MC.f90:738-746 compute it from
   lambda), does MC.f90:756-785 and returns dU = U_new - U_old and the overlap flag;
   yamc_volume_commit then keeps the new box (accepted != 0) or restores the old one
   (MC.f90:807-818). */
int yamc_volume_eval(yamc_ctx *ctx, double new_box_length, double *du, int32_t *overlap);
int yamc_volume_commit(yamc_ctx *ctx, int32_t accepted);
/* The parameters as they stand (BoxLength and everything Parameters_recalc derives from it
   change with accepted volume steps). */
int yamc_get_params(yamc_ctx *ctx, yamc_params *p);

/* ---- exchange moves (mc_xchange, MC.f90:1325-1954) ----
   init_freq with the exchange column of a frequencies file (runmc.f90:25-173): weights[nmol]
   give xchange_freq (BiasedRandom_init) and the probability Sxch / (Smv + Sxch) that a move
   step of run_mc is an exchange step (Smv: the move weights' sum).  With a positive
   probability the chain kernel stops before each exchange step (its exchange draw below the
   probability) and yamc_run_mc runs the step on the host (two molecules from xchange_freq,
   different, swap their centres of mass; acceptance by MonteCarloMove_accept_or_decline_simple)
   before relaunching the chain; exchange records have flags bit2 set, imol = the first
   molecule and the second in flags bits 8..31.
   yamc_run_chain refuses a context with exchange steps on. */
int yamc_set_xchange_weights(yamc_ctx *ctx, const double *weights);
/* The exchange step as a drop-in for the body of mc_xchange, for a host that draws its own
   random numbers: yamc_xchange_eval(imol1 != imol2, 1-based) returns du = {dU_real, dU_k_coulomb,
   dU_k_LJ, dU_ext} as the reference forms them (its real-space part holds the 1-2 pair energy
   change twice, MC.f90:1451-1452, 1639-1642) and *overlap (then du = 0 and the step is
   rejected without a draw); yamc_xchange_commit keeps the swap (accepted != 0) or drops it. */
int yamc_xchange_eval(yamc_ctx *ctx, int32_t imol1, int32_t imol2, double du[4], int32_t *overlap);
int yamc_xchange_commit(yamc_ctx *ctx, int32_t accepted);

/* ---- radial distribution functions of molecule centres (mcrdf2.f90:110-440) ----
   The reference computes them offline from the trajectory; here frames are added on the GPU,
   from host arrays of molecule centres (a trajectory frame) or straight from a context's
   device-resident positions.  For every frame: every ordered pair (i, j) of centres and, when
   rmax reaches past L/2, the periodic images, counted per species pair (t1 <= t2) into bins of
   width dr (count_distances, mcrdf2.f90:110-333).  mol_type[nmol]: 1-based species of each
   molecule (composition order); mol_numbers[ntypes]: molecules per species.  nbin =
   aint((rmax - 1e-10)/dr) + 2.  yamc_rdf_result: counts[(t1*ntypes + t2)*nbin + b] (0-based
   species) and the written g(r) of save_rdfs (mcrdf2.f90:371-440) at r = (b + 1/2) dr:
   counts / N_frame / <1/V> / N_t1 / N_t2 / dV / (2 if t1 != t2), dV = 4 pi dr (r^2 + r dr) +
   4/3 pi dr^3.  The reference's interpolated and 1/r^2-weighted histograms, which save_rdfs does
   not write, are not formed. */
typedef struct yamc_rdf yamc_rdf;
int yamc_rdf_create(int32_t nmol, const int32_t *mol_type, int32_t ntypes, const int32_t *mol_numbers,
                    double dr, double rmax, int32_t device, yamc_rdf **out);
int yamc_rdf_destroy(yamc_rdf *h);
int yamc_rdf_nbin(yamc_rdf *h, int32_t *nbin);
/* centres in box units (HOST arrays, nmol each), box length in Angstrom */
int yamc_rdf_add_frame(yamc_rdf *h, const double *x, const double *y, const double *z, double box_length);
/* the context's current configuration: centres of mass (center_of_mass, geometry.f90:170-201)
   computed on the device from its positions; the context must be on the RDF's device */
int yamc_rdf_add_ctx(yamc_rdf *h, yamc_ctx *ctx);
/* g and counts: ntypes*ntypes*nbin each (entries with t1 > t2 are 0); either may be NULL */
int yamc_rdf_result(yamc_rdf *h, double *g, double *counts, int32_t *n_frames);

/* Mixed form (params.precision = YAMC_MIXED): the chain kernel recomputes rho(k)
   and the k-space energies in FP64 from the positions after every
   `accepted_moves` accepted moves (default 10000; 0 = never), bounding the drift
   of the running sums that FP32 deltas update.  yamc_refresh_count returns how
   many refreshes ran. */
int yamc_set_refresh(yamc_ctx *ctx, int64_t accepted_moves);
int yamc_refresh_count(yamc_ctx *ctx, int64_t *count);

/* ---- launch configuration and diagnostics ---- */
/* Threads per block and blocks per cluster of the persistent chain kernel
   (0 = autotuned); takes effect on the next yamc_run_chain. */
int yamc_set_launch(yamc_ctx *ctx, int32_t cluster_blocks, int32_t threads);
/* Where the chain kernel keeps the signed k entries (k, beta, beta_LJ, rho(k)):
   in registers, at most 2 per worker thread, for the whole launch; or streamed
   from device memory (L2-resident) by every pass, any k-set size.  AUTO takes
   registers when they fit. */
#define YAMC_KSPACE_AUTO 0
#define YAMC_KSPACE_REGISTERS 1
#define YAMC_KSPACE_STREAMED 2
int yamc_set_kspace_layout(yamc_ctx *ctx, int32_t layout);
/* out: cluster blocks, threads, entries per thread (0 = streamed), shared memory bytes */
int yamc_get_launch(yamc_ctx *ctx, int32_t out[4]);
/* device time (ms) of the last run_chain kernel, measured with CUDA events on its stream */
int yamc_last_kernel_ms(yamc_ctx *ctx, double *ms);
/* Per-phase clock64 cycles of the chain kernel, summed over moves by block 0, in the order
   choose, speculate, propose, tables, kspace, pair_filter, pairs, reduce, old_pass,
   metropolis, commit, kspace_next (control warp: molecule choice, speculation of the next
   move, proposal, reduction, the force-biased old pass with its reduction, Metropolis,
   commit; worker warps: phase tables, k-space, pair filter, pairs; kspace_next is unused).
   mode 1 = reset and enable, 0 = disable,
   2 = read only; out receives min(n, 12) counters in that order. */
int yamc_phase_cycles(yamc_ctx *ctx, int32_t mode, int64_t *out, int32_t n);
/* No counterpart in the reference (whose checked build is gfortran's -ffpe-trap=invalid debug
   Makefile): *checked = 1 for the bounds-checked build of this library, 0 otherwise; and one
   checked read of a 4-value device array at `index` with the array taken as `size` long (at most
   4), on device `device`, with no context: *value = the value read (array[0] when the index is
   out of bounds) and *line = the source line the check recorded (0 when the index was in
   bounds) -- the index check on its own, in every build, for tests. */
int yamc_checked_build(int32_t *checked);
int yamc_bounds_check_selftest(int32_t device, int64_t index, int64_t size, double *value, int32_t *line);
const char *yamc_error_string(int status);
const char *yamc_last_error_detail(void);

/* ---- batched replicas ----
   No counterpart in the reference, which runs one chain per process (run_mc,
   runmc.f90:178-334).  A batch holds n independent replicas -- each a full system
   with its own size, box, temperature, composition and random stream -- and
   advances all of them together: one persistent cluster launch per group of
   replicas that share a kernel variant (LJ type count, force bias on or off), the
   groups concurrently, the whole step replayed as one CUDA graph. */
typedef struct yamc_batch yamc_batch;
/* systems[n], params[n] as for yamc_create (initmc of every replica). */
int yamc_batch_create(int32_t n, const yamc_system *systems, const yamc_params *params,
                      int32_t device, yamc_batch **out);
int yamc_batch_destroy(yamc_batch *b);
/* Replica i as a context (owned by the batch): yamc_energies, yamc_full_sums,
   yamc_get_positions and the other per-context calls work on it between steps. */
int yamc_batch_replica(yamc_batch *b, int32_t i, yamc_ctx **ctx);
/* n_moves movemc calls of every replica.  Replica i's random stream is
   d_rng[i][0 .. n_rng[i]) (device memory); cursors[i] (in/out) indexes it.
   moves_done[i], status[i] (optional) as for yamc_run_chain; d_log: NULL or
   n x n_moves records, replica i from i*n_moves.  Returns the first error of any
   replica, else YAMC_ERNG_EXHAUSTED if some stream ran out (that replica stops
   at the move it could not complete and resumes from its cursor). */
int yamc_batch_run_device(yamc_batch *b, const float *const *d_rng, const int64_t *n_rng,
                          int64_t *cursors, int64_t n_moves, int64_t *moves_done,
                          int32_t *status, yamc_move_record *d_log);
/* The same with the streams in host memory (each replica's unread window
   [cursors[i], n_rng[i]) is copied to the device) and the log in host memory. */
int yamc_batch_run(yamc_batch *b, const float *const *rng, const int64_t *n_rng, int64_t *cursors,
                   int64_t n_moves, int64_t *moves_done, int32_t *status, yamc_move_record *log);
/* Replicas are grouped by kernel variant (LJ type count, force bias, precision)
   and size class (atom count up to 1024 / 2048 / 4096 / 8192 / more); each group
   is one cluster launch with a shape of its own, the groups run concurrently.
   Autotuner: for each group alone, times every launch shape (k-space layout x
   cluster size x threads per block) that fits its replicas on n_moves moves of
   each and keeps the one with the most moves/s per SM it occupies (the groups
   share the GPU); then, with all groups running together, tries each group's next
   three shapes by that measure and its three fastest shapes alone, keeping a change
   when the whole batch's moves/s rises by 2 %.  The replicas' state is put back after every trial, so the chains do not
   advance.  best_moves_per_s: the whole batch's moves/s with the chosen shapes. */
int yamc_batch_tune(yamc_batch *b, const float *const *d_rng, const int64_t *n_rng,
                    const int64_t *cursors, int64_t n_moves, double *best_moves_per_s);
int yamc_batch_set_launch(yamc_batch *b, int32_t cluster_blocks, int32_t threads);
int yamc_batch_set_kspace_layout(yamc_batch *b, int32_t layout);
/* out: cluster blocks, threads, entries per thread, shared memory bytes, clusters
   resident at once (of the first group) */
int yamc_batch_get_launch(yamc_batch *b, int32_t out[5]);
/* the groups: their number, and per group the out[5] above plus its replica count
   and precision (1 = mixed) */
int yamc_batch_groups(yamc_batch *b, int32_t *n);
int yamc_batch_group_launch(yamc_batch *b, int32_t group, int32_t out[7]);
/* device time (ms, CUDA events on the batch stream) of the last run, and the kernels it
   launched (per variant group: the staging-order kernel and the chain kernel) */
int yamc_batch_last_kernel_ms(yamc_batch *b, double *ms);
int yamc_batch_last_launches(yamc_batch *b, int32_t *n);

/* ---- allocation-free real-space sums ----
   No counterpart in the reference: an extra entry point for callers that cannot
   call cudaMalloc where they need an energy (a host whose own pool holds the
   device memory, or one that cannot take the synchronisation that cudaMalloc and
   cudaFree may cause).  It computes the full real-space Ewald sum of a whole
   configuration -- the real-space half of yamc_full_sums -- from the caller's
   DEVICE arrays into the caller's DEVICE outputs and allocates nothing: its only
   scratch is a fixed static device array, sized for YAMC_STATIC_MAX_ATOMS atoms
   (64 KiB, held by every GPU that loads the library until the process exits).
   Inputs, all device pointers on the current device: x, y, z (box units), charge,
   mol (any molecule id per atom; equal ids = same molecule, intra pairs use
   -erf_Luc), lj_type (0 = no LJ, else 1..n_types), hard_core_angstr, and the
   n_types x n_types tables sigma6_tab (sigma^6 in box units) and four_eps_tab
   (4 epsilon / kT) at offset (t1-1)*n_types + t2-1, as LJTypes builds them.  From
   p: BoxLength, alpha, rmax2, xclb, two_alpha_over_sqrt_pi.  Outputs: uu, fx, fy,
   fz (natom doubles each, per-atom energy and force; any may be NULL) and sums[8]
   = uu_ew, uu_lj6, uu_lj12, their intra-molecular parts, overlap (1 when two LJ
   sites of different molecules are closer than their mean hard-core diameter)
   and bad_type (1 when some lj_type is outside 0..n_types; those atoms get no LJ).
   Asynchronous on `stream` (a cudaStream_t, NULL = default stream): read the
   outputs after that stream has finished.  natom above YAMC_STATIC_MAX_ATOMS is
   rejected with YAMC_ELIMITS.  Every call looks up the static array's device
   address in the current context (cudaGetSymbolAddress, which allocates nothing),
   so a device reset between calls is followed; the first call on a device loads
   the library's device code and should come before any stream capture.  Every
   call on a device shares the one scratch array: calls that overlap on the GPU
   (other streams, other host threads) race on it. */
#define YAMC_STATIC_MAX_ATOMS 262144
int yamc_realspace_sums_static(const yamc_params *p, int32_t natom, const double *x, const double *y,
                               const double *z, const double *charge, const int32_t *mol,
                               const int32_t *lj_type, const double *hard_core_angstr, int32_t n_types,
                               const double *sigma6_tab, const double *four_eps_tab, double *uu,
                               double *fx, double *fy, double *fz, double *sums, void *stream);

/* ---- measurement ----
   No counterpart in the reference.  The FP64 (fp64 != 0) or FP32 fused-multiply-add
   throughput of GPU `device` in TFLOP/s (2 flops per FMA), measured: independent FMA
   recurrences on every SM, the median of 5 timed launches of about 10-20 ms after one
   warm-up.  The trial move is not a contraction, so this -- not the tensor-core peak --
   is the compute roofline of the chain kernel.  Allocates and frees a few MB of device
   memory and its own stream; synchronous. */
int yamc_fma_peak(int32_t device, int32_t fp64, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
