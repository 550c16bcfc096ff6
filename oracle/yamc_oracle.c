/*
 * yamc_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the YAMC
 * per-trial-move energy path.  A plain-C restatement of the reference
 * Fortran; each routine cites the reference file:line it follows.  Paths
 * are the reference project's own file names.  Build: oracle/Makefile
 * (gcc -O2 -ffp-contract=off for parity; a second -O3 -march=native build
 * is the timed CPU baseline).
 *
 * Indexing: the reference is 1-based; here atoms and molecules are 0-based
 * internally, molecule numbers stored per atom (molnum) and the imol given
 * to movemc stay 1-based like the Fortran.
 */
#include "yamc_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* constants.f90:5-13 */
static const double PI = 3.14159265358979323846;
static const double TWO_PI = 2.0 * 3.14159265358979323846;
static const double FOUR_PI = 4.0 * 3.14159265358979323846;
static const double BOLTZ = 1.38065e-23;
static const double ELEC = 1.602176e-19;
static const double EPSI0 = 8.854187e-12;
static const double KCAL_MOL = 6.9477e-21;

#define MAX_LJ_TYPE 20      /* LJTypes.f90:20 */
#define MAX_MOL_TYPES 16
#define MAX_MOL_ATOMS 64

/* gfortran expands x**n (integer n) into multiplications; square-and-multiply
   keeps the value within an ulp of that expansion. */
static double ipow(double x, int n) {
    double r = 1.0, b = x;
    int first = 1;
    while (n > 0) {
        if (n & 1) { r = first ? b : r * b; first = 0; }
        n >>= 1;
        if (n) b = b * b;
    }
    return r;
}

/* ------------------------------------------------------------------ */
/* parameters.f90                                                      */
/* ------------------------------------------------------------------ */

/* parameters.f90:18-72 defaults */
void orc_params_defaults(orc_params *p) {
    memset(p, 0, sizeof(*p));
    p->sr = 4.0; p->sk = 4.0; p->alphaL = 0.0; p->temp = 298.15;
    p->external_permutivity = 50.0; p->BoxLength = 0.0; p->density = 33.33;
    p->dr_a = 0.4; p->d_angle_degree = 40.0; p->xlambda_c = 0.5; p->xlambda_f = 0.5;
    p->rnd_seed = 0; p->pressure = 0.0; p->pressure_step_multiplier = 0.0;
    p->max_volume_scaling = 1.05; p->max_cycle = 1000000;
    p->n_store_traj_interval = 100.0; p->n_store_energy_interval = 100.0;
    p->input_nbytes_xyz = 2; p->input_nbytes_ang = 2;
    p->output_nbytes_xyz = 2; p->output_nbytes_ang = 2;
    strcpy(p->freq_file, "none");
}

/* read_parameter (parameters.f90:102-148): name/value dispatch */
static void read_parameter(orc_params *p, const char *nam, const char *val) {
#define RD(key, field) if (!strcmp(nam, key)) p->field = strtod(val, NULL)
#define RI(key, field) if (!strcmp(nam, key)) p->field = (int32_t)strtol(val, NULL, 10)
    RD("sr", sr); RD("sk", sk); RD("alphaL", alphaL); RD("temp", temp);
    RD("external_permutivity", external_permutivity); RD("BoxLength", BoxLength);
    RD("density", density); RD("dr_a", dr_a); RD("d_angle_degree", d_angle_degree);
    RD("xlambda_c", xlambda_c); RD("xlambda_f", xlambda_f);
    RI("input_nbytes_xyz", input_nbytes_xyz); RI("input_nbytes_ang", input_nbytes_ang);
    RI("output_nbytes_xyz", output_nbytes_xyz); RI("output_nbytes_ang", output_nbytes_ang);
    RD("pressure_step_multiplier", pressure_step_multiplier);
    RD("max_volume_scaling", max_volume_scaling);
    RD("n_store_traj_interval", n_store_traj_interval);
    RD("n_store_energy_interval", n_store_energy_interval);
    RI("max_cycle", max_cycle); RD("pressure", pressure); RI("random_seed", rnd_seed);
    if (!strcmp(nam, "freq_file")) { strncpy(p->freq_file, val, 255); p->freq_file[255] = 0; }
#undef RD
#undef RI
}

/* Parameters_read (parameters.f90:266-305): '=' becomes a blank, the first two
   list-directed tokens are name and value, a name starting with '#' is a comment */
int orc_params_read(orc_params *p, const char *path) {
    FILE *f = fopen(path, "r");
    if (!f) return -2;
    char line[1024];
    while (fgets(line, sizeof line, f)) {
        for (char *c = line; *c; c++) if (*c == '=' || *c == ',' || *c == '\t' || *c == '\n' || *c == '\r') *c = ' ';
        char nam[256], val[512];
        int n = sscanf(line, "%255s %511s", nam, val);
        if (n <= 0) continue;           /* empty line */
        if (nam[0] == '#') continue;     /* comment */
        if (n < 2) continue;
        read_parameter(p, nam, val);
    }
    fclose(f);
    p->are_read = 1;
    return 0;
}

/* Parameters_read_string (parameters.f90:209-263): "nam1=val1,nam2=val2" */
int orc_params_read_string(orc_params *p, const char *str) {
    char buf[2048];
    strncpy(buf, str, sizeof buf - 1); buf[sizeof buf - 1] = 0;
    char *save = NULL;
    for (char *tok = strtok_r(buf, ",", &save); tok; tok = strtok_r(NULL, ",", &save)) {
        char *eq = strchr(tok, '=');
        if (!eq) return -4;
        *eq = 0;
        char nam[256], val[512];
        if (sscanf(tok, "%255s", nam) != 1 || sscanf(eq + 1, "%511s", val) != 1) return -4;
        read_parameter(p, nam, val);
    }
    return 0;
}

/* Parameters_recalc (parameters.f90:355-413) */
int orc_params_recalc(orc_params *p, double box_length) {
    if (!p->are_read) return -5;
    p->BoxLength = box_length;
    p->alpha = p->alphaL;
    if (p->alpha < 1e-9) p->alpha = 2.0 * p->sr;
    p->rmax = p->sr / p->alpha;
    p->kmax = (int32_t)lround(p->sk * p->alpha / PI);
    /* the reference build folds the constant ratio first: parameters.out holds
       (boltz/kcal_mol)*temp and 2*xclb*(pi/(2*eps+1)) to the bit */
    p->kT_kcal_mol = (BOLTZ / KCAL_MOL) * p->temp;
    p->dbjr_a = ELEC * ELEC / (4.0 * PI * EPSI0 * BOLTZ * p->temp) / 1.0e-10;
    p->dbjr = p->dbjr_a / p->BoxLength;
    p->xclb = p->dbjr;
    p->dr = p->dr_a / p->BoxLength;
    p->d_angle = p->d_angle_degree * PI / 180.0;
    p->alpha_over_sqrt_pi = p->alpha / sqrt(PI);
    p->two_alpha_over_sqrt_pi = 2.0 * p->alpha_over_sqrt_pi;
    p->kext = 2.0 * p->xclb * (PI / (2.0 * p->external_permutivity + 1.0));
    p->minus_two_kext = -2 * p->kext;
    p->rmax2 = p->rmax * p->rmax;
    p->log_max_volume_scaling = log(p->max_volume_scaling);
    p->pressure_angstr_kT = p->pressure / (BOLTZ * p->temp) * 1.0e-30;
    p->alphaL = p->alpha;
    return 0;
}

/* Parameters_init (parameters.f90:323-352) + BoxLength_from_density (:307-321) */
int orc_params_init(orc_params *p, int32_t nmol) {
    if (fabs(p->BoxLength) < 1e-9) {
        if (fabs(p->density) < 1e-9) return -4;
        double volume = nmol / p->density;
        p->BoxLength = pow(volume, 1.0 / 3.0) * 10.0;
    }
    return orc_params_recalc(p, p->BoxLength);
}

/* ------------------------------------------------------------------ */
/* Functions.f90                                                       */
/* ------------------------------------------------------------------ */

/* erfc_Luc (Functions.f90:116-142) with x2 = x^2 and ee2 = exp(-x^2) given */
static double erfc_luc3(double x, double x2, double ee2) {
    const double P = 0.3275911, A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741,
                 A4 = -1.453152027, A5 = 1.061405429, pi05 = 1.7724538509055;
    if (x < 0.455) {
        return 1.0 - 2.0 / pi05 * x * (1.0 - x2 * (1.0 / 3.0 - x2 * (0.1 - x2 * (1.0 / 42.0 - x2 / 216.0))));
    } else if (x > 3.0) {
        double ax = (1.0 - 0.5 * (1.0 - 1.5 / x2) / x2) / (pi05 * x);
        return ax * ee2;
    } else {
        double t = 1.0 / (1.0 + P * x);
        double ax = t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5))));
        return ax * ee2;
    }
}

/* erf_Luc (Functions.f90:145-171) */
static double erf_luc3(double x, double x2, double ee2) {
    const double P = 0.3275911, A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741,
                 A4 = -1.453152027, A5 = 1.061405429, pi05 = 1.7724538509055;
    if (x < 0.455) {
        return 2.0 / pi05 * x * (1.0 - x2 * (1.0 / 3.0 - x2 * (0.1 - x2 * (1.0 / 42.0 - x2 / 216.0))));
    } else if (x > 3.0) {
        double ax = (1.0 - 0.5 * (1.0 - 1.5 / x2) / x2) / (pi05 * x);
        return 1.0 - ax * ee2;
    } else {
        double t = 1.0 / (1.0 + P * x);
        double ax = t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5))));
        return 1.0 - ax * ee2;
    }
}

double orc_erfc_luc(double x) { double x2 = x * x; return erfc_luc3(x, x2, exp(-x2)); }
double orc_erf_luc(double x) { double x2 = x * x; return erf_luc3(x, x2, exp(-x2)); }

/* erfc_Luc_bet6_bet12 (Functions.f90:26-111); n and i are implicit integers */
void orc_erfc_bet6_bet12(double x, double x2, double e2, double *erfk, double *bet6, double *bet12) {
    double pi = 4.0 * atan(1.0);
    double pi12 = sqrt(pi);
    double pi15 = pow(pi, 1.5);
    const double xmin = 0.5, xmax = 8.0;
    if (x <= xmin) {
        *erfk = erfc_luc3(x, x2, e2);
        *bet6 = pi15 / 3.0 * ipow(x, 3) * (pi12 * (*erfk) + (0.5 / x2 - 1.0) / x * e2);
        *bet12 = pi15 / 1080.0 * ipow(x, 9) *
                 (-16.0 * pi12 / 105.0 * (*erfk) +
                  (((((1.0 / x2 - 2.0 / 7.0) / x2 + 4.0 / 35.0) / x2 - 8.0 / 105.0) / x2 + 16.0 / 105.0)) / x * e2);
    } else if (x >= xmax) {
        *erfk = e2 / pi12 / x * (1.0 - 0.5 / x2 * (1.0 - 1.5 / x2 * (1.0 - 2.5 / x2)));
        *bet6 = pi15 * e2 / 4.0 / ipow(x, 2) * (1.0 - 2.5 / x2 * (1.0 - 3.5 / x2 * (1.0 - 4.5 / x2)));
        *bet12 = pi15 * e2 / 240.0 / ipow(x, 2) * (1.0 - 5.5 / x2 * (1.0 - 6.5 / x2 * (1.0 - 7.5 / x2)));
    } else {
        double dx = 1.0e-3;
        int n = (int)((xmax - x) / dx + 2);
        dx = (xmax - x) / (n - 1);
        double som = dx * e2 / 2.0 - dx * dx / 12.0 * 2.0 * x * e2;
        double som6 = dx * e2 / ipow(x, 4) / 2.0 - dx * dx / 12.0 * (2.0 / ipow(x, 3) + 4.0 / ipow(x, 5)) * e2;
        double som12 = dx * e2 / ipow(x, 10) / 2.0 - dx * dx / 12.0 * (2.0 / ipow(x, 9) + 10.0 / ipow(x, 11)) * e2;
        double y = x, e = e2;
        for (int i = 2; i <= n; i++) {
            y = x + (double)(i - 1) * dx;
            e = exp(-(y * y));
            som = som + dx * e;
            som6 = som6 + dx * e / ipow(y, 4);
            som12 = som12 + dx * e / ipow(y, 10);
        }
        som = som - dx * e / 2.0 + dx * dx / 12.0 * 2.0 * y * e;
        double y2 = y * y;
        som = som + e / 2.0 / y * (1.0 - 0.5 / y2 * (1.0 - 1.5 / y2 * (1.0 - 2.5 / y2)));
        *erfk = 2.0 / pi12 * som;
        som6 = som6 - dx * e / ipow(y, 4) / 2.0 + dx * dx / 12.0 * (2.0 / ipow(y, 3) + 4.0 / ipow(y, 5)) * e;
        som6 = som6 + e / 2.0 / ipow(y, 5) * (1.0 - 2.5 / y2 * (1.0 - 3.5 / y2 * (1.0 - 4.5 / y2)));
        *bet6 = pi15 * ipow(x, 3) / 2.0 * som6;
        som12 = som12 - dx * e / ipow(y, 10) / 2.0 + dx * dx / 12.0 * (2.0 / ipow(y, 9) + 10.0 / ipow(y, 11)) * e;
        som12 = som12 + e / 2.0 / ipow(y, 11) * (1.0 - 5.5 / y2 * (1.0 - 6.5 / y2 * (1.0 - 7.5 / y2)));
        *bet12 = pi15 * ipow(x, 9) / 120.0 * som12;
    }
}

/* shi_sans_exp_f (Functions.f90:225-289): Shi(x) exp(-x) */
double orc_shi_sans_exp(double x) {
    const double dx0 = 0.2;
    double shi_f, x1;
    if (x <= 1.0) {
        double x2 = x * x, fac = 1.0, xn = x;
        shi_f = x;
        for (int i = 1; i <= 4; i++) {
            double deuxi = 2.0 * i;
            xn = xn * x2;
            fac = fac * (deuxi) * (deuxi + 1.0);
            shi_f = shi_f + xn / (deuxi + 1.0) / fac;
        }
        return exp(-x) * shi_f;
    } else if (x > 20.0) {
        double som = 1.0, term = 1.0;
        for (int i = 1; i <= 6; i++) { term = term * i / x; som = som + term; }
        return 1.0 / 2.0 / x * som;
    } else if (x < 5.0) { x1 = 1.0; shi_f = 1.057250875; }
    else if (x < 10.0) { x1 = 5.0; shi_f = 20.093211826; }
    else if (x < 15.0) { x1 = 10.0; shi_f = 1246.11449; }
    else { x1 = 15.0; shi_f = 117477.926; }
    int n = (int)((x - x1) / dx0 + 2);
    double dx = (x - x1) / (n - 1);
    shi_f = shi_f + dx * sinh(x1) / x1 / 2.0 + dx * dx / 12.0 * (cosh(x1) / x1 - sinh(x1) / (x1 * x1));
    double t = x1, s = 0.0;
    for (int i = 2; i <= n; i++) {
        t = x1 + (double)(i - 1) * dx;
        s = sinh(t);
        shi_f = shi_f + dx * s / t;
    }
    shi_f = shi_f - dx * s / t / 2.0 - dx * dx / 12.0 * (cosh(t) / t - s / (t * t));
    return exp(-x) * shi_f;
}

/* ------------------------------------------------------------------ */
/* FourierGrid.f90                                                     */
/* ------------------------------------------------------------------ */
typedef struct {
    int kmax, nk;
    int *kx, *ky, *kz, *ip, *iq;
    double *xk, *xk2;
} grid_t;

/* FourierGrid_calcNalloc (FourierGrid.f90:37-78) */
int32_t orc_grid_count(int32_t kmax) {
    double xkmax2 = (double)(kmax * kmax);
    int kk = 0;
    for (int kx = 0; kx <= kmax; kx++) {
        double xkx2 = (double)(kx * kx);
        int kymax = (int)sqrt(xkmax2 - xkx2);
        for (int ky = 0; ky <= kymax; ky++) {
            double xky2 = (double)(ky * ky);
            int kzmax = (int)sqrt(xkmax2 - xkx2 - xky2);
            for (int kz = 0; kz <= kzmax; kz++) {
                double xk2 = xkx2 + xky2 + (double)(kz * kz);
                if (xk2 < 0.1) continue;
                kk++;
            }
        }
    }
    return kk;
}

/* FourierGrid_init (FourierGrid.f90:118-189) */
static void grid_init(grid_t *g, int kmax) {
    int n = orc_grid_count(kmax);
    g->kmax = kmax; g->nk = n;
    g->kx = calloc(n, sizeof(int)); g->ky = calloc(n, sizeof(int)); g->kz = calloc(n, sizeof(int));
    g->ip = calloc(n, sizeof(int)); g->iq = calloc(n, sizeof(int));
    g->xk = calloc(n, sizeof(double)); g->xk2 = calloc(n, sizeof(double));
    double xkmax2 = (double)(kmax * kmax);
    int kk = 0;
    for (int kx = 0; kx <= kmax; kx++) {
        double xkx2 = (double)(kx * kx);
        int kymax = (int)sqrt(xkmax2 - xkx2);
        for (int ky = 0; ky <= kymax; ky++) {
            double xky2 = (double)(ky * ky);
            int kzmax = (int)sqrt(xkmax2 - xkx2 - xky2);
            for (int kz = 0; kz <= kzmax; kz++) {
                double xk2 = xkx2 + xky2 + (double)(kz * kz);
                if (xk2 < 0.1) continue;
                g->kx[kk] = kx; g->ky[kk] = ky; g->kz[kk] = kz;
                g->xk2[kk] = xk2; g->xk[kk] = sqrt(xk2);
                if (ky == 0) g->iq[kk] = (kz == 0) ? 1 : 3;
                else g->iq[kk] = (kz == 0) ? 2 : 4;
                g->ip[kk] = 0;
                kk++;
            }
            if (kk > 0) g->ip[kk - 1] = 1;
        }
        if (kk > 0) g->ip[kk - 1] = 2;
    }
    if (kk > 0) g->ip[kk - 1] = 3;
}

static void grid_free(grid_t *g) {
    free(g->kx); free(g->ky); free(g->kz); free(g->ip); free(g->iq); free(g->xk); free(g->xk2);
}

/* ------------------------------------------------------------------ */
/* SumSinCosKR.f90: 8 arrays per structure in the order                 */
/* cos_ppp, sin_ppp, cos_ppm, sin_ppm, cos_pmp, sin_pmp, cos_pmm, sin_pmm */
/* ------------------------------------------------------------------ */
enum { CPPP = 0, SPPP, CPPM, SPPM, CPMP, SPMP, CPMM, SPMM };

typedef struct { double *a[8]; } sck_t; /* TSinCosKR / TSumSinCosKR */

static void sck_alloc(sck_t *s, int nk) {
    double *blk = calloc((size_t)8 * nk, sizeof(double));
    for (int i = 0; i < 8; i++) s->a[i] = blk + (size_t)i * nk;
}
static void sck_free(sck_t *s) { free(s->a[0]); }
static void sck_zero(sck_t *s, int nk) { memset(s->a[0], 0, sizeof(double) * 8 * (size_t)nk); }
static void sck_copy(sck_t *d, const sck_t *s, int nk) { memcpy(d->a[0], s->a[0], sizeof(double) * 8 * (size_t)nk); }
/* SumSinCosKR_addAtom / addSum (SumSinCosKR.f90:590-630) */
static void sck_add(sck_t *d, const sck_t *s, int nk) {
    for (int c = 0; c < 8; c++) for (int k = 0; k < nk; k++) d->a[c][k] = d->a[c][k] + s->a[c][k];
}
/* SumSinCosKR_subSum (SumSinCosKR.f90:632-648) */
static void sck_sub(sck_t *d, const sck_t *s, int nk) {
    for (int c = 0; c < 8; c++) for (int k = 0; k < nk; k++) d->a[c][k] = d->a[c][k] - s->a[c][k];
}
/* SinCosKR_mulScalar (SumSinCosKR.f90:496-515) */
static void sck_mul(sck_t *d, double m, int nk) {
    for (int c = 0; c < 8; c++) for (int k = 0; k < nk; k++) d->a[c][k] = d->a[c][k] * m;
}

typedef struct { double *cx, *cy, *cz, *sx, *sy, *sz; } scxyz_t; /* TSinCosXYZ, 0..kmax */

/* SinCosXYZ_fill (SumSinCosKR.f90:181-223) */
static void scxyz_fill(scxyz_t *t, double x, double y, double z, int kmax) {
    double cx = cos(TWO_PI * x), sx = sin(TWO_PI * x);
    double cy = cos(TWO_PI * y), sy = sin(TWO_PI * y);
    double cz = cos(TWO_PI * z), sz = sin(TWO_PI * z);
    t->cx[0] = 1.0; t->sx[0] = 0.0; t->cy[0] = 1.0; t->sy[0] = 0.0; t->cz[0] = 1.0; t->sz[0] = 0.0;
    for (int k = 1; k <= kmax; k++) {
        t->cx[k] = t->cx[k - 1] * cx - t->sx[k - 1] * sx;
        t->sx[k] = t->sx[k - 1] * cx + t->cx[k - 1] * sx;
        t->cy[k] = t->cy[k - 1] * cy - t->sy[k - 1] * sy;
        t->sy[k] = t->sy[k - 1] * cy + t->cy[k - 1] * sy;
        t->cz[k] = t->cz[k - 1] * cz - t->sz[k - 1] * sz;
        t->sz[k] = t->sz[k - 1] * cz + t->cz[k - 1] * sz;
    }
}

/* SinCosKR_fill (SumSinCosKR.f90:297-455): row recurrence over the half-space list */
static void sck_fill(sck_t *o, const scxyz_t *t, double charge, const grid_t *g) {
    double qcp = charge, qsp = 0.0, qcm = charge, qsm = 0.0; /* cos/sin(xkx +- yky) * q */
    int nk = g->nk;
    for (int kk = 0; kk < nk; kk++) {
        int kz = g->kz[kk], ky = g->ky[kk];
        double q_cosxy_cosz = qcp * t->cz[kz];
        double q_sinxy_sinz = qsp * t->sz[kz];
        double q_sinxy_cosz = qsp * t->cz[kz];
        double q_cosxy_sinz = qcp * t->sz[kz];
        o->a[CPPP][kk] = q_cosxy_cosz - q_sinxy_sinz;
        o->a[SPPP][kk] = q_sinxy_cosz + q_cosxy_sinz;
        if (kz > 0) { o->a[CPPM][kk] = q_cosxy_cosz + q_sinxy_sinz; o->a[SPPM][kk] = q_sinxy_cosz - q_cosxy_sinz; }
        else { o->a[CPPM][kk] = 0.0; o->a[SPPM][kk] = 0.0; }
        double q_cosxmy_cosz = qcm * t->cz[kz];
        double q_sinxmy_sinz = qsm * t->sz[kz];
        double q_sinxmy_cosz = qsm * t->cz[kz];
        double q_cosxmy_sinz = qcm * t->sz[kz];
        if (ky > 0) { o->a[CPMP][kk] = q_cosxmy_cosz - q_sinxmy_sinz; o->a[SPMP][kk] = q_sinxmy_cosz + q_cosxmy_sinz; }
        else { o->a[CPMP][kk] = 0.0; o->a[SPMP][kk] = 0.0; }
        if (kz > 0 && ky > 0) { o->a[CPMM][kk] = q_cosxmy_cosz + q_sinxmy_sinz; o->a[SPMM][kk] = q_sinxmy_cosz - q_cosxmy_sinz; }
        else { o->a[CPMM][kk] = 0.0; o->a[SPMM][kk] = 0.0; }
        if (g->ip[kk] != 0 && kk < nk - 1) {
            int kx1 = g->kx[kk + 1], ky1 = g->ky[kk + 1];
            double q_cosx_cosy = charge * t->cx[kx1] * t->cy[ky1];
            double q_sinx_siny = charge * t->sx[kx1] * t->sy[ky1];
            double q_sinx_cosy = charge * t->sx[kx1] * t->cy[ky1];
            double q_cosx_siny = charge * t->cx[kx1] * t->sy[ky1];
            qcp = q_cosx_cosy - q_sinx_siny;
            qsp = q_sinx_cosy + q_cosx_siny;
            qcm = q_cosx_cosy + q_sinx_siny;
            qsm = q_sinx_cosy - q_cosx_siny;
        }
    }
}

/* ------------------------------------------------------------------ */
/* LJTypes.f90                                                         */
/* ------------------------------------------------------------------ */
typedef struct {
    int ntype;
    double sigma[MAX_LJ_TYPE], epsilon[MAX_LJ_TYPE];
    int *type_by_index;
    double *lj6, *lj12, *four_eps, *sigma6, *sigma2; /* ntype^2, offset (t1-1)*ntype+t2 - 1 */
} ljtypes_t;

/* LJTypes_fill_LJ_tab_index (LJTypes.f90:202-232) */
static void lj_fill_index(ljtypes_t *L, int i, int j, double sigma12, double epsilon12) {
    int o12 = (i - 1) * L->ntype + j - 1;
    double sp2 = sigma12 * sigma12;
    double sp6 = sp2 * sp2 * sp2;
    L->lj6[o12] = 4 * epsilon12 * sp6;
    L->lj12[o12] = L->lj6[o12] * sp6;
    L->sigma2[o12] = sp2;
    L->sigma6[o12] = sp6;
    L->four_eps[o12] = 4 * epsilon12;
    if (i == j) return;
    int o21 = (j - 1) * L->ntype + i - 1;
    L->lj6[o21] = L->lj6[o12];
    /* LJ12Tab(offset21) is a self-assignment in the reference (LJTypes.f90:230) and never read */
    L->sigma2[o21] = sp2;
    L->sigma6[o21] = sp6;
    L->four_eps[o21] = 4 * epsilon12;
}

/* LJTypes_fill_LJ_tab (LJTypes.f90:273-308): Lorentz-Berthelot tables from the type list */
static void lj_fill_tab(ljtypes_t *L) {
    int nt = L->ntype;
    for (int i = 1; i <= nt; i++) {
        double s1 = L->sigma[i - 1], e1 = L->epsilon[i - 1];
        lj_fill_index(L, i, i, s1, e1);
        for (int j = i + 1; j <= nt; j++) {
            double s2 = L->sigma[j - 1], e2 = L->epsilon[j - 1];
            lj_fill_index(L, i, j, (s1 + s2) / 2, sqrt(e1 * e2));
        }
    }
}

/* LJTypes_fill (LJTypes.f90:134-200) + LJTypes_fill_LJ_tab (:273-308) */
static int lj_fill(ljtypes_t *L, const double *sig, const double *eps, int n) {
    int nt = 0;
    for (int i = 0; i < n; i++) {
        if (sig[i] < (double)1e-8f) continue;
        int found = 0;
        for (int t = 0; t < nt; t++)
            if (fabs(sig[i] - L->sigma[t]) < 1e-8 && fabs(eps[i] - L->epsilon[t]) < 1e-8) { found = 1; break; }
        if (!found) {
            if (nt >= MAX_LJ_TYPE) return -3;
            L->sigma[nt] = sig[i]; L->epsilon[nt] = eps[i]; nt++;
        }
    }
    L->ntype = nt;
    L->type_by_index = calloc(n, sizeof(int));
    for (int i = 0; i < n; i++)
        for (int t = 0; t < nt; t++)
            if (fabs(sig[i] - L->sigma[t]) < 1e-8 && fabs(eps[i] - L->epsilon[t]) < 1e-8) { L->type_by_index[i] = t + 1; break; }
    int n2 = nt * nt > 0 ? nt * nt : 1;
    L->lj6 = calloc(n2, sizeof(double)); L->lj12 = calloc(n2, sizeof(double));
    L->four_eps = calloc(n2, sizeof(double)); L->sigma6 = calloc(n2, sizeof(double)); L->sigma2 = calloc(n2, sizeof(double));
    lj_fill_tab(L);
    return 0;
}

/* LJTypes_scale_sigma (LJTypes.f90:238-252): every type's sigma times c, tables refilled */
static void lj_scale_sigma(ljtypes_t *L, double c) {
    for (int i = 0; i < L->ntype; i++) L->sigma[i] = L->sigma[i] * c;
    lj_fill_tab(L);
}

/* ------------------------------------------------------------------ */
/* state (MC.f90:18-95 module globals)                                  */
/* ------------------------------------------------------------------ */
typedef struct {
    int natoms;
    double x[MAX_MOL_ATOMS], y[MAX_MOL_ATOMS], z[MAX_MOL_ATOMS], sigma[MAX_MOL_ATOMS];
    double epsilon[MAX_MOL_ATOMS], charge[MAX_MOL_ATOMS], mass[MAX_MOL_ATOMS], hard_core[MAX_MOL_ATOMS];
} mol_t;

typedef struct {           /* TRhoSquared (RhoSquared.f90:9-45) */
    sck_t coul;
    sck_t lj[MAX_LJ_TYPE];
    int present[MAX_LJ_TYPE];
} rho_t;

typedef struct {           /* TEwaldSumRealSpace partial sum (EwaldSumRealSpace.f90:32-58) */
    double uu_ew, uu_lj6, uu_lj12, uu_ew_intra, uu_lj6_intra, uu_lj12_intra;
    double uu[MAX_MOL_ATOMS], fx[MAX_MOL_ATOMS], fy[MAX_MOL_ATOMS], fz[MAX_MOL_ATOMS];
    double *uu_back, *fx_back, *fy_back, *fz_back;
} partial_t;

struct orc_state {
    orc_params p;
    int nmoltypes; mol_t moltypes[MAX_MOL_TYPES]; int mol_numbers[MAX_MOL_TYPES];
    /* molecule table */
    int nmol, max_mol_atom;
    int *mol_type, *first_atom, *last_atom; /* 0-based atom ranges, inclusive */
    double *mx, *my, *mz, *mtheta, *mphi, *mpsi;
    /* atomic data (AtomicData.f90:9-22) */
    int N;
    double *xx, *yy, *zz, *sigma, *epsilon, *charge, *hard_core, *mass;
    int *molnum; /* 1-based */
    ljtypes_t lj;
    grid_t g;
    double *beta, *beta6, *beta12;
    double **beta_lj; /* ntype^2 pointers, (t2,t1) aliases (t1,t2) */
    rho_t rho_total, mol_old, mol_new, total_new;
    sck_t *skr_coul, *skr_lj; /* per molecule atom (MC.f90:55-56) */
    scxyz_t xyz;
    double *tc[4], *ts[4]; /* twoC_plus_dC / twoS_plus_dS temporaries (EwaldSumKSpace.f90:79-83) */
    /* full real-space sum */
    double *uu, *fx, *fy, *fz;
    double uu_ew, uu_lj6, uu_lj12, uu_ew_intra, uu_lj6_intra, uu_lj12_intra;
    partial_t ps_old, ps_new;
    double E_k, E_k_coul, E_k_lj;
    double mu_x, mu_y, mu_z;
    double U_tail, U_tail_coul, U_tail_lj6, U_tail_lj12, U_ext, U_total, U_total_ew, U_total_lj;
    /* run_mc state */
    double *freq_beg, *freq_end;
    double *xfreq_beg, *xfreq_end;     /* xchange_freq intervals (BiasedRandom_init on exchange weights) */
    double smv, xchange_probability;   /* SUM(mv_num) and Sxch / (Smv + Sxch) (init_freq, runmc.f90:25-67) */
    int64_t icycle, move_in_cycle;
    double n_mv_steps, n_mv_accepted, n_vol_steps, n_vol_accepted;
    /* RNG binding for the current call */
    const float *rng; int64_t n_rng; int64_t *cursor; int rng_out;
};

/* ------------------------------------------------------------------ */
/* random.f90 rand(): gfortran random_number with the [eps,1-eps] redraw */
/* ------------------------------------------------------------------ */
static double orc_rand(orc_state *s) {
    const double eps = 1e-14;
    float v = 0.0f;
    while ((double)v < eps || (double)v > 1.0 - eps) {
        if (*s->cursor >= s->n_rng) { s->rng_out = 1; return 0.5; }
        v = s->rng[(*s->cursor)++];
    }
    return (double)v;
}

/* ------------------------------------------------------------------ */
/* RhoSquared.f90                                                       */
/* ------------------------------------------------------------------ */
static void rho_alloc(rho_t *r, int nk, int nt) {
    sck_alloc(&r->coul, nk);
    for (int t = 0; t < nt; t++) sck_alloc(&r->lj[t], nk);
    memset(r->present, 0, sizeof r->present);
}
static void rho_free(rho_t *r, int nt) { sck_free(&r->coul); for (int t = 0; t < nt; t++) sck_free(&r->lj[t]); }
/* RhoSquared_nulify (:128-144) */
static void rho_zero(rho_t *r, int nk, int nt) {
    sck_zero(&r->coul, nk); for (int t = 0; t < nt; t++) sck_zero(&r->lj[t], nk);
    memset(r->present, 0, sizeof r->present);
}
/* RhoSquared_copy / _add / _sub (:296-341) */
static void rho_copy(rho_t *d, const rho_t *s, int nk, int nt) { sck_copy(&d->coul, &s->coul, nk); for (int t = 0; t < nt; t++) sck_copy(&d->lj[t], &s->lj[t], nk); }
static void rho_add(rho_t *d, const rho_t *s, int nk, int nt) { sck_add(&d->coul, &s->coul, nk); for (int t = 0; t < nt; t++) sck_add(&d->lj[t], &s->lj[t], nk); }
static void rho_sub(rho_t *d, const rho_t *s, int nk, int nt) { sck_sub(&d->coul, &s->coul, nk); for (int t = 0; t < nt; t++) sck_sub(&d->lj[t], &s->lj[t], nk); }

/* RhoSquared_addAtom (RhoSquared.f90:147-185) */
static void rho_add_atom(orc_state *s, rho_t *r, double x, double y, double z, double charge, int lj_type,
                         sck_t *kr_coul, sck_t *kr_lj) {
    int nk = s->g.nk;
    if (charge != 0.0) {
        scxyz_fill(&s->xyz, x, y, z, s->g.kmax);
        sck_fill(kr_coul, &s->xyz, charge, &s->g);
        sck_add(&r->coul, kr_coul, nk);
    } else {
        sck_zero(kr_coul, nk);
    }
    if (lj_type > 0) {
        if (charge != 0.0) {
            sck_copy(kr_lj, kr_coul, nk);
            sck_mul(kr_lj, 1.0 / charge, nk);
        } else {
            scxyz_fill(&s->xyz, x, y, z, s->g.kmax);
            sck_fill(kr_lj, &s->xyz, 1.0, &s->g);
        }
        sck_add(&r->lj[lj_type - 1], kr_lj, nk);
        r->present[lj_type - 1] = 1;
    }
}

/* ------------------------------------------------------------------ */
/* EwaldSumKSpace.f90                                                   */
/* ------------------------------------------------------------------ */

/* EwaldSumKSpace_initBeta (EwaldSumKSpace.f90:263-350) */
static void init_beta(orc_state *s) {
    double alpha = s->p.alpha, xclb = s->p.xclb;
    double pi_over_alpha = PI / alpha;
    double poa2 = pi_over_alpha * pi_over_alpha;
    for (int kk = 0; kk < s->g.nk; kk++) {
        double b2 = poa2 * s->g.xk2[kk];
        double e = exp(-b2);
        s->beta[kk] = xclb * e / s->g.xk2[kk] / TWO_PI;
        double b = pi_over_alpha * s->g.xk[kk];
        double erfc_b, B6, B12;
        orc_erfc_bet6_bet12(b, b2, e, &erfc_b, &B6, &B12);
        s->beta6[kk] = ipow(alpha, 3) * B6;
        s->beta12[kk] = ipow(alpha, 9) * B12;
        if (s->g.kx[kk] > 0) {
            s->beta[kk] = 2.0 * s->beta[kk];
            s->beta6[kk] = 2.0 * s->beta6[kk];
            s->beta12[kk] = 2.0 * s->beta12[kk];
        }
    }
}

/* EwaldSumKSpace_initBetaLJ (EwaldSumKSpace.f90:352-386) */
static void init_beta_lj(orc_state *s) {
    int nt = s->lj.ntype, nk = s->g.nk;
    for (int t1 = 1; t1 <= nt; t1++)
        for (int t2 = t1; t2 <= nt; t2++) {
            int o = (t1 - 1) * nt + t2 - 1;
            double a6 = s->lj.lj6[o], a12 = s->lj.lj12[o];
            for (int k = 0; k < nk; k++) s->beta_lj[o][k] = a12 * s->beta12[k] - a6 * s->beta6[k];
        }
}

/* EwaldSumKSpace_calc_coulomb_energy + RhoSquared_calc_rho_squared (:389-416, RhoSquared.f90:245-294) */
static double kspace_coulomb_energy(orc_state *s) {
    sck_t *r = &s->rho_total.coul;
    double U = 0;
    for (int kk = 0; kk < s->g.nk; kk++) {
        double r2 = r->a[CPPP][kk] * r->a[CPPP][kk] + r->a[SPPP][kk] * r->a[SPPP][kk];
        int sy = s->g.ky[kk] > 0, sz = s->g.kz[kk] > 0;
        if (sy) r2 = r2 + r->a[CPMP][kk] * r->a[CPMP][kk] + r->a[SPMP][kk] * r->a[SPMP][kk];
        if (sz) r2 = r2 + r->a[CPPM][kk] * r->a[CPPM][kk] + r->a[SPPM][kk] * r->a[SPPM][kk];
        if (sy && sz) r2 = r2 + r->a[CPMM][kk] * r->a[CPMM][kk] + r->a[SPMM][kk] * r->a[SPMM][kk];
        U = U + s->beta[kk] * r2;
    }
    return U;
}

/* EwaldSumKSpace_calc_LJ_energy (EwaldSumKSpace.f90:418-526) */
static double kspace_lj_energy(orc_state *s) {
    int nt = s->lj.ntype, nk = s->g.nk;
    double U = 0;
    for (int t1 = 1; t1 <= nt; t1++) {
        sck_t *a = &s->rho_total.lj[t1 - 1];
        for (int t2 = t1; t2 <= nt; t2++) {
            sck_t *b = &s->rho_total.lj[t2 - 1];
            double *bl = s->beta_lj[(t1 - 1) * nt + t2 - 1];
            double sk = 0;
            for (int kk = 0; kk < nk; kk++) {
                double l = a->a[CPPP][kk] * b->a[CPPP][kk] + a->a[SPPP][kk] * b->a[SPPP][kk];
                if (s->g.ky[kk] > 0) l = l + a->a[CPMP][kk] * b->a[CPMP][kk] + a->a[SPMP][kk] * b->a[SPMP][kk];
                if (s->g.kz[kk] > 0) l = l + a->a[CPPM][kk] * b->a[CPPM][kk] + a->a[SPPM][kk] * b->a[SPPM][kk];
                if (s->g.ky[kk] > 0 && s->g.kz[kk] > 0) l = l + a->a[CPMM][kk] * b->a[CPMM][kk] + a->a[SPMM][kk] * b->a[SPMM][kk];
                sk = sk + bl[kk] * l;
            }
            if (t1 != t2) sk = sk + sk;
            U = U + sk;
        }
    }
    return U;
}

/* EwaldSumKSpace_calc_total_energy (EwaldSumKSpace.f90:225-260) with RhoSquared_addAtoms (RhoSquared.f90:188-243) */
static void kspace_total_energy(orc_state *s) {
    int nk = s->g.nk, nt = s->lj.ntype;
    rho_zero(&s->rho_total, nk, nt);
    sck_t kc, kl; sck_alloc(&kc, nk); sck_alloc(&kl, nk);
    for (int i = 0; i < s->N; i++)
        rho_add_atom(s, &s->rho_total, s->xx[i], s->yy[i], s->zz[i], s->charge[i], s->lj.type_by_index[i], &kc, &kl);
    sck_free(&kc); sck_free(&kl);
    s->E_k_coul = kspace_coulomb_energy(s);
    s->E_k_lj = kspace_lj_energy(s);
    s->E_k = s->E_k_coul + s->E_k_lj;
}

/* EwaldSumKSpace_calc_dU_coulomb (EwaldSumKSpace.f90:528-620) */
static double kspace_du_coulomb(orc_state *s, const sck_t *d) {
    const sck_t *c = &s->rho_total.coul;
    double total = 0;
    for (int kk = 0; kk < s->g.nk; kk++) {
        double two_C = c->a[CPPP][kk] + c->a[CPPP][kk], dC = d->a[CPPP][kk];
        double two_S = c->a[SPPP][kk] + c->a[SPPP][kk], dS = d->a[SPPP][kk];
        double l = (two_C + dC) * dC + (two_S + dS) * dS;
        if (s->g.ky[kk] > 0) {
            two_C = c->a[CPMP][kk] + c->a[CPMP][kk]; dC = d->a[CPMP][kk];
            two_S = c->a[SPMP][kk] + c->a[SPMP][kk]; dS = d->a[SPMP][kk];
            l = l + (two_C + dC) * dC + (two_S + dS) * dS;
        }
        if (s->g.kz[kk] > 0) {
            two_C = c->a[CPPM][kk] + c->a[CPPM][kk]; dC = d->a[CPPM][kk];
            two_S = c->a[SPPM][kk] + c->a[SPPM][kk]; dS = d->a[SPPM][kk];
            l = l + (two_C + dC) * dC + (two_S + dS) * dS;
        }
        if (s->g.ky[kk] > 0 && s->g.kz[kk] > 0) {
            two_C = c->a[CPMM][kk] + c->a[CPMM][kk]; dC = d->a[CPMM][kk];
            two_S = c->a[SPMM][kk] + c->a[SPMM][kk]; dS = d->a[SPMM][kk];
            l = l + (two_C + dC) * dC + (two_S + dS) * dS;
        }
        total = total + l * s->beta[kk];
    }
    return total;
}

/* EwaldSumKSpace_calc_dU_LJ (EwaldSumKSpace.f90:623-753) */
static double kspace_du_lj(orc_state *s, const rho_t *delta) {
    int nt = s->lj.ntype, nk = s->g.nk;
    double total = 0;
    for (int t1 = 1; t1 <= nt; t1++) {
        const sck_t *C1 = &s->rho_total.lj[t1 - 1], *D1 = &delta->lj[t1 - 1];
        /* twoC_plus_dC_* = C1 + C1 + DeltaC1 (:699-707); index order ppp, ppm, pmp, pmm */
        for (int c = 0; c < 4; c++)
            for (int k = 0; k < nk; k++) {
                s->tc[c][k] = C1->a[2 * c][k] + C1->a[2 * c][k] + D1->a[2 * c][k];
                s->ts[c][k] = C1->a[2 * c + 1][k] + C1->a[2 * c + 1][k] + D1->a[2 * c + 1][k];
            }
        for (int t2 = 1; t2 <= nt; t2++) {
            if (!delta->present[t2 - 1]) continue;
            const double *bl = s->beta_lj[(t1 - 1) * nt + t2 - 1];
            const sck_t *D2 = &delta->lj[t2 - 1];
            for (int kk = 0; kk < nk; kk++) {
                double l = s->tc[0][kk] * D2->a[CPPP][kk] + s->ts[0][kk] * D2->a[SPPP][kk];
                if (s->g.ky[kk] > 0) l = l + s->tc[2][kk] * D2->a[CPMP][kk] + s->ts[2][kk] * D2->a[SPMP][kk];
                if (s->g.kz[kk] > 0) l = l + s->tc[1][kk] * D2->a[CPPM][kk] + s->ts[1][kk] * D2->a[SPPM][kk];
                if (s->g.ky[kk] > 0 && s->g.kz[kk] > 0) l = l + s->tc[3][kk] * D2->a[CPMM][kk] + s->ts[3][kk] * D2->a[SPMM][kk];
                total = total + l * bl[kk];
            }
        }
    }
    return total;
}

/* ------------------------------------------------------------------ */
/* ForceKSpace.f90                                                      */
/* ------------------------------------------------------------------ */
/* one k term of the force sum: A per combo with the y/z sign flips (ForceKSpace.f90:117-156) */
static void force_k_accum(const sck_t *C, const sck_t *kr, const grid_t *g, const double *beta,
                          double *fxt, double *fyt, double *fzt) {
    for (int kk = 0; kk < g->nk; kk++) {
        double A = C->a[CPPP][kk] * kr->a[SPPP][kk] - C->a[SPPP][kk] * kr->a[CPPP][kk];
        double fx = A, fy = A, fz = A;
        if (g->ky[kk] > 0) {
            A = C->a[CPMP][kk] * kr->a[SPMP][kk] - C->a[SPMP][kk] * kr->a[CPMP][kk];
            fx = fx + A; fy = fy - A; fz = fz + A;
        }
        if (g->kz[kk] > 0) {
            A = C->a[CPPM][kk] * kr->a[SPPM][kk] - C->a[SPPM][kk] * kr->a[CPPM][kk];
            fx = fx + A; fy = fy + A; fz = fz - A;
        }
        if (g->ky[kk] > 0 && g->kz[kk] > 0) {
            A = C->a[CPMM][kk] * kr->a[SPMM][kk] - C->a[SPMM][kk] * kr->a[CPMM][kk];
            fx = fx + A; fy = fy - A; fz = fz - A;
        }
        fx = fx * g->kx[kk] * beta[kk];
        fy = fy * g->ky[kk] * beta[kk];
        fz = fz * g->kz[kk] * beta[kk];
        *fxt = *fxt + fx; *fyt = *fyt + fy; *fzt = *fzt + fz;
    }
}

/* ForceKSpace_coulomb (ForceKSpace.f90:59-167) */
static void force_k_coulomb(orc_state *s, const sck_t *C, const sck_t *kr, double f[3]) {
    double fx = 0, fy = 0, fz = 0;
    force_k_accum(C, kr, &s->g, s->beta, &fx, &fy, &fz);
    f[0] = FOUR_PI * fx; f[1] = FOUR_PI * fy; f[2] = FOUR_PI * fz;
}

/* ForceKSpace_LJ (ForceKSpace.f90:171-302) */
static void force_k_lj(orc_state *s, const rho_t *R, int ityp, const sck_t *kr, double f[3]) {
    int nt = s->lj.ntype;
    double fx = 0, fy = 0, fz = 0;
    for (int typ = 1; typ <= nt; typ++)
        force_k_accum(&R->lj[typ - 1], kr, &s->g, s->beta_lj[(ityp - 1) * nt + typ - 1], &fx, &fy, &fz);
    f[0] = FOUR_PI * fx; f[1] = FOUR_PI * fy; f[2] = FOUR_PI * fz;
}

/* ------------------------------------------------------------------ */
/* EwaldSumRealSpace.f90 + RealSumLocal.f90                             */
/* ------------------------------------------------------------------ */
typedef struct { double r, r2, a, a2, a6, e2, erfc_a, C6, C12, so6, potew, potlj6, potlj12, pot, FR; } rsl_t;

/* RealSumLocal_init/calc_electrostatics (RealSumLocal.f90:63-108) */
static void rsl_elec(rsl_t *L, const orc_params *p, double r2, int same, double qi, double qj) {
    L->r = sqrt(r2); L->r2 = r2; L->a = p->alpha * L->r; L->a2 = L->a * L->a; L->e2 = exp(-L->a2);
    L->erfc_a = same ? -erf_luc3(L->a, L->a2, L->e2) : erfc_luc3(L->a, L->a2, L->e2);
    L->potew = p->xclb * qi * qj * L->erfc_a / L->r;
    L->pot = L->potew;
    L->FR = p->xclb * qi * qj * (L->erfc_a / L->r + p->two_alpha_over_sqrt_pi * L->e2) / L->r2;
}

/* RealSumLocal_init_LJ / calc_LJ (RealSumLocal.f90:110-168) */
static void rsl_lj(rsl_t *L, double sigma6, double four_eps) {
    double a2 = L->a2;
    double r6 = L->r2 * L->r2 * L->r2;
    L->so6 = sigma6 / r6;
    L->C6 = 1.0 + a2 * (1.0 + a2 / 2.0);
    L->a6 = a2 * a2 * a2;
    L->C12 = L->C6 + L->a6 * (1.0 + a2 * (1.0 + a2 / 5.0) / 4.0) / 6.0;
    L->potlj6 = four_eps * L->so6 * L->e2 * L->C6;
    L->potlj12 = four_eps * (L->so6 * L->so6) * L->e2 * L->C12;
    L->pot = L->pot + L->potlj12 - L->potlj6;
    L->FR = L->FR + four_eps * 6.0 * L->so6 * L->e2 *
                        (2.0 * L->so6 * (L->C12 + L->a6 * L->a6 / 720.0) - (L->C6 + L->a6 / 6.0)) / L->r2;
}

/* EwaldSumRealSpace_calc (EwaldSumRealSpace.f90:233-500).
   full != 0: full sum (i over all atoms, j0 = i+1, uu_back == uu).
   otherwise: partial sum of molecule atoms [first,last] placed at (xn,yn,zn).
   Returns the overlap flag (early return like the reference). */
/* EwaldSumRealSpace_calc (EwaldSumRealSpace.f90:233-500); the partial form runs j over
   [jlo, jhi) only (the optional first/last of the reference's call, used by mc_xchange for the
   1-2 cross sum) */
static int realspace_calc_j(orc_state *s, int full, partial_t *ps, const double *xn, const double *yn,
                            const double *zn, int first, int last, int jlo, int jhi);
static int realspace_calc(orc_state *s, int full, partial_t *ps, const double *xn, const double *yn,
                          const double *zn, int first, int last) {
    return realspace_calc_j(s, full, ps, xn, yn, zn, first, last, 0, s->N);
}
static int realspace_calc_j(orc_state *s, int full, partial_t *ps, const double *xn, const double *yn,
                            const double *zn, int first, int last, int jlo, int jhi) {
    const orc_params *p = &s->p;
    int ntot = s->N, nt = s->lj.ntype;
    int natom = full ? ntot : (last - first + 1);
    double *uu, *uub, *fx, *fxb, *fy, *fyb, *fz, *fzb;
    double *e_ew, *e_lj6, *e_lj12, *e_ewi, *e_lj6i, *e_lj12i;
    if (full) {
        uu = uub = s->uu; fx = fxb = s->fx; fy = fyb = s->fy; fz = fzb = s->fz;
        e_ew = &s->uu_ew; e_lj6 = &s->uu_lj6; e_lj12 = &s->uu_lj12;
        e_ewi = &s->uu_ew_intra; e_lj6i = &s->uu_lj6_intra; e_lj12i = &s->uu_lj12_intra;
        memset(uu, 0, sizeof(double) * ntot); memset(fx, 0, sizeof(double) * ntot);
        memset(fy, 0, sizeof(double) * ntot); memset(fz, 0, sizeof(double) * ntot);
    } else {
        uu = ps->uu; fx = ps->fx; fy = ps->fy; fz = ps->fz;
        uub = ps->uu_back; fxb = ps->fx_back; fyb = ps->fy_back; fzb = ps->fz_back;
        e_ew = &ps->uu_ew; e_lj6 = &ps->uu_lj6; e_lj12 = &ps->uu_lj12;
        e_ewi = &ps->uu_ew_intra; e_lj6i = &ps->uu_lj6_intra; e_lj12i = &ps->uu_lj12_intra;
        memset(uu, 0, sizeof(double) * MAX_MOL_ATOMS); memset(fx, 0, sizeof(double) * MAX_MOL_ATOMS);
        memset(fy, 0, sizeof(double) * MAX_MOL_ATOMS); memset(fz, 0, sizeof(double) * MAX_MOL_ATOMS);
        memset(uub, 0, sizeof(double) * ntot); memset(fxb, 0, sizeof(double) * ntot);
        memset(fyb, 0, sizeof(double) * ntot); memset(fzb, 0, sizeof(double) * ntot);
    }
    *e_ew = *e_lj6 = *e_lj12 = *e_ewi = *e_lj6i = *e_lj12i = 0;
    for (int i = 0; i < natom; i++) {
        int j0 = full ? i + 1 : jlo;
        int ii = full ? i : i + first;
        int imol = s->molnum[ii], ityp = s->lj.type_by_index[ii];
        double qi = s->charge[ii];
        double dhs_i = s->hard_core[ii] / p->BoxLength;
        int base = ityp > 0 ? (ityp - 1) * nt : -1000;
        double xi = full ? s->xx[i] : xn[i], yi = full ? s->yy[i] : yn[i], zi = full ? s->zz[i] : zn[i];
        for (int j = j0; j < (full ? ntot : jhi); j++) {
            int jmol = s->molnum[j], jtyp = s->lj.type_by_index[j];
            if (!full && imol == jmol) continue;
            double qj = s->charge[j];
            double dhs_j = s->hard_core[j] / p->BoxLength;
            double d12 = (dhs_i + dhs_j) / 2;
            int off = 0;
            if (ityp > 0 && jtyp > 0) off = base + jtyp - 1;
            double xij = xi - s->xx[j], yij = yi - s->yy[j], zij = zi - s->zz[j];
            if (xij > 0.5) xij = xij - 1.0;
            if (xij < -0.5) xij = xij + 1.0;
            if (yij > 0.5) yij = yij - 1.0;
            if (yij < -0.5) yij = yij + 1.0;
            if (zij > 0.5) zij = zij - 1.0;
            if (zij < -0.5) zij = zij + 1.0;
            double r2 = xij * xij + yij * yij + zij * zij;
            if (ityp > 0 && jtyp > 0 && imol != jmol && r2 < d12 * d12) return 1; /* overlap */
            if (r2 >= p->rmax2) continue;
            rsl_t L;
            rsl_elec(&L, p, r2, imol == jmol, qi, qj);
            *e_ew = *e_ew + L.potew;
            if (imol == jmol) *e_ewi = *e_ewi + L.potew;
            if (ityp != 0 && jtyp != 0) {
                rsl_lj(&L, s->lj.sigma6[off], s->lj.four_eps[off]);
                *e_lj6 = *e_lj6 + L.potlj6;
                *e_lj12 = *e_lj12 + L.potlj12;
                if (imol == jmol) { *e_lj6i = *e_lj6i + L.potlj6; *e_lj12i = *e_lj12i + L.potlj12; }
            }
            if (imol != jmol) {
                uu[i] = uu[i] + L.pot;
                uub[j] = uub[j] + L.pot;
                double fxij = xij * L.FR;
                fx[i] = fx[i] + fxij; fxb[j] = fxb[j] - fxij;
                double fyij = yij * L.FR;
                fy[i] = fy[i] + fyij; fyb[j] = fyb[j] - fyij;
                double fzij = zij * L.FR;
                fz[i] = fz[i] + fzij; fzb[j] = fzb[j] - fzij;
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* EwaldSumExternal.f90 / EwaldSumTails.f90 / mc_total_energy          */
/* ------------------------------------------------------------------ */
/* EwaldSumExternal_calc_mu (EwaldSumExternal.f90:34-52) */
static void calc_mu(const double *x, const double *y, const double *z, const double *q, int n,
                    double *mx, double *my, double *mz) {
    double a = 0, b = 0, c = 0;
    for (int i = 0; i < n; i++) { a = a + q[i] * x[i]; b = b + q[i] * y[i]; c = c + q[i] * z[i]; }
    *mx = a; *my = b; *mz = c;
}

/* ewald_sum_coulomb_tail / ewald_sum_lj_tails (EwaldSumTails.f90:18-127) */
static void tails(orc_state *s) {
    double S = 0;
    for (int i = 0; i < s->N; i++) S = S + s->charge[i] * s->charge[i];
    s->U_tail_coul = -(s->p.xclb * s->p.alpha_over_sqrt_pi * S);
    double alpha = s->p.alpha;
    double a3 = ipow(alpha, 3), a6 = a3 * a3, a9 = a3 * a6, a12 = a6 * a6;
    double pisp = pow(PI, 1.5);
    int nt = s->lj.ntype;
    double sij6 = 0, sij12 = 0, sj6 = 0, sj12 = 0;
    /* mol_numbers indexed by LJ type: the reference's quirk (EwaldSumTails.f90:88) */
    for (int t1 = 1; t1 <= nt; t1++)
        for (int t2 = t1; t2 <= nt; t2++) {
            int o = (t1 - 1) * nt + t2 - 1;
            int n1n2 = s->mol_numbers[t1 - 1] * s->mol_numbers[t2 - 1];
            double l6 = s->lj.lj6[o] * n1n2, l12 = s->lj.lj12[o] * n1n2;
            if (t1 != t2) { l6 = l6 + l6; l12 = l12 + l12; }
            sij6 = sij6 + l6; sij12 = sij12 + l12;
        }
    for (int t = 1; t <= nt; t++) {
        int o = (t - 1) * nt + t - 1;
        sj6 = sj6 + s->lj.lj6[o] * s->mol_numbers[t - 1];
        sj12 = sj12 + s->lj.lj12[o] * s->mol_numbers[t - 1];
    }
    s->U_tail_lj6 = pisp * a3 / 6.0 * sij6 - a6 / 12.0 * sj6;
    s->U_tail_lj12 = pisp * a9 / 1080.0 * sij12 - a12 / 1440.0 * sj12;
    s->U_tail = s->U_tail_coul + s->U_tail_lj12 - s->U_tail_lj6;
}

/* mc_total_energy (MC.f90:681-698) */
static double total_energy(orc_state *s) {
    s->U_tail = s->U_tail_coul + s->U_tail_lj12 - s->U_tail_lj6;
    s->U_ext = s->p.kext * (s->mu_x * s->mu_x + s->mu_y * s->mu_y + s->mu_z * s->mu_z);
    s->U_total_ew = s->uu_ew + s->E_k_coul + s->U_tail_coul + s->U_ext;
    s->U_total_lj = s->uu_lj12 - s->uu_lj6 + s->E_k_lj + s->U_tail_lj12 - s->U_tail_lj6;
    s->U_total = s->U_total_ew + s->U_total_lj;
    return s->U_total;
}

void orc_energies(orc_state *s, double e[8]) {
    e[0] = total_energy(s); e[1] = s->U_total_ew; e[2] = s->U_total_lj;
    e[3] = s->uu_ew; e[4] = s->uu_lj6; e[5] = s->uu_lj12; e[6] = s->E_k_coul; e[7] = s->E_k_lj;
}

/* mc_calc_total_sums (MC.f90:477-585) */
int32_t orc_full_sums(orc_state *s, double e[8]) {
    int ov = realspace_calc(s, 1, NULL, NULL, NULL, NULL, 0, 0);
    init_beta(s);
    init_beta_lj(s);
    kspace_total_energy(s);
    calc_mu(s->xx, s->yy, s->zz, s->charge, s->N, &s->mu_x, &s->mu_y, &s->mu_z);
    tails(s);
    total_energy(s);
    if (e) orc_energies(s, e);
    return ov ? 1 : 0;
}

/* ------------------------------------------------------------------ */
/* geometry.f90                                                         */
/* ------------------------------------------------------------------ */
/* rot_vect (geometry.f90:28-63) */
static void rot_vect(double x, double y, double z, double *x1, double *y1, double *z1, double cc, double ss, int i) {
    if (i == 1) { double y2 = y; *x1 = x; *y1 = cc * y2 - ss * z; *z1 = ss * y2 + cc * z; }
    if (i == 2) { double x2 = x; *y1 = y; *x1 = cc * x2 + ss * z; *z1 = -ss * x2 + cc * z; }
    if (i == 3) { double x2 = x; *z1 = z; *x1 = cc * x2 - ss * y; *y1 = ss * x2 + cc * y; }
}
/* prod_vect (geometry.f90:65-101) */
static void prod_vect(double x1, double y1, double z1, double x2, double y2, double z2, double *xp, double *yp, double *zp) {
    *xp = y1 * z2 - z1 * y2; *yp = z1 * x2 - x1 * z2; *zp = x1 * y2 - y1 * x2;
}
/* center_of_mass (geometry.f90:170-201) */
static void center_of_mass(const double *x, const double *y, const double *z, const double *m, int n,
                           double *xc, double *yc, double *zc) {
    double sx = 0, sy = 0, sz = 0, tm = 0;
    for (int i = 0; i < n; i++) { sx = sx + m[i] * x[i]; sy = sy + m[i] * y[i]; sz = sz + m[i] * z[i]; tm = tm + m[i]; }
    *xc = sx / tm; *yc = sy / tm; *zc = sz / tm;
}

typedef struct { double cphi, sphi, ct, st, ca, sa; } rot_t;
typedef struct { double xx, xy, xz, yx, yy, yz, zx, zy, zz; } rotm_t;

/* fill_rot_matrix (geometry.f90:103-138) */
static void fill_rot_matrix(const rot_t *r, rotm_t *m) {
    double cphi = r->cphi, sphi = r->sphi, st = r->st, ct = r->ct, ca = r->ca, sa = r->sa, ca1 = 1 - ca;
    m->xx = (cphi * cphi * (st * st) * ca1 + ca);
    m->xy = (sphi * cphi * (st * st) * ca1 - ct * sa);
    m->xz = st * (ct * ca1 * cphi + sa * sphi);
    m->yx = (cphi * sphi * (st * st) * ca1 + ct * sa);
    m->yy = (sphi * sphi * (st * st) * ca1 + ca);
    m->yz = st * (ct * ca1 * sphi - sa * cphi);
    m->zx = st * (ct * ca1 * cphi - sa * sphi);
    m->zy = st * (ct * ca1 * sphi + sa * cphi);
    m->zz = (st * st * ca + ct * ct);
}

/* ------------------------------------------------------------------ */
/* MonteCarloMove.f90                                                   */
/* ------------------------------------------------------------------ */
typedef struct {
    double fxo, fyo, fzo, fo, cxo, cyo, czo, co, umaxold, vmaxold, cold, qold;
    double vx, vy, vz, deltx, delty, deltz, angle;
    double fxn, fyn, fzn, fn, cxn, cyn, czn, cn, umaxnew, vmaxnew, cnew, qnew;
} mcmove_t;

/* MonteCarloMove_init_old (MonteCarloMove.f90:34-54) */
static void mcm_init_old(mcmove_t *m, double fx, double fy, double fz, double tx, double ty, double tz) {
    m->fxo = fx; m->fyo = fy; m->fzo = fz; m->fo = sqrt(fx * fx + fy * fy + fz * fz);
    m->cxo = tx; m->cyo = ty; m->czo = tz; m->co = sqrt(tx * tx + ty * ty + tz * tz);
}

/* MonteCarloMove_init_new (MonteCarloMove.f90:56-106) */
static void mcm_init_new(mcmove_t *m, const orc_params *p, double fx, double fy, double fz, double tx, double ty, double tz) {
    m->fxn = fx; m->fyn = fy; m->fzn = fz; m->fn = sqrt(fx * fx + fy * fy + fz * fz);
    m->cxn = tx; m->cyn = ty; m->czn = tz; m->cn = sqrt(tx * tx + ty * ty + tz * tz);
    double umaxnew = p->xlambda_f * m->fn * p->dr, cnew;
    if (umaxnew > 1e-2) {
        double e = exp(-2.0 * umaxnew);
        double t = (umaxnew * (1.0 + e) - (1.0 - e)) / 2.0;
        cnew = 3.0 * t / (umaxnew * umaxnew * umaxnew);
    } else { umaxnew = 0.0; cnew = 1.0; }
    m->umaxnew = umaxnew; m->cnew = cnew;
    double vmaxnew = p->xlambda_c * m->cn * p->d_angle, qnew;
    if (vmaxnew > 1e-2) qnew = orc_shi_sans_exp(vmaxnew) / vmaxnew;
    else { vmaxnew = 0.0; qnew = 1.0; }
    m->vmaxnew = vmaxnew; m->qnew = qnew;
}

/* MonteCarloMove_chooseDisplacement (MonteCarloMove.f90:109-266) */
static void mcm_choose_displacement(orc_state *s, mcmove_t *m, double *dx_, double *dy_, double *dz_) {
    const orc_params *p = &s->p;
    double fxo = m->fxo, fyo = m->fyo, fzo = m->fzo, fo = m->fo;
    double umax = p->xlambda_f * fo * p->dr, cold, deltx, delty, deltz;
    if (umax > 1e-2) {
        double e = exp(-2.0 * umax);
        double t = (umax * (1.0 + e) - (1.0 - e)) / 2.0;
        cold = 3.0 * t / (umax * umax * umax);
        double xksi = 0.0;
        while (xksi < 1e-10) xksi = orc_rand(s);
        double z = umax + log(xksi * t), u;
        if (z <= log(4.0)) { double ss = exp(z); u = pow(3.0 * ss, 1.0 / 3.0) - ss / 10.0; }
        else u = z - log(z / 2.0);
        double h = 0, h1, g, sh, ch;
        for (int k = 1; k <= 10; k++) {
            e = exp(-2.0 * u);
            ch = (1.0 + e) / 2.0;
            sh = (1.0 - e) / 2.0;
            if (u < 1e-5) sh = u - u * u;
            g = u * ch - sh;
            if (u < 1e-3) g = u * u * u / 3.0;
            h = u + log(g);
            h1 = u * sh / g;
            if (k < 10) u = u + (z - h) / h1;
        }
        double deltar = u / (p->xlambda_f * fo);
        xksi = 1.0;
        while (xksi > (1.0 - 1e-10) || xksi < 1e-10) xksi = orc_rand(s);
        double xc = 1.0 + log(xksi + (1.0 - xksi) * e) / u;
        if (u < 1e-7) xc = 1.0 - 2.0 * (1.0 - xksi);
        if (xc > 1.0 - 1e-14) xc = 1.0 - 1e-14;
        if (xc < -1.0 + 1e-14) xc = -1.0 + 1e-14;
        double xs = sqrt(1.0 - xc * xc);
        double w = -1.0, wx = 0, wy = 0, wz = 0;
        while (w <= 1e-10) {
            double v2 = 2.0, vx = 0, vy = 0, vz = 0;
            while (v2 > 1.0) {
                vx = 2.0 * orc_rand(s) - 1.0; vy = 2.0 * orc_rand(s) - 1.0; vz = 2.0 * orc_rand(s) - 1.0;
                v2 = vx * vx + vy * vy + vz * vz;
                if (s->rng_out) break;
            }
            prod_vect(vx, vy, vz, fxo, fyo, fzo, &wx, &wy, &wz);
            w = sqrt(wx * wx + wy * wy + wz * wz);
            if (s->rng_out) break;
        }
        deltx = deltar * (xc * fxo / fo + xs * wx / w);
        delty = deltar * (xc * fyo / fo + xs * wy / w);
        deltz = deltar * (xc * fzo / fo + xs * wz / w);
    } else {
        double v2 = 2.0, vx = 0, vy = 0, vz = 0;
        while (v2 > 1.0) {
            vx = 2.0 * orc_rand(s) - 1.0; vy = 2.0 * orc_rand(s) - 1.0; vz = 2.0 * orc_rand(s) - 1.0;
            v2 = vx * vx + vy * vy + vz * vz;
            if (s->rng_out) break;
        }
        deltx = p->dr * vx; delty = p->dr * vy; deltz = p->dr * vz;
        umax = 0.0; cold = 1.0;
    }
    m->deltx = deltx; m->delty = delty; m->deltz = deltz;
    m->cold = cold; m->umaxold = umax;
    *dx_ = deltx; *dy_ = delty; *dz_ = deltz;
}

/* MonteCarloMove_chooseRotation (MonteCarloMove.f90:269-444) */
static void mcm_choose_rotation(orc_state *s, mcmove_t *m, rot_t *rot) {
    const orc_params *p = &s->p;
    double cxo = m->cxo, cyo = m->cyo, czo = m->czo, co = m->co;
    double vmax = p->xlambda_c * co * p->d_angle, vx, vy, vz, angle, qold;
    if (vmax > 1e-2) {
        double emax = exp(-2.0 * vmax);
        double shmax = (1.0 - emax) / 2.0;
        double xksi = 1.0, proba = 0.0, v = 0, e = 0;
        while (xksi >= proba) {
            v = 0.0;
            while (fabs(v) < 1e-10) {
                xksi = orc_rand(s);
                double xs = xksi * shmax;
                v = vmax + log(xs + sqrt(xs * xs + emax));
                if (xs * xs < 1e-14 * emax) v = xs / sqrt(emax);
                if (s->rng_out) break;
            }
            e = exp(-2.0 * v);
            proba = (1.0 - e) / v / (1.0 + e);
            if (v < 1e-5) proba = (2.0 * v - 2.0 * v * v) / v / (1.0 + e);
            xksi = orc_rand(s);
            if (s->rng_out) break;
        }
        double cosx = v / vmax;
        qold = orc_shi_sans_exp(vmax) / vmax;
        xksi = 1.0;
        while (xksi > (1.0 - 1e-10)) { xksi = orc_rand(s); if (s->rng_out) break; }
        angle = p->d_angle * (1.0 + log(xksi + (1.0 - xksi) * e) / v);
        if (v < 1e-7) angle = p->d_angle * (1.0 - 2.0 * (1.0 - xksi));
        double w = -1.0, wx = 0, wy = 0, wz = 0;
        vx = vy = vz = 0;
        while (w <= 1e-10) {
            double v2 = 2.0;
            while (v2 > 1.0 || v2 < 1e-10) {
                vx = 2.0 * orc_rand(s) - 1.0; vy = 2.0 * orc_rand(s) - 1.0; vz = 2.0 * orc_rand(s) - 1.0;
                v2 = vx * vx + vy * vy + vz * vz;
                if (s->rng_out) break;
            }
            prod_vect(vx, vy, vz, cxo, cyo, czo, &wx, &wy, &wz);
            w = sqrt(wx * wx + wy * wy + wz * wz);
            if (s->rng_out) break;
        }
        double sinx = sqrt(1.0 - cosx * cosx);
        vx = cxo / co * cosx + wx / w * sinx;
        vy = cyo / co * cosx + wy / w * sinx;
        vz = czo / co * cosx + wz / w * sinx;
    } else {
        double v2 = 2.0;
        vx = vy = vz = 0;
        while (v2 > 1.0 || v2 < 1e-10) {
            vx = 2.0 * orc_rand(s) - 1.0; vy = 2.0 * orc_rand(s) - 1.0; vz = 2.0 * orc_rand(s) - 1.0;
            v2 = vx * vx + vy * vy + vz * vz;
            if (s->rng_out) break;
        }
        double v = sqrt(v2);
        vx = vx / v; vy = vy / v; vz = vz / v;
        angle = p->d_angle * (2.0 * orc_rand(s) - 1.0);
        vmax = 0.0; qold = 1.0;
    }
    double ca = cos(angle), sa = sin(angle);
    double ct = vz, st = sqrt(1.0 - ct * ct), cphi = 0.0, sphi = 0.0;
    if (st > 0.0) { cphi = vx / st; sphi = vy / st; }
    rot->cphi = cphi; rot->sphi = sphi; rot->ct = ct; rot->st = st; rot->ca = ca; rot->sa = sa;
    m->vx = vx; m->vy = vy; m->vz = vz; m->vmaxold = vmax; m->angle = angle; m->qold = qold;
}

/* MonteCarloMove_accept_or_decline (MonteCarloMove.f90:447-570) */
static int mcm_accept(orc_state *s, const mcmove_t *m, double dutot) {
    const orc_params *p = &s->p;
    double exposu = -dutot;
    double exposf = -p->xlambda_f * ((m->fxo + m->fxn) * m->deltx + (m->fyo + m->fyn) * m->delty + (m->fzo + m->fzn) * m->deltz);
    double exposfcorr = m->umaxold - m->umaxnew;
    double exposc = -p->xlambda_c * m->angle * ((m->cxo + m->cxn) * m->vx + (m->cyo + m->cyn) * m->vy + (m->czo + m->czn) * m->vz);
    double exposccorr = m->vmaxold - m->vmaxnew;
    double factor = m->cold * m->qold / (m->cnew * m->qnew) * exp(exposu + exposf + exposfcorr + exposc + exposccorr);
    double xksi = orc_rand(s);
    if (xksi > factor) return 0;
    return 1;
}

/* ------------------------------------------------------------------ */
/* movemc (MC.f90:831-1322), split into the stages the per-move C ABI    */
/* exposes: old (Steps 0-4), eval (Steps 6-12), accept + commit (13-14)  */
/* ------------------------------------------------------------------ */
typedef struct {
    int im, first, last, natom;
    const double *mass;
    double fxo[MAX_MOL_ATOMS], fyo[MAX_MOL_ATOMS], fzo[MAX_MOL_ATOMS];
    double fxn[MAX_MOL_ATOMS], fyn[MAX_MOL_ATOMS], fzn[MAX_MOL_ATOMS];
    double xn[MAX_MOL_ATOMS], yn[MAX_MOL_ATOMS], zn[MAX_MOL_ATOMS];
    double E_old, mo_x, mo_y, mo_z, xc, yc, zc;
    double Fo[3], To[3], Fn[3], Tn[3];
    double dU_real, du_kc, du_kl, dU_ext, mux_new, muy_new, muz_new;
    int overlap;
} mvctx_t;

/* Steps 0-4 */
static void movemc_old(orc_state *s, int imol1, mvctx_t *c) {
    const orc_params *p = &s->p;
    int nk = s->g.nk, nt = s->lj.ntype;
    double fk[3], fl[3];
    c->im = imol1 - 1;
    c->first = s->first_atom[c->im]; c->last = s->last_atom[c->im];
    c->natom = c->last - c->first + 1;
    c->mass = s->moltypes[s->mol_type[c->im]].mass;
    int first = c->first, natom = c->natom;
    double *xo = s->xx + first, *yo = s->yy + first, *zo = s->zz + first;
    /* FOR TEST ONLY (MC.f90:915-916): mu recomputed from all atoms every move */
    calc_mu(s->xx, s->yy, s->zz, s->charge, s->N, &s->mu_x, &s->mu_y, &s->mu_z);
    /* Step 2 (:934-939) */
    double E_old = 0;
    for (int i = first; i <= c->last; i++) E_old = E_old + s->uu[i];
    c->E_old = E_old;
    for (int i = 0; i < natom; i++) { c->fxo[i] = s->fx[first + i]; c->fyo[i] = s->fy[first + i]; c->fzo[i] = s->fz[first + i]; }
    /* Step 3 (:946-982): old structure factors and k-space forces against the current total rho */
    rho_zero(&s->mol_old, nk, nt);
    for (int i = 0; i < natom; i++) {
        int ii = first + i, ityp = s->lj.type_by_index[ii];
        rho_add_atom(s, &s->mol_old, s->xx[ii], s->yy[ii], s->zz[ii], s->charge[ii], ityp, &s->skr_coul[i], &s->skr_lj[i]);
        force_k_coulomb(s, &s->rho_total.coul, &s->skr_coul[i], fk);
        if (ityp > 0) force_k_lj(s, &s->rho_total, ityp, &s->skr_lj[i], fl);
        else fl[0] = fl[1] = fl[2] = 0;
        c->fxo[i] = c->fxo[i] + fk[0] + fl[0];
        c->fyo[i] = c->fyo[i] + fk[1] + fl[1];
        c->fzo[i] = c->fzo[i] + fk[2] + fl[2];
    }
    /* Step 3A (:988-997): external-field forces, molecule dipole (old) */
    for (int i = 0; i < natom; i++) {
        double q = s->charge[first + i];
        c->fxo[i] = c->fxo[i] + p->minus_two_kext * q * s->mu_x;
        c->fyo[i] = c->fyo[i] + p->minus_two_kext * q * s->mu_y;
        c->fzo[i] = c->fzo[i] + p->minus_two_kext * q * s->mu_z;
    }
    calc_mu(xo, yo, zo, s->charge + first, natom, &c->mo_x, &c->mo_y, &c->mo_z);
    /* Step 4 (:1002-1025) */
    double Fx = 0, Fy = 0, Fz = 0;
    for (int i = 0; i < natom; i++) { Fx = Fx + c->fxo[i]; Fy = Fy + c->fyo[i]; Fz = Fz + c->fzo[i]; }
    center_of_mass(xo, yo, zo, c->mass, natom, &c->xc, &c->yc, &c->zc);
    double Tx = 0, Ty = 0, Tz = 0;
    for (int i = 0; i < natom; i++) {
        double tx, ty, tz;
        prod_vect(xo[i] - c->xc, yo[i] - c->yc, zo[i] - c->zc, c->fxo[i], c->fyo[i], c->fzo[i], &tx, &ty, &tz);
        Tx = Tx + tx; Ty = Ty + ty; Tz = Tz + tz;
    }
    c->Fo[0] = Fx; c->Fo[1] = Fy; c->Fo[2] = Fz; c->To[0] = Tx; c->To[1] = Ty; c->To[2] = Tz;
}

/* Steps 6-12 for new positions c->xn/yn/zn; returns the overlap flag */
static int movemc_eval(orc_state *s, mvctx_t *c) {
    const orc_params *p = &s->p;
    int nk = s->g.nk, nt = s->lj.ntype;
    int first = c->first, natom = c->natom;
    double fk[3], fl[3];
    /* Step 6 (:1077-1084) */
    c->overlap = realspace_calc(s, 0, &s->ps_new, c->xn, c->yn, c->zn, first, c->last);
    if (c->overlap) return 1;
    double E_new = 0;
    for (int i = 0; i < natom; i++) E_new = E_new + s->ps_new.uu[i];
    c->dU_real = E_new - c->E_old;  /* Step 7 */
    /* Step 8 (:1096-1112) */
    rho_zero(&s->mol_new, nk, nt);
    for (int i = 0; i < natom; i++) {
        int ii = first + i;
        rho_add_atom(s, &s->mol_new, c->xn[i], c->yn[i], c->zn[i], s->charge[ii], s->lj.type_by_index[ii], &s->skr_coul[i], &s->skr_lj[i]);
    }
    /* Step 9: delta = new - old */
    rho_sub(&s->mol_new, &s->mol_old, nk, nt);
    /* Step 9A (:1136-1163): forces with total_new = total + delta */
    rho_copy(&s->total_new, &s->rho_total, nk, nt);
    rho_add(&s->total_new, &s->mol_new, nk, nt);
    for (int i = 0; i < natom; i++) {
        int ii = first + i, ityp = s->lj.type_by_index[ii];
        force_k_coulomb(s, &s->total_new.coul, &s->skr_coul[i], fk);
        if (ityp > 0) force_k_lj(s, &s->total_new, ityp, &s->skr_lj[i], fl);
        else fl[0] = fl[1] = fl[2] = 0;
        c->fxn[i] = s->ps_new.fx[i] + fk[0] + fl[0];
        c->fyn[i] = s->ps_new.fy[i] + fk[1] + fl[1];
        c->fzn[i] = s->ps_new.fz[i] + fk[2] + fl[2];
    }
    /* Steps 10-11 */
    c->du_kc = kspace_du_coulomb(s, &s->mol_new.coul);
    c->du_kl = kspace_du_lj(s, &s->mol_new);
    /* Step 11A */
    double mn_x, mn_y, mn_z;
    calc_mu(c->xn, c->yn, c->zn, s->charge + first, natom, &mn_x, &mn_y, &mn_z);
    double dmx = mn_x - c->mo_x, dmy = mn_y - c->mo_y, dmz = mn_z - c->mo_z;
    c->dU_ext = p->kext * ((2 * s->mu_x + dmx) * dmx + (2 * s->mu_y + dmy) * dmy + (2 * s->mu_z + dmz) * dmz);
    /* Step 11B */
    c->mux_new = s->mu_x + dmx; c->muy_new = s->mu_y + dmy; c->muz_new = s->mu_z + dmz;
    for (int i = 0; i < natom; i++) {
        double q = s->charge[first + i];
        c->fxn[i] = c->fxn[i] + p->minus_two_kext * q * c->mux_new;
        c->fyn[i] = c->fyn[i] + p->minus_two_kext * q * c->muy_new;
        c->fzn[i] = c->fzn[i] + p->minus_two_kext * q * c->muz_new;
    }
    /* Step 12 */
    double Fx = 0, Fy = 0, Fz = 0, xc, yc, zc;
    for (int i = 0; i < natom; i++) { Fx = Fx + c->fxn[i]; Fy = Fy + c->fyn[i]; Fz = Fz + c->fzn[i]; }
    center_of_mass(c->xn, c->yn, c->zn, c->mass, natom, &xc, &yc, &zc);
    double Tx = 0, Ty = 0, Tz = 0;
    for (int i = 0; i < natom; i++) {
        double tx, ty, tz;
        prod_vect(c->xn[i] - xc, c->yn[i] - yc, c->zn[i] - zc, c->fxn[i], c->fyn[i], c->fzn[i], &tx, &ty, &tz);
        Tx = Tx + tx; Ty = Ty + ty; Tz = Tz + tz;
    }
    c->Fn[0] = Fx; c->Fn[1] = Fy; c->Fn[2] = Fz; c->Tn[0] = Tx; c->Tn[1] = Ty; c->Tn[2] = Tz;
    return 0;
}

/* Step 14 (:1242-1320) */
static void movemc_commit(orc_state *s, mvctx_t *c) {
    int nk = s->g.nk, nt = s->lj.ntype, first = c->first, natom = c->natom;
    double *xo = s->xx + first, *yo = s->yy + first, *zo = s->zz + first;
    rho_add(&s->rho_total, &s->mol_new, nk, nt);
    realspace_calc(s, 0, &s->ps_old, xo, yo, zo, first, c->last);
    for (int i = 0; i < s->N; i++) {
        s->uu[i] = s->uu[i] + s->ps_new.uu_back[i] - s->ps_old.uu_back[i];
        s->fx[i] = s->fx[i] + s->ps_new.fx_back[i] - s->ps_old.fx_back[i];
        s->fy[i] = s->fy[i] + s->ps_new.fy_back[i] - s->ps_old.fy_back[i];
        s->fz[i] = s->fz[i] + s->ps_new.fz_back[i] - s->ps_old.fz_back[i];
    }
    for (int i = 0; i < natom; i++) {
        s->uu[first + i] = s->ps_new.uu[i];
        s->fx[first + i] = s->ps_new.fx[i]; s->fy[first + i] = s->ps_new.fy[i]; s->fz[first + i] = s->ps_new.fz[i];
    }
    s->E_k_coul = s->E_k_coul + c->du_kc;
    s->E_k_lj = s->E_k_lj + c->du_kl;
    s->E_k = s->E_k_coul + s->E_k_lj;
    s->uu_ew = s->uu_ew + s->ps_new.uu_ew - s->ps_old.uu_ew;
    s->uu_lj6 = s->uu_lj6 + s->ps_new.uu_lj6 - s->ps_old.uu_lj6;
    s->uu_lj12 = s->uu_lj12 + s->ps_new.uu_lj12 - s->ps_old.uu_lj12;
    s->mu_x = c->mux_new; s->mu_y = c->muy_new; s->mu_z = c->muz_new;
    total_energy(s);
    for (int i = 0; i < natom; i++) { xo[i] = c->xn[i]; yo[i] = c->yn[i]; zo[i] = c->zn[i]; }
}

static void fill_rec(const mvctx_t *c, orc_move_rec *rec) {
    for (int k = 0; k < 3; k++) {
        rec->f_old[k] = c->Fo[k]; rec->t_old[k] = c->To[k]; rec->f_new[k] = c->Fn[k]; rec->t_new[k] = c->Tn[k];
    }
    rec->du_real = c->dU_real; rec->du_k_coul = c->du_kc; rec->du_k_lj = c->du_kl; rec->du_ext = c->dU_ext;
}

static int movemc(orc_state *s, int imol1, orc_move_rec *rec) {
    const orc_params *p = &s->p;
    mvctx_t c;
    memset(&c, 0, sizeof c);
    memset(rec, 0, sizeof(*rec));
    rec->imol = imol1;
    movemc_old(s, imol1, &c);
    int first = c.first, natom = c.natom;
    double *xo = s->xx + first, *yo = s->yy + first, *zo = s->zz + first;
    /* Step 5 (:1031-1067) */
    mcmove_t mv;
    memset(&mv, 0, sizeof mv);
    mcm_init_old(&mv, c.Fo[0], c.Fo[1], c.Fo[2], c.To[0], c.To[1], c.To[2]);
    double deltx, delty, deltz;
    mcm_choose_displacement(s, &mv, &deltx, &delty, &deltz);
    rot_t rot;
    mcm_choose_rotation(s, &mv, &rot);
    if (s->rng_out) return -6;
    double xcn = c.xc + deltx - round(c.xc + deltx);
    double ycn = c.yc + delty - round(c.yc + delty);
    double zcn = c.zc + deltz - round(c.zc + deltz);
    if (natom > 1) {
        rotm_t R;
        fill_rot_matrix(&rot, &R);
        for (int i = 0; i < natom; i++) {
            double xr0 = xo[i] - c.xc, yr0 = yo[i] - c.yc, zr0 = zo[i] - c.zc;
            double xr = R.xx * xr0 + R.xy * yr0 + R.xz * zr0;
            double yr = R.yx * xr0 + R.yy * yr0 + R.yz * zr0;
            double zr = R.zx * xr0 + R.zy * yr0 + R.zz * zr0;
            c.xn[i] = xr + xcn; c.yn[i] = yr + ycn; c.zn[i] = zr + zcn;
        }
    } else { c.xn[0] = xcn; c.yn[0] = ycn; c.zn[0] = zcn; }
    if (movemc_eval(s, &c)) { fill_rec(&c, rec); rec->flags = 2; return 0; }
    /* Step 13 */
    double du_total = c.dU_real + (c.du_kc + c.du_kl) + c.dU_ext;
    mcm_init_new(&mv, p, c.Fn[0], c.Fn[1], c.Fn[2], c.Tn[0], c.Tn[1], c.Tn[2]);
    int acc = mcm_accept(s, &mv, du_total);
    if (s->rng_out) return -6;
    fill_rec(&c, rec);
    rec->flags = acc ? 1 : 0;
    if (acc) movemc_commit(s, &c);
    return 0;
}

/* per-move entry points (the stages a host-driven movemc calls) */
static mvctx_t g_api;
int32_t orc_move_old(orc_state *s, int32_t imol, double f[3], double t[3]) {
    if (imol < 1 || imol > s->nmol) return -4;
    memset(&g_api, 0, sizeof g_api);
    movemc_old(s, imol, &g_api);
    for (int k = 0; k < 3; k++) { f[k] = g_api.Fo[k]; t[k] = g_api.To[k]; }
    return 0;
}
int32_t orc_move_eval(orc_state *s, const double *xn, const double *yn, const double *zn, double du[4],
                      int32_t *overlap, double f[3], double t[3]) {
    for (int i = 0; i < g_api.natom; i++) { g_api.xn[i] = xn[i]; g_api.yn[i] = yn[i]; g_api.zn[i] = zn[i]; }
    *overlap = movemc_eval(s, &g_api);
    du[0] = g_api.dU_real; du[1] = g_api.du_kc; du[2] = g_api.du_kl; du[3] = g_api.dU_ext;
    for (int k = 0; k < 3; k++) { f[k] = g_api.Fn[k]; t[k] = g_api.Tn[k]; }
    return 0;
}
int32_t orc_move_commit(orc_state *s) { movemc_commit(s, &g_api); return 0; }

/* BiasedRandom_choose (BiasedRandom.f90:81-109) */
static int biased_choose(orc_state *s) {
    double rnd = orc_rand(s);
    int interval = 1;
    for (int i = 0; i < s->nmol; i++)
        if (rnd > s->freq_beg[i] && rnd < s->freq_end[i]) { interval = i + 1; break; }
    return interval;
}

/* BiasedRandom_choose on xchange_freq */
static int biased_choose_x(orc_state *s) {
    double rnd = orc_rand(s);
    int interval = 1;
    for (int i = 0; i < s->nmol; i++)
        if (rnd > s->xfreq_beg[i] && rnd < s->xfreq_end[i]) { interval = i + 1; break; }
    return interval;
}

static void partial_alloc(partial_t *p, int N) {
    memset(p, 0, sizeof *p);
    p->uu_back = calloc(N, sizeof(double)); p->fx_back = calloc(N, sizeof(double));
    p->fy_back = calloc(N, sizeof(double)); p->fz_back = calloc(N, sizeof(double));
}
static void partial_free(partial_t *p) { free(p->uu_back); free(p->fx_back); free(p->fy_back); free(p->fz_back); }

/* mc_xchange (MC.f90:1325-1954): molecules imol1 and imol2 (1-based) swap their centres of mass,
   each keeping its orientation.  The real-space change is, as in the reference, the sum of the
   two molecules' per-atom energies after minus before (MC.f90:1451-1452, 1639-1642), so the 1-2
   pair energy enters the acceptance twice (the bookkeeping on acceptance takes it once,
   :1813-1826).  No acceptance draw after a hard-core overlap; otherwise
   MonteCarloMove_accept_or_decline_simple (MonteCarloMove.f90:572-597). */
static int mc_xchange(orc_state *s, int imol1, int imol2, orc_move_rec *rec) {
    const orc_params *p = &s->p;
    int nk = s->g.nk, nt = s->lj.ntype, N = s->N;
    int m1 = imol1 - 1, m2 = imol2 - 1;
    int f1 = s->first_atom[m1], l1 = s->last_atom[m1], n1 = l1 - f1 + 1;
    int f2 = s->first_atom[m2], l2 = s->last_atom[m2], n2 = l2 - f2 + 1;
    const double *mass1 = s->moltypes[s->mol_type[m1]].mass, *mass2 = s->moltypes[s->mol_type[m2]].mass;
    memset(rec, 0, sizeof *rec);
    rec->imol = imol1;
    /* FOR TEST ONLY (MC.f90:1420): mu from all atoms */
    calc_mu(s->xx, s->yy, s->zz, s->charge, N, &s->mu_x, &s->mu_y, &s->mu_z);
    /* Step 2 (:1451-1452) */
    double S1 = 0, S2 = 0;
    for (int i = f1; i <= l1; i++) S1 = S1 + s->uu[i];
    for (int i = f2; i <= l2; i++) S2 = S2 + s->uu[i];
    double E_old = S1 + S2;
    /* Step 3 (:1467-1490): old structure factors of both molecules */
    rho_zero(&s->mol_old, nk, nt);
    for (int i = f1; i <= l1; i++)
        rho_add_atom(s, &s->mol_old, s->xx[i], s->yy[i], s->zz[i], s->charge[i], s->lj.type_by_index[i], &s->skr_coul[0], &s->skr_lj[0]);
    for (int i = f2; i <= l2; i++)
        rho_add_atom(s, &s->mol_old, s->xx[i], s->yy[i], s->zz[i], s->charge[i], s->lj.type_by_index[i], &s->skr_coul[0], &s->skr_lj[0]);
    double mo1[3], mo2[3], c1[3], c2[3];
    calc_mu(s->xx + f1, s->yy + f1, s->zz + f1, s->charge + f1, n1, &mo1[0], &mo1[1], &mo1[2]);
    calc_mu(s->xx + f2, s->yy + f2, s->zz + f2, s->charge + f2, n2, &mo2[0], &mo2[1], &mo2[2]);
    center_of_mass(s->xx + f1, s->yy + f1, s->zz + f1, mass1, n1, &c1[0], &c1[1], &c1[2]);
    center_of_mass(s->xx + f2, s->yy + f2, s->zz + f2, mass2, n2, &c2[0], &c2[1], &c2[2]);
    /* the swapped positions (:1516-1524), not wrapped into the box */
    double xn1[MAX_MOL_ATOMS], yn1[MAX_MOL_ATOMS], zn1[MAX_MOL_ATOMS];
    double xn2[MAX_MOL_ATOMS], yn2[MAX_MOL_ATOMS], zn2[MAX_MOL_ATOMS];
    double xo1[MAX_MOL_ATOMS], yo1[MAX_MOL_ATOMS], zo1[MAX_MOL_ATOMS];
    double xo2[MAX_MOL_ATOMS], yo2[MAX_MOL_ATOMS], zo2[MAX_MOL_ATOMS];
    for (int i = 0; i < n1; i++) {
        xo1[i] = s->xx[f1 + i]; yo1[i] = s->yy[f1 + i]; zo1[i] = s->zz[f1 + i];
        xn1[i] = xo1[i] - c1[0] + c2[0]; yn1[i] = yo1[i] - c1[1] + c2[1]; zn1[i] = zo1[i] - c1[2] + c2[2];
    }
    for (int i = 0; i < n2; i++) {
        xo2[i] = s->xx[f2 + i]; yo2[i] = s->yy[f2 + i]; zo2[i] = s->zz[f2 + i];
        xn2[i] = xo2[i] - c2[0] + c1[0]; yn2[i] = yo2[i] - c2[1] + c1[1]; zn2[i] = zo2[i] - c2[2] + c1[2];
    }
    /* real space with both molecules at their new positions (:1534-1570) */
    partial_t pn1, pn2, pn12;
    partial_alloc(&pn1, N); partial_alloc(&pn2, N); partial_alloc(&pn12, N);
    for (int i = 0; i < n1; i++) { s->xx[f1 + i] = xn1[i]; s->yy[f1 + i] = yn1[i]; s->zz[f1 + i] = zn1[i]; }
    for (int i = 0; i < n2; i++) { s->xx[f2 + i] = xn2[i]; s->yy[f2 + i] = yn2[i]; s->zz[f2 + i] = zn2[i]; }
    int ov1 = realspace_calc_j(s, 0, &pn1, xn1, yn1, zn1, f1, l1, 0, N);
    int ov2 = realspace_calc_j(s, 0, &pn2, xn2, yn2, zn2, f2, l2, 0, N);
    (void)realspace_calc_j(s, 0, &pn12, xn1, yn1, zn1, f1, l1, f2, l2 + 1);
    for (int i = 0; i < n1; i++) { s->xx[f1 + i] = xo1[i]; s->yy[f1 + i] = yo1[i]; s->zz[f1 + i] = zo1[i]; }
    for (int i = 0; i < n2; i++) { s->xx[f2 + i] = xo2[i]; s->yy[f2 + i] = yo2[i]; s->zz[f2 + i] = zo2[i]; }
    rec->flags = 4 | (imol2 << 8);
    if (ov1 || ov2) {
        rec->flags |= 2;
        partial_free(&pn1); partial_free(&pn2); partial_free(&pn12);
        return 0;
    }
    double T1 = 0, T2 = 0;
    for (int i = 0; i < n1; i++) T1 = T1 + pn1.uu[i];
    for (int i = 0; i < n2; i++) T2 = T2 + pn2.uu[i];
    double E_new = T1 + T2;
    double dU_real = E_new - E_old;
    /* new structure factors and the k-space change (:1652-1700) */
    rho_zero(&s->mol_new, nk, nt);
    for (int i = 0; i < n1; i++)
        rho_add_atom(s, &s->mol_new, xn1[i], yn1[i], zn1[i], s->charge[f1 + i], s->lj.type_by_index[f1 + i], &s->skr_coul[0], &s->skr_lj[0]);
    for (int i = 0; i < n2; i++)
        rho_add_atom(s, &s->mol_new, xn2[i], yn2[i], zn2[i], s->charge[f2 + i], s->lj.type_by_index[f2 + i], &s->skr_coul[0], &s->skr_lj[0]);
    rho_sub(&s->mol_new, &s->mol_old, nk, nt);
    double du_kc = kspace_du_coulomb(s, &s->mol_new.coul);
    double du_kl = kspace_du_lj(s, &s->mol_new);
    /* external field (:1706-1738) */
    double mn1[3], mn2[3];
    calc_mu(xn1, yn1, zn1, s->charge + f1, n1, &mn1[0], &mn1[1], &mn1[2]);
    calc_mu(xn2, yn2, zn2, s->charge + f2, n2, &mn2[0], &mn2[1], &mn2[2]);
    double dmx = (mn1[0] - mo1[0]) + (mn2[0] - mo2[0]);
    double dmy = (mn1[1] - mo1[1]) + (mn2[1] - mo2[1]);
    double dmz = (mn1[2] - mo1[2]) + (mn2[2] - mo2[2]);
    double dU_ext = p->kext * ((2 * s->mu_x + dmx) * dmx + (2 * s->mu_y + dmy) * dmy + (2 * s->mu_z + dmz) * dmz);
    double du_total = dU_real + (du_kc + du_kl) + dU_ext;
    rec->du_real = dU_real; rec->du_k_coul = du_kc; rec->du_k_lj = du_kl; rec->du_ext = dU_ext;
    /* MonteCarloMove_accept_or_decline_simple */
    double factor = exp(-du_total);
    double xksi = orc_rand(s);
    if (s->rng_out) { partial_free(&pn1); partial_free(&pn2); partial_free(&pn12); return -6; }
    int acc = !(xksi > factor);
    if (acc) {
        /* :1758-1848 */
        rho_add(&s->rho_total, &s->mol_new, nk, nt);
        partial_t po1, po2, po12;
        partial_alloc(&po1, N); partial_alloc(&po2, N); partial_alloc(&po12, N);
        realspace_calc_j(s, 0, &po1, xo1, yo1, zo1, f1, l1, 0, N);
        realspace_calc_j(s, 0, &po2, xo2, yo2, zo2, f2, l2, 0, N);
        realspace_calc_j(s, 0, &po12, xo1, yo1, zo1, f1, l1, f2, l2 + 1);
        for (int i = 0; i < N; i++) {
            s->uu[i] = s->uu[i] + pn1.uu_back[i] - po1.uu_back[i] + pn2.uu_back[i] - po2.uu_back[i];
            s->fx[i] = s->fx[i] + pn1.fx_back[i] - po1.fx_back[i] + pn2.fx_back[i] - po2.fx_back[i];
            s->fy[i] = s->fy[i] + pn1.fy_back[i] - po1.fy_back[i] + pn2.fy_back[i] - po2.fy_back[i];
            s->fz[i] = s->fz[i] + pn1.fz_back[i] - po1.fz_back[i] + pn2.fz_back[i] - po2.fz_back[i];
        }
        for (int i = 0; i < n1; i++) {
            s->uu[f1 + i] = pn1.uu[i]; s->fx[f1 + i] = pn1.fx[i]; s->fy[f1 + i] = pn1.fy[i]; s->fz[f1 + i] = pn1.fz[i];
        }
        for (int i = 0; i < n2; i++) {
            s->uu[f2 + i] = pn2.uu[i]; s->fx[f2 + i] = pn2.fx[i]; s->fy[f2 + i] = pn2.fy[i]; s->fz[f2 + i] = pn2.fz[i];
        }
        s->E_k_coul = s->E_k_coul + du_kc;
        s->E_k_lj = s->E_k_lj + du_kl;
        s->E_k = s->E_k_coul + s->E_k_lj;
        s->uu_ew = s->uu_ew + pn1.uu_ew - po1.uu_ew + pn2.uu_ew - po2.uu_ew - (pn12.uu_ew - po12.uu_ew);
        s->uu_lj6 = s->uu_lj6 + pn1.uu_lj6 - po1.uu_lj6 + pn2.uu_lj6 - po2.uu_lj6 - (pn12.uu_lj6 - po12.uu_lj6);
        s->uu_lj12 = s->uu_lj12 + pn1.uu_lj12 - po1.uu_lj12 + pn2.uu_lj12 - po2.uu_lj12 - (pn12.uu_lj12 - po12.uu_lj12);
        s->mu_x = s->mu_x + dmx; s->mu_y = s->mu_y + dmy; s->mu_z = s->mu_z + dmz;
        total_energy(s);
        for (int i = 0; i < n1; i++) { s->xx[f1 + i] = xn1[i]; s->yy[f1 + i] = yn1[i]; s->zz[f1 + i] = zn1[i]; }
        for (int i = 0; i < n2; i++) { s->xx[f2 + i] = xn2[i]; s->yy[f2 + i] = yn2[i]; s->zz[f2 + i] = zn2[i]; }
        partial_free(&po1); partial_free(&po2); partial_free(&po12);
        rec->flags |= 1;
    }
    partial_free(&pn1); partial_free(&pn2); partial_free(&pn12);
    return 0;
}

int32_t orc_xchange(orc_state *s, int32_t imol1, int32_t imol2, const float *rng, int64_t n_rng, int64_t *cursor,
                    orc_move_rec *rec) {
    s->rng = rng; s->n_rng = n_rng; s->cursor = cursor; s->rng_out = 0;
    if (imol1 < 1 || imol1 > s->nmol || imol2 < 1 || imol2 > s->nmol || imol1 == imol2) return -4;
    int r = mc_xchange(s, imol1, imol2, rec);
    rec->cursor = *cursor;
    return r;
}

int32_t orc_movemc(orc_state *s, int32_t imol, const float *rng, int64_t n_rng, int64_t *cursor, orc_move_rec *rec) {
    s->rng = rng; s->n_rng = n_rng; s->cursor = cursor; s->rng_out = 0;
    if (imol < 1 || imol > s->nmol) return -4;
    int r = movemc(s, imol, rec);
    rec->cursor = *cursor;
    return r;
}

/* energy.dat row at the end of a cycle (runmc.f90:276-279), frame = the cycle number */
static void cycle_end(orc_state *s, double *rows, int32_t max_rows, int32_t *n_rows) {
    if (fmod(s->n_mv_steps / s->nmol + s->n_vol_steps, s->p.n_store_energy_interval) < 1e-10) {
        if (rows && n_rows && *n_rows < max_rows) {
            double e[8];
            orc_energies(s, e);
            double *row = rows + 9 * (size_t)(*n_rows);
            row[0] = (double)s->icycle;
            for (int c = 0; c < 8; c++) row[1 + c] = e[c];
            (*n_rows)++;
        }
    }
    s->icycle++;
}

static int32_t run_moves(orc_state *s, int64_t n_moves, orc_move_rec *log, double *rows, int32_t max_rows,
                         int32_t *n_rows);
static int biased_choose_x(orc_state *s);
static int mc_xchange(orc_state *s, int imol1, int imol2, orc_move_rec *rec);

/* run_mc (runmc.f90:178-334), NVT single-molecule moves only */
int32_t orc_run_mc(orc_state *s, const float *rng, int64_t n_rng, int64_t *cursor, int64_t n_moves,
                   orc_move_rec *log, double *rows, int32_t max_rows, int32_t *n_rows) {
    s->rng = rng; s->n_rng = n_rng; s->cursor = cursor; s->rng_out = 0;
    if (s->p.pressure_step_multiplier > 0) return -4; /* NPT runs through orc_run_cycles */
    if (n_rows) *n_rows = 0;
    return run_moves(s, n_moves, log, rows, max_rows, n_rows);
}

/* the movemc calls of run_mc's move cycles (runmc.f90:224-272): the cycle's pressure draw
   at a cycle start (a move cycle: the caller has checked it), the exchange draw, the
   molecule choice, movemc */
static int32_t run_moves(orc_state *s, int64_t n_moves, orc_move_rec *log, double *rows, int32_t max_rows,
                         int32_t *n_rows) {
    for (int64_t m = 0; m < n_moves; m++) {
        const int64_t c_move = *s->cursor;  /* an interrupted move resumes from here */
        if (s->move_in_cycle == 0) {
            double rnd = orc_rand(s) * (s->p.pressure_step_multiplier + 1);
            (void)rnd;
        }
        double rnd = orc_rand(s);
        orc_move_rec rec;
        int r;
        if (rnd < s->xchange_probability) {
            /* exchange step (runmc.f90:238-259): two different molecules from xchange_freq */
            int imol1 = biased_choose_x(s), imol2 = imol1;
            while (imol2 == imol1 && !s->rng_out) imol2 = biased_choose_x(s);
            if (s->rng_out) { *s->cursor = c_move; return -6; }
            r = mc_xchange(s, imol1, imol2, &rec);
        } else {
            int imol = biased_choose(s);
            if (s->rng_out) { *s->cursor = c_move; return -6; }
            r = movemc(s, imol, &rec);
        }
        if (r == -6) *s->cursor = c_move;
        if (r) return r;
        rec.cursor = *s->cursor;
        if (rec.flags & 1) s->n_mv_accepted += 1;
        s->n_mv_steps += 1;
        if (log) log[m] = rec;
        s->move_in_cycle++;
        if (s->move_in_cycle == s->nmol) {
            s->move_in_cycle = 0;
            cycle_end(s, rows, max_rows, n_rows);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* NPT volume move: mcvol (MC.f90:701-825)                              */
/* ------------------------------------------------------------------ */
/* TMCState (MC.f90:149-255): what mc_save_state keeps; the parameters, the LJ
   type list and beta are kept too, only to undo a step that ran out of random
   numbers (the reference has no such case) */
typedef struct {
    double U_tail, U_tail_coul, U_tail_lj6, U_tail_lj12, U_ext, U_total, U_total_ew, U_total_lj;
    double E_k, E_k_coul, E_k_lj, uu_ew, uu_lj6, uu_lj12, uu_ew_intra, uu_lj6_intra, uu_lj12_intra;
    double *xx, *yy, *zz, *sigma, *fx, *fy, *fz, *uu;
    rho_t rho;
    double mu_x, mu_y, mu_z;
    orc_params p;
    double lj_sigma[MAX_LJ_TYPE];
    double *beta;
} mcstate_t;

static void mcstate_save(orc_state *s, mcstate_t *t) {
    int N = s->N, nk = s->g.nk, nt = s->lj.ntype;
    t->U_tail = s->U_tail; t->U_tail_coul = s->U_tail_coul; t->U_tail_lj6 = s->U_tail_lj6; t->U_tail_lj12 = s->U_tail_lj12;
    t->U_ext = s->U_ext; t->U_total = s->U_total; t->U_total_ew = s->U_total_ew; t->U_total_lj = s->U_total_lj;
    t->E_k = s->E_k; t->E_k_coul = s->E_k_coul; t->E_k_lj = s->E_k_lj;
    t->uu_ew = s->uu_ew; t->uu_lj6 = s->uu_lj6; t->uu_lj12 = s->uu_lj12;
    t->uu_ew_intra = s->uu_ew_intra; t->uu_lj6_intra = s->uu_lj6_intra; t->uu_lj12_intra = s->uu_lj12_intra;
    double **dst[8] = {&t->xx, &t->yy, &t->zz, &t->sigma, &t->fx, &t->fy, &t->fz, &t->uu};
    double *src[8] = {s->xx, s->yy, s->zz, s->sigma, s->fx, s->fy, s->fz, s->uu};
    for (int a = 0; a < 8; a++) { *dst[a] = malloc(sizeof(double) * N); memcpy(*dst[a], src[a], sizeof(double) * N); }
    rho_alloc(&t->rho, nk, nt);
    rho_copy(&t->rho, &s->rho_total, nk, nt);
    memcpy(t->rho.present, s->rho_total.present, sizeof t->rho.present);
    t->mu_x = s->mu_x; t->mu_y = s->mu_y; t->mu_z = s->mu_z;
    t->p = s->p;
    memcpy(t->lj_sigma, s->lj.sigma, sizeof t->lj_sigma);
    t->beta = malloc(sizeof(double) * nk);
    memcpy(t->beta, s->beta, sizeof(double) * nk);
}

/* mc_restore_state (MC.f90:205-255) */
static void mcstate_restore(orc_state *s, const mcstate_t *t) {
    int N = s->N, nk = s->g.nk, nt = s->lj.ntype;
    s->U_tail = t->U_tail; s->U_tail_coul = t->U_tail_coul; s->U_tail_lj6 = t->U_tail_lj6; s->U_tail_lj12 = t->U_tail_lj12;
    s->U_ext = t->U_ext; s->U_total = t->U_total; s->U_total_ew = t->U_total_ew; s->U_total_lj = t->U_total_lj;
    s->E_k = t->E_k; s->E_k_coul = t->E_k_coul; s->E_k_lj = t->E_k_lj;
    s->uu_ew = t->uu_ew; s->uu_lj6 = t->uu_lj6; s->uu_lj12 = t->uu_lj12;
    s->uu_ew_intra = t->uu_ew_intra; s->uu_lj6_intra = t->uu_lj6_intra; s->uu_lj12_intra = t->uu_lj12_intra;
    double *dst[8] = {s->xx, s->yy, s->zz, s->sigma, s->fx, s->fy, s->fz, s->uu};
    const double *src[8] = {t->xx, t->yy, t->zz, t->sigma, t->fx, t->fy, t->fz, t->uu};
    for (int a = 0; a < 8; a++) memcpy(dst[a], src[a], sizeof(double) * N);
    rho_copy(&s->rho_total, &t->rho, nk, nt);
    s->mu_x = t->mu_x; s->mu_y = t->mu_y; s->mu_z = t->mu_z;
}

static void mcstate_free(orc_state *s, mcstate_t *t) {
    free(t->xx); free(t->yy); free(t->zz); free(t->sigma); free(t->fx); free(t->fy); free(t->fz); free(t->uu);
    rho_free(&t->rho, s->lj.ntype);
    free(t->beta);
}

/* scale_box (scale_box.f90:6-62): molecule centres of mass keep their box coordinates,
   the atoms' offsets from them scale by L_old / L_new (bond lengths in Angstrom stay);
   single-atom molecules are left as they are; atomic sigma (box units) scales too */
static void scale_box(orc_state *s, double new_L) {
    double c = s->p.BoxLength / new_L;
    for (int m = 0; m < s->nmol; m++) {
        int f = s->first_atom[m], l = s->last_atom[m], n = l - f + 1;
        if (n == 1) continue;
        double xc, yc, zc;
        center_of_mass(&s->xx[f], &s->yy[f], &s->zz[f], &s->mass[f], n, &xc, &yc, &zc);
        for (int j = f; j <= l; j++) {
            s->xx[j] = (s->xx[j] - xc) * c + xc;
            s->yy[j] = (s->yy[j] - yc) * c + yc;
            s->zz[j] = (s->zz[j] - zc) * c + zc;
        }
    }
    for (int i = 0; i < s->N; i++) s->sigma[i] = s->sigma[i] * c;
}

/* mc_calc_total_sums with scale_beta (MC.f90:477-585, EwaldSumKSpace_init :197-223):
   beta is scaled instead of recomputed (alpha*L, hence beta6/beta12, stays fixed) */
static int full_sums_scaled(orc_state *s, double scale_beta) {
    int ov = realspace_calc(s, 1, NULL, NULL, NULL, NULL, 0, 0);
    if (scale_beta > (double)1e-9f)
        for (int k = 0; k < s->g.nk; k++) s->beta[k] = s->beta[k] * scale_beta;
    else { init_beta(s); init_beta_lj(s); }
    kspace_total_energy(s);
    calc_mu(s->xx, s->yy, s->zz, s->charge, s->N, &s->mu_x, &s->mu_y, &s->mu_z);
    tails(s);
    total_energy(s);
    return ov;
}

/* mcvol (MC.f90:701-825): a random walk in ln V, Frenkel & Smit algorithm 11.
   Draws: lambda, then the acceptance draw only when the probability is not above 1
   (`(proba > 1) .or. (rand() < proba)`, evaluated left to right with short-circuit as
   gfortran's optimised builds do); an overlap gives proba = -1, so it draws and rejects.
   Returns 0, or -6 when the random buffer ran out (the state is put back exactly). */
static int mcvol(orc_state *s, orc_vol_rec *rec) {
    int64_t cur0 = *s->cursor;
    double old_L = s->p.BoxLength;
    double old_V = old_L * old_L * old_L;
    double lambda = 2 * orc_rand(s) - 1.0;
    if (s->rng_out) return -6;
    double log_new_V = log(old_V) + lambda * s->p.log_max_volume_scaling;
    double new_V = exp(log_new_V);
    double new_L = pow(new_V, 1.0 / 3.0);
    double U_old = total_energy(s);
    mcstate_t st;
    mcstate_save(s, &st);
    scale_box(s, new_L);
    double xclb_old = s->p.xclb;
    orc_params_recalc(&s->p, new_L);
    double xclb_new = s->p.xclb;
    lj_scale_sigma(&s->lj, old_L / new_L);
    init_beta_lj(s);
    int ov = full_sums_scaled(s, xclb_new / xclb_old);
    double proba, dU = 0, arg = 0;
    if (!ov) {
        double U_new = total_energy(s);
        dU = U_new - U_old;
        double dV = new_V - old_V;
        arg = -dU - s->p.pressure_angstr_kT * dV + (s->nmol + 1) * log(new_V / old_V);
        proba = exp(arg);
    } else {
        proba = -1.0;
    }
    int acc = 1;
    if (!(proba > 1)) {
        double r = orc_rand(s);
        if (s->rng_out) {  /* undo exactly and rewind to before lambda */
            mcstate_restore(s, &st);
            s->p = st.p;
            memcpy(s->lj.sigma, st.lj_sigma, sizeof st.lj_sigma);
            lj_fill_tab(&s->lj);
            memcpy(s->beta, st.beta, sizeof(double) * s->g.nk);
            init_beta_lj(s);
            total_energy(s);
            mcstate_free(s, &st);
            *s->cursor = cur0;
            return -6;
        }
        acc = r < proba;
    }
    if (!acc) {
        mcstate_restore(s, &st);
        orc_params_recalc(&s->p, old_L);
        lj_scale_sigma(&s->lj, new_L / old_L);
        init_beta_lj(s);
        for (int k = 0; k < s->g.nk; k++) s->beta[k] = s->beta[k] * xclb_old / xclb_new;
        total_energy(s);
    }
    mcstate_free(s, &st);
    rec->flags = (acc ? 1 : 0) | (ov ? 2 : 0);
    rec->pad = 0;
    rec->box_old = old_L; rec->box_new = new_L; rec->du = dU; rec->arg = arg;
    rec->cursor = *s->cursor;
    return 0;
}

int32_t orc_mcvol(orc_state *s, const float *rng, int64_t n_rng, int64_t *cursor, orc_vol_rec *rec) {
    s->rng = rng; s->n_rng = n_rng; s->cursor = cursor; s->rng_out = 0;
    rec->cycle = s->icycle;
    return mcvol(s, rec);
}

/* run_mc (runmc.f90:178-334) by cycles, NPT included: each cycle draws
   rnd = rand()*(pressure_step_multiplier+1); above pressure_step_multiplier (when it is
   positive) the cycle is one mcvol, otherwise nmol movemc calls.  A call that starts in
   the middle of a move cycle finishes that cycle first (it counts as one of n_cycles). */
int32_t orc_run_cycles(orc_state *s, const float *rng, int64_t n_rng, int64_t *cursor, int64_t n_cycles,
                       int64_t *cycles_done, orc_move_rec *log, int64_t max_log, int64_t *n_log,
                       orc_vol_rec *vlog, int64_t max_vlog, int64_t *n_vlog, double *rows, int32_t max_rows,
                       int32_t *n_rows) {
    s->rng = rng; s->n_rng = n_rng; s->cursor = cursor; s->rng_out = 0;
    if (n_rows) *n_rows = 0;
    if (n_log) *n_log = 0;
    if (n_vlog) *n_vlog = 0;
    if (cycles_done) *cycles_done = 0;
    double psm = s->p.pressure_step_multiplier;
    for (int64_t c = 0; c < n_cycles; c++) {
        if (s->move_in_cycle == 0) {
            int64_t c0 = *cursor;
            double rnd = orc_rand(s) * (psm + 1);
            if (s->rng_out) { *cursor = c0; return -6; }
            if (psm > 0 && rnd > psm) {
                orc_vol_rec vr;
                vr.cycle = s->icycle;
                int r = mcvol(s, &vr);
                if (r) { *cursor = c0; return r; }
                if (vr.flags & 1) s->n_vol_accepted += 1;
                s->n_vol_steps += 1;
                if (vlog && n_vlog && *n_vlog < max_vlog) vlog[(*n_vlog)++] = vr;
                cycle_end(s, rows, max_rows, n_rows);
                if (cycles_done) (*cycles_done)++;
                continue;
            }
            *cursor = c0;  /* a move cycle: run_moves takes the draw again */
        }
        int64_t mic0 = s->move_in_cycle;
        int64_t n = s->nmol - mic0;
        int64_t room = log ? max_log - *n_log : 0;
        orc_move_rec *lg = (log && room >= n) ? log + *n_log : NULL;
        int r = run_moves(s, n, lg, rows, max_rows, n_rows);
        if (r == -6 && lg) *n_log += s->move_in_cycle - mic0;  /* the moves done before the stream ran out */
        if (r) return r;
        if (lg) *n_log += n;
        if (cycles_done) (*cycles_done)++;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* input files: Molecule.f90, composition.f90, MoleculeTable.f90        */
/* ------------------------------------------------------------------ */
static void dir_of(const char *path, char *out, size_t n) {
    strncpy(out, path, n - 1); out[n - 1] = 0;
    char *sl = strrchr(out, '/');
    if (sl) sl[1] = 0; else out[0] = 0;
}

/* Molecule_read_from_file (Molecule.f90:142-188) + Molecule_centrate (:190-209) */
static int read_mol(mol_t *m, const char *path) {
    FILE *f = fopen(path, "r");
    if (!f) return -2;
    char line[1024];
    int n = 0;
    while (fgets(line, sizeof line, f)) {
        char name[32];
        double v[8];
        int k = sscanf(line, "%31s %lf %lf %lf %lf %lf %lf %lf %lf", name, &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7]);
        if (k <= 0) continue;
        if (k < 9) { fclose(f); return -2; }
        if (n >= MAX_MOL_ATOMS) { fclose(f); return -3; }
        m->x[n] = v[0]; m->y[n] = v[1]; m->z[n] = v[2]; m->sigma[n] = v[3]; m->epsilon[n] = v[4];
        m->charge[n] = v[5]; m->mass[n] = v[6]; m->hard_core[n] = v[7];
        if (m->hard_core[n] < (double)1e-9f) m->hard_core[n] = m->sigma[n] * (double)sqrtf(0.4f);
        n++;
    }
    fclose(f);
    m->natoms = n;
    double xc, yc, zc;
    center_of_mass(m->x, m->y, m->z, m->mass, n, &xc, &yc, &zc);
    for (int i = 0; i < n; i++) { m->x[i] = m->x[i] - xc; m->y[i] = m->y[i] - yc; m->z[i] = m->z[i] - zc; }
    return 0;
}

/* read_little_endian (io.f90:224-259) */
static int read_le(FILE *f, int n, int *val) {
    int v = 0, power = 1;
    for (int i = 0; i < n; i++) {
        int c = fgetc(f);
        if (c == EOF) return -2;
        v = v + c * power;
        power = power * 256;
    }
    *val = v;
    return 0;
}

orc_state *orc_create(const orc_params *pin, const char *composition_path, const char *moltab_path, int32_t *status) {
    orc_state *s = calloc(1, sizeof(orc_state));
    *status = 0;
    s->p = *pin;
    /* Composition_read_from_file (composition.f90:84-142) */
    FILE *f = fopen(composition_path, "r");
    if (!f) { *status = -2; free(s); return NULL; }
    char dir[1024];
    dir_of(composition_path, dir, sizeof dir);
    if (fscanf(f, "%d", &s->nmoltypes) != 1 || s->nmoltypes < 1 || s->nmoltypes > MAX_MOL_TYPES) {
        fclose(f); *status = -2; free(s); return NULL;
    }
    int total_mol = 0, total_atoms = 0;
    for (int t = 0; t < s->nmoltypes; t++) {
        char name[512], path[1600];
        if (fscanf(f, "%511s %d", name, &s->mol_numbers[t]) != 2) { fclose(f); *status = -2; free(s); return NULL; }
        if (name[0] == '/') snprintf(path, sizeof path, "%s", name);
        else snprintf(path, sizeof path, "%s%s", dir, name);
        int r = read_mol(&s->moltypes[t], path);
        if (r) { fclose(f); *status = r; free(s); return NULL; }
        total_mol += s->mol_numbers[t];
        total_atoms += s->mol_numbers[t] * s->moltypes[t].natoms;
    }
    fclose(f);
    /* parameters: BoxLength from density needs the molecule count (mc_main.f90:527-536) */
    if (!s->p.are_read) s->p.are_read = 1;
    int r = orc_params_init(&s->p, total_mol);
    if (r) { *status = r; free(s); return NULL; }
    const orc_params *p = &s->p;

    /* MoleculeTable_load_binary (MoleculeTable.f90:240-319) */
    s->nmol = total_mol;
    s->mol_type = calloc(total_mol, sizeof(int)); s->first_atom = calloc(total_mol, sizeof(int));
    s->last_atom = calloc(total_mol, sizeof(int));
    s->mx = calloc(total_mol, sizeof(double)); s->my = calloc(total_mol, sizeof(double)); s->mz = calloc(total_mol, sizeof(double));
    s->mtheta = calloc(total_mol, sizeof(double)); s->mphi = calloc(total_mol, sizeof(double)); s->mpsi = calloc(total_mol, sizeof(double));
    int ii = 0;
    for (int t = 0; t < s->nmoltypes; t++) for (int i = 0; i < s->mol_numbers[t]; i++) s->mol_type[ii++] = t;
    f = fopen(moltab_path, "rb");
    if (!f) { *status = -2; return s; }
    double pow_xyz = 1, pow_ang = 1;
    for (int i = 0; i < p->input_nbytes_xyz; i++) pow_xyz = pow_xyz * 256;
    for (int i = 0; i < p->input_nbytes_ang; i++) pow_ang = pow_ang * 256;
    for (int i = 0; i < total_mol; i++) {
        int xi, yi, zi, it, ip, is;
        if (read_le(f, p->input_nbytes_xyz, &xi) || read_le(f, p->input_nbytes_xyz, &yi) ||
            read_le(f, p->input_nbytes_xyz, &zi) || read_le(f, p->input_nbytes_ang, &it) ||
            read_le(f, p->input_nbytes_ang, &ip) || read_le(f, p->input_nbytes_ang, &is)) {
            fclose(f); *status = -2; return s;
        }
        s->mx[i] = xi / pow_xyz - 0.5; s->my[i] = yi / pow_xyz - 0.5; s->mz[i] = zi / pow_xyz - 0.5;
        s->mtheta[i] = it / pow_ang * TWO_PI; s->mphi[i] = ip / pow_ang * TWO_PI; s->mpsi[i] = is / pow_ang * TWO_PI;
    }
    fclose(f);

    /* MoleculeTable_fillAtomicData (MoleculeTable.f90:584-705) */
    s->N = total_atoms;
    int N = total_atoms;
    s->xx = calloc(N, sizeof(double)); s->yy = calloc(N, sizeof(double)); s->zz = calloc(N, sizeof(double));
    s->sigma = calloc(N, sizeof(double)); s->epsilon = calloc(N, sizeof(double)); s->charge = calloc(N, sizeof(double));
    s->hard_core = calloc(N, sizeof(double)); s->mass = calloc(N, sizeof(double)); s->molnum = calloc(N, sizeof(int));
    int natom = 0;
    s->max_mol_atom = 0;
    for (int im = 0; im < total_mol; im++) {
        const mol_t *m = &s->moltypes[s->mol_type[im]];
        if (s->max_mol_atom < m->natoms) s->max_mol_atom = m->natoms;
        s->first_atom[im] = natom; s->last_atom[im] = natom + m->natoms - 1;
        double ct = cos(s->mtheta[im]), st = sin(s->mtheta[im]);
        double cp = cos(s->mphi[im]), sp = sin(s->mphi[im]);
        double cs = cos(s->mpsi[im]), ss = sin(s->mpsi[im]);
        for (int a = 0; a < m->natoms; a++) {
            double xm, ym, zm;
            rot_vect(m->x[a], m->y[a], m->z[a], &xm, &ym, &zm, cs, ss, 3);
            rot_vect(xm, ym, zm, &xm, &ym, &zm, ct, st, 2);
            rot_vect(xm, ym, zm, &xm, &ym, &zm, cp, sp, 3);
            s->xx[natom] = xm / p->BoxLength + s->mx[im];
            s->yy[natom] = ym / p->BoxLength + s->my[im];
            s->zz[natom] = zm / p->BoxLength + s->mz[im];
            s->charge[natom] = m->charge[a];
            s->sigma[natom] = m->sigma[a] / p->BoxLength;
            s->hard_core[natom] = m->hard_core[a];
            s->epsilon[natom] = m->epsilon[a] / p->kT_kcal_mol;
            s->mass[natom] = m->mass[a];
            s->molnum[natom] = im + 1;
            natom++;
        }
    }
    /* LJTypes_fill (mc_main.f90:548) */
    if ((r = lj_fill(&s->lj, s->sigma, s->epsilon, N))) { *status = r; return s; }
    int nt = s->lj.ntype;
    /* the LJ tails read comp%mol_numbers(t) by LJ type t (EwaldSumTails.f90:88) */
    if (nt > s->nmoltypes) { *status = -3; return s; }

    /* mc_alloc (MC.f90:257-379) */
    grid_init(&s->g, p->kmax);
    int nk = s->g.nk;
    s->beta = calloc(nk, sizeof(double)); s->beta6 = calloc(nk, sizeof(double)); s->beta12 = calloc(nk, sizeof(double));
    s->beta_lj = calloc(nt * nt > 0 ? nt * nt : 1, sizeof(double *));
    for (int t1 = 1; t1 <= nt; t1++)
        for (int t2 = t1; t2 <= nt; t2++) {
            int o12 = (t1 - 1) * nt + t2 - 1;
            s->beta_lj[o12] = calloc(nk, sizeof(double));
            if (t1 != t2) s->beta_lj[(t2 - 1) * nt + t1 - 1] = s->beta_lj[o12];
        }
    rho_alloc(&s->rho_total, nk, nt); rho_alloc(&s->mol_old, nk, nt);
    rho_alloc(&s->mol_new, nk, nt); rho_alloc(&s->total_new, nk, nt);
    s->skr_coul = calloc(s->max_mol_atom, sizeof(sck_t)); s->skr_lj = calloc(s->max_mol_atom, sizeof(sck_t));
    for (int i = 0; i < s->max_mol_atom; i++) { sck_alloc(&s->skr_coul[i], nk); sck_alloc(&s->skr_lj[i], nk); }
    int km = p->kmax + 1;
    s->xyz.cx = calloc(km, sizeof(double)); s->xyz.cy = calloc(km, sizeof(double)); s->xyz.cz = calloc(km, sizeof(double));
    s->xyz.sx = calloc(km, sizeof(double)); s->xyz.sy = calloc(km, sizeof(double)); s->xyz.sz = calloc(km, sizeof(double));
    for (int c = 0; c < 4; c++) { s->tc[c] = calloc(nk, sizeof(double)); s->ts[c] = calloc(nk, sizeof(double)); }
    s->uu = calloc(N, sizeof(double)); s->fx = calloc(N, sizeof(double)); s->fy = calloc(N, sizeof(double)); s->fz = calloc(N, sizeof(double));
    partial_t *pp[2] = {&s->ps_old, &s->ps_new};
    for (int k = 0; k < 2; k++) {
        pp[k]->uu_back = calloc(N, sizeof(double)); pp[k]->fx_back = calloc(N, sizeof(double));
        pp[k]->fy_back = calloc(N, sizeof(double)); pp[k]->fz_back = calloc(N, sizeof(double));
    }
    /* init_freq (runmc.f90:25-67) with no frequencies file: flat weights */
    s->freq_beg = calloc(total_mol, sizeof(double)); s->freq_end = calloc(total_mol, sizeof(double));
    double S = 0;
    for (int i = 0; i < total_mol; i++) S = S + 1.0;
    double prob = 1.0 / S;
    s->freq_beg[0] = 0.0; s->freq_end[0] = prob;
    for (int i = 1; i < total_mol; i++) { s->freq_beg[i] = s->freq_end[i - 1]; s->freq_end[i] = s->freq_beg[i] + prob; }
    s->smv = S;
    s->xfreq_beg = calloc(total_mol, sizeof(double)); s->xfreq_end = calloc(total_mol, sizeof(double));
    s->xchange_probability = 0.0;
    s->icycle = 1;
    /* initmc -> mc_calc_total_sums (MC.f90:587-602) */
    if (orc_full_sums(s, NULL)) *status = 1; /* overlap in the initial configuration */
    return s;
}

/* BiasedRandom_init (BiasedRandom.f90:44-79) on given move weights (init_freq with a frequencies
   file, runmc.f90:25-67): probabilities w/S (flat when S == 0), running-sum intervals, and
   end = -1 for a zero weight when S > 0. */
static double biased_random_init(double *beg, double *end, const double *w, int n) {
    double S = 0;
    for (int i = 0; i < n; i++) S = S + w[i];
    double *prob = malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) prob[i] = (S == 0) ? 1.0 / n : w[i] / S;
    beg[0] = 0.0; end[0] = prob[0];
    for (int i = 1; i < n; i++) { beg[i] = end[i - 1]; end[i] = beg[i] + prob[i]; }
    if (S > 0)
        for (int i = 0; i < n; i++) if (w[i] == 0) end[i] = -1.0;
    free(prob);
    return S;
}

int32_t orc_set_move_weights(orc_state *s, const double *w, int32_t n) {
    if (n != s->nmol) return -3;
    s->smv = biased_random_init(s->freq_beg, s->freq_end, w, n);
    return 0;
}

/* init_freq with exchange weights (runmc.f90:25-67): xchange_freq from the exchange weights,
   xchange_probability = Sxch / (Smv + Sxch) with Smv the move weights' sum */
int32_t orc_set_xchange_weights(orc_state *s, const double *w, int32_t n) {
    if (n != s->nmol) return -3;
    double sx = biased_random_init(s->xfreq_beg, s->xfreq_end, w, n);
    s->xchange_probability = sx / (s->smv + sx);
    return 0;
}

void orc_destroy(orc_state *s) {
    if (!s) return;
    int nt = s->lj.ntype;
    free(s->mol_type); free(s->first_atom); free(s->last_atom);
    free(s->mx); free(s->my); free(s->mz); free(s->mtheta); free(s->mphi); free(s->mpsi);
    free(s->xx); free(s->yy); free(s->zz); free(s->sigma); free(s->epsilon); free(s->charge);
    free(s->hard_core); free(s->mass); free(s->molnum);
    free(s->lj.type_by_index); free(s->lj.lj6); free(s->lj.lj12); free(s->lj.four_eps); free(s->lj.sigma6); free(s->lj.sigma2);
    if (s->g.kx) {
        rho_free(&s->rho_total, nt); rho_free(&s->mol_old, nt); rho_free(&s->mol_new, nt); rho_free(&s->total_new, nt);
        for (int i = 0; i < s->max_mol_atom; i++) { sck_free(&s->skr_coul[i]); sck_free(&s->skr_lj[i]); }
        free(s->skr_coul); free(s->skr_lj);
        for (int t1 = 1; t1 <= nt; t1++) for (int t2 = t1; t2 <= nt; t2++) free(s->beta_lj[(t1 - 1) * nt + t2 - 1]);
        free(s->beta_lj); free(s->beta); free(s->beta6); free(s->beta12);
        free(s->xyz.cx); free(s->xyz.cy); free(s->xyz.cz); free(s->xyz.sx); free(s->xyz.sy); free(s->xyz.sz);
        for (int c = 0; c < 4; c++) { free(s->tc[c]); free(s->ts[c]); }
        free(s->uu); free(s->fx); free(s->fy); free(s->fz);
        free(s->ps_old.uu_back); free(s->ps_old.fx_back); free(s->ps_old.fy_back); free(s->ps_old.fz_back);
        free(s->ps_new.uu_back); free(s->ps_new.fx_back); free(s->ps_new.fy_back); free(s->ps_new.fz_back);
        grid_free(&s->g);
    }
    free(s->freq_beg); free(s->freq_end); free(s->xfreq_beg); free(s->xfreq_end);
    free(s);
}

int32_t orc_natom(const orc_state *s) { return s->N; }
int32_t orc_nmol(const orc_state *s) { return s->nmol; }
int32_t orc_nk(const orc_state *s) { return s->g.nk; }
int32_t orc_ntype(const orc_state *s) { return s->lj.ntype; }
void orc_get_params(const orc_state *s, orc_params *p) { *p = s->p; }
void orc_get_atoms(const orc_state *s, double *x, double *y, double *z, double *q, int32_t *tbi, int32_t *molnum) {
    for (int i = 0; i < s->N; i++) {
        if (x) x[i] = s->xx[i];
        if (y) y[i] = s->yy[i];
        if (z) z[i] = s->zz[i];
        if (q) q[i] = s->charge[i];
        if (tbi) tbi[i] = s->lj.type_by_index[i];
        if (molnum) molnum[i] = s->molnum[i];
    }
}
void orc_get_mols(const orc_state *s, int32_t *first_atom, int32_t *last_atom) {
    for (int i = 0; i < s->nmol; i++) { first_atom[i] = s->first_atom[i] + 1; last_atom[i] = s->last_atom[i] + 1; }
}
void orc_get_uuF(const orc_state *s, double *uu, double *fx, double *fy, double *fz) {
    memcpy(uu, s->uu, sizeof(double) * s->N); memcpy(fx, s->fx, sizeof(double) * s->N);
    memcpy(fy, s->fy, sizeof(double) * s->N); memcpy(fz, s->fz, sizeof(double) * s->N);
}
void orc_get_rho(const orc_state *s, double *out) {
    int nk = s->g.nk, nt = s->lj.ntype;
    for (int st = 0; st <= nt; st++) {
        const sck_t *c = st == 0 ? &s->rho_total.coul : &s->rho_total.lj[st - 1];
        for (int a = 0; a < 8; a++) memcpy(out + ((size_t)st * 8 + a) * nk, c->a[a], sizeof(double) * nk);
    }
}
double orc_mu(const orc_state *s, int32_t c) { return c == 0 ? s->mu_x : c == 1 ? s->mu_y : s->mu_z; }
/* the intra-molecular parts of the last full real-space sum (uu_ew_intra, uu_lj6_intra,
   uu_lj12_intra of mc_calc_total_sums, EwaldSumRealSpace.f90:444-474) */
void orc_intra_sums(const orc_state *s, double out[3]) {
    out[0] = s->uu_ew_intra; out[1] = s->uu_lj6_intra; out[2] = s->uu_lj12_intra;
}

void orc_force_kspace_atom(orc_state *s, int32_t atom1, double x, double y, double z, double f[3]) {
    int a = atom1 - 1, ityp = s->lj.type_by_index[a];
    double fk[3], fl[3] = {0, 0, 0};
    rho_t tmp;
    rho_alloc(&tmp, s->g.nk, s->lj.ntype);
    rho_zero(&tmp, s->g.nk, s->lj.ntype);
    rho_add_atom(s, &tmp, x, y, z, s->charge[a], ityp, &s->skr_coul[0], &s->skr_lj[0]);
    force_k_coulomb(s, &s->rho_total.coul, &s->skr_coul[0], fk);
    if (ityp > 0) force_k_lj(s, &s->rho_total, ityp, &s->skr_lj[0], fl);
    f[0] = fk[0] + fl[0]; f[1] = fk[1] + fl[1]; f[2] = fk[2] + fl[2];
    rho_free(&tmp, s->lj.ntype);
}
double orc_box_length(const orc_state *s) { return s->p.BoxLength; }

/* ------------------------------------------------------------------ */
/* radial distribution functions: mcrdf2 count_distances / save_rdfs    */
/* ------------------------------------------------------------------ */
/* count_distances (mcrdf2.f90:110-333) for one frame: every ordered pair (i, j) of molecule
   centres (box units) and, when Rmax reaches past L/2, the periodic images up to Nbox boxes
   away; j shifted by one box where |x_i - x_j| > 0.5 first.  cnt4[(t1*ntypes + t2)*nbin + b]
   (t1 <= t2, 0-based species) counts the pairs with r in bin b = aint(r/dr), n_total[t1*ntypes+t2]
   all of them.  The interpolated, 1/r^2 and 1/(r^2 V) histograms of the reference are not
   formed: its output (save_rdfs) reads only cnt4.  nbin = aint((Rmax - 1e-10)/dr) + 2. */
void orc_rdf_count(int32_t M, const double *x, const double *y, const double *z, const int32_t *type, int32_t ntypes,
                   double L, double dr, double rmax, double *cnt4, double *n_total) {
    int nbin = (int)((rmax - 1e-10) / dr) + 2;
    double rmax2 = rmax * rmax;
    int nbox = rmax < L / 2 ? 0 : (int)((rmax - L / 2) / L) + 1;
    for (int i = 0; i < M; i++) {
        int ti = type[i] - 1;
        for (int j = 0; j < M; j++) {
            int tj = type[j] - 1;
            double x2 = x[j], y2 = y[j], z2 = z[j];
            if (x[i] - x2 > 0.5) x2 = x2 + 1.0;
            if (x[i] - x2 < -0.5) x2 = x2 - 1.0;
            if (y[i] - y2 > 0.5) y2 = y2 + 1.0;
            if (y[i] - y2 < -0.5) y2 = y2 - 1.0;
            if (z[i] - z2 > 0.5) z2 = z2 + 1.0;
            if (z[i] - z2 < -0.5) z2 = z2 - 1.0;
            for (int nx = -nbox; nx <= nbox; nx++)
                for (int ny = -nbox; ny <= nbox; ny++)
                    for (int nz = -nbox; nz <= nbox; nz++) {
                        if (i == j && nx == 0 && ny == 0 && nz == 0) continue;
                        double dx = (x[i] - x2 + nx) * L, dy = (y[i] - y2 + ny) * L, dz = (z[i] - z2 + nz) * L;
                        double r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 > rmax2 - 1e-10) continue;
                        double r = sqrt(r2);
                        int b = (int)(r / dr);
                        int off = ti < tj ? ti * ntypes + tj : tj * ntypes + ti;
                        n_total[off] += 1.0;
                        if (b < nbin) cnt4[(size_t)off * nbin + b] += 1.0;
                    }
        }
    }
}

/* save_rdfs (mcrdf2.f90:371-440), the written column: g(r_k + dr/2) = cnt4 / N_frame / <1/V> /
   N_i / N_j / dV / factor with dV = 4 pi dr (r^2 + r dr) + 4/3 pi dr^3, factor 2 for i != j */
void orc_rdf_normalize(int32_t ntypes, const int32_t *mol_numbers, double dr, double rmax, const double *cnt4,
                       const double *n_total, int32_t n_frame, double avg_inv_vol, double *g) {
    int nbin = (int)((rmax - 1e-10) / dr) + 2;
    double four_pi_dr = 4.0 * PI * dr, small_ball = 4.0 / 3.0 * PI * dr * dr * dr;
    for (int i = 0; i < ntypes; i++)
        for (int j = i; j < ntypes; j++) {
            int off = i * ntypes + j;
            double r = 0.0;
            for (int k = 0; k < nbin; k++) {
                double dV = four_pi_dr * (r * r + r * dr) + small_ball;
                double factor = i == j ? 1.0 : 2.0;
                double v = 0.0;
                if (n_total[off] > 0)
                    v = cnt4[(size_t)off * nbin + k] / n_frame / avg_inv_vol / mol_numbers[i] / mol_numbers[j] / dV / factor;
                g[(size_t)off * nbin + k] = v;
                r = r + dr;
            }
        }
}
