/* CPU restatement of the Rast-3DMHD RK3 step on one global domain (test infrastructure).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this library, and
 * only as the checker.  The product (rast-3dmhd_b200/) never links or calls it.
 *
 * Layout: every 3D array is the global (npx+2) x (npy+2) x (npz+2) domain, x fastest,
 * idx = i + NX*(j + NY*k), interior i in [1,npx], j in [1,npy], k in [1,npz].  The
 * arithmetic follows the reference statement by statement (file:line in r3d_oracle.c).
 */
#ifndef R3D_ORACLE_H
#define R3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_sim ora_sim;

/* Field ids for ora_field(). */
enum {
    ORA_RU = 0, ORA_RV, ORA_RW, ORA_RO, ORA_TT, ORA_UU, ORA_VV, ORA_WW,
    ORA_FU, ORA_FV, ORA_FW, ORA_FR, ORA_FT, ORA_ZRU, ORA_ZRV, ORA_ZRW, ORA_ZRO, ORA_ZTT,
    ORA_WW1, ORA_WW2, ORA_WW3, ORA_BX, ORA_BY, ORA_BZ, ORA_ZBX, ORA_ZBY, ORA_ZBZ,
    ORA_NFIELDS
};
/* 1D ids for ora_line(). */
enum {
    ORA_EXX = 0, ORA_DXXDX, ORA_D2XXDX2, ORA_DDX, ORA_WYY, ORA_DYYDY, ORA_D2YYDY2, ORA_DDY,
    ORA_ZEE, ORA_DZZDZ, ORA_D2ZZDZ2, ORA_DDZ, ORA_RKAPA, ORA_DKAPA, ORA_NLINES
};

/* Parse reference-style flags ("--npx 32", "--lmag=1", ...).  Returns NULL on error. */
ora_sim* ora_create(int argc, const char** argv);
void ora_destroy(ora_sim* s);
const char* ora_error(void);

/* Grid metrics + conductivity + static IC (+ seeded RAN2 perturbation) + ghost fill. */
int ora_init(ora_sim* s, int seed);
/* One RK3 step (nstages = 1..3 substages, as the reference's step(nstages, ...)). */
int ora_step(ora_sim* s, int nstages);
/* One FLUXES evaluation on the current state (overwrites RO with 1/RO like the reference). */
int ora_fluxes(ora_sim* s);
/* The halo exchange of the primaries (+B) on the global domain (periodic x/y copies). */
void ora_communicate(ora_sim* s);

double* ora_field(ora_sim* s, int id);
double* ora_line(ora_sim* s, int id);
/* scalars: dt timc timt timi umach tb nit */
void ora_get_scalars(const ora_sim* s, double* out7);
void ora_set_scalars(ora_sim* s, const double* in7);
void ora_dims(const ora_sim* s, int* out3);
/* Static polytrope T(k), R(k), k = 0..npz-1. */
int ora_static_profile(ora_sim* s, double* t, double* r);
void ora_ran2(int seed, int n, double* out);
void ora_mkgrid(ora_sim* s, double scode, int icoord, double* out3);
/* Copy of the parsed parameters as doubles in a fixed order (see r3d_oracle.c). */
int ora_param(const ora_sim* s, const char* name, double* out);

/* The itcon-2 embedded heat-loss term of the current state added to ft (test of the
   restatement against the Fortran block). */
int ora_heat_loss(ora_sim* s, double* ft);
/* density-diffusion terms (ID 1, 2) of the current state added to fr */
int ora_density_diffusion(ora_sim* s, double* fr);

#ifdef __cplusplus
}
#endif
#endif
