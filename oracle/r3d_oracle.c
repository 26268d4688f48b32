/* CPU restatement of the Rast-3DMHD time step (test infrastructure; see r3d_oracle.h).
 *
 * Statement-level restatement of:
 *   set-up      src/params.cpp:14-66 (derive), src/grid.cpp:28-276 (mkgrid, x/y/zjacobi),
 *               src/ode.cpp:20-174 (static profile, Bulirsch-Stoer), src/ran2.cpp:13-32,
 *               src/static_ic.cpp:24-161, src/main.cpp:134-154
 *   time step   src/step.cpp:37-257, src/fluxes.cpp:44-542, src/bcon.cpp:12-141,
 *               src/communicate.cpp:70-182 (periodic ghost fill of the global domain)
 *   MHD         golden/fortran/3dmhdsub.f:2146-2650 (FLUXES LMAG branch),
 *               3dmhdsub.f:907-1177 (B save/update/mix through WW1..WW3)
 * on a single global domain.  The reference splits y/z over MPI ranks; with one domain the
 * halo exchange reduces to the x/y periodic copies, and the global z ghost planes are the top
 * and bottom ranks' outer planes (never refreshed, as in the reference).  Every floating-point
 * expression keeps the reference's association; build with -ffp-contract=off.
 *
 * Pinning: the hydro path is checked bit for bit against the reference CPU sources compiled
 * unmodified (oracle/_ref) and against the reference's known-answer tests
 * (tests/test_oracle_pins.py).  The MHD flux branch has no reference C++ implementation
 * (src/fluxes.cpp:539-541 aborts) and the Fortran cannot be compiled here; it is checked bit
 * for bit against the reference's Fortran source executed statement by statement
 * (oracle/fortran_lmag.py, tests/test_oracle_mhd_pin.py).  The MHD initial condition and dt
 * terms are checked against the reference C++, which implements them.
 */
#include "r3d_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define F4(x) ((double)(float)(x))

/* ------------------------------------------------------------------ parameters ---- */
typedef struct {
    int npx, npy, npz, npey, ix, iy, ilap, ipad, ngrid, id, ncol, nrow;
    int ixcon, iycon, izcon, itcon, ibcon;
    int lrot, lmag, lpot, lrem, lshr;
    int ncase, ncasep, ntotal, nstep0, nstart, ntube, gpu_id, backend;
    double re, pr, theta, grav, r_y, ang, rm, beta, pzp, sigma, polys, tp, tc, xp, yp, zp;
    double xmax, ymax, zmax, ampt, ampb, bfh, bzp, qfh, gamma, hh, dh, dv, tstart, toff, rlax;
    double xx1, xx2, yy1, yy2, zz1, zz2, xa, xb, xc, xd, ya, yb, yc, yd, za, zb, zc, zd;
    double xcent, zcent, rmax, cmt, a_tube, lambda, vz0, sf;
} ora_params;

/* Defaults: include/params.hpp:26-113 (single-precision literals widened). */
static void params_default(ora_params* p) {
    memset(p, 0, sizeof(*p));
    p->npx = 504; p->npy = 504; p->npz = 2048; p->npey = 8;
    p->ix = 2; p->iy = 2; p->ilap = 2; p->ngrid = 1;
    p->itcon = 1;
    p->ncase = 1; p->ncasep = 1; p->ntotal = 1000; p->nstep0 = 100;
    p->re = 2.0; p->pr = F4(5.0e-2f); p->theta = 2.5e-1; p->grav = 6.25e-1;
    p->tp = 2.0; p->xp = 10.0; p->yp = 10.0;
    p->xmax = 20.0; p->ymax = 20.0; p->zmax = 40.0;
    p->ampt = F4(5.0e-3f); p->gamma = F4(5.0f / 3.0f); p->hh = 1.0;
    p->xx1 = -7.0; p->xx2 = 7.0; p->yy1 = -7.0; p->yy2 = 7.0; p->zz1 = -2.0; p->zz2 = 1.0e-2;
    p->xa = 0.5; p->xb = 0.48; p->xc = 28.0; p->xd = 0.025;
    p->ya = 0.5; p->yb = 0.48; p->yc = 28.0; p->yd = 0.025;
    p->za = 0.65; p->zb = 1.0; p->zc = 5.0; p->zd = 0.2;
    p->sf = F4(0.315f);
}

typedef struct { const char* name; char kind; size_t off; } flagdef;
#define FI(n, f) {n, 'i', offsetof(ora_params, f)}
#define FD(n, f) {n, 'd', offsetof(ora_params, f)}
#define FB(n, f) {n, 'b', offsetof(ora_params, f)}
/* Flag set: src/params.cpp:113-224. */
static const flagdef FLAGS[] = {
    FI("--npx", npx), FI("--npy", npy), FI("--npz", npz), FI("--npey", npey), FI("--ix", ix),
    FI("--iy", iy), FI("--ilap", ilap), FI("--ngrid", ngrid), FI("--id", id), FI("--ncol", ncol),
    FI("--nrow", nrow), FI("--ixcon", ixcon), FI("--iycon", iycon), FI("--izcon", izcon),
    FI("--itcon", itcon), FI("--ibcon", ibcon), FI("--ncase", ncase), FI("--ncasep", ncasep),
    FI("--ntotal", ntotal), FI("--nstep0", nstep0), FI("--nstart", nstart),
    FI("--ntube", ntube), FI("--gpu", gpu_id),
    FD("--re", re), FD("--pr", pr), FD("--theta", theta), FD("--grav", grav), FD("--ry", r_y),
    FD("--ang", ang), FD("--rm", rm), FD("--beta", beta), FD("--pzp", pzp),
    FD("--sigma", sigma), FD("--polys", polys), FD("--tp", tp), FD("--tc", tc), FD("--xp", xp),
    FD("--yp", yp), FD("--zp", zp), FD("--xmax", xmax), FD("--ymax", ymax), FD("--zmax", zmax),
    FD("--ampt", ampt), FD("--ampb", ampb), FD("--bfh", bfh), FD("--bzp", bzp), FD("--qfh", qfh),
    FD("--gamma", gamma), FD("--hh", hh), FD("--dh", dh), FD("--dv", dv),
    FD("--tstart", tstart), FD("--toff", toff), FD("--rlax", rlax), FD("--xx1", xx1),
    FD("--xx2", xx2), FD("--yy1", yy1), FD("--yy2", yy2), FD("--zz1", zz1), FD("--zz2", zz2),
    FD("--xa", xa), FD("--xb", xb), FD("--xc", xc), FD("--xd", xd), FD("--ya", ya),
    FD("--yb", yb), FD("--yc", yc), FD("--yd", yd), FD("--za", za), FD("--zb", zb),
    FD("--zc", zc), FD("--zd", zd), FD("--xcent", xcent), FD("--zcent", zcent),
    FD("--rmax", rmax), FD("--cmt", cmt), FD("--a", a_tube), FD("--lambda", lambda),
    FD("--vz0", vz0), FD("--sff", sf),
    FB("--lrot", lrot), FB("--lmag", lmag), FB("--lpot", lpot), FB("--lrem", lrem),
    FB("--lshr", lshr),
};

static char g_err[512];
static void set_err(const char* m) { snprintf(g_err, sizeof g_err, "%s", m); }
const char* ora_error(void) { return g_err; }

static int parse(int argc, const char** argv, ora_params* p) {
    for (int a = 0; a < argc; ++a) {
        const char* arg = argv[a];
        const char* val = NULL;
        int matched = 0;
        if (strncmp(arg, "--backend", 9) == 0 && (arg[9] == 0 || arg[9] == '=')) {
            val = arg[9] == '=' ? arg + 10 : (a + 1 < argc ? argv[++a] : NULL);
            if (!val) { set_err("missing value for --backend"); return -1; }
            if (strcmp(val, "cpu") == 0) p->backend = 0;
            else if (strcmp(val, "gpu") == 0) p->backend = 1;
            else { set_err("--backend must be 'cpu' or 'gpu'"); return -1; }
            continue;
        }
        for (size_t f = 0; f < sizeof FLAGS / sizeof FLAGS[0]; ++f) {
            size_t n = strlen(FLAGS[f].name);
            if (strncmp(arg, FLAGS[f].name, n) != 0) continue;
            if (arg[n] == '=') val = arg + n + 1;
            else if (arg[n] == 0) {
                if (a + 1 >= argc) { snprintf(g_err, sizeof g_err, "missing value for %s", arg); return -1; }
                val = argv[++a];
            } else continue;
            char* base = (char*)p + FLAGS[f].off;
            if (FLAGS[f].kind == 'i') *(int*)base = atoi(val);
            else if (FLAGS[f].kind == 'd') *(double*)base = atof(val);
            else *(int*)base = (!strcmp(val, "1") || !strcmp(val, "true") || !strcmp(val, "yes") || !strcmp(val, "on"));
            matched = 1;
            break;
        }
        if (!matched) { snprintf(g_err, sizeof g_err, "unknown option '%s'", arg); return -1; }
    }
    return 0;
}

/* ------------------------------------------------------------------- state -------- */
struct ora_sim {
    ora_params p;
    int NX, NY, NZ;
    long N;
    /* derived: src/params.cpp:29-64 */
    double c13, c23, c43, gam1, gam2, gam3, zeta1, zeta2, hx, h2x, hy, h2y, hz, h2z;
    double repr, ore, cv, ocv, rkapst, orm, obeta, omx, omz;
    double* f[ORA_NFIELDS];
    double* line[ORA_NLINES];
    double* scr[4]; /* MHD scratch standing in for RU/RV/RW/TT reuse (interior only) */
    double dt, timc, timt, timi, umach, tb;
    int nit;
};

#define IDX(i, j, k) ((long)(k) * s->NX * s->NY + (long)(j) * s->NX + (i))

static void derive(ora_sim* s) {
    const ora_params* p = &s->p;
    s->c13 = F4(1.0f / 3.0f);
    s->c23 = 2.0 * s->c13;
    s->c43 = 4.0 * s->c13;
    s->gam1 = F4(8.0f / 15.0f);
    s->gam2 = F4(5.0f / 12.0f);
    s->gam3 = F4(3.0f / 4.0f);
    s->zeta1 = F4(-17.0f / 60.0f);
    s->zeta2 = F4(-5.0f / 12.0f);
    s->hx = F4(0.5f * (float)(p->npx - 1));
    s->h2x = F4((float)(p->npx - 1) * (float)(p->npx - 1));
    s->hy = F4(0.5f * (float)(p->npy - 1));
    s->h2y = F4((float)(p->npy - 1) * (float)(p->npy - 1));
    s->hz = F4(0.5f * (float)(p->npz - 1));
    s->h2z = F4((float)(p->npz - 1) * (float)(p->npz - 1));
    s->repr = p->re * p->pr;
    s->ore = 1.0 / p->re;
    s->cv = 1.0 / (p->gamma - 1.0);
    s->ocv = 1.0 / s->cv;
    s->rkapst = (p->grav == 0.0) ? 1.0 : (p->polys + 1.0) * p->theta / p->grav;
    if (p->lmag) { s->orm = 1.0 / p->rm; s->obeta = 2.0 / p->beta; }
    else { s->orm = 0.0; s->obeta = 0.0; }
    if (p->lrot) { s->omx = sin(p->ang) / p->r_y; s->omz = cos(p->ang) / p->r_y; }
    else { s->omx = 0.0; s->omz = 0.0; }
}

ora_sim* ora_create(int argc, const char** argv) {
    ora_sim* s = (ora_sim*)calloc(1, sizeof(ora_sim));
    params_default(&s->p);
    if (parse(argc, argv, &s->p) != 0) { free(s); return NULL; }
    const ora_params* p = &s->p;
    if (p->npx < 1 || p->npy < 1 || p->npz < 1) { set_err("grid extents must be positive"); free(s); return NULL; }
    s->NX = p->npx + 2; s->NY = p->npy + 2; s->NZ = p->npz + 2;
    s->N = (long)s->NX * s->NY * s->NZ;
    for (int q = 0; q < ORA_NFIELDS; ++q) s->f[q] = (double*)calloc(s->N, sizeof(double));
    for (int q = 0; q < 4; ++q) s->scr[q] = (double*)calloc(s->N, sizeof(double));
    for (int q = 0; q < ORA_NLINES; ++q) {
        int n = q < 4 ? s->NX : (q < 8 ? s->NY : s->NZ);
        s->line[q] = (double*)calloc(n, sizeof(double));
    }
    derive(s);
    s->tb = 1.0;
    return s;
}

void ora_destroy(ora_sim* s) {
    if (!s) return;
    for (int q = 0; q < ORA_NFIELDS; ++q) free(s->f[q]);
    for (int q = 0; q < 4; ++q) free(s->scr[q]);
    for (int q = 0; q < ORA_NLINES; ++q) free(s->line[q]);
    free(s);
}

double* ora_field(ora_sim* s, int id) { return (id >= 0 && id < ORA_NFIELDS) ? s->f[id] : NULL; }
double* ora_line(ora_sim* s, int id) { return (id >= 0 && id < ORA_NLINES) ? s->line[id] : NULL; }
void ora_dims(const ora_sim* s, int* o) { o[0] = s->NX; o[1] = s->NY; o[2] = s->NZ; }
void ora_get_scalars(const ora_sim* s, double* o) {
    o[0] = s->dt; o[1] = s->timc; o[2] = s->timt; o[3] = s->timi; o[4] = s->umach; o[5] = s->tb;
    o[6] = (double)s->nit;
}
void ora_set_scalars(ora_sim* s, const double* v) {
    s->dt = v[0]; s->timc = v[1]; s->timt = v[2]; s->timi = v[3]; s->umach = v[4]; s->tb = v[5];
    s->nit = (int)v[6];
}

int ora_param(const ora_sim* s, const char* name, double* out) {
    for (size_t f = 0; f < sizeof FLAGS / sizeof FLAGS[0]; ++f) {
        if (strcmp(FLAGS[f].name, name) != 0) continue;
        const char* base = (const char*)&s->p + FLAGS[f].off;
        *out = FLAGS[f].kind == 'd' ? *(const double*)base : (double)*(const int*)base;
        return 0;
    }
    if (!strcmp(name, "--backend")) { *out = s->p.backend; return 0; }
    /* derived constants */
    struct { const char* n; double v; } dv[] = {
        {"c13", s->c13}, {"c23", s->c23}, {"c43", s->c43}, {"gam1", s->gam1}, {"gam2", s->gam2},
        {"gam3", s->gam3}, {"zeta1", s->zeta1}, {"zeta2", s->zeta2}, {"hx", s->hx}, {"h2x", s->h2x},
        {"hy", s->hy}, {"h2y", s->h2y}, {"hz", s->hz}, {"h2z", s->h2z}, {"repr", s->repr},
        {"ore", s->ore}, {"cv", s->cv}, {"ocv", s->ocv}, {"rkapst", s->rkapst}, {"orm", s->orm},
        {"obeta", s->obeta}, {"omx", s->omx}, {"omz", s->omz}};
    for (size_t q = 0; q < sizeof dv / sizeof dv[0]; ++q)
        if (!strcmp(dv[q].n, name)) { *out = dv[q].v; return 0; }
    return -1;
}

/* ---------------------------------------------------------------- RAN2 ------------ */
/* src/ran2.cpp:13-32 (Numerical Recipes RAN2, RM = f4(1/714025)). */
typedef struct { int idum, iiy, iir[97]; } ran2_state;
static double ran2(ran2_state* st) {
    const int M = 714025, IA = 1366, IC = 150889;
    const double RM = F4(1.0f / 714025.0f);
    if (st->idum < 0) {
        st->idum = (IC - st->idum) % M;
        for (int j = 0; j < 97; ++j) {
            st->idum = (IA * st->idum + IC) % M;
            st->iir[j] = st->idum;
        }
        st->idum = (IA * st->idum + IC) % M;
        st->iiy = st->idum;
    }
    int j = 1 + (97 * st->iiy) / M;
    if (j > 97 || j < 1) abort();
    st->iiy = st->iir[j - 1];
    double r = (double)st->iiy * RM;
    st->idum = (IA * st->idum + IC) % M;
    st->iir[j - 1] = st->idum;
    return r;
}
void ora_ran2(int seed, int n, double* out) {
    ran2_state st; memset(&st, 0, sizeof st); st.idum = -seed;
    for (int i = 0; i < n; ++i) out[i] = ran2(&st);
}

/* ---------------------------------------------------------------- MKGRID ---------- */
/* src/grid.cpp:28-146 */
static void mkgrid(const ora_params* p, double scode, int icoord, double* sphys, double* dsds,
                   double* d2sds2) {
    const double onepi = 2.0 * asin(1.0);
    if (p->ngrid == 0) {
        double smax = icoord == 1 ? p->xmax : (icoord == 2 ? p->ymax : p->zmax);
        *sphys = scode * smax;
        *dsds = 1.0 / smax;
        *d2sds2 = 0.0;
        return;
    }
    if (p->ngrid == 1) {
        double s1, s2, smax;
        if (icoord == 1) { s1 = p->xx1; s2 = p->xx2; smax = p->xmax; }
        else if (icoord == 2) { s1 = p->yy1; s2 = p->yy2; smax = p->ymax; }
        else { s1 = p->zz1; s2 = p->zz2; smax = p->zmax; }
        double a1 = (s2 - s1) / smax;
        double a3 = atan(s1);
        double a2 = atan(s2) - a3;
        if (scode == 0.0) *sphys = 0.0;
        else if (scode == 1.0) *sphys = smax;
        else *sphys = (tan(a2 * scode + a3) - s1) / a1;
        *dsds = a1 / a2 / (1.0 + (s1 + a1 * *sphys) * (s1 + a1 * *sphys));
        double t = (s1 + a1 * *sphys);
        double den = (1.0 + t * t);
        *d2sds2 = -2.0 * a1 * a1 * t / a2 / (den * den);
        return;
    }
    /* ngrid == 2 */
    double a, b, c, dp, smax;
    if (icoord == 1) { a = p->xa; b = p->xb; c = p->xc; dp = p->xd; smax = p->xmax; }
    else if (icoord == 2) { a = p->ya; b = p->yb; c = p->yc; dp = p->yd; smax = p->ymax; }
    else { a = p->za; b = p->zb; c = p->zc; dp = p->zd; smax = p->zmax; }
    if (c <= 1.0e-9) {
        *sphys = scode * smax;
        *dsds = 1.0 / smax;
        *d2sds2 = 0.0;
        return;
    }
    double sh = (1.0 - dp) * onepi /
                (dp * atan((a - b) * c) + 2.0 * atan(b * c) - dp * atan((a + b) * c));
    double sk = 2.0 * c * onepi * smax /
                (2.0 * c * onepi +
                 sh * (2.0 * c *
                           (atan((a - b) * c) * (a - b) - atan((a + b) * c) * (a + b) +
                            atan((a - b - 1.0) * c) + atan((a + b - 1.0) * c) * (a + b - 1.0) +
                            atan((1.0 - a + b) * c) * (a - b)) -
                       log(1.0 + (a - b) * (a - b) * c * c) + log(1.0 + (a + b) * (a + b) * c * c) -
                       log(1.0 + (a + b - 1.0) * (a + b - 1.0) * c * c) +
                       log(1.0 + (1.0 - a + b) * (1.0 - a + b) * c * c)));
    *dsds = 1.0 / (sk * (1.0 + sh / onepi * (atan(c * (scode - a - b)) + atan(c * (a - scode - b)))));
    *d2sds2 = -*dsds * *dsds * *dsds * c * sh * sk / onepi *
              (1.0 / (1.0 + c * c * (a + b - scode) * (a + b - scode)) -
               1.0 / (1.0 + c * c * (a - b - scode) * (a - b - scode)));
    *sphys = sk / (2.0 * c * onepi) *
             (2.0 * c * onepi * scode +
              sh * (2.0 * c *
                        (atan((a - b) * c) * (a - b) - atan((a + b) * c) * (a + b) +
                         atan((a - b - scode) * c) * scode + atan((a + b - scode) * c) * (a + b - scode) +
                         atan((scode - a + b) * c) * (a - b)) -
                    log(1.0 + (a - b) * (a - b) * c * c) + log(1.0 + (a + b) * (a + b) * c * c) -
                    log(1.0 + (a + b - scode) * (a + b - scode) * c * c) +
                    log(1.0 + (scode - a + b) * (scode - a + b) * c * c)));
    if (scode == 0.0) *sphys = 0.0;
    if (scode == 1.0) *sphys = smax;
}
void ora_mkgrid(ora_sim* s, double scode, int icoord, double* o) {
    mkgrid(&s->p, scode, icoord, &o[0], &o[1], &o[2]);
}

/* Global (stitched) metrics.  x: src/grid.cpp:148-167.  y/z: grid.cpp:169-276 evaluated as
 * the multi-rank result stitched together: ghost 0 -> mkgrid(0), interior g -> mkgrid(s[g-1])
 * with s[n] = n*f4(1/(np-1)), s[0]=0, s[np-1]=1, ghost np+1 -> mkgrid(1). */
static void build_metrics(ora_sim* s) {
    const ora_params* p = &s->p;
    double* exx = s->line[ORA_EXX]; double* dxxdx = s->line[ORA_DXXDX];
    double* d2xxdx2 = s->line[ORA_D2XXDX2]; double* ddx = s->line[ORA_DDX];
    const int nx = s->NX;
    double orx = F4(1.0f / (float)(nx - p->ix - 1));
    for (int i = 0; i < nx - p->ix - 1; ++i) exx[i + 1] = i * orx;
    exx[1] = 0.0;
    exx[nx - p->ix] = 1.0;
    for (int i = 1; i <= nx - p->ix; ++i) {
        double sp, ds, d2;
        mkgrid(p, exx[i], 1, &sp, &ds, &d2);
        exx[i] = sp; dxxdx[i] = ds; d2xxdx2[i] = d2; ddx[i] = orx * (1.0 / ds);
    }
    for (int ax = 2; ax <= 3; ++ax) {
        int np = ax == 2 ? p->npy : p->npz;
        int n = np + 2;
        double* e = s->line[ax == 2 ? ORA_WYY : ORA_ZEE];
        double* d1 = s->line[ax == 2 ? ORA_DYYDY : ORA_DZZDZ];
        double* d2a = s->line[ax == 2 ? ORA_D2YYDY2 : ORA_D2ZZDZ2];
        double* dd = s->line[ax == 2 ? ORA_DDY : ORA_DDZ];
        double o = F4(1.0f / (float)(np - 1));
        for (int g = 0; g < n; ++g) {
            double sc;
            if (g == 0) sc = 0.0;
            else if (g == n - 1) sc = 1.0;
            else if (g == 1) sc = 0.0;
            else if (g == np) sc = 1.0;
            else sc = (g - 1) * o;
            double sp, ds, d2;
            mkgrid(p, sc, ax, &sp, &ds, &d2);
            e[g] = sp; d1[g] = ds; d2a[g] = d2;
        }
        for (int g = 0; g < n; ++g) dd[g] = o * (1.0 / d1[g]);
    }
    /* conductivity: src/main.cpp:135-146 */
    for (int k = 0; k < s->NZ; ++k) {
        if (p->pzp == 0.0) { s->line[ORA_RKAPA][k] = 1.0; s->line[ORA_DKAPA][k] = 0.0; }
        else {
            double xe = s->line[ORA_ZEE][k];
            s->line[ORA_RKAPA][k] = 1.0 + (s->rkapst - 1.0) / 2.0 * (1.0 + tanh((xe - p->pzp) / p->sigma));
            s->line[ORA_DKAPA][k] = (s->rkapst - 1.0) / 2.0 / p->sigma / cosh((xe - p->pzp) / p->sigma) /
                                    cosh((xe - p->pzp) / p->sigma);
        }
    }
}

/* ------------------------------------------------------- static profile (BS) ----- */
/* src/ode.cpp:20-174 (DERIVS, RZEXTR, MMID, BSSTEP, static_profile). */
#define KNMAX 10
#define KIMAX 11
#define KNUSE 7
static const int NSEQ[KIMAX] = {2, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96};

static void derivs(const ora_params* p, double zz, const double* y, double* dydx) {
    double z, dzzdz, d2;
    mkgrid(p, zz, 3, &z, &dzzdz, &d2);
    double rkapst = (p->grav == 0.0) ? 1.0 : (p->polys + 1.0) * p->theta / p->grav;
    double rkap = (p->pzp == 0.0) ? 1.0 : 1.0 + (rkapst - 1.0) / 2.0 * (1.0 + tanh((z - p->pzp) / p->sigma));
    dydx[0] = p->theta / rkap / dzzdz;
    dydx[1] = p->grav / (1.0 + y[0]) / dzzdz;
}

static void rzextr(int iest, double xest, const double* yest, double* yz, double d[KNMAX][KNUSE],
                   double* dy, int nv, double* xbuf) {
    xbuf[iest - 1] = xest;
    if (iest == 1) {
        for (int j = 0; j < nv; ++j) { yz[j] = yest[j]; d[j][0] = yest[j]; dy[j] = yest[j]; }
        return;
    }
    int m1 = iest < KNUSE ? iest : KNUSE;
    double fx[KNUSE + 1];
    for (int k = 0; k < m1 - 1; ++k) fx[k + 1] = xbuf[iest - k - 2] / xest;
    for (int j = 0; j < nv; ++j) {
        double yy = yest[j], v = d[j][0], c = yy, ddy = 0.0;
        d[j][0] = yy;
        for (int k = 1; k < m1; ++k) {
            double b1 = fx[k] * v;
            double b = b1 - c;
            if (b != 0.0) { b = (c - v) / b; ddy = c * b; c = b1 * b; }
            else ddy = v;
            v = d[j][k];
            d[j][k] = ddy;
            yy += ddy;
        }
        dy[j] = ddy;
        yz[j] = yy;
    }
}

static void mmid(const ora_params* p, const double* y, const double* dydx, int nvar, double xs,
                 double htot, int nstp, double* yout) {
    double h = htot / nstp, ym[KNMAX], yn[KNMAX], yt[KNMAX];
    for (int i = 0; i < nvar; ++i) { ym[i] = y[i]; yn[i] = y[i] + h * dydx[i]; }
    double x = xs + h;
    derivs(p, x, yn, yt);
    double h2 = 2.0 * h;
    for (int n = 1; n < nstp; ++n) {
        for (int i = 0; i < nvar; ++i) { double sw = ym[i] + h2 * yt[i]; ym[i] = yn[i]; yn[i] = sw; }
        x += h;
        derivs(p, x, yn, yt);
    }
    for (int i = 0; i < nvar; ++i) yout[i] = 0.5 * (ym[i] + yn[i] + h * yt[i]);
}

static int bsstep(const ora_params* p, double* y, double* dydx, int nv, double* x, double htry,
                  double eps, double* hdid, double* hnext, double* xbuf) {
    double h = htry, xsav = *x, ysav[KNMAX], dysav[KNMAX], yseq[KNMAX], yerr[KNMAX];
    double d[KNMAX][KNUSE];
    for (int i = 0; i < nv; ++i) { ysav[i] = y[i]; dysav[i] = dydx[i]; }
    for (;;) {
        for (int i = 1; i <= KIMAX; ++i) {
            mmid(p, ysav, dysav, nv, xsav, h, NSEQ[i - 1], yseq);
            double xest = (h / NSEQ[i - 1]) * (h / NSEQ[i - 1]);
            rzextr(i, xest, yseq, y, d, yerr, nv, xbuf);
            double errmax = 0.0;
            for (int j = 0; j < nv; ++j) { double e = fabs(yerr[j] / y[j]); if (e > errmax) errmax = e; }
            errmax /= eps;
            if (errmax < 1.0) {
                *x += h;
                *hdid = h;
                if (i == KNUSE) *hnext = h * 0.95;
                else if (i == KNUSE - 1) *hnext = h * 1.2;
                else *hnext = (h * NSEQ[KNUSE - 1]) / NSEQ[i - 1];
                return 0;
            }
        }
        h = 0.25 * h / pow(2.0, (double)((KIMAX - KNUSE) / 2));
        if (*x + h == *x) return -1;
    }
}

static int static_profile(const ora_params* p, int npz, double* tp, double* rp) {
    double dzz = F4(1.0f / (float)(npz - 1));
    double y[2] = {0.0, 0.0}, zz = 0.0, xbuf[KIMAX];
    tp[0] = 1.0; rp[0] = 1.0;
    for (int k = 1; k < npz; ++k) {
        double dydx[2], hdid, hnext;
        derivs(p, zz, y, dydx);
        if (bsstep(p, y, dydx, 2, &zz, dzz, 1.0e-12, &hdid, &hnext, xbuf) != 0) return -1;
        if (hdid != dzz) return -1;
        tp[k] = 1.0 + y[0];
        rp[k] = exp(y[1]) / (1.0 + y[0]);
    }
    return 0;
}
int ora_static_profile(ora_sim* s, double* t, double* r) { return static_profile(&s->p, s->p.npz, t, r); }

/* ------------------------------------------------------------- ghost fill --------- */
/* src/communicate.cpp:70-168 on one domain: y periodic copy of one plane, then x periodic
 * copy of one column, over every k (the global z ghost planes included). */
static void ghost_fill(ora_sim* s, double* f) {
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < NZ; ++k) {
        double* pl = f + (long)k * NX * NY;
        memcpy(pl + 0 * (long)NX, pl + (long)(NY - 2) * NX, sizeof(double) * NX);
        memcpy(pl + (long)(NY - 1) * NX, pl + 1 * (long)NX, sizeof(double) * NX);
        for (int j = 0; j < NY; ++j) {
            pl[(long)j * NX + 0] = pl[(long)j * NX + NX - 2];
            pl[(long)j * NX + NX - 1] = pl[(long)j * NX + 1];
        }
    }
}
static void communicate(ora_sim* s) {
    ghost_fill(s, s->f[ORA_RU]); ghost_fill(s, s->f[ORA_RV]); ghost_fill(s, s->f[ORA_RW]);
    ghost_fill(s, s->f[ORA_TT]); ghost_fill(s, s->f[ORA_RO]);
    if (s->p.lmag) { ghost_fill(s, s->f[ORA_BX]); ghost_fill(s, s->f[ORA_BY]); ghost_fill(s, s->f[ORA_BZ]); }
}

/* --------------------------------------------------------------- static IC -------- */
/* src/static_ic.cpp:24-161 + src/main.cpp:148-154 on the global domain. */
int ora_init(ora_sim* s, int seed) {
    const ora_params* p = &s->p;
    if (p->ix != 2 || p->iy != 2 || p->ilap != 2) { set_err("ix/iy/ilap must be 2"); return -1; }
    if (p->npx < 3 || p->npy < 3 || p->npz < 4) { set_err("grid too small"); return -1; }
    if (p->nstart != 0) { set_err("restart (nstart != 0) is not supported"); return -1; }
    if (p->lshr || p->lrem) { set_err("LSHR/LREM not supported"); return -1; }
    if (p->lmag && p->ntube != 0) { set_err("TUBE models not supported"); return -1; }
    if (p->ampb != 0.0 && !p->lmag) { set_err("AMPB requires LMAG"); return -1; }
    build_metrics(s);
    const int NX = s->NX, NY = s->NY, NZ = s->NZ, npz = p->npz;
    for (int q = 0; q < ORA_NFIELDS; ++q) memset(s->f[q], 0, sizeof(double) * s->N);
    double* T = (double*)malloc(sizeof(double) * npz);
    double* R = (double*)malloc(sizeof(double) * npz);
    if (static_profile(p, npz, T, R) != 0) { free(T); free(R); set_err("static profile failed"); return -1; }
    const double tb = T[npz - 1], rb = R[npz - 1];
    s->tb = tb;
    double* tt = s->f[ORA_TT]; double* ro = s->f[ORA_RO];
    for (int k = 0; k < NZ; ++k) {
        double tv = k == 0 ? T[0] : (k == NZ - 1 ? tb : T[k - 1]);
        double rv = k == 0 ? R[0] : (k == NZ - 1 ? rb : R[k - 1]);
        for (int j = 1; j <= NY - 2; ++j)
            for (int i = 1; i <= NX - 2; ++i) { tt[IDX(i, j, k)] = tv; ro[IDX(i, j, k)] = rv; }
    }
    if (p->lmag) {
        /* src/static_ic.cpp:94-108 (C++ association cln = f4(-4 log 2)/(bfh*bfh)) */
        double cln = F4(-4.0f * logf(2.0f)) / (p->bfh * p->bfh);
        double* bx = s->f[ORA_BX];
        const double* zee = s->line[ORA_ZEE];
        for (int k = 1; k <= NZ - 2; ++k) {
            double bfac = p->ampb * exp(cln * (zee[k] - p->bzp) * (zee[k] - p->bzp));
            for (int j = 0; j < NY; ++j)
                for (int i = 0; i < NX; ++i) bx[IDX(i, j, k)] = bfac;
        }
        for (int k = 1; k <= NZ - 2; ++k)
            for (int j = 1; j <= NY - 2; ++j)
                for (int i = 1; i <= NX - 2; ++i) {
                    long n = IDX(i, j, k);
                    ro[n] = ro[n] - bx[n] * bx[n] / tt[n] * s->obeta;
                }
    }
    if (p->ampt != 0.0) {
        /* The reference draw order (z-rank, local k, y-rank, plane rows, x fastest) is the
         * global (k, j, i) order for every decomposition. */
        ran2_state st; memset(&st, 0, sizeof st); st.idum = -seed;
        double* w = s->f[ORA_WW1];
        for (int k = 1; k <= NZ - 2; ++k)
            for (int j = 1; j <= NY - 2; ++j)
                for (int i = 1; i <= NX - 2; ++i) w[IDX(i, j, k)] = 1.0 + p->ampt * (ran2(&st) - 0.5);
        for (int k = 1; k <= NZ - 2; ++k)
            for (int j = 1; j <= NY - 2; ++j)
                for (int i = 1; i <= NX - 2; ++i) tt[IDX(i, j, k)] *= w[IDX(i, j, k)];
    }
    free(T); free(R);
    s->timi = 0.0; s->timc = 0.0; s->timt = 0.0; s->nit = 0; s->dt = 0.0; s->umach = 0.0;
    communicate(s);
    return 0;
}

/* ----------------------------------------------------------------- FLUXES --------- */
#define LOOP_INT for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i)
#define OMP _Pragma("omp parallel for schedule(static)")

/* Localized embedded heat loss (itcon 2), 3dmhdsub.f:1799-1821: FT -= TP*OCV[*0.5*(1 +
   TANH(LOG(3)/QFH*(TIMT-TC)))]*RO*EXP(CLN*(EXX-XP)**2)/HH*EXP(CLN*(WYY-YP)**2)/HH*EXP(..ZEE..)/HH
   over the interior, with RI holding 1/rho (the Fortran's RO at that point).  CLN =
   -4.0E00*LOG(2.0E00)/HH/HH and LOG(3.0E00) are single-precision literals; x**2 is x*x; TIMT is
   the time at the start of the step (STEP advances it after the stages). */
static void heat_loss(ora_sim* s, const double* RI, double* FT) {
    const ora_params* p = &s->p;
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
    const int i1 = 1, i2 = NX - 2, j1 = 1, j2 = NY - 2, k1 = 1, k2 = NZ - 2;
    const double *exx = s->line[ORA_EXX], *wyy = s->line[ORA_WYY], *zee = s->line[ORA_ZEE];
    const double cln = F4(-4.0f * logf(2.0f)) / p->hh / p->hh, hh = p->hh, timt = s->timi + s->timc;
    OMP for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
        long n = IDX(i, j, k);
        if (p->tc != 0.0)
            FT[n] = FT[n] - p->tp * s->ocv * 0.5 * (1.0 + tanh(F4(logf(3.0f)) / p->qfh * (timt - p->tc))) * RI[n] *
                                exp(cln * ((exx[i] - p->xp) * (exx[i] - p->xp))) / hh *
                                exp(cln * ((wyy[j] - p->yp) * (wyy[j] - p->yp))) / hh *
                                exp(cln * ((zee[k] - p->zp) * (zee[k] - p->zp))) / hh;
        else
            FT[n] = FT[n] - p->tp * s->ocv * RI[n] * exp(cln * ((exx[i] - p->xp) * (exx[i] - p->xp))) / hh *
                                exp(cln * ((wyy[j] - p->yp) * (wyy[j] - p->yp))) / hh *
                                exp(cln * ((zee[k] - p->zp) * (zee[k] - p->zp))) / hh;
    }
    (void)NZ;
}

/* The heat-loss term alone (added to ft, normally zeros) for the current state: the pin of
   heat_loss against the Fortran block executed statement by statement. */
int ora_heat_loss(ora_sim* s, double* ft) {
    const long n = (long)s->NX * s->NY * s->NZ;
    double* ri = (double*)malloc(sizeof(double) * (size_t)n);
    if (!ri) { set_err("out of memory"); return -1; }
    const double* ro = s->f[ORA_RO];
    for (long q = 0; q < n; ++q) ri[q] = 1.0 / ro[q];
    heat_loss(s, ri, ft);
    free(ri);
    return 0;
}

/* Density diffusion (ID 1 or 2), 3dmhdsub.f:1316-1382, the part of FLUXES after FR's
   continuity terms: the density ghost planes are loaded with their mirror planes (RO(k=0) =
   RO(2), RO(NZ-1) = RO(NZ-3); kept in the state, as the Fortran does), ROM(k) is the horizontal
   mean of every plane (HORIZONTAL_MEAN, 3dmhdsub.f:3160-3186, the uniform grid it requires: the
   interior (j, i) sum in loop order over FLOAT(NPX*NPY), a single rank in y), WW1 = RO - ROM,
   and FR receives DH*ORE*WWZ times its x and y second-difference operators and DV*ORE*WWZ times
   its z one.  WWZ = 1/ROM (ID 1) or exp(CLN*ZEE**2) + exp(CLN*(ZEE-ZMAX)**2) with SGM = 0.1E00
   and CLN = -4.0E00*LOG(2.0E00)/SGM/SGM (ID 2; single-precision literals as written). */
static void density_diffusion(ora_sim* s, double* FR) {
    const ora_params* p = &s->p;
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
    const int i1 = 1, i2 = NX - 2, j1 = 1, j2 = NY - 2, k1 = 1, k2 = NZ - 2;
    double* RO = s->f[ORA_RO];
    double *W1 = s->f[ORA_WW1], *W2 = s->f[ORA_WW2], *W3 = s->f[ORA_WW3];
    const double *dxxdx = s->line[ORA_DXXDX], *d2xxdx2 = s->line[ORA_D2XXDX2];
    const double *dyydy = s->line[ORA_DYYDY], *d2yydy2 = s->line[ORA_D2YYDY2];
    const double *dzzdz = s->line[ORA_DZZDZ], *d2zzdz2 = s->line[ORA_D2ZZDZ2], *zee = s->line[ORA_ZEE];
    const double hx = s->hx, h2x = s->h2x, hy = s->hy, h2y = s->h2y, hz = s->hz, h2z = s->h2z;
    const long sx = 1, sy = NX, sz = (long)NX * NY;
    for (int j = 0; j < NY; ++j) for (int i = 0; i < NX; ++i) {
        RO[IDX(i, j, 0)] = RO[IDX(i, j, 2)];
        RO[IDX(i, j, NZ - 1)] = RO[IDX(i, j, NZ - 3)];
    }
    double* rom = (double*)malloc(sizeof(double) * (size_t)NZ * 2);
    double* wwz = rom + NZ;
    const double cnt = F4((float)(p->npx * p->npy));
    for (int k = 0; k < NZ; ++k) {
        double sum = 0.0;
        for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) sum = sum + RO[IDX(i, j, k)];
        rom[k] = sum / cnt;
    }
    for (int k = 0; k < NZ; ++k) for (int j = 0; j < NY; ++j) for (int i = 0; i < NX; ++i) {
        long n = IDX(i, j, k);
        W1[n] = RO[n] - rom[k];
    }
    if (p->id == 1) {
        for (int k = 0; k < NZ; ++k) wwz[k] = 1.0 / rom[k];
    } else {
        const double sgm = F4(0.1f);
        const double cln = F4(-4.0f * logf(2.0f)) / sgm / sgm;
        for (int k = 0; k < NZ; ++k)
            wwz[k] = exp(cln * (zee[k] * zee[k])) + exp(cln * ((zee[k] - p->zmax) * (zee[k] - p->zmax)));
    }
#define A(F, di, dj, dk) F[n + (di) * sx + (dj) * sy + (dk) * sz]
    if (p->dh != 0.0) {
        for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
            long n = IDX(i, j, k);
            W2[n] = (A(W1, 1, 0, 0) - A(W1, -1, 0, 0)) * hx * d2xxdx2[i] +
                    (A(W1, 1, 0, 0) - 2.0 * W1[n] + A(W1, -1, 0, 0)) * h2x * dxxdx[i] * dxxdx[i];
        }
        for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) {
            const double tmpy1 = hy * d2yydy2[j], tmpy2 = h2y * dyydy[j] * dyydy[j];
            for (int i = i1; i <= i2; ++i) {
                long n = IDX(i, j, k);
                W3[n] = (A(W1, 0, 1, 0) - A(W1, 0, -1, 0)) * tmpy1 +
                        (A(W1, 0, 1, 0) - 2.0 * W1[n] + A(W1, 0, -1, 0)) * tmpy2;
            }
        }
        for (int k = k1; k <= k2; ++k) {
            const double tmp = p->dh * s->ore * wwz[k];
            for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
                long n = IDX(i, j, k);
                FR[n] = FR[n] + (W2[n] + W3[n]) * tmp;
            }
        }
    }
    if (p->dv != 0.0) {
        for (int k = k1; k <= k2; ++k) {
            const double tmpz1 = hz * d2zzdz2[k], tmpz2 = h2z * dzzdz[k] * dzzdz[k];
            for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
                long n = IDX(i, j, k);
                W2[n] = (A(W1, 0, 0, 1) - A(W1, 0, 0, -1)) * tmpz1 +
                        (A(W1, 0, 0, 1) - 2.0 * W1[n] + A(W1, 0, 0, -1)) * tmpz2;
            }
        }
        for (int k = k1; k <= k2; ++k) {
            const double tmp = p->dv * s->ore * wwz[k];
            for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
                long n = IDX(i, j, k);
                FR[n] = FR[n] + W2[n] * tmp;
            }
        }
    }
#undef A
    free(rom);
}

/* The density-diffusion terms alone (added to fr, normally zeros) for the current state, with
   rho in RO (its value at the start of FLUXES): the pin of density_diffusion against the
   Fortran block executed statement by statement.  The state's ghost planes are restored. */
int ora_density_diffusion(ora_sim* s, double* fr) {
    if (s->p.id != 1 && s->p.id != 2) { set_err("ID must be 1 or 2"); return -1; }
    const long plane = (long)s->NX * s->NY;
    double* RO = s->f[ORA_RO];
    double* keep = (double*)malloc(sizeof(double) * (size_t)plane * 2);
    if (!keep) { set_err("out of memory"); return -1; }
    memcpy(keep, RO, sizeof(double) * (size_t)plane);
    memcpy(keep + plane, RO + (s->NZ - 1) * plane, sizeof(double) * (size_t)plane);
    density_diffusion(s, fr);
    memcpy(RO, keep, sizeof(double) * (size_t)plane);
    memcpy(RO + (s->NZ - 1) * plane, keep + plane, sizeof(double) * (size_t)plane);
    free(keep);
    return 0;
}

static void fluxes(ora_sim* s) {
    const ora_params* p = &s->p;
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
    const int i1 = 1, i2 = NX - 2, j1 = 1, j2 = NY - 2, k1 = 1, k2 = NZ - 2;
    double *RU = s->f[ORA_RU], *RV = s->f[ORA_RV], *RW = s->f[ORA_RW], *RO = s->f[ORA_RO], *TT = s->f[ORA_TT];
    double *UU = s->f[ORA_UU], *VV = s->f[ORA_VV], *WW = s->f[ORA_WW];
    double *FU = s->f[ORA_FU], *FV = s->f[ORA_FV], *FW = s->f[ORA_FW], *FR = s->f[ORA_FR], *FT = s->f[ORA_FT];
    double *W1 = s->f[ORA_WW1], *W2 = s->f[ORA_WW2], *W3 = s->f[ORA_WW3];
    const double *dxxdx = s->line[ORA_DXXDX], *d2xxdx2 = s->line[ORA_D2XXDX2];
    const double *dyydy = s->line[ORA_DYYDY], *d2yydy2 = s->line[ORA_D2YYDY2];
    const double *dzzdz = s->line[ORA_DZZDZ], *d2zzdz2 = s->line[ORA_D2ZZDZ2];
    const double *rkapa = s->line[ORA_RKAPA], *dkapa = s->line[ORA_DKAPA];
    const double c13 = s->c13, c43 = s->c43, ore = s->ore;
    const double hx = s->hx, h2x = s->h2x, hy = s->hy, h2y = s->h2y, hz = s->hz, h2z = s->h2z;
    const long sx = 1, sy = NX, sz = (long)NX * NY;
#define A(F, di, dj, dk) F[n + (di) * sx + (dj) * sy + (dk) * sz]
    (void)NZ;

    /* FR: src/fluxes.cpp:87-121 */
    OMP for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) {
        double tmpy = hy * dyydy[j];
        for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k);
            FR[n] = (A(RU, -1, 0, 0) - A(RU, 1, 0, 0)) * hx * dxxdx[i];
            FR[n] -= (A(RV, 0, 1, 0) - A(RV, 0, -1, 0)) * tmpy; } }
    OMP for (int k = k1; k <= k2; ++k) { double tmpz = hz * dzzdz[k];
        for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k);
            W1[n] = (A(RW, 0, 0, 1) - A(RW, 0, 0, -1)) * tmpz; } }
    { double tmpz = hz * dzzdz[k1];
      for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k1);
          W1[n] = (4.0 * A(RW, 0, 0, 1) - A(RW, 0, 0, 2)) * tmpz; } }
    { double tmpz = hz * dzzdz[k2];
      for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k2);
          W1[n] = (A(RW, 0, 0, -2) - 4.0 * A(RW, 0, 0, -1)) * tmpz; } }
    OMP LOOP_INT { long n = IDX(i, j, k); FR[n] -= W1[n]; }
    if (p->id != 0) density_diffusion(s, FR);

    /* buoyancy, pressure, 1/rho, velocities: src/fluxes.cpp:126-166 */
    OMP LOOP_INT { long n = IDX(i, j, k); FW[n] = p->grav * RO[n]; }
    OMP for (long n = 0; n < s->N; ++n) { W1[n] = RO[n] * TT[n]; RO[n] = 1.0 / RO[n]; }
    OMP for (int k = k1; k <= k2; ++k) { double tmpz = hz * dzzdz[k];
        for (int j = j1; j <= j2; ++j) { double tmpy = hy * dyydy[j];
            for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k);
                FW[n] -= (A(W1, 0, 0, 1) - A(W1, 0, 0, -1)) * tmpz;
                FV[n] = (A(W1, 0, -1, 0) - A(W1, 0, 1, 0)) * tmpy;
                FU[n] = (A(W1, -1, 0, 0) - A(W1, 1, 0, 0)) * hx * dxxdx[i]; } } }
    OMP for (long n = 0; n < s->N; ++n) { UU[n] = RU[n] * RO[n]; }
    OMP for (long n = 0; n < s->N; ++n) { VV[n] = RV[n] * RO[n]; }
    OMP for (long n = 0; n < s->N; ++n) { WW[n] = RW[n] * RO[n]; }

    /* momentum advection: src/fluxes.cpp:171-224 */
    double* Fm[3] = {FU, FV, FW};
    double* Rm[3] = {RU, RV, RW};
    for (int c = 0; c < 3; ++c) {
        double* F = Fm[c]; double* R = Rm[c];
        OMP for (int k = k1; k <= k2; ++k) { double tmpz = hz * dzzdz[k];
            for (int j = j1; j <= j2; ++j) { double tmpy = hy * dyydy[j];
                for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k);
                    F[n] -= (A(R, 1, 0, 0) * A(UU, 1, 0, 0) - A(R, -1, 0, 0) * A(UU, -1, 0, 0)) * hx * dxxdx[i];
                    F[n] -= (A(R, 0, 1, 0) * A(VV, 0, 1, 0) - A(R, 0, -1, 0) * A(VV, 0, -1, 0)) * tmpy;
                    F[n] -= (A(R, 0, 0, 1) * A(WW, 0, 0, 1) - A(R, 0, 0, -1) * A(WW, 0, 0, -1)) * tmpz; } } }
    }

    /* energy advection: src/fluxes.cpp:229-243 */
    OMP for (int k = k1; k <= k2; ++k) { double tmpz = hz * dzzdz[k];
        for (int j = j1; j <= j2; ++j) { double tmpy = hy * dyydy[j];
            for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k);
                FT[n] = -1.0 * UU[n] * (A(TT, 1, 0, 0) - A(TT, -1, 0, 0)) * hx * dxxdx[i];
                FT[n] -= VV[n] * (A(TT, 0, 1, 0) - A(TT, 0, -1, 0)) * tmpy;
                FT[n] -= WW[n] * (A(TT, 0, 0, 1) - A(TT, 0, 0, -1)) * tmpz; } } }

    /* thermal diffusion: src/fluxes.cpp:246-276 */
    { const double tmp = s->ocv / s->repr;
      OMP for (int k = k1; k <= k2; ++k) {
        const double tmpz1 = hz * d2zzdz2[k], tmpz2 = h2z * dzzdz[k] * dzzdz[k];
        for (int j = j1; j <= j2; ++j) {
            const double tmpy1 = hy * d2yydy2[j], tmpy2 = h2y * dyydy[j] * dyydy[j];
            for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k);
                FT[n] += ((A(TT, 1, 0, 0) - A(TT, -1, 0, 0)) * hx * d2xxdx2[i] +
                          (A(TT, 1, 0, 0) - 2.0 * TT[n] + A(TT, -1, 0, 0)) * h2x * dxxdx[i] * dxxdx[i]) *
                         RO[n] * tmp * rkapa[k];
                FT[n] += ((A(TT, 0, 1, 0) - A(TT, 0, -1, 0)) * tmpy1 +
                          (A(TT, 0, 1, 0) - 2.0 * TT[n] + A(TT, 0, -1, 0)) * tmpy2) * RO[n] * tmp * rkapa[k];
                FT[n] += ((A(TT, 0, 0, 1) - A(TT, 0, 0, -1)) * tmpz1 +
                          (A(TT, 0, 0, 1) - 2.0 * TT[n] + A(TT, 0, 0, -1)) * tmpz2) * RO[n] * tmp * rkapa[k];
                FT[n] += (A(TT, 0, 0, 1) - A(TT, 0, 0, -1)) * hz * dzzdz[k] * RO[n] * tmp * dkapa[k]; } } } }

    /* localized embedded heat loss (itcon 2), after the diffusion and before the viscous terms
       as in 3dmhdsub.f; RO holds 1/rho at this point (3dmhdsub.f:1405) */
    if (p->itcon == 2) heat_loss(s, RO, FT);

    /* viscous momentum: src/fluxes.cpp:281-320 */
    OMP for (int k = k1; k <= k2; ++k) {
        const double tmpz1 = hz * d2zzdz2[k], tmpz2 = h2z * dzzdz[k] * dzzdz[k];
        for (int j = j1; j <= j2; ++j) {
            const double tmpy1 = hy * d2yydy2[j], tmpy2 = h2y * dyydy[j] * dyydy[j];
            for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k);
                FU[n] += ore * (c43 * ((A(UU, 1, 0, 0) - A(UU, -1, 0, 0)) * hx * d2xxdx2[i] +
                                       (A(UU, 1, 0, 0) - 2.0 * UU[n] + A(UU, -1, 0, 0)) * h2x * dxxdx[i] * dxxdx[i]) +
                                (A(UU, 0, 1, 0) - A(UU, 0, -1, 0)) * tmpy1 +
                                (A(UU, 0, 1, 0) - 2.0 * UU[n] + A(UU, 0, -1, 0)) * tmpy2 +
                                (A(UU, 0, 0, 1) - A(UU, 0, 0, -1)) * tmpz1 +
                                (A(UU, 0, 0, 1) - 2.0 * UU[n] + A(UU, 0, 0, -1)) * tmpz2);
                FV[n] += ore * (((A(VV, 1, 0, 0) - A(VV, -1, 0, 0)) * hx * d2xxdx2[i] +
                                 (A(VV, 1, 0, 0) - 2.0 * VV[n] + A(VV, -1, 0, 0)) * h2x * dxxdx[i] * dxxdx[i]) +
                                c43 * ((A(VV, 0, 1, 0) - A(VV, 0, -1, 0)) * tmpy1 +
                                       (A(VV, 0, 1, 0) - 2.0 * VV[n] + A(VV, 0, -1, 0)) * tmpy2) +
                                (A(VV, 0, 0, 1) - A(VV, 0, 0, -1)) * tmpz1 +
                                (A(VV, 0, 0, 1) - 2.0 * VV[n] + A(VV, 0, 0, -1)) * tmpz2);
                FW[n] += ore * (((A(WW, 1, 0, 0) - A(WW, -1, 0, 0)) * hx * d2xxdx2[i] +
                                 (A(WW, 1, 0, 0) - 2.0 * WW[n] + A(WW, -1, 0, 0)) * h2x * dxxdx[i] * dxxdx[i]) +
                                (A(WW, 0, 1, 0) - A(WW, 0, -1, 0)) * tmpy1 +
                                (A(WW, 0, 1, 0) - 2.0 * WW[n] + A(WW, 0, -1, 0)) * tmpy2 +
                                c43 * ((A(WW, 0, 0, 1) - A(WW, 0, 0, -1)) * tmpz1 +
                                       (A(WW, 0, 0, 1) - 2.0 * WW[n] + A(WW, 0, 0, -1)) * tmpz2)); } } }

    /* viscous heating, p dV, cross terms: src/fluxes.cpp:327-514 */
    OMP for (int k = k1; k <= k2; ++k) for (int j = 0; j < NY; ++j) for (int i = i1; i <= i2; ++i) {
        long n = IDX(i, j, k); W1[n] = (A(UU, 1, 0, 0) - A(UU, -1, 0, 0)) * hx * dxxdx[i]; }
    OMP for (int k = k1; k <= k2; ++k) for (int j = 0; j < NY; ++j) for (int i = i1; i <= i2; ++i) {
        long n = IDX(i, j, k); W2[n] = (A(VV, 1, 0, 0) - A(VV, -1, 0, 0)) * hx * dxxdx[i]; }
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = (A(WW, 1, 0, 0) - A(WW, -1, 0, 0)) * hx * dxxdx[i]; }
    { const double tmp = s->ocv * ore;
      OMP LOOP_INT { long n = IDX(i, j, k);
          FT[n] += (c43 * W1[n] * W1[n] + W2[n] * W2[n] + W3[n] * W3[n]) * RO[n] * tmp; }
      OMP LOOP_INT { long n = IDX(i, j, k); FT[n] -= s->ocv * W1[n] * TT[n]; } }
    { const double tmp = c13 * ore;
      OMP LOOP_INT { long n = IDX(i, j, k); FU[n] += tmp * (A(W2, 0, 1, 0) - A(W2, 0, -1, 0)) * hy * dyydy[j]; }
      OMP LOOP_INT { long n = IDX(i, j, k); FV[n] += tmp * (A(W1, 0, 1, 0) - A(W1, 0, -1, 0)) * hy * dyydy[j]; } }
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = (A(UU, 0, 1, 0) - A(UU, 0, -1, 0)) * hy * dyydy[j]; }
    { const double tmp = s->ocv * ore;
      OMP LOOP_INT { long n = IDX(i, j, k); FT[n] += (W1[n] * W1[n] + 2.0 * W1[n] * W2[n]) * RO[n] * tmp; } }
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = (A(VV, 0, 1, 0) - A(VV, 0, -1, 0)) * hy * dyydy[j]; }
    { const double tmp = c43 * s->ocv * ore;
      OMP LOOP_INT { long n = IDX(i, j, k); FT[n] += W2[n] * W2[n] * RO[n] * tmp; }
      OMP LOOP_INT { long n = IDX(i, j, k); FT[n] -= s->ocv * W2[n] * TT[n]; } }
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = (A(UU, 1, 0, 0) - A(UU, -1, 0, 0)) * hx * dxxdx[i]; }
    OMP for (int k = k1; k <= k2; ++k) for (int j = 0; j < NY; ++j) for (int i = 0; i < NX; ++i) {
        long n = IDX(i, j, k); W3[n] = (A(WW, 0, 0, 1) - A(WW, 0, 0, -1)) * hz * dzzdz[k]; }
    { const double tmp = c43 * s->ocv * ore;
      OMP LOOP_INT { long n = IDX(i, j, k);
          FT[n] += (W3[n] * W3[n] - W1[n] * W3[n] - W1[n] * W2[n] - W2[n] * W3[n]) * RO[n] * tmp; }
      OMP LOOP_INT { long n = IDX(i, j, k); FT[n] -= s->ocv * W3[n] * TT[n]; } }
    { const double tmp = c13 * ore;
      OMP LOOP_INT { long n = IDX(i, j, k); FU[n] += tmp * (A(W3, 1, 0, 0) - A(W3, -1, 0, 0)) * hx * dxxdx[i]; }
      OMP LOOP_INT { long n = IDX(i, j, k); FV[n] += tmp * (A(W3, 0, 1, 0) - A(W3, 0, -1, 0)) * hy * dyydy[j]; } }
    OMP for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) for (int i = 0; i < NX; ++i) {
        long n = IDX(i, j, k); W1[n] = (A(UU, 0, 0, 1) - A(UU, 0, 0, -1)) * hz * dzzdz[k]; }
    OMP for (int k = k1; k <= k2; ++k) for (int j = 0; j < NY; ++j) for (int i = i1; i <= i2; ++i) {
        long n = IDX(i, j, k); W2[n] = (A(VV, 0, 0, 1) - A(VV, 0, 0, -1)) * hz * dzzdz[k]; }
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = (A(WW, 0, 1, 0) - A(WW, 0, -1, 0)) * hy * dyydy[j]; }
    { const double tmp = s->ocv * ore;
      OMP LOOP_INT { long n = IDX(i, j, k);
          FT[n] += (W1[n] * W1[n] + W2[n] * W2[n] + W3[n] * W3[n] + 2.0 * W2[n] * W3[n]) * RO[n] * tmp; } }
    { const double tmp = c13 * ore;
      OMP LOOP_INT { long n = IDX(i, j, k);
          FW[n] += tmp * ((A(W1, 1, 0, 0) - A(W1, -1, 0, 0)) * hx * dxxdx[i] +
                          (A(W2, 0, 1, 0) - A(W2, 0, -1, 0)) * hy * dyydy[j]); } }
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = (A(WW, 1, 0, 0) - A(WW, -1, 0, 0)) * hx * dxxdx[i]; }
    { const double tmp = s->ocv * ore;
      OMP LOOP_INT { long n = IDX(i, j, k); FT[n] += 2.0 * W1[n] * W3[n] * RO[n] * tmp; } }

    /* rotation: src/fluxes.cpp:519-533 */
    if (p->lrot) {
        OMP LOOP_INT { long n = IDX(i, j, k); FU[n] += s->omz * RV[n]; }
        OMP LOOP_INT { long n = IDX(i, j, k); FV[n] += -s->omz * RU[n] + s->omx * RW[n]; }
        OMP LOOP_INT { long n = IDX(i, j, k); FW[n] += -s->omx * RV[n]; }
    }

    if (!p->lmag) return;
    /* MHD: golden/fortran/3dmhdsub.f:2146-2650.  The Fortran reuses RU/RV/RW/TT as
     * interior-only scratch; every scratch value is written and read at the same cell, and
     * STEP overwrites those interiors from ZRU.. right after, so separate scratch arrays give
     * the same numbers.  XU/XV/XW/XT below stand for that scratch. */
    double *XU = s->scr[0], *XV = s->scr[1], *XW = s->scr[2], *XT = s->scr[3];
    double *BX = s->f[ORA_BX], *BY = s->f[ORA_BY], *BZ = s->f[ORA_BZ];
    const double obeta = s->obeta, orm = s->orm, ocv = s->ocv;
#define DX(F) ((A(F, 1, 0, 0) - A(F, -1, 0, 0)) * hx * dxxdx[i])
#define DY(F) ((A(F, 0, 1, 0) - A(F, 0, -1, 0)) * hy * dyydy[j])
#define DZ(F) ((A(F, 0, 0, 1) - A(F, 0, 0, -1)) * hz * dzzdz[k])
#define D2X(F) ((A(F, 1, 0, 0) - A(F, -1, 0, 0)) * hx * d2xxdx2[i] + (A(F, 1, 0, 0) - 2.0 * F[n] + A(F, -1, 0, 0)) * h2x * dxxdx[i] * dxxdx[i])
#define D2Y(F) ((A(F, 0, 1, 0) - A(F, 0, -1, 0)) * hy * d2yydy2[j] + (A(F, 0, 1, 0) - 2.0 * F[n] + A(F, 0, -1, 0)) * h2y * dyydy[j] * dyydy[j])
#define D2Z(F) ((A(F, 0, 0, 1) - A(F, 0, 0, -1)) * hz * d2zzdz2[k] + (A(F, 0, 0, 1) - 2.0 * F[n] + A(F, 0, 0, -1)) * h2z * dzzdz[k] * dzzdz[k])
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = DX(UU); }                                      /* 1000 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = DX(VV); }                                      /* 1010 */
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = DX(WW); }                                      /* 1020 */
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = BX[n] * XV[n] - BY[n] * XU[n]; }               /* 1030 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = BX[n] * XW[n] - BZ[n] * XU[n]; }               /* 1040 */
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = DY(UU); }                                      /* 1050 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = DY(VV); }                                      /* 1060 */
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = DY(WW); }                                      /* 1070 */
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = BY[n] * XU[n] - BX[n] * XV[n]; }               /* 1080 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = W3[n] + BY[n] * XW[n] - BZ[n] * XV[n]; }       /* 1090 */
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = DZ(UU); }                                      /* 1100 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = DZ(VV); }                                      /* 1110 */
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = DZ(WW); }                                      /* 1120 */
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {                                /* 1125 */
        long n = IDX(i, j, k1); XW[n] = (4.0 * A(WW, 0, 0, 1) - A(WW, 0, 0, 2)) * hz * dzzdz[k1]; }
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {                                /* 1126 */
        long n = IDX(i, j, k2); XW[n] = (A(WW, 0, 0, -2) - 4.0 * A(WW, 0, 0, -1)) * hz * dzzdz[k2]; }
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = W1[n] + BZ[n] * XU[n] - BX[n] * XW[n]; }       /* 1130 */
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = W2[n] + BZ[n] * XV[n] - BY[n] * XW[n]; }       /* 1140 */
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = DX(BX); }                                      /* 1150 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = DX(BY); }                                      /* 1160 */
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = DX(BZ); }                                      /* 1170 */
    OMP LOOP_INT { long n = IDX(i, j, k); XT[n] = DY(BX); }                                      /* 1180 */
    OMP LOOP_INT { long n = IDX(i, j, k); FU[n] = FU[n] + obeta * BY[n] * (XT[n] - XV[n]) - obeta * BZ[n] * XW[n]; } /* 1190 */
    OMP LOOP_INT { long n = IDX(i, j, k); FV[n] = FV[n] + obeta * BX[n] * (XV[n] - XT[n]); }     /* 1200 */
    OMP LOOP_INT { long n = IDX(i, j, k); FW[n] = FW[n] + obeta * BX[n] * XW[n]; }               /* 1210 */
    { const double tmp = obeta * orm * ocv;                                                        /* 1220 */
      OMP LOOP_INT { long n = IDX(i, j, k);
          FT[n] = FT[n] + (XT[n] * XT[n] + XV[n] * XV[n] + XW[n] * XW[n] - 2.0 * XV[n] * XT[n]) * RO[n] * tmp; } }
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = W1[n] - UU[n] * XU[n] - VV[n] * XT[n]; }       /* 1230 */
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = W2[n] - UU[n] * XV[n]; }                       /* 1240 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = W3[n] - UU[n] * XW[n]; }                       /* 1250 */
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = D2X(BX); }                                     /* 1260 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = D2X(BY); }                                     /* 1265 */
    OMP LOOP_INT { long n = IDX(i, j, k); XT[n] = D2Y(BX); }                                     /* 1270 */
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = W1[n] + orm * (XU[n] + XT[n]); }               /* 1280 */
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = W2[n] + orm * XV[n]; }                         /* 1290 */
    OMP LOOP_INT { long n = IDX(i, j, k); XT[n] = D2X(BZ); }                                     /* 1300 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = W3[n] + orm * XT[n]; }                         /* 1310 */
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = DZ(BX); }                                      /* 1320 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = DY(BY); }                                      /* 1330 */
    OMP LOOP_INT { long n = IDX(i, j, k); FU[n] = FU[n] + obeta * BZ[n] * XU[n]; }               /* 1340 */
    OMP LOOP_INT { long n = IDX(i, j, k); FW[n] = FW[n] - obeta * BX[n] * XU[n]; }               /* 1350 */
    { const double tmp = obeta * orm * ocv;                                                        /* 1360 */
      OMP LOOP_INT { long n = IDX(i, j, k);
          FT[n] = FT[n] + (XU[n] * XU[n] - 2.0 * XU[n] * XW[n]) * RO[n] * tmp; } }
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = W1[n] - WW[n] * XU[n]; }                       /* 1370 */
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = W2[n] - VV[n] * XV[n]; }                       /* 1380 */
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = D2Z(BX); }                                     /* 1390 */
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {                                /* 1391 */
        long n = IDX(i, j, k1);
        XU[n] = (-3.0 * BX[n] + 4.0 * A(BX, 0, 0, 1) - A(BX, 0, 0, 2)) * hz * d2zzdz2[k1] +
                (2.0 * BX[n] - 5.0 * A(BX, 0, 0, 1) + 4.0 * A(BX, 0, 0, 2) - A(BX, 0, 0, 3)) * h2z * dzzdz[k1] * dzzdz[k1]; }
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {                                /* 1392 */
        long n = IDX(i, j, k2);
        XU[n] = (3.0 * BX[n] - 4.0 * A(BX, 0, 0, -1) + A(BX, 0, 0, -2)) * hz * d2zzdz2[k2] +
                (2.0 * BX[n] - 5.0 * A(BX, 0, 0, -1) + 4.0 * A(BX, 0, 0, -2) - A(BX, 0, 0, -3)) * h2z * dzzdz[k2] * dzzdz[k2]; }
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = D2Y(BY); }                                     /* 1400 */
    OMP LOOP_INT { long n = IDX(i, j, k); W1[n] = W1[n] + orm * XU[n]; }                         /* 1410 */
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = W2[n] + orm * XV[n]; }                         /* 1420 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = DZ(BY); }                                      /* 1430 */
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = DY(BZ); }                                      /* 1440 */
    OMP LOOP_INT { long n = IDX(i, j, k); XU[n] = XV[n] - XW[n]; }                               /* 1450 */
    OMP LOOP_INT { long n = IDX(i, j, k); FV[n] = FV[n] + obeta * BZ[n] * XU[n]; }               /* 1460 */
    OMP LOOP_INT { long n = IDX(i, j, k); FW[n] = FW[n] - obeta * BY[n] * XU[n]; }               /* 1470 */
    { const double tmp = obeta * orm * ocv;                                                        /* 1480 */
      OMP LOOP_INT { long n = IDX(i, j, k);
          FT[n] = FT[n] + (XV[n] * XV[n] + XW[n] * XW[n] - 2.0 * XV[n] * XW[n]) * RO[n] * tmp; } }
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = W2[n] - WW[n] * XV[n]; }                       /* 1490 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = W3[n] - VV[n] * XW[n]; }                       /* 1500 */
    OMP LOOP_INT { long n = IDX(i, j, k); XV[n] = D2Z(BY); }                                     /* 1510 */
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {                                /* 1511 */
        long n = IDX(i, j, k1);
        XV[n] = (-3.0 * BY[n] + 4.0 * A(BY, 0, 0, 1) - A(BY, 0, 0, 2)) * hz * d2zzdz2[k1] +
                (2.0 * BY[n] - 5.0 * A(BY, 0, 0, 1) + 4.0 * A(BY, 0, 0, 2) - A(BY, 0, 0, 3)) * h2z * dzzdz[k1] * dzzdz[k1]; }
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {                                /* 1513 */
        long n = IDX(i, j, k2);
        XV[n] = (3.0 * BY[n] - 4.0 * A(BY, 0, 0, -1) + A(BY, 0, 0, -2)) * hz * d2zzdz2[k2] +
                (2.0 * BY[n] - 5.0 * A(BY, 0, 0, -1) + 4.0 * A(BY, 0, 0, -2) - A(BY, 0, 0, -3)) * h2z * dzzdz[k2] * dzzdz[k2]; }
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = D2Y(BZ); }                                     /* 1520 */
    OMP LOOP_INT { long n = IDX(i, j, k); W2[n] = W2[n] + orm * XV[n]; }                         /* 1530 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = W3[n] + orm * XW[n]; }                         /* 1540 */
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = DZ(BZ); }                                      /* 1550 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = W3[n] - WW[n] * XW[n]; }                       /* 1560 */
    OMP LOOP_INT { long n = IDX(i, j, k); XW[n] = D2Z(BZ); }                                     /* 1570 */
    OMP LOOP_INT { long n = IDX(i, j, k); W3[n] = W3[n] + orm * XW[n]; }                         /* 1580 */
#undef DX
#undef DY
#undef DZ
#undef D2X
#undef D2Y
#undef D2Z
#undef A
}

int ora_fluxes(ora_sim* s) { fluxes(s); return 0; }
void ora_communicate(ora_sim* s) { communicate(s); }

/* ------------------------------------------------------------------- BCON --------- */
/* src/bcon.cpp:12-141 for the global top (k=1) and bottom (k=npz) planes. */
static int bcon(ora_sim* s) {
    const ora_params* p = &s->p;
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
    const int i1 = 1, i2 = NX - 2, j1 = 1, j2 = NY - 2, k1 = 1, k2 = NZ - 2;
    const double c13 = s->c13, c23 = s->c23, c43 = s->c43;
    const double timt = s->timc + s->timi;
    double *ru = s->f[ORA_RU], *rv = s->f[ORA_RV], *rw = s->f[ORA_RW], *ro = s->f[ORA_RO], *tt = s->f[ORA_TT];
    const double *exx = s->line[ORA_EXX], *wyy = s->line[ORA_WYY], *dzzdz = s->line[ORA_DZZDZ];
    const long sz = (long)NX * NY;
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k1);
        ru[n] = ro[n] * (c43 * ru[n + sz] / ro[n + sz] - c13 * ru[n + 2 * sz] / ro[n + 2 * sz]); }
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k1);
        rv[n] = ro[n] * (c43 * rv[n + sz] / ro[n + sz] - c13 * rv[n + 2 * sz] / ro[n + 2 * sz]); }
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) rw[IDX(i, j, k1)] = 0.0;
    if ((p->tp != 0.0) && (p->itcon == 0 || p->itcon == 1)) {
        double tpr = (p->tc != 0.0) ? p->tp + (1.0 - p->tp) * exp(-timt / p->tc) : p->tp;
        const double cln = F4(-4.0f * logf(2.0f)) / (p->hh * p->hh);
        if (p->itcon == 0) {
            for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i)
                tt[IDX(i, j, k1)] = 1.0 - (1.0 - tpr) * exp(cln * (exx[i] - p->xp) * (exx[i] - p->xp)) / p->hh *
                                              exp(cln * (wyy[j] - p->yp) * (wyy[j] - p->yp)) / p->hh;
        } else {
            const double dz = F4(1.0f / (float)(p->npz - 1)) / dzzdz[k1];
            for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k1);
                tt[n] = c43 * tt[n + sz] - c13 * tt[n + 2 * sz] -
                        c23 * dz * (p->theta - (p->theta - tpr) * exp(cln * ((exx[i] - p->xp) * (exx[i] - p->xp))) / p->hh *
                                                   exp(cln * ((wyy[j] - p->yp) * (wyy[j] - p->yp))) / p->hh); }
        }
    } else {
        if (p->itcon == 0 || p->itcon == 2 || p->itcon == 4) {
            for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
                long n = IDX(i, j, k1);
                tt[n] = 1.0;
                if (p->itcon == 4 && i <= NX / 2) tt[n] = 1.0 - p->tp;
            }
        }
        if (p->itcon == 1) {
            const double dz = F4(1.0f / (float)(p->npz - 1)) / dzzdz[k1];
            for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k1);
                tt[n] = c43 * tt[n + sz] - c13 * tt[n + 2 * sz] - c23 * dz * p->theta; }
        }
    }
    if (p->lmag && p->ibcon == 0)
        for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) s->f[ORA_BZ][IDX(i, j, k1)] = 0.0;

    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k2);
        ru[n] = ro[n] * (c43 * ru[n - sz] / ro[n - sz] - c13 * ru[n - 2 * sz] / ro[n - 2 * sz]); }
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k2);
        rv[n] = ro[n] * (c43 * rv[n - sz] / ro[n - sz] - c13 * rv[n - 2 * sz] / ro[n - 2 * sz]); }
    for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) rw[IDX(i, j, k2)] = 0.0;
    if (p->izcon == 0) {
        for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) tt[IDX(i, j, k2)] = s->tb;
    } else if (p->izcon == 1) {
        const double dz = F4(1.0f / (float)(p->npz - 1)) / dzzdz[k2];
        for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) { long n = IDX(i, j, k2);
            tt[n] = c43 * tt[n - sz] - c13 * tt[n - 2 * sz] + c23 * dz * p->theta / s->line[ORA_RKAPA][k2]; }
    } else {
        set_err("invalid IZCON");
        return -1;
    }
    if (p->lmag && p->ibcon == 0)
        for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) s->f[ORA_BZ][IDX(i, j, k2)] = 0.0;
    return 0;
}

/* ------------------------------------------------------------------- STEP --------- */
/* src/step.cpp:114-257 (+ B terms of 3dmhdsub.f STEP when lmag). */
int ora_step(ora_sim* s, int nstages) {
    const ora_params* p = &s->p;
    if (p->lshr || p->lrem || p->rlax > 0.0 || (p->id != 0 && (p->ngrid != 0 || (p->id != 1 && p->id != 2))) ||
        p->ixcon != 0 || p->iycon != 0) { set_err("unsupported FLUXES feature"); return -1; }
    const int NX = s->NX, NY = s->NY, NZ = s->NZ;
    const int i1 = 1, i2 = NX - 2, j1 = 1, j2 = NY - 2, k1 = 1, k2 = NZ - 2;
    double *ru = s->f[ORA_RU], *rv = s->f[ORA_RV], *rw = s->f[ORA_RW], *ro = s->f[ORA_RO], *tt = s->f[ORA_TT];
    double *uu = s->f[ORA_UU], *vv = s->f[ORA_VV];
    double *w1 = s->f[ORA_WW1], *w2 = s->f[ORA_WW2], *w3 = s->f[ORA_WW3];
    double *bx = s->f[ORA_BX], *by = s->f[ORA_BY], *bz = s->f[ORA_BZ];
    const double *ddx = s->line[ORA_DDX], *ddy = s->line[ORA_DDY], *ddz = s->line[ORA_DDZ];
    const double *rkapa = s->line[ORA_RKAPA];
    const double sff = p->sf, ogamma = 1.0 / p->gamma;

    OMP LOOP_INT { long n = IDX(i, j, k);
        uu[n] = (ru[n] * ru[n] + rv[n] * rv[n] + rw[n] * rw[n]) * (1.0 / ro[n]) * (1.0 / ro[n]); }
    double um = 0.0;
    LOOP_INT { long n = IDX(i, j, k); double v = ogamma * uu[n] / tt[n]; um = (um < v) ? v : um; }
    s->umach = sqrt(um);
    if (p->lmag) {
        OMP LOOP_INT { long n = IDX(i, j, k);
            double b2 = (bx[n] * bx[n] + by[n] * by[n] + bz[n] * bz[n]) * s->obeta / ro[n];
            uu[n] = uu[n] + p->gamma * tt[n] + b2 + 2.0 * sqrt(uu[n] * (p->gamma * tt[n] + b2)); }
    } else {
        OMP LOOP_INT { long n = IDX(i, j, k);
            uu[n] = uu[n] + p->gamma * tt[n] + 2.0 * sqrt(uu[n] * p->gamma * tt[n]); }
    }
    OMP LOOP_INT { long n = IDX(i, j, k);
        double a = ddx[i], b = ddy[j], c = ddz[k];
        double m = (b < a) ? b : a;
        double dd = (c < m) ? c : m;
        w1[n] = dd / sqrt(uu[n]);
        w2[n] = 0.5 * dd * dd * s->repr * s->cv * ro[n] / rkapa[k];
        w3[n] = 0.375 * dd * dd * p->re * ro[n];
        if (p->lmag) vv[n] = 0.5 * dd * dd * p->rm; }
    double m0 = 1e300, m1 = 1e300, m2 = 1e300, m3 = 1e300;
    LOOP_INT { long n = IDX(i, j, k);
        m0 = (w1[n] < m0) ? w1[n] : m0; m1 = (w2[n] < m1) ? w2[n] : m1; m2 = (w3[n] < m2) ? w3[n] : m2;
        if (p->lmag) m3 = (vv[n] < m3) ? vv[n] : m3; }
    double a = (m1 < m0) ? m1 : m0;
    a = (m2 < a) ? m2 : a;
    if (p->lmag) a = (m3 < a) ? m3 : a;
    s->dt = sff * a;

    double* X[8] = {ru, rv, rw, ro, tt, bx, by, bz};
    double* Z[8] = {s->f[ORA_ZRU], s->f[ORA_ZRV], s->f[ORA_ZRW], s->f[ORA_ZRO], s->f[ORA_ZTT],
                    s->f[ORA_ZBX], s->f[ORA_ZBY], s->f[ORA_ZBZ]};
    double* F[8] = {s->f[ORA_FU], s->f[ORA_FV], s->f[ORA_FW], s->f[ORA_FR], s->f[ORA_FT], w1, w2, w3};
    const int nv = p->lmag ? 8 : 5;
    for (int q = 0; q < nv; ++q) { double *x = X[q], *z = Z[q]; OMP LOOP_INT { long n = IDX(i, j, k); z[n] = x[n]; } }
    const double gam[3] = {s->gam1, s->gam2, s->gam3};
    const double zeta[3] = {0.0, s->zeta1, s->zeta2};
    for (int st = 0; st < nstages; ++st) {
        if (st > 0) {
            const double coef = zeta[st] * s->dt;
            for (int q = 0; q < nv; ++q) { double *x = X[q], *z = Z[q], *f = F[q];
                OMP LOOP_INT { long n = IDX(i, j, k); z[n] = x[n] + coef * f[n]; } }
        }
        fluxes(s);
        const double coef = gam[st] * s->dt;
        for (int q = 0; q < nv; ++q) { double *x = X[q], *z = Z[q], *f = F[q];
            OMP LOOP_INT { long n = IDX(i, j, k); x[n] = z[n] + coef * f[n]; } }
        if (bcon(s) != 0) return -1;
        communicate(s);
    }
    s->nit += 1;
    s->timc += s->dt;
    s->timt = s->timi + s->timc;
    return 0;
}
