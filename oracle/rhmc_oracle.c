/*
 * rhmc_oracle.c -- CPU restatement of the RHMC hot path, TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA path: only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg load it.  Nothing in the product library links, calls or
 * falls back to it.
 *
 * It restates, in plain C with runtime lattice sizes, the FP64 CPU algorithms of
 * coppolachan/RHMC-on-GPU (each function cites the reference file:line it follows) using
 * the reference's own data layouts:
 *   links    double[4*V][3][3][2]   index mu*V + site, site in even/odd order (u_work)
 *   spinor   double[Vh][3][2]       one parity (Fermion)
 *   algebra  double[4*V][3][3][2]   full 3x3 complex (Momenta / Ipdot)
 * and the reference's operation order (so that, compiled without FMA contraction, its
 * results agree with the reference binary to the last bit or within a few ulp).
 *
 * Parity of this restatement is pinned against the reference itself: oracle/build_ref.py
 * compiles the unmodified reference CPU sources with a harness into oracle/_ref/ and
 * tests/golden/make_golden.py records their outputs as fixtures.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b) { cplx r; r.re = a.re * b.re - a.im * b.im; r.im = a.re * b.im + a.im * b.re; return r; }
static inline cplx cadd(cplx a, cplx b) { cplx r = { a.re + b.re, a.im + b.im }; return r; }
static inline cplx csub(cplx a, cplx b) { cplx r = { a.re - b.re, a.im - b.im }; return r; }
static inline cplx cconj(cplx a) { cplx r = { a.re, -a.im }; return r; }
static inline cplx cscal(double s, cplx a) { cplx r = { a.re * s, a.im * s }; return r; }

typedef struct { cplx c[3][3]; } su3;
typedef struct { cplx c[3]; } vec3;

/* ---------------------------------------------------------------- lattice state */
static int g_nx, g_ny, g_nz, g_nt, g_bc;
static long g_V, g_Vh;
static long *g_nnp, *g_nnm;   /* [V][4] */
static int *g_eta;            /* [4V]   */

/* snum: lib/Main/Geometry/geometry.cc:5-11 */
static long snum(int x, int y, int z, int t)
{
    long r = x + (long)y * g_nx + (long)z * g_nx * g_ny + (long)t * g_nx * g_ny * g_nz;
    return r / 2;
}

/* init_geo: lib/Main/Geometry/geometry.cc:26-161 (nnp/nnm periodic, eta with antiperiodic t
 * for the fermions when bc == 0). */
int orc_init(int nx, int ny, int nz, int nt, int bc)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || nt <= 0 || (nx & 1) || (ny & 1) || (nz & 1) || (nt & 1)) return -1;
    free(g_nnp); free(g_nnm); free(g_eta);
    g_nx = nx; g_ny = ny; g_nz = nz; g_nt = nt; g_bc = bc;
    g_V = (long)nx * ny * nz * nt; g_Vh = g_V / 2;
    g_nnp = (long *)malloc(sizeof(long) * 4 * g_V);
    g_nnm = (long *)malloc(sizeof(long) * 4 * g_V);
    g_eta = (int *)malloc(sizeof(int) * 4 * g_V);
    for (int t = 0; t < nt; t++) {
        int tp = (t == nt - 1) ? 0 : t + 1, tm = (t == 0) ? nt - 1 : t - 1;
        for (int z = 0; z < nz; z++) {
            int zp = (z == nz - 1) ? 0 : z + 1, zm = (z == 0) ? nz - 1 : z - 1;
            for (int y = 0; y < ny; y++) {
                int yp = (y == ny - 1) ? 0 : y + 1, ym = (y == 0) ? ny - 1 : y - 1;
                for (int x = 0; x < nx; x++) {
                    int xp = (x == nx - 1) ? 0 : x + 1, xm = (x == 0) ? nx - 1 : x - 1;
                    int par = (x + y + z + t) % 2;
                    long num = par * g_Vh + snum(x, y, z, t);
                    long o = (1 - par) * g_Vh;
                    g_nnp[num * 4 + 0] = o + snum(xp, y, z, t); g_nnm[num * 4 + 0] = o + snum(xm, y, z, t);
                    g_nnp[num * 4 + 1] = o + snum(x, yp, z, t); g_nnm[num * 4 + 1] = o + snum(x, ym, z, t);
                    g_nnp[num * 4 + 2] = o + snum(x, y, zp, t); g_nnm[num * 4 + 2] = o + snum(x, y, zm, t);
                    g_nnp[num * 4 + 3] = o + snum(x, y, z, tp); g_nnm[num * 4 + 3] = o + snum(x, y, z, tm);
                    g_eta[num] = 1;
                    g_eta[num + g_V] = (x % 2 == 0) ? 1 : -1;
                    g_eta[num + 2 * g_V] = ((x + y) % 2 == 0) ? 1 : -1;
                    g_eta[num + 3 * g_V] = ((x + y + z) % 2 == 0) ? 1 : -1;
                    if (bc == 0 && t == nt - 1) g_eta[num + 3 * g_V] = -g_eta[num + 3 * g_V];
                }
            }
        }
    }
    return 0;
}

long orc_volume(void) { return g_V; }

/* make_shift_table: lib/Tools/Packer/packer.cc:415-439 (nnm mu0..3 then nnp mu0..3, int[8V]) */
void orc_tables(int *table, int *eta)
{
    for (long i = 0; i < g_V; i++)
        for (int mu = 0; mu < 4; mu++) {
            table[i + mu * g_V] = (int)g_nnm[i * 4 + mu];
            table[i + (4 + mu) * g_V] = (int)g_nnp[i * 4 + mu];
        }
    if (eta) memcpy(eta, g_eta, sizeof(int) * 4 * g_V);
}

/* ---------------------------------------------------------------- SU(3) algebra */
/* matrix*vector: lib/Action/su3.h:489-509 (column-by-column accumulation) */
static vec3 su3_mul_vec(const su3 *m, const vec3 *v)
{
    vec3 r;
    for (int i = 0; i < 3; i++) r.c[i] = cmul(v->c[0], m->c[i][0]);
    for (int i = 0; i < 3; i++) r.c[i] = cadd(r.c[i], cmul(v->c[1], m->c[i][1]));
    for (int i = 0; i < 3; i++) r.c[i] = cadd(r.c[i], cmul(v->c[2], m->c[i][2]));
    return r;
}

/* operator~ (hermitian conjugate): su3.h:109-126 */
static su3 su3_dag(const su3 *m)
{
    su3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.c[i][j] = cconj(m->c[j][i]);
    return r;
}

/* a *= b (a = a*b): su3.h:251-305, column by column */
static void su3_mulassign(su3 *a, const su3 *b)
{
    su3 aux = *a;
    for (int j = 0; j < 3; j++) {
        cplx p0 = b->c[0][j], p1 = b->c[1][j], p2 = b->c[2][j];
        for (int i = 0; i < 3; i++) a->c[i][j] = cmul(p0, aux.c[i][0]);
        for (int i = 0; i < 3; i++) a->c[i][j] = cadd(a->c[i][j], cmul(p1, aux.c[i][1]));
        for (int i = 0; i < 3; i++) a->c[i][j] = cadd(a->c[i][j], cmul(p2, aux.c[i][2]));
    }
}

static void su3_scal_assign(su3 *a, double s)
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a->c[i][j] = cscal(s, a->c[i][j]);
}

static void su3_cscal_assign(su3 *a, cplx s)
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a->c[i][j] = cmul(a->c[i][j], s);
}

static void su3_addassign(su3 *a, const su3 *b)
{
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) a->c[i][j] = cadd(a->c[i][j], b->c[i][j]);
}

static void su3_one(su3 *a)
{
    memset(a, 0, sizeof(*a));
    a->c[0][0].re = a->c[1][1].re = a->c[2][2].re = 1.0;
}

/* sunitarize: lib/Action/su3.cc:69-112 (normalise row 0, Gram-Schmidt row 1, row 2 = conj(r0 x r1)) */
static void su3_sunitarize(su3 *m)
{
    double norm = 0.0;
    for (int i = 0; i < 3; i++) norm += m->c[0][i].re * m->c[0][i].re + m->c[0][i].im * m->c[0][i].im;
    norm = 1.0 / sqrt(norm);
    for (int i = 0; i < 3; i++) m->c[0][i] = cscal(norm, m->c[0][i]);
    cplx prod = { 0.0, 0.0 };
    for (int i = 0; i < 3; i++) prod = cadd(prod, cmul(cconj(m->c[0][i]), m->c[1][i]));
    for (int i = 0; i < 3; i++) m->c[1][i] = csub(m->c[1][i], cmul(prod, m->c[0][i]));
    norm = 0.0;
    for (int i = 0; i < 3; i++) norm += m->c[1][i].re * m->c[1][i].re + m->c[1][i].im * m->c[1][i].im;
    norm = 1.0 / sqrt(norm);
    for (int i = 0; i < 3; i++) m->c[1][i] = cscal(norm, m->c[1][i]);
    prod = csub(cmul(m->c[0][1], m->c[1][2]), cmul(m->c[0][2], m->c[1][1]));
    m->c[2][0] = cconj(prod);
    prod = csub(cmul(m->c[0][2], m->c[1][0]), cmul(m->c[0][0], m->c[1][2]));
    m->c[2][1] = cconj(prod);
    prod = csub(cmul(m->c[0][0], m->c[1][1]), cmul(m->c[0][1], m->c[1][0]));
    m->c[2][2] = cconj(prod);
}

/* ta (traceless anti-hermitian part): lib/Action/su3.cc:161-183 */
static void su3_ta(su3 *m)
{
    su3 aux = *m;
    cplx trace = { 0.0, 0.0 };
    const cplx half = { 0.5, 0.0 };
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) m->c[i][j] = cmul(csub(aux.c[i][j], cconj(aux.c[j][i])), half);
        trace = cadd(trace, m->c[i][i]);
    }
    trace = cmul(trace, (cplx){ 0.3333333333333333333333333333333, 0.0 });
    for (int i = 0; i < 3; i++) m->c[i][i] = csub(m->c[i][i], trace);
}

/* exp: lib/Action/su3.cc:187-219 (6th-order Taylor, then sunitarize) */
static void su3_exp(su3 *m)
{
    su3 aux, ris;
    su3_one(&ris);
    aux = *m;
    su3_addassign(&ris, &aux);
    su3_mulassign(&aux, m); su3_scal_assign(&aux, 0.5); su3_addassign(&ris, &aux);
    su3_mulassign(&aux, m); su3_scal_assign(&aux, 0.3333333333333333333333333333333); su3_addassign(&ris, &aux);
    su3_mulassign(&aux, m); su3_scal_assign(&aux, 0.25); su3_addassign(&ris, &aux);
    su3_mulassign(&aux, m); su3_scal_assign(&aux, 0.2); su3_addassign(&ris, &aux);
    su3_mulassign(&aux, m); su3_scal_assign(&aux, 0.166666666666666666); su3_addassign(&ris, &aux);
    su3_sunitarize(&ris);
    *m = ris;
}

static double su3_retr(const su3 *m) { return m->c[0][0].re + m->c[1][1].re + m->c[2][2].re; }

/* operator^ (outer product, no conjugation): su3.h:513-530 */
static su3 vec_outer(const vec3 *a, const vec3 *b)
{
    su3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.c[i][j] = cmul(a->c[i], b->c[j]);
    return r;
}

static vec3 vec_conj(const vec3 *a) { vec3 r; for (int i = 0; i < 3; i++) r.c[i] = cconj(a->c[i]); return r; }

/* l2norm2 of a Vec3 and r_scalprod: lib/Tools/vec3.h:240-250 */
static double vec_l2norm2(const vec3 *a)
{
    double s = 0.0;
    for (int i = 0; i < 3; i++) s += a->c[i].re * a->c[i].re + a->c[i].im * a->c[i].im;
    return s;
}

static double vec_rscal(const vec3 *a, const vec3 *b)
{
    cplx r = { 0.0, 0.0 };
    for (int i = 0; i < 3; i++) r = cadd(r, cmul(cconj(a->c[i]), b->c[i]));
    return r.re;
}

/* global_sum: include/tools.h:25-57 (pairwise tree sum; destroys vec) */
static void global_sum(double *vec, long n)
{
    while (n > 1) {
        if (n % 2 == 0) {
            long j = n / 2;
            for (long k = 0; k < j; k++) vec[k] += vec[k + j];
            n = j;
        } else {
            long j1 = n / 2, j2 = j1 + 1;
            for (long k = 0; k < j1; k++) vec[k] += vec[k + j2];
            n = j2;
        }
    }
}

/* ---------------------------------------------------------------- Dslash */
/* Deo: lib/Action/fermionmatrix.cc:8-50.  out_e(x) = 1/2 sum_mu [U_mu(x) in(x+mu) - U_mu(x-mu)^dag in(x-mu)] */
void orc_deo(double *out_, const double *in_, const double *u_)
{
    vec3 *out = (vec3 *)out_;
    const vec3 *in = (const vec3 *)in_;
    const su3 *u = (const su3 *)u_;
    for (long e = 0; e < g_Vh; e++) {
        vec3 aux = su3_mul_vec(&u[e], &in[g_nnp[e * 4 + 0] - g_Vh]);
        for (int mu = 1; mu < 4; mu++) {
            vec3 t = su3_mul_vec(&u[e + mu * g_V], &in[g_nnp[e * 4 + mu] - g_Vh]);
            for (int c = 0; c < 3; c++) aux.c[c] = cadd(aux.c[c], t.c[c]);
        }
        for (int mu = 0; mu < 4; mu++) {
            su3 ud = su3_dag(&u[g_nnm[e * 4 + mu] + mu * g_V]);
            vec3 t = su3_mul_vec(&ud, &in[g_nnm[e * 4 + mu] - g_Vh]);
            for (int c = 0; c < 3; c++) aux.c[c] = csub(aux.c[c], t.c[c]);
        }
        for (int c = 0; c < 3; c++) aux.c[c] = cscal(0.5, aux.c[c]);
        out[e] = aux;
    }
}

/* Doe: lib/Action/fermionmatrix.cc:58-97 */
void orc_doe(double *out_, const double *in_, const double *u_)
{
    vec3 *out = (vec3 *)out_;
    const vec3 *in = (const vec3 *)in_;
    const su3 *u = (const su3 *)u_;
    for (long o = g_Vh; o < g_V; o++) {
        vec3 aux = su3_mul_vec(&u[o], &in[g_nnp[o * 4 + 0]]);
        for (int mu = 1; mu < 4; mu++) {
            vec3 t = su3_mul_vec(&u[o + mu * g_V], &in[g_nnp[o * 4 + mu]]);
            for (int c = 0; c < 3; c++) aux.c[c] = cadd(aux.c[c], t.c[c]);
        }
        for (int mu = 0; mu < 4; mu++) {
            su3 ud = su3_dag(&u[g_nnm[o * 4 + mu] + mu * g_V]);
            vec3 t = su3_mul_vec(&ud, &in[g_nnm[o * 4 + mu]]);
            for (int c = 0; c < 3; c++) aux.c[c] = csub(aux.c[c], t.c[c]);
        }
        for (int c = 0; c < 3; c++) aux.c[c] = cscal(0.5, aux.c[c]);
        out[o - g_Vh] = aux;
    }
}

/* (M^dag M + shift) x = (mass^2 + shift) x - Deo Doe x: lib/Action/Inverter/inverter.cc:3, 206-216 */
void orc_mdagm(double *out_, const double *in_, const double *u_, double mass, double shift)
{
    vec3 *h = (vec3 *)malloc(sizeof(vec3) * g_Vh);
    vec3 *s = (vec3 *)malloc(sizeof(vec3) * g_Vh);
    orc_doe((double *)h, in_, u_);
    orc_deo((double *)s, (double *)h, u_);
    const vec3 *in = (const vec3 *)in_;
    vec3 *out = (vec3 *)out_;
    double m2 = mass * mass + shift;
    for (long i = 0; i < g_Vh; i++)
        for (int c = 0; c < 3; c++) out[i].c[c] = csub(cscal(m2, in[i].c[c]), s[i].c[c]);
    free(h); free(s);
}

/* ---------------------------------------------------------------- multi-shift CG */
/* multips_shifted_invert, one pseudofermion: lib/Action/Inverter/inverter.cc:142-299.
 * x: [nshift][Vh] spinors (output), b: [Vh] spinor.  Returns the iteration count.
 * Stops on sqrt(|r|^2) <= res (absolute, base unshifted system) or cg == max_cg; a shift
 * is frozen when sqrt(delta*zeta^2) < res with the lagged residual, as the reference does. */
int orc_msolve(double *x_, const double *b_, const double *u_, double mass,
               int nshift, const double *shifts, double res, int max_cg)
{
    const vec3 *b = (const vec3 *)b_;
    vec3 *x = (vec3 *)x_;
    long Vh = g_Vh;
    double mass2 = mass * mass;
    vec3 *r = (vec3 *)malloc(sizeof(vec3) * Vh), *p = (vec3 *)malloc(sizeof(vec3) * Vh);
    vec3 *h = (vec3 *)malloc(sizeof(vec3) * Vh), *s = (vec3 *)malloc(sizeof(vec3) * Vh);
    vec3 *ps = (vec3 *)malloc(sizeof(vec3) * Vh * nshift);
    double *dv = (double *)malloc(sizeof(double) * Vh);
    double *zi = malloc(sizeof(double) * nshift), *zii = malloc(sizeof(double) * nshift);
    double *ziii = malloc(sizeof(double) * nshift), *oms = malloc(sizeof(double) * nshift);
    double *gms = malloc(sizeof(double) * nshift);
    int *flag = malloc(sizeof(int) * nshift);

    for (int k = 0; k < nshift; k++) {
        memset(&x[k * Vh], 0, sizeof(vec3) * Vh);
        flag[k] = 1;
    }
    for (long i = 0; i < Vh; i++) { r[i] = b[i]; p[i] = b[i]; dv[i] = vec_l2norm2(&b[i]); }
    global_sum(dv, Vh);
    double delta = dv[0], omega = 1.0, omega_save, alpha, lambda, gammag = 0.0;
    for (int k = 0; k < nshift; k++) {
        memcpy(&ps[k * Vh], b, sizeof(vec3) * Vh);
        zi[k] = 1.0; zii[k] = 1.0; gms[k] = 0.0;
    }
    int cg = 0;
    do {
        cg++;
        orc_doe((double *)h, (double *)p, u_);
        orc_deo((double *)s, (double *)h, u_);
        for (long i = 0; i < Vh; i++) {
            vec3 v3;
            for (int c = 0; c < 3; c++) v3.c[c] = csub(cscal(mass2, p[i].c[c]), s[i].c[c]);
            s[i] = v3;
            dv[i] = vec_rscal(&p[i], &v3);
        }
        global_sum(dv, Vh);
        alpha = dv[0];
        omega_save = omega;
        omega = -delta / alpha;
        for (int k = 0; k < nshift; k++) {
            if (flag[k] == 1) {
                ziii[k] = (zi[k] * zii[k] * omega_save) /
                          (omega * gammag * (zi[k] - zii[k]) + zi[k] * omega_save * (1.0 - shifts[k] * omega));
                oms[k] = omega * ziii[k] / zii[k];
                vec3 *xk = &x[k * Vh], *pk = &ps[k * Vh];
                for (long i = 0; i < Vh; i++)
                    for (int c = 0; c < 3; c++) xk[i].c[c] = csub(xk[i].c[c], cscal(oms[k], pk[i].c[c]));
            }
        }
        for (long i = 0; i < Vh; i++) {
            for (int c = 0; c < 3; c++) r[i].c[c] = cadd(r[i].c[c], cscal(omega, s[i].c[c]));
            dv[i] = vec_l2norm2(&r[i]);
        }
        global_sum(dv, Vh);
        lambda = dv[0];
        gammag = lambda / delta;
        for (long i = 0; i < Vh; i++)
            for (int c = 0; c < 3; c++) p[i].c[c] = cadd(r[i].c[c], cscal(gammag, p[i].c[c]));
        for (int k = 0; k < nshift; k++) {
            if (flag[k] == 1) {
                gms[k] = gammag * ziii[k] * oms[k] / (zii[k] * omega);
                vec3 *pk = &ps[k * Vh];
                for (long i = 0; i < Vh; i++)
                    for (int c = 0; c < 3; c++)
                        pk[i].c[c] = cadd(cscal(ziii[k], r[i].c[c]), cscal(gms[k], pk[i].c[c]));
                double fact = sqrt(delta * zii[k] * zii[k]);
                if (fact < res) flag[k] = 0;
                zi[k] = zii[k];
                zii[k] = ziii[k];
            }
        }
        delta = lambda;
    } while (sqrt(lambda) > res && cg < max_cg);

    free(r); free(p); free(h); free(s); free(ps); free(dv);
    free(zi); free(zii); free(ziii); free(oms); free(gms); free(flag);
    return cg;
}

/* chi = a0*b + sum_i a_i x_i: lib/Tools/RationalApprox/rationalapprox.cc:300-311 */
void orc_rational_sum(double *out_, const double *b_, const double *x_, double a0, const double *a, int nshift)
{
    vec3 *out = (vec3 *)out_;
    const vec3 *b = (const vec3 *)b_, *x = (const vec3 *)x_;
    for (long i = 0; i < g_Vh; i++) {
        vec3 v;
        for (int c = 0; c < 3; c++) v.c[c] = cscal(a0, b[i].c[c]);
        for (int k = 0; k < nshift; k++)
            for (int c = 0; c < 3; c++) v.c[c] = cadd(v.c[c], cscal(a[k], x[k * g_Vh + i].c[c]));
        out[i] = v;
    }
}

/* ---------------------------------------------------------------- fermion force */
/* fermionforce (CPU branch), outer products only: lib/Action/fermionforce.cc:46-104.
 * F (4V su3, accumulated): for each shift, h = Doe x; even x: F_mu(x) += a h(x+mu) (x) conj(x(x));
 * odd x: F_mu(x) += -a x(x+mu) (x) conj(h(x)). */
void orc_fermion_force_accum(double *F_, const double *u_, const double *x_, const double *a, int nshift)
{
    su3 *F = (su3 *)F_;
    const vec3 *xs = (const vec3 *)x_;
    vec3 *h = (vec3 *)malloc(sizeof(vec3) * g_Vh);
    for (int k = 0; k < nshift; k++) {
        const vec3 *s = &xs[k * g_Vh];
        orc_doe((double *)h, (const double *)s, u_);
        for (long e = 0; e < g_Vh; e++) {
            long o = e + g_Vh;
            for (int mu = 0; mu < 4; mu++) {
                vec3 v1 = h[g_nnp[e * 4 + mu] - g_Vh];
                vec3 v2 = vec_conj(&s[e]);
                for (int c = 0; c < 3; c++) v1.c[c] = cmul(v1.c[c], (cplx){ a[k], 0.0 });
                su3 aux = vec_outer(&v1, &v2);
                su3_addassign(&F[mu * g_V + e], &aux);

                v1 = s[g_nnp[o * 4 + mu]];
                v2 = vec_conj(&h[e]);
                for (int c = 0; c < 3; c++) v1.c[c] = cmul(v1.c[c], (cplx){ -a[k], 0.0 });
                aux = vec_outer(&v1, &v2);
                su3_addassign(&F[mu * g_V + o], &aux);
            }
        }
    }
    free(h);
}

/* ---------------------------------------------------------------- gauge staples / forces */
/* calc_staples: lib/Action/staples.cc:16-74 */
void orc_staples(double *st_, const double *u_)
{
    su3 *st = (su3 *)st_;
    const su3 *u = (const su3 *)u_;
    for (long pos = 0; pos < g_V; pos++)
        for (int mu = 0; mu < 4; mu++) {
            long imu = mu * g_V;
            su3 acc;
            memset(&acc, 0, sizeof(acc));
            for (int nu = 0; nu < 4; nu++) {
                if (nu == mu) continue;
                long inu = nu * g_V;
                su3 aux = u[inu + g_nnp[pos * 4 + mu]];
                su3 d = su3_dag(&u[imu + g_nnp[pos * 4 + nu]]);
                su3_mulassign(&aux, &d);
                d = su3_dag(&u[inu + pos]);
                su3_mulassign(&aux, &d);
                su3_addassign(&acc, &aux);

                long helper = g_nnm[pos * 4 + nu];
                aux = su3_dag(&u[inu + g_nnp[helper * 4 + mu]]);
                d = su3_dag(&u[imu + helper]);
                su3_mulassign(&aux, &d);
                su3_mulassign(&aux, &u[inu + helper]);
                su3_addassign(&acc, &aux);
            }
            st[imu + pos] = acc;
        }
}

/* First half of calc_ipdot: lib/Update/ipdot.cc:164-170 (CPU branch): buf = beta/3 * staples.
 * The fermion outer products (orc_fermion_force_accum) are then added on top of it, in the
 * reference's order. */
void orc_ipdot_gauge_init(double *buf_, const double *u_, double beta)
{
    su3 *buf = (su3 *)buf_;
    double bb3 = beta / 3.0;
    orc_staples(buf_, u_);
    for (long r = 0; r < 4 * g_V; r++) su3_scal_assign(&buf[r], bb3);
}

/* Second half of calc_ipdot / calc_ipdot_fermion: ipdot.cc:176-183 and 104-111:
 * ipdot = TA(U * buf). */
void orc_u_times_ta(double *ipdot_, const double *u_, const double *buf_)
{
    su3 *ip = (su3 *)ipdot_;
    const su3 *u = (const su3 *)u_, *buf = (const su3 *)buf_;
    for (long r = 0; r < 4 * g_V; r++) {
        su3 aux = u[r];
        su3_mulassign(&aux, &buf[r]);
        su3_ta(&aux);
        ip[r] = aux;
    }
}

/* calc_ipdot_gauge: lib/Update/ipdot.cc:25-49 (CPU branch): ipdot = TA((U * beta/3) * staples) */
void orc_ipdot_gauge(double *ipdot_, const double *u_, double beta)
{
    su3 *ip = (su3 *)ipdot_;
    const su3 *u = (const su3 *)u_;
    su3 *st = (su3 *)malloc(sizeof(su3) * 4 * g_V);
    orc_staples((double *)st, u_);
    double bb3 = beta / 3.0;
    for (long r = 0; r < 4 * g_V; r++) {
        su3 aux = u[r];
        su3_scal_assign(&aux, bb3);
        su3_mulassign(&aux, &st[r]);
        su3_ta(&aux);
        ip[r] = aux;
    }
    free(st);
}

/* ---------------------------------------------------------------- updates */
/* momenta_sum_multiply(p=i*step): lib/Update/momenta.cc:82-115 (P += p * ipdot) */
void orc_mom_update(double *P_, const double *ipdot_, double step)
{
    su3 *P = (su3 *)P_;
    const su3 *ip = (const su3 *)ipdot_;
    cplx p = { 0.0, step };
    for (long i = 0; i < 4 * g_V; i++) {
        su3 aux = ip[i];
        su3_cscal_assign(&aux, p);
        su3_addassign(&P[i], &aux);
    }
}

/* conf_left_exp_multiply(p=i*step): lib/Update/momenta.cc:42-78 + Conf::unitarize_with_eta
 * (lib/Main/Conf/conf.cc:235-251): U <- exp(p P) U, then sunitarize and row 2 times eta. */
void orc_link_update(double *u_, const double *P_, double step)
{
    su3 *u = (su3 *)u_;
    const su3 *P = (const su3 *)P_;
    cplx p = { 0.0, step };
    for (long i = 0; i < 4 * g_V; i++) {
        su3 aux = P[i];
        su3_cscal_assign(&aux, p);
        su3_exp(&aux);
        su3_mulassign(&aux, &u[i]);
        u[i] = aux;
    }
    for (long i = 0; i < 4 * g_V; i++) {
        su3_sunitarize(&u[i]);
        for (int j = 0; j < 3; j++) u[i].c[2][j] = cscal((double)g_eta[i], u[i].c[2][j]);
    }
}

/* sunitarize + eta on row 2 for every link (Conf::unitarize_with_eta, conf.cc:235-251) */
void orc_unitarize_with_eta(double *u_)
{
    su3 *u = (su3 *)u_;
    for (long i = 0; i < 4 * g_V; i++) {
        su3_sunitarize(&u[i]);
        for (int j = 0; j < 3; j++) u[i].c[2][j] = cscal((double)g_eta[i], u[i].c[2][j]);
    }
}

/* ---------------------------------------------------------------- actions and measurements */
/* Gauge action sum_r sum_{mu<nu} beta/3 ReTr(plaquette with eta): lib/Action/action.cc:6-61 */
double orc_gauge_action(const double *u_, double beta)
{
    const su3 *u = (const su3 *)u_;
    double *v = (double *)malloc(sizeof(double) * g_V);
    double bb3 = beta / 3.0;
    for (long r = 0; r < g_V; r++) {
        v[r] = 0.0;
        for (int mu = 0; mu < 3; mu++)
            for (int nu = mu + 1; nu < 4; nu++) {
                su3 aux = u[mu * g_V + r];
                su3_mulassign(&aux, &u[nu * g_V + g_nnp[r * 4 + mu]]);
                su3 d = su3_dag(&u[mu * g_V + g_nnp[r * 4 + nu]]);
                su3_mulassign(&aux, &d);
                d = su3_dag(&u[nu * g_V + r]);
                su3_mulassign(&aux, &d);
                v[r] += bb3 * su3_retr(&aux);
            }
    }
    global_sum(v, g_V);
    double s = v[0];
    free(v);
    return s;
}

/* Momentum action sum 1/2 ReTr(P^2): lib/Action/action.cc:122-134 */
double orc_momentum_action(const double *P_)
{
    const su3 *P = (const su3 *)P_;
    double *v = (double *)malloc(sizeof(double) * g_V);
    for (long r = 0; r < g_V; r++) {
        v[r] = 0.0;
        for (int mu = 0; mu < 4; mu++) {
            su3 aux = P[r + mu * g_V];
            su3_mulassign(&aux, &P[r + mu * g_V]);
            v[r] += 0.5 * su3_retr(&aux);
        }
    }
    global_sum(v, g_V);
    double s = v[0];
    free(v);
    return s;
}

/* sum_i Re<a_i, b_i> over one parity (fermion_action, action.cc:65-107) */
double orc_rdot(const double *a_, const double *b_)
{
    const vec3 *a = (const vec3 *)a_, *b = (const vec3 *)b_;
    double *v = (double *)malloc(sizeof(double) * g_Vh);
    for (long i = 0; i < g_Vh; i++) v[i] = vec_rscal(&a[i], &b[i]);
    global_sum(v, g_Vh);
    double s = v[0];
    free(v);
    return s;
}

/* Conf::calc_plaq: lib/Measurements/gaugemeas.cc:7-65 (spatial, temporal; minus sign for eta) */
void orc_plaquette(const double *u_, double *pls, double *plt)
{
    const su3 *u = (const su3 *)u_;
    double *d1 = (double *)malloc(sizeof(double) * g_V), *d2 = (double *)malloc(sizeof(double) * g_V);
    for (long r = 0; r < g_V; r++) {
        d1[r] = 0.0; d2[r] = 0.0;
        for (int mu = 0; mu < 3; mu++)
            for (int nu = mu + 1; nu < 4; nu++) {
                su3 aux = u[mu * g_V + r];
                su3_mulassign(&aux, &u[nu * g_V + g_nnp[r * 4 + mu]]);
                su3 d = su3_dag(&u[mu * g_V + g_nnp[r * 4 + nu]]);
                su3_mulassign(&aux, &d);
                d = su3_dag(&u[nu * g_V + r]);
                su3_mulassign(&aux, &d);
                if (nu == 3) d1[r] -= su3_retr(&aux);
                else d2[r] -= su3_retr(&aux);
            }
    }
    global_sum(d1, g_V);
    global_sum(d2, g_V);
    double inv = 1.0 / (double)g_V;
    double inv3 = inv / 3.0;
    *plt = d1[0] * inv3 * 0.3333333333333333333333333333333;
    *pls = d2[0] * inv3 * 0.3333333333333333333333333333333;
    free(d1); free(d2);
}

/* ---------------------------------------------------------------- measurements */
/* Conf::calc_poly: lib/Measurements/gaugemeas.cc:66-106.  From each of the reference's sites
 * r < vol3 (the even sites of the slabs t = 0 and t = 1: one per spatial point) the ordered
 * product of the nt temporal links; minus sign for the antiperiodic phase folded into them. */
void orc_polyakov(const double *u_, double *re, double *im)
{
    const su3 *u = (const su3 *)u_;
    long vol3 = (long)g_nx * g_ny * g_nz;
    double *d1 = (double *)malloc(sizeof(double) * vol3), *d2 = (double *)malloc(sizeof(double) * vol3);
    for (long r = 0; r < vol3; r++) {
        su3 aux;
        su3_one(&aux);
        long r2 = r;
        for (int t = 0; t < g_nt; t++) {
            su3_mulassign(&aux, &u[r2 + 3 * g_V]);
            r2 = g_nnp[r2 * 4 + 3];
        }
        d1[r] = -su3_retr(&aux);
        d2[r] = -(aux.c[0][0].im + aux.c[1][1].im + aux.c[2][2].im);
    }
    global_sum(d1, vol3);
    global_sum(d2, vol3);
    const double inv_vol3 = 1.0 / (double)vol3, one_by_three = 1.0 / 3.0;
    *re = d1[0] * inv_vol3 * one_by_three;
    *im = d2[0] * inv_vol3 * one_by_three;
    free(d1); free(d2);
}

static cplx vec_cscal(const vec3 *a, const vec3 *b)  /* c_scalprod, lib/Tools/vec3.h:227-235 */
{
    cplx r = { 0.0, 0.0 };
    for (int c = 0; c < 3; c++) r = cadd(r, cmul(cconj(a->c[c]), b->c[c]));
    return r;
}

/* chiral_meas for one pair of Z2 noise vectors: lib/Measurements/chiralmeas.cc:44-183 (the
 * branch without imaginary chemical potential).  out: chiral condensate, energy, baryon and
 * pressure densities as (re, im) pairs.  The even solve is (M^dag M) chi_e = phi_e to the
 * absolute residual res (the reference's invert, started here from zero). */
int orc_chiral_meas(const double *u_, const double *ne_, const double *no_, double mass, int nf, double res, int max_cg,
                    double *out)
{
    const su3 *u = (const su3 *)u_;
    const vec3 *rnd_e = (const vec3 *)ne_, *rnd_o = (const vec3 *)no_;
    long Vh = g_Vh;
    vec3 *phi_e = (vec3 *)malloc(sizeof(vec3) * Vh), *chi_e = (vec3 *)malloc(sizeof(vec3) * Vh);
    vec3 *phi_o = (vec3 *)malloc(sizeof(vec3) * Vh), *chi_o = (vec3 *)malloc(sizeof(vec3) * Vh);
    double *v[8];
    for (int j = 0; j < 8; j++) v[j] = (double *)malloc(sizeof(double) * Vh);
    orc_deo((double *)phi_e, no_, u_);
    for (long i = 0; i < Vh; i++)
        for (int c = 0; c < 3; c++) phi_e[i].c[c] = csub(cscal(mass, rnd_e[i].c[c]), phi_e[i].c[c]);
    const double zero = 0.0;
    int cg = orc_msolve((double *)chi_e, (const double *)phi_e, u_, mass, 1, &zero, res, max_cg);
    orc_doe((double *)phi_o, (const double *)chi_e, u_);
    const double one_by_mass = 1.0 / mass;
    for (long i = 0; i < Vh; i++)
        for (int c = 0; c < 3; c++) chi_o[i].c[c] = cscal(one_by_mass, csub(rnd_o[i].c[c], phi_o[i].c[c]));
    for (long i = 0; i < Vh; i++) {
        const long j = i + Vh;
        cplx ch = cadd(vec_cscal(&rnd_o[i], &chi_o[i]), vec_cscal(&rnd_e[i], &chi_e[i]));
        /* temporal hops: energy (p1 - p2) and baryon (p1 + p2) densities */
        vec3 ve = su3_mul_vec(&u[i + 3 * g_V], &chi_o[g_nnp[i * 4 + 3] - Vh]);
        vec3 we = su3_mul_vec(&u[i + 3 * g_V], &rnd_o[g_nnp[i * 4 + 3] - Vh]);
        cplx p1 = vec_cscal(&rnd_e[i], &ve), p2 = vec_cscal(&we, &chi_e[i]);
        cplx c1 = csub(p1, p2), c2 = cadd(p1, p2);
        vec3 vo = su3_mul_vec(&u[j + 3 * g_V], &chi_e[g_nnp[j * 4 + 3]]);
        vec3 wo = su3_mul_vec(&u[j + 3 * g_V], &rnd_e[g_nnp[j * 4 + 3]]);
        p1 = vec_cscal(&rnd_o[i], &vo);
        p2 = vec_cscal(&wo, &chi_o[i]);
        c1 = cadd(c1, csub(p1, p2));
        c2 = cadd(c2, cadd(p1, p2));
        /* spatial hops: pressure density */
        cplx cp = { 0.0, 0.0 };
        for (int k = 0; k < 3; k++) {
            ve = su3_mul_vec(&u[i + k * g_V], &chi_o[g_nnp[i * 4 + k] - Vh]);
            we = su3_mul_vec(&u[i + k * g_V], &rnd_o[g_nnp[i * 4 + k] - Vh]);
            cp = cadd(cp, vec_cscal(&rnd_e[i], &ve));
            cp = csub(cp, vec_cscal(&we, &chi_e[i]));
            vo = su3_mul_vec(&u[j + k * g_V], &chi_e[g_nnp[j * 4 + k]]);
            wo = su3_mul_vec(&u[j + k * g_V], &rnd_e[g_nnp[j * 4 + k]]);
            cp = cadd(cp, vec_cscal(&rnd_o[i], &vo));
            cp = csub(cp, vec_cscal(&wo, &chi_o[i]));
        }
        v[0][i] = ch.re; v[1][i] = ch.im;
        v[2][i] = c1.re; v[3][i] = c1.im;
        v[4][i] = c2.re; v[5][i] = c2.im;
        v[6][i] = cp.re; v[7][i] = cp.im;
    }
    const double inv_size = 1.0 / (double)g_V;
    for (int j = 0; j < 8; j++) {
        global_sum(v[j], Vh);
        out[j] = v[j][0] * ((j < 2 ? 1.0 : 0.5) * nf * 0.25 * inv_size);
        free(v[j]);
    }
    free(phi_e); free(chi_e); free(phi_o); free(chi_o);
    return cg;
}
