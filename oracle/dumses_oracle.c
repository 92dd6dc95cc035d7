/*
 * dumses_oracle.c -- TEST INFRASTRUCTURE ONLY (see dumses_oracle.h).
 *
 * CPU restatement of the DUMSES-Hybrid v2.2.0 second-order Godunov MHD step,
 * Cartesian geometry, NDIM = 2 or 3, adiabatic or isothermal EOS.  Each
 * function cites the reference routine it restates (path:line within the
 * reference project) and keeps its statement order and arithmetic order.
 * Fortran MIN/MAX are the ternaries MN/MX below; SIGN(one,x) is copysign.
 */
#include "dumses_oracle.h"
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* constants, src/modules/commons.f90:37-52 */
static const double zero = 0.0, one = 1.0, two = 2.0, half = 0.5, forth = 0.25;
static const double smallr = 1.0e-10, smallc = 1.0e-10;

static inline double MN(double a, double b) { return a < b ? a : b; }
static inline double MX(double a, double b) { return a > b ? a : b; }
static inline double SGN1(double x) { return copysign(1.0, x); }

/* ------------------------------------------------------------------------- */
/* Fortran-style arrays: arbitrary lower bounds, column-major                 */
/* ------------------------------------------------------------------------- */
typedef struct {
    double *d;
    int l0, l1, l2;          /* lower bounds of the three spatial indices */
    int n0, n1, n2, nv, nd;  /* extents */
    long s1, s2, s3, s4;     /* strides of index 2,3,4,5 */
    long size;
} farr;

static farr fa_alloc(int l0, int h0, int l1, int h1, int l2, int h2, int nv, int nd)
{
    farr a;
    a.l0 = l0; a.l1 = l1; a.l2 = l2;
    a.n0 = h0 - l0 + 1; a.n1 = h1 - l1 + 1; a.n2 = h2 - l2 + 1; a.nv = nv; a.nd = nd;
    a.s1 = a.n0; a.s2 = a.s1 * a.n1; a.s3 = a.s2 * a.n2; a.s4 = a.s3 * nv;
    a.size = a.s4 * nd;
    a.d = (double *)calloc((size_t)a.size, sizeof(double));
    return a;
}

#ifdef OR_CHECK_BOUNDS
static double *fa_chk(const farr *a, int i, int j, int k, int v, int d, int line)
{
    if (i < a->l0 || i >= a->l0 + a->n0 || j < a->l1 || j >= a->l1 + a->n1 ||
        k < a->l2 || k >= a->l2 + a->n2 || v < 1 || v > a->nv || d < 1 || d > a->nd) {
        fprintf(stderr, "oracle: out of bounds at line %d: (%d,%d,%d,%d,%d)\n", line, i, j, k, v, d);
        abort();
    }
    return a->d + (i - a->l0) + a->s1 * (j - a->l1) + a->s2 * (k - a->l2) + a->s3 * (v - 1) + a->s4 * (d - 1);
}
#define AT(a, i, j, k, v, dd) (*fa_chk(&(a), (i), (j), (k), (v), (dd), __LINE__))
#else
#define AT(a, i, j, k, v, dd) ((a).d[((i) - (a).l0) + (a).s1 * ((j) - (a).l1) + (a).s2 * ((k) - (a).l2) \
                                     + (a).s3 * ((v) - 1) + (a).s4 * ((dd) - 1)])
#endif
#define A3(a, i, j, k) AT(a, i, j, k, 1, 1)
#define A4(a, i, j, k, v) AT(a, i, j, k, v, 1)
#define A5(a, i, j, k, v, dd) AT(a, i, j, k, v, dd)

/* variable indices, commons.f90:70-80 */
enum { ir = 1, iu = 2, iv = 3, iw = 4, ip = 5, iA = 6, iB = 7, iC = 8 };
enum { nvar = 8, nghost = 3 };

struct or_state {
    dg_params p;
    int ndim, ndim_act;
    int iu1, iu2, ju1, ju2, ku1, ku2;
    int if1, if2, jf1, jf2, kf1, kf2;
    int nx, ny, nz;
    double dx, dy, dz;
    double *xc, *yc, *zc;          /* x(iu1:iu2) etc. */
    farr uin, uin_old, qin, duin;
    farr flux, emfx, emfy, emfz, Ex, Ey, Ez;
    farr bfc, dq, dbfc, qm, qp, qRT, qRB, qLT, qLB;
    farr fgodunov, fgodunov_pre, rgstar, ugstar, vgstar, wgstar, bgstar, cgstar, pgstar;
    farr dv, ds;
};

#define XC(i) (s->xc[(i) - s->iu1])
#define YC(j) (s->yc[(j) - s->ju1])
#define ZC(k) (s->zc[(k) - s->ku1])

void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* init_param bounds (init.f90:33-54), allocate_workspace (init.f90:348-419),
 * init_grid (init.f90:423-560, Cartesian, single rank) */
or_state *or_create(const dg_params *p)
{
    or_state *s = (or_state *)calloc(1, sizeof(or_state));
    s->p = *p;
    s->ndim = p->ndim;
    s->nx = p->nx; s->ny = p->ny; s->nz = p->nz;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    /* read_input: ndim_act (init.f90:203-213) */
    if ((nx == 1 && ny == 1) || (nx == 1 && nz == 1) || (ny == 1 && nz == 1)) s->ndim_act = 1;
    else if ((nx == 1 && ny > 1 && nz > 1) || (nx > 1 && ny == 1 && nz > 1) || (nx > 1 && ny > 1 && nz == 1))
        s->ndim_act = 2;
    else s->ndim_act = 3;

    s->iu1 = 1 - nghost; s->iu2 = nx + nghost;
    s->ju1 = 1; s->ju2 = 1; s->ku1 = 1; s->ku2 = 1;
    if (s->ndim > 1) { s->ju1 = 1 - nghost; s->ju2 = ny + nghost; }
    if (s->ndim == 3) { s->ku1 = 1 - nghost; s->ku2 = nz + nghost; }
    s->if1 = 1; s->if2 = nx + 1; s->jf1 = 1; s->jf2 = 1; s->kf1 = 1; s->kf2 = 1;
    if (s->ndim > 1) { s->jf1 = 1; s->jf2 = ny + 1; }
    if (s->ndim == 3) { s->kf1 = 1; s->kf2 = nz + 1; }

    int iu1 = s->iu1, iu2 = s->iu2, ju1 = s->ju1, ju2 = s->ju2, ku1 = s->ku1, ku2 = s->ku2;
    int nd = s->ndim;
    s->uin = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar + 3, 1);
    s->uin_old = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar + 3, 1);
    s->qin = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, 1);
    s->duin = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, 1);
    s->flux = fa_alloc(s->if1, s->if2, s->jf1, s->jf2, s->kf1, s->kf2, nvar, nd);
    s->emfx = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->emfy = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->emfz = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->Ex = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->Ey = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->Ez = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->dv = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->ds = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nd, 1);
    s->bfc = fa_alloc(iu1, iu2 + 1, ju1, ju2 + 1, ku1, ku2 + 1, 3, 1);
    s->dq = fa_alloc(iu1, iu2 + 1, ju1, ju2 + 1, ku1, ku2 + 1, nvar, nd);
    s->dbfc = fa_alloc(iu1, iu2 + 1, ju1, ju2 + 1, ku1, ku2 + 1, 3, nd);
    s->qm = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, nd);
    s->qp = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, nd);
    s->qRT = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, 3);
    s->qRB = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, 3);
    s->qLT = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, 3);
    s->qLB = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, 3);
    s->fgodunov = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nvar, nd);
    s->fgodunov_pre = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, nd, 1);
    s->rgstar = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->ugstar = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->vgstar = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->wgstar = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->bgstar = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->cgstar = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);
    s->pgstar = fa_alloc(iu1, iu2, ju1, ju2, ku1, ku2, 1, 1);

    /* init_grid, init.f90:447-519 (no MPI): dx = (xmax-xmin)/nxglob ... */
    s->dx = (p->xmax - p->xmin) / nx;
    s->dy = (p->ymax - p->ymin) / ny;
    s->dz = (p->zmax - p->zmin) / nz;
    s->xc = (double *)calloc((size_t)(iu2 - iu1 + 1), sizeof(double));
    s->yc = (double *)calloc((size_t)(ju2 - ju1 + 1), sizeof(double));
    s->zc = (double *)calloc((size_t)(ku2 - ku1 + 1), sizeof(double));
    for (int i = iu1; i <= iu2; i++) XC(i) = p->xmin + s->dx / 2 + (i - 1) * s->dx;
    for (int j = ju1; j <= ju2; j++) YC(j) = (s->ndim > 1) ? p->ymin + s->dy / 2 + (j - 1) * s->dy : 0.0;
    for (int k = ku1; k <= ku2; k++) ZC(k) = (s->ndim == 3) ? p->zmin + s->dz / 2 + (k - 1) * s->dz : 0.0;
    /* dv, ds on ilo..ihi (init.f90:521-536) */
    int ilo = (1 < iu1 + 1) ? 1 : iu1 + 1, ihi = (1 > iu2 - 1) ? 1 : iu2 - 1;
    int jlo = (1 < ju1 + 1) ? 1 : ju1 + 1, jhi = (1 > ju2 - 1) ? 1 : ju2 - 1;
    int klo = (1 < ku1 + 1) ? 1 : ku1 + 1, khi = (1 > ku2 - 1) ? 1 : ku2 - 1;
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                A3(s->dv, i, j, k) = s->dx * s->dy * s->dz;
                for (int idim = 1; idim <= nd; idim++) {
                    if (idim == 1) A4(s->ds, i, j, k, idim) = s->dy * s->dz;
                    if (idim == 2) A4(s->ds, i, j, k, idim) = s->dx * s->dz;
                    if (idim == 3) A4(s->ds, i, j, k, idim) = s->dx * s->dy;
                }
            }
    return s;
}

void or_destroy(or_state *s)
{
    if (!s) return;
    farr *all[] = {&s->uin, &s->uin_old, &s->qin, &s->duin, &s->flux, &s->emfx, &s->emfy, &s->emfz,
                   &s->Ex, &s->Ey, &s->Ez, &s->bfc, &s->dq, &s->dbfc, &s->qm, &s->qp, &s->qRT,
                   &s->qRB, &s->qLT, &s->qLB, &s->fgodunov, &s->fgodunov_pre, &s->rgstar, &s->ugstar,
                   &s->vgstar, &s->wgstar, &s->bgstar, &s->cgstar, &s->pgstar, &s->dv, &s->ds};
    for (size_t n = 0; n < sizeof(all) / sizeof(all[0]); n++) free(all[n]->d);
    free(s->xc); free(s->yc); free(s->zc);
    free(s);
}

double *or_uin(or_state *s) { return s->uin.d; }
long long or_uin_size(const or_state *s) { return s->uin.size; }

double *or_array(or_state *s, int which, long long *count)
{
    farr *a = NULL;
    switch (which) {
    case 0: a = &s->flux; break;
    case 1: a = &s->emfx; break;
    case 2: a = &s->emfy; break;
    case 3: a = &s->emfz; break;
    case 4: a = &s->fgodunov_pre; break;
    case 5: a = &s->qin; break;
    default: return NULL;
    }
    if (count) *count = a->size;
    return a->d;
}

/* ------------------------------------------------------------------------- */
/* primitive, src/subroutines/scheme.f90:20-91                                */
/* ------------------------------------------------------------------------- */
void or_primitive(or_state *s, double dt)
{
    const dg_params *p = &s->p;
    double smallp;
    if (p->iso) smallp = smallr * (p->ciso * p->ciso);
    else smallp = smallr * (smallc * smallc) / p->gamma;
    const double gamma = p->gamma, ciso = p->ciso, Omega0 = p->omega0;
#pragma omp parallel for schedule(static)
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = s->iu1; i <= s->iu2; i++) {
                A4(s->qin, i, j, k, ir) = MX(A4(s->uin, i, j, k, ir), smallr);
                A4(s->qin, i, j, k, iu) = A4(s->uin, i, j, k, iu) / A4(s->uin, i, j, k, ir);
                A4(s->qin, i, j, k, iv) = A4(s->uin, i, j, k, iv) / A4(s->uin, i, j, k, ir);
                A4(s->qin, i, j, k, iw) = A4(s->uin, i, j, k, iw) / A4(s->uin, i, j, k, ir);
                A4(s->qin, i, j, k, iA) = half * (A4(s->uin, i, j, k, iA) + A4(s->uin, i, j, k, iA + 3));
                A4(s->qin, i, j, k, iB) = half * (A4(s->uin, i, j, k, iB) + A4(s->uin, i, j, k, iB + 3));
                A4(s->qin, i, j, k, iC) = half * (A4(s->uin, i, j, k, iC) + A4(s->uin, i, j, k, iC + 3));
                if (p->iso) {
                    A4(s->qin, i, j, k, ip) = A4(s->uin, i, j, k, ir) * (ciso * ciso);
                } else {
                    double qu = A4(s->qin, i, j, k, iu), qv = A4(s->qin, i, j, k, iv), qw = A4(s->qin, i, j, k, iw);
                    double qa = A4(s->qin, i, j, k, iA), qb = A4(s->qin, i, j, k, iB), qc = A4(s->qin, i, j, k, iC);
                    double eken = half * (qu * qu + qv * qv + qw * qw);
                    double emag = half * (qa * qa + qb * qb + qc * qc);
                    double eint = (A4(s->uin, i, j, k, ip) - emag) / A4(s->uin, i, j, k, ir) - eken;
                    A4(s->qin, i, j, k, ip) = MX((gamma - one) * A4(s->qin, i, j, k, ir) * eint, smallp);
                }
                if (Omega0 > zero) {
                    double dvx = two * Omega0 * A4(s->qin, i, j, k, iv);
                    double dvy = -(half * Omega0 * A4(s->qin, i, j, k, iu));
                    A4(s->qin, i, j, k, iu) = A4(s->qin, i, j, k, iu) + dvx * dt * half;
                    A4(s->qin, i, j, k, iv) = A4(s->qin, i, j, k, iv) + dvy * dt * half;
                }
            }
}

/* comp_speed, physics.f90:148-164 */
static inline double comp_speed(double gamma, double rho, double p, double v, double bn, double bt1, double bt2)
{
    double c2 = gamma * p / rho;
    double b2 = bn * bn + bt1 * bt1 + bt2 * bt2;
    double d2 = half * (c2 + b2 / rho);
    double cf = sqrt(d2 + sqrt(d2 * d2 - c2 * bn * bn / rho));
    return cf + fabs(v);
}

/* compute_dt, physics.f90:18-132 (CPU branch, Cartesian, single rank) */
double or_compute_dt(or_state *s)
{
    const dg_params *p = &s->p;
    or_primitive(s, zero);
    double dt = p->courant * s->dx / smallc;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for schedule(static) reduction(min : dt)
    for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) {
                double rho = A4(s->qin, i, j, k, ir), vx = A4(s->qin, i, j, k, iu);
                double vy = A4(s->qin, i, j, k, iv), vz = A4(s->qin, i, j, k, iw);
                double pp = A4(s->qin, i, j, k, ip), bx = A4(s->qin, i, j, k, iA);
                double by = A4(s->qin, i, j, k, iB), bz = A4(s->qin, i, j, k, iC);
                double velx, vely = 0, velz = 0;
                velx = comp_speed(p->gamma, rho, pp, vx, bx, by, bz);
                if (nx == 1) velx = zero;
                if (s->ndim > 1) {
                    vely = comp_speed(p->gamma, rho, pp, vy, by, bz, bx);
                    if ((p->omega0 > zero) && !p->fargo) vely = vely + 1.5 * p->omega0 * (p->xmax - p->xmin) * half;
                    if (ny == 1) vely = zero;
                }
                if (s->ndim == 3) {
                    velz = comp_speed(p->gamma, rho, pp, vz, bz, bx, by);
                    if (nz == 1) velz = zero;
                }
                double c;
                if (s->ndim == 1) c = s->dx / velx;  /* physics.f90:101-103 */
                else if (s->ndim == 2) c = one / (velx / s->dx + vely / s->dy);
                else c = one / (velx / s->dx + vely / s->dy + velz / s->dz);
                dt = MN(dt, c);
            }
    return p->courant * dt;
}

/* fc_magnetic, scheme.f90:193-249 */
static void fc_magnetic(or_state *s)
{
#pragma omp parallel for schedule(static)
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = s->iu1; i <= s->iu2 + 1; i++)
                A4(s->bfc, i, j, k, 1) = (i <= s->iu2) ? A4(s->uin, i, j, k, iA) : A4(s->uin, i - 1, j, k, iA + 3);
#pragma omp parallel for schedule(static)
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2 + 1; j++)
            for (int i = s->iu1; i <= s->iu2; i++)
                A4(s->bfc, i, j, k, 2) = (j <= s->ju2) ? A4(s->uin, i, j, k, iB) : A4(s->uin, i, j - 1, k, iB + 3);
#pragma omp parallel for schedule(static)
    for (int k = s->ku1; k <= s->ku2 + 1; k++)
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = s->iu1; i <= s->iu2; i++)
                A4(s->bfc, i, j, k, 3) = (k <= s->ku2) ? A4(s->uin, i, j, k, iC) : A4(s->uin, i, j, k - 1, iC + 3);
}

/* the one-dimensional limiter used by slope() for slope_type 1 and 2 (scheme.f90:450-458) */
static inline double limit1(double st, double qm1, double q0, double qp1)
{
    double dlft = st * (q0 - qm1);
    double drgt = st * (qp1 - q0);
    double dcen = half * (dlft + drgt) / st;
    double dsgn = SGN1(dcen);
    double slop = MN(fabs(dlft), fabs(drgt));
    double dlim = slop;
    if ((dlft * drgt) <= zero) dlim = zero;
    return dsgn * MN(dlim, fabs(dcen));
}

/* slope, scheme.f90:253-656 (NDIM 2 and 3) */
static void slope(or_state *s)
{
    const int st = s->p.slope_type;
    int ilo = MN(1, s->iu1 + 1), ihi = MX(1, s->iu2 - 1);
    int jlo = MN(1, s->ju1 + 1), jhi = MX(1, s->ju2 - 1);
    int klo = MN(1, s->ku1 + 1), khi = MX(1, s->ku2 - 1);
    if (st == 0) {
        memset(s->dq.d, 0, sizeof(double) * s->dq.size);
        memset(s->dbfc.d, 0, sizeof(double) * s->dbfc.size);
        return;
    }
    const double stl = (double)MN(st, 2);
    const double sd = (double)st;
    const farr q = s->qin;
    if (s->ndim == 1) {
        /* scheme.f90:289-316: slope_type 1 or 2 (the reference stops on any other) */
        if (st >= 3) return;
#pragma omp parallel for schedule(static)
        for (int k = klo; k <= khi; k++)
            for (int j = jlo; j <= jhi; j++)
                for (int i = ilo; i <= ihi; i++)
                    for (int ivar = 1; ivar <= nvar; ivar++)
                        A5(s->dq, i, j, k, ivar, 1) = limit1(sd, A4(q, i - 1, j, k, ivar), A4(q, i, j, k, ivar), A4(q, i + 1, j, k, ivar));
        return;
    }
    if (s->ndim == 2) {
        if (st < 3) {
#pragma omp parallel for schedule(static)
            for (int k = klo; k <= khi; k++)
                for (int j = jlo; j <= jhi; j++)
                    for (int i = ilo; i <= ihi; i++)
                        for (int v = 1; v <= nvar; v++) {
                            A5(s->dq, i, j, k, v, 1) = limit1(sd, A4(q, i - 1, j, k, v), A4(q, i, j, k, v), A4(q, i + 1, j, k, v));
                            A5(s->dq, i, j, k, v, 2) = limit1(sd, A4(q, i, j - 1, k, v), A4(q, i, j, k, v), A4(q, i, j + 1, k, v));
                        }
        } else {
            /* multidimensional limiter, scheme.f90:355-391 */
#pragma omp parallel for schedule(static)
            for (int k = klo; k <= khi; k++)
                for (int j = jlo; j <= jhi; j++)
                    for (int i = ilo; i <= ihi; i++)
                        for (int v = 1; v <= nvar; v++) {
                            double c = A4(q, i, j, k, v);
                            double dfll = A4(q, i - 1, j - 1, k, v) - c;
                            double dflm = A4(q, i - 1, j, k, v) - c;
                            double dflr = A4(q, i, j - 1, k, v) - c;
                            double dfml = A4(q, i, j - 1, k, v) - c;
                            double dfmm = A4(q, i, j, k, v) - c;
                            double dfmr = A4(q, i, j + 1, k, v) - c;
                            double dfrl = A4(q, i + 1, j - 1, k, v) - c;
                            double dfrm = A4(q, i + 1, j, k, v) - c;
                            double dfrr = A4(q, i + 1, j + 1, k, v) - c;
                            double vals[9] = {dfll, dflm, dflr, dfml, dfmm, dfmr, dfrl, dfrm, dfrr};
                            double vmin = vals[0], vmax = vals[0];
                            for (int n = 1; n < 9; n++) { vmin = MN(vmin, vals[n]); vmax = MX(vmax, vals[n]); }
                            double dfx = half * (A4(q, i + 1, j, k, v) - A4(q, i - 1, j, k, v));
                            double dfy = half * (A4(q, i, j + 1, k, v) - A4(q, i, j - 1, k, v));
                            double dff = half * (fabs(dfx) + fabs(dfy));
                            double slop;
                            if (dff > zero) slop = MN(one, MN(fabs(vmin), fabs(vmax)) / dff);
                            else slop = one;
                            double dlim = slop;
                            A5(s->dq, i, j, k, v, 1) = dlim * dfx;
                            A5(s->dq, i, j, k, v, 2) = dlim * dfy;
                        }
        }
        /* Bx along Y, By along X (scheme.f90:399-434) */
#pragma omp parallel for schedule(static)
        for (int k = klo; k <= khi; k++)
            for (int j = jlo; j <= jhi; j++)
                for (int i = ilo; i <= ihi + 1; i++)
                    A5(s->dbfc, i, j, k, 1, 2) = limit1(stl, A4(s->bfc, i, j - 1, k, 1), A4(s->bfc, i, j, k, 1), A4(s->bfc, i, j + 1, k, 1));
#pragma omp parallel for schedule(static)
        for (int k = klo; k <= khi; k++)
            for (int j = jlo; j <= jhi + 1; j++)
                for (int i = ilo; i <= ihi; i++)
                    A5(s->dbfc, i, j, k, 2, 1) = limit1(stl, A4(s->bfc, i - 1, j, k, 2), A4(s->bfc, i, j, k, 2), A4(s->bfc, i + 1, j, k, 2));
        return;
    }
    /* NDIM == 3, scheme.f90:440-653 */
    if (st < 3) {
#pragma omp parallel for schedule(static)
        for (int k = klo; k <= khi; k++)
            for (int j = jlo; j <= jhi; j++)
                for (int i = ilo; i <= ihi; i++)
                    for (int v = 1; v <= nvar; v++) {
                        A5(s->dq, i, j, k, v, 1) = limit1(sd, A4(q, i - 1, j, k, v), A4(q, i, j, k, v), A4(q, i + 1, j, k, v));
                        A5(s->dq, i, j, k, v, 2) = limit1(sd, A4(q, i, j - 1, k, v), A4(q, i, j, k, v), A4(q, i, j + 1, k, v));
                        A5(s->dq, i, j, k, v, 3) = limit1(sd, A4(q, i, j, k - 1, v), A4(q, i, j, k, v), A4(q, i, j, k + 1, v));
                    }
    } else {
        /* scheme.f90:484-557: 27-point min/max in the order the reference lists them */
#pragma omp parallel for schedule(static)
        for (int k = klo; k <= khi; k++)
            for (int j = jlo; j <= jhi; j++)
                for (int i = ilo; i <= ihi; i++)
                    for (int v = 1; v <= nvar; v++) {
                        double c = A4(q, i, j, k, v);
                        double vals[27];
                        int n = 0;
                        for (int dk = -1; dk <= 1; dk++)
                            for (int di = -1; di <= 1; di++)
                                for (int dj = -1; dj <= 1; dj++)
                                    vals[n++] = A4(q, i + di, j + dj, k + dk, v) - c;
                        double vmin = vals[0], vmax = vals[0];
                        for (n = 1; n < 27; n++) { vmin = MN(vmin, vals[n]); vmax = MX(vmax, vals[n]); }
                        double dfx = half * (A4(q, i + 1, j, k, v) - A4(q, i - 1, j, k, v));
                        double dfy = half * (A4(q, i, j + 1, k, v) - A4(q, i, j - 1, k, v));
                        double dfz = half * (A4(q, i, j, k + 1, v) - A4(q, i, j, k - 1, v));
                        double dff = half * (fabs(dfx) + fabs(dfy) + fabs(dfz));
                        double slop;
                        if (dff > zero) slop = MN(one, MN(fabs(vmin), fabs(vmax)) / dff);
                        else slop = one;
                        double dlim = slop;
                        A5(s->dq, i, j, k, v, 1) = dlim * dfx;
                        A5(s->dq, i, j, k, v, 2) = dlim * dfy;
                        A5(s->dq, i, j, k, v, 3) = dlim * dfz;
                    }
    }
#pragma omp parallel for schedule(static)
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi + 1; i++) {
                A5(s->dbfc, i, j, k, 1, 2) = limit1(stl, A4(s->bfc, i, j - 1, k, 1), A4(s->bfc, i, j, k, 1), A4(s->bfc, i, j + 1, k, 1));
                A5(s->dbfc, i, j, k, 1, 3) = limit1(stl, A4(s->bfc, i, j, k - 1, 1), A4(s->bfc, i, j, k, 1), A4(s->bfc, i, j, k + 1, 1));
            }
#pragma omp parallel for schedule(static)
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi + 1; j++)
            for (int i = ilo; i <= ihi; i++) {
                A5(s->dbfc, i, j, k, 2, 1) = limit1(stl, A4(s->bfc, i - 1, j, k, 2), A4(s->bfc, i, j, k, 2), A4(s->bfc, i + 1, j, k, 2));
                A5(s->dbfc, i, j, k, 2, 3) = limit1(stl, A4(s->bfc, i, j, k - 1, 2), A4(s->bfc, i, j, k, 2), A4(s->bfc, i, j, k + 1, 2));
            }
#pragma omp parallel for schedule(static)
    for (int k = klo; k <= khi + 1; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                A5(s->dbfc, i, j, k, 3, 1) = limit1(stl, A4(s->bfc, i - 1, j, k, 3), A4(s->bfc, i, j, k, 3), A4(s->bfc, i + 1, j, k, 3));
                A5(s->dbfc, i, j, k, 3, 2) = limit1(stl, A4(s->bfc, i, j - 1, k, 3), A4(s->bfc, i, j, k, 3), A4(s->bfc, i, j + 1, k, 3));
            }
}

/* store one traced state with the rho/P floors of the reference */
#define PUT8(arr, i, j, k, d, R, U, V, W, P, AA, BB, CC)                            \
    do {                                                                           \
        A5(arr, i, j, k, ir, d) = MX(smallr, (R));                                 \
        A5(arr, i, j, k, iu, d) = (U);                                             \
        A5(arr, i, j, k, iv, d) = (V);                                             \
        A5(arr, i, j, k, iw, d) = (W);                                             \
        A5(arr, i, j, k, ip, d) = MX(smallp, (P));                                 \
        A5(arr, i, j, k, iA, d) = (AA);                                            \
        A5(arr, i, j, k, iB, d) = (BB);                                            \
        A5(arr, i, j, k, iC, d) = (CC);                                            \
    } while (0)

/* trace3d, scheme.f90:1149-1711 (Cartesian branch) */
static void trace3d(or_state *s, double dt)
{
    const dg_params *p = &s->p;
    const double gamma = p->gamma, Omega0 = p->omega0;
    const int fargo = p->fargo;
    const double smallp = smallr * (smallc * smallc) / gamma;
    int ilo = MN(1, s->iu1 + 1), ihi = MX(1, s->iu2 - 1);
    int jlo = MN(1, s->ju1 + 1), jhi = MX(1, s->ju2 - 1);
    int klo = MN(1, s->ku1 + 1), khi = MX(1, s->ku2 - 1);
    const double dtdx = dt / s->dx, dtdy = dt / s->dy, dtdz = dt / s->dz, dx = s->dx;
    const farr q = s->qin, bfc = s->bfc;

    /* edge electric fields, scheme.f90:1194-1239 */
#pragma omp parallel for schedule(static)
    for (int k = klo; k <= s->ku2; k++)
        for (int j = jlo; j <= s->ju2; j++)
            for (int i = ilo; i <= s->iu2; i++) {
                double u, v, w, A, B, C, shear;
                v = forth * (A4(q, i, j - 1, k - 1, iv) + A4(q, i, j - 1, k, iv) + A4(q, i, j, k - 1, iv) + A4(q, i, j, k, iv));
                w = forth * (A4(q, i, j - 1, k - 1, iw) + A4(q, i, j - 1, k, iw) + A4(q, i, j, k - 1, iw) + A4(q, i, j, k, iw));
                B = half * (A4(bfc, i, j, k - 1, 2) + A4(bfc, i, j, k, 2));
                C = half * (A4(bfc, i, j - 1, k, 3) + A4(bfc, i, j, k, 3));
                A3(s->Ex, i, j, k) = v * C - w * B;
                if ((Omega0 > zero) && !fargo) {
                    shear = -1.5 * Omega0 * XC(i);
                    A3(s->Ex, i, j, k) = A3(s->Ex, i, j, k) + shear * C;
                }
                u = forth * (A4(q, i - 1, j, k - 1, iu) + A4(q, i - 1, j, k, iu) + A4(q, i, j, k - 1, iu) + A4(q, i, j, k, iu));
                w = forth * (A4(q, i - 1, j, k - 1, iw) + A4(q, i - 1, j, k, iw) + A4(q, i, j, k - 1, iw) + A4(q, i, j, k, iw));
                A = half * (A4(bfc, i, j, k - 1, 1) + A4(bfc, i, j, k, 1));
                C = half * (A4(bfc, i - 1, j, k, 3) + A4(bfc, i, j, k, 3));
                A3(s->Ey, i, j, k) = w * A - u * C;
                u = forth * (A4(q, i - 1, j - 1, k, iu) + A4(q, i - 1, j, k, iu) + A4(q, i, j - 1, k, iu) + A4(q, i, j, k, iu));
                v = forth * (A4(q, i - 1, j - 1, k, iv) + A4(q, i - 1, j, k, iv) + A4(q, i, j - 1, k, iv) + A4(q, i, j, k, iv));
                A = half * (A4(bfc, i, j - 1, k, 1) + A4(bfc, i, j, k, 1));
                B = half * (A4(bfc, i - 1, j, k, 2) + A4(bfc, i, j, k, 2));
                A3(s->Ez, i, j, k) = u * B - v * A;
                if ((Omega0 > zero) && !fargo) {
                    shear = -1.5 * Omega0 * half * (XC(i) + XC(i - 1));
                    A3(s->Ez, i, j, k) = A3(s->Ez, i, j, k) - shear * A;
                }
            }

#pragma omp parallel for schedule(static)
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                double r = A4(q, i, j, k, ir), u = A4(q, i, j, k, iu), v = A4(q, i, j, k, iv), w = A4(q, i, j, k, iw);
                double pp = A4(q, i, j, k, ip), A = A4(q, i, j, k, iA), B = A4(q, i, j, k, iB), C = A4(q, i, j, k, iC);
                double drx = half * A5(s->dq, i, j, k, ir, 1), dux = half * A5(s->dq, i, j, k, iu, 1);
                double dvx = half * A5(s->dq, i, j, k, iv, 1), dwx = half * A5(s->dq, i, j, k, iw, 1);
                double dpx = half * A5(s->dq, i, j, k, ip, 1), dBx = half * A5(s->dq, i, j, k, iB, 1);
                double dCx = half * A5(s->dq, i, j, k, iC, 1);
                double dry = half * A5(s->dq, i, j, k, ir, 2), duy = half * A5(s->dq, i, j, k, iu, 2);
                double dvy = half * A5(s->dq, i, j, k, iv, 2), dwy = half * A5(s->dq, i, j, k, iw, 2);
                double dpy = half * A5(s->dq, i, j, k, ip, 2), dAy = half * A5(s->dq, i, j, k, iA, 2);
                double dCy = half * A5(s->dq, i, j, k, iC, 2);
                double drz = half * A5(s->dq, i, j, k, ir, 3), duz = half * A5(s->dq, i, j, k, iu, 3);
                double dvz = half * A5(s->dq, i, j, k, iv, 3), dwz = half * A5(s->dq, i, j, k, iw, 3);
                double dpz = half * A5(s->dq, i, j, k, ip, 3), dAz = half * A5(s->dq, i, j, k, iA, 3);
                double dBz = half * A5(s->dq, i, j, k, iB, 3);
                double AL = A4(bfc, i, j, k, 1), AR = A4(bfc, i + 1, j, k, 1);
                double BL = A4(bfc, i, j, k, 2), BR = A4(bfc, i, j + 1, k, 2);
                double CL = A4(bfc, i, j, k, 3), CR = A4(bfc, i, j, k + 1, 3);
                double dAx = half * (AR - AL), dBy = half * (BR - BL), dCz = half * (CR - CL);
                double dALy = half * A5(s->dbfc, i, j, k, 1, 2), dARy = half * A5(s->dbfc, i + 1, j, k, 1, 2);
                double dALz = half * A5(s->dbfc, i, j, k, 1, 3), dARz = half * A5(s->dbfc, i + 1, j, k, 1, 3);
                double dBLx = half * A5(s->dbfc, i, j, k, 2, 1), dBRx = half * A5(s->dbfc, i, j + 1, k, 2, 1);
                double dBLz = half * A5(s->dbfc, i, j, k, 2, 3), dBRz = half * A5(s->dbfc, i, j + 1, k, 2, 3);
                double dCLx = half * A5(s->dbfc, i, j, k, 3, 1), dCRx = half * A5(s->dbfc, i, j, k + 1, 3, 1);
                double dCLy = half * A5(s->dbfc, i, j, k, 3, 2), dCRy = half * A5(s->dbfc, i, j, k + 1, 3, 2);
                double ELL = A3(s->Ex, i, j, k), ELR = A3(s->Ex, i, j, k + 1);
                double ERL = A3(s->Ex, i, j + 1, k), ERR = A3(s->Ex, i, j + 1, k + 1);
                double FLL = A3(s->Ey, i, j, k), FLR = A3(s->Ey, i, j, k + 1);
                double FRL = A3(s->Ey, i + 1, j, k), FRR = A3(s->Ey, i + 1, j, k + 1);
                double GLL = A3(s->Ez, i, j, k), GLR = A3(s->Ez, i, j + 1, k);
                double GRL = A3(s->Ez, i + 1, j, k), GRR = A3(s->Ez, i + 1, j + 1, k);

                /* source terms, scheme.f90:1351-1389 */
                double sr0 = (-u * drx - dux * r) * dtdx + (-v * dry - dvy * r) * dtdy + (-w * drz - dwz * r) * dtdz;
                double su0 = (-u * dux - (dpx + B * dBx + C * dCx) / r) * dtdx + (-v * duy + B * dAy / r) * dtdy
                           + (-w * duz + C * dAz / r) * dtdz;
                double sv0 = (-u * dvx + A * dBx / r) * dtdx + (-v * dvy - (dpy + A * dAy + C * dCy) / r) * dtdy
                           + (-w * dvz + C * dBz / r) * dtdz;
                double sw0 = (-u * dwx + A * dCx / r) * dtdx + (-v * dwy + B * dCy / r) * dtdy
                           + (-w * dwz - (dpz + A * dAz + B * dBz) / r) * dtdz;
                double sp0 = (-u * dpx - dux * gamma * pp) * dtdx + (-v * dpy - dvy * gamma * pp) * dtdy
                           + (-w * dpz - dwz * gamma * pp) * dtdz;
                double sA0 = (u * dBy + B * duy - v * dAy - A * dvy) * dtdy + (u * dCz + C * duz - w * dAz - A * dwz) * dtdz;
                double sB0 = (v * dAx + A * dvx - u * dBx - B * dux) * dtdx + (v * dCz + C * dvz - w * dBz - B * dwz) * dtdz;
                double sC0 = (w * dAx + A * dwx - u * dCx - C * dux) * dtdx + (w * dBy + B * dwy - v * dCy - C * dvy) * dtdy;
                if ((Omega0 > zero) && !fargo) {
                    double shear = -1.5 * Omega0 * XC(i);
                    sr0 = sr0 - shear * dry * dtdy;
                    su0 = su0 - shear * duy * dtdy;
                    sv0 = sv0 - shear * dvy * dtdy;
                    sw0 = sw0 - shear * dwy * dtdy;
                    sp0 = sp0 - shear * dpy * dtdy;
                    sA0 = sA0 - shear * dAy * dtdy;
                    sB0 = sB0 + (shear * dAx - 1.5 * Omega0 * A * dx) * dtdx + shear * dBz * dtdz;
                    sC0 = sC0 - shear * dCy * dtdy;
                }
                double sAL0 = +(GLR - GLL) * dtdy * half - (FLR - FLL) * dtdz * half;
                double sAR0 = +(GRR - GRL) * dtdy * half - (FRR - FRL) * dtdz * half;
                double sBL0 = -(GRL - GLL) * dtdx * half + (ELR - ELL) * dtdz * half;
                double sBR0 = -(GRR - GLR) * dtdx * half + (ERR - ERL) * dtdz * half;
                double sCL0 = +(FRL - FLL) * dtdx * half - (ERL - ELL) * dtdy * half;
                double sCR0 = +(FRR - FLR) * dtdx * half - (ERR - ELR) * dtdy * half;

                r = r + sr0; u = u + su0; v = v + sv0; w = w + sw0; pp = pp + sp0;
                A = A + sA0; B = B + sB0; C = C + sC0;
                AL = AL + sAL0; AR = AR + sAR0; BL = BL + sBL0; BR = BR + sBR0; CL = CL + sCL0; CR = CR + sCR0;

                /* face states, scheme.f90:1489-1553 */
                PUT8(s->qp, i, j, k, 1, r - drx, u - dux, v - dvx, w - dwx, pp - dpx, AL, B - dBx, C - dCx);
                PUT8(s->qm, i, j, k, 1, r + drx, u + dux, v + dvx, w + dwx, pp + dpx, AR, B + dBx, C + dCx);
                PUT8(s->qp, i, j, k, 2, r - dry, u - duy, v - dvy, w - dwy, pp - dpy, A - dAy, BL, C - dCy);
                PUT8(s->qm, i, j, k, 2, r + dry, u + duy, v + dvy, w + dwy, pp + dpy, A + dAy, BR, C + dCy);
                PUT8(s->qp, i, j, k, 3, r - drz, u - duz, v - dvz, w - dwz, pp - dpz, A - dAz, B - dBz, CL);
                PUT8(s->qm, i, j, k, 3, r + drz, u + duz, v + dvz, w + dwz, pp + dpz, A + dAz, B + dBz, CR);
                /* x-edge corners, scheme.f90:1555-1601 */
                PUT8(s->qRT, i, j, k, 1, r + (+dry + drz), u + (+duy + duz), v + (+dvy + dvz), w + (+dwy + dwz),
                     pp + (+dpy + dpz), A + (+dAy + dAz), BR + dBRz, CR + dCRy);
                PUT8(s->qRB, i, j, k, 1, r + (+dry - drz), u + (+duy - duz), v + (+dvy - dvz), w + (+dwy - dwz),
                     pp + (+dpy - dpz), A + (+dAy - dAz), BR - dBRz, CL + dCLy);
                PUT8(s->qLT, i, j, k, 1, r + (-dry + drz), u + (-duy + duz), v + (-dvy + dvz), w + (-dwy + dwz),
                     pp + (-dpy + dpz), A + (-dAy + dAz), BL + dBLz, CR - dCRy);
                PUT8(s->qLB, i, j, k, 1, r + (-dry - drz), u + (-duy - duz), v + (-dvy - dvz), w + (-dwy - dwz),
                     pp + (-dpy - dpz), A + (-dAy - dAz), BL - dBLz, CL - dCLy);
                /* y-edge corners, scheme.f90:1603-1649 */
                PUT8(s->qRT, i, j, k, 2, r + (+drx + drz), u + (+dux + duz), v + (+dvx + dvz), w + (+dwx + dwz),
                     pp + (+dpx + dpz), AR + dARz, B + (+dBx + dBz), CR + dCRx);
                PUT8(s->qRB, i, j, k, 2, r + (+drx - drz), u + (+dux - duz), v + (+dvx - dvz), w + (+dwx - dwz),
                     pp + (+dpx - dpz), AR - dARz, B + (+dBx - dBz), CL + dCLx);
                PUT8(s->qLT, i, j, k, 2, r + (-drx + drz), u + (-dux + duz), v + (-dvx + dvz), w + (-dwx + dwz),
                     pp + (-dpx + dpz), AL + dALz, B + (-dBx + dBz), CR - dCRx);
                PUT8(s->qLB, i, j, k, 2, r + (-drx - drz), u + (-dux - duz), v + (-dvx - dvz), w + (-dwx - dwz),
                     pp + (-dpx - dpz), AL - dALz, B + (-dBx - dBz), CL - dCLx);
                /* z-edge corners, scheme.f90:1651-1697 */
                PUT8(s->qRT, i, j, k, 3, r + (+drx + dry), u + (+dux + duy), v + (+dvx + dvy), w + (+dwx + dwy),
                     pp + (+dpx + dpy), AR + dARy, BR + dBRx, C + (+dCx + dCy));
                PUT8(s->qRB, i, j, k, 3, r + (+drx - dry), u + (+dux - duy), v + (+dvx - dvy), w + (+dwx - dwy),
                     pp + (+dpx - dpy), AR - dARy, BL + dBLx, C + (+dCx - dCy));
                PUT8(s->qLT, i, j, k, 3, r + (-drx + dry), u + (-dux + duy), v + (-dvx + dvy), w + (-dwx + dwy),
                     pp + (-dpx + dpy), AL + dALy, BR - dBRx, C + (-dCx + dCy));
                PUT8(s->qLB, i, j, k, 3, r + (-drx - dry), u + (-dux - duy), v + (-dvx - dvy), w + (-dwx - dwy),
                     pp + (-dpx - dpy), AL - dALy, BL - dBLx, C + (-dCx - dCy));
            }
}

/* trace2d, scheme.f90:807-1143 (Cartesian branch) */
/* trace1d, scheme.f90:661-805 (Cartesian): the predicted cell state and its face states in x;
 * the face B_x is the cell-centred value, the density has a floor, the pressure none, and the
 * rotation term of :777-781 changes only the local sC0 after its last use (no effect) */
static void trace1d(or_state *s, double dt)
{
    const dg_params *p = &s->p;
    const double gamma = p->gamma;
    int ilo = MN(1, s->iu1 + 1), ihi = MX(1, s->iu2 - 1);
    int jlo = MN(1, s->ju1 + 1), jhi = MX(1, s->ju2 - 1);
    int klo = MN(1, s->ku1 + 1), khi = MX(1, s->ku2 - 1);
    const double dtdx = dt / s->dx;
    const farr q = s->qin;
#pragma omp parallel for schedule(static)
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                double r = A4(q, i, j, k, ir), u = A4(q, i, j, k, iu), v = A4(q, i, j, k, iv), w = A4(q, i, j, k, iw);
                double pp = A4(q, i, j, k, ip), A = A4(q, i, j, k, iA), B = A4(q, i, j, k, iB), C = A4(q, i, j, k, iC);
                double drx = half * A5(s->dq, i, j, k, ir, 1), dux = half * A5(s->dq, i, j, k, iu, 1);
                double dvx = half * A5(s->dq, i, j, k, iv, 1), dwx = half * A5(s->dq, i, j, k, iw, 1);
                double dpx = half * A5(s->dq, i, j, k, ip, 1), dBx = half * A5(s->dq, i, j, k, iB, 1);
                double dCx = half * A5(s->dq, i, j, k, iC, 1);
                double sr0 = -u * drx - r * dux;                   sr0 = sr0 * dtdx;
                double su0 = -u * dux - (dpx + B * dBx + C * dCx) / r; su0 = su0 * dtdx;
                double sv0 = -u * dvx + (A * dBx) / r;              sv0 = sv0 * dtdx;
                double sw0 = -u * dwx + (A * dCx) / r;              sw0 = sw0 * dtdx;
                double sp0 = -u * dpx - gamma * pp * dux;          sp0 = sp0 * dtdx;
                double sB0 = -u * dBx + A * dvx - B * dux;          sB0 = sB0 * dtdx;
                double sC0 = -u * dCx + A * dwx - C * dux;          sC0 = sC0 * dtdx;
                r = r + sr0; u = u + su0; v = v + sv0; w = w + sw0; pp = pp + sp0; B = B + sB0; C = C + sC0;
                A5(s->qp, i, j, k, ir, 1) = r - drx;
                A5(s->qp, i, j, k, iu, 1) = u - dux;
                A5(s->qp, i, j, k, iv, 1) = v - dvx;
                A5(s->qp, i, j, k, iw, 1) = w - dwx;
                A5(s->qp, i, j, k, ip, 1) = pp - dpx;
                A5(s->qp, i, j, k, iA, 1) = A;
                A5(s->qp, i, j, k, iB, 1) = B - dBx;
                A5(s->qp, i, j, k, iC, 1) = C - dCx;
                A5(s->qp, i, j, k, ir, 1) = MX(smallr, A5(s->qp, i, j, k, ir, 1));
                A5(s->qm, i, j, k, ir, 1) = r + drx;
                A5(s->qm, i, j, k, iu, 1) = u + dux;
                A5(s->qm, i, j, k, iv, 1) = v + dvx;
                A5(s->qm, i, j, k, iw, 1) = w + dwx;
                A5(s->qm, i, j, k, ip, 1) = pp + dpx;
                A5(s->qm, i, j, k, iA, 1) = A;
                A5(s->qm, i, j, k, iB, 1) = B + dBx;
                A5(s->qm, i, j, k, iC, 1) = C + dCx;
                A5(s->qm, i, j, k, ir, 1) = MX(smallr, A5(s->qm, i, j, k, ir, 1));
            }
}

static void trace2d(or_state *s, double dt)
{
    const dg_params *p = &s->p;
    const double gamma = p->gamma, Omega0 = p->omega0;
    const double smallp = smallr * (smallc * smallc) / gamma;
    int ilo = MN(1, s->iu1 + 1), ihi = MX(1, s->iu2 - 1);
    int jlo = MN(1, s->ju1 + 1), jhi = MX(1, s->ju2 - 1);
    int klo = MN(1, s->ku1 + 1), khi = MX(1, s->ku2 - 1);
    const double dtdx = dt / s->dx, dtdy = dt / s->dy;
    const farr q = s->qin, bfc = s->bfc;

    /* scheme.f90:856-872 */
#pragma omp parallel for schedule(static)
    for (int k = klo; k <= s->ku2; k++)
        for (int j = jlo; j <= s->ju2; j++)
            for (int i = ilo; i <= s->iu2; i++) {
                double u = 0.25 * (A4(q, i - 1, j - 1, k, iu) + A4(q, i - 1, j, k, iu) + A4(q, i, j - 1, k, iu) + A4(q, i, j, k, iu));
                double v = 0.25 * (A4(q, i - 1, j - 1, k, iv) + A4(q, i - 1, j, k, iv) + A4(q, i, j - 1, k, iv) + A4(q, i, j, k, iv));
                double A = 0.5 * (A4(bfc, i, j - 1, k, 1) + A4(bfc, i, j, k, 1));
                double B = 0.5 * (A4(bfc, i - 1, j, k, 2) + A4(bfc, i, j, k, 2));
                A3(s->Ez, i, j, k) = u * B - v * A;
            }

#pragma omp parallel for schedule(static)
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                double r = A4(q, i, j, k, ir), u = A4(q, i, j, k, iu), v = A4(q, i, j, k, iv), w = A4(q, i, j, k, iw);
                double pp = A4(q, i, j, k, ip), A = A4(q, i, j, k, iA), B = A4(q, i, j, k, iB), C = A4(q, i, j, k, iC);
                double AL = A4(bfc, i, j, k, 1), AR = A4(bfc, i + 1, j, k, 1);
                double BL = A4(bfc, i, j, k, 2), BR = A4(bfc, i, j + 1, k, 2);
                double ELL = A3(s->Ez, i, j, k), ELR = A3(s->Ez, i, j + 1, k);
                double ERL = A3(s->Ez, i + 1, j, k), ERR = A3(s->Ez, i + 1, j + 1, k);
                double drx = half * A5(s->dq, i, j, k, ir, 1), dux = half * A5(s->dq, i, j, k, iu, 1);
                double dvx = half * A5(s->dq, i, j, k, iv, 1), dwx = half * A5(s->dq, i, j, k, iw, 1);
                double dCx = half * A5(s->dq, i, j, k, iC, 1), dpx = half * A5(s->dq, i, j, k, ip, 1);
                double dBx = half * A5(s->dq, i, j, k, iB, 1);
                double dry = half * A5(s->dq, i, j, k, ir, 2), duy = half * A5(s->dq, i, j, k, iu, 2);
                double dvy = half * A5(s->dq, i, j, k, iv, 2), dwy = half * A5(s->dq, i, j, k, iw, 2);
                double dCy = half * A5(s->dq, i, j, k, iC, 2), dpy = half * A5(s->dq, i, j, k, ip, 2);
                double dAy = half * A5(s->dq, i, j, k, iA, 2);
                double dALy = half * A5(s->dbfc, i, j, k, 1, 2), dARy = half * A5(s->dbfc, i + 1, j, k, 1, 2);
                double dBLx = half * A5(s->dbfc, i, j, k, 2, 1), dBRx = half * A5(s->dbfc, i, j + 1, k, 2, 1);
                double dAx = half * (AR - AL), dBy = half * (BR - BL);

                /* scheme.f90:946-967 */
                double sr0 = (-u * drx - dux * r) * dtdx + (-v * dry - dvy * r) * dtdy;
                double su0 = (-u * dux - dpx / r - B * dBx / r - C * dCx / r) * dtdx + (-v * duy + B * dAy / r) * dtdy;
                double sv0 = (-u * dvx + A * dBx / r) * dtdx + (-v * dvy - dpy / r - A * dAy / r - C * dCy / r) * dtdy;
                double sw0 = (-u * dwx + A * dCx / r) * dtdx + (-v * dwy + B * dCy / r) * dtdy;
                double sp0 = (-u * dpx - dux * gamma * pp) * dtdx + (-v * dpy - dvy * gamma * pp) * dtdy;
                double sA0 = (u * dBy + B * duy - v * dAy - A * dvy) * dtdy;
                double sB0 = (-u * dBx - B * dux + v * dAx + A * dvx) * dtdx;
                double sC0 = (w * dAx + A * dwx - u * dCx - C * dux) * dtdx + (-v * dCy - C * dvy + w * dBy + B * dwy) * dtdy;
                if (Omega0 > zero) {
                    double shear = -1.5 * Omega0 * XC(i);
                    sC0 = sC0 + (shear * dAx - 1.5 * Omega0 * A) * dtdx + shear * dBy * dtdy;
                }
                double sAL0 = +(ELR - ELL) * half * dtdy;
                double sAR0 = +(ERR - ERL) * half * dtdy;
                double sBL0 = -(ERL - ELL) * half * dtdx;
                double sBR0 = -(ERR - ELR) * half * dtdx;

                r = r + sr0; u = u + su0; v = v + sv0; w = w + sw0; pp = pp + sp0;
                A = A + sA0; B = B + sB0; C = C + sC0;
                AL = AL + sAL0; AR = AR + sAR0; BL = BL + sBL0; BR = BR + sBR0;

                /* scheme.f90:1062-1139 */
                PUT8(s->qp, i, j, k, 1, r - drx, u - dux, v - dvx, w - dwx, pp - dpx, AL, B - dBx, C - dCx);
                PUT8(s->qm, i, j, k, 1, r + drx, u + dux, v + dvx, w + dwx, pp + dpx, AR, B + dBx, C + dCx);
                PUT8(s->qp, i, j, k, 2, r - dry, u - duy, v - dvy, w - dwy, pp - dpy, A - dAy, BL, C - dCy);
                PUT8(s->qm, i, j, k, 2, r + dry, u + duy, v + dvy, w + dwy, pp + dpy, A + dAy, BR, C + dCy);
                PUT8(s->qRT, i, j, k, 3, r + (+drx + dry), u + (+dux + duy), v + (+dvx + dvy), w + (+dwx + dwy),
                     pp + (+dpx + dpy), AR + (+dARy), BR + (+dBRx), C + (+dCx + dCy));
                PUT8(s->qRB, i, j, k, 3, r + (+drx - dry), u + (+dux - duy), v + (+dvx - dvy), w + (+dwx - dwy),
                     pp + (+dpx - dpy), AR + (-dARy), BL + (+dBLx), C + (+dCx - dCy));
                PUT8(s->qLB, i, j, k, 3, r + (-drx - dry), u + (-dux - duy), v + (-dvx - dvy), w + (-dwx - dwy),
                     pp + (-dpx - dpy), AL + (-dALy), BL + (-dBLx), C + (-dCx - dCy));
                PUT8(s->qLT, i, j, k, 3, r + (-drx + dry), u + (-dux + duy), v + (-dvx + dvy), w + (-dwx + dwy),
                     pp + (-dpx + dpy), AL + (+dALy), BR + (-dBRx), C + (-dCx + dCy));
            }
}

/* ------------------------------------------------------------------------- */
/* 1D Riemann solvers, src/modules/solvers/solver.f90                         */
/* states: 1 rho, 2 P, 3 u_n, 4 B_n, 5 v_t1, 6 B_t1, 7 v_t2, 8 B_t2           */
/* ------------------------------------------------------------------------- */
typedef struct { double r, pg, u, v, w, b, c, p; } gstar_t;

static inline double cfast(double gamma, double ploc, double rho, double a, double b, double c)
{
    double c2 = gamma * ploc / rho;
    double b2 = a * a + b * b + c * c;
    double d2 = half * (c2 + b2 / rho);
    return sqrt(d2 + sqrt(d2 * d2 - c2 * a * a / rho));
}

/* llf (solver.f90:393-498), hll (:504-612), upwind (:842-935): shared flux pieces */
static void lr_fluxes(const double *ql, const double *qr, double gamma, double ciso, int iso,
                      double *fl, double *cl, double *fr, double *cr, double *ploc_o, double *proc_o, double *a_o)
{
    double rl = ql[0], pl = ql[1], ul = ql[2], al = ql[3], vl = ql[4], bl = ql[5], wl = ql[6], clv = ql[7];
    double rr = qr[0], pr = qr[1], ur = qr[2], ar = qr[3], vr = qr[4], br = qr[5], wr = qr[6], crv = qr[7];
    double entho = one / (gamma - one);
    double a = half * (al + ar);
    al = a; ar = a;
    double ploc, proc;
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); }
    else { ploc = pl; proc = pr; }
    double ecin = half * (ul * ul + vl * vl + wl * wl) * rl;
    double emag = half * (a * a + bl * bl + clv * clv);
    double etot = ploc * entho + ecin + emag;
    double ptot = ploc + emag;
    fl[0] = rl * ul;
    fl[1] = (etot + ptot) * ul - al * (ul * al + vl * bl + wl * clv);
    fl[2] = rl * ul * ul + ptot - al * al;
    fl[3] = zero;
    fl[4] = rl * ul * vl - al * bl;
    fl[5] = bl * ul - al * vl;
    fl[6] = rl * ul * wl - al * clv;
    fl[7] = clv * ul - al * wl;
    cl[0] = rl; cl[1] = etot; cl[2] = rl * ul; cl[3] = al; cl[4] = rl * vl; cl[5] = bl; cl[6] = rl * wl; cl[7] = clv;
    ecin = half * (ur * ur + vr * vr + wr * wr) * rr;
    emag = half * (a * a + br * br + crv * crv);
    etot = proc * entho + ecin + emag;
    ptot = proc + emag;
    fr[0] = rr * ur;
    fr[1] = (etot + ptot) * ur - ar * (ur * ar + vr * br + wr * crv);
    fr[2] = rr * ur * ur + ptot - ar * ar;
    fr[3] = zero;
    fr[4] = rr * ur * vr - ar * br;
    fr[5] = br * ur - ar * vr;
    fr[6] = rr * ur * wr - ar * crv;
    fr[7] = crv * ur - ar * wr;
    cr[0] = rr; cr[1] = etot; cr[2] = rr * ur; cr[3] = ar; cr[4] = rr * vr; cr[5] = br; cr[6] = rr * wr; cr[7] = crv;
    *ploc_o = ploc; *proc_o = proc; *a_o = a;
}

static void llf1d(const double *ql, const double *qr, double *f, double gamma, double ciso, int iso)
{
    double fl[8], cl[8], fr[8], cr[8], ploc, proc, a;
    lr_fluxes(ql, qr, gamma, ciso, iso, fl, cl, fr, cr, &ploc, &proc, &a);
    double vleft = cfast(gamma, ploc, ql[0], a, ql[5], ql[7]) + fabs(ql[2]);
    double vright = cfast(gamma, proc, qr[0], a, qr[5], qr[7]) + fabs(qr[2]);
    double vel_info = MX(vleft, vright);
    for (int n = 0; n < 8; n++) f[n] = half * (fl[n] + fr[n]) - vel_info * half * (cr[n] - cl[n]);
}

static void hll1d(const double *ql, const double *qr, double *f, double gamma, double ciso, int iso)
{
    double fl[8], cl[8], fr[8], cr[8], ploc, proc, a;
    lr_fluxes(ql, qr, gamma, ciso, iso, fl, cl, fr, cr, &ploc, &proc, &a);
    double vleft = cfast(gamma, ploc, ql[0], a, ql[5], ql[7]);
    double vright = cfast(gamma, proc, qr[0], a, qr[5], qr[7]);
    double ul = ql[2], ur = qr[2];
    double sl = MN(MN(ul, ur) - MX(vleft, vright), zero);
    double sr = MX(MX(ul, ur) + MX(vleft, vright), zero);
    for (int n = 0; n < 8; n++) f[n] = (sr * fl[n] - sl * fr[n] + sr * sl * (cr[n] - cl[n])) / (sr - sl);
}

static void upwind1d(const double *ql, const double *qr, double *f, double gamma, double ciso, int iso)
{
    double fl[8], cl[8], fr[8], cr[8], ploc, proc, a;
    lr_fluxes(ql, qr, gamma, ciso, iso, fl, cl, fr, cr, &ploc, &proc, &a);
    double vleft = half * (ql[2] + qr[2]);
    for (int n = 0; n < 8; n++) f[n] = half * (fl[n] + fr[n]) - fabs(vleft) * half * (cr[n] - cl[n]);
}

/* hlld, solver.f90:618-836 */
static void hlld1d(const double *ql, const double *qr, double *f, gstar_t *g, double gamma, double ciso, int iso)
{
    double rl = ql[0], pl = ql[1], ul = ql[2], al = ql[3], vl = ql[4], bl = ql[5], wl = ql[6], cl = ql[7];
    double rr = qr[0], pr = qr[1], ur = qr[2], ar = qr[3], vr = qr[4], br = qr[5], wr = qr[6], cr = qr[7];
    double entho = one / (gamma - one);
    double a = half * (al + ar);
    double sgnm = SGN1(a);
    double ploc, proc;
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); }
    else { ploc = pl; proc = pr; }
    double ecinl = half * (ul * ul + vl * vl + wl * wl) * rl;
    double emagl = half * (a * a + bl * bl + cl * cl);
    double etotl = ploc * entho + ecinl + emagl;
    double ptotl = ploc + emagl;
    double vdotbl = ul * a + vl * bl + wl * cl;
    double ecinr = half * (ur * ur + vr * vr + wr * wr) * rr;
    double emagr = half * (a * a + br * br + cr * cr);
    double etotr = proc * entho + ecinr + emagr;
    double ptotr = proc + emagr;
    double vdotbr = ur * a + vr * br + wr * cr;
    double cfastl = cfast(gamma, ploc, rl, a, bl, cl);
    double cfastr = cfast(gamma, proc, rr, a, br, cr);
    double sl = MN(ul, ur) - MX(cfastl, cfastr);
    double sr = MX(ul, ur) + MX(cfastl, cfastr);
    double rcl = rl * (ul - sl);
    double rcr = rr * (sr - ur);
    double ustar = (rcr * ur + rcl * ul + (ptotl - ptotr)) / (rcr + rcl);
    double ptotstar = (rcr * ptotl + rcl * ptotr + rcl * rcr * (ul - ur)) / (rcr + rcl);
    double rstarl = rl * (sl - ul) / (sl - ustar);
    double estar = rl * (sl - ul) * (sl - ustar) - a * a;
    double el = rl * (sl - ul) * (sl - ul) - a * a;
    double vstarl, bstarl, wstarl, cstarl;
    if (estar == zero) { vstarl = vl; bstarl = bl; wstarl = wl; cstarl = cl; }
    else {
        vstarl = vl - a * bl * (ustar - ul) / estar;
        bstarl = bl * el / estar;
        wstarl = wl - a * cl * (ustar - ul) / estar;
        cstarl = cl * el / estar;
    }
    double vdotbstarl = ustar * a + vstarl * bstarl + wstarl * cstarl;
    double etotstarl = ((sl - ul) * etotl - ptotl * ul + ptotstar * ustar + a * (vdotbl - vdotbstarl)) / (sl - ustar);
    double sqrrstarl = sqrt(rstarl);
    double calfvenl = fabs(a) / sqrrstarl;
    double sal = ustar - calfvenl;
    double rstarr = rr * (sr - ur) / (sr - ustar);
    estar = rr * (sr - ur) * (sr - ustar) - a * a;
    double er = rr * (sr - ur) * (sr - ur) - a * a;
    double vstarr, bstarr, wstarr, cstarr;
    if (estar == zero) { vstarr = vr; bstarr = br; wstarr = wr; cstarr = cr; }
    else {
        vstarr = vr - a * br * (ustar - ur) / estar;
        bstarr = br * er / estar;
        wstarr = wr - a * cr * (ustar - ur) / estar;
        cstarr = cr * er / estar;
    }
    double vdotbstarr = ustar * a + vstarr * bstarr + wstarr * cstarr;
    double etotstarr = ((sr - ur) * etotr - ptotr * ur + ptotstar * ustar + a * (vdotbr - vdotbstarr)) / (sr - ustar);
    double sqrrstarr = sqrt(rstarr);
    double calfvenr = fabs(a) / sqrrstarr;
    double sar = ustar + calfvenr;
    double vstarstar = (sqrrstarl * vstarl + sqrrstarr * vstarr + sgnm * (bstarr - bstarl)) / (sqrrstarl + sqrrstarr);
    double wstarstar = (sqrrstarl * wstarl + sqrrstarr * wstarr + sgnm * (cstarr - cstarl)) / (sqrrstarl + sqrrstarr);
    double bstarstar = (sqrrstarl * bstarr + sqrrstarr * bstarl + sgnm * sqrrstarl * sqrrstarr * (vstarr - vstarl))
                     / (sqrrstarl + sqrrstarr);
    double cstarstar = (sqrrstarl * cstarr + sqrrstarr * cstarl + sgnm * sqrrstarl * sqrrstarr * (wstarr - wstarl))
                     / (sqrrstarl + sqrrstarr);
    double vdotbstarstar = ustar * a + vstarstar * bstarstar + wstarstar * cstarstar;
    double etotstarstarl = etotstarl - sgnm * sqrrstarl * (vdotbstarl - vdotbstarstar);
    double etotstarstarr = etotstarr + sgnm * sqrrstarr * (vdotbstarr - vdotbstarstar);
    double ro, uo, vo, wo, bo, co, ptoto, etoto, vdotbo;
    if (sl > zero) {
        ro = rl; uo = ul; vo = vl; wo = wl; bo = bl; co = cl; ptoto = ptotl; etoto = etotl; vdotbo = vdotbl;
    } else if (sal > zero) {
        ro = rstarl; uo = ustar; vo = vstarl; wo = wstarl; bo = bstarl; co = cstarl;
        ptoto = ptotstar; etoto = etotstarl; vdotbo = vdotbstarl;
    } else if (ustar > zero) {
        ro = rstarl; uo = ustar; vo = vstarstar; wo = wstarstar; bo = bstarstar; co = cstarstar;
        ptoto = ptotstar; etoto = etotstarstarl; vdotbo = vdotbstarstar;
    } else if (sar > zero) {
        ro = rstarr; uo = ustar; vo = vstarstar; wo = wstarstar; bo = bstarstar; co = cstarstar;
        ptoto = ptotstar; etoto = etotstarstarr; vdotbo = vdotbstarstar;
    } else if (sr > zero) {
        ro = rstarr; uo = ustar; vo = vstarr; wo = wstarr; bo = bstarr; co = cstarr;
        ptoto = ptotstar; etoto = etotstarr; vdotbo = vdotbstarr;
    } else {
        ro = rr; uo = ur; vo = vr; wo = wr; bo = br; co = cr; ptoto = ptotr; etoto = etotr; vdotbo = vdotbr;
    }
    f[0] = ro * uo;
    f[1] = (etoto + ptoto) * uo - a * vdotbo;
    f[2] = ro * uo * uo - a * a;
    f[3] = zero;
    f[4] = ro * uo * vo - a * bo;
    f[5] = bo * uo - a * vo;
    f[6] = ro * uo * wo - a * co;
    f[7] = co * uo - a * wo;
    g->r = ro; g->u = uo; g->v = vo; g->w = wo; g->b = bo; g->c = co; g->p = ptoto;
}

/* riemann_solver, solver.f90:65-387 (Cartesian) */
static void riemann_solver(or_state *s, double dt)
{
    const dg_params *p = &s->p;
    const double gamma = p->gamma, ciso = p->ciso, Omega0 = p->omega0;
    const int iso = p->iso, fargo = p->fargo, ndim = s->ndim;
    memset(s->rgstar.d, 0, sizeof(double) * s->rgstar.size);
    memset(s->ugstar.d, 0, sizeof(double) * s->ugstar.size);
    memset(s->vgstar.d, 0, sizeof(double) * s->vgstar.size);
    memset(s->wgstar.d, 0, sizeof(double) * s->wgstar.size);
    memset(s->bgstar.d, 0, sizeof(double) * s->bgstar.size);
    memset(s->cgstar.d, 0, sizeof(double) * s->cgstar.size);
    memset(s->pgstar.d, 0, sizeof(double) * s->pgstar.size);
    for (int idim = 1; idim <= ndim; idim++) {
        int ln, lt1, lt2, bn, bt1, bt2, ilo, ihi, jlo, jhi, klo, khi, io, jo, ko;
        if (idim == 1) {
            ln = 2; lt1 = 3; lt2 = 4; bn = 6; bt1 = 7; bt2 = 8;
            ilo = s->if1; ihi = s->if2;
            jlo = MN(1, s->ju1 + 3); jhi = MX(1, s->ju2 - 3);
            klo = MN(1, s->ku1 + 3); khi = MX(1, s->ku2 - 3);
            io = 1; jo = 0; ko = 0;
        } else if (idim == 2) {
            ln = 3; lt1 = 2; lt2 = 4; bn = 7; bt1 = 6; bt2 = 8;
            ilo = MN(1, s->iu1 + 3); ihi = MX(1, s->iu2 - 3);
            jlo = s->jf1; jhi = s->jf2;
            klo = MN(1, s->ku1 + 3); khi = MX(1, s->ku2 - 3);
            io = 0; jo = 1; ko = 0;
        } else {
            ln = 4; lt1 = 2; lt2 = 3; bn = 8; bt1 = 6; bt2 = 7;
            ilo = MN(1, s->iu1 + 3); ihi = MX(1, s->iu2 - 3);
            jlo = MN(1, s->ju1 + 3); jhi = MX(1, s->ju2 - 3);
            klo = s->kf1; khi = s->kf2;
            io = 0; jo = 0; ko = 1;
        }
#pragma omp parallel for schedule(static)
        for (int k = klo; k <= khi; k++)
            for (int j = jlo; j <= jhi; j++)
                for (int i = ilo; i <= ihi; i++) {
                    int im = i - io, jm = j - jo, km = k - ko;
                    double ql[8], qr[8], f[8];
                    double bn_mean = half * (A5(s->qm, im, jm, km, bn, idim) + A5(s->qp, i, j, k, bn, idim));
                    ql[0] = A5(s->qm, im, jm, km, 1, idim);
                    ql[1] = A5(s->qm, im, jm, km, 5, idim);
                    ql[2] = A5(s->qm, im, jm, km, ln, idim);
                    ql[3] = bn_mean;
                    ql[4] = A5(s->qm, im, jm, km, lt1, idim);
                    ql[5] = A5(s->qm, im, jm, km, bt1, idim);
                    ql[6] = A5(s->qm, im, jm, km, lt2, idim);
                    ql[7] = A5(s->qm, im, jm, km, bt2, idim);
                    qr[0] = A5(s->qp, i, j, k, 1, idim);
                    qr[1] = A5(s->qp, i, j, k, 5, idim);
                    qr[2] = A5(s->qp, i, j, k, ln, idim);
                    qr[3] = bn_mean;
                    qr[4] = A5(s->qp, i, j, k, lt1, idim);
                    qr[5] = A5(s->qp, i, j, k, bt1, idim);
                    qr[6] = A5(s->qp, i, j, k, lt2, idim);
                    qr[7] = A5(s->qp, i, j, k, bt2, idim);
                    int have = 1;
                    if (p->iriemann == DG_RIEMANN_HLLD) {
                        gstar_t g;
                        hlld1d(ql, qr, f, &g, gamma, ciso, iso);
                        A3(s->rgstar, i, j, k) = g.r; A3(s->ugstar, i, j, k) = g.u; A3(s->vgstar, i, j, k) = g.v;
                        A3(s->wgstar, i, j, k) = g.w; A3(s->bgstar, i, j, k) = g.b; A3(s->cgstar, i, j, k) = g.c;
                        A3(s->pgstar, i, j, k) = g.p;
                    } else if (p->iriemann == DG_RIEMANN_HLL) hll1d(ql, qr, f, gamma, ciso, iso);
                    else if (p->iriemann == DG_RIEMANN_LLF) llf1d(ql, qr, f, gamma, ciso, iso);
                    else if (p->iriemann == DG_RIEMANN_UPWIND) upwind1d(ql, qr, f, gamma, ciso, iso);
                    else have = 0;
                    if (have)
                        for (int n = 0; n < 8; n++) A5(s->fgodunov, i, j, k, n + 1, idim) = f[n];
                    /* shearing-box upwind terms, solver.f90:199-241 */
                    if (ndim == 1) {
                        if (Omega0 > zero) {
                            double shear = -1.5 * Omega0 * (XC(i) + XC(i - 1));
                            A5(s->fgodunov, i, j, k, 8, idim) = A5(s->fgodunov, i, j, k, 8, idim) + shear * bn_mean;
                        }
                    } else if (ndim == 2) {
                        if (Omega0 > zero) {
                            double shear = -1.5 * Omega0 * XC(i);
                            if (idim == 1) shear = -1.5 * Omega0 * (XC(i) + XC(i - 1));
                            if (idim == 2) shear = -1.5 * Omega0 * XC(i);
                            A5(s->fgodunov, i, j, k, 8, idim) = A5(s->fgodunov, i, j, k, 8, idim) + shear * bn_mean;
                        }
                    } else if ((Omega0 > zero) && (idim == 2) && !fargo) {
                        double shear = -1.5 * Omega0 * XC(i);
                        const double *qs = (shear > zero) ? ql : qr;
                        double rs = qs[0], ps = qs[1], us = qs[2], as = qs[3], vs = qs[4], bs = qs[5], ws = qs[6], cs = qs[7];
                        double Emag = half * (as * as + bs * bs + cs * cs);
                        double Ekin = half * (us * us + vs * vs + ws * ws);
                        double Etot = Ekin + Emag + ps / (gamma - one);
                        A5(s->fgodunov, i, j, k, 1, idim) = A5(s->fgodunov, i, j, k, 1, idim) + shear * rs;
                        A5(s->fgodunov, i, j, k, 2, idim) = A5(s->fgodunov, i, j, k, 2, idim) + shear * (Etot + Emag - bn_mean * bn_mean);
                        A5(s->fgodunov, i, j, k, 3, idim) = A5(s->fgodunov, i, j, k, 3, idim) + shear * rs * us;
                        A5(s->fgodunov, i, j, k, 5, idim) = A5(s->fgodunov, i, j, k, 5, idim) + shear * rs * vs;
                        A5(s->fgodunov, i, j, k, 7, idim) = A5(s->fgodunov, i, j, k, 7, idim) + shear * rs * ws;
                    }
                }
        /* pressure term, solver.f90:246-262 */
#pragma omp parallel for schedule(static)
        for (int k = klo; k <= khi - ko; k++)
            for (int j = jlo; j <= jhi - jo; j++)
                for (int i = ilo; i <= ihi - io; i++) {
                    int ii = i + io, ji = j + jo, ki = k + ko;
                    A4(s->fgodunov_pre, i, j, k, idim) =
                        -(A3(s->pgstar, ii, ji, ki) * A4(s->ds, ii, ji, ki, idim) - A3(s->pgstar, i, j, k) * A4(s->ds, i, j, k, idim)) * dt;
                }
    }
}

/* ------------------------------------------------------------------------- */
/* 2D Riemann solvers for edge EMFs, src/modules/solvers/solver_magnetic.f90  */
/* corner state: 1 rho, 2 P, 3 u, 4 v, 5 A, 6 B, 7 C, 8 E                     */
/* ------------------------------------------------------------------------- */
typedef struct {
    double rLL, rLR, rRL, rRR, pLL, pLR, pRL, pRR, uLL, uLR, uRL, uRR;
    double vLL, vLR, vRL, vRR, ALL, ALR, ARL, ARR, BLL, BLR, BRL, BRR;
    double CLL, CLR, CRL, CRR, ELL, ELR, ERL, ERR;
} corners_t;

/* solver_magnetic_utils, solver_magnetic.f90:32-49 */
static void mag_utils(corners_t *c, const double *qLL, const double *qLR, const double *qRL, const double *qRR)
{
    c->rLL = qLL[0]; c->uLL = qLL[2]; c->ALL = qLL[4]; c->CLL = qLL[6];
    c->rRL = qRL[0]; c->uRL = qRL[2]; c->ARL = qRL[4]; c->CRL = qRL[6];
    c->rLR = qLR[0]; c->uLR = qLR[2]; c->ALR = qLR[4]; c->CLR = qLR[6];
    c->rRR = qRR[0]; c->uRR = qRR[2]; c->ARR = qRR[4]; c->CRR = qRR[6];
    c->pLL = qLL[1]; c->vLL = qLL[3]; c->BLL = qLL[5]; c->ELL = qLL[7];
    c->pRL = qRL[1]; c->vRL = qRL[3]; c->BRL = qRL[5]; c->ERL = qRL[7];
    c->pLR = qLR[1]; c->vLR = qLR[3]; c->BLR = qLR[5]; c->ELR = qLR[7];
    c->pRR = qRR[1]; c->vRR = qRR[3]; c->BRR = qRR[5]; c->ERR = qRR[7];
}

static inline double mn4(double a, double b, double c, double d) { return MN(MN(MN(a, b), c), d); }
static inline double mx4(double a, double b, double c, double d) { return MX(MX(MX(a, b), c), d); }

/* llf, solver_magnetic.f90:241-356 */
static double llf2d(const corners_t *c, double dt, double gamma, double ciso, int iso)
{
    double E = forth * (c->ELL + c->ERL + c->ELR + c->ERR);
    double rl = half * (c->rLL + c->rLR), pl = half * (c->pLL + c->pLR), ul = half * (c->uLL + c->uLR);
    double al = half * (c->ALL + c->ALR), bl = half * (c->BLL + c->BLR), cl = half * (c->CLL + c->CLR);
    double rr = half * (c->rRR + c->rRL), pr = half * (c->pRR + c->pRL), ur = half * (c->uRR + c->uRL);
    double ar = half * (c->ARR + c->ARL), br = half * (c->BRR + c->BRL), cr = half * (c->CRR + c->CRL);
    double ploc, proc;
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); } else { ploc = pl; proc = pr; }
    al = half * (al + ar); ar = al;
    double vleft = cfast(gamma, ploc, rl, al, bl, cl) + fabs(ul);
    double vright = cfast(gamma, proc, rr, ar, br, cr) + fabs(ur);
    double vel_info = MX(vleft, vright);
    double flux_x = -vel_info * half * (br - bl);
    rl = half * (c->rLL + c->rRL); pl = half * (c->pLL + c->pRL); ul = half * (c->vLL + c->vRL);
    al = half * (c->BLL + c->BRL); bl = half * (c->ALL + c->ARL); cl = half * (c->CLL + c->CRL);
    rr = half * (c->rRR + c->rLR); pr = half * (c->pRR + c->pLR); ur = half * (c->vRR + c->vLR);
    ar = half * (c->BRR + c->BLR); br = half * (c->ARR + c->ALR); cr = half * (c->CRR + c->CLR);
    if (iso) { ploc = rl * (ciso * ciso); proc = rr * (ciso * ciso); } else { ploc = pl; proc = pr; }
    al = half * (al + ar); ar = al;
    vleft = cfast(gamma, ploc, rl, al, bl, cl) + fabs(ul);
    vright = cfast(gamma, proc, rr, ar, br, cr) + fabs(ur);
    vel_info = MX(vleft, vright);
    double flux_y = -vel_info * half * (br - bl);
    double emf = E + (flux_x - flux_y);
    return emf * dt;
}

/* hlld, solver_magnetic.f90:362-548 */
static double hlld2d(const corners_t *c, double dt, double gamma)
{
    double cfastLLx = cfast(gamma, c->pLL, c->rLL, c->ALL, c->BLL, c->CLL);
    double cfastLRx = cfast(gamma, c->pLR, c->rLR, c->ALR, c->BLR, c->CLR);
    double cfastRLx = cfast(gamma, c->pRL, c->rRL, c->ARL, c->BRL, c->CRL);
    double cfastRRx = cfast(gamma, c->pRR, c->rRR, c->ARR, c->BRR, c->CRR);
    double cfastLLy = cfast(gamma, c->pLL, c->rLL, c->BLL, c->ALL, c->CLL);
    double cfastLRy = cfast(gamma, c->pLR, c->rLR, c->BLR, c->ALR, c->CLR);
    double cfastRLy = cfast(gamma, c->pRL, c->rRL, c->BRL, c->ARL, c->CRL);
    double cfastRRy = cfast(gamma, c->pRR, c->rRR, c->BRR, c->ARR, c->CRR);
    double SL = mn4(c->uLL, c->uLR, c->uRL, c->uRR) - mx4(cfastLLx, cfastLRx, cfastRLx, cfastRRx);
    double SR = mx4(c->uLL, c->uLR, c->uRL, c->uRR) + mx4(cfastLLx, cfastLRx, cfastRLx, cfastRRx);
    double SB = mn4(c->vLL, c->vLR, c->vRL, c->vRR) - mx4(cfastLLy, cfastLRy, cfastRLy, cfastRRy);
    double ST = mx4(c->vLL, c->vLR, c->vRL, c->vRR) + mx4(cfastLLy, cfastLRy, cfastRLy, cfastRRy);
    double PtotLL = c->pLL + half * (c->ALL * c->ALL + c->BLL * c->BLL + c->CLL * c->CLL);
    double PtotLR = c->pLR + half * (c->ALR * c->ALR + c->BLR * c->BLR + c->CLR * c->CLR);
    double PtotRL = c->pRL + half * (c->ARL * c->ARL + c->BRL * c->BRL + c->CRL * c->CRL);
    double PtotRR = c->pRR + half * (c->ARR * c->ARR + c->BRR * c->BRR + c->CRR * c->CRR);
    double rcLLx = c->rLL * (c->uLL - SL), rcRLx = c->rRL * (SR - c->uRL);
    double rcLRx = c->rLR * (c->uLR - SL), rcRRx = c->rRR * (SR - c->uRR);
    double rcLLy = c->rLL * (c->vLL - SB), rcLRy = c->rLR * (ST - c->vLR);
    double rcRLy = c->rRL * (c->vRL - SB), rcRRy = c->rRR * (ST - c->vRR);
    double ustar = (rcLLx * c->uLL + rcLRx * c->uLR + rcRLx * c->uRL + rcRRx * c->uRR + (PtotLL - PtotRL + PtotLR - PtotRR))
                 / (rcLLx + rcLRx + rcRLx + rcRRx);
    double vstar = (rcLLy * c->vLL + rcLRy * c->vLR + rcRLy * c->vRL + rcRRy * c->vRR + (PtotLL - PtotLR + PtotRL - PtotRR))
                 / (rcLLy + rcLRy + rcRLy + rcRRy);
    double SLustar = one / (SL - ustar), SRustar = one / (SR - ustar);
    double SBvstar = one / (SB - vstar), STvstar = one / (ST - vstar);
    double rstarLLx = c->rLL * (SL - c->uLL) * SLustar;
    double BstarLL = c->BLL * (SL - c->uLL) * SLustar;
    double rstarLLy = c->rLL * (SB - c->vLL) * SBvstar;
    double AstarLL = c->ALL * (SB - c->vLL) * SBvstar;
    double rstarLL = c->rLL * (SL - c->uLL) * SLustar * (SB - c->vLL) * SBvstar;
    double EstarLLx = ustar * BstarLL - c->vLL * c->ALL;
    double EstarLLy = c->uLL * c->BLL - vstar * AstarLL;
    double EstarLL = ustar * BstarLL - vstar * AstarLL;
    double rstarLRx = c->rLR * (SL - c->uLR) * SLustar;
    double BstarLR = c->BLR * (SL - c->uLR) * SLustar;
    double rstarLRy = c->rLR * (ST - c->vLR) * STvstar;
    double AstarLR = c->ALR * (ST - c->vLR) * STvstar;
    double rstarLR = c->rLR * (SL - c->uLR) * SLustar * (ST - c->vLR) * STvstar;
    double EstarLRx = ustar * BstarLR - c->vLR * c->ALR;
    double EstarLRy = c->uLR * c->BLR - vstar * AstarLR;
    double EstarLR = ustar * BstarLR - vstar * AstarLR;
    double rstarRLx = c->rRL * (SR - c->uRL) * SRustar;
    double BstarRL = c->BRL * (SR - c->uRL) * SRustar;
    double rstarRLy = c->rRL * (SB - c->vRL) * SBvstar;
    double AstarRL = c->ARL * (SB - c->vRL) * SBvstar;
    double rstarRL = c->rRL * (SR - c->uRL) * SRustar * (SB - c->vRL) * SBvstar;
    double EstarRLx = ustar * BstarRL - c->vRL * c->ARL;
    double EstarRLy = c->uRL * c->BRL - vstar * AstarRL;
    double EstarRL = ustar * BstarRL - vstar * AstarRL;
    double rstarRRx = c->rRR * (SR - c->uRR) * SRustar;
    double BstarRR = c->BRR * (SR - c->uRR) * SRustar;
    double rstarRRy = c->rRR * (ST - c->vRR) * STvstar;
    double AstarRR = c->ARR * (ST - c->vRR) * STvstar;
    double rstarRR = c->rRR * (SR - c->uRR) * SRustar * (ST - c->vRR) * STvstar;
    double EstarRRx = ustar * BstarRR - c->vRR * c->ARR;
    double EstarRRy = c->uRR * c->BRR - vstar * AstarRR;
    double EstarRR = ustar * BstarRR - vstar * AstarRR;
    double sqrtrstarLR = one / sqrt(rstarLR);
    double sqrtrstarRL = one / sqrt(rstarRL);
    double sqrtrstarRR = one / sqrt(rstarRR);
    double sqrtrstarLL = one / sqrt(rstarLL);
    double calfvenL = MX(MX(MX(MX(fabs(c->ALR) / sqrt(rstarLRx), fabs(AstarLR) * sqrtrstarLR),
                               fabs(c->ALL) / sqrt(rstarLLx)), fabs(AstarLL) * sqrtrstarLL), smallc);
    double calfvenR = MX(MX(MX(MX(fabs(c->ARR) / sqrt(rstarRRx), fabs(AstarRR) * sqrtrstarRR),
                               fabs(c->ARL) / sqrt(rstarRLx)), fabs(AstarRL) * sqrtrstarRL), smallc);
    double calfvenB = MX(MX(MX(MX(fabs(c->BLL) / sqrt(rstarLLy), fabs(BstarLL) * sqrtrstarLL),
                               fabs(c->BRL) / sqrt(rstarRLy)), fabs(BstarRL) * sqrtrstarRL), smallc);
    double calfvenT = MX(MX(MX(MX(fabs(c->BLR) / sqrt(rstarLRy), fabs(BstarLR) * sqrtrstarLR),
                               fabs(c->BRR) / sqrt(rstarRRy)), fabs(BstarRR) * sqrtrstarRR), smallc);
    double SAL = MN(ustar - calfvenL, zero), SAR = MX(ustar + calfvenR, zero);
    double SAB = MN(vstar - calfvenB, zero), SAT = MX(vstar + calfvenT, zero);
    double SARSAL = one / (SAR - SAL);
    double SATSAB = one / (SAT - SAB);
    double AstarT = (SAR * AstarRR - SAL * AstarLR) * SARSAL;
    double AstarB = (SAR * AstarRL - SAL * AstarLL) * SARSAL;
    double BstarR = (SAT * BstarRR - SAB * BstarRL) * SATSAB;
    double BstarL = (SAT * BstarLR - SAB * BstarLL) * SATSAB;
    double E;
    if (SB > zero) {
        if (SL > zero) E = c->ELL;
        else if (SR < zero) E = c->ERL;
        else E = (SAR * EstarLLx - SAL * EstarRLx + SAR * SAL * (c->BRL - c->BLL)) * SARSAL;
    } else if (ST < zero) {
        if (SL > zero) E = c->ELR;
        else if (SR < zero) E = c->ERR;
        else E = (SAR * EstarLRx - SAL * EstarRRx + SAR * SAL * (c->BRR - c->BLR)) * SARSAL;
    } else if (SL > zero) {
        E = (SAT * EstarLLy - SAB * EstarLRy - SAT * SAB * (c->ALR - c->ALL)) * SATSAB;
    } else if (SR < zero) {
        E = (SAT * EstarRLy - SAB * EstarRRy - SAT * SAB * (c->ARR - c->ARL)) * SATSAB;
    } else {
        E = (SAL * SAB * EstarRR - SAL * SAT * EstarRL - SAR * SAB * EstarLR + SAR * SAT * EstarLL) * SARSAL * SATSAB
          - SAT * SAB * SATSAB * (AstarT - AstarB) + SAR * SAL * SARSAL * (BstarR - BstarL);
    }
    return E * dt;
}

/* upwind, solver_magnetic.f90:554-600 */
static double upwind2d(const corners_t *c, double dt)
{
    double E = forth * (c->ELL + c->ERL + c->ELR + c->ERR);
    double ul = half * (c->uLL + c->uLR), bl = half * (c->BLL + c->BLR);
    double ur = half * (c->uRR + c->uRL), br = half * (c->BRR + c->BRL);
    double vel_info = half * (ul + ur);
    double flux_x = -fabs(vel_info) * half * (br - bl);
    ul = half * (c->vLL + c->vRL); bl = half * (c->ALL + c->ARL);
    ur = half * (c->vRR + c->vLR); br = half * (c->ARR + c->ALR);
    vel_info = half * (ul + ur);
    double flux_y = -fabs(vel_info) * half * (br - bl);
    double emf = E + (flux_x - flux_y);
    return emf * dt;
}

/* hlla, solver_magnetic.f90:688-727 */
static double hlla2d(const corners_t *c, double dt)
{
    double cLLx = sqrt(c->ALL * c->ALL / c->rLL), cLRx = sqrt(c->ALR * c->ALR / c->rLR);
    double cRLx = sqrt(c->ARL * c->ARL / c->rRL), cRRx = sqrt(c->ARR * c->ARR / c->rRR);
    double cLLy = sqrt(c->BLL * c->BLL / c->rLL), cLRy = sqrt(c->BLR * c->BLR / c->rLR);
    double cRLy = sqrt(c->BRL * c->BRL / c->rRL), cRRy = sqrt(c->BRR * c->BRR / c->rRR);
    double SL = MN(mn4(c->uLL, c->uLR, c->uRL, c->uRR) - MX(mx4(cLLx, cLRx, cRLx, cRRx), smallc), zero);
    double SR = MX(mx4(c->uLL, c->uLR, c->uRL, c->uRR) + MX(mx4(cLLx, cLRx, cRLx, cRRx), smallc), zero);
    double SB = MN(mn4(c->vLL, c->vLR, c->vRL, c->vRR) - MX(mx4(cLLy, cLRy, cRLy, cRRy), smallc), zero);
    double ST = MX(mx4(c->vLL, c->vLR, c->vRL, c->vRR) + MX(mx4(cLLy, cLRy, cRLy, cRRy), smallc), zero);
    double emf = (SL * SB * c->ERR - SL * ST * c->ERL - SR * SB * c->ELR + SR * ST * c->ELL) / (SR - SL) / (ST - SB)
               - ST * SB / (ST - SB) * (c->ARR - c->ALL) + SR * SL / (SR - SL) * (c->BRR - c->BLL);
    return emf * dt;
}

/* riemann_solver_magnetic, solver_magnetic.f90:55-235.  The four corner arrays
 * are passed in the order of the call site (scheme.f90:162-168). */
static void riemann_solver_magnetic(or_state *s, const farr *qRT, const farr *qRB, const farr *qLT, const farr *qLB,
                                    farr *emf, int idim, double dt)
{
    const dg_params *p = &s->p;
    const double gamma = p->gamma, ciso = p->ciso, Omega0 = p->omega0;
    const int iso = p->iso;
    int ilo, ihi, jlo, jhi, klo, khi, ln, lt1, lt2, bn, bt1, bt2;
    int irto, irbo, ilto, ilbo, jrto, jrbo, jlto, jlbo, krto, krbo, klto, klbo;
    if (idim == 1) {
        ilo = MN(1, s->iu1 + 3); ihi = MX(1, s->iu2 - 3); jlo = s->jf1; jhi = s->jf2; klo = s->kf1; khi = s->kf2;
        ln = 2; lt1 = 3; lt2 = 4; bn = 6; bt1 = 7; bt2 = 8;
        irto = 0; irbo = 0; ilto = 0; ilbo = 0; jrto = -1; jrbo = -1; jlto = 0; jlbo = 0;
        krto = -1; krbo = 0; klto = -1; klbo = 0;
    } else if (idim == 2) {
        ilo = s->if1; ihi = s->if2; jlo = MN(1, s->ju1 + 3); jhi = MX(1, s->ju2 - 3); klo = s->kf1; khi = s->kf2;
        ln = 3; lt1 = 4; lt2 = 2; bn = 7; bt1 = 8; bt2 = 6;
        irto = -1; irbo = 0; ilto = -1; ilbo = 0; jrto = 0; jrbo = 0; jlto = 0; jlbo = 0;
        krto = -1; krbo = -1; klto = 0; klbo = 0;
    } else {
        ilo = s->if1; ihi = s->if2; jlo = s->jf1; jhi = s->jf2; klo = MN(1, s->ku1 + 3); khi = MX(1, s->ku2 - 3);
        ln = 4; lt1 = 2; lt2 = 3; bn = 8; bt1 = 6; bt2 = 7;
        irto = -1; irbo = -1; ilto = 0; ilbo = 0; jrto = -1; jrbo = 0; jlto = -1; jlbo = 0;
        krto = 0; krbo = 0; klto = 0; klbo = 0;
    }
    (void)ln;
#pragma omp parallel for schedule(static)
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                int irt = i + irto, irb = i + irbo, ilt = i + ilto, ilb = i + ilbo;
                int jrt = j + jrto, jrb = j + jrbo, jlt = j + jlto, jlb = j + jlbo;
                int krt = k + krto, krb = k + krbo, klt = k + klto, klb = k + klbo;
                double qLL[8], qRL[8], qLR[8], qRR[8];
#define QRT(v) AT(*qRT, irt, jrt, krt, v, idim)
#define QLT(v) AT(*qLT, ilt, jlt, klt, v, idim)
#define QRB(v) AT(*qRB, irb, jrb, krb, v, idim)
#define QLB(v) AT(*qLB, ilb, jlb, klb, v, idim)
                qLL[0] = QRT(1); qRL[0] = QLT(1); qLR[0] = QRB(1); qRR[0] = QLB(1);
                if (iso) {
                    qLL[1] = qLL[0] * (ciso * ciso); qRL[1] = qRL[0] * (ciso * ciso);
                    qLR[1] = qLR[0] * (ciso * ciso); qRR[1] = qRR[0] * (ciso * ciso);
                } else {
                    qLL[1] = QRT(5); qRL[1] = QLT(5); qLR[1] = QRB(5); qRR[1] = QLB(5);
                }
                qLL[2] = QRT(lt1); qRL[2] = QLT(lt1); qLR[2] = QRB(lt1); qRR[2] = QLB(lt1);
                qLL[3] = QRT(lt2); qRL[3] = QLT(lt2); qLR[3] = QRB(lt2); qRR[3] = QLB(lt2);
                qLL[4] = half * (QRT(bt1) + QLT(bt1));
                qRL[4] = half * (QRT(bt1) + QLT(bt1));
                qLR[4] = half * (QRB(bt1) + QLB(bt1));
                qRR[4] = half * (QRB(bt1) + QLB(bt1));
                qLL[5] = half * (QRT(bt2) + QRB(bt2));
                qRL[5] = half * (QLT(bt2) + QLB(bt2));
                qLR[5] = half * (QRT(bt2) + QRB(bt2));
                qRR[5] = half * (QLT(bt2) + QLB(bt2));
                qLL[6] = QRT(bn); qRL[6] = QLT(bn); qLR[6] = QRB(bn); qRR[6] = QLB(bn);
#undef QRT
#undef QLT
#undef QRB
#undef QLB
                qLL[7] = qLL[2] * qLL[5] - qLL[3] * qLL[4];
                qRL[7] = qRL[2] * qRL[5] - qRL[3] * qRL[4];
                qLR[7] = qLR[2] * qLR[5] - qLR[3] * qLR[4];
                qRR[7] = qRR[2] * qRR[5] - qRR[3] * qRR[4];
                corners_t c;
                mag_utils(&c, qLL, qLR, qRL, qRR);
                double emf_tmp = 0.0;
                if (p->iriemann2d == DG_RIEMANN_LLF) emf_tmp = llf2d(&c, dt, gamma, ciso, iso);
                else if (p->iriemann2d == DG_RIEMANN_HLLD) emf_tmp = hlld2d(&c, dt, gamma);
                else if (p->iriemann2d == DG_RIEMANN_UPWIND) emf_tmp = upwind2d(&c, dt);
                else if (p->iriemann2d == DG_RIEMANN_HLLA) emf_tmp = hlla2d(&c, dt);
                if ((Omega0 > zero) && !p->fargo) {
                    if (idim == 1) {
                        double shear = -1.5 * Omega0 * XC(i);
                        if (shear > zero) emf_tmp = emf_tmp + shear * c.BLL * dt;
                        else emf_tmp = emf_tmp + shear * c.BRR * dt;
                    }
                    if (idim == 3) {
                        double shear = -1.5 * Omega0 * half * (XC(i) + XC(i - 1));
                        if (shear > zero) emf_tmp = emf_tmp - shear * c.ALL * dt;
                        else emf_tmp = emf_tmp - shear * c.ARR * dt;
                    }
                }
                A3(*emf, i, j, k) = emf_tmp;
            }
}

/* compflux, scheme.f90:1716-1760 */
static void compflux(or_state *s, double dt)
{
    for (int idim = 1; idim <= s->ndim; idim++) {
        int ln, lt1, lt2, bn, bt1, bt2;
        if (idim == 1) { ln = 2; lt1 = 3; lt2 = 4; bn = 6; bt1 = 7; bt2 = 8; }
        else if (idim == 2) { ln = 3; lt1 = 2; lt2 = 4; bn = 7; bt1 = 6; bt2 = 8; }
        else { ln = 4; lt1 = 2; lt2 = 3; bn = 8; bt1 = 6; bt2 = 7; }
#pragma omp parallel for schedule(static)
        for (int k = s->kf1; k <= s->kf2; k++)
            for (int j = s->jf1; j <= s->jf2; j++)
                for (int i = s->if1; i <= s->if2; i++) {
                    double ds = A4(s->ds, i, j, k, idim);
                    A5(s->flux, i, j, k, ir, idim) = A5(s->fgodunov, i, j, k, 1, idim) * ds * dt;
                    A5(s->flux, i, j, k, ip, idim) = A5(s->fgodunov, i, j, k, 2, idim) * ds * dt;
                    A5(s->flux, i, j, k, ln, idim) = A5(s->fgodunov, i, j, k, 3, idim) * ds * dt;
                    A5(s->flux, i, j, k, bn, idim) = A5(s->fgodunov, i, j, k, 4, idim) * ds * dt;
                    A5(s->flux, i, j, k, lt1, idim) = A5(s->fgodunov, i, j, k, 5, idim) * ds * dt;
                    A5(s->flux, i, j, k, bt1, idim) = A5(s->fgodunov, i, j, k, 6, idim) * ds * dt;
                    A5(s->flux, i, j, k, lt2, idim) = A5(s->fgodunov, i, j, k, 7, idim) * ds * dt;
                    A5(s->flux, i, j, k, bt2, idim) = A5(s->fgodunov, i, j, k, 8, idim) * ds * dt;
                }
    }
}

/* shear offset of the x boundaries at time itime (shearingbox.f90:34-37) */
static void shear_offset(const or_state *s, double itime, double *epsi, int *jp)
{
    const dg_params *p = &s->p;
    double deltay = 1.5 * p->omega0 * (p->xmax - p->xmin) * itime;
    deltay = fmod(deltay, (p->ymax - p->ymin));
    *epsi = fmod(deltay, s->dy);
    *jp = (int)(deltay / s->dy);
}

/* shearing_emf, shearingbox.f90:298-390 (single rank) */
static void shearing_emf(or_state *s, double itime)
{
    double epsi; int jp;
    shear_offset(s, itime, &epsi, &jp);
    const int ny = s->ny, iin = s->iu1 + nghost, iout = s->iu2 - nghost + 1;
    int nj = s->ju2 - s->ju1 + 1, nk = s->ku2 - s->ku1 + 1;
    double *inner = (double *)malloc(sizeof(double) * nj * nk), *outer = (double *)malloc(sizeof(double) * nj * nk);
#define IO(a, j, k) a[((j) - s->ju1) + nj * ((k) - s->ku1)]
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2; j++) {
            IO(inner, j, k) = A3(s->emfy, iin, j, k);
            IO(outer, j, k) = A3(s->emfy, iout, j, k);
        }
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1 + 1; j <= s->ju2; j++) {
            int jremap = j - jp - 1, jremapp = jremap + 1;
            if (jremap <= 0) jremap = jremap + ny;
            if (jremapp <= 0) jremapp = jremapp + ny;
            double eps = one - epsi / s->dy;
            A3(s->emfy, iin, j, k) = A3(s->emfy, iin, j, k) + (one - eps) * IO(outer, jremap, k) + eps * IO(outer, jremapp, k);
            A3(s->emfy, iin, j, k) = half * A3(s->emfy, iin, j, k);
        }
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2 - 1; j++) {
            int jremap = j + jp, jremapp = jremap + 1;
            if (jremap > ny) jremap = jremap - ny;
            if (jremapp > ny) jremapp = jremapp - ny;
            double eps = epsi / s->dy;
            A3(s->emfy, iout, j, k) = A3(s->emfy, iout, j, k) + (one - eps) * IO(inner, jremap, k) + eps * IO(inner, jremapp, k);
            A3(s->emfy, iout, j, k) = half * A3(s->emfy, iout, j, k);
        }
#undef IO
    free(inner); free(outer);
}

/* shearing_flux, shearingbox.f90:207-294 (single rank) */
static void shearing_flux(or_state *s, double itime)
{
    double epsi; int jp;
    shear_offset(s, itime, &epsi, &jp);
    const int ny = s->ny;
    const int jf1 = s->jf1, jf2 = s->jf2, kf1 = s->kf1, kf2 = s->kf2;
    int nj = jf2 + 2 - (jf1 - 1) + 1, nk = kf2 - kf1 + 1;
    /* inner(jf1:jf2+1,kf1:kf2), outer(jf1-1:jf2,kf1:kf2); use a common base jf1-1 */
    double *inner = (double *)calloc((size_t)nj * nk, sizeof(double)), *outer = (double *)calloc((size_t)nj * nk, sizeof(double));
#define IO(a, j, k) a[((j) - (jf1 - 1)) + nj * ((k) - kf1)]
    for (int k = kf1; k <= kf2; k++)
        for (int j = jf1; j <= jf2; j++) {
            IO(inner, j, k) = A5(s->flux, s->if1, j, k, 1, 1);
            IO(outer, j, k) = A5(s->flux, s->if2, j, k, 1, 1);
        }
    const int iin = s->iu1 + nghost, iout = s->iu2 - nghost + 1;
    for (int k = kf1; k <= kf2; k++)
        for (int j = jf1; j <= jf2; j++) {
            int jremap = j - jp - 1, jremapp = jremap + 1;
            if (jremap <= 0) jremap = jremap + ny;
            if (jremapp <= 0) jremapp = jremapp + ny;
            double eps = one - epsi / s->dy;
            A5(s->flux, iin, j, k, 1, 1) = A5(s->flux, iin, j, k, 1, 1) + (one - eps) * IO(outer, jremap, k) + eps * IO(outer, jremapp, k);
            A5(s->flux, iin, j, k, 1, 1) = half * A5(s->flux, iin, j, k, 1, 1);
            jremap = j + jp; jremapp = jremap + 1;
            if (jremap > ny) jremap = jremap - ny;
            if (jremapp > ny) jremapp = jremapp - ny;
            eps = epsi / s->dy;
            A5(s->flux, iout, j, k, 1, 1) = A5(s->flux, iout, j, k, 1, 1) + (one - eps) * IO(inner, jremap, k) + eps * IO(inner, jremapp, k);
            A5(s->flux, iout, j, k, 1, 1) = half * A5(s->flux, iout, j, k, 1, 1);
        }
#undef IO
    free(inner); free(outer);
    shearing_emf(s, itime);
}

/* constrained_transport, scheme.f90:1940-1993 (Cartesian) */
static void constrained_transport(or_state *s)
{
    int ihi = MX(1, s->if2 - 1), jhi = MX(1, s->jf2 - 1), khi = MX(1, s->kf2 - 1);
    const double dx = s->dx, dy = s->dy, dz = s->dz;
    if (s->ndim >= 2) {
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= khi; k++)
            for (int j = 1; j <= jhi + 1; j++)
                for (int i = 1; i <= ihi + 1; i++) {
                    A4(s->uin, i, j, k, iA) = A4(s->uin, i, j, k, iA) + (A3(s->emfz, i, j + 1, k) - A3(s->emfz, i, j, k)) / dy;
                    A4(s->uin, i, j, k, iB) = A4(s->uin, i, j, k, iB) - (A3(s->emfz, i + 1, j, k) - A3(s->emfz, i, j, k)) / dx;
                }
    }
    if (s->ndim == 3) {
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= khi + 1; k++)
            for (int j = 1; j <= jhi + 1; j++)
                for (int i = 1; i <= ihi + 1; i++) {
                    A4(s->uin, i, j, k, iA) = A4(s->uin, i, j, k, iA) - (A3(s->emfy, i, j, k + 1) - A3(s->emfy, i, j, k)) / dz;
                    A4(s->uin, i, j, k, iB) = A4(s->uin, i, j, k, iB) + (A3(s->emfx, i, j, k + 1) - A3(s->emfx, i, j, k)) / dz;
                    A4(s->uin, i, j, k, iC) = A4(s->uin, i, j, k, iC) + (A3(s->emfy, i + 1, j, k) - A3(s->emfy, i, j, k)) / dx
                                            - (A3(s->emfx, i, j + 1, k) - A3(s->emfx, i, j, k)) / dy;
                }
    }
}

/* right-face B copy, scheme.f90:1927-1932 and boundary.f90:82-88 */
static void right_faces(or_state *s)
{
#pragma omp parallel for schedule(static)
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = s->iu1; i <= s->iu2 - 1; i++) A4(s->uin, i, j, k, iA + 3) = A4(s->uin, i + 1, j, k, iA);
#pragma omp parallel for schedule(static)
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2 - 1; j++)
            for (int i = s->iu1; i <= s->iu2; i++) A4(s->uin, i, j, k, iB + 3) = A4(s->uin, i, j + 1, k, iB);
#pragma omp parallel for schedule(static)
    for (int k = s->ku1; k <= s->ku2 - 1; k++)
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = s->iu1; i <= s->iu2; i++) A4(s->uin, i, j, k, iC + 3) = A4(s->uin, i, j, k + 1, iC);
}

/* update, scheme.f90:1764-1936 (Cartesian) */
static void update(or_state *s, double dt)
{
    const dg_params *p = &s->p;
    const double Omega0 = p->omega0;
    const int ndim = s->ndim;
    double lambda = 0.0, ratio = 0.0;
    if (Omega0 > zero) {
        lambda = Omega0 * dt; lambda = 2.5e-1 * lambda * lambda;
        ratio = (one - lambda) / (one + lambda);
    }
    int ihi = MX(1, s->if2 - 1), jhi = MX(1, s->jf2 - 1), khi = MX(1, s->kf2 - 1);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= khi; k++)
        for (int j = 1; j <= jhi; j++)
            for (int i = 1; i <= ihi; i++) {
                double dvloc = one / A3(s->dv, i, j, k);
                if (Omega0 > zero) {
                    double dsx = two * Omega0 * dt * A4(s->uin, i, j, k, iv) / (one + lambda);
                    double dsy = -(half * Omega0 * dt * A4(s->uin, i, j, k, iu)) / (one + lambda);
                    A4(s->uin, i, j, k, iu) = A4(s->uin, i, j, k, iu) * ratio + dsx;
                    A4(s->uin, i, j, k, iv) = A4(s->uin, i, j, k, iv) * ratio + dsy;
                }
                for (int idim = 1; idim <= ndim; idim++) {
                    int i0 = (idim == 1), j0 = (idim == 2), k0 = (idim == 3);
                    /* radius(...) = one in Cartesian geometry */
                    A4(s->uin, i, j, k, ir) = A4(s->uin, i, j, k, ir) + (A5(s->flux, i, j, k, ir, idim) - A5(s->flux, i + i0, j + j0, k + k0, ir, idim)) * dvloc;
                    A4(s->uin, i, j, k, iw) = A4(s->uin, i, j, k, iw)
                        + (A5(s->flux, i, j, k, iw, idim) * one - A5(s->flux, i + i0, j + j0, k + k0, iw, idim) * one) * dvloc / one;
                    A4(s->uin, i, j, k, ip) = A4(s->uin, i, j, k, ip) + (A5(s->flux, i, j, k, ip, idim) - A5(s->flux, i + i0, j + j0, k + k0, ip, idim)) * dvloc;
                    if (ndim == 1) {
                        for (int b = iA; b <= iC; b++)
                            A4(s->uin, i, j, k, b) = A4(s->uin, i, j, k, b) + (A5(s->flux, i, j, k, b, idim) - A5(s->flux, i + i0, j + j0, k + k0, b, idim)) * dvloc;
                    } else if (ndim == 2)
                        A4(s->uin, i, j, k, iC) = A4(s->uin, i, j, k, iC) + (A5(s->flux, i, j, k, iC, idim) - A5(s->flux, i + i0, j + j0, k + k0, iC, idim)) * dvloc;
                    if (Omega0 > zero) {
                        double dfn2 = (A5(s->flux, i, j, k, iu, idim) - A5(s->flux, i + i0, j + j0, k + k0, iu, idim)) * dvloc;
                        if (idim == 1) dfn2 = dfn2 + A4(s->fgodunov_pre, i, j, k, 1) * dvloc;
                        double dfn3 = (A5(s->flux, i, j, k, iv, idim) - A5(s->flux, i + i0, j + j0, k + k0, iv, idim)) * dvloc;
                        if (idim == 2) dfn3 = dfn3 + A4(s->fgodunov_pre, i, j, k, 2) * dvloc;
                        A4(s->uin, i, j, k, iu) = A4(s->uin, i, j, k, iu) + dfn2 / (one + lambda) + Omega0 * dt / (one + lambda) * dfn3;
                        A4(s->uin, i, j, k, iv) = A4(s->uin, i, j, k, iv) + dfn3 / (one + lambda) - 2.5e-1 * Omega0 * dt / (one + lambda) * dfn2;
                    } else {
                        A4(s->uin, i, j, k, iu) = A4(s->uin, i, j, k, iu)
                            + (A5(s->flux, i, j, k, iu, idim) * one - A5(s->flux, i + i0, j + j0, k + k0, iu, idim) * one) * dvloc / one;
                        A4(s->uin, i, j, k, iv) = A4(s->uin, i, j, k, iv)
                            + (A5(s->flux, i, j, k, iv, idim) * one - A5(s->flux, i + i0, j + j0, k + k0, iv, idim) * one) * dvloc / one;
                    }
                }
                if (Omega0 == 0) {
                    A4(s->uin, i, j, k, iu) = A4(s->uin, i, j, k, iu) + A4(s->fgodunov_pre, i, j, k, 1) * dvloc;
                    if (ndim > 1)
                        A4(s->uin, i, j, k, iv) = A4(s->uin, i, j, k, iv) + A4(s->fgodunov_pre, i, j, k, 2) * dvloc;
                }
                if (ndim > 2)
                    A4(s->uin, i, j, k, iw) = A4(s->uin, i, j, k, iw) + A4(s->fgodunov_pre, i, j, k, 3) * dvloc;
            }
    if (s->ndim_act > 1) constrained_transport(s);
    right_faces(s);
}

/* godunov, scheme.f90:104-189 */
void or_godunov(or_state *s, double dt, double time)
{
    fc_magnetic(s);
    or_primitive(s, dt);
    slope(s);
    if (s->ndim == 3) trace3d(s, dt);
    else if (s->ndim == 2) trace2d(s, dt);
    else trace1d(s, dt);
    riemann_solver(s, dt);
    if (s->ndim > 1) riemann_solver_magnetic(s, &s->qRT, &s->qRB, &s->qLT, &s->qLB, &s->emfz, 3, dt);
    if (s->ndim == 3) {
        riemann_solver_magnetic(s, &s->qRT, &s->qLT, &s->qRB, &s->qLB, &s->emfy, 2, dt);
        riemann_solver_magnetic(s, &s->qRT, &s->qRB, &s->qLT, &s->qLB, &s->emfx, 1, dt);
    }
    compflux(s, dt);
    if (s->ndim == 3 && s->p.bc[0] == DG_BC_SHEARINGBOX) shearing_flux(s, time + half * dt);
    update(s, dt);
}

/* ------------------------------------------------------------------------- */
/* boundaries, src/subroutines/boundary.f90 and shearingbox.f90               */
/* ------------------------------------------------------------------------- */
static void copy_cell(or_state *s, int id, int jd, int kd, int is, int js, int ks)
{
    for (int v = 1; v <= nvar + 3; v++) A4(s->uin, id, jd, kd, v) = A4(s->uin, is, js, ks, v);
}

static void bc_x(or_state *s)
{
    int t = s->p.bc[0], nx = s->nx, iu1 = s->iu1, iu2 = s->iu2;
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1; j <= s->ju2; j++) {
            if (t == DG_BC_PERIODIC) {
                copy_cell(s, iu1, j, k, nx - 2, j, k); copy_cell(s, iu1 + 1, j, k, nx - 1, j, k); copy_cell(s, iu1 + 2, j, k, nx, j, k);
                copy_cell(s, iu2 - 2, j, k, 1, j, k); copy_cell(s, iu2 - 1, j, k, 2, j, k); copy_cell(s, iu2, j, k, 3, j, k);
            } else if (t == DG_BC_ZERO_GRADIENT) {
                for (int g = 0; g < 3; g++) { copy_cell(s, iu1 + g, j, k, 1, j, k); copy_cell(s, iu2 - 2 + g, j, k, nx, j, k); }
            }
        }
}

static void bc_y(or_state *s)
{
    int t = s->p.bc[1], ny = s->ny, ju1 = s->ju1, ju2 = s->ju2;
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int i = s->iu1; i <= s->iu2; i++) {
            if (t == DG_BC_PERIODIC) {
                copy_cell(s, i, ju1, k, i, ny - 2, k); copy_cell(s, i, ju1 + 1, k, i, ny - 1, k); copy_cell(s, i, ju1 + 2, k, i, ny, k);
                copy_cell(s, i, ju2 - 2, k, i, 1, k); copy_cell(s, i, ju2 - 1, k, i, 2, k); copy_cell(s, i, ju2, k, i, 3, k);
            } else if (t == DG_BC_ZERO_GRADIENT) {
                for (int g = 0; g < 3; g++) { copy_cell(s, i, ju1 + g, k, i, 1, k); copy_cell(s, i, ju2 - 2 + g, k, i, ny, k); }
            }
        }
}

static void bc_z(or_state *s)
{
    int t = s->p.bc[2], nz = s->nz, ku1 = s->ku1, ku2 = s->ku2;
    for (int j = s->ju1; j <= s->ju2; j++)
        for (int i = s->iu1; i <= s->iu2; i++) {
            if (t == DG_BC_PERIODIC) {
                copy_cell(s, i, j, ku1, i, j, nz - 2); copy_cell(s, i, j, ku1 + 1, i, j, nz - 1); copy_cell(s, i, j, ku1 + 2, i, j, nz);
                copy_cell(s, i, j, ku2 - 2, i, j, 1); copy_cell(s, i, j, ku2 - 1, i, j, 2); copy_cell(s, i, j, ku2, i, j, 3);
            } else if (t == DG_BC_ZERO_GRADIENT) {
                for (int g = 0; g < 3; g++) { copy_cell(s, i, j, ku1 + g, i, j, 1); copy_cell(s, i, j, ku2 - 2 + g, i, j, nz); }
            }
        }
}

/* shearing_slope, shearingbox.f90:394-508; quant/dq are (1:3, ju1:ju2, ku1:ku2, 1:11) */
static void shearing_slope(or_state *s, const farr *quant, farr *dq)
{
    int jst = MN(s->p.slope_type, 2);
    if (jst == 0) { memset(dq->d, 0, sizeof(double) * dq->size); return; }
    const double st = (double)jst;
    for (int g = 1; g <= nghost; g++)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int j = s->ju1 + 1; j <= s->ju2 - 1; j++) {
                for (int v = 1; v <= nvar - 2; v++)
                    A4(*dq, g, j, k, v) = limit1(st, A4(*quant, g, j - 1, k, v), A4(*quant, g, j, k, v), A4(*quant, g, j + 1, k, v));
                A4(*dq, g, j, k, nvar) = limit1(st, A4(*quant, g, j - 1, k, nvar), A4(*quant, g, j, k, nvar), A4(*quant, g, j + 1, k, nvar));
                for (int v = nvar + 1; v <= nvar + 3; v += 2)
                    A4(*dq, g, j, k, v) = limit1(st, A4(*quant, g, j - 1, k, v), A4(*quant, g, j, k, v), A4(*quant, g, j + 1, k, v));
                A4(*dq, g, j, k, nvar - 1) = A4(*quant, g, j + 1, k, nvar - 1) - A4(*quant, g, j, k, nvar - 1);
                A4(*dq, g, j, k, nvar + 2) = A4(*quant, g, j + 1, k, nvar + 2) - A4(*quant, g, j, k, nvar + 2);
            }
}

/* shearing_boundary, shearingbox.f90:19-203 (single rank) */
static void shearing_boundary(or_state *s, double itime)
{
    double epsi; int jp;
    shear_offset(s, itime, &epsi, &jp);
    const int ny = s->ny, iu1 = s->iu1, iu2 = s->iu2;
    farr inner = fa_alloc(1, nghost, s->ju1, s->ju2, s->ku1, s->ku2, nvar + 3, 1);
    farr outer = fa_alloc(1, nghost, s->ju1, s->ju2, s->ku1, s->ku2, nvar + 3, 1);
    farr inner_dq = fa_alloc(1, nghost, s->ju1, s->ju2, s->ku1, s->ku2, nvar + 3, 1);
    farr outer_dq = fa_alloc(1, nghost, s->ju1, s->ju2, s->ku1, s->ku2, nvar + 3, 1);
    for (int v = 1; v <= nvar + 3; v++)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int j = s->ju1; j <= s->ju2; j++)
                for (int g = 1; g <= nghost; g++) {
                    A4(inner, g, j, k, v) = A4(s->uin, iu1 + nghost + g - 1, j, k, v);
                    A4(outer, g, j, k, v) = A4(s->uin, iu2 - 2 * nghost + g, j, k, v);
                }
    shearing_slope(s, &inner, &inner_dq);
    shearing_slope(s, &outer, &outer_dq);
    for (int k = s->ku1; k <= s->ku2; k++)
        for (int j = s->ju1 + 1; j <= s->ju2 - 1; j++) {
            /* inner x boundary */
            int jremap = j - jp - 1, jremapp = jremap + 1;
            if (jremap <= 0) jremap = jremap + ny;
            if (jremapp <= 0) jremapp = jremapp + ny;
            double eps = one - epsi / s->dy;
            double lambda = half * eps * (eps - one);
            for (int g = 1; g <= nghost; g++) {
                for (int v = 1; v <= nvar - 2; v++)
                    A4(s->uin, iu1 + g - 1, j, k, v) = (one - eps) * A4(outer, g, jremap, k, v) + eps * A4(outer, g, jremapp, k, v)
                        + lambda * (A4(outer_dq, g, jremap, k, v) - A4(outer_dq, g, jremapp, k, v));
                A4(s->uin, iu1 + g - 1, j, k, nvar - 1) = A4(outer, g, jremap, k, nvar - 1) + eps * A4(outer_dq, g, jremap, k, nvar - 1);
                A4(s->uin, iu1 + g - 1, j, k, nvar) = (one - eps) * A4(outer, g, jremap, k, nvar) + eps * A4(outer, g, jremapp, k, nvar)
                    + lambda * (A4(outer_dq, g, jremap, k, nvar) - A4(outer_dq, g, jremapp, k, nvar));
            }
            /* outer x boundary */
            jremap = j + jp; jremapp = jremap + 1;
            if (jremap > ny) jremap = jremap - ny;
            if (jremapp > ny) jremapp = jremapp - ny;
            eps = epsi / s->dy;
            lambda = half * eps * (eps - one);
            for (int g = 1; g <= nghost; g++) {
                for (int v = 1; v <= nvar - 3; v++)
                    A4(s->uin, iu2 - 3 + g, j, k, v) = (one - eps) * A4(inner, g, jremap, k, v) + eps * A4(inner, g, jremapp, k, v)
                        + lambda * (A4(inner_dq, g, jremapp, k, v) - A4(inner_dq, g, jremap, k, v));
            }
            for (int g = 2; g <= nghost; g++)
                A4(s->uin, iu2 - 3 + g, j, k, iA) = (one - eps) * A4(inner, g, jremap, k, iA) + eps * A4(inner, g, jremapp, k, iA)
                    + lambda * (A4(inner_dq, g, jremapp, k, iA) - A4(inner_dq, g, jremap, k, iA));
            for (int g = 1; g <= nghost; g++) {
                A4(s->uin, iu2 - 3 + g, j, k, iB) = A4(inner, g, jremap, k, iB) + eps * A4(inner_dq, g, jremap, k, iB);
                A4(s->uin, iu2 - 3 + g, j, k, iC) = (one - eps) * A4(inner, g, jremap, k, iC) + eps * A4(inner, g, jremapp, k, iC)
                    + lambda * (A4(inner_dq, g, jremapp, k, iC) - A4(inner_dq, g, jremap, k, iC));
            }
            A4(s->uin, iu2, j, k, iA + 3) = (one - eps) * A4(inner, nghost, jremap, k, iA + 3) + eps * A4(inner, nghost, jremapp, k, iA + 3)
                + lambda * (A4(inner_dq, nghost, jremapp, k, iA + 3) - A4(inner_dq, nghost, jremap, k, iA + 3));
        }
    /* right-face B of the ghost slabs, shearingbox.f90:150-196 */
    for (int i = iu1 + 2; i >= iu1; i--)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int j = s->ju1; j <= s->ju2; j++) A4(s->uin, i, j, k, iA + 3) = A4(s->uin, i + 1, j, k, iA);
    for (int j = s->ju1; j <= s->ju2 - 1; j++)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int i = iu1; i <= iu1 + 2; i++) A4(s->uin, i, j, k, iB + 3) = A4(s->uin, i, j + 1, k, iB);
    for (int k = s->ku1; k <= s->ku2 - 1; k++)
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = iu1; i <= iu1 + 2; i++) A4(s->uin, i, j, k, iC + 3) = A4(s->uin, i, j, k + 1, iC);
    for (int i = iu2 - 2; i <= iu2 - 1; i++)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int j = s->ju1; j <= s->ju2; j++) A4(s->uin, i, j, k, iA + 3) = A4(s->uin, i + 1, j, k, iA);
    for (int j = s->ju1; j <= s->ju2 - 1; j++)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int i = iu2 - 2; i <= iu2; i++) A4(s->uin, i, j, k, iB + 3) = A4(s->uin, i, j + 1, k, iB);
    for (int k = s->ku1; k <= s->ku2 - 1; k++)
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = iu2 - 2; i <= iu2; i++) A4(s->uin, i, j, k, iC + 3) = A4(s->uin, i, j, k + 1, iC);
    free(inner.d); free(outer.d); free(inner_dq.d); free(outer_dq.d);
}

/* boundary, boundary.f90:18-92 (single rank) */
void or_boundary(or_state *s, double time, double dt)
{
    bc_x(s);
    if (s->ndim == 3 && s->p.bc[0] == DG_BC_SHEARINGBOX) {
        bc_y(s);
        shearing_boundary(s, time + dt);
    }
    if (s->ndim == 3) bc_z(s);
    if (s->ndim > 1) bc_y(s);
    right_faces(s);
}

/* ------------------------------------------------------------------------- */
/* FARGO, src/subroutines/fargo.f90                                          */
/* ------------------------------------------------------------------------- */
/* uin_slope, fargo.f90:244-288 */
static void uin_slope(or_state *s)
{
    int stl = MN(s->p.slope_type, 2);
    if (stl == 0) { memset(s->duin.d, 0, sizeof(double) * s->duin.size); return; }
    const double st = (double)stl;
    for (int v = 1; v <= nvar; v++) {
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= s->nz + 1; k++)
            for (int j = 1; j <= s->ny + 1; j++)
                for (int i = 1; i <= s->nx + 1; i++)
                    A4(s->duin, i, j, k, v) = limit1(st, A4(s->uin, i, j - 1, k, v), A4(s->uin, i, j, k, v), A4(s->uin, i, j + 1, k, v));
    }
}

/* fargo_update, fargo.f90:17-124 with get_emfx (:128-182) and get_emfz (:186-240) */
void or_fargo_update(or_state *s, double dt)
{
    const dg_params *p = &s->p;
    const double Omega0 = p->omega0, dx = s->dx, dy = s->dy, dz = s->dz;
    const int nx = s->nx, ny = s->ny;
    memset(s->emfx.d, 0, sizeof(double) * s->emfx.size);
    memset(s->emfz.d, 0, sizeof(double) * s->emfz.size);
    int ihi = MX(1, s->if2 - 1), jhi = MX(1, s->jf2 - 1), khi = MX(1, s->kf2 - 1);
    if (s->ndim > 1) bc_y(s);
    if (s->ndim == 3) bc_z(s);
    uin_slope(s);
    memcpy(s->uin_old.d, s->uin.d, sizeof(double) * s->uin.size);
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; i++) {
        double vK = -1.5 * Omega0 * XC(i);
        int nshft = (int)(fabs(vK * dt) / dy);
        double eps = fmod(fabs(vK * dt), dy);
        eps = eps / dy;
        for (int j = 1; j <= ny; j++) {
            int jshft, jshftp;
            if (vK > zero) {
                jshft = j - nshft - 1;
                if (jshft < 1) jshft = jshft + ny;
                jshftp = jshft + 1;
                if (jshftp > ny) jshftp = jshftp - ny;
            } else {
                jshft = j + nshft;
                if (jshft > ny) jshft = jshft - ny;
                jshftp = jshft + 1;
                if (jshftp > ny) jshftp = jshftp - ny;
            }
            for (int k = s->ku1; k <= s->ku2; k++)
                for (int v = ir; v <= ip; v++) {
                    double val;
                    if (vK > zero) val = A4(s->uin_old, i, jshft, k, v) * eps + A4(s->uin_old, i, jshftp, k, v) * (one - eps);
                    else val = A4(s->uin_old, i, jshft, k, v) * (one - eps) + A4(s->uin_old, i, jshftp, k, v) * eps;
                    double hme = half - eps;
                    val = val + half * A4(s->duin, i, jshft, k, v) * (forth - hme * hme)
                              + half * A4(s->duin, i, jshftp, k, v) * (hme * hme - forth);
                    A4(s->uin, i, j, k, v) = val;
                }
        }
    }
    /* get_emfx */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx; i++) {
        double vK = -1.5 * Omega0 * XC(i);
        int nshft = (int)(fabs(vK * dt) / dy);
        double eps = fmod(fabs(vK * dt), dy);
        eps = eps / dy;
        for (int j = 1; j <= ny + 1; j++) {
            if (vK > zero) {
                double lambda = half * eps * (one - eps);
                for (int jj = 1; jj <= nshft; jj++) {
                    int jshft = j - jj;
                    if (jshft < 1) jshft = jshft + ny;
                    for (int k = s->ku1; k <= s->ku2; k++) A3(s->emfx, i, j, k) = A3(s->emfx, i, j, k) + A4(s->uin, i, jshft, k, iC) * dy;
                }
                int jshft = j - nshft - 1;
                if (jshft < 1) jshft = jshft + ny;
                for (int k = s->ku1; k <= s->ku2; k++) {
                    double demf = eps * A4(s->uin, i, jshft, k, iC) + lambda * A4(s->duin, i, jshft, k, iC);
                    A3(s->emfx, i, j, k) = A3(s->emfx, i, j, k) + demf * dy;
                }
            } else {
                double lambda = half * eps * (eps - one);
                for (int jj = 0; jj <= nshft - 1; jj++) {
                    int jshft = j + jj;
                    if (jshft > ny) jshft = jshft - ny;
                    for (int k = s->ku1; k <= s->ku2; k++) A3(s->emfx, i, j, k) = A3(s->emfx, i, j, k) - A4(s->uin, i, jshft, k, iC) * dy;
                }
                int jshft = j + nshft;
                if (jshft > ny) jshft = jshft - ny;
                for (int k = s->ku1; k <= s->ku2; k++) {
                    double demf = -eps * A4(s->uin, i, jshft, k, iC) - lambda * A4(s->duin, i, jshft, k, iC);
                    A3(s->emfx, i, j, k) = A3(s->emfx, i, j, k) + demf * dy;
                }
            }
        }
    }
    /* get_emfz */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= nx + 1; i++) {
        double vK = -1.5 * Omega0 * half * (XC(i) + XC(i - 1));
        int nshft = (int)(fabs(vK * dt) / dy);
        double eps = fmod(fabs(vK * dt), dy);
        eps = eps / dy;
        for (int j = 1; j <= ny + 1; j++) {
            if (vK > zero) {
                double lambda = half * eps * (one - eps);
                for (int jj = 1; jj <= nshft; jj++) {
                    int jshft = j - jj;
                    if (jshft < 1) jshft = jshft + ny;
                    for (int k = s->ku1; k <= s->ku2; k++) A3(s->emfz, i, j, k) = A3(s->emfz, i, j, k) - A4(s->uin, i, jshft, k, iA) * dy;
                }
                int jshft = j - nshft - 1;
                if (jshft < 1) jshft = jshft + ny;
                for (int k = s->ku1; k <= s->ku2; k++) {
                    double demf = eps * A4(s->uin, i, jshft, k, iA) + lambda * A4(s->duin, i, jshft, k, iA);
                    A3(s->emfz, i, j, k) = A3(s->emfz, i, j, k) - demf * dy;
                }
            } else {
                double lambda = half * eps * (eps - one);
                for (int jj = 0; jj <= nshft - 1; jj++) {
                    int jshft = j + jj;
                    if (jshft > ny) jshft = jshft - ny;
                    for (int k = s->ku1; k <= s->ku2; k++) A3(s->emfz, i, j, k) = A3(s->emfz, i, j, k) + A4(s->uin, i, jshft, k, iA) * dy;
                }
                int jshft = j + nshft;
                if (jshft > ny) jshft = jshft - ny;
                for (int k = s->ku1; k <= s->ku2; k++) {
                    double demf = -eps * A4(s->uin, i, jshft, k, iA) - lambda * A4(s->duin, i, jshft, k, iA);
                    A3(s->emfz, i, j, k) = A3(s->emfz, i, j, k) - demf * dy;
                }
            }
        }
    }
    /* constrained transport, fargo.f90:100-119 */
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= khi + 1; k++)
        for (int j = 1; j <= jhi + 1; j++)
            for (int i = 1; i <= ihi + 1; i++) {
                A4(s->uin, i, j, k, iA) = A4(s->uin, i, j, k, iA) + (A3(s->emfz, i, j + 1, k) - A3(s->emfz, i, j, k)) / dy;
                A4(s->uin, i, j, k, iB) = A4(s->uin, i, j, k, iB) - (A3(s->emfz, i + 1, j, k) - A3(s->emfz, i, j, k)) / dx
                                        + (A3(s->emfx, i, j, k + 1) - A3(s->emfx, i, j, k)) / dz;
                A4(s->uin, i, j, k, iC) = A4(s->uin, i, j, k, iC) - (A3(s->emfx, i, j + 1, k) - A3(s->emfx, i, j, k)) / dy;
                A4(s->uin, i, j, k, iA + 3) = A4(s->uin, i, j, k, iA) + (A3(s->emfz, i + 1, j + 1, k) - A3(s->emfz, i, j, k)) / dy;
                A4(s->uin, i, j, k, iB + 3) = A4(s->uin, i, j, k, iB) - (A3(s->emfz, i + 1, j + 1, k) - A3(s->emfz, i, j, k)) / dx
                                            + (A3(s->emfx, i, j + 1, k + 1) - A3(s->emfx, i, j, k)) / dz;
                A4(s->uin, i, j, k, iC + 3) = A4(s->uin, i, j, k, iC) - (A3(s->emfx, i, j + 1, k + 1) - A3(s->emfx, i, j, k)) / dy;
            }
}

/* ------------------------------------------------------------------------- */
/* MRI history, src/problem/mri/history.f90:60-125                            */
/* ------------------------------------------------------------------------- */
/* The history sums of the MRI problem (src/problem/mri/history.f90:19-174) and of the default
 * routine of the other problems (src/subroutines/history.f90:57-125, NDIM = 3): the same loop,
 * with the Maxwell stress of B_x and face component ib2 and the Reynolds stress of v_x and
 * velocity iv2 about their y-z means (MRI: B_y and v_y; default: B_z and v_z). */
static void history_sums(or_state *s, int iv2, int ib2, double out[9])
{
    const dg_params *p = &s->p;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    double dtau = s->dx * s->dy * s->dz / (p->xmax - p->xmin) / (p->ymax - p->ymin) / (p->zmax - p->zmin);
    /* compute_yz_mean of v_x and the second velocity (history.f90:247-288, single rank) */
    int ni = s->iu2 - s->iu1 + 1;
    double *mvx = (double *)calloc((size_t)ni, sizeof(double)), *mvy = (double *)calloc((size_t)ni, sizeof(double));
    for (int i = s->iu1; i <= s->iu2; i++) {
        double a = zero, b = zero;
        for (int k = 1; k <= nz; k++)
            for (int j = 1; j <= ny; j++) {
                a = a + A4(s->uin, i, j, k, iu) / A4(s->uin, i, j, k, ir);
                b = b + A4(s->uin, i, j, k, iv2) / A4(s->uin, i, j, k, ir);
            }
        mvx[i - s->iu1] = a / ny / nz;
        mvy[i - s->iu1] = b / ny / nz;
    }
    double mass = zero, magp = zero, maxwell = zero, reynolds = zero, divB = zero;
    double mB[3] = {zero, zero, zero};
    for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) {
                double bxc = A4(s->uin, i, j, k, iA) + A4(s->uin, i + 1, j, k, iA);
                double byc = A4(s->uin, i, j, k, iB) + A4(s->uin, i, j + 1, k, iB);
                double bzc = A4(s->uin, i, j, k, iC) + A4(s->uin, i, j, k + 1, iC);
                mass = mass + A4(s->uin, i, j, k, ir);
                magp = magp + forth * (bxc * bxc) + forth * (byc * byc) + forth * (bzc * bzc);
                maxwell = maxwell - forth * bxc * (ib2 == iB ? byc : bzc);
                mB[0] = mB[0] + A4(s->uin, i, j, k, iA);
                mB[1] = mB[1] + A4(s->uin, i, j, k, iB);
                mB[2] = mB[2] + A4(s->uin, i, j, k, iC);
                reynolds = reynolds + A4(s->uin, i, j, k, ir) * dtau
                         * (A4(s->uin, i, j, k, iu) / A4(s->uin, i, j, k, ir) - mvx[i - s->iu1])
                         * (A4(s->uin, i, j, k, iv2) / A4(s->uin, i, j, k, ir) - mvy[i - s->iu1]);
                divB = divB + (A4(s->uin, i + 1, j, k, iA) - A4(s->uin, i, j, k, iA)) / s->dx
                            + (A4(s->uin, i, j + 1, k, iB) - A4(s->uin, i, j, k, iB)) / s->dy
                            + (A4(s->uin, i, j, k + 1, iC) - A4(s->uin, i, j, k, iC)) / s->dz;
            }
    free(mvx); free(mvy);
    magp = half * magp * dtau;
    mass = mass * dtau;
    maxwell = maxwell * dtau;
    out[0] = mass; out[1] = maxwell; out[2] = reynolds; out[3] = maxwell + reynolds; out[4] = magp;
    out[5] = mB[0] * dtau; out[6] = mB[1] * dtau; out[7] = mB[2] * dtau; out[8] = divB;
}

void or_history_mri(or_state *s, double out[9]) { history_sums(s, iv, iB, out); }
void or_history_default(or_state *s, double out[9]) { history_sums(s, iw, iC, out); }

/* the one-dimensional history line (src/subroutines/history.f90:37-59): rho, rho u_x and E of
 * the first cell whose centre is at x >= 1/2 (the loop's exit value nx+1, a ghost cell, if none) */
void or_history_1d(or_state *s, double out[3])
{
    int ipos = 1;
    for (ipos = 1; ipos <= s->nx; ipos++)
        if (XC(ipos) >= half) break;
    out[0] = A4(s->uin, ipos, 1, 1, ir);
    out[1] = A4(s->uin, ipos, 1, 1, iu);
    out[2] = A4(s->uin, ipos, 1, 1, ip);
}

/* ------------------------------------------------------------------------- */
/* dissipation, src/subroutines/physics.f90:272-664                           */
/* ------------------------------------------------------------------------- */
static const double two3rd = 0.66666666666666667; /* commons.f90:45 */

/* resistivity, physics.f90:295-455: edge EMFs -eta J dt, then constrained_transport.
 * The ISO = 0 loop of :350-451 adds a resistive energy flux to flux(:,:,:,ip,:); that
 * array is zeroed by dissipation before viscosity (:284-285) and overwritten by the next
 * godunov's compflux, so the flux never reaches uin and is not restated here. */
static void resistivity(or_state *s, double dt)
{
    const double eta = s->p.eta, dx = s->dx, dy = s->dy, dz = s->dz;
    memset(s->emfx.d, 0, sizeof(double) * s->emfx.size);
    memset(s->emfy.d, 0, sizeof(double) * s->emfy.size);
    memset(s->emfz.d, 0, sizeof(double) * s->emfz.size);
#pragma omp parallel for schedule(static)
    for (int k = s->kf1; k <= s->kf2; k++)
        for (int j = s->jf1; j <= s->jf2; j++)
            for (int i = s->if1; i <= s->if2; i++) {
                double dBxdy = zero, dBxdz = zero, dBydz = zero, dBzdy = zero, jx = zero;
                const double dBydx = (A4(s->uin, i, j, k, iB) - A4(s->uin, i - 1, j, k, iB)) / dx;
                const double dBzdx = (A4(s->uin, i, j, k, iC) - A4(s->uin, i - 1, j, k, iC)) / dx;
                if (s->ndim > 1) {
                    dBxdy = (A4(s->uin, i, j, k, iA) - A4(s->uin, i, j - 1, k, iA)) / dy;
                    dBzdy = (A4(s->uin, i, j, k, iC) - A4(s->uin, i, j - 1, k, iC)) / dy;
                }
                if (s->ndim == 3) {
                    dBxdz = (A4(s->uin, i, j, k, iA) - A4(s->uin, i, j, k - 1, iA)) / dz;
                    dBydz = (A4(s->uin, i, j, k, iB) - A4(s->uin, i, j, k - 1, iB)) / dz;
                }
                if (s->ndim > 1) jx = dBzdy - dBydz;
                const double jy = dBxdz - dBzdx, jz = dBydx - dBxdy;
                if (s->ndim > 1) A3(s->emfx, i, j, k) = -eta * jx * dt;
                A3(s->emfy, i, j, k) = -eta * jy * dt;
                A3(s->emfz, i, j, k) = -eta * jz * dt;
            }
    constrained_transport(s);
}

/* velocity component m (1..3) of cell (i,j,k) over the density of cell (ii,jj,kk) */
#define VEL(m, i, j, k, ii, jj, kk) (A4(s->uin, i, j, k, (m) + 1) / A4(s->uin, ii, jj, kk, ir))

/* viscosity, physics.f90:459-664: viscous fluxes of momentum (and energy when ISO = 0)
 * on the faces, then the conservative update.  The reference runs the update's idim
 * loop as an OpenMP/OpenACC parallel loop although every idim updates the same cells;
 * the restatement takes the serial order idim = 1, 2, 3. */
static void viscosity(or_state *s, double dt)
{
    const double nu = s->p.nu, dx = s->dx, dy = s->dy, dz = s->dz;
    const int iso = s->p.iso, nd = s->ndim;
#pragma omp parallel for schedule(static)
    for (int k = s->kf1; k <= s->kf2; k++)
        for (int j = s->jf1; j <= s->jf2; j++)
            for (int i = s->if1; i <= s->if2; i++) {
                double dudx[4] = {0, 0, 0, 0}, dudy[4] = {0, 0, 0, 0}, dudz[4] = {0, 0, 0, 0};
                double rho, u = zero, v = zero, w = zero, uR, uL, uRR, uRL, uLR, uLL, txx, tyy, tzz, txy, txz, tyz;
                /* first direction, :482-541 */
                rho = half * (A4(s->uin, i, j, k, ir) + A4(s->uin, i - 1, j, k, ir));
                if (!iso) {
                    u = half * (VEL(1, i, j, k, i, j, k) + VEL(1, i - 1, j, k, i - 1, j, k));
                    v = half * (VEL(2, i, j, k, i, j, k) + VEL(2, i - 1, j, k, i - 1, j, k));
                    w = half * (VEL(3, i, j, k, i, j, k) + VEL(3, i - 1, j, k, i - 1, j, k));
                }
                for (int m = 1; m <= 3; m++) {
                    uR = VEL(m, i, j, k, i, j, k);
                    uL = VEL(m, i - 1, j, k, i, j, k); /* :495, over the density of cell i */
                    dudx[m] = (uR - uL) / dx;
                }
                if (nd > 1) {
                    for (int m = 1; m <= 2; m++) {
                        uRR = VEL(m, i, j + 1, k, i, j + 1, k);
                        uRL = VEL(m, i - 1, j + 1, k, i - 1, j + 1, k);
                        uLR = VEL(m, i, j - 1, k, i, j - 1, k);
                        uLL = VEL(m, i - 1, j - 1, k, i - 1, j - 1, k);
                        uR = uRR + uRL; uL = uLR + uLL;
                        dudy[m] = forth * (uR - uL) / dy;
                    }
                } else {
                    dudy[1] = dudy[2] = dudy[3] = zero;
                }
                if (nd == 3) {
                    for (int m = 1; m <= 3; m += 2) {
                        uRR = VEL(m, i, j, k + 1, i, j, k + 1);
                        uRL = VEL(m, i - 1, j, k + 1, i - 1, j, k + 1);
                        uLR = VEL(m, i, j, k - 1, i, j, k - 1);
                        uLL = VEL(m, i - 1, j, k - 1, i - 1, j, k - 1);
                        uR = uRR + uRL; uL = uLR + uLL;
                        dudz[m] = forth * (uR - uL) / dz;
                    }
                } else {
                    dudz[1] = dudz[2] = dudz[3] = zero;
                }
                txx = -two3rd * nu * rho * (two * dudx[1] - dudy[2] - dudz[3]);
                txy = -nu * rho * (dudy[1] + dudx[2]);
                txz = -nu * rho * (dudz[1] + dudx[3]);
                A5(s->flux, i, j, k, iu, 1) = txx * dt / dx;
                A5(s->flux, i, j, k, iv, 1) = txy * dt / dx;
                A5(s->flux, i, j, k, iw, 1) = txz * dt / dx;
                if (!iso) {
                    A5(s->flux, i, j, k, ip, 1) = u * txx + v * txy + w * txz;
                    A5(s->flux, i, j, k, ip, 1) = A5(s->flux, i, j, k, ip, 1) * dt / dx;
                }
                /* second direction, :544-593 */
                if (nd > 1) {
                    rho = half * (A4(s->uin, i, j, k, ir) + A4(s->uin, i, j - 1, k, ir));
                    if (!iso) {
                        u = half * (VEL(1, i, j, k, i, j, k) + VEL(1, i, j - 1, k, i, j - 1, k));
                        v = half * (VEL(2, i, j, k, i, j, k) + VEL(2, i, j - 1, k, i, j - 1, k));
                        w = half * (VEL(3, i, j, k, i, j, k) + VEL(3, i, j - 1, k, i, j - 1, k));
                    }
                    for (int m = 1; m <= 3; m++) {
                        uR = VEL(m, i, j, k, i, j, k);
                        uL = VEL(m, i, j - 1, k, i, j - 1, k);
                        dudy[m] = (uR - uL) / dy;
                    }
                    for (int m = 1; m <= 2; m++) {
                        uRR = VEL(m, i + 1, j, k, i + 1, j, k);
                        uRL = VEL(m, i + 1, j - 1, k, i + 1, j - 1, k);
                        uLR = VEL(m, i - 1, j, k, i - 1, j, k);
                        uLL = VEL(m, i - 1, j - 1, k, i - 1, j - 1, k);
                        uR = uRR + uRL; uL = uLR + uLL;
                        dudx[m] = forth * (uR - uL) / dx;
                    }
                    if (nd == 3) {
                        for (int m = 2; m <= 3; m++) {
                            uRR = VEL(m, i, j, k + 1, i, j, k + 1);
                            uRL = VEL(m, i, j - 1, k + 1, i, j - 1, k + 1);
                            uLR = VEL(m, i, j, k - 1, i, j, k - 1);
                            uLL = VEL(m, i, j - 1, k - 1, i, j - 1, k - 1);
                            uR = uRR + uRL; uL = uLR + uLL;
                            dudz[m] = forth * (uR - uL) / dz;
                        }
                    } else {
                        dudz[1] = dudz[2] = dudz[3] = zero;
                    }
                    tyy = -two3rd * nu * rho * (two * dudy[2] - dudx[1] - dudz[3]);
                    txy = -nu * rho * (dudy[1] + dudx[2]);
                    tyz = -nu * rho * (dudz[2] + dudy[3]);
                    A5(s->flux, i, j, k, iu, 2) = txy * dt / dy;
                    A5(s->flux, i, j, k, iv, 2) = tyy * dt / dy;
                    A5(s->flux, i, j, k, iw, 2) = tyz * dt / dy;
                    if (!iso) {
                        A5(s->flux, i, j, k, ip, 2) = u * txy + v * tyy + w * tyz;
                        A5(s->flux, i, j, k, ip, 2) = A5(s->flux, i, j, k, ip, 2) * dt / dy;
                    }
                }
                /* third direction, :596-643 */
                if (nd == 3) {
                    rho = half * (A4(s->uin, i, j, k, ir) + A4(s->uin, i, j, k - 1, ir));
                    if (!iso) {
                        u = half * (VEL(1, i, j, k, i, j, k) + VEL(1, i, j, k - 1, i, j, k - 1));
                        v = half * (VEL(2, i, j, k, i, j, k) + VEL(2, i, j, k - 1, i, j, k - 1));
                        w = half * (VEL(3, i, j, k, i, j, k) + VEL(3, i, j, k - 1, i, j, k - 1));
                    }
                    for (int m = 1; m <= 3; m++) {
                        uR = VEL(m, i, j, k, i, j, k);
                        uL = VEL(m, i, j, k - 1, i, j, k - 1);
                        dudz[m] = (uR - uL) / dz;
                    }
                    for (int m = 1; m <= 3; m += 2) {
                        uRR = VEL(m, i + 1, j, k, i + 1, j, k);
                        uRL = VEL(m, i + 1, j, k - 1, i + 1, j, k - 1);
                        uLR = VEL(m, i - 1, j, k, i - 1, j, k);
                        uLL = VEL(m, i - 1, j, k - 1, i - 1, j, k - 1);
                        uR = uRR + uRL; uL = uLR + uLL;
                        dudx[m] = forth * (uR - uL) / dx;
                    }
                    for (int m = 2; m <= 3; m++) {
                        uRR = VEL(m, i, j + 1, k, i, j + 1, k);
                        uRL = VEL(m, i, j + 1, k - 1, i, j + 1, k - 1);
                        uLR = VEL(m, i, j - 1, k, i, j - 1, k);
                        uLL = VEL(m, i, j - 1, k - 1, i, j - 1, k - 1);
                        uR = uRR + uRL; uL = uLR + uLL;
                        dudy[m] = forth * (uR - uL) / dy;
                    }
                    tzz = -two3rd * nu * rho * (two * dudz[3] - dudx[1] - dudy[2]);
                    txz = -nu * rho * (dudz[1] + dudx[3]);
                    tyz = -nu * rho * (dudz[2] + dudy[3]);
                    A5(s->flux, i, j, k, iu, 3) = txz * dt / dz;
                    A5(s->flux, i, j, k, iv, 3) = tyz * dt / dz;
                    A5(s->flux, i, j, k, iw, 3) = tzz * dt / dz;
                    if (!iso) {
                        A5(s->flux, i, j, k, ip, 3) = u * txz + v * tyz + w * tzz;
                        A5(s->flux, i, j, k, ip, 3) = A5(s->flux, i, j, k, ip, 3) * dt / dz;
                    }
                }
            }
    /* conservative update, :647-663 */
    for (int idim = 1; idim <= nd; idim++) {
        const int i0 = idim == 1, j0 = idim == 2, k0 = idim == 3;
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= s->nz; k++)
            for (int j = 1; j <= s->ny; j++)
                for (int i = 1; i <= s->nx; i++)
                    for (int v = iu; v <= ip; v++)
                        A4(s->uin, i, j, k, v) = A4(s->uin, i, j, k, v)
                            + (A5(s->flux, i, j, k, v, idim) - A5(s->flux, i + i0, j + j0, k + k0, v, idim));
    }
}
#undef VEL

/* dissipation, physics.f90:272-291, called after boundary when nu > 0 or eta > 0
 * (dumses.f90:104) */
void or_dissipation(or_state *s, double time, double dt)
{
    if (s->p.eta > zero) resistivity(s, dt);
    if (s->p.nu > zero) {
        memset(s->flux.d, 0, sizeof(double) * s->flux.size);
        viscosity(s, dt);
    }
    or_boundary(s, time, dt);
}

/* ------------------------------------------------------------------------- */
/* driver loop, src/dumses.f90:75-160                                         */
/* ------------------------------------------------------------------------- */
double or_step(or_state *s, double *time)
{
    double dt = or_compute_dt(s);
    or_godunov(s, dt, *time);
    if (s->p.fargo) or_fargo_update(s, dt);
    or_boundary(s, *time, dt);
    if (s->p.nu > zero || s->p.eta > zero) or_dissipation(s, *time, dt);
    *time = *time + dt;
    return dt;
}

int or_run_history(or_state *s, double tlim, double dthist, double *rows, int max_rows)
{
    int n = 0;
    double time = 0.0, dt = 0.0, h[9];
    if (n < max_rows) {
        or_history_mri(s, h);
        rows[0] = time; rows[1] = dt;
        for (int c = 0; c < 9; c++) rows[2 + c] = h[c];
        n++;
    }
    double thist = time;
    for (;;) {
        dt = or_step(s, &time);
        if (((time - dt) <= (thist + dthist)) && (time > (thist + dthist))) {
            if (n < max_rows) {
                or_history_mri(s, h);
                double *r = rows + 11 * n;
                r[0] = time; r[1] = dt;
                for (int c = 0; c < 9; c++) r[2 + c] = h[c];
                n++;
            }
            thist = thist + dthist;
        }
        if ((time - dt) > tlim) break;
    }
    return n;
}

/* ------------------------------------------------------------------------- */
/* initial conditions (the problem plug-ins src/problem/<p>/condinit.f90)     */
/* ------------------------------------------------------------------------- */
/* Counter-based uniform variates in [0,1): splitmix64 of (seed, stream, cell).  The
 * reference seeds random_number from the wall clock (mri/condinit.f90:52-61), which no
 * two runs share; a counter-based generator gives every cell the same kick on any
 * thread count, and the same value as the library's own initial-condition generator. */
static uint64_t or_mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
static double or_uniform01(uint64_t seed, uint64_t stream, uint64_t counter)
{
    const uint64_t h = or_mix64(seed ^ or_mix64(stream * 0x100000001B3ull + counter));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

int or_condinit(or_state *s, int ic, double beta, double amp, unsigned long long seed)
{
    const double twopi = 4.0 * asin(1.0), pi = 2.0 * asin(1.0); /* commons.f90:47 */
    memset(s->uin.d, 0, sizeof(double) * s->uin.size);
    if (ic == DG_IC_MRI || ic == DG_IC_MRI_TEST) {
        /* mri/condinit.f90:30-105: rho = 1, p0 = rho ciso^2, B0 = sqrt(2 p0 / beta) */
        if (s->ndim != 3) return DG_ERR_ARG;
        const double d0 = 1.0, p0 = d0 * s->p.ciso * s->p.ciso, B0 = sqrt(2.0 * p0 / beta);
#pragma omp parallel for collapse(2)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int j = s->ju1; j <= s->ju2; j++)
                for (int i = s->iu1; i <= s->iu2; i++) {
                    /* the kick stream's counter: the cell's offset in the uin array */
                    const uint64_t cell = (uint64_t)(&A4(s->uin, i, j, k, 1) - s->uin.d);
                    A4(s->uin, i, j, k, ir) = d0;
                    if (ic == DG_IC_MRI_TEST) {
                        /* the regression set-up ('Test', amp = 0): one vx mode, B_z = B0 sin(2 pi x) */
                        A4(s->uin, i, j, k, iu) = 1.e-2 * 1.e-3 * cos(twopi * 10.0 * ZC(k)) * cos(twopi * 5.0 * XC(i));
                        A4(s->uin, i, j, k, iC) = B0 * sin(twopi * XC(i));
                        A4(s->uin, i, j, k, 11) = B0 * sin(twopi * XC(i));
                    } else {
                        /* 'fluxZ' with uniform kicks amp (r - 1/2) sqrt(p0) per component */
                        for (int c = 0; c < 3; c++)
                            A4(s->uin, i, j, k, iu + c) =
                                A4(s->uin, i, j, k, ir) * amp * (or_uniform01(seed, (uint64_t)(c + 1), cell) - 0.5) * sqrt(p0);
                        A4(s->uin, i, j, k, iC) = B0;
                        A4(s->uin, i, j, k, 11) = B0;
                    }
                }
        return DG_OK;
    }
    if (ic == DG_IC_ORSZAG_TANG) {
        /* the 3D form of orszag_tang/condinit.f90:33-56: rho = 25/(36 pi), P = 5/(12 pi),
         * v = (-sin 2 pi y, sin 2 pi x, 0.2 sin 2 pi z), B = (-sin 2 pi y, sin 4 pi x, 0)/sqrt(4 pi) */
        if (s->ndim != 3) return DG_ERR_ARG;
        const double rho = 25.0 / (36.0 * pi), pres = 5.0 / (12.0 * pi), b0 = 1.0 / sqrt(4.0 * pi);
        const double gamma = s->p.gamma;
#pragma omp parallel for collapse(2)
        for (int k = s->ku1; k <= s->ku2; k++)
            for (int j = s->ju1; j <= s->ju2; j++)
                for (int i = s->iu1; i <= s->iu2; i++) {
                    const double x = XC(i), y = YC(j), z = ZC(k);
                    const double vx = -sin(twopi * y), vy = sin(twopi * x), vz = 0.2 * sin(twopi * z);
                    const double bx = -b0 * sin(twopi * y), by = b0 * sin(2.0 * twopi * x);
                    A4(s->uin, i, j, k, ir) = rho;
                    A4(s->uin, i, j, k, iu) = rho * vx;
                    A4(s->uin, i, j, k, iv) = rho * vy;
                    A4(s->uin, i, j, k, iw) = rho * vz;
                    A4(s->uin, i, j, k, iA) = bx; A4(s->uin, i, j, k, 9) = bx;
                    A4(s->uin, i, j, k, iB) = by; A4(s->uin, i, j, k, 10) = by;
                    A4(s->uin, i, j, k, ip) = pres / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
                                              + 0.5 * (bx * bx + by * by);
                }
        return DG_OK;
    }
    if (ic == DG_IC_FIELD_LOOP) {
        /* magnetic_loop/condinit.f90:40-104 (direction 'x') with A0 = 1e-3, R = 0.3, v = (2, 1):
         * A_z = A0 (R - r) for r <= R, face B from its differences */
        if (s->ndim != 2) return DG_ERR_ARG;
        const double A0 = 1.e-3, R = 0.3, rho = 1.0, pres = 1.0, vx = 2.0, vy = 1.0, gamma = s->p.gamma;
        const double dx = s->dx, dy = s->dy, xmin = s->p.xmin, ymin = s->p.ymin;
        const int k = 1;
        for (int j = s->ju1; j <= s->ju2; j++)
            for (int i = s->iu1; i <= s->iu2; i++) {
                /* A_z at the cell's lower-left corner, from the centre formula of init_grid */
                double az[2][2];
                for (int a = 0; a < 2; a++)
                    for (int b = 0; b < 2; b++) {
                        const double x = xmin + dx / 2 + (i + a - 1) * dx, y = ymin + dy / 2 + (j + b - 1) * dy;
                        const double dist = sqrt(x * x + y * y);
                        az[a][b] = dist <= R ? A0 * (R - dist) : 0.0;
                    }
                const double bxl = (az[0][1] - az[0][0]) / dy, bxr = (az[1][1] - az[1][0]) / dy;
                const double byl = -(az[1][0] - az[0][0]) / dx, byr = -(az[1][1] - az[0][1]) / dx;
                A4(s->uin, i, j, k, ir) = rho;
                A4(s->uin, i, j, k, iu) = rho * vx;
                A4(s->uin, i, j, k, iv) = rho * vy;
                A4(s->uin, i, j, k, iA) = bxl; A4(s->uin, i, j, k, 9) = bxr;
                A4(s->uin, i, j, k, iB) = byl; A4(s->uin, i, j, k, 10) = byr;
                const double bcx = 0.5 * (bxl + bxr), bcy = 0.5 * (byl + byr);
                A4(s->uin, i, j, k, ip) = pres / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy)
                                          + 0.5 * (bcx * bcx + bcy * bcy);
            }
        return DG_OK;
    }
    return DG_ERR_ARG;
}
