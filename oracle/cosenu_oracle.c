/*
 * cosenu_oracle.c -- CPU restatement of COSEnu's RK4 time-stepping path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the CUDA path is
 * compared against; it is imported only by tests/, by __graft_entry__.smoke()
 * and by bench.py's cpu_baseline leg.  Nothing in the product links it.
 *
 * Every routine below restates one reference routine (paths relative to the
 * COSEnu project root) in plain C, on the reference's own memory layout:
 * one array per component, v-major rows of length nz+2*gz, z contiguous,
 * idx(i,j) = i*(nz+2gz) + j + gz   (src/nuosc.hpp:145-148).
 * Buffers handed in here are contiguous [8][nvz][nz+2gz] blocks; component
 * order is ee, xx, ex_re, ex_im, bee, bxx, bex_re, bex_im
 * (src/structures.hpp:5-13).
 *
 * Parity pin: tests/golden/ holds outputs of the reference binary itself
 * (compiled from its own sources by oracle/build_ref.sh) on seeded inputs;
 * tests/test_oracle_golden.py checks this file against them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NCOMP 8
enum { EE = 0, XX, EXR, EXI, BEE, BXX, BEXR, BEXI };

typedef struct {
    int nz, nvz, gz;
    double z0, z1, v0, v1, cfl;
    double pmo, omega, theta_deg, mu;
    int scheme;      /* 0 = FV (WENO7), 1 = FD */
    int bc;          /* 0 = periodic, 1 = open */
    int vac, mat, coll, advec_off;
    int fd_advec;    /* 0 = central FD4, 1 = upwind, 2 = lopsided */
    int ko_order;    /* 3 or 5 (FD only) */
    int coll_direct; /* 1 = per-v' loop as the reference, 0 = velocity-moment form */
    int nthreads;
} orc_params;

typedef struct {
    int nz, nvz, gz, ld;
    long cs; /* component stride */
    double dz, dv, dt, ct, st;
    double *Z, *vz, *Hm;
} orc_grid;

/* Grid set-up, src/nuosc.hpp:47-96 (dz, dv, dt = CFL*dz, cell-centred Z and vz,
 * Hm) and set_vac_pars src/nuosc.hpp:132-138 (theta given in degrees). */
static void grid_make(const orc_params *p, orc_grid *g)
{
    g->nz = p->nz;
    g->nvz = p->nvz;
    g->gz = p->gz;
    g->ld = p->nz + 2 * p->gz;
    g->cs = (long)g->ld * p->nvz;
    g->dz = (p->z1 - p->z0) / p->nz;
    g->dv = (p->v1 - p->v0) / p->nvz;
    g->dt = p->cfl * g->dz;
    double th = p->theta_deg * M_PI / 180.0;
    g->ct = 0.5 * p->omega * cos(2.0 * th);
    g->st = 0.5 * p->omega * sin(2.0 * th);
    g->Z = (double *)malloc(sizeof(double) * p->nz);
    g->vz = (double *)malloc(sizeof(double) * p->nvz);
    g->Hm = (double *)malloc(sizeof(double) * p->nz);
    for (int j = 0; j < p->nz; j++) {
        g->Z[j] = p->z0 + (j + 0.5) * g->dz;
        g->Hm[j] = -1.0e-3 * (g->Z[j] + 600.0);
    }
    for (int i = 0; i < p->nvz; i++)
        g->vz[i] = p->v0 + (i + 0.5) * g->dv;
}

static void grid_free(orc_grid *g)
{
    free(g->Z);
    free(g->vz);
    free(g->Hm);
}

static inline long at(const orc_grid *g, int i, int j) { return (long)i * g->ld + j + g->gz; }

static inline int sgn_d(double x) { return (0.0 < x) - (x < 0.0); }

void orc_grid_info(const orc_params *p, double *Z, double *vz, double *scal /* dz dv dt ct st */)
{
    orc_grid g;
    grid_make(p, &g);
    if (Z) memcpy(Z, g.Z, sizeof(double) * p->nz);
    if (vz) memcpy(vz, g.vz, sizeof(double) * p->nvz);
    if (scal) {
        scal[0] = g.dz; scal[1] = g.dv; scal[2] = g.dt; scal[3] = g.ct; scal[4] = g.st;
    }
    grid_free(&g);
}

/* Ghost-zone fill, src/nuosc.hpp:212-278.  Periodic: low ghosts copy the last
 * gz interior cells, high ghosts the first gz.  Open: low ghosts hold cell 0,
 * high ghosts are a linear extrapolation that reuses the ghost just written
 * (the serial order of the reference loop). */
static void fill_ghosts(const orc_grid *g, int bc, double *f, int ncomp)
{
    for (int c = 0; c < ncomp; c++) {
        double *a = f + c * g->cs;
        for (int i = 0; i < g->nvz; i++) {
            for (int j = 0; j < g->gz; j++) {
                if (bc == 0) {
                    a[at(g, i, -j - 1)] = a[at(g, i, g->nz - j - 1)];
                    a[at(g, i, g->nz + j)] = a[at(g, i, j)];
                } else {
                    a[at(g, i, -j - 1)] = a[at(g, i, 0)];
                    a[at(g, i, g->nz + j)] =
                        a[at(g, i, g->nz + j - 1)] * 2 - a[at(g, i, g->nz + j - 2)];
                }
            }
        }
    }
}

void orc_fill_ghosts(const orc_params *p, double *f, int ncomp)
{
    orc_grid g;
    grid_make(p, &g);
    fill_ghosts(&g, p->bc, f, ncomp);
    grid_free(&g);
}

/* 7th-order WENO reconstruction of one component, src/rhs_fv.hpp:6-95.
 * For every row and j in [-1, nz], rflux[j] is the left-biased value at face
 * j+1/2 and lflux[j] the right-biased value at face j-1/2, from the four
 * 4-point candidate stencils with linear weights (4,18,12,1)/35 and
 * (1,12,18,4)/35 and the Jiang-Shu style indicators with eps = 1e-6. */
static void weno7(const orc_grid *g, const double *in, double *rflux, double *lflux)
{
    const double eps = 1e-6;
    const double gr[4] = {4. / 35., 18. / 35., 12. / 35., 1. / 35.};
    const double gl[4] = {1. / 35., 12. / 35., 18. / 35., 4. / 35.};
#pragma omp parallel for collapse(2)
    for (int i = 0; i < g->nvz; i++) {
        for (int j = -1; j < g->nz + 1; j++) {
            const double *u = in + at(g, i, j);
            double b[4];
            b[0] = u[0] * (2107 * u[0] - 9402 * u[1] + 7042 * u[2] - 1854 * u[3]) +
                   u[1] * (11003 * u[1] - 17246 * u[2] + 4642 * u[3]) +
                   u[2] * (7043 * u[2] - 3882 * u[3]) + 547 * u[3] * u[3];
            b[1] = u[-1] * (547 * u[-1] - 2522 * u[0] + 1922 * u[1] - 494 * u[2]) +
                   u[0] * (3443 * u[0] - 5966 * u[1] + 1602 * u[2]) +
                   u[1] * (2843 * u[1] - 1642 * u[2]) + 267 * u[2] * u[2];
            b[2] = u[-2] * (267 * u[-2] - 1642 * u[-1] + 1602 * u[0] - 494 * u[1]) +
                   u[-1] * (2843 * u[-1] - 5966 * u[0] + 1922 * u[1]) +
                   u[0] * (3443 * u[0] - 2522 * u[1]) + 547 * u[1] * u[1];
            b[3] = u[-3] * (547 * u[-3] - 3882 * u[-2] + 4642 * u[-1] - 1854 * u[0]) +
                   u[-2] * (7043 * u[-2] - 17246 * u[-1] + 7042 * u[0]) +
                   u[-1] * (11003 * u[-1] - 9402 * u[0]) + 2107 * u[0] * u[0];
            double qr[4], ql[4];
            qr[0] = (1. / 4.) * u[0] + (13. / 12.) * u[1] - (5. / 12.) * u[2] + (1. / 12.) * u[3];
            qr[1] = (-1. / 12.) * u[-1] + (7. / 12.) * u[0] + (7. / 12.) * u[1] - (1. / 12.) * u[2];
            qr[2] = (1. / 12.) * u[-2] - (5. / 12.) * u[-1] + (13. / 12.) * u[0] + (1. / 4.) * u[1];
            qr[3] = (-1. / 4.) * u[-3] + (13. / 12.) * u[-2] - (23. / 12.) * u[-1] + (25. / 12.) * u[0];
            ql[0] = (-1. / 4.) * u[3] + (13. / 12.) * u[2] - (23. / 12.) * u[1] + (25. / 12.) * u[0];
            ql[1] = (1. / 12.) * u[2] - (5. / 12.) * u[1] + (13. / 12.) * u[0] + (1. / 4.) * u[-1];
            ql[2] = (-1. / 12.) * u[1] + (7. / 12.) * u[0] + (7. / 12.) * u[-1] - (1. / 12.) * u[-2];
            ql[3] = (1. / 4.) * u[0] + (13. / 12.) * u[-1] - (5. / 12.) * u[-2] + (1. / 12.) * u[-3];
            double ar[4], al[4], sr = 0, sl = 0;
            for (int r = 0; r < 4; r++) {
                double d = (eps + b[r]) * (eps + b[r]);
                ar[r] = gr[r] / d;
                al[r] = gl[r] / d;
                sr += ar[r];
                sl += al[r];
            }
            double fr = 0, fl = 0;
            for (int r = 0; r < 4; r++) {
                fr += (ar[r] / sr) * qr[r];
                fl += (al[r] / sl) * ql[r];
            }
            rflux[at(g, i, j)] = fr;
            lflux[at(g, i, j)] = fl;
        }
    }
}

void orc_weno7(const orc_params *p, const double *in, double *rflux, double *lflux)
{
    orc_grid g;
    grid_make(p, &g);
    weno7(&g, in, rflux, lflux);
    grid_free(&g);
}

/* Per-z velocity moments of the three combinations the collective term needs
 * (rhs_fv.hpp:188-233 / rhs_fd.hpp:85-126 depend on v' only through these):
 *   A = ex_im + bex_im,  B = ex_re - bex_re,  C = ee - xx - bee + bxx,
 * m[0..2][j] = sum_k {A,B,C}(k,j),  m[3..5][j] = sum_k v_k {A,B,C}(k,j). */
static void velocity_moments(const orc_grid *g, const double *in, double *m)
{
    const double *ee = in + EE * g->cs, *xx = in + XX * g->cs, *exr = in + EXR * g->cs,
                 *exi = in + EXI * g->cs, *bee = in + BEE * g->cs, *bxx = in + BXX * g->cs,
                 *bexr = in + BEXR * g->cs, *bexi = in + BEXI * g->cs;
    for (int j = 0; j < g->nz; j++) {
        double s[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < g->nvz; k++) {
            long q = at(g, k, j);
            double A = exi[q] + bexi[q];
            double B = exr[q] - bexr[q];
            double C = ee[q] - xx[q] - bee[q] + bxx[q];
            s[0] += A; s[1] += B; s[2] += C;
            s[3] += g->vz[k] * A; s[4] += g->vz[k] * B; s[5] += g->vz[k] * C;
        }
        for (int t = 0; t < 6; t++) m[t * g->nz + j] = s[t];
    }
}

/* Collective nu-nu term for cell (i,j), added into o[8].  The direct form
 * keeps the reference's per-v' accumulation and its operand order
 * (rhs_fv.hpp:188-233; rhs_fd.hpp:85-126 is the same arithmetic with
 * vw[k] = 1 and sign-symmetric rewrites that round identically), so it
 * reproduces the reference bit for bit.  The moment form uses
 *   sum_k (1 - v_i v_k) X_k = M0[X] - v_i M1[X]
 * and differs from it only by summation order. */
static void collective(const orc_grid *g, const orc_params *p, const double *in, const double *mom,
                       int i, int j, const double *c, double *o)
{
    double vi = g->vz[i];
    if (p->coll_direct) {
        double Iee = 0, Ixx = 0, Iexr = 0, Iexi = 0, Ibee = 0, Ibxx = 0, Ibexr = 0, Ibexi = 0;
        for (int k = 0; k < g->nvz; k++) {
            long q = at(g, k, j);
            double eep = in[EE * g->cs + q], xxp = in[XX * g->cs + q];
            double expr = in[EXR * g->cs + q], expi = in[EXI * g->cs + q];
            double beep = in[BEE * g->cs + q], bxxp = in[BXX * g->cs + q];
            double bexpr = in[BEXR * g->cs + q], bexpi = in[BEXI * g->cs + q];
            double A = expi + bexpi;
            double B = expr - bexpr;
            double C = eep - xxp - beep + bxxp;
            double w2 = 2.0 * p->mu * (1.0 - vi * g->vz[k]);
            double w1 = 1.0 * p->mu * (1.0 - vi * g->vz[k]);
            double t = c[EXR] * A - c[EXI] * B;
            Iee += w2 * t;
            Ixx += -w2 * t;
            Iexr += w1 * ((c[XX] - c[EE]) * A + c[EXI] * C);
            Iexi += w1 * (-(c[XX] - c[EE]) * B - c[EXR] * C);
            double bt = c[BEXR] * A + c[BEXI] * B;
            Ibee += w2 * bt;
            Ibxx += -w2 * bt;
            Ibexr += w1 * ((c[BXX] - c[BEE]) * A - c[BEXI] * C);
            Ibexi += w1 * ((c[BXX] - c[BEE]) * B + c[BEXR] * C);
        }
        o[EE] += g->dv * Iee;
        o[XX] += g->dv * Ixx;
        o[EXR] += g->dv * Iexr;
        o[EXI] += g->dv * Iexi;
        o[BEE] += g->dv * Ibee;
        o[BXX] += g->dv * Ibxx;
        o[BEXR] += g->dv * Ibexr;
        o[BEXI] += g->dv * Ibexi;
        return;
    }
    double SA = mom[0 * g->nz + j] - vi * mom[3 * g->nz + j];
    double SB = mom[1 * g->nz + j] - vi * mom[4 * g->nz + j];
    double SC = mom[2 * g->nz + j] - vi * mom[5 * g->nz + j];
    double f = p->mu * g->dv;
    double Iee = 2.0 * (c[EXR] * SA - c[EXI] * SB);
    double Ibee = 2.0 * (c[BEXR] * SA + c[BEXI] * SB);
    o[EE] += f * Iee;
    o[XX] += f * (-Iee);
    o[EXR] += f * ((c[XX] - c[EE]) * SA + c[EXI] * SC);
    o[EXI] += f * (-(c[XX] - c[EE]) * SB - c[EXR] * SC);
    o[BEE] += f * Ibee;
    o[BXX] += f * (-Ibee);
    o[BEXR] += f * ((c[BXX] - c[BEE]) * SA - c[BEXI] * SC);
    o[BEXI] += f * ((c[BXX] - c[BEE]) * SB + c[BEXR] * SC);
}

/* Vacuum term -i[H0, rho].  The two schemes write it with different operand
 * order (rhs_fv.hpp:164-174 accumulates, rhs_fd.hpp:33-43 assigns); each is
 * kept so that the rounding matches. */
static void vacuum(const orc_grid *g, const orc_params *p, const double *c, double *o)
{
    double pmo = p->pmo, ct = g->ct, st = g->st;
    if (p->scheme == 0) {
        o[EE] += -2.0 * st * c[EXI] * pmo;
        o[XX] += 2.0 * st * c[EXI] * pmo;
        o[EXR] += -2.0 * ct * c[EXI] * pmo;
        o[EXI] += (2.0 * ct * c[EXR] + st * (c[EE] - c[XX])) * pmo;
        o[BEE] += -2.0 * st * c[BEXI] * pmo;
        o[BXX] += 2.0 * st * c[BEXI] * pmo;
        o[BEXR] += -2.0 * ct * c[BEXI] * pmo;
        o[BEXI] += (2.0 * ct * c[BEXR] + st * (c[BEE] - c[BXX])) * pmo;
    } else {
        o[EE] = -pmo * 2 * st * c[EXI];
        o[XX] = pmo * 2 * st * c[EXI];
        o[EXR] = -pmo * 2 * ct * c[EXI];
        o[EXI] = pmo * (2 * ct * c[EXR] + st * (c[EE] - c[XX]));
        o[BEE] = -pmo * 2 * st * c[BEXI];
        o[BXX] = pmo * 2 * st * c[BEXI];
        o[BEXR] = -pmo * 2 * ct * c[BEXI];
        o[BEXI] = pmo * (2 * ct * c[BEXR] + st * (c[BEE] - c[BXX]));
    }
}

/* Matter term with the built-in Hm(z) profile, rhs_fv.hpp:176-186. */
static void matter(const orc_grid *g, int j, const double *c, double *o)
{
    double h = g->Hm[j];
    o[EXR] += h * c[EXI];
    o[EXI] += -h * c[EXR];
    o[BEXR] += -h * c[BEXI];
    o[BEXI] += h * c[BEXR];
}

/* FD advection and Kreiss-Oliger stencils, rhs_fd.hpp:53-79 and 128-145. */
static double fd_advect(const orc_params *p, const double *x, double vi, double dz)
{
    if (p->fd_advec == 0) {
        double factor = -vi / (12 * dz);
        return factor * ((x[-2] - x[2]) - 8.0 * (x[-1] - x[1]));
    }
    int sv = sgn_d(vi);
    if (p->fd_advec == 1) {
        double factor = -sv * vi / (12 * dz);
        return factor * (-4 * x[-3 * sv] + 18 * x[-2 * sv] - 36 * x[-sv] + 22 * x[0]);
    }
    double factor = sv * vi / (12 * dz);
    return factor * (x[-3 * sv] - 6 * x[-2 * sv] + 18 * x[-sv] - 10 * x[0] - 3 * x[sv]);
}

static double fd_ko(const orc_params *p, const double *x, double dz, double ko)
{
    if (p->ko_order == 5) {
        double e = -ko / dz / 64.0;
        return e * (x[-3] + x[3] - 6 * (x[-2] + x[2]) + 15 * (x[-1] + x[1]) - 20 * x[0]);
    }
    double e = -ko / dz / 16.0;
    return e * (x[-2] + x[2] - 4 * (x[-1] + x[1]) + 6 * x[0]);
}

/* Right-hand side, FV (src/rhs_fv.hpp:115-236) or FD (src/rhs_fd.hpp:6-148).
 * `in` must have its ghost zones filled; `rfl`/`lfl` are 8-component flux
 * scratch of the same shape (FV only). */
static void rhs(const orc_grid *g, const orc_params *p, double *out, const double *in, double *rfl,
                double *lfl, double *mom)
{
    if (p->coll && !p->coll_direct) velocity_moments(g, in, mom);
    if (p->scheme == 0) {
        for (int c = 0; c < NCOMP; c++) weno7(g, in + c * g->cs, rfl + c * g->cs, lfl + c * g->cs);
        fill_ghosts(g, p->bc, rfl, NCOMP);
        fill_ghosts(g, p->bc, lfl, NCOMP);
    }
    const double ko = 1.0e-1; /* src/nuosc.hpp:60 */
#pragma omp parallel for collapse(2)
    for (int i = 0; i < g->nvz; i++) {
        for (int j = 0; j < g->nz; j++) {
            long q = at(g, i, j);
            double c[NCOMP], o[NCOMP];
            for (int k = 0; k < NCOMP; k++) {
                c[k] = in[k * g->cs + q];
                o[k] = 0.0;
            }
            double vi = g->vz[i];
            if (p->scheme == 0) {
                if (!p->advec_off) {
                    double fac = -vi / g->dz;
                    int s = sgn_d(vi);
                    for (int k = 0; k < NCOMP; k++) {
                        const double *R = rfl + k * g->cs, *L = lfl + k * g->cs;
                        o[k] += fac * fabs(1.0 + s) / 2 * (R[q] - R[q - 1]) +
                                fac * fabs(1.0 - s) / 2 * (L[q + 1] - L[q]);
                    }
                }
                if (p->vac) vacuum(g, p, c, o);
                if (p->mat) matter(g, j, c, o);
                if (p->coll) collective(g, p, in, mom, i, j, c, o);
            } else {
                if (p->vac) vacuum(g, p, c, o);
                if (p->mat) matter(g, j, c, o);
                if (!p->advec_off)
                    for (int k = 0; k < NCOMP; k++) o[k] += fd_advect(p, in + k * g->cs + q, vi, g->dz);
                if (p->coll) collective(g, p, in, mom, i, j, c, o);
                for (int k = 0; k < NCOMP; k++) o[k] += fd_ko(p, in + k * g->cs + q, g->dz, ko);
            }
            for (int k = 0; k < NCOMP; k++) out[k * g->cs + q] = o[k];
        }
    }
}

/* v0 = v1 + a*v2 (and v0 = v1 + a*(v2+v3)) over interior cells,
 * src/nuosc.hpp:281-318. */
static void axpy(const orc_grid *g, double *v0, const double *v1, double a, const double *v2,
                 const double *v3)
{
#pragma omp parallel for collapse(2)
    for (int c = 0; c < NCOMP; c++)
        for (int i = 0; i < g->nvz; i++)
            for (int j = 0; j < g->nz; j++) {
                long q = c * g->cs + at(g, i, j);
                v0[q] = v3 ? v1[q] + a * (v2[q] + v3[q]) : v1[q] + a * v2[q];
            }
}

void orc_rhs(const orc_params *p, double *out, const double *in_ghosted)
{
    orc_grid g;
    grid_make(p, &g);
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
    size_t n = (size_t)NCOMP * g.cs;
    double *rfl = (double *)calloc(n, sizeof(double));
    double *lfl = (double *)calloc(n, sizeof(double));
    double *mom = (double *)calloc(6 * (size_t)g.nz, sizeof(double));
    rhs(&g, p, out, in_ghosted, rfl, lfl, mom);
    free(rfl); free(lfl); free(mom);
    grid_free(&g);
}

/* Classical RK4 over four buffers with the reference's combine order and
 * pointer swaps, src/nuosc.hpp:320-348.  `y` is advanced in place `nsteps`
 * times; ghost zones of `y` are refreshed on return. */
int orc_step_rk4(const orc_params *p, double *y, int nsteps)
{
    orc_grid g;
    grid_make(p, &g);
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif
    size_t n = (size_t)NCOMP * g.cs;
    double *stat = (double *)malloc(n * sizeof(double));
    double *krhs = (double *)calloc(n, sizeof(double));
    double *pre = (double *)calloc(n, sizeof(double));
    double *cor = (double *)calloc(n, sizeof(double));
    double *rfl = (double *)calloc(n, sizeof(double));
    double *lfl = (double *)calloc(n, sizeof(double));
    double *mom = (double *)calloc(6 * (size_t)g.nz, sizeof(double));
    if (!stat || !krhs || !pre || !cor || !rfl || !lfl || !mom) return -1;
    memcpy(stat, y, n * sizeof(double));
    double dt = g.dt;
    for (int s = 0; s < nsteps; s++) {
        double *t;
        fill_ghosts(&g, p->bc, stat, NCOMP);
        rhs(&g, p, krhs, stat, rfl, lfl, mom);
        axpy(&g, pre, stat, 0.5 * dt, krhs, NULL);

        fill_ghosts(&g, p->bc, pre, NCOMP);
        rhs(&g, p, cor, pre, rfl, lfl, mom);
        axpy(&g, krhs, krhs, 2.0, cor, NULL);
        axpy(&g, cor, stat, 0.5 * dt, cor, NULL);
        t = pre; pre = cor; cor = t;

        fill_ghosts(&g, p->bc, pre, NCOMP);
        rhs(&g, p, cor, pre, rfl, lfl, mom);
        axpy(&g, krhs, krhs, 2.0, cor, NULL);
        axpy(&g, cor, stat, dt, cor, NULL);
        t = pre; pre = cor; cor = t;

        fill_ghosts(&g, p->bc, pre, NCOMP);
        rhs(&g, p, cor, pre, rfl, lfl, mom);
        axpy(&g, pre, stat, 1.0 / 6.0 * dt, cor, krhs);
        t = pre; pre = stat; stat = t;
    }
    fill_ghosts(&g, p->bc, stat, NCOMP);
    memcpy(y, stat, n * sizeof(double));
    free(stat); free(krhs); free(pre); free(cor); free(rfl); free(lfl); free(mom);
    grid_free(&g);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Initial conditions.                                                       */

/* Philox-4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11), the published
 * round function and Weyl key schedule. */
static void philox4x32(uint32_t ctr[4], uint32_t key0, uint32_t key1, uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key0, k1 = key1;
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void orc_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t *out)
{
    uint32_t ctr[4] = {c0, c1, c2, c3};
    philox4x32(ctr, k0, k1, out);
}

/* Normalised Gaussian angular profile on v in [-1, 1],
 * src/miscellaneous_funcs.hpp:57-62. */
static double gprof(double v, double v0, double sigma)
{
    double e = (v - v0) * (v - v0) / (2.0 * sigma * sigma);
    double N = sigma * sqrt(M_PI / 2.0) *
               (erf((1.0 + v0) / sigma / sqrt(2.0)) + erf((1.0 - v0) / sigma / sqrt(2.0)));
    return exp(-e) / N;
}

/* Seeded initial condition: G = g(v,1,sig_nu), bG = alpha*g(v,1,sig_nubar);
 * per cell two uniform draws in [-amp, amp] for (Re, Im) ex of nu and two for
 * nubar from Philox keyed by the seed with counter (j, i, instance, 0);
 * ee,xx = G/2 (1 +- sqrt(1 - er^2 - ei^2)), ex = G/2 (er + i ei), following
 * the shape of src/initialize.hpp:30-38.  Writes G/bG per cell and the
 * 8-component state (reference layout, ghosts filled for `bc`). */
void orc_init_seeded(const orc_params *p, uint64_t seed, uint32_t instance, double sig_nu,
                     double sig_nubar, double alpha, double amp, double *G, double *bG, double *state)
{
    orc_grid g;
    grid_make(p, &g);
    for (int i = 0; i < g.nvz; i++) {
        double gv = gprof(g.vz[i], 1.0, sig_nu);
        double bgv = alpha * gprof(g.vz[i], 1.0, sig_nubar);
        for (int j = 0; j < g.nz; j++) {
            long q = at(&g, i, j);
            uint32_t ctr[4] = {(uint32_t)j, (uint32_t)i, instance, 0u}, r[4];
            philox4x32(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), r);
            double e[4];
            for (int t = 0; t < 4; t++) e[t] = amp * (2.0 * (((double)r[t] + 0.5) / 4294967296.0) - 1.0);
            double s = sqrt(1.0 - e[0] * e[0] - e[1] * e[1]);
            double bs = sqrt(1.0 - e[2] * e[2] - e[3] * e[3]);
            G[q] = gv;
            bG[q] = bgv;
            state[EE * g.cs + q] = 0.5 * gv * (1.0 + s);
            state[XX * g.cs + q] = 0.5 * gv * (1.0 - s);
            state[EXR * g.cs + q] = 0.5 * gv * e[0];
            state[EXI * g.cs + q] = 0.5 * gv * e[1];
            state[BEE * g.cs + q] = 0.5 * bgv * (1.0 + bs);
            state[BXX * g.cs + q] = 0.5 * bgv * (1.0 - bs);
            state[BEXR * g.cs + q] = 0.5 * bgv * e[2];
            state[BEXI * g.cs + q] = 0.5 * bgv * e[3];
        }
    }
    fill_ghosts(&g, p->bc, state, NCOMP);
    grid_free(&g);
}

/* The reference's own default initial condition, src/initialize.hpp:6-47
 * with eps/eps_ from src/miscellaneous_funcs.hpp:66-78. */
void orc_init_reference(const orc_params *p, double perturbation_size, double *G, double *bG, double *state)
{
    orc_grid g;
    grid_make(p, &g);
    const double signu = 0.6, sigbnu = 0.6, alpha = 0.90;
    for (int i = 0; i < g.nvz; i++) {
        for (int j = 0; j < g.nz; j++) {
            long q = at(&g, i, j);
            double z = g.Z[j];
            double e = perturbation_size * exp(-(z - 0.0) * (z - 0.0) / 50.0);
            double e_ = sqrt(1.0 - e * e);
            G[q] = gprof(g.vz[i], 1.0, signu);
            bG[q] = alpha * gprof(g.vz[i], 1.0, sigbnu);
            state[EE * g.cs + q] = 0.5 * G[q] * (1.0 + e_);
            state[XX * g.cs + q] = 0.5 * G[q] * (1.0 - e_);
            state[EXR * g.cs + q] = 0.5 * G[q] * (0.0 + e);
            state[EXI * g.cs + q] = -0.0;
            state[BEE * g.cs + q] = 0.5 * bG[q] * (1.0 + e_);
            state[BXX * g.cs + q] = 0.5 * bG[q] * (1.0 - e_);
            state[BEXR * g.cs + q] = 0.5 * bG[q] * (0.0 + e);
            state[BEXI * g.cs + q] = 0.0;
        }
    }
    fill_ghosts(&g, p->bc, state, NCOMP);
    grid_free(&g);
}

/* ------------------------------------------------------------------------ */
/* Analysis, src/analysis.hpp.                                               */

/* Output slots of orc_analyse. */
enum {
    D_DPMAX = 0, /* max(max|dP|, max|dbP|)            dcon, analysis.hpp:108-125 */
    D_AVDP,      /* sum |d|P|| G / sum G                                          */
    D_AVBDP,     /* sum |d|bP|| bG / sum bG                                       */
    D_M0NORM,    /* |M0|                               cal_Mn, analysis.hpp:50-67  */
    D_M0E1, D_M0E2, D_M0E3,
    D_PEE,       /* <Pee>  = sum ee / sum ee0          surv_prob, analysis.hpp:169-182 */
    D_PBEE,      /* <Pbee> = sum bee / sum bee0                                     */
    D_TRACE,     /* sum (ee+xx) dz dv                                               */
    D_BTRACE,    /* sum (bee+bxx) dz dv                                             */
    D_ELN,       /* sum (ee - bee) dz dv                                            */
    D_NSLOTS
};

/* Polarisation of one cell, cal_pol analysis.hpp:27-46 (note the + sign on
 * bP2). */
static void pol(const double *c, double G, double bG, double P[3], double bP[3], double *n, double *bn)
{
    P[0] = 2.0 * c[EXR] / G;
    P[1] = -2.0 * c[EXI] / G;
    P[2] = (c[EE] - c[XX]) / G;
    *n = fabs(sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]));
    bP[0] = 2.0 * c[BEXR] / bG;
    bP[1] = 2.0 * c[BEXI] / bG;
    bP[2] = (c[BEE] - c[BXX]) / bG;
    *bn = fabs(sqrt(bP[0] * bP[0] + bP[1] * bP[1] + bP[2] * bP[2]));
}

/* analyse + surv_prob in the reference's summation order (i outer, j inner). */
void orc_analyse(const orc_params *p, const double *state, const double *G, const double *bG,
                 const double *state0, double *out)
{
    orc_grid g;
    grid_make(p, &g);
    double dP = 0, dbP = 0, avdP = 0, avbdP = 0, N0 = 0, bN0 = 0;
    double e1 = 0, e2 = 0, e3 = 0;
    double nee = 0, nbee = 0, dee = 0, dbee = 0, tr = 0, btr = 0, eln = 0;
    double dzdv = g.dz * g.dv;
    for (int i = 0; i < g.nvz; i++) {
        for (int j = 0; j < g.nz; j++) {
            long q = at(&g, i, j);
            double c[NCOMP], c0[NCOMP], P[3], bP[3], P0[3], bP0[3], n, bn, n0, bn0;
            for (int k = 0; k < NCOMP; k++) {
                c[k] = state[k * g.cs + q];
                c0[k] = state0[k * g.cs + q];
            }
            pol(c, G[q], bG[q], P, bP, &n, &bn);
            pol(c0, G[q], bG[q], P0, bP0, &n0, &bn0);
            /* L(v, 0) == 1 */
            e1 += 1.0 * (G[q] * P[0] - bG[q] * bP[0]) * g.dz * g.dv;
            e2 += 1.0 * (G[q] * P[1] - bG[q] * bP[1]) * g.dz * g.dv;
            e3 += 1.0 * (G[q] * P[2] - bG[q] * bP[2]) * g.dz * g.dv;
            double a = fabs(n - n0), b = fabs(bn - bn0);
            dP = (dP >= a) ? dP : a;
            dbP = (dbP >= b) ? dbP : b;
            avdP += a * G[q];
            avbdP += b * bG[q];
            N0 += G[q];
            bN0 += bG[q];
            nee += c[EE] * g.dz * g.dv;
            nbee += c[BEE] * g.dz * g.dv;
            dee += c0[EE] * g.dz * g.dv;
            dbee += c0[BEE] * g.dz * g.dv;
            tr += (c[EE] + c[XX]) * dzdv;
            btr += (c[BEE] + c[BXX]) * dzdv;
            eln += (c[EE] - c[BEE]) * dzdv;
        }
    }
    out[D_DPMAX] = (dP >= dbP) ? dP : dbP;
    out[D_AVDP] = avdP / N0;
    out[D_AVBDP] = avbdP / bN0;
    out[D_M0E1] = e1;
    out[D_M0E2] = e2;
    out[D_M0E3] = e3;
    out[D_M0NORM] = sqrt(e1 * e1 + e2 * e2 + e3 * e3);
    out[D_PEE] = nee / dee;
    out[D_PBEE] = nbee / dbee;
    out[D_TRACE] = tr;
    out[D_BTRACE] = btr;
    out[D_ELN] = eln;
    grid_free(&g);
}

/* Angle-resolved survival probability P_ee(v) = sum_z ee / sum_z ee0 per
 * velocity bin (the per-v analogue of surv_prob, analysis.hpp:169-176). */
void orc_pee_v(const orc_params *p, const double *state, const double *state0, double *pee, double *pbee)
{
    orc_grid g;
    grid_make(p, &g);
    for (int i = 0; i < g.nvz; i++) {
        double a = 0, b = 0, a0 = 0, b0 = 0;
        for (int j = 0; j < g.nz; j++) {
            long q = at(&g, i, j);
            a += state[EE * g.cs + q];
            b += state[BEE * g.cs + q];
            a0 += state0[EE * g.cs + q];
            b0 += state0[BEE * g.cs + q];
        }
        pee[i] = a / a0;
        pbee[i] = b / b0;
    }
    grid_free(&g);
}
