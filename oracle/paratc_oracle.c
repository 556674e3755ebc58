/*
 * paratc_oracle.c -- TEST INFRASTRUCTURE, not product code.
 *
 * A CPU restatement (C11 + OpenMP) of the per-RK3-substep hot path of ParaTC
 * (GongZheng-Justin/ParaTC, Fortran 2003 + MPI).  Only tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py load it, as the
 * checker the CUDA library is compared against; the library never calls it.
 *
 * Fidelity: every routine follows the Fortran routine named beside it, keeping
 * the loop order over a z-plane, the halo'd array bounds of mb1 (x -1..nxc+2,
 * y 0..nyp, z -1..nzc+2), the halo exchange of a single rank (self copies of
 * myupdate_halo, src/m_Decomp2d.f90:1554-1709) and the grouping of every
 * floating-point expression (Fortran evaluates a+b+c and a*b*c left to right;
 * so does C).  Built with -ffp-contract=off so that no FMA is formed.
 * Reductions are summed per z-plane and then over the planes in order, so the
 * result does not depend on the thread count.
 *
 * Third-party arithmetic: the reference transforms with FFTW 3.3.9
 * (src/ThirdParty/install_thirdParty.sh:12) through fftw_plan_guru_r2r with
 * FFTW_R2HC / FFTW_HC2R (src/m_Poisson.f90:180-244).  FFTW is built by its own
 * configure system, so under the rules of this build it counts as
 * unbuildable; its published transform is restated here instead: R2HC gives
 * r_0..r_{n/2}, i_{(n+1)/2-1}..i_1 of X_k = sum_j x_j exp(-2 pi i j k / n),
 * HC2R is the unnormalised inverse.  The transform itself is a mixed-radix
 * Cooley-Tukey FFT of two real rows packed into one complex row, with
 * twiddles evaluated in long double.  tests/ pin it against numpy.fft.
 *
 * PARITY UNPINNED: the reference ships no tests, golden vectors or fixtures,
 * and it cannot be run in this container (no Fortran compiler, no MPI), so no
 * output of the reference itself pins this restatement.  What pins it instead
 * (tests/test_oracle_*.py): an independent numpy restatement of the same
 * routines at small sizes, numpy's FFT for the halfcomplex convention,
 * scipy's banded solver for the Thomas sweeps, and discrete identities of the
 * scheme (4th-order modified wavenumber = symbol of D4 o D4, so the divergence
 * after a projection is at round-off; a manufactured single-mode Poisson
 * solution; the laminar Poiseuille profile as a fixed point).
 */
#include "paratc_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

#define FFT_MAXF 40
#define FFT_MAXP 64

typedef struct {
    int n, nf;
    int fac[FFT_MAXF];
    cplx* w;            /* w[k] = exp(-2 pi i k / n) */
} fftplan;

struct orc {
    paratc_params p;
    int nxc, nyc, nzc, nyp;
    size_t nxt, nyt, nzt, nh, ni;
    /* m_MeshAndMetries */
    double dx, dy, dz, rdx, rdy, rdz, dx2, dy2, dz2, rdx2, rdy2, rdz2;
    double *yp, *yc, *dyp, *dyc, *rdyp, *rdyc, *yinterp;          /* 0..nyp */
    double *ap2ph, *ac2ph, *am2ph, *ap2c, *ac2c, *am2c;           /* 1..nyc */
    double *ap2cCN, *ac2cCN, *am2cCN, *ap2p, *ac2p, *am2p;
    double *ap2cSc, *ac2cSc, *am2cSc, *ap2cScCN, *ac2cScCN, *am2cScCN;
    double dxC[4], dzC[4], dxxC[5], dzzC[5], IC[4];
    /* m_Poisson */
    double *wnx, *wnz;                                            /* 1..n */
    double normfft;
    fftplan px, pz;
    /* m_Parameters */
    int iadvance;
    double gamc[3], thec[3], alpc[3];
    double pmGamma, pmTheta, pmAlpha, pmAlphaC, pmBeta, pmBetaSc;
    double dt, sim_time, pr_grad_aver;
    /* m_Variables */
    double *ux, *uy, *uz, *pr, *sc, *phi;                          /* halo */
    double *hx, *hy, *hz, *hc;                                     /* interior */
    double *rhsx, *rhsy, *rhsz, *rhsc, *prsrc, *phi_int;           /* interior */
    double *uy_ym, *duy_ym;                                        /* nxc*nzc */
    double *uxhx, *uyhx, *uzhx, *uxhz, *uyhz, *uzhz;               /* halo temps */
    double *pln;                                                    /* per-plane partials */
};

/* Fortran index helpers: halo'd arrays (mb1 bounds) and interior arrays */
#define HX(o, i, j, k) ((((size_t)((k) + 1)) * (o)->nyt + (size_t)(j)) * (o)->nxt + (size_t)((i) + 1))
#define IX(o, i, j, k) ((((size_t)((k) - 1)) * (size_t)(o)->nyc + (size_t)((j) - 1)) * (size_t)(o)->nxc + (size_t)((i) - 1))

static const double zero = 0.0, quarter = 0.25, half = 0.5, one = 1.0, two = 2.0,
                    three = 3.0, four = 4.0, five = 5.0, eight = 8.0, twelve = 12.0,
                    fifteen = 15.0, seventeen = 17.0, sixty = 60.0;
static const double twopi = 6.283185307179586476925286766559005768;

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------
 * FFT (restating the DFT definition FFTW documents for R2HC / HC2R)
 * ---------------------------------------------------------------------- */
static int fft_plan_init(fftplan* pl, int n) {
    int m = n, nf = 0;
    pl->n = n;
    while (m % 4 == 0 && nf < FFT_MAXF) { pl->fac[nf++] = 4; m /= 4; }
    while (m % 2 == 0 && nf < FFT_MAXF) { pl->fac[nf++] = 2; m /= 2; }
    for (int f = 3; m > 1 && nf < FFT_MAXF; f += 2)
        while (m % f == 0) { pl->fac[nf++] = f; m /= f; }
    pl->nf = nf;
    for (int i = 0; i < nf; i++) if (pl->fac[i] > FFT_MAXP) return -1;
    pl->w = (cplx*)malloc(sizeof(cplx) * (size_t)n);
    if (!pl->w) return -1;
    for (int k = 0; k < n; k++) {
        long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
        pl->w[k].re = (double)cosl(a);
        pl->w[k].im = (double)sinl(a);
    }
    return 0;
}

static void fft_rec(const fftplan* pl, int n, int fi, const cplx* in, size_t s, cplx* out) {
    if (n == 1) { out[0] = in[0]; return; }
    const int p = pl->fac[fi], m = n / p, N = pl->n, tm = N / n, tp = N / p;
    for (int r = 0; r < p; r++) fft_rec(pl, m, fi + 1, in + (size_t)r * s, s * (size_t)p, out + (size_t)r * m);
    cplx t[FFT_MAXP];
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) {
            cplx y = out[(size_t)r * m + k];
            cplx w = pl->w[((size_t)r * k * tm) % N];
            t[r].re = y.re * w.re - y.im * w.im;
            t[r].im = y.re * w.im + y.im * w.re;
        }
        for (int q = 0; q < p; q++) {
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < p; r++) {
                cplx w = pl->w[((size_t)r * q * tp) % N];
                sr += t[r].re * w.re - t[r].im * w.im;
                si += t[r].re * w.im + t[r].im * w.re;
            }
            out[k + (size_t)q * m].re = sr;
            out[k + (size_t)q * m].im = si;
        }
    }
}

/* two real rows a,b (length n) -> halfcomplex ha,hb */
static void r2hc_pair(const fftplan* pl, const double* a, const double* b, double* ha, double* hb,
                      cplx* zin, cplx* zout) {
    const int n = pl->n;
    for (int j = 0; j < n; j++) { zin[j].re = a[j]; zin[j].im = b[j]; }
    fft_rec(pl, n, 0, zin, 1, zout);
    for (int k = 0; k <= n / 2; k++) {
        cplx zk = zout[k], zn = zout[(n - k) % n];
        double are = half * (zk.re + zn.re), aim = half * (zk.im - zn.im);
        double bre = half * (zk.im + zn.im), bim = half * (zn.re - zk.re);
        ha[k] = are; hb[k] = bre;
        if (k > 0 && 2 * k < n) { ha[n - k] = aim; hb[n - k] = bim; }
    }
}

/* halfcomplex ha,hb -> unnormalised inverse real rows a,b */
static void hc2r_pair(const fftplan* pl, const double* ha, const double* hb, double* a, double* b,
                      cplx* zin, cplx* zout) {
    const int n = pl->n;
    for (int k = 0; k < n; k++) {
        double are, aim, bre, bim;
        if (k == 0) { are = ha[0]; aim = 0.0; bre = hb[0]; bim = 0.0; }
        else if (2 * k == n) { are = ha[k]; aim = 0.0; bre = hb[k]; bim = 0.0; }
        else if (2 * k < n) { are = ha[k]; aim = ha[n - k]; bre = hb[k]; bim = hb[n - k]; }
        else { are = ha[n - k]; aim = -ha[k]; bre = hb[n - k]; bim = -hb[k]; }
        /* Z = A + i B, conjugated for the inverse-by-forward trick */
        zin[k].re = are - bim;
        zin[k].im = -(aim + bre);
    }
    fft_rec(pl, n, 0, zin, 1, zout);
    for (int j = 0; j < n; j++) { a[j] = zout[j].re; b[j] = -zout[j].im; }
}

int orc_r2hc(int n, const double* in, double* out) {
    fftplan pl;
    if (n < 1 || fft_plan_init(&pl, n)) return PARATC_ERR_BAD_ARG;
    cplx* z = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)n);
    double* zb = (double*)calloc((size_t)n * 2, sizeof(double));
    r2hc_pair(&pl, in, zb, out, zb + n, z, z + n);
    free(z); free(zb); free(pl.w);
    return 0;
}

int orc_hc2r(int n, const double* in, double* out) {
    fftplan pl;
    if (n < 1 || fft_plan_init(&pl, n)) return PARATC_ERR_BAD_ARG;
    cplx* z = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)n);
    double* zb = (double*)calloc((size_t)n * 2, sizeof(double));
    hc2r_pair(&pl, in, zb, out, zb + n, z, z + n);
    free(z); free(zb); free(pl.w);
    return 0;
}

/* ------------------------------------------------------------------------
 * clcYcoord  (src/m_MeshAndMetries.f90:340-408) for all sections
 * (section loop: src/m_MeshAndMetries.f90:166-181)
 * ---------------------------------------------------------------------- */
static void clc_ycoord(double* yc1 /* yc1[j] = ycoord(j), 1-based */, int nid1, int nid2,
                       double ys1, double ys2, int stret_type, double cstret, int stret_option) {
    int m = nid2 - nid1;
    double ylen = ys2 - ys1, tstr, xi, y0;
    yc1[nid1] = ys1;
    yc1[nid2] = ys2;
    switch (stret_type) {
    case 0:
        for (int j = 0; j <= m; j++) yc1[nid1 + j] = ys1 + (double)j / (double)m * ylen;
        break;
    case 1:
        tstr = tanh(cstret);
        for (int j = 0; j <= m; j++) {
            xi = (double)j / (double)(float)m;
            y0 = tanh(cstret * (xi - one)) / tstr + one;
            if (stret_option == 0) yc1[nid1 + j] = ys1 + y0 * ylen;
            else                   yc1[nid2 - j] = ys2 - y0 * ylen;
        }
        break;
    case 2: {
        const double PI = 3.141592653589793238462643383279502884;
        tstr = sin(half * cstret * PI);
        for (int j = 0; j <= m; j++) {
            xi = (double)j / (double)m - one;
            y0 = sin(cstret * xi * PI * half) / tstr + one;
            if (stret_option == 0) yc1[nid1 + j] = ys1 + y0 * ylen;
            else                   yc1[nid2 - j] = ys2 - y0 * ylen;
        }
        break;
    }
    case 3:
        if (cstret == one) {
            for (int j = 0; j <= m; j++) yc1[j + nid1] = ys1 + (double)j / (double)m * ylen;
        } else {
            tstr = (pow(cstret, m) - one) / (cstret - one);
            for (int j = 0; j <= m - 1; j++) {
                y0 = pow(cstret, j) / tstr;
                if (stret_option == 0) { int jt = nid1 + j; yc1[jt + 1] = yc1[jt] + y0 * ylen; }
                else                   { int jt = nid2 - j; yc1[jt - 1] = yc1[jt] - y0 * ylen; }
            }
        }
        break;
    }
    yc1[nid1] = ys1;
    yc1[nid2] = ys2;
}

int orc_ycoord(int nsection, const double* section_length, const double* section_cstret,
               const int32_t* nyc_section, const int32_t* stret_type,
               const int32_t* stret_option, double yly, double* yp_out) {
    if (nsection < 1) return PARATC_ERR_BAD_ARG;
    int nyc = 0;
    double sumlen = 0.0;
    for (int s = 0; s < nsection; s++) {
        if (section_length[s] < 0 || section_cstret[s] < 0 || nyc_section[s] < 1 ||
            stret_type[s] < 0 || stret_type[s] > 3 || stret_option[s] < 0 || stret_option[s] > 1)
            return PARATC_ERR_BAD_ARG;
        nyc += nyc_section[s];
        sumlen += section_length[s];
    }
    int nyp = nyc + 1;
    double* y1 = (double*)calloc((size_t)nyp + 2, sizeof(double));
    int* nid = (int*)malloc(sizeof(int) * (size_t)(nsection + 1));
    double* ysc = (double*)malloc(sizeof(double) * (size_t)(nsection + 1));
    nid[0] = 1; ysc[0] = 0.0;
    for (int s = 0; s < nsection; s++) {
        nid[s + 1] = nid[s] + nyc_section[s];
        ysc[s + 1] = ysc[s] + section_length[s] / sumlen * yly;
    }
    ysc[nsection] = yly;
    for (int s = 0; s < nsection; s++)
        clc_ycoord(y1, nid[s], nid[s + 1], ysc[s], ysc[s + 1], stret_type[s], section_cstret[s], stret_option[s]);
    for (int j = 1; j <= nyp; j++) yp_out[j - 1] = y1[j];
    free(y1); free(nid); free(ysc);
    return 0;
}

/* ------------------------------------------------------------------------
 * myupdate_halo for the y pencil of a single rank: periodic self copies
 * (src/m_Decomp2d.f90:1612-1706). y halos are never requested on the hot path.
 * ---------------------------------------------------------------------- */
static void upd_halo(orc_t* o, double* a, int xmh, int xph, int zmh, int zph) {
    const int nxc = o->nxc, nzc = o->nzc, nyp = o->nyp;
    /* step 3: x- halo over y 0..nyp, z -1..nzc+2 */
    if (xmh > 0) {
#pragma omp parallel for schedule(static)
        for (int k = -1; k <= nzc + 2; k++)
            for (int j = 0; j <= nyp; j++)
                for (int h = 0; h < xmh; h++)
                    a[HX(o, 1 - xmh + h, j, k)] = a[HX(o, nxc - xmh + 1 + h, j, k)];
    }
    /* step 4: x+ halo */
    if (xph > 0) {
#pragma omp parallel for schedule(static)
        for (int k = -1; k <= nzc + 2; k++)
            for (int j = 0; j <= nyp; j++)
                for (int h = 0; h < xph; h++)
                    a[HX(o, nxc + 1 + h, j, k)] = a[HX(o, 1 + h, j, k)];
    }
    /* step 5: z- halo over x -1..nxc+2, y 0..nyp */
    for (int h = 0; h < zmh; h++) {
        int kr = 1 - zmh + h, ks = nzc - zmh + 1 + h;
        memcpy(&a[HX(o, -1, 0, kr)], &a[HX(o, -1, 0, ks)], sizeof(double) * o->nxt * o->nyt);
    }
    /* step 6: z+ halo */
    for (int h = 0; h < zph; h++) {
        int kr = nzc + 1 + h, ks = 1 + h;
        memcpy(&a[HX(o, -1, 0, kr)], &a[HX(o, -1, 0, ks)], sizeof(double) * o->nxt * o->nyt);
    }
}

/* ------------------------------------------------------------------------
 * m_BC_and_Halo
 * ---------------------------------------------------------------------- */
/* SetBC_and_UpdateHalo (src/m_BC_and_Halo.f90:23-64) */
static void bc_vel(orc_t* o) {
    const int nxc = o->nxc, nzc = o->nzc, nyc = o->nyc, nyp = o->nyp;
    const paratc_params* P = &o->p;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++)
        for (int ic = 1; ic <= nxc; ic++) {
            if (P->flow_type == PARATC_FT_CH) {
                o->ux[HX(o, ic, nyp, kc)] = P->ux_bc[3] * two - o->ux[HX(o, ic, nyc, kc)];
                o->uy[HX(o, ic, nyp, kc)] = P->uy_bc[3];
                o->uz[HX(o, ic, nyp, kc)] = P->uz_bc[3] * two - o->uz[HX(o, ic, nyc, kc)];
            } else {
                o->ux[HX(o, ic, nyp, kc)] = o->ux[HX(o, ic, nyc, kc)];
                o->uy[HX(o, ic, nyp, kc)] = zero;
                o->uz[HX(o, ic, nyp, kc)] = o->uz[HX(o, ic, nyc, kc)];
            }
            o->ux[HX(o, ic, 0, kc)] = P->ux_bc[2] * two - o->ux[HX(o, ic, 1, kc)];
            o->uy[HX(o, ic, 1, kc)] = o->uy_ym[(size_t)(kc - 1) * nxc + (ic - 1)];
            o->uz[HX(o, ic, 0, kc)] = P->uz_bc[2] * two - o->uz[HX(o, ic, 1, kc)];
        }
    upd_halo(o, o->ux, 2, 2, 2, 2);
    upd_halo(o, o->uy, 2, 2, 2, 2);
    upd_halo(o, o->uz, 2, 2, 2, 2);
}

/* SetBC_and_UpdateHaloForPrSrc (src/m_BC_and_Halo.f90:69-103) */
static void bc_prsrc(orc_t* o) {
    const int nxc = o->nxc, nzc = o->nzc, nyp = o->nyp;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++)
        for (int ic = 1; ic <= nxc; ic++) {
            o->uy[HX(o, ic, nyp, kc)] = (o->p.flow_type == PARATC_FT_CH) ? o->p.uy_bc[3] : zero;
            o->uy[HX(o, ic, 1, kc)] = o->uy_ym[(size_t)(kc - 1) * nxc + (ic - 1)];
        }
    upd_halo(o, o->ux, 1, 2, 0, 0);
    upd_halo(o, o->uz, 0, 0, 1, 2);
}

/* SetBC_and_UpdateHalo_pr (src/m_BC_and_Halo.f90:108-122) */
static void bc_pr(orc_t* o, double* a) {
    const int nxc = o->nxc, nzc = o->nzc, nyc = o->nyc, nyp = o->nyp;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++)
        for (int ic = 1; ic <= nxc; ic++) {
            a[HX(o, ic, 0, kc)] = a[HX(o, ic, 1, kc)];
            a[HX(o, ic, nyp, kc)] = a[HX(o, ic, nyc, kc)];
        }
    upd_halo(o, a, 2, 1, 2, 1);
}

/* SetBC_and_UpdateHalo_scalar (src/m_BC_and_Halo.f90:128-178) */
static void bc_scalar(orc_t* o) {
    const int nxc = o->nxc, nzc = o->nzc, nyc = o->nyc, nyp = o->nyp;
    const double* v = o->p.scalar_bc_values;
    double r1b = 0, r2b = 0, r1t = 0, r2t = 0;
    switch (o->p.scalar_bc_option[0]) {
    case -1: r1b = -one; r2b = two * v[0]; break;
    case -2: r1b = one; r2b = -o->dyc[1] * v[2]; break;
    case -3: r1b = (two + v[0] * o->dyc[1]) / (two - v[0] * o->dyc[1]);
             r2b = -(two * v[2] * o->dyc[1] / (two - v[0] * o->dyc[1])); break;
    }
    switch (o->p.scalar_bc_option[1]) {
    case -1: r1t = -one; r2t = two * v[1]; break;
    case -2: r1t = one; r2t = o->dyc[nyp] * v[3]; break;
    case -3: r1t = (two - v[1] * o->dyc[nyp]) / (two + v[1] * o->dyc[nyp]);
             r2t = two * v[3] * o->dyc[nyp] / (two + v[1] * o->dyc[nyp]); break;
    }
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++)
        for (int ic = 1; ic <= nxc; ic++) {
            o->sc[HX(o, ic, 0, kc)] = r1b * o->sc[HX(o, ic, 1, kc)] + r2b;
            o->sc[HX(o, ic, nyp, kc)] = r1t * o->sc[HX(o, ic, nyc, kc)] + r2t;
        }
    upd_halo(o, o->sc, 2, 2, 2, 2);
}

/* ------------------------------------------------------------------------
 * set-up: InitMeshAndMetries (src/m_MeshAndMetries.f90:86-335),
 * ReadAndInitParameters RK constants (src/m_Parameters.f90:159-174),
 * InitPoissonSolver wavenumbers (src/m_Poisson.f90:36-48),
 * AllocateVariables (src/m_Variables.f90:41-105)
 * ---------------------------------------------------------------------- */
static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

static int metrics_init(orc_t* o, const double* yp_in) {
    const paratc_params* P = &o->p;
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc, nyp = o->nyp;
    o->dx = P->xlx / (double)nxc; o->dy = P->yly / (double)nyc; o->dz = P->zlz / (double)nzc;
    o->rdx = (double)nxc / P->xlx; o->rdy = (double)nyc / P->yly; o->rdz = (double)nzc / P->zlz;
    o->dx2 = o->dx * o->dx; o->rdx2 = o->rdx * o->rdx;
    o->dy2 = o->dy * o->dy; o->rdy2 = o->rdy * o->rdy;
    o->dz2 = o->dz * o->dz; o->rdz2 = o->rdz * o->rdz;
    const double rdx = o->rdx, rdz = o->rdz, rdx2 = o->rdx2, rdz2 = o->rdz2;
    o->dxC[0] = rdx / 24.0; o->dxC[1] = -rdx * 1.125; o->dxC[2] = rdx * 1.125; o->dxC[3] = -rdx / 24.0;
    o->dzC[0] = rdz / 24.0; o->dzC[1] = -rdz * 1.125; o->dzC[2] = rdz * 1.125; o->dzC[3] = -rdz / 24.0;
    o->dxxC[0] = -rdx2 / 12.0; o->dxxC[1] = 4.0 / 3.0 * rdx2; o->dxxC[2] = -2.5 * rdx2;
    o->dxxC[3] = 4.0 / 3.0 * rdx2; o->dxxC[4] = -rdx2 / 12.0;
    o->dzzC[0] = -rdz2 / 12.0; o->dzzC[1] = 4.0 / 3.0 * rdz2; o->dzzC[2] = -2.5 * rdz2;
    o->dzzC[3] = 4.0 / 3.0 * rdz2; o->dzzC[4] = -rdz2 / 12.0;
    o->IC[0] = -1.0 / 16.0; o->IC[1] = 9.0 / 16.0; o->IC[2] = 9.0 / 16.0; o->IC[3] = -1.0 / 16.0;

    size_t ny1 = (size_t)nyp + 1;
    double** arrs[] = {&o->yp, &o->yc, &o->dyp, &o->dyc, &o->rdyp, &o->rdyc, &o->yinterp,
                       &o->ap2ph, &o->ac2ph, &o->am2ph, &o->ap2c, &o->ac2c, &o->am2c,
                       &o->ap2cCN, &o->ac2cCN, &o->am2cCN, &o->ap2p, &o->ac2p, &o->am2p,
                       &o->ap2cSc, &o->ac2cSc, &o->am2cSc, &o->ap2cScCN, &o->ac2cScCN, &o->am2cScCN};
    for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++) {
        *arrs[a] = dalloc(ny1);
        if (!*arrs[a]) return PARATC_ERR_OOM;
    }
    double *yp = o->yp, *yc = o->yc, *dyp = o->dyp, *dyc = o->dyc, *rdyp = o->rdyp, *rdyc = o->rdyc;
    for (int j = 1; j <= nyp; j++) yp[j] = yp_in[j - 1];
    for (int j = 1; j <= nyc; j++) yc[j] = half * (yp[j] + yp[j + 1]);
    yc[0] = two * yp[1] - yc[1];
    yc[nyp] = two * yp[nyp] - yc[nyc];
    for (int j = 1; j <= nyc; j++) dyp[j] = yp[j + 1] - yp[j];
    dyp[0] = dyp[1];
    dyp[nyp] = dyp[nyc];
    for (int j = 2; j <= nyc; j++) dyc[j] = yc[j] - yc[j - 1];
    dyc[1] = dyp[1];
    dyc[nyp] = dyp[nyc];
    for (int j = 0; j <= nyp; j++) rdyp[j] = one / dyp[j];
    for (int j = 1; j <= nyp; j++) rdyc[j] = one / dyc[j];
    for (int j = 1; j <= nyp; j++) o->yinterp[j] = dyp[j] / (dyp[j] + dyp[j - 1]);
    /* pressure */
    for (int j = 1; j <= nyc; j++) { o->am2ph[j] = rdyp[j] * rdyc[j]; o->ap2ph[j] = rdyp[j] * rdyc[j + 1]; }
    o->am2ph[1] = zero; o->ap2ph[1] = rdyp[1] * rdyc[2];
    o->am2ph[nyc] = rdyp[nyc] * rdyc[nyc]; o->ap2ph[nyc] = zero;
    for (int j = 1; j <= nyc; j++) o->ac2ph[j] = -(o->am2ph[j] + o->ap2ph[j]);
    /* ux/uz */
    for (int j = 1; j <= nyc; j++) { o->am2c[j] = rdyp[j] * rdyc[j]; o->ap2c[j] = rdyp[j] * rdyc[j + 1]; }
    o->am2c[1] = four * rdyc[1] / (dyc[1] + two * dyc[2]);
    o->ap2c[1] = four * rdyc[2] / (dyc[1] + two * dyc[2]);
    if (o->p.flow_type == PARATC_FT_CH) {
        o->am2c[nyc] = four * rdyc[nyc] / (dyc[nyp] + two * dyc[nyc]);
        o->ap2c[nyc] = four * rdyc[nyp] / (dyc[nyp] + two * dyc[nyc]);
    } else {
        o->am2c[nyc] = rdyp[nyc] * rdyc[nyc];
        o->ap2c[nyc] = zero;
    }
    for (int j = 1; j <= nyc; j++) o->ac2c[j] = -(o->am2c[j] + o->ap2c[j]);
    for (int j = 1; j <= nyc; j++) { o->ap2cCN[j] = o->ap2c[j]; o->ac2cCN[j] = o->ac2c[j]; o->am2cCN[j] = o->am2c[j]; }
    o->ap2cCN[1] = o->ap2c[1];
    o->ac2cCN[1] = o->ac2c[1] - o->am2c[1];
    o->am2cCN[1] = two * o->am2c[1];
    if (o->p.flow_type == PARATC_FT_CH) {
        o->am2cCN[nyc] = o->am2c[nyc];
        o->ac2cCN[nyc] = o->ac2c[nyc] - o->ap2c[nyc];
        o->ap2cCN[nyc] = two * o->ap2c[nyc];
    }
    /* uy */
    for (int j = 1; j <= nyc; j++) { o->am2p[j] = rdyc[j] * rdyp[j - 1]; o->ap2p[j] = rdyc[j] * rdyp[j]; }
    for (int j = 1; j <= nyc; j++) o->ac2p[j] = -(o->am2p[j] + o->ap2p[j]);
    /* scalar (src/m_MeshAndMetries.f90:283-334) */
    if (o->p.scalar_on) {
        const int* opt = o->p.scalar_bc_option;
        const double* v = o->p.scalar_bc_values;
        for (int j = 1; j <= nyc; j++) { o->am2cSc[j] = rdyp[j] * rdyc[j]; o->ap2cSc[j] = rdyp[j] * rdyc[j + 1]; }
        if (opt[0] == -1) {
            o->am2cSc[1] = four * rdyc[1] / (dyc[1] + two * dyc[2]);
            o->ap2cSc[1] = four * rdyc[2] / (dyc[1] + two * dyc[2]);
        }
        if (opt[1] == -1) {
            o->am2cSc[nyc] = four * rdyc[nyc] / (dyc[nyp] + two * dyc[nyc]);
            o->ap2cSc[nyc] = four * rdyc[nyp] / (dyc[nyp] + two * dyc[nyc]);
        }
        for (int j = 1; j <= nyc; j++) o->ac2cSc[j] = -(o->am2cSc[j] + o->ap2cSc[j]);
        for (int j = 1; j <= nyc; j++) { o->am2cScCN[j] = rdyp[j] * rdyc[j]; o->ap2cScCN[j] = rdyp[j] * rdyc[j + 1]; }
        for (int j = 1; j <= nyc; j++) o->ac2cScCN[j] = -(o->am2cScCN[j] + o->ap2cScCN[j]);
        switch (opt[0]) {
        case -1:
            o->am2cScCN[1] = eight * rdyc[1] / (dyc[1] + two * dyc[2]);
            o->ap2cScCN[1] = four * rdyc[2] / (dyc[1] + two * dyc[2]);
            o->ac2cScCN[1] = -(eight * rdyc[1] + four * rdyc[2]) / (dyc[1] + two * dyc[2]);
            break;
        case -2:
            o->ap2cScCN[1] = rdyp[1] * rdyc[2];
            o->ac2cScCN[1] = -rdyp[1] * rdyc[2];
            o->am2cScCN[1] = zero;
            break;
        case -3:
            o->ap2cScCN[1] = rdyp[1] * rdyc[2];
            o->ac2cScCN[1] = o->ac2cScCN[1] + o->am2cScCN[1] * (two + v[0] * dyc[1]) / (two - v[0] * dyc[1]);
            o->am2cScCN[1] = zero;
            break;
        }
        switch (opt[1]) {
        case -1:
            o->am2cScCN[nyc] = four * rdyc[nyc] / (dyc[nyp] + two * dyc[nyc]);
            o->ap2cScCN[nyc] = eight * rdyc[nyp] / (dyc[nyp] + two * dyc[nyc]);
            o->ac2cScCN[nyc] = -(eight * rdyc[nyp] + four * rdyc[nyc]) / (dyc[nyp] + two * dyc[nyc]);
            break;
        case -2:
            o->am2cScCN[nyc] = rdyp[nyc] * rdyc[nyc];
            o->ac2cScCN[nyc] = -rdyp[nyc] * rdyc[nyc];
            o->ap2cScCN[nyc] = zero;
            break;
        case -3:
            o->am2cScCN[nyc] = rdyp[nyc] * rdyc[nyc];
            o->ac2cScCN[nyc] = o->ac2cScCN[nyc] + o->ap2cScCN[nyc] * (two - v[1] * dyc[nyp]) / (two + v[1] * dyc[nyp]);
            o->ap2cScCN[nyc] = zero;
            break;
        }
    }
    /* wavenumbers (src/m_Poisson.f90:40-48) */
    o->wnx = dalloc((size_t)nxc + 1);
    o->wnz = dalloc((size_t)nzc + 1);
    if (!o->wnx || !o->wnz) return PARATC_ERR_OOM;
    for (int i = 1; i <= nxc; i++) {
        double wa1 = twopi * (double)(i - 1) / (double)nxc;
        o->wnx[i] = rdx2 / 288.0 * (cos(three * wa1) - 54.0 * cos(two * wa1) + 783.0 * cos(wa1) - 730.0);
    }
    for (int k = 1; k <= nzc; k++) {
        double wa3 = twopi * (double)(k - 1) / (double)nzc;
        o->wnz[k] = rdz2 / 288.0 * (cos(three * wa3) - 54.0 * cos(two * wa3) + 783.0 * cos(wa3) - 730.0);
    }
    o->normfft = one / ((double)nxc * (double)nzc);
    return 0;
}

void orc_destroy(orc_t* o) {
    if (!o) return;
    double** arrs[] = {&o->yp, &o->yc, &o->dyp, &o->dyc, &o->rdyp, &o->rdyc, &o->yinterp,
                       &o->ap2ph, &o->ac2ph, &o->am2ph, &o->ap2c, &o->ac2c, &o->am2c,
                       &o->ap2cCN, &o->ac2cCN, &o->am2cCN, &o->ap2p, &o->ac2p, &o->am2p,
                       &o->ap2cSc, &o->ac2cSc, &o->am2cSc, &o->ap2cScCN, &o->ac2cScCN, &o->am2cScCN,
                       &o->wnx, &o->wnz, &o->ux, &o->uy, &o->uz, &o->pr, &o->sc, &o->phi,
                       &o->hx, &o->hy, &o->hz, &o->hc, &o->rhsx, &o->rhsy, &o->rhsz, &o->rhsc,
                       &o->prsrc, &o->phi_int, &o->uy_ym, &o->duy_ym, &o->uxhx, &o->uyhx, &o->uzhx,
                       &o->uxhz, &o->uyhz, &o->uzhz, &o->pln};
    for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); a++) free(*arrs[a]);
    free(o->px.w);
    free(o->pz.w);
    free(o);
}

int orc_create(const paratc_params* prm, const double* yp, orc_t** out) {
    if (!prm || !yp || !out) return PARATC_ERR_BAD_ARG;
    if (prm->nxc < 4 || prm->nyc < 4 || prm->nzc < 4 || prm->nxc % 2 || prm->nzc % 2) return PARATC_ERR_BAD_ARG;
    if (prm->flow_type == PARATC_FT_CH && prm->nyc % 2) return PARATC_ERR_BAD_ARG;
    if (prm->ischeme < 1 || prm->ischeme > 3) return PARATC_ERR_BAD_ARG;
    orc_t* o = (orc_t*)calloc(1, sizeof(orc_t));
    if (!o) return PARATC_ERR_OOM;
    o->p = *prm;
    o->nxc = prm->nxc; o->nyc = prm->nyc; o->nzc = prm->nzc; o->nyp = prm->nyc + 1;
    o->nxt = (size_t)o->nxc + 4; o->nyt = (size_t)o->nyc + 2; o->nzt = (size_t)o->nzc + 4;
    o->nh = o->nxt * o->nyt * o->nzt;
    o->ni = (size_t)o->nxc * o->nyc * o->nzc;
    int rc = metrics_init(o, yp);
    if (rc) { orc_destroy(o); return rc; }
    if (fft_plan_init(&o->px, o->nxc) || fft_plan_init(&o->pz, o->nzc)) { orc_destroy(o); return PARATC_ERR_BAD_ARG; }
    /* RK constants (src/m_Parameters.f90:159-174) */
    if (prm->ischeme == PARATC_AB2) {
        o->iadvance = 1;
        o->gamc[0] = three / two; o->gamc[1] = zero; o->gamc[2] = zero;
        o->thec[0] = -half; o->thec[1] = zero; o->thec[2] = zero;
    } else if (prm->ischeme == PARATC_RK2) {
        o->iadvance = 2;
        o->gamc[0] = half; o->gamc[1] = one; o->gamc[2] = zero;
        o->thec[0] = zero; o->thec[1] = -half; o->thec[2] = zero;
    } else {
        o->iadvance = 3;
        o->gamc[0] = eight / fifteen; o->gamc[1] = five / twelve; o->gamc[2] = three / four;
        o->thec[0] = zero; o->thec[1] = -seventeen / sixty; o->thec[2] = -five / twelve;
    }
    for (int i = 0; i < 3; i++) o->alpc[i] = o->gamc[i] + o->thec[i];
    /* fields */
    double** H[] = {&o->ux, &o->uy, &o->uz, &o->pr, &o->phi, &o->uxhx, &o->uyhx, &o->uzhx, &o->uxhz, &o->uyhz, &o->uzhz};
    for (size_t a = 0; a < sizeof(H) / sizeof(H[0]); a++) if (!(*H[a] = dalloc(o->nh))) { orc_destroy(o); return PARATC_ERR_OOM; }
    double** I[] = {&o->hx, &o->hy, &o->hz, &o->rhsx, &o->rhsy, &o->rhsz, &o->prsrc, &o->phi_int};
    for (size_t a = 0; a < sizeof(I) / sizeof(I[0]); a++) if (!(*I[a] = dalloc(o->ni))) { orc_destroy(o); return PARATC_ERR_OOM; }
    o->uy_ym = dalloc((size_t)o->nxc * o->nzc);
    o->duy_ym = dalloc((size_t)o->nxc * o->nzc);
    o->pln = dalloc((size_t)o->nzc * 4);
    if (!o->uy_ym || !o->duy_ym || !o->pln) { orc_destroy(o); return PARATC_ERR_OOM; }
    if (prm->scalar_on) {
        if (!(o->sc = dalloc(o->nh)) || !(o->hc = dalloc(o->ni)) || !(o->rhsc = dalloc(o->ni))) { orc_destroy(o); return PARATC_ERR_OOM; }
        for (size_t i = 0; i < o->nh; i++) o->sc[i] = prm->scalar_init_value;
    }
    o->sim_time = zero;
    o->dt = prm->dt_max;
    *out = o;
    return 0;
}

/* ------------------------------------------------------------------------
 * PMcoeUpdate (src/m_Parameters.f90:215-230)
 * ---------------------------------------------------------------------- */
static void pm_update(orc_t* o, int ns) {
    const double dt = o->dt;
    o->pmGamma = o->gamc[ns - 1] * dt;
    o->pmTheta = o->thec[ns - 1] * dt;
    o->pmAlpha = o->alpc[ns - 1] * dt;
    o->pmBeta = half * o->alpc[ns - 1] * o->p.xnu * dt;
    o->pmBetaSc = half * o->alpc[ns - 1] * o->p.sdiff * dt;
    o->sim_time = o->sim_time + dt * o->alpc[ns - 1];
    o->pmAlphaC = o->alpc[ns - 1];
    if (ns == 1) o->pr_grad_aver = zero;
}

/* Update_uy_ym (src/m_FlowCase.f90:112-122): no wall transpiration */
static void update_uy_ym(orc_t* o) {
    size_t n = (size_t)o->nxc * o->nzc;
    for (size_t i = 0; i < n; i++) {
        o->duy_ym[i] = o->uy_ym[i];
        o->uy_ym[i] = zero;
        o->duy_ym[i] = o->uy_ym[i] - o->duy_ym[i];
    }
}

/* ------------------------------------------------------------------------
 * clcRhsXYZ (src/m_TScheme.f90:113-360)
 * ---------------------------------------------------------------------- */
static double sum_planes(const double* pl, int nz) {
    double s = 0.0;
    for (int k = 0; k < nz; k++) s += pl[k];
    return s;
}

static void clc_rhs(orc_t* o) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc, nyp = o->nyp;
    const double *ux = o->ux, *uy = o->uy, *uz = o->uz, *pr = o->pr;
    double *uxhx = o->uxhx, *uyhx = o->uyhx, *uzhx = o->uzhx, *uxhz = o->uxhz, *uyhz = o->uyhz, *uzhz = o->uzhz;
    const double I1 = o->IC[0], I2 = o->IC[1], I3 = o->IC[2], I4 = o->IC[3];
    const double *dxC = o->dxC, *dzC = o->dzC, *dxxC = o->dxxC, *dzzC = o->dzzC;
    const double uCRF = o->p.ucrf, xnu = o->p.xnu;
    const double pmGamma = o->pmGamma, pmTheta = o->pmTheta, pmAlpha = o->pmAlpha, pmBeta = o->pmBeta;

    /* Update_VelInterp_uvw (:143-161) */
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
        for (int jc = 1; jc <= nyc; jc++)
            for (int ic = 1; ic <= nxc; ic++) {
                int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
                uxhx[HX(o, ic, jc, kc)] = I1 * ux[HX(o, im, jc, kc)] + I2 * ux[HX(o, ic, jc, kc)] + I3 * ux[HX(o, ip, jc, kc)] + I4 * ux[HX(o, iu, jc, kc)];
                uyhx[HX(o, ic, jc, kc)] = I1 * uy[HX(o, is, jc, kc)] + I2 * uy[HX(o, im, jc, kc)] + I3 * uy[HX(o, ic, jc, kc)] + I4 * uy[HX(o, ip, jc, kc)];
                uzhx[HX(o, ic, jc, kc)] = I1 * uz[HX(o, is, jc, kc)] + I2 * uz[HX(o, im, jc, kc)] + I3 * uz[HX(o, ic, jc, kc)] + I4 * uz[HX(o, ip, jc, kc)];
                uxhz[HX(o, ic, jc, kc)] = I1 * ux[HX(o, ic, jc, ks)] + I2 * ux[HX(o, ic, jc, km)] + I3 * ux[HX(o, ic, jc, kc)] + I4 * ux[HX(o, ic, jc, kp)];
                uyhz[HX(o, ic, jc, kc)] = I1 * uy[HX(o, ic, jc, ks)] + I2 * uy[HX(o, ic, jc, km)] + I3 * uy[HX(o, ic, jc, kc)] + I4 * uy[HX(o, ic, jc, kp)];
                uzhz[HX(o, ic, jc, kc)] = I1 * uz[HX(o, ic, jc, km)] + I2 * uz[HX(o, ic, jc, kc)] + I3 * uz[HX(o, ic, jc, kp)] + I4 * uz[HX(o, ic, jc, ku)];
            }
        for (int ic = 1; ic <= nxc; ic++) { uyhx[HX(o, ic, nyp, kc)] = zero; uyhz[HX(o, ic, nyp, kc)] = zero; }
    }
    upd_halo(o, uxhx, 2, 1, 0, 0);
    upd_halo(o, uyhx, 1, 2, 0, 0);
    upd_halo(o, uzhx, 1, 2, 1, 2);
    upd_halo(o, uxhz, 1, 2, 1, 2);
    upd_halo(o, uyhz, 0, 0, 1, 2);
    upd_halo(o, uzhz, 0, 0, 2, 1);

    /* RhsX (:169-204) */
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
        double s3 = zero;
        for (int jc = 1; jc <= nyc; jc++) {
            int jm = jc - 1, jp = jc + 1;
            double sucaj = o->rdyp[jc];
            double IY1 = o->yinterp[jc], IY2 = one - IY1, IY3 = o->yinterp[jp], IY4 = one - IY3;
            for (int ic = 1; ic <= nxc; ic++) {
                int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
                double uxhyc = IY1 * ux[HX(o, ic, jm, kc)] + IY2 * ux[HX(o, ic, jc, kc)];
                double uxhyp = IY3 * ux[HX(o, ic, jc, kc)] + IY4 * ux[HX(o, ic, jp, kc)];
                double h11 = dxC[0] * uxhx[HX(o, is, jc, kc)] * (uxhx[HX(o, is, jc, kc)] + uCRF) + dxC[1] * uxhx[HX(o, im, jc, kc)] * (uxhx[HX(o, im, jc, kc)] + uCRF)
                           + dxC[2] * uxhx[HX(o, ic, jc, kc)] * (uxhx[HX(o, ic, jc, kc)] + uCRF) + dxC[3] * uxhx[HX(o, ip, jc, kc)] * (uxhx[HX(o, ip, jc, kc)] + uCRF);
                double h12 = (uyhx[HX(o, ic, jp, kc)] * uxhyp - uyhx[HX(o, ic, jc, kc)] * uxhyc) * sucaj;
                double h13 = dzC[0] * uxhz[HX(o, ic, jc, km)] * uzhx[HX(o, ic, jc, km)] + dzC[1] * uxhz[HX(o, ic, jc, kc)] * uzhx[HX(o, ic, jc, kc)]
                           + dzC[2] * uxhz[HX(o, ic, jc, kp)] * uzhx[HX(o, ic, jc, kp)] + dzC[3] * uxhz[HX(o, ic, jc, ku)] * uzhx[HX(o, ic, jc, ku)];
                double d11 = dxxC[0] * ux[HX(o, is, jc, kc)] + dxxC[1] * ux[HX(o, im, jc, kc)] + dxxC[2] * ux[HX(o, ic, jc, kc)] + dxxC[3] * ux[HX(o, ip, jc, kc)] + dxxC[4] * ux[HX(o, iu, jc, kc)];
                double d22 = o->ap2c[jc] * ux[HX(o, ic, jp, kc)] + o->ac2c[jc] * ux[HX(o, ic, jc, kc)] + o->am2c[jc] * ux[HX(o, ic, jm, kc)];
                double d33 = dzzC[0] * ux[HX(o, ic, jc, ks)] + dzzC[1] * ux[HX(o, ic, jc, km)] + dzzC[2] * ux[HX(o, ic, jc, kc)] + dzzC[3] * ux[HX(o, ic, jc, kp)] + dzzC[4] * ux[HX(o, ic, jc, ku)];
                double dcq13 = d11 + d33;
                if (o->p.scalar_on) s3 = s3 + ux[HX(o, ic, jc, kc)] * o->dyp[jc];
                else                s3 = s3 + (dcq13 + d22) * o->dyp[jc];
                double conv = -h11 - h12 - h13 + xnu * dcq13 + o->p.gravity[0];
                double gradp = dxC[0] * pr[HX(o, is, jc, kc)] + dxC[1] * pr[HX(o, im, jc, kc)] + dxC[2] * pr[HX(o, ic, jc, kc)] + dxC[3] * pr[HX(o, ip, jc, kc)];
                size_t q = IX(o, ic, jc, kc);
                o->rhsx[q] = pmGamma * conv + pmTheta * o->hx[q] - pmAlpha * gradp + two * pmBeta * d22;
                o->hx[q] = conv;
            }
        }
        o->pln[kc - 1] = s3;
    }

    /* RhsY (:206-236) */
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
        for (int jc = 1; jc <= nyc; jc++) {
            int jm = jc - 1, jp = jc + 1;
            double sucac = o->rdyc[jc], qsucac = quarter * sucac;
            double IY1 = o->yinterp[jc], IY2 = one - IY1;
            for (int ic = 1; ic <= nxc; ic++) {
                int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
                double uxhym = IY1 * ux[HX(o, im, jm, kc)] + IY2 * ux[HX(o, im, jc, kc)] + uCRF, uzhym = IY1 * uz[HX(o, ic, jm, km)] + IY2 * uz[HX(o, ic, jc, km)];
                double uxhyc = IY1 * ux[HX(o, ic, jm, kc)] + IY2 * ux[HX(o, ic, jc, kc)] + uCRF, uzhyc = IY1 * uz[HX(o, ic, jm, kc)] + IY2 * uz[HX(o, ic, jc, kc)];
                double uxhyp = IY1 * ux[HX(o, ip, jm, kc)] + IY2 * ux[HX(o, ip, jc, kc)] + uCRF, uzhyp = IY1 * uz[HX(o, ic, jm, kp)] + IY2 * uz[HX(o, ic, jc, kp)];
                double uxhyu = IY1 * ux[HX(o, iu, jm, kc)] + IY2 * ux[HX(o, iu, jc, kc)] + uCRF, uzhyu = IY1 * uz[HX(o, ic, jm, ku)] + IY2 * uz[HX(o, ic, jc, ku)];
                double h21 = dxC[0] * uyhx[HX(o, im, jc, kc)] * uxhym + dxC[1] * uyhx[HX(o, ic, jc, kc)] * uxhyc + dxC[2] * uyhx[HX(o, ip, jc, kc)] * uxhyp + dxC[3] * uyhx[HX(o, iu, jc, kc)] * uxhyu;
                double vp = uy[HX(o, ic, jp, kc)], vc = uy[HX(o, ic, jc, kc)], vm = uy[HX(o, ic, jm, kc)];
                double h22 = ((vp + vc) * (vp + vc) - (vc + vm) * (vc + vm)) * qsucac;
                double h23 = dzC[0] * uyhz[HX(o, ic, jc, km)] * uzhym + dzC[1] * uyhz[HX(o, ic, jc, kc)] * uzhyc + dzC[2] * uyhz[HX(o, ic, jc, kp)] * uzhyp + dzC[3] * uyhz[HX(o, ic, jc, ku)] * uzhyu;
                double d11 = dxxC[0] * uy[HX(o, is, jc, kc)] + dxxC[1] * uy[HX(o, im, jc, kc)] + dxxC[2] * vc + dxxC[3] * uy[HX(o, ip, jc, kc)] + dxxC[4] * uy[HX(o, iu, jc, kc)];
                double d22 = o->ap2p[jc] * vp + o->ac2p[jc] * vc + o->am2p[jc] * vm;
                double d33 = dzzC[0] * uy[HX(o, ic, jc, ks)] + dzzC[1] * uy[HX(o, ic, jc, km)] + dzzC[2] * vc + dzzC[3] * uy[HX(o, ic, jc, kp)] + dzzC[4] * uy[HX(o, ic, jc, ku)];
                double dcq13 = d11 + d33;
                double conv = -h21 - h22 - h23 + xnu * dcq13 + o->p.gravity[1];
                double gradp = (pr[HX(o, ic, jc, kc)] - pr[HX(o, ic, jm, kc)]) * sucac;
                size_t q = IX(o, ic, jc, kc);
                o->rhsy[q] = pmGamma * conv + pmTheta * o->hy[q] - pmAlpha * gradp + two * pmBeta * d22;
                o->hy[q] = conv;
            }
        }
    }

    /* RhsZ (:238-267) */
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
        for (int jc = 1; jc <= nyc; jc++) {
            int jm = jc - 1, jp = jc + 1;
            double sucaj = o->rdyp[jc];
            double IY1 = o->yinterp[jc], IY2 = one - IY1, IY3 = o->yinterp[jp], IY4 = one - IY3;
            for (int ic = 1; ic <= nxc; ic++) {
                int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
                double uzhyc = IY1 * uz[HX(o, ic, jm, kc)] + IY2 * uz[HX(o, ic, jc, kc)];
                double uzhyp = IY3 * uz[HX(o, ic, jc, kc)] + IY4 * uz[HX(o, ic, jp, kc)];
                double h31 = dxC[0] * uzhx[HX(o, im, jc, kc)] * (uxhz[HX(o, im, jc, kc)] + uCRF) + dxC[1] * uzhx[HX(o, ic, jc, kc)] * (uxhz[HX(o, ic, jc, kc)] + uCRF)
                           + dxC[2] * uzhx[HX(o, ip, jc, kc)] * (uxhz[HX(o, ip, jc, kc)] + uCRF) + dxC[3] * uzhx[HX(o, iu, jc, kc)] * (uxhz[HX(o, iu, jc, kc)] + uCRF);
                double h32 = (uyhz[HX(o, ic, jp, kc)] * uzhyp - uyhz[HX(o, ic, jc, kc)] * uzhyc) * sucaj;
                double h33 = dzC[0] * uzhz[HX(o, ic, jc, ks)] * uzhz[HX(o, ic, jc, ks)] + dzC[1] * uzhz[HX(o, ic, jc, km)] * uzhz[HX(o, ic, jc, km)]
                           + dzC[2] * uzhz[HX(o, ic, jc, kc)] * uzhz[HX(o, ic, jc, kc)] + dzC[3] * uzhz[HX(o, ic, jc, kp)] * uzhz[HX(o, ic, jc, kp)];
                double d11 = dxxC[0] * uz[HX(o, is, jc, kc)] + dxxC[1] * uz[HX(o, im, jc, kc)] + dxxC[2] * uz[HX(o, ic, jc, kc)] + dxxC[3] * uz[HX(o, ip, jc, kc)] + dxxC[4] * uz[HX(o, iu, jc, kc)];
                double d22 = o->ap2c[jc] * uz[HX(o, ic, jp, kc)] + o->ac2c[jc] * uz[HX(o, ic, jc, kc)] + o->am2c[jc] * uz[HX(o, ic, jm, kc)];
                double d33 = dzzC[0] * uz[HX(o, ic, jc, ks)] + dzzC[1] * uz[HX(o, ic, jc, km)] + dzzC[2] * uz[HX(o, ic, jc, kc)] + dzzC[3] * uz[HX(o, ic, jc, kp)] + dzzC[4] * uz[HX(o, ic, jc, ku)];
                double dcq13 = d11 + d33;
                double conv = -h31 - h32 - h33 + xnu * dcq13 + o->p.gravity[2];
                double gradp = dzC[0] * pr[HX(o, ic, jc, ks)] + dzC[1] * pr[HX(o, ic, jc, km)] + dzC[2] * pr[HX(o, ic, jc, kc)] + dzC[3] * pr[HX(o, ic, jc, kp)];
                size_t q = IX(o, ic, jc, kc);
                o->rhsz[q] = pmGamma * conv + pmTheta * o->hz[q] - pmAlpha * gradp + two * pmBeta * d22;
                o->hz[q] = conv;
            }
        }
    }

    /* mean pressure gradient / flow-rate constraint (:269-300) */
    if (o->p.is_ux_const) {
        double s3tot1 = sum_planes(o->pln, nzc), dpmdxns, dp1ns;
        if (o->p.scalar_on) {
            s3tot1 = s3tot1 / (double)(nxc * nzc) / o->p.yly;
            dpmdxns = o->p.ubulk - uCRF - s3tot1;
            dp1ns = o->pmAlphaC * dpmdxns;
            for (size_t q = 0; q < o->ni; q++) o->rhsx[q] = o->rhsx[q] + dp1ns;
            o->pr_grad_aver = o->pr_grad_aver + dpmdxns * o->pmAlphaC / o->dt;
        } else {
            dpmdxns = xnu * s3tot1 / (double)(nxc * nzc) / o->p.yly;
            dp1ns = pmAlpha * dpmdxns;
            for (size_t q = 0; q < o->ni; q++) o->rhsx[q] = o->rhsx[q] - dp1ns;
            o->pr_grad_aver = o->pr_grad_aver + dpmdxns * o->pmAlphaC;
        }
    }

    if (!o->p.scalar_on) return;
    /* scalar transport (:302-357); shx/shz reuse uyhx/uyhz as in the reference */
    const double* sc = o->sc;
    double *shx = uyhx, *shz = uyhz;
    const double* GE = o->p.gravity_eff_vec;
    const double* FV = o->p.falling_vel_vec;
    const double SD = o->p.sdiff, pmBetaSc = o->pmBetaSc;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int ks = kc - 2, km = kc - 1, kp = kc + 1;
        for (int jc = 1; jc <= nyc; jc++)
            for (int ic = 1; ic <= nxc; ic++) {
                int is = ic - 2, im = ic - 1, ip = ic + 1;
                shx[HX(o, ic, jc, kc)] = I1 * sc[HX(o, is, jc, kc)] + I2 * sc[HX(o, im, jc, kc)] + I3 * sc[HX(o, ic, jc, kc)] + I4 * sc[HX(o, ip, jc, kc)];
                shz[HX(o, ic, jc, kc)] = I1 * sc[HX(o, ic, jc, ks)] + I2 * sc[HX(o, ic, jc, km)] + I3 * sc[HX(o, ic, jc, kc)] + I4 * sc[HX(o, ic, jc, kp)];
            }
    }
    upd_halo(o, shx, 1, 2, 0, 0);
    upd_halo(o, shz, 0, 0, 1, 2);
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
        for (int jc = 1; jc <= nyc; jc++) {
            int jm = jc - 1, jp = jc + 1;
            double sucaj = o->rdyp[jc];
            double IY1 = o->yinterp[jc], IY2 = one - IY1, IY3 = o->yinterp[jp], IY4 = one - IY3;
            for (int ic = 1; ic <= nxc; ic++) {
                int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
                double shyc = IY1 * sc[HX(o, ic, jm, kc)] + IY2 * sc[HX(o, ic, jc, kc)];
                double shyp = IY3 * sc[HX(o, ic, jc, kc)] + IY4 * sc[HX(o, ic, jp, kc)];
                double c1 = GE[0] * shx[HX(o, ic, jc, kc)], c2 = GE[1] * shyc, c3 = GE[2] * shz[HX(o, ic, jc, kc)];
                size_t q = IX(o, ic, jc, kc);
                o->rhsx[q] = o->rhsx[q] + pmGamma * c1;
                o->rhsy[q] = o->rhsy[q] + pmGamma * c2;
                o->rhsz[q] = o->rhsz[q] + pmGamma * c3;
                o->hx[q] = o->hx[q] + c1;
                o->hy[q] = o->hy[q] + c2;
                o->hz[q] = o->hz[q] + c3;
                double hc1 = dxC[0] * (ux[HX(o, im, jc, kc)] + FV[0]) * shx[HX(o, im, jc, kc)] + dxC[1] * (ux[HX(o, ic, jc, kc)] + FV[0]) * shx[HX(o, ic, jc, kc)]
                           + dxC[2] * (ux[HX(o, ip, jc, kc)] + FV[0]) * shx[HX(o, ip, jc, kc)] + dxC[3] * (ux[HX(o, iu, jc, kc)] + FV[0]) * shx[HX(o, iu, jc, kc)];
                double hc2 = ((uy[HX(o, ic, jp, kc)] + FV[1]) * shyp - (uy[HX(o, ic, jc, kc)] + FV[1]) * shyc) * sucaj;
                double hc3 = dzC[0] * (uz[HX(o, ic, jc, km)] + FV[2]) * shz[HX(o, ic, jc, km)] + dzC[1] * (uz[HX(o, ic, jc, kc)] + FV[2]) * shz[HX(o, ic, jc, kc)]
                           + dzC[2] * (uz[HX(o, ic, jc, kp)] + FV[2]) * shz[HX(o, ic, jc, kp)] + dzC[3] * (uz[HX(o, ic, jc, ku)] + FV[2]) * shz[HX(o, ic, jc, ku)];
                double d11 = dxxC[0] * sc[HX(o, is, jc, kc)] + dxxC[1] * sc[HX(o, im, jc, kc)] + dxxC[2] * sc[HX(o, ic, jc, kc)] + dxxC[3] * sc[HX(o, ip, jc, kc)] + dxxC[4] * sc[HX(o, iu, jc, kc)];
                double d22 = o->ap2cSc[jc] * sc[HX(o, ic, jp, kc)] + o->ac2cSc[jc] * sc[HX(o, ic, jc, kc)] + o->am2cSc[jc] * sc[HX(o, ic, jm, kc)];
                double d33 = dzzC[0] * sc[HX(o, ic, jc, ks)] + dzzC[1] * sc[HX(o, ic, jc, km)] + dzzC[2] * sc[HX(o, ic, jc, kc)] + dzzC[3] * sc[HX(o, ic, jc, kp)] + dzzC[4] * sc[HX(o, ic, jc, ku)];
                double convc = -hc1 - hc2 - hc3 + SD * (d11 + d33);
                o->rhsc[q] = pmGamma * convc + pmTheta * o->hc[q] + two * pmBetaSc * d22;
                o->hc[q] = convc;
            }
        }
    }
}

/* ------------------------------------------------------------------------
 * InverseTridiagonal (src/m_Tools.f90:224-251) for one column
 * ---------------------------------------------------------------------- */
static void thomas_col(int n, const double* aj, const double* bj, const double* cj, double* f,
                       size_t fs, double* arr) {
    /* aj/bj/cj/arr 1-based (index 1..n); f strided */
    double vecm = bj[1];
    f[0] = f[0] / vecm;
    for (int j = 2; j <= n; j++) {
        arr[j] = cj[j - 1] / vecm;
        vecm = bj[j] - aj[j] * arr[j];
        f[(size_t)(j - 1) * fs] = (f[(size_t)(j - 1) * fs] - aj[j] * f[(size_t)(j - 2) * fs]) / vecm;
    }
    for (int j = n - 1; j >= 1; j--) f[(size_t)(j - 1) * fs] = f[(size_t)(j - 1) * fs] - arr[j + 1] * f[(size_t)j * fs];
}

/* clcU1Hat / clcU3Hat / clcScalar (src/m_TScheme.f90:365-394,442-471,477-506):
 * u(ic,jc,kc) += (I - beta*L_CN)^-1 Rhs along y */
static void helm_cn(orc_t* o, double* u, double* rhs, double beta, const double* ap, const double* ac,
                    const double* am) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    double *tp = dalloc((size_t)nyc + 2), *tc = dalloc((size_t)nyc + 2), *tm = dalloc((size_t)nyc + 2);
    for (int jc = 1; jc <= nyc; jc++) {
        tp[jc] = -(beta * ap[jc]);
        tc[jc] = -(beta * ac[jc]) + one;
        tm[jc] = -(beta * am[jc]);
    }
#pragma omp parallel
    {
        double* arr = dalloc((size_t)nyc + 2);
#pragma omp for schedule(static)
        for (int kc = 1; kc <= nzc; kc++)
            for (int ic = 1; ic <= nxc; ic++) {
                double* f = &rhs[IX(o, ic, 1, kc)];
                thomas_col(nyc, tm, tc, tp, f, (size_t)nxc, arr);
                for (int jc = 1; jc <= nyc; jc++) u[HX(o, ic, jc, kc)] = u[HX(o, ic, jc, kc)] + f[(size_t)(jc - 1) * nxc];
            }
        free(arr);
    }
    free(tp); free(tc); free(tm);
}

/* clcU2Hat (src/m_TScheme.f90:399-437) */
static void helm_v(orc_t* o) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    double *tp = dalloc((size_t)nyc + 2), *tc = dalloc((size_t)nyc + 2), *tm = dalloc((size_t)nyc + 2);
    tp[1] = zero; tc[1] = one; tm[1] = zero;
    for (int jc = 2; jc <= nyc; jc++) {
        tp[jc] = -(o->pmBeta * o->ap2p[jc]);
        tc[jc] = -(o->pmBeta * o->ac2p[jc]) + one;
        tm[jc] = -(o->pmBeta * o->am2p[jc]);
    }
#pragma omp parallel
    {
        double* arr = dalloc((size_t)nyc + 2);
#pragma omp for schedule(static)
        for (int kc = 1; kc <= nzc; kc++)
            for (int ic = 1; ic <= nxc; ic++) {
                double* f = &o->rhsy[IX(o, ic, 1, kc)];
                f[0] = o->duy_ym[(size_t)(kc - 1) * nxc + (ic - 1)];
                thomas_col(nyc, tm, tc, tp, f, (size_t)nxc, arr);
                for (int jc = 1; jc <= nyc; jc++) o->uy[HX(o, ic, jc, kc)] = o->uy[HX(o, ic, jc, kc)] + f[(size_t)(jc - 1) * nxc];
            }
        free(arr);
    }
    free(tp); free(tc); free(tm);
}

/* ------------------------------------------------------------------------
 * clcPrSrc (src/m_TScheme.f90:48-77); scale = 1/pmAlpha (sudtal)
 * ---------------------------------------------------------------------- */
static double clc_prsrc(orc_t* o, double* src, double sudtal) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    const double *ux = o->ux, *uy = o->uy, *uz = o->uz, *dxC = o->dxC, *dzC = o->dzC;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int km = kc - 1, kp = kc + 1, ku = kc + 2;
        double dm = zero;
        for (int jc = 1; jc <= nyc; jc++) {
            int jp = jc + 1;
            double sucaj = o->rdyp[jc];
            for (int ic = 1; ic <= nxc; ic++) {
                int im = ic - 1, ip = ic + 1, iu = ic + 2;
                double dudx = dxC[0] * ux[HX(o, im, jc, kc)] + dxC[1] * ux[HX(o, ic, jc, kc)] + dxC[2] * ux[HX(o, ip, jc, kc)] + dxC[3] * ux[HX(o, iu, jc, kc)];
                double dvdy = (uy[HX(o, ic, jp, kc)] - uy[HX(o, ic, jc, kc)]) * sucaj;
                double dwdz = dzC[0] * uz[HX(o, ic, jc, km)] + dzC[1] * uz[HX(o, ic, jc, kc)] + dzC[2] * uz[HX(o, ic, jc, kp)] + dzC[3] * uz[HX(o, ic, jc, ku)];
                double rdiv = dudx + dvdy + dwdz;
                if (fabs(rdiv) > dm) dm = fabs(rdiv);
                if (src) src[IX(o, ic, jc, kc)] = sudtal * rdiv;
            }
        }
        o->pln[kc - 1] = dm;
    }
    double m = zero;
    for (int k = 0; k < nzc; k++) if (o->pln[k] > m) m = o->pln[k];
    return m;
}

/* ------------------------------------------------------------------------
 * clcPPE_x1 (src/m_Poisson.f90:352-452), single rank: the transposes are
 * identities in value, the x transform runs over contiguous rows and the z
 * transform over rows strided by nxc*nyc.
 * ---------------------------------------------------------------------- */
static void clc_ppe(orc_t* o, const double* src, double* phi_int) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    const size_t ni = o->ni, pl = (size_t)nxc * nyc;
    double* a = phi_int;
    if (a != src) memcpy(a, src, sizeof(double) * ni);
    const int nrows = nyc * nzc;
#pragma omp parallel
    {
        int nmax = nxc > nzc ? nxc : nzc;
        cplx* zb = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)nmax);
        double* rb = (double*)malloc(sizeof(double) * 4 * (size_t)nmax);
        /* forward x (R2HC) */
#pragma omp for schedule(static)
        for (int q = 0; q < nrows / 2; q++) {
            double* r0 = a + (size_t)(2 * q) * nxc;
            double* r1 = r0 + nxc;
            r2hc_pair(&o->px, r0, r1, rb, rb + nxc, zb, zb + nxc);
            memcpy(r0, rb, sizeof(double) * nxc);
            memcpy(r1, rb + nxc, sizeof(double) * nxc);
        }
        /* forward z (R2HC), pairs of x slots */
#pragma omp for schedule(static) collapse(2)
        for (int jc = 0; jc < nyc; jc++)
            for (int ip = 0; ip < nxc / 2; ip++) {
                double* b0 = a + (size_t)jc * nxc + 2 * ip;
                for (int k = 0; k < nzc; k++) { rb[k] = b0[(size_t)k * pl]; rb[nzc + k] = b0[(size_t)k * pl + 1]; }
                r2hc_pair(&o->pz, rb, rb + nzc, rb + 2 * nzc, rb + 3 * nzc, zb, zb + nzc);
                for (int k = 0; k < nzc; k++) { b0[(size_t)k * pl] = rb[2 * nzc + k]; b0[(size_t)k * pl + 1] = rb[3 * nzc + k]; }
            }
        free(zb); free(rb);
    }
    /* y: (am2ph, ac2ph + lx(i) + lz(k), ap2ph) per (i,k); DC row 1 pinned */
#pragma omp parallel
    {
        double* tc = dalloc((size_t)nyc + 2);
        double* tp = dalloc((size_t)nyc + 2);
        double* arr = dalloc((size_t)nyc + 2);
#pragma omp for schedule(static)
        for (int kc = 1; kc <= nzc; kc++)
            for (int ic = 1; ic <= nxc; ic++) {
                for (int jc = 1; jc <= nyc; jc++) { tc[jc] = o->ac2ph[jc] + o->wnx[ic] + o->wnz[kc]; tp[jc] = o->ap2ph[jc]; }
                double* f = &a[IX(o, ic, 1, kc)];
                if (kc == 1 && ic == 1) { tp[1] = zero; tc[1] = one; f[0] = zero; }
                /* tridmj(1,1) = 0 is never read by the Thomas sweep */
                thomas_col(nyc, o->am2ph, tc, tp, f, (size_t)nxc, arr);
            }
        free(tc); free(tp); free(arr);
    }
#pragma omp parallel
    {
        int nmax = nxc > nzc ? nxc : nzc;
        cplx* zb = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)nmax);
        double* rb = (double*)malloc(sizeof(double) * 4 * (size_t)nmax);
        /* backward z (HC2R) */
#pragma omp for schedule(static) collapse(2)
        for (int jc = 0; jc < nyc; jc++)
            for (int ip = 0; ip < nxc / 2; ip++) {
                double* b0 = a + (size_t)jc * nxc + 2 * ip;
                for (int k = 0; k < nzc; k++) { rb[k] = b0[(size_t)k * pl]; rb[nzc + k] = b0[(size_t)k * pl + 1]; }
                hc2r_pair(&o->pz, rb, rb + nzc, rb + 2 * nzc, rb + 3 * nzc, zb, zb + nzc);
                for (int k = 0; k < nzc; k++) { b0[(size_t)k * pl] = rb[2 * nzc + k]; b0[(size_t)k * pl + 1] = rb[3 * nzc + k]; }
            }
        /* backward x (HC2R) and the normfft scaling */
#pragma omp for schedule(static)
        for (int q = 0; q < nrows / 2; q++) {
            double* r0 = a + (size_t)(2 * q) * nxc;
            double* r1 = r0 + nxc;
            hc2r_pair(&o->px, r0, r1, rb, rb + nxc, zb, zb + nxc);
            for (int i = 0; i < nxc; i++) { r0[i] = rb[i] * o->normfft; r1[i] = rb[nxc + i] * o->normfft; }
        }
        free(zb); free(rb);
    }
}

static void phi_to_halo(orc_t* o) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++)
        for (int jc = 1; jc <= nyc; jc++)
            memcpy(&o->phi[HX(o, 1, jc, kc)], &o->phi_int[IX(o, 1, jc, kc)], sizeof(double) * nxc);
    bc_pr(o, o->phi);
}

/* FluidVelUpdate (src/m_TScheme.f90:82-107) */
static void fluid_vel_update(orc_t* o, double alpha) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    const double *ph = o->phi, *dxC = o->dxC, *dzC = o->dzC;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int ks = kc - 2, km = kc - 1, kp = kc + 1;
        for (int jc = 1; jc <= nyc; jc++) {
            int jm = jc - 1;
            double sucac = o->rdyc[jc];
            for (int ic = 1; ic <= nxc; ic++) {
                int is = ic - 2, im = ic - 1, ip = ic + 1;
                double dpdx = dxC[0] * ph[HX(o, is, jc, kc)] + dxC[1] * ph[HX(o, im, jc, kc)] + dxC[2] * ph[HX(o, ic, jc, kc)] + dxC[3] * ph[HX(o, ip, jc, kc)];
                double dpdy = (ph[HX(o, ic, jc, kc)] - ph[HX(o, ic, jm, kc)]) * sucac;
                double dpdz = dzC[0] * ph[HX(o, ic, jc, ks)] + dzC[1] * ph[HX(o, ic, jc, km)] + dzC[2] * ph[HX(o, ic, jc, kc)] + dzC[3] * ph[HX(o, ic, jc, kp)];
                o->ux[HX(o, ic, jc, kc)] = o->ux[HX(o, ic, jc, kc)] - alpha * dpdx;
                o->uy[HX(o, ic, jc, kc)] = o->uy[HX(o, ic, jc, kc)] - alpha * dpdy;
                o->uz[HX(o, ic, jc, kc)] = o->uz[HX(o, ic, jc, kc)] - alpha * dpdz;
            }
        }
    }
}

/* PressureUpdate (src/m_TScheme.f90:512-532) */
static void pressure_update(orc_t* o) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    const double* ph = o->phi;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++)
        for (int jc = 1; jc <= nyc; jc++) {
            int jp = jc + 1, jm = jc - 1;
            double bp = -(o->pmBeta * o->ap2ph[jc]);
            double bc = -(o->pmBeta * o->ac2ph[jc]) + one;
            double bm = -(o->pmBeta * o->am2ph[jc]);
            for (int ic = 1; ic <= nxc; ic++)
                o->pr[HX(o, ic, jc, kc)] = o->pr[HX(o, ic, jc, kc)] + bp * ph[HX(o, ic, jp, kc)] + bc * ph[HX(o, ic, jc, kc)] + bm * ph[HX(o, ic, jm, kc)];
        }
}

/* ------------------------------------------------------------------------
 * m_Tools reductions (src/m_Tools.f90:24-110,256-301)
 * ---------------------------------------------------------------------- */
static double calc_max_cfl(orc_t* o) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        int kp = kc + 1;
        double m = zero;
        for (int jc = 1; jc <= nyc; jc++) {
            int jp = jc + 1;
            for (int ic = 1; ic <= nxc; ic++) {
                int ip = ic + 1;
                double vcf = fabs(o->ux[HX(o, ic, jc, kc)] + o->ux[HX(o, ip, jc, kc)]) * o->rdx + fabs(o->uy[HX(o, ic, jc, kc)] + o->uy[HX(o, ic, jp, kc)]) * o->rdyp[jc]
                           + fabs(o->uz[HX(o, ic, jc, kc)] + o->uz[HX(o, ic, jc, kp)]) * o->rdz;
                if (vcf > m) m = vcf;
            }
        }
        o->pln[kc - 1] = m;
    }
    double m = zero;
    for (int k = 0; k < nzc; k++) if (o->pln[k] > m) m = o->pln[k];
    return m * half;
}

static void calc_vmax(orc_t* o, double* v) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        double a = zero, b = zero, c = zero;
        for (int jc = 1; jc <= nyc; jc++)
            for (int ic = 1; ic <= nxc; ic++) {
                double x = fabs(o->ux[HX(o, ic, jc, kc)]), y = fabs(o->uy[HX(o, ic, jc, kc)]), z = fabs(o->uz[HX(o, ic, jc, kc)]);
                if (x > a) a = x;
                if (y > b) b = y;
                if (z > c) c = z;
            }
        o->pln[4 * (kc - 1)] = a; o->pln[4 * (kc - 1) + 1] = b; o->pln[4 * (kc - 1) + 2] = c;
    }
    v[0] = v[1] = v[2] = zero;
    for (int k = 0; k < nzc; k++)
        for (int d = 0; d < 3; d++) if (o->pln[4 * k + d] > v[d]) v[d] = o->pln[4 * k + d];
}

static void calc_means(orc_t* o, double* r) {
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= nzc; kc++) {
        double a = zero, b = zero, c = zero;
        for (int jc = 1; jc <= nyc; jc++) {
            double dy = o->dyp[jc];
            for (int ic = 1; ic <= nxc; ic++) {
                a = a + o->ux[HX(o, ic, jc, kc)] * dy;
                if (o->p.scalar_on) {
                    double s = o->sc[HX(o, ic, jc, kc)];
                    b = b + dy * s;
                    c = c + dy * s * s;
                }
            }
        }
        o->pln[4 * (kc - 1)] = a; o->pln[4 * (kc - 1) + 1] = b; o->pln[4 * (kc - 1) + 2] = c;
    }
    r[0] = r[1] = r[2] = zero;
    for (int k = 0; k < nzc; k++)
        for (int d = 0; d < 3; d++) r[d] += o->pln[4 * k + d];
    for (int d = 0; d < 3; d++) r[d] = r[d] / (double)(nxc * nzc) / o->p.yly;
}

int orc_diagnostics(orc_t* o, paratc_diag* d) {
    if (!o || !d) return PARATC_ERR_BAD_ARG;
    double m[3];
    d->divmax = clc_prsrc(o, NULL, one);
    calc_vmax(o, d->vmax);
    calc_means(o, m);
    d->ux_mean = m[0]; d->sc_mean = m[1]; d->sc2_mean = m[2];
    d->cfl = calc_max_cfl(o) * o->dt;
    d->dt = o->dt; d->sim_time = o->sim_time; d->pr_grad_aver = o->pr_grad_aver;
    return 0;
}

/* ------------------------------------------------------------------------
 * clcStat (src/m_FlowCase.f90:257-428): one call's contribution
 * SumVec(k)*inxz to SumStat(k, jc), jc = 1..nyp, k fastest in out[]; nst = 35
 * (40 with the scalar).  Loop order and expressions as the reference.
 * ---------------------------------------------------------------------- */
int orc_stats(orc_t* o, double* out) {
    if (!o || !out) return PARATC_ERR_BAD_ARG;
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc, nyp = o->nyp;
    const int nst = o->p.scalar_on ? 40 : 35;
    const double *ux = o->ux, *uy = o->uy, *uz = o->uz, *pr = o->pr, *sc = o->sc;
    const double *dxC = o->dxC, *dzC = o->dzC, *dxxC = o->dxxC, *dzzC = o->dzzC, *IC = o->IC;
    const double uCRF = o->p.ucrf;
    upd_halo(o, o->ux, 2, 2, 2, 2);
    upd_halo(o, o->uy, 2, 2, 2, 2);
    upd_halo(o, o->uz, 2, 2, 2, 2);
    upd_halo(o, o->pr, 2, 1, 2, 1);
    if (o->p.scalar_on) upd_halo(o, o->sc, 2, 2, 2, 2);
    const double rdxt = o->rdx / 12.0, rdzt = o->rdz / 12.0;
    const double inxz = one / ((double)nxc * (double)nzc);
#pragma omp parallel for schedule(static)
    for (int jc = 1; jc <= nyc; jc++) {
        const int jp = jc + 1, jm = jc - 1;
        const double InterpY1 = o->yinterp[jc], InterpY2 = one - InterpY1;
        const double cac = o->rdyc[jc], cacU = o->rdyc[jp], caj = o->rdyp[jc];
        double SumVec[40];
        for (int q = 0; q < 40; q++) SumVec[q] = zero;
        for (int kc = 1; kc <= nzc; kc++) {
            const int ks = kc - 2, km = kc - 1, kp = kc + 1, ku = kc + 2;
            for (int ic = 1; ic <= nxc; ic++) {
                const int is = ic - 2, im = ic - 1, ip = ic + 1, iu = ic + 2;
#define A(a, i, j, k) (a)[HX(o, i, j, k)]
                double uxloc = A(ux, ic, jc, kc) + uCRF;
                double uyloc = A(uy, ic, jc, kc);
                double uzloc = A(uz, ic, jc, kc);
                double prloc = A(pr, ic, jc, kc);
                double uxCell = IC[0] * A(ux, im, jc, kc) + IC[1] * A(ux, ic, jc, kc) + IC[2] * A(ux, ip, jc, kc) + IC[3] * A(ux, iu, jc, kc) + uCRF;
                double uyCell = (uyloc + A(uy, ic, jp, kc)) * half;
                double uy_xc = IC[0] * A(uy, is, jc, kc) + IC[1] * A(uy, im, jc, kc) + IC[2] * A(uy, ic, jc, kc) + IC[3] * A(uy, ip, jc, kc);
                double uy_xp = IC[0] * A(uy, is, jp, kc) + IC[1] * A(uy, im, jp, kc) + IC[2] * A(uy, ic, jp, kc) + IC[3] * A(uy, ip, jp, kc);
                double uzCell = IC[0] * A(uz, ic, jc, km) + IC[1] * A(uz, ic, jc, kc) + IC[2] * A(uz, ic, jc, kp) + IC[3] * A(uz, ic, jc, ku);
                double prloc2 = InterpY1 * (IC[0] * A(pr, is, jm, kc) + IC[1] * A(pr, im, jm, kc) + IC[2] * A(pr, ic, jm, kc) + IC[3] * A(pr, ip, jm, kc)) +
                                InterpY2 * (IC[0] * A(pr, is, jc, kc) + IC[1] * A(pr, im, jc, kc) + IC[2] * A(pr, ic, jc, kc) + IC[3] * A(pr, ip, jc, kc));
                double dudx = dxC[0] * A(ux, im, jc, kc) + dxC[1] * A(ux, ic, jc, kc) + dxC[2] * A(ux, ip, jc, kc) + dxC[3] * A(ux, iu, jc, kc);
                double dudy = (A(ux, ic, jc, kc) - A(ux, ic, jm, kc)) * cac;
                double dudz = dzC[0] * A(ux, ic, jc, ks) + dzC[1] * A(ux, ic, jc, km) + dzC[2] * A(ux, ic, jc, kc) + dzC[3] * A(ux, ic, jc, kp);
                double dvdx = dxC[0] * A(uy, is, jc, kc) + dxC[1] * A(uy, im, jc, kc) + dxC[2] * A(uy, ic, jc, kc) + dxC[3] * A(uy, ip, jc, kc);
                double dvdy = (A(uy, ic, jp, kc) - uyloc) * caj;
                double dvdz = dzC[0] * A(uy, ic, jc, ks) + dzC[1] * A(uy, ic, jc, km) + dzC[2] * A(uy, ic, jc, kc) + dzC[3] * A(uy, ic, jc, kp);
                double dwdx = dxC[0] * A(uz, is, jc, kc) + dxC[1] * A(uz, im, jc, kc) + dxC[2] * A(uz, ic, jc, kc) + dxC[3] * A(uz, ip, jc, kc);
                double dwdy = (uzloc - A(uz, ic, jm, kc)) * cac;
                double dwdz = dzC[0] * A(uz, ic, jc, km) + dzC[1] * A(uz, ic, jc, kc) + dzC[2] * A(uz, ic, jc, kp) + dzC[3] * A(uz, ic, jc, ku);
                double dudxx = dxxC[0] * A(ux, is, jc, kc) + dxxC[1] * A(ux, im, jc, kc) + dxxC[2] * A(ux, ic, jc, kc) + dxxC[3] * A(ux, ip, jc, kc) + dxxC[4] * A(ux, iu, jc, kc);
                double dudyy = o->ap2c[jc] * A(ux, ic, jp, kc) + o->ac2c[jc] * A(ux, ic, jc, kc) + o->am2c[jc] * A(ux, ic, jm, kc);
                double dudzz = dzzC[0] * A(ux, ic, jc, ks) + dzzC[1] * A(ux, ic, jc, km) + dzzC[2] * A(ux, ic, jc, kc) + dzzC[3] * A(ux, ic, jc, kp) + dzzC[4] * A(ux, ic, jc, ku);
                double dvdxx = dxxC[0] * A(uy, is, jc, kc) + dxxC[1] * A(uy, im, jc, kc) + dxxC[2] * A(uy, ic, jc, kc) + dxxC[3] * A(uy, ip, jc, kc) + dxxC[4] * A(uy, iu, jc, kc);
                double dvdyy = o->ap2p[jc] * A(uy, ic, jp, kc) + o->ac2p[jc] * A(uy, ic, jc, kc) + o->am2p[jc] * A(uy, ic, jm, kc);
                double dvdzz = dzzC[0] * A(uy, ic, jc, ks) + dzzC[1] * A(uy, ic, jc, km) + dzzC[2] * A(uy, ic, jc, kc) + dzzC[3] * A(uy, ic, jc, kp) + dzzC[4] * A(uy, ic, jc, ku);
                double dwdxx = dxxC[0] * A(uz, is, jc, kc) + dxxC[1] * A(uz, im, jc, kc) + dxxC[2] * A(uz, ic, jc, kc) + dxxC[3] * A(uz, ip, jc, kc) + dxxC[4] * A(uz, iu, jc, kc);
                double dwdyy = o->ap2c[jc] * A(uz, ic, jp, kc) + o->ac2c[jc] * A(uz, ic, jc, kc) + o->am2c[jc] * A(uz, ic, jm, kc);
                double dwdzz = dzzC[0] * A(uz, ic, jc, ks) + dzzC[1] * A(uz, ic, jc, km) + dzzC[2] * A(uz, ic, jc, kc) + dzzC[3] * A(uz, ic, jc, kp) + dzzC[4] * A(uz, ic, jc, ku);
                double vor_x = dwdy - dvdz, vor_y = dudz - dwdx, vor_z = dvdx - dudy;
                double dudxC = (-A(ux, iu, jc, kc) + eight * A(ux, ip, jc, kc) - eight * A(ux, im, jc, kc) + A(ux, is, jc, kc)) * rdxt;
                double dvdxU = dxC[0] * A(uy, is, jp, kc) + dxC[1] * A(uy, im, jp, kc) + dxC[2] * A(uy, ic, jp, kc) + dxC[3] * A(uy, ip, jp, kc);
                double dudyU = (A(ux, ic, jp, kc) - A(ux, ic, jc, kc)) * cacU;
                double dudzC = (InterpY1 * (-A(ux, ic, jm, ku) + eight * A(ux, ic, jm, kp) - eight * A(ux, ic, jm, km) + A(ux, ic, jm, ks)) +
                                InterpY2 * (-A(ux, ic, jc, ku) + eight * A(ux, ic, jc, kp) - eight * A(ux, ic, jc, km) + A(ux, ic, jc, ks))) * rdzt;
                double dvdzC = ((-A(uy, is, jc, ku) + eight * A(uy, is, jc, kp) - eight * A(uy, is, jc, km) + A(uy, is, jc, ks)) * IC[0] +
                                (-A(uy, im, jc, ku) + eight * A(uy, im, jc, kp) - eight * A(uy, im, jc, km) + A(uy, im, jc, ks)) * IC[1] +
                                (-A(uy, ic, jc, ku) + eight * A(uy, ic, jc, kp) - eight * A(uy, ic, jc, km) + A(uy, ic, jc, ks)) * IC[2] +
                                (-A(uy, ip, jc, ku) + eight * A(uy, ip, jc, kp) - eight * A(uy, ip, jc, km) + A(uy, ip, jc, ks)) * IC[3]) * rdzt;
                SumVec[0] += uxloc;
                SumVec[1] += uyloc;
                SumVec[2] += uzloc;
                SumVec[3] += prloc;
                SumVec[4] += uxloc * uxloc;
                SumVec[5] += uyloc * uyloc;
                SumVec[6] += uzloc * uzloc;
                SumVec[7] += prloc * prloc;
                SumVec[8] += uxCell * uyCell;
                SumVec[9] += uyCell * uzCell;
                SumVec[10] += uxCell * uzCell;
                SumVec[11] += uxCell * prloc;
                SumVec[12] += uyCell * prloc;
                SumVec[13] += uzCell * prloc;
                SumVec[14] += uxCell * uxCell * uyCell;
                SumVec[15] += uyloc * uyloc * uyloc;
                SumVec[16] += uzCell * uzCell * uyCell;
                SumVec[17] += uxCell * uyCell * uyCell;
                SumVec[18] += uxloc * uxloc * uxloc;
                SumVec[19] += uzloc * uzloc * uzloc;
                SumVec[20] += uxloc * uxloc * uxloc * uxloc;
                SumVec[21] += uyloc * uyloc * uyloc * uyloc;
                SumVec[22] += uzloc * uzloc * uzloc * uzloc;
                SumVec[23] += prloc * dudx;
                SumVec[24] += prloc * dvdy;
                SumVec[25] += prloc * dwdz;
                SumVec[26] += prloc2 * (dudy + dvdx);
                SumVec[27] += uxloc * (dudxx + dudyy + dudzz);
                SumVec[28] += uyloc * (dvdxx + dvdyy + dvdzz);
                SumVec[29] += uzloc * (dwdxx + dwdyy + dwdzz);
                SumVec[30] += (dudxC * (dvdxU + dvdx) + (dudyU + dudy) * (uy_xp - uy_xc) * caj) * half;
                SumVec[31] += dudzC * dvdzC;
                SumVec[32] += vor_x * vor_x;
                SumVec[33] += vor_y * vor_y;
                SumVec[34] += vor_z * vor_z;
                if (nst > 35) {
                    double scloc = A(sc, ic, jc, kc);
                    SumVec[35] += scloc;
                    SumVec[36] += scloc * scloc;
                    SumVec[37] += scloc * uxCell;
                    SumVec[38] += scloc * uyCell;
                    SumVec[39] += scloc * uzCell;
                }
            }
        }
        for (int q = 0; q < nst; q++) out[(size_t)(jc - 1) * nst + q] = SumVec[q] * inxz;
    }
    /* nyp only */
    {
        const int jc = nyp, jm = jc - 1;
        const double cac = o->rdyc[jc];
        const double InterpY1 = o->yinterp[jc], InterpY2 = one - InterpY1;
        double SumVec[40];
        for (int q = 0; q < 40; q++) SumVec[q] = zero;
        for (int kc = 1; kc <= nzc; kc++)
            for (int ic = 1; ic <= nxc; ic++) {
                const int is = ic - 2, im = ic - 1, ip = ic + 1;
                double prloc2 = InterpY1 * (IC[0] * A(pr, is, jm, kc) + IC[1] * A(pr, im, jm, kc) + IC[2] * A(pr, ic, jm, kc) + IC[3] * A(pr, ip, jm, kc)) +
                                InterpY2 * (IC[0] * A(pr, is, jc, kc) + IC[1] * A(pr, im, jc, kc) + IC[2] * A(pr, ic, jc, kc) + IC[3] * A(pr, ip, jc, kc));
                double dudy = (A(ux, ic, jc, kc) - A(ux, ic, jm, kc)) * cac;
                double dwdy = (A(uz, ic, jc, kc) - A(uz, ic, jm, kc)) * cac;
                double vor_x = dwdy, vor_z = -dudy;
                SumVec[26] += prloc2 * (dudy + zero);
                SumVec[32] += vor_x * vor_x;
                SumVec[34] += vor_z * vor_z;
            }
#undef A
        for (int q = 0; q < nst; q++) out[(size_t)(jc - 1) * nst + q] = SumVec[q] * inxz;
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * 1-D spectra of clcStat (src/m_FlowCase.f90:430-806) with the helpers
 * clcEnergySpectraX/Z, clcLTS_x/z_real, clcLTS_x/z_imag and clcCospectraX/Z
 * (:954-1180), on halfcomplex rows h[0..n-1].  Index a = ic-1 of the
 * Fortran arrays; the mirror icCnter = n+2-ic is c = n-a.
 * ---------------------------------------------------------------------- */
static void spec_energy(int n, const double* h, double* E) {        /* :954-977 */
    const int nh = n / 2;
    E[0] = E[0] + h[0] * h[0];
    E[nh] = E[nh] + h[nh] * h[nh];
    for (int a = 1; a < nh; a++) {
        const int c = n - a;
        E[a] = E[a] + (h[a] * h[a] + h[c] * h[c]) * two;
    }
}
static void spec_cos(int n, const double* h, const double* g, double* E) {   /* :1032-1055 */
    const int nh = n / 2;
    E[0] = E[0] + h[0] * g[0];
    E[nh] = E[nh] + h[nh] * g[nh];
    for (int a = 1; a < nh; a++) {
        const int c = n - a;
        E[a] = E[a] + (h[a] * g[a] + h[c] * g[c]) * two;
    }
}
/* clcLTS_real on the product array P[a] = h[a]*r[a] (:471-510, :982-1003) */
static void spec_lcs_real(int n, const double* h, const double* r, double* E) {
    const int nh = n / 2;
    E[0] = E[0] + h[0] * r[0];
    E[nh] = E[nh] + h[nh] * r[nh];
    for (int a = 1; a < nh; a++) {
        const int c = n - a;
        E[a] = E[a] + (h[a] * r[a] + h[c] * r[c]);
    }
}
/* clcLTS_imag on Q[a] = h[n-a]*r[a] (the swapped row of :513-520 times the
 * reference plane, :521-545, :1008-1027); the two end modes stay zero */
static void spec_lcs_imag(int n, const double* h, const double* r, double* E) {
    const int nh = n / 2;
    E[0] = zero;
    E[nh] = zero;
    for (int a = 1; a < nh; a++) {
        const int c = n - a;
        E[a] = E[a] + (h[c] * r[a] - h[a] * r[c]);
    }
}

/* one row of every field along the transform direction: r[0] ux+uCRF, r[1]
 * ux+uCRF on the LCS reference row, r[2] uy, r[3] uz, r[4] p, r[5] uy at the
 * cell centre, r[6] ux at the cell centre (+uCRF), r[7] the scalar (or 0);
 * E[m][a] gets spectrum m+1 of the reference's numbering */
static void spec_rows(const fftplan* pl, int n, double* const* r, double* const* h, cplx* z, int nsp, int nhp,
                      double* E) {
    r2hc_pair(pl, r[0], r[1], h[0], h[1], z, z + n);
    r2hc_pair(pl, r[2], r[3], h[2], h[3], z, z + n);
    r2hc_pair(pl, r[4], r[5], h[4], h[5], z, z + n);
    r2hc_pair(pl, r[6], r[7], h[6], h[7], z, z + n);
    spec_energy(n, h[0], E + 0 * nhp);
    spec_lcs_real(n, h[0], h[1], E + 6 * nhp);
    spec_lcs_imag(n, h[0], h[1], E + 7 * nhp);
    spec_energy(n, h[2], E + 1 * nhp);
    spec_energy(n, h[3], E + 2 * nhp);
    spec_energy(n, h[4], E + 3 * nhp);
    spec_cos(n, h[0], h[5], E + 4 * nhp);
    spec_cos(n, h[6], h[5], E + 5 * nhp);
    if (nsp > 8) spec_energy(n, h[7], E + 8 * nhp);
}

int orc_spectra(orc_t* o, int jlcs, double* egx, double* egz) {
    if (!o || !egx || !egz || jlcs < 1 || jlcs > o->nyc) return PARATC_ERR_BAD_ARG;
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    const int nsp = o->p.scalar_on ? 9 : 8;
    const int nxhp = nxc / 2 + 1, nzhp = nzc / 2 + 1;
    const double *ux = o->ux, *uy = o->uy, *uz = o->uz, *pr = o->pr, *sc = o->sc, *IC = o->IC;
    const double uCRF = o->p.ucrf;
    const int is_hc = (o->p.flow_type == PARATC_FT_HC);
    upd_halo(o, o->ux, 2, 2, 2, 2);
    const double normx = one / ((double)nxc * (double)nxc * (double)nzc);
    const double normz = one / ((double)nxc * (double)nzc * (double)nzc);
    for (int dir = 0; dir < 2; dir++) {
        const int n = dir == 0 ? nxc : nzc, nhp = dir == 0 ? nxhp : nzhp, nl = dir == 0 ? nzc : nxc;
        const fftplan* pl = dir == 0 ? &o->px : &o->pz;
        double* out = dir == 0 ? egx : egz;
        const double norm = dir == 0 ? normx : normz;
#pragma omp parallel
        {
            double* wk = (double*)malloc(sizeof(double) * (16 * (size_t)n + 9 * (size_t)nhp));
            cplx* z = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)n);
            double *r[8], *h[8];
            for (int q = 0; q < 8; q++) { r[q] = wk + (size_t)q * n; h[q] = wk + (size_t)(8 + q) * n; }
            double* E = wk + 16 * (size_t)n;
#pragma omp for schedule(static)
            for (int jc = 1; jc <= nyc; jc++) {
                const int jr = (is_hc || jc <= nyc / 2) ? jlcs : nyc + 1 - jlcs;
                for (int q = 0; q < 9 * nhp; q++) E[q] = zero;
                for (int l = 1; l <= nl; l++) {
                    for (int e = 1; e <= n; e++) {
                        const int ic = dir == 0 ? e : l, kc = dir == 0 ? l : e;
                        const int im = ic - 1, ip = ic + 1, iu = ic + 2;
#define A(a, i, j, k) (a)[HX(o, i, j, k)]
                        r[0][e - 1] = A(ux, ic, jc, kc) + uCRF;
                        r[1][e - 1] = A(ux, ic, jr, kc) + uCRF;
                        r[2][e - 1] = A(uy, ic, jc, kc);
                        r[3][e - 1] = A(uz, ic, jc, kc);
                        r[4][e - 1] = A(pr, ic, jc, kc);
                        r[5][e - 1] = half * (A(uy, ic, jc, kc) + A(uy, ic, jc + 1, kc));
                        r[6][e - 1] = IC[0] * A(ux, im, jc, kc) + IC[1] * A(ux, ic, jc, kc) + IC[2] * A(ux, ip, jc, kc) +
                                      IC[3] * A(ux, iu, jc, kc) + uCRF;
                        r[7][e - 1] = nsp > 8 ? A(sc, ic, jc, kc) : zero;
#undef A
                    }
                    spec_rows(pl, n, r, h, z, nsp, nhp, E);
                }
                for (int m = 0; m < nsp; m++)
                    for (int a = 0; a < nhp; a++)
                        out[((size_t)m * nyc + (jc - 1)) * nhp + a] = E[(size_t)m * nhp + a] * norm;
            }
            free(wk);
            free(z);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * 2-D spectra of clcStat (src/m_FlowCase.f90:780-803) with
 * clcEnergySpectra2D and clcCosSpectra2D (:1186-1375): the field is
 * transformed R2HC along x, then R2HC along z (a halfcomplex-of-halfcomplex
 * array, not a complex 2-D transform), and at the rows iySpec2D the squares
 * (products for the cospectrum) are added with normEgy = (1/(nxc nzc))^2,
 * halved in a channel, where the mirrored row is added too (nyp+1-jct for the
 * uy faces, nyc+1-jct otherwise; the cospectrum subtracts it, IsSymmetry =
 * .false.).  Fields: 1 ux (no uCRF), 2 uy, 3 uz, 4 p, 5 <ux_c uy_c> with ux_c
 * the cell-centre interpolation + uCRF (:434-444) and uy_c = (uy_j +
 * uy_j+1)/2 (:784-793) [, 6 scalar].  out[((m*nzc + kc)*nsel + q)*nxc + ic]
 * gets one call's contribution (EnergySpec2D's Fortran order).
 * ---------------------------------------------------------------------- */
/* hc-hc transform of one y row of field f: H[kc*nxc + ic] */
static void hc2d_row(orc_t* o, int f, int j, double* H, double* row, double* hrow, cplx* z) {
    const int nxc = o->nxc, nzc = o->nzc;
    const double *ux = o->ux, *uy = o->uy, *uz = o->uz, *pr = o->pr, *sc = o->sc, *IC = o->IC;
    const double uCRF = o->p.ucrf;
    double* zero_row = row + (nxc > nzc ? nxc : nzc);
    for (int q = 0; q < (nxc > nzc ? nxc : nzc); q++) zero_row[q] = zero;
    for (int kc = 1; kc <= nzc; kc++) {
        for (int ic = 1; ic <= nxc; ic++) {
#define A(a, i, jj, k) (a)[HX(o, i, jj, k)]
            double v;
            switch (f) {
                case 0: v = A(ux, ic, j, kc); break;
                case 1: v = A(uy, ic, j, kc); break;
                case 2: v = A(uz, ic, j, kc); break;
                case 3: v = A(pr, ic, j, kc); break;
                case 4: v = IC[0] * A(ux, ic - 1, j, kc) + IC[1] * A(ux, ic, j, kc) + IC[2] * A(ux, ic + 1, j, kc) +
                            IC[3] * A(ux, ic + 2, j, kc) + uCRF; break;
                case 5: v = half * (A(uy, ic, j, kc) + A(uy, ic, j + 1, kc)); break;
                default: v = A(sc, ic, j, kc); break;
            }
#undef A
            row[ic - 1] = v;
        }
        r2hc_pair(&o->px, row, zero_row, H + (size_t)(kc - 1) * nxc, hrow, z, z + nxc);
    }
    for (int ic = 0; ic < nxc; ic++) {
        for (int kc = 0; kc < nzc; kc++) row[kc] = H[(size_t)kc * nxc + ic];
        r2hc_pair(&o->pz, row, zero_row, hrow, hrow + nzc, z, z + nzc);
        for (int kc = 0; kc < nzc; kc++) H[(size_t)kc * nxc + ic] = hrow[kc];
    }
}

int orc_spectra2d(orc_t* o, int nsel, const int* iy, double* out) {
    if (!o || !out || !iy || nsel < 1) return PARATC_ERR_BAD_ARG;
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc, nyp = o->nyp;
    const int is_hc = (o->p.flow_type == PARATC_FT_HC);
    for (int q = 0; q < nsel; q++)
        if (iy[q] < 2 || iy[q] > (o->p.flow_type == PARATC_FT_CH ? nyc / 2 : nyc)) return PARATC_ERR_BAD_ARG;
    const int nsp = o->p.scalar_on ? 6 : 5;
    upd_halo(o, o->ux, 2, 2, 2, 2);
    double normEgy = one / ((double)nxc * (double)nzc);
    normEgy = normEgy * normEgy;
    if (o->p.flow_type == PARATC_FT_CH) normEgy = normEgy * half;
    const size_t pl = (size_t)nxc * nzc;
    const int nmax = nxc > nzc ? nxc : nzc;
#pragma omp parallel
    {
        double* H = (double*)malloc(sizeof(double) * 4 * pl);
        double* row = (double*)malloc(sizeof(double) * 4 * (size_t)nmax);
        cplx* z = (cplx*)malloc(sizeof(cplx) * 2 * (size_t)nmax);
#pragma omp for schedule(static) collapse(2)
        for (int q = 0; q < nsel; q++) {
            for (int m = 0; m < nsp; m++) {
                const int jct = iy[q];
                double *H1 = H, *H2 = H + pl, *H3 = H + 2 * pl, *H4 = H + 3 * pl;
                if (m == 4) {                                   /* clcCosSpectra2D(ArrTemp1, ArrTemp2, 5, .false.) */
                    hc2d_row(o, 4, jct, H1, row, row + 2 * nmax, z);
                    hc2d_row(o, 5, jct, H2, row, row + 2 * nmax, z);
                    if (!is_hc) {
                        const int jcs = nyc + 1 - jct;
                        hc2d_row(o, 4, jcs, H3, row, row + 2 * nmax, z);
                        hc2d_row(o, 5, jcs, H4, row, row + 2 * nmax, z);
                    }
                    for (size_t e = 0; e < pl; e++) {
                        const double rt1 = H1[e] * H2[e];
                        double v;
                        if (is_hc) v = normEgy * rt1;
                        else { const double rt2 = H3[e] * H4[e]; v = normEgy * (rt1 + (-one) * rt2); }
                        const size_t kc = e / nxc, ic = e % nxc;
                        out[(((size_t)m * nzc + kc) * nsel + q) * nxc + ic] = v;
                    }
                } else {                                         /* clcEnergySpectra2D */
                    const int f = m < 4 ? m : 6;
                    hc2d_row(o, f, jct, H1, row, row + 2 * nmax, z);
                    if (!is_hc) hc2d_row(o, f, (f == 1 ? nyp : nyc) + 1 - jct, H2, row, row + 2 * nmax, z);
                    for (size_t e = 0; e < pl; e++) {
                        const double rt1 = H1[e];
                        double v;
                        if (is_hc) v = normEgy * rt1 * rt1;
                        else { const double rt2 = H2[e]; v = normEgy * (rt1 * rt1 + rt2 * rt2); }
                        const size_t kc = e / nxc, ic = e % nxc;
                        out[(((size_t)m * nzc + kc) * nsel + q) * nxc + ic] = v;
                    }
                }
            }
        }
        free(H);
        free(row);
        free(z);
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * one substep: body of the ns loop of ChannelIterate
 * (src/m_ChannelSystem.f90:102-140)
 * ---------------------------------------------------------------------- */
int orc_substep(orc_t* o, int ns, double dt, int stop_stage, double* divmax_src) {
    if (!o || ns < 1 || ns > o->iadvance) return PARATC_ERR_BAD_ARG;
    o->dt = dt;
    pm_update(o, ns);
    update_uy_ym(o);
    clc_rhs(o);
    if (stop_stage == 1) return 0;
    if (o->p.scalar_on) helm_cn(o, o->sc, o->rhsc, o->pmBetaSc, o->ap2cScCN, o->ac2cScCN, o->am2cScCN);
    helm_cn(o, o->ux, o->rhsx, o->pmBeta, o->ap2cCN, o->ac2cCN, o->am2cCN);
    helm_v(o);
    helm_cn(o, o->uz, o->rhsz, o->pmBeta, o->ap2cCN, o->ac2cCN, o->am2cCN);
    if (stop_stage == 2) return 0;
    bc_prsrc(o);
    double dm = clc_prsrc(o, o->prsrc, one / o->pmAlpha);
    if (divmax_src) *divmax_src = dm;
    if (stop_stage == 3) return 0;
    clc_ppe(o, o->prsrc, o->phi_int);
    phi_to_halo(o);
    if (stop_stage == 4) return 0;
    fluid_vel_update(o, o->pmAlpha);
    pressure_update(o);
    bc_vel(o);
    bc_pr(o, o->pr);
    if (o->p.scalar_on) bc_scalar(o);
    return 0;
}

/* ChannelIterate without statistics / visu / restart IO
 * (src/m_ChannelSystem.f90:80-187) */
int orc_step(orc_t* o, paratc_diag* diag) {
    if (!o) return PARATC_ERR_BAD_ARG;
    double uddxmax = calc_max_cfl(o);
    double cflmp = uddxmax * o->dt;
    double dt;
    if (o->p.icfl == 1) {
        dt = o->p.cflc / uddxmax;
        if (o->p.dt_max < dt) dt = o->p.dt_max;
    } else {
        dt = o->p.dt_max;
    }
    double dm1 = 0.0;
    for (int ns = 1; ns <= o->iadvance; ns++) orc_substep(o, ns, dt, 5, &dm1);
    double dm2 = clc_prsrc(o, NULL, one);
    double vm[3];
    calc_vmax(o, vm);
    if (diag) {
        double m[3];
        calc_means(o, m);
        diag->dt = dt; diag->cfl = cflmp; diag->sim_time = o->sim_time;
        diag->divmax_src = dm1; diag->divmax = dm2;
        diag->vmax[0] = vm[0]; diag->vmax[1] = vm[1]; diag->vmax[2] = vm[2];
        diag->pr_grad_aver = o->pr_grad_aver;
        diag->ux_mean = m[0]; diag->sc_mean = m[1]; diag->sc2_mean = m[2];
    }
    if (dm2 > o->p.div_limit) return PARATC_ERR_DIV_LIMIT;
    double vmin = vm[0];
    if (vm[1] < vmin) vmin = vm[1];
    if (vm[2] < vmin) vmin = vm[2];
    if (vmin > o->p.vel_limit) return PARATC_ERR_VEL_LIMIT;
    return 0;
}

int orc_poisson(orc_t* o, const double* src, double* phi) {
    if (!o || !src || !phi) return PARATC_ERR_BAD_ARG;
    clc_ppe(o, src, phi);
    return 0;
}

/* one pressure-free projection of the current velocity (pmAlpha = 1) */
int orc_project(orc_t* o, double* divmax_out) {
    if (!o) return PARATC_ERR_BAD_ARG;
    bc_prsrc(o);
    clc_prsrc(o, o->prsrc, one);
    clc_ppe(o, o->prsrc, o->phi_int);
    phi_to_halo(o);
    fluid_vel_update(o, one);
    bc_vel(o);
    double dm = clc_prsrc(o, NULL, one);
    if (divmax_out) *divmax_out = dm;
    return 0;
}

/* ------------------------------------------------------------------------
 * field access
 * ---------------------------------------------------------------------- */
static void put_int(orc_t* o, double* h, const double* in) {
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= o->nzc; kc++)
        for (int jc = 1; jc <= o->nyc; jc++)
            memcpy(&h[HX(o, 1, jc, kc)], &in[IX(o, 1, jc, kc)], sizeof(double) * o->nxc);
}
static void get_int(orc_t* o, const double* h, double* out) {
#pragma omp parallel for schedule(static)
    for (int kc = 1; kc <= o->nzc; kc++)
        for (int jc = 1; jc <= o->nyc; jc++)
            memcpy(&out[IX(o, 1, jc, kc)], &h[HX(o, 1, jc, kc)], sizeof(double) * o->nxc);
}

/* state load as ChannelInitialize does after read_restart
 * (src/m_ChannelSystem.f90:63-68) */
int orc_set_fields(orc_t* o, const double* ux, const double* uy, const double* uz, const double* p,
                   const double* c, const double* hx, const double* hy, const double* hz,
                   const double* hc) {
    if (!o) return PARATC_ERR_BAD_ARG;
    if (ux) put_int(o, o->ux, ux);
    if (uy) put_int(o, o->uy, uy);
    if (uz) put_int(o, o->uz, uz);
    if (p) put_int(o, o->pr, p);
    if (o->p.scalar_on && c) put_int(o, o->sc, c);
    size_t nb = sizeof(double) * o->ni;
    if (hx) memcpy(o->hx, hx, nb); else memset(o->hx, 0, nb);
    if (hy) memcpy(o->hy, hy, nb); else memset(o->hy, 0, nb);
    if (hz) memcpy(o->hz, hz, nb); else memset(o->hz, 0, nb);
    if (o->p.scalar_on) { if (hc) memcpy(o->hc, hc, nb); else memset(o->hc, 0, nb); }
    update_uy_ym(o);
    o->sim_time = zero;
    o->dt = o->p.dt_max;
    bc_vel(o);
    bc_pr(o, o->pr);
    if (o->p.scalar_on) bc_scalar(o);
    return 0;
}

int orc_get_fields(orc_t* o, double* ux, double* uy, double* uz, double* p, double* c, double* hx,
                   double* hy, double* hz, double* hc) {
    if (!o) return PARATC_ERR_BAD_ARG;
    size_t nb = sizeof(double) * o->ni;
    if (ux) get_int(o, o->ux, ux);
    if (uy) get_int(o, o->uy, uy);
    if (uz) get_int(o, o->uz, uz);
    if (p) get_int(o, o->pr, p);
    if (c && o->p.scalar_on) get_int(o, o->sc, c);
    if (hx) memcpy(hx, o->hx, nb);
    if (hy) memcpy(hy, o->hy, nb);
    if (hz) memcpy(hz, o->hz, nb);
    if (hc && o->p.scalar_on) memcpy(hc, o->hc, nb);
    return 0;
}

int orc_get_halo(orc_t* o, int which, double* out) {
    double* src[] = {o->ux, o->uy, o->uz, o->pr, o->sc, o->phi};
    if (!o || which < 0 || which > 5 || !src[which]) return PARATC_ERR_BAD_ARG;
    memcpy(out, src[which], sizeof(double) * o->nh);
    return 0;
}

int orc_get_work(orc_t* o, int which, double* out) {
    double* src[] = {o->rhsx, o->rhsy, o->rhsz, o->rhsc, o->prsrc, o->phi_int};
    if (!o || which < 0 || which > 5 || !src[which]) return PARATC_ERR_BAD_ARG;
    memcpy(out, src[which], sizeof(double) * o->ni);
    return 0;
}

int orc_set_time(orc_t* o, double sim_time, double dt) {
    if (!o) return PARATC_ERR_BAD_ARG;
    o->sim_time = sim_time; o->dt = dt;
    return 0;
}

int orc_get_time(orc_t* o, double* sim_time, double* dt, double* pga) {
    if (!o) return PARATC_ERR_BAD_ARG;
    if (sim_time) *sim_time = o->sim_time;
    if (dt) *dt = o->dt;
    if (pga) *pga = o->pr_grad_aver;
    return 0;
}

int orc_metric(orc_t* o, const char* name, double* out, int cap) {
    struct { const char* n; const double* a; int lo, hi; } tab[] = {
        {"yp", o->yp, 1, o->nyp}, {"yc", o->yc, 0, o->nyp}, {"dyp", o->dyp, 0, o->nyp},
        {"dyc", o->dyc, 1, o->nyp}, {"rdyp", o->rdyp, 0, o->nyp}, {"rdyc", o->rdyc, 1, o->nyp},
        {"YinterpCoe", o->yinterp, 1, o->nyp},
        {"ap2ph", o->ap2ph, 1, o->nyc}, {"ac2ph", o->ac2ph, 1, o->nyc}, {"am2ph", o->am2ph, 1, o->nyc},
        {"ap2c", o->ap2c, 1, o->nyc}, {"ac2c", o->ac2c, 1, o->nyc}, {"am2c", o->am2c, 1, o->nyc},
        {"ap2cForCN", o->ap2cCN, 1, o->nyc}, {"ac2cForCN", o->ac2cCN, 1, o->nyc}, {"am2cForCN", o->am2cCN, 1, o->nyc},
        {"ap2p", o->ap2p, 1, o->nyc}, {"ac2p", o->ac2p, 1, o->nyc}, {"am2p", o->am2p, 1, o->nyc},
        {"ap2cSc", o->ap2cSc, 1, o->nyc}, {"ac2cSc", o->ac2cSc, 1, o->nyc}, {"am2cSc", o->am2cSc, 1, o->nyc},
        {"ap2cScCN", o->ap2cScCN, 1, o->nyc}, {"ac2cScCN", o->ac2cScCN, 1, o->nyc}, {"am2cScCN", o->am2cScCN, 1, o->nyc},
        {"WaveNumX", o->wnx, 1, o->nxc}, {"WaveNumZ", o->wnz, 1, o->nzc},
    };
    for (size_t t = 0; t < sizeof(tab) / sizeof(tab[0]); t++) {
        if (strcmp(tab[t].n, name) == 0) {
            int n = tab[t].hi - tab[t].lo + 1;
            if (n > cap) return PARATC_ERR_BAD_ARG;
            for (int i = 0; i < n; i++) out[i] = tab[t].a[tab[t].lo + i];
            return n;
        }
    }
    return PARATC_ERR_BAD_ARG;
}


/* ------------------------------------------------------------------------
 * dump_visu (src/m_IOAndVisu.f90:182-385) with Clc_Q_vor, Clc_lamda2 and
 * CubicRoot (src/m_Tools.f90:305-440, 494-570), at the points
 * decomp_2d_write_every keeps with from1 = .true. (src/m_Decomp2d.f90:
 * 1232-1389): ic = 1, 1+iskip, ... (likewise j, k), Fortran order.
 * Quantity numbers as PARATC_VISU_*.  Returns PARATC_ERR_NUMERIC after
 * filling out when lambda2 met complex roots (the reference stops there).
 * ---------------------------------------------------------------------- */
static double cubic_root2(double b, double c, double d, int* allreal) {
    const double SMALL = 1.0E-12, OneThird = 0.3333333333333333333333;
    const double Pi = 3.141592653589793238462643383279502884;
    double p = c - OneThird * b * b;
    double q = (2.0 * b * b * b - 9.0 * b * c + 27.0 * d) / 27.0;
    double t = q * q / 4.0 + p * p * p / 27.0;
    if (t < 0.0) {
        *allreal = 1;
        t = -OneThird * b;
        double rho = pow(-p, 1.5) / sqrt(27.0);
        double eta = acos(0.5 * q / rho);
        rho = -2.0 * pow(rho, OneThird);
        double root1 = cos(OneThird * eta) * rho + t;
        double root2 = cos(OneThird * (2.0 * Pi + eta)) * rho + t;
        double root3 = cos(OneThird * (4.0 * Pi + eta)) * rho + t;
        if (root1 < root2 && root1 < root3) return root2 < root3 ? root2 : root3;
        else if (root1 > root2 && root1 > root3) return root2 < root3 ? root3 : root2;
        else return root1;
    } else if (t < SMALL) {
        *allreal = 1;
        double rho = 0.5 * q;
        if (rho < 0.0) rho = pow(-rho, OneThird);
        else rho = -pow(rho, OneThird);
        return -rho - OneThird * b;
    }
    *allreal = 0;
    t = sqrt(t);
    double rho = 0.5 * q + t, eta = 0.5 * q - t;
    if (rho < 0.0) rho = pow(-rho, OneThird); else rho = -pow(rho, OneThird);
    if (eta < 0.0) eta = pow(-eta, OneThird); else eta = -pow(eta, OneThird);
    return -0.5 * (rho + eta) - OneThird * b;
}

int orc_visu(orc_t* o, int qn, int iskip, int jskip, int kskip, int node, double* out) {
    if (!o || !out || qn < 0 || qn > 10 || iskip < 1 || jskip < 1 || kskip < 1) return PARATC_ERR_BAD_ARG;
    if (qn == 10 && !o->p.scalar_on) return PARATC_ERR_BAD_ARG;
    const int nxc = o->nxc, nyc = o->nyc, nzc = o->nzc;
    const int nxo = (nxc + iskip - 1) / iskip, nyo = (nyc + jskip - 1) / jskip, nzo = (nzc + kskip - 1) / kskip;
    const double *ux = o->ux, *uy = o->uy, *uz = o->uz, *pr = o->pr, *sc = o->sc;
    const double rdx = o->rdx, rdz = o->rdz, uCRF = o->p.ucrf;
    upd_halo(o, o->ux, 2, 2, 2, 2);
    upd_halo(o, o->uy, 2, 2, 2, 2);
    upd_halo(o, o->uz, 2, 2, 2, 2);
    int nbad = 0;
#pragma omp parallel for schedule(static) reduction(+ : nbad)
    for (int ko = 0; ko < nzo; ko++) {
        const int kc = 1 + ko * kskip, kp = kc + 1, km = kc - 1;
        for (int jo = 0; jo < nyo; jo++) {
            const int jc = 1 + jo * jskip, jp = jc + 1, jm = jc - 1;
            const double caj = o->rdyp[jc], cac1 = o->rdyc[jc], cac2 = o->rdyc[jp], cac12 = cac1 - cac2;
            for (int io = 0; io < nxo; io++) {
                const int ic = 1 + io * iskip, ip = ic + 1, im = ic - 1;
#define A(a, i, j, k) (a)[HX(o, i, j, k)]
                double v;
                if (qn == 0) v = node ? A(ux, ic, jc, kc) + uCRF : half * (A(ux, ic + 1, jc, kc) + A(ux, ic, jc, kc)) + uCRF;
                else if (qn == 1) v = node ? A(uy, ic, jc, kc) : half * (A(uy, ic, jc + 1, kc) + A(uy, ic, jc, kc));
                else if (qn == 2) v = node ? A(uz, ic, jc, kc) : half * (A(uz, ic, jc, kc + 1) + A(uz, ic, jc, kc));
                else if (qn == 3) v = A(pr, ic, jc, kc);
                else if (qn == 10) v = A(sc, ic, jc, kc);
                else {
                    double dudx = (A(ux, ip, jc, kc) - A(ux, ic, jc, kc)) * rdx;
                    double dudy = ((A(ux, ip, jp, kc) + A(ux, ic, jp, kc)) * cac2 + (A(ux, ip, jc, kc) + A(ux, ic, jc, kc)) * cac12 -
                                   (A(ux, ip, jm, kc) + A(ux, ic, jm, kc)) * cac1) * quarter;
                    double dudz = (A(ux, ip, jc, kp) + A(ux, ic, jc, kp) - A(ux, ip, jc, km) - A(ux, ic, jc, km)) * rdz * quarter;
                    double dvdx = (A(uy, ip, jp, kc) - A(uy, im, jp, kc) + A(uy, ip, jc, kc) - A(uy, im, jc, kc)) * rdx * quarter;
                    double dvdy = (A(uy, ic, jp, kc) - A(uy, ic, jc, kc)) * caj;
                    double dvdz = (A(uy, ic, jp, kp) + A(uy, ic, jc, kp) - A(uy, ic, jp, km) - A(uy, ic, jc, km)) * rdz * quarter;
                    double dwdx = (A(uz, ip, jc, kp) - A(uz, im, jc, kp) + A(uz, ip, jc, kc) - A(uz, im, jc, kc)) * rdx * quarter;
                    double dwdy = ((A(uz, ic, jp, kp) + A(uz, ic, jp, kc)) * cac2 + (A(uz, ic, jc, kp) + A(uz, ic, jc, kc)) * cac12 -
                                   (A(uz, ic, jm, kp) + A(uz, ic, jm, kc)) * cac1) * quarter;
                    double dwdz = (A(uz, ic, jc, kp) - A(uz, ic, jc, kc)) * rdz;
#undef A
                    if (qn == 4) v = dwdy - dvdz;
                    else if (qn == 5) v = dudz - dwdx;
                    else if (qn == 6) v = dvdx - dudy;
                    else if (qn == 7) {
                        double vor_x = dwdy - dvdz, vor_y = dudz - dwdx, vor_z = dvdx - dudy;
                        v = sqrt(vor_x * vor_x + vor_y * vor_y + vor_z * vor_z);
                    } else if (qn == 8) {
                        double udiv = dudx + dvdy + dwdz;
                        v = half * (udiv * udiv - dudx * dudx - dvdy * dvdy - dwdz * dwdz) - dudy * dvdx - dudz * dwdx - dvdz * dwdy;
                    } else {
                        double Ome12 = dvdx - dudy, Ome23 = dwdy - dvdz, Ome31 = dudz - dwdx;
                        double Eps11 = dudx + dudx, Eps12 = dudy + dvdx, Eps13 = dudz + dwdx;
                        double Eps22 = dvdy + dvdy, Eps23 = dvdz + dwdy, Eps33 = dwdz + dwdz;
                        double Lam12 = Eps11 * Eps12 + Eps12 * Eps22 + Eps13 * Eps23 + Ome31 * Ome23;
                        double Lam13 = Eps11 * Eps13 + Eps12 * Eps23 + Eps13 * Eps33 + Ome12 * Ome23;
                        double Lam23 = Eps12 * Eps13 + Eps22 * Eps23 + Eps23 * Eps33 + Ome12 * Ome31;
                        double Lam11 = Eps11 * Eps11 + Eps12 * Eps12 + Eps13 * Eps13 - Ome12 * Ome12 - Ome31 * Ome31;
                        double Lam22 = Eps12 * Eps12 + Eps22 * Eps22 + Eps23 * Eps23 - Ome12 * Ome12 - Ome23 * Ome23;
                        double Lam33 = Eps13 * Eps13 + Eps23 * Eps23 + Eps33 * Eps33 - Ome31 * Ome31 - Ome23 * Ome23;
                        double rb = -(Lam11 + Lam22 + Lam33);
                        double rc = Lam11 * Lam22 + Lam22 * Lam33 + Lam33 * Lam11 - Lam12 * Lam12 - Lam13 * Lam13 - Lam23 * Lam23;
                        double rd = Lam12 * Lam12 * Lam33 + Lam13 * Lam13 * Lam22 + Lam23 * Lam23 * Lam11 - Lam11 * Lam22 * Lam33 -
                                    2.0 * Lam12 * Lam23 * Lam13;
                        int allreal;
                        v = quarter * cubic_root2(rb, rc, rd, &allreal);
                        if (!allreal) nbad++;
                    }
                }
                out[((size_t)ko * nyo + jo) * nxo + io] = v;
            }
        }
    }
    return nbad ? PARATC_ERR_NUMERIC : 0;
}
