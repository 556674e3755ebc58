/*
 * paratc_oracle.h -- TEST INFRASTRUCTURE, not product code.
 *
 * CPU restatement (C, OpenMP) of ParaTC's per-RK3-substep hot path, used only
 * by tests/, __graft_entry__.smoke() and the CPU baseline of bench.py as the
 * checker.  See paratc_oracle.c for the file:line each routine follows and for
 * the parity-pinning status.
 */
#ifndef PARATC_ORACLE_H
#define PARATC_ORACLE_H
#include "../include/paratc.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc_t;

int  orc_ycoord(int nsection, const double* section_length, const double* section_cstret,
                const int32_t* nyc_section, const int32_t* stret_type,
                const int32_t* stret_option, double yly, double* yp_out);
int  orc_create(const paratc_params* prm, const double* yp, orc_t** out);
void orc_destroy(orc_t* o);
void orc_set_threads(int n);

/* interior (nxc*nyc*nzc, Fortran order) in/out; NULL pointers skipped / zero */
int  orc_set_fields(orc_t* o, const double* ux, const double* uy, const double* uz,
                    const double* p, const double* c, const double* hx,
                    const double* hy, const double* hz, const double* hc);
int  orc_get_fields(orc_t* o, double* ux, double* uy, double* uz, double* p,
                    double* c, double* hx, double* hy, double* hz, double* hc);
/* halo'd ((nxc+4)*(nyc+2)*(nzc+4)) copies of ux,uy,uz,p,c (which = 0..4) */
int  orc_get_halo(orc_t* o, int which, double* out);

int  orc_set_time(orc_t* o, double sim_time, double dt);
int  orc_get_time(orc_t* o, double* sim_time, double* dt, double* pr_grad_aver);

int  orc_step(orc_t* o, paratc_diag* diag);
/* substep ns with dt; stop after stage (1 rhs, 2 helmholtz, 3 prsrc, 4 ppe,
 * 5 complete). */
int  orc_substep(orc_t* o, int ns, double dt, int stop_stage, double* divmax_src);
/* intermediate arrays (interior): 0 RhsX, 1 RhsY, 2 RhsZ, 3 RhsC, 4 prsrc, 5 phi */
int  orc_get_work(orc_t* o, int which, double* out);

int  orc_poisson(orc_t* o, const double* src, double* phi);
int  orc_project(orc_t* o, double* divmax_out);
int  orc_diagnostics(orc_t* o, paratc_diag* diag);

/* 1D metric arrays by name (e.g. "yp", "ac2ph", "am2cForCN"); returns the
 * number of values written (Fortran index from the array's lower bound). */
int  orc_metric(orc_t* o, const char* name, double* out, int cap);
/* clcStat: one call's SumVec*inxz per row jc = 1..nyp (k fastest; 35 or 40) */
int  orc_stats(orc_t* o, double* out);
/* clcStat's 1-D spectra: one call's EgyX*normEgy / EgyZ*normEgy,
 * egx[(m*nyc + jc-1)*(nxc/2+1) + kx], egz likewise with nzc/2+1 modes, for
 * the reference's spectra m = 1..8 (9 with the scalar) in its order: ux, uy,
 * uz, p, the cospectra <ux uy_c> and <ux_c uy_c>, LCS real, LCS imaginary
 * [, scalar]; jlcs is jForLCS (1..nyc). */
int  orc_spectra(orc_t* o, int jlcs, double* egx, double* egz);
/* clcStat's 2-D spectra at the rows iy[0..nsel-1] (iySpec2D): one call's
 * contribution, out[((m*nzc + kc)*nsel + q)*nxc + ic] for m = 1..5 (6 with
 * the scalar): ux, uy, uz, p, <ux_c uy_c> [, scalar] of the halfcomplex-of-
 * halfcomplex x-z transform. */
int  orc_spectra2d(orc_t* o, int nsel, const int* iy, double* out);
/* dump_visu's quantity q (PARATC_VISU_* numbering) at the points
 * decomp_2d_write_every keeps (1, 1+skip, ...), Fortran order; node != 0 is
 * the SaveNode build.  PARATC_ERR_NUMERIC when lambda2 met complex roots. */
int  orc_visu(orc_t* o, int q, int iskip, int jskip, int kskip, int node, double* out);

/* real DFT helpers in FFTW's halfcomplex convention (for pinning) */
int  orc_r2hc(int n, const double* in, double* out);
int  orc_hc2r(int n, const double* in, double* out);

#ifdef __cplusplus
}
#endif
#endif
