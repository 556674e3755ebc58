// kernels.cuh -- host-side launchers of the hot-path kernels.
#pragma once
#include "common.cuh"

namespace ptc {

// device pointers of the fields of one context (padded layout, see common.cuh)
struct Fields {
    double *ux, *uy, *uz, *pr, *sc;   // state (sc may be null)
    double *hx, *hy, *hz, *hc;        // explicit history HistX/Y/Z/C
    double *rx, *ry, *rz, *rc;        // right-hand sides of the Helmholtz solves
};

// k_stencil.cu
size_t cell_grid_blocks(const DConst& c);
void launch_coef(cudaStream_t st, DCoef* coef, int ns, double gam, double the, double alp, double xnu, double sdiff);
void launch_rhs(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f, double* part);
void launch_flowrate(cudaStream_t st, const DConst& c, DCoef* coef, const double* part, int nparts);
void launch_prsrc(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int unit_scale,
                  const Fields& f, double* src, double* part, double* out_max);
void launch_project(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int mode, const double* phi,
                    const Fields& f, const double* uy_ym);
void launch_bc_all(cudaStream_t st, const DConst& c, const Fields& f, const double* uy_ym);
void launch_update_uy_ym(cudaStream_t st, int n, double* uy_ym, double* duy_ym);
void launch_cfl(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, DCoef* coef, double* part);
void launch_check(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, const DCoef* coef, DDiag* diag,
                  double* part);

// k_tridiag.cu
int tridiag_partitions(int ny);
bool tridiag_supported(int ny);
void tridiag_init();
void launch_helm(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f,
                 const double* duy_ym, const double* uy_ym);
void launch_helm_scalar(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f);
void launch_ysolve(cudaStream_t st, const DConst& c, const DMetric& m, double2* spec);

// k_fft.cu
void fft_init();
size_t fft_smem_need(int nx, int nz);
void launch_fft_x_r2c(cudaStream_t st, int nx, int nrows, const double* src, double2* spec, const FftPlan& pl,
                      const double2* tw, const double2* post);
void launch_fft_z(cudaStream_t st, int dir, int nx, int ny, int nz, double2* spec, const FftPlan& pl, const double2* tw);
void launch_fft_x_c2r(cudaStream_t st, int nx, int ny, int nrows, const double2* spec, double* phi, const FftPlan& pl,
                      const double2* tw, const double2* post, double scale, int padded);

}  // namespace ptc
