// kernels.cuh -- host-side launchers of the hot-path kernels.
#pragma once
#include <utility>

#include "common.cuh"

namespace ptc {

// true unless the environment sets PARATC_NO_PDL (read once)
bool pdl_enabled();

// launch with programmatic stream serialization, so that the kernel's CTAs
// can be scheduled while the previous kernel in the stream drains; the
// kernel itself calls pdl_wait() before touching data of earlier kernels
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// device pointers of the fields of one context (padded layout, see
// common.cuh), in storage type V: double for the FP64 forms, float for the
// FP32 storage form.  The pressure, which accumulates the potential of every
// substep, is FP64 in every form.
template <class V>
struct FieldSet {
    V *ux, *uy, *uz;          // velocity state
    double* pr;               // pressure
    V* sc;                    // scalar (may be null)
    V *hx, *hy, *hz, *hc;     // explicit history HistX/Y/Z/C
    V *rx, *ry, *rz, *rc;     // right-hand sides of the Helmholtz solves
};
using Fields = FieldSet<double>;
using Fields32 = FieldSet<float>;

// k_stencil.cu (each for the FP64 fields and for the FP32 storage form)
size_t cell_grid_blocks(const DConst& c);
void launch_prsrc(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int unit_scale,
                  const Fields& f, double* src, double* part, double* out_max);
void launch_prsrc(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int unit_scale,
                  const Fields32& f, double* src, double* part, double* out_max);
void launch_project(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int mode, const double* phi,
                    const Fields& f, const double* uy_ym);
void launch_project(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int mode, const float* phi,
                    const Fields32& f, const double* uy_ym);
void launch_bc_all(cudaStream_t st, const DConst& c, const Fields& f, const double* uy_ym);
void launch_bc_all(cudaStream_t st, const DConst& c, const Fields32& f, const double* uy_ym);
void launch_update_uy_ym(cudaStream_t st, int n, double* uy_ym, double* duy_ym);
void launch_cfl(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, DCoef* coef, double* part);
void launch_cfl(cudaStream_t st, const DConst& c, const DMetric& m, const Fields32& f, DCoef* coef, double* part);
size_t endstep_blocks(const DConst& c);
void launch_endstep(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, DCoef* coef, DDiag* diag,
                    double* part, unsigned int* counter, int next);
void launch_endstep(cudaStream_t st, const DConst& c, const DMetric& m, const Fields32& f, DCoef* coef, DDiag* diag,
                    double* part, unsigned int* counter, int next);
// storage conversions (FP32 storage form)
void launch_cast(cudaStream_t st, size_t n, const double* a, float* b);
void launch_cast(cudaStream_t st, size_t n, const float* a, double* b);
// r = src - L phi (compact arrays) without the pinned kx = kz = 0 equation of
// row 1, max|r| and max|src| to out[0..1], the row-1 plane means of r and phi
// to out[2..3]; part holds 4 doubles per cell block
void launch_residual(cudaStream_t st, const DConst& c, const DMetric& m, const double* src, const double* phi,
                     double* r, double* part, unsigned int* counter, double* out);
// x profile of a padded field averaged over y (dyp weights) and z; part holds nx*nz doubles
void launch_xprofile(cudaStream_t st, const DConst& c, const DMetric& m, const double* q, double* part, double* out);
void launch_xprofile(cudaStream_t st, const DConst& c, const DMetric& m, const float* q, double* part, double* out);

// k_rhs.cu
size_t rhs_grid_blocks(const DConst& c);
void rhs_init();
void launch_rhs_tile(cudaStream_t st, const DConst& c, const DMetric& m, DCoef* coef, const Fields& f, double* uy_ym,
                     double* duy_ym, int ns, double gam, double the, double alp, double* part, unsigned int* counter);
// FP32 storage form: float fields, FP64 pressure, FP32 arithmetic
void launch_rhs_tile(cudaStream_t st, const DConst& c, const DMetric& m, DCoef* coef, const Fields32& f, double* uy_ym,
                     double* duy_ym, int ns, double gam, double the, double alp, double* part, unsigned int* counter);

// k_tridiag.cu
int tridiag_partitions(int ny);
bool tridiag_supported(int ny);
void tridiag_init();
int tridiag_part_len(int ny);
size_t helm_fac_doubles(int ny);
int helm_variants();  // compiled Helmholtz launch shapes (DConst::helm_var < helm_variants())
int helm_variants(int prec);  // the shapes of precision form prec: FP64 and mixed 2, FP32 storage 3 (float sweeps)
int rhs_variants();          // compiled FP64 right-hand-side launch shapes (DConst::rhs_var < rhs_variants())
int rhs_variants(int prec);  // the shapes of precision form prec (PARATC_PREC_*): FP64 3, FP32 storage 2, mixed 1
void launch_helm_factors(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int ns0, int nsub,
                         const double* alp, double* fac);
void launch_helm(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields& f, const double* duy_ym,
                 const double* uy_ym, const double* fac);
void launch_helm(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields32& f, const double* duy_ym,
                 const double* uy_ym, const double* fac);
void launch_helm_scalar(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields& f, const double* fac);
void launch_helm_scalar(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields32& f, const double* fac);
void launch_ysolve(cudaStream_t st, const DConst& c, const DMetric& m, double2* spec);

// k_tridiag.cu: spectral y-solve with the pivots computed once per context
void launch_pois_factors(cudaStream_t st, const DConst& c, const DMetric& m, double* fac);
// a z-slab rank's x-mode slab (dc_here: its column 0 is kx = kz = 0)
void launch_pois_factors_slab(cudaStream_t st, const DConst& c, const DMetric& m, double* fac, int dc_here);
void launch_ysolve_fac_slab(cudaStream_t st, const DConst& c, const DMetric& m, double2* spec, const double* fac,
                            int dc_here);
void launch_ysolve_fac(cudaStream_t st, const DConst& c, const DMetric& m, double2* spec, const double* fac);
// FP32 storage form: the streaming solve on a float2 spectrum, FP64 sweeps and pivots
void launch_ysolve_fac(cudaStream_t st, const DConst& c, const DMetric& m, float2* spec, const double* fac);

// k_stats.cu: clcStat accumulation
int stats_count(const DConst& c);
int stats_splits(const DConst& c);
size_t stats_part_doubles(const DConst& c);
void launch_stats(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, const DCoef* coef,
                  double* part, double* sumstat, double* prgradsum);

// k_spectra.cu: clcStat's 1-D spectra (energy, cospectra, linear coherence)
bool spectra_supported(int n);
int spectra_count(const DConst& c);
int spectra_splits(const DConst& c, int axis);
size_t spectra_part_doubles(const DConst& c);
void spectra_init();
void launch_spectra(cudaStream_t st, int axis, const DConst& c, const Fields& f, int jlcs, const double2* tw,
                    double* part, double* out);
void launch_spectra2d(cudaStream_t st, const DConst& c, const Fields& f, const int2* fj, int nfj, int nsel, int nmir,
                      int nfld, const double2* twx, const double2* twz, double* S, double* out);

// k_visu.cu: the quantities of dump_visu at the kept points
int visu_count(int n, int skip);
void launch_visu(cudaStream_t st, int q, int iskip, int jskip, int kskip, int node, const DConst& c, const DMetric& m,
                 const Fields& f, double* out, unsigned int* nbad);

// k_pfft_zt.cu: z transforms fed by TMA (persistent CTAs, two stages)
bool zt_tma_supported(int nz);
void zt_tma_init();
bool zt_tma_prepare(double2* spec, int ncol, int nz, void* tmap_out);
// the FP32 storage form's float2 spectrum (float passes); needs ncol even
bool zt_tma_prepare(float2* spec, int ncol, int nz, void* tmap_out);
void launch_zt_tma32(cudaStream_t st, int dir, int ncol, int nz, const void* tmap, const double2* twz, int nsm,
                     unsigned int* err);
void launch_zt_tma(cudaStream_t st, int dir, int ncol, int nz, const void* tmap, const double2* twz, int nsm,
                   unsigned int* err);

// k_pfft_xt.cu: x transforms fed by bulk copies (persistent CTAs, two stages);
// row pointers must be 16-byte aligned
bool xt_tma_supported(int n);
// the x-slabs of the ranks of a z-slab decomposition (device addresses,
// mapped here where they are other GPUs' memory), this rank's first plane
struct XtGather {
    const double2* p[64];
    int G, k0;
};
// the inverse x transform of this rank's planes, its spectrum rows gathered
// from the x-slabs (compact phi rows)
void launch_xb_tma_gather(cudaStream_t st, int nx, int ny, int nz, const XtGather& gt, double* phi, const double2* twx,
                          const double2* post, double scale, int nsm, unsigned int* err);
// the forward x transform of this rank's planes (compact source rows), every
// mode stored into its owner's x-slab
void launch_xf_tma_scatter(cudaStream_t st, int nx, int ny, int nz, const double* src, const XtGather& gt,
                           const double2* twx, const double2* post, int nsm, unsigned int* err);
void xt_tma_init();
void launch_xb_tma(cudaStream_t st, int nx, int ny, int nz, const double2* spec, double* phi, const double2* twx,
                   const double2* post, double scale, int padded, int nsm, unsigned int* err);
void launch_xf_tma(cudaStream_t st, int nx, int ny, int nz, const double* src, double2* spec, const double2* twx,
                   const double2* post, int nsm, unsigned int* err);
// FP32 storage form: float2 spectrum rows in (two per bulk copy), float phi out
void launch_xb_tma(cudaStream_t st, int nx, int ny, int nz, const float2* spec, float* phi, const double2* twx,
                   const double2* post, double scale, int padded, int nsm, unsigned int* err);
// the divergence source of clcPrSrc (mode 0: / pmAlpha, 1: unscaled) and its
// forward x transform, warp-specialised (one CTA per SM; grid records to part)
int xf_div_grid(int n, int nrows, int nsm);
void launch_xf_div(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f,
                   double2* spec, const double2* twx, const double2* post, double* part, unsigned int* counter,
                   double* out_max, unsigned int* err);
// FP32 storage form: float velocity in, float2 spectrum rows out
void launch_xf_div(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                   const Fields32& f, float2* spec, const double2* twx, const double2* post, double* part,
                   unsigned int* counter, double* out_max, unsigned int* err);

// k_plane.cu: both transforms of a y-plane in one CTA (planes that fit shared memory)
bool plane_supported(int nx, int nz);
void plane_init();
void launch_plane_f(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f,
                    const double* src, double2* spec, const double2* twx, const double2* post, const double2* twz,
                    double* part, unsigned int* counter, double* out_max);
void launch_plane_b(cudaStream_t st, int nx, int ny, int nz, const double2* spec, double* phi, const double2* twx,
                    const double2* post, const double2* twz, double scale, int padded);
void plane_init32();  // the FP32 storage instantiations (k_plane32.cu)
// FP32 storage form: the step's solve and the refined solve (as launch_pfft_xf / _xb)
void launch_plane_f(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                    const Fields32& f, const double* src, float2* spec, const double2* twx, const double2* post,
                    const double2* twz, double* part, unsigned int* counter, double* out_max);
void launch_plane_f(cudaStream_t st, const DConst& c, const double* src, float2* spec, const double2* twx,
                    const double2* post, const double2* twz);
void launch_plane_b(cudaStream_t st, int nx, int ny, int nz, const float2* spec, float* phi, const double2* twx,
                    const double2* post, const double2* twz, double scale, int padded);
void launch_plane_b(cudaStream_t st, int nx, int ny, int nz, const float2* spec, double* phi, const double2* twx,
                    const double2* post, const double2* twz, double scale, int accumulate, const double* shift);

// k_pfft_x.cu / k_pfft_z.cu: compile-time-length transforms of the Poisson solve
bool pfft_x_supported(int n);
bool pfft_z_supported(int n);
int pfft_x_blocks(int nx, int ny, int nz);
void pfft_x_init();
void pfft_x_init32();  // the FP32 storage instantiations (k_pfft_x32.cu)
void pfft_z_init();
void launch_pfft_xf(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f,
                    const double* src, double2* spec, const double2* twx, const double2* post, double* part,
                    unsigned int* counter, double* out_max);
void launch_pfft_xb(cudaStream_t st, int nx, int ny, int nz, const double2* spec, double* phi, const double2* twx,
                    const double2* post, double scale, int padded);
void launch_pfft_z(cudaStream_t st, int dir, int nx, int ny, int nz, double2* spec, const double2* twz);
// FP32 storage form: the step's solve (float velocity, float2 spectrum, float potential)
void launch_pfft_xf(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                    const Fields32& f, const double* src, float2* spec, const double2* twx, const double2* post,
                    double* part, unsigned int* counter, double* out_max);
void launch_pfft_xb(cudaStream_t st, int nx, int ny, int nz, const float2* spec, float* phi, const double2* twx,
                    const double2* post, double scale, int padded);
// f32arith: the passes in float (the FP32 storage form's step), else in
// double (the refined solve)
void launch_pfft_z(cudaStream_t st, int dir, int nx, int ny, int nz, float2* spec, const double2* twz, int f32arith);
// the refined solve: an FP64 source array into a float2 spectrum, and the
// inverse into an FP64 potential (compact rows), added to it when accumulate != 0
void launch_pfft_xf(cudaStream_t st, const DConst& c, const double* src, float2* spec, const double2* twx,
                    const double2* post);
void launch_pfft_xb(cudaStream_t st, int nx, int ny, int nz, const float2* spec, double* phi, const double2* twx,
                    const double2* post, double scale, int accumulate, const double* shift);

// ---- grouped launches over the members of an ensemble.  One launch runs
// one kernel instantiation for every member of a table (GrpTab in
// common.cuh): member i's CTAs take its own launch shape (the *_member_grid
// functions, the same shape its own launch has) on its own fields, so each
// member computes exactly what its own launches compute.  Argument records:
template <class V>
struct RhsArgs {  // k_rhs_tile
    DConst c;
    DMetric m;
    DCoef* coef;
    FieldSet<V> fl;
    double *uy_ym, *duy_ym;
    double gam, the, alp;  // the substep's RK3 coefficients
    double* part;
    unsigned int* counter;
    int nlog;  // blocks of the member's own launch (its flow-rate records)
    int pad;
};
template <class V>
struct HelmArgs {  // k_helm, components comp0 .. comp0 + grid z - 1
    DConst c;
    const DCoef* coef;
    FieldSet<V> fl;
    const double *duy_ym, *uy_ym, *fac;
    int comp0;
};
template <class V, class S>
struct XfArgs {  // k_xf, divergence source of the substep (mode 0)
    DConst c;
    DMetric m;
    const DCoef* coef;
    const V *ux, *uy, *uz;
    S* spec;
    const double2 *tw, *post;
    double* part;
    unsigned int* counter;
    double* out_max;
};
template <class S>
struct ZtArgs {  // k_zt
    int ncol;
    S* spec;
    const double2* tw;
};
template <class S>
struct YsArgs {  // k_ys_staged / k_ys_global
    int ny, M1, nz;
    const double* am2ph;
    S* spec;
    const double* fac;
};
template <class S, class PH>
struct XbArgs {  // k_xb into the padded potential
    int ny, nz;
    const S* spec;
    PH* phi;
    const double2 *tw, *post;
    double scale;
};
template <class V>
struct ProjArgs {  // k_project, substep mode
    DConst c;
    DMetric m;
    const DCoef* coef;
    const V* phi;
    V *ux, *uy, *uz;
    double* pr;
    const double* uy_ym;
};
template <class V>
struct EndArgs {  // k_endstep with the next step's clcCFL
    DConst c;
    DMetric m;
    const V *ux, *uy, *uz, *sc;
    DCoef* coef;
    DDiag* diag;
    double* part;
    unsigned int* counter;
};

// key: the member whose DConst selects the instantiation (scalar_on,
// fp32_rhs, rhs_var, helm_var, nx, nz, ...); nblk: the table's total CTAs
dim3 rhs_member_grid(const DConst& c, int f32arith);
long long rhs_work_rows(const DConst& c);  // (tile, row) work items of the right-hand side
int rhs_wave(const DConst& c);             // resident right-hand-side CTAs of the device
void launch_rhs_grp(cudaStream_t st, const DConst& key, const GrpTab<RhsArgs<double>>* t, int nblk, int ns);
void launch_rhs_grp(cudaStream_t st, const DConst& key, const GrpTab<RhsArgs<float>>* t, int nblk, int ns);
dim3 helm_member_grid(const DConst& c, int ncomp);
size_t helm_smem(const DConst& c);
void launch_helm_grp(cudaStream_t st, const DConst& key, const GrpTab<HelmArgs<double>>* t, int nblk, size_t smem);
void launch_helm_grp(cudaStream_t st, const DConst& key, const GrpTab<HelmArgs<float>>* t, int nblk, size_t smem);
// the y-solve: kind 0 staged, 1 streaming (ys_kind), per member
int ys_kind(const DConst& c);
dim3 ys_member_grid(const DConst& c, int kind);
size_t ys_smem(const DConst& c, int kind);
void launch_ys_grp(cudaStream_t st, int kind, const GrpTab<YsArgs<double2>>* t, int nblk, size_t smem);
void launch_ys_grp(cudaStream_t st, int kind, const GrpTab<YsArgs<float2>>* t, int nblk, size_t smem);
dim3 pfft_x_member_grid(const DConst& c);
void launch_xf_grp(cudaStream_t st, int nx, const GrpTab<XfArgs<double, double2>>* t, int nblk);
void launch_xf_grp(cudaStream_t st, int nx, const GrpTab<XfArgs<float, float2>>* t, int nblk);
void launch_xb_grp(cudaStream_t st, int nx, const GrpTab<XbArgs<double2, double>>* t, int nblk);
void launch_xb_grp(cudaStream_t st, int nx, const GrpTab<XbArgs<float2, float>>* t, int nblk);
dim3 pfft_z_member_grid(const DConst& c);
void launch_zt_grp(cudaStream_t st, int dir, int nz, const GrpTab<ZtArgs<double2>>* t, int nblk);
void launch_zt_grp(cudaStream_t st, int dir, int nz, const GrpTab<ZtArgs<float2>>* t, int nblk);
dim3 cell_member_grid(const DConst& c);
void launch_project_grp(cudaStream_t st, const GrpTab<ProjArgs<double>>* t, int nblk);
void launch_project_grp(cudaStream_t st, const GrpTab<ProjArgs<float>>* t, int nblk);
dim3 endstep_member_grid(const DConst& c);
void launch_endstep_grp(cudaStream_t st, const GrpTab<EndArgs<double>>* t, int nblk);
void launch_endstep_grp(cudaStream_t st, const GrpTab<EndArgs<float>>* t, int nblk);

// k_fft.cu
void fft_init();
size_t fft_smem_need(int nx, int nz);
void launch_fft_x_r2c(cudaStream_t st, int nx, int nrows, const double* src, double2* spec, const FftPlan& pl,
                      const double2* tw, const double2* post);
void launch_fft_z(cudaStream_t st, int dir, int nx, int ny, int nz, double2* spec, const FftPlan& pl, const double2* tw);
void launch_fft_x_c2r(cudaStream_t st, int nx, int ny, int nrows, const double2* spec, double* phi, const FftPlan& pl,
                      const double2* tw, const double2* post, double scale, int padded);

}  // namespace ptc
