// api.cu -- paratc_ctx and the C ABI of include/paratc.h.
//
// A context is the B200 counterpart of one ParaTC rank's module state
// (m_Variables, m_MeshAndMetries, m_Poisson, m_Parameters): all fields live in
// HBM for the life of the context, one CUDA stream orders every kernel, and a
// step is enqueued as the fixed kernel sequence of ChannelIterate
// (src/m_ChannelSystem.f90:80-187) with dt, the RK coefficients and the
// guards kept on the device, so a step needs no host round trip until its
// diagnostics are read.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/paratc.h"
#include "common.cuh"
#include "host_setup.h"
#include "kernels.cuh"

using namespace ptc;

bool ptc::pdl_enabled() {
    static const bool on = std::getenv("PARATC_NO_PDL") == nullptr;
    return on;
}

// kernel classes of the per-kernel timer
enum ProfK {
    PK_COEF = 0, PK_UYYM, PK_RHS, PK_FLOWRATE, PK_HELM, PK_HELM_SC, PK_PRSRC, PK_FFTX_F, PK_FFTZ_F, PK_YSOLVE,
    PK_FFTZ_B, PK_FFTX_B, PK_PROJECT, PK_CFL, PK_CHECK, PK_BC
};
static const char* kProfNames[PARATC_PROF_NKERNELS] = {
    "helm_factors", "uy_ym", "rhs", "flowrate", "helmholtz", "helmholtz_scalar", "prsrc", "fft_x_fwd", "fft_z_fwd",
    "ysolve", "fft_z_bwd", "fft_x_bwd", "project", "cfl", "check", "bc"};

struct paratc_ctx {
    paratc_params prm;
    int dev = 0;
    cudaStream_t st = nullptr;
    int nx = 0, ny = 0, nz = 0, nyp = 0, nyt = 0, M1 = 0;
    size_t nf = 0, ni = 0, npart = 0;
    HostMetrics hm;
    DConst kc;
    DMetric dm;
    FftPlan plx, plz;
    Fields f;
    int prec = PARATC_PREC_FP64;  // PARATC_PREC_FP64 / _MIXED / _FP32
    int tune_from_cache = 0;      // the launch shapes and schedule came from the tuning cache
    double tune_step_ms = 0.0;    // ms per step of the tuned combination (0: not timed here)
    Fields32 f32{};               // float fields of the FP32 storage form (pr = f.pr), allocated on first use
    float* d_phi32 = nullptr;     // its potential (padded)
    std::vector<void*> allocs;
    double *d_src = nullptr, *d_phi = nullptr, *d_part = nullptr, *d_uy_ym = nullptr, *d_duy_ym = nullptr;
    double *d_metric = nullptr, *d_scal = nullptr;
    double2 *d_spec = nullptr, *d_twx = nullptr, *d_postx = nullptr, *d_twz = nullptr;
    bool pfft = false;   // compile-time-length transforms exist for nx/2 and nz
    bool plane = false;  // a whole y-plane of the spectrum fits one CTA: fused 2-D transforms
    bool ztma = false;   // z transforms through the TMA-fed persistent kernel (split path)
    bool ztma_ok = false;  // its tensor map is encoded (nz supported, driver entry point found)
    bool xtma = false;     // x transforms through the bulk-copy-fed persistent kernels (split path)
    bool xdiv = false;     // the divergence source by producer warps of the forward x transform
    alignas(64) unsigned char zt_tmap[128];  // its tensor map (a CUtensorMap)
    alignas(64) unsigned char zt_tmap32[128];  // the same over the float2 spectrum of the FP32 storage form
    bool ztma32_ok = false;                    // that map is encoded (ncol even, nz supported)
    unsigned int* d_zt_err = nullptr;        // set by a TMA-fed kernel whose bounded wait ran out
    int sched_gen = 0;   // bumped whenever the Poisson schedule changes (captured graphs hold the old one)
    double* d_pfac = nullptr;   // pivots of the spectral y systems (1/vecm, then arr), computed once
    DCoef* d_coef = nullptr;
    DDiag* d_diag = nullptr;
    DDiag* d_diag2 = nullptr;
    unsigned int* d_counter = nullptr;  // grid-completion counters of the last-block reductions
    double* d_hfac = nullptr;           // Helmholtz pivots of the substeps of a step (3 matrix types each)
    double hfac_dt = -1.0;              // the fixed dt d_hfac holds pivots for (iCFL != 1), else < 0
    bool next_ready = false;            // the last step's end kernel already computed this step's dt
    double* d_stats = nullptr;          // SumStat [nyp][nstat] then PrGradsum (FP64 accumulators)
    double* d_stats_part = nullptr;     // per-slice partial sums of clcStat
    int nfstime = 0;                    // statistics steps accumulated
    double* d_specx = nullptr;          // 1-D spectra accumulators [nsp][ny][nx/2+1], [nsp][ny][nz/2+1]
    double* d_specz = nullptr;          //   (created on first use)
    double* d_spec_part = nullptr;      // per-slice partial records of the spectra kernels
    double2* d_twxf = nullptr;          // exp(-2 pi i m / nx), m < nx (full-length x transforms)
    int nspectime = 0;                  // spectra samples accumulated
    double* d_spec2d = nullptr;         // 2-D spectra accumulators [nsp2][nz][nsel][nx]
    double* d_s2 = nullptr;             // hc-hc transforms of the listed (field, row) pairs
    int2* d_fj = nullptr;               // the (field, row) pairs
    int nsel2 = 0, nfj2 = 0, nmir2 = 0, nfld2 = 0;
    size_t spec2d_cap = 0, s2_cap = 0, fj_cap = 0;  // capacities of the three buffers (elements)
    int nspectime2 = 0;                 // 2-D spectra samples accumulated
    double* d_visu = nullptr;           // one visu quantity at the kept points (nx*ny*nz doubles, first use)
    unsigned int* d_visu_bad = nullptr; // lambda2 points with complex roots
    DDiag* h_diag = nullptr;   // pinned
    DCoef* h_coef = nullptr;   // pinned
    DCoef* h_coef0 = nullptr;  // pinned, the coefficient block of a freshly loaded state (never rewritten)
    double* h_scal = nullptr;  // pinned
    std::string err;
    int64_t launches = 0;
    // per-kernel timer
    bool prof_on = false;
    std::vector<cudaEvent_t> ev;          // pool, pairs (2q, 2q+1)
    std::vector<int> ev_class;            // class of pending pair q
    int ev_used = 0;
    double prof_ms[PARATC_PROF_NKERNELS] = {0};
    int64_t prof_n[PARATC_PROF_NKERNELS] = {0};
};

// tuning cache (defined with paratc_autotune_all)
static std::string tune_key(const paratc_ctx* ctx);
static bool tune_cache_read(const char* path, const std::string& key, paratc_tuning* t);
static bool tuning_valid(const paratc_ctx* ctx, const paratc_tuning& t);
static void tuning_apply(paratc_ctx* ctx, const paratc_tuning& t);

namespace {

void prof_flush(paratc_ctx* ctx);

// brackets one launch with a pair of events when the timer is on
struct ProfScope {
    paratc_ctx* ctx;
    int q = -1;
    ProfScope(paratc_ctx* c, int cls) : ctx(c) {
        if (!ctx->prof_on) return;
        if (ctx->ev_used * 2 + 2 > (int)ctx->ev.size()) prof_flush(ctx);
        q = ctx->ev_used++;
        ctx->ev_class[q] = cls;
        cudaEventRecord(ctx->ev[2 * q], ctx->st);
    }
    ~ProfScope() {
        if (q >= 0) cudaEventRecord(ctx->ev[2 * q + 1], ctx->st);
    }
};
#define PT_CAT2(a, b) a##b
#define PT_CAT(a, b) PT_CAT2(a, b)
#define PROF(cls) ProfScope PT_CAT(prof_scope_, __LINE__)(ctx, cls)

void prof_flush(paratc_ctx* ctx) {
    if (ctx->ev_used == 0) return;
    cudaStreamSynchronize(ctx->st);
    for (int q = 0; q < ctx->ev_used; q++) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev[2 * q], ctx->ev[2 * q + 1]) == cudaSuccess) {
            ctx->prof_ms[ctx->ev_class[q]] += ms;
            ctx->prof_n[ctx->ev_class[q]] += 1;
        }
    }
    ctx->ev_used = 0;
}

int set_err(paratc_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_err(ctx, PARATC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// releases a buffer from dalloc before its context ends (a buffer that grows)
template <class T>
void dfree(paratc_ctx* ctx, T** p) {
    if (!*p) return;
    for (size_t a = 0; a < ctx->allocs.size(); a++)
        if (ctx->allocs[a] == (void*)*p) {
            cudaFree(ctx->allocs[a]);
            ctx->allocs.erase(ctx->allocs.begin() + (long)a);
            break;
        }
    *p = nullptr;
}

template <class T>
int dalloc(paratc_ctx* ctx, T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T) + 256);
    if (e != cudaSuccess) return set_err(ctx, PARATC_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    ctx->allocs.push_back(q);
    cudaMemsetAsync(q, 0, n * sizeof(T) + 256, ctx->st);
    *p = (T*)q;
    return PARATC_OK;
}

int make_plan(int n, FftPlan& pl) {
    pl.n = n;
    pl.nr = 0;
    int m = n;
    while (m % 4 == 0 && pl.nr < PT_MAX_RADIX_PASSES) { pl.rad[pl.nr++] = 4; m /= 4; }
    while (m % 2 == 0 && pl.nr < PT_MAX_RADIX_PASSES) { pl.rad[pl.nr++] = 2; m /= 2; }
    while (m % 3 == 0 && pl.nr < PT_MAX_RADIX_PASSES) { pl.rad[pl.nr++] = 3; m /= 3; }
    while (m % 5 == 0 && pl.nr < PT_MAX_RADIX_PASSES) { pl.rad[pl.nr++] = 5; m /= 5; }
    pl.code = 0;
    for (int s = 0; s < pl.nr && s < 16; s++) pl.code |= (unsigned long long)pl.rad[s] << (4 * s);
    return (m == 1 && pl.nr <= 16) ? PARATC_OK : PARATC_ERR_BAD_ARG;
}

std::vector<double2> twiddles(int n, int count) {
    std::vector<double2> w(count);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < count; k++) {
        long double a = -2.0L * pi * (long double)k / (long double)n;
        w[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    return w;
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// the z transforms, the y-solve and the x inverse, after the forward x
// transform has filled d_spec
void enqueue_poisson_tail(paratc_ctx* ctx, double* out, int padded) {
    cudaStream_t st = ctx->st;
    if (ctx->plane) {
        { PROF(PK_YSOLVE); launch_ysolve_fac(st, ctx->kc, ctx->dm, ctx->d_spec, ctx->d_pfac); }
        { PROF(PK_FFTX_B); launch_plane_b(st, ctx->nx, ctx->ny, ctx->nz, ctx->d_spec, out, ctx->d_twx, ctx->d_postx,
                                          ctx->d_twz, ctx->hm.normfft, padded); }
        ctx->launches += 2;
        return;
    }
    if (ctx->pfft) {
        const int ncol = ctx->ny * (ctx->nx / 2 + 1);
        if (ctx->ztma) { PROF(PK_FFTZ_F); launch_zt_tma(st, -1, ncol, ctx->nz, ctx->zt_tmap, ctx->d_twz, ctx->kc.nsm, ctx->d_zt_err); }
        else { PROF(PK_FFTZ_F); launch_pfft_z(st, -1, ctx->nx, ctx->ny, ctx->nz, ctx->d_spec, ctx->d_twz); }
        { PROF(PK_YSOLVE); launch_ysolve_fac(st, ctx->kc, ctx->dm, ctx->d_spec, ctx->d_pfac); }
        if (ctx->ztma) { PROF(PK_FFTZ_B); launch_zt_tma(st, +1, ncol, ctx->nz, ctx->zt_tmap, ctx->d_twz, ctx->kc.nsm, ctx->d_zt_err); }
        else { PROF(PK_FFTZ_B); launch_pfft_z(st, +1, ctx->nx, ctx->ny, ctx->nz, ctx->d_spec, ctx->d_twz); }
        if (ctx->xtma && aligned16(out)) {
            PROF(PK_FFTX_B);
            launch_xb_tma(st, ctx->nx, ctx->ny, ctx->nz, ctx->d_spec, out, ctx->d_twx, ctx->d_postx, ctx->hm.normfft,
                          padded, ctx->kc.nsm, ctx->d_zt_err);
        } else {
            PROF(PK_FFTX_B);
            launch_pfft_xb(st, ctx->nx, ctx->ny, ctx->nz, ctx->d_spec, out, ctx->d_twx, ctx->d_postx, ctx->hm.normfft,
                           padded);
        }
    } else {
        const int nrows = ctx->ny * ctx->nz;
        { PROF(PK_FFTZ_F); launch_fft_z(st, -1, ctx->nx, ctx->ny, ctx->nz, ctx->d_spec, ctx->plz, ctx->d_twz); }
        { PROF(PK_YSOLVE); launch_ysolve_fac(st, ctx->kc, ctx->dm, ctx->d_spec, ctx->d_pfac); }
        { PROF(PK_FFTZ_B); launch_fft_z(st, +1, ctx->nx, ctx->ny, ctx->nz, ctx->d_spec, ctx->plz, ctx->d_twz); }
        { PROF(PK_FFTX_B); launch_fft_x_c2r(st, ctx->nx, ctx->ny, nrows, ctx->d_spec, out, ctx->plx, ctx->d_twx,
                                             ctx->d_postx, ctx->hm.normfft, padded); }
    }
    ctx->launches += 4;
}

// forward x transform of the source; mode 0: divergence of u* / pmAlpha
// (clcPrSrc, max|div| to out_max), 1: unscaled divergence, 2: array src
void enqueue_poisson_head(paratc_ctx* ctx, int mode, const double* src, double* out_max) {
    cudaStream_t st = ctx->st;
    if (ctx->plane) {
        PROF(mode == 2 ? PK_FFTX_F : PK_PRSRC);
        launch_plane_f(st, mode, ctx->kc, ctx->dm, ctx->d_coef, ctx->f, src, ctx->d_spec, ctx->d_twx, ctx->d_postx,
                       ctx->d_twz, ctx->d_part, ctx->d_counter + 1, out_max);
        ctx->launches += 1;
        return;
    }
    if (ctx->pfft && mode == 2 && ctx->xtma && aligned16(src)) {
        PROF(PK_FFTX_F);
        launch_xf_tma(st, ctx->nx, ctx->ny, ctx->nz, src, ctx->d_spec, ctx->d_twx, ctx->d_postx, ctx->kc.nsm,
                      ctx->d_zt_err);
        ctx->launches += 1;
        return;
    }
    if (ctx->pfft && mode != 2 && ctx->xdiv) {
        PROF(PK_PRSRC);
        launch_xf_div(st, mode, ctx->kc, ctx->dm, ctx->d_coef, ctx->f, ctx->d_spec, ctx->d_twx, ctx->d_postx,
                      ctx->d_part, ctx->d_counter + 1, out_max, ctx->d_zt_err);
        ctx->launches += 1;
        return;
    }
    if (ctx->pfft) {
        PROF(mode == 2 ? PK_FFTX_F : PK_PRSRC);
        launch_pfft_xf(st, mode, ctx->kc, ctx->dm, ctx->d_coef, ctx->f, src, ctx->d_spec, ctx->d_twx, ctx->d_postx,
                       ctx->d_part, ctx->d_counter + 1, out_max);
        ctx->launches += 1;
        return;
    }
    if (mode != 2) {
        { PROF(PK_PRSRC); launch_prsrc(st, ctx->kc, ctx->dm, ctx->d_coef, mode, ctx->f, ctx->d_src, ctx->d_part, out_max); }
        ctx->launches += 2;
        src = ctx->d_src;
    }
    { PROF(PK_FFTX_F); launch_fft_x_r2c(st, ctx->nx, ctx->ny * ctx->nz, src, ctx->d_spec, ctx->plx, ctx->d_twx, ctx->d_postx); }
    ctx->launches += 1;
}

void enqueue_poisson(paratc_ctx* ctx, const double* src, double* out, int padded) {
    enqueue_poisson_head(ctx, 2, src, nullptr);
    enqueue_poisson_tail(ctx, out, padded);
}

// ---- the FP32 storage form: the same solve on a float2 spectrum (the
// passes compute in double) with the compile-time-length transforms, one CTA
// per plane where the plane fits, else the separate x and z kernels
float2* spec32(paratc_ctx* ctx) { return reinterpret_cast<float2*>(ctx->d_spec); }

// forward transform of the divergence of the float velocity (mode 0:
// clcPrSrc's source / pmAlpha, max|div| to out_max; 1: unscaled)
void enqueue_poisson_head32(paratc_ctx* ctx, int mode, double* out_max) {
    cudaStream_t st = ctx->st;
    PROF(PK_PRSRC);
    if (ctx->plane)
        launch_plane_f(st, mode, ctx->kc, ctx->dm, ctx->d_coef, ctx->f32, nullptr, spec32(ctx), ctx->d_twx,
                       ctx->d_postx, ctx->d_twz, ctx->d_part, ctx->d_counter + 1, out_max);
    else if (ctx->xdiv)
        launch_xf_div(st, mode, ctx->kc, ctx->dm, ctx->d_coef, ctx->f32, spec32(ctx), ctx->d_twx, ctx->d_postx,
                      ctx->d_part, ctx->d_counter + 1, out_max, ctx->d_zt_err);
    else
        launch_pfft_xf(st, mode, ctx->kc, ctx->dm, ctx->d_coef, ctx->f32, nullptr, spec32(ctx), ctx->d_twx,
                       ctx->d_postx, ctx->d_part, ctx->d_counter + 1, out_max);
    ctx->launches += 1;
}

void enqueue_poisson_tail32(paratc_ctx* ctx, float* out, int padded) {
    cudaStream_t st = ctx->st;
    if (ctx->plane) {
        { PROF(PK_YSOLVE); launch_ysolve_fac(st, ctx->kc, ctx->dm, spec32(ctx), ctx->d_pfac); }
        { PROF(PK_FFTX_B); launch_plane_b(st, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), out, ctx->d_twx, ctx->d_postx,
                                          ctx->d_twz, ctx->hm.normfft, padded); }
        ctx->launches += 2;
        return;
    }
    const int ncol = ctx->ny * (ctx->nx / 2 + 1);
    const bool zt = ctx->ztma && ctx->ztma32_ok;
    if (zt) { PROF(PK_FFTZ_F); launch_zt_tma32(st, -1, ncol, ctx->nz, ctx->zt_tmap32, ctx->d_twz, ctx->kc.nsm, ctx->d_zt_err); }
    else { PROF(PK_FFTZ_F); launch_pfft_z(st, -1, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), ctx->d_twz, 1); }
    { PROF(PK_YSOLVE); launch_ysolve_fac(st, ctx->kc, ctx->dm, spec32(ctx), ctx->d_pfac); }
    if (zt) { PROF(PK_FFTZ_B); launch_zt_tma32(st, +1, ncol, ctx->nz, ctx->zt_tmap32, ctx->d_twz, ctx->kc.nsm, ctx->d_zt_err); }
    else { PROF(PK_FFTZ_B); launch_pfft_z(st, +1, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), ctx->d_twz, 1); }
    // (the bulk-copy-fed kernel loads the odd-length float2 rows in pairs: an
    // even row count, which every compiled nz gives)
    if (ctx->xtma && aligned16(out) && (ctx->ny * ctx->nz) % 2 == 0) {
        PROF(PK_FFTX_B);
        launch_xb_tma(st, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), out, ctx->d_twx, ctx->d_postx, ctx->hm.normfft,
                      padded, ctx->kc.nsm, ctx->d_zt_err);
    } else {
        PROF(PK_FFTX_B);
        launch_pfft_xb(st, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), out, ctx->d_twx, ctx->d_postx, ctx->hm.normfft,
                       padded);
    }
    ctx->launches += 4;
}

// one solve of the refined standalone Poisson equation: the FP64 array src
// (compact) through a float2 spectrum into the FP64 potential phi (compact),
// written (accumulate = 0) or added to it (the corrections)
// (the correction also subtracts *shift, the row-1 plane mean of phi, from phi)
void enqueue_solve32(paratc_ctx* ctx, const double* src, double* phi, int accumulate, const double* shift) {
    cudaStream_t st = ctx->st;
    if (ctx->plane) {
        { PROF(PK_FFTX_F); launch_plane_f(st, ctx->kc, src, spec32(ctx), ctx->d_twx, ctx->d_postx, ctx->d_twz); }
        { PROF(PK_YSOLVE); launch_ysolve_fac(st, ctx->kc, ctx->dm, spec32(ctx), ctx->d_pfac); }
        { PROF(PK_FFTX_B); launch_plane_b(st, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), phi, ctx->d_twx, ctx->d_postx,
                                          ctx->d_twz, ctx->hm.normfft, accumulate, shift); }
        ctx->launches += 3;
        return;
    }
    { PROF(PK_FFTX_F); launch_pfft_xf(st, ctx->kc, src, spec32(ctx), ctx->d_twx, ctx->d_postx); }
    { PROF(PK_FFTZ_F); launch_pfft_z(st, -1, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), ctx->d_twz, 0); }
    { PROF(PK_YSOLVE); launch_ysolve_fac(st, ctx->kc, ctx->dm, spec32(ctx), ctx->d_pfac); }
    { PROF(PK_FFTZ_B); launch_pfft_z(st, +1, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), ctx->d_twz, 0); }
    { PROF(PK_FFTX_B); launch_pfft_xb(st, ctx->nx, ctx->ny, ctx->nz, spec32(ctx), phi, ctx->d_twx, ctx->d_postx,
                                      ctx->hm.normfft, accumulate, shift); }
    ctx->launches += 5;
}

// the substep of the FP32 storage form: float u, v, w, c, histories,
// right-hand sides, spectrum and potential, FP64 pressure; the right-hand
// side in FP32 arithmetic, the Helmholtz sweeps and the transforms in FP64
// arithmetic, the flow-rate sum and every reduction in FP64
void enqueue_substep32(paratc_ctx* ctx, int ns, int stop) {
    cudaStream_t st = ctx->st;
    const HostMetrics& h = ctx->hm;
    {
        PROF(PK_RHS);
        launch_rhs_tile(st, ctx->kc, ctx->dm, ctx->d_coef, ctx->f32, ctx->d_uy_ym, ctx->d_duy_ym, ns, h.gam[ns - 1],
                        h.the[ns - 1], h.alp[ns - 1], ctx->d_part, ctx->d_counter);
    }
    ctx->launches += 1;
    if (stop == 1) return;
    if (ctx->prm.scalar_on) { PROF(PK_HELM_SC); launch_helm_scalar(st, ctx->kc, ctx->d_coef, ctx->f32, ctx->d_hfac); ctx->launches++; }
    { PROF(PK_HELM); launch_helm(st, ctx->kc, ctx->d_coef, ctx->f32, ctx->d_duy_ym, ctx->d_uy_ym, ctx->d_hfac); }
    ctx->launches += 1;
    if (stop == 2) return;
    if (stop == 3) {
        { PROF(PK_PRSRC); launch_prsrc(st, ctx->kc, ctx->dm, ctx->d_coef, 0, ctx->f32, ctx->d_src, ctx->d_part, &ctx->d_coef->divmax_src); }
        ctx->launches += 2;
        return;
    }
    enqueue_poisson_head32(ctx, 0, &ctx->d_coef->divmax_src);
    enqueue_poisson_tail32(ctx, ctx->d_phi32, 1);
    if (stop == 4) return;
    { PROF(PK_PROJECT); launch_project(st, ctx->kc, ctx->dm, ctx->d_coef, 0, ctx->d_phi32, ctx->f32, ctx->d_uy_ym); }
    ctx->launches += 1;
}

// body of the ns loop of ChannelIterate (src/m_ChannelSystem.f90:102-140),
// optionally stopped after stage `stop` (1 rhs, 2 helmholtz, 3 prsrc, 4 ppe)
void enqueue_substep(paratc_ctx* ctx, int ns, int stop = 5) {
    if (ctx->prec == PARATC_PREC_FP32) {
        enqueue_substep32(ctx, ns, stop);
        return;
    }
    cudaStream_t st = ctx->st;
    const HostMetrics& h = ctx->hm;
    {
        PROF(PK_RHS);
        launch_rhs_tile(st, ctx->kc, ctx->dm, ctx->d_coef, ctx->f, ctx->d_uy_ym, ctx->d_duy_ym, ns, h.gam[ns - 1],
                        h.the[ns - 1], h.alp[ns - 1], ctx->d_part, ctx->d_counter);
    }
    ctx->launches += 1;
    if (stop == 1) return;
    if (ctx->prm.scalar_on) { PROF(PK_HELM_SC); launch_helm_scalar(st, ctx->kc, ctx->d_coef, ctx->f, ctx->d_hfac); ctx->launches++; }
    { PROF(PK_HELM); launch_helm(st, ctx->kc, ctx->d_coef, ctx->f, ctx->d_duy_ym, ctx->d_uy_ym, ctx->d_hfac); }
    ctx->launches += 1;
    if (stop == 2) return;
    if (stop == 3) {
        // the source alone (for a stage-by-stage comparison)
        { PROF(PK_PRSRC); launch_prsrc(st, ctx->kc, ctx->dm, ctx->d_coef, 0, ctx->f, ctx->d_src, ctx->d_part, &ctx->d_coef->divmax_src); }
        ctx->launches += 2;
        return;
    }
    // clcPrSrc fused into the forward x transform
    enqueue_poisson_head(ctx, 0, nullptr, &ctx->d_coef->divmax_src);
    enqueue_poisson_tail(ctx, ctx->d_phi, 1);
    if (stop == 4) return;
    { PROF(PK_PROJECT); launch_project(st, ctx->kc, ctx->dm, ctx->d_coef, 0, ctx->d_phi, ctx->f, ctx->d_uy_ym); }
    ctx->launches += 1;
}

void enqueue_step(paratc_ctx* ctx) {
    // clcCFL: done by the previous step's end kernel unless the state changed since
    const bool fp32 = ctx->prec == PARATC_PREC_FP32;
    if (!ctx->next_ready) {
        PROF(PK_CFL);
        if (fp32) launch_cfl(ctx->st, ctx->kc, ctx->dm, ctx->f32, ctx->d_coef, ctx->d_part);
        else launch_cfl(ctx->st, ctx->kc, ctx->dm, ctx->f, ctx->d_coef, ctx->d_part);
        ctx->launches += 2;
    }
    // with a fixed time step (iCFL != 1) the Helmholtz matrices never change:
    // their pivots are computed once and kept
    if (ctx->prm.icfl == 1 || ctx->hfac_dt != ctx->prm.dt_max) {
        { PROF(PK_COEF); launch_helm_factors(ctx->st, ctx->kc, ctx->dm, ctx->d_coef, 1, ctx->hm.iadvance, ctx->hm.alp, ctx->d_hfac); }
        ctx->launches += 1;
        ctx->hfac_dt = (ctx->prm.icfl == 1) ? -1.0 : ctx->prm.dt_max;
    }
    for (int ns = 1; ns <= ctx->hm.iadvance; ns++) enqueue_substep(ctx, ns);
    {
        PROF(PK_CHECK);
        if (fp32) launch_endstep(ctx->st, ctx->kc, ctx->dm, ctx->f32, ctx->d_coef, ctx->d_diag, ctx->d_part, ctx->d_counter + 3, 1);
        else launch_endstep(ctx->st, ctx->kc, ctx->dm, ctx->f, ctx->d_coef, ctx->d_diag, ctx->d_part, ctx->d_counter + 3, 1);
    }
    ctx->next_ready = true;
    ctx->launches += 1;
}

void diag_out(const DDiag& d, paratc_diag* o) {
    if (!o) return;
    o->dt = d.dt; o->cfl = d.cfl; o->sim_time = d.sim_time; o->divmax_src = d.divmax_src; o->divmax = d.divmax;
    for (int q = 0; q < 3; q++) o->vmax[q] = d.vmax[q];
    o->pr_grad_aver = d.pr_grad_aver; o->ux_mean = d.ux_mean; o->sc_mean = d.sc_mean; o->sc2_mean = d.sc2_mean;
}

int sync(paratc_ctx* ctx) {
    // the error word of the TMA-fed kernels comes back with the same wait:
    // bit 1 z transform, 2 x transform, 4 divergence-fed transform (a bounded
    // wait that ran out)
    unsigned int* hb = reinterpret_cast<unsigned int*>(ctx->h_scal + 15);
    *hb = 0u;
    cudaError_t e = cudaMemcpyAsync(hb, ctx->d_zt_err, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) return set_err(ctx, PARATC_ERR_CUDA, std::string("kernel execution: ") + cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(ctx, PARATC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    if (*hb) {
        std::string m;
        const char* names[3] = {"z transform", "x transform", "divergence-fed x transform"};
        for (int b = 0; b < 3; b++)
            if (*hb & (1u << b)) m += (m.empty() ? "" : ", ") + std::string(names[b]);
        return set_err(ctx, PARATC_ERR_TIMEOUT, m + ": a bounded wait on a copy pipeline gave up");
    }
    return PARATC_OK;
}

// host <-> device copies of one field between a host layout and the padded
// device layout (rows j = 1..ny of every z slab)
int copy_field(paratc_ctx* ctx, double* dev, const double* host_src, double* host_dst, int layout, bool dev_is_host_side) {
    (void)dev_is_host_side;
    cudaMemcpy3DParms p;
    std::memset(&p, 0, sizeof(p));
    const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    cudaPitchedPtr dp = make_cudaPitchedPtr(dev, (size_t)nx * sizeof(double), (size_t)nx, (size_t)ctx->nyt);
    cudaPitchedPtr hp;
    cudaPos hpos = make_cudaPos(0, 0, 0);
    if (layout == PARATC_LAYOUT_HALO) {
        hp = make_cudaPitchedPtr((void*)(host_src ? host_src : host_dst), (size_t)(nx + 4) * sizeof(double), (size_t)(nx + 4),
                                 (size_t)(ny + 2));
        hpos = make_cudaPos(2 * sizeof(double), 1, 2);
    } else {
        hp = make_cudaPitchedPtr((void*)(host_src ? host_src : host_dst), (size_t)nx * sizeof(double), (size_t)nx, (size_t)ny);
    }
    p.extent = make_cudaExtent((size_t)nx * sizeof(double), (size_t)ny, (size_t)nz);
    if (host_src) {
        p.srcPtr = hp; p.srcPos = hpos;
        p.dstPtr = dp; p.dstPos = make_cudaPos(0, 1, 0);
    } else {
        p.srcPtr = dp; p.srcPos = make_cudaPos(0, 1, 0);
        p.dstPtr = hp; p.dstPos = hpos;
    }
    p.kind = cudaMemcpyDefault;
    CK(cudaMemcpy3DAsync(&p, ctx->st));
    return PARATC_OK;
}

// the float arrays of the FP32 storage form, created on first use
int alloc_fp32(paratc_ctx* ctx) {
    if (ctx->f32.ux) return PARATC_OK;
    Fields32& g = ctx->f32;
    float** a[] = {&g.ux, &g.uy, &g.uz, &g.hx, &g.hy, &g.hz, &g.rx, &g.ry, &g.rz, &ctx->d_phi32};
    int rc;
    for (float** q : a)
        if ((rc = dalloc(ctx, q, ctx->nf))) return rc;
    if (ctx->prm.scalar_on) {
        float** b[] = {&g.sc, &g.hc, &g.rc};
        for (float** q : b)
            if ((rc = dalloc(ctx, q, ctx->nf))) return rc;
    }
    g.pr = ctx->f.pr;  // the pressure stays FP64
    if (ctx->pfft && zt_tma_supported(ctx->nz))
        ctx->ztma32_ok = zt_tma_prepare(spec32(ctx), ctx->ny * (ctx->nx / 2 + 1), ctx->nz, ctx->zt_tmap32);
    return PARATC_OK;
}

// the state (u, v, w, c, ghost rows included) and the explicit histories
// between the FP64 arrays and the float arrays of the FP32 storage form
void state_to32(paratc_ctx* ctx) {
    const Fields& a = ctx->f;
    const Fields32& b = ctx->f32;
    const double* src[] = {a.ux, a.uy, a.uz, a.hx, a.hy, a.hz, a.sc, a.hc};
    float* dst[] = {b.ux, b.uy, b.uz, b.hx, b.hy, b.hz, b.sc, b.hc};
    for (int q = 0; q < 8; q++)
        if (src[q] && dst[q]) { launch_cast(ctx->st, ctx->nf, src[q], dst[q]); ctx->launches++; }
}
void state_to64(paratc_ctx* ctx) {
    const Fields& a = ctx->f;
    const Fields32& b = ctx->f32;
    const float* src[] = {b.ux, b.uy, b.uz, b.hx, b.hy, b.hz, b.sc, b.hc};
    double* dst[] = {a.ux, a.uy, a.uz, a.hx, a.hy, a.hz, a.sc, a.hc};
    for (int q = 0; q < 8; q++)
        if (src[q] && dst[q]) { launch_cast(ctx->st, ctx->nf, src[q], dst[q]); ctx->launches++; }
}
// before a reader of the FP64 arrays (statistics, spectra, visualisation,
// restart, get_fields) in the FP32 storage form
void refresh64(paratc_ctx* ctx) {
    if (ctx->prec == PARATC_PREC_FP32) state_to64(ctx);
}

int load_state_common(paratc_ctx* ctx, bool wait) {
    // ChannelInitialize after read_restart (src/m_ChannelSystem.f90:63-68)
    launch_update_uy_ym(ctx->st, ctx->nx * ctx->nz, ctx->d_uy_ym, ctx->d_duy_ym);
    CK(cudaMemcpyAsync(ctx->d_coef, ctx->h_coef0, sizeof(DCoef), cudaMemcpyHostToDevice, ctx->st));
    launch_bc_all(ctx->st, ctx->kc, ctx->f, ctx->d_uy_ym);
    ctx->launches += 2;
    if (ctx->prec == PARATC_PREC_FP32) state_to32(ctx);
    return wait ? sync(ctx) : PARATC_OK;
}

}  // namespace

extern "C" {

const char* paratc_strerror(int status) {
    switch (status) {
    case PARATC_OK: return "ok";
    case PARATC_ERR_BAD_ARG: return "invalid argument";
    case PARATC_ERR_OOM: return "out of memory";
    case PARATC_ERR_CUDA: return "CUDA error";
    case PARATC_ERR_NONFINITE: return "non-finite value in a field";
    case PARATC_ERR_DIV_LIMIT: return "too big div";
    case PARATC_ERR_VEL_LIMIT: return "too big velocity";
    case PARATC_ERR_TIMEOUT: return "device wait timed out";
    case PARATC_ERR_IO: return "restart/input file error";
    case PARATC_ERR_NO_DEVICE: return "no CUDA device";
    case PARATC_ERR_NUMERIC: return "lamda2 wrong";
    default: return "unknown status";
    }
}

const char* paratc_last_error(paratc_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }
int64_t paratc_launch_count(paratc_ctx* ctx) { return ctx ? ctx->launches : 0; }
void* paratc_stream(paratc_ctx* ctx) { return ctx ? (void*)ctx->st : nullptr; }

int paratc_profile_enable(paratc_ctx* ctx, int on) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (on) {
        if (ctx->ev.empty()) {
            ctx->ev.resize(4096);
            ctx->ev_class.resize(2048);
            for (auto& e : ctx->ev) CK(cudaEventCreate(&e));
        }
        prof_flush(ctx);
        for (int k = 0; k < PARATC_PROF_NKERNELS; k++) { ctx->prof_ms[k] = 0.0; ctx->prof_n[k] = 0; }
        ctx->prof_on = true;
    } else {
        prof_flush(ctx);
        ctx->prof_on = false;
    }
    return PARATC_OK;
}

int paratc_profile_get(paratc_ctx* ctx, int k, double* total_ms, int64_t* launches) {
    if (!ctx || k < 0 || k >= PARATC_PROF_NKERNELS) return PARATC_ERR_BAD_ARG;
    prof_flush(ctx);
    if (total_ms) *total_ms = ctx->prof_ms[k];
    if (launches) *launches = ctx->prof_n[k];
    return PARATC_OK;
}

const char* paratc_profile_name(int k) { return (k >= 0 && k < PARATC_PROF_NKERNELS) ? kProfNames[k] : ""; }

int paratc_destroy(paratc_ctx* ctx) {
    if (!ctx) return PARATC_OK;
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    for (auto& e : ctx->ev) cudaEventDestroy(e);
    for (void* p : ctx->allocs) cudaFree(p);
    if (ctx->h_diag) cudaFreeHost(ctx->h_diag);
    if (ctx->h_coef) cudaFreeHost(ctx->h_coef);
    if (ctx->h_coef0) cudaFreeHost(ctx->h_coef0);
    if (ctx->h_scal) cudaFreeHost(ctx->h_scal);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
    return PARATC_OK;
}

int paratc_create(const paratc_params* prm, const double* yp, int device, paratc_ctx** out) {
    if (!prm || !yp || !out) return PARATC_ERR_BAD_ARG;
    *out = nullptr;
    std::string why;
    int rc = validate_params(*prm, why);
    if (rc != PARATC_OK) {
        std::fprintf(stderr, "paratc_create: %s\n", why.c_str());
        return rc;
    }
    if (!tridiag_supported(prm->nyc)) {
        std::fprintf(stderr, "paratc_create: nyc=%d outside the supported 3..256\n", prm->nyc);
        return PARATC_ERR_BAD_ARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return PARATC_ERR_NO_DEVICE;
    paratc_ctx* ctx = new paratc_ctx();
    ctx->prm = *prm;
    if (device < 0) cudaGetDevice(&ctx->dev);
    else ctx->dev = device;
    if (ctx->dev >= ndev) { delete ctx; return PARATC_ERR_BAD_ARG; }
    CK(cudaSetDevice(ctx->dev));
    rc = build_metrics(*prm, yp, ctx->hm);
    if (rc != PARATC_OK) { delete ctx; return rc; }
    ctx->nx = prm->nxc; ctx->ny = prm->nyc; ctx->nz = prm->nzc; ctx->nyp = prm->nyc + 1; ctx->nyt = prm->nyc + 2;
    ctx->M1 = ctx->nx / 2 + 1;
    ctx->nf = (size_t)ctx->nz * ctx->nyt * ctx->nx;
    ctx->ni = (size_t)ctx->nz * ctx->ny * ctx->nx;
    if (make_plan(ctx->nx / 2, ctx->plx) != PARATC_OK || make_plan(ctx->nz, ctx->plz) != PARATC_OK) {
        std::fprintf(stderr, "paratc_create: nxc/2 and nzc must factor into 2, 3 and 5\n");
        delete ctx;
        return PARATC_ERR_BAD_ARG;
    }
    if (fft_smem_need(ctx->nx, ctx->nz) > 160 * 1024) {
        std::fprintf(stderr, "paratc_create: grid too large for the shared-memory FFT\n");
        delete ctx;
        return PARATC_ERR_BAD_ARG;
    }
    ctx->pfft = pfft_x_supported(ctx->nx / 2) && pfft_z_supported(ctx->nz) && std::getenv("PARATC_GENERIC_FFT") == nullptr;
    // PARATC_NO_PLANE keeps the separate x and z transform kernels (both exact)
    ctx->plane = ctx->pfft && plane_supported(ctx->nx, ctx->nz) && std::getenv("PARATC_NO_PLANE") == nullptr;
    cudaError_t ce = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking);
    if (ce != cudaSuccess) { delete ctx; return PARATC_ERR_CUDA; }
    // the kernels' shared-memory limits are attributes of each device: set
    // them once per device, with that device current
    {
        static std::mutex mu;
        static std::vector<int> done;
        std::lock_guard<std::mutex> lock(mu);
        if (std::find(done.begin(), done.end(), ctx->dev) == done.end()) {
            fft_init();
            tridiag_init();
            rhs_init();
            pfft_x_init();
            pfft_z_init();
            plane_init();
            zt_tma_init();
            xt_tma_init();
            spectra_init();
            done.push_back(ctx->dev);
        }
    }
    const HostMetrics& h = ctx->hm;
    // ---- constants
    DConst& kc = ctx->kc;
    std::memset(&kc, 0, sizeof(kc));
    kc.nx = ctx->nx; kc.ny = ctx->ny; kc.nz = ctx->nz; kc.nyp = ctx->nyp; kc.nyt = ctx->nyt;
    kc.flow_type = prm->flow_type; kc.scalar_on = prm->scalar_on; kc.is_ux_const = prm->is_ux_const; kc.icfl = prm->icfl;
    cudaDeviceGetAttribute(&kc.nsm, cudaDevAttrMultiProcessorCount, ctx->dev);
    {
        // PARATC_YSOLVER=staged|streaming pins the variant of the y-solve
        // kernels (both are exact; the choice is normally made by size)
        const char* e = std::getenv("PARATC_YSOLVER");
        kc.solver_sel = !e ? 0 : (std::strcmp(e, "staged") == 0 ? 1 : (std::strcmp(e, "streaming") == 0 ? 2 : 0));
    }
    for (int q = 0; q < 4; q++) { kc.dxC[q] = h.dxC[q]; kc.dzC[q] = h.dzC[q]; kc.IC[q] = h.IC[q]; }
    for (int q = 0; q < 5; q++) { kc.dxxC[q] = h.dxxC[q]; kc.dzzC[q] = h.dzzC[q]; }
    kc.rdx = h.rdx; kc.rdz = h.rdz;
    kc.ucrf = prm->ucrf; kc.xnu = prm->xnu; kc.sdiff = prm->sdiff;
    for (int q = 0; q < 3; q++) { kc.grav[q] = prm->gravity[q]; kc.gev[q] = prm->gravity_eff_vec[q]; kc.fvv[q] = prm->falling_vel_vec[q]; }
    kc.uxbc_ym = prm->ux_bc[2]; kc.uxbc_yp = prm->ux_bc[3]; kc.uybc_yp = prm->uy_bc[3];
    kc.uzbc_ym = prm->uz_bc[2]; kc.uzbc_yp = prm->uz_bc[3];
    kc.ubulk = prm->ubulk; kc.yly = prm->yly; kc.normfft = h.normfft; kc.dt_max = prm->dt_max; kc.cflc = prm->cflc;
    kc.sc_r1b = h.sc_r1b; kc.sc_r2b = h.sc_r2b; kc.sc_r1t = h.sc_r1t; kc.sc_r2t = h.sc_r2t;
    kc.vel_limit = prm->vel_limit; kc.div_limit = prm->div_limit;
    for (int q = 0; q < 4; q++) { kc.fdxC[q] = (float)kc.dxC[q]; kc.fdzC[q] = (float)kc.dzC[q]; kc.fIC[q] = (float)kc.IC[q]; }
    for (int q = 0; q < 5; q++) { kc.fdxxC[q] = (float)kc.dxxC[q]; kc.fdzzC[q] = (float)kc.dzzC[q]; }
    for (int q = 0; q < 3; q++) { kc.fgrav[q] = (float)kc.grav[q]; kc.fgev[q] = (float)kc.gev[q]; kc.ffvv[q] = (float)kc.fvv[q]; }
    kc.fucrf = (float)kc.ucrf; kc.fxnu = (float)kc.xnu; kc.fsdiff = (float)kc.sdiff;

    // ---- device memory
    const size_t nf = ctx->nf;
    Fields& f = ctx->f;
    std::memset(&f, 0, sizeof(f));
    double** fl[] = {&f.ux, &f.uy, &f.uz, &f.pr, &f.hx, &f.hy, &f.hz, &f.rx, &f.ry, &f.rz, &ctx->d_phi};
    for (double** p : fl)
        if ((rc = dalloc(ctx, p, nf)) != PARATC_OK) { paratc_destroy(ctx); return rc; }
    if (prm->scalar_on) {
        double** fs[] = {&f.sc, &f.hc, &f.rc};
        for (double** p : fs)
            if ((rc = dalloc(ctx, p, nf)) != PARATC_OK) { paratc_destroy(ctx); return rc; }
    }
    // partial-result records of the grid reductions: one per block of k_prsrc /
    // k_cfl, one per block of the RHS and forward-x kernels, 8 per block of the
    // end-of-step kernel
    ctx->npart = std::max(std::max(4 * cell_grid_blocks(kc), rhs_grid_blocks(kc)),
                          std::max((size_t)pfft_x_blocks(ctx->nx, ctx->ny, ctx->nz), endstep_blocks(kc) * 8)) + 64;
    if ((rc = dalloc(ctx, &ctx->d_src, ctx->ni)) || (rc = dalloc(ctx, &ctx->d_spec, (size_t)ctx->M1 * ctx->ny * ctx->nz)) ||
        (rc = dalloc(ctx, &ctx->d_part, ctx->npart)) || (rc = dalloc(ctx, &ctx->d_uy_ym, (size_t)ctx->nx * ctx->nz)) ||
        (rc = dalloc(ctx, &ctx->d_duy_ym, (size_t)ctx->nx * ctx->nz)) || (rc = dalloc(ctx, &ctx->d_coef, 1)) ||
        (rc = dalloc(ctx, &ctx->d_diag, 1)) || (rc = dalloc(ctx, &ctx->d_diag2, 1)) || (rc = dalloc(ctx, &ctx->d_scal, 16)) ||
        (rc = dalloc(ctx, &ctx->d_counter, 16)) ||
        (rc = dalloc(ctx, &ctx->d_hfac, helm_fac_doubles(ctx->ny))) ||
        (rc = dalloc(ctx, &ctx->d_pfac, (size_t)2 * ctx->M1 * ctx->nz * ctx->ny)) ||
        (rc = dalloc(ctx, &ctx->d_stats, (size_t)ctx->nyp * 40 + 1)) ||
        (rc = dalloc(ctx, &ctx->d_stats_part, stats_part_doubles(kc))) ||
        (rc = dalloc(ctx, &ctx->d_zt_err, 1))) {
        paratc_destroy(ctx);
        return rc;
    }
    // metrics: 25 y-arrays of nyp+1 plus wavenumbers
    {
        const size_t ny1 = (size_t)ctx->nyp + 1;
        std::vector<double> buf;
        HostMetrics& hm = ctx->hm;
        std::vector<const std::vector<double>*> ys = {&hm.rdyp, &hm.rdyc, &hm.dyp, &hm.yinterp, &hm.ap2c, &hm.ac2c, &hm.am2c,
                                                      &hm.ap2p, &hm.ac2p, &hm.am2p, &hm.ap2ph, &hm.ac2ph, &hm.am2ph,
                                                      &hm.ap2cCN, &hm.ac2cCN, &hm.am2cCN, &hm.ap2cSc, &hm.ac2cSc, &hm.am2cSc,
                                                      &hm.ap2cScCN, &hm.ac2cScCN, &hm.am2cScCN};
        for (auto* v : ys) buf.insert(buf.end(), v->begin(), v->end());
        buf.insert(buf.end(), hm.wnx.begin(), hm.wnx.end());
        buf.insert(buf.end(), hm.wnz.begin(), hm.wnz.end());
        // per-row coefficient records of the right-hand side (DMetric::rowmet),
        // 16-double aligned in the buffer
        while (buf.size() % ROWMET) buf.push_back(0.0);
        const size_t o_rowmet = buf.size();
        for (size_t j = 0; j < ny1; j++) {
            const double rec[ROWMET] = {hm.yinterp[j], j + 1 < ny1 ? hm.yinterp[j + 1] : 0.0, hm.rdyp[j], hm.rdyc[j],
                                        hm.dyp[j], hm.ap2c[j], hm.ac2c[j], hm.am2c[j], hm.ap2p[j], hm.ac2p[j],
                                        hm.am2p[j], hm.ap2cSc[j], hm.ac2cSc[j], hm.am2cSc[j], 0.0, 0.0};
            buf.insert(buf.end(), rec, rec + ROWMET);
        }
        if ((rc = dalloc(ctx, &ctx->d_metric, buf.size()))) { paratc_destroy(ctx); return rc; }
        CK(cudaMemcpyAsync(ctx->d_metric, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        const double* b = ctx->d_metric;
        const double** dst[] = {&ctx->dm.rdyp, &ctx->dm.rdyc, &ctx->dm.dyp, &ctx->dm.yinterp, &ctx->dm.ap2c, &ctx->dm.ac2c,
                                &ctx->dm.am2c, &ctx->dm.ap2p, &ctx->dm.ac2p, &ctx->dm.am2p, &ctx->dm.ap2ph, &ctx->dm.ac2ph,
                                &ctx->dm.am2ph, &ctx->dm.ap2cCN, &ctx->dm.ac2cCN, &ctx->dm.am2cCN, &ctx->dm.ap2cSc,
                                &ctx->dm.ac2cSc, &ctx->dm.am2cSc, &ctx->dm.ap2cScCN, &ctx->dm.ac2cScCN, &ctx->dm.am2cScCN};
        for (size_t a = 0; a < sizeof(dst) / sizeof(dst[0]); a++) *dst[a] = b + a * ny1;
        ctx->dm.wnx = b + ys.size() * ny1;
        ctx->dm.wnz = ctx->dm.wnx + ctx->nx;
        ctx->dm.rowmet = b + o_rowmet;
        // pivots of the spectral y systems (constant for the life of the context)
        launch_pois_factors(ctx->st, kc, ctx->dm, ctx->d_pfac);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->st));
    }
    // z transforms fed by TMA: the default of the separate-transform path
    // where nz has a kernel; PARATC_ZT_TMA=0 keeps the register-fed k_zt
    if (ctx->pfft && zt_tma_supported(ctx->nz))
        ctx->ztma_ok = zt_tma_prepare(ctx->d_spec, ctx->ny * (ctx->nx / 2 + 1), ctx->nz, ctx->zt_tmap);
    {
        const char* e = std::getenv("PARATC_ZT_TMA");
        ctx->ztma = ctx->ztma_ok && !ctx->plane && !(e && std::atoi(e) == 0);
        const char* ex = std::getenv("PARATC_XT_TMA");
        ctx->xtma = ctx->pfft && xt_tma_supported(ctx->nx / 2) && !(ex && std::atoi(ex) == 0);
    }
    // twiddles
    {
        std::vector<double2> twx = twiddles(ctx->nx / 2, ctx->nx / 2);
        std::vector<double2> post = twiddles(ctx->nx, ctx->nx / 2 + 1);
        std::vector<double2> twz = twiddles(ctx->nz, ctx->nz);
        if ((rc = dalloc(ctx, &ctx->d_twx, twx.size())) || (rc = dalloc(ctx, &ctx->d_postx, post.size())) ||
            (rc = dalloc(ctx, &ctx->d_twz, twz.size()))) {
            paratc_destroy(ctx);
            return rc;
        }
        // on the context's stream, after dalloc's zero fill; the host vectors live until the sync
        CK(cudaMemcpyAsync(ctx->d_twx, twx.data(), twx.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->d_postx, post.data(), post.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(ctx->d_twz, twz.data(), twz.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    CK(cudaMallocHost(&ctx->h_diag, sizeof(DDiag)));
    CK(cudaMallocHost(&ctx->h_coef, sizeof(DCoef)));
    CK(cudaMallocHost(&ctx->h_coef0, sizeof(DCoef)));
    std::memset(ctx->h_coef0, 0, sizeof(DCoef));
    ctx->h_coef0->dt = ctx->prm.dt_max;
    CK(cudaMallocHost(&ctx->h_scal, 16 * sizeof(double)));
    // AllocateVariables: scalar = Scalar_InitValue everywhere (src/m_Variables.f90:84)
    if (prm->scalar_on) {
        std::vector<double> init(nf, prm->scalar_init_value);
        CK(cudaMemcpy(f.sc, init.data(), nf * sizeof(double), cudaMemcpyHostToDevice));
    }
    rc = load_state_common(ctx, true);
    if (rc != PARATC_OK) { paratc_destroy(ctx); return rc; }
    // picks of an earlier tuning run on this GPU and grid (paratc_autotune_all)
    if (const char* cache = std::getenv("PARATC_TUNE_CACHE")) {
        paratc_tuning t;
        std::memset(&t, 0, sizeof(t));
        if (tune_cache_read(cache, tune_key(ctx), &t) && tuning_valid(ctx, t)) {
            tuning_apply(ctx, t);
            ctx->tune_from_cache = 1;
            ctx->tune_step_ms = t.step_ms;
        }
    }
    *out = ctx;
    return PARATC_OK;
}

static int set_fields_impl(paratc_ctx* ctx, const double* ux, const double* uy, const double* uz, const double* p,
                           const double* c, const double* hx, const double* hy, const double* hz, const double* hc,
                           int layout, bool wait) {
    if (!ctx || (layout != PARATC_LAYOUT_INTERIOR && layout != PARATC_LAYOUT_HALO)) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    ctx->next_ready = false;
    struct { double* d; const double* h; bool hist; } tab[] = {
        {ctx->f.ux, ux, false}, {ctx->f.uy, uy, false}, {ctx->f.uz, uz, false}, {ctx->f.pr, p, false},
        {ctx->f.sc, c, false}, {ctx->f.hx, hx, true}, {ctx->f.hy, hy, true}, {ctx->f.hz, hz, true}, {ctx->f.hc, hc, true}};
    for (auto& t : tab) {
        if (!t.d) continue;
        if (t.h) {
            int rc = copy_field(ctx, t.d, t.h, nullptr, layout, false);
            if (rc) return rc;
        } else if (t.hist) {
            CK(cudaMemsetAsync(t.d, 0, ctx->nf * sizeof(double), ctx->st));
        }
    }
    return load_state_common(ctx, wait);
}

int paratc_set_fields(paratc_ctx* ctx, const double* ux, const double* uy, const double* uz, const double* p,
                      const double* c, const double* hx, const double* hy, const double* hz, const double* hc, int layout) {
    return set_fields_impl(ctx, ux, uy, uz, p, c, hx, hy, hz, hc, layout, true);
}

int paratc_set_fields_async(paratc_ctx* ctx, const double* ux, const double* uy, const double* uz, const double* p,
                            const double* c, const double* hx, const double* hy, const double* hz, const double* hc,
                            int layout) {
    return set_fields_impl(ctx, ux, uy, uz, p, c, hx, hy, hz, hc, layout, false);
}

static int get_fields_impl(paratc_ctx* ctx, double* ux, double* uy, double* uz, double* p, double* c, double* hx,
                           double* hy, double* hz, double* hc, int layout, bool wait) {
    if (!ctx || (layout != PARATC_LAYOUT_INTERIOR && layout != PARATC_LAYOUT_HALO)) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    refresh64(ctx);
    struct { double* d; double* h; } tab[] = {{ctx->f.ux, ux}, {ctx->f.uy, uy}, {ctx->f.uz, uz}, {ctx->f.pr, p},
                                             {ctx->f.sc, c}, {ctx->f.hx, hx}, {ctx->f.hy, hy}, {ctx->f.hz, hz}, {ctx->f.hc, hc}};
    for (auto& t : tab) {
        if (!t.d || !t.h) continue;
        int rc = copy_field(ctx, t.d, nullptr, t.h, layout, false);
        if (rc) return rc;
    }
    return wait ? sync(ctx) : PARATC_OK;
}

int paratc_get_fields(paratc_ctx* ctx, double* ux, double* uy, double* uz, double* p, double* c, double* hx, double* hy,
                      double* hz, double* hc, int layout) {
    return get_fields_impl(ctx, ux, uy, uz, p, c, hx, hy, hz, hc, layout, true);
}

int paratc_get_fields_async(paratc_ctx* ctx, double* ux, double* uy, double* uz, double* p, double* c, double* hx,
                            double* hy, double* hz, double* hc, int layout) {
    return get_fields_impl(ctx, ux, uy, uz, p, c, hx, hy, hz, hc, layout, false);
}

int paratc_sync(paratc_ctx* ctx) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    return sync(ctx);
}

int paratc_set_fields_device(paratc_ctx* ctx, const double* ux, const double* uy, const double* uz, const double* p,
                             const double* c, const double* hx, const double* hy, const double* hz, const double* hc) {
    return paratc_set_fields(ctx, ux, uy, uz, p, c, hx, hy, hz, hc, PARATC_LAYOUT_INTERIOR);
}

int paratc_get_fields_device(paratc_ctx* ctx, double* ux, double* uy, double* uz, double* p, double* c, double* hx,
                             double* hy, double* hz, double* hc) {
    return paratc_get_fields(ctx, ux, uy, uz, p, c, hx, hy, hz, hc, PARATC_LAYOUT_INTERIOR);
}

int paratc_set_time(paratc_ctx* ctx, double sim_time, double dt) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaMemcpyAsync(ctx->h_coef, ctx->d_coef, sizeof(DCoef), cudaMemcpyDeviceToHost, ctx->st));
    int rc = sync(ctx);
    if (rc) return rc;
    ctx->h_coef->sim_time = sim_time;
    ctx->h_coef->dt = dt;
    ctx->next_ready = false;
    CK(cudaMemcpyAsync(ctx->d_coef, ctx->h_coef, sizeof(DCoef), cudaMemcpyHostToDevice, ctx->st));
    return sync(ctx);
}

int paratc_get_time(paratc_ctx* ctx, double* sim_time, double* dt) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaMemcpyAsync(ctx->h_coef, ctx->d_coef, sizeof(DCoef), cudaMemcpyDeviceToHost, ctx->st));
    int rc = sync(ctx);
    if (rc) return rc;
    if (sim_time) *sim_time = ctx->h_coef->sim_time;
    // after a step the device already holds the next step's dt; report the last one
    if (dt) *dt = ctx->next_ready ? ctx->h_coef->dt_last : ctx->h_coef->dt;
    return PARATC_OK;
}

int paratc_steps(paratc_ctx* ctx, int n, paratc_diag* diag) {
    if (!ctx || n < 1) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaMemsetAsync(ctx->d_diag, 0, sizeof(DDiag), ctx->st));
    for (int s = 0; s < n; s++) enqueue_step(ctx);
    CK(cudaMemcpyAsync(ctx->h_diag, ctx->d_diag, sizeof(DDiag), cudaMemcpyDeviceToHost, ctx->st));
    int rc = sync(ctx);
    if (rc) return rc;
    diag_out(*ctx->h_diag, diag);
    if (ctx->h_diag->status != 0) {
        char b[160];
        std::snprintf(b, sizeof(b), "%s at step %d of %d (divmax %.6e, vmax %.6e %.6e %.6e)",
                      paratc_strerror(ctx->h_diag->status), ctx->h_diag->failed_step, n, ctx->h_diag->divmax,
                      ctx->h_diag->vmax[0], ctx->h_diag->vmax[1], ctx->h_diag->vmax[2]);
        return set_err(ctx, ctx->h_diag->status, b);
    }
    return PARATC_OK;
}

int paratc_step(paratc_ctx* ctx, paratc_diag* diag) { return paratc_steps(ctx, 1, diag); }

int paratc_steps_async(paratc_ctx* ctx, int n) {
    if (!ctx || n < 1) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    for (int s = 0; s < n; s++) enqueue_step(ctx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(ctx, PARATC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return PARATC_OK;
}

int paratc_last_diag(paratc_ctx* ctx, paratc_diag* diag) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaMemcpyAsync(ctx->h_diag, ctx->d_diag, sizeof(DDiag), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemsetAsync(ctx->d_diag, 0, sizeof(DDiag), ctx->st));
    int rc = sync(ctx);
    if (rc) return rc;
    diag_out(*ctx->h_diag, diag);
    if (ctx->h_diag->status != 0) {
        char b[160];
        std::snprintf(b, sizeof(b), "%s at step %d (divmax %.6e)", paratc_strerror(ctx->h_diag->status),
                      ctx->h_diag->failed_step, ctx->h_diag->divmax);
        return set_err(ctx, ctx->h_diag->status, b);
    }
    return PARATC_OK;
}

int paratc_substep(paratc_ctx* ctx, int ns, double dt, double* divmax_src) {
    return paratc_substep_stage(ctx, ns, dt, 5, divmax_src);
}

int paratc_substep_stage(paratc_ctx* ctx, int ns, double dt, int stop_stage, double* divmax_src) {
    if (!ctx || ns < 1 || ns > ctx->hm.iadvance || stop_stage < 1 || stop_stage > 5) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    ctx->next_ready = false;
    CK(cudaMemcpyAsync(ctx->h_coef, ctx->d_coef, sizeof(DCoef), cudaMemcpyDeviceToHost, ctx->st));
    int rc = sync(ctx);
    if (rc) return rc;
    ctx->h_coef->dt = dt;
    CK(cudaMemcpyAsync(ctx->d_coef, ctx->h_coef, sizeof(DCoef), cudaMemcpyHostToDevice, ctx->st));
    launch_helm_factors(ctx->st, ctx->kc, ctx->dm, ctx->d_coef, ns, 1, ctx->hm.alp, ctx->d_hfac);
    ctx->hfac_dt = -1.0;  // pivots of substep ns now hold this call's dt
    ctx->launches += 1;
    enqueue_substep(ctx, ns, stop_stage);
    CK(cudaMemcpyAsync(ctx->h_coef, ctx->d_coef, sizeof(DCoef), cudaMemcpyDeviceToHost, ctx->st));
    rc = sync(ctx);
    if (rc) return rc;
    if (divmax_src) *divmax_src = ctx->h_coef->divmax_src;
    return PARATC_OK;
}

int paratc_get_work(paratc_ctx* ctx, int which, double* out) {
    if (!ctx || !out || which < 0 || which > 5) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    double* src[] = {ctx->f.rx, ctx->f.ry, ctx->f.rz, ctx->f.rc, ctx->d_src, ctx->d_phi};
    if (!src[which]) return PARATC_ERR_BAD_ARG;
    if (ctx->prec == PARATC_PREC_FP32 && which != 4) {
        // the FP32 storage form's work arrays, widened into the FP64 ones
        const float* w32[] = {ctx->f32.rx, ctx->f32.ry, ctx->f32.rz, ctx->f32.rc, nullptr, ctx->d_phi32};
        launch_cast(ctx->st, ctx->nf, w32[which], src[which]);
        ctx->launches += 1;
    }
    int rc;
    if (which == 4) {
        CK(cudaMemcpyAsync(out, ctx->d_src, ctx->ni * sizeof(double), cudaMemcpyDefault, ctx->st));
        rc = sync(ctx);
    } else {
        rc = copy_field(ctx, src[which], nullptr, out, PARATC_LAYOUT_INTERIOR, false);
        if (rc == PARATC_OK) rc = sync(ctx);
    }
    if (rc) return rc;
    if (which == 0) {
        CK(cudaMemcpyAsync(ctx->h_coef, ctx->d_coef, sizeof(DCoef), cudaMemcpyDeviceToHost, ctx->st));
        rc = sync(ctx);
        if (rc) return rc;
        const double add = ctx->h_coef->rhsx_add;
        for (size_t q = 0; q < ctx->ni; q++) out[q] = out[q] + add;
    }
    return PARATC_OK;
}

int paratc_poisson_device(paratc_ctx* ctx, const double* d_src, double* d_phi) {
    if (!ctx || !d_src || !d_phi) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    enqueue_poisson(ctx, d_src, d_phi, 0);
    return sync(ctx);
}

int paratc_poisson_device_async(paratc_ctx* ctx, const double* d_src, double* d_phi) {
    if (!ctx || !d_src || !d_phi) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    enqueue_poisson(ctx, d_src, d_phi, 0);
    CK(cudaGetLastError());
    return PARATC_OK;
}

int paratc_poisson_refined_async(paratc_ctx* ctx, const double* d_src, double* d_phi, int ncorr) {
    if (!ctx || !d_src || !d_phi || ncorr < 0 || d_src == d_phi) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (!ctx->pfft) return set_err(ctx, PARATC_ERR_BAD_ARG, "the refined solve needs compile-time-length transforms");
    enqueue_solve32(ctx, d_src, d_phi, 0, nullptr);
    for (int q = 0; q < ncorr; q++) {
        // r = src - L phi in FP64 (into the context's compact work array), then
        // its FP32-spectrum solve added to phi
        launch_residual(ctx->st, ctx->kc, ctx->dm, d_src, d_phi, ctx->d_src, ctx->d_part, ctx->d_counter + 5,
                        ctx->d_scal + 4);
        ctx->launches += 1;
        enqueue_solve32(ctx, ctx->d_src, d_phi, 1, ctx->d_scal + 7);
    }
    CK(cudaGetLastError());
    return PARATC_OK;
}

int paratc_poisson_refined(paratc_ctx* ctx, const double* d_src, double* d_phi, double rtol, int max_corr,
                           int* ncorr, double* relres) {
    if (!ctx || !d_src || !d_phi || max_corr < 0 || d_src == d_phi) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (!ctx->pfft) return set_err(ctx, PARATC_ERR_BAD_ARG, "the refined solve needs compile-time-length transforms");
    enqueue_solve32(ctx, d_src, d_phi, 0, nullptr);
    int q = 0;
    double rel = 0.0;
    for (;;) {
        launch_residual(ctx->st, ctx->kc, ctx->dm, d_src, d_phi, ctx->d_src, ctx->d_part, ctx->d_counter + 5,
                        ctx->d_scal + 4);
        ctx->launches += 1;
        CK(cudaMemcpyAsync(ctx->h_scal + 4, ctx->d_scal + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        const int rc = sync(ctx);
        if (rc) return rc;
        rel = ctx->h_scal[4] / std::max(ctx->h_scal[5], 1e-300);
        if (!(rel > rtol) || q >= max_corr) break;
        enqueue_solve32(ctx, ctx->d_src, d_phi, 1, ctx->d_scal + 7);
        q++;
    }
    if (ncorr) *ncorr = q;
    if (relres) *relres = rel;
    return PARATC_OK;
}

int paratc_poisson(paratc_ctx* ctx, const double* src, double* phi) {
    if (!ctx || !src || !phi) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaMemcpyAsync(ctx->d_src, src, ctx->ni * sizeof(double), cudaMemcpyDefault, ctx->st));
    enqueue_poisson(ctx, ctx->d_src, ctx->d_src, 0);
    CK(cudaMemcpyAsync(phi, ctx->d_src, ctx->ni * sizeof(double), cudaMemcpyDefault, ctx->st));
    return sync(ctx);
}

// Poisson schedules: 2*s + (y-1), s 0 fused y-plane transforms, 1 separate
// compile-time-length x / z transforms, 2 generic mixed-radix transforms, 3
// as 1 with TMA-fed z transforms; y 1 staged, 2 streaming spectral y-solve
static bool sched_supported(const paratc_ctx* ctx, int choice) {
    if (choice < 0 || choice >= PARATC_SCHED_NCHOICES) return false;
    const int sc = choice / 2;
    const bool pfft_ok = pfft_x_supported(ctx->nx / 2) && pfft_z_supported(ctx->nz);
    if (sc == 0) return pfft_ok && plane_supported(ctx->nx, ctx->nz);
    if (sc == 1) return pfft_ok;
    if (sc == 3) return pfft_ok && ctx->ztma_ok;
    if (sc == 4) return pfft_ok && ctx->xtma;
    if (sc == 5) return pfft_ok && ctx->ztma_ok && ctx->xtma;
    return true;
}

static void sched_apply(paratc_ctx* ctx, int choice) {
    const int sc = choice / 2;
    ctx->plane = sc == 0;
    ctx->pfft = sc == 0 || sc == 1 || sc >= 3;
    ctx->ztma = sc == 3 || sc == 5;
    ctx->xdiv = sc == 4 || sc == 5;
    ctx->kc.solver_sel = choice % 2 + 1;
    ctx->sched_gen++;
}

int paratc_get_schedule(paratc_ctx* ctx, int* choice) {
    if (!ctx || !choice) return PARATC_ERR_BAD_ARG;
    const int sc = ctx->plane ? 0 : (ctx->xdiv ? (ctx->ztma ? 5 : 4) : (ctx->ztma ? 3 : (ctx->pfft ? 1 : 2)));
    *choice = 2 * sc + (ctx->kc.solver_sel == 2 ? 1 : 0);
    return PARATC_OK;
}

int paratc_set_schedule(paratc_ctx* ctx, int choice) {
    if (!ctx || !sched_supported(ctx, choice)) return PARATC_ERR_BAD_ARG;
    sched_apply(ctx, choice);
    return PARATC_OK;
}

int paratc_set_wait_limit(paratc_ctx* ctx, long long polls) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    // word 1 after the error word, read by every TMA-fed kernel at its start
    const unsigned int v = polls < 0 ? 0u : (unsigned int)std::min<long long>(polls + 1, 0xffffffffLL);
    CK(cudaMemcpyAsync(ctx->d_zt_err + 1, &v, sizeof(v), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));  // v lives on this stack frame
    return PARATC_OK;
}

int paratc_set_precision(paratc_ctx* ctx, int prec) {
    if (!ctx || (prec != PARATC_PREC_FP64 && prec != PARATC_PREC_MIXED && prec != PARATC_PREC_FP32))
        return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (prec == PARATC_PREC_FP32 && !(pfft_x_supported(ctx->nx / 2) && pfft_z_supported(ctx->nz) && ctx->nx % 4 == 0))
        return set_err(ctx, PARATC_ERR_BAD_ARG,
                       "the FP32 storage form needs nxc % 4 == 0 and compile-time-length transforms for nxc/2 and nzc");
    if (prec == PARATC_PREC_FP32 && ctx->prec != PARATC_PREC_FP32) {
        int rc = alloc_fp32(ctx);
        if (rc) return rc;
        state_to32(ctx);
        // the generic-length transforms have no float2 form
        if (!ctx->pfft) sched_apply(ctx, plane_supported(ctx->nx, ctx->nz) ? 0 : 2);
    } else if (prec != PARATC_PREC_FP32 && ctx->prec == PARATC_PREC_FP32) {
        state_to64(ctx);
    }
    ctx->prec = prec;
    ctx->kc.fp32_rhs = prec == PARATC_PREC_MIXED ? 1 : 0;
    ctx->next_ready = false;  // the next step takes its CFL from the converted state
    ctx->sched_gen++;         // captured graphs hold the other kernels
    return sync(ctx);
}

int paratc_get_precision(paratc_ctx* ctx, int* prec) {
    if (!ctx || !prec) return PARATC_ERR_BAD_ARG;
    *prec = ctx->prec;
    return PARATC_OK;
}

int paratc_autotune(paratc_ctx* ctx, int nrep, int* choice, double* times_ms) {
    if (!ctx || nrep < 1) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float tbest[PARATC_SCHED_NCHOICES];
    for (int c = 0; c < PARATC_SCHED_NCHOICES; c++) tbest[c] = -1.f;
    int rc = PARATC_OK;
    // three interleaved rounds over the choices, each choice keeping its
    // fastest round, so that a clock that drifts during the search (power
    // or thermal limits on the largest grids) favours no choice
    constexpr int kRounds = 3;
    for (int round = 0; round < kRounds && rc == PARATC_OK; round++) {
        for (int q = 0; q < PARATC_SCHED_NCHOICES && rc == PARATC_OK; q++) {
            const int c = (q + round * 3) % PARATC_SCHED_NCHOICES;  // another order each round
            if (!sched_supported(ctx, c)) continue;
            const bool f32 = ctx->prec == PARATC_PREC_FP32;
            if (f32 && c / 2 == 2) continue;  // the generic transforms have no float2 form
            sched_apply(ctx, c);
            // the step's form of the solve: divergence source, transforms,
            // y-solve, inverse into phi with its Neumann ghosts (state
            // untouched), in the context's storage form
            for (int r = 0; r < nrep + 1; r++) {
                if (r == 1) cudaEventRecord(e0, ctx->st);
                if (f32) {
                    enqueue_poisson_head32(ctx, 1, ctx->d_scal);
                    enqueue_poisson_tail32(ctx, ctx->d_phi32, 1);
                } else {
                    enqueue_poisson_head(ctx, 1, nullptr, ctx->d_scal);
                    enqueue_poisson_tail(ctx, ctx->d_phi, 1);
                }
            }
            cudaEventRecord(e1, ctx->st);
            rc = sync(ctx);
            float ms = 0.f;
            if (rc == PARATC_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) rc = PARATC_ERR_CUDA;
            if (rc != PARATC_OK) break;
            if (tbest[c] < 0.f || ms < tbest[c]) tbest[c] = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != PARATC_OK) return rc;
    int best = -1;
    for (int c = 0; c < PARATC_SCHED_NCHOICES; c++) {
        if (times_ms) times_ms[c] = tbest[c];
        if (tbest[c] >= 0.f && (best < 0 || tbest[c] < tbest[best])) best = c;
    }
    sched_apply(ctx, best);
    if (choice) *choice = best;
    return PARATC_OK;
}

extern "C++" {
// ---- tuning of the launch shapes and the Poisson schedule, with a cache
// file.  The key names the GPU, the grid, the scalar, the precision and the
// flow type; one entry per line,
//   "NVIDIA B200|128x96x128|s0|p0|f1": {"schedule": 6, "rhs_var": 0, "helm_var": 1, "step_ms": 0.5},
// so the file is JSON and a line-by-line reader finds an entry.
static std::string tune_key(const paratc_ctx* ctx) {
    cudaDeviceProp pr;
    std::memset(&pr, 0, sizeof(pr));
    cudaGetDeviceProperties(&pr, ctx->dev);
    char b[384];
    std::snprintf(b, sizeof(b), "%s|%dx%dx%d|s%d|p%d|f%d", pr.name, ctx->nx, ctx->ny, ctx->nz, ctx->prm.scalar_on ? 1 : 0,
                  ctx->prec, ctx->prm.flow_type);
    return b;
}

static bool tune_field(const std::string& line, const char* name, double* v) {
    const std::string pat = std::string("\"") + name + "\":";
    const size_t p = line.find(pat);
    if (p == std::string::npos) return false;
    return std::sscanf(line.c_str() + p + pat.size(), "%lf", v) == 1;
}

// the cached entry of `key` in `path` (false when the file or the entry is missing)
static bool tune_cache_read(const char* path, const std::string& key, paratc_tuning* t) {
    FILE* fp = path ? std::fopen(path, "r") : nullptr;
    if (!fp) return false;
    char buf[1024];
    bool found = false;
    const std::string k = "\"" + key + "\":";
    while (!found && std::fgets(buf, sizeof(buf), fp)) {
        const std::string line(buf);
        if (line.find(k) == std::string::npos) continue;
        double sc, rv, hv, ms = 0.0;
        if (tune_field(line, "schedule", &sc) && tune_field(line, "rhs_var", &rv) && tune_field(line, "helm_var", &hv)) {
            tune_field(line, "step_ms", &ms);
            t->schedule = (int32_t)sc;
            t->rhs_var = (int32_t)rv;
            t->helm_var = (int32_t)hv;
            t->step_ms = ms;
            found = true;
        }
    }
    std::fclose(fp);
    return found;
}

// adds or replaces the entry of `key`, keeping the others
static int tune_cache_write(const char* path, const std::string& key, const paratc_tuning& t) {
    std::vector<std::string> keep;
    const std::string k = "\"" + key + "\":";
    if (FILE* fp = std::fopen(path, "r")) {
        char buf[1024];
        while (std::fgets(buf, sizeof(buf), fp)) {
            std::string line(buf);
            while (!line.empty() && (line.back() == '\n' || line.back() == ',' || line.back() == ' ')) line.pop_back();
            if (line.find("\": {") == std::string::npos || line.find(k) != std::string::npos) continue;
            keep.push_back(line);
        }
        std::fclose(fp);
    }
    char b[640];
    std::snprintf(b, sizeof(b), "  \"%s\": {\"schedule\": %d, \"rhs_var\": %d, \"helm_var\": %d, \"step_ms\": %.6f}",
                  key.c_str(), t.schedule, t.rhs_var, t.helm_var, t.step_ms);
    keep.push_back(b);
    FILE* fp = std::fopen(path, "w");
    if (!fp) return PARATC_ERR_IO;
    std::fprintf(fp, "{\n");
    for (size_t q = 0; q < keep.size(); q++) std::fprintf(fp, "%s%s\n", keep[q].c_str(), q + 1 < keep.size() ? "," : "");
    std::fprintf(fp, "}\n");
    std::fclose(fp);
    return PARATC_OK;
}

static bool tuning_valid(const paratc_ctx* ctx, const paratc_tuning& t) {
    return sched_supported(ctx, t.schedule) && t.rhs_var >= 0 && t.rhs_var < rhs_variants(ctx->prec) && t.helm_var >= 0 &&
           t.helm_var < helm_variants(ctx->prec) && !(ctx->prec == PARATC_PREC_FP32 && t.schedule / 2 == 2);
}

static void tuning_apply(paratc_ctx* ctx, const paratc_tuning& t) {
    sched_apply(ctx, t.schedule);
    ctx->kc.rhs_var = t.rhs_var;
    ctx->kc.helm_var = t.helm_var;
}

}  // extern "C++"

int paratc_get_tuning(paratc_ctx* ctx, paratc_tuning* t) {
    if (!ctx || !t) return PARATC_ERR_BAD_ARG;
    int sc = 0;
    paratc_get_schedule(ctx, &sc);
    t->schedule = sc;
    t->rhs_var = ctx->kc.rhs_var;
    t->helm_var = ctx->kc.helm_var;
    t->from_cache = ctx->tune_from_cache;
    t->step_ms = ctx->tune_step_ms;
    return PARATC_OK;
}

int paratc_set_tuning(paratc_ctx* ctx, const paratc_tuning* t) {
    if (!ctx || !t || !tuning_valid(ctx, *t)) return PARATC_ERR_BAD_ARG;
    tuning_apply(ctx, *t);
    ctx->tune_from_cache = 0;
    return PARATC_OK;
}

int paratc_autotune_all(paratc_ctx* ctx, int nrep, const char* cache_path, paratc_tuning* out) {
    if (!ctx || nrep < 1) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    const std::string key = tune_key(ctx);
    paratc_tuning t;
    std::memset(&t, 0, sizeof(t));
    if (tune_cache_read(cache_path, key, &t) && tuning_valid(ctx, t)) {
        tuning_apply(ctx, t);
        ctx->tune_from_cache = 1;
        ctx->tune_step_ms = t.step_ms;
        return paratc_get_tuning(ctx, out ? out : &t);
    }
    // 1. the Poisson schedule (InitPoissonSolver's search, src/m_Poisson.f90:50-175)
    int sched = 0;
    int rc = paratc_autotune(ctx, nrep, &sched, nullptr);
    if (rc) return rc;
    // 2. the launch shapes, timed by whole steps from a saved state that is
    // put back afterwards (u, v, w, p, c, histories, uy_ym, the coefficients)
    rc = sync(ctx);
    if (rc) return rc;
    const bool fp32 = ctx->prec == PARATC_PREC_FP32;
    std::vector<std::pair<void*, size_t>> st;
    const size_t nb64 = ctx->nf * sizeof(double), nb32 = ctx->nf * sizeof(float);
    if (fp32) {
        for (float* q : {ctx->f32.ux, ctx->f32.uy, ctx->f32.uz, ctx->f32.hx, ctx->f32.hy, ctx->f32.hz, ctx->f32.sc, ctx->f32.hc})
            if (q) st.push_back({q, nb32});
    } else {
        for (double* q : {ctx->f.ux, ctx->f.uy, ctx->f.uz, ctx->f.hx, ctx->f.hy, ctx->f.hz, ctx->f.sc, ctx->f.hc})
            if (q) st.push_back({q, nb64});
    }
    st.push_back({ctx->f.pr, nb64});
    st.push_back({ctx->d_uy_ym, (size_t)ctx->nx * ctx->nz * sizeof(double)});
    st.push_back({ctx->d_duy_ym, (size_t)ctx->nx * ctx->nz * sizeof(double)});
    st.push_back({ctx->d_coef, sizeof(DCoef)});
    size_t total = 0;
    for (auto& e : st) total += (e.second + 255) & ~(size_t)255;
    char* save = nullptr;
    CK(cudaMalloc(&save, total));
    auto copy_all = [&](bool to_save) {
        size_t o = 0;
        for (auto& e : st) {
            cudaMemcpyAsync(to_save ? save + o : e.first, to_save ? e.first : save + o, e.second,
                            cudaMemcpyDeviceToDevice, ctx->st);
            o += (e.second + 255) & ~(size_t)255;
        }
    };
    copy_all(true);
    const bool ready0 = ctx->next_ready;
    const double hdt0 = ctx->hfac_dt;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int nr = rhs_variants(ctx->prec);  // FP64 3 launch shapes, FP32 storage 2, mixed 1
    float best = -1.f;
    paratc_tuning bt = {sched, 0, 0, 0, 0.0};
    for (int rv = 0; rv < nr; rv++)
        for (int hv = 0; hv < helm_variants(ctx->prec); hv++) {
            ctx->kc.rhs_var = rv;
            ctx->kc.helm_var = hv;
            copy_all(false);
            ctx->next_ready = false;
            ctx->hfac_dt = -1.0;
            enqueue_step(ctx);  // warm-up
            cudaEventRecord(e0, ctx->st);
            for (int q = 0; q < nrep; q++) enqueue_step(ctx);
            cudaEventRecord(e1, ctx->st);
            if ((rc = sync(ctx))) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= (float)nrep;
            if (best < 0.f || ms < best) { best = ms; bt.rhs_var = rv; bt.helm_var = hv; }
        }
    copy_all(false);
    CK(cudaMemsetAsync(ctx->d_diag, 0, sizeof(DDiag), ctx->st));
    const int rc2 = sync(ctx);
    cudaFree(save);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->next_ready = false;
    ctx->hfac_dt = -1.0;
    (void)ready0;
    (void)hdt0;
    if (rc) return rc;
    if (rc2) return rc2;
    bt.step_ms = best;
    tuning_apply(ctx, bt);
    ctx->sched_gen++;
    ctx->tune_from_cache = 0;
    ctx->tune_step_ms = best;
    if (cache_path && (rc = tune_cache_write(cache_path, key, bt)))
        return set_err(ctx, rc, std::string("cannot write the tuning cache ") + cache_path);
    return paratc_get_tuning(ctx, out ? out : &bt);
}

int paratc_project(paratc_ctx* ctx, double* divmax_out) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    ctx->next_ready = false;
    if (ctx->prec == PARATC_PREC_FP32) {
        launch_bc_all(ctx->st, ctx->kc, ctx->f32, ctx->d_uy_ym);
        enqueue_poisson_head32(ctx, 1, ctx->d_scal);
        enqueue_poisson_tail32(ctx, ctx->d_phi32, 1);
        launch_project(ctx->st, ctx->kc, ctx->dm, ctx->d_coef, 1, ctx->d_phi32, ctx->f32, ctx->d_uy_ym);
        launch_prsrc(ctx->st, ctx->kc, ctx->dm, ctx->d_coef, 1, ctx->f32, nullptr, ctx->d_part, ctx->d_scal + 1);
    } else {
        launch_bc_all(ctx->st, ctx->kc, ctx->f, ctx->d_uy_ym);
        enqueue_poisson_head(ctx, 1, nullptr, ctx->d_scal);
        enqueue_poisson_tail(ctx, ctx->d_phi, 1);
        launch_project(ctx->st, ctx->kc, ctx->dm, ctx->d_coef, 1, ctx->d_phi, ctx->f, ctx->d_uy_ym);
        launch_prsrc(ctx->st, ctx->kc, ctx->dm, ctx->d_coef, 1, ctx->f, nullptr, ctx->d_part, ctx->d_scal + 1);
    }
    ctx->launches += 4;
    CK(cudaMemcpyAsync(ctx->h_scal, ctx->d_scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    int rc = sync(ctx);
    if (rc) return rc;
    if (divmax_out) *divmax_out = ctx->h_scal[1];
    return PARATC_OK;
}

int paratc_diagnostics(paratc_ctx* ctx, paratc_diag* diag) {
    if (!ctx || !diag) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaMemsetAsync(ctx->d_diag2, 0, sizeof(DDiag), ctx->st));
    if (ctx->prec == PARATC_PREC_FP32)
        launch_endstep(ctx->st, ctx->kc, ctx->dm, ctx->f32, ctx->d_coef, ctx->d_diag2, ctx->d_part, ctx->d_counter + 3, 0);
    else
        launch_endstep(ctx->st, ctx->kc, ctx->dm, ctx->f, ctx->d_coef, ctx->d_diag2, ctx->d_part, ctx->d_counter + 3, 0);
    ctx->launches += 1;
    CK(cudaMemcpyAsync(ctx->h_diag, ctx->d_diag2, sizeof(DDiag), cudaMemcpyDeviceToHost, ctx->st));
    int rc = sync(ctx);
    if (rc) return rc;
    diag_out(*ctx->h_diag, diag);
    return PARATC_OK;
}

int paratc_xprofile(paratc_ctx* ctx, int field, double* out) {
    if (!ctx || !out || field < 0 || field > 4) return PARATC_ERR_BAD_ARG;
    const double* q[5] = {ctx->f.ux, ctx->f.uy, ctx->f.uz, ctx->f.pr, ctx->f.sc};
    if (!q[field]) return set_err(ctx, PARATC_ERR_BAD_ARG, "xprofile: no scalar in this context");
    CK(cudaSetDevice(ctx->dev));
    // d_src (nx*ny*nz doubles, ny >= 3) is free between substeps: the nx*nz
    // column sums, then the profile
    double* part = ctx->d_src;
    double* prof = ctx->d_src + (size_t)ctx->nx * ctx->nz;
    const float* q32[5] = {ctx->f32.ux, ctx->f32.uy, ctx->f32.uz, nullptr, ctx->f32.sc};
    if (ctx->prec == PARATC_PREC_FP32 && field != 3) launch_xprofile(ctx->st, ctx->kc, ctx->dm, q32[field], part, prof);
    else launch_xprofile(ctx->st, ctx->kc, ctx->dm, q[field], part, prof);
    ctx->launches += 2;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, prof, (size_t)ctx->nx * sizeof(double), cudaMemcpyDefault, ctx->st));
    return sync(ctx);
}

int paratc_front_position(paratc_ctx* ctx, double x_from, double level, double* x_front) {
    if (!ctx || !x_front) return PARATC_ERR_BAD_ARG;
    if (!ctx->prm.scalar_on) return set_err(ctx, PARATC_ERR_BAD_ARG, "front position: no scalar in this context");
    std::vector<double> prof(ctx->nx);
    int rc = paratc_xprofile(ctx, 4, prof.data());
    if (rc) return rc;
    // the nose: the furthest cell centre right of x_from, within half the
    // periodic domain, whose depth average is at least `level`, and the
    // linear crossing of the level between it and the next cell
    const int nx = ctx->nx;
    const double dx = ctx->prm.xlx / nx;
    *x_front = -1.0;
    int last = -1;
    for (int i = 0; i < nx; i++) {
        const double x = (i + 0.5) * dx;
        if (x > x_from && x < x_from + 0.5 * ctx->prm.xlx && prof[i] >= level) last = i;
    }
    if (last < 0) return PARATC_OK;
    const double xl = (last + 0.5) * dx;
    const double pn = prof[(last + 1) % nx];
    *x_front = pn < level ? xl + (prof[last] - level) / (prof[last] - pn) * dx : xl;
    return PARATC_OK;
}

// restart files: write_restart / read_restart (src/m_IOAndVisu.f90:408-512)
int paratc_write_restart(paratc_ctx* ctx, const char* path, int with_hist) {
    if (!ctx || !path) return PARATC_ERR_BAD_ARG;
    const size_t n = ctx->ni;
    std::vector<double> buf(n);
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return set_err(ctx, PARATC_ERR_IO, std::string("cannot open ") + path);
    refresh64(ctx);
    std::vector<double*> order = {ctx->f.ux, ctx->f.uy, ctx->f.uz, ctx->f.pr};
    if (ctx->prm.scalar_on) order.push_back(ctx->f.sc);
    if (with_hist) {
        order.push_back(ctx->f.hx); order.push_back(ctx->f.hy); order.push_back(ctx->f.hz);
        if (ctx->prm.scalar_on) order.push_back(ctx->f.hc);
    }
    for (size_t a = 0; a < order.size(); a++) {
        int rc = copy_field(ctx, order[a], nullptr, buf.data(), PARATC_LAYOUT_INTERIOR, false);
        if (rc == PARATC_OK) rc = sync(ctx);
        if (rc) { std::fclose(fp); return rc; }
        if (a == 0)
            for (size_t q = 0; q < n; q++) buf[q] = buf[q] + ctx->prm.ucrf;
        if (std::fwrite(buf.data(), sizeof(double), n, fp) != n) {
            std::fclose(fp);
            return set_err(ctx, PARATC_ERR_IO, "short write");
        }
    }
    std::fclose(fp);
    return PARATC_OK;
}

int paratc_read_restart(paratc_ctx* ctx, const char* path) {
    if (!ctx || !path) return PARATC_ERR_BAD_ARG;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return set_err(ctx, PARATC_ERR_IO, std::string("Cannot open file: ") + path);
    std::fseek(fp, 0, SEEK_END);
    const long long bytes = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    const size_t n = ctx->ni;
    const long long unit = (long long)n * (long long)sizeof(double);
    const int nb = ctx->prm.scalar_on ? 5 : 4, nh = ctx->prm.scalar_on ? 9 : 7;
    if (bytes != unit * nb && bytes != unit * nh) {
        std::fclose(fp);
        return set_err(ctx, PARATC_ERR_IO, "file byte wrong");
    }
    const bool hist = (bytes == unit * nh);
    std::vector<std::vector<double>> arr(nh, std::vector<double>());
    const int nread = hist ? nh : nb;
    for (int a = 0; a < nread; a++) {
        arr[a].resize(n);
        if (std::fread(arr[a].data(), sizeof(double), n, fp) != n) {
            std::fclose(fp);
            return set_err(ctx, PARATC_ERR_IO, "short read");
        }
    }
    std::fclose(fp);
    for (size_t q = 0; q < n; q++) arr[0][q] = arr[0][q] - ctx->prm.ucrf;
    const double* c = ctx->prm.scalar_on ? arr[4].data() : nullptr;
    const int h0 = nb;
    const double* hx = hist ? arr[h0].data() : nullptr;
    const double* hy = hist ? arr[h0 + 1].data() : nullptr;
    const double* hz = hist ? arr[h0 + 2].data() : nullptr;
    const double* hc = (hist && ctx->prm.scalar_on) ? arr[h0 + 3].data() : nullptr;
    int rc = paratc_set_fields(ctx, arr[0].data(), arr[1].data(), arr[2].data(), arr[3].data(), c, hx, hy, hz, hc,
                               PARATC_LAYOUT_INTERIOR);
    return rc;
}

int paratc_stats_reset(paratc_ctx* ctx) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    CK(cudaMemsetAsync(ctx->d_stats, 0, ((size_t)ctx->nyp * 40 + 1) * sizeof(double), ctx->st));
    ctx->nfstime = 0;
    return sync(ctx);
}

int paratc_stats_accumulate(paratc_ctx* ctx) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    refresh64(ctx);
    const int ns = stats_count(ctx->kc);
    launch_stats(ctx->st, ctx->kc, ctx->dm, ctx->f, ctx->d_coef, ctx->d_stats_part, ctx->d_stats,
                 ctx->d_stats + (size_t)ctx->nyp * ns);
    ctx->launches += 2;
    ctx->nfstime += 1;
    CK(cudaGetLastError());
    return PARATC_OK;
}

int paratc_stats_get(paratc_ctx* ctx, double* sumstat, int* nstat, int* nfstime, double* prgradsum) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    const int ns = stats_count(ctx->kc);
    if (nstat) *nstat = ns;
    if (nfstime) *nfstime = ctx->nfstime;
    if (sumstat) CK(cudaMemcpyAsync(sumstat, ctx->d_stats, (size_t)ctx->nyp * ns * sizeof(double), cudaMemcpyDefault, ctx->st));
    if (prgradsum) CK(cudaMemcpyAsync(prgradsum, ctx->d_stats + (size_t)ctx->nyp * ns, sizeof(double), cudaMemcpyDefault, ctx->st));
    return sync(ctx);
}


// the spectra accumulators, partial records and full-length x twiddles, on first use
static int spectra_alloc(paratc_ctx* ctx) {
    if (ctx->d_specx) return PARATC_OK;
    if (!spectra_supported(ctx->nx) || !spectra_supported(ctx->nz))
        return set_err(ctx, PARATC_ERR_BAD_ARG, "spectra: no transform kernel for nx or nz");
    int rc;
    const std::vector<double2> tw = twiddles(ctx->nx, ctx->nx);
    if ((rc = dalloc(ctx, &ctx->d_specx, (size_t)9 * ctx->ny * (ctx->nx / 2 + 1))) ||
        (rc = dalloc(ctx, &ctx->d_specz, (size_t)9 * ctx->ny * (ctx->nz / 2 + 1))) ||
        (rc = dalloc(ctx, &ctx->d_spec_part, spectra_part_doubles(ctx->kc))) ||
        (rc = dalloc(ctx, &ctx->d_twxf, tw.size())))
        return rc;
    CK(cudaMemcpyAsync(ctx->d_twxf, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    ctx->nspectime = 0;
    return sync(ctx);
}

int paratc_spectra_reset(paratc_ctx* ctx) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    int rc = spectra_alloc(ctx);
    if (rc != PARATC_OK) return rc;
    CK(cudaMemsetAsync(ctx->d_specx, 0, (size_t)9 * ctx->ny * (ctx->nx / 2 + 1) * sizeof(double), ctx->st));
    CK(cudaMemsetAsync(ctx->d_specz, 0, (size_t)9 * ctx->ny * (ctx->nz / 2 + 1) * sizeof(double), ctx->st));
    ctx->nspectime = 0;
    return sync(ctx);
}

int paratc_spectra_accumulate(paratc_ctx* ctx, int jlcs) {
    if (!ctx || jlcs < 1 || jlcs > ctx->ny) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    int rc = spectra_alloc(ctx);
    if (rc != PARATC_OK) return rc;
    refresh64(ctx);
    launch_spectra(ctx->st, 0, ctx->kc, ctx->f, jlcs, ctx->d_twxf, ctx->d_spec_part, ctx->d_specx);
    launch_spectra(ctx->st, 1, ctx->kc, ctx->f, jlcs, ctx->d_twz, ctx->d_spec_part, ctx->d_specz);
    ctx->launches += 4;
    ctx->nspectime += 1;
    CK(cudaGetLastError());
    return PARATC_OK;
}

int paratc_spectra_get(paratc_ctx* ctx, double* spec_x, double* spec_z, int* nspec, int* nspectime) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    const int nsp = spectra_count(ctx->kc);
    if (nspec) *nspec = nsp;
    if (nspectime) *nspectime = ctx->nspectime;
    if (!spec_x && !spec_z) return PARATC_OK;
    int rc = spectra_alloc(ctx);
    if (rc != PARATC_OK) return rc;
    if (spec_x)
        CK(cudaMemcpyAsync(spec_x, ctx->d_specx, (size_t)nsp * ctx->ny * (ctx->nx / 2 + 1) * sizeof(double),
                           cudaMemcpyDefault, ctx->st));
    if (spec_z)
        CK(cudaMemcpyAsync(spec_z, ctx->d_specz, (size_t)nsp * ctx->ny * (ctx->nz / 2 + 1) * sizeof(double),
                           cudaMemcpyDefault, ctx->st));
    return sync(ctx);
}

int paratc_spectra2d_setup(paratc_ctx* ctx, int nsel, const int* iy) {
    if (!ctx || nsel < 1 || !iy) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    const int ny = ctx->ny, nyp = ctx->nyp;
    const int jmax = ctx->prm.flow_type == PARATC_FT_CH ? ny / 2 : ny;
    for (int q = 0; q < nsel; q++)
        if (iy[q] < 2 || iy[q] > jmax) return set_err(ctx, PARATC_ERR_BAD_ARG, "spectra2d: iySpec2D out of range");
    int rc = spectra_alloc(ctx);  // the full-length x twiddles
    if (rc != PARATC_OK) return rc;
    const int nmir = ctx->prm.flow_type == PARATC_FT_HC ? 1 : 2;
    const int nfld = ctx->prm.scalar_on ? 7 : 6;
    std::vector<int2> fj;
    for (int q = 0; q < nsel; q++)
        for (int f = 0; f < nfld; f++)
            for (int h = 0; h < nmir; h++) {
                const int jct = iy[q];
                const int row = h == 0 ? jct : (f == 1 ? nyp + 1 - jct : ny + 1 - jct);
                fj.push_back(make_int2(f, row));
            }
    const int nsp = ctx->prm.scalar_on ? 6 : 5;
    const size_t pl = (size_t)ctx->nx * ctx->nz;
    const size_t need_out = (size_t)nsp * nsel * pl, need_s = fj.size() * pl;
    // grow the buffers (the old ones are released; nothing is in flight on
    // them once the stream is idle)
    if (need_out > ctx->spec2d_cap || need_s > ctx->s2_cap || fj.size() > ctx->fj_cap) {
        if ((rc = sync(ctx))) return rc;
    }
    if (need_out > ctx->spec2d_cap) {
        dfree(ctx, &ctx->d_spec2d);
        ctx->spec2d_cap = 0;
        if ((rc = dalloc(ctx, &ctx->d_spec2d, need_out))) return rc;
        ctx->spec2d_cap = need_out;
    }
    if (need_s > ctx->s2_cap) {
        dfree(ctx, &ctx->d_s2);
        ctx->s2_cap = 0;
        if ((rc = dalloc(ctx, &ctx->d_s2, need_s))) return rc;
        ctx->s2_cap = need_s;
    }
    if (fj.size() > ctx->fj_cap) {
        dfree(ctx, &ctx->d_fj);
        ctx->fj_cap = 0;
        if ((rc = dalloc(ctx, &ctx->d_fj, fj.size()))) return rc;
        ctx->fj_cap = fj.size();
    }
    CK(cudaMemcpyAsync(ctx->d_fj, fj.data(), fj.size() * sizeof(int2), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemsetAsync(ctx->d_spec2d, 0, need_out * sizeof(double), ctx->st));
    ctx->nsel2 = nsel;
    ctx->nfj2 = (int)fj.size();
    ctx->nmir2 = nmir;
    ctx->nfld2 = nfld;
    ctx->nspectime2 = 0;
    return sync(ctx);
}

int paratc_spectra2d_reset(paratc_ctx* ctx) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    if (ctx->nsel2 == 0) return set_err(ctx, PARATC_ERR_BAD_ARG, "spectra2d: not set up");
    CK(cudaSetDevice(ctx->dev));
    const size_t n = (size_t)(ctx->prm.scalar_on ? 6 : 5) * ctx->nsel2 * ctx->nx * ctx->nz;
    CK(cudaMemsetAsync(ctx->d_spec2d, 0, n * sizeof(double), ctx->st));
    ctx->nspectime2 = 0;
    return sync(ctx);
}

int paratc_spectra2d_accumulate(paratc_ctx* ctx) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    if (ctx->nsel2 == 0) return set_err(ctx, PARATC_ERR_BAD_ARG, "spectra2d: not set up");
    CK(cudaSetDevice(ctx->dev));
    refresh64(ctx);
    launch_spectra2d(ctx->st, ctx->kc, ctx->f, ctx->d_fj, ctx->nfj2, ctx->nsel2, ctx->nmir2, ctx->nfld2, ctx->d_twxf,
                     ctx->d_twz, ctx->d_s2, ctx->d_spec2d);
    ctx->launches += 3;
    ctx->nspectime2 += 1;
    CK(cudaGetLastError());
    return PARATC_OK;
}

int paratc_spectra2d_get(paratc_ctx* ctx, double* out, int* nspec, int* nsel, int* nspectime) {
    if (!ctx) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    const int nsp = ctx->prm.scalar_on ? 6 : 5;
    if (nspec) *nspec = nsp;
    if (nsel) *nsel = ctx->nsel2;
    if (nspectime) *nspectime = ctx->nspectime2;
    if (!out || ctx->nsel2 == 0) return PARATC_OK;
    CK(cudaMemcpyAsync(out, ctx->d_spec2d, (size_t)nsp * ctx->nsel2 * ctx->nx * ctx->nz * sizeof(double),
                       cudaMemcpyDefault, ctx->st));
    return sync(ctx);
}

const char* paratc_visu_name(int q) {
    static const char* names[PARATC_VISU_NQ] = {"ux", "uy", "uz", "pr", "wx", "wy", "wz", "wMag", "Q", "lamda2", "scalar"};
    return (q >= 0 && q < PARATC_VISU_NQ) ? names[q] : "";
}

int paratc_visu_quantity(paratc_ctx* ctx, int q, int iskip, int jskip, int kskip, int node, double* out,
                         int64_t* count) {
    if (!ctx || q < 0 || q >= PARATC_VISU_NQ || iskip < 1 || jskip < 1 || kskip < 1) return PARATC_ERR_BAD_ARG;
    if (q == PARATC_VISU_SCALAR && !ctx->prm.scalar_on) return PARATC_ERR_BAD_ARG;
    const int64_t n = (int64_t)visu_count(ctx->nx, iskip) * visu_count(ctx->ny, jskip) * visu_count(ctx->nz, kskip);
    if (count) *count = n;
    if (!out) return PARATC_OK;
    CK(cudaSetDevice(ctx->dev));
    int rc;
    if (!ctx->d_visu) {
        if ((rc = dalloc(ctx, &ctx->d_visu, ctx->ni)) || (rc = dalloc(ctx, &ctx->d_visu_bad, 1))) return rc;
    }
    CK(cudaMemsetAsync(ctx->d_visu_bad, 0, sizeof(unsigned int), ctx->st));
    refresh64(ctx);
    launch_visu(ctx->st, q, iskip, jskip, kskip, node, ctx->kc, ctx->dm, ctx->f, ctx->d_visu, ctx->d_visu_bad);
    ctx->launches += 1;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->d_visu, (size_t)n * sizeof(double), cudaMemcpyDefault, ctx->st));
    unsigned int* hb = reinterpret_cast<unsigned int*>(ctx->h_scal);
    CK(cudaMemcpyAsync(hb, ctx->d_visu_bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->st));
    if ((rc = sync(ctx))) return rc;
    if (*hb) {
        char b[128];
        std::snprintf(b, sizeof(b), "lamda2 wrong: %u points with complex roots", *hb);
        return set_err(ctx, PARATC_ERR_NUMERIC, b);
    }
    return PARATC_OK;
}

int paratc_visu_quantity_device(paratc_ctx* ctx, int q, int iskip, int jskip, int kskip, int node, double* d_out,
                                unsigned int* d_nbad) {
    if (!ctx || !d_out || q < 0 || q >= PARATC_VISU_NQ || iskip < 1 || jskip < 1 || kskip < 1) return PARATC_ERR_BAD_ARG;
    if (q == PARATC_VISU_SCALAR && !ctx->prm.scalar_on) return PARATC_ERR_BAD_ARG;
    CK(cudaSetDevice(ctx->dev));
    if (!d_nbad) {
        if (!ctx->d_visu_bad) {
            int rc = dalloc(ctx, &ctx->d_visu_bad, 1);
            if (rc) return rc;
        }
        d_nbad = ctx->d_visu_bad;
    }
    refresh64(ctx);
    launch_visu(ctx->st, q, iskip, jskip, kskip, node, ctx->kc, ctx->dm, ctx->f, d_out, d_nbad);
    ctx->launches += 1;
    CK(cudaGetLastError());
    return PARATC_OK;
}

int paratc_dump_visu(paratc_ctx* ctx, const char* res_dir, const char* run_name, int ntime, int save_mask, int iskip,
                     int jskip, int kskip, int node, int single) {
    if (!ctx || !res_dir || !run_name || ntime < 0) return PARATC_ERR_BAD_ARG;
    // the order dump_visu writes them in
    const int order[PARATC_VISU_NQ] = {PARATC_VISU_UX, PARATC_VISU_UY, PARATC_VISU_UZ, PARATC_VISU_PR,
                                       PARATC_VISU_SCALAR, PARATC_VISU_WX, PARATC_VISU_WY, PARATC_VISU_WZ,
                                       PARATC_VISU_WMAG, PARATC_VISU_Q, PARATC_VISU_LAMDA2};
    int64_t n = 0;
    int rc = paratc_visu_quantity(ctx, PARATC_VISU_UX, iskip, jskip, kskip, node, nullptr, &n);
    if (rc) return rc;
    std::vector<double> buf((size_t)n);
    std::vector<float> fbuf(single ? (size_t)n : 0);
    for (int a = 0; a < PARATC_VISU_NQ; a++) {
        const int q = order[a];
        if (!(save_mask & (1 << q))) continue;
        if (q == PARATC_VISU_SCALAR && !ctx->prm.scalar_on) continue;
        if ((rc = paratc_visu_quantity(ctx, q, iskip, jskip, kskip, node, buf.data(), nullptr))) return rc;
        char tail[32];
        std::snprintf(tail, sizeof(tail), "_%010d", ntime);
        const std::string path = std::string(res_dir) + "VisuFor" + run_name + "_" + paratc_visu_name(q) + tail;
        FILE* fp = std::fopen(path.c_str(), "wb");
        if (!fp) return set_err(ctx, PARATC_ERR_IO, "Cannot open file: " + path);
        size_t w;
        if (single) {
            for (size_t e = 0; e < buf.size(); e++) fbuf[e] = (float)buf[e];
            w = std::fwrite(fbuf.data(), sizeof(float), fbuf.size(), fp);
        } else {
            w = std::fwrite(buf.data(), sizeof(double), buf.size(), fp);
        }
        std::fclose(fp);
        if (w != buf.size()) return set_err(ctx, PARATC_ERR_IO, "short write: " + path);
    }
    return PARATC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// ensembles
// ---------------------------------------------------------------------------
namespace {

// one launch of a grouped step
struct GrpLaunch {
    std::function<void(cudaStream_t)> run;
};

// the grouped form of a step: every stage is one launch per kernel
// instantiation over the members that share it (GrpTab, kernels.cuh)
struct GrpPlan {
    std::vector<void*> dev;                   // device tables
    std::vector<paratc_ctx*> fac;             // members whose Helmholtz pivots change every step (iCFL = 1)
    std::vector<std::vector<GrpLaunch>> sub;  // the launches of substep ns at index ns - 1
    std::vector<GrpLaunch> end;               // end of step
    std::vector<int> gens;                    // the members' sched_gen the tables were built from
    int64_t kernels = 0;                      // launches per step
    bool built = false;
};

void grp_free(GrpPlan& P) {
    for (void* d : P.dev) cudaFree(d);
    P = GrpPlan();
}

}  // namespace

struct paratc_batch {
    int n = 0, dev = 0;
    std::vector<paratc_ctx*> m;
    cudaStream_t st = nullptr;          // stream the graph is captured on and launched from
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;      // one per member
    cudaGraphExec_t exec = nullptr;
    std::vector<int> gens;              // the members' sched_gen when the graph was captured
    bool graph_failed = false;
    int64_t graph_kernels = 0;
    int mode = PARATC_BATCH_STREAMS;    // PARATC_BATCH_STREAMS or PARATC_BATCH_GROUPED
    GrpPlan plan;                       // the grouped launches (PARATC_BATCH_GROUPED)
    std::string err;
};

namespace {

// a member whose next step is the steady step the graph holds: clcCFL done by
// its last end-of-step kernel, Helmholtz pivots current (or recomputed every
// step, iCFL = 1)
bool member_steady(const paratc_ctx* c) {
    return c->next_ready && (c->prm.icfl == 1 || c->hfac_dt == c->prm.dt_max);
}

void batch_free_graph(paratc_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
}

// b->st waits for everything already queued on the member streams
cudaError_t batch_join_members(paratc_batch* b) {
    for (int i = 0; i < b->n; i++) {
        cudaError_t e = cudaEventRecord(b->join[i], b->m[i]->st);
        if (e != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(b->st, b->join[i], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// the member streams wait for everything queued on b->st
cudaError_t batch_fork_members(paratc_batch* b) {
    cudaError_t e = cudaEventRecord(b->done, b->st);
    if (e != cudaSuccess) return e;
    for (int i = 0; i < b->n; i++)
        if ((e = cudaStreamWaitEvent(b->m[i]->st, b->done, 0)) != cudaSuccess) return e;
    return cudaSuccess;
}

// ---- grouped launches -------------------------------------------------------

// the members gathered for one kernel instantiation
template <class E>
struct GrpAcc {
    DConst key{};  // a member's constants: the launcher picks the instantiation from them
    std::vector<E> e;
    std::vector<dim3> g;
    size_t smem = 0;  // the largest member's dynamic shared memory
    void add(const DConst& k, const E& x, dim3 grid, size_t sm = 0) {
        if ((size_t)grid.x * grid.y * grid.z == 0) return;  // nothing to do for this member
        if (e.empty()) key = k;
        e.push_back(x);
        g.push_back(grid);
        smem = std::max(smem, sm);
    }
};

// the tables of one instantiation on the device, PT_MAXMEM members each,
// with the CTA count of each
template <class E>
bool grp_upload(GrpPlan& P, const GrpAcc<E>& a, std::vector<std::pair<const GrpTab<E>*, int>>& out) {
    for (size_t s0 = 0; s0 < a.e.size(); s0 += PT_MAXMEM) {
        const int n = (int)std::min<size_t>(PT_MAXMEM, a.e.size() - s0);
        std::unique_ptr<GrpTab<E>> h(new GrpTab<E>());
        h->nmem = n;
        long long blk = 0;
        for (int i = 0; i < n; i++) {
            const dim3 g = a.g[s0 + i];
            h->b0[i] = (int)blk;
            h->g[i][0] = g.x;
            h->g[i][1] = g.y;
            h->g[i][2] = g.z;
            h->e[i] = a.e[s0 + i];
            blk += (long long)g.x * g.y * g.z;
        }
        if (blk > 0x7fffffffLL) return false;
        h->b0[n] = (int)blk;
        void* d = nullptr;
        if (cudaMalloc(&d, sizeof(GrpTab<E>)) != cudaSuccess) return false;
        P.dev.push_back(d);
        if (cudaMemcpy(d, h.get(), sizeof(GrpTab<E>), cudaMemcpyHostToDevice) != cudaSuccess) return false;
        out.push_back({static_cast<const GrpTab<E>*>(d), (int)blk});
    }
    return true;
}

// the right-hand-side CTAs of a group: one wave of the device shared by the
// members in proportion to their rows, at least one each and at most the
// member's own block count (each CTA runs consecutive logical blocks of its
// member, see rhs_body)
template <class K, class V>
void grp_balance_rhs(std::map<K, GrpAcc<RhsArgs<V>>>& m) {
    for (auto& kv : m) {
        GrpAcc<RhsArgs<V>>& a = kv.second;
        long long tot = 0;
        for (auto& e : a.e) tot += rhs_work_rows(e.c);
        if (tot <= 0 || a.e.empty()) continue;
        const long long wave = rhs_wave(a.e[0].c);
        for (size_t i = 0; i < a.e.size(); i++) {
            const long long w = rhs_work_rows(a.e[i].c);
            long long b = (wave * w + tot / 2) / tot;
            b = std::max(1LL, std::min(b, (long long)a.e[i].nlog));
            a.g[i] = dim3((unsigned)b);
        }
    }
}

// one launch per table of every instantiation in m, in key order
template <class K, class E, class F>
bool grp_emit(GrpPlan& P, std::map<K, GrpAcc<E>>& m, std::vector<GrpLaunch>& out, F launch) {
    for (auto& kv : m) {
        std::vector<std::pair<const GrpTab<E>*, int>> tabs;
        if (!grp_upload(P, kv.second, tabs)) return false;
        const K key = kv.first;
        const DConst kc = kv.second.key;
        const size_t smem = kv.second.smem;
        for (auto& t : tabs) {
            const GrpTab<E>* tab = t.first;
            const int nblk = t.second;
            out.push_back({[=](cudaStream_t st) { launch(st, key, kc, tab, nblk, smem); }});
        }
    }
    return true;
}

// the Poisson schedule of the grouped step: the separate compile-time-length
// x and z transforms with register-fed z passes (choice 2 or 3, the y-solve
// kind kept), the form every member of a table shares
bool grp_schedule(paratc_ctx* c) {
    const int y = c->kc.solver_sel == 2 ? 1 : 0;
    const bool ok = c->pfft && !c->plane && !c->ztma && !c->xdiv;
    if (ok) return true;
    if (!sched_supported(c, 2 + y)) return false;
    sched_apply(c, 2 + y);
    return true;
}

// the grouped form of the k_xb launch: the plain kernel (no bulk copies)
int grp_build(paratc_batch* b) {
    grp_free(b->plan);
    GrpPlan& P = b->plan;
    for (auto* c : b->m)
        if (!grp_schedule(c)) {
            b->err = "grouped batch: a member has no compile-time-length transforms for nxc/2 and nzc";
            return PARATC_ERR_BAD_ARG;
        }
    int maxiad = 0;
    for (auto* c : b->m) maxiad = std::max(maxiad, c->hm.iadvance);
    P.sub.assign(maxiad, {});
    using K4 = std::tuple<int, int, int, int>;
    bool ok = true;
    for (int ns = 1; ns <= maxiad && ok; ns++) {
        std::map<K4, GrpAcc<RhsArgs<double>>> rhs64;
        std::map<int, GrpAcc<RhsArgs<float>>> rhs32;
        std::map<int, GrpAcc<HelmArgs<double>>> hs64, h64;
        std::map<int, GrpAcc<HelmArgs<float>>> hs32, h32;
        std::map<int, GrpAcc<XfArgs<double, double2>>> xf64;
        std::map<int, GrpAcc<XfArgs<float, float2>>> xf32;
        std::map<int, GrpAcc<ZtArgs<double2>>> zt64;
        std::map<int, GrpAcc<ZtArgs<float2>>> zt32;
        std::map<int, GrpAcc<YsArgs<double2>>> ys64;
        std::map<int, GrpAcc<YsArgs<float2>>> ys32;
        std::map<int, GrpAcc<XbArgs<double2, double>>> xb64;
        std::map<int, GrpAcc<XbArgs<float2, float>>> xb32;
        std::map<int, GrpAcc<ProjArgs<double>>> pj64;
        std::map<int, GrpAcc<ProjArgs<float>>> pj32;
        for (auto* c : b->m) {
            if (c->hm.iadvance < ns) continue;
            const DConst& k = c->kc;
            const HostMetrics& h = c->hm;
            const int M1 = c->nx / 2 + 1, kind = ys_kind(k);
            const double gam = h.gam[ns - 1], the = h.the[ns - 1], alp = h.alp[ns - 1];
            if (c->prec == PARATC_PREC_FP32) {
                float2* sp = spec32(c);
                rhs32[k.scalar_on].add(k, RhsArgs<float>{k, c->dm, c->d_coef, c->f32, c->d_uy_ym, c->d_duy_ym, gam,
                                                          the, alp, c->d_part, c->d_counter,
                                                          (int)rhs_member_grid(k, 1).x, 0},
                                       rhs_member_grid(k, 1));
                if (c->prm.scalar_on)
                    hs32[k.helm_var].add(k, HelmArgs<float>{k, c->d_coef, c->f32, nullptr, nullptr, c->d_hfac, 3},
                                         helm_member_grid(k, 1), helm_smem(k));
                h32[k.helm_var].add(k, HelmArgs<float>{k, c->d_coef, c->f32, c->d_duy_ym, c->d_uy_ym, c->d_hfac, 0},
                                    helm_member_grid(k, 3), helm_smem(k));
                xf32[c->nx].add(k, XfArgs<float, float2>{k, c->dm, c->d_coef, c->f32.ux, c->f32.uy, c->f32.uz, sp,
                                                         c->d_twx, c->d_postx, c->d_part, c->d_counter + 1,
                                                         &c->d_coef->divmax_src},
                                pfft_x_member_grid(k));
                zt32[c->nz].add(k, ZtArgs<float2>{c->ny * M1, sp, c->d_twz}, pfft_z_member_grid(k));
                ys32[kind].add(k, YsArgs<float2>{c->ny, M1, c->nz, c->dm.am2ph, sp, c->d_pfac},
                               ys_member_grid(k, kind), ys_smem(k, kind));
                xb32[c->nx].add(k, XbArgs<float2, float>{c->ny, c->nz, sp, c->d_phi32, c->d_twx, c->d_postx,
                                                         h.normfft},
                                pfft_x_member_grid(k));
                pj32[0].add(k, ProjArgs<float>{k, c->dm, c->d_coef, c->d_phi32, c->f32.ux, c->f32.uy, c->f32.uz,
                                               c->f32.pr, c->d_uy_ym},
                            cell_member_grid(k));
            } else {
                double2* sp = c->d_spec;
                rhs64[K4(k.scalar_on, k.fp32_rhs, k.fp32_rhs ? 0 : k.rhs_var, 0)].add(
                    k, RhsArgs<double>{k, c->dm, c->d_coef, c->f, c->d_uy_ym, c->d_duy_ym, gam, the, alp, c->d_part,
                                       c->d_counter, (int)rhs_member_grid(k, k.fp32_rhs).x, 0},
                    rhs_member_grid(k, k.fp32_rhs));
                if (c->prm.scalar_on)
                    hs64[k.helm_var].add(k, HelmArgs<double>{k, c->d_coef, c->f, nullptr, nullptr, c->d_hfac, 3},
                                         helm_member_grid(k, 1), helm_smem(k));
                h64[k.helm_var].add(k, HelmArgs<double>{k, c->d_coef, c->f, c->d_duy_ym, c->d_uy_ym, c->d_hfac, 0},
                                    helm_member_grid(k, 3), helm_smem(k));
                xf64[c->nx].add(k, XfArgs<double, double2>{k, c->dm, c->d_coef, c->f.ux, c->f.uy, c->f.uz, sp,
                                                           c->d_twx, c->d_postx, c->d_part, c->d_counter + 1,
                                                           &c->d_coef->divmax_src},
                                pfft_x_member_grid(k));
                zt64[c->nz].add(k, ZtArgs<double2>{c->ny * M1, sp, c->d_twz}, pfft_z_member_grid(k));
                ys64[kind].add(k, YsArgs<double2>{c->ny, M1, c->nz, c->dm.am2ph, sp, c->d_pfac},
                               ys_member_grid(k, kind), ys_smem(k, kind));
                xb64[c->nx].add(k, XbArgs<double2, double>{c->ny, c->nz, sp, c->d_phi, c->d_twx, c->d_postx,
                                                           h.normfft},
                                pfft_x_member_grid(k));
                pj64[0].add(k, ProjArgs<double>{k, c->dm, c->d_coef, c->d_phi, c->f.ux, c->f.uy, c->f.uz, c->f.pr,
                                                c->d_uy_ym},
                            cell_member_grid(k));
            }
        }
        std::vector<GrpLaunch>& L = P.sub[ns - 1];
        const int nsv = ns;
        auto rhs = [nsv](cudaStream_t st, auto, const DConst& kc, auto tab, int nblk, size_t) {
            launch_rhs_grp(st, kc, tab, nblk, nsv);
        };
        auto helm = [](cudaStream_t st, int, const DConst& kc, auto tab, int nblk, size_t sm) {
            launch_helm_grp(st, kc, tab, nblk, sm);
        };
        auto xf = [](cudaStream_t st, int nx, const DConst&, auto tab, int nblk, size_t) { launch_xf_grp(st, nx, tab, nblk); };
        auto ztf = [](cudaStream_t st, int nz, const DConst&, auto tab, int nblk, size_t) {
            launch_zt_grp(st, -1, nz, tab, nblk);
        };
        auto ztb = [](cudaStream_t st, int nz, const DConst&, auto tab, int nblk, size_t) {
            launch_zt_grp(st, 1, nz, tab, nblk);
        };
        auto ys = [](cudaStream_t st, int kind, const DConst&, auto tab, int nblk, size_t sm) {
            launch_ys_grp(st, kind, tab, nblk, sm);
        };
        auto xb = [](cudaStream_t st, int nx, const DConst&, auto tab, int nblk, size_t) { launch_xb_grp(st, nx, tab, nblk); };
        auto pj = [](cudaStream_t st, int, const DConst&, auto tab, int nblk, size_t) { launch_project_grp(st, tab, nblk); };
        // the substep's stages in the order of enqueue_substep, each stage's
        // instantiations one after another
        grp_balance_rhs(rhs64);
        grp_balance_rhs(rhs32);
        ok = ok && grp_emit(P, rhs64, L, rhs) && grp_emit(P, rhs32, L, rhs);
        ok = ok && grp_emit(P, hs64, L, helm) && grp_emit(P, hs32, L, helm);
        ok = ok && grp_emit(P, h64, L, helm) && grp_emit(P, h32, L, helm);
        ok = ok && grp_emit(P, xf64, L, xf) && grp_emit(P, xf32, L, xf);
        ok = ok && grp_emit(P, zt64, L, ztf) && grp_emit(P, zt32, L, ztf);
        ok = ok && grp_emit(P, ys64, L, ys) && grp_emit(P, ys32, L, ys);
        ok = ok && grp_emit(P, zt64, L, ztb) && grp_emit(P, zt32, L, ztb);
        ok = ok && grp_emit(P, xb64, L, xb) && grp_emit(P, xb32, L, xb);
        ok = ok && grp_emit(P, pj64, L, pj) && grp_emit(P, pj32, L, pj);
        P.kernels += (int64_t)L.size();
    }
    if (ok) {
        std::map<int, GrpAcc<EndArgs<double>>> e64;
        std::map<int, GrpAcc<EndArgs<float>>> e32;
        for (auto* c : b->m) {
            const DConst& k = c->kc;
            if (c->prec == PARATC_PREC_FP32)
                e32[0].add(k, EndArgs<float>{k, c->dm, c->f32.ux, c->f32.uy, c->f32.uz, c->f32.sc, c->d_coef,
                                             c->d_diag, c->d_part, c->d_counter + 3},
                           endstep_member_grid(k));
            else
                e64[0].add(k, EndArgs<double>{k, c->dm, c->f.ux, c->f.uy, c->f.uz, c->f.sc, c->d_coef, c->d_diag,
                                              c->d_part, c->d_counter + 3},
                           endstep_member_grid(k));
            if (c->prm.icfl == 1) P.fac.push_back(c);
        }
        auto es = [](cudaStream_t st, int, const DConst&, auto tab, int nblk, size_t) { launch_endstep_grp(st, tab, nblk); };
        ok = grp_emit(P, e64, P.end, es) && grp_emit(P, e32, P.end, es);
        P.kernels += (int64_t)P.end.size() + (int64_t)P.fac.size();
    }
    if (!ok) {
        grp_free(b->plan);
        b->err = "grouped batch: could not build the launch tables";
        return PARATC_ERR_CUDA;
    }
    for (auto* c : b->m) P.gens.push_back(c->sched_gen);
    P.built = true;
    return PARATC_OK;
}

// the plan is current: built from the members' present schedules and forms
bool grp_current(const paratc_batch* b) {
    if (!b->plan.built) return false;
    for (int i = 0; i < b->n; i++)
        if (b->m[i]->sched_gen != b->plan.gens[i]) return false;
    return true;
}

// one grouped step of every member on b->st (every member steady)
void grp_enqueue_step(paratc_batch* b) {
    cudaStream_t st = b->st;
    for (auto* c : b->plan.fac)
        launch_helm_factors(st, c->kc, c->dm, c->d_coef, 1, c->hm.iadvance, c->hm.alp, c->d_hfac);
    for (auto& v : b->plan.sub)
        for (auto& l : v) l.run(st);
    for (auto& l : b->plan.end) l.run(st);
    for (auto* c : b->m) {
        c->next_ready = true;
        c->launches += b->plan.kernels / b->n;
    }
}

int batch_capture(paratc_batch* b) {
    cudaGraph_t g = nullptr;
    int64_t l0 = 0;
    for (auto* c : b->m) l0 += c->launches;
    cudaError_t e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return (int)e;
    bool ok = true;
    if (b->mode == PARATC_BATCH_GROUPED) {
        grp_enqueue_step(b);  // every launch on b->st
    } else {
        ok = cudaEventRecord(b->fork, b->st) == cudaSuccess;
        for (int i = 0; ok && i < b->n; i++) {
            paratc_ctx* c = b->m[i];
            ok = cudaStreamWaitEvent(c->st, b->fork, 0) == cudaSuccess;
            if (ok) enqueue_step(c);
            ok = ok && cudaEventRecord(b->join[i], c->st) == cudaSuccess;
            ok = ok && cudaStreamWaitEvent(b->st, b->join[i], 0) == cudaSuccess;
        }
    }
    e = cudaStreamEndCapture(b->st, &g);
    if (!ok || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return ok ? (int)e : -1;
    }
    e = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->exec = nullptr;
        cudaGetLastError();
        return (int)e;
    }
    int64_t l1 = 0;
    for (auto* c : b->m) l1 += c->launches;
    b->graph_kernels = b->mode == PARATC_BATCH_GROUPED ? b->plan.kernels : l1 - l0;
    b->gens.clear();
    for (auto* c : b->m) b->gens.push_back(c->sched_gen);
    return 0;
}

}  // namespace

extern "C" {

int paratc_batch_create(int n, const paratc_params* prm, const double* const* yp, int device, paratc_batch** out) {
    if (n < 1 || !prm || !yp || !out) return PARATC_ERR_BAD_ARG;
    *out = nullptr;
    paratc_batch* b = new paratc_batch();
    b->n = n;
    b->dev = device;
    for (int i = 0; i < n; i++) {
        paratc_ctx* c = nullptr;
        int rc = paratc_create(&prm[i], yp[i], device, &c);
        if (rc != PARATC_OK) {
            paratc_batch_destroy(b);
            return rc;
        }
        b->m.push_back(c);
    }
    b->dev = b->m[0]->dev;  // the device paratc_create resolved (device < 0: the current one)
    b->join.assign(n, nullptr);
    bool ok = cudaSetDevice(b->dev) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < n; i++) ok = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        paratc_batch_destroy(b);
        return PARATC_ERR_CUDA;
    }
    *out = b;
    return PARATC_OK;
}

int paratc_batch_destroy(paratc_batch* b) {
    if (!b) return PARATC_OK;
    if (b->st) cudaStreamSynchronize(b->st);
    batch_free_graph(b);
    grp_free(b->plan);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->st) cudaStreamDestroy(b->st);
    for (auto* c : b->m) paratc_destroy(c);
    delete b;
    return PARATC_OK;
}

int paratc_batch_member(paratc_batch* b, int i, paratc_ctx** ctx) {
    if (!b || !ctx || i < 0 || i >= b->n) return PARATC_ERR_BAD_ARG;
    *ctx = b->m[i];
    return PARATC_OK;
}

int64_t paratc_batch_graph_kernels(paratc_batch* b) { return b ? b->graph_kernels : 0; }

int paratc_batch_set_mode(paratc_batch* b, int mode) {
    if (!b || (mode != PARATC_BATCH_STREAMS && mode != PARATC_BATCH_GROUPED)) return PARATC_ERR_BAD_ARG;
    if (cudaSetDevice(b->dev) != cudaSuccess) return PARATC_ERR_CUDA;
    if (cudaStreamSynchronize(b->st) != cudaSuccess) return PARATC_ERR_CUDA;  // no graph of the old mode in flight
    batch_free_graph(b);
    b->graph_failed = false;
    b->graph_kernels = 0;
    grp_free(b->plan);
    b->mode = mode;
    if (mode == PARATC_BATCH_GROUPED) {
        const int rc = grp_build(b);
        if (rc != PARATC_OK) {
            b->mode = PARATC_BATCH_STREAMS;
            return rc;
        }
    }
    return PARATC_OK;
}

int paratc_batch_get_mode(paratc_batch* b, int* mode) {
    if (!b || !mode) return PARATC_ERR_BAD_ARG;
    *mode = b->mode;
    return PARATC_OK;
}

int64_t paratc_batch_step_launches(paratc_batch* b) {
    if (!b) return 0;
    if (b->mode == PARATC_BATCH_GROUPED) return b->plan.built ? b->plan.kernels : 0;
    return b->graph_kernels;
}

void* paratc_batch_stream(paratc_batch* b) { return b ? (void*)b->st : nullptr; }

int paratc_batch_steps(paratc_batch* b, int nsteps, int use_graph, paratc_diag* diag) {
    if (!b || nsteps < 1) return PARATC_ERR_BAD_ARG;
    if (cudaSetDevice(b->dev) != cudaSuccess) return PARATC_ERR_CUDA;
    if (batch_fork_members(b) != cudaSuccess) return PARATC_ERR_CUDA;  // after what the caller queued on b->st
    for (auto* c : b->m) {
        c->prof_on = false;  // the event timer cannot live inside a graph
        if (cudaMemsetAsync(c->d_diag, 0, sizeof(DDiag), c->st) != cudaSuccess) return PARATC_ERR_CUDA;
    }
    int s = 0;
    const bool graph = use_graph && !b->graph_failed;
    if (b->mode == PARATC_BATCH_GROUPED && !grp_current(b)) {
        // a member changed its schedule, form or launch shapes: new tables
        batch_free_graph(b);
        const int rc = grp_build(b);
        if (rc != PARATC_OK) return rc;
    }
    if (graph && b->exec) {
        // a member re-tuned since the capture: the graph holds its old kernels
        for (int i = 0; i < b->n; i++)
            if (b->m[i]->sched_gen != b->gens[i]) { batch_free_graph(b); break; }
    }
    if (b->mode == PARATC_BATCH_GROUPED) {
        // the grouped launches need every member in the steady state: a member
        // that is not takes one ordinary step first (all of them, in step)
        bool steady = true;
        for (auto* c : b->m) steady = steady && member_steady(c);
        if (!steady) {
            for (auto* c : b->m) enqueue_step(c);
            s++;
        }
        if (s < nsteps) {
            if (batch_join_members(b) != cudaSuccess) return PARATC_ERR_CUDA;
            if (graph && !b->exec && batch_capture(b) != 0) {
                b->graph_failed = true;
                batch_free_graph(b);
            }
            for (; s < nsteps; s++) {
                if (b->exec) {
                    if (cudaGraphLaunch(b->exec, b->st) != cudaSuccess) return PARATC_ERR_CUDA;
                    for (auto* c : b->m) c->launches += b->graph_kernels / b->n;
                } else {
                    grp_enqueue_step(b);
                }
            }
            if (batch_fork_members(b) != cudaSuccess) return PARATC_ERR_CUDA;
        }
    } else if (graph) {
        bool steady = true;
        for (auto* c : b->m) steady = steady && member_steady(c);
        if (!steady) {
            for (auto* c : b->m) enqueue_step(c);
            s++;
        }
        if (s < nsteps && !b->exec) {
            // the capture needs every member in the steady state first
            bool st2 = true;
            for (auto* c : b->m) st2 = st2 && member_steady(c);
            if (!st2 || batch_capture(b) != 0) {
                b->graph_failed = true;
                batch_free_graph(b);
            }
        }
        if (b->exec && s < nsteps) {
            if (batch_join_members(b) != cudaSuccess) return PARATC_ERR_CUDA;
            for (; s < nsteps; s++)
                if (cudaGraphLaunch(b->exec, b->st) != cudaSuccess) return PARATC_ERR_CUDA;
            for (auto* c : b->m) c->launches += b->graph_kernels / b->n;
            if (batch_fork_members(b) != cudaSuccess) return PARATC_ERR_CUDA;
        }
    }
    for (; s < nsteps; s++)
        for (auto* c : b->m) enqueue_step(c);
    if (batch_join_members(b) != cudaSuccess) return PARATC_ERR_CUDA;  // b->st follows every member
    int first = PARATC_OK;
    for (int i = 0; i < b->n; i++) {
        paratc_ctx* c = b->m[i];
        if (cudaMemcpyAsync(c->h_diag, c->d_diag, sizeof(DDiag), cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
            return PARATC_ERR_CUDA;
    }
    for (int i = 0; i < b->n; i++) {
        paratc_ctx* c = b->m[i];
        int rc = sync(c);
        if (rc) return rc;
        if (diag) diag_out(*c->h_diag, &diag[i]);
        if (c->h_diag->status != 0 && first == PARATC_OK) {
            first = c->h_diag->status;
            char msg[160];
            std::snprintf(msg, sizeof(msg), "member %d: %s at step %d (divmax %.6e)", i,
                          paratc_strerror(c->h_diag->status), c->h_diag->failed_step, c->h_diag->divmax);
            b->err = msg;
            set_err(c, first, msg);
        }
    }
    return first;
}

}  // extern "C"
