// common.cuh -- device-side data structures shared by the kernels of the
// ParaTC hot path.
//
// HBM layout of a 3-D field ("padded layout"): x fastest, then y, then z,
// index (i, j, k) -> (k*(ny+2) + j)*nx + i with i in [0,nx), j in [0,ny+1],
// k in [0,nz).  j keeps the Fortran numbering of the reference: j = 0 and
// j = nyp = ny+1 are the wall ghost rows of mb1 (src/m_Variables.f90:47-50),
// j = 1..ny the interior.  There are no x/z halo cells: the periodic halos of
// myupdate_halo (src/m_Decomp2d.f90:1554-1709) become index wrap, which reads
// the same values because every halo width the reference updates covers what
// its stencils read.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define PT_MAX_RADIX_PASSES 24

namespace ptc {

// y-direction metric arrays of m_MeshAndMetries, indexed by the Fortran j
// (entries 0..nyp); wavenumbers by the 0-based mode number.
struct DMetric {
    const double *rdyp, *rdyc, *dyp, *yinterp;
    const double *ap2c, *ac2c, *am2c;
    const double *ap2p, *ac2p, *am2p;
    const double *ap2ph, *ac2ph, *am2ph;
    const double *ap2cCN, *ac2cCN, *am2cCN;
    const double *ap2cSc, *ac2cSc, *am2cSc;
    const double *ap2cScCN, *ac2cScCN, *am2cScCN;
    const double *wnx, *wnz;
    // the coefficients one row j of the right-hand side reads, 16 doubles per
    // row j = 0..nyp (one 128-byte bulk copy): yinterp(j), yinterp(j+1), rdyp,
    // rdyc, dyp, ap2c, ac2c, am2c, ap2p, ac2p, am2p, ap2cSc, ac2cSc, am2cSc, 0, 0
    const double* rowmet;
};
constexpr int ROWMET = 16;

// grid sizes and the scalar constants every stencil needs
struct DConst {
    int nx, ny, nz, nyp, nyt;
    int flow_type, scalar_on, is_ux_const, icfl;
    int nsm;  // streaming multiprocessors of the device
    int solver_sel;  // 0 automatic; 1 forces the staged, 2 the streaming y-solve kernels (tests)
    int fp32_rhs;    // 1: the explicit right-hand side computed in FP32 arithmetic (FP64 state)
    int rhs_var;     // compiled launch shape of the FP64 right-hand side (the tuner's pick)
    int helm_var;    // compiled launch shape of the Helmholtz sweeps (the tuner's pick)
    double dxC[4], dzC[4], dxxC[5], dzzC[5], IC[4];
    double rdx, rdz;
    double ucrf, xnu, grav[3], sdiff, gev[3], fvv[3];
    double uxbc_ym, uxbc_yp, uybc_yp, uzbc_ym, uzbc_yp;
    double ubulk, yly, normfft, dt_max, cflc;
    double sc_r1b, sc_r2b, sc_r1t, sc_r2t;   // scalar ghost: c0 = r1b*c1 + r2b, ...
    double vel_limit, div_limit;
    // FP32 copies of the stencil constants for the FP32 right-hand side
    float fdxC[4], fdzC[4], fdxxC[5], fdzzC[5], fIC[4], fgrav[3], fgev[3], ffvv[3];
    float fucrf, fxnu, fsdiff;
};

// per-substep coefficients (PMcoeUpdate, src/m_Parameters.f90:215-230) and
// the running scalars of a step; lives in device memory so that dt computed
// on the device (iCFL = 1) needs no host round trip
struct DCoef {
    double dt, pmGamma, pmTheta, pmAlpha, pmAlphaC, pmBeta, pmBetaSc;
    double rhsx_add;        // -dp1ns (no scalar) or +dp1ns (scalar) of the flow-rate constraint
    double sim_time, pr_grad_aver, cflmp;
    double divmax_src;
    double dt_last;         // dt of the last completed step, once dt holds the next step's
    int ns, pad;
};

// diagnostics of one step, copied to pinned host memory at the end
struct DDiag {
    double dt, cfl, sim_time, divmax_src, divmax, vmax[3], pr_grad_aver, ux_mean, sc_mean, sc2_mean;
    int status;             // 0, or the PARATC_ERR_* of the first guard that failed
    int failed_step;        // 1-based index of that step inside a multi-step call
    int step_counter;
    int pad;
};

struct FftPlan {
    int n;          // transform length
    int nr;         // number of radix passes
    int rad[PT_MAX_RADIX_PASSES];
    unsigned long long code;  // the radices again, 4 bits each (pass s at bits 4s..4s+3)
};

// Programmatic dependent launch: a kernel launched with launch_pdl may start
// while its predecessor in the stream drains; pdl_wait() blocks until the
// predecessor grid has completed and its memory is visible, so every read of
// data an earlier kernel produced, and every global write, comes after it.
// pdl_trigger() lets the successor launch now.  Both are no-ops when the
// launch carried no programmatic attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// The block a CTA works as.  OwnGrid: its own launch (blockIdx, gridDim).
// SubGrid: its block within one member's launch shape inside a grouped
// launch over the members of an ensemble (every member keeps the block
// counts of its own launch, so its reductions see the same partial records).
struct OwnGrid {
    __device__ __forceinline__ unsigned x() const { return blockIdx.x; }
    __device__ __forceinline__ unsigned y() const { return blockIdx.y; }
    __device__ __forceinline__ unsigned z() const { return blockIdx.z; }
    __device__ __forceinline__ unsigned gx() const { return gridDim.x; }
    __device__ __forceinline__ unsigned gy() const { return gridDim.y; }
    __device__ __forceinline__ unsigned gz() const { return gridDim.z; }
};
struct SubGrid {
    unsigned bx, by, bz, nx, ny, nz;
    __device__ __forceinline__ unsigned x() const { return bx; }
    __device__ __forceinline__ unsigned y() const { return by; }
    __device__ __forceinline__ unsigned z() const { return bz; }
    __device__ __forceinline__ unsigned gx() const { return nx; }
    __device__ __forceinline__ unsigned gy() const { return ny; }
    __device__ __forceinline__ unsigned gz() const { return nz; }
};

// a grouped launch's table: member i owns blocks [b0[i], b0[i+1]) of a
// one-dimensional grid and launches with shape (gx, gy, gz) of its own
constexpr int PT_MAXMEM = 64;
template <class E>
struct GrpTab {
    int nmem;
    int b0[PT_MAXMEM + 1];
    unsigned g[PT_MAXMEM][3];
    E e[PT_MAXMEM];
};
// the member of this CTA, and its block in the member's launch shape (Tab:
// a GrpTab, or any table with the same nmem / b0 / g members)
template <class Tab>
__device__ __forceinline__ int grp_member(const Tab* __restrict__ t, SubGrid& sg) {
    int lo = 0, hi = t->nmem - 1;
    const int b = (int)blockIdx.x;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t->b0[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const unsigned l = (unsigned)(b - t->b0[lo]);
    sg.nx = t->g[lo][0];
    sg.ny = t->g[lo][1];
    sg.nz = t->g[lo][2];
    sg.bx = l % sg.nx;
    sg.by = (l / sg.nx) % sg.ny;
    sg.bz = l / (sg.nx * sg.ny);
    return lo;
}

// maximum that keeps a NaN: fmax(x, NaN) returns x, so a field that is NaN
// everywhere would report a maximum of 0 and pass every guard; with nmax a
// NaN anywhere reaches the grid-wide result (the non-finite guard's input)
__device__ __forceinline__ double nmax(double a, double b) { return (a > b || a != a) ? a : b; }

// Loads and stores between either storage precision and FP64 registers: the
// FP32 storage form keeps fields and spectra in float / float2 while every
// kernel computes in double (loads widen exactly, stores round to nearest).
// ld_pair / st_pair move the two values at an even index p[0], p[1].
__device__ __forceinline__ double2 ld_pair(const double* p) { return __ldg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ double2 ld_pair(const float* p) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return make_double2(v.x, v.y);
}
__device__ __forceinline__ void st_pair(double* p, double2 v) { *reinterpret_cast<double2*>(p) = v; }
__device__ __forceinline__ void st_pair(float* p, double2 v) {
    *reinterpret_cast<float2*>(p) = make_float2((float)v.x, (float)v.y);
}
__device__ __forceinline__ double2 ld_c(const double2* p) { return *p; }
__device__ __forceinline__ double2 ld_c(const float2* p) {
    const float2 v = *p;
    return make_double2(v.x, v.y);
}
__device__ __forceinline__ void st_c(double2* p, double2 v) { *p = v; }
__device__ __forceinline__ void st_c(float2* p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// the same for float2 (the FP32 arithmetic of the transforms)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// a complex type's real type and constructor, and conversions between the
// two complex types
template <class C>
struct Cx;
template <>
struct Cx<double2> {
    using R = double;
    static __device__ __forceinline__ double2 make(double x, double y) { return make_double2(x, y); }
};
template <>
struct Cx<float2> {
    using R = float;
    static __device__ __forceinline__ float2 make(float x, float y) { return make_float2(x, y); }
};
template <class C, class D>
__device__ __forceinline__ C cto(D v) {
    return Cx<C>::make((typename Cx<C>::R)v.x, (typename Cx<C>::R)v.y);
}

}  // namespace ptc
