// k_pfft_x.cu -- x transforms of the pressure Poisson solve, compile-time
// lengths.
//
// clcPPE (src/m_Poisson.f90:352-452) transforms the source along x with
// FFTW's R2HC and back with HC2R.  Here the real row of nx values is packed
// into nx/2 complex values z[m] = x[2m] + i x[2m+1], transformed with an
// nx/2-point complex FFT (fft_fixed.cuh) and split into the nx/2+1 modes of
// the real transform (forward), or merged and transformed back (inverse).
// The modified wavenumber is even in the mode number, so these modes carry
// the same eigenvalues as the reference's halfcomplex ones.
//
// Forward kernel: the source of a row is the divergence of u* computed on
// the fly (clcPrSrc, src/m_TScheme.f90:48-77: scaled by 1/pmAlpha in mode 0,
// unscaled in mode 1, with max|div| reduced over the grid by the last CTA)
// or a given compact source array (mode 2).  Inverse kernel: the merge, the
// inverse FFT, 1/(nx*nz) and the Neumann ghost rows phi(0) = phi(1),
// phi(nyp) = phi(nyc) of SetBC_and_UpdateHalo_pr (src/m_BC_and_Halo.f90:
// 115-120).  A CTA owns B consecutive rows g = k*ny + (jc-1), so its spectral
// rows spec[g*(nx/2+1) + kx] form one contiguous block.
#include <type_traits>

#include "common.cuh"
#include "fft_fixed.cuh"
#include "kernels.cuh"
#include "div_src.cuh"
#include "reduce.cuh"

namespace ptc {
namespace {

constexpr int XF_DIV_U = 2;  // divergence point pairs in flight per thread

__device__ __forceinline__ void cpa16(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpa_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// A: the complex type the passes compute in (double2; float2 for the FP32
// storage form's step, whose transforms then compute in FP32)
template <int N, class A = double2>
struct XK {
    static constexpr int B = ff::Shape<N>::B;
    static constexpr int P = ff::Shape<N>::P;
    static constexpr int PITCH = B + 1;  // odd pitch: row-order accesses hit distinct banks
    static constexpr size_t smem = ((size_t)(N + 1) * PITCH + N) * sizeof(A);
    // resident CTAs the launch bounds of k_xf ask for: 24 warps per SM (80
    // registers, a few spills; the FP32 form's k_xf<64> at C1 went from 0.14
    // to 0.17 of the HBM peak)
    static constexpr int MINB = 768 / P;
};

// V: storage of the velocity (mode 0/1), S: storage of the spectrum; the
// given source of mode 2 is FP64
// G: the block this CTA works as (OwnGrid, or SubGrid in a grouped launch)
template <int N, class V, class S, class A, class G>
__device__ __forceinline__ void xf_body(const G& grid, int mode, const DConst& c, const DMetric& m,
                                        const DCoef* __restrict__ coef, const V* __restrict__ ux,
                                        const V* __restrict__ uy, const V* __restrict__ uz,
                                        const double* __restrict__ src, S* __restrict__ spec,
                                        const double2* __restrict__ twN, const double2* __restrict__ post,
                                        double* __restrict__ part, unsigned int* __restrict__ counter,
                                        double* __restrict__ out_max) {
    using R = typename Cx<A>::R;
    constexpr int B = XK<N, A>::B, P = XK<N, A>::P, PITCH = XK<N, A>::PITCH, M1 = N + 1;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ double2 smx[];
    A* buf = reinterpret_cast<A*>(smx);
    A* tws = buf + (N + 1) * PITCH;
    const int tid = threadIdx.x;
    const int nx = 2 * N, nrows = c.ny * c.nz;
    const int g0 = grid.x() * B;
    for (int t = tid; t < N; t += P) tws[t] = cto<A>(twN[t]);
    pdl_wait();
    pdl_trigger();
    double dm = 0.0;
    if (mode == 2) {
        for (int f = tid; f < B * N; f += P) {
            const int b = f / N, e = f - b * N;
            const int g = g0 + b;
            if constexpr (sizeof(A) == sizeof(double2)) {
                if (g < nrows) cpa16(&buf[e * PITCH + b], src + (size_t)g * nx + 2 * e);
                else buf[e * PITCH + b] = Cx<A>::make(0, 0);
            } else {
                buf[e * PITCH + b] = g < nrows ? cto<A>(ld_pair(src + (size_t)g * nx + 2 * e)) : Cx<A>::make(0, 0);
            }
        }
        cpa_wait_all();
    } else {
        const double sudtal = (mode == 0) ? 1.0 / coef->pmAlpha : 1.0;
        div_batch<N, B, P, XF_DIV_U>(c, m, ux, uy, uz, g0, nrows, sudtal, tid, dm,
                                     [&](int b, int e, double2 v) { buf[e * PITCH + b] = cto<A>(v); });
    }
    __syncthreads();
    ff::smem_passes<N, B, PITCH, P, -1, 0, SC.np>(buf, tws, tid);
    // split the packed transform into the nx/2+1 modes of the real row
    const R h = (R)0.5;
    for (int f = tid; f < B * M1; f += P) {
        const int b = f / M1, a = f - b * M1;
        if (g0 + b >= nrows) continue;
        const A za = buf[(a == N ? 0 : a) * PITCH + b];
        const A zb = buf[(a == 0 ? 0 : N - a) * PITCH + b];
        const A E = Cx<A>::make(h * (za.x + zb.x), h * (za.y - zb.y));
        const A O = Cx<A>::make(h * (za.y + zb.y), -h * (za.x - zb.x));
        spec[(size_t)g0 * M1 + f] = cto<S>(cadd(E, cmul(cto<A>(__ldg(&post[a])), O)));
    }
    if (mode == 2) return;
    double v[1] = {dm};
    const unsigned int nblocks = grid.gx();
    block_max_store<1>(v, part + grid.x());
    if (!last_block_arrive(counter, nblocks)) return;
    double tot[1];
    reduce_records<1, true>(part, (int)nblocks, tot);
    if (tid == 0) *out_max = tot[0];
}

template <int N, class V, class S, class A>
__global__ void __launch_bounds__(XK<N, A>::P, XK<N, A>::MINB)
    k_xf(int mode, DConst c, DMetric m, const DCoef* __restrict__ coef, const V* __restrict__ ux,
         const V* __restrict__ uy, const V* __restrict__ uz, const double* __restrict__ src,
         S* __restrict__ spec, const double2* __restrict__ twN, const double2* __restrict__ post,
         double* __restrict__ part, unsigned int* __restrict__ counter, double* __restrict__ out_max) {
    xf_body<N, V, S, A>(OwnGrid{}, mode, c, m, coef, ux, uy, uz, src, spec, twN, post, part, counter, out_max);
}

template <int N, class V, class S, class A>
__global__ void __launch_bounds__(XK<N, A>::P) k_xf_grp(const GrpTab<XfArgs<V, S>>* __restrict__ t) {
    SubGrid g;
    const XfArgs<V, S>& a = t->e[grp_member(t, g)];
    xf_body<N, V, S, A>(g, 0, a.c, a.m, a.coef, a.ux, a.uy, a.uz, (const double*)nullptr, a.spec, a.tw, a.post,
                        a.part, a.counter, a.out_max);
}

// S: storage of the spectrum, P: of the potential; accumulate != 0 adds the
// result to phi (unpadded rows: the corrections of the refined solve)
template <int N, class S, class PH, class A, class G>
__device__ __forceinline__ void xb_body(const G& grid, int ny, int nz, const S* __restrict__ spec,
                                        PH* __restrict__ phi, const double2* __restrict__ twN,
                                        const double2* __restrict__ post, double scale, int padded, int accumulate,
                                        const double* __restrict__ shift) {
    using R = typename Cx<A>::R;
    constexpr int B = XK<N, A>::B, P = XK<N, A>::P, PITCH = XK<N, A>::PITCH, M1 = N + 1;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ double2 smx[];
    A* buf = reinterpret_cast<A*>(smx);
    A* tws = buf + (N + 1) * PITCH;
    const int tid = threadIdx.x;
    const int nx = 2 * N, nrows = ny * nz;
    const int g0 = grid.x() * B;
    for (int t = tid; t < N; t += P) tws[t] = cto<A>(twN[t]);
    pdl_wait();
    pdl_trigger();
    for (int f = tid; f < B * M1; f += P) {
        const int b = f / M1, a = f - b * M1;
        if (g0 + b >= nrows) buf[a * PITCH + b] = Cx<A>::make(0, 0);
        else if constexpr (sizeof(S) == sizeof(double2) && sizeof(A) == sizeof(double2))
            cpa16(&buf[a * PITCH + b], spec + (size_t)g0 * M1 + f);
        else buf[a * PITCH + b] = cto<A>(spec[(size_t)g0 * M1 + f]);
    }
    cpa_wait_all();
    __syncthreads();
    // merge modes a and N-a of every row into z[a], z[N-a] (the DC and
    // Nyquist coefficients are real)
    for (int f = tid; f < B * (N / 2 + 1); f += P) {
        const int a = f / B, b = f - a * B;
        const int bn = N - a;
        A xa = buf[a * PITCH + b], xb = buf[bn * PITCH + b];
        if (a == 0) { xa.y = 0; xb.y = 0; }
        const A e2a = Cx<A>::make(xa.x + xb.x, xa.y - xb.y);
        const A da = Cx<A>::make(xa.x - xb.x, xa.y + xb.y);
        const A o2a = cmulc(da, cto<A>(__ldg(&post[a])));
        const A za = Cx<A>::make(e2a.x - o2a.y, e2a.y + o2a.x);
        if (a == 0) {
            buf[b] = za;
        } else {
            const A e2b = Cx<A>::make(xb.x + xa.x, xb.y - xa.y);
            const A db = Cx<A>::make(xb.x - xa.x, xb.y + xa.y);
            const A o2b = cmulc(db, cto<A>(__ldg(&post[bn])));
            const A zb = Cx<A>::make(e2b.x - o2b.y, e2b.y + o2b.x);
            buf[a * PITCH + b] = za;
            if (bn != a) buf[bn * PITCH + b] = zb;
        }
    }
    __syncthreads();
    ff::smem_passes<N, B, PITCH, P, 1, 0, SC.np>(buf, tws, tid);
    const int nyt = ny + 2;
    const R sc = (R)scale;
    for (int f = tid; f < B * N; f += P) {
        const int b = f / N, e = f - b * N;
        const int g = g0 + b;
        if (g >= nrows) continue;
        const A z = buf[e * PITCH + b];
        double2 v = make_double2(z.x * sc, z.y * sc);
        if (!padded) {
            PH* dst = phi + (size_t)g * nx + 2 * e;
            if (accumulate) {
                // phi += correction - the row-1 plane mean of phi (the gauge)
                const double2 o = ld_pair(dst);
                const double sh = shift ? *shift : 0.0;
                v = make_double2(o.x + v.x - sh, o.y + v.y - sh);
            }
            st_pair(dst, v);
            continue;
        }
        const int k = g / ny, jc = g - k * ny + 1;
        PH* rowp = phi + ((size_t)k * nyt + jc) * nx + 2 * e;
        st_pair(rowp, v);
        if (jc == 1) st_pair(rowp - nx, v);
        if (jc == ny) st_pair(rowp + nx, v);
    }
}

template <int N, class S, class PH, class A>
__global__ void __launch_bounds__(XK<N, A>::P)
    k_xb(int ny, int nz, const S* __restrict__ spec, PH* __restrict__ phi, const double2* __restrict__ twN,
         const double2* __restrict__ post, double scale, int padded, int accumulate,
         const double* __restrict__ shift) {
    xb_body<N, S, PH, A>(OwnGrid{}, ny, nz, spec, phi, twN, post, scale, padded, accumulate, shift);
}

template <int N, class S, class PH, class A>
__global__ void __launch_bounds__(XK<N, A>::P) k_xb_grp(const GrpTab<XbArgs<S, PH>>* __restrict__ t) {
    SubGrid g;
    const XbArgs<S, PH>& a = t->e[grp_member(t, g)];
    xb_body<N, S, PH, A>(g, a.ny, a.nz, a.spec, a.phi, a.tw, a.post, a.scale, 1, 0, (const double*)nullptr);
}

#define PFFT_X_SIZES(X) X(8) X(12) X(16) X(24) X(32) X(40) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) \
    X(768) X(1024) X(1152) X(1536)

}  // namespace

#ifndef PTC_STORE32
// FP64 instantiations; the FP32 storage forms (float2 spectra) are compiled
// in k_pfft_x32.cu from these same kernels
bool pfft_x_supported(int n) {
    switch (n) {
#define X_CASE(n) case n:
        PFFT_X_SIZES(X_CASE)
#undef X_CASE
        return true;
        default: return false;
    }
}

int pfft_x_blocks(int nx, int ny, int nz) {
    int b = 1;
    switch (nx / 2) {
#define X_CASE(n) case n: b = XK<n>::B; break;
        PFFT_X_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
    return (ny * nz + b - 1) / b;
}
// (velocity or potential, spectrum, arithmetic): the FP32 storage form's
// step computes in float; the refined solve's FP64 source and FP64
// corrections keep double arithmetic
#define XF_TYPES(X, n) X(n, double, double2, double2)
#define XB_TYPES(X, n) X(n, double2, double, double2)
#define XG_V double
#define XG_S double2
#define XG_A double2
#else
#define XF_TYPES(X, n) X(n, float, float2, float2) X(n, double, float2, double2)
#define XB_TYPES(X, n) X(n, float2, float, float2) X(n, float2, double, double2)
#define XG_V float
#define XG_S float2
#define XG_A float2
#endif

#ifndef PTC_STORE32
void pfft_x_init() {
    pfft_x_init32();
#else
void pfft_x_init32() {
#endif
#define XF_ATTR(n, V, S, A)                                                                                     \
    cudaFuncSetAttribute(k_xf<n, V, S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XK<n, A>::smem);
#define XB_ATTR(n, S, PH, A)                                                                                    \
    cudaFuncSetAttribute(k_xb<n, S, PH, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XK<n, A>::smem);
#define XG_ATTR(n)                                                                                              \
    cudaFuncSetAttribute(k_xf_grp<n, XG_V, XG_S, XG_A>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                         (int)XK<n, XG_A>::smem);                                                               \
    cudaFuncSetAttribute(k_xb_grp<n, XG_S, XG_V, XG_A>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                         (int)XK<n, XG_A>::smem);
#define X_CASE(n) XF_TYPES(XF_ATTR, n) XB_TYPES(XB_ATTR, n) XG_ATTR(n)
    PFFT_X_SIZES(X_CASE)
#undef X_CASE
#undef XG_ATTR
#undef XF_ATTR
#undef XB_ATTR
}

// float velocity: the FP32 storage form's step, float arithmetic
template <class V, class S>
static void pfft_xf_t(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                      const FieldSet<V>& f, const double* src, S* spec, const double2* twx, const double2* post,
                      double* part, unsigned int* counter, double* out_max) {
    using A = std::conditional_t<sizeof(V) == 4, float2, double2>;
    const int nrows = c.ny * c.nz;
    switch (c.nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xf<n, V, S, A>, dim3((nrows + XK<n, A>::B - 1) / XK<n, A>::B), dim3(XK<n, A>::P),        \
                   XK<n, A>::smem, st, mode, c, m, coef, f.ux, f.uy, f.uz, src, spec, twx, post, part, counter,  \
                   out_max);                                                                                   \
        break;
        PFFT_X_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

// float potential: the FP32 storage form's step, float arithmetic
template <class S, class PH>
static void pfft_xb_t(cudaStream_t st, int nx, int ny, int nz, const S* spec, PH* phi, const double2* twx,
                      const double2* post, double scale, int padded, int accumulate, const double* shift) {
    using A = std::conditional_t<sizeof(PH) == 4, float2, double2>;
    const int nrows = ny * nz;
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xb<n, S, PH, A>, dim3((nrows + XK<n, A>::B - 1) / XK<n, A>::B), dim3(XK<n, A>::P),      \
                   XK<n, A>::smem, st, ny, nz, spec, phi, twx, post, scale, padded, accumulate, shift);        \
        break;
        PFFT_X_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

// grouped launches of the step's forward (divergence source) and inverse
// (padded potential) transforms: one member's shape is its row blocks
void launch_xf_grp(cudaStream_t st, int nx, const GrpTab<XfArgs<XG_V, XG_S>>* t, int nblk) {
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xf_grp<n, XG_V, XG_S, XG_A>, dim3((unsigned)nblk), dim3(XK<n, XG_A>::P), XK<n, XG_A>::smem, \
                   st, t);                                                                                     \
        break;
        PFFT_X_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}
void launch_xb_grp(cudaStream_t st, int nx, const GrpTab<XbArgs<XG_S, XG_V>>* t, int nblk) {
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xb_grp<n, XG_S, XG_V, XG_A>, dim3((unsigned)nblk), dim3(XK<n, XG_A>::P), XK<n, XG_A>::smem, \
                   st, t);                                                                                     \
        break;
        PFFT_X_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

#ifndef PTC_STORE32
dim3 pfft_x_member_grid(const DConst& c) { return dim3((unsigned)pfft_x_blocks(c.nx, c.ny, c.nz)); }

void launch_pfft_xf(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f,
                    const double* src, double2* spec, const double2* twx, const double2* post, double* part,
                    unsigned int* counter, double* out_max) {
    pfft_xf_t(st, mode, c, m, coef, f, src, spec, twx, post, part, counter, out_max);
}
void launch_pfft_xb(cudaStream_t st, int nx, int ny, int nz, const double2* spec, double* phi, const double2* twx,
                    const double2* post, double scale, int padded) {
    pfft_xb_t(st, nx, ny, nz, spec, phi, twx, post, scale, padded, 0, nullptr);
}
#else
void launch_pfft_xf(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                    const Fields32& f, const double* src, float2* spec, const double2* twx, const double2* post,
                    double* part, unsigned int* counter, double* out_max) {
    pfft_xf_t(st, mode, c, m, coef, f, src, spec, twx, post, part, counter, out_max);
}
void launch_pfft_xf(cudaStream_t st, const DConst& c, const double* src, float2* spec, const double2* twx,
                    const double2* post) {
    const Fields none = {};
    pfft_xf_t(st, 2, c, DMetric{}, nullptr, none, src, spec, twx, post, nullptr, nullptr, nullptr);
}
void launch_pfft_xb(cudaStream_t st, int nx, int ny, int nz, const float2* spec, float* phi, const double2* twx,
                    const double2* post, double scale, int padded) {
    pfft_xb_t(st, nx, ny, nz, spec, phi, twx, post, scale, padded, 0, nullptr);
}
void launch_pfft_xb(cudaStream_t st, int nx, int ny, int nz, const float2* spec, double* phi, const double2* twx,
                    const double2* post, double scale, int accumulate, const double* shift) {
    pfft_xb_t(st, nx, ny, nz, spec, phi, twx, post, scale, 0, accumulate, shift);
}
#endif

}  // namespace ptc
