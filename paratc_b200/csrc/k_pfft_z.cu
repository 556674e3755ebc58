// k_pfft_z.cu -- z transforms of the pressure Poisson solve, compile-time
// lengths.
//
// After the x transform the spectrum is spec[(kz*ny + j)*(nx/2+1) + kx]; for
// a fixed kz the (j, kx) pairs form one contiguous run of ncol = ny*(nx/2+1)
// complex values, so the z transform works on "columns" q = j*(nx/2+1) + kx
// whose element kz sits at spec[kz*ncol + q].  A CTA owns B consecutive
// columns: every load and store of a pass moves B contiguous 16-byte values.
// The first pass reads its inputs straight from global memory and the last
// pass writes its outputs straight back, so a two-pass length (64, 128, 256)
// touches shared memory once.  Unnormalised, as FFTW's R2HC / HC2R along z in
// clcPPE (src/m_Poisson.f90:352-452); the 1/(nx*nz) is applied after the x
// inverse.
#include "common.cuh"
#include "fft_fixed.cuh"
#include "kernels.cuh"

namespace ptc {
namespace {

// A: the complex type the passes compute in (double2; float2 for the FP32
// storage form's step)
template <int N, class A = double2>
struct ZK {
    static constexpr int B = ff::Shape<N>::B < 4 ? 4 : ff::Shape<N>::B;
    static constexpr int P = B * N / ff::Shape<N>::RMAX;
    static constexpr size_t smem = ((size_t)N * B + N) * sizeof(A);
};

// global element e of column b, in the spectrum's storage type S (double2,
// or float2 in the FP32 storage form), converted to and from A
template <class S, class A>
struct GLd {
    const S* base;
    int ncol, nvalid;
    __device__ __forceinline__ A operator()(int e, int b) const {
        return b < nvalid ? cto<A>(base[(size_t)e * ncol + b]) : Cx<A>::make(0, 0);
    }
};
template <class S, class A>
struct GSt {
    S* base;
    int ncol, nvalid;
    __device__ __forceinline__ void operator()(int e, int b, A v) const {
        if (b < nvalid) base[(size_t)e * ncol + b] = cto<S>(v);
    }
};

// G: the block this CTA works as (OwnGrid, or SubGrid in a grouped launch)
template <int N, int DIR, class S, class A, class G>
__device__ __forceinline__ void zt_body(const G& grid, int ncol, S* __restrict__ spec,
                                        const double2* __restrict__ twN) {
    constexpr int B = ZK<N, A>::B, P = ZK<N, A>::P;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ double2 smz[];
    A* buf = reinterpret_cast<A*>(smz);
    A* tws = buf + N * B;
    const int tid = threadIdx.x;
    const int q0 = grid.x() * B;
    const int nvalid = min(B, ncol - q0);
    const GLd<S, A> gl{spec + q0, ncol, nvalid};
    const GSt<S, A> gs{spec + q0, ncol, nvalid};
    if constexpr (SC.np == 1) {
        pdl_wait();
        pdl_trigger();
        ff::pass<N, B, P, SC.r[0], 1, DIR, false>(gl, gs, static_cast<const A*>(tws), tid);
    } else {
        for (int t = tid; t < N; t += P) tws[t] = cto<A>(twN[t]);
        pdl_wait();
        pdl_trigger();
        ff::pass<N, B, P, SC.r[0], 1, DIR, false>(gl, ff::SmemSt<B, A>{buf}, static_cast<const A*>(tws), tid);
        __syncthreads();
        ff::smem_passes<N, B, B, P, DIR, 1, SC.np - 1>(buf, static_cast<const A*>(tws), tid);
        constexpr int L = SC.np - 1;
        ff::pass<N, B, P, SC.r[L], ff::sched_ns(N, L), DIR, false>(ff::SmemLd<B, A>{buf}, gs,
                                                                   static_cast<const A*>(tws), tid);
    }
}

template <int N, int DIR, class S, class A>
__global__ void __launch_bounds__(ZK<N, A>::P) k_zt(int ncol, S* __restrict__ spec, const double2* __restrict__ twN) {
    zt_body<N, DIR, S, A>(OwnGrid{}, ncol, spec, twN);
}

template <int N, int DIR, class S, class A>
__global__ void __launch_bounds__(ZK<N, A>::P) k_zt_grp(const GrpTab<ZtArgs<S>>* __restrict__ t) {
    SubGrid g;
    const ZtArgs<S>& a = t->e[grp_member(t, g)];
    zt_body<N, DIR, S, A>(g, a.ncol, a.spec, a.tw);
}

#define PFFT_Z_SIZES(X) X(8) X(12) X(16) X(24) X(30) X(32) X(40) X(48) X(64) X(96) X(128) X(192) X(256) X(384) \
    X(512) X(768) X(1024) X(1152) X(1536)

}  // namespace

bool pfft_z_supported(int n) {
    switch (n) {
#define Z_CASE(n) case n:
        PFFT_Z_SIZES(Z_CASE)
#undef Z_CASE
        return true;
        default: return false;
    }
}

// (spectrum, arithmetic): FP64; the FP32 storage form's step (float); the
// refined solve's float2 spectrum in double arithmetic
#define ZT_ATTR(n, S, A)                                                                                          \
    cudaFuncSetAttribute(k_zt<n, -1, S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n, A>::smem);    \
    cudaFuncSetAttribute(k_zt<n, 1, S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n, A>::smem);
#define ZG_ATTR(n, S, A)                                                                                          \
    cudaFuncSetAttribute(k_zt_grp<n, -1, S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n, A>::smem); \
    cudaFuncSetAttribute(k_zt_grp<n, 1, S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n, A>::smem);

void pfft_z_init() {
#define Z_CASE(n) ZT_ATTR(n, double2, double2) ZT_ATTR(n, float2, float2) ZT_ATTR(n, float2, double2) \
    ZG_ATTR(n, double2, double2) ZG_ATTR(n, float2, float2)
    PFFT_Z_SIZES(Z_CASE)
#undef Z_CASE
}

dim3 pfft_z_member_grid(const DConst& c) {
    const int ncol = c.ny * (c.nx / 2 + 1);
    switch (c.nz) {
#define Z_CASE(n) case n: return dim3((ncol + ZK<n>::B - 1) / ZK<n>::B);
        PFFT_Z_SIZES(Z_CASE)
#undef Z_CASE
        default: return dim3(0);
    }
}

// grouped: a float2 spectrum is an FP32-storage member's step (float arithmetic)
template <class S>
static void zt_grp_t(cudaStream_t st, int dir, int nz, const GrpTab<ZtArgs<S>>* t, int nblk) {
    using A = S;
    switch (nz) {
#define Z_CASE(n)                                                                                               \
    case n:                                                                                                     \
        if (dir < 0) launch_pdl(k_zt_grp<n, -1, S, A>, dim3((unsigned)nblk), dim3(ZK<n, A>::P), ZK<n, A>::smem, \
                                st, t);                                                                         \
        else launch_pdl(k_zt_grp<n, 1, S, A>, dim3((unsigned)nblk), dim3(ZK<n, A>::P), ZK<n, A>::smem, st, t);  \
        break;
        PFFT_Z_SIZES(Z_CASE)
#undef Z_CASE
        default: break;
    }
}
void launch_zt_grp(cudaStream_t st, int dir, int nz, const GrpTab<ZtArgs<double2>>* t, int nblk) {
    zt_grp_t(st, dir, nz, t, nblk);
}
void launch_zt_grp(cudaStream_t st, int dir, int nz, const GrpTab<ZtArgs<float2>>* t, int nblk) {
    zt_grp_t(st, dir, nz, t, nblk);
}

template <class S, class A>
static void pfft_z_t(cudaStream_t st, int dir, int nx, int ny, int nz, S* spec, const double2* twz) {
    const int ncol = ny * (nx / 2 + 1);
    switch (nz) {
#define Z_CASE(n)                                                                                                 \
    case n: {                                                                                                     \
        const int grid = (ncol + ZK<n, A>::B - 1) / ZK<n, A>::B;                                                  \
        if (dir < 0)                                                                                              \
            launch_pdl(k_zt<n, -1, S, A>, dim3(grid), dim3(ZK<n, A>::P), ZK<n, A>::smem, st, ncol, spec, twz);    \
        else launch_pdl(k_zt<n, 1, S, A>, dim3(grid), dim3(ZK<n, A>::P), ZK<n, A>::smem, st, ncol, spec, twz);    \
        break;                                                                                                    \
    }
        PFFT_Z_SIZES(Z_CASE)
#undef Z_CASE
        default: break;
    }
}
void launch_pfft_z(cudaStream_t st, int dir, int nx, int ny, int nz, double2* spec, const double2* twz) {
    pfft_z_t<double2, double2>(st, dir, nx, ny, nz, spec, twz);
}
void launch_pfft_z(cudaStream_t st, int dir, int nx, int ny, int nz, float2* spec, const double2* twz, int f32arith) {
    if (f32arith) pfft_z_t<float2, float2>(st, dir, nx, ny, nz, spec, twz);
    else pfft_z_t<float2, double2>(st, dir, nx, ny, nz, spec, twz);
}

}  // namespace ptc
