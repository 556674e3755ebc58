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

template <int N>
struct ZK {
    static constexpr int B = ff::Shape<N>::B < 4 ? 4 : ff::Shape<N>::B;
    static constexpr int P = B * N / ff::Shape<N>::RMAX;
    static constexpr size_t smem = ((size_t)N * B + N) * sizeof(double2);
};

// global element e of column b, in the spectrum's storage type S (double2,
// or float2 in the FP32 storage form; the passes compute in double either way)
template <class S>
struct GLd {
    const S* base;
    int ncol, nvalid;
    __device__ __forceinline__ double2 operator()(int e, int b) const {
        return b < nvalid ? ld_c(base + (size_t)e * ncol + b) : make_double2(0.0, 0.0);
    }
};
template <class S>
struct GSt {
    S* base;
    int ncol, nvalid;
    __device__ __forceinline__ void operator()(int e, int b, double2 v) const {
        if (b < nvalid) st_c(base + (size_t)e * ncol + b, v);
    }
};

// G: the block this CTA works as (OwnGrid, or SubGrid in a grouped launch)
template <int N, int DIR, class S, class G>
__device__ __forceinline__ void zt_body(const G& grid, int ncol, S* __restrict__ spec,
                                        const double2* __restrict__ twN) {
    constexpr int B = ZK<N>::B, P = ZK<N>::P;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ double2 smz[];
    double2* buf = smz;
    double2* tws = smz + N * B;
    const int tid = threadIdx.x;
    const int q0 = grid.x() * B;
    const int nvalid = min(B, ncol - q0);
    const GLd<S> gl{spec + q0, ncol, nvalid};
    const GSt<S> gs{spec + q0, ncol, nvalid};
    if constexpr (SC.np == 1) {
        pdl_wait();
        pdl_trigger();
        ff::pass<N, B, P, SC.r[0], 1, DIR, false>(gl, gs, tws, tid);
    } else {
        for (int t = tid; t < N; t += P) tws[t] = twN[t];
        pdl_wait();
        pdl_trigger();
        ff::pass<N, B, P, SC.r[0], 1, DIR, false>(gl, ff::SmemSt<B>{buf}, tws, tid);
        __syncthreads();
        ff::smem_passes<N, B, B, P, DIR, 1, SC.np - 1>(buf, tws, tid);
        constexpr int L = SC.np - 1;
        ff::pass<N, B, P, SC.r[L], ff::sched_ns(N, L), DIR, false>(ff::SmemLd<B>{buf}, gs, tws, tid);
    }
}

template <int N, int DIR, class S>
__global__ void __launch_bounds__(ZK<N>::P) k_zt(int ncol, S* __restrict__ spec, const double2* __restrict__ twN) {
    zt_body<N, DIR>(OwnGrid{}, ncol, spec, twN);
}

template <int N, int DIR, class S>
__global__ void __launch_bounds__(ZK<N>::P) k_zt_grp(const GrpTab<ZtArgs<S>>* __restrict__ t) {
    SubGrid g;
    const ZtArgs<S>& a = t->e[grp_member(t, g)];
    zt_body<N, DIR>(g, a.ncol, a.spec, a.tw);
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

void pfft_z_init() {
#define Z_CASE(n)                                                                                              \
    cudaFuncSetAttribute(k_zt<n, -1, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem); \
    cudaFuncSetAttribute(k_zt<n, 1, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem);  \
    cudaFuncSetAttribute(k_zt<n, -1, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem);  \
    cudaFuncSetAttribute(k_zt<n, 1, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem);      \
    cudaFuncSetAttribute(k_zt_grp<n, -1, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem); \
    cudaFuncSetAttribute(k_zt_grp<n, 1, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem);  \
    cudaFuncSetAttribute(k_zt_grp<n, -1, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem);  \
    cudaFuncSetAttribute(k_zt_grp<n, 1, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZK<n>::smem);
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

template <class S>
static void zt_grp_t(cudaStream_t st, int dir, int nz, const GrpTab<ZtArgs<S>>* t, int nblk) {
    switch (nz) {
#define Z_CASE(n)                                                                                               \
    case n:                                                                                                     \
        if (dir < 0) launch_pdl(k_zt_grp<n, -1, S>, dim3((unsigned)nblk), dim3(ZK<n>::P), ZK<n>::smem, st, t);  \
        else launch_pdl(k_zt_grp<n, 1, S>, dim3((unsigned)nblk), dim3(ZK<n>::P), ZK<n>::smem, st, t);           \
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

template <class S>
static void pfft_z_t(cudaStream_t st, int dir, int nx, int ny, int nz, S* spec, const double2* twz) {
    const int ncol = ny * (nx / 2 + 1);
    switch (nz) {
#define Z_CASE(n)                                                                                                 \
    case n: {                                                                                                     \
        const int grid = (ncol + ZK<n>::B - 1) / ZK<n>::B;                                                        \
        if (dir < 0) launch_pdl(k_zt<n, -1, S>, dim3(grid), dim3(ZK<n>::P), ZK<n>::smem, st, ncol, spec, twz);     \
        else launch_pdl(k_zt<n, 1, S>, dim3(grid), dim3(ZK<n>::P), ZK<n>::smem, st, ncol, spec, twz);              \
        break;                                                                                                    \
    }
        PFFT_Z_SIZES(Z_CASE)
#undef Z_CASE
        default: break;
    }
}
void launch_pfft_z(cudaStream_t st, int dir, int nx, int ny, int nz, double2* spec, const double2* twz) {
    pfft_z_t(st, dir, nx, ny, nz, spec, twz);
}
void launch_pfft_z(cudaStream_t st, int dir, int nx, int ny, int nz, float2* spec, const double2* twz) {
    pfft_z_t(st, dir, nx, ny, nz, spec, twz);
}

}  // namespace ptc
