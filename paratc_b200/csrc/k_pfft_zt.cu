// k_pfft_zt.cu -- the z transforms of the Poisson solve fed by TMA.
//
// Same transform as k_zt (k_pfft_z.cu): the spectrum for a fixed kz is one
// contiguous run of ncol = ny*(nx/2+1) complex values, and a batch is B
// consecutive columns, i.e. a (2B doubles) x (nz rows) box of the 2-D tensor
// [nz][2*ncol] -- a plain tiled TMA box.  A persistent CTA walks its batches
// with two shared-memory stages: while it transforms batch n in place, the
// tensor-memory accelerator loads batch n+1 into the other stage
// (cp.async.bulk.tensor, completion on an mbarrier) and the store of batch n
// (cp.async.bulk.tensor from shared memory) overlaps the next batch's
// passes.  Every wait on an mbarrier or a bulk group is bounded: after
// kSpinLimit polls the CTA records an error (*err |= 1) and stops.  No
// multicast; only this GPU's memory.
#include <cstdio>

#include "common.cuh"
#include "fft_fixed.cuh"
#include "kernels.cuh"
#include "tma.cuh"

namespace ptc {
namespace {

// W = 1: the wide batch (8 columns) for nz = 512 and 768 on large spectra.
// A batch reads one run of 2B doubles from every one of the nz rows; when
// those rows span more than 1 GB, runs of 64 B per row leave the copies bound
// by address translation (nz = 768: 0.36 of peak at 2304 x 192 x 768, 2.7 GB;
// 0.79 at 512 x 96 x 768), and 128 B per row restores them (0.71) at one CTA
// per SM.
// A: the complex type of the spectrum and of the passes (double2, or float2
// for the FP32 storage form's step)
template <int N, int W = 0, class A = double2>
struct ZT {
    static constexpr int B = (W && (N == 512 || N == 768)) ? 8 : (ff::Shape<N>::B < 4 ? 4 : ff::Shape<N>::B);
    static constexpr int P = B * N / ff::Shape<N>::RMAX;
    static constexpr int ROWS = N < 256 ? N : 256;  // TMA box rows (at most 256)
    static constexpr int NBOX = N / ROWS;
    static constexpr unsigned STAGE_BYTES = (unsigned)N * B * (unsigned)sizeof(A);
    static constexpr size_t smem = 1024 + 2 * (size_t)STAGE_BYTES + (size_t)N * sizeof(A);
};

// whether the CTA's iteration i has a batch (and so a load was issued for it)
__device__ __forceinline__ bool b_first_unused(int i, int nb) {
    return (long long)blockIdx.x + (long long)i * gridDim.x < nb;
}

template <int N, int DIR, int W, class A>
__global__ void __launch_bounds__(ZT<N, W, A>::P) k_zt_tma(const __grid_constant__ CUtensorMap tm, int nb,
                                                             const double2* __restrict__ twN,
                                                             unsigned int* __restrict__ err) {
    constexpr int B = ZT<N, W, A>::B, P = ZT<N, W, A>::P, ROWS = ZT<N, W, A>::ROWS, NBOX = ZT<N, W, A>::NBOX;
    constexpr unsigned SB = ZT<N, W, A>::STAGE_BYTES;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ unsigned char smraw[];
    // 1 KB-aligned stages (TMA destinations), then the twiddles, then the barriers
    unsigned char* base = smraw + ((1024 - (tma::smem_addr(smraw) & 1023)) & 1023);
    A* stage[2] = {reinterpret_cast<A*>(base), reinterpret_cast<A*>(base + SB)};
    A* tws = reinterpret_cast<A*>(base + 2 * SB);
    __shared__ unsigned long long mbar[2];
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    const long long lim = tma::wait_limit(err);
    for (int t = tid; t < N; t += P) tws[t] = cto<A>(twN[t]);
    if (tid == 0) {
        tma::mbar_init(&mbar[0], 1);
        tma::mbar_init(&mbar[1], 1);
        tma::fence_mbar_init();
        s_bad = 0;
    }
    __syncthreads();
    pdl_wait();  // the spectrum is written by the kernel before this one
    pdl_trigger();
    auto issue = [&](int s, int b) {
        tma::mbar_expect_tx(&mbar[s], SB);
#pragma unroll
        for (int r = 0; r < NBOX; r++)
            tma::load_2d(stage[s] + (size_t)r * ROWS * B, &tm, 2 * B * b, r * ROWS, &mbar[s]);
    };
    if (tid == 0) {
        if ((int)blockIdx.x < nb) issue(0, blockIdx.x);
        if ((int)(blockIdx.x + gridDim.x) < nb) issue(1, blockIdx.x + gridDim.x);
    }
    int it = 0;
    for (int b = blockIdx.x; b < nb; b += gridDim.x, it++) {
        const int s = it & 1;
        A* buf = stage[s];
        // one decision for the whole CTA: a flag read after a plain barrier
        // could be set by a faster thread's next wait before a slower one
        // reads it, and the two would then part at the next barrier
        if (__syncthreads_or(tma::mbar_wait(&mbar[s], (unsigned)((it >> 1) & 1), lim) ? 0 : 1)) {
            s_bad = 1;
            break;
        }
        ff::smem_passes<N, B, B, P, DIR, 0, SC.np>(buf, static_cast<const A*>(tws), tid);
        tma::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
#pragma unroll
            for (int r = 0; r < NBOX; r++) tma::store_2d(&tm, 2 * B * b, r * ROWS, buf + (size_t)r * ROWS * B);
            tma::bulk_commit();
            const int bn = b + 2 * gridDim.x;
            if (bn < nb) {
                tma::bulk_wait_read0();  // the store has read this stage
                issue(s, bn);
            }
        }
    }
    if (tid == 0) {
        tma::bulk_wait0();
        if (s_bad) {
            atomicOr(err, 1u);
            // loads still in flight land in this CTA's stages: wait for them (bounded)
            for (int t = 0; t < 2; t++) {
                const int i = ((it & 1) == t) ? it : it + 1;  // the stage's oldest unconsumed use
                if (b_first_unused(i, nb)) tma::mbar_wait(&mbar[t], (unsigned)((i >> 1) & 1));
            }
        }
    }
}

#define ZT_SIZES(X) X(128) X(256) X(512) X(768) X(1024)

template <int N, int W>
int zt_batch() { return ZT<N, W>::B; }

// the wide batch where it exists and a batch's rows span more than 1 GB
// (esize: bytes of a complex value)
bool zt_wide(int ncol, int nz, int esize = 16) {
    return (nz == 512 || nz == 768) && (size_t)ncol * esize * (size_t)nz > ((size_t)1 << 30);
}

}  // namespace

PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

bool zt_tma_supported(int nz) {
    switch (nz) {
#define X_CASE(n) case n:
        ZT_SIZES(X_CASE)
#undef X_CASE
        return true;
        default: return false;
    }
}

#define ZT_ATTR(n, w, A)                                                                                       \
    cudaFuncSetAttribute(k_zt_tma<n, -1, w, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,                  \
                         (int)ZT<n, w, A>::smem);                                                              \
    cudaFuncSetAttribute(k_zt_tma<n, 1, w, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZT<n, w, A>::smem);

void zt_tma_init() {
#define X_CASE(n) ZT_ATTR(n, 0, double2) ZT_ATTR(n, 0, float2)
    ZT_SIZES(X_CASE)
#undef X_CASE
    ZT_ATTR(512, 1, double2) ZT_ATTR(768, 1, double2) ZT_ATTR(512, 1, float2) ZT_ATTR(768, 1, float2)
}

// the tensor map of the spectrum viewed as [nz][2*ncol] reals (FP64, or FP32
// for a float2 spectrum: esize 8) with the batch box (2B x min(nz, 256));
// false when the driver cannot encode it (a float2 spectrum also needs ncol
// even, the row stride a multiple of 16 bytes)
static bool zt_prepare(void* spec, int ncol, int nz, int esize, void* tmap_out) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encode_fn();
    if (!enc || !zt_tma_supported(nz)) return false;
    if (((size_t)ncol * esize) % 16 != 0) return false;
    int B = 0;
    if (zt_wide(ncol, nz, esize)) B = nz == 512 ? zt_batch<512, 1>() : zt_batch<768, 1>();
    else switch (nz) {
#define X_CASE(n) case n: B = zt_batch<n, 0>(); break;
        ZT_SIZES(X_CASE)
#undef X_CASE
        default: return false;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)2 * ncol, (cuuint64_t)nz};
    const cuuint64_t strides[1] = {(cuuint64_t)ncol * esize};
    const cuuint32_t box[2] = {(cuuint32_t)(2 * B), (cuuint32_t)(nz < 256 ? nz : 256)};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(reinterpret_cast<CUtensorMap*>(tmap_out),
                           esize == 16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, spec,
                           dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}
bool zt_tma_prepare(double2* spec, int ncol, int nz, void* tmap_out) { return zt_prepare(spec, ncol, nz, 16, tmap_out); }
bool zt_tma_prepare(float2* spec, int ncol, int nz, void* tmap_out) { return zt_prepare(spec, ncol, nz, 8, tmap_out); }

template <class A>
static void zt_tma_t(cudaStream_t st, int dir, int ncol, int nz, const void* tmap, const double2* twz, int nsm,
                     unsigned int* err) {
    const CUtensorMap& tm = *reinterpret_cast<const CUtensorMap*>(tmap);
#define ZT_LAUNCH(n, w)                                                                                        \
    {                                                                                                          \
        using Z = ZT<n, w, A>;                                                                                 \
        const int nb = (ncol + Z::B - 1) / Z::B;                                                               \
        const int per_sm = (int)((220 * 1024) / Z::smem);                                                      \
        int grid = (per_sm > 0 ? per_sm : 1) * nsm;                                                            \
        if (grid > nb) grid = nb;                                                                              \
        if (dir < 0) launch_pdl(k_zt_tma<n, -1, w, A>, dim3(grid), dim3(Z::P), Z::smem, st, tm, nb, twz, err);  \
        else launch_pdl(k_zt_tma<n, 1, w, A>, dim3(grid), dim3(Z::P), Z::smem, st, tm, nb, twz, err);           \
    }
    if (zt_wide(ncol, nz, (int)sizeof(A))) {
        if (nz == 512) ZT_LAUNCH(512, 1)
        else ZT_LAUNCH(768, 1)
        return;
    }
    switch (nz) {
#define X_CASE(n)                                                                                              \
    case n: ZT_LAUNCH(n, 0) break;
        ZT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
#undef ZT_LAUNCH
}
void launch_zt_tma(cudaStream_t st, int dir, int ncol, int nz, const void* tmap, const double2* twz, int nsm,
                   unsigned int* err) {
    zt_tma_t<double2>(st, dir, ncol, nz, tmap, twz, nsm, err);
}
void launch_zt_tma32(cudaStream_t st, int dir, int ncol, int nz, const void* tmap, const double2* twz, int nsm,
                     unsigned int* err) {
    zt_tma_t<float2>(st, dir, ncol, nz, tmap, twz, nsm, err);
}

}  // namespace ptc
