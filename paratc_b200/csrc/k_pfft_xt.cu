// k_pfft_xt.cu -- the x transforms of the Poisson solve fed by bulk copies.
//
// The same packed real transforms as k_xf (given source) and k_xb
// (k_pfft_x.cu), with the rows moved by the tensor-memory accelerator
// instead of by threads.  A persistent CTA keeps two shared-memory stages of
// B rows, each row contiguous (row b at b*PITCH complex values, which is the
// layout the bulk copies need), and walks its batches: while it transforms
// one stage, cp.async.bulk loads (completion on an mbarrier) fill the other,
// and the previous results leave through bulk stores from shared memory.
//
// Inverse (k_xb_tma): spectrum rows of nx/2+1 complex values in, merge of
// modes a and N-a with 1/(nx*nz) folded in, inverse FFT, phi rows out, with
// the Neumann ghost copies phi(0) = phi(1), phi(nyp) = phi(nyc) of the
// padded layout (SetBC_and_UpdateHalo_pr, src/m_BC_and_Halo.f90:115-120).
// Forward (k_xf_tma): rows of a given source in, FFT, split in place into
// the nx/2+1 modes of the real transform, spectrum rows out.  Forward of the
// divergence source (k_xf_div, Poisson schedules 8-11): the same consumer
// side, with producer warps computing the source rows into the stages.
//
// Every wait is bounded: after kSpinLimit polls the CTA records an error
// (*err |= 2, or 4 for k_xf_div), waits (bounded) for its own copies in
// flight and stops.  No multicast; only this GPU's memory.
#include <type_traits>

#include "common.cuh"
#include "fft_fixed.cuh"
#include "kernels.cuh"
#include "div_src.cuh"
#include "reduce.cuh"
#include "tma.cuh"

namespace ptc {
namespace {

template <int N>
struct XT {
    // at least two rows per batch: single-row batches of nx = 3072 ran at 0.40
    // of peak, two-row ones at 0.47 (one CTA per SM)
    static constexpr int BM = ff::Shape<N>::B < 2 ? 2 : 1;
    static constexpr int B = ff::Shape<N>::B * BM;
    static constexpr int P = ff::Shape<N>::P * BM;
    static constexpr int M1 = N + 1;
    // row pitch in complex values: at least N+1, with B*PITCH residues that
    // spread a quarter warp's (row, element) pairs over the eight 16-byte
    // bank groups (b fastest across lanes, then consecutive elements)
    static constexpr int pitch() {
        const int want = B >= 8 ? 1 : 8 / B;
        int p = M1;
        while (B > 1 && p % 8 != want % 8) p++;
        return p;
    }
    static constexpr int PITCH = pitch();
    static constexpr unsigned STAGE = (unsigned)B * PITCH;  // complex values per stage
    static constexpr size_t smem = 2 * (size_t)STAGE * sizeof(double2);
    // resident CTAs that the shared memory allows: the register target of
    // the launch bounds (without it k_xb_tma<1152> takes 236 registers and
    // runs one CTA per SM: 0.28 of peak against 0.39)
    static constexpr int mcalc() {
        const int m = (int)((220 * 1024) / (smem + 1024));
        return m < 1 ? 1 : (m > 8 ? 8 : m);
    }
    static constexpr int MINB = mcalc();
    // between passes the rows are kept in the swizzled order (fft_fixed.cuh):
    // with 1 or 2 rows per batch, a first pass's stores otherwise fall in one
    // bank group
    static constexpr bool SWZ = N % 8 == 0;
};

// whether the CTA's iteration i has a batch (and so a load was issued for it)
__device__ __forceinline__ bool xt_has(int i, int nb) {
    return (long long)blockIdx.x + (long long)i * gridDim.x < nb;
}

// the error path: record, then wait (bounded) for the loads still in flight
// into this CTA's stages; it runs in thread 0 after its stores drained
__device__ __forceinline__ void xt_fail(unsigned long long* mbar, int it, int nb, unsigned int* err) {
    atomicOr(err, 2u);
    for (int t = 0; t < 2; t++) {
        const int i = ((it & 1) == t) ? it : it + 1;  // the stage's oldest unconsumed use
        if (xt_has(i, nb)) tma::mbar_wait(&mbar[t], (unsigned)((i >> 1) & 1));
    }
}

// Where the inverse finds spectrum row g: one contiguous row of the
// spectrum (RowsContig), or the segments of the row that the ranks of a
// z-slab decomposition hold in their x-slabs (RowsGathered: modes
// [kx0_q, kx0_q + nxl_q) of local row g = (kl, jc) in rank q's x-slab at
// ((k0*ny + g)*nxl_q), one bulk copy per segment; the x-slabs may be other
// GPUs' memory, mapped here, read by plain (non-multicast) bulk copies).
struct RowsContig {
    const double2* spec;
    __device__ __forceinline__ void load(double2* dst, int g, int M1, unsigned long long* mbar) const {
        tma::bulk_load(dst, spec + (size_t)g * M1, M1 * (unsigned)sizeof(double2), mbar);
    }
};
struct RowsGathered {
    const XtGather* t;  // the kernel's __grid_constant__ parameter
    int ny;
    __device__ __forceinline__ void load(double2* dst, int g, int M1, unsigned long long* mbar) const {
        const int G = t->G, base = M1 / G, rem = M1 - base * G;
        const size_t row = (size_t)t->k0 * ny + g;
        for (int q = 0; q < G; q++) {
            const int kx0 = q * base + (q < rem ? q : rem), nxl = base + (q < rem ? 1 : 0);
            tma::bulk_load(dst + kx0, t->p[q] + row * nxl, nxl * (unsigned)sizeof(double2), mbar);
        }
    }
};

template <int N, class Rows>
__device__ __forceinline__ void xb_tma_body(int nrows, int ny, const Rows& rows, double* __restrict__ phi,
                                            const double2* __restrict__ twN, const double2* __restrict__ post,
                                            double scale, int padded, unsigned int* __restrict__ err) {
    constexpr int B = XT<N>::B, P = XT<N>::P, PITCH = XT<N>::PITCH, M1 = N + 1;
    constexpr unsigned SB = XT<N>::STAGE;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ __align__(128) unsigned char smraw[];
    double2* stage[2] = {reinterpret_cast<double2*>(smraw), reinterpret_cast<double2*>(smraw) + SB};
    __shared__ unsigned long long mbar[2];
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    const long long lim = tma::wait_limit(err);
    const int nb = (nrows + B - 1) / B;
    const int nx = 2 * N, nyt = ny + 2;
    if (tid == 0) {
        tma::mbar_init(&mbar[0], 1);
        tma::mbar_init(&mbar[1], 1);
        tma::fence_mbar_init();
        s_bad = 0;
    }
    __syncthreads();
    pdl_wait();  // the spectrum is written by the kernel before this one
    pdl_trigger();
    auto issue = [&](int s, int bt) {
        const int g0 = bt * B, nv = min(B, nrows - g0);
        tma::mbar_expect_tx(&mbar[s], (unsigned)nv * M1 * (unsigned)sizeof(double2));
        for (int b = 0; b < nv; b++) rows.load(stage[s] + b * PITCH, g0 + b, M1, &mbar[s]);
    };
    if (tid == 0) {
        if ((int)blockIdx.x < nb) issue(0, blockIdx.x);
        if ((int)(blockIdx.x + gridDim.x) < nb) issue(1, blockIdx.x + gridDim.x);
    }
    int it = 0;
    for (int bt = blockIdx.x; bt < nb; bt += gridDim.x, it++) {
        const int s = it & 1;
        double2* buf = stage[s];
        // one decision for the whole CTA: a flag read after a plain barrier
        // could be set by a faster thread's next wait before a slower one
        // reads it, and the two would then part at the next barrier
        if (__syncthreads_or(tma::mbar_wait(&mbar[s], (unsigned)((it >> 1) & 1), lim) ? 0 : 1)) {
            s_bad = 1;
            break;
        }
        // merge modes a and N-a of every row into z[a], z[N-a] (the DC and
        // Nyquist coefficients are real), scaled by 1/(nx*nz)
        for (int f = tid; f < B * (N / 2 + 1); f += P) {
            const int a = f / B, b = f - a * B;
            const int bn = N - a;
            double2* rb = buf + b * PITCH;
            double2 xa = rb[a], xb = rb[bn];
            if (a == 0) { xa.y = 0.0; xb.y = 0.0; }
            const double2 e2a = make_double2(xa.x + xb.x, xa.y - xb.y);
            const double2 da = make_double2(xa.x - xb.x, xa.y + xb.y);
            const double2 o2a = cmulc(da, __ldg(&post[a]));
            const double2 za = make_double2(scale * (e2a.x - o2a.y), scale * (e2a.y + o2a.x));
            if (a == 0) {
                rb[0] = za;
            } else {
                const double2 e2b = make_double2(xb.x + xa.x, xb.y - xa.y);
                const double2 db = make_double2(xb.x - xa.x, xb.y + xa.y);
                const double2 o2b = cmulc(db, __ldg(&post[bn]));
                rb[a] = za;
                if (bn != a) rb[bn] = make_double2(scale * (e2b.x - o2b.y), scale * (e2b.y + o2b.x));
            }
        }
        __syncthreads();
        ff::smem_passes<N, B, PITCH, P, 1, 0, SC.np, 4, true, 0, XT<N>::SWZ>(buf, twN, tid);
        tma::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            const int g0 = bt * B, nv = min(B, nrows - g0);
            constexpr unsigned RB = N * (unsigned)sizeof(double2);
            for (int b = 0; b < nv; b++) {
                const int g = g0 + b;
                const double2* row = buf + b * PITCH;
                if (!padded) {
                    tma::bulk_store(phi + (size_t)g * nx, row, RB);
                    continue;
                }
                const int k = g / ny, jc = g - k * ny + 1;
                double* rowp = phi + ((size_t)k * nyt + jc) * nx;
                tma::bulk_store(rowp, row, RB);
                if (jc == 1) tma::bulk_store(rowp - nx, row, RB);
                if (jc == ny) tma::bulk_store(rowp + nx, row, RB);
            }
            tma::bulk_commit();
            const int bn = bt + 2 * gridDim.x;
            if (bn < nb) {
                tma::bulk_wait_read0();  // the stores have read this stage
                issue(s, bn);
            }
        }
    }
    if (tid == 0) {
        tma::bulk_wait0();
        if (s_bad) xt_fail(mbar, it, nb, err);
    }
}

template <int N>
__global__ void __launch_bounds__(XT<N>::P, XT<N>::MINB)
    k_xb_tma(int nrows, int ny, const double2* __restrict__ spec, double* __restrict__ phi,
             const double2* __restrict__ twN, const double2* __restrict__ post, double scale, int padded,
             unsigned int* __restrict__ err) {
    xb_tma_body<N>(nrows, ny, RowsContig{spec}, phi, twN, post, scale, padded, err);
}

// the same inverse with the rows gathered from the ranks' x-slabs
template <int N>
__global__ void __launch_bounds__(XT<N>::P, XT<N>::MINB)
    k_xb_tma_gather(int nrows, int ny, const __grid_constant__ XtGather gt, double* __restrict__ phi,
                    const double2* __restrict__ twN, const double2* __restrict__ post, double scale,
                    unsigned int* __restrict__ err) {
    xb_tma_body<N>(nrows, ny, RowsGathered{&gt, ny}, phi, twN, post, scale, 0, err);
}

// The inverse of the FP32 storage form: float2 spectrum rows in, float phi
// rows out, the merge and the passes in float (the stages hold float2, half
// the FP64 stage, and the float2 twiddles sit after them).  A float2 row has
// N+1 (odd) values, so a row starts 16-byte aligned only at an even index:
// rows are loaded two at a time (the batches hold an even number of rows and
// start at an even row, and the host launches the kernel for an even row
// count only; an odd last row would be loaded with the one float2 after it,
// inside the spectrum's allocation, which holds the FP64 spectrum's bytes).
// The rows land contiguously at the start of the stage
// and are moved to the pitched layout by the merge, which reads all its
// inputs before a barrier and writes after it; the phi rows leave through
// coalesced stores of the threads.
template <int N>
__global__ void __launch_bounds__(XT<N>::P, XT<N>::MINB)
    k_xb_tma32(int nrows, int ny, const float2* __restrict__ spec, float* __restrict__ phi,
               const double2* __restrict__ twN, const double2* __restrict__ post, double scale, int padded,
               unsigned int* __restrict__ err) {
    constexpr int B = XT<N>::B, P = XT<N>::P, PITCH = XT<N>::PITCH, M1 = N + 1;
    static_assert(B % 2 == 0, "row pairs");
    constexpr int NPAIR = B * (N / 2 + 1);
    constexpr int KP = (NPAIR + P - 1) / P;  // merge pairs per thread
    constexpr unsigned SB = XT<N>::STAGE;
    static_assert(2 * SB >= (unsigned)N, "the twiddles fit after the float2 stages");
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ __align__(128) unsigned char smraw[];
    float2* stage[2] = {reinterpret_cast<float2*>(smraw), reinterpret_cast<float2*>(smraw) + SB};
    float2* tws = reinterpret_cast<float2*>(smraw) + 2 * SB;
    __shared__ unsigned long long mbar[2];
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    const long long lim = tma::wait_limit(err);
    const int nb = (nrows + B - 1) / B;
    const int nx = 2 * N, nyt = ny + 2;
    for (int t = tid; t < N; t += P) tws[t] = cto<float2>(twN[t]);
    if (tid == 0) {
        tma::mbar_init(&mbar[0], 1);
        tma::mbar_init(&mbar[1], 1);
        tma::fence_mbar_init();
        s_bad = 0;
    }
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    auto issue = [&](int s, int bt) {
        const int g0 = bt * B, nv = min(B, nrows - g0);
        unsigned bytes = 0;
        for (int b = 0; b < nv; b += 2) bytes += (unsigned)(b + 1 < nv ? 2 * M1 : M1 + 1) * (unsigned)sizeof(float2);
        tma::mbar_expect_tx(&mbar[s], bytes);
        for (int b = 0; b < nv; b += 2) {
            const unsigned n2 = (unsigned)(b + 1 < nv ? 2 * M1 : M1 + 1) * (unsigned)sizeof(float2);
            tma::bulk_load(stage[s] + b * M1, spec + (size_t)(g0 + b) * M1, n2, &mbar[s]);
        }
    };
    if (tid == 0) {
        if ((int)blockIdx.x < nb) issue(0, blockIdx.x);
        if ((int)(blockIdx.x + gridDim.x) < nb) issue(1, blockIdx.x + gridDim.x);
    }
    const float fsc = (float)scale;
    int it = 0;
    for (int bt = blockIdx.x; bt < nb; bt += gridDim.x, it++) {
        const int s = it & 1;
        float2* buf = stage[s];
        if (__syncthreads_or(tma::mbar_wait(&mbar[s], (unsigned)((it >> 1) & 1), lim) ? 0 : 1)) {
            s_bad = 1;
            break;
        }
        const int g0 = bt * B, nv = min(B, nrows - g0);
        // merge, reading every input first (the pitched rows overlay them)
        float2 xa_[KP], xb_[KP];
#pragma unroll
        for (int k = 0; k < KP; k++) {
            const int f = tid + k * P;
            if (f < NPAIR) {
                const int a = f / B, b = f - a * B;
                xa_[k] = buf[b * M1 + a];
                xb_[k] = buf[b * M1 + (N - a)];
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < KP; k++) {
            const int f = tid + k * P;
            if (f >= NPAIR) continue;
            const int a = f / B, b = f - a * B;
            const int bn = N - a;
            float2* rb = buf + b * PITCH;
            float2 xa = xa_[k], xb = xb_[k];
            if (a == 0) { xa.y = 0.f; xb.y = 0.f; }
            const float2 e2a = make_float2(xa.x + xb.x, xa.y - xb.y);
            const float2 da = make_float2(xa.x - xb.x, xa.y + xb.y);
            const float2 o2a = cmulc(da, cto<float2>(__ldg(&post[a])));
            const float2 za = make_float2(fsc * (e2a.x - o2a.y), fsc * (e2a.y + o2a.x));
            if (a == 0) {
                rb[0] = za;
            } else {
                const float2 e2b = make_float2(xb.x + xa.x, xb.y - xa.y);
                const float2 db = make_float2(xb.x - xa.x, xb.y + xa.y);
                const float2 o2b = cmulc(db, cto<float2>(__ldg(&post[bn])));
                rb[a] = za;
                if (bn != a) rb[bn] = make_float2(fsc * (e2b.x - o2b.y), fsc * (e2b.y + o2b.x));
            }
        }
        __syncthreads();
        ff::smem_passes<N, B, PITCH, P, 1, 0, SC.np, 4, true, 0, XT<N>::SWZ>(buf, static_cast<const float2*>(tws),
                                                                             tid);
        __syncthreads();
        // phi rows (and the Neumann ghost copies) by coalesced float2 stores
        for (int e = tid; e < nv * N; e += P) {
            const int b = e / N, i = e - b * N;
            const float2 v = buf[b * PITCH + i];
            const int g = g0 + b;
            if (!padded) {
                reinterpret_cast<float2*>(phi + (size_t)g * nx)[i] = v;
                continue;
            }
            const int k = g / ny, jc = g - k * ny + 1;
            float2* rowp = reinterpret_cast<float2*>(phi + ((size_t)k * nyt + jc) * nx);
            rowp[i] = v;
            if (jc == 1) rowp[i - N] = v;
            if (jc == ny) rowp[i + N] = v;
        }
        // the stage's generic reads are done before the next bulk load writes it
        tma::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            const int bn = bt + 2 * gridDim.x;
            if (bn < nb) issue(s, bn);
        }
    }
    if (tid == 0 && s_bad) xt_fail(mbar, it, nb, err);
}

// Where the forward sends spectrum row g: one contiguous row of the spectrum
// by bulk stores from thread 0 (RowsToSpec), or every mode straight into its
// owner's x-slab of a z-slab decomposition by plain stores of all threads
// (RowsScattered: mode kx of local row g = (kl, jc) to rank q's x-slab at
// ((k0*ny + g)*nxl_q + kx - kx0_q); the x-slabs may be other GPUs' memory,
// written over NVLink).  `bulk` tells the kernel which of the two it is.
struct RowsToSpec {
    static constexpr bool bulk = true;
    double2* spec;
    __device__ __forceinline__ void store(int g, const double2* row, int M1) const {
        tma::bulk_store(spec + (size_t)g * M1, row, M1 * (unsigned)sizeof(double2));
    }
};
struct RowsScattered {
    static constexpr bool bulk = false;
    const XtGather* t;  // the kernel's __grid_constant__ parameter (pointers written through)
    int ny;
    __device__ __forceinline__ void put(int g, int kx, double2 v, int M1) const {
        const int G = t->G, base = M1 / G, rem = M1 - base * G, cut = rem * (base + 1);
        const int q = kx < cut ? kx / (base + 1) : rem + (kx - cut) / base;
        const int kx0 = q * base + (q < rem ? q : rem), nxl = base + (q < rem ? 1 : 0);
        const_cast<double2*>(t->p[q])[((size_t)t->k0 * ny + g) * nxl + (kx - kx0)] = v;
    }
};

template <int N, class Out>
__device__ __forceinline__ void xf_tma_body(int nrows, const double* __restrict__ src, const Out& out,
                                            const double2* __restrict__ twN, const double2* __restrict__ post,
                                            unsigned int* __restrict__ err) {
    constexpr int B = XT<N>::B, P = XT<N>::P, PITCH = XT<N>::PITCH, M1 = N + 1;
    constexpr unsigned SB = XT<N>::STAGE;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ __align__(128) unsigned char smraw[];
    double2* stage[2] = {reinterpret_cast<double2*>(smraw), reinterpret_cast<double2*>(smraw) + SB};
    __shared__ unsigned long long mbar[2];
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    const long long lim = tma::wait_limit(err);
    const int nb = (nrows + B - 1) / B;
    const int nx = 2 * N;
    if (tid == 0) {
        tma::mbar_init(&mbar[0], 1);
        tma::mbar_init(&mbar[1], 1);
        tma::fence_mbar_init();
        s_bad = 0;
    }
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    auto issue = [&](int s, int bt) {
        const int g0 = bt * B, nv = min(B, nrows - g0);
        tma::mbar_expect_tx(&mbar[s], (unsigned)nv * N * (unsigned)sizeof(double2));
        for (int b = 0; b < nv; b++)
            tma::bulk_load(stage[s] + b * PITCH, src + (size_t)(g0 + b) * nx, N * (unsigned)sizeof(double2), &mbar[s]);
    };
    if (tid == 0) {
        if ((int)blockIdx.x < nb) issue(0, blockIdx.x);
        if ((int)(blockIdx.x + gridDim.x) < nb) issue(1, blockIdx.x + gridDim.x);
    }
    int it = 0;
    for (int bt = blockIdx.x; bt < nb; bt += gridDim.x, it++) {
        const int s = it & 1;
        double2* buf = stage[s];
        // one decision for the whole CTA: a flag read after a plain barrier
        // could be set by a faster thread's next wait before a slower one
        // reads it, and the two would then part at the next barrier
        if (__syncthreads_or(tma::mbar_wait(&mbar[s], (unsigned)((it >> 1) & 1), lim) ? 0 : 1)) {
            s_bad = 1;
            break;
        }
        ff::smem_passes<N, B, PITCH, P, -1, 0, SC.np, 4, true, 0, XT<N>::SWZ>(buf, twN, tid);
        // split the packed transform into the nx/2+1 modes, in place: one
        // thread takes the pair (a, N-a) (and a = 0 also writes mode N)
        for (int f = tid; f < B * (N / 2 + 1); f += P) {
            const int a = f / B, b = f - a * B;
            const int bn = N - a;
            double2* rb = buf + b * PITCH;
            const double2 za = rb[a], zb = rb[a == 0 ? 0 : bn];
            const double2 E = make_double2(0.5 * (za.x + zb.x), 0.5 * (za.y - zb.y));
            const double2 O = make_double2(0.5 * (za.y + zb.y), -0.5 * (za.x - zb.x));
            const double2 xa = cadd(E, cmul(__ldg(&post[a]), O));
            if (a == 0) {
                rb[0] = xa;
                rb[N] = cadd(E, cmul(__ldg(&post[N]), O));
            } else if (bn != a) {
                const double2 E2 = make_double2(0.5 * (zb.x + za.x), 0.5 * (zb.y - za.y));
                const double2 O2 = make_double2(0.5 * (zb.y + za.y), -0.5 * (zb.x - za.x));
                rb[a] = xa;
                rb[bn] = cadd(E2, cmul(__ldg(&post[bn]), O2));
            } else {
                rb[a] = xa;
            }
        }
        if constexpr (Out::bulk) {
            tma::fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                const int g0 = bt * B, nv = min(B, nrows - g0);
                for (int b = 0; b < nv; b++) out.store(g0 + b, buf + b * PITCH, M1);
                tma::bulk_commit();
                const int bn = bt + 2 * gridDim.x;
                if (bn < nb) {
                    tma::bulk_wait_read0();
                    issue(s, bn);
                }
            }
        } else {
            __syncthreads();
            const int g0 = bt * B, nv = min(B, nrows - g0);
            for (int f = tid; f < nv * M1; f += P) {
                const int b = f / M1, kx = f - b * M1;
                out.put(g0 + b, kx, buf[b * PITCH + kx], M1);
            }
            tma::fence_async_smem();  // this thread's stage accesses before the refill's async writes
            __syncthreads();          // every thread has read the stage before it is refilled
            const int bn = bt + 2 * gridDim.x;
            if (tid == 0 && bn < nb) issue(s, bn);
        }
    }
    if (tid == 0) {
        tma::bulk_wait0();
        if (s_bad) xt_fail(mbar, it, nb, err);
    }
}

template <int N>
__global__ void __launch_bounds__(XT<N>::P, XT<N>::MINB)
    k_xf_tma(int nrows, const double* __restrict__ src, double2* __restrict__ spec, const double2* __restrict__ twN,
             const double2* __restrict__ post, unsigned int* __restrict__ err) {
    xf_tma_body<N>(nrows, src, RowsToSpec{spec}, twN, post, err);
}

// the same forward transform with every mode stored straight into its
// owner's x-slab
template <int N>
__global__ void __launch_bounds__(XT<N>::P, XT<N>::MINB)
    k_xf_tma_scatter(int nrows, int ny, const double* __restrict__ src, const __grid_constant__ XtGather gt,
                     const double2* __restrict__ twN, const double2* __restrict__ post, unsigned int* __restrict__ err) {
    xf_tma_body<N>(nrows, src, RowsScattered{&gt, ny}, twN, post, err);
}

// ---------------------------------------------------------------------------
// Forward transform of the divergence source (clcPrSrc, src/m_TScheme.f90:
// 48-77: scaled by 1/pmAlpha in mode 0, unscaled in mode 1, max|div| reduced
// over the grid by the last CTA), warp-specialised: XD_Q producer threads
// compute the divergence of the next batch's rows from u, v, w into one
// stage while the P consumer threads transform the other stage, split it
// into the nx/2+1 modes and send the spectrum rows out by bulk stores.
// Stages change hands through mbarriers: full[s] (the producers' arrivals,
// release) and empty[s] (consumer thread 0, once the stores have read the
// stage).  The consumers synchronise among themselves on named barrier 1,
// the producers on named barrier 2; a group decides to stop on a barrier
// that reduces the predicate, so all its threads decide alike.  Every wait is
// bounded; a group that gives up leaves its loop, the other group's waits
// then run out too, and the CTA records *err |= 4.
// ---------------------------------------------------------------------------
constexpr int XD_Q = 256;      // producer threads
constexpr int XD_DIV_U = 2;    // divergence point pairs in flight per producer thread

template <int N>
struct XD {
    static constexpr int RMAX = ff::Shape<N>::RMAX;
    // rows per batch: the transform's batch, doubled until its thread count
    // is whole warps (named barriers count warps)
    static constexpr int bcalc() {
        int b = ff::Shape<N>::B;
        while ((b * N / RMAX) % 32 != 0 && b < 64) b *= 2;
        return b;
    }
    static constexpr int B = bcalc();
    static constexpr int P = B * N / RMAX;
    static constexpr int pitch() {
        const int want = B >= 8 ? 1 : 8 / B;
        int p = N + 1;
        while (B > 1 && p % 8 != want % 8) p++;
        return p;
    }
    static constexpr int PITCH = pitch();
    static constexpr unsigned STAGE = (unsigned)B * PITCH;
    static constexpr int NT = P + XD_Q;
    static constexpr size_t smem = 2 * (size_t)STAGE * sizeof(double2);
};

// V: storage of the velocity, S: of the spectrum.  The FP32 storage form
// (float, float2) writes the spectrum rows with the consumers' own coalesced
// stores: a float2 row of N+1 values starts 16-byte aligned only at even
// rows, which a bulk store needs.
template <int N, class V, class S>
__global__ void __launch_bounds__(XD<N>::NT, 1)
    k_xf_div(int mode, DConst c, DMetric m, const DCoef* __restrict__ coef, const V* __restrict__ ux,
             const V* __restrict__ uy, const V* __restrict__ uz, S* __restrict__ spec,
             const double2* __restrict__ twN, const double2* __restrict__ post, double* __restrict__ part,
             unsigned int* __restrict__ counter, double* __restrict__ out_max, unsigned int* __restrict__ err) {
    constexpr int B = XD<N>::B, P = XD<N>::P, PITCH = XD<N>::PITCH, M1 = N + 1, Q = XD_Q;
    static_assert(P % 32 == 0, "the consumer group is whole warps");
    // the passes' complex type: float2 for the FP32 storage form (the stages
    // hold float2, half the FP64 stage, and the float2 twiddles sit after
    // them), double2 otherwise (the twiddles read from the global table)
    using A = std::conditional_t<sizeof(S) == sizeof(float2), float2, double2>;
    constexpr bool F32 = sizeof(A) == sizeof(float2);
    constexpr unsigned SB = XD<N>::STAGE;
    static_assert(!F32 || 2 * SB >= (unsigned)N, "the twiddles fit after the float2 stages");
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ __align__(128) unsigned char smraw[];
    A* stage[2] = {reinterpret_cast<A*>(smraw), reinterpret_cast<A*>(smraw) + SB};
    float2* tws32 = reinterpret_cast<float2*>(smraw) + 2 * SB;
    __shared__ unsigned long long full[2], empty[2];
    __shared__ int bad_c, bad_p;
    const int tid = threadIdx.x;
    const int nrows = c.ny * c.nz;
    const int nb = (nrows + B - 1) / B;
    const long long lim = tma::wait_limit(err);
    if constexpr (F32)
        for (int t = tid; t < N; t += XD<N>::NT) tws32[t] = cto<float2>(twN[t]);
    const A* tw;
    if constexpr (F32) tw = reinterpret_cast<const A*>(tws32);
    else tw = reinterpret_cast<const A*>(twN);
    if (tid == 0) {
        tma::mbar_init(&full[0], Q);
        tma::mbar_init(&full[1], Q);
        tma::mbar_init(&empty[0], 1);
        tma::mbar_init(&empty[1], 1);
        tma::fence_mbar_init();
        bad_c = bad_p = 0;
    }
    __syncthreads();
    pdl_wait();  // u* is written by the kernel before this one
    pdl_trigger();
    double dm = 0.0;
    if (tid >= P) {
        // producers
        const int tp = tid - P;
        const double sudtal = (mode == 0) ? 1.0 / coef->pmAlpha : 1.0;
        int it = 0;
        for (int bt = blockIdx.x; bt < nb; bt += gridDim.x, it++) {
            const int s = it & 1;
            const bool ok = it < 2 || tma::mbar_wait(&empty[s], (unsigned)(((it >> 1) + 1) & 1), lim);
            if (ff::group_any<2, Q>(!ok)) {
                bad_p = 1;
                break;
            }
            A* buf = stage[s];
            div_batch<N, B, Q, XD_DIV_U>(c, m, ux, uy, uz, bt * B, nrows, sudtal, tp, dm,
                                         [&](int b, int e, double2 v) { buf[b * PITCH + e] = cto<A>(v); });
            tma::mbar_arrive(&full[s]);
        }
    } else {
        // consumers
        int it = 0;
        for (int bt = blockIdx.x; bt < nb; bt += gridDim.x, it++) {
            const int s = it & 1;
            A* buf = stage[s];
            if (ff::group_any<1, P>(!tma::mbar_wait(&full[s], (unsigned)((it >> 1) & 1), lim))) {
                bad_c = 1;
                break;
            }
            ff::smem_passes<N, B, PITCH, P, -1, 0, SC.np, 4, true, 1, N % 8 == 0>(buf, tw, tid);
            if constexpr (sizeof(S) != sizeof(double2)) {
                // the split straight to the float2 spectrum rows (consecutive
                // threads take consecutive modes of one row: coalesced stores)
                const int g0 = bt * B, nv = min(B, nrows - g0);
                for (int f = tid; f < nv * (N / 2 + 1); f += P) {
                    const int b = f / (N / 2 + 1), a = f - b * (N / 2 + 1);
                    const int bn = N - a;
                    const A* rb = buf + b * PITCH;
                    S* out = spec + (size_t)(g0 + b) * M1;
                    const A za = rb[a], zb = rb[a == 0 ? 0 : bn];
                    const float h = 0.5f;
                    const A E = Cx<A>::make(h * (za.x + zb.x), h * (za.y - zb.y));
                    const A O = Cx<A>::make(h * (za.y + zb.y), -h * (za.x - zb.x));
                    out[a] = cto<S>(cadd(E, cmul(cto<A>(__ldg(&post[a])), O)));
                    if (a == 0) {
                        out[N] = cto<S>(cadd(E, cmul(cto<A>(__ldg(&post[N])), O)));
                    } else if (bn != a) {
                        const A E2 = Cx<A>::make(h * (zb.x + za.x), h * (zb.y - za.y));
                        const A O2 = Cx<A>::make(h * (zb.y + za.y), -h * (zb.x - za.x));
                        out[bn] = cto<S>(cadd(E2, cmul(cto<A>(__ldg(&post[bn])), O2)));
                    }
                }
                ff::group_sync<1, P>();  // every consumer has read the stage
                if (tid == 0) tma::mbar_arrive(&empty[s]);
            } else {
            for (int f = tid; f < B * (N / 2 + 1); f += P) {
                const int a = f / B, b = f - a * B;
                const int bn = N - a;
                A* rb = buf + b * PITCH;
                const double2 za = rb[a], zb = rb[a == 0 ? 0 : bn];
                const double2 E = make_double2(0.5 * (za.x + zb.x), 0.5 * (za.y - zb.y));
                const double2 O = make_double2(0.5 * (za.y + zb.y), -0.5 * (za.x - zb.x));
                const double2 xa = cadd(E, cmul(__ldg(&post[a]), O));
                if (a == 0) {
                    rb[0] = xa;
                    rb[N] = cadd(E, cmul(__ldg(&post[N]), O));
                } else if (bn != a) {
                    const double2 E2 = make_double2(0.5 * (zb.x + za.x), 0.5 * (zb.y - za.y));
                    const double2 O2 = make_double2(0.5 * (zb.y + za.y), -0.5 * (zb.x - za.x));
                    rb[a] = xa;
                    rb[bn] = cadd(E2, cmul(__ldg(&post[bn]), O2));
                } else {
                    rb[a] = xa;
                }
            }
            tma::fence_async_smem();
            ff::group_sync<1, P>();
            if (tid == 0) {
                const int g0 = bt * B, nv = min(B, nrows - g0);
                for (int b = 0; b < nv; b++)
                    tma::bulk_store(reinterpret_cast<double2*>(spec) + (size_t)(g0 + b) * M1, buf + b * PITCH,
                                    M1 * (unsigned)sizeof(double2));
                tma::bulk_commit();
                tma::bulk_wait_read0();  // the stores have read the stage
                tma::mbar_arrive(&empty[s]);
            }
            }
        }
        if (tid == 0) tma::bulk_wait0();
    }
    __syncthreads();
    if (tid == 0 && (bad_c | bad_p)) atomicOr(err, 4u);
    double v[1] = {dm};
    block_max_store<1>(v, part + blockIdx.x);
    if (!last_block_arrive(counter, gridDim.x)) return;
    double tot[1];
    reduce_records<1, true>(part, (int)gridDim.x, tot);
    if (tid == 0) *out_max = tot[0];
}

#define XT_SIZES(X) X(8) X(12) X(16) X(24) X(32) X(40) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) \
    X(768) X(1024) X(1152) X(1536)

template <int N>
int xt_grid(int nrows, int nsm) {
    const int nb = (nrows + XT<N>::B - 1) / XT<N>::B;
    const int per_sm = (int)((220 * 1024) / (XT<N>::smem + 1024));
    int grid = (per_sm > 0 ? per_sm : 1) * nsm;
    return grid < nb ? grid : nb;
}

}  // namespace

bool xt_tma_supported(int n) {
    switch (n) {
#define X_CASE(n) case n:
        XT_SIZES(X_CASE)
#undef X_CASE
        return true;
        default: return false;
    }
}

void xt_tma_init() {
#define X_CASE(n)                                                                                              \
    cudaFuncSetAttribute(k_xb_tma<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XT<n>::smem);          \
    cudaFuncSetAttribute(k_xb_tma32<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XT<n>::smem);        \
    cudaFuncSetAttribute(k_xf_tma<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XT<n>::smem);       \
    cudaFuncSetAttribute(k_xb_tma_gather<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XT<n>::smem);\
    cudaFuncSetAttribute(k_xf_tma_scatter<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XT<n>::smem);\
    cudaFuncSetAttribute(k_xf_div<n, double, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                         (int)XD<n>::smem);                                                                    \
    cudaFuncSetAttribute(k_xf_div<n, float, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XD<n>::smem);
    XT_SIZES(X_CASE)
#undef X_CASE
}

void launch_xb_tma(cudaStream_t st, int nx, int ny, int nz, const double2* spec, double* phi, const double2* twx,
                   const double2* post, double scale, int padded, int nsm, unsigned int* err) {
    const int nrows = ny * nz;
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xb_tma<n>, dim3(xt_grid<n>(nrows, nsm)), dim3(XT<n>::P), XT<n>::smem, st, nrows, ny, spec, \
                   phi, twx, post, scale, padded, err);                                                        \
        break;
        XT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

void launch_xb_tma(cudaStream_t st, int nx, int ny, int nz, const float2* spec, float* phi, const double2* twx,
                   const double2* post, double scale, int padded, int nsm, unsigned int* err) {
    const int nrows = ny * nz;
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xb_tma32<n>, dim3(xt_grid<n>(nrows, nsm)), dim3(XT<n>::P), XT<n>::smem, st, nrows, ny,   \
                   spec, phi, twx, post, scale, padded, err);                                                  \
        break;
        XT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

void launch_xb_tma_gather(cudaStream_t st, int nx, int ny, int nz, const XtGather& gt, double* phi, const double2* twx,
                          const double2* post, double scale, int nsm, unsigned int* err) {
    const int nrows = ny * nz;
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xb_tma_gather<n>, dim3(xt_grid<n>(nrows, nsm)), dim3(XT<n>::P), XT<n>::smem, st, nrows, ny, \
                   gt, phi, twx, post, scale, err);                                                            \
        break;
        XT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

void launch_xf_tma_scatter(cudaStream_t st, int nx, int ny, int nz, const double* src, const XtGather& gt,
                           const double2* twx, const double2* post, int nsm, unsigned int* err) {
    const int nrows = ny * nz;
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xf_tma_scatter<n>, dim3(xt_grid<n>(nrows, nsm)), dim3(XT<n>::P), XT<n>::smem, st, nrows,   \
                   ny, src, gt, twx, post, err);                                                               \
        break;
        XT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

void launch_xf_tma(cudaStream_t st, int nx, int ny, int nz, const double* src, double2* spec, const double2* twx,
                   const double2* post, int nsm, unsigned int* err) {
    const int nrows = ny * nz;
    switch (nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xf_tma<n>, dim3(xt_grid<n>(nrows, nsm)), dim3(XT<n>::P), XT<n>::smem, st, nrows, src, spec, \
                   twx, post, err);                                                                            \
        break;
        XT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}

// one CTA per SM (the producers' loads and the consumers' transforms share
// it), at most one batch per CTA
int xf_div_grid(int n, int nrows, int nsm) {
    int b = 1;
    switch (n) {
#define X_CASE(n) case n: b = XD<n>::B; break;
        XT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
    const int nb = (nrows + b - 1) / b;
    return nb < nsm ? nb : nsm;
}

template <class V, class S>
static void xf_div_t(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                     const FieldSet<V>& f, S* spec, const double2* twx, const double2* post, double* part,
                     unsigned int* counter, double* out_max, unsigned int* err) {
    const int nrows = c.ny * c.nz;
    const int grid = xf_div_grid(c.nx / 2, nrows, c.nsm > 0 ? c.nsm : 148);
    switch (c.nx / 2) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        launch_pdl(k_xf_div<n, V, S>, dim3(grid), dim3(XD<n>::NT), XD<n>::smem, st, mode, c, m, coef, f.ux, f.uy, \
                   f.uz, spec, twx, post, part, counter, out_max, err);                                        \
        break;
        XT_SIZES(X_CASE)
#undef X_CASE
        default: break;
    }
}
void launch_xf_div(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f,
                   double2* spec, const double2* twx, const double2* post, double* part, unsigned int* counter,
                   double* out_max, unsigned int* err) {
    xf_div_t(st, mode, c, m, coef, f, spec, twx, post, part, counter, out_max, err);
}
void launch_xf_div(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                   const Fields32& f, float2* spec, const double2* twx, const double2* post, double* part,
                   unsigned int* counter, double* out_max, unsigned int* err) {
    xf_div_t(st, mode, c, m, coef, f, spec, twx, post, part, counter, out_max, err);
}

}  // namespace ptc
