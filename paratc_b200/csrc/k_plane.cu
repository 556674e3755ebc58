// k_plane.cu -- the 2-D transforms of one y-plane of the Poisson solve in
// one CTA, for planes that fit shared memory.
//
// clcPPE (src/m_Poisson.f90:352-452) transforms the source along x and then
// along z.  When the (nx/2+1) x nz complex plane of one wall-normal row fits
// a CTA (C1: 65 x 128 x 16 B = 133 KB), one CTA per row does both transforms
// of that row between a single load and a single store: the forward kernel
// computes the source (the divergence of u*, clcPrSrc src/m_TScheme.f90:48-77,
// or a given array), the nx/2-point FFTs of the nz packed rows, their split
// into nx/2+1 modes and the nz-point FFTs of the nx/2+1 mode columns; the
// inverse kernel does the reverse and writes phi with its Neumann ghost rows.
// Both transforms run on the compile-time-length Stockham engine
// (fft_fixed.cuh) with radices of at most 8, on the plane stored as
// buf[kx*PITCH + k] (PITCH = nz + 1, odd): the x transform sees nz sequences
// of element stride PITCH, the z transform nx/2+1 sequences of element stride
// 1, and consecutive lanes always touch addresses PITCH or 1 apart.
#include "common.cuh"
#include "fft_fixed.cuh"
#include "kernels.cuh"
#include "reduce.cuh"

namespace ptc {
namespace {

constexpr int PL_P = 512;     // threads per plane CTA
constexpr int PL_BITS = 3;    // radix <= 8: register-held butterflies per thread stay small

__device__ __forceinline__ void cpa16p(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}

// largest number of complex values a thread holds in one pass of a
// length-N transform over B sequences
__host__ __device__ constexpr int max_regs_cplx(int N, int B) {
    const ff::Sched s = ff::make_sched(N, PL_BITS);
    int m = 0;
    for (int q = 0; q < s.np; q++) {
        const int tot = B * (N / s.r[q]);
        const int v = ((tot + PL_P - 1) / PL_P) * s.r[q];
        m = v > m ? v : m;
    }
    return m;
}

template <int M, int NZ>
struct PK {
    static constexpr int M1 = M + 1, PITCH = NZ + 1;
    static constexpr size_t smem = ((size_t)M1 * PITCH + M + M1 + NZ) * sizeof(double2);
    static constexpr bool fits = smem <= 200 * 1024 && max_regs_cplx(M, NZ) <= 24 && max_regs_cplx(NZ, M1) <= 24;
};

template <int M, int NZ>
__device__ __forceinline__ void load_tw(double2* tx, double2* tp, double2* tz, const double2* __restrict__ twx,
                                        const double2* __restrict__ post, const double2* __restrict__ twz, int tid) {
    for (int t = tid; t < M; t += PL_P) tx[t] = twx[t];
    for (int t = tid; t < M + 1; t += PL_P) tp[t] = post[t];
    for (int t = tid; t < NZ; t += PL_P) tz[t] = twz[t];
}

// MODE 0: source = divergence of u* / pmAlpha (clcPrSrc) with max|div| to
// out_max; 1: the divergence unscaled; 2: the compact source array src
// V: storage of the velocity, S: of the spectrum (the given source of mode 2
// is FP64); the transforms compute in double either way
template <int M, int NZ, class V, class S>
__global__ void __launch_bounds__(PL_P, 1)
    k_plane_f(int mode, DConst c, DMetric m, const DCoef* __restrict__ coef, const V* __restrict__ ux,
              const V* __restrict__ uy, const V* __restrict__ uz, const double* __restrict__ src,
              S* __restrict__ spec, const double2* __restrict__ twx, const double2* __restrict__ post,
              const double2* __restrict__ twz, double* __restrict__ part, unsigned int* __restrict__ counter,
              double* __restrict__ out_max) {
    constexpr int M1 = PK<M, NZ>::M1, PITCH = PK<M, NZ>::PITCH;
    constexpr ff::Sched SX = ff::make_sched(M, PL_BITS), SZ = ff::make_sched(NZ, PL_BITS);
    extern __shared__ double2 smp[];
    double2* buf = smp;
    double2* tx = smp + (size_t)M1 * PITCH;
    double2* tp = tx + M;
    double2* tz = tp + M1;
    const int tid = threadIdx.x;
    const int nx = 2 * M, ny = c.ny;
    const int j = blockIdx.x, jc = j + 1;
    load_tw<M, NZ>(tx, tp, tz, twx, post, twz, tid);
    pdl_wait();
    pdl_trigger();
    double dm = 0.0;
    if (mode == 2) {
        for (int f = tid; f < NZ * M; f += PL_P) {
            const int k = f / M, e = f - k * M;
            cpa16p(&buf[e * PITCH + k], src + ((size_t)k * ny + j) * nx + 2 * e);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    } else {
        const double sudtal = (mode == 0) ? 1.0 / coef->pmAlpha : 1.0;
        const size_t pl = (size_t)c.nyt * nx, r0 = (size_t)jc * nx;
        const double rdyp = __ldg(&m.rdyp[jc]);
#pragma unroll 2
        for (int f = tid; f < NZ * M; f += PL_P) {
            const int k = f / M, e = f - k * M;
            const int km = k == 0 ? NZ - 1 : k - 1, kp = k == NZ - 1 ? 0 : k + 1, ku = kp == NZ - 1 ? 0 : kp + 1;
            const int i0 = 2 * e, im = i0 == 0 ? nx - 1 : i0 - 1, i2 = i0 + 2 == nx ? 0 : i0 + 2;
            const V* ur = ux + (size_t)k * pl + r0;
            const V* vr = uy + (size_t)k * pl + r0;
            const double2 u01 = ld_pair(ur + i0);
            const double2 u23 = ld_pair(ur + i2);
            const double um = (double)__ldg(ur + im);
            const double2 v0 = ld_pair(vr + i0);
            const double2 v1 = ld_pair(vr + nx + i0);
            const double2 w0 = ld_pair(uz + (size_t)km * pl + r0 + i0);
            const double2 w1 = ld_pair(uz + (size_t)k * pl + r0 + i0);
            const double2 w2 = ld_pair(uz + (size_t)kp * pl + r0 + i0);
            const double2 w3 = ld_pair(uz + (size_t)ku * pl + r0 + i0);
            const double dudx0 = c.dxC[0] * um + c.dxC[1] * u01.x + c.dxC[2] * u01.y + c.dxC[3] * u23.x;
            const double dudx1 = c.dxC[0] * u01.x + c.dxC[1] * u01.y + c.dxC[2] * u23.x + c.dxC[3] * u23.y;
            const double dvdy0 = (v1.x - v0.x) * rdyp, dvdy1 = (v1.y - v0.y) * rdyp;
            const double dwdz0 = c.dzC[0] * w0.x + c.dzC[1] * w1.x + c.dzC[2] * w2.x + c.dzC[3] * w3.x;
            const double dwdz1 = c.dzC[0] * w0.y + c.dzC[1] * w1.y + c.dzC[2] * w2.y + c.dzC[3] * w3.y;
            const double d0 = dudx0 + dvdy0 + dwdz0, d1 = dudx1 + dvdy1 + dwdz1;
            dm = nmax(dm, nmax(fabs(d0), fabs(d1)));
            buf[e * PITCH + k] = make_double2(sudtal * d0, sudtal * d1);
        }
    }
    __syncthreads();
    // x: M-point transforms of the NZ packed rows
    ff::smem_passes<M, NZ, PITCH, PL_P, -1, 0, SX.np, PL_BITS, false>(buf, tx, tid);
    // split every row into the M+1 modes of the real transform (pairs a, M-a)
    for (int f = tid; f < NZ * (M / 2 + 1); f += PL_P) {
        const int a = f / NZ, k = f - a * NZ;
        const int b = M - a;
        const double2 za = buf[a * PITCH + k], zb = buf[(a == 0 ? 0 : b) * PITCH + k];
        // X[a] from Z[a], Z[M-a]; X[b] from Z[b], Z[M-b] = Z[a] (b = M: Z[0], Z[0])
        const double2 Ea = make_double2(0.5 * (za.x + zb.x), 0.5 * (za.y - zb.y));
        const double2 Oa = make_double2(0.5 * (za.y + zb.y), -0.5 * (za.x - zb.x));
        const double2 Xa = cadd(Ea, cmul(tp[a], Oa));
        const double2 Eb = make_double2(0.5 * (zb.x + za.x), 0.5 * (zb.y - za.y));
        const double2 Ob = make_double2(0.5 * (zb.y + za.y), -0.5 * (zb.x - za.x));
        const double2 Xb = cadd(Eb, cmul(tp[b], Ob));
        buf[a * PITCH + k] = Xa;
        if (b != a) buf[b * PITCH + k] = Xb;
    }
    __syncthreads();
    // z: NZ-point transforms of the M+1 mode columns
    ff::smem_passes<NZ, M1, PITCH, PL_P, -1, 0, SZ.np, PL_BITS, true>(buf, tz, tid);
    for (int f = tid; f < M1 * NZ; f += PL_P) {
        const int k = f / M1, kx = f - k * M1;
        st_c(spec + ((size_t)k * ny + j) * M1 + kx, buf[kx * PITCH + k]);
    }
    if (mode == 2) return;
    double v[1] = {dm};
    const unsigned int nblocks = gridDim.x;
    block_max_store<1>(v, part + blockIdx.x);
    if (!last_block_arrive(counter, nblocks)) return;
    double tot[1];
    reduce_records<1, true>(part, (int)nblocks, tot);
    if (tid == 0) *out_max = tot[0];
}

// S: storage of the spectrum, PH: of the potential; accumulate != 0 adds the
// result to phi (unpadded rows: the corrections of the refined solve)
template <int M, int NZ, class S, class PH>
__global__ void __launch_bounds__(PL_P, 1)
    k_plane_b(int ny, const S* __restrict__ spec, PH* __restrict__ phi, const double2* __restrict__ twx,
              const double2* __restrict__ post, const double2* __restrict__ twz, double scale, int padded,
              int accumulate, const double* __restrict__ shift) {
    constexpr int M1 = PK<M, NZ>::M1, PITCH = PK<M, NZ>::PITCH;
    constexpr ff::Sched SX = ff::make_sched(M, PL_BITS), SZ = ff::make_sched(NZ, PL_BITS);
    extern __shared__ double2 smp[];
    double2* buf = smp;
    double2* tx = smp + (size_t)M1 * PITCH;
    double2* tp = tx + M;
    double2* tz = tp + M1;
    const int tid = threadIdx.x;
    const int nx = 2 * M;
    const int j = blockIdx.x;
    load_tw<M, NZ>(tx, tp, tz, twx, post, twz, tid);
    pdl_wait();
    pdl_trigger();
    for (int f = tid; f < M1 * NZ; f += PL_P) {
        const int k = f / M1, kx = f - k * M1;
        if constexpr (sizeof(S) == sizeof(double2)) cpa16p(&buf[kx * PITCH + k], spec + ((size_t)k * ny + j) * M1 + kx);
        else buf[kx * PITCH + k] = ld_c(spec + ((size_t)k * ny + j) * M1 + kx);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    ff::smem_passes<NZ, M1, PITCH, PL_P, 1, 0, SZ.np, PL_BITS, true>(buf, tz, tid);
    // merge modes a and M-a of every row (the DC and Nyquist coefficients are real)
    for (int f = tid; f < NZ * (M / 2 + 1); f += PL_P) {
        const int a = f / NZ, k = f - a * NZ;
        const int b = M - a;
        double2 xa = buf[a * PITCH + k], xb = buf[b * PITCH + k];
        if (a == 0) { xa.y = 0.0; xb.y = 0.0; }
        const double2 e2a = make_double2(xa.x + xb.x, xa.y - xb.y);
        const double2 da = make_double2(xa.x - xb.x, xa.y + xb.y);
        const double2 o2a = cmulc(da, tp[a]);
        const double2 za = make_double2(e2a.x - o2a.y, e2a.y + o2a.x);
        if (a == 0) {
            buf[k] = za;
        } else {
            const double2 e2b = make_double2(xb.x + xa.x, xb.y - xa.y);
            const double2 db = make_double2(xb.x - xa.x, xb.y + xa.y);
            const double2 o2b = cmulc(db, tp[b]);
            const double2 zb = make_double2(e2b.x - o2b.y, e2b.y + o2b.x);
            buf[a * PITCH + k] = za;
            if (b != a) buf[b * PITCH + k] = zb;
        }
    }
    __syncthreads();
    ff::smem_passes<M, NZ, PITCH, PL_P, 1, 0, SX.np, PL_BITS, false>(buf, tx, tid);
    const int nyt = ny + 2;
    for (int f = tid; f < NZ * M; f += PL_P) {
        const int k = f / M, e = f - k * M;
        const double2 z = buf[e * PITCH + k];
        double2 v = make_double2(z.x * scale, z.y * scale);
        if (!padded) {
            PH* dst = phi + ((size_t)k * ny + j) * nx + 2 * e;
            if (accumulate) {
                // phi += correction - the row-1 plane mean of phi (the gauge)
                const double2 o = ld_pair(dst);
                const double sh = shift ? *shift : 0.0;
                v = make_double2(o.x + v.x - sh, o.y + v.y - sh);
            }
            st_pair(dst, v);
            continue;
        }
        PH* rowp = phi + ((size_t)k * nyt + (j + 1)) * nx + 2 * e;
        st_pair(rowp, v);
        if (j == 0) st_pair(rowp - nx, v);
        if (j == ny - 1) st_pair(rowp + nx, v);
    }
}

#define PLANE_PAIRS(X)                                                                                        \
    X(32, 32) X(32, 48) X(32, 64) X(32, 96) X(32, 128) X(48, 48) X(48, 64) X(48, 96) X(48, 128) X(64, 48)     \
    X(64, 64) X(64, 96) X(64, 128) X(96, 64) X(96, 96)

}  // namespace

#ifndef PTC_STORE32
// FP64 instantiations; the FP32 storage forms are compiled in k_plane32.cu
bool plane_supported(int nx, int nz) {
#define P_CASE(a, b) \
    if (nx / 2 == a && nz == b) return PK<a, b>::fits;
    PLANE_PAIRS(P_CASE)
#undef P_CASE
    return false;
}
#define PF_TYPES(X, a, b) X(a, b, double, double2)
#define PB_TYPES(X, a, b) X(a, b, double2, double)
void plane_init() {
    plane_init32();
#else
#define PF_TYPES(X, a, b) X(a, b, float, float2) X(a, b, double, float2)
#define PB_TYPES(X, a, b) X(a, b, float2, float) X(a, b, float2, double)
void plane_init32() {
#endif
#define PF_ATTR(a, b, V, S) \
    cudaFuncSetAttribute(k_plane_f<a, b, V, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PK<a, b>::smem);
#define PB_ATTR(a, b, S, PH) \
    cudaFuncSetAttribute(k_plane_b<a, b, S, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PK<a, b>::smem);
#define P_CASE(a, b)                       \
    if constexpr (PK<a, b>::fits) {        \
        PF_TYPES(PF_ATTR, a, b)            \
        PB_TYPES(PB_ATTR, a, b)            \
    }
    PLANE_PAIRS(P_CASE)
#undef P_CASE
#undef PF_ATTR
#undef PB_ATTR
}

template <class V, class S>
static void plane_f_t(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                      const FieldSet<V>& f, const double* src, S* spec, const double2* twx, const double2* post,
                      const double2* twz, double* part, unsigned int* counter, double* out_max) {
#define P_CASE(a, b)                                                                                           \
    if constexpr (PK<a, b>::fits) {                                                                            \
        if (c.nx / 2 == a && c.nz == b) {                                                                      \
            launch_pdl(k_plane_f<a, b, V, S>, dim3(c.ny), dim3(PL_P), PK<a, b>::smem, st, mode, c, m, coef, f.ux, \
                       f.uy, f.uz, src, spec, twx, post, twz, part, counter, out_max);                         \
            return;                                                                                            \
        }                                                                                                      \
    }
    PLANE_PAIRS(P_CASE)
#undef P_CASE
}

template <class S, class PH>
static void plane_b_t(cudaStream_t st, int nx, int ny, int nz, const S* spec, PH* phi, const double2* twx,
                      const double2* post, const double2* twz, double scale, int padded, int accumulate,
                      const double* shift) {
#define P_CASE(a, b)                                                                                           \
    if constexpr (PK<a, b>::fits) {                                                                            \
        if (nx / 2 == a && nz == b) {                                                                          \
            launch_pdl(k_plane_b<a, b, S, PH>, dim3(ny), dim3(PL_P), PK<a, b>::smem, st, ny, spec, phi, twx, post, \
                       twz, scale, padded, accumulate, shift);                                                 \
            return;                                                                                            \
        }                                                                                                      \
    }
    PLANE_PAIRS(P_CASE)
#undef P_CASE
}

#ifndef PTC_STORE32
void launch_plane_f(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f,
                    const double* src, double2* spec, const double2* twx, const double2* post, const double2* twz,
                    double* part, unsigned int* counter, double* out_max) {
    plane_f_t(st, mode, c, m, coef, f, src, spec, twx, post, twz, part, counter, out_max);
}
void launch_plane_b(cudaStream_t st, int nx, int ny, int nz, const double2* spec, double* phi, const double2* twx,
                    const double2* post, const double2* twz, double scale, int padded) {
    plane_b_t(st, nx, ny, nz, spec, phi, twx, post, twz, scale, padded, 0, nullptr);
}
#else
void launch_plane_f(cudaStream_t st, int mode, const DConst& c, const DMetric& m, const DCoef* coef,
                    const Fields32& f, const double* src, float2* spec, const double2* twx, const double2* post,
                    const double2* twz, double* part, unsigned int* counter, double* out_max) {
    plane_f_t(st, mode, c, m, coef, f, src, spec, twx, post, twz, part, counter, out_max);
}
void launch_plane_f(cudaStream_t st, const DConst& c, const double* src, float2* spec, const double2* twx,
                    const double2* post, const double2* twz) {
    const Fields none = {};
    plane_f_t(st, 2, c, DMetric{}, nullptr, none, src, spec, twx, post, twz, nullptr, nullptr, nullptr);
}
void launch_plane_b(cudaStream_t st, int nx, int ny, int nz, const float2* spec, float* phi, const double2* twx,
                    const double2* post, const double2* twz, double scale, int padded) {
    plane_b_t(st, nx, ny, nz, spec, phi, twx, post, twz, scale, padded, 0, nullptr);
}
void launch_plane_b(cudaStream_t st, int nx, int ny, int nz, const float2* spec, double* phi, const double2* twx,
                    const double2* post, const double2* twz, double scale, int accumulate, const double* shift) {
    plane_b_t(st, nx, ny, nz, spec, phi, twx, post, twz, scale, 0, accumulate, shift);
}
#endif

}  // namespace ptc
