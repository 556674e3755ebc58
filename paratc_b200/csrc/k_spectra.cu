// k_spectra.cu -- 1-D energy spectra, cospectra and linear coherence spectra
// of clcStat (src/m_FlowCase.f90:430-806, with clcEnergySpectraX/Z,
// clcLTS_x/z_real/imag and clcCospectraX/Z at :954-1180) on B200.
//
// For every wall-normal row jc the reference transforms, along x (then along
// z), the rows of ux+uCRF, uy, uz, p, uy at the cell centre (uy_c), ux at the
// cell centre by the 4th-order interpolation (ux_c, +uCRF) and the scalar, and
// sums over the other homogeneous direction, per mode k of the real transform:
//   spectra 1-4, 9:  w_k |X_k|^2                  (ux', uy, uz, p, scalar)
//   spectrum 5:      w_k Re(X_k conj Y_k)         (ux' with uy_c)
//   spectrum 6:      w_k Re(U_k conj Y_k)         (ux_c with uy_c)
//   spectra 7, 8:    Re, Im of X_k conj R_k       (ux' with ux' on the row
//                    jForLCS, mirrored to nyc+1-jForLCS in the upper half of
//                    a channel; the imaginary part is zero at the end modes)
// with w_k = 2 except at k = 0 and k = n/2, and times 1/(n^2 n_other).  The
// end modes use only the real parts, as the reference's halfcomplex loops do.
//
// Here two real rows are packed into one complex sequence (a + i b) and
// transformed with the compile-time-length FFT engine of fft_fixed.cuh; the
// two real transforms are split off mode by mode (A_k = (Z_k + conj Z_{n-k})/2,
// B_k = (Z_k - conj Z_{n-k})/2i).  Four packed sequences per row, in the order
// (ux', ux'_ref), (uy_c, ux_c), (uy, uz), (p, scalar or 0), give every
// spectrum from one pass over the fields; the ux' modes of the batch stay in
// shared memory for the cospectrum with uy_c.  A CTA owns one row jc and a
// contiguous slice of the other direction, B sequences at a time; each thread
// owns a fixed set of modes and adds its batch sums to the CTA's FP64
// partial record in a fixed order, and a second kernel adds the slices of a
// row in index order, times the norm, to the accumulators.  Results are
// independent of scheduling.
#include <algorithm>

#include "common.cuh"
#include "fft_fixed.cuh"
#include "kernels.cuh"

namespace ptc {
namespace {

constexpr size_t SPEC_SMEM_BUDGET = 160 * 1024;

// launch shape of the length-N spectra kernel: B packed sequences per batch
// (buffer, ux' modes and twiddles within the shared-memory budget), P threads
template <int N>
struct SpK {
    static constexpr int NH = N / 2 + 1;
    static constexpr size_t bytes(int b) { return ((size_t)N * (b + 1) + (size_t)b * NH + N) * sizeof(double2); }
    static constexpr int bcalc() {
        int b = 16;
        while (b > 1 && bytes(b) > SPEC_SMEM_BUDGET) b /= 2;
        return b;
    }
    static constexpr int B = bcalc();
    static constexpr int PITCH = B + 1;
    static constexpr int RMAX = ff::sched_rmax(N);
    static constexpr int pcalc() {
        int p = B * N / RMAX;
        p = (p + 31) / 32 * 32;
        return p < 64 ? 64 : (p > 256 ? 256 : p);
    }
    static constexpr int P = pcalc();
    static constexpr size_t smem = bytes(B);
};

// one record per CTA: NSPEC spectra of NH modes
constexpr int NSPEC = 9;

struct SpecTerms {
    // real transforms of the two rows packed in sequence b at mode a
    __device__ __forceinline__ static void split(double2 zk, double2 zn, double2& fa, double2& fb) {
        fa = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y - zn.y));
        fb = make_double2(0.5 * (zk.y + zn.y), 0.5 * (zn.x - zk.x));
    }
    __device__ __forceinline__ static double energy(double2 x, bool edge) {
        return edge ? x.x * x.x : (x.x * x.x + x.y * x.y) * 2.0;
    }
    __device__ __forceinline__ static double cosp(double2 x, double2 y, bool edge) {
        return edge ? x.x * y.x : (x.x * y.x + x.y * y.y) * 2.0;
    }
};

template <int N>
__global__ void __launch_bounds__(SpK<N>::P)
    k_spec(int axis, DConst c, const double* __restrict__ ux, const double* __restrict__ uy,
           const double* __restrict__ uz, const double* __restrict__ pr, const double* __restrict__ sc, int jlcs,
           int splits, const double2* __restrict__ twN, double* __restrict__ part) {
    constexpr int B = SpK<N>::B, P = SpK<N>::P, PITCH = SpK<N>::PITCH, NH = SpK<N>::NH;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ double2 sms[];
    double2* buf = sms;                     // N * PITCH: the packed sequences
    double2* xm = sms + (size_t)N * PITCH;  // B * NH: ux' modes of the batch
    double2* tws = xm + (size_t)B * NH;     // N twiddles
    const int tid = threadIdx.x;
    const int nx = c.nx, ny = c.ny, nz = c.nz;
    const int jc = blockIdx.x + 1;
    const int s = blockIdx.y;
    const int nl = axis == 0 ? nz : nx;  // sequences of the row: z planes (x spectra) or x points (z spectra)
    const int l0 = (int)((long long)nl * s / splits), l1 = (int)((long long)nl * (s + 1) / splits);
    const int jr = (c.flow_type == 2 || jc <= ny / 2) ? jlcs : ny + 1 - jlcs;
    const size_t pl = (size_t)c.nyt * nx;
    const double I1 = c.IC[0], I2 = c.IC[1], I3 = c.IC[2], I4 = c.IC[3], ucrf = c.ucrf;
    const bool has_sc = c.scalar_on != 0;
    double* rec = part + ((size_t)blockIdx.x * splits + s) * NSPEC * NH;
    for (int t = tid; t < N; t += P) tws[t] = twN[t];
    // a thread zeroes, and later updates, only the modes a = tid + q P of every spectrum
    for (int a = tid; a < NH; a += P)
        for (int m = 0; m < NSPEC; m++) rec[m * NH + a] = 0.0;
    for (int lb = l0; lb < l1; lb += B) {
        const int nb = min(B, l1 - lb);
#pragma unroll 1
        for (int q = 0; q < 4; q++) {
            __syncthreads();  // the previous extraction has finished reading buf
            for (int f = tid; f < B * N; f += P) {
                int b, e;
                if (axis == 0) { b = f / N; e = f - b * N; }  // along x: consecutive threads, consecutive i
                else { e = f / B; b = f - e * B; }             // along z: consecutive threads, consecutive i
                double va = 0.0, vb = 0.0;
                if (b < nb) {
                    const int k = axis == 0 ? lb + b : e, i = axis == 0 ? e : lb + b;
                    const size_t o = (size_t)k * pl + (size_t)jc * nx + i;
                    if (q == 0) {
                        va = __ldg(&ux[o]) + ucrf;
                        vb = __ldg(&ux[(size_t)k * pl + (size_t)jr * nx + i]) + ucrf;
                    } else if (q == 1) {
                        const int im = i >= 1 ? i - 1 : nx - 1, ip = i + 1 < nx ? i + 1 : i + 1 - nx;
                        const int iu = i + 2 < nx ? i + 2 : i + 2 - nx;
                        const size_t r = o - i;
                        va = 0.5 * (__ldg(&uy[o]) + __ldg(&uy[o + nx]));
                        vb = I1 * __ldg(&ux[r + im]) + I2 * __ldg(&ux[o]) + I3 * __ldg(&ux[r + ip]) + I4 * __ldg(&ux[r + iu]) + ucrf;
                    } else if (q == 2) {
                        va = __ldg(&uy[o]);
                        vb = __ldg(&uz[o]);
                    } else {
                        va = __ldg(&pr[o]);
                        vb = has_sc ? __ldg(&sc[o]) : 0.0;
                    }
                }
                buf[e * PITCH + b] = make_double2(va, vb);
            }
            __syncthreads();
            ff::smem_passes<N, B, PITCH, P, -1, 0, SC.np>(buf, tws, tid);
            // each thread: its modes a, the batch's sequences in order
            for (int a = tid; a < NH; a += P) {
                const int an = a == 0 ? 0 : N - a;
                const bool edge = (a == 0) || (a == N / 2);
                double t0 = 0.0, t1 = 0.0, t2 = 0.0;
                for (int b = 0; b < nb; b++) {
                    double2 fa, fb;
                    SpecTerms::split(buf[a * PITCH + b], buf[an * PITCH + b], fa, fb);
                    if (q == 0) {
                        xm[b * NH + a] = fa;
                        t0 += SpecTerms::energy(fa, edge);
                        t1 += edge ? fa.x * fb.x : fa.x * fb.x + fa.y * fb.y;
                        t2 += edge ? 0.0 : fa.y * fb.x - fa.x * fb.y;
                    } else if (q == 1) {
                        t0 += SpecTerms::cosp(xm[b * NH + a], fa, edge);
                        t1 += SpecTerms::cosp(fb, fa, edge);
                    } else {
                        t0 += SpecTerms::energy(fa, edge);
                        t1 += SpecTerms::energy(fb, edge);
                    }
                }
                if (q == 0) {
                    rec[0 * NH + a] += t0;
                    rec[6 * NH + a] += t1;
                    rec[7 * NH + a] += t2;
                } else if (q == 1) {
                    rec[4 * NH + a] += t0;
                    rec[5 * NH + a] += t1;
                } else if (q == 2) {
                    rec[1 * NH + a] += t0;
                    rec[2 * NH + a] += t1;
                } else {
                    rec[3 * NH + a] += t0;
                    rec[8 * NH + a] += t1;
                }
            }
        }
    }
}

// out[(m*ny + jc-1)*nh + a] += (sum over the row's slices, in order) * norm
__global__ void k_spec_final(int ny, int nh, int nsp, int splits, double norm, const double* __restrict__ part,
                             double* __restrict__ out) {
    const int jr = blockIdx.x, m = blockIdx.y;
    if (m >= nsp) return;
    for (int a = threadIdx.x; a < nh; a += blockDim.x) {
        double t = 0.0;
        for (int s = 0; s < splits; s++) t += part[(((size_t)jr * splits + s) * NSPEC + m) * nh + a];
        out[((size_t)m * ny + jr) * nh + a] += t * norm;
    }
}

// ---------------------------------------------------------------------------
// 2-D spectra (clcEnergySpectra2D / clcCosSpectra2D, src/m_FlowCase.f90:
// 1186-1375): R2HC along x, then R2HC along z, of whole x-z rows of the
// fields, in FFTW's halfcomplex order (r_0..r_{n/2}, then i_k at n-k), two
// real sequences packed per complex FFT.  Mode 0 transforms the x rows of
// the listed (field, row) pairs fj[q] into S[(q*nz + k)*nx + a]; mode 1
// transforms the columns of S along z in place (a CTA reads all its columns
// before it writes them).  Fields: 0 ux, 1 uy, 2 uz, 3 p, 4 ux at the cell
// centre + uCRF, 5 uy at the cell centre, 6 the scalar.
template <int N>
__global__ void __launch_bounds__(SpK<N>::P)
    k_hc(int mode, DConst c, const double* __restrict__ ux, const double* __restrict__ uy,
         const double* __restrict__ uz, const double* __restrict__ pr, const double* __restrict__ sc,
         const int2* __restrict__ fj, int nseq, const double2* __restrict__ twN, double* S) {
    constexpr int B = SpK<N>::B, P = SpK<N>::P, PITCH = SpK<N>::PITCH;
    constexpr ff::Sched SC = ff::make_sched(N);
    extern __shared__ double2 sms[];
    double2* buf = sms;
    double* bufd = reinterpret_cast<double*>(sms);
    double2* tws = sms + (size_t)N * PITCH;
    const int tid = threadIdx.x;
    const int nx = c.nx, nz = c.nz;
    const size_t pl = (size_t)c.nyt * nx;
    const double I1 = c.IC[0], I2 = c.IC[1], I3 = c.IC[2], I4 = c.IC[3], ucrf = c.ucrf;
    const int s0 = blockIdx.x * 2 * B;
    for (int t = tid; t < N; t += P) tws[t] = twN[t];
    // real sequence r of the CTA (0..2B-1) is the real (r even) or imaginary
    // part of complex sequence r/2; mode 0 reads along rows, mode 1 across
    // columns (consecutive threads, consecutive sequences)
    for (int f = tid; f < 2 * B * N; f += P) {
        int r, e;
        if (mode == 0) { r = f / N; e = f - r * N; }
        else { e = f / (2 * B); r = f - e * 2 * B; }
        const int s = s0 + r;
        double v = 0.0;
        if (s < nseq) {
            if (mode == 0) {
                const int q = s / nz, k = s - q * nz;
                const int2 d = fj[q];
                const int i = e;
                const size_t rw = (size_t)k * pl + (size_t)d.y * nx, o = rw + i;
                switch (d.x) {
                    case 0: v = __ldg(&ux[o]); break;
                    case 1: v = __ldg(&uy[o]); break;
                    case 2: v = __ldg(&uz[o]); break;
                    case 3: v = __ldg(&pr[o]); break;
                    case 4: {
                        const int im = i >= 1 ? i - 1 : nx - 1, ip = i + 1 < nx ? i + 1 : i + 1 - nx;
                        const int iu = i + 2 < nx ? i + 2 : i + 2 - nx;
                        v = I1 * __ldg(&ux[rw + im]) + I2 * __ldg(&ux[o]) + I3 * __ldg(&ux[rw + ip]) + I4 * __ldg(&ux[rw + iu]) + ucrf;
                        break;
                    }
                    case 5: v = 0.5 * (__ldg(&uy[o]) + __ldg(&uy[o + nx])); break;
                    default: v = __ldg(&sc[o]); break;
                }
            } else {
                const int q = s / nx, a = s - q * nx;
                v = S[((size_t)q * nz + e) * nx + a];
            }
        }
        bufd[2 * (e * PITCH + (r >> 1)) + (r & 1)] = v;
    }
    __syncthreads();
    ff::smem_passes<N, B, PITCH, P, -1, 0, SC.np>(buf, tws, tid);
    for (int f = tid; f < 2 * B * N; f += P) {
        int r, a;
        if (mode == 0) { r = f / N; a = f - r * N; }
        else { a = f / (2 * B); r = f - a * 2 * B; }
        const int s = s0 + r;
        if (s >= nseq) continue;
        const int b = r >> 1;
        double v;
        if (a <= N / 2) {  // Re of mode a
            const double2 za = buf[a * PITCH + b], zn = buf[(a == 0 ? 0 : N - a) * PITCH + b];
            v = (r & 1) == 0 ? 0.5 * (za.x + zn.x) : 0.5 * (za.y + zn.y);
        } else {  // Im of mode N - a
            const double2 zk = buf[(N - a) * PITCH + b], za = buf[a * PITCH + b];
            v = (r & 1) == 0 ? 0.5 * (zk.y - za.y) : 0.5 * (za.x - zk.x);
        }
        if (mode == 0) {
            const int q = s / nz, k = s - q * nz;
            S[((size_t)q * nz + k) * nx + a] = v;
        } else {
            const int q = s / nx, col = s - q * nx;
            S[((size_t)q * nz + a) * nx + col] = v;
        }
    }
}

// EnergySpec2D(ic, q, kc, m) += normEgy * (H^2 [+ H_mirror^2]) for m = ux, uy,
// uz, p [, scalar]; the cospectrum m = 5 takes H_uxc H_uyc [- the mirrored
// product].  fj of (row q, field f, mirror h) = (q*nfld + f)*nmir + h.
__global__ void k_spec2d_acc(int nx, int nz, int nsel, int nsp, int nmir, int nfld, double norm,
                             const double* __restrict__ S, double* __restrict__ out) {
    const size_t tot = (size_t)nsp * nz * nsel * nx;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x) {
        const int ic = (int)(t % nx);
        size_t r = t / nx;
        const int q = (int)(r % nsel);
        r /= nsel;
        const int kc = (int)(r % nz);
        const int m = (int)(r / nz);
        const size_t e = (size_t)kc * nx + ic, pl = (size_t)nx * nz;
        const double* Sq = S + (size_t)q * nfld * nmir * pl;
        double v;
        if (m == 4) {
            const double rt1 = Sq[(4 * nmir) * pl + e] * Sq[(5 * nmir) * pl + e];
            if (nmir == 1) v = norm * rt1;
            else v = norm * (rt1 + (-1.0) * (Sq[(4 * nmir + 1) * pl + e] * Sq[(5 * nmir + 1) * pl + e]));
        } else {
            const int f = m < 4 ? m : 6;
            const double rt1 = Sq[(f * nmir) * pl + e];
            if (nmir == 1) v = norm * rt1 * rt1;
            else {
                const double rt2 = Sq[(f * nmir + 1) * pl + e];
                v = norm * (rt1 * rt1 + rt2 * rt2);
            }
        }
        out[t] += v;
    }
}

#define SPEC_SIZES(X) X(8) X(12) X(16) X(24) X(30) X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(192) X(256) \
    X(384) X(512) X(768) X(1024) X(1152) X(1536) X(2048) X(2304) X(3072)

int spec_batch(int n) {
    switch (n) {
#define X_CASE(n) case n: return SpK<n>::B;
        SPEC_SIZES(X_CASE)
#undef X_CASE
        default: return 0;
    }
}

}  // namespace

bool spectra_supported(int n) { return spec_batch(n) > 0; }

int spectra_count(const DConst& c) { return c.scalar_on ? 9 : 8; }

int spectra_splits(const DConst& c, int axis) {
    const int n = axis == 0 ? c.nx : c.nz, nl = axis == 0 ? c.nz : c.nx;
    const int b = spec_batch(n);
    if (b <= 0) return 1;
    int s = (2 * (c.nsm > 0 ? c.nsm : 148) + c.ny - 1) / c.ny;
    const int nbatch = (nl + b - 1) / b;
    if (s > nbatch) s = nbatch;
    return s < 1 ? 1 : s;
}

size_t spectra_part_doubles(const DConst& c) {
    size_t a = (size_t)c.ny * spectra_splits(c, 0) * NSPEC * (c.nx / 2 + 1);
    size_t b = (size_t)c.ny * spectra_splits(c, 1) * NSPEC * (c.nz / 2 + 1);
    return a > b ? a : b;
}

void spectra_init() {
#define X_CASE(n)                                                                                              \
    cudaFuncSetAttribute(k_spec<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SpK<n>::smem);           \
    cudaFuncSetAttribute(k_hc<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SpK<n>::smem);
    SPEC_SIZES(X_CASE)
#undef X_CASE
}

// axis 0: spectra along x (tw: exp(-2 pi i m / nx), out [nsp][ny][nx/2+1]);
// axis 1: along z (tw for nz, out [nsp][ny][nz/2+1])
void launch_spectra(cudaStream_t st, int axis, const DConst& c, const Fields& f, int jlcs, const double2* tw,
                    double* part, double* out) {
    const int n = axis == 0 ? c.nx : c.nz;
    const int splits = spectra_splits(c, axis);
    const dim3 grid(c.ny, splits);
    switch (n) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        k_spec<n><<<grid, SpK<n>::P, SpK<n>::smem, st>>>(axis, c, f.ux, f.uy, f.uz, f.pr, f.sc, jlcs, splits, tw, \
                                                          part);                                               \
        break;
        SPEC_SIZES(X_CASE)
#undef X_CASE
        default: return;
    }
    const double norm = axis == 0 ? 1.0 / ((double)c.nx * (double)c.nx * (double)c.nz)
                                  : 1.0 / ((double)c.nx * (double)c.nz * (double)c.nz);
    const int nsp = spectra_count(c);
    k_spec_final<<<dim3(c.ny, nsp), 128, 0, st>>>(c.ny, n / 2 + 1, nsp, splits, norm, part, out);
}

// 2-D spectra of the nfj (field, row) pairs fj: hc-hc transforms into S
// (nfj*nx*nz doubles), then the accumulation into out
// [nsp][nz][nsel][nx]; twx / twz: exp(-2 pi i m / n) for n = nx, nz
void launch_spectra2d(cudaStream_t st, const DConst& c, const Fields& f, const int2* fj, int nfj, int nsel, int nmir,
                      int nfld, const double2* twx, const double2* twz, double* S, double* out) {
    for (int mode = 0; mode < 2; mode++) {
        const int n = mode == 0 ? c.nx : c.nz;
        const int nseq = nfj * (mode == 0 ? c.nz : c.nx);
        const double2* tw = mode == 0 ? twx : twz;
        switch (n) {
#define X_CASE(n)                                                                                              \
    case n:                                                                                                    \
        k_hc<n><<<(nseq + 2 * SpK<n>::B - 1) / (2 * SpK<n>::B), SpK<n>::P, SpK<n>::smem, st>>>(                \
            mode, c, f.ux, f.uy, f.uz, f.pr, f.sc, fj, nseq, tw, S);                                          \
        break;
            SPEC_SIZES(X_CASE)
#undef X_CASE
            default: return;
        }
    }
    double norm = 1.0 / ((double)c.nx * (double)c.nz);
    norm = norm * norm;
    if (c.flow_type == 1) norm = norm * 0.5;
    const int nsp = c.scalar_on ? 6 : 5;
    const size_t tot = (size_t)nsp * c.nz * nsel * c.nx;
    const int blocks = (int)std::min<size_t>((tot + 255) / 256, (size_t)8 * (c.nsm > 0 ? c.nsm : 148));
    k_spec2d_acc<<<blocks, 256, 0, st>>>(c.nx, c.nz, nsel, nsp, nmir, nfld, norm, S, out);
}

}  // namespace ptc
