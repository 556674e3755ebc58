// k_plane.cu -- the 2-D FFT of one y-plane of the Poisson solve in one CTA.
//
// clcPPE (src/m_Poisson.f90:352-452) transforms the source along x and then
// along z, one y-plane at a time in effect.  When a whole complex plane of
// (nx/2+1) x nz values fits in shared memory (133 KB at 128 x 128), one CTA
// owns one plane: it loads it once, transforms it in place and writes it once,
// instead of two HBM round trips through separate x and z kernels.
//
// Forward kernel: the source is either the divergence of u* computed on the fly
// (clcPrSrc, src/m_TScheme.f90:48-77, with its max|div| reduced across the
// grid by the last CTA) or a given source array; then the nx/2-point complex
// FFT of every even/odd packed row and its split into nx/2+1 modes, then the
// nz-point FFT of every mode column.  Inverse kernel: the z inverse, the merge
// of every row into nx/2 complex values, the x inverse, 1/(nx*nz) and the
// Neumann ghost rows of phi (SetBC_and_UpdateHalo_pr).
//
// The transforms are Stockham passes done in place: every thread loads the
// inputs of its butterflies into registers, the block synchronises, and the
// outputs are written over the same buffer.  Twiddles live in shared memory.
#include "common.cuh"
#include "kernels.cuh"
#include "reduce.cuh"

namespace ptc {
namespace {

constexpr int PT = 512;    // threads per plane CTA
constexpr int MAXE = 5;    // complex values a thread holds in one pass (no spill at 512 threads)

template <int DIR>
__device__ __forceinline__ void dft2p(double2 (&v)[2]) {
    const double2 t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
}
template <int DIR>
__device__ __forceinline__ void dft3p(double2 (&v)[3]) {
    const double c = -0.5, s = DIR * 0.86602540378443864676;
    const double2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    const double2 mm = make_double2(v[0].x + c * t1.x, v[0].y + c * t1.y);
    const double2 it = make_double2(-s * t2.y, s * t2.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(mm, it);
    v[2] = csub(mm, it);
}
template <int DIR>
__device__ __forceinline__ void dft4p(double2 (&v)[4]) {
    const double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const double2 t2 = cadd(v[1], v[3]);
    double2 t3 = csub(v[1], v[3]);
    t3 = (DIR < 0) ? make_double2(t3.y, -t3.x) : make_double2(-t3.y, t3.x);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}
template <int DIR>
__device__ __forceinline__ void dft5p(double2 (&v)[5]) {
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const double s1 = DIR * 0.95105651629515357212, s2 = DIR * 0.58778525229247312917;
    const double2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const double2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const double2 m1 = make_double2(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    const double2 m2 = make_double2(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    const double2 n1 = make_double2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
    const double2 n2 = make_double2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
    const double2 in1 = make_double2(-n1.y, n1.x), in2 = make_double2(-n2.y, n2.x);
    v[0] = make_double2(v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y);
    v[1] = cadd(m1, in1);
    v[4] = csub(m1, in1);
    v[2] = cadd(m2, in2);
    v[3] = csub(m2, in2);
}

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8p(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// t = q*d + r for 0 <= t < 2^22 and 1 <= d < 2^16: float reciprocal, one fix-up
__device__ __forceinline__ void fdivmod(int t, int d, float inv, int& q, int& r) {
    q = __float2int_rz(__int2float_rn(t) * inv);
    r = t - q * d;
    if (r < 0) { q -= 1; r += d; }
    else if (r >= d) { q += 1; r -= d; }
}

// one in-place Stockham pass of radix R over nb sequences of length n
// (element e of sequence b at buf[e*sE + b*sB]); tw[e] = exp(-2 pi i e / n)
template <int R, int DIR>
__device__ __forceinline__ void pass_inplace(double2* buf, int n, int Ns, int nb, int sE, int sB, bool bfast,
                                             const double2* tw, int tid) {
    constexpr int MAXB = MAXE / R;
    const int nbf = n / R;
    const int total = nb * nbf;
    const int tstep = n / (Ns * R);
    const int dsplit = bfast ? nb : nbf;
    const float inv_split = 1.0f / (float)dsplit, inv_ns = 1.0f / (float)Ns;
    double2 v[MAXB][R];
    int ob[MAXB];
#pragma unroll
    for (int c = 0; c < MAXB; c++) {
        const int t = tid + c * PT;
        ob[c] = -1;
        if (t < total) {
            int b, j, q, rr;
            fdivmod(t, dsplit, inv_split, q, rr);
            if (bfast) { b = rr; j = q; }
            else { j = rr; b = q; }
            int jq, kk;
            fdivmod(j, Ns, inv_ns, jq, kk);
#pragma unroll
            for (int r = 0; r < R; r++) v[c][r] = buf[(j + r * nbf) * sE + b * sB];
#pragma unroll
            for (int r = 1; r < R; r++) {
                const double2 w = tw[kk * r * tstep];
                v[c][r] = (DIR < 0) ? cmul(v[c][r], w) : cmulc(v[c][r], w);
            }
            if constexpr (R == 2) dft2p<DIR>(v[c]);
            else if constexpr (R == 3) dft3p<DIR>(v[c]);
            else if constexpr (R == 4) dft4p<DIR>(v[c]);
            else dft5p<DIR>(v[c]);
            ob[c] = (jq * Ns * R + kk) * sE + b * sB;
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < MAXB; c++)
        if (ob[c] >= 0)
#pragma unroll
            for (int r = 0; r < R; r++) buf[ob[c] + r * Ns * sE] = v[c][r];
    __syncthreads();
}

// sequences a batch can hold: every pass must fit MAXE/R butterflies per thread
__host__ __device__ inline int batch_seqs(const FftPlan& pl) {
    int cap = 1 << 30;
    for (int s = 0; s < pl.nr; s++) {
        const int R = (int)((pl.code >> (4 * s)) & 15ull);
        const int c = PT * (MAXE / R) * R;
        cap = c < cap ? c : cap;
    }
    return cap / pl.n;
}

// all passes of the plan over nb sequences, in batches whose values fit the
// registers of the block (batches touch disjoint sequences)
template <int DIR>
__device__ __forceinline__ void fft_inplace(double2* buf, int n, int nr, unsigned long long code, int B, int nb, int sE,
                                            int sB, bool bfast, const double2* tw, int tid) {
    for (int b0 = 0; b0 < nb; b0 += B) {
        const int nbb = min(B, nb - b0);
        double2* bb = buf + (size_t)b0 * sB;
        int Ns = 1;
        for (int s = 0; s < nr; s++) {
            const int R = (int)((code >> (4 * s)) & 15ull);
            if (R == 4) pass_inplace<4, DIR>(bb, n, Ns, nbb, sE, sB, bfast, tw, tid);
            else if (R == 2) pass_inplace<2, DIR>(bb, n, Ns, nbb, sE, sB, bfast, tw, tid);
            else if (R == 3) pass_inplace<3, DIR>(bb, n, Ns, nbb, sE, sB, bfast, tw, tid);
            else pass_inplace<5, DIR>(bb, n, Ns, nbb, sE, sB, bfast, tw, tid);
            Ns *= R;
        }
    }
}

// shared memory of a plane CTA: plane [nz][M1] complex, then twiddles
// twx[M], post[M1], twz[nz]
__device__ __forceinline__ void load_twiddles(double2* tws, int M, int M1, int nz, const double2* __restrict__ twx,
                                              const double2* __restrict__ post, const double2* __restrict__ twz,
                                              int tid) {
    for (int t = tid; t < M; t += PT) tws[t] = twx[t];
    for (int t = tid; t < M1; t += PT) tws[M + t] = post[t];
    for (int t = tid; t < nz; t += PT) tws[M + M1 + t] = twz[t];
}

}  // namespace

// MODE 0: source = divergence of u* / pmAlpha (clcPrSrc); 1: divergence
// unscaled (projection of a given field); 2: source array src (compact)
template <int MODE>
__global__ void __launch_bounds__(PT, 1)
    k_plane_fwd(DConst c, DMetric m, DCoef* __restrict__ coef, const double* __restrict__ ux,
                const double* __restrict__ uy, const double* __restrict__ uz, const double* __restrict__ src,
                double2* __restrict__ spec, int nrx, unsigned long long cx, int Bx, int nrz, unsigned long long cz, int Bz,
                const double2* __restrict__ twx,
                const double2* __restrict__ post, const double2* __restrict__ twz, double* __restrict__ part,
                unsigned int* __restrict__ counter, double* __restrict__ out_max) {
    extern __shared__ double2 smp[];
    const int nx = c.nx, ny = c.ny, nz = c.nz, M = nx / 2, M1 = M + 1;
    double2* plane = smp;
    double2* tws = smp + (size_t)nz * M1;
    const int tid = threadIdx.x;
    const int jc = blockIdx.x + 1;  // Fortran row of this plane
    load_twiddles(tws, M, M1, nz, twx, post, twz, tid);
    double* pr = reinterpret_cast<double*>(plane);
    double dm = 0.0;
    const int lane = tid & 31, warp = tid >> 5;
    constexpr int NW = PT / 32;
    if (MODE == 2) {
        for (int k = warp; k < nz; k += NW)
            for (int i = lane; i < nx; i += 32)
                cp_async8p(&pr[(size_t)k * 2 * M1 + i], &src[((size_t)k * ny + (jc - 1)) * nx + i]);
        cp_async_all();
    } else {
        // divergence, 4 cells of a row per thread with all 40 loads issued first
        const size_t pl = (size_t)c.nyt * nx, r0 = (size_t)jc * nx;
        const double sudtal = (MODE == 0) ? 1.0 / coef->pmAlpha : 1.0;
        const double rdyp = __ldg(&m.rdyp[jc]);
        for (int k = warp; k < nz; k += NW) {
            const int km = k == 0 ? nz - 1 : k - 1, kp = k == nz - 1 ? 0 : k + 1, ku = kp == nz - 1 ? 0 : kp + 1;
            const double* ur = ux + (size_t)k * pl + r0;
            const double* vr = uy + (size_t)k * pl + r0;
            const double* w0 = uz + (size_t)km * pl + r0;
            const double* w1 = uz + (size_t)k * pl + r0;
            const double* w2 = uz + (size_t)kp * pl + r0;
            const double* w3 = uz + (size_t)ku * pl + r0;
            for (int i0 = 0; i0 < nx; i0 += 128) {
                double a[4][10];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int i = i0 + lane + 32 * u;
                    const int ii = i < nx ? i : nx - 1;
                    const int im = ii == 0 ? nx - 1 : ii - 1, ip = ii == nx - 1 ? 0 : ii + 1, iu = ip == nx - 1 ? 0 : ip + 1;
                    a[u][0] = __ldg(&ur[im]); a[u][1] = __ldg(&ur[ii]); a[u][2] = __ldg(&ur[ip]); a[u][3] = __ldg(&ur[iu]);
                    a[u][4] = __ldg(&vr[nx + ii]); a[u][5] = __ldg(&vr[ii]);
                    a[u][6] = __ldg(&w0[ii]); a[u][7] = __ldg(&w1[ii]); a[u][8] = __ldg(&w2[ii]); a[u][9] = __ldg(&w3[ii]);
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int i = i0 + lane + 32 * u;
                    const double dudx = c.dxC[0] * a[u][0] + c.dxC[1] * a[u][1] + c.dxC[2] * a[u][2] + c.dxC[3] * a[u][3];
                    const double dvdy = (a[u][4] - a[u][5]) * rdyp;
                    const double dwdz = c.dzC[0] * a[u][6] + c.dzC[1] * a[u][7] + c.dzC[2] * a[u][8] + c.dzC[3] * a[u][9];
                    const double rdiv = dudx + dvdy + dwdz;
                    if (i < nx) {
                        dm = fmax(dm, fabs(rdiv));
                        pr[(size_t)k * 2 * M1 + i] = sudtal * rdiv;
                    }
                }
            }
        }
    }
    __syncthreads();
    // x: M-point complex FFT of every row (even/odd packed), then the split
    fft_inplace<-1>(plane, M, nrx, cx, Bx, nz, 1, M1, false, tws, tid);
    const double2* pst = tws + M;
    for (int k = warp; k < nz; k += NW)
    for (int a = lane; a <= M / 2; a += 32) {
        double2* row = plane + (size_t)k * M1;
        const int b = M - a;  // partner mode
        const double2 za = row[a == M ? 0 : a], zb = row[a == 0 ? 0 : b];
        // X[a] from Z[a], Z[M-a]; X[b] from Z[b], Z[M-b] = Z[a]
        const double2 Ea = make_double2(0.5 * (za.x + zb.x), 0.5 * (za.y - zb.y));
        const double2 Oa = make_double2(0.5 * (za.y + zb.y), -0.5 * (za.x - zb.x));
        const double2 Xa = cadd(Ea, cmul(pst[a], Oa));
        const double2 Eb = make_double2(0.5 * (zb.x + za.x), 0.5 * (zb.y - za.y));
        const double2 Ob = make_double2(0.5 * (zb.y + za.y), -0.5 * (zb.x - za.x));
        const double2 Xb = cadd(Eb, cmul(pst[b], Ob));
        row[a] = Xa;
        if (b != a) row[b] = Xb;
    }
    __syncthreads();
    // z: nz-point FFT of every mode column
    fft_inplace<-1>(plane, nz, nrz, cz, Bz, M1, M1, 1, true, tws + M + M1, tid);
    for (int k = warp; k < nz; k += NW)
        for (int kx = lane; kx < M1; kx += 32)
            spec[((size_t)k * ny + (jc - 1)) * M1 + kx] = plane[(size_t)k * M1 + kx];
    if (MODE == 2) return;
    double v[1] = {dm};
    const unsigned int nblocks = gridDim.x;
    block_max_store<1>(v, part + blockIdx.x);
    if (!last_block_arrive(counter, nblocks)) return;
    double tot[1];
    reduce_records<1, true>(part, (int)nblocks, tot);
    if (tid == 0) *out_max = tot[0];
}

// inverse: spec plane -> phi rows (padded with ghosts, or compact), scaled
__global__ void __launch_bounds__(PT, 1)
    k_plane_inv(int nx, int ny, int nz, const double2* __restrict__ spec, double* __restrict__ phi, int nrx,
                unsigned long long cx, int Bx, int nrz, unsigned long long cz, int Bz, const double2* __restrict__ twx,
                const double2* __restrict__ post,
                const double2* __restrict__ twz, double scale, int padded) {
    extern __shared__ double2 smp[];
    const int M = nx / 2, M1 = M + 1;
    double2* plane = smp;
    double2* tws = smp + (size_t)nz * M1;
    const int tid = threadIdx.x;
    const int j = blockIdx.x;  // 0-based interior row
    load_twiddles(tws, M, M1, nz, twx, post, twz, tid);
    const int lane = tid & 31, warp = tid >> 5;
    constexpr int NW = PT / 32;
    for (int k = warp; k < nz; k += NW)
        for (int kx = lane; kx < M1; kx += 32)
            cp_async16(&plane[(size_t)k * M1 + kx], &spec[((size_t)k * ny + j) * M1 + kx]);
    cp_async_all();
    __syncthreads();
    fft_inplace<1>(plane, nz, nrz, cz, Bz, M1, M1, 1, true, tws + M + M1, tid);
    // merge the modes of every row into M complex values (DC and Nyquist real)
    const double2* pst = tws + M;
    for (int k = warp; k < nz; k += NW)
    for (int a = lane; a <= M / 2; a += 32) {
        double2* row = plane + (size_t)k * M1;
        const int b = M - a;
        double2 xa = row[a], xb = row[b];
        if (a == 0) { xa.y = 0.0; xb.y = 0.0; }
        // Z[a] from X[a], X[M-a]; Z[b] from X[b], X[M-b] = X[a]
        const double2 e2a = make_double2(xa.x + xb.x, xa.y - xb.y);
        const double2 da = make_double2(xa.x - xb.x, xa.y + xb.y);
        const double2 o2a = cmulc(da, pst[a]);
        const double2 Za = make_double2(e2a.x - o2a.y, e2a.y + o2a.x);
        if (a == 0) {
            row[0] = Za;
        } else {
            const double2 e2b = make_double2(xb.x + xa.x, xb.y - xa.y);
            const double2 db = make_double2(xb.x - xa.x, xb.y + xa.y);
            const double2 o2b = cmulc(db, pst[b]);
            const double2 Zb = make_double2(e2b.x - o2b.y, e2b.y + o2b.x);
            row[a] = Za;
            if (b != a) row[b] = Zb;
        }
    }
    __syncthreads();
    fft_inplace<1>(plane, M, nrx, cx, Bx, nz, 1, M1, false, tws, tid);
    const double* pr = reinterpret_cast<const double*>(plane);
    const int nyt = ny + 2;
    for (int k = warp; k < nz; k += NW)
    for (int i = lane; i < nx; i += 32) {
        const double v = pr[(size_t)k * 2 * M1 + i] * scale;
        if (!padded) {
            phi[((size_t)k * ny + j) * nx + i] = v;
            continue;
        }
        double* rowp = phi + ((size_t)k * nyt + (j + 1)) * nx;
        rowp[i] = v;
        if (j == 0) rowp[i - nx] = v;
        if (j == ny - 1) rowp[i + nx] = v;
    }
}

// ---------------------------------------------------------------------------
static size_t plane_smem(int nx, int nz) {
    const int M = nx / 2, M1 = M + 1;
    return ((size_t)nz * M1 + M + M1 + nz) * sizeof(double2);
}

bool plane_supported(int nx, int nz, const FftPlan& plx, const FftPlan& plz) {
    if (plane_smem(nx, nz) > 200 * 1024) return false;
    // every radix must fit at least one butterfly per thread, and a batch at
    // least one sequence
    for (int s = 0; s < plx.nr; s++) if (MAXE / plx.rad[s] < 1) return false;
    for (int s = 0; s < plz.nr; s++) if (MAXE / plz.rad[s] < 1) return false;
    return batch_seqs(plx) >= 1 && batch_seqs(plz) >= 1;
}

void plane_init() {
    cudaFuncSetAttribute(k_plane_fwd<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_plane_fwd<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_plane_fwd<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_plane_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

void launch_plane_fwd(cudaStream_t st, int mode, const DConst& c, const DMetric& m, DCoef* coef, const Fields& f,
                      const double* src, double2* spec, const FftPlan& plx, const FftPlan& plz, const double2* twx,
                      const double2* post, const double2* twz, double* part, unsigned int* counter, double* out_max) {
    const size_t sm = plane_smem(c.nx, c.nz);
    const int Bx = batch_seqs(plx), Bz = batch_seqs(plz);
#define PF_ARGS c, m, coef, f.ux, f.uy, f.uz, src, spec, plx.nr, plx.code, Bx, plz.nr, plz.code, Bz, twx, post, twz, part, counter, out_max
    if (mode == 0) k_plane_fwd<0><<<c.ny, PT, sm, st>>>(PF_ARGS);
    else if (mode == 1) k_plane_fwd<1><<<c.ny, PT, sm, st>>>(PF_ARGS);
    else k_plane_fwd<2><<<c.ny, PT, sm, st>>>(PF_ARGS);
#undef PF_ARGS
}

void launch_plane_inv(cudaStream_t st, int nx, int ny, int nz, const double2* spec, double* phi, const FftPlan& plx,
                      const FftPlan& plz, const double2* twx, const double2* post, const double2* twz, double scale,
                      int padded) {
    k_plane_inv<<<ny, PT, plane_smem(nx, nz), st>>>(nx, ny, nz, spec, phi, plx.nr, plx.code, batch_seqs(plx), plz.nr,
                                                    plz.code, batch_seqs(plz), twx, post, twz, scale, padded);
}

}  // namespace ptc
