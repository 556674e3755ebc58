// k_fft.cu -- batched real FFTs of the pressure Poisson solve on B200.
//
// clcPPE (src/m_Poisson.f90:352-452) transforms the source with FFTW's
// R2HC along x, then R2HC along z, solves one real tridiagonal system in y
// per halfcomplex coefficient and transforms back with HC2R.  Because the
// modified wavenumber is even in the mode number and the y operator is real,
// the same solution comes out of any real transform pair with the same
// per-|k| eigenvalue and the same gauge phi_hat(kx=0,kz=0,jc=1) = 0; this
// file uses a real-to-complex transform in x (nx/2+1 complex modes, computed
// as an nx/2-point complex FFT of the even/odd packed row) and a complex
// transform in z, both unnormalised, with the 1/(nx*nz) of normfft applied
// once at the end as in the reference.
//
// Transforms run in shared memory as Stockham autosort passes of radix 4, 2,
// 3 and 5 (the grids of ParaTC's inputs factor into 2^a*3^b*5^c); twiddles
// come from tables computed on the host in long double.
#include "common.cuh"
#include "kernels.cuh"

namespace ptc {

// R-point DFTs, DIR = -1 forward (exp(-i...)), +1 backward
template <int DIR>
__device__ __forceinline__ void dft2(double2 (&v)[2]) {
    const double2 t = v[0];
    v[0] = cadd(t, v[1]);
    v[1] = csub(t, v[1]);
}

template <int DIR>
__device__ __forceinline__ void dft3(double2 (&v)[3]) {
    const double c = -0.5;
    const double s = DIR * 0.86602540378443864676;  // sin(2 pi / 3)
    const double2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    const double2 mm = make_double2(v[0].x + c * t1.x, v[0].y + c * t1.y);
    const double2 it = make_double2(-s * t2.y, s * t2.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(mm, it);
    v[2] = csub(mm, it);
}

template <int DIR>
__device__ __forceinline__ void dft4(double2 (&v)[4]) {
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
__device__ __forceinline__ void dft5(double2 (&v)[5]) {
    const double c1 = 0.30901699437494742410;   // cos(2 pi / 5)
    const double c2 = -0.80901699437494742410;  // cos(4 pi / 5)
    const double s1 = DIR * 0.95105651629515357212;  // sin(2 pi / 5)
    const double s2 = DIR * 0.58778525229247312917;  // sin(4 pi / 5)
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

template <int R, int DIR>
__device__ __forceinline__ void dftR(double2 (&v)[R]) {
    if constexpr (R == 2) dft2<DIR>(v);
    else if constexpr (R == 3) dft3<DIR>(v);
    else if constexpr (R == 4) dft4<DIR>(v);
    else dft5<DIR>(v);
}

// one Stockham pass over nb sequences of length n; element e of sequence b
// sits at e*sE + b*sB
template <int R, int DIR>
__device__ __forceinline__ void stockham_pass(const double2* __restrict__ in, double2* __restrict__ out, int n, int Ns,
                                              int nb, int sE, int sB, bool bfast,
                                              const double2* __restrict__ tw, int tid, int nthr) {
    const int nbf = n / R;
    const int total = nb * nbf;
    const int tstep = n / (Ns * R);
    for (int t = tid; t < total; t += nthr) {
        int b, j;
        if (bfast) { b = t % nb; j = t / nb; }
        else       { j = t % nbf; b = t / nbf; }
        const int kk = j % Ns;
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = in[(j + r * nbf) * sE + b * sB];
#pragma unroll
        for (int r = 1; r < R; r++) {
            double2 w = __ldg(&tw[kk * r * tstep]);
            v[r] = (DIR < 0) ? cmul(v[r], w) : cmulc(v[r], w);
        }
        dftR<R, DIR>(v);
        const int base = (j - kk) * R + kk;
#pragma unroll
        for (int r = 0; r < R; r++) out[(base + r * Ns) * sE + b * sB] = v[r];
    }
}

template <int DIR>
__device__ double2* smem_fft(double2* a, double2* b, const FftPlan& pl, int nb, int sE, int sB, bool bfast,
                             const double2* __restrict__ tw, int tid, int nthr) {
    int Ns = 1;
    for (int s = 0; s < pl.nr; s++) {
        const int R = pl.rad[s];
        if (R == 4) stockham_pass<4, DIR>(a, b, pl.n, Ns, nb, sE, sB, bfast, tw, tid, nthr);
        else if (R == 2) stockham_pass<2, DIR>(a, b, pl.n, Ns, nb, sE, sB, bfast, tw, tid, nthr);
        else if (R == 3) stockham_pass<3, DIR>(a, b, pl.n, Ns, nb, sE, sB, bfast, tw, tid, nthr);
        else stockham_pass<5, DIR>(a, b, pl.n, Ns, nb, sE, sB, bfast, tw, tid, nthr);
        __syncthreads();
        double2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// forward real transform along x of compact rows src[row*nx + i] into
// spec[row*(nx/2+1) + kx], row = k*ny + (jc-1)
__global__ void __launch_bounds__(256) k_fft_x_r2c(int nx, const double* __restrict__ src, double2* __restrict__ spec,
                                                   int nrows, int rpc, FftPlan pl, const double2* __restrict__ tw,
                                                   const double2* __restrict__ post) {
    extern __shared__ double2 smc[];
    const int M = nx / 2, M1 = M + 1, ld = M + 1;
    double2* A = smc;
    double2* B = smc + (size_t)rpc * ld;
    const int row0 = blockIdx.x * rpc;
    const int nr = min(rpc, nrows - row0);
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int t = tid; t < nr * M; t += nthr) {
        const int r = t / M, mm = t - r * M;
        A[r * ld + mm] = reinterpret_cast<const double2*>(src + (size_t)(row0 + r) * nx)[mm];
    }
    __syncthreads();
    const double2* Rz = smem_fft<-1>(A, B, pl, nr, 1, ld, false, tw, tid, nthr);
    for (int t = tid; t < nr * M1; t += nthr) {
        const int r = t / M1, kx = t - r * M1;
        const double2 zk = Rz[r * ld + (kx == M ? 0 : kx)];
        const double2 zm = Rz[r * ld + (kx == 0 ? 0 : M - kx)];
        const double2 E = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        const double2 O = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
        spec[(size_t)(row0 + r) * M1 + kx] = cadd(E, cmul(__ldg(&post[kx]), O));
    }
}

// complex transform along z, in place, on tiles of T consecutive kx of one y row
template <int DIR>
__global__ void __launch_bounds__(256) k_fft_z(int nx, int ny, int nz, double2* __restrict__ spec, int T, FftPlan pl,
                                               const double2* __restrict__ tw) {
    extern __shared__ double2 smc[];
    const int M1 = nx / 2 + 1;
    const int j = blockIdx.y;
    const int kx0 = blockIdx.x * T;
    const int nb = min(T, M1 - kx0);
    double2* A = smc;
    double2* B = smc + (size_t)nz * T;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int t = tid; t < nz * T; t += nthr) {
        const int e = t / T, b = t - e * T;
        A[t] = (b < nb) ? spec[((size_t)e * ny + j) * M1 + kx0 + b] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const double2* Rz = smem_fft<DIR>(A, B, pl, T, T, 1, true, tw, tid, nthr);
    for (int t = tid; t < nz * T; t += nthr) {
        const int e = t / T, b = t - e * T;
        if (b < nb) spec[((size_t)e * ny + j) * M1 + kx0 + b] = Rz[t];
    }
}

// backward real transform along x into the padded field phi (rows jc and,
// at the walls, the Neumann ghost rows phi(0) = phi(1), phi(nyp) = phi(nyc)
// of SetBC_and_UpdateHalo_pr, src/m_BC_and_Halo.f90:115-120), scaled by s
__global__ void __launch_bounds__(256) k_fft_x_c2r(int nx, int ny, const double2* __restrict__ spec,
                                                   double* __restrict__ phi, int nrows, int rpc, FftPlan pl,
                                                   const double2* __restrict__ tw, const double2* __restrict__ post,
                                                   double scale, int padded) {
    extern __shared__ double2 smc[];
    const int M = nx / 2, M1 = M + 1, ld = M + 1;
    double2* A = smc;
    double2* B = smc + (size_t)rpc * ld;
    const int row0 = blockIdx.x * rpc;
    const int nr = min(rpc, nrows - row0);
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int t = tid; t < nr * M; t += nthr) {
        const int r = t / M, kx = t - r * M;
        const double2* srow = spec + (size_t)(row0 + r) * M1;
        double2 xk = srow[kx];
        double2 xm = srow[M - kx];
        if (kx == 0) { xk.y = 0.0; xm.y = 0.0; }  // DC and Nyquist coefficients are real
        const double2 e2 = make_double2(xk.x + xm.x, xk.y - xm.y);
        const double2 d = make_double2(xk.x - xm.x, xk.y + xm.y);
        const double2 o2 = cmulc(d, __ldg(&post[kx]));
        A[r * ld + kx] = make_double2(e2.x - o2.y, e2.y + o2.x);
    }
    __syncthreads();
    const double2* Rz = smem_fft<1>(A, B, pl, nr, 1, ld, false, tw, tid, nthr);
    const int nyt = ny + 2;
    for (int t = tid; t < nr * M; t += nthr) {
        const int r = t / M, mm = t - r * M;
        const double2 z = Rz[r * ld + mm];
        const double2 v = make_double2(z.x * scale, z.y * scale);
        const int g = row0 + r;
        if (!padded) {
            reinterpret_cast<double2*>(phi + (size_t)g * nx)[mm] = v;
            continue;
        }
        const int k = g / ny, jc = g - k * ny + 1;
        double* rowp = phi + ((size_t)k * nyt + jc) * nx;
        reinterpret_cast<double2*>(rowp)[mm] = v;
        if (jc == 1) reinterpret_cast<double2*>(rowp - nx)[mm] = v;
        if (jc == ny) reinterpret_cast<double2*>(rowp + nx)[mm] = v;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int x_rows_per_cta(int nx) {
    const size_t per_row = (size_t)2 * (nx / 2 + 1) * sizeof(double2);
    int r = (int)((64 * 1024) / per_row);
    if (r > 16) r = 16;
    if (r < 1) r = 1;
    return r;
}

static int z_tile(int nz) {
    const size_t per_col = (size_t)2 * nz * sizeof(double2);
    int t = (int)((96 * 1024) / per_col);
    if (t >= 16) return 16;
    if (t >= 8) return 8;
    if (t >= 4) return 4;
    if (t >= 2) return 2;
    return 1;
}

void fft_init() {
    cudaFuncSetAttribute(k_fft_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_fft_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_fft_z<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_fft_z<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
}

size_t fft_smem_need(int nx, int nz) {
    const size_t sx = (size_t)x_rows_per_cta(nx) * 2 * (nx / 2 + 1) * sizeof(double2);
    const size_t sz = (size_t)2 * nz * z_tile(nz) * sizeof(double2);
    return sx > sz ? sx : sz;
}

void launch_fft_x_r2c(cudaStream_t st, int nx, int nrows, const double* src, double2* spec, const FftPlan& pl,
                      const double2* tw, const double2* post) {
    const int rpc = x_rows_per_cta(nx);
    const size_t smem = (size_t)rpc * 2 * (nx / 2 + 1) * sizeof(double2);
    k_fft_x_r2c<<<(nrows + rpc - 1) / rpc, 256, smem, st>>>(nx, src, spec, nrows, rpc, pl, tw, post);
}

void launch_fft_z(cudaStream_t st, int dir, int nx, int ny, int nz, double2* spec, const FftPlan& pl, const double2* tw) {
    const int T = z_tile(nz);
    const size_t smem = (size_t)2 * nz * T * sizeof(double2);
    dim3 grd((nx / 2 + 1 + T - 1) / T, ny);
    if (dir < 0) k_fft_z<-1><<<grd, 256, smem, st>>>(nx, ny, nz, spec, T, pl, tw);
    else k_fft_z<1><<<grd, 256, smem, st>>>(nx, ny, nz, spec, T, pl, tw);
}

void launch_fft_x_c2r(cudaStream_t st, int nx, int ny, int nrows, const double2* spec, double* phi, const FftPlan& pl,
                      const double2* tw, const double2* post, double scale, int padded) {
    const int rpc = x_rows_per_cta(nx);
    const size_t smem = (size_t)rpc * 2 * (nx / 2 + 1) * sizeof(double2);
    k_fft_x_c2r<<<(nrows + rpc - 1) / rpc, 256, smem, st>>>(nx, ny, spec, phi, nrows, rpc, pl, tw, post, scale, padded);
}

}  // namespace ptc
