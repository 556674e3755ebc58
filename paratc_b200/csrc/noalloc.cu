// noalloc.cu -- a pressure Poisson solve that allocates no memory.
//
// Why it exists: some callers cannot call cudaMalloc.  Typical cases are a
// host program that hands the GPU to this library from inside a region where
// it must not allocate (a real-time loop with a fixed memory budget, a code
// whose allocator owns all device memory and forbids other allocations, or a
// caller that cannot hold a library context between calls).  For them
// paratc_poisson_noalloc() solves the same system as paratc_poisson_device()
// but takes its working memory from one fixed array that lives in the
// library image itself.
//
// The working memory is the file-scope array g_noalloc_scratch below: a
// static __device__ array of PARATC_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB).
// Every GPU that loads the library holds it until the process exits.  It
// carries the spectral coefficients of the solve, the y metrics, the
// wavenumbers and the FFT twiddle tables, all rewritten by every call before
// they are read (the forward x transform overwrites every spectral entry), so
// nothing has to start at zero.
//
// In host code the name g_noalloc_scratch is only a host-side stand-in for the
// device array, not a device address; passing it to a kernel would fault (or,
// where the GPU can reach host memory, silently use the wrong memory).  The
// device address is obtained once per device, with that device current, by
// cudaGetSymbolAddress() in noalloc_setup(); the first call of the entry point
// on a device performs that set-up (and sets the shared-memory limits of the
// FFT kernels) under a per-device std::call_once, so first calls from several
// host threads are safe.  The address is kept for the life of the process:
// cudaDeviceReset() after the first call is not supported.
//
// The entry point must not be called while its stream is being captured into
// a CUDA graph (it returns PARATC_ERR_BAD_ARG then): it copies tables from
// its stack frame to the device and waits for the stream.
//
// All calls share the one array: two calls whose work overlaps on the GPU
// (different streams, or different host threads) race and corrupt each other.
// The entry point calls no cudaMalloc, cudaFree or other allocating routine;
// host-side tables live on the stack (about 68 KB at the largest sizes).
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/paratc.h"
#include "common.cuh"
#include "kernels.cuh"

using namespace ptc;

namespace {

static __device__ __align__(256) double g_noalloc_scratch[PARATC_NOALLOC_SCRATCH_DOUBLES];

constexpr int kMaxDevices = 64;
constexpr int kMaxNxz = 1024;    // largest nxc / nzc accepted (host stack tables)
constexpr int kMaxNy = 256;      // largest nyc accepted (the tridiagonal kernels)
std::once_flag g_setup_once[kMaxDevices];
std::atomic<double*> g_scratch_dev[kMaxDevices];

// once per device, with that device current: the device address of the
// array and the kernels' shared-memory limits
int noalloc_setup(int dev) {
    std::call_once(g_setup_once[dev], [dev] {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            std::fprintf(stderr, "paratc_poisson_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return;
        }
        fft_init();
        tridiag_init();
        g_scratch_dev[dev].store(static_cast<double*>(p), std::memory_order_release);
    });
    return g_scratch_dev[dev].load(std::memory_order_acquire) ? PARATC_OK : PARATC_ERR_CUDA;
}

bool plan_of(int n, FftPlan& pl) {
    pl.n = n;
    pl.nr = 0;
    int m = n;
    const int rads[4] = {4, 2, 3, 5};
    for (int r : rads)
        while (m % r == 0 && pl.nr < PT_MAX_RADIX_PASSES) { pl.rad[pl.nr++] = r; m /= r; }
    pl.code = 0;
    for (int s = 0; s < pl.nr && s < 16; s++) pl.code |= (unsigned long long)pl.rad[s] << (4 * s);
    return m == 1 && pl.nr <= 16;
}

void fill_twiddles(double2* w, int n, int count) {
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < count; k++) {
        const long double a = -2.0L * pi * (long double)k / (long double)n;
        w[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
}

size_t align32(size_t n) { return (n + 31) & ~(size_t)31; }

}  // namespace

extern "C" int paratc_poisson_noalloc(const paratc_params* prm, const double* yp, const double* d_src, double* d_phi,
                                      void* stream) {
    if (!prm || !yp || !d_src || !d_phi) return PARATC_ERR_BAD_ARG;
    const int nx = prm->nxc, ny = prm->nyc, nz = prm->nzc;
    if (nx < 4 || nz < 4 || ny < 3 || nx % 2 || nz % 2 || nx > kMaxNxz || nz > kMaxNxz || ny > kMaxNy ||
        !tridiag_supported(ny) || !(prm->xlx > 0) || !(prm->zlz > 0)) {
        std::fprintf(stderr, "paratc_poisson_noalloc: grid %dx%dx%d outside the supported range\n", nx, ny, nz);
        return PARATC_ERR_BAD_ARG;
    }
    FftPlan plx, plz;
    if (!plan_of(nx / 2, plx) || !plan_of(nz, plz) || fft_smem_need(nx, nz) > 160 * 1024) {
        std::fprintf(stderr, "paratc_poisson_noalloc: nxc/2 and nzc must factor into 2, 3 and 5\n");
        return PARATC_ERR_BAD_ARG;
    }
    const int M1 = nx / 2 + 1, nyp = ny + 1;
    // scratch layout (doubles): spectral | am2ph ac2ph ap2ph | wnx wnz | twx postx twz
    const size_t o_spec = 0;
    const size_t o_m = align32(o_spec + (size_t)2 * M1 * ny * nz);
    const size_t o_w = align32(o_m + (size_t)3 * (nyp + 1));
    const size_t o_t = align32(o_w + (size_t)nx + nz);
    const size_t need = o_t + (size_t)2 * (nx / 2 + M1 + nz);
    if (need > (size_t)PARATC_NOALLOC_SCRATCH_DOUBLES) {
        std::fprintf(stderr,
                     "paratc_poisson_noalloc: grid %dx%dx%d needs %zu scratch doubles, the fixed array holds %d\n",
                     nx, ny, nz, need, PARATC_NOALLOC_SCRATCH_DOUBLES);
        return PARATC_ERR_BAD_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PARATC_ERR_NO_DEVICE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // an error left by an earlier, unrelated call would otherwise be reported
    // as this call's own by the launch check at the end
    (void)cudaGetLastError();
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
        std::fprintf(stderr, "paratc_poisson_noalloc: the stream is being captured; call it outside stream capture\n");
        return PARATC_ERR_BAD_ARG;
    }
    int rc = noalloc_setup(dev);
    if (rc != PARATC_OK) return rc;
    double* scr = g_scratch_dev[dev].load(std::memory_order_acquire);

    // pressure y operator (InitMeshAndMetries, src/m_MeshAndMetries.f90:194-247)
    // and the modified wavenumbers (src/m_Poisson.f90:40-48), on the stack
    double ypl[kMaxNy + 3], yc[kMaxNy + 3], dyp[kMaxNy + 3], dyc[kMaxNy + 3], rdyp[kMaxNy + 3], rdyc[kMaxNy + 3];
    double met[3 * (kMaxNy + 3)];
    for (int j = 1; j <= nyp; j++) ypl[j] = yp[j - 1];
    for (int j = 1; j < nyp; j++)
        if (!(ypl[j + 1] > ypl[j])) return PARATC_ERR_BAD_ARG;
    for (int j = 1; j <= ny; j++) yc[j] = 0.5 * (ypl[j] + ypl[j + 1]);
    for (int j = 1; j <= ny; j++) dyp[j] = ypl[j + 1] - ypl[j];
    dyp[0] = dyp[1];
    dyp[nyp] = dyp[ny];
    for (int j = 2; j <= ny; j++) dyc[j] = yc[j] - yc[j - 1];
    dyc[1] = dyp[1];
    dyc[nyp] = dyp[ny];
    for (int j = 0; j <= nyp; j++) rdyp[j] = 1.0 / dyp[j];
    for (int j = 1; j <= nyp; j++) rdyc[j] = 1.0 / dyc[j];
    double* am = met;
    double* ac = met + (nyp + 1);
    double* ap = met + 2 * (nyp + 1);
    for (int j = 0; j <= nyp; j++) am[j] = ac[j] = ap[j] = 0.0;
    for (int j = 1; j <= ny; j++) { am[j] = rdyp[j] * rdyc[j]; ap[j] = rdyp[j] * rdyc[j + 1]; }
    am[1] = 0.0; ap[1] = rdyp[1] * rdyc[2];
    am[ny] = rdyp[ny] * rdyc[ny]; ap[ny] = 0.0;
    for (int j = 1; j <= ny; j++) ac[j] = -(am[j] + ap[j]);
    double wn[2 * kMaxNxz];
    const double twopi = 6.283185307179586476925286766559005768;
    const double rdx = (double)nx / prm->xlx, rdz = (double)nz / prm->zlz;
    const double rdx2 = rdx * rdx, rdz2 = rdz * rdz;
    for (int i = 1; i <= nx; i++) {
        const double w = twopi * (double)(i - 1) / (double)nx;
        wn[i - 1] = rdx2 / 288.0 * (std::cos(3.0 * w) - 54.0 * std::cos(2.0 * w) + 783.0 * std::cos(w) - 730.0);
    }
    for (int k = 1; k <= nz; k++) {
        const double w = twopi * (double)(k - 1) / (double)nz;
        wn[nx + k - 1] = rdz2 / 288.0 * (std::cos(3.0 * w) - 54.0 * std::cos(2.0 * w) + 783.0 * std::cos(w) - 730.0);
    }
    double2 tw[kMaxNxz / 2 + (kMaxNxz / 2 + 1) + kMaxNxz];
    fill_twiddles(tw, nx / 2, nx / 2);
    fill_twiddles(tw + nx / 2, nx, M1);
    fill_twiddles(tw + nx / 2 + M1, nz, nz);

    cudaError_t e;
    if ((e = cudaMemcpyAsync(scr + o_m, met, sizeof(double) * 3 * (nyp + 1), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(scr + o_w, wn, sizeof(double) * (nx + nz), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(scr + o_t, tw, sizeof(double2) * (nx / 2 + M1 + nz), cudaMemcpyHostToDevice, st)) != cudaSuccess) {
        std::fprintf(stderr, "paratc_poisson_noalloc: %s\n", cudaGetErrorString(e));
        return PARATC_ERR_CUDA;
    }
    DConst kc;
    std::memset(&kc, 0, sizeof(kc));
    kc.nx = nx; kc.ny = ny; kc.nz = nz; kc.nyp = nyp; kc.nyt = ny + 2;
    DMetric dm;
    std::memset(&dm, 0, sizeof(dm));
    dm.am2ph = scr + o_m;
    dm.ac2ph = scr + o_m + (nyp + 1);
    dm.ap2ph = scr + o_m + 2 * (nyp + 1);
    dm.wnx = scr + o_w;
    dm.wnz = scr + o_w + nx;
    double2* spec = reinterpret_cast<double2*>(scr + o_spec);
    const double2* twx = reinterpret_cast<const double2*>(scr + o_t);
    const double2* postx = twx + nx / 2;
    const double2* twz = postx + M1;
    const int nrows = ny * nz;
    launch_fft_x_r2c(st, nx, nrows, d_src, spec, plx, twx, postx);
    launch_fft_z(st, -1, nx, ny, nz, spec, plz, twz);
    launch_ysolve(st, kc, dm, spec);
    launch_fft_z(st, +1, nx, ny, nz, spec, plz, twz);
    launch_fft_x_c2r(st, nx, ny, nrows, spec, d_phi, plx, twx, postx, 1.0 / ((double)nx * (double)nz), 0);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        std::fprintf(stderr, "paratc_poisson_noalloc: %s\n", cudaGetErrorString(e));
        return PARATC_ERR_CUDA;
    }
    return PARATC_OK;
}
