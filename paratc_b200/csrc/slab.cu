// slab.cu -- the pressure Poisson solve of clcPPE_x1 (src/m_Poisson.f90:352-452)
// over a z-slab decomposition of several GPUs.
//
// The reference solves on 2-D pencils and moves the array through six
// MPI_ALLTOALLW transposes per solve (y1->x1, x1->z2, z2->y2 and back;
// src/m_Decomp2d.f90:585-1000).  On GPUs joined by NVSwitch every peer is
// one hop at full bandwidth, so a 1-D decomposition needs only two
// exchanges: rank r of G holds the planes kc in [k0_r, k0_r+nzl_r) of the
// source, transforms them along x (a local operation), and one all-to-all
// regroups the x spectrum so that rank r holds every plane of the modes kx
// in [kx0_r, kx0_r+nxl_r) (an "x-slab").  The z transform, the y-Thomas
// solve of each (kx, kz) column and the inverse z transform are then local;
// a second all-to-all returns the planes, and the inverse x transform gives
// the rank's planes of phi.
//
// Layouts (complex values as double2):
//   spectrum of the local planes  [kl][jc][kx]      kl < nzl, kx < nxc/2+1
//   send / recv buffer            for each peer q in rank order, the block
//                                 [kl][jc][kx - kx0_q] of q's modes
//                                 (offset nzl*nyc*kx0_q)
//   x-slab                        [kc][jc][kx - kx0_r]: the block received
//                                 from peer s holds its planes, so the blocks
//                                 in rank order ARE the x-slab (no unpack)
// After the middle step, the planes of peer s are the contiguous block at
// kc = k0_s of the x-slab, so the backward exchange needs no pack either.
// The only reordering is the pack of the forward exchange and the matching
// unpack of the backward one (k_slab_pack), an HBM-bound copy.
//
// Peer form (no collective library): every rank's plan owns its x-slab,
// whose device address the other ranks map (CUDA IPC, paratc_ipc_*); the
// forward scatter (k_slab_scatter) stores each value of the local planes'
// spectrum straight into its owner's x-slab over NVLink, and the backward
// gather loads them back from there, so pack, exchange and unpack are one
// kernel each way, with plain loads and stores to peer memory (no TMA, no
// multicast).  The ordering between ranks is the caller's: all ranks'
// scatters complete before any rank's middle step, all middle steps before
// any gather, all gathers before the next scatter (a stream synchronisation
// and a barrier of the host processes at each of the three points).
//
// The kernels are the library's own: the bulk-copy-fed x transforms
// (k_xf_tma / k_xb_tma) where nxc/2 has a compiled length and the arrays are
// 16-byte aligned, else the generic k_fft_x_r2c / k_fft_x_c2r; the TMA-fed z
// transform (k_zt_tma, its tensor map encoded over the caller's x-slab)
// where nzc has a compiled length, else the generic k_fft_z; and the
// stored-pivot y-Thomas sweeps of the one-GPU solve (k_ys_staged /
// k_ys_global bodies), their pivots computed once per plan for the rank's
// modes (m.wnx offset to kx0; only the rank holding kx = 0 has the
// kx = kz = 0 system with row 1 replaced by phi = 0).  The solve is the
// same discrete system as paratc_poisson_device().
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/paratc.h"
#include "common.cuh"
#include "host_setup.h"
#include "kernels.cuh"

using namespace ptc;

namespace {

// a balanced split: the first n % g ranks get one item more
__host__ __device__ inline int split_start(int n, int g, int r) {
    const int base = n / g, rem = n % g;
    return r * base + (r < rem ? r : rem);
}
__host__ __device__ inline int split_count(int n, int g, int r) { return n / g + (r < n % g ? 1 : 0); }
// the rank that owns item i
__device__ inline int split_owner(int n, int g, int i) {
    const int base = n / g, rem = n % g;
    const int cut = rem * (base + 1);
    return i < cut ? i / (base + 1) : rem + (i - cut) / base;
}

// Forward exchange pack (dir 0: spec -> buf) and backward exchange unpack
// (dir 1: buf -> spec).  One thread per complex value of the local planes'
// spectrum, in its own order, so the spectrum side is read or written
// coalesced and the buffer side in runs of nxl_q values.
__global__ void __launch_bounds__(256) k_slab_pack(int dir, int nzl, int ny, int M1, int G, double2* __restrict__ spec,
                                                   double2* __restrict__ buf) {
    const size_t total = (size_t)nzl * ny * M1;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int kx = (int)(e % M1);
        const size_t row = e / M1;  // kl*ny + jc-1
        const int q = split_owner(M1, G, kx);
        const int kx0 = split_start(M1, G, q), nxl = split_count(M1, G, q);
        const size_t o = (size_t)nzl * ny * kx0 + row * nxl + (kx - kx0);
        if (dir == 0) buf[o] = spec[e];
        else spec[e] = buf[o];
    }
}

struct SlabPeers {
    double2* p[PARATC_SLAB_MAX_RANKS];
};
static_assert(PARATC_SLAB_MAX_RANKS <= sizeof(XtGather::p) / sizeof(XtGather::p[0]), "gather table size");

// dir 0: scatter the local planes' spectrum into every rank's x-slab;
// dir 1: gather it back.  Value (kl, jc, kx) of this rank (planes from k0)
// lives in owner q's x-slab at ((k0 + kl)*ny + jc-1)*nxl_q + kx - kx0_q.
__global__ void __launch_bounds__(256) k_slab_scatter(int dir, int nzl, int ny, int M1, int G, int k0,
                                                      double2* __restrict__ spec, SlabPeers peers) {
    const size_t total = (size_t)nzl * ny * M1;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int kx = (int)(e % M1);
        const size_t row = e / M1;
        const int q = split_owner(M1, G, kx);
        const int kx0 = split_start(M1, G, q), nxl = split_count(M1, G, q);
        double2* x = peers.p[q] + ((size_t)k0 * ny + row) * nxl + (kx - kx0);
        if (dir == 0) *x = spec[e];
        else spec[e] = *x;
    }
}

bool radix_plan(int n, FftPlan& pl) {
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

std::vector<double2> twiddle_table(int n, int count) {
    std::vector<double2> w(count);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < count; k++) {
        const long double a = -2.0L * pi * (long double)k / (long double)n;
        w[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    return w;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int grid_blocks(size_t n, int nsm) {
    const size_t b = (n + 255) / 256;
    const size_t cap = (size_t)nsm * 8;
    return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

}  // namespace

struct paratc_slab {
    int dev = 0, rank = 0, nranks = 1, nsm = 148;
    int nx = 0, ny = 0, nz = 0, M1 = 0;
    int k0 = 0, nzl = 0, kx0 = 0, nxl = 0;
    double normfft = 0.0;
    FftPlan plx{}, plz{};
    double2* d_spec = nullptr;  // [nzl][ny][M1]
    double2* d_xslab = nullptr; // [nz][ny][nxl], the plan's own x-slab (peer form)
    unsigned int* d_err = nullptr;  // bounded-wait failure word of the TMA-fed kernels (+ their poll setting)
    bool xt = false, zt = false;    // compiled-length x / z transforms available
    const void* zt_for = nullptr;   // the x-slab the tensor map below was encoded for
    alignas(64) unsigned char zt_map[128];
    double* d_fac = nullptr;    // pivots of the x-slab's columns: 1/vecm then arr, nyc*nxl*nzc each
    double* d_tab = nullptr;    // am2ph ac2ph ap2ph (nyp+1 each) | wnx (M1) | wnz (nz) | twx postx twz
    DConst kc{};
    DMetric dm{};
    const double2 *twx = nullptr, *postx = nullptr, *twz = nullptr;
};

extern "C" int paratc_slab_partition(int n, int nranks, int rank, int* start, int* count) {
    if (n < 1 || nranks < 1 || nranks > n || rank < 0 || rank >= nranks || !start || !count) return PARATC_ERR_BAD_ARG;
    *start = split_start(n, nranks, rank);
    *count = split_count(n, nranks, rank);
    return PARATC_OK;
}

extern "C" int paratc_slab_create(const paratc_params* prm, const double* yp, int device, int rank, int nranks,
                                  paratc_slab** out) {
    if (!prm || !yp || !out) return PARATC_ERR_BAD_ARG;
    *out = nullptr;
    const int nx = prm->nxc, ny = prm->nyc, nz = prm->nzc;
    const int M1 = nx / 2 + 1;
    if (nranks < 1 || nranks > PARATC_SLAB_MAX_RANKS || rank < 0 || rank >= nranks || nranks > nz || nranks > M1) {
        std::fprintf(stderr, "paratc_slab_create: rank %d of %d does not fit nzc = %d, nxc/2+1 = %d\n", rank, nranks,
                     nz, M1);
        return PARATC_ERR_BAD_ARG;
    }
    if (nx < 4 || nx % 2 || nz < 2 || !tridiag_supported(ny)) {
        std::fprintf(stderr, "paratc_slab_create: grid %dx%dx%d outside the supported range\n", nx, ny, nz);
        return PARATC_ERR_BAD_ARG;
    }
    std::string why;
    int rc = validate_params(*prm, why);
    if (rc != PARATC_OK) {
        std::fprintf(stderr, "paratc_slab_create: %s\n", why.c_str());
        return rc;
    }
    paratc_slab* s = new (std::nothrow) paratc_slab;
    if (!s) return PARATC_ERR_OOM;
    s->rank = rank; s->nranks = nranks;
    s->nx = nx; s->ny = ny; s->nz = nz; s->M1 = M1;
    s->k0 = split_start(nz, nranks, rank); s->nzl = split_count(nz, nranks, rank);
    s->kx0 = split_start(M1, nranks, rank); s->nxl = split_count(M1, nranks, rank);
    if (!radix_plan(nx / 2, s->plx) || !radix_plan(nz, s->plz) || fft_smem_need(nx, nz) > 160 * 1024) {
        std::fprintf(stderr, "paratc_slab_create: nxc/2 and nzc must factor into 2, 3 and 5\n");
        delete s;
        return PARATC_ERR_BAD_ARG;
    }
    HostMetrics h;
    rc = build_metrics(*prm, yp, h);
    if (rc != PARATC_OK) { delete s; return rc; }
    s->normfft = h.normfft;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { delete s; return PARATC_ERR_NO_DEVICE; }
    if (device < 0 || device >= ndev || cudaSetDevice(device) != cudaSuccess) { delete s; return PARATC_ERR_BAD_ARG; }
    s->dev = device;
    cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, device);
    // the transforms' and the partitioned y-solve's shared-memory limits
    // (attributes of the device; setting them again is harmless)
    fft_init();
    tridiag_init();
    xt_tma_init();
    zt_tma_init();

    const int nyp = ny + 1;
    std::vector<double> tab;
    auto put = [&tab](const std::vector<double>& v, size_t n) {
        for (size_t i = 0; i < n; i++) tab.push_back(i < v.size() ? v[i] : 0.0);
    };
    put(h.am2ph, nyp + 1);
    put(h.ac2ph, nyp + 1);
    put(h.ap2ph, nyp + 1);
    const size_t o_wnx = tab.size();
    put(h.wnx, M1);
    const size_t o_wnz = tab.size();
    put(h.wnz, nz);
    while (tab.size() % 2) tab.push_back(0.0);  // double2 alignment of the twiddles
    const size_t o_tw = tab.size();
    for (const auto& w : {twiddle_table(nx / 2, nx / 2), twiddle_table(nx, M1), twiddle_table(nz, nz)})
        for (const double2& c : w) { tab.push_back(c.x); tab.push_back(c.y); }
    cudaError_t e;
    if ((e = cudaMalloc(&s->d_tab, tab.size() * sizeof(double))) != cudaSuccess ||
        (e = cudaMemcpy(s->d_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&s->d_spec, (size_t)s->nzl * ny * M1 * sizeof(double2))) != cudaSuccess ||
        (e = cudaMalloc(&s->d_err, 2 * sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaMemset(s->d_err, 0, 2 * sizeof(unsigned int))) != cudaSuccess) {
        std::fprintf(stderr, "paratc_slab_create: %s\n", cudaGetErrorString(e));
        paratc_slab_destroy(s);
        return e == cudaErrorMemoryAllocation ? PARATC_ERR_OOM : PARATC_ERR_CUDA;
    }
    std::memset(&s->kc, 0, sizeof(s->kc));
    // the y-solve sees an x-slab of nxl modes: nx such that nx/2+1 = nxl,
    // its column 0 being the global mode kx0
    s->kc.nx = 2 * (s->nxl - 1);
    s->kc.ny = ny; s->kc.nz = nz; s->kc.nyp = nyp; s->kc.nyt = ny + 2;
    s->kc.nsm = s->nsm;
    // the staged sweep copies pivot pairs as 16-byte units: an even column count
    if ((s->nxl * nz) % 2) s->kc.solver_sel = 2;
    std::memset(&s->dm, 0, sizeof(s->dm));
    s->dm.am2ph = s->d_tab;
    s->dm.ac2ph = s->d_tab + (nyp + 1);
    s->dm.ap2ph = s->d_tab + 2 * (nyp + 1);
    s->dm.wnx = s->d_tab + o_wnx + s->kx0;
    s->dm.wnz = s->d_tab + o_wnz;
    s->twx = reinterpret_cast<const double2*>(s->d_tab + o_tw);
    s->postx = s->twx + nx / 2;
    s->twz = s->postx + M1;
    const size_t nq = (size_t)s->nxl * nz;
    if ((e = cudaMalloc(&s->d_fac, 2 * nq * ny * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&s->d_xslab, nq * ny * sizeof(double2))) != cudaSuccess) {
        std::fprintf(stderr, "paratc_slab_create: %s\n", cudaGetErrorString(e));
        paratc_slab_destroy(s);
        return e == cudaErrorMemoryAllocation ? PARATC_ERR_OOM : PARATC_ERR_CUDA;
    }
    launch_pois_factors_slab(0, s->kc, s->dm, s->d_fac, s->kx0 == 0);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaDeviceSynchronize()) != cudaSuccess) {
        std::fprintf(stderr, "paratc_slab_create: %s\n", cudaGetErrorString(e));
        paratc_slab_destroy(s);
        return PARATC_ERR_CUDA;
    }
    s->xt = xt_tma_supported(nx / 2);
    s->zt = zt_tma_supported(nz);
    *out = s;
    return PARATC_OK;
}

extern "C" int paratc_slab_destroy(paratc_slab* s) {
    if (!s) return PARATC_OK;
    cudaSetDevice(s->dev);
    if (s->d_spec) cudaFree(s->d_spec);
    if (s->d_tab) cudaFree(s->d_tab);
    if (s->d_err) cudaFree(s->d_err);
    if (s->d_fac) cudaFree(s->d_fac);
    if (s->d_xslab) cudaFree(s->d_xslab);
    delete s;
    return PARATC_OK;
}

extern "C" int paratc_slab_counts(const paratc_slab* s, int64_t* send, int64_t* recv) {
    if (!s) return PARATC_ERR_BAD_ARG;
    for (int q = 0; q < s->nranks; q++) {
        if (send) send[q] = 2LL * s->nzl * s->ny * split_count(s->M1, s->nranks, q);
        if (recv) recv[q] = 2LL * split_count(s->nz, s->nranks, q) * s->ny * s->nxl;
    }
    return PARATC_OK;
}

static int slab_finish(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return PARATC_OK;
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    return PARATC_ERR_CUDA;
}

extern "C" int paratc_slab_forward(paratc_slab* s, const double* d_src, double* d_send, void* stream) {
    if (!s || !d_src || !d_send) return PARATC_ERR_BAD_ARG;
    cudaSetDevice(s->dev);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->nzl * s->ny * s->M1;
    if (s->xt && aligned16(d_src))
        launch_xf_tma(st, s->nx, s->ny, s->nzl, d_src, s->d_spec, s->twx, s->postx, s->nsm, s->d_err);
    else
        launch_fft_x_r2c(st, s->nx, s->nzl * s->ny, d_src, s->d_spec, s->plx, s->twx, s->postx);
    k_slab_pack<<<grid_blocks(n, s->nsm), 256, 0, st>>>(0, s->nzl, s->ny, s->M1, s->nranks, s->d_spec,
                                                        reinterpret_cast<double2*>(d_send));
    return slab_finish("paratc_slab_forward");
}

extern "C" int paratc_slab_middle(paratc_slab* s, double* d_xslab, void* stream) {
    if (!s || !d_xslab) return PARATC_ERR_BAD_ARG;
    cudaSetDevice(s->dev);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double2* xs = reinterpret_cast<double2*>(d_xslab);
    const int ncol = s->ny * s->nxl;
    if (s->zt && s->zt_for != xs) s->zt_for = zt_tma_prepare(xs, ncol, s->nz, s->zt_map) ? xs : nullptr;
    const bool zt = s->zt && s->zt_for == xs;
    if (zt) launch_zt_tma(st, -1, ncol, s->nz, s->zt_map, s->twz, s->nsm, s->d_err);
    else launch_fft_z(st, -1, s->kc.nx, s->ny, s->nz, xs, s->plz, s->twz);
    launch_ysolve_fac_slab(st, s->kc, s->dm, xs, s->d_fac, s->kx0 == 0);
    if (zt) launch_zt_tma(st, +1, ncol, s->nz, s->zt_map, s->twz, s->nsm, s->d_err);
    else launch_fft_z(st, +1, s->kc.nx, s->ny, s->nz, xs, s->plz, s->twz);
    return slab_finish("paratc_slab_middle");
}

extern "C" int paratc_slab_backward(paratc_slab* s, const double* d_recv, double* d_phi, void* stream) {
    if (!s || !d_recv || !d_phi) return PARATC_ERR_BAD_ARG;
    cudaSetDevice(s->dev);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->nzl * s->ny * s->M1;
    k_slab_pack<<<grid_blocks(n, s->nsm), 256, 0, st>>>(1, s->nzl, s->ny, s->M1, s->nranks, s->d_spec,
                                                        const_cast<double2*>(reinterpret_cast<const double2*>(d_recv)));
    if (s->xt && aligned16(d_phi))
        launch_xb_tma(st, s->nx, s->ny, s->nzl, s->d_spec, d_phi, s->twx, s->postx, s->normfft, 0, s->nsm, s->d_err);
    else
        launch_fft_x_c2r(st, s->nx, s->ny, s->nzl * s->ny, s->d_spec, d_phi, s->plx, s->twx, s->postx, s->normfft, 0);
    return slab_finish("paratc_slab_backward");
}

extern "C" double* paratc_slab_xslab(paratc_slab* s) { return s ? reinterpret_cast<double*>(s->d_xslab) : nullptr; }

static int slab_peers(const paratc_slab* s, const double* const* xslabs, SlabPeers& pp) {
    if (!xslabs) return PARATC_ERR_BAD_ARG;
    for (int q = 0; q < s->nranks; q++) {
        if (!xslabs[q] || !aligned16(xslabs[q])) return PARATC_ERR_BAD_ARG;
        pp.p[q] = const_cast<double2*>(reinterpret_cast<const double2*>(xslabs[q]));
    }
    return PARATC_OK;
}

extern "C" int paratc_slab_forward_peers(paratc_slab* s, const double* d_src, const double* const* xslabs,
                                         void* stream) {
    SlabPeers pp{};
    if (!s || !d_src || slab_peers(s, xslabs, pp) != PARATC_OK) return PARATC_ERR_BAD_ARG;
    cudaSetDevice(s->dev);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->nzl * s->ny * s->M1;
    if (s->xt && aligned16(d_src)) {
        // transform and scatter in one kernel: the modes leave shared memory
        // straight for their owners' x-slabs
        XtGather gt{};
        for (int q = 0; q < s->nranks; q++) gt.p[q] = pp.p[q];
        gt.G = s->nranks;
        gt.k0 = s->k0;
        launch_xf_tma_scatter(st, s->nx, s->ny, s->nzl, d_src, gt, s->twx, s->postx, s->nsm, s->d_err);
    } else {
        launch_fft_x_r2c(st, s->nx, s->nzl * s->ny, d_src, s->d_spec, s->plx, s->twx, s->postx);
        k_slab_scatter<<<grid_blocks(n, s->nsm), 256, 0, st>>>(0, s->nzl, s->ny, s->M1, s->nranks, s->k0, s->d_spec,
                                                               pp);
    }
    return slab_finish("paratc_slab_forward_peers");
}

extern "C" int paratc_slab_backward_peers(paratc_slab* s, const double* const* xslabs, double* d_phi, void* stream) {
    SlabPeers pp{};
    if (!s || !d_phi || slab_peers(s, xslabs, pp) != PARATC_OK) return PARATC_ERR_BAD_ARG;
    cudaSetDevice(s->dev);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)s->nzl * s->ny * s->M1;
    if (s->xt && aligned16(d_phi)) {
        // the inverse x transform loads its rows' segments straight from the
        // x-slabs (bulk copies, peer memory included): gather and transform
        // in one kernel
        XtGather gt{};
        for (int q = 0; q < s->nranks; q++) gt.p[q] = pp.p[q];
        gt.G = s->nranks;
        gt.k0 = s->k0;
        launch_xb_tma_gather(st, s->nx, s->ny, s->nzl, gt, d_phi, s->twx, s->postx, s->normfft, s->nsm, s->d_err);
    } else {
        k_slab_scatter<<<grid_blocks(n, s->nsm), 256, 0, st>>>(1, s->nzl, s->ny, s->M1, s->nranks, s->k0, s->d_spec,
                                                               pp);
        launch_fft_x_c2r(st, s->nx, s->ny, s->nzl * s->ny, s->d_spec, d_phi, s->plx, s->twx, s->postx, s->normfft, 0);
    }
    return slab_finish("paratc_slab_backward_peers");
}

extern "C" int paratc_ipc_get_handle(const void* d_ptr, void* handle) {
    if (!d_ptr || !handle) return PARATC_ERR_BAD_ARG;
    cudaIpcMemHandle_t h;
    const cudaError_t e = cudaIpcGetMemHandle(&h, const_cast<void*>(d_ptr));
    if (e != cudaSuccess) {
        std::fprintf(stderr, "paratc_ipc_get_handle: %s\n", cudaGetErrorString(e));
        return PARATC_ERR_CUDA;
    }
    static_assert(sizeof(h) <= PARATC_IPC_HANDLE_BYTES, "IPC handle size");
    std::memcpy(handle, &h, sizeof(h));
    return PARATC_OK;
}

extern "C" int paratc_ipc_open(const void* handle, void** d_ptr) {
    if (!handle || !d_ptr) return PARATC_ERR_BAD_ARG;
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle, sizeof(h));
    const cudaError_t e = cudaIpcOpenMemHandle(d_ptr, h, cudaIpcMemLazyEnablePeerAccess);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "paratc_ipc_open: %s\n", cudaGetErrorString(e));
        return PARATC_ERR_CUDA;
    }
    return PARATC_OK;
}

extern "C" int paratc_ipc_close(void* d_ptr) {
    if (!d_ptr) return PARATC_ERR_BAD_ARG;
    return cudaIpcCloseMemHandle(d_ptr) == cudaSuccess ? PARATC_OK : PARATC_ERR_CUDA;
}

extern "C" int paratc_slab_sync(paratc_slab* s, void* stream) {
    if (!s) return PARATC_ERR_BAD_ARG;
    cudaSetDevice(s->dev);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned int err = 0;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(&err, s->d_err, sizeof(err), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        std::fprintf(stderr, "paratc_slab_sync: %s\n", cudaGetErrorString(e));
        return PARATC_ERR_CUDA;
    }
    return err ? PARATC_ERR_TIMEOUT : PARATC_OK;
}
