// k_stencil.cu -- explicit stencils of the ParaTC substep on B200.
//
// One thread per cell, x fastest (coalesced 256-byte rows of doubles); the
// interpolated face velocities that clcRhsXYZ stores in six halo'd arrays
// (src/m_TScheme.f90:143-167) are recomputed in registers from the raw
// fields, so they never touch HBM.  The x/z periodic halos of the reference
// are index wrap (see common.cuh).  Reductions are per-block tree reductions
// followed by one single-block pass in a fixed order, so every result is
// bitwise reproducible run to run.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "reduce.cuh"

namespace ptc {

#define LD(A, off) __ldg(&(A)[off])

// ---------------------------------------------------------------------------
// clcPrSrc (src/m_TScheme.f90:48-77) / CheckDivergence (src/m_Tools.f90:54-81)
// src is the compact interior array (k, j-1, i); scale = 1/pmAlpha, or 1
// ---------------------------------------------------------------------------
template <class V>
__global__ void __launch_bounds__(256) k_prsrc(DConst c, DMetric m, const DCoef* __restrict__ coef, int unit_scale,
                                               const V* __restrict__ ux, const V* __restrict__ uy,
                                               const V* __restrict__ uz, double* __restrict__ src,
                                               double* __restrict__ part) {
    const int nx = c.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int jc = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z;
    double dm[1] = {0.0};
    if (i < nx && jc <= c.ny) {
        const size_t pl = (size_t)c.nyt * nx;
        const size_t r0 = (size_t)jc * nx;
        const size_t zc = (size_t)k * pl;
        const int im = wrapi(i - 1, nx), ip = wrapi(i + 1, nx), iu = wrapi(i + 2, nx);
        const size_t zm = (size_t)wrapi(k - 1, c.nz) * pl, zp = (size_t)wrapi(k + 1, c.nz) * pl, zu = (size_t)wrapi(k + 2, c.nz) * pl;
        const double dudx = c.dxC[0] * LD(ux, zc + r0 + im) + c.dxC[1] * LD(ux, zc + r0 + i) + c.dxC[2] * LD(ux, zc + r0 + ip) + c.dxC[3] * LD(ux, zc + r0 + iu);
        const double dvdy = (LD(uy, zc + r0 + nx + i) - LD(uy, zc + r0 + i)) * __ldg(&m.rdyp[jc]);
        const double dwdz = c.dzC[0] * LD(uz, zm + r0 + i) + c.dzC[1] * LD(uz, zc + r0 + i) + c.dzC[2] * LD(uz, zp + r0 + i) + c.dzC[3] * LD(uz, zu + r0 + i);
        const double rdiv = dudx + dvdy + dwdz;
        dm[0] = fabs(rdiv);
        if (src) {
            const double sudtal = unit_scale ? 1.0 : 1.0 / coef->pmAlpha;
            src[((size_t)k * c.ny + (jc - 1)) * nx + i] = sudtal * rdiv;
        }
    }
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_max_store<1>(dm, part + bid);
}

__global__ void k_reduce_max(const double* __restrict__ part, int nparts, double* __restrict__ out) {
    double v[1];
    reduce_parts<1, true>(part, nparts, v);
    if (threadIdx.x == 0) *out = v[0];
}

// ---------------------------------------------------------------------------
// FluidVelUpdate + PressureUpdate + SetBC_and_UpdateHalo(_pr)
// (src/m_TScheme.f90:82-107,512-532; src/m_BC_and_Halo.f90:23-64,108-122)
// mode 0: substep; mode 1: pressure-free projection (alpha = 1, p untouched)
// ---------------------------------------------------------------------------
// G: the block this CTA works as (OwnGrid, or SubGrid in a grouped launch)
// KZ: z planes per thread (1; the grouped launch takes 4, so that a thread
// reads its member's constants once for four cells)
template <class V, int KZ = 1, class G>
__device__ __forceinline__ void project_body(const G& grid, const DConst& c, const DMetric& m,
                                             const DCoef* __restrict__ coef, int mode, const V* __restrict__ phi,
                                             V* __restrict__ ux, V* __restrict__ uy, V* __restrict__ uz,
                                             double* __restrict__ pr, const double* __restrict__ uy_ym) {
    const int nx = c.nx;
    const int i = grid.x() * blockDim.x + threadIdx.x;
    const int jc = grid.y() * blockDim.y + threadIdx.y + 1;
    pdl_wait();
    if (i >= nx || jc > c.ny) return;
    const double alpha = mode == 0 ? coef->pmAlpha : 1.0;
#pragma unroll
    for (int kk = 0; kk < KZ; kk++) {
    const int k = grid.z() * KZ + kk;
    if (KZ > 1 && k >= c.nz) break;
    const size_t pl = (size_t)c.nyt * nx;
    const size_t r0 = (size_t)jc * nx, zc = (size_t)k * pl;
    const int is = wrapi(i - 2, nx), im = wrapi(i - 1, nx), ip = wrapi(i + 1, nx);
    const size_t zs = (size_t)wrapi(k - 2, c.nz) * pl, zm = (size_t)wrapi(k - 1, c.nz) * pl, zp = (size_t)wrapi(k + 1, c.nz) * pl;
    const size_t q = zc + r0 + i;
    const double pc = LD(phi, q), pjm = LD(phi, q - nx), pjp = LD(phi, q + nx);  // in FP64 from either storage
    const double dpdx = c.dxC[0] * LD(phi, zc + r0 + is) + c.dxC[1] * LD(phi, zc + r0 + im) + c.dxC[2] * pc + c.dxC[3] * LD(phi, zc + r0 + ip);
    const double dpdy = (pc - pjm) * __ldg(&m.rdyc[jc]);
    const double dpdz = c.dzC[0] * LD(phi, zs + r0 + i) + c.dzC[1] * LD(phi, zm + r0 + i) + c.dzC[2] * pc + c.dzC[3] * LD(phi, zp + r0 + i);
    const double uxn = ux[q] - alpha * dpdx;
    double uyn = uy[q] - alpha * dpdy;
    const double uzn = uz[q] - alpha * dpdz;
    const bool ft_ch = (c.flow_type == 1);
    if (jc == 1) uyn = uy_ym[(size_t)k * nx + i];
    ux[q] = uxn;
    uy[q] = uyn;
    uz[q] = uzn;
    if (jc == 1) {
        ux[q - nx] = c.uxbc_ym * 2.0 - uxn;
        uz[q - nx] = c.uzbc_ym * 2.0 - uzn;
    }
    if (jc == c.ny) {
        ux[q + nx] = ft_ch ? c.uxbc_yp * 2.0 - uxn : uxn;
        uy[q + nx] = ft_ch ? c.uybc_yp : 0.0;
        uz[q + nx] = ft_ch ? c.uzbc_yp * 2.0 - uzn : uzn;
    }
    if (mode == 0) {
        const double beta = coef->pmBeta;
        const double bp = -(beta * __ldg(&m.ap2ph[jc]));
        const double bc = -(beta * __ldg(&m.ac2ph[jc])) + 1.0;
        const double bm = -(beta * __ldg(&m.am2ph[jc]));
        const double pn = pr[q] + bp * pjp + bc * pc + bm * pjm;
        pr[q] = pn;
        if (jc == 1) pr[q - nx] = pn;
        if (jc == c.ny) pr[q + nx] = pn;
    }
    }
}

// z planes per thread of the one-context projection (2 measured slower at
// C1: 0.596 of the HBM peak against 0.648)
constexpr int PROJ_KZ1 = 1;
template <class V>
__global__ void __launch_bounds__(256) k_project(DConst c, DMetric m, const DCoef* __restrict__ coef, int mode,
                                                 const V* __restrict__ phi, V* __restrict__ ux,
                                                 V* __restrict__ uy, V* __restrict__ uz,
                                                 double* __restrict__ pr, const double* __restrict__ uy_ym) {
    project_body<V, PROJ_KZ1>(OwnGrid{}, c, m, coef, mode, phi, ux, uy, uz, pr, uy_ym);
}

// The one-context projection with two x-adjacent cells per thread (nx even):
// the cells' loads and stores move as pairs at an even index (float2 /
// double2), so a thread issues 12 loads for two cells instead of 13 per
// cell, and the x taps of the pair share two of their five values.  Every
// cell's arithmetic is project_body's, in the same order, so the two kernels
// give the same bits.
namespace {
__device__ __forceinline__ double2 ld_pv(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ double2 ld_pv(const float* p) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    return make_double2(v.x, v.y);
}
}  // namespace

template <class V>
__global__ void __launch_bounds__(256) k_project2(DConst c, DMetric m, const DCoef* __restrict__ coef, int mode,
                                                  const V* __restrict__ phi, V* __restrict__ ux, V* __restrict__ uy,
                                                  V* __restrict__ uz, double* __restrict__ pr,
                                                  const double* __restrict__ uy_ym) {
    const int nx = c.nx;
    const int i = 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int jc = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z;
    pdl_wait();
    if (i >= nx || jc > c.ny) return;
    const double alpha = mode == 0 ? coef->pmAlpha : 1.0;
    const size_t pl = (size_t)c.nyt * nx;
    const size_t r0 = (size_t)jc * nx, zc = (size_t)k * pl;
    const size_t zs = (size_t)wrapi(k - 2, c.nz) * pl, zm = (size_t)wrapi(k - 1, c.nz) * pl, zp = (size_t)wrapi(k + 1, c.nz) * pl;
    const size_t q = zc + r0 + i;
    // phi at i-2 .. i+3 of the row (pairs at even indices, wrapped), and the pair's y and z neighbours
    const double2 xm = ld_pair(phi + zc + r0 + wrapi(i - 2, nx));
    const double2 x0 = ld_pair(phi + q);
    const double2 xp = ld_pair(phi + zc + r0 + wrapi(i + 2, nx));
    const double2 ym = ld_pair(phi + q - nx), yp = ld_pair(phi + q + nx);
    const double2 z2 = ld_pair(phi + zs + r0 + i), z1 = ld_pair(phi + zm + r0 + i), z3 = ld_pair(phi + zp + r0 + i);
    const double2 u0 = ld_pv(ux + q), v0 = ld_pv(uy + q), w0 = ld_pv(uz + q);
    const double rdyc = __ldg(&m.rdyc[jc]);
    // cell i: x taps i-2, i-1, i, i+1; cell i+1: i-1, i, i+1, i+2
    const double pc[2] = {x0.x, x0.y}, pjm[2] = {ym.x, ym.y}, pjp[2] = {yp.x, yp.y};
    const double ps[2] = {xm.x, xm.y}, pm[2] = {xm.y, x0.x}, pp[2] = {x0.y, xp.x};
    const double zsv[2] = {z2.x, z2.y}, zmv[2] = {z1.x, z1.y}, zpv[2] = {z3.x, z3.y};
    const double uv[2] = {u0.x, u0.y}, vv[2] = {v0.x, v0.y}, wv[2] = {w0.x, w0.y};
    double uxn[2], uyn[2], uzn[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const double dpdx = c.dxC[0] * ps[h] + c.dxC[1] * pm[h] + c.dxC[2] * pc[h] + c.dxC[3] * pp[h];
        const double dpdy = (pc[h] - pjm[h]) * rdyc;
        const double dpdz = c.dzC[0] * zsv[h] + c.dzC[1] * zmv[h] + c.dzC[2] * pc[h] + c.dzC[3] * zpv[h];
        uxn[h] = uv[h] - alpha * dpdx;
        uyn[h] = vv[h] - alpha * dpdy;
        uzn[h] = wv[h] - alpha * dpdz;
    }
    const bool ft_ch = (c.flow_type == 1);
    if (jc == 1) {
        const double2 w = *reinterpret_cast<const double2*>(uy_ym + (size_t)k * nx + i);
        uyn[0] = w.x;
        uyn[1] = w.y;
    }
    st_pair(ux + q, make_double2(uxn[0], uxn[1]));
    st_pair(uy + q, make_double2(uyn[0], uyn[1]));
    st_pair(uz + q, make_double2(uzn[0], uzn[1]));
    if (jc == 1) {
        st_pair(ux + q - nx, make_double2(c.uxbc_ym * 2.0 - uxn[0], c.uxbc_ym * 2.0 - uxn[1]));
        st_pair(uz + q - nx, make_double2(c.uzbc_ym * 2.0 - uzn[0], c.uzbc_ym * 2.0 - uzn[1]));
    }
    if (jc == c.ny) {
        st_pair(ux + q + nx, ft_ch ? make_double2(c.uxbc_yp * 2.0 - uxn[0], c.uxbc_yp * 2.0 - uxn[1])
                                   : make_double2(uxn[0], uxn[1]));
        st_pair(uy + q + nx, ft_ch ? make_double2(c.uybc_yp, c.uybc_yp) : make_double2(0.0, 0.0));
        st_pair(uz + q + nx, ft_ch ? make_double2(c.uzbc_yp * 2.0 - uzn[0], c.uzbc_yp * 2.0 - uzn[1])
                                   : make_double2(uzn[0], uzn[1]));
    }
    if (mode == 0) {
        const double beta = coef->pmBeta;
        const double bp = -(beta * __ldg(&m.ap2ph[jc]));
        const double bc = -(beta * __ldg(&m.ac2ph[jc])) + 1.0;
        const double bm = -(beta * __ldg(&m.am2ph[jc]));
        const double2 p0 = *reinterpret_cast<const double2*>(pr + q);
        const double2 pn = make_double2(p0.x + bp * pjp[0] + bc * pc[0] + bm * pjm[0],
                                        p0.y + bp * pjp[1] + bc * pc[1] + bm * pjm[1]);
        st_pair(pr + q, pn);
        if (jc == 1) st_pair(pr + q - nx, pn);
        if (jc == c.ny) st_pair(pr + q + nx, pn);
    }
}

constexpr int PROJ_KZ = 4;
template <class V>
__global__ void __launch_bounds__(256) k_project_grp(const GrpTab<ProjArgs<V>>* __restrict__ t) {
    SubGrid g;
    const ProjArgs<V>& a = t->e[grp_member(t, g)];
    project_body<V, PROJ_KZ>(g, a.c, a.m, a.coef, 0, a.phi, a.ux, a.uy, a.uz, a.pr, a.uy_ym);
}

// ---------------------------------------------------------------------------
// ghost rows from the interior: SetBC_and_UpdateHalo, _pr and _scalar
// (src/m_BC_and_Halo.f90:23-178); one thread per (i, k)
// ---------------------------------------------------------------------------
template <class V>
__global__ void k_bc_all(DConst c, V* __restrict__ ux, V* __restrict__ uy, V* __restrict__ uz,
                         double* __restrict__ pr, V* __restrict__ sc, const double* __restrict__ uy_ym) {
    const int nx = c.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= nx) return;
    const size_t pl = (size_t)c.nyt * nx, zc = (size_t)k * pl;
    const size_t g0 = zc + i, r1 = zc + nx + i, rn = zc + (size_t)c.ny * nx + i, gt = zc + (size_t)c.nyp * nx + i;
    const bool ft_ch = (c.flow_type == 1);
    ux[gt] = (V)(ft_ch ? c.uxbc_yp * 2.0 - (double)ux[rn] : (double)ux[rn]);
    uy[gt] = (V)(ft_ch ? c.uybc_yp : 0.0);
    uz[gt] = (V)(ft_ch ? c.uzbc_yp * 2.0 - (double)uz[rn] : (double)uz[rn]);
    ux[g0] = (V)(c.uxbc_ym * 2.0 - (double)ux[r1]);
    uy[r1] = (V)uy_ym[(size_t)k * nx + i];
    uz[g0] = (V)(c.uzbc_ym * 2.0 - (double)uz[r1]);
    pr[g0] = pr[r1];
    pr[gt] = pr[rn];
    if (c.scalar_on && sc) {
        sc[g0] = (V)(c.sc_r1b * (double)sc[r1] + c.sc_r2b);
        sc[gt] = (V)(c.sc_r1t * (double)sc[rn] + c.sc_r2t);
    }
}

// Update_uy_ym (src/m_FlowCase.f90:112-122): no transpiration
__global__ void k_update_uy_ym(int n, double* __restrict__ uy_ym, double* __restrict__ duy_ym) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double d = uy_ym[t];
    uy_ym[t] = 0.0;
    duy_ym[t] = uy_ym[t] - d;
}

// ---------------------------------------------------------------------------
// CalcMaxCFL (src/m_Tools.f90:24-49) and the dt choice of ChannelIterate
// (src/m_ChannelSystem.f90:93-100)
// ---------------------------------------------------------------------------
template <class V>
__global__ void __launch_bounds__(256) k_cfl(DConst c, DMetric m, const V* __restrict__ ux,
                                             const V* __restrict__ uy, const V* __restrict__ uz,
                                             double* __restrict__ part) {
    const int nx = c.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int jc = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z;
    double v[1] = {0.0};
    if (i < nx && jc <= c.ny) {
        const size_t pl = (size_t)c.nyt * nx, zc = (size_t)k * pl, r0 = (size_t)jc * nx;
        const size_t q = zc + r0 + i;
        const size_t zp = (size_t)wrapi(k + 1, c.nz) * pl;
        const int ip = wrapi(i + 1, nx);
        v[0] = fabs(LD(ux, q) + LD(ux, zc + r0 + ip)) * c.rdx + fabs(LD(uy, q) + LD(uy, q + nx)) * __ldg(&m.rdyp[jc]) +
               fabs(LD(uz, q) + LD(uz, zp + r0 + i)) * c.rdz;
    }
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_max_store<1>(v, part + bid);
}

__global__ void k_cfl_final(DConst c, DCoef* coef, const double* __restrict__ part, int nparts) {
    double v[1];
    reduce_parts<1, true>(part, nparts, v);
    if (threadIdx.x != 0) return;
    DCoef f = *coef;
    const double uddxmax = v[0] * 0.5;
    f.cflmp = uddxmax * f.dt;
    if (c.icfl == 1) {
        double dt = c.cflc / uddxmax;
        f.dt = fmin(dt, c.dt_max);
    } else {
        f.dt = c.dt_max;
    }
    *coef = f;
}

// ---------------------------------------------------------------------------
// End of a step, one pass over the velocity: CheckDivergence, CalcVmax,
// CalcUxAver / ClcMeanValue (src/m_Tools.f90:54-110,256-301) for the step's
// diagnostics and guards, and (next != 0) clcCFL (src/m_TScheme.f90:20-46)
// of the step that follows, which reads the same velocity.  A warp takes whole
// x rows (grid-stride over the (jc, k) rows, k fastest, one wave of CTAs); every CTA
// stores one record of 5 maxima and 3 sums and the last CTA to finish reduces
// the records in index order.  It first fills the diagnostics from this
// step's dt and CFL number, then writes the next step's: cflmp = uddxmax*dt
// with the dt just used, dt = min(cflc/uddxmax, dt_max) for iCFL = 1 (or
// dt_max), exactly as clcCFL would at the start of the next step.
// ---------------------------------------------------------------------------
constexpr int ENDSTEP_THREADS = 256;
constexpr int ENDSTEP_U = 4;

template <class V, class G>
__device__ __forceinline__ void endstep_body(const G& grid, const DConst& c, const DMetric& m, const V* __restrict__ ux,
                                             const V* __restrict__ uy, const V* __restrict__ uz,
                                             const V* __restrict__ sc, DCoef* __restrict__ coef,
                                             DDiag* __restrict__ diag, double* __restrict__ part,
                                             unsigned int* __restrict__ counter, int next) {
    const int nx = c.nx, ny = c.ny, nz = c.nz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = grid.gx() * (ENDSTEP_THREADS / 32);
    const size_t pl = (size_t)c.nyt * nx;
    double mx[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double sm[3] = {0.0, 0.0, 0.0};
    pdl_wait();
    pdl_trigger();
    for (int r = grid.x() * (ENDSTEP_THREADS / 32) + warp; r < ny * nz; r += nwarps) {
        // k fastest: the warps of a CTA take consecutive z planes of one row
        // jc, so the four w planes of dw/dz are shared through L1
        const int jm = r / nz, k = r - jm * nz, jc = jm + 1;
        const int km = k == 0 ? nz - 1 : k - 1, kp = k == nz - 1 ? 0 : k + 1, ku = kp == nz - 1 ? 0 : kp + 1;
        const size_t r0 = (size_t)jc * nx;
        const V* ur = ux + (size_t)k * pl + r0;
        const V* vr = uy + (size_t)k * pl + r0;
        const V* w1 = uz + (size_t)k * pl + r0;
        const V* w0 = uz + (size_t)km * pl + r0;
        const V* w2 = uz + (size_t)kp * pl + r0;
        const V* w3 = uz + (size_t)ku * pl + r0;
        const double rdyp = __ldg(&m.rdyp[jc]), dy = __ldg(&m.dyp[jc]);
        // one cell's contribution: a = ux(i-1), ux(i), ux(i+1), ux(i+2), uy(j),
        // uy(j+1), uz(k-1 .. k+2), scalar
        auto cell = [&](const double (&a)[11]) {
            const double u0 = a[1], up = a[2], v0 = a[4], vp = a[5], z1 = a[7], z2 = a[8];
            const double dudx = c.dxC[0] * a[0] + c.dxC[1] * u0 + c.dxC[2] * up + c.dxC[3] * a[3];
            const double dvdy = (vp - v0) * rdyp;
            const double dwdz = c.dzC[0] * a[6] + c.dzC[1] * z1 + c.dzC[2] * z2 + c.dzC[3] * a[9];
            mx[0] = nmax(mx[0], fabs(dudx + dvdy + dwdz));
            mx[1] = nmax(mx[1], fabs(u0));
            mx[2] = nmax(mx[2], fabs(v0));
            mx[3] = nmax(mx[3], fabs(z1));
            if (next) mx[4] = nmax(mx[4], fabs(u0 + up) * c.rdx + fabs(v0 + vp) * rdyp + fabs(z1 + z2) * c.rdz);
            sm[0] += u0 * dy;
            if (c.scalar_on) {
                const double s = a[10];
                sm[1] += dy * s;
                sm[2] += dy * s * s;
            }
        };
        if (nx % 2 == 0) {
            // nx even: two adjacent cells per lane and pair, every load a pair at
            // an even index (ux at i-2 .. i+3 in three pairs), ENDSTEP_U / 2
            // pairs per lane in flight
            constexpr int EP = ENDSTEP_U / 2;
            const V* sr = c.scalar_on ? sc + (size_t)k * pl + r0 : nullptr;
            for (int i0 = 0; i0 < nx; i0 += 64 * EP) {
                double2 t[EP][10];
#pragma unroll
                for (int u = 0; u < EP; u++) {
                    const int i = min(i0 + 2 * lane + 64 * u, nx - 2);
                    t[u][0] = ld_pair(ur + wrapi(i - 2, nx)); t[u][1] = ld_pair(ur + i); t[u][2] = ld_pair(ur + wrapi(i + 2, nx));
                    t[u][3] = ld_pair(vr + i); t[u][4] = ld_pair(vr + nx + i);
                    t[u][5] = ld_pair(w0 + i); t[u][6] = ld_pair(w1 + i); t[u][7] = ld_pair(w2 + i); t[u][8] = ld_pair(w3 + i);
                    t[u][9] = sr ? ld_pair(sr + i) : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < EP; u++) {
                    if (i0 + 2 * lane + 64 * u >= nx) continue;
                    const double a0[11] = {t[u][0].y, t[u][1].x, t[u][1].y, t[u][2].x, t[u][3].x, t[u][4].x,
                                           t[u][5].x, t[u][6].x, t[u][7].x, t[u][8].x, t[u][9].x};
                    const double a1[11] = {t[u][1].x, t[u][1].y, t[u][2].x, t[u][2].y, t[u][3].y, t[u][4].y,
                                           t[u][5].y, t[u][6].y, t[u][7].y, t[u][8].y, t[u][9].y};
                    cell(a0);
                    cell(a1);
                }
            }
            continue;
        }
        // nx odd: ENDSTEP_U cells per lane with every load issued before the arithmetic
        for (int i0 = 0; i0 < nx; i0 += 32 * ENDSTEP_U) {
            double a[ENDSTEP_U][11];
#pragma unroll
            for (int u = 0; u < ENDSTEP_U; u++) {
                const int i = min(i0 + lane + 32 * u, nx - 1);
                const int im = i == 0 ? nx - 1 : i - 1, ip = i == nx - 1 ? 0 : i + 1, iu = ip == nx - 1 ? 0 : ip + 1;
                a[u][0] = __ldg(&ur[im]); a[u][1] = __ldg(&ur[i]); a[u][2] = __ldg(&ur[ip]); a[u][3] = __ldg(&ur[iu]);
                a[u][4] = __ldg(&vr[i]); a[u][5] = __ldg(&vr[nx + i]);
                a[u][6] = __ldg(&w0[i]); a[u][7] = __ldg(&w1[i]); a[u][8] = __ldg(&w2[i]); a[u][9] = __ldg(&w3[i]);
                a[u][10] = c.scalar_on ? __ldg(&sc[(size_t)k * pl + r0 + i]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < ENDSTEP_U; u++) {
                if (i0 + lane + 32 * u >= nx) continue;
                cell(a[u]);
            }
        }
    }
    block_max_store<5>(mx, part + (size_t)grid.x() * 8);
    __syncthreads();
    block_sum_store<3>(sm, part + (size_t)grid.x() * 8 + 5);
    if (!last_block_arrive(counter, grid.gx())) return;
    // the last CTA: records in index order, thread t takes records t, t+256, ...
    __shared__ double sh[ENDSTEP_THREADS / 32][8];
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < (int)grid.gx(); b += ENDSTEP_THREADS) {
        const double* p = part + (size_t)b * 8;
#pragma unroll
        for (int q = 0; q < 5; q++) v[q] = nmax(v[q], __ldcg(&p[q]));
#pragma unroll
        for (int q = 5; q < 8; q++) v[q] += __ldcg(&p[q]);
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = q < 5 ? nmax(v[q], y) : v[q] + y;
        }
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 8; q++) sh[warp][q] = v[q];
    __syncthreads();
    if (threadIdx.x != 0) return;
    double r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int w = 0; w < ENDSTEP_THREADS / 32; w++)
        for (int q = 0; q < 8; q++) r[q] = q < 5 ? nmax(r[q], sh[w][q]) : r[q] + sh[w][q];
    DDiag d = *diag;
    DCoef f = *coef;
    d.step_counter += 1;
    d.dt = f.dt;
    d.cfl = f.cflmp;
    d.sim_time = f.sim_time;
    d.divmax_src = f.divmax_src;
    d.divmax = r[0];
    d.vmax[0] = r[1]; d.vmax[1] = r[2]; d.vmax[2] = r[3];
    d.pr_grad_aver = f.pr_grad_aver;
    const double nxz = (double)(c.nx * c.nz);
    d.ux_mean = r[5] / nxz / c.yly;
    d.sc_mean = r[6] / nxz / c.yly;
    d.sc2_mean = r[7] / nxz / c.yly;
    if (d.status == 0) {
        // the maxima keep a NaN (nmax) and |Inf| stays Inf, so one non-finite
        // value of u, v, w or div u anywhere makes one of these non-finite;
        // the sums catch a non-finite scalar.  ChannelIterate's own tests
        // (src/m_ChannelSystem.f90:143,145) follow: div_limit, then the
        // smallest of the three velocity maxima against vel_limit.
        bool finite = true;
        for (int q = 0; q < 8; q++) finite = finite && isfinite(r[q]);
        const double vmin = fmin(fmin(r[1], r[2]), r[3]);
        if (!finite) { d.status = -4; d.failed_step = d.step_counter; }
        else if (r[0] > c.div_limit) { d.status = -5; d.failed_step = d.step_counter; }
        else if (vmin > c.vel_limit) { d.status = -6; d.failed_step = d.step_counter; }
    }
    *diag = d;
    if (next) {
        const double uddxmax = r[4] * 0.5;
        f.dt_last = f.dt;
        f.cflmp = uddxmax * f.dt;
        f.dt = (c.icfl == 1) ? fmin(c.cflc / uddxmax, c.dt_max) : c.dt_max;
        *coef = f;
    }
}

template <class V>
__global__ void __launch_bounds__(ENDSTEP_THREADS, 2)
    k_endstep(DConst c, DMetric m, const V* __restrict__ ux, const V* __restrict__ uy,
              const V* __restrict__ uz, const V* __restrict__ sc, DCoef* __restrict__ coef,
              DDiag* __restrict__ diag, double* __restrict__ part, unsigned int* __restrict__ counter, int next) {
    endstep_body(OwnGrid{}, c, m, ux, uy, uz, sc, coef, diag, part, counter, next);
}

template <class V>
__global__ void __launch_bounds__(ENDSTEP_THREADS, 2) k_endstep_grp(const GrpTab<EndArgs<V>>* __restrict__ t) {
    SubGrid g;
    const EndArgs<V>& a = t->e[grp_member(t, g)];
    endstep_body(g, a.c, a.m, a.ux, a.uy, a.uz, a.sc, a.coef, a.diag, a.part, a.counter, 1);
}

// ---------------------------------------------------------------------------
// x profile of a field averaged over the depth and the span:
// prof(i) = sum_k sum_j q(i, j, k) dyp(j) / (nz * yly), the depth-averaged
// concentration whose 0.5 crossing is the front of a gravity current.  One
// thread per (i, k) sums its column over j in order; the second kernel adds
// the nz columns of an i in order, so the result is deterministic.
// ---------------------------------------------------------------------------
template <class V>
__global__ void k_xprof_part(DConst c, DMetric m, const V* __restrict__ q, double* __restrict__ part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= c.nx) return;
    const V* col = q + (size_t)k * c.nyt * c.nx + i;
    double s = 0.0;
    for (int j = 1; j <= c.ny; j++) s += __ldg(&col[(size_t)j * c.nx]) * __ldg(&m.dyp[j]);
    part[(size_t)k * c.nx + i] = s;
}

__global__ void k_xprof_final(DConst c, const double* __restrict__ part, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.nx) return;
    double s = 0.0;
    for (int k = 0; k < c.nz; k++) s += part[(size_t)k * c.nx + i];
    out[i] = s / (double)c.nz / c.yly;
}

// elementwise conversion between the storage precisions (round to nearest
// one way, exact the other), for loading and reading the FP32 storage form
template <class A, class B>
__global__ void k_cast(size_t n, const A* __restrict__ a, B* __restrict__ b) {
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        b[t] = (B)a[t];
}

// the residual of the discrete pressure Poisson equation r = src - L phi on
// compact arrays (k*ny + jc-1)*nx + i: L = D4x D4x + D4z D4z + Lyy, the
// operator whose eigenvalues the spectral solve inverts (D4 the 4th-order
// staggered first difference of clcPrSrc / FluidVelUpdate, so D4 D4 has the
// modified wavenumber of src/m_Poisson.f90:40-48 as its symbol; Lyy the
// Neumann wall-normal operator am2ph/ac2ph/ap2ph).  The spectral solve
// replaces the kx = kz = 0 equation of row 1 by phi_hat = 0
// (src/m_Poisson.f90:399-404); that equation's residual is the plane mean of
// r at row 1, nonzero whenever the source's dy-weighted mean is, and it is
// removed (k_resid_row1) so that the corrections see only the equations the
// solve keeps.  The same pinned equation fixes the additive constant of phi
// (the plane mean of phi at row 1 is zero); out[3] receives that mean of the
// current phi, which the next correction subtracts (a constant is invisible
// to the residual, and FP32 rounding in the inverse transforms shifts it).
// Record per CTA: max|r| over rows 2..ny, max|src|, and the sums of r and
// phi over its row-1 cells; the last CTA writes out[0] = max|r| (rows
// 2..ny), out[1] = max|src|, out[2], out[3] = the row-1 plane means of r, phi.
__global__ void __launch_bounds__(256) k_residual(DConst c, DMetric m, const double* __restrict__ src,
                                                  const double* __restrict__ phi, double* __restrict__ r,
                                                  double* __restrict__ part, unsigned int* __restrict__ counter,
                                                  double* __restrict__ out) {
    const int nx = c.nx, ny = c.ny, nz = c.nz;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int jc = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z;
    // the 7-point D4 D4 weights of offsets -3..3 (a face derivative of cell
    // values, then the cell derivative of face values)
    double wx[7], wz[7];
#pragma unroll
    for (int q = 0; q < 7; q++) { wx[q] = 0.0; wz[q] = 0.0; }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
            wx[a + b] += c.dxC[a] * c.dxC[b];
            wz[a + b] += c.dzC[a] * c.dzC[b];
        }
    double v[2] = {0.0, 0.0}, s1[2] = {0.0, 0.0};
    if (i < nx && jc <= ny) {
        const size_t row = (size_t)ny * nx;
        const double* pk = phi + (size_t)k * row + (size_t)(jc - 1) * nx;
        double lx = 0.0, lz = 0.0;
#pragma unroll
        for (int q = 0; q < 7; q++) {
            lx += wx[q] * __ldg(&pk[wrapi(i - 3 + q, nx)]);
            const int kq = ((k - 3 + q) % nz + nz) % nz;
            lz += wz[q] * __ldg(&phi[(size_t)kq * row + (size_t)(jc - 1) * nx + i]);
        }
        const double pc = __ldg(&pk[i]);
        double ly = __ldg(&m.ac2ph[jc]) * pc;
        if (jc > 1) ly += __ldg(&m.am2ph[jc]) * __ldg(&pk[i - nx]);
        if (jc < ny) ly += __ldg(&m.ap2ph[jc]) * __ldg(&pk[i + nx]);
        const size_t q0 = (size_t)k * row + (size_t)(jc - 1) * nx + i;
        const double s = __ldg(&src[q0]);
        const double res = s - (lx + lz + ly);
        r[q0] = res;
        if (jc == 1) { s1[0] = res; s1[1] = pc; }
        else v[0] = fabs(res);
        v[1] = fabs(s);
    }
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_max_store<2>(v, part + (size_t)bid * 2);
    __syncthreads();
    block_sum_store<2>(s1, part + (size_t)nb * 2 + (size_t)bid * 2);
    if (!last_block_arrive(counter, nb)) return;
    double tot[2], sum[2];
    reduce_records<2, true>(part, (int)nb, tot);
    reduce_records<2, false>(part + (size_t)nb * 2, (int)nb, sum);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
        out[2] = sum[0] / ((double)nx * (double)nz);
        out[3] = sum[1] / ((double)nx * (double)nz);
    }
}

// row 1 of the residual minus its plane mean (the dropped kx = kz = 0
// equation), and out[0] = max(out[0], max|r| of the corrected row 1)
__global__ void __launch_bounds__(256) k_resid_row1(DConst c, double* __restrict__ r, double* __restrict__ part,
                                                    unsigned int* __restrict__ counter, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = c.nx;
    double v[1] = {0.0};
    if (t < nx * c.nz) {
        const int k = t / nx, i = t - k * nx;
        double* q = r + (size_t)k * c.ny * nx + i;
        const double x = *q - out[2];
        *q = x;
        v[0] = fabs(x);
    }
    block_max_store<1>(v, part + blockIdx.x);
    if (!last_block_arrive(counter, gridDim.x)) return;
    double tot[1];
    reduce_records<1, true>(part, (int)gridDim.x, tot);
    if (threadIdx.x == 0) out[0] = nmax(out[0], tot[0]);
}

__global__ void k_store_divsrc(DCoef* coef, const double* __restrict__ v) {
    if (threadIdx.x == 0) coef->divmax_src = *v;
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static dim3 cell_block() { return dim3(32, 8, 1); }
static dim3 cell_grid(const DConst& c) { return dim3((c.nx + 31) / 32, (c.ny + 7) / 8, c.nz); }

size_t cell_grid_blocks(const DConst& c) {
    dim3 g = cell_grid(c);
    return (size_t)g.x * g.y * g.z;
}

template <class V>
static void prsrc_t(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int unit_scale,
                    const FieldSet<V>& f, double* src, double* part, double* out_max) {
    k_prsrc<V><<<cell_grid(c), cell_block(), 0, st>>>(c, m, coef, unit_scale, f.ux, f.uy, f.uz, src, part);
    k_reduce_max<<<1, 1024, 0, st>>>(part, (int)cell_grid_blocks(c), out_max);
}
void launch_prsrc(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int unit_scale,
                  const Fields& f, double* src, double* part, double* out_max) {
    prsrc_t(st, c, m, coef, unit_scale, f, src, part, out_max);
}
void launch_prsrc(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int unit_scale,
                  const Fields32& f, double* src, double* part, double* out_max) {
    prsrc_t(st, c, m, coef, unit_scale, f, src, part, out_max);
}

void launch_store_divsrc(cudaStream_t st, DCoef* coef, const double* v) { k_store_divsrc<<<1, 32, 0, st>>>(coef, v); }

static dim3 project_grid(const DConst& c) {
    const dim3 g = cell_grid(c);
    return dim3(g.x, g.y, (g.z + PROJ_KZ1 - 1) / PROJ_KZ1);
}
// two cells per thread where nx is even (k_project2), one otherwise
template <class V>
static void project_t(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int mode, const V* phi,
                      const FieldSet<V>& f, const double* uy_ym) {
    if (c.nx % 2 == 0)
        launch_pdl(k_project2<V>, dim3((c.nx + 63) / 64, (c.ny + 7) / 8, c.nz), cell_block(), 0, st, c, m, coef, mode,
                   phi, f.ux, f.uy, f.uz, f.pr, uy_ym);
    else
        launch_pdl(k_project<V>, project_grid(c), cell_block(), 0, st, c, m, coef, mode, phi, f.ux, f.uy, f.uz, f.pr,
                   uy_ym);
}
void launch_project(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int mode, const double* phi,
                    const Fields& f, const double* uy_ym) {
    project_t(st, c, m, coef, mode, phi, f, uy_ym);
}
void launch_project(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int mode, const float* phi,
                    const Fields32& f, const double* uy_ym) {
    project_t(st, c, m, coef, mode, phi, f, uy_ym);
}

void launch_bc_all(cudaStream_t st, const DConst& c, const Fields& f, const double* uy_ym) {
    k_bc_all<double><<<dim3((c.nx + 127) / 128, c.nz), 128, 0, st>>>(c, f.ux, f.uy, f.uz, f.pr, f.sc, uy_ym);
}
void launch_bc_all(cudaStream_t st, const DConst& c, const Fields32& f, const double* uy_ym) {
    k_bc_all<float><<<dim3((c.nx + 127) / 128, c.nz), 128, 0, st>>>(c, f.ux, f.uy, f.uz, f.pr, f.sc, uy_ym);
}

void launch_update_uy_ym(cudaStream_t st, int n, double* uy_ym, double* duy_ym) {
    k_update_uy_ym<<<(n + 255) / 256, 256, 0, st>>>(n, uy_ym, duy_ym);
}

template <class V>
static void cfl_t(cudaStream_t st, const DConst& c, const DMetric& m, const FieldSet<V>& f, DCoef* coef, double* part) {
    k_cfl<V><<<cell_grid(c), cell_block(), 0, st>>>(c, m, f.ux, f.uy, f.uz, part);
    k_cfl_final<<<1, 1024, 0, st>>>(c, coef, part, (int)cell_grid_blocks(c));
}
void launch_cfl(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, DCoef* coef, double* part) {
    cfl_t(st, c, m, f, coef, part);
}
void launch_cfl(cudaStream_t st, const DConst& c, const DMetric& m, const Fields32& f, DCoef* coef, double* part) {
    cfl_t(st, c, m, f, coef, part);
}

template <class V>
static void xprofile_t(cudaStream_t st, const DConst& c, const DMetric& m, const V* q, double* part, double* out) {
    k_xprof_part<V><<<dim3((c.nx + 127) / 128, c.nz), 128, 0, st>>>(c, m, q, part);
    k_xprof_final<<<(c.nx + 127) / 128, 128, 0, st>>>(c, part, out);
}
void launch_xprofile(cudaStream_t st, const DConst& c, const DMetric& m, const double* q, double* part, double* out) {
    xprofile_t(st, c, m, q, part, out);
}
void launch_xprofile(cudaStream_t st, const DConst& c, const DMetric& m, const float* q, double* part, double* out) {
    xprofile_t(st, c, m, q, part, out);
}

void launch_cast(cudaStream_t st, size_t n, const double* a, float* b) {
    k_cast<double, float><<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, st>>>(n, a, b);
}
void launch_cast(cudaStream_t st, size_t n, const float* a, double* b) {
    k_cast<float, double><<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, st>>>(n, a, b);
}

void launch_residual(cudaStream_t st, const DConst& c, const DMetric& m, const double* src, const double* phi,
                     double* r, double* part, unsigned int* counter, double* out) {
    k_residual<<<cell_grid(c), cell_block(), 0, st>>>(c, m, src, phi, r, part, counter, out);
    k_resid_row1<<<(c.nx * c.nz + 255) / 256, 256, 0, st>>>(c, r, part, counter, out);
}

size_t endstep_blocks(const DConst& c) { return (size_t)2 * (c.nsm > 0 ? c.nsm : 148); }

// grouped launches (one member's shape: its own launch's)
dim3 cell_member_grid(const DConst& c) {
    const dim3 g = cell_grid(c);
    return dim3(g.x, g.y, (g.z + PROJ_KZ - 1) / PROJ_KZ);  // the grouped projection's shape
}
dim3 endstep_member_grid(const DConst& c) { return dim3((unsigned)endstep_blocks(c)); }
void launch_project_grp(cudaStream_t st, const GrpTab<ProjArgs<double>>* t, int nblk) {
    launch_pdl(k_project_grp<double>, dim3((unsigned)nblk), cell_block(), 0, st, t);
}
void launch_project_grp(cudaStream_t st, const GrpTab<ProjArgs<float>>* t, int nblk) {
    launch_pdl(k_project_grp<float>, dim3((unsigned)nblk), cell_block(), 0, st, t);
}
void launch_endstep_grp(cudaStream_t st, const GrpTab<EndArgs<double>>* t, int nblk) {
    launch_pdl(k_endstep_grp<double>, dim3((unsigned)nblk), dim3(ENDSTEP_THREADS), 0, st, t);
}
void launch_endstep_grp(cudaStream_t st, const GrpTab<EndArgs<float>>* t, int nblk) {
    launch_pdl(k_endstep_grp<float>, dim3((unsigned)nblk), dim3(ENDSTEP_THREADS), 0, st, t);
}

void launch_endstep(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, DCoef* coef, DDiag* diag,
                    double* part, unsigned int* counter, int next) {
    launch_pdl(k_endstep<double>, dim3((unsigned)endstep_blocks(c)), dim3(ENDSTEP_THREADS), 0, st, c, m, f.ux, f.uy,
               f.uz, f.sc, coef, diag, part, counter, next);
}
void launch_endstep(cudaStream_t st, const DConst& c, const DMetric& m, const Fields32& f, DCoef* coef, DDiag* diag,
                    double* part, unsigned int* counter, int next) {
    launch_pdl(k_endstep<float>, dim3((unsigned)endstep_blocks(c)), dim3(ENDSTEP_THREADS), 0, st, c, m, f.ux, f.uy,
               f.uz, f.sc, coef, diag, part, counter, next);
}

}  // namespace ptc
