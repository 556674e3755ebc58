// k_stencil.cu -- explicit stencils of the ParaTC substep on B200.
//
// One thread per cell, x fastest (coalesced 256-byte rows of doubles); the
// interpolated face velocities that clcRhsXYZ stores in six halo'd arrays
// (src/m_TScheme.f90:143-167) are recomputed in registers from the raw
// fields, so they never touch HBM.  The x/z periodic halos of the reference
// are index wrap (see common.cuh).  Reductions are per-block tree reductions
// followed by one single-block pass in a fixed order, so every result is
// bitwise reproducible run to run.
#include "common.cuh"
#include "kernels.cuh"

namespace ptc {

// ---------------------------------------------------------------------------
// block reductions (deterministic)
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double* __restrict__ out_block) {
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[wid][q] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = lane < nw ? sh[lane][q] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) out_block[q] = x;
        }
    }
}

template <int NV>
__device__ __forceinline__ void block_max_store(double (&v)[NV], double* __restrict__ out_block) {
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nthr + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] = fmax(v[q], __shfl_down_sync(0xffffffffu, v[q], o));
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[wid][q] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = lane < nw ? sh[lane][q] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
            if (lane == 0) out_block[q] = x;
        }
    }
}

// single-block reduction of nparts partial records of NV values, fixed order
template <int NV, bool MAX>
__device__ void reduce_parts(const double* __restrict__ parts, int nparts, double (&out)[NV]) {
    __shared__ double sh[32][NV];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = (blockDim.x + 31) >> 5;
    double v[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = 0.0;
    for (int b = tid; b < nparts; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] = MAX ? fmax(v[q], parts[(size_t)b * NV + q]) : v[q] + parts[(size_t)b * NV + q];
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) {
            double y = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = MAX ? fmax(v[q], y) : v[q] + y;
        }
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[wid][q] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double x = 0.0;
        if (wid == 0) {
            x = lane < nw ? sh[lane][q] : 0.0;
            for (int o = 16; o > 0; o >>= 1) {
                double y = __shfl_down_sync(0xffffffffu, x, o);
                x = MAX ? fmax(x, y) : x + y;
            }
        }
        out[q] = x;  // valid in thread 0
    }
}

// ---------------------------------------------------------------------------
// PMcoeUpdate (src/m_Parameters.f90:215-230), one thread
// ---------------------------------------------------------------------------
__global__ void k_coef(DCoef* coef, int ns, double gam, double the, double alp, double xnu, double sdiff) {
    if (threadIdx.x != 0) return;
    DCoef c = *coef;
    const double dt = c.dt;
    c.pmGamma = gam * dt;
    c.pmTheta = the * dt;
    c.pmAlpha = alp * dt;
    c.pmBeta = 0.5 * alp * xnu * dt;
    c.pmBetaSc = 0.5 * alp * sdiff * dt;
    c.sim_time = c.sim_time + dt * alp;
    c.pmAlphaC = alp;
    if (ns == 1) c.pr_grad_aver = 0.0;
    c.rhsx_add = 0.0;
    c.ns = ns;
    *coef = c;
}

// ---------------------------------------------------------------------------
// clcRhsXYZ (src/m_TScheme.f90:113-360)
// ---------------------------------------------------------------------------
#define LD(A, off) __ldg(&(A)[off])

template <bool SCALAR>
__global__ void __launch_bounds__(256) k_rhs(DConst c, DMetric m, const DCoef* __restrict__ coef,
                                             const double* __restrict__ ux, const double* __restrict__ uy,
                                             const double* __restrict__ uz, const double* __restrict__ pr,
                                             const double* __restrict__ sc, double* __restrict__ hx,
                                             double* __restrict__ hy, double* __restrict__ hz,
                                             double* __restrict__ hc, double* __restrict__ rx,
                                             double* __restrict__ ry, double* __restrict__ rz,
                                             double* __restrict__ rc, double* __restrict__ part) {
    const int nx = c.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int jc = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z;
    double s3[1] = {0.0};
    if (i < nx && jc <= c.ny) {
        const double pmGamma = coef->pmGamma, pmTheta = coef->pmTheta, pmAlpha = coef->pmAlpha;
        const double tb = 2.0 * coef->pmBeta;
        const size_t pl = (size_t)c.nyt * nx;
        int xo[7];
        size_t zo[7];
#pragma unroll
        for (int d = 0; d < 7; d++) {
            xo[d] = wrapi(i + d - 3, nx);
            zo[d] = (size_t)wrapi(k + d - 3, c.nz) * pl;
        }
        const size_t r0 = (size_t)jc * nx, rm = r0 - nx, rp = r0 + nx;
#define AT(A, dx, row, dz) LD(A, zo[3 + (dz)] + (row) + xo[3 + (dx)])
        const double I1 = c.IC[0], I2 = c.IC[1], I3 = c.IC[2], I4 = c.IC[3];
        const double ucrf = c.ucrf, xnu = c.xnu;
        const bool top = (jc == c.ny);
        const double IY1 = __ldg(&m.yinterp[jc]), IY2 = 1.0 - IY1;
        const double IY3 = __ldg(&m.yinterp[jc + 1]), IY4 = 1.0 - IY3;
        const double rdyp = __ldg(&m.rdyp[jc]), rdyc = __ldg(&m.rdyc[jc]), dyp = __ldg(&m.dyp[jc]);
        const size_t q0 = zo[3] + r0 + i;

        // ---------------- RhsX (:169-204)
        double uxx[7], uxz[7];
#pragma unroll
        for (int d = 0; d < 7; d++) { uxx[d] = AT(ux, d - 3, r0, 0); uxz[d] = AT(ux, 0, r0, d - 3); }
        const double uxc = uxx[3], uxjm = AT(ux, 0, rm, 0), uxjp = AT(ux, 0, rp, 0);
        double conv_x, rhs_x;
        {
            const double uxhyc = IY1 * uxjm + IY2 * uxc;
            const double uxhyp = IY3 * uxc + IY4 * uxjp;
            double uxhx[4];
#pragma unroll
            for (int q = 0; q < 4; q++) uxhx[q] = I1 * uxx[q] + I2 * uxx[q + 1] + I3 * uxx[q + 2] + I4 * uxx[q + 3];
            const double h11 = c.dxC[0] * uxhx[0] * (uxhx[0] + ucrf) + c.dxC[1] * uxhx[1] * (uxhx[1] + ucrf) +
                               c.dxC[2] * uxhx[2] * (uxhx[2] + ucrf) + c.dxC[3] * uxhx[3] * (uxhx[3] + ucrf);
            const double uyhx_j = I1 * AT(uy, -2, r0, 0) + I2 * AT(uy, -1, r0, 0) + I3 * AT(uy, 0, r0, 0) + I4 * AT(uy, 1, r0, 0);
            const double uyhx_p = top ? 0.0 : I1 * AT(uy, -2, rp, 0) + I2 * AT(uy, -1, rp, 0) + I3 * AT(uy, 0, rp, 0) + I4 * AT(uy, 1, rp, 0);
            const double h12 = (uyhx_p * uxhyp - uyhx_j * uxhyc) * rdyp;
            double h13 = 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++) {  // z offsets -1..2
                const double uxhz = I1 * uxz[q] + I2 * uxz[q + 1] + I3 * uxz[q + 2] + I4 * uxz[q + 3];
                const double uzhx = I1 * AT(uz, -2, r0, q - 1) + I2 * AT(uz, -1, r0, q - 1) + I3 * AT(uz, 0, r0, q - 1) + I4 * AT(uz, 1, r0, q - 1);
                h13 = (q == 0) ? c.dzC[0] * uxhz * uzhx : h13 + c.dzC[q] * uxhz * uzhx;
            }
            const double d11 = c.dxxC[0] * uxx[1] + c.dxxC[1] * uxx[2] + c.dxxC[2] * uxx[3] + c.dxxC[3] * uxx[4] + c.dxxC[4] * uxx[5];
            const double d22 = __ldg(&m.ap2c[jc]) * uxjp + __ldg(&m.ac2c[jc]) * uxc + __ldg(&m.am2c[jc]) * uxjm;
            const double d33 = c.dzzC[0] * uxz[1] + c.dzzC[1] * uxz[2] + c.dzzC[2] * uxz[3] + c.dzzC[3] * uxz[4] + c.dzzC[4] * uxz[5];
            const double dcq13 = d11 + d33;
            s3[0] = SCALAR ? uxc * dyp : (dcq13 + d22) * dyp;
            conv_x = -h11 - h12 - h13 + xnu * dcq13 + c.grav[0];
            const double gradp = c.dxC[0] * AT(pr, -2, r0, 0) + c.dxC[1] * AT(pr, -1, r0, 0) + c.dxC[2] * AT(pr, 0, r0, 0) + c.dxC[3] * AT(pr, 1, r0, 0);
            rhs_x = pmGamma * conv_x + pmTheta * hx[q0] - pmAlpha * gradp + tb * d22;
        }

        // ---------------- RhsY (:206-236)
        double uyx[7], uyz[7];
#pragma unroll
        for (int d = 0; d < 7; d++) { uyx[d] = AT(uy, d - 3, r0, 0); uyz[d] = AT(uy, 0, r0, d - 3); }
        double conv_y, rhs_y;
        {
            const double qsucac = 0.25 * rdyc;
            double uxh[4], uzh[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {  // offsets -1..2
                uxh[q] = IY1 * AT(ux, q - 1, rm, 0) + IY2 * uxx[q + 2] + ucrf;
                uzh[q] = IY1 * AT(uz, 0, rm, q - 1) + IY2 * AT(uz, 0, r0, q - 1);
            }
            double h21 = 0.0, h23 = 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const double uyhx = I1 * uyx[q] + I2 * uyx[q + 1] + I3 * uyx[q + 2] + I4 * uyx[q + 3];
                const double uyhz = I1 * uyz[q] + I2 * uyz[q + 1] + I3 * uyz[q + 2] + I4 * uyz[q + 3];
                h21 = (q == 0) ? c.dxC[0] * uyhx * uxh[0] : h21 + c.dxC[q] * uyhx * uxh[q];
                h23 = (q == 0) ? c.dzC[0] * uyhz * uzh[0] : h23 + c.dzC[q] * uyhz * uzh[q];
            }
            const double vp = AT(uy, 0, rp, 0), vc = uyx[3], vm = AT(uy, 0, rm, 0);
            const double h22 = ((vp + vc) * (vp + vc) - (vc + vm) * (vc + vm)) * qsucac;
            const double d11 = c.dxxC[0] * uyx[1] + c.dxxC[1] * uyx[2] + c.dxxC[2] * uyx[3] + c.dxxC[3] * uyx[4] + c.dxxC[4] * uyx[5];
            const double d22 = __ldg(&m.ap2p[jc]) * vp + __ldg(&m.ac2p[jc]) * vc + __ldg(&m.am2p[jc]) * vm;
            const double d33 = c.dzzC[0] * uyz[1] + c.dzzC[1] * uyz[2] + c.dzzC[2] * uyz[3] + c.dzzC[3] * uyz[4] + c.dzzC[4] * uyz[5];
            conv_y = -h21 - h22 - h23 + xnu * (d11 + d33) + c.grav[1];
            const double gradp = (AT(pr, 0, r0, 0) - AT(pr, 0, rm, 0)) * rdyc;
            rhs_y = pmGamma * conv_y + pmTheta * hy[q0] - pmAlpha * gradp + tb * d22;
        }

        // ---------------- RhsZ (:238-267)
        double uzx[7], uzz[7];
#pragma unroll
        for (int d = 0; d < 7; d++) { uzx[d] = AT(uz, d - 3, r0, 0); uzz[d] = AT(uz, 0, r0, d - 3); }
        double conv_z, rhs_z;
        {
            const double uzc = uzx[3];
            const double uzhyc = IY1 * AT(uz, 0, rm, 0) + IY2 * uzc;
            const double uzhyp = IY3 * uzc + IY4 * AT(uz, 0, rp, 0);
            double h31 = 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++) {  // x offsets -1..2
                const double uzhx = I1 * uzx[q] + I2 * uzx[q + 1] + I3 * uzx[q + 2] + I4 * uzx[q + 3];
                const double uxhz = I1 * AT(ux, q - 1, r0, -2) + I2 * AT(ux, q - 1, r0, -1) + I3 * AT(ux, q - 1, r0, 0) + I4 * AT(ux, q - 1, r0, 1);
                h31 = (q == 0) ? c.dxC[0] * uzhx * (uxhz + ucrf) : h31 + c.dxC[q] * uzhx * (uxhz + ucrf);
            }
            const double uyhz_j = I1 * uyz[1] + I2 * uyz[2] + I3 * uyz[3] + I4 * uyz[4];
            const double uyhz_p = top ? 0.0 : I1 * AT(uy, 0, rp, -2) + I2 * AT(uy, 0, rp, -1) + I3 * AT(uy, 0, rp, 0) + I4 * AT(uy, 0, rp, 1);
            const double h32 = (uyhz_p * uzhyp - uyhz_j * uzhyc) * rdyp;
            double h33 = 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++) {  // z offsets -2..1
                const double uzhz = I1 * uzz[q] + I2 * uzz[q + 1] + I3 * uzz[q + 2] + I4 * uzz[q + 3];
                h33 = (q == 0) ? c.dzC[0] * uzhz * uzhz : h33 + c.dzC[q] * uzhz * uzhz;
            }
            const double d11 = c.dxxC[0] * uzx[1] + c.dxxC[1] * uzx[2] + c.dxxC[2] * uzx[3] + c.dxxC[3] * uzx[4] + c.dxxC[4] * uzx[5];
            const double d22 = __ldg(&m.ap2c[jc]) * AT(uz, 0, rp, 0) + __ldg(&m.ac2c[jc]) * uzc + __ldg(&m.am2c[jc]) * AT(uz, 0, rm, 0);
            const double d33 = c.dzzC[0] * uzz[1] + c.dzzC[1] * uzz[2] + c.dzzC[2] * uzz[3] + c.dzzC[3] * uzz[4] + c.dzzC[4] * uzz[5];
            conv_z = -h31 - h32 - h33 + xnu * (d11 + d33) + c.grav[2];
            const double gradp = c.dzC[0] * AT(pr, 0, r0, -2) + c.dzC[1] * AT(pr, 0, r0, -1) + c.dzC[2] * AT(pr, 0, r0, 0) + c.dzC[3] * AT(pr, 0, r0, 1);
            rhs_z = pmGamma * conv_z + pmTheta * hz[q0] - pmAlpha * gradp + tb * d22;
        }

        if (SCALAR) {
            // ---------------- scalar transport (:302-357)
            double scx[7], scz[7];
#pragma unroll
            for (int d = 0; d < 7; d++) { scx[d] = AT(sc, d - 3, r0, 0); scz[d] = AT(sc, 0, r0, d - 3); }
            const double scc = scx[3];
            double shx[4], shz[4];  // offsets -1..2
#pragma unroll
            for (int q = 0; q < 4; q++) {
                shx[q] = I1 * scx[q] + I2 * scx[q + 1] + I3 * scx[q + 2] + I4 * scx[q + 3];
                shz[q] = I1 * scz[q] + I2 * scz[q + 1] + I3 * scz[q + 2] + I4 * scz[q + 3];
            }
            const double scjm = AT(sc, 0, rm, 0), scjp = AT(sc, 0, rp, 0);
            const double shyc = IY1 * scjm + IY2 * scc;
            const double shyp = IY3 * scc + IY4 * scjp;
            const double c1 = c.gev[0] * shx[1], c2 = c.gev[1] * shyc, c3 = c.gev[2] * shz[1];
            rhs_x = rhs_x + pmGamma * c1;
            rhs_y = rhs_y + pmGamma * c2;
            rhs_z = rhs_z + pmGamma * c3;
            conv_x = conv_x + c1;
            conv_y = conv_y + c2;
            conv_z = conv_z + c3;
            double hc1 = 0.0, hc3 = 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const double ua = AT(ux, q - 1, r0, 0) + c.fvv[0];
                const double wa = AT(uz, 0, r0, q - 1) + c.fvv[2];
                hc1 = (q == 0) ? c.dxC[0] * ua * shx[0] : hc1 + c.dxC[q] * ua * shx[q];
                hc3 = (q == 0) ? c.dzC[0] * wa * shz[0] : hc3 + c.dzC[q] * wa * shz[q];
            }
            const double hc2 = ((AT(uy, 0, rp, 0) + c.fvv[1]) * shyp - (uyx[3] + c.fvv[1]) * shyc) * rdyp;
            const double d11 = c.dxxC[0] * scx[1] + c.dxxC[1] * scx[2] + c.dxxC[2] * scc + c.dxxC[3] * scx[4] + c.dxxC[4] * scx[5];
            const double d22 = __ldg(&m.ap2cSc[jc]) * scjp + __ldg(&m.ac2cSc[jc]) * scc + __ldg(&m.am2cSc[jc]) * scjm;
            const double d33 = c.dzzC[0] * scz[1] + c.dzzC[1] * scz[2] + c.dzzC[2] * scc + c.dzzC[3] * scz[4] + c.dzzC[4] * scz[5];
            const double convc = -hc1 - hc2 - hc3 + c.sdiff * (d11 + d33);
            rc[q0] = coef->pmGamma * convc + pmTheta * hc[q0] + 2.0 * coef->pmBetaSc * d22;
            hc[q0] = convc;
        }
#undef AT
        rx[q0] = rhs_x;
        ry[q0] = rhs_y;
        rz[q0] = rhs_z;
        hx[q0] = conv_x;
        hy[q0] = conv_y;
        hz[q0] = conv_z;
    }
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_sum_store<1>(s3, part + bid);
}

// flow-rate constraint (src/m_TScheme.f90:269-300): reduce s3tot, set the
// uniform RhsX correction and accumulate PrGradAver
__global__ void k_flowrate(DConst c, DCoef* coef, const double* __restrict__ part, int nparts) {
    double s[1];
    reduce_parts<1, false>(part, nparts, s);
    if (threadIdx.x != 0) return;
    DCoef f = *coef;
    if (!c.is_ux_const) { f.rhsx_add = 0.0; *coef = f; return; }
    double s3tot1 = s[0];
    const double nxz = (double)(c.nx * c.nz);
    if (c.scalar_on) {
        s3tot1 = s3tot1 / nxz / c.yly;
        const double dpmdxns = c.ubulk - c.ucrf - s3tot1;
        f.rhsx_add = f.pmAlphaC * dpmdxns;
        f.pr_grad_aver = f.pr_grad_aver + dpmdxns * f.pmAlphaC / f.dt;
    } else {
        const double dpmdxns = c.xnu * s3tot1 / nxz / c.yly;
        f.rhsx_add = -(f.pmAlpha * dpmdxns);
        f.pr_grad_aver = f.pr_grad_aver + dpmdxns * f.pmAlphaC;
    }
    *coef = f;
}

// ---------------------------------------------------------------------------
// clcPrSrc (src/m_TScheme.f90:48-77) / CheckDivergence (src/m_Tools.f90:54-81)
// src is the compact interior array (k, j-1, i); scale = 1/pmAlpha, or 1
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_prsrc(DConst c, DMetric m, const DCoef* __restrict__ coef, int unit_scale,
                                               const double* __restrict__ ux, const double* __restrict__ uy,
                                               const double* __restrict__ uz, double* __restrict__ src,
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
__global__ void __launch_bounds__(256) k_project(DConst c, DMetric m, const DCoef* __restrict__ coef, int mode,
                                                 const double* __restrict__ phi, double* __restrict__ ux,
                                                 double* __restrict__ uy, double* __restrict__ uz,
                                                 double* __restrict__ pr, const double* __restrict__ uy_ym) {
    const int nx = c.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int jc = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z;
    if (i >= nx || jc > c.ny) return;
    const double alpha = mode == 0 ? coef->pmAlpha : 1.0;
    const size_t pl = (size_t)c.nyt * nx;
    const size_t r0 = (size_t)jc * nx, zc = (size_t)k * pl;
    const int is = wrapi(i - 2, nx), im = wrapi(i - 1, nx), ip = wrapi(i + 1, nx);
    const size_t zs = (size_t)wrapi(k - 2, c.nz) * pl, zm = (size_t)wrapi(k - 1, c.nz) * pl, zp = (size_t)wrapi(k + 1, c.nz) * pl;
    const size_t q = zc + r0 + i;
    const double pc = LD(phi, q), pjm = LD(phi, q - nx), pjp = LD(phi, q + nx);
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

// ---------------------------------------------------------------------------
// ghost rows from the interior: SetBC_and_UpdateHalo, _pr and _scalar
// (src/m_BC_and_Halo.f90:23-178); one thread per (i, k)
// ---------------------------------------------------------------------------
__global__ void k_bc_all(DConst c, double* __restrict__ ux, double* __restrict__ uy, double* __restrict__ uz,
                         double* __restrict__ pr, double* __restrict__ sc, const double* __restrict__ uy_ym) {
    const int nx = c.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (i >= nx) return;
    const size_t pl = (size_t)c.nyt * nx, zc = (size_t)k * pl;
    const size_t g0 = zc + i, r1 = zc + nx + i, rn = zc + (size_t)c.ny * nx + i, gt = zc + (size_t)c.nyp * nx + i;
    const bool ft_ch = (c.flow_type == 1);
    ux[gt] = ft_ch ? c.uxbc_yp * 2.0 - ux[rn] : ux[rn];
    uy[gt] = ft_ch ? c.uybc_yp : 0.0;
    uz[gt] = ft_ch ? c.uzbc_yp * 2.0 - uz[rn] : uz[rn];
    ux[g0] = c.uxbc_ym * 2.0 - ux[r1];
    uy[r1] = uy_ym[(size_t)k * nx + i];
    uz[g0] = c.uzbc_ym * 2.0 - uz[r1];
    pr[g0] = pr[r1];
    pr[gt] = pr[rn];
    if (c.scalar_on && sc) {
        sc[g0] = c.sc_r1b * sc[r1] + c.sc_r2b;
        sc[gt] = c.sc_r1t * sc[rn] + c.sc_r2t;
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
__global__ void __launch_bounds__(256) k_cfl(DConst c, DMetric m, const double* __restrict__ ux,
                                             const double* __restrict__ uy, const double* __restrict__ uz,
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
// end-of-step checks: CheckDivergence, CalcVmax, CalcUxAver / ClcMeanValue
// (src/m_Tools.f90:54-110,256-301); per block: 4 maxima + 3 sums
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_check(DConst c, DMetric m, const double* __restrict__ ux,
                                               const double* __restrict__ uy, const double* __restrict__ uz,
                                               const double* __restrict__ sc, double* __restrict__ part) {
    const int nx = c.nx;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int jc = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z;
    double mx[4] = {0.0, 0.0, 0.0, 0.0};
    double sm[3] = {0.0, 0.0, 0.0};
    if (i < nx && jc <= c.ny) {
        const size_t pl = (size_t)c.nyt * nx, zc = (size_t)k * pl, r0 = (size_t)jc * nx;
        const size_t q = zc + r0 + i;
        const int im = wrapi(i - 1, nx), ip = wrapi(i + 1, nx), iu = wrapi(i + 2, nx);
        const size_t zm = (size_t)wrapi(k - 1, c.nz) * pl, zp = (size_t)wrapi(k + 1, c.nz) * pl, zu = (size_t)wrapi(k + 2, c.nz) * pl;
        const double dudx = c.dxC[0] * LD(ux, zc + r0 + im) + c.dxC[1] * LD(ux, q) + c.dxC[2] * LD(ux, zc + r0 + ip) + c.dxC[3] * LD(ux, zc + r0 + iu);
        const double dvdy = (LD(uy, q + nx) - LD(uy, q)) * __ldg(&m.rdyp[jc]);
        const double dwdz = c.dzC[0] * LD(uz, zm + r0 + i) + c.dzC[1] * LD(uz, q) + c.dzC[2] * LD(uz, zp + r0 + i) + c.dzC[3] * LD(uz, zu + r0 + i);
        mx[0] = fabs(dudx + dvdy + dwdz);
        const double u = LD(ux, q);
        mx[1] = fabs(u);
        mx[2] = fabs(LD(uy, q));
        mx[3] = fabs(LD(uz, q));
        const double dy = __ldg(&m.dyp[jc]);
        sm[0] = u * dy;
        if (c.scalar_on) {
            const double s = LD(sc, q);
            sm[1] = dy * s;
            sm[2] = dy * s * s;
        }
    }
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_max_store<4>(mx, part + (size_t)bid * 7);
    __syncthreads();
    block_sum_store<3>(sm, part + (size_t)bid * 7 + 4);
}

__global__ void k_check_final(DConst c, const DCoef* __restrict__ coef, DDiag* __restrict__ diag,
                              const double* __restrict__ part, int nparts) {
    // maxima and sums are interleaved per block: reduce in two passes
    __shared__ double sh[32][7];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = (blockDim.x + 31) >> 5;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = tid; b < nparts; b += blockDim.x) {
        const double* p = part + (size_t)b * 7;
        for (int q = 0; q < 4; q++) v[q] = fmax(v[q], p[q]);
        for (int q = 4; q < 7; q++) v[q] += p[q];
    }
    for (int q = 0; q < 7; q++)
        for (int o = 16; o > 0; o >>= 1) {
            double y = __shfl_down_sync(0xffffffffu, v[q], o);
            v[q] = q < 4 ? fmax(v[q], y) : v[q] + y;
        }
    if (lane == 0)
        for (int q = 0; q < 7; q++) sh[wid][q] = v[q];
    __syncthreads();
    if (tid != 0) return;
    double r[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int w = 0; w < nw; w++)
        for (int q = 0; q < 7; q++) r[q] = q < 4 ? fmax(r[q], sh[w][q]) : r[q] + sh[w][q];
    DDiag d = *diag;
    const DCoef f = *coef;
    d.step_counter += 1;
    d.dt = f.dt;
    d.cfl = f.cflmp;
    d.sim_time = f.sim_time;
    d.divmax_src = f.divmax_src;
    d.divmax = r[0];
    d.vmax[0] = r[1]; d.vmax[1] = r[2]; d.vmax[2] = r[3];
    d.pr_grad_aver = f.pr_grad_aver;
    const double nxz = (double)(c.nx * c.nz);
    d.ux_mean = r[4] / nxz / c.yly;
    d.sc_mean = r[5] / nxz / c.yly;
    d.sc2_mean = r[6] / nxz / c.yly;
    if (d.status == 0) {
        double vmin = fmin(fmin(r[1], r[2]), r[3]);
        if (!(r[0] == r[0]) || !(vmin == vmin)) { d.status = -4; d.failed_step = d.step_counter; }
        else if (r[0] > c.div_limit) { d.status = -5; d.failed_step = d.step_counter; }
        else if (vmin > c.vel_limit) { d.status = -6; d.failed_step = d.step_counter; }
    }
    *diag = d;
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

void launch_coef(cudaStream_t st, DCoef* coef, int ns, double gam, double the, double alp, double xnu, double sdiff) {
    k_coef<<<1, 32, 0, st>>>(coef, ns, gam, the, alp, xnu, sdiff);
}

void launch_rhs(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, const Fields& f, double* part) {
    if (c.scalar_on)
        k_rhs<true><<<cell_grid(c), cell_block(), 0, st>>>(c, m, coef, f.ux, f.uy, f.uz, f.pr, f.sc, f.hx, f.hy, f.hz, f.hc,
                                                            f.rx, f.ry, f.rz, f.rc, part);
    else
        k_rhs<false><<<cell_grid(c), cell_block(), 0, st>>>(c, m, coef, f.ux, f.uy, f.uz, f.pr, f.sc, f.hx, f.hy, f.hz, f.hc,
                                                             f.rx, f.ry, f.rz, f.rc, part);
}

void launch_flowrate(cudaStream_t st, const DConst& c, DCoef* coef, const double* part, int nparts) {
    k_flowrate<<<1, 1024, 0, st>>>(c, coef, part, nparts);
}

void launch_prsrc(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int unit_scale,
                  const Fields& f, double* src, double* part, double* out_max) {
    k_prsrc<<<cell_grid(c), cell_block(), 0, st>>>(c, m, coef, unit_scale, f.ux, f.uy, f.uz, src, part);
    k_reduce_max<<<1, 1024, 0, st>>>(part, (int)cell_grid_blocks(c), out_max);
}

void launch_store_divsrc(cudaStream_t st, DCoef* coef, const double* v) { k_store_divsrc<<<1, 32, 0, st>>>(coef, v); }

void launch_project(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int mode, const double* phi,
                    const Fields& f, const double* uy_ym) {
    k_project<<<cell_grid(c), cell_block(), 0, st>>>(c, m, coef, mode, phi, f.ux, f.uy, f.uz, f.pr, uy_ym);
}

void launch_bc_all(cudaStream_t st, const DConst& c, const Fields& f, const double* uy_ym) {
    k_bc_all<<<dim3((c.nx + 127) / 128, c.nz), 128, 0, st>>>(c, f.ux, f.uy, f.uz, f.pr, f.sc, uy_ym);
}

void launch_update_uy_ym(cudaStream_t st, int n, double* uy_ym, double* duy_ym) {
    k_update_uy_ym<<<(n + 255) / 256, 256, 0, st>>>(n, uy_ym, duy_ym);
}

void launch_cfl(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, DCoef* coef, double* part) {
    k_cfl<<<cell_grid(c), cell_block(), 0, st>>>(c, m, f.ux, f.uy, f.uz, part);
    k_cfl_final<<<1, 1024, 0, st>>>(c, coef, part, (int)cell_grid_blocks(c));
}

void launch_check(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, const DCoef* coef, DDiag* diag,
                  double* part) {
    k_check<<<cell_grid(c), cell_block(), 0, st>>>(c, m, f.ux, f.uy, f.uz, f.sc, part);
    k_check_final<<<1, 1024, 0, st>>>(c, coef, diag, part, (int)cell_grid_blocks(c));
}

}  // namespace ptc
