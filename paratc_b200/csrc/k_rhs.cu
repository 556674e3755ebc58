// k_rhs.cu -- clcRhsXYZ (src/m_TScheme.f90:113-360) on B200 with
// shared-memory row-slab tiles.
//
// A CTA owns a 32 (x) by 8 (z) column tile and marches up a chunk of y rows.
// For every row j it needs rows j-1, j, j+1 of ux, uy, uz, p (and the
// scalar) over the tile plus the x/z halo of 3 cells that the interpolated
// face velocities and the 4th-order stencils read (38 x 14 values per field
// and row).  Those row-slabs sit in a ring of 4 slots in shared memory; the
// slab of row j+2 is copied in with cp.async while row j is computed, so the
// HBM loads of one row overlap the arithmetic of the previous one.  Each
// thread computes one cell per row: RhsX/RhsY/RhsZ (and RhsC) and the new
// explicit histories, reading every neighbour from shared memory; the six
// interpolated fields of the reference and their halo updates never exist.
//
// The same kernel performs PMcoeUpdate (src/m_Parameters.f90:215-230),
// Update_uy_ym (src/m_FlowCase.f90:112-122) and the flow-rate constraint
// (src/m_TScheme.f90:269-300): every CTA writes its partial of s3tot and the
// last CTA to finish reduces them in a fixed order and stores the uniform
// RhsX correction and the substep coefficients for the kernels that follow.
#include "common.cuh"
#include "kernels.cuh"
#include "reduce.cuh"

namespace ptc {
namespace {

constexpr int TX = 32, TZ = 8, HX = 3, HZ = 3;
constexpr int SX = TX + 2 * HX;  // 38
constexpr int SZ = TZ + 2 * HZ;  // 14
constexpr int SLAB = SX * SZ;    // 532 doubles per field and row
constexpr int NB = 4;            // ring slots
constexpr int ZC = 2;            // z-adjacent cells per thread: their shared stencil taps are loaded once
constexpr int NTHR = TX * TZ / ZC;  // 128
constexpr int NSLOT = (SLAB + NTHR - 1) / NTHR;

__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ int modp(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

}  // namespace

template <bool SCALAR>
__global__ void __launch_bounds__(NTHR, 2)
    k_rhs_tile(DConst c, DMetric m, DCoef* __restrict__ coef, Fields fl, double* __restrict__ uy_ym,
               double* __restrict__ duy_ym, int ns, double gam, double the, double alp, int ychunk,
               double* __restrict__ part, unsigned int* __restrict__ counter) {
    constexpr int NF = SCALAR ? 5 : 4;
    extern __shared__ double sm[];  // [NB][NF][SLAB]
    const int lane = threadIdx.x, wq = threadIdx.y, tid = wq * 32 + lane;
    const int nx = c.nx, nz = c.nz, ny = c.ny;
    const size_t pl = (size_t)c.nyt * nx;
    // work = the (tile, row) pairs in tile-major order; block b takes the
    // contiguous range [b*W/B, (b+1)*W/B), so one wave of resident blocks
    // covers the grid with at most one row of imbalance
    const int ntx = (nx + TX - 1) / TX, ntz = (nz + TZ - 1) / TZ;
    const long long W = (long long)ntx * ntz * ny;
    const long long gbeg = W * blockIdx.x / gridDim.x, gend = W * (blockIdx.x + 1) / gridDim.x;
    (void)ychunk;
    pdl_wait();
    pdl_trigger();

    // PMcoeUpdate from the device dt
    const double dt = coef->dt;
    const double pmGamma = gam * dt, pmTheta = the * dt, pmAlpha = alp * dt;
    const double pmBeta = 0.5 * alp * c.xnu * dt, pmBetaSc = 0.5 * alp * c.sdiff * dt;
    const double tb = 2.0 * pmBeta, tbs = 2.0 * pmBetaSc;
    const double I1 = c.IC[0], I2 = c.IC[1], I3 = c.IC[2], I4 = c.IC[3];
    const double ucrf = c.ucrf, xnu = c.xnu;
    const double* fsrc[5] = {fl.ux, fl.uy, fl.uz, fl.pr, fl.sc};
    double s3 = 0.0;

    for (long long g = gbeg; g < gend;) {
        const int tile = (int)(g / ny);
        const int j0 = (int)(g - (long long)tile * ny) + 1;
        const int j1 = (int)min((long long)ny, (long long)j0 + (gend - g) - 1);
        g += j1 - j0 + 1;
        const int i0 = (tile % ntx) * TX, k0 = (tile / ntx) * TZ;
        size_t goff[NSLOT];
        int soff[NSLOT];
        bool sval[NSLOT];
#pragma unroll
        for (int s = 0; s < NSLOT; s++) {
            const int e = tid + s * NTHR;
            sval[s] = e < SLAB;
            const int zz = e / SX, xx = e - zz * SX;
            goff[s] = (size_t)modp(k0 - HZ + zz, nz) * pl + (size_t)modp(i0 - HX + xx, nx);
            soff[s] = e;
        }
#define LOAD_ROW(jrow)                                                                   \
    do {                                                                                 \
        double* dst_ = sm + (size_t)((jrow) % NB) * NF * SLAB;                           \
        const size_t ro_ = (size_t)(jrow) * nx;                                          \
        _Pragma("unroll") for (int f_ = 0; f_ < NF; f_++)                                \
            _Pragma("unroll") for (int s_ = 0; s_ < NSLOT; s_++) if (sval[s_])           \
                cp_async8(dst_ + f_ * SLAB + soff[s_], fsrc[f_] + goff[s_] + ro_);       \
    } while (0)

        LOAD_ROW(j0 - 1);
        LOAD_ROW(j0);
        LOAD_ROW(j0 + 1);
        cp_async_commit();

        const int i = i0 + lane;
        int kk[ZC];
        bool act[ZC];
        // explicit histories of the next row are loaded one row ahead
        double hxn[ZC], hyn[ZC], hzn[ZC], hcn[ZC];
#pragma unroll
        for (int cz = 0; cz < ZC; cz++) {
            kk[cz] = k0 + wq * ZC + cz;
            act[cz] = (i < nx) && (kk[cz] < nz);
            if (act[cz] && j0 == 1) {
                const size_t t = (size_t)kk[cz] * nx + i;
                const double d = uy_ym[t];
                uy_ym[t] = 0.0;
                duy_ym[t] = uy_ym[t] - d;
            }
            hxn[cz] = hyn[cz] = hzn[cz] = hcn[cz] = 0.0;
            if (act[cz]) {
                const size_t q = (size_t)kk[cz] * pl + (size_t)j0 * nx + i;
                hxn[cz] = fl.hx[q]; hyn[cz] = fl.hy[q]; hzn[cz] = fl.hz[q];
                if (SCALAR) hcn[cz] = fl.hc[q];
            }
        }

        for (int j = j0; j <= j1; j++) {
            if (j + 2 <= j1 + 1) LOAD_ROW(j + 2);
            cp_async_commit();
            double hx0a[ZC], hy0a[ZC], hz0a[ZC], hc0a[ZC];
            size_t q0a[ZC];
#pragma unroll
            for (int cz = 0; cz < ZC; cz++) {
                hx0a[cz] = hxn[cz]; hy0a[cz] = hyn[cz]; hz0a[cz] = hzn[cz]; hc0a[cz] = hcn[cz];
                q0a[cz] = (size_t)kk[cz] * pl + (size_t)j * nx + i;
                if (act[cz] && j + 1 <= j1) {
                    hxn[cz] = fl.hx[q0a[cz] + nx]; hyn[cz] = fl.hy[q0a[cz] + nx]; hzn[cz] = fl.hz[q0a[cz] + nx];
                    if (SCALAR) hcn[cz] = fl.hc[q0a[cz] + nx];
                }
            }
            cp_async_wait<1>();
            __syncthreads();
            // both cells are computed before any global store, so that the
            // compiler may load a tap the two cells share once
            double o_rx[ZC], o_ry[ZC], o_rz[ZC], o_hx[ZC], o_hy[ZC], o_hz[ZC], o_rc[ZC], o_hc[ZC];
            {
                const double* Sm = sm + (size_t)((j - 1) % NB) * NF * SLAB;
                const double* Sc = sm + (size_t)(j % NB) * NF * SLAB;
                const double* Sp = sm + (size_t)((j + 1) % NB) * NF * SLAB;
#define V(S, f, dx, dz) (S)[(f) * SLAB + (w + HZ + (dz)) * SX + (lane + HX + (dx))]
            const bool top = (j == ny);
            const double IY1 = __ldg(&m.yinterp[j]), IY2 = 1.0 - IY1;
            const double IY3 = __ldg(&m.yinterp[j + 1]), IY4 = 1.0 - IY3;
            const double rdyp = __ldg(&m.rdyp[j]), rdyc = __ldg(&m.rdyc[j]), dyp = __ldg(&m.dyp[j]);
#pragma unroll
            for (int cz = 0; cz < ZC; cz++) {
            const int w = wq * ZC + cz;
            const double hx0 = hx0a[cz], hy0 = hy0a[cz], hz0 = hz0a[cz], hc0 = hc0a[cz];
            (void)hc0;

            // ---------------- RhsX (:169-204)
            double conv_x, rhs_x;
            {
                const double uxc = V(Sc, 0, 0, 0), uxjm = V(Sm, 0, 0, 0), uxjp = V(Sp, 0, 0, 0);
                const double uxhyc = IY1 * uxjm + IY2 * uxc;
                const double uxhyp = IY3 * uxc + IY4 * uxjp;
                double h11 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) {  // uxhx at x offsets -2..1
                    const int d = q - 2;
                    const double uh = I1 * V(Sc, 0, d - 1, 0) + I2 * V(Sc, 0, d, 0) + I3 * V(Sc, 0, d + 1, 0) + I4 * V(Sc, 0, d + 2, 0);
                    h11 = (q == 0) ? c.dxC[0] * uh * (uh + ucrf) : h11 + c.dxC[q] * uh * (uh + ucrf);
                }
                const double uyhx_j = I1 * V(Sc, 1, -2, 0) + I2 * V(Sc, 1, -1, 0) + I3 * V(Sc, 1, 0, 0) + I4 * V(Sc, 1, 1, 0);
                const double uyhx_p = top ? 0.0 : I1 * V(Sp, 1, -2, 0) + I2 * V(Sp, 1, -1, 0) + I3 * V(Sp, 1, 0, 0) + I4 * V(Sp, 1, 1, 0);
                const double h12 = (uyhx_p * uxhyp - uyhx_j * uxhyc) * rdyp;
                double h13 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) {  // z offsets -1..2
                    const int d = q - 1;
                    const double uxhz = I1 * V(Sc, 0, 0, d - 2) + I2 * V(Sc, 0, 0, d - 1) + I3 * V(Sc, 0, 0, d) + I4 * V(Sc, 0, 0, d + 1);
                    const double uzhx = I1 * V(Sc, 2, -2, d) + I2 * V(Sc, 2, -1, d) + I3 * V(Sc, 2, 0, d) + I4 * V(Sc, 2, 1, d);
                    h13 = (q == 0) ? c.dzC[0] * uxhz * uzhx : h13 + c.dzC[q] * uxhz * uzhx;
                }
                const double d11 = c.dxxC[0] * V(Sc, 0, -2, 0) + c.dxxC[1] * V(Sc, 0, -1, 0) + c.dxxC[2] * uxc + c.dxxC[3] * V(Sc, 0, 1, 0) + c.dxxC[4] * V(Sc, 0, 2, 0);
                const double d22 = __ldg(&m.ap2c[j]) * uxjp + __ldg(&m.ac2c[j]) * uxc + __ldg(&m.am2c[j]) * uxjm;
                const double d33 = c.dzzC[0] * V(Sc, 0, 0, -2) + c.dzzC[1] * V(Sc, 0, 0, -1) + c.dzzC[2] * uxc + c.dzzC[3] * V(Sc, 0, 0, 1) + c.dzzC[4] * V(Sc, 0, 0, 2);
                const double dcq13 = d11 + d33;
                if (act[cz]) s3 += SCALAR ? uxc * dyp : (dcq13 + d22) * dyp;
                conv_x = -h11 - h12 - h13 + xnu * dcq13 + c.grav[0];
                const double gradp = c.dxC[0] * V(Sc, 3, -2, 0) + c.dxC[1] * V(Sc, 3, -1, 0) + c.dxC[2] * V(Sc, 3, 0, 0) + c.dxC[3] * V(Sc, 3, 1, 0);
                rhs_x = pmGamma * conv_x + pmTheta * hx0 - pmAlpha * gradp + tb * d22;
            }
            // ---------------- RhsY (:206-236)
            double conv_y, rhs_y;
            {
                const double qsucac = 0.25 * rdyc;
                double h21 = 0.0, h23 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) {  // offsets -1..2
                    const int d = q - 1;
                    const double uxh = IY1 * V(Sm, 0, d, 0) + IY2 * V(Sc, 0, d, 0) + ucrf;
                    const double uzh = IY1 * V(Sm, 2, 0, d) + IY2 * V(Sc, 2, 0, d);
                    const double uyhx = I1 * V(Sc, 1, d - 2, 0) + I2 * V(Sc, 1, d - 1, 0) + I3 * V(Sc, 1, d, 0) + I4 * V(Sc, 1, d + 1, 0);
                    const double uyhz = I1 * V(Sc, 1, 0, d - 2) + I2 * V(Sc, 1, 0, d - 1) + I3 * V(Sc, 1, 0, d) + I4 * V(Sc, 1, 0, d + 1);
                    h21 = (q == 0) ? c.dxC[0] * uyhx * uxh : h21 + c.dxC[q] * uyhx * uxh;
                    h23 = (q == 0) ? c.dzC[0] * uyhz * uzh : h23 + c.dzC[q] * uyhz * uzh;
                }
                const double vp = V(Sp, 1, 0, 0), vc = V(Sc, 1, 0, 0), vm = V(Sm, 1, 0, 0);
                const double h22 = ((vp + vc) * (vp + vc) - (vc + vm) * (vc + vm)) * qsucac;
                const double d11 = c.dxxC[0] * V(Sc, 1, -2, 0) + c.dxxC[1] * V(Sc, 1, -1, 0) + c.dxxC[2] * vc + c.dxxC[3] * V(Sc, 1, 1, 0) + c.dxxC[4] * V(Sc, 1, 2, 0);
                const double d22 = __ldg(&m.ap2p[j]) * vp + __ldg(&m.ac2p[j]) * vc + __ldg(&m.am2p[j]) * vm;
                const double d33 = c.dzzC[0] * V(Sc, 1, 0, -2) + c.dzzC[1] * V(Sc, 1, 0, -1) + c.dzzC[2] * vc + c.dzzC[3] * V(Sc, 1, 0, 1) + c.dzzC[4] * V(Sc, 1, 0, 2);
                conv_y = -h21 - h22 - h23 + xnu * (d11 + d33) + c.grav[1];
                const double gradp = (V(Sc, 3, 0, 0) - V(Sm, 3, 0, 0)) * rdyc;
                rhs_y = pmGamma * conv_y + pmTheta * hy0 - pmAlpha * gradp + tb * d22;
            }
            // ---------------- RhsZ (:238-267)
            double conv_z, rhs_z;
            {
                const double uzc = V(Sc, 2, 0, 0);
                const double uzhyc = IY1 * V(Sm, 2, 0, 0) + IY2 * uzc;
                const double uzhyp = IY3 * uzc + IY4 * V(Sp, 2, 0, 0);
                double h31 = 0.0, h33 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int d = q - 1;  // x offsets -1..2 for h31
                    const double uzhx = I1 * V(Sc, 2, d - 2, 0) + I2 * V(Sc, 2, d - 1, 0) + I3 * V(Sc, 2, d, 0) + I4 * V(Sc, 2, d + 1, 0);
                    const double uxhz = I1 * V(Sc, 0, d, -2) + I2 * V(Sc, 0, d, -1) + I3 * V(Sc, 0, d, 0) + I4 * V(Sc, 0, d, 1);
                    h31 = (q == 0) ? c.dxC[0] * uzhx * (uxhz + ucrf) : h31 + c.dxC[q] * uzhx * (uxhz + ucrf);
                    const int e = q - 2;  // z offsets -2..1 for h33
                    const double uzhz = I1 * V(Sc, 2, 0, e - 1) + I2 * V(Sc, 2, 0, e) + I3 * V(Sc, 2, 0, e + 1) + I4 * V(Sc, 2, 0, e + 2);
                    h33 = (q == 0) ? c.dzC[0] * uzhz * uzhz : h33 + c.dzC[q] * uzhz * uzhz;
                }
                const double uyhz_j = I1 * V(Sc, 1, 0, -2) + I2 * V(Sc, 1, 0, -1) + I3 * V(Sc, 1, 0, 0) + I4 * V(Sc, 1, 0, 1);
                const double uyhz_p = top ? 0.0 : I1 * V(Sp, 1, 0, -2) + I2 * V(Sp, 1, 0, -1) + I3 * V(Sp, 1, 0, 0) + I4 * V(Sp, 1, 0, 1);
                const double h32 = (uyhz_p * uzhyp - uyhz_j * uzhyc) * rdyp;
                const double d11 = c.dxxC[0] * V(Sc, 2, -2, 0) + c.dxxC[1] * V(Sc, 2, -1, 0) + c.dxxC[2] * uzc + c.dxxC[3] * V(Sc, 2, 1, 0) + c.dxxC[4] * V(Sc, 2, 2, 0);
                const double d22 = __ldg(&m.ap2c[j]) * V(Sp, 2, 0, 0) + __ldg(&m.ac2c[j]) * uzc + __ldg(&m.am2c[j]) * V(Sm, 2, 0, 0);
                const double d33 = c.dzzC[0] * V(Sc, 2, 0, -2) + c.dzzC[1] * V(Sc, 2, 0, -1) + c.dzzC[2] * uzc + c.dzzC[3] * V(Sc, 2, 0, 1) + c.dzzC[4] * V(Sc, 2, 0, 2);
                conv_z = -h31 - h32 - h33 + xnu * (d11 + d33) + c.grav[2];
                const double gradp = c.dzC[0] * V(Sc, 3, 0, -2) + c.dzC[1] * V(Sc, 3, 0, -1) + c.dzC[2] * V(Sc, 3, 0, 0) + c.dzC[3] * V(Sc, 3, 0, 1);
                rhs_z = pmGamma * conv_z + pmTheta * hz0 - pmAlpha * gradp + tb * d22;
            }
            if (SCALAR) {
                // ---------------- scalar transport (:302-357)
                const double scc = V(Sc, 4, 0, 0), scjm = V(Sm, 4, 0, 0), scjp = V(Sp, 4, 0, 0);
                const double shyc = IY1 * scjm + IY2 * scc;
                const double shyp = IY3 * scc + IY4 * scjp;
                double hc1 = 0.0, hc3 = 0.0, shx0 = 0.0, shz0 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int d = q - 1;
                    const double shx = I1 * V(Sc, 4, d - 2, 0) + I2 * V(Sc, 4, d - 1, 0) + I3 * V(Sc, 4, d, 0) + I4 * V(Sc, 4, d + 1, 0);
                    const double shz = I1 * V(Sc, 4, 0, d - 2) + I2 * V(Sc, 4, 0, d - 1) + I3 * V(Sc, 4, 0, d) + I4 * V(Sc, 4, 0, d + 1);
                    if (q == 1) { shx0 = shx; shz0 = shz; }
                    const double ua = V(Sc, 0, d, 0) + c.fvv[0];
                    const double wa = V(Sc, 2, 0, d) + c.fvv[2];
                    hc1 = (q == 0) ? c.dxC[0] * ua * shx : hc1 + c.dxC[q] * ua * shx;
                    hc3 = (q == 0) ? c.dzC[0] * wa * shz : hc3 + c.dzC[q] * wa * shz;
                }
                const double c1 = c.gev[0] * shx0, c2 = c.gev[1] * shyc, c3 = c.gev[2] * shz0;
                rhs_x = rhs_x + pmGamma * c1;
                rhs_y = rhs_y + pmGamma * c2;
                rhs_z = rhs_z + pmGamma * c3;
                conv_x = conv_x + c1;
                conv_y = conv_y + c2;
                conv_z = conv_z + c3;
                const double hc2 = ((V(Sp, 1, 0, 0) + c.fvv[1]) * shyp - (V(Sc, 1, 0, 0) + c.fvv[1]) * shyc) * rdyp;
                const double d11 = c.dxxC[0] * V(Sc, 4, -2, 0) + c.dxxC[1] * V(Sc, 4, -1, 0) + c.dxxC[2] * scc + c.dxxC[3] * V(Sc, 4, 1, 0) + c.dxxC[4] * V(Sc, 4, 2, 0);
                const double d22 = __ldg(&m.ap2cSc[j]) * scjp + __ldg(&m.ac2cSc[j]) * scc + __ldg(&m.am2cSc[j]) * scjm;
                const double d33 = c.dzzC[0] * V(Sc, 4, 0, -2) + c.dzzC[1] * V(Sc, 4, 0, -1) + c.dzzC[2] * scc + c.dzzC[3] * V(Sc, 4, 0, 1) + c.dzzC[4] * V(Sc, 4, 0, 2);
                const double convc = -hc1 - hc2 - hc3 + c.sdiff * (d11 + d33);
                o_rc[cz] = pmGamma * convc + pmTheta * hc0 + tbs * d22;
                o_hc[cz] = convc;
            }
#undef V
            o_rx[cz] = rhs_x; o_ry[cz] = rhs_y; o_rz[cz] = rhs_z;
            o_hx[cz] = conv_x; o_hy[cz] = conv_y; o_hz[cz] = conv_z;
            }
            }
#pragma unroll
            for (int cz = 0; cz < ZC; cz++) {
                if (!act[cz]) continue;
                const size_t q0 = q0a[cz];
                fl.rx[q0] = o_rx[cz];
                fl.ry[q0] = o_ry[cz];
                fl.rz[q0] = o_rz[cz];
                fl.hx[q0] = o_hx[cz];
                fl.hy[q0] = o_hy[cz];
                fl.hz[q0] = o_hz[cz];
                if (SCALAR) {
                    fl.rc[q0] = o_rc[cz];
                    fl.hc[q0] = o_hc[cz];
                }
            }
        __syncthreads();
        }
#undef LOAD_ROW
    }
    cp_async_wait<0>();

    // flow-rate constraint and the substep coefficients (last CTA)
    double s3v[1] = {s3};
    const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_sum_store<1>(s3v, part + bid);
    if (!last_block_arrive(counter, nblocks)) return;
    double tot[1];
    reduce_records<1, false>(part, (int)nblocks, tot);
    if (tid != 0) return;
    DCoef f = *coef;
    f.pmGamma = pmGamma;
    f.pmTheta = pmTheta;
    f.pmAlpha = pmAlpha;
    f.pmBeta = pmBeta;
    f.pmBetaSc = pmBetaSc;
    f.sim_time = f.sim_time + dt * alp;
    f.pmAlphaC = alp;
    if (ns == 1) f.pr_grad_aver = 0.0;
    f.ns = ns;
    f.rhsx_add = 0.0;
    if (c.is_ux_const) {
        double s3tot1 = tot[0];
        const double nxz = (double)(c.nx * c.nz);
        if (SCALAR) {
            s3tot1 = s3tot1 / nxz / c.yly;
            const double dpmdxns = c.ubulk - c.ucrf - s3tot1;
            f.rhsx_add = f.pmAlphaC * dpmdxns;
            f.pr_grad_aver = f.pr_grad_aver + dpmdxns * f.pmAlphaC / f.dt;
        } else {
            const double dpmdxns = c.xnu * s3tot1 / nxz / c.yly;
            f.rhsx_add = -(f.pmAlpha * dpmdxns);
            f.pr_grad_aver = f.pr_grad_aver + dpmdxns * f.pmAlphaC;
        }
    }
    *coef = f;
}

// ---------------------------------------------------------------------------
static int rhs_ychunk(const DConst& c) {
    const int nxz = ((c.nx + TX - 1) / TX) * ((c.nz + TZ - 1) / TZ);
    int nch = (4 * 148 + nxz - 1) / nxz;
    if (nch > c.ny / 4) nch = c.ny / 4;
    if (nch < 1) nch = 1;
    return (c.ny + nch - 1) / nch;
}

// one wave: two resident CTAs per SM (shared memory and registers allow 2)
size_t rhs_grid_blocks(const DConst& c) {
    const long long rows = (long long)((c.nx + TX - 1) / TX) * ((c.nz + TZ - 1) / TZ) * c.ny;
    const long long b = 2LL * (c.nsm > 0 ? c.nsm : 148);
    return (size_t)(rows < b ? rows : b);
}

void rhs_init() {
    cudaFuncSetAttribute(k_rhs_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, NB * 4 * SLAB * 8);
    cudaFuncSetAttribute(k_rhs_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, NB * 5 * SLAB * 8);
}

void launch_rhs_tile(cudaStream_t st, const DConst& c, const DMetric& m, DCoef* coef, const Fields& f, double* uy_ym,
                     double* duy_ym, int ns, double gam, double the, double alp, double* part, unsigned int* counter) {
    const int yc = rhs_ychunk(c);
    dim3 grd((unsigned)rhs_grid_blocks(c));
    dim3 blk(32, TZ / ZC);
    if (c.scalar_on)
        launch_pdl(k_rhs_tile<true>, grd, blk, NB * 5 * SLAB * 8, st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp,
                   yc, part, counter);
    else
        launch_pdl(k_rhs_tile<false>, grd, blk, NB * 4 * SLAB * 8, st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp,
                   yc, part, counter);
}

}  // namespace ptc
