// div_src.cuh -- the source of the pressure Poisson equation, computed where
// the forward x transform consumes it: the divergence of u* at the two x
// points 2e, 2e+1 of row g = k*ny + (jc-1) (clcPrSrc, src/m_TScheme.f90:
// 48-77: 4th-order staggered differences in x and z, 2nd-order in y).  The
// loads of a point pair are separated from its arithmetic so that a thread
// can put the loads of several pairs in flight before it uses any of them.
#pragma once
#include "common.cuh"

namespace ptc {

struct DivTaps {
    double2 u01, u23, v0, v1, w0, w1, w2, w3;
    double um, rdyp;
};

template <class V>
__device__ __forceinline__ void div_load(DivTaps& t, const DConst& c, const DMetric& m, const V* __restrict__ ux,
                                         const V* __restrict__ uy, const V* __restrict__ uz, int g, int e) {
    const int nx = c.nx, ny = c.ny, nz = c.nz;
    const size_t pl = (size_t)c.nyt * nx;
    const int k = g / ny, jc = g - k * ny + 1;
    const int km = k == 0 ? nz - 1 : k - 1, kp = k == nz - 1 ? 0 : k + 1, ku = kp == nz - 1 ? 0 : kp + 1;
    const int i0 = 2 * e, im = i0 == 0 ? nx - 1 : i0 - 1, i2 = i0 + 2 == nx ? 0 : i0 + 2;
    const size_t r0 = (size_t)jc * nx;
    const V* ur = ux + (size_t)k * pl + r0;
    const V* vr = uy + (size_t)k * pl + r0;
    t.u01 = ld_pair(ur + i0);
    t.u23 = ld_pair(ur + i2);
    t.um = (double)__ldg(ur + im);
    t.v0 = ld_pair(vr + i0);
    t.v1 = ld_pair(vr + nx + i0);
    t.w0 = ld_pair(uz + (size_t)km * pl + r0 + i0);
    t.w1 = ld_pair(uz + (size_t)k * pl + r0 + i0);
    t.w2 = ld_pair(uz + (size_t)kp * pl + r0 + i0);
    t.w3 = ld_pair(uz + (size_t)ku * pl + r0 + i0);
    t.rdyp = __ldg(&m.rdyp[jc]);
}

// (div at 2e, div at 2e+1)
__device__ __forceinline__ double2 div_eval(const DivTaps& t, const DConst& c) {
    const double dudx0 = c.dxC[0] * t.um + c.dxC[1] * t.u01.x + c.dxC[2] * t.u01.y + c.dxC[3] * t.u23.x;
    const double dudx1 = c.dxC[0] * t.u01.x + c.dxC[1] * t.u01.y + c.dxC[2] * t.u23.x + c.dxC[3] * t.u23.y;
    const double dvdy0 = (t.v1.x - t.v0.x) * t.rdyp, dvdy1 = (t.v1.y - t.v0.y) * t.rdyp;
    const double dwdz0 = c.dzC[0] * t.w0.x + c.dzC[1] * t.w1.x + c.dzC[2] * t.w2.x + c.dzC[3] * t.w3.x;
    const double dwdz1 = c.dzC[0] * t.w0.y + c.dzC[1] * t.w1.y + c.dzC[2] * t.w2.y + c.dzC[3] * t.w3.y;
    return make_double2(dudx0 + dvdy0 + dwdz0, dudx1 + dvdy1 + dwdz1);
}

// the source of every point pair f = start, start + STRIDE, ... < B*N of a
// batch of B rows from g0 (pair e of row b = f / N), U pairs in flight per
// thread: st(b, e, value) stores it, the running max|div| goes to dm
template <int N, int B, int STRIDE, int U, class V, class ST>
__device__ __forceinline__ void div_batch(const DConst& c, const DMetric& m, const V* __restrict__ ux,
                                          const V* __restrict__ uy, const V* __restrict__ uz, int g0,
                                          int nrows, double sudtal, int start, double& dm, const ST& st) {
    for (int f0 = start; f0 < B * N; f0 += U * STRIDE) {
        DivTaps tp[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int f = f0 + u * STRIDE;
            const int b = f / N, e = f - b * N;
            ok[u] = f < B * N && g0 + b < nrows;
            if (ok[u]) div_load(tp[u], c, m, ux, uy, uz, g0 + b, e);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int f = f0 + u * STRIDE;
            if (f >= B * N) continue;
            const int b = f / N, e = f - b * N;
            double2 val = make_double2(0.0, 0.0);
            if (ok[u]) {
                const double2 d = div_eval(tp[u], c);
                dm = nmax(dm, nmax(fabs(d.x), fabs(d.y)));
                val = make_double2(sudtal * d.x, sudtal * d.y);
            }
            st(b, e, val);
        }
    }
}

}  // namespace ptc
