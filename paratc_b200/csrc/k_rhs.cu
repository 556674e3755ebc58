// k_rhs.cu -- clcRhsXYZ (src/m_TScheme.f90:113-360) on B200 with
// shared-memory row-slab tiles.
//
// A CTA owns a 32 (x) by 8 (z) column tile and marches up a chunk of y rows.
// For every row j it needs rows j-1, j, j+1 of ux, uy, uz, p (and the
// scalar) over the tile plus the x/z halo of 3 cells that the interpolated
// face velocities and the 4th-order stencils read.  Those row-slabs
// (40 x 14 values per field and row: the x range starts 4 cells left of the
// tile so that every 16-byte pair of values is aligned and never straddles
// the periodic wrap) sit in a ring of 3 + PF slots in shared memory.  In FP64
// the slabs of rows j+2 .. j+1+PF are copied in with 16-byte cp.async while
// row j is computed, one commit group per row, so the HBM loads overlap the
// arithmetic.  The row's metric coefficients (interpolation weights, 1/dy,
// the d2/dy2 stencils) come as one 128-byte record (DMetric::rowmet) in the
// same group, so no global
// load sits on a row's dependent path.  Each thread computes
// two z-adjacent cells per row (FP64; one in the FP32 form): RhsX/RhsY/RhsZ
// (and RhsC) and the new explicit histories, reading every neighbour from
// shared memory; the six interpolated fields of the reference and their halo
// updates never exist.
//
// Two precisions of the same kernel: FP64 (the reference's arithmetic) and a
// mixed form whose stencil arithmetic and row slabs are FP32 while the state,
// the outputs and the flow-rate sum stay FP64.  In the FP32 form the slabs
// take half the shared memory and the registers, so a CTA runs 256 threads
// with one cell each; its row slabs are loaded into registers one row ahead
// and converted when stored, and s3tot sums the wall-normal viscous term
// d22 from FP64 loads of the thread's own column (the x and z second
// differences sum to zero over a periodic line, so they carry nothing into
// s3tot but rounding).
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

constexpr int TX = 32, TZ = 8, HX = 4, HZ = 3;
constexpr int SX = TX + 2 * HX;  // 40: x offsets -4 .. 35 of the tile (the stencils read -3 .. 34)
constexpr int SZ = TZ + 2 * HZ;  // 14
constexpr int SLAB = SX * SZ;    // 560 doubles per field and row
// The launch shape, per precision and compiled variant VAR (the tuner's
// choice, paratc_autotune_all): PF rows loaded ahead beyond row j+1 (copy
// groups in flight; FP64), ZC z-adjacent cells per thread (2 lets the shared
// stencil taps of the two cells load once) and the threads per CTA.
// FP64 variants: 0 PF 1, ZC 2 (128 threads); 1 PF 2, ZC 2; 2 PF 1, ZC 1
// (256 threads).  FP32 storage: 0 ZC 1 (256 threads), 1 ZC 2 (128 threads).
// The mixed form (FP32 arithmetic on FP64 fields) has one variant.
constexpr int RHS_NVAR = 3;
template <class T, int VAR = 0>
struct RhsCfg {
    static constexpr bool F64 = sizeof(T) == 8;
    static constexpr int PF = (F64 && VAR == 1) ? 2 : 1;
    static constexpr int NB = F64 ? 3 + PF : 4;  // ring slots: rows j-1..j+1 and the rows in flight
    // resident CTAs per SM: 2 (FP64 with 2 cells: 3 spills and is slower);
    // 3 for the FP32 storage form's two-cell shape (168 registers, no spills)
    static constexpr int MINB = (!F64 && VAR == 1) ? 3 : 2;
    static constexpr int ZC = F64 ? (VAR != 2 ? 2 : 1) : (VAR == 1 ? 2 : 1);
    static constexpr int NTHR = TX * TZ / ZC;  // 128 or 256
    static constexpr int NSLOT = (SLAB + NTHR - 1) / NTHR;
};
template <bool SCALAR, class T, int VAR = 0>
constexpr size_t rhs_smem_bytes() {
    return (size_t)RhsCfg<T, VAR>::NB * (SCALAR ? 5 : 4) * SLAB * sizeof(T);
}

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// the field a copy reads (f = 0 ux, 1 uy, 2 uz, 3 p, 4 scalar)
__device__ __forceinline__ const double* field_of(const Fields& fl, int f) {
    return f == 0 ? fl.ux : f == 1 ? fl.uy : f == 2 ? fl.uz : f == 3 ? fl.pr : fl.sc;
}
// the float field f (0 ux, 1 uy, 2 uz, 4 scalar) of the FP32 storage form
template <class V>
__device__ __forceinline__ const V* fieldv(const FieldSet<V>& fl, int f) {
    return f == 0 ? fl.ux : f == 1 ? fl.uy : f == 2 ? fl.uz : fl.sc;
}
// one value of field f at offset off, widened to double (the pressure is
// FP64 in every storage form)
template <class V>
__device__ __forceinline__ double ld_field(const FieldSet<V>& fl, int f, size_t off) {
    if (f == 3) return __ldg(fl.pr + off);
    const V* q = f == 0 ? fl.ux : f == 1 ? fl.uy : f == 2 ? fl.uz : fl.sc;
    return (double)__ldg(q + off);
}

__device__ __forceinline__ int modp(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

}  // namespace

// SCALAR: with the scalar transport; T: arithmetic (double, or float for the
// mixed and FP32 storage forms); V: storage of u, v, w, c, Hist and Rhs
// (float only in the FP32 storage form, whose arithmetic is float)
// G: the block this CTA works as (OwnGrid, or SubGrid in a grouped launch).
// MULTI (grouped launches): the member's own launch shape has nlog blocks
// ("logical blocks"), and this CTA runs the consecutive logical blocks
// [nlog*b/B, nlog*(b+1)/B) of the B CTAs the member has here, one after
// another without restarting its row pipeline; it stores the flow-rate
// partial of each logical block as that block's own CTA would, so the
// member's records, and its result, are those of its own launch.
template <bool SCALAR, class T, class V, int VAR, bool MULTI = false, class G>
__device__ __forceinline__ void rhs_body(const G& grid, const DConst& c, const DMetric& m, DCoef* __restrict__ coef,
                                         const FieldSet<V>& fl, double* __restrict__ uy_ym,
                                         double* __restrict__ duy_ym, int ns, double gam, double the, double alp,
                                         double* __restrict__ part, unsigned int* __restrict__ counter,
                                         int nlog = 0) {
    constexpr int NF = SCALAR ? 5 : 4;
    constexpr bool F64 = sizeof(T) == 8;
    static_assert(!F64 || sizeof(V) == 8, "the FP64 arithmetic form keeps FP64 fields");
    using CFG = RhsCfg<T, VAR>;
    constexpr int ZC = CFG::ZC, NTHR = CFG::NTHR, NSLOT = CFG::NSLOT, NB = CFG::NB, PF = CFG::PF;
    // FP64 copies: 16-byte pairs, NPAIR per (field, z-plane) row, NP2 per thread and field
    constexpr int NPAIR = SX / 2, NPR = SZ * NPAIR, NP2 = (NPR + NTHR - 1) / NTHR;
    // FP32 storage: u, v, w (and c) come as 16-byte quads by cp.async (SZ *
    // SX / 4 = 140 per field, NQ2 per thread), the FP64 pressure through
    // registers, converted; needs nx % 4 == 0 (paratc_set_precision checks)
    constexpr bool F32S = !F64 && sizeof(V) == 4;
    constexpr int NQUAD = SZ * (SX / 4), NQ2 = (NQUAD + NTHR - 1) / NTHR;
    extern __shared__ __align__(128) unsigned char sm_raw[];
    T* sm = reinterpret_cast<T*>(sm_raw);  // [NB][NF][SLAB]
    __shared__ __align__(128) double smet[NB][ROWMET];
    const int lane = threadIdx.x, wq = threadIdx.y, tid = wq * 32 + lane;
    const int nx = c.nx, nz = c.nz, ny = c.ny;
    const size_t pl = (size_t)c.nyt * nx;
    // work = the (tile, row) pairs in tile-major order; block b takes the
    // contiguous range [b*W/B, (b+1)*W/B), so one wave of resident blocks
    // covers the grid with at most one row of imbalance
    const int ntx = (nx + TX - 1) / TX, ntz = (nz + TZ - 1) / TZ;
    const long long W = (long long)ntx * ntz * ny;
    long long gbeg = W * grid.x() / grid.gx(), gend = W * (grid.x() + 1) / grid.gx();
    int lb = 0, lb1 = 0;      // MULTI: the logical block being run, and the end of this CTA's
    long long lb_end = 0;     // the work index where logical block lb ends
    if constexpr (MULTI) {
        lb = (int)((long long)nlog * grid.x() / grid.gx());
        lb1 = (int)((long long)nlog * (grid.x() + 1) / grid.gx());
        gbeg = W * lb / nlog;
        gend = W * lb1 / nlog;
        lb_end = W * (lb + 1) / nlog;
    }
    pdl_wait();
    pdl_trigger();

    // PMcoeUpdate from the device dt
    const double dt = coef->dt;
    const double pmGamma = gam * dt, pmTheta = the * dt, pmAlpha = alp * dt;
    const double pmBeta = 0.5 * alp * c.xnu * dt, pmBetaSc = 0.5 * alp * c.sdiff * dt;
    const double tb = 2.0 * pmBeta, tbs = 2.0 * pmBetaSc;
    // stencil constants straight from the parameter bank, in the kernel's precision
#define KC(a64, a32, q) (F64 ? (T)c.a64[q] : (T)c.a32[q])
#define dxC(q) KC(dxC, fdxC, q)
#define dzC(q) KC(dzC, fdzC, q)
#define dxxC(q) KC(dxxC, fdxxC, q)
#define dzzC(q) KC(dzzC, fdzzC, q)
#define grav(q) KC(grav, fgrav, q)
#define gev(q) KC(gev, fgev, q)
#define fvv(q) KC(fvv, ffvv, q)
    const T I1 = KC(IC, fIC, 0), I2 = KC(IC, fIC, 1), I3 = KC(IC, fIC, 2), I4 = KC(IC, fIC, 3);
    const T ucrf = F64 ? (T)c.ucrf : (T)c.fucrf, xnu = F64 ? (T)c.xnu : (T)c.fxnu;
    const T tpG = (T)pmGamma, tpT = (T)pmTheta, tpA = (T)pmAlpha, ttb = (T)tb, ttbs = (T)tbs;
    const T tsdiff = F64 ? (T)c.sdiff : (T)c.fsdiff;
    double s3 = 0.0;

    for (long long g = gbeg; g < gend;) {
        const int tile = (int)(g / ny);
        const int j0 = (int)(g - (long long)tile * ny) + 1;
        const int j1 = (int)min((long long)ny, (long long)j0 + (gend - g) - 1);
        g += j1 - j0 + 1;
        const int i0 = (tile % ntx) * TX, k0 = (tile / ntx) * TZ;
        // FP32 storage: the quads this thread copies for every float field
        size_t gq[NQ2];
        int sq[NQ2];
        bool vq[NQ2];
#pragma unroll
        for (int s4 = 0; s4 < NQ2; s4++) {
            const int e = tid + s4 * NTHR;
            vq[s4] = F32S && e < NQUAD;
            const int zz = e / (SX / 4), qq = e - zz * (SX / 4);
            gq[s4] = vq[s4] ? (size_t)modp(k0 - HZ + zz, nz) * pl + (size_t)modp(i0 - HX + 4 * qq, nx) : 0;
            sq[s4] = zz * SX + 4 * qq;
        }
        // FP32 form: per-thread slab elements, loaded and converted
        size_t goff[F64 ? 1 : NSLOT];
        int soff[F64 ? 1 : NSLOT];
        bool sval[F64 ? 1 : NSLOT];
        if constexpr (!F64) {
#pragma unroll
            for (int s = 0; s < NSLOT; s++) {
                const int e = tid + s * NTHR;
                sval[s] = e < SLAB;
                const int zz = e / SX, xx = e - zz * SX;
                goff[s] = (size_t)modp(k0 - HZ + zz, nz) * pl + (size_t)modp(i0 - HX + xx, nx);
                soff[s] = e;
            }
        }
        // FP64: the 16-byte pairs this thread copies (the same for every field)
        size_t gp[F64 ? NP2 : 1];
        int sp[F64 ? NP2 : 1];
        bool vp[F64 ? NP2 : 1];
        if constexpr (F64) {
#pragma unroll
            for (int q = 0; q < NP2; q++) {
                const int e = tid + q * NTHR;
                vp[q] = e < NPR;
                const int zz = e / NPAIR, pp = e - zz * NPAIR;
                gp[q] = (size_t)modp(k0 - HZ + zz, nz) * pl + (size_t)modp(i0 - HX + 2 * pp, nx);
                sp[q] = zz * SX + 2 * pp;
            }
        }
#define LOAD_ROW64(jrow)                                                                             \
    do {                                                                                             \
        double* dst_ = reinterpret_cast<double*>(sm) + (size_t)((jrow) % NB) * NF * SLAB;           \
        const size_t ro_ = (size_t)(jrow) * nx;                                                      \
        _Pragma("unroll") for (int f_ = 0; f_ < NF; f_++)                                            \
            _Pragma("unroll") for (int q_ = 0; q_ < NP2; q_++) if (vp[q_])                           \
                cp_async16(dst_ + f_ * SLAB + sp[q_], field_of(fl, f_) + gp[q_] + ro_);              \
        if (tid < ROWMET / 2) cp_async16(&smet[(jrow) % NB][2 * tid], m.rowmet + (size_t)(jrow) * ROWMET + 2 * tid); \
    } while (0)
        // FP32: load, convert, store (FP32 storage: the float fields by
        // cp.async quads, the pressure converted)
#define LOAD_ROW32(jrow)                                                                 \
    do {                                                                                 \
        T* dst_ = sm + (size_t)((jrow) % NB) * NF * SLAB;                                \
        const size_t ro_ = (size_t)(jrow) * nx;                                          \
        _Pragma("unroll") for (int f_ = 0; f_ < NF; f_++) {                              \
            if (F32S && f_ != 3) {                                                       \
                _Pragma("unroll") for (int s4_ = 0; s4_ < NQ2; s4_++) if (vq[s4_])       \
                    cp_async16(dst_ + f_ * SLAB + sq[s4_], fieldv(fl, f_) + gq[s4_] + ro_); \
                continue;                                                                \
            }                                                                            \
            _Pragma("unroll") for (int s_ = 0; s_ < NSLOT; s_++) if (sval[s_])           \
                dst_[f_ * SLAB + soff[s_]] = (T)ld_field(fl, f_, goff[s_] + ro_);           \
        }                                                                                \
        if (tid < ROWMET) smet[(jrow) % NB][tid] = __ldg(m.rowmet + (size_t)(jrow) * ROWMET + tid); \
    } while (0)

        if constexpr (F64) {
            // rows j0-1 .. j0+1 in one commit group, rows j0+2 .. j0+PF one group each
            LOAD_ROW64(j0 - 1);
            LOAD_ROW64(j0);
            LOAD_ROW64(j0 + 1);
            cp_async_commit();
#pragma unroll
            for (int d = 2; d <= PF; d++) {
                if (j0 + d <= j1 + 1) LOAD_ROW64(j0 + d);
                cp_async_commit();
            }
        } else {
            LOAD_ROW32(j0 - 1);
            LOAD_ROW32(j0);
            LOAD_ROW32(j0 + 1);
            if constexpr (F32S) {
                cp_async_commit();
                cp_async_wait<0>();
            }
            __syncthreads();
        }

        const int i = i0 + lane;
        int kk[ZC];
        bool act[ZC];
        // explicit histories of the next row are loaded one row ahead, held
        // in their storage type (widened where used, so the loads stay in flight)
        V hxn[ZC], hyn[ZC], hzn[ZC], hcn[ZC];
        V u64m[ZC], u64c[ZC], u64p[ZC];  // FP32 forms: ux of the own column, rows j-1, j, j+1
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
            u64m[cz] = u64c[cz] = u64p[cz] = 0.0;
            if (act[cz]) {
                const size_t q = (size_t)kk[cz] * pl + (size_t)j0 * nx + i;
                hxn[cz] = fl.hx[q]; hyn[cz] = fl.hy[q]; hzn[cz] = fl.hz[q];
                if (SCALAR) hcn[cz] = fl.hc[q];
                if constexpr (!F64) {
                    u64m[cz] = __ldg(&fl.ux[q - nx]);
                    u64c[cz] = __ldg(&fl.ux[q]);
                    u64p[cz] = __ldg(&fl.ux[q + nx]);
                }
            }
        }

        for (int j = j0; j <= j1; j++) {
            // FP32 form: row j+2 in registers now, converted and stored after
            // the arithmetic of row j
            double pre[F64 ? 1 : NF][F64 ? 1 : NSLOT];
            double mpre = 0.0;
            const bool more = j + 2 <= j1 + 1;
            if constexpr (F64) {
                // the slot of row j+1+PF was last read by row j-1's arithmetic,
                // which every thread finished at the barrier closing it
                if (j + 1 + PF <= j1 + 1) LOAD_ROW64(j + 1 + PF);
                cp_async_commit();
            } else {
                if (more) {
                    const size_t ro = (size_t)(j + 2) * nx;
                    T* dst = sm + (size_t)((j + 2) % NB) * NF * SLAB;
#pragma unroll
                    for (int f = 0; f < NF; f++) {
                        if (F32S && f != 3) {
                            // the slot of row j+2 was last read by row j-2's arithmetic
#pragma unroll
                            for (int s4 = 0; s4 < NQ2; s4++)
                                if (vq[s4]) cp_async16(dst + f * SLAB + sq[s4], fieldv(fl, f) + gq[s4] + ro);
                            continue;
                        }
#pragma unroll
                        for (int sl = 0; sl < NSLOT; sl++)
                            pre[f][sl] = sval[sl] ? ld_field(fl, f, goff[sl] + ro) : 0.0;
                    }
                    if (tid < ROWMET) mpre = __ldg(m.rowmet + (size_t)(j + 2) * ROWMET + tid);
                }
                if constexpr (F32S) cp_async_commit();  // one group per row, empty or not
            }
            V hx0a[ZC], hy0a[ZC], hz0a[ZC], hc0a[ZC];
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
            // FP32 form: ux of row j+2 for the next row's s3tot term, one row ahead
            V u64n[ZC];
#pragma unroll
            for (int cz = 0; cz < ZC; cz++)
                u64n[cz] = (!F64 && act[cz] && j + 2 <= ny + 1) ? __ldg(&fl.ux[q0a[cz] + 2 * nx]) : (V)0;
            if constexpr (F64) {
                cp_async_wait<PF>();  // the group holding row j+1 is complete
                __syncthreads();
            } else if constexpr (F32S) {
                cp_async_wait<1>();  // row j+1's quads (the newest group is row j+2's)
                __syncthreads();
            }
            // both cells are computed before any global store, so that the
            // compiler may load a tap the two cells share once
            T o_rx[ZC], o_ry[ZC], o_rz[ZC], o_hx[ZC], o_hy[ZC], o_hz[ZC], o_rc[ZC], o_hc[ZC];
            {
                const T* Sm = sm + (size_t)((j - 1) % NB) * NF * SLAB;
                const T* Sc = sm + (size_t)(j % NB) * NF * SLAB;
                const T* Sp = sm + (size_t)((j + 1) % NB) * NF * SLAB;
#define V(S, f, dx, dz) (S)[(f) * SLAB + (w + HZ + (dz)) * SX + (lane + HX + (dx))]
            const bool top = (j == ny);
            const double* M = smet[j % NB];
#define MET(q) M[q]
            const double IY1d = MET(0), IY3d = MET(1);
            const T IY1 = (T)IY1d, IY2 = (T)(1.0 - IY1d), IY3 = (T)IY3d, IY4 = (T)(1.0 - IY3d);
            const T rdyp = (T)MET(2), rdyc = (T)MET(3);
            const double dyp = MET(4);
            const T ap2c = (T)MET(5), ac2c = (T)MET(6), am2c = (T)MET(7);
#pragma unroll
            for (int cz = 0; cz < ZC; cz++) {
            const int w = wq * ZC + cz;
            const T hx0 = (T)hx0a[cz], hy0 = (T)hy0a[cz], hz0 = (T)hz0a[cz], hc0 = (T)hc0a[cz];
            (void)hc0;

            // ---------------- RhsX (:169-204)
            T conv_x, rhs_x;
            {
                const T uxc = V(Sc, 0, 0, 0), uxjm = V(Sm, 0, 0, 0), uxjp = V(Sp, 0, 0, 0);
                const T uxhyc = IY1 * uxjm + IY2 * uxc;
                const T uxhyp = IY3 * uxc + IY4 * uxjp;
                T h11 = 0;
#pragma unroll
                for (int q = 0; q < 4; q++) {  // uxhx at x offsets -2..1
                    const int d = q - 2;
                    const T uh = I1 * V(Sc, 0, d - 1, 0) + I2 * V(Sc, 0, d, 0) + I3 * V(Sc, 0, d + 1, 0) + I4 * V(Sc, 0, d + 2, 0);
                    h11 = (q == 0) ? dxC(0) * uh * (uh + ucrf) : h11 + dxC(q) * uh * (uh + ucrf);
                }
                const T uyhx_j = I1 * V(Sc, 1, -2, 0) + I2 * V(Sc, 1, -1, 0) + I3 * V(Sc, 1, 0, 0) + I4 * V(Sc, 1, 1, 0);
                const T uyhx_p = top ? T(0) : I1 * V(Sp, 1, -2, 0) + I2 * V(Sp, 1, -1, 0) + I3 * V(Sp, 1, 0, 0) + I4 * V(Sp, 1, 1, 0);
                const T h12 = (uyhx_p * uxhyp - uyhx_j * uxhyc) * rdyp;
                T h13 = 0;
#pragma unroll
                for (int q = 0; q < 4; q++) {  // z offsets -1..2
                    const int d = q - 1;
                    const T uxhz = I1 * V(Sc, 0, 0, d - 2) + I2 * V(Sc, 0, 0, d - 1) + I3 * V(Sc, 0, 0, d) + I4 * V(Sc, 0, 0, d + 1);
                    const T uzhx = I1 * V(Sc, 2, -2, d) + I2 * V(Sc, 2, -1, d) + I3 * V(Sc, 2, 0, d) + I4 * V(Sc, 2, 1, d);
                    h13 = (q == 0) ? dzC(0) * uxhz * uzhx : h13 + dzC(q) * uxhz * uzhx;
                }
                const T d11 = dxxC(0) * V(Sc, 0, -2, 0) + dxxC(1) * V(Sc, 0, -1, 0) + dxxC(2) * uxc + dxxC(3) * V(Sc, 0, 1, 0) + dxxC(4) * V(Sc, 0, 2, 0);
                const T d22 = ap2c * uxjp + ac2c * uxc + am2c * uxjm;
                const T d33 = dzzC(0) * V(Sc, 0, 0, -2) + dzzC(1) * V(Sc, 0, 0, -1) + dzzC(2) * uxc + dzzC(3) * V(Sc, 0, 0, 1) + dzzC(4) * V(Sc, 0, 0, 2);
                const T dcq13 = d11 + d33;
                if constexpr (F64) {
                    if (act[cz]) s3 += SCALAR ? uxc * dyp : (dcq13 + d22) * dyp;
                } else if (act[cz]) {
                    s3 += SCALAR ? u64c[cz] * dyp
                                 : (MET(5) * u64p[cz] + MET(6) * u64c[cz] + MET(7) * u64m[cz]) * dyp;
                }
                conv_x = -h11 - h12 - h13 + xnu * dcq13 + grav(0);
                const T gradp = dxC(0) * V(Sc, 3, -2, 0) + dxC(1) * V(Sc, 3, -1, 0) + dxC(2) * V(Sc, 3, 0, 0) + dxC(3) * V(Sc, 3, 1, 0);
                rhs_x = tpG * conv_x + tpT * hx0 - tpA * gradp + ttb * d22;
            }
            // ---------------- RhsY (:206-236)
            T conv_y, rhs_y;
            {
                const T qsucac = T(0.25) * rdyc;
                T h21 = 0.0, h23 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) {  // offsets -1..2
                    const int d = q - 1;
                    const T uxh = IY1 * V(Sm, 0, d, 0) + IY2 * V(Sc, 0, d, 0) + ucrf;
                    const T uzh = IY1 * V(Sm, 2, 0, d) + IY2 * V(Sc, 2, 0, d);
                    const T uyhx = I1 * V(Sc, 1, d - 2, 0) + I2 * V(Sc, 1, d - 1, 0) + I3 * V(Sc, 1, d, 0) + I4 * V(Sc, 1, d + 1, 0);
                    const T uyhz = I1 * V(Sc, 1, 0, d - 2) + I2 * V(Sc, 1, 0, d - 1) + I3 * V(Sc, 1, 0, d) + I4 * V(Sc, 1, 0, d + 1);
                    h21 = (q == 0) ? dxC(0) * uyhx * uxh : h21 + dxC(q) * uyhx * uxh;
                    h23 = (q == 0) ? dzC(0) * uyhz * uzh : h23 + dzC(q) * uyhz * uzh;
                }
                const T vp = V(Sp, 1, 0, 0), vc = V(Sc, 1, 0, 0), vm = V(Sm, 1, 0, 0);
                const T h22 = ((vp + vc) * (vp + vc) - (vc + vm) * (vc + vm)) * qsucac;
                const T d11 = dxxC(0) * V(Sc, 1, -2, 0) + dxxC(1) * V(Sc, 1, -1, 0) + dxxC(2) * vc + dxxC(3) * V(Sc, 1, 1, 0) + dxxC(4) * V(Sc, 1, 2, 0);
                const T d22 = (T)MET(8) * vp + (T)MET(9) * vc + (T)MET(10) * vm;
                const T d33 = dzzC(0) * V(Sc, 1, 0, -2) + dzzC(1) * V(Sc, 1, 0, -1) + dzzC(2) * vc + dzzC(3) * V(Sc, 1, 0, 1) + dzzC(4) * V(Sc, 1, 0, 2);
                conv_y = -h21 - h22 - h23 + xnu * (d11 + d33) + grav(1);
                const T gradp = (V(Sc, 3, 0, 0) - V(Sm, 3, 0, 0)) * rdyc;
                rhs_y = tpG * conv_y + tpT * hy0 - tpA * gradp + ttb * d22;
            }
            // ---------------- RhsZ (:238-267)
            T conv_z, rhs_z;
            {
                const T uzc = V(Sc, 2, 0, 0);
                const T uzhyc = IY1 * V(Sm, 2, 0, 0) + IY2 * uzc;
                const T uzhyp = IY3 * uzc + IY4 * V(Sp, 2, 0, 0);
                T h31 = 0.0, h33 = 0.0;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int d = q - 1;  // x offsets -1..2 for h31
                    const T uzhx = I1 * V(Sc, 2, d - 2, 0) + I2 * V(Sc, 2, d - 1, 0) + I3 * V(Sc, 2, d, 0) + I4 * V(Sc, 2, d + 1, 0);
                    const T uxhz = I1 * V(Sc, 0, d, -2) + I2 * V(Sc, 0, d, -1) + I3 * V(Sc, 0, d, 0) + I4 * V(Sc, 0, d, 1);
                    h31 = (q == 0) ? dxC(0) * uzhx * (uxhz + ucrf) : h31 + dxC(q) * uzhx * (uxhz + ucrf);
                    const int e = q - 2;  // z offsets -2..1 for h33
                    const T uzhz = I1 * V(Sc, 2, 0, e - 1) + I2 * V(Sc, 2, 0, e) + I3 * V(Sc, 2, 0, e + 1) + I4 * V(Sc, 2, 0, e + 2);
                    h33 = (q == 0) ? dzC(0) * uzhz * uzhz : h33 + dzC(q) * uzhz * uzhz;
                }
                const T uyhz_j = I1 * V(Sc, 1, 0, -2) + I2 * V(Sc, 1, 0, -1) + I3 * V(Sc, 1, 0, 0) + I4 * V(Sc, 1, 0, 1);
                const T uyhz_p = top ? T(0) : I1 * V(Sp, 1, 0, -2) + I2 * V(Sp, 1, 0, -1) + I3 * V(Sp, 1, 0, 0) + I4 * V(Sp, 1, 0, 1);
                const T h32 = (uyhz_p * uzhyp - uyhz_j * uzhyc) * rdyp;
                const T d11 = dxxC(0) * V(Sc, 2, -2, 0) + dxxC(1) * V(Sc, 2, -1, 0) + dxxC(2) * uzc + dxxC(3) * V(Sc, 2, 1, 0) + dxxC(4) * V(Sc, 2, 2, 0);
                const T d22 = ap2c * V(Sp, 2, 0, 0) + ac2c * uzc + am2c * V(Sm, 2, 0, 0);
                const T d33 = dzzC(0) * V(Sc, 2, 0, -2) + dzzC(1) * V(Sc, 2, 0, -1) + dzzC(2) * uzc + dzzC(3) * V(Sc, 2, 0, 1) + dzzC(4) * V(Sc, 2, 0, 2);
                conv_z = -h31 - h32 - h33 + xnu * (d11 + d33) + grav(2);
                const T gradp = dzC(0) * V(Sc, 3, 0, -2) + dzC(1) * V(Sc, 3, 0, -1) + dzC(2) * V(Sc, 3, 0, 0) + dzC(3) * V(Sc, 3, 0, 1);
                rhs_z = tpG * conv_z + tpT * hz0 - tpA * gradp + ttb * d22;
            }
            if (SCALAR) {
                // ---------------- scalar transport (:302-357)
                const T scc = V(Sc, 4, 0, 0), scjm = V(Sm, 4, 0, 0), scjp = V(Sp, 4, 0, 0);
                const T shyc = IY1 * scjm + IY2 * scc;
                const T shyp = IY3 * scc + IY4 * scjp;
                T hc1 = 0, hc3 = 0, shx0 = 0, shz0 = 0;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int d = q - 1;
                    const T shx = I1 * V(Sc, 4, d - 2, 0) + I2 * V(Sc, 4, d - 1, 0) + I3 * V(Sc, 4, d, 0) + I4 * V(Sc, 4, d + 1, 0);
                    const T shz = I1 * V(Sc, 4, 0, d - 2) + I2 * V(Sc, 4, 0, d - 1) + I3 * V(Sc, 4, 0, d) + I4 * V(Sc, 4, 0, d + 1);
                    if (q == 1) { shx0 = shx; shz0 = shz; }
                    const T ua = V(Sc, 0, d, 0) + fvv(0);
                    const T wa = V(Sc, 2, 0, d) + fvv(2);
                    hc1 = (q == 0) ? dxC(0) * ua * shx : hc1 + dxC(q) * ua * shx;
                    hc3 = (q == 0) ? dzC(0) * wa * shz : hc3 + dzC(q) * wa * shz;
                }
                const T c1 = gev(0) * shx0, c2 = gev(1) * shyc, c3 = gev(2) * shz0;
                rhs_x = rhs_x + tpG * c1;
                rhs_y = rhs_y + tpG * c2;
                rhs_z = rhs_z + tpG * c3;
                conv_x = conv_x + c1;
                conv_y = conv_y + c2;
                conv_z = conv_z + c3;
                const T hc2 = ((V(Sp, 1, 0, 0) + fvv(1)) * shyp - (V(Sc, 1, 0, 0) + fvv(1)) * shyc) * rdyp;
                const T d11 = dxxC(0) * V(Sc, 4, -2, 0) + dxxC(1) * V(Sc, 4, -1, 0) + dxxC(2) * scc + dxxC(3) * V(Sc, 4, 1, 0) + dxxC(4) * V(Sc, 4, 2, 0);
                const T d22 = (T)MET(11) * scjp + (T)MET(12) * scc + (T)MET(13) * scjm;
                const T d33 = dzzC(0) * V(Sc, 4, 0, -2) + dzzC(1) * V(Sc, 4, 0, -1) + dzzC(2) * scc + dzzC(3) * V(Sc, 4, 0, 1) + dzzC(4) * V(Sc, 4, 0, 2);
                const T convc = -hc1 - hc2 - hc3 + tsdiff * (d11 + d33);
                o_rc[cz] = tpG * convc + tpT * hc0 + ttbs * d22;
                o_hc[cz] = convc;
            }
#undef V
#undef MET
            o_rx[cz] = rhs_x; o_ry[cz] = rhs_y; o_rz[cz] = rhs_z;
            o_hx[cz] = conv_x; o_hy[cz] = conv_y; o_hz[cz] = conv_z;
            }
            }
#pragma unroll
            for (int cz = 0; cz < ZC; cz++) {
                if (!act[cz]) continue;
                const size_t q0 = q0a[cz];
                fl.rx[q0] = (V)o_rx[cz];
                fl.ry[q0] = (V)o_ry[cz];
                fl.rz[q0] = (V)o_rz[cz];
                fl.hx[q0] = (V)o_hx[cz];
                fl.hy[q0] = (V)o_hy[cz];
                fl.hz[q0] = (V)o_hz[cz];
                if (SCALAR) {
                    fl.rc[q0] = (V)o_rc[cz];
                    fl.hc[q0] = (V)o_hc[cz];
                }
            }
            if constexpr (!F64) {
                if (more) {
                    T* dst = sm + (size_t)((j + 2) % NB) * NF * SLAB;
#pragma unroll
                    for (int f = 0; f < NF; f++) {
                        if (F32S && f != 3) continue;  // copied by cp.async
#pragma unroll
                        for (int sl = 0; sl < NSLOT; sl++)
                            if (sval[sl]) dst[f * SLAB + soff[sl]] = (T)pre[f][sl];
                    }
                    if (tid < ROWMET) smet[(j + 2) % NB][tid] = mpre;
                }
#pragma unroll
                for (int cz = 0; cz < ZC; cz++) { u64m[cz] = u64c[cz]; u64c[cz] = u64p[cz]; u64p[cz] = u64n[cz]; }
            }
        __syncthreads();
            if constexpr (MULTI) {
                // row j was work item tile*ny + j - 1: a logical block ends here
                if ((long long)tile * ny + j == lb_end && lb + 1 < lb1) {
                    double v[1] = {s3};
                    block_sum_store<1>(v, part + lb);
                    __syncthreads();  // its scratch is reused by the next store
                    s3 = 0.0;
                    lb++;
                    lb_end = W * (lb + 1) / nlog;
                }
            }
        }
#undef LOAD_ROW32
#undef LOAD_ROW64
    }
    if constexpr (F64) cp_async_wait<0>();
#undef KC
#undef dxC
#undef dzC
#undef dxxC
#undef dzzC
#undef grav
#undef gev
#undef fvv

    // flow-rate constraint and the substep coefficients (last CTA)
    double s3v[1] = {s3};
    const unsigned int nblocks = grid.gx() * grid.gy() * grid.gz();
    const int bid = grid.x() + grid.gx() * (grid.y() + grid.gy() * grid.z());
    block_sum_store<1>(s3v, part + (MULTI ? lb : bid));
    if (!last_block_arrive(counter, nblocks)) return;
    double tot[1];
    reduce_records<1, false>(part, MULTI ? nlog : (int)nblocks, tot);
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

// the arguments of a grouped launch's member, read from shared memory; fill(a)
// writes the record
template <bool SCALAR, class T, class V, int VAR, bool MULTI, class Fill>
__device__ __forceinline__ void rhs_from_shared(const SubGrid& g, Fill fill, int ns) {
    __shared__ RhsArgs<V> a;
    fill(a);
    __syncthreads();
    rhs_body<SCALAR, T, V, VAR, MULTI>(g, a.c, a.m, a.coef, a.fl, a.uy_ym, a.duy_ym, ns, a.gam, a.the, a.alp,
                                       a.part, a.counter, a.nlog);
}

template <bool SCALAR, class T, class V, int VAR>
__global__ void __launch_bounds__(RhsCfg<T, VAR>::NTHR, RhsCfg<T, VAR>::MINB)
    k_rhs_tile(DConst c, DMetric m, DCoef* __restrict__ coef, FieldSet<V> fl, double* __restrict__ uy_ym,
               double* __restrict__ duy_ym, int ns, double gam, double the, double alp, double* __restrict__ part,
               unsigned int* __restrict__ counter) {
    rhs_body<SCALAR, T, V, VAR>(OwnGrid{}, c, m, coef, fl, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
}

// the members of an ensemble in one launch: member i's blocks run its own
// launch shape on its own fields
// (the member's record is copied to shared memory first: read from there,
// its constants are reloaded after the barriers of the row loop rather than
// held in registers, which the one-context FP64 kernel takes straight from
// its parameter bank)
template <bool SCALAR, class T, class V, int VAR>
__global__ void __launch_bounds__(RhsCfg<T, VAR>::NTHR, RhsCfg<T, VAR>::MINB)
    k_rhs_grp(const GrpTab<RhsArgs<V>>* __restrict__ t, int ns) {
    static_assert(sizeof(RhsArgs<V>) % 8 == 0, "copied in 8-byte words");
    SubGrid g;
    const int mi = grp_member(t, g);
    rhs_from_shared<SCALAR, T, V, VAR, true>(
        g,
        [&](RhsArgs<V>& a) {
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&t->e[mi]);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(&a);
            for (int w = threadIdx.y * 32 + threadIdx.x; w < (int)(sizeof(RhsArgs<V>) / 8);
                 w += RhsCfg<T, VAR>::NTHR)
                dst[w] = __ldg(&src[w]);
        },
        ns);
}

// ---------------------------------------------------------------------------
// one wave of resident CTAs (MINB per SM for the precision; the record
// count is sized for the larger)
static size_t rhs_blocks(const DConst& c, int minb) {
    const long long rows = (long long)((c.nx + TX - 1) / TX) * ((c.nz + TZ - 1) / TZ) * c.ny;
    const long long b = (long long)minb * (c.nsm > 0 ? c.nsm : 148);
    return (size_t)(rows < b ? rows : b);
}

size_t rhs_grid_blocks(const DConst& c) {
    return rhs_blocks(c, 3);  // the largest MINB of the variants
}

int rhs_variants() { return RHS_NVAR; }
// the launch shapes the tuner tries per precision form: FP64 3, FP32
// storage 2, mixed 1
int rhs_variants(int prec) { return prec == 0 ? RHS_NVAR : (prec == 2 ? 2 : 1); }

void rhs_init() {
#define RHS_ATTR(S, T, V, VAR)                                                                            \
    cudaFuncSetAttribute(k_rhs_tile<S, T, V, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                         (int)rhs_smem_bytes<S, T, VAR>());                                            \
    cudaFuncSetAttribute(k_rhs_grp<S, T, V, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                         (int)rhs_smem_bytes<S, T, VAR>());
    RHS_ATTR(false, double, double, 0) RHS_ATTR(true, double, double, 0)
    RHS_ATTR(false, double, double, 1) RHS_ATTR(true, double, double, 1)
    RHS_ATTR(false, double, double, 2) RHS_ATTR(true, double, double, 2)
    RHS_ATTR(false, float, double, 0) RHS_ATTR(true, float, double, 0)
    RHS_ATTR(false, float, float, 0) RHS_ATTR(true, float, float, 0)
    RHS_ATTR(false, float, float, 1) RHS_ATTR(true, float, float, 1)
#undef RHS_ATTR
}

template <bool SCALAR, class T, int VAR, class V>
static void launch_rhs_t(cudaStream_t st, const DConst& c, const DMetric& m, DCoef* coef, const FieldSet<V>& f,
                         double* uy_ym, double* duy_ym, int ns, double gam, double the, double alp, double* part,
                         unsigned int* counter) {
    using CFG = RhsCfg<T, VAR>;
    const dim3 grd((unsigned)rhs_blocks(c, CFG::MINB));
    const dim3 blk(32, TZ / CFG::ZC);
    launch_pdl(k_rhs_tile<SCALAR, T, V, VAR>, grd, blk, rhs_smem_bytes<SCALAR, T, VAR>(), st, c, m, coef, f, uy_ym,
               duy_ym, ns, gam, the, alp, part, counter);
}

template <bool SCALAR>
static void launch_rhs64(cudaStream_t st, const DConst& c, const DMetric& m, DCoef* coef, const Fields& f,
                         double* uy_ym, double* duy_ym, int ns, double gam, double the, double alp, double* part,
                         unsigned int* counter) {
    if (c.rhs_var == 1)
        launch_rhs_t<SCALAR, double, 1>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
    else if (c.rhs_var == 2)
        launch_rhs_t<SCALAR, double, 2>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
    else
        launch_rhs_t<SCALAR, double, 0>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
}

void launch_rhs_tile(cudaStream_t st, const DConst& c, const DMetric& m, DCoef* coef, const Fields& f, double* uy_ym,
                     double* duy_ym, int ns, double gam, double the, double alp, double* part, unsigned int* counter) {
    if (c.fp32_rhs) {
        if (c.scalar_on) launch_rhs_t<true, float, 0>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
        else launch_rhs_t<false, float, 0>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
    } else {
        if (c.scalar_on) launch_rhs64<true>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
        else launch_rhs64<false>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
    }
}

// ---- grouped launches: the shape of one member's launch, and one launch
// over a table of members that share the instantiation (scalar, arithmetic,
// storage, launch shape)
dim3 rhs_member_grid(const DConst& c, int f32arith) {
    return dim3((unsigned)rhs_blocks(c, f32arith ? RhsCfg<float, 0>::MINB : RhsCfg<double, 0>::MINB));
}

long long rhs_work_rows(const DConst& c) { return (long long)((c.nx + TX - 1) / TX) * ((c.nz + TZ - 1) / TZ) * c.ny; }

int rhs_wave(const DConst& c) { return RhsCfg<double, 0>::MINB * (c.nsm > 0 ? c.nsm : 148); }

template <bool SCALAR, class T, int VAR, class V>
static void rhs_grp_t(cudaStream_t st, const GrpTab<RhsArgs<V>>* t, int nblk, int ns) {
    using CFG = RhsCfg<T, VAR>;
    launch_pdl(k_rhs_grp<SCALAR, T, V, VAR>, dim3((unsigned)nblk), dim3(32, TZ / CFG::ZC),
               rhs_smem_bytes<SCALAR, T, VAR>(), st, t, ns);
}

void launch_rhs_grp(cudaStream_t st, const DConst& key, const GrpTab<RhsArgs<double>>* t, int nblk, int ns) {
    const bool s = key.scalar_on != 0;
    if (key.fp32_rhs) {
        if (s) rhs_grp_t<true, float, 0>(st, t, nblk, ns);
        else rhs_grp_t<false, float, 0>(st, t, nblk, ns);
    } else if (key.rhs_var == 1) {
        if (s) rhs_grp_t<true, double, 1>(st, t, nblk, ns);
        else rhs_grp_t<false, double, 1>(st, t, nblk, ns);
    } else if (key.rhs_var == 2) {
        if (s) rhs_grp_t<true, double, 2>(st, t, nblk, ns);
        else rhs_grp_t<false, double, 2>(st, t, nblk, ns);
    } else {
        if (s) rhs_grp_t<true, double, 0>(st, t, nblk, ns);
        else rhs_grp_t<false, double, 0>(st, t, nblk, ns);
    }
}

void launch_rhs_grp(cudaStream_t st, const DConst& key, const GrpTab<RhsArgs<float>>* t, int nblk, int ns) {
    if (key.scalar_on) rhs_grp_t<true, float, 0>(st, t, nblk, ns);
    else rhs_grp_t<false, float, 0>(st, t, nblk, ns);
}

void launch_rhs_tile(cudaStream_t st, const DConst& c, const DMetric& m, DCoef* coef, const Fields32& f, double* uy_ym,
                     double* duy_ym, int ns, double gam, double the, double alp, double* part, unsigned int* counter) {
    if (c.rhs_var == 1) {
        if (c.scalar_on) launch_rhs_t<true, float, 1>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
        else launch_rhs_t<false, float, 1>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
    } else {
        if (c.scalar_on) launch_rhs_t<true, float, 0>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
        else launch_rhs_t<false, float, 0>(st, c, m, coef, f, uy_ym, duy_ym, ns, gam, the, alp, part, counter);
    }
}

}  // namespace ptc
