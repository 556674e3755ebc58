// k_tridiag.cu -- wall-normal tridiagonal solves on B200.
//
// Both the implicit Helmholtz systems (I - beta*Lyy) du = Rhs of clcU1Hat /
// clcU2Hat / clcU3Hat / clcScalar (src/m_TScheme.f90:365-506) and the
// spectral Poisson systems (Lyy + lambda_x + lambda_z) phi = f of clcPPE
// (src/m_Poisson.f90:383-430) are many independent tridiagonal systems along
// y, one per (x, z) column.  The reference sweeps them with the serial Thomas
// algorithm InverseTridiagonal (src/m_Tools.f90:224-251), and across ranks
// with the reduced-system ("PaScaL") Thomas of clcPPE_x1_reduce
// (src/m_Poisson.f90:457-695).
//
// The matrices never depend on the column's data, only on the row (the
// Helmholtz systems, per step) or on the row and the wavenumber pair (the
// Poisson systems, per context).  So the Thomas pivots are computed apart
// from the solves, and a solve is a chain of multiply-adds per column with
// its loads issued ahead: k_helm (pivots per step, k_helm_factors) and
// k_ys_staged / k_ys_global (pivots per context, k_pois_factors).  The
// partitioned reduced-system solver (part_eliminate / part_reduced /
// k_ysolve) computes its pivots in place; the allocation-free Poisson entry
// point uses it because it has no room to keep pivots between calls.
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"

namespace ptc {

// local elimination of one partition of MR rows (MR >= 3), the modified
// Thomas sweep of src/m_Poisson.f90:496-537 in registers.  On exit row 0 reads
// a0*x_prev + x0 + c0*x_last = f0, row r (1..MR-2) a_r*x0 + x_r + c_r*x_last
// = f_r, row MR-1 a*x0 + x_last + c*x_next = f.  MR is a compile-time
// constant so that every register array index is static; rows past ny are
// identity rows (a = c = f = 0, b = 1), decoupled from the system.
template <int MAXM, int NC, class GetB>
__device__ __forceinline__ void part_eliminate(double (&a)[MAXM], double (&c)[MAXM], double (&f)[MAXM][NC],
                                               const GetB& getb) {
    {
        const double b0 = getb(0), b1 = getb(1);
        a[0] = a[0] / b0;
        c[0] = c[0] / b0;
        a[1] = a[1] / b1;
        c[1] = c[1] / b1;
#pragma unroll
        for (int q = 0; q < NC; q++) {
            f[0][q] = f[0][q] / b0;
            f[1][q] = f[1][q] / b1;
        }
    }
#pragma unroll
    for (int r = 2; r < MAXM; r++) {
        const double rr = 1.0 / (getb(r) - a[r] * c[r - 1]);
#pragma unroll
        for (int q = 0; q < NC; q++) f[r][q] = rr * (f[r][q] - a[r] * f[r - 1][q]);
        c[r] = rr * c[r];
        a[r] = -(rr * a[r] * a[r - 1]);
    }
#pragma unroll
    for (int r = MAXM - 3; r >= 1; r--) {
#pragma unroll
        for (int q = 0; q < NC; q++) f[r][q] = f[r][q] - c[r] * f[r + 1][q];
        a[r] = a[r] - c[r] * a[r + 1];
        c[r] = -(c[r] * c[r + 1]);
    }
    {
        const double rr = 1.0 / (1.0 - a[1] * c[0]);
#pragma unroll
        for (int q = 0; q < NC; q++) f[0][q] = rr * (f[0][q] - c[0] * f[1][q]);
        a[0] = rr * a[0];
        c[0] = -(rr * c[0] * c[1]);
    }
}

// writes the two reduced rows of this partition, solves the reduced systems
// (one column per lane of warp 0), returns x_first / x_last of the partition
template <int MAXM, int NC>
__device__ __forceinline__ void part_reduced(int P, int w, int lane, const double (&a)[MAXM], const double (&c)[MAXM],
                                             const double (&f)[MAXM][NC], double* sm, double (&xf)[NC], double (&xl)[NC]) {
    const int n2 = 2 * P;
    double* RA = sm;                          // [n2][32]
    double* RC = RA + n2 * 32;                // [n2][32]
    double* RW = RC + n2 * 32;                // [n2][32] Thomas factors
    double* RF = RW + n2 * 32;                // [n2][NC][32]
    const double al = a[MAXM - 1], cl = c[MAXM - 1];
    double fl[NC];
#pragma unroll
    for (int q = 0; q < NC; q++) fl[q] = f[MAXM - 1][q];
    const int r0 = 2 * w, r1 = 2 * w + 1;
    RA[r0 * 32 + lane] = a[0];
    RC[r0 * 32 + lane] = c[0];
    RA[r1 * 32 + lane] = al;
    RC[r1 * 32 + lane] = cl;
#pragma unroll
    for (int q = 0; q < NC; q++) {
        RF[(r0 * NC + q) * 32 + lane] = f[0][q];
        RF[(r1 * NC + q) * 32 + lane] = fl[q];
    }
    __syncthreads();
    if (w == 0) {
        // unit-diagonal Thomas (InverseTridiagonal, src/m_Tools.f90:224-251)
        double vecm = 1.0;
        double fp[NC];
#pragma unroll
        for (int q = 0; q < NC; q++) fp[q] = RF[(0 * NC + q) * 32 + lane];
        for (int r = 1; r < n2; r++) {
            const double arr = RC[(r - 1) * 32 + lane] / vecm;
            const double ar = RA[r * 32 + lane];
            RW[r * 32 + lane] = arr;
            vecm = 1.0 - ar * arr;
#pragma unroll
            for (int q = 0; q < NC; q++) {
                const double v = (RF[(r * NC + q) * 32 + lane] - ar * fp[q]) / vecm;
                RF[(r * NC + q) * 32 + lane] = v;
                fp[q] = v;
            }
        }
        for (int r = n2 - 2; r >= 0; r--) {
            const double arr = RW[(r + 1) * 32 + lane];
#pragma unroll
            for (int q = 0; q < NC; q++) {
                const double v = RF[(r * NC + q) * 32 + lane] - arr * fp[q];
                RF[(r * NC + q) * 32 + lane] = v;
                fp[q] = v;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NC; q++) {
        xf[q] = RF[(r0 * NC + q) * 32 + lane];
        xl[q] = RF[(r1 * NC + q) * 32 + lane];
    }
}

// diagonal of row r of a partition starting at Fortran row s
struct PoisDiag {
    const double* ac2ph;
    double lam;
    int s, ny;
    bool dc;  // kx = kz = 0: row 1 is the identity
    __device__ __forceinline__ double operator()(int r) const {
        const int jc = s + r;
        if (jc > ny || (dc && jc == 1)) return 1.0;
        return __ldg(&ac2ph[jc]) + lam;
    }
};

// ---------------------------------------------------------------------------
// Helmholtz: comp 0 ux (clcU1Hat), 1 uy (clcU2Hat), 2 uz (clcU3Hat),
// 3 scalar (clcScalar); u(jc) += du(jc) with (I - beta*Lyy) du = Rhs
// (src/m_TScheme.f90:365-506).  The matrices depend on the row only, so
// their Thomas pivots (InverseTridiagonal, src/m_Tools.f90:224-251) are
// computed once per step by k_helm_factors: for matrix (ns, type) and row jc,
// A = a(jc), RV = 1/vecm(jc), AR = arr(jc), evaluated in the reference's
// order without contraction.  A warp then sweeps 32 adjacent columns (i)
// straight from memory: rows come in chunks of HY_U held in a three-chunk
// register ring, so two chunks are in flight while one is on the dependent
// chain.  The forward sweep writes f(jc) back over Rhs (it stays in L2 for
// the backward sweep), the backward sweep adds the solution to u.
// uy and the scalar also get the ghost values that
// SetBC_and_UpdateHaloForPrSrc / _scalar give them.
// ---------------------------------------------------------------------------
namespace {
// rows per chunk (three chunks in registers, two in flight): 8, or 4 in the
// tuner's second variant (DConst::helm_var = 1); twice that for float storage
constexpr int HY_U = 8;
constexpr int HELM_NVAR = 2;
__host__ __device__ inline int helm_stride(int ny) { return 3 * (ny + 2); }
}  // namespace

// thread = column i = 128*blockIdx.x + 32*threadIdx.y + lane at z index
// blockIdx.y, component comp0 + blockIdx.z: the four warps of a CTA read
// one contiguous 1 KB stretch of a row together.  The pivots sit in shared
// memory; rows are addressed by pointer steps; the wall rows need no case of
// their own in the sweeps (a(1) = 0, arr(ny+1) = 0, and clcU2Hat's row-1
// value is substituted before the sweep and its result after it).
// G: the block this CTA works as (OwnGrid, or SubGrid in a grouped launch).
// Z4: the grouped launch's CTA shape, 32 columns of 4 z planes (one per
// warp), so that a narrow member (nx < 128) leaves no warp idle.
// W: the sweeps' arithmetic, double (FP64 in every form), or float for the
// FP32 storage form's third launch shape, whose rows are stored in float
// anyway: widening each value to FP64 and rounding it back put conversions
// and FP64 latencies on every row of the chain
template <class V, int HU, bool Z4 = false, class W = double, class G>
__device__ __forceinline__ void helm_body(const G& grid, const DConst& cst, const DCoef* __restrict__ coef, int comp0,
                                          const FieldSet<V>& fl, const double* __restrict__ duy_ym,
                                          const double* __restrict__ uy_ym, const double* __restrict__ facs) {
    extern __shared__ double shf[];
    const int nx = cst.nx, ny = cst.ny;
    const int comp = comp0 + (int)grid.z();
    const int t = comp == 1 ? 1 : (comp == 3 ? 2 : 0);
    pdl_wait();
    pdl_trigger();
    {
        const double* F = facs + (size_t)((coef->ns - 1) * 3 + t) * helm_stride(ny);
        const int tid = threadIdx.y * 32 + threadIdx.x;
        W* shw = reinterpret_cast<W*>(shf);
        for (int q = tid; q < helm_stride(ny); q += 128) shw[q] = (W)F[q];
    }
    __syncthreads();
    const W* SA = reinterpret_cast<const W*>(shf);
    const W* SR = SA + (ny + 2);
    const W* SW = SA + 2 * (ny + 2);
    const int i = Z4 ? (int)grid.x() * 32 + (int)threadIdx.x : (int)(grid.x() * 4 + threadIdx.y) * 32 + (int)threadIdx.x;
    const int k = Z4 ? (int)grid.y() * 4 + (int)threadIdx.y : (int)grid.y();
    if (i >= nx || (Z4 && k >= cst.nz)) return;
    V* u;
    V* rhs;
    double add = 0.0;
    if (comp == 0)      { u = fl.ux; rhs = fl.rx; add = coef->rhsx_add; }
    else if (comp == 1) { u = fl.uy; rhs = fl.ry; }
    else if (comp == 2) { u = fl.uz; rhs = fl.rz; }
    else                { u = fl.sc; rhs = fl.rc; }
    const size_t col = (size_t)k * cst.nyt * nx + i;
    // the sweeps run in W (FP64 unless chosen otherwise): loads convert, stores round
    const W addw = (W)add;
    V* rc = rhs + col;
    V* uc = u + col;
    const int nch = (ny + HU - 1) / HU;

    // forward sweep, rows 1..ny: f = ((r + add) - a f_prev) / vecm, written over Rhs
    const double a0 = (comp == 1) ? duy_ym[(size_t)k * nx + i] : 0.0;
    // the register ring holds rows in their storage type and widens them
    // where they are used, so that the loads of later chunks stay in flight
    V A[HU], B[HU], C[HU];
    auto ldr = [&](V (&X)[HU], int cc) {
        if (cc >= nch) return;
        const V* b = rc + (size_t)(cc * HU + 1) * nx;
        const int nr = ny - cc * HU;
#pragma unroll
        for (int q = 0; q < HU; q++) {
            if (q < nr) X[q] = *b;
            b += nx;
        }
    };
    W fp = 0;
    V* wp = rc + nx;
    auto fwd = [&](const V (&X)[HU], int cc) {
        if (cc >= nch) return;
        const int nr = ny - cc * HU;
        const W* sa = SA + cc * HU + 1;
        const W* sr = SR + cc * HU + 1;
#pragma unroll
        for (int q = 0; q < HU; q++) {
            if (q < nr) {
                // clcU2Hat: the row-1 value is the wall increment (kept in FP64)
                const W xq = (comp == 1 && cc == 0 && q == 0) ? (W)a0 : (W)X[q];
                const W f = ((xq + addw) - sa[q] * fp) * sr[q];
                *wp = (V)f;
                fp = f;  // the chain stays in W (no conversion on the dependent path)
            }
            wp += nx;
        }
    };
    ldr(A, 0);
    ldr(B, 1);
    ldr(C, 2);
    for (int c = 0; c < nch; c += 3) {
        fwd(A, c);
        ldr(A, c + 3);
        fwd(B, c + 1);
        ldr(B, c + 4);
        fwd(C, c + 2);
        ldr(C, c + 5);
    }
    // backward sweep, rows ny..1: x = f - arr(j+1) x(j+1), u += x
    V DA[HU], DB[HU], DC[HU], UA[HU], UB[HU], UC[HU];
    auto ldb = [&](V (&D)[HU], V (&U)[HU], int cc) {
        if (cc >= nch) return;
        const size_t off = (size_t)(ny - cc * HU) * nx;
        const V* bd = rc + off;
        const V* bu = uc + off;
        const int nr = ny - cc * HU;
#pragma unroll
        for (int q = 0; q < HU; q++) {
            if (q < nr) { D[q] = *bd; U[q] = *bu; }
            bd -= nx;
            bu -= nx;
        }
    };
    W xn = 0, unew = 0, utop = 0;
    V* up = uc + (size_t)ny * nx;
    auto bwd = [&](const V (&D)[HU], const V (&U)[HU], int cc) {
        if (cc >= nch) return;
        const int nr = ny - cc * HU;
        const W* sw = SW + ny + 1 - cc * HU;
#pragma unroll
        for (int q = 0; q < HU; q++) {
            if (q < nr) {
                const W x = (W)D[q] - sw[-q] * xn;
                xn = x;
                unew = (W)U[q] + x;
                *up = (V)unew;
            }
            up -= nx;
        }
    };
    ldb(DA, UA, 0);
    ldb(DB, UB, 1);
    ldb(DC, UC, 2);
    for (int c = 0; c < nch; c += 3) {
        bwd(DA, UA, c);
        if (c == 0) utop = (W)DA[0] + (W)UA[0];  // u(ny): x(ny) = f(ny)
        ldb(DA, UA, c + 3);
        bwd(DB, UB, c + 1);
        ldb(DB, UB, c + 4);
        bwd(DC, UC, c + 2);
        ldb(DC, UC, c + 5);
    }
    // wall rows: unew now holds u(1)
    if (comp == 1) {
        uc[nx] = (V)uy_ym[(size_t)k * nx + i];
        uc[(size_t)(ny + 1) * nx] = (V)((cst.flow_type == 1) ? cst.uybc_yp : 0.0);
    } else if (comp == 3) {
        uc[0] = (V)(cst.sc_r1b * (double)unew + cst.sc_r2b);
        uc[(size_t)(ny + 1) * nx] = (V)(cst.sc_r1t * (double)utop + cst.sc_r2t);
    }
}

template <class V, int HU, class W = double>
__global__ void __launch_bounds__(128, 4) k_helm(DConst cst, const DCoef* __restrict__ coef, int comp0, FieldSet<V> fl,
                                              const double* __restrict__ duy_ym, const double* __restrict__ uy_ym,
                                              const double* __restrict__ facs) {
    helm_body<V, HU, false, W>(OwnGrid{}, cst, coef, comp0, fl, duy_ym, uy_ym, facs);
}

template <class V, int HU, class W = double>
__global__ void __launch_bounds__(128, 4) k_helm_grp(const GrpTab<HelmArgs<V>>* __restrict__ t) {
    SubGrid g;
    const HelmArgs<V>& a = t->e[grp_member(t, g)];
    helm_body<V, HU, true, W>(g, a.c, a.coef, a.comp0, a.fl, a.duy_ym, a.uy_ym, a.fac);
}

// ---------------------------------------------------------------------------
// spectral y-solve of clcPPE_x1 (src/m_Poisson.f90:383-430) on the complex
// coefficients spec[(k*ny + j)*(nx/2+1) + kx].  The real and imaginary parts
// are two real right-hand sides of the same real matrix, so the array is
// treated as 2*(nx/2+1) real columns: lane pairs share kx and a warp reads
// 256 contiguous bytes per row.  The kx = kz = 0 system has its first row
// replaced by phi = 0 (src/m_Poisson.f90:399-404).
// ---------------------------------------------------------------------------
template <int MR>
__global__ void __launch_bounds__(512) k_ysolve(DConst cst, DMetric m, double* __restrict__ specd) {
    extern __shared__ double sm[];
    const int lane = threadIdx.x, w = threadIdx.y, P = blockDim.y;
    const int ny = cst.ny, ncol = 2 * (cst.nx / 2 + 1);
    const int cr = blockIdx.x * 32 + lane;
    const int kx = cr >> 1;
    const int k = blockIdx.y;
    const bool act = cr < ncol;
    const int s = w * MR + 1;
    const double lam = act ? __ldg(&m.wnx[kx]) + __ldg(&m.wnz[k]) : 0.0;
    const bool dc = (kx == 0 && k == 0);
    double* col = specd + (size_t)k * ny * ncol + (act ? cr : 0);
    double a[MR], c[MR], f[MR][1];
#pragma unroll
    for (int r = 0; r < MR; r++) {
        a[r] = 0.0; c[r] = 0.0; f[r][0] = 0.0;
        const int jc = s + r;
        if (jc <= ny && !(dc && jc == 1)) {
            a[r] = (jc == 1) ? 0.0 : __ldg(&m.am2ph[jc]);
            c[r] = (jc == ny) ? 0.0 : __ldg(&m.ap2ph[jc]);
            if (act) f[r][0] = col[(size_t)(jc - 1) * ncol];
        }
    }
    part_eliminate<MR, 1>(a, c, f, PoisDiag{m.ac2ph, lam, s, ny, dc});
    double xf[1], xl[1];
    part_reduced<MR, 1>(P, w, lane, a, c, f, sm, xf, xl);
    if (!act) return;
#pragma unroll
    for (int r = 0; r < MR; r++) {
        const int jc = s + r;
        if (jc <= ny) {
            double x;
            if (r == 0) x = xf[0];
            else if (r == MR - 1) x = xl[0];
            else x = f[r][0] - a[r] * xf[0] - c[r] * xl[0];
            col[(size_t)(jc - 1) * ncol] = x;
        }
    }
}

// ---------------------------------------------------------------------------
// Spectral y-solve with the factors computed once.  The Poisson matrices
// (am2ph, ac2ph + lambda_x(kx) + lambda_z(kz), ap2ph) depend on the mesh and
// the wavenumbers only, so the pivots of InverseTridiagonal
// (src/m_Tools.f90:224-251) are computed once per context: for complex
// column q = kz*(nx/2+1) + kx and Fortran row jc, rv[(jc-1)*NQ + q] =
// 1/vecm(jc) and ar[(jc-1)*NQ + q] = arr(jc) (two arrays, so that each sweep
// reads only the one it needs) with vecm(1) = b(1), arr(jc) = c(jc-1)/vecm(jc-1),
// vecm(jc) = b(jc) - a(jc)*arr(jc), evaluated in the reference's order
// without contraction.  A solve is then the two sweeps
//   f(1) = f(1)/vecm(1),  f(jc) = (f(jc) - a(jc) f(jc-1)) / vecm(jc),
//   f(jc) = f(jc) - arr(jc+1) f(jc+1),
// with no division left on the dependent chain (1/vecm is a multiply).
// The kx = kz = 0 system has row 1 replaced by phi = 0 (b = 1, c = 0,
// f = 0; src/m_Poisson.f90:399-404).
// ---------------------------------------------------------------------------
// dc_here: column 0 is the kx = kz = 0 system (false for a z-slab rank
// whose modes start above kx = 0; m.wnx then starts at its first mode)
__device__ __forceinline__ void pois_factors_body(int ny, int M1, int nz, const DMetric& m, double* __restrict__ rv,
                                                  double* __restrict__ ar, bool dc_here) {
    const int NQ = M1 * nz;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= NQ) return;
    const int kz = q / M1, kx = q - kz * M1;
    const double wx = m.wnx[kx], wz = m.wnz[kz];
    const bool dc = dc_here && (q == 0);
    double vecm = dc ? 1.0 : __dadd_rn(__dadd_rn(m.ac2ph[1], wx), wz);
    rv[q] = 1.0 / vecm;
    ar[q] = 0.0;
    for (int jc = 2; jc <= ny; jc++) {
        const double cp = (dc && jc == 2) ? 0.0 : m.ap2ph[jc - 1];
        const double arr = cp / vecm;
        const double b = __dadd_rn(__dadd_rn(m.ac2ph[jc], wx), wz);
        vecm = __dsub_rn(b, __dmul_rn(m.am2ph[jc], arr));
        rv[(size_t)(jc - 1) * NQ + q] = 1.0 / vecm;
        ar[(size_t)(jc - 1) * NQ + q] = arr;
    }
}
__global__ void k_pois_factors(int ny, int M1, int nz, DMetric m, double* __restrict__ rv, double* __restrict__ ar) {
    pois_factors_body(ny, M1, nz, m, rv, ar, true);
}
__global__ void k_pois_factors_slab(int ny, int M1, int nz, DMetric m, double* __restrict__ rv, double* __restrict__ ar,
                                    int dc_here) {
    pois_factors_body(ny, M1, nz, m, rv, ar, dc_here != 0);
}

namespace {
__device__ __forceinline__ void cpa16t(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpa8t(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
constexpr int YS_U = 8;  // rows loaded ahead of the dependent chain
}  // namespace

// Small grids (one wave): a one-warp CTA stages 16 complex columns of the
// spectrum and their factors in shared memory with cp.async, then lane l
// sweeps the real (l even) or imaginary (l odd) part of column l/2.  S: the
// spectrum's storage (double2, or float2 in the FP32 storage form; the
// sweeps run in double either way).
template <class S, class G>
__device__ __forceinline__ void ys_staged_body(const G& grid, int ny, int M1, int nz, const double* __restrict__ am2ph,
                                               S* __restrict__ spec, const double* __restrict__ fac,
                                               bool dc_here = true) {
    using R = decltype(S::x);
    extern __shared__ double2 sy[];
    const int lane = threadIdx.x;
    const int NQ = M1 * nz;
    const int q0 = grid.x() * 16;
    const int nv = min(16, NQ - q0);
    S* sd = reinterpret_cast<S*>(sy);                          // [ny][16] spectrum
    double* srv = reinterpret_cast<double*>(sy + ny * 16);     // [ny][16] 1/vecm
    double* sar = srv + ny * 16;                               // [ny][16] arr
    double* sa = sar + ny * 16;                                // am2ph[0..ny]
    pdl_wait();
    pdl_trigger();
    // one 16-byte copy per lane and row: lanes 0-15 the spectrum of column
    // q0+lane, lanes 16-23 two 1/vecm of columns q0+2(lane-16)+{0,1}, lanes
    // 24-31 two arr (NQ is even, so the pairs are aligned and never split)
    const int cq = lane & 15, half = lane >> 4;
    const bool cval = cq < nv;
    const int qq = q0 + (cval ? cq : 0);
    const int kz = qq / M1, kx = qq - kz * M1;
    S* scol = spec + (size_t)kz * ny * M1 + kx;
    const char* gsrc;
    char* sdst;
    size_t gstride;
    int sstride;
    bool cvalid;
    if (lane < 16) {
        gsrc = reinterpret_cast<const char*>(scol);
        gstride = (size_t)M1 * sizeof(S);
        sdst = reinterpret_cast<char*>(sd + lane);
        sstride = 16 * sizeof(S);
        cvalid = cval;
    } else {
        const int pr = (lane & 7) * 2;
        const double* base = fac + (lane < 24 ? (size_t)0 : (size_t)NQ * ny) + q0 + pr;
        gsrc = reinterpret_cast<const char*>(base);
        gstride = (size_t)NQ * sizeof(double);
        sdst = reinterpret_cast<char*>((lane < 24 ? srv : sar) + pr);
        sstride = 16 * sizeof(double);
        cvalid = pr < nv;
    }
    if (cvalid) {
        if (lane < 16 && sizeof(S) == 8)
            for (int j = 0; j < ny; j++) cpa8t(sdst + (size_t)j * sstride, gsrc + (size_t)j * gstride);
        else
            for (int j = 0; j < ny; j++) cpa16t(sdst + (size_t)j * sstride, gsrc + (size_t)j * gstride);
    }
    for (int j = lane; j <= ny; j += 32) sa[j] = __ldg(&am2ph[j]);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    R* sdd = reinterpret_cast<R*>(sd);
    const int cp = lane >> 1;  // complex column of this lane's real or imaginary part
    const bool dc = dc_here && (q0 + cp) == 0;
    double fp = 0.0;
    for (int j0 = 0; j0 < ny; j0 += YS_U) {
        double d[YS_U], rv[YS_U], a[YS_U];
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 + u;
            if (j < ny) {
                d[u] = (double)sdd[j * 32 + lane];
                rv[u] = srv[j * 16 + cp];
                a[u] = sa[j + 1];
            }
        }
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 + u;
            if (j < ny) {
                const double f = (j == 0) ? (dc ? 0.0 : d[u]) * rv[u] : (d[u] - a[u] * fp) * rv[u];
                sdd[j * 32 + lane] = (R)f;
                fp = f;
            }
        }
    }
    double xn = fp;
    for (int j0 = ny - 2; j0 >= 0; j0 -= YS_U) {
        double d[YS_U], ar[YS_U];
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 - u;
            if (j >= 0) {
                d[u] = (double)sdd[j * 32 + lane];
                ar[u] = sar[(j + 1) * 16 + cp];
            }
        }
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 - u;
            if (j >= 0) {
                const double x = d[u] - ar[u] * xn;
                sdd[j * 32 + lane] = (R)x;
                xn = x;
            }
        }
    }
    __syncthreads();
    if (cval)
        for (int j = half; j < ny; j += 2) scol[(size_t)j * M1] = sd[j * 16 + cq];
}

template <class S>
__global__ void __launch_bounds__(32) k_ys_staged(int ny, int M1, int nz, const double* __restrict__ am2ph,
                                                  S* __restrict__ spec, const double* __restrict__ fac) {
    ys_staged_body(OwnGrid{}, ny, M1, nz, am2ph, spec, fac);
}

// Large grids: one thread per real column straight from global memory, the
// rows of a chunk loaded ahead of its chain, latency hidden by occupancy.
// R: storage of the spectrum's real parts (double, or float in the FP32
// storage form); the sweeps run in double either way
template <class R, class G>
__device__ __forceinline__ void ys_global_body(const G& grid, int ny, int M1, int nz, const double* __restrict__ am2ph,
                                               R* __restrict__ specd, const double* __restrict__ fac,
                                               bool dc_here = true) {
    const int W = 2 * M1, NQ = M1 * nz;
    const int g = grid.x() * blockDim.x + threadIdx.x;
    pdl_wait();
    pdl_trigger();
    if (g >= W * nz) return;
    const int kz = g / W, cr = g - kz * W, q = g >> 1;
    R* col = specd + (size_t)kz * ny * W + cr;
    const double* frv = fac + q;
    const double* far = fac + (size_t)NQ * ny + q;
    const bool dc = dc_here && (q == 0);
    double fp = 0.0;
    for (int j0 = 0; j0 < ny; j0 += YS_U) {
        R d[YS_U];  // in the storage type: widened at use, so the loads stay in flight
        double rv[YS_U], a[YS_U];
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 + u;
            if (j < ny) {
                d[u] = col[(size_t)j * W];
                rv[u] = __ldg(&frv[(size_t)j * NQ]);
                a[u] = __ldg(&am2ph[j + 1]);
            }
        }
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 + u;
            if (j < ny) {
                const double du = (double)d[u];
                const double f = (j == 0) ? (dc ? 0.0 : du) * rv[u] : (du - a[u] * fp) * rv[u];
                col[(size_t)j * W] = (R)f;
                fp = f;  // the chain stays FP64 (no conversion on the dependent path)
            }
        }
    }
    double xn = fp;
    for (int j0 = ny - 2; j0 >= 0; j0 -= YS_U) {
        R d[YS_U];
        double ar[YS_U];
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 - u;
            if (j >= 0) {
                d[u] = col[(size_t)j * W];
                ar[u] = __ldg(&far[(size_t)(j + 1) * NQ]);
            }
        }
#pragma unroll
        for (int u = 0; u < YS_U; u++) {
            const int j = j0 - u;
            if (j >= 0) {
                const double x = (double)d[u] - ar[u] * xn;
                col[(size_t)j * W] = (R)x;
                xn = x;
            }
        }
    }
}

template <class R>
__global__ void __launch_bounds__(128) k_ys_global(int ny, int M1, int nz, const double* __restrict__ am2ph,
                                                   R* __restrict__ specd, const double* __restrict__ fac) {
    ys_global_body(OwnGrid{}, ny, M1, nz, am2ph, specd, fac);
}

// grouped: kind 0 staged (S the spectrum), 1 streaming (its real parts)
template <class S>
__global__ void __launch_bounds__(32) k_ys_staged_grp(const GrpTab<YsArgs<S>>* __restrict__ t) {
    SubGrid g;
    const YsArgs<S>& a = t->e[grp_member(t, g)];
    ys_staged_body(g, a.ny, a.M1, a.nz, a.am2ph, a.spec, a.fac);
}
template <class S>
__global__ void __launch_bounds__(128) k_ys_global_grp(const GrpTab<YsArgs<S>>* __restrict__ t) {
    using R = decltype(S::x);
    SubGrid g;
    const YsArgs<S>& a = t->e[grp_member(t, g)];
    ys_global_body(g, a.ny, a.M1, a.nz, a.am2ph, reinterpret_cast<R*>(a.spec), a.fac);
}

void launch_pois_factors(cudaStream_t st, const DConst& c, const DMetric& m, double* fac) {
    const int M1 = c.nx / 2 + 1, NQ = M1 * c.nz;
    k_pois_factors<<<(NQ + 127) / 128, 128, 0, st>>>(c.ny, M1, c.nz, m, fac, fac + (size_t)NQ * c.ny);
}

// the same kernels for a z-slab rank's x-mode slab, whose column 0 is the
// kx = kz = 0 system only on the rank holding kx = 0
__global__ void __launch_bounds__(32) k_ys_staged_slab(int ny, int M1, int nz, const double* __restrict__ am2ph,
                                                       double2* __restrict__ spec, const double* __restrict__ fac,
                                                       int dc_here) {
    ys_staged_body(OwnGrid{}, ny, M1, nz, am2ph, spec, fac, dc_here != 0);
}
__global__ void __launch_bounds__(128) k_ys_global_slab(int ny, int M1, int nz, const double* __restrict__ am2ph,
                                                        double* __restrict__ specd, const double* __restrict__ fac,
                                                        int dc_here) {
    ys_global_body(OwnGrid{}, ny, M1, nz, am2ph, specd, fac, dc_here != 0);
}
void launch_pois_factors_slab(cudaStream_t st, const DConst& c, const DMetric& m, double* fac, int dc_here) {
    const int M1 = c.nx / 2 + 1, NQ = M1 * c.nz;
    k_pois_factors_slab<<<(NQ + 127) / 128, 128, 0, st>>>(c.ny, M1, c.nz, m, fac, fac + (size_t)NQ * c.ny, dc_here);
}

// the staged kernel's shared memory: the spectrum block (16 B per complex
// value, whatever the storage, so that the factor arrays stay 16-byte
// aligned), the two factor blocks and am2ph
static size_t ys_staged_smem(int ny) { return (size_t)ny * 16 * 2 * sizeof(double2) + (size_t)(ny + 1) * sizeof(double); }

// 0: the staged kernel (the grid fits one wave of it, or solver_sel = 1),
// 1: the streaming one
int ys_kind(const DConst& c) {
    const int M1 = c.nx / 2 + 1, NQ = M1 * c.nz;
    const size_t sm = ys_staged_smem(c.ny);
    const int per_sm = sm > 0 ? (int)((220 * 1024) / sm) : 0;
    const int ctas = (NQ + 15) / 16;
    return (per_sm >= 1 && (c.solver_sel == 1 || (c.solver_sel == 0 && ctas <= per_sm * c.nsm))) ? 0 : 1;
}
dim3 ys_member_grid(const DConst& c, int kind) {
    const int M1 = c.nx / 2 + 1, NQ = M1 * c.nz;
    return kind == 0 ? dim3((NQ + 15) / 16) : dim3((2 * M1 * c.nz + 127) / 128);
}
size_t ys_smem(const DConst& c, int kind) { return kind == 0 ? ys_staged_smem(c.ny) : 0; }

template <class S>
static void ysolve_fac_t(cudaStream_t st, const DConst& c, const DMetric& m, S* spec, const double* fac) {
    using R = decltype(S::x);
    const int M1 = c.nx / 2 + 1;
    const int kind = ys_kind(c);
    if (kind == 0) {
        launch_pdl(k_ys_staged<S>, ys_member_grid(c, 0), dim3(32), ys_smem(c, 0), st, c.ny, M1, c.nz, m.am2ph, spec,
                   fac);
    } else {
        launch_pdl(k_ys_global<R>, ys_member_grid(c, 1), dim3(128), 0, st, c.ny, M1, c.nz, m.am2ph,
                   reinterpret_cast<R*>(spec), fac);
    }
}

template <class S>
static void ys_grp_t(cudaStream_t st, int kind, const GrpTab<YsArgs<S>>* t, int nblk, size_t smem) {
    if (kind == 0) launch_pdl(k_ys_staged_grp<S>, dim3((unsigned)nblk), dim3(32), smem, st, t);
    else launch_pdl(k_ys_global_grp<S>, dim3((unsigned)nblk), dim3(128), 0, st, t);
}
void launch_ys_grp(cudaStream_t st, int kind, const GrpTab<YsArgs<double2>>* t, int nblk, size_t smem) {
    ys_grp_t(st, kind, t, nblk, smem);
}
void launch_ys_grp(cudaStream_t st, int kind, const GrpTab<YsArgs<float2>>* t, int nblk, size_t smem) {
    ys_grp_t(st, kind, t, nblk, smem);
}
void launch_ysolve_fac(cudaStream_t st, const DConst& c, const DMetric& m, double2* spec, const double* fac) {
    ysolve_fac_t(st, c, m, spec, fac);
}
void launch_ysolve_fac_slab(cudaStream_t st, const DConst& c, const DMetric& m, double2* spec, const double* fac,
                            int dc_here) {
    const int M1 = c.nx / 2 + 1;
    if (ys_kind(c) == 0)
        launch_pdl(k_ys_staged_slab, ys_member_grid(c, 0), dim3(32), ys_smem(c, 0), st, c.ny, M1, c.nz, m.am2ph, spec,
                   fac, dc_here);
    else
        launch_pdl(k_ys_global_slab, ys_member_grid(c, 1), dim3(128), 0, st, c.ny, M1, c.nz, m.am2ph,
                   reinterpret_cast<double*>(spec), fac, dc_here);
}
void launch_ysolve_fac(cudaStream_t st, const DConst& c, const DMetric& m, float2* spec, const double* fac) {
    ysolve_fac_t(st, c, m, spec, fac);
}

// ---------------------------------------------------------------------------
// launchers: partition length MR in {8, 12, 16}, P = ceil(ny/MR) <= 16 warps
// ---------------------------------------------------------------------------
__host__ __device__ inline int part_len_dev(int ny) { return ny <= 64 ? 8 : (ny <= 192 ? 12 : 16); }
__host__ __device__ inline int tridiag_partitions_dev(int ny) {
    const int mr = part_len_dev(ny);
    return (ny + mr - 1) / mr;
}
static int part_len(int ny) { return part_len_dev(ny); }

int tridiag_partitions(int ny) { return tridiag_partitions_dev(ny); }

bool tridiag_supported(int ny) { return ny >= 3 && ny <= 256; }

static size_t red_smem(int P, int nc) { return (size_t)2 * P * 32 * (3 + nc) * sizeof(double); }

__global__ void k_helm_factors(DConst cst, DMetric m, const DCoef* __restrict__ coef, int ns0, int nsub, double a1,
                               double a2, double a3, double* __restrict__ facs);

void tridiag_init() {
    cudaFuncSetAttribute(k_ysolve<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_ysolve<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_ysolve<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_ys_staged<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(k_ys_staged<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(k_ys_staged_grp<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(k_ys_staged_grp<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(k_ys_staged_slab, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(k_helm_factors, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
}

int tridiag_part_len(int ny) { return part_len(ny); }

size_t helm_fac_doubles(int ny) { return (size_t)9 * helm_stride(ny); }
int helm_variants() { return HELM_NVAR; }
// the Helmholtz launch shapes of precision form prec: FP32 storage adds
// float-arithmetic sweeps (helm_var 2)
int helm_variants(int prec) { return prec == 2 ? HELM_NVAR + 1 : HELM_NVAR; }

// pivots of the Helmholtz matrices of substeps ns0..ns0+nsub-1 for the
// current dt (coef->dt): one thread per (substep, type) runs the forward
// elimination of InverseTridiagonal on the coefficients of clcU1Hat /
// clcU2Hat / clcScalar (src/m_TScheme.f90:374-380,409-420,486-492)
__global__ void __launch_bounds__(32) k_helm_factors(DConst cst, DMetric m, const DCoef* __restrict__ coef, int ns0,
                                                     int nsub, double a1, double a2, double a3,
                                                     double* __restrict__ facs) {
    extern __shared__ double shm[];  // ap, ac, am of the three types, rows 0..ny+1
    const int ny = cst.ny, L = ny + 2;
    const double* srcs[9] = {m.ap2cCN, m.ac2cCN, m.am2cCN, m.ap2p, m.ac2p, m.am2p, m.ap2cScCN, m.ac2cScCN, m.am2cScCN};
    for (int a = 0; a < 9; a++)
        for (int j = threadIdx.x; j < L; j += blockDim.x) shm[a * L + j] = srcs[a][j];
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    const int q = threadIdx.x;
    if (q >= 3 * nsub) return;
    const int ns = ns0 + q / 3, t = q % 3;
    const double alp = ns == 1 ? a1 : (ns == 2 ? a2 : a3);
    const double dt = coef->dt;
    const double beta = (t == 2) ? 0.5 * alp * cst.sdiff * dt : 0.5 * alp * cst.xnu * dt;
    const double* ap = shm + (3 * t) * L;
    const double* ac = ap + L;
    const double* am = ac + L;
    double* F = facs + (size_t)((ns - 1) * 3 + t) * helm_stride(ny);
    double* FA = F;
    double* FR = F + (ny + 2);
    double* FW = F + 2 * (ny + 2);
    const bool vrow1 = (t == 1);  // clcU2Hat: row 1 is the identity
    double vecm = vrow1 ? 1.0 : __dadd_rn(-__dmul_rn(beta, ac[1]), 1.0);
    double cprev = vrow1 ? 0.0 : -__dmul_rn(beta, ap[1]);
    FA[0] = FR[0] = FW[0] = 0.0;
    FA[1] = 0.0;
    FR[1] = 1.0 / vecm;
    FW[1] = 0.0;
    for (int jc = 2; jc <= ny; jc++) {
        const double arr = cprev / vecm;
        const double a = -__dmul_rn(beta, am[jc]);
        const double b = __dadd_rn(-__dmul_rn(beta, ac[jc]), 1.0);
        vecm = __dsub_rn(b, __dmul_rn(a, arr));
        FA[jc] = a;
        FR[jc] = 1.0 / vecm;
        FW[jc] = arr;
        cprev = -__dmul_rn(beta, ap[jc]);
    }
    FA[ny + 1] = FR[ny + 1] = FW[ny + 1] = 0.0;
}

void launch_helm_factors(cudaStream_t st, const DConst& c, const DMetric& m, const DCoef* coef, int ns0, int nsub,
                         const double* alp, double* fac) {
    launch_pdl(k_helm_factors, dim3(1), dim3(32), (size_t)9 * (c.ny + 2) * sizeof(double), st, c, m, coef, ns0, nsub,
               alp[0], alp[1], alp[2], fac);
}

static dim3 helm_grid(const DConst& c, int ncomp) { return dim3((c.nx + 127) / 128, c.nz, ncomp); }
// the grouped launch's shape (32 columns x 4 z planes per CTA)
dim3 helm_member_grid(const DConst& c, int ncomp) { return dim3((c.nx + 31) / 32, (c.nz + 3) / 4, ncomp); }
size_t helm_smem(const DConst& c) { return helm_stride(c.ny) * sizeof(double); }

template <class V>
static void helm_grp_t(cudaStream_t st, const DConst& key, const GrpTab<HelmArgs<V>>* t, int nblk, size_t smem) {
    constexpr int H0 = sizeof(V) == 4 ? 2 * HY_U : HY_U;
    using WF = std::conditional_t<sizeof(V) == 4, float, double>;  // helm_var 2: float sweeps (FP32 storage)
    if (key.helm_var == 1) launch_pdl(k_helm_grp<V, H0 / 2>, dim3((unsigned)nblk), dim3(32, 4), smem, st, t);
    else if (key.helm_var == 2) launch_pdl(k_helm_grp<V, H0, WF>, dim3((unsigned)nblk), dim3(32, 4), smem, st, t);
    else launch_pdl(k_helm_grp<V, H0>, dim3((unsigned)nblk), dim3(32, 4), smem, st, t);
}
void launch_helm_grp(cudaStream_t st, const DConst& key, const GrpTab<HelmArgs<double>>* t, int nblk, size_t smem) {
    helm_grp_t(st, key, t, nblk, smem);
}
void launch_helm_grp(cudaStream_t st, const DConst& key, const GrpTab<HelmArgs<float>>* t, int nblk, size_t smem) {
    helm_grp_t(st, key, t, nblk, smem);
}

template <class V>
static void helm_dispatch(cudaStream_t st, const DConst& c, const DCoef* coef, int comp0, int ncomp,
                          const FieldSet<V>& f, const double* duy_ym, const double* uy_ym, const double* fac) {
    dim3 blk(32, 4);
    dim3 grd = helm_grid(c, ncomp);
    // rows per chunk: FP64 8 (variant 1: 4); float storage, whose ring takes
    // half the registers, 16 (variant 1: 8)
    constexpr int H0 = sizeof(V) == 4 ? 2 * HY_U : HY_U;
    using WF = std::conditional_t<sizeof(V) == 4, float, double>;  // helm_var 2: float sweeps (FP32 storage)
    if (c.helm_var == 1)
        launch_pdl(k_helm<V, H0 / 2>, grd, blk, helm_stride(c.ny) * sizeof(double), st, c, coef, comp0, f, duy_ym,
                   uy_ym, fac);
    else if (c.helm_var == 2)
        launch_pdl(k_helm<V, H0, WF>, grd, blk, helm_stride(c.ny) * sizeof(double), st, c, coef, comp0, f, duy_ym,
                   uy_ym, fac);
    else
        launch_pdl(k_helm<V, H0>, grd, blk, helm_stride(c.ny) * sizeof(double), st, c, coef, comp0, f, duy_ym,
                   uy_ym, fac);
}

void launch_helm(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields& f, const double* duy_ym,
                 const double* uy_ym, const double* fac) {
    helm_dispatch(st, c, coef, 0, 3, f, duy_ym, uy_ym, fac);
}
void launch_helm(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields32& f, const double* duy_ym,
                 const double* uy_ym, const double* fac) {
    helm_dispatch(st, c, coef, 0, 3, f, duy_ym, uy_ym, fac);
}

void launch_helm_scalar(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields& f, const double* fac) {
    helm_dispatch(st, c, coef, 3, 1, f, nullptr, nullptr, fac);
}
void launch_helm_scalar(cudaStream_t st, const DConst& c, const DCoef* coef, const Fields32& f, const double* fac) {
    helm_dispatch(st, c, coef, 3, 1, f, nullptr, nullptr, fac);
}

void launch_ysolve(cudaStream_t st, const DConst& c, const DMetric& m, double2* spec) {
    const int mr = part_len(c.ny), P = tridiag_partitions(c.ny);
    dim3 blk(32, P);
    dim3 grd((2 * (c.nx / 2 + 1) + 31) / 32, c.nz);
    const size_t sm = red_smem(P, 1);
    double* sd = reinterpret_cast<double*>(spec);
    if (mr == 8) k_ysolve<8><<<grd, blk, sm, st>>>(c, m, sd);
    else if (mr == 12) k_ysolve<12><<<grd, blk, sm, st>>>(c, m, sd);
    else k_ysolve<16><<<grd, blk, sm, st>>>(c, m, sd);
}

}  // namespace ptc
