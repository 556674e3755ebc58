// helm_factor.cuh -- factors of the implicit wall-normal Helmholtz systems.
//
// The matrices (I - beta*Lyy) of clcU1Hat/clcU3Hat (a?2cForCN), clcU2Hat
// (a?2p, row 1 the identity) and clcScalar (a?2cScCN) depend only on the row
// (src/m_TScheme.f90:374-380,409-420,451-457,486-492), not on the column.  So
// the partitioned elimination (see k_tridiag.cu) is factored once per
// substep: per partition the multipliers of the modified Thomas sweep, and the
// Thomas factors of the 2P-row reduced system.  Applying them to a column is
// then a fixed sequence of multiply-adds.
#pragma once
#include "common.cuh"

namespace ptc {

struct HelmFacLayout {
    int MR, P, NG;
    int F0, A0, CB, AF, CF, R0, C0, RA, IV, W, RI, stride;
};

__host__ __device__ inline HelmFacLayout helm_fac_layout(int MR, int P) {
    HelmFacLayout L;
    L.MR = MR;
    L.P = P;
    L.NG = MR * P;
    L.F0 = 0;              // 1/b (rows 0,1) or the forward pivot reciprocal
    L.A0 = L.NG;           // original sub-diagonal a
    L.CB = 2 * L.NG;       // super-diagonal used by the backward sweep
    L.AF = 3 * L.NG;       // final coefficient of x_first
    L.CF = 4 * L.NG;       // final coefficient of x_last
    L.R0 = 5 * L.NG;       // row-0 pivot reciprocal, per partition
    L.C0 = L.R0 + P;       // row-0 c after normalisation
    L.RA = L.C0 + P;       // reduced sub-diagonal
    L.IV = L.RA + 2 * P;   // reduced pivot reciprocals
    L.W = L.IV + 2 * P;    // reduced multipliers
    L.RI = L.W + 2 * P;    // dense inverse of the reduced matrix, row major [2P][2P]
    L.stride = L.RI + 4 * P * P;
    return L;
}

// coefficients of Fortran row jc of matrix type t (0: u/w, 1: v, 2: scalar);
// rows past ny are identity rows; aj(1) and cj(nyc) are never read by
// InverseTridiagonal and are zero here
__device__ inline void helm_row(const DMetric& m, int t, double beta, int ny, int jc, double& a, double& b, double& c) {
    if (jc > ny || (t == 1 && jc == 1)) { a = 0.0; b = 1.0; c = 0.0; return; }
    const double *ap, *ac, *am;
    if (t == 0) { ap = m.ap2cCN; ac = m.ac2cCN; am = m.am2cCN; }
    else if (t == 1) { ap = m.ap2p; ac = m.ac2p; am = m.am2p; }
    else { ap = m.ap2cScCN; ac = m.ac2cScCN; am = m.am2cScCN; }
    a = (jc == 1) ? 0.0 : -(beta * am[jc]);
    b = -(beta * ac[jc]) + 1.0;
    c = (jc == ny) ? 0.0 : -(beta * ap[jc]);
}

// factors of partition w (rows w*MR .. w*MR+MR-1), the modified Thomas sweep
// of src/m_Poisson.f90:496-537 with the multipliers recorded
__device__ inline void helm_factor_partition(const DMetric& m, int t, double beta, int ny, const HelmFacLayout& L, int w,
                                             double* fac) {
    double a[16], c[16];
    const int MR = L.MR, g0 = w * MR;
    for (int r = 0; r < MR; r++) {
        double b;
        helm_row(m, t, beta, ny, g0 + r + 1, a[r], b, c[r]);
        fac[L.A0 + g0 + r] = a[r];
        if (r < 2) {
            fac[L.F0 + g0 + r] = 1.0 / b;
            a[r] = a[r] / b;
            c[r] = c[r] / b;
        } else {
            const double rr = 1.0 / (b - a[r] * c[r - 1]);
            fac[L.F0 + g0 + r] = rr;
            c[r] = rr * c[r];
            a[r] = -(rr * a[r] * a[r - 1]);
        }
    }
    for (int r = 0; r < MR; r++) fac[L.CB + g0 + r] = 0.0;
    for (int r = MR - 3; r >= 1; r--) {
        fac[L.CB + g0 + r] = c[r];
        a[r] = a[r] - c[r] * a[r + 1];
        c[r] = -(c[r] * c[r + 1]);
    }
    const double rr0 = 1.0 / (1.0 - a[1] * c[0]);
    fac[L.R0 + w] = rr0;
    fac[L.C0 + w] = c[0];
    a[0] = rr0 * a[0];
    c[0] = -(rr0 * c[0] * c[1]);
    for (int r = 0; r < MR; r++) {
        fac[L.AF + g0 + r] = a[r];
        fac[L.CF + g0 + r] = c[r];
    }
}

// Whole-block computation of the factors of `nmat` matrices (one per
// (substep, type) pair): partitions in parallel, then the Thomas factors of
// each reduced system, then the columns of its dense inverse in parallel.
// betas[q] and types[q] describe matrix q; its factors go to fac + q*stride.
// Shared memory: red[nmat][2P][2] + ra/iv/w [nmat][2P] (<= 9*32*5 doubles).
__device__ inline void helm_factor_block(const DMetric& m, int ny, const HelmFacLayout& L, int nmat, const double* betas,
                                         const int* types, double* fac) {
    __shared__ double red[9][32][2];
    __shared__ double sra[9][32], siv[9][32], sw[9][32];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int n2 = 2 * L.P, MR = L.MR;
    for (int q = tid; q < nmat * L.P; q += nthr) {
        const int mat = q / L.P, w = q - mat * L.P;
        double* f = fac + (size_t)mat * L.stride;
        helm_factor_partition(m, types[mat], betas[mat], ny, L, w, f);
        red[mat][2 * w][0] = f[L.AF + w * MR];
        red[mat][2 * w][1] = f[L.CF + w * MR];
        red[mat][2 * w + 1][0] = f[L.AF + w * MR + MR - 1];
        red[mat][2 * w + 1][1] = f[L.CF + w * MR + MR - 1];
    }
    __syncthreads();
    if (tid < nmat) {
        const int mat = tid;
        double* f = fac + (size_t)mat * L.stride;
        double vecm = 1.0;
        sra[mat][0] = red[mat][0][0];
        siv[mat][0] = 1.0;
        sw[mat][0] = 0.0;
        for (int i = 1; i < n2; i++) {
            const double wgt = red[mat][i - 1][1] / vecm;
            const double ai = red[mat][i][0];
            vecm = 1.0 - ai * wgt;
            sra[mat][i] = ai;
            sw[mat][i] = wgt;
            siv[mat][i] = 1.0 / vecm;
        }
        for (int i = 0; i < n2; i++) {
            f[L.RA + i] = sra[mat][i];
            f[L.IV + i] = siv[mat][i];
            f[L.W + i] = sw[mat][i];
        }
    }
    __syncthreads();
    for (int q = tid; q < nmat * n2; q += nthr) {
        const int mat = q / n2, col = q - mat * n2;
        double* f = fac + (size_t)mat * L.stride;
        double v[32];
        double fp = (col == 0) ? 1.0 : 0.0;
        v[0] = fp;
        for (int i = 1; i < n2; i++) {
            fp = ((i == col ? 1.0 : 0.0) - sra[mat][i] * fp) * siv[mat][i];
            v[i] = fp;
        }
        for (int i = n2 - 2; i >= 0; i--) {
            fp = v[i] - sw[mat][i + 1] * fp;
            v[i] = fp;
        }
        for (int i = 0; i < n2; i++) f[L.RI + i * n2 + col] = v[i];
    }
}

}  // namespace ptc
