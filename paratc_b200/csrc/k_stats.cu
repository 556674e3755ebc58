// k_stats.cu -- FP64 statistics accumulation of clcStat
// (src/m_FlowCase.f90:257-428) on B200.
//
// clcStat adds, at every statistics step, the x-z plane averages of 35
// moments (40 with the scalar) per wall-normal row to SumStat(k, jc): means,
// second to fourth moments, pressure-strain and dissipation terms and the
// squared vorticity, from the staggered fields with their 4th-order
// interpolations and derivatives; the top wall row nyp adds three of them.
// Here a CTA sums one slice of the cells of one row (the row's z range cut
// into `splits` pieces), every thread in a fixed cell order, the block in a
// fixed shuffle order, and a second kernel adds the slices of a row in index
// order and then SumVec/(nx nz) to SumStat, so the accumulators are FP64 and
// independent of scheduling.  Periodic neighbours are index wrap (the same
// values as the reference's halos of width 2, 1 for p on the + side).
#include "common.cuh"
#include "kernels.cuh"
#include "reduce.cuh"

namespace ptc {
namespace {

constexpr int STAT_THREADS = 256;

template <int NS>
__global__ void __launch_bounds__(STAT_THREADS)
    k_stats(DConst c, DMetric m, const double* __restrict__ ux, const double* __restrict__ uy,
            const double* __restrict__ uz, const double* __restrict__ pr, const double* __restrict__ sc, int splits,
            double* __restrict__ part) {
    const int nx = c.nx, ny = c.ny, nz = c.nz;
    const int jc = blockIdx.x + 1;  // 1..nyp
    const int s = blockIdx.y;
    const int k0 = (int)((long long)nz * s / splits), k1 = (int)((long long)nz * (s + 1) / splits);
    const size_t pl = (size_t)c.nyt * nx;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double v[NS];
#pragma unroll
    for (int q = 0; q < NS; q++) v[q] = 0.0;
    const double I1 = c.IC[0], I2 = c.IC[1], I3 = c.IC[2], I4 = c.IC[3];
    const double IY1 = m.yinterp[jc], IY2 = 1.0 - IY1;
    const double rdxt = c.rdx / 12.0, rdzt = c.rdz / 12.0;
    if (jc <= ny) {
        const int jm = jc - 1, jp = jc + 1;
        const double cac = m.rdyc[jc], cacU = m.rdyc[jp], caj = m.rdyp[jc];
        const double ap2c = m.ap2c[jc], ac2c = m.ac2c[jc], am2c = m.am2c[jc];
        const double ap2p = m.ap2p[jc], ac2p = m.ac2p[jc], am2p = m.am2p[jc];
        for (int k = k0 + warp; k < k1; k += STAT_THREADS / 32) {
            const size_t kc = (size_t)k * pl;
            const size_t ks = (size_t)(k >= 2 ? k - 2 : k - 2 + nz) * pl, km = (size_t)(k >= 1 ? k - 1 : nz - 1) * pl;
            const size_t kp = (size_t)(k + 1 < nz ? k + 1 : k + 1 - nz) * pl, ku = (size_t)(k + 2 < nz ? k + 2 : k + 2 - nz) * pl;
            const size_t rc = (size_t)jc * nx, rm = (size_t)jm * nx, rp = (size_t)jp * nx;
            for (int i = lane; i < nx; i += 32) {
                const int is = i >= 2 ? i - 2 : i - 2 + nx, im = i >= 1 ? i - 1 : nx - 1;
                const int ip = i + 1 < nx ? i + 1 : i + 1 - nx, iu = i + 2 < nx ? i + 2 : i + 2 - nx;
#define U(a, kk, rr, ii) __ldg(&(a)[(kk) + (rr) + (ii)])
                const double uxloc = U(ux, kc, rc, i) + c.ucrf;
                const double uyloc = U(uy, kc, rc, i);
                const double uzloc = U(uz, kc, rc, i);
                const double prloc = U(pr, kc, rc, i);
                const double uxCell = I1 * U(ux, kc, rc, im) + I2 * U(ux, kc, rc, i) + I3 * U(ux, kc, rc, ip) + I4 * U(ux, kc, rc, iu) + c.ucrf;
                const double uyCell = (uyloc + U(uy, kc, rp, i)) * 0.5;
                const double uy_xc = I1 * U(uy, kc, rc, is) + I2 * U(uy, kc, rc, im) + I3 * U(uy, kc, rc, i) + I4 * U(uy, kc, rc, ip);
                const double uy_xp = I1 * U(uy, kc, rp, is) + I2 * U(uy, kc, rp, im) + I3 * U(uy, kc, rp, i) + I4 * U(uy, kc, rp, ip);
                const double uzCell = I1 * U(uz, km, rc, i) + I2 * U(uz, kc, rc, i) + I3 * U(uz, kp, rc, i) + I4 * U(uz, ku, rc, i);
                const double prloc2 = IY1 * (I1 * U(pr, kc, rm, is) + I2 * U(pr, kc, rm, im) + I3 * U(pr, kc, rm, i) + I4 * U(pr, kc, rm, ip)) +
                                      IY2 * (I1 * U(pr, kc, rc, is) + I2 * U(pr, kc, rc, im) + I3 * U(pr, kc, rc, i) + I4 * U(pr, kc, rc, ip));
                const double dudx = c.dxC[0] * U(ux, kc, rc, im) + c.dxC[1] * U(ux, kc, rc, i) + c.dxC[2] * U(ux, kc, rc, ip) + c.dxC[3] * U(ux, kc, rc, iu);
                const double dudy = (U(ux, kc, rc, i) - U(ux, kc, rm, i)) * cac;
                const double dudz = c.dzC[0] * U(ux, ks, rc, i) + c.dzC[1] * U(ux, km, rc, i) + c.dzC[2] * U(ux, kc, rc, i) + c.dzC[3] * U(ux, kp, rc, i);
                const double dvdx = c.dxC[0] * U(uy, kc, rc, is) + c.dxC[1] * U(uy, kc, rc, im) + c.dxC[2] * U(uy, kc, rc, i) + c.dxC[3] * U(uy, kc, rc, ip);
                const double dvdy = (U(uy, kc, rp, i) - uyloc) * caj;
                const double dvdz = c.dzC[0] * U(uy, ks, rc, i) + c.dzC[1] * U(uy, km, rc, i) + c.dzC[2] * U(uy, kc, rc, i) + c.dzC[3] * U(uy, kp, rc, i);
                const double dwdx = c.dxC[0] * U(uz, kc, rc, is) + c.dxC[1] * U(uz, kc, rc, im) + c.dxC[2] * U(uz, kc, rc, i) + c.dxC[3] * U(uz, kc, rc, ip);
                const double dwdy = (uzloc - U(uz, kc, rm, i)) * cac;
                const double dwdz = c.dzC[0] * U(uz, km, rc, i) + c.dzC[1] * U(uz, kc, rc, i) + c.dzC[2] * U(uz, kp, rc, i) + c.dzC[3] * U(uz, ku, rc, i);
                const double dudxx = c.dxxC[0] * U(ux, kc, rc, is) + c.dxxC[1] * U(ux, kc, rc, im) + c.dxxC[2] * U(ux, kc, rc, i) + c.dxxC[3] * U(ux, kc, rc, ip) + c.dxxC[4] * U(ux, kc, rc, iu);
                const double dudyy = ap2c * U(ux, kc, rp, i) + ac2c * U(ux, kc, rc, i) + am2c * U(ux, kc, rm, i);
                const double dudzz = c.dzzC[0] * U(ux, ks, rc, i) + c.dzzC[1] * U(ux, km, rc, i) + c.dzzC[2] * U(ux, kc, rc, i) + c.dzzC[3] * U(ux, kp, rc, i) + c.dzzC[4] * U(ux, ku, rc, i);
                const double dvdxx = c.dxxC[0] * U(uy, kc, rc, is) + c.dxxC[1] * U(uy, kc, rc, im) + c.dxxC[2] * U(uy, kc, rc, i) + c.dxxC[3] * U(uy, kc, rc, ip) + c.dxxC[4] * U(uy, kc, rc, iu);
                const double dvdyy = ap2p * U(uy, kc, rp, i) + ac2p * U(uy, kc, rc, i) + am2p * U(uy, kc, rm, i);
                const double dvdzz = c.dzzC[0] * U(uy, ks, rc, i) + c.dzzC[1] * U(uy, km, rc, i) + c.dzzC[2] * U(uy, kc, rc, i) + c.dzzC[3] * U(uy, kp, rc, i) + c.dzzC[4] * U(uy, ku, rc, i);
                const double dwdxx = c.dxxC[0] * U(uz, kc, rc, is) + c.dxxC[1] * U(uz, kc, rc, im) + c.dxxC[2] * U(uz, kc, rc, i) + c.dxxC[3] * U(uz, kc, rc, ip) + c.dxxC[4] * U(uz, kc, rc, iu);
                const double dwdyy = ap2c * U(uz, kc, rp, i) + ac2c * U(uz, kc, rc, i) + am2c * U(uz, kc, rm, i);
                const double dwdzz = c.dzzC[0] * U(uz, ks, rc, i) + c.dzzC[1] * U(uz, km, rc, i) + c.dzzC[2] * U(uz, kc, rc, i) + c.dzzC[3] * U(uz, kp, rc, i) + c.dzzC[4] * U(uz, ku, rc, i);
                const double vor_x = dwdy - dvdz, vor_y = dudz - dwdx, vor_z = dvdx - dudy;
                const double dudxC = (-U(ux, kc, rc, iu) + 8.0 * U(ux, kc, rc, ip) - 8.0 * U(ux, kc, rc, im) + U(ux, kc, rc, is)) * rdxt;
                const double dvdxU = c.dxC[0] * U(uy, kc, rp, is) + c.dxC[1] * U(uy, kc, rp, im) + c.dxC[2] * U(uy, kc, rp, i) + c.dxC[3] * U(uy, kc, rp, ip);
                const double dudyU = (U(ux, kc, rp, i) - U(ux, kc, rc, i)) * cacU;
                const double dudzC = (IY1 * (-U(ux, ku, rm, i) + 8.0 * U(ux, kp, rm, i) - 8.0 * U(ux, km, rm, i) + U(ux, ks, rm, i)) +
                                      IY2 * (-U(ux, ku, rc, i) + 8.0 * U(ux, kp, rc, i) - 8.0 * U(ux, km, rc, i) + U(ux, ks, rc, i))) * rdzt;
                const double dvdzC = ((-U(uy, ku, rc, is) + 8.0 * U(uy, kp, rc, is) - 8.0 * U(uy, km, rc, is) + U(uy, ks, rc, is)) * I1 +
                                      (-U(uy, ku, rc, im) + 8.0 * U(uy, kp, rc, im) - 8.0 * U(uy, km, rc, im) + U(uy, ks, rc, im)) * I2 +
                                      (-U(uy, ku, rc, i) + 8.0 * U(uy, kp, rc, i) - 8.0 * U(uy, km, rc, i) + U(uy, ks, rc, i)) * I3 +
                                      (-U(uy, ku, rc, ip) + 8.0 * U(uy, kp, rc, ip) - 8.0 * U(uy, km, rc, ip) + U(uy, ks, rc, ip)) * I4) * rdzt;
                v[0] += uxloc;
                v[1] += uyloc;
                v[2] += uzloc;
                v[3] += prloc;
                v[4] += uxloc * uxloc;
                v[5] += uyloc * uyloc;
                v[6] += uzloc * uzloc;
                v[7] += prloc * prloc;
                v[8] += uxCell * uyCell;
                v[9] += uyCell * uzCell;
                v[10] += uxCell * uzCell;
                v[11] += uxCell * prloc;
                v[12] += uyCell * prloc;
                v[13] += uzCell * prloc;
                v[14] += uxCell * uxCell * uyCell;
                v[15] += uyloc * uyloc * uyloc;
                v[16] += uzCell * uzCell * uyCell;
                v[17] += uxCell * uyCell * uyCell;
                v[18] += uxloc * uxloc * uxloc;
                v[19] += uzloc * uzloc * uzloc;
                v[20] += uxloc * uxloc * uxloc * uxloc;
                v[21] += uyloc * uyloc * uyloc * uyloc;
                v[22] += uzloc * uzloc * uzloc * uzloc;
                v[23] += prloc * dudx;
                v[24] += prloc * dvdy;
                v[25] += prloc * dwdz;
                v[26] += prloc2 * (dudy + dvdx);
                v[27] += uxloc * (dudxx + dudyy + dudzz);
                v[28] += uyloc * (dvdxx + dvdyy + dvdzz);
                v[29] += uzloc * (dwdxx + dwdyy + dwdzz);
                v[30] += (dudxC * (dvdxU + dvdx) + (dudyU + dudy) * (uy_xp - uy_xc) * caj) * 0.5;
                v[31] += dudzC * dvdzC;
                v[32] += vor_x * vor_x;
                v[33] += vor_y * vor_y;
                v[34] += vor_z * vor_z;
                if constexpr (NS > 35) {
                    const double scloc = U(sc, kc, rc, i);
                    v[35] += scloc;
                    v[36] += scloc * scloc;
                    v[37] += scloc * uxCell;
                    v[38] += scloc * uyCell;
                    v[39] += scloc * uzCell;
                }
            }
        }
    } else {
        // the top wall row nyp: moments 27, 33, 35 only
        const int jm = jc - 1;
        const double cac = m.rdyc[jc];
        for (int k = k0 + warp; k < k1; k += STAT_THREADS / 32) {
            const size_t kc = (size_t)k * pl;
            const size_t rc = (size_t)jc * nx, rm = (size_t)jm * nx;
            for (int i = lane; i < nx; i += 32) {
                const int is = i >= 2 ? i - 2 : i - 2 + nx, im = i >= 1 ? i - 1 : nx - 1;
                const int ip = i + 1 < nx ? i + 1 : i + 1 - nx;
                const double prloc2 = IY1 * (I1 * U(pr, kc, rm, is) + I2 * U(pr, kc, rm, im) + I3 * U(pr, kc, rm, i) + I4 * U(pr, kc, rm, ip)) +
                                      IY2 * (I1 * U(pr, kc, rc, is) + I2 * U(pr, kc, rc, im) + I3 * U(pr, kc, rc, i) + I4 * U(pr, kc, rc, ip));
                const double dudy = (U(ux, kc, rc, i) - U(ux, kc, rm, i)) * cac;
                const double dwdy = (U(uz, kc, rc, i) - U(uz, kc, rm, i)) * cac;
                const double vor_x = dwdy, vor_z = -dudy;
                v[26] += prloc2 * (dudy + 0.0);
                v[32] += vor_x * vor_x;
                v[34] += vor_z * vor_z;
            }
        }
#undef U
    }
    block_sum_store<NS>(v, part + ((size_t)blockIdx.x * splits + s) * NS);
}

// SumStat[jc-1][q] += (sum over the row's slices, in order) / (nx nz);
// thread 0 of block 0 also adds PrGradAver to PrGradsum
template <int NS>
__global__ void k_stats_final(int nyp, int splits, double inxz, const double* __restrict__ part,
                              double* __restrict__ sumstat, const DCoef* __restrict__ coef,
                              double* __restrict__ prgradsum) {
    const int jr = blockIdx.x;
    for (int q = threadIdx.x; q < NS; q += blockDim.x) {
        double t = 0.0;
        for (int s = 0; s < splits; s++) t += part[((size_t)jr * splits + s) * NS + q];
        sumstat[(size_t)jr * NS + q] += t * inxz;
    }
    if (jr == 0 && threadIdx.x == 0) *prgradsum += coef->pr_grad_aver;
}

}  // namespace

int stats_count(const DConst& c) { return c.scalar_on ? 40 : 35; }

int stats_splits(const DConst& c) {
    int s = (4 * (c.nsm > 0 ? c.nsm : 148) + c.nyp - 1) / c.nyp;
    if (s > c.nz) s = c.nz;
    return s < 1 ? 1 : s;
}

size_t stats_part_doubles(const DConst& c) { return (size_t)c.nyp * stats_splits(c) * stats_count(c); }

void launch_stats(cudaStream_t st, const DConst& c, const DMetric& m, const Fields& f, const DCoef* coef,
                  double* part, double* sumstat, double* prgradsum) {
    const int splits = stats_splits(c);
    const dim3 grid(c.nyp, splits);
    const double inxz = 1.0 / ((double)c.nx * (double)c.nz);
    if (c.scalar_on) {
        k_stats<40><<<grid, STAT_THREADS, 0, st>>>(c, m, f.ux, f.uy, f.uz, f.pr, f.sc, splits, part);
        k_stats_final<40><<<c.nyp, 64, 0, st>>>(c.nyp, splits, inxz, part, sumstat, coef, prgradsum);
    } else {
        k_stats<35><<<grid, STAT_THREADS, 0, st>>>(c, m, f.ux, f.uy, f.uz, f.pr, f.sc, splits, part);
        k_stats_final<35><<<c.nyp, 64, 0, st>>>(c.nyp, splits, inxz, part, sumstat, coef, prgradsum);
    }
}

}  // namespace ptc
