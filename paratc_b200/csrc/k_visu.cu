// k_visu.cu -- the quantities dump_visu writes (src/m_IOAndVisu.f90:182-385):
// cell-centre (or, with SaveNode, staggered) velocities, pressure, scalar,
// the vorticity components and magnitude, Q (Clc_Q_vor, src/m_Tools.f90:
// 305-353) and lambda2 (Clc_lamda2 with CubicRoot, :356-440, :494-570), at
// the points decomp_2d_write_every keeps with from1 = .true.
// (src/m_Decomp2d.f90:1232-1389): global indices 1, 1+skip, 1+2 skip, ...
// in each direction.  One thread per kept point, consecutive threads on
// consecutive x, so a skip of 1 reads and writes whole rows.
#include <algorithm>

#include "../../include/paratc.h"
#include "common.cuh"
#include "kernels.cuh"

namespace ptc {
namespace {

struct VisuArgs {
    int q, iskip, jskip, kskip, node, nxo, nyo, nzo;
};

// CubicRoot (src/m_Tools.f90:494-570): the middle root of
// x^3 + b x^2 + c x + d (real branch: roots sorted ascending); *complex is
// set when the discriminant says the roots are not all real, where the
// reference stops with "lamda2 wrong"
__device__ double cubic_middle_root(double b, double c, double d, bool* complex_roots) {
    const double SMALL = 1.0e-12, third = 1.0 / 3.0;
    const double pi = 3.141592653589793238462643383279502884;
    const double p = c - third * b * b;
    const double q = (2.0 * b * b * b - 9.0 * b * c + 27.0 * d) / 27.0;
    const double t = q * q / 4.0 + p * p * p / 27.0;
    *complex_roots = false;
    if (t < 0.0) {
        const double tt = -third * b;
        double rho = pow(-p, 1.5) / sqrt(27.0);
        const double eta = acos(0.5 * q / rho);
        rho = -2.0 * pow(rho, third);
        const double r1 = cos(third * eta) * rho + tt;
        const double r2 = cos(third * (2.0 * pi + eta)) * rho + tt;
        const double r3 = cos(third * (4.0 * pi + eta)) * rho + tt;
        if (r1 < r2 && r1 < r3) return r2 < r3 ? r2 : r3;
        if (r1 > r2 && r1 > r3) return r2 < r3 ? r3 : r2;
        return r1;
    }
    if (t < SMALL) {
        double rho = 0.5 * q;
        rho = rho < 0.0 ? pow(-rho, third) : -pow(rho, third);
        return -rho - third * b;
    }
    *complex_roots = true;
    const double ts = sqrt(t);
    double rho = 0.5 * q + ts, eta = 0.5 * q - ts;
    rho = rho < 0.0 ? pow(-rho, third) : -pow(rho, third);
    eta = eta < 0.0 ? pow(-eta, third) : -pow(eta, third);
    return -0.5 * (rho + eta) - third * b;
}

__global__ void k_visu(VisuArgs a, DConst c, DMetric m, const double* __restrict__ ux, const double* __restrict__ uy,
                       const double* __restrict__ uz, const double* __restrict__ pr, const double* __restrict__ sc,
                       double* __restrict__ out, unsigned int* __restrict__ nbad) {
    const int nx = c.nx, nz = c.nz;
    const size_t pl = (size_t)c.nyt * nx;
    const long long tot = (long long)a.nxo * a.nyo * a.nzo;
    const double quarter = 0.25;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int io = (int)(t % a.nxo);
        const long long r = t / a.nxo;
        const int jo = (int)(r % a.nyo), ko = (int)(r / a.nyo);
        const int i = io * a.iskip, jc = 1 + jo * a.jskip, k = ko * a.kskip;
        const int ip = i + 1 < nx ? i + 1 : 0, im = i >= 1 ? i - 1 : nx - 1;
        const int kp = k + 1 < nz ? k + 1 : 0, km = k >= 1 ? k - 1 : nz - 1;
        const int jp = jc + 1, jm = jc - 1;
#define V(f, kk, jj, ii) __ldg(&(f)[(size_t)(kk) * pl + (size_t)(jj) * nx + (ii)])
        double v = 0.0;
        switch (a.q) {
            case PARATC_VISU_UX:
                v = a.node ? V(ux, k, jc, i) + c.ucrf : 0.5 * (V(ux, k, jc, ip) + V(ux, k, jc, i)) + c.ucrf;
                break;
            case PARATC_VISU_UY:
                v = a.node ? V(uy, k, jc, i) : 0.5 * (V(uy, k, jp, i) + V(uy, k, jc, i));
                break;
            case PARATC_VISU_UZ:
                v = a.node ? V(uz, k, jc, i) : 0.5 * (V(uz, kp, jc, i) + V(uz, k, jc, i));
                break;
            case PARATC_VISU_PR: v = V(pr, k, jc, i); break;
            case PARATC_VISU_SCALAR: v = V(sc, k, jc, i); break;
            default: {
                const double rdx = c.rdx, rdz = c.rdz;
                const double cac1 = m.rdyc[jc], cac2 = m.rdyc[jp], cac12 = cac1 - cac2;
                const double dudy = ((V(ux, k, jp, ip) + V(ux, k, jp, i)) * cac2 + (V(ux, k, jc, ip) + V(ux, k, jc, i)) * cac12 -
                                     (V(ux, k, jm, ip) + V(ux, k, jm, i)) * cac1) * quarter;
                const double dudz = (V(ux, kp, jc, ip) + V(ux, kp, jc, i) - V(ux, km, jc, ip) - V(ux, km, jc, i)) * rdz * quarter;
                const double dvdx = (V(uy, k, jp, ip) - V(uy, k, jp, im) + V(uy, k, jc, ip) - V(uy, k, jc, im)) * rdx * quarter;
                const double dvdz = (V(uy, kp, jp, i) + V(uy, kp, jc, i) - V(uy, km, jp, i) - V(uy, km, jc, i)) * rdz * quarter;
                const double dwdx = (V(uz, kp, jc, ip) - V(uz, kp, jc, im) + V(uz, k, jc, ip) - V(uz, k, jc, im)) * rdx * quarter;
                const double dwdy = ((V(uz, kp, jp, i) + V(uz, k, jp, i)) * cac2 + (V(uz, kp, jc, i) + V(uz, k, jc, i)) * cac12 -
                                     (V(uz, kp, jm, i) + V(uz, k, jm, i)) * cac1) * quarter;
                if (a.q == PARATC_VISU_WX) { v = dwdy - dvdz; break; }
                if (a.q == PARATC_VISU_WY) { v = dudz - dwdx; break; }
                if (a.q == PARATC_VISU_WZ) { v = dvdx - dudy; break; }
                if (a.q == PARATC_VISU_WMAG) {
                    const double vx = dwdy - dvdz, vy = dudz - dwdx, vz = dvdx - dudy;
                    v = sqrt(vx * vx + vy * vy + vz * vz);
                    break;
                }
                const double dudx = (V(ux, k, jc, ip) - V(ux, k, jc, i)) * rdx;
                const double dvdy = (V(uy, k, jp, i) - V(uy, k, jc, i)) * m.rdyp[jc];
                const double dwdz = (V(uz, kp, jc, i) - V(uz, k, jc, i)) * rdz;
                if (a.q == PARATC_VISU_Q) {
                    const double udiv = dudx + dvdy + dwdz;
                    v = 0.5 * (udiv * udiv - dudx * dudx - dvdy * dvdy - dwdz * dwdz) - dudy * dvdx - dudz * dwdx - dvdz * dwdy;
                    break;
                }
                // lambda2: middle eigenvalue of Ome.Ome + Eps.Eps (with the
                // reference's factor-2 Ome and Eps, hence the quarter)
                const double O12 = dvdx - dudy, O23 = dwdy - dvdz, O31 = dudz - dwdx;
                const double E11 = dudx + dudx, E12 = dudy + dvdx, E13 = dudz + dwdx;
                const double E22 = dvdy + dvdy, E23 = dvdz + dwdy, E33 = dwdz + dwdz;
                const double L12 = E11 * E12 + E12 * E22 + E13 * E23 + O31 * O23;
                const double L13 = E11 * E13 + E12 * E23 + E13 * E33 + O12 * O23;
                const double L23 = E12 * E13 + E22 * E23 + E23 * E33 + O12 * O31;
                const double L11 = E11 * E11 + E12 * E12 + E13 * E13 - O12 * O12 - O31 * O31;
                const double L22 = E12 * E12 + E22 * E22 + E23 * E23 - O12 * O12 - O23 * O23;
                const double L33 = E13 * E13 + E23 * E23 + E33 * E33 - O31 * O31 - O23 * O23;
                const double rb = -(L11 + L22 + L33);
                const double rc = L11 * L22 + L22 * L33 + L33 * L11 - L12 * L12 - L13 * L13 - L23 * L23;
                const double rd = L12 * L12 * L33 + L13 * L13 * L22 + L23 * L23 * L11 - L11 * L22 * L33 - 2.0 * L12 * L23 * L13;
                bool cplx;
                v = quarter * cubic_middle_root(rb, rc, rd, &cplx);
                if (cplx) atomicAdd(nbad, 1u);
                break;
            }
        }
#undef V
        out[t] = v;
    }
}

}  // namespace

// count of kept points along one direction: global indices 1, 1+skip, ..., <= n
int visu_count(int n, int skip) { return skip >= 1 ? (n + skip - 1) / skip : 0; }

void launch_visu(cudaStream_t st, int q, int iskip, int jskip, int kskip, int node, const DConst& c, const DMetric& m,
                 const Fields& f, double* out, unsigned int* nbad) {
    VisuArgs a{q, iskip, jskip, kskip, node, visu_count(c.nx, iskip), visu_count(c.ny, jskip), visu_count(c.nz, kskip)};
    const long long tot = (long long)a.nxo * a.nyo * a.nzo;
    const long long cap = 16LL * (c.nsm > 0 ? c.nsm : 148);
    const int blocks = (int)std::max(1LL, std::min((tot + 255) / 256, cap));
    k_visu<<<blocks, 256, 0, st>>>(a, c, m, f.ux, f.uy, f.uz, f.pr, f.sc, out, nbad);
}

}  // namespace ptc
