// host_setup.h -- host-side set-up helpers (metrics, y-grid, namelist).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/paratc.h"

namespace ptc {

// coefficients of m_MeshAndMetries / m_Poisson / m_Parameters for one grid
struct HostMetrics {
    double dx, dy, dz, rdx, rdy, rdz, rdx2, rdz2;
    double dxC[4], dzC[4], dxxC[5], dzzC[5], IC[4];
    std::vector<double> yp, yc, dyp, dyc, rdyp, rdyc, yinterp;
    std::vector<double> ap2ph, ac2ph, am2ph, ap2c, ac2c, am2c, ap2cCN, ac2cCN, am2cCN, ap2p, ac2p, am2p;
    std::vector<double> ap2cSc, ac2cSc, am2cSc, ap2cScCN, ac2cScCN, am2cScCN;
    std::vector<double> wnx, wnz;
    double normfft;
    double sc_r1b = 0, sc_r2b = 0, sc_r1t = 0, sc_r2t = 0;
    int iadvance;
    double gam[3], the[3], alp[3];
    std::vector<std::vector<double>*> arrays() {
        return {&yp, &yc, &dyp, &dyc, &rdyp, &rdyc, &yinterp, &ap2ph, &ac2ph, &am2ph, &ap2c, &ac2c, &am2c,
                &ap2cCN, &ac2cCN, &am2cCN, &ap2p, &ac2p, &am2p, &ap2cSc, &ac2cSc, &am2cSc, &ap2cScCN, &ac2cScCN,
                &am2cScCN};
    }
};

struct RunOptions {
    int ifirst = 1, ilast = 0, restart_flag = 0, backup_freq = 0, cmd_lfile_freq = 1;
    char run_name[64] = {0};
    char res_dir[256] = {0};
    char restart_dir[256] = {0};
};

int mesh_ycoord(int nsection, const double* section_length, const double* section_cstret, const int32_t* nyc_section,
                const int32_t* stret_type, const int32_t* stret_option, double yly, double* yp_out);
int validate_params(const paratc_params& p, std::string& why);
int build_metrics(const paratc_params& p, const double* yp, HostMetrics& h);
int parse_namelist(const char* path, int scalar_on, paratc_params& P, std::vector<double>* yp, RunOptions* ro,
                   std::string& why);

}  // namespace ptc
