// host_setup.cpp -- host-side set-up of the hot path: y-grid, metrics,
// wavenumbers, RK constants and the ParaTC namelist input format.
//
// These run once per context on the CPU (they are O(ny) and O(nx+nz)) and
// follow the reference routine named beside each function, expression by
// expression, so that the device kernels see the same coefficients as the
// Fortran code.
#include "host_setup.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace ptc {

// clcYcoord (src/m_MeshAndMetries.f90:340-408); y is 1-based
static void clc_ycoord(std::vector<double>& y, int nid1, int nid2, double ys1, double ys2, int stret_type,
                       double cstret, int stret_option) {
    const int m = nid2 - nid1;
    const double ylen = ys2 - ys1;
    y[nid1] = ys1;
    y[nid2] = ys2;
    if (stret_type == 0) {
        for (int j = 0; j <= m; j++) y[nid1 + j] = ys1 + (double)j / (double)m * ylen;
    } else if (stret_type == 1) {
        const double tstr = std::tanh(cstret);
        for (int j = 0; j <= m; j++) {
            const double xi = (double)j / (double)(float)m;  // real(m) is default real
            const double y0 = std::tanh(cstret * (xi - 1.0)) / tstr + 1.0;
            if (stret_option == 0) y[nid1 + j] = ys1 + y0 * ylen;
            else y[nid2 - j] = ys2 - y0 * ylen;
        }
    } else if (stret_type == 2) {
        const double PI = 3.141592653589793238462643383279502884;
        const double tstr = std::sin(0.5 * cstret * PI);
        for (int j = 0; j <= m; j++) {
            const double xi = (double)j / (double)m - 1.0;
            const double y0 = std::sin(cstret * xi * PI * 0.5) / tstr + 1.0;
            if (stret_option == 0) y[nid1 + j] = ys1 + y0 * ylen;
            else y[nid2 - j] = ys2 - y0 * ylen;
        }
    } else if (stret_type == 3) {
        if (cstret == 1.0) {
            for (int j = 0; j <= m; j++) y[j + nid1] = ys1 + (double)j / (double)m * ylen;
        } else {
            const double tstr = (std::pow(cstret, m) - 1.0) / (cstret - 1.0);
            for (int j = 0; j <= m - 1; j++) {
                const double y0 = std::pow(cstret, j) / tstr;
                if (stret_option == 0) { const int jt = nid1 + j; y[jt + 1] = y[jt] + y0 * ylen; }
                else { const int jt = nid2 - j; y[jt - 1] = y[jt] - y0 * ylen; }
            }
        }
    }
    y[nid1] = ys1;
    y[nid2] = ys2;
}

// section loop of InitMeshAndMetries (src/m_MeshAndMetries.f90:143-181)
int mesh_ycoord(int nsection, const double* section_length, const double* section_cstret, const int32_t* nyc_section,
                const int32_t* stret_type, const int32_t* stret_option, double yly, double* yp_out) {
    if (nsection < 1 || !section_length || !section_cstret || !nyc_section || !stret_type || !stret_option || !yp_out)
        return PARATC_ERR_BAD_ARG;
    int nyc = 0;
    double sumlen = 0.0;
    for (int s = 0; s < nsection; s++) {
        if (section_length[s] < 0.0 || section_cstret[s] < 0.0 || nyc_section[s] < 1 || stret_type[s] < 0 ||
            stret_type[s] > 3 || stret_option[s] < 0 || stret_option[s] > 1)
            return PARATC_ERR_BAD_ARG;
        nyc += nyc_section[s];
        sumlen += section_length[s];
    }
    const int nyp = nyc + 1;
    std::vector<double> y(nyp + 2, 0.0);
    std::vector<int> nid(nsection + 1);
    std::vector<double> ysc(nsection + 1);
    nid[0] = 1;
    ysc[0] = 0.0;
    for (int s = 0; s < nsection; s++) {
        nid[s + 1] = nid[s] + nyc_section[s];
        ysc[s + 1] = ysc[s] + section_length[s] / sumlen * yly;
    }
    ysc[nsection] = yly;
    for (int s = 0; s < nsection; s++)
        clc_ycoord(y, nid[s], nid[s + 1], ysc[s], ysc[s + 1], stret_type[s], section_cstret[s], stret_option[s]);
    for (int j = 1; j <= nyp; j++) yp_out[j - 1] = y[j];
    return PARATC_OK;
}

int validate_params(const paratc_params& p, std::string& why) {
    if (p.nxc < 4 || p.nyc < 3 || p.nzc < 4) { why = "grid too small (nxc, nzc >= 4, nyc >= 3)"; return PARATC_ERR_BAD_ARG; }
    if (p.nxc % 2 != 0 || p.nzc % 2 != 0) { why = "mod(nxc,2)/=0 || mod(nzc,2)/=0"; return PARATC_ERR_BAD_ARG; }
    if (p.flow_type == PARATC_FT_CH && p.nyc % 2 != 0) { why = "mod(nyc,2)/=0 for channel geometry"; return PARATC_ERR_BAD_ARG; }
    if (p.flow_type != PARATC_FT_CH && p.flow_type != PARATC_FT_HC) { why = "FlowType must be 1 or 2"; return PARATC_ERR_BAD_ARG; }
    if (p.ischeme < 1 || p.ischeme > 3) { why = "ischeme must be 1, 2 or 3"; return PARATC_ERR_BAD_ARG; }
    if (p.icfl != 1 && p.icfl != 2) { why = "iCFL must be 1 or 2"; return PARATC_ERR_BAD_ARG; }
    if (!(p.xlx > 0) || !(p.yly > 0) || !(p.zlz > 0)) { why = "domain lengths must be positive"; return PARATC_ERR_BAD_ARG; }
    if (!(p.dt_max > 0)) { why = "dtMax must be positive"; return PARATC_ERR_BAD_ARG; }
    if (p.scalar_on) {
        for (int s = 0; s < 2; s++)
            if (p.scalar_bc_option[s] < -3 || p.scalar_bc_option[s] > -1) {
                why = "ScalarBcOption must be -1, -2 or -3";
                return PARATC_ERR_BAD_ARG;
            }
    }
    return PARATC_OK;
}

// InitMeshAndMetries (src/m_MeshAndMetries.f90:86-335) and the wavenumbers of
// InitPoissonSolver (src/m_Poisson.f90:36-48)
int build_metrics(const paratc_params& p, const double* yp_in, HostMetrics& h) {
    const int nxc = p.nxc, nyc = p.nyc, nzc = p.nzc, nyp = nyc + 1;
    h.dx = p.xlx / (double)nxc; h.dy = p.yly / (double)nyc; h.dz = p.zlz / (double)nzc;
    h.rdx = (double)nxc / p.xlx; h.rdy = (double)nyc / p.yly; h.rdz = (double)nzc / p.zlz;
    h.rdx2 = h.rdx * h.rdx; h.rdz2 = h.rdz * h.rdz;
    const double rdx = h.rdx, rdz = h.rdz, rdx2 = h.rdx2, rdz2 = h.rdz2;
    h.dxC[0] = rdx / 24.0; h.dxC[1] = -rdx * 1.125; h.dxC[2] = rdx * 1.125; h.dxC[3] = -rdx / 24.0;
    h.dzC[0] = rdz / 24.0; h.dzC[1] = -rdz * 1.125; h.dzC[2] = rdz * 1.125; h.dzC[3] = -rdz / 24.0;
    h.dxxC[0] = -rdx2 / 12.0; h.dxxC[1] = 4.0 / 3.0 * rdx2; h.dxxC[2] = -2.5 * rdx2; h.dxxC[3] = 4.0 / 3.0 * rdx2; h.dxxC[4] = -rdx2 / 12.0;
    h.dzzC[0] = -rdz2 / 12.0; h.dzzC[1] = 4.0 / 3.0 * rdz2; h.dzzC[2] = -2.5 * rdz2; h.dzzC[3] = 4.0 / 3.0 * rdz2; h.dzzC[4] = -rdz2 / 12.0;
    h.IC[0] = -1.0 / 16.0; h.IC[1] = 9.0 / 16.0; h.IC[2] = 9.0 / 16.0; h.IC[3] = -1.0 / 16.0;

    for (auto* v : h.arrays()) v->assign(nyp + 1, 0.0);
    auto &yp = h.yp, &yc = h.yc, &dyp = h.dyp, &dyc = h.dyc, &rdyp = h.rdyp, &rdyc = h.rdyc;
    for (int j = 1; j <= nyp; j++) yp[j] = yp_in[j - 1];
    for (int j = 1; j < nyp; j++)
        if (!(yp[j + 1] > yp[j])) return PARATC_ERR_BAD_ARG;
    for (int j = 1; j <= nyc; j++) yc[j] = 0.5 * (yp[j] + yp[j + 1]);
    yc[0] = 2.0 * yp[1] - yc[1];
    yc[nyp] = 2.0 * yp[nyp] - yc[nyc];
    for (int j = 1; j <= nyc; j++) dyp[j] = yp[j + 1] - yp[j];
    dyp[0] = dyp[1];
    dyp[nyp] = dyp[nyc];
    for (int j = 2; j <= nyc; j++) dyc[j] = yc[j] - yc[j - 1];
    dyc[1] = dyp[1];
    dyc[nyp] = dyp[nyc];
    for (int j = 0; j <= nyp; j++) rdyp[j] = 1.0 / dyp[j];
    for (int j = 1; j <= nyp; j++) rdyc[j] = 1.0 / dyc[j];
    for (int j = 1; j <= nyp; j++) h.yinterp[j] = dyp[j] / (dyp[j] + dyp[j - 1]);

    for (int j = 1; j <= nyc; j++) { h.am2ph[j] = rdyp[j] * rdyc[j]; h.ap2ph[j] = rdyp[j] * rdyc[j + 1]; }
    h.am2ph[1] = 0.0; h.ap2ph[1] = rdyp[1] * rdyc[2];
    h.am2ph[nyc] = rdyp[nyc] * rdyc[nyc]; h.ap2ph[nyc] = 0.0;
    for (int j = 1; j <= nyc; j++) h.ac2ph[j] = -(h.am2ph[j] + h.ap2ph[j]);

    for (int j = 1; j <= nyc; j++) { h.am2c[j] = rdyp[j] * rdyc[j]; h.ap2c[j] = rdyp[j] * rdyc[j + 1]; }
    h.am2c[1] = 4.0 * rdyc[1] / (dyc[1] + 2.0 * dyc[2]);
    h.ap2c[1] = 4.0 * rdyc[2] / (dyc[1] + 2.0 * dyc[2]);
    if (p.flow_type == PARATC_FT_CH) {
        h.am2c[nyc] = 4.0 * rdyc[nyc] / (dyc[nyp] + 2.0 * dyc[nyc]);
        h.ap2c[nyc] = 4.0 * rdyc[nyp] / (dyc[nyp] + 2.0 * dyc[nyc]);
    } else {
        h.am2c[nyc] = rdyp[nyc] * rdyc[nyc];
        h.ap2c[nyc] = 0.0;
    }
    for (int j = 1; j <= nyc; j++) h.ac2c[j] = -(h.am2c[j] + h.ap2c[j]);
    for (int j = 1; j <= nyc; j++) { h.ap2cCN[j] = h.ap2c[j]; h.ac2cCN[j] = h.ac2c[j]; h.am2cCN[j] = h.am2c[j]; }
    h.ap2cCN[1] = h.ap2c[1];
    h.ac2cCN[1] = h.ac2c[1] - h.am2c[1];
    h.am2cCN[1] = 2.0 * h.am2c[1];
    if (p.flow_type == PARATC_FT_CH) {
        h.am2cCN[nyc] = h.am2c[nyc];
        h.ac2cCN[nyc] = h.ac2c[nyc] - h.ap2c[nyc];
        h.ap2cCN[nyc] = 2.0 * h.ap2c[nyc];
    }
    for (int j = 1; j <= nyc; j++) { h.am2p[j] = rdyc[j] * rdyp[j - 1]; h.ap2p[j] = rdyc[j] * rdyp[j]; }
    for (int j = 1; j <= nyc; j++) h.ac2p[j] = -(h.am2p[j] + h.ap2p[j]);

    if (p.scalar_on) {
        const int* opt = p.scalar_bc_option;
        const double* v = p.scalar_bc_values;
        for (int j = 1; j <= nyc; j++) { h.am2cSc[j] = rdyp[j] * rdyc[j]; h.ap2cSc[j] = rdyp[j] * rdyc[j + 1]; }
        if (opt[0] == -1) {
            h.am2cSc[1] = 4.0 * rdyc[1] / (dyc[1] + 2.0 * dyc[2]);
            h.ap2cSc[1] = 4.0 * rdyc[2] / (dyc[1] + 2.0 * dyc[2]);
        }
        if (opt[1] == -1) {
            h.am2cSc[nyc] = 4.0 * rdyc[nyc] / (dyc[nyp] + 2.0 * dyc[nyc]);
            h.ap2cSc[nyc] = 4.0 * rdyc[nyp] / (dyc[nyp] + 2.0 * dyc[nyc]);
        }
        for (int j = 1; j <= nyc; j++) h.ac2cSc[j] = -(h.am2cSc[j] + h.ap2cSc[j]);
        for (int j = 1; j <= nyc; j++) { h.am2cScCN[j] = rdyp[j] * rdyc[j]; h.ap2cScCN[j] = rdyp[j] * rdyc[j + 1]; }
        for (int j = 1; j <= nyc; j++) h.ac2cScCN[j] = -(h.am2cScCN[j] + h.ap2cScCN[j]);
        if (opt[0] == -1) {
            h.am2cScCN[1] = 8.0 * rdyc[1] / (dyc[1] + 2.0 * dyc[2]);
            h.ap2cScCN[1] = 4.0 * rdyc[2] / (dyc[1] + 2.0 * dyc[2]);
            h.ac2cScCN[1] = -(8.0 * rdyc[1] + 4.0 * rdyc[2]) / (dyc[1] + 2.0 * dyc[2]);
        } else if (opt[0] == -2) {
            h.ap2cScCN[1] = rdyp[1] * rdyc[2];
            h.ac2cScCN[1] = -rdyp[1] * rdyc[2];
            h.am2cScCN[1] = 0.0;
        } else if (opt[0] == -3) {
            h.ap2cScCN[1] = rdyp[1] * rdyc[2];
            h.ac2cScCN[1] = h.ac2cScCN[1] + h.am2cScCN[1] * (2.0 + v[0] * dyc[1]) / (2.0 - v[0] * dyc[1]);
            h.am2cScCN[1] = 0.0;
        }
        if (opt[1] == -1) {
            h.am2cScCN[nyc] = 4.0 * rdyc[nyc] / (dyc[nyp] + 2.0 * dyc[nyc]);
            h.ap2cScCN[nyc] = 8.0 * rdyc[nyp] / (dyc[nyp] + 2.0 * dyc[nyc]);
            h.ac2cScCN[nyc] = -(8.0 * rdyc[nyp] + 4.0 * rdyc[nyc]) / (dyc[nyp] + 2.0 * dyc[nyc]);
        } else if (opt[1] == -2) {
            h.am2cScCN[nyc] = rdyp[nyc] * rdyc[nyc];
            h.ac2cScCN[nyc] = -rdyp[nyc] * rdyc[nyc];
            h.ap2cScCN[nyc] = 0.0;
        } else if (opt[1] == -3) {
            h.am2cScCN[nyc] = rdyp[nyc] * rdyc[nyc];
            h.ac2cScCN[nyc] = h.ac2cScCN[nyc] + h.ap2cScCN[nyc] * (2.0 - v[1] * dyc[nyp]) / (2.0 + v[1] * dyc[nyp]);
            h.ap2cScCN[nyc] = 0.0;
        }
        // ghost coefficients of SetBC_and_UpdateHalo_scalar (src/m_BC_and_Halo.f90:137-176)
        if (opt[0] == -1) { h.sc_r1b = -1.0; h.sc_r2b = 2.0 * v[0]; }
        else if (opt[0] == -2) { h.sc_r1b = 1.0; h.sc_r2b = -dyc[1] * v[2]; }
        else { h.sc_r1b = (2.0 + v[0] * dyc[1]) / (2.0 - v[0] * dyc[1]); h.sc_r2b = -(2.0 * v[2] * dyc[1] / (2.0 - v[0] * dyc[1])); }
        if (opt[1] == -1) { h.sc_r1t = -1.0; h.sc_r2t = 2.0 * v[1]; }
        else if (opt[1] == -2) { h.sc_r1t = 1.0; h.sc_r2t = dyc[nyp] * v[3]; }
        else { h.sc_r1t = (2.0 - v[1] * dyc[nyp]) / (2.0 + v[1] * dyc[nyp]); h.sc_r2t = 2.0 * v[3] * dyc[nyp] / (2.0 + v[1] * dyc[nyp]); }
    }

    const double twopi = 6.283185307179586476925286766559005768;
    h.wnx.assign(nxc, 0.0);
    h.wnz.assign(nzc, 0.0);
    for (int i = 1; i <= nxc; i++) {
        const double wa1 = twopi * (double)(i - 1) / (double)nxc;
        h.wnx[i - 1] = rdx2 / 288.0 * (std::cos(3.0 * wa1) - 54.0 * std::cos(2.0 * wa1) + 783.0 * std::cos(wa1) - 730.0);
    }
    for (int k = 1; k <= nzc; k++) {
        const double wa3 = twopi * (double)(k - 1) / (double)nzc;
        h.wnz[k - 1] = rdz2 / 288.0 * (std::cos(3.0 * wa3) - 54.0 * std::cos(2.0 * wa3) + 783.0 * std::cos(wa3) - 730.0);
    }
    h.normfft = 1.0 / ((double)nxc * (double)nzc);

    // RK coefficients of ReadAndInitParameters (src/m_Parameters.f90:159-174)
    if (p.ischeme == PARATC_AB2) {
        h.iadvance = 1;
        h.gam[0] = 3.0 / 2.0; h.gam[1] = 0.0; h.gam[2] = 0.0;
        h.the[0] = -0.5; h.the[1] = 0.0; h.the[2] = 0.0;
    } else if (p.ischeme == PARATC_RK2) {
        h.iadvance = 2;
        h.gam[0] = 0.5; h.gam[1] = 1.0; h.gam[2] = 0.0;
        h.the[0] = 0.0; h.the[1] = -0.5; h.the[2] = 0.0;
    } else {
        h.iadvance = 3;
        h.gam[0] = 8.0 / 15.0; h.gam[1] = 5.0 / 12.0; h.gam[2] = 3.0 / 4.0;
        h.the[0] = 0.0; h.the[1] = -17.0 / 60.0; h.the[2] = -5.0 / 12.0;
    }
    for (int q = 0; q < 3; q++) h.alp[q] = h.gam[q] + h.the[q];
    return PARATC_OK;
}

// ---------------------------------------------------------------------------
// namelist input (src/m_Parameters.f90:112-188, src/m_MeshAndMetries.f90:143-165;
// the format is described in doc/ParaTC_prm.md)
// ---------------------------------------------------------------------------
static std::string lower(std::string s) {
    for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
    return s;
}

// returns name -> list of value tokens for one "&group ... /" block
static int read_group(const std::string& text, const std::string& group, std::map<std::string, std::vector<std::string>>& out) {
    // strip comments ('!' outside quotes), keep line structure
    std::string clean;
    {
        bool inq = false;
        char q = 0;
        bool comment = false;
        for (char ch : text) {
            if (ch == '\n') { comment = false; clean.push_back('\n'); continue; }
            if (comment) continue;
            if (inq) { clean.push_back(ch); if (ch == q) inq = false; continue; }
            if (ch == '"' || ch == '\'') { inq = true; q = ch; clean.push_back(ch); continue; }
            if (ch == '!') { comment = true; continue; }
            clean.push_back(ch);
        }
    }
    const std::string lc = lower(clean);
    const std::string key = "&" + lower(group);
    size_t pos = 0, start = std::string::npos;
    while ((pos = lc.find(key, pos)) != std::string::npos) {
        const size_t e = pos + key.size();
        if (e >= lc.size() || !(std::isalnum((unsigned char)lc[e]) || lc[e] == '_')) { start = e; break; }
        pos = e;
    }
    if (start == std::string::npos) return PARATC_ERR_IO;
    // body ends at the first '/' outside quotes
    size_t end = start;
    {
        bool inq = false;
        char q = 0;
        for (; end < clean.size(); end++) {
            const char ch = clean[end];
            if (inq) { if (ch == q) inq = false; continue; }
            if (ch == '"' || ch == '\'') { inq = true; q = ch; continue; }
            if (ch == '/') break;
        }
    }
    const std::string body = clean.substr(start, end - start);
    // tokens: identifiers, '=', quoted strings, values; commas/whitespace separate
    std::vector<std::string> tok;
    for (size_t i = 0; i < body.size();) {
        const char ch = body[i];
        if (std::isspace((unsigned char)ch) || ch == ',') { i++; continue; }
        if (ch == '=') { tok.push_back("="); i++; continue; }
        if (ch == '"' || ch == '\'') {
            size_t j = body.find(ch, i + 1);
            if (j == std::string::npos) j = body.size();
            tok.push_back(body.substr(i, j - i + 1));
            i = j + 1;
            continue;
        }
        size_t j = i;
        while (j < body.size() && !std::isspace((unsigned char)body[j]) && body[j] != ',' && body[j] != '=') j++;
        tok.push_back(body.substr(i, j - i));
        i = j;
    }
    std::string cur;
    for (size_t t = 0; t < tok.size(); t++) {
        if (t + 1 < tok.size() && tok[t + 1] == "=") {
            cur = lower(tok[t]);
            out[cur].clear();
            t++;
            continue;
        }
        if (cur.empty() || tok[t] == "=") return PARATC_ERR_BAD_ARG;
        // r*value repeat form
        const std::string& v = tok[t];
        const size_t star = v.find('*');
        if (star != std::string::npos && star > 0 && v[0] != '"' && v[0] != '\'') {
            const int rep = std::atoi(v.substr(0, star).c_str());
            for (int r = 0; r < rep; r++) out[cur].push_back(v.substr(star + 1));
        } else {
            out[cur].push_back(v);
        }
    }
    return PARATC_OK;
}

static double to_d(const std::string& s) {
    std::string t = s;
    for (auto& ch : t) if (ch == 'd' || ch == 'D') ch = 'e';
    return std::strtod(t.c_str(), nullptr);
}
static bool to_b(const std::string& s) {
    std::string t = lower(s);
    if (!t.empty() && t[0] == '.') t = t.substr(1);
    return !t.empty() && t[0] == 't';
}
static std::string to_s(const std::string& s) {
    if (s.size() >= 2 && (s[0] == '"' || s[0] == '\'')) return s.substr(1, s.size() - 2);
    return s;
}

int parse_namelist(const char* path, int scalar_on, paratc_params& P, std::vector<double>* yp, RunOptions* ro,
                   std::string& why) {
    std::ifstream in(path);
    if (!in) { why = std::string("Cannot open file: ") + path; return PARATC_ERR_IO; }
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string text = ss.str();
    std::map<std::string, std::vector<std::string>> bp, ms, mo, so;
    if (read_group(text, "BasicParam", bp) != PARATC_OK) { why = "&BasicParam missing or malformed"; return PARATC_ERR_BAD_ARG; }
    auto getd = [&](std::map<std::string, std::vector<std::string>>& g, const char* n, int idx, double dflt) {
        auto it = g.find(lower(n));
        if (it == g.end() || (int)it->second.size() <= idx) return dflt;
        return to_d(it->second[idx]);
    };
    auto geti = [&](std::map<std::string, std::vector<std::string>>& g, const char* n, int idx, int dflt) {
        auto it = g.find(lower(n));
        if (it == g.end() || (int)it->second.size() <= idx) return dflt;
        return (int)std::lround(to_d(it->second[idx]));
    };
    auto getb = [&](std::map<std::string, std::vector<std::string>>& g, const char* n, bool dflt) {
        auto it = g.find(lower(n));
        if (it == g.end() || it->second.empty()) return dflt;
        return to_b(it->second[0]);
    };
    std::memset(&P, 0, sizeof(P));
    P.flow_type = geti(bp, "FlowType", 0, 1);
    P.ubulk = getd(bp, "ubulk", 0, 0.0);
    P.xlx = getd(bp, "xlx", 0, 0.0);
    P.yly = getd(bp, "yly", 0, 0.0);
    P.zlz = getd(bp, "zlz", 0, 0.0);
    const int nxp = geti(bp, "nxp", 0, 0), nyp = geti(bp, "nyp", 0, 0), nzp = geti(bp, "nzp", 0, 0);
    P.nxc = nxp - 1; P.nyc = nyp - 1; P.nzc = nzp - 1;
    P.xnu = getd(bp, "xnu", 0, 0.0);
    P.dt_max = getd(bp, "dtMax", 0, 0.0);
    P.icfl = geti(bp, "iCFL", 0, 2);
    P.cflc = getd(bp, "CFLc", 0, 0.0);
    P.ischeme = geti(bp, "ischeme", 0, 3);
    for (int q = 0; q < 3; q++) P.gravity[q] = getd(bp, "gravity", q, 0.0);
    for (int q = 0; q < 6; q++) {
        P.ux_bc[q] = getd(bp, "uxBcValue", q, 0.0);
        P.uy_bc[q] = getd(bp, "uyBcValue", q, 0.0);
        P.uz_bc[q] = getd(bp, "uzBcValue", q, 0.0);
    }
    P.is_ux_const = getb(bp, "IsUxConst", false) ? 1 : 0;
    const bool use_crf = getb(bp, "IsUseCRF", false);
    P.ucrf = getd(bp, "uCRF", 0, 0.0);
    P.vel_limit = getd(bp, "vel_limit", 0, 0.0);
    P.div_limit = getd(bp, "div_limit", 0, 0.0);
    P.scalar_on = scalar_on ? 1 : 0;
    if (ro) {
        ro->ifirst = geti(bp, "ifirst", 0, 1);
        ro->ilast = geti(bp, "ilast", 0, 0);
        ro->restart_flag = getb(bp, "RestartFlag", false) ? 1 : 0;
        ro->backup_freq = geti(bp, "BackupFreq", 0, 0);
        ro->cmd_lfile_freq = geti(bp, "Cmd_LFile_Freq", 0, 1);
        auto gs = [&](const char* n) {
            auto it = bp.find(lower(n));
            return (it == bp.end() || it->second.empty()) ? std::string() : to_s(it->second[0]);
        };
        std::snprintf(ro->run_name, sizeof(ro->run_name), "%s", gs("RunName").c_str());
        std::snprintf(ro->res_dir, sizeof(ro->res_dir), "%s", gs("Res_Dir").c_str());
        std::snprintf(ro->restart_dir, sizeof(ro->restart_dir), "%s", gs("RestartDir").c_str());
    }
    // derived values (src/m_Parameters.f90:144-157)
    if (P.nxc % 2 != 0 || P.nzc % 2 != 0) { why = "mod(nxc,2)/=0 || mod(nzc,2)/=0 WRONG"; return PARATC_ERR_BAD_ARG; }
    if (P.flow_type == PARATC_FT_CH && P.nyc % 2 != 0) { why = "mod(nyc,2)/=0 For channel geomotry. WRONG"; return PARATC_ERR_BAD_ARG; }
    if (P.ischeme < 1 || P.ischeme > 3) { why = "Time scheme WRONG"; return PARATC_ERR_BAD_ARG; }
    if (use_crf) {
        for (int q = 0; q < 6; q++) P.ux_bc[q] = P.ux_bc[q] - P.ucrf;
    } else {
        P.ucrf = 0.0;
    }
    if (scalar_on) {
        if (read_group(text, "ScalarFlowOptions", so) != PARATC_OK) { why = "&ScalarFlowOptions missing"; return PARATC_ERR_BAD_ARG; }
        const double sc = getd(so, "SchmidtNumber", 0, 1.0);
        P.scalar_init_value = getd(so, "Scalar_InitValue", 0, 0.0);
        const double geff = getd(so, "GravityEff", 0, 0.0);
        const double fvel = getd(so, "FallingVel", 0, 0.0);
        double gd[3];
        for (int q = 0; q < 3; q++) gd[q] = getd(so, "GravityDir", q, 0.0);
        for (int q = 0; q < 2; q++) P.scalar_bc_option[q] = geti(so, "ScalarBcOption", q, -2);
        for (int q = 0; q < 4; q++) P.scalar_bc_values[q] = getd(so, "ScalarBcValues", q, 0.0);
        // src/m_Parameters.f90:177-186
        const double rt = std::sqrt(gd[0] * gd[0] + gd[1] * gd[1] + gd[2] * gd[2]);
        if (rt > 1.0e-10) { for (int q = 0; q < 3; q++) gd[q] = gd[q] / rt; }
        else { gd[0] = 0.0; gd[1] = -1.0; gd[2] = 0.0; }
        P.sdiff = P.xnu / sc;
        for (int q = 0; q < 3; q++) { P.gravity_eff_vec[q] = gd[q] * geff; P.falling_vel_vec[q] = gd[q] * fvel; }
        P.falling_vel_vec[0] = P.falling_vel_vec[0] + P.ucrf;
    }
    if (yp) {
        if (read_group(text, "MeshSection", ms) != PARATC_OK) { why = "&MeshSection missing"; return PARATC_ERR_BAD_ARG; }
        if (read_group(text, "MeshOptions", mo) != PARATC_OK) { why = "&MeshOptions missing"; return PARATC_ERR_BAD_ARG; }
        const int ns = geti(ms, "nSection", 0, -1);
        if (ns < 1) { why = "nSection Wrong !!!"; return PARATC_ERR_BAD_ARG; }
        std::vector<double> sl(ns), cs(ns);
        std::vector<int32_t> ny(ns), st(ns), so2(ns);
        int sum = 0;
        for (int s = 0; s < ns; s++) {
            sl[s] = getd(mo, "SectionLength", s, -1.0);
            cs[s] = getd(mo, "SectioncStret", s, -1.0);
            ny[s] = geti(mo, "nycSection", s, 0);
            st[s] = geti(mo, "StretType", s, -1);
            so2[s] = geti(mo, "StretOption", s, -1);
            sum += ny[s];
        }
        if (sum != P.nyc) { why = "nycSection Wrong 2 !!!"; return PARATC_ERR_BAD_ARG; }
        yp->assign(P.nyc + 1, 0.0);
        int rc = mesh_ycoord(ns, sl.data(), cs.data(), ny.data(), st.data(), so2.data(), P.yly, yp->data());
        if (rc != PARATC_OK) { why = "MeshOptions out of range"; return rc; }
    }
    return PARATC_OK;
}

}  // namespace ptc

extern "C" int paratc_mesh_ycoord(int nsection, const double* section_length, const double* section_cstret,
                                  const int32_t* nyc_section, const int32_t* stret_type, const int32_t* stret_option,
                                  double yly, double* yp_out) {
    return ptc::mesh_ycoord(nsection, section_length, section_cstret, nyc_section, stret_type, stret_option, yly, yp_out);
}

extern "C" int paratc_params_from_namelist(const char* path, int scalar_on, paratc_params* out, double* yp_out,
                                           int nyp_cap) {
    if (!path || !out) return PARATC_ERR_BAD_ARG;
    std::string why;
    std::vector<double> yp;
    int rc = ptc::parse_namelist(path, scalar_on, *out, yp_out ? &yp : nullptr, nullptr, why);
    if (rc != PARATC_OK) {
        std::fprintf(stderr, "paratc_params_from_namelist: %s\n", why.c_str());
        return rc;
    }
    if (yp_out) {
        if ((int)yp.size() > nyp_cap) return PARATC_ERR_BAD_ARG;
        std::copy(yp.begin(), yp.end(), yp_out);
    }
    return PARATC_OK;
}

extern "C" int paratc_run_options_from_namelist(const char* path, paratc_run_options* out) {
    if (!path || !out) return PARATC_ERR_BAD_ARG;
    paratc_params p;
    std::string why;
    std::memset(out, 0, sizeof(*out));
    ptc::RunOptions ro;
    int rc = ptc::parse_namelist(path, 0, p, nullptr, &ro, why);
    if (rc != PARATC_OK) return rc;
    out->ifirst = ro.ifirst;
    out->ilast = ro.ilast;
    out->restart_flag = ro.restart_flag;
    out->backup_freq = ro.backup_freq;
    out->cmd_lfile_freq = ro.cmd_lfile_freq;
    std::snprintf(out->run_name, sizeof(out->run_name), "%s", ro.run_name);
    std::snprintf(out->res_dir, sizeof(out->res_dir), "%s", ro.res_dir);
    std::snprintf(out->restart_dir, sizeof(out->restart_dir), "%s", ro.restart_dir);
    return PARATC_OK;
}

// ---------------------------------------------------------------------------
// output options: &IO_Options and &SaveScalarOption (InitVisu,
// src/m_IOAndVisu.f90:29-53), &SpectraOptions and &Spectra2DOpt
// (InitStatVar, src/m_FlowCase.f90:127-235) and the output cadences of
// &BasicParam, with the checks those routines make
// ---------------------------------------------------------------------------
extern "C" int paratc_io_options_from_namelist(const char* path, int scalar_on, paratc_io_options* out) {
    if (!path || !out) return PARATC_ERR_BAD_ARG;
    std::memset(out, 0, sizeof(*out));
    std::ifstream in(path);
    if (!in) { std::fprintf(stderr, "paratc_io_options_from_namelist: Cannot open file: %s\n", path); return PARATC_ERR_IO; }
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string text = ss.str();
    using Group = std::map<std::string, std::vector<std::string>>;
    Group bp, io, sso, sp, s2;
    auto fail = [&](const char* why) {
        std::fprintf(stderr, "paratc_io_options_from_namelist: %s\n", why);
        return PARATC_ERR_BAD_ARG;
    };
    if (ptc::read_group(text, "BasicParam", bp) != PARATC_OK) return fail("&BasicParam missing or malformed");
    if (ptc::read_group(text, "IO_Options", io) != PARATC_OK) return fail("&IO_Options missing or malformed");
    if (ptc::read_group(text, "SpectraOptions", sp) != PARATC_OK) return fail("&SpectraOptions missing or malformed");
    if (scalar_on && ptc::read_group(text, "SaveScalarOption", sso) != PARATC_OK)
        return fail("&SaveScalarOption missing or malformed");
    auto geti = [&](Group& g, const char* n, int idx, int dflt) {
        auto it = g.find(ptc::lower(n));
        if (it == g.end() || (int)it->second.size() <= idx) return dflt;
        return (int)std::lround(ptc::to_d(it->second[idx]));
    };
    auto getb = [&](Group& g, const char* n, bool dflt) {
        auto it = g.find(ptc::lower(n));
        if (it == g.end() || it->second.empty()) return dflt;
        return ptc::to_b(it->second[0]);
    };
    out->ivstats = geti(bp, "ivstats", 0, 1);
    out->save_stat = geti(bp, "SaveStat", 0, 1);
    out->save_visu = geti(bp, "SaveVisu", 0, 1);
    out->iskip = geti(io, "iskip", 0, 1);
    out->jskip = geti(io, "jskip", 0, 1);
    out->kskip = geti(io, "kskip", 0, 1);
    out->xdmf_set_type = geti(io, "XDMF_SET_TYPE", 0, 0);
    const char* flags[PARATC_VISU_NQ] = {"save_ux", "save_uy", "save_uz", "save_pr", "save_wx", "save_wy",
                                         "save_wz", "save_wMag", "save_Q_vor", "save_lamda2", nullptr};
    for (int q = 0; q < PARATC_VISU_NQ; q++) {
        const bool on = (q == PARATC_VISU_SCALAR) ? (scalar_on && getb(sso, "save_scalar", false)) : getb(io, flags[q], false);
        if (on) out->save_mask |= 1 << q;
    }
    out->write_hist_old = getb(io, "WriteHistOld", false) ? 1 : 0;
    out->read_hist_old = getb(io, "ReadHistOld", false) ? 1 : 0;
    out->clc_spectra1d = getb(sp, "clcSpectra1D", false) ? 1 : 0;
    out->iv_spec = geti(sp, "ivSpec", 0, 1);
    out->j_for_lcs = geti(sp, "jForLCS", 0, 1);
    out->clc_spectra2d = getb(sp, "clcSpectra2D", false) ? 1 : 0;
    out->ny_spec2d = geti(sp, "nySpec2D", 0, 0);
    if (out->ivstats < 1 || out->save_stat < 1 || out->save_visu < 1 || out->iskip < 1 || out->jskip < 1 || out->kskip < 1)
        return fail("ivstats, SaveStat, SaveVisu and the skips must be >= 1");
    if (out->save_stat % out->ivstats != 0) return fail("ivstats wrong !!!");
    if (out->clc_spectra1d && (out->iv_spec < 1 || out->save_stat % out->iv_spec != 0 || out->iv_spec % out->ivstats != 0))
        return fail("ivSpec wrong !!!");
    if (out->ny_spec2d < 1) out->clc_spectra2d = 0;
    if (out->clc_spectra2d) {
        if (out->ny_spec2d > PARATC_MAX_SPEC2D) return fail("nySpec2D above PARATC_MAX_SPEC2D");
        if (ptc::read_group(text, "Spectra2DOpt", s2) != PARATC_OK) return fail("&Spectra2DOpt missing or malformed");
        for (int q = 0; q < out->ny_spec2d; q++) out->iy_spec2d[q] = geti(s2, "iySpec2D", q, 0);
    }
    return PARATC_OK;
}

// Fortran's Ew.d edit descriptor for w = d + 7 (the coordinates of the XDMF
// index are written with E14.7): right-justified [-]0.ddddddd E+ee
static std::string fortran_e(double v, int w, int d) {
    char m[64];
    std::snprintf(m, sizeof(m), "%.*e", d - 1, v);  // d significant digits: x.xxxxxxe+yy
    std::string s(m);
    const bool neg = s[0] == '-';
    if (neg) s = s.substr(1);
    const size_t epos = s.find('e');
    std::string digits = s.substr(0, 1) + s.substr(2, epos - 2);
    int ex = std::atoi(s.c_str() + epos + 1) + 1;
    if (v == 0.0) ex = 0;
    char e[16];
    std::snprintf(e, sizeof(e), "E%c%02d", ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    std::string r = std::string(neg ? "-" : "") + "0." + digits + e;
    if ((int)r.size() < w) r = std::string(w - r.size(), ' ') + r;
    return r;
}

extern "C" int paratc_write_xdmf(const paratc_params* prm, const double* yp, const char* res_dir, const char* run_name,
                                 int ifirst, int ilast, int save_visu, int save_mask, int xdmf_set_type, int single) {
    if (!prm || !yp || !res_dir || !run_name || save_visu < 1) return PARATC_ERR_BAD_ARG;
    const int nxc = prm->nxc, nyc = prm->nyc, nzc = prm->nzc;
    const int iprec = single ? 4 : 8;
    const double dx = prm->xlx / (double)nxc, dz = prm->zlz / (double)nzc, half = 0.5;
    const std::string path = std::string(res_dir) + "VisuFor" + run_name + ".xmf";
    FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) { std::fprintf(stderr, "paratc_write_xdmf: Cannot open file: %s\n", path.c_str()); return PARATC_ERR_IO; }
    const char* set_str = xdmf_set_type == 0 ? "\" Center=\"Cell\">" : "\" Center=\"Node\">";
    const int nxo = xdmf_set_type == 0 ? nxc + 1 : nxc, nyo = xdmf_set_type == 0 ? nyc + 1 : nyc;
    const int nzo = xdmf_set_type == 0 ? nzc + 1 : nzc;
    std::fprintf(fp, "<?xml version=\"1.0\" ?>\n");
    std::fprintf(fp, "<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n");
    std::fprintf(fp, "<Xdmf xmlns:xi=\"http://www.w3.org/2001/XInclude\" Version=\"2.0\">\n");
    std::fprintf(fp, "<Domain>\n");
    std::fprintf(fp, "    <Topology name=\"TOPO\" TopologyType=\"3DRectMesh\" Dimensions=\"%5d%5d%5d\"/>\n", nzo, nyo, nxo);
    std::fprintf(fp, "    <Geometry name=\"GEO\" GeometryType=\"VXVYVZ\">\n");
    auto axis = [&](int n, auto coord) {
        std::fprintf(fp, "        <DataItem Format=\"XML\" DataType=\"Float\" Precision=\"%1d\" Endian=\"Native\" Dimensions=\"%5d\">\n",
                     iprec, n);
        std::fprintf(fp, "        ");
        for (int i = 1; i <= n; i++) std::fprintf(fp, "%s", fortran_e(coord(i), 14, 7).c_str());
        std::fprintf(fp, " \n");
        std::fprintf(fp, "        </DataItem>\n");
    };
    axis(nxo, [&](int i) { return xdmf_set_type == 0 ? (double)(i - 1) * dx : (double)(i - 1) * dx + dx * half; });
    axis(nyo, [&](int j) { return xdmf_set_type == 0 ? yp[j - 1] : half * (yp[j - 1] + yp[j]); });
    axis(nzo, [&](int k) { return xdmf_set_type == 0 ? (double)(k - 1) * dz : (double)(k - 1) * dz + dz * half; });
    std::fprintf(fp, "    </Geometry>\n");
    const int nflds = (ilast - ifirst + 1) / save_visu + 1;
    std::fprintf(fp, "    <Grid Name=\"TimeSeries\" GridType=\"Collection\" CollectionType=\"Temporal\">\n");
    std::fprintf(fp, "        <Time TimeType=\"List\">\n");
    std::fprintf(fp, "        <DataItem Format=\"XML\" NumberType=\"Int\" Dimensions=\"%6d\">\n", nflds);
    std::fprintf(fp, "        ");
    for (int f = ifirst - 1; f <= ilast; f += save_visu) std::fprintf(fp, "%10d", f);
    std::fprintf(fp, "        </DataItem>\n");
    std::fprintf(fp, " \n");
    std::fprintf(fp, "       </Time>\n");
    // the order of InitVisu's Write_XDMF_One calls
    const int order[PARATC_VISU_NQ] = {PARATC_VISU_UX, PARATC_VISU_UY, PARATC_VISU_UZ, PARATC_VISU_PR,
                                       PARATC_VISU_WX, PARATC_VISU_WY, PARATC_VISU_WZ, PARATC_VISU_WMAG,
                                       PARATC_VISU_Q, PARATC_VISU_LAMDA2, PARATC_VISU_SCALAR};
    for (int f = ifirst - 1; f <= ilast; f += save_visu) {
        std::fprintf(fp, "        <Grid Name=\"T%010d\" GridType=\"Uniform\">\n", f);
        std::fprintf(fp, "            <Topology Reference=\"/Xdmf/Domain/Topology[1]\"/>\n");
        std::fprintf(fp, "            <Geometry Reference=\"/Xdmf/Domain/Geometry[1]\"/>\n");
        for (int a = 0; a < PARATC_VISU_NQ; a++) {
            const int q = order[a];
            if (!(save_mask & (1 << q)) || (q == PARATC_VISU_SCALAR && !prm->scalar_on)) continue;
            const char* name = paratc_visu_name(q);
            std::fprintf(fp, "            <Attribute Name=\"%s%s\n", name, set_str);
            std::fprintf(fp, "                <DataItem Format=\"Binary\" DataType=\"Float\" Precision=\"%1d\" Endian=\"Native\" Dimensions=\"%5d%5d%5d\">\n",
                         iprec, nzc, nyc, nxc);
            std::fprintf(fp, "                    VisuFor%s_%s_%010d\n", run_name, name, f);
            std::fprintf(fp, "                </DataItem>\n");
            std::fprintf(fp, "            </Attribute>\n");
        }
        std::fprintf(fp, "        </Grid>\n");
    }
    std::fprintf(fp, "    </Grid>\n");
    std::fprintf(fp, "</Domain>\n");
    std::fprintf(fp, "</Xdmf>\n");
    return std::fclose(fp) == 0 ? PARATC_OK : PARATC_ERR_IO;
}
