// Plane-wave basis set-up (host).  See pw_basis.h for the reference functions mirrored.
#include "pw_basis.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>

namespace b200 {
namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;

// 3x3 helpers on row-major arrays.  The determinant is expanded in ModuleBase::Matrix3::Det's order
// (module_base/matrix3.cpp:29-37) and a zero determinant replaced by 1 as Matrix3::Inverse does (:44-59), so
// that G, kvec_c, tpiba and omega carry the reference's bits (a wavefunction file is checked against them
// exactly, read_wfc_pw.cpp:121-160).
double det3(const double* a) {
    return a[0] * a[4] * a[8] - a[0] * a[7] * a[5] + a[3] * a[7] * a[2] - a[3] * a[1] * a[8] + a[6] * a[1] * a[5] -
           a[6] * a[4] * a[2];
}
void inv3(const double* a, double* r) {
    double det = det3(a);
    if (det == 0.0) det = 1.0;
    r[0] = (a[4] * a[8] - a[5] * a[7]) / det;
    r[1] = (a[2] * a[7] - a[1] * a[8]) / det;
    r[2] = (a[1] * a[5] - a[2] * a[4]) / det;
    r[3] = (a[5] * a[6] - a[3] * a[8]) / det;
    r[4] = (a[0] * a[8] - a[2] * a[6]) / det;
    r[5] = (a[2] * a[3] - a[0] * a[5]) / det;
    r[6] = (a[3] * a[7] - a[4] * a[6]) / det;
    r[7] = (a[1] * a[6] - a[0] * a[7]) / det;
    r[8] = (a[0] * a[4] - a[1] * a[3]) / det;
}
// f . (M f) with M row-major, evaluated as (M*f) then the dot product
double quad(const double* M, double x, double y, double z) {
    const double vx = M[0] * x + M[1] * y + M[2] * z;
    const double vy = M[3] * x + M[4] * y + M[5] * z;
    const double vz = M[6] * x + M[7] * y + M[8] * z;
    return x * vx + y * vy + z * vz;
}
int smooth235(int n) {
    for (int m = n;; ++m) {
        int b = m;
        while (b % 2 == 0) b /= 2;
        while (b % 3 == 0) b /= 3;
        while (b % 5 == 0) b /= 5;
        if (b == 1) return m;
    }
}

}  // namespace

int PWBasisK::setup(double lat0_in, const double* latvec_in, double ecutwfc_in, double ecutrho_in, int nx_in,
                    int ny_in, int nz_in, int nks_in, const double* kvec_d_in) {
    if (lat0_in <= 0.0 || ecutwfc_in <= 0.0 || nks_in <= 0 || latvec_in == nullptr || kvec_d_in == nullptr) return 1;
    lat0 = lat0_in;
    std::copy(latvec_in, latvec_in + 9, latvec);
    ecutwfc = ecutwfc_in;
    ecutrho = ecutrho_in > 0.0 ? ecutrho_in : 4.0 * ecutwfc_in;
    nks = nks_in;
    kvec_d.assign(kvec_d_in, kvec_d_in + 3 * nks);
    if (std::fabs(det3(latvec)) < 1e-12) return 1;

    // PW_Basis::initgrids (pw_init.cpp:24-140)
    tpiba = kTwoPi / lat0;
    tpiba2 = tpiba * tpiba;
    omega = std::fabs(det3(latvec)) * lat0 * lat0 * lat0;
    double GT[9];
    inv3(latvec, GT);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G[i * 3 + j] = GT[j * 3 + i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += G[i * 3 + k] * GT[k * 3 + j];
            GGT[i * 3 + j] = s;
        }
    gridecut_lat = ecutrho / tpiba2;
    const bool explicit_grid = nx_in > 0 && ny_in > 0 && nz_in > 0;
    if (ecutrho_in < 0.0) {
        // the cutoff an explicit grid holds (initgrids(lat0, latvec, nx, ny, nz), pw_init.cpp:157-207): the
        // smallest |G|^2 on the shell just outside the box of half-widths (n-1)/2, less 1e-6
        if (!explicit_grid) return 1;
        const int bx = (nx_in - 1) / 2 + 1, by = (ny_in - 1) / 2 + 1, bz = (nz_in - 1) / 2 + 1;
        double m = 1e20;
        for (int igz = -bz; igz <= bz; ++igz)
            for (int igy = -by; igy <= by; ++igy)
                for (int igx = -bx; igx <= bx; ++igx) {
                    if (std::abs(igx) <= bx - 1 && std::abs(igy) <= by - 1 && std::abs(igz) <= bz - 1) continue;
                    m = std::min(m, quad(GGT, igx, igy, igz));
                }
        gridecut_lat = m - 1e-6;
        ecutrho = gridecut_lat * tpiba2;
    }
    int ibox[3];
    for (int i = 0; i < 3; ++i) {
        const double* l = latvec + 3 * i;
        ibox[i] = int(std::sqrt(gridecut_lat) * std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2])) + 1;
    }
    int n1 = 0, n2 = 0, n3 = 0;
    for (int igz = -ibox[2]; igz <= ibox[2]; ++igz)
        for (int igy = -ibox[1]; igy <= ibox[1]; ++igy)
            for (int igx = -ibox[0]; igx <= ibox[0]; ++igx) {
                if (quad(GGT, igx, igy, igz) <= gridecut_lat) {
                    n1 = std::max(n1, std::abs(igx));
                    n2 = std::max(n2, std::abs(igy));
                    n3 = std::max(n3, std::abs(igz));
                }
            }
    if (explicit_grid) {
        nx = nx_in;
        ny = ny_in;
        nz = nz_in;
    } else {
        nx = smooth235(2 * n1 + 1);
        ny = smooth235(2 * n2 + 1);
        nz = smooth235(2 * n3 + 1);
    }

    // PW_Basis_K::initparameters (pw_basis_k.cpp:53-116)
    kvec_c.assign(3 * nks, 0.0);
    double kmaxmod = 0.0;
    for (int ik = 0; ik < nks; ++ik) {
        const double* kd = &kvec_d[3 * ik];
        for (int j = 0; j < 3; ++j) kvec_c[3 * ik + j] = kd[0] * G[0 * 3 + j] + kd[1] * G[1 * 3 + j] + kd[2] * G[2 * 3 + j];
        const double* kc = &kvec_c[3 * ik];
        kmaxmod = std::max(kmaxmod, std::sqrt(kc[0] * kc[0] + kc[1] * kc[1] + kc[2] * kc[2]));
    }
    gk_ecut = ecutwfc / tpiba2;
    ggecut = std::pow(std::sqrt(gk_ecut) + kmaxmod, 2);
    if (ggecut > gridecut_lat) {
        ggecut = gridecut_lat;
        gk_ecut = std::pow(std::sqrt(ggecut) - kmaxmod, 2);
    }

    // count_pw_st + get_ig2isz_is2fftixy (pw_distributeg.cpp:44-200); sticks in ixy order
    const int fftny = ny;
    std::vector<int> st_len(size_t(nx) * ny, 0), st_bot(size_t(nx) * ny, 0);
    const int ix_end = nx / 2 + 1, iy_end = ny / 2 + 1, iz_end = nz / 2 + 1;
    for (int ix = -ix_end; ix <= ix_end; ++ix)
        for (int iy = -iy_end; iy <= iy_end; ++iy) {
            const int x = ix < 0 ? ix + nx : ix;
            const int y = iy < 0 ? iy + ny : iy;
            if (x < 0 || x >= nx || y < 0 || y >= ny) continue;
            const int index = x * fftny + y;
            int length = 0;
            for (int iz = -iz_end; iz <= iz_end; ++iz) {
                if (quad(GGT, ix, iy, iz) <= ggecut) {
                    if (length == 0) st_bot[index] = iz;
                    ++length;
                }
            }
            if (length > 0) st_len[index] = length;
        }
    is2fftixy.clear();
    ig2isz.clear();
    for (int ixy = 0; ixy < nx * ny; ++ixy) {
        if (st_len[ixy] <= 0) continue;
        const int s = int(is2fftixy.size());
        for (int iz = st_bot[ixy]; iz < st_bot[ixy] + st_len[ixy]; ++iz) {
            const int z = iz < 0 ? iz + nz : iz;
            ig2isz.push_back(s * nz + z);
        }
        is2fftixy.push_back(ixy);
    }
    nst = int(is2fftixy.size());
    npw = int(ig2isz.size());

    // Miller indices of the ggecut sphere (cal_GplusK_cartesian, pw_basis_k.cpp:291-306)
    std::vector<int> mil(size_t(npw) * 3);
    for (int ig = 0; ig < npw; ++ig) {
        const int isz = ig2isz[ig];
        int iz = isz % nz;
        const int is = isz / nz;
        int ix = is2fftixy[is] / fftny;
        int iy = is2fftixy[is] % fftny;
        if (ix >= nx / 2 + 1) ix -= nx;
        if (iy >= ny / 2 + 1) iy -= ny;
        if (iz >= nz / 2 + 1) iz -= nz;
        mil[3 * ig] = ix;
        mil[3 * ig + 1] = iy;
        mil[3 * ig + 2] = iz;
    }

    // setupIndGk (pw_basis_k.cpp:118-168)
    npwk.assign(nks, 0);
    std::vector<std::vector<int>> sel(nks);
    for (int ik = 0; ik < nks; ++ik) {
        const double* kc = &kvec_c[3 * ik];
        for (int ig = 0; ig < npw; ++ig) {
            double q[3];
            for (int j = 0; j < 3; ++j)
                q[j] = kc[j] + mil[3 * ig] * G[0 * 3 + j] + mil[3 * ig + 1] * G[1 * 3 + j] + mil[3 * ig + 2] * G[2 * 3 + j];
            if (q[0] * q[0] + q[1] * q[1] + q[2] * q[2] <= gk_ecut) sel[ik].push_back(ig);
        }
        npwk[ik] = int(sel[ik].size());
        if (npwk[ik] == 0) return 2;
    }
    npwk_max = *std::max_element(npwk.begin(), npwk.end());
    const size_t L = size_t(npwk_max);
    igl2isz_k.assign(nks * L, 0);
    ig2ixyz_k.assign(nks * L, 0);
    gk2.assign(nks * L, 0.0);
    gcar.assign(nks * L * 3, 0.0);
    for (int ik = 0; ik < nks; ++ik) {
        const double* kd = &kvec_d[3 * ik];
        for (int igl = 0; igl < npwk[ik]; ++igl) {
            const int ig = sel[ik][igl];
            const int isz = ig2isz[ig];
            igl2isz_k[ik * L + igl] = isz;
            // collect_local_pw (pw_basis_k.cpp:209-231)
            const double fx = mil[3 * ig] + kd[0], fy = mil[3 * ig + 1] + kd[1], fz = mil[3 * ig + 2] + kd[2];
            gk2[ik * L + igl] = quad(GGT, fx, fy, fz);
            for (int j = 0; j < 3; ++j)
                gcar[(ik * L + igl) * 3 + j] =
                    mil[3 * ig] * G[0 * 3 + j] + mil[3 * ig + 1] * G[1 * 3 + j] + mil[3 * ig + 2] * G[2 * 3 + j];
            // get_ig2ixyz_k (pw_basis_k.cpp:319-344)
            const int iz = isz % nz;
            const int is = isz / nz;
            const int ixy = is2fftixy[is];
            ig2ixyz_k[ik * L + igl] = iz + (ixy % ny) * nz + (ixy / ny) * ny * nz;
        }
    }
    return 0;
}

}  // namespace b200
