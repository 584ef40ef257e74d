// io.cu -- the reference's text formats on the host, over the C ABI.
//
// data_end.dat (save_data_end, LBM.cu:1506-1566, and read_data,
// LBM.cu:1597-1643), the Tecplot ASCII file (save_data_tecplot,
// LBM.cu:1427-1503) and the uz file for DMD post-processing (save_data_dmd,
// LBM.cu:1569-1594), so a driver that replaces the reference's time loop
// keeps its output and restart files.
#include <cstdio>
#include <vector>

#include "ehd.h"
#include "kernels.h"

namespace {

struct Fields {
    int nx, ny, nz;
    std::vector<double> a[9];  // rho u v w q phi ex ey ez
    size_t idx(int x, int y, int z) const { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); }
};

int fetch(ehd_ctx *c, Fields &f) {
    const ehd_params *p = ehd::ctx_params(c);
    f.nx = p->nx;
    f.ny = p->ny;
    f.nz = p->nz;
    const size_t n = (size_t)f.nx * f.ny * f.nz;
    for (auto &v : f.a) v.assign(n, 0.0);
    return ehd_get_fields(c, f.a[0].data(), f.a[1].data(), f.a[2].data(), f.a[3].data(),
                          f.a[4].data(), f.a[5].data(), f.a[6].data(), f.a[7].data(),
                          f.a[8].data());
}

// rho, q, u, v, w on both walls replaced by a linear extrapolation from the
// two planes inside (LBM.cu:1465-1478, 1531-1544)
void extrapolate_walls(Fields &f) {
    const int K[5] = {0, 4, 1, 2, 3};
    for (int y = 0; y < f.ny; ++y)
        for (int x = 0; x < f.nx; ++x)
            for (int k : K) {
                std::vector<double> &a = f.a[k];
                a[f.idx(x, y, 0)] = 2.0 * a[f.idx(x, y, 1)] - a[f.idx(x, y, 2)];
                a[f.idx(x, y, f.nz - 1)] = 2.0 * a[f.idx(x, y, f.nz - 2)] - a[f.idx(x, y, f.nz - 3)];
            }
}

}  // namespace

extern "C" int ehd_write_data_end(ehd_ctx *c, const char *path) {
    if (!c || !path) return ehd::set_error(EHD_ERR_INVALID, "NULL argument");
    Fields f;
    int r = fetch(c, f);
    if (r != EHD_OK) return r;
    extrapolate_walls(f);
    FILE *fp = std::fopen(path, "w");
    if (!fp) return ehd::set_error(EHD_ERR_IO, "cannot open the data_end file for writing");
    const double t = *ehd::ctx_time(c);
    for (int z = 0; z < f.nz; ++z)
        for (int y = 0; y < f.ny; ++y)
            for (int x = 0; x < f.nx; ++x) {
                const size_t i = f.idx(x, y, z);
                std::fprintf(fp,
                             "%10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f "
                             "%10.6f\n",
                             t, f.a[1][i], f.a[2][i], f.a[3][i], f.a[0][i], f.a[4][i], f.a[5][i],
                             f.a[6][i], f.a[7][i], f.a[8][i]);
            }
    if (std::fclose(fp) != 0) return ehd::set_error(EHD_ERR_IO, "writing the data_end file failed");
    return EHD_OK;
}

// save_data_dmd (LBM.cu:1569-1594): "t uz" per node, %10.6f, uz extrapolated
// onto both walls from the two planes inside
extern "C" int ehd_write_dmd(ehd_ctx *c, const char *path) {
    if (!c || !path) return ehd::set_error(EHD_ERR_INVALID, "NULL argument");
    const ehd_params *p = ehd::ctx_params(c);
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    if (nz < 3) return ehd::set_error(EHD_ERR_INVALID, "the DMD file needs nz >= 3");
    const size_t nxy = (size_t)nx * ny;
    std::vector<double> w(nxy * nz);
    int r = ehd_get_fields(c, nullptr, nullptr, nullptr, w.data(), nullptr, nullptr, nullptr,
                           nullptr, nullptr);
    if (r != EHD_OK) return r;
    for (size_t i = 0; i < nxy; ++i) {
        w[i] = 2.0 * w[nxy + i] - w[2 * nxy + i];
        w[(nz - 1) * nxy + i] = 2.0 * w[(nz - 2) * nxy + i] - w[(nz - 3) * nxy + i];
    }
    FILE *fp = std::fopen(path, "w");
    if (!fp) return ehd::set_error(EHD_ERR_IO, "cannot open the DMD file for writing");
    const double t = *ehd::ctx_time(c);
    for (size_t i = 0; i < w.size(); ++i) std::fprintf(fp, "%10.6f %10.6f\n", t, w[i]);
    if (std::fclose(fp) != 0) return ehd::set_error(EHD_ERR_IO, "writing the DMD file failed");
    return EHD_OK;
}

extern "C" int ehd_read_data_end(ehd_ctx *c, const char *path) {
    if (!c || !path) return ehd::set_error(EHD_ERR_INVALID, "NULL argument");
    const ehd_params *p = ehd::ctx_params(c);
    Fields f;
    f.nx = p->nx;
    f.ny = p->ny;
    f.nz = p->nz;
    const size_t n = (size_t)f.nx * f.ny * f.nz;
    for (auto &v : f.a) v.assign(n, 0.0);
    FILE *fp = std::fopen(path, "r");
    if (!fp) return ehd::set_error(EHD_ERR_IO, "cannot open the data_end file");
    double t = 0.0;
    for (size_t i = 0; i < n; ++i) {
        // time, ux, uy, uz, rho, charge, phi, Ex, Ey, Ez (LBM.cu:1614-1616)
        if (std::fscanf(fp, "%lf %lf %lf %lf %lf %lf %lf %lf %lf %lf", &t, &f.a[1][i],
                        &f.a[2][i], &f.a[3][i], &f.a[0][i], &f.a[4][i], &f.a[5][i], &f.a[6][i],
                        &f.a[7][i], &f.a[8][i]) != 10) {
            std::fclose(fp);
            return ehd::set_error(EHD_ERR_IO, "data_end file is short or malformed");
        }
    }
    std::fclose(fp);
    int r = ehd_set_fields(c, f.a[0].data(), f.a[1].data(), f.a[2].data(), f.a[3].data(),
                           f.a[4].data(), f.a[5].data(), f.a[6].data(), f.a[7].data(),
                           f.a[8].data());
    if (r != EHD_OK) return r;
    *ehd::ctx_time(c) = t;
    return EHD_OK;
}

extern "C" int ehd_write_tecplot(ehd_ctx *c, const char *path, int first) {
    if (!c || !path) return ehd::set_error(EHD_ERR_INVALID, "NULL argument");
    Fields f;
    int r = fetch(c, f);
    if (r != EHD_OK) return r;
    extrapolate_walls(f);
    const ehd_params *p = ehd::ctx_params(c);
    FILE *fp = std::fopen(path, first ? "w" : "a");
    if (!fp) return ehd::set_error(EHD_ERR_IO, "cannot open the Tecplot file");
    if (first)
        std::fprintf(fp, "%s\n",
                     "VARIABLES=\"x\",\"y\",\"z\",\"u\",\"v\",\"w\",\"p\",\"charge\",\"phi\","
                     "\"Ex\",\"Ey\",\"Ez\"");
    std::fprintf(fp, "\n");
    std::fprintf(fp, "ZONE T=\"t=%g\", F=POINT, I = %d, J = %d, K = %d\n", *ehd::ctx_time(c),
                 f.nx, f.ny, f.nz);
    for (int z = 0; z < f.nz; ++z)
        for (int y = 0; y < f.ny; ++y)
            for (int x = 0; x < f.nx; ++x) {
                const size_t i = f.idx(x, y, z);
                std::fprintf(fp, "%g %g %g %g %g %g %g %g %10.6f %10.6f %10.6f %10.6f\n",
                             p->dx * x, p->dy * y, p->dz * z, f.a[1][i], f.a[2][i], f.a[3][i],
                             f.a[0][i], f.a[4][i], f.a[5][i], f.a[6][i], f.a[7][i], f.a[8][i]);
            }
    if (std::fclose(fp) != 0) return ehd::set_error(EHD_ERR_IO, "writing the Tecplot file failed");
    return EHD_OK;
}
