// The reference's restart state file (cfd_state) for an instance: write the
// level set and the velocities a REEF3D run restarts from, and read such a
// file back into an instance.
//
// File layout (cfd_state::write_result, src/cfd_state_write.cpp:34-146; read
// back by cfd_state::read, src/cfd_state_read.cpp:44-160), native byte order:
//   int count, int printcount,
//   double simtime, printtime, sedprinttime, fsfprinttime, probeprinttime,
//          stateprinttime,
//   then float blocks, each in the reference's loop order (i outermost, k
//   innermost, src/looping.h:35-37):
//   topo  ALOOP  every cell (no solid cells here)
//   u     ULOOP  i < nx - ulast, all j, k
//   v     VLOOP  j < ny - vlast
//   w     WLOOP  k < nz - wlast
//   press, phi, kin, eps, eddyv  LOOP  every cell
//   qbe   SLICELOOP4  every (i, j)
//   conc  LOOP
// A single rank without periodic faces has ulast = vlast = wlast = 1 (the
// wall face at the far end is not written, src/lexer_gridsize.cpp:66-90); on
// a 2D grid (ny == 1) that leaves no v block.  Every cell counts as fluid
// (flag4 > 0): the library holds no solid flags.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handle.h"

namespace {

int state_fail(r3d_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

// padded REEF3D index of cell (i, j, k) (src/field_base.h:32-47; 2D grids keep
// the y ghost planes)
inline size_t ridx(const r3d_grid_desc& d, int i, int j, int k) {
    return ((size_t)(i + 3) * (d.ny + 6) + (size_t)(j + 3)) * (d.nz + 6) + (size_t)(k + 3);
}

struct Extents {
    int ux, vy, wz;  // u faces in x, v faces in y, w faces in z
};

Extents extents(const r3d_grid_desc& d) { return {d.nx - 1, d.ny - 1, d.nz - 1}; }

// the seven fields of the file the library does not hold, dense
// (R3D_LAYOUT_DENSE, qbe: i + nx*j); a NULL pointer stands for zeros
enum { X_TOPO, X_PRESS, X_KIN, X_EPS, X_EDDYV, X_QBE, X_CONC, X_COUNT };

inline size_t didx(const r3d_grid_desc& d, int i, int j, int k) {
    return (size_t)i + (size_t)d.nx * ((size_t)j + (size_t)d.ny * k);
}

}  // namespace

extern "C" int r3d_write_reef3d_state(r3d_handle* h, const char* path, const r3d_state_info* info,
                                      const double* const* extra) {
    if (!h || !path || !info) return state_fail(h, R3D_EINVAL, "null argument");
    const r3d_grid_desc& d = h->desc;
    const size_t np = (size_t)(d.nx + 6) * (d.ny + 6) * (d.nz + 6);
    std::vector<double> phi(np), u(np), v(np), w(np);
    const int ids[4] = {R3D_PHI, R3D_U, R3D_V, R3D_W};
    std::vector<double>* dst[4] = {&phi, &u, &v, &w};
    for (int q = 0; q < 4; ++q)
        if (int rc = r3d_download(h, ids[q], dst[q]->data(), R3D_LAYOUT_REEF3D)) return rc;

    const Extents e = extents(d);
    const size_t ncell = (size_t)d.nx * d.ny * d.nz;
    std::vector<float> buf;
    buf.reserve(8 * ncell + (size_t)d.nx * d.ny);
    auto cells = [&](auto&& value) {
        for (int i = 0; i < d.nx; ++i)
            for (int j = 0; j < d.ny; ++j)
                for (int k = 0; k < d.nz; ++k) buf.push_back((float)value(i, j, k));
    };
    auto extra_at = [&](int which) {
        const double* a = extra ? extra[which] : nullptr;
        return [a, &d](int i, int j, int k) { return a ? a[didx(d, i, j, k)] : 0.0; };
    };
    cells(extra_at(X_TOPO));
    for (int i = 0; i < e.ux; ++i)
        for (int j = 0; j < d.ny; ++j)
            for (int k = 0; k < d.nz; ++k) buf.push_back((float)u[ridx(d, i, j, k)]);
    for (int i = 0; i < d.nx; ++i)
        for (int j = 0; j < e.vy; ++j)
            for (int k = 0; k < d.nz; ++k) buf.push_back((float)v[ridx(d, i, j, k)]);
    for (int i = 0; i < d.nx; ++i)
        for (int j = 0; j < d.ny; ++j)
            for (int k = 0; k < e.wz; ++k) buf.push_back((float)w[ridx(d, i, j, k)]);
    cells(extra_at(X_PRESS));
    cells([&](int i, int j, int k) { return phi[ridx(d, i, j, k)]; });
    cells(extra_at(X_KIN));
    cells(extra_at(X_EPS));
    cells(extra_at(X_EDDYV));
    {
        const double* qb = extra ? extra[X_QBE] : nullptr;
        for (int i = 0; i < d.nx; ++i)
            for (int j = 0; j < d.ny; ++j) buf.push_back(qb ? (float)qb[(size_t)i + (size_t)d.nx * j] : 0.0f);
    }
    cells(extra_at(X_CONC));

    FILE* f = std::fopen(path, "wb");
    if (!f) return state_fail(h, R3D_EINVAL, std::string("cannot open ") + path + " for writing");
    const int iv[2] = {info->count, info->printcount};
    const double dv[6] = {info->simtime, info->printtime, info->sedprinttime,
                          info->fsfprinttime, info->probeprinttime, info->stateprinttime};
    const bool ok = std::fwrite(iv, sizeof(int), 2, f) == 2 && std::fwrite(dv, sizeof(double), 6, f) == 6 &&
                    std::fwrite(buf.data(), sizeof(float), buf.size(), f) == buf.size();
    if (std::fclose(f) != 0 || !ok) return state_fail(h, R3D_EINVAL, std::string("write failed: ") + path);
    return R3D_OK;
}

extern "C" int r3d_read_reef3d_state(r3d_handle* h, const char* path, r3d_state_info* info, double* const* extra) {
    if (!h || !path) return state_fail(h, R3D_EINVAL, "null argument");
    const r3d_grid_desc& d = h->desc;
    const Extents e = extents(d);
    const size_t ncell = (size_t)d.nx * d.ny * d.nz;
    // seven cell blocks (topo, press, phi, kin, eps, eddyv, conc), the three
    // velocity blocks and the bed-load slice
    const size_t expect = 7 * ncell + (size_t)e.ux * d.ny * d.nz + (size_t)d.nx * e.vy * d.nz +
                          (size_t)d.nx * d.ny * e.wz + (size_t)d.nx * d.ny;
    FILE* f = std::fopen(path, "rb");
    if (!f) return state_fail(h, R3D_EINVAL, std::string("cannot open ") + path);
    int iv[2];
    double dv[6];
    std::vector<float> buf(expect);
    bool ok = std::fread(iv, sizeof(int), 2, f) == 2 && std::fread(dv, sizeof(double), 6, f) == 6 &&
              std::fread(buf.data(), sizeof(float), expect, f) == expect;
    const bool at_end = ok && std::fgetc(f) == EOF;
    std::fclose(f);
    if (!ok || !at_end)
        return state_fail(h, R3D_EINVAL, std::string(path) + ": not a state file of this grid (size mismatch)");

    // the instance's current fields keep every value the file does not
    // hold (ghost cells, the wall faces of u, v, w)
    const size_t np = (size_t)(d.nx + 6) * (d.ny + 6) * (d.nz + 6);
    std::vector<double> phi(np), u(np), v(np), w(np);
    const int ids[4] = {R3D_PHI, R3D_U, R3D_V, R3D_W};
    std::vector<double>* fld[4] = {&phi, &u, &v, &w};
    for (int q = 0; q < 4; ++q)
        if (int rc = r3d_download(h, ids[q], fld[q]->data(), R3D_LAYOUT_REEF3D)) return rc;

    size_t pos = 0;
    auto cells = [&](double* dense) {
        for (int i = 0; i < d.nx; ++i)
            for (int j = 0; j < d.ny; ++j)
                for (int k = 0; k < d.nz; ++k) {
                    const float x = buf[pos++];
                    if (dense) dense[didx(d, i, j, k)] = (double)x;
                }
    };
    auto extra_out = [&](int which) { return extra ? extra[which] : nullptr; };
    cells(extra_out(X_TOPO));
    for (int i = 0; i < e.ux; ++i)
        for (int j = 0; j < d.ny; ++j)
            for (int k = 0; k < d.nz; ++k) u[ridx(d, i, j, k)] = (double)buf[pos++];
    for (int i = 0; i < d.nx; ++i)
        for (int j = 0; j < e.vy; ++j)
            for (int k = 0; k < d.nz; ++k) v[ridx(d, i, j, k)] = (double)buf[pos++];
    for (int i = 0; i < d.nx; ++i)
        for (int j = 0; j < d.ny; ++j)
            for (int k = 0; k < e.wz; ++k) w[ridx(d, i, j, k)] = (double)buf[pos++];
    cells(extra_out(X_PRESS));
    for (int i = 0; i < d.nx; ++i)
        for (int j = 0; j < d.ny; ++j)
            for (int k = 0; k < d.nz; ++k) phi[ridx(d, i, j, k)] = (double)buf[pos++];
    cells(extra_out(X_KIN));
    cells(extra_out(X_EPS));
    cells(extra_out(X_EDDYV));
    {
        double* qb = extra_out(X_QBE);
        for (int i = 0; i < d.nx; ++i)
            for (int j = 0; j < d.ny; ++j) {
                const float x = buf[pos++];
                if (qb) qb[(size_t)i + (size_t)d.nx * j] = (double)x;
            }
    }
    cells(extra_out(X_CONC));

    for (int q = 0; q < 4; ++q)
        if (int rc = r3d_upload(h, ids[q], fld[q]->data(), R3D_LAYOUT_REEF3D)) return rc;
    // the level set's ghost cells as cfd_state::read refills them
    // (ghostcell::start4, src/cfd_state_read.cpp:183)
    if (int rc = r3d_ghost_fill(h, R3D_PHI)) return rc;
    if (info) {
        info->count = iv[0];
        info->printcount = iv[1];
        info->simtime = dv[0];
        info->printtime = dv[1];
        info->sedprinttime = dv[2];
        info->fsfprinttime = dv[3];
        info->probeprinttime = dv[4];
        info->stateprinttime = dv[5];
    }
    return R3D_OK;
}
