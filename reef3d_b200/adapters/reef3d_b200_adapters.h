// REEF3D-side adapter classes for the B200 level-set library.
//
// These are the classes a REEF3D maintainer adds to REEF3D's source tree to
// run the level-set path on the GPU through include/reef3d_b200.h.  Each one
// derives from the REEF3D interface it replaces and keeps that interface's
// contract; the file compiles only inside a REEF3D build (it includes
// REEF3D's headers) and links against libreef3d_b200.so:
//
//   levelset_RK3_gpu : freesurface   replaces levelset_RK3 (src/levelset_RK3.h)
//   levelset_RK3_domain : freesurface  the same over z slabs on several GPUs
//   weno_hj_gpu      : convection    replaces weno_hj_df_nug (src/weno_hj_df_nug.h)
//   reinidisc_gpu    : reinidisc     replaces reinidisc_f / reinidisc_fsf
//   reini_RK3_gpu    : reini         replaces reini_RK3 (src/reini_RK3.h)
//
// Fields cross the boundary in REEF3D's own layout (field_base::V,
// R3D_LAYOUT_REEF3D).  Errors: the library returns a status, the adapters
// print r3d_last_error and stop the run with exit(1), as REEF3D does on a
// fatal error.
#pragma once

#include <cstdlib>
#include <iostream>
#include <vector>

#include "convection.h"
#include "fdm.h"
#include "field.h"
#include "freesurface.h"
#include "ghostcell.h"
#include "lexer.h"
#include "reef3d_b200.h"
#include "reini.h"
#include "reinidisc.h"
// the wave generator: its relaxation weights and targets are private to
// iowave; the adapter reads them as a friend -- a maintainer adds
//   namespace r3d_adapter { struct WaveState; }   (before class iowave)
//   friend struct r3d_adapter::WaveState;          (inside it)
// to src/iowave.h
#include "iowave.h"

namespace r3d_adapter {

inline void check(r3d_handle* h, int rc) {
    if (rc != R3D_OK) {
        std::cout << "reef3d_b200: " << r3d_last_error(h) << std::endl;
        std::exit(1);
    }
}

// One device instance for the grid and control flags of a REEF3D run: the
// node coordinates DIVEMesh wrote (p->XN etc., node indices -5..n+5) and the
// level-set flags of the control file.  precision: R3D_FP64 (the reference's
// arithmetic) or R3D_FP32 (the FP32 form).
inline r3d_grid_desc grid_desc(const lexer* p, int precision) {
    r3d_grid_desc d{};
    d.nx = p->knox;
    d.ny = p->knoy;
    d.nz = p->knoz;
    d.xn = p->XN;
    d.yn = p->YN;
    d.zn = p->ZN;
    d.f43 = p->F43;
    d.f44 = p->F44;
    d.f45 = p->F45;
    d.f49 = p->F49;
    d.n47 = p->N47;
    d.precision = precision;
    d.f46 = p->F46;
    d.f47 = p->F47;
    return d;
}

inline r3d_handle* make_handle(lexer* p, int precision) {
    const r3d_grid_desc d = grid_desc(p, precision);
    r3d_handle* h = nullptr;
    check(nullptr, r3d_create(&d, &h));
    return h;
}

inline void check_domain(r3d_domain* d, int rc) {
    if (rc != R3D_OK) {
        std::cout << "reef3d_b200: " << (d ? r3d_domain_last_error(d) : r3d_last_error(nullptr)) << std::endl;
        std::exit(1);
    }
}

// Interior cell (i,j,k) of a REEF3D field array (src/field_base.h:47).
inline long ijk(const lexer* p, int i, int j, int k) {
    return (long)(i - p->imin) * p->jmax * p->kmax + (long)(j - p->jmin) * p->kmax + (k - p->kmin);
}

// Copies the cells the device owns -- the interior, plus the face ghost
// layers when `faces` (a 2D grid has no y ghost planes on the device) --
// from a full REEF3D-layout array into a field; every other cell of the
// field keeps its value, as it would under the reference object.
inline void copy_owned(const lexer* p, const std::vector<double>& src, field& f, bool faces) {
    const int nx = p->knox, ny = p->knoy, nz = p->knoz;
    const int gy = ny == 1 ? 0 : 3;
    for (int i = -3; i < nx + 3; ++i)
        for (int j = -gy; j < ny + gy; ++j)
            for (int k = -3; k < nz + 3; ++k) {
                const int outside = (i < 0 || i >= nx) + (j < 0 || j >= ny) + (k < 0 || k >= nz);
                if (outside > (faces ? 1 : 0)) continue;
                const long c = ijk(p, i, j, k);
                f.V[c] = src[c];
            }
}

inline void download_owned(r3d_handle* h, int id, const lexer* p, field& f, bool faces,
                           std::vector<double>& buf) {
    buf.resize((size_t)p->imax * p->jmax * p->kmax);
    check(h, r3d_download(h, id, buf.data(), R3D_LAYOUT_REEF3D));
    copy_owned(p, buf, f, faces);
}

// Ghost-cell type of the level set for ghostcell::start4, chosen from F50
// as levelset_RK3 and reini_RK3 choose it (src/levelset_RK3.cpp:50-60,
// src/reini_RK3.cpp:35-62).
inline int gcval_phi(const lexer* p) { return 50 + (p->F50 >= 1 && p->F50 <= 4 ? p->F50 : 0); }
inline int gcval_iniphi(const lexer* p) {
    int g = 50;
    if ((p->F61 > 1.0e-20 || p->F60 > 1.0e-20) && p->F50 == 1) g = 51;
    if ((p->F62 > 1.0e-20 || p->F60 > 1.0e-20) && p->F50 == 2) g = 52;
    if (((p->F61 > 1.0e-20 && p->F62 > 1.0e-20) || p->F60 > 1.0e-20) && p->F50 == 3) g = 53;
    return g;
}

// Inflow / outflow faces of a run whose flow object is ioflow_f (B60 >= 1,
// src/driver_logic_cfd.cpp:509-510) for the level-set gcv `gcv`: the
// device models an inflow boundary on the whole x-min face and an outflow
// boundary on the whole x-max face, with ioflow_f's hooks
// (r3d_set_ioflow).  false: closed box (ioflow_v, or gcv 50, whose ghost
// label is 4 on every face).  iowave and the gravity flow (B90, B180) have
// relaxation zones and hooks of their own, not on the device.
inline bool ioflow_desc(const lexer* p, int gcv, r3d_ioflow_desc* d, bool* waves) {
    *waves = p->B90 >= 1;
    if (p->B180 == 1 || p->B191 == 1 || p->B192 == 1) {
        std::cout << "reef3d_b200: ioflow_gravity level-set hooks are not on the device" << std::endl;
        std::exit(1);
    }
    // the wave generator's level-set hooks on the device: relaxation-zone
    // generation (B98 = 2) and beach (B99 = 2) in phi_relax, the face copies
    // of fsfrkin / fsfrkout; faces without flow-file input (I230 = 0).  The
    // Dirichlet and active wave makers (B98 = 3, 4) and active beaches (B99 =
    // 3..5) set the velocities at the faces (iowave::inflow,
    // src/iowave_inflow.cpp:30-52), which reach the device with the host's
    // u, v, w; of the level set they only read phi, and phi_relax leaves it
    // alone for them (src/iowave_relax.cpp:346-378)
    if (*waves && (p->B98 < 0 || p->B98 > 4 || p->B99 < 0 || p->B99 > 5 || p->I230 > 0)) {
        std::cout << "reef3d_b200: iowave's level-set hooks run on the device for B98 = 0..4, B99 = 0..5 "
                     "without flow-file input" << std::endl;
        std::exit(1);
    }
    if ((p->B60 < 1 && !*waves) || gcv == 50) return false;
    const int face = p->knoy * p->knoz;
    for (int n = 0; n < p->gcin_count; ++n)
        if (p->gcin[n][3] != 1 || p->gcin_count != face) {
            std::cout << "reef3d_b200: the device's inflow boundary is the whole x-min face" << std::endl;
            std::exit(1);
        }
    for (int n = 0; n < p->gcout_count; ++n)
        if (p->gcout[n][3] != 4 || p->gcout_count != face) {
            std::cout << "reef3d_b200: the device's outflow boundary is the whole x-max face" << std::endl;
            std::exit(1);
        }
    *d = r3d_ioflow_desc{};
    d->inflow = p->gcin_count > 0 ? 1 : 0;
    d->outflow = p->gcout_count > 0 ? 1 : 0;
    if (!d->inflow && !d->outflow) return false;
    d->f50 = gcv - 50;
    d->b77 = p->B77;
    d->f56 = p->F56;
    d->f60 = p->F60;
    d->f61 = p->F61;
    d->f62 = p->F62;
    d->f64 = p->F64;
    d->qi = p->Qi;
    d->qo = p->Qo;
    return true;
}

// Direct-forcing convection stencils (X45 != 0, src/weno_hj_df_nug.cpp:
// 398-987): enables them on the instance (FP64 only).
inline void set_direct_forcing(r3d_handle* h, const lexer* p) {
    if (p->X45 != 0) check(h, r3d_set_direct_forcing(h, p->X45));
}

// The body field those stencils read, from the fdm: fb (X45 1), fbh5 (2, 4),
// fbh4 (3, 6), min(solid, topo) (5: both > 0 exactly when the minimum is).
inline void upload_body(r3d_handle* h, const lexer* p, fdm* a, std::vector<double>& buf) {
    if (p->X45 == 0) return;
    const double* src = nullptr;
    if (p->X45 == 1) src = a->fb.V;
    if (p->X45 == 2 || p->X45 == 4) src = a->fbh5.V;
    if (p->X45 == 3 || p->X45 == 6) src = a->fbh4.V;
    if (p->X45 == 5) {
        const long n = (long)p->imax * p->jmax * p->kmax;
        buf.resize((size_t)n);
        for (long q = 0; q < n; ++q) buf[q] = a->solid.V[q] < a->topo.V[q] ? a->solid.V[q] : a->topo.V[q];
        src = buf.data();
    }
    check(h, r3d_upload(h, R3D_BODY, src, R3D_LAYOUT_REEF3D));
}

// The solid forcing of the level set (X48 = 1): the direct-forcing boundary
// list gcdf4 (src/gcdf_update.cpp), handed to the device when it changed
// (moving bodies rebuild it).
struct SolidForcingState {
    std::vector<int> last;
    bool on = false;
    void sync(r3d_handle* h, const lexer* p) {
        std::vector<int> cells;
        if (p->X48 == 1)
            for (int n = 0; n < p->gcdf4_count; ++n)
                for (int c = 0; c < 4; ++c) cells.push_back(p->gcdf4[n][c]);
        if (cells != last || on != (p->X48 == 1)) {
            check(h, r3d_set_solid_forcing(h, (int)(cells.size() / 4), cells.data()));
            last = cells;
            on = p->X48 == 1;
        }
    }
};

inline bool same_ioflow(const r3d_ioflow_desc& a, const r3d_ioflow_desc& b) {
    return a.inflow == b.inflow && a.outflow == b.outflow && a.f50 == b.f50 && a.b77 == b.b77 && a.f56 == b.f56 &&
           a.f60 == b.f60 && a.f61 == b.f61 && a.f62 == b.f62 && a.f64 == b.f64 && a.qi == b.qi && a.qo == b.qo;
}

// Brings the instance's inflow / outflow configuration and step count
// (lexer::count, read by the outflow ramp and picard_lsm) up to date.
struct IoflowState {
    bool on = false;
    r3d_ioflow_desc last{};
    void sync(r3d_handle* h, const lexer* p, int gcv) {
        r3d_ioflow_desc d{};
        bool waves = false;
        const bool now = ioflow_desc(p, gcv, &d, &waves);
        if (now != on || (now && !same_ioflow(d, last))) {
            if (now && waves) check(h, r3d_set_ioflow_waves(h, &d));
            else check(h, r3d_set_ioflow(h, now ? &d : nullptr));
            on = now;
            last = d;
        }
        check(h, r3d_set_step_count(h, p->count));
    }
    // the same for a slab domain: the faces on every slab, the step count
    // on every slab (the grid's levels are taken from slab 0's)
    void sync(r3d_domain* dm, const lexer* p, int gcv) {
        r3d_ioflow_desc d{};
        bool waves = false;
        const bool now = ioflow_desc(p, gcv, &d, &waves);
        if (waves) {
            std::cout << "reef3d_b200: the slab domain runs without the wave generator" << std::endl;
            std::exit(1);
        }
        if (now != on || (now && !same_ioflow(d, last))) {
            check_domain(dm, r3d_domain_set_ioflow(dm, now ? &d : nullptr));
            on = now;
            last = d;
        }
        r3d_handle* h = nullptr;
        for (int s = 0; r3d_domain_slab(dm, s, &h, nullptr, nullptr) == R3D_OK; ++s)
            check(h, r3d_set_step_count(h, p->count));
    }
};

// The wave generator's relaxation zones on the level set (iowave::phi_relax,
// src/iowave_relax.cpp:346-378, after every convection stage): the zones'
// weights relax4_wg / relax4_nb of every column inside them (distgen /
// distbeach < 1e20) go to the device once, and each step the targets lsval
// that the driver's wavegen_precalc computed for it (src/driver_loop_cfd.cpp:78)
// with the step's ramp.  Generation applies with B98 = 2 (and iowave's
// h_switch), the beach with B99 = 2.
struct WaveState {
    bool set = false;
    double phimean = 0.0;
    bool gen = false, beach = false;
    std::vector<double> wg, wb;
    void sync(r3d_handle* h, lexer* p, ioflow* pflow) {
        if (p->B90 < 1) return;
        iowave* w = dynamic_cast<iowave*>(pflow);
        if (!w) {
            std::cout << "reef3d_b200: B90 >= 1 without the iowave flow object" << std::endl;
            std::exit(1);
        }
        if (!set || phimean != p->phimean) {
            gen = p->B98 == 2 && w->h_switch == 1;
            beach = p->B99 == 2;
            const int nx = p->knox, ny = p->knoy;
            wg.assign((size_t)nx * ny, -1.0);
            wb.assign((size_t)nx * ny, -1.0);
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j) {
                    increment::i = i;
                    increment::j = j;
                    increment::k = 0;
                    if (gen && w->distgen(p) < 1.0e20) wg[(size_t)i * ny + j] = w->relax4_wg(i, j);
                    if (beach && w->distbeach(p) < 1.0e20) wb[(size_t)i * ny + j] = w->relax4_nb(i, j);
                }
            check(h, r3d_set_relaxation(h, gen ? wg.data() : nullptr, beach ? wb.data() : nullptr, p->phimean));
            phimean = p->phimean;
            set = true;
        }
        long long n = 0;
        if (gen)
            for (double x : wg) n += x >= 0.0 ? p->knoz : 0;
        if (gen || beach) check(h, r3d_set_relaxation_target(h, w->lsval, n, w->ramp(p)));
    }
};

}  // namespace r3d_adapter

// The device writes the interior and the face ghost layers of every field it
// returns; the adapters then run REEF3D's own ghostcell::start4 on the host
// copy, which also fills the edge and corner ghosts (dgcpol4) and, in a
// multi-rank run, exchanges the halo.  (The device step knows walls, the
// inflow / outflow x faces of ioflow_f, the X45 stencils and the solid
// forcing.  A REEF3D run split over several MPI ranks needs a halo exchange
// in every stage; the library has it for z slabs -- r3d_set_halo,
// r3d_halo_copy, reef3d_b200/slab.py -- but these adapters drive one
// single-subdomain instance.)

// freesurface: one level-set step on the device (three WENO5-HJ convection
// RK stages with the wall ghost fill, F44 reinitialisation pseudo-steps, the
// picard correction the control file selects, the volume integral and the
// density/viscosity update), src/levelset_RK3.cpp:103-178.  The level set
// goes up at every call unless `resident` is set, in which case it stays on
// the device after the first call (for runs where only this object writes
// a->phi); the velocities go up at every call because the momentum solver
// owns them on the host.  a->phi, a->ro, a->visc and p->volume1/2 come back.
class levelset_RK3_gpu final : public freesurface {
public:
    levelset_RK3_gpu(lexer* p, fdm*, ghostcell*, int precision = R3D_FP64, bool resident = false)
        : h(r3d_adapter::make_handle(p, precision)), resident(resident) {
        r3d_adapter::check(h, r3d_set_fluid(h, p->W1, p->W2, p->W3, p->W4));
        r3d_adapter::set_direct_forcing(h, p);
    }
    ~levelset_RK3_gpu() { r3d_destroy(h); }

    void start(fdm* a, lexer* p, convection*, solver*, ghostcell* pgc, ioflow* pflow, reini*, particle_corr*,
               field& ls) override {
        using r3d_adapter::check;
        io.sync(h, p, r3d_adapter::gcval_phi(p));
        wave.sync(h, p, pflow);
        sf.sync(h, p);
        if (!resident || first) check(h, r3d_upload(h, R3D_PHI, ls.V, R3D_LAYOUT_REEF3D));
        first = false;
        check(h, r3d_upload(h, R3D_U, a->u.V, R3D_LAYOUT_REEF3D));
        check(h, r3d_upload(h, R3D_V, a->v.V, R3D_LAYOUT_REEF3D));
        check(h, r3d_upload(h, R3D_W, a->w.V, R3D_LAYOUT_REEF3D));
        r3d_adapter::upload_body(h, p, a, buf);
        check(h, r3d_ls_step(h, p->dt));
        r3d_adapter::download_owned(h, R3D_PHI, p, ls, true, buf);
        r3d_adapter::download_owned(h, R3D_RO, p, a->ro, true, buf);
        r3d_adapter::download_owned(h, R3D_VISC, p, a->visc, true, buf);
        check(h, r3d_last_volume(h, &p->volume1, &p->volume2));
        // the reference fills the ghosts of ls in the last reinitialisation
        // stage; a picard correction after it moves the interior only
        if (p->F46 == 0) pgc->start4(p, ls, r3d_adapter::gcval_phi(p));
        pgc->start4(p, a->ro, 1);  // gcval_ro of fluid_update_fsf
        pgc->start4(p, a->visc, 1);
    }

    // levelset_RK3::update: the density/viscosity update on a->phi
    // (src/levelset_RK3.cpp:180-183).
    void update(lexer* p, fdm* a, ghostcell* pgc, field&) override {
        using r3d_adapter::check;
        check(h, r3d_upload(h, R3D_PHI, a->phi.V, R3D_LAYOUT_REEF3D));
        first = false;
        check(h, r3d_fluid_update(h, &p->volume1, &p->volume2));
        r3d_adapter::download_owned(h, R3D_RO, p, a->ro, true, buf);
        r3d_adapter::download_owned(h, R3D_VISC, p, a->visc, true, buf);
        pgc->start4(p, a->ro, 1);
        pgc->start4(p, a->visc, 1);
    }

    r3d_handle* handle() { return h; }

private:
    r3d_handle* h;
    bool resident;
    bool first = true;
    r3d_adapter::IoflowState io;
    r3d_adapter::WaveState wave;
    r3d_adapter::SolidForcingState sf;
    std::vector<double> buf;
};

// freesurface over several slabs of the grid: the grid split along z into
// nslabs slabs (r3d_domain_*; slab r on devices[r], or all on the current
// GPU), stepped as one with the halo exchange between stages -- one
// REEF3D process spreading its level set over the GPUs of a node.  The same
// contract as levelset_RK3_gpu (the picard correction F46 selects and the
// ioflow_f inflow/outflow faces included, over the whole grid), for runs
// without X45 stencils or solid forcing (the run stops on them).
class levelset_RK3_domain final : public freesurface {
public:
    levelset_RK3_domain(lexer* p, fdm*, ghostcell*, int nslabs, const int* devices = nullptr,
                        int precision = R3D_FP64) {
        if (p->X45 != 0 || p->X48 == 1) {
            std::cout << "reef3d_b200: the slab domain runs without X45 or X48" << std::endl;
            std::exit(1);
        }
        const r3d_grid_desc g = r3d_adapter::grid_desc(p, precision);
        r3d_adapter::check_domain(nullptr, r3d_domain_create(&g, nslabs, devices, &d));
        r3d_adapter::check_domain(d, r3d_domain_set_fluid(d, p->W1, p->W2, p->W3, p->W4));
    }
    ~levelset_RK3_domain() { r3d_domain_destroy(d); }

    void start(fdm* a, lexer* p, convection*, solver*, ghostcell* pgc, ioflow*, reini*, particle_corr*,
               field& ls) override {
        using r3d_adapter::check_domain;
        io.sync(d, p, r3d_adapter::gcval_phi(p));
        check_domain(d, r3d_domain_upload(d, R3D_PHI, ls.V));
        check_domain(d, r3d_domain_upload(d, R3D_U, a->u.V));
        check_domain(d, r3d_domain_upload(d, R3D_V, a->v.V));
        check_domain(d, r3d_domain_upload(d, R3D_W, a->w.V));
        check_domain(d, r3d_domain_run(d, 1, p->dt));
        download(p, R3D_PHI, ls);
        download(p, R3D_RO, a->ro);
        download(p, R3D_VISC, a->visc);
        check_domain(d, r3d_domain_last_volume(d, &p->volume1, &p->volume2));
        if (p->F46 == 0) pgc->start4(p, ls, r3d_adapter::gcval_phi(p));  // picard moves the interior only
        pgc->start4(p, a->ro, 1);
        pgc->start4(p, a->visc, 1);
    }

    void update(lexer* p, fdm* a, ghostcell* pgc, field&) override {
        using r3d_adapter::check_domain;
        check_domain(d, r3d_domain_upload(d, R3D_PHI, a->phi.V));
        check_domain(d, r3d_domain_fluid_update(d, &p->volume1, &p->volume2));
        download(p, R3D_RO, a->ro);
        download(p, R3D_VISC, a->visc);
        pgc->start4(p, a->ro, 1);
        pgc->start4(p, a->visc, 1);
    }

private:
    void download(const lexer* p, int id, field& f) {
        buf.resize((size_t)p->imax * p->jmax * p->kmax);
        r3d_adapter::check_domain(d, r3d_domain_download(d, id, buf.data()));
        r3d_adapter::copy_owned(p, buf, f, true);
    }
    r3d_domain* d = nullptr;
    r3d_adapter::IoflowState io;
    std::vector<double> buf;
};

// convection: the WENO5-HJ operator of the level set (ipol 4), accumulated
// into a->L over the LOOP cells as weno_hj_df_nug::start does
// (src/weno_hj_df_nug.cpp:58-110).
class weno_hj_gpu final : public convection {
public:
    explicit weno_hj_gpu(lexer* p, int precision = R3D_FP64)
        : h(r3d_adapter::make_handle(p, precision)), buf((size_t)p->imax * p->jmax * p->kmax) {
        r3d_adapter::set_direct_forcing(h, p);
    }
    ~weno_hj_gpu() { r3d_destroy(h); }

    void start(lexer* p, fdm* a, field& f, int ipol, field& u, field& v, field& w) override {
        using r3d_adapter::check;
        if (ipol != 4) {
            std::cout << "weno_hj_gpu: only the level set (ipol 4) is on the device" << std::endl;
            std::exit(1);
        }
        check(h, r3d_upload(h, R3D_WORK1, f.V, R3D_LAYOUT_REEF3D));
        check(h, r3d_upload(h, R3D_U, u.V, R3D_LAYOUT_REEF3D));
        check(h, r3d_upload(h, R3D_V, v.V, R3D_LAYOUT_REEF3D));
        check(h, r3d_upload(h, R3D_W, w.V, R3D_LAYOUT_REEF3D));
        r3d_adapter::upload_body(h, p, a, body);
        check(h, r3d_convection_L(h, R3D_WORK1));
        check(h, r3d_download(h, R3D_L, buf.data(), R3D_LAYOUT_REEF3D));
        for (int i = 0; i < p->knox; ++i)
            for (int j = 0; j < p->knoy; ++j)
                for (int k = 0; k < p->knoz; ++k) {
                    const long c = r3d_adapter::ijk(p, i, j, k);
                    if (p->flag4[c] > 0) a->L.V[c] += buf[c];
                }
    }

private:
    r3d_handle* h;
    std::vector<double> buf, body;
};

// reinidisc: the reinitialisation right-hand side (reinidisc_f, or
// reinidisc_fsf when F49 = 0), written to L over the interior
// (src/reinidisc_f.cpp:37-127, src/reinidisc_fsf.cpp:37-141).
class reinidisc_gpu final : public reinidisc {
public:
    explicit reinidisc_gpu(lexer* p, int precision = R3D_FP64) : h(r3d_adapter::make_handle(p, precision)) {}
    ~reinidisc_gpu() { r3d_destroy(h); }

    void start(lexer* p, fdm*, ghostcell*, field& f, field& L, int) override {
        using r3d_adapter::check;
        check(h, r3d_upload(h, R3D_WORK1, f.V, R3D_LAYOUT_REEF3D));
        check(h, r3d_reinidisc_L(h, R3D_WORK1));
        r3d_adapter::download_owned(h, R3D_L, p, L, false, buf);  // BASELOOP cells only
    }

private:
    r3d_handle* h;
    std::vector<double> buf;
};

// reini: the RK3 pseudo-time reinitialisation, 2 int(maxlength/(F43 DXM))
// pseudo-steps on the first call of a run (p->count == 0) and F44 after
// (src/reini_RK3.cpp:84-143), with the picard correction when F46 = 1.
class reini_RK3_gpu final : public reini {
public:
    explicit reini_RK3_gpu(lexer* p, int precision = R3D_FP64) : h(r3d_adapter::make_handle(p, precision)) {}
    ~reini_RK3_gpu() { r3d_destroy(h); }

    void start(fdm*, lexer* p, field& f, ghostcell* pgc, ioflow*) override {
        using r3d_adapter::check;
        const int iters = p->count == 0 ? 2 * int(p->maxlength / (p->F43 * p->DXM)) : p->F44;
        io.sync(h, p, p->count == 0 ? r3d_adapter::gcval_iniphi(p) : r3d_adapter::gcval_phi(p));
        check(h, r3d_upload(h, R3D_PHI, f.V, R3D_LAYOUT_REEF3D));
        check(h, r3d_reinit(h, iters));
        r3d_adapter::download_owned(h, R3D_PHI, p, f, true, buf);
        if (p->F46 != 1)  // (with picard the last shift leaves the ghosts as they were)
            pgc->start4(p, f, p->count == 0 ? r3d_adapter::gcval_iniphi(p) : r3d_adapter::gcval_phi(p));
    }

private:
    r3d_handle* h;
    r3d_adapter::IoflowState io;
    std::vector<double> buf;
};
