// Oracle harness around the reference's OWN level-set objects (test
// infrastructure, never shipped).  It is compiled together with the
// reference sources listed in oracle/Makefile.ref and the single-rank MPI
// stub, and exposes a tiny C API that tests and fixture scripts call through
// ctypes.  One grid per process: the reference keeps loop indices and WENO
// coefficient tables in static members (src/increment.h:38,
// src/weno_nug_func.h:198-202), so a second grid in the same process would
// silently reuse the first grid's tables.
//
// Set-up mirrors the reference's start-up order
//   src/driver.cpp:33-57   (lexer, ghostcell, lexer_read, vellast, gc_ini,
//                           gcx_ini, gridini)
//   src/driver.cpp:116-120 (flagini, flagfield, makegrid)
//   src/driver_makegrid.cpp:29-62
// except that the DIVEMesh grid file is replaced by assigning the same
// lexer members read_grid() assigns (src/read_grid.cpp:29-911) for a closed
// box whose six faces are walls (boundary group 21), and the control file
// is replaced by assigning the few control flags the path reads.

#include "lexer.h"
#include "fdm.h"
#include "ghostcell.h"
#include "grid_helper.h"
#include "levelset_RK3.h"
#include "weno_hj_df_nug.h"
#include "reini_RK3.h"
#include "reinidisc_f.h"
#include "reinidisc_fsf.h"
#include "ioflow_void.h"
#include "ioflow_f.h"
#include "particle_pls_void.h"
#include "heat.h"
#include "concentration.h"
#include "fluid_update_fsf.h"
#include "patchBC_void.h"
#include "mgcslice1.h"
#include "ietimestep.h"
#include "kepsilon_void.h"
#include "mgcslice2.h"
#include "mgcslice4.h"
// iowave (the wave generator's relaxation zones): its own headers first, then
// the class with its private members readable by this harness (test
// infrastructure reading relax4_wg / relax4_nb / lsval, which the reference
// keeps private; nothing of the reference is modified)
#include "ioflow.h"
#include "wave_interface.h"
#include "field1.h"
#include "field2.h"
#include "slice1.h"
#include "slice2.h"
#include "slice4.h"
#include "sliceint4.h"
#include "flowfile_in.h"
#define private public
#include "iowave.h"
#include "cfd_state.h"
#include "sediment_void.h"
#undef private

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#include <unistd.h>

namespace {

lexer* P = nullptr;
ghostcell* PGC = nullptr;
fdm* A = nullptr;
weno_hj_df_nug* CONV = nullptr;
reini_RK3* REINI = nullptr;
levelset_RK3* LS = nullptr;
ioflow* FLOW = nullptr;
particle_corr* PART = nullptr;
reinidisc* DISC = nullptr;
heat* HEAT = nullptr;
concentration* CONC = nullptr;
field4* TMP = nullptr;
int G_F46 = 0, G_F47 = 10;  // picard mass correction flags for the next refls_init
int G_X45 = 0;              // level-set convection stencil at bodies for the next refls_init
std::vector<int> G_SF;      // gcdf4 entries (i, j, k, side) of the solid forcing (X48 = 1)
// inflow (x-min) / outflow (x-max) boundaries and ioflow_f flags for the next
// refls_init; io.on == 0 keeps the closed box and ioflow_v
struct IoFlags {
    int on = 0, inflow = 0, outflow = 0, f50 = 2, b77 = 1, f64 = 0;
    double f56 = 1.0e20, f60 = -1.0e20, f61 = -1.0e20, f62 = -1.0e20, qi = 0.0, qo = 0.0;
} G_IO;
// iowave (B90 = 1) for the next refls_init, wave maker B98 (2: relaxation
// zone, 3: Dirichlet, 4: active) and beach B99 (2: relaxation zone, 3-5:
// active); on == 0: no wave generator
struct WaveFlags {
    int on = 0, b92 = 2, b101 = 0, b98 = 2, b99 = 2;
    double amp = 0.0, period = 0.0, depth = 0.0, b96_1 = 0.0, b96_2 = 0.0, phimean = 0.0, b102 = 1.0;
} G_IOW;
iowave* WAVE = nullptr;
ietimestep* TSTEP = nullptr;
turbulence* TURB = nullptr;

long ncells_padded() { return (long)P->imax * P->jmax * P->kmax; }

field* field_by_id(int id) {
    switch (id) {
        case 0: return &A->phi;
        case 1: return &A->u;
        case 2: return &A->v;
        case 3: return &A->w;
        case 4: return &A->L;
        case 5: return TMP;
        case 6: return &A->ro;
        case 7: return &A->visc;
        // body fields the direct-forcing WENO stencils read (X45 1..6,
        // src/weno_hj_df_nug.cpp:398-987)
        case 8: return &A->fb;
        case 9: return &A->fbh4;
        case 10: return &A->fbh5;
        case 11: return &A->solid;
        case 12: return &A->topo;
        // further fields of the restart state file (src/cfd_state_write.cpp)
        case 13: return &A->press;
        case 14: return &A->eddyv;
        case 15: return &A->conc;
        default: return nullptr;
    }
}

int ijk(int i, int j, int k) {
    return (i - P->imin) * P->jmax * P->kmax + (j - P->jmin) * P->kmax + (k - P->kmin);
}

}  // namespace

// The harness's objects, for oracle/ref_adapter.cpp (the adapter test).
namespace refh {
lexer* lex() { return P; }
fdm* fd() { return A; }
ghostcell* gc() { return PGC; }
ioflow* flow() { return FLOW; }
field4* tmp() { return TMP; }
}  // namespace refh

extern "C" {

// Picard mass correction of the next refls_init: f46 = 1 (in reini_RK3,
// src/reini_RK3.cpp:92,140), 2 (picard_f in levelset_RK3,
// src/levelset_RK3.cpp:110,171) or 3 (picard_lsm there), f47 iterations
// (src/picard_f.cpp:82-113, src/picard_lsm.cpp:89-116).
void refls_set_picard(int f46, int f47) { G_F46 = f46; G_F47 = f47; }

// X45 of the next refls_init: the direct-forcing variant of the level-set
// WENO stencils (0 plain; 1..6 mask or weight the divided differences by
// the body fields fb, fbh4, fbh5, solid, topo, src/weno_hj_df_nug.cpp:398-987).
void refls_set_x45(int x45) { G_X45 = x45; }

// The solid forcing of the level set after each convection stage
// (ghostcell::solid_forcing_lsm, src/gc_solid_forcing_lsm.cpp:27-78, X48 = 1):
// n entries (i, j, k, side) of the direct-forcing boundary list gcdf4, which
// a solid geometry would produce (src/gcdf_update.cpp).
void refls_set_solid_forcing(int n, const int* cells) { G_SF.assign(cells, cells + 4 * n); }

// Inflow / outflow boundaries of the next refls_init.  inflow: the x-min face
// is boundary type 1, outflow: the x-max face type 2 (the other faces stay
// walls, type 21); the flow object becomes ioflow_f (B60 = 1,
// src/driver_logic_cfd.cpp:509-510) with the level-set flags F50, B77,
// F56, F60, F61, F62, F64 (src/ini.cpp:208-441) and discharges Qi, Qo.
void refls_set_ioflow(int inflow, int outflow, int f50, int b77, double f56, double f60, double f61,
                      double f62, int f64, double qi, double qo) {
    G_IO.on = 1;
    G_IO.inflow = inflow; G_IO.outflow = outflow; G_IO.f50 = f50; G_IO.b77 = b77;
    G_IO.f56 = f56; G_IO.f60 = f60; G_IO.f61 = f61; G_IO.f62 = f62; G_IO.f64 = f64;
    G_IO.qi = qi; G_IO.qo = qo;
}

// Wave generator of the next refls_init: REEF3D's iowave (B90 = 1) with the
// x-min face as inflow and the x-max face as outflow, wave theory b92 (2:
// linear waves, src/wave_interface.cpp:60-80) of amplitude amp and period
// (B93 = 1), water depth (B94 = 1), the wave maker b98 (2: relaxation-zone
// generation over b96_1 from the x-min face; 3 Dirichlet, 4 active) and the
// beach b99 (2: relaxation zone over b96_2 before the x-max face, the default
// zone lines of src/iowave.cpp:130-170; 3-5 active absorption), still water
// level phimean (F56), ramp B101/B102.
void refls_set_iowave(int b92, double amp, double period, double depth, double b96_1, double b96_2,
                      double phimean, int b101, double b102, int b98, int b99) {
    G_IOW.on = 1;
    G_IOW.b98 = b98; G_IOW.b99 = b99;
    G_IOW.b92 = b92; G_IOW.amp = amp; G_IOW.period = period; G_IOW.depth = depth;
    G_IOW.b96_1 = b96_1; G_IOW.b96_2 = b96_2; G_IOW.phimean = phimean; G_IOW.b101 = b101; G_IOW.b102 = b102;
    G_IO.on = 1;
    G_IO.inflow = 1;
    G_IO.outflow = 1;
}

// xn/yn/zn: node coordinates for index -5 .. n+5 (n+11 values), the same
// arrays DIVEMesh writes (src/read_grid.cpp:417-433, marge=5).
// f49 selects reinidisc_f (1) or reinidisc_fsf (0); f44 the reinit
// pseudo-steps per physical step; f43 the reinit time-step factor; f45 the
// interface-thickness factor.
int refls_init(int nx, int ny, int nz, const double* xn, const double* yn, const double* zn,
               int f44, double f43, double f45, int f49) {
    if (P) return -1;
    int argc = 0;
    char** argv = nullptr;
    // members the reference never assigns are read as zero, as the fresh
    // heap of a REEF3D process gives them (e.g. gcsldfbed4_count, read by
    // ghostcell::solid_forcing_bed from iowave's set-up): the lexer is
    // constructed in zeroed memory
    P = new (std::calloc(1, sizeof(lexer))) lexer;
    PGC = new ghostcell(argc, argv, P);
    lexer* p = P;

    // control flags on this path (defaults src/ini.cpp:400-416)
    p->F30 = 3; p->F35 = 5; p->F40 = 3;
    p->F43 = f43; p->F44 = f44; p->F45 = f45; p->F46 = G_F46; p->F47 = G_F47; p->F49 = f49; p->F50 = 2;
    if (G_IO.on) {
        p->F50 = G_IO.f50; p->B60 = 1; p->B77 = G_IO.b77;
        p->F56 = G_IO.f56; p->F60 = G_IO.f60; p->F61 = G_IO.f61; p->F62 = G_IO.f62; p->F64 = G_IO.f64;
    }
    p->X45 = G_X45; p->X48 = 0; p->M10 = 1; p->P12 = 1000000000;
    if (G_IOW.on) {  // control letters of the wave generator (src/ini.cpp:224-240)
        p->B60 = 0;
        p->B90 = 1; p->B92 = G_IOW.b92;
        p->B93 = 1; p->B93_1 = G_IOW.amp; p->B93_2 = G_IOW.period;
        p->B94 = 1; p->B94_wdt = G_IOW.depth;
        p->B96_1 = G_IOW.b96_1; p->B96_2 = G_IOW.b96_2;
        p->B98 = G_IOW.b98; p->B99 = G_IOW.b99; p->B101 = G_IOW.b101; p->B102 = G_IOW.b102;
        p->F56 = G_IOW.phimean; p->phimean = G_IOW.phimean; p->phiout = G_IOW.phimean;
        p->A10 = 6;
        p->xcoormin = xn[5]; p->xcoormax = xn[5 + nx];
        p->ycoormin = yn[5]; p->ycoormax = yn[5 + ny];
        p->simtime = 0.0;
    }

    // --- what read_grid() assigns (src/read_grid.cpp:78-300)
    p->knox = nx; p->knoy = ny; p->knoz = nz;
    p->gknox = nx; p->gknoy = ny; p->gknoz = nz;
    p->origin_i = p->origin_j = p->origin_k = 0;
    p->dx = xn[5 + 1] - xn[5];
    p->DXM = xn[5 + 1] - xn[5];
    p->DYM = yn[5 + 1] - yn[5];
    p->DZM = zn[5 + 1] - zn[5];
    p->originx = p->global_xmin = xn[5];
    p->originy = p->global_ymin = yn[5];
    p->originz = p->global_zmin = zn[5];
    p->endx = p->global_xmax = xn[5 + nx];
    p->endy = p->global_ymax = yn[5 + ny];
    p->endz = p->global_zmax = zn[5 + nz];
    p->nb1 = p->nb2 = p->nb3 = p->nb4 = p->nb5 = p->nb6 = -2;
    p->mx = p->my = p->mz = 1;
    p->periodic1 = p->periodic2 = p->periodic3 = 0;
    p->periodicX1 = p->periodicX2 = p->periodicX3 = 0;
    p->periodicX4 = p->periodicX5 = p->periodicX6 = 0;
    p->i_dir = 1; p->j_dir = (ny > 1) ? 1 : 0; p->k_dir = 1;
    p->P150 = 0; p->solidread = 0; p->toporead = 0;
    p->solid_gcb_est = p->topo_gcb_est = 0;
    p->solid_gcbextra_est = p->topo_gcbextra_est = p->tot_gcbextra_est = 0;
    p->global_orig_x = p->global_orig_y = p->alpha_grid = 0.0;
    p->gcpara1_count = p->gcpara2_count = p->gcpara3_count = 0;
    p->gcpara4_count = p->gcpara5_count = p->gcpara6_count = 0;
    p->gcparaco1_count = p->gcparaco2_count = p->gcparaco3_count = 0;
    p->gcparaco4_count = p->gcparaco5_count = p->gcparaco6_count = 0;
    p->gcslpara1_count = p->gcslpara2_count = p->gcslpara3_count = p->gcslpara4_count = 0;
    p->gcslparaco1_count = p->gcslparaco2_count = p->gcslparaco3_count = p->gcslparaco4_count = 0;
    p->gcin_count = p->gcout_count = 0;
    // never assigned by the reference (read by lexer::vecsize,
    // src/lexer_vectorsize.cpp:37); zero, as in a fresh process heap
    p->gcextra4 = 0;

    // wall list: every interior cell on each face, one entry per face side
    // (side codes of src/gc_neumann.cpp:29-54: 1 -x, 4 +x, 3 -y, 2 +y, 5 -z, 6 +z)
    std::vector<int> wall;
    auto add = [&](int i, int j, int k, int side) {
        wall.push_back(i); wall.push_back(j); wall.push_back(k); wall.push_back(side);
    };
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                if (i == 0) add(i, j, k, 1);
                if (i == nx - 1) add(i, j, k, 4);
                if (j == 0) add(i, j, k, 3);
                if (j == ny - 1) add(i, j, k, 2);
                if (k == 0) add(i, j, k, 5);
                if (k == nz - 1) add(i, j, k, 6);
            }
    p->gcwall_count = (int)(wall.size() / 4);

    p->topo_gcb_est *= 4;
    p->gcb1_count = p->gcb2_count = p->gcb3_count = p->gcb4_count = p->gcb4a_count = p->gcb_fix =
        p->gcb_solid = p->gcb_topo = p->gcb_fb = p->gcwall_count;
    p->gcpara_sum = 0;
    p->gcparaco_sum = 0;
    p->assign_margin();

    p->Iarray(p->flag4, p->imax * p->jmax * p->kmax);
    p->Darray(p->flag_solid, p->imax * p->jmax * p->kmax);
    p->Darray(p->flag_topo, p->imax * p->jmax * p->kmax);
    p->Darray(p->solidbed, p->imax * p->jmax);
    p->Darray(p->topobed, p->imax * p->jmax);
    p->Darray(p->bed, p->imax * p->jmax);
    p->Iarray(p->wet, p->imax * p->jmax);
    p->Iarray(p->wet_n, p->imax * p->jmax);
    p->Iarray(p->deep, p->imax * p->jmax);
    p->Darray(p->depth, p->imax * p->jmax);
    p->Darray(p->data, p->imax * p->jmax);
    p->Iarray(p->flagslice1, p->imax * p->jmax);
    p->Iarray(p->flagslice2, p->imax * p->jmax);
    p->Iarray(p->flagslice4, p->imax * p->jmax);
    for (long n = 0; n < (long)p->imax * p->jmax * p->kmax; ++n) p->flag4[n] = -1;
    for (long n = 0; n < (long)p->imax * p->jmax; ++n) {
        p->flagslice1[n] = -10; p->flagslice2[n] = -10; p->flagslice4[n] = -10;
    }
    p->Iarray(p->gcb1, p->gcb1_count, 6);
    p->Iarray(p->gcb2, p->gcb2_count, 6);
    p->Iarray(p->gcb3, p->gcb3_count, 6);
    p->Iarray(p->gcb4, p->gcb4_count, 6);
    p->Iarray(p->gcb4a, p->gcb4a_count, 6);
    p->Darray(p->gcd1, p->gcb1_count);
    p->Darray(p->gcd2, p->gcb2_count);
    p->Darray(p->gcd3, p->gcb3_count);
    p->Darray(p->gcd4, p->gcb4_count);
    p->Darray(p->gcd4a, p->gcb4a_count);
    p->Iarray(p->gcpara1, 0, 16); p->Iarray(p->gcpara2, 0, 16); p->Iarray(p->gcpara3, 0, 16);
    p->Iarray(p->gcpara4, 0, 16); p->Iarray(p->gcpara5, 0, 16); p->Iarray(p->gcpara6, 0, 16);
    p->Iarray(p->gcparaco1, 0, 3); p->Iarray(p->gcparaco2, 0, 3); p->Iarray(p->gcparaco3, 0, 3);
    p->Iarray(p->gcparaco4, 0, 3); p->Iarray(p->gcparaco5, 0, 3); p->Iarray(p->gcparaco6, 0, 3);
    p->gcbsl1_count = p->gcbsl2_count = p->gcbsl3_count = p->gcbsl4_count = p->gcbsl4a_count = 1;
    p->Iarray(p->gcbsl1, 1, 6); p->Iarray(p->gcbsl2, 1, 6); p->Iarray(p->gcbsl3, 1, 6);
    p->Iarray(p->gcbsl4, 1, 6); p->Iarray(p->gcbsl4a, 1, 6);
    p->Iarray(p->gcslin, 0, 6); p->Iarray(p->gcslout, 0, 6);
    p->Iarray(p->gcslpara1, 0, 2); p->Iarray(p->gcslpara2, 0, 2);
    p->Iarray(p->gcslpara3, 0, 2); p->Iarray(p->gcslpara4, 0, 2);
    p->Iarray(p->gcslparaco1, 0, 4); p->Iarray(p->gcslparaco2, 0, 4);
    p->Iarray(p->gcslparaco3, 0, 4); p->Iarray(p->gcslparaco4, 0, 4);
    p->Darray(p->XN, nx + 1 + 4 * p->marge);
    p->Darray(p->YN, ny + 1 + 4 * p->marge);
    p->Darray(p->ZN, nz + 1 + 4 * p->marge);

    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) p->flag4[ijk(i, j, k)] = WATER_FLAG;
    // the wave generator works on the water-surface slices (SLICELOOP4 over
    // flagslice4 > 0, src/looping2D.h:51), which a DIVEMesh grid marks for
    // every interior column (src/read_grid.cpp:753-758)
    if (G_IOW.on)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) p->flagslice4[(i - p->imin) * p->jmax + (j - p->jmin)] = 1;
    for (int n = 0; n < nx + 1 + 2 * p->marge; ++n) p->XN[n] = xn[n];
    for (int n = 0; n < ny + 1 + 2 * p->marge; ++n) p->YN[n] = yn[n];
    for (int n = 0; n < nz + 1 + 2 * p->marge; ++n) p->ZN[n] = zn[n];
    for (int q = 0; q < p->gcb4_count; ++q) {
        p->gcb4[q][0] = wall[4 * q + 0];
        p->gcb4[q][1] = wall[4 * q + 1];
        p->gcb4[q][2] = wall[4 * q + 2];
        p->gcb4[q][3] = wall[4 * q + 3];
        const int side = wall[4 * q + 3];
        p->gcb4[q][4] = (G_IO.on && G_IO.inflow && side == 1) ? 1
                        : (G_IO.on && G_IO.outflow && side == 4) ? 2 : 21;
    }
    p->Iarray(p->gcin, 0, 6); p->Iarray(p->gcout, 0, 6);
    p->Iarray(p->gcin4a, 0, 6); p->Iarray(p->gcout4a, 0, 6);
    p->gcin4a_count = 0; p->gcout4a_count = 0;

    // --- driver start-up (src/driver.cpp:51-57, 116-120)
    p->lexer_ini();
    p->vellast();
    PGC->gc_ini(p);
    PGC->gcx_ini(p);
    p->gridini(PGC);
    p->flagini();
    PGC->flagfield(p);
    {   // body of driver::makegrid (src/driver_makegrid.cpp:29-62)
        PGC->flagx(p, p->flagsf1); PGC->flagx(p, p->flagsf2);
        PGC->flagx(p, p->flagsf3); PGC->flagx(p, p->flagsf4);
        PGC->flagx(p, p->flag1); PGC->flagx(p, p->flag2); PGC->flagx(p, p->flag3);
        PGC->flagx(p, p->flag4); PGC->flagx(p, p->flag);
        PGC->gcxupdate(p);
        p->vecsize(PGC);
        grid_helper gridgen(p);
        gridgen.fillgcb1(p);
        gridgen.fillgcb2(p);
        gridgen.fillgcb3(p);
        gridgen.fillgcb4a(p);
        gridgen.fillgcb4_wall(p);
        gridgen.make_dgc(p);
        gridgen.fill_dgc1(p);
        gridgen.fill_dgc2(p);
        gridgen.fill_dgc3(p);
        gridgen.fill_dgc4(p);
    }
    {   // body of driver::makegrid2D (src/driver_makgrid_2D.cpp:31-74): the
        // slice ghost lists sized here are allocated by every fdm
        PGC->gcslflagx(p, p->flagslice4);
        mgcslice1 m1(p);
        mgcslice2 m2(p);
        mgcslice4 m4(p);
        m1.makemgc(p); PGC->gcslflagx(p, p->flagslice1);
        m1.gcb_seed(p); m1.mgcsetup(p); m1.fillmgc(p); m1.gcdirfill(p);
        m2.makemgc(p); PGC->gcslflagx(p, p->flagslice2);
        m2.gcb_seed(p); m2.mgcsetup(p); m2.fillmgc(p); m2.gcdirfill(p);
        m4.makemgc(p);
        m4.gcb_seed(p); m4.mgcsetup(p); m4.fillmgc(p); m4.gcdirfill(p);
        m1.make_ggc(p); m1.fill_ggc(p);
        m2.make_ggc(p); m2.fill_ggc(p);
        m4.make_ggc(p); m4.fill_ggc(p);
        PGC->gcsl_setbc1(p); PGC->gcsl_setbc2(p); PGC->gcsl_setbc4(p);
        PGC->gcsl_setbcio(p);
        PGC->dgcslini1(p); PGC->dgcslini2(p); PGC->dgcslini4(p);
    }

    A = new fdm(p);
    PGC->fdm_update(A);
    // porosity is 1 everywhere without VRANS structures
    for (long n = 0; n < ncells_padded(); ++n) A->porosity.V[n] = 1.0;

    // psi (src/ini_psi.cpp:33-37)
    if (p->j_dir == 0) p->psi = p->F45 * (1.0 / 2.0) * (p->DXM + p->DZM);
    if (p->j_dir == 1) p->psi = p->F45 * (1.0 / 3.0) * (p->DXM + p->DYM + p->DZM);

    CONV = new weno_hj_df_nug(p);
    // no patch boundaries: driver::patchBC_logic picks patchBC_void
    // (src/driver_logic_cfd.cpp:661-672)
    if (G_IOW.on) {
        p->phimean = p->phiout = p->phiin = G_IOW.phimean;  // src/ini_phi.cpp:33
        // iowave's constructor writes the wave time series into
        // ./REEF3D_Log-Wave (src/iowave_timeseries.cpp:38-58): construct it
        // from a scratch directory so the caller's working directory stays clean
        char cwd[4096];
        char scratch[] = "/tmp/refls_wave_XXXXXX";
        bool moved = getcwd(cwd, sizeof cwd) != nullptr && mkdtemp(scratch) != nullptr && chdir(scratch) == 0;
        FLOW = WAVE = new iowave(p, PGC, new patchBC_void(p));
        if (moved && chdir(cwd) != 0) return -2;
    }
    else if (G_IO.on) FLOW = new ioflow_f(p, PGC, new patchBC_void(p));
    else FLOW = new ioflow_v(p, PGC, new patchBC_void(p));
    PART = new particle_pls_void();
    REINI = new reini_RK3(p, 0);
    LS = new levelset_RK3(p, A, PGC, HEAT, CONC);
    if (f49 == 1) DISC = new reinidisc_f(p);
    else DISC = new reinidisc_fsf(p);
    TMP = new field4(p);
    TSTEP = new ietimestep(p);
    TURB = new kepsilon_void(p, A, PGC);
    if (!G_SF.empty()) {
        const int n = (int)(G_SF.size() / 4);
        p->X48 = 1;
        p->Iarray(p->gcdf4, n, 6);
        for (int q = 0; q < n; ++q)
            for (int c = 0; c < 4; ++c) p->gcdf4[q][c] = G_SF[4 * q + c];
        p->gcdf4_count = n;
    }
    p->count = 1;
    p->dt = 0.0;
    p->Qi = p->Qo = 0.0;  // closed box: no discharge (read by picard_lsm, src/picard_lsm.cpp:95)
    if (G_IO.on) {
        p->Qi = G_IO.qi; p->Qo = G_IO.qo;
        // inflow / outflow cell lists gcin, gcout (src/ioflow_util.cpp:30-81);
        // iowave also fills the gcb4a lists gcin4a / gcout4a without
        // resizing them (src/iowave_util.cpp:101-128): room for every entry
        if (WAVE) {
            p->Iarray(p->gcin4a, p->gcb4a_count, 6);
            p->Iarray(p->gcout4a, p->gcb4a_count, 6);
        }
        FLOW->gcio_update(p, A, PGC);
    }
    if (WAVE) FLOW->ini(p, A, PGC);  // relaxation functions and the first targets (src/iowave_ini.cpp:29-50)
    return 0;
}

// The clock (lexer::simtime) the wave generator's targets and ramp read.
void refls_set_time(double t) { P->simtime = t; }

// The wave generator's per-step targets (iowave::wavegen_precalc,
// src/driver_loop_cfd.cpp:78), as the driver computes them before each
// free-surface step.
int refls_wavegen_precalc() {
    if (!WAVE) return -1;
    FLOW->wavegen_precalc(P, PGC);
    return 0;
}

// Relaxation weights per interior column (i * ny + j): relax4_wg(i,j) where
// distgen < 1e20 (the generation zone), relax4_nb(i,j) where distbeach <
// 1e20 (the beach), -1 elsewhere (src/iowave_relax.cpp:346-378).
int refls_iowave_weights(double* wg, double* wb) {
    if (!WAVE) return -1;
    lexer* p = P;
    for (int i = 0; i < p->knox; ++i)
        for (int j = 0; j < p->knoy; ++j) {
            increment::i = i;
            increment::j = j;
            increment::k = 0;
            const double dg = WAVE->distgen(p), db = WAVE->distbeach(p);
            wg[i * p->knoy + j] = dg < 1.0e20 ? WAVE->relax4_wg(i, j) : -1.0;
            wb[i * p->knoy + j] = db < 1.0e20 ? WAVE->relax4_nb(i, j) : -1.0;
        }
    return 0;
}

// The generation zone's current targets (iowave::lsval, LOOP order over the
// zone, src/iowave_precalc_relax.cpp) and iowave::ramp; returns their count
// (n = capacity of lsval; -1 when larger).
long refls_iowave_targets(double* lsval, long n, double* ramp) {
    if (!WAVE) return -1;
    lexer* p = P;
    long count = 0;
    for (int i = 0; i < p->knox; ++i)
        for (int j = 0; j < p->knoy; ++j) {
            increment::i = i;
            increment::j = j;
            increment::k = 0;
            if (WAVE->distgen(p) < 1.0e20) count += p->knoz;
        }
    if (count > n) return -1;
    for (long q = 0; q < count; ++q) lsval[q] = WAVE->lsval[q];
    *ramp = WAVE->ramp(p);
    return count;
}

long refls_padded_size() { return P ? ncells_padded() : -1; }
int refls_dims(int* out) {
    if (!P) return -1;
    out[0] = P->imax; out[1] = P->jmax; out[2] = P->kmax; out[3] = P->j_dir;
    return 0;
}

int refls_set_field(int id, const double* src) {
    field* f = field_by_id(id);
    if (!f) return -1;
    std::memcpy(f->V, src, sizeof(double) * ncells_padded());
    return 0;
}

int refls_get_field(int id, double* dst) {
    field* f = field_by_id(id);
    if (!f) return -1;
    std::memcpy(dst, f->V, sizeof(double) * ncells_padded());
    return 0;
}

void refls_set_dt(double dt) { P->dt = dt; }
void refls_set_count(int c) { P->count = c; }
double refls_psi() { return P->psi; }
double refls_dxm() { return P->DXM; }
double refls_volume1() { return P->volume1; }
double refls_volume2() { return P->volume2; }
// Point data of the reference's VTU printer over the TPLOOP nodes (i
// fastest, src/printer_CFD.cpp:678-727): ipol4phi(a->phi), ipol4_a(a->ro),
// ipol4(a->visc), each stored as float like the printer.
int refls_vtu_point_data(float* phi, float* ro, float* visc) {
    lexer* p = P;
    long n = 0;
    for (int k = -1; k < p->knoz; ++k)
        for (int j = -1; j < p->knoy; ++j)
            for (int i = -1; i < p->knox; ++i) {
                increment::i = i;
                increment::j = j;
                increment::k = k;
                phi[n] = float(p->ipol4phi(A, A->phi));
                ro[n] = float(p->ipol4_a(A->ro));
                visc[n] = float(p->ipol4(A->visc));
                ++n;
            }
    return 0;
}

// Water levels of the last ioflow_f::fsfinflow (src/ioflow_waterlevel.cpp:29-141).
int refls_io_levels(double* out) {
    out[0] = P->phimean; out[1] = P->phiout;
    out[2] = P->gcin_count; out[3] = P->gcout_count;
    return 0;
}

// Metric arrays as the reference derives them from the node coordinates
// (src/grid.cpp:55-100): which 0..8 = DXN,DYN,DZN,DXP,DYP,DZP,XP,YP,ZP.
int refls_get_metric(int which, double* dst, int n) {
    double* src[9] = {P->DXN, P->DYN, P->DZN, P->DXP, P->DYP, P->DZP, P->XP, P->YP, P->ZP};
    if (which < 0 || which > 8) return -1;
    std::memcpy(dst, src[which], sizeof(double) * n);
    return 0;
}

// WENO coefficient tables for axis 0..2 (uf=0 node tables): qf [n][6][2],
// cf [n][6], isf [n][6][3], for index IP = -1+5 .. knox+5 (as built by
// src/weno_nug_func_precalc_*.cpp).  n entries starting at table index 0.
int refls_get_weno_tables(int axis, double* qf, double* cf, double* isf, int n) {
    double**** q = axis == 0 ? weno_nug_func::qfx : axis == 1 ? weno_nug_func::qfy : weno_nug_func::qfz;
    double*** c = axis == 0 ? weno_nug_func::cfx : axis == 1 ? weno_nug_func::cfy : weno_nug_func::cfz;
    double**** s = axis == 0 ? weno_nug_func::isfx : axis == 1 ? weno_nug_func::isfy : weno_nug_func::isfz;
    for (int t = 0; t < n; ++t)
        for (int r = 0; r < 6; ++r) {
            qf[(t * 6 + r) * 2 + 0] = q[t][0][r][0];
            qf[(t * 6 + r) * 2 + 1] = q[t][0][r][1];
            cf[t * 6 + r] = c[t][0][r];
            for (int m = 0; m < 3; ++m) isf[(t * 6 + r) * 3 + m] = s[t][0][r][m];
        }
    return 0;
}

// L = convection operator of src/weno_hj_df_nug.cpp:58-91 (ipol=4) applied to
// field `src` with the stored velocities; the caller's L is zeroed first as
// src/levelset_RK3.cpp:115-116 does.
int refls_weno_L(const double* src, double* L) {
    std::memcpy(TMP->V, src, sizeof(double) * ncells_padded());
    for (long n = 0; n < ncells_padded(); ++n) A->L.V[n] = 0.0;
    CONV->start(P, A, *TMP, 4, A->u, A->v, A->w);
    std::memcpy(L, A->L.V, sizeof(double) * ncells_padded());
    return 0;
}

// L = reinitialisation operator (src/reinidisc_f.cpp:37-127 or
// src/reinidisc_fsf.cpp:37-141) applied to `src`.
int refls_reinidisc_L(const double* src, double* L) {
    std::memcpy(TMP->V, src, sizeof(double) * ncells_padded());
    for (long n = 0; n < ncells_padded(); ++n) A->L.V[n] = 0.0;
    DISC->start(P, A, PGC, *TMP, A->L, 4);
    std::memcpy(L, A->L.V, sizeof(double) * ncells_padded());
    return 0;
}

// Ghost fill of a level-set field: ghostcell::start4 with the level set's
// gcv 50+F50 (52 for the default F50 = 2; src/gc_start.cpp:146-185,
// src/levelset_RK3.cpp:50-60).
int refls_ghost_fill(double* f) {
    std::memcpy(TMP->V, f, sizeof(double) * ncells_padded());
    PGC->start4(P, *TMP, 50 + P->F50);
    std::memcpy(f, TMP->V, sizeof(double) * ncells_padded());
    return 0;
}

// F44 reinitialisation pseudo-steps on phi (src/reini_RK3.cpp:84-143).
int refls_reini() {
    REINI->start(A, P, A->phi, PGC, FLOW);
    return 0;
}

// One physical level-set step on phi with the current dt and velocities
// (src/levelset_RK3.cpp:103-172), including reinitialisation and the
// density/volume update.
int refls_step() {
    convection* pc = CONV;
    LS->start(A, P, pc, nullptr, PGC, FLOW, REINI, PART, A->phi);
    return 0;
}

// Adaptive time step from the stored velocities with CFL factor n47
// (src/ietimestep.cpp:38-206; maxF=maxG=maxH=0 for a prescribed velocity).
double refls_cfl_dt(double n47) {
    P->N47 = n47;
    A->maxF = A->maxG = A->maxH = 0.0;
    TSTEP->start(A, P, PGC, TURB);
    return P->dt;
}

// Density/volume update only (src/fluid_update_fsf.cpp:39-104).
int refls_update() {
    LS->update(P, A, PGC, A->phi);
    return 0;
}

// The reference's restart state file of the current fields: cfd_state::write
// (src/cfd_state.cpp:201-220, i.e. write_result, src/cfd_state_write.cpp:34-146)
// with the step count, print count and time given, from the working
// directory `dir` (the file lands in dir/REEF3D_CFD_STATE/, named
// REEF3D-CFD-State-00000000-000001.r3d: the first file of a single rank,
// P15 = 1).  Turbulence and sediment are the void models (k, epsilon and the
// bed-load slice written as their zeros).  P45 = 1: no continuous file.
// The water-surface slices of every interior column, as a DIVEMesh grid
// marks them (src/read_grid.cpp:753-758), while a state file is written or
// read (its bed-load block is a SLICELOOP4); the harness's marks otherwise.
struct SliceMarks {
    std::vector<int> saved;
    SliceMarks() {
        const long n = (long)P->imax * P->jmax;
        saved.assign(P->flagslice4, P->flagslice4 + n);
        for (int i = 0; i < P->knox; ++i)
            for (int j = 0; j < P->knoy; ++j) P->flagslice4[(i - P->imin) * P->jmax + (j - P->jmin)] = 1;
    }
    ~SliceMarks() { std::copy(saved.begin(), saved.end(), P->flagslice4); }
};

int refls_write_state(const char* dir, int count, int printcount, double simtime) {
    char cwd[4096];
    if (!P || !getcwd(cwd, sizeof cwd) || chdir(dir) != 0) return -1;
    SliceMarks marks;
    P->count = count;
    P->printcount = printcount;
    P->simtime = simtime;
    P->P15 = 1; P->P40 = 0; P->P43 = 0; P->P45 = 1;
    {
        sediment_void sed;
        cfd_state st(P, A, PGC, 0);
        st.write(P, A, PGC, TURB, &sed);
    }
    return chdir(cwd) == 0 ? 0 : -2;
}

// cfd_state::read (src/cfd_state_read.cpp) of state number num from
// dir/REEF3D_CFD_STATE/, with the control file's defaults for the topo
// ghost condition (S50 = 4, src/ini.cpp:783); the fields and p->count /
// p->simtime are then the file's.
int refls_read_state(const char* dir, int num, int* count, double* simtime) {
    char cwd[4096];
    if (!P || !getcwd(cwd, sizeof cwd) || chdir(dir) != 0) return -1;
    P->I41 = num; P->P43 = 0; P->P45 = 1; P->S50 = 4;
    SliceMarks marks;
    {
        sediment_void sed;
        cfd_state st(P, A, PGC, 1);
        st.read(P, A, PGC, TURB, &sed);
    }
    *count = P->count;
    *simtime = P->simtime;
    return chdir(cwd) == 0 ? 0 : -2;
}

}  // extern "C"
