// Test infrastructure, never shipped: runs the REEF3D-side adapter classes
// (reef3d_b200/adapters/reef3d_b200_adapters.h) on the harness's own REEF3D
// objects (lexer, fdm, ghostcell; oracle/ref_harness.cpp), so a test can
// compare, in one process and on the same REEF3D data structures, what the
// reference's levelset_RK3 / weno_hj_df_nug / reinidisc / reini_RK3 compute
// on the CPU with what the adapters compute through libreef3d_b200.so.
// Built into oracle/_ref/libreef3d_adapter.so by oracle/Makefile.ref.

// iowave's relaxation weights and targets are private; the adapter reads
// them as the friend a REEF3D maintainer declares in src/iowave.h.  This
// test build, which leaves the reference untouched, opens them instead.
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
#undef private
#include "reef3d_b200_adapters.h"

#include <cstring>

namespace refh {
lexer* lex();
fdm* fd();
ghostcell* gc();
ioflow* flow();
field4* tmp();
}  // namespace refh

namespace {
levelset_RK3_gpu* G_LS = nullptr;
levelset_RK3_domain* G_LSD = nullptr;
weno_hj_gpu* G_CONV = nullptr;
reinidisc_gpu* G_DISC = nullptr;
reini_RK3_gpu* G_REINI = nullptr;

long ncell() {
    lexer* p = refh::lex();
    return (long)p->imax * p->jmax * p->kmax;
}
}  // namespace

extern "C" {

// Adapters on the current harness grid (after refls_init); precision
// R3D_FP64 or R3D_FP32; resident: the freesurface adapter keeps phi on the
// device between steps.
int refad_create(int precision, int resident) {
    lexer* p = refh::lex();
    G_LS = new levelset_RK3_gpu(p, refh::fd(), refh::gc(), precision, resident != 0);
    G_CONV = new weno_hj_gpu(p, precision);
    G_DISC = new reinidisc_gpu(p, precision);
    G_REINI = new reini_RK3_gpu(p, precision);
    return 0;
}

// The slab-domain free-surface adapter with nslabs slabs on the current GPU.
int refad_create_domain(int precision, int nslabs) {
    G_LSD = new levelset_RK3_domain(refh::lex(), refh::fd(), refh::gc(), nslabs, nullptr, precision);
    return 0;
}
// freesurface::start of levelset_RK3_domain on a->phi.
int refad_step_domain() {
    G_LSD->start(refh::fd(), refh::lex(), nullptr, nullptr, refh::gc(), refh::flow(), nullptr, nullptr,
                 refh::fd()->phi);
    return 0;
}
void refad_destroy() {
    delete G_LSD;
    G_LSD = nullptr;
    delete G_LS;
    delete G_CONV;
    delete G_DISC;
    delete G_REINI;
    G_LS = nullptr;
    G_CONV = nullptr;
    G_DISC = nullptr;
    G_REINI = nullptr;
}

// freesurface::start on a->phi with the harness's dt (levelset_RK3_gpu).
int refad_step() {
    G_LS->start(refh::fd(), refh::lex(), nullptr, nullptr, refh::gc(), refh::flow(), nullptr, nullptr,
                refh::fd()->phi);
    return 0;
}

// freesurface::update (the density/viscosity update on a->phi).
int refad_update() {
    G_LS->update(refh::lex(), refh::fd(), refh::gc(), refh::fd()->phi);
    return 0;
}

// L = convection operator of `src` accumulated on a zeroed a->L, as
// refls_weno_L does with weno_hj_df_nug.
int refad_weno_L(const double* src, double* L) {
    fdm* a = refh::fd();
    field4* t = refh::tmp();
    std::memcpy(t->V, src, sizeof(double) * ncell());
    for (long n = 0; n < ncell(); ++n) a->L.V[n] = 0.0;
    G_CONV->start(refh::lex(), a, *t, 4, a->u, a->v, a->w);
    std::memcpy(L, a->L.V, sizeof(double) * ncell());
    return 0;
}

// L = reinitialisation operator of `src` (reinidisc_gpu).
int refad_reinidisc_L(const double* src, double* L) {
    fdm* a = refh::fd();
    field4* t = refh::tmp();
    std::memcpy(t->V, src, sizeof(double) * ncell());
    for (long n = 0; n < ncell(); ++n) a->L.V[n] = 0.0;
    G_DISC->start(refh::lex(), a, refh::gc(), *t, a->L, 4);
    std::memcpy(L, a->L.V, sizeof(double) * ncell());
    return 0;
}

// reini::start on a->phi (reini_RK3_gpu).
int refad_reini() {
    G_REINI->start(refh::fd(), refh::lex(), refh::fd()->phi, refh::gc(), refh::flow());
    return 0;
}

}  // extern "C"
