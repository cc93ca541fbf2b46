/* CPU restatement of REEF3D's level-set transport path (WENO5-HJ convection
 * in TVD-RK3 stages, PDE reinitialisation, wall ghost fill, CFL and volume
 * reductions).
 *
 * TEST INFRASTRUCTURE ONLY.  Tests, the smoke check and the CPU-baseline leg
 * of the benchmark call it as the checker; the shipped library never links,
 * loads or calls it.
 *
 * Parity is pinned against the reference's own code compiled in
 * oracle/_ref (ref_harness.cpp) through golden vectors in tests/golden/.
 *
 * Layout: the reference's padded field layout (src/field_base.h:32-47):
 * margin 3 on every side (also the degenerate y axis of a 2D grid),
 * index (i+3)*jmax*kmax + (j+3)*kmax + (k+3), k contiguous.  1D metric
 * arrays are indexed like the reference's (offset marge=5,
 * src/iterators1D.h:25-60).  Unlike the reference it is re-entrant: all
 * state lives in lso_grid.
 */
#ifndef LS_ORACLE_H
#define LS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define LSO_MARGIN 3
#define LSO_MARGE 5

typedef struct {
    int nx, ny, nz;     /* interior cells; ny == 1 selects the 2D (x-z) form */
    int jdir;           /* 0 for 2D, 1 for 3D (src/read_grid.cpp:253-258) */
    int imax, jmax, kmax;
    long ncell;         /* imax*jmax*kmax */
    /* control flags (src/ini.cpp:400-416) */
    double f43, f45, n47;
    int f44, f49;
    int f46, f47;       /* picard mass correction (0 off, 1 in reinit, 2 in the step, 3 picard_lsm) */
    int count;          /* steps taken (lexer::count of the first step is 1) */
    double netvol;      /* picard_lsm target volume */
    /* metrics, length n+1+4*marge like the reference (src/grid.cpp:55-100) */
    double *xn, *yn, *zn, *xp, *yp, *zp;
    double *dxn, *dyn, *dzn, *dxp, *dyp, *dzp;
    double dxm, dym, dzm;  /* DIVEMesh header means (first node spacing) */
    double dxm_mean;       /* grid::gridspacing mean spacing (src/grid.cpp:102-148) */
    double psi;            /* src/ini_psi.cpp:33-37 */
    /* WENO node tables per axis (uf=0): qf[n][6][2], cf[n][6], isf[n][6][3],
     * n = cells+8, built like src/weno_nug_func_precalc_*.cpp */
    double *qf[3], *cf[3], *isf[3];
    /* inflow (x-min, boundary type 1) / outflow (x-max, type 2) faces and
     * ioflow_f's level-set flags (src/ioflow_waterlevel.cpp); io_on == 0 is
     * the closed box with ioflow_v (every hook void) */
    int io_on, io_in, io_out, f50, b77, f64;
    double f56, f60, f61, f62, qi, qo;
    double phimean, phiout;  /* water levels of the last fsfinflow */
    /* direct-forcing convection stencils (X45, src/weno_hj_df_nug.cpp:398-987):
     * body1 = fb (X45 1), fbh5 (2, 4), fbh4 (3, 6) or solid (5), body2 = topo
     * (5); caller-owned padded fields */
    int x45;
    const double *body1, *body2;
    /* solid forcing after each convection stage (X48 = 1): nsf entries
     * (i, j, k, side), caller-owned */
    int nsf;
    const int* sf;
    /* the inflow / outflow faces belong to iowave (B90 = 1): fsfinflow
     * imposes nothing, fsfrkin / fsfrkout copy phi's ghosts */
    int io_waves;
    /* relaxation zones (iowave::phi_relax): per interior column i*ny + j
     * the generation / beach weight, < 0 outside; the generation targets
     * (LOOP order over the zone), the ramp, the still water level;
     * caller-owned */
    const double *rz_wg, *rz_wb, *rz_lsval;
    double rz_ramp, rz_phimean;
} lso_grid;

/* xn/yn/zn: node coordinates for indices -5..n+5 (n+11 values). */
int lso_grid_init(lso_grid* g, int nx, int ny, int nz, const double* xn, const double* yn,
                  const double* zn, double f43, int f44, double f45, int f49, double n47);
void lso_grid_free(lso_grid* g);
long lso_index(const lso_grid* g, int i, int j, int k);

/* L = -u.grad(phi) by WENO5-HJ on interior cells (others untouched), the
 * operator levelset_RK3 accumulates into a zeroed L. */
void lso_weno_L(const lso_grid* g, const double* phi, const double* u, const double* v,
                const double* w, double* L);
/* L of the reinitialisation equation on interior cells (F49 selects the
 * form); L is zeroed on interior cells first. */
void lso_reinidisc_L(const lso_grid* g, const double* f, double* L);
/* Neumann copy of the wall cells into the three face ghost layers. */
void lso_ghost_fill(const lso_grid* g, double* f);
/* F44 reinit pseudo-steps (3 RK stages each) on f in place; a1, a2, L work. */
void lso_reini(const lso_grid* g, double* f, double* a1, double* a2, double* L, int iters);
/* One physical step: 3 convection RK stages, then F44 reinit steps.
 * a1, a2, L are work fields of ncell doubles. */
void lso_ls_step(lso_grid* g, double* phi, const double* u, const double* v,
                 const double* w, double dt, double* a1, double* a2, double* L);
/* Smoothed-Heaviside volume sums (volume1, volume2) over interior cells. */
void lso_volume(const lso_grid* g, const double* phi, double* vol1, double* vol2);
/* Next time step from the velocity maxima (src/ietimestep.cpp:38-188 with a
 * prescribed velocity: no source term, no turbulence). */
double lso_cfl_dt(const lso_grid* g, const double* u, const double* v, const double* w);

/* src/fluid_update_fsf.cpp:39-104: ro/visc with wall ghosts (w1..w4 = W1..W4). */
void lso_fluid(const lso_grid* g, const double* phi, double* ro, double* visc, double w1, double w2, double w3,
               double w4);

/* Picard mass correction flags (src/picard_f.cpp, src/picard_lsm.cpp): f46 1, 2 or 3,
 * f47 iterations.  Resets the step count. */
void lso_set_picard(lso_grid* g, int f46, int f47);

/* Inflow / outflow faces with ioflow_f's hooks (B60 >= 1): fsfinflow at the
 * start of each step, fsfrkin/fsfrkout on the RK buffers of the step and of
 * each reinitialisation, and the ghost rule of gcval 50+f50 on those faces
 * (src/gc_epol4.cpp:26-58).  qi, qo: discharges of picard_lsm's netvol. */
void lso_set_ioflow(lso_grid* g, int inflow, int outflow, int f50, int b77, double f56, double f60, double f61,
                    double f62, int f64, double qi, double qo);
/* out[0] = phimean, out[1] = phiout of the last step */
void lso_io_levels(const lso_grid* g, double* out);
/* lexer::count the next step runs as minus one (the step increments it) */
void lso_set_count(lso_grid* g, int count);

/* X45 direct-forcing variant of the convection stencils and the body
 * fields it reads (kept by pointer). */
void lso_set_direct_forcing(lso_grid* g, int x45, const double* body1, const double* body2);

/* solid_forcing_lsm entries (src/gc_solid_forcing_lsm.cpp:27-78), kept by pointer */
void lso_set_solid_forcing(lso_grid* g, int n, const int* cells);

/* The faces of lso_set_ioflow owned by iowave instead of ioflow_f. */
void lso_set_io_waves(lso_grid* g, int on);
/* iowave::phi_relax after every convection stage (src/iowave_relax.cpp:346-378):
 * weights per column (kept by pointer; NULL: no zone), still water level. */
void lso_set_relaxation(lso_grid* g, const double* wg, const double* wb, double phimean);
/* the generation targets of the next step (kept by pointer) and its ramp */
void lso_set_relaxation_target(lso_grid* g, const double* lsval, double ramp);

/* opaque handle helpers (used through ctypes) */
lso_grid* lso_new(int nx, int ny, int nz, const double* xn, const double* yn, const double* zn,
                  double f43, int f44, double f45, int f49, double n47);
void lso_delete(lso_grid* g);
long lso_ncell(const lso_grid* g);
double lso_psi(const lso_grid* g);
double lso_dxm(const lso_grid* g);
int lso_get_metric(const lso_grid* g, int which, double* dst, int n);
int lso_get_weno_tables(const lso_grid* g, int axis, double* qf, double* cf, double* isf, int n);

#ifdef __cplusplus
}
#endif
#endif
