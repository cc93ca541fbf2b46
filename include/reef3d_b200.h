/* reef3d_b200 -- B200-native level-set transport for REEF3D.
 *
 * C-ABI of the shared library libreef3d_b200.so.  Plain pointers and sizes
 * only; every entry point returns an int status (R3D_OK on success) and
 * never throws.  The text of the last error of a handle is available from
 * r3d_last_error(); errors raised before a handle exists go to the
 * thread's last error, r3d_last_error(NULL).
 *
 * One handle = one level-set instance (one grid) whose fields live in device
 * memory of the GPU current at creation.  Calls on one handle are not
 * thread-safe; distinct handles may be used from distinct threads.
 *
 * Each entry point names the reference interface it replaces (paths are
 * relative to the REEF3D source tree).
 */
#ifndef REEF3D_B200_H
#define REEF3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define R3D_OK 0
#define R3D_EINVAL 1     /* bad argument (size, id, layout, null pointer) */
#define R3D_ENOMEM 2     /* device or host allocation failed / over budget */
#define R3D_EDEVICE 3    /* CUDA runtime error */
#define R3D_ETIMEOUT 4   /* a bounded device wait gave up */
#define R3D_ESTATE 5     /* call not valid in the handle's current state */

/* arithmetic of an instance */
#define R3D_FP64 0       /* plain FP64: same operations and order as the reference */
#define R3D_FP32 1       /* FP32 stencils and RK stages, FP64 reductions */

/* field ids (the fdm members the path reads and writes, src/fdm.h) */
#define R3D_PHI 0        /* a->phi, level set (cell centres) */
#define R3D_U 1          /* a->u, x velocity on x faces (i+1/2) */
#define R3D_V 2          /* a->v, y velocity on y faces */
#define R3D_W 3          /* a->w, z velocity on z faces */
#define R3D_L 4          /* a->L, right-hand side of the last operator call */
#define R3D_WORK1 5      /* RK stage buffer (ark1 / frk1) */
#define R3D_WORK2 6      /* RK stage buffer (ark2 / frk2) */
#define R3D_RO 7         /* a->ro, density (exists once r3d_set_fluid enabled it) */
#define R3D_VISC 8       /* a->visc, kinematic viscosity (likewise) */
#define R3D_BODY 9       /* body field of the direct-forcing stencils (exists once
                            r3d_set_direct_forcing enabled them) */

/* host array layouts for upload/download */
#define R3D_LAYOUT_REEF3D 0  /* the reference's padded field: (nx+6)(ny+6)(nz+6) doubles,
                                index (i+3)(ny+6)(nz+6)+(j+3)(nz+6)+(k+3), k contiguous
                                (src/field_base.h:32-47); 2D grids keep the 6 y ghost planes */
#define R3D_LAYOUT_DENSE 1   /* interior cells only, nx*ny*nz doubles, x contiguous:
                                index i + nx*(j + ny*k) */

typedef struct r3d_handle r3d_handle;

/* Grid and control flags of one instance.  Node coordinates follow the
 * DIVEMesh grid the reference reads (src/read_grid.cpp:417-433): n+11 values
 * for node indices -5..n+5.  ny == 1 selects the 2D x-z form (j_dir = 0).
 * Flags carry the reference's control-file meaning (src/ini.cpp:400-416,
 * 587-596): f43 reinit time-step factor, f44 reinit pseudo-steps per
 * physical step, f45 interface thickness factor, f49 reinit form (1 every
 * cell, 0 freeze cells next to the interface), n47 CFL factor, f46 picard
 * mass correction (0 off; 1 picard_f around each reinitialisation as
 * reini_RK3 does, src/reini_RK3.cpp:65-69; 2 picard_f around each step as
 * levelset_RK3 does, src/levelset_RK3.cpp:84-91; 3 picard_lsm there, whose
 * target is the volume of the instance's first step, src/picard_lsm.cpp,
 * with no inflow or outflow), f47 picard iterations.
 * f46/f47 come last so that a zero-initialised descriptor leaves the
 * correction off. */
typedef struct {
    int nx, ny, nz;
    const double* xn;
    const double* yn;
    const double* zn;
    double f43;
    int f44;
    double f45;
    int f49;
    double n47;
    int precision;      /* R3D_FP64 or R3D_FP32 */
    int f46;            /* 0, 1 or 2 */
    int f47;            /* >= 0 */
} r3d_grid_desc;

/* Create an instance on the current CUDA device: allocates the level set,
 * two stage buffers, L, the three velocity fields and reduction scratch,
 * builds the grid metrics and WENO coefficient tables the way
 * src/grid.cpp:55-148 and src/weno_nug_func_precalc_*.cpp do, and zeroes
 * every field.  Replaces the construction of levelset_RK3, weno_hj_df_nug
 * and reini_RK3 (src/driver_logic_cfd.cpp:145-146,377-385). */
int r3d_create(const r3d_grid_desc* desc, r3d_handle** out);
int r3d_destroy(r3d_handle* h);
const char* r3d_last_error(const r3d_handle* h);

/* Device bytes an instance of this description holds (for admission). */
int r3d_footprint(const r3d_grid_desc* desc, size_t* bytes);

/* Host <-> device field copies (explicit copy-in/copy-out of the
 * reference's field objects, src/field_base.h:28-54).  Synchronous. */
int r3d_upload(r3d_handle* h, int field, const double* host, int layout);
int r3d_download(r3d_handle* h, int field, double* host, int layout);

/* Time step used by r3d_ls_step when dt <= 0 is passed there. */
int r3d_set_dt(r3d_handle* h, double dt);
/* Adaptive time step from the stored velocities, FP64 on the device:
 * src/ietimestep.cpp:38-206 for a prescribed velocity (N50=1, no source
 * term).  Stores it as the handle's dt and returns it in *dt (may be NULL). */
int r3d_cfl_dt(r3d_handle* h, double* dt);

/* One physical level-set step: three WENO5-HJ convection RK stages with
 * ghost fill, then f44 reinitialisation pseudo-steps, then the volume
 * integral.  Replaces levelset_RK3::start (src/levelset_RK3.cpp:103-172)
 * with particles, ioflow hooks and solid forcing void, as in the
 * reference's default configuration; the picard mass correction runs as
 * the descriptor's f46 selects (the volume integral then follows the
 * correction, as fluid_update_fsf follows correct_ls at :171-174).
 * dt <= 0 uses the handle's dt.
 * Asynchronous on the handle's stream. */
int r3d_ls_step(r3d_handle* h, double dt);
/* n steps, each preceded by r3d_cfl_dt when adaptive != 0 (the timestep
 * control of src/driver_loop_cfd.cpp:104-105), all on the device. */
int r3d_ls_run(r3d_handle* h, int nsteps, int adaptive);

/* Reinitialisation only: `iters` pseudo-steps on the level set
 * (reini_RK3::start, src/reini_RK3.cpp:84-143; iters <= 0 uses f44), inside
 * the picard volume/correction when f46 == 1 (:92, :140). */
int r3d_reinit(r3d_handle* h, int iters);

/* Operator-level drop-ins on device fields:
 *  r3d_convection_L: L(field_in) = -u.grad(field_in) by WENO5-HJ, written
 *    to R3D_L (convection::start with ipol 4 on a zeroed L,
 *    src/weno_hj_df_nug.cpp:58-111).
 *  r3d_reinidisc_L: reinitialisation operator (reinidisc::start,
 *    src/reinidisc_f.cpp:37-127 / src/reinidisc_fsf.cpp:37-141).
 *  r3d_ghost_fill: wall ghost fill of a field (ghostcell::start4 with a
 *    level-set gcv, src/gc_start.cpp:146-185). */
int r3d_convection_L(r3d_handle* h, int field_in);
int r3d_reinidisc_L(r3d_handle* h, int field_in);
int r3d_ghost_fill(r3d_handle* h, int field);

/* Writes the instance's level set (and, with the fluid update on, its
 * density and viscosity) as a VTK unstructured-grid file the way the
 * reference's printer does (printer_CFD::print_vtu, src/printer_CFD.cpp:
 * 356-727; src/vtu3D.cpp): Float32 point data "phi", "rho", "viscosity" at
 * the grid nodes with the reference's interpolations (ipol4phi, ipol4_a,
 * ipol4, src/interpolation_ipol.cpp), node coordinates, hexahedral cells,
 * appended raw data, and the device clock as TimeValue.  The point data is
 * formed on the device; the eight triple-corner ghost cells, which the
 * reference never writes, enter the corner nodes as their corner cell.
 * Synchronous. */
int r3d_write_vtu(r3d_handle* h, const char* path);

/* Checkpoint and resume of an instance (the role of the reference's state
 * files, src/cfd_state_write.cpp / cfd_state_read.cpp, for the fields this
 * library holds): r3d_save_state writes every device field (level set,
 * stage buffers, velocities, and ro, visc, body when enabled) in the
 * instance's own precision, bit for bit, with the device scalars a step
 * reads (dt, clock, velocity factor, picard and inflow/outflow state);
 * r3d_load_state restores them into an instance created from the same grid
 * description and configured the same way (fluid update, direct forcing,
 * inflow/outflow), so that a resumed run continues exactly as the
 * uninterrupted one.  Unlike the reference's state files (single precision)
 * nothing is rounded.  Synchronous. */
int r3d_save_state(r3d_handle* h, const char* path);
int r3d_load_state(r3d_handle* h, const char* path);

/* The reference's restart state file, so that a REEF3D run restarts from a
 * state this library wrote and the reverse: replaces cfd_state::write
 * (src/cfd_state.cpp:201-220 -> write_result, src/cfd_state_write.cpp:34-146)
 * and cfd_state::read (src/cfd_state_read.cpp:44-195) for a single rank.
 * The file holds the header below and single-precision blocks in the
 * reference's loop order: topo, u, v, w, press, phi, kin, eps, eddyv, the
 * bed-load slice qbe, conc (u, v, w without the far wall face, ulast =
 * vlast = wlast = 1; no v block on a 2D grid; every cell fluid).  The level
 * set and the velocities come from / go to the instance; the other fields
 * from / to `extra` (7 pointers in the order topo, press, kin, eps, eddyv,
 * qbe, conc: dense x-contiguous arrays, qbe nx*ny; a NULL array, or a NULL
 * `extra`, writes zeros / skips the field).  The reference names the file
 * REEF3D_CFD_STATE/REEF3D-CFD-State-<num %08d>-<rank+1 %06d>.r3d.  Reading
 * keeps the instance's values where the file has none (ghost cells, the far
 * wall faces), then refills the level set's ghost cells (ghostcell::start4,
 * as the reference does).  Synchronous. */
typedef struct r3d_state_info {
    int count;       /* p->count, the step number */
    int printcount;  /* p->printcount */
    double simtime, printtime, sedprinttime, fsfprinttime, probeprinttime, stateprinttime;
} r3d_state_info;
int r3d_write_reef3d_state(r3d_handle* h, const char* path, const r3d_state_info* info,
                           const double* const* extra);
int r3d_read_reef3d_state(r3d_handle* h, const char* path, r3d_state_info* info, double* const* extra);

/* Volume sums of the smoothed Heaviside (fluid_update_fsf::start,
 * src/fluid_update_fsf.cpp:39-74), FP64.  Synchronous. */
int r3d_volume(r3d_handle* h, double* volume1, double* volume2);

/* Density and viscosity update of fluid_update_fsf (src/fluid_update_fsf.cpp:
 * 39-104): allocates R3D_RO and R3D_VISC and from then on ends every step
 * with ro = ro_water H + ro_air (1-H), visc = visc_water H + visc_air (1-H)
 * of the smoothed Heaviside H(phi; psi) on the interior, their wall ghost
 * layers (a Neumann copy, gcval 1) and the volume sums -- the call
 * levelset_RK3::start makes after the reinitialisation (src/levelset_RK3.cpp:
 * 174).  The reference takes the constants from W1, W2, W3, W4 (defaults
 * 998.2, 1.004e-6, 1.205, 1.41e-5, src/ini.cpp:831-834).  Synchronous.
 * Not for batch members. */
int r3d_set_fluid(r3d_handle* h, double ro_water, double visc_water, double ro_air, double visc_air);
/* The update alone on the current level set (fluid_update_fsf::start),
 * returning the volume sums; needs r3d_set_fluid.  Synchronous. */
int r3d_fluid_update(r3d_handle* h, double* volume1, double* volume2);

/* Volume sums accumulated by the last r3d_ls_step / r3d_ls_run step
 * (fused into the step's final stage, or taken after the picard correction
 * or by the fluid update when those are on).  Synchronous. */
int r3d_last_volume(r3d_handle* h, double* volume1, double* volume2);

/* Factor applied to the stored face velocities by every convection stage
 * and by r3d_cfl_dt (default 1, which leaves them bit-exact).  Lets a
 * caller advance a velocity field u(x,t) = u(x) g(t) without re-uploading
 * it; the reference multiplies the same way when it evaluates its analytic
 * benchmark velocities (src/benchmark_vortex3D.cpp:77-95). */
int r3d_set_velocity_scale(r3d_handle* h, double scale);
/* With period T > 0 the factor follows the device clock:
 * g = cos(pi t / T), recomputed after every step (0 turns it off). */
int r3d_set_velocity_period(r3d_handle* h, double period);
/* Velocity generator for wave-tank runs (no counterpart in the level-set
 * path of the reference, whose velocities come from its momentum solver):
 * before every step (and in r3d_cfl_dt) u and w are rewritten on every
 * stored cell with the linear (Airy) orbital velocity of a wave
 *   eta = amplitude cos(kw x - om t), kw = 2 pi / wavelength,
 *   om = sqrt(gravity kw tanh(kw depth)), bed at z = 0:
 *   u = a cosh(kw z') cos(kw x - om t), w = a sinh(kw z') sin(kw x - om t),
 *   a = amplitude om / sinh(kw depth), z' = min(z, depth) (above the
 *   still-water level the surface value, not the linear solution's
 *   exponential growth into the air),
 * at the device clock t (u on x faces, w on z faces); v is zeroed and the
 * velocity factor set to 1.  wavelength <= 0 turns the generator off.
 * Synchronous.  Not for batch members. */
int r3d_set_velocity_airy(r3d_handle* h, double amplitude, double wavelength, double depth, double gravity);
/* Subdomain (slab) decomposition along z, the role of the reference's MPI
 * halo exchange (ghostcell::gcparax, src/gcx_parax.cpp) for a grid split
 * into slabs of consecutive z cells, one instance per slab (per GPU, or
 * several on one GPU).  The instance's node coordinates are the slab's own
 * (zn: node indices -5..nz+5 of the slab, taken from the global grid).
 *  r3d_set_halo: zlo / zhi = 1 marks the z-min / z-max face as a subdomain
 *    boundary: no kernel writes wall copies into its three ghost planes
 *    (a neighbour's halo fills them), and with zhi the faces at nz-1 take
 *    part in the CFL maximum (wlast = 0 with a neighbour above,
 *    src/lexer_gridsize.cpp:78-79).  Not with picard (f46 != 0) or
 *    inflow/outflow faces, whose sums the reference takes globally inside
 *    the step.
 *  r3d_halo_copy: dir 0 packs the three interior z planes next to `side`
 *    (0 z-min, 1 z-max) of `field` into the device buffer buf; dir 1 unpacks
 *    buf into the three ghost planes on that side.  r3d_halo_bytes gives
 *    the buffer size (3 padded planes).  Asynchronous on the handle's
 *    stream.
 *  r3d_cfl_max: the instance's |u|, |v|, |w| face maxima of the stored
 *    velocities (the first half of ietimestep, src/ietimestep.cpp:72-88;
 *    the caller takes the maximum over subdomains, as pgc->globalmax does).
 *  r3d_cfl_dt_from_max: the time step from given maxima with this
 *    instance's smallest cell (the second half, :160-188); the minimum of
 *    it over subdomains is the undivided grid's time step, which the caller
 *    then sets with r3d_set_dt.
 * A step over subdomains is then: r3d_stage per RK stage, and after each
 * stage the stage's output field exchanged (pack on one instance, unpack
 * into its neighbour); volumes are summed over subdomains (r3d_volume). */
int r3d_set_halo(r3d_handle* h, int zlo, int zhi);
/* The grid-wide spacing constants of src/grid.cpp:102-148 (DXM, the mean
 * cell spacing over the three axes, summed over all subdomains) and of the
 * DIVEMesh header (DYM, DZM), from which the interface thickness psi
 * (src/ini_psi.cpp:33-37), the picard epsi and the X45 = 1 threshold derive.
 * r3d_grid_spacing computes them for a description (out[0..3] = DXM, DYM,
 * DZM, psi; host only); r3d_set_grid_spacing gives a subdomain instance the
 * whole grid's values in place of its own. */
int r3d_grid_spacing(const r3d_grid_desc* desc, double* out);
int r3d_set_grid_spacing(r3d_handle* h, double dxm, double dym, double dzm);
int r3d_halo_bytes(const r3d_handle* h, size_t* bytes);
int r3d_halo_copy(r3d_handle* h, int field, int side, int dir, void* buf);
int r3d_cfl_max(r3d_handle* h, double* vmax);
int r3d_cfl_dt_from_max(r3d_handle* h, const double* vmax, double* dt);

/* Direct-forcing variant of the level-set convection stencils (control
 * flag X45, src/weno_hj_df_nug.cpp:115-342 selecting :398-987): the five
 * divided differences of each WENO5 stencil are masked or weighted by a
 * body field at the two cells of each difference --
 *   X45 1: zero unless |fb| > 0.6 DXM at both cells        (body = a->fb)
 *       2: times 0.5 (fbh5 + fbh5) of the two cells         (body = a->fbh5)
 *       3: zero unless fbh4 < 0.5 at both                   (body = a->fbh4)
 *       4: times fbh5 of the upwind-most cell of the pair   (body = a->fbh5)
 *       5: zero unless solid > 0 and topo > 0 at both       (body = min(a->solid, a->topo))
 *       6: as 3, but 1e20 where masked                      (body = a->fbh4)
 * The body field is R3D_BODY, allocated (zeroed) by the first call with
 * x45 != 0 and uploaded like any field (REEF3D layout: its ghost cells are
 * read too); it is held in FP64 in both arithmetic forms, so the mask
 * decisions are the reference's.  The reinitialisation is unchanged (the
 * reference applies X45 to the convection only).  FP32 instances run the
 * one-cell-per-thread kernels; with X45 6 (masked differences 1e20, whose
 * squares pass the FP32 range) a stencil holding a masked difference gets
 * weight 0 (~1e-80 relative in the reference's FP64), and a cell whose
 * three stencils all hold one is evaluated in FP64.  0 turns it off.
 * Synchronous.  Not for batch members. */
int r3d_set_direct_forcing(r3d_handle* h, int x45);

/* Relaxation zones of REEF3D's wave generator and numerical beach on the
 * level set (iowave::phi_relax, src/iowave_relax.cpp:346-378, called by
 * levelset_RK3::start after every convection stage,
 * src/levelset_RK3.cpp:125,142,158).  w_gen[i*ny + j] is the generation
 * zone's weight relax4_wg(i,j) of column (i,j), w_beach the beach zone's
 * relax4_nb(i,j); a negative weight marks a column outside that zone
 * (iowave's distgen / distbeach >= 1e20); NULL: no such zone (B98 != 2, or
 * B99 != 2).  After each convection stage, on the columns of the zones:
 *   generation: f = (1 - w_gen) ramp lsval + w_gen f
 *   beach:      f = (1 - w_beach) (phimean - z) + w_beach f
 * with z the cell-centre height, and the relaxed values go into the wall
 * ghost layers.  Both NULL turns the zones off.  Synchronous.  Not for
 * batch members or slabs of a domain. */
int r3d_set_relaxation(r3d_handle* h, const double* w_gen, const double* w_beach, double phimean);
/* The generation zone's target level set of the coming step (iowave's
 * lsval, filled by wavegen_precalc, src/iowave_precalc_relax.cpp) in the
 * reference's LOOP order over the zone (columns i-major, j, then k), n =
 * nz x the zone's columns, and the wave generation ramp of the step
 * (iowave::ramp).  Synchronous. */
int r3d_set_relaxation_target(r3d_handle* h, const double* lsval, long long n, double ramp);

/* Solid forcing of the level set after each convection stage
 * (ghostcell::solid_forcing_lsm, src/gc_solid_forcing_lsm.cpp:27-78, called
 * at src/levelset_RK3.cpp:128,145,160 with X48 = 1): for each of the n
 * entries (i, j, k, side) of the direct-forcing boundary list gcdf4
 * (src/gcdf_update.cpp; side 1 -x, 4 +x, 3 -y, 2 +y, 5 -z, 6 +z; entries with
 * side <= 0 are skipped), in list order, the two cells beyond the side take
 * the value of cell (i, j, k).  Entries that touch the same cells keep the
 * list order (the library runs the list in dependency levels).  n = 0 turns
 * it off.  Synchronous.  Not for batch members. */
int r3d_set_solid_forcing(r3d_handle* h, int n, const int* cells);

/* Inflow and outflow boundaries with the level-set hooks of REEF3D's
 * ioflow_f (B60 >= 1, src/driver_logic_cfd.cpp:509-510), which the
 * closed box's ioflow_v leaves void.  The x-min face becomes an inflow
 * boundary (boundary type 1) and the x-max face an outflow boundary (type
 * 2); the other faces stay walls.  Per step (levelset_RK3::start,
 * src/levelset_RK3.cpp:105-109):
 *  - fsfinflow (src/ioflow_waterlevel.cpp:29-141): the inflow water level
 *    phimean from the zero crossings of phi in the first ghost column
 *    (else F56, or F60 when set) is imposed on the inflow ghosts when f50 is
 *    2 or 4; the outflow level phiout is measured the same way on the last
 *    interior column; with F62 set and B77 = 2 the outflow ghosts take the
 *    level F62 (ramped from F60 over the first F64 steps);
 *  - fsfrkin / fsfrkout (:143-177) on the RK buffers, also at the start of
 *    every reinitialisation (src/reini_RK3.cpp:107-110);
 *  - the ghost fill of the level set follows gcval 50+f50
 *    (src/gc_epol4.cpp:26-58): the inflow face is a Neumann copy for f50 2
 *    and 4 and untouched otherwise, the outflow face a Neumann copy for f50
 *    1 and 4 and for 2 with B77 = 1, untouched otherwise.
 * Values as the reference's control file gives them; "unset" is its
 * default (F56 1e20, F60/F61/F62 -1e20).  qi, qo: the discharges picard_lsm
 * adds to its target volume each step, netvol += Qi dt - Qo dt
 * (src/picard_lsm.cpp:93), which the flow solver computes.  ioflow_f's
 * phi_relax (src/ioflow_relax.cpp:49) acts only at step count 0, the
 * reference's initialisation step, and is not part of a step here.
 * Not for batch members; instances with inflow/outflow run the
 * one-cell-per-thread kernels.  NULL restores the closed box.  Synchronous. */
typedef struct {
    int inflow;         /* 1: x-min face is an inflow boundary, 0: wall */
    int outflow;        /* 1: x-max face is an outflow boundary, 0: wall */
    int f50;            /* 1..4, level-set ghost rule gcval 50+f50 (src/levelset_RK3.cpp:50-60) */
    int b77;            /* 1 or 2: outflow pressure-controlled / fixed water level */
    double f56, f60, f61, f62;
    int f64;            /* >= 0 */
    double qi, qo;
} r3d_ioflow_desc;
int r3d_set_ioflow(r3d_handle* h, const r3d_ioflow_desc* io);
/* The same faces owned by REEF3D's wave generator iowave (B90 >= 1) instead
 * of ioflow_f: the ghost labels of gcval 50+F50 as above, while
 * iowave::fsfinflow imposes no ghosts (src/iowave_waterlevel.cpp:29-35,
 * without flow-file input or patch boundaries) and fsfrkin / fsfrkout copy
 * the level set's ghost layers at the faces into both stage buffers
 * (:37-63).  F56 .. F64, qi, qo are not read; r3d_io_levels reports
 * nothing measured.  Pair with r3d_set_relaxation. */
int r3d_set_ioflow_waves(r3d_handle* h, const r3d_ioflow_desc* io);
/* Water levels phimean and phiout of the last step's fsfinflow (both may be
 * NULL).  Synchronous. */
int r3d_io_levels(r3d_handle* h, double* phimean, double* phiout);
/* lexer::count of the next step (default: 1 for the first step of the
 * instance).  The outflow ramp (F64) and picard_lsm's first-step target
 * read it. */
int r3d_set_step_count(r3d_handle* h, long long count);

/* Device clock (the reference's p->simtime, advanced by dt every step,
 * src/driver_loop_cfd.cpp:104). */
int r3d_set_time(r3d_handle* h, double t);
int r3d_get_time(r3d_handle* h, double* t);

/* One fused RK stage on the device fields (stage 1..3): the convection
 * stages of src/levelset_RK3.cpp:112-159 (phi -> WORK1 -> WORK2 -> phi) or
 * the reinitialisation stages of src/reini_RK3.cpp:113-137, each with its
 * wall ghost fill.  Used to time and test a single stage. */
#define R3D_STAGE_CONVECTION 0
#define R3D_STAGE_REINIT 1
int r3d_stage(r3d_handle* h, int kind, int stage);

/* Device-side initial fields of the ensemble and serving workloads (the role
 * of the reference's analytic benchmark setups, src/benchmark_*.cpp):
 * phi = union of nspheres signed-distance spheres (circles in the x-z plane
 * for 2D grids), spheres[4q..4q+3] = centre x, y, z and radius; the stored
 * velocities = sum of nmodes Taylor-Green modes, modes[2q] = integer
 * wavenumber k, modes[2q+1] = amplitude A:
 *   u = A sin(k pi x) cos(k pi y) cos(k pi z), v = -A cos(k pi x) sin(k pi y) cos(k pi z), w = 0
 *   (2D: u = A sin(k pi x) cos(k pi z), w = -A cos(k pi x) sin(k pi z)),
 * evaluated on every stored cell at the staggered positions.  Synchronous. */
int r3d_init_spheres_tg(r3d_handle* h, int nspheres, const double* spheres, int nmodes, const double* modes);

/* Execution options of an instance (no effect on results beyond the
 * rounding of the FP32 form):
 *  R3D_OPT_TILED  1 = TMA-tiled FP32x2 stage kernels on 3D uniform FP32
 *                 grids (default), 0 = one-cell-per-thread kernels;
 *                 reading it returns whether the tiled path is in use.
 *  R3D_OPT_CHUNK  z-planes per CTA of the tiled kernels (default 16); sets
 *                 both stage kinds, R3D_OPT_CHUNK_REINIT then sets the
 *                 reinitialisation stages' alone (reading CHUNK returns the
 *                 convection stages' value).
 *  R3D_OPT_BAND64 1 = FP64 re-anchoring of interface-band cells in the FP32
 *                 reinitialisation (default), 0 = FP32 everywhere.
 *  R3D_OPT_WAIT_TEST  diagnostic for the bounded waits of the tiled kernels:
 *                 1 makes every CTA of the next r3d_ls_step wait (with a
 *                 short limit) for a copy that is never issued, so the
 *                 kernels take their timeout path -- raise the error flag,
 *                 wait for their own copies, return -- and the next
 *                 r3d_sync reports R3D_ETIMEOUT; the instance stays usable.
 *                 Cleared by that step.  No effect off the tiled path.
 *  R3D_OPT_TILE_CFG  tile configuration of the tiled kernels, 0 ..
 *                 r3d_tile_config_count()-1 (r3d_tile_config_describe: tile
 *                 shape, rows per thread, ring depth); the level set is the
 *                 same under every configuration.  Sets both stage kinds;
 *                 R3D_OPT_TILE_CFG_REINIT then sets the reinitialisation
 *                 stages' alone.  r3d_autotune picks both with the chunks. */
#define R3D_OPT_TILED 0
#define R3D_OPT_CHUNK 1
#define R3D_OPT_BAND64 2
#define R3D_OPT_WAIT_TEST 3
#define R3D_OPT_TILE_CFG 4
#define R3D_OPT_TILE_CFG_REINIT 6
#define R3D_OPT_CHUNK_REINIT 7
int r3d_set_option(r3d_handle* h, int option, int value);
int r3d_get_option(r3d_handle* h, int option, int* value);

/* Tile configurations of the tiled kernels: how many there are, and for
 * id cfg the tile (tx x ty cells per CTA), rows per thread, plane slots of
 * the shared-memory ring and threads per CTA (R3D_EINVAL for a bad id). */
int r3d_tile_config_count(void);
int r3d_tile_config_describe(int cfg, int* tx, int* ty, int* rows_per_thread, int* ring, int* threads);
/* The z chunks (planes per CTA work item) the autotuners try: writes up to
 * max of them to out and returns how many there are. */
int r3d_tile_chunk_candidates(int* out, int max);
/* Picks the instance's tile configuration and z chunk, for the convection
 * and the reinitialisation stages separately, by timing stages 1 and 2 of
 * each kind under every candidate (the level set is untouched: those stages
 * write only the stage buffers), and caches the choice per grid size, in
 * memory and in cache_path (may be NULL; the file r3d_batch_autotune
 * uses).  cfg/chunk receive the convection stages' choice (the
 * reinitialisation stages': R3D_OPT_TILE_CFG_REINIT, R3D_OPT_CHUNK_REINIT).
 * No effect (and no timing) off the tiled path.  Synchronous. */
int r3d_autotune(r3d_handle* h, const char* cache_path, int* cfg, int* chunk);

/* Wait for the handle's stream; R3D_ETIMEOUT if a bounded device wait of a
 * kernel gave up since the last check. */
int r3d_sync(r3d_handle* h);
/* The handle's cudaStream_t, as void*. */
int r3d_stream(r3d_handle* h, void** stream);
/* Kernel launches issued on this handle since creation. */
int r3d_launch_count(const r3d_handle* h, long long* count);

/* Volume sums of a level set, allocating nothing (no counterpart in the
 * reference: it is a variant of r3d_volume for callers that cannot allocate
 * device memory at the time of the call -- a host code that has handed all
 * of the GPU's memory to its own pool, or a time loop that must not take
 * cudaMalloc's implicit device synchronisation).  phi: device array of
 * nx*ny*nz doubles, dense x-contiguous layout (R3D_LAYOUT_DENSE); dx, dy,
 * dz: uniform cell sizes; psi: interface half-thickness; out: device array
 * of 2 doubles receiving volume1 and volume2 (the smoothed-Heaviside sums of
 * src/fluid_update_fsf.cpp:50-74).  Asynchronous on `stream` (a
 * cudaStream_t, NULL for the default stream).
 * Its scratch is a fixed 1 MiB device array inside the library, kept by
 * every GPU that loads it until the process exits: at most ny*nz = 65536
 * rows (R3D_EINVAL beyond).  All calls share that array, so calls whose
 * kernels may overlap on one GPU race and must be ordered by the caller.
 * The first call on a device looks up the array's device address (once per
 * device); make that first call before any stream capture.
 * Errors: r3d_last_error(NULL). */
int r3d_volume_dense_noalloc(const double* phi, int nx, int ny, int nz, double dx, double dy, double dz,
                             double psi, double* out, void* stream);

/* ---------------------------------------------------------------- batches
 * Many FP32 instances of uneven sizes (2D and 3D mixed) advanced together:
 * one persistent launch per RK stage over a packed tile list of all members,
 * the whole step captured in a CUDA graph.  The reference has no
 * counterpart (it runs one grid per process, src/weno_nug_func.h:198-202);
 * each member's step is levelset_RK3::start (src/levelset_RK3.cpp:103-172)
 * with its own CFL time step (src/ietimestep.cpp:38-206), clock and volume.
 * A member's results do not depend on the other members.  While an
 * instance is a member, calls on its handle first wait for the batch.
 * Members are FP32 instances with f46 = 0 (no picard mass correction),
 * without the fluid update and without the Airy velocity generator. */
typedef struct r3d_batch r3d_batch;
int r3d_batch_create(r3d_batch** out);
int r3d_batch_destroy(r3d_batch* b);
const char* r3d_batch_last_error(const r3d_batch* b);
int r3d_batch_add(r3d_batch* b, r3d_handle* h);
int r3d_batch_remove(r3d_batch* b, r3d_handle* h);
int r3d_batch_size(const r3d_batch* b, int* n);
/* Members on the one-cell-per-thread kernels (2D, stretched): tile rows
 * (2, 4, 8: tiles of 32 x rows cells, 32*rows threads) and persistent CTAs
 * per SM. */
int r3d_batch_set_config(r3d_batch* b, int rows, int ctas_per_sm);
int r3d_batch_get_config(const r3d_batch* b, int* rows, int* ctas_per_sm);
/* Members on the tiled kernels (3D uniform FP32): tile configuration (as
 * R3D_OPT_TILE_CFG) and z chunk of the batch's persistent launches. */
int r3d_batch_set_tile_config(r3d_batch* b, int cfg, int chunk);
int r3d_batch_get_tile_config(const r3d_batch* b, int* cfg, int* chunk);
/* Times the candidate configurations on the batch (state-preserving): tile
 * configuration x z chunk of the tiled members, then rows x CTAs per SM of
 * the others; caches the best per size class, in memory and in cache_path
 * (may be NULL); a cached class is reused without timing. */
int r3d_batch_autotune(r3d_batch* b, const char* cache_path, int* rows, int* ctas_per_sm);
int r3d_batch_use_graph(r3d_batch* b, int on);
/* nsteps adaptive steps of every member; asynchronous on the batch stream. */
int r3d_batch_step(r3d_batch* b, int nsteps);
int r3d_batch_sync(r3d_batch* b);
int r3d_batch_stream(r3d_batch* b, void** stream);
int r3d_batch_launch_count(const r3d_batch* b, long long* count);

/* One grid split along z into nslabs slabs -- on the current device, or
 * slab r on devices[r] -- and stepped as one (the role of the reference's
 * MPI decomposition with
 * ghostcell::gcparax, src/gcx_parax.cpp, for z splits): each slab is an
 * instance with halo faces towards its neighbours (r3d_set_halo) and the
 * whole grid's spacing constants; a step runs every RK stage on all slabs,
 * each on its own stream, then moves the three halo planes between
 * neighbours by peer copies (over NVLink between GPUs), then the next
 * stage; the adaptive time step takes the maxima over all slabs
 * (pgc->globalmax) at the grid's smallest cell.  The step is captured in one
 * CUDA graph.  The level set, dt and clock equal the
 * undivided grid's; the volume sums are taken per slab and added.
 * r3d_domain_upload / download take the whole grid in the reference's
 * layout.  r3d_domain_run: nsteps steps with time step dt, or adaptive ones
 * when dt <= 0; synchronous.  The picard correction the descriptor selects
 * (f46, f47) runs over the whole grid: each volume summed per slab, the
 * slabs' shares added on slab 0's device (pgc->globalsum), w written back to
 * every slab, the phi halos exchanged after the last shift.
 * r3d_domain_set_ioflow opens inflow/outflow faces on every slab
 * (r3d_set_ioflow's faces; nullptr closes them): the water levels come from
 * the crossing heights of all slabs gathered in the whole grid's order, so
 * they equal the undivided grid's; the step count is slab 0's
 * (r3d_set_step_count through r3d_domain_slab).  r3d_domain_set_fluid
 * turns on the density/viscosity update on every slab (its ro, visc halos
 * exchanged too); the slabs' own settings (velocity generator, X45
 * stencils, solid forcing) apply, set through r3d_domain_slab.  One process per GPU runs the same
 * decomposition with reef3d_b200.slab.DistSlab (NCCL). */
typedef struct r3d_domain r3d_domain;
int r3d_domain_create(const r3d_grid_desc* desc, int nslabs, const int* devices, r3d_domain** out);
int r3d_domain_destroy(r3d_domain* d);
const char* r3d_domain_last_error(const r3d_domain* d);
int r3d_domain_slab(r3d_domain* d, int s, r3d_handle** h, int* k0, int* k1);
int r3d_domain_upload(r3d_domain* d, int field, const double* host);
int r3d_domain_download(r3d_domain* d, int field, double* host);
int r3d_domain_run(r3d_domain* d, int nsteps, double dt);
int r3d_domain_last_volume(r3d_domain* d, double* volume1, double* volume2);
int r3d_domain_get_dt(r3d_domain* d, double* dt);
int r3d_domain_set_ioflow(r3d_domain* d, const r3d_ioflow_desc* io);
int r3d_domain_set_fluid(r3d_domain* d, double ro_water, double visc_water, double ro_air, double visc_air);
/* The density/viscosity update alone on the current level set of every slab
 * (fluid_update_fsf::start), with the ro, visc halos; volume sums added. */
int r3d_domain_fluid_update(r3d_domain* d, double* volume1, double* volume2);

/* Continuous-batching job server (no counterpart in the reference, which
 * runs one case per process).  A job is a level set on a uniform grid of the
 * unit box made of nspheres spheres (spheres[4q..4q+3] = centre x, y, z,
 * radius) advected by nmodes Taylor-Green modes (modes[2q] = wavenumber,
 * modes[2q+1] = amplitude; r3d_init_spheres_tg) for `steps` adaptive steps
 * with f44 reinitialisation pseudo-steps and CFL factor n47 (f43 0.5, f45
 * 2.1, f49 1).  Submitted jobs wait in arrival order until their device
 * footprint (r3d_footprint) fits the HBM budget; admitted jobs stay
 * resident and advance together between polls -- FP32 jobs as members of
 * one batch (one persistent launch per RK stage over all members, CUDA
 * graph), FP64 jobs each on its own instance -- and leave when done.  A
 * job's results do not depend on which jobs shared its steps.
 *  r3d_serve_poll: admits what fits, then advances every active job by up
 *    to max_steps steps, stopping at the first job to finish (which is
 *    retired: volume sums and clock recorded, instance destroyed unless the
 *    server keeps fields); *nfinished = jobs retired by this call.
 *  r3d_serve_result: state (0 queued, 1 active, 2 finished, 3 released),
 *    times on the server's clock (seconds since creation; -1 not yet), and
 *    with keep_fields the finished job's instance (read its fields, then
 *    r3d_serve_release). */
typedef struct r3d_server r3d_server;
typedef struct {
    int nx, ny, nz;
    int steps;
    int f44;
    double n47;
    int nspheres;
    const double* spheres;
    int nmodes;
    const double* modes;
} r3d_job_desc;
typedef struct {
    int state;
    int steps_done;
    double volume1, volume2;
    double sim_time;
    double t_submit, t_admit, t_done;
    r3d_handle* instance;
} r3d_job_result;
int r3d_serve_create(double budget_bytes, int precision, int keep_fields, r3d_server** out);
int r3d_serve_destroy(r3d_server* s);
const char* r3d_serve_last_error(const r3d_server* s);
int r3d_serve_submit(r3d_server* s, const r3d_job_desc* job, long long* id);
int r3d_serve_poll(r3d_server* s, int max_steps, int* nfinished);
int r3d_serve_status(const r3d_server* s, int* queued, int* active, double* used_bytes, double* peak_bytes,
                     int* max_active);
int r3d_serve_result(const r3d_server* s, long long id, r3d_job_result* out);
int r3d_serve_release(r3d_server* s, long long id);
/* The FP32 server's batch (for r3d_batch_autotune / r3d_batch_set_config);
 * NULL for an FP64 server. */
int r3d_serve_batch(r3d_server* s, r3d_batch** batch);

#ifdef __cplusplus
}
#endif
#endif
