// FP32 form, 3D uniform grids: TMA-tiled fused stage kernels.
//
// A CTA owns a TX x TY (x, y) column of cells and marches a chunk of kc
// z-planes.  Each plane of the stage input is staged once into shared memory
// by one TMA box copy ((TX+8) x (TY+6) floats: the tile plus its 3-cell x/y
// halo, x rounded down to a 16-byte boundary) into a ring of RING slots
// guarded by mbarriers; the ring holds the seven planes of the z stencil as
// well as the planes being prefetched.  Every thread computes two
// x-adjacent cells in each of RY consecutive rows with packed FP32x2
// arithmetic (Blackwell FFMA2/FADD2/FMUL2); the rows of a thread are
// independent chains of arithmetic and share their y-stencil loads.  The
// WENO5-HJ upwind side and the Godunov branch of the reinitialisation are
// chosen with selects: the plus-side derivative is the minus-side formula on
// the mirrored difference sequence, so one evaluation per axis serves both
// sides.  The tile shape, the rows per thread and the ring depth form a
// configuration (TileCfg, kTileCfgs); the autotuner picks one per size
// class, with the z chunk.
//
// Waits on the mbarriers are bounded: on a timeout the kernel raises the
// instance's error flag, waits (bounded) for its copies in flight and
// returns; the host reports R3D_ETIMEOUT.
#include <cuda.h>

#include <string>

#include "stencil_f32.cuh"
#include "tile_host.h"



namespace r3d {

namespace {

constexpr long long kSpin = 1ll << 22;

// ------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit = kSpin) {
    for (long long it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// plain tiled TMA load of one box into this CTA's own shared memory
__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ------------------------------------------------------------ packed math
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
__device__ __forceinline__ float2 sel2(bool cx, bool cy, float2 a, float2 b) {
    return make_float2(cx ? a.x : b.x, cy ? a.y : b.y);
}

// WENO5 (Jiang-Peng) derivative times h from the undivided differences
// d1..d5 of the minus-side upwind set; the plus side passes the mirrored
// set (d1..d5 = D2, D1, D0, D-1, D-2).  Ideal weights 0.1/0.6/0.3 for the
// stencils (d1,d2,d3)/(d2,d3,d4)/(d3,d4,d5).
// The smoothness indicators are formed at the scale of divided differences
// (IS coefficients times 1/h^2, so s = IS + psi with the reference's
// psi = 1e-6 exactly as in src/weno_nug_func.h:133-143), and the nonlinear
// weights w_r = (c_r/s_r^2) / sum_q (c_q/s_q^2) are evaluated with one
// reciprocal as n_r / sum_q n_q, n_r = prod_{q!=r} t_q^2, where
// t_q = s_q / sqrt(c_q) (the 1/sqrt(c_q) folded into the coefficients of s_q).
// ih2 = 1/h^2 of the axis.
__device__ __forceinline__ float2 weno5_2(float2 d1, float2 d2, float2 d3, float2 d4, float2 d5, float ih2) {
    const float2 a1 = sub2(d3, d4), b1 = sub2(d5, d4);
    const float2 b2 = sub2(d2, d3), b3 = sub2(d1, d2);
    // s_r scaled by 1/sqrt(c_r) (c = 0.3, 0.6, 0.1): n_r = prod_{q!=r} s_q^2;
    // s1 = IS1 + psi = (10/3 a1 + 11/3 b1) a1 + 4/3 b1^2 + psi,
    // IS2 = (4/3 a1 - 5/3 b2) a1 + 4/3 b2^2, IS3 = (10/3 b2 - 11/3 b3) b2 + 4/3 b3^2
    constexpr float G1 = 1.8257418583505538f, G2 = 1.2909944487358056f, G3 = 3.1622776601683795f;
    const float2 s1 = fma2(fma2(f2(ih2 * (10.0f / 3.0f * G1)), a1, mul2(f2(ih2 * (11.0f / 3.0f * G1)), b1)), a1,
                           fma2(mul2(f2(ih2 * (4.0f / 3.0f * G1)), b1), b1, f2(1.0e-6f * G1)));
    const float2 s2 = fma2(fma2(f2(ih2 * (4.0f / 3.0f * G2)), a1, mul2(f2(ih2 * (-5.0f / 3.0f * G2)), b2)), a1,
                           fma2(mul2(f2(ih2 * (4.0f / 3.0f * G2)), b2), b2, f2(1.0e-6f * G2)));
    const float2 s3 = fma2(fma2(f2(ih2 * (10.0f / 3.0f * G3)), b2, mul2(f2(ih2 * (-11.0f / 3.0f * G3)), b3)), b2,
                           fma2(mul2(f2(ih2 * (4.0f / 3.0f * G3)), b3), b3, f2(1.0e-6f * G3)));
    // IS + psi clamped at 1e6 (fields far from a distance function): the
    // products below stay inside the FP32 range
    const float2 c1 = make_float2(fminf(s1.x, 1.0e6f * G1), fminf(s1.y, 1.0e6f * G1));
    const float2 c2 = make_float2(fminf(s2.x, 1.0e6f * G2), fminf(s2.y, 1.0e6f * G2));
    const float2 c3 = make_float2(fminf(s3.x, 1.0e6f * G3), fminf(s3.y, 1.0e6f * G3));
    const float2 q1 = mul2(c1, c1), q2 = mul2(c2, c2), q3 = mul2(c3, c3);
    const float2 n1 = mul2(q2, q3);
    const float2 n2 = mul2(q1, q3);
    const float2 n3 = mul2(q1, q2);
    const float2 inv = rcp2(add2(add2(n1, n2), n3));
    // p1 = d4 + a1/3 - b1/6, p2 = d3 - a1/3 - b2/6, p3 = d2 + b3/3 - 11/6 b2
    const float2 p1 = fma2(f2(-1.0f / 6.0f), b1, fma2(f2(1.0f / 3.0f), a1, d4));
    const float2 p2 = fma2(f2(-1.0f / 6.0f), b2, fma2(f2(-1.0f / 3.0f), a1, d3));
    const float2 p3 = fma2(f2(-11.0f / 6.0f), b2, fma2(f2(1.0f / 3.0f), b3, d2));
    return mul2(fma2(n3, p3, fma2(n2, p2, mul2(n1, p1))), inv);
}

// Upwind derivative (times h) of an axis from its six packed undivided
// differences D[m] = f[m+1] - f[m] of the 7-point stencil f[0..6] (f[3] the
// cells), plus side where `plus` is set per cell.
__device__ __forceinline__ float2 deriv2(const float2* D, bool px, bool py, float ih2) {
    // minus: (D0..D4); plus (mirrored): (D5, D4, D3, D2, D1)
    return weno5_2(sel2(px, py, D[5], D[0]), sel2(px, py, D[4], D[1]), sel2(px, py, D[3], D[2]),
                   sel2(px, py, D[2], D[3]), sel2(px, py, D[1], D[4]), ih2);
}

__device__ __forceinline__ void diffs2(const float2* f, float2* D) {
#pragma unroll
    for (int m = 0; m < 6; ++m) D[m] = sub2(f[m + 1], f[m]);
}

// WENO5 (Jiang-Peng) derivative times h in FP64 from the undivided
// differences d1..d5 of the minus-side upwind set (the plus side passes the
// mirrored set), the weights with one division:
// w_r = c_r prod_{q!=r} s_q^2 / sum_q c_q prod_{p!=q} s_p^2.
__device__ __forceinline__ double weno5_d(double d1, double d2, double d3, double d4, double d5, double eps) {
    const double a1 = d3 - d4, b1 = d5 - d4, b2 = d2 - d3, b3 = d1 - d2;
    const double s1 = ((10.0 / 3.0) * a1 + (11.0 / 3.0) * b1) * a1 + (4.0 / 3.0) * b1 * b1 + eps;
    const double s2 = ((4.0 / 3.0) * a1 - (5.0 / 3.0) * b2) * a1 + (4.0 / 3.0) * b2 * b2 + eps;
    const double s3 = ((10.0 / 3.0) * b2 - (11.0 / 3.0) * b3) * b2 + (4.0 / 3.0) * b3 * b3 + eps;
    const double q1 = s1 * s1, q2 = s2 * s2, q3 = s3 * s3;
    const double n1 = 0.3 * q2 * q3, n2 = 0.6 * q1 * q3, n3 = 0.1 * q1 * q2;
    const double p1 = d4 + (1.0 / 3.0) * a1 - (1.0 / 6.0) * b1;
    const double p2 = d3 - (1.0 / 3.0) * a1 - (1.0 / 6.0) * b2;
    const double p3 = d2 + (1.0 / 3.0) * b3 - (11.0 / 6.0) * b2;
    return (n1 * p1 + n2 * p2 + n3 * p3) / (n1 + n2 + n3);
}

// Reinitialisation right-hand side of one cell in FP64 from its FP32
// stencils (the interface band): Godunov selection, one-sided WENO5 per
// axis and the smoothed sign of src/reinidisc_f.cpp:58-127 on a uniform
// grid.  X, Y, Z: the 7-point stencils along x, y, z (centre at [3]); rh*:
// the FP32 1/h per axis, eps* = 1e-6 h^2 with h = 1/(double)rh (host-made).
__device__ __noinline__ float reini_cell_fp64(const float* X, const float* Y, const float* Z, float rhx, float rhy,
                                              float rhz, double epsx, double epsy, double epsz, float deltax) {
    const float rh[3] = {rhx, rhy, rhz};
    const double epsd[3] = {epsx, epsy, epsz};
    const double f0 = X[3];
    const double sg = fabs(f0) < 1.0e-8 ? 1.0 : (f0 > 0.0 ? 1.0 : -1.0);
    const float* ax[3] = {X, Y, Z};
    double g2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float* f = ax[d];
        double D[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) D[m] = (double)f[m + 1] - (double)f[m];
        const double ms = D[2] * sg, ps = D[3] * sg, sum = ms + ps;
        const bool c1 = ms > 0.0 && sum > 0.0, c2 = ps < 0.0 && sum < 0.0;
        if (c1 || c2) {
            const double eps = epsd[d];
            const double w = c2 ? weno5_d(D[5], D[4], D[3], D[2], D[1], eps)
                                : weno5_d(D[0], D[1], D[2], D[3], D[4], eps);
            const double gd = w * (double)rh[d];
            g2 += gd * gd;
        }
    }
    const double dn = sqrt(g2);
    const double dl = deltax;
    double S = f0 / sqrt(f0 * f0 + dn * dn * dl * dl);
    if (S != S) S = 1.0;
    return (float)(S - S * dn);  // -(S |grad| - S)
}

// Position of the n-th (from 0) set bit of m, for n < popc(m): a binary
// search on the set-bit counts of halves, quarters, ... (always 0..31).
__device__ __forceinline__ int nth_set_bit(unsigned m, int n) {
    int pos = 0;
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) {
        const unsigned low = m & ((1u << w) - 1u);
        const int c = __popc(low);
        if (n >= c) {
            n -= c;
            m >>= w;
            pos += w;
        } else {
            m = low;
        }
    }
    return pos;
}

// 3-input minimum / maximum (one instruction on sm_100)
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// One tile configuration: TX x TY cells per CTA (TX/2 threads per row
// group, RY rows per thread), RING plane slots in shared memory, MINB CTAs
// per SM the registers are limited for.
template <int TX_, int TY_, int RY_, int RING_, int MINB_>
struct TileCfg {
    static constexpr int TX = TX_, TY = TY_, RY = RY_, RING = RING_, MINB = MINB_;
    static constexpr int TPR = TX / 2;           // threads per row group
    static constexpr int NT = TPR * (TY / RY);   // threads per CTA
    static constexpr int NW = NT / 32;
    static constexpr int BX = TX + 8, BY = TY + 6;
    static constexpr int SLOT = (BX * BY + 31) / 32 * 32;  // floats per slot (128-byte aligned)
    static constexpr unsigned BOX_BYTES = BX * BY * 4;
    static_assert(NT % 32 == 0 && TY % RY == 0, "whole warps, whole row groups");
    static_assert(RING >= 8, "the ring holds the 7-plane stencil and one plane in flight");
    static_assert(BX <= 256 && BY <= 256 && (BX * 4) % 16 == 0, "TMA box limits");
    static constexpr size_t smem() { return (size_t)RING * SLOT * 4 + RING * sizeof(uint64_t) + (RING + 2) * sizeof(int); }
};

// The configurations the library is built with (id = position).
#define R3D_TILE_CFGS(X)        \
    X(0, 64, 8, 1, 16, 3)       \
    X(1, 64, 8, 2, 12, 4)       \
    X(2, 64, 16, 2, 10, 2)      \
    X(3, 32, 16, 2, 12, 4)      \
    X(4, 128, 8, 2, 8, 2)       \
    X(5, 64, 8, 1, 10, 4)       \
    X(6, 32, 16, 2, 12, 5)

#define R3D_CFG_TYPE(id, tx, ty, ry, ring, minb) using Cfg##id = TileCfg<tx, ty, ry, ring, minb>;
R3D_TILE_CFGS(R3D_CFG_TYPE)
#undef R3D_CFG_TYPE

// One work item: the TX x TY column (bx, by) over planes [bz*kc, bz*kc+kc)
// of one instance.  Returns false when a bounded wait gave up (the error
// flag is raised and the copies in flight have been waited for).  The
// item's volume partials (when `volume`) go to partial_out[0..1].  The
// mbarriers are initialised at the start of the item and invalidated at its
// end, so a persistent CTA can run items back to back.
// ISO: the three axes have bitwise-equal spacing constants (cubic cells), so
// axis 0's are used for all three and held once.
//
// Shared memory is a ring of RING plane boxes: the x and y stencils of
// plane k come from its box, the z stencil from the thread's own column in
// the seven boxes k-3..k+3.  Each box has a "full" mbarrier (the TMA copy
// landed).  After plane k the box of plane k-3 is refilled with plane
// k-3+RING by the last warp to count itself out of the box (a per-box
// release counter), so that warps drift apart where their work differs
// (interface-band cells in FP64, wall ghosts) instead of meeting at a CTA
// barrier every plane.
template <class C, bool REINI, int STAGE, bool ISO>
__device__ __forceinline__ bool tile_item(const CUtensorMap* tmap, const TileArgs& a, int bx, int by, int bz,
                                          bool volume, unsigned char* smem_raw, double* red_a, double* red_b,
                                          double* partial_out) {
    constexpr int RY = C::RY, BX = C::BX, RING = C::RING, SLOT = C::SLOT;
    float* ring = reinterpret_cast<float*>(smem_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(ring + RING * SLOT);  // full
    int* rel = reinterpret_cast<int*>(bar + RING);                    // release counters
    volatile int* s_abort = rel + RING;
    int* s_issued = rel + RING + 1;  // last plane issued

    const Layout& L = a.L;
    const int sy = (int)L.sy, sz = (int)L.sz;
    const int tid = threadIdx.x, lane = tid & 31;
    const int tx = tid % C::TPR, tg = tid / C::TPR;
    const int i0 = bx * C::TX + 2 * tx;
    const int jb = by * C::TY + tg * RY;  // the thread's first row
    const int k0 = bz * a.kc;
    const int k1 = min(k0 + a.kc, L.nz);
    const int xbox = bx * C::TX + L.gx - 4;  // 16-byte aligned x start
    const int ybox = by * C::TY + L.gy - 3;
    const int pfirst = k0 - 3;  // first plane staged (ring position 0)
    const int plast = k1 + 2;   // last plane staged
    const int rowb = tg * RY;   // box row of the first y-stencil point of the thread's first row
    bool act0[RY], act1[RY], gside[RY], gxlo[RY], gxhi1[RY], gxhi2[RY], gylo[RY], gyhi[RY];
    int col[RY];  // 32-bit offsets: the host enables tiles only for fields of < 2^31 cells
    int own[RY];  // the thread's two cells of row r in a box
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        const int j = jb + r;
        act0[r] = i0 < L.nx && j < L.ny;
        act1[r] = i0 + 1 < L.nx && j < L.ny;
        col[r] = (j + L.gy) * sy + (i0 + L.gx);
        own[r] = (rowb + r + 3) * BX + 2 * tx + 4;
        // wall ghost layers this thread writes on every plane (x, y faces)
        gxlo[r] = act0[r] && i0 == 0;
        gxhi2[r] = act1[r] && i0 + 1 == L.nx - 1;  // second cell is the last one
        gxhi1[r] = act0[r] && !act1[r];             // first cell is the last one
        gylo[r] = act0[r] && j == 0;
        gyhi[r] = act0[r] && j == L.ny - 1;
        gside[r] = gxlo[r] || gxhi2[r] || gxhi1[r] || gylo[r] || gyhi[r];
    }

    if (tid == 0) {
        for (int s = 0; s < RING; ++s) {
            mbar_init(bar + s, 1);
            rel[s] = 0;
        }
        *s_abort = 0;
        mbar_fence_init();
        for (int p = pfirst; p <= min(pfirst + RING - 1, plast); ++p) {
            const int s = p - pfirst;
            mbar_expect_tx(bar + s, C::BOX_BYTES);
            tma_load_3d(ring + s * SLOT, tmap, bar + s, xbox, ybox, p + L.gz);
            *s_issued = p;
        }
    }
    __syncthreads();

    // planes k0-3 .. k0+2: the first window without its top plane
    const long long spin = a.spin > 0 ? a.spin : kSpin;
    bool ok = true;
#pragma unroll
    for (int m = 0; m < 6; ++m) ok = ok && mbar_wait_bounded(bar + m, 0, spin);
    // timeout-path test: the second completion of box 0 needs a refill that
    // only the plane loop issues, so this wait gives up after `spin` tries
    if (a.wait_test) ok = ok && mbar_wait_bounded(bar, 1, spin);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok) *s_abort = 1;

    const float vs = (float)*a.vscale;
    const float dtc = REINI ? a.dtr : (float)*a.dt;
    const int c0 = (k0 + L.gz) * sz;
    float2 wprev[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        wprev[r] = make_float2(0.f, 0.f);
        if (!REINI && act0[r]) {
            const float* wp = a.w + c0 + col[r] - sz;
            wprev[r] = act1[r] ? __ldg(reinterpret_cast<const float2*>(wp)) : make_float2(__ldg(wp), 0.f);
        }
    }
    double vol_a = 0.0, vol_b = 0.0;

    // cell-local global operands of a plane (velocities, step start value),
    // fetched one plane ahead so their latency overlaps the current plane;
    // v on the face below row r is v of row r-1 for r > 0
    float2 nu[RY], nv[RY], nw[RY], nfn[RY], nvm0;
    float num[RY];
#pragma unroll
    for (int r = 0; r < RY; ++r) {
        nu[r] = nv[r] = nw[r] = nfn[r] = make_float2(0.f, 0.f);
        num[r] = 0.f;
    }
    nvm0 = make_float2(0.f, 0.f);
    auto fetch = [&](int cz) {
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (!act0[r]) continue;
            const int cc = cz + col[r];
            if (!REINI) {
                if (act1[r]) {
                    nu[r] = __ldg(reinterpret_cast<const float2*>(a.u + cc));
                    nv[r] = __ldg(reinterpret_cast<const float2*>(a.v + cc));
                    nw[r] = __ldg(reinterpret_cast<const float2*>(a.w + cc));
                    if (r == 0) nvm0 = __ldg(reinterpret_cast<const float2*>(a.v + cc - sy));
                } else {
                    nu[r].x = __ldg(a.u + cc);
                    nv[r].x = __ldg(a.v + cc);
                    nw[r].x = __ldg(a.w + cc);
                    if (r == 0) nvm0.x = __ldg(a.v + cc - sy);
                }
                num[r] = __ldg(a.u + cc - 1);
            }
            // the step start value may be this stage's output (stage 3): plain loads
            if (STAGE != 1) nfn[r] = act1[r] ? *reinterpret_cast<const float2*>(a.fn + cc) : make_float2(a.fn[cc], 0.f);
        }
    };
    fetch(c0);

    int sb = 0;          // ring slot of position n = k - k0 (plane k-3)
    int ws = 6, wp = 0;  // ring slot and phase parity of position n + 6 (plane k+3)
    int cz = c0;
    for (int k = k0; k < k1; ++k, cz += sz) {
        ok = __all_sync(0xffffffffu, mbar_wait_bounded(bar + ws, (uint32_t)wp, spin));
        if (!ok) *s_abort = 1;
        if (__any_sync(0xffffffffu, *s_abort != 0)) break;
        const float* slot[7];
#pragma unroll
        for (int m = 0; m < 7; ++m) {
            int s = sb + m;
            if (RING < 16 || (RING & (RING - 1))) s -= s >= RING ? RING : 0;
            else s &= RING - 1;
            slot[m] = ring + s * SLOT;
        }
        const float* sl = slot[3];  // plane k

        // y stencil values of all RY rows (rows rowb .. rowb+RY+5 of the box)
        float2 DY[RY + 5];
        float2 fy2[RY], fy4[RY];
        {
            float2 fy[RY + 6];
#pragma unroll
            for (int m = 0; m < RY + 6; ++m) fy[m] = *reinterpret_cast<const float2*>(sl + (rowb + m) * BX + 2 * tx + 4);
#pragma unroll
            for (int m = 0; m < RY + 5; ++m) DY[m] = sub2(fy[m + 1], fy[m]);
#pragma unroll
            for (int r = 0; r < RY; ++r) { fy2[r] = fy[r + 2]; fy4[r] = fy[r + 4]; }
        }
        // this plane's operands, then the next plane's loads in flight
        // through the whole computation of this one
        float2 fnr[RY], ucr[RY], vcr[RY], wcr[RY], vm0;
        float umr[RY];
#pragma unroll
        for (int r = 0; r < RY; ++r) { fnr[r] = nfn[r]; ucr[r] = nu[r]; vcr[r] = nv[r]; wcr[r] = nw[r]; umr[r] = num[r]; }
        vm0 = nvm0;
        if (k + 1 < k1) fetch(cz + sz);

        float2 f0[RY], Lc[RY];
        bool bandx[RY], bandy[RY];
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            // x stencil: the row's columns 2tx .. 2tx+9 (the cells at 2tx+4, 2tx+5)
            float xv[10];
            {
                const float* rp = sl + (rowb + r + 3) * BX + 2 * tx;
#pragma unroll
                for (int q = 0; q < 5; ++q) {
                    const float2 t = *reinterpret_cast<const float2*>(rp + 2 * q);
                    xv[2 * q] = t.x;
                    xv[2 * q + 1] = t.y;
                }
            }
            float2 Dx[6], Dz[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) Dx[m] = make_float2(xv[m + 2] - xv[m + 1], xv[m + 3] - xv[m + 2]);
            float2 fz2, fz4;
            {
                float2 fz[7];
#pragma unroll
                for (int m = 0; m < 7; ++m) fz[m] = *reinterpret_cast<const float2*>(slot[m] + own[r]);
                diffs2(fz, Dz);
                fz2 = fz[2];
                fz4 = fz[4];
            }
            const float2* Dy = DY + r;
            f0[r] = make_float2(xv[4], xv[5]);
            bandx[r] = bandy[r] = false;
            if (!REINI) {
                const float2 h2 = f2(0.5f * vs);
                const float2 vm = r == 0 ? vm0 : vcr[r - 1];
                const float2 ia = mul2(h2, add2(make_float2(umr[r], ucr[r].x), ucr[r]));
                const float2 ja = mul2(h2, add2(vcr[r], vm));
                const float2 ka = mul2(h2, add2(wcr[r], wprev[r]));
                wprev[r] = wcr[r];
                const float2 gx = mul2(f2(a.rh[0]), deriv2(Dx, ia.x < 0.f, ia.y < 0.f, a.eps[0]));
                constexpr int AY = ISO ? 0 : 1, AZ = ISO ? 0 : 2;
                const float2 gy = mul2(f2(a.rh[AY]), deriv2(Dy, ja.x < 0.f, ja.y < 0.f, a.eps[AY]));
                const float2 gz = mul2(f2(a.rh[AZ]), deriv2(Dz, ka.x < 0.f, ka.y < 0.f, a.eps[AZ]));
                Lc[r] = mul2(f2(-1.f), fma2(ka, gz, fma2(ja, gy, mul2(ia, gx))));
            } else {
                // Godunov selection per axis (src/reinidisc_f.cpp:70-109) on the
                // backward and forward differences D[2], D[3] times the sign s
                // (the grid factor 1/h > 0 leaves every test unchanged):
                //   upwind minus side: m > 0 && p > -m, i.e. m > 0 && m + p > 0
                //   upwind plus side:  p < 0 && m < -p, i.e. p < 0 && m + p < 0
                // (the sign of a rounded sum is the sign of the exact sum)
                const float2 fc = f0[r];
                const float2 sg = make_float2(fabsf(fc.x) < 1.0e-8f ? 1.f : (fc.x > 0.f ? 1.f : -1.f),
                                              fabsf(fc.y) < 1.0e-8f ? 1.f : (fc.y > 0.f ? 1.f : -1.f));
                const float2* ax[3] = {Dx, Dy, Dz};
                float2 g2 = make_float2(0.f, 0.f);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const float2* D = ax[d];
                    const float2 ms = mul2(D[2], sg), ps = mul2(D[3], sg);
                    const float2 sum = add2(ms, ps);
                    const bool c1x = ms.x > 0.f && sum.x > 0.f, c2x = ps.x < 0.f && sum.x < 0.f;
                    const bool c1y = ms.y > 0.f && sum.y > 0.f, c2y = ps.y < 0.f && sum.y < 0.f;
                    const int ad = ISO ? 0 : d;
                    float2 g = mul2(f2(a.rh[ad]), deriv2(D, c2x, c2y, a.eps[ad]));
                    g.x = (c1x || c2x) ? g.x : 0.f;
                    g.y = (c1y || c2y) ? g.y : 0.f;
                    g2 = fma2(g, g, g2);
                }
                const float2 dn = make_float2(sqrt_approx(g2.x), sqrt_approx(g2.y));
                const float2 dl = f2(a.deltax);
                const float2 den = fma2(mul2(mul2(dn, dn), dl), dl, mul2(fc, fc));
                float2 S = mul2(fc, make_float2(rsqrtf(den.x), rsqrtf(den.y)));
                if (S.x != S.x) S.x = 1.f;
                if (S.y != S.y) S.y = 1.f;
                Lc[r] = sub2(S, mul2(S, dn));  // -(S |grad| - S)
                // interface band: the 7-point stencil changes sign, i.e. neither
                // all values >= 0 (min >= 0) nor all < 0 (max < 0)
                const float lox = min3f(min3f(fc.x, xv[3], xv[5]), min3f(fy2[r].x, fy4[r].x, fz2.x), fz4.x);
                const float hix = max3f(max3f(fc.x, xv[3], xv[5]), max3f(fy2[r].x, fy4[r].x, fz2.x), fz4.x);
                const float loy = min3f(min3f(fc.y, xv[4], xv[6]), min3f(fy2[r].y, fy4[r].y, fz2.y), fz4.y);
                const float hiy = max3f(max3f(fc.y, xv[4], xv[6]), max3f(fy2[r].y, fy4[r].y, fz2.y), fz4.y);
                bandx[r] = lox < 0.f && hix >= 0.f;
                bandy[r] = loy < 0.f && hiy >= 0.f;
                if (a.f49 == 0) {
                    if (bandx[r]) Lc[r].x = 0.f;  // src/reinidisc_fsf.cpp:70-72
                    if (bandy[r]) Lc[r].y = 0.f;
                }
            }
        }
        bool band_here = false;
        if (REINI && a.f49 != 0 && a.band64) {
#pragma unroll
            for (int r = 0; r < RY; ++r) band_here = band_here || (act0[r] && bandx[r]) || (act1[r] && bandy[r]);
        }
        // one vote for the plane: most warps hold no band cell in it
        if (REINI && a.f49 != 0 && a.band64 && __any_sync(0xffffffffu, band_here)) {
            // The warp's band cells of row r (at most 64) are dealt out to
            // its lanes, one FP64 evaluation each, stencils from shared
            // memory; results go back to the owning lanes by shuffles.
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                const unsigned mx = __ballot_sync(0xffffffffu, act0[r] && bandx[r]);
                const unsigned my = __ballot_sync(0xffffffffu, act1[r] && bandy[r]);
                if (mx | my) {
                    const int cx = __popc(mx), total = cx + __popc(my);
                    const unsigned below = (1u << lane) - 1u;
                    const int bxi = __popc(mx & below), byi = cx + __popc(my & below);
                    for (int base = 0; base < total; base += 32) {
                        float res = 0.f;
                        const int b = base + lane;
                        if (b < total) {
                            const bool isy = b >= cx;
                            // the lane holding the (b or b-cx)-th set bit of the mask
                            const int src = nth_set_bit(isy ? my : mx, isy ? b - cx : b);
                            const int st = (tid & ~31) + src;  // the source lane's thread
                            const int sx = 2 * (st % C::TPR) + (isy ? 1 : 0);
                            const int srow = (st / C::TPR) * RY + r;  // its y-stencil base row
                            float X[7], Y[7], Z[7];
#pragma unroll
                            for (int m = 0; m < 7; ++m) {
                                X[m] = sl[(srow + 3) * BX + sx + 1 + m];
                                Y[m] = sl[(srow + m) * BX + sx + 4];
                                Z[m] = slot[m][(srow + 3) * BX + sx + 4];
                            }
                            res = reini_cell_fp64(X, Y, Z, a.rh[0], a.rh[1], a.rh[2], a.beps[0], a.beps[1],
                                                  a.beps[2], a.deltax);
                        }
                        const float rx = __shfl_sync(0xffffffffu, res, (bxi - base) & 31);
                        const float ry = __shfl_sync(0xffffffffu, res, (byi - base) & 31);
                        if (act0[r] && bandx[r] && bxi >= base && bxi < base + 32) Lc[r].x = rx;
                        if (act1[r] && bandy[r] && byi >= base && byi < base + 32) Lc[r].y = ry;
                    }
                }
            }
        }

        // the warp's shared-memory reads of this plane are done, so it counts
        // itself out of the box of plane k-3 (before its global stores and
        // loads, so the fence waits on nothing in flight), and the last warp
        // out refills the box with plane k-3+RING
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            if (atomicAdd(rel + sb, 1) == C::NW - 1) {
                __threadfence_block();
                rel[sb] = 0;
                if (k - 3 + RING <= plast) {
                    fence_proxy_async();
                    mbar_expect_tx(bar + sb, C::BOX_BYTES);
                    tma_load_3d(ring + sb * SLOT, tmap, bar + sb, xbox, ybox, k - 3 + RING + L.gz);
                    atomicMax(s_issued, k - 3 + RING);
                }
            }
        }

#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (!act0[r]) continue;
            // RK combine (src/levelset_RK3.cpp:121-156, src/reini_RK3.cpp:118-135)
            float2 val;
            const float2 sdl = fma2(f2(dtc), Lc[r], f0[r]);  // stage input + dt L
            if (STAGE == 1) {
                val = sdl;
            } else {
                if (STAGE == 2) val = fma2(f2(0.75f), fnr[r], mul2(f2(0.25f), sdl));
                else val = fma2(f2(1.0f / 3.0f), fnr[r], mul2(f2(2.0f / 3.0f), sdl));
            }
            const int c = cz + col[r];
            if (act1[r]) *reinterpret_cast<float2*>(a.out + c) = val;
            else a.out[c] = val.x;
            // wall ghost copies (src/gc_neumann.cpp:29-54)
            if (gside[r] || k == 0 || k == L.nz - 1) {
                if (gxlo[r]) { a.out[c - 1] = val.x; a.out[c - 2] = val.x; a.out[c - 3] = val.x; }
                if (gxhi2[r]) { a.out[c + 2] = val.y; a.out[c + 3] = val.y; a.out[c + 4] = val.y; }
                if (gxhi1[r]) { a.out[c + 1] = val.x; a.out[c + 2] = val.x; a.out[c + 3] = val.x; }
                const int nw = act1[r] ? 2 : 1;
                if (gylo[r])
                    for (int q = 1; q <= 3; ++q)
                        for (int e = 0; e < nw; ++e) a.out[c - q * sy + e] = e ? val.y : val.x;
                if (gyhi[r])
                    for (int q = 1; q <= 3; ++q)
                        for (int e = 0; e < nw; ++e) a.out[c + q * sy + e] = e ? val.y : val.x;
                if (k == 0 && !(L.io & kHaloZLo))  // a slab face's ghosts come from the neighbour
                    for (int q = 1; q <= 3; ++q)
                        for (int e = 0; e < nw; ++e) a.out[c - q * sz + e] = e ? val.y : val.x;
                if (k == L.nz - 1 && !(L.io & kHaloZHi))
                    for (int q = 1; q <= 3; ++q)
                        for (int e = 0; e < nw; ++e) a.out[c + q * sz + e] = e ? val.y : val.x;
            }
            if (volume) {
                // smoothed Heaviside in FP64 (src/fluid_update_fsf.cpp:50-71)
                const double PI_REF = 3.14159265359;
                const int nw = act1[r] ? 2 : 1;
                for (int e = 0; e < nw; ++e) {
                    const double ph = e ? val.y : val.x;
                    double H = 0.0;
                    if (ph > a.psi) H = 1.0;
                    if (ph < -a.psi) H = 0.0;
                    if (fabs(ph) <= a.psi) H = 0.5 * (1.0 + ph / a.psi + (1.0 / PI_REF) * sin((PI_REF * ph) / a.psi));
                    vol_a += a.cellvol * H;
                    vol_b += a.cellvol * (1.0 - H);
                }
            }
        }

        sb = sb + 1 == RING ? 0 : sb + 1;
        if (++ws == RING) {
            ws = 0;
            wp ^= 1;
        }
    }
    __syncthreads();
    const bool aborted = *s_abort != 0;

    if (aborted) {
        if (tid == 0) {
            atomicExch(a.err, 1);
            // wait (bounded) for every copy still in flight before leaving
            for (int p = pfirst; p <= *s_issued; ++p) {
                const int q = p - pfirst;
                mbar_wait_bounded(bar + (q % RING), (uint32_t)((q / RING) & 1));
            }
        }
        return false;
    }
    if (volume) {
        for (int o = 16; o > 0; o >>= 1) {
            vol_a += __shfl_down_sync(0xffffffffu, vol_a, o);
            vol_b += __shfl_down_sync(0xffffffffu, vol_b, o);
        }
        if (lane == 0) { red_a[tid >> 5] = vol_a; red_b[tid >> 5] = vol_b; }
        __syncthreads();
        if (tid == 0) {
            double sa = 0.0, sb2 = 0.0;
            for (int q = 0; q < C::NW; ++q) { sa += red_a[q]; sb2 += red_b[q]; }
            partial_out[0] = sa;
            partial_out[1] = sb2;
        }
    }
    // every wait of the item has completed: retire the barriers
    __syncthreads();
    if (tid == 0)
        for (int s = 0; s < RING; ++s) mbar_inval(bar + s);
    __syncthreads();
    return true;
}

template <class C, bool REINI, int STAGE, bool VOLUME, bool ISO>
__global__ void __launch_bounds__(C::NT, C::MINB) tile_kernel(const __grid_constant__ CUtensorMap tmap, TileArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_a[C::NW], red_b[C::NW];
    const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    tile_item<C, REINI, STAGE, ISO>(&tmap, a, blockIdx.x, blockIdx.y, blockIdx.z, VOLUME, smem_raw, red_a, red_b,
                               a.partial + 2 * b);
}

// Persistent batched form: CTAs take the work items of all tiled members
// (member m owns items [tile0[m], tile0[m+1]); item = (bx, by, bz) of that
// member) one at a time from a global counter, so CTAs whose items hold
// more work (FP64 interface band, wall ghosts) take fewer of them.  The
// last CTA to leave resets the counter pair work[0..1] for the next launch
// on the stream.  Reinitialisation pseudo-step q is skipped by members with
// f44 <= q; the last stage of a member's step adds its volume partials.
template <class C, bool REINI, int STAGE, bool ISO>
__global__ void __launch_bounds__(C::NT, C::MINB) batch_tile_kernel(const TiledMember* __restrict__ members,
                                                                    const CUtensorMap* __restrict__ maps,
                                                                    const long long* __restrict__ tile0, int nm,
                                                                    int q, double* __restrict__ vol_part,
                                                                    unsigned* __restrict__ work) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red_a[C::NW], red_b[C::NW];
    __shared__ TileArgs sa;
    __shared__ int s_member;
    __shared__ long long s_t;
    const long long nt = tile0[nm];
    for (;;) {
        if (threadIdx.x == 0) {
            const long long t0 = (long long)atomicAdd(work, 1u);
            s_t = t0;
            if (t0 < nt) {
                int lo = 0, hi = nm - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (tile0[mid] <= t0) lo = mid;
                    else hi = mid - 1;
                }
                s_member = lo;
                sa = members[lo].args;
                sa.out = STAGE == 1 ? members[lo].a1 : STAGE == 2 ? members[lo].a2 : members[lo].phi;
            }
        }
        __syncthreads();
        const long long t = s_t;
        if (t >= nt) break;
        const int m = s_member;
        const int f44 = members[m].f44;
        if (REINI && f44 <= q) {
            __syncthreads();
            continue;
        }
        const bool volume = STAGE == 3 && (REINI ? q == f44 - 1 : f44 == 0);
        const long long lt = t - tile0[m];
        const int ntx = (sa.L.nx + C::TX - 1) / C::TX, nty = (sa.L.ny + C::TY - 1) / C::TY;
        const int bx = (int)(lt % ntx);
        const int by = (int)((lt / ntx) % nty);
        const int bz = (int)(lt / ((long long)ntx * nty));
        // the item's arguments in a thread-local copy: the plane loop reads
        // them across CTA barriers, after which shared memory would be reread
        const TileArgs a = sa;
        if (!tile_item<C, REINI, STAGE, ISO>(maps + 3 * m + (STAGE - 1), a, bx, by, bz, volume, smem_raw, red_a, red_b,
                                        vol_part + 2 * t))
            break;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(work + 1, 1u) == gridDim.x - 1) {
            work[0] = 0u;
            work[1] = 0u;
            __threadfence();
        }
    }
}

// Face maxima over the cells of one item (x faces 0..nx-2, y 0..ny-2, z
// 0..nz-2, src/ietimestep.cpp:72-88) for every tiled member's item.
template <class C>
__global__ void __launch_bounds__(C::NT) batch_tile_vmax_kernel(const TiledMember* __restrict__ members,
                                                                const long long* __restrict__ tile0, int nm,
                                                                double* __restrict__ vmax_part) {
    __shared__ unsigned s[3][C::NW];
    const long long nt = tile0[nm];
    for (long long t = blockIdx.x; t < nt; t += gridDim.x) {
        int lo = 0, hi = nm - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tile0[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const TileArgs& a = members[lo].args;
        const Layout& L = a.L;
        const long long lt = t - tile0[lo];
        const int ntx = (L.nx + C::TX - 1) / C::TX, nty = (L.ny + C::TY - 1) / C::TY;
        const int bx = (int)(lt % ntx), by = (int)((lt / ntx) % nty), bz = (int)(lt / ((long long)ntx * nty));
        const int tx = threadIdx.x % C::TPR, tg = threadIdx.x / C::TPR;
        const int i0 = bx * C::TX + 2 * tx;
        const int k0 = bz * a.kc, k1 = min(k0 + a.kc, L.nz);
        // |x| compared as the float's bit pattern with the sign cleared (exact)
        unsigned mu = 0u, mv = 0u, mw = 0u;
        for (int r = 0; r < C::RY; ++r) {
            const int j = by * C::TY + tg * C::RY + r;
            if (j >= L.ny || i0 >= L.nx) continue;
            const bool two = i0 + 1 < L.nx;
            const long long col = (long long)(j + L.gy) * L.sy + (i0 + L.gx);
            for (int k = k0; k < k1; ++k) {
                const long long c = (long long)(k + L.gz) * L.sz + col;
                float2 fu, fv, fw;
                if (two) {
                    fu = __ldg(reinterpret_cast<const float2*>(a.u + c));
                    fv = __ldg(reinterpret_cast<const float2*>(a.v + c));
                    fw = __ldg(reinterpret_cast<const float2*>(a.w + c));
                } else {
                    fu = make_float2(__ldg(a.u + c), 0.f);
                    fv = make_float2(__ldg(a.v + c), 0.f);
                    fw = make_float2(__ldg(a.w + c), 0.f);
                }
                if (i0 < L.nx - 1) mu = max(mu, __float_as_uint(fu.x) & 0x7fffffffu);
                if (i0 + 1 < L.nx - 1) mu = max(mu, __float_as_uint(fu.y) & 0x7fffffffu);
                if (j < L.ny - 1) mv = max(mv, max(__float_as_uint(fv.x) & 0x7fffffffu, __float_as_uint(fv.y) & 0x7fffffffu));
                if (k < L.nz - 1) mw = max(mw, max(__float_as_uint(fw.x) & 0x7fffffffu, __float_as_uint(fw.y) & 0x7fffffffu));
            }
        }
        mu = __reduce_max_sync(0xffffffffu, mu);
        mv = __reduce_max_sync(0xffffffffu, mv);
        mw = __reduce_max_sync(0xffffffffu, mw);
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { s[0][w] = mu; s[1][w] = mv; s[2][w] = mw; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int q = 1; q < C::NW; ++q) { mu = max(mu, s[0][q]); mv = max(mv, s[1][q]); mw = max(mw, s[2][q]); }
            vmax_part[3 * t] = (double)__uint_as_float(mu);
            vmax_part[3 * t + 1] = (double)__uint_as_float(mv);
            vmax_part[3 * t + 2] = (double)__uint_as_float(mw);
        }
        __syncthreads();
    }
}

// The ring needs more than the default 48 KB of dynamic shared memory, and a
// full shared-memory carveout lets several CTAs share an SM.
template <typename K>
bool tile_attr(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess &&
           cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100) == cudaSuccess;
}

template <class C, bool ISO>
bool cfg_prepare_iso(size_t b) {
    return tile_attr(tile_kernel<C, false, 1, false, ISO>, b) && tile_attr(tile_kernel<C, false, 2, false, ISO>, b) &&
           tile_attr(tile_kernel<C, false, 3, false, ISO>, b) && tile_attr(tile_kernel<C, false, 1, true, ISO>, b) &&
           tile_attr(tile_kernel<C, false, 2, true, ISO>, b) && tile_attr(tile_kernel<C, false, 3, true, ISO>, b) &&
           tile_attr(tile_kernel<C, true, 1, false, ISO>, b) && tile_attr(tile_kernel<C, true, 2, false, ISO>, b) &&
           tile_attr(tile_kernel<C, true, 3, false, ISO>, b) && tile_attr(tile_kernel<C, true, 1, true, ISO>, b) &&
           tile_attr(tile_kernel<C, true, 2, true, ISO>, b) && tile_attr(tile_kernel<C, true, 3, true, ISO>, b) &&
           tile_attr(batch_tile_kernel<C, false, 1, ISO>, b) && tile_attr(batch_tile_kernel<C, false, 2, ISO>, b) &&
           tile_attr(batch_tile_kernel<C, false, 3, ISO>, b) && tile_attr(batch_tile_kernel<C, true, 1, ISO>, b) &&
           tile_attr(batch_tile_kernel<C, true, 2, ISO>, b) && tile_attr(batch_tile_kernel<C, true, 3, ISO>, b);
}

template <class C>
bool cfg_prepare() {
    return cfg_prepare_iso<C, false>(C::smem()) && cfg_prepare_iso<C, true>(C::smem());
}

template <class C, bool ISO>
void launch_stage_cfg(const CUtensorMap& map, const TileArgs& a, bool reini, int stage, bool volume,
                      cudaStream_t st) {
    const dim3 grid((a.L.nx + C::TX - 1) / C::TX, (a.L.ny + C::TY - 1) / C::TY, (a.L.nz + a.kc - 1) / a.kc);
    const dim3 block(C::NT);
    const size_t sm = C::smem();
#define R3D_TL(R, S, V) tile_kernel<C, R, S, V, ISO><<<grid, block, sm, st>>>(map, a)
    if (reini) {
        if (stage == 1) { if (volume) R3D_TL(true, 1, true); else R3D_TL(true, 1, false); }
        else if (stage == 2) { if (volume) R3D_TL(true, 2, true); else R3D_TL(true, 2, false); }
        else { if (volume) R3D_TL(true, 3, true); else R3D_TL(true, 3, false); }
    } else {
        if (stage == 1) { if (volume) R3D_TL(false, 1, true); else R3D_TL(false, 1, false); }
        else if (stage == 2) { if (volume) R3D_TL(false, 2, true); else R3D_TL(false, 2, false); }
        else { if (volume) R3D_TL(false, 3, true); else R3D_TL(false, 3, false); }
    }
#undef R3D_TL
}

template <class C, bool ISO>
void launch_batch_cfg(const TiledMember* members, const CUtensorMap* maps, const long long* tile0, int nm,
                      bool reini, int stage, int q, double* vol_part, unsigned* work, unsigned grid,
                      cudaStream_t st) {
    const size_t sm = C::smem();
    const dim3 g(grid), block(C::NT);
#define R3D_BT(R, S) batch_tile_kernel<C, R, S, ISO><<<g, block, sm, st>>>(members, maps, tile0, nm, q, vol_part, work)
    if (reini) {
        if (stage == 1) R3D_BT(true, 1);
        else if (stage == 2) R3D_BT(true, 2);
        else R3D_BT(true, 3);
    } else {
        if (stage == 1) R3D_BT(false, 1);
        else if (stage == 2) R3D_BT(false, 2);
        else R3D_BT(false, 3);
    }
#undef R3D_BT
}

struct CfgInfo {
    int tx, ty, ry, ring, minb, threads;
    size_t smem;
};

const CfgInfo kCfgInfo[] = {
#define R3D_CFG_INFO(id, tx, ty, ry, ring, minb) {tx, ty, ry, ring, minb, Cfg##id::NT, Cfg##id::smem()},
    R3D_TILE_CFGS(R3D_CFG_INFO)
#undef R3D_CFG_INFO
};
constexpr int kNumCfg = sizeof(kCfgInfo) / sizeof(kCfgInfo[0]);

const CfgInfo& info(int cfg) { return kCfgInfo[(cfg >= 0 && cfg < kNumCfg) ? cfg : 0]; }

}  // namespace

int tile_cfg_count() { return kNumCfg; }

int tile_cfg_describe(int cfg, int* tx, int* ty, int* ry, int* ring, int* threads) {
    if (cfg < 0 || cfg >= kNumCfg) return 1;
    const CfgInfo& c = kCfgInfo[cfg];
    if (tx) *tx = c.tx;
    if (ty) *ty = c.ty;
    if (ry) *ry = c.ry;
    if (ring) *ring = c.ring;
    if (threads) *threads = c.threads;
    return 0;
}

int tile_ctas_per_sm(int cfg) { return info(cfg).minb; }

// Sets the attributes of every instantiation once per device.
bool tile_prepare() {
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (dev >= 0 && dev < 64 && done[dev]) return true;
    bool ok = true;
#define R3D_CFG_PREP(id, tx, ty, ry, ring, minb) ok = ok && cfg_prepare<Cfg##id>();
    R3D_TILE_CFGS(R3D_CFG_PREP)
#undef R3D_CFG_PREP
    if (!ok) {
        cudaGetLastError();
        return false;
    }
    if (dev >= 0 && dev < 64) done[dev] = true;
    return true;
}

long long tile_items_of(const Layout& L, int kc, int cfg) {
    const dim3 g = tile_grid(L, kc, cfg);
    return (long long)g.x * g.y * g.z;
}

int launch_batch_tile_stage(const TiledMember* members, const CUtensorMap* maps, const long long* tile0, int nm,
                            int cfg, bool iso, bool reini, int stage, int q, double* vol_part, unsigned* work,
                            unsigned grid, cudaStream_t st) {
    tile_prepare();  // a failure here makes the launch below fail, which the caller reports
#define R3D_BATCH(C, I) launch_batch_cfg<C, I>(members, maps, tile0, nm, reini, stage, q, vol_part, work, grid, st)
    switch (cfg) {
#define R3D_CFG_CASE(id, tx, ty, ry, ring, minb) \
    case id: if (iso) R3D_BATCH(Cfg##id, true); else R3D_BATCH(Cfg##id, false); break;
        R3D_TILE_CFGS(R3D_CFG_CASE)
#undef R3D_CFG_CASE
        default: if (iso) R3D_BATCH(Cfg0, true); else R3D_BATCH(Cfg0, false);
    }
#undef R3D_BATCH
    return 1;
}

int launch_batch_tile_vmax(const TiledMember* members, const long long* tile0, int nm, int cfg, double* vmax_part,
                           unsigned grid, cudaStream_t st) {
    switch (cfg) {
#define R3D_CFG_CASE(id, tx, ty, ry, ring, minb) \
    case id: batch_tile_vmax_kernel<Cfg##id><<<grid, Cfg##id::NT, 0, st>>>(members, tile0, nm, vmax_part); break;
        R3D_TILE_CFGS(R3D_CFG_CASE)
#undef R3D_CFG_CASE
        default: batch_tile_vmax_kernel<Cfg0><<<grid, Cfg0::NT, 0, st>>>(members, tile0, nm, vmax_part);
    }
    return 1;
}

int encode_plane_map(const Layout& L, const float* base, int cfg, CUtensorMap* out, std::string* why) {
    using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeFn encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            if (why) *why = "cuTensorMapEncodeTiled unavailable";
            return 1;
        }
        encode = reinterpret_cast<EncodeFn>(fn);
    }
    // strides must be multiples of 16 bytes and the base 16-byte aligned
    if ((L.px * 4) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) {
        if (why) *why = "field not 16-byte aligned for TMA";
        return 1;
    }
    const CfgInfo& c = info(cfg);
    const cuuint64_t dims[3] = {(cuuint64_t)L.px, (cuuint64_t)L.py, (cuuint64_t)L.pz};
    const cuuint64_t strides[2] = {(cuuint64_t)L.px * 4, (cuuint64_t)L.px * L.py * 4};
    const cuuint32_t box[3] = {(cuuint32_t)(c.tx + 8), (cuuint32_t)(c.ty + 6), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        if (why) *why = "cuTensorMapEncodeTiled failed";
        return 1;
    }
    return 0;
}

size_t tile_smem_bytes(int cfg) { return info(cfg).smem; }

dim3 tile_grid(const Layout& L, int kc, int cfg) {
    const CfgInfo& c = info(cfg);
    return dim3((L.nx + c.tx - 1) / c.tx, (L.ny + c.ty - 1) / c.ty, (L.nz + kc - 1) / kc);
}

int launch_tile_stage(const CUtensorMap& map, const TileArgs& a, int cfg, bool reini, int stage, bool volume,
                      cudaStream_t st) {
    tile_prepare();  // a failure here makes the launch below fail, which the caller reports
    const bool iso = tile_args_iso(a);
#define R3D_STAGE(C, I) launch_stage_cfg<C, I>(map, a, reini, stage, volume, st)
    switch (cfg) {
#define R3D_CFG_CASE(id, tx, ty, ry, ring, minb) \
    case id: if (iso) R3D_STAGE(Cfg##id, true); else R3D_STAGE(Cfg##id, false); break;
        R3D_TILE_CFGS(R3D_CFG_CASE)
#undef R3D_CFG_CASE
        default: if (iso) R3D_STAGE(Cfg0, true); else R3D_STAGE(Cfg0, false);
    }
#undef R3D_STAGE
    return 1;
}

}  // namespace r3d
