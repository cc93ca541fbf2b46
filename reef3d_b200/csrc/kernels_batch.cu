// Batched persistent kernels: many FP32 instances of uneven sizes, 2D and
// 3D mixed, advanced together.  The work of a stage is a packed list of
// tiles (32 x ROWS cells: x by y rows of one z plane in 3D, x by z rows in
// 2D) over all members; a persistent grid walks the list, each CTA looking
// up its member by binary search over the members' first tile index.
// Everything a member needs (fields, grid, its own dt, clock, velocity
// factor and reductions) is in its descriptor, so no value crosses members
// and a member's result does not depend on the batch around it: its tiles
// and its reductions are processed with the same arithmetic and in the same
// order alone or in any mix.
#include "batch_internal.h"
#include "cell_f32.cuh"

namespace r3d {
namespace {

using namespace f32c;

__device__ __forceinline__ int find_member(const long long* __restrict__ tile0, int nm, long long t) {
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile0[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int ROWS>
__device__ __forceinline__ void tile_cell(const MemberDesc& m, long long lt, int& i, int& j, int& k) {
    const Layout& L = m.g.L;
    const int tx = (L.nx + 31) / 32;
    if (L.two_d) {
        const int tz = (int)(lt / tx), bx = (int)(lt % tx);
        i = bx * 32 + (threadIdx.x & 31);
        j = 0;
        k = tz * ROWS + (threadIdx.x >> 5);
    } else {
        const int ty = (L.ny + ROWS - 1) / ROWS;
        const long long per_plane = (long long)tx * ty;
        k = (int)(lt / per_plane);
        const int r = (int)(lt % per_plane);
        const int by = r / tx, bx = r % tx;
        i = bx * 32 + (threadIdx.x & 31);
        j = by * ROWS + (threadIdx.x >> 5);
    }
}

// Deterministic CTA sum of two doubles (fixed tree); thread 0 writes.
template <int ROWS>
__device__ __forceinline__ void cta_sum2(double a, double b, double* dst) {
    __shared__ double sa[ROWS], sb[ROWS];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sa[warp] = a; sb[warp] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int q = 0; q < ROWS; ++q) { x += sa[q]; y += sb[q]; }
        dst[0] = x;
        dst[1] = y;
    }
    __syncthreads();
}

// One RK stage of every member.  conv: convection stage; else reinit
// pseudo-step q (members with f44 <= q sit it out).
template <int ROWS>
__global__ void __launch_bounds__(32 * ROWS) batch_stage_kernel(const MemberDesc* __restrict__ members,
                                                                const long long* __restrict__ tile0, int nm,
                                                                long long t_begin, long long ntiles, int conv,
                                                                int stage, int q, double* __restrict__ partial) {
    __shared__ MemberDesc sm;
    for (long long t = t_begin + blockIdx.x; t < ntiles; t += gridDim.x) {
        const int mi = find_member(tile0, nm, t);
        __syncthreads();
        if (threadIdx.x == 0) sm = members[mi];
        __syncthreads();
        const MemberDesc& m = sm;
        if (!conv && m.f44 <= q) continue;  // uniform across the CTA
        const bool volume = stage == 3 && (conv ? m.f44 == 0 : q == m.f44 - 1);
        int i, j, k;
        tile_cell<ROWS>(m, t - tile0[mi], i, j, k);
        const Layout& L = m.g.L;
        const bool active = i < L.nx && j < L.ny && k < L.nz;
        double v1 = 0.0, v2 = 0.0;
        if (active) {
            const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
            const float* fs = stage == 1 ? m.phi : stage == 2 ? m.a1 : m.a2;
            float* out = stage == 1 ? m.a1 : stage == 2 ? m.a2 : m.phi;
            float Lc, dtc;
            const bool uni = m.g.h[0] > 0.0f;
            if (conv) {
                const float vs = (float)*m.vscale;
                if (L.two_d) Lc = uni ? conv_L<true, true>(m.g, fs, m.u, m.v, m.w, c, i, j, k, vs)
                                      : conv_L<true, false>(m.g, fs, m.u, m.v, m.w, c, i, j, k, vs);
                else Lc = uni ? conv_L<false, true>(m.g, fs, m.u, m.v, m.w, c, i, j, k, vs)
                              : conv_L<false, false>(m.g, fs, m.u, m.v, m.w, c, i, j, k, vs);
                dtc = (float)*m.dt;
            } else {
                if (L.two_d) {
                    Lc = uni ? reini_L<true, true>(m.g, fs, c, i, j, k) : reini_L<true, false>(m.g, fs, c, i, j, k);
                    dtc = reini_dt32<true>(m.g, i, j, k);
                } else {
                    Lc = uni ? reini_L<false, true>(m.g, fs, c, i, j, k) : reini_L<false, false>(m.g, fs, c, i, j, k);
                    dtc = reini_dt32<false>(m.g, i, j, k);
                }
            }
            const float fn = m.phi[c];
            float val;
            if (stage == 1) val = fn + dtc * Lc;
            else if (stage == 2) val = 0.75f * fn + 0.25f * (__ldg(fs + c) + dtc * Lc);
            else val = (1.0f / 3.0f) * fn + (2.0f / 3.0f) * (__ldg(fs + c) + dtc * Lc);
            out[c] = val;
            if (i == 0) { out[c - 1] = val; out[c - 2] = val; out[c - 3] = val; }
            if (i == L.nx - 1) { out[c + 1] = val; out[c + 2] = val; out[c + 3] = val; }
            if (!L.two_d) {
                if (j == 0) { out[c - L.sy] = val; out[c - 2 * L.sy] = val; out[c - 3 * L.sy] = val; }
                if (j == L.ny - 1) { out[c + L.sy] = val; out[c + 2 * L.sy] = val; out[c + 3 * L.sy] = val; }
            }
            if (k == 0) { out[c - L.sz] = val; out[c - 2 * L.sz] = val; out[c - 3 * L.sz] = val; }
            if (k == L.nz - 1) { out[c + L.sz] = val; out[c + 2 * L.sz] = val; out[c + 3 * L.sz] = val; }
            if (volume) {
                const double PI_REF = 3.14159265359;  // src/definitions.h:37
                const double p = val, psi = m.g.psi;
                double H = 0.0;
                if (p > psi) H = 1.0;
                if (p < -psi) H = 0.0;
                if (fabs(p) <= psi) H = 0.5 * (1.0 + p / psi + (1.0 / PI_REF) * sin((PI_REF * p) / psi));
                const double vol = __ldg(m.g.dxn_d[0] + i + 5) * __ldg(m.g.dxn_d[1] + j + 5) *
                                   __ldg(m.g.dxn_d[2] + k + 5);
                v1 = vol * H;
                v2 = vol * (1.0 - H);
            }
        }
        if (volume) cta_sum2<ROWS>(v1, v2, partial + 2 * t);
    }
}

// Per-tile face maxima for the CFL step (x faces 0..nx-2, y 0..ny-2,
// z 0..nz-2, src/ietimestep.cpp:72-88), written to the tile's slots.
template <int ROWS>
__global__ void __launch_bounds__(32 * ROWS) batch_vmax_kernel(const MemberDesc* __restrict__ members,
                                                               const long long* __restrict__ tile0, int nm,
                                                               long long t_begin, long long ntiles,
                                                               double* __restrict__ partial) {
    __shared__ MemberDesc sm;
    __shared__ double s[3][ROWS];
    for (long long t = t_begin + blockIdx.x; t < ntiles; t += gridDim.x) {
        const int mi = find_member(tile0, nm, t);
        __syncthreads();
        if (threadIdx.x == 0) sm = members[mi];
        __syncthreads();
        const MemberDesc& m = sm;
        int i, j, k;
        tile_cell<ROWS>(m, t - tile0[mi], i, j, k);
        const Layout& L = m.g.L;
        double mu = 0.0, mv = 0.0, mw = 0.0;
        if (i < L.nx && j < L.ny && k < L.nz) {
            const long long c = (long long)(k + L.gz) * L.sz + (long long)(j + L.gy) * L.sy + (i + L.gx);
            if (i < L.nx - 1) mu = fabs((double)m.u[c]);
            if (j < L.ny - 1) mv = fabs((double)m.v[c]);
            if (k < L.nz - 1) mw = fabs((double)m.w[c]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            mu = fmax(mu, __shfl_down_sync(0xffffffffu, mu, o));
            mv = fmax(mv, __shfl_down_sync(0xffffffffu, mv, o));
            mw = fmax(mw, __shfl_down_sync(0xffffffffu, mw, o));
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) { s[0][warp] = mu; s[1][warp] = mv; s[2][warp] = mw; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int q = 1; q < ROWS; ++q) { mu = fmax(mu, s[0][q]); mv = fmax(mv, s[1][q]); mw = fmax(mw, s[2][q]); }
            partial[3 * t] = mu;
            partial[3 * t + 1] = mv;
            partial[3 * t + 2] = mw;
        }
    }
}

// One CTA per member: mode 0 reduces the tile maxima to the member's dt
// (src/ietimestep.cpp:160-188); mode 1 reduces the volume partials of the
// member's tiles in a fixed order, advances its clock by dt and updates its
// velocity factor.
__global__ void __launch_bounds__(256) batch_member_kernel(const MemberDesc* __restrict__ members,
                                                           const long long* __restrict__ tile0, int nm, int mode,
                                                           const double* __restrict__ vmax_part,
                                                           const double* __restrict__ vol_part) {
    const int mi = blockIdx.x;
    if (mi >= nm) return;
    const MemberDesc& m = members[mi];
    const long long t0 = tile0[mi], t1 = tile0[mi + 1];
    __shared__ double s0[256], s1[256], s2[256];
    double a = 0.0, b = 0.0, c = 0.0;
    for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        if (mode == 0) {
            a = fmax(a, vmax_part[3 * t]);
            b = fmax(b, vmax_part[3 * t + 1]);
            c = fmax(c, vmax_part[3 * t + 2]);
        } else {
            a += vol_part[2 * t];
            b += vol_part[2 * t + 1];
        }
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = b;
    s2[threadIdx.x] = c;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) {
            if (mode == 0) {
                s0[threadIdx.x] = fmax(s0[threadIdx.x], s0[threadIdx.x + st]);
                s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + st]);
                s2[threadIdx.x] = fmax(s2[threadIdx.x], s2[threadIdx.x + st]);
            } else {
                s0[threadIdx.x] += s0[threadIdx.x + st];
                s1[threadIdx.x] += s1[threadIdx.x + st];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (mode == 0) {
            const double sc = fabs(*m.vscale);
            const double umax = sc * s0[0], vmax = sc * s1[0], wmax = sc * s2[0];
            double cu = 1.0e10;
            const double cand = 2.0 / ((sqrt(umax * umax + vmax * vmax + wmax * wmax)) / m.dxmin +
                                       sqrt((4.0 * fabs(0.0)) / m.dxmin));
            cu = cu < cand ? cu : cand;
            *m.dt = m.n47 * cu;
        } else {
            m.vol[0] = s0[0];
            m.vol[1] = s1[0];
            *m.t += *m.dt;
            if (m.period > 0.0) *m.vscale = cos(3.141592653589793 * *m.t / m.period);
        }
    }
}

}  // namespace

long long batch_tiles_of(const Layout& L, int rows) {
    const long long tx = (L.nx + 31) / 32;
    if (L.two_d) return tx * ((L.nz + rows - 1) / rows);
    return tx * ((L.ny + rows - 1) / rows) * L.nz;
}

int launch_batch_stage(const BatchLaunch& b, int conv, int stage, int q, cudaStream_t st) {
    const dim3 grid(b.grid), block(32 * b.rows);
    switch (b.rows) {
        case 2: batch_stage_kernel<2><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, conv, stage, q, b.vol_part); break;
        case 8: batch_stage_kernel<8><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, conv, stage, q, b.vol_part); break;
        default: batch_stage_kernel<4><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, conv, stage, q, b.vol_part); break;
    }
    return 1;
}

int launch_batch_vmax(const BatchLaunch& b, cudaStream_t st) {
    const dim3 grid(b.grid), block(32 * b.rows);
    switch (b.rows) {
        case 2: batch_vmax_kernel<2><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, b.vmax_part); break;
        case 8: batch_vmax_kernel<8><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, b.vmax_part); break;
        default: batch_vmax_kernel<4><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, b.vmax_part); break;
    }
    return 1;
}

int launch_batch_dt(const BatchLaunch& b, cudaStream_t st) {
    batch_member_kernel<<<b.nm, 256, 0, st>>>(b.members, b.tile0, b.nm, 0, b.vmax_part, b.vol_part);
    return 1;
}

int launch_batch_cfl(const BatchLaunch& b, cudaStream_t st) {
    const dim3 grid(b.grid), block(32 * b.rows);
    switch (b.rows) {
        case 2: batch_vmax_kernel<2><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, b.vmax_part); break;
        case 8: batch_vmax_kernel<8><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, b.vmax_part); break;
        default: batch_vmax_kernel<4><<<grid, block, 0, st>>>(b.members, b.tile0, b.nm, b.t_begin, b.ntiles, b.vmax_part); break;
    }
    batch_member_kernel<<<b.nm, 256, 0, st>>>(b.members, b.tile0, b.nm, 0, b.vmax_part, b.vol_part);
    return 2;
}

int launch_batch_finish(const BatchLaunch& b, cudaStream_t st) {
    batch_member_kernel<<<b.nm, 256, 0, st>>>(b.members, b.tile0, b.nm, 1, b.vmax_part, b.vol_part);
    return 1;
}

}  // namespace r3d
