// Fused 2D TMz step (Ez, Hx, Hy) over a strip table: one launch advances every grid of a batch.
//
// The batch is a set of independent 2D grids of any sizes. Each grid keeps its own plan (fields, CPML
// memories, sources, monitors in its own arena); the kernel receives a table of their Grid structs and a
// table of strips (grid index, x0, y0, y1). Uneven grids therefore share one launch with no per-grid launch
// or cohort (reference: grouped_batch.py:38-77 runs each distinct shape as its own cohort, tensor_batch.py:
// 45-113 one kernel per cohort).
//
// One warp owns one strip: 31 columns [x0, x0+31) and rows [y0, y1). Lane l holds column x0+l; lane 31 is
// the +x halo whose new Ez the Hy update of lane 30 needs (it is computed, never stored). The warp marches
// along y with no shared memory and no block barrier: at row y it has Hx, Hy, Ez and 1/eps of row y in
// registers (coalesced 128-byte rows, loaded K rows ahead), takes Hy(x-1) from the lane below by shuffle
// (lane 0 loads it), computes Ez_new(y) with Hx(y-1) kept from the previous row, and then finishes the H
// update of row y-1, which needed Ez_new of rows y-1 and y (and Ez_new(x+1) by shuffle). Row y1 is a halo
// row: its Ez_new is computed for Hx(y1-1) and not stored. E and H are double-buffered over steps
// (parity = step & 1) and the E-family CPML memories too, so strips never wait on each other; H-family
// memories are updated in place by their owning lane only.
//
// Arithmetic in the reference order (torchfdtd/boundaries.py:363-438): for Ez the terms dx(Hy) then
// -dy(Hx), for Hx the term dy(Ez), for Hy the term -dx(Ez), CPML psi = psi*b + c*d; d = d/kappa + psi on the
// slabs, soft sources added after each family's update (E sources before Ez_new feeds the H update).
// Grids of a batch may have different step counts: a grid whose run has ended is skipped, so its state stays
// that of its last step while longer grids continue. Supported: x/y faces PML or PEC (periodic 2D grids run
// the gather kernel). A grid on a nonuniform mesh has no interior strips: the general path multiplies each
// plain difference by the metric factor of the updated cell before its CPML terms.
#pragma once
#include <algorithm>

#include "internal.cuh"

namespace tfd {

constexpr int k2dOwnX = 31;
constexpr int k2dWarps = 8;
constexpr int k2dThreads = 32 * k2dWarps;
constexpr int k2dRowsAhead = 3;                  // rows in flight in the interior path (FP32)

// Default rows per strip for a strip table covering `cells` cells: about 4 strips per resident warp of a
// B200 (148 SMs x 24 warps), at least 8 rows (the halo row costs 1/rows extra E work), at most 128.
inline int strip_rows(long long cells) {
    const long long target = 148LL * 24 * 4;
    const long long rows = (cells + (long long)k2dOwnX * target - 1) / ((long long)k2dOwnX * target);
    return (int)std::max(8LL, std::min(128LL, rows));
}

// A strip: owned columns [x0, x0+31), rows [y0, y1). kind 1: an interior strip (no CPML slab, grid edge or
// source meets it; the host checks), run by the lean path; kind 0: the general path.
struct Tile2D { int grid, x0, y0, y1, kind; };

template <typename T>
struct Row2D { T hx, hy, ez, ie, hyl; };

// Interior strip: every lane's column and every row (the halo row y1 included) lies inside the grid with
// x-1 and y-1 present, and no CPML slab or source meets the strip, so the update is the bare stencil with
// the general path's operation order. Row offsets stay 32-bit (the plan checks nx * ny < 2^31).
template <typename T>
__device__ __forceinline__ void strip_interior(const Grid<T> &g, const Tile2D &st, int par, int lane) {
    constexpr unsigned kAll = 0xffffffffu;
    constexpr int K = sizeof(T) == 4 ? k2dRowsAhead : 2;   // rows in flight (a ring of K row slots)
    const int pitch = g.pitch;
    const int base = st.y0 * pitch + st.x0 + lane;
    const T *__restrict__ Hx = g.H[par][0] + base;
    const T *__restrict__ Hy = g.H[par][1] + base;
    const T *__restrict__ Ez = g.E[par][2] + base;
    const T *__restrict__ iep = g.inv_eps[2] + base;
    T *__restrict__ Hxn = g.H[par ^ 1][0] + base;
    T *__restrict__ Hyn = g.H[par ^ 1][1] + base;
    T *__restrict__ Ezn = g.E[par ^ 1][2] + base;
    const T cn = g.cn;
    const bool own = lane < k2dOwnX;
    const int rows = st.y1 - st.y0;                    // owned rows; row `rows` is the halo row
    T hx_prev = Hx[-pitch];
    T hy_prev = T(0), ez_prev = T(0);
    auto load = [&](Row2D<T> &r, int k) {
        const bool live = k <= rows;
        const int o = k * pitch;
        r.hx = live ? Hx[o] : T(0);
        r.hy = live ? Hy[o] : T(0);
        r.ez = live ? Ez[o] : T(0);
        r.ie = live ? iep[o] : T(0);
        r.hyl = (live && lane == 0) ? Hy[o - 1] : T(0);
    };
    Row2D<T> ring[K];
#pragma unroll
    for (int k = 0; k < K; ++k) load(ring[k], k);
    for (int rb = 0; rb <= rows; rb += K) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int r = rb + k;
            if (r > rows) break;                       // warp-uniform
            const Row2D<T> c = ring[k];
            load(ring[k], r + K);                      // refill the slot K rows ahead
            T hy_left = __shfl_up_sync(kAll, c.hy, 1);
            if (lane == 0) hy_left = c.hyl;
            T acc = T(0) + (c.hy - hy_left);
            acc = acc + (-(c.hx - hx_prev));
            const T ez_new = c.ez + (cn * c.ie) * acc;
            const int o = r * pitch;
            if (own && r < rows) Ezn[o] = ez_new;
            const T ez_right = __shfl_down_sync(kAll, ez_prev, 1);
            if (r > 0) {
                const T hxn = hx_prev - cn * (T(0) + (ez_new - ez_prev));
                const T hyn = hy_prev - cn * (T(0) + (-(ez_right - ez_prev)));
                if (own) {
                    Hxn[o - pitch] = hxn;
                    Hyn[o - pitch] = hyn;
                }
            }
            hx_prev = c.hx;
            hy_prev = c.hy;
            ez_prev = ez_new;
        }
    }
}

// Everything of row y the general path reads, fetched K rows ahead: the fields, Hy(x-1) for lane 0, the
// E-family CPML memories of row y (x slab of this lane, y slab of this row) and the H-family memories of
// row y-1, which this iteration completes, with the y-slab rows of both.
template <typename T>
struct GRow2D {
    T hx, hy, ez, ie, hyl, pex, pey, phx, phy;
    int rye, ryh;
};

template <typename T>
__device__ __forceinline__ void strip_general(const Grid<T> &g, const Tile2D &st, long long n, int par, int lane) {
    constexpr unsigned kAll = 0xffffffffu;
    constexpr int K = 2;
    const long long steps = g.steps;
    const int nx = g.n[0], ny = g.n[1], pitch = g.pitch;
    const int x = st.x0 + lane, y0 = st.y0, y1 = st.y1;
    const bool in_x = x < nx;
    const bool own = in_x && lane < k2dOwnX;
    const T *__restrict__ Hx = g.H[par][0];
    const T *__restrict__ Hy = g.H[par][1];
    const T *__restrict__ Ez = g.E[par][2];
    const T *__restrict__ iep = g.inv_eps[2];
    T *__restrict__ Hxn = g.H[par ^ 1][0];
    T *__restrict__ Hyn = g.H[par ^ 1][1];
    T *__restrict__ Ezn = g.E[par ^ 1][2];
    const T cn = g.cn;
    // x-axis CPML of this lane: E term of Ez (axis 0, j 1) and H term of Hy (axis 0, j 0).
    const int *rxp_e = g.row[0][0], *rxp_h = g.row[1][0];
    const int rxE = (rxp_e != nullptr && in_x && x > 0) ? rxp_e[x] : -1;
    const int rxH = (rxp_h != nullptr && in_x && x < nx - 1) ? rxp_h[x] : -1;
    T bxE = T(0), cxE = T(0), kxE = T(0), bxH = T(0), cxH = T(0), kxH = T(0);
    if (rxE >= 0) { bxE = g.cb[0][0][x]; cxE = g.cc[0][0][x]; kxE = g.ck[0][0][x]; }
    if (rxH >= 0) { bxH = g.cb[1][0][x]; cxH = g.cc[1][0][x]; kxH = g.ck[1][0][x]; }
    const int RxE = g.rows[0][0], RxH = g.rows[1][0];
    const int *ryp_e = g.row[0][1], *ryp_h = g.row[1][1];
    const T *psiEx = g.psiE[par][0][1];
    T *psiExn = g.psiE[par ^ 1][0][1];
    const T *psiEy = g.psiE[par][1][1];
    T *psiEyn = g.psiE[par ^ 1][1][1];
    T *psiHy = g.psiH[1][0];                           // Hx term dy(Ez), updated in place
    T *psiHx = g.psiH[0][0];                           // Hy term dx(Ez), updated in place
    const bool pec_x = g.pec_on[0] != 0, pec_y = g.pec_on[1] != 0;
    const T pneg_x = g.pec_neg[0], pneg_y = g.pec_neg[1];
    // Nonuniform mesh: x factors of this lane's column, y factors read per row (nullptr: uniform axis).
    const T *my_e = g.metric[0][1], *my_h = g.metric[1][1];
    const T mx_e = (g.metric[0][0] != nullptr && in_x) ? g.metric[0][0][x] : T(1);
    const T mx_h = (g.metric[1][0] != nullptr && in_x) ? g.metric[1][0][x] : T(1);
    const bool mx = g.metric[0][0] != nullptr;
    // Sources meeting this strip (E with the halo lane and halo row), tested once per strip.
    unsigned src_e = 0, src_hx = 0, src_hy = 0;
    for (int t = 0; t < g.n_src; ++t) {
        const SourceTerm &q = g.src[t];
        const bool hit_e = q.lo[0] < st.x0 + 32 && st.x0 < q.hi[0] && q.lo[1] <= y1 && y0 < q.hi[1];
        const bool hit_h = q.lo[0] < st.x0 + k2dOwnX && st.x0 < q.hi[0] && q.lo[1] < y1 && y0 < q.hi[1];
        if (q.family == 0 && q.comp == 2 && hit_e) src_e |= 1u << t;
        if (q.family == 1 && q.comp == 0 && hit_h) src_hx |= 1u << t;
        if (q.family == 1 && q.comp == 1 && hit_h) src_hy |= 1u << t;
    }
    auto add_sources = [&](unsigned mask, int y, T v) {
        for (; mask; mask &= mask - 1) {
            const int t = __ffs(mask) - 1;
            const SourceTerm &q = g.src[t];
            if (x >= q.lo[0] && x < q.hi[0] && y >= q.lo[1] && y < q.hi[1]) v = v + g.src_values[(long long)t * steps + n];
        }
        return v;
    };
    auto load = [&](GRow2D<T> &r, int y) {
        const bool row = y <= y1 && y < ny;            // E row y exists in this strip
        const bool live = row && in_x;
        const long long i = (long long)y * pitch + x;
        r.hx = live ? Hx[i] : T(0);
        r.hy = live ? Hy[i] : T(0);
        r.ez = live ? Ez[i] : T(0);
        r.ie = live ? iep[i] : T(0);
        r.hyl = (row && lane == 0 && x > 0) ? Hy[i - 1] : T(0);
        r.pex = (live && rxE >= 0) ? psiEx[(long long)y * RxE + rxE] : T(0);
        r.rye = (row && ryp_e != nullptr && y > 0) ? ryp_e[y] : -1;
        r.pey = (r.rye >= 0 && in_x) ? psiEy[(long long)r.rye * pitch + x] : T(0);
        const int h = y - 1;                           // H row completed at iteration y
        const bool hrow = y > y0 && y <= y1;
        r.ryh = (hrow && ryp_h != nullptr && h < ny - 1) ? ryp_h[h] : -1;
        r.phy = (r.ryh >= 0 && in_x) ? psiHy[(long long)r.ryh * pitch + x] : T(0);
        r.phx = (hrow && rxH >= 0) ? psiHx[(long long)h * RxH + rxH] : T(0);
    };

    T hx_prev = (y0 > 0 && in_x) ? Hx[(long long)(y0 - 1) * pitch + x] : T(0);   // Hx_old(y-1)
    T hy_prev = T(0), ez_prev = T(0);                 // Hy_old(y-1), Ez_new(y-1)
    GRow2D<T> ring[K];
#pragma unroll
    for (int k = 0; k < K; ++k) load(ring[k], y0 + k);
    for (int yb = y0; yb <= y1; yb += K) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int y = yb + k;
            if (y > y1) break;                         // warp-uniform
            const GRow2D<T> r = ring[k];
            load(ring[k], y + K);                      // refill the slot K rows ahead
            T ez_new = T(0);
            if (y < ny) {
                T hy_left = __shfl_up_sync(kAll, r.hy, 1);
                if (lane == 0) hy_left = r.hyl;
                // Ez: dx(Hy) ...
                T d = x > 0 ? r.hy - hy_left : T(0);
                if (mx && x > 0) d = d * mx_e;
                if (rxE >= 0) {
                    const T mem = r.pex * bxE + cxE * d;
                    if (own && y < y1) psiExn[(long long)y * RxE + rxE] = mem;
                    d = d * kxE + mem;
                }
                T acc = T(0) + d;
                // ... then -dy(Hx)
                d = y > 0 ? r.hx - hx_prev : T(0);
                if (my_e != nullptr && y > 0) d = d * my_e[y];
                if (r.rye >= 0 && in_x) {
                    const T mem = r.pey * g.cb[0][1][y] + g.cc[0][1][y] * d;
                    if (own && y < y1) psiEyn[(long long)r.rye * pitch + x] = mem;
                    d = d * g.ck[0][1][y] + mem;
                }
                acc = acc + (-d);
                ez_new = r.ez + (cn * r.ie) * acc;
                if (src_e) ez_new = add_sources(src_e, y, ez_new);
                if (own && y < y1) Ezn[(long long)y * pitch + x] = ez_new;
            }
            const T ez_right = __shfl_down_sync(kAll, ez_prev, 1);
            if (y > y0) {
                const int h = y - 1;                   // the H row this iteration completes
                // Hx: dy(Ez)
                T d = T(0);
                if (h < ny - 1) {
                    d = ez_new - ez_prev;
                    if (my_h != nullptr) d = d * my_h[h];
                    if (r.ryh >= 0 && in_x) {
                        const T mem = r.phy * g.cb[1][1][h] + g.cc[1][1][h] * d;
                        if (own) psiHy[(long long)r.ryh * pitch + x] = mem;
                        d = d * g.ck[1][1][h] + mem;
                    }
                } else if (pec_y) {
                    d = pneg_y * ez_prev;
                }
                T acc = T(0) + d;
                T hxn = hx_prev - cn * acc;
                // Hy: -dx(Ez)
                d = T(0);
                if (x < nx - 1) {
                    d = ez_right - ez_prev;
                    if (mx) d = d * mx_h;
                    if (rxH >= 0) {
                        const T mem = r.phx * bxH + cxH * d;
                        if (own) psiHx[(long long)h * RxH + rxH] = mem;
                        d = d * kxH + mem;
                    }
                } else if (pec_x) {
                    d = pneg_x * ez_prev;
                }
                acc = T(0) + (-d);
                T hyn = hy_prev - cn * acc;
                if (src_hx) hxn = add_sources(src_hx, h, hxn);
                if (src_hy) hyn = add_sources(src_hy, h, hyn);
                if (own) {
                    const long long i = (long long)h * pitch + x;
                    Hxn[i] = hxn;
                    Hyn[i] = hyn;
                }
            }
            hx_prev = r.hx;
            hy_prev = r.hy;
            ez_prev = ez_new;
        }
    }
}

// Two kernels walk the two parts of a strip table, interior strips first: the lean path fits 64 registers
// (4 CTAs, 32 warps per SM), the general path gets up to 128. Both read only old-parity state and write
// disjoint owned cells, so they need no ordering between them within a step.
template <typename T>
__global__ void __launch_bounds__(k2dThreads, 4) k_step2d_interior(const Grid<T> *__restrict__ grids,
                                                                  const Tile2D *__restrict__ strips, int nstrips,
                                                                  const long long *counter) {
    const long long n = *counter;
    const int par = (int)(n & 1);
    const int lane = threadIdx.x & 31;
    const int warps_total = gridDim.x * k2dWarps;
    for (int s = blockIdx.x * k2dWarps + (threadIdx.x >> 5); s < nstrips; s += warps_total) {
        const Tile2D st = strips[s];
        const Grid<T> &g = grids[st.grid];
        if (n >= g.steps) continue;                    // this grid has finished its run (warp-uniform)
        // The lean path reads x0-1, x0+31, y0-1 and y1 unchecked: refuse a strip that is not interior.
        if (st.kind != 1 || st.x0 < 1 || st.x0 + 31 > g.n[0] - 1 || st.y0 < 1 || st.y1 > g.n[1] - 1 || st.y1 < st.y0) {
            if (lane == 0) atomicExch(g.status, kStatusBadStrip);
            continue;
        }
        strip_interior(g, st, par, lane);
    }
}

template <typename T>
__global__ void __launch_bounds__(k2dThreads, 2) k_step2d_general(const Grid<T> *__restrict__ grids,
                                                                 const Tile2D *__restrict__ strips, int nstrips,
                                                                 const long long *counter) {
    const long long n = *counter;
    const int par = (int)(n & 1);
    const int lane = threadIdx.x & 31;
    const int warps_total = gridDim.x * k2dWarps;
    for (int s = blockIdx.x * k2dWarps + (threadIdx.x >> 5); s < nstrips; s += warps_total) {
        const Tile2D st = strips[s];
        const Grid<T> &g = grids[st.grid];
        if (n >= g.steps) continue;
        strip_general(g, st, n, par, lane);
    }
}

}  // namespace tfd
