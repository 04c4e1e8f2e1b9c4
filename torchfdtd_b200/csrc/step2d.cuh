// Fused 2D TMz step (Ez, Hx, Hy) over a tile table: one launch advances every grid of a batch.
//
// The batch is a set of independent 2D grids of any sizes. Each grid keeps its own plan (fields, CPML
// memories, sources, monitors in its own arena); the kernel receives a table of their Grid structs and a
// table of tiles (grid index, x0, y0). A persistent grid of CTAs strides over the tiles, so uneven grids
// share one launch with no per-grid launch or cohort (reference: grouped_batch.py:38-77 runs each distinct
// shape as its own cohort, tensor_batch.py:45-113 one kernel per cohort).
//
// A tile owns 31 x 15 cells and computes Ez on 32 x 16 (lane 31 and row 15 are the +x / +y halo its H
// update borrows). Thread (lane, warp) holds one cell: H(x, y) and the x-1 / y-1 halo go to shared memory,
// Ez_new of the 32 x 16 tile goes to shared memory, then Hx, Hy of the owned cells. E and H are
// double-buffered over steps (parity = step & 1), so tiles never wait on each other. Arithmetic in the
// reference order (torchfdtd/boundaries.py:363-438): for Ez the terms dx(Hy) then -dy(Hx), for Hx the term
// dy(Ez), for Hy the term -dx(Ez), CPML on the slabs, soft sources after each family's update.
// Grids of a batch may have different step counts: a grid whose run has ended is skipped, so its state
// stays that of its last step while longer grids continue.
// Supported: x/y faces PML or PEC (periodic 2D grids run the gather kernel).
#pragma once
#include "internal.cuh"

namespace tfd {

constexpr int k2dLanes = 32, k2dRows = 16, k2dOwnX = 31, k2dOwnY = 15;
constexpr int k2dThreads = k2dLanes * k2dRows;

struct Tile2D { int grid, x0, y0, pad; };

template <typename T>
__device__ __forceinline__ T src2d(const Grid<T> &g, int comp_family, int comp, long long n, int x, int y, T v) {
    if (n < g.steps)
        for (int s = 0; s < g.n_src; ++s) {
            const SourceTerm &t = g.src[s];
            if (t.family == comp_family && t.comp == comp && x >= t.lo[0] && x < t.hi[0] && y >= t.lo[1] && y < t.hi[1])
                v = v + g.src_values[(long long)s * g.steps + n];
        }
    return v;
}

template <typename T>
__global__ void __launch_bounds__(k2dThreads) k_step2d_tm(const Grid<T> *__restrict__ grids, const Tile2D *__restrict__ tiles,
                                                         int ntiles, const long long *counter) {
    __shared__ T sHx[k2dRows + 1][k2dLanes];          // row 0 = y0-1
    __shared__ T sHy[k2dRows][k2dLanes + 1];          // column 0 = x0-1
    __shared__ T sEz[k2dRows][k2dLanes];
    const long long n = *counter;
    const int par = (int)(n & 1);
    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile2D tile = tiles[t];
        const Grid<T> &g = grids[tile.grid];
        if (n >= g.steps) continue;                   // this grid has finished its run (uniform per block)
        const int nx = g.n[0], ny = g.n[1], pitch = g.pitch;
        const int x = tile.x0 + lane, y = tile.y0 + r;
        const bool in = x < nx && y < ny;
        const bool own = in && lane < k2dOwnX && r < k2dOwnY;
        const long long i = (long long)y * pitch + x;
        const T *Hx = g.H[par][0], *Hy = g.H[par][1];
        T hx = T(0), hy = T(0), ez = T(0), ie = T(0);
        if (in) {
            hx = Hx[i];
            hy = Hy[i];
            ez = g.E[par][2][i];
            ie = g.inv_eps[2][i];
        }
        sHx[r + 1][lane] = hx;
        sHy[r][lane + 1] = hy;
        if (lane == 0) sHy[r][0] = (in && x > 0) ? Hy[i - 1] : T(0);
        if (r == 0) sHx[0][lane] = (in && y > 0) ? Hx[i - pitch] : T(0);
        __syncthreads();
        if (in) {
            // Ez: dx(Hy) then -dy(Hx) (reference curl-term order)
            T acc = T(0);
            T d = x > 0 ? sHy[r][lane + 1] - sHy[r][lane] : T(0);
            const int *rx = g.row[0][0];
            if (rx != nullptr && x > 0) {
                const int q = rx[x];
                if (q >= 0) {
                    const long long p = g.psi_index(0, x, y, 0, q, g.rows[0][0]);
                    const T mem = g.psiE[par][0][1][p] * g.cb[0][0][x] + g.cc[0][0][x] * d;
                    if (own) g.psiE[par ^ 1][0][1][p] = mem;
                    d = d * g.ck[0][0][x] + mem;
                }
            }
            acc = acc + d;
            d = y > 0 ? sHx[r + 1][lane] - sHx[r][lane] : T(0);
            const int *ry = g.row[0][1];
            if (ry != nullptr && y > 0) {
                const int q = ry[y];
                if (q >= 0) {
                    const long long p = g.psi_index(1, x, y, 0, q, g.rows[0][1]);
                    const T mem = g.psiE[par][1][1][p] * g.cb[0][1][y] + g.cc[0][1][y] * d;
                    if (own) g.psiE[par ^ 1][1][1][p] = mem;
                    d = d * g.ck[0][1][y] + mem;
                }
            }
            acc = acc + (-d);
            ez = ez + (g.cn * ie) * acc;
            if (g.n_src) ez = src2d(g, 0, 2, n, x, y, ez);
            sEz[r][lane] = ez;
            if (own) g.E[par ^ 1][2][i] = ez;
        }
        __syncthreads();
        if (own) {
            // Hx: dy(Ez)
            T d = T(0);
            if (y < ny - 1) {
                d = sEz[r + 1][lane] - sEz[r][lane];
                const int *ry = g.row[1][1];
                if (ry != nullptr) {
                    const int q = ry[y];
                    if (q >= 0) {
                        const long long p = g.psi_index(1, x, y, 0, q, g.rows[1][1]);
                        T *psi = g.psiH[1][0];
                        const T mem = psi[p] * g.cb[1][1][y] + g.cc[1][1][y] * d;
                        psi[p] = mem;
                        d = d * g.ck[1][1][y] + mem;
                    }
                }
            } else if (g.pec_on[1]) {
                d = g.pec_neg[1] * sEz[r][lane];
            }
            T acc = T(0) + d;
            T hxn = hx - g.cn * acc;
            // Hy: -dx(Ez)
            d = T(0);
            if (x < nx - 1) {
                d = sEz[r][lane + 1] - sEz[r][lane];
                const int *rx = g.row[1][0];
                if (rx != nullptr) {
                    const int q = rx[x];
                    if (q >= 0) {
                        const long long p = g.psi_index(0, x, y, 0, q, g.rows[1][0]);
                        T *psi = g.psiH[0][0];
                        const T mem = psi[p] * g.cb[1][0][x] + g.cc[1][0][x] * d;
                        psi[p] = mem;
                        d = d * g.ck[1][0][x] + mem;
                    }
                }
            } else if (g.pec_on[0]) {
                d = g.pec_neg[0] * sEz[r][lane];
            }
            acc = T(0) + (-d);
            T hyn = hy - g.cn * acc;
            if (g.n_src) {
                hxn = src2d(g, 1, 0, n, x, y, hxn);
                hyn = src2d(g, 1, 1, n, x, y, hyn);
            }
            g.H[par ^ 1][0][i] = hxn;
            g.H[par ^ 1][1][i] = hyn;
        }
        __syncthreads();
    }
}

}  // namespace tfd
