// 2D TMz stepping entirely on chip: one thread-block cluster holds a whole small grid in distributed shared
// memory and runs every step of a tfd_step call without touching HBM between steps.
//
// A 320 x 240 TMz grid is about 1.4 MB of fields, inverse permittivity and CPML memories: more than one CTA's
// shared memory, less than a cluster's (8 or 16 CTAs of up to 227 KB on a B200). Each CTA of the cluster owns a
// band of rows [r0, r1) and keeps Ez, Hx, Hy, 1/eps and the CPML memories of its rows in its own shared memory.
// A step is
//   E phase: Ez of every own cell from Hy (same row) and Hx (row y - 1: the CTA below for the first row, read
//            through distributed shared memory), the E-family CPML memories, the E soft sources;
//   cluster barrier;
//   H phase: Hx from Ez (row y + 1: the CTA above for the last row), Hy from Ez (x + 1), the H-family memories,
//            the H soft sources, then the point traces of the step (the owning CTA writes them to HBM);
//   cluster barrier.
// A warp takes a 32-column segment of a group of consecutive rows and marches up through them (E pass: Hx of the
// row below kept in a register; H pass: Ez of the row above), with the x neighbours by shuffle. Each phase
// reads only the other family, so the updates are in place. The arithmetic per cell is that of
// the strip kernels' general path (step2d.cuh: strip_general), so the fields are bitwise the same. The state
// is loaded from the parity the step counter names at the start of the launch and written back, with the
// counter, at the end. Scope: 2D TMz plans without DFT planes (the traces are the only observations).
#pragma once
#include <cooperative_groups.h>

#include "internal.cuh"

namespace tfd {

namespace cg = cooperative_groups;

constexpr int kCl2dThreads = 1024;
constexpr int kCl2dWarps = kCl2dThreads / 32;
constexpr int kCl2dMaxRanks = 16;

struct Cluster2D {
    int ranks;                       // CTAs in the cluster
    int r0[kCl2dMaxRanks + 1];       // band of rank c: rows [r0[c], r0[c + 1])
    int rows_max;                    // the largest band
    int w;                           // shared-memory row width (nx)
    int h;                           // rows of the grid (ny): length of the per-row coefficient tables
    int rx_e, rx_h;                  // x-slab memory widths (rows of both x slabs) of the E and H families
    int rye_lo[kCl2dMaxRanks], rye_n[kCl2dMaxRanks];   // per rank: first y-slab memory row of its band, count (E)
    int ryh_lo[kCl2dMaxRanks], ryh_n[kCl2dMaxRanks];   // the same for the H family
    int rye_max, ryh_max;
    int count;                       // steps of this launch
};

// Shared-memory arrays of one rank, at element offsets fixed by the launch (every rank uses the same layout, so
// a neighbour's row sits at the same offset in its shared memory). After the fields and memories: per family f
// and axis a (x: nx entries, y: ny entries) the CPML coefficients b, c, 1/kappa and the metric factor of each
// column / row (tab), and the memory row of each column / row (-1: no CPML term there; slab).
struct Cl2dLayout {
    int ez, hx, hy, ie, pex, pey, phx, phy;
    int tab[2][2];                   // 4 consecutive T arrays (b, c, k, metric) of n[a] entries
    int slab[2][2];                  // int arrays, element offsets from the start of the int region
    int ints;                        // start of the int region (in T elements)
    int total;                       // T elements including the int region
};

__host__ __device__ inline Cl2dLayout cl2d_layout(const Cluster2D &c, int tsize) {
    Cl2dLayout L;
    const int cells = c.rows_max * c.w;
    L.ez = 0;
    L.hx = L.ez + cells;
    L.hy = L.hx + cells;
    L.ie = L.hy + cells;
    L.pex = L.ie + cells;
    L.pey = L.pex + c.rows_max * c.rx_e;
    L.phx = L.pey + c.rye_max * c.w;
    L.phy = L.phx + c.rows_max * c.rx_h;
    int o = L.phy + c.ryh_max * c.w;
    int io = 0;
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 2; ++a) {
            const int n = a == 0 ? c.w : c.h;
            L.tab[f][a] = o;
            o += 4 * n;
            L.slab[f][a] = io;
            io += n;
        }
    L.ints = o;
    L.total = o + (io * 4 + tsize - 1) / tsize;
    return L;
}

template <typename T>
__global__ void __launch_bounds__(kCl2dThreads, 1) k_step2d_cluster(const __grid_constant__ Grid<T> g, const __grid_constant__ Cluster2D c,
                                                                   const TraceDev *__restrict__ traces, int n_traces, T *trace_out) {
    extern __shared__ __align__(16) unsigned char cl_raw[];
    T *const sm = reinterpret_cast<T *>(cl_raw);
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const Cl2dLayout L = cl2d_layout(c, (int)sizeof(T));
    const int nx = g.n[0], ny = g.n[1], W = c.w, pitch = g.pitch;
    const int r0 = c.r0[rank], r1 = c.r0[rank + 1], rows = r1 - r0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long n0 = *g.counter;
    const int par0 = (int)(n0 & 1);
    T *Ez = sm + L.ez, *Hx = sm + L.hx, *Hy = sm + L.hy, *ie = sm + L.ie;
    T *pex = sm + L.pex, *pey = sm + L.pey, *phx = sm + L.phx, *phy = sm + L.phy;
    int *const ints = reinterpret_cast<int *>(sm + L.ints);
    // The neighbours' bands: the last Hx row of the rank below, the first Ez row of the rank above.
    const T *hx_below = rank > 0 ? cluster.map_shared_rank(sm + L.hx, rank - 1) : nullptr;
    const T *ez_above = rank + 1 < c.ranks ? cluster.map_shared_rank(sm + L.ez, rank + 1) : nullptr;
    const int rows_below = rank > 0 ? c.r0[rank] - c.r0[rank - 1] : 0;
    const int RxE = g.rows[0][0], RxH = g.rows[1][0];

    // Load the band (parity par0) and its CPML memories.
    for (int q = tid; q < rows * W; q += kCl2dThreads) {
        const int y = r0 + q / W, x = q % W;
        const long long i = (long long)y * pitch + x;
        Ez[q] = g.E[par0][2][i];
        Hx[q] = g.H[par0][0][i];
        Hy[q] = g.H[par0][1][i];
        ie[q] = g.inv_eps[2][i];
    }
    if (RxE) for (int q = tid; q < rows * RxE; q += kCl2dThreads) pex[q] = g.psiE[par0][0][1][(long long)(r0 + q / RxE) * RxE + q % RxE];
    if (RxH) for (int q = tid; q < rows * RxH; q += kCl2dThreads) phx[q] = g.psiH[0][0][(long long)(r0 + q / RxH) * RxH + q % RxH];
    for (int q = tid; q < c.rye_n[rank] * W; q += kCl2dThreads) pey[q] = g.psiE[par0][1][1][(long long)(c.rye_lo[rank] + q / W) * pitch + q % W];
    for (int q = tid; q < c.ryh_n[rank] * W; q += kCl2dThreads) phy[q] = g.psiH[1][0][(long long)(c.ryh_lo[rank] + q / W) * pitch + q % W];
    // Coefficient tables. A column / row whose difference the update does not take (E: x = 0, y = 0; H: the last
    // column / row) gets no memory row, so the tables alone decide where CPML terms apply.
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 2; ++a) {
            const int len = a == 0 ? nx : ny;
            T *tb = sm + L.tab[f][a];
            int *ts = ints + L.slab[f][a];
            const int *rowp = g.row[f][a];
            const T *m = g.metric[f][a];
            for (int i = tid; i < len; i += kCl2dThreads) {
                const bool diff = f == 0 ? i > 0 : i < len - 1;
                const int r = (rowp != nullptr && diff) ? rowp[i] : -1;
                ts[i] = r;
                tb[i] = r >= 0 ? g.cb[f][a][i] : T(0);
                tb[len + i] = r >= 0 ? g.cc[f][a][i] : T(0);
                tb[2 * len + i] = r >= 0 ? g.ck[f][a][i] : T(1);
                tb[3 * len + i] = m != nullptr ? m[i] : T(1);
            }
        }
    // Sources that meet the band (E: its rows; H: its rows), tested once.
    unsigned src_e = 0, src_hx = 0, src_hy = 0;
    for (int t = 0; t < g.n_src; ++t) {
        const SourceTerm &s = g.src[t];
        const bool hit = s.lo[1] < r1 && r0 < s.hi[1];
        if (s.family == 0 && s.comp == 2 && hit) src_e |= 1u << t;
        if (s.family == 1 && s.comp == 0 && hit) src_hx |= 1u << t;
        if (s.family == 1 && s.comp == 1 && hit) src_hy |= 1u << t;
    }
    bool band_traces = false;
    for (int t = 0; t < n_traces; ++t) {
        const int y = (int)(traces[t].offset / pitch);
        band_traces |= y >= r0 && y < r1;
    }
    // Soft sources of a family, after its update pass: the cells of each source box in the band get the source
    // value added, one source after the other (ascending index, the order of the strip kernels), so each cell
    // sees the same additions in the same order as an update that adds them in place.
    // Source values of the step, loaded at its top by thread t for term t so that their latency overlaps the E
    // pass (a source mask has 32 bits, so at most 32 terms reach here).
    __shared__ T src_val[32];
    const unsigned src_any = src_e | src_hx | src_hy;
    auto add_sources = [&](unsigned mask, T *field, long long n) {
        for (; mask; mask &= mask - 1) {
            const int t = __ffs(mask) - 1;
            const SourceTerm &s = g.src[t];
            const int ylo = max(s.lo[1], r0), yhi = min(s.hi[1], r1), xlo = max(s.lo[0], 0), xhi = min(s.hi[0], nx);
            const int w = xhi - xlo, cnt = (w > 0 && yhi > ylo) ? w * (yhi - ylo) : 0;
            __syncthreads();
            const T v = src_val[t];                   // prefetched at the top of the step
            for (int q = tid; q < cnt; q += kCl2dThreads) {
                const int e = (ylo - r0 + q / w) * W + xlo + q % w;
                field[e] = field[e] + v;
            }
        }
    };
    const bool pec_x = g.pec_on[0] != 0, pec_y = g.pec_on[1] != 0;
    const T pneg_x = g.pec_neg[0], pneg_y = g.pec_neg[1], cn = g.cn;
    const bool mx_e = g.metric[0][0] != nullptr, my_e = g.metric[0][1] != nullptr;
    const bool mx_h = g.metric[1][0] != nullptr, my_h = g.metric[1][1] != nullptr;
    const T *const xb_e = sm + L.tab[0][0], *const yb_e = sm + L.tab[0][1];
    const T *const xb_h = sm + L.tab[1][0], *const yb_h = sm + L.tab[1][1];
    const int *const xs_e = ints + L.slab[0][0], *const ys_e = ints + L.slab[0][1];
    const int *const xs_h = ints + L.slab[1][0], *const ys_h = ints + L.slab[1][1];
    // Work units: a warp takes a 32-column segment (cg) of a group of consecutive rows (rg) and marches up
    // through its rows, keeping the row below (E pass: Hx(y-1)) or above (H pass: Ez(y+1)) in registers and
    // taking the x neighbours by shuffle. XU segments per row, RG row groups (as many as the warps allow), each
    // of RPG rows; unit u = w, w + 32, ... is segment u % XU of row group u / XU.
    const int XU = (nx + 31) / 32;
    const int RG = max(1, min(rows, kCl2dWarps / XU));
    const int RPG = (rows + RG - 1) / RG;
    const int units = XU * RG;
    cluster.sync();                                       // every band and table loaded before any neighbour reads it

    // Point traces: a thread keeps the band-local index of its trace (-1: another band's cell) and the field.
    int tr_e = -1, tr_f = 0;
    if (tid < n_traces) {
        const TraceDev tr = traces[tid];
        const int y = (int)(tr.offset / pitch), x = (int)(tr.offset % pitch);
        if (y >= r0 && y < r1) tr_e = (y - r0) * W + x;
        tr_f = (tr.family == 0 && tr.comp == 2) ? 1 : (tr.family == 1 && tr.comp == 0) ? 2 : (tr.family == 1 && tr.comp == 1) ? 3 : 0;
    }
    long long n = n0;
    for (int k = 0; k < c.count && n < g.steps; ++k, ++n) {
        if (tid < 32 && ((src_any >> tid) & 1u)) src_val[tid] = g.src_values[(long long)tid * g.steps + n];
        // ---- E pass ----
        for (int u = warp; u < units; u += kCl2dWarps) {
            const int x = (u % XU) * 32 + lane, ylo = (u / XU) * RPG, yhi = min(ylo + RPG, rows);
            const bool in = x < nx;
            // This lane's x terms: CPML row and coefficients, metric factor.
            const int rxE = in ? xs_e[x] : -1;
            // A plain segment: every lane has its -x neighbour and no x memory, on a uniform mesh; its rows clear of
            // the y slabs and the y = 0 face take the bare update (the general arithmetic reduces to it there).
            const bool xplain = __all_sync(0xffffffffu, in && x > 0 && rxE < 0) && !mx_e && !my_e;
            T bx = T(0), cx = T(0), kx = T(1), mxv = T(1);
            if (rxE >= 0) { bx = xb_e[x]; cx = xb_e[nx + x]; kx = xb_e[2 * nx + x]; }
            if (mx_e && in) mxv = xb_e[3 * nx + x];
            // Hx of the row below the group: this band's row, the band below (DSMEM), or none at y = 0.
            T hx_prev = T(0);
            if (in && ylo > 0 && ylo <= rows) hx_prev = Hx[(ylo - 1) * W + x];
            else if (in && hx_below != nullptr) hx_prev = hx_below[(rows_below - 1) * W + x];
            for (int yl = ylo; yl < yhi; ++yl) {
                const int y = r0 + yl, e = yl * W + x;
                const T hy = in ? Hy[e] : T(0);
                const T hx = in ? Hx[e] : T(0);
                T hy_left = __shfl_up_sync(0xffffffffu, hy, 1);
                if (lane == 0 && x > 0 && in) hy_left = Hy[e - 1];
                if (xplain && y > 0 && ys_e[y] < 0) {
                    T acc = T(0) + (hy - hy_left);
                    acc = acc + (-(hx - hx_prev));
                    Ez[e] = Ez[e] + (cn * ie[e]) * acc;
                } else if (in) {
                    T d = x > 0 ? hy - hy_left : T(0);
                    if (mx_e && x > 0) d = d * mxv;
                    if (rxE >= 0) {
                        const T mem = pex[yl * RxE + rxE] * bx + cx * d;
                        pex[yl * RxE + rxE] = mem;
                        d = d * kx + mem;
                    }
                    T acc = T(0) + d;
                    d = y > 0 ? hx - hx_prev : T(0);
                    if (my_e && y > 0) d = d * yb_e[3 * ny + y];
                    const int rye = ys_e[y];
                    if (rye >= 0) {
                        const int pi = (rye - c.rye_lo[rank]) * W + x;
                        const T mem = pey[pi] * yb_e[y] + yb_e[ny + y] * d;
                        pey[pi] = mem;
                        d = d * yb_e[2 * ny + y] + mem;
                    }
                    acc = acc + (-d);
                    Ez[e] = Ez[e] + (cn * ie[e]) * acc;
                }
                hx_prev = hx;
            }
        }
        if (src_e) add_sources(src_e, Ez, n);             // CTA-uniform
        // A CTA enters the cluster barrier once all its warps are done.
        __syncthreads();
        cluster.sync();
        // ---- H pass ----
        for (int u = warp; u < units; u += kCl2dWarps) {
            const int x = (u % XU) * 32 + lane, ylo = (u / XU) * RPG, yhi = min(ylo + RPG, rows);
            const bool in = x < nx;
            const int rxH = in ? xs_h[x] : -1;
            // A plain segment: every lane has its +x neighbour and no x memory, on a uniform mesh.
            const bool xplain = __all_sync(0xffffffffu, x < nx - 1 && rxH < 0) && !mx_h && !my_h;
            T bx = T(0), cx = T(0), kx = T(1), mxv = T(1);
            if (rxH >= 0) { bx = xb_h[x]; cx = xb_h[nx + x]; kx = xb_h[2 * nx + x]; }
            if (mx_h && in) mxv = xb_h[3 * nx + x];
            T ez_cur = (in && ylo < rows) ? Ez[ylo * W + x] : T(0);
            for (int yl = ylo; yl < yhi; ++yl) {
                const int h = r0 + yl, e = yl * W + x;
                // Ez of the row above: this band's row, the band above (DSMEM); none above the last grid row.
                T ez_up = T(0);
                if (in && yl + 1 < rows) ez_up = Ez[e + W];
                else if (in && ez_above != nullptr) ez_up = ez_above[x];
                T ez_right = __shfl_down_sync(0xffffffffu, ez_cur, 1);
                if (lane == 31 && x + 1 < nx) ez_right = Ez[e + 1];
                if (xplain && h < ny - 1 && ys_h[h] < 0) {
                    const T hxn = Hx[e] - cn * (T(0) + (ez_up - ez_cur));
                    Hy[e] = Hy[e] - cn * (T(0) + (-(ez_right - ez_cur)));
                    Hx[e] = hxn;
                } else if (in) {
                    // Hx: dy(Ez)
                    T d = T(0);
                    if (h < ny - 1) {
                        d = ez_up - ez_cur;
                        if (my_h) d = d * yb_h[3 * ny + h];
                        const int ryh = ys_h[h];
                        if (ryh >= 0) {
                            const int pi = (ryh - c.ryh_lo[rank]) * W + x;
                            const T mem = phy[pi] * yb_h[h] + yb_h[ny + h] * d;
                            phy[pi] = mem;
                            d = d * yb_h[2 * ny + h] + mem;
                        }
                    } else if (pec_y) {
                        d = pneg_y * ez_cur;
                    }
                    T acc = T(0) + d;
                    const T hxn = Hx[e] - cn * acc;
                    // Hy: -dx(Ez)
                    d = T(0);
                    if (x < nx - 1) {
                        d = ez_right - ez_cur;
                        if (mx_h) d = d * mxv;
                        if (rxH >= 0) {
                            const T mem = phx[yl * RxH + rxH] * bx + cx * d;
                            phx[yl * RxH + rxH] = mem;
                            d = d * kx + mem;
                        }
                    } else if (pec_x) {
                        d = pneg_x * ez_cur;
                    }
                    acc = T(0) + (-d);
                    Hx[e] = hxn;
                    Hy[e] = Hy[e] - cn * acc;
                }
                ez_cur = ez_up;
            }
        }
        if (src_hx) add_sources(src_hx, Hx, n);
        if (src_hy) add_sources(src_hy, Hy, n);
        if (band_traces) {
            // Point traces of step n sampled by the rank that owns the cell (a CTA-uniform branch).
            __syncthreads();
            if (tid < n_traces && tr_e >= 0) {
                const T v = tr_f == 1 ? Ez[tr_e] : tr_f == 2 ? Hx[tr_e] : tr_f == 3 ? Hy[tr_e] : T(0);
                trace_out[n * n_traces + tid] = v;
            }
            for (int t = tid + kCl2dThreads; t < n_traces; t += kCl2dThreads) {
                const TraceDev tr = traces[t];
                const int y = (int)(tr.offset / pitch), x = (int)(tr.offset % pitch);
                if (y < r0 || y >= r1) continue;
                const int e = (y - r0) * W + x;
                T v = T(0);
                if (tr.family == 0 && tr.comp == 2) v = Ez[e];
                else if (tr.family == 1 && tr.comp == 0) v = Hx[e];
                else if (tr.family == 1 && tr.comp == 1) v = Hy[e];
                trace_out[n * n_traces + t] = v;
            }
        }
        __syncthreads();
        cluster.sync();
    }
    // Write the band back at the parity of the step count reached, and the counter.
    const int par = (int)(n & 1);
    for (int q = tid; q < rows * W; q += kCl2dThreads) {
        const int y = r0 + q / W, x = q % W;
        const long long i = (long long)y * pitch + x;
        g.E[par][2][i] = Ez[q];
        g.H[par][0][i] = Hx[q];
        g.H[par][1][i] = Hy[q];
    }
    if (RxE) for (int q = tid; q < rows * RxE; q += kCl2dThreads) g.psiE[par][0][1][(long long)(r0 + q / RxE) * RxE + q % RxE] = pex[q];
    if (RxH) for (int q = tid; q < rows * RxH; q += kCl2dThreads) g.psiH[0][0][(long long)(r0 + q / RxH) * RxH + q % RxH] = phx[q];
    for (int q = tid; q < c.rye_n[rank] * W; q += kCl2dThreads) g.psiE[par][1][1][(long long)(c.rye_lo[rank] + q / W) * pitch + q % W] = pey[q];
    for (int q = tid; q < c.ryh_n[rank] * W; q += kCl2dThreads) g.psiH[1][0][(long long)(c.ryh_lo[rank] + q / W) * pitch + q % W] = phy[q];
    if (rank == 0 && tid == 0) *g.counter = n;
    cluster.sync();                                       // no rank leaves while a neighbour may still read it
}

}  // namespace tfd
