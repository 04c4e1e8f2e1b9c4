// Fused E+H step, 2.5D marching form with TMA-staged planes (sm_100a).
//
// A CTA owns a 31 x 15 tile of (x, y) and a chunk [z0, z1) of planes, and computes E
// on the 32 x 16 tile that adds the +x column and +y row its H update borrows: lane 31
// of every warp row is the x halo and row 15 the y halo, so all warps carry the same
// work. It marches along z: for each plane k the old H(k), E(k) and inverse
// permittivity of the tile plus a one-cell halo arrive in shared memory through
// cp.async.bulk.tensor (TMA, no multicast) into an S-stage ring guarded by mbarriers,
// issued S-1 planes ahead by one elected thread. Then:
//   1. E_new(k) on the 32 x 16 tile from shared memory: H(k), H(k) at x-1 / y-1 and
//      H(k-1) of the previous stage. Owned cells are stored to global memory with their
//      E-family CPML memory; all values go to a shared E buffer double-buffered over k.
//   2. H_new(k-1) on the owned tile from E_new(k-1) (with its halo) and E_new(k).
// The last plane of a chunk recomputes E_new(z1) of the next chunk as a halo plane, so
// chunks are independent. E and H are double-buffered in HBM (ping-pong over steps),
// so a halo value is recomputed from the same old inputs with the same arithmetic as
// by its owner: bitwise identical, no inter-CTA synchronisation. The arithmetic is the
// reference operation order (see step_gather.cuh). Global traffic per cell: one read
// and one write of each field component, one read of the permittivity, and the CPML
// memories of slab cells only; halos are re-read from L2.
//
// CPML slab rows come from the (lo, hi) slab bounds in registers (no table lookups
// outside slabs); coefficients are read only on slab cells. Index arithmetic is 32-bit
// (the plan refuses grids whose component arrays exceed 2^31 elements).
//
// Supported here: x/y faces PML or PEC (periodic x/y run the gather kernel), z faces
// PML, PEC or periodic, 3D grids. Every mbarrier wait is bounded: on timeout the
// kernel records kStatusPipelineTimeout in the device status word and returns.
#pragma once
#include <cuda.h>

#include "internal.cuh"

namespace tfd {

constexpr int kMarchLanes = 32;     // computed columns: 31 owned + the +x halo
constexpr int kMarchOwnX = 31;
constexpr int kMarchRows = 16;      // computed E rows: 15 owned + the +y halo
constexpr int kMarchOwnY = 15;
constexpr int kMarchThreads = 256;
constexpr int kMarchStages = 4;
constexpr long long kWaitLimit = 1LL << 24;

template <typename T>
struct MarchArgs {
    CUtensorMap field[6];        // Ex Ey Ez Hx Hy Hz: dims (nx, ny, nz, parity), box (BXW, BY, 1, 1)
    CUtensorMap eps[3];          // inverse permittivity per stored sample: dims (nx, ny, nz), box (BXW, BY, 1)
    Grid<T> g;
    int lz;                      // planes per chunk
    int slab[2][3][4];           // per family and axis: lo0, hi0, lo1, hi1 of the two CPML slabs
};

template <typename T, int SAMPLES>
struct MarchShape {
    static constexpr int A = 16 / sizeof(T);                 // TMA x alignment in elements
    static constexpr int BXW = kMarchLanes + A;              // box columns from floor_A(x0-1)
    static constexpr int BY = kMarchRows + 1;                // box rows y0-1 .. y0+15
    static constexpr int BOX = BXW * BY;
    static constexpr int BOX_BYTES = BOX * sizeof(T);
    static constexpr int BOX_STRIDE = (BOX_BYTES + 127) / 128 * 128;
    static constexpr int ARRAYS = 6 + SAMPLES;
    static constexpr int STAGE_BYTES = ARRAYS * BOX_STRIDE;
    static constexpr int EBUF = kMarchLanes * kMarchRows;    // one component of the E buffer
    static constexpr size_t SMEM = (size_t)kMarchStages * STAGE_BYTES + 2 * 3 * EBUF * sizeof(T) + kMarchStages * 8 + 128;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait on phase `parity`; false when the limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (long long it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z, int w) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Slab row of coordinate c, or -1: rows of the low slab first, then of the high slab.
__device__ __forceinline__ int slab_row(const int *s, int c) {
    return (c >= s[0] && c < s[1]) ? c - s[0] : (c >= s[2] && c < s[3]) ? (s[1] - s[0]) + (c - s[2]) : -1;
}

// Index of a CPML memory element (32-bit; the plan bounds every array below 2^31 elements).
__device__ __forceinline__ int psi_index32(int a, int x, int y, int z, int r, int R, int ny, int pitch) {
    return a == 0 ? (z * ny + y) * R + r : a == 1 ? (z * R + r) * pitch + x : (r * ny + y) * pitch + x;
}

template <typename T>
__device__ __forceinline__ T cpml_e32(const Grid<T> &g, int par, int a, int j, int coord, int r, int x, int y, int z, bool own, T d) {
    const int p = psi_index32(a, x, y, z, r, g.rows[0][a], g.n[1], g.pitch);
    const T mem = g.psiE[par][a][j][p] * __ldg(&g.cb[0][a][coord]) + __ldg(&g.cc[0][a][coord]) * d;
    if (own) g.psiE[par ^ 1][a][j][p] = mem;
    return d * __ldg(&g.ck[0][a][coord]) + mem;
}

template <typename T>
__device__ __forceinline__ T cpml_h32(const Grid<T> &g, int a, int j, int coord, int r, int x, int y, int z, T d) {
    const int p = psi_index32(a, x, y, z, r, g.rows[1][a], g.n[1], g.pitch);
    T *psi = g.psiH[a][j];
    const T mem = psi[p] * __ldg(&g.cb[1][a][coord]) + __ldg(&g.cc[1][a][coord]) * d;
    psi[p] = mem;
    return d * __ldg(&g.ck[1][a][coord]) + mem;
}

// Source injection restricted to the terms that touch this tile and plane (bit s of mask).
template <typename T>
__device__ __noinline__ T inject_masked(const Grid<T> &g, unsigned mask, int family, int comp, long long n, int x, int y, int z, T v) {
    while (mask) {
        const int s = __ffs(mask) - 1;
        mask &= mask - 1;
        const SourceTerm &t = g.src[s];
        if (t.family == family && t.comp == comp && x >= t.lo[0] && x < t.hi[0] && y >= t.lo[1] && y < t.hi[1] && z >= t.lo[2] &&
            z < t.hi[2])
            v = v + g.src_values[(long long)s * g.steps + n];
    }
    return v;
}

template <typename T>
__device__ __forceinline__ unsigned source_mask(const Grid<T> &g, int family, int xlo, int xhi, int ylo, int yhi, int z, long long n) {
    unsigned m = 0;
    if (n >= g.steps) return 0;
    for (int s = 0; s < g.n_src; ++s) {
        const SourceTerm &t = g.src[s];
        if (t.family == family && z >= t.lo[2] && z < t.hi[2] && t.lo[0] < xhi && xlo < t.hi[0] && t.lo[1] < yhi && ylo < t.hi[1])
            m |= 1u << s;
    }
    return m;
}

// Per-cell slab rows (E family): x from the lane, y from the warp row, z from the plane.
struct Rows { int x, y, z; };

// E_new of component C at stage index s. hk: plane k stage base, hm: plane k-1 stage base.
template <typename T, int SAMPLES, int C>
__device__ __forceinline__ T march_e(const Grid<T> &g, int par, const T *hk, const T *hm, int s, int x, int y, int z, bool zprev,
                                     bool own, Rows rw) {
    using S = MarchShape<T, SAMPLES>;
    constexpr int ES = S::BOX_STRIDE / sizeof(T);          // element stride between stage arrays
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const Term t = term_of(C, k);
        const T *h = hk + (3 + t.in) * ES;
        T d;
        if (t.axis == 0) {
            const T diff = h[s] - h[s - 1];
            d = x > 0 ? diff : T(0);
            if (rw.x >= 0) d = cpml_e32(g, par, 0, t.j, x, rw.x, x, y, z, own, d);
        } else if (t.axis == 1) {
            const T diff = h[s] - h[s - S::BXW];
            d = y > 0 ? diff : T(0);
            if (rw.y >= 0) d = cpml_e32(g, par, 1, t.j, y, rw.y, x, y, z, own, d);
        } else {
            d = T(0);
            if (zprev) {
                d = h[s] - hm[(3 + t.in) * ES + s];
                if (rw.z >= 0) d = cpml_e32(g, par, 2, t.j, z, rw.z, x, y, z, own, d);
            }
        }
        acc = acc + (t.sign > 0 ? d : -d);
    }
    return hk[C * ES + s] + (g.cn * hk[(6 + (SAMPLES == 3 ? C : 0)) * ES + s]) * acc;
}

template <typename T, int SAMPLES>
__global__ void __launch_bounds__(kMarchThreads, 2) k_step_march(const __grid_constant__ MarchArgs<T> args) {
    using S = MarchShape<T, SAMPLES>;
    constexpr int ES = S::BOX_STRIDE / sizeof(T);
    const Grid<T> &g = args.g;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    T *ebuf = (T *)(smem + (size_t)kMarchStages * S::STAGE_BYTES);
    uint64_t *bars = (uint64_t *)(ebuf + 2 * 3 * S::EBUF);

    const long long n = *g.counter;
    const int par = (int)(n & 1);
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int x0 = blockIdx.x * kMarchOwnX, y0 = blockIdx.y * kMarchOwnY;
    const int z0 = blockIdx.z * args.lz;
    if (z0 >= nz) return;
    const int z1 = min(z0 + args.lz, nz);
    const bool zper = g.periodic[2] != 0;
    const bool has_prev = z0 > 0 || zper;                    // plane z0-1 exists (wrapped when periodic)
    const bool has_halo = z1 < nz || zper;                   // plane z1 exists (wrapped when periodic)
    const int planes = (z1 - z0) + 1 + (has_halo ? 1 : 0);  // ring sequence q holds plane z0-1+q
    const int bx = (x0 - 1) & ~(S::A - 1);                   // TMA box origin: x0-1 rounded down to 16 bytes
    const int off = x0 - bx;                                 // smem column of x0
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    auto issue = [&](int q) {
        uint64_t *bar = &bars[q % kMarchStages];
        T *dst = (T *)(smem + (size_t)(q % kMarchStages) * S::STAGE_BYTES);
        int z = z0 - 1 + q;
        const bool exists = (q == 0) ? has_prev : (z < nz || zper);
        if (z < 0) z += nz;
        if (z >= nz) z -= nz;
        if (!exists) {
            mbar_expect_tx(bar, 0);
            return;
        }
        mbar_expect_tx(bar, (uint32_t)(S::ARRAYS * S::BOX_BYTES));
#pragma unroll
        for (int c = 0; c < 6; ++c) tma_load_4d(dst + c * ES, &args.field[c], bar, bx, y0 - 1, z, par);
#pragma unroll
        for (int c = 0; c < SAMPLES; ++c) tma_load_3d(dst + (6 + c) * ES, &args.eps[c], bar, bx, y0 - 1, z);
    };

    if (tid == 0) {
        for (int s = 0; s < kMarchStages; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0)
        for (int q = 0; q < min(kMarchStages, planes); ++q) issue(q);

    auto stage = [&](int q) { return (const T *)(smem + (size_t)(q % kMarchStages) * S::STAGE_BYTES); };
    auto wait_stage = [&](int q) -> bool { return mbar_wait(&bars[q % kMarchStages], (uint32_t)((q / kMarchStages) & 1)); };

    // Per-thread invariants: column, rows of this warp, CPML slab rows, store offsets.
    const int x = x0 + lane;
    const bool lane_own = lane < kMarchOwnX && x < nx;
    const bool lane_in = x < nx;
    const int rxE = slab_row(args.slab[0][0], x), rxH = slab_row(args.slab[1][0], x);
    int yrow[2], ryE[2], ryH[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        yrow[h] = y0 + warp + 8 * h;
        ryE[h] = slab_row(args.slab[0][1], yrow[h]);
        ryH[h] = slab_row(args.slab[1][1], yrow[h]);
    }
    const int smask_all = g.n_src;

    if (!wait_stage(0)) {
        if (tid == 0) atomicExch(g.status, kStatusPipelineTimeout);
        return;
    }
    for (int k = z0; k <= z1; ++k) {
        const int q = k - z0 + 1;
        const bool halo_plane = k == z1;
        const bool compute_e = !halo_plane || has_halo;
        if (compute_e && !wait_stage(q)) {
            if (tid == 0) atomicExch(g.status, kStatusPipelineTimeout);
            return;
        }
        const int kz = k >= nz ? k - nz : k;
        T *ecur = ebuf + (k & 1) * 3 * S::EBUF;
        const T *eprv = ebuf + ((k - 1) & 1) * 3 * S::EBUF;
        if (compute_e) {
            const T *hk = stage(q), *hm = stage(q - 1);
            const bool zprev = kz > 0 || zper;
            const int rzE = slab_row(args.slab[0][2], kz);
            const unsigned smask = smask_all ? source_mask(g, 0, x0, x0 + kMarchLanes, y0, y0 + kMarchRows, kz, n) : 0u;
            T *gE0 = g.E[par ^ 1][0] + (size_t)kz * g.plane, *gE1 = g.E[par ^ 1][1] + (size_t)kz * g.plane,
              *gE2 = g.E[par ^ 1][2] + (size_t)kz * g.plane;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = warp + 8 * h;
                const int y = yrow[h];
                if (!lane_in || y >= ny) continue;
                const bool own = !halo_plane && lane_own && r < kMarchOwnY;
                const int s = (r + 1) * S::BXW + off + lane;
                const Rows rw{rxE, ryE[h], rzE};
                T ex = march_e<T, SAMPLES, 0>(g, par, hk, hm, s, x, y, kz, zprev, own, rw);
                T ey = march_e<T, SAMPLES, 1>(g, par, hk, hm, s, x, y, kz, zprev, own, rw);
                T ez = march_e<T, SAMPLES, 2>(g, par, hk, hm, s, x, y, kz, zprev, own, rw);
                if (smask) {
                    ex = inject_masked(g, smask, 0, 0, n, x, y, kz, ex);
                    ey = inject_masked(g, smask, 0, 1, n, x, y, kz, ey);
                    ez = inject_masked(g, smask, 0, 2, n, x, y, kz, ez);
                }
                const int e = r * kMarchLanes + lane;
                ecur[e] = ex;
                ecur[S::EBUF + e] = ey;
                ecur[2 * S::EBUF + e] = ez;
                if (own) {
                    const int i = y * g.pitch + x;
                    gE0[i] = ex;
                    gE1[i] = ey;
                    gE2[i] = ez;
                }
            }
        }
        __syncthreads();
        if (k > z0) {
            // H_new(k-1) on the owned tile.
            const int km = k - 1;
            const T *hs = stage(q - 1);
            const bool znext = compute_e;
            const int rzH = slab_row(args.slab[1][2], km);
            const unsigned hmask = smask_all ? source_mask(g, 1, x0, x0 + kMarchOwnX, y0, y0 + kMarchOwnY, km, n) : 0u;
            T *gH[3] = {g.H[par ^ 1][0] + (size_t)km * g.plane, g.H[par ^ 1][1] + (size_t)km * g.plane,
                        g.H[par ^ 1][2] + (size_t)km * g.plane};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = warp + 8 * h;
                const int y = yrow[h];
                if (!lane_own || r >= kMarchOwnY || y >= ny) continue;
                const int s = (r + 1) * S::BXW + off + lane;
                const int e = r * kMarchLanes + lane;
                const int i = y * g.pitch + x;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    T acc = T(0);
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const Term t = term_of(c, kk);
                        const T *ep = eprv + t.in * S::EBUF;
                        T d = T(0);
                        if (t.axis == 0) {
                            if (x < nx - 1) {
                                d = ep[e + 1] - ep[e];
                                if (rxH >= 0) d = cpml_h32(g, 0, t.j, x, rxH, x, y, km, d);
                            } else if (g.pec_on[0]) {
                                d = g.pec_neg[0] * ep[e];
                            }
                        } else if (t.axis == 1) {
                            if (y < ny - 1) {
                                d = ep[e + kMarchLanes] - ep[e];
                                if (ryH[h] >= 0) d = cpml_h32(g, 1, t.j, y, ryH[h], x, y, km, d);
                            } else if (g.pec_on[1]) {
                                d = g.pec_neg[1] * ep[e];
                            }
                        } else {
                            if (znext) {
                                d = ecur[t.in * S::EBUF + e] - ep[e];
                                if (rzH >= 0) d = cpml_h32(g, 2, t.j, km, rzH, x, y, km, d);
                            } else if (g.pec_on[2]) {
                                d = g.pec_neg[2] * ep[e];
                            }
                        }
                        acc = acc + (t.sign > 0 ? d : -d);
                    }
                    T hv = hs[(3 + c) * ES + s] - g.cn * acc;
                    if (hmask) hv = inject_masked(g, hmask, 1, c, n, x, y, km, hv);
                    gH[c][i] = hv;
                }
            }
        }
        __syncthreads();
        // Stage q-1 is free: refill it with plane q-1+S.
        if (tid == 0 && q - 1 + kMarchStages < planes) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(q - 1 + kMarchStages);
        }
    }
}

}  // namespace tfd
