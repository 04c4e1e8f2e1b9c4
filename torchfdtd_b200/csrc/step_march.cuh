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
// Supported here: x/y faces PML, PEC or periodic, z faces PML, PEC or periodic, 3D grids.
// Periodic x/y run the MODE 2 instantiation: after a stage lands, tiles at a periodic seam
// overwrite the box cells that fall outside the domain (TMA fills them with zeros) with the
// cells one period away, so the seam columns / rows difference the same two values as the
// reference's periodic branch, and the +x / +y halo lane or row that lies one past the last
// cell recomputes E of the first column / row. Every mbarrier wait is bounded, and the decision
// is taken by the whole CTA (a barrier reduction): on timeout the kernel records
// kStatusPipelineTimeout in the device status word, waits once more (bounded) for the copies it
// issued, and every thread of the CTA returns together. The fields of a timed-out launch are
// undefined; the plan must be reset (tfd_reset) before it steps again.
#pragma once
#include <cuda.h>

#include "internal.cuh"

namespace tfd {

constexpr int kMarchLanes = 32;     // computed columns: 31 owned + the +x halo
constexpr int kMarchOwnX = 31;
constexpr int kMarchRows = 16;      // computed E rows: 15 owned + the +y halo
constexpr int kMarchOwnY = 15;
// Warps per CTA; each thread computes kMarchRows / kMarchWarps rows of the tile per plane.
#ifndef TFD_MARCH_WARPS
#define TFD_MARCH_WARPS 8
#endif
constexpr int kMarchWarps = TFD_MARCH_WARPS;
constexpr int kMarchThreads = 32 * kMarchWarps;
constexpr int kMarchRowsPerThread = kMarchRows / kMarchWarps;
static_assert(kMarchRows % kMarchWarps == 0, "tile rows must split evenly over the warps");

template <typename T>
struct MarchArgs {
    CUtensorMap field[6];        // Ex Ey Ez Hx Hy Hz: dims (nx, ny, nz, parity), box (BXW, BY, 1, 1)
    CUtensorMap eps[3];          // inverse permittivity per stored sample: dims (nx, ny, nz), box (BXW, BY, 1)
    Grid<T> g;
    int slab[2][3][4];           // per family and axis: lo0, hi0, lo1, hi1 of the two CPML slabs
    int psi_parity[3];           // elements between the two parities of an E-family CPML memory, per axis
};

// Shared-memory layout of the marching kernel. D = planes of TMA prefetch; the H ring holds
// D + 2 planes (k-1 and k in use), the E ring (old E and inverse permittivity) D + 1 (k in use).
template <typename T, int SAMPLES, int D>
struct MarchShape {
    static constexpr int A = 16 / sizeof(T);                 // TMA x alignment in elements
    static constexpr int BXW = kMarchLanes + A;              // box columns from floor_A(x0-1)
    static constexpr int BYH = kMarchRows + 1;               // H box rows y0-1 .. y0+15
    static constexpr int BYE = kMarchRows;                   // E / eps box rows y0 .. y0+15
    static constexpr int BOXH_BYTES = BXW * BYH * (int)sizeof(T);
    static constexpr int BOXE_BYTES = BXW * BYE * (int)sizeof(T);
    static constexpr int BOXH_STRIDE = (BOXH_BYTES + 127) / 128 * 128;
    static constexpr int BOXE_STRIDE = (BOXE_BYTES + 127) / 128 * 128;
    static constexpr int NH = D + 2, NE = D + 1;
    static constexpr int EARR = 3 + SAMPLES;
    static constexpr int HSLOT = 3 * BOXH_STRIDE, ESLOT = EARR * BOXE_STRIDE;
    static constexpr int EBUF = kMarchLanes * kMarchRows;    // one component of the E buffer
    static constexpr size_t HRING = (size_t)NH * HSLOT, ERING = (size_t)NE * ESLOT;
    static constexpr size_t SMEM = HRING + ERING + 2 * 3 * EBUF * sizeof(T) + (NH + NE) * 8;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait on phase `parity`; false when the limit is reached. Each try_wait suspends the
// warp in hardware for up to kSuspendNs (it wakes when the phase completes), so waiting warps do
// not take issue slots from the computing ones; the loop bounds the total wait to about 2 s.
constexpr uint32_t kSuspendNs = 1000000;
constexpr int kWaitTries = 2000;
constexpr int kDrainTries = 500;     // the second wait of a timed-out CTA for its copies in flight (about 0.5 s)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int tries = kWaitTries) {
    const uint32_t addr = smem_u32(bar);
    for (int it = 0; it < tries; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(addr), "r"(parity), "r"(kSuspendNs) : "memory");
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

// Slab row of coordinate c, or -1: rows of the low slab [l0, h0) first, then of the high slab [l1, h1).
__device__ __forceinline__ int slab_row(int l0, int h0, int l1, int h1, int c) {
    return (c >= l0 && c < h0) ? c - l0 : (c >= l1 && c < h1) ? (h0 - l0) + (c - l1) : -1;
}
#define TFD_SLAB_ROW(args, f, a, c) \
    slab_row((args).slab[f][a][0], (args).slab[f][a][1], (args).slab[f][a][2], (args).slab[f][a][3], (c))
// Whether [lo, hi) meets a slab of (family, axis).
#define TFD_SLAB_MEETS(args, f, a, lo, hi) \
    (((lo) < (args).slab[f][a][1] && (args).slab[f][a][0] < (hi)) || ((lo) < (args).slab[f][a][3] && (args).slab[f][a][2] < (hi)))

// Index of a CPML memory element (32-bit; the plan bounds every array below 2^31 elements).
__device__ __forceinline__ int psi_index32(int a, int x, int y, int z, int r, int R, int ny, int pitch) {
    return a == 0 ? (z * ny + y) * R + r : a == 1 ? (z * R + r) * pitch + x : (r * ny + y) * pitch + x;
}

// CPML coefficients of one slab row: decay b, coupling c, 1/kappa.
template <typename T>
struct Coef { T b, c, k; };

template <typename T>
__device__ __forceinline__ Coef<T> coef_at(const Grid<T> &g, int f, int a, int coord, int row) {
    Coef<T> q{T(0), T(0), T(1)};
    if (row >= 0) {
        q.b = __ldg(&g.cb[f][a][coord]);
        q.c = __ldg(&g.cc[f][a][coord]);
        q.k = __ldg(&g.ck[f][a][coord]);
    }
    return q;
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

// Per-cell slab rows (E family): x from the lane, y from the warp row, z from the plane, with
// their coefficients; po/pn: old/new parity offsets of the E-family memories of axis 0, 1, 2.
template <typename T>
struct Rows { int x, y, z; int po[3], pn[3]; Coef<T> qx, qy, qz; };

// E_new of component C on the fast path (the row meets no CPML slab, no domain face and no source, and
// plane z has a previous plane): plain differences in the reference order. hk / hm: H stage of plane
// k / k-1 (box row 0 = y0-1, stride HS); ek: E stage of plane k (box row 0 = y0, stride ES); s / se: the
// cell's element index in those boxes.
// METRIC: nonuniform mesh, each difference times the cell's factor of its axis (m[0..2]).
template <typename T, int SAMPLES, int D, int C, bool METRIC = false>
__device__ __forceinline__ T march_e_fast(const Grid<T> &g, const T *hk, const T *hm, const T *ek, int s, int se,
                                         const T *m = nullptr) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int ES = S::BOXE_STRIDE / sizeof(T);
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const Term t = term_of(C, k);
        const T *h = hk + t.in * HS;
        T d = t.axis == 0 ? h[s] - h[s - 1] : t.axis == 1 ? h[s] - h[s - S::BXW] : h[s] - hm[t.in * HS + s];
        if constexpr (METRIC) d = d * m[t.axis];
        acc = acc + (t.sign > 0 ? d : -d);
    }
    return ek[C * ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? C : 0)) * ES + se]) * acc;
}

// E_new of one cell on a z row (general and z-pure bodies): the row meets no x / y slab, x / y face or source.
// The x / y terms are plain differences. The z terms of Ex and Ey: zero on the first plane of a grid without
// a previous plane (zprev false), through the z memories when zm (z in a z slab and zprev; old at po + iz,
// new at pn + iz, stored by the owner). The terms and their order are those of march_e_row on such a row.
template <typename T, int SAMPLES, int D>
__device__ __forceinline__ void march_e_zslab(const Grid<T> &g, const T *hk, const T *hm, const T *ek, int s, int se, bool zprev,
                                              bool zm, int iz, int po, int pn, bool own, const Coef<T> &q, T &ex, T &ey, T &ez) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int ES = S::BOXE_STRIDE / sizeof(T);
    T o0 = T(0), o1 = T(0);
    if (zm) {
        o0 = g.psiE[0][2][0][po + iz];
        o1 = g.psiE[0][2][1][po + iz];
    }
    const T *Hx = hk, *Hy = hk + HS, *Hz = hk + 2 * HS;
    T d, acc, m;
    // Ex: (y, Hz, +), (z, Hy, -, memory j0)
    d = Hz[s] - Hz[s - S::BXW];
    acc = T(0);
    acc = acc + d;
    d = zprev ? Hy[s] - hm[HS + s] : T(0);
    if (zm) {
        m = o0 * q.b + q.c * d;
        if (own) g.psiE[0][2][0][pn + iz] = m;
        d = d * q.k + m;
    }
    acc = acc + (-d);
    ex = ek[se] + (g.cn * ek[3 * ES + se]) * acc;
    // Ey: (x, Hz, -), (z, Hx, +, memory j1)
    d = Hz[s] - Hz[s - 1];
    acc = T(0);
    acc = acc + (-d);
    d = zprev ? Hx[s] - hm[s] : T(0);
    if (zm) {
        m = o1 * q.b + q.c * d;
        if (own) g.psiE[0][2][1][pn + iz] = m;
        d = d * q.k + m;
    }
    acc = acc + d;
    ey = ek[ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? 1 : 0)) * ES + se]) * acc;
    ez = march_e_fast<T, SAMPLES, D, 2>(g, hk, hm, ek, s, se);
}

// H_new of one owned cell on a z row: no x / y slab, x / y face or source. The z terms: the difference to plane
// km + 1 when znext, else the PEC ghost term or 0 (the last plane of a grid without a next plane); through the
// H-family z memories (at iz, updated in place) when zm (km in a z slab and znext). The terms and their order
// are those of march_h_row.
template <typename T, int SAMPLES, int D>
__device__ __forceinline__ void march_h_zslab(const Grid<T> &g, const T *ep, const T *ec, const T *hs, int sh, int e, bool znext,
                                              bool zm, int iz, const Coef<T> &q, T &hx, T &hy, T &hz) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int EB = S::EBUF;
    T o0 = T(0), o1 = T(0);
    if (zm) {
        o0 = g.psiH[2][0][iz];
        o1 = g.psiH[2][1][iz];
    }
    const T *Ex = ep, *Ey = ep + EB, *Ez = ep + 2 * EB;
    auto dz = [&](int c) -> T { return znext ? ec[c * EB + e] - ep[c * EB + e] : (g.pec_on[2] ? g.pec_neg[2] * ep[c * EB + e] : T(0)); };
    T d, acc, m;
    // Hx: (y, Ez, +), (z, Ey, -, memory j0)
    d = Ez[e + kMarchLanes] - Ez[e];
    acc = T(0);
    acc = acc + d;
    d = dz(1);
    if (zm) {
        m = o0 * q.b + q.c * d;
        g.psiH[2][0][iz] = m;
        d = d * q.k + m;
    }
    acc = acc + (-d);
    hx = hs[sh] - g.cn * acc;
    // Hy: (x, Ez, -), (z, Ex, +, memory j1)
    d = Ez[e + 1] - Ez[e];
    acc = T(0);
    acc = acc + (-d);
    d = dz(0);
    if (zm) {
        m = o1 * q.b + q.c * d;
        g.psiH[2][1][iz] = m;
        d = d * q.k + m;
    }
    acc = acc + d;
    hy = hs[HS + sh] - g.cn * acc;
    // Hz: (x, Ey, +), (y, Ex, -)
    d = Ey[e + 1] - Ey[e];
    acc = T(0);
    acc = acc + d;
    d = Ex[e + kMarchLanes] - Ex[e];
    acc = acc + (-d);
    hz = hs[2 * HS + sh] - g.cn * acc;
}

// E_new of the three components of one cell on a row that is not on the fast path (general kernel).
// Faces become selects (x / y / z > 0, or a periodic seam). CPML: the row meets a CPML slab; the old
// memories of the cell's active slabs are loaded first, so their loads are in flight together, then
// the terms run in the reference order (y-term, z-term of Ex; x, z of Ey; x, y of Ez) and the owner
// stores the new memories. rw.x / rw.y / rw.z: slab rows (-1 outside); x, y: the cell's coordinates.
template <typename T, int SAMPLES, int D, bool CPML, bool WRAP, bool METRIC = false>
__device__ __forceinline__ void march_e_row(const Grid<T> &g, const T *hk, const T *hm, const T *ek, int s, int se, int x, int y,
                                            int z, bool zprev, bool own, const Rows<T> &rw, T &ex, T &ey, T &ez,
                                            const T *m = nullptr) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int ES = S::BOXE_STRIDE / sizeof(T);
    const bool xin = x > 0 || (WRAP && g.periodic[0]);
    const bool yin = y > 0 || (WRAP && g.periodic[1]);
    const T *Hx = hk, *Hy = hk + HS, *Hz = hk + 2 * HS;
    bool ax = false, ay = false, az = false;
    int ix = 0, iy = 0, iz = 0;
    T ox0 = T(0), ox1 = T(0), oy0 = T(0), oy1 = T(0), oz0 = T(0), oz1 = T(0);
    if (CPML) {
        const int ny = g.n[1], pitch = g.pitch;
        ax = rw.x >= 0;
        ay = rw.y >= 0;
        az = zprev && rw.z >= 0;
        ix = (z * ny + y) * g.rows[0][0] + rw.x;
        iy = (z * g.rows[0][1] + rw.y) * pitch + x;
        iz = (rw.z * ny + y) * pitch + x;
        if (ax) { ox0 = g.psiE[0][0][0][rw.po[0] + ix]; ox1 = g.psiE[0][0][1][rw.po[0] + ix]; }
        if (ay) { oy0 = g.psiE[0][1][0][rw.po[1] + iy]; oy1 = g.psiE[0][1][1][rw.po[1] + iy]; }
        if (az) { oz0 = g.psiE[0][2][0][rw.po[2] + iz]; oz1 = g.psiE[0][2][1][rw.po[2] + iz]; }
    }
    auto mem = [&](int a, int j, int idx, T old, const Coef<T> &q, T d) -> T {
        const T m = old * q.b + q.c * d;
        if (own) g.psiE[0][a][j][rw.pn[a] + idx] = m;
        return d * q.k + m;
    };
    T d, acc;
    // Ex: (y, Hz, +, j0), (z, Hy, -, j0)
    // Nonuniform mesh: a plain difference (periodic seam included) times the cell's factor of its axis.
    auto scale = [&](bool live, int a, T d) -> T {
        if constexpr (METRIC) return live ? d * m[a] : d;
        return d;
    };
    d = scale(yin, 1, yin ? Hz[s] - Hz[s - S::BXW] : T(0));
    if (CPML && ay) d = mem(1, 0, iy, oy0, rw.qy, d);
    acc = T(0);
    acc = acc + d;
    d = scale(zprev, 2, zprev ? Hy[s] - hm[HS + s] : T(0));
    if (CPML && az) d = mem(2, 0, iz, oz0, rw.qz, d);
    acc = acc + (-d);
    ex = ek[se] + (g.cn * ek[3 * ES + se]) * acc;
    // Ey: (x, Hz, -, j0), (z, Hx, +, j1)
    d = scale(xin, 0, xin ? Hz[s] - Hz[s - 1] : T(0));
    if (CPML && ax) d = mem(0, 0, ix, ox0, rw.qx, d);
    acc = T(0);
    acc = acc + (-d);
    d = scale(zprev, 2, zprev ? Hx[s] - hm[s] : T(0));
    if (CPML && az) d = mem(2, 1, iz, oz1, rw.qz, d);
    acc = acc + d;
    ey = ek[ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? 1 : 0)) * ES + se]) * acc;
    // Ez: (x, Hy, +, j1), (y, Hx, -, j1)
    d = scale(xin, 0, xin ? Hy[s] - Hy[s - 1] : T(0));
    if (CPML && ax) d = mem(0, 1, ix, ox1, rw.qx, d);
    acc = T(0);
    acc = acc + d;
    d = scale(yin, 1, yin ? Hx[s] - Hx[s - S::BXW] : T(0));
    if (CPML && ay) d = mem(1, 1, iy, oy1, rw.qy, d);
    acc = acc + (-d);
    ez = ek[2 * ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? 2 : 0)) * ES + se]) * acc;
}

// H_new of the three components of one owned cell on a row that is not on the fast path. Upper faces
// become selects: the difference to the +x / +y / +z neighbour, else the PEC ghost term, else 0.
// CPML: as for E, with the H-family memories updated in place. ep: E_new of plane km (the cell's
// plane, with the +x column and +y row), ec: E_new of plane km + 1; e: the cell's index in both.
template <typename T, int SAMPLES, int D, bool CPML, bool METRIC = false>
__device__ __forceinline__ void march_h_row(const Grid<T> &g, const T *ep, const T *ec, const T *hs, int sh, int e, int x, int y,
                                            int km, bool xn, bool yn, bool znext, int rx, int ry, int rz, const Coef<T> &qx,
                                            const Coef<T> &qy, const Coef<T> &qz, T &hx, T &hy, T &hz, const T *m = nullptr) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int EB = S::EBUF;
    bool ax = false, ay = false, az = false;
    int ix = 0, iy = 0, iz = 0;
    T ox0 = T(0), ox1 = T(0), oy0 = T(0), oy1 = T(0), oz0 = T(0), oz1 = T(0);
    if (CPML) {
        const int ny = g.n[1], pitch = g.pitch;
        ax = xn && rx >= 0;
        ay = yn && ry >= 0;
        az = znext && rz >= 0;
        ix = (km * ny + y) * g.rows[1][0] + rx;
        iy = (km * g.rows[1][1] + ry) * pitch + x;
        iz = (rz * ny + y) * pitch + x;
        if (ax) { ox0 = g.psiH[0][0][ix]; ox1 = g.psiH[0][1][ix]; }
        if (ay) { oy0 = g.psiH[1][0][iy]; oy1 = g.psiH[1][1][iy]; }
        if (az) { oz0 = g.psiH[2][0][iz]; oz1 = g.psiH[2][1][iz]; }
    }
    auto mem = [&](int a, int j, int idx, T old, const Coef<T> &q, T d) -> T {
        const T m = old * q.b + q.c * d;
        g.psiH[a][j][idx] = m;
        return d * q.k + m;
    };
    // A neighbour difference (periodic seam included) times the cell's factor of its axis on a nonuniform mesh;
    // the PEC ghost term is not scaled.
    auto nb = [&](int a, T d) -> T {
        if constexpr (METRIC) return d * m[a];
        return d;
    };
    auto dx = [&](const T *f) -> T { return xn ? nb(0, f[e + 1] - f[e]) : (g.pec_on[0] ? g.pec_neg[0] * f[e] : T(0)); };
    auto dy = [&](const T *f) -> T { return yn ? nb(1, f[e + kMarchLanes] - f[e]) : (g.pec_on[1] ? g.pec_neg[1] * f[e] : T(0)); };
    auto dz = [&](int c) -> T {
        return znext ? nb(2, ec[c * EB + e] - ep[c * EB + e]) : (g.pec_on[2] ? g.pec_neg[2] * ep[c * EB + e] : T(0));
    };
    const T *Ex = ep, *Ey = ep + EB, *Ez = ep + 2 * EB;
    T d, acc;
    // Hx: (y, Ez, +, j0), (z, Ey, -, j0)
    d = dy(Ez);
    if (CPML && ay) d = mem(1, 0, iy, oy0, qy, d);
    acc = T(0);
    acc = acc + d;
    d = dz(1);
    if (CPML && az) d = mem(2, 0, iz, oz0, qz, d);
    acc = acc + (-d);
    hx = hs[sh] - g.cn * acc;
    // Hy: (x, Ez, -, j0), (z, Ex, +, j1)
    d = dx(Ez);
    if (CPML && ax) d = mem(0, 0, ix, ox0, qx, d);
    acc = T(0);
    acc = acc + (-d);
    d = dz(0);
    if (CPML && az) d = mem(2, 1, iz, oz1, qz, d);
    acc = acc + d;
    hy = hs[HS + sh] - g.cn * acc;
    // Hz: (x, Ey, +, j1), (y, Ex, -, j1)
    d = dx(Ey);
    if (CPML && ax) d = mem(0, 1, ix, ox1, qx, d);
    acc = T(0);
    acc = acc + d;
    d = dy(Ex);
    if (CPML && ay) d = mem(1, 1, iy, oy1, qy, d);
    acc = acc + (-d);
    hz = hs[2 * HS + sh] - g.cn * acc;
}

// The x tier of the x-boundary body (MODE 5): a row of a tile that meets an x slab or an x face but no y / z
// slab or face. Only the x differences carry CPML memories (per lane: rx >= 0) and the x faces are selects;
// the y and z differences are plain. The operations are those of march_e_row / march_h_row with the y and z
// terms plain, in the same order. rx, q: this lane's x slab row and coefficients (fixed over the tile);
// ix: the memory element of the lane's cell; po / pn: old / new parity offsets of the E-family x memories.
template <typename T, int SAMPLES, int D>
__device__ __forceinline__ void march_e_xtier(const Grid<T> &g, const T *hk, const T *hm, const T *ek, int s, int se, bool xin, int rx,
                                              int ix, int po, int pn, bool own, const Coef<T> &q, T &ex, T &ey, T &ez) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int ES = S::BOXE_STRIDE / sizeof(T);
    const T *Hx = hk, *Hy = hk + HS, *Hz = hk + 2 * HS;
    const bool ax = rx >= 0;
    T o0 = T(0), o1 = T(0);
    if (ax) {
        o0 = g.psiE[0][0][0][po + ix];
        o1 = g.psiE[0][0][1][po + ix];
    }
    T d, acc, m;
    // Ex: (y, Hz, +), (z, Hy, -)
    d = Hz[s] - Hz[s - S::BXW];
    acc = T(0);
    acc = acc + d;
    d = Hy[s] - hm[HS + s];
    acc = acc + (-d);
    ex = ek[se] + (g.cn * ek[3 * ES + se]) * acc;
    // Ey: (x, Hz, -, j0), (z, Hx, +)
    d = xin ? Hz[s] - Hz[s - 1] : T(0);
    if (ax) {
        m = o0 * q.b + q.c * d;
        if (own) g.psiE[0][0][0][pn + ix] = m;
        d = d * q.k + m;
    }
    acc = T(0);
    acc = acc + (-d);
    d = Hx[s] - hm[s];
    acc = acc + d;
    ey = ek[ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? 1 : 0)) * ES + se]) * acc;
    // Ez: (x, Hy, +, j1), (y, Hx, -)
    d = xin ? Hy[s] - Hy[s - 1] : T(0);
    if (ax) {
        m = o1 * q.b + q.c * d;
        if (own) g.psiE[0][0][1][pn + ix] = m;
        d = d * q.k + m;
    }
    acc = T(0);
    acc = acc + d;
    d = Hx[s] - Hx[s - S::BXW];
    acc = acc + (-d);
    ez = ek[2 * ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? 2 : 0)) * ES + se]) * acc;
}

// ep / ec: E_new of the cell's plane and of the plane above; xn: the +x neighbour exists (else the PEC ghost
// term or 0); the H-family x memories are updated in place.
template <typename T, int SAMPLES, int D>
__device__ __forceinline__ void march_h_xtier(const Grid<T> &g, const T *ep, const T *ec, const T *hs, int sh, int e, bool xn, int rx,
                                              int ix, const Coef<T> &q, T &hx, T &hy, T &hz) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int EB = S::EBUF;
    const bool ax = xn && rx >= 0;
    T o0 = T(0), o1 = T(0);
    if (ax) {
        o0 = g.psiH[0][0][ix];
        o1 = g.psiH[0][1][ix];
    }
    const T *Ex = ep, *Ey = ep + EB, *Ez = ep + 2 * EB;
    auto dx = [&](const T *f) -> T { return xn ? f[e + 1] - f[e] : (g.pec_on[0] ? g.pec_neg[0] * f[e] : T(0)); };
    T d, acc, m;
    // Hx: (y, Ez, +), (z, Ey, -)
    d = Ez[e + kMarchLanes] - Ez[e];
    acc = T(0);
    acc = acc + d;
    d = ec[EB + e] - ep[EB + e];
    acc = acc + (-d);
    hx = hs[sh] - g.cn * acc;
    // Hy: (x, Ez, -, j0), (z, Ex, +)
    d = dx(Ez);
    if (ax) {
        m = o0 * q.b + q.c * d;
        g.psiH[0][0][ix] = m;
        d = d * q.k + m;
    }
    acc = T(0);
    acc = acc + (-d);
    d = ec[e] - ep[e];
    acc = acc + d;
    hy = hs[HS + sh] - g.cn * acc;
    // Hz: (x, Ey, +, j1), (y, Ex, -)
    d = dx(Ey);
    if (ax) {
        m = o1 * q.b + q.c * d;
        g.psiH[0][1][ix] = m;
        d = d * q.k + m;
    }
    acc = T(0);
    acc = acc + d;
    d = Ex[e + kMarchLanes] - Ex[e];
    acc = acc + (-d);
    hz = hs[2 * HS + sh] - g.cn * acc;
}

// The y tier of the y-boundary body (MODE 6): a row of a tile inside the interior x range that meets a y slab
// or a y face but no z slab or face. Only the y differences carry CPML memories (ry >= 0, the row's slab row)
// and the y faces are selects; the x and z differences are plain. Same operations and order as march_e_row /
// march_h_row with the x and z terms plain. iy: the memory element of the cell.
template <typename T, int SAMPLES, int D>
__device__ __forceinline__ void march_e_ytier(const Grid<T> &g, const T *hk, const T *hm, const T *ek, int s, int se, bool yin, int ry,
                                              int iy, int po, int pn, bool own, const Coef<T> &q, T &ex, T &ey, T &ez) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int ES = S::BOXE_STRIDE / sizeof(T);
    const T *Hx = hk, *Hy = hk + HS, *Hz = hk + 2 * HS;
    const bool ay = ry >= 0;
    T o0 = T(0), o1 = T(0);
    if (ay) {
        o0 = g.psiE[0][1][0][po + iy];
        o1 = g.psiE[0][1][1][po + iy];
    }
    T d, acc, m;
    // Ex: (y, Hz, +, j0), (z, Hy, -)
    d = yin ? Hz[s] - Hz[s - S::BXW] : T(0);
    if (ay) {
        m = o0 * q.b + q.c * d;
        if (own) g.psiE[0][1][0][pn + iy] = m;
        d = d * q.k + m;
    }
    acc = T(0);
    acc = acc + d;
    d = Hy[s] - hm[HS + s];
    acc = acc + (-d);
    ex = ek[se] + (g.cn * ek[3 * ES + se]) * acc;
    // Ey: (x, Hz, -), (z, Hx, +)
    d = Hz[s] - Hz[s - 1];
    acc = T(0);
    acc = acc + (-d);
    d = Hx[s] - hm[s];
    acc = acc + d;
    ey = ek[ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? 1 : 0)) * ES + se]) * acc;
    // Ez: (x, Hy, +), (y, Hx, -, j1)
    d = Hy[s] - Hy[s - 1];
    acc = T(0);
    acc = acc + d;
    d = yin ? Hx[s] - Hx[s - S::BXW] : T(0);
    if (ay) {
        m = o1 * q.b + q.c * d;
        if (own) g.psiE[0][1][1][pn + iy] = m;
        d = d * q.k + m;
    }
    acc = acc + (-d);
    ez = ek[2 * ES + se] + (g.cn * ek[(3 + (SAMPLES == 3 ? 2 : 0)) * ES + se]) * acc;
}

template <typename T, int SAMPLES, int D>
__device__ __forceinline__ void march_h_ytier(const Grid<T> &g, const T *ep, const T *ec, const T *hs, int sh, int e, bool yn, int ry,
                                              int iy, const Coef<T> &q, T &hx, T &hy, T &hz) {
    using S = MarchShape<T, SAMPLES, D>;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int EB = S::EBUF;
    const bool ay = yn && ry >= 0;
    T o0 = T(0), o1 = T(0);
    if (ay) {
        o0 = g.psiH[1][0][iy];
        o1 = g.psiH[1][1][iy];
    }
    const T *Ex = ep, *Ey = ep + EB, *Ez = ep + 2 * EB;
    auto dy = [&](const T *f) -> T { return yn ? f[e + kMarchLanes] - f[e] : (g.pec_on[1] ? g.pec_neg[1] * f[e] : T(0)); };
    T d, acc, m;
    // Hx: (y, Ez, +, j0), (z, Ey, -)
    d = dy(Ez);
    if (ay) {
        m = o0 * q.b + q.c * d;
        g.psiH[1][0][iy] = m;
        d = d * q.k + m;
    }
    acc = T(0);
    acc = acc + d;
    d = ec[EB + e] - ep[EB + e];
    acc = acc + (-d);
    hx = hs[sh] - g.cn * acc;
    // Hy: (x, Ez, -), (z, Ex, +)
    d = Ez[e + 1] - Ez[e];
    acc = T(0);
    acc = acc + (-d);
    d = ec[e] - ep[e];
    acc = acc + d;
    hy = hs[HS + sh] - g.cn * acc;
    // Hz: (x, Ey, +), (y, Ex, -, j1)
    d = Ey[e + 1] - Ey[e];
    acc = T(0);
    acc = acc + d;
    d = dy(Ex);
    if (ay) {
        m = o1 * q.b + q.c * d;
        g.psiH[1][1][iy] = m;
        d = d * q.k + m;
    }
    acc = acc + (-d);
    hz = hs[2 * HS + sh] - g.cn * acc;
}

// D planes of TMA prefetch; MINB CTAs per SM requested from the register allocator.
// MODE 0 (general) runs any tile. MODE 1 (pure) has only the fast path (plus source injection): the host
// launches it over tiles whose computed 32 x 16 cells lie inside the domain and outside every x/y CPML
// slab, and over planes whose chunks (with their halo plane) meet no z slab of either family, and the
// general kernel over the rest; compiled without the face and CPML code, the fast path gets the whole
// 64-register budget. MODE 2 is MODE 0 with periodic x / y seams (the host launches it when the grid has
// them). MODE 4 (z-pure) takes the same interior tiles on the other planes (k_step_march_mixed only): fast
// rows, and z rows in march_e_zslab / march_h_zslab. Tile (tx, ty) of a launch is (blockIdx.x + tx_off, blockIdx.y + ty_off); chunk blockIdx.z
// covers planes [z_lo + blockIdx.z * lz, min(that + lz, z_hi)).
// The body of one CTA: tile (tx, ty), planes [z0, z1).
// METRIC (general bodies only): a nonuniform mesh; every plain difference is scaled by the updated cell's factor
// of its axis (1 on a uniform axis), the z tier is off and z-slab rows take the general CPML rows.
template <typename T, int SAMPLES, int D, int MODE, bool METRIC = false>
__device__ __forceinline__ void march_body(const MarchArgs<T> &args, int tx, int ty, int z0, int z1) {
    using S = MarchShape<T, SAMPLES, D>;
    // MODE 4 (z-pure) runs interior tiles (as MODE 1) on any planes: fast rows, and z rows (a z slab, or the
    // first / last plane of a grid with z faces) in march_e_zslab / march_h_zslab.
    constexpr bool ZPURE = MODE == 4;
    // MODE 5 (x-boundary) runs tiles outside the interior block's x range whose rows meet no y slab or face, on
    // planes clear of the z slabs and faces (k_step_march_mixed only): every row takes the x tier.
    constexpr bool XPURE = MODE == 5;
    // MODE 6 (y-boundary) runs tiles of the interior x range outside its y range on the same planes: fast rows,
    // and rows with a y slab, a y face or a source in the y tier.
    constexpr bool YPURE = MODE == 6;
    constexpr bool INTERIOR = MODE == 1 || ZPURE;
    constexpr bool PXY = MODE == 2;
    // Rows that meet only a z slab get their own tier (plain x / y differences, z memories) in the periodic
    // x / y body, where such rows are most of the general work (CPML on z only): 0.575 against 0.612 ms per
    // step at 512 x 512 x 128. With x / y slabs the general work is mostly x / y slab rows, and the extra tier
    // cost the 512 x 512 x 256 CPML step 1.3 % (instruction cache); there the z-pure body takes them.
    constexpr bool ZTIER = (MODE == 2 || ZPURE) && !METRIC;
    static_assert(!METRIC || MODE == 0 || MODE == 1 || MODE == 2, "the metric variants are the general and pure bodies");
    static_assert(!(XPURE || YPURE) || !METRIC, "the x- and y-boundary bodies assume a uniform mesh");
    // The general and z-pure bodies keep their row loops rolled: unrolled, the general body's three row tiers
    // exist once per row and the code outgrows the instruction cache once a pure body shares the SM
    // (measured: 75 % vs 94 % hits).
    constexpr int kRowUnroll = (MODE == 1 || XPURE) ? kMarchRowsPerThread : 1;
    constexpr int HS = S::BOXH_STRIDE / sizeof(T);
    constexpr int ES = S::BOXE_STRIDE / sizeof(T);
    const Grid<T> &g = args.g;
    // Dynamic shared memory (16-byte aligned, enough for non-swizzled TMA boxes whose strides are
    // multiples of 128 bytes), addressed as element offsets from the __shared__ array so every access
    // stays a 32-bit shared-window load.
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T *const sm = reinterpret_cast<T *>(smem_raw);
    constexpr int HSLOT_E = S::HSLOT / sizeof(T), ESLOT_E = S::ESLOT / sizeof(T);
    constexpr int ERING_OFF = S::HRING / sizeof(T);
    constexpr int EBUF_OFF = (S::HRING + S::ERING) / sizeof(T);
    uint64_t *barh = reinterpret_cast<uint64_t *>(smem_raw + S::HRING + S::ERING + 2 * 3 * S::EBUF * sizeof(T));
    uint64_t *bare = barh + S::NH;

    const long long n = *g.counter;
    if (n >= g.steps) return;                   // past the plan's last step: a step is a no-op
    const int par = (int)(n & 1);
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int x0 = tx * kMarchOwnX, y0 = ty * kMarchOwnY;
    if (z0 >= z1) return;
    const bool zper = g.periodic[2] != 0;
    const bool has_prev = z0 > 0 || zper;                    // plane z0-1 exists (wrapped when periodic)
    const bool has_halo = z1 < nz || zper;                   // plane z1 exists (wrapped when periodic)
    const int nh = (z1 - z0) + 1 + (has_halo ? 1 : 0);      // H sequence i holds plane z0-1+i
    const int ne = (z1 - z0) + (has_halo ? 1 : 0);          // E sequence i holds plane z0+i
    const int bx = (x0 - 1) & ~(S::A - 1);                   // TMA box origin: x0-1 rounded down to 16 bytes
    const int off = x0 - bx;                                 // smem column of x0
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    auto wrap = [&](int z) { return z < 0 ? z + nz : (z >= nz ? z - nz : z); };
    auto issue_h = [&](int i) {
        uint64_t *bar = &barh[i % S::NH];
        T *dst = sm + (i % S::NH) * HSLOT_E;
        const int z = z0 - 1 + i;
        if (i == 0 && !has_prev) {
            mbar_expect_tx(bar, 0);
            return;
        }
        mbar_expect_tx(bar, (uint32_t)(3 * S::BOXH_BYTES));
#pragma unroll
        for (int c = 0; c < 3; ++c) tma_load_4d(dst + c * HS, &args.field[3 + c], bar, bx, y0 - 1, wrap(z), par);
    };
    auto issue_e = [&](int i) {
        uint64_t *bar = &bare[i % S::NE];
        T *dst = sm + ERING_OFF + (i % S::NE) * ESLOT_E;
        const int z = wrap(z0 + i);
        mbar_expect_tx(bar, (uint32_t)(S::EARR * S::BOXE_BYTES));
#pragma unroll
        for (int c = 0; c < 3; ++c) tma_load_4d(dst + c * ES, &args.field[c], bar, bx, y0, z, par);
#pragma unroll
        for (int c = 0; c < SAMPLES; ++c) tma_load_3d(dst + (3 + c) * ES, &args.eps[c], bar, bx, y0, z);
    };

    if (tid == 0) {
        for (int s = 0; s < S::NH + S::NE; ++s) mbar_init(&barh[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        for (int i = 0; i < min(S::NH, nh); ++i) issue_h(i);
        for (int i = 0; i < min(S::NE, ne); ++i) issue_e(i);
    }

    auto hstage = [&](int i) -> const T * { return sm + (i % S::NH) * HSLOT_E; };
    auto estage = [&](int i) -> const T * { return sm + ERING_OFF + (i % S::NE) * ESLOT_E; };
    auto wait_h = [&](int i) -> bool { return mbar_wait(&barh[i % S::NH], (uint32_t)((i / S::NH) & 1)); };
    auto wait_e = [&](int i) -> bool { return mbar_wait(&bare[i % S::NE], (uint32_t)((i / S::NE) & 1)); };

    // Per-thread invariants: column, rows of this warp, CPML slab rows and coefficients.
    // px / py: periodic seams (MODE 2 only). xc: the cell this lane computes E of (the lane one past
    // the last column wraps to column 0).
    const bool px = PXY && g.periodic[0] != 0, py = PXY && g.periodic[1] != 0;
    const int x = x0 + lane;
    const int xc = (px && x == nx) ? 0 : x;
    const bool lane_own = lane < kMarchOwnX && x < nx;
    const bool lane_in = x < nx || (px && x == nx);
    // Nonuniform mesh: this lane's x factors (E at column xc, H at column x), 1 on a uniform axis.
    T mxE = T(1), mxH = T(1);
    if constexpr (METRIC) {
        if (g.metric[0][0] != nullptr && lane_in) mxE = g.metric[0][0][xc];
        if (g.metric[1][0] != nullptr && x < nx) mxH = g.metric[1][0][x];
    }
    // Per-thread CPML state (slab rows, coefficients) is built on the rows that meet a slab, where it
    // is used, and not kept across the plane loop: under the 64-register budget of 4 CTAs per SM it
    // would crowd the fast path.
    int yrow[kMarchRowsPerThread];
#pragma unroll
    for (int h = 0; h < kMarchRowsPerThread; ++h) yrow[h] = y0 + warp + kMarchWarps * h;
    auto e_rows = [&](int xx, int yy, int kz, int rz) {
        Rows<T> rw;
        rw.x = TFD_SLAB_ROW(args, 0, 0, xx);
        rw.y = TFD_SLAB_ROW(args, 0, 1, yy);
        rw.z = rz;
        rw.qx = coef_at(g, 0, 0, xx, rw.x);
        rw.qy = coef_at(g, 0, 1, yy, rw.y);
        rw.qz = coef_at(g, 0, 2, kz, rz);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            rw.po[a] = par ? args.psi_parity[a] : 0;
            rw.pn[a] = par ? 0 : args.psi_parity[a];
        }
        return rw;
    };
    // Warp-uniform path of each row: fast (plain differences: no face, CPML slab or source), edge (faces
    // as selects) or CPML (the row meets a slab). Lanes past the last column skip the row, so the last
    // tile column takes the fast E path; its H update has the x = nx-1 face unless x is periodic.
    // The tile and row parts of that choice, packed in one register (R rows per thread): bit h, the E row
    // meets an x or y slab; bit R + h, it has a domain face; bits 2R + h and 3R + h, the same for H.
    constexpr int R = kMarchRowsPerThread;
    unsigned rowbits = 0;
    // x-boundary body: this lane's x slab rows and coefficients, fixed over the tile.
    int rx_e = -1, rx_h = -1;
    Coef<T> qx_e{T(0), T(0), T(1)}, qx_h{T(0), T(0), T(1)};
    if constexpr (XPURE) {
        rx_e = TFD_SLAB_ROW(args, 0, 0, xc);
        qx_e = coef_at(g, 0, 0, xc, rx_e);
        rx_h = TFD_SLAB_ROW(args, 1, 0, x);
        qx_h = coef_at(g, 1, 0, x, rx_h);
    }
    if (!INTERIOR && !XPURE && !YPURE) {
        const bool slab_x_e = TFD_SLAB_MEETS(args, 0, 0, x0, x0 + kMarchLanes);
        const bool slab_x_h = TFD_SLAB_MEETS(args, 1, 0, x0, x0 + kMarchOwnX);
        const bool face_x_e = x0 == 0 && !px;
        const bool face_x_h = x0 + kMarchLanes > nx && !px;
#pragma unroll
        for (int h = 0; h < R; ++h) {
            const int yc = (py && yrow[h] == ny) ? 0 : yrow[h];
            if (slab_x_e || TFD_SLAB_ROW(args, 0, 1, yc) >= 0) rowbits |= 1u << h;
            if (face_x_e || (yrow[h] == 0 && !py)) rowbits |= 1u << (R + h);
            if (slab_x_h || TFD_SLAB_ROW(args, 1, 1, yrow[h]) >= 0) rowbits |= 1u << (2 * R + h);
            if (face_x_h || (yrow[h] >= ny - 1 && !py)) rowbits |= 1u << (3 * R + h);
        }
    }
    // Source terms whose x/y box meets this tile (E: with the halo), tested once per CTA.
    unsigned tile_src_e = 0, tile_src_h = 0;
    // A tile at a periodic seam also computes E of the wrapped first column / row: test every x / y.
    const bool wrap_x = px && x0 + kMarchLanes > nx, wrap_y = py && y0 + kMarchRows > ny;
    for (int t = 0; t < g.n_src; ++t) {
        const SourceTerm &st = g.src[t];
        const bool e_hit = (wrap_x || (st.lo[0] < x0 + kMarchLanes && x0 < st.hi[0])) &&
                           (wrap_y || (st.lo[1] < y0 + kMarchRows && y0 < st.hi[1]));
        const bool h_hit = st.lo[0] < x0 + kMarchOwnX && x0 < st.hi[0] && st.lo[1] < y0 + kMarchOwnY && y0 < st.hi[1];
        if (st.family == 0 && e_hit) tile_src_e |= 1u << t;
        if (st.family == 1 && h_hit) tile_src_h |= 1u << t;
    }
    // New-parity offset of the fields; old/new offsets of the E-family CPML memories.
    const size_t fn = par ? 0 : (size_t)g.count;
    // Periodic seams: box cells outside the domain on a periodic axis take the cell one period away
    // (old fields at parity par, inverse permittivity), written over the TMA zero fill once the
    // stage has landed. Only tiles whose box crosses a seam do this.
    const bool patch = wrap_x || wrap_y || (px && x0 == 0) || (py && y0 == 0);
    // kind 0: H fields, 1: E fields, 2: inverse permittivity.
    auto patch_box = [&](T *dst, int stride, int rows, int ry0, int z, int comps, int kind) {
        const size_t zo = (size_t)z * g.plane;
        for (int q = tid; q < S::BXW * rows; q += kMarchThreads) {
            const int cx = bx + q % S::BXW, cy = ry0 + q / S::BXW;
            const bool ox = cx < 0 || cx >= nx, oy = cy < 0 || cy >= ny;
            if ((!ox && !oy) || (ox && !px) || (oy && !py)) continue;
            const size_t gi = zo + (size_t)(((cy % ny) + ny) % ny) * g.pitch + (((cx % nx) + nx) % nx);
            for (int c = 0; c < comps; ++c) {
                const T *src = kind == 2 ? g.inv_eps[c] : (kind == 0 ? g.H[0][c] : g.E[0][c]) + (size_t)par * g.count;
                dst[c * stride + q] = src[gi];
            }
        }
    };
    auto patch_h = [&](int i) { patch_box(sm + (i % S::NH) * HSLOT_E, HS, S::BYH, y0 - 1, wrap(z0 - 1 + i), 3, 0); };
    auto patch_e = [&](int i) {
        T *dst = sm + ERING_OFF + (i % S::NE) * ESLOT_E;
        patch_box(dst, ES, S::BYE, y0, wrap(z0 + i), 3, 1);
        patch_box(dst + 3 * ES, ES, S::BYE, y0, wrap(z0 + i), SAMPLES, 2);
    };
    const Rows<T> no_rows{};
    // A wait of plane step t ran out: the status is recorded, thread 0 waits once more (bounded) for the copies
    // still in flight, and the caller returns with the whole CTA. Before the waits of step t, thread 0 has issued
    // the H sequence up to min(nh, NH + t) and the E sequence up to min(ne, NE + t); everything older than one
    // ring was waited on.
    auto give_up = [&](int t) {
        if (tid == 0) {
            atomicExch(g.status, kStatusPipelineTimeout);
            const int issued_h = min(nh, S::NH + t), issued_e = min(ne, S::NE + t);
            for (int i = max(0, issued_h - S::NH); i < issued_h; ++i) mbar_wait(&barh[i % S::NH], (uint32_t)((i / S::NH) & 1), kDrainTries);
            for (int i = max(0, issued_e - S::NE); i < issued_e; ++i) mbar_wait(&bare[i % S::NE], (uint32_t)((i / S::NE) & 1), kDrainTries);
        }
    };

    if (__syncthreads_or(!wait_h(0))) {
        give_up(0);
        return;
    }
    for (int k = z0; k <= z1; ++k) {
        const int t = k - z0;                                // E sequence index of plane k; H index is t + 1
        const bool halo_plane = k == z1;
        const bool compute_e = !halo_plane || has_halo;
        // A thread whose wait runs out still computes this plane (in-bounds shared-memory reads of a stage that
        // may not have landed); the barrier after the E phase then takes the CTA-wide decision.
        const bool late = compute_e && !(wait_h(t + 1) && wait_e(t));
        if (PXY && patch && compute_e) {
            if (t == 0 && has_prev) patch_h(0);
            patch_h(t + 1);
            patch_e(t);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
        }
        const int kz = k >= nz ? k - nz : k;
        T *ecur = sm + EBUF_OFF + (k & 1) * 3 * S::EBUF;
        const T *eprv = sm + EBUF_OFF + ((k - 1) & 1) * 3 * S::EBUF;
        if (compute_e) {
            const T *hk = hstage(t + 1), *hm = hstage(t), *ek = estage(t);
            const bool zprev = kz > 0 || zper;
            const int rzE = TFD_SLAB_ROW(args, 0, 2, kz);
            const unsigned smask = tile_src_e ? source_mask(g, 0, wrap_x ? 0 : x0, wrap_x ? nx : x0 + kMarchLanes, wrap_y ? 0 : y0,
                                                            wrap_y ? ny : y0 + kMarchRows, kz, n) & tile_src_e
                                              : 0u;
            T *gE0 = g.E[0][0] + fn + (size_t)kz * g.plane, *gE1 = g.E[0][1] + fn + (size_t)kz * g.plane,
              *gE2 = g.E[0][2] + fn + (size_t)kz * g.plane;
            T mzE = T(1);
            if constexpr (METRIC) {
                if (g.metric[0][2] != nullptr) mzE = g.metric[0][2][kz];
            }
#pragma unroll kRowUnroll
            for (int h = 0; h < kMarchRowsPerThread; ++h) {
                const int r = warp + kMarchWarps * h;
                const int y = y0 + warp + kMarchWarps * h;
                const bool row_wraps = py && y == ny;               // computes E of row 0
                if (!lane_in || (y >= ny && !row_wraps)) continue;
                const int yc = row_wraps ? 0 : y;
                const bool own = !halo_plane && lane_own && r < kMarchOwnY && !row_wraps;
                const int sh = (r + 1) * S::BXW + off + lane;
                const int se = r * S::BXW + off + lane;
                const Rows<T> &rw = no_rows;
                T mE[3] = {mxE, T(1), mzE};
                if constexpr (METRIC) {
                    if (g.metric[0][1] != nullptr) mE[1] = g.metric[0][1][yc];
                }
                T ex, ey, ez;
                const bool cpml_row = ((rowbits >> h) & 1u) || rzE >= 0;
                const bool plain_xy = !((rowbits >> h) & 1u) && !((rowbits >> (R + h)) & 1u) && zprev && !smask;
                const bool fast = MODE == 1 || (ZPURE ? rzE < 0 && zprev : !cpml_row && plain_xy);
                if (XPURE) {
                    const int pxo = args.psi_parity[0];
                    march_e_xtier<T, SAMPLES, D>(g, hk, hm, ek, sh, se, xc > 0, rx_e, (kz * ny + yc) * g.rows[0][0] + rx_e,
                                                 par ? pxo : 0, par ? 0 : pxo, own, qx_e, ex, ey, ez);
                } else if (YPURE) {
                    const int ry = TFD_SLAB_ROW(args, 0, 1, yc);
                    if (ry < 0 && yc > 0 && !smask) {
                        ex = march_e_fast<T, SAMPLES, D, 0>(g, hk, hm, ek, sh, se);
                        ey = march_e_fast<T, SAMPLES, D, 1>(g, hk, hm, ek, sh, se);
                        ez = march_e_fast<T, SAMPLES, D, 2>(g, hk, hm, ek, sh, se);
                    } else {
                        const int pyo = args.psi_parity[1];
                        march_e_ytier<T, SAMPLES, D>(g, hk, hm, ek, sh, se, yc > 0, ry, (kz * g.rows[0][1] + ry) * g.pitch + xc,
                                                     par ? pyo : 0, par ? 0 : pyo, own, coef_at(g, 0, 1, yc, ry), ex, ey, ez);
                    }
                } else if (fast) {
                    ex = march_e_fast<T, SAMPLES, D, 0, METRIC>(g, hk, hm, ek, sh, se, mE);
                    ey = march_e_fast<T, SAMPLES, D, 1, METRIC>(g, hk, hm, ek, sh, se, mE);
                    ez = march_e_fast<T, SAMPLES, D, 2, METRIC>(g, hk, hm, ek, sh, se, mE);
                } else if (ZPURE || (ZTIER && plain_xy)) {
                    // A z-slab row (rzE >= 0), or in the z-pure body also the first plane of the grid (!zprev).
                    const int pz = args.psi_parity[2];
                    march_e_zslab<T, SAMPLES, D>(g, hk, hm, ek, sh, se, zprev, zprev && rzE >= 0, (rzE * ny + yc) * g.pitch + xc,
                                                 par ? pz : 0, par ? 0 : pz, own, coef_at(g, 0, 2, kz, rzE), ex, ey, ez);
                } else if (!cpml_row) {
                    march_e_row<T, SAMPLES, D, false, PXY, METRIC>(g, hk, hm, ek, sh, se, xc, yc, kz, zprev, own, rw, ex, ey, ez, mE);
                } else {
                    const Rows<T> rc = e_rows(xc, yc, kz, rzE);
                    march_e_row<T, SAMPLES, D, true, PXY, METRIC>(g, hk, hm, ek, sh, se, xc, yc, kz, zprev, own, rc, ex, ey, ez, mE);
                }
                if (smask) {
                    ex = inject_masked(g, smask, 0, 0, n, xc, yc, kz, ex);
                    ey = inject_masked(g, smask, 0, 1, n, xc, yc, kz, ey);
                    ez = inject_masked(g, smask, 0, 2, n, xc, yc, kz, ez);
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
        if (__syncthreads_or(late)) {
            give_up(t);
            return;
        }
        // The E slot of plane k is free: refill it D+1 planes ahead.
        if (tid == 0 && compute_e && t + S::NE < ne) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue_e(t + S::NE);
        }
        if (k > z0) {
            // H_new(k-1) on the owned tile.
            const int km = k - 1;
            const T *hs = hstage(t);
            const bool znext = compute_e;
            const int rzH = TFD_SLAB_ROW(args, 1, 2, km);
            const unsigned hmask = tile_src_h ? source_mask(g, 1, x0, x0 + kMarchOwnX, y0, y0 + kMarchOwnY, km, n) & tile_src_h : 0u;
            T *gH[3] = {g.H[0][0] + fn + (size_t)km * g.plane, g.H[0][1] + fn + (size_t)km * g.plane,
                        g.H[0][2] + fn + (size_t)km * g.plane};
            T mzH = T(1);
            if constexpr (METRIC) {
                if (g.metric[1][2] != nullptr) mzH = g.metric[1][2][km];
            }
#pragma unroll kRowUnroll
            for (int h = 0; h < kMarchRowsPerThread; ++h) {
                const int r = warp + kMarchWarps * h;
                const int y = y0 + warp + kMarchWarps * h;
                if (!lane_own || r >= kMarchOwnY || y >= ny) continue;
                const int sh = (r + 1) * S::BXW + off + lane;
                const int e = r * kMarchLanes + lane;
                const int i = y * g.pitch + x;
                const bool cpml_row = ((rowbits >> (2 * R + h)) & 1u) || rzH >= 0;
                const bool fast = !XPURE && (MODE == 1 || (YPURE ? TFD_SLAB_ROW(args, 1, 1, y) < 0 && y < ny - 1 && !hmask
                                                          : ZPURE ? rzH < 0 && znext
                                                                  : !cpml_row && !((rowbits >> (3 * R + h)) & 1u) && znext && !hmask));
                T mH[3] = {mxH, T(1), mzH};
                if constexpr (METRIC) {
                    if (g.metric[1][1] != nullptr) mH[1] = g.metric[1][1][y];
                }
                if (fast) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const Term t0 = term_of(c, 0), t1 = term_of(c, 1);
                        auto dif = [&](const Term &tm) -> T {
                            const T *ep = eprv + tm.in * S::EBUF;
                            const T d = tm.axis == 0 ? ep[e + 1] - ep[e]
                                      : tm.axis == 1 ? ep[e + kMarchLanes] - ep[e] : ecur[tm.in * S::EBUF + e] - ep[e];
                            if constexpr (METRIC) return d * mH[tm.axis];
                            return d;
                        };
                        const T d0 = dif(t0), d1 = dif(t1);
                        T acc = T(0);
                        acc = acc + (t0.sign > 0 ? d0 : -d0);
                        acc = acc + (t1.sign > 0 ? d1 : -d1);
                        T hv = hs[c * HS + sh] - g.cn * acc;
                        if (INTERIOR && hmask) hv = inject_masked(g, hmask, 1, c, n, x, y, km, hv);
                        gH[c][i] = hv;
                    }
                    continue;
                }
                if constexpr (!INTERIOR || ZPURE) {
                    // Interior tiles have their +x / +y neighbours.
                    const bool xn = ZPURE || x < nx - 1 || px, yn = ZPURE || y < ny - 1 || py;
                    T hv[3];
                    if (XPURE) {
                        march_h_xtier<T, SAMPLES, D>(g, eprv, ecur, hs, sh, e, xn, rx_h, (km * ny + y) * g.rows[1][0] + rx_h, qx_h, hv[0],
                                                     hv[1], hv[2]);
                    } else if (YPURE) {
                        const int ry = TFD_SLAB_ROW(args, 1, 1, y);
                        march_h_ytier<T, SAMPLES, D>(g, eprv, ecur, hs, sh, e, yn, ry, (km * g.rows[1][1] + ry) * g.pitch + x,
                                                     coef_at(g, 1, 1, y, ry), hv[0], hv[1], hv[2]);
                    } else if (ZPURE || (ZTIER && !((rowbits >> (2 * R + h)) & 1u) && !((rowbits >> (3 * R + h)) & 1u) && znext && !hmask)) {
                        // A z-slab row (rzH >= 0), or in the z-pure body also the last plane of the grid (!znext).
                        march_h_zslab<T, SAMPLES, D>(g, eprv, ecur, hs, sh, e, znext, znext && rzH >= 0, (rzH * ny + y) * g.pitch + x,
                                                     coef_at(g, 1, 2, km, rzH), hv[0], hv[1], hv[2]);
                    } else if (cpml_row) {
                        const int rx = TFD_SLAB_ROW(args, 1, 0, x), ry = TFD_SLAB_ROW(args, 1, 1, y);
                        march_h_row<T, SAMPLES, D, true, METRIC>(g, eprv, ecur, hs, sh, e, x, y, km, xn, yn, znext, rx, ry, rzH,
                                                                 coef_at(g, 1, 0, x, rx), coef_at(g, 1, 1, y, ry),
                                                                 coef_at(g, 1, 2, km, rzH), hv[0], hv[1], hv[2], mH);
                    } else {
                        const Coef<T> q0{T(0), T(0), T(1)};
                        march_h_row<T, SAMPLES, D, false, METRIC>(g, eprv, ecur, hs, sh, e, x, y, km, xn, yn, znext, -1, -1, -1, q0, q0,
                                                                  q0, hv[0], hv[1], hv[2], mH);
                    }
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        if (hmask) hv[c] = inject_masked(g, hmask, 1, c, n, x, y, km, hv[c]);
                        gH[c][i] = hv[c];
                    }
                }
            }
        }
        __syncthreads();
        // The H slot of plane k-1 is free: refill it D+2 planes ahead.
        if (tid == 0 && t + S::NH < nh) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue_h(t + S::NH);
        }
    }
}

template <typename T, int SAMPLES, int D, int MINB, int MODE, bool METRIC = false>
__global__ void __launch_bounds__(kMarchThreads, MINB) k_step_march(const __grid_constant__ MarchArgs<T> args, int tx_off, int ty_off,
                                                                    int lz, int z_lo, int z_hi) {
    const int z0 = z_lo + blockIdx.z * lz;
    march_body<T, SAMPLES, D, MODE, METRIC>(args, blockIdx.x + tx_off, blockIdx.y + ty_off, z0, min(z0 + lz, z_hi));
}

// One launch over every tile and z chunk in which each CTA takes the pure body (MODE 1) when its tile is in
// the interior block [ix0, ix1) x [iy0, iy1) and its chunk in the pure z segment, the z-pure body (MODE 4)
// for the interior block's other chunks, else the general body (GEN: 0, or 2 with periodic seams). The planes are cut into three segments, [zb0, zb1), [zb1, zb2) (the
// pure one) and [zb2, zb3), chunked separately (chunks[s] of lz[s] planes; blockIdx.z runs over all).
// The two bodies share no state inside the plane loop, so the pure one is compiled as lean as in its own
// kernel, while its CTAs interleave with the general ones as in one launch.
struct MarchMix {
    int ix0, ix1, iy0, iy1;
    int xband;                   // 1: on pure planes, x-boundary tiles of the interior y range take the x-boundary body and
                                 // y-boundary tiles of the interior x range the y-boundary body
    int zb[4];
    int lz[3], chunks[3];
};

// METRIC (a nonuniform mesh, GEN 0): the pure body with the metric factors on the interior block's pure planes,
// the general metric body elsewhere (the z-pure and boundary bodies assume unit factors).
template <typename T, int SAMPLES, int D, int MINB, int GEN, bool METRIC = false>
__global__ void __launch_bounds__(kMarchThreads, MINB) k_step_march_mixed(const __grid_constant__ MarchArgs<T> args,
                                                                          const __grid_constant__ MarchMix mx) {
    int zc = blockIdx.z, seg = 0;
    while (seg < 2 && zc >= mx.chunks[seg]) {
        zc -= mx.chunks[seg];
        ++seg;
    }
    const int z0 = mx.zb[seg] + zc * mx.lz[seg];
    const int z1 = min(z0 + mx.lz[seg], mx.zb[seg + 1]);
    const int tx = blockIdx.x, ty = blockIdx.y;
    const bool yband = ty >= mx.iy0 && ty < mx.iy1;
    const bool interior = tx >= mx.ix0 && tx < mx.ix1 && yband;
    if constexpr (METRIC) {
        if (interior && seg == 1) march_body<T, SAMPLES, D, 1, true>(args, tx, ty, z0, z1);
        else march_body<T, SAMPLES, D, 0, true>(args, tx, ty, z0, z1);
        return;
    }
    if (interior && seg == 1)
        march_body<T, SAMPLES, D, 1>(args, tx, ty, z0, z1);
    else if (interior)
        march_body<T, SAMPLES, D, 4>(args, tx, ty, z0, z1);
    else if (GEN == 0 && mx.xband && yband && seg == 1)
        march_body<T, SAMPLES, D, 5>(args, tx, ty, z0, z1);
    else if (GEN == 0 && mx.xband && tx >= mx.ix0 && tx < mx.ix1 && seg == 1)
        march_body<T, SAMPLES, D, 6>(args, tx, ty, z0, z1);
    else
        march_body<T, SAMPLES, D, GEN>(args, tx, ty, z0, z1);
}

}  // namespace tfd
