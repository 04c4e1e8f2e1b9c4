// Discrete adjoint of one Yee/CPML step, gather form: one thread per cell.
//
// The forward step n maps the state s_n = (E, H, psi) to s_{n+1}:
//     E' = E + (cn / eps) curl_b(H; psi_E)      then E sources
//     H' = H - cn curl_f(E'; psi_H)             then H sources
// and observations sample s_{n+1}. Its transpose (reference torchfdtd/differentiable.py:489-519,
// _System.transpose_step, with the CPML memory transpose of curl_faces_transpose :369-432) maps the
// adjoint lambda_{n+1} = (e_bar, h_bar, psi_bar) to lambda_n:
//     e_bar += curl_f^T(-cn h_bar)              (psi_H bars: m = psi_bar + v, psi_bar <- b m, v <- v/kappa + c m)
//     dJ/d eps += -cn e_bar curl_b(H_n; psi_E,n) / eps^2
//     h_bar += curl_b^T((cn / eps) e_bar)       (psi_E bars likewise)
// Sources are additive constants and drop out; observation seeds are added to e_bar / h_bar before
// the transpose of the step whose result they sampled. On a nonuniform mesh the forward scales each plain
// difference by the cell's metric factor before its CPML terms, so the transpose scales each D value after
// the CPML memory transpose (reference torchfdtd/differentiable.py:409-418).
//
// curl_f^T is a backward difference of the per-H-cell values D(k) (k = 0..n-2, plus the periodic wrap or
// PEC edge at n-1) and curl_b^T a forward difference of per-E-cell values D(k) (k = 1..n-1, plus the
// periodic edge at 0), so the adjoint step has the forward step's stencil shape. It runs as two
// launches, one thread per cell: k_adjoint_e writes e_bar_new (and accumulates the sensitivity),
// k_adjoint_h reads e_bar_new of its own cell and its +x, +y, +z neighbours back and writes h_bar_new.
// (A single launch that recomputes the neighbours' e_bar_new, as the forward gather kernel recomputes E,
// ran about 4x slower: each h_bar term needs a neighbour's e_bar, which needs CPML-transposed D values
// at two cells.) Adjoint fields and both families' adjoint CPML memories are double-buffered by
// reverse-step parity; each memory is written once, by the thread that owns its cell. The forward state comes from a restart snapshot (tfd_state_save)
// of s_n, so no forward buffer is disturbed.
//
// The material sensitivity is accumulated as S_c = sum_n e_bar_c * curl_b(H)_c per component; the host
// forms dJ/d eps = -cn S / eps^2 (summed over components for a per-cell permittivity).
#pragma once
#include "internal.cuh"

namespace tfd {

// Terms of the curl whose INPUT is component C, in reference CURL_TERMS order (ascending axis):
// {axis, out, sign, j}.
struct RevTerm { int axis, out, sign, j; };
__host__ __device__ constexpr RevTerm rev_of(int in, int k) {
    return in == 0 ? (k == 0 ? RevTerm{1, 2, -1, 1} : RevTerm{2, 1, +1, 1})
         : in == 1 ? (k == 0 ? RevTerm{0, 2, +1, 1} : RevTerm{2, 0, -1, 0})
                   : (k == 0 ? RevTerm{0, 1, -1, 0} : RevTerm{1, 0, +1, 0});
}

template <typename T>
struct AdjArgs {
    Grid<T> g;                   // geometry, CPML tables, 1/eps; its field pointers are not used
    long long sE[3], sH[3];      // element offsets of the snapshot's arrays (-1: absent)
    long long sPsiE[3][2];
    T *eb[2][3], *hb[2][3];      // adjoint fields [parity][component]
    T *pEb[2][3][2], *pHb[2][3][2];   // adjoint CPML memories [parity][axis][term j]
    T *S[3];                     // material sensitivity per E component
    int slab[2][3][4];           // per family and axis: lo0, hi0, lo1, hi1 of the two CPML slabs
};

// Slab row of coordinate c from the (lo, hi) bounds of a (family, axis), or -1: rows of the low slab first.
// The bounds sit in the kernel parameters, so no dependent table load precedes the CPML work.
__device__ __forceinline__ int adj_slab_row(const int *b, int c) {
    return (c >= b[0] && c < b[1]) ? c - b[0] : (c >= b[2] && c < b[3]) ? (b[1] - b[0]) + (c - b[2]) : -1;
}

template <typename T>
__device__ __forceinline__ int coord_of(int a, int x, int y, int z) { return a == 0 ? x : (a == 1 ? y : z); }

// D of an H-family term (output H component `out`, axis a) at H cell k: the transposed forward-difference
// value sign * (-cn h_bar_out[k]) through the CPML memory transpose. Writes the memory when own.
template <typename T>
__device__ __forceinline__ T d_h(const AdjArgs<T> &A, int q, const RevTerm t, int x, int y, int z, long long k, bool own) {
    const Grid<T> &g = A.g;
    const int a = t.axis;
    const int c = coord_of<T>(a, x, y, z);
    const T dst = -g.cn * A.hb[q][t.out][k];
    T v = t.sign > 0 ? dst : -dst;
    const T *mt = g.metric[1][a];
    if (c < g.n[a] - 1) {
        if (A.pHb[q][a][t.j] != nullptr) {
            const int r = adj_slab_row(A.slab[1][a], c);
            if (r >= 0) {
                const long long p = g.psi_index(a, x, y, z, r, g.rows[1][a]);
                const T m = A.pHb[q][a][t.j][p] + v;
                if (own) A.pHb[q ^ 1][a][t.j][p] = g.cb[1][a][c] * m;
                v = v * g.ck[1][a][c] + g.cc[1][a][c] * m;
            }
        }
        return mt != nullptr ? v * mt[c] : v;       // the forward scales before its CPML terms
    }
    if (g.periodic[a]) return mt != nullptr ? v * mt[c] : v;
    if (g.pec_on[a]) return -g.pec_neg[a] * v;       // sign * pec * dst
    return T(0);
}

// e_bar_new of component C at cell (x, y, z), index i.
template <typename T, int C>
__device__ __forceinline__ T ebar_value(const AdjArgs<T> &A, int q, int x, int y, int z, long long i, bool own) {
    const Grid<T> &g = A.g;
    T contrib = T(0);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const RevTerm t = rev_of(C, k);
        const int a = t.axis;
        if (g.n[a] == 1) continue;
        const int out_bit = 1 << (3 + t.out);
        if (!(g.active & out_bit)) continue;
        const int c = coord_of<T>(a, x, y, z);
        const int n = g.n[a];
        const long long s = g.stride(a);
        if (c >= 1) {                                   // src[c] += D(c-1)
            const int xm = a == 0 ? x - 1 : x, ym = a == 1 ? y - 1 : y, zm = a == 2 ? z - 1 : z;
            contrib = contrib + d_h(A, q, t, xm, ym, zm, i - s, false);
        }
        if (c <= n - 2) contrib = contrib - d_h(A, q, t, x, y, z, i, own);   // src[c] -= D(c)
        if (g.periodic[a]) {                            // wrap edge D(n-1): src[0] += D, src[n-1] -= D
            if (c == 0) {
                const int xw = a == 0 ? n - 1 : x, yw = a == 1 ? n - 1 : y, zw = a == 2 ? n - 1 : z;
                contrib = contrib + d_h(A, q, t, xw, yw, zw, i + (long long)(n - 1) * s, false);
            }
            if (c == n - 1) contrib = contrib - d_h(A, q, t, x, y, z, i, false);
        } else if (g.pec_on[a] && c == n - 1) {
            contrib = contrib - d_h(A, q, t, x, y, z, i, false);
        }
    }
    return A.eb[q][C][i] + contrib;
}

// D of an E-family term (output E component `out`, axis a) at E cell k: sign * (cn / eps) e_bar_new_out[k]
// through the CPML memory transpose. Writes the memory when own.
template <typename T>
__device__ __forceinline__ T d_e(const AdjArgs<T> &A, int q, const RevTerm t, int x, int y, int z, long long k, T ebar_out,
                                 bool own) {
    const Grid<T> &g = A.g;
    const int a = t.axis;
    const int c = coord_of<T>(a, x, y, z);
    const T dst = (g.cn * g.inv_eps[t.out][k]) * ebar_out;
    T v = t.sign > 0 ? dst : -dst;
    const T *mt = g.metric[0][a];
    if (c >= 1) {
        if (A.pEb[q][a][t.j] != nullptr) {
            const int r = adj_slab_row(A.slab[0][a], c);
            if (r >= 0) {
                const long long p = g.psi_index(a, x, y, z, r, g.rows[0][a]);
                const T m = A.pEb[q][a][t.j][p] + v;
                if (own) A.pEb[q ^ 1][a][t.j][p] = g.cb[0][a][c] * m;
                v = v * g.ck[0][a][c] + g.cc[0][a][c] * m;
            }
        }
        return mt != nullptr ? v * mt[c] : v;
    }
    return g.periodic[a] ? (mt != nullptr ? v * mt[0] : v) : T(0);
}

template <typename T, int C>
__device__ __forceinline__ T ebar_at(const AdjArgs<T> &A, int q, int x, int y, int z, long long i) {
    return ebar_value<T, C>(A, q, x, y, z, i, false);
}

// e_bar_new of component `out` at a neighbour (runtime component).
template <typename T>
__device__ __forceinline__ T ebar_any(const AdjArgs<T> &A, int q, int out, int x, int y, int z, long long i) {
    return out == 0 ? ebar_at<T, 0>(A, q, x, y, z, i) : out == 1 ? ebar_at<T, 1>(A, q, x, y, z, i) : ebar_at<T, 2>(A, q, x, y, z, i);
}

// h_bar_new of H component C at its own cell; e_own[] holds e_bar_new of the own cell. STORED: the
// neighbours' e_bar_new are read from the new buffer (written by k_adjoint_e) instead of recomputed.
template <typename T, int C, bool STORED = false>
__device__ __forceinline__ T hbar_value(const AdjArgs<T> &A, int q, int x, int y, int z, long long i, const T *e_own) {
    const Grid<T> &g = A.g;
    T contrib = T(0);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const RevTerm t = rev_of(C, k);
        const int a = t.axis;
        if (g.n[a] == 1) continue;
        if (!(g.active & (1 << t.out))) continue;
        const int c = coord_of<T>(a, x, y, z);
        const int n = g.n[a];
        const long long s = g.stride(a);
        if (c >= 1) contrib = contrib + d_e(A, q, t, x, y, z, i, e_own[t.out], true);          // src[c] += D(c)
        if (c + 1 <= n - 1) {                                                                   // src[c] -= D(c+1)
            const int xp = a == 0 ? x + 1 : x, yp = a == 1 ? y + 1 : y, zp = a == 2 ? z + 1 : z;
            const T eb = STORED ? A.eb[q ^ 1][t.out][i + s] : ebar_any(A, q, t.out, xp, yp, zp, i + s);
            contrib = contrib - d_e(A, q, t, xp, yp, zp, i + s, eb, false);
        }
        if (g.periodic[a]) {                             // edge D(0): src[0] += D, src[n-1] -= D
            if (c == 0) contrib = contrib + d_e(A, q, t, x, y, z, i, e_own[t.out], false);
            if (c == n - 1) {
                const int x0 = a == 0 ? 0 : x, y0 = a == 1 ? 0 : y, z0 = a == 2 ? 0 : z;
                const long long i0 = i - (long long)(n - 1) * s;
                const T eb = STORED ? A.eb[q ^ 1][t.out][i0] : ebar_any(A, q, t.out, x0, y0, z0, i0);
                contrib = contrib - d_e(A, q, t, x0, y0, z0, i0, eb, false);
            }
        }
    }
    return A.hb[q][C][i] + contrib;
}

// Forward E curl of component C from the snapshot (same arithmetic as the forward E update).
template <typename T, int C>
__device__ __forceinline__ T forward_curl(const AdjArgs<T> &A, const T *slot, int x, int y, int z, long long i) {
    const Grid<T> &g = A.g;
    T acc = T(0);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const Term t = term_of(C, k);
        const int a = t.axis;
        if (g.n[a] == 1) continue;
        const int c = coord_of<T>(a, x, y, z);
        const T *h = slot + A.sH[t.in];
        const T *mt = g.metric[0][a];
        T d = T(0);
        if (c > 0) {
            d = h[i] - h[i - g.stride(a)];
            if (mt != nullptr) d = d * mt[c];
            if (A.sPsiE[a][t.j] >= 0) {
                const int r = adj_slab_row(A.slab[0][a], c);
                if (r >= 0) {
                    const long long p = g.psi_index(a, x, y, z, r, g.rows[0][a]);
                    const T mem = slot[A.sPsiE[a][t.j] + p] * g.cb[0][a][c] + g.cc[0][a][c] * d;
                    d = d * g.ck[0][a][c] + mem;
                }
            }
        } else if (g.periodic[a]) {
            d = h[i] - h[i + (long long)(g.n[a] - 1) * g.stride(a)];
            if (mt != nullptr) d = d * mt[0];
        }
        acc = acc + (t.sign > 0 ? d : -d);
    }
    return acc;
}

// ACTIVE: bitmask of advanced components (bit c: E_c, bit 3+c: H_c). Blocks of kAdjX x kAdjY cells of one
// z plane (blockIdx.x, blockIdx.y: x and y tile; blockIdx.z: plane), so the x and y neighbours a cell reads
// are mostly in its block's L1 lines. The tile origins are shifted by (xs, ys) cells (tile (bx, by) starts at
// (bx kAdjX - xs, by kAdjY - ys)) so that tiles start at x = 1 and y = 1; tiles clear of the grid faces take a
// fast path unless `fast` is 0 (the general path alone, for comparisons). Reads parity q, writes q^1.
constexpr int kAdjX = 32, kAdjY = 8;

// Whether the CPML slab bounds b = {lo0, hi0, lo1, hi1} (half-open) meet the coordinates [lo, hi].
__host__ __device__ __forceinline__ bool adj_meets(const int *b, int lo, int hi) {
    return (lo < b[1] && b[0] <= hi) || (lo < b[3] && b[2] <= hi);
}

// Block classes for the fast paths. Every cell of the block lies in [1, n-2] on every axis (both neighbours
// inside the grid: no face or periodic edge); otherwise the block takes the general path (class -1). Else the
// class is a mask with bit a set when a CPML term may apply to a D value the block's cells evaluate on axis a:
// the H family on [lo - 1, hi] (HFAM: the e_bar update differences D(c-1) and D(c)) and the E family on
// [lo, hi + e_hi]. Terms on the axes of the mask go through the general D functions; the others are the plain
// transposed differences, to which the general path's arithmetic reduces there, in the same order.
template <typename T>
__device__ __forceinline__ int adj_class(const AdjArgs<T> &A, int x0, int y0, int z, bool hfam, int e_hi) {
    const Grid<T> &g = A.g;
    const int lo[3] = {max(x0, 0), max(y0, 0), z};
    const int hi[3] = {min(x0 + kAdjX, g.n[0]) - 1, min(y0 + kAdjY, g.n[1]) - 1, z};
    int mask = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (lo[a] < 1 || hi[a] > g.n[a] - 2) return -1;
        if ((hfam && adj_meets(A.slab[1][a], lo[a] - 1, hi[a])) || adj_meets(A.slab[0][a], lo[a], hi[a] + e_hi)) mask |= 1 << a;
    }
    return mask;
}

// e_bar_new and the sensitivity of the three components of a cell of a fast-path block; GEN: the axes whose
// terms go through the general D functions (the mask above). Every input of the plain terms is loaded before
// the first store (the stores could alias the loads for the compiler, which would otherwise serialise the three
// components' memory round trips).
template <typename T, int GEN>
__device__ __forceinline__ void adj_e_fast(const AdjArgs<T> &A, const T *__restrict__ slot, int q, int x, int y, int z, long long i) {
    const Grid<T> &g = A.g;
    const int co[3] = {x, y, z};
    T hc[3], sc[3], hm[3][2], smv[3][2], eb[3], S0[3];
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        hc[o] = __ldg(A.hb[q][o] + i);
        sc[o] = __ldg(slot + A.sH[o] + i);
        eb[o] = __ldg(A.eb[q][o] + i);
        S0[o] = A.S[o][i];
    }
#pragma unroll
    for (int C = 0; C < 3; ++C)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const RevTerm t = rev_of(C, k);
            if (!((GEN >> t.axis) & 1)) hm[C][k] = __ldg(A.hb[q][t.out] + i - g.stride(t.axis));
            const Term f = term_of(C, k);
            smv[C][k] = __ldg(slot + A.sH[f.in] + i - g.stride(f.axis));
        }
    T e[3], s[3];
#pragma unroll
    for (int C = 0; C < 3; ++C) {
        T contrib = T(0);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const RevTerm t = rev_of(C, k);
            const int a = t.axis, c = co[a];
            if ((GEN >> a) & 1) {
                const int xm = a == 0 ? x - 1 : x, ym = a == 1 ? y - 1 : y, zm = a == 2 ? z - 1 : z;
                contrib = contrib + d_h(A, q, t, xm, ym, zm, i - g.stride(a), false);   // src[c] += D(c-1)
                contrib = contrib - d_h(A, q, t, x, y, z, i, true);                    // src[c] -= D(c)
                continue;
            }
            const T *mt = g.metric[1][a];
            auto dh = [&](T h, int cc) -> T {
                const T dst = -g.cn * h;
                const T v = t.sign > 0 ? dst : -dst;
                return mt != nullptr ? v * mt[cc] : v;
            };
            contrib = contrib + dh(hm[C][k], c - 1);      // src[c] += D(c-1)
            contrib = contrib - dh(hc[t.out], c);         // src[c] -= D(c)
        }
        e[C] = eb[C] + contrib;
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const Term t = term_of(C, k);
            const int a = t.axis, c = co[a];
            const T *mt = g.metric[0][a];
            T d = sc[t.in] - smv[C][k];
            if (mt != nullptr) d = d * mt[c];
            if (((GEN >> a) & 1) && A.sPsiE[a][t.j] >= 0) {
                const int r = adj_slab_row(A.slab[0][a], c);
                if (r >= 0) {
                    const long long p = g.psi_index(a, x, y, z, r, g.rows[0][a]);
                    const T mem = slot[A.sPsiE[a][t.j] + p] * g.cb[0][a][c] + g.cc[0][a][c] * d;
                    d = d * g.ck[0][a][c] + mem;
                }
            }
            acc = acc + (t.sign > 0 ? d : -d);
        }
        s[C] = S0[C] + e[C] * acc;
    }
#pragma unroll
    for (int C = 0; C < 3; ++C) {
        A.eb[q ^ 1][C][i] = e[C];
        A.S[C][i] = s[C];
    }
}

// h_bar_new of the three components of a cell of a fast-path block; e_own: the cell's e_bar_new.
template <typename T, int GEN>
__device__ __forceinline__ void adj_h_fast(const AdjArgs<T> &A, int q, int x, int y, int z, long long i, const T *e_own) {
    const Grid<T> &g = A.g;
    const int co[3] = {x, y, z};
    T ep[3][2], ie0[3], iep[3][2], hb[3];
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        ie0[o] = __ldg(g.inv_eps[o] + i);
        hb[o] = __ldg(A.hb[q][o] + i);
    }
#pragma unroll
    for (int C = 0; C < 3; ++C)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const RevTerm t = rev_of(C, k);
            ep[C][k] = __ldg(A.eb[q ^ 1][t.out] + i + g.stride(t.axis));
            if (!((GEN >> t.axis) & 1)) iep[C][k] = __ldg(g.inv_eps[t.out] + i + g.stride(t.axis));
        }
    T out[3];
#pragma unroll
    for (int C = 0; C < 3; ++C) {
        T contrib = T(0);
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const RevTerm t = rev_of(C, k);
            const int a = t.axis, c = co[a];
            if ((GEN >> a) & 1) {
                const int xp = a == 0 ? x + 1 : x, yp = a == 1 ? y + 1 : y, zp = a == 2 ? z + 1 : z;
                contrib = contrib + d_e(A, q, t, x, y, z, i, e_own[t.out], true);                   // src[c] += D(c)
                contrib = contrib - d_e(A, q, t, xp, yp, zp, i + g.stride(a), ep[C][k], false);    // src[c] -= D(c+1)
                continue;
            }
            const T *mt = g.metric[0][a];
            auto de = [&](T ie, int cc, T eb) -> T {
                const T dst = (g.cn * ie) * eb;
                const T v = t.sign > 0 ? dst : -dst;
                return mt != nullptr ? v * mt[cc] : v;
            };
            contrib = contrib + de(ie0[t.out], c, e_own[t.out]);       // src[c] += D(c)
            contrib = contrib - de(iep[C][k], c + 1, ep[C][k]);        // src[c] -= D(c+1)
        }
        out[C] = hb[C] + contrib;
    }
#pragma unroll
    for (int C = 0; C < 3; ++C) A.hb[q ^ 1][C][i] = out[C];
}

// Part 1 of the reverse step: e_bar_new of the own cell, and S += e_bar_new * curl_b(H_n).
template <typename T, int ACTIVE>
__global__ void __launch_bounds__(kAdjX * kAdjY) k_adjoint_e(const __grid_constant__ AdjArgs<T> A, const T *__restrict__ slot, int q,
                                                             int xs, int ys, int fast) {
    const Grid<T> &g = A.g;
    const int x0 = blockIdx.x * kAdjX - xs, y0 = blockIdx.y * kAdjY - ys;
    const int x = x0 + threadIdx.x;
    const int y = y0 + threadIdx.y;
    const int z = blockIdx.z;
    if (x < 0 || y < 0 || x >= g.n[0] || y >= g.n[1]) return;
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    if (ACTIVE == 63 && fast && g.active == 63) {
        switch (adj_class(A, x0, y0, z, true, 0)) {
            case 0: adj_e_fast<T, 0>(A, slot, q, x, y, z, i); return;
            case 1: adj_e_fast<T, 1>(A, slot, q, x, y, z, i); return;
            case 2: adj_e_fast<T, 2>(A, slot, q, x, y, z, i); return;
            case 3: adj_e_fast<T, 3>(A, slot, q, x, y, z, i); return;
            case 4: adj_e_fast<T, 4>(A, slot, q, x, y, z, i); return;
            case 5: adj_e_fast<T, 5>(A, slot, q, x, y, z, i); return;
            case 6: adj_e_fast<T, 6>(A, slot, q, x, y, z, i); return;
            case 7: adj_e_fast<T, 7>(A, slot, q, x, y, z, i); return;
            default: break;
        }
    }
    if (ACTIVE & 1) {
        const T e = ebar_value<T, 0>(A, q, x, y, z, i, true);
        A.eb[q ^ 1][0][i] = e;
        A.S[0][i] = A.S[0][i] + e * forward_curl<T, 0>(A, slot, x, y, z, i);
    }
    if (ACTIVE & 2) {
        const T e = ebar_value<T, 1>(A, q, x, y, z, i, true);
        A.eb[q ^ 1][1][i] = e;
        A.S[1][i] = A.S[1][i] + e * forward_curl<T, 1>(A, slot, x, y, z, i);
    }
    if (ACTIVE & 4) {
        const T e = ebar_value<T, 2>(A, q, x, y, z, i, true);
        A.eb[q ^ 1][2][i] = e;
        A.S[2][i] = A.S[2][i] + e * forward_curl<T, 2>(A, slot, x, y, z, i);
    }
}

// Part 2: h_bar_new of the own cell from the e_bar_new that part 1 stored (own cell and +x/+y/+z).
template <typename T, int ACTIVE>
__global__ void __launch_bounds__(kAdjX * kAdjY) k_adjoint_h(const __grid_constant__ AdjArgs<T> A, int q, int xs, int ys, int fast) {
    const Grid<T> &g = A.g;
    const int x0 = blockIdx.x * kAdjX - xs, y0 = blockIdx.y * kAdjY - ys;
    const int x = x0 + threadIdx.x;
    const int y = y0 + threadIdx.y;
    const int z = blockIdx.z;
    if (x < 0 || y < 0 || x >= g.n[0] || y >= g.n[1]) return;
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    T e[3] = {T(0), T(0), T(0)};
    if (ACTIVE & 1) e[0] = A.eb[q ^ 1][0][i];
    if (ACTIVE & 2) e[1] = A.eb[q ^ 1][1][i];
    if (ACTIVE & 4) e[2] = A.eb[q ^ 1][2][i];
    if (ACTIVE == 63 && fast && g.active == 63) {
        switch (adj_class(A, x0, y0, z, false, 1)) {
            case 0: adj_h_fast<T, 0>(A, q, x, y, z, i, e); return;
            case 1: adj_h_fast<T, 1>(A, q, x, y, z, i, e); return;
            case 2: adj_h_fast<T, 2>(A, q, x, y, z, i, e); return;
            case 3: adj_h_fast<T, 3>(A, q, x, y, z, i, e); return;
            case 4: adj_h_fast<T, 4>(A, q, x, y, z, i, e); return;
            case 5: adj_h_fast<T, 5>(A, q, x, y, z, i, e); return;
            case 6: adj_h_fast<T, 6>(A, q, x, y, z, i, e); return;
            case 7: adj_h_fast<T, 7>(A, q, x, y, z, i, e); return;
            default: break;
        }
    }
    if (ACTIVE & 8) A.hb[q ^ 1][0][i] = hbar_value<T, 0, true>(A, q, x, y, z, i, e);
    if (ACTIVE & 16) A.hb[q ^ 1][1][i] = hbar_value<T, 1, true>(A, q, x, y, z, i, e);
    if (ACTIVE & 32) A.hb[q ^ 1][2][i] = hbar_value<T, 2, true>(A, q, x, y, z, i, e);
}

// Observation seeds of one step: bar[family][comp][offset] += seed[k] (observers are distinct cells).
template <typename T>
__global__ void k_adjoint_seed(const __grid_constant__ AdjArgs<T> A, const TraceDev *__restrict__ obs, int n_obs,
                               const T *__restrict__ seed, int q) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_obs; k += gridDim.x * blockDim.x) {
        const TraceDev o = obs[k];
        T *bar = o.family == 0 ? A.eb[q][o.comp] : A.hb[q][o.comp];
        if (bar != nullptr) bar[o.offset] = bar[o.offset] + seed[k];
    }
}

}  // namespace tfd
