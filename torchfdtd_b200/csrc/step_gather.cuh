// Fused E+H step, gather form: one thread per cell.
//
// Thread (x, y, z) computes E_new at its own cell (writing E and the E-family CPML
// memory), then H_new at its own cell. The H update's forward differences need
// E_new at (x+1), (y+1), (z+1); the thread recomputes those values from the old
// buffers with the same arithmetic their owners use (bitwise identical, including
// CPML and soft sources) instead of waiting for them, so a single launch advances a
// whole step with no grid-wide synchronisation. Every arithmetic step follows the
// reference operation order (torchfdtd/boundaries.py:363-438, torchfdtd/cuda_kernels.py:
// 186-259,327-347): d = F[i] - F[i-1]; psi = psi*b + c*d; d = d*(1/kappa) + psi;
// curl = (0 + s0*d0) + s1*d1; E += (cn*inv_eps)*curl; H -= cn*curl; soft sources are
// added after the family update. On a nonuniform mesh each plain difference (periodic wrap
// included, PEC ghost excluded) is first multiplied by the metric factor of the updated cell. The library is compiled with --fmad=false so no
// multiply-add is contracted, as in the reference's NVRTC build.
//
// This kernel is the parity baseline and the fallback for shapes the marching
// kernel does not tile; its extra work is three recomputed E components per H
// component, served from L1/L2.
#pragma once
#include "internal.cuh"

namespace tfd {

template <typename T>
__device__ __forceinline__ T inject(const Grid<T> &g, int family, int comp, long long n, int x, int y, int z, T v) {
    if (n < g.steps) {
        for (int s = 0; s < g.n_src; ++s) {
            const SourceTerm &t = g.src[s];
            if (t.family == family && t.comp == comp && x >= t.lo[0] && x < t.hi[0] && y >= t.lo[1] && y < t.hi[1] &&
                z >= t.lo[2] && z < t.hi[2])
                v = v + g.src_values[(long long)s * g.steps + n];
        }
    }
    return v;
}

// One backward-difference curl term of E component C (k-th of its two terms).
template <typename T, int C, int K>
__device__ __forceinline__ void e_term(const Grid<T> &g, int par, int x, int y, int z, long long i, bool own, T &acc) {
    constexpr Term t = term_of(C, K);
    const int a = t.axis;
    if (g.n[a] == 1) return;
    const int coord = a == 0 ? x : (a == 1 ? y : z);
    const T *h = g.H[par][t.in];
    const T *mt = g.metric[0][a];
    T d = T(0);
    if (coord > 0) {
        d = h[i] - h[i - g.stride(a)];
        if (mt != nullptr) d = d * mt[coord];
        const int *rm = g.row[0][a];
        if (rm != nullptr) {
            const int r = rm[coord];
            if (r >= 0) {
                const long long p = g.psi_index(a, x, y, z, r, g.rows[0][a]);
                const T mem = g.psiE[par][a][t.j][p] * g.cb[0][a][coord] + g.cc[0][a][coord] * d;
                if (own) g.psiE[par ^ 1][a][t.j][p] = mem;
                d = d * g.ck[0][a][coord] + mem;
            }
        }
    } else if (g.periodic[a]) {
        d = h[i] - h[i + (long long)(g.n[a] - 1) * g.stride(a)];
        if (mt != nullptr) d = d * mt[0];
    }
    acc = acc + (t.sign > 0 ? d : -d);
}

// The coupled trapezoidal ADE of dispersive sample j: E_new from the free update and the old E, and (when own)
// the pole states advanced. Reference operation order (torchfdtd/materials.py:67-88).
template <typename T>
__device__ __forceinline__ T ade_correct(const Grid<T> &g, int j, T old, T free, bool own) {
    int s = 0;
    while (s + 1 < g.n_ade && j >= g.ade[s + 1].start) ++s;
    const AdeDev<T> &st = g.ade[s];
    const int l = j - st.start, ns = st.samples;
    auto response = [&](int p) -> T { return (st.Q[p * ns + l] - st.a[p] * st.P[p * ns + l]) / st.d[p]; };
    T total = response(0);
    for (int p = 1; p < st.poles; ++p) total = total + response(p);
    const T e = (st.eps * free - st.ksum * old - total) / st.denom;
    if (own) {
        for (int p = 0; p < st.poles; ++p) {
            const T delta = response(p) + st.k[p] * (e + old);
            st.P[p * ns + l] = st.P[p * ns + l] + delta;
            st.Q[p * ns + l] = -st.Q[p * ns + l] + T(2) * delta;
        }
    }
    return e;
}

template <typename T, int C>
__device__ __forceinline__ T e_value(const Grid<T> &g, int par, long long n, int x, int y, int z, long long i, bool own) {
    T acc = T(0);
    e_term<T, C, 0>(g, par, x, y, z, i, own, acc);
    e_term<T, C, 1>(g, par, x, y, z, i, own, acc);
    T e = g.E[par][C][i] + (g.cn * g.inv_eps[C][i]) * acc;
    if (g.ade_map[C] != nullptr) {
        const int j = g.ade_map[C][i];
        if (j >= 0) e = ade_correct(g, j, g.E[par][C][i], e, own);
    }
    return inject(g, 0, C, n, x, y, z, e);
}

template <typename T, int IN>
__device__ __forceinline__ T e_neighbour(const Grid<T> &g, int par, long long n, int a, int x, int y, int z, long long i, int coord_to) {
    // E_new of component IN at the cell whose axis-a coordinate is coord_to (not owned).
    long long j = i + (long long)(coord_to - (a == 0 ? x : a == 1 ? y : z)) * g.stride(a);
    int xx = a == 0 ? coord_to : x, yy = a == 1 ? coord_to : y, zz = a == 2 ? coord_to : z;
    return e_value<T, IN>(g, par, n, xx, yy, zz, j, false);
}

// STORED: the neighbour's E_new is read from the new buffer (written by the split E kernel, with the TFSF E
// corrections) instead of recomputed.
template <typename T, int C, int K, bool STORED = false>
__device__ __forceinline__ void h_term(const Grid<T> &g, int par, long long n, int x, int y, int z, long long i, const T *e_own,
                                       T &acc) {
    constexpr Term t = term_of(C, K);
    const int a = t.axis;
    if (g.n[a] == 1) return;
    const int coord = a == 0 ? x : (a == 1 ? y : z);
    const T *mt = g.metric[1][a];
    auto e_at = [&](int to) -> T {
        if constexpr (STORED) return g.E[par ^ 1][t.in][i + (long long)(to - coord) * g.stride(a)];
        return e_neighbour<T, t.in>(g, par, n, a, x, y, z, i, to);
    };
    T d = T(0);
    if (coord < g.n[a] - 1) {
        d = e_at(coord + 1) - e_own[t.in];
        if (mt != nullptr) d = d * mt[coord];
        const int *rm = g.row[1][a];
        if (rm != nullptr) {
            const int r = rm[coord];
            if (r >= 0) {
                const long long p = g.psi_index(a, x, y, z, r, g.rows[1][a]);
                T *psi = g.psiH[a][t.j];
                const T mem = psi[p] * g.cb[1][a][coord] + g.cc[1][a][coord] * d;
                psi[p] = mem;
                d = d * g.ck[1][a][coord] + mem;
            }
        }
    } else if (g.periodic[a]) {
        d = e_at(0) - e_own[t.in];
        if (mt != nullptr) d = d * mt[coord];
    } else if (g.pec_on[a]) {
        d = g.pec_neg[a] * e_own[t.in];
    }
    acc = acc + (t.sign > 0 ? d : -d);
}

template <typename T, int C, bool STORED = false>
__device__ __forceinline__ T h_value(const Grid<T> &g, int par, long long n, int x, int y, int z, long long i, const T *e_own) {
    T acc = T(0);
    h_term<T, C, 0, STORED>(g, par, n, x, y, z, i, e_own, acc);
    h_term<T, C, 1, STORED>(g, par, n, x, y, z, i, e_own, acc);
    const T h = g.H[par][C][i] - g.cn * acc;
    return inject(g, 1, C, n, x, y, z, h);
}

// ACTIVE: bitmask of advanced components (bit c: E_c, bit 3+c: H_c).
// Launch: blockIdx.x = row (z*ny + y), blockIdx.y = 128-cell chunk of the row.
template <typename T, int ACTIVE>
__global__ void __launch_bounds__(128) k_step_gather_rows(const __grid_constant__ Grid<T> g) {
    const long long n = *g.counter;
    if (n >= g.steps) return;                   // past the plan's last step: a step is a no-op
    const int par = (int)(n & 1);
    const int x = blockIdx.y * blockDim.x + threadIdx.x;
    const int y = blockIdx.x % g.n[1];
    const int z = blockIdx.x / g.n[1];
    if (x >= g.n[0]) return;
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    T e[3] = {T(0), T(0), T(0)};
    if (ACTIVE & 1) { e[0] = e_value<T, 0>(g, par, n, x, y, z, i, true); g.E[par ^ 1][0][i] = e[0]; }
    if (ACTIVE & 2) { e[1] = e_value<T, 1>(g, par, n, x, y, z, i, true); g.E[par ^ 1][1][i] = e[1]; }
    if (ACTIVE & 4) { e[2] = e_value<T, 2>(g, par, n, x, y, z, i, true); g.E[par ^ 1][2][i] = e[2]; }
    if (ACTIVE & 8) g.H[par ^ 1][0][i] = h_value<T, 0>(g, par, n, x, y, z, i, e);
    if (ACTIVE & 16) g.H[par ^ 1][1][i] = h_value<T, 1>(g, par, n, x, y, z, i, e);
    if (ACTIVE & 32) g.H[par ^ 1][2][i] = h_value<T, 2>(g, par, n, x, y, z, i, e);
}

// The step split in two launches (plans with TFSF boxes, whose E corrections must land between the E and the
// H update, and plans with dispersive materials, whose pole states each E sample advances exactly once): the E
// kernel writes E_new and the E-family CPML memories, the H kernel reads E_new back.
// Whether the cell's family-f CPML row on axis a is absent (no slab there) and no metric factor applies.
template <typename T>
__device__ __forceinline__ bool gather_plain_axis(const Grid<T> &g, int f, int a, int coord) {
    return g.metric[f][a] == nullptr && (g.row[f][a] == nullptr || g.row[f][a][coord] < 0);
}

template <typename T, int ACTIVE>
__global__ void __launch_bounds__(128) k_step_gather_e(const __grid_constant__ Grid<T> g) {
    const long long n = *g.counter;
    if (n >= g.steps) return;
    const int par = (int)(n & 1);
    const int x = blockIdx.y * blockDim.x + threadIdx.x;
    const int y = blockIdx.x % g.n[1];
    const int z = blockIdx.x / g.n[1];
    if (x >= g.n[0]) return;
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    // Plain cells (all six components advanced; on every axis of the grid the -1 neighbour exists and no
    // E-family CPML term or metric factor applies): the bare backward differences, every H value loaded before
    // the stores; the general path's arithmetic reduces to exactly this there (then ADE and sources as usual).
    if (ACTIVE == 63 && g.active == 63 && x >= 1 && gather_plain_axis(g, 0, 0, x) && (y >= 1 || g.n[1] == 1) &&
        (g.n[1] == 1 || gather_plain_axis(g, 0, 1, y)) && (z >= 1 || g.n[2] == 1) && (g.n[2] == 1 || gather_plain_axis(g, 0, 2, z))) {
        T hc[3], hm[3][2], eo[3], ie[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            hc[c] = g.H[par][c][i];
            eo[c] = g.E[par][c][i];
            ie[c] = g.inv_eps[c][i];
        }
#pragma unroll
        for (int C = 0; C < 3; ++C)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const Term t = term_of(C, k);
                hm[C][k] = g.n[t.axis] == 1 ? T(0) : g.H[par][t.in][i - g.stride(t.axis)];
            }
        int jc[3];
#pragma unroll
        for (int C = 0; C < 3; ++C) jc[C] = g.ade_map[C] != nullptr ? g.ade_map[C][i] : -1;
        T e[3];
#pragma unroll
        for (int C = 0; C < 3; ++C) {
            T acc = T(0);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const Term t = term_of(C, k);
                if (g.n[t.axis] == 1) continue;
                const T d = hc[t.in] - hm[C][k];
                acc = acc + (t.sign > 0 ? d : -d);
            }
            e[C] = eo[C] + (g.cn * ie[C]) * acc;
        }
        if (jc[0] >= 0 || jc[1] >= 0 || jc[2] >= 0) {
            // Dispersive samples: the pole states of every component are loaded before any correction is computed
            // (single-pole states; several poles take ade_correct). Same arithmetic as ade_correct.
            int st_of[3], l_of[3];
            T Pv[3], Qv[3];
#pragma unroll
            for (int C = 0; C < 3; ++C) {
                st_of[C] = -1;
                if (jc[C] < 0) continue;
                int s = 0;
                while (s + 1 < g.n_ade && jc[C] >= g.ade[s + 1].start) ++s;
                st_of[C] = s;
                l_of[C] = jc[C] - g.ade[s].start;
                if (g.ade[s].poles == 1) {
                    Pv[C] = g.ade[s].P[l_of[C]];
                    Qv[C] = g.ade[s].Q[l_of[C]];
                }
            }
#pragma unroll
            for (int C = 0; C < 3; ++C) {
                if (jc[C] < 0) continue;
                const AdeDev<T> &st = g.ade[st_of[C]];
                if (st.poles != 1) {
                    e[C] = ade_correct(g, jc[C], eo[C], e[C], true);
                    continue;
                }
                const T resp = (Qv[C] - st.a[0] * Pv[C]) / st.d[0];
                const T total = resp;
                const T v = (st.eps * e[C] - st.ksum * eo[C] - total) / st.denom;
                const T delta = resp + st.k[0] * (v + eo[C]);
                st.P[l_of[C]] = Pv[C] + delta;
                st.Q[l_of[C]] = -Qv[C] + T(2) * delta;
                e[C] = v;
            }
        }
#pragma unroll
        for (int C = 0; C < 3; ++C) e[C] = inject(g, 0, C, n, x, y, z, e[C]);
#pragma unroll
        for (int C = 0; C < 3; ++C) g.E[par ^ 1][C][i] = e[C];
        return;
    }
    if (ACTIVE & 1) g.E[par ^ 1][0][i] = e_value<T, 0>(g, par, n, x, y, z, i, true);
    if (ACTIVE & 2) g.E[par ^ 1][1][i] = e_value<T, 1>(g, par, n, x, y, z, i, true);
    if (ACTIVE & 4) g.E[par ^ 1][2][i] = e_value<T, 2>(g, par, n, x, y, z, i, true);
}

template <typename T, int ACTIVE>
__global__ void __launch_bounds__(128) k_step_gather_h(const __grid_constant__ Grid<T> g) {
    const long long n = *g.counter;
    if (n >= g.steps) return;
    const int par = (int)(n & 1);
    const int x = blockIdx.y * blockDim.x + threadIdx.x;
    const int y = blockIdx.x % g.n[1];
    const int z = blockIdx.x / g.n[1];
    if (x >= g.n[0]) return;
    const long long i = (long long)z * g.plane + (long long)y * g.pitch + x;
    T e[3] = {T(0), T(0), T(0)};
    if (ACTIVE & 1) e[0] = g.E[par ^ 1][0][i];
    if (ACTIVE & 2) e[1] = g.E[par ^ 1][1][i];
    if (ACTIVE & 4) e[2] = g.E[par ^ 1][2][i];
    // Plain cells: on every axis of the grid the +1 neighbour exists and no H-family CPML term or metric factor
    // applies; the bare forward differences of the stored E_new.
    if (ACTIVE == 63 && g.active == 63 && x < g.n[0] - 1 && gather_plain_axis(g, 1, 0, x) && (y < g.n[1] - 1 || g.n[1] == 1) &&
        (g.n[1] == 1 || gather_plain_axis(g, 1, 1, y)) && (z < g.n[2] - 1 || g.n[2] == 1) && (g.n[2] == 1 || gather_plain_axis(g, 1, 2, z))) {
        T ep[3][2], ho[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) ho[c] = g.H[par][c][i];
#pragma unroll
        for (int C = 0; C < 3; ++C)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const Term t = term_of(C, k);
                ep[C][k] = g.n[t.axis] == 1 ? T(0) : g.E[par ^ 1][t.in][i + g.stride(t.axis)];
            }
        T h[3];
#pragma unroll
        for (int C = 0; C < 3; ++C) {
            T acc = T(0);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const Term t = term_of(C, k);
                if (g.n[t.axis] == 1) continue;
                const T d = ep[C][k] - e[t.in];
                acc = acc + (t.sign > 0 ? d : -d);
            }
            h[C] = inject(g, 1, C, n, x, y, z, ho[C] - g.cn * acc);
        }
#pragma unroll
        for (int C = 0; C < 3; ++C) g.H[par ^ 1][C][i] = h[C];
        return;
    }
    if (ACTIVE & 8) g.H[par ^ 1][0][i] = h_value<T, 0, true>(g, par, n, x, y, z, i, e);
    if (ACTIVE & 16) g.H[par ^ 1][1][i] = h_value<T, 1, true>(g, par, n, x, y, z, i, e);
    if (ACTIVE & 32) g.H[par ^ 1][2][i] = h_value<T, 2, true>(g, par, n, x, y, z, i, e);
}

}  // namespace tfd
