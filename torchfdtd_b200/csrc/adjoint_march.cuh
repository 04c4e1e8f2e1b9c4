// Discrete adjoint of one Yee/CPML step, marching form: one launch per reverse step, every transposed D value
// evaluated once per cell.
//
// The gather pair (adjoint.cuh: k_adjoint_e, k_adjoint_h) evaluates a CPML-transposed D value in the cell that
// owns it and again in each neighbour that differences it, and round-trips e_bar_new through global memory
// between its two launches. Here a CTA owns a 32 x 8 (x, y) tile and a chunk of z planes and marches up in z.
// For each plane k it
//   A. evaluates the H-family D values of plane k on the tile widened by one cell on every side (34 x 10), the
//      owner writing the H-family CPML memory bars, into shared memory;
//   B. forms e_bar_new of plane k on the tile plus its +x column and +y row (the neighbours the H update below
//      differences), from D(c - e_a) - D(c) in the reference term order, the D values of plane k - 1 kept from
//      the previous plane; owned cells store e_bar_new and accumulate the sensitivity S += e_bar_new curl_b(H_n);
//   C. evaluates the E-family D values of those cells from e_bar_new (owners write the E-family memory bars),
//      into a shared buffer double-buffered over the plane parity;
//   D. forms h_bar_new of plane k - 1 on the owned tile from D(c) - D(c + e_a), the +z values being plane k's.
// The last plane of a chunk is followed by a halo plane (steps A-C without stores) for the H update of the
// chunk's last plane, and its first plane needs the z D values of the plane below (step A without stores).
// Each value is computed with the same device functions and the same operation order as the gather pair, so
// the gradients are bitwise the same. Scope: 3D grids with all six components and no periodic faces (PML / PEC);
// other plans keep the gather pair.
#pragma once
#include "adjoint.cuh"

namespace tfd {

constexpr int kAmX = 32, kAmY = 8, kAmThreads = kAmX * kAmY;
constexpr int kAmHx = kAmX + 2, kAmHy = kAmY + 2;      // H-family D grid: x0-1 .. x0+32, y0-1 .. y0+8
constexpr int kAmEx = kAmX + 1, kAmEy = kAmY + 1;      // e_bar_new / E-family D grid: x0 .. x0+32, y0 .. y0+8

template <typename T>
struct AdjMarchSmem {
    T dh[6][kAmHy][kAmHx];       // H-family D of plane k, term 2*in + kk (rev_of(in, kk))
    T dhz[2][kAmHy][kAmHx];      // the z terms (in 0 and 1, kk 1) of plane k - 1
    T de[2][6][kAmEy][kAmEx];    // E-family D by plane parity, term 2*C + kk
};

template <typename T>
__global__ void __launch_bounds__(kAmThreads) k_adjoint_march(const __grid_constant__ AdjArgs<T> A, const T *__restrict__ slot,
                                                              int q, int lz) {
    extern __shared__ __align__(16) unsigned char am_raw[];
    AdjMarchSmem<T> &sm = *reinterpret_cast<AdjMarchSmem<T> *>(am_raw);
    const Grid<T> &g = A.g;
    const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
    const int x0 = blockIdx.x * kAmX, y0 = blockIdx.y * kAmY;
    const int z0 = blockIdx.z * lz, z1 = min(z0 + lz, nz);
    const int tid = threadIdx.x;
    const long long pitch = g.pitch, plane = g.plane;
    auto index = [&](int x, int y, int z) { return (long long)z * plane + (long long)y * pitch + x; };

    // Step A over the widened grid (own: the cell is in the owned tile and the plane is an owned plane).
    auto d_h_plane = [&](int k, bool owned_plane, bool z_only) {
        for (int c = tid; c < kAmHx * kAmHy; c += kAmThreads) {
            const int xi = c % kAmHx, yi = c / kAmHx;
            const int x = x0 - 1 + xi, y = y0 - 1 + yi;
            const bool valid = x >= 0 && x < nx && y >= 0 && y < ny;
            const bool own = owned_plane && valid && xi >= 1 && xi <= kAmX && yi >= 1 && yi <= kAmY;
            const long long i = valid ? index(x, y, k) : 0;
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                if (z_only && !(t == 1 || t == 3)) continue;
                const RevTerm rt = rev_of(t >> 1, t & 1);
                const T v = valid ? d_h(A, q, rt, x, y, k, i, own) : T(0);
                if (z_only) sm.dhz[t >> 1][yi][xi] = v;
                else sm.dh[t][yi][xi] = v;
            }
        }
    };

    if (z0 > 0) d_h_plane(z0 - 1, false, true);       // z D values of the plane below the chunk
    __syncthreads();
    const int last = z1 < nz ? z1 : z1 - 1;            // the halo plane z1, when it exists
    for (int k = z0; k <= z1; ++k) {
        const bool compute_e = k <= last;
        const bool owned_plane = k < z1;
        if (compute_e) {
            d_h_plane(k, owned_plane, false);
            __syncthreads();
            // Steps B and C over the tile plus its +x column and +y row.
            for (int c = tid; c < kAmEx * kAmEy; c += kAmThreads) {
                const int xf = c % kAmEx, yf = c / kAmEx;
                if (xf == kAmX && yf == kAmY) continue;           // the corner is never differenced
                const int x = x0 + xf, y = y0 + yf;
                if (x >= nx || y >= ny) {
#pragma unroll
                    for (int t = 0; t < 6; ++t) sm.de[k & 1][t][yf][xf] = T(0);
                    continue;
                }
                const bool own = owned_plane && xf < kAmX && yf < kAmY;
                const long long i = index(x, y, k);
                const int co[3] = {x, y, k};
                const int n3[3] = {nx, ny, nz};
                T e[3];
#pragma unroll
                for (int in = 0; in < 3; ++in) {
                    T contrib = T(0);
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const RevTerm rt = rev_of(in, kk);
                        const int a = rt.axis, cc = co[a], n = n3[a];
                        const int t = 2 * in + kk;
                        if (cc >= 1) {                                  // + D(c - e_a)
                            const T dm = a == 0 ? sm.dh[t][yf + 1][xf] : a == 1 ? sm.dh[t][yf][xf + 1] : sm.dhz[in][yf + 1][xf + 1];
                            contrib = contrib + dm;
                        }
                        if (cc <= n - 2) contrib = contrib - sm.dh[t][yf + 1][xf + 1];   // - D(c)
                        else if (g.pec_on[a] && cc == n - 1) contrib = contrib - sm.dh[t][yf + 1][xf + 1];
                    }
                    e[in] = A.eb[q][in][i] + contrib;
                }
                if (own) {
#pragma unroll
                    for (int in = 0; in < 3; ++in) A.eb[q ^ 1][in][i] = e[in];
                    A.S[0][i] = A.S[0][i] + e[0] * forward_curl<T, 0>(A, slot, x, y, k, i);
                    A.S[1][i] = A.S[1][i] + e[1] * forward_curl<T, 1>(A, slot, x, y, k, i);
                    A.S[2][i] = A.S[2][i] + e[2] * forward_curl<T, 2>(A, slot, x, y, k, i);
                }
#pragma unroll
                for (int t = 0; t < 6; ++t) {
                    const RevTerm rt = rev_of(t >> 1, t & 1);
                    sm.de[k & 1][t][yf][xf] = d_e(A, q, rt, x, y, k, i, e[rt.out], own);
                }
            }
        }
        __syncthreads();
        // Step D: h_bar_new of plane k - 1 on the owned tile.
        if (k > z0) {
            const int km = k - 1;
            const int xf = tid % kAmX, yf = tid / kAmX;
            const int x = x0 + xf, y = y0 + yf;
            if (x < nx && y < ny) {
                const long long i = index(x, y, km);
                const int co[3] = {x, y, km};
                const int n3[3] = {nx, ny, nz};
#pragma unroll
                for (int C = 0; C < 3; ++C) {
                    T contrib = T(0);
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const RevTerm rt = rev_of(C, kk);
                        const int a = rt.axis, cc = co[a], n = n3[a];
                        const int t = 2 * C + kk;
                        if (cc >= 1) contrib = contrib + sm.de[km & 1][t][yf][xf];             // + D(c)
                        if (cc + 1 <= n - 1) {                                                 // - D(c + e_a)
                            const T dp = a == 0 ? sm.de[km & 1][t][yf][xf + 1] : a == 1 ? sm.de[km & 1][t][yf + 1][xf]
                                                                                          : sm.de[k & 1][t][yf][xf];
                            contrib = contrib - dp;
                        }
                    }
                    A.hb[q ^ 1][C][i] = A.hb[q][C][i] + contrib;
                }
            }
        }
        // The z D values of plane k serve plane k + 1 (after every reader of plane k - 1's finished above).
        if (compute_e)
            for (int c = tid; c < kAmHx * kAmHy; c += kAmThreads) {
                const int xi = c % kAmHx, yi = c / kAmHx;
                sm.dhz[0][yi][xi] = sm.dh[1][yi][xi];
                sm.dhz[1][yi][xi] = sm.dh[3][yi][xi];
            }
        __syncthreads();
    }
}

}  // namespace tfd
