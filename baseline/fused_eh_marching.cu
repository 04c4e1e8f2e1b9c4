// The reference's one-pass marching E+H update, restated in CUDA as the comparison kernel for the
// periodic-x/y, z-CPML scenes it admits (reference: torchfdtd/reversible_cuda_fused.py:259-326,
// FusedEHMarching; its operand and CPML expressions: _EHBase._e_code / _h_code, :154-196).
//
// This is NOT the product path. It exists so that the product's TMA z-march kernel can be timed and
// checked bitwise against the reference's own GPU algorithm on the same device. Layout and schedule
// follow the reference:
//   * fields E, H and the inverse permittivity are AoS (nx, ny, nz, 3), z fastest;
//   * a CTA owns TY y-rows and all z (blockDim = (ZB, TY + 2), ZB = nz rounded up to 32; thread
//     rows 0 and TY + 1 are the y halo) and marches along an x chunk [x0, x1);
//   * per plane x it loads H_old(x + 1) of its TY + 2 rows into shared memory, computes E_new(x + 1)
//     once on rows 1 .. TY + 1 (row TY + 1 is the halo the H update's y difference needs; plane x1
//     is the next chunk's first plane, recomputed here and not stored), then H_new(x) on its own rows;
//   * x / y are periodic (rows and planes wrap), z-CPML memories are (nx, ny, hi - lo) per slab,
//     E-family ones double-buffered (old / new), H-family ones updated in place;
//   * curl terms in the reference order, built with --fmad=false like the reference's kernels.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int kMaxSlabs = 2;
constexpr int kMaxSources = 8;

}  // namespace

extern "C" {

// j indexes the two z-derivative terms: E family j = 0 -> Ex (d Hy / dz), j = 1 -> Ey (d Hx / dz);
// H family j = 0 -> Hx (d Ey / dz), j = 1 -> Hy (d Ex / dz).
struct fem_args {
    const float *Eo, *Ho;
    float *En, *Hn;
    const float *inv;
    float cn, cn_imu;
    int nx, ny, nz, zb, rows, chunk;
    int n_eslab, n_hslab;
    int elo[kMaxSlabs], ehi[kMaxSlabs], hlo[kMaxSlabs], hhi[kMaxSlabs];
    const float *eb[kMaxSlabs], *ec[kMaxSlabs], *ek[kMaxSlabs];
    const float *hb[kMaxSlabs], *hc[kMaxSlabs], *hk[kMaxSlabs];
    const float *epo[kMaxSlabs][2];
    float *epn[kMaxSlabs][2];
    float *hpsi[kMaxSlabs][2];
    int n_src;
    int src_comp[kMaxSources], src_lo[kMaxSources][3], src_hi[kMaxSources][3];
    const float *src_w[kMaxSources];
};

}  // extern "C"

namespace {

__device__ __forceinline__ float e_zterm(const fem_args &a, int j, int X, int Y, int Z, bool own, float d) {
    for (int s = 0; s < a.n_eslab; ++s) {
        const int lo = a.elo[s], hi = a.ehi[s];
        if (Z >= lo && Z < hi) {
            const int p = (X * a.ny + Y) * (hi - lo) + (Z - lo);
            const int q = Z - lo;
            const float memory = a.epo[s][j][p] * a.eb[s][q] + a.ec[s][q] * d;
            if (own) a.epn[s][j][p] = memory;
            d = d * a.ek[s][q] + memory;
        }
    }
    return d;
}

__device__ __forceinline__ float h_zterm(const fem_args &a, int j, int X, int Y, int Z, float d) {
    for (int s = 0; s < a.n_hslab; ++s) {
        const int lo = a.hlo[s], hi = a.hhi[s];
        if (Z >= lo && Z < hi) {
            const int p = (X * a.ny + Y) * (hi - lo) + (Z - lo);
            const int q = Z - lo;
            const float memory = a.hpsi[s][j][p] * a.hb[s][q] + a.hc[s][q] * d;
            a.hpsi[s][j][p] = memory;
            d = d * a.hk[s][q] + memory;
        }
    }
    return d;
}

__global__ void k_fused_eh_marching(const __grid_constant__ fem_args a, int n) {
    extern __shared__ float smem[];
    const int ZB = a.zb, R = a.rows + 2, P = R * ZB * 3;
    float *SH[2] = {smem, smem + P};
    float *SE[2] = {smem + 2 * P, smem + 3 * P};
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int z = threadIdx.x, ty = threadIdx.y;
    const int y0 = blockIdx.x * a.rows, nrows = min(a.rows, ny - y0);
    const int x0 = blockIdx.y * a.chunk, x1 = min(x0 + a.chunk, nx);
    if (x0 >= x1) return;
    const int y = ((y0 - 1 + ty) % ny + ny) % ny;
    const bool zin = z < nz;
    const bool hrow = ty <= nrows + 1;
    const bool erow = ty >= 1 && ty <= nrows + 1;
    const bool own = ty >= 1 && ty <= nrows;
    auto s = [&](int row, int zz, int c) { return (row * ZB + zz) * 3 + c; };

    int cur = 0;
    {
        const int xm = x0 == 0 ? nx - 1 : x0 - 1;
        if (hrow && zin) {
            const int j = (xm * ny + y) * nz + z;
            for (int c = 0; c < 3; ++c) SH[0][s(ty, z, c)] = a.Ho[3 * j + c];
        }
    }
    for (int x = x0 - 1; x < x1; ++x) {
        const int nxt = cur ^ 1;
        const int xe = x + 1 == nx ? 0 : x + 1;
        float *Hn_ = SH[nxt], *Hc_ = SH[cur], *En_ = SE[nxt], *Ec_ = SE[cur];
        if (hrow && zin) {
            const int j = (xe * ny + y) * nz + z;
            for (int c = 0; c < 3; ++c) Hn_[s(ty, z, c)] = a.Ho[3 * j + c];
        }
        __syncthreads();
        if (erow && zin) {
            // E_new(xe, y, z). H operands: the cell (Hn_ row ty), -x (Hc_: plane x), -y (row ty - 1), -z.
            const int j = (xe * ny + y) * nz + z;
            const bool eown = own && x + 1 < x1;
            float e[3];
            {   // Ex: (axis 1, Hz, +), (axis 2, Hy, -)
                float cc = 0;
                float d = Hn_[s(ty, z, 2)] - Hn_[s(ty - 1, z, 2)];
                cc += d;
                d = 0;
                if (z > 0) d = e_zterm(a, 0, xe, y, z, eown, Hn_[s(ty, z, 1)] - Hn_[s(ty, z - 1, 1)]);
                cc += -d;
                e[0] = a.Eo[3 * j + 0] + (a.cn * a.inv[3 * j + 0]) * cc;
            }
            {   // Ey: (axis 0, Hz, -), (axis 2, Hx, +)
                float cc = 0;
                float d = Hn_[s(ty, z, 2)] - Hc_[s(ty, z, 2)];
                cc += -d;
                d = 0;
                if (z > 0) d = e_zterm(a, 1, xe, y, z, eown, Hn_[s(ty, z, 0)] - Hn_[s(ty, z - 1, 0)]);
                cc += d;
                e[1] = a.Eo[3 * j + 1] + (a.cn * a.inv[3 * j + 1]) * cc;
            }
            {   // Ez: (axis 0, Hy, +), (axis 1, Hx, -)
                float cc = 0;
                float d = Hn_[s(ty, z, 1)] - Hc_[s(ty, z, 1)];
                cc += d;
                d = Hn_[s(ty, z, 0)] - Hn_[s(ty - 1, z, 0)];
                cc += -d;
                e[2] = a.Eo[3 * j + 2] + (a.cn * a.inv[3 * j + 2]) * cc;
            }
            for (int q = 0; q < a.n_src; ++q) {
                const int c = a.src_comp[q];
                if (xe >= a.src_lo[q][0] && xe < a.src_hi[q][0] && y >= a.src_lo[q][1] && y < a.src_hi[q][1] &&
                    z >= a.src_lo[q][2] && z < a.src_hi[q][2])
                    e[c] = e[c] + a.src_w[q][n];
            }
            for (int c = 0; c < 3; ++c) En_[s(ty, z, c)] = e[c];
            if (eown)
                for (int c = 0; c < 3; ++c) a.En[3 * j + c] = e[c];
        }
        __syncthreads();
        if (x >= x0 && own && zin) {
            // H_new(x, y, z). E_new operands: the cell (Ec_), +x (En_: plane x + 1), +y (row ty + 1), +z.
            const int i = (x * ny + y) * nz + z;
            float c0 = 0, c1 = 0, c2 = 0, d;
            d = En_[s(ty, z, 2)] - Ec_[s(ty, z, 2)];         // (axis 0, Ez, out 1, -)
            c1 += -d;
            d = En_[s(ty, z, 1)] - Ec_[s(ty, z, 1)];         // (axis 0, Ey, out 2, +)
            c2 += d;
            d = Ec_[s(ty + 1, z, 2)] - Ec_[s(ty, z, 2)];     // (axis 1, Ez, out 0, +)
            c0 += d;
            d = Ec_[s(ty + 1, z, 0)] - Ec_[s(ty, z, 0)];     // (axis 1, Ex, out 2, -)
            c2 += -d;
            d = 0;                                           // (axis 2, Ey, out 0, -)
            if (z < nz - 1) d = h_zterm(a, 0, x, y, z, Ec_[s(ty, z + 1, 1)] - Ec_[s(ty, z, 1)]);
            c0 += -d;
            d = 0;                                           // (axis 2, Ex, out 1, +)
            if (z < nz - 1) d = h_zterm(a, 1, x, y, z, Ec_[s(ty, z + 1, 0)] - Ec_[s(ty, z, 0)]);
            c1 += d;
            a.Hn[3 * i + 0] = Hc_[s(ty, z, 0)] - a.cn_imu * c0;
            a.Hn[3 * i + 1] = Hc_[s(ty, z, 1)] - a.cn_imu * c1;
            a.Hn[3 * i + 2] = Hc_[s(ty, z, 2)] - a.cn_imu * c2;
        }
        __syncthreads();
        cur = nxt;
    }
}

}  // namespace

extern "C" {

int fem_args_size(void) { return (int)sizeof(fem_args); }

// Shared-memory bytes of one CTA: H and E, two planes each, (rows + 2) x zb x 3 floats.
int fem_smem_bytes(int rows, int zb) { return 4 * (rows + 2) * zb * 3 * (int)sizeof(float); }

// One step: grid (ceil(ny / rows), ceil(nx / chunk)), block (zb, rows + 2). Returns a cudaError_t.
int fem_step(const fem_args *args, int n, void *stream) {
    const int yblocks = (args->ny + args->rows - 1) / args->rows;
    const int xchunks = (args->nx + args->chunk - 1) / args->chunk;
    const int smem = fem_smem_bytes(args->rows, args->zb);
    cudaError_t e = cudaFuncSetAttribute(k_fused_eh_marching, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return (int)e;
    k_fused_eh_marching<<<dim3(yblocks, xchunks), dim3(args->zb, args->rows + 2), smem, (cudaStream_t)stream>>>(*args, n);
    return (int)cudaGetLastError();
}

}  // extern "C"
