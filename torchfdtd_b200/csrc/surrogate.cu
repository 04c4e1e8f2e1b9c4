// Learned surrogate: a small convolutional neural operator (8 conv layers, 64 channels) mapping a 2D design
// density to its complex transmission spectrum, trained and evaluated by these kernels.
//
// Numerics: BF16 operands, FP32 accumulation (tcgen05 kind::f16 into tensor memory by default, or warp-level
// mma.sync m16n8k16 as the selectable legacy path; bf16 x bf16 -> f32), FP32
// master weights, bias, head (linear on the flattened last feature map), loss and Adam state. Activations are NHWC bf16 with C = 16 (the packed input:
// density, x, y, 1, zeros) or C = 64, so one pixel is one or four 16-byte vectors.
//
// Each conv is 3x3, zero padding 1, stride 1 or 2, Cout = 64, followed by GELU (tanh form):
//   forward          z[p, co] = bias[co] + sum_{tap, ci} x[in(p, tap), ci] w[tap, co, ci];  a = gelu(z)
//   backward (data)  dx[q, ci] = sum_{tap, co} dz[out(q, tap), co] w[tap, co, ci]  (then * gelu'(z_prev))
//   backward (weight) dw[tap, co, ci] = sum_p dz[p, co] x[in(p, tap), ci]; dbias[co] = sum_p dz[p, co]
// All three are implicit GEMMs. The tcgen05 kernels (k_conv_shift for the stride-1 layers and the stride-2 input
// gradient, k_conv_tc for the other forward and backward-data cases, k_wgrad_tc for backward weight) stage cp.async
// loads in shared memory for MMAs issued by one thread into tensor memory. The
// mma.sync kernels work on 64 x 64 tiles: 4 warps, each 16 rows x 64 columns of m16n8k16 MMAs, with the operands
// staged in shared memory (row-major A, column-major B, both padded to 144-byte rows so the fragment loads are
// bank-conflict free).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/tfdtd.h"

namespace tfd {
void set_error(const std::string &msg);
}

namespace {

using bf16 = __nv_bfloat16;
constexpr int kCo = 64;
constexpr int kTile = 64;
constexpr int kThreads = 128;

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

// acc[nt] += A[16 rows of this warp][K] * B[K][8 nt .. 8 nt + 7]; A row-major with leading dimension lda,
// B stored as [n][k] with leading dimension ldb (k contiguous).
template <int NT>
__device__ __forceinline__ void warp_gemm(float (&acc)[NT][4], const bf16 *A, int lda, const bf16 *B, int ldb, int K, int lane) {
    const int g = lane >> 2, t = lane & 3;
    for (int kk = 0; kk < K; kk += 16) {
        const uint32_t a0 = ld32(A + g * lda + kk + 2 * t);
        const uint32_t a1 = ld32(A + (g + 8) * lda + kk + 2 * t);
        const uint32_t a2 = ld32(A + g * lda + kk + 2 * t + 8);
        const uint32_t a3 = ld32(A + (g + 8) * lda + kk + 2 * t + 8);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const uint32_t b0 = ld32(B + (nt * 8 + g) * ldb + kk + 2 * t);
            const uint32_t b1 = ld32(B + (nt * 8 + g) * ldb + kk + 2 * t + 8);
            mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
        }
    }
}

// GELU (tanh form) with the hardware tanh (tanh.approx.f32, one MUFU operation, relative error about 2^-11): the
// activations are rounded to BF16 (2^-8) right after, and the epilogues of the conv kernels are bound by this
// arithmetic, not by their memory traffic.
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu(float z) {
    const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
    return 0.5f * z * (1.0f + tanh_hw(u));
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
    const float th = tanh_hw(u);
    return 0.5f * (1.0f + th) + 0.5f * z * (1.0f - th * th) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * z * z);
}

// ---- forward ------------------------------------------------------------------------------------------
template <int CI>
__global__ void __launch_bounds__(kThreads) k_conv_fwd(const bf16 *__restrict__ X, const bf16 *__restrict__ Wt,
                                                      const float *__restrict__ bias, bf16 *__restrict__ Z, bf16 *__restrict__ Aout,
                                                      int N, int H, int W, int Ho, int Wo, int stride) {
    constexpr int LD = CI + 8;
    __shared__ __align__(16) bf16 As[kTile * LD];
    __shared__ __align__(16) bf16 Bs[kCo * LD];
    const long long P = (long long)N * Ho * Wo;
    const long long p0 = (long long)blockIdx.x * kTile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float acc[8][4] = {};
    for (int tap = 0; tap < 9; ++tap) {
        const int ky = tap / 3, kx = tap % 3;
        for (int e = threadIdx.x; e < kTile * CI / 8; e += kThreads) {
            const int row = e / (CI / 8), ch = (e % (CI / 8)) * 8;
            const long long p = p0 + row;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < P) {
                const int n = (int)(p / ((long long)Ho * Wo));
                const int rem = (int)(p % ((long long)Ho * Wo));
                const int iy = (rem / Wo) * stride + ky - 1, ix = (rem % Wo) * stride + kx - 1;
                if (iy >= 0 && iy < H && ix >= 0 && ix < W)
                    v = *reinterpret_cast<const uint4 *>(X + (((long long)n * H + iy) * W + ix) * CI + ch);
            }
            *reinterpret_cast<uint4 *>(As + row * LD + ch) = v;
        }
        for (int e = threadIdx.x; e < kCo * CI / 8; e += kThreads) {
            const int co = e / (CI / 8), ch = (e % (CI / 8)) * 8;
            *reinterpret_cast<uint4 *>(Bs + co * LD + ch) = *reinterpret_cast<const uint4 *>(Wt + ((long long)tap * kCo + co) * CI + ch);
        }
        __syncthreads();
        warp_gemm<8>(acc, As + warp * 16 * LD, LD, Bs, LD, CI, lane);
        __syncthreads();
    }
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const long long p = p0 + warp * 16 + g + 8 * h;
            if (p >= P) continue;
            const int co = nt * 8 + 2 * t;
            const float z0 = acc[nt][2 * h] + bias[co], z1 = acc[nt][2 * h + 1] + bias[co + 1];
            *reinterpret_cast<__nv_bfloat162 *>(Z + p * kCo + co) = __floats2bfloat162_rn(z0, z1);
            *reinterpret_cast<__nv_bfloat162 *>(Aout + p * kCo + co) = __floats2bfloat162_rn(gelu(z0), gelu(z1));
        }
}

// ---- backward, data -------------------------------------------------------------------------------------
// Rows: input pixels q; columns: input channels; K: (tap, co). Wt_t is the weight stored [tap][ci][co].
// With Zprev, writes dz_prev = bf16(dx * gelu'(z_prev)); otherwise writes dx in FP32.
template <int CI>
__global__ void __launch_bounds__(kThreads) k_conv_dgrad(const bf16 *__restrict__ dZ, const bf16 *__restrict__ Wt_t,
                                                        const bf16 *__restrict__ Zprev, void *__restrict__ out, int N, int H, int W,
                                                        int Ho, int Wo, int stride) {
    constexpr int LD = kCo + 8;
    constexpr int NT = CI / 8;
    __shared__ __align__(16) bf16 As[kTile * LD];
    __shared__ __align__(16) bf16 Bs[CI * LD];
    const long long Q = (long long)N * H * W;
    const long long q0 = (long long)blockIdx.x * kTile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float acc[NT][4] = {};
    for (int tap = 0; tap < 9; ++tap) {
        const int ky = tap / 3, kx = tap % 3;
        for (int e = threadIdx.x; e < kTile * kCo / 8; e += kThreads) {
            const int row = e / (kCo / 8), ch = (e % (kCo / 8)) * 8;
            const long long q = q0 + row;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (q < Q) {
                const int n = (int)(q / ((long long)H * W));
                const int rem = (int)(q % ((long long)H * W));
                const int ty = rem / W + 1 - ky, tx = rem % W + 1 - kx;      // = o * stride
                if (ty >= 0 && tx >= 0 && ty % stride == 0 && tx % stride == 0) {
                    const int oy = ty / stride, ox = tx / stride;
                    if (oy < Ho && ox < Wo) v = *reinterpret_cast<const uint4 *>(dZ + (((long long)n * Ho + oy) * Wo + ox) * kCo + ch);
                }
            }
            *reinterpret_cast<uint4 *>(As + row * LD + ch) = v;
        }
        for (int e = threadIdx.x; e < CI * kCo / 8; e += kThreads) {
            const int ci = e / (kCo / 8), ch = (e % (kCo / 8)) * 8;
            *reinterpret_cast<uint4 *>(Bs + ci * LD + ch) = *reinterpret_cast<const uint4 *>(Wt_t + ((long long)tap * CI + ci) * kCo + ch);
        }
        __syncthreads();
        warp_gemm<NT>(acc, As + warp * 16 * LD, LD, Bs, LD, kCo, lane);
        __syncthreads();
    }
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const long long q = q0 + warp * 16 + g + 8 * h;
            if (q >= Q) continue;
            const int ci = nt * 8 + 2 * t;
            float d0 = acc[nt][2 * h], d1 = acc[nt][2 * h + 1];
            if (Zprev) {
                const __nv_bfloat162 z = *reinterpret_cast<const __nv_bfloat162 *>(Zprev + q * CI + ci);
                d0 *= gelu_grad(__bfloat162float(z.x));
                d1 *= gelu_grad(__bfloat162float(z.y));
                *reinterpret_cast<__nv_bfloat162 *>((bf16 *)out + q * CI + ci) = __floats2bfloat162_rn(d0, d1);
            } else {
                float *o = (float *)out + q * CI + ci;
                o[0] = d0;
                o[1] = d1;
            }
        }
}

// ---- backward, weight -----------------------------------------------------------------------------------
// One CTA: one tap, one chunk of output pixels; rows co, columns ci, K = pixels. Writes its partial sums
// (and, for the centre tap, the partial bias gradient); k_reduce_partials adds the chunks in a fixed order.
template <int CI>
__global__ void __launch_bounds__(kThreads) k_conv_wgrad(const bf16 *__restrict__ dZ, const bf16 *__restrict__ X,
                                                        float *__restrict__ partial, float *__restrict__ partial_bias, int N, int H,
                                                        int W, int Ho, int Wo, int stride, int chunk) {
    constexpr int LD = kTile + 8;
    constexpr int NT = CI / 8;
    __shared__ __align__(16) bf16 As[kCo * LD];     // [co][pixel]
    __shared__ __align__(16) bf16 Bs[CI * LD];      // [ci][pixel]
    const int tap = blockIdx.y, ky = tap / 3, kx = tap % 3;
    const long long P = (long long)N * Ho * Wo;
    const long long begin = (long long)blockIdx.x * chunk;
    const long long end = begin + chunk < P ? begin + chunk : P;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float acc[NT][4] = {};
    float bias_acc = 0.f;                              // thread c < 64 sums column c of dz (centre tap)
    for (long long p0 = begin; p0 < end; p0 += kTile) {
        for (int e = threadIdx.x; e < kTile * kCo / 8; e += kThreads) {
            const int pix = e / (kCo / 8), ch = (e % (kCo / 8)) * 8;
            const long long p = p0 + pix;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < end) v = *reinterpret_cast<const uint4 *>(dZ + p * kCo + ch);
            const bf16 *s = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
            for (int j = 0; j < 8; ++j) As[(ch + j) * LD + pix] = s[j];
        }
        for (int e = threadIdx.x; e < kTile * CI / 8; e += kThreads) {
            const int pix = e / (CI / 8), ch = (e % (CI / 8)) * 8;
            const long long p = p0 + pix;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (p < end) {
                const int n = (int)(p / ((long long)Ho * Wo));
                const int rem = (int)(p % ((long long)Ho * Wo));
                const int iy = (rem / Wo) * stride + ky - 1, ix = (rem % Wo) * stride + kx - 1;
                if (iy >= 0 && iy < H && ix >= 0 && ix < W)
                    v = *reinterpret_cast<const uint4 *>(X + (((long long)n * H + iy) * W + ix) * CI + ch);
            }
            const bf16 *s = reinterpret_cast<const bf16 *>(&v);
#pragma unroll
            for (int j = 0; j < 8; ++j) Bs[(ch + j) * LD + pix] = s[j];
        }
        __syncthreads();
        if (tap == 4 && threadIdx.x < kCo)
            for (int pix = 0; pix < kTile; ++pix) bias_acc += __bfloat162float(As[threadIdx.x * LD + pix]);
        warp_gemm<NT>(acc, As + warp * 16 * LD, LD, Bs, LD, kTile, lane);
        __syncthreads();
    }
    const int g = lane >> 2, t = lane & 3;
    float *out = partial + ((long long)blockIdx.x * 9 + tap) * kCo * CI;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int co = warp * 16 + g + 8 * h, ci = nt * 8 + 2 * t;
            out[co * CI + ci] = acc[nt][2 * h];
            out[co * CI + ci + 1] = acc[nt][2 * h + 1];
        }
    if (tap == 4 && threadIdx.x < kCo) partial_bias[(long long)blockIdx.x * kCo + threadIdx.x] = bias_acc;
}

// out[e] = the sum over chunks c of partial[c * len + e]; elements past the weights reduce the bias partials
// (len_b per chunk) the same way. A block of 256 threads takes 64 elements: thread group g (64 threads) sums chunks
// g, g + 4, g + 8, ... in order with eight loads in flight, and the four group sums are added in the order 0, 1, 2,
// 3, so the result does not depend on scheduling.
__global__ void __launch_bounds__(256) k_reduce_partials(const float *__restrict__ partial, int chunks, long long len,
                                                         float *__restrict__ out, const float *__restrict__ partial_b, int len_b,
                                                         float *__restrict__ out_b) {
    __shared__ float part[4][64];
    const int g = threadIdx.x >> 6, l = threadIdx.x & 63;
    const long long e = blockIdx.x * 64LL + l;
    const float *src = nullptr;
    long long stride = 0;
    float *dst = nullptr;
    if (e < len) {
        src = partial + e, stride = len, dst = out + e;
    } else if (e < len + len_b) {
        src = partial_b + (e - len), stride = len_b, dst = out_b + (e - len);
    }
    float s = 0.f;
    if (src) {
        int c = g;
        for (; c + 28 < chunks; c += 32) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = src[(long long)(c + 4 * i) * stride];
#pragma unroll
            for (int i = 0; i < 8; ++i) s += v[i];
        }
        for (; c < chunks; c += 4) s += src[(long long)c * stride];
    }
    part[g][l] = s;
    __syncthreads();
    if (g == 0 && dst) *dst = ((part[0][l] + part[1][l]) + part[2][l]) + part[3][l];
}

// ---- input packing, head, loss, optimiser ---------------------------------------------------------------
// x0[n, y, x, :] = (2 rho - 1, xc, yc, 1, 0 ...) with coordinates in [-1, 1]; two 16-byte stores per pixel.
__global__ void k_pack_input(const float *__restrict__ rho, bf16 *__restrict__ x0, int total, int H, int W) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
        const int rem = p % (H * W);
        const int y = rem / W, x = rem % W;
        __align__(16) bf16 v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16_rn(0.f);
        v[0] = __float2bfloat16_rn(2.f * rho[p] - 1.f);
        v[1] = __float2bfloat16_rn(W > 1 ? -1.f + 2.f * x / (W - 1) : 0.f);
        v[2] = __float2bfloat16_rn(H > 1 ? -1.f + 2.f * y / (H - 1) : 0.f);
        v[3] = __float2bfloat16_rn(1.f);
        uint4 *o = reinterpret_cast<uint4 *>(x0 + (long long)p * 16);
        o[0] = reinterpret_cast<const uint4 *>(v)[0];
        o[1] = reinterpret_cast<const uint4 *>(v)[1];
    }
}

// Linear head on the flattened last feature map: out[n, j] = bh[j] + sum_f wh[j, f] a[n, f], f = p * 64 + c
// (the positions stay distinct: the scene is not translation invariant). One block per sample, one warp per
// output at a time, warp-shuffle reductions.
__global__ void k_head_fwd(const bf16 *__restrict__ a, const float *__restrict__ wh, const float *__restrict__ bh,
                           float *__restrict__ out, int F, int K) {
    const int n = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const bf16 *an = a + (long long)n * F;
    for (int j = warp; j < K; j += warps) {
        const float *w = wh + (long long)j * F;
        float s = 0.f;
        for (int f = lane; f < F; f += 32) s += w[f] * __bfloat162float(an[f]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[n * K + j] = bh[j] + s;
    }
}

// loss = mean (out - y)^2; dout = 2 (out - y) / (N K). Single block.
__global__ void k_mse(const float *__restrict__ out, const float *__restrict__ y, float *__restrict__ dout, float *__restrict__ loss,
                      int total) {
    __shared__ float red[256];
    float s = 0.f;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const float d = out[e] - y[e];
        s += d * d;
        if (dout) dout[e] = 2.f * d / total;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] / total;
}

// Head backward: dwh[j, f] = sum_n dout[n, j] a[n, f], dbh[j] = sum_n dout[n, j] (deterministic), and
// dz_last[n, f] = (sum_j dout[n, j] wh[j, f]) * gelu'(z_last[n, f]).
__global__ void k_head_bwd_params(const float *__restrict__ dout, const bf16 *__restrict__ a, float *__restrict__ dwh,
                                  float *__restrict__ dbh, int N, int F, int K) {
    const long long total = (long long)K * F;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / F);
        const long long f = e % F;
        float s = 0.f;
        for (int n = 0; n < N; ++n) s += dout[n * K + j] * __bfloat162float(a[(long long)n * F + f]);
        dwh[e] = s;
    }
    if (blockIdx.x == 0)
        for (int j = threadIdx.x; j < K; j += blockDim.x) {
            float s = 0.f;
            for (int n = 0; n < N; ++n) s += dout[n * K + j];
            dbh[j] = s;
        }
}

__global__ void k_head_bwd_data(const float *__restrict__ dout, const float *__restrict__ wh, const bf16 *__restrict__ z,
                                bf16 *__restrict__ dz, int N, int F, int K) {
    const long long total = (long long)N * F;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int n = (int)(e / F);
        const long long f = e % F;
        float s = 0.f;
        for (int j = 0; j < K; ++j) s += dout[n * K + j] * wh[(long long)j * F + f];
        dz[e] = __float2bfloat16_rn(s * gelu_grad(__bfloat162float(z[e])));
    }
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v, long long n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const float gr = g[e];
        const float mm = b1 * m[e] + (1.f - b1) * gr;
        const float vv = b2 * v[e] + (1.f - b2) * gr * gr;
        m[e] = mm;
        v[e] = vv;
        p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

// w [9][64][ci] fp32 -> w_bf16 [9][64][ci] and wt_bf16 [9][ci][64].
__global__ void k_cast_weights(const float *__restrict__ w, bf16 *__restrict__ wb, bf16 *__restrict__ wt, int ci) {
    const int total = 9 * kCo * ci;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int tap = e / (kCo * ci), rem = e % (kCo * ci), co = rem / ci, c = rem % ci;
        const bf16 v = __float2bfloat16_rn(w[e]);
        wb[e] = v;
        wt[(tap * ci + c) * kCo + co] = v;
    }
}

// ---- tcgen05 path: 5th-generation tensor cores, accumulators in tensor memory -------------------------
// One CTA = 128 output rows (pixels) x N columns. Per tap, the 128 threads gather their row's K = 16..64
// input channels (16-byte vectors) and the tap's weights into a shared-memory stage laid out K-major without
// swizzle (8-row x 16-byte core matrices: rows 16 bytes apart, 8-row groups 128 bytes apart (SBO), 16-byte
// K chunks one 128- or N-row block apart (LBO)); one thread issues the tap's tcgen05.mma instructions
// (M = 128, K = 16 each) into the tensor-memory accumulator and commits them to the stage's mbarrier, while
// the CTA gathers the next tap into the other stage. The epilogue reads the accumulator with tcgen05.ld
// (warp w: tensor-memory lanes 32w..32w+31 = its 32 rows). Every wait is bounded: on a timeout the kernel
// records g_sg_status, waits (bounded) for its own MMAs, frees its tensor memory and returns.
__device__ int g_sg_status;

__device__ __forceinline__ uint32_t sh_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;                    // descriptor version of sm_100; no swizzle, base offset 0
    return d;
}

// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(sh_addr(bar)) : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sh_addr(bar)) : "memory");
}

__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t addr = sh_addr(bar);
    for (int it = 0; it < 2000; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(addr), "r"(parity), "r"(1000000u) : "memory");
        if (done) return true;
    }
    return false;
}

template <int COLS>
__device__ __forceinline__ void tmem_alloc(uint32_t *slot) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sh_addr(slot)), "r"(COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

template <int COLS>
__device__ __forceinline__ void tmem_free(uint32_t tmem) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS) : "memory");
}

// 32 lanes x 16 columns of 32-bit accumulators (one warp, its own lane quarter), then wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 32 columns in one load and one wait.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,"
        "%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory bytes of one tcgen05 conv CTA: three A stages (128 x K), three B stages (N x K), barriers, slot.
constexpr int kStages = 3;
__host__ __device__ constexpr int tc_smem(int K, int N) { return kStages * (K * 128 * 2) + kStages * (K * N * 2) + 64; }

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sh_addr(dst)), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// MODE 0 forward (K = CI input channels per tap, N = 64 output channels);
// MODE 1 backward data (K = 64 output channels per tap, N = CI input channels).
// The gathers of tap t+2 (cp.async, zero-filled outside the image) are in flight while the tensor cores
// work on tap t; a stage is refilled once the commit of the MMAs that read it has arrived.
// Backward data with stride 2 (cls != nullptr): input pixel (y, x) takes dz only through the taps with
// ky = y + 1 and kx = x + 1 (mod 2), one tap for (even, even), two for (even, odd) and (odd, even), four for
// (odd, odd). The rows are grouped by that parity class (CTAs [cls[c], cls[c + 1]) take class c = 2 (y & 1) +
// (x & 1), rows in (n, y / 2, x / 2) order) and a CTA runs only its class's taps.
template <int MODE, int CI>
__global__ void __launch_bounds__(128) k_conv_tc(const bf16 *__restrict__ src, const bf16 *__restrict__ wsrc,
                                                const float *__restrict__ bias, const bf16 *__restrict__ zprev, bf16 *__restrict__ out0,
                                                void *__restrict__ out1, int N, int H, int W, int Ho, int Wo, int stride,
                                                const int4 cls = make_int4(0, 0, 0, 0)) {
    constexpr int K = MODE == 0 ? CI : kCo;              // reduction channels per tap
    constexpr int NC = MODE == 0 ? kCo : CI;             // output columns
    constexpr int KC = K / 8;                            // 16-byte K chunks per tap
    constexpr int A_BYTES = KC * 128 * 16, B_BYTES = KC * NC * 16;
    constexpr int COLS = NC < 32 ? 32 : NC;
    constexpr uint32_t IDESC = umma_idesc(128, NC);
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *As = smem, *Bs = smem + kStages * A_BYTES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(Bs + kStages * B_BYTES);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + kStages);
    const int tid = threadIdx.x, warp = tid >> 5;
    // Output rows: MODE 0 output pixels (n, oy, ox); MODE 1 input pixels (n, y, x).
    const bool classes = MODE == 1 && cls.w > 0;
    int cy = 0, cx = 0, blk = blockIdx.x;
    if (classes) {
        const int c = (int)blockIdx.x >= cls.z ? 3 : (int)blockIdx.x >= cls.y ? 2 : (int)blockIdx.x >= cls.x ? 1 : 0;
        blk -= c == 0 ? 0 : c == 1 ? cls.x : c == 2 ? cls.y : cls.z;
        cy = c >> 1, cx = c & 1;
    }
    // Rows of this CTA's class: y = 2 u + cy, x = 2 v + cx (all pixels with one class when there are no classes).
    const int RH = MODE == 0 ? Ho : classes ? (H - cy + 1) / 2 : H, RW = MODE == 0 ? Wo : classes ? (W - cx + 1) / 2 : W;
    const long long rows = (long long)N * RH * RW;
    const long long crow = (long long)blk * 128 + tid;
    const bool live = crow < rows;
    const int n = live ? (int)(crow / ((long long)RH * RW)) : 0;
    const int rem = live ? (int)(crow % ((long long)RH * RW)) : 0;
    const int ry = classes ? 2 * (rem / RW) + cy : rem / RW, rx = classes ? 2 * (rem % RW) + cx : rem % RW;
    const long long row = classes ? ((long long)n * H + ry) * W + rx : crow;     // the pixel this thread writes
    // Taps of this CTA: all 9, or the class's 1, 2 or 4 (tap index i -> (ky, kx)).
    const int nkx = classes ? (cx ? 2 : 1) : 3;
    const int taps = classes ? (cy ? 2 : 1) * nkx : 9;
    auto tap_of = [&](int i) {
        if (!classes) return i;
        const int ky = cy ? 2 * (i / nkx) : 1, kx = cx ? 2 * (i % nkx) : 1;
        return ky * 3 + kx;
    };
    if (warp == 0) tmem_alloc<COLS>(slot);
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) bar_init(&bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;

    // Gathers of one tap into its stage: this thread's row (K channels of the tap's neighbour, zero outside
    // the image or off the stride grid) and its share of the tap's weights ([K chunk][column][16 bytes]).
    auto issue = [&](int i) {
        const int s = i % kStages, tap = tap_of(i), ky = tap / 3, kx = tap % 3;
        const bf16 *a = nullptr;
        if (live) {
            if (MODE == 0) {
                const int iy = ry * stride + ky - 1, ix = rx * stride + kx - 1;
                if (iy >= 0 && iy < H && ix >= 0 && ix < W) a = src + (((long long)n * H + iy) * W + ix) * CI;
            } else {
                const int ty = ry + 1 - ky, tx = rx + 1 - kx;
                if (ty >= 0 && tx >= 0 && ty % stride == 0 && tx % stride == 0 && ty / stride < Ho && tx / stride < Wo)
                    a = src + (((long long)n * Ho + ty / stride) * Wo + tx / stride) * kCo;
            }
        }
        unsigned char *as = As + s * A_BYTES;
#pragma unroll
        for (int kc = 0; kc < KC; ++kc) cp_async16(as + (kc * 128 + tid) * 16, a ? a + kc * 8 : src, a ? 16 : 0);
        unsigned char *bs = Bs + s * B_BYTES;
        for (int e = tid; e < NC * KC; e += 128) {
            const int col = e / KC, kc = e % KC;
            cp_async16(bs + (kc * NC + col) * 16, wsrc + ((long long)tap * NC + col) * K + kc * 8, 16);
        }
        cp_async_commit();
    };

    bool ok = true;
    int issued = 0;                                      // taps whose MMAs were committed
    issue(0);
    if (taps > 1) issue(1);
    else cp_async_commit();
    for (int tap = 0; tap < taps; ++tap) {
        const int s = tap % kStages;
        if (tap + 2 < taps) {
            // Stage (tap + 2) % 3 was last read by the MMAs of tap - 1.
            if (tap >= 1 && !bar_wait(&bar[(tap - 1) % kStages], ((tap - 1) / kStages) & 1)) ok = false;
            if (__syncthreads_or(!ok)) break;
            issue(tap + 2);
        } else {
            cp_async_commit();                           // empty group: keeps "tap's group is 2 groups back"
        }
        cp_async_wait<2>();
        proxy_fence();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const unsigned char *as = As + s * A_BYTES, *bs = Bs + s * B_BYTES;
#pragma unroll
            for (int kk = 0; kk < K / 16; ++kk) {
                const uint64_t ad = umma_desc(sh_addr(as) + kk * 2 * (128 * 16), 128 * 16, 128);
                const uint64_t bd = umma_desc(sh_addr(bs) + kk * 2 * (NC * 16), NC * 16, 128);
                umma_bf16(tmem, ad, bd, IDESC, (tap | kk) != 0);
            }
            umma_commit(&bar[s]);
        }
        issued = tap + 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // Wait for the last committed tap (its commit covers every earlier MMA of this thread).
    if (issued > 0 && !bar_wait(&bar[(issued - 1) % kStages], ((issued - 1) / kStages) & 1)) ok = false;
    tc_fence_after();
    if (__syncthreads_or(!ok) || issued < taps) {
        if (tid == 0) atomicExch(&g_sg_status, 1);
    } else {
#pragma unroll
        for (int c0 = 0; c0 < NC; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
            if (!live) continue;
            if (MODE == 0) {
                __align__(16) bf16 zb[16], ab[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const float z = v[i] + bias[c0 + i];
                    zb[i] = __float2bfloat16_rn(z);
                    ab[i] = __float2bfloat16_rn(gelu(z));
                }
                uint4 *zd = reinterpret_cast<uint4 *>(out0 + row * kCo + c0);
                uint4 *adst = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(out1) + row * kCo + c0);
                zd[0] = reinterpret_cast<const uint4 *>(zb)[0];
                zd[1] = reinterpret_cast<const uint4 *>(zb)[1];
                adst[0] = reinterpret_cast<const uint4 *>(ab)[0];
                adst[1] = reinterpret_cast<const uint4 *>(ab)[1];
            } else if (zprev) {
                __align__(16) bf16 db[16];
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    db[i] = __float2bfloat16_rn(v[i] * gelu_grad(__bfloat162float(zprev[row * CI + c0 + i])));
                uint4 *dd = reinterpret_cast<uint4 *>(out0 + row * CI + c0);
                dd[0] = reinterpret_cast<const uint4 *>(db)[0];
                dd[1] = reinterpret_cast<const uint4 *>(db)[1];
            } else {
                float *o = reinterpret_cast<float *>(out1) + row * CI + c0;
#pragma unroll
                for (int i = 0; i < 16; ++i) o[i] = v[i];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_free<COLS>(tmem);
}

// ---- tcgen05 backward weight ----------------------------------------------------------------------------
// dW^T as one GEMM per chunk of output pixels: rows (tap, ci) -- all 9 taps stacked, 9 * CI rows, plus one row
// of ones whose product with dz is the bias gradient -- times columns co, K = pixels. Both operands are staged
// MN-major (no swizzle): for each 8-element chunk of rows (or of co), the stage's 32 pixels lie 16 bytes apart
// (8-pixel core matrices 128 bytes apart = LBO, row chunks KB * 16 bytes apart = SBO), so a pixel's gathered
// 16-byte vector lands whole. The rows are split into MT tiles of M = 128, each with its own 64-column
// accumulator in tensor memory; the padding rows past the ones row stay zero. Three stages: the cp.async gathers
// of block b+2 are in flight while the tensor cores work on block b. Bounded waits as in k_conv_tc.
constexpr int kWgKB = 32;                          // pixels per stage (two K = 16 MMA steps)
constexpr int kWgThreads = 256;                    // 8 warps: more gathers in flight (one CTA per SM: 512 tensor-memory columns)
template <int CI>
struct WgradShape {
    static constexpr int ROWS = 9 * CI;                    // (tap, ci) rows; row ROWS is the ones row
    static constexpr int MT = (ROWS + 1 + 127) / 128;      // M = 128 tiles
    static constexpr int MCH = MT * 16;                    // 8-row chunks of A
    static constexpr int A_BYTES = MCH * kWgKB * 16;
    static constexpr int B_BYTES = 8 * kWgKB * 16;         // 64 co = 8 chunks
    static constexpr int COLS = MT * 64 <= 32 ? 32 : MT * 64 <= 64 ? 64 : MT * 64 <= 128 ? 128 : MT * 64 <= 256 ? 256 : 512;
    static constexpr int SMEM = kStages * (A_BYTES + B_BYTES) + 64;
};

template <int CI>
__global__ void __launch_bounds__(kWgThreads) k_wgrad_tc(const bf16 *__restrict__ dZ, const bf16 *__restrict__ X, float *__restrict__ partial,
                                                 float *__restrict__ partial_bias, int N, int H, int W, int Ho, int Wo, int stride,
                                                 int chunk) {
    using S = WgradShape<CI>;
    constexpr int CC = CI / 8;                             // 16-byte chunks of one input pixel
    constexpr uint32_t IDESC = umma_idesc(128, kCo) | (1u << 15) | (1u << 16);   // A and B MN-major
    constexpr uint32_t LBO = 8 * 16, SBO = kWgKB * 16;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *As = smem, *Bs = smem + kStages * S::A_BYTES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(Bs + kStages * S::B_BYTES);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + kStages);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long P = (long long)N * Ho * Wo;
    const long long begin = (long long)blockIdx.x * chunk;
    const long long end = begin + chunk < P ? begin + chunk : P;
    const int blocks = (int)((end - begin + kWgKB - 1) / kWgKB);
    if (warp == 0) tmem_alloc<S::COLS>(slot);
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) bar_init(&bar[s]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // The rows past the gathered ones never change: the ones row (element 0 of its chunk) and zero padding.
    for (int e = tid; e < kStages * (S::MCH - S::ROWS / 8) * kWgKB; e += kWgThreads) {
        const int s = e / ((S::MCH - S::ROWS / 8) * kWgKB), r = e % ((S::MCH - S::ROWS / 8) * kWgKB);
        const int mc = S::ROWS / 8 + r / kWgKB, j = r % kWgKB;
        *reinterpret_cast<uint4 *>(As + s * S::A_BYTES + (mc * kWgKB + j) * 16) =
            make_uint4(mc == S::ROWS / 8 ? 0x3F80u : 0u, 0u, 0u, 0u);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;

    // Gathers of pixel block b into its stage: lane = pixel of the block, warp = an eighth of the chunks.
    auto issue = [&](int b) {
        const int s = b % kStages;
        const long long p = begin + (long long)b * kWgKB + lane;
        const bool live = p < end;
        const int n = live ? (int)(p / ((long long)Ho * Wo)) : 0;
        const int rem = live ? (int)(p % ((long long)Ho * Wo)) : 0;
        const int oy = rem / Wo, ox = rem % Wo;
        unsigned char *as = As + s * S::A_BYTES + lane * 16;
        for (int i = warp; i < 9 * CC; i += kWgThreads / 32) {
            const int t = i / CC, c = i % CC;
            const int iy = oy * stride + t / 3 - 1, ix = ox * stride + t % 3 - 1;
            const bool in = live && iy >= 0 && iy < H && ix >= 0 && ix < W;
            const bf16 *src = in ? X + (((long long)n * H + iy) * W + ix) * CI + c * 8 : X;
            cp_async16(as + i * (kWgKB * 16), src, in ? 16 : 0);
        }
        unsigned char *bs = Bs + s * S::B_BYTES + lane * 16;
        for (int c = warp; c < 8; c += kWgThreads / 32) cp_async16(bs + c * (kWgKB * 16), live ? dZ + p * kCo + c * 8 : dZ, live ? 16 : 0);
        cp_async_commit();
    };

    bool ok = true;
    int issued = 0;
    issue(0);
    if (blocks > 1) issue(1);
    else cp_async_commit();
    for (int b = 0; b < blocks; ++b) {
        const int s = b % kStages;
        if (b + 2 < blocks) {
            // Stage (b + 2) % 3 was last read by the MMAs of block b - 1.
            if (b >= 1 && !bar_wait(&bar[(b - 1) % kStages], ((b - 1) / kStages) & 1)) ok = false;
            if (__syncthreads_or(!ok)) break;
            issue(b + 2);
        } else {
            cp_async_commit();
        }
        cp_async_wait<2>();
        proxy_fence();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t as = sh_addr(As + s * S::A_BYTES), bs = sh_addr(Bs + s * S::B_BYTES);
#pragma unroll
            for (int kk = 0; kk < kWgKB / 16; ++kk) {
                const uint64_t bd = umma_desc(bs + kk * 256, LBO, SBO);
#pragma unroll
                for (int m = 0; m < S::MT; ++m)
                    umma_bf16(tmem + m * kCo, umma_desc(as + m * 16 * SBO + kk * 256, LBO, SBO), bd, IDESC, (b | kk) != 0);
            }
            umma_commit(&bar[s]);
        }
        issued = b + 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (issued > 0 && !bar_wait(&bar[(issued - 1) % kStages], ((issued - 1) / kStages) & 1)) ok = false;
    tc_fence_after();
    if (__syncthreads_or(!ok) || issued < blocks) {
        if (tid == 0) atomicExch(&g_sg_status, 1);
    } else {
        // Warp w reads tensor-memory lanes 32 (w % 4) .. + 31 of the tiles m = w / 4, w / 4 + 2, ...
#pragma unroll 1
        for (int m = warp >> 2; m < S::MT; m += 2) {
            const int q = warp & 3;
            const int r = m * 128 + q * 32 + lane;            // this lane's row: (tap, ci) or the ones row
#pragma unroll
            for (int c0 = 0; c0 < kCo; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + m * kCo + c0, v);
                if (r < S::ROWS) {
                    float *o = partial + ((long long)blockIdx.x * 9 + r / CI) * kCo * CI + r % CI;
#pragma unroll
                    for (int i = 0; i < 16; ++i) o[(c0 + i) * CI] = v[i];
                } else if (r == S::ROWS) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) partial_bias[(long long)blockIdx.x * kCo + c0 + i] = v[i];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_free<S::COLS>(tmem);
}

// ---- tcgen05 shifted-window conv (stride 1) -------------------------------------------------------------
// With stride 1, a tap of the 3x3 conv is a shift of a flattened, zero-padded image: give the image a zero
// border (width Wp = W + 2) and number its pixels g = py * Wp + px; output pixel (y, x) at f = y * Wp + x
// reads tap (ky, kx) of the forward conv at g = f + ky * Wp + kx, and backward data (a conv of dz with the
// taps flipped) at g = f + (2 - ky) * Wp + (2 - kx). A CTA takes M = 128 consecutive f of one image (the two
// border columns of each row are computed and dropped) and loads the padded pixels [f0, f0 + NP) once, NP =
// 128 + 2 Wp + 2, into shared memory in the K-major no-swizzle layout with rows 16 bytes apart ([K chunk]
// [pixel][16 bytes], K chunks LBO apart): the A operand of every tap is then the same patch with the
// descriptor's start moved by 16 bytes per pixel of shift. The 9 taps' weights stay in shared memory for the
// whole persistent tile loop. A ring of NB = 2..4 patch buffers (as many as fit) and two tensor-memory
// accumulators, with loads, MMAs and stores in separate warps: while the tensor cores work on tile j, the
// storing warps drain tile j-1 and the loading warps fill the buffers of the tiles after j. Every wait is bounded;
// a role that times out sets the CTA's abort flag and the status word, and the other roles give up their waits.
template <int MODE, int CI>
struct ShiftShape {
    static constexpr int K = MODE == 0 ? CI : kCo;         // reduction channels per tap
    static constexpr int NC = MODE == 0 ? kCo : CI;        // output columns
    static constexpr int KC = K / 8;                        // 16-byte K chunks
    static constexpr int W_BYTES = 9 * KC * NC * 16;       // resident weights: [tap][K chunk][column][16 bytes]
    static constexpr int COLS = 2 * NC < 32 ? 32 : 2 * NC;  // two accumulators
    // K chunks of a patch lie (NP + LPAD) * 16 bytes apart: with NP a multiple of 8, the 8 (or 2) chunks of a
    // pixel that a quarter-warp stores land on distinct banks.
    static constexpr int LPAD = KC == 8 ? 1 : 4;
};
constexpr int kShiftThreads = 384;                        // 12 warps: MMA issue, 3 loading, 8 storing
constexpr int kShiftMaxSmem = 227 * 1024;
constexpr int kShiftSmPerSm = 228 * 1024;                  // shared memory of an SM (1 KB of it reserved per CTA)
__host__ __device__ constexpr int shift_np(int W) { return (128 + 2 * (W + 2) + 2 + 7) / 8 * 8; }
// MODE 2 (stride-2 backward data by parity class): the dz image with one zero column and row at its far edges
// (row width Wo + 1), read at offsets 0 or 1 along each axis.
__host__ __device__ constexpr int shift_np2(int Wo) { return (128 + (Wo + 1) + 1 + 7) / 8 * 8; }

// Bounded wait that also gives up once another role of the CTA has aborted (*abort set).
__device__ __forceinline__ bool bar_wait_or_abort(uint64_t *bar, uint32_t parity, volatile int *abort) {
    const uint32_t addr = sh_addr(bar);
    for (int it = 0; it < 20000; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(addr), "r"(parity), "r"(100000u) : "memory");
        if (done) return true;
        if (*abort) return false;
    }
    *abort = 1;
    atomicExch(&g_sg_status, 1);
    return false;
}

__device__ __forceinline__ void bar_init_count(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sh_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sh_addr(bar)) : "memory");
}

// Warp roles: warp 0 issues the MMAs (one elected thread), warps 1-3 load patches, warps 4-11 store outputs (warp
// 4 + q and 8 + q read tensor-memory lanes 32q..32q+31, one half of the columns each; with 16 columns warps 4-7
// store alone). full[i]: the 96 loaders' patch of buffer i has landed (each loader waits for its own copies,
// fences them for the tensor cores and arrives); empty[i]: the MMAs that read buffer i are done
// (tcgen05.commit); accf[a]: accumulator a holds a finished tile (commit); acce[a]: the storing threads have
// read accumulator a. A loader keeps two tiles of copies in flight and runs up to NB
// tiles ahead of the tensor cores; the tensor cores run one tile ahead of the stores.
// Register budget: three CTAs per SM for the 16-channel input layer (its shared memory allows three), one otherwise.
template <int MODE, int CI>
__global__ void __launch_bounds__(kShiftThreads, MODE == 0 && CI == 16 ? 3 : 1) k_conv_shift(const bf16 *__restrict__ src, const bf16 *__restrict__ wsrc,
                                                             const float *__restrict__ bias, const bf16 *__restrict__ zprev,
                                                             bf16 *__restrict__ out0, void *__restrict__ out1, int N, int H, int W, int NB) {
    using S = ShiftShape<MODE, CI>;
    constexpr int K = S::K, NC = S::NC, KC = S::KC;
    constexpr int LOADERS = 96;
    constexpr int STORERS = NC >= 32 ? 256 : 128;          // threads that read an accumulator
    constexpr int SPAN = NC >= 32 ? NC / 2 : NC;           // columns per storing warp
    constexpr uint32_t IDESC = umma_idesc(128, NC);
    extern __shared__ __align__(1024) unsigned char smem[];
    // MODE 2: input pixels (y, x) = (2u + cy, 2v + cx) of parity class c = 2 cy + cx take dz[u + dy][v + dx] through
    // the taps ky = y + 1, kx = x + 1 (mod 2), dy = (cy + 1 - ky) / 2 in {0, 1} (likewise dx): per class a conv of
    // the dz image with 1, 2 or 4 taps, on rows f = u (Wo + 1) + v. MODES 0 and 1: rows f = y (W + 2) + x.
    constexpr bool CLS = MODE == 2;
    const int Ho = (H - 1) / 2 + 1, Wo = (W - 1) / 2 + 1;
    const int Wp = CLS ? Wo + 1 : W + 2, np = CLS ? shift_np2(Wo) : shift_np(W);
    const int lbo = (np + S::LPAD) * 16, pbytes = KC * lbo;
    unsigned char *ws = smem, *ps = smem + S::W_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(ps + NB * pbytes);
    uint64_t *empty = full + 4, *accf = full + 8, *acce = full + 10;
    uint32_t *slot = reinterpret_cast<uint32_t *>(full + 12);
    volatile int *abort = reinterpret_cast<volatile int *>(slot + 1);
    float *sbias = reinterpret_cast<float *>(full + 13);      // forward: the 64 biases
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_img = (H * Wp + 127) / 128;
    int tend[4] = {0, 0, 0, 0}, tiles = N * tiles_img;      // MODE 2: tiles of classes 0..c
    if (CLS) {
        for (int c = 0, t = 0; c < 4; ++c) {
            t += N * ((((H - (c >> 1) + 1) / 2) * Wp + 127) / 128);
            tend[c] = t;
        }
        tiles = tend[3];
    }
    // Image n, first row f0 and parity class c of a tile.
    auto decode = [&](int tile, int &n, int &f0, int &c) {
        if (!CLS) {
            n = tile / tiles_img, f0 = (tile % tiles_img) * 128, c = 0;
            return;
        }
        c = tile >= tend[2] ? 3 : tile >= tend[1] ? 2 : tile >= tend[0] ? 1 : 0;
        const int local = tile - (c ? tend[c - 1] : 0), per = ((((H - (c >> 1) + 1) / 2) * Wp + 127) / 128);
        n = local / per, f0 = (local % per) * 128;
    };
    const int count = (int)blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;   // local tiles
    if (warp == 0) tmem_alloc<S::COLS>(slot);
    if (tid == 0) {
        for (int i = 0; i < NB; ++i) {
            bar_init_count(&full[i], LOADERS);
            bar_init_count(&empty[i], 1);
        }
        for (int a = 0; a < 2; ++a) {
            bar_init_count(&accf[a], 1);
            bar_init_count(&acce[a], STORERS);
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int e = tid; e < 9 * NC * KC; e += kShiftThreads) {
        const int kc = e % KC, col = (e / KC) % NC, tap = e / (KC * NC);
        cp_async16(ws + ((tap * KC + kc) * NC + col) * 16, wsrc + ((long long)tap * NC + col) * K + kc * 8, 16);
    }
    if (MODE == 0 && tid < kCo) sbias[tid] = bias[tid];
    cp_async_commit();
    cp_async_wait<0>();
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;

    if (warp >= 1 && warp <= 3) {
        // Loaders: patch of local tile j = padded pixels [f0, f0 + np) of its image into buffer j % NB.
        const int lt = tid - 32;
        for (int j = 0; j < count; ++j) {
            const int b = j % NB;
            if (j >= NB && !bar_wait_or_abort(&empty[b], (j / NB - 1) & 1, abort)) break;
            int n, f0, c;
            decode(blockIdx.x + j * gridDim.x, n, f0, c);
            unsigned char *p = ps + b * pbytes;
            for (int e = lt; e < np * KC; e += LOADERS) {
                const int kc = e % KC, i = e / KC, g = f0 + i;
                const int py = g / Wp, px = g - py * Wp;
                const bool in = CLS ? py < Ho && px < Wo : py >= 1 && py <= H && px >= 1 && px <= W;
                const bf16 *s = !in ? src
                              : CLS ? src + (((long long)n * Ho + py) * Wo + px) * K + kc * 8
                                    : src + (((long long)n * H + py - 1) * W + px - 1) * K + kc * 8;
                cp_async16(p + kc * lbo + i * 16, s, in ? 16 : 0);
            }
            cp_async_commit();
            if (j >= 1) {                                 // tile j-1's copies have landed
                cp_async_wait<1>();
                proxy_fence();
                bar_arrive(&full[(j - 1) % NB]);
            }
        }
        cp_async_wait<0>();
        proxy_fence();
        if (count > 0 && !*abort) bar_arrive(&full[(count - 1) % NB]);
    } else if (warp == 0) {
        // The MMAs of local tile j into accumulator j & 1, one elected thread.
        int committed = 0;
        if (lane == 0) {
            for (int j = 0; j < count; ++j) {
                const int b = j % NB, a = j & 1;
                if (!bar_wait_or_abort(&full[b], (j / NB) & 1, abort)) break;
                if (j >= 2 && !bar_wait_or_abort(&acce[a], (j / 2 - 1) & 1, abort)) break;
                tc_fence_after();
                const uint32_t pa = sh_addr(ps + b * pbytes), wa = sh_addr(ws);
                int n, f0, c;
                decode(blockIdx.x + j * gridDim.x, n, f0, c);
                // Tap i of the tile: weights of tap t, patch shifted by `shift` pixels.
                auto mma_tap = [&](int i, int t, int shift) {
#pragma unroll
                    for (int kk = 0; kk < K / 16; ++kk) {
                        const uint64_t ad = umma_desc(pa + shift * 16 + kk * 2 * lbo, lbo, 128);
                        const uint64_t bd = umma_desc(wa + (t * KC + 2 * kk) * NC * 16, NC * 16, 128);
                        umma_bf16(tmem + a * NC, ad, bd, IDESC, (i | kk) != 0);
                    }
                };
                if constexpr (CLS) {
                    const int nkx = c & 1 ? 2 : 1, taps = (c >> 1 ? 2 : 1) * nkx;
                    for (int i = 0; i < taps; ++i) {
                        const int ky = c >> 1 ? 2 * (i / nkx) : 1, kx = c & 1 ? 2 * (i % nkx) : 1;
                        mma_tap(i, ky * 3 + kx, (ky == 0) * Wp + (kx == 0));
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 9; ++i) {
                        const int ky = i / 3, kx = i % 3;
                        mma_tap(i, i, MODE == 0 ? ky * Wp + kx : (2 - ky) * Wp + (2 - kx));
                    }
                }
                umma_commit(&empty[b]);
                umma_commit(&accf[a]);
                committed = j + 1;
            }
            // On an abort, wait (bounded, whatever the flag) for the MMAs already issued before tensor memory is freed.
            if (*abort && committed > 0) {
                const int last = committed - 1;
                uint32_t done = 0;
                for (int it = 0; it < 20000 && !done; ++it)
                    asm volatile(
                        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
                        : "=r"(done) : "r"(sh_addr(&accf[last & 1])), "r"((last / 2) & 1), "r"(100000u) : "memory");
            }
        }
        __syncwarp();
    } else if ((warp - 4) * 32 < STORERS) {
        // Stores of local tile j from accumulator j & 1: this thread's row (tensor-memory lane), SPAN columns.
        const int quarter = (warp - 4) & 3, cbeg = ((warp - 4) >> 2) * SPAN;
        for (int j = 0; j < count; ++j) {
            const int a = j & 1;
            if (!bar_wait_or_abort(&accf[a], (j / 2) & 1, abort)) break;
            tc_fence_after();
            int n, f0, c;
            decode(blockIdx.x + j * gridDim.x, n, f0, c);
            const int f = f0 + quarter * 32 + lane;
            const int u = f / Wp, v = f - u * Wp;
            const int cy = c >> 1, cx = c & 1;
            const bool live = CLS ? u < (H - cy + 1) / 2 && v < (W - cx + 1) / 2 : u < H && v < W;
            const long long row = CLS ? ((long long)n * H + 2 * u + cy) * W + 2 * v + cx : ((long long)n * H + u) * W + v;
            // This warp's SPAN columns in one tensor-memory load (one wait), then 16 at a time.
            float vs[SPAN];
            if constexpr (SPAN == 32) {
                tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + a * NC + cbeg, vs);
            } else {
                float v16[16];
                tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + a * NC + cbeg, v16);
#pragma unroll
                for (int i = 0; i < 16; ++i) vs[i] = v16[i];
            }
#pragma unroll
            for (int c0 = cbeg; c0 < cbeg + SPAN; c0 += 16) {
                const float *v = vs + (c0 - cbeg);
                if (!live) continue;
                if (MODE == 0) {
                    __align__(16) bf16 zb[16], ab[16];
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const float z = v[i] + sbias[c0 + i];
                        zb[i] = __float2bfloat16_rn(z);
                        ab[i] = __float2bfloat16_rn(gelu(z));
                    }
                    uint4 *zd = reinterpret_cast<uint4 *>(out0 + row * kCo + c0);
                    uint4 *adst = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(out1) + row * kCo + c0);
                    zd[0] = reinterpret_cast<const uint4 *>(zb)[0];
                    zd[1] = reinterpret_cast<const uint4 *>(zb)[1];
                    adst[0] = reinterpret_cast<const uint4 *>(ab)[0];
                    adst[1] = reinterpret_cast<const uint4 *>(ab)[1];
                } else if (zprev) {
                    __align__(16) bf16 zp[16], db[16];
                    reinterpret_cast<uint4 *>(zp)[0] = reinterpret_cast<const uint4 *>(zprev + row * CI + c0)[0];
                    reinterpret_cast<uint4 *>(zp)[1] = reinterpret_cast<const uint4 *>(zprev + row * CI + c0)[1];
#pragma unroll
                    for (int i = 0; i < 16; ++i) db[i] = __float2bfloat16_rn(v[i] * gelu_grad(__bfloat162float(zp[i])));
                    uint4 *dd = reinterpret_cast<uint4 *>(out0 + row * CI + c0);
                    dd[0] = reinterpret_cast<const uint4 *>(db)[0];
                    dd[1] = reinterpret_cast<const uint4 *>(db)[1];
                } else {
                    float4 *o = reinterpret_cast<float4 *>(reinterpret_cast<float *>(out1) + row * CI + c0);
#pragma unroll
                    for (int i = 0; i < 4; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                }
            }
            tc_fence_before();
            bar_arrive(&acce[a]);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free<S::COLS>(tmem);
}

// Launches the shifted-window kernel when at least two patch buffers fit in shared memory (image rows up to a
// few hundred pixels); false when the caller should use the gather kernel instead.
template <int MODE, int CI>
bool launch_shift(const bf16 *src, const bf16 *w, const float *bias, const bf16 *zprev, bf16 *o0, void *o1, int n, int h, int wd,
                  cudaStream_t s) {
    using S = ShiftShape<MODE, CI>;
    const int wo = (wd - 1) / 2 + 1, wp = MODE == 2 ? wo + 1 : wd + 2;
    const long long pbytes = (long long)S::KC * ((MODE == 2 ? shift_np2(wo) : shift_np(wd)) + S::LPAD) * 16;
    int nb = 4;                          // + 384 bytes: 12 mbarriers, the tensor-memory slot, the abort flag, 64 biases
    while (nb >= 2 && S::W_BYTES + nb * pbytes + 384 > kShiftMaxSmem) --nb;
    if (nb < 2) return false;
    const int smem = (int)(S::W_BYTES + nb * pbytes + 384);
    static const cudaError_t attr = cudaFuncSetAttribute(k_conv_shift<MODE, CI>, cudaFuncAttributeMaxDynamicSharedMemorySize, kShiftMaxSmem);
    (void)attr;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            sms = 148;
    }
    static int regs = 0;
    if (!regs) {
        cudaFuncAttributes fa;
        regs = cudaFuncGetAttributes(&fa, k_conv_shift<MODE, CI>) == cudaSuccess && fa.numRegs > 0 ? fa.numRegs : 255;
    }
    int per_sm = kShiftSmPerSm / (smem + 1024);
    const int regs_cta = (regs * 32 + 255) / 256 * 256 * (kShiftThreads / 32);   // registers are allocated per warp
    per_sm = per_sm < 65536 / regs_cta ? per_sm : 65536 / regs_cta;
    per_sm = per_sm < 512 / S::COLS ? per_sm : 512 / S::COLS;      // tensor-memory columns of an SM
    per_sm = per_sm < 2048 / kShiftThreads ? per_sm : 2048 / kShiftThreads;
    per_sm = per_sm < 1 ? 1 : per_sm;
    long long tiles = (long long)n * ((h * wp + 127) / 128);
    if (MODE == 2) {
        tiles = 0;
        for (int c = 0; c < 4; ++c) tiles += (long long)n * ((((h - (c >> 1) + 1) / 2) * wp + 127) / 128);
    }
    const long long grid = tiles < (long long)sms * per_sm ? tiles : (long long)sms * per_sm;
    k_conv_shift<MODE, CI><<<(unsigned)grid, kShiftThreads, (size_t)smem, s>>>(src, w, bias, zprev, o0, o1, n, h, wd, nb);
    return true;
}

// 0: mma.sync kernels; 1: tcgen05 kernels, the shifted-window form where it fits (default: stride-1 layers, and the
// stride-2 input gradient by parity class); 2: tcgen05 kernels, the per-tap gather form for every layer.
int g_tensor_path = 1;

int blocks_for(long long work, int threads) {
    const long long b = (work + threads - 1) / threads;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

int check_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        tfd::set_error(std::string(what) + ": " + cudaGetErrorString(e));
        return TFD_ERR_CUDA;
    }
    return TFD_OK;
}

int bad(const char *what) {
    tfd::set_error(what);
    return TFD_ERR_INVALID;
}

int out_size(int n, int stride) { return (n - 1) / stride + 1; }

}  // namespace

extern "C" {

// 1: conv forward, backward data and backward weight on the tcgen05 kernels, stride-1 layers in the
// shifted-window form where it fits (default); 2: the same with the per-tap gather form for every layer;
// 0: on the mma.sync kernels.
int tfd_sg_set_tensor_path(int32_t mode) {
    if (mode < 0 || mode > 2) return bad("tfd_sg_set_tensor_path: mode 0, 1 or 2");
    g_tensor_path = mode;
    return TFD_OK;
}

// Device status of the surrogate kernels (1: a bounded tensor-core wait timed out); reading clears it.
int tfd_sg_status(int32_t *status) {
    if (!status) return bad("tfd_sg_status: null argument");
    int v = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_sg_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_sg_status, &zero, sizeof(int));
    if (e != cudaSuccess) {
        tfd::set_error(std::string("tfd_sg_status: ") + cudaGetErrorString(e));
        return TFD_ERR_CUDA;
    }
    *status = v;
    return TFD_OK;
}

int tfd_sg_pack_input(const float *rho, int32_t n, int32_t h, int32_t w, void *x0, void *stream) {
    if (!rho || !x0 || n < 1 || h < 1 || w < 1) return bad("tfd_sg_pack_input: bad arguments");
    if ((long long)n * h * w >= (1LL << 31)) return bad("tfd_sg_pack_input: more than 2^31 pixels");
    k_pack_input<<<blocks_for((long long)n * h * w, 256), 256, 0, (cudaStream_t)stream>>>(rho, (bf16 *)x0, n * h * w, h, w);
    return check_launch("tfd_sg_pack_input");
}

int tfd_sg_conv_forward(const void *x, const void *w, const float *bias, void *z, void *a, int32_t n, int32_t h, int32_t wd,
                        int32_t ci, int32_t stride, void *stream) {
    if (!x || !w || !bias || !z || !a || (ci != 16 && ci != 64) || (stride != 1 && stride != 2) || n < 1 || h < 1 || wd < 1)
        return bad("tfd_sg_conv_forward: bad arguments (ci 16 or 64, stride 1 or 2)");
    const int ho = out_size(h, stride), wo = out_size(wd, stride);
    const long long P = (long long)n * ho * wo;
    cudaStream_t s = (cudaStream_t)stream;
    if (g_tensor_path == 1 && stride == 1) {
        const bool done = ci == 16 ? launch_shift<0, 16>((const bf16 *)x, (const bf16 *)w, bias, nullptr, (bf16 *)z, a, n, h, wd, s)
                                   : launch_shift<0, 64>((const bf16 *)x, (const bf16 *)w, bias, nullptr, (bf16 *)z, a, n, h, wd, s);
        if (done) return check_launch("tfd_sg_conv_forward (tcgen05, shifted window)");
    }
    if (g_tensor_path) {
        const dim3 grid((unsigned)((P + 127) / 128));
        if (ci == 16) {
            static const cudaError_t attr = cudaFuncSetAttribute(k_conv_tc<0, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem(16, 64));
            (void)attr;
            k_conv_tc<0, 16><<<grid, 128, tc_smem(16, 64), s>>>((const bf16 *)x, (const bf16 *)w, bias, nullptr, (bf16 *)z, a, n, h, wd, ho, wo, stride);
        } else {
            static const cudaError_t attr = cudaFuncSetAttribute(k_conv_tc<0, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem(64, 64));
            (void)attr;
            k_conv_tc<0, 64><<<grid, 128, tc_smem(64, 64), s>>>((const bf16 *)x, (const bf16 *)w, bias, nullptr, (bf16 *)z, a, n, h, wd, ho, wo, stride);
        }
        return check_launch("tfd_sg_conv_forward (tcgen05)");
    }
    const dim3 grid((unsigned)((P + kTile - 1) / kTile));
    if (ci == 16) k_conv_fwd<16><<<grid, kThreads, 0, s>>>((const bf16 *)x, (const bf16 *)w, bias, (bf16 *)z, (bf16 *)a, n, h, wd, ho, wo, stride);
    else k_conv_fwd<64><<<grid, kThreads, 0, s>>>((const bf16 *)x, (const bf16 *)w, bias, (bf16 *)z, (bf16 *)a, n, h, wd, ho, wo, stride);
    return check_launch("tfd_sg_conv_forward");
}

int tfd_sg_conv_backward_data(const void *dz, const void *wt, const void *zprev, void *out, int32_t n, int32_t h, int32_t wd,
                              int32_t ci, int32_t stride, void *stream) {
    if (!dz || !wt || !out || (ci != 16 && ci != 64) || (stride != 1 && stride != 2) || n < 1 || h < 1 || wd < 1)
        return bad("tfd_sg_conv_backward_data: bad arguments");
    const int ho = out_size(h, stride), wo = out_size(wd, stride);
    const long long Q = (long long)n * h * wd;
    cudaStream_t s = (cudaStream_t)stream;
    bf16 *o0 = zprev ? (bf16 *)out : nullptr;
    void *o1 = zprev ? nullptr : out;
    if (g_tensor_path == 1) {
        bool done;
        if (stride == 1)
            done = ci == 16 ? launch_shift<1, 16>((const bf16 *)dz, (const bf16 *)wt, nullptr, (const bf16 *)zprev, o0, o1, n, h, wd, s)
                            : launch_shift<1, 64>((const bf16 *)dz, (const bf16 *)wt, nullptr, (const bf16 *)zprev, o0, o1, n, h, wd, s);
        else
            done = ci == 16 ? launch_shift<2, 16>((const bf16 *)dz, (const bf16 *)wt, nullptr, (const bf16 *)zprev, o0, o1, n, h, wd, s)
                            : launch_shift<2, 64>((const bf16 *)dz, (const bf16 *)wt, nullptr, (const bf16 *)zprev, o0, o1, n, h, wd, s);
        if (done) return check_launch("tfd_sg_conv_backward_data (tcgen05, shifted window)");
    }
    if (g_tensor_path) {
        dim3 grid((unsigned)((Q + 127) / 128));
        int4 cls = make_int4(0, 0, 0, 0);
        if (stride == 2) {
            // CTAs by parity class: class c = 2 (y & 1) + (x & 1) takes blocks [end of class c-1, end of class c).
            long long end[4], total = 0;
            for (int c = 0; c < 4; ++c) {
                const long long rows = (long long)n * ((h - (c >> 1) + 1) / 2) * ((wd - (c & 1) + 1) / 2);
                total += (rows + 127) / 128;
                end[c] = total;
            }
            cls = make_int4((int)end[0], (int)end[1], (int)end[2], 1);
            grid = dim3((unsigned)total);
        }
        if (ci == 16) {
            static const cudaError_t attr = cudaFuncSetAttribute(k_conv_tc<1, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem(64, 16));
            (void)attr;
            k_conv_tc<1, 16><<<grid, 128, tc_smem(64, 16), s>>>((const bf16 *)dz, (const bf16 *)wt, nullptr, (const bf16 *)zprev, o0, o1, n, h, wd,
                                                               ho, wo, stride, cls);
        } else {
            static const cudaError_t attr = cudaFuncSetAttribute(k_conv_tc<1, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem(64, 64));
            (void)attr;
            k_conv_tc<1, 64><<<grid, 128, tc_smem(64, 64), s>>>((const bf16 *)dz, (const bf16 *)wt, nullptr, (const bf16 *)zprev, o0, o1, n, h, wd,
                                                               ho, wo, stride, cls);
        }
        return check_launch("tfd_sg_conv_backward_data (tcgen05)");
    }
    const dim3 grid((unsigned)((Q + kTile - 1) / kTile));
    if (ci == 16) k_conv_dgrad<16><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)wt, (const bf16 *)zprev, out, n, h, wd, ho, wo, stride);
    else k_conv_dgrad<64><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)wt, (const bf16 *)zprev, out, n, h, wd, ho, wo, stride);
    return check_launch("tfd_sg_conv_backward_data");
}

// Output pixels per partial sum of the weight gradient: at most `chunk`, and fewer on small layers so that about
// two CTAs per SM (296) sum side by side (a multiple of 64 pixels).
static long long wgrad_chunk(long long P, int chunk) {
    long long want = (P + 295) / 296;
    want = (want + kTile - 1) / kTile * kTile;
    return want < chunk ? want : chunk;
}

int tfd_sg_wgrad_scratch(int32_t n, int32_t h, int32_t wd, int32_t ci, int32_t stride, int32_t chunk, size_t *bytes) {
    if (!bytes || chunk < kTile || chunk % kTile) return bad("tfd_sg_wgrad_scratch: chunk must be a positive multiple of 64");
    const long long P = (long long)n * out_size(h, stride) * out_size(wd, stride);
    const long long c = wgrad_chunk(P, chunk);
    const long long chunks = (P + c - 1) / c;
    *bytes = (size_t)(chunks * 9 * kCo * ci + chunks * kCo) * sizeof(float);
    return TFD_OK;
}

int tfd_sg_conv_backward_weight(const void *dz, const void *x, float *dw, float *dbias, float *scratch, size_t scratch_bytes,
                                int32_t n, int32_t h, int32_t wd, int32_t ci, int32_t stride, int32_t chunk, void *stream) {
    if (!dz || !x || !dw || !dbias || !scratch || (ci != 16 && ci != 64) || (stride != 1 && stride != 2))
        return bad("tfd_sg_conv_backward_weight: bad arguments");
    size_t need = 0;
    int rc = tfd_sg_wgrad_scratch(n, h, wd, ci, stride, chunk, &need);
    if (rc) return rc;
    if (scratch_bytes < need) return bad("tfd_sg_conv_backward_weight: scratch smaller than tfd_sg_wgrad_scratch()");
    const int ho = out_size(h, stride), wo = out_size(wd, stride);
    const long long P = (long long)n * ho * wo;
    chunk = (int32_t)wgrad_chunk(P, chunk);
    const int chunks = (int)((P + chunk - 1) / chunk);
    float *partial = scratch, *partial_bias = scratch + (long long)chunks * 9 * kCo * ci;
    cudaStream_t s = (cudaStream_t)stream;
    if (g_tensor_path) {
        if (ci == 16) {
            static const cudaError_t attr = cudaFuncSetAttribute(k_wgrad_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, WgradShape<16>::SMEM);
            (void)attr;
            k_wgrad_tc<16><<<chunks, kWgThreads, WgradShape<16>::SMEM, s>>>((const bf16 *)dz, (const bf16 *)x, partial, partial_bias, n, h, wd, ho, wo,
                                                                    stride, chunk);
        } else {
            static const cudaError_t attr = cudaFuncSetAttribute(k_wgrad_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, WgradShape<64>::SMEM);
            (void)attr;
            k_wgrad_tc<64><<<chunks, kWgThreads, WgradShape<64>::SMEM, s>>>((const bf16 *)dz, (const bf16 *)x, partial, partial_bias, n, h, wd, ho, wo,
                                                                    stride, chunk);
        }
        if ((rc = check_launch("tfd_sg_conv_backward_weight (tcgen05)"))) return rc;
    } else {
        const dim3 grid((unsigned)chunks, 9);
        if (ci == 16) k_conv_wgrad<16><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)x, partial, partial_bias, n, h, wd, ho, wo, stride, chunk);
        else k_conv_wgrad<64><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)x, partial, partial_bias, n, h, wd, ho, wo, stride, chunk);
        if ((rc = check_launch("tfd_sg_conv_backward_weight"))) return rc;
    }
    const long long len = 9LL * kCo * ci;
    k_reduce_partials<<<(unsigned)((len + kCo + 63) / 64), 256, 0, s>>>(partial, chunks, len, dw, partial_bias, kCo, dbias);
    return check_launch("tfd_sg_conv_backward_weight reduce");
}

int tfd_sg_head_forward(const void *a, const float *wh, const float *bh, float *out, int32_t n, int32_t features, int32_t k,
                        void *stream) {
    if (!a || !wh || !bh || !out || n < 1 || features < 1 || k < 1) return bad("tfd_sg_head_forward: bad arguments");
    k_head_fwd<<<n, 256, 0, (cudaStream_t)stream>>>((const bf16 *)a, wh, bh, out, features, k);
    return check_launch("tfd_sg_head_forward");
}

int tfd_sg_mse(const float *out, const float *y, float *dout, float *loss, int32_t total, void *stream) {
    if (!out || !y || !loss || total < 1) return bad("tfd_sg_mse: bad arguments");
    k_mse<<<1, 256, 0, (cudaStream_t)stream>>>(out, y, dout, loss, total);
    return check_launch("tfd_sg_mse");
}

int tfd_sg_head_backward(const float *dout, const void *a_last, const float *wh, const void *z_last, float *dwh, float *dbh,
                         void *dz_last, int32_t n, int32_t features, int32_t k, void *stream) {
    if (!dout || !a_last || !wh || !z_last || !dz_last || n < 1 || features < 1 || k < 1) return bad("tfd_sg_head_backward: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (dwh && dbh)
        k_head_bwd_params<<<blocks_for((long long)k * features, 256), 256, 0, s>>>(dout, (const bf16 *)a_last, dwh, dbh, n, features, k);
    k_head_bwd_data<<<blocks_for((long long)n * features, 256), 256, 0, s>>>(dout, wh, (const bf16 *)z_last, (bf16 *)dz_last, n, features, k);
    return check_launch("tfd_sg_head_backward");
}

int tfd_sg_adam(float *p, const float *g, float *m, float *v, int64_t count, float lr, float b1, float b2, float eps, int32_t step,
                void *stream) {
    if (!p || !g || !m || !v || count < 0 || step < 1) return bad("tfd_sg_adam: bad arguments");
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, count, lr, b1, b2, eps, c1, c2);
    return check_launch("tfd_sg_adam");
}

int tfd_sg_cast_weights(const float *w, void *w_bf16, void *wt_bf16, int32_t ci, void *stream) {
    if (!w || !w_bf16 || !wt_bf16 || (ci != 16 && ci != 64)) return bad("tfd_sg_cast_weights: bad arguments");
    k_cast_weights<<<blocks_for(9LL * kCo * ci, 256), 256, 0, (cudaStream_t)stream>>>(w, (bf16 *)w_bf16, (bf16 *)wt_bf16, ci);
    return check_launch("tfd_sg_cast_weights");
}

}  // extern "C"
