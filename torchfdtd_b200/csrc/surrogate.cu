// Learned surrogate: a small convolutional neural operator (8 conv layers, 64 channels) mapping a 2D design
// density to its complex transmission spectrum, trained and evaluated by these kernels.
//
// Numerics: BF16 operands, FP32 accumulation (tensor-core mma.sync m16n8k16, bf16 x bf16 -> f32), FP32
// master weights, bias, head (linear on the flattened last feature map), loss and Adam state. Activations are NHWC bf16 with C = 16 (the packed input:
// density, x, y, 1, zeros) or C = 64, so one pixel is one or four 16-byte vectors.
//
// Each conv is 3x3, zero padding 1, stride 1 or 2, Cout = 64, followed by GELU (tanh form):
//   forward          z[p, co] = bias[co] + sum_{tap, ci} x[in(p, tap), ci] w[tap, co, ci];  a = gelu(z)
//   backward (data)  dx[q, ci] = sum_{tap, co} dz[out(q, tap), co] w[tap, co, ci]  (then * gelu'(z_prev))
//   backward (weight) dw[tap, co, ci] = sum_p dz[p, co] x[in(p, tap), ci]; dbias[co] = sum_p dz[p, co]
// All three are implicit GEMMs on 64 x 64 tiles: 4 warps, each 16 rows x 64 columns of m16n8k16 MMAs, with
// the operands staged in shared memory (row-major A, column-major B, both padded to 144-byte rows so the
// fragment loads are bank-conflict free).
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

__device__ __forceinline__ float gelu(float z) {
    const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
    return 0.5f * z * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
    const float th = tanhf(u);
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
// (and, for the centre tap, the partial bias gradient); k_reduce_partials adds the chunks in order.
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

__global__ void k_reduce_partials(const float *__restrict__ partial, int chunks, long long len, float *__restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < len; e += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int c = 0; c < chunks; ++c) s += partial[(long long)c * len + e];
        out[e] = s;
    }
}

// ---- input packing, head, loss, optimiser ---------------------------------------------------------------
// x0[n, y, x, :] = (2 rho - 1, xc, yc, 1, 0 ...) with coordinates in [-1, 1].
__global__ void k_pack_input(const float *__restrict__ rho, bf16 *__restrict__ x0, int N, int H, int W) {
    const long long total = (long long)N * H * W;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < total; p += (long long)gridDim.x * blockDim.x) {
        const int rem = (int)(p % ((long long)H * W));
        const int y = rem / W, x = rem % W;
        float v[16] = {};
        v[0] = 2.f * rho[p] - 1.f;
        v[1] = W > 1 ? -1.f + 2.f * x / (W - 1) : 0.f;
        v[2] = H > 1 ? -1.f + 2.f * y / (H - 1) : 0.f;
        v[3] = 1.f;
        bf16 *o = x0 + p * 16;
#pragma unroll
        for (int c = 0; c < 16; ++c) o[c] = __float2bfloat16_rn(v[c]);
    }
}

// Linear head on the flattened last feature map: out[n, j] = bh[j] + sum_f wh[j, f] a[n, f], f = p * 64 + c
// (the positions stay distinct: the scene is not translation invariant). One block per sample.
__global__ void k_head_fwd(const bf16 *__restrict__ a, const float *__restrict__ wh, const float *__restrict__ bh,
                           float *__restrict__ out, int F, int K) {
    __shared__ float red[256];
    const int n = blockIdx.x;
    for (int j = 0; j < K; ++j) {
        float s = 0.f;
        for (int f = threadIdx.x; f < F; f += blockDim.x) s += wh[(long long)j * F + f] * __bfloat162float(a[(long long)n * F + f]);
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[n * K + j] = bh[j] + red[0];
        __syncthreads();
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

int tfd_sg_pack_input(const float *rho, int32_t n, int32_t h, int32_t w, void *x0, void *stream) {
    if (!rho || !x0 || n < 1 || h < 1 || w < 1) return bad("tfd_sg_pack_input: bad arguments");
    k_pack_input<<<blocks_for((long long)n * h * w, 256), 256, 0, (cudaStream_t)stream>>>(rho, (bf16 *)x0, n, h, w);
    return check_launch("tfd_sg_pack_input");
}

int tfd_sg_conv_forward(const void *x, const void *w, const float *bias, void *z, void *a, int32_t n, int32_t h, int32_t wd,
                        int32_t ci, int32_t stride, void *stream) {
    if (!x || !w || !bias || !z || !a || (ci != 16 && ci != 64) || (stride != 1 && stride != 2) || n < 1 || h < 1 || wd < 1)
        return bad("tfd_sg_conv_forward: bad arguments (ci 16 or 64, stride 1 or 2)");
    const int ho = out_size(h, stride), wo = out_size(wd, stride);
    const long long P = (long long)n * ho * wo;
    const dim3 grid((unsigned)((P + kTile - 1) / kTile));
    cudaStream_t s = (cudaStream_t)stream;
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
    const dim3 grid((unsigned)((Q + kTile - 1) / kTile));
    cudaStream_t s = (cudaStream_t)stream;
    if (ci == 16) k_conv_dgrad<16><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)wt, (const bf16 *)zprev, out, n, h, wd, ho, wo, stride);
    else k_conv_dgrad<64><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)wt, (const bf16 *)zprev, out, n, h, wd, ho, wo, stride);
    return check_launch("tfd_sg_conv_backward_data");
}

int tfd_sg_wgrad_scratch(int32_t n, int32_t h, int32_t wd, int32_t ci, int32_t stride, int32_t chunk, size_t *bytes) {
    if (!bytes || chunk < kTile || chunk % kTile) return bad("tfd_sg_wgrad_scratch: chunk must be a positive multiple of 64");
    const long long P = (long long)n * out_size(h, stride) * out_size(wd, stride);
    const long long chunks = (P + chunk - 1) / chunk;
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
    const int chunks = (int)((P + chunk - 1) / chunk);
    float *partial = scratch, *partial_bias = scratch + (long long)chunks * 9 * kCo * ci;
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid((unsigned)chunks, 9);
    if (ci == 16) k_conv_wgrad<16><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)x, partial, partial_bias, n, h, wd, ho, wo, stride, chunk);
    else k_conv_wgrad<64><<<grid, kThreads, 0, s>>>((const bf16 *)dz, (const bf16 *)x, partial, partial_bias, n, h, wd, ho, wo, stride, chunk);
    if ((rc = check_launch("tfd_sg_conv_backward_weight"))) return rc;
    const long long len = 9LL * kCo * ci;
    k_reduce_partials<<<blocks_for(len, 256), 256, 0, s>>>(partial, chunks, len, dw);
    k_reduce_partials<<<1, kCo, 0, s>>>(partial_bias, chunks, kCo, dbias);
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
