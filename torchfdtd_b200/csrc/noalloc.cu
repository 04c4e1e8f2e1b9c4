// tfd_field_norm_static: the divergence-diagnostic reduction (energy and peak of E and H) for callers
// that cannot allocate device memory.
//
// Who needs it: a health check that must still work when the device is out of memory (it runs after an
// allocation has failed, exactly when a new allocation would fail too), and hosts whose device memory is
// owned by a pool or budget they must not bypass with their own cudaMalloc. tfd_diagnose needs a plan,
// whose arena the caller allocated; this entry point needs only the field arrays the caller already holds.
//
// Scratch: the per-block partial sums live in g_norm_scratch, a file-scope __device__ array of
// kNoAllocBlocks x 4 doubles (32 KiB) that every GPU loading the library holds until the process exits.
// Host code cannot use the symbol as a device address, so the first call on each device looks its address
// up with cudaGetSymbolAddress (with that device current) and caches it; that first call should come
// before any stream capture. Each call writes every partial it later reads, so nothing needs clearing
// between calls, but all calls share the one array: calls that overlap on the GPU (on different streams)
// race on it and must be serialised by the caller.
#include <algorithm>
#include <mutex>
#include <string>

#include "aux.cuh"
#include "internal.cuh"

namespace tfd {
void set_error(const std::string &msg);   // api.cu: message for tfd_last_error()
}

namespace {

constexpr int kNoAllocBlocks = 1024;
constexpr int kNoAllocThreads = 256;
constexpr long long kCellsPerThread = 256;
// Largest input: every block reduces at most kNoAllocThreads * kCellsPerThread cells.
constexpr long long kNoAllocMaxCells = (long long)kNoAllocBlocks * kNoAllocThreads * kCellsPerThread;

static __device__ __align__(256) double g_norm_scratch[kNoAllocBlocks * 4];

constexpr int kMaxDevices = 64;         // devices per process whose scratch address is cached
std::mutex g_symbol_mutex;
void *g_symbol_ptr[kMaxDevices] = {nullptr};

template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads) k_norm_partial(const T *__restrict__ E, const T *__restrict__ H,
                                                                  const T *__restrict__ inv_eps, int samples, long long cells,
                                                                  double *partial) {
    __shared__ double sh[3][kNoAllocThreads / 32];
    double energy = 0.0, peak = 0.0, nan_seen = 0.0;
    for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < cells;
         cell += (long long)gridDim.x * blockDim.x) {
        for (int c = 0; c < 3; ++c) {
            const double e = (double)E[cell * 3 + c], h = (double)H[cell * 3 + c];
            const double ie = (double)inv_eps[samples == 3 ? cell * 3 + c : cell];
            energy += e * e * (1.0 / ie) + h * h;
            if (isnan(e) || isnan(h)) nan_seen = 1.0;
            else peak = fmax(peak, fmax(fabs(e), fabs(h)));
        }
    }
    energy = tfd::warp_sum(energy);
    peak = tfd::warp_max(peak);
    nan_seen = tfd::warp_max(nan_seen);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sh[0][w] = energy; sh[1][w] = peak; sh[2][w] = nan_seen; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, q = 0.0;
        for (int k = 0; k < kNoAllocThreads / 32; ++k) {
            a += sh[0][k];
            b = fmax(b, sh[1][k]);
            q = fmax(q, sh[2][k]);
        }
        partial[4 * blockIdx.x] = a;
        partial[4 * blockIdx.x + 1] = b;
        partial[4 * blockIdx.x + 2] = q;
    }
}

__global__ void k_norm_final(const double *partial, int blocks, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double energy = 0.0, peak = 0.0, nan_seen = 0.0;
    for (int b = 0; b < blocks; ++b) {      // fixed order: the result does not depend on scheduling
        energy += partial[4 * b];
        peak = fmax(peak, partial[4 * b + 1]);
        nan_seen = fmax(nan_seen, partial[4 * b + 2]);
    }
    out[0] = energy;
    out[1] = nan_seen > 0.0 ? __longlong_as_double(0x7ff8000000000000LL) : peak;
}

int scratch_pointer(double **ptr) {
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess || device < 0) {
        tfd::set_error(std::string("tfd_field_norm_static: no current CUDA device: ") + cudaGetErrorString(e));
        return TFD_ERR_CUDA;
    }
    if (device >= kMaxDevices) {
        tfd::set_error("tfd_field_norm_static: device index " + std::to_string(device) + " exceeds the " +
                       std::to_string(kMaxDevices) + " devices whose scratch address this library caches");
        return TFD_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_symbol_mutex);
    if (!g_symbol_ptr[device]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_norm_scratch);
        if (e != cudaSuccess || !p) {
            tfd::set_error(std::string("tfd_field_norm_static: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return TFD_ERR_CUDA;
        }
        g_symbol_ptr[device] = p;
    }
    *ptr = (double *)g_symbol_ptr[device];
    return TFD_OK;
}

}  // namespace

extern "C" int tfd_field_norm_static(const void *E, const void *H, const void *inv_eps, int64_t cells, int32_t material_samples,
                                     int32_t precision, double *out, void *stream) {
    if (!E || !H || !inv_eps || !out) {
        tfd::set_error("tfd_field_norm_static: null argument");
        return TFD_ERR_INVALID;
    }
    if ((precision != 4 && precision != 8) || (material_samples != 1 && material_samples != 3) || cells < 0) {
        tfd::set_error("tfd_field_norm_static: precision must be 4 or 8, material_samples 1 or 3, cells >= 0");
        return TFD_ERR_INVALID;
    }
    if (cells > kNoAllocMaxCells) {
        tfd::set_error("tfd_field_norm_static: " + std::to_string(cells) + " cells exceed the static scratch limit of " +
                       std::to_string(kNoAllocMaxCells) + " cells; use tfd_diagnose on a plan");
        return TFD_ERR_INVALID;
    }
    double *scratch = nullptr;
    int rc = scratch_pointer(&scratch);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const long long per_block = (long long)kNoAllocThreads * kCellsPerThread;
    const int blocks = (int)std::max(1LL, std::min<long long>(kNoAllocBlocks, (cells + per_block - 1) / per_block));
    if (precision == 8)
        k_norm_partial<double><<<blocks, kNoAllocThreads, 0, s>>>((const double *)E, (const double *)H, (const double *)inv_eps,
                                                                  material_samples, cells, scratch);
    else
        k_norm_partial<float><<<blocks, kNoAllocThreads, 0, s>>>((const float *)E, (const float *)H, (const float *)inv_eps,
                                                                material_samples, cells, scratch);
    k_norm_final<<<1, 32, 0, s>>>(scratch, blocks, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        tfd::set_error(std::string("tfd_field_norm_static: launch failed: ") + cudaGetErrorString(e));
        return TFD_ERR_CUDA;
    }
    return TFD_OK;
}
