// Persistent 2D TMz stepping for grids too small to fill the GPU in one step.
//
// A 320 x 240 TMz grid is about 2 MB of state: one fused strip step takes a few microseconds of work,
// less than the launch and dependency latency of the two launches per step (strips, observations)
// that the per-step path costs. Here one cooperative launch runs many steps: every warp walks the
// plan's strip table (interior strips on the lean path, the rest on the general path, as the per-step
// kernels do), a grid-wide barrier separates the steps, and the observations of step n - 1 (traces, DFT
// planes) are taken while step n computes: they read the parity step n - 1 wrote, step n writes the other
// one, and they finish before the barrier after step n, that is before step n + 1 overwrites what they
// read. The step counter is written once, at the end of the launch. The arithmetic per cell is the
// per-step kernels' (strip_interior / strip_general), so the fields are bitwise the same.
//
// The barrier is a generation counter with a bounded wait: a block that waits longer than about a
// second records kStatusBarrierTimeout in the device status word and the launch ends (all blocks give
// up within the same bound). The launch is cooperative, so all its blocks are resident together.
#pragma once
#include "aux.cuh"
#include "step2d.cuh"

namespace tfd {

constexpr int kGridWaitTries = 1 << 23;          // x ~128 ns sleep: about a second
constexpr unsigned kGridSleepNs = 128;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of a cooperative launch: bar[0] counts arrivals, bar[1] is the generation. Returns
// false (and records the timeout) when the wait runs out.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *status) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        const unsigned gen = ld_acquire_u32(bar + 1);
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            int it = 0;
            while (ld_acquire_u32(bar + 1) == gen) {
                if (++it > kGridWaitTries) {
                    good = 0;
                    atomicExch(status, kStatusBarrierTimeout);
                    break;
                }
                __nanosleep(kGridSleepNs);
            }
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Observations of step n, spread over the launch's blocks as the per-step observation kernel spreads them
// over its (mgx x mgy) grid.
template <typename T>
__device__ __forceinline__ void observe_step(const MonitorArgs<T> &m, int mgx, int mgy, long long n) {
    for (int b = blockIdx.x; b < mgx * mgy; b += gridDim.x) monitor_work(m, b % mgx, b / mgx, n, mgx);
}

// `count` steps of one 2D TMz plan: strips [0, interior) take the lean path, [interior, all) the general
// one; warps are strided over the table. bar: the plan's barrier words (the launcher zeroes them before
// every launch, so a launch that timed out leaves no stale arrival count to the next one).
template <typename T>
__global__ void __launch_bounds__(k2dThreads, 2) k_step2d_persistent(const Grid<T> *__restrict__ grids,
                                                                    const Tile2D *__restrict__ strips, int interior, int all,
                                                                    const __grid_constant__ MonitorArgs<T> m, int mgx, int mgy,
                                                                    int count, unsigned *bar) {
    const Grid<T> &g = grids[0];
    const long long n0 = *m.counter;
    const int lane = threadIdx.x & 31;
    const int warps_total = gridDim.x * k2dWarps;
    const int w0 = blockIdx.x * k2dWarps + (threadIdx.x >> 5);
    long long n = n0;
    for (int k = 0; k < count && n < m.steps; ++k, ++n) {
        const int par = (int)(n & 1);
        if (k > 0) observe_step(m, mgx, mgy, n - 1);
        for (int s = w0; s < all; s += warps_total) {
            const Tile2D st = strips[s];
            if (s < interior) {
                // The lean path reads x0-1, x0+31, y0-1 and y1 unchecked: refuse a strip that is not interior.
                if (st.kind != 1 || st.x0 < 1 || st.x0 + 31 > g.n[0] - 1 || st.y0 < 1 || st.y1 > g.n[1] - 1 || st.y1 < st.y0) {
                    if (lane == 0) atomicExch(g.status, kStatusBadStrip);
                    continue;
                }
                strip_interior(g, st, par, lane);
            } else {
                strip_general(g, st, n, par, lane);
            }
        }
        if (!grid_barrier(bar, g.status)) return;
    }
    if (n > n0) observe_step(m, mgx, mgy, n - 1);
    if (blockIdx.x == 0 && threadIdx.x == 0) *m.counter = n;
}

// `count` steps of a batch of 2D TMz plans of any sizes in one cooperative launch: the batch's strip table
// (interior strips of every member first) walked by all warps each step, a member whose run has ended skipped
// (its state stays that of its last step), the observations of every member for step n - 1 taken while step n
// computes (plan = work item / (mgx * mgy)), a bounded grid barrier between steps, and the batch's shared step
// counter written once at the end. Per strip the arithmetic is the per-step kernels' (strip_interior /
// strip_general), so the fields are bitwise the same as with one launch per step.
template <typename T>
__global__ void __launch_bounds__(k2dThreads, 2) k_step2d_batch_persistent(const Grid<T> *__restrict__ grids,
                                                                          const Tile2D *__restrict__ strips, int interior, int all,
                                                                          const MonitorArgs<T> *__restrict__ mons, int plans, int mgx,
                                                                          int mgy, long long *counter, int count, unsigned *bar,
                                                                          int *status) {
    const long long n0 = *counter;
    const int lane = threadIdx.x & 31;
    const int warps_total = gridDim.x * k2dWarps;
    const int w0 = blockIdx.x * k2dWarps + (threadIdx.x >> 5);
    const int items = plans * mgx * mgy;
    auto observe = [&](long long step) {
        for (int b = blockIdx.x; b < items; b += gridDim.x) {
            const int q = b / (mgx * mgy), r = b % (mgx * mgy);
            monitor_work(mons[q], r % mgx, r / mgx, step, mgx);
        }
    };
    long long n = n0;
    for (int k = 0; k < count; ++k, ++n) {
        const int par = (int)(n & 1);
        if (k > 0) observe(n - 1);
        for (int s = w0; s < all; s += warps_total) {
            const Tile2D st = strips[s];
            const Grid<T> &g = grids[st.grid];
            if (n >= g.steps) continue;                // this member has finished its run (warp-uniform)
            if (s < interior) {
                if (st.kind != 1 || st.x0 < 1 || st.x0 + 31 > g.n[0] - 1 || st.y0 < 1 || st.y1 > g.n[1] - 1 || st.y1 < st.y0) {
                    if (lane == 0) atomicExch(g.status, kStatusBadStrip);
                    continue;
                }
                strip_interior(g, st, par, lane);
            } else {
                strip_general(g, st, n, par, lane);
            }
        }
        if (!grid_barrier(bar, status)) return;
    }
    if (n > n0) observe(n - 1);
    if (blockIdx.x == 0 && threadIdx.x == 0) *counter = n;
}

}  // namespace tfd
