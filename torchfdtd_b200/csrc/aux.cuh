// Per-step monitor kernel and the layout conversion / diagnostics kernels.
#pragma once
#include "internal.cuh"

namespace tfd {

// ---- per-step observations ---------------------------------------------------------------
// Point traces (reference torchfdtd/solver.py:790-796) and the online DFT planes
// (reference torchfdtd/field_monitors.py:144-160, torchfdtd/cuda_monitors.py:68-120),
// then the step counter. Runs after the step kernel, on the new parity.
//
// Plane samples: sum over interpolation corners in corner order, in the field precision,
// times the window (apodization * dt * downsample mask). Accumulation is complex float64
// with the phase exp(i*omega*(n+1)) evaluated from the absolute step (never a recurrence),
// and exp(i*pi*f*dt) more for H samples, half a step later.
template <typename T>
struct MonitorArgs {
    T *field[6];                 // parity-0 component arrays (parity 1 = field[c] + count); null if not advanced
    long long count;
    int steps;
    long long *counter;
    unsigned *done;
    int n_traces;
    const TraceDev *traces;
    T *trace_out;                // [steps][n_traces]
    int n_planes;
    const PlaneDev *planes;
    int max_samples;             // max over planes of points*components, and the trace count
};

constexpr int kMonitorThreads = 256;
constexpr int kPhaseChunk = 256;

// Observations of step n for one plan: block (bx, by) of a (gx x ...) grid handles sample chunk bx of plane
// by; the blocks of row by = 0 also record the point traces, strided over the row.
template <typename T>
__device__ __forceinline__ void monitor_work(const MonitorArgs<T> &m, int bx, int by, long long n, int gx) {
    __shared__ double2 phase_e[kPhaseChunk], phase_h[kPhaseChunk];
    const long long shift = ((n + 1) & 1) ? m.count : 0;   // current (new) parity
    if (n >= m.steps) return;
    if (by == 0) {
        for (int k = bx * blockDim.x + threadIdx.x; k < m.n_traces; k += gx * blockDim.x) {
            const TraceDev t = m.traces[k];
            const T *base = m.field[3 * t.family + t.comp];   // null: a component 2D does not advance (zero)
            m.trace_out[n * m.n_traces + k] = base ? base[shift + t.offset] : T(0);
        }
    }
    if (by >= m.n_planes) return;
    const PlaneDev &pl = m.planes[by];
    const int samples = pl.points * pl.components;
    if (bx * (int)blockDim.x >= samples) return;          // uniform per block: no barrier below is skipped by part of it
    const int s = bx * blockDim.x + threadIdx.x;
    const T *win = (const T *)pl.window;
    double value = 0.0;
    int p = 0, c = 0;
    const bool live = s < samples;
    if (live) {
        p = s / pl.components;
        c = s % pl.components;
        const int comp = pl.comp[c];
        const T *f = m.field[comp];
        const T *w = (const T *)pl.weight + (long long)c * pl.corners * pl.points;
        const long long *cell = pl.cell + (long long)c * pl.corners * pl.points;
        T sum = T(0);
        if (f != nullptr) {
            f += shift;
            for (int k = 0; k < pl.corners; ++k)
                sum = sum + f[cell[(long long)k * pl.points + p]] * w[(long long)k * pl.points + p];
        }
        const T wv = win[(comp >= 3 ? m.steps : 0) + n];
        value = (double)(sum * wv);
    }
    const bool magnetic = live && pl.comp[c] >= 3;
    for (int f0 = 0; f0 < pl.frequencies; f0 += kPhaseChunk) {
        const int nf = min(kPhaseChunk, pl.frequencies - f0);
        __syncthreads();
        for (int f = threadIdx.x; f < nf; f += blockDim.x) {
            double si, co;
            sincos(pl.omega[f0 + f] * (double)(n + 1), &si, &co);
            const double hr = pl.half[2 * (f0 + f)], hi = pl.half[2 * (f0 + f) + 1];
            phase_e[f] = make_double2(co, si);
            phase_h[f] = make_double2(co * hr - si * hi, co * hi + si * hr);
        }
        __syncthreads();
        if (live) {
            for (int f = 0; f < nf; ++f) {
                const double2 ph = magnetic ? phase_h[f] : phase_e[f];
                double *acc = pl.acc + 2 * (((long long)(f0 + f) * pl.points + p) * pl.components + c);
                acc[0] += ph.x * value;
                acc[1] += ph.y * value;
            }
        }
    }
}

// The last block of a launch to finish advances the step counter; every block read it first.
__device__ __forceinline__ void finish_step(long long *counter, unsigned *done, long long n) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned total = gridDim.x * gridDim.y * gridDim.z;
        const unsigned prev = atomicAdd(done, 1u);
        if (prev == total - 1) {
            *done = 0;
            __threadfence();
            *counter = n + 1;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kMonitorThreads) k_monitor(const __grid_constant__ MonitorArgs<T> m) {
    const long long n = *m.counter;
    if (n >= m.steps) return;                  // past the plan's last step: no observation, the counter stays
    monitor_work(m, blockIdx.x, blockIdx.y, n, gridDim.x);
    finish_step(m.counter, m.done, n);
}

// Observations of every plan of a batch (plan = blockIdx.z), then the batch's shared step counter.
template <typename T>
__global__ void __launch_bounds__(kMonitorThreads) k_monitor_batch(const MonitorArgs<T> *__restrict__ args, long long *counter,
                                                                  unsigned *done) {
    const long long n = *counter;
    monitor_work(args[blockIdx.z], blockIdx.x, blockIdx.y, n, gridDim.x);
    finish_step(counter, done, n);
}

// ---- layout conversion ----------------------------------------------------------------------
// Reference layout: (nx, ny, nz, S) C order, z fastest. Internal: [S][nz][ny][pitch].
template <typename T>
__global__ void k_reference_to_internal(const T *__restrict__ src, int S, int nx, int ny, int nz, int pitch,
                                        T *d0, T *d1, T *d2) {
    const long long total = (long long)nx * ny * nz * S;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e % S);
        const long long cell = e / S;
        const int z = (int)(cell % nz);
        const int y = (int)((cell / nz) % ny);
        const int x = (int)(cell / ((long long)nz * ny));
        T *d = s == 0 ? d0 : (s == 1 ? d1 : d2);
        d[((long long)z * ny + y) * pitch + x] = src[e];
    }
}

// Permittivity in the reference layout to the internal inverse-permittivity arrays: 1 / eps by IEEE division
// (the host's values); *bad is set when a value is not finite or below 1.
template <typename T>
__global__ void k_permittivity_to_internal(const T *__restrict__ src, int S, int nx, int ny, int nz, int pitch, T *d0, T *d1,
                                           T *d2, int *bad) {
    const long long total = (long long)nx * ny * nz * S;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e % S);
        const long long cell = e / S;
        const int z = (int)(cell % nz);
        const int y = (int)((cell / nz) % ny);
        const int x = (int)(cell / ((long long)nz * ny));
        T *d = s == 0 ? d0 : (s == 1 ? d1 : d2);
        const T v = src[e];
        if (!(v >= T(1)) || !isfinite(v)) atomicExch(bad, 1);
        d[((long long)z * ny + y) * pitch + x] = T(1) / v;
    }
}

template <typename T>
__global__ void k_internal_to_reference(T *__restrict__ dst, int S, int nx, int ny, int nz, int pitch, const T *s0,
                                        const T *s1, const T *s2) {
    const long long total = (long long)nx * ny * nz * S;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e % S);
        const long long cell = e / S;
        const int z = (int)(cell % nz);
        const int y = (int)((cell / nz) % ny);
        const int x = (int)(cell / ((long long)nz * ny));
        const T *src = s == 0 ? s0 : (s == 1 ? s1 : s2);
        dst[e] = src == nullptr ? T(0) : src[((long long)z * ny + y) * pitch + x];
    }
}

// Field arrays of the parity the counter selects: [parity][6 components], a component that
// is not advanced (2D) has a null pointer and reads as zero / ignores writes.
template <typename T>
struct FieldSet { T *f[2][6]; };

// ---- tiled layout conversion ---------------------------------------------------------------------
// The reference layout is z (then sample) fastest, the internal one x fastest: converting is a transpose of
// (x, z) for every y. A block of kTileThreads takes a 32 x 32 (x, z) tile of one y row through shared memory,
// so both sides move in coalesced runs: internal rows of 32 x values, reference runs of 32 * S values per x.
// Used when nz >= kTileMinNz (below it a tile would be mostly empty); the grid-stride kernels above serve the
// rest. Arrays: [parity][sample], parity from *counter (or 0 without a counter); a null array reads as zero
// and ignores writes.
constexpr int kTile = 32;
constexpr int kTileThreads = 256;
constexpr int kTileMinNz = 16;
constexpr int kTileStride = kTile * (kTile + 1) + 1;          // per sample; +1 keeps the samples' banks apart

template <typename T>
struct TileArrays { T *p[2][3]; };

__device__ __forceinline__ void tile_coords(int nx, int nz, int &x0, int &z0, int &y) {
    const int tx = (nx + kTile - 1) / kTile, tz = (nz + kTile - 1) / kTile;
    int b = blockIdx.x;
    x0 = (b % tx) * kTile;
    b /= tx;
    z0 = (b % tz) * kTile;
    y = b / tz;
}

// Internal -> reference: dst (nx, ny, nz, S) from src[parity][s] ([nz][ny][pitch]).
template <typename T>
__global__ void __launch_bounds__(kTileThreads) k_to_reference_tiled(T *__restrict__ dst, const __grid_constant__ TileArrays<T> src,
                                                                    const long long *counter, int S, int nx, int ny, int nz,
                                                                    int pitch) {
    __shared__ T tile[3 * kTileStride];
    int x0, z0, y;
    tile_coords(nx, nz, x0, z0, y);
    const int par = counter ? (int)(*counter & 1) : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = kTileThreads / 32;
    const int x = x0 + lane;
    for (int s = 0; s < S; ++s) {
        const T *a = src.p[par][s];
        for (int zz = w; zz < kTile; zz += nw) {
            const int z = z0 + zz;
            tile[s * kTileStride + zz * (kTile + 1) + lane] = (a && z < nz && x < nx) ? a[((long long)z * ny + y) * pitch + x] : T(0);
        }
    }
    __syncthreads();
    const int run = min(kTile, nz - z0) * S;
    for (int xx = w; xx < kTile && x0 + xx < nx; xx += nw) {
        T *out = dst + (((long long)(x0 + xx) * ny + y) * nz + z0) * S;
        for (int q = lane; q < run; q += 32) {
            const int zz = q / S, s = q - zz * S;
            out[q] = tile[s * kTileStride + zz * (kTile + 1) + xx];
        }
    }
}

// Reference -> internal: dst[parity][s] from src (nx, ny, nz, S). INVERT: the source is the permittivity;
// 1 / eps (IEEE division) is stored and *bad set when a value is not finite or below 1.
template <typename T, bool INVERT>
__global__ void __launch_bounds__(kTileThreads) k_from_reference_tiled(const T *__restrict__ src, const __grid_constant__ TileArrays<T> dst,
                                                                      const long long *counter, int S, int nx, int ny, int nz,
                                                                      int pitch, int *bad) {
    __shared__ T tile[3 * kTileStride];
    int x0, z0, y;
    tile_coords(nx, nz, x0, z0, y);
    const int par = counter ? (int)(*counter & 1) : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = kTileThreads / 32;
    const int zn = min(kTile, nz - z0), run = zn * S;
    bool wrong = false;
    for (int xx = w; xx < kTile && x0 + xx < nx; xx += nw) {
        const T *in = src + (((long long)(x0 + xx) * ny + y) * nz + z0) * S;
        for (int q = lane; q < run; q += 32) {
            const int zz = q / S, s = q - zz * S;
            T v = in[q];
            if (INVERT) {
                wrong |= !(v >= T(1)) || !isfinite(v);
                v = T(1) / v;
            }
            tile[s * kTileStride + zz * (kTile + 1) + xx] = v;
        }
    }
    if (INVERT && wrong) atomicExch(bad, 1);
    __syncthreads();
    const int x = x0 + lane;
    if (x >= nx) return;
    for (int s = 0; s < S; ++s) {
        T *a = dst.p[par][s];
        if (!a) continue;
        for (int zz = w; zz < zn; zz += nw) a[((long long)(z0 + zz) * ny + y) * pitch + x] = tile[s * kTileStride + zz * (kTile + 1) + lane];
    }
}

// The largest |E| and whether any E or H value of the current parity is not finite. out[0]: the bit pattern of
// the largest |E| (non-negative values order like their bit patterns); out[1]: 1 when a value is NaN or
// infinite. Both start at zero.
template <typename T>
__global__ void k_field_check(const __grid_constant__ FieldSet<T> fs, long long count, const long long *counter,
                              unsigned long long *out) {
    const int par = (int)(*counter & 1);
    T peak = T(0);
    int bad = 0;
#pragma unroll 1
    for (int c = 0; c < 6; ++c) {
        const T *f = fs.f[par][c];
        if (f == nullptr) continue;
        for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count; e += (long long)gridDim.x * blockDim.x) {
            const T v = f[e];
            if (!isfinite(v)) bad = 1;
            else if (c < 3) peak = fmax(peak, fabs(v));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        peak = fmax(peak, __shfl_xor_sync(0xffffffffu, peak, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        const unsigned long long bits = sizeof(T) == 4 ? (unsigned long long)__float_as_uint((float)peak)
                                                       : (unsigned long long)__double_as_longlong((double)peak);
        atomicMax(&out[0], bits);
        if (bad) atomicOr(&out[1], 1ull);
    }
}

template <typename T>
__global__ void k_fields_to_reference(T *__restrict__ E, T *__restrict__ H, int nx, int ny, int nz, int pitch,
                                      const __grid_constant__ FieldSet<T> fs, const long long *counter) {
    const int par = (int)(*counter & 1);
    const long long total = (long long)nx * ny * nz * 3;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e % 3);
        const long long cell = e / 3;
        const int z = (int)(cell % nz);
        const int y = (int)((cell / nz) % ny);
        const int x = (int)(cell / ((long long)nz * ny));
        const long long i = ((long long)z * ny + y) * pitch + x;
        const T *a = fs.f[par][c], *b = fs.f[par][3 + c];
        if (E) E[e] = a ? a[i] : T(0);
        if (H) H[e] = b ? b[i] : T(0);
    }
}

template <typename T>
__global__ void k_reference_to_fields(const T *__restrict__ E, const T *__restrict__ H, int nx, int ny, int nz, int pitch,
                                      const __grid_constant__ FieldSet<T> fs, const long long *counter) {
    const int par = (int)(*counter & 1);
    const long long total = (long long)nx * ny * nz * 3;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e % 3);
        const long long cell = e / 3;
        const int z = (int)(cell % nz);
        const int y = (int)((cell / nz) % ny);
        const int x = (int)(cell / ((long long)nz * ny));
        const long long i = ((long long)z * ny + y) * pitch + x;
        T *a = fs.f[par][c], *b = fs.f[par][3 + c];
        if (a && E) a[i] = E[e];
        if (b && H) b[i] = H[e];
    }
}

// One plane of one component: dst[(u*nv + v)] over the two remaining axes in order.
template <typename T>
__global__ void k_slice(T *__restrict__ dst, const __grid_constant__ FieldSet<T> fs, int comp, int axis, int index, int nx,
                        int ny, int nz, int pitch, const long long *counter) {
    const int par = (int)(*counter & 1);
    const int n[3] = {nx, ny, nz};
    const int ua = axis == 0 ? 1 : 0, va = axis == 2 ? 1 : 2;
    const long long total = (long long)n[ua] * n[va];
    const T *f = fs.f[par][comp];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        int c[3];
        c[axis] = index;
        c[ua] = (int)(e / n[va]);
        c[va] = (int)(e % n[va]);
        dst[e] = f ? f[((long long)c[2] * ny + c[1]) * pitch + c[0]] : T(0);
    }
}

// CPML memories <-> the reference's memory_states order. One segment = one reference psi
// array: family f, axis a, term j, cells [lo, hi) on axis a, full extent elsewhere.
struct PsiSegment {
    long long offset;            // element offset in the concatenated reference vector
    int f, a, j, lo, hi;
};

template <typename T>
struct PsiArgs {
    int n_seg;
    PsiSegment seg[24];
    int n[3];
    int pitch;
    const int *row[2][3];
    int rows[2][3];
    T *psiE[2][3][2];
    T *psiH[3][2];
    const long long *counter;
};

template <typename T>
__global__ void k_psi_copy(T *vec, const __grid_constant__ PsiArgs<T> a, int to_reference) {
    const int s = blockIdx.y;
    const PsiSegment sg = a.seg[s];
    int ext[3] = {a.n[0], a.n[1], a.n[2]};
    ext[sg.a] = sg.hi - sg.lo;
    const long long total = (long long)ext[0] * ext[1] * ext[2];
    const int par = (int)(*a.counter & 1);
    T *psi = sg.f == 0 ? a.psiE[par][sg.a][sg.j] : a.psiH[sg.a][sg.j];
    const int R = a.rows[sg.f][sg.a];
    if (psi == nullptr) {   // a term of a 2D polarization this plan does not advance: identically zero
        if (to_reference)
            for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x)
                vec[sg.offset + e] = T(0);
        return;
    }
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        int c[3];
        c[2] = (int)(e % ext[2]);
        c[1] = (int)((e / ext[2]) % ext[1]);
        c[0] = (int)(e / ((long long)ext[2] * ext[1]));
        c[sg.a] += sg.lo;
        const int r = a.row[sg.f][sg.a][c[sg.a]];
        const long long p = sg.a == 0 ? ((long long)c[2] * a.n[1] + c[1]) * R + r
                          : sg.a == 1 ? ((long long)c[2] * R + r) * a.pitch + c[0]
                                      : ((long long)r * a.n[1] + c[1]) * a.pitch + c[0];
        if (to_reference) vec[sg.offset + e] = psi[p];
        else psi[p] = vec[sg.offset + e];
    }
}

// ---- divergence diagnostics (reference torchfdtd/run_control.py:127-159) -----------------
constexpr int kDiagThreads = 256;

template <typename T>
struct DiagArgs {
    FieldSet<T> fs;
    const T *inv_eps[3];
    int nx, ny, nz, pitch;
    const long long *counter;
    int n_psi;
    const T *psi[40];
    long long psi_len[40];
    const double *volume[3];     // per-axis cell widths over the reference step (nullptr: 1)
    // Incident lines of TFSF boxes: their E (times the background index) and H enter the norm with a weight.
    int n_lines;
    const T *line[8];
    int line_len[8];
    double line_factor[8], line_weight[8];
    // Dispersive states: per state P and Q ([poles][samples]); the norm adds (Q / cq_p)^2 + (P cp_p)^2 per pole,
    // weighed by the sample's volume (rounded to the field precision; nullptr: 1).
    int n_ade;
    const T *ade_P[kMaxAde], *ade_Q[kMaxAde];
    int ade_samples[kMaxAde], ade_poles[kMaxAde];
    double ade_cq[kMaxAde][kMaxPoles], ade_cp[kMaxAde][kMaxPoles];
    const double *ade_weight[kMaxAde];
    double *partial;             // [gridDim.x][4]
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <typename T>
__global__ void __launch_bounds__(kDiagThreads) k_diag(const __grid_constant__ DiagArgs<T> d) {
    // Per block: [0] sum of E^2/inv_eps + H^2, [1] max |E|,|H| over non-NaN values,
    // [2] 1 when every CPML memory is finite else 0, [3] 1 when a field value is NaN.
    __shared__ double sh[4][kDiagThreads / 32];
    const int par = (int)(*d.counter & 1);
    const long long cells = (long long)d.nx * d.ny * d.nz;
    double energy = 0.0, peak = 0.0, finite = 1.0, nan_seen = 0.0;
    const bool weighted = d.volume[0] || d.volume[1] || d.volume[2];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cells; e += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(e % d.nx);
        const long long i = (e / d.nx) * d.pitch + x;   // e / nx = z*ny + y
        // Cell volume in reference-step units, rounded to the field precision as the reference stores it.
        double vol = 1.0;
        if (weighted) {
            const int y = (int)((e / d.nx) % d.ny), z = (int)(e / ((long long)d.nx * d.ny));
            const double wx = d.volume[0] ? d.volume[0][x] : 1.0, wy = d.volume[1] ? d.volume[1][y] : 1.0,
                         wz = d.volume[2] ? d.volume[2][z] : 1.0;
            vol = (double)(T)((wx * wy) * wz);
        }
        for (int c = 0; c < 3; ++c) {
            const T *a = d.fs.f[par][c], *b = d.fs.f[par][3 + c];
            if (a) {
                const double v = (double)a[i];
                energy += v * v * ((weighted ? vol : 1.0) / (double)d.inv_eps[c][i]);
                if (isnan(v)) nan_seen = 1.0; else peak = fmax(peak, fabs(v));
            }
            if (b) {
                const double v = (double)b[i];
                energy += weighted ? v * v * vol : v * v;
                if (isnan(v)) nan_seen = 1.0; else peak = fmax(peak, fabs(v));
            }
        }
    }
    for (int k = 0; k < d.n_lines; ++k)
        for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < d.line_len[k]; e += (long long)gridDim.x * blockDim.x) {
            const double v = (double)d.line[k][e] * d.line_factor[k];
            energy += v * v * d.line_weight[k];
        }
    for (int k = 0; k < d.n_ade; ++k) {
        const int ns = d.ade_samples[k];
        for (int p = 0; p < d.ade_poles[k]; ++p)
            for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ns; e += (long long)gridDim.x * blockDim.x) {
                const double w = d.ade_weight[k] ? (double)(T)d.ade_weight[k][e] : 1.0;
                const double q = (double)d.ade_Q[k][p * ns + e] / d.ade_cq[k][p];
                const double v = (double)d.ade_P[k][p * ns + e] * d.ade_cp[k][p];
                energy += q * q * w;
                energy += v * v * w;
            }
    }
    for (int k = 0; k < d.n_psi; ++k)
        for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < d.psi_len[k]; e += (long long)gridDim.x * blockDim.x)
            if (!isfinite((double)d.psi[k][e])) finite = 0.0;
    energy = warp_sum(energy);
    peak = warp_max(peak);
    finite = -warp_max(-finite);
    nan_seen = warp_max(nan_seen);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { sh[0][w] = energy; sh[1][w] = peak; sh[2][w] = finite; sh[3][w] = nan_seen; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, c = 1.0, q = 0.0;
        for (int k = 0; k < kDiagThreads / 32; ++k) {
            a += sh[0][k];
            b = fmax(b, sh[1][k]);
            c = fmin(c, sh[2][k]);
            q = fmax(q, sh[3][k]);
        }
        d.partial[4 * blockIdx.x] = a;
        d.partial[4 * blockIdx.x + 1] = b;
        d.partial[4 * blockIdx.x + 2] = c;
        d.partial[4 * blockIdx.x + 3] = q;
    }
}

}  // namespace tfd
