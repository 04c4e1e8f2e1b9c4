// Internal types shared by the kernels and the C ABI of libtfdtd.
//
// Layout in HBM (owned by the library inside the caller's arena):
//   * every field component is its own array [nz][ny][pitch] (x fastest), pitch =
//     nx rounded up to 32 elements so that each x-row starts on a 128-byte line;
//   * E and H are double-buffered ("ping-pong"): step n reads parity n&1 and writes
//     parity (n+1)&1, so one fused kernel can advance E and H of a step without
//     cross-CTA hazards (a CTA recomputes, never re-reads, the E values it borrows
//     from its neighbours' cells);
//   * CPML memories exist only on slab rows: per (family, axis, curl term) one array
//     [nz][ny][R] (x slabs), [nz][R][pitch] (y slabs) or [R][ny][pitch] (z slabs),
//     R = rows in both slabs of that axis; E-family memories are double-buffered like
//     E (halo recomputation reads the old value), H-family ones are updated in place;
//   * per (family, axis) 1-D tables b, c, 1/kappa and a row map (slab row or -1).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tfdtd.h"

namespace tfd {

constexpr int kMaxSources = 16;
constexpr int kPitchAlign = 32;

// Curl terms of the reference (torchfdtd/boundaries.py:21-23), grouped by output
// component in the order the reference accumulates them:
// out 0: (axis 1, in 2, +), (axis 2, in 1, -)
// out 1: (axis 0, in 2, -), (axis 2, in 0, +)
// out 2: (axis 0, in 1, +), (axis 1, in 0, -)
// j is the term's position among the two terms of its axis (psi array index).
struct Term { int axis, in, sign, j; };
__host__ __device__ constexpr Term term_of(int out, int k) {
    return out == 0 ? (k == 0 ? Term{1, 2, +1, 0} : Term{2, 1, -1, 0})
         : out == 1 ? (k == 0 ? Term{0, 2, -1, 0} : Term{2, 0, +1, 1})
                    : (k == 0 ? Term{0, 1, +1, 1} : Term{1, 0, -1, 1});
}
// Input / output component of term j on axis a (reference CURL_TERMS[2a+j]).
__host__ __device__ constexpr int term_in(int a, int j) { return a == 0 ? (j == 0 ? 2 : 1) : a == 1 ? (j == 0 ? 2 : 0) : (j == 0 ? 1 : 0); }
__host__ __device__ constexpr int term_out(int a, int j) { return a == 0 ? (j == 0 ? 1 : 2) : a == 1 ? (j == 0 ? 0 : 2) : (j == 0 ? 0 : 1); }

struct SourceTerm {
    int family, comp;
    int lo[3], hi[3];
};

constexpr int kMaxAde = 8;
constexpr int kMaxPoles = 16;

// One dispersive material state on the device: samples [start, start + samples) of the plan's sample list,
// P and Q as [poles][samples], coefficients in the field precision.
template <typename T>
struct AdeDev {
    int start, samples, poles;
    T eps, ksum, denom;          // eps_inf, sum of k, the denominator eps_inf + k_sum
    const T *a, *d, *k;          // [poles]
    T *P, *Q;
};

template <typename T>
struct Grid {
    int n[3];
    int pitch;
    long long plane;             // ny * pitch
    long long count;             // nz * ny * pitch
    int steps;
    int active;                  // component bitmask
    T cn;                        // Courant number rounded to T
    int periodic[3];
    int pec_on[3];
    T pec_neg[3];                // -(pec factor), rounded to T
    T *E[2][3], *H[2][3];
    const T *inv_eps[3];
    // CPML tables per family (0 E, 1 H) and axis
    const T *cb[2][3], *cc[2][3], *ck[2][3];
    const int *row[2][3];
    int rows[2][3];
    // Nonuniform-mesh factors per family and axis, indexed by the updated cell (nullptr: uniform axis).
    const T *metric[2][3];
    T *psiE[2][3][2];            // [parity][axis][term j]
    T *psiH[3][2];               // [axis][term j]
    int n_src;
    SourceTerm src[kMaxSources];
    const T *src_values;         // [n_src][steps]
    // Dispersive materials: per E component the sample index of each cell (-1: none); nullptr without any.
    const int *ade_map[3];
    int n_ade;
    AdeDev<T> ade[kMaxAde];
    long long *counter;
    int *status;

    __host__ __device__ __forceinline__ long long psi_index(int a, int x, int y, int z, int r, int R) const {
        return a == 0 ? ((long long)z * n[1] + y) * R + r
             : a == 1 ? ((long long)z * R + r) * pitch + x
                      : ((long long)r * n[1] + y) * pitch + x;
    }
    __host__ __device__ __forceinline__ long long stride(int a) const { return a == 0 ? 1 : a == 1 ? (long long)pitch : plane; }
};

// Device status codes (reported through tfd_device_status).
enum : int { kStatusOk = 0, kStatusCounterRange = 1, kStatusPipelineTimeout = 2, kStatusBadStrip = 3, kStatusBarrierTimeout = 4 };

struct PlaneDev {
    int points, frequencies, components, corners, ne;
    int comp[6];
    const long long *cell;      // [components][corners][points] offsets into a component array
    const void *weight;         // T [components][corners][points]
    const double *omega;        // [frequencies]: 2*pi*f*dt
    const double *half;         // [frequencies][2]: exp(i*pi*f*dt)
    const void *window;         // T [2][steps]
    double *acc;                // [frequencies][points][components][2]
};

struct TraceDev { int family, comp; long long offset; };

}  // namespace tfd
