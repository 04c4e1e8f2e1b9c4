// Total-field / scattered-field boxes: the live incident line and the face corrections (one launch per family
// and step, all boxes of a plan in blockIdx.y).
//
// Threads [0, count) of a box advance its scalar incident line by the family's half step (CPML memory first,
// then the line field, then the soft drive on the E half step); threads [count, count + n) add the family's
// corrections to the grid's new field buffer: E[target] += weight * h_line[sample] after the E update (the
// line's old H: the E half step writes e only) and H[target] += weight * e_line[sample] after the H update
// (the line's new E: the H half step writes h only). Neither half step reads what it writes, so the line
// update and the corrections share the launch without ordering. Arithmetic in the field precision, in the
// reference order (torchfdtd/tfsf.py:125-176, torchfdtd/cuda_tfsf.py:19-49): psi = psi*b + c*diff;
// line -= factor*(diff + psi); field += weight*incident.
//
// The grid's E and H updates run as the split gather kernels (k_step_gather_e / k_step_gather_h) so that
// the E corrections land before the H update reads E.
#pragma once
#include "internal.cuh"

namespace tfd {

constexpr int kMaxTfsf = 4;
constexpr int kTfsfThreads = 256;

struct TfsfTarget {
    long long idx;               // element of the component array (internal layout)
    int comp;                    // component 0..2 of the family
    int sample;                  // incident-line cell
};

template <typename T>
struct TfsfBoxDev {
    int count, drive_at;
    int n[2];                    // corrections per family
    T fac[2];                    // line update factors: courant / index^2 (E), courant (H)
    T *e, *h, *pe, *ph;          // line state
    const T *b[2], *c[2];        // line CPML per family
    const T *drive;              // [steps]
    const TfsfTarget *tgt[2];
    const T *w[2];
};

template <typename T>
struct TfsfArgs {
    int boxes;
    TfsfBoxDev<T> box[kMaxTfsf];
    T *E[2][3], *H[2][3];
    const long long *counter;
    int steps;
};

template <typename T>
__global__ void __launch_bounds__(kTfsfThreads) k_tfsf(const __grid_constant__ TfsfArgs<T> a, int family) {
    const TfsfBoxDev<T> &b = a.box[blockIdx.y];
    const long long n = *a.counter;
    if (n >= a.steps) return;                   // past the plan's last step: a step is a no-op
    const int par = (int)(n & 1);
    const bool fwd = family == 1;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < b.count) {
        T diff, *psi, *line;
        if (fwd) {
            diff = i + 1 < b.count ? b.e[i + 1] - b.e[i] : T(0);
            psi = b.ph;
            line = b.h;
        } else {
            diff = i > 0 ? b.h[i] - b.h[i - 1] : T(0);
            psi = b.pe;
            line = b.e;
        }
        const T p = psi[i] * b.b[family][i] + b.c[family][i] * diff;
        psi[i] = p;
        T v = line[i] - b.fac[family] * (diff + p);
        if (!fwd && i == b.drive_at) v = v + b.drive[n];
        line[i] = v;
    } else if (i < b.count + b.n[family]) {
        const long long j = i - b.count;
        const TfsfTarget t = b.tgt[family][j];
        T *field = (fwd ? a.H : a.E)[par ^ 1][t.comp];
        const T *incident = fwd ? b.e : b.h;
        field[t.idx] = field[t.idx] + b.w[family][j] * incident[t.sample];
    }
}

}  // namespace tfd
