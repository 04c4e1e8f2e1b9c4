/*
 * CPU oracle of the fused Yee/CPML step in plain C + OpenMP
 * (TEST INFRASTRUCTURE and CPU baseline, not product code).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm load this library (oracle/_build/libyee_oracle.so), and only as the checker
 * or as the timed CPU baseline. It restates, per element and in the same
 * floating-point operation order, the reference CPU path
 * (torchfdtd/boundaries.py:363-438, torchfdtd/solver.py:778-797):
 *   E pass:  d = H[i]-H[i-1]; (nonuniform mesh) d = d*metric; (CPML) psi = psi*b + c*d; d = d*(1/kappa) + psi;
 *            acc = (0 + s0*d0) + s1*d1; E = E + (cn*inv_eps)*acc; then E sources;
 *   H pass:  d = E[i+1]-E[i] (periodic wrap / PEC ghost at the upper end), CPML,
 *            H = H - cn*acc; then H sources; then point traces.
 * Built with -ffp-contract=off so no multiply-add is fused: its results are
 * bitwise equal to the NumPy restatement (oracle/yee_oracle.py) and to the
 * reference. State layout is the reference's: E, H as (nx, ny, nz, 3) C order and
 * CPML memories in the reference's memory_states order and shapes.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct oc_segment { int32_t forward, axis, lo, hi; const double *b, *c, *inv_kappa; } oc_segment;
typedef struct oc_source { int32_t family, component, lo[3], hi[3]; const double *values; } oc_source;
typedef struct oc_trace { int32_t family, component, index[3]; } oc_trace;

typedef struct oc_desc {
    int32_t nx, ny, nz, steps, material_samples;
    double courant;
    int32_t periodic[3], pec_on[3];
    double pec_upper[3];
    int32_t n_segments;
    const oc_segment *segments;
    int32_t n_sources;
    const oc_source *sources;
    int32_t n_traces;
    const oc_trace *traces;
    /* nonuniform mesh: per family and axis n factors indexed by the updated cell, or NULL (uniform axis);
     * reference torchfdtd/boundaries.py:276-284,376-393 */
    const double *metric[2][3];
} oc_desc;

/* Curl terms grouped by output component, in reference accumulation order:
 * {axis, input component, sign, j (term index on its axis)}. */
static const int TERMS[3][2][4] = {
    {{1, 2, +1, 0}, {2, 1, -1, 0}},
    {{0, 2, -1, 0}, {2, 0, +1, 1}},
    {{0, 1, +1, 1}, {1, 0, -1, 1}},
};

/* Per (family, axis): which segment and local row a coordinate falls in (-1: none). */
typedef struct { int *seg, *local; int n_seg; int order[4]; } oc_rows;

static int build_rows(const oc_desc *d, oc_rows rows[2][3]) {
    const int n[3] = {d->nx, d->ny, d->nz};
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) {
            oc_rows *r = &rows[f][a];
            r->seg = (int *)malloc(sizeof(int) * n[a]);
            r->local = (int *)malloc(sizeof(int) * n[a]);
            if (!r->seg || !r->local) return -1;
            for (int i = 0; i < n[a]; ++i) r->seg[i] = r->local[i] = -1;
            r->n_seg = 0;
            for (int k = 0; k < d->n_segments; ++k) {
                const oc_segment *s = &d->segments[k];
                if (s->forward != f || s->axis != a) continue;
                for (int i = s->lo; i < s->hi; ++i) { r->seg[i] = k; r->local[i] = i - s->lo; }
            }
        }
    return 0;
}

static void free_rows(oc_rows rows[2][3]) {
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) { free(rows[f][a].seg); free(rows[f][a].local); }
}

/* psi pointer table: psi_of[f][a][j][segment index] = array in the reference order. */
#define OC_DEFINE(REAL, SUFFIX)                                                                                  \
int oc_run_##SUFFIX(const oc_desc *d, REAL *E, REAL *H, const REAL *inv_eps, REAL **psi, int64_t start, int32_t nsteps, \
                    REAL *traces, int32_t threads) {                                                             \
    const int nx = d->nx, ny = d->ny, nz = d->nz, S = d->material_samples;                                       \
    const int n[3] = {nx, ny, nz};                                                                               \
    const long long st[3] = {(long long)ny * nz * 3, (long long)nz * 3, 3};                                       \
    const REAL cn = (REAL)d->courant;                                                                            \
    REAL pec_neg[3];                                                                                             \
    for (int a = 0; a < 3; ++a) pec_neg[a] = (REAL)(-d->pec_upper[a]);                                           \
    oc_rows rows[2][3];                                                                                          \
    if (build_rows(d, rows)) return -1;                                                                          \
    /* coefficient tables rounded to REAL, as the reference stores them */                                        \
    REAL *cb[2][3], *cc[2][3], *ck[2][3], *mt[2][3];                                                             \
    for (int f = 0; f < 2; ++f)                                                                                  \
        for (int a = 0; a < 3; ++a) {                                                                            \
            mt[f][a] = NULL;                                                                                     \
            if (d->metric[f][a]) {                                                                               \
                mt[f][a] = (REAL *)calloc(n[a], sizeof(REAL));                                                   \
                for (int i = 0; i < n[a]; ++i) mt[f][a][i] = (REAL)d->metric[f][a][i];                           \
            }                                                                                                    \
            cb[f][a] = (REAL *)calloc(n[a], sizeof(REAL));                                                       \
            cc[f][a] = (REAL *)calloc(n[a], sizeof(REAL));                                                       \
            ck[f][a] = (REAL *)calloc(n[a], sizeof(REAL));                                                       \
            for (int i = 0; i < n[a]; ++i) {                                                                     \
                const int k = rows[f][a].seg[i];                                                                 \
                if (k < 0) continue;                                                                             \
                const oc_segment *s = &d->segments[k];                                                           \
                cb[f][a][i] = (REAL)s->b[i - s->lo];                                                             \
                cc[f][a][i] = (REAL)s->c[i - s->lo];                                                             \
                ck[f][a][i] = (REAL)s->inv_kappa[i - s->lo];                                                     \
            }                                                                                                    \
        }                                                                                                        \
    /* psi slot of (family, axis, term j, segment k) in the reference memory_states order */                      \
    int slot[2][3][2][12];                                                                                       \
    {                                                                                                            \
        int q = 0;                                                                                               \
        for (int f = 0; f < 2; ++f)                                                                              \
            for (int a = 0; a < 3; ++a)                                                                          \
                for (int j = 0; j < 2; ++j) {                                                                    \
                    if (n[a] == 1) continue;                                                                     \
                    int order[12], m = 0;                                                                        \
                    for (int k = 0; k < d->n_segments; ++k)                                                      \
                        if (d->segments[k].forward == f && d->segments[k].axis == a) order[m++] = k;             \
                    for (int x = 0; x < m; ++x) /* by lo */                                                       \
                        for (int y = x + 1; y < m; ++y)                                                          \
                            if (d->segments[order[y]].lo < d->segments[order[x]].lo) { int t = order[x]; order[x] = order[y]; order[y] = t; } \
                    for (int x = 0; x < m; ++x) slot[f][a][j][order[x]] = q++;                                   \
                }                                                                                                \
    }                                                                                                            \
    for (int32_t step = 0; step < nsteps; ++step) {                                                             \
        const int64_t nstep = start + step;                                                                      \
        /* ---- E pass ---- */                                                                                   \
        _Pragma("omp parallel for num_threads(threads) schedule(static)")                                        \
        for (int x = 0; x < nx; ++x)                                                                             \
            for (int y = 0; y < ny; ++y)                                                                         \
                for (int z = 0; z < nz; ++z) {                                                                   \
                    const int co[3] = {x, y, z};                                                                 \
                    const long long cell = ((long long)x * ny + y) * nz + z;                                     \
                    for (int c = 0; c < 3; ++c) {                                                                \
                        REAL acc = (REAL)0;                                                                      \
                        for (int t = 0; t < 2; ++t) {                                                            \
                            const int a = TERMS[c][t][0], in = TERMS[c][t][1], sg = TERMS[c][t][2], j = TERMS[c][t][3]; \
                            if (n[a] == 1) continue;                                                             \
                            REAL dd = (REAL)0;                                                                   \
                            if (co[a] > 0) {                                                                     \
                                dd = H[cell * 3 + in] - H[cell * 3 - st[a] + in];                                \
                                if (mt[0][a]) dd = dd * mt[0][a][co[a]];                                         \
                                const int k = rows[0][a].seg[co[a]];                                             \
                                if (k >= 0) {                                                                    \
                                    int e[3] = {nx, ny, nz}, q[3] = {x, y, z};                                   \
                                    e[a] = d->segments[k].hi - d->segments[k].lo;                                \
                                    q[a] = rows[0][a].local[co[a]];                                              \
                                    REAL *ps = psi[slot[0][a][j][k]] + ((long long)q[0] * e[1] + q[1]) * e[2] + q[2]; \
                                    const REAL mem = *ps * cb[0][a][co[a]] + cc[0][a][co[a]] * dd;               \
                                    *ps = mem;                                                                   \
                                    dd = dd * ck[0][a][co[a]] + mem;                                             \
                                }                                                                                \
                            } else if (d->periodic[a]) {                                                         \
                                dd = H[cell * 3 + in] - H[cell * 3 + (long long)(n[a] - 1) * st[a] + in];        \
                                if (mt[0][a]) dd = dd * mt[0][a][0];                                             \
                            }                                                                                    \
                            acc = acc + (sg > 0 ? dd : -dd);                                                     \
                        }                                                                                        \
                        const REAL ie = inv_eps[S == 3 ? cell * 3 + c : cell];                                   \
                        E[cell * 3 + c] = E[cell * 3 + c] + (cn * ie) * acc;                                     \
                    }                                                                                            \
                }                                                                                                \
        for (int s = 0; s < d->n_sources; ++s) {                                                                 \
            const oc_source *t = &d->sources[s];                                                                 \
            if (t->family != 0 || nstep >= d->steps) continue;                                                   \
            const REAL v = (REAL)t->values[nstep];                                                               \
            for (int x = t->lo[0]; x < t->hi[0]; ++x)                                                            \
                for (int y = t->lo[1]; y < t->hi[1]; ++y)                                                        \
                    for (int z = t->lo[2]; z < t->hi[2]; ++z) {                                                  \
                        const long long i = (((long long)x * ny + y) * nz + z) * 3 + t->component;               \
                        E[i] = E[i] + v;                                                                         \
                    }                                                                                            \
        }                                                                                                        \
        /* ---- H pass ---- */                                                                                   \
        _Pragma("omp parallel for num_threads(threads) schedule(static)")                                        \
        for (int x = 0; x < nx; ++x)                                                                             \
            for (int y = 0; y < ny; ++y)                                                                         \
                for (int z = 0; z < nz; ++z) {                                                                   \
                    const int co[3] = {x, y, z};                                                                 \
                    const long long cell = ((long long)x * ny + y) * nz + z;                                     \
                    for (int c = 0; c < 3; ++c) {                                                                \
                        REAL acc = (REAL)0;                                                                      \
                        for (int t = 0; t < 2; ++t) {                                                            \
                            const int a = TERMS[c][t][0], in = TERMS[c][t][1], sg = TERMS[c][t][2], j = TERMS[c][t][3]; \
                            if (n[a] == 1) continue;                                                             \
                            REAL dd = (REAL)0;                                                                   \
                            if (co[a] < n[a] - 1) {                                                              \
                                dd = E[cell * 3 + st[a] + in] - E[cell * 3 + in];                                \
                                if (mt[1][a]) dd = dd * mt[1][a][co[a]];                                         \
                                const int k = rows[1][a].seg[co[a]];                                             \
                                if (k >= 0) {                                                                    \
                                    int e[3] = {nx, ny, nz}, q[3] = {x, y, z};                                   \
                                    e[a] = d->segments[k].hi - d->segments[k].lo;                                \
                                    q[a] = rows[1][a].local[co[a]];                                              \
                                    REAL *ps = psi[slot[1][a][j][k]] + ((long long)q[0] * e[1] + q[1]) * e[2] + q[2]; \
                                    const REAL mem = *ps * cb[1][a][co[a]] + cc[1][a][co[a]] * dd;               \
                                    *ps = mem;                                                                   \
                                    dd = dd * ck[1][a][co[a]] + mem;                                             \
                                }                                                                                \
                            } else if (d->periodic[a]) {                                                         \
                                dd = E[cell * 3 - (long long)(n[a] - 1) * st[a] + in] - E[cell * 3 + in];        \
                                if (mt[1][a]) dd = dd * mt[1][a][co[a]];                                         \
                            } else if (d->pec_on[a]) {                                                           \
                                dd = pec_neg[a] * E[cell * 3 + in];                                              \
                            }                                                                                    \
                            acc = acc + (sg > 0 ? dd : -dd);                                                     \
                        }                                                                                        \
                        H[cell * 3 + c] = H[cell * 3 + c] - cn * acc;                                            \
                    }                                                                                            \
                }                                                                                                \
        for (int s = 0; s < d->n_sources; ++s) {                                                                 \
            const oc_source *t = &d->sources[s];                                                                 \
            if (t->family != 1 || nstep >= d->steps) continue;                                                   \
            const REAL v = (REAL)t->values[nstep];                                                               \
            for (int x = t->lo[0]; x < t->hi[0]; ++x)                                                            \
                for (int y = t->lo[1]; y < t->hi[1]; ++y)                                                        \
                    for (int z = t->lo[2]; z < t->hi[2]; ++z) {                                                  \
                        const long long i = (((long long)x * ny + y) * nz + z) * 3 + t->component;               \
                        H[i] = H[i] + v;                                                                         \
                    }                                                                                            \
        }                                                                                                        \
        if (traces && nstep < d->steps)                                                                          \
            for (int k = 0; k < d->n_traces; ++k) {                                                              \
                const oc_trace *t = &d->traces[k];                                                               \
                const long long i = (((long long)t->index[0] * ny + t->index[1]) * nz + t->index[2]) * 3 + t->component; \
                traces[nstep * d->n_traces + k] = t->family ? H[i] : E[i];                                       \
            }                                                                                                    \
    }                                                                                                            \
    for (int f = 0; f < 2; ++f)                                                                                  \
        for (int a = 0; a < 3; ++a) { free(cb[f][a]); free(cc[f][a]); free(ck[f][a]); free(mt[f][a]); }          \
    free_rows(rows);                                                                                             \
    return 0;                                                                                                    \
}

OC_DEFINE(float, f32)
OC_DEFINE(double, f64)
