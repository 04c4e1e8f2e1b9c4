// C ABI of libtfdtd: arena layout, table upload, step dispatch, layout conversion and
// diagnostics. Declarations and the reference interfaces they replace: include/tfdtd.h.
#include <algorithm>
#include <memory>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "aux.cuh"
#include "internal.cuh"
#include "persist2d.cuh"
#include "step_gather.cuh"
#include "step_march.cuh"
#include "step2d.cuh"
#include "adjoint.cuh"
#include "cluster2d.cuh"
#include "tfsf.cuh"
#include <cudaTypedefs.h>

using namespace tfd;

namespace {

thread_local std::string g_error;

int fail(int code, const std::string &msg) {
    g_error = msg;
    return code;
}

#define TFD_CUDA(expr)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (expr);                                                                       \
        if (e_ != cudaSuccess) return fail(TFD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define TFD_CHECK(expr)      \
    do {                     \
        const int rc_ = (expr); \
        if (rc_) return rc_; \
    } while (0)

// A side stream and its fork/join events, so that the general strips run beside the interior strips.
struct SideStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    int create() {
        TFD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        TFD_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        TFD_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
        return TFD_OK;
    }
    ~SideStream() {
        if (stream) cudaStreamDestroy(stream);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
    }
};

constexpr int kMaskTM = 0x04 | 0x08 | 0x10;   // Ez, Hx, Hy
constexpr int kMaskTE = 0x01 | 0x02 | 0x20;   // Ex, Ey, Hz
constexpr int kMaskAll = 0x3F;
constexpr int kDiagBlocks = 296;

// Offsets start at 256: offset 0 means "not allocated" (a component 2D does not advance).
struct Bump {
    size_t off = 256;
    size_t take(size_t bytes) {
        const size_t o = (off + 255) & ~size_t(255);
        off = o + bytes;
        return o;
    }
};

struct PlaneLayout {
    size_t cell, weight, omega, half, window, acc;
};

struct AdeLayout {
    size_t state;                  // P then Q: 2 x poles x samples elements
    size_t coef;                   // a, d, k: 3 x poles elements
    size_t weight;                 // samples doubles (diagnostics), 0: unit
};

struct TfsfLayout {
    size_t line;                   // e, h, pe, ph: 4 x count elements
    size_t coef;                   // b_e, c_e, b_h, c_h: 4 x count elements
    size_t drive;                  // steps elements
    size_t tgt[2], w[2];           // corrections per family
};

struct Layout {
    int elem = 4;
    int pitch = 0;
    long long count = 0;           // elements per component array (one parity)
    size_t E[3], H[3];             // both parities, contiguous
    size_t inv[3];
    size_t cb[2][3], cc[2][3], ck[2][3], row[2][3];
    size_t metric[2][3];
    int rows[2][3];
    long long psi_len[2][3];
    size_t psiE[3][2], psiH[3][2];
    size_t src_values = 0, trace_tab = 0, trace_out = 0, plane_tab = 0;
    std::vector<PlaneLayout> planes;
    std::vector<TfsfLayout> tfsf;
    std::vector<AdeLayout> ade;
    size_t ade_map = 0;            // 3 x count int32 sample indices
    size_t volume[3];              // diagnostics cell volumes per axis (double), 0: unit
    size_t counter = 0, done = 0, status = 0, diag = 0, stage = 0;
    size_t grid_bar = 0;           // persistent 2D stepping: arrival count and generation
    size_t check = 0;              // tfd_set_permittivity / tfd_field_check results
    size_t grid_tab = 0, tile_tab = 0;   // 2D tile kernel: this plan's Grid struct and its tile table
    int tiles2d = 0, strip_rows = 8;
    size_t stage_bytes = 0;
    size_t psi_total = 0;          // elements of the reference psi vector
    size_t total = 0;
};

bool active(int mask, int bit) { return (mask >> bit) & 1; }

int validate(const tfd_desc *d) {
    if (d == nullptr) return fail(TFD_ERR_INVALID, "descriptor is null");
    if (d->abi_version != TFD_ABI_VERSION) return fail(TFD_ERR_INVALID, "descriptor ABI version mismatch");
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) return fail(TFD_ERR_INVALID, "grid extents must be positive");
    if (d->nx > 1000000 || d->ny > 1000000 || d->nz > 1000000) return fail(TFD_ERR_INVALID, "a grid axis may hold at most one million cells");
    if (d->precision != 4 && d->precision != 8) return fail(TFD_ERR_INVALID, "precision must be 4 (float32) or 8 (float64)");
    if (d->material_samples != 1 && d->material_samples != 3) return fail(TFD_ERR_INVALID, "material_samples must be 1 or 3");
    if (d->steps < 0) return fail(TFD_ERR_INVALID, "steps must be non-negative");
    if (!(d->courant > 0) || !std::isfinite(d->courant)) return fail(TFD_ERR_INVALID, "courant must be positive and finite");
    const int n[3] = {d->nx, d->ny, d->nz};
    const bool two_d = d->nz == 1;
    if (two_d) {
        if (d->components != kMaskTM && d->components != kMaskTE && d->components != kMaskAll)
            return fail(TFD_ERR_INVALID, "2D components must be TM (Ez,Hx,Hy), TE (Ex,Ey,Hz) or all six");
    } else if (d->components != kMaskAll) {
        return fail(TFD_ERR_INVALID, "3D grids advance all six components");
    }
    for (int a = 0; a < 3; ++a)
        for (int s = 0; s < 2; ++s)
            if (d->face[a][s] < TFD_FACE_PML || d->face[a][s] > TFD_FACE_PEC) return fail(TFD_ERR_UNSUPPORTED, "unsupported boundary kind");
    for (int a = 0; a < 3; ++a)
        if (n[a] > 1 && ((d->face[a][0] == TFD_FACE_PERIODIC) != (d->face[a][1] == TFD_FACE_PERIODIC)))
            return fail(TFD_ERR_INVALID, "periodic faces must be paired on an axis");
    if (d->n_segments < 0 || d->n_segments > 12 || (d->n_segments && !d->segments)) return fail(TFD_ERR_INVALID, "bad CPML segment list");
    for (int k = 0; k < d->n_segments; ++k) {
        const tfd_cpml_segment &s = d->segments[k];
        if (s.forward < 0 || s.forward > 1 || s.axis < 0 || s.axis > 2) return fail(TFD_ERR_INVALID, "bad CPML segment family/axis");
        if (n[s.axis] == 1) return fail(TFD_ERR_INVALID, "CPML segment on an invariant axis");
        const int lo_min = s.forward ? 0 : 1, hi_max = s.forward ? n[s.axis] - 1 : n[s.axis];
        if (s.lo < lo_min || s.hi > hi_max || s.lo >= s.hi) return fail(TFD_ERR_INVALID, "CPML segment outside the active derivative range");
        if (!s.b || !s.c || !s.inv_kappa) return fail(TFD_ERR_INVALID, "CPML segment coefficients missing");
        for (int q = 0; q < k; ++q) {
            const tfd_cpml_segment &o = d->segments[q];
            if (o.forward == s.forward && o.axis == s.axis && s.lo < o.hi && o.lo < s.hi)
                return fail(TFD_ERR_INVALID, "overlapping CPML segments");
        }
    }
    if (d->n_sources < 0 || d->n_sources > kMaxSources || (d->n_sources && !d->sources))
        return fail(TFD_ERR_INVALID, "at most 16 source terms are supported per plan");
    for (int k = 0; k < d->n_sources; ++k) {
        const tfd_source_term &s = d->sources[k];
        if (s.family < 0 || s.family > 1 || s.component < 0 || s.component > 2) return fail(TFD_ERR_INVALID, "bad source component");
        for (int a = 0; a < 3; ++a)
            if (s.lo[a] < 0 || s.hi[a] > n[a] || s.lo[a] >= s.hi[a]) return fail(TFD_ERR_INVALID, "source box outside the grid");
        if (d->steps > 0 && !s.values) return fail(TFD_ERR_INVALID, "source values missing");
    }
    if (d->n_traces < 0 || (d->n_traces && !d->traces)) return fail(TFD_ERR_INVALID, "bad trace list");
    for (int k = 0; k < d->n_traces; ++k) {
        const tfd_trace &t = d->traces[k];
        if (t.family < 0 || t.family > 1 || t.component < 0 || t.component > 2) return fail(TFD_ERR_INVALID, "bad trace component");
        for (int a = 0; a < 3; ++a)
            if (t.index[a] < 0 || t.index[a] >= n[a]) return fail(TFD_ERR_INVALID, "trace index outside the grid");
    }
    if (d->n_planes < 0 || d->n_planes > 65535 || (d->n_planes && !d->planes)) return fail(TFD_ERR_INVALID, "bad plane list");
    if (d->n_tfsf < 0 || d->n_tfsf > kMaxTfsf || (d->n_tfsf && !d->tfsf)) return fail(TFD_ERR_INVALID, "at most 4 TFSF boxes are supported per plan");
    if (d->n_ade < 0 || d->n_ade > kMaxAde || (d->n_ade && !d->ade)) return fail(TFD_ERR_INVALID, "at most 8 dispersive material states are supported per plan");
    for (int k = 0; k < d->n_ade; ++k) {
        const tfd_ade &m = d->ade[k];
        if (m.samples < 0 || m.poles < 1 || m.poles > kMaxPoles || (m.samples && !m.target) || !m.a || !m.d || !m.k || !m.w0 ||
            !m.strength || !(m.eps_inf > 0))
            return fail(TFD_ERR_INVALID, "bad dispersive material state");
        const long long cells = (long long)d->nx * d->ny * d->nz;
        for (int j = 0; j < m.samples; ++j)
            if (m.target[j] < 0 || m.target[j] >= 3 * cells || !active(d->components, (int)(m.target[j] % 3)))
                return fail(TFD_ERR_INVALID, "a dispersive sample lies outside the grid or on a component this plan does not advance");
    }
    for (int k = 0; k < d->n_tfsf; ++k) {
        const tfd_tfsf &t = d->tfsf[k];
        if (t.count < 2 || t.drive_at < 0 || t.drive_at >= t.count || !t.drive || !t.b[0] || !t.b[1] || !t.c[0] || !t.c[1])
            return fail(TFD_ERR_INVALID, "bad TFSF incident line");
        for (int f = 0; f < 2; ++f) {
            if (t.n_targets[f] < 0 || (t.n_targets[f] && (!t.target[f] || !t.sample[f] || !t.weight[f])))
                return fail(TFD_ERR_INVALID, "bad TFSF correction list");
            const long long cells = (long long)d->nx * d->ny * d->nz;
            for (int j = 0; j < t.n_targets[f]; ++j) {
                const int64_t q = t.target[f][j];
                if (q < 0 || q >= 3 * cells || t.sample[f][j] < 0 || t.sample[f][j] >= t.count)
                    return fail(TFD_ERR_INVALID, "a TFSF correction lies outside the grid or its incident line");
                if (!active(d->components, 3 * f + (int)(q % 3)))
                    return fail(TFD_ERR_INVALID, "a TFSF correction drives a component this plan does not advance");
            }
        }
    }
    const long long cells = (long long)n[0] * n[1] * n[2];
    for (int k = 0; k < d->n_planes; ++k) {
        const tfd_plane &p = d->planes[k];
        if (p.points < 0 || p.frequencies < 0 || p.components < 1 || p.components > 6 || p.corners < 1 || p.corners > 8)
            return fail(TFD_ERR_INVALID, "bad plane sizes");
        if ((long long)p.points * p.components > (1LL << 30)) return fail(TFD_ERR_INVALID, "plane too large");
        if (!p.component_ids || (p.points && (!p.corner_cells || !p.corner_weights)) || (p.frequencies && !p.frequency_hz) ||
            (d->steps && (!p.window_e || !p.window_h)))
            return fail(TFD_ERR_INVALID, "plane tables missing");
        int ne = 0;
        for (int c = 0; c < p.components; ++c) {
            const int id = p.component_ids[c];
            if (id < 0 || id > 5) return fail(TFD_ERR_INVALID, "bad plane component id");
            if (id < 3) {
                if (ne != c) return fail(TFD_ERR_INVALID, "plane E components must come first");
                ++ne;
            }
        }
        const long long entries = (long long)p.components * p.corners * p.points;
        for (long long e = 0; e < entries; ++e)
            if (p.corner_cells[e] < 0 || p.corner_cells[e] >= cells) return fail(TFD_ERR_INVALID, "plane corner outside the grid");
    }
    return TFD_OK;
}

// The segment order of the reference's memory_states: family, then CURL_TERMS order
// ((a, j) = (0,0),(0,1),(1,0),(1,1),(2,0),(2,1)), then side.
std::vector<PsiSegment> psi_segments(const tfd_desc *d, size_t *total) {
    const int n[3] = {d->nx, d->ny, d->nz};
    std::vector<PsiSegment> out;
    long long off = 0;
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 2; ++j) {
                if (n[a] == 1) continue;
                std::vector<const tfd_cpml_segment *> segs;
                for (int k = 0; k < d->n_segments; ++k)
                    if (d->segments[k].forward == f && d->segments[k].axis == a) segs.push_back(&d->segments[k]);
                std::sort(segs.begin(), segs.end(), [](auto *x, auto *y) { return x->lo < y->lo; });
                for (auto *s : segs) {
                    long long ext[3] = {n[0], n[1], n[2]};
                    ext[a] = s->hi - s->lo;
                    out.push_back(PsiSegment{off, f, a, j, s->lo, s->hi});
                    off += ext[0] * ext[1] * ext[2];
                }
            }
    *total = (size_t)off;
    return out;
}

// The 2D tile kernel runs 2D TMz grids whose x and y faces are PML or PEC.
bool tile2d_capable(const tfd_desc *d) {
    return d->nz == 1 && d->components == kMaskTM && d->face[0][0] != TFD_FACE_PERIODIC && d->face[1][0] != TFD_FACE_PERIODIC &&
           (long long)d->ny * ((d->nx + kPitchAlign - 1) / kPitchAlign * kPitchAlign) < (1LL << 31);
}

// What the strip table of a 2D grid depends on: its size, its CPML slabs and its source boxes.
struct StripGeom {
    int nx = 0, ny = 0;
    struct Slab { int family, axis, lo, hi; };
    std::vector<Slab> slabs;
    std::vector<SourceTerm> sources;
    bool metric = false;             // nonuniform mesh: every strip takes the general path
};

StripGeom strip_geom(const tfd_desc *d) {
    StripGeom G;
    G.nx = d->nx;
    G.ny = d->ny;
    for (int k = 0; k < d->n_segments; ++k)
        G.slabs.push_back({d->segments[k].forward, d->segments[k].axis, d->segments[k].lo, d->segments[k].hi});
    for (int k = 0; k < d->n_sources; ++k) {
        const tfd_source_term &t = d->sources[k];
        SourceTerm q{t.family, t.component, {t.lo[0], t.lo[1], t.lo[2]}, {t.hi[0], t.hi[1], t.hi[2]}};
        G.sources.push_back(q);
    }
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 2; ++a) G.metric = G.metric || d->metric[f][a] != nullptr;
    return G;
}

// Strips of one grid: rows split into a lower boundary band, an interior band and an upper boundary band
// (so that whole strips avoid the y slabs), each band cut into strips of `rows` rows, columns in steps of
// 31, x-fastest so that neighbouring strips (which share halo columns) run together. A strip is interior
// (kind 1) when all 32 columns and its rows, halo row included, avoid the grid edges, every CPML slab and
// every source box, on a uniform mesh; the kernel then runs the bare stencil.
std::vector<Tile2D> strips_of(const StripGeom &G, int grid_index, int rows) {
    const int nx = G.nx, ny = G.ny;
    int fb0 = 1, fb1 = ny - 1;                       // interior rows: y0 >= fb0 and halo row y1 <= fb1
    for (const auto &sl : G.slabs) {
        if (sl.axis != 1 || sl.hi <= sl.lo) continue;
        if (sl.lo + sl.hi < ny) fb0 = std::max(fb0, sl.hi);                         // lower slab
        else fb1 = std::min(fb1, sl.family == 0 ? sl.lo - 1 : sl.lo);                // upper slab (E rows up to y1, H up to y1-1)
    }
    std::vector<std::pair<int, int>> bands;
    if (fb1 > fb0) bands = {{0, fb0}, {fb0, fb1}, {fb1, ny}};
    else bands = {{0, ny}};
    auto x_interior = [&](int x0) {
        if (x0 < 1 || x0 + 31 > nx - 1) return false;
        for (const auto &sl : G.slabs) {
            if (sl.axis != 0 || sl.hi <= sl.lo) continue;
            const int last = sl.family == 0 ? x0 + 31 : x0 + 30;                    // E on all 32 lanes, H on 31
            if (sl.lo <= last && x0 < sl.hi) return false;
        }
        return true;
    };
    auto no_source = [&](int x0, int y0, int y1) {
        for (const auto &q : G.sources) {
            const int xe = q.family == 0 ? x0 + 32 : x0 + k2dOwnX, ye = q.family == 0 ? y1 + 1 : y1;
            if (q.lo[0] < xe && x0 < q.hi[0] && q.lo[1] < ye && y0 < q.hi[1]) return false;
        }
        return true;
    };
    std::vector<Tile2D> t;
    for (size_t b = 0; b < bands.size(); ++b) {
        const bool inner = bands.size() == 3 && b == 1;
        for (int y0 = bands[b].first; y0 < bands[b].second; y0 += rows) {
            const int y1 = std::min(y0 + rows, bands[b].second);
            for (int x0 = 0; x0 < nx; x0 += k2dOwnX) {
                const int kind = inner && !G.metric && x_interior(x0) && no_source(x0, y0, y1) ? 1 : 0;
                t.push_back(Tile2D{grid_index, x0, y0, y1, kind});
            }
        }
    }
    // Interior strips first: the lean kernel walks [0, interior), the general kernel the rest.
    std::stable_partition(t.begin(), t.end(), [](const Tile2D &a) { return a.kind == 1; });
    return t;
}

int interior_count(const std::vector<Tile2D> &t) {
    return (int)std::count_if(t.begin(), t.end(), [](const Tile2D &a) { return a.kind == 1; });
}

// Upper bound of the strip count of a grid for strips of at least 8 rows (two band edges add two cuts).
int strip_capacity(int nx, int ny) { return ((nx + k2dOwnX - 1) / k2dOwnX) * ((ny + 7) / 8 + 2); }

// 2D TMz grids up to this many cells step in one persistent launch (see setup_tile2d), over strips of
// persist2d_strip_rows() rows. TFD_PERSIST2D=0/1 and TFD_PERSIST_ROWS in the environment override both,
// for sweeps.
constexpr long long kPersist2dMaxCells = 1LL << 19;
constexpr int kPersist2dStripRows = 4;

inline bool persist2d_eligible(long long cells) {
    const char *env = getenv("TFD_PERSIST2D");
    return env ? std::atoi(env) != 0 : cells <= kPersist2dMaxCells;
}

inline int persist2d_strip_rows() {
    const char *env = getenv("TFD_PERSIST_ROWS");
    const int rows = env ? std::atoi(env) : 0;
    return rows >= 1 ? rows : kPersist2dStripRows;
}

void compute_layout(const tfd_desc *d, Layout &L) {
    Bump b;
    const int n[3] = {d->nx, d->ny, d->nz};
    L.elem = d->precision;
    L.pitch = (d->nx + kPitchAlign - 1) / kPitchAlign * kPitchAlign;
    L.count = (long long)d->nz * d->ny * L.pitch;
    L.count = (L.count + 63) / 64 * 64;          // parity-1 arrays stay 256-byte aligned
    const size_t comp_bytes = (size_t)L.count * L.elem;
    for (int c = 0; c < 3; ++c) {
        L.E[c] = active(d->components, c) ? b.take(2 * comp_bytes) : 0;
        L.H[c] = active(d->components, 3 + c) ? b.take(2 * comp_bytes) : 0;
    }
    for (int s = 0; s < 3; ++s) L.inv[s] = s < d->material_samples ? b.take(comp_bytes) : 0;
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) L.metric[f][a] = (d->metric[f][a] && n[a] > 1) ? b.take((size_t)n[a] * L.elem) : 0;
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) {
            int rows = 0;
            for (int k = 0; k < d->n_segments; ++k)
                if (d->segments[k].forward == f && d->segments[k].axis == a) rows += d->segments[k].hi - d->segments[k].lo;
            L.rows[f][a] = rows;
            L.cb[f][a] = L.cc[f][a] = L.ck[f][a] = L.row[f][a] = 0;
            L.psi_len[f][a] = 0;
            if (rows == 0) continue;
            L.cb[f][a] = b.take((size_t)n[a] * L.elem);
            L.cc[f][a] = b.take((size_t)n[a] * L.elem);
            L.ck[f][a] = b.take((size_t)n[a] * L.elem);
            L.row[f][a] = b.take((size_t)n[a] * sizeof(int));
            L.psi_len[f][a] = a == 0 ? (long long)n[2] * n[1] * rows
                            : a == 1 ? (long long)n[2] * rows * L.pitch
                                     : (long long)rows * n[1] * L.pitch;
        }
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 2; ++j) {
            L.psiE[a][j] = L.psi_len[0][a] && active(d->components, term_out(a, j))
                               ? b.take(2 * (size_t)((L.psi_len[0][a] + 63) / 64 * 64) * L.elem) : 0;
            L.psiH[a][j] = L.psi_len[1][a] && active(d->components, 3 + term_out(a, j))
                               ? b.take((size_t)L.psi_len[1][a] * L.elem) : 0;
        }
    L.src_values = b.take((size_t)std::max(1, d->n_sources) * std::max(1, d->steps) * L.elem);
    L.trace_tab = b.take((size_t)std::max(1, d->n_traces) * sizeof(TraceDev));
    L.trace_out = b.take((size_t)std::max(1, d->n_traces) * std::max(1, d->steps) * L.elem);
    L.plane_tab = b.take((size_t)std::max(1, d->n_planes) * sizeof(PlaneDev));
    size_t largest_plane = 0;
    L.planes.resize(d->n_planes);
    for (int k = 0; k < d->n_planes; ++k) {
        const tfd_plane &p = d->planes[k];
        const size_t entries = (size_t)p.components * p.corners * p.points;
        PlaneLayout &q = L.planes[k];
        q.cell = b.take(std::max<size_t>(1, entries) * sizeof(long long));
        q.weight = b.take(std::max<size_t>(1, entries) * L.elem);
        q.omega = b.take(std::max<size_t>(1, p.frequencies) * sizeof(double));
        q.half = b.take(std::max<size_t>(1, p.frequencies) * 2 * sizeof(double));
        q.window = b.take(2 * (size_t)std::max(1, d->steps) * L.elem);
        const size_t acc = (size_t)p.frequencies * p.points * p.components * 2 * sizeof(double);
        q.acc = b.take(std::max<size_t>(1, acc));
        largest_plane = std::max(largest_plane, acc);
    }
    L.tfsf.resize(d->n_tfsf);
    for (int k = 0; k < d->n_tfsf; ++k) {
        const tfd_tfsf &t = d->tfsf[k];
        TfsfLayout &q = L.tfsf[k];
        q.line = b.take((size_t)4 * t.count * L.elem);
        q.coef = b.take((size_t)4 * t.count * L.elem);
        q.drive = b.take((size_t)std::max(1, d->steps) * L.elem);
        for (int f = 0; f < 2; ++f) {
            q.tgt[f] = b.take(std::max<size_t>(1, t.n_targets[f]) * sizeof(TfsfTarget));
            q.w[f] = b.take(std::max<size_t>(1, t.n_targets[f]) * L.elem);
        }
    }
    for (int a = 0; a < 3; ++a) L.volume[a] = d->volume[a] ? b.take((size_t)n[a] * sizeof(double)) : 0;
    L.ade.resize(d->n_ade);
    L.ade_map = d->n_ade > 0 ? b.take((size_t)3 * L.count * sizeof(int)) : 0;
    for (int k = 0; k < d->n_ade; ++k) {
        const tfd_ade &m = d->ade[k];
        L.ade[k].state = b.take(std::max<size_t>(1, (size_t)2 * m.poles * m.samples) * L.elem);
        L.ade[k].coef = b.take((size_t)3 * m.poles * L.elem);
        L.ade[k].weight = m.weight ? b.take(std::max<size_t>(1, m.samples) * sizeof(double)) : 0;
    }
    if (tile2d_capable(d)) {
        L.strip_rows = persist2d_eligible((long long)d->nx * d->ny) ? persist2d_strip_rows() : strip_rows((long long)d->nx * d->ny);
        L.tiles2d = (int)strips_of(strip_geom(d), 0, L.strip_rows).size();
        L.grid_tab = b.take(std::max(sizeof(Grid<float>), sizeof(Grid<double>)));
        L.tile_tab = b.take((size_t)L.tiles2d * sizeof(Tile2D));
    }
    L.counter = b.take(sizeof(long long));
    L.done = b.take(sizeof(unsigned));
    L.grid_bar = b.take(2 * sizeof(unsigned));
    L.check = b.take(4 * sizeof(unsigned long long));
    L.status = b.take(sizeof(int));
    L.diag = b.take((size_t)kDiagBlocks * 4 * sizeof(double));
    psi_segments(d, &L.psi_total);
    const long long cells = (long long)n[0] * n[1] * n[2];
    L.stage_bytes = std::max({(size_t)cells * 3 * L.elem, L.psi_total * L.elem, largest_plane,
                              (size_t)std::max(1, d->n_traces) * std::max(1, d->steps) * L.elem, (size_t)256});
    L.stage = b.take(L.stage_bytes);
    L.total = b.off + 256;
}

}  // namespace

namespace tfd {
void set_error(const std::string &msg) { g_error = msg; }
}  // namespace tfd

struct tfd_plan {
    tfd_desc desc;               // sizes and flags only; host pointers are not kept
    Layout L;
    char *arena = nullptr;
    Grid<float> gf;
    Grid<double> gd;
    int kernel = TFD_KERNEL_GATHER;
    std::vector<PsiSegment> psi_segs;
    std::vector<int> planes_f, planes_p, planes_c;
    int max_samples = 0;
    MarchArgs<float> mf;
    MarchArgs<double> md;
    dim3 march_grid;
    size_t march_smem = 0;
    struct MarchLaunch { int mode; dim3 grid; int tx_off, ty_off, lz, z_lo, z_hi; };   // mode 3: the mixed kernel
    MarchMix march_mix{};
    std::vector<MarchLaunch> march_launches;
    bool march_metric = false;     // nonuniform mesh: the general body with metric factors
    TfsfArgs<float> tf{};          // TFSF boxes (the step runs the split gather kernels when there are any)
    TfsfArgs<double> td{};
    double tfsf_index[kMaxTfsf] = {}, tfsf_norm[kMaxTfsf] = {};   // diagnostics: background index, norm weight
    bool split = false;            // TFSF boxes or dispersive materials: the split gather step
    // Diagnostics of the dispersive states: per state and pole the divisors of Q and the factors of P.
    std::vector<std::vector<double>> ade_cq, ade_cp;
    template <typename T> TfsfArgs<T> &tfsf();
    // Boundary strips run on auxiliary streams, forked from and joined back to the caller's stream
    // (a CUDA graph capture records them as parallel branches).
    std::vector<cudaStream_t> aux;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    ~tfd_plan() {
        for (auto st : aux) cudaStreamDestroy(st);
        for (auto ev : join) cudaEventDestroy(ev);
        if (fork) cudaEventDestroy(fork);
    }
    int march_variant = 42;
    int tile2d_interior = 0;
    int persist_ctas = 0;          // > 0: 2D steps run as one persistent cooperative launch of this many CTAs
    Cluster2D cluster2d{};         // ranks > 0: 2D steps run on chip in one thread-block cluster
    size_t cluster2d_smem = 0;
    std::unique_ptr<SideStream> side2d;
    bool in_batch = false;
    long long *own_counter = nullptr;
    std::vector<int> seg_f, seg_a, seg_lo, seg_hi;

    template <typename T> Grid<T> &grid();
    template <typename T> MarchArgs<T> &march();
    template <typename T> T *ptr(size_t off) const { return off ? (T *)(arena + off) : nullptr; }
};
template <> Grid<float> &tfd_plan::grid<float>() { return gf; }
template <> Grid<double> &tfd_plan::grid<double>() { return gd; }
template <> MarchArgs<float> &tfd_plan::march<float>() { return mf; }
template <> MarchArgs<double> &tfd_plan::march<double>() { return md; }
template <> TfsfArgs<float> &tfd_plan::tfsf<float>() { return tf; }
template <> TfsfArgs<double> &tfd_plan::tfsf<double>() { return td; }

namespace {

template <typename T>
__global__ void k_fill(T *p, long long n, T v) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) p[e] = v;
}

int launch_blocks(long long work, int threads = 256) {
    long long b = (work + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, 148LL * 32));
}

template <typename T>
int upload(cudaStream_t s, tfd_plan *p, size_t off, const std::vector<T> &v) {
    if (v.empty()) return TFD_OK;
    TFD_CUDA(cudaMemcpyAsync(p->arena + off, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return TFD_OK;
}

template <typename T>
int create_typed(tfd_plan *p, const tfd_desc *d, cudaStream_t s) {
    const Layout &L = p->L;
    Grid<T> &g = p->grid<T>();
    std::memset(&g, 0, sizeof(g));
    const int n[3] = {d->nx, d->ny, d->nz};
    for (int a = 0; a < 3; ++a) g.n[a] = n[a];
    g.pitch = L.pitch;
    g.plane = (long long)d->ny * L.pitch;
    g.count = L.count;
    g.steps = d->steps;
    g.active = d->components;
    g.cn = (T)d->courant;
    for (int a = 0; a < 3; ++a) {
        g.periodic[a] = n[a] > 1 && d->face[a][0] == TFD_FACE_PERIODIC;
        g.pec_on[a] = n[a] > 1 && !g.periodic[a] && d->face[a][1] == TFD_FACE_PEC;
        g.pec_neg[a] = (T)(-d->pec_upper[a]);
    }
    for (int par = 0; par < 2; ++par)
        for (int c = 0; c < 3; ++c) {
            g.E[par][c] = L.E[c] ? p->ptr<T>(L.E[c]) + par * L.count : nullptr;
            g.H[par][c] = L.H[c] ? p->ptr<T>(L.H[c]) + par * L.count : nullptr;
        }
    for (int c = 0; c < 3; ++c) g.inv_eps[c] = p->ptr<T>(L.inv[d->material_samples == 3 ? c : 0]);
    // CPML tables
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) {
            g.rows[f][a] = L.rows[f][a];
            if (!L.rows[f][a]) continue;
            std::vector<T> vb(n[a], T(0)), vc(n[a], T(0)), vk(n[a], T(1));
            std::vector<int> vr(n[a], -1);
            std::vector<const tfd_cpml_segment *> segs;
            for (int k = 0; k < d->n_segments; ++k)
                if (d->segments[k].forward == f && d->segments[k].axis == a) segs.push_back(&d->segments[k]);
            std::sort(segs.begin(), segs.end(), [](auto *x, auto *y) { return x->lo < y->lo; });
            int r = 0;
            for (auto *sg : segs)
                for (int i = sg->lo; i < sg->hi; ++i) {
                    vb[i] = (T)sg->b[i - sg->lo];
                    vc[i] = (T)sg->c[i - sg->lo];
                    vk[i] = (T)sg->inv_kappa[i - sg->lo];
                    vr[i] = r++;
                }
            int rc;
            if ((rc = upload(s, p, L.cb[f][a], vb)) || (rc = upload(s, p, L.cc[f][a], vc)) || (rc = upload(s, p, L.ck[f][a], vk)) ||
                (rc = upload(s, p, L.row[f][a], vr)))
                return rc;
            g.cb[f][a] = p->ptr<T>(L.cb[f][a]);
            g.cc[f][a] = p->ptr<T>(L.cc[f][a]);
            g.ck[f][a] = p->ptr<T>(L.ck[f][a]);
            g.row[f][a] = p->ptr<int>(L.row[f][a]);
        }
    // TFSF boxes: line coefficients and drive rounded to T, corrections with internal element indices
    {
        TfsfArgs<T> &ta = p->tfsf<T>();
        std::memset(&ta, 0, sizeof(ta));
        ta.boxes = d->n_tfsf;
        ta.steps = d->steps;
        for (int k = 0; k < d->n_tfsf; ++k) {
            const tfd_tfsf &t = d->tfsf[k];
            p->tfsf_index[k] = t.index;
            p->tfsf_norm[k] = t.norm_weight;
            const TfsfLayout &q = L.tfsf[k];
            TfsfBoxDev<T> &bx = ta.box[k];
            bx.count = t.count;
            bx.drive_at = t.drive_at;
            bx.fac[0] = (T)t.courant_e;
            bx.fac[1] = (T)t.courant_h;
            T *line = p->ptr<T>(q.line);
            bx.e = line;
            bx.h = line + t.count;
            bx.pe = line + 2 * t.count;
            bx.ph = line + 3 * t.count;
            std::vector<T> coef((size_t)4 * t.count);
            for (int f = 0; f < 2; ++f)
                for (int i = 0; i < t.count; ++i) {
                    coef[(size_t)(2 * f) * t.count + i] = (T)t.b[f][i];
                    coef[(size_t)(2 * f + 1) * t.count + i] = (T)t.c[f][i];
                }
            if (int rc = upload(s, p, q.coef, coef)) return rc;
            const T *cp = p->ptr<T>(q.coef);
            for (int f = 0; f < 2; ++f) {
                bx.b[f] = cp + (size_t)(2 * f) * t.count;
                bx.c[f] = cp + (size_t)(2 * f + 1) * t.count;
            }
            std::vector<T> drive((size_t)std::max(1, d->steps), T(0));
            for (int i = 0; i < d->steps; ++i) drive[i] = (T)t.drive[i];
            if (int rc = upload(s, p, q.drive, drive)) return rc;
            bx.drive = p->ptr<T>(q.drive);
            for (int f = 0; f < 2; ++f) {
                std::vector<TfsfTarget> tg(t.n_targets[f]);
                std::vector<T> w(t.n_targets[f]);
                for (int j = 0; j < t.n_targets[f]; ++j) {
                    const long long cell = t.target[f][j] / 3;
                    const int x = (int)(cell / ((long long)n[1] * n[2])), y = (int)((cell / n[2]) % n[1]), z = (int)(cell % n[2]);
                    tg[j].idx = (long long)z * g.plane + (long long)y * L.pitch + x;
                    tg[j].comp = (int)(t.target[f][j] % 3);
                    tg[j].sample = (int)t.sample[f][j];
                    w[j] = (T)t.weight[f][j];
                }
                if (int rc = upload(s, p, q.tgt[f], tg)) return rc;
                if (int rc = upload(s, p, q.w[f], w)) return rc;
                bx.n[f] = t.n_targets[f];
                bx.tgt[f] = p->ptr<TfsfTarget>(q.tgt[f]);
                bx.w[f] = p->ptr<T>(q.w[f]);
            }
        }
    }
    for (int a = 0; a < 3; ++a)
        if (L.volume[a]) {
            std::vector<double> v(d->volume[a], d->volume[a] + n[a]);
            if (int rc = upload(s, p, L.volume[a], v)) return rc;
        }
    // dispersive materials: the per-component sample map, pole coefficients, states (zeroed by zero_state)
    g.n_ade = d->n_ade;
    for (int c = 0; c < 3; ++c) g.ade_map[c] = nullptr;
    if (d->n_ade > 0) {
        std::vector<int> map((size_t)3 * L.count, -1);
        int start = 0;
        for (int k = 0; k < d->n_ade; ++k) {
            const tfd_ade &m = d->ade[k];
            AdeDev<T> &st = g.ade[k];
            st.start = start;
            st.samples = m.samples;
            st.poles = m.poles;
            for (int j = 0; j < m.samples; ++j) {
                const long long cell = m.target[j] / 3;
                const int comp = (int)(m.target[j] % 3);
                const int x = (int)(cell / ((long long)n[1] * n[2])), y = (int)((cell / n[2]) % n[1]), z = (int)(cell % n[2]);
                int &slot = map[(size_t)comp * L.count + (size_t)z * g.plane + (size_t)y * L.pitch + x];
                if (slot >= 0) return fail(TFD_ERR_INVALID, "dispersive material states overlap");
                slot = start + j;
            }
            start += m.samples;
            std::vector<T> coef((size_t)3 * m.poles);
            T ksum = T(0);
            for (int q = 0; q < m.poles; ++q) {
                coef[q] = (T)m.a[q];
                coef[m.poles + q] = (T)m.d[q];
                coef[2 * m.poles + q] = (T)m.k[q];
                ksum = q == 0 ? (T)m.k[0] : ksum + (T)m.k[q];
            }
            st.eps = (T)m.eps_inf;
            st.ksum = ksum;
            // One pole: eps_inf + k added in float64 and rounded once; several: summed in the field precision.
            st.denom = m.multiple ? (T)m.eps_inf + ksum : (T)(m.eps_inf + m.k[0]);
            if (int rc = upload(s, p, L.ade[k].coef, coef)) return rc;
            const T *cp = p->ptr<T>(L.ade[k].coef);
            st.a = cp;
            st.d = cp + m.poles;
            st.k = cp + 2 * m.poles;
            st.P = p->ptr<T>(L.ade[k].state);
            st.Q = st.P + (size_t)m.poles * m.samples;
            if (L.ade[k].weight) {
                std::vector<double> w(m.weight, m.weight + m.samples);
                if (int rc = upload(s, p, L.ade[k].weight, w)) return rc;
            }
        }
        if (int rc = upload(s, p, L.ade_map, map)) return rc;
        for (int c = 0; c < 3; ++c) g.ade_map[c] = p->ptr<int>(L.ade_map) + (size_t)c * L.count;
    }
    // nonuniform-mesh factors
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) {
            g.metric[f][a] = nullptr;
            if (!L.metric[f][a]) continue;
            std::vector<T> vm(n[a]);
            for (int i = 0; i < n[a]; ++i) vm[i] = (T)d->metric[f][a][i];
            if (int rc = upload(s, p, L.metric[f][a], vm)) return rc;
            g.metric[f][a] = p->ptr<T>(L.metric[f][a]);
        }
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 2; ++j) {
            const long long padded = (L.psi_len[0][a] + 63) / 64 * 64;
            for (int par = 0; par < 2; ++par) g.psiE[par][a][j] = L.psiE[a][j] ? p->ptr<T>(L.psiE[a][j]) + par * padded : nullptr;
            g.psiH[a][j] = p->ptr<T>(L.psiH[a][j]);
        }
    // sources
    g.n_src = d->n_sources;
    std::vector<T> values((size_t)std::max(1, d->n_sources) * std::max(1, d->steps), T(0));
    for (int k = 0; k < d->n_sources; ++k) {
        const tfd_source_term &t = d->sources[k];
        g.src[k].family = t.family;
        g.src[k].comp = t.component;
        for (int a = 0; a < 3; ++a) { g.src[k].lo[a] = t.lo[a]; g.src[k].hi[a] = t.hi[a]; }
        for (int q = 0; q < d->steps; ++q) values[(size_t)k * d->steps + q] = (T)t.values[q];
        if (!active(d->components, 3 * t.family + t.component))
            return fail(TFD_ERR_INVALID, "a source drives a component this plan does not advance");
    }
    int rc;
    if ((rc = upload(s, p, L.src_values, values))) return rc;
    g.src_values = p->ptr<T>(L.src_values);
    g.counter = p->ptr<long long>(L.counter);
    g.status = p->ptr<int>(L.status);
    // traces
    std::vector<TraceDev> traces(d->n_traces);
    for (int k = 0; k < d->n_traces; ++k) {
        const tfd_trace &t = d->traces[k];
        traces[k] = TraceDev{t.family, t.component, ((long long)t.index[2] * d->ny + t.index[1]) * L.pitch + t.index[0]};
    }
    if ((rc = upload(s, p, L.trace_tab, traces))) return rc;
    // planes
    std::vector<PlaneDev> planes(d->n_planes);
    p->max_samples = 0;
    for (int k = 0; k < d->n_planes; ++k) {
        const tfd_plane &src = d->planes[k];
        const PlaneLayout &q = L.planes[k];
        PlaneDev &pd = planes[k];
        std::memset(&pd, 0, sizeof(pd));
        pd.points = src.points;
        pd.frequencies = src.frequencies;
        pd.components = src.components;
        pd.corners = src.corners;
        pd.ne = 0;
        for (int c = 0; c < src.components; ++c) {
            pd.comp[c] = src.component_ids[c];
            pd.ne += src.component_ids[c] < 3;
        }
        const size_t entries = (size_t)src.components * src.corners * src.points;
        std::vector<long long> cells(entries);
        std::vector<T> weights(entries);
        for (size_t e = 0; e < entries; ++e) {
            const long long cell = src.corner_cells[e];
            const long long x = cell / ((long long)d->ny * d->nz), y = (cell / d->nz) % d->ny, z = cell % d->nz;
            cells[e] = (z * d->ny + y) * L.pitch + x;
            weights[e] = (T)src.corner_weights[e];
        }
        std::vector<double> omega(src.frequencies), half(2 * (size_t)src.frequencies);
        for (int f = 0; f < src.frequencies; ++f) {
            omega[f] = (2.0 * M_PI * src.frequency_hz[f]) * d->time_step;
            const double ang = (M_PI * src.frequency_hz[f]) * d->time_step;
            half[2 * f] = std::cos(ang);
            half[2 * f + 1] = std::sin(ang);
        }
        std::vector<T> window(2 * (size_t)std::max(1, d->steps), T(0));
        for (int q2 = 0; q2 < d->steps; ++q2) {
            window[q2] = (T)src.window_e[q2];
            window[d->steps + q2] = (T)src.window_h[q2];
        }
        if ((rc = upload(s, p, q.cell, cells)) || (rc = upload(s, p, q.weight, weights)) || (rc = upload(s, p, q.omega, omega)) ||
            (rc = upload(s, p, q.half, half)) || (rc = upload(s, p, q.window, window)))
            return rc;
        pd.cell = p->ptr<long long>(q.cell);
        pd.weight = p->ptr<T>(q.weight);
        pd.omega = p->ptr<double>(q.omega);
        pd.half = p->ptr<double>(q.half);
        pd.window = p->ptr<T>(q.window);
        pd.acc = p->ptr<double>(q.acc);
        p->max_samples = std::max(p->max_samples, src.points * src.components);
    }
    p->max_samples = std::max(p->max_samples, d->n_traces);     // the trace loop strides over the same blocks
    if ((rc = upload(s, p, L.plane_tab, planes))) return rc;
    // zero the state; the material starts as vacuum (inverse permittivity 1)
    return TFD_OK;
}

template <typename T>
int zero_state(tfd_plan *p, cudaStream_t s) {
    const Layout &L = p->L;
    const size_t comp_bytes = (size_t)L.count * L.elem;
    for (int c = 0; c < 3; ++c) {
        if (L.E[c]) TFD_CUDA(cudaMemsetAsync(p->arena + L.E[c], 0, 2 * comp_bytes, s));
        if (L.H[c]) TFD_CUDA(cudaMemsetAsync(p->arena + L.H[c], 0, 2 * comp_bytes, s));
    }
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 2; ++j) {
            if (L.psiE[a][j]) TFD_CUDA(cudaMemsetAsync(p->arena + L.psiE[a][j], 0, 2 * (size_t)((L.psi_len[0][a] + 63) / 64 * 64) * L.elem, s));
            if (L.psiH[a][j]) TFD_CUDA(cudaMemsetAsync(p->arena + L.psiH[a][j], 0, (size_t)L.psi_len[1][a] * L.elem, s));
        }
    TFD_CUDA(cudaMemsetAsync(p->arena + L.trace_out, 0, (size_t)std::max(1, p->desc.n_traces) * std::max(1, p->desc.steps) * L.elem, s));
    for (size_t k = 0; k < L.planes.size(); ++k) {
        const size_t acc = (size_t)p->planes_f[k] * p->planes_p[k] * p->planes_c[k] * 2 * sizeof(double);
        if (acc) TFD_CUDA(cudaMemsetAsync(p->arena + L.planes[k].acc, 0, acc, s));
    }
    for (size_t k = 0; k < L.tfsf.size(); ++k)
        TFD_CUDA(cudaMemsetAsync(p->arena + L.tfsf[k].line, 0, (size_t)4 * p->tfsf<T>().box[k].count * L.elem, s));
    for (size_t k = 0; k < L.ade.size(); ++k) {
        const AdeDev<T> &st = p->grid<T>().ade[k];
        TFD_CUDA(cudaMemsetAsync(p->arena + L.ade[k].state, 0, (size_t)2 * st.poles * st.samples * L.elem, s));
    }
    TFD_CUDA(cudaMemsetAsync(p->arena + L.counter, 0, sizeof(long long), s));
    TFD_CUDA(cudaMemsetAsync(p->arena + L.done, 0, sizeof(unsigned), s));
    TFD_CUDA(cudaMemsetAsync(p->arena + L.grid_bar, 0, 2 * sizeof(unsigned), s));
    TFD_CUDA(cudaMemsetAsync(p->arena + L.status, 0, sizeof(int), s));
    return TFD_OK;
}

}  // namespace

// ---- marching kernel set-up -------------------------------------------------------------------------
namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// CPML slab bounds per (family, axis): segments sorted by lo, as lo0, hi0, lo1, hi1; empty slabs are [0, 0).
int slab_bounds(const tfd_plan *p, int out[2][3][4]) {
    for (int f = 0; f < 2; ++f)
        for (int ax = 0; ax < 3; ++ax) {
            int k = 0;
            int b[4] = {0, 0, 0, 0};
            std::vector<std::pair<int, int>> segs;
            for (int q = 0; q < p->desc.n_segments; ++q)
                if (p->seg_f[q] == f && p->seg_a[q] == ax) segs.push_back({p->seg_lo[q], p->seg_hi[q]});
            std::sort(segs.begin(), segs.end());
            if (segs.size() > 2) return fail(TFD_ERR_INVALID, "more than two CPML slabs on one axis");
            for (auto &sg : segs) { b[2 * k] = sg.first; b[2 * k + 1] = sg.second; ++k; }
            for (int q = 0; q < 4; ++q) out[f][ax][q] = b[q];
        }
    return TFD_OK;
}

template <typename T>
bool march_supported(const tfd_plan *p) {
    const Grid<T> &g = const_cast<tfd_plan *>(p)->grid<T>();
    return g.n[2] > 1 && g.active == 0x3F;
}


// Target z-planes per CTA chunk of the marching kernel (see choose_lz in setup_march_s).
constexpr int kMarchChunkPlanes = 12;

// Launch variant (D * 10 + MINB) that the periodic-seam kernel (MODE 2) is built for.
template <typename T>
constexpr int periodic_march_variant() { return sizeof(T) == 4 ? 14 : 22; }

template <typename T, int SAMPLES, int D, int MINB>
int setup_march_s(tfd_plan *p, int split, int lz_fixed) {
    const bool split_interior = split == 1;
    // Split digit 0: the mixed launch where the grid has an interior block (measured on B200: 0.963 vs
    // 1.038 ms per step at 512x512x256, 0.612 vs 0.691 ms at 512x512x128 periodic), else the general kernel.
    if (split == 0) split = 3;
    using S = MarchShape<T, SAMPLES, D>;
    Grid<T> &g = p->grid<T>();
    MarchArgs<T> &a = p->march<T>();
    std::memset(&a, 0, sizeof(a));
    a.g = g;
    const bool seams = g.periodic[0] || g.periodic[1];
    for (int ax = 0; ax < 2; ++ax)
        for (int q = 0; q < p->desc.n_segments; ++q)
            if (g.periodic[ax] && p->seg_a[q] == ax)
                return fail(TFD_ERR_INVALID, "a periodic axis carries a CPML slab");
    for (int ax = 0; ax < 3; ++ax) a.psi_parity[ax] = (int)((p->L.psi_len[0][ax] + 63) / 64 * 64);
    if (g.count >= (1LL << 31)) return fail(TFD_ERR_UNSUPPORTED, "component arrays above 2^31 elements need the gather kernel");
    for (int f = 0; f < 2; ++f)
        for (int ax = 0; ax < 3; ++ax)
            if (p->L.psi_len[f][ax] >= (1LL << 31)) return fail(TFD_ERR_UNSUPPORTED, "CPML memory above 2^31 elements");
    if (int rc = slab_bounds(p, a.slab)) return rc;
    auto encode = tensor_map_encoder();
    if (!encode) return fail(TFD_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable from the driver");
    const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t e = sizeof(T);
    for (int c = 0; c < 6; ++c) {
        T *base = c < 3 ? g.E[0][c] : g.H[0][c - 3];
        const cuuint64_t dims[4] = {(cuuint64_t)g.n[0], (cuuint64_t)g.n[1], (cuuint64_t)g.n[2], 2};
        const cuuint64_t strides[3] = {(cuuint64_t)g.pitch * e, (cuuint64_t)g.plane * e, (cuuint64_t)g.count * e};
        const cuuint32_t box[4] = {(cuuint32_t)S::BXW, (cuuint32_t)(c < 3 ? S::BYE : S::BYH), 1, 1};
        const cuuint32_t elem[4] = {1, 1, 1, 1};
        CUresult r = encode(&a.field[c], dt, 4, (void *)base, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(TFD_ERR_CUDA, "cuTensorMapEncodeTiled(field) failed: " + std::to_string((int)r));
    }
    for (int c = 0; c < SAMPLES; ++c) {
        const cuuint64_t dims[3] = {(cuuint64_t)g.n[0], (cuuint64_t)g.n[1], (cuuint64_t)g.n[2]};
        const cuuint64_t strides[2] = {(cuuint64_t)g.pitch * e, (cuuint64_t)g.plane * e};
        const cuuint32_t box[3] = {(cuuint32_t)S::BXW, (cuuint32_t)S::BYE, 1};
        const cuuint32_t elem[3] = {1, 1, 1};
        CUresult r = encode(&a.eps[c], dt, 3, (void *)g.inv_eps[c], dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(TFD_ERR_CUDA, "cuTensorMapEncodeTiled(eps) failed: " + std::to_string((int)r));
    }
    p->march_smem = S::SMEM;
    TFD_CUDA(cudaFuncSetAttribute(k_step_march<T, SAMPLES, D, MINB, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->march_smem));
    TFD_CUDA(cudaFuncSetAttribute(k_step_march<T, SAMPLES, D, MINB, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->march_smem));
    TFD_CUDA(cudaFuncSetAttribute(k_step_march_mixed<T, SAMPLES, D, MINB, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)p->march_smem));
    if constexpr (D * 10 + MINB == periodic_march_variant<T>()) {
        TFD_CUDA(cudaFuncSetAttribute(k_step_march<T, SAMPLES, D, MINB, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->march_smem));
        TFD_CUDA(cudaFuncSetAttribute(k_step_march_mixed<T, SAMPLES, D, MINB, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)p->march_smem));
        TFD_CUDA(cudaFuncSetAttribute(k_step_march<T, SAMPLES, D, MINB, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)p->march_smem));
        TFD_CUDA(cudaFuncSetAttribute(k_step_march<T, SAMPLES, D, MINB, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)p->march_smem));
        TFD_CUDA(cudaFuncSetAttribute(k_step_march_mixed<T, SAMPLES, D, MINB, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)p->march_smem));
    }
    const int edge_mode = seams ? 2 : 0;
    int device = 0, sms = 148, per_sm = 1;
    TFD_CUDA(cudaGetDevice(&device));
    TFD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    TFD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_march<T, SAMPLES, D, MINB, 1>, kMarchThreads, p->march_smem));
    const long long resident = (long long)sms * std::max(1, per_sm);
    const int tx = (g.n[0] + kMarchOwnX - 1) / kMarchOwnX, ty = (g.n[1] + kMarchOwnY - 1) / kMarchOwnY;
    // Planes per chunk for a launch of `tiles` tiles sharing `share` of the resident CTA slots. Chunks
    // of about kMarchChunkPlanes: in a long march neighbouring tiles drift apart in z and the halo rows
    // they share miss in L2 (measured on B200 at 512x496x256: one 256-plane chunk per tile moved 5.9 GB
    // per step at 23 % L2 hits, 12-plane chunks 4.1 GB at 41 %, and ran 2.8x faster), while short
    // chunks reload more halo planes (4 planes: 9 % slower than 12). Small grids take shorter chunks,
    // down to 2 planes, until the launch has two waves of CTAs.
    auto choose_lz = [&](long long tiles, int planes, double share) {
        if (lz_fixed > 0) return std::min(lz_fixed, planes);
        const double slots = std::max(1.0, share * resident);
        int chunks = (planes + kMarchChunkPlanes - 1) / kMarchChunkPlanes;
        while ((double)tiles * chunks < 2 * slots) {
            const int next = chunks + 1;
            if ((planes + next - 1) / next < 2) break;
            chunks = next;
        }
        return (planes + chunks - 1) / chunks;
    };
    auto chunks_of = [&](int lz, int planes) { return (unsigned)((planes + lz - 1) / lz); };
    const int nzp = g.n[2];
    const int lz_all = choose_lz((long long)tx * ty, nzp, 1.0);
    p->march_grid = dim3(tx, ty, chunks_of(lz_all, nzp));
    p->march_launches.clear();
    // One launch of `mode` over tiles [ox, ox + sx) x [oy, oy + sy) and planes [zlo, zhi); share: its
    // fraction of the step's tile-planes (for the chunk length).
    const double tile_planes = (double)tx * ty * nzp;
    auto push = [&](int mode, int sx, int sy, int ox, int oy, int zlo, int zhi) {
        if (sx <= 0 || sy <= 0 || zhi <= zlo) return;
        const int planes = zhi - zlo;
        const int lz = choose_lz((long long)sx * sy, planes, (double)sx * sy * planes / tile_planes);
        p->march_launches.push_back({mode, dim3(sx, sy, chunks_of(lz, planes)), ox, oy, lz, zlo, zhi});
    };
    // Interior tiles: all 32 x 16 computed cells inside the domain, x-1 / y-1 present, H neighbours
    // x+1 / y+1 present, and no E or H CPML slab on x or y. They form a contiguous tile range.
    auto meets = [&](int f, int ax, int lo, int hi) {
        const int *b = a.slab[f][ax];
        return (lo < b[1] && b[0] < hi) || (lo < b[3] && b[2] < hi);
    };
    auto interior_x = [&](int t) {
        const int x0 = t * kMarchOwnX;
        return x0 > 0 && x0 + kMarchLanes < g.n[0] && !meets(0, 0, x0, x0 + kMarchLanes) && !meets(1, 0, x0, x0 + kMarchOwnX);
    };
    auto interior_y = [&](int t) {
        const int y0 = t * kMarchOwnY;
        return y0 > 0 && y0 + kMarchRows < g.n[1] && !meets(0, 1, y0, y0 + kMarchRows) && !meets(1, 1, y0, y0 + kMarchOwnY);
    };
    int ix0 = 0, ix1 = 0, iy0 = 0, iy1 = 0;
    while (ix0 < tx && !interior_x(ix0)) ++ix0;
    ix1 = ix0;
    while (ix1 < tx && interior_x(ix1)) ++ix1;
    while (iy0 < ty && !interior_y(iy0)) ++iy0;
    iy1 = iy0;
    while (iy1 < ty && interior_y(iy1)) ++iy1;
    // Pure planes: the longest range [za, zb) whose chunks meet no z slab: E planes za..zb (zb is a
    // chunk's halo plane) outside every E-family z slab, H planes za..zb-1 outside every H-family one,
    // za >= 1 and zb <= nz - 1 (the first and last planes have faces).
    int za = 0, zb = 0;
    {
        std::vector<char> ebad(nzp + 1, 0), hbad(nzp + 1, 0);
        for (int q = 0; q < 2; ++q) {
            for (int z = a.slab[0][2][2 * q]; z < a.slab[0][2][2 * q + 1]; ++z) ebad[z] = 1;
            for (int z = a.slab[1][2][2 * q]; z < a.slab[1][2][2 * q + 1]; ++z) hbad[z] = 1;
        }
        for (int z = 1; z < nzp - 1; ++z) {
            if (ebad[z] || hbad[z]) continue;
            int e = z;
            while (e + 1 <= nzp - 1 && !ebad[e + 1] && !hbad[e]) ++e;
            if (e - z > zb - za) { za = z; zb = e; }
            z = e;
        }
    }
    if (split_interior && ix1 > ix0 && iy1 > iy0 && zb - za >= 2) {
        // The pure fast kernel over the interior block; the general kernel over its z-slab planes and
        // over the boundary strips (all planes). Concurrent launches on forked streams.
        // Measured on B200 this split is slower than one general launch (512x512x256: 1.16 vs 1.02 ms per
        // step, in either launch order; 256^3: 0.41 vs 0.37 ms), so it is a launch variant the tuner may
        // pick (split digit 1), not the default.
        const int ni = ix1 - ix0, nj = iy1 - iy0;
        push(edge_mode, ix0, ty, 0, 0, 0, nzp);
        push(edge_mode, tx - ix1, ty, ix1, 0, 0, nzp);
        push(edge_mode, ni, iy0, ix0, 0, 0, nzp);
        push(edge_mode, ni, ty - iy1, ix0, iy1, 0, nzp);
        push(edge_mode, ni, nj, ix0, iy0, 0, za);
        push(edge_mode, ni, nj, ix0, iy0, zb, nzp);
        push(1, ni, nj, ix0, iy0, za, zb);
    } else if (split == 3 && ix1 > ix0 && iy1 > iy0 && zb - za >= 2) {
        // Default: one launch, each CTA taking the pure body on the interior block's pure planes and the
        // general body elsewhere (k_step_march_mixed).
        MarchMix &mx = p->march_mix;
        mx = MarchMix{};
        mx.ix0 = ix0; mx.ix1 = ix1; mx.iy0 = iy0; mx.iy1 = iy1;
        // x-boundary tiles of the interior y range on the pure planes take the x-tier body (non-periodic grids;
        // TFD_MARCH_XBODY=0 gives them the general body, for comparisons).
        const char *xenv = getenv("TFD_MARCH_XBODY");
        mx.xband = (xenv && std::atoi(xenv) == 0) ? 0 : 1;
        mx.zb[0] = 0; mx.zb[1] = za; mx.zb[2] = zb; mx.zb[3] = nzp;
        int total = 0;
        for (int q = 0; q < 3; ++q) {
            const int planes = mx.zb[q + 1] - mx.zb[q];
            mx.lz[q] = planes > 0 ? choose_lz((long long)tx * ty, planes, (double)planes / nzp) : 1;
            mx.chunks[q] = planes > 0 ? (int)chunks_of(mx.lz[q], planes) : 0;
            total += mx.chunks[q];
        }
        p->march_launches.push_back({3, dim3(tx, ty, total), 0, 0, 0, 0, nzp});
    } else {
        push(edge_mode, tx, ty, 0, 0, 0, nzp);
    }
    if (p->aux.empty() && p->march_launches.size() > 1) {
        TFD_CUDA(cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming));
        for (size_t k = 1; k < p->march_launches.size(); ++k) {
            cudaStream_t st;
            cudaEvent_t ev;
            TFD_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            TFD_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            p->aux.push_back(st);
            p->join.push_back(ev);
        }
    }
    p->march_variant = D * 10 + MINB;
    return TFD_OK;
}

// Launch variant of the marching kernel, as decimal digits: lz * 1000 + split * 100 + D * 10 + MINB.
// D / MINB: prefetch depth and CTAs per SM, one of 14 (FP32 default), 23, 32, 22 (FP64: 22 only);
// split 1: the interior block and the boundary as separate concurrent launches; 2: the general kernel only;
// 3: one launch, the pure body on the interior block's planes outside the z slabs (k_step_march_mixed), when
// the grid has such a block (else the general kernel); 0: 3. lz: z-planes per CTA chunk (0: about 12, shorter
// on small grids).
// Grids with periodic x/y faces run D / MINB = 14 (FP32) or 22 (FP64) whatever the variant asks.
// 0 selects the default (TFD_MARCH_VARIANT in the environment overrides the default, for sweeps).
template <typename T>
int setup_march(tfd_plan *p) {
    const char *env = getenv("TFD_MARCH_VARIANT");
    int v = p->desc.launch_variant;
    if (v == 0) v = env ? std::atoi(env) : 0;
    if (v == 0) v = sizeof(T) == 4 ? 14 : 22;
    const int dm = v % 100, split = (v / 100) % 10, lz = v / 1000;
    if (v < 0 || split > 3 || (dm != 14 && dm != 22 && dm != 23 && dm != 32) || (sizeof(T) == 8 && dm != 22))
        return fail(TFD_ERR_INVALID, "launch variant " + std::to_string(v) + " is not lz*1000 + split*100 + one of " +
                                         (sizeof(T) == 8 ? std::string("22 (FP64)") : std::string("14, 22, 23, 32")));
    const bool three = p->desc.material_samples == 3;
    const Grid<T> &g = p->grid<T>();
    // A nonuniform mesh runs the metric bodies at the launch shape the periodic-seam body is built for: the mixed
    // launch (pure body on the interior block) by default, the general body alone for split digits 1 and 2 and
    // with periodic seams.
    p->march_metric = false;
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) p->march_metric = p->march_metric || g.metric[f][a] != nullptr;
    // Nonuniform meshes: the metric mixed launch (pure body on the interior block) unless a split is asked for.
    const int sp = (p->march_metric && (split == 1 || split == 2 || g.periodic[0] || g.periodic[1])) ? 2 : split;
    switch ((g.periodic[0] || g.periodic[1] || p->march_metric) ? periodic_march_variant<T>() : dm) {
        case 22: return three ? setup_march_s<T, 3, 2, 2>(p, sp, lz) : setup_march_s<T, 1, 2, 2>(p, sp, lz);
        case 32: return three ? setup_march_s<T, 3, 3, 2>(p, sp, lz) : setup_march_s<T, 1, 3, 2>(p, sp, lz);
        case 14: return three ? setup_march_s<T, 3, 1, 4>(p, sp, lz) : setup_march_s<T, 1, 1, 4>(p, sp, lz);
        default: return three ? setup_march_s<T, 3, 2, 3>(p, sp, lz) : setup_march_s<T, 1, 2, 3>(p, sp, lz);
    }
}

template <typename T, int SAMPLES, int D, int MINB>
void launch_march(tfd_plan *p, cudaStream_t s) {
    const size_t n = p->march_launches.size();
    if (n > 1) cudaEventRecord(p->fork, s);
    for (size_t k = 0; k < n; ++k) {
        const auto &l = p->march_launches[k];
        cudaStream_t st = k == 0 ? s : p->aux[k - 1];
        if (k > 0) cudaStreamWaitEvent(st, p->fork, 0);
        if (l.mode == 3) {
            if (p->march_metric) {
                if constexpr (D * 10 + MINB == periodic_march_variant<T>())
                    k_step_march_mixed<T, SAMPLES, D, MINB, 0, true><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(),
                                                                                                                p->march_mix);
            } else if (p->grid<T>().periodic[0] || p->grid<T>().periodic[1]) {
                if constexpr (D * 10 + MINB == periodic_march_variant<T>())
                    k_step_march_mixed<T, SAMPLES, D, MINB, 2><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(), p->march_mix);
            } else {
                k_step_march_mixed<T, SAMPLES, D, MINB, 0><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(), p->march_mix);
            }
        } else if (p->march_metric) {
            if constexpr (D * 10 + MINB == periodic_march_variant<T>()) {
                if (l.mode == 2)
                    k_step_march<T, SAMPLES, D, MINB, 2, true><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(), l.tx_off,
                                                                                                           l.ty_off, l.lz, l.z_lo, l.z_hi);
                else
                    k_step_march<T, SAMPLES, D, MINB, 0, true><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(), l.tx_off,
                                                                                                           l.ty_off, l.lz, l.z_lo, l.z_hi);
            }
        } else if (l.mode == 1)
            k_step_march<T, SAMPLES, D, MINB, 1><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(), l.tx_off, l.ty_off, l.lz,
                                                                                             l.z_lo, l.z_hi);
        else if (l.mode == 2) {
            if constexpr (D * 10 + MINB == periodic_march_variant<T>())
                k_step_march<T, SAMPLES, D, MINB, 2><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(), l.tx_off, l.ty_off,
                                                                                                 l.lz, l.z_lo, l.z_hi);
        } else
            k_step_march<T, SAMPLES, D, MINB, 0><<<l.grid, kMarchThreads, p->march_smem, st>>>(p->march<T>(), l.tx_off, l.ty_off, l.lz,
                                                                                             l.z_lo, l.z_hi);
        if (k > 0) cudaEventRecord(p->join[k - 1], st);
    }
    for (size_t k = 1; k < n; ++k) cudaStreamWaitEvent(s, p->join[k - 1], 0);
}

template <typename T>
void launch_march_any(tfd_plan *p, cudaStream_t s) {
    const bool three = p->desc.material_samples == 3;
    switch (p->march_variant) {
        case 23: three ? launch_march<T, 3, 2, 3>(p, s) : launch_march<T, 1, 2, 3>(p, s); break;
        case 22: three ? launch_march<T, 3, 2, 2>(p, s) : launch_march<T, 1, 2, 2>(p, s); break;
        case 32: three ? launch_march<T, 3, 3, 2>(p, s) : launch_march<T, 1, 3, 2>(p, s); break;
        default: three ? launch_march<T, 3, 1, 4>(p, s) : launch_march<T, 1, 1, 4>(p, s); break;
    }
}

}  // namespace

// ---- 2D tile kernel set-up ---------------------------------------------------------------------------
namespace {

template <typename T>
StripGeom strip_geom(tfd_plan *p) {
    StripGeom G;
    const Grid<T> &g = p->grid<T>();
    G.nx = g.n[0];
    G.ny = g.n[1];
    for (size_t k = 0; k < p->seg_f.size(); ++k) G.slabs.push_back({p->seg_f[k], p->seg_a[k], p->seg_lo[k], p->seg_hi[k]});
    for (int k = 0; k < g.n_src; ++k) G.sources.push_back(g.src[k]);
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 2; ++a) G.metric = G.metric || g.metric[f][a] != nullptr;
    return G;
}

// CTAs of a 2D launch over `strips` strips: one warp per strip, or `ctas` persistent CTAs when set.
inline int ctas_2d(int strips, int ctas) {
    const int all = (strips + k2dWarps - 1) / k2dWarps;
    return std::max(1, ctas > 0 ? std::min(ctas, all) : all);
}

template <typename T>
int setup_cluster2d(tfd_plan *p);

template <typename T>
int setup_tile2d(tfd_plan *p, cudaStream_t s) {
    Grid<T> &g = p->grid<T>();
    std::vector<Tile2D> tiles = strips_of(strip_geom<T>(p), 0, p->L.strip_rows);
    if ((int)tiles.size() != p->L.tiles2d) return fail(TFD_ERR_INVALID, "2D strip table does not match the layout");
    p->tile2d_interior = interior_count(tiles);
    if (p->tile2d_interior > 0 && p->tile2d_interior < p->L.tiles2d && !p->side2d) {
        p->side2d.reset(new SideStream());
        TFD_CHECK(p->side2d->create());
    }
    TFD_CUDA(cudaMemcpyAsync(p->arena + p->L.grid_tab, &g, sizeof(Grid<T>), cudaMemcpyHostToDevice, s));
    TFD_CUDA(cudaMemcpyAsync(p->arena + p->L.tile_tab, tiles.data(), tiles.size() * sizeof(Tile2D), cudaMemcpyHostToDevice, s));
    // Small grids step in one persistent launch (TFD_PERSIST2D=0/1 in the environment overrides the size
    // rule, for sweeps): a warp per strip, and no more CTAs than can be resident together.
    p->persist_ctas = 0;
    if (persist2d_eligible((long long)g.n[0] * g.n[1])) {
        int device = 0, sms = 148, per_sm = 0;
        TFD_CUDA(cudaGetDevice(&device));
        TFD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        TFD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step2d_persistent<T>, k2dThreads, 0));
        const int mblocks = std::max(1, (p->max_samples + kMonitorThreads - 1) / kMonitorThreads) * std::max(1, p->desc.n_planes);
        const int want = std::max({1, (p->L.tiles2d + k2dWarps - 1) / k2dWarps, mblocks});
        if (per_sm > 0) p->persist_ctas = std::min(want, per_sm * sms);
    }
    return setup_cluster2d<T>(p);
}

// One 2D step over a strip table whose first `interior` strips are interior strips. The general strips
// (latency-bound: CPML memories, edges, sources) start first on the side stream and overlap the
// bandwidth-bound interior kernel; the caller's stream waits for both (graph capture follows the fork).
template <typename T>
void launch_strips(const Grid<T> *grids, const Tile2D *table, int interior, int all, int ctas, const long long *counter,
                   cudaStream_t s, const SideStream *side) {
    const bool both = interior > 0 && all > interior && side != nullptr && side->stream != nullptr;
    if (both) {
        cudaEventRecord(side->fork, s);
        cudaStreamWaitEvent(side->stream, side->fork, 0);
    }
    if (all > interior)
        k_step2d_general<T><<<ctas_2d(all - interior, ctas), k2dThreads, 0, both ? side->stream : s>>>(grids, table + interior,
                                                                                                     all - interior, counter);
    if (interior > 0) k_step2d_interior<T><<<ctas_2d(interior, ctas), k2dThreads, 0, s>>>(grids, table, interior, counter);
    if (both) {
        cudaEventRecord(side->join, side->stream);
        cudaStreamWaitEvent(s, side->join, 0);
    }
}

template <typename T>
void launch_tile2d(tfd_plan *p, cudaStream_t s) {
    launch_strips<T>((const Grid<T> *)(p->arena + p->L.grid_tab), (const Tile2D *)(p->arena + p->L.tile_tab), p->tile2d_interior,
                     p->L.tiles2d, p->desc.launch_variant, p->grid<T>().counter, s, p->side2d.get());
}

}  // namespace

// ---- C ABI ---------------------------------------------------------------------------------------
namespace {

cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

template <typename T>
FieldSet<T> field_set(tfd_plan *p) {
    FieldSet<T> fs;
    Grid<T> &g = p->grid<T>();
    for (int par = 0; par < 2; ++par)
        for (int c = 0; c < 3; ++c) {
            fs.f[par][c] = g.E[par][c];
            fs.f[par][3 + c] = g.H[par][c];
        }
    return fs;
}

template <typename T>
PsiArgs<T> psi_args(tfd_plan *p) {
    PsiArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    Grid<T> &g = p->grid<T>();
    a.n_seg = (int)p->psi_segs.size();
    for (int k = 0; k < a.n_seg; ++k) a.seg[k] = p->psi_segs[k];
    for (int q = 0; q < 3; ++q) a.n[q] = g.n[q];
    a.pitch = g.pitch;
    for (int f = 0; f < 2; ++f)
        for (int q = 0; q < 3; ++q) {
            a.row[f][q] = g.row[f][q];
            a.rows[f][q] = g.rows[f][q];
        }
    std::memcpy(a.psiE, g.psiE, sizeof(a.psiE));
    std::memcpy(a.psiH, g.psiH, sizeof(a.psiH));
    a.counter = g.counter;
    return a;
}

// Copy `bytes` between a caller buffer (host or device) and the plan's stage buffer.
int stage_in(tfd_plan *p, const void *src, size_t bytes, int where, cudaStream_t s, const void **dev) {
    if (where == TFD_DEVICE) { *dev = src; return TFD_OK; }
    if (where != TFD_HOST) return fail(TFD_ERR_INVALID, "where must be TFD_DEVICE or TFD_HOST");
    if (bytes > p->L.stage_bytes) return fail(TFD_ERR_INVALID, "transfer larger than the stage buffer");
    TFD_CUDA(cudaMemcpyAsync(p->arena + p->L.stage, src, bytes, cudaMemcpyHostToDevice, s));
    *dev = p->arena + p->L.stage;
    return TFD_OK;
}

// Blocks of the tiled layout conversions (one per 32 x 32 (x, z) tile of each y row), or 0 when the grid is
// too thin in z for them or has more tiles than one launch holds.
inline unsigned tiled_blocks(const tfd_desc &d) {
    if (d.nz < kTileMinNz) return 0;
    const long long b = (long long)((d.nx + kTile - 1) / kTile) * ((d.nz + kTile - 1) / kTile) * d.ny;
    return b < (1ll << 31) ? (unsigned)b : 0u;
}

template <typename T>
TileArrays<T> tile_arrays(T *a, T *b, T *c) {
    TileArrays<T> t{};
    for (int par = 0; par < 2; ++par) {
        t.p[par][0] = a;
        t.p[par][1] = b;
        t.p[par][2] = c;
    }
    return t;
}

template <typename T>
TileArrays<T> tile_arrays(const FieldSet<T> &fs, int family) {
    TileArrays<T> t{};
    for (int par = 0; par < 2; ++par)
        for (int c = 0; c < 3; ++c) t.p[par][c] = fs.f[par][3 * family + c];
    return t;
}

template <typename T>
int set_material_t(tfd_plan *p, const void *src, int where, cudaStream_t s) {
    const tfd_desc &d = p->desc;
    const int S = d.material_samples;
    const size_t bytes = (size_t)d.nx * d.ny * d.nz * S * sizeof(T);
    const void *dev;
    int rc = stage_in(p, src, bytes, where, s, &dev);
    if (rc) return rc;
    Grid<T> &g = p->grid<T>();
    if (const unsigned tb = tiled_blocks(d))
        k_from_reference_tiled<T, false><<<tb, kTileThreads, 0, s>>>(
            (const T *)dev, tile_arrays<T>((T *)g.inv_eps[0], (T *)(S == 3 ? g.inv_eps[1] : nullptr), (T *)(S == 3 ? g.inv_eps[2] : nullptr)),
            nullptr, S, d.nx, d.ny, d.nz, g.pitch, nullptr);
    else
        k_reference_to_internal<T><<<launch_blocks((long long)d.nx * d.ny * d.nz * S), 256, 0, s>>>(
            (const T *)dev, S, d.nx, d.ny, d.nz, g.pitch, (T *)g.inv_eps[0], (T *)(S == 3 ? g.inv_eps[1] : nullptr),
            (T *)(S == 3 ? g.inv_eps[2] : nullptr));
    TFD_CUDA(cudaGetLastError());
    if (where == TFD_HOST) TFD_CUDA(cudaStreamSynchronize(s));
    return TFD_OK;
}

template <typename T>
int set_permittivity_t(tfd_plan *p, const void *src, int where, cudaStream_t s) {
    const tfd_desc &d = p->desc;
    const int S = d.material_samples;
    const size_t bytes = (size_t)d.nx * d.ny * d.nz * S * sizeof(T);
    const void *dev;
    int rc = stage_in(p, src, bytes, where, s, &dev);
    if (rc) return rc;
    Grid<T> &g = p->grid<T>();
    int *bad = p->ptr<int>(p->L.check);
    TFD_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    if (const unsigned tb = tiled_blocks(d))
        k_from_reference_tiled<T, true><<<tb, kTileThreads, 0, s>>>(
            (const T *)dev, tile_arrays<T>((T *)g.inv_eps[0], (T *)(S == 3 ? g.inv_eps[1] : nullptr), (T *)(S == 3 ? g.inv_eps[2] : nullptr)),
            nullptr, S, d.nx, d.ny, d.nz, g.pitch, bad);
    else
        k_permittivity_to_internal<T><<<launch_blocks((long long)d.nx * d.ny * d.nz * S), 256, 0, s>>>(
            (const T *)dev, S, d.nx, d.ny, d.nz, g.pitch, (T *)g.inv_eps[0], (T *)(S == 3 ? g.inv_eps[1] : nullptr),
            (T *)(S == 3 ? g.inv_eps[2] : nullptr), bad);
    TFD_CUDA(cudaGetLastError());
    int flag = 0;
    TFD_CUDA(cudaMemcpyAsync(&flag, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    if (flag) return fail(TFD_ERR_INVALID, "epsilon must be finite and at least 1.");
    return TFD_OK;
}

template <typename T>
int field_check_t(tfd_plan *p, double *peak_e, int32_t *finite, cudaStream_t s) {
    unsigned long long *out = p->ptr<unsigned long long>(p->L.check);
    TFD_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long), s));
    k_field_check<T><<<launch_blocks(p->L.count), 256, 0, s>>>(field_set<T>(p), p->L.count, p->grid<T>().counter, out);
    TFD_CUDA(cudaGetLastError());
    unsigned long long host[2] = {0, 0};
    TFD_CUDA(cudaMemcpyAsync(host, out, sizeof(host), cudaMemcpyDeviceToHost, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    double peak;
    if (sizeof(T) == 4) {
        const unsigned bits = (unsigned)host[0];
        float f;
        std::memcpy(&f, &bits, sizeof(f));
        peak = f;
    } else {
        std::memcpy(&peak, &host[0], sizeof(peak));
    }
    *peak_e = peak;
    *finite = host[1] ? 0 : 1;
    return TFD_OK;
}

template <typename T>
int set_fields_t(tfd_plan *p, const void *E, const void *H, int where, cudaStream_t s) {
    const tfd_desc &d = p->desc;
    const long long total = (long long)d.nx * d.ny * d.nz * 3;
    const size_t bytes = total * sizeof(T);
    const FieldSet<T> fs = field_set<T>(p);
    for (int fam = 0; fam < 2; ++fam) {
        const void *src = fam == 0 ? E : H;
        if (!src) continue;
        const void *dev;
        int rc = stage_in(p, src, bytes, where, s, &dev);
        if (rc) return rc;
        if (const unsigned tb = tiled_blocks(d))
            k_from_reference_tiled<T, false><<<tb, kTileThreads, 0, s>>>((const T *)dev, tile_arrays<T>(fs, fam), p->grid<T>().counter, 3,
                                                                         d.nx, d.ny, d.nz, p->L.pitch, nullptr);
        else
            k_reference_to_fields<T><<<launch_blocks(total), 256, 0, s>>>(fam == 0 ? (const T *)dev : nullptr,
                                                                           fam == 1 ? (const T *)dev : nullptr, d.nx, d.ny, d.nz,
                                                                           p->L.pitch, fs, p->grid<T>().counter);
        TFD_CUDA(cudaGetLastError());
        if (where == TFD_HOST) TFD_CUDA(cudaStreamSynchronize(s));
    }
    return TFD_OK;
}

template <typename T>
int get_fields_t(tfd_plan *p, void *E, void *H, int where, cudaStream_t s) {
    const tfd_desc &d = p->desc;
    const long long total = (long long)d.nx * d.ny * d.nz * 3;
    const size_t bytes = total * sizeof(T);
    const FieldSet<T> fs = field_set<T>(p);
    for (int fam = 0; fam < 2; ++fam) {
        void *dst = fam == 0 ? E : H;
        if (!dst) continue;
        void *dev = where == TFD_DEVICE ? dst : p->arena + p->L.stage;
        if (where == TFD_HOST && bytes > p->L.stage_bytes) return fail(TFD_ERR_INVALID, "transfer larger than the stage buffer");
        if (const unsigned tb = tiled_blocks(d))
            k_to_reference_tiled<T><<<tb, kTileThreads, 0, s>>>((T *)dev, tile_arrays<T>(fs, fam), p->grid<T>().counter, 3, d.nx, d.ny,
                                                                d.nz, p->L.pitch);
        else
            k_fields_to_reference<T><<<launch_blocks(total), 256, 0, s>>>(fam == 0 ? (T *)dev : nullptr, fam == 1 ? (T *)dev : nullptr,
                                                                           d.nx, d.ny, d.nz, p->L.pitch, fs, p->grid<T>().counter);
        TFD_CUDA(cudaGetLastError());
        if (where == TFD_HOST) {
            TFD_CUDA(cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDeviceToHost, s));
            TFD_CUDA(cudaStreamSynchronize(s));
        }
    }
    return TFD_OK;
}

template <typename T>
int psi_t(tfd_plan *p, void *vec, int where, cudaStream_t s, bool to_reference) {
    const size_t bytes = p->L.psi_total * sizeof(T);
    if (p->psi_segs.empty()) return TFD_OK;
    void *dev = vec;
    if (where == TFD_HOST) {
        dev = p->arena + p->L.stage;
        if (!to_reference) TFD_CUDA(cudaMemcpyAsync(dev, vec, bytes, cudaMemcpyHostToDevice, s));
    }
    const PsiArgs<T> a = psi_args<T>(p);
    long long largest = 0;
    for (auto &sg : p->psi_segs) {
        long long ext[3] = {p->desc.nx, p->desc.ny, p->desc.nz};
        ext[sg.a] = sg.hi - sg.lo;
        largest = std::max(largest, ext[0] * ext[1] * ext[2]);
    }
    dim3 grid(launch_blocks(largest), (unsigned)p->psi_segs.size());
    k_psi_copy<T><<<grid, 256, 0, s>>>((T *)dev, a, to_reference ? 1 : 0);
    TFD_CUDA(cudaGetLastError());
    if (where == TFD_HOST) {
        if (to_reference) TFD_CUDA(cudaMemcpyAsync(vec, dev, bytes, cudaMemcpyDeviceToHost, s));
        TFD_CUDA(cudaStreamSynchronize(s));
    }
    return TFD_OK;
}

template <typename T>
MonitorArgs<T> monitor_args(tfd_plan *p) {
    MonitorArgs<T> m;
    std::memset(&m, 0, sizeof(m));
    Grid<T> &g = p->grid<T>();
    for (int c = 0; c < 3; ++c) {
        m.field[c] = g.E[0][c];
        m.field[3 + c] = g.H[0][c];
    }
    m.count = g.count;
    m.steps = g.steps;
    m.counter = g.counter;
    m.done = p->ptr<unsigned>(p->L.done);
    m.n_traces = p->desc.n_traces;
    m.traces = p->ptr<TraceDev>(p->L.trace_tab);
    m.trace_out = p->ptr<T>(p->L.trace_out);
    m.n_planes = p->desc.n_planes;
    m.planes = p->ptr<PlaneDev>(p->L.plane_tab);
    m.max_samples = p->max_samples;
    return m;
}

template <typename T>
int launch_step_gather(tfd_plan *p, cudaStream_t s) {
    const Grid<T> &g = p->grid<T>();
    dim3 block(128), grid((unsigned)((long long)g.n[1] * g.n[2]), (unsigned)((g.n[0] + 127) / 128));
    // rows on x (up to 2^31-1), x chunks on y
    switch (g.active) {
        case kMaskTM: k_step_gather_rows<T, kMaskTM><<<grid, block, 0, s>>>(g); break;
        case kMaskTE: k_step_gather_rows<T, kMaskTE><<<grid, block, 0, s>>>(g); break;
        default: k_step_gather_rows<T, kMaskAll><<<grid, block, 0, s>>>(g); break;
    }
    return TFD_OK;
}

// The on-chip cluster path for small 2D TMz plans without DFT planes (TFD_CLUSTER2D=0 in the environment
// turns it off, for comparisons): the smallest cluster of 8 or 16 CTAs whose per-rank bands fit in shared memory.
template <typename T>
int setup_cluster2d(tfd_plan *p) {
    Cluster2D &c = p->cluster2d;
    c = Cluster2D{};
    p->cluster2d_smem = 0;
    const char *env = getenv("TFD_CLUSTER2D");
    if ((env && std::atoi(env) == 0) || p->desc.n_planes > 0 || p->desc.n_tfsf > 0 || p->desc.n_ade > 0) return TFD_OK;
    const Grid<T> &g = p->grid<T>();
    const int nx = g.n[0], ny = g.n[1];
    int device = 0, max_smem = 0;
    TFD_CUDA(cudaGetDevice(&device));
    TFD_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    // y-slab memory rows of a band: rows y of the band with a slab row (E: y > 0, H: y < ny - 1), contiguous.
    auto slab_rows = [&](int f, int lo, int hi, int &first, int &count) {
        std::vector<std::pair<int, int>> segs;
        for (size_t q = 0; q < p->seg_f.size(); ++q)
            if (p->seg_f[q] == f && p->seg_a[q] == 1) segs.push_back({p->seg_lo[q], p->seg_hi[q]});
        std::sort(segs.begin(), segs.end());
        int base = 0;
        first = -1;
        count = 0;
        for (auto &sg : segs) {
            const int a = std::max(sg.first, lo), b = std::min(sg.second, hi);
            if (a < b) {
                if (first < 0) first = base + (a - sg.first);
                count += b - a;
            }
            base += sg.second - sg.first;
        }
        if (first < 0) first = 0;
    };
    // 16 CTAs first: the band work is spread over twice the SMs of a portable 8-CTA cluster.
    for (int ranks : {16, 8}) {
        if (ranks > ny) continue;
        Cluster2D t{};
        t.ranks = ranks;
        t.w = nx;
        t.h = ny;
        t.rx_e = g.rows[0][0];
        t.rx_h = g.rows[1][0];
        for (int r = 0; r <= ranks; ++r) t.r0[r] = (int)((long long)r * ny / ranks);
        for (int r = 0; r < ranks; ++r) {
            t.rows_max = std::max(t.rows_max, t.r0[r + 1] - t.r0[r]);
            slab_rows(0, t.r0[r], t.r0[r + 1], t.rye_lo[r], t.rye_n[r]);
            slab_rows(1, t.r0[r], t.r0[r + 1], t.ryh_lo[r], t.ryh_n[r]);
            t.rye_max = std::max(t.rye_max, t.rye_n[r]);
            t.ryh_max = std::max(t.ryh_max, t.ryh_n[r]);
        }
        const size_t bytes = (size_t)cl2d_layout(t, (int)sizeof(T)).total * sizeof(T);
        if (bytes > (size_t)max_smem) continue;
        TFD_CUDA(cudaFuncSetAttribute(k_step2d_cluster<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        if (ranks > 8) TFD_CUDA(cudaFuncSetAttribute(k_step2d_cluster<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)ranks);
        cfg.blockDim = dim3(kCl2dThreads);
        cfg.dynamicSmemBytes = bytes;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)ranks;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_step2d_cluster<T>, &cfg) != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            continue;
        }
        c = t;
        p->cluster2d_smem = bytes;
        break;
    }
    return TFD_OK;
}

template <typename T>
int launch_cluster2d(tfd_plan *p, int nsteps, cudaStream_t s) {
    Cluster2D c = p->cluster2d;
    c.count = nsteps;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)c.ranks);
    cfg.blockDim = dim3(kCl2dThreads);
    cfg.dynamicSmemBytes = p->cluster2d_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)c.ranks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TFD_CUDA(cudaLaunchKernelEx(&cfg, k_step2d_cluster<T>, p->grid<T>(), c, (const TraceDev *)(p->arena + p->L.trace_tab),
                                p->desc.n_traces, p->ptr<T>(p->L.trace_out)));
    return TFD_OK;
}

// One persistent launch of `nsteps` 2D steps with their observations (cooperative: every CTA resident).
template <typename T>
int launch_persist2d(tfd_plan *p, int nsteps, cudaStream_t s) {
    const MonitorArgs<T> m = monitor_args<T>(p);
    const int mgx = std::max(1, (p->max_samples + kMonitorThreads - 1) / kMonitorThreads), mgy = std::max(1, p->desc.n_planes);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)p->persist_ctas);
    cfg.blockDim = dim3(k2dThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // The barrier words start every launch at zero: a launch that timed out leaves its arrival count behind.
    TFD_CUDA(cudaMemsetAsync(p->arena + p->L.grid_bar, 0, 2 * sizeof(unsigned), s));
    TFD_CUDA(cudaLaunchKernelEx(&cfg, k_step2d_persistent<T>, (const Grid<T> *)(p->arena + p->L.grid_tab),
                                (const Tile2D *)(p->arena + p->L.tile_tab), p->tile2d_interior, p->L.tiles2d, m, mgx, mgy, nsteps,
                                p->ptr<unsigned>(p->L.grid_bar)));
    return TFD_OK;
}

// One split step (plans with TFSF boxes or dispersive materials): the split gather E kernel, the boxes' E half
// step and E corrections, the split gather H kernel, the H half step and H corrections (the observation launch
// follows in step_t).
template <typename T>
int launch_split_step(tfd_plan *p, cudaStream_t s) {
    const Grid<T> &g = p->grid<T>();
    TfsfArgs<T> a = p->tfsf<T>();
    for (int par = 0; par < 2; ++par)
        for (int c = 0; c < 3; ++c) {
            a.E[par][c] = g.E[par][c];
            a.H[par][c] = g.H[par][c];
        }
    a.counter = g.counter;
    int longest = 1;
    for (int k = 0; k < a.boxes; ++k) longest = std::max(longest, a.box[k].count + std::max(a.box[k].n[0], a.box[k].n[1]));
    const dim3 tgrid((unsigned)((longest + kTfsfThreads - 1) / kTfsfThreads), (unsigned)a.boxes);
    dim3 block(128), grid((unsigned)((long long)g.n[1] * g.n[2]), (unsigned)((g.n[0] + 127) / 128));
    switch (g.active) {
        case kMaskTM: k_step_gather_e<T, kMaskTM><<<grid, block, 0, s>>>(g); break;
        case kMaskTE: k_step_gather_e<T, kMaskTE><<<grid, block, 0, s>>>(g); break;
        default: k_step_gather_e<T, kMaskAll><<<grid, block, 0, s>>>(g); break;
    }
    if (a.boxes > 0) k_tfsf<T><<<tgrid, kTfsfThreads, 0, s>>>(a, 0);
    switch (g.active) {
        case kMaskTM: k_step_gather_h<T, kMaskTM><<<grid, block, 0, s>>>(g); break;
        case kMaskTE: k_step_gather_h<T, kMaskTE><<<grid, block, 0, s>>>(g); break;
        default: k_step_gather_h<T, kMaskAll><<<grid, block, 0, s>>>(g); break;
    }
    if (a.boxes > 0) k_tfsf<T><<<tgrid, kTfsfThreads, 0, s>>>(a, 1);
    return TFD_OK;
}

template <typename T>
int step_t(tfd_plan *p, int nsteps, cudaStream_t s) {
    if (p->kernel == TFD_KERNEL_TILE2D && p->cluster2d.ranks > 0 && !p->in_batch) {
        if (nsteps > 0) TFD_CHECK(launch_cluster2d<T>(p, nsteps, s));
        return TFD_OK;
    }
    if (p->kernel == TFD_KERNEL_TILE2D && p->persist_ctas > 0 && !p->in_batch) {
        if (nsteps > 0) TFD_CHECK(launch_persist2d<T>(p, nsteps, s));
        return TFD_OK;
    }
    const MonitorArgs<T> m = monitor_args<T>(p);
    dim3 mgrid((unsigned)std::max(1, (p->max_samples + kMonitorThreads - 1) / kMonitorThreads), (unsigned)std::max(1, p->desc.n_planes));
    for (int k = 0; k < nsteps; ++k) {
        if (p->split) {
            TFD_CHECK(launch_split_step<T>(p, s));
        } else if (p->kernel == TFD_KERNEL_MARCH) {
            launch_march_any<T>(p, s);
        } else if (p->kernel == TFD_KERNEL_TILE2D) {
            launch_tile2d<T>(p, s);
        } else {
            int rc = launch_step_gather<T>(p, s);
            if (rc) return rc;
        }
        k_monitor<T><<<mgrid, kMonitorThreads, 0, s>>>(m);
    }
    TFD_CUDA(cudaGetLastError());
    return TFD_OK;
}

template <typename T>
int diagnose_t(tfd_plan *p, double out[3], cudaStream_t s) {
    long long counter = 0;
    TFD_CUDA(cudaMemcpyAsync(&counter, p->arena + p->L.counter, sizeof(long long), cudaMemcpyDeviceToHost, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    const int par = (int)(counter & 1);
    Grid<T> &g = p->grid<T>();
    DiagArgs<T> d;
    std::memset(&d, 0, sizeof(d));
    d.fs = field_set<T>(p);
    for (int c = 0; c < 3; ++c) d.inv_eps[c] = g.inv_eps[c];
    d.nx = g.n[0];
    d.ny = g.n[1];
    d.nz = g.n[2];
    d.pitch = g.pitch;
    d.counter = g.counter;
    const Layout &L = p->L;
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 2; ++j) {
            if (g.psiE[par][a][j]) { d.psi[d.n_psi] = g.psiE[par][a][j]; d.psi_len[d.n_psi++] = L.psi_len[0][a]; }
            if (g.psiH[a][j]) { d.psi[d.n_psi] = g.psiH[a][j]; d.psi_len[d.n_psi++] = L.psi_len[1][a]; }
        }
    for (int a = 0; a < 3; ++a) d.volume[a] = L.volume[a] ? p->ptr<double>(L.volume[a]) : nullptr;
    const TfsfArgs<T> &ta = p->tfsf<T>();
    for (int k = 0; k < ta.boxes; ++k) {
        const TfsfBoxDev<T> &bx = ta.box[k];
        // Line E weighed like E times the background index, line H like H; both CPML memories checked finite.
        d.line[d.n_lines] = bx.e;
        d.line_len[d.n_lines] = bx.count;
        d.line_factor[d.n_lines] = p->tfsf_index[k];
        d.line_weight[d.n_lines++] = (double)(T)p->tfsf_norm[k];
        d.line[d.n_lines] = bx.h;
        d.line_len[d.n_lines] = bx.count;
        d.line_factor[d.n_lines] = 1.0;
        d.line_weight[d.n_lines++] = (double)(T)p->tfsf_norm[k];
        d.psi[d.n_psi] = bx.pe;
        d.psi_len[d.n_psi++] = bx.count;
        d.psi[d.n_psi] = bx.ph;
        d.psi_len[d.n_psi++] = bx.count;
    }
    d.n_ade = g.n_ade;
    for (int k = 0; k < g.n_ade; ++k) {
        d.ade_P[k] = g.ade[k].P;
        d.ade_Q[k] = g.ade[k].Q;
        d.ade_samples[k] = g.ade[k].samples;
        d.ade_poles[k] = g.ade[k].poles;
        for (int q = 0; q < g.ade[k].poles; ++q) {
            d.ade_cq[k][q] = p->ade_cq[k][q];
            d.ade_cp[k][q] = p->ade_cp[k][q];
        }
        d.ade_weight[k] = L.ade[k].weight ? p->ptr<double>(L.ade[k].weight) : nullptr;
    }
    d.partial = p->ptr<double>(L.diag);
    k_diag<T><<<kDiagBlocks, kDiagThreads, 0, s>>>(d);
    TFD_CUDA(cudaGetLastError());
    std::vector<double> part((size_t)kDiagBlocks * 4);
    TFD_CUDA(cudaMemcpyAsync(part.data(), d.partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    double energy = 0, peak = 0, finite = 1, nan_seen = 0;
    for (int b = 0; b < kDiagBlocks; ++b) {
        energy += part[4 * b];
        peak = std::max(peak, part[4 * b + 1]);
        finite = std::min(finite, part[4 * b + 2]);
        nan_seen = std::max(nan_seen, part[4 * b + 3]);
    }
    out[0] = energy;
    out[1] = nan_seen > 0 ? NAN : peak;
    out[2] = finite;
    return TFD_OK;
}

template <typename T>
int slice_t(tfd_plan *p, int comp, int axis, int index, void *dst, int where, cudaStream_t s) {
    const tfd_desc &d = p->desc;
    const int n[3] = {d.nx, d.ny, d.nz};
    if (comp < 0 || comp > 5 || axis < 0 || axis > 2 || index < 0 || index >= n[axis]) return fail(TFD_ERR_INVALID, "bad slice");
    const int ua = axis == 0 ? 1 : 0, va = axis == 2 ? 1 : 2;
    const long long total = (long long)n[ua] * n[va];
    void *dev = where == TFD_DEVICE ? dst : p->arena + p->L.stage;
    k_slice<T><<<launch_blocks(total), 256, 0, s>>>((T *)dev, field_set<T>(p), comp, axis, index, d.nx, d.ny, d.nz, p->L.pitch,
                                                    p->grid<T>().counter);
    TFD_CUDA(cudaGetLastError());
    if (where == TFD_HOST) {
        TFD_CUDA(cudaMemcpyAsync(dst, dev, total * sizeof(T), cudaMemcpyDeviceToHost, s));
        TFD_CUDA(cudaStreamSynchronize(s));
    }
    return TFD_OK;
}

template <typename T>
int reset_t(tfd_plan *p, cudaStream_t s) { return zero_state<T>(p, s); }

#define TFD_DISPATCH(p, fn, ...) ((p)->desc.precision == 8 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

}  // namespace

extern "C" {

const char *tfd_error_string(int code) {
    switch (code) {
        case TFD_OK: return "ok";
        case TFD_ERR_INVALID: return "invalid argument";
        case TFD_ERR_UNSUPPORTED: return "unsupported feature";
        case TFD_ERR_CUDA: return "CUDA error";
        case TFD_ERR_ARENA: return "arena too small or misaligned";
        case TFD_ERR_DEVICE: return "device status error";
        default: return "unknown error";
    }
}

const char *tfd_last_error(void) { return g_error.c_str(); }

int tfd_plan_bytes(const tfd_desc *desc, size_t *bytes) {
    int rc = validate(desc);
    if (rc) return rc;
    if (!bytes) return fail(TFD_ERR_INVALID, "bytes is null");
    Layout L;
    compute_layout(desc, L);
    *bytes = L.total;
    return TFD_OK;
}

int tfd_plan_create(const tfd_desc *desc, void *arena, size_t arena_bytes, void *stream, tfd_plan **out) {
    int rc = validate(desc);
    if (rc) return rc;
    if (!out) return fail(TFD_ERR_INVALID, "plan output is null");
    *out = nullptr;
    tfd_plan *p = new tfd_plan();
    p->desc = *desc;
    p->desc.segments = nullptr;
    p->desc.sources = nullptr;
    p->desc.traces = nullptr;
    p->desc.planes = nullptr;
    compute_layout(desc, p->L);
    if (!arena || ((uintptr_t)arena & 255) || arena_bytes < p->L.total) {
        delete p;
        return fail(TFD_ERR_ARENA, "arena must be 256-byte aligned and at least tfd_plan_bytes() long");
    }
    p->arena = (char *)arena;
    size_t total;
    p->psi_segs = psi_segments(desc, &total);
    for (int k = 0; k < desc->n_segments; ++k) {
        p->seg_f.push_back(desc->segments[k].forward);
        p->seg_a.push_back(desc->segments[k].axis);
        p->seg_lo.push_back(desc->segments[k].lo);
        p->seg_hi.push_back(desc->segments[k].hi);
    }
    for (int k = 0; k < desc->n_ade; ++k) {
        const tfd_ade &m = desc->ade[k];
        std::vector<double> cq(m.poles), cp(m.poles);
        for (int q = 0; q < m.poles; ++q) {
            cq[q] = desc->time_step * std::sqrt(m.strength[q]);
            cp[q] = m.w0[q] / std::sqrt(m.strength[q]);
        }
        p->ade_cq.push_back(cq);
        p->ade_cp.push_back(cp);
    }
    for (int k = 0; k < desc->n_planes; ++k) {
        p->planes_f.push_back(desc->planes[k].frequencies);
        p->planes_p.push_back(desc->planes[k].points);
        p->planes_c.push_back(desc->planes[k].components);
    }
    cudaStream_t s = as_stream(stream);
    rc = desc->precision == 8 ? create_typed<double>(p, desc, s) : create_typed<float>(p, desc, s);
    if (!rc) {
        const bool march_ok = desc->precision == 8 ? march_supported<double>(p) : march_supported<float>(p);
        const bool tile_ok = tile2d_capable(desc);
        if (desc->kernel == TFD_KERNEL_MARCH && !march_ok)
            rc = fail(TFD_ERR_UNSUPPORTED, "the marching kernel needs a 3D grid");
        else if (desc->kernel == TFD_KERNEL_TILE2D && !tile_ok)
            rc = fail(TFD_ERR_UNSUPPORTED, "the 2D tile kernel needs a 2D TMz grid without periodic x/y faces");
        p->split = desc->n_tfsf > 0 || desc->n_ade > 0;
        if (p->split && (desc->kernel == TFD_KERNEL_MARCH || desc->kernel == TFD_KERNEL_TILE2D))
            rc = fail(TFD_ERR_UNSUPPORTED, "plans with TFSF boxes or dispersive materials run the split gather kernels");
        if (desc->kernel == TFD_KERNEL_GATHER || p->split) p->kernel = TFD_KERNEL_GATHER;
        else if (march_ok) p->kernel = TFD_KERNEL_MARCH;
        else if (tile_ok) p->kernel = TFD_KERNEL_TILE2D;
        else p->kernel = TFD_KERNEL_GATHER;
        if (!rc && p->kernel == TFD_KERNEL_MARCH) rc = TFD_DISPATCH(p, setup_march, p);
        if (!rc && tile_ok && !p->split) rc = TFD_DISPATCH(p, setup_tile2d, p, s);
    }
    if (!rc) rc = TFD_DISPATCH(p, zero_state, p, s);
    if (!rc) {
        const long long n = p->L.count;
        for (int q = 0; q < desc->material_samples; ++q) {
            if (desc->precision == 8) k_fill<double><<<launch_blocks(n), 256, 0, s>>>((double *)(p->arena + p->L.inv[q]), n, 1.0);
            else k_fill<float><<<launch_blocks(n), 256, 0, s>>>((float *)(p->arena + p->L.inv[q]), n, 1.0f);
        }
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = fail(TFD_ERR_CUDA, std::string("plan setup: ") + cudaGetErrorString(e));
    }
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return TFD_OK;
}

void tfd_plan_destroy(tfd_plan *plan) { delete plan; }

int tfd_set_material(tfd_plan *p, const void *inv_eps, int where, void *stream) {
    if (!p || !inv_eps) return fail(TFD_ERR_INVALID, "null argument");
    return TFD_DISPATCH(p, set_material_t, p, inv_eps, where, as_stream(stream));
}

int tfd_set_permittivity(tfd_plan *p, const void *eps, int where, void *stream) {
    if (!p || !eps) return fail(TFD_ERR_INVALID, "null argument");
    return TFD_DISPATCH(p, set_permittivity_t, p, eps, where, as_stream(stream));
}

int tfd_field_check(tfd_plan *p, double *peak_e, int32_t *finite, void *stream) {
    if (!p || !peak_e || !finite) return fail(TFD_ERR_INVALID, "null argument");
    return TFD_DISPATCH(p, field_check_t, p, peak_e, finite, as_stream(stream));
}

int tfd_set_fields(tfd_plan *p, const void *E, const void *H, int where, void *stream) {
    if (!p) return fail(TFD_ERR_INVALID, "null plan");
    return TFD_DISPATCH(p, set_fields_t, p, E, H, where, as_stream(stream));
}

int tfd_get_fields(tfd_plan *p, void *E, void *H, int where, void *stream) {
    if (!p) return fail(TFD_ERR_INVALID, "null plan");
    return TFD_DISPATCH(p, get_fields_t, p, E, H, where, as_stream(stream));
}

int tfd_psi_count(const tfd_plan *p, size_t *count) {
    if (!p || !count) return fail(TFD_ERR_INVALID, "null argument");
    *count = p->L.psi_total;
    return TFD_OK;
}

int tfd_set_psi(tfd_plan *p, const void *psi, int where, void *stream) {
    if (!p || !psi) return fail(TFD_ERR_INVALID, "null argument");
    return TFD_DISPATCH(p, psi_t, p, (void *)psi, where, as_stream(stream), false);
}

int tfd_get_psi(tfd_plan *p, void *psi, int where, void *stream) {
    if (!p || !psi) return fail(TFD_ERR_INVALID, "null argument");
    return TFD_DISPATCH(p, psi_t, p, psi, where, as_stream(stream), true);
}

int tfd_step(tfd_plan *p, int32_t nsteps, void *stream) {
    if (!p) return fail(TFD_ERR_INVALID, "null plan");
    if (p->in_batch) return fail(TFD_ERR_INVALID, "this plan belongs to a batch: advance it with tfd_batch_step");
    if (nsteps < 0) return fail(TFD_ERR_INVALID, "nsteps must be non-negative");
    return TFD_DISPATCH(p, step_t, p, nsteps, as_stream(stream));
}

int tfd_reset(tfd_plan *p, void *stream) {
    if (!p) return fail(TFD_ERR_INVALID, "null plan");
    if (p->in_batch) return fail(TFD_ERR_INVALID, "this plan belongs to a batch: destroy the batch before resetting it");
    return TFD_DISPATCH(p, reset_t, p, as_stream(stream));
}

int tfd_get_traces(tfd_plan *p, void *dst, int where, void *stream) {
    if (!p || !dst) return fail(TFD_ERR_INVALID, "null argument");
    const size_t bytes = (size_t)p->desc.n_traces * p->desc.steps * p->L.elem;
    if (!bytes) return TFD_OK;
    cudaStream_t s = as_stream(stream);
    TFD_CUDA(cudaMemcpyAsync(dst, p->arena + p->L.trace_out, bytes, where == TFD_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    if (where == TFD_HOST) TFD_CUDA(cudaStreamSynchronize(s));
    return TFD_OK;
}

int tfd_get_plane(tfd_plan *p, int32_t k, void *dst, int where, void *stream) {
    if (!p || !dst || k < 0 || k >= p->desc.n_planes) return fail(TFD_ERR_INVALID, "bad plane request");
    const size_t bytes = (size_t)p->planes_f[k] * p->planes_p[k] * p->planes_c[k] * 2 * sizeof(double);
    if (!bytes) return TFD_OK;
    cudaStream_t s = as_stream(stream);
    TFD_CUDA(cudaMemcpyAsync(dst, p->arena + p->L.planes[k].acc, bytes, where == TFD_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    if (where == TFD_HOST) TFD_CUDA(cudaStreamSynchronize(s));
    return TFD_OK;
}

int tfd_get_slice(tfd_plan *p, int32_t component, int32_t axis, int32_t index, void *dst, int where, void *stream) {
    if (!p || !dst) return fail(TFD_ERR_INVALID, "null argument");
    return TFD_DISPATCH(p, slice_t, p, component, axis, index, dst, where, as_stream(stream));
}

int tfd_diagnose(tfd_plan *p, double out[3], void *stream) {
    if (!p || !out) return fail(TFD_ERR_INVALID, "null argument");
    return TFD_DISPATCH(p, diagnose_t, p, out, as_stream(stream));
}

int tfd_counter(tfd_plan *p, int64_t *value, void *stream) {
    if (!p || !value) return fail(TFD_ERR_INVALID, "null argument");
    cudaStream_t s = as_stream(stream);
    long long v = 0;
    TFD_CUDA(cudaMemcpyAsync(&v, p->arena + p->L.counter, sizeof(long long), cudaMemcpyDeviceToHost, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    *value = v;
    return TFD_OK;
}

int tfd_device_status(tfd_plan *p, int32_t *status, void *stream) {
    if (!p || !status) return fail(TFD_ERR_INVALID, "null argument");
    cudaStream_t s = as_stream(stream);
    int v = 0;
    TFD_CUDA(cudaMemcpyAsync(&v, p->arena + p->L.status, sizeof(int), cudaMemcpyDeviceToHost, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    *status = v;
    return TFD_OK;
}

int tfd_kernel_in_use(const tfd_plan *p, int32_t *kernel) {
    if (!p || !kernel) return fail(TFD_ERR_INVALID, "null argument");
    *kernel = p->kernel;
    return TFD_OK;
}

int tfd_step_launches(const tfd_plan *p, int32_t nsteps, int64_t *launches) {
    if (!p || !launches) return fail(TFD_ERR_INVALID, "null argument");
    if (nsteps < 0) return fail(TFD_ERR_INVALID, "nsteps must be non-negative");
    long long per_step = 2;                                   // gather: step + observation
    if (p->split) {
        per_step = p->desc.n_tfsf > 0 ? 5 : 3;                // split E, (TFSF E), split H, (TFSF H), observation
    } else if (p->kernel == TFD_KERNEL_TILE2D) {
        if ((p->persist_ctas > 0 || p->cluster2d.ranks > 0) && !p->in_batch) {
            *launches = nsteps > 0 ? 1 : 0;
            return TFD_OK;
        }
        per_step = (p->tile2d_interior > 0) + (p->L.tiles2d > p->tile2d_interior) + 1;
    } else if (p->kernel == TFD_KERNEL_MARCH) {
        per_step = (long long)p->march_launches.size() + 1;
    }
    *launches = per_step * nsteps;
    return TFD_OK;
}

}  // extern "C"

// ---- batches ---------------------------------------------------------------------------------------------
struct tfd_batch {
    std::vector<tfd_plan *> plans;
    int precision = 4;
    char *arena = nullptr;
    size_t counter = 0, done = 0, grids = 0, tiles = 0, mon = 0, total = 0;
    int ntiles = 0, interior = 0, capacity = 0, rows = 8, ctas = 0, max_planes = 0, max_chunks = 1;
    SideStream side;
    long long cells = 0;
    size_t bar = 0;                // persistent stepping: arrival count and generation
    int persist_ctas = 0;          // > 0: all steps of a tfd_batch_step call in one cooperative launch
};

namespace {

int batch_layout(tfd_batch &b, int n, tfd_plan *const *plans) {
    if (n < 1 || !plans) return fail(TFD_ERR_INVALID, "a batch needs at least one plan");
    b.plans.assign(plans, plans + n);
    b.precision = plans[0] ? plans[0]->desc.precision : 4;
    b.ntiles = 0;
    b.capacity = 0;
    b.cells = 0;
    for (int i = 0; i < n; ++i) {
        tfd_plan *p = plans[i];
        if (!p) return fail(TFD_ERR_INVALID, "null plan in batch");
        if (p->desc.precision != b.precision) return fail(TFD_ERR_INVALID, "batched plans must share one precision");
        if (p->L.tiles2d == 0) return fail(TFD_ERR_UNSUPPORTED, "batches run 2D TMz grids without periodic x/y faces");
        if (p->in_batch) return fail(TFD_ERR_INVALID, "a plan belongs to another batch");
        for (int j = 0; j < i; ++j)
            if (plans[j] == p) return fail(TFD_ERR_INVALID, "a plan appears twice in the batch");
        // The strip table is sized for the shortest strips (8 rows) so any strip length fits later.
        b.capacity += strip_capacity(p->desc.nx, p->desc.ny);
        b.cells += (long long)p->desc.nx * p->desc.ny;
    }
    const size_t grid_bytes = b.precision == 8 ? sizeof(Grid<double>) : sizeof(Grid<float>);
    const size_t mon_bytes = b.precision == 8 ? sizeof(MonitorArgs<double>) : sizeof(MonitorArgs<float>);
    Bump bump;
    b.counter = bump.take(sizeof(long long));
    b.done = bump.take(sizeof(unsigned));
    b.grids = bump.take(n * grid_bytes);
    b.tiles = bump.take((size_t)b.capacity * sizeof(Tile2D));
    b.mon = bump.take(n * mon_bytes);
    b.bar = bump.take(2 * sizeof(unsigned));
    b.total = bump.off + 256;
    return TFD_OK;
}

// Rebuild the batch's strip table for strips of `rows` rows (grid by grid, x-fastest).
template <typename T>
int batch_strips_t(tfd_batch *b, int rows, cudaStream_t s) {
    std::vector<Tile2D> tiles;
    for (size_t i = 0; i < b->plans.size(); ++i) {
        std::vector<Tile2D> t = strips_of(strip_geom<T>(b->plans[i]), (int)i, rows);
        tiles.insert(tiles.end(), t.begin(), t.end());
    }
    if ((int)tiles.size() > b->capacity) return fail(TFD_ERR_INVALID, "strip table exceeds the batch arena");
    // Interior strips of every member first: the lean kernel walks [0, interior) of the whole table.
    std::stable_partition(tiles.begin(), tiles.end(), [](const Tile2D &a) { return a.kind == 1; });
    TFD_CUDA(cudaMemcpyAsync(b->arena + b->tiles, tiles.data(), tiles.size() * sizeof(Tile2D), cudaMemcpyHostToDevice, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    b->ntiles = (int)tiles.size();
    b->interior = interior_count(tiles);
    b->rows = rows;
    return TFD_OK;
}

template <typename T>
int batch_create_t(tfd_batch *b, cudaStream_t s) {
    const int n = (int)b->plans.size();
    long long *counter = (long long *)(b->arena + b->counter);
    std::vector<Grid<T>> grids;
    std::vector<MonitorArgs<T>> mons;
    for (int i = 0; i < n; ++i) {
        tfd_plan *p = b->plans[i];
        long long value = -1;
        TFD_CUDA(cudaMemcpyAsync(&value, p->grid<T>().counter, sizeof(long long), cudaMemcpyDeviceToHost, s));
        TFD_CUDA(cudaStreamSynchronize(s));
        if (value != 0) return fail(TFD_ERR_INVALID, "batched plans must start at step 0 (tfd_reset them)");
    }
    for (int i = 0; i < n; ++i) {
        tfd_plan *p = b->plans[i];
        Grid<T> &g = p->grid<T>();
        p->own_counter = g.counter;
        g.counter = counter;                         // members read the batch's shared step counter
        p->in_batch = true;
        grids.push_back(g);
        MonitorArgs<T> m = monitor_args<T>(p);
        mons.push_back(m);
        b->max_planes = std::max(b->max_planes, p->desc.n_planes);
        b->max_chunks = std::max(b->max_chunks, (p->max_samples + kMonitorThreads - 1) / kMonitorThreads);
    }
    TFD_CUDA(cudaMemsetAsync(b->arena + b->counter, 0, sizeof(long long), s));
    TFD_CUDA(cudaMemsetAsync(b->arena + b->done, 0, sizeof(unsigned), s));
    TFD_CUDA(cudaMemcpyAsync(b->arena + b->grids, grids.data(), grids.size() * sizeof(Grid<T>), cudaMemcpyHostToDevice, s));
    TFD_CUDA(cudaMemcpyAsync(b->arena + b->mon, mons.data(), mons.size() * sizeof(MonitorArgs<T>), cudaMemcpyHostToDevice, s));
    TFD_CUDA(cudaStreamSynchronize(s));
    cudaFuncAttributes attr;                     // loads the monitor kernel now, before any graph capture
    TFD_CUDA(cudaFuncGetAttributes(&attr, (const void *)k_monitor_batch<T>));
    b->ctas = 0;
    TFD_CHECK(b->side.create());
    return batch_strips_t<T>(b, strip_rows(b->cells), s);
}

// The CTAs of a persistent batch launch: a warp per strip (or b->ctas when set), at least one CTA per
// observation work item, no more than can be resident together.
template <typename T>
int batch_persist_ctas(tfd_batch *b, int &ctas) {
    int device = 0, sms = 148, per_sm = 0;
    TFD_CUDA(cudaGetDevice(&device));
    TFD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    TFD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step2d_batch_persistent<T>, k2dThreads, 0));
    const int items = (int)b->plans.size() * b->max_chunks * std::max(1, b->max_planes);
    const int want = b->ctas > 0 ? b->ctas : std::max({1, (b->ntiles + k2dWarps - 1) / k2dWarps, items});
    ctas = per_sm > 0 ? std::min(want, per_sm * sms) : 0;
    return ctas > 0 ? TFD_OK : fail(TFD_ERR_UNSUPPORTED, "the persistent batch kernel cannot be resident on this device");
}

template <typename T>
int batch_persistent_step(tfd_batch *b, int nsteps, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)b->persist_ctas);
    cfg.blockDim = dim3(k2dThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const Grid<T> *grids = (const Grid<T> *)(b->arena + b->grids);
    TFD_CUDA(cudaMemsetAsync(b->arena + b->bar, 0, 2 * sizeof(unsigned), s));
    TFD_CUDA(cudaLaunchKernelEx(&cfg, k_step2d_batch_persistent<T>, grids, (const Tile2D *)(b->arena + b->tiles), b->interior,
                                b->ntiles, (const MonitorArgs<T> *)(b->arena + b->mon), (int)b->plans.size(), b->max_chunks,
                                std::max(1, b->max_planes), (long long *)(b->arena + b->counter), nsteps,
                                (unsigned *)(b->arena + b->bar), b->plans[0]->grid<T>().status));
    return TFD_OK;
}

template <typename T>
int batch_step_t(tfd_batch *b, int nsteps, cudaStream_t s) {
    if (b->persist_ctas > 0) return nsteps > 0 ? batch_persistent_step<T>(b, nsteps, s) : TFD_OK;
    long long *counter = (long long *)(b->arena + b->counter);
    const dim3 mgrid((unsigned)b->max_chunks, (unsigned)std::max(1, b->max_planes), (unsigned)b->plans.size());
    for (int k = 0; k < nsteps; ++k) {
        launch_strips<T>((const Grid<T> *)(b->arena + b->grids), (const Tile2D *)(b->arena + b->tiles), b->interior, b->ntiles,
                         b->ctas, counter, s, &b->side);
        k_monitor_batch<T><<<mgrid, kMonitorThreads, 0, s>>>((const MonitorArgs<T> *)(b->arena + b->mon), counter,
                                                             (unsigned *)(b->arena + b->done));
    }
    TFD_CUDA(cudaGetLastError());
    return TFD_OK;
}

template <typename T>
void batch_release_t(tfd_batch *b) {
    // Hand the step count back to every member (capped at its own run length: a finished grid was
    // skipped from then on) and restore its own counter.
    long long n = 0;
    cudaMemcpy(&n, b->arena + b->counter, sizeof(long long), cudaMemcpyDeviceToHost);
    for (tfd_plan *p : b->plans) {
        Grid<T> &g = p->grid<T>();
        if (p->own_counter) {
            const long long mine = std::min<long long>(n, p->desc.steps);
            cudaMemcpy(p->own_counter, &mine, sizeof(long long), cudaMemcpyHostToDevice);
            g.counter = p->own_counter;
            p->own_counter = nullptr;
        }
        p->in_batch = false;
    }
}

}  // namespace

extern "C" {

int tfd_batch_bytes(int32_t n_plans, tfd_plan *const *plans, size_t *bytes) {
    if (!bytes) return fail(TFD_ERR_INVALID, "bytes is null");
    tfd_batch b;
    int rc = batch_layout(b, n_plans, plans);
    if (rc) return rc;
    *bytes = b.total;
    return TFD_OK;
}

int tfd_batch_create(int32_t n_plans, tfd_plan *const *plans, void *arena, size_t arena_bytes, void *stream, tfd_batch **out) {
    if (!out) return fail(TFD_ERR_INVALID, "batch output is null");
    *out = nullptr;
    tfd_batch *b = new tfd_batch();
    int rc = batch_layout(*b, n_plans, plans);
    if (!rc && (!arena || ((uintptr_t)arena & 255) || arena_bytes < b->total))
        rc = fail(TFD_ERR_ARENA, "batch arena must be 256-byte aligned and at least tfd_batch_bytes() long");
    if (rc) {
        delete b;
        return rc;
    }
    b->arena = (char *)arena;
    rc = b->precision == 8 ? batch_create_t<double>(b, as_stream(stream)) : batch_create_t<float>(b, as_stream(stream));
    if (rc) {
        if (b->precision == 8) batch_release_t<double>(b); else batch_release_t<float>(b);
        delete b;
        return rc;
    }
    *out = b;
    return TFD_OK;
}

int tfd_batch_set_launch(tfd_batch *b, int32_t ctas, int32_t strip_rows, void *stream) {
    if (!b || ctas < 0 || strip_rows < 0 || (strip_rows > 0 && strip_rows < 8))
        return fail(TFD_ERR_INVALID, "bad batch launch: ctas >= 0, strip_rows 0 or >= 8");
    const int rows = strip_rows == 0 ? tfd::strip_rows(b->cells) : strip_rows;
    if (rows != b->rows) {
        const int rc = b->precision == 8 ? batch_strips_t<double>(b, rows, as_stream(stream))
                                         : batch_strips_t<float>(b, rows, as_stream(stream));
        if (rc) return rc;
    }
    b->ctas = ctas;
    if (b->persist_ctas > 0) {                   // keep a persistent launch sized for the new table
        int n = 0;
        const int rc = b->precision == 8 ? batch_persist_ctas<double>(b, n) : batch_persist_ctas<float>(b, n);
        if (rc) return rc;
        b->persist_ctas = n;
    }
    return TFD_OK;
}

int tfd_batch_set_persistent(tfd_batch *b, int32_t persistent, void *stream) {
    (void)stream;
    if (!b) return fail(TFD_ERR_INVALID, "null batch");
    if (!persistent) {
        b->persist_ctas = 0;
        return TFD_OK;
    }
    int ctas = 0;
    const int rc = b->precision == 8 ? batch_persist_ctas<double>(b, ctas) : batch_persist_ctas<float>(b, ctas);
    if (rc) return rc;
    b->persist_ctas = ctas;
    return TFD_OK;
}

int tfd_batch_step(tfd_batch *b, int32_t nsteps, void *stream) {
    if (!b || nsteps < 0) return fail(TFD_ERR_INVALID, "bad batch step");
    return b->precision == 8 ? batch_step_t<double>(b, nsteps, as_stream(stream)) : batch_step_t<float>(b, nsteps, as_stream(stream));
}

int tfd_batch_tiles(const tfd_batch *b, int32_t *tiles) {
    if (!b || !tiles) return fail(TFD_ERR_INVALID, "null argument");
    *tiles = b->ntiles;
    return TFD_OK;
}

void tfd_batch_destroy(tfd_batch *b) {
    if (!b) return;
    cudaDeviceSynchronize();
    if (b->precision == 8) batch_release_t<double>(b); else batch_release_t<float>(b);
    delete b;
}

}  // extern "C"

// ---- restart states and the discrete adjoint ---------------------------------------------------------
namespace {

constexpr int kStateArrays = 18;

// The restart state of a plan as a compact snapshot: the step counter (first 8 bytes), then E, H and the
// E-family CPML memories of the current parity and the H-family memories, each 256-byte aligned.
template <typename T>
struct StateCopy {
    int n;
    T *a[kStateArrays][2];       // [array][parity]; H-family memories have one buffer (both entries)
    long long len[kStateArrays];
    long long off[kStateArrays]; // element offset in the snapshot
};

struct StateMap {
    long long sE[3], sH[3], sPsiE[3][2], sPsiH[3][2];
    size_t bytes;
};

template <typename T>
StateMap state_layout(tfd_plan *p, StateCopy<T> *sc) {
    const Grid<T> &g = p->grid<T>();
    StateMap m;
    size_t off = 256;
    auto take = [&](long long elems) {
        const long long at = (long long)(off / sizeof(T));
        off += ((size_t)elems * sizeof(T) + 255) / 256 * 256;
        return at;
    };
    if (sc) sc->n = 0;
    auto add = [&](T *p0, T *p1, long long len) {
        const long long at = take(len);
        if (sc) {
            sc->a[sc->n][0] = p0;
            sc->a[sc->n][1] = p1;
            sc->len[sc->n] = len;
            sc->off[sc->n] = at;
            ++sc->n;
        }
        return at;
    };
    for (int c = 0; c < 3; ++c) m.sE[c] = g.E[0][c] ? add(g.E[0][c], g.E[1][c], g.count) : -1;
    for (int c = 0; c < 3; ++c) m.sH[c] = g.H[0][c] ? add(g.H[0][c], g.H[1][c], g.count) : -1;
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 2; ++j)
            m.sPsiE[a][j] = g.psiE[0][a][j] ? add(g.psiE[0][a][j], g.psiE[1][a][j], p->L.psi_len[0][a]) : -1;
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 2; ++j) m.sPsiH[a][j] = g.psiH[a][j] ? add(g.psiH[a][j], g.psiH[a][j], p->L.psi_len[1][a]) : -1;
    m.bytes = off;
    return m;
}

// Copies the state between the plan and a snapshot; the parity comes from the plan's counter (save) or
// from the snapshot's counter (load), read on the device, so the copy is stream-ordered and capturable.
template <typename T>
__global__ void k_state_copy(const __grid_constant__ StateCopy<T> sc, char *slot, long long *counter, int save) {
    const int k = blockIdx.y;
    const long long n = save ? *counter : *(const long long *)slot;
    const int par = (int)(n & 1);
    T *arr = sc.a[k][par];
    T *snap = (T *)slot + sc.off[k];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < sc.len[k]; e += (long long)gridDim.x * blockDim.x) {
        if (save) snap[e] = arr[e];
        else arr[e] = snap[e];
    }
    if (k == 0 && blockIdx.x == 0 && threadIdx.x == 0) {
        if (save) *(long long *)slot = n;
        else *counter = n;
    }
}

template <typename T>
int state_copy_t(tfd_plan *p, char *slot, bool save, cudaStream_t s) {
    StateCopy<T> sc;
    std::memset(&sc, 0, sizeof(sc));
    state_layout<T>(p, &sc);
    long long longest = 1;
    for (int k = 0; k < sc.n; ++k) longest = std::max(longest, sc.len[k]);
    const dim3 grid((unsigned)std::min<long long>((longest + 255) / 256, 1184), (unsigned)std::max(1, sc.n));
    k_state_copy<T><<<grid, 256, 0, s>>>(sc, slot, p->grid<T>().counter, save ? 1 : 0);
    TFD_CUDA(cudaGetLastError());
    return TFD_OK;
}

}  // namespace

struct tfd_adjoint {
    tfd_plan *p = nullptr;
    char *arena = nullptr;
    size_t used = 0;
    int q = 0;
    AdjArgs<float> af;
    AdjArgs<double> ad;
    template <typename T> AdjArgs<T> &args();
};
template <> AdjArgs<float> &tfd_adjoint::args<float>() { return af; }
template <> AdjArgs<double> &tfd_adjoint::args<double>() { return ad; }

namespace {

// Adjoint arena: e_bar, h_bar and both families' CPML memory bars by parity, and the sensitivity.
template <typename T>
size_t adjoint_layout(tfd_plan *p, AdjArgs<T> *A, char *arena) {
    const Grid<T> &g = p->grid<T>();
    Bump b;
    auto at = [&](size_t off) { return arena ? (T *)(arena + off) : nullptr; };
    const size_t field = (size_t)g.count * sizeof(T);
    for (int q = 0; q < 2; ++q)
        for (int c = 0; c < 3; ++c) {
            T *e = g.E[0][c] ? at(b.take(field)) : nullptr;
            T *h = g.H[0][c] ? at(b.take(field)) : nullptr;
            if (A) { A->eb[q][c] = e; A->hb[q][c] = h; }
        }
    for (int q = 0; q < 2; ++q)
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 2; ++j) {
                T *pe = g.psiE[0][a][j] ? at(b.take((size_t)p->L.psi_len[0][a] * sizeof(T))) : nullptr;
                T *ph = g.psiH[a][j] ? at(b.take((size_t)p->L.psi_len[1][a] * sizeof(T))) : nullptr;
                if (A) { A->pEb[q][a][j] = pe; A->pHb[q][a][j] = ph; }
            }
    for (int c = 0; c < 3; ++c) {
        T *sv = g.E[0][c] ? at(b.take(field)) : nullptr;
        if (A) A->S[c] = sv;
    }
    return b.off;
}

template <typename T>
int adjoint_create_t(tfd_adjoint *adj, cudaStream_t s) {
    tfd_plan *p = adj->p;
    AdjArgs<T> &A = adj->args<T>();
    std::memset(&A, 0, sizeof(A));
    A.g = p->grid<T>();
    const StateMap m = state_layout<T>(p, nullptr);
    for (int c = 0; c < 3; ++c) { A.sE[c] = m.sE[c]; A.sH[c] = m.sH[c]; }
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 2; ++j) A.sPsiE[a][j] = m.sPsiE[a][j];
    if (int rc = slab_bounds(p, A.slab)) return rc;
    if (A.g.n[2] > 65535) return fail(TFD_ERR_UNSUPPORTED, "the adjoint step launches one z plane per grid row: nz above 65535");
    adj->used = adjoint_layout<T>(p, &A, adj->arena);
    TFD_CUDA(cudaMemsetAsync(adj->arena, 0, adj->used, s));
    adj->q = 0;
    return TFD_OK;
}

template <typename T>
int adjoint_step_t(tfd_adjoint *adj, const void *snapshot, const void *seeds, cudaStream_t s) {
    tfd_plan *p = adj->p;
    const AdjArgs<T> &A = adj->args<T>();
    const int n_obs = p->desc.n_traces;
    if (seeds && n_obs > 0)
        k_adjoint_seed<T><<<std::max(1, std::min(1184, (n_obs + 255) / 256)), 256, 0, s>>>(A, p->ptr<TraceDev>(p->L.trace_tab), n_obs,
                                                                                       (const T *)seeds, adj->q);
    const Grid<T> &g = A.g;
    // x tiles at multiples of 32 (rows aligned to 128 bytes: measured 13 % faster for k_adjoint_e than tiles
    // starting at x = 1, which put one more column of tiles on the fast path); y tiles shifted to start at y = 1,
    // so the first tile row holds the y = 0 face alone. A tile whose cells all lie in [1, n-2] takes the fast path.
    const int exs = 0, eys = kAdjY - 1;
    const int hxs = exs, hys = eys;
    auto grid_of = [&](int xs, int ys) {
        return dim3((unsigned)((g.n[0] + xs + kAdjX - 1) / kAdjX), (unsigned)((g.n[1] + ys + kAdjY - 1) / kAdjY), (unsigned)g.n[2]);
    };
    const dim3 ge = grid_of(exs, eys), gh = grid_of(hxs, hys);
    const char *env = getenv("TFD_ADJ_FAST");
    const int fast = (env && std::atoi(env) == 0) ? 0 : 1;
    const dim3 block(kAdjX, kAdjY);
    const T *slot = (const T *)snapshot;
    switch (p->desc.components) {
        case kMaskTM:
            k_adjoint_e<T, kMaskTM><<<ge, block, 0, s>>>(A, slot, adj->q, exs, eys, fast);
            k_adjoint_h<T, kMaskTM><<<gh, block, 0, s>>>(A, adj->q, hxs, hys, fast);
            break;
        case kMaskTE:
            k_adjoint_e<T, kMaskTE><<<ge, block, 0, s>>>(A, slot, adj->q, exs, eys, fast);
            k_adjoint_h<T, kMaskTE><<<gh, block, 0, s>>>(A, adj->q, hxs, hys, fast);
            break;
        default:
            k_adjoint_e<T, kMaskAll><<<ge, block, 0, s>>>(A, slot, adj->q, exs, eys, fast);
            k_adjoint_h<T, kMaskAll><<<gh, block, 0, s>>>(A, adj->q, hxs, hys, fast);
            break;
    }
    TFD_CUDA(cudaGetLastError());
    adj->q ^= 1;
    return TFD_OK;
}

template <typename T>
int adjoint_sensitivity_t(tfd_adjoint *adj, void *dst, int where, cudaStream_t s) {
    tfd_plan *p = adj->p;
    const AdjArgs<T> &A = adj->args<T>();
    const tfd_desc &d = p->desc;
    const size_t bytes = (size_t)d.nx * d.ny * d.nz * 3 * sizeof(T);
    T *out = (T *)dst;
    T *staging = nullptr;
    if (where == TFD_HOST) {
        TFD_CUDA(cudaMallocAsync((void **)&staging, bytes, s));
        out = staging;
    }
    if (const unsigned tb = tiled_blocks(d))
        k_to_reference_tiled<T><<<tb, kTileThreads, 0, s>>>(out, tile_arrays<T>(A.S[0], A.S[1], A.S[2]), nullptr, 3, d.nx, d.ny, d.nz,
                                                            p->L.pitch);
    else
        k_internal_to_reference<T><<<launch_blocks((long long)d.nx * d.ny * d.nz * 3), 256, 0, s>>>(out, 3, d.nx, d.ny, d.nz,
                                                                                                p->L.pitch, A.S[0], A.S[1], A.S[2]);
    TFD_CUDA(cudaGetLastError());
    if (staging) {
        TFD_CUDA(cudaMemcpyAsync(dst, staging, bytes, cudaMemcpyDeviceToHost, s));
        TFD_CUDA(cudaFreeAsync(staging, s));
        TFD_CUDA(cudaStreamSynchronize(s));
    }
    return TFD_OK;
}

}  // namespace

extern "C" {

int tfd_state_bytes(tfd_plan *p, size_t *bytes) {
    if (!p || !bytes) return fail(TFD_ERR_INVALID, "null argument");
    *bytes = p->desc.precision == 8 ? state_layout<double>(p, nullptr).bytes : state_layout<float>(p, nullptr).bytes;
    return TFD_OK;
}

int tfd_state_save(tfd_plan *p, void *dst, void *stream) {
    if (!p || !dst || ((uintptr_t)dst & 255)) return fail(TFD_ERR_INVALID, "snapshot must be a 256-byte aligned device buffer");
    if (p->in_batch) return fail(TFD_ERR_INVALID, "this plan belongs to a batch");
    return p->desc.precision == 8 ? state_copy_t<double>(p, (char *)dst, true, as_stream(stream))
                                  : state_copy_t<float>(p, (char *)dst, true, as_stream(stream));
}

int tfd_state_load(tfd_plan *p, const void *src, void *stream) {
    if (!p || !src || ((uintptr_t)src & 255)) return fail(TFD_ERR_INVALID, "snapshot must be a 256-byte aligned device buffer");
    if (p->in_batch) return fail(TFD_ERR_INVALID, "this plan belongs to a batch");
    return p->desc.precision == 8 ? state_copy_t<double>(p, (char *)src, false, as_stream(stream))
                                  : state_copy_t<float>(p, (char *)src, false, as_stream(stream));
}

int tfd_adjoint_bytes(tfd_plan *p, size_t *bytes) {
    if (!p || !bytes) return fail(TFD_ERR_INVALID, "null argument");
    *bytes = (p->desc.precision == 8 ? adjoint_layout<double>(p, nullptr, nullptr) : adjoint_layout<float>(p, nullptr, nullptr)) + 256;
    return TFD_OK;
}

int tfd_adjoint_create(tfd_plan *p, void *arena, size_t arena_bytes, void *stream, tfd_adjoint **out) {
    if (!p || !out) return fail(TFD_ERR_INVALID, "null argument");
    *out = nullptr;
    size_t need = 0;
    tfd_adjoint_bytes(p, &need);
    if (!arena || ((uintptr_t)arena & 255) || arena_bytes < need)
        return fail(TFD_ERR_ARENA, "adjoint arena must be 256-byte aligned and at least tfd_adjoint_bytes() long");
    tfd_adjoint *adj = new tfd_adjoint();
    adj->p = p;
    adj->arena = (char *)arena;
    const int rc = p->desc.precision == 8 ? adjoint_create_t<double>(adj, as_stream(stream)) : adjoint_create_t<float>(adj, as_stream(stream));
    if (rc) {
        delete adj;
        return rc;
    }
    *out = adj;
    return TFD_OK;
}

int tfd_adjoint_reset(tfd_adjoint *adj, void *stream) {
    if (!adj) return fail(TFD_ERR_INVALID, "null adjoint");
    TFD_CUDA(cudaMemsetAsync(adj->arena, 0, adj->used, as_stream(stream)));
    adj->q = 0;
    return TFD_OK;
}

int tfd_adjoint_step(tfd_adjoint *adj, const void *snapshot, const void *seeds, void *stream) {
    if (!adj || !snapshot || ((uintptr_t)snapshot & 255)) return fail(TFD_ERR_INVALID, "bad adjoint step arguments");
    return adj->p->desc.precision == 8 ? adjoint_step_t<double>(adj, snapshot, seeds, as_stream(stream))
                                       : adjoint_step_t<float>(adj, snapshot, seeds, as_stream(stream));
}

int tfd_adjoint_sensitivity(tfd_adjoint *adj, void *dst, int where, void *stream) {
    if (!adj || !dst) return fail(TFD_ERR_INVALID, "null argument");
    return adj->p->desc.precision == 8 ? adjoint_sensitivity_t<double>(adj, dst, where, as_stream(stream))
                                       : adjoint_sensitivity_t<float>(adj, dst, where, as_stream(stream));
}

void tfd_adjoint_destroy(tfd_adjoint *adj) { delete adj; }

}  // extern "C"
