/*
 * tfdtd.h - C ABI of the B200-native fused Yee/CPML engine (libtfdtd.so).
 *
 * This is the drop-in boundary for TorchFDTD's fused CUDA path. In the
 * reference the path is reached from Python through
 *   Simulation(project).run()                      torchfdtd/solver.py:662-908
 *   configure_cuda_kernel(grid, 'fused')           torchfdtd/cuda_kernels.py:368-373
 *   FusedYeeCUDA.update_E / update_H               torchfdtd/cuda_kernels.py:349-365
 *   FusedFrequencyPlanes.update(counter)           torchfdtd/cuda_monitors.py:135-155
 *   CudaStepGraphs(step, states, steps, width)     torchfdtd/cuda_graph.py:187-218
 * Here the same work sits behind plain C entry points (pointers, sizes, int
 * status codes, no exceptions, no torch types) that any host language can bind;
 * the Python package binds them with ctypes.
 *
 * Memory: the caller allocates ONE device arena of tfd_plan_bytes() bytes
 * (PyTorch does, mirroring the reference, where torch owns every array,
 * torchfdtd/cuda_kernels.py:120-128) and the library lays out fields, CPML
 * memories, material, tables and monitor accumulators inside it. The main
 * entry points never call cudaMalloc.
 *
 * Streams: every call takes a cudaStream_t (as void*); work is enqueued on it.
 * tfd_step is capturable in a CUDA graph (no allocation, no synchronisation,
 * the time step is read from a device counter). Calls with TFD_HOST buffers
 * synchronise the stream before returning.
 *
 * Every function returns TFD_OK (0) or an error code; tfd_last_error() gives a
 * message for the calling thread's last failure.
 */
#ifndef TFDTD_H
#define TFDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TFD_ABI_VERSION 2

enum tfd_code {
    TFD_OK = 0,
    TFD_ERR_INVALID = 1,       /* bad argument or descriptor; reference: ValueError */
    TFD_ERR_UNSUPPORTED = 2,   /* feature outside the fused path; reference: ValueError naming it */
    TFD_ERR_CUDA = 3,          /* CUDA runtime error; reference: RuntimeError */
    TFD_ERR_ARENA = 4,         /* arena too small or misaligned */
    TFD_ERR_DEVICE = 5         /* a kernel reported a failure in the device status word */
};

enum tfd_face { TFD_FACE_PML = 0, TFD_FACE_PERIODIC = 1, TFD_FACE_PEC = 2 };
enum tfd_where { TFD_DEVICE = 0, TFD_HOST = 1 };
enum tfd_kernel { TFD_KERNEL_AUTO = 0, TFD_KERNEL_MARCH = 1, TFD_KERNEL_GATHER = 2, TFD_KERNEL_TILE2D = 3 };

/* One CPML slab of one field family on one axis (both curl terms of that axis share it).
 * forward = 0: E family (backward differences), 1: H family (forward differences).
 * Targets are cells [lo, hi) along axis; b, c, inv_kappa hold hi-lo float64 values.
 * Reference: YeeGrid._prepare_boundaries, torchfdtd/boundaries.py:307-355. */
typedef struct tfd_cpml_segment {
    int32_t forward, axis, lo, hi;
    const double *b, *c, *inv_kappa;
} tfd_cpml_segment;

/* A soft source term: values[n] is ADDED to component `component` of family
 * `family` (0 E, 1 H) on cells [lo, hi) right after that family's update of
 * step n. Reference: torchfdtd/injection.py:117-141, torchfdtd/solver.py:778-789. */
typedef struct tfd_source_term {
    int32_t family, component;
    int32_t lo[3], hi[3];
    const double *values;     /* steps samples, rounded to the field precision */
} tfd_source_term;

/* A point trace, recorded after the H update of each step.
 * Reference: torchfdtd/solver.py:765,790-796. */
typedef struct tfd_trace {
    int32_t family, component;
    int32_t index[3];
} tfd_trace;

/* An online DFT plane: per step n, sample = sum_k field[corner k] * weight k (field
 * precision, in corner order) * window[n]; then for every frequency f
 * acc[f][p][c] += exp(i*omega_f*(n+1)) * sample, times exp(i*pi*f*dt) for H samples.
 * Accumulators are complex float64. E components come first.
 * Reference: torchfdtd/field_monitors.py:121-164, torchfdtd/cuda_monitors.py:65-155. */
typedef struct tfd_plane {
    int32_t points, frequencies, components, corners;
    const int32_t *component_ids;  /* components entries, 0..5 = Ex Ey Ez Hx Hy Hz */
    const int64_t *corner_cells;   /* [components][corners][points] flat (x*ny+y)*nz+z */
    const double *corner_weights;  /* same shape */
    const double *frequency_hz;    /* frequencies */
    const double *window_e;        /* steps: apodization * dt * downsample mask, E samples */
    const double *window_h;        /* steps, H samples (half a step later) */
} tfd_plane;

/* A total-field / scattered-field box: a live scalar incident line stepped with the grid and the sparse
 * corrections on the box faces. Per step, after the grid's E update and soft sources: the line's E half-step
 *   diff[i] = h[i] - h[i-1] (0 at i = 0); pe[i] = b_e[i] pe[i] + c_e[i] diff[i]; e[i] -= courant_e (diff[i] + pe[i]);
 *   e[drive_at] += drive[n]
 * then E[target] += weight * h[sample] for every E correction; after the H update and H sources the line's H
 * half-step (forward differences of e, 0 at the last cell, b_h / c_h, courant_h) and H[target] += weight *
 * e[sample]. Line arithmetic runs in the field precision. Targets are flat reference-layout elements
 * ((x*ny + y)*nz + z)*3 + component, one correction per target and family.
 * Reference: torchfdtd/tfsf.py:19-176 (tfsf_plan, surface_maps, IncidentLine, TfsfState.inject),
 * torchfdtd/cuda_tfsf.py:19-49 (the fused line + correction kernel). */
typedef struct tfd_tfsf {
    int32_t count;                 /* incident-line cells */
    int32_t drive_at;              /* line cell of the soft drive */
    double courant_e, courant_h;   /* line update factors: courant / index^2 (E), courant (H) */
    double index;                  /* background index (the diagnostics weigh line E by it) */
    double norm_weight;            /* diagnostics weight of every line cell */
    const double *b[2], *c[2];     /* line CPML decay / coupling per family (0 E, 1 H), count values each */
    const double *drive;           /* steps waveform samples */
    int32_t n_targets[2];          /* corrections per family */
    const int64_t *target[2];
    const int64_t *sample[2];      /* line cell each correction reads */
    const double *weight[2];
} tfd_tfsf;

/* The samples one dispersive material owns and its poles (coupled trapezoidal ADE). Per step, after the free
 * E update of a sample (with 1 / eps_inf) and before the soft sources:
 *   r_p = (Q_p - a_p P_p) / d_p;  E = (eps_inf E_free - k_sum E_old - sum_p r_p) / (eps_inf + k_sum);
 *   delta_p = r_p + k_p (E + E_old);  P_p += delta_p;  Q_p = -Q_p + 2 delta_p.
 * multiple = 0 (one pole): a, d, k rounded to the field precision at each use and eps_inf + k rounded once;
 * multiple = 1: a, d, k rounded to the field precision, k_sum and eps_inf + k_sum summed in it (pole order).
 * Reference: MaterialADE, torchfdtd/materials.py:29-88, configure_materials :117-193. */
typedef struct tfd_ade {
    int32_t samples, poles, multiple;
    const int64_t *target;         /* samples: flat reference-layout element ((x*ny + y)*nz + z)*3 + component */
    double eps_inf;
    const double *a, *d, *k;       /* poles values */
    const double *w0, *strength;   /* poles: the state norm adds (Q / (dt sqrt(strength)))^2 + (P w0 / sqrt(strength))^2 */
    const double *weight;          /* samples: diagnostics volume weights, or NULL for 1 */
} tfd_ade;

typedef struct tfd_desc {
    int32_t abi_version;           /* TFD_ABI_VERSION */
    int32_t nx, ny, nz;            /* Yee cells; nz = 1 for 2D */
    int32_t precision;             /* 4: float32 fields, 8: float64 fields */
    int32_t material_samples;      /* 1 (one inverse permittivity per cell) or 3 (per E component) */
    int32_t components;            /* bit c (0..5) set = component advanced; 0x3F in 3D */
    int32_t steps;                 /* length of every per-step table (sources, windows, traces) */
    int32_t kernel;                /* enum tfd_kernel */
    int32_t launch_variant;        /* 0: default launch shape; otherwise a kernel-specific variant (autotuner) */
    int32_t face[3][2];            /* enum tfd_face per axis and side */
    double courant;                /* rectangular Courant number c*dt/dx */
    double time_step;              /* seconds */
    double pec_upper[3];           /* H ghost factor on PEC upper faces (reference_step / last width) */
    int32_t n_segments;
    const tfd_cpml_segment *segments;
    int32_t n_sources;
    const tfd_source_term *sources;
    int32_t n_traces;
    const tfd_trace *traces;
    int32_t n_planes;
    const tfd_plane *planes;
    /* Nonuniform meshes: per family (0 E, 1 H) and axis, n float64 factors indexed by the updated cell, or NULL on
     * an axis whose cells all have the reference step. The plain difference of the cell's curl term along that axis
     * is multiplied by the factor (rounded to the field precision) before the CPML terms: E at cell i >= 1 by
     * h / ((w[i-1] + w[i]) / 2), at i = 0 by the periodic wrap factor 2 h / (w[0] + w[n-1]); H at cell i <= n-2 by
     * h / w[i], at i = n-1 by the wrap factor h / w[n-1] (h: reference step, w: cell widths). PEC ghost terms are
     * not scaled. Reference: the metric of YeeGrid._prepare_boundaries / curl, torchfdtd/boundaries.py:276-284,
     * 376-393, and its fused kernel, torchfdtd/cuda_kernels.py:203-236. */
    const double *metric[2][3];
    /* Diagnostics cell volumes: per axis the cell widths over the reference step (n values), or NULL for 1. The
     * state norm weighs E^2 / inv_eps and H^2 by (w_x * w_y) * w_z rounded to the field precision (reference
     * StateDiagnostics, torchfdtd/run_control.py:88-146). */
    const double *volume[3];
    int32_t n_tfsf;                /* TFSF boxes, in source order (at most 4) */
    const tfd_tfsf *tfsf;
    int32_t n_ade;                 /* dispersive material states (at most 8), samples disjoint */
    const tfd_ade *ade;
} tfd_desc;

typedef struct tfd_plan tfd_plan;

/* Arena size for a descriptor. Replaces the reference's per-array torch allocations
 * (torchfdtd/boundaries.py:231-256, torchfdtd/solver.py:769-771, field_monitors.py:136). */
int tfd_plan_bytes(const tfd_desc *desc, size_t *bytes);

/* Lay out the arena, upload the tables and zero the state (fields, CPML memories,
 * monitors, step counter). Replaces YeeGrid(...) + configure_cuda_kernel(grid, 'fused')
 * + FrequencyUpdates(...) (torchfdtd/solver.py:741-776). The arena must be 256-byte
 * aligned and stay allocated until tfd_plan_destroy. */
int tfd_plan_create(const tfd_desc *desc, void *arena, size_t arena_bytes, void *stream, tfd_plan **plan);
void tfd_plan_destroy(tfd_plan *plan);

/* Inverse permittivity in the reference layout (nx, ny, nz[, 3]) C order, z fastest,
 * field precision. Replaces g.inverse_permittivity[:] = 1/eps (torchfdtd/solver.py:742-745). */
int tfd_set_material(tfd_plan *plan, const void *inv_eps, int where, void *stream);

/* The relative permittivity itself, same layout: every value is checked (finite, at least 1) and inverted on
 * the device (IEEE division, the host's 1/eps values) into the plan's material, saving the caller a host pass
 * over the array. Returns TFD_ERR_INVALID when a value fails the check; synchronizes the stream. No
 * counterpart in the reference (its solver inverts on the host). */
int tfd_set_permittivity(tfd_plan *plan, const void *eps, int where, void *stream);

/* The largest |E| over the current fields and whether every E and H value is finite (1) or not (0);
 * synchronizes the stream. No counterpart in the reference (its Result checks the host copies). */
int tfd_field_check(tfd_plan *plan, double *peak_e, int32_t *finite, void *stream);

/* E and H in the reference layout (nx, ny, nz, 3), field precision (g.E, g.H). */
int tfd_set_fields(tfd_plan *plan, const void *E, const void *H, int where, void *stream);
int tfd_get_fields(tfd_plan *plan, void *E, void *H, int where, void *stream);

/* Every CPML memory concatenated in the reference's YeeGrid.memory_states order and
 * shapes (torchfdtd/boundaries.py:307-355); tfd_psi_count gives the element count. */
int tfd_psi_count(const tfd_plan *plan, size_t *count);
int tfd_set_psi(tfd_plan *plan, const void *psi, int where, void *stream);
int tfd_get_psi(tfd_plan *plan, void *psi, int where, void *stream);

/* Advance nsteps time steps: fused E update + E sources + H update + H sources, then
 * the point traces, the DFT planes and the step counter. Replaces one replay of the
 * reference's captured step (torchfdtd/solver.py:785-797, cuda_graph.py:62-63).
 * Capturable in a CUDA graph. */
int tfd_step(tfd_plan *plan, int32_t nsteps, void *stream);

/* Zero fields, CPML memories, traces, DFT accumulators and the step counter. */
int tfd_reset(tfd_plan *plan, void *stream);

/* Point traces, (steps, n_traces) field precision (torchfdtd/solver.py:771,908). */
int tfd_get_traces(tfd_plan *plan, void *dst, int where, void *stream);

/* DFT plane k accumulators as complex float64 (frequencies, points, components). */
int tfd_get_plane(tfd_plan *plan, int32_t k, void *dst, int where, void *stream);

/* One plane of one component (0..5) at `index` on `axis`, reference order of the two
 * remaining axes, field precision: the snapshot frame (torchfdtd/solver.py:821-863). */
int tfd_get_slice(tfd_plan *plan, int32_t component, int32_t axis, int32_t index, void *dst, int where, void *stream);

/* Divergence diagnostics of torchfdtd/run_control.py:127-159: out[0] = sum over cells and
 * components of E^2/inv_eps + H^2 (float64), out[1] = max |E|, |H|, out[2] = 1 when every
 * CPML memory is finite. Synchronises the stream. */
int tfd_diagnose(tfd_plan *plan, double out[3], void *stream);

/* The device step counter (synchronises the stream). */
int tfd_counter(tfd_plan *plan, int64_t *value, void *stream);

/* The device status word: 0, or the code a kernel recorded (synchronises the stream): 1 step counter out of
 * range, 2 a bounded pipeline wait timed out, 3 a strip table entry failed the 2D kernel's own checks. */
int tfd_device_status(tfd_plan *plan, int32_t *status, void *stream);

/* Field energy and peak without any device allocation and without a plan. No counterpart in the
 * reference. For callers that cannot allocate device memory: a health check that runs after an
 * out-of-memory failure (when an allocation would fail again), or a host whose device memory belongs to
 * a pool or budget it must not bypass. E, H: (cells, 3) and inv_eps: (cells, material_samples) device
 * arrays in the field precision (4 or 8); out: 2 device doubles, set to the sum of E^2/inv_eps + H^2 and
 * to max |E|, |H| (NaN if a field value is NaN) -- the first two values tfd_diagnose reports. Scratch is a
 * static 32 KiB device array inside the library, so at most 67,108,864 cells are accepted (larger inputs
 * return TFD_ERR_INVALID; use tfd_diagnose). The first call on a device looks the array up and should
 * come before any stream capture; calls that overlap on the GPU share the array and race. */
int tfd_field_norm_static(const void *E, const void *H, const void *inv_eps, int64_t cells, int32_t material_samples,
                          int32_t precision, double *out, void *stream);

/* Which step kernel the plan runs (enum tfd_kernel) after TFD_KERNEL_AUTO is resolved. */
int tfd_kernel_in_use(const tfd_plan *plan, int32_t *kernel);

/* How many kernel launches tfd_step(plan, nsteps) issues (small 2D TMz plans run all their steps in one
 * persistent launch; the other paths launch per step). No counterpart in the reference. */
int tfd_step_launches(const tfd_plan *plan, int32_t nsteps, int64_t *launches);

/* ---- batches: many independent 2D TMz grids of uneven size advanced by one launch per step ----
 * Replaces run_tensor_batch / run_grouped_batch cohorts (torchfdtd/tensor_batch.py:45-337,
 * torchfdtd/grouped_batch.py:38-146, torchfdtd/cuda_batch.py:19-169), which need identical shapes per
 * cohort and launch one kernel per cohort. Members are ordinary plans (2D TMz, same precision, non-periodic,
 * step counter 0); while batched they share the batch's step counter and must be advanced only through
 * tfd_batch_step (tfd_step and tfd_reset refuse them). Members may have different step counts: a member
 * whose run has ended is skipped by later batch steps. Its fields, traces, planes and diagnostics stay
 * readable through the plan entry points while the batch's step is at most the member's own step count,
 * and always after tfd_batch_destroy, which hands every member its step count (capped at its own). */
typedef struct tfd_batch tfd_batch;
int tfd_batch_bytes(int32_t n_plans, tfd_plan *const *plans, size_t *bytes);
int tfd_batch_create(int32_t n_plans, tfd_plan *const *plans, void *arena, size_t arena_bytes, void *stream, tfd_batch **batch);
/* Launch shape of the batched step kernel, the autotuner's knobs: ctas = persistent CTA count (0: one warp
 * per strip), strip_rows = rows per strip (0: default for the batch's cell count; else >= 8). Rebuilds the
 * strip table on the stream when strip_rows changes; call it outside graph capture. */
int tfd_batch_set_launch(tfd_batch *batch, int32_t ctas, int32_t strip_rows, void *stream);
/* persistent = 1: every tfd_batch_step call runs all its steps in ONE cooperative launch over the strip table
 * (with the observations of every member, a bounded grid barrier between steps; ctas as set above, capped at
 * the resident limit), bitwise equal to the per-step launches; 0: one strip launch and one observation launch
 * per step. Call it outside graph capture (it queries the occupancy). The north-star shape of the batched
 * path; the reference has no counterpart (its cohorts launch per step, torchfdtd/cuda_batch.py:139-169). */
int tfd_batch_set_persistent(tfd_batch *batch, int32_t persistent, void *stream);
int tfd_batch_step(tfd_batch *batch, int32_t nsteps, void *stream);
int tfd_batch_tiles(const tfd_batch *batch, int32_t *tiles);
void tfd_batch_destroy(tfd_batch *batch);

/* ---- restart states: the checkpoints of the discrete adjoint ----
 * Replace _Checkpoints.save / restore (torchfdtd/differentiable.py:539-624), which clone E, H and every
 * CPML memory as torch tensors. A snapshot is one device buffer (256-byte aligned, tfd_state_bytes long)
 * holding the step counter, E, H and E-family memories of the current parity and the H-family memories.
 * Save and load are stream-ordered kernels (the parity is read on the device), so they can be captured. */
int tfd_state_bytes(tfd_plan *plan, size_t *bytes);
int tfd_state_save(tfd_plan *plan, void *snapshot, void *stream);
int tfd_state_load(tfd_plan *plan, const void *snapshot, void *stream);

/* ---- discrete adjoint ----
 * Replaces _System.transpose_step / FusedAdjointCUDA (torchfdtd/differentiable.py:489-519,
 * torchfdtd/cuda_adjoint.py:16-234): the transpose of one Yee/CPML step, with the CPML memory transpose,
 * accumulating the material sensitivity S_c = sum over steps of e_bar_c * curl_b(H)_c (the gradient with
 * respect to the permittivity is -courant * S / eps^2). The observers are the plan's traces: they must be
 * distinct cells. tfd_adjoint_step transposes the step that took s_n to s_{n+1}: it first adds `seeds`
 * (one value per trace, the derivative of the objective with respect to the traces recorded after step n;
 * device pointer in the plan's precision, or null) and then reads the forward state s_n from `snapshot`
 * (a tfd_state_save buffer). Call it for n = steps-1 down to 0. */
typedef struct tfd_adjoint tfd_adjoint;
int tfd_adjoint_bytes(tfd_plan *plan, size_t *bytes);
int tfd_adjoint_create(tfd_plan *plan, void *arena, size_t arena_bytes, void *stream, tfd_adjoint **adjoint);
int tfd_adjoint_reset(tfd_adjoint *adjoint, void *stream);
int tfd_adjoint_step(tfd_adjoint *adjoint, const void *snapshot, const void *seeds, void *stream);
/* S in the reference layout (nx, ny, nz, 3), one value per E component (zero for components 2D does not
 * advance); TFD_HOST or TFD_DEVICE destination. */
int tfd_adjoint_sensitivity(tfd_adjoint *adjoint, void *dst, int where, void *stream);
void tfd_adjoint_destroy(tfd_adjoint *adjoint);

const char *tfd_error_string(int code);
const char *tfd_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* TFDTD_H */
