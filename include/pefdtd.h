/*
 * pefdtd — C ABI of the B200 label-indexed anisotropic elastic FDTD solver.
 *
 * This is the boundary a non-Python caller binds (ctypes / cffi / cgo / JNI).
 * It replaces the reference's solver entry point
 *   fdtd.forward_fused_labels(lab, axes, h, dt, nt, src_pts, wavelet,
 *                             rec_groups, order, coeffs, sponge_width,
 *                             sponge_strength, damp_mask, c_couplant,
 *                             rho_couplant, record, slab, stress_smem,
 *                             progress, mat_tables)
 *   (Jerome-Graves/pulse-echo-azimuthal-simulation sim/core/fdtd.py:1618-1816)
 * and its dense siblings fdtd.forward_fused (:831-921) and fdtd.forward
 * (:236-376), which the reference drives through CuPy RawKernel launches
 * (:586-591, :1786-1815). Everything crossing this boundary is a plain
 * pointer, size or enum; no PyTorch or CuPy type appears.
 *
 * Conventions
 *  - Grids are (nz, ny, nx), C order, x fastest; flat cell index
 *    i = (iz * ny + iy) * nx + ix (the reference's np.ravel_multi_index).
 *  - "dev" pointers are CUDA device memory on the current device; all other
 *    pointers are host memory, read during the call only.
 *  - Material index m is the reference's (label + 1): m = 0 is the fluid
 *    couplant, m = g + 1 is grain g. At most PE_MAX_MATERIALS materials.
 *  - Every function returns PE_OK or an error code; pe_last_error() gives the
 *    message of the last failure on the calling thread. PE_ERR_INVALID is the
 *    condition the reference reports as ValueError.
 */
#ifndef PEFDTD_H
#define PEFDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PE_ABI_VERSION 1
#define PE_MAX_MATERIALS 16383

enum PeStatus {
    PE_OK = 0,
    PE_ERR_INVALID = 1,     /* bad argument (reference: ValueError) */
    PE_ERR_CUDA = 2,        /* CUDA runtime error */
    PE_ERR_NOMEM = 3,       /* device or host allocation failed */
    PE_ERR_UNSUPPORTED = 4, /* valid request this build cannot serve */
    PE_ERR_TIMEOUT = 5      /* a bounded device-side wait gave up */
};

enum PeDtype { PE_F32 = 0, PE_F64 = 1 };

/* What a receiver records (reference `record=`, sim/core/fdtd.py:1806-1812). */
enum PeRecord { PE_REC_PRESSURE = 0, PE_REC_VX = 1, PE_REC_VY = 2, PE_REC_VZ = 3 };

/* Solve description. Scalars only. */
typedef struct PeConfig {
    int32_t nz, ny, nx;
    int32_t dtype;          /* PeDtype: arithmetic of fields, tables, traces */
    int32_t n_coeffs;       /* 1..4 staggered coefficients (order = 2 * n) */
    double coeffs[4];       /* reference `coeffs` (optimised_coeffs(order)) */
    double h, dt;           /* grid step [m], time step [s] */
    int32_t record;         /* PeRecord */
    int32_t damped_record;  /* 0: pressure from the stored (pre-deferred-
                               damping) stress, as forward_fused_labels;
                               1: from the end-of-step damped stress, as
                               forward_fused / forward (:909-915, :361-367) */
    int32_t n_mat;          /* rows in the material tables, 1..PE_MAX_MATERIALS */
    int32_t chunk_steps;    /* steps per captured CUDA graph (0 = 200) */
    int32_t tile_x, tile_y; /* simple-kernel tile (0 = default) */
    int32_t z_chunk;        /* planes per z-march (0 = tuned default) */
    int32_t variant;        /* PeKernelVariant (0 = tiled, the default) */
} PeConfig;

/* Kernel family; all are bit-identical. TILED picks the fastest tiled kernels
 * the grid allows: in FP32 on grids whose rows are 16-byte multiples the
 * pair-column kernels (each thread updates two x-adjacent cells), else the
 * one-column tiled kernels. COLUMN forces the one-column tiled kernels and
 * SIMPLE the untiled ones (every tap read through the L1 cache); both are
 * kept as independent cross-checks of TILED. */
enum PeKernelVariant { PE_KERNEL_TILED = 0, PE_KERNEL_SIMPLE = 1, PE_KERNEL_COLUMN = 2, PE_KERNEL_DENSE = 3 };
/* PE_KERNEL_DENSE: per-cell media, the reference's dense path (forward_fused
 * with 21 arbitrary stiffness maps, sim/core/fdtd.py:831-921, kernels K1-K3
 * :392-583): the medium tables hold one row per cell (n_mat == nz * ny * nx,
 * row i for the cell of linear index i; PE_MAX_MATERIALS does not apply),
 * labels_dev is not read (may be NULL). Runs the untiled kernels with the
 * row looked up by cell index; same arithmetic, so a medium that also fits a
 * table gives bit-identical results either way. Not available to batches or
 * the adjoint. */

/* The medium. Volumes live on the device; tables are small host arrays. */
typedef struct PeMedium {
    const uint16_t *labels_dev;    /* (nz, ny, nx) material index (< n_mat) */
    const float *damp_volume_dev;  /* (nz, ny, nx) f32 per-step multiplier
                                      (reference damp_mask) or NULL */
    const void *ctab;              /* (n_mat, 36) dtype: full symmetric Voigt
                                      rows, row-major I*6+J (reference Ct) */
    const void *rho;               /* (n_mat,) dtype density (reference rho_t) */
    const float *sponge_z;         /* (nz,) f32 sponge taper or NULL */
    const float *sponge_y;         /* (ny,) */
    const float *sponge_x;         /* (nx,); all three or none. The damping
                                      applied to a cell is
                                      ((sz*sy)*sx)*volume in f32, the
                                      reference's sponge_profile(..)*damp_mask */
} PeMedium;

/* Source and receivers (host arrays, copied at create). */
typedef struct PeProbe {
    int32_t n_src;
    const int64_t *src_idx;  /* flat cell index; s1,s2,s3 += wavelet[n]*w after
                                the stress update (reference :1798-1800). A
                                repeated cell keeps its last entry. */
    const void *src_w;       /* (n_src,) dtype */
    int32_t n_groups;        /* receiver groups = trace columns */
    const int64_t *rec_off;  /* (n_groups + 1) CSR offsets into rec_idx/rec_w */
    const int64_t *rec_idx;  /* flat cell index per entry */
    const void *rec_w;       /* dtype weight per entry; a trace sample is the
                                weighted sum over its group, in list order */
} PeProbe;

/* The nine state fields, device memory of dtype, (nz, ny, nx) each. */
typedef struct PeState {
    void *v[3];  /* vx, vy, vz */
    void *s[6];  /* s1..s6 (Voigt order xx, yy, zz, yz, xz, xy) */
} PeState;

typedef struct PeSolver PeSolver;

/* ABI version of the loaded library (PE_ABI_VERSION). */
int pe_abi_version(void);

/* Message of the last failure on the calling thread ("" if none). */
const char *pe_last_error(void);

/* Validate and prepare a solve: copies the labels (marking source and
 * receiver cells), tables, profiles and probe into solver-owned device
 * memory. labels out of range -> PE_ERR_INVALID (reference :1650-1658,
 * :1674-1677); n_coeffs outside 1..4 -> PE_ERR_INVALID (:1638-1643). */
int pe_solver_create(const PeConfig *cfg, const PeMedium *medium, const PeProbe *probe,
                     PeSolver **out);

/* Upload the source wavelet (host, dtype, nt samples). */
int pe_solver_set_wavelet(PeSolver *s, const void *wavelet, int64_t nt);

/* Advance `state` over steps [step_begin, step_end) on `stream`
 * (cudaStream_t, NULL = legacy default stream) and write trace rows
 * traces_dev[n * n_groups + g] for those steps (traces_dev: device, dtype,
 * at least step_end * n_groups elements). Asynchronous with respect to the
 * host. Full chunks run as one captured CUDA graph each. */
int pe_solver_run(PeSolver *s, const PeState *state, void *traces_dev, int64_t step_begin,
                  int64_t step_end, void *stream);

/* Wait for the solver's queued work and report its device status: PE_OK, or
 * PE_ERR_TIMEOUT if a bounded device-side wait (TMA arrival) gave up, in
 * which case the traces of the affected run are invalid. Clears the status. */
int pe_solver_status(PeSolver *s);

/* Kernel launches issued by the last pe_solver_run (diagnostics). */
int64_t pe_solver_launch_count(const PeSolver *s);

/* Diagnostics for roofline reporting: advance `state` by n_steps from step 0
 * one kernel at a time, with CUDA events around each launch, and write the
 * mean per-step milliseconds of the stress and velocity kernels to
 * ms_out[0], ms_out[1]. Synchronous. No reference counterpart (the
 * reference times whole solves with time.time()). */
int pe_solver_profile(PeSolver *s, const PeState *state, int n_steps, float *ms_out,
                      void *stream);

int pe_solver_destroy(PeSolver *s);

/* One call, host buffers in and out: the reference's forward_fused_labels
 * contract (sim/core/fdtd.py:1618-1816) for callers without device memory
 * management. Uploads the labels, zeroes the state on the device, runs nt
 * steps and copies the (nt, n_groups) traces (dtype) back into traces_host.
 * labels_host is (nz, ny, nx) uint16, damp_volume_host f32 or NULL;
 * medium->labels_dev/damp_volume_dev are ignored. The device buffers (state,
 * labels, damping, traces) are kept per device between calls, grown when a
 * call needs more, so that repeated calls allocate nothing; calls on one
 * device run one at a time. */
int pe_forward_host(const PeConfig *cfg, const uint16_t *labels_host,
                    const float *damp_volume_host, const PeMedium *medium,
                    const PeProbe *probe, const void *wavelet_host, int64_t nt,
                    void *traces_host);
/* Give back to the driver the device memory the library keeps for reuse:
 * pe_forward_host's buffers and the cache of freed solver and batch buffers
 * (a destroyed solve's buffers are kept, up to 8 GiB per device, and reused
 * by a later solve of the same sizes, so that repeated solves allocate and
 * free nothing). Call with no solve, batch or host-entry call in flight. No
 * reference counterpart. */
void pe_release_cached_memory(void);

/* ---- Adjoint ---------------------------------------------------------------
 * One reverse step of the exact discrete adjoint of pe_solver_run's step n
 * (the reference's only FDTD adjoint is the order-2, undamped, cell-density
 * vendor/ringfwi/elastic3d.py:348-463; this is the adjoint of the full
 * scheme: order 2..8, face density, sponge and damping volume, deferred
 * damping, every record kind). On entry lv, ls hold dJ/d(v^n, s^n) from the
 * later steps; the call adds the trace adjoint residual[n][g] at the
 * receivers, then transposes the velocity and stress updates, leaving
 * dJ/d(v^{n-1}, s^{n-1}) and adding dJ/dC of this step to grad. v_prev must
 * hold the forward velocity at the start of step n (the caller recomputes
 * it from checkpoints). All pointers are device memory of the solver's dtype
 * except grad (f64). Asynchronous on `stream`. */
typedef struct PeAdjoint {
    void *lv[3];             /* adjoint of vx, vy, vz */
    void *ls[6];             /* adjoint of s1..s6 */
    const void *v_prev[3];   /* forward v^{n-1} */
    void *scratch;           /* 33 fields of (nz, ny, nx) */
    double *grad;            /* (n_mat, 21) dJ/dC upper triangle, accumulated */
} PeAdjoint;

int pe_solver_adjoint_step(PeSolver *s, const PeAdjoint *adj, int64_t n, const void *residual,
                           void *stream);

/* One checkpoint segment of the reverse sweep in a single call: `state`
 * holds the forward state before step `step_begin` (restored from its
 * checkpoint by the caller); the call recomputes steps [step_begin,
 * step_end) forward on `state`, keeping v before each step in `v_hist`
 * (device, (step_end - step_begin, 3, nz, ny, nx) of dtype), then applies
 * pe_solver_adjoint_step for n = step_end - 1 down to step_begin (v_prev
 * from v_hist). Asynchronous on `stream`; the trace buffer is not written.
 * Same result as the per-step calls, without a host round trip per step
 * (reference counterpart: the reverse loop of vendor/ringfwi/elastic3d.py
 * :386-463, which stores the whole history instead of recomputing). */
int pe_solver_adjoint_segment(PeSolver *s, const PeState *state, const PeAdjoint *adj, void *v_hist,
                              int64_t step_begin, int64_t step_end, const void *residual, void *stream);

/* ---- Batches: many independent solves advanced together ----------------
 * No counterpart in the reference, which runs one azimuth at a time in a
 * Python loop (sim/pipeline/sweep_runner.py:322-390); the closest precedent
 * is ringfwi's elastic3d.forward_batch (vendor/ringfwi/elastic3d.py:474-632),
 * which stacks transmits on a leading array axis. Every solve keeps the
 * single-solve contract above (own grid size, medium, probe, wavelet, state
 * and traces); all share one dtype and the tiled kernels. Each step is one
 * stress and one velocity launch covering every solve with nx a multiple of
 * 4 (state buffers 16-byte aligned), plus one launch pair per solve whose
 * rows are not whole 16-byte units (the cp.async kernels); when the batched
 * kernels' shared memory cannot hold the largest table (FP64), every solve
 * runs its own pair. Chunks of steps replay as CUDA graphs. */
typedef struct PeBatch PeBatch;

int pe_batch_create(int n, const PeConfig *cfgs, const PeMedium *media, const PeProbe *probes,
                    PeBatch **out);
/* Work layout: planes per z-march (0 = 40) and steps per captured graph
 * (0 = keep). Chosen by pefdtd.autotune. */
int pe_batch_schedule(PeBatch *b, int z_chunk, int chunk_steps);
/* Persistent batch mode (on = 1): one cooperative launch per graph chunk
 * advances every batched solve by the chunk's steps, its blocks alternating
 * a stress and a velocity phase separated by bounded grid-wide barriers
 * (a timed-out barrier sets PE_ERR_TIMEOUT in pe_batch_status; nothing
 * hangs). Bit-identical to the per-step launches (on = 0, the default).
 * FP32 batches of pair-column solves only, else PE_ERR_UNSUPPORTED. The
 * reference has no counterpart: it runs one solve at a time, one CuPy launch
 * per kernel and step (sim/pipeline/sweep_runner.py:322-390,
 * sim/core/fdtd.py:1784-1813). */
int pe_batch_set_persistent(PeBatch *B, int on);
int pe_batch_set_wavelet(PeBatch *b, int i, const void *wavelet, int64_t nt);
/* Advance every solve i over [step_begin, step_end): states[i], traces[i] as
 * in pe_solver_run. Asynchronous on `stream`. */
int pe_batch_run(PeBatch *b, const PeState *states, void *const *traces, int64_t step_begin,
                 int64_t step_end, void *stream);
int pe_batch_status(PeBatch *b);
int64_t pe_batch_launch_count(const PeBatch *b);
int pe_batch_destroy(PeBatch *b);

/* Power-diagram labels of a cylinder (specimen builder, reference
 * sim/core/specimen.py:298-337): out_dev[(iz*ny + iy)*nx + ix] = the seed
 * minimising ((x-sx)^2 + (y-sy)^2) - w + (z-sz)^2 in float64 at point
 * (xs[ix], ys[iy], zs[iz]), first index on ties, or -1 where
 * x^2 + y^2 > R2. seeds (ns, 3) and weights (ns, NULL = 0) are host arrays;
 * out_dev is device int32. Synchronous on `stream`. */
int pe_label_cylinder(const double *xs, int nx, const double *ys, int ny, const double *zs,
                      int nz, double R2, const double *seeds, const double *weights, int ns,
                      int32_t *out_dev, void *stream);

/* Solver grid of a specimen rotated by -rot about z (azimuth sweep; replaces
 * the reference's rotated_grid, sim/core/rotation_test.py:60-137, with its
 * nearest resample by np.rint). labels_dev: device int32 (nx_s, nx_s, nz_s)
 * specimen labels (x, y, z order, -1 outside) at spacing h_spec. out_dev:
 * device int32 (ndz + 2m, nd + 2m, nd + 2m) solver labels (z, y, x), -1 in
 * the padding and where the rotated sample leaves the specimen; nd and ndz
 * the core extents (round(nx_s*h_spec/h), round(nz_s*h_spec/h)), m the
 * padding (sponge + 3), cos_a / sin_a of the rotation angle. Bit-identical
 * to the host computation. Synchronous on `stream`. */
int pe_rotated_grid(const int32_t *labels_dev, int nx_s, int nz_s, double h_spec, double h, int nd,
                    int ndz, double cos_a, double sin_a, int m, int32_t *out_dev, void *stream);

/* Batched trace post-processing, float64 on the device. A batch is `batch`
 * traces packed back to back in one device array: trace i is samples
 * off[i] .. off[i+1]-1 (off: host int64 (batch + 1), off[0] = 0, every trace
 * non-empty). x_dev is PE_F32 or PE_F64 (`dtype`); results are device f64.
 * Window bounds, time steps and filter coefficients come from the host,
 * computed as the reference's Python computes them. All synchronous on
 * `stream`.
 *
 * pe_trace_envelope: env = |x + i H(x)| with H the discrete Hilbert
 * transform of the whole trace (scipy.signal.hilbert, as used by
 * sim/core/fdtd.py:976 and sim/pipeline/sweep_runner.py:210). */
int pe_trace_envelope(const void *x_dev, int32_t dtype, const int64_t *off, int32_t batch, double *env_dev,
                      void *stream);

/* pe_trace_detrend: n_ab == 0: x - mean(x) per trace (sim/core/fdtd.py:974);
 * else filtfilt(b, a, x) with odd padding of `padlen` samples at each end and
 * initial state zi * (first sample) (scipy.signal.filtfilt defaults; the
 * reference's detrend_hp, sim/core/fdtd.py:943-948). b, a: host (n_ab,)
 * normalised so a[0] = 1, 2 <= n_ab <= 8; zi: host (n_ab - 1,)
 * (scipy.signal.lfilter_zi); padlen <= 24 and every trace longer than padlen. */
int pe_trace_detrend(const void *x_dev, int32_t dtype, const int64_t *off, int32_t batch, const double *b,
                     const double *a, int32_t n_ab, const double *zi, int32_t padlen, double *out_dev,
                     void *stream);

/* pe_trace_pick: envelope peak in [lo, hi) per trace (win: host int64
 * (batch, 2), hi > lo + 2), first index on ties, parabolic refinement;
 * out_dev (batch, 3): pick time (refined index * dt[i]), peak value, and 1.0
 * when the peak is not on a window edge (sim/core/fdtd.py:977-984). */
int pe_trace_pick(const double *env_dev, const int64_t *off, int32_t batch, const int64_t *win, const double *dt,
                  double *out_dev, void *stream);

/* pe_trace_analyse: the sweep driver's per-trace figures
 * (sim/pipeline/sweep_runner.py:209-225). win: host int64 (batch, 4) = E1
 * window [a, b) (b > a) and coda window [lo, hi); dt_fs: host (batch, 2) =
 * dt and 1/dt. out_dev (batch, 4): E1 (envelope max in [a, b)), t1 (its
 * index * dt), coda = 20 log10(sqrt(mean(env[lo:hi]^2)) / E1 + 1e-30) and
 * tail = max |x[k:]| / max(E1, 1e-30) with k = int((t1 + 3e-6) * fs), NaN
 * unless k < n - 8. */
int pe_trace_analyse(const void *x_dev, int32_t dtype, const double *env_dev, const int64_t *off, int32_t batch,
                     const int64_t *win, const double *dt_fs, double *out_dev, void *stream);

/* Allocation-free variant of pe_label_cylinder, with no counterpart in the
 * reference. For callers that may not allocate device memory (an application
 * whose framework has reserved the device pool for its own allocator, or a
 * pipeline stage that must not pay cudaMalloc/cudaFree's implicit device
 * synchronisation): the staged coordinates, seeds and weights go to a
 * fixed-size file-scope device array instead of a cudaMalloc buffer, which
 * every device that loads the library holds until exit
 * (PE_NOALLOC_SCRATCH_BYTES). Same arguments and result as
 * pe_label_cylinder; out_dev is still the caller's. Limits: nx + ny + nz <=
 * PE_NOALLOC_MAX_COORDS and ns <= PE_NOALLOC_MAX_SEEDS, else PE_ERR_INVALID
 * (message: pe_label_cylinder_noalloc_error). The first call on a device
 * looks the array up (make it before any stream capture on that device). All
 * calls on a device share the array: calls that can overlap on the GPU race
 * and must be serialised by the caller. Synchronous on `stream`. */
#define PE_NOALLOC_MAX_COORDS 12288
#define PE_NOALLOC_MAX_SEEDS 16384
#define PE_NOALLOC_SCRATCH_BYTES (8 * (PE_NOALLOC_MAX_COORDS + 4 * PE_NOALLOC_MAX_SEEDS))
int pe_label_cylinder_noalloc(const double *xs, int nx, const double *ys, int ny, const double *zs,
                              int nz, double R2, const double *seeds, const double *weights, int ns,
                              int32_t *out_dev, void *stream);
const char *pe_label_cylinder_noalloc_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PEFDTD_H */
