/*
 * feelmri_b200.h -- C ABI of the B200 (sm_100a) implementation of FEelMRI's
 * simulation hot path.
 *
 * Every entry point here replaces one native routine that python/feelmri
 * imports from the reference's four pybind11 modules (cpp/feelmri/*.h).  The
 * replaced interface is cited beside each declaration as file:line inside the
 * reference project.
 *
 * Conventions
 *  - All array arguments are DEVICE pointers on the context's device unless a
 *    comment says otherwise.  Complex numbers are interleaved (re, im).
 *  - Layouts are the reference's numpy layouts: (N,3) node arrays are
 *    row-major, Bloch histories are column-major (N, n_time) like the Eigen
 *    matrices solve_mri returns, Signal's output is row-major
 *    (n_ro, n_lines, n_kz, V) like the RowMajor Eigen tensor it returns.
 *  - Every entry point returns an int status (FM_OK == 0).  The message of the
 *    last failure on the calling host thread is read with fm_last_error().
 *    No C++ exception crosses this boundary.
 *  - The library never frees caller memory.  Scratch memory is passed in by
 *    the caller (workspace pointer + size); each *_workspace_size() query
 *    returns the bytes that call needs.
 *  - Calls are asynchronous on the context's stream; a context is used by one
 *    host thread at a time.
 */
#ifndef FEELMRI_B200_H
#define FEELMRI_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FM_API __attribute__((visibility("default")))
#else
#define FM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define FM_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define FM_OK 0
#define FM_ERR_SHAPE 1       /* inconsistent sizes between arguments        */
#define FM_ERR_DTYPE 2       /* unsupported element type / kind code         */
#define FM_ERR_CUDA 3        /* a CUDA runtime call failed                    */
#define FM_ERR_NOMEM 4       /* workspace or output capacity too small        */
#define FM_ERR_TIMEOUT 5     /* a bounded device wait ran out                  */
#define FM_ERR_ARG 6         /* null pointer / invalid enum / bad handle       */
#define FM_ERR_UNSUPPORTED 7 /* valid request this build does not implement   */
#define FM_ERR_CANCELLED 8   /* request cancelled before completion            */

/* ---- numeric kinds: how a Python scalar takes part in NumPy 2 arithmetic.
 * The reference's motion callables combine the time passed from C++ (a
 * Python float) with a timeshift and a period whose NumPy types decide the
 * precision of the fold (python/feelmri/Motion.py:142-149, :248).         */
#define FM_NUM_NONE 0        /* absent (non-periodic motion)                  */
#define FM_NUM_PYFLOAT 1     /* Python float / int: weak, double arithmetic   */
#define FM_NUM_F32 2         /* numpy.float32: float arithmetic               */
#define FM_NUM_F64 3         /* numpy.float64 (or numpy integer): double      */

/* ---- motion descriptors ------------------------------------------------ */
#define FM_MOTION_NONE 0     /* pod_trajectory is None                        */
#define FM_MOTION_TERMS 1    /* sum of POD / PODVelocity / respiratory terms   */
#define FM_MOTION_TABLE 2    /* displacements sampled by the caller            */

#define FM_TERM_POD 0          /* Motion.py:240-254                            */
#define FM_TERM_POD_VELOCITY 1 /* Motion.py:272-290 (weights *= unfolded t)    */
#define FM_TERM_RESPIRATORY 2  /* Motion.py:58-103 (scalar spline x direction) */

#define FM_MAX_MOTION_TERMS 4

typedef struct fm_motion_term {
  int32_t kind;            /* FM_TERM_*                                         */
  int32_t n_modes;         /* r: number of POD modes (1 for respiratory)       */
  const float *modes;      /* POD: (N, 3, r) C-contiguous float32              */
  const double *pp_c;      /* PPoly coefficients (k, n_intervals, r) float64   */
  const double *pp_x;      /* PPoly breakpoints (n_intervals + 1,) float64     */
  int32_t pp_k;            /* polynomial order + 1 (4 for cubic)               */
  int32_t pp_intervals;    /* number of intervals                              */
  double timeshift;        /* value of .timeshift                              */
  int32_t timeshift_kind;  /* FM_NUM_* of .timeshift                           */
  int32_t period_kind;     /* FM_NUM_NONE unless periodic                      */
  double period;           /* value of ._period                                */
  float direction[3];      /* respiratory: normalised direction (float32)     */
  int32_t extrapolate;     /* PPoly(extrapolate=...); the reference uses 0     */
} fm_motion_term;

typedef struct fm_motion {
  int32_t kind;                               /* FM_MOTION_*                   */
  int32_t n_terms;                            /* TERMS: summed left to right   */
  fm_motion_term terms[FM_MAX_MOTION_TERMS];
  const void *table;                          /* TABLE: (n_calls, N, 3), float
                                                 (double for FM_PREC_F64)      */
  int64_t table_calls;                        /* TABLE: number of sampled calls*/
} fm_motion;

/* ---- lifecycle --------------------------------------------------------- */
typedef struct fm_ctx fm_ctx;

/* Creates a context bound to CUDA device `device`; the stream starts as the
 * legacy default stream.  New component: the reference has no GPU context. */
FM_API int fm_ctx_create(int device, fm_ctx **out);
FM_API int fm_ctx_destroy(fm_ctx *ctx);
/* `stream` is a cudaStream_t passed as void*. */
FM_API int fm_ctx_set_stream(fm_ctx *ctx, void *stream);
/* Blocks until all work queued on the context's stream has finished. */
FM_API int fm_ctx_synchronize(fm_ctx *ctx);
/* Copies the last error message of the calling thread into buf (NUL
 * terminated, truncated to len).  Returns the last status code. */
FM_API int fm_last_error(char *buf, size_t len);
FM_API int fm_abi_version(void);
/* Number of kernel launches issued by this library since load (all
 * contexts); used by benchmarks to report launches inside a timed region. */
FM_API int64_t fm_launch_count(void);
/* Kernel timing: while enabled, the context records CUDA events on its
 * stream around each launch of its main kernels (the Bloch sweep and the
 * Signal contraction kernels).  fm_ctx_timing_query synchronises those
 * events and returns the summed duration (ms) and launch count of the
 * kernels whose name starts with `prefix`; fm_ctx_timing_reset clears them.
 * New component: the reference has no kernels to time. */
FM_API int fm_ctx_timing_enable(fm_ctx *ctx, int on);
FM_API int fm_ctx_timing_reset(fm_ctx *ctx);
FM_API int fm_ctx_timing_query(fm_ctx *ctx, const char *prefix, double *total_ms, int64_t *launches);

/* ---- POD: tensordot_modes_weights -------------------------------------- */
/* Replaces POD.tensordot_modes_weights<float|double>
 * (cpp/feelmri/POD.cpp:5-38, bound at cpp/feelmri/POD.h:16-24):
 * out[p, c] = sum_m modes[p, c, m] * weights[m].
 * modes (P, C, M) C-contiguous, weights (M,), out (P, C) C-contiguous. */
FM_API int fm_pod_tensordot_f32(fm_ctx *ctx, const float *modes, const float *weights,
                         int64_t P, int64_t C, int64_t M, float *out);
FM_API int fm_pod_tensordot_f64(fm_ctx *ctx, const double *modes,
                         const double *weights, int64_t P, int64_t C,
                         int64_t M, double *out);

/* Snapshot products of POD.calculate_pod (python/feelmri/Motion.py:174-211),
 * the O(rows t^2) part of building a POD, on the device.  X is the
 * (rows x t) snapshot matrix data.reshape(-1, t) (rows = P * C), row-major.
 *   fm_pod_gram_*:    gram = X^T X, (t x t) float64            (Motion.py:189)
 *   fm_pod_project_*: phi = X E (rows x n_modes, X's type) and
 *                     weights = X^T phi (t x n_modes, float64)   (Motion.py:202-204)
 * with E (t x n_modes, float64) the scaled eigenvectors; the t x t
 * eigenproblem stays on the host.  Sums are accumulated in FP64 in a fixed
 * order (reproducible run to run); 1 <= t <= 1024.  All pointers are device
 * memory; the workspace is sized by fm_pod_build_workspace_size.  New
 * component: the reference builds the POD with numpy on the host. */
FM_API int fm_pod_build_workspace_size(int64_t rows, int32_t t, int32_t n_modes, size_t *bytes);
FM_API int fm_pod_gram_f32(fm_ctx *ctx, const float *X, int64_t rows, int32_t t, double *gram, void *workspace,
                           size_t workspace_bytes);
FM_API int fm_pod_gram_f64(fm_ctx *ctx, const double *X, int64_t rows, int32_t t, double *gram, void *workspace,
                           size_t workspace_bytes);
FM_API int fm_pod_project_f32(fm_ctx *ctx, const float *X, int64_t rows, int32_t t, const double *E,
                              int32_t n_modes, float *phi, double *weights, void *workspace, size_t workspace_bytes);
FM_API int fm_pod_project_f64(fm_ctx *ctx, const double *X, int64_t rows, int32_t t, const double *E,
                              int32_t n_modes, double *phi, double *weights, void *workspace,
                              size_t workspace_bytes);

/* Evaluates a lowered motion callable at n_times host-given times, exactly as
 * pod_trajectory(t) would (python/feelmri/Motion.py:237-254, :272-290,
 * :303-309, :58-103): out (n_times, N, 3) float32.  `times` is a HOST array
 * of the float64 values passed to the callable. */
FM_API int fm_motion_eval(fm_ctx *ctx, const fm_motion *motion, int64_t n_nodes,
                   const double *times, int64_t n_times, float *out,
                   void *workspace, size_t workspace_bytes);
FM_API int fm_motion_eval_workspace_size(const fm_motion *motion, int64_t n_nodes,
                                  int64_t n_times, size_t *bytes);

/* Receive-coil columns: out[n, c] = m[n] * sens[n, c] (complex64), the (N, C)
 * Mxy that Signal sums per coil.  New component: the reference's Signal
 * takes no coil sensitivities (cpp/feelmri/MRI.cpp:38-48). */
FM_API int fm_coil_expand(fm_ctx *ctx, const float *m, const float *sens, int64_t N, int64_t C, float *out);

/* ---- BlochSimulator.solve_mri ------------------------------------------ */
typedef struct fm_bloch_args {
  int64_t n_pos;           /* N                                             */
  int64_t n_time;          /* n_t = rf_all.size()                           */
  const float *r0;         /* (N, 3) row-major                              */
  const float *T1;         /* (N,) ms                                       */
  const float *T2;         /* (N,) ms                                       */
  const float *delta_B;    /* (N,) mT                                       */
  float M0;
  float gamma;             /* rad / (ms mT)                                 */
  const float *rf;         /* (n_t,) complex64, mT                          */
  const float *G;          /* (n_t, 3) row-major, mT/m                       */
  const float *dt;         /* (n_t,) ms; dt[0] is ignored                    */
  const float *Mxy0;       /* (N,) complex64                                */
  const float *Mz0;        /* (N,)                                          */
  const fm_motion *motion; /* NULL or kind NONE for the static overload     */
  float *Mxy_hist;         /* (N, n_t) column-major complex64, or NULL      */
  float *Mz_hist;          /* (N, n_t) column-major float32, or NULL        */
  float *Mxy_final;        /* (N,) complex64 state after the last step, or NULL */
  float *Mz_final;         /* (N,) float32, or NULL                         */
  float *Mxy_carry;        /* (N,) complex64 receiving 0 * final Mxy, or NULL:
                              BlochSolver's artificial spoiling of the state
                              carried past a non-empty block (Bloch.py:363-367) */
  int64_t final_stride;    /* element stride of Mxy_final (0 or 1: contiguous);
                              lets a sweep write one column of an (N, V) matrix */
} fm_bloch_args;

/* Replaces solve_mri<float>(..., py::function) (cpp/feelmri/BlochSimulator.cpp:12-148,
 * bound at cpp/feelmri/BlochSimulator.h:53-66) and solve_mri<float>(..., py::none)
 * (BlochSimulator.cpp:151-277, bound at BlochSimulator.h:67-80).  With both
 * history pointers set it is the API-exact form; with only the *_final
 * pointers it is the final-state form BlochSolver.solve needs
 * (python/feelmri/Bloch.py:355-359).  A TABLE motion holds n_t entries:
 * entry 0 is the pod_trajectory(0.0) call, entry i (i >= 1) the call at the
 * float32 running time of step i-1 -> i. */
FM_API int fm_bloch_solve_f32(fm_ctx *ctx, const fm_bloch_args *args, void *workspace,
                       size_t workspace_bytes);
FM_API int fm_bloch_workspace_size(const fm_bloch_args *args, size_t *bytes);

/* ---- BlochSolver.solve: a whole block sequence in one sweep ------------- */
/* One block of a sequence (host array). */
typedef struct fm_bloch_block {
  int64_t offset;          /* first sample of the block in rf / G / dt      */
  int64_t n_time;          /* samples of the block (>= 1); the first sample
                              is the block's initial-state column            */
  int32_t empty;           /* nonzero: the final Mxy is carried on; zero:
                              0 * Mxy is carried (Bloch.py:363-367)          */
  int32_t store;           /* row of Mxy_out / Mz_out for the block's final
                              state (store_magnetization), or -1            */
  double timeshift[FM_MAX_MOTION_TERMS];       /* each motion term's .timeshift
                              during the block (update_timeshift(t0))       */
  int32_t timeshift_kind[FM_MAX_MOTION_TERMS]; /* FM_NUM_* of those values   */
} fm_bloch_block;

typedef struct fm_bloch_sequence_args {
  int64_t n_pos;           /* N                                             */
  const float *r0;         /* (N, 3) row-major                              */
  const float *T1, *T2;    /* (N,) ms                                       */
  const float *delta_B;    /* (N,) mT                                       */
  float M0;
  float gamma;             /* rad / (ms mT)                                 */
  int32_t n_blocks;
  const fm_bloch_block *blocks; /* host array of n_blocks, offsets contiguous
                              from 0 in block order                          */
  int64_t n_samples;       /* sum of the blocks' n_time                     */
  const float *rf;         /* (n_samples,) complex64, mT, blocks concatenated */
  const float *G;          /* (n_samples, 3) row-major, mT/m                 */
  const float *dt;         /* (n_samples,) ms; each block's first is ignored */
  const float *Mxy0;       /* (N,) complex64 state before the first block   */
  const float *Mz0;        /* (N,)                                          */
  const fm_motion *motion; /* NULL, NONE or TERMS (a TABLE motion is not
                              accepted); the per-block timeshifts replace
                              terms[k].timeshift                             */
  int32_t n_store;         /* rows of Mxy_out / Mz_out                      */
  float *Mxy_out;          /* (n_store, N) complex64 stored final states    */
  float *Mz_out;           /* (n_store, N) float32                          */
  float *Mxy_carry;        /* (N,) state carried past the last block, or
                              NULL; may alias Mxy0                          */
  float *Mz_carry;         /* (N,) or NULL; may alias Mz0                   */
} fm_bloch_sequence_args;

/* Replaces BlochSolver.solve's block loop (python/feelmri/Bloch.py:332-368),
 * which calls solve_mri (cpp/feelmri/BlochSimulator.cpp:12-148 / :151-277)
 * once per block and carries the state on the host: here every block runs in
 * one sweep with the magnetisation in registers.  Per block: the motion
 * terms' timeshift is the block's, each block's dt[0] is ignored and its
 * running time restarts at 0; after the block its final state is stored when
 * requested and 0 * Mxy is carried on unless the block is empty.  Stored rows
 * and the carried state equal the per-block fm_bloch_solve_f32 loop's bit for
 * bit.  The block table is copied to the device from host memory, so this
 * call is not meant for stream capture. */
FM_API int fm_bloch_sequence_f32(fm_ctx *ctx, const fm_bloch_sequence_args *args, void *workspace,
                                 size_t workspace_bytes);
FM_API int fm_bloch_sequence_workspace_size(const fm_bloch_sequence_args *args, size_t *bytes);

/* Scratch held by the library for fm_bloch_solve_f32_noalloc, per device. */
#define FM_NOALLOC_BLOCH_SCRATCH_BYTES (4u << 20)

/* Same computation as fm_bloch_solve_f32, for callers that cannot allocate
 * device memory: code running where allocation is forbidden (inside a
 * region another runtime is capturing, a real-time loop, or a host
 * framework that owns every allocation through its own pool and offers no
 * way to hand out a workspace).  The caller still provides every input and
 * output buffer; the per-step scratch lives in a fixed-size array of device
 * memory inside this library (FM_NOALLOC_BLOCH_SCRATCH_BYTES, enough for
 * about 50,000 time steps with a 10-mode motion; larger requests are rejected
 * with FM_ERR_NOMEM and the size they would need).  Every GPU that loads the
 * library keeps that array until the process exits.
 * The first call on a device looks up the array's device address (with that
 * device current); make that first call before any stream capture.  All calls
 * on a device share the one array, which keeps the previous call's contents
 * (nothing in it needs to start at zero: each call writes every entry it
 * reads), so calls that may overlap on the GPU -- on different streams or
 * from different threads -- race and must be serialised by the caller.
 * No counterpart in the reference: its solve_mri runs on the CPU. */
FM_API int fm_bloch_solve_f32_noalloc(fm_ctx *ctx, const fm_bloch_args *args);

/* ---- MRI.Signal -------------------------------------------------------- */
#define FM_PREC_F32 0        /* plain FP32 CUDA-core form (drop-in)            */
#define FM_PREC_F64 1        /* FP64 form (the reference's double overload)    */
#define FM_PREC_BF16X3 2     /* split-BF16 tcgen05 tensor-core form            */

typedef struct fm_signal_args {
  int64_t n_nodes;         /* N = r0.rows()                                 */
  int64_t n_vencs;         /* V = Mxy.cols()                                */
  int64_t n_ro, n_lines, n_kz; /* sample grid (kloc[0].dimensions)          */
  /* M: sparse (m_rows x m_cols) in CSC, element type = precision's real. */
  int64_t m_rows, m_cols, m_nnz;
  const int32_t *m_indptr; /* (m_cols + 1,)                                 */
  const int32_t *m_indices;/* (m_nnz,)                                      */
  const void *m_data;      /* (m_nnz,)                                      */
  const void *kx, *ky, *kz;/* (n_ro*n_lines*n_kz,) C-order, 1/m             */
  const void *t;           /* (n_ro*n_lines*n_kz,) C-order, ms              */
  const void *r0;          /* (N, 3) row-major, m                           */
  const void *phi;         /* (N,) rad/ms                                   */
  const void *T2;          /* (N,) ms                                       */
  const void *Mxy;         /* (N, V) row-major complex                      */
  const fm_motion *motion; /* NULL/NONE, TERMS, or TABLE with one entry per
                              distinct-time run of t (in sample order)      */
  void *out;               /* (n_ro*n_lines*n_kz, V) row-major complex      */
} fm_signal_args;

/* Replaces Signal<T>(..., py::function) (cpp/feelmri/MRI.cpp:38-159, bound at
 * cpp/feelmri/MRI.h:46-53 (float) and :65-72 (double)) and Signal<T>(...,
 * py::none) (MRI.cpp:196-298, bound at MRI.h:55-62 and :74-81).
 * precision: FM_PREC_F32 reads float inputs, FM_PREC_F64 double inputs,
 * FM_PREC_BF16X3 float inputs (split-BF16 tensor-core contraction with the
 * phase reduced modulo one cycle in FP64). */
FM_API int fm_signal(fm_ctx *ctx, const fm_signal_args *args, int precision,
              void *workspace, size_t workspace_bytes);
/* fm_signal in two halves.  fm_signal_enqueue only queues work on the
 * context's stream: it never waits for the device, so a sequence of calls
 * can be captured in a CUDA graph or overlapped with other streams.  Errors
 * found on the device (a sparse row index out of range, a TABLE motion with
 * the wrong number of entries, a tensor-core wait that ran out) are kept in
 * the workspace; fm_signal_status waits for the stream and reports them for
 * the call that used that workspace. */
FM_API int fm_signal_enqueue(fm_ctx *ctx, const fm_signal_args *args, int precision,
                             void *workspace, size_t workspace_bytes);
FM_API int fm_signal_status(fm_ctx *ctx, const fm_signal_args *args, int precision,
                            void *workspace, size_t workspace_bytes);
FM_API int fm_signal_workspace_size(const fm_signal_args *args, int precision,
                             size_t *bytes);
/* Self-test of the bounded device waits the tensor-core kernels use (no
 * counterpart in the reference): one thread waits on an mbarrier that
 * nothing arrives on, gives up after `limit_ns` of device wall time and
 * records the timeout; the call returns FM_ERR_TIMEOUT (the expected
 * outcome) after synchronising the context's stream.  The context and the
 * device stay usable.  Lets a host check its failure handling without a
 * GPU fault. */
FM_API int fm_selftest_wait(fm_ctx *ctx, uint64_t limit_ns);

/* Batched split-BF16 Signal (no counterpart in the reference, which calls
 * Signal once per phantom, e.g. examples/phase_contrast.py:207): n problems,
 * each an fm_signal_args with its own mesh, trajectory, columns, motion and
 * output (float inputs, as FM_PREC_BF16X3), prepared one after another and
 * then contracted by ONE persistent tensor-core launch over the work units
 * of all of them.  Enqueue-only (capturable in a CUDA graph); the status
 * call waits and reports device errors.  A problem's result depends on the
 * problem and the tuning only, not on the rest of the batch.  `tune` may be
 * NULL (defaults). */
typedef struct fm_tc_tuning {
  int32_t split_nodes;  /* nodes per unit along the node range (0: spread one
                           problem's units evenly over the SMs)             */
  int32_t kz_cap;       /* most kz values per tile of a factored run (0: up
                           to 64 within 128 (kz, column) pairs)             */
  int32_t reserved[2];
} fm_tc_tuning;

FM_API int fm_signal_batch_workspace_size(const fm_signal_args *probs, int n_probs, size_t *bytes);
FM_API int fm_signal_batch_enqueue(fm_ctx *ctx, const fm_signal_args *probs, int n_probs,
                                   const fm_tc_tuning *tune, void *workspace, size_t workspace_bytes);
FM_API int fm_signal_batch_status(fm_ctx *ctx, const fm_signal_args *probs, int n_probs,
                                  void *workspace, size_t workspace_bytes);

/* Number of distinct-time runs of t (MRI.cpp:109-134 refreshes positions,
 * off-resonance and decay once per run).  `t` is a HOST array here. */
FM_API int64_t fm_signal_count_time_runs(const void *t_host, int64_t n_samples,
                                  int is_double);

/* ---- Assemble.MassAssemble ---------------------------------------------- */
typedef struct fm_mass_args {
  int64_t n_elems;         /* E                                             */
  int32_t nodes_per_elem;  /* nb (4 for P1 tetrahedra; at most 10)          */
  const int32_t *elems;    /* (E, nb) row-major                             */
  int64_t n_nodes;         /* N                                             */
  const void *nodes;       /* (N, 3) row-major, float or double             */
  int32_t n_qpoints;       /* Q                                             */
  const void *qweights;    /* (Q,)                                          */
  const void *tabulated;   /* (Q, 4, nb): value, d/dr, d/ds, d/dt of each
                              basis function at each quadrature point        */
} fm_mass_args;

/* Replaces MassAssemble<T> -> LocalMassAssemble<T> -> IsoMapping<T>
 * (cpp/feelmri/Assemble.cpp:79-116, :59-75, :16-55; bound at
 * cpp/feelmri/Assemble.h:26-38).  Produces the CSC matrix Eigen's
 * setFromTriplets builds: duplicates summed in element order, row indices
 * sorted within each column.  Two-phase: with indices/data NULL only
 * *nnz_out (and indptr when non-NULL) are produced.  is_double selects T. */
FM_API int fm_mass_assemble(fm_ctx *ctx, const fm_mass_args *args, int is_double,
                     int64_t *nnz_out, int32_t *indptr, int32_t *indices,
                     void *data, int64_t capacity, void *workspace,
                     size_t workspace_bytes);
/* Lumped mass as FEMPhantom.mass_matrix(lumped=True) forms it
 * (python/feelmri/Phantom.py:395-398): row sums of the assembled matrix in
 * scipy's csc @ ones order.  out (N,) of type T. */
FM_API int fm_mass_lumped(fm_ctx *ctx, const fm_mass_args *args, int is_double,
                   void *out, void *workspace, size_t workspace_bytes);
FM_API int fm_mass_workspace_size(const fm_mass_args *args, int is_double,
                           size_t *bytes);

#ifdef __cplusplus
}
#endif
#endif /* FEELMRI_B200_H */
