// Pieces shared by the Signal forms: the mass-weighted magnetisation M * Mxy,
// the distinct-time runs of the sample times, and the tile list that maps
// thread blocks to runs.
#pragma once
#include "motion.cuh"

namespace fm {

// Samples per tile of the plain (CUDA-core) forms.
constexpr int kPlainThreads = 256;
// SM count of a B200; sizes split-K fan-out so workspace queries need no device.
constexpr int kSmCount = 148;

// Device view of the sample runs ("time groups"): run g covers samples
// [start[g], start[g+1]) which share one time t_g.
struct Runs {
  int *flag;        // (S,) 1 where a run starts
  int *gid;         // (S,) inclusive scan of flag
  int *start;       // (S + 1,) run starts; start[n_runs] = S
  int *tile_off;    // (S + 1,) first tile of each run
  int *tile_run;    // (max_tiles,) run of each tile
  int *tile_s0;     // (max_tiles,) first sample of each tile
  double *run_t;    // (S,) time of each run, widened to double
  int *counts;      // (8,) n_runs, n_tiles, then per-form plan values
  int *error;       // (1,) error bits of the call (kErr*)
  void *cub_tmp;
  size_t cub_bytes;
};

// CSR view of the sparse mass matrix, rows in Eigen's accumulation order.
struct Csr {
  int *rowptr;   // (rows + 1,)
  int *fill;     // (rows,)
  int *col;      // (nnz,)
  int *pos;      // (nnz,) position of the entry in the CSC arrays
  void *cub_tmp;
  size_t cub_bytes;
};

int64_t max_tiles_for(int64_t S, int tile);

void carve_runs(Carve &c, int64_t S, int tile, Runs &r);
void carve_csr(Carve &c, int64_t rows, int64_t nnz, Csr &m);

// Error bits recorded on the device during a Signal call.
constexpr int kErrTimeout = 1;      // a tensor-core pipeline wait ran out
constexpr int kErrSparseRow = 2;    // a row index of M outside [0, rows)
constexpr int kErrTableCalls = 4;   // TABLE motion entries != distinct-time runs
constexpr int kErrPhaseRange = 8;   // a tensor-core phase k . r may reach 2^27 cycles

// Builds runs and tiles of `tile` samples on the device: counts[0] = runs,
// counts[1] = tiles.  No host synchronisation.
template <typename T>
int build_runs(const T *t, int64_t S, int tile, Runs &r, cudaStream_t st);

// Sets kErrTableCalls when a TABLE motion does not hold one entry per run.
int check_table_calls(const fm_motion *m, Runs &r, cudaStream_t st);

// Reads and clears the error word (synchronises the stream) and maps it to a
// status with a message.
int report_errors(Runs &r, cudaStream_t st, const char *who);

// MM[i, v] = sum_j M[i, j] * Mxy[j, v] accumulated over j ascending (Eigen's
// column-major sparse x dense product, cpp/feelmri/MRI.cpp:92).
template <typename T>
int sparse_times_dense(const fm_signal_args *a, Csr &m, const T *Mxy, T *MM, int *error, cudaStream_t st);

// Motion weights for the runs, with the run count read on the device.
int launch_run_weights(const MotionDev &md, const double *run_t, const int *n_runs, int64_t max_runs,
                       float *weights, cudaStream_t st);

}  // namespace fm
