// Shared Signal preprocessing: distinct-time runs and the sparse product.
#include <cub/cub.cuh>

#include "signal_common.cuh"

namespace fm {

int64_t max_tiles_for(int64_t S, int tile) { return S + S / tile + 1; }

static size_t cub_scan_bytes(int64_t n) {
  size_t b = 0;
  cub::DeviceScan::InclusiveSum(nullptr, b, (int *)nullptr, (int *)nullptr, (int)(n > 0 ? n : 1));
  size_t b2 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, b2, (int *)nullptr, (int *)nullptr, (int)(n > 0 ? n : 1));
  return b > b2 ? b : b2;
}

void carve_runs(Carve &c, int64_t S, int tile, Runs &r) {
  const int64_t mt = max_tiles_for(S, tile);
  r.flag = c.take<int>(S + 1);
  r.gid = c.take<int>(S + 1);
  r.start = c.take<int>(S + 1);
  r.tile_off = c.take<int>(S + 1);
  r.tile_run = c.take<int>(mt);
  r.tile_s0 = c.take<int>(mt);
  r.run_t = c.take<double>(S + 1);
  r.counts = c.take<int>(8);
  r.error = c.take<int>(4);
  r.cub_bytes = cub_scan_bytes(S + 1);
  r.cub_tmp = c.take<char>(r.cub_bytes);
}

void carve_csr(Carve &c, int64_t rows, int64_t nnz, Csr &m) {
  m.rowptr = c.take<int>(rows + 1);
  m.fill = c.take<int>(rows + 1);
  m.col = c.take<int>(nnz + 1);
  m.pos = c.take<int>(nnz + 1);
  m.cub_bytes = cub_scan_bytes(rows + 1);
  m.cub_tmp = c.take<char>(m.cub_bytes);
}

// A run starts where t differs from the previous sample (MRI.cpp:109); the
// first sample always starts one.  NaN never equals anything, so every NaN
// sample starts its own run, as in the reference's `t_old == t` test.
template <typename T>
__global__ void run_flags_kernel(const T *__restrict__ t, int64_t S, int *__restrict__ flag) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  flag[s] = (s == 0) ? 1 : (t[s] == t[s - 1] ? 0 : 1);
}

template <typename T>
__global__ void run_starts_kernel(const T *__restrict__ t, int64_t S, const int *__restrict__ flag,
                                  const int *__restrict__ gid, int *__restrict__ start, double *__restrict__ run_t,
                                  int *__restrict__ counts) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  if (flag[s]) {
    const int g = gid[s] - 1;
    start[g] = (int)s;
    run_t[g] = (double)t[s];
  }
  if (s == S - 1) {
    const int n = gid[s];
    start[n] = (int)S;
    counts[0] = n;
  }
}

__global__ void run_ntiles_kernel(const int *__restrict__ start, const int *__restrict__ counts, int tile,
                                  int *__restrict__ ntiles, int64_t S) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = counts[0];
  if (g > S) return;
  ntiles[g] = (g >= n) ? 0 : (start[g + 1] - start[g] + tile - 1) / tile;
}

__global__ void run_tiles_kernel(const int *__restrict__ start, const int *__restrict__ tile_off,
                                 int *__restrict__ counts, int tile, int *__restrict__ tile_run,
                                 int *__restrict__ tile_s0) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = counts[0];
  if (g >= n) {
    if (g == n) counts[1] = tile_off[n];
    return;
  }
  const int k0 = tile_off[g], k1 = tile_off[g + 1];
  for (int k = k0; k < k1; ++k) {
    tile_run[k] = g;
    tile_s0[k] = start[g] + (k - k0) * tile;
  }
}

template <typename T>
int build_runs(const T *t, int64_t S, int tile, Runs &r, cudaStream_t st) {
  const unsigned b = (unsigned)ceil_div(S, 256);
  FM_CUDA(cudaMemsetAsync(r.error, 0, sizeof(int), st));
  run_flags_kernel<T><<<b, 256, 0, st>>>(t, S, r.flag);
  count_launch();
  FM_TRY(check_launch("run_flags_kernel"));
  size_t cb = r.cub_bytes;
  FM_CUDA(cub::DeviceScan::InclusiveSum(r.cub_tmp, cb, r.flag, r.gid, (int)S, st));
  count_launch();
  run_starts_kernel<T><<<b, 256, 0, st>>>(t, S, r.flag, r.gid, r.start, r.run_t, r.counts);
  count_launch();
  FM_TRY(check_launch("run_starts_kernel"));
  // tile counts per run, then exclusive scan over n_runs + 1 entries (the
  // scan length is bounded by S + 1; unused tail entries are zero).
  run_ntiles_kernel<<<(unsigned)ceil_div(S + 1, 256), 256, 0, st>>>(r.start, r.counts, tile, r.flag, S);
  count_launch();
  FM_TRY(check_launch("run_ntiles_kernel"));
  cb = r.cub_bytes;
  FM_CUDA(cub::DeviceScan::ExclusiveSum(r.cub_tmp, cb, r.flag, r.tile_off, (int)(S + 1), st));
  count_launch();
  run_tiles_kernel<<<(unsigned)ceil_div(S + 1, 256), 256, 0, st>>>(r.start, r.tile_off, r.counts, tile, r.tile_run,
                                                                   r.tile_s0);
  count_launch();
  return check_launch("run_tiles_kernel");
}

__global__ void table_calls_kernel(const int *__restrict__ counts, int64_t calls, int *__restrict__ error) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && counts[0] != calls) atomicOr(error, kErrTableCalls);
}

int check_table_calls(const fm_motion *m, Runs &r, cudaStream_t st) {
  if (m == nullptr || m->kind != FM_MOTION_TABLE) return FM_OK;
  table_calls_kernel<<<1, 32, 0, st>>>(r.counts, m->table_calls, r.error);
  count_launch();
  return check_launch("table_calls_kernel");
}

int report_errors(Runs &r, cudaStream_t st, const char *who) {
  int h = 0;
  FM_CUDA(cudaMemcpyAsync(&h, r.error, sizeof(int), cudaMemcpyDeviceToHost, st));
  FM_CUDA(cudaStreamSynchronize(st));
  FM_REQUIRE(!(h & kErrSparseRow), FM_ERR_SHAPE, "%s: sparse M has a row index outside [0, rows)", who);
  FM_REQUIRE(!(h & kErrTableCalls), FM_ERR_SHAPE,
             "%s: TABLE motion must hold one entry per distinct-time run of t", who);
  FM_REQUIRE(!(h & kErrTimeout), FM_ERR_TIMEOUT, "%s: a tensor-core pipeline wait timed out", who);
  FM_REQUIRE(!(h & kErrPhaseRange), FM_ERR_ARG,
             "%s: the split-BF16 form reduces phases k . r in fixed point and needs (|kx|+|ky|+|kz|) * "
             "(|x|+|y|+|z|) below 2^27 cycles for every sample and moved node (or finite positions); use "
             "precision f32 or f64",
             who);
  return FM_OK;
}

__global__ void run_weights_kernel(MotionDev md, const double *__restrict__ times, const int *__restrict__ n_runs,
                                   float *__restrict__ weights) {
  const int64_t total = (int64_t)n_runs[0] * md.slots;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = idx / md.slots;
    const int s = (int)(idx - c * md.slots);
    int k = 0;
    while (k + 1 < md.n_terms && s >= md.slot0[k + 1]) ++k;
    const fm_motion_term &T = md.terms[k];
    const double t = times[c];
    const double v = ppoly_eval(T.pp_c, T.pp_x, T.pp_k, T.pp_intervals, T.n_modes, s - md.slot0[k],
                                term_time(t, T), T.extrapolate);
    float w = __double2float_rn(v);
    if (T.kind == FM_TERM_POD_VELOCITY) w = __fmul_rn(w, __double2float_rn(t));
    weights[idx] = w;
  }
}

int launch_run_weights(const MotionDev &md, const double *run_t, const int *n_runs, int64_t max_runs,
                       float *weights, cudaStream_t st) {
  if (md.kind != FM_MOTION_TERMS || max_runs == 0) return FM_OK;
  const int64_t total = max_runs * md.slots;
  int64_t blocks = ceil_div(total, 256);
  if (blocks > 4 * kSmCount) blocks = 4 * kSmCount;
  run_weights_kernel<<<(unsigned)blocks, 256, 0, st>>>(md, run_t, n_runs, weights);
  count_launch();
  return check_launch("run_weights_kernel");
}

template int build_runs<float>(const float *, int64_t, int, Runs &, cudaStream_t);
template int build_runs<double>(const double *, int64_t, int, Runs &, cudaStream_t);

// ---- CSC -> CSR in Eigen's accumulation order ---------------------------

__global__ void csr_count_kernel(const int *__restrict__ indices, int64_t nnz, int64_t rows, int *__restrict__ cnt,
                                 int *__restrict__ bad) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int i = indices[k];
  if (i < 0 || i >= rows) {
    atomicOr(bad, kErrSparseRow);
    return;
  }
  atomicAdd(cnt + i, 1);
}

__global__ void csr_scatter_kernel(const int *__restrict__ indptr, const int *__restrict__ indices, int64_t cols,
                                   int64_t rows, const int *__restrict__ rowptr, int *__restrict__ fill,
                                   int *__restrict__ col, int *__restrict__ pos) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  for (int k = indptr[j]; k < indptr[j + 1]; ++k) {
    const int i = indices[k];
    if (i < 0 || i >= rows) continue;
    const int slot = atomicAdd(fill + i, 1);
    col[rowptr[i] + slot] = (int)j;
    pos[rowptr[i] + slot] = k;
  }
}

// Entries of a row sorted by CSC position, which orders them by column and,
// inside a column, by storage order: the order Eigen visits them.
__global__ void csr_sort_kernel(const int *__restrict__ rowptr, int64_t rows, int *__restrict__ col,
                                int *__restrict__ pos) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  const int b = rowptr[i], e = rowptr[i + 1];
  for (int k = b + 1; k < e; ++k) {
    const int pk = pos[k], ck = col[k];
    int m = k - 1;
    while (m >= b && pos[m] > pk) {
      pos[m + 1] = pos[m];
      col[m + 1] = col[m];
      --m;
    }
    pos[m + 1] = pk;
    col[m + 1] = ck;
  }
}

template <typename T>
struct Cplx;
template <>
struct Cplx<float> {
  using type = float2;
};
template <>
struct Cplx<double> {
  using type = double2;
};

template <typename T>
__global__ void spmm_kernel(const int *__restrict__ rowptr, const int *__restrict__ col, const int *__restrict__ pos,
                            const T *__restrict__ data, int64_t rows, int64_t V,
                            const typename Cplx<T>::type *__restrict__ Mxy, typename Cplx<T>::type *__restrict__ MM) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rows * V) return;
  const int64_t i = idx / V, v = idx - (idx / V) * V;
  T re = T(0), im = T(0);
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    const T m = data[pos[k]];
    const typename Cplx<T>::type x = Mxy[(int64_t)col[k] * V + v];
    re = fma(m, x.x, re);
    im = fma(m, x.y, im);
  }
  MM[idx].x = re;
  MM[idx].y = im;
}

template <typename T>
int sparse_times_dense(const fm_signal_args *a, Csr &m, const T *Mxy, T *MM, int *error, cudaStream_t st) {
  const int64_t rows = a->m_rows, cols = a->m_cols, nnz = a->m_nnz, V = a->n_vencs;
  FM_CUDA(cudaMemsetAsync(m.fill, 0, (rows + 1) * sizeof(int), st));
  if (nnz > 0) {
    csr_count_kernel<<<(unsigned)ceil_div(nnz, 256), 256, 0, st>>>(a->m_indices, nnz, rows, m.fill, error);
    count_launch();
    FM_TRY(check_launch("csr_count_kernel"));
  }
  size_t cb = m.cub_bytes;
  FM_CUDA(cub::DeviceScan::ExclusiveSum(m.cub_tmp, cb, m.fill, m.rowptr, (int)(rows + 1), st));
  count_launch();
  FM_CUDA(cudaMemsetAsync(m.fill, 0, (rows + 1) * sizeof(int), st));
  if (cols > 0 && nnz > 0) {
    csr_scatter_kernel<<<(unsigned)ceil_div(cols, 256), 256, 0, st>>>(a->m_indptr, a->m_indices, cols, rows,
                                                                      m.rowptr, m.fill, m.col, m.pos);
    count_launch();
    FM_TRY(check_launch("csr_scatter_kernel"));
    csr_sort_kernel<<<(unsigned)ceil_div(rows, 256), 256, 0, st>>>(m.rowptr, rows, m.col, m.pos);
    count_launch();
    FM_TRY(check_launch("csr_sort_kernel"));
  }
  if (rows * V > 0) {
    using C = typename Cplx<T>::type;
    spmm_kernel<T><<<(unsigned)ceil_div(rows * V, 256), 256, 0, st>>>(
        m.rowptr, m.col, m.pos, static_cast<const T *>(a->m_data), rows, V, reinterpret_cast<const C *>(Mxy),
        reinterpret_cast<C *>(MM));
    count_launch();
    FM_TRY(check_launch("spmm_kernel"));
  }
  return FM_OK;
}

template int sparse_times_dense<float>(const fm_signal_args *, Csr &, const float *, float *, int *, cudaStream_t);
template int sparse_times_dense<double>(const fm_signal_args *, Csr &, const double *, double *, int *,
                                        cudaStream_t);

}  // namespace fm
