// POD tensordot (cpp/feelmri/POD.cpp:5-38) and the device-side evaluation of
// the motion callables of python/feelmri/Motion.py.
#include "motion.cuh"

namespace fm {

int validate_motion(const fm_motion *m, int64_t n_nodes, const char *who) {
  if (m == nullptr || m->kind == FM_MOTION_NONE) return FM_OK;
  if (m->kind == FM_MOTION_TABLE) {
    FM_REQUIRE(m->table != nullptr, FM_ERR_ARG, "%s: TABLE motion without a table", who);
    FM_REQUIRE(m->table_calls >= 0, FM_ERR_SHAPE, "%s: negative table_calls", who);
    return FM_OK;
  }
  FM_REQUIRE(m->kind == FM_MOTION_TERMS, FM_ERR_ARG, "%s: unknown motion kind %d", who, m->kind);
  FM_REQUIRE(m->n_terms >= 1 && m->n_terms <= FM_MAX_MOTION_TERMS, FM_ERR_ARG, "%s: n_terms=%d out of [1,%d]",
             who, m->n_terms, FM_MAX_MOTION_TERMS);
  for (int k = 0; k < m->n_terms; ++k) {
    const fm_motion_term &T = m->terms[k];
    FM_REQUIRE(T.kind == FM_TERM_POD || T.kind == FM_TERM_POD_VELOCITY || T.kind == FM_TERM_RESPIRATORY,
               FM_ERR_ARG, "%s: term %d has unknown kind %d", who, k, T.kind);
    FM_REQUIRE(T.pp_c != nullptr && T.pp_x != nullptr, FM_ERR_ARG, "%s: term %d lacks spline data", who, k);
    FM_REQUIRE(T.pp_k >= 1 && T.pp_intervals >= 1, FM_ERR_SHAPE, "%s: term %d has an empty spline", who, k);
    FM_REQUIRE(T.timeshift_kind >= FM_NUM_PYFLOAT && T.timeshift_kind <= FM_NUM_F64, FM_ERR_DTYPE,
               "%s: term %d timeshift kind %d invalid", who, k, T.timeshift_kind);
    FM_REQUIRE(T.period_kind >= FM_NUM_NONE && T.period_kind <= FM_NUM_F64, FM_ERR_DTYPE,
               "%s: term %d period kind %d invalid", who, k, T.period_kind);
    if (T.kind == FM_TERM_RESPIRATORY) {
      FM_REQUIRE(T.n_modes == 1, FM_ERR_SHAPE, "%s: respiratory term %d must have one spline column", who, k);
    } else {
      FM_REQUIRE(T.modes != nullptr && T.n_modes >= 1, FM_ERR_ARG, "%s: POD term %d lacks modes", who, k);
      (void)n_nodes;
    }
  }
  return FM_OK;
}

// One thread per (call, slot).
__global__ void motion_weights_kernel(MotionDev md, const double *__restrict__ times, int64_t n_calls,
                                      float *__restrict__ weights) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_calls * md.slots) return;
  const int64_t c = idx / md.slots;
  const int s = (int)(idx - c * md.slots);
  int k = 0;
  while (k + 1 < md.n_terms && s >= md.slot0[k + 1]) ++k;
  const fm_motion_term &T = md.terms[k];
  const int col = s - md.slot0[k];
  const double t = times[c];
  const double te = term_time(t, T);
  const double v = ppoly_eval(T.pp_c, T.pp_x, T.pp_k, T.pp_intervals, T.n_modes, col, te, T.extrapolate);
  float w = __double2float_rn(v);
  if (T.kind == FM_TERM_POD_VELOCITY) w = __fmul_rn(w, __double2float_rn(t));
  weights[idx] = w;
}

int launch_motion_weights(const MotionDev &md, const double *times_dev, int64_t n_calls, float *weights,
                          cudaStream_t st) {
  if (md.kind != FM_MOTION_TERMS || n_calls == 0) return FM_OK;
  const int64_t total = n_calls * md.slots;
  const int threads = 128;
  motion_weights_kernel<<<(unsigned)ceil_div(total, threads), threads, 0, st>>>(md, times_dev, n_calls, weights);
  count_launch();
  return check_launch("motion_weights_kernel");
}

// out[c, n, :] = displacement of node n at call c.
__global__ void motion_disp_kernel(MotionDev md, const float *__restrict__ weights, int64_t n_nodes,
                                   int64_t n_calls, float *__restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_calls * n_nodes) return;
  const int64_t c = idx / n_nodes;
  const int64_t n = idx - c * n_nodes;
  float dx, dy, dz;
  motion_disp(md, weights + c * md.slots, n, n_nodes, dx, dy, dz);
  out[idx * 3 + 0] = dx;
  out[idx * 3 + 1] = dy;
  out[idx * 3 + 2] = dz;
}

// GEMV over rows of a (rows x M) row-major matrix; one warp per row group.
template <typename T>
__global__ void tensordot_kernel(const T *__restrict__ A, const T *__restrict__ w, int64_t rows, int64_t M,
                                 T *__restrict__ out) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  const T *a = A + row * M;
  T acc = T(0);
  for (int64_t m = 0; m < M; ++m) acc = fma(__ldg(a + m), __ldg(w + m), acc);
  out[row] = acc;
}

// Row-parallel GEMV with the matrix staged through shared memory so that
// the loads of a warp are contiguous (rows are M elements long).
template <typename T, int ROWS>
__global__ void tensordot_tiled_kernel(const T *__restrict__ A, const T *__restrict__ w, int64_t rows, int M,
                                       T *__restrict__ out) {
  extern __shared__ unsigned char smem_raw[];
  T *tile = reinterpret_cast<T *>(smem_raw);   // ROWS * M
  T *ws = tile + (size_t)ROWS * M;             // M
  const int64_t row0 = (int64_t)blockIdx.x * ROWS;
  const int64_t nrows = min((int64_t)ROWS, rows - row0);
  for (int m = threadIdx.x; m < M; m += blockDim.x) ws[m] = w[m];
  const T *src = A + row0 * M;
  const int64_t total = nrows * M;
  for (int64_t i = threadIdx.x; i < total; i += blockDim.x) tile[i] = __ldg(src + i);
  __syncthreads();
  for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
    const T *a = tile + (size_t)r * M;
    T acc = T(0);
    for (int m = 0; m < M; ++m) acc = fma(a[m], ws[m], acc);
    out[row0 + r] = acc;
  }
}

template <typename T>
static int tensordot_impl(fm_ctx *ctx, const T *modes, const T *weights, int64_t P, int64_t C, int64_t M, T *out,
                          const char *who) {
  FM_TRY(ctx_ok(ctx));
  FM_REQUIRE(P >= 0 && C >= 0 && M >= 0, FM_ERR_SHAPE, "%s: negative extent", who);
  const int64_t rows = P * C;
  if (rows == 0) return FM_OK;
  FM_REQUIRE(out != nullptr, FM_ERR_ARG, "%s: null output", who);
  DeviceGuard g(ctx->device);
  if (M == 0) {
    FM_CUDA(cudaMemsetAsync(out, 0, rows * sizeof(T), ctx->stream));
    return FM_OK;
  }
  FM_REQUIRE(modes != nullptr && weights != nullptr, FM_ERR_ARG, "%s: null input", who);
  constexpr int ROWS = 256;
  const size_t smem = ((size_t)ROWS * M + M) * sizeof(T);
  if (smem <= 48 * 1024) {
    tensordot_tiled_kernel<T, ROWS><<<(unsigned)ceil_div(rows, ROWS), 256, smem, ctx->stream>>>(modes, weights, rows,
                                                                                                   (int)M, out);
  } else {
    tensordot_kernel<T><<<(unsigned)ceil_div(rows, 256), 256, 0, ctx->stream>>>(modes, weights, rows, M, out);
  }
  count_launch();
  return check_launch(who);
}

}  // namespace fm

using namespace fm;

extern "C" {

int fm_pod_tensordot_f32(fm_ctx *ctx, const float *modes, const float *weights, int64_t P, int64_t C, int64_t M,
                         float *out) {
  return tensordot_impl<float>(ctx, modes, weights, P, C, M, out, "fm_pod_tensordot_f32");
}

int fm_pod_tensordot_f64(fm_ctx *ctx, const double *modes, const double *weights, int64_t P, int64_t C, int64_t M,
                         double *out) {
  return tensordot_impl<double>(ctx, modes, weights, P, C, M, out, "fm_pod_tensordot_f64");
}

int fm_motion_eval_workspace_size(const fm_motion *motion, int64_t n_nodes, int64_t n_times, size_t *bytes) {
  FM_REQUIRE(bytes != nullptr, FM_ERR_ARG, "fm_motion_eval_workspace_size: null output");
  Carve c(nullptr, 0);
  c.take<double>(n_times);
  c.take<float>((size_t)n_times * motion_slots(motion));
  *bytes = c.used;
  (void)n_nodes;
  return FM_OK;
}

int fm_motion_eval(fm_ctx *ctx, const fm_motion *motion, int64_t n_nodes, const double *times, int64_t n_times,
                   float *out, void *workspace, size_t workspace_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_REQUIRE(motion != nullptr, FM_ERR_ARG, "fm_motion_eval: null motion");
  FM_REQUIRE(motion->kind == FM_MOTION_TERMS, FM_ERR_ARG, "fm_motion_eval: only TERMS motion can be evaluated");
  FM_TRY(validate_motion(motion, n_nodes, "fm_motion_eval"));
  FM_REQUIRE(n_nodes >= 0 && n_times >= 0, FM_ERR_SHAPE, "fm_motion_eval: negative extent");
  if (n_nodes == 0 || n_times == 0) return FM_OK;
  FM_REQUIRE(times != nullptr && out != nullptr, FM_ERR_ARG, "fm_motion_eval: null pointer");
  DeviceGuard g(ctx->device);
  MotionDev md = make_motion_dev(motion);
  Carve cv(workspace, workspace_bytes);
  double *tdev = cv.take<double>(n_times);
  float *w = cv.take<float>((size_t)n_times * md.slots);
  FM_TRY(carve_ok(cv, "fm_motion_eval"));
  FM_CUDA(cudaMemcpyAsync(tdev, times, n_times * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  FM_TRY(launch_motion_weights(md, tdev, n_times, w, ctx->stream));
  const int64_t total = n_times * n_nodes;
  motion_disp_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, ctx->stream>>>(md, w, n_nodes, n_times, out);
  count_launch();
  FM_TRY(check_launch("motion_disp_kernel"));
  // The host times array may be reused by the caller as soon as we return.
  FM_CUDA(cudaStreamSynchronize(ctx->stream));
  return FM_OK;
}

}  // extern "C"

// ---- coil columns ---------------------------------------------------------
// out[n, c] = m[n] * sens[n, c]: the transverse magnetisation seen by each
// receive coil, the columns of Signal's Mxy when coils are simulated.  New
// component: the reference's Signal takes no coil sensitivities.
namespace fm {
__global__ void coil_expand_kernel(const float2 *__restrict__ m, const float2 *__restrict__ sens, int64_t N,
                                   int64_t C, float2 *__restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N * C) return;
  const int64_t n = idx / C;
  const float2 a = m[n], b = sens[idx];
  out[idx] = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
}  // namespace fm

extern "C" int fm_coil_expand(fm_ctx *ctx, const float *m, const float *sens, int64_t N, int64_t C, float *out) {
  using namespace fm;
  FM_TRY(ctx_ok(ctx));
  FM_REQUIRE(N >= 0 && C >= 0, FM_ERR_SHAPE, "fm_coil_expand: negative extent");
  if (N * C == 0) return FM_OK;
  FM_REQUIRE(m && sens && out, FM_ERR_ARG, "fm_coil_expand: null pointer");
  DeviceGuard g(ctx->device);
  coil_expand_kernel<<<(unsigned)ceil_div(N * C, 256), 256, 0, ctx->stream>>>(
      reinterpret_cast<const float2 *>(m), reinterpret_cast<const float2 *>(sens), N, C, reinterpret_cast<float2 *>(out));
  count_launch();
  return check_launch("coil_expand_kernel");
}
