// fm_signal entry point: argument validation and dispatch over the forms.
#include "signal_common.cuh"
#include "tc_ptx.cuh"

namespace fm {

template <typename T>
int signal_plain(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes);
template <typename T>
size_t plain_workspace(const fm_signal_args *a);
int signal_tc(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes);
size_t tc_workspace(const fm_signal_args *a);
template <typename T>
int signal_plain_errors(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes);
int signal_tc_errors(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes);
int signal_tc_batch(fm_ctx *ctx, const fm_signal_args *probs, int n, const fm_tc_tuning *tune, void *ws,
                    size_t ws_bytes);
int signal_tc_batch_errors(fm_ctx *ctx, const fm_signal_args *probs, int n, void *ws, size_t ws_bytes);
size_t tc_batch_workspace_size(const fm_signal_args *probs, int n);

int validate_signal(const fm_signal_args *a, const char *who) {
  FM_REQUIRE(a != nullptr, FM_ERR_ARG, "%s: null args", who);
  FM_REQUIRE(a->n_nodes >= 0 && a->n_vencs >= 0 && a->n_ro >= 0 && a->n_lines >= 0 && a->n_kz >= 0, FM_ERR_SHAPE,
             "%s: negative extent", who);
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  FM_REQUIRE(S < (1LL << 31) - 2, FM_ERR_SHAPE, "%s: %lld samples exceed the 2^31 limit", who, (long long)S);
  FM_REQUIRE(a->n_nodes < (1LL << 31) - 2, FM_ERR_SHAPE, "%s: too many nodes", who);
  // M * Mxy needs M.cols() == N rows of Mxy and yields M.rows() rows, which
  // must match r0.rows() (Eigen leaves both unchecked in release builds).
  FM_REQUIRE(a->m_cols == a->n_nodes, FM_ERR_SHAPE, "%s: M has %lld columns but Mxy has %lld rows", who,
             (long long)a->m_cols, (long long)a->n_nodes);
  FM_REQUIRE(a->m_rows == a->n_nodes, FM_ERR_SHAPE, "%s: M has %lld rows but r0 has %lld nodes", who,
             (long long)a->m_rows, (long long)a->n_nodes);
  FM_REQUIRE(a->m_nnz >= 0 && a->m_nnz < (1LL << 31) - 2, FM_ERR_SHAPE, "%s: bad nnz", who);
  if (S > 0 && a->n_vencs > 0) {
    FM_REQUIRE(a->out != nullptr, FM_ERR_ARG, "%s: null output", who);
    FM_REQUIRE(a->kx && a->ky && a->kz && a->t, FM_ERR_ARG, "%s: null trajectory array", who);
    if (a->n_nodes > 0) {
      FM_REQUIRE(a->r0 && a->phi && a->T2 && a->Mxy && a->m_indptr, FM_ERR_ARG, "%s: null node array", who);
      FM_REQUIRE(a->m_nnz == 0 || (a->m_indices && a->m_data), FM_ERR_ARG, "%s: null sparse array", who);
    }
  }
  FM_TRY(validate_motion(a->motion, a->n_nodes, who));
  return FM_OK;
}

}  // namespace fm

using namespace fm;

extern "C" {

int fm_signal_workspace_size(const fm_signal_args *a, int precision, size_t *bytes) {
  FM_REQUIRE(bytes != nullptr, FM_ERR_ARG, "fm_signal_workspace_size: null output");
  FM_TRY(validate_signal(a, "fm_signal_workspace_size"));
  switch (precision) {
    case FM_PREC_F32: *bytes = plain_workspace<float>(a); return FM_OK;
    case FM_PREC_F64: *bytes = plain_workspace<double>(a); return FM_OK;
    case FM_PREC_BF16X3: *bytes = tc_workspace(a); return FM_OK;
    default: break;
  }
  set_error(FM_ERR_ARG, "fm_signal_workspace_size: unknown precision %d", precision);
  return FM_ERR_ARG;
}

int fm_signal_enqueue(fm_ctx *ctx, const fm_signal_args *a, int precision, void *ws, size_t ws_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_signal(a, "fm_signal_enqueue"));
  DeviceGuard g(ctx->device);
  FM_REQUIRE(g.ok, FM_ERR_CUDA, "fm_signal_enqueue: cannot select device %d", ctx->device);
  switch (precision) {
    case FM_PREC_F32: return signal_plain<float>(ctx, a, ws, ws_bytes);
    case FM_PREC_F64: return signal_plain<double>(ctx, a, ws, ws_bytes);
    case FM_PREC_BF16X3: return signal_tc(ctx, a, ws, ws_bytes);
    default: break;
  }
  set_error(FM_ERR_ARG, "fm_signal_enqueue: unknown precision %d", precision);
  return FM_ERR_ARG;
}

int fm_signal_status(fm_ctx *ctx, const fm_signal_args *a, int precision, void *ws, size_t ws_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_signal(a, "fm_signal_status"));
  DeviceGuard g(ctx->device);
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  if (S == 0 || a->n_vencs == 0 || a->n_nodes == 0) {
    FM_CUDA(cudaStreamSynchronize(ctx->stream));
    return FM_OK;
  }
  switch (precision) {
    case FM_PREC_F32: return signal_plain_errors<float>(ctx, a, ws, ws_bytes);
    case FM_PREC_F64: return signal_plain_errors<double>(ctx, a, ws, ws_bytes);
    case FM_PREC_BF16X3: return signal_tc_errors(ctx, a, ws, ws_bytes);
    default: break;
  }
  set_error(FM_ERR_ARG, "fm_signal_status: unknown precision %d", precision);
  return FM_ERR_ARG;
}

int fm_signal(fm_ctx *ctx, const fm_signal_args *a, int precision, void *ws, size_t ws_bytes) {
  FM_TRY(fm_signal_enqueue(ctx, a, precision, ws, ws_bytes));
  return fm_signal_status(ctx, a, precision, ws, ws_bytes);
}

// One thread waits on an mbarrier that nothing arrives on; the bounded wait
// runs out and the kernel records where it gave up.
__global__ void selftest_wait_kernel(uint64_t limit_ns, int *status) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  ptx::mbar_init(&bar, 1);
  ptx::fence_mbar_init();
  const bool done = ptx::mbar_wait(&bar, 0, limit_ns);
  *status = done ? 0 : 1;
}

static int validate_batch(const fm_signal_args *probs, int n, const char *who) {
  FM_REQUIRE(n >= 0, FM_ERR_SHAPE, "%s: negative problem count", who);
  FM_REQUIRE(n == 0 || probs != nullptr, FM_ERR_ARG, "%s: null problem array", who);
  for (int i = 0; i < n; ++i) FM_TRY(validate_signal(&probs[i], who));
  return FM_OK;
}

int fm_signal_batch_workspace_size(const fm_signal_args *probs, int n, size_t *bytes) {
  FM_REQUIRE(bytes != nullptr, FM_ERR_ARG, "fm_signal_batch_workspace_size: null output");
  FM_TRY(validate_batch(probs, n, "fm_signal_batch_workspace_size"));
  *bytes = tc_batch_workspace_size(probs, n);
  return FM_OK;
}

int fm_signal_batch_enqueue(fm_ctx *ctx, const fm_signal_args *probs, int n, const fm_tc_tuning *tune, void *ws,
                            size_t ws_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_batch(probs, n, "fm_signal_batch_enqueue"));
  if (tune) {
    FM_REQUIRE(tune->split_nodes >= 0 && tune->kz_cap >= 0, FM_ERR_ARG,
               "fm_signal_batch_enqueue: negative tuning value");
  }
  DeviceGuard g(ctx->device);
  FM_REQUIRE(g.ok, FM_ERR_CUDA, "fm_signal_batch_enqueue: cannot select device %d", ctx->device);
  return signal_tc_batch(ctx, probs, n, tune, ws, ws_bytes);
}

int fm_signal_batch_status(fm_ctx *ctx, const fm_signal_args *probs, int n, void *ws, size_t ws_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_batch(probs, n, "fm_signal_batch_status"));
  DeviceGuard g(ctx->device);
  return signal_tc_batch_errors(ctx, probs, n, ws, ws_bytes);
}

int fm_selftest_wait(fm_ctx *ctx, uint64_t limit_ns) {
  FM_TRY(ctx_ok(ctx));
  FM_REQUIRE(limit_ns > 0 && limit_ns <= 2000000000ull, FM_ERR_ARG, "fm_selftest_wait: limit must be in (0, 2 s]");
  DeviceGuard g(ctx->device);
  FM_REQUIRE(g.ok, FM_ERR_CUDA, "fm_selftest_wait: cannot select device %d", ctx->device);
  int *d = nullptr;
  FM_CUDA(cudaMallocAsync(&d, sizeof(int), ctx->stream));
  FM_CUDA(cudaMemsetAsync(d, 0, sizeof(int), ctx->stream));
  selftest_wait_kernel<<<1, 32, 0, ctx->stream>>>(limit_ns, d);
  count_launch();
  int h = 0;
  FM_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  FM_CUDA(cudaFreeAsync(d, ctx->stream));
  FM_CUDA(cudaStreamSynchronize(ctx->stream));
  FM_TRY(check_launch("selftest_wait_kernel"));
  if (h != 0) {
    set_error(FM_ERR_TIMEOUT, "fm_selftest_wait: the device wait ran out after %llu ns (expected)",
              (unsigned long long)limit_ns);
    return FM_ERR_TIMEOUT;
  }
  return FM_OK;
}

int64_t fm_signal_count_time_runs(const void *t_host, int64_t n_samples, int is_double) {
  if (t_host == nullptr || n_samples <= 0) return 0;
  int64_t runs = 1;
  if (is_double) {
    const double *t = static_cast<const double *>(t_host);
    for (int64_t s = 1; s < n_samples; ++s) runs += (t[s] == t[s - 1]) ? 0 : 1;
  } else {
    const float *t = static_cast<const float *>(t_host);
    for (int64_t s = 1; s < n_samples; ++s) runs += (t[s] == t[s - 1]) ? 0 : 1;
  }
  return runs;
}

}  // extern "C"
