// Context lifecycle and error reporting of the C ABI.
#include <stdarg.h>
#include <string.h>

#include "common.cuh"

namespace fm {

static thread_local int t_code = FM_OK;
static thread_local char t_msg[1024] = {0};
std::atomic<int64_t> g_launches{0};

void set_error(int code, const char *fmt, ...) {
  t_code = code;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_msg, sizeof(t_msg), fmt, ap);
  va_end(ap);
}

int last_code() { return t_code; }

int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(FM_ERR_CUDA, "%s: kernel launch failed: %s", what, cudaGetErrorString(e));
    return FM_ERR_CUDA;
  }
  return FM_OK;
}

static cudaEvent_t pooled_event(fm_ctx *ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

int timer_start(fm_ctx *ctx, const char *name) {
  if (ctx == nullptr || !ctx->timing) return -1;
  fm_timed_launch t;
  t.name = name;
  t.start = pooled_event(ctx);
  t.stop = pooled_event(ctx);
  if (t.start == nullptr || t.stop == nullptr) return -1;
  cudaEventRecord(t.start, ctx->stream);
  ctx->timed.push_back(t);
  return (int)ctx->timed.size() - 1;
}

void timer_stop(fm_ctx *ctx, int slot) {
  if (ctx == nullptr || slot < 0 || slot >= (int)ctx->timed.size()) return;
  cudaEventRecord(ctx->timed[slot].stop, ctx->stream);
}

int ctx_side_streams(fm_ctx *ctx, int k) {
  if ((int)ctx->side.size() >= k) return FM_OK;
  DeviceGuard g(ctx->device);
  FM_REQUIRE(g.ok, FM_ERR_CUDA, "cudaSetDevice(%d) failed", ctx->device);
  if (ctx->side_ev.empty()) {
    cudaEvent_t e = nullptr;
    FM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->side_ev.push_back(e);  // the fork event
  }
  while ((int)ctx->side.size() < k) {
    cudaStream_t s = nullptr;
    FM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaStreamDestroy(s);
      set_error(FM_ERR_CUDA, "cudaEventCreateWithFlags failed");
      return FM_ERR_CUDA;
    }
    ctx->side.push_back(s);
    ctx->side_ev.push_back(e);  // its join event
  }
  return FM_OK;
}

int ctx_fork(fm_ctx *ctx, int k) {
  FM_CUDA(cudaEventRecord(ctx->side_ev[0], ctx->stream));
  for (int i = 0; i < k; ++i) FM_CUDA(cudaStreamWaitEvent(ctx->side[i], ctx->side_ev[0], 0));
  return FM_OK;
}

int ctx_join(fm_ctx *ctx, int k) {
  for (int i = 0; i < k; ++i) {
    FM_CUDA(cudaEventRecord(ctx->side_ev[1 + i], ctx->side[i]));
    FM_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->side_ev[1 + i], 0));
  }
  return FM_OK;
}

}  // namespace fm

extern "C" {

int fm_ctx_timing_enable(fm_ctx *ctx, int on) {
  FM_TRY(fm::ctx_ok(ctx));
  ctx->timing = (on != 0);
  return FM_OK;
}

int fm_ctx_timing_reset(fm_ctx *ctx) {
  FM_TRY(fm::ctx_ok(ctx));
  fm::DeviceGuard g(ctx->device);
  for (auto &t : ctx->timed) {
    ctx->event_pool.push_back(t.start);
    ctx->event_pool.push_back(t.stop);
  }
  ctx->timed.clear();
  return FM_OK;
}

int fm_ctx_timing_query(fm_ctx *ctx, const char *prefix, double *total_ms, int64_t *launches) {
  FM_TRY(fm::ctx_ok(ctx));
  FM_REQUIRE(total_ms != nullptr && launches != nullptr, FM_ERR_ARG, "fm_ctx_timing_query: null output");
  fm::DeviceGuard g(ctx->device);
  double sum = 0.0;
  int64_t n = 0;
  const size_t plen = prefix ? strlen(prefix) : 0;
  for (auto &t : ctx->timed) {
    if (plen && t.name.compare(0, plen, prefix) != 0) continue;
    FM_CUDA(cudaEventSynchronize(t.stop));
    float ms = 0.f;
    FM_CUDA(cudaEventElapsedTime(&ms, t.start, t.stop));
    sum += ms;
    ++n;
  }
  *total_ms = sum;
  *launches = n;
  return FM_OK;
}

int fm_abi_version(void) { return FM_ABI_VERSION; }

int64_t fm_launch_count(void) { return fm::g_launches.load(); }

int fm_last_error(char *buf, size_t len) {
  if (buf != nullptr && len > 0) {
    strncpy(buf, fm::t_msg, len - 1);
    buf[len - 1] = '\0';
  }
  return fm::t_code;
}

int fm_ctx_create(int device, fm_ctx **out) {
  FM_REQUIRE(out != nullptr, FM_ERR_ARG, "fm_ctx_create: null output pointer");
  int n = 0;
  FM_CUDA(cudaGetDeviceCount(&n));
  FM_REQUIRE(device >= 0 && device < n, FM_ERR_ARG, "fm_ctx_create: device %d out of range (%d devices)", device, n);
  fm::DeviceGuard g(device);
  FM_REQUIRE(g.ok, FM_ERR_CUDA, "fm_ctx_create: cudaSetDevice(%d) failed", device);
  cudaDeviceProp prop;
  FM_CUDA(cudaGetDeviceProperties(&prop, device));
  FM_REQUIRE(prop.major == 10, FM_ERR_UNSUPPORTED,
             "fm_ctx_create: device %d is sm_%d%d; this library is built for sm_100a only", device, prop.major,
             prop.minor);
  fm_ctx *c = new fm_ctx;
  c->device = device;
  c->stream = nullptr;
  c->num_sms = prop.multiProcessorCount;
  *out = c;
  return FM_OK;
}

int fm_ctx_destroy(fm_ctx *ctx) {
  FM_TRY(fm::ctx_ok(ctx));
  fm_ctx_timing_reset(ctx);
  for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
  {
    fm::DeviceGuard g(ctx->device);
    for (cudaEvent_t e : ctx->side_ev) cudaEventDestroy(e);
    for (cudaStream_t s : ctx->side) cudaStreamDestroy(s);
  }
  delete ctx;
  return FM_OK;
}

int fm_ctx_set_stream(fm_ctx *ctx, void *stream) {
  FM_TRY(fm::ctx_ok(ctx));
  ctx->stream = static_cast<cudaStream_t>(stream);
  return FM_OK;
}

int fm_ctx_synchronize(fm_ctx *ctx) {
  FM_TRY(fm::ctx_ok(ctx));
  fm::DeviceGuard g(ctx->device);
  FM_CUDA(cudaStreamSynchronize(ctx->stream));
  return FM_OK;
}

}  // extern "C"
