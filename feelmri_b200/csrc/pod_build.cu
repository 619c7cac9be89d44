// Snapshot products of the POD construction, POD.calculate_pod
// (python/feelmri/Motion.py:174-211): with X the (rows x t) snapshot matrix
// (data.reshape(-1, t), rows = P * C),
//   gram    = X^T X                      (t x t)          Motion.py:189
//   phi     = X E                        (rows x r)       Motion.py:202
//   weights = X^T phi                    (t x r)          Motion.py:204
// where E (t x r) holds the leading eigenvectors of gram scaled by
// 1/sqrt(eigenvalue).  The t x t eigenproblem itself stays on the host
// (numpy.linalg.eigh, as the reference computes it).
//
// The reference evaluates these in the data's type with BLAS.  Here every sum
// is accumulated in FP64 in a fixed order (per block over its rows, then over
// the blocks in block order), so results are reproducible run to run and at
// least as accurate; phi is rounded to the data's type before it enters the
// weights, as the reference's phi array is.
#include <algorithm>

#include "common.cuh"

namespace fm {

constexpr int kPodThreads = 256;
constexpr int kSmCountPod = 148;   // SMs of a B200: sizes the block count without a device query
constexpr int kPodTileRows = 32;    // rows staged per shared-memory tile
constexpr int kPodPerThread = 16;   // output elements a thread accumulates at once

// partials[b][e] = sum over block b's rows of A[row, e / nb] * B[row, e % nb]
// for e in [0, na * nb).  A and B are row-major with leading dimensions na, nb.
template <typename TA, typename TB>
__global__ void __launch_bounds__(kPodThreads) pod_cross_partial_kernel(const TA *__restrict__ A, int na,
                                                                      const TB *__restrict__ B, int nb,
                                                                      int64_t rows, int64_t rows_per_block,
                                                                      double *__restrict__ partials) {
  extern __shared__ double sm[];
  double *ta = sm;                          // [kPodTileRows][na]
  double *tb = sm + kPodTileRows * na;      // [kPodTileRows][nb]
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
  const int64_t r1 = (rows < r0 + rows_per_block) ? rows : r0 + rows_per_block;
  const int n_el = na * nb;
  double *out = partials + (int64_t)blockIdx.x * n_el;
  for (int e0 = 0; e0 < n_el; e0 += kPodThreads * kPodPerThread) {
    double acc[kPodPerThread];
#pragma unroll
    for (int q = 0; q < kPodPerThread; ++q) acc[q] = 0.0;
    for (int64_t rt = r0; rt < r1; rt += kPodTileRows) {
      const int nr = (r1 - rt < (int64_t)kPodTileRows) ? (int)(r1 - rt) : kPodTileRows;
      __syncthreads();
      for (int i = threadIdx.x; i < nr * na; i += kPodThreads) ta[i] = (double)A[rt * na + i];
      for (int i = threadIdx.x; i < nr * nb; i += kPodThreads) tb[i] = (double)B[rt * nb + i];
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kPodPerThread; ++q) {
        const int e = e0 + q * kPodThreads + threadIdx.x;
        if (e < n_el) {
          const int a = e / nb, b = e - (e / nb) * nb;
          double s = acc[q];
          for (int r = 0; r < nr; ++r) s = fma(ta[r * na + a], tb[r * nb + b], s);
          acc[q] = s;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kPodPerThread; ++q) {
      const int e = e0 + q * kPodThreads + threadIdx.x;
      if (e < n_el) out[e] = acc[q];
    }
  }
}

// out[e] = sum over b of partials[b][e], in block order.
__global__ void pod_reduce_kernel(const double *__restrict__ partials, int n_parts, int n_el,
                                  double *__restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_el) return;
  double s = 0.0;
  for (int b = 0; b < n_parts; ++b) s += partials[(int64_t)b * n_el + e];
  out[e] = s;
}

// phi[row, m] = T(sum_k X[row, k] E[k, m]), k ascending, FP64 accumulation.
template <typename T>
__global__ void pod_project_kernel(const T *__restrict__ X, int64_t rows, int t, const double *__restrict__ E, int r,
                                   T *__restrict__ phi) {
  extern __shared__ double se[];  // E, t x r
  for (int i = threadIdx.x; i < t * r; i += blockDim.x) se[i] = E[i];
  __syncthreads();
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < rows;
       row += (int64_t)gridDim.x * blockDim.x) {
    const T *x = X + row * t;
    for (int m0 = 0; m0 < r; m0 += 8) {
      double acc[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[q] = 0.0;
      for (int k = 0; k < t; ++k) {
        const double xv = (double)x[k];
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (m0 + q < r) acc[q] = fma(xv, se[k * r + m0 + q], acc[q]);
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (m0 + q < r) phi[row * r + m0 + q] = (T)acc[q];
    }
  }
}

static int pod_blocks(int64_t rows) {
  const int64_t want = ceil_div(rows, (int64_t)4 * kPodTileRows);
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, 4 * kSmCountPod));
}

static int validate_pod(const void *X, int64_t rows, int t, int r, const char *who) {
  FM_REQUIRE(rows >= 0 && t >= 1 && t <= 1024, FM_ERR_SHAPE, "%s: rows=%lld, t=%d (1 <= t <= 1024)", who,
             (long long)rows, t);
  FM_REQUIRE(r >= 0 && r <= t, FM_ERR_SHAPE, "%s: %d modes for %d snapshots", who, r, t);
  FM_REQUIRE(rows == 0 || X != nullptr, FM_ERR_ARG, "%s: null snapshot matrix", who);
  return FM_OK;
}

static size_t pod_ws_bytes(int64_t rows, int t, int r) {
  const int nb = pod_blocks(rows);
  const int64_t el = std::max<int64_t>((int64_t)t * t, (int64_t)t * r);
  return (size_t)nb * el * sizeof(double) + 256;
}

template <typename T>
static int cross_products(fm_ctx *ctx, const T *A, int na, const T *B, int nb_cols, int64_t rows, double *out,
                          void *ws, size_t ws_bytes, const char *who) {
  const int nb = pod_blocks(rows);
  const int n_el = na * nb_cols;
  Carve cv(ws, ws_bytes);
  double *partials = cv.take<double>((size_t)nb * n_el);
  FM_TRY(carve_ok(cv, who));
  const int64_t per = ceil_div(rows, (int64_t)nb);
  const size_t smem = sizeof(double) * kPodTileRows * (size_t)(na + nb_cols);
  FM_REQUIRE(smem <= 200 * 1024, FM_ERR_SHAPE, "%s: %d + %d columns do not fit a shared-memory tile", who, na,
             nb_cols);
  auto kern = pod_cross_partial_kernel<T, T>;
  if (smem > 48 * 1024) FM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<nb, kPodThreads, smem, ctx->stream>>>(A, na, B, nb_cols, rows, per, partials);
  count_launch();
  FM_TRY(check_launch("pod_cross_partial_kernel"));
  pod_reduce_kernel<<<(unsigned)ceil_div(n_el, 256), 256, 0, ctx->stream>>>(partials, nb, n_el, out);
  count_launch();
  return check_launch("pod_reduce_kernel");
}

template <typename T>
static int pod_gram_impl(fm_ctx *ctx, const T *X, int64_t rows, int t, double *gram, void *ws, size_t ws_bytes,
                         const char *who) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_pod(X, rows, t, 0, who));
  FM_REQUIRE(gram != nullptr, FM_ERR_ARG, "%s: null output", who);
  DeviceGuard g(ctx->device);
  if (rows == 0) {
    FM_CUDA(cudaMemsetAsync(gram, 0, sizeof(double) * t * t, ctx->stream));
    return FM_OK;
  }
  return cross_products<T>(ctx, X, t, X, t, rows, gram, ws, ws_bytes, who);
}

template <typename T>
static int pod_project_impl(fm_ctx *ctx, const T *X, int64_t rows, int t, const double *E, int r, T *phi,
                            double *weights, void *ws, size_t ws_bytes, const char *who) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_pod(X, rows, t, r, who));
  FM_REQUIRE(r >= 1 && E != nullptr && phi != nullptr && weights != nullptr, FM_ERR_ARG, "%s: null argument",
             who);
  DeviceGuard g(ctx->device);
  if (rows == 0) {
    FM_CUDA(cudaMemsetAsync(weights, 0, sizeof(double) * t * r, ctx->stream));
    return FM_OK;
  }
  const size_t smem = sizeof(double) * (size_t)t * r;
  FM_REQUIRE(smem <= 200 * 1024, FM_ERR_SHAPE, "%s: E (%d x %d) does not fit shared memory", who, t, r);
  auto kern = pod_project_kernel<T>;
  if (smem > 48 * 1024) FM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(rows, (int64_t)256), 8 * kSmCountPod));
  kern<<<blocks, 256, smem, ctx->stream>>>(X, rows, t, E, r, phi);
  count_launch();
  FM_TRY(check_launch("pod_project_kernel"));
  // weights = X^T phi (t x r), phi as rounded to the data's type
  return cross_products<T>(ctx, X, t, phi, r, rows, weights, ws, ws_bytes, who);
}

}  // namespace fm

using namespace fm;

extern "C" {

int fm_pod_build_workspace_size(int64_t rows, int32_t t, int32_t n_modes, size_t *bytes) {
  FM_REQUIRE(bytes != nullptr, FM_ERR_ARG, "fm_pod_build_workspace_size: null output");
  FM_TRY(validate_pod(reinterpret_cast<const void *>(1), rows, t, n_modes, "fm_pod_build_workspace_size"));
  *bytes = pod_ws_bytes(rows, t, n_modes);
  return FM_OK;
}

int fm_pod_gram_f32(fm_ctx *ctx, const float *X, int64_t rows, int32_t t, double *gram, void *ws, size_t ws_bytes) {
  return pod_gram_impl<float>(ctx, X, rows, t, gram, ws, ws_bytes, "fm_pod_gram_f32");
}

int fm_pod_gram_f64(fm_ctx *ctx, const double *X, int64_t rows, int32_t t, double *gram, void *ws,
                    size_t ws_bytes) {
  return pod_gram_impl<double>(ctx, X, rows, t, gram, ws, ws_bytes, "fm_pod_gram_f64");
}

int fm_pod_project_f32(fm_ctx *ctx, const float *X, int64_t rows, int32_t t, const double *E, int32_t n_modes,
                       float *phi, double *weights, void *ws, size_t ws_bytes) {
  return pod_project_impl<float>(ctx, X, rows, t, E, n_modes, phi, weights, ws, ws_bytes, "fm_pod_project_f32");
}

int fm_pod_project_f64(fm_ctx *ctx, const double *X, int64_t rows, int32_t t, const double *E, int32_t n_modes,
                       double *phi, double *weights, void *ws, size_t ws_bytes) {
  return pod_project_impl<double>(ctx, X, rows, t, E, n_modes, phi, weights, ws, ws_bytes, "fm_pod_project_f64");
}

}  // extern "C"
