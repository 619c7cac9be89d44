// Plain CUDA-core forms of Signal (FP32 drop-in and FP64).
//
// Restates Signal<T> (cpp/feelmri/MRI.cpp:38-159 with motion, :196-298
// without): for every sample s of run g (time t_g)
//   K[s, v] = sum_n exp(i * (-2pi k_s . r_n(t_g) + phi_n t_g)) * MM[n, v] * exp(-t_g / T2_n)
// with MM = M * Mxy, 2pi built from a float-rounded pi (MRI.h:13, MRI.cpp:73),
// the phase summed in T as the reference does (MRI.cpp:138-146) and sin/cos
// taken of the phase in radians.  One thread block covers up to
// kPlainThreads * SPT samples of one run and sweeps a node range staged in
// shared memory; the per-run node quantities (moved position, phase offset,
// decayed weight) are formed once per block and node.  Node ranges may be
// split over blocks; partial sums are then added in a fixed order.
#include "signal_common.cuh"

namespace fm {

template <typename T>
struct V4;
template <>
struct V4<float> {
  using type = float4;
};
template <>
struct V4<double> {
  using type = double4;
};

template <typename T>
struct PlainDev {
  int64_t N, S, V;
  const T *kx, *ky, *kz;
  const T *r0, *phi, *T2;
  const T *MM;  // (N, V) complex interleaved
  MotionDev md;
  const float *weights;   // (n_runs, slots) TERMS motion weights
  const T *table;         // TABLE motion (n_runs, N, 3) in T
  const int *tile_run, *tile_s0, *run_start;
  const int *n_tiles;     // device: number of tiles
  const double *run_t;
  int64_t chunk;          // nodes per split
  int splits;
  T *out;                 // (S, V) complex or partials (splits, S, V)
  T two_pi;
};

template <typename T>
__device__ inline void sincos_t(T x, T *s, T *c);
template <>
__device__ inline void sincos_t<float>(float x, float *s, float *c) { sincosf(x, s, c); }
template <>
__device__ inline void sincos_t<double>(double x, double *s, double *c) { sincos(x, s, c); }

template <typename T>
__device__ inline T exp_t(T x);
template <>
__device__ inline float exp_t<float>(float x) { return expf(x); }
template <>
__device__ inline double exp_t<double>(double x) { return exp(x); }

template <typename T, int VMAX, int SPT, int NT>
__global__ void __launch_bounds__(kPlainThreads) signal_plain_kernel(PlainDev<T> p, int v0) {
  using T4 = typename V4<T>::type;
  __shared__ T4 s_pos[NT];             // moved x, y, z and phi * t
  __shared__ T s_w[NT][2 * VMAX];      // decayed M * Mxy columns v0 .. v0 + VMAX

  const int n_tiles = *p.n_tiles;
  const int split = blockIdx.y;
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
  __syncthreads();  // the previous tile's readers of s_pos / s_w are done
  const int g = p.tile_run[tile];
  const int s_begin = p.tile_s0[tile];
  const int s_end = min(p.run_start[g + 1], s_begin + kPlainThreads * SPT);
  const T tg = (T)p.run_t[g];
  const int nv = (int)min((int64_t)VMAX, p.V - v0);

  T kxs[SPT], kys[SPT], kzs[SPT];
  T acc_r[SPT][VMAX], acc_i[SPT][VMAX];
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    const int s = s_begin + q * kPlainThreads + threadIdx.x;
    const bool ok = s < s_end;
    // kx_ = two_pi * kloc[0](i,j,k)   (MRI.cpp:138-140)
    kxs[q] = ok ? p.two_pi * p.kx[s] : T(0);
    kys[q] = ok ? p.two_pi * p.ky[s] : T(0);
    kzs[q] = ok ? p.two_pi * p.kz[s] : T(0);
#pragma unroll
    for (int v = 0; v < VMAX; ++v) {
      acc_r[q][v] = T(0);
      acc_i[q][v] = T(0);
    }
  }

  const int64_t n_begin = (int64_t)split * p.chunk;
  const int64_t n_end = min(p.N, n_begin + p.chunk);
  const float *wrun = p.weights ? p.weights + (int64_t)g * p.md.slots : nullptr;
  for (int64_t nb = n_begin; nb < n_end; nb += NT) {
    const int cnt = (int)min((int64_t)NT, n_end - nb);
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += kPlainThreads) {
      const int64_t n = nb + j;
      T x = p.r0[3 * n + 0], y = p.r0[3 * n + 1], z = p.r0[3 * n + 2];
      if (p.md.kind == FM_MOTION_TERMS) {
        float dx, dy, dz;
        motion_disp(p.md, wrun, n, p.N, dx, dy, dz);
        x = x + (T)dx; y = y + (T)dy; z = z + (T)dz;
      } else if (p.table) {
        const T *d = p.table + ((int64_t)g * p.N + n) * 3;
        x = x + (T)d[0]; y = y + (T)d[1]; z = z + (T)d[2];
      }
      T4 pp;
      pp.x = x; pp.y = y; pp.z = z;
      pp.w = p.phi[n] * tg;                       // phi_off (MRI.cpp:124)
      s_pos[j] = pp;
      const T invT2 = T(1) / p.T2[n];
      const T decay = exp_t<T>(-tg * invT2);      // T2_decay (MRI.cpp:127)
      const T *mm = p.MM + (n * p.V + v0) * 2;
#pragma unroll
      for (int v = 0; v < VMAX; ++v) {
        s_w[j][2 * v + 0] = (v < nv) ? mm[2 * v + 0] * decay : T(0);
        s_w[j][2 * v + 1] = (v < nv) ? mm[2 * v + 1] * decay : T(0);
      }
    }
    __syncthreads();
    for (int j = 0; j < cnt; ++j) {
      const T4 pp = s_pos[j];
#pragma unroll
      for (int q = 0; q < SPT; ++q) {
        // phase = -kx_ x - ky_ y - kz_ z + phi_off   (MRI.cpp:143-146)
        const T ph = fma(-kzs[q], pp.z, fma(-kys[q], pp.y, -kxs[q] * pp.x)) + pp.w;
        T sn, cs;
        sincos_t<T>(ph, &sn, &cs);
#pragma unroll
        for (int v = 0; v < VMAX; ++v) {
          const T wr = s_w[j][2 * v + 0], wi = s_w[j][2 * v + 1];
          acc_r[q][v] = fma(cs, wr, fma(-sn, wi, acc_r[q][v]));
          acc_i[q][v] = fma(cs, wi, fma(sn, wr, acc_i[q][v]));
        }
      }
    }
  }

  T *dst = p.out + (int64_t)split * p.S * p.V * 2;
#pragma unroll
  for (int q = 0; q < SPT; ++q) {
    const int s = s_begin + q * kPlainThreads + threadIdx.x;
    if (s >= s_end) continue;
#pragma unroll
    for (int v = 0; v < VMAX; ++v) {
      if (v < nv) {
        dst[((int64_t)s * p.V + v0 + v) * 2 + 0] = acc_r[q][v];
        dst[((int64_t)s * p.V + v0 + v) * 2 + 1] = acc_i[q][v];
      }
    }
  }
  }  // tiles
}

// out[e] = sum over splits in order of partial[split][e].
template <typename T>
__global__ void split_reduce_kernel(const T *__restrict__ part, int splits, int64_t count, T *__restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  T acc = part[e];
  for (int k = 1; k < splits; ++k) acc += part[(int64_t)k * count + e];
  out[e] = acc;
}

template <typename T, int VMAX>
static void launch_plain(const PlainDev<T> &p, int64_t max_tiles, int v0, int spt, cudaStream_t st) {
  constexpr int NT = 128;
  const int64_t per_split = (4LL * kSmCount + p.splits - 1) / p.splits;
  dim3 grid((unsigned)(max_tiles < per_split ? max_tiles : per_split), (unsigned)p.splits);
  if (spt == 2) signal_plain_kernel<T, VMAX, 2, NT><<<grid, kPlainThreads, 0, st>>>(p, v0);
  else signal_plain_kernel<T, VMAX, 1, NT><<<grid, kPlainThreads, 0, st>>>(p, v0);
}

// Samples per thread: two for FP32 with few columns, else one.
template <typename T>
static int samples_per_thread(int64_t V) {
  return (sizeof(T) == 4 && V <= 4) ? 2 : 1;
}

// Split count: enough blocks to fill the GPU, bounded by the node count.
static int choose_splits(int64_t n_tiles_min, int64_t N) {
  const int64_t want = 4LL * kSmCount;
  int64_t s = (n_tiles_min >= want) ? 1 : ceil_div(want, n_tiles_min > 0 ? n_tiles_min : 1);
  s = s < 1 ? 1 : s;
  const int64_t by_nodes = ceil_div(N, 1024);
  if (s > by_nodes) s = by_nodes;
  if (s > 64) s = 64;
  return (int)(s < 1 ? 1 : s);
}

template <typename T>
struct PlainPlan {
  T *MM;
  Csr csr;
  Runs runs;
  float *weights;
  T *partials;
  int splits;
  int tile;
};

template <typename T>
static void carve_plain(Carve &c, const fm_signal_args *a, PlainPlan<T> &pl) {
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  const int64_t N = a->n_nodes, V = a->n_vencs;
  pl.tile = samples_per_thread<T>(V) * kPlainThreads;
  pl.MM = c.take<T>((size_t)N * V * 2);
  carve_csr(c, a->m_rows, a->m_nnz, pl.csr);
  carve_runs(c, S, pl.tile, pl.runs);
  pl.weights = c.take<float>((size_t)(S + 1) * motion_slots(a->motion));
  pl.splits = choose_splits(ceil_div(S, pl.tile), N);
  pl.partials = (pl.splits > 1) ? c.take<T>((size_t)pl.splits * S * V * 2) : nullptr;
}

int validate_signal(const fm_signal_args *a, const char *who);

template <typename T>
int signal_plain(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes) {
  const char *who = sizeof(T) == 4 ? "fm_signal(F32)" : "fm_signal(F64)";
  cudaStream_t st = ctx->stream;
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  const int64_t N = a->n_nodes, V = a->n_vencs;
  Carve cv(ws, ws_bytes);
  PlainPlan<T> pl;
  carve_plain<T>(cv, a, pl);
  FM_TRY(carve_ok(cv, who));
  if (S == 0 || V == 0) return FM_OK;
  T *out = static_cast<T *>(a->out);
  if (N == 0) {
    FM_CUDA(cudaMemsetAsync(out, 0, (size_t)S * V * 2 * sizeof(T), st));
    return FM_OK;
  }
  FM_TRY(build_runs<T>(static_cast<const T *>(a->t), S, pl.tile, pl.runs, st));
  FM_TRY(sparse_times_dense<T>(a, pl.csr, static_cast<const T *>(a->Mxy), pl.MM, pl.runs.error, st));
  FM_TRY(check_table_calls(a->motion, pl.runs, st));
  const MotionDev md = make_motion_dev(a->motion);
  FM_TRY(launch_run_weights(md, pl.runs.run_t, pl.runs.counts, S, pl.weights, st));
  const int64_t max_tiles = max_tiles_for(S, pl.tile);

  PlainDev<T> p{};
  p.N = N; p.S = S; p.V = V;
  p.kx = static_cast<const T *>(a->kx);
  p.ky = static_cast<const T *>(a->ky);
  p.kz = static_cast<const T *>(a->kz);
  p.r0 = static_cast<const T *>(a->r0);
  p.phi = static_cast<const T *>(a->phi);
  p.T2 = static_cast<const T *>(a->T2);
  p.MM = pl.MM;
  p.md = md;
  p.weights = (md.kind == FM_MOTION_TERMS) ? pl.weights : nullptr;
  p.table = (a->motion && a->motion->kind == FM_MOTION_TABLE) ? static_cast<const T *>(a->motion->table) : nullptr;
  p.n_tiles = pl.runs.counts + 1;
  p.tile_run = pl.runs.tile_run;
  p.tile_s0 = pl.runs.tile_s0;
  p.run_start = pl.runs.start;
  p.run_t = pl.runs.run_t;
  p.splits = pl.splits;
  p.chunk = ceil_div(N, pl.splits);
  p.out = (pl.splits > 1) ? pl.partials : out;
  // two_pi = 2.0 * PI with PI = (float)M_PI   (MRI.h:13, MRI.cpp:73)
  const float pi_f = 3.14159265358979323846f;
  p.two_pi = (T)2.0 * (T)pi_f;

  const int spt = samples_per_thread<T>(V);
  ScopedTimer timer(ctx, sizeof(T) == 4 ? "signal_f32" : "signal_f64");
  for (int v0 = 0; v0 < V; v0 += 8) {
    const int64_t nv = V - v0;
    if (nv <= 1) launch_plain<T, 1>(p, max_tiles, v0, spt, st);
    else if (nv <= 2) launch_plain<T, 2>(p, max_tiles, v0, spt, st);
    else if (nv <= 4) launch_plain<T, 4>(p, max_tiles, v0, spt, st);
    else launch_plain<T, 8>(p, max_tiles, v0, spt, st);
    count_launch();
    FM_TRY(check_launch("signal_plain_kernel"));
  }
  if (pl.splits > 1) {
    const int64_t count = S * V * 2;
    split_reduce_kernel<T><<<(unsigned)ceil_div(count, 256), 256, 0, st>>>(pl.partials, pl.splits, count, out);
    count_launch();
    FM_TRY(check_launch("split_reduce_kernel"));
  }
  return FM_OK;
}

template <typename T>
int signal_plain_errors(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes) {
  Carve cv(ws, ws_bytes);
  PlainPlan<T> pl;
  carve_plain<T>(cv, a, pl);
  FM_TRY(carve_ok(cv, "fm_signal"));
  return report_errors(pl.runs, ctx->stream, sizeof(T) == 4 ? "fm_signal(F32)" : "fm_signal(F64)");
}
template int signal_plain_errors<float>(fm_ctx *, const fm_signal_args *, void *, size_t);
template int signal_plain_errors<double>(fm_ctx *, const fm_signal_args *, void *, size_t);

template int signal_plain<float>(fm_ctx *, const fm_signal_args *, void *, size_t);
template int signal_plain<double>(fm_ctx *, const fm_signal_args *, void *, size_t);

template <typename T>
size_t plain_workspace(const fm_signal_args *a) {
  Carve c(nullptr, 0);
  PlainPlan<T> pl;
  carve_plain<T>(c, a, pl);
  return c.used;
}
template size_t plain_workspace<float>(const fm_signal_args *);
template size_t plain_workspace<double>(const fm_signal_args *);

}  // namespace fm
