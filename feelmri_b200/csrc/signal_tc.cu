// Split-BF16 tcgen05 tensor-core form of Signal.
//
// Same result as Signal<float> (cpp/feelmri/MRI.cpp:38-159 / :196-298): for
// each sample s of run g (time t_g, node positions r_n = r0_n + d_n(t_g))
//   K[s, v] = sum_n exp(-2 pi i k_s . r_n) * W_g[n, v],
//   W_g[n, v] = (M * Mxy)[n, v] * exp(-t_g / T2_n) * exp(i phi_n t_g),
// computed as a dense complex GEMM on the 5th-generation tensor cores:
//
// * Factoring.  A run whose samples form one complete Cartesian (line, kz)
//   slab with k(j, k) == kp_j + kq_k exactly (checked in FP64) is written as
//   C[p, (q, v)] = sum_n A[p, n] B[n, (q, v)] with A = exp(-2 pi i kp . r) and
//   B = exp(-2 pi i kq . r) W: P = lines rows, Q = kz values times V columns.
//   Every other run uses P = its samples and Q = 1 (B = W).
// * Real stacking.  Node n contributes two K entries: A'[p][2n..2n+1] =
//   (Re A, Im A) and B'^T[(q,v,re)][2n..] = (Re B, -Im B),
//   B'^T[(q,v,im)][2n..] = (Im B, Re B), so C'[p][2(q,v)+{0,1}] = (Re, Im).
// * Split BF16.  Each operand x is stored as hi = bf16(x), lo = bf16(x - hi);
//   hi*hi + hi*lo + lo*hi accumulate in FP32 in tensor memory.
// * Phases.  k . r is evaluated in FP64 and reduced modulo one cycle before
//   the FP32 sin/cos, so far nodes at high k keep their digits.
//
// Block: warps 0-3 produce operand tiles (16 nodes per pipeline stage, 4
// stages of shared memory in the UMMA no-swizzle K-major layout) and run the
// epilogue; warp 4 owns the tensor memory and one of its threads issues the
// MMAs.  Stages are handed over with mbarriers; tcgen05.commit frees a stage
// when the MMAs that read it have completed.  All waits are bounded: on
// timeout the block records an error, drains and frees its tensor memory.
#include <cuda_bf16.h>
#include <cub/cub.cuh>

#include "signal_common.cuh"
#include "tc_ptx.cuh"

namespace fm {

constexpr int kTcRows = 128;        // UMMA M
constexpr int kTcNodes = 16;        // nodes per stage -> K = 32 (two UMMA K steps)
constexpr int kTcStages = 4;
constexpr int kTcBlockNodes = 128;  // nodes whose per-run data is formed together
constexpr int kTcProducers = 128;
constexpr int kTcThreads = 160;
constexpr int kTcVGroup = 16;       // Mxy columns per launch
constexpr uint64_t kTcWaitNs = 2000000000ull;
constexpr uint32_t kAStageBytes = kTcRows * 2 * kTcNodes * 2;  // 128 rows x 32 K x bf16 = 8 KB

struct TcRun {
  int start, P, Q, factored;
};
struct TcItem {
  int run, p0, q0;
};

struct TcDev {
  int64_t N, S, V;
  int v0, VG;
  int n_lines, n_kz;
  const float *kx, *ky, *kz;
  const float *r0, *phi, *T2;
  const float2 *MM;
  MotionDev md;
  const float *weights;
  const float *table;
  const double *run_t;
  const TcRun *runs;
  const TcItem *items;
  int item0;
  int Qt, NT, tmem_cols;
  int splits;
  int64_t chunk;
  float2 *out;
  int *error;
};

struct TcSmem {
  uint32_t stage_bytes, a_hi, a_lo, b_hi, b_lo;  // offsets inside a stage
  uint32_t pos, w, etab, kq, bars, misc, total;
};

__host__ __device__ inline TcSmem tc_smem_layout(int NT, int VG, int Qt) {
  TcSmem L;
  L.a_hi = 0;
  L.a_lo = kAStageBytes;
  L.b_hi = 2 * kAStageBytes;
  L.b_lo = 2 * kAStageBytes + NT * 2 * kTcNodes * 2;
  L.stage_bytes = 2 * kAStageBytes + 2 * NT * 2 * kTcNodes * 2;
  uint32_t off = kTcStages * L.stage_bytes;
  L.pos = off;
  off += kTcBlockNodes * 16;
  L.w = off;
  off += kTcBlockNodes * VG * 8;
  L.etab = off;
  off += Qt * kTcNodes * 8;
  L.kq = off;
  off += ((Qt * 24 + 15) / 16) * 16;
  L.bars = off;
  off += 16 * 8;
  L.misc = off;
  off += 16;
  L.total = off;
  return L;
}

// Byte offset of element (row, k) of a K-major, no-swizzle operand tile with
// `rows` rows and 32 K elements: two K steps of 16, each made of 8-row x
// 16-byte core matrices (LBO = 128 between K halves, SBO = 256 between row
// groups).
__device__ inline uint32_t kmajor_offset(uint32_t row, uint32_t k, uint32_t rows) {
  return (k >> 4) * (rows * 32) + (row >> 3) * 256 + ((k >> 3) & 1) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ inline uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}

// hi/lo split of 8 consecutive K values written as one 16-byte chunk each.
__device__ inline void store_split8(uint32_t hi_addr, uint32_t lo_addr, const float (&x)[8]) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
    const float2 hf = __bfloat1622float2(hb);
    h[i] = *reinterpret_cast<uint32_t *>(&hb);
    l[i] = pack_bf16(x[2 * i] - hf.x, x[2 * i + 1] - hf.y);
  }
  ptx::st_shared_v4(hi_addr, h[0], h[1], h[2], h[3]);
  ptx::st_shared_v4(lo_addr, l[0], l[1], l[2], l[3]);
}

// exp(-2 pi i c) for c in cycles given in FP64: reduce modulo one, then FP32.
__device__ inline float2 cis_neg_cycles(double c) {
  const double f = c - rint(c);
  float s, co;
  __sincosf(6.283185307179586f * (float)f, &s, &co);
  return make_float2(co, -s);
}

__device__ inline bool producers_any(bool x) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, 1, 128, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)x)
      : "memory");
  return out != 0;
}

__global__ void __launch_bounds__(kTcThreads, 1) signal_tc_kernel(TcDev p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const TcSmem L = tc_smem_layout(p.NT, p.VG, p.Qt);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L.bars);
  uint64_t *empty = full + kTcStages;
  uint64_t *accum = empty + kTcStages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L.misc);
  float4 *pos = reinterpret_cast<float4 *>(smem + L.pos);
  float2 *wblk = reinterpret_cast<float2 *>(smem + L.w);
  float2 *etab = reinterpret_cast<float2 *>(smem + L.etab);
  double *kq = reinterpret_cast<double *>(smem + L.kq);
  const uint32_t sbase = ptx::smem_addr(smem);

  const TcItem it = p.items[p.item0 + blockIdx.x];
  const TcRun run = p.runs[it.run];
  const int split = blockIdx.y;
  const int P_tile = min(kTcRows, run.P - it.p0);
  const int Q_tile = min(p.Qt, run.Q - it.q0);
  const int64_t n_begin = (int64_t)split * p.chunk;
  const int64_t n_end = min(p.N, n_begin + p.chunk);
  const int n_stages = n_end > n_begin ? (int)ceil_div(n_end - n_begin, kTcNodes) : 0;
  const double tg_d = p.run_t[it.run];
  const float tg = (float)tg_d;

  // ---- set-up: zero operand ring, barriers, tensor memory, k vectors ----
  for (uint32_t o = tid * 16; o < kTcStages * L.stage_bytes; o += kTcThreads * 16)
    ptx::st_shared_v4(sbase + o, 0u, 0u, 0u, 0u);
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      ptx::mbar_init(&full[s], kTcProducers);
      ptx::mbar_init(&empty[s], 1);
    }
    ptx::mbar_init(accum, 1);
    tmem_slot[1] = 0;  // abort flag of the MMA thread
    ptx::fence_mbar_init();
  }
  if (warp == 4) ptx::tmem_alloc(tmem_slot, p.tmem_cols);
  // kq_q = k(start + q) - k(start) for the columns of this tile (factored)
  for (int q = tid; q < Q_tile; q += kTcThreads) {
    const int s_q = run.start + it.q0 + q, s_0 = run.start;
    kq[3 * q + 0] = run.factored ? (double)p.kx[s_q] - (double)p.kx[s_0] : 0.0;
    kq[3 * q + 1] = run.factored ? (double)p.ky[s_q] - (double)p.ky[s_0] : 0.0;
    kq[3 * q + 2] = run.factored ? (double)p.kz[s_q] - (double)p.kz[s_0] : 0.0;
  }
  ptx::fence_proxy_async_smem();
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = tmem_slot[0];
  const uint32_t idesc = ptx::idesc_bf16_f32(kTcRows, p.NT);
  bool ok = true;

  if (warp < 4) {
    // ------------------------------------------------------ producers --
    const int prow = tid;  // A row handled by this thread
    double kpx = 0, kpy = 0, kpz = 0;
    const bool a_active = prow < P_tile;
    if (a_active) {
      const int s_p = run.start + (run.factored ? (it.p0 + prow) * p.n_kz : it.p0 + prow);
      kpx = p.kx[s_p];
      kpy = p.ky[s_p];
      kpz = p.kz[s_p];
    }
    const int bj = tid;  // (q, v) pair handled by this thread for B
    const bool b_active = bj < Q_tile * p.VG;
    const int bq = b_active ? bj / p.VG : 0, bv = b_active ? bj % p.VG : 0;
    const float *wrun = p.weights ? p.weights + (int64_t)it.run * p.md.slots : nullptr;

    for (int st = 0; st < n_stages; ++st) {
      const int s = st % kTcStages;
      const uint32_t round = st / kTcStages;
      const int j = st % (kTcBlockNodes / kTcNodes);
      if (j == 0) {
        // per-run node data for the next 128 nodes
        ptx::named_barrier(1, kTcProducers);
        const int64_t n = n_begin + (int64_t)st * kTcNodes + tid;
        float4 pp = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 wv[kTcVGroup];
#pragma unroll
        for (int v = 0; v < kTcVGroup; ++v) wv[v] = make_float2(0.f, 0.f);
        if (n < n_end) {
          float x = p.r0[3 * n + 0], y = p.r0[3 * n + 1], z = p.r0[3 * n + 2];
          if (p.md.kind == FM_MOTION_TERMS) {
            float dx, dy, dz;
            motion_disp(p.md, wrun, n, p.N, dx, dy, dz);
            x = x + dx; y = y + dy; z = z + dz;
          } else if (p.table) {
            const float *d = p.table + ((int64_t)it.run * p.N + n) * 3;
            x = x + d[0]; y = y + d[1]; z = z + d[2];
          }
          pp = make_float4(x, y, z, 1.f);
          const float decay = expf(-tg * (1.0f / p.T2[n]));
          float so, co;
          sincosf(p.phi[n] * tg, &so, &co);
          const float er = decay * co, ei = decay * so;
          for (int v = 0; v < p.VG; ++v) {
            const float2 m = p.MM[n * p.V + p.v0 + v];
            wv[v] = make_float2(m.x * er - m.y * ei, m.x * ei + m.y * er);
          }
        }
        pos[tid] = pp;
        for (int v = 0; v < p.VG; ++v) wblk[tid * p.VG + v] = wv[v];
        ptx::named_barrier(1, kTcProducers);
      }
      // wait until the MMAs that last read stage s are done
      const bool waited = ptx::mbar_wait(&empty[s], (round & 1) ^ 1, kTcWaitNs);
      if (producers_any(!waited)) {
        ok = false;
        break;
      }
      const float4 *pn = pos + j * kTcNodes;
      const float2 *wn = wblk + j * kTcNodes * p.VG;
      // e_q(n) = exp(-2 pi i kq_q . r_n) for this stage's nodes
      for (int idx = tid; idx < Q_tile * kTcNodes; idx += kTcProducers) {
        const int q = idx / kTcNodes, n = idx % kTcNodes;
        const float4 r = pn[n];
        float2 e = make_float2(1.f, 0.f);
        if (run.factored) {
          const double c = kq[3 * q] * (double)r.x + kq[3 * q + 1] * (double)r.y + kq[3 * q + 2] * (double)r.z;
          e = cis_neg_cycles(c);
        }
        etab[idx] = e;
      }
      ptx::named_barrier(1, kTcProducers);
      const uint32_t stage = sbase + s * L.stage_bytes;
      if (a_active) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {  // 4 chunks of 4 nodes (8 K values)
          float x[8];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float4 r = pn[4 * h + u];
            const double c = kpx * (double)r.x + kpy * (double)r.y + kpz * (double)r.z;
            float2 e = cis_neg_cycles(c);
            if (r.w == 0.f) e = make_float2(0.f, 0.f);
            x[2 * u] = e.x;
            x[2 * u + 1] = e.y;
          }
          const uint32_t off = kmajor_offset(prow, 8 * h, kTcRows);
          store_split8(stage + L.a_hi + off, stage + L.a_lo + off, x);
        }
      }
      if (b_active) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          float xr[8], xi[8];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int n = 4 * h + u;
            const float2 e = etab[bq * kTcNodes + n];
            const float2 w = wn[n * p.VG + bv];
            const float br = e.x * w.x - e.y * w.y, bi = e.x * w.y + e.y * w.x;
            xr[2 * u] = br;
            xr[2 * u + 1] = -bi;
            xi[2 * u] = bi;
            xi[2 * u + 1] = br;
          }
          const uint32_t o_re = kmajor_offset(2 * bj, 8 * h, p.NT);
          const uint32_t o_im = kmajor_offset(2 * bj + 1, 8 * h, p.NT);
          store_split8(stage + L.b_hi + o_re, stage + L.b_lo + o_re, xr);
          store_split8(stage + L.b_hi + o_im, stage + L.b_lo + o_im, xi);
        }
      }
      ptx::fence_proxy_async_smem();
      ptx::mbar_arrive(&full[s]);
    }
  } else if (tid == 4 * 32) {
    // ------------------------------------------------------ MMA issue --
    for (int st = 0; st < n_stages; ++st) {
      const int s = st % kTcStages;
      const uint32_t round = st / kTcStages;
      if (!ptx::mbar_wait(&full[s], round & 1, kTcWaitNs)) {
        ok = false;
        break;
      }
      ptx::tc_fence_after();
      const uint32_t stage = sbase + s * L.stage_bytes;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const uint64_t ah = ptx::smem_desc(stage + L.a_hi + ks * kTcRows * 32, 128, 256);
        const uint64_t al = ptx::smem_desc(stage + L.a_lo + ks * kTcRows * 32, 128, 256);
        const uint64_t bh = ptx::smem_desc(stage + L.b_hi + ks * p.NT * 32, 128, 256);
        const uint64_t bl = ptx::smem_desc(stage + L.b_lo + ks * p.NT * 32, 128, 256);
        ptx::mma_bf16(tmem, ah, bh, idesc, (st > 0 || ks > 0) ? 1u : 0u);
        ptx::mma_bf16(tmem, ah, bl, idesc, 1u);
        ptx::mma_bf16(tmem, al, bh, idesc, 1u);
      }
      ptx::mma_commit(&empty[s]);
    }
    ptx::mma_commit(accum);
    if (!ok) tmem_slot[1] = 1;
  }

  // ---------------------------------------------------------- epilogue --
  if (warp < 4) {
    const bool done = ptx::mbar_wait(accum, 0, kTcWaitNs);
    ptx::tc_fence_after();
    if (!done || !ok) atomicExch(p.error, 1);
    const int prow = warp * 32 + (tid & 31);
    float2 *dst = p.out + (int64_t)split * p.S * p.V;
    const bool row_ok = prow < P_tile;
    const int s_row = run.start + (run.factored ? (it.p0 + prow) * p.n_kz + it.q0 : it.p0 + prow);
    for (int c0 = 0; c0 < p.NT; c0 += 16) {
      uint32_t r[16];
      if (n_stages > 0 && done) {
        ptx::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
        ptx::tmem_wait_ld();
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) r[i] = 0u;
      }
      if (!row_ok) continue;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int jj = (c0 >> 1) + i;
        const int q = jj / p.VG, v = jj % p.VG;
        if (q < Q_tile) {
          dst[(int64_t)(s_row + q) * p.V + p.v0 + v] = make_float2(__uint_as_float(r[2 * i]),
                                                                   __uint_as_float(r[2 * i + 1]));
        }
      }
    }
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 4) {
    ptx::tc_fence_after();
    if (tid == 4 * 32 && tmem_slot[1]) atomicExch(p.error, 2);
    ptx::tmem_dealloc(tmem, p.tmem_cols);
  }
}

// ---- run classification and work items ---------------------------------

// One block per run: a run is factored when it covers exactly one
// (lines x kz) slab and every sample satisfies k = kp_j + kq_k in FP64.
__global__ void tc_classify_kernel(const float *__restrict__ kx, const float *__restrict__ ky,
                                   const float *__restrict__ kz, const int *__restrict__ start,
                                   const int *__restrict__ counts, int n_lines, int n_kz, TcRun *__restrict__ runs) {
  const int g = blockIdx.x;
  if (g >= counts[0]) return;
  const int s0 = start[g], len = start[g + 1] - s0;
  const int Ls = n_lines * n_kz;
  __shared__ int sep;
  if (threadIdx.x == 0) sep = (len == Ls && Ls > 1 && n_kz > 1 && s0 % Ls == 0) ? 1 : 0;
  __syncthreads();
  if (sep) {
    const double b0[3] = {kx[s0], ky[s0], kz[s0]};
    for (int idx = threadIdx.x; idx < Ls; idx += blockDim.x) {
      const int jl = idx / n_kz, kk = idx % n_kz;
      const int s = s0 + idx, sj = s0 + jl * n_kz, sk = s0 + kk;
      const double a[3] = {kx[s], ky[s], kz[s]};
      const double pj[3] = {kx[sj], ky[sj], kz[sj]};
      const double qk[3] = {kx[sk], ky[sk], kz[sk]};
      bool good = true;
      for (int c = 0; c < 3; ++c) good = good && (a[c] == pj[c] + (qk[c] - b0[c]));
      if (!good) atomicExch(&sep, 0);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    TcRun r;
    r.start = s0;
    r.factored = sep;
    r.P = sep ? n_lines : len;
    r.Q = sep ? n_kz : 1;
    runs[g] = r;
  }
}

// Item counts per run, factored runs in one list and the rest in another.
__global__ void tc_count_kernel(const TcRun *__restrict__ runs, const int *__restrict__ counts, int Qt,
                                int *__restrict__ nf, int *__restrict__ ng) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = counts[0];
  if (g > n) return;
  if (g == n) {
    nf[g] = 0;
    ng[g] = 0;
    return;
  }
  const TcRun r = runs[g];
  const int items = (int)(ceil_div(r.P, kTcRows) * ceil_div(r.Q, r.factored ? Qt : 1));
  nf[g] = r.factored ? items : 0;
  ng[g] = r.factored ? 0 : items;
}

__global__ void tc_fill_kernel(const TcRun *__restrict__ runs, int *__restrict__ counts, int Qt,
                               const int *__restrict__ of, const int *__restrict__ og, TcItem *__restrict__ items) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = counts[0];
  if (g > n) return;
  if (g == n) {
    counts[2] = of[n];
    counts[3] = og[n];
    return;
  }
  const TcRun r = runs[g];
  const int qt = r.factored ? Qt : 1;
  const int nq = (int)ceil_div(r.Q, qt);
  const int np = (int)ceil_div(r.P, kTcRows);
  // factored items first, then the generic ones (offset by the factored total)
  const int base = r.factored ? of[g] : of[n] + og[g];
  for (int a = 0; a < np; ++a)
    for (int b = 0; b < nq; ++b) {
      TcItem t;
      t.run = g;
      t.p0 = a * kTcRows;
      t.q0 = b * qt;
      items[base + a * nq + b] = t;
    }
}

__global__ void tc_reduce_kernel(const float2 *__restrict__ part, int splits, int64_t count, float2 *__restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  float2 acc = part[e];
  for (int k = 1; k < splits; ++k) {
    const float2 v = part[(int64_t)k * count + e];
    acc.x += v.x;
    acc.y += v.y;
  }
  out[e] = acc;
}

struct TcPlan {
  float *MM;
  Csr csr;
  Runs runs;
  float *weights;
  TcRun *tcruns;
  TcItem *items;
  int *nf, *ng, *of, *og;
  int *error;
  float2 *partials;
  int max_splits;
};

static int tc_max_splits(int64_t S, int64_t V) {
  const int64_t bytes_per = S * V * 8;
  int64_t s = bytes_per > 0 ? (1LL << 30) / bytes_per : 16;
  if (s > 16) s = 16;
  return (int)(s < 1 ? 1 : s);
}

static void carve_tc(Carve &c, const fm_signal_args *a, TcPlan &pl) {
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  const int64_t N = a->n_nodes, V = a->n_vencs;
  pl.MM = c.take<float>((size_t)N * V * 2);
  carve_csr(c, a->m_rows, a->m_nnz, pl.csr);
  carve_runs(c, S, kTcRows, pl.runs);
  pl.weights = c.take<float>((size_t)(S + 1) * motion_slots(a->motion));
  pl.tcruns = c.take<TcRun>(S + 1);
  pl.items = c.take<TcItem>(2 * S + 2);
  pl.nf = c.take<int>(S + 2);
  pl.ng = c.take<int>(S + 2);
  pl.of = c.take<int>(S + 2);
  pl.og = c.take<int>(S + 2);
  pl.error = c.take<int>(4);
  pl.max_splits = tc_max_splits(S, V);
  pl.partials = c.take<float2>((size_t)pl.max_splits * S * V);
}

size_t tc_workspace(const fm_signal_args *a) {
  Carve c(nullptr, 0);
  TcPlan pl;
  carve_tc(c, a, pl);
  return c.used;
}

// Splits of the node range: enough blocks to cover the SMs a few times with
// little tail, each split at least 2048 nodes.
static int tc_choose_splits(int64_t items, int64_t N, int max_splits) {
  if (items <= 0) return 1;
  int best = 1;
  double best_cost = 1e30;
  for (int s = 1; s <= max_splits; ++s) {
    if (s > 1 && ceil_div(N, s) < 2048) break;
    const int64_t blocks = items * s;
    const int64_t waves = ceil_div(blocks, kSmCount);
    // time ~ waves x (work per block) ; work per block ~ 1/s
    const double cost = (double)waves / s + (blocks < kSmCount ? 1.0 : 0.0) * 0.0;
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = s;
    }
  }
  return best;
}

int signal_tc(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes) {
  const char *who = "fm_signal(BF16X3)";
  cudaStream_t st = ctx->stream;
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  const int64_t N = a->n_nodes, V = a->n_vencs;
  Carve cv(ws, ws_bytes);
  TcPlan pl;
  carve_tc(cv, a, pl);
  FM_TRY(carve_ok(cv, who));
  if (S == 0 || V == 0) return FM_OK;
  float2 *out = static_cast<float2 *>(a->out);
  if (N == 0) {
    FM_CUDA(cudaMemsetAsync(out, 0, (size_t)S * V * sizeof(float2), st));
    return FM_OK;
  }
  FM_REQUIRE(a->n_lines * a->n_kz < (1LL << 30), FM_ERR_SHAPE, "%s: slab too large", who);
  FM_TRY(sparse_times_dense<float>(a, pl.csr, static_cast<const float *>(a->Mxy), pl.MM, st));
  int n_runs = 0, n_tiles = 0;
  FM_TRY(build_runs<float>(static_cast<const float *>(a->t), S, kTcRows, pl.runs, st, &n_runs, &n_tiles));
  const MotionDev md = make_motion_dev(a->motion);
  if (a->motion && a->motion->kind == FM_MOTION_TABLE) {
    FM_REQUIRE(a->motion->table_calls == n_runs, FM_ERR_SHAPE,
               "%s: TABLE motion holds %lld entries but t has %d distinct-time runs", who,
               (long long)a->motion->table_calls, n_runs);
  }
  FM_TRY(launch_motion_weights(md, pl.runs.run_t, n_runs, pl.weights, st));
  const float *kx = static_cast<const float *>(a->kx), *ky = static_cast<const float *>(a->ky),
              *kz = static_cast<const float *>(a->kz);
  tc_classify_kernel<<<n_runs, 256, 0, st>>>(kx, ky, kz, pl.runs.start, pl.runs.counts, (int)a->n_lines,
                                             (int)a->n_kz, pl.tcruns);
  count_launch();
  FM_TRY(check_launch("tc_classify_kernel"));
  FM_CUDA(cudaMemsetAsync(pl.error, 0, 4 * sizeof(int), st));

  for (int64_t v0 = 0; v0 < V; v0 += kTcVGroup) {
    const int VG = (int)((V - v0) < kTcVGroup ? (V - v0) : kTcVGroup);
    const int Qt_f = (int)((a->n_kz < 128 / VG) ? a->n_kz : (128 / VG > 0 ? 128 / VG : 1));
    const unsigned gb = (unsigned)ceil_div(n_runs + 1, 256);
    tc_count_kernel<<<gb, 256, 0, st>>>(pl.tcruns, pl.runs.counts, Qt_f, pl.nf, pl.ng);
    count_launch();
    FM_TRY(check_launch("tc_count_kernel"));
    size_t cb = pl.runs.cub_bytes;
    FM_CUDA(cub::DeviceScan::ExclusiveSum(pl.runs.cub_tmp, cb, pl.nf, pl.of, n_runs + 1, st));
    cb = pl.runs.cub_bytes;
    FM_CUDA(cub::DeviceScan::ExclusiveSum(pl.runs.cub_tmp, cb, pl.ng, pl.og, n_runs + 1, st));
    count_launch(2);
    tc_fill_kernel<<<gb, 256, 0, st>>>(pl.tcruns, pl.runs.counts, Qt_f, pl.of, pl.og, pl.items);
    count_launch();
    FM_TRY(check_launch("tc_fill_kernel"));
    int h[4] = {0, 0, 0, 0};
    FM_CUDA(cudaMemcpyAsync(h, pl.runs.counts, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    FM_CUDA(cudaStreamSynchronize(st));
    const int n_fact = h[2], n_gen = h[3];
    const int splits = tc_choose_splits(n_fact + n_gen, N, pl.max_splits);

    TcDev p{};
    p.N = N; p.S = S; p.V = V;
    p.v0 = (int)v0; p.VG = VG;
    p.n_lines = (int)a->n_lines; p.n_kz = (int)a->n_kz;
    p.kx = kx; p.ky = ky; p.kz = kz;
    p.r0 = static_cast<const float *>(a->r0);
    p.phi = static_cast<const float *>(a->phi);
    p.T2 = static_cast<const float *>(a->T2);
    p.MM = reinterpret_cast<const float2 *>(pl.MM);
    p.md = md;
    p.weights = (md.kind == FM_MOTION_TERMS) ? pl.weights : nullptr;
    p.table = (a->motion && a->motion->kind == FM_MOTION_TABLE) ? static_cast<const float *>(a->motion->table)
                                                                 : nullptr;
    p.run_t = pl.runs.run_t;
    p.runs = pl.tcruns;
    p.items = pl.items;
    p.splits = splits;
    p.chunk = ceil_div(ceil_div(N, splits), kTcNodes) * kTcNodes;
    p.out = (splits > 1) ? pl.partials : out;
    p.error = pl.error;
    if (splits > 1) FM_CUDA(cudaMemsetAsync(pl.partials, 0, (size_t)splits * S * V * sizeof(float2), st));

    ScopedTimer timer(ctx, "signal_tc");
    for (int kind = 0; kind < 2; ++kind) {
      const int count = kind == 0 ? n_fact : n_gen;
      if (count == 0) continue;
      p.item0 = kind == 0 ? 0 : n_fact;
      p.Qt = kind == 0 ? Qt_f : 1;
      const int cols = 2 * p.Qt * VG;
      p.NT = (int)ceil_div(cols, 16) * 16;
      p.tmem_cols = 32;
      while (p.tmem_cols < p.NT) p.tmem_cols <<= 1;
      const TcSmem Ls = tc_smem_layout(p.NT, VG, p.Qt);
      const size_t smem = Ls.total + 1024;
      FM_REQUIRE(smem <= 232448, FM_ERR_UNSUPPORTED, "%s: tile needs %zu bytes of shared memory", who, smem);
      FM_CUDA(cudaFuncSetAttribute(signal_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      dim3 grid((unsigned)count, (unsigned)splits);
      signal_tc_kernel<<<grid, kTcThreads, smem, st>>>(p);
      count_launch();
      FM_TRY(check_launch("signal_tc_kernel"));
    }
    if (splits > 1) {
      const int64_t count = S * V;
      tc_reduce_kernel<<<(unsigned)ceil_div(count, 256), 256, 0, st>>>(pl.partials, splits, count, out);
      count_launch();
      FM_TRY(check_launch("tc_reduce_kernel"));
    }
  }
  int herr = 0;
  FM_CUDA(cudaMemcpyAsync(&herr, pl.error, sizeof(int), cudaMemcpyDeviceToHost, st));
  FM_CUDA(cudaStreamSynchronize(st));
  FM_REQUIRE(herr == 0, FM_ERR_TIMEOUT, "%s: a tensor-core pipeline wait timed out (code %d)", who, herr);
  return FM_OK;
}

}  // namespace fm
