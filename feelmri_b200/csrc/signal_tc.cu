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
// Block (persistent, one per SM): warps 0-7 produce operand tiles (16 nodes
// per pipeline stage, 4 stages of shared memory in the UMMA no-swizzle
// K-major layout) and drain the accumulators; one thread of warp 8 issues the
// MMAs and warp 8 owns the tensor memory.  Stages are handed over with
// mbarriers; tcgen05.commit frees a stage when the MMAs that read it have
// completed.  The tensor core's FP32 accumulation truncates, so each
// accumulator only collects 32 stages: two accumulators alternate in tensor
// memory and the producers drain the idle one into an FP32 (round-to-nearest)
// running sum.  Blocks loop over work units (row/column tile of a run x node
// range).  All waits are bounded: on timeout the block records an error,
// lets its MMAs finish and frees its tensor memory.
#include <cuda_bf16.h>
#include <cmath>
#include <cub/cub.cuh>

#include "signal_common.cuh"
#include "tc_ptx.cuh"

namespace fm {

constexpr int kTcRows = 128;        // UMMA M
constexpr int kTcNodes = 16;        // nodes per stage -> K = 32 (two UMMA K steps)
constexpr int kTcStages = 4;
constexpr int kTcBlockNodes = 128;  // nodes whose per-run data is formed together
constexpr int kTcProducers = 256;   // warps 0-7
constexpr int kTcMmaWarp = 8;
constexpr int kTcThreads = 288;
constexpr int kTcVGroup = 16;       // Mxy columns per launch
// Stages accumulated in one tensor-memory accumulator before it is drained
// into an FP32 round-to-nearest running sum.  The tensor core's FP32
// accumulation truncates, so its error grows with the number of MMAs added
// into one accumulator; 32 stages (512 nodes, 192 MMAs) keep it near 1e-5.
constexpr int kTcDrain = 32;
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
  int item0, n_items;
  int Qt, NT, acc_cols;
  int splits;
  int64_t chunk;
  float2 *out;
  float *scratch;  // per block: 128 x NT running sums
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

__device__ inline void store_zero8(uint32_t hi_addr, uint32_t lo_addr) {
  ptx::st_shared_v4(hi_addr, 0u, 0u, 0u, 0u);
  ptx::st_shared_v4(lo_addr, 0u, 0u, 0u, 0u);
}

// exp(-2 pi i c) for c in cycles given in FP64: reduce modulo one, then FP32.
__device__ inline float2 cis_neg_cycles(double c) {
  const double f = c - rint(c);
  float s, co;
  __sincosf(6.283185307179586f * (float)f, &s, &co);
  return make_float2(co, -s);
}

// OR of a predicate over the 256 producer threads (named barrier 1): used
// for every decision that must be uniform across them.
__device__ inline bool producers_any(bool x) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\t"
      "setp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, 1, 256, pi;\n\t"
      "selp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)x)
      : "memory");
  return out != 0;
}

struct TcUnit {
  TcItem it;
  TcRun run;
  int split, P_tile, Q_tile, n_stages, n_groups;
  int64_t n_begin, n_end;
};

__device__ inline TcUnit tc_unit(const TcDev &p, int u) {
  TcUnit U;
  const int item = u % p.n_items;
  U.split = u / p.n_items;
  U.it = p.items[p.item0 + item];
  U.run = p.runs[U.it.run];
  U.P_tile = min(kTcRows, U.run.P - U.it.p0);
  U.Q_tile = min(p.Qt, U.run.Q - U.it.q0);
  U.n_begin = (int64_t)U.split * p.chunk;
  U.n_end = min(p.N, U.n_begin + p.chunk);
  U.n_stages = U.n_end > U.n_begin ? (int)ceil_div(U.n_end - U.n_begin, kTcNodes) : 0;
  U.n_groups = (int)ceil_div(U.n_stages, kTcDrain);
  return U;
}

// Adds accumulator `buf` (one drained group) into the block's running sums,
// or, for the unit's last group, writes running sums + accumulator to the
// output samples.  Executed by all 256 producers: warp w reads TMEM lanes of
// quarter w % 4 and column half w / 4.
__device__ inline bool tc_drain(const TcDev &p, const TcUnit &U, uint64_t *accfull, uint64_t *accfree, uint32_t tmem,
                                int gg, bool first, bool final, bool ok_in) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const int b = gg & 1;
  const bool waited = ptx::mbar_wait(&accfull[b], (gg >> 1) & 1, kTcWaitNs);
  const bool ok = ok_in && !producers_any(!waited);
  ptx::tc_fence_after();
  const int quarter = warp & 3, half = warp >> 2;
  const int row = quarter * 32 + (tid & 31);
  const int cph = ((p.NT / 2 + 15) / 16) * 16;
  const int c_begin = half * cph, c_end = min(p.NT, c_begin + cph);
  float *srow = p.scratch + ((size_t)blockIdx.x * kTcRows + row) * p.NT;
  const bool row_ok = row < U.P_tile;
  float2 *dst = p.out + (int64_t)U.split * p.S * p.V;
  const int s_row = U.run.start + (U.run.factored ? (U.it.p0 + row) * p.n_kz + U.it.q0 : U.it.p0 + row);
  for (int c0 = c_begin; c0 < c_end; c0 += 16) {
    uint32_t r[16];
    if (ok) {
      ptx::tmem_ld16(tmem + (uint32_t)(b * p.acc_cols) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0, r);
      ptx::tmem_wait_ld();
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) r[i] = 0u;
    }
    if (!row_ok) continue;
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
    if (!first) {
      const float4 *src = reinterpret_cast<const float4 *>(srow + c0);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float4 a = src[i];
        v[4 * i] += a.x; v[4 * i + 1] += a.y; v[4 * i + 2] += a.z; v[4 * i + 3] += a.w;
      }
    }
    if (!final) {
      float4 *d4 = reinterpret_cast<float4 *>(srow + c0);
#pragma unroll
      for (int i = 0; i < 4; ++i) d4[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int jj = (c0 >> 1) + i;
        const int q = jj / p.VG, vv = jj % p.VG;
        if (q < U.Q_tile) dst[(int64_t)(s_row + q) * p.V + p.v0 + vv] = make_float2(v[2 * i], v[2 * i + 1]);
      }
    }
  }
  ptx::tc_fence_before();
  ptx::mbar_arrive(&accfree[b]);
  return ok;
}

__global__ void __launch_bounds__(kTcThreads, 1) signal_tc_kernel(TcDev p, int n_units) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const TcSmem L = tc_smem_layout(p.NT, p.VG, p.Qt);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L.bars);
  uint64_t *empty = full + kTcStages;
  uint64_t *accfull = empty + kTcStages;
  uint64_t *accfree = accfull + 2;
  uint64_t *done = accfree + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L.misc);
  float4 *pos = reinterpret_cast<float4 *>(smem + L.pos);
  float2 *wblk = reinterpret_cast<float2 *>(smem + L.w);
  float2 *etab = reinterpret_cast<float2 *>(smem + L.etab);
  double *kq = reinterpret_cast<double *>(smem + L.kq);
  const uint32_t sbase = ptx::smem_addr(smem);

  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      ptx::mbar_init(&full[s], kTcProducers);
      ptx::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      ptx::mbar_init(&accfull[b], 1);
      ptx::mbar_init(&accfree[b], kTcProducers);
    }
    ptx::mbar_init(done, 1);
    ptx::fence_mbar_init();
  }
  if (warp == kTcMmaWarp) ptx::tmem_alloc(tmem_slot, 2 * p.acc_cols);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = tmem_slot[0];
  const uint32_t idesc = ptx::idesc_bf16_f32(kTcRows, p.NT);
  bool ok = true;

  if (warp < kTcMmaWarp) {
    // ------------------------------------------------------ producers --
    const int row = tid & (kTcRows - 1);  // A row / B (q, v) pair of this thread
    const int half = tid >> 7;            // which 8 of the 16 nodes of a stage
    int gst = 0, gbase = 0;
    for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
      const TcUnit U = tc_unit(p, u);
      ptx::named_barrier(1, kTcProducers);  // previous unit's readers of kq are done
      for (int q = tid; q < U.Q_tile; q += kTcProducers) {
        const int s_q = U.run.start + U.it.q0 + q, s_0 = U.run.start;
        kq[3 * q + 0] = U.run.factored ? (double)p.kx[s_q] - (double)p.kx[s_0] : 0.0;
        kq[3 * q + 1] = U.run.factored ? (double)p.ky[s_q] - (double)p.ky[s_0] : 0.0;
        kq[3 * q + 2] = U.run.factored ? (double)p.kz[s_q] - (double)p.kz[s_0] : 0.0;
      }
      const bool a_active = row < U.P_tile;
      double kpx = 0, kpy = 0, kpz = 0;
      if (a_active) {
        const int s_p = U.run.start + (U.run.factored ? (U.it.p0 + row) * p.n_kz : U.it.p0 + row);
        kpx = p.kx[s_p];
        kpy = p.ky[s_p];
        kpz = p.kz[s_p];
      }
      const bool b_rows = 2 * row < p.NT;
      const bool b_active = row < U.Q_tile * p.VG;
      const int bq = b_active ? row / p.VG : 0, bv = b_active ? row % p.VG : 0;
      const float *wrun = p.weights ? p.weights + (int64_t)U.it.run * p.md.slots : nullptr;
      const float tg = (float)p.run_t[U.it.run];
      int next_drain = 0;

      for (int st = 0; st < U.n_stages; ++st, ++gst) {
        const int s = gst % kTcStages;
        const uint32_t round = gst / kTcStages;
        const int j = st % (kTcBlockNodes / kTcNodes);
        if (j == 0) {
          ptx::named_barrier(1, kTcProducers);
          if (tid < kTcBlockNodes) {
            const int64_t n = U.n_begin + (int64_t)st * kTcNodes + tid;
            float4 pp = make_float4(0.f, 0.f, 0.f, 0.f);
            if (n < U.n_end) {
              float x = p.r0[3 * n + 0], y = p.r0[3 * n + 1], z = p.r0[3 * n + 2];
              if (p.md.kind == FM_MOTION_TERMS) {
                float dx, dy, dz;
                motion_disp(p.md, wrun, n, p.N, dx, dy, dz);
                x = x + dx; y = y + dy; z = z + dz;
              } else if (p.table) {
                const float *d = p.table + ((int64_t)U.it.run * p.N + n) * 3;
                x = x + d[0]; y = y + d[1]; z = z + d[2];
              }
              pp = make_float4(x, y, z, 1.f);
              const float decay = expf(-tg * (1.0f / p.T2[n]));
              float so, co;
              sincosf(p.phi[n] * tg, &so, &co);
              const float er = decay * co, ei = decay * so;
              for (int v = 0; v < p.VG; ++v) {
                const float2 m = p.MM[n * p.V + p.v0 + v];
                wblk[tid * p.VG + v] = make_float2(m.x * er - m.y * ei, m.x * ei + m.y * er);
              }
            } else {
              for (int v = 0; v < p.VG; ++v) wblk[tid * p.VG + v] = make_float2(0.f, 0.f);
            }
            pos[tid] = pp;
          }
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
        for (int idx = tid; idx < U.Q_tile * kTcNodes; idx += kTcProducers) {
          const int q = idx / kTcNodes, n = idx % kTcNodes;
          const float4 r = pn[n];
          float2 e = make_float2(1.f, 0.f);
          if (U.run.factored) {
            const double c = kq[3 * q] * (double)r.x + kq[3 * q + 1] * (double)r.y + kq[3 * q + 2] * (double)r.z;
            e = cis_neg_cycles(c);
          }
          etab[idx] = e;
        }
        ptx::named_barrier(1, kTcProducers);
        const uint32_t stage = sbase + s * L.stage_bytes;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {  // two chunks of 4 nodes (8 K values)
          const int h = 2 * half + hh;
          const uint32_t off = kmajor_offset(row, 8 * h, kTcRows);
          if (a_active) {
            float x[8];
#pragma unroll
            for (int u4 = 0; u4 < 4; ++u4) {
              const float4 r = pn[4 * h + u4];
              const double c = kpx * (double)r.x + kpy * (double)r.y + kpz * (double)r.z;
              float2 e = cis_neg_cycles(c);
              if (r.w == 0.f) e = make_float2(0.f, 0.f);
              x[2 * u4] = e.x;
              x[2 * u4 + 1] = e.y;
            }
            store_split8(stage + L.a_hi + off, stage + L.a_lo + off, x);
          } else {
            store_zero8(stage + L.a_hi + off, stage + L.a_lo + off);
          }
          if (b_rows) {
            const uint32_t o_re = kmajor_offset(2 * row, 8 * h, p.NT);
            const uint32_t o_im = kmajor_offset(2 * row + 1, 8 * h, p.NT);
            if (b_active) {
              float xr[8], xi[8];
#pragma unroll
              for (int u4 = 0; u4 < 4; ++u4) {
                const int n = 4 * h + u4;
                const float2 e = etab[bq * kTcNodes + n];
                const float2 w = wn[n * p.VG + bv];
                const float br = e.x * w.x - e.y * w.y, bi = e.x * w.y + e.y * w.x;
                xr[2 * u4] = br;
                xr[2 * u4 + 1] = -bi;
                xi[2 * u4] = bi;
                xi[2 * u4 + 1] = br;
              }
              store_split8(stage + L.b_hi + o_re, stage + L.b_lo + o_re, xr);
              store_split8(stage + L.b_hi + o_im, stage + L.b_lo + o_im, xi);
            } else {
              store_zero8(stage + L.b_hi + o_re, stage + L.b_lo + o_re);
              store_zero8(stage + L.b_hi + o_im, stage + L.b_lo + o_im);
            }
          }
        }
        ptx::fence_proxy_async_smem();
        ptx::mbar_arrive(&full[s]);
        // drain the previous group a few stages into the current one, when the
        // MMAs that wrote it have (almost surely) completed
        if (st % kTcDrain == kTcStages - 1 && st / kTcDrain >= 1 && next_drain == st / kTcDrain - 1) {
          ok = tc_drain(p, U, accfull, accfree, tmem, gbase + next_drain, next_drain == 0, false, ok);
          ++next_drain;
          if (!ok) break;
        }
      }
      while (ok && next_drain < U.n_groups) {
        ok = tc_drain(p, U, accfull, accfree, tmem, gbase + next_drain, next_drain == 0,
                      next_drain == U.n_groups - 1, ok);
        ++next_drain;
      }
      if (ok && U.n_groups == 0 && row == tid) {
        // no nodes in this split: its share of the tile is zero
        float2 *dst = p.out + (int64_t)U.split * p.S * p.V;
        if (row < U.P_tile) {
          const int s_row = U.run.start + (U.run.factored ? (U.it.p0 + row) * p.n_kz + U.it.q0 : U.it.p0 + row);
          for (int q = 0; q < U.Q_tile; ++q)
            for (int v = 0; v < p.VG; ++v) dst[(int64_t)(s_row + q) * p.V + p.v0 + v] = make_float2(0.f, 0.f);
        }
      }
      gbase += U.n_groups;
    }
    if (!ok) atomicExch(p.error, 1);
  } else if (tid == kTcMmaWarp * 32) {
    // ------------------------------------------------------ MMA issue --
    int gst = 0, gbase = 0;
    for (int u = blockIdx.x; u < n_units && ok; u += gridDim.x) {
      const TcUnit U = tc_unit(p, u);
      for (int st = 0; st < U.n_stages; ++st, ++gst) {
        const int s = gst % kTcStages;
        const uint32_t round = gst / kTcStages;
        const int gg = gbase + st / kTcDrain;
        const int b = gg & 1;
        const bool group_start = (st % kTcDrain) == 0;
        if (group_start && gg >= 2 && !ptx::mbar_wait(&accfree[b], ((gg - 2) >> 1) & 1, kTcWaitNs)) {
          ok = false;
          break;
        }
        if (!ptx::mbar_wait(&full[s], round & 1, kTcWaitNs)) {
          ok = false;
          break;
        }
        ptx::tc_fence_after();
        const uint32_t stage = sbase + s * L.stage_bytes;
        const uint32_t acc = tmem + (uint32_t)(b * p.acc_cols);
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const uint64_t ah = ptx::smem_desc(stage + L.a_hi + ks * kTcRows * 32, 128, 256);
          const uint64_t al = ptx::smem_desc(stage + L.a_lo + ks * kTcRows * 32, 128, 256);
          const uint64_t bh = ptx::smem_desc(stage + L.b_hi + ks * p.NT * 32, 128, 256);
          const uint64_t bl = ptx::smem_desc(stage + L.b_lo + ks * p.NT * 32, 128, 256);
          ptx::mma_bf16(acc, ah, bh, idesc, (group_start && ks == 0) ? 0u : 1u);
          ptx::mma_bf16(acc, ah, bl, idesc, 1u);
          ptx::mma_bf16(acc, al, bh, idesc, 1u);
        }
        ptx::mma_commit(&empty[s]);
        if ((st % kTcDrain) == kTcDrain - 1 || st == U.n_stages - 1) ptx::mma_commit(&accfull[b]);
      }
      gbase += U.n_groups;
    }
    // all issued MMAs complete before the tensor memory is released
    ptx::mma_commit(done);
    if (!ptx::mbar_wait(done, 0, kTcWaitNs)) ok = false;
    if (!ok) atomicExch(p.error, 2);
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == kTcMmaWarp) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, 2 * p.acc_cols);
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
  float *scratch;
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
  pl.scratch = c.take<float>((size_t)kSmCount * kTcRows * 256);
  pl.max_splits = tc_max_splits(S, V);
  pl.partials = c.take<float2>((size_t)pl.max_splits * S * V);
}

size_t tc_workspace(const fm_signal_args *a) {
  Carve c(nullptr, 0);
  TcPlan pl;
  carve_tc(c, a, pl);
  return c.used;
}

// Node-range splits: enough work units that the persistent blocks finish
// together (units per block close to an integer), each split at least 2048
// nodes; fewer splits win ties.
static int tc_choose_splits(int64_t items, int64_t N, int max_splits) {
  if (items <= 0) return 1;
  int best = 1;
  double best_eff = -1.0;
  for (int s = 1; s <= max_splits; ++s) {
    if (s > 1 && ceil_div(N, s) < 2048) break;
    const double units = (double)items * s;
    const double per_block = units / kSmCount;
    const double eff = per_block / std::ceil(per_block) * (units < kSmCount ? units / kSmCount : 1.0);
    if (eff > best_eff + 0.02) {
      best_eff = eff;
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
    p.scratch = pl.scratch;
    p.error = pl.error;

    ScopedTimer timer(ctx, "signal_tc");
    for (int kind = 0; kind < 2; ++kind) {
      const int count = kind == 0 ? n_fact : n_gen;
      if (count == 0) continue;
      p.item0 = kind == 0 ? 0 : n_fact;
      p.n_items = count;
      p.Qt = kind == 0 ? Qt_f : 1;
      const int cols = 2 * p.Qt * VG;
      p.NT = (int)ceil_div(cols, 16) * 16;
      p.acc_cols = 32;
      while (p.acc_cols < p.NT) p.acc_cols <<= 1;
      const TcSmem Ls = tc_smem_layout(p.NT, VG, p.Qt);
      const size_t smem = Ls.total + 1024;
      FM_REQUIRE(smem <= 232448, FM_ERR_UNSUPPORTED, "%s: tile needs %zu bytes of shared memory", who, smem);
      FM_CUDA(cudaFuncSetAttribute(signal_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const int n_units = count * splits;
      const int grid = n_units < kSmCount ? n_units : kSmCount;
      signal_tc_kernel<<<grid, kTcThreads, smem, st>>>(p, n_units);
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
