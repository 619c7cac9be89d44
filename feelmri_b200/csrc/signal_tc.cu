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
constexpr int kTcVGroup = 8;        // Mxy columns per launch
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
  const int *plan;  // device: [2] factored items, [3] generic items, [4] splits, [5] nodes per split
  float2 *partials; // (splits, S, V) when splits > 1
  float2 *out;
  float *scratch;  // per block: 128 x NT running sums
  int *error;
};

struct TcSmem {
  uint32_t stage_bytes, a_hi, a_lo, b_hi, b_lo;  // offsets inside a stage
  uint32_t posd, valid, w, etab, kq, bars, misc, total;
};

// Node data is double-buffered: block b is read while block b + 1 is written.
__host__ __device__ inline TcSmem tc_smem_layout(int NT, int VG, int Qt) {
  TcSmem L;
  L.a_hi = 0;
  L.a_lo = kAStageBytes;
  L.b_hi = 2 * kAStageBytes;
  L.b_lo = 2 * kAStageBytes + NT * 2 * kTcNodes * 2;
  L.stage_bytes = 2 * kAStageBytes + 2 * NT * 2 * kTcNodes * 2;
  uint32_t off = kTcStages * L.stage_bytes;
  L.posd = off;  // [2][128] double4 (x, y, z, unused)
  off += 2 * kTcBlockNodes * 32;
  L.valid = off;  // [2][128] float
  off += 2 * kTcBlockNodes * 4;
  L.w = off;  // [2][128][VG] float2
  off += 2 * kTcBlockNodes * VG * 8;
  L.etab = off;  // [2][Qt][16] float2, by stage parity
  off += 2 * Qt * kTcNodes * 8;
  L.kq = off;  // [Qt][3] double
  off += ((Qt * 24 + 15) / 16) * 16;
  L.bars = off;
  off += 16 * 8;
  L.misc = off;  // tmem address, abort flag
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

__device__ inline uint32_t bf16x2_bits(__nv_bfloat162 h) { return *reinterpret_cast<uint32_t *>(&h); }

// hi = bf16(x), lo = bf16(x - hi) for the pair (a, b); bits of (hi_a, hi_b)
// and (lo_a, lo_b) with a in the low half.
__device__ inline void split_pair(float a, float b, uint32_t &hi, uint32_t &lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  hi = bf16x2_bits(h);
  lo = bf16x2_bits(__floats2bfloat162_rn(a - hf.x, b - hf.y));
}

// exp(-2 pi i c) for c in cycles given in FP64: reduce modulo one with an
// exact round-to-integer (add/subtract 1.5 * 2^52), then FP32 sin/cos.
__device__ inline float2 cis_neg_cycles(double c) {
  const double kRound = 6755399441055744.0;
  const double n = __dsub_rn(__dadd_rn(c, kRound), kRound);
  const float f = __double2float_rn(__dsub_rn(c, n));
  float s, co;
  __sincosf(6.283185307179586f * f, &s, &co);
  return make_float2(co, -s);
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

// Bounded wait that gives up at once after any earlier timeout of the block
// (the flag lives in shared memory), so a broken pipeline ends quickly.
__device__ inline bool tc_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  if (*abort_flag) return false;
  if (ptx::mbar_wait(bar, parity, kTcWaitNs)) return true;
  *abort_flag = 1;
  return false;
}

// Raw node data loaded one node block ahead (global loads in flight while
// the current block is processed).
struct TcRaw {
  float x, y, z, t2, phi;
  float2 m[kTcVGroup];
};

__device__ inline void tc_load_raw(const TcDev &p, int64_t n, TcRaw &r) {
  r.x = p.r0[3 * n + 0];
  r.y = p.r0[3 * n + 1];
  r.z = p.r0[3 * n + 2];
  r.t2 = p.T2[n];
  r.phi = p.phi[n];
#pragma unroll
  for (int v = 0; v < kTcVGroup; ++v)
    if (v < p.VG) r.m[v] = p.MM[n * p.V + p.v0 + v];
}

// Per-run node quantities of one node into buffer `buf`: moved position (in
// FP64 for the phase products), validity and the decayed, off-resonance
// rotated weights W' = (M Mxy)[n, v] exp(-t / T2) exp(i phi t).
__device__ inline void tc_derive(const TcDev &p, const TcUnit &U, int64_t n, const TcRaw &r, const float *wrun,
                                 float tg, double4 *posd, float *valid, float2 *wblk, int slot) {
  if (n < U.n_end) {
    float x = r.x, y = r.y, z = r.z;
    if (p.md.kind == FM_MOTION_TERMS) {
      float dx, dy, dz;
      motion_disp(p.md, wrun, n, p.N, dx, dy, dz);
      x = x + dx; y = y + dy; z = z + dz;
    } else if (p.table) {
      const float *d = p.table + ((int64_t)U.it.run * p.N + n) * 3;
      x = x + d[0]; y = y + d[1]; z = z + d[2];
    }
    posd[slot] = make_double4((double)x, (double)y, (double)z, 0.0);
    valid[slot] = 1.f;
    const float decay = expf(-tg * (1.0f / r.t2));
    float so, co;
    sincosf(r.phi * tg, &so, &co);
    const float er = decay * co, ei = decay * so;
#pragma unroll
    for (int v = 0; v < kTcVGroup; ++v)
      if (v < p.VG) wblk[slot * p.VG + v] = make_float2(r.m[v].x * er - r.m[v].y * ei, r.m[v].x * ei + r.m[v].y * er);
  } else {
    posd[slot] = make_double4(0.0, 0.0, 0.0, 0.0);
    valid[slot] = 0.f;
    for (int v = 0; v < p.VG; ++v) wblk[slot * p.VG + v] = make_float2(0.f, 0.f);
  }
}

// Adds accumulator `b` (one drained group) into the block's running sums,
// or, for the unit's last group, writes running sums + accumulator to the
// output samples.  Executed by all 256 producers: warp w reads TMEM lanes of
// quarter w % 4 and column half w / 4.
__device__ inline void tc_drain(const TcDev &p, const TcUnit &U, uint64_t *accfull, uint64_t *accfree, uint32_t tmem,
                                int gg, bool first, bool final, volatile int *abort_flag) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const int b = gg & 1;
  tc_wait(&accfull[b], (gg >> 1) & 1, abort_flag);
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
    ptx::tmem_ld16(tmem + (uint32_t)(b * p.acc_cols) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0, r);
    ptx::tmem_wait_ld();
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
}

__global__ void __launch_bounds__(kTcThreads, 1) signal_tc_kernel(TcDev p_in, int kind) {
  extern __shared__ __align__(1024) unsigned char smem[];
  // work sizes come from the device-side plan, so the launch needs no host
  // synchronisation (and can be captured in a CUDA graph)
  TcDev p = p_in;
  p.splits = p_in.plan[4];
  p.chunk = p_in.plan[5];
  p.item0 = kind == 0 ? 0 : p_in.plan[2];
  p.n_items = kind == 0 ? p_in.plan[2] : p_in.plan[3];
  p.out = p.splits > 1 ? p_in.partials : p_in.out;
  const int n_units = p.n_items * p.splits;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const TcSmem L = tc_smem_layout(p.NT, p.VG, p.Qt);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + L.bars);
  uint64_t *empty = full + kTcStages;
  uint64_t *accfull = empty + kTcStages;
  uint64_t *accfree = accfull + 2;
  uint64_t *done = accfree + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L.misc);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + L.misc + 4);
  double4 *posd_all = reinterpret_cast<double4 *>(smem + L.posd);
  float *valid_all = reinterpret_cast<float *>(smem + L.valid);
  float2 *w_all = reinterpret_cast<float2 *>(smem + L.w);
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
    *abort_flag = 0;
    ptx::fence_mbar_init();
  }
  if (warp == kTcMmaWarp) ptx::tmem_alloc(tmem_slot, 2 * p.acc_cols);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = tmem_slot[0];
  const uint32_t idesc = ptx::idesc_bf16_f32(kTcRows, p.NT);

  if (warp < kTcMmaWarp) {
    // ------------------------------------------------------ producers --
    const int row = tid & (kTcRows - 1);  // A row / B (q, v) pair of this thread
    const int half = tid >> 7;            // which 8 of the 16 nodes of a stage
    const bool loader = tid < kTcBlockNodes;
    int gst = 0, gbase = 0;
    TcRaw raw;
    for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
      const TcUnit U = tc_unit(p, u);
      ptx::named_barrier(1, kTcProducers);  // the previous unit's readers are done
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
      const int n_blocks = (int)ceil_div(U.n_stages, kTcBlockNodes / kTcNodes);
      // prologue: node block 0 into buffer 0, block 1's loads in flight
      if (loader && U.n_stages > 0) {
        const int64_t n = U.n_begin + tid;
        if (n < U.n_end) tc_load_raw(p, n, raw);
        tc_derive(p, U, n, raw, wrun, tg, posd_all, valid_all, w_all, tid);
        const int64_t n1 = n + kTcBlockNodes;
        if (n_blocks > 1 && n1 < U.n_end) tc_load_raw(p, n1, raw);
      }
      int next_drain = 0;

      for (int st = 0; st < U.n_stages; ++st, ++gst) {
        const int s = gst % kTcStages;
        const uint32_t round = gst / kTcStages;
        const int j = st % (kTcBlockNodes / kTcNodes);
        const int blk = st / (kTcBlockNodes / kTcNodes);
        const int buf = blk & 1;
        if (j == 0) {
          // buffer `buf` (written during the previous block) is complete, and
          // every producer is done with the other buffer
          ptx::named_barrier(1, kTcProducers);
          if (loader && blk >= 1 && blk + 1 < n_blocks) {
            const int64_t n2 = U.n_begin + (int64_t)(blk + 1) * kTcBlockNodes + tid;
            if (n2 < U.n_end) tc_load_raw(p, n2, raw);
          }
        }
        if (j == 4 && loader && blk + 1 < n_blocks) {
          const int64_t n1 = U.n_begin + (int64_t)(blk + 1) * kTcBlockNodes + tid;
          tc_derive(p, U, n1, raw, wrun, tg, posd_all + (buf ^ 1) * kTcBlockNodes,
                    valid_all + (buf ^ 1) * kTcBlockNodes, w_all + (buf ^ 1) * kTcBlockNodes * p.VG, tid);
        }
        const double4 *pn = posd_all + buf * kTcBlockNodes + j * kTcNodes;
        const float *vn = valid_all + buf * kTcBlockNodes + j * kTcNodes;
        const float2 *wn = w_all + (buf * kTcBlockNodes + j * kTcNodes) * p.VG;
        // wait until the MMAs that last read stage s are done
        tc_wait(&empty[s], (round & 1) ^ 1, abort_flag);
        // e_q(n) = exp(-2 pi i kq_q . r_n) for this stage's nodes.  Buffers
        // alternate by stage: a thread that writes stage st's table has passed
        // the barrier of stage st - 1, so every reader of stage st - 2 is done.
        float2 *et = etab + (st & 1) * p.Qt * kTcNodes;
        for (int idx = tid; idx < U.Q_tile * kTcNodes; idx += kTcProducers) {
          const int q = idx / kTcNodes, n = idx % kTcNodes;
          float2 e = make_float2(1.f, 0.f);
          if (U.run.factored) {
            const double4 r = pn[n];
            e = cis_neg_cycles(kq[3 * q] * r.x + kq[3 * q + 1] * r.y + kq[3 * q + 2] * r.z);
          }
          et[idx] = e;
        }
        ptx::named_barrier(1, kTcProducers);
        const uint32_t stage = sbase + s * L.stage_bytes;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {  // two chunks of 4 nodes (8 K values)
          const int h = 2 * half + hh;
          const uint32_t off = kmajor_offset(row, 8 * h, kTcRows);
          if (a_active) {
            uint32_t ah[4], al[4];
#pragma unroll
            for (int u4 = 0; u4 < 4; ++u4) {
              const int n = 4 * h + u4;
              const double4 r = pn[n];
              float2 e = cis_neg_cycles(kpx * r.x + kpy * r.y + kpz * r.z);
              if (vn[n] == 0.f) e = make_float2(0.f, 0.f);
              split_pair(e.x, e.y, ah[u4], al[u4]);
            }
            ptx::st_shared_v4(stage + L.a_hi + off, ah[0], ah[1], ah[2], ah[3]);
            ptx::st_shared_v4(stage + L.a_lo + off, al[0], al[1], al[2], al[3]);
          } else {
            ptx::st_shared_v4(stage + L.a_hi + off, 0u, 0u, 0u, 0u);
            ptx::st_shared_v4(stage + L.a_lo + off, 0u, 0u, 0u, 0u);
          }
          if (b_rows) {
            const uint32_t o_re = kmajor_offset(2 * row, 8 * h, p.NT);
            const uint32_t o_im = kmajor_offset(2 * row + 1, 8 * h, p.NT);
            uint32_t rh[4] = {0u, 0u, 0u, 0u}, rl[4] = {0u, 0u, 0u, 0u};
            uint32_t ih[4] = {0u, 0u, 0u, 0u}, il[4] = {0u, 0u, 0u, 0u};
            if (b_active) {
#pragma unroll
              for (int u4 = 0; u4 < 4; ++u4) {
                const int n = 4 * h + u4;
                const float2 e = et[bq * kTcNodes + n];
                const float2 w = wn[n * p.VG + bv];
                const float br = e.x * w.x - e.y * w.y, bi = e.x * w.y + e.y * w.x;
                uint32_t hb, lb;
                split_pair(br, bi, hb, lb);  // (br, bi) halves
                // row (q,v,re) holds (Re B, -Im B); row (q,v,im) holds (Im B, Re B)
                rh[u4] = hb ^ 0x80000000u;
                rl[u4] = lb ^ 0x80000000u;
                ih[u4] = __byte_perm(hb, 0u, 0x1032);
                il[u4] = __byte_perm(lb, 0u, 0x1032);
              }
            }
            ptx::st_shared_v4(stage + L.b_hi + o_re, rh[0], rh[1], rh[2], rh[3]);
            ptx::st_shared_v4(stage + L.b_lo + o_re, rl[0], rl[1], rl[2], rl[3]);
            ptx::st_shared_v4(stage + L.b_hi + o_im, ih[0], ih[1], ih[2], ih[3]);
            ptx::st_shared_v4(stage + L.b_lo + o_im, il[0], il[1], il[2], il[3]);
          }
        }
        ptx::fence_proxy_async_smem();
        ptx::mbar_arrive(&full[s]);
        // drain the previous group a few stages into the current one, when the
        // MMAs that wrote it have (almost surely) completed
        if (st % kTcDrain == kTcStages - 1 && st / kTcDrain >= 1 && next_drain == st / kTcDrain - 1) {
          tc_drain(p, U, accfull, accfree, tmem, gbase + next_drain, next_drain == 0, false, abort_flag);
          ++next_drain;
        }
      }
      while (next_drain < U.n_groups) {
        tc_drain(p, U, accfull, accfree, tmem, gbase + next_drain, next_drain == 0, next_drain == U.n_groups - 1,
                 abort_flag);
        ++next_drain;
      }
      if (U.n_groups == 0 && tid < kTcRows && row < U.P_tile) {
        // no nodes in this split: its share of the tile is zero
        float2 *dst = p.out + (int64_t)U.split * p.S * p.V;
        const int s_row = U.run.start + (U.run.factored ? (U.it.p0 + row) * p.n_kz + U.it.q0 : U.it.p0 + row);
        for (int q = 0; q < U.Q_tile; ++q)
          for (int v = 0; v < p.VG; ++v) dst[(int64_t)(s_row + q) * p.V + p.v0 + v] = make_float2(0.f, 0.f);
      }
      gbase += U.n_groups;
    }
  } else if (tid == kTcMmaWarp * 32) {
    // ------------------------------------------------------ MMA issue --
    int gst = 0, gbase = 0;
    for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
      const TcUnit U = tc_unit(p, u);
      for (int st = 0; st < U.n_stages; ++st, ++gst) {
        const int s = gst % kTcStages;
        const uint32_t round = gst / kTcStages;
        const int gg = gbase + st / kTcDrain;
        const int b = gg & 1;
        const bool group_start = (st % kTcDrain) == 0;
        if (group_start && gg >= 2) tc_wait(&accfree[b], ((gg - 2) >> 1) & 1, abort_flag);
        tc_wait(&full[s], round & 1, abort_flag);
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
    if (!ptx::mbar_wait(done, 0, kTcWaitNs)) *abort_flag = 1;
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (tid == 0 && *abort_flag) atomicOr(p.error, kErrTimeout);
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
  const int n_runs = counts[0];
  for (int g = blockIdx.x; g < n_runs; g += gridDim.x) {
  __syncthreads();
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
  }  // runs
}

// Item counts per run, factored runs in one list and the rest in another.
__global__ void tc_count_kernel(const TcRun *__restrict__ runs, const int *__restrict__ counts, int Qt,
                                int *__restrict__ nf, int *__restrict__ ng, int64_t S) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = counts[0];
  if (g > S) return;
  if (g >= n) {
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

// Node-range splits: enough work units that the persistent blocks finish
// together (units per block close to an integer), each split at least 2048
// nodes; fewer splits win ties.
__host__ __device__ inline int tc_choose_splits(int64_t items, int64_t N, int max_splits) {
  if (items <= 0) return 1;
  int best = 1;
  double best_eff = -1.0;
  for (int s = 1; s <= max_splits; ++s) {
    if (s > 1 && ceil_div(N, s) < 2048) break;
    const double units = (double)items * s;
    const double per_block = units / kSmCount;
    const double eff = per_block / ceil(per_block) * (units < kSmCount ? units / kSmCount : 1.0);
    if (eff > best_eff + 0.02) {
      best_eff = eff;
      best = s;
    }
  }
  return best;
}

__global__ void tc_plan_kernel(int *__restrict__ counts, int64_t N, int max_splits) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int splits = tc_choose_splits((int64_t)counts[2] + counts[3], N, max_splits);
  counts[4] = splits;
  counts[5] = (int)(ceil_div(ceil_div(N, splits), kTcNodes) * kTcNodes);
}

__global__ void tc_reduce_kernel(const float2 *__restrict__ part, const int *__restrict__ plan, int64_t count,
                                 float2 *__restrict__ out) {
  const int splits = plan[4];
  if (splits <= 1) return;
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
  const float *kx = static_cast<const float *>(a->kx), *ky = static_cast<const float *>(a->ky),
              *kz = static_cast<const float *>(a->kz);
  FM_TRY(build_runs<float>(static_cast<const float *>(a->t), S, kTcRows, pl.runs, st));
  FM_TRY(sparse_times_dense<float>(a, pl.csr, static_cast<const float *>(a->Mxy), pl.MM, pl.runs.error, st));
  FM_TRY(check_table_calls(a->motion, pl.runs, st));
  const MotionDev md = make_motion_dev(a->motion);
  FM_TRY(launch_run_weights(md, pl.runs.run_t, pl.runs.counts, S, pl.weights, st));
  const int64_t cls_blocks = S < 8 * kSmCount ? S : 8 * kSmCount;
  tc_classify_kernel<<<(unsigned)cls_blocks, 256, 0, st>>>(kx, ky, kz, pl.runs.start, pl.runs.counts,
                                                           (int)a->n_lines, (int)a->n_kz, pl.tcruns);
  count_launch();
  FM_TRY(check_launch("tc_classify_kernel"));

  for (int64_t v0 = 0; v0 < V; v0 += kTcVGroup) {
    const int VG = (int)((V - v0) < kTcVGroup ? (V - v0) : kTcVGroup);
    // columns per tile: up to 128 (q, v) pairs and at most 64 kz values
    const int q_cap = (128 / VG < 64) ? 128 / VG : 64;
    const int Qt_f = (int)((a->n_kz < q_cap) ? a->n_kz : q_cap);
    const unsigned gb = (unsigned)ceil_div(S + 1, 256);
    tc_count_kernel<<<gb, 256, 0, st>>>(pl.tcruns, pl.runs.counts, Qt_f, pl.nf, pl.ng, S);
    count_launch();
    FM_TRY(check_launch("tc_count_kernel"));
    size_t cb = pl.runs.cub_bytes;
    FM_CUDA(cub::DeviceScan::ExclusiveSum(pl.runs.cub_tmp, cb, pl.nf, pl.of, (int)(S + 1), st));
    cb = pl.runs.cub_bytes;
    FM_CUDA(cub::DeviceScan::ExclusiveSum(pl.runs.cub_tmp, cb, pl.ng, pl.og, (int)(S + 1), st));
    count_launch(2);
    tc_fill_kernel<<<gb, 256, 0, st>>>(pl.tcruns, pl.runs.counts, Qt_f, pl.of, pl.og, pl.items);
    count_launch();
    FM_TRY(check_launch("tc_fill_kernel"));
    tc_plan_kernel<<<1, 32, 0, st>>>(pl.runs.counts, N, pl.max_splits);
    count_launch();
    FM_TRY(check_launch("tc_plan_kernel"));

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
    p.plan = pl.runs.counts;
    p.partials = pl.partials;
    p.out = out;
    p.scratch = pl.scratch;
    p.error = pl.runs.error;

    ScopedTimer timer(ctx, "signal_tc");
    for (int kind = 0; kind < 2; ++kind) {
      p.Qt = kind == 0 ? Qt_f : 1;
      const int cols = 2 * p.Qt * VG;
      p.NT = (int)ceil_div(cols, 16) * 16;
      p.acc_cols = 32;
      while (p.acc_cols < p.NT) p.acc_cols <<= 1;
      const TcSmem Ls = tc_smem_layout(p.NT, VG, p.Qt);
      const size_t smem = Ls.total + 1024;
      FM_REQUIRE(smem <= 232448, FM_ERR_UNSUPPORTED, "%s: tile needs %zu bytes of shared memory", who, smem);
      FM_CUDA(cudaFuncSetAttribute(signal_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      signal_tc_kernel<<<kSmCount, kTcThreads, smem, st>>>(p, kind);
      count_launch();
      FM_TRY(check_launch("signal_tc_kernel"));
    }
    const int64_t count = S * V;
    tc_reduce_kernel<<<(unsigned)ceil_div(count, 256), 256, 0, st>>>(pl.partials, pl.runs.counts, count, out);
    count_launch();
    FM_TRY(check_launch("tc_reduce_kernel"));
  }
  return FM_OK;
}

int signal_tc_errors(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes) {
  Carve cv(ws, ws_bytes);
  TcPlan pl;
  carve_tc(cv, a, pl);
  FM_TRY(carve_ok(cv, "fm_signal(BF16X3)"));
  return report_errors(pl.runs, ctx->stream, "fm_signal(BF16X3)");
}

}  // namespace fm
