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
//   (Re A, -Im A) and, in two blocks of B rows, B'^T[(q,v,re)][2n..] =
//   (Re B, Im B) and B'^T[(q,v,im)][2n..] = (Im B, -Re B), so column
//   (q,v,re) of C' is Re C and column (q,v,im) is Im C.
// * Split BF16.  Each operand x is stored as hi = bf16(x), lo = bf16(x - hi);
//   hi*hi + hi*lo + lo*hi accumulate in FP32 in tensor memory.
// * Phases.  k . r is evaluated in FP64 and reduced modulo one cycle (in
//   fixed point, to 2^-24 cycles) before the FP32 sin/cos, so far nodes at
//   high k keep their digits.
//
// Block (persistent, one per SM, 16 warps): in factored units warps 0-7
// write the A tiles and warps 8-15 the B tiles and the phase tables; in
// generic units every warp writes A (16 nodes per pipeline stage, a ring of
// 4 stages in shared memory in the 64-byte swizzled K-major layout).
// Threads 0-127 also derive the node blocks.  After each group's
// barrier one thread (warp 7, lane 0) issues the group's MMAs; warp 0 owns
// the tensor memory.  tcgen05.commit frees a ring slot when the MMAs that
// read it have completed.  The tensor core's FP32 accumulation truncates, so
// the accumulator only collects 32 stages; all warps then fold it into an FP32
// (round-to-nearest) running sum kept in the other half of tensor memory.
// Blocks loop over work units (row/column tile of a run x node range).  All
// waits are bounded: on timeout the block records an error, lets its MMAs
// finish and frees its tensor memory.
#include <cmath>
#include <vector>
#include <cub/cub.cuh>

#include "signal_common.cuh"
#include "tc_ptx.cuh"

namespace fm {

constexpr int kTcRows = 128;        // UMMA M
constexpr int kTcNodes = 16;        // nodes per stage -> K = 32 (two UMMA K steps)
constexpr int kTcStages = 4;
// Generic units use a ring of their own (kTcRingGen slots of their small
// stages, which always fit), with their own barriers and stage counter, so
// that a group's producers need not wait for the previous group's MMAs.  At
// a unit's end every MMA has completed, so the two rings may share the
// shared memory.
constexpr int kTcRingGen = 8;
constexpr int kTcBlockNodes = 128;  // nodes whose per-run data is formed together
constexpr int kTcStagesPerBlock = kTcBlockNodes / kTcNodes;
constexpr int kTcProducerWarps = 16;
constexpr int kTcProducers = 32 * kTcProducerWarps;  // every thread of the block
constexpr int kTcThreads = kTcProducers;
constexpr int kTcVGroup = 8;        // Mxy columns per launch
// Stages accumulated in the tensor-memory accumulator before it is folded
// into an FP32 round-to-nearest running sum (also in tensor memory).  The
// tensor core's FP32 accumulation truncates, so its error grows with the
// number of MMAs added into one accumulator; 32 stages (512 nodes, 192 MMAs)
// keep it near 1e-5.
constexpr int kTcDrain = 32;
// Stages a generic (unfactored, N = 16) unit writes between two barriers.  At
// most kTcStages: a group's stages must use distinct ring slots, whose
// previous MMAs went out at an earlier barrier (so no wait can depend on the
// group's own MMAs).
constexpr int kTcGenGroup = 4;
// Stages a factored unit writes between two barriers.  The B warps compute
// the phase table of stage st + kTcFacGroup during stage st, so the table
// ring holds 2 kTcFacGroup buffers (kTcEBufs).
constexpr int kTcFacGroup = 2;
constexpr int kTcEBufs = 2 * kTcFacGroup;
constexpr uint64_t kTcWaitNs = 2000000000ull;
static_assert(kTcGenGroup <= kTcStages && (kTcRingGen & (kTcRingGen - 1)) == 0 &&
                  kTcStagesPerBlock % kTcGenGroup == 0 && kTcDrain % kTcGenGroup == 0,
              "generic stage groups must fit the ring, the node blocks and the accumulation groups");
static_assert(kTcFacGroup <= kTcStages && kTcStagesPerBlock % kTcFacGroup == 0 && kTcDrain % kTcFacGroup == 0 &&
                  (kTcEBufs & (kTcEBufs - 1)) == 0 && kTcFacGroup <= 2,
              "factored stage groups: the node block is requested at stage 2 and derived at stage 4 of 8");
constexpr uint32_t kAStageBytes = kTcRows * 2 * kTcNodes * 2;  // 128 rows x 32 K x bf16 = 8 KB

struct TcRun {
  int start, P, Q, factored;
};
// A work item: `rows` lines from line p0 and columns q0.. of run `run`, or
// (stacked problems) `rows` consecutive lines of the problem's runs laid end
// to end, from line p0 of run `run` on: unit row i is line (p0 + i) % P of
// run run + (p0 + i) / P (P lines per run), nrun runs in all, and every run
// shares the columns.  The runs then differ only in their times, so each
// run's decay and off-resonance factor D_r(n) = exp(-t_r / T2_n)
// exp(i phi_n t_r) moves into its A rows (A = exp(-2 pi i kp . r) D_r) and
// B = exp(-2 pi i kq . r) (M Mxy) is the same for all of them: the whole
// product is read.
struct TcItem {
  int run, p0, q0, nrun, rows;
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
  int Qt, NT, kind;  // kind 0: factored runs, 1: generic runs
  int wrows;         // rows per node buffer: VG weight rows, then (stacked runs) nrun D rows
  int stacked;       // items hold several runs (D in the A rows, B without decay)
  int mm_ld;         // row stride of MM (float2): this group's columns, padded to even
  int tma;           // node blocks are staged by bulk copies (aligned inputs, room in smem)
  int mstage;        // 3 r: a single POD term's mode rows are staged with each node block (0: read from global)
  const int *plan;  // device: [2] factored items, [3] generic items, [4] splits, [5] nodes per split
  float2 *partials; // (splits, S, V) when splits > 1
  float2 *out;
  int *error;
};

// One launch works through a table of entries (one per problem, Mxy column
// group and run kind); the device-side plan gives each entry's units.
struct TcBatchDev {
  const TcDev *entries;
  const int *offsets;  // device: n_entries + 1 running unit counts
  int n_entries;
  int acc_cols;  // tensor-memory columns of the widest entry (accumulator; the running sum follows)
};

// Work list of one entry, read from the device-side plan.
struct TcWork {
  int splits, item0, n_items;
  int64_t chunk;
  float2 *out;
};

__device__ inline TcWork tc_work(const TcDev &p) {
  const int kind = p.kind;
  TcWork W;
  W.splits = p.plan[4];
  W.chunk = p.plan[5];
  W.item0 = kind == 0 ? 0 : p.plan[2];
  W.n_items = kind == 0 ? p.plan[2] : p.plan[3];
  W.out = W.splits > 1 ? p.partials : p.out;
  return W;
}

// Shared-memory layout.  Strides of the weight and phase tables are padded
// (130 and 18 complex values) so that the B producers' 16-byte reads of
// different columns fall in different banks.
constexpr int kWStride = kTcBlockNodes + 2;
constexpr uint32_t kTcSmemMax = 232448;  // dynamic shared memory a block may opt in to
constexpr int kEStride = kTcNodes + 2;

// Barriers and the tensor-memory address live in the first kTcFront bytes
// (fixed, since the tile layout after them changes from unit to unit).
constexpr uint32_t kTcFront = 1024;
constexpr uint32_t kTcBars = 0, kTcMisc = 128;

struct TcSmem {
  uint32_t stage_bytes, a_hi, a_lo, b_hi, b_lo;  // offsets inside a stage
  uint32_t stages, pos, w, etab, raw, total;
};

// Node data is double-buffered: block b is read while block b + 1 is written.
__host__ __device__ inline TcSmem tc_smem_layout(int NT, int VG, int Qt, int ring = kTcStages) {
  // VG here is the weight rows per node buffer (TcDev::wrows)
  TcSmem L;
  L.a_hi = 0;
  L.a_lo = kAStageBytes;
  L.b_hi = 2 * kAStageBytes;
  L.b_lo = 2 * kAStageBytes + NT * 2 * kTcNodes * 2;
  L.stage_bytes = 2 * kAStageBytes + 2 * NT * 2 * kTcNodes * 2;
  L.stages = kTcFront;
  uint32_t off = kTcFront + (uint32_t)ring * L.stage_bytes;
  L.pos = off;  // [2][3][128] double: x, y, z of the moved nodes
  off += 2 * 3 * kTcBlockNodes * 8;
  L.w = off;  // [2][VG][kWStride] float2
  off += 2 * VG * kWStride * 8;
  L.etab = off;  // [kTcEBufs][Qt][kEStride] float2, by stage
  off += kTcEBufs * Qt * kEStride * 8;
  L.raw = off;  // staging of one raw node block (bulk copies), when used
  L.total = off;
  return L;
}

// Bytes of one raw node block: positions, T2, phi and the group's M Mxy rows.
__host__ __device__ inline uint32_t tc_raw_bytes(int mm_ld) {
  return kTcBlockNodes * (12 + 4 + 4 + 8 * mm_ld);
}

// Bytes of one node block's POD mode rows ([128][3 r] floats), staged after
// the raw block when TcDev::mstage (= 3 r) is set.
__host__ __device__ inline uint32_t tc_mode_bytes(int mstage) { return kTcBlockNodes * 4 * (uint32_t)mstage; }

// Byte offset of element (row, k) of a K-major operand tile with 32 K
// elements (64-byte rows) in the 64-byte swizzled layout: row r at r * 64,
// its 16-byte chunk c (elements 8c .. 8c + 7) stored at chunk position
// c ^ ((r >> 1) & 3), i.e. address bits 4-5 XOR bits 7-8.  Tiles start on
// 512-byte boundaries (8-row groups, SBO = 512), so the swizzle of a byte
// offset is the swizzle of its shared-memory address.  The tensor core reads
// this layout at full shared-memory bandwidth; the unswizzled layout's
// 16-byte core-matrix rows cap its operand reads, which dominates narrow
// (small N) MMAs.
__host__ __device__ inline uint32_t sw64_offset(uint32_t row, uint32_t k) {
  return row * 64 + ((((k >> 3) ^ (row >> 1)) & 3) << 4) + (k & 7) * 2;
}

// hi = bf16(x), lo = bf16(x - hi) for the pair (a, b); bits of (hi_a, hi_b)
// and (lo_a, lo_b) with a in the low half (cvt.rn.bf16x2 puts its first
// source in the upper half).
__device__ inline void split_pair(float a, float b, uint32_t &hi, uint32_t &lo) {
  uint32_t h, l;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(h) : "f"(b), "f"(a));
  const float ha = __uint_as_float(h << 16), hb = __uint_as_float(h & 0xffff0000u);
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(l) : "f"(b - hb), "f"(a - ha));
  hi = h;
  lo = l;
}

// cos and sin of 2 pi c for c in cycles given in FP64.  c is reduced modulo
// one in fixed point: adding 1.5 * 2^29 leaves a double whose last place is
// 2^-23, so its low 32 bits hold round(c * 2^23) modulo 2^32 and their low
// 23 bits, sign-extended, are c - rint(c) in units of 2^-23 (error at most
// 2^-24 cycles, for |c| < 2^28).  This keeps the reduction off the
// transcendental unit (no rint, no double-to-float conversion): one FP64
// add, a signed bit-field extract and an integer-to-float conversion, then
// the FP32 sin/cos.
__device__ inline void cycles_cos_sin(double c, float &co, float &s) {
  const int lo = __double2loint(__dadd_rn(c, 805306368.0));
  int frac;  // the low 23 bits, sign-extended
  asm("bfe.s32 %0, %1, 0, 23;" : "=r"(frac) : "r"(lo));
  __sincosf(__int2float_rn(frac) * 7.490140565847157e-07f, &s, &co);  // 2 pi / 2^23
}

__device__ inline void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  // no memory clobber: the stores are ordered before the proxy fence (also
  // volatile) that publishes them, and no generic load reads them back
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d));
}

struct TcUnit {
  TcItem it;
  TcRun run;  // the first run
  int split, P_tile, Q_tile, n_stages, n_groups;
  int rows, pairs;  // active A rows and column pairs (Q_tile VG); P_tile: lines per run when stacked
  int64_t n_begin, n_end;
};

__device__ inline TcUnit tc_unit(const TcDev &p, const TcWork &W, int u) {
  TcUnit U;
  const int item = u % W.n_items;
  U.split = u / W.n_items;
  U.it = p.items[W.item0 + item];
  U.run = p.runs[U.it.run];
  U.P_tile = p.stacked ? U.run.P : min(kTcRows, U.run.P - U.it.p0);
  U.Q_tile = min(p.Qt, U.run.Q - U.it.q0);
  U.rows = U.it.rows;
  U.pairs = U.Q_tile * p.VG;
  U.n_begin = (int64_t)U.split * W.chunk;
  U.n_end = min(p.N, U.n_begin + W.chunk);
  U.n_stages = U.n_end > U.n_begin ? (int)ceil_div(U.n_end - U.n_begin, kTcNodes) : 0;
  U.n_groups = (int)ceil_div(U.n_stages, kTcDrain);
  return U;
}

// Run (relative to the unit's first) and line of unit row `row` (TcItem).
__device__ inline void tc_row_line(const TcDev &p, const TcUnit &U, int row, int &r, int &line) {
  if (p.stacked) {
    const int lr = U.it.p0 + row;
    r = lr / U.P_tile;
    line = lr % U.P_tile;
  } else {
    r = 0;
    line = U.it.p0 + row;
  }
}

// Bounded wait that gives up at once after any earlier timeout of the block
// (the flag lives in shared memory), so a broken pipeline ends quickly.
__device__ inline bool tc_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  if (ptx::mbar_try_wait(bar, parity)) return true;
  if (*abort_flag) return false;
  if (ptx::mbar_wait(bar, parity, kTcWaitNs)) return true;
  *abort_flag = 1;
  return false;
}

// Before a group of stages ending with global stage gl is written: the MMAs
// that last read its ring slots are done.  They complete in issue order, so
// waiting for the slot of the group's last stage (stage gl - kTcStages)
// covers the earlier ones.
__device__ inline void tc_wait_group(uint64_t *empty, uint32_t gl, volatile int *abort_flag) {
  tc_wait(&empty[gl & (kTcStages - 1)], ((gl / kTcStages) & 1) ^ 1, abort_flag);
}

// Shared-memory maximum of non-negative ints over the active lanes of a
// warp: one atomic per warp instead of one per thread on the same address.
__device__ inline void tc_note_max(int *dst, int v) {
  const unsigned mask = __activemask();
  const int m = __reduce_max_sync(mask, v);
  if ((threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(dst, m);
}

// Records |kx| + |ky| + |kz| of a phase row (float bits; a NaN counts as too large).
__device__ inline void tc_note_k(int *kmax, double kx, double ky, double kz) {
  const float s = (float)(fabs(kx) + fabs(ky) + fabs(kz));
  tc_note_max(kmax, __float_as_int(s) & 0x7fffffff);
}

__device__ inline void prefetch_l1(const void *ptr) { asm volatile("prefetch.global.L1 [%0];" ::"l"(ptr)); }

// Raw node data loaded two stages before it is derived (global loads in
// flight meanwhile).  With a single rank-1 POD term (the flow and respiratory
// POD fits of the examples) the node's mode row is loaded into registers with
// it; otherwise the mode rows are prefetched into L1 for the displacement.
constexpr int kTcRegModes = 1;
struct TcRaw {
  float x, y, z, t2, phi;
  float2 m[kTcVGroup];
  float pmx[kTcRegModes], pmy[kTcRegModes], pmz[kTcRegModes];
};
// Mode count of the register-resident displacement, or -1 when the motion
// is not a single POD term of at most kTcRegModes modes.
__device__ inline int tc_reg_modes(const TcDev &p) {
  return (p.md.kind == FM_MOTION_TERMS && p.md.n_terms == 1 && p.md.terms[0].kind != FM_TERM_RESPIRATORY &&
          p.md.terms[0].n_modes <= kTcRegModes) ? p.md.terms[0].n_modes : -1;
}

__device__ inline void tc_prefetch_modes(const TcDev &p, int64_t n, TcRaw &rr) {
  if (p.md.kind != FM_MOTION_TERMS) return;
  const int rm = tc_reg_modes(p);
  if (rm >= 0) {
    const float *Phi = p.md.terms[0].modes + (size_t)n * 3 * rm;
#pragma unroll
    for (int m = 0; m < kTcRegModes; ++m) {
      rr.pmx[m] = m < rm ? __ldg(Phi + m) : 0.f;
      rr.pmy[m] = m < rm ? __ldg(Phi + rm + m) : 0.f;
      rr.pmz[m] = m < rm ? __ldg(Phi + 2 * rm + m) : 0.f;
    }
    return;
  }
  for (int k = 0; k < p.md.n_terms; ++k) {
    const fm_motion_term &T = p.md.terms[k];
    if (T.kind == FM_TERM_RESPIRATORY) continue;
    const float *Phi = T.modes + (size_t)n * 3 * T.n_modes;
    prefetch_l1(Phi);
    prefetch_l1(Phi + 3 * T.n_modes - 1);
  }
}

__device__ inline void tc_load_raw(const TcDev &p, int64_t n, TcRaw &r) {
  r.x = p.r0[3 * n + 0];
  r.y = p.r0[3 * n + 1];
  r.z = p.r0[3 * n + 2];
  r.t2 = p.T2[n];
  r.phi = p.phi[n];
#pragma unroll
  for (int v = 0; v < kTcVGroup; ++v)
    if (v < p.VG) r.m[v] = p.MM[n * p.mm_ld + v];
  tc_prefetch_modes(p, n, r);
}

// Per-run node quantities of one node into slot `slot` of a node buffer:
// moved position (in FP64 for the phase products) and the decayed,
// off-resonance rotated weights W' = (M Mxy)[n, v] exp(-t / T2) exp(i phi t).
// Nodes past the range get position 0 and zero weights, so they add nothing.
__device__ inline void tc_derive(const TcDev &p, const TcUnit &U, int64_t n, const TcRaw &r, const float *wrun,
                                 double *pos, float2 *wblk, int slot, int *rmax, const float *smodes = nullptr) {
  if (n < U.n_end) {
    float x = r.x, y = r.y, z = r.z;
    const int rm = tc_reg_modes(p);
    if (rm >= 0) {
      // motion_disp for one POD term, modes from registers (same arithmetic)
      const float *wk = wrun + p.md.slot0[0];
      float tx = 0.f, ty = 0.f, tz = 0.f;
#pragma unroll
      for (int m = 0; m < kTcRegModes; ++m) {
        const float wm = m < rm ? wk[m] : 0.f;
        tx = fmaf(r.pmx[m], wm, tx);
        ty = fmaf(r.pmy[m], wm, ty);
        tz = fmaf(r.pmz[m], wm, tz);
      }
      x = x + tx; y = y + ty; z = z + tz;
    } else if (p.md.kind == FM_MOTION_TERMS) {
      float dx, dy, dz;
      if (smodes) {
        // the single POD term's sum (motion_disp's products in its order),
        // the mode row read from the staged block
        const int rk = p.md.terms[0].n_modes;
        const float *Phi = smodes + slot * 3 * rk, *wk = wrun + p.md.slot0[0];
        dx = 0.f; dy = 0.f; dz = 0.f;
#pragma unroll 1
        for (int m = 0; m < rk; ++m) {
          const float wm = wk[m];
          dx = fmaf(Phi[m], wm, dx);
          dy = fmaf(Phi[rk + m], wm, dy);
          dz = fmaf(Phi[2 * rk + m], wm, dz);
        }
      } else {
        motion_disp(p.md, wrun, n, p.N, dx, dy, dz);
      }
      x = x + dx; y = y + dy; z = z + dz;
    } else if (p.table) {
      const float *d = p.table + ((int64_t)U.it.run * p.N + n) * 3;
      x = x + d[0]; y = y + d[1]; z = z + d[2];
    }
    pos[slot] = (double)x;
    pos[kTcBlockNodes + slot] = (double)y;
    pos[2 * kTcBlockNodes + slot] = (double)z;
    // |x| + |y| + |z| for the phase range check (a NaN counts as too large)
    tc_note_max(rmax, __float_as_int(fabsf(x) + fabsf(y) + fabsf(z)) & 0x7fffffff);
    // decay exp(-t / T2) and off-resonance rotation exp(i phi t) of a run:
    // the fast exponential of -t (1 / T2), and the phase phi t reduced in
    // cycles in FP64 before the fast sin/cos (cycles_cos_sin), as the A and B
    // tiles do (both within a few 1e-7 of the accurate functions)
    const float inv_t2 = __frcp_rn(r.t2);
    if (p.stacked) {
      // the weights without decay (B), then one D_r = decay e^{i phi t_r} row per run (A)
#pragma unroll
      for (int v = 0; v < kTcVGroup; ++v)
        if (v < p.VG) wblk[v * kWStride + slot] = r.m[v];
      for (int k = 0; k < U.it.nrun; ++k) {
        const float tg = (float)p.run_t[U.it.run + k];
        const float decay = __expf(-tg * inv_t2);
        float so, co;
        cycles_cos_sin((double)(r.phi * tg) * 0.15915494309189535, co, so);
        wblk[(p.VG + k) * kWStride + slot] = make_float2(decay * co, decay * so);
      }
    } else {
      const float tg = (float)p.run_t[U.it.run];
      const float decay = __expf(-tg * inv_t2);
      float so, co;
      cycles_cos_sin((double)(r.phi * tg) * 0.15915494309189535, co, so);
      const float er = decay * co, ei = decay * so;
#pragma unroll
      for (int v = 0; v < kTcVGroup; ++v)
        if (v < p.VG)
          wblk[v * kWStride + slot] = make_float2(r.m[v].x * er - r.m[v].y * ei, r.m[v].x * ei + r.m[v].y * er);
    }
  } else {
    pos[slot] = 0.0;
    pos[kTcBlockNodes + slot] = 0.0;
    pos[2 * kTcBlockNodes + slot] = 0.0;
    for (int v = 0; v < p.wrows; ++v) wblk[v * kWStride + slot] = make_float2(0.f, 0.f);
  }
}

// Node block blk + 1 of a unit (threads 0-127, one node each), in two calls
// some stages apart.  request: a full block with p.tma is requested by bulk
// copies into the staging area (thread 0; completion on rawfull), any other
// block by register loads.  Otherwise the block is derived into the other
// node buffer.  raw_seq counts the staged blocks (the rawfull phase).
template <bool kModes>
__device__ inline void tc_stage_block(const TcDev &p, const TcUnit &U, int tid, uint32_t blk, bool request,
                                      TcRaw &raw, uint32_t &raw_seq, unsigned char *staging, uint64_t *rawfull,
                                      const float *wrun, double *pos_next, float2 *w_next,
                                      volatile int *abort_flag, int *rmax) {
  const int64_t n0 = U.n_begin + (int64_t)(blk + 1) * kTcBlockNodes;
  const int64_t n1 = n0 + tid;
  const bool staged = p.tma && n0 + kTcBlockNodes <= U.n_end;
  float *sr0 = reinterpret_cast<float *>(staging);
  float *sT2 = sr0 + 3 * kTcBlockNodes;
  float *sphi = sT2 + kTcBlockNodes;
  float2 *sMM = reinterpret_cast<float2 *>(sphi + kTcBlockNodes);
  // the block's POD mode rows, after the raw block (TcDev::mstage)
  float *smodes = reinterpret_cast<float *>(staging + tc_raw_bytes(p.mm_ld));
  if (request) {
    if (staged) {
      if (tid == 0) {
        // the staging area's previous readers (the last block's derive) are
        // past this stage's barriers; order their reads before the copies
        ptx::fence_proxy_async_smem();
        ptx::mbar_arrive_expect_tx(rawfull, tc_raw_bytes(p.mm_ld) + (kModes ? tc_mode_bytes(p.mstage) : 0u));
        ptx::bulk_copy_g2s(sr0, p.r0 + 3 * n0, 12 * kTcBlockNodes, rawfull);
        ptx::bulk_copy_g2s(sT2, p.T2 + n0, 4 * kTcBlockNodes, rawfull);
        ptx::bulk_copy_g2s(sphi, p.phi + n0, 4 * kTcBlockNodes, rawfull);
        ptx::bulk_copy_g2s(sMM, p.MM + n0 * p.mm_ld, 8 * kTcBlockNodes * p.mm_ld, rawfull);
        // mode rows of node n0 onwards: 12 r bytes per node, n0 a multiple of
        // 16 and the rows 16-byte aligned (checked on the host)
        if (kModes && p.mstage)
          ptx::bulk_copy_g2s(smodes, p.md.terms[0].modes + n0 * p.mstage, tc_mode_bytes(p.mstage), rawfull);
      }
      if (!(kModes && p.mstage)) tc_prefetch_modes(p, n1, raw);
    } else if (n1 < U.n_end) {
      tc_load_raw(p, n1, raw);
    }
  } else {
    if (staged) {
      tc_wait(rawfull, raw_seq & 1, abort_flag);
      ++raw_seq;
      raw.x = sr0[3 * tid];
      raw.y = sr0[3 * tid + 1];
      raw.z = sr0[3 * tid + 2];
      raw.t2 = sT2[tid];
      raw.phi = sphi[tid];
#pragma unroll
      for (int v = 0; v < kTcVGroup; ++v)
        if (v < p.VG) raw.m[v] = sMM[tid * p.mm_ld + v];
    }
    tc_derive(p, U, n1, raw, wrun, pos_next, w_next, tid, rmax, kModes && staged && p.mstage ? smodes : nullptr);
  }
}

// Phase table of one stage of a factored unit: e_q(n) = exp(-2 pi i kq_q . r_n)
// for q = q0 (and q0 + 32) and the two nodes n0, n0 + 1 of this thread.
__device__ inline void tc_phase_pair(const double *pb, float2 *et, int q, int n0, double kx, double ky, double kz) {
  const double2 x = *reinterpret_cast<const double2 *>(pb + n0);
  const double2 y = *reinterpret_cast<const double2 *>(pb + kTcBlockNodes + n0);
  const double2 z = *reinterpret_cast<const double2 *>(pb + 2 * kTcBlockNodes + n0);
  float c0, s0, c1, s1;
  cycles_cos_sin(fma(kz, z.x, fma(ky, y.x, kx * x.x)), c0, s0);
  cycles_cos_sin(fma(kz, z.y, fma(ky, y.y, kx * x.y)), c1, s1);
  *reinterpret_cast<float4 *>(et + q * kEStride + n0) = make_float4(c0, -s0, c1, -s1);
}

// Tensor memory (all 512 columns of the SM).  Wide tiles (NT > 128): the
// accumulator in columns [0, NT) collects all three products.  Narrow tiles
// (NT <= 128): the B hi and lo tiles are contiguous, so one MMA with
// N = 2 NT gives A_hi B_hi in columns [0, NT) and A_hi B_lo in [NT, 2 NT), and
// a second MMA adds A_lo B_hi into [0, NT): two MMAs per K step instead of
// three.  A narrow tile's MMAs cost about as much as wide ones to issue
// (the tensor core takes ~45 cycles per MMA at N <= 64 against 128 at
// N = 256), so their count, not their size, sets the pace.  The FP32 running
// sum follows at column sum_col.  In each part, column j < NT/2 is the real
// part of pair j and column NT/2 + j its imaginary part.
constexpr uint32_t kTcTmemCols = 512;
__host__ __device__ inline bool tc_narrow(int NT) { return NT <= 128; }
__host__ __device__ inline int tc_parts(int NT) { return tc_narrow(NT) ? 2 : 1; }
__host__ __device__ inline int tc_sum_col(int NT) { return ((tc_parts(NT) * NT) + 31) & ~31; }

// Folds the accumulator (group gg, complete once accfull's phase gg & 1
// has flipped) into the running sum: sum = part_0 (+ part_1) for the first
// group, else sum + (part_0 (+ part_1)), in FP32 round-to-nearest.  Warp w
// handles TMEM lanes of quarter w % 4 and column quarter w / 4.  The next MMA
// into the accumulator is issued after a block barrier.
__device__ inline void tc_fold(const TcDev &p, uint64_t *accfull, uint32_t tmem, int gg, bool first,
                               volatile int *abort_flag) {
  const int warp = threadIdx.x >> 5;
  tc_wait(accfull, gg & 1, abort_flag);
  ptx::tc_fence_after();
  const int NT = p.NT, n_acc = tc_parts(NT), sum_col = tc_sum_col(NT);
  const int quarter = warp & 3, cq = warp >> 2;
  const int cpq = ((NT / 4 + 15) / 16) * 16;
  const int c_begin = cq * cpq, c_end = min(NT, c_begin + cpq);
  const uint32_t lanes = (uint32_t)(quarter * 32) << 16;
  for (int c0 = c_begin; c0 < c_end; c0 += 16) {
    uint32_t a[16];
    ptx::tmem_ld16(tmem + lanes + (uint32_t)c0, a);
    ptx::tmem_wait_ld();
    // the other accumulators, then the running sum, in halves of 8 columns
    for (int k = 1; k <= n_acc; ++k) {
      if (k == n_acc && first) break;
      const int col = (k == n_acc ? sum_col : k * NT) + c0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t r[8];
        ptx::tmem_ld8(tmem + lanes + (uint32_t)(col + 8 * h), r);
        ptx::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i)
          a[8 * h + i] = k == n_acc ? __float_as_uint(__uint_as_float(r[i]) + __uint_as_float(a[8 * h + i]))
                                    : __float_as_uint(__uint_as_float(a[8 * h + i]) + __uint_as_float(r[i]));
      }
    }
    ptx::tmem_st16(tmem + lanes + (uint32_t)(sum_col + c0), a);
  }
  ptx::tmem_wait_st();
  ptx::tc_fence_before();
}

// Writes the unit's result: running sum (when earlier groups were folded) +
// the accumulator of the last group gg (its parts added in order), to the
// output samples.  Warp w reads TMEM lanes of quarter w % 4 and every fourth
// chunk of 8 pairs starting at w / 4.
__device__ inline void tc_final(const TcDev &p, const TcWork &W, const TcUnit &U, uint64_t *accfull,
                                uint32_t tmem, int gg, bool has_sum, volatile int *abort_flag) {
  const int tid = threadIdx.x, warp = tid >> 5;
  tc_wait(accfull, gg & 1, abort_flag);
  ptx::tc_fence_after();
  const int quarter = warp & 3;
  const int row = quarter * 32 + (tid & 31);
  const int NH = p.NT >> 1;
  const bool row_ok = row < U.rows;
  float2 *dst = W.out + (int64_t)U.split * p.S * p.V;
  // every run of a stacked unit shares the column pairs
  int r_row = 0, line = 0;
  if (row_ok) tc_row_line(p, U, row, r_row, line);
  const int qvg = U.Q_tile * p.VG;
  const int start = row_ok ? p.runs[U.it.run + r_row].start : 0;
  const int s_row = start + (U.run.factored ? line * p.n_kz + U.it.q0 : line);
  const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16);
  const int n_acc = tc_parts(p.NT), AW = p.NT, sum_col = tc_sum_col(p.NT);
  for (int c0 = (warp >> 2) * 8; c0 < NH; c0 += 32) {
    uint32_t r[8], m[8];
    ptx::tmem_ld8(taddr + (uint32_t)c0, r);
    ptx::tmem_ld8(taddr + (uint32_t)(NH + c0), m);
    ptx::tmem_wait_ld();
    float re8[8], im8[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      re8[i] = __uint_as_float(r[i]);
      im8[i] = __uint_as_float(m[i]);
    }
    for (int k = 1; k < n_acc; ++k) {
      ptx::tmem_ld8(taddr + (uint32_t)(k * AW + c0), r);
      ptx::tmem_ld8(taddr + (uint32_t)(k * AW + NH + c0), m);
      ptx::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        re8[i] = re8[i] + __uint_as_float(r[i]);
        im8[i] = im8[i] + __uint_as_float(m[i]);
      }
    }
    if (has_sum) {
      ptx::tmem_ld8(taddr + (uint32_t)(sum_col + c0), r);
      ptx::tmem_ld8(taddr + (uint32_t)(sum_col + NH + c0), m);
      ptx::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        re8[i] = __uint_as_float(r[i]) + re8[i];
        im8[i] = __uint_as_float(m[i]) + im8[i];
      }
    }
    if (!row_ok) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float re = re8[i], im = im8[i];
      const int jj = c0 + i;  // pair (q, v)
      if (jj >= qvg) continue;
      const int q = jj / p.VG, vv = jj % p.VG;
      if (q < U.Q_tile) dst[(int64_t)(s_row + q) * p.V + p.v0 + vv] = make_float2(re, im);
    }
  }
  ptx::tc_fence_before();
}

// MMAs of one stage (global stage index g, stage-local st of a unit with
// n_stages stages): A_hi B_hi + A_hi B_lo + A_lo B_hi over the two K steps
// into the accumulator (overwritten at a group's first stage); the stage's
// shared memory is released by a commit to empty[s], and the group's
// accumulator by a commit to accfull after the group's last stage.  kFence:
// the call orders its MMAs after the group barrier itself (otherwise the
// caller has done so once for the group).  Called by
// the whole issuing warp (warp 7): the descriptors are warp-uniform, and
// lane 0 issues the MMAs and commits (it is the thread whose operations the
// commits track).
template <bool kFence>
__device__ inline void tc_issue(const TcSmem &L, uint32_t sbase, uint32_t tmem, uint32_t idesc, int NT,
                                uint64_t *empty, uint64_t *accfull, uint32_t s, uint32_t st, uint32_t n_stages,
                                uint32_t lane) {
  if (kFence) ptx::tc_fence_after();
  // Descriptors (ptx::smem_desc_sw64): the tiles of a stage differ only in
  // the start-address field, address / 16 (below 2^14 in shared memory, and
  // every tile and stage offset a multiple of 16), so the stage's field is
  // formed once and each tile's is one add; the high word is constant.
  const uint32_t f0 = ((sbase + L.stages + s * L.stage_bytes) >> 4) | (1u << 16);  // + LBO
  constexpr uint32_t kDescHi = (512u >> 4) | (1u << 14) | (4u << 29);            // SBO, version, 64B swizzle
  // the drain group's first stage overwrites the accumulator; everything is
  // computed before the first MMA goes out
  const uint32_t acc0 = (st % kTcDrain) == 0 ? 0u : 1u;
  uint64_t ad[2][2], bd[2][2];
#pragma unroll
  for (int ks = 0; ks < 2; ++ks) {
    // K step ks: elements 16 ks .. 16 ks + 15, bytes 32 ks .. of every row
    ad[ks][0] = ((uint64_t)kDescHi << 32) | (f0 + ((L.a_hi + ks * 32) >> 4));
    ad[ks][1] = ((uint64_t)kDescHi << 32) | (f0 + ((L.a_lo + ks * 32) >> 4));
    bd[ks][0] = ((uint64_t)kDescHi << 32) | (f0 + ((L.b_hi + ks * 32) >> 4));
    bd[ks][1] = ((uint64_t)kDescHi << 32) | (f0 + ((L.b_lo + ks * 32) >> 4));
  }
  if (tc_narrow(NT)) {
    // A_hi [B_hi; B_lo] (N = 2 NT, both tiles from b_hi on), then A_lo B_hi
    const uint32_t idesc2 = ptx::idesc_bf16_f32(kTcRows, 2 * NT);
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      ptx::mma_bf16_lane0(tmem, ad[ks][0], bd[ks][0], idesc2, ks == 0 ? acc0 : 1u, lane);
      ptx::mma_bf16_lane0(tmem, ad[ks][1], bd[ks][0], idesc, 1u, lane);
    }
  } else {
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      ptx::mma_bf16_lane0(tmem, ad[ks][0], bd[ks][0], idesc, ks == 0 ? acc0 : 1u, lane);
      ptx::mma_bf16_lane0(tmem, ad[ks][0], bd[ks][1], idesc, 1u, lane);
      ptx::mma_bf16_lane0(tmem, ad[ks][1], bd[ks][0], idesc, 1u, lane);
    }
  }
  ptx::mma_commit_lane0(&empty[s], lane);
  if ((st % kTcDrain) == kTcDrain - 1 || st == n_stages - 1) ptx::mma_commit_lane0(accfull, lane);
}

// kModes: some entry stages POD mode rows with its node blocks (TcDev::mstage);
// the instance without that code is the one every other launch uses.
template <bool kModes>
__global__ void __launch_bounds__(kTcThreads, 1) signal_tc_kernel(const __grid_constant__ TcBatchDev B) {
  extern __shared__ __align__(1024) unsigned char smem[];
  // work sizes come from the device-side plan, so the launch needs no host
  // synchronisation (and can be captured in a CUDA graph)
  const int n_units = B.offsets[B.n_entries];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  uint64_t *empty = reinterpret_cast<uint64_t *>(smem + kTcBars);
  uint64_t *gempty = empty + kTcStages;  // the generic ring's slots
  uint64_t *accfull = gempty + kTcRingGen;
  uint64_t *done = accfull + 1;
  uint64_t *rawfull = done + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kTcMisc);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + kTcMisc + 4);
  // largest |kx|+|ky|+|kz| of the unit's phases and |x|+|y|+|z| of its moved
  // nodes (float bits), for the check that the fixed-point phase reduction
  // applies (cycles_cos_sin)
  int *kmax = reinterpret_cast<int *>(smem + kTcMisc + 8);
  int *rmax = reinterpret_cast<int *>(smem + kTcMisc + 12);
  const uint32_t sbase = ptx::smem_addr(smem);

  if (tid == 0) {
    for (int s = 0; s < kTcStages + kTcRingGen; ++s) ptx::mbar_init(&empty[s], 1);
    ptx::mbar_init(accfull, 1);
    ptx::mbar_init(done, 1);
    ptx::mbar_init(rawfull, 1);
    *abort_flag = 0;
    *kmax = 0;
    *rmax = 0;
    ptx::fence_mbar_init();
  }
  if (warp == 0) ptx::tmem_alloc(tmem_slot, kTcTmemCols);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = tmem_slot[0];

  // Roles (warp-uniform).  Warps 0-7 write A: rows 32 (w >> 1) + lane, nodes
  // 8 (w & 1) .. + 7 of every stage.  Warps 8-15 write B: pairs
  // 32 ((w - 8) >> 1) + lane, same node halves, and the next stage's phase
  // table.  Threads 0-127 also derive the node blocks.  One thread of warp 7
  // issues a stage's MMAs after the block barrier that follows the stage
  // (every writer has fenced its stores to the async proxy by then).  Both
  // roles pass the same barriers and drains in the same order.
  const bool a_role = warp < 8;
  const int rw = a_role ? warp : warp - 8;
  const int row = (rw >> 1) * 32 + lane;  // A row or B pair
  const int half = rw & 1;                // nodes 8 half .. 8 half + 7 of a stage
  const bool loader = tid < kTcBlockNodes;
  const bool issuer = tid == 7 * 32;  // lane 0 of warp 7: the thread that issues every MMA
  // phase-table thread: q = (tid - 256) / 8 (+ 32), nodes 2 ((tid - 256) % 8) + {0, 1}
  const int tq = (tid - 256) >> 3, tn = ((tid - 256) & 7) * 2;
  uint32_t gst = 0, raw_seq = 0;
  uint32_t gsg = 0;  // stages of generic units so far (their ring's counter)
  int gbase = 0;
  TcRaw raw;
  for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
    // the unit's entry: offsets[e] <= u < offsets[e + 1]
    int e_lo = 0, e_hi = B.n_entries;
    while (e_hi - e_lo > 1) {
      const int mid = (e_lo + e_hi) >> 1;
      if (B.offsets[mid] <= u) e_lo = mid; else e_hi = mid;
    }
    const TcDev &p = B.entries[e_lo];
    const TcWork W = tc_work(p);
    const int NT = p.NT, NH = NT >> 1, VG = p.VG, Qt = p.Qt, WR = p.wrows;
    const TcSmem L = tc_smem_layout(NT, WR, Qt, p.kind == 0 ? kTcStages : kTcRingGen);
    double *pos_all = reinterpret_cast<double *>(smem + L.pos);
    float2 *w_all = reinterpret_cast<float2 *>(smem + L.w);
    float2 *etab = reinterpret_cast<float2 *>(smem + L.etab);
    const uint32_t sstages = sbase + L.stages;
    const uint32_t idesc = ptx::idesc_bf16_f32(kTcRows, NT);
    // operand addresses inside a stage: the thread's first 8-K chunk; the
    // second chunk is d_k2 = +/-16 bytes from it (swizzled chunk positions
    // 2 half and 2 half + 1 differ in their lowest bit), the lo tile d_lo
    // bytes on and (B) the imaginary row block d_im bytes on
    const uint32_t o_hi = (a_role ? L.a_hi : L.b_hi) + sw64_offset(row, 16 * half);
    const int d_k2 = ((((2 * half) ^ (row >> 1)) & 1) != 0) ? -16 : 16;
    const uint32_t d_lo = a_role ? L.a_lo - L.a_hi : L.b_lo - L.b_hi;
    const uint32_t d_im = (uint32_t)NH * 64;
    const bool b_rows = row < NH;
    const TcUnit U = tc_unit(p, W, u - B.offsets[e_lo]);
    const bool fac = U.run.factored != 0;
    const uint32_t nst = (uint32_t)U.n_stages;
    ptx::named_barrier(1, kTcProducers);  // the previous unit's readers are done
    // per-unit row data in registers
    double kx0 = 0, ky0 = 0, kz0 = 0, kx1 = 0, ky1 = 0, kz1 = 0;  // A: kp of the row; B: kq of q and q + 32
    int bq = 0, bw = 0;  // B: phase-table row and weight row of the pair
    int a_drow = 0;      // A of a stacked unit: the row's D row in the node buffer
    if (a_role) {
      if (row < U.rows) {
        // the row's run (r = 0 unless stacked) and line
        int r, line;
        tc_row_line(p, U, row, r, line);
        a_drow = VG + r;
        const int start = r == 0 ? U.run.start : p.runs[U.it.run + r].start;
        const int s_p = start + (fac ? line * p.n_kz : line);
        kx0 = p.kx[s_p];
        ky0 = p.ky[s_p];
        kz0 = p.kz[s_p];
        if (nst > 0) tc_note_k(kmax, kx0, ky0, kz0);
      }
    } else {
      if (row < U.pairs) {
        bq = row / VG;
        bw = row % VG;
      }
      if (fac) {
        const int s_0 = U.run.start;
        if (tq < U.Q_tile) {
          const int s_q = U.run.start + U.it.q0 + tq;
          kx0 = (double)p.kx[s_q] - (double)p.kx[s_0];
          ky0 = (double)p.ky[s_q] - (double)p.ky[s_0];
          kz0 = (double)p.kz[s_q] - (double)p.kz[s_0];
          if (nst > 0) tc_note_k(kmax, kx0, ky0, kz0);
        }
        if (tq + 32 < U.Q_tile) {
          const int s_q = U.run.start + U.it.q0 + tq + 32;
          kx1 = (double)p.kx[s_q] - (double)p.kx[s_0];
          ky1 = (double)p.ky[s_q] - (double)p.ky[s_0];
          kz1 = (double)p.kz[s_q] - (double)p.kz[s_0];
          if (nst > 0) tc_note_k(kmax, kx1, ky1, kz1);
        }
      }
    }
    const bool t_on0 = !a_role && fac && tq < U.Q_tile, t_on1 = !a_role && fac && tq + 32 < U.Q_tile;
    const float *wrun = p.weights ? p.weights + (int64_t)U.it.run * p.md.slots : nullptr;
    const uint32_t n_blocks = (nst + kTcStagesPerBlock - 1) / kTcStagesPerBlock;
    // prologue: node block 0 into buffer 0
    if (loader && nst > 0) {
      const int64_t n = U.n_begin + tid;
      if (n < U.n_end) tc_load_raw(p, n, raw);
      tc_derive(p, U, n, raw, wrun, pos_all, w_all, tid, rmax);
    }
    ptx::named_barrier(1, kTcProducers);  // block 0 is visible
    // phase tables of the first group's stages (block 0, buffers 0 ..)
    for (uint32_t st = 0; st < kTcFacGroup && st < nst; ++st) {
      float2 *et = etab + st * Qt * kEStride;
      if (t_on0) tc_phase_pair(pos_all + st * kTcNodes, et, tq, tn, kx0, ky0, kz0);
      if (t_on1) tc_phase_pair(pos_all + st * kTcNodes, et, tq + 32, tn, kx1, ky1, kz1);
    }
    // the first group's tables are read by other warps than their writers
    if (fac) ptx::named_barrier(1, kTcProducers);
    const uint32_t g0 = gst, gg0 = gsg;
    int next_drain = 0;
    if (!fac) {
      // ------------------------------------------- generic unit, all warps --
      // B is only the weights of the unit's VG columns (NT = 16), so every
      // warp writes A: rows 32 (w % 4) + lane, nodes 4 (w / 4) .. + 3 of a
      // stage; threads 0-127 also write one B element (pair tid % 8, node
      // tid / 8).  Pairs past VG hold values no output reads.
      const int grow = (warp & 3) * 32 + lane, gc = warp >> 2;
      double gx = 0, gy = 0, gz = 0;
      if (grow < U.P_tile) {
        const int s_p = U.run.start + U.it.p0 + grow;
        gx = p.kx[s_p];
        gy = p.ky[s_p];
        gz = p.kz[s_p];
        if (nst > 0) tc_note_k(kmax, gx, gy, gz);
      }
      const bool g_active = (warp & 3) * 32 < U.P_tile;
      const uint32_t ga0 = L.a_hi + sw64_offset(grow, 8 * gc);
      const uint32_t gl0 = L.a_lo + sw64_offset(grow, 8 * gc);
      const int gpair = tid & 7, gnode = tid >> 3;
      const bool g_b = tid < kTcRows && gpair < NH;
      const int gv = gpair < VG ? gpair : 0;
      const uint32_t gbr = sw64_offset(gpair, 2 * gnode), gbi = sw64_offset(NH + gpair, 2 * gnode);
      // The MMAs of a generic stage are small (N = 16), so the producers
      // write kTcGenGroup stages between barriers and the issuer sends them
      // together: one barrier per group instead of one per stage.  Groups
      // divide the 8-stage node blocks, so a block derived at stage 6 is
      // visible after its group's barrier, before any stage of it is read.
      for (uint32_t sg = 0; sg < nst; sg += kTcGenGroup) {
        const uint32_t s_end = min(nst, sg + (uint32_t)kTcGenGroup);
        for (uint32_t st = sg; st < s_end; ++st) {
          const uint32_t g = gg0 + st, s = g & (kTcRingGen - 1);
          const uint32_t j = st & (kTcStagesPerBlock - 1), blk = st / kTcStagesPerBlock, buf = blk & 1;
          if (loader && blk + 1 < n_blocks && (j == 0 || j == 4))
            tc_stage_block<kModes>(p, U, tid, blk, j == 0, raw, raw_seq, smem + L.raw, rawfull, wrun,
                           pos_all + (buf ^ 1) * 3 * kTcBlockNodes, w_all + (buf ^ 1) * WR * kWStride, abort_flag,
                           rmax);
          // the MMAs that last read stage s were sent at an earlier barrier
          tc_wait(&gempty[s], ((g / kTcRingGen) & 1) ^ 1, abort_flag);
          const uint32_t stg = sstages + s * L.stage_bytes;
          if (g_active) {
            const double *px = pos_all + buf * 3 * kTcBlockNodes + j * kTcNodes + 4 * gc;
            uint32_t h[4], l[4];
#pragma unroll
            for (int u4 = 0; u4 < 4; u4 += 2) {
              const double2 x = *reinterpret_cast<const double2 *>(px + u4);
              const double2 y = *reinterpret_cast<const double2 *>(px + kTcBlockNodes + u4);
              const double2 z = *reinterpret_cast<const double2 *>(px + 2 * kTcBlockNodes + u4);
              float c0, s0, c1, s1;
              cycles_cos_sin(fma(gz, z.x, fma(gy, y.x, gx * x.x)), c0, s0);
              cycles_cos_sin(fma(gz, z.y, fma(gy, y.y, gx * x.y)), c1, s1);
              split_pair(c0, s0, h[u4], l[u4]);
              split_pair(c1, s1, h[u4 + 1], l[u4 + 1]);
            }
            st_shared_v4(stg + ga0, h[0], h[1], h[2], h[3]);
            st_shared_v4(stg + gl0, l[0], l[1], l[2], l[3]);
          }
          if (g_b) {
            const float2 wv = w_all[(buf * WR + gv) * kWStride + j * kTcNodes + gnode];
            uint32_t hb, lb;
            split_pair(wv.x, wv.y, hb, lb);
            const uint32_t hm = __byte_perm(hb, 0u, 0x1032) ^ 0x80000000u, lm = __byte_perm(lb, 0u, 0x1032) ^ 0x80000000u;
            asm volatile("st.shared.b32 [%0], %1;" ::"r"(stg + L.b_hi + gbr), "r"(hb));
            asm volatile("st.shared.b32 [%0], %1;" ::"r"(stg + L.b_lo + gbr), "r"(lb));
            asm volatile("st.shared.b32 [%0], %1;" ::"r"(stg + L.b_hi + gbi), "r"(hm));
            asm volatile("st.shared.b32 [%0], %1;" ::"r"(stg + L.b_lo + gbi), "r"(lm));
          }
        }
        ptx::fence_proxy_async_smem();
        // every writer of the group is done: its MMAs go out now
        ptx::named_barrier(1, kTcProducers);
        if (warp == 7) {
          ptx::tc_fence_after();
          for (uint32_t st = sg; st < s_end; ++st)
            tc_issue<false>(L, sbase, tmem, idesc, NT, gempty, accfull, (gg0 + st) & (kTcRingGen - 1), st, nst, lane);
        }
        // an accumulation group ended with this group: fold it before the
        // next group's MMAs (which go out at the next barrier)
        if (s_end < nst && (s_end & (kTcDrain - 1)) == 0) {
          tc_fold(p, accfull, tmem, gbase + next_drain, next_drain == 0, abort_flag);
          ++next_drain;
        }
      }
    } else if (a_role) {
      // ------------------------------------------------------- A rows --
      // kTcFacGroup stages between barriers; the group's MMAs go out at its
      // barrier.  Node block blk + 1 is requested at j == 2 and derived at
      // j == 4 into the other buffer: that buffer's readers (block blk - 1)
      // are done, and the phase tables of block blk + 1's first stages are
      // computed after the barrier that ends the derive's group.
      const bool active = (rw >> 1) * 32 < U.rows;
      for (uint32_t sg = 0; sg < nst; sg += kTcFacGroup) {
        const uint32_t s_end = min(nst, sg + (uint32_t)kTcFacGroup);
        // a group's stages lie in one node block (groups divide the blocks)
        const uint32_t jg = sg & (kTcStagesPerBlock - 1), blk = sg / kTcStagesPerBlock, buf = blk & 1;
        if (loader && blk + 1 < n_blocks && (jg == 2 || jg == 4))
          tc_stage_block<kModes>(p, U, tid, blk, jg == 2, raw, raw_seq, smem + L.raw, rawfull, wrun,
                         pos_all + (buf ^ 1) * 3 * kTcBlockNodes, w_all + (buf ^ 1) * WR * kWStride, abort_flag,
                         rmax);
        tc_wait_group(empty, g0 + s_end - 1, abort_flag);
#pragma unroll
        for (uint32_t i = 0; i < (uint32_t)kTcFacGroup; ++i) {
          const uint32_t st = sg + i;
          if (st >= s_end) break;
          const uint32_t s = (g0 + st) & (kTcStages - 1), j = jg + i;
          if (active) {
            // A'[row][2n..2n+1] = (Re A, -Im A) = (cos, sin) of 2 pi kp . r_n;
            // in a stacked unit A is multiplied by the row's run factor D_r(n):
            // (Re, -Im) of (cos - i sin)(dr + i di) = (cos dr + sin di, sin dr - cos di)
            const uint32_t stg = sstages + s * L.stage_bytes;
            const double *px = pos_all + buf * 3 * kTcBlockNodes + j * kTcNodes + 8 * half;
            uint32_t h[8], l[8];
            if (p.stacked) {
              const float4 *dp = reinterpret_cast<const float4 *>(w_all + (buf * WR + a_drow) * kWStride +
                                                                  j * kTcNodes + 8 * half);
#pragma unroll
              for (int u4 = 0; u4 < 8; u4 += 2) {
                const double2 x = *reinterpret_cast<const double2 *>(px + u4);
                const double2 y = *reinterpret_cast<const double2 *>(px + kTcBlockNodes + u4);
                const double2 z = *reinterpret_cast<const double2 *>(px + 2 * kTcBlockNodes + u4);
                float c0, s0, c1, s1;
                cycles_cos_sin(fma(kz0, z.x, fma(ky0, y.x, kx0 * x.x)), c0, s0);
                cycles_cos_sin(fma(kz0, z.y, fma(ky0, y.y, kx0 * x.y)), c1, s1);
                const float4 d = dp[u4 >> 1];
                split_pair(fmaf(c0, d.x, s0 * d.y), fmaf(s0, d.x, -(c0 * d.y)), h[u4], l[u4]);
                split_pair(fmaf(c1, d.z, s1 * d.w), fmaf(s1, d.z, -(c1 * d.w)), h[u4 + 1], l[u4 + 1]);
              }
            } else {
#pragma unroll
              for (int u4 = 0; u4 < 8; u4 += 2) {
                const double2 x = *reinterpret_cast<const double2 *>(px + u4);
                const double2 y = *reinterpret_cast<const double2 *>(px + kTcBlockNodes + u4);
                const double2 z = *reinterpret_cast<const double2 *>(px + 2 * kTcBlockNodes + u4);
                float c0, s0, c1, s1;
                cycles_cos_sin(fma(kz0, z.x, fma(ky0, y.x, kx0 * x.x)), c0, s0);
                cycles_cos_sin(fma(kz0, z.y, fma(ky0, y.y, kx0 * x.y)), c1, s1);
                split_pair(c0, s0, h[u4], l[u4]);
                split_pair(c1, s1, h[u4 + 1], l[u4 + 1]);
              }
            }
            const uint32_t a_st = stg + o_hi;
            st_shared_v4(a_st, h[0], h[1], h[2], h[3]);
            st_shared_v4(a_st + d_k2, h[4], h[5], h[6], h[7]);
            st_shared_v4(a_st + d_lo, l[0], l[1], l[2], l[3]);
            st_shared_v4(a_st + d_lo + d_k2, l[4], l[5], l[6], l[7]);
          }
        }
        ptx::fence_proxy_async_smem();
        // every writer of the group is done (and its phase tables of the next
        // group are visible after this barrier): its MMAs go out now
        ptx::named_barrier(1, kTcProducers);
        if (warp == 7)
          for (uint32_t st = sg; st < s_end; ++st)
            tc_issue<true>(L, sbase, tmem, idesc, NT, empty, accfull, (g0 + st) % kTcStages, st, nst, lane);
        // an accumulation group ended with this group: fold it before the
        // next group's MMAs go out
        if (s_end < nst && (s_end & (kTcDrain - 1)) == 0) {
          tc_fold(p, accfull, tmem, gbase + next_drain, next_drain == 0, abort_flag);
          ++next_drain;
        }
      }
    } else {
      // ------------------------------------------------------- B rows --
      for (uint32_t sg = 0; sg < nst; sg += kTcFacGroup) {
        const uint32_t s_end = min(nst, sg + (uint32_t)kTcFacGroup);
        const uint32_t jg = sg & (kTcStagesPerBlock - 1), buf = (sg / kTcStagesPerBlock) & 1;
        tc_wait_group(empty, g0 + s_end - 1, abort_flag);
#pragma unroll
        for (uint32_t i = 0; i < (uint32_t)kTcFacGroup; ++i) {
          const uint32_t st = sg + i;
          if (st >= s_end) break;
          const uint32_t s = (g0 + st) & (kTcStages - 1), j = jg + i;
          // B'^T rows: re row `row` = (Re B, Im B), im row NT/2 + row =
          // (Im B, -Re B), B = e_q(n) W'(n, v).  Pairs past Q_tile VG hold
          // values no output reads.  Threads past the tile's NT/2 pairs have
          // no B element (their warps only take part in the phase table).
          if (b_rows) {
          const float4 *wp =
              reinterpret_cast<const float4 *>(w_all + (buf * WR + bw) * kWStride + j * kTcNodes + 8 * half);
          float br[8], bi[8];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float4 w2 = wp[i];
            br[2 * i] = w2.x; bi[2 * i] = w2.y; br[2 * i + 1] = w2.z; bi[2 * i + 1] = w2.w;
          }
          {
            const float4 *ep = reinterpret_cast<const float4 *>(etab + ((st & (kTcEBufs - 1)) * Qt + bq) * kEStride +
                                                                8 * half);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const float4 e2 = ep[i];
              const float wr0 = br[2 * i], wi0 = bi[2 * i], wr1 = br[2 * i + 1], wi1 = bi[2 * i + 1];
              br[2 * i] = e2.x * wr0 - e2.y * wi0;
              bi[2 * i] = e2.x * wi0 + e2.y * wr0;
              br[2 * i + 1] = e2.z * wr1 - e2.w * wi1;
              bi[2 * i + 1] = e2.z * wi1 + e2.w * wr1;
            }
          }
          uint32_t hr[8], lr[8], hm[8], lm[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            split_pair(br[i], bi[i], hr[i], lr[i]);
            hm[i] = __byte_perm(hr[i], 0u, 0x1032) ^ 0x80000000u;
            lm[i] = __byte_perm(lr[i], 0u, 0x1032) ^ 0x80000000u;
          }
          {
            const uint32_t stg = sstages + s * L.stage_bytes;
            const uint32_t b_st = stg + o_hi;
            st_shared_v4(b_st, hr[0], hr[1], hr[2], hr[3]);
            st_shared_v4(b_st + d_k2, hr[4], hr[5], hr[6], hr[7]);
            st_shared_v4(b_st + d_lo, lr[0], lr[1], lr[2], lr[3]);
            st_shared_v4(b_st + d_lo + d_k2, lr[4], lr[5], lr[6], lr[7]);
            st_shared_v4(b_st + d_im, hm[0], hm[1], hm[2], hm[3]);
            st_shared_v4(b_st + d_im + d_k2, hm[4], hm[5], hm[6], hm[7]);
            st_shared_v4(b_st + d_im + d_lo, lm[0], lm[1], lm[2], lm[3]);
            st_shared_v4(b_st + d_im + d_lo + d_k2, lm[4], lm[5], lm[6], lm[7]);
          }
          }  // b_rows
          // the phase table of stage st + kTcFacGroup (next group) into its
          // buffer, whose last readers (stage st - kTcFacGroup) are past the
          // previous group's barrier
          if (t_on0 && st + kTcFacGroup < nst) {
            const uint32_t st1 = st + kTcFacGroup;
            const double *pb = pos_all + ((st1 / kTcStagesPerBlock) & 1) * 3 * kTcBlockNodes +
                               (st1 & (kTcStagesPerBlock - 1)) * kTcNodes;
            float2 *et = etab + (st1 & (kTcEBufs - 1)) * Qt * kEStride;
            tc_phase_pair(pb, et, tq, tn, kx0, ky0, kz0);
            if (t_on1) tc_phase_pair(pb, et, tq + 32, tn, kx1, ky1, kz1);
          }
        }
        ptx::fence_proxy_async_smem();
        ptx::named_barrier(1, kTcProducers);
        if (s_end < nst && (s_end & (kTcDrain - 1)) == 0) {
          tc_fold(p, accfull, tmem, gbase + next_drain, next_drain == 0, abort_flag);
          ++next_drain;
        }
      }
    }
    if (fac) gst = g0 + nst;
    else gsg = gg0 + nst;
    if (nst > 0) {
      ptx::named_barrier(1, kTcProducers);  // the unit's last stage is written
      if (tid == 0) {
        // every phase of the unit had |k . r| <= kmax rmax: the fixed-point
        // reduction holds below 2^28 cycles (2^27 leaves a margin)
        if (!((double)__int_as_float(*kmax) * (double)__int_as_float(*rmax) < 134217728.0))
          atomicOr(p.error, kErrPhaseRange);
        *kmax = 0;
        *rmax = 0;
      }
    }
    if (U.n_groups > 0) tc_final(p, W, U, accfull, tmem, gbase + U.n_groups - 1, U.n_groups > 1, abort_flag);
    if (U.n_groups == 0 && tid < U.rows) {
      // no nodes in this split: its share of the tile is zero
      float2 *dst = W.out + (int64_t)U.split * p.S * p.V;
      int r, line;
      tc_row_line(p, U, tid, r, line);
      const int start = p.runs[U.it.run + r].start;
      const int s_row = start + (fac ? line * p.n_kz + U.it.q0 : line);
      for (int q = 0; q < U.Q_tile; ++q)
        for (int v = 0; v < VG; ++v) dst[(int64_t)(s_row + q) * p.V + p.v0 + v] = make_float2(0.f, 0.f);
    }
    gbase += U.n_groups;
  }
  if (issuer) {
    // all issued MMAs complete before the tensor memory is released
    ptx::mma_commit(done);
    if (!ptx::mbar_wait(done, 0, kTcWaitNs)) *abort_flag = 1;
  }
  ptx::tc_fence_before();
  __syncthreads();
  // a wait that ran out is reported for every problem of the launch
  if (*abort_flag)
    for (int e = tid; e < B.n_entries; e += kTcThreads) atomicOr(B.entries[e].error, kErrTimeout);
  if (warp == 0) {
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, kTcTmemCols);
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

// Runs can be stacked into one unit when the positions do not depend on the
// run (no motion) and every run is a factored slab of the full (lines x kz)
// shape with the same kz offsets kq = k(q) - k(first sample), exactly.
// `flag` starts non-zero; any run that breaks a condition clears it.
__global__ void tc_stack_check_kernel(const float *__restrict__ kx, const float *__restrict__ ky,
                                      const float *__restrict__ kz, const TcRun *__restrict__ runs,
                                      const int *__restrict__ counts, int n_lines, int n_kz, int *__restrict__ flag) {
  const int n_runs = counts[0];
  if (n_runs <= 0) return;
  const int s0 = runs[0].start;
  const int64_t total = (int64_t)n_runs * n_kz;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int g = (int)(idx / n_kz), q = (int)(idx % n_kz);
    const TcRun r = runs[g];
    bool ok = r.factored && r.P == n_lines && r.Q == n_kz;
    if (ok) {
      const int a = r.start, b = s0;
      ok = ((double)kx[a + q] - (double)kx[a]) == ((double)kx[b + q] - (double)kx[b]) &&
           ((double)ky[a + q] - (double)ky[a]) == ((double)ky[b + q] - (double)ky[b]) &&
           ((double)kz[a + q] - (double)kz[a]) == ((double)kz[b + q] - (double)kz[b]);
    }
    if (!ok) atomicExch(flag, 0);
  }
}

// Item counts per run, factored runs in one list and the rest in another.
// With stacking (stack != nullptr and *stack set) the runs' P lines are laid
// end to end and cut into items of RU lines: run g opens the items whose
// first line falls in it.
__device__ inline int64_t tc_packed_first(int64_t g, int P, int RU) { return ceil_div(g * P, (int64_t)RU); }
__global__ void tc_count_kernel(const TcRun *__restrict__ runs, const int *__restrict__ counts, int Qt,
                                int *__restrict__ nf, int *__restrict__ ng, int64_t S, const int *__restrict__ stack,
                                int P, int RU) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = counts[0];
  if (g > S) return;
  if (g >= n) {
    nf[g] = 0;
    ng[g] = 0;
    return;
  }
  if (stack && *stack) {
    nf[g] = (int)(tc_packed_first(g + 1, P, RU) - tc_packed_first(g, P, RU));
    ng[g] = 0;
    return;
  }
  const TcRun r = runs[g];
  const int items = (int)(ceil_div(r.P, kTcRows) * ceil_div(r.Q, r.factored ? Qt : 1));
  nf[g] = r.factored ? items : 0;
  ng[g] = r.factored ? 0 : items;
}

// Items of one Mxy column group: factored first, then generic; their counts
// go to plan[2] and plan[3].
__global__ void tc_fill_kernel(const TcRun *__restrict__ runs, const int *__restrict__ counts, int Qt,
                               const int *__restrict__ of, const int *__restrict__ og, TcItem *__restrict__ items,
                               int *__restrict__ plan, const int *__restrict__ stack, int P, int RU) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = counts[0];
  if (g > n) return;
  if (g == n) {
    plan[2] = of[n];
    plan[3] = og[n];
    return;
  }
  if (stack && *stack) {
    const int64_t i0 = tc_packed_first(g, P, RU), i1 = tc_packed_first(g + 1, P, RU);
    const int64_t total = (int64_t)n * P;
    for (int64_t i = i0; i < i1; ++i) {
      const int64_t L0 = i * RU;
      TcItem t;
      t.run = g;
      t.p0 = (int)(L0 - (int64_t)g * P);
      t.q0 = 0;
      t.rows = (int)((total - L0) < RU ? (total - L0) : RU);
      t.nrun = (int)((L0 + t.rows - 1) / P - g + 1);
      items[of[g] + (i - i0)] = t;
    }
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
      t.nrun = 1;
      t.rows = (r.P - t.p0) < kTcRows ? (r.P - t.p0) : kTcRows;
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

// Splits of one problem, shared by all its column groups (plan rows of 8
// ints): from the node count per split when tuned, else balanced over the SMs.
__global__ void tc_plan_kernel(int *__restrict__ plan, int n_groups, int64_t N, int max_splits, int split_nodes) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int64_t items = 0;
  for (int g = 0; g < n_groups; ++g) items += plan[8 * g + 2] + plan[8 * g + 3];
  int splits;
  if (split_nodes > 0) {
    const int64_t s = ceil_div(N, (int64_t)split_nodes);
    splits = (int)(s < 1 ? 1 : (s > max_splits ? max_splits : s));
  } else {
    splits = tc_choose_splits(items, N, max_splits);
  }
  const int chunk = (int)(ceil_div(ceil_div(N, splits), kTcNodes) * kTcNodes);
  for (int g = 0; g < n_groups; ++g) {
    plan[8 * g + 4] = splits;
    plan[8 * g + 5] = chunk;
  }
}

// Running unit counts of the launch's entries.
__global__ void tc_batch_plan_kernel(const TcDev *__restrict__ entries, int n, int *__restrict__ offsets) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int acc = 0;
  offsets[0] = 0;
  for (int e = 0; e < n; ++e) {
    const int *pl = entries[e].plan;
    acc += (entries[e].kind == 0 ? pl[2] : pl[3]) * pl[4];
    offsets[e + 1] = acc;
  }
}

constexpr int kTcEntriesPerWrite = 16;
struct TcEntryChunk {
  TcDev e[kTcEntriesPerWrite];
  int n;
};

// Copies entry descriptors (passed by value) to device memory, so that the
// launch sequence holds no pointer to host memory and can be captured.
__global__ void tc_write_entries_kernel(const __grid_constant__ TcEntryChunk c, TcDev *__restrict__ dst) {
  const int words = c.n * (int)(sizeof(TcDev) / 4);
  const uint32_t *src = reinterpret_cast<const uint32_t *>(c.e);
  uint32_t *d = reinterpret_cast<uint32_t *>(dst);
  for (int i = threadIdx.x; i < words; i += blockDim.x) d[i] = src[i];
}

// M Mxy regrouped per column group: group g holds (N, mm_ld_g) rows with
// mm_ld_g = its column count rounded up to even (16-byte rows for the bulk
// copies); groups of 8 columns are consecutive.
__global__ void tc_group_mm_kernel(const float2 *__restrict__ MM, int64_t N, int V, float2 *__restrict__ MMg) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * V) return;
  const int64_t n = e / V;
  const int v = (int)(e % V);
  const int g = v / kTcVGroup, vi = v % kTcVGroup;
  const int vg = (V - g * kTcVGroup) < kTcVGroup ? (V - g * kTcVGroup) : kTcVGroup;
  const int ld = (vg + 1) & ~1;
  MMg[(int64_t)g * N * kTcVGroup + n * ld + vi] = MM[e];
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

// Workspace of one problem.
struct TcPlan {
  float *MM;
  float2 *MMg;    // M Mxy per column group (tc_group_mm_kernel)
  Csr csr;
  Runs runs;
  float *weights;
  TcRun *tcruns;
  TcItem *items;  // n_groups lists of 2 S + 2
  int *nf, *ng, *of, *og;
  int *plan;      // n_groups rows of 8 ints
  int *stack;     // runs can be stacked (set on the device)
  float2 *partials;
  int n_groups, max_splits;
};

static int tc_max_splits(int64_t S, int64_t V) {
  const int64_t bytes_per = S * V * 8;
  int64_t s = bytes_per > 0 ? (1LL << 30) / bytes_per : 16;
  if (s > 16) s = 16;
  return (int)(s < 1 ? 1 : s);
}

static int tc_groups(int64_t V) { return (int)ceil_div(V, (int64_t)kTcVGroup); }

static void carve_tc(Carve &c, const fm_signal_args *a, TcPlan &pl) {
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  const int64_t N = a->n_nodes, V = a->n_vencs;
  pl.n_groups = tc_groups(V);
  pl.MM = c.take<float>((size_t)N * V * 2);
  pl.MMg = c.take<float2>((size_t)pl.n_groups * N * kTcVGroup);
  carve_csr(c, a->m_rows, a->m_nnz, pl.csr);
  carve_runs(c, S, kTcRows, pl.runs);
  pl.weights = c.take<float>((size_t)(S + 1) * motion_slots(a->motion));
  pl.tcruns = c.take<TcRun>(S + 1);
  pl.items = c.take<TcItem>((size_t)pl.n_groups * (2 * S + 2));
  pl.nf = c.take<int>(S + 2);
  pl.ng = c.take<int>(S + 2);
  pl.of = c.take<int>(S + 2);
  pl.og = c.take<int>(S + 2);
  pl.plan = c.take<int>((size_t)8 * (pl.n_groups > 0 ? pl.n_groups : 1));
  pl.stack = c.take<int>(4);
  pl.max_splits = tc_max_splits(S, V);
  pl.partials = c.take<float2>((size_t)pl.max_splits * S * V);
}

// Entries of a launch: per problem, per column group, both run kinds.
static int tc_n_entries(const fm_signal_args *probs, int n) {
  int e = 0;
  for (int i = 0; i < n; ++i) e += 2 * tc_groups(probs[i].n_vencs);
  return e;
}

static void carve_batch(Carve &c, const fm_signal_args *probs, int n, TcPlan *plans, TcDev **entries,
                        int **offsets) {
  for (int i = 0; i < n; ++i) carve_tc(c, &probs[i], plans[i]);
  const int ne = tc_n_entries(probs, n);
  *entries = c.take<TcDev>(ne > 0 ? ne : 1);
  *offsets = c.take<int>(ne + 1);
}

// Tile shape of a column group: up to 128 (q, v) pairs per tile and at most
// 64 kz values (fewer when tuned).
static void tc_shape(int Qt, int VG, int &NT, int &acc_cols);

static int tc_qt(const fm_signal_args *a, int VG, const fm_tc_tuning *tune) {
  int cap = (128 / VG < 64) ? 128 / VG : 64;
  if (tune && tune->kz_cap > 0 && tune->kz_cap < cap) cap = tune->kz_cap;
  int Qt = (int)((a->n_kz < cap) ? a->n_kz : cap);
  // narrower tiles until the tiles, node buffers and phase-table ring fit in
  // shared memory (stacked runs are limited to what then fits)
  for (;;) {
    int NT, acc;
    tc_shape(Qt, VG, NT, acc);
    if (Qt <= 8 || tc_smem_layout(NT, VG, Qt).total <= kTcSmemMax) return Qt;
    Qt -= 8;
  }
}

// Runs a stacked unit may touch, for a column group: stacking needs whole
// kz slabs within one tile and no motion (the runs then share node
// positions).  Units take 128 consecutive lines of the runs laid end to end,
// so a unit touches 128 / P runs when P divides 128, else up to
// ceil(127 / P) + 1; at most kTcMaxStack, and fewer when the node buffers (VG
// weight rows and one D row per run) would not fit in shared memory.
constexpr int kTcMaxStack = 16;
static int tc_stack_runs(const fm_signal_args *a, int VG, int Qt) {
  if (a->motion && a->motion->kind != FM_MOTION_NONE) return 1;
  if (a->n_kz < 2 || a->n_lines * a->n_kz < 2 || a->n_kz > Qt) return 1;
  const int P = (int)a->n_lines;
  int R = P >= kTcRows ? 2 : (kTcRows % P == 0 ? kTcRows / P : (kTcRows - 1 + P - 1) / P + 1);
  if (R > kTcMaxStack) R = kTcMaxStack;
  // the tiles and node buffers must fit in shared memory
  int NT, acc;
  tc_shape(Qt, VG, NT, acc);
  while (R > 1 && tc_smem_layout(NT, VG + R, Qt).total > kTcSmemMax) --R;
  return R < 2 ? 1 : R;
}

// Lines per stacked unit (RU) for P lines per run and units touching at most
// R runs: all 128 rows when that keeps within R runs, else whole runs
// (R P lines, units then start at run boundaries) or (R - 1) P lines (a unit
// starting inside a run then still touches at most R runs).
static int tc_pack_rows(int P, int R) {
  if ((int64_t)R * P <= kTcRows) return R * P;
  if (kTcRows % P == 0) return kTcRows;
  if ((kTcRows - 1 + P - 1) / P + 1 <= R) return kTcRows;
  return (R - 1) * P;
}

static void tc_shape(int Qt, int VG, int &NT, int &acc_cols) {
  NT = (int)ceil_div(2 * Qt * VG, 16) * 16;
  acc_cols = 32;
  while (acc_cols < NT) acc_cols <<= 1;
}

static size_t tc_batch_workspace(const fm_signal_args *probs, int n) {
  Carve c(nullptr, 0);
  std::vector<TcPlan> plans(n > 0 ? n : 1);
  TcDev *entries;
  int *offsets;
  carve_batch(c, probs, n, plans.data(), &entries, &offsets);
  return c.used;
}

size_t tc_workspace(const fm_signal_args *a) { return tc_batch_workspace(a, 1); }

// Preparation of one problem (runs, M Mxy, motion weights, run kinds, items
// and splits); fills its launch entries.  Returns the number of entries.
static int tc_prepare(const fm_signal_args *a, TcPlan &pl, const fm_tc_tuning *tune, TcDev *host_entries,
                      cudaStream_t st, const char *who) {
  const int64_t S = a->n_ro * a->n_lines * a->n_kz;
  const int64_t N = a->n_nodes, V = a->n_vencs;
  if (S == 0 || V == 0) return 0;
  float2 *out = static_cast<float2 *>(a->out);
  if (N == 0) {
    FM_CUDA(cudaMemsetAsync(out, 0, (size_t)S * V * sizeof(float2), st));
    return 0;
  }
  FM_REQUIRE(a->n_lines * a->n_kz < (1LL << 30), FM_ERR_SHAPE, "%s: slab too large", who);
  const float *kx = static_cast<const float *>(a->kx), *ky = static_cast<const float *>(a->ky),
              *kz = static_cast<const float *>(a->kz);
  FM_TRY(build_runs<float>(static_cast<const float *>(a->t), S, kTcRows, pl.runs, st));
  FM_TRY(sparse_times_dense<float>(a, pl.csr, static_cast<const float *>(a->Mxy), pl.MM, pl.runs.error, st));
  FM_TRY(check_table_calls(a->motion, pl.runs, st));
  tc_group_mm_kernel<<<(unsigned)ceil_div(N * V, 256), 256, 0, st>>>(reinterpret_cast<const float2 *>(pl.MM), N,
                                                                     (int)V, pl.MMg);
  count_launch();
  FM_TRY(check_launch("tc_group_mm_kernel"));
  const MotionDev md = make_motion_dev(a->motion);
  FM_TRY(launch_run_weights(md, pl.runs.run_t, pl.runs.counts, S, pl.weights, st));
  const int64_t cls_blocks = S < 8 * kSmCount ? S : 8 * kSmCount;
  tc_classify_kernel<<<(unsigned)cls_blocks, 256, 0, st>>>(kx, ky, kz, pl.runs.start, pl.runs.counts,
                                                           (int)a->n_lines, (int)a->n_kz, pl.tcruns);
  count_launch();
  FM_TRY(check_launch("tc_classify_kernel"));
  // stacking check (the same for every column group)
  bool may_stack = false;
  for (int g = 0; g < pl.n_groups; ++g) {
    const int64_t v0 = (int64_t)g * kTcVGroup;
    const int VG = (int)((V - v0) < kTcVGroup ? (V - v0) : kTcVGroup);
    if (tc_stack_runs(a, VG, tc_qt(a, VG, tune)) > 1) may_stack = true;
  }
  if (may_stack) {
    FM_CUDA(cudaMemsetAsync(pl.stack, 1, sizeof(int), st));
    const int64_t work = S;  // n_runs x n_kz <= S
    const unsigned blocks = (unsigned)(work / 256 + 1 < 4 * kSmCount ? work / 256 + 1 : 4 * kSmCount);
    tc_stack_check_kernel<<<blocks, 256, 0, st>>>(kx, ky, kz, pl.tcruns, pl.runs.counts, (int)a->n_lines,
                                                   (int)a->n_kz, pl.stack);
    count_launch();
    FM_TRY(check_launch("tc_stack_check_kernel"));
  }
  int ne = 0;
  for (int g = 0; g < pl.n_groups; ++g) {
    const int64_t v0 = (int64_t)g * kTcVGroup;
    const int VG = (int)((V - v0) < kTcVGroup ? (V - v0) : kTcVGroup);
    const int Qt_f = tc_qt(a, VG, tune);
    const int R = tc_stack_runs(a, VG, Qt_f);
    const int RU = R > 1 ? tc_pack_rows((int)a->n_lines, R) : 0;
    const int *stack = R > 1 ? pl.stack : nullptr;
    TcItem *items = pl.items + (size_t)g * (2 * S + 2);
    int *plan = pl.plan + 8 * g;
    const unsigned gb = (unsigned)ceil_div(S + 1, 256);
    tc_count_kernel<<<gb, 256, 0, st>>>(pl.tcruns, pl.runs.counts, Qt_f, pl.nf, pl.ng, S, stack, (int)a->n_lines, RU);
    count_launch();
    FM_TRY(check_launch("tc_count_kernel"));
    size_t cb = pl.runs.cub_bytes;
    FM_CUDA(cub::DeviceScan::ExclusiveSum(pl.runs.cub_tmp, cb, pl.nf, pl.of, (int)(S + 1), st));
    cb = pl.runs.cub_bytes;
    FM_CUDA(cub::DeviceScan::ExclusiveSum(pl.runs.cub_tmp, cb, pl.ng, pl.og, (int)(S + 1), st));
    count_launch(2);
    tc_fill_kernel<<<gb, 256, 0, st>>>(pl.tcruns, pl.runs.counts, Qt_f, pl.of, pl.og, items, plan, stack,
                                       (int)a->n_lines, RU);
    count_launch();
    FM_TRY(check_launch("tc_fill_kernel"));
    for (int kind = 0; kind < 2; ++kind) {
      TcDev &p = host_entries[ne++];
      p = TcDev{};
      p.N = N; p.S = S; p.V = V;
      p.v0 = (int)v0; p.VG = VG;
      p.n_lines = (int)a->n_lines; p.n_kz = (int)a->n_kz;
      p.kx = kx; p.ky = ky; p.kz = kz;
      p.r0 = static_cast<const float *>(a->r0);
      p.phi = static_cast<const float *>(a->phi);
      p.T2 = static_cast<const float *>(a->T2);
      p.MM = pl.MMg + (size_t)g * N * kTcVGroup;
      p.mm_ld = (VG + 1) & ~1;
      p.md = md;
      p.weights = (md.kind == FM_MOTION_TERMS) ? pl.weights : nullptr;
      p.table = (a->motion && a->motion->kind == FM_MOTION_TABLE) ? static_cast<const float *>(a->motion->table)
                                                                   : nullptr;
      p.run_t = pl.runs.run_t;
      p.runs = pl.tcruns;
      p.items = items;
      p.plan = plan;
      p.partials = pl.partials;
      p.out = out;
      p.error = pl.runs.error;
      p.kind = kind;
      p.Qt = kind == 0 ? Qt_f : 1;
      // a stacked unit's node buffers add one D row per run
      const int Rk = kind == 0 ? R : 1;
      p.stacked = Rk > 1 ? 1 : 0;
      p.wrows = VG + (Rk > 1 ? Rk : 0);
      int acc_cols;
      tc_shape(p.Qt, VG, p.NT, acc_cols);
      // node blocks by bulk copies when the inputs are 16-byte aligned and the
      // staging area fits next to the tiles
      const bool aligned = ((uintptr_t)p.r0 % 16 == 0) && ((uintptr_t)p.T2 % 16 == 0) &&
                           ((uintptr_t)p.phi % 16 == 0) && ((uintptr_t)p.MM % 16 == 0);
      const int ring = kind == 0 ? kTcStages : kTcRingGen;
      p.tma = aligned && tc_smem_layout(p.NT, p.wrows, p.Qt, ring).total + tc_raw_bytes(p.mm_ld) <= kTcSmemMax;
      // the mode rows of a single POD term of several modes are staged with
      // the node blocks (a rank-1 term is held in registers instead) when
      // they are 16-byte aligned and there is room after the raw block
      if (p.tma && md.kind == FM_MOTION_TERMS && md.n_terms == 1 && md.terms[0].kind != FM_TERM_RESPIRATORY &&
          md.terms[0].n_modes > kTcRegModes && (uintptr_t)md.terms[0].modes % 16 == 0 &&
          tc_smem_layout(p.NT, p.wrows, p.Qt, ring).total + tc_raw_bytes(p.mm_ld) +
                  tc_mode_bytes(3 * md.terms[0].n_modes) <= kTcSmemMax)
        p.mstage = 3 * md.terms[0].n_modes;
    }
  }
  tc_plan_kernel<<<1, 32, 0, st>>>(pl.plan, pl.n_groups, N, pl.max_splits, tune ? tune->split_nodes : 0);
  count_launch();
  FM_TRY(check_launch("tc_plan_kernel"));
  return ne;
}

// Signal for n problems: per-problem preparation, then one persistent
// tensor-core launch over all of their work units, then the split sums.
constexpr int kTcSideStreams = 8;  // helper streams for the per-problem preparations of a batch

static int tc_batch(fm_ctx *ctx, const fm_signal_args *probs, int n, const fm_tc_tuning *tune, void *ws,
                    size_t ws_bytes, const char *who) {
  cudaStream_t st = ctx->stream;
  Carve cv(ws, ws_bytes);
  std::vector<TcPlan> plans(n > 0 ? n : 1);
  TcDev *entries;
  int *offsets;
  carve_batch(cv, probs, n, plans.data(), &entries, &offsets);
  FM_TRY(carve_ok(cv, who));
  std::vector<TcDev> host(tc_n_entries(probs, n) + 1);
  int ne = 0;
  // the problems' preparations are independent: with several problems they
  // run on helper streams forked from the launch stream and joined back
  // before the persistent launch (in a captured graph: parallel branches)
  const int K = n >= 4 ? kTcSideStreams : 0;
  if (K > 0) {
    FM_TRY(ctx_side_streams(ctx, K));
    FM_TRY(ctx_fork(ctx, K));
  }
  int prep = FM_OK;
  for (int i = 0; i < n && prep == FM_OK; ++i) {
    const int k = tc_prepare(&probs[i], plans[i], tune, host.data() + ne, K > 0 ? ctx->side[i % K] : st, who);
    if (k < 0) prep = k;
    else ne += k;
  }
  if (K > 0) FM_TRY(ctx_join(ctx, K));
  if (prep != FM_OK) return prep;
  if (ne == 0) return FM_OK;
  int acc_cols = 32;
  size_t smem = 0;
  bool modes = false;
  auto staging = [&](const TcDev &d) -> size_t {
    return d.tma ? tc_raw_bytes(d.mm_ld) + tc_mode_bytes(d.mstage) : 0;
  };
  for (int e = 0; e < ne; ++e) {
    modes = modes || host[e].mstage != 0;
    int NT = host[e].NT, ac = 32;
    while (ac < NT) ac <<= 1;
    if (ac > acc_cols) acc_cols = ac;
    const int ring = host[e].kind == 0 ? kTcStages : kTcRingGen;
    const size_t sm = tc_smem_layout(NT, host[e].wrows, host[e].Qt, ring).total + staging(host[e]);
    if (sm > smem) smem = sm;
  }
  FM_REQUIRE(smem <= kTcSmemMax, FM_ERR_UNSUPPORTED, "%s: tile needs %zu bytes of shared memory", who, smem);
  for (int e0 = 0; e0 < ne; e0 += kTcEntriesPerWrite) {
    TcEntryChunk c;
    c.n = (ne - e0) < kTcEntriesPerWrite ? (ne - e0) : kTcEntriesPerWrite;
    for (int k = 0; k < c.n; ++k) c.e[k] = host[e0 + k];
    tc_write_entries_kernel<<<1, 256, 0, st>>>(c, entries + e0);
    count_launch();
    FM_TRY(check_launch("tc_write_entries_kernel"));
  }
  tc_batch_plan_kernel<<<1, 32, 0, st>>>(entries, ne, offsets);
  count_launch();
  FM_TRY(check_launch("tc_batch_plan_kernel"));
  TcBatchDev B;
  B.entries = entries;
  B.offsets = offsets;
  B.n_entries = ne;
  B.acc_cols = acc_cols;
  {
    ScopedTimer timer(ctx, "signal_tc");
    auto kernel = modes ? signal_tc_kernel<true> : signal_tc_kernel<false>;
    FM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kernel<<<kSmCount, kTcThreads, smem, st>>>(B);
    count_launch();
    FM_TRY(check_launch("signal_tc_kernel"));
  }
  for (int i = 0; i < n; ++i) {
    const fm_signal_args *a = &probs[i];
    const int64_t count = a->n_ro * a->n_lines * a->n_kz * a->n_vencs;
    if (count == 0 || a->n_nodes == 0) continue;
    tc_reduce_kernel<<<(unsigned)ceil_div(count, 256), 256, 0, st>>>(plans[i].partials, plans[i].plan, count,
                                                                      static_cast<float2 *>(a->out));
    count_launch();
    FM_TRY(check_launch("tc_reduce_kernel"));
  }
  return FM_OK;
}

int signal_tc(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes) {
  return tc_batch(ctx, a, 1, nullptr, ws, ws_bytes, "fm_signal(BF16X3)");
}

static int tc_batch_errors(fm_ctx *ctx, const fm_signal_args *probs, int n, void *ws, size_t ws_bytes,
                           const char *who) {
  Carve cv(ws, ws_bytes);
  std::vector<TcPlan> plans(n > 0 ? n : 1);
  TcDev *entries;
  int *offsets;
  carve_batch(cv, probs, n, plans.data(), &entries, &offsets);
  FM_TRY(carve_ok(cv, who));
  int rc = FM_OK;
  for (int i = 0; i < n; ++i) {
    const fm_signal_args *a = &probs[i];
    if (a->n_ro * a->n_lines * a->n_kz == 0 || a->n_vencs == 0 || a->n_nodes == 0) continue;
    const int r = report_errors(plans[i].runs, ctx->stream, who);
    if (r != FM_OK && rc == FM_OK) rc = r;
  }
  if (n == 0) FM_CUDA(cudaStreamSynchronize(ctx->stream));
  return rc;
}

int signal_tc_errors(fm_ctx *ctx, const fm_signal_args *a, void *ws, size_t ws_bytes) {
  return tc_batch_errors(ctx, a, 1, ws, ws_bytes, "fm_signal(BF16X3)");
}

int signal_tc_batch(fm_ctx *ctx, const fm_signal_args *probs, int n, const fm_tc_tuning *tune, void *ws,
                    size_t ws_bytes) {
  return tc_batch(ctx, probs, n, tune, ws, ws_bytes, "fm_signal_batch");
}

int signal_tc_batch_errors(fm_ctx *ctx, const fm_signal_args *probs, int n, void *ws, size_t ws_bytes) {
  return tc_batch_errors(ctx, probs, n, ws, ws_bytes, "fm_signal_batch");
}

size_t tc_batch_workspace_size(const fm_signal_args *probs, int n) { return tc_batch_workspace(probs, n); }

}  // namespace fm
