// Bloch rotation + relaxation sweep with fused POD motion.
//
// Restates solve_mri<float> (cpp/feelmri/BlochSimulator.cpp:12-148 with a
// motion callable, :151-277 without) as one pass: one thread per node keeps
// its magnetisation, relaxation factors and motion modes in registers for
// all time steps; per-step scalars (rf, G, dt, motion weights) are read as
// warp-uniform loads.  Step i -> i+1 uses rf[i+1], G[i+1], dt[i+1]; dt[0] is
// ignored; e1/e2 are recomputed only when dt changes (BlochSimulator.cpp:69-99).
#include <mutex>

#include <math_constants.h>

#include "motion.cuh"

namespace fm {

// Step segments: runs of consecutive steps with the same dt and the same
// RF-off state, so that the sweep tests neither per step.  seg[0] holds the
// count G; seg[1 + g] the first step of segment g with the flags below;
// seg[1 + G] the number of steps.
constexpr int kSegNoRf = 1 << 30;  // rf = 0 on every step of the segment
constexpr int kSegDt = 1 << 29;    // dt changes at the first step (e1, e2 recomputed)
constexpr int kSegStep = kSegDt - 1;

// Sequential pass over the n_time samples of one solve (or one block of a
// sequence): float32 running time (BlochSimulator.cpp:82-83), the
// dt-changed flags (:72), the step segments and the motion call times.
__device__ inline void bloch_prep_range(int64_t n_time, float gamma, const float2 *__restrict__ rf,
                                        const float *__restrict__ G, const float *__restrict__ dt,
                                        float4 *__restrict__ sa, float4 *__restrict__ sb, int *__restrict__ seg,
                                        double *__restrict__ call_t) {
  float ti = 0.0f, dti = -1.0f;
  const float mhg = __fmul_rn(-0.5f, gamma);
  if (call_t) call_t[0] = 0.0;
  int n_seg = 0;
  bool prev_norf = false;
  for (int64_t i = 0; i + 1 < n_time; ++i) {
    const float d = dt[i + 1];
    const bool changed = dti != d;
    dti = d;
    ti = __fadd_rn(ti, dti);
    if (call_t) call_t[i + 1] = (double)ti;
    const float2 r = rf[i + 1];
    sa[i] = make_float4(r.x, r.y, __fmaf_rn(r.x, r.x, __fmul_rn(r.y, r.y)), __fmul_rn(mhg, dti));
    sb[i] = make_float4(G[3 * (i + 1) + 0], G[3 * (i + 1) + 1], G[3 * (i + 1) + 2], dti);
    const bool norf = r.x == 0.f && r.y == 0.f;
    if (i == 0 || changed || norf != prev_norf)
      seg[1 + n_seg++] = (int)i | (norf ? kSegNoRf : 0) | (changed ? kSegDt : 0);
    prev_norf = norf;
  }
  seg[0] = n_seg;
  seg[1 + n_seg] = (int)(n_time > 1 ? n_time - 1 : 0);
}

__global__ void bloch_prep_kernel(int64_t n_time, float gamma, const float2 *__restrict__ rf,
                                  const float *__restrict__ G, const float *__restrict__ dt, float4 *__restrict__ sa,
                                  float4 *__restrict__ sb, int *__restrict__ seg, double *__restrict__ call_t) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  bloch_prep_range(n_time, gamma, rf, G, dt, sa, sb, seg, call_t);
}

// Sequence form: one thread per block.  Block b's samples start at
// offset_b; its steps at offset_b - b (every earlier block has one sample
// more than steps); its segment list at offset_b + b (n_time_b + 1 ints).
// Its motion calls are the samples offset_b .. offset_b + n_time_b - 1.
__global__ void bloch_seq_prep_kernel(const fm_bloch_block *__restrict__ blocks, int n_blocks, float gamma,
                                      const float2 *__restrict__ rf, const float *__restrict__ G,
                                      const float *__restrict__ dt, float4 *__restrict__ sa,
                                      float4 *__restrict__ sb, int *__restrict__ seg, double *__restrict__ call_t,
                                      int *__restrict__ call_block) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n_blocks) return;
  const int64_t o = blocks[b].offset, nt = blocks[b].n_time, step0 = o - b;
  bloch_prep_range(nt, gamma, rf + o, G + 3 * o, dt + o, sa + step0, sb + step0, seg + o + b,
                   call_t ? call_t + o : nullptr);
  if (call_block)
    for (int64_t i = 0; i < nt; ++i) call_block[o + i] = b;
}

struct BlochDev {
  int64_t n, n_time;
  const float *r0, *T1, *T2, *dB;
  float M0;
  const float2 *Mxy0;
  const float *Mz0;
  const float4 *sa, *sb;
  const int *seg;  // step segments (bloch_prep_kernel)
  MotionDev md;
  const float *weights;  // (n_time, slots) motion weights per call
  const float *table;    // TABLE motion: (n_time, N, 3)
  int pod_term;          // index of the register-resident POD term, -1 if none
  float2 *Mxy_hist;
  float *Mz_hist;
  float2 *Mxy_final;
  float *Mz_final;
  float2 *Mxy_carry;
  int64_t final_stride;
};

// One node's registers during a sweep.
template <int RMAX>
struct BlochNode {
  int64_t n;
  float x, y, z, db, invT1, invT2;
  float phx[RMAX > 0 ? RMAX : 1], phy[RMAX > 0 ? RMAX : 1], phz[RMAX > 0 ? RMAX : 1];
  int r_pod;
  float2 mxy;
  float mz;
  float e1, e2, rec;  // rec = (1 - e1) M0, recomputed with e1
};

// MODE: 0 static, 1 TERMS with the POD modes of one term in registers,
//       2 TERMS read from global memory (several POD terms), 3 TABLE,
//       4 one POD term and nothing else (modes in registers; the common
//         pod_trajectory of the examples): no per-step term loop.
template <int MODE, int RMAX>
__device__ __forceinline__ void bloch_node_load(const BlochDev &p, int64_t n, BlochNode<RMAX> &s) {
  s.n = n;
  s.x = p.r0[3 * n + 0]; s.y = p.r0[3 * n + 1]; s.z = p.r0[3 * n + 2];
  s.db = p.dB[n];
  s.invT1 = __frcp_rn(p.T1[n]);
  s.invT2 = __frcp_rn(p.T2[n]);
  s.mxy = p.Mxy0[n];
  s.mz = p.Mz0[n];
  s.e1 = 0.f; s.e2 = 0.f; s.rec = 0.f;
  s.r_pod = 0;
  if (MODE == 1 || MODE == 4) {
    const fm_motion_term &T = p.md.terms[p.pod_term];
    s.r_pod = T.n_modes;
    const float *Phi = T.modes + (size_t)n * 3 * s.r_pod;
#pragma unroll
    for (int m = 0; m < RMAX; ++m) {
      s.phx[m] = (m < s.r_pod) ? __ldg(Phi + m) : 0.f;
      s.phy[m] = (m < s.r_pod) ? __ldg(Phi + s.r_pod + m) : 0.f;
      s.phz[m] = (m < s.r_pod) ? __ldg(Phi + 2 * s.r_pod + m) : 0.f;
    }
  }
}

// Node position at motion call `call` (call 0 is the pod_trajectory(0.0)
// call; step i of a solve uses call i + 1).  wrow: MODE 4's weight row.
template <int MODE, int RMAX>
__device__ __forceinline__ void bloch_position(const BlochDev &p, const BlochNode<RMAX> &s, int64_t call,
                                               const float *wrow, float &px, float &py, float &pz) {
  px = s.x; py = s.y; pz = s.z;
  if (MODE == 4) {
    // the single term's sum, as the k == 0 case of the term loop below
    float tx = 0.f, ty = 0.f, tz = 0.f;
#pragma unroll
    for (int m = 0; m < RMAX; ++m) {
      const float wm = (m < s.r_pod) ? wrow[m] : 0.f;
      tx = fmaf(s.phx[m], wm, tx);
      ty = fmaf(s.phy[m], wm, ty);
      tz = fmaf(s.phz[m], wm, tz);
    }
    px = __fadd_rn(s.x, tx); py = __fadd_rn(s.y, ty); pz = __fadd_rn(s.z, tz);
  } else if (MODE == 1 || MODE == 2) {
    const float *w = p.weights + call * p.md.slots;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (int k = 0; k < p.md.n_terms; ++k) {
      const fm_motion_term &T = p.md.terms[k];
      const float *wk = w + p.md.slot0[k];
      float tx, ty, tz;
      if (T.kind == FM_TERM_RESPIRATORY) {
        const float amp = wk[0];
        tx = __fmul_rn(amp, T.direction[0]);
        ty = __fmul_rn(amp, T.direction[1]);
        tz = __fmul_rn(amp, T.direction[2]);
      } else if (MODE == 1) {
        tx = 0.f; ty = 0.f; tz = 0.f;
#pragma unroll
        for (int m = 0; m < RMAX; ++m) {
          const float wm = (m < s.r_pod) ? wk[m] : 0.f;
          tx = fmaf(s.phx[m], wm, tx);
          ty = fmaf(s.phy[m], wm, ty);
          tz = fmaf(s.phz[m], wm, tz);
        }
      } else {
        const int r = T.n_modes;
        const float *Phi = T.modes + (size_t)s.n * 3 * r;
        tx = 0.f; ty = 0.f; tz = 0.f;
        for (int m = 0; m < r; ++m) {
          const float wm = wk[m];
          tx = fmaf(__ldg(Phi + m), wm, tx);
          ty = fmaf(__ldg(Phi + r + m), wm, ty);
          tz = fmaf(__ldg(Phi + 2 * r + m), wm, tz);
        }
      }
      if (k == 0) { sx = tx; sy = ty; sz = tz; }
      else { sx = __fadd_rn(sx, tx); sy = __fadd_rn(sy, ty); sz = __fadd_rn(sz, tz); }
    }
    px = __fadd_rn(s.x, sx); py = __fadd_rn(s.y, sy); pz = __fadd_rn(s.z, sz);
  } else if (MODE == 3) {
    const float *d = p.table + (call * p.n + s.n) * 3;
    px = __fadd_rn(s.x, d[0]); py = __fadd_rn(s.y, d[1]); pz = __fadd_rn(s.z, d[2]);
  }
}

// One segment of `count` steps (one dt, one RF state; flags from the prep
// pass), step parameters from sa / sb, first motion call call0.  HIST:
// history columns written through hist_m / hist_z (the first step's column).
template <int MODE, int RMAX, bool HIST>
__device__ __forceinline__ void bloch_segment(const BlochDev &p, BlochNode<RMAX> &s, int flags, const float4 *sa,
                                              const float4 *sb, int count, int64_t call0, float2 *hist_m,
                                              float *hist_z) {
  const float *wrow = (MODE == 4) ? p.weights + call0 * p.md.slots + p.md.slot0[p.pod_term] : nullptr;
  const float M0 = p.M0;
  if (flags & kSegDt) {
    // e1, e2 = exp(-dt / T) rounded once to float (the float64 exponential
    // of the float32 product, then one rounding), as a correctly rounded
    // host expf gives them.  (1 - e1) M0 cancels all but a few digits of e1
    // when dt << T1, so an ulp of difference in e1 would be amplified by
    // T1 / dt in the recovery; once per segment, so the cost is nil.
    const float dtw = sb->w;
    s.e1 = __double2float_rn(exp((double)__fmul_rn(-dtw, s.invT1)));
    s.rec = (1.f - s.e1) * M0;
    s.e2 = __double2float_rn(exp((double)__fmul_rn(-dtw, s.invT2)));
  }
  float2 mxy = s.mxy;
  float mz = s.mz;
  const float e1 = s.e1, e2 = s.e2, rec = s.rec;
  if (flags & kSegNoRf) {
    // No RF on these steps: beta = 0, so the update reduces to
    // Mxy' = conj(alpha)^2 Mxy, Mz' = |alpha|^2 Mz; the dropped terms of
    // the general form below are exact zeros.  |rf|^2 is 0, and
    // clamp(sqrt(RN(Bz^2))) needs no sqrt: sqrt(RN(Bz^2)) = |Bz| exactly
    // whenever Bz^2 is a normal float (checked for every float32
    // mantissa); below |Bz| = 1e-18 both forms clamp to 1e-12 (Bz = 0 on
    // gradient-free steps included); an overflowing square gives +inf and
    // a NaN stays NaN in both.
    // unrolled: the position, Bz and sin/cos of the next steps do not
    // depend on this step's magnetisation, so they overlap its update
#pragma unroll 4
    for (int i = 0; i < count; ++i, ++sa, ++sb) {
      const float aw = sa->w;
      const float4 b = *sb;
      float px, py, pz;
      bloch_position<MODE, RMAX>(p, s, call0 + i, wrow, px, py, pz);
      if (MODE == 4) wrow += p.md.slots;
      // Bz = r . G + dB  (BlochSimulator.cpp:104-107)
      const float Bz = __fadd_rn(fmaf(pz, b.z, fmaf(py, b.y, __fmul_rn(px, b.x))), s.db);
      const float sq = __fmul_rn(Bz, Bz);
      float Bn = (sq == CUDART_INF_F) ? sq : fabsf(Bz);
      Bn = (Bn < 1e-12f) ? 1e-12f : Bn;
      const float nz = __fmul_rn(Bz, __frcp_rn(Bn));
      float sn, c;
      sincosf(__fmul_rn(Bn, aw), &sn, &c);
      const float ca_i = nz * sn;  // conj(alpha) = c + i nz s
      const float a2 = fmaf(c, c, ca_i * ca_i);
      const float ca2r = c * c - ca_i * ca_i, ca2i = 2.f * c * ca_i;
      const float nmr = ca2r * mxy.x - ca2i * mxy.y;
      const float nmi = ca2r * mxy.y + ca2i * mxy.x;
      mxy.x = nmr * e2;
      mxy.y = nmi * e2;
      mz = fmaf(a2 * mz, e1, rec);
      if (HIST) {
        *hist_m = mxy;
        *hist_z = mz;
        hist_m += p.n;
        hist_z += p.n;
      }
    }
  } else {
#pragma unroll 4
    for (int i = 0; i < count; ++i, ++sa, ++sb) {
      const float4 a = *sa;
      const float4 b = *sb;
      float px, py, pz;
      bloch_position<MODE, RMAX>(p, s, call0 + i, wrow, px, py, pz);
      if (MODE == 4) wrow += p.md.slots;
      // Bz = r . G + dB  (BlochSimulator.cpp:104-107)
      const float Bz = __fadd_rn(fmaf(pz, b.z, fmaf(py, b.y, __fmul_rn(px, b.x))), s.db);
      float Bn = sqrtf(fmaf(Bz, Bz, a.z));
      Bn = (Bn < 1e-12f) ? 1e-12f : Bn;
      const float invB = __frcp_rn(Bn);
      const float nz = __fmul_rn(Bz, invB);
      const float hp = __fmul_rn(Bn, a.w);
      float sn, c;
      sincosf(hp, &sn, &c);
      // alpha = c - i nz s ; beta = -i (rf/B) s   (BlochSimulator.cpp:114-126)
      const float al_i = -nz * sn;
      const float nxr = __fmul_rn(a.x, invB), nxi = __fmul_rn(a.y, invB);
      const float be_r = nxi * sn, be_i = -nxr * sn;
      const float a2 = fmaf(c, c, al_i * al_i);
      const float b2 = fmaf(be_r, be_r, be_i * be_i);
      // conj(alpha) = c + i nz s  -> ca = (c, -al_i)
      const float ca_r = c, ca_i = -al_i;
      // 2 conj(a) beta Mz
      const float t1r = 2.f * (ca_r * be_r - ca_i * be_i) * mz;
      const float t1i = 2.f * (ca_r * be_i + ca_i * be_r) * mz;
      // conj(a)^2 Mxy
      const float ca2r = ca_r * ca_r - ca_i * ca_i, ca2i = 2.f * ca_r * ca_i;
      const float t2r = ca2r * mxy.x - ca2i * mxy.y;
      const float t2i = ca2r * mxy.y + ca2i * mxy.x;
      // beta^2 conj(Mxy)
      const float bb_r = be_r * be_r - be_i * be_i, bb_i = 2.f * be_r * be_i;
      const float t3r = bb_r * mxy.x + bb_i * mxy.y;
      const float t3i = bb_i * mxy.x - bb_r * mxy.y;
      const float nmr = t1r + t2r - t3r;
      const float nmi = t1i + t2i - t3i;
      // Re(alpha beta conj(Mxy))
      const float ab_r = c * be_r - al_i * be_i, ab_i = c * be_i + al_i * be_r;
      const float re_abm = ab_r * mxy.x + ab_i * mxy.y;
      const float nmz = (a2 - b2) * mz - 2.f * re_abm;
      // relaxation (BlochSimulator.cpp:141-142)
      mxy.x = nmr * e2;
      mxy.y = nmi * e2;
      mz = fmaf(nmz, e1, rec);
      if (HIST) {
        *hist_m = mxy;
        *hist_z = mz;
        hist_m += p.n;
        hist_z += p.n;
      }
    }
  }
  s.mxy = mxy;
  s.mz = mz;
}

// One solve: one thread per node, every step in registers.  Segments of
// steps with one dt and one RF-off state; inside a segment the loop has no
// per-step test.  32-bit step indices (n_time <= 2^29 is checked on the
// host) and running pointers.
template <int MODE, int RMAX, bool HIST>
__global__ void __launch_bounds__(128) bloch_kernel(BlochDev p) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.n) return;
  BlochNode<RMAX> s;
  bloch_node_load<MODE, RMAX>(p, n, s);
  if (HIST) {
    p.Mxy_hist[n] = s.mxy;
    p.Mz_hist[n] = s.mz;
  }
  const int n_seg = p.seg[0];
  const int *segp = p.seg + 1;
  for (int g = 0; g < n_seg; ++g) {
    const int e0 = segp[g];
    const int i0 = e0 & kSegStep, i1 = segp[g + 1] & kSegStep;
    bloch_segment<MODE, RMAX, HIST>(p, s, e0, p.sa + i0, p.sb + i0, i1 - i0, (int64_t)i0 + 1,
                                    HIST ? p.Mxy_hist + (int64_t)(i0 + 1) * p.n + n : nullptr,
                                    HIST ? p.Mz_hist + (int64_t)(i0 + 1) * p.n + n : nullptr);
  }
  if (p.Mxy_final) p.Mxy_final[n * p.final_stride] = s.mxy;
  if (p.Mz_final) p.Mz_final[n] = s.mz;
  if (p.Mxy_carry) p.Mxy_carry[n] = make_float2(0.f * s.mxy.x, 0.f * s.mxy.y);
}

// A block sequence in one sweep (fm_bloch_sequence_f32).
struct BlochSeqDev {
  const fm_bloch_block *blocks;
  int n_blocks;
  const int *seg;
  float2 *Mxy_out;
  float *Mz_out;
  float2 *Mxy_carry;
  float *Mz_carry;
};

// Each block as its own solve (relaxation factors restart at 0, as a fresh
// solve_mri call's do), its final state stored when asked for, then 0 * Mxy
// carried on unless the block is empty (Bloch.py:355-368).
template <int MODE, int RMAX>
__global__ void __launch_bounds__(128) bloch_seq_kernel(BlochDev p, BlochSeqDev q) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.n) return;
  BlochNode<RMAX> s;
  bloch_node_load<MODE, RMAX>(p, n, s);
  for (int b = 0; b < q.n_blocks; ++b) {
    const fm_bloch_block &B = q.blocks[b];
    const int64_t o = B.offset, step0 = o - b;
    const int *segp = q.seg + o + b;
    const int n_seg = segp[0];
    s.e1 = 0.f; s.e2 = 0.f; s.rec = 0.f;
    for (int g = 0; g < n_seg; ++g) {
      const int e0 = segp[1 + g];
      const int i0 = e0 & kSegStep, i1 = segp[2 + g] & kSegStep;
      bloch_segment<MODE, RMAX, false>(p, s, e0, p.sa + step0 + i0, p.sb + step0 + i0, i1 - i0, o + i0 + 1,
                                       nullptr, nullptr);
    }
    if (B.store >= 0) {
      q.Mxy_out[(int64_t)B.store * p.n + n] = s.mxy;
      q.Mz_out[(int64_t)B.store * p.n + n] = s.mz;
    }
    if (!B.empty) s.mxy = make_float2(0.f * s.mxy.x, 0.f * s.mxy.y);
  }
  if (q.Mxy_carry) q.Mxy_carry[n] = s.mxy;
  if (q.Mz_carry) q.Mz_carry[n] = s.mz;
}

// Motion weights of a sequence: call c belongs to block call_block[c], whose
// timeshifts replace the terms' (update_timeshift(t0) before each block).
__global__ void motion_weights_seq_kernel(MotionDev md, const double *__restrict__ times, int64_t n_calls,
                                          const int *__restrict__ call_block,
                                          const fm_bloch_block *__restrict__ blocks, float *__restrict__ weights) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_calls * md.slots) return;
  const int64_t c = idx / md.slots;
  const int sl = (int)(idx - c * md.slots);
  int k = 0;
  while (k + 1 < md.n_terms && sl >= md.slot0[k + 1]) ++k;
  fm_motion_term T = md.terms[k];
  const fm_bloch_block &B = blocks[call_block[c]];
  T.timeshift = B.timeshift[k];
  T.timeshift_kind = B.timeshift_kind[k];
  const int col = sl - md.slot0[k];
  const double t = times[c];
  const double te = term_time(t, T);
  const double v = ppoly_eval(T.pp_c, T.pp_x, T.pp_k, T.pp_intervals, T.n_modes, col, te, T.extrapolate);
  float w = __double2float_rn(v);
  if (T.kind == FM_TERM_POD_VELOCITY) w = __fmul_rn(w, __double2float_rn(t));
  weights[idx] = w;
}

template <int MODE, int RMAX>
static void launch_bloch(const BlochDev &p, bool hist, cudaStream_t st) {
  const int threads = 128;
  const unsigned blocks = (unsigned)ceil_div(p.n, threads);
  if (hist) bloch_kernel<MODE, RMAX, true><<<blocks, threads, 0, st>>>(p);
  else bloch_kernel<MODE, RMAX, false><<<blocks, threads, 0, st>>>(p);
}

static void carve_bloch(Carve &c, const fm_bloch_args *a, float4 **sa, float4 **sb, int **seg, double **call_t,
                        float **weights) {
  const int64_t steps = a->n_time > 1 ? a->n_time - 1 : 1;
  *sa = c.take<float4>(steps);
  *sb = c.take<float4>(steps);
  *seg = c.take<int>(steps + 2);
  *call_t = c.take<double>(a->n_time);
  *weights = c.take<float>((size_t)a->n_time * motion_slots(a->motion));
}

static int validate_bloch(const fm_bloch_args *a) {
  FM_REQUIRE(a != nullptr, FM_ERR_ARG, "fm_bloch_solve_f32: null args");
  FM_REQUIRE(a->n_pos >= 0, FM_ERR_SHAPE, "fm_bloch_solve_f32: negative n_pos");
  FM_REQUIRE(a->n_time >= 1, FM_ERR_SHAPE,
             "fm_bloch_solve_f32: rf_all must hold at least one sample (the initial state column)");
  FM_REQUIRE(a->n_time <= (int64_t)kSegStep, FM_ERR_SHAPE, "fm_bloch_solve_f32: %lld time steps (at most 2^29 - 1)",
             (long long)a->n_time);
  FM_REQUIRE((a->Mxy_hist == nullptr) == (a->Mz_hist == nullptr), FM_ERR_ARG,
             "fm_bloch_solve_f32: Mxy_hist and Mz_hist must be given together");
  if (a->n_pos > 0) {
    FM_REQUIRE(a->r0 && a->T1 && a->T2 && a->delta_B && a->Mxy0 && a->Mz0, FM_ERR_ARG,
               "fm_bloch_solve_f32: null node array");
  }
  FM_REQUIRE(a->rf && a->G && a->dt, FM_ERR_ARG, "fm_bloch_solve_f32: null sequence array");
  FM_TRY(validate_motion(a->motion, a->n_pos, "fm_bloch_solve_f32"));
  if (a->motion && a->motion->kind == FM_MOTION_TABLE) {
    FM_REQUIRE(a->motion->table_calls == a->n_time, FM_ERR_SHAPE,
               "fm_bloch_solve_f32: TABLE motion holds %lld calls, the solve makes %lld",
               (long long)a->motion->table_calls, (long long)a->n_time);
  }
  return FM_OK;
}

}  // namespace fm

using namespace fm;

// Kernel instantiation for a motion descriptor: MODE (see bloch_kernel) and
// the bound on the register-resident POD modes.  Sets pod_term.
template <class L>
static void dispatch_bloch_mode(const MotionDev &md, int &pod_term, L &l) {
  if (md.kind == FM_MOTION_NONE) {
    l.template run<0, 0>();
  } else if (md.kind == FM_MOTION_TABLE) {
    l.template run<3, 0>();
  } else {
    int n_pod = 0, r = 0;
    for (int k = 0; k < md.n_terms; ++k)
      if (md.terms[k].kind != FM_TERM_RESPIRATORY) {
        ++n_pod;
        pod_term = k;
        r = md.terms[k].n_modes;
      }
    if (n_pod == 1 && md.n_terms == 1 && r <= 32) {
      if (r <= 1) l.template run<4, 1>();
      else if (r <= 4) l.template run<4, 4>();
      else if (r <= 8) l.template run<4, 8>();
      else if (r <= 16) l.template run<4, 16>();
      else l.template run<4, 32>();
    } else if (n_pod == 0 || n_pod > 1 || r > 32) {
      l.template run<2, 0>();
    } else if (r <= 1) {
      l.template run<1, 1>();
    } else if (r <= 4) {
      l.template run<1, 4>();
    } else if (r <= 8) {
      l.template run<1, 8>();
    } else if (r <= 16) {
      l.template run<1, 16>();
    } else {
      l.template run<1, 32>();
    }
  }
}

struct SolveLaunch {
  const BlochDev &p;
  bool hist;
  cudaStream_t st;
  template <int MODE, int RMAX>
  void run() { launch_bloch<MODE, RMAX>(p, hist, st); }
};

struct SequenceLaunch {
  const BlochDev &p;
  const BlochSeqDev &q;
  cudaStream_t st;
  template <int MODE, int RMAX>
  void run() {
    if constexpr (MODE != 3) {  // a TABLE motion is rejected by validate_sequence
      bloch_seq_kernel<MODE, RMAX><<<(unsigned)ceil_div(p.n, 128), 128, 0, st>>>(p, q);
    }
  }
};

struct SeqScratch {
  fm_bloch_block *blocks;
  float4 *sa, *sb;
  int *seg;
  double *call_t;
  int *call_block;
  float *weights;
};

static void carve_sequence(Carve &c, const fm_bloch_sequence_args *a, SeqScratch &w) {
  const int64_t steps = a->n_samples - a->n_blocks > 0 ? a->n_samples - a->n_blocks : 1;
  w.blocks = c.take<fm_bloch_block>(a->n_blocks > 0 ? a->n_blocks : 1);
  w.sa = c.take<float4>(steps);
  w.sb = c.take<float4>(steps);
  w.seg = c.take<int>(a->n_samples + a->n_blocks);
  w.call_t = c.take<double>(a->n_samples);
  w.call_block = c.take<int>(a->n_samples);
  w.weights = c.take<float>((size_t)a->n_samples * motion_slots(a->motion));
}

static int validate_sequence(const fm_bloch_sequence_args *a) {
  FM_REQUIRE(a != nullptr, FM_ERR_ARG, "fm_bloch_sequence_f32: null args");
  FM_REQUIRE(a->n_pos >= 0, FM_ERR_SHAPE, "fm_bloch_sequence_f32: negative n_pos");
  FM_REQUIRE(a->n_blocks >= 1 && a->blocks != nullptr, FM_ERR_ARG, "fm_bloch_sequence_f32: no blocks");
  FM_REQUIRE(a->n_store >= 0, FM_ERR_SHAPE, "fm_bloch_sequence_f32: negative n_store");
  int64_t off = 0;
  for (int b = 0; b < a->n_blocks; ++b) {
    const fm_bloch_block &B = a->blocks[b];
    FM_REQUIRE(B.offset == off, FM_ERR_SHAPE, "fm_bloch_sequence_f32: block %d starts at sample %lld, expected %lld",
               b, (long long)B.offset, (long long)off);
    FM_REQUIRE(B.n_time >= 1, FM_ERR_SHAPE, "fm_bloch_sequence_f32: block %d has no samples", b);
    FM_REQUIRE(B.store >= -1 && B.store < a->n_store, FM_ERR_SHAPE,
               "fm_bloch_sequence_f32: block %d stores into row %d of %d", b, B.store, a->n_store);
    for (int k = 0; k < FM_MAX_MOTION_TERMS; ++k)
      FM_REQUIRE(a->motion == nullptr || a->motion->kind != FM_MOTION_TERMS || k >= a->motion->n_terms ||
                     (B.timeshift_kind[k] >= FM_NUM_PYFLOAT && B.timeshift_kind[k] <= FM_NUM_F64),
                 FM_ERR_DTYPE, "fm_bloch_sequence_f32: block %d term %d timeshift kind %d invalid", b, k,
                 B.timeshift_kind[k]);
    off += B.n_time;
  }
  FM_REQUIRE(off == a->n_samples, FM_ERR_SHAPE, "fm_bloch_sequence_f32: blocks cover %lld samples, n_samples is %lld",
             (long long)off, (long long)a->n_samples);
  FM_REQUIRE(a->n_samples + a->n_blocks <= (int64_t)kSegStep, FM_ERR_SHAPE,
             "fm_bloch_sequence_f32: %lld samples (at most 2^29 - 1 with the blocks)", (long long)a->n_samples);
  if (a->n_pos > 0) {
    FM_REQUIRE(a->r0 && a->T1 && a->T2 && a->delta_B && a->Mxy0 && a->Mz0, FM_ERR_ARG,
               "fm_bloch_sequence_f32: null node array");
    FM_REQUIRE(a->n_store == 0 || (a->Mxy_out && a->Mz_out), FM_ERR_ARG,
               "fm_bloch_sequence_f32: n_store > 0 needs Mxy_out and Mz_out");
  }
  FM_REQUIRE(a->rf && a->G && a->dt, FM_ERR_ARG, "fm_bloch_sequence_f32: null sequence array");
  FM_REQUIRE(a->motion == nullptr || a->motion->kind != FM_MOTION_TABLE, FM_ERR_ARG,
             "fm_bloch_sequence_f32: a TABLE motion is not accepted (run the blocks with fm_bloch_solve_f32)");
  FM_TRY(validate_motion(a->motion, a->n_pos, "fm_bloch_sequence_f32"));
  return FM_OK;
}

extern "C" {

int fm_bloch_workspace_size(const fm_bloch_args *a, size_t *bytes) {
  FM_REQUIRE(bytes != nullptr, FM_ERR_ARG, "fm_bloch_workspace_size: null output");
  FM_TRY(validate_bloch(a));
  Carve c(nullptr, 0);
  float4 *sa, *sb;
  int *ch;
  double *ct;
  float *w;
  carve_bloch(c, a, &sa, &sb, &ch, &ct, &w);
  *bytes = c.used;
  return FM_OK;
}

int fm_bloch_solve_f32(fm_ctx *ctx, const fm_bloch_args *a, void *workspace, size_t workspace_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_bloch(a));
  DeviceGuard g(ctx->device);
  cudaStream_t st = ctx->stream;
  Carve cv(workspace, workspace_bytes);
  float4 *sa, *sb;
  int *seg;
  double *call_t;
  float *weights;
  carve_bloch(cv, a, &sa, &sb, &seg, &call_t, &weights);
  FM_TRY(carve_ok(cv, "fm_bloch_solve_f32"));
  if (a->n_pos == 0) return FM_OK;

  const MotionDev md = make_motion_dev(a->motion);
  bloch_prep_kernel<<<1, 1, 0, st>>>(a->n_time, a->gamma, reinterpret_cast<const float2 *>(a->rf), a->G, a->dt, sa,
                                     sb, seg, md.kind == FM_MOTION_TERMS ? call_t : nullptr);
  count_launch();
  FM_TRY(check_launch("bloch_prep_kernel"));
  FM_TRY(launch_motion_weights(md, call_t, a->n_time, weights, st));

  BlochDev p{};
  p.n = a->n_pos;
  p.n_time = a->n_time;
  p.r0 = a->r0; p.T1 = a->T1; p.T2 = a->T2; p.dB = a->delta_B;
  p.M0 = a->M0;
  p.Mxy0 = reinterpret_cast<const float2 *>(a->Mxy0);
  p.Mz0 = a->Mz0;
  p.sa = sa; p.sb = sb; p.seg = seg;
  p.md = md;
  p.weights = weights;
  p.table = (a->motion && a->motion->kind == FM_MOTION_TABLE) ? static_cast<const float *>(a->motion->table) : nullptr;
  p.Mxy_hist = reinterpret_cast<float2 *>(a->Mxy_hist);
  p.Mz_hist = a->Mz_hist;
  p.Mxy_final = reinterpret_cast<float2 *>(a->Mxy_final);
  p.Mz_final = a->Mz_final;
  p.Mxy_carry = reinterpret_cast<float2 *>(a->Mxy_carry);
  p.final_stride = a->final_stride > 1 ? a->final_stride : 1;
  p.pod_term = -1;
  const bool hist = a->Mxy_hist != nullptr;
  ScopedTimer timer(ctx, hist ? "bloch_history" : "bloch_final");

  SolveLaunch L{p, hist, st};
  dispatch_bloch_mode(md, p.pod_term, L);
  count_launch();
  return check_launch("bloch_kernel");
}

int fm_bloch_sequence_workspace_size(const fm_bloch_sequence_args *a, size_t *bytes) {
  FM_REQUIRE(bytes != nullptr, FM_ERR_ARG, "fm_bloch_sequence_workspace_size: null output");
  FM_TRY(validate_sequence(a));
  Carve c(nullptr, 0);
  SeqScratch w;
  carve_sequence(c, a, w);
  *bytes = c.used;
  return FM_OK;
}

int fm_bloch_sequence_f32(fm_ctx *ctx, const fm_bloch_sequence_args *a, void *workspace, size_t workspace_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_sequence(a));
  DeviceGuard g(ctx->device);
  cudaStream_t st = ctx->stream;
  Carve cv(workspace, workspace_bytes);
  SeqScratch w;
  carve_sequence(cv, a, w);
  FM_TRY(carve_ok(cv, "fm_bloch_sequence_f32"));
  if (a->n_pos == 0) return FM_OK;

  const MotionDev md = make_motion_dev(a->motion);
  FM_CUDA(cudaMemcpyAsync(w.blocks, a->blocks, sizeof(fm_bloch_block) * (size_t)a->n_blocks, cudaMemcpyHostToDevice,
                          st));
  const bool terms = md.kind == FM_MOTION_TERMS;
  bloch_seq_prep_kernel<<<(unsigned)ceil_div(a->n_blocks, 64), 64, 0, st>>>(
      w.blocks, a->n_blocks, a->gamma, reinterpret_cast<const float2 *>(a->rf), a->G, a->dt, w.sa, w.sb, w.seg,
      terms ? w.call_t : nullptr, terms ? w.call_block : nullptr);
  count_launch();
  FM_TRY(check_launch("bloch_seq_prep_kernel"));
  if (terms) {
    const int64_t total = a->n_samples * md.slots;
    motion_weights_seq_kernel<<<(unsigned)ceil_div(total, 128), 128, 0, st>>>(md, w.call_t, a->n_samples,
                                                                               w.call_block, w.blocks, w.weights);
    count_launch();
    FM_TRY(check_launch("motion_weights_seq_kernel"));
  }

  BlochDev p{};
  p.n = a->n_pos;
  p.n_time = a->n_samples;
  p.r0 = a->r0; p.T1 = a->T1; p.T2 = a->T2; p.dB = a->delta_B;
  p.M0 = a->M0;
  p.Mxy0 = reinterpret_cast<const float2 *>(a->Mxy0);
  p.Mz0 = a->Mz0;
  p.sa = w.sa; p.sb = w.sb; p.seg = nullptr;
  p.md = md;
  p.weights = w.weights;
  p.pod_term = -1;
  p.final_stride = 1;
  BlochSeqDev q{w.blocks, a->n_blocks, w.seg, reinterpret_cast<float2 *>(a->Mxy_out), a->Mz_out,
                reinterpret_cast<float2 *>(a->Mxy_carry), a->Mz_carry};
  ScopedTimer timer(ctx, "bloch_sequence");
  SequenceLaunch L{p, q, st};
  dispatch_bloch_mode(md, p.pod_term, L);
  count_launch();
  return check_launch("bloch_seq_kernel");
}

}  // extern "C"

// ---- no-allocation variant ---------------------------------------------
// The per-step scratch of the sweep (step parameters, dt flags, motion call
// times and weights) lives in this fixed array instead of a caller-provided
// workspace.  Host code must not use the array's name as a device address:
// its address is looked up once per device with cudaGetSymbolAddress.
namespace fm {

static __device__ __align__(256) unsigned char g_bloch_noalloc_scratch[FM_NOALLOC_BLOCH_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void *g_noalloc_addr[128];

// Device address of the scratch array on `device` (the current device).
static int noalloc_scratch(int device, void **out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  FM_REQUIRE(device >= 0 && device < 128, FM_ERR_ARG, "fm_bloch_solve_f32_noalloc: device %d out of range", device);
  if (g_noalloc_addr[device] == nullptr) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_bloch_noalloc_scratch);
    FM_REQUIRE(e == cudaSuccess && ptr != nullptr, FM_ERR_CUDA,
               "fm_bloch_solve_f32_noalloc: cudaGetSymbolAddress failed on device %d: %s", device,
               cudaGetErrorString(e));
    g_noalloc_addr[device] = ptr;
  }
  *out = g_noalloc_addr[device];
  return FM_OK;
}

}  // namespace fm

extern "C" int fm_bloch_solve_f32_noalloc(fm_ctx *ctx, const fm_bloch_args *a) {
  using namespace fm;
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_bloch(a));
  DeviceGuard g(ctx->device);
  FM_REQUIRE(g.ok, FM_ERR_CUDA, "fm_bloch_solve_f32_noalloc: cannot select device %d", ctx->device);
  size_t need = 0;
  FM_TRY(fm_bloch_workspace_size(a, &need));
  FM_REQUIRE(need <= FM_NOALLOC_BLOCH_SCRATCH_BYTES, FM_ERR_NOMEM,
             "fm_bloch_solve_f32_noalloc: %lld time steps need %zu bytes of scratch, more than the %u bytes this "
             "entry point holds; use fm_bloch_solve_f32 with a workspace",
             (long long)a->n_time, need, (unsigned)FM_NOALLOC_BLOCH_SCRATCH_BYTES);
  void *scratch = nullptr;
  FM_TRY(noalloc_scratch(ctx->device, &scratch));
  return fm_bloch_solve_f32(ctx, a, scratch, FM_NOALLOC_BLOCH_SCRATCH_BYTES);
}
