// Device evaluation of the reference's motion callables.
//
// The reference passes the simulation time to a Python callable once per
// Bloch step or per distinct readout time (cpp/feelmri/BlochSimulator.cpp:86,
// cpp/feelmri/MRI.cpp:114).  For the callables python/feelmri/Motion.py
// defines, the callable's arithmetic is reproduced here:
//   t_eff = fold(t + timeshift)                         Motion.py:248, :279
//   fold(x) = x - T * floor(x / T)  (periodic only)       Motion.py:146-148
//   w = float32(PPoly(t_eff))       (float64 evaluation)  Motion.py:237-238
//   w *= t                          (PODVelocity only)     Motion.py:283-287
//   disp = tensordot(modes, w)      (float32 GEMV)         Motion.py:254 -> POD.cpp:5-38
//   respiratory: float32(spline(t_eff)) * direction         Motion.py:101-103, :63-66
//   PODSum: term1(t) + term2(t)      (float32 adds)         Motion.py:303-309
// The precision of `t + timeshift` and of the fold follows NumPy 2's scalar
// promotion: a Python float is weak (it adopts numpy.float32 when combined
// with one), numpy.float64 dominates.
#pragma once
#include <math.h>

#include "common.cuh"

namespace fm {

// Total number of weight slots a motion descriptor needs per call time.
inline int motion_slots(const fm_motion *m) {
  if (m == nullptr || m->kind != FM_MOTION_TERMS) return 0;
  int s = 0;
  for (int k = 0; k < m->n_terms; ++k) s += m->terms[k].n_modes;
  return s;
}

__host__ __device__ inline int promote_kind(int a, int b) {
  if (a == FM_NUM_F64 || b == FM_NUM_F64) return FM_NUM_F64;
  if (a == FM_NUM_F32 || b == FM_NUM_F32) return FM_NUM_F32;
  return FM_NUM_PYFLOAT;
}

// t_eff for one term, returned widened to double.
__device__ inline double term_time(double t, const fm_motion_term &T) {
  const int kx = promote_kind(FM_NUM_PYFLOAT, T.timeshift_kind);
  double x;
  if (kx == FM_NUM_F32) {
    x = (double)__fadd_rn((float)t, (float)T.timeshift);
  } else {
    x = __dadd_rn(t, T.timeshift);
  }
  if (T.period_kind == FM_NUM_NONE) return x;
  const int kf = promote_kind(kx, T.period_kind);
  if (kf == FM_NUM_F32) {
    const float xf = (float)x, Tf = (float)T.period;
    const float q = floorf(__fdiv_rn(xf, Tf));
    return (double)__fsub_rn(xf, __fmul_rn(Tf, q));
  }
  const double q = floor(__ddiv_rn(x, T.period));
  return __dsub_rn(x, __dmul_rn(T.period, q));
}

// Index of the PPoly interval holding xv (scipy's find_interval for
// ascending breakpoints): x[i] <= xv < x[i+1], closed on the right at the
// last breakpoint; -1 when out of range (or NaN) and not extrapolating.
__device__ inline int ppoly_interval(const double *x, int nint, double xv, int extrapolate) {
  const double a = x[0], b = x[nint];
  if (!(a <= xv && xv <= b)) {
    if (extrapolate && xv < a) return 0;
    if (extrapolate && xv > b) return nint - 1;
    return -1;
  }
  if (xv == b) return nint - 1;
  int lo = 0, hi = nint;  // invariant x[lo] <= xv < x[hi]
  while (lo < hi - 1) {
    const int mid = (lo + hi) >> 1;
    if (xv >= x[mid]) lo = mid; else hi = mid;
  }
  return lo;
}

// Power-basis evaluation from the lowest order term up, as scipy's PPoly
// evaluates (res += c[k-1-j] * s^j), with every operation rounded on its own.
__device__ inline double ppoly_eval(const double *c, const double *x, int k, int nint, int ncols, int col,
                                    double xv, int extrapolate) {
  const int iv = ppoly_interval(x, nint, xv, extrapolate);
  if (iv < 0) return __longlong_as_double(0x7ff8000000000000LL);
  const double s = __dsub_rn(xv, x[iv]);
  double res = 0.0, z = 1.0;
  for (int j = 0; j < k; ++j) {
    const double cj = c[((size_t)(k - 1 - j) * nint + iv) * ncols + col];
    res = __dadd_rn(res, __dmul_rn(cj, z));
    if (j < k - 1) z = __dmul_rn(z, s);
  }
  return res;
}

// Weight table: for call c and slot s, the float32 weight (POD modes) or
// amplitude (respiratory) the callable computes at times[c].
struct MotionDev {
  int kind;
  int n_terms;
  int slots;
  fm_motion_term terms[FM_MAX_MOTION_TERMS];
  int slot0[FM_MAX_MOTION_TERMS];
};

inline MotionDev make_motion_dev(const fm_motion *m) {
  MotionDev d{};
  d.kind = (m == nullptr) ? FM_MOTION_NONE : m->kind;
  if (d.kind == FM_MOTION_TERMS) {
    d.n_terms = m->n_terms;
    int s = 0;
    for (int k = 0; k < m->n_terms; ++k) {
      d.terms[k] = m->terms[k];
      d.slot0[k] = s;
      s += m->terms[k].n_modes;
    }
    d.slots = s;
  }
  return d;
}

int validate_motion(const fm_motion *m, int64_t n_nodes, const char *who);

// Fills weights[c * slots + s] for n_calls call times (device array).
int launch_motion_weights(const MotionDev &md, const double *times_dev, int64_t n_calls, float *weights,
                          cudaStream_t st);

// Displacement of node n at one call from the weights of that call.
__device__ inline void motion_disp(const MotionDev &md, const float *__restrict__ w, int64_t n, int64_t n_nodes,
                                   float &dx, float &dy, float &dz) {
  float sx = 0.f, sy = 0.f, sz = 0.f;
  for (int k = 0; k < md.n_terms; ++k) {
    const fm_motion_term &T = md.terms[k];
    const float *wk = w + md.slot0[k];
    float tx, ty, tz;
    if (T.kind == FM_TERM_RESPIRATORY) {
      tx = __fmul_rn(wk[0], T.direction[0]);
      ty = __fmul_rn(wk[0], T.direction[1]);
      tz = __fmul_rn(wk[0], T.direction[2]);
    } else {
      const int r = T.n_modes;
      const float *Phi = T.modes + (size_t)n * 3 * r;
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
  dx = sx; dy = sy; dz = sz;
}

}  // namespace fm
