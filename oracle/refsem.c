/*
 * ORACLE -- test infrastructure, not product code.
 *
 * Plain-C restatement of the reference's native hot path with the
 * reference's own loop order and precision, used by tests/ as the checker of
 * the GPU kernels and by bench.py as the timed CPU baseline ("port").  Nothing
 * in the product (feelmri_b200/) links or calls this file.
 *
 * Parity pinning: the reference's own tests hold no golden vectors for this
 * path and its native modules cannot be built here (Eigen is fetched over the
 * network), so this restatement is pinned by analytic known answers and by
 * golden vectors produced with the reference's python/feelmri/Motion.py
 * (tests/golden/).  The summation order of Eigen's vectorised reductions is
 * not reproduced bit for bit; comparisons use relative tolerances.
 *
 * Follows:
 *   solve_mri     cpp/feelmri/BlochSimulator.cpp:12-148 (motion) / :151-277
 *   Signal<T>     cpp/feelmri/MRI.cpp:38-159 (motion) / :196-298, MRI.h:13
 *   MassAssemble  cpp/feelmri/Assemble.cpp:16-116
 *   lumping       python/feelmri/Phantom.py:395-398 (scipy csc @ ones)
 *   tensordot     cpp/feelmri/POD.cpp:5-38
 *
 * Node loops may run in parallel over node ranges (OpenMP), mirroring the
 * reference's MPI node partition + gather_data sum
 * (python/feelmri/MPIUtilities.py:13-26).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------ Bloch ---- */
/* disp: NULL or (n_time, N, 3) displacements, entry i+1 for step i.
 * Mxy_hist/Mz_hist: (n_time, N) (== (N, n_time) column-major) or NULL;
 * Mxy_out/Mz_out: final state (N,) or NULL. */
void oracle_bloch_f32(int64_t N, int64_t n_time, const float *r0, const float *T1, const float *T2,
                      const float *dB, float M0, float gamma, const float *rf, const float *G, const float *dt,
                      const float *Mxy0, const float *Mz0, const float *disp, float *Mxy_hist, float *Mz_hist,
                      float *Mxy_out, float *Mz_out) {
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < N; ++p) {
    const float invT1 = 1.0f / T1[p], invT2 = 1.0f / T2[p];
    float complex m = Mxy0[2 * p] + I * Mxy0[2 * p + 1];
    float mz = Mz0[p];
    if (Mxy_hist) {
      Mxy_hist[2 * p] = crealf(m);
      Mxy_hist[2 * p + 1] = cimagf(m);
      Mz_hist[p] = mz;
    }
    float e1 = 0.f, e2 = 0.f, dti = -1.0f;
    for (int64_t i = 0; i + 1 < n_time; ++i) {
      const float d = dt[i + 1];
      if (dti != d) {
        e1 = expf(-d * invT1);
        e2 = expf(-d * invT2);
      }
      dti = d;
      const float complex rfc = rf[2 * (i + 1)] + I * rf[2 * (i + 1) + 1];
      const float rf2 = crealf(rfc) * crealf(rfc) + cimagf(rfc) * cimagf(rfc);
      const float kappa = -0.5f * gamma * dti;
      const float Gx = G[3 * (i + 1)], Gy = G[3 * (i + 1) + 1], Gz = G[3 * (i + 1) + 2];
      float x = r0[3 * p], y = r0[3 * p + 1], z = r0[3 * p + 2];
      if (disp) {
        const float *dd = disp + ((i + 1) * N + p) * 3;
        x = x + dd[0];
        y = y + dd[1];
        z = z + dd[2];
      }
      const float Bz = x * Gx + y * Gy + z * Gz + dB[p];
      float Bn = sqrtf(Bz * Bz + rf2);
      if (Bn < 1e-12f) Bn = 1e-12f;
      const float nz = Bz / Bn;
      const float hp = Bn * kappa;
      const float c = cosf(hp), s = sinf(hp);
      const float complex alpha = c - I * (nz * s);
      const float complex ca = conjf(alpha);
      const float a2 = crealf(alpha) * crealf(alpha) + cimagf(alpha) * cimagf(alpha);
      const float complex nxy = rfc / Bn;
      const float complex beta = -I * nxy * s;
      const float complex mn = 2.0f * ca * beta * mz + ca * ca * m - beta * beta * conjf(m);
      const float b2 = crealf(beta) * crealf(beta) + cimagf(beta) * cimagf(beta);
      const float mzn = (a2 - b2) * mz - 2.0f * crealf(alpha * beta * conjf(m));
      m = mn * e2;
      mz = mzn * e1 + (1.0f - e1) * M0;
      if (Mxy_hist) {
        Mxy_hist[2 * ((i + 1) * N + p)] = crealf(m);
        Mxy_hist[2 * ((i + 1) * N + p) + 1] = cimagf(m);
        Mz_hist[(i + 1) * N + p] = mz;
      }
    }
    if (Mxy_out) {
      Mxy_out[2 * p] = crealf(m);
      Mxy_out[2 * p + 1] = cimagf(m);
    }
    if (Mz_out) Mz_out[p] = mz;
  }
}

/* ----------------------------------------------------------- Signal ---- */
#define LANES 8

/* T: element type, CT: complex type, SUF: math suffix */
#define DEFINE_SIGNAL(NAME, T, SINF, COSF, EXPF)                                                              \
  void NAME(int64_t N, int64_t V, int64_t S, const int32_t *indptr, const int32_t *indices, const T *mdata,     \
            const T *kx, const T *ky, const T *kz, const T *t, const T *r0, const T *phi, const T *T2,          \
            const T *Mxy, const T *disp, int64_t n_runs, int pi_exact, int64_t node_begin, int64_t node_end,    \
            T *out) {                                                                                           \
    /* M * Mxy (MRI.cpp:92): columns j ascending, entries in storage order */                                  \
    T *MM = (T *)calloc((size_t)N * V * 2, sizeof(T));                                                          \
    for (int64_t j = 0; j < N; ++j)                                                                             \
      for (int32_t k = indptr[j]; k < indptr[j + 1]; ++k) {                                                     \
        const int64_t i = indices[k];                                                                           \
        for (int64_t v = 0; v < V; ++v) {                                                                       \
          MM[(i * V + v) * 2] += mdata[k] * Mxy[(j * V + v) * 2];                                               \
          MM[(i * V + v) * 2 + 1] += mdata[k] * Mxy[(j * V + v) * 2 + 1];                                       \
        }                                                                                                       \
      }                                                                                                         \
    const float pi_f = 3.14159265358979323846f;                                                                 \
    const T two_pi = pi_exact ? (T)(2.0 * 3.14159265358979323846) : (T)2.0 * (T)pi_f;                           \
    const int64_t n0 = node_begin, n1 = node_end < N ? node_end : N;                                            \
    const int64_t nn = n1 > n0 ? n1 - n0 : 0;                                                                   \
    T *x = (T *)malloc(sizeof(T) * (nn + 1) * 3);                                                               \
    T *phoff = (T *)malloc(sizeof(T) * (nn + 1));                                                               \
    T *W = (T *)malloc(sizeof(T) * (nn + 1) * V * 2);                                                           \
    T *fc = (T *)malloc(sizeof(T) * (nn + 1)); /* the sample's Fourier vector (MRI.cpp:143-149) */              \
    T *fs = (T *)malloc(sizeof(T) * (nn + 1));                                                                  \
    T t_old = (T)-1.0;                                                                                          \
    int64_t run = -1;                                                                                           \
    for (int64_t s = 0; s < S; ++s) {                                                                           \
      if (s == 0 || !(t_old == t[s])) {                                                                         \
        ++run;                                                                                                  \
        const T ts = t[s];                                                                                      \
        for (int64_t q = 0; q < nn; ++q) {                                                                      \
          const int64_t n = n0 + q;                                                                             \
          T px = r0[3 * n], py = r0[3 * n + 1], pz = r0[3 * n + 2];                                             \
          if (disp) {                                                                                           \
            const T *dd = disp + ((run < n_runs ? run : n_runs - 1) * N + n) * 3;                               \
            px = px + dd[0];                                                                                    \
            py = py + dd[1];                                                                                    \
            pz = pz + dd[2];                                                                                    \
          }                                                                                                     \
          x[3 * q] = px;                                                                                        \
          x[3 * q + 1] = py;                                                                                    \
          x[3 * q + 2] = pz;                                                                                    \
          phoff[q] = phi[n] * ts;                                                                               \
          const T dec = EXPF(-ts * ((T)1 / T2[n]));                                                             \
          for (int64_t v = 0; v < V; ++v) {                                                                     \
            W[(q * V + v) * 2] = MM[(n * V + v) * 2] * dec;                                                     \
            W[(q * V + v) * 2 + 1] = MM[(n * V + v) * 2 + 1] * dec;                                             \
          }                                                                                                     \
        }                                                                                                       \
        t_old = ts;                                                                                             \
      }                                                                                                         \
      const T kx_ = two_pi * kx[s], ky_ = two_pi * ky[s], kz_ = two_pi * kz[s];                                 \
      /* one phase and one sin/cos per node-sample, then the V columns (MRI.cpp:143-152) */                     \
      for (int64_t q = 0; q < nn; ++q) {                                                                        \
        const T ph = -kx_ * x[3 * q] - ky_ * x[3 * q + 1] - kz_ * x[3 * q + 2] + phoff[q];                      \
        fc[q] = COSF(ph);                                                                                       \
        fs[q] = SINF(ph);                                                                                       \
      }                                                                                                         \
      for (int64_t v = 0; v < V; ++v) {                                                                         \
        T ar[LANES], ai[LANES];                                                                                 \
        for (int l = 0; l < LANES; ++l) ar[l] = ai[l] = (T)0;                                                   \
        for (int64_t q = 0; q < nn; ++q) {                                                                      \
          const T c = fc[q], sn = fs[q];                                                                        \
          const T wr = W[(q * V + v) * 2], wi = W[(q * V + v) * 2 + 1];                                         \
          ar[q % LANES] += c * wr - sn * wi;                                                                    \
          ai[q % LANES] += c * wi + sn * wr;                                                                    \
        }                                                                                                       \
        T sr = 0, si = 0;                                                                                       \
        for (int l = 0; l < LANES; ++l) {                                                                       \
          sr += ar[l];                                                                                          \
          si += ai[l];                                                                                          \
        }                                                                                                       \
        out[(s * V + v) * 2] = sr;                                                                              \
        out[(s * V + v) * 2 + 1] = si;                                                                          \
      }                                                                                                         \
    }                                                                                                           \
    free(x);                                                                                                    \
    free(phoff);                                                                                                \
    free(W);                                                                                                    \
    free(fc);                                                                                                   \
    free(fs);                                                                                                   \
    free(MM);                                                                                                   \
  }

DEFINE_SIGNAL(oracle_signal_f32_range, float, sinf, cosf, expf)
DEFINE_SIGNAL(oracle_signal_f64_range, double, sin, cos, exp)

/* Whole-node Signal, split over threads by node range (one partial k-space
 * per thread, summed in thread order like gather_data's Reduce). */
#define DEFINE_SIGNAL_PAR(NAME, RANGE, T)                                                                      \
  void NAME(int64_t N, int64_t V, int64_t S, const int32_t *indptr, const int32_t *indices, const T *mdata,     \
            const T *kx, const T *ky, const T *kz, const T *t, const T *r0, const T *phi, const T *T2,          \
            const T *Mxy, const T *disp, int64_t n_runs, int pi_exact, int threads, T *out) {                    \
    if (threads < 1) threads = 1;                                                                               \
    T *part = (T *)calloc((size_t)threads * S * V * 2, sizeof(T));                                              \
    _Pragma("omp parallel for num_threads(threads) schedule(static,1)")                                         \
    for (int k = 0; k < threads; ++k) {                                                                         \
      const int64_t b = N * k / threads, e = N * (k + 1) / threads;                                             \
      RANGE(N, V, S, indptr, indices, mdata, kx, ky, kz, t, r0, phi, T2, Mxy, disp, n_runs, pi_exact, b, e,    \
            part + (size_t)k * S * V * 2);                                                                      \
    }                                                                                                           \
    for (int64_t i = 0; i < S * V * 2; ++i) {                                                                   \
      T acc = 0;                                                                                                \
      for (int k = 0; k < threads; ++k) acc += part[(size_t)k * S * V * 2 + i];                                 \
      out[i] = acc;                                                                                             \
    }                                                                                                           \
    free(part);                                                                                                 \
  }

DEFINE_SIGNAL_PAR(oracle_signal_f32, oracle_signal_f32_range, float)
DEFINE_SIGNAL_PAR(oracle_signal_f64, oracle_signal_f64_range, double)

/* --------------------------------------------------------- tensordot ---- */
void oracle_tensordot_f32(const float *A, const float *w, int64_t rows, int64_t M, float *out) {
  for (int64_t r = 0; r < rows; ++r) {
    float acc = 0.f;
    for (int64_t m = 0; m < M; ++m) acc += A[r * M + m] * w[m];
    out[r] = acc;
  }
}

void oracle_tensordot_f64(const double *A, const double *w, int64_t rows, int64_t M, double *out) {
  for (int64_t r = 0; r < rows; ++r) {
    double acc = 0.0;
    for (int64_t m = 0; m < M; ++m) acc += A[r * M + m] * w[m];
    out[r] = acc;
  }
}

/* ------------------------------------------------------------- Mass ---- */
typedef struct {
  int64_t key; /* col * N + row */
  int64_t ord; /* insertion order */
} trip_t;

static int trip_cmp(const void *a, const void *b) {
  const trip_t *x = (const trip_t *)a, *y = (const trip_t *)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->ord < y->ord ? -1 : (x->ord > y->ord);
}

/* Returns nnz; with indices/data non-NULL writes the CSC (duplicates summed
 * in insertion order, rows sorted per column) as setFromTriplets builds it. */
#define DEFINE_MASS(NAME, T, FABS)                                                                             \
  int64_t NAME(int64_t E, int nb, const int32_t *elems, int64_t N, const T *nodes, int Q, const T *qw,          \
               const T *tab, int32_t *indptr, int32_t *indices, T *data) {                                      \
    const int64_t K = E * nb * nb;                                                                              \
    trip_t *tr = (trip_t *)malloc(sizeof(trip_t) * (K + 1));                                                    \
    T *val = (T *)malloc(sizeof(T) * (K + 1));                                                                  \
    for (int64_t e = 0; e < E; ++e) {                                                                           \
      T Me[100];                                                                                                \
      memset(Me, 0, sizeof(Me));                                                                                \
      for (int q = 0; q < Q; ++q) {                                                                             \
        const T *Sq = tab + (size_t)q * 4 * nb;                                                                 \
        T J[3][3];                                                                                              \
        for (int a = 0; a < 3; ++a)                                                                             \
          for (int c = 0; c < 3; ++c) {                                                                         \
            T s = 0;                                                                                            \
            for (int i = 0; i < nb; ++i) s += Sq[(a + 1) * nb + i] * nodes[3 * (int64_t)elems[e * nb + i] + c]; \
            J[a][c] = s;                                                                                        \
          }                                                                                                     \
        const T det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -                                       \
                      J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +                                       \
                      J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);                                        \
        const T ad = FABS(det);                                                                                 \
        for (int i = 0; i < nb; ++i)                                                                            \
          for (int j = 0; j < nb; ++j) Me[i * nb + j] += ((Sq[i] * Sq[j]) * ad) * qw[q];                        \
      }                                                                                                         \
      for (int i = 0; i < nb; ++i)                                                                              \
        for (int j = 0; j < nb; ++j) {                                                                          \
          const int64_t k = e * nb * nb + i * nb + j;                                                           \
          tr[k].key = (int64_t)elems[e * nb + j] * N + elems[e * nb + i];                                       \
          tr[k].ord = k;                                                                                        \
          val[k] = Me[i * nb + j];                                                                              \
        }                                                                                                       \
    }                                                                                                           \
    qsort(tr, (size_t)K, sizeof(trip_t), trip_cmp);                                                             \
    int64_t nnz = 0;                                                                                            \
    if (indptr) memset(indptr, 0, sizeof(int32_t) * (N + 1));                                                   \
    for (int64_t k = 0; k < K;) {                                                                               \
      int64_t m = k + 1;                                                                                        \
      T acc = val[tr[k].ord];                                                                                   \
      while (m < K && tr[m].key == tr[k].key) acc += val[tr[m++].ord];                                          \
      const int64_t col = tr[k].key / N, row = tr[k].key % N;                                                   \
      if (indices) {                                                                                            \
        indices[nnz] = (int32_t)row;                                                                            \
        data[nnz] = acc;                                                                                        \
      }                                                                                                         \
      if (indptr) indptr[col + 1] += 1;                                                                         \
      ++nnz;                                                                                                    \
      k = m;                                                                                                    \
    }                                                                                                           \
    if (indptr)                                                                                                 \
      for (int64_t c = 0; c < N; ++c) indptr[c + 1] += indptr[c];                                               \
    free(tr);                                                                                                   \
    free(val);                                                                                                  \
    return nnz;                                                                                                 \
  }

DEFINE_MASS(oracle_mass_f32, float, fabsf)
DEFINE_MASS(oracle_mass_f64, double, fabs)

/* y = M @ ones for a CSC matrix, as scipy's csc_matvec accumulates it. */
void oracle_csc_rowsum_f64(int64_t N, const int32_t *indptr, const int32_t *indices, const double *data,
                           double *y) {
  for (int64_t i = 0; i < N; ++i) y[i] = 0.0;
  for (int64_t j = 0; j < N; ++j)
    for (int32_t k = indptr[j]; k < indptr[j + 1]; ++k) y[indices[k]] += data[k] * 1.0;
}

void oracle_csc_rowsum_f32(int64_t N, const int32_t *indptr, const int32_t *indices, const float *data, float *y) {
  for (int64_t i = 0; i < N; ++i) y[i] = 0.0f;
  for (int64_t j = 0; j < N; ++j)
    for (int32_t k = indptr[j]; k < indptr[j + 1]; ++k) y[indices[k]] += data[k] * 1.0f;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
