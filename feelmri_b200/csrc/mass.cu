// Finite-element mass assembly and lumping.
//
// Restates MassAssemble<T> (cpp/feelmri/Assemble.cpp:79-116): per element
// the local matrix Me = sum_q (S S^T) |det J| w_q (LocalMassAssemble,
// Assemble.cpp:59-75; J from the tabulated reference gradients, IsoMapping
// Assemble.cpp:16-55), emitted as triplets (elem(i), elem(j), Me(i,j)) in
// element order and combined as Eigen's setFromTriplets does: duplicates
// summed in insertion order, CSC with row indices sorted inside each column.
// On the device the triplets are ordered by a stable radix sort on
// (column, row), which keeps insertion order among duplicates.
//
// Lumping restates FEMPhantom.mass_matrix(lumped=True)
// (python/feelmri/Phantom.py:395-398): row sums as scipy forms them for a
// CSC matrix (csc @ ones: columns visited in ascending order).  The
// assembled matrix is symmetric entry for entry (S_i S_j == S_j S_i, and
// both entries collect the same elements in the same order), so row i summed
// over ascending columns equals column i summed over ascending rows.
#include <cub/cub.cuh>

#include "common.cuh"

namespace fm {

constexpr int kMaxNb = 10;

template <typename T>
__global__ void mass_local_kernel(int64_t E, int nb, const int *__restrict__ elems, int64_t N,
                                  const T *__restrict__ nodes, int Q, const T *__restrict__ qw,
                                  const T *__restrict__ tab, unsigned long long *__restrict__ keys,
                                  int *__restrict__ order, T *__restrict__ vals, int *__restrict__ bad) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  int id[kMaxNb];
  T X[kMaxNb][3];
  for (int i = 0; i < nb; ++i) {
    int v = elems[e * nb + i];
    if (v < 0 || v >= N) {
      atomicExch(bad, 1);
      v = 0;
    }
    id[i] = v;
    X[i][0] = nodes[3 * (int64_t)v + 0];
    X[i][1] = nodes[3 * (int64_t)v + 1];
    X[i][2] = nodes[3 * (int64_t)v + 2];
  }
  T Me[kMaxNb * kMaxNb];
  for (int k = 0; k < nb * nb; ++k) Me[k] = T(0);
  for (int q = 0; q < Q; ++q) {
    const T *Sq = tab + (size_t)q * 4 * nb;
    // J(a, c) = sum_i dS_a[i] * X[i][c]   (Assemble.cpp:36-44)
    T J[3][3];
    for (int a = 0; a < 3; ++a) {
      const T *dS = Sq + (size_t)(a + 1) * nb;
      for (int c = 0; c < 3; ++c) {
        T s = T(0);
        for (int i = 0; i < nb; ++i) s = s + dS[i] * X[i][c];
        J[a][c] = s;
      }
    }
    // Cofactor expansion along the first row (Eigen's 3x3 determinant).
    const T det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                  J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                  J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    const T adet = det < T(0) ? -det : det;
    const T w = qw[q];
    // Me += (S S^T) * |detJ| * w_q   (Assemble.cpp:72)
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) Me[i * nb + j] = Me[i * nb + j] + ((Sq[i] * Sq[j]) * adet) * w;
  }
  const int64_t base = e * nb * nb;
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      const int64_t k = base + i * nb + j;
      keys[k] = ((unsigned long long)(unsigned)id[j] << 32) | (unsigned)id[i];  // (col, row)
      order[k] = (int)k;
      vals[k] = Me[i * nb + j];
    }
}

__global__ void mass_heads_kernel(const unsigned long long *__restrict__ keys, int64_t K, int *__restrict__ head) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  head[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1 : 0;
}

// One thread per distinct (col, row): its column is counted, and (when
// writing) its duplicates are summed in insertion order (the sort is stable).
template <typename T>
__global__ void mass_collapse_kernel(const unsigned long long *__restrict__ keys, const int *__restrict__ order,
                                     const T *__restrict__ vals, const int *__restrict__ head,
                                     const int *__restrict__ uid, int64_t K, int *__restrict__ indices,
                                     T *__restrict__ data, int *__restrict__ colcount, int write) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K || !head[k]) return;
  const unsigned long long key = keys[k];
  if (colcount) atomicAdd(colcount + (int)(key >> 32), 1);
  if (!write) return;
  T acc = vals[order[k]];
  for (int64_t m = k + 1; m < K && !head[m]; ++m) acc = acc + vals[order[m]];
  const int u = uid[k] - 1;
  if (indices) indices[u] = (int)(key & 0xffffffffULL);
  data[u] = acc;
}

// lumped[c] = sum over the entries of column c in ascending row order.
template <typename T>
__global__ void mass_lump_kernel(const int *__restrict__ indptr, const T *__restrict__ data, int64_t N,
                                 T *__restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  T acc = T(0);
  for (int k = indptr[c]; k < indptr[c + 1]; ++k) acc = acc + data[k];
  out[c] = acc;
}

struct MassPlan {
  unsigned long long *keys_in, *keys_out;
  int *ord_in, *ord_out;
  void *vals;
  int *head, *uid;
  int *colcount, *indptr;
  int *bad;
  int *data_idx;
  void *lump_data;
  void *cub_tmp;
  size_t cub_bytes;
};

static int64_t n_triplets(const fm_mass_args *a) { return a->n_elems * a->nodes_per_elem * a->nodes_per_elem; }

static void carve_mass(Carve &c, const fm_mass_args *a, int is_double, MassPlan &p) {
  const int64_t K = n_triplets(a);
  const size_t tsz = is_double ? sizeof(double) : sizeof(float);
  p.keys_in = c.take<unsigned long long>(K + 1);
  p.keys_out = c.take<unsigned long long>(K + 1);
  p.ord_in = c.take<int>(K + 1);
  p.ord_out = c.take<int>(K + 1);
  p.vals = c.take<char>((K + 1) * tsz);
  p.head = c.take<int>(K + 1);
  p.uid = c.take<int>(K + 1);
  p.colcount = c.take<int>(a->n_nodes + 2);
  p.indptr = c.take<int>(a->n_nodes + 2);
  p.bad = c.take<int>(2);
  p.lump_data = c.take<char>((K + 1) * tsz);
  size_t b1 = 0, b2 = 0, b3 = 0;
  const int Ki = (int)(K > 0 ? K : 1);
  cub::DeviceRadixSort::SortPairs(nullptr, b1, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                  (int *)nullptr, (int *)nullptr, Ki);
  cub::DeviceScan::InclusiveSum(nullptr, b2, (int *)nullptr, (int *)nullptr, Ki);
  cub::DeviceScan::ExclusiveSum(nullptr, b3, (int *)nullptr, (int *)nullptr, (int)(a->n_nodes + 1));
  p.cub_bytes = b1 > b2 ? b1 : b2;
  p.cub_bytes = p.cub_bytes > b3 ? p.cub_bytes : b3;
  p.cub_tmp = c.take<char>(p.cub_bytes);
}

static int validate_mass(const fm_mass_args *a, const char *who) {
  FM_REQUIRE(a != nullptr, FM_ERR_ARG, "%s: null args", who);
  FM_REQUIRE(a->n_elems >= 0 && a->n_nodes >= 0 && a->n_qpoints >= 0, FM_ERR_SHAPE, "%s: negative extent", who);
  FM_REQUIRE(a->nodes_per_elem >= 1 && a->nodes_per_elem <= kMaxNb, FM_ERR_SHAPE,
             "%s: nodes_per_elem=%d outside [1, %d]", who, a->nodes_per_elem, kMaxNb);
  FM_REQUIRE(a->n_nodes < (1LL << 31) - 2, FM_ERR_SHAPE, "%s: too many nodes", who);
  FM_REQUIRE(n_triplets(a) < (1LL << 31) - 2, FM_ERR_SHAPE, "%s: %lld triplets exceed the 2^31 limit", who,
             (long long)n_triplets(a));
  if (a->n_elems > 0) {
    FM_REQUIRE(a->elems && a->nodes && a->tabulated && (a->n_qpoints == 0 || a->qweights), FM_ERR_ARG,
               "%s: null input", who);
  }
  return FM_OK;
}

// Builds the CSC of the assembled matrix in the plan: indptr in p.indptr,
// values in `data` (capacity entries) and rows in `indices` when non-null.
template <typename T>
static int mass_build(fm_ctx *ctx, const fm_mass_args *a, MassPlan &p, int64_t *nnz_out, int32_t *indices, T *data,
                      int64_t capacity, const char *who) {
  cudaStream_t st = ctx->stream;
  const int64_t K = n_triplets(a), N = a->n_nodes;
  FM_CUDA(cudaMemsetAsync(p.bad, 0, 2 * sizeof(int), st));
  FM_CUDA(cudaMemsetAsync(p.colcount, 0, (N + 2) * sizeof(int), st));
  if (K > 0) {
    mass_local_kernel<T><<<(unsigned)ceil_div(a->n_elems, 128), 128, 0, st>>>(
        a->n_elems, a->nodes_per_elem, a->elems, N, static_cast<const T *>(a->nodes), a->n_qpoints,
        static_cast<const T *>(a->qweights), static_cast<const T *>(a->tabulated), p.keys_in, p.ord_in,
        static_cast<T *>(p.vals), p.bad);
    count_launch();
    FM_TRY(check_launch("mass_local_kernel"));
    size_t cb = p.cub_bytes;
    FM_CUDA(cub::DeviceRadixSort::SortPairs(p.cub_tmp, cb, p.keys_in, p.keys_out, p.ord_in, p.ord_out, (int)K, 0, 64,
                                            st));
    count_launch();
    mass_heads_kernel<<<(unsigned)ceil_div(K, 256), 256, 0, st>>>(p.keys_out, K, p.head);
    count_launch();
    FM_TRY(check_launch("mass_heads_kernel"));
    cb = p.cub_bytes;
    FM_CUDA(cub::DeviceScan::InclusiveSum(p.cub_tmp, cb, p.head, p.uid, (int)K, st));
    count_launch();
  }
  int h[2] = {0, 0};
  if (K > 0) {
    FM_CUDA(cudaMemcpyAsync(h, p.uid + (K - 1), sizeof(int), cudaMemcpyDeviceToHost, st));
    FM_CUDA(cudaMemcpyAsync(h + 1, p.bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  FM_CUDA(cudaStreamSynchronize(st));
  FM_REQUIRE(h[1] == 0, FM_ERR_SHAPE, "%s: element connectivity refers to a node outside [0, %lld)", who,
             (long long)N);
  const int64_t nnz = h[0];
  if (nnz_out) *nnz_out = nnz;
  const bool write = (data != nullptr);
  if (write) {
    FM_REQUIRE(capacity >= nnz, FM_ERR_NOMEM, "%s: output capacity %lld < nnz %lld", who, (long long)capacity,
               (long long)nnz);
  }
  if (K > 0) {
    mass_collapse_kernel<T><<<(unsigned)ceil_div(K, 256), 256, 0, st>>>(
        p.keys_out, p.ord_out, static_cast<const T *>(p.vals), p.head, p.uid, K, indices, data, p.colcount,
        write ? 1 : 0);
    count_launch();
    FM_TRY(check_launch("mass_collapse_kernel"));
  }
  size_t cb = p.cub_bytes;
  FM_CUDA(cub::DeviceScan::ExclusiveSum(p.cub_tmp, cb, p.colcount, p.indptr, (int)(N + 1), st));
  count_launch();
  return FM_OK;
}

}  // namespace fm

using namespace fm;

extern "C" {

int fm_mass_workspace_size(const fm_mass_args *a, int is_double, size_t *bytes) {
  FM_REQUIRE(bytes != nullptr, FM_ERR_ARG, "fm_mass_workspace_size: null output");
  FM_TRY(validate_mass(a, "fm_mass_workspace_size"));
  Carve c(nullptr, 0);
  MassPlan p;
  carve_mass(c, a, is_double, p);
  *bytes = c.used;
  return FM_OK;
}

int fm_mass_assemble(fm_ctx *ctx, const fm_mass_args *a, int is_double, int64_t *nnz_out, int32_t *indptr,
                     int32_t *indices, void *data, int64_t capacity, void *workspace, size_t workspace_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_mass(a, "fm_mass_assemble"));
  FM_REQUIRE(nnz_out != nullptr, FM_ERR_ARG, "fm_mass_assemble: null nnz_out");
  FM_REQUIRE((indices == nullptr) == (data == nullptr), FM_ERR_ARG,
             "fm_mass_assemble: indices and data must be given together");
  DeviceGuard g(ctx->device);
  Carve cv(workspace, workspace_bytes);
  MassPlan p;
  carve_mass(cv, a, is_double, p);
  FM_TRY(carve_ok(cv, "fm_mass_assemble"));
  int st;
  if (is_double)
    st = mass_build<double>(ctx, a, p, nnz_out, indices, static_cast<double *>(data), capacity, "fm_mass_assemble");
  else
    st = mass_build<float>(ctx, a, p, nnz_out, indices, static_cast<float *>(data), capacity, "fm_mass_assemble");
  FM_TRY(st);
  if (indptr) {
    FM_CUDA(cudaMemcpyAsync(indptr, p.indptr, (a->n_nodes + 1) * sizeof(int), cudaMemcpyDeviceToDevice,
                            ctx->stream));
  }
  return FM_OK;
}

int fm_mass_lumped(fm_ctx *ctx, const fm_mass_args *a, int is_double, void *out, void *workspace,
                   size_t workspace_bytes) {
  FM_TRY(ctx_ok(ctx));
  FM_TRY(validate_mass(a, "fm_mass_lumped"));
  FM_REQUIRE(out != nullptr || a->n_nodes == 0, FM_ERR_ARG, "fm_mass_lumped: null output");
  DeviceGuard g(ctx->device);
  Carve cv(workspace, workspace_bytes);
  MassPlan p;
  carve_mass(cv, a, is_double, p);
  FM_TRY(carve_ok(cv, "fm_mass_lumped"));
  int64_t nnz = 0;
  const int64_t N = a->n_nodes;
  if (N == 0) return FM_OK;
  if (is_double) {
    FM_TRY(mass_build<double>(ctx, a, p, &nnz, nullptr, static_cast<double *>(p.lump_data), n_triplets(a) + 1,
                              "fm_mass_lumped"));
    mass_lump_kernel<double><<<(unsigned)ceil_div(N, 256), 256, 0, ctx->stream>>>(
        p.indptr, static_cast<const double *>(p.lump_data), N, static_cast<double *>(out));
  } else {
    FM_TRY(mass_build<float>(ctx, a, p, &nnz, nullptr, static_cast<float *>(p.lump_data), n_triplets(a) + 1,
                             "fm_mass_lumped"));
    mass_lump_kernel<float><<<(unsigned)ceil_div(N, 256), 256, 0, ctx->stream>>>(
        p.indptr, static_cast<const float *>(p.lump_data), N, static_cast<float *>(out));
  }
  count_launch();
  return check_launch("mass_lump_kernel");
}

}  // extern "C"
