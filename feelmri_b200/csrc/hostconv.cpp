// Host-side argument conversion for the Signal shim.
//
// The reference's pybind11 sparse caster turns any scipy matrix into CSC by
// calling scipy.sparse.csc_matrix(obj) (pybind11 eigen/matrix.h, sparse
// type_caster::load).  The lumped mass that the reference's examples pass to
// Signal is a lil_matrix (python/feelmri/Phantom.py:395-398), so every Signal
// call pays scipy's lil -> csr -> csc conversion, which walks one Python list
// per row.  lil_to_csc produces the same three arrays:
//
//   * the row lists are read in row order and each list in its stored order
//     (scipy's lil_flatten_to_array);
//   * entries are distributed to their columns in that order, so the row
//     indices of every column come out in the order scipy's csr_tocsc gives
//     them (sorted when the lists are);
//   * values are read as C doubles (np.float64 and np.float32 scalars both
//     convert exactly) and returned as float64; the caller force-casts them
//     to the solver's type as the caster does.
//
// The row lists are read on several threads when every index is a plain int
// and every value a float (see row_items_plain); otherwise one thread reads
// them through the C API.  Anything unexpected (a row that is not a list,
// lists of unequal length, a column index out of range, a value that does not
// convert) returns None and the caller lets scipy handle the matrix, so scipy
// raises its own errors.
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#include <numpy/arrayobject.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Ref {
  PyObject *p = nullptr;
  explicit Ref(PyObject *o) : p(o) {}
  ~Ref() { Py_XDECREF(p); }
};

PyObject *give_up() {
  if (PyErr_Occurred()) PyErr_Clear();
  Py_RETURN_NONE;
}

// Row i's list lengths, read without any C API call that may run Python code.
inline bool row_len_plain(PyObject *r, PyObject *d, int32_t *len) {
  if (!PyList_Check(r) || !PyList_Check(d)) return false;
  const Py_ssize_t n = PyList_GET_SIZE(r);
  if (PyList_GET_SIZE(d) != n || n > INT32_MAX) return false;
  *len = (int32_t)n;
  return true;
}

// Row i's items when every index is an exact int with a compact value and
// every value a float (or a float subclass, such as np.float64).  These are
// plain memory reads of immutable objects, so worker threads may do them
// while the calling thread holds the GIL.  False for anything else.
inline bool row_items_plain(PyObject *r, PyObject *d, Py_ssize_t n_cols, int32_t *cols, double *vals) {
  const Py_ssize_t n = PyList_GET_SIZE(r);
  for (Py_ssize_t k = 0; k < n; ++k) {
    PyObject *jo = PyList_GET_ITEM(r, k);
    PyObject *vo = PyList_GET_ITEM(d, k);
    if (!PyLong_CheckExact(jo) || !PyUnstable_Long_IsCompact(reinterpret_cast<PyLongObject *>(jo))) return false;
    const Py_ssize_t j = PyUnstable_Long_CompactValue(reinterpret_cast<PyLongObject *>(jo));
    if (j < 0 || j >= n_cols || !PyFloat_Check(vo)) return false;
    cols[k] = (int32_t)j;
    vals[k] = PyFloat_AS_DOUBLE(vo);
  }
  return true;
}

// Runs fn(begin, end) over [0, n) on up to `threads` threads (the calling
// thread takes the first range).
template <class F>
void parallel_rows(Py_ssize_t n, int threads, F fn) {
  if (threads <= 1 || n < 4096) {
    fn((Py_ssize_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  const Py_ssize_t chunk = (n + threads - 1) / threads;
  for (int t = 1; t < threads; ++t) {
    const Py_ssize_t b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) pool.emplace_back(fn, b, e);
  }
  fn((Py_ssize_t)0, std::min(n, chunk));
  for (auto &th : pool) th.join();
}

// Single-threaded flattening through the C API (any int-like index, any value
// with __float__); false when scipy should take over.
bool flatten_generic(PyArrayObject *ra, PyArrayObject *da, Py_ssize_t n_rows, Py_ssize_t n_cols,
                     std::vector<int32_t> &row_ptr, std::vector<int32_t> &cols, std::vector<double> &vals) {
  cols.clear();
  vals.clear();
  for (Py_ssize_t i = 0; i < n_rows; ++i) {
    PyObject *r = *reinterpret_cast<PyObject **>(PyArray_GETPTR1(ra, i));
    PyObject *d = *reinterpret_cast<PyObject **>(PyArray_GETPTR1(da, i));
    if (!PyList_Check(r) || !PyList_Check(d)) return false;
    const Py_ssize_t len = PyList_GET_SIZE(r);
    if (PyList_GET_SIZE(d) != len) return false;
    for (Py_ssize_t k = 0; k < len; ++k) {
      const long j = PyLong_AsLong(PyList_GET_ITEM(r, k));
      if (j == -1 && PyErr_Occurred()) return false;
      if (j < 0 || j >= n_cols) return false;
      const double v = PyFloat_AsDouble(PyList_GET_ITEM(d, k));
      if (v == -1.0 && PyErr_Occurred()) return false;
      cols.push_back((int32_t)j);
      vals.push_back(v);
    }
    if (cols.size() > (size_t)INT32_MAX) return false;
    row_ptr[(size_t)i + 1] = (int32_t)cols.size();
  }
  return true;
}

// lil_to_csc(rows, data, n_rows, n_cols[, threads]) -> (indptr int32, indices int32, data float64) or None
PyObject *lil_to_csc(PyObject *, PyObject *args) {
  PyObject *rows_o = nullptr, *data_o = nullptr;
  Py_ssize_t n_rows = 0, n_cols = 0;
  int threads = 0;
  if (!PyArg_ParseTuple(args, "OOnn|i", &rows_o, &data_o, &n_rows, &n_cols, &threads)) return nullptr;
  if (!PyArray_Check(rows_o) || !PyArray_Check(data_o)) return give_up();
  PyArrayObject *ra = reinterpret_cast<PyArrayObject *>(rows_o);
  PyArrayObject *da = reinterpret_cast<PyArrayObject *>(data_o);
  if (PyArray_TYPE(ra) != NPY_OBJECT || PyArray_TYPE(da) != NPY_OBJECT || PyArray_NDIM(ra) != 1 ||
      PyArray_NDIM(da) != 1 || PyArray_DIM(ra, 0) != n_rows || PyArray_DIM(da, 0) != n_rows || n_rows < 0 ||
      n_cols < 0 || n_rows > INT32_MAX || n_cols >= INT32_MAX)
    return give_up();
  if (threads <= 0) threads = (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
  auto row_at = [&](Py_ssize_t i) { return *reinterpret_cast<PyObject **>(PyArray_GETPTR1(ra, i)); };
  auto dat_at = [&](Py_ssize_t i) { return *reinterpret_cast<PyObject **>(PyArray_GETPTR1(da, i)); };

  // Scratch kept between calls (calls are serialised by the GIL), so that
  // repeated conversions of one size do not page-fault fresh memory.
  static std::vector<int32_t> row_ptr, cols;
  static std::vector<double> vals;
  static std::vector<int64_t> count;
  row_ptr.assign((size_t)n_rows + 1, 0);
  cols.clear();
  vals.clear();

  // Pass 1: flatten the row lists into CSR order (row order, list order).
  // The lists are scattered Python objects, so reading them is memory
  // latency: rows are split over threads, first for the lengths, then for
  // the items at their row offsets.
  std::atomic<bool> plain{true};
  parallel_rows(n_rows, threads, [&](Py_ssize_t b, Py_ssize_t e) {
    for (Py_ssize_t i = b; i < e; ++i) {
      if (!row_len_plain(row_at(i), dat_at(i), &row_ptr[(size_t)i + 1])) {
        plain.store(false, std::memory_order_relaxed);
        return;
      }
    }
  });
  if (plain.load()) {
    int64_t nnz64 = 0;
    for (Py_ssize_t i = 0; i < n_rows; ++i) {
      nnz64 += row_ptr[(size_t)i + 1];
      if (nnz64 > INT32_MAX) return give_up();
      row_ptr[(size_t)i + 1] = (int32_t)nnz64;
    }
    cols.resize((size_t)nnz64);
    vals.resize((size_t)nnz64);
    parallel_rows(n_rows, threads, [&](Py_ssize_t b, Py_ssize_t e) {
      for (Py_ssize_t i = b; i < e && plain.load(std::memory_order_relaxed); ++i) {
        const size_t o = (size_t)row_ptr[(size_t)i];
        if (!row_items_plain(row_at(i), dat_at(i), n_cols, cols.data() + o, vals.data() + o)) {
          plain.store(false, std::memory_order_relaxed);
          return;
        }
      }
    });
  }
  if (!plain.load() && !flatten_generic(ra, da, n_rows, n_cols, row_ptr, cols, vals)) return give_up();
  const npy_intp nnz = (npy_intp)cols.size();

  npy_intp dp = n_cols + 1;
  Ref indptr(PyArray_SimpleNew(1, &dp, NPY_INT32));
  Ref indices(PyArray_SimpleNew(1, &nnz, NPY_INT32));
  Ref data(PyArray_SimpleNew(1, &nnz, NPY_FLOAT64));
  if (!indptr.p || !indices.p || !data.p) return nullptr;
  int32_t *ip = static_cast<int32_t *>(PyArray_DATA(reinterpret_cast<PyArrayObject *>(indptr.p)));
  int32_t *ix = static_cast<int32_t *>(PyArray_DATA(reinterpret_cast<PyArrayObject *>(indices.p)));
  double *dv = static_cast<double *>(PyArray_DATA(reinterpret_cast<PyArrayObject *>(data.p)));

  // Pass 2: the CSC arrays, by a stable scatter in row order (the order of
  // scipy's csr_tocsc).  When the column indices already increase strictly
  // in row order (a diagonal, such as the lumped mass), every column holds
  // at most one entry and the scatter keeps the order: the values are copied
  // as they are and the column pointers come from a merge walk.  The output
  // arrays are fresh memory, so that case is split over the threads too.
  bool monotone = true;
  for (npy_intp k = 1; k < nnz && monotone; ++k) monotone = cols[(size_t)k - 1] < cols[(size_t)k];
  if (monotone) {
    parallel_rows(n_rows, threads, [&](Py_ssize_t b, Py_ssize_t e) {
      const int32_t k0 = row_ptr[(size_t)b], k1 = row_ptr[(size_t)e];
      if (k1 > k0) std::memcpy(dv + k0, vals.data() + k0, sizeof(double) * (size_t)(k1 - k0));
      for (Py_ssize_t i = b; i < e; ++i)
        for (int32_t k = row_ptr[(size_t)i]; k < row_ptr[(size_t)i + 1]; ++k) ix[k] = (int32_t)i;
    });
    parallel_rows(n_cols + 1, threads, [&](Py_ssize_t b, Py_ssize_t e) {
      npy_intp k = std::lower_bound(cols.begin(), cols.begin() + nnz, (int32_t)b) - cols.begin();
      for (Py_ssize_t j = b; j < e; ++j) {
        while (k < nnz && cols[(size_t)k] < j) ++k;
        ip[j] = (int32_t)k;
      }
    });
  } else {
    count.assign((size_t)n_cols + 1, 0);
    for (npy_intp k = 0; k < nnz; ++k) count[(size_t)cols[(size_t)k] + 1] += 1;
    for (Py_ssize_t j = 0; j < n_cols; ++j) count[(size_t)j + 1] += count[(size_t)j];
    for (Py_ssize_t j = 0; j <= n_cols; ++j) ip[j] = (int32_t)count[(size_t)j];
    for (Py_ssize_t i = 0; i < n_rows; ++i) {
      for (int32_t k = row_ptr[(size_t)i]; k < row_ptr[(size_t)i + 1]; ++k) {
        const int64_t pos = count[(size_t)cols[(size_t)k]]++;
        ix[pos] = (int32_t)i;
        dv[pos] = vals[(size_t)k];
      }
    }
  }
  return PyTuple_Pack(3, indptr.p, indices.p, data.p);
}

PyMethodDef kMethods[] = {
    {"lil_to_csc", lil_to_csc, METH_VARARGS,
     "lil_to_csc(rows, data, n_rows, n_cols[, threads]) -> (indptr, indices, data) of the CSC form, or None"},
    {nullptr, nullptr, 0, nullptr}};

PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "_hostconv", "Host-side argument conversion.", -1, kMethods,
                       nullptr, nullptr, nullptr, nullptr};

}  // namespace

PyMODINIT_FUNC PyInit__hostconv(void) {
  import_array();
  return PyModule_Create(&kModule);
}
