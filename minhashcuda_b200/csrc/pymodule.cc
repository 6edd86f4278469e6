// CPython module `libMHCUDA`: the Python surface of src-d/minhashcuda
// (python.cc:30-42, README.md:105-159) on top of this engine's C ABI.
//
// Same function names, keyword names, defaults, return shapes and exception
// mapping as the reference (python.cc:86-96,119-142):
//   mhcudaInvalidArguments        -> ValueError
//   mhcudaNoSuchDevice            -> ValueError("No such CUDA device exists")
//   mhcudaMemoryAllocationFailure -> MemoryError
//   mhcudaMemoryCopyError         -> RuntimeError
//   mhcudaRuntimeError            -> AssertionError
// Additions: minhash_cuda_assign_random_vars (alias of minhash_cuda_assign_vars,
// the name README.md:125 uses), minhash_cuda_calc_batch, acceptance of
// scipy.sparse.csr_array besides csr_matrix, and casting of float64 (or
// integer) data and parameter arrays to float32 where the reference accepts
// only what numpy casts safely.
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#include <numpy/arrayobject.h>

#include <algorithm>
#include <ctime>
#include <string>
#include <unordered_map>
#include <vector>

#include "minhashcuda.h"
#include "minhashcuda_b200.h"

namespace {

// Owning PyObject reference.
class Ref {
 public:
  Ref() = default;
  explicit Ref(PyObject *p) : p_(p) {}
  Ref(const Ref &) = delete;
  Ref &operator=(const Ref &) = delete;
  Ref(Ref &&o) noexcept : p_(o.p_) { o.p_ = nullptr; }
  Ref &operator=(Ref &&o) noexcept {
    if (this != &o) {
      Py_XDECREF(p_);
      p_ = o.p_;
      o.p_ = nullptr;
    }
    return *this;
  }
  ~Ref() { Py_XDECREF(p_); }
  PyObject *get() const { return p_; }
  PyArrayObject *arr() const { return reinterpret_cast<PyArrayObject *>(p_); }
  PyObject *release() {
    PyObject *p = p_;
    p_ = nullptr;
    return p;
  }
  explicit operator bool() const { return p_ != nullptr; }

 private:
  PyObject *p_ = nullptr;
};

// Sets the Python exception for a failed call; returns false on failure.
bool check(MHCUDAResult r, const char *fn) {
  switch (r) {
    case mhcudaSuccess:
      return true;
    case mhcudaInvalidArguments:
      PyErr_Format(PyExc_ValueError, "Invalid arguments were passed to %s", fn);
      return false;
    case mhcudaNoSuchDevice:
      PyErr_SetString(PyExc_ValueError, "No such CUDA device exists");
      return false;
    case mhcudaMemoryAllocationFailure:
      PyErr_SetString(PyExc_MemoryError, "Failed to allocate memory on GPU");
      return false;
    case mhcudaMemoryCopyError:
      PyErr_SetString(PyExc_RuntimeError, "cudaMemcpy failed");
      return false;
    case mhcudaRuntimeError:
      PyErr_Format(PyExc_AssertionError, "%s failure (bug?)", fn);
      return false;
    default:
      PyErr_Format(PyExc_AssertionError, "Unknown error code returned from %s", fn);
      return false;
  }
}

MinhashCudaGenerator *gen_from(unsigned long long v) {
  MinhashCudaGenerator *gen = reinterpret_cast<MinhashCudaGenerator *>(static_cast<uintptr_t>(v));
  if (!gen) PyErr_SetString(PyExc_ValueError, "MinHashCuda Generator pointer is null.");
  return gen;
}

// A CSR matrix viewed as three C arrays and their element types
// (MHCUDAElementType).  For mhcuda_calc_batch they are always
// float32/uint32-bit; for mhcuda_calc_typed also float64 and 64-bit.
struct Csr {
  Ref data, indices, indptr;
  const void *weights = nullptr;
  const void *cols = nullptr;
  const void *rows = nullptr;
  int wtype = mhcudaFloat32, ctype = mhcudaUInt32, rtype = mhcudaUInt32;
  uint32_t length = 0;
};

bool is_csr(PyObject *m) {
  Ref sparse(PyImport_ImportModule("scipy.sparse"));
  if (!sparse) {
    PyErr_SetString(PyExc_ImportError, "Failed to import scipy.sparse.csr_matrix");
    return false;
  }
  for (const char *name : {"csr_matrix", "csr_array"}) {
    Ref type(PyObject_GetAttrString(sparse.get(), name));
    if (!type) {
      PyErr_Clear();
      continue;
    }
    if (PyType_Check(type.get()) &&
        PyObject_TypeCheck(m, reinterpret_cast<PyTypeObject *>(type.get())))
      return true;
  }
  PyErr_SetString(PyExc_TypeError, "The second argument must be of type scipy.sparse.csr_matrix");
  return false;
}

// An array in a type the engine reads in place, else cast (a copy), as
// python.cc:310-327 always casts to float32 / uint32.  In place: contiguous,
// aligned, native-order arrays of float32 (and float64 if `wide`) for data;
// of int32/uint32 (and int64/uint64 if `wide`) for indices -- the bits of an
// int32 index equal its uint32 for every valid index, and a negative one
// reads as a column >= dim, which the device rejects.
Ref as_engine_array(PyObject *obj, bool floating, bool wide, int *type) {
  if (PyArray_Check(obj)) {
    PyArrayObject *a = reinterpret_cast<PyArrayObject *>(obj);
    if (PyArray_ISCARRAY_RO(a) && PyArray_ISNOTSWAPPED(a)) {
      int t = -1;
      switch (PyArray_TYPE(a)) {
        case NPY_FLOAT32: t = floating ? mhcudaFloat32 : -1; break;
        case NPY_FLOAT64: t = floating && wide ? mhcudaFloat64 : -1; break;
        case NPY_UINT32: t = floating ? -1 : mhcudaUInt32; break;
        case NPY_INT32: t = floating ? -1 : mhcudaInt32; break;
        case NPY_INT64: t = !floating && wide ? mhcudaInt64 : -1; break;
        case NPY_UINT64: t = !floating && wide ? mhcudaUInt64 : -1; break;
        default: break;
      }
      // npy_intp-sized longs alias NPY_INT64 / NPY_UINT64 on LP64.
      if (t < 0 && !floating && wide && PyArray_ITEMSIZE(a) == 8 && PyArray_ISINTEGER(a))
        t = PyArray_ISSIGNED(a) ? mhcudaInt64 : mhcudaUInt64;
      if (t >= 0) {
        *type = t;
        Py_INCREF(obj);
        return Ref(obj);
      }
    }
  }
  *type = floating ? mhcudaFloat32 : mhcudaUInt32;
  return Ref(PyArray_FROM_OTF(obj, floating ? NPY_FLOAT32 : NPY_UINT32,
                              NPY_ARRAY_FORCECAST | NPY_ARRAY_IN_ARRAY));
}

bool csr_view(PyObject *m, Csr *out, bool wide) {
  if (!is_csr(m)) return false;
  Ref d(PyObject_GetAttrString(m, "data"));
  if (d) out->data = as_engine_array(d.get(), true, wide, &out->wtype);
  if (!out->data) {
    PyErr_SetString(PyExc_ValueError, "Failed to convert csr_matrix.data to numpy.array");
    return false;
  }
  Ref i(PyObject_GetAttrString(m, "indices"));
  if (i) out->indices = as_engine_array(i.get(), false, wide, &out->ctype);
  if (!out->indices) {
    PyErr_SetString(PyExc_ValueError, "Failed to convert csr_matrix.indices to numpy.array");
    return false;
  }
  Ref p(PyObject_GetAttrString(m, "indptr"));
  if (p) out->indptr = as_engine_array(p.get(), false, wide, &out->rtype);
  if (!out->indptr) {
    PyErr_SetString(PyExc_ValueError, "Failed to convert csr_matrix.indptr to numpy.array");
    return false;
  }
  out->weights = PyArray_DATA(out->data.arr());
  out->cols = PyArray_DATA(out->indices.arr());
  out->rows = PyArray_DATA(out->indptr.arr());
  const npy_intp n = PyArray_SIZE(out->indptr.arr());
  out->length = n > 0 ? static_cast<uint32_t>(n - 1) : 0;
  return true;
}

PyObject *py_init(PyObject *, PyObject *args, PyObject *kwargs) {
  unsigned int dim = 0, seed = static_cast<unsigned int>(time(nullptr)), devices = 0;
  unsigned short samples = 0;
  int deferred = 0, verbosity = 0;
  static const char *kwlist[] = {"dim", "samples", "seed", "deferred", "devices", "verbosity",
                                 nullptr};
  if (!PyArg_ParseTupleAndKeywords(args, kwargs, "IH|IpIi", const_cast<char **>(kwlist), &dim,
                                   &samples, &seed, &deferred, &devices, &verbosity))
    return nullptr;
  MHCUDAResult r = mhcudaSuccess;
  MinhashCudaGenerator *gen;
  Py_BEGIN_ALLOW_THREADS
  gen = mhcuda_init(dim, samples, seed, deferred, devices, verbosity, &r);
  Py_END_ALLOW_THREADS
  if (!check(r, "minhash_cuda_init")) return nullptr;
  return PyLong_FromUnsignedLongLong(reinterpret_cast<uintptr_t>(gen));
}

PyObject *py_retrieve_vars(PyObject *, PyObject *args) {
  unsigned long long g = 0;
  if (!PyArg_ParseTuple(args, "K", &g)) return nullptr;
  MinhashCudaGenerator *gen = gen_from(g);
  if (!gen) return nullptr;
  const MinhashCudaGeneratorParameters p = mhcuda_get_parameters(gen);
  npy_intp dims[2] = {p.samples, static_cast<npy_intp>(p.dim)};
  Ref rs(PyArray_EMPTY(2, dims, NPY_FLOAT32, 0));
  Ref ln_cs(PyArray_EMPTY(2, dims, NPY_FLOAT32, 0));
  Ref betas(PyArray_EMPTY(2, dims, NPY_FLOAT32, 0));
  if (!rs || !ln_cs || !betas) return nullptr;
  float *a = static_cast<float *>(PyArray_DATA(rs.arr()));
  float *b = static_cast<float *>(PyArray_DATA(ln_cs.arr()));
  float *c = static_cast<float *>(PyArray_DATA(betas.arr()));
  MHCUDAResult r;
  Py_BEGIN_ALLOW_THREADS
  r = mhcuda_retrieve_random_vars(gen, a, b, c);
  Py_END_ALLOW_THREADS
  if (!check(r, "minhash_cuda_retrieve_vars")) return nullptr;
  return Py_BuildValue("NNN", rs.release(), ln_cs.release(), betas.release());
}

PyObject *py_assign_vars(PyObject *, PyObject *args) {
  unsigned long long g = 0;
  PyObject *objs[3];
  if (!PyArg_ParseTuple(args, "KOOO", &g, &objs[0], &objs[1], &objs[2])) return nullptr;
  MinhashCudaGenerator *gen = gen_from(g);
  if (!gen) return nullptr;
  const MinhashCudaGeneratorParameters p = mhcuda_get_parameters(gen);
  const npy_intp want = static_cast<npy_intp>(p.dim) * p.samples;
  static const char *names[3] = {"rs", "ln_cs", "betas"};
  Ref arrs[3];
  const float *ptrs[3];
  for (int i = 0; i < 3; ++i) {
    arrs[i] = Ref(PyArray_FROM_OTF(objs[i], NPY_FLOAT32, NPY_ARRAY_FORCECAST | NPY_ARRAY_IN_ARRAY));
    if (!arrs[i]) {
      PyErr_Format(PyExc_ValueError, "Failed to convert %s to numpy array", names[i]);
      return nullptr;
    }
    if (PyArray_SIZE(arrs[i].arr()) != want) {
      PyErr_Format(PyExc_ValueError, "%s.size must be equal to dim * samples", names[i]);
      return nullptr;
    }
    ptrs[i] = static_cast<const float *>(PyArray_DATA(arrs[i].arr()));
  }
  MHCUDAResult r;
  Py_BEGIN_ALLOW_THREADS
  r = mhcuda_assign_random_vars(gen, ptrs[0], ptrs[1], ptrs[2]);
  Py_END_ALLOW_THREADS
  if (!check(r, "minhash_cuda_assign_vars")) return nullptr;
  Py_RETURN_NONE;
}

PyObject *py_calc(PyObject *, PyObject *args, PyObject *kwargs) {
  unsigned long long g = 0;
  PyObject *matrix = nullptr;
  unsigned int row_start = 0, row_finish = 0xFFFFFFFFu;
  static const char *kwlist[] = {"gen", "matrix", "row_start", "row_finish", nullptr};
  if (!PyArg_ParseTupleAndKeywords(args, kwargs, "KO|II", const_cast<char **>(kwlist), &g,
                                   &matrix, &row_start, &row_finish))
    return nullptr;
  MinhashCudaGenerator *gen = gen_from(g);
  if (!gen) return nullptr;
  Csr m;
  if (!csr_view(matrix, &m, /*wide=*/true)) return nullptr;
  if (row_start >= m.length) {
    PyErr_SetString(PyExc_ValueError,
                    "minhash_cuda_calc: row_start must be less than the total number of rows "
                    "in the input matrix.");
    return nullptr;
  }
  row_finish = std::min(row_finish, m.length);
  if (row_finish <= row_start) {
    PyErr_SetString(PyExc_ValueError,
                    "minhash_cuda_calc: row_finish must be greater than row_start.");
    return nullptr;
  }
  const uint32_t length = row_finish - row_start;
  const MinhashCudaGeneratorParameters p = mhcuda_get_parameters(gen);
  npy_intp dims[3] = {static_cast<npy_intp>(length), p.samples, 2};
  Ref out(PyArray_EMPTY(3, dims, NPY_UINT32, 0));
  if (!out) return nullptr;
  uint32_t *o = static_cast<uint32_t *>(PyArray_DATA(out.arr()));
  // mhcuda_calc_typed honours rows[0] != 0 as an offset, so a row slice is a
  // pointer offset into indptr: no rebased copy (python.cc:349-359 copies).
  const void *rows = static_cast<const char *>(m.rows) +
                     static_cast<size_t>(row_start) * PyArray_ITEMSIZE(m.indptr.arr());
  MHCUDAResult r;
  Py_BEGIN_ALLOW_THREADS
  r = mhcuda_calc_typed(gen, m.weights, m.wtype, m.cols, m.ctype, rows, m.rtype, length, o);
  Py_END_ALLOW_THREADS
  if (!check(r, "minhash_cuda_calc")) return nullptr;
  return out.release();
}

PyObject *py_calc_batch(PyObject *, PyObject *args) {
  unsigned long long g = 0;
  PyObject *seq = nullptr;
  if (!PyArg_ParseTuple(args, "KO", &g, &seq)) return nullptr;
  MinhashCudaGenerator *gen = gen_from(g);
  if (!gen) return nullptr;
  Ref fast(PySequence_Fast(seq, "minhash_cuda_calc_batch: expected a sequence of CSR matrices"));
  if (!fast) return nullptr;
  const Py_ssize_t n = PySequence_Fast_GET_SIZE(fast.get());
  const MinhashCudaGeneratorParameters p = mhcuda_get_parameters(gen);
  std::vector<Csr> mats(static_cast<size_t>(n));
  std::vector<const float *> w(n);
  std::vector<const uint32_t *> c(n), rw(n);
  std::vector<uint32_t> len(n);
  std::vector<uint32_t *> outp(n);
  Ref result(PyList_New(n));
  if (!result) return nullptr;
  for (Py_ssize_t i = 0; i < n; ++i) {
    PyObject *m = PySequence_Fast_GET_ITEM(fast.get(), i);
    if (!csr_view(m, &mats[i], /*wide=*/false)) return nullptr;
    w[i] = static_cast<const float *>(mats[i].weights);
    c[i] = static_cast<const uint32_t *>(mats[i].cols);
    rw[i] = static_cast<const uint32_t *>(mats[i].rows);
    len[i] = mats[i].length;
    npy_intp dims[3] = {static_cast<npy_intp>(len[i]), p.samples, 2};
    PyObject *o = PyArray_EMPTY(3, dims, NPY_UINT32, 0);
    if (!o) return nullptr;
    outp[i] = static_cast<uint32_t *>(PyArray_DATA(reinterpret_cast<PyArrayObject *>(o)));
    PyList_SET_ITEM(result.get(), i, o);
  }
  MHCUDAResult r;
  Py_BEGIN_ALLOW_THREADS
  r = mhcuda_calc_batch(gen, static_cast<uint32_t>(n), w.data(), c.data(), rw.data(), len.data(),
                        outp.data());
  Py_END_ALLOW_THREADS
  if (!check(r, "minhash_cuda_calc_batch")) return nullptr;
  return result.release();
}

// Matrices page-locked by minhash_cuda_pin: handle -> the registered arrays
// (held, so their memory stays valid while registered) and the device mask.
struct Pinned {
  std::vector<PyObject *> arrays;
  uint32_t devices = 0;
};
std::unordered_map<unsigned long long, Pinned> g_pinned;
unsigned long long g_next_pin = 1;

void release_pinned(Pinned &p) {
  for (PyObject *a : p.arrays) {
    const void *ptr = PyArray_DATA(reinterpret_cast<PyArrayObject *>(a));
    Py_BEGIN_ALLOW_THREADS
    mhcuda_host_unregister(p.devices, ptr);
    Py_END_ALLOW_THREADS
    Py_DECREF(a);
  }
  p.arrays.clear();
}

// minhash_cuda_pin(matrix, devices=0) -> handle.  Page-locks the float32
// data and 32-bit indices/indptr of a CSR matrix in place, so that
// minhash_cuda_calc copies them to the device directly -- the case of a large
// matrix hashed in several row_start/row_finish blocks, several times or by
// several generators.  The arrays are kept alive until minhash_cuda_unpin.
PyObject *py_pin(PyObject *, PyObject *args, PyObject *kwargs) {
  static const char *kw[] = {"matrix", "devices", nullptr};
  PyObject *m = nullptr;
  unsigned int devices = 0;
  if (!PyArg_ParseTupleAndKeywords(args, kwargs, "O|I", const_cast<char **>(kw), &m, &devices))
    return nullptr;
  Csr v;
  if (!csr_view(m, &v, /*wide=*/true)) return nullptr;
  const bool native = v.wtype == mhcudaFloat32 &&
                      (v.ctype == mhcudaUInt32 || v.ctype == mhcudaInt32) &&
                      (v.rtype == mhcudaUInt32 || v.rtype == mhcudaInt32);
  const char *attrs[3] = {"data", "indices", "indptr"};
  PyArrayObject *views[3] = {v.data.arr(), v.indices.arr(), v.indptr.arr()};
  Pinned p;
  p.devices = devices;
  for (int i = 0; i < 3; ++i) {
    // Only the matrix's own arrays: pinning a converted copy would not
    // reach the buffers the calls read.
    Ref own(PyObject_GetAttrString(m, attrs[i]));
    if (!native || !own || !PyArray_Check(own.get()) ||
        PyArray_DATA(reinterpret_cast<PyArrayObject *>(own.get())) != PyArray_DATA(views[i])) {
      release_pinned(p);
      PyErr_SetString(PyExc_ValueError,
                      "minhash_cuda_pin needs contiguous float32 data and 32-bit indices and "
                      "indptr");
      return nullptr;
    }
    const void *ptr = PyArray_DATA(views[i]);
    const uint64_t bytes = static_cast<uint64_t>(PyArray_NBYTES(views[i]));
    if (bytes == 0) continue;
    MHCUDAResult r;
    Py_BEGIN_ALLOW_THREADS
    r = mhcuda_host_register(devices, ptr, bytes);
    Py_END_ALLOW_THREADS
    if (!check(r, "minhash_cuda_pin")) {
      release_pinned(p);
      return nullptr;
    }
    Py_INCREF(reinterpret_cast<PyObject *>(views[i]));
    p.arrays.push_back(reinterpret_cast<PyObject *>(views[i]));
  }
  const unsigned long long h = g_next_pin++;
  g_pinned.emplace(h, std::move(p));
  return PyLong_FromUnsignedLongLong(h);
}

// minhash_cuda_unpin(handle): releases a minhash_cuda_pin registration.
PyObject *py_unpin(PyObject *, PyObject *args) {
  unsigned long long h = 0;
  if (!PyArg_ParseTuple(args, "K", &h)) return nullptr;
  auto it = g_pinned.find(h);
  if (it == g_pinned.end()) {
    PyErr_SetString(PyExc_ValueError, "minhash_cuda_unpin: unknown handle");
    return nullptr;
  }
  release_pinned(it->second);
  g_pinned.erase(it);
  Py_RETURN_NONE;
}

PyObject *py_fini(PyObject *, PyObject *args) {
  unsigned long long g = 0;
  if (!PyArg_ParseTuple(args, "K", &g)) return nullptr;
  MinhashCudaGenerator *gen = reinterpret_cast<MinhashCudaGenerator *>(static_cast<uintptr_t>(g));
  Py_BEGIN_ALLOW_THREADS
  mhcuda_fini(gen);
  Py_END_ALLOW_THREADS
  Py_RETURN_NONE;
}

PyMethodDef kMethods[] = {
    {"minhash_cuda_init", reinterpret_cast<PyCFunction>(reinterpret_cast<void (*)(void)>(py_init)),
     METH_VARARGS | METH_KEYWORDS, "Prepares Weighted Minhash internal state on GPU."},
    {"minhash_cuda_retrieve_vars", py_retrieve_vars, METH_VARARGS,
     "Copies the random variables rs, ln_cs and betas from the generator to the host."},
    {"minhash_cuda_assign_vars", py_assign_vars, METH_VARARGS,
     "Assigns random variables rs, ln_cs and betas to the generator."},
    {"minhash_cuda_assign_random_vars", py_assign_vars, METH_VARARGS,
     "Alias of minhash_cuda_assign_vars."},
    {"minhash_cuda_calc", reinterpret_cast<PyCFunction>(reinterpret_cast<void (*)(void)>(py_calc)),
     METH_VARARGS | METH_KEYWORDS, "Calculates Weighted Minhashes."},
    {"minhash_cuda_calc_batch", py_calc_batch, METH_VARARGS,
     "Calculates Weighted Minhashes of several CSR matrices in one device pass."},
    {"minhash_cuda_fini", py_fini, METH_VARARGS, "Disposes Weighted Minhash internal state on GPU."},
    {"minhash_cuda_pin", reinterpret_cast<PyCFunction>(reinterpret_cast<void (*)(void)>(py_pin)),
     METH_VARARGS | METH_KEYWORDS,
     "Page-locks a CSR matrix's arrays in place for direct copies; returns a handle."},
    {"minhash_cuda_unpin", py_unpin, METH_VARARGS, "Releases a minhash_cuda_pin handle."},
    {nullptr, nullptr, 0, nullptr}};

PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "libMHCUDA",
                       "Weighted MinHash (Ioffe) on one NVIDIA B200, drop-in for libMHCUDA.", -1,
                       kMethods, nullptr, nullptr, nullptr, nullptr};

}  // namespace

PyMODINIT_FUNC PyInit_libMHCUDA(void) {
  PyObject *m = PyModule_Create(&kModule);
  if (!m) return nullptr;
  import_array();
  return m;
}
