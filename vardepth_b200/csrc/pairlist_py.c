/* _pairlist: the Python side of the pair-list drop-in (score_pairs / CudaPairHMM.score).
 *
 * gather(pairs) walks a sequence of (read, qualities, haplotype) triples once
 * and returns the pointer arrays of the reference's C calling convention
 * (caller/native/caller/batch_hmm.cpp:192: reads**, quals**, rn*, haps**,
 * hn*), pointing straight into the Python objects: a read or haplotype str
 * that is ASCII is used in place (CPython keeps it as one byte per character),
 * and so are bytes / bytearray / C-contiguous uint8 buffers of qualities.
 * Other quality containers (int lists and tuples, numpy arrays of another
 * dtype) are converted once per object into a bytes object that the returned
 * keep-alive list holds.  The caller must keep `pairs` (and the returned
 * tuple) alive while the pointers are used.
 *
 * Checks here are the ones that need Python objects, with the messages of
 * caller/native/caller/accelerator.py:25-40: a read or haplotype that is not
 * an ASCII str -> ValueError("Uppercase DNA required"); qualities that are not
 * integer Phred scores in [0, 255] -> ValueError("Base qualities must be
 * integer Phred scores in [0,255]"); a read/quality length mismatch ->
 * ValueError("Read/quality lengths differ").  The ACGTN content of the bases
 * is checked in the library (vd_score_pair_list).
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

static const char kDnaMsg[] = "Uppercase DNA required";
static const char kQualMsg[] = "Base qualities must be integer Phred scores in [0,255]";

/* Bases of a read or haplotype: an ASCII str, used in place. */
static int dna_view(PyObject* o, const char** p, Py_ssize_t* n) {
  if (!PyUnicode_Check(o) || !PyUnicode_IS_ASCII(o)) {
    PyErr_SetString(PyExc_ValueError, kDnaMsg);
    return -1;
  }
  *p = PyUnicode_AsUTF8AndSize(o, n); /* ASCII: the object's own bytes, no copy */
  return *p ? 0 : -1;
}

static int put_phred(double v, unsigned char* dst) {
  if (!(v >= 0.0 && v <= 255.0) || v != floor(v)) return -1;
  *dst = (unsigned char)v;
  return 0;
}

/* Qualities converted into a new bytes object (lists, tuples, numpy arrays of
 * other dtypes, any buffer that is not contiguous uint8). */
static PyObject* convert_quals(PyObject* o) {
  Py_buffer view;
  if (PyObject_CheckBuffer(o) && PyObject_GetBuffer(o, &view, PyBUF_RECORDS_RO) == 0) {
    PyObject* res = NULL;
    const char* f = view.format ? view.format : "B";
    if (*f == '<' || *f == '=' || *f == '@' || *f == '|') ++f;
    if (view.ndim > 1 || strlen(f) != 1 || !strchr("bBhHiIlLqQfd?", *f)) {
      PyBuffer_Release(&view);
      PyErr_SetString(PyExc_ValueError, kQualMsg);
      return NULL;
    }
    const Py_ssize_t n = view.ndim == 0 ? 1 : view.shape[0];
    const Py_ssize_t stride = view.ndim == 0 ? view.itemsize : (view.strides ? view.strides[0] : view.itemsize);
    res = PyBytes_FromStringAndSize(NULL, n);
    if (!res) { PyBuffer_Release(&view); return NULL; }
    unsigned char* dst = (unsigned char*)PyBytes_AS_STRING(res);
    for (Py_ssize_t i = 0; i < n; ++i) {
      const char* src = (const char*)view.buf + i * stride;
      double v;
      switch (*f) {
        case 'b': v = *(const signed char*)src; break;
        case 'B': case '?': v = *(const unsigned char*)src; break;
        case 'h': v = *(const short*)src; break;
        case 'H': v = *(const unsigned short*)src; break;
        case 'i': v = *(const int*)src; break;
        case 'I': v = *(const unsigned int*)src; break;
        case 'l': v = (double)*(const long*)src; break;
        case 'L': v = (double)*(const unsigned long*)src; break;
        case 'q': v = (double)*(const long long*)src; break;
        case 'Q': v = (double)*(const unsigned long long*)src; break;
        case 'f': v = *(const float*)src; break;
        default: v = *(const double*)src; break;
      }
      if (put_phred(v, dst + i)) {
        Py_DECREF(res);
        PyBuffer_Release(&view);
        PyErr_SetString(PyExc_ValueError, kQualMsg);
        return NULL;
      }
    }
    PyBuffer_Release(&view);
    if (view.ndim == 0) { /* a scalar is not a quality string */
      Py_DECREF(res);
      PyErr_SetString(PyExc_ValueError, kQualMsg);
      return NULL;
    }
    return res;
  }
  PyErr_Clear();
  PyObject* seq = PySequence_Fast(o, kQualMsg);
  if (!seq) {
    PyErr_SetString(PyExc_ValueError, kQualMsg);
    return NULL;
  }
  const Py_ssize_t n = PySequence_Fast_GET_SIZE(seq);
  PyObject* res = PyBytes_FromStringAndSize(NULL, n);
  if (!res) { Py_DECREF(seq); return NULL; }
  unsigned char* dst = (unsigned char*)PyBytes_AS_STRING(res);
  PyObject** items = PySequence_Fast_ITEMS(seq);
  for (Py_ssize_t i = 0; i < n; ++i) {
    PyObject* it = items[i];
    double v = -1.0;
    if (PyLong_Check(it)) {
      int overflow = 0;
      const long long x = PyLong_AsLongLongAndOverflow(it, &overflow);
      v = overflow ? -1.0 : (double)x;
    } else if (PyFloat_Check(it)) {
      v = PyFloat_AS_DOUBLE(it);
    } else {
      PyObject* f = PyNumber_Float(it); /* numpy scalars */
      if (!f) { PyErr_Clear(); v = -1.0; }
      else { v = PyFloat_AS_DOUBLE(f); Py_DECREF(f); }
    }
    if (put_phred(v, dst + i)) {
      Py_DECREF(res);
      Py_DECREF(seq);
      PyErr_SetString(PyExc_ValueError, kQualMsg);
      return NULL;
    }
  }
  Py_DECREF(seq);
  return res;
}

/* Qualities in place where the object already is contiguous bytes. */
static int qual_view(PyObject* o, const unsigned char** p, Py_ssize_t* n, PyObject* keep, PyObject* converted) {
  if (PyBytes_CheckExact(o)) {
    *p = (const unsigned char*)PyBytes_AS_STRING(o);
    *n = PyBytes_GET_SIZE(o);
    return 0;
  }
  if (PyByteArray_CheckExact(o)) {
    *p = (const unsigned char*)PyByteArray_AS_STRING(o);
    *n = PyByteArray_GET_SIZE(o);
    return 0;
  }
  /* one conversion per object: callers pass the same quality array with every haplotype */
  PyObject* key = PyLong_FromVoidPtr(o);
  if (!key) return -1;
  PyObject* done = PyDict_GetItemWithError(converted, key);
  if (!done && PyErr_Occurred()) { Py_DECREF(key); return -1; }
  if (!done) {
    Py_buffer view;
    int inplace = 0;
    if (PyObject_CheckBuffer(o) && PyObject_GetBuffer(o, &view, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) == 0) {
      const char* f = view.format ? view.format : "B";
      if (*f == '|' || *f == '=' || *f == '<' || *f == '@') ++f;
      inplace = view.ndim == 1 && view.itemsize == 1 && (strcmp(f, "B") == 0 || strcmp(f, "c") == 0);
      PyBuffer_Release(&view);
    } else {
      PyErr_Clear();
    }
    if (inplace) {
      done = o; /* the object's own memory (the caller keeps it alive) */
    } else {
      done = convert_quals(o);
      if (!done) { Py_DECREF(key); return -1; }
      if (PyList_Append(keep, done)) { Py_DECREF(done); Py_DECREF(key); return -1; }
      Py_DECREF(done); /* the keep list holds it */
    }
    /* the dict entry holds the source object too, so its address is not reused during the walk */
    PyObject* entry = PyTuple_Pack(2, done, o);
    if (!entry || PyDict_SetItem(converted, key, entry)) { Py_XDECREF(entry); Py_DECREF(key); return -1; }
    Py_DECREF(entry);
  } else {
    done = PyTuple_GET_ITEM(done, 0);
  }
  Py_DECREF(key);
  if (PyBytes_Check(done)) {
    *p = (const unsigned char*)PyBytes_AS_STRING(done);
    *n = PyBytes_GET_SIZE(done);
    return 0;
  }
  Py_buffer view;
  if (PyObject_GetBuffer(done, &view, PyBUF_C_CONTIGUOUS) != 0) return -1;
  *p = (const unsigned char*)view.buf;
  *n = view.len;
  PyBuffer_Release(&view); /* the exporter (kept alive by the caller) still owns the memory */
  return 0;
}

static PyObject* gather(PyObject* self, PyObject* args) {
  (void)self;
  PyObject* pairs;
  if (!PyArg_ParseTuple(args, "O", &pairs)) return NULL;
  PyObject* seq = PySequence_Fast(pairs, "pairs must be a sequence of (read, qualities, haplotype)");
  if (!seq) return NULL;
  const Py_ssize_t count = PySequence_Fast_GET_SIZE(seq);
  PyObject** items = PySequence_Fast_ITEMS(seq);
  PyObject* keep = PyList_New(0);
  PyObject* converted = PyDict_New();
  PyObject* reads = PyBytes_FromStringAndSize(NULL, count * (Py_ssize_t)sizeof(const char*));
  PyObject* quals = PyBytes_FromStringAndSize(NULL, count * (Py_ssize_t)sizeof(const unsigned char*));
  PyObject* haps = PyBytes_FromStringAndSize(NULL, count * (Py_ssize_t)sizeof(const char*));
  PyObject* rn = PyBytes_FromStringAndSize(NULL, count * (Py_ssize_t)sizeof(int));
  PyObject* hn = PyBytes_FromStringAndSize(NULL, count * (Py_ssize_t)sizeof(int));
  PyObject* result = NULL;
  if (!keep || !converted || !reads || !quals || !haps || !rn || !hn) goto done;
  {
    const char** rp = (const char**)PyBytes_AS_STRING(reads);
    const unsigned char** qp = (const unsigned char**)PyBytes_AS_STRING(quals);
    const char** hp = (const char**)PyBytes_AS_STRING(haps);
    int* rl = (int*)PyBytes_AS_STRING(rn);
    int* hl = (int*)PyBytes_AS_STRING(hn);
    PyObject* last_q = NULL; /* consecutive pairs usually share the read's quality object */
    const unsigned char* last_qp = NULL;
    Py_ssize_t last_qn = 0;
    for (Py_ssize_t i = 0; i < count; ++i) {
      PyObject* t = items[i];
      PyObject *s, *q, *h;
      if (PyTuple_CheckExact(t) && PyTuple_GET_SIZE(t) == 3) {
        s = PyTuple_GET_ITEM(t, 0);
        q = PyTuple_GET_ITEM(t, 1);
        h = PyTuple_GET_ITEM(t, 2);
      } else if (PyList_CheckExact(t) && PyList_GET_SIZE(t) == 3) {
        s = PyList_GET_ITEM(t, 0);
        q = PyList_GET_ITEM(t, 1);
        h = PyList_GET_ITEM(t, 2);
      } else {
        PyErr_SetString(PyExc_ValueError, "each pair must be (read, qualities, haplotype)");
        goto done;
      }
      Py_ssize_t n, m, nq;
      if (dna_view(s, &rp[i], &n) || dna_view(h, &hp[i], &m)) goto done;
      if (q == last_q) {
        qp[i] = last_qp;
        nq = last_qn;
      } else {
        if (qual_view(q, &qp[i], &nq, keep, converted)) goto done;
        last_q = q;
        last_qp = qp[i];
        last_qn = nq;
      }
      if (nq != n) {
        PyErr_SetString(PyExc_ValueError, "Read/quality lengths differ");
        goto done;
      }
      if (n > INT32_MAX || m > INT32_MAX) {
        PyErr_SetString(PyExc_ValueError, "read or haplotype longer than 2^31-1 bases");
        goto done;
      }
      rl[i] = (int)n;
      hl[i] = (int)m;
    }
    result = Py_BuildValue("(nOOOOOO)", count, reads, quals, rn, haps, hn, keep);
  }
done:
  Py_XDECREF(keep);
  Py_XDECREF(converted);
  Py_XDECREF(reads);
  Py_XDECREF(quals);
  Py_XDECREF(haps);
  Py_XDECREF(rn);
  Py_XDECREF(hn);
  Py_DECREF(seq);
  return result;
}

static PyMethodDef methods[] = {
    {"gather", gather, METH_VARARGS,
     "gather(pairs) -> (count, reads, quals, rn, haps, hn, keep): pointer arrays (bytes) of the "
     "reference's pair-list calling convention, pointing into the Python objects."},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_pairlist", NULL, -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pairlist(void) { return PyModule_Create(&module); }
