/*
 * qs_fast.c — a CPython extension that forwards the per-gate calls of the
 * blackwell_kernels API (and the measurement and sampling calls) to libqsim's C ABI
 * with no argument marshalling.
 *
 * The reference binds its kernels with pybind11 (bwk/csrc/apply_gate_sm120.cu:
 * 398-489); through ctypes the same calls spend about 1.5 us each converting
 * arguments, more than the gate kernel itself at 20 qubits.  These functions
 * take the handle, state and gate as integers (raw pointers obtained on the
 * Python side) and call the declared entry points of include/qsim.h
 * directly; a non-zero status raises the exception class given to set_error
 * (qsim_b200's QsimError, a RuntimeError) with qs_last_error's text.
 * No torch type crosses into C.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>

#include "../../include/qsim.h"

/* Exception class for a non-zero status (set_error; RuntimeError until then),
 * constructed as cls(status, message). */
static PyObject* g_error = NULL;

static PyObject* fail(void* h, int rc) {
  const char* m = qs_last_error((qs_handle_t)h);
  if (!g_error) {
    PyErr_Format(PyExc_RuntimeError, "qsim error %d: %s", rc, m ? m : "");
    return NULL;
  }
  PyObject* e = PyObject_CallFunction(g_error, "is", rc, m ? m : "");
  if (e) {
    PyErr_SetObject((PyObject*)Py_TYPE(e), e);
    Py_DECREF(e);
  }
  return NULL;
}

static PyObject* f_set_error(PyObject* self, PyObject* cls) {
  Py_XDECREF(g_error);
  g_error = Py_NewRef(cls);
  return Py_NewRef(Py_None);
}

#define PTR(i) PyLong_AsVoidPtr(args[i])
#define INT(i) ((int)PyLong_AsLong(args[i]))

static int check_n(Py_ssize_t nargs, Py_ssize_t want) {
  if (nargs != want) {
    PyErr_Format(PyExc_TypeError, "expected %zd arguments, got %zd", want, nargs);
    return 0;
  }
  return 1;
}

/* controls: a Python sequence of at most QS_MAX_CONTROLS ints */
static int controls_of(PyObject* seq, int* out, int* n) {
  PyObject* f = PySequence_Fast(seq, "controls must be a sequence");
  if (!f) return 0;
  const Py_ssize_t k = PySequence_Fast_GET_SIZE(f);
  if (k > QS_MAX_CONTROLS) {
    Py_DECREF(f);
    PyErr_SetString(PyExc_RuntimeError, "controls must have 0-7 elements");
    return 0;
  }
  for (Py_ssize_t i = 0; i < k; ++i) out[i] = (int)PyLong_AsLong(PySequence_Fast_GET_ITEM(f, i));
  Py_DECREF(f);
  *n = (int)k;
  return !PyErr_Occurred();
}

/* apply_1q_dev(h, state, n, gate, t) */
static PyObject* f_apply_1q_dev(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 5)) return NULL;
  void* h = PTR(0);
  const int rc = qs_apply_1q_dev((qs_handle_t)h, PTR(1), INT(2), PTR(3), INT(4));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* apply_gates_fused_dev(h, state, n, gates, targets, k) */
static PyObject* f_apply_gates_fused_dev(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 6)) return NULL;
  void* h = PTR(0);
  const int rc = qs_apply_gates_fused_dev((qs_handle_t)h, PTR(1), INT(2), PTR(3), PTR(4), INT(5));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* apply_2q_dev(h, state, n, gate, q0, q1) */
static PyObject* f_apply_2q_dev(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 6)) return NULL;
  void* h = PTR(0);
  const int rc = qs_apply_2q_dev((qs_handle_t)h, PTR(1), INT(2), PTR(3), INT(4), INT(5));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* apply_diag1_dev(h, state, n, diag, t) */
static PyObject* f_apply_diag1_dev(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 5)) return NULL;
  void* h = PTR(0);
  const int rc = qs_apply_diag1_dev((qs_handle_t)h, PTR(1), INT(2), PTR(3), INT(4));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* apply_diag2_dev(h, state, n, diag, q0, q1) */
static PyObject* f_apply_diag2_dev(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 6)) return NULL;
  void* h = PTR(0);
  const int rc = qs_apply_diag2_dev((qs_handle_t)h, PTR(1), INT(2), PTR(3), INT(4), INT(5));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* apply_phase(h, state, n, re, im, t) */
static PyObject* f_apply_phase(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 6)) return NULL;
  void* h = PTR(0);
  const float re = (float)PyFloat_AsDouble(args[3]), im = (float)PyFloat_AsDouble(args[4]);
  const int rc = qs_apply_phase((qs_handle_t)h, PTR(1), INT(2), re, im, INT(5));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* apply_mc1q_dev(h, state, n, gate, controls, t) */
static PyObject* f_apply_mc1q_dev(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 6)) return NULL;
  int c[QS_MAX_CONTROLS], nc = 0;
  if (!controls_of(args[4], c, &nc)) return NULL;
  void* h = PTR(0);
  const int rc = qs_apply_mc1q_dev((qs_handle_t)h, PTR(1), INT(2), PTR(3), c, nc, INT(5));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* apply_mc2q_dev(h, state, n, gate, controls, t0, t1) */
static PyObject* f_apply_mc2q_dev(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 7)) return NULL;
  int c[QS_MAX_CONTROLS], nc = 0;
  if (!controls_of(args[4], c, &nc)) return NULL;
  void* h = PTR(0);
  const int rc = qs_apply_mc2q_dev((qs_handle_t)h, PTR(1), INT(2), PTR(3), c, nc, INT(5), INT(6));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

/* measure(h, state, n, t, u) -> outcome (0 or 1) */
static PyObject* f_measure(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 5)) return NULL;
  void* h = PTR(0);
  const double u = PyFloat_AsDouble(args[4]);
  int outcome = 0;
  const int rc = qs_measure((qs_handle_t)h, PTR(1), INT(2), INT(3), u, &outcome);
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : PyLong_FromLong(outcome);
}

/* sample(h, state, n, u, nshots, out) */
static PyObject* f_sample(PyObject* self, PyObject* const* args, Py_ssize_t nargs) {
  if (!check_n(nargs, 6)) return NULL;
  void* h = PTR(0);
  const long long nshots = PyLong_AsLongLong(args[4]);
  const int rc = qs_sample((qs_handle_t)h, PTR(1), INT(2), (const double*)PTR(3), (int64_t)nshots, (int64_t*)PTR(5));
  if (PyErr_Occurred()) return NULL;
  return rc ? fail(h, rc) : Py_NewRef(Py_None);
}

static PyMethodDef kMethods[] = {
    {"set_error", (PyCFunction)f_set_error, METH_O, "exception class raised for a non-zero status"},
    {"apply_1q_dev", (PyCFunction)(void (*)(void))f_apply_1q_dev, METH_FASTCALL, "qs_apply_1q_dev"},
    {"apply_2q_dev", (PyCFunction)(void (*)(void))f_apply_2q_dev, METH_FASTCALL, "qs_apply_2q_dev"},
    {"apply_gates_fused_dev", (PyCFunction)(void (*)(void))f_apply_gates_fused_dev, METH_FASTCALL,
     "qs_apply_gates_fused_dev"},
    {"apply_diag1_dev", (PyCFunction)(void (*)(void))f_apply_diag1_dev, METH_FASTCALL, "qs_apply_diag1_dev"},
    {"apply_diag2_dev", (PyCFunction)(void (*)(void))f_apply_diag2_dev, METH_FASTCALL, "qs_apply_diag2_dev"},
    {"apply_phase", (PyCFunction)(void (*)(void))f_apply_phase, METH_FASTCALL, "qs_apply_phase"},
    {"apply_mc1q_dev", (PyCFunction)(void (*)(void))f_apply_mc1q_dev, METH_FASTCALL, "qs_apply_mc1q_dev"},
    {"apply_mc2q_dev", (PyCFunction)(void (*)(void))f_apply_mc2q_dev, METH_FASTCALL, "qs_apply_mc2q_dev"},
    {"measure", (PyCFunction)(void (*)(void))f_measure, METH_FASTCALL, "qs_measure"},
    {"sample", (PyCFunction)(void (*)(void))f_sample, METH_FASTCALL, "qs_sample"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef kModule = {PyModuleDef_HEAD_INIT, "_qsfast",
                                     "Direct calls into libqsim's per-gate entry points.", -1, kMethods};

PyMODINIT_FUNC PyInit__qsfast(void) { return PyModule_Create(&kModule); }
