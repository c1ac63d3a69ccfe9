/* ha_pyfast.c -- CPython entry point for the host-buffer throughput loop.
 *
 * ha_throughput_host_ex_c takes about 48 us per call on a B200, of which the
 * ctypes wrapper adds about 4 (argument conversion, the foreign call).  This
 * module calls the same C ABI function from a METH_FASTCALL function: eleven
 * integer arguments, in the C ABI's order, converted without building a
 * ctypes call frame.  The GIL is released around the call, as ctypes does.
 * It is a binding, not another implementation: the work is done by
 * libhalloc_b200.so.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>

#include "halloc_c.h"

/* throughput_host(h_sizes, d_sizes, nbytes, nthreads, block, nallocs, niters,
 *                 d_out, h_out, transfer, stream) -> the C ABI's return code */
static PyObject *throughput_host(PyObject *self, PyObject *const *args, Py_ssize_t nargs) {
  (void)self;
  if (nargs != 11) {
    PyErr_SetString(PyExc_TypeError, "throughput_host takes 11 integer arguments");
    return NULL;
  }
  unsigned long long v[11];
  for (int i = 0; i < 11; i++) {
    v[i] = PyLong_AsUnsignedLongLong(args[i]);
    if (v[i] == (unsigned long long)-1 && PyErr_Occurred()) return NULL;
  }
  /* nbytes, nthreads, block, nallocs, niters and transfer are 32-bit */
  static const int narrow[] = {2, 3, 4, 5, 6, 9};
  for (int i = 0; i < 6; i++) {
    if (v[narrow[i]] > 0xffffffffull) {
      PyErr_Format(PyExc_OverflowError, "argument %d does not fit in 32 bits", narrow[i]);
      return NULL;
    }
  }
  int rc;
  Py_BEGIN_ALLOW_THREADS
  rc = ha_throughput_host_ex_c((const uint32_t *)(uintptr_t)v[0], (uint32_t *)(uintptr_t)v[1],
                               (uint32_t)v[2], (uint32_t)v[3], (uint32_t)v[4], (uint32_t)v[5],
                               (uint32_t)v[6], (uint64_t *)(uintptr_t)v[7],
                               (uint64_t *)(uintptr_t)v[8], (uint32_t)v[9], (void *)(uintptr_t)v[10]);
  Py_END_ALLOW_THREADS
  return PyLong_FromLong(rc);
}

static PyMethodDef methods[] = {
    {"throughput_host", (PyCFunction)(void (*)(void))throughput_host, METH_FASTCALL,
     "ha_throughput_host_ex_c with plain integer arguments"},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_pyfast", NULL, -1, methods,
                                    NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pyfast(void) { return PyModule_Create(&module); }
