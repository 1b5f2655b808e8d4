/* Per-execute call into the provider's C ABI from Python without ctypes argument marshalling.
 *
 * Plan.execute calls execute(fn, plan, in, out, stream, err, cap): fn is the address of the
 * provider table's execute entry (syclfft_b200_provider_v1::execute, whose signature this
 * file repeats), the rest its arguments as Python ints (pointers and the error-buffer
 * address). ctypes spends about two microseconds converting those arguments; a FASTCALL
 * function reads them directly. The GIL is released around the call, as ctypes does. */
#define PY_SSIZE_T_CLEAN
#include <Python.h>

typedef int (*execute_fn)(void *plan, const void *in, void *out, void *stream, char *err, size_t cap);

static PyObject *fc_execute(PyObject *self, PyObject *const *args, Py_ssize_t nargs) {
    (void)self;
    if (nargs != 7) {
        PyErr_SetString(PyExc_TypeError, "execute(fn, plan, in, out, stream, err, cap) takes 7 arguments");
        return NULL;
    }
    void *p[6];
    for (int i = 0; i < 6; ++i) {
        p[i] = args[i] == Py_None ? NULL : PyLong_AsVoidPtr(args[i]);
        if (p[i] == NULL && PyErr_Occurred()) return NULL;
    }
    const size_t cap = PyLong_AsSize_t(args[6]);
    if (cap == (size_t)-1 && PyErr_Occurred()) return NULL;
    if (p[0] == NULL) {
        PyErr_SetString(PyExc_ValueError, "null execute entry");
        return NULL;
    }
    execute_fn fn = (execute_fn)p[0];
    int rc;
    Py_BEGIN_ALLOW_THREADS
    rc = fn(p[1], p[2], p[3], p[4], (char *)p[5], cap);
    Py_END_ALLOW_THREADS
    return PyLong_FromLong(rc);
}

static PyMethodDef fc_methods[] = {
    {"execute", (PyCFunction)(void (*)(void))fc_execute, METH_FASTCALL, "Call a provider execute entry."},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef fc_module = {PyModuleDef_HEAD_INIT, "_fastcall", NULL, -1, fc_methods,
                                       NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__fastcall(void) { return PyModule_Create(&fc_module); }
