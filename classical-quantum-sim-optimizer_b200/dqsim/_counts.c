/* Builds the {bitstring: count} dictionary that simulate_shots returns.
 *
 * The C ABI hands back the distinct count keys as one buffer of fixed-width
 * ASCII bitstrings and their counts as uint64 (dq_counts_copy).  At 30 qubits
 * and 10^5 shots nearly every key is distinct, and building 10^5 strings and
 * dictionary entries in the interpreter took about as long as sampling itself;
 * this module builds them directly with the CPython API: one ASCII string per
 * key, the dictionary sized for all keys up front.
 *
 * build(keys: bytes-like, width: int, counts: bytes-like of uint64) -> dict
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

static PyObject* build(PyObject* self, PyObject* args) {
    (void)self;
    Py_buffer keys, counts;
    Py_ssize_t width;
    if (!PyArg_ParseTuple(args, "y*ny*", &keys, &width, &counts)) return NULL;
    PyObject* out = NULL;
    const Py_ssize_t n = counts.len / 8;
    if (width < 0 || counts.len % 8 != 0 || keys.len < n * width) {
        PyErr_SetString(PyExc_ValueError, "counts buffers do not match");
        goto done;
    }
#if PY_VERSION_HEX >= 0x030D0000
    out = PyDict_New();  /* the presizing helper is private from 3.13 on */
#else
    out = _PyDict_NewPresized(n);
#endif
    if (!out) goto done;
    const char* k = (const char*)keys.buf;
    const unsigned char* c = (const unsigned char*)counts.buf;
    for (Py_ssize_t i = 0; i < n; i++) {
        PyObject* key = PyUnicode_New(width, 127);
        if (!key) goto fail;
        memcpy(PyUnicode_1BYTE_DATA(key), k + i * width, (size_t)width);
        uint64_t v;
        memcpy(&v, c + 8 * i, 8);
        PyObject* val = PyLong_FromUnsignedLongLong(v);
        if (!val) {
            Py_DECREF(key);
            goto fail;
        }
        const int rc = PyDict_SetItem(out, key, val);
        Py_DECREF(key);
        Py_DECREF(val);
        if (rc < 0) goto fail;
    }
    goto done;
fail:
    Py_CLEAR(out);
done:
    PyBuffer_Release(&keys);
    PyBuffer_Release(&counts);
    return out;
}

static PyMethodDef methods[] = {
    {"build", build, METH_VARARGS, "build(keys, width, counts) -> {key: count}"},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_counts", NULL, -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__counts(void) { return PyModule_Create(&module); }
