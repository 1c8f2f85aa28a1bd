// Host-side helper of the Python batch constructor (libuva_pyhost.so, loaded
// with the GIL held): one pass over the charts list that reads, through the
// buffer protocol, each chart's position, triangle and UV array: data
// pointer, rows and element code, for the arrays the parallel host copies
// read as they are (C-contiguous, two dimensions, 3 or 2 columns, float32 /
// float64 positions and UVs, int32 / int64 triangles). A chart with any
// other array gets ok = 0 and is prepared by the Python path. Separate from
// libuva_b200.so, whose C ABI stays free of the Python runtime.
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

namespace {

// Element code of a buffer format: floats 0 float32 / 1 float64, ints 0
// int32 / 1 int64; -1 for anything else.
int float_code(const char* f) {
    if (!f) return -1;
    if (*f == '<' || *f == '=' || *f == '@') ++f;
    if (f[0] == 'f' && f[1] == 0) return 0;
    if (f[0] == 'd' && f[1] == 0) return 1;
    return -1;
}

int int_code(const char* f, Py_ssize_t itemsize) {
    if (!f) return -1;
    if (*f == '<' || *f == '=' || *f == '@') ++f;
    if (f[1] != 0) return -1;
    switch (f[0]) {
        case 'i': case 'l': case 'q':
            return itemsize == 4 ? 0 : (itemsize == 8 ? 1 : -1);
        default:
            return -1;
    }
}

// Data pointer, rows and code of a C-contiguous 2-D buffer with `width`
// columns; false when the object is not one.
bool probe(PyObject* o, int width, bool is_int, uint64_t* ptr, int64_t* rows, int8_t* code) {
    if (!PyObject_CheckBuffer(o)) return false;
    Py_buffer v;
    if (PyObject_GetBuffer(o, &v, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) != 0) {
        PyErr_Clear();
        return false;
    }
    bool ok = v.ndim == 2 && v.shape && v.shape[1] == width;
    int c = -1;
    if (ok) c = is_int ? int_code(v.format, v.itemsize) : float_code(v.format);
    ok = ok && c >= 0;
    if (ok) {
        *ptr = reinterpret_cast<uint64_t>(v.buf);
        *rows = static_cast<int64_t>(v.shape[0]);
        *code = static_cast<int8_t>(c);
    }
    PyBuffer_Release(&v);   // the array itself stays referenced by the charts list
    return ok;
}

}  // namespace

// charts: a list or tuple of sequences (P, T[, U]). Per chart i: pp / pdt /
// nv of P (n x 3), tp / tdt / nt of T (t x 3), up / udt of U (n x 2, udt -1:
// none or None), ok[i] = 1 when all present arrays passed. Returns the
// number of charts, or -1 (a Python error is set) when `charts` is not a
// list or tuple or an item is not a sequence of at least two.
extern "C" int64_t uva_py_charts(PyObject* charts, int32_t with_uv, uint64_t* pp, int8_t* pdt, uint64_t* tp,
                                 int8_t* tdt, uint64_t* up, int8_t* udt, int64_t* nv, int64_t* nt, int8_t* ok) {
    PyObject* seq = PySequence_Fast(charts, "uva_py_charts: charts must be a sequence");
    if (!seq) return -1;
    const Py_ssize_t n = PySequence_Fast_GET_SIZE(seq);
    PyObject** items = PySequence_Fast_ITEMS(seq);
    for (Py_ssize_t i = 0; i < n; ++i) {
        PyObject* ch = items[i];
        ok[i] = 0;
        udt[i] = -1;
        up[i] = 0;
        const Py_ssize_t len = PySequence_Size(ch);
        if (len < 2) {
            if (len < 0) PyErr_Clear();
            continue;   // the Python path reports it
        }
        PyObject* a = PySequence_GetItem(ch, 0);
        PyObject* t = PySequence_GetItem(ch, 1);
        bool good = a && t && probe(a, 3, false, pp + i, nv + i, pdt + i) && probe(t, 3, true, tp + i, nt + i, tdt + i);
        if (good && with_uv && len > 2) {
            PyObject* u = PySequence_GetItem(ch, 2);
            if (!u) {
                PyErr_Clear();
                good = false;
            } else {
                if (u != Py_None) {
                    int64_t urows = 0;
                    good = probe(u, 2, false, up + i, &urows, udt + i) && urows == nv[i];
                }
                Py_DECREF(u);
            }
        }
        if (!a || !t) PyErr_Clear();
        Py_XDECREF(a);
        Py_XDECREF(t);
        ok[i] = good ? 1 : 0;
    }
    Py_DECREF(seq);
    return static_cast<int64_t>(n);
}
