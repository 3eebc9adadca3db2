/* Test infrastructure (oracle only): exported entry points for the reference's
 * own MoG evaluators, whose C text oracle/build_ref.sh copies verbatim out of
 * tractor/mix.i into ref_mix_blocks.c.  The functions there are `static`, so
 * this file includes that text and re-exports them unchanged.
 *
 *   c_gauss_2d_grid     tractor/mix.i:452-524
 *   c_gauss_2d_approx3  tractor/approx3.c:1-465 (declared mix.i:1095-1113)
 *   c_gauss_2d_masked   tractor/gauss_masked.c:1-159 (mix.i:1116-1128)
 *
 * Called through ctypes.PyDLL with py_object arguments (numpy arrays), as
 * SWIG's generated wrapper would pass them.
 */
#include <Python.h>
#include "ref_mix_blocks.c"

int ref_mix_init(void) {
    if (_import_array() < 0) {
        PyErr_Print();
        return -1;
    }
    return 0;
}

int ref_c_gauss_2d_grid(int x0, int x1, int y0, int y1, double fx, double fy,
                        PyObject* amp, PyObject* mean, PyObject* var,
                        PyObject* result) {
    return c_gauss_2d_grid(x0, x1, y0, y1, fx, fy, amp, mean, var, result);
}

int ref_c_gauss_2d_approx3(int x0, int x1, int y0, int y1, double fx,
                           double fy, double minval, PyObject* amp,
                           PyObject* mean, PyObject* var, PyObject* result,
                           PyObject* xderiv, PyObject* yderiv, int xc, int yc,
                           int minradius, int* sx0, int* sx1, int* sy0,
                           int* sy1) {
    return c_gauss_2d_approx3(x0, x1, y0, y1, fx, fy, minval, amp, mean, var,
                              result, xderiv, yderiv, xc, yc, minradius,
                              sx0, sx1, sy0, sy1);
}

int ref_c_gauss_2d_masked(int x0, int y0, int W, int H, double fx, double fy,
                          PyObject* amp, PyObject* mean, PyObject* var,
                          PyObject* result, PyObject* xderiv,
                          PyObject* yderiv, PyObject* mask) {
    return c_gauss_2d_masked(x0, y0, W, H, fx, fy, amp, mean, var, result,
                             xderiv, yderiv, mask);
}
