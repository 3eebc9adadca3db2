/* Test infrastructure (oracle only): an exported entry point for the
 * reference's EM fit of a Gaussian mixture to an image, whose C text
 * oracle/build_ref.sh copies verbatim out of tractor/emfit.i into
 * ref_emfit_blocks.c (static functions there; emfit2.c is #included from
 * where it lies in the reference tree).
 *
 *   em_fit_2d_reg   tractor/emfit.i:274-557
 *   em_fit_2d_reg2  tractor/emfit2.c (the EM fit with a flat sky term)
 *
 * Called through ctypes.PyDLL with py_object arguments (numpy arrays), as
 * SWIG's generated wrapper would pass them; amp / mean / var are updated in
 * place.
 */
#include <Python.h>
#include "ref_emfit_blocks.c"

int ref_emfit_init(void) {
    if (_import_array() < 0) {
        PyErr_Print();
        return -1;
    }
    return 0;
}

int ref_em_fit_2d_reg(PyObject* img, int x0, int y0, PyObject* amp, PyObject* mean,
                      PyObject* var, double alpha, int steps) {
    return em_fit_2d_reg(img, x0, y0, amp, mean, var, alpha, steps);
}

int ref_em_fit_2d_reg2(PyObject* img, int x0, int y0, PyObject* amp, PyObject* mean,
                       PyObject* var, double alpha, int steps, double approx, double* skyamp) {
    return em_fit_2d_reg2(img, x0, y0, amp, mean, var, alpha, steps, approx, skyamp);
}
