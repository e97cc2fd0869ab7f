// Test harness: the FFTLog coefficient helpers of lngamma.cuh (complex log-Gamma, digamma, the
// kernel coefficient M_l(p) and its derivative along the grid spacing) compiled for the host, so
// that they can be compared with scipy and with difference quotients on a CPU.  Test
// infrastructure only; the library that ships is the CUDA build of the same header.
#include "lngamma.cuh"

using namespace dscb::cplx;

extern "C" {

void shim_lngamma(double re, double im, double* out)
{
    const Cx v = lngamma_c(cx(re, im));
    out[0] = v.re;
    out[1] = v.im;
}

void shim_digamma(double re, double im, double* out)
{
    const Cx v = digamma_c(cx(re, im));
    out[0] = v.re;
    out[1] = v.im;
}

void shim_mcoef(int l, int q, int n_fft, double bias, double dl, double dl_dot, double* b, double* b_dot)
{
    fftlog_mcoef(l, q, n_fft, bias, dl, dl_dot, b, b_dot);
}

void shim_mcoef_run(int l0, int count, int q, int n_fft, double bias, double dl, double dl_dot, double* b,
                    double* b_dot)
{
    fftlog_mcoef_run(l0, count, q, n_fft, bias, dl, dl_dot, 2, b, b_dot);
}

}  // extern "C"
