// Observables of the linear power spectrum (perturbations.py:1409-1569 and util.py:291-327 of the
// reference): the field amplitudes sqrt(P) of the output fields, a Savitzky-Golay smoothed log P(k),
// the Kaiser redshift-space P(k, mu), its multipoles l = 0, 2, 4, and the FFTLog correlation
// function xi_l(r) (cuFFT D2Z / Z2D around a phase kernel with the complex log Gamma).
//
// Elementwise kernels: one thread per output entry, grid-stride loops.  All arrays are device
// arrays of the caller; the FFTLog call takes a caller workspace (discoeb_xi_workspace_bytes).
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdint>

#include "discoeb.h"
#include "fft_plans.cuh"
#include "lngamma.cuh"

using namespace dscb::cplx;

namespace {

int blocks_for(long long n, int threads)
{
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
}

// squared = 0: amp_i = sqrt(2 pi^2 A_s (k_i/k_p)^(n_s-1) k_i^-3) y[i, idx]   (perturbations.py:1515-1516)
// squared = 1: P_i = 2 pi^2 A_s (k_i/k_p)^(n_s-1) k_i^-3 y[i, idx]^2        (get_power, :1468)
__global__ void amplitude_kernel(int n_k, const double* __restrict__ k, const double* __restrict__ y, int stride,
                                 int idx, double A_s, double n_s, double k_p, int squared, double* amp)
{
    const double fac = 2.0 * (M_PI * M_PI) * A_s;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_k; i += gridDim.x * blockDim.x) {
        const double yi = y[(size_t)i * stride + idx];
        const double w = fac * pow(k[i] / k_p, n_s - 1.0) * pow(k[i], -3.0);
        amp[i] = squared ? w * (yi * yi) : sqrt(w) * yi;
    }
}

// out = exp(convolve(log P, c, 'same')) in the interior; the first w/2 and the last (w+1)/2 entries
// keep P (perturbations.py:1481-1490; numpy's convolve 'same' zero-pads log P)
__global__ void savgol_kernel(int n_k, const double* __restrict__ P, int w, const double* __restrict__ c, double* out)
{
    const int h = (w - 1) / 2;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_k; i += gridDim.x * blockDim.x) {
        if (i < w / 2 || i >= n_k - (w + 1) / 2) {
            out[i] = P[i];
            continue;
        }
        double acc = 0.0;
        for (int j = 0; j < w; ++j) {
            const int m = i + h - j;
            if (m >= 0 && m < n_k) acc += c[j] * log(P[m]);
        }
        out[i] = exp(acc);
    }
}

// P(k_i, mu_j) = (b delta_i - mu_j^2 theta_i)^2   (perturbations.py:1520-1523)
__global__ void kaiser_kernel(int n_k, const double* __restrict__ delta, const double* __restrict__ theta, double b,
                              int n_mu, const double* __restrict__ mu, double* pkmu)
{
    const long long n = (long long)n_k * n_mu;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n_mu), j = (int)(t - (long long)i * n_mu);
        const double v = b * delta[i] - (mu[j] * mu[j]) * theta[i];
        pkmu[t] = v * v;
    }
}

// multipoles of the Kaiser spectrum (perturbations.py:1559-1562)
__global__ void multipole_kernel(int n_k, const double* __restrict__ delta, const double* __restrict__ theta, double b,
                                 double* P0, double* P2, double* P4)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_k; i += gridDim.x * blockDim.x) {
        const double d = delta[i], th = theta[i];
        P0[i] = (b * b) * (d * d) - 2.0 * b / 3.0 * d * th + 0.2 * (th * th);
        P2[i] = -4.0 * b / 3.0 * d * th + 4.0 / 7.0 * (th * th);
        P4[i] = 8.0 / 35.0 * (th * th);
    }
}

// FFTLog (perturbations.py:1409-1442): f_i = P_i k_i^1.5 before the forward transform
__global__ void xi_in_kernel(int n_k, const double* __restrict__ k, const double* __restrict__ Pk, double* f)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_k; i += gridDim.x * blockDim.x)
        f[i] = Pk[i] * pow(k[i], 1.5);
}

// F_m *= exp(2i (Im lnGamma((1.5 + l)/2 + i kappa_m) - ln(pi) kappa_m)), kappa_m = pi m / ln(k_max/k_min)
__global__ void xi_phase_kernel(int n_k, const double* __restrict__ k, int n_freq, int ell, double* F)
{
    const double L = log(k[n_k - 1] / k[0]);
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n_freq; m += gridDim.x * blockDim.x) {
        const double ki = M_PI * m / L;
        const double th = lngamma_c(cx(0.5 * (1.5 + ell), ki)).im;
        double sn, cs;
        sincos(2.0 * (th - log(M_PI) * ki), &sn, &cs);
        double* c = F + 2 * (size_t)m;
        const double re = c[0], im = c[1];
        c[0] = re * cs - im * sn;
        c[1] = re * sn + im * cs;
    }
}

// xi and r in increasing r (the reverse of the k order), with the inverse transform's 1/N and the
// factor Re(i^l) (the reference takes the real part of i^l times a real array)
__global__ void xi_out_kernel(int n_k, const double* __restrict__ k, const double* __restrict__ g, double sign,
                              double* xi, double* r)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_k; i += gridDim.x * blockDim.x) {
        const double ri = 2.0 * M_PI / k[i];
        xi[n_k - 1 - i] = sign * (g[i] / n_k) / pow(2.0 * M_PI * ri, 1.5);
        r[n_k - 1 - i] = ri;
    }
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// workspace: real buffer [N], complex buffer [N/2 + 1], cuFFT work area (shared by both plans)
struct XiLayout {
    size_t f, F, work, total, cufft_bytes;
};

// the cached forward (D2Z) and inverse (Z2D) plans of one length-n transform; the caller holds
// discoeb_fft::plan_mutex()
int xi_plans(int n, cufftHandle* fwd, cufftHandle* inv, size_t* work)
{
    size_t w1 = 0, w2 = 0;
    const long long nf = n / 2 + 1;
    if (!discoeb_fft::cached_plan(CUFFT_D2Z, n, 1, n, nf, fwd, &w1) ||
        !discoeb_fft::cached_plan(CUFFT_Z2D, n, 1, nf, n, inv, &w2))
        return DISCOEB_ECUDA;
    *work = w1 > w2 ? w1 : w2;
    return DISCOEB_SUCCESS;
}

XiLayout xi_layout(int n, size_t cufft_bytes)
{
    XiLayout L;
    size_t o = 0;
    L.f = o;
    o = align256(o + sizeof(double) * (size_t)n);
    L.F = o;
    o = align256(o + 2 * sizeof(double) * (size_t)(n / 2 + 1));
    L.work = o;
    o = align256(o + cufft_bytes);
    L.total = o;
    L.cufft_bytes = cufft_bytes;
    return L;
}

}  // namespace

extern "C" {

int32_t discoeb_power_amplitudes(int32_t n_k, const double* kmodes, const double* y, int32_t y_stride, int32_t idx,
                                 double A_s, double n_s, double k_p, int32_t squared, double* amp, void* stream)
{
    if (n_k < 1 || !kmodes || !y || !amp || idx < 0 || y_stride <= idx) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    amplitude_kernel<<<blocks_for(n_k, 128), 128, 0, s>>>(n_k, kmodes, y, y_stride, idx, A_s, n_s, k_p, squared != 0,
                                                          amp);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

int32_t discoeb_savgol_log_power(int32_t n_k, const double* P, int32_t window_length, const double* coeffs,
                                 double* out, void* stream)
{
    if (n_k < 1 || !P || !coeffs || !out || window_length < 1 || window_length % 2 == 0) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    savgol_kernel<<<blocks_for(n_k, 128), 128, 0, s>>>(n_k, P, window_length, coeffs, out);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

int32_t discoeb_power_kaiser(int32_t n_k, const double* delta, const double* theta, double bias, int32_t n_mu,
                             const double* mu, double* pkmu, void* stream)
{
    if (n_k < 1 || n_mu < 1 || !delta || !theta || !mu || !pkmu) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    kaiser_kernel<<<blocks_for((long long)n_k * n_mu, 256), 256, 0, s>>>(n_k, delta, theta, bias, n_mu, mu, pkmu);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

int32_t discoeb_power_multipoles(int32_t n_k, const double* delta, const double* theta, double b, double* P0,
                                 double* P2, double* P4, void* stream)
{
    if (n_k < 1 || !delta || !theta || !P0 || !P2 || !P4) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    multipole_kernel<<<blocks_for(n_k, 128), 128, 0, s>>>(n_k, delta, theta, b, P0, P2, P4);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

int64_t discoeb_xi_workspace_bytes(int32_t n_k)
{
    if (n_k < 2 || n_k % 2 != 0) return -1;
    cufftHandle a, b;
    size_t work = 0;
    std::lock_guard<std::mutex> lock(discoeb_fft::plan_mutex());
    if (xi_plans(n_k, &a, &b, &work) != DISCOEB_SUCCESS) return -1;
    return (int64_t)xi_layout(n_k, work).total;
}

int32_t discoeb_xi_from_power(int32_t n_k, const double* kmodes, const double* Pk, int32_t ell, void* workspace,
                              int64_t workspace_bytes, double* xi, double* r, void* stream)
{
    if (n_k < 2 || n_k % 2 != 0 || ell < 0 || !kmodes || !Pk || !workspace || !xi || !r) return DISCOEB_EINVAL;
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return DISCOEB_EINVAL;
    cufftHandle fwd, inv;
    size_t work = 0;
    std::lock_guard<std::mutex> lock(discoeb_fft::plan_mutex());
    if (xi_plans(n_k, &fwd, &inv, &work) != DISCOEB_SUCCESS) return DISCOEB_ECUDA;
    const XiLayout L = xi_layout(n_k, work);
    if ((int64_t)L.total > workspace_bytes) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(workspace);
    double* f = reinterpret_cast<double*>(ws + L.f);
    double* F = reinterpret_cast<double*>(ws + L.F);
    int rc = DISCOEB_SUCCESS;
    const int n_freq = n_k / 2 + 1;
    // Re(i^l): 1, 0, -1, 0 for l = 0, 1, 2, 3 (mod 4)
    const double sign = (ell % 2 == 1) ? 0.0 : ((ell % 4 == 0) ? 1.0 : -1.0);
    cufftSetWorkArea(fwd, ws + L.work);
    cufftSetWorkArea(inv, ws + L.work);
    cufftSetStream(fwd, s);
    cufftSetStream(inv, s);
    xi_in_kernel<<<blocks_for(n_k, 128), 128, 0, s>>>(n_k, kmodes, Pk, f);
    if (cufftExecD2Z(fwd, f, reinterpret_cast<cufftDoubleComplex*>(F)) != CUFFT_SUCCESS) rc = DISCOEB_ECUDA;
    if (rc == DISCOEB_SUCCESS) {
        xi_phase_kernel<<<blocks_for(n_freq, 128), 128, 0, s>>>(n_k, kmodes, n_freq, ell, F);
        if (cufftExecZ2D(inv, reinterpret_cast<cufftDoubleComplex*>(F), f) != CUFFT_SUCCESS) rc = DISCOEB_ECUDA;
    }
    if (rc == DISCOEB_SUCCESS) xi_out_kernel<<<blocks_for(n_k, 128), 128, 0, s>>>(n_k, kmodes, f, sign, xi, r);
    if (cudaGetLastError() != cudaSuccess) rc = DISCOEB_ECUDA;
    return rc;
}

}  // extern "C"
