// Entries of the background and Recfast thermal history.  discoeb_background (host): the double
// pass for the values, one forward-mode pass per parameter direction for the tangents, each
// direction on its own host thread.  discoeb_background_batch (device): the same passes for many
// cosmologies at once, one GPU thread per (cosmology, pass), each with its own workspace.
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <type_traits>
#include <vector>

#include "background.cuh"
#include "discoeb.h"

namespace {

using dscb::bgn::Fw;
using dscb::bgn::Params;

BGF int64_t layout_size(int N)
{
    return (int64_t)DISCOEB_BGS_COUNT + (int64_t)DISCOEB_BGN_COUNT * DISCOEB_NU_KNOTS + (int64_t)DISCOEB_BGT_COUNT * N;
}

template <class T> void run(const Params<T>& P, int N, std::vector<T>& buf)
{
    const int64_t size = layout_size(N);
    buf.assign((size_t)size + (size_t)dscb::bgn::bg_work_count(N), T(0.0));
    std::vector<double> agrid((size_t)N + 1);
    T* scal = buf.data();
    T* nu = scal + DISCOEB_BGS_COUNT;
    T* th = nu + (size_t)DISCOEB_BGN_COUNT * DISCOEB_NU_KNOTS;
    dscb::bgn::evolve_background_core(P, N, scal, nu, th, buf.data() + size, agrid.data());
}

BGF Params<double> params_of(const DiscoebCosmoParams& c)
{
    Params<double> p;
    p.H0 = c.H0; p.Omegab = c.Omegab; p.Omegam = c.Omegam; p.mnu = c.mnu; p.w0 = c.w_DE_0; p.wa = c.w_DE_a;
    p.Tcmb = c.Tcmb; p.YHe = c.YHe; p.Neff = c.Neff; p.Nmnu = c.Nmnu; p.cs2_DE = c.cs2_DE; p.Omegak = c.Omegak;
    return p;
}

BGF Params<Fw<double>> params_dual(const DiscoebCosmoParams& c, const DiscoebCosmoParams& d)
{
    Params<Fw<double>> p;
    p.H0 = Fw<double>(c.H0, d.H0);
    p.Omegab = Fw<double>(c.Omegab, d.Omegab);
    p.Omegam = Fw<double>(c.Omegam, d.Omegam);
    p.mnu = Fw<double>(c.mnu, d.mnu);
    p.w0 = Fw<double>(c.w_DE_0, d.w_DE_0);
    p.wa = Fw<double>(c.w_DE_a, d.w_DE_a);
    p.Tcmb = c.Tcmb; p.YHe = c.YHe; p.Neff = c.Neff; p.Nmnu = c.Nmnu; p.cs2_DE = c.cs2_DE; p.Omegak = c.Omegak;
    return p;
}

// bytes of one device thread's workspace: the output image, the core's work arrays, the a-grid
template <class T> size_t thread_bytes(int N)
{
    const size_t b = sizeof(T) * ((size_t)layout_size(N) + (size_t)dscb::bgn::bg_work_count(N)) +
                     sizeof(double) * ((size_t)N + 1);
    return (b + 255) & ~(size_t)255;
}

// one thread per (cosmology c, pass d): T = double gives the values (one pass per cosmology),
// T = Fw<double> the values and the tangent along direction d
template <class T>
__global__ void __launch_bounds__(64) background_batch_kernel(const DiscoebCosmoParams* __restrict__ par,
                                                              const DiscoebCosmoParams* __restrict__ dots,
                                                              int n_cosmo, int n_pass, int N, unsigned char* ws,
                                                              size_t per_thread, double* out, double* out_dot)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_cosmo * n_pass) return;
    const int c = t / n_pass, d = t - c * n_pass;
    const int64_t size = layout_size(N);
    T* buf = reinterpret_cast<T*>(ws + (size_t)t * per_thread);
    double* agrid = reinterpret_cast<double*>(buf + size + dscb::bgn::bg_work_count(N));
    T* scal = buf;
    T* nu = scal + DISCOEB_BGS_COUNT;
    T* th = nu + (size_t)DISCOEB_BGN_COUNT * DISCOEB_NU_KNOTS;
    if constexpr (std::is_same<T, double>::value) {
        dscb::bgn::evolve_background_core(params_of(par[c]), N, scal, nu, th, buf + size, agrid);
        double* o = out + (size_t)c * size;
        for (int64_t i = 0; i < size; ++i) o[i] = buf[i];
    } else {
        dscb::bgn::evolve_background_core(params_dual(par[c], dots[(size_t)c * n_pass + d]), N, scal, nu, th,
                                          buf + size, agrid);
        double* od = out_dot + ((size_t)c * n_pass + d) * size;
        for (int64_t i = 0; i < size; ++i) od[i] = buf[i].d;
        if (d == 0) {
            double* o = out + (size_t)c * size;
            for (int64_t i = 0; i < size; ++i) o[i] = buf[i].v;
        }
    }
}

}  // namespace

extern "C" int64_t discoeb_background_batch_workspace_bytes(int32_t n_cosmo, int32_t n_dir, int32_t num_thermo)
{
    if (n_cosmo < 1 || n_dir < 0 || num_thermo < 32) return -1;
    const size_t per = n_dir == 0 ? thread_bytes<double>(num_thermo) : thread_bytes<Fw<double>>(num_thermo);
    return (int64_t)(per * (size_t)n_cosmo * (size_t)(n_dir == 0 ? 1 : n_dir));
}

extern "C" int32_t discoeb_background_batch(const DiscoebCosmoParams* par_dev, const DiscoebCosmoParams* par_dot_dev,
                                            int32_t n_cosmo, int32_t n_dir, int32_t num_thermo, void* workspace,
                                            int64_t workspace_bytes, double* out_dev, double* out_dot_dev, void* stream)
{
    if (!par_dev || !out_dev || !workspace || n_cosmo < 1 || n_dir < 0 || num_thermo < 32 ||
        (n_dir > 0 && (!par_dot_dev || !out_dot_dev)))
        return DISCOEB_EINVAL;
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return DISCOEB_EINVAL;
    if (workspace_bytes < discoeb_background_batch_workspace_bytes(n_cosmo, n_dir, num_thermo)) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    const int n_pass = n_dir == 0 ? 1 : n_dir;
    const int threads = n_cosmo * n_pass, block = 64, grid = (threads + block - 1) / block;
    if (n_dir == 0)
        background_batch_kernel<double><<<grid, block, 0, s>>>(par_dev, nullptr, n_cosmo, 1, num_thermo, ws,
                                                               thread_bytes<double>(num_thermo), out_dev, nullptr);
    else
        background_batch_kernel<Fw<double>><<<grid, block, 0, s>>>(par_dev, par_dot_dev, n_cosmo, n_dir, num_thermo,
                                                                   ws, thread_bytes<Fw<double>>(num_thermo), out_dev,
                                                                   out_dot_dev);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

extern "C" int64_t discoeb_background_size(int32_t num_thermo)
{
    return num_thermo < 32 ? -1 : layout_size(num_thermo);
}

extern "C" int32_t discoeb_background(const DiscoebCosmoParams* par, const DiscoebCosmoParams* par_dot,
                                      int32_t n_dir, int32_t num_thermo, double* out, double* out_dot,
                                      int32_t n_threads)
{
    if (!par || !out || num_thermo < 32 || n_dir < 0 || (n_dir > 0 && (!par_dot || !out_dot))) return DISCOEB_EINVAL;
    const int N = num_thermo;
    const int64_t size = layout_size(N);
    if (n_dir == 0) {
        std::vector<double> buf;
        run(params_of(*par), N, buf);
        std::copy(buf.begin(), buf.begin() + size, out);
        return DISCOEB_SUCCESS;
    }
    // each direction's pass also yields the values (its value part is the double computation);
    // direction 0 writes them
    auto one = [&](int d) {
        std::vector<Fw<double>> buf;
        run(params_dual(*par, par_dot[d]), N, buf);
        double* od = out_dot + (int64_t)d * size;
        for (int64_t i = 0; i < size; ++i) od[i] = buf[(size_t)i].d;
        if (d == 0)
            for (int64_t i = 0; i < size; ++i) out[i] = buf[(size_t)i].v;
    };
    int nt = n_threads > 0 ? n_threads : n_dir;
    nt = std::max(1, std::min(nt, n_dir));
    if (nt == 1) {
        for (int d = 0; d < n_dir; ++d) one(d);
        return DISCOEB_SUCCESS;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t]() {
            for (int d = t; d < n_dir; d += nt) one(d);
        });
    for (auto& th : pool) th.join();
    return DISCOEB_SUCCESS;
}

// Knot second derivatives of the natural cubic spline through (x[i], y[i]), i < n: the Thomas
// recurrence of the reference's spline_interpolation (spline_interpolation.py:19-75), operation
// for operation (host code, IEEE double, no contraction), so that host tables built here equal
// those of the Python restatement bit for bit.
extern "C" int32_t discoeb_natural_spline_second(int32_t n, const double* x, const double* y, double* S)
{
    if (n < 2 || !x || !y || !S) return DISCOEB_EINVAL;
    S[0] = 0.0;
    S[n - 1] = 0.0;
    const int m = n - 2;
    if (m <= 0) return DISCOEB_SUCCESS;
    std::vector<double> cp(m), dp(m);
    for (int i = 0; i < m; ++i) {
        const double h0 = x[i + 1] - x[i], h1 = x[i + 2] - x[i + 1];
        const double a = h0, b = 2.0 * (h0 + h1), c = h1;
        const double d = 6.0 * ((y[i + 2] - y[i + 1]) / h1 - (y[i + 1] - y[i]) / h0);
        if (i == 0) {
            cp[0] = c / b;
            dp[0] = d / b;
        } else {
            const double denom = b - a * cp[i - 1];
            cp[i] = (i < m - 1) ? c / denom : 0.0;
            dp[i] = (d - a * dp[i - 1]) / denom;
        }
    }
    S[m] = dp[m - 1];
    for (int i = m - 2; i >= 0; --i) S[i + 1] = dp[i] - cp[i] * S[i + 2];
    return DISCOEB_SUCCESS;
}
