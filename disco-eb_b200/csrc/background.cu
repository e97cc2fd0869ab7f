// Host entry of the background and Recfast thermal history (discoeb_background): the double
// pass for the values, one forward-mode pass per parameter direction for the tangents, each
// direction on its own host thread.
#include <algorithm>
#include <thread>
#include <vector>

#include "background.cuh"
#include "discoeb.h"

namespace {

using dscb::bgn::Fw;
using dscb::bgn::Params;

int64_t layout_size(int N)
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

Params<double> params_of(const DiscoebCosmoParams& c)
{
    Params<double> p;
    p.H0 = c.H0; p.Omegab = c.Omegab; p.Omegam = c.Omegam; p.mnu = c.mnu; p.w0 = c.w_DE_0; p.wa = c.w_DE_a;
    p.Tcmb = c.Tcmb; p.YHe = c.YHe; p.Neff = c.Neff; p.Nmnu = c.Nmnu; p.cs2_DE = c.cs2_DE; p.Omegak = c.Omegak;
    return p;
}

Params<Fw<double>> params_dual(const DiscoebCosmoParams& c, const DiscoebCosmoParams& d)
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

}  // namespace

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
