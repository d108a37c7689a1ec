// Host-side parts of the C ABI that need no device: the seeded Haar-random start and the
// metadynamics bias potential (one 801-point grid; negligible next to the lattice work).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "lettuce_b200.h"
#include "lt_host.h"
#include "lt_math.cuh"

using cd = std::complex<double>;

namespace {

// Haar-random SU(3) matrix for link `link` (Mezzadri's method): a complex Gaussian 3x3
// matrix from Philox calls j = 0..8 of tag TAG_HAAR (Box-Muller), orthonormalised by
// Gram-Schmidt on its columns (the QR factor with positive diagonal R, which is Haar on
// U(3)), then divided by the principal cube root of its determinant.
void haar_link(uint32_t link, uint64_t seed, double* out)
{
    cd z[3][3];
    for (int j = 0; j < 9; ++j)
    {
        lt::U4 w = lt::philox4x32(link, 0u, 0u, (lt::TAG_HAAR << 24) | (uint32_t)j, (uint32_t)seed,
                                  (uint32_t)(seed >> 32));
        double u1 = lt::u01_from(w.x, w.y), u2 = lt::u01_from(w.z, w.w);
        double r = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::sqrt(0.5);
        z[j / 3][j % 3] = cd(r * std::cos(2.0 * M_PI * u2), r * std::sin(2.0 * M_PI * u2));
    }
    for (int c = 0; c < 3; ++c)
    {
        for (int p = 0; p < c; ++p)
        {
            cd d = 0.0;
            for (int r = 0; r < 3; ++r) d += std::conj(z[r][p]) * z[r][c];
            for (int r = 0; r < 3; ++r) z[r][c] -= d * z[r][p];
        }
        double n = 0.0;
        for (int r = 0; r < 3; ++r) n += std::norm(z[r][c]);
        n = 1.0 / std::sqrt(n);
        for (int r = 0; r < 3; ++r) z[r][c] *= n;
    }
    cd det = z[0][0] * (z[1][1] * z[2][2] - z[1][2] * z[2][1]) - z[0][1] * (z[1][0] * z[2][2] - z[1][2] * z[2][0])
           + z[0][2] * (z[1][0] * z[2][1] - z[1][1] * z[2][0]);
    cd inv = 1.0 / std::pow(det, 1.0 / 3.0);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
        {
            cd v = z[a][b] * inv;
            out[6 * a + 2 * b] = v.real();
            out[6 * a + 2 * b + 1] = v.imag();
        }
}

} // namespace

namespace lt {

void haar_links(const int ext[4], uint64_t seed, double* out)
{
    const long long nlink = 4LL * ext[0] * ext[1] * ext[2] * ext[3];
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (nlink < 4096) nt = 1;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([=] {
            for (long long l = t; l < nlink; l += nt) haar_link((uint32_t)l, seed, out + 18 * l);
        });
    for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------- bias potential
Bias::Bias(double cv_min_, double cv_max_, int bins_, double weight_, double width_, double wt_, double thr_)
    : cv_min(cv_min_), cv_max(cv_max_), bins(bins_), bin_width((cv_max_ - cv_min_) / bins_),
      bin_width_inv(1.0 / ((cv_max_ - cv_min_) / bins_)), weight(weight_), width(width_), wt(wt_), thr(thr_),
      grid((size_t)bins_ + 1, 0.0)
{
}

void Bias::update(double cv)
{
    if (mode == 1) update_binned(cv);
    else update_gaussian(cv);
}

// Gaussian-free binned deposit (not in the reference, whose deposits are Gaussians): the weight
// goes to the two grid points that bracket the CV, split linearly (cloud in cell), so the
// linearly interpolated potential (ReturnPotential) gains exactly `weight` of area per deposit
// and its value at a grid point rises by `weight`.  Each point's share is well-tempered by its
// own current value, exp(-V_i / wt), as the reference tempers each grid point
// (metadynamics.hpp:116-118).  A CV outside [cv_min, cv_max) deposits nothing -- there is no
// grid point to carry it -- and is counted in `exceeded` like the reference's out-of-range CVs.
void Bias::update_binned(double cv)
{
    if (!(cv >= cv_min && cv < cv_max))
    {
        ++exceeded;
        return;
    }
    // the bracketing points i, i + 1 (clamped against rounding at the upper edge) and the
    // linear share a of point i + 1
    const int i = std::min(std::max((int)std::floor((cv - cv_min) * bin_width_inv), 0), bins - 1);
    const double a = std::min(std::max((cv - (cv_min + i * bin_width)) * bin_width_inv, 0.0), 1.0);
    const double w0 = weight * (1.0 - a) * std::exp(-grid[i] / wt);
    const double w1 = weight * a * std::exp(-grid[i + 1] / wt);
    grid[i] += w0;
    grid[i + 1] += w1;
}

// UpdatePotential, well-tempered branch (metadynamics.hpp:103-124)
void Bias::update_gaussian(double cv)
{
    if (cv < cv_min || cv >= cv_max) ++exceeded;
    const double wis = 1.0 / (width * width);
    for (size_t i = 0; i < grid.size(); ++i)
    {
        const double d = cv - (cv_min + (double)i * bin_width);
        grid[i] += weight * std::exp(-0.5 * wis * d * d - grid[i] / wt);
    }
}

// ReturnPotential (metadynamics.hpp:151-179)
double Bias::potential(double cv) const
{
    const int i = (int)std::floor((cv - cv_min) * bin_width_inv);
    if ((unsigned)i < (unsigned)bins)
    {
        const double a = (cv - (cv_min + i * bin_width)) * bin_width_inv;
        return grid[i] * (1.0 - a) + a * grid[i + 1];
    }
    if (i < 0)
    {
        const double d = cv - cv_min;
        return grid.front() + thr * d * d;
    }
    const double d = cv - cv_max;
    return grid.back() + thr * d * d;
}

// ReturnDerivative (metadynamics.hpp:181-187)
double Bias::derivative(double cv) const
{
    const double h = 0.5 * bin_width;
    return bin_width_inv * (potential(cv + h) - potential(cv - h));
}

} // namespace lt

extern "C" {

int lt_haar_links(const int ext[4], uint64_t seed, double* links_out)
{
    if (!ext || !links_out) return lt::set_error(LT_ERR_ARG, "lt_haar_links: null pointer");
    for (int d = 0; d < 4; ++d)
        if (ext[d] < 2 || ext[d] % 2) return lt::set_error(LT_ERR_ARG, "lt_haar_links: extents must be even and >= 2");
    lt::haar_links(ext, seed, links_out);
    return LT_OK;
}

int lt_bias_create(double cv_min, double cv_max, int bin_number, double weight, double width,
                   double well_tempered_parameter, double threshold_weight, lt_bias** out)
{
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_bias_create: null output pointer");
    *out = nullptr;
    if (!(cv_min < cv_max)) return lt::set_error(LT_ERR_ARG, "CV_min < CV_max required");
    if (bin_number <= 0) return lt::set_error(LT_ERR_ARG, "bin_number > 0 required");
    auto* b = new (std::nothrow) lt::Bias(cv_min, cv_max, bin_number, weight, width, well_tempered_parameter,
                                          threshold_weight);
    if (!b) return lt::set_error(LT_ERR_NOMEM, "lt_bias_create: out of host memory");
    *out = reinterpret_cast<lt_bias*>(b);
    return LT_OK;
}

int lt_bias_destroy(lt_bias* b)
{
    delete reinterpret_cast<lt::Bias*>(b);
    return LT_OK;
}

int lt_bias_update(lt_bias* b, const double* cv, int n, int symmetric)
{
    if (!b || (n > 0 && !cv) || n < 0) return lt::set_error(LT_ERR_ARG, "lt_bias_update: bad arguments");
    auto* p = reinterpret_cast<lt::Bias*>(b);
    for (int k = 0; k < n; ++k)
    {
        p->update(cv[k]);
        if (symmetric) p->update(-cv[k]);
    }
    return LT_OK;
}

int lt_bias_set_update_mode(lt_bias* b, int mode)
{
    if (!b) return lt::set_error(LT_ERR_ARG, "lt_bias_set_update_mode: null bias");
    if (mode != LT_BIAS_GAUSSIAN && mode != LT_BIAS_BINNED)
        return lt::set_error(LT_ERR_ARG, "lt_bias_set_update_mode: unknown mode");
    reinterpret_cast<lt::Bias*>(b)->mode = mode;
    return LT_OK;
}

int lt_bias_get_update_mode(const lt_bias* b, int* mode)
{
    if (!b || !mode) return lt::set_error(LT_ERR_ARG, "lt_bias_get_update_mode: null pointer");
    *mode = reinterpret_cast<const lt::Bias*>(b)->mode;
    return LT_OK;
}

int lt_bias_potential(const lt_bias* b, double cv, double* out)
{
    if (!b || !out) return lt::set_error(LT_ERR_ARG, "lt_bias_potential: null pointer");
    *out = reinterpret_cast<const lt::Bias*>(b)->potential(cv);
    return LT_OK;
}

int lt_bias_derivative(const lt_bias* b, double cv, double* out)
{
    if (!b || !out) return lt::set_error(LT_ERR_ARG, "lt_bias_derivative: null pointer");
    *out = reinterpret_cast<const lt::Bias*>(b)->derivative(cv);
    return LT_OK;
}

int lt_bias_get_grid(const lt_bias* b, double* grid_out, int n)
{
    if (!b || !grid_out) return lt::set_error(LT_ERR_ARG, "lt_bias_get_grid: null pointer");
    auto* p = reinterpret_cast<const lt::Bias*>(b);
    if (n != (int)p->grid.size()) return lt::set_error(LT_ERR_ARG, "lt_bias_get_grid: n must be bin_number + 1");
    std::memcpy(grid_out, p->grid.data(), sizeof(double) * p->grid.size());
    return LT_OK;
}

int lt_bias_set_grid(lt_bias* b, const double* grid, int n)
{
    if (!b || !grid) return lt::set_error(LT_ERR_ARG, "lt_bias_set_grid: null pointer");
    auto* p = reinterpret_cast<lt::Bias*>(b);
    if (n != (int)p->grid.size()) return lt::set_error(LT_ERR_ARG, "lt_bias_set_grid: n must be bin_number + 1");
    std::memcpy(p->grid.data(), grid, sizeof(double) * p->grid.size());
    return LT_OK;
}

} // extern "C"
