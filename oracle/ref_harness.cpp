// Test-infrastructure harness around the reference (timo-eichhorn/Lettuce) CPU code.
//
// This file is NOT part of the product.  It is compiled by oracle/build_ref.py against a
// copy of the reference headers whose compile-time lattice extents
// (LettuceGauge/defines.hpp:34-37) are replaced by the macros LT_NT..LT_NZ, one shared
// library per extent tuple, into oracle/_ref/.  Tests and the CPU-baseline leg of bench.py
// load it through ctypes to
//   * pin the C restatement in oracle/lt_oracle.c against the reference itself, and
//   * generate the golden fixtures under tests/golden/.
// Every entry point calls the reference's own functions/functors; nothing here restates
// an algorithm.  Links cross this boundary in the reference AoS layout
// double[V][4][3][3][2] (site index ((t*Nx+x)*Ny+y)*Nz+z, mu fastest, row-major 3x3,
// re/im interleaved; LettuceGauge/lattice.hpp:366-382).
//
// Private members of the reference HMC functors (integrator hooks, Hamiltonian, the MetaD
// force) are reached by compiling the two HMC headers with `private` mapped to `public`;
// all standard, Eigen and other reference headers are included first so only those
// classes are affected.

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include <omp.h>
#include <Eigen/Dense>
#include <unsupported/Eigen/MatrixFunctions>
#include "PCG/pcg_random.hpp"

#include "LettuceGauge/defines.hpp"
#include "LettuceGauge/coords.hpp"
#include "LettuceGauge/lattice.hpp"
#include "LettuceGauge/actions/bias_potential/metadynamics.hpp"
#include "LettuceGauge/actions/gauge/rectangular_action.hpp"
#include "LettuceGauge/actions/gauge/wilson_action.hpp"
#include "LettuceGauge/iterators/iterators.hpp"
#include "LettuceGauge/math/su2.hpp"
#include "LettuceGauge/math/su3.hpp"
#include "LettuceGauge/math/su3_exp.hpp"
#include "LettuceGauge/observables/clover.hpp"
#include "LettuceGauge/observables/plaquette.hpp"
#include "LettuceGauge/observables/field_strength_tensor.hpp"
#include "LettuceGauge/observables/topological_charge.hpp"
#include "LettuceGauge/observables/wilson_loop.hpp"
#include "LettuceGauge/observables/polyakov_loop.hpp"
#include "LettuceGauge/smearing/stout_smearing.hpp"
#include "LettuceGauge/smearing/gradient_flow.hpp"
#include "LettuceGauge/updates/heatbath.hpp"
#include "LettuceGauge/updates/overrelaxation.hpp"
#include "LettuceGauge/IO/config_io/bmw_format.hpp"
#include "LettuceGauge/updates/parity_update.hpp"
#include "LettuceGauge/updates/tempering.hpp"
// Only the two HMC headers are compiled with `private` mapped to `public` (they hold no
// OpenMP `private(...)` clauses, which the mapping would break).
#define private public
#include "LettuceGauge/updates/hmc_gauge.hpp"
#include "LettuceGauge/updates/hmc_metadynamics.hpp"
#undef private

namespace
{
// The reference announces every field construction on std::cout (lattice.hpp:96-104); the
// harness runs inside other processes (tests, bench.py) whose stdout must stay clean.
const bool g_quiet = (std::cout.rdbuf(nullptr), true);

constexpr std::size_t kV = static_cast<std::size_t>(Nt) * Nx * Ny * Nz;
constexpr std::size_t kL = 4 * kV;

void load(GaugeField& U, const double* a)
{
    #pragma omp parallel for
    for (std::size_t l = 0; l < kL; ++l)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                const double* p = a + 18 * l + 2 * (3 * i + j);
                U(l)(i, j) = std::complex<double>(p[0], p[1]);
            }
}

void store(const GaugeField& U, double* a)
{
    #pragma omp parallel for
    for (std::size_t l = 0; l < kL; ++l)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                double* p = a + 18 * l + 2 * (3 * i + j);
                p[0] = std::real(U(l)(i, j));
                p[1] = std::imag(U(l)(i, j));
            }
}

void set_beta(double b)
{
    beta = b;                                  // defines.hpp:52 (used by HMC momentum update)
    GaugeAction::WilsonAction.SetBeta(b);      // rectangular_action.hpp:43
}

using PRNG = PRNG4D<Nt, Nx, Ny, Nz, pcg64, floatT, int>;
std::unique_ptr<PRNG> g_prng;

PRNG& prng()
{
    if (!g_prng)
    {
        auto gen = MakeRandomGenerator();
        g_prng = std::make_unique<PRNG>(gen);
    }
    return *g_prng;
}

// A bias whose grid holds V(Q) = slope * Q, so that MetaBiasPotential::ReturnDerivative
// returns `slope` (metadynamics.hpp:181-187) and the MetaD force is slope * dQ/dU.
std::unique_ptr<MetaBiasPotential> linear_bias(double slope)
{
    auto bias = std::make_unique<MetaBiasPotential>(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0);
    bias->GeneratePotentialFrom([slope](double cv) { return slope * cv; });
    return bias;
}
// The integrator hooks of HMCMetaDKernel with the Metadynamics momentum update preceded by
// CalculateTopologicalForce on the current links, so that the multiple-timescale integrators
// of hmc_metadynamics.hpp:26-238 apply the bias force of the field they are at (the kernel's
// own UpdateMetadynamicsMomenta, :478-491, adds the force it last stored).
template <typename KernelT>
struct RefreshedMetaD
{
    KernelT& k;
    void UpdateGaugeMomenta(const floatT e) { k.UpdateGaugeMomenta(e); }
    void UpdateMetadynamicsMomenta(const floatT e)
    {
        k.CalculateTopologicalForce();
        k.UpdateMetadynamicsMomenta(e);
    }
    void UpdateMomenta(const floatT e, const bool sub = false) { k.UpdateMomenta(e, sub); }
    void UpdateFields(const floatT e) { k.UpdateFields(e); }
};

// Run integrator `id` (the LT_MD_* numbering of the C ABI) of the reference on `kernel`
template <typename HMCFunctor>
bool run_integrator(int id, HMCFunctor& kernel, double tau, int n)
{
    using namespace Integrators::HMC;
    switch (id)
    {
    case 0: Leapfrog_slow{}(kernel, tau, n); return true;
    case 1: Leapfrog{}(kernel, tau, n); return true;
    case 2: OMF_2_slow{}(kernel, tau, n); return true;
    case 3: OMF_2{}(kernel, tau, n); return true;
    case 4: OMF_4_slow{}(kernel, tau, n); return true;
    case 5: OMF_4{}(kernel, tau, n); return true;
    default: return false;
    }
}
// Run f(action) with GaugeAction::Rectangular<radius>(beta, c_plaq, c_rect)
template <typename F>
void with_action(int radius, double b, double cp, double cr, F&& f)
{
    if (radius == 2)
    {
        GaugeAction::Rectangular<2> act(b, cp, cr);
        f(act);
    }
    else
    {
        GaugeAction::Rectangular<1> act(b, cp, cr);
        f(act);
    }
}

} // namespace

extern "C"
{
int ref_extent(int d)
{
    switch (d)
    {
        case 0: return Nt;
        case 1: return Nx;
        case 2: return Ny;
        case 3: return Nz;
        default: return 0;
    }
}

int ref_threads()
{
    return omp_get_max_threads();
}

// plaquette.hpp:26-43
double ref_plaquette_sum(const double* links)
{
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    return PlaquetteSum(*U);
}

// rectangular_action.hpp:61-94 with (c_plaq, c_rect) = (1, 0)
double ref_wilson_action(const double* links, double b)
{
    set_beta(b);
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    return GaugeAction::WilsonAction.Action(*U);
}

// rectangular_action.hpp:104-184 for every link
void ref_staples(const double* links, double* out)
{
    auto U = std::make_unique<GaugeField>();
    auto S = std::make_unique<GaugeField>();
    load(*U, links);
    #pragma omp parallel for collapse(2)
    for (int t = 0; t < Nt; ++t)
    for (int x = 0; x < Nx; ++x)
    for (int y = 0; y < Ny; ++y)
    for (int z = 0; z < Nz; ++z)
    for (int mu = 0; mu < 4; ++mu)
    {
        link_coord l {t, x, y, z, mu};
        (*S)(l) = GaugeAction::WilsonAction.Staple(*U, l);
    }
    store(*S, out);
}

// overrelaxation.hpp:68-117 driven by iterators.hpp:65-87
void ref_or_sweeps(double* links, int n)
{
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    OverrelaxationSubgroupKernel OR(*U, GaugeAction::WilsonAction);
    Iterator::Checkerboard(OR, n);
    store(*U, links);
}

void ref_reset_prng()
{
    g_prng.reset();
}

// Reseed the per-link pcg64 streams (PRNG4D::SeedPRNG, random/prng_wrapper.hpp:154-157):
// link i gets seed i + offset * (number of links), so chains with different offsets draw
// independent streams (FIXED_SEED seeds link i with i, prng_wrapper.hpp:104-109).
void ref_reseed(std::uint64_t offset)
{
    PRNG& p = prng();
    for (std::size_t i = 0; i < kL; ++i) p.SeedPRNG(i, i + offset * kL);
}

// heatbath.hpp:30-130 driven by iterators.hpp:65-87; the per-link pcg64 streams persist
// across calls until ref_reset_prng().
void ref_hb_sweeps(double* links, double b, int n)
{
    set_beta(b);
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    HeatbathKernel HB(*U, GaugeAction::WilsonAction, prng());
    Iterator::Checkerboard(HB, n);
    store(*U, links);
}

// n_sweep rounds of (n_hb heatbath + n_or overrelaxation), plaquette sum recorded after each round
void ref_hb_or_chain(double* links, double b, int n_sweep, int n_hb, int n_or, double* plaq)
{
    set_beta(b);
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    HeatbathKernel HB(*U, GaugeAction::WilsonAction, prng());
    OverrelaxationSubgroupKernel OR(*U, GaugeAction::WilsonAction);
    for (int s = 0; s < n_sweep; ++s)
    {
        Iterator::Checkerboard(HB, n_hb);
        Iterator::Checkerboard(OR, n_or);
        if (plaq) plaq[s] = PlaquetteSum(*U);
    }
    store(*U, links);
}

// gradient_flow.hpp:120-168 (RK3) and :252-367 (GradientFlowKernel)
void ref_flow_rk3(const double* in, double* out, double eps, int n_step)
{
    auto U0 = std::make_unique<GaugeField>();
    auto U1 = std::make_unique<GaugeField>();
    auto Z  = std::make_unique<GaugeField>();
    load(*U0, in);
    Integrators::GradientFlow::RK3 rk3(*Z);
    GradientFlowKernel Flow(*U0, *U1, rk3, GaugeAction::WilsonAction, eps);
    Flow(n_step);
    store(*U1, out);
}

// Flow with measurements every `every` steps: plaquette sum, clover Q (topological_charge.hpp:97-200)
// and clover energy density (field_strength_tensor.hpp:28-66, :107-134, :154-175).
void ref_flow_rk3_measure(const double* in, double eps, int n_meas, int every,
                          double* plaq, double* q, double* e)
{
    auto U0 = std::make_unique<GaugeField>();
    auto U1 = std::make_unique<GaugeField>();
    auto Z  = std::make_unique<GaugeField>();
    auto F  = std::make_unique<FullTensor>();
    load(*U0, in);
    Integrators::GradientFlow::RK3 rk3(*Z);
    GradientFlowKernel Flow(*U0, *U1, rk3, GaugeAction::WilsonAction, eps);
    for (int m = 0; m < n_meas; ++m)
    {
        if (m == 0) Flow(every); else Flow.Resume(every);
        plaq[m] = PlaquetteSum(*U1);
        q[m]    = TopChargeClover(*U1);
        FieldStrengthTensor::Clover(*U1, *F);
        FieldStrengthTensor::MakeComponentsTraceless(*F);
        e[m]    = EnergyDensity::Clover(*F);
    }
}

// stout_smearing.hpp:29-57 applied n times
void ref_stout(const double* in, double* out, double rho, int n)
{
    auto A = std::make_unique<GaugeField>();
    auto B = std::make_unique<GaugeField>();
    load(*A, in);
    for (int k = 0; k < n; ++k)
    {
        StoutSmearing4D(*A, *B, rho);
        std::swap(A, B);
    }
    store(*A, out);
}

// topological_charge.hpp:97-200
double ref_topcharge_clover(const double* links)
{
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    return TopChargeClover(*U);
}

// E = sum_{mu<nu} ReTr(F_munu^2) / V with the traceless clover F, as measured by the driver
// (SU3_main.cpp:128-141 through field_strength_tensor.hpp)
double ref_energy_clover(const double* links)
{
    auto U = std::make_unique<GaugeField>();
    auto F = std::make_unique<FullTensor>();
    load(*U, links);
    FieldStrengthTensor::Clover(*U, *F);
    FieldStrengthTensor::MakeComponentsTraceless(*F);
    return EnergyDensity::Clover(*F);
}

// Gauge force beta/6 * Algebra(st U^dagger) per link: the HMC momentum kick
// (hmc_gauge.hpp:450-464) applied with epsilon = 1 to zero momenta.
void ref_gauge_force(const double* links, double b, double* out)
{
    set_beta(b);
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    P->SetToZero();
    Integrators::HMC::OMF_2 omf2;
    RunStatistics stats;
    GaugeUpdates::HMCKernel hmc(*U, *Uc, *P, omf2, GaugeAction::WilsonAction, prng(), stats, std::cout, 1.0);
    hmc.UpdateMomenta(1.0);
    store(*P, out);
}

// dQ/dU_mu(x) of the clover charge on the given field (clover.hpp:94-152, :279-321)
void ref_clover_derivative(const double* links, double* out)
{
    auto U = std::make_unique<GaugeField>();
    auto C = std::make_unique<FullTensor>();
    auto D = std::make_unique<GaugeField>();
    load(*U, links);
    CalculateClover<1>(*U, *C);
    #pragma omp parallel for collapse(2)
    for (int t = 0; t < Nt; ++t)
    for (int x = 0; x < Nx; ++x)
    for (int y = 0; y < Ny; ++y)
    for (int z = 0; z < Nz; ++z)
    for (int mu = 0; mu < 4; ++mu)
    {
        site_coord s {t, x, y, z};
        (*D)(s, mu) = CloverDerivative(*U, *C, s, mu);
    }
    store(*D, out);
}

// CalculateClover<1, 1> (observables/clover.hpp:94-152) into the FullTensor layout
// double[V][4][4][3][3][2] (lattice.hpp:447-590), and TopChargeClover(const FullTensor&)
// (topological_charge.hpp:202-231) of that tensor
double ref_clover_tensor(const double* links, double* tensor_out)
{
    auto U = std::make_unique<GaugeField>();
    auto C = std::make_unique<FullTensor>();
    load(*U, links);
    CalculateClover<1>(*U, *C);
    for (std::size_t k = 0; k < kV * 16; ++k)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                tensor_out[18 * k + 6 * i + 2 * j]     = std::real((*C)(k)(i, j));
                tensor_out[18 * k + 6 * i + 2 * j + 1] = std::imag((*C)(k)(i, j));
            }
    return TopChargeClover(*C);
}

// The MetaD force chain of HMCMetaDKernel::CalculateTopologicalForce (hmc_metadynamics.hpp:374-436)
// with n_smear_meta (= 4, defines.hpp:74) stout levels of parameter rho, under a bias with
// dV/dQ = slope.  Writes ForceFatLink (the force on the thin links) and returns the CV.
double ref_metad_force(const double* links, double rho, double slope, double* out)
{
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    auto bias = linear_bias(slope);
    auto data = std::make_unique<GaugeUpdates::HMCMetaDData>(n_smear_meta);
    Integrators::HMC::OMF_2 omf2;
    RunStatistics stats;
    std::string log_path {"/dev/null"};
    GaugeUpdates::HMCMetaDKernel kern(*U, *Uc, *P, *bias, *data, omf2, GaugeAction::WilsonAction, prng(), stats,
                                      std::cout, log_path, 1.0, rho);
    kern.CalculateTopologicalForce(false);
    store(data->ForceFatLink, out);
    CalculateClover<1>(data->SmearedFields[n_smear_meta], data->Clover);
    return TopChargeClover(data->Clover);
}

// Wall-clock seconds of n calls of HMCMetaDKernel::CalculateTopologicalForce (the reference's
// MetaD force, hmc_metadynamics.hpp:374-436) on the given links, after one untimed call; the
// kernel, its fields and the bias are set up once outside the timed region.  For the CPU
// baseline of the force evaluations/s.
double ref_metad_force_seconds(const double* links, double rho, double slope, int n)
{
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    auto bias = linear_bias(slope);
    auto data = std::make_unique<GaugeUpdates::HMCMetaDData>(n_smear_meta);
    Integrators::HMC::OMF_2 omf2;
    RunStatistics stats;
    std::string log_path {"/dev/null"};
    GaugeUpdates::HMCMetaDKernel kern(*U, *Uc, *P, *bias, *data, omf2, GaugeAction::WilsonAction, prng(), stats,
                                      std::cout, log_path, 1.0, rho);
    kern.CalculateTopologicalForce(false);
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < n; ++k) kern.CalculateTopologicalForce(false);
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int ref_n_smear_meta()
{
    return n_smear_meta;
}

// Q after n_smear_meta stout steps (HMCMetaDKernel::MetaCharge, hmc_metadynamics.hpp:302-310)
double ref_metad_charge(const double* links, double rho)
{
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    auto bias = linear_bias(1.0);
    auto data = std::make_unique<GaugeUpdates::HMCMetaDData>(n_smear_meta);
    Integrators::HMC::OMF_2 omf2;
    RunStatistics stats;
    std::string log_path {"/dev/null"};
    GaugeUpdates::HMCMetaDKernel kern(*U, *Uc, *P, *bias, *data, omf2, GaugeAction::WilsonAction, prng(), stats,
                                      std::cout, log_path, 1.0, rho);
    return kern.MetaCharge();
}

// Deterministic OMF2 molecular dynamics from given links and momenta (hmc_gauge.hpp:155-190,
// :450-541).  Returns H before and after; links and momenta are updated in place.
void ref_omf2(double* links, double* momenta, double b, double tau, int n_step, double* h_old, double* h_new)
{
    set_beta(b);
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    load(*P, momenta);
    Integrators::HMC::OMF_2 omf2;
    RunStatistics stats;
    GaugeUpdates::HMCKernel hmc(*U, *Uc, *P, omf2, GaugeAction::WilsonAction, prng(), stats, std::cout, tau);
    *h_old = hmc.Hamiltonian();
    omf2(hmc, tau, n_step);
    *h_new = hmc.Hamiltonian();
    store(*U, links);
    store(*P, momenta);
}

// Deterministic OMF2 MetaD molecular dynamics (hmc_metadynamics.hpp:441-535) under a linear
// bias V(Q) = slope * Q.  Returns H + V before and after.
void ref_metad_omf2(double* links, double* momenta, double b, double tau, int n_step, double rho, double slope,
                    double* h_old, double* h_new)
{
    set_beta(b);
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    load(*P, momenta);
    auto bias = linear_bias(slope);
    auto data = std::make_unique<GaugeUpdates::HMCMetaDData>(n_smear_meta);
    Integrators::HMC::OMF_2 omf2;
    RunStatistics stats;
    std::string log_path {"/dev/null"};
    GaugeUpdates::HMCMetaDKernel kern(*U, *Uc, *P, *bias, *data, omf2, GaugeAction::WilsonAction, prng(), stats,
                                      std::cout, log_path, tau, rho);
    kern.cv_path_samples.clear();
    *h_old = kern.Hamiltonian() + bias->ReturnPotential(kern.MetaCharge());
    omf2(kern, tau, n_step);
    *h_new = kern.Hamiltonian() + bias->ReturnPotential(kern.MetaCharge());
    store(*U, links);
    store(*P, momenta);
}

// MetaBiasPotential (metadynamics.hpp:29-187): deposits then samples potential and derivative.
void ref_bias_probe(double cv_min, double cv_max, int bins, double weight, double width, double wt, double thr,
                    const double* deposits, int n_dep, int symmetric,
                    const double* probes, int n_probe, double* pot, double* der)
{
    MetaBiasPotential bias(cv_min, cv_max, bins, weight, width, wt, thr);
    std::vector<double> cvs(deposits, deposits + n_dep);
    if (symmetric) bias.UpdatePotentialSymmetric(cvs); else bias.UpdatePotential(cvs);
    for (int i = 0; i < n_probe; ++i)
    {
        pot[i] = bias.ReturnPotential(probes[i]);
        der[i] = bias.ReturnDerivative(probes[i]);
    }
}

// MetadynamicsTemperingKernel::operator() (updates/tempering.hpp:51-72) once, on the
// unbiased stream's links `links_u` (Gluon) and the biased stream's `links_temper`
// (Gluon_temper), with the bias of the reference driver (SU3_main.cpp:566-578) after
// well-tempered deposits at `deposits`, and CV_current = cv_current.  The kernel draws its
// uniform from a fresh FIXED_SEED generator; a second fresh generator gives the same first
// draw, recorded here.  out = {CV_new (MetaCharge of links_u), CV_old, delta_V_tempering,
// uniform, accepted, CV_current afterwards}; on acceptance the two fields come back swapped.
void ref_tempering(double* links_u, double* links_temper, double rho, double cv_current, const double* deposits,
                   int n_dep, double* out)
{
    auto U  = std::make_unique<GaugeField>();
    auto Ut = std::make_unique<GaugeField>();
    auto C1 = std::make_unique<GaugeField>();
    auto C2 = std::make_unique<GaugeField>();
    load(*U, links_u);
    load(*Ut, links_temper);
    MetaBiasPotential bias(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0);
    std::vector<double> cvs(deposits, deposits + n_dep);
    if (n_dep > 0) bias.UpdatePotential(cvs);
    bias.SetCV_current(cv_current);
    auto gen_probe = MakeRandomGenerator();
    PRNG probe(gen_probe);
    const double q = probe.UniformReal();
    auto gen = MakeRandomGenerator();
    auto p = std::make_unique<PRNG>(gen);
    RunStatistics stats;
    GaugeUpdates::MetadynamicsTemperingKernel<PRNG> kern(*U, *Ut, *C1, *C2, bias, *p, stats, rho);
    out[0] = kern.MetaCharge(*U, *C1, *C2, n_smear_meta, rho);
    out[1] = bias.ReturnCV_current();
    out[4] = kern() ? 1.0 : 0.0;
    out[2] = stats.delta_V_tempering;
    out[3] = q;
    out[5] = bias.ReturnCV_current();
    store(*U, links_u);
    store(*Ut, links_temper);
}

// A field kept resident in the library between calls, so timed CPU-baseline samples do
// not include the layout conversion of ref_* entry points above.
static std::unique_ptr<GaugeField> g_field, g_flowed, g_force;

void ref_field_load(const double* links)
{
    if (!g_field) g_field = std::make_unique<GaugeField>();
    load(*g_field, links);
}

void ref_field_store(double* links)
{
    if (g_field) store(*g_field, links);
}

// n_hb heatbath then n_or overrelaxation sweeps (Iterator::Checkerboard, iterators.hpp:65-87)
// on the resident field; returns the plaquette sum afterwards.
double ref_field_sweeps(double b, int n_hb, int n_or)
{
    set_beta(b);
    HeatbathKernel HB(*g_field, GaugeAction::WilsonAction, prng());
    OverrelaxationSubgroupKernel OR(*g_field, GaugeAction::WilsonAction);
    Iterator::Checkerboard(HB, n_hb);
    Iterator::Checkerboard(OR, n_or);
    return PlaquetteSum(*g_field);
}

// n_round rounds of (n_hb heatbath + n_or overrelaxation sweeps) on the resident field, as
// the reference driver's update loop runs them (SU3_main.cpp: Iterator::Checkerboard of the
// heatbath kernel, then of the overrelaxation kernel, per round); no observable in between.
// This is the timed CPU baseline.
void ref_field_rounds(double b, int n_round, int n_hb, int n_or)
{
    set_beta(b);
    HeatbathKernel HB(*g_field, GaugeAction::WilsonAction, prng());
    OverrelaxationSubgroupKernel OR(*g_field, GaugeAction::WilsonAction);
    for (int r = 0; r < n_round; ++r)
    {
        Iterator::Checkerboard(HB, n_hb);
        Iterator::Checkerboard(OR, n_or);
    }
}

// n RK3 flow steps of the resident field into a second resident field, nothing measured
// (the timed flow baseline)
void ref_field_flow_steps(double eps, int n)
{
    if (!g_flowed) g_flowed = std::make_unique<GaugeField>();
    if (!g_force) g_force = std::make_unique<GaugeField>();
    Integrators::GradientFlow::RK3 rk3(*g_force);
    GradientFlowKernel Flow(*g_field, *g_flowed, rk3, GaugeAction::WilsonAction, eps);
    Flow(n);
}

// n RK3 flow steps of the resident field into a second resident field; returns its plaquette sum
double ref_field_flow(double eps, int n)
{
    if (!g_flowed) g_flowed = std::make_unique<GaugeField>();
    if (!g_force) g_force = std::make_unique<GaugeField>();
    Integrators::GradientFlow::RK3 rk3(*g_force);
    GradientFlowKernel Flow(*g_field, *g_flowed, rk3, GaugeAction::WilsonAction, eps);
    Flow(n);
    return PlaquetteSum(*g_flowed);
}

// GradientFlowKernel with the Euler / RK2 / RK3 / RK3W7 integrator (gradient_flow.hpp:31-168)
void ref_flow(const double* in, double* out, double eps, int n, int integrator)
{
    auto U = std::make_unique<GaugeField>();
    auto V = std::make_unique<GaugeField>();
    auto F = std::make_unique<GaugeField>();
    load(*U, in);
    switch (integrator)
    {
        case 0: { Integrators::GradientFlow::Euler it(*F); GradientFlowKernel k(*U, *V, it, GaugeAction::WilsonAction, eps); k(n); break; }
        case 1: { Integrators::GradientFlow::RK2 it(*F); GradientFlowKernel k(*U, *V, it, GaugeAction::WilsonAction, eps); k(n); break; }
        case 2: { Integrators::GradientFlow::RK3 it(*F); GradientFlowKernel k(*U, *V, it, GaugeAction::WilsonAction, eps); k(n); break; }
        default: { Integrators::GradientFlow::RK3W7 it(*F); GradientFlowKernel k(*U, *V, it, GaugeAction::WilsonAction, eps); k(n); break; }
    }
    store(*V, out);
}

// The measurement bundle of SU3_main.cpp:89-235 on one field: out = {Symanzik action
// (normalised), TopChargePlaquette, W(L=2), W(L=4), W(L=8), Re P, Im P}; q_t, e_t = the
// clover charge and energy per timeslice (Nt each)
void ref_measure(const double* links, double b, double* out, double* q_t, double* e_t)
{
    auto U = std::make_unique<GaugeField>();
    auto chain = std::make_unique<GaugeField>();
    auto F = std::make_unique<FullTensor>();
    load(*U, links);
    GaugeAction::Rectangular<2> Symanzik(b, 1.0 + 8.0 * 1.0 / 12.0, -1.0 / 12.0);
    out[0] = Symanzik.ActionNormalized(*U);
    out[1] = TopChargePlaquette(*U);
    out[2] = WilsonLoop<0, 2, true>(*U, *chain);
    out[3] = WilsonLoop<2, 4, false>(*U, *chain);
    out[4] = WilsonLoop<4, 8, false>(*U, *chain);
    const std::complex<double> P = PolyakovLoop(*U);
    out[5] = std::real(P);
    out[6] = std::imag(P);
    FieldStrengthTensor::Clover(*U, *F);
    for (int t = 0; t < Nt; ++t) q_t[t] = TopChargeCloverTimeslice(*F, t);
    FieldStrengthTensor::MakeComponentsTraceless(*F);
    for (int t = 0; t < Nt; ++t) e_t[t] = EnergyDensity::CloverTimeslice(*F, t);
}

// SaveConfigBMW / SaveConfigBMWFull (IO/config_io/bmw_format.hpp:294-394, :564-645) of the
// given links to `path` (overwriting); returns 1 on success
int ref_save_bmw(const double* links, const char* path, int full)
{
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    return (full ? SaveConfigBMWFull(*U, path, true) : SaveConfigBMW(*U, path, true)) ? 1 : 0;
}

// LoadConfigBMW / LoadConfigBMWFull (bmw_format.hpp:153-290, :425-560) of `path` into
// links_out; returns 1 when the reference accepts the file (its links pass IsGroupElement)
int ref_load_bmw(const char* path, int full, double* links_out)
{
    auto U = std::make_unique<GaugeField>();
    const bool ok = full ? LoadConfigBMWFull(*U, path) : LoadConfigBMW(*U, path);
    store(*U, links_out);
    return ok ? 1 : 0;
}

// Deterministic molecular dynamics with any of the reference's integrators from given links
// and momenta: HMCKernel (metad = 0; ids 0-7, the friction variants 6 and 7 included) or
// HMCMetaDKernel under the linear bias slope * Q (metad = 1; ids 0-5 and the
// multiple-timescale ids 8-10).  Returns 0 for a combination the reference does not offer.
int ref_md_integrate(double* links, double* momenta, double b, double tau, int n_step, int id, int metad, double rho,
                     double slope, double* h_old, double* h_new)
{
    set_beta(b);
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    load(*P, momenta);
    RunStatistics stats;
    Integrators::HMC::OMF_2 omf2;
    bool ok = true;
    if (!metad)
    {
        GaugeUpdates::HMCKernel hmc(*U, *Uc, *P, omf2, GaugeAction::WilsonAction, prng(), stats, std::cout, tau);
        *h_old = hmc.Hamiltonian();
        if (id == 6) Integrators::HMC::Leapfrog_friction_slow{}(hmc, tau, n_step);
        else if (id == 7) Integrators::HMC::OMF_4_friction_slow{}(hmc, tau, n_step);
        else ok = run_integrator(id, hmc, tau, n_step);
        *h_new = hmc.Hamiltonian();
    }
    else
    {
        auto bias = linear_bias(slope);
        auto data = std::make_unique<GaugeUpdates::HMCMetaDData>(n_smear_meta);
        std::string log_path {"/dev/null"};
        GaugeUpdates::HMCMetaDKernel kern(*U, *Uc, *P, *bias, *data, omf2, GaugeAction::WilsonAction, prng(), stats,
                                          std::cout, log_path, tau, rho);
        kern.cv_path_samples.clear();
        *h_old = kern.Hamiltonian() + bias->ReturnPotential(kern.MetaCharge());
        RefreshedMetaD<decltype(kern)> hooks {kern};
        if (id == 8) Integrators::HMC::Leapfrog_OMF_4{}(hooks, tau, n_step);
        else if (id == 9) Integrators::HMC::OMF_2_OMF_4_slow{}(hooks, tau, n_step);
        else if (id == 10) Integrators::HMC::OMF_2_OMF_4{}(hooks, tau, n_step);
        else ok = run_integrator(id, kern, tau, n_step);
        *h_new = kern.Hamiltonian() + bias->ReturnPotential(kern.MetaCharge());
    }
    store(*U, links);
    store(*P, momenta);
    return ok ? 1 : 0;
}

// Rectangular<radius>::Staple (rectangular_action.hpp:236-246) for every link
void ref_action_staples(const double* links, double* out, int radius, double cp, double cr)
{
    auto U = std::make_unique<GaugeField>();
    auto S = std::make_unique<GaugeField>();
    load(*U, links);
    with_action(radius, 6.0, cp, cr, [&](auto& act) {
        #pragma omp parallel for collapse(2)
        for (int t = 0; t < Nt; ++t)
        for (int x = 0; x < Nx; ++x)
        for (int y = 0; y < Ny; ++y)
        for (int z = 0; z < Nz; ++z)
        for (int mu = 0; mu < 4; ++mu)
        {
            link_coord l {t, x, y, z, mu};
            (*S)(l) = act.Staple(*U, l);
        }
    });
    store(*S, out);
}

// n sweeps of OverrelaxationSubgroupKernel with the action over Iterator::Checkerboard4
// (iterators.hpp:141-166); every extent must be a multiple of 4 (the reference exits otherwise)
int ref_or_sweeps4(double* links, int n, int radius, double cp, double cr)
{
    if (Nt % 4 != 0 || Nx % 4 != 0 || Ny % 4 != 0 || Nz % 4 != 0) return 0;
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
    with_action(radius, 6.0, cp, cr, [&](auto& act) {
        OverrelaxationSubgroupKernel OR(*U, act);
        Iterator::Checkerboard4(OR, n);
    });
    store(*U, links);
    return 1;
}

// Gauge-only MD with integrator `id` (0-7) under Rectangular<radius>(beta, cp, cr): H before and after
int ref_md_action(double* links, double* momenta, double b, double tau, int n_step, int id, int radius, double cp,
                  double cr, double* h_old, double* h_new)
{
    set_beta(b);
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    auto P  = std::make_unique<GaugeField>();
    load(*U, links);
    load(*P, momenta);
    RunStatistics stats;
    Integrators::HMC::OMF_2 omf2;
    bool ok = true;
    with_action(radius, b, cp, cr, [&](auto& act) {
        GaugeUpdates::HMCKernel hmc(*U, *Uc, *P, omf2, act, prng(), stats, std::cout, tau);
        *h_old = hmc.Hamiltonian();
        if (id == 6) Integrators::HMC::Leapfrog_friction_slow{}(hmc, tau, n_step);
        else if (id == 7) Integrators::HMC::OMF_4_friction_slow{}(hmc, tau, n_step);
        else ok = run_integrator(id, hmc, tau, n_step);
        *h_new = hmc.Hamiltonian();
    });
    store(*U, links);
    store(*P, momenta);
    return ok ? 1 : 0;
}

// GradientFlowKernel with integrator 0-3 (Euler, RK2, RK3, RK3W7) and Rectangular<radius>
void ref_flow_action(const double* in, double* out, double eps, int n, int integrator, int radius, double cp, double cr)
{
    auto U = std::make_unique<GaugeField>();
    auto V = std::make_unique<GaugeField>();
    auto F = std::make_unique<GaugeField>();
    load(*U, in);
    with_action(radius, 6.0, cp, cr, [&](auto& act) {
        switch (integrator)
        {
            case 0: { Integrators::GradientFlow::Euler it(*F); GradientFlowKernel k(*U, *V, it, act, eps); k(n); break; }
            case 1: { Integrators::GradientFlow::RK2 it(*F); GradientFlowKernel k(*U, *V, it, act, eps); k(n); break; }
            case 2: { Integrators::GradientFlow::RK3 it(*F); GradientFlowKernel k(*U, *V, it, act, eps); k(n); break; }
            default: { Integrators::GradientFlow::RK3W7 it(*F); GradientFlowKernel k(*U, *V, it, act, eps); k(n); break; }
        }
    });
    store(*V, out);
}

// WilsonLoop<start, end, reset>(U, U_chain) (wilson_loop.hpp:63-124) with start/end among
// the instantiated pairs and U_chain kept in the library between calls
double ref_wilson_loop_chain(const double* links, int start, int end, int reset)
{
    static std::unique_ptr<GaugeField> chain;
    if (!chain) chain = std::make_unique<GaugeField>();
    auto U = std::make_unique<GaugeField>();
    load(*U, links);
#define LT_WL(S, E)                                                                               \
    if (start == S && end == E) return reset ? WilsonLoop<S, E, true>(*U, *chain) : WilsonLoop<S, E, false>(*U, *chain);
    LT_WL(0, 1) LT_WL(0, 2) LT_WL(0, 3) LT_WL(2, 4) LT_WL(4, 8) LT_WL(3, 5) LT_WL(1, 3) LT_WL(2, 3) LT_WL(5, 6)
#undef LT_WL
    return std::nan("");
}

// ParityUpdate (parity_update.hpp:22-47) in place
void ref_parity_update(double* links)
{
    auto U  = std::make_unique<GaugeField>();
    auto Uc = std::make_unique<GaugeField>();
    load(*U, links);
    ParityUpdate(*U, *Uc);
    store(*U, links);
}

// SU3::exp (su3_exp.hpp:419-425) of n traceless Hermitian matrices (18 doubles each)
void ref_su3_exp(const double* in, double* out, int n)
{
    for (int k = 0; k < n; ++k)
    {
        Matrix_3x3 M;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                M(i, j) = std::complex<double>(in[18 * k + 6 * i + 2 * j], in[18 * k + 6 * i + 2 * j + 1]);
        Matrix_SU3 E = SU3::exp(M);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                out[18 * k + 6 * i + 2 * j]     = std::real(E(i, j));
                out[18 * k + 6 * i + 2 * j + 1] = std::imag(E(i, j));
            }
    }
}
} // extern "C"
