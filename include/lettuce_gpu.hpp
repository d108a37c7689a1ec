// lettuce_gpu.hpp -- C++20 drop-in header over the lettuce_b200 C ABI.
//
// Keeps the call surface of the CPU reference timo-eichhorn/Lettuce (LettuceGauge/...) so
// that SU3_main.cpp-style host code recompiles against the B200 path with only its includes
// changed.  Differences that cannot be hidden:
//   * lattice extents are constructor arguments, not compile-time constants
//     (defines.hpp:34-37), and beta is passed to the action instead of a global (:52);
//   * a per-link functor cannot cross to the device, so Iterator::Checkerboard is
//     overloaded for the update kernels and runs a whole sweep per call
//     (iterators/iterators.hpp:65-87);
//   * random numbers come from counter-based Philox streams (seed + counter) instead of
//     one pcg64 per link (random/prng_wrapper.hpp:43-114).
// A non-OK status from the C ABI throws lettuce_gpu::Error (the reference exits or
// throws std::invalid_argument on the corresponding misuse).
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "lettuce_b200.h"

namespace lettuce_gpu
{
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int code)
{
    if (code != LT_OK) throw Error(code, lt_last_error());
}

// GaugeField4D (lattice.hpp:87-394)
class GaugeField
{
public:
    explicit GaugeField(std::array<int, 4> ext, int prec = LT_PREC_FP64) : ext_(ext)
    {
        check(lt_create(ext.data(), prec, &h_));
    }
    GaugeField(const GaugeField& o) : ext_(o.ext_)
    {
        int prec;
        check(lt_get_extents(o.h_, nullptr, &prec));
        check(lt_create(ext_.data(), prec, &h_));
        check(lt_copy(h_, o.h_));
    }
    GaugeField& operator=(const GaugeField& o)
    {
        if (this != &o) check(lt_copy(h_, o.h_));
        return *this;
    }
    GaugeField(GaugeField&& o) noexcept : ext_(o.ext_), h_(std::exchange(o.h_, nullptr)) {}
    ~GaugeField() { lt_destroy(h_); }

    void SetToIdentity() { check(lt_set_identity(h_)); }
    void SetToHaarRandom(std::uint64_t seed) { check(lt_set_haar_random(h_, seed)); }
    std::size_t Volume() const { return (std::size_t)ext_[0] * ext_[1] * ext_[2] * ext_[3]; }
    std::size_t SpatialVolume() const { return (std::size_t)ext_[1] * ext_[2] * ext_[3]; }   // lattice.hpp:201-204
    int Length(int d) const { return ext_[d]; }
    std::array<int, 4> Shape() const { return ext_; }

    // Whole field in the reference layout double[V][4][3][3][2]
    void Upload(const std::vector<double>& links) { check(lt_upload_links(h_, links.data())); }
    std::vector<double> Download() const
    {
        std::vector<double> v(Volume() * 72);
        check(lt_download_links(h_, v.data()));
        return v;
    }
    // operator()(link_coord) as explicit get/set of 18 doubles
    std::array<double, 18> GetLink(std::int64_t site, int mu) const
    {
        std::array<double, 18> m;
        check(lt_get_link(h_, site, mu, m.data()));
        return m;
    }
    void SetLink(std::int64_t site, int mu, const std::array<double, 18>& m) { check(lt_set_link(h_, site, mu, m.data())); }

    friend void Swap(GaugeField& a, GaugeField& b) { check(lt_swap(a.h_, b.h_)); }
    lt_lattice* handle() const { return h_; }

private:
    std::array<int, 4> ext_;
    lt_lattice* h_ = nullptr;
};

// observables/plaquette.hpp:26-43
inline double PlaquetteSum(const GaugeField& U)
{
    double v;
    check(lt_plaquette_sum(U.handle(), &v));
    return v;
}

// observables/topological_charge.hpp:97-200
inline double TopChargeClover(const GaugeField& U)
{
    double v;
    check(lt_topcharge_clover(U.handle(), &v));
    return v;
}

// FullTensor4D (lattice.hpp:447-590): 16 3x3 complex matrices per site in host memory, layout
// double[V][4][4][3][3][2]; CalculateClover<1, 1> (observables/clover.hpp:94-152) fills it on
// the device, TopChargeClover(const FullTensor&) (topological_charge.hpp:202-231) reads it
class FullTensor
{
public:
    explicit FullTensor(std::array<int, 4> ext)
        : ext_(ext), data_((std::size_t)ext[0] * ext[1] * ext[2] * ext[3] * 16 * 18, 0.0)
    {
    }
    std::array<int, 4> Shape() const { return ext_; }
    std::size_t Volume() const { return data_.size() / (16 * 18); }
    // the 18 doubles of C_{mu nu} at site (reference site index)
    const double* operator()(std::size_t site, int mu, int nu) const { return data_.data() + 18 * ((site * 4 + mu) * 4 + nu); }
    double* operator()(std::size_t site, int mu, int nu) { return data_.data() + 18 * ((site * 4 + mu) * 4 + nu); }
    const std::vector<double>& Data() const { return data_; }
    std::vector<double>& Data() { return data_; }

private:
    std::array<int, 4> ext_;
    std::vector<double> data_;
};

template <int N = 1>
inline void CalculateClover(const GaugeField& U, FullTensor& Clov)
{
    static_assert(N == 1, "only the plaquette clover CalculateClover<1, 1> is provided");
    if (Clov.Shape() != U.Shape()) throw Error(LT_ERR_ARG, "CalculateClover: tensor and field extents differ");
    check(lt_clover_tensor(U.handle(), Clov.Data().data()));
}

inline double TopChargeClover(const FullTensor& Clov)
{
    GaugeField scratch(Clov.Shape());   // supplies the extents, stream and reduction scratch
    double v;
    check(lt_topcharge_clover_tensor(scratch.handle(), Clov.Data().data(), &v));
    return v;
}

// EnergyDensity::Clover of the traceless clover field strength (field_strength_tensor.hpp:154-175)
inline double EnergyDensityClover(const GaugeField& U)
{
    double v;
    check(lt_energy_clover(U.handle(), &v));
    return v;
}

namespace GaugeAction
{
// Rectangular<stencil_radius> (actions/gauge/rectangular_action.hpp:23-246): radius 1 is the
// plaquette action (its staple is the plaquette staple whatever c_plaq), radius 2 adds the
// 1x2 and 2x1 rectangles with weight c_rect.  Apply() makes it the action of a field's
// device staples, sweeps, HMC force and Hamiltonian, and flow.
template <int stencil_radius_>
struct Rectangular
{
    static_assert(stencil_radius_ > 0 && stencil_radius_ <= 2, "Invalid stencil_radius!");
    static constexpr int stencil_radius = stencil_radius_;
    double beta = 6.0;
    const double c_plaq = 1.0;
    const double c_rect = 0.0;
    Rectangular(double beta_in, double c_plaq_in, double c_rect_in) : beta(beta_in), c_plaq(c_plaq_in), c_rect(c_rect_in) {}
    Rectangular() = default;
    void SetBeta(double b) { beta = b; }
    double GetBeta() const { return beta; }
    double Action(const GaugeField& U) const
    {
        double v;
        if constexpr (stencil_radius == 1)
        {
            check(lt_wilson_action(U.handle(), beta, &v));
            return c_plaq * v;
        }
        else
        {
            check(lt_rect_action(U.handle(), beta, c_plaq, c_rect, &v));
            return v;
        }
    }
    double ActionNormalized(const GaugeField& U) const { return Action(U) / (6.0 * beta * (double)U.Volume()); }
    void Apply(const GaugeField& U) const { check(lt_set_gauge_action(U.handle(), stencil_radius, c_plaq, c_rect)); }
};
using Wilson = Rectangular<1>;

// The named actions of rectangular_action.hpp:273-276 (c_plaq = 1 - 8 c_rect)
inline Rectangular<1> WilsonAction(6.0, 1.0, 0.0);
inline Rectangular<2> LüscherWeiszAction(6.0, 1.0 + 8.0 * 1.0 / 12.0, -1.0 / 12.0);
inline Rectangular<2>& LuescherWeiszAction = LüscherWeiszAction;
inline Rectangular<2> IwasakiAction(6.0, 1.0 + 8.0 * 0.331, -0.331);
inline Rectangular<2> DBW2Action(6.0, 1.0 + 8.0 * 1.4088, -1.4088);

// The Zeuthen flow (Ramos and Sint, arXiv:1508.05552) as the ActionT of a GradientFlowKernel:
// the Luescher-Weisz force acted on by 1 + 1/12 nabla*_mu nabla_mu (lt_set_flow_action).  Not
// in the reference, which flows with its gauge actions only.
struct ZeuthenFlow
{
    double beta = 6.0;
    double GetBeta() const { return beta; }
};
inline ZeuthenFlow ZeuthenFlowAction;
} // namespace GaugeAction

// The action a kernel runs with: its device form and a view of its coupling, which the kernels
// read at each call as the reference's kernels read their action
struct ActionRef
{
    int radius;
    double c_plaq, c_rect;
    const double* beta;
    int flow = LT_FLOW_ACTION_GAUGE;
    template <int R>
    ActionRef(const GaugeAction::Rectangular<R>& a) : radius(R), c_plaq(a.c_plaq), c_rect(a.c_rect), beta(&a.beta)
    {
    }
    // as the action of a flow: the Zeuthen force (the gauge action of the field is left alone)
    ActionRef(const GaugeAction::ZeuthenFlow& a)
        : radius(0), c_plaq(0.0), c_rect(0.0), beta(&a.beta), flow(LT_FLOW_ACTION_ZEUTHEN)
    {
    }
    void Apply(const GaugeField& U) const
    {
        check(lt_set_flow_action(U.handle(), flow));
        if (flow == LT_FLOW_ACTION_GAUGE) check(lt_set_gauge_action(U.handle(), radius, c_plaq, c_rect));
    }
    double GetBeta() const { return *beta; }
};

// TopChargeCloverTimeslice (observables/topological_charge.hpp:233-364) and
// EnergyDensity::CloverTimeslice (observables/field_strength_tensor.hpp:178-195): one launch
// computes every timeslice; the vector forms return all of them.
inline std::vector<double> TopChargeCloverTimeslices(const GaugeField& U)
{
    std::vector<double> q((size_t)U.Length(0));
    check(lt_clover_timeslices(U.handle(), q.data(), nullptr));
    return q;
}
inline double TopChargeCloverTimeslice(const GaugeField& U, int t) { return TopChargeCloverTimeslices(U).at((size_t)t); }

namespace EnergyDensity
{
inline double Clover(const GaugeField& U) { return EnergyDensityClover(U); }
inline std::vector<double> CloverTimeslices(const GaugeField& U)
{
    std::vector<double> e((size_t)U.Length(0));
    check(lt_clover_timeslices(U.handle(), nullptr, e.data()));
    return e;
}
inline double CloverTimeslice(const GaugeField& U, int t) { return CloverTimeslices(U).at((size_t)t); }
} // namespace EnergyDensity

// observables/topological_charge.hpp:366-416
inline double TopChargePlaquette(const GaugeField& U)
{
    double v;
    check(lt_topcharge_plaquette(U.handle(), &v));
    return v;
}

// WilsonLoop<N_mu_start, N_mu_end, reset>(U, U_chain) (observables/wilson_loop.hpp:63-124):
// 1 - sum Re tr W / (18 V) over the square N_mu_end x N_mu_end loops.  The chain of link
// products lives in U's handle on the device (the same reset / extend semantics), so U_chain
// is accepted for the signature and left untouched.
template <int N_mu_start, int N_mu_end, bool reset>
double WilsonLoop(const GaugeField& U, GaugeField& /*U_chain*/)
{
    static_assert(N_mu_start >= 0 && N_mu_end >= 0, "The template parameters of WilsonLoop are not allowed to be negative!");
    double v;
    check(lt_wilson_loop_chain(U.handle(), N_mu_start, N_mu_end, reset ? 1 : 0, &v));
    return v;
}

// observables/polyakov_loop.hpp:32-49
inline std::complex<double> PolyakovLoop(const GaugeField& U)
{
    double re, im;
    check(lt_polyakov_loop(U.handle(), &re, &im));
    return {re, im};
}

// HeatbathKernel (updates/heatbath.hpp:30-130); beta fixed at construction (:40).  Its random
// stream is (seed, counter) of Philox4x32-10, so SaveState / LoadState (the PRNG's checkpoint
// calls in the reference, random/prng_wrapper.hpp:268-279) write and read those two numbers;
// the second file, the reference's normal-distribution state, has no counterpart and is
// written as a marker only.
struct HeatbathKernel
{
    GaugeField& U;
    ActionRef action;
    double beta;
    std::uint64_t seed, counter;
    HeatbathKernel(GaugeField& U_in, ActionRef action_in, std::uint64_t seed_in = 1, std::uint64_t counter_in = 0)
        : U(U_in), action(action_in), beta(action_in.GetBeta()), seed(seed_in), counter(counter_in)
    {
    }
    bool SaveState(const std::filesystem::path& state, const std::filesystem::path& normal, bool overwrite = false) const
    {
        if (!overwrite && (std::filesystem::exists(state) || std::filesystem::exists(normal))) return false;
        std::ofstream s(state, std::ios::trunc), n(normal, std::ios::trunc);
        s << "philox4x32-10 " << seed << ' ' << counter << '\n';
        n << "counter-based stream: no distribution state\n";
        return static_cast<bool>(s) && static_cast<bool>(n);
    }
    bool LoadState(const std::filesystem::path& state, const std::filesystem::path&)
    {
        std::ifstream s(state);
        std::string tag;
        std::uint64_t sd = 0, ct = 0;
        if (!(s >> tag >> sd >> ct) || tag != "philox4x32-10") return false;
        seed = sd;
        counter = ct;
        return true;
    }
};

// OverrelaxationSubgroupKernel (updates/overrelaxation.hpp:68-117)
struct OverrelaxationSubgroupKernel
{
    GaugeField& U;
    ActionRef action;
    OverrelaxationSubgroupKernel(GaugeField& U_in, ActionRef action_in) : U(U_in), action(action_in) {}
};

namespace Iterator
{
// Iterator::Checkerboard (iterators/iterators.hpp:65-87): whole sweeps per call; a radius-2
// action throws (its rectangle staples reach links of the same colour)
inline void Checkerboard(HeatbathKernel& k, int n_sweep = 1)
{
    k.action.Apply(k.U);
    check(lt_heatbath_sweeps(k.U.handle(), k.beta, n_sweep, k.seed, &k.counter));
}
inline void Checkerboard(OverrelaxationSubgroupKernel& k, int n_sweep = 1)
{
    k.action.Apply(k.U);
    check(lt_overrelax_sweeps(k.U.handle(), n_sweep));
}
// Iterator::Checkerboard4 (:141-166): four sublattices per direction, any action; every
// extent a multiple of 4
inline void Checkerboard4(HeatbathKernel& k, int n_sweep = 1)
{
    k.action.Apply(k.U);
    check(lt_heatbath_sweeps4(k.U.handle(), k.beta, n_sweep, k.seed, &k.counter));
}
inline void Checkerboard4(OverrelaxationSubgroupKernel& k, int n_sweep = 1)
{
    k.action.Apply(k.U);
    check(lt_overrelax_sweeps4(k.U.handle(), n_sweep));
}
} // namespace Iterator

namespace Integrators::GradientFlow
{
struct Euler   // smearing/gradient_flow.hpp:31-56
{
    static constexpr int ID = LT_FLOW_EULER;
    static std::string ReturnName() { return "Euler/StoutSmearing"; }
};
struct RK2   // smearing/gradient_flow.hpp:89-118
{
    static constexpr int ID = LT_FLOW_RK2;
    static std::string ReturnName() { return "RK2"; }
};
struct RK3   // smearing/gradient_flow.hpp:120-168
{
    static constexpr int ID = LT_FLOW_RK3;
    static std::string ReturnName() { return "RK3"; }
};
struct RK3W7   // smearing/gradient_flow.hpp:170-218
{
    static constexpr int ID = LT_FLOW_RK3W7;
    static std::string ReturnName() { return "RK3W7"; }
};
} // namespace Integrators::GradientFlow

// GradientFlowKernel (smearing/gradient_flow.hpp:252-367) with any of the integrators above
template <typename IntegratorT = Integrators::GradientFlow::RK3, typename ActionT = GaugeAction::Rectangular<1>>
struct GradientFlowKernel
{
    const GaugeField& U_unflowed;
    GaugeField& U_flowed;
    ActionRef action;
    double epsilon;
    GradientFlowKernel(const GaugeField& in, GaugeField& out, IntegratorT&, ActionT& act, double eps)
        : U_unflowed(in), U_flowed(out), action(act), epsilon(eps)
    {
    }
    void operator()(int n_step) const
    {
        action.Apply(U_flowed);
        check(lt_flow(U_unflowed.handle(), U_flowed.handle(), IntegratorT::ID, epsilon, n_step));
    }
    void Resume(int n_step) const
    {
        action.Apply(U_flowed);
        check(lt_flow(U_flowed.handle(), U_flowed.handle(), IntegratorT::ID, epsilon, n_step));
    }
    void SetEpsilon(double e) { epsilon = e; }
    double GetEpsilon() const { return epsilon; }
    std::string ReturnIntegratorName() const { return IntegratorT::ReturnName(); }
};

// StoutSmearing4D (smearing/stout_smearing.hpp:29-57)
inline void StoutSmearing4D(const GaugeField& in, GaugeField& out, double smear_param = 0.12)
{
    check(lt_stout(in.handle(), out.handle(), smear_param, 1));
}

// Configuration files in the BMW format (IO/config_io/bmw_format.hpp): the reference's
// signatures and return values (false for a missing or malformed file, a shape mismatch or an
// existing file without overwrite; loading returns whether every link is an SU(3) element).
// LoadConfigBMWChecked also returns what the reference only prints: whether the recomputed
// Adler-64 checksum equals the header's (no counterpart in the reference).
inline bool LoadConfigBMWChecked(GaugeField& U, const std::string& filename, bool full, bool& checksum_ok)
{
    int ok = 0, in_group = 0;
    const int r = lt_load_bmw(U.handle(), filename.c_str(), full ? 1 : 0, &ok, &in_group);
    checksum_ok = false;
    if (r == LT_ERR_IO || r == LT_ERR_ARG) return false;
    check(r);
    checksum_ok = ok != 0;
    return in_group != 0;
}

namespace detail
{
inline bool save_bmw(const GaugeField& U, const std::string& filename, bool overwrite, int full)
{
    const int r = lt_save_bmw(U.handle(), filename.c_str(), full, overwrite ? 1 : 0, nullptr);
    if (r == LT_ERR_IO) return false;
    check(r);
    return true;
}
} // namespace detail

// SaveConfigBMW (:294-394) / LoadConfigBMW (:153-290): first two rows per link, "#BMW" header
inline bool SaveConfigBMW(const GaugeField& U, const std::string& filename, const bool overwrite = false)
{
    return detail::save_bmw(U, filename, overwrite, 0);
}
inline bool LoadConfigBMW(GaugeField& U, const std::string& filename)
{
    bool checksum_ok;
    return LoadConfigBMWChecked(U, filename, false, checksum_ok);
}
// SaveConfigBMWFull (:564-645) / LoadConfigBMWFull (:425-560): all three rows, "#18BMW" header
inline bool SaveConfigBMWFull(const GaugeField& U, const std::string& filename, const bool overwrite = false)
{
    return detail::save_bmw(U, filename, overwrite, 1);
}
inline bool LoadConfigBMWFull(GaugeField& U, const std::string& filename)
{
    bool checksum_ok;
    return LoadConfigBMWChecked(U, filename, true, checksum_ok);
}

// CheckpointManager (IO/config_io/checkpoint_manager.hpp:12-161): rotating checkpoint copies in
// backup1..backup<n-1> subdirectories; the save / load functions are passed in as in the
// reference (for example SaveConfigBMWFull and LoadConfigBMWFull), the PRNG is any object with
// SaveState / LoadState (HeatbathKernel above)
struct CheckpointManager
{
private:
    std::filesystem::path checkpoint_directory;

public:
    const int n_checkpoint_files;

    CheckpointManager(const std::filesystem::path& dir, const int n_files, const bool create_subdirectories)
        : checkpoint_directory(dir), n_checkpoint_files(n_files)
    {
        if (create_subdirectories) CreateSubdirectories();
    }
    std::filesystem::path CheckpointDirectory() const { return checkpoint_directory; }
    void CheckpointDirectory(const std::filesystem::path& dir) { checkpoint_directory = dir; }
    std::string ReturnBackupSubdirectory(const int counter) const
    {
        return counter == 0 ? std::string() : "backup" + std::to_string(counter);
    }
    void CreateSubdirectories() const
    {
        std::error_code err;
        for (int k = 1; k < n_checkpoint_files; ++k)
            std::filesystem::create_directories(checkpoint_directory / ReturnBackupSubdirectory(k), err);
    }
    void RotateFiles(const std::filesystem::path& current, const std::filesystem::path& old, const bool copy_file = true) const
    {
        if (!std::filesystem::exists(current)) return;
        std::error_code err;
        if (copy_file) std::filesystem::copy_file(current, old, std::filesystem::copy_options::overwrite_existing, err);
        else std::filesystem::rename(current, old, err);
    }
    template <typename FuncT>
    void AlternatingConfigCheckpoints(FuncT&& SaveFunction, const GaugeField& U, const std::string& filename_config) const
    {
        for (int k = n_checkpoint_files - 1; k > 0; --k)
            RotateFiles(checkpoint_directory / ReturnBackupSubdirectory(k - 1) / filename_config,
                        checkpoint_directory / ReturnBackupSubdirectory(k) / filename_config, k != 1);
        SaveFunction(U, (checkpoint_directory / filename_config).string(), true);
    }
    template <typename FuncT, typename prngT>
    void AlternatingCheckpoints(FuncT&& SaveFunction, prngT& prng, const GaugeField& U, const std::string& filename_config,
                                const std::string& filename_prng, const std::string& filename_normal_distribution) const
    {
        for (int k = n_checkpoint_files - 1; k > 0; --k)
        {
            const auto old_dir = checkpoint_directory / ReturnBackupSubdirectory(k);
            const auto cur_dir = checkpoint_directory / ReturnBackupSubdirectory(k - 1);
            RotateFiles(cur_dir / filename_config, old_dir / filename_config, k != 1);
            RotateFiles(cur_dir / filename_prng, old_dir / filename_prng, k != 1);
            RotateFiles(cur_dir / filename_normal_distribution, old_dir / filename_normal_distribution, k != 1);
        }
        SaveFunction(U, (checkpoint_directory / filename_config).string(), true);
        prng.SaveState(checkpoint_directory / filename_prng, checkpoint_directory / filename_normal_distribution, true);
    }
    template <typename FuncT, typename prngT>
    void LoadCheckpoint(FuncT&& LoadFunction, prngT& prng, GaugeField& U, const std::string& filename_config,
                        const std::string& filename_prng, const std::string& filename_normal_distribution) const
    {
        LoadFunction(U, (checkpoint_directory / filename_config).string());
        prng.LoadState(checkpoint_directory / filename_prng, checkpoint_directory / filename_normal_distribution);
    }
};

// MetaBiasPotential (actions/bias_potential/metadynamics.hpp:29-507)
class MetaBiasPotential
{
public:
    MetaBiasPotential(double CV_min, double CV_max, int bin_number, double weight, double width,
                      double well_tempered_parameter, double threshold_weight)
    {
        if (lt_bias_create(CV_min, CV_max, bin_number, weight, width, well_tempered_parameter, threshold_weight, &b_)
            != LT_OK)
            throw std::invalid_argument(lt_last_error());
    }
    MetaBiasPotential(const MetaBiasPotential&) = delete;
    MetaBiasPotential& operator=(const MetaBiasPotential&) = delete;
    ~MetaBiasPotential() { lt_bias_destroy(b_); }
    // the deposit of the updates and of MetaD trajectories: LT_BIAS_GAUSSIAN (the reference's)
    // or LT_BIAS_BINNED (Gaussian-free binned weights; no counterpart in the reference)
    void SetUpdateMode(int mode) { check(lt_bias_set_update_mode(b_, mode)); }
    void UpdatePotential(double cv) { check(lt_bias_update(b_, &cv, 1, 0)); }
    void UpdatePotentialSymmetric(double cv) { check(lt_bias_update(b_, &cv, 1, 1)); }
    void UpdatePotentialSymmetric(const std::vector<double>& cv)
    {
        check(lt_bias_update(b_, cv.data(), (int)cv.size(), 1));
    }
    double ReturnPotential(double cv) const
    {
        double v;
        check(lt_bias_potential(b_, cv, &v));
        return v;
    }
    double ReturnDerivative(double cv) const
    {
        double v;
        check(lt_bias_derivative(b_, cv, &v));
        return v;
    }
    lt_bias* handle() const { return b_; }

private:
    lt_bias* b_ = nullptr;
};

struct RunStatistics   // defines.hpp:93-106 (the fields this path fills)
{
    double delta_H_hmc = 0.0;
    std::uint64_t acceptances_hmc = 0;
    std::uint64_t acceptances_metadynamics_hmc = 0;
};

// The integrators of updates/hmc_gauge.hpp:19-377 and updates/hmc_metadynamics.hpp:26-238;
// ID selects the device program.  The friction variants run on HMCKernel only, the
// multiple-timescale ones on HMCMetaDKernel only (as in the reference, whose HMCKernel has no
// UpdateGaugeMomenta / UpdateMetadynamicsMomenta and whose HMCMetaDKernel no
// UpdateMomentaFriction).
namespace Integrators::HMC
{
#define LT_HMC_INTEGRATOR(NAME, ID_, GAUGE, METAD)                                        \
    struct NAME                                                                            \
    {                                                                                      \
        static constexpr int ID = ID_;                                                     \
        static constexpr bool gauge_kernel = GAUGE, metad_kernel = METAD;                  \
    };
LT_HMC_INTEGRATOR(Leapfrog_slow, LT_MD_LEAPFROG_SLOW, true, true)                 // hmc_gauge.hpp:21-44
LT_HMC_INTEGRATOR(Leapfrog, LT_MD_LEAPFROG, true, true)                           // :47-70
LT_HMC_INTEGRATOR(OMF_2_slow, LT_MD_OMF2_SLOW, true, true)                        // :121-151
LT_HMC_INTEGRATOR(OMF_2, LT_MD_OMF2, true, true)                                  // :155-190
LT_HMC_INTEGRATOR(OMF_4_slow, LT_MD_OMF4_SLOW, true, true)                        // :195-237
LT_HMC_INTEGRATOR(OMF_4, LT_MD_OMF4, true, true)                                  // :241-294
LT_HMC_INTEGRATOR(Leapfrog_friction_slow, LT_MD_LEAPFROG_FRICTION_SLOW, true, false)   // :74-116
LT_HMC_INTEGRATOR(OMF_4_friction_slow, LT_MD_OMF4_FRICTION_SLOW, true, false)     // :298-376
LT_HMC_INTEGRATOR(Leapfrog_OMF_4, LT_MD_LEAPFROG_OMF4, false, true)               // hmc_metadynamics.hpp:28-83
LT_HMC_INTEGRATOR(OMF_2_OMF_4_slow, LT_MD_OMF2_OMF4_SLOW, false, true)            // :85-143
LT_HMC_INTEGRATOR(OMF_2_OMF_4, LT_MD_OMF2_OMF4, false, true)                      // :145-237
#undef LT_HMC_INTEGRATOR
} // namespace Integrators::HMC

// ParityUpdate (updates/parity_update.hpp:22-47); the copy lives on the device, so U_copy is
// accepted for the signature and left untouched
inline void ParityUpdate(GaugeField& U, GaugeField& /*U_copy*/) { check(lt_parity_update(U.handle())); }

namespace GaugeUpdates
{
// HMCKernel (updates/hmc_gauge.hpp:381-600); U_copy and Momentum live on the device
template <typename IntegratorT>
struct HMCKernel
{
    static_assert(IntegratorT::gauge_kernel, "this integrator needs the Metadynamics kernel");
    GaugeField& U;
    ActionRef Action;
    RunStatistics& statistics;
    double trajectory_length;
    std::uint64_t seed, counter;
    HMCKernel(GaugeField& U_in, IntegratorT&, ActionRef action, RunStatistics& stats, double tau = 1.0,
              std::uint64_t seed_in = 1, std::uint64_t counter_in = 0)
        : U(U_in), Action(action), statistics(stats), trajectory_length(tau), seed(seed_in), counter(counter_in)
    {
    }
    bool operator()(int n_step, bool metropolis_step)
    {
        double dH;
        int acc;
        Action.Apply(U);
        check(lt_md_trajectory(U.handle(), nullptr, IntegratorT::ID, Action.GetBeta(), trajectory_length, n_step, 0.0,
                               0, seed, &counter, metropolis_step ? 1 : 0, &dH, &acc, nullptr));
        statistics.delta_H_hmc = dH;
        statistics.acceptances_hmc += (std::uint64_t)acc;
        return acc != 0;
    }
    // ReversibilityTest (:585-598): returns H after the forward-reverse-forward run minus H before
    double ReversibilityTest(int n_step)
    {
        double ho, hn;
        Action.Apply(U);
        check(lt_random_momenta(U.handle(), seed, counter));
        check(lt_md_integrate(U.handle(), nullptr, IntegratorT::ID, Action.GetBeta(), trajectory_length, n_step, 0.0, 0,
                              &ho, nullptr));
        check(lt_reverse_momenta(U.handle()));
        check(lt_md_integrate(U.handle(), nullptr, IntegratorT::ID, Action.GetBeta(), trajectory_length, n_step, 0.0, 0,
                              nullptr, &hn));
        return hn - ho;
    }
};

// HMCMetaDKernel (updates/hmc_metadynamics.hpp:264-675)
template <typename IntegratorT>
struct HMCMetaDKernel
{
    static_assert(IntegratorT::metad_kernel, "this integrator needs the gauge-only kernel");
    GaugeField& U;
    MetaBiasPotential& Metapotential;
    ActionRef Action;
    RunStatistics& statistics;
    double trajectory_length, rho_stout_cv;
    int n_smear_meta;
    std::uint64_t seed, counter;
    double cv_current = 0.0;
    HMCMetaDKernel(GaugeField& U_in, MetaBiasPotential& bias, IntegratorT&, ActionRef action,
                   RunStatistics& stats, double tau, double rho, int n_smear = 4, std::uint64_t seed_in = 1,
                   std::uint64_t counter_in = 0)
        : U(U_in), Metapotential(bias), Action(action), statistics(stats), trajectory_length(tau), rho_stout_cv(rho),
          n_smear_meta(n_smear), seed(seed_in), counter(counter_in)
    {
    }
    bool operator()(int n_step, bool metropolis_step)
    {
        double dH, cv;
        int acc;
        Action.Apply(U);
        check(lt_md_trajectory(U.handle(), Metapotential.handle(), IntegratorT::ID, Action.GetBeta(), trajectory_length,
                               n_step, rho_stout_cv, n_smear_meta, seed, &counter, metropolis_step ? 1 : 0, &dH, &acc,
                               &cv));
        statistics.delta_H_hmc = dH;
        statistics.acceptances_metadynamics_hmc += (std::uint64_t)acc;
        cv_current = cv;
        return acc != 0;
    }
    double MetaCharge() const
    {
        double q;
        check(lt_metad_charge(U.handle(), rho_stout_cv, n_smear_meta, &q));
        return q;
    }
    double ReversibilityTest(int n_step)
    {
        double ho, hn;
        Action.Apply(U);
        check(lt_random_momenta(U.handle(), seed, counter));
        check(lt_md_integrate(U.handle(), Metapotential.handle(), IntegratorT::ID, Action.GetBeta(), trajectory_length,
                              n_step, rho_stout_cv, n_smear_meta, &ho, nullptr));
        check(lt_reverse_momenta(U.handle()));
        check(lt_md_integrate(U.handle(), Metapotential.handle(), IntegratorT::ID, Action.GetBeta(), trajectory_length,
                              n_step, rho_stout_cv, n_smear_meta, nullptr, &hn));
        return hn - ho;
    }
};
} // namespace GaugeUpdates
} // namespace lettuce_gpu
