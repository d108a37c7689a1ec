// C ABI of the lattice handle: device memory, one stream per handle, and the sequencing
// of kernels for sweeps, flow, stout smearing, HMC and the metadynamics force.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <cmath>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "lt_handle.h"

namespace lt {

static thread_local std::string g_last_error;

int set_error(int code, const char* msg)
{
    g_last_error = msg ? msg : "";
    return code;
}

int cuda_error(cudaError_t e, const char* what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    g_last_error = m;
    return e == cudaErrorMemoryAllocation ? LT_ERR_NOMEM : LT_ERR_CUDA;
}

} // namespace lt

namespace {

int check_h(const lt_lattice* h, const char* fn)
{
    if (!h) return lt::set_error(LT_ERR_ARG, (std::string(fn) + ": null handle").c_str());
    return LT_OK;
}

int ensure(lt_lattice* h, void** p, size_t bytes)
{
    if (*p) return LT_OK;
    LT_CK(cudaMalloc(p, bytes));
    return LT_OK;
}

int ensure_aos(lt_lattice* h) { return ensure(h, (void**)&h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double)); }

// Kernel-launch status after a batch of launches
int launched(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return lt::cuda_error(e, what);
    return LT_OK;
}

// Copy results[slot..slot+n) to host and wait for the stream.
int fetch(lt_lattice* h, int slot, int n, double* out)
{
    LT_TRY(launched("reduction"));
    LT_CK(cudaMemcpyAsync(h->h_results, h->results + slot, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < n; ++k) out[k] = h->h_results[k];
    return LT_OK;
}

// Make `dst` wait for all work queued on `src`.
int order_after(lt_lattice* dst, const lt_lattice* src)
{
    if (dst == src) return LT_OK;
    cudaEvent_t ev;
    LT_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    LT_CK(cudaEventRecord(ev, src->stream));
    LT_CK(cudaStreamWaitEvent(dst->stream, ev, 0));
    LT_CK(cudaEventDestroy(ev));
    return LT_OK;
}

const double kPi = 3.14159265358979323846;

// Stages of the reference's flow integrators (smearing/gradient_flow.hpp:31-168), each one
// fused Z update + exponential update: Z <- c_old Z + c_new eps Algebra(st U^dag),
// U <- exp(c_exp Z) U
struct FlowStage
{
    double c_old, c_new, c_exp;
    int read_z, write_z;
};
constexpr FlowStage kEuler[] = { { 0.0, 1.0, 1.0, 0, 0 } };
constexpr FlowStage kRK2[] = { { 0.0, 1.0, 0.5, 0, 1 }, { -0.5, 1.0, 1.0, 1, 0 } };
constexpr FlowStage kRK3[] = { { 0.0, 1.0, 0.25, 0, 1 }, { -17.0 / 36.0, 8.0 / 9.0, 1.0, 1, 1 }, { -1.0, 3.0 / 4.0, 1.0, 1, 0 } };
constexpr FlowStage kRK3W7[] = { { 0.0, 1.0, 1.0 / 3.0, 0, 1 },
                                 { -25.0 / 48.0, 15.0 / 16.0, 1.0, 1, 1 },
                                 { -17.0 / 25.0, 8.0 / 15.0, 1.0, 1, 0 } };

int flow_steps(lt_lattice* h, double eps, int n_step, int integrator = LT_FLOW_RK3)
{
    const FlowStage* st = integrator == LT_FLOW_EULER ? kEuler
                        : integrator == LT_FLOW_RK2   ? kRK2
                        : integrator == LT_FLOW_RK3W7 ? kRK3W7 : kRK3;
    const int ns = integrator == LT_FLOW_EULER ? 1 : integrator == LT_FLOW_RK2 ? 2 : 3;
    LT_TRY(ensure(h, &h->U2, h->be->gauge_bytes(h->g)));
    if (ns > 1) LT_TRY(ensure(h, &h->Z, h->be->alg_bytes(h->g)));
    const bool zeuthen = h->flow_action == LT_FLOW_ACTION_ZEUTHEN;
    if (zeuthen || h->be->flow_split()) LT_TRY(ensure(h, &h->Xz, h->be->alg_bytes(h->g)));
    const lt::Ctx c = h->ctx();
    for (int k = 0; k < n_step; ++k)
        for (int j = 0; j < ns; ++j)
        {
            if (zeuthen)
                // the Zeuthen flow's force is that of the Luescher-Weisz action whatever the
                // handle's gauge action (c_plaq = 5/3, c_rect = -1/12)
                h->be->flow_zeuthen_stage(c, h->U, h->U2, h->Z, h->Xz, st[j].c_old, st[j].c_new * eps, st[j].c_exp,
                                          st[j].read_z, st[j].write_z, 5.0 / 3.0, -1.0 / 12.0);
            else
                h->be->flow_stage(c, h->U, h->U2, h->Z, st[j].c_old, st[j].c_new * eps, st[j].c_exp, st[j].read_z,
                                  st[j].write_z, h->be->flow_split() ? h->Xz : nullptr);
            std::swap(h->U, h->U2);
        }
    return launched("flow");
}

int stout_steps(lt_lattice* h, double rho, int n)
{
    LT_TRY(ensure(h, &h->U2, h->be->gauge_bytes(h->g)));
    const lt::Ctx c = h->ctx();
    for (int k = 0; k < n; ++k)
    {
        h->be->stout(c, h->U, h->U2, rho, nullptr);
        std::swap(h->U, h->U2);
    }
    return launched("stout");
}

int clover_q_e(lt_lattice* h, const void* U, double* q, double* e)
{
    h->be->clover_obs(h->ctx(), U, 2);
    double r[2];
    LT_TRY(fetch(h, 2, 2, r));
    if (q) *q = -1.0 / (64.0 * 4.0 * kPi * kPi) * r[0];
    if (e) *e = r[1] / (double)h->g.V;
    return LT_OK;
}

int plaq_of(lt_lattice* h, const void* U, double* out)
{
    h->be->plaquette(h->ctx(), U, 0);
    return fetch(h, 0, 1, out);
}

// Forward stout chain U -> levels[1..n] (StoutSmearing4DWithConstants,
// smearing/stout_smearing.hpp:92-119): the exponential constants are not stored (the adjoint
// recomputes them), the staple of every level is (the adjoint's Lambda step reads it back
// instead of computing it again)
int metad_forward(lt_lattice* h, double rho, int n_stout)
{
    while ((int)h->levels.size() < n_stout)
    {
        void* p = nullptr;
        LT_CK(cudaMalloc(&p, h->be->gauge_bytes(h->g)));
        h->levels.push_back(p);
    }
    while ((int)h->staples.size() < n_stout)
    {
        void* p = nullptr;
        LT_CK(cudaMalloc(&p, h->be->full_bytes(h->g)));
        h->staples.push_back(p);
    }
    const lt::Ctx c = h->ctx();
    const void* prev = h->U;
    for (int k = 0; k < n_stout; ++k)
    {
        h->be->stout(c, prev, h->levels[k], rho, h->staples[k]);
        prev = h->levels[k];
    }
    return launched("metad_forward");
}

const void* level(const lt_lattice* h, int k) { return k == 0 ? h->U : h->levels[k - 1]; }

// dvdq * dQ/dU into h->F, given the forward chain (CalculateTopologicalForce,
// updates/hmc_metadynamics.hpp:374-436)
// The clover planes R of the most smeared level (CalculateClover, hmc_metadynamics.hpp:397-399)
int metad_clover(lt_lattice* h, int n_stout)
{
    LT_TRY(ensure(h, &h->R, h->be->clov_bytes(h->g)));
    h->be->clover_R(h->ctx(), level(h, n_stout), h->R);
    return launched("metad_clover");
}

// Q of the most smeared level from its clover planes (TopChargeClover(Clover),
// topological_charge.hpp:202-231)
int charge_from_R(lt_lattice* h, double* q)
{
    h->be->topcharge_R(h->ctx(), h->R, 7);
    double r;
    LT_TRY(fetch(h, 7, 1, &r));
    *q = -1.0 / (64.0 * 4.0 * kPi * kPi) * r;
    return LT_OK;
}

int metad_backward(lt_lattice* h, double rho, int n_stout, double dvdq, bool have_R = false)
{
    LT_TRY(ensure(h, &h->F, h->be->alg_bytes(h->g)));
    LT_TRY(ensure(h, &h->Lam, h->be->alg_bytes(h->g)));
    LT_TRY(ensure(h, &h->Tloc, h->be->full_bytes(h->g)));
    if (!have_R) LT_TRY(metad_clover(h, n_stout));
    const lt::Ctx c = h->ctx();
    const void* top = level(h, n_stout);
    h->be->clover_deriv(c, top, h->R, h->F, dvdq);
    for (int k = n_stout; k > 0; --k)
    {
        h->be->stout_lambda(c, level(h, k - 1), level(h, k), h->F, h->Lam, h->Tloc, rho, h->staples[k - 1]);
        h->be->stout_recursion(c, level(h, k - 1), h->Lam, h->Tloc, h->F, rho);
    }
    return launched("metad_backward");
}

// Action(U) of the handle's gauge action (rectangular_action.hpp:61-94) + (-sum ReTr P^2)
int hamiltonian(lt_lattice* h, double beta, double* out)
{
    const lt::Ctx c = h->ctx();
    const double V = (double)h->g.V;
    if (h->act_radius == 2)
    {
        h->be->loops(c, h->U, 4);
        h->be->kinetic(c, h->P, 1);
        double r[3], k;
        LT_TRY(fetch(h, 4, 3, r));
        LT_TRY(fetch(h, 1, 1, &k));
        *out = beta * (h->act_cp * (6.0 * V - r[0] / 3.0) + h->act_cr * (12.0 * V - r[1] / 3.0)) + k;
        return LT_OK;
    }
    h->be->plaquette(c, h->U, 0);
    h->be->kinetic(c, h->P, 1);
    double r[2];
    LT_TRY(fetch(h, 0, 2, r));
    *out = beta * h->act_cp * (6.0 * V - r[0] / 3.0) + r[1];
    return LT_OK;
}

// Momentum kick with optional MetaD force.  For MetaD the force is evaluated on the
// current links first (UpdateMomenta, updates/hmc_metadynamics.hpp:441-459).
struct MetaDParams
{
    lt::Bias* bias;
    double rho;
    int n_stout;
    std::vector<double>* samples;
};

// dV/dQ * dQ/dU into h->F at the current links (CalculateTopologicalForce,
// updates/hmc_metadynamics.hpp:374-436); with submeasure the CV is recorded as the
// reference's path samples are (:405-412)
int metad_force_now(lt_lattice* h, const MetaDParams* md, bool submeasure)
{
    LT_TRY(metad_forward(h, md->rho, md->n_stout));
    LT_TRY(metad_clover(h, md->n_stout));
    double q;
    LT_TRY(charge_from_R(h, &q));
    if (submeasure && md->samples) md->samples->push_back(q);
    return metad_backward(h, md->rho, md->n_stout, md->bias->derivative(q), true);
}

int kick(lt_lattice* h, double beta, double eps, const MetaDParams* md, bool submeasure)
{
    const void* F = nullptr;
    if (md)
    {
        LT_TRY(metad_force_now(h, md, submeasure));
        F = h->F;
    }
    h->be->momenta(h->ctx(), h->U, h->P, F, beta / 6.0, eps);
    return launched("momenta");
}

int drift(lt_lattice* h, double eps)
{
    h->be->fields(h->ctx(), h->U, h->P, eps);
    return launched("fields");
}

// One step of a molecular-dynamics program:
//   KICK          UpdateMomenta: gauge force plus, under MetaD, the force at the current links
//   KICK_GAUGE    UpdateGaugeMomenta (hmc_metadynamics.hpp:464-476)
//   KICK_METAD    UpdateMetadynamicsMomenta (:478-491); the force is evaluated at the current
//                 links first (the reference adds its stored ForceFatLink as it stands)
//   FRICTION_PRE  UpdateMomentaFriction with friction_without_kick (hmc_gauge.hpp:469-484):
//                 P <- e P + eps beta/6 Alg(st U^dag), e = exp(-friction eps)
//   FRICTION_POST the other branch (:485-500): P <- e (P + eps beta/6 Alg(st U^dag))
//   DRIFT         UpdateFields
enum class Md : unsigned char { KICK, KICK_GAUGE, KICK_METAD, FRICTION_PRE, FRICTION_POST, DRIFT };
struct MdOp
{
    Md kind;
    double eps;
    bool sub = false;        // record the CV (path samples)
    double friction = 0.0;
};

// The integrators of updates/hmc_gauge.hpp:19-377 and updates/hmc_metadynamics.hpp:26-238 as
// programs of the steps above; eps = tau / n_step.
bool md_program(int integ, double tau, int n, std::vector<MdOp>& ops)
{
    ops.clear();
    if (integ < LT_MD_LEAPFROG_SLOW || integ > LT_MD_OMF2_OMF4) return false;
    if (n <= 0) return true;
    const double e = tau / n;
    auto K = [&](double x, bool sub = false) { ops.push_back({ Md::KICK, x, sub }); };
    auto G = [&](double x) { ops.push_back({ Md::KICK_GAUGE, x }); };
    auto M = [&](double x) { ops.push_back({ Md::KICK_METAD, x }); };
    auto D = [&](double x) { ops.push_back({ Md::DRIFT, x }); };
    auto FP = [&](double x, double f, bool pre) { ops.push_back({ pre ? Md::FRICTION_PRE : Md::FRICTION_POST, x, false, f }); };
    // OMF2 (hep-lat/0505020) and OMF4 coefficients
    const double l2 = 0.1931833275037836;
    const double a4 = 0.08398315262876693, b4 = 0.2539785108410595, g4 = 0.6822365335719091,
                 d4 = -0.03230286765269967;
    const double m4 = 0.5 - g4 - a4, n4 = 1.0 - 2.0 * d4 - 2.0 * b4;
    // one OMF4 step of the gauge part with kicks `kick` and the first / last kick left out
    auto omf4_inner = [&](double s, auto kick) {
        D(s * b4 * e); kick(s * g4 * e); D(s * d4 * e);
        kick(s * m4 * e); D(s * n4 * e); kick(s * m4 * e);
        D(s * d4 * e); kick(s * g4 * e); D(s * b4 * e);
    };
    auto kfull = [&](double x) { K(x); };
    switch (integ)
    {
    case LT_MD_LEAPFROG_SLOW:   // hmc_gauge.hpp:21-44
        for (int k = 0; k < n; ++k) { K(0.5 * e); D(e); K(0.5 * e, true); }
        break;
    case LT_MD_LEAPFROG:        // :47-70
        K(0.5 * e);
        for (int k = 0; k < n - 1; ++k) { D(e); K(e, true); }
        D(e); K(0.5 * e, true);
        break;
    case LT_MD_OMF2_SLOW:       // :121-151
        for (int k = 0; k < n; ++k) { K(l2 * e); D(0.5 * e); K((1.0 - 2.0 * l2) * e); D(0.5 * e); K(l2 * e, true); }
        break;
    case LT_MD_OMF2:            // :155-190
        K(l2 * e); D(0.5 * e); K((1.0 - 2.0 * l2) * e); D(0.5 * e);
        for (int k = 0; k < n - 1; ++k) { K(2.0 * l2 * e, true); D(0.5 * e); K((1.0 - 2.0 * l2) * e); D(0.5 * e); }
        K(l2 * e, true);
        break;
    case LT_MD_OMF4_SLOW:       // :195-237
        for (int k = 0; k < n; ++k) { K(a4 * e); omf4_inner(1.0, kfull); K(a4 * e, true); }
        break;
    case LT_MD_OMF4:            // :241-294
        K(a4 * e); omf4_inner(1.0, kfull);
        for (int k = 0; k < n - 1; ++k) { K(2.0 * a4 * e, true); omf4_inner(1.0, kfull); }
        K(a4 * e, true);
        break;
    case LT_MD_LEAPFROG_FRICTION_SLOW:   // :74-116 (RAHMC, 2403.04607)
    case LT_MD_OMF4_FRICTION_SLOW:       // :298-376
    {
        double f = 0.01;
        const int half = n / 2;
        auto step = [&](bool flip_mid) {
            if (integ == LT_MD_LEAPFROG_FRICTION_SLOW)
            {
                FP(0.5 * e, f, true); D(e);
                if (flip_mid) f = -f;
                FP(0.5 * e, f, false);
            }
            else
            {
                FP(a4 * e, f, true); D(b4 * e); FP(g4 * e, f, true); D(d4 * e);
                FP(m4 * e, f, true); D(n4 * e);
                if (flip_mid) f = -f;
                FP(m4 * e, f, false);
                D(d4 * e); FP(g4 * e, f, false); D(b4 * e); FP(a4 * e, f, false);
            }
        };
        for (int k = 0; k < half; ++k) step(false);
        if (n % 2 != 0) step(true);
        else f = -f;
        for (int k = 0; k < half; ++k) step(false);
        break;
    }
    case LT_MD_LEAPFROG_OMF4:   // hmc_metadynamics.hpp:28-83
    {
        auto kg = [&](double x) { G(x); };
        M(0.5 * e);
        for (int k = 0; k < n; ++k)
        {
            G(a4 * e); omf4_inner(1.0, kg); G(a4 * e);
            M(k < n - 1 ? e : 0.5 * e);
        }
        break;
    }
    case LT_MD_OMF2_OMF4_SLOW:  // :85-143
    {
        auto kg = [&](double x) { G(x); };
        for (int k = 0; k < n; ++k)
        {
            M(l2 * e);
            G(a4 * e); omf4_inner(1.0, kg); G(a4 * e);
            M((1.0 - 2.0 * l2) * e);
            G(a4 * e); omf4_inner(1.0, kg); G(a4 * e);
            M(l2 * e);
        }
        break;
    }
    case LT_MD_OMF2_OMF4:       // :145-237 (inner OMF4 at half steps)
    {
        auto kg = [&](double x) { G(x); };
        M(l2 * e);
        for (int k = 0; k < n; ++k)
        {
            G(0.5 * a4 * e); omf4_inner(0.5, kg); G(0.5 * a4 * e);
            M((1.0 - 2.0 * l2) * e);
            G(0.5 * a4 * e); omf4_inner(0.5, kg); G(0.5 * a4 * e);
            M(k < n - 1 ? 2.0 * l2 * e : l2 * e);
        }
        break;
    }
    }
    return true;
}

bool md_needs_bias(int integ) { return integ >= LT_MD_LEAPFROG_OMF4; }
bool md_friction(int integ) { return integ == LT_MD_LEAPFROG_FRICTION_SLOW || integ == LT_MD_OMF4_FRICTION_SLOW; }

int md_check(int integ, bool metad, const char* fn)
{
    if (integ < LT_MD_LEAPFROG_SLOW || integ > LT_MD_OMF2_OMF4)
        return lt::set_error(LT_ERR_ARG, (std::string(fn) + ": unknown integrator").c_str());
    if (md_needs_bias(integ) && !metad)
        return lt::set_error(LT_ERR_ARG, (std::string(fn) + ": multiple-timescale integrators need a bias").c_str());
    if (md_friction(integ) && metad)
        return lt::set_error(LT_ERR_ARG, (std::string(fn) + ": friction integrators are gauge-only").c_str());
    return LT_OK;
}

// Run a program on (h->U, h->P); md null for the gauge action alone
int integrate(lt_lattice* h, double beta, const std::vector<MdOp>& ops, const MetaDParams* md)
{
    const lt::Ctx c = h->ctx();
    for (const MdOp& op : ops)
    {
        switch (op.kind)
        {
        case Md::KICK: LT_TRY(kick(h, beta, op.eps, md, op.sub)); break;
        case Md::KICK_GAUGE: LT_TRY(kick(h, beta, op.eps, nullptr, false)); break;
        case Md::KICK_METAD:
            LT_TRY(metad_force_now(h, md, op.sub));
            h->be->alg_axpby(c, h->P, h->F, 1.0, op.eps);
            LT_TRY(launched("metad momenta"));
            break;
        case Md::FRICTION_PRE:
            h->be->alg_axpby(c, h->P, nullptr, std::exp(-op.friction * op.eps), 0.0);
            LT_TRY(kick(h, beta, op.eps, nullptr, false));
            break;
        case Md::FRICTION_POST:
            LT_TRY(kick(h, beta, op.eps, nullptr, false));
            h->be->alg_axpby(c, h->P, nullptr, std::exp(-op.friction * op.eps), 0.0);
            LT_TRY(launched("friction"));
            break;
        case Md::DRIFT: LT_TRY(drift(h, op.eps)); break;
        }
    }
    return LT_OK;
}

// Integrators::HMC::OMF_2 (updates/hmc_gauge.hpp:155-190)
int omf2(lt_lattice* h, double beta, double tau, int n_step, const MetaDParams* md)
{
    std::vector<MdOp> ops;
    md_program(LT_MD_OMF2, tau, n_step, ops);
    return integrate(h, beta, ops, md);
}

int metad_charge(lt_lattice* h, double rho, int n_stout, double* q)
{
    LT_TRY(metad_forward(h, rho, n_stout));
    return clover_q_e(h, level(h, n_stout), q, nullptr);
}

double accept_uniform(uint64_t seed, uint64_t counter)
{
    lt::U4 w = lt::philox4x32(0u, (uint32_t)counter, (uint32_t)(counter >> 32), lt::TAG_ACCEPT << 24, (uint32_t)seed,
                              (uint32_t)(seed >> 32));
    return lt::u01_from(w.x, w.y);
}

} // namespace

// Two-row FP32 storage: the reference-layout FP64 links are rounded and packed into the device
// layout on the host, by a pool of host threads, chunk by chunk into a pinned staging buffer,
// and each chunk is copied to the device while the threads pack the next: the PCIe link then
// carries the stored 48 bytes per link instead of the 144 of the FP64 input.  From pinned
// input a share of the sites goes over PCIe as FP64 at the same time and is converted on the
// device, so that the copy engine and the host's memory bandwidth are both used (one 32^4
// upload: 6.4 to 6.8 ms, against 8.0 ms packed whole and 11.2 ms for the FP64 copy at 55 GB/s).
// A handle's first upload takes the device conversion: the pinned staging buffer (its
// allocation costs more than one upload) is set up for handles that are uploaded again.  The
// 18-real FP32 storage keeps the device conversion: its host packing (72 bytes per link) was
// slower than the FP64 copy.  The rounding (IEEE round to nearest, double to float) and the
// layout are those of the device conversion k_from_aos.
namespace {

#ifndef LT_UPLOAD_CHUNKS
#define LT_UPLOAD_CHUNKS 8
#endif
constexpr int kUploadChunks = LT_UPLOAD_CHUNKS;

// Packs the sites [i0, i1) (reference site order; i0 and i1 even) of the FP64 links into dst
// in the device layout of the storage (nr = 2: three float4 chunks per link; nr = 3: nine
// complex planes).  Sites 2s and 2s + 1 share the checkerboard index s and have opposite
// parities (the z extent is even), so the loop walks site pairs and steps the coordinates
// with carries instead of dividing.
//
// Two-row storage goes block by block: kPackBlock site pairs' input records (74 KB, held in
// the core's L2) are located first, then each of the 24 (direction, parity, chunk) planes
// receives one contiguous run of kPackBlock float4 by streaming stores, so the pinned staging
// buffer is written in whole cache lines without being read first.  Site by site, every site
// would touch 12 planes and the plain stores would read each destination line before writing
// it (packing a 32^4 field on 8 cores: 25.3 ms site by site, 16.2 ms blocked with plain stores,
// 12.2 ms blocked with streaming stores).
// Share of the checkerboard indices packed on the host when the input is pinned (the rest is
// copied as FP64 and converted on the device).  Host packing alone is bound by the host's
// memory bandwidth, the FP64 copy by PCIe; one 32^4 upload from pinned memory takes 8.0 ms
// packed whole, 6.6 to 6.8 ms with 0.65 to 0.75 packed, 8.0 ms with 0.85
#ifndef LT_PACK_SHARE
#define LT_PACK_SHARE 0.7
#endif
constexpr double kPackShare = LT_PACK_SHARE;

#ifndef LT_PACK_RESERVE
#define LT_PACK_RESERVE 2
#endif
// host threads left to the callers: the uploading thread, which hands the chunks to the copy
// engine, and a second handle's thread waiting on its kernels (32^4 streamed through two
// handles: 3.34e9 link updates/s end to end with 2 left, 3.14e9 with 1, 3.05e9 with none)
constexpr unsigned kPackReserve = LT_PACK_RESERVE;

#ifndef LT_PACK_BLOCK
#define LT_PACK_BLOCK 64
#endif
constexpr int kPackBlock = LT_PACK_BLOCK;

void pack_sites(const lt::Geom& g, int nr, const double* aos, float* dst, long long i0, long long i1)
{
    const size_t vh = (size_t)g.vh;
    if (i0 >= i1) return;
    long long r = i0;
    int z = (int)(r % g.n[3]);
    r /= g.n[3];
    int y = (int)(r % g.n[2]);
    r /= g.n[2];
    int x = (int)(r % g.n[1]);
    int t = (int)(r / g.n[1]);
    auto next_pair = [&] {
        z += 2;
        if (z == g.n[3])
        {
            z = 0;
            if (++y == g.n[2])
            {
                y = 0;
                if (++x == g.n[1])
                {
                    x = 0;
                    ++t;
                }
            }
        }
    };
    if (nr == 2)
    {
        const double* src[2][kPackBlock];   // input record of checkerboard index sa + k, by parity
        for (long long i = i0; i < i1;)
        {
            const size_t sa = (size_t)(i >> 1);
            int n = 0;
            for (; n < kPackBlock && i < i1; ++n, i += 2)
            {
                const int p0 = (t + x + y + z) & 1;   // parity of site i; site i + 1 has the other
                src[p0][n] = aos + (size_t)72 * (size_t)i;
                src[p0 ^ 1][n] = aos + (size_t)72 * (size_t)(i + 1);
                next_pair();
            }
            for (int par = 0; par < 2; ++par)
                for (int mu = 0; mu < 4; ++mu)
                    for (int c = 0; c < 3; ++c)
                    {
                        // chunk c of plane (mu, par) holds floats 4c .. 4c + 3 of rows 0-1
                        float* q = dst + 4 * (((size_t)(mu * 2 + par) * 3 + c) * vh + sa);
                        const int off = 18 * mu + 4 * c;
                        for (int k = 0; k < n; ++k)
                        {
                            const double* a = src[par][k] + off;
#if defined(__SSE2__)
                            const __m128 lo = _mm_cvtpd_ps(_mm_loadu_pd(a));
                            const __m128 hi = _mm_cvtpd_ps(_mm_loadu_pd(a + 2));
                            _mm_stream_ps(q + 4 * k, _mm_movelh_ps(lo, hi));
#else
                            for (int e = 0; e < 4; ++e) q[4 * k + e] = (float)a[e];
#endif
                        }
                    }
        }
#if defined(__SSE2__)
        _mm_sfence();   // the streamed chunks are visible before the caller reports them packed
#endif
        return;
    }
    for (long long i = i0; i < i1; i += 2)
    {
        const int p0 = (t + x + y + z) & 1;
        const size_t s = (size_t)(i >> 1);
        for (int h = 0; h < 2; ++h)
        {
            const int par = p0 ^ h;
            const double* site = aos + (size_t)72 * (size_t)(i + h);
            for (int mu = 0; mu < 4; ++mu)
            {
                const double* a = site + 18 * mu;
                for (int e = 0; e < 9; ++e)
                {
                    float* q = dst + 2 * (((size_t)(mu * 2 + par) * 9 + e) * vh + s);
                    q[0] = (float)a[2 * e];
                    q[1] = (float)a[2 * e + 1];
                }
            }
        }
        next_pair();
    }
}

// One packing upload at a time per process: the packing is bound by host memory bandwidth and
// uses the cores, so handles packing at once only contend; serialised, one handle packs while
// the other's copy and kernels run (two handles streamed from two host threads at 32^4,
// measured before the split uploads: 2.10e9 link updates/s end to end, against 1.98e9 to
// 2.05e9 with the cores shared).
std::mutex g_pack_mutex;

// The packing threads: started by the first packing upload and kept for the life of the
// process (starting and joining 16 threads cost about 0.4 ms of an 8 ms upload).  They are
// detached and the pool is never freed, so nothing waits for them at exit; each waits on a
// condition variable between jobs.  Jobs run one at a time (under g_pack_mutex).
class PackPool
{
public:
    static PackPool& get()
    {
        static PackPool* pool = new PackPool();
        return *pool;
    }
    unsigned size() const { return n_; }

    // runs job(t) on workers t = 0 .. size() - 1 and returns without waiting
    void start(const std::function<void(unsigned)>& job)
    {
        std::lock_guard<std::mutex> lk(m_);
        job_ = job;
        finished_ = 0;
        ++gen_;
        cv_.notify_all();
    }
    // waits until every worker has returned from the current job
    void wait()
    {
        std::unique_lock<std::mutex> lk(m_);
        idle_.wait(lk, [this] { return finished_ == n_; });
    }

private:
    PackPool()
    {
        const unsigned hc = std::thread::hardware_concurrency();
        n_ = hc > kPackReserve ? hc - kPackReserve : 1;
        for (unsigned t = 0; t < n_; ++t) std::thread([this, t] { loop(t); }).detach();
    }
    void loop(unsigned t)
    {
        unsigned long long seen = 0;
        for (;;)
        {
            std::function<void(unsigned)> job;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                job = job_;
            }
            job(t);
            std::lock_guard<std::mutex> lk(m_);
            if (++finished_ == n_) idle_.notify_all();
        }
    }
    std::mutex m_;
    std::condition_variable cv_, idle_;
    std::function<void(unsigned)> job_;
    unsigned long long gen_ = 0;
    unsigned finished_ = 0;
    unsigned n_ = 1;
};

// From pinned input, the sites of the checkerboard indices [pack_split, vh) cross PCIe as FP64
// straight from the caller's buffer and are converted on the device, while the host threads
// pack the rest: the copy engine and the host cores then share the field
long long pack_split(const lt_lattice* h, const double* links)
{
    cudaPointerAttributes attr;
    const bool pinned = cudaPointerGetAttributes(&attr, links) == cudaSuccess && attr.type == cudaMemoryTypeHost;
    (void)cudaGetLastError();   // an unregistered pointer may leave an error behind on old drivers
    return pinned && h->g.V >= 65536 ? (long long)(h->g.vh * kPackShare) : h->g.vh;
}

int upload_packed_fp32(lt_lattice* h, const double* links)
{
    std::lock_guard<std::mutex> pack_lock(g_pack_mutex);
    const int nr = h->prec == LT_PREC_FP32_12 ? 2 : 3;
    const size_t elem = nr == 2 ? 16 : 8;           // bytes of one plane entry
    const int planes = nr == 2 ? 24 : 72;           // (mu, par) x chunks or elements
    const size_t bytes = h->be->gauge_bytes(h->g);
    if (!h->h_stage) LT_CK(cudaMallocHost(&h->h_stage, bytes));
    // the staging buffers may still feed a copy of an earlier call on this stream
    LT_CK(cudaStreamSynchronize(h->stream));
    const long long vh = h->g.vh;
    const long long s_split = pack_split(h, links);
    if (s_split < vh)
    {
        LT_TRY(ensure_aos(h));
        const size_t first = (size_t)72 * (size_t)(2 * s_split);   // doubles before the first raw site
        LT_CK(cudaMemcpyAsync(h->d_aos + first, links + first, (size_t)72 * (size_t)(h->g.V - 2 * s_split) * sizeof(double),
                              cudaMemcpyHostToDevice, h->stream));
        h->be->from_aos_sites(h->ctx(), h->U, h->d_aos, 2 * s_split, h->g.V);
        LT_TRY(launched("lt_upload_links"));
    }
    long long bound[kUploadChunks + 1];
    for (int k = 0; k <= kUploadChunks; ++k) bound[k] = s_split * k / kUploadChunks;   // checkerboard indices
    // small lattices pack on the calling thread, chunk by chunk
    PackPool* pool = h->g.V < 65536 ? nullptr : &PackPool::get();
    const unsigned nt = pool ? pool->size() : 1;
    std::atomic<int> done[kUploadChunks];
    for (auto& d : done) d.store(0);
    float* dst = static_cast<float*>(h->h_stage);
    const lt::Geom g = h->g;
    // sites 2s and 2s + 1 share checkerboard index s (the z extent is even), so chunk k of
    // checkerboard indices is the contiguous site range [2 bound[k], 2 bound[k+1])
    auto pack_chunk = [&](unsigned t, int k) {
        // whole site pairs per thread: pair range [bound[k], bound[k+1]) split evenly
        const long long n = bound[k + 1] - bound[k];
        const long long a = bound[k] + n * t / nt, b = bound[k] + n * (t + 1) / nt;
        pack_sites(g, nr, links, dst, 2 * a, 2 * b);
        done[k].fetch_add(1, std::memory_order_release);
    };
    if (pool)
        pool->start([&](unsigned t) {
            for (int k = 0; k < kUploadChunks; ++k) pack_chunk(t, k);
        });
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < kUploadChunks; ++k)
    {
        if (!pool) pack_chunk(0, k);
        while (done[k].load(std::memory_order_acquire) < (int)nt) std::this_thread::yield();
        const size_t off = (size_t)bound[k] * elem, width = (size_t)(bound[k + 1] - bound[k]) * elem;
        if (e == cudaSuccess && width)
            e = cudaMemcpy2DAsync(static_cast<char*>(h->U) + off, (size_t)vh * elem,
                                  reinterpret_cast<const char*>(dst) + off, (size_t)vh * elem, width, planes,
                                  cudaMemcpyHostToDevice, h->stream);
    }
    if (pool) pool->wait();
    if (e != cudaSuccess) return lt::cuda_error(e, "lt_upload_links: copy");
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

} // namespace

extern "C" {

const char* lt_last_error(void) { return lt::g_last_error.c_str(); }

int lt_version(void) { return 100; }

int lt_create(const int ext[4], int prec, lt_lattice** out)
{
    if (!out || !ext) return lt::set_error(LT_ERR_ARG, "lt_create: null pointer");
    *out = nullptr;
    // 4 V 9 complex entries index the field in 32-bit arithmetic: the running product is checked
    // after every factor, so huge extents are refused before any multiplication can wrap
    long long V = 1;
    for (int d = 0; d < 4; ++d)
    {
        if (ext[d] < 2 || ext[d] % 2) return lt::set_error(LT_ERR_ARG, "lt_create: extents must be even and >= 2");
        V *= ext[d];
        if (V * 4 * 9 >= (1LL << 31)) return lt::set_error(LT_ERR_ARG, "lt_create: lattice too large");
    }
    const lt::Backend* be = prec == LT_PREC_FP64 ? lt::backend_fp64()
                          : prec == LT_PREC_FP32 ? lt::backend_fp32()
                          : prec == LT_PREC_FP32_12 ? lt::backend_fp32_12() : nullptr;
    if (!be) return lt::set_error(LT_ERR_ARG, "lt_create: unknown precision");
    auto* h = new (std::nothrow) lt_lattice();
    if (!h) return lt::set_error(LT_ERR_NOMEM, "lt_create: out of host memory");
    std::memcpy(h->ext, ext, sizeof(h->ext));
    h->prec = prec;
    h->g = lt::make_geom(ext);
    h->be = be;
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&h->U, be->gauge_bytes(h->g));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->partials, sizeof(double) * lt::kNumSlots * lt::kRedBlocks);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->results, sizeof(double) * lt::kNumSlots);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&h->h_results, sizeof(double) * lt::kNumSlots);
    // status[0]: the status word; status[1]: scratch of lt_check_links; status[2]: of lt_load_bmw
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->status, 4 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(h->status, 0, 4 * sizeof(unsigned), h->stream);
    if (e != cudaSuccess)
    {
        int r = lt::cuda_error(e, "lt_create");
        lt_destroy(h);
        return r;
    }
    be->set_unit(h->ctx(), h->U);
    int r = launched("lt_create");
    if (r != LT_OK)
    {
        lt_destroy(h);
        return r;
    }
    *out = h;
    return LT_OK;
}

int lt_destroy(lt_lattice* h)
{
    if (!h) return LT_OK;
    const lt::DeviceScope device_scope(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void* bufs[] = { h->U,   h->U2,   h->Z,        h->P,       h->F,     h->Ubak,   h->R,      h->chainA,
                     h->Lam, h->Tloc, h->partials, h->results, h->d_aos, h->status, h->chainB, h->Xz,
                     h->tensor };
    for (void* p : bufs)
        if (p) cudaFree(p);
    for (void* p : h->levels) cudaFree(p);
    for (void* p : h->staples) cudaFree(p);
    if (h->h_results) cudaFreeHost(h->h_results);
    if (h->h_stage) cudaFreeHost(h->h_stage);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LT_OK;
}

int lt_get_extents(const lt_lattice* h, int ext[4], int* prec)
{
    LT_TRY(check_h(h, "lt_get_extents"));
    const lt::DeviceScope device_scope(h->device);
    if (ext) std::memcpy(ext, h->ext, sizeof(h->ext));
    if (prec) *prec = h->prec;
    return LT_OK;
}

int lt_upload_links(lt_lattice* h, const double* links)
{
    LT_TRY(check_h(h, "lt_upload_links"));
    const lt::DeviceScope device_scope(h->device);
    if (!links) return lt::set_error(LT_ERR_ARG, "lt_upload_links: null pointer");
    // a handle uploaded more than once (a field streamed in step after step) packs on the host;
    // a single upload does not pay the pinned staging buffer's allocation
    if (h->prec == LT_PREC_FP32_12 && h->uploads++ > 0) return upload_packed_fp32(h, links);
    LT_TRY(ensure_aos(h));
    LT_CK(cudaMemcpyAsync(h->d_aos, links, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyHostToDevice,
                          h->stream));
    h->be->from_aos(h->ctx(), h->U, h->d_aos);
    LT_TRY(launched("lt_upload_links"));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_upload_bytes(const lt_lattice* h, const double* links, uint64_t* h2d_bytes)
{
    LT_TRY(check_h(h, "lt_upload_bytes"));
    if (!links || !h2d_bytes) return lt::set_error(LT_ERR_ARG, "lt_upload_bytes: null pointer");
    const lt::DeviceScope device_scope(h->device);
    const uint64_t V = (uint64_t)h->g.V;
    if (h->prec == LT_PREC_FP32_12 && h->uploads > 0)
    {
        const uint64_t s_split = (uint64_t)pack_split(h, links);
        *h2d_bytes = s_split * 24 * 16 + (V - 2 * s_split) * 72 * sizeof(double);
    }
    else
        *h2d_bytes = V * 72 * sizeof(double);
    return LT_OK;
}

int lt_pack_links_test(const int ext[4], const double* links, float* out)
{
    if (!ext || !links || !out) return lt::set_error(LT_ERR_ARG, "lt_pack_links_test: null pointer");
    if (reinterpret_cast<uintptr_t>(out) % 16) return lt::set_error(LT_ERR_ARG, "lt_pack_links_test: out not 16-byte aligned");
    long long V = 1;
    for (int d = 0; d < 4; ++d)
    {
        if (ext[d] < 2 || ext[d] % 2) return lt::set_error(LT_ERR_ARG, "lt_pack_links_test: extents must be even and >= 2");
        V *= ext[d];
        if (V * 4 * 9 >= (1LL << 31)) return lt::set_error(LT_ERR_ARG, "lt_pack_links_test: lattice too large");
    }
    const lt::Geom g = lt::make_geom(ext);
    pack_sites(g, 2, links, out, 0, g.V);
    return LT_OK;
}

int lt_download_links(lt_lattice* h, double* links)
{
    LT_TRY(check_h(h, "lt_download_links"));
    const lt::DeviceScope device_scope(h->device);
    if (!links) return lt::set_error(LT_ERR_ARG, "lt_download_links: null pointer");
    LT_TRY(ensure_aos(h));
    h->be->to_aos(h->ctx(), h->U, h->d_aos);
    LT_TRY(launched("lt_download_links"));
    LT_CK(cudaMemcpyAsync(links, h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyDeviceToHost,
                          h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

static int link_access(lt_lattice* h, int64_t site, int mu, double* m, int write)
{
    if (!m || site < 0 || site >= h->g.V || mu < 0 || mu > 3)
        return lt::set_error(LT_ERR_ARG, "lt_set_link/lt_get_link: bad site, direction or pointer");
    LT_TRY(ensure_aos(h));
    if (write) LT_CK(cudaMemcpyAsync(h->d_aos, m, 18 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->be->link_io(h->ctx(), h->U, (int)site, mu, h->d_aos, write);
    LT_TRY(launched("link access"));
    if (!write) LT_CK(cudaMemcpyAsync(m, h->d_aos, 18 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_set_link(lt_lattice* h, int64_t site, int mu, const double* m)
{
    LT_TRY(check_h(h, "lt_set_link"));
    const lt::DeviceScope device_scope(h->device);
    return link_access(h, site, mu, const_cast<double*>(m), 1);
}

int lt_get_link(lt_lattice* h, int64_t site, int mu, double* m_out)
{
    LT_TRY(check_h(h, "lt_get_link"));
    const lt::DeviceScope device_scope(h->device);
    return link_access(h, site, mu, m_out, 0);
}

int lt_copy(lt_lattice* dst, const lt_lattice* src)
{
    LT_TRY(check_h(dst, "lt_copy"));
    LT_TRY(check_h(src, "lt_copy"));
    const lt::DeviceScope device_scope(dst->device);
    if (dst == src) return LT_OK;
    if (std::memcmp(dst->ext, src->ext, sizeof(dst->ext)))
        return lt::set_error(LT_ERR_ARG, "lt_copy: extents differ");
    LT_TRY(order_after(dst, src));
    if (dst->prec == src->prec)
    {
        LT_CK(cudaMemcpyAsync(dst->U, src->U, dst->be->gauge_bytes(dst->g), cudaMemcpyDeviceToDevice, dst->stream));
    }
    else
    {
        LT_TRY(ensure_aos(dst));
        src->be->to_aos(dst->ctx(), src->U, dst->d_aos);
        dst->be->from_aos(dst->ctx(), dst->U, dst->d_aos);
    }
    LT_TRY(launched("lt_copy"));
    // src may be reused by its owner right after this returns
    LT_CK(cudaStreamSynchronize(dst->stream));
    return LT_OK;
}

int lt_swap(lt_lattice* a, lt_lattice* b)
{
    LT_TRY(check_h(a, "lt_swap"));
    LT_TRY(check_h(b, "lt_swap"));
    const lt::DeviceScope device_scope(a->device);
    if (std::memcmp(a->ext, b->ext, sizeof(a->ext)) || a->prec != b->prec)
        return lt::set_error(LT_ERR_ARG, "lt_swap: extents or formats differ");
    // the link buffers change owners: a buffer on another GPU would be read by this handle's
    // kernels through a pointer its device cannot dereference
    if (a->device != b->device) return lt::set_error(LT_ERR_ARG, "lt_swap: handles live on different devices");
    LT_CK(cudaStreamSynchronize(a->stream));
    LT_CK(cudaStreamSynchronize(b->stream));
    std::swap(a->U, b->U);
    return LT_OK;
}

int lt_set_identity(lt_lattice* h)
{
    LT_TRY(check_h(h, "lt_set_identity"));
    const lt::DeviceScope device_scope(h->device);
    h->be->set_unit(h->ctx(), h->U);
    return launched("lt_set_identity");
}

int lt_set_haar_random(lt_lattice* h, uint64_t seed)
{
    LT_TRY(check_h(h, "lt_set_haar_random"));
    const lt::DeviceScope device_scope(h->device);
    std::vector<double> buf;
    try
    {
        buf.resize((size_t)4 * h->g.V * 18);
    }
    catch (...)
    {
        return lt::set_error(LT_ERR_NOMEM, "lt_set_haar_random: out of host memory");
    }
    lt::haar_links(h->ext, seed, buf.data());
    return lt_upload_links(h, buf.data());
}

int lt_synchronize(lt_lattice* h)
{
    LT_TRY(check_h(h, "lt_synchronize"));
    const lt::DeviceScope device_scope(h->device);
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_get_stream(const lt_lattice* h, void** stream_out)
{
    LT_TRY(check_h(h, "lt_get_stream"));
    const lt::DeviceScope device_scope(h->device);
    if (!stream_out) return lt::set_error(LT_ERR_ARG, "lt_get_stream: null pointer");
    *stream_out = (void*)h->stream;
    return LT_OK;
}

static_assert(LT_STATUS_NONFINITE == lt::kStatusNonFinite && LT_STATUS_UNITARITY == lt::kStatusUnitarity &&
                  LT_STATUS_HB_CAP == lt::kStatusHbCap,
              "status bits of the C ABI and the kernels differ");

int lt_status_word(lt_lattice* h, uint32_t* word, int clear)
{
    LT_TRY(check_h(h, "lt_status_word"));
    const lt::DeviceScope device_scope(h->device);
    if (!word) return lt::set_error(LT_ERR_ARG, "lt_status_word: null pointer");
    LT_CK(cudaMemcpyAsync(h->h_results, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    if (clear) LT_CK(cudaMemsetAsync(h->status, 0, sizeof(unsigned), h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    unsigned w;
    std::memcpy(&w, h->h_results, sizeof(w));
    *word = w;
    return LT_OK;
}

int lt_check_links(lt_lattice* h, double* max_dev)
{
    LT_TRY(check_h(h, "lt_check_links"));
    const lt::DeviceScope device_scope(h->device);
    unsigned* maxbits = h->status + 1;
    LT_CK(cudaMemsetAsync(maxbits, 0, sizeof(unsigned), h->stream));
    const double tol = h->be->real_bytes() == 8 ? 1e-10 : 1e-4;
    h->be->check_links(h->ctx(), h->U, tol, maxbits);
    LT_TRY(launched("lt_check_links"));
    LT_CK(cudaMemcpyAsync(h->h_results, maxbits, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    float f;
    std::memcpy(&f, h->h_results, sizeof(f));
    if (max_dev) *max_dev = (double)f;
    return LT_OK;
}

// ---------------------------------------------------------------- observables
int lt_plaquette_sum(lt_lattice* h, double* out)
{
    LT_TRY(check_h(h, "lt_plaquette_sum"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_plaquette_sum: null pointer");
    return plaq_of(h, h->U, out);
}

int lt_wilson_action(lt_lattice* h, double beta, double* out)
{
    LT_TRY(check_h(h, "lt_wilson_action"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_wilson_action: null pointer");
    double p;
    LT_TRY(plaq_of(h, h->U, &p));
    *out = beta * (6.0 * (double)h->g.V - p / 3.0);
    return LT_OK;
}

int lt_topcharge_clover(lt_lattice* h, double* out)
{
    LT_TRY(check_h(h, "lt_topcharge_clover"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_topcharge_clover: null pointer");
    return clover_q_e(h, h->U, out, nullptr);
}

int lt_energy_clover(lt_lattice* h, double* out)
{
    LT_TRY(check_h(h, "lt_energy_clover"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_energy_clover: null pointer");
    return clover_q_e(h, h->U, nullptr, out);
}

int lt_clover_timeslices(lt_lattice* h, double* q_t, double* e_t)
{
    LT_TRY(check_h(h, "lt_clover_timeslices"));
    const lt::DeviceScope device_scope(h->device);
    if (!q_t && !e_t) return lt::set_error(LT_ERR_ARG, "lt_clover_timeslices: null pointers");
    const int nt = h->g.n[0];
    const int nbx = std::max(1, std::min(lt::kRedBlocks / nt, (h->g.V / nt + lt::kRedThreads - 1) / lt::kRedThreads));
    if (2 * nt * nbx > lt::kNumSlots * lt::kRedBlocks)
        return lt::set_error(LT_ERR_ARG, "lt_clover_timeslices: more timeslices than the partial-sum buffer holds");
    h->be->clover_timeslices(h->ctx(), h->U, h->partials, nbx);
    LT_TRY(launched("lt_clover_timeslices"));
    std::vector<double> p((size_t)2 * nt * nbx);
    LT_CK(cudaMemcpyAsync(p.data(), h->partials, sizeof(double) * p.size(), cudaMemcpyDeviceToHost, h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    for (int t = 0; t < nt; ++t)
    {
        double sq = 0.0, cq = 0.0, se = 0.0, ce = 0.0;   // Kahan, fixed order
        for (int b = 0; b < nbx; ++b)
        {
            double y = p[(size_t)t * nbx + b] - cq, s2 = sq + y;
            cq = (s2 - sq) - y;
            sq = s2;
            y = p[(size_t)(nt + t) * nbx + b] - ce;
            s2 = se + y;
            ce = (s2 - se) - y;
            se = s2;
        }
        if (q_t) q_t[t] = -1.0 / (64.0 * 4.0 * kPi * kPi) * sq;
        if (e_t) e_t[t] = se / (double)h->g.V;
    }
    return LT_OK;
}

int lt_topcharge_plaquette(lt_lattice* h, double* out)
{
    LT_TRY(check_h(h, "lt_topcharge_plaquette"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_topcharge_plaquette: null pointer");
    h->be->loops(h->ctx(), h->U, 4);
    double r[3];
    LT_TRY(fetch(h, 4, 3, r));
    *out = 1.0 / (16.0 * kPi * kPi) * r[2];
    return LT_OK;
}

int lt_rect_action(lt_lattice* h, double beta, double c_plaq, double c_rect, double* out)
{
    LT_TRY(check_h(h, "lt_rect_action"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_rect_action: null pointer");
    h->be->loops(h->ctx(), h->U, 4);
    double r[3];
    LT_TRY(fetch(h, 4, 3, r));
    const double V = (double)h->g.V;
    *out = beta * (c_plaq * (6.0 * V - r[0] / 3.0) + c_rect * (12.0 * V - r[1] / 3.0));
    return LT_OK;
}

int lt_wilson_loop(lt_lattice* h, int L, double* out)
{
    LT_TRY(check_h(h, "lt_wilson_loop"));
    const lt::DeviceScope device_scope(h->device);
    if (!out || L < 1) return lt::set_error(LT_ERR_ARG, "lt_wilson_loop: null pointer or L < 1");
    const size_t bytes = (size_t)4 * h->g.V * 9 * 2 * sizeof(double);
    LT_TRY(ensure(h, &h->chainA, bytes));
    LT_TRY(ensure(h, &h->chainB, bytes));
    const lt::Ctx c = h->ctx();
    h->be->chain_init(c, h->U, h->chainA);
    void *cur = h->chainA, *nxt = h->chainB;
    // the buffers are the ones lt_wilson_loop_chain keeps its chain in
    h->chain_len = -1;
    h->chain_cur = nullptr;
    if ((L & (L - 1)) == 0)
        for (int len = 1; len < L; len *= 2)
        {
            h->be->chain_double(c, cur, nxt, len);
            std::swap(cur, nxt);
        }
    else
        for (int len = 1; len < L; ++len)
        {
            h->be->chain_extend(c, cur, h->U, nxt, len);
            std::swap(cur, nxt);
        }
    h->be->wilson_square(c, cur, L, 0);
    double w;
    LT_TRY(fetch(h, 0, 1, &w));
    *out = 1.0 - w / (18.0 * (double)h->g.V);
    return LT_OK;
}

int lt_wilson_loop_chain(lt_lattice* h, int start, int end, int reset, double* out)
{
    LT_TRY(check_h(h, "lt_wilson_loop_chain"));
    const lt::DeviceScope device_scope(h->device);
    if (!out || start < 0 || end < 1 || end < start)
        return lt::set_error(LT_ERR_ARG, "lt_wilson_loop_chain: null pointer or not 0 <= start <= end, end >= 1");
    if (!reset && h->chain_len < 0)
        return lt::set_error(LT_ERR_STATE, "lt_wilson_loop_chain: no chain to extend (call with reset first)");
    const size_t bytes = (size_t)4 * h->g.V * 9 * 2 * sizeof(double);
    LT_TRY(ensure(h, &h->chainA, bytes));
    LT_TRY(ensure(h, &h->chainB, bytes));
    const lt::Ctx c = h->ctx();
    void* cur = h->chain_cur ? h->chain_cur : h->chainA;
    int n = start;   // the next factor is U(x + n mu)
    if (reset)
    {
        // U_chain = 1, then the factors n = start..end-1 (wilson_loop.hpp:75-88); from the
        // origin the first factor is a copy of the links
        cur = h->chainA;
        h->chain_origin = start;
        h->chain_contig = true;
        if (start == 0 && end > 0)
        {
            h->be->chain_init(c, h->U, cur);
            h->chain_len = 1;
            n = 1;
        }
        else
        {
            h->be->chain_unit(c, cur);
            h->chain_len = 0;
        }
    }
    else if (h->chain_origin + h->chain_len != start)
        h->chain_contig = false;   // the chain no longer holds one straight run of links
    while (n < end)
    {
        void* nxt = cur == h->chainA ? h->chainB : h->chainA;
        if (h->chain_contig && h->chain_origin == 0 && h->chain_len == n && 2 * n <= end)
        {
            // C(x) C(x + n mu): the run of length n doubles with one product per link
            h->be->chain_double(c, cur, nxt, n);
            h->chain_len = 2 * n;
            n *= 2;
        }
        else
        {
            h->be->chain_extend(c, cur, h->U, nxt, n);
            if (h->chain_contig && h->chain_origin + h->chain_len == n) ++h->chain_len;
            else h->chain_contig = false;
            ++n;
        }
        cur = nxt;
    }
    h->chain_cur = cur;
    LT_TRY(launched("lt_wilson_loop_chain"));
    h->be->wilson_square(c, cur, end, 0);
    double w;
    LT_TRY(fetch(h, 0, 1, &w));
    *out = 1.0 - w / (18.0 * (double)h->g.V);
    return LT_OK;
}

int lt_polyakov_loop(lt_lattice* h, double* re, double* im)
{
    LT_TRY(check_h(h, "lt_polyakov_loop"));
    const lt::DeviceScope device_scope(h->device);
    if (!re || !im) return lt::set_error(LT_ERR_ARG, "lt_polyakov_loop: null pointer");
    h->be->polyakov(h->ctx(), h->U, 0);
    double r[2];
    LT_TRY(fetch(h, 0, 2, r));
    const double vs = (double)(h->g.V / h->g.n[0]);
    *re = r[0] / vs;
    *im = r[1] / vs;
    return LT_OK;
}

int lt_clover_observables(lt_lattice* h, double* q_out, double* e_out)
{
    LT_TRY(check_h(h, "lt_clover_observables"));
    const lt::DeviceScope device_scope(h->device);
    return clover_q_e(h, h->U, q_out, e_out);
}

int lt_staples(lt_lattice* h, double* staples_out)
{
    LT_TRY(check_h(h, "lt_staples"));
    const lt::DeviceScope device_scope(h->device);
    if (!staples_out) return lt::set_error(LT_ERR_ARG, "lt_staples: null pointer");
    LT_TRY(ensure_aos(h));
    h->be->staples_aos(h->ctx(), h->U, h->d_aos);
    LT_TRY(launched("lt_staples"));
    LT_CK(cudaMemcpyAsync(staples_out, h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyDeviceToHost,
                          h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

// ---------------------------------------------------------------- local updates
int lt_set_gauge_action(lt_lattice* h, int stencil_radius, double c_plaq, double c_rect)
{
    LT_TRY(check_h(h, "lt_set_gauge_action"));
    const lt::DeviceScope device_scope(h->device);
    if ((stencil_radius != 1 && stencil_radius != 2) || !std::isfinite(c_plaq) || !std::isfinite(c_rect))
        return lt::set_error(LT_ERR_ARG, "lt_set_gauge_action: stencil radius 1 or 2 and finite coefficients");
    h->act_radius = stencil_radius;
    h->act_cp = c_plaq;
    h->act_cr = stencil_radius == 2 ? c_rect : 0.0;
    return LT_OK;
}

int lt_get_gauge_action(lt_lattice* h, int* stencil_radius, double* c_plaq, double* c_rect)
{
    LT_TRY(check_h(h, "lt_get_gauge_action"));
    const lt::DeviceScope device_scope(h->device);
    if (stencil_radius) *stencil_radius = h->act_radius;
    if (c_plaq) *c_plaq = h->act_cp;
    if (c_rect) *c_rect = h->act_cr;
    return LT_OK;
}

int lt_overrelax_sweeps(lt_lattice* h, int n_sweep)
{
    LT_TRY(check_h(h, "lt_overrelax_sweeps"));
    const lt::DeviceScope device_scope(h->device);
    if (n_sweep < 0) return lt::set_error(LT_ERR_ARG, "lt_overrelax_sweeps: n_sweep < 0");
    if (h->act_radius == 2)
        return lt::set_error(LT_ERR_ARG, "lt_overrelax_sweeps: a rectangular action needs Checkerboard4 (lt_overrelax_sweeps4)");
    const lt::Ctx c = h->ctx();
    for (int s = 0; s < n_sweep; ++s)
        for (int mu = 0; mu < 4; ++mu)
            for (int par = 0; par < 2; ++par) h->be->overrelax(c, h->U, mu, par);
    return launched("lt_overrelax_sweeps");
}

int lt_heatbath_sweeps(lt_lattice* h, double beta, int n_sweep, uint64_t seed, uint64_t* counter)
{
    LT_TRY(check_h(h, "lt_heatbath_sweeps"));
    const lt::DeviceScope device_scope(h->device);
    if (n_sweep < 0 || !counter || !(beta > 0.0))
        return lt::set_error(LT_ERR_ARG, "lt_heatbath_sweeps: bad arguments");
    if (h->act_radius == 2)
        return lt::set_error(LT_ERR_ARG, "lt_heatbath_sweeps: a rectangular action needs Checkerboard4 (lt_heatbath_sweeps4)");
    const lt::Ctx c = h->ctx();
    for (int s = 0; s < n_sweep; ++s)
    {
        for (int mu = 0; mu < 4; ++mu)
            for (int par = 0; par < 2; ++par) h->be->heatbath(c, h->U, mu, par, 3.0 / beta, *counter, seed, 10);
        ++*counter;
    }
    return launched("lt_heatbath_sweeps");
}

int lt_update_sweeps(lt_lattice* h, double beta, int n_sweep, int n_hb, int n_or, uint64_t seed, uint64_t* counter)
{
    LT_TRY(check_h(h, "lt_update_sweeps"));
    const lt::DeviceScope device_scope(h->device);
    if (n_sweep < 0 || n_hb < 0 || n_or < 0 || !counter || !(beta > 0.0))
        return lt::set_error(LT_ERR_ARG, "lt_update_sweeps: bad arguments");
    for (int s = 0; s < n_sweep; ++s)
    {
        LT_TRY(lt_heatbath_sweeps(h, beta, n_hb, seed, counter));
        LT_TRY(lt_overrelax_sweeps(h, n_or));
    }
    return LT_OK;
}

static int check_cb4(const lt_lattice* h, const char* fn)
{
    for (int d = 0; d < 4; ++d)
        if (h->ext[d] % 4 != 0)
            return lt::set_error(LT_ERR_ARG, (std::string(fn) + ": Checkerboard4 needs every extent a multiple of 4").c_str());
    return LT_OK;
}

int lt_overrelax_sweeps4(lt_lattice* h, int n_sweep)
{
    LT_TRY(check_h(h, "lt_overrelax_sweeps4"));
    const lt::DeviceScope device_scope(h->device);
    if (n_sweep < 0) return lt::set_error(LT_ERR_ARG, "lt_overrelax_sweeps4: n_sweep < 0");
    LT_TRY(check_cb4(h, "lt_overrelax_sweeps4"));
    const lt::Ctx c = h->ctx();
    for (int s = 0; s < n_sweep; ++s)
        for (int mu = 0; mu < 4; ++mu)
            for (int sub = 0; sub < 4; ++sub) h->be->sweep4(c, h->U, 1, mu, sub, 0.0, 0, 0, 0);
    return launched("lt_overrelax_sweeps4");
}

int lt_heatbath_sweeps4(lt_lattice* h, double beta, int n_sweep, uint64_t seed, uint64_t* counter)
{
    LT_TRY(check_h(h, "lt_heatbath_sweeps4"));
    const lt::DeviceScope device_scope(h->device);
    if (n_sweep < 0 || !counter || !(beta > 0.0))
        return lt::set_error(LT_ERR_ARG, "lt_heatbath_sweeps4: bad arguments");
    LT_TRY(check_cb4(h, "lt_heatbath_sweeps4"));
    const lt::Ctx c = h->ctx();
    for (int s = 0; s < n_sweep; ++s)
    {
        for (int mu = 0; mu < 4; ++mu)
            for (int sub = 0; sub < 4; ++sub) h->be->sweep4(c, h->U, 0, mu, sub, 3.0 / beta, *counter, seed, 10);
        ++*counter;
    }
    return launched("lt_heatbath_sweeps4");
}

int lt_update_sweeps4(lt_lattice* h, double beta, int n_sweep, int n_hb, int n_or, uint64_t seed, uint64_t* counter)
{
    LT_TRY(check_h(h, "lt_update_sweeps4"));
    const lt::DeviceScope device_scope(h->device);
    if (n_sweep < 0 || n_hb < 0 || n_or < 0 || !counter || !(beta > 0.0))
        return lt::set_error(LT_ERR_ARG, "lt_update_sweeps4: bad arguments");
    for (int s = 0; s < n_sweep; ++s)
    {
        LT_TRY(lt_heatbath_sweeps4(h, beta, n_hb, seed, counter));
        LT_TRY(lt_overrelax_sweeps4(h, n_or));
    }
    return LT_OK;
}

// ---------------------------------------------------------------- smearing
int lt_flow_rk3(lt_lattice* in, lt_lattice* out, double eps, int n_step)
{
    LT_TRY(check_h(in, "lt_flow_rk3"));
    LT_TRY(check_h(out, "lt_flow_rk3"));
    const lt::DeviceScope device_scope(in->device);
    if (n_step < 0) return lt::set_error(LT_ERR_ARG, "lt_flow_rk3: n_step < 0");
    LT_TRY(lt_copy(out, in));
    return flow_steps(out, eps, n_step);
}

int lt_flow(lt_lattice* in, lt_lattice* out, int integrator, double eps, int n_step)
{
    LT_TRY(check_h(in, "lt_flow"));
    LT_TRY(check_h(out, "lt_flow"));
    const lt::DeviceScope device_scope(in->device);
    if (n_step < 0 || integrator < LT_FLOW_EULER || integrator > LT_FLOW_RK3W7)
        return lt::set_error(LT_ERR_ARG, "lt_flow: n_step < 0 or unknown integrator");
    LT_TRY(lt_copy(out, in));
    return flow_steps(out, eps, n_step, integrator);
}

// ---------------------------------------------------------------- clover tensor
int lt_clover_tensor(lt_lattice* h, double* tensor_out)
{
    LT_TRY(check_h(h, "lt_clover_tensor"));
    const lt::DeviceScope device_scope(h->device);
    const size_t bytes = (size_t)h->g.V * 16 * 18 * sizeof(double);
    LT_TRY(ensure(h, (void**)&h->tensor, bytes));
    LT_CK(cudaMemsetAsync(h->tensor, 0, bytes, h->stream));
    h->be->clover_tensor(h->ctx(), h->U, h->tensor);
    LT_TRY(launched("lt_clover_tensor"));
    if (tensor_out)
    {
        LT_CK(cudaMemcpyAsync(tensor_out, h->tensor, bytes, cudaMemcpyDeviceToHost, h->stream));
        LT_CK(cudaStreamSynchronize(h->stream));
    }
    return LT_OK;
}

int lt_topcharge_clover_tensor(lt_lattice* h, const double* tensor, double* q_out)
{
    LT_TRY(check_h(h, "lt_topcharge_clover_tensor"));
    if (!q_out) return lt::set_error(LT_ERR_ARG, "lt_topcharge_clover_tensor: null output");
    const lt::DeviceScope device_scope(h->device);
    const size_t bytes = (size_t)h->g.V * 16 * 18 * sizeof(double);
    if (tensor)
    {
        LT_TRY(ensure(h, (void**)&h->tensor, bytes));
        LT_CK(cudaMemcpyAsync(h->tensor, tensor, bytes, cudaMemcpyHostToDevice, h->stream));
    }
    else if (!h->tensor)
        return lt::set_error(LT_ERR_STATE, "lt_topcharge_clover_tensor: no tensor given and none computed");
    h->be->topcharge_tensor(h->ctx(), h->tensor, 0);
    double r;
    LT_TRY(fetch(h, 0, 1, &r));
    *q_out = -1.0 / (64.0 * 4.0 * kPi * kPi) * r;
    return LT_OK;
}

int lt_set_flow_action(lt_lattice* h, int flow_action)
{
    LT_TRY(check_h(h, "lt_set_flow_action"));
    if (flow_action != LT_FLOW_ACTION_GAUGE && flow_action != LT_FLOW_ACTION_ZEUTHEN)
        return lt::set_error(LT_ERR_ARG, "lt_set_flow_action: unknown flow action");
    h->flow_action = flow_action;
    return LT_OK;
}

int lt_get_flow_action(lt_lattice* h, int* flow_action)
{
    LT_TRY(check_h(h, "lt_get_flow_action"));
    if (!flow_action) return lt::set_error(LT_ERR_ARG, "lt_get_flow_action: null pointer");
    *flow_action = h->flow_action;
    return LT_OK;
}

int lt_flow_rk3_measure(lt_lattice* in, lt_lattice* out, double eps, int n_meas, int every, double* plaq_out,
                        double* q_out, double* e_out)
{
    LT_TRY(check_h(in, "lt_flow_rk3_measure"));
    LT_TRY(check_h(out, "lt_flow_rk3_measure"));
    const lt::DeviceScope device_scope(in->device);
    if (n_meas < 0 || every < 0) return lt::set_error(LT_ERR_ARG, "lt_flow_rk3_measure: negative count");
    LT_TRY(lt_copy(out, in));
    for (int m = 0; m < n_meas; ++m)
    {
        LT_TRY(flow_steps(out, eps, every));
        if (plaq_out) LT_TRY(plaq_of(out, out->U, &plaq_out[m]));
        if (q_out || e_out)
            LT_TRY(clover_q_e(out, out->U, q_out ? &q_out[m] : nullptr, e_out ? &e_out[m] : nullptr));
    }
    return LT_OK;
}

int lt_flow_t0(lt_lattice* in, lt_lattice* out, double eps, double target, int max_steps, double* t0_out,
               double* q_out)
{
    LT_TRY(check_h(in, "lt_flow_t0"));
    LT_TRY(check_h(out, "lt_flow_t0"));
    const lt::DeviceScope device_scope(in->device);
    if (!t0_out || !(eps > 0.0) || max_steps < 1) return lt::set_error(LT_ERR_ARG, "lt_flow_t0: bad arguments");
    LT_TRY(lt_copy(out, in));
    double t_prev = 0.0, y_prev = 0.0, q = 0.0, e = 0.0;
    for (int k = 1; k <= max_steps; ++k)
    {
        LT_TRY(flow_steps(out, eps, 1));
        LT_TRY(clover_q_e(out, out->U, &q, &e));
        const double t = k * eps, y = t * t * e;
        if (y >= target)
        {
            *t0_out = k == 1 ? t : t_prev + (target - y_prev) / (y - y_prev) * (t - t_prev);
            if (q_out) *q_out = q;
            return LT_OK;
        }
        t_prev = t;
        y_prev = y;
    }
    if (q_out) *q_out = q;
    return lt::set_error(LT_ERR_STATE, "lt_flow_t0: t^2 E did not reach the target within max_steps");
}

int lt_stout(lt_lattice* in, lt_lattice* out, double rho, int n)
{
    LT_TRY(check_h(in, "lt_stout"));
    LT_TRY(check_h(out, "lt_stout"));
    const lt::DeviceScope device_scope(in->device);
    if (n < 0) return lt::set_error(LT_ERR_ARG, "lt_stout: n < 0");
    LT_TRY(lt_copy(out, in));
    return stout_steps(out, rho, n);
}

// ---------------------------------------------------------------- HMC
int lt_gauge_force(lt_lattice* h, double beta, double* force_out)
{
    LT_TRY(check_h(h, "lt_gauge_force"));
    const lt::DeviceScope device_scope(h->device);
    if (!force_out) return lt::set_error(LT_ERR_ARG, "lt_gauge_force: null pointer");
    LT_TRY(ensure(h, &h->F, h->be->alg_bytes(h->g)));
    LT_CK(cudaMemsetAsync(h->F, 0, h->be->alg_bytes(h->g), h->stream));
    h->be->momenta(h->ctx(), h->U, h->F, nullptr, beta / 6.0, 1.0);
    LT_TRY(ensure_aos(h));
    h->be->alg_to_aos(h->ctx(), h->F, h->d_aos);
    LT_TRY(launched("lt_gauge_force"));
    LT_CK(cudaMemcpyAsync(force_out, h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyDeviceToHost,
                          h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_set_momenta(lt_lattice* h, const double* p)
{
    LT_TRY(check_h(h, "lt_set_momenta"));
    const lt::DeviceScope device_scope(h->device);
    if (!p) return lt::set_error(LT_ERR_ARG, "lt_set_momenta: null pointer");
    LT_TRY(ensure(h, &h->P, h->be->alg_bytes(h->g)));
    LT_TRY(ensure_aos(h));
    LT_CK(cudaMemcpyAsync(h->d_aos, p, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->be->alg_from_aos(h->ctx(), h->P, h->d_aos);
    LT_TRY(launched("lt_set_momenta"));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_get_momenta(lt_lattice* h, double* p_out)
{
    LT_TRY(check_h(h, "lt_get_momenta"));
    const lt::DeviceScope device_scope(h->device);
    if (!p_out) return lt::set_error(LT_ERR_ARG, "lt_get_momenta: null pointer");
    if (!h->P) return lt::set_error(LT_ERR_STATE, "lt_get_momenta: no momenta set");
    LT_TRY(ensure_aos(h));
    h->be->alg_to_aos(h->ctx(), h->P, h->d_aos);
    LT_TRY(launched("lt_get_momenta"));
    LT_CK(cudaMemcpyAsync(p_out, h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyDeviceToHost,
                          h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_random_momenta(lt_lattice* h, uint64_t seed, uint64_t counter)
{
    LT_TRY(check_h(h, "lt_random_momenta"));
    const lt::DeviceScope device_scope(h->device);
    LT_TRY(ensure(h, &h->P, h->be->alg_bytes(h->g)));
    h->be->random_momenta(h->ctx(), h->P, counter, seed);
    return launched("lt_random_momenta");
}

int lt_hamiltonian(lt_lattice* h, double beta, double* out)
{
    LT_TRY(check_h(h, "lt_hamiltonian"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_hamiltonian: null pointer");
    if (!h->P) return lt::set_error(LT_ERR_STATE, "lt_hamiltonian: no momenta set");
    return hamiltonian(h, beta, out);
}

int lt_omf2(lt_lattice* h, double beta, double tau, int n_step, double* h_old, double* h_new)
{
    LT_TRY(check_h(h, "lt_omf2"));
    const lt::DeviceScope device_scope(h->device);
    if (!h->P) return lt::set_error(LT_ERR_STATE, "lt_omf2: no momenta set");
    if (h_old) LT_TRY(hamiltonian(h, beta, h_old));
    LT_TRY(omf2(h, beta, tau, n_step, nullptr));
    if (h_new) LT_TRY(hamiltonian(h, beta, h_new));
    return LT_OK;
}

int lt_hmc_trajectory(lt_lattice* h, double beta, double tau, int n_step, uint64_t seed, uint64_t* counter,
                      int metropolis, double* dH, int* accepted)
{
    return lt_md_trajectory(h, nullptr, LT_MD_OMF2, beta, tau, n_step, 0.0, 0, seed, counter, metropolis, dH, accepted,
                            nullptr);
}

int lt_reverse_momenta(lt_lattice* h)
{
    LT_TRY(check_h(h, "lt_reverse_momenta"));
    const lt::DeviceScope device_scope(h->device);
    if (!h->P) return lt::set_error(LT_ERR_STATE, "lt_reverse_momenta: no momenta set");
    h->be->alg_axpby(h->ctx(), h->P, nullptr, -1.0, 0.0);
    return launched("lt_reverse_momenta");
}

int lt_parity_update(lt_lattice* h)
{
    LT_TRY(check_h(h, "lt_parity_update"));
    const lt::DeviceScope device_scope(h->device);
    LT_TRY(ensure(h, &h->U2, h->be->gauge_bytes(h->g)));
    h->be->parity(h->ctx(), h->U, h->U2);
    std::swap(h->U, h->U2);
    return launched("lt_parity_update");
}

// ---------------------------------------------------------------- metadynamics
int lt_clover_derivative(lt_lattice* h, double* out)
{
    LT_TRY(check_h(h, "lt_clover_derivative"));
    const lt::DeviceScope device_scope(h->device);
    if (!out) return lt::set_error(LT_ERR_ARG, "lt_clover_derivative: null pointer");
    LT_TRY(metad_backward(h, 0.0, 0, 1.0));
    LT_TRY(ensure_aos(h));
    h->be->alg_to_aos(h->ctx(), h->F, h->d_aos);
    LT_TRY(launched("lt_clover_derivative"));
    LT_CK(cudaMemcpyAsync(out, h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_metad_charge(lt_lattice* h, double rho, int n_stout, double* q_out)
{
    LT_TRY(check_h(h, "lt_metad_charge"));
    const lt::DeviceScope device_scope(h->device);
    if (!q_out || n_stout < 0) return lt::set_error(LT_ERR_ARG, "lt_metad_charge: bad arguments");
    return metad_charge(h, rho, n_stout, q_out);
}

int lt_metad_force(lt_lattice* h, double rho, int n_stout, double dvdq, double* force_out, double* q_out)
{
    LT_TRY(check_h(h, "lt_metad_force"));
    const lt::DeviceScope device_scope(h->device);
    if (n_stout < 0) return lt::set_error(LT_ERR_ARG, "lt_metad_force: n_stout < 0");
    LT_TRY(metad_forward(h, rho, n_stout));
    LT_TRY(metad_clover(h, n_stout));
    // the charge is summed before the backward chain but read after it, so the host does not
    // wait between the two halves of the force
    if (q_out) h->be->topcharge_R(h->ctx(), h->R, 7);
    LT_TRY(metad_backward(h, rho, n_stout, dvdq, true));
    if (q_out)
    {
        double r;
        LT_TRY(fetch(h, 7, 1, &r));
        *q_out = -1.0 / (64.0 * 4.0 * kPi * kPi) * r;
    }
    if (force_out)
    {
        LT_TRY(ensure_aos(h));
        h->be->alg_to_aos(h->ctx(), h->F, h->d_aos);
        LT_TRY(launched("lt_metad_force"));
        LT_CK(cudaMemcpyAsync(force_out, h->d_aos, (size_t)4 * h->g.V * 18 * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream));
    }
    LT_CK(cudaStreamSynchronize(h->stream));
    return LT_OK;
}

int lt_metad_omf2(lt_lattice* h, lt_bias* bias, double beta, double tau, int n_step, double rho, int n_stout,
                  double* h_old, double* h_new)
{
    LT_TRY(check_h(h, "lt_metad_omf2"));
    const lt::DeviceScope device_scope(h->device);
    if (!bias) return lt::set_error(LT_ERR_ARG, "lt_metad_omf2: null bias");
    return lt_md_integrate(h, bias, LT_MD_OMF2, beta, tau, n_step, rho, n_stout, h_old, h_new);
}

int lt_metad_hmc_trajectory(lt_lattice* h, lt_bias* bias, double beta, double tau, int n_step, double rho,
                            int n_stout, uint64_t seed, uint64_t* counter, int metropolis, double* dH, int* accepted,
                            double* cv_out)
{
    LT_TRY(check_h(h, "lt_metad_hmc_trajectory"));
    const lt::DeviceScope device_scope(h->device);
    if (!bias) return lt::set_error(LT_ERR_ARG, "lt_metad_hmc_trajectory: null bias");
    return lt_md_trajectory(h, bias, LT_MD_OMF2, beta, tau, n_step, rho, n_stout, seed, counter, metropolis, dH,
                            accepted, cv_out);
}

// H (+ V(CV) under MetaD) of the current links and momenta
static int md_energy(lt_lattice* h, lt::Bias* b, double beta, double rho, int n_stout, double* e, double* cv)
{
    double hh;
    if (b)
    {
        LT_TRY(metad_charge(h, rho, n_stout, cv));
        LT_TRY(hamiltonian(h, beta, &hh));
        *e = hh + b->potential(*cv);
        return LT_OK;
    }
    LT_TRY(hamiltonian(h, beta, &hh));
    *e = hh;
    return LT_OK;
}

int lt_md_integrate(lt_lattice* h, lt_bias* bias, int integrator, double beta, double tau, int n_step, double rho,
                    int n_stout, double* h_old, double* h_new)
{
    LT_TRY(check_h(h, "lt_md_integrate"));
    const lt::DeviceScope device_scope(h->device);
    if (!h->P) return lt::set_error(LT_ERR_STATE, "lt_md_integrate: no momenta set");
    if (bias && n_stout < 0) return lt::set_error(LT_ERR_ARG, "lt_md_integrate: n_stout < 0");
    LT_TRY(md_check(integrator, bias != nullptr, "lt_md_integrate"));
    auto* b = reinterpret_cast<lt::Bias*>(bias);
    double cv;
    if (h_old) LT_TRY(md_energy(h, b, beta, rho, n_stout, h_old, &cv));
    std::vector<MdOp> ops;
    md_program(integrator, tau, n_step, ops);
    MetaDParams md { b, rho, n_stout, nullptr };
    LT_TRY(integrate(h, beta, ops, b ? &md : nullptr));
    if (h_new) LT_TRY(md_energy(h, b, beta, rho, n_stout, h_new, &cv));
    return LT_OK;
}

int lt_md_trajectory(lt_lattice* h, lt_bias* bias, int integrator, double beta, double tau, int n_step, double rho,
                     int n_stout, uint64_t seed, uint64_t* counter, int metropolis, double* dH, int* accepted,
                     double* cv_out)
{
    LT_TRY(check_h(h, "lt_md_trajectory"));
    const lt::DeviceScope device_scope(h->device);
    if (!counter) return lt::set_error(LT_ERR_ARG, "lt_md_trajectory: null counter");
    if (bias && n_stout < 0) return lt::set_error(LT_ERR_ARG, "lt_md_trajectory: n_stout < 0");
    LT_TRY(md_check(integrator, bias != nullptr, "lt_md_trajectory"));
    auto* b = reinterpret_cast<lt::Bias*>(bias);
    LT_TRY(ensure(h, &h->Ubak, h->be->gauge_bytes(h->g)));
    LT_CK(cudaMemcpyAsync(h->Ubak, h->U, h->be->gauge_bytes(h->g), cudaMemcpyDeviceToDevice, h->stream));
    LT_TRY(lt_random_momenta(h, seed, *counter));
    double cv_old = 0.0, cv_new = 0.0, e_old, e_new;
    LT_TRY(md_energy(h, b, beta, rho, n_stout, &e_old, &cv_old));
    std::vector<double> samples;
    samples.reserve((size_t)n_step);
    std::vector<MdOp> ops;
    md_program(integrator, tau, n_step, ops);
    MetaDParams md { b, rho, n_stout, &samples };
    LT_TRY(integrate(h, beta, ops, b ? &md : nullptr));
    LT_TRY(md_energy(h, b, beta, rho, n_stout, &e_new, &cv_new));
    const double d = e_new - e_old;
    bool acc = true;
    if (metropolis)
    {
        acc = accept_uniform(seed, *counter) <= std::exp(-d);
        if (!acc) LT_CK(cudaMemcpyAsync(h->U, h->Ubak, h->be->gauge_bytes(h->g), cudaMemcpyDeviceToDevice, h->stream));
    }
    if (b)
    {
        // the visited CVs (or, for the multiple-timescale integrators, which record none, the
        // final CV) are deposited symmetrically; a rejected trajectory deposits CV_old
        // (updates/hmc_metadynamics.hpp:583-626)
        b->cv_current = acc ? cv_new : cv_old;
        if (samples.empty()) samples.push_back(b->cv_current);
        if (!acc)
            for (double& s : samples) s = cv_old;
        for (double s : samples)
        {
            b->update(s);
            b->update(-s);
        }
    }
    ++*counter;
    LT_CK(cudaStreamSynchronize(h->stream));
    if (dH) *dH = d;
    if (accepted) *accepted = acc ? 1 : 0;
    if (cv_out) *cv_out = b ? b->cv_current : 0.0;
    if (!std::isfinite(d)) return lt::set_error(LT_ERR_NUMERIC, "lt_md_trajectory: non-finite dH");
    return LT_OK;
}

} // extern "C"
