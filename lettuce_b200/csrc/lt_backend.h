// Precision-independent interface between the C ABI (lt_capi.cu) and the kernels.  One
// implementation per storage format (FP64 18 reals, FP32 18 reals, FP32 12 reals) lives in
// its own translation unit so the three are compiled in parallel.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "lt_field.cuh"

namespace lt {

// Launch context: geometry, stream and the reduction scratch of one lattice handle.
struct Ctx
{
    Geom g;
    cudaStream_t stream;
    double* partials;   // kNumSlots * kRedBlocks doubles
    double* results;    // kNumSlots doubles
    unsigned* status = nullptr;   // the handle's device status word (LT_STATUS_* bits)
    // the handle's gauge action: Rectangular<2> (rect = 1: c_plaq StaplePlaq + c_rect StapleRect)
    // or Rectangular<1> (rect = 0: the plaquette staple)
    int rect = 0;
    double cp = 1.0, cr = 0.0;
    unsigned* order = nullptr;    // the handle's launch counter for alternating site orders
};

constexpr int kNumSlots = 8;

class Backend
{
public:
    virtual ~Backend() = default;
    virtual int real_bytes() const = 0;                     // 8 (FP64) or 4 (FP32)
    virtual size_t gauge_bytes(const Geom& g) const = 0;     // one link field
    virtual size_t alg_bytes(const Geom& g) const = 0;       // one algebra field (8 reals/link)
    virtual size_t full_bytes(const Geom& g) const = 0;      // one 3x3 complex per link
    virtual size_t clov_bytes(const Geom& g) const = 0;      // six anti-Hermitian planes per site

    virtual void from_aos(const Ctx& c, void* U, const double* aos) const = 0;
    // sites [i0, i1) only (reference site order; aos is the whole field's base)
    virtual void from_aos_sites(const Ctx& c, void* U, const double* aos, long long i0, long long i1) const = 0;
    virtual void to_aos(const Ctx& c, const void* U, double* aos) const = 0;
    virtual void alg_from_aos(const Ctx& c, void* P, const double* aos) const = 0;
    virtual void alg_to_aos(const Ctx& c, const void* P, double* aos) const = 0;
    virtual void set_unit(const Ctx& c, void* U) const = 0;
    // single link (site = reference site index) from / to 18 doubles in device memory
    virtual void link_io(const Ctx& c, void* U, int site, int mu, double* m, int write) const = 0;
    virtual void staples_aos(const Ctx& c, const void* U, double* aos) const = 0;

    // reductions write ctx.results[slot] (and slot+1 for clover_obs: q then e)
    virtual void plaquette(const Ctx& c, const void* U, int slot) const = 0;
    virtual void clover_obs(const Ctx& c, const void* U, int slot) const = 0;
    virtual void kinetic(const Ctx& c, const void* P, int slot) const = 0;

    // link health: sets kStatusNonFinite / kStatusUnitarity (tolerance tol) in c.status and
    // atomically maxes the float bits of the largest |U U^dag - 1| entry into *maxbits
    virtual void check_links(const Ctx& c, const void* U, double tol, unsigned* maxbits) const = 0;

    // measurement bundle (SU3_main.cpp:89-235): clover densities per timeslice into partials
    // (q then e, nbx blocks per timeslice); plaquette, rectangle and plaquette-charge sums into
    // results[slot..slot+2]; Polyakov loop re, im into results[slot..slot+1]; straight-line
    // products of the links (full FP64 matrices) for square Wilson loops
    virtual void clover_timeslices(const Ctx& c, const void* U, double* partials, int nbx) const = 0;
    virtual void loops(const Ctx& c, const void* U, int slot) const = 0;
    virtual void polyakov(const Ctx& c, const void* U, int slot) const = 0;
    virtual void chain_init(const Ctx& c, const void* U, void* C) const = 0;
    virtual void chain_unit(const Ctx& c, void* C) const = 0;
    virtual void chain_extend(const Ctx& c, const void* Cin, const void* U, void* Cout, int L) const = 0;
    virtual void chain_double(const Ctx& c, const void* Cin, void* Cout, int L) const = 0;
    virtual void wilson_square(const Ctx& c, const void* C, int L, int slot) const = 0;

    // BMW payload (full: 18 reals per link, else 12) to / from device memory; Adler-64 partial
    // sums (A then B, kRedBlocks each) into partials; unpack sets bit 0 of *flags for a link
    // that fails the reference's group-element test
    virtual void bmw_pack(const Ctx& c, const void* U, int full, void* out, unsigned long long* partials) const = 0;
    virtual void bmw_unpack(const Ctx& c, void* U, int full, const void* in, unsigned long long* partials,
                            unsigned* flags) const = 0;

    virtual void overrelax(const Ctx& c, void* U, int mu, int par) const = 0;
    // one (mu, sublattice) sub-sweep of Iterator::Checkerboard4 with the context's action:
    // heatbath (op 0, Philox counter/seed as heatbath()) or overrelaxation (op 1)
    virtual void sweep4(const Ctx& c, void* U, int op, int mu, int sub, double prefactor, uint64_t counter,
                        uint64_t seed, int max_iter) const = 0;
    virtual void heatbath(const Ctx& c, void* U, int mu, int par, double prefactor, uint64_t counter,
                          uint64_t seed, int max_iter) const = 0;
    // flow_split(): the format runs a flow stage as two kernels and wants an algebra scratch
    // field X (flow_stage's last argument; null: the fused stage)
    virtual bool flow_split() const = 0;
    virtual void flow_stage(const Ctx& c, const void* Uin, void* Uout, void* Z, double c_old, double c_new,
                            double c_exp, int read_z, int write_z, void* X) const = 0;
    // st_out (may be null): the staple of every link, one full 3x3 per link
    virtual void stout(const Ctx& c, const void* Uin, void* Uout, double rho, void* st_out) const = 0;
    // Zeuthen flow stage: X <- the Luescher-Weisz force (c_plaq cp, c_rect cr) of Uin, then the
    // Zeuthen force from X and the stage's Z and link update Uin -> Uout
    virtual void flow_zeuthen_stage(const Ctx& c, const void* Uin, void* Uout, void* Z, void* X, double c_old,
                                    double c_new, double c_exp, int read_z, int write_z, double cp,
                                    double cr) const = 0;

    virtual void momenta(const Ctx& c, const void* U, void* P, const void* F, double coef, double eps) const = 0;
    virtual void fields(const Ctx& c, void* U, const void* P, double eps) const = 0;
    virtual void random_momenta(const Ctx& c, void* P, uint64_t counter, uint64_t seed) const = 0;
    // P <- a P + b F on algebra fields (F may be null); the spatial parity reflection Uin -> Uout
    virtual void alg_axpby(const Ctx& c, void* P, const void* F, double a, double b) const = 0;
    virtual void parity(const Ctx& c, const void* Uin, void* Uout) const = 0;

    // One (mu, parity) sub-sweep of heatbath (op 0) or overrelaxation (op 1) over a batch of
    // lattices described by the device array desc (LatDesc[n_lat]); sel picks 64/128/256
    // threads per block and n_blocks is the batch's block count for that size.
    virtual void batch_sweep(cudaStream_t s, const void* desc, int n_lat, int n_blocks, int sel, int op, int mu,
                             int par, const uint64_t* counter, int max_iter, int flip) const = 0;

    // FullTensor4D of CalculateClover<1, 1> in the reference layout (FP64, device memory,
    // zeroed by the caller); Q sum of a tensor into results[slot] (unnormalised)
    virtual void clover_tensor(const Ctx& c, const void* U, double* tensor) const = 0;
    virtual void topcharge_tensor(const Ctx& c, const double* tensor, int slot) const = 0;
    // One persistent cooperative launch of a whole round (n_hb heatbath + n_or overrelaxation
    // sweeps) over a batch of lattices (blocks of 128 threads: n_units = the batch's block
    // count), blocks_per_sm blocks resident per SM; bar = {count, gen, status} words for the
    // bounded grid barrier (count zero at launch) followed by one work-unit counter per
    // sub-sweep from bar[4] on (8 (n_hb + n_or) words, zeroed here), polls = its wait bound.
    // Returns the launch status.  max_blocks_per_sm: the occupancy limit of that kernel.
    virtual cudaError_t batch_round(cudaStream_t s, const void* desc, int n_lat, int n_units, int blocks_per_sm,
                                    int n_hb, int n_or, int reverse, uint64_t* counter, int max_iter, unsigned* bar,
                                    long long polls) const = 0;
    virtual int batch_round_max_blocks_per_sm() const = 0;
    virtual void clover_R(const Ctx& c, const void* U, void* R) const = 0;
    // sum over sites of ReTr(R01 R23 - R02 R13 + R03 R12) into results[slot]
    virtual void topcharge_R(const Ctx& c, const void* R, int slot) const = 0;
    virtual void clover_deriv(const Ctx& c, const void* U, const void* R, void* out, double scale) const = 0;
    virtual void stout_lambda(const Ctx& c, const void* U, const void* Up, const void* Sigma, void* Lam,
                              void* Tloc, double rho, const void* st_in) const = 0;
    virtual void stout_recursion(const Ctx& c, const void* U, const void* Lam, const void* Tloc, void* Sigma,
                                 double rho) const = 0;
};

const Backend* backend_fp64();
const Backend* backend_fp32();
const Backend* backend_fp32_12();

} // namespace lt
