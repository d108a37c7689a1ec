/*
 * lettuce_b200 -- C ABI of the B200-native pure-gauge SU(3) hot path.
 *
 * Drop-in boundary for the CPU reference timo-eichhorn/Lettuce (header-only C++20).  The
 * reference has no FFI of its own; each entry point below replaces the reference
 * function, functor or container member named beside it (paths relative to the
 * reference project root).  Plain C types only: opaque handles, plain pointers and sizes,
 * int status codes, no exceptions across the boundary.
 *
 * Link and algebra fields cross the boundary in the reference layout
 * double[V][4][3][3][2]: site index ((t*Nx + x)*Ny + y)*Nz + z, direction mu fastest,
 * row-major 3x3, real/imaginary interleaved (LettuceGauge/lattice.hpp:366-382).
 *
 * Threading: every lattice handle owns one CUDA stream on the device that was current when
 * it was created; each call runs on that device and restores the caller's current device.
 * Calls on one handle are serialised by the caller; distinct handles may be driven from
 * distinct host threads.  Calls that return a host value synchronise the handle's stream.
 * No device wait in this library spins without a bound.
 */
#ifndef LETTUCE_B200_H
#define LETTUCE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define LT_OK          0
#define LT_ERR_ARG     1   /* invalid argument: null pointer, odd extent, mismatched handles */
#define LT_ERR_CUDA    2   /* CUDA runtime error (no device, launch failure, ...)            */
#define LT_ERR_NOMEM   3   /* device or host allocation failed                                */
#define LT_ERR_STATE   4   /* operation not valid in the handle's current state              */
#define LT_ERR_NUMERIC 5   /* non-finite value detected in a result                          */
#define LT_ERR_IO      6   /* file cannot be opened, read or written, or has a malformed header */
#define LT_ERR_TIMEOUT 7   /* a bounded device-side wait gave up (the result is not valid)     */

/* Storage format of the link field. */
#define LT_PREC_FP64    0  /* 18 doubles per link (the reference's Matrix_SU3, defines.hpp:122)   */
#define LT_PREC_FP32    1  /* 18 floats per link                                                  */
#define LT_PREC_FP32_12 2  /* 12 floats per link; third row rebuilt by RestoreLastRow
                              (math/su3.hpp:362-367)                                              */

typedef struct lt_lattice lt_lattice;
typedef struct lt_bias lt_bias;

/* Message of the last failing call on this host thread ("" if none). */
const char* lt_last_error(void);
/* Library version, major*10000 + minor*100 + patch. */
int lt_version(void);

/* ---- gauge field container: GaugeField4D (lattice.hpp:87-394) ---------------------- */
/* Constructor; ext = {Nt, Nx, Ny, Nz}, all even and >= 2 (iterators/iterators.hpp:68).
 * Links start as the unit matrix. */
int lt_create(const int ext[4], int prec, lt_lattice** out);
/* Destructor. */
int lt_destroy(lt_lattice* h);
int lt_get_extents(const lt_lattice* h, int ext[4], int* prec);
/* Copy links from / to host memory in the reference layout (GaugeField4D element access,
 * lattice.hpp:113-136). */
int lt_upload_links(lt_lattice* h, const double* links);
int lt_download_links(lt_lattice* h, double* links);
/* The bytes the next lt_upload_links(h, links) copies host to device (no counterpart in the
 * reference): the FP64 field, or for a two-row FP32 handle uploaded before the packed field,
 * with a share of the sites as FP64 when links is pinned host memory. */
int lt_upload_bytes(const lt_lattice* h, const double* links, uint64_t* h2d_bytes);
/* One link: GaugeField4D::operator()(link_coord) (lattice.hpp:113-136); site index as in
 * the reference layout, m = 18 doubles (row-major 3x3, re/im interleaved). */
int lt_set_link(lt_lattice* h, int64_t site, int mu, const double* m);
int lt_get_link(lt_lattice* h, int64_t site, int mu, double* m_out);
/* Device-side copy dst = src (GaugeField4D::operator=, lattice.hpp:106-112); same extents,
 * any storage formats. */
int lt_copy(lt_lattice* dst, const lt_lattice* src);
/* Exchange the link storage of two handles with identical extents and format
 * (Swap, lattice.hpp:238-246). */
int lt_swap(lt_lattice* a, lt_lattice* b);
/* SetToIdentity (lattice.hpp:138-150). */
int lt_set_identity(lt_lattice* h);
/* Seeded Haar-random SU(3) start (the reference has none: SU3_main.cpp:296 starts cold).
 * Host-only generator; no device needed. */
int lt_haar_links(const int ext[4], uint64_t seed, double* links_out);
/* lt_haar_links + lt_upload_links. */
int lt_set_haar_random(lt_lattice* h, uint64_t seed);
/* Block the calling thread until the handle's stream is idle. */
int lt_synchronize(lt_lattice* h);
/* The handle's CUDA stream (a cudaStream_t), for callers that time or order work on it. */
int lt_get_stream(const lt_lattice* h, void** stream_out);

/* ---- status word ----------------------------------------------------------------------- */
/* No counterpart in the reference, which has no error channel (its kernels are noexcept and
 * the heatbath silently falls back to the unit matrix, updates/heatbath.hpp:72-76).  Each
 * handle keeps a device status word; kernels set bits, the host reads them here. */
#define LT_STATUS_NONFINITE 1u /* a link holds NaN or Inf (set by lt_check_links) */
#define LT_STATUS_UNITARITY 2u /* a link has an entry of |U U^dag - 1| above 1e-4 (FP32) or 1e-10 (FP64) */
#define LT_STATUS_HB_CAP 4u    /* a heatbath subgroup update hit the 10-retry cap and took the unit matrix */
#define LT_STATUS_BARRIER_TIMEOUT 8u /* a grid barrier of a persistent ensemble round gave up waiting */
/* Reads the status word (synchronising the handle's stream); clear = 1 resets it to 0. */
int lt_status_word(lt_lattice* h, uint32_t* word, int clear);
/* Scans every link, sets LT_STATUS_NONFINITE / LT_STATUS_UNITARITY, and returns the largest
 * entry of |U U^dag - 1| over the lattice (for FP32 storage: the reunitarisation error left
 * by the Gram-Schmidt projection after every update). */
int lt_check_links(lt_lattice* h, double* max_dev);

/* ---- configuration files: the BMW format (IO/config_io/bmw_format.hpp) ------------------ */
/* full = 0: "#BMW" files with the first two rows of each link; full = 1: "#18BMW" files with
 * all three rows.  A 4096-byte ASCII header "#BMW Nx Ny Nz Nt <checksum>" is followed by the
 * links in t, z, y, x order, directions x, y, z, t, as big-endian doubles; the checksum is
 * Checksum_Adler64 (:63-118) of the link data.  The device packs the records and computes the
 * checksum; the host writes the bytes. */
/* SaveConfigBMW / SaveConfigBMWFull (:294-394, :564-645).  Fails with LT_ERR_IO when the file
 * exists and overwrite = 0 (the reference returns false).  checksum_hex (17 bytes, may be
 * NULL) receives the header's checksum string. */
int lt_save_bmw(lt_lattice* h, const char* path, int full, int overwrite, char* checksum_hex);
/* LoadConfigBMW / LoadConfigBMWFull (:153-290, :425-560): reads the links (two-row files get
 * their third row from RestoreLastRow, su3.hpp:362-367, in the reference's rounding).
 * *checksum_ok = 1 when the recomputed checksum string equals the header's (the reference
 * only prints the comparison); *in_group = 1 when every link passes SU3::Tests::IsGroupElement
 * (su3.hpp:568-595, tolerance 1e-6), the reference's return value.  LT_ERR_IO for a missing
 * file, a malformed header or a short file; LT_ERR_ARG when the shape differs from the handle's. */
int lt_load_bmw(lt_lattice* h, const char* path, int full, int* checksum_ok, int* in_group);
/* Checksum_Adler64 of the handle's links as a BMW file would hold them, without file IO.
 * No counterpart in the reference (which computes it only inside save and load). */
int lt_bmw_checksum(lt_lattice* h, int full, uint64_t* checksum);

/* ---- observables --------------------------------------------------------------------- */
/* PlaquetteSum (observables/plaquette.hpp:26-43): sum over sites, mu<nu of ReTr P. */
int lt_plaquette_sum(lt_lattice* h, double* out);
/* WilsonAction::Action / Rectangular<1>::Action (actions/gauge/wilson_action.hpp:24-41,
 * rectangular_action.hpp:61-94): beta (6V - sum ReTr P / 3). */
int lt_wilson_action(lt_lattice* h, double beta, double* out);
/* TopChargeClover (observables/topological_charge.hpp:97-200). */
int lt_topcharge_clover(lt_lattice* h, double* out);
/* EnergyDensity::Clover on the traceless clover field strength
 * (observables/field_strength_tensor.hpp:28-66, :107-134, :154-175). */
int lt_energy_clover(lt_lattice* h, double* out);
/* Both of the above from one pass over the clover leaves. */
int lt_clover_observables(lt_lattice* h, double* q_out, double* e_out);
/* The measurement bundle of the reference driver (SU3_main.cpp:89-235).
 * TopChargeCloverTimeslice and EnergyDensity::CloverTimeslice (topological_charge.hpp:338-364,
 * field_strength_tensor.hpp:178-195) for every t = 0..Nt-1 (each array Nt doubles; either may
 * be NULL); the timeslices sum to lt_topcharge_clover / lt_energy_clover. */
int lt_clover_timeslices(lt_lattice* h, double* q_t, double* e_t);
/* TopChargePlaquette (topological_charge.hpp:366-416). */
int lt_topcharge_plaquette(lt_lattice* h, double* out);
/* GaugeAction::Rectangular<2>::Action (actions/gauge/rectangular_action.hpp:61-94) with
 * coefficients c_plaq, c_rect (the driver's Symanzik action: 5/3, -1/12); divide by 6 beta V
 * for ActionNormalized. */
int lt_rect_action(lt_lattice* h, double beta, double c_plaq, double c_rect, double* out);
/* WilsonLoop (observables/wilson_loop.hpp:63-124): 1 - sum Re tr W_LxL / (18 V) over all sites
 * and the six planes, for square L x L loops (the driver measures L = 2, 4, 8). */
int lt_wilson_loop(lt_lattice* h, int L, double* out);
/* WilsonLoop<start, end, reset>(U, U_chain) (observables/wilson_loop.hpp:63-124) with the
 * chain U_chain kept in the handle between calls: reset sets it to 1, then the links
 * U(x + n mu) for n = start..end-1 are multiplied on, and the square loops of side `end` are
 * evaluated from it.  The driver's sequence (0, 2, reset), (2, 4), (4, 8) builds each chain
 * once (a straight run from the origin doubles with one product per link).  Without reset
 * the previous call's chain is extended as it stands; LT_ERR_STATE if there is none
 * (lt_wilson_loop reuses the chain's buffers and drops it). */
int lt_wilson_loop_chain(lt_lattice* h, int start, int end, int reset, double* out);
/* PolyakovLoop (observables/polyakov_loop.hpp:32-49): mean over the spatial sites of the trace
 * of the product of the links in direction t. */
int lt_polyakov_loop(lt_lattice* h, double* re, double* im);
/* CalculateClover<1, 1> (observables/clover.hpp:94-152): the clover field of the handle's
 * links as a FullTensor4D (lattice.hpp:447-590) in its layout double[V][4][4][3][3][2]
 * (index ((site * 4 + mu) * 4 + nu)), FP64 products whatever the storage.  The tensor is kept
 * in device memory with the handle (16 V 3x3 complex: 2304 bytes per site) and copied to
 * tensor_out unless that is NULL. */
int lt_clover_tensor(lt_lattice* h, double* tensor_out);
/* TopChargeClover(const FullTensor&) (observables/topological_charge.hpp:202-231): Q of the
 * tensor `tensor` (host memory, the layout above, the handle's extents), or of the tensor the
 * handle keeps from lt_clover_tensor when tensor is NULL. */
int lt_topcharge_clover_tensor(lt_lattice* h, const double* tensor, double* q_out);
/* WilsonAction::Staple for every link (rectangular_action.hpp:104-184), reference layout. */
int lt_staples(lt_lattice* h, double* staples_out);
/* Plaquette sum of a field that the caller already holds in device memory, in the reference
 * layout double[V][4][3][3][2], written as one double to the caller's device pointer
 * out_dev, on the caller's stream (NULL = default stream).  No counterpart in the reference:
 * this entry point exists for callers that may not allocate device memory -- frameworks whose
 * memory pool owns all device memory (a raw cudaMalloc escapes its accounting), and timing or
 * monitoring loops that cudaMalloc/cudaFree would stall by synchronising the device.  It
 * allocates nothing: its scratch is a fixed 128 KiB static device array (present on every
 * GPU that loads the library), so volumes above 16,777,216 sites (64^4) are rejected with
 * LT_ERR_ARG.  The first call on a device looks up that array's address (make it before
 * any stream capture).  All calls share the array: calls that overlap on the GPU race. */
int lt_plaquette_sum_noalloc(const double* links_dev, const int ext[4], double* out_dev, void* stream);

/* ---- gauge action: GaugeAction::Rectangular (actions/gauge/rectangular_action.hpp) ------ */
/* The handle's simulated action, used by lt_staples, the sweeps, the HMC force and
 * Hamiltonian (lt_gauge_force, lt_hamiltonian, lt_omf2, lt_md_*, lt_hmc_trajectory and the
 * MetaD variants) and the gradient flow (lt_flow*, lt_flow_t0).  stencil_radius 1:
 * Rectangular<1>, whose staple is the plaquette staple and whose action is
 * beta c_plaq (6V - sum ReTr P / 3) (the default, (1, 1.0, 0.0), is WilsonAction);
 * 2: Rectangular<2>, staple c_plaq StaplePlaq + c_rect StapleRect (:187-246), action
 * beta (c_plaq (6V - ReTr P/3) + c_rect (12V - ReTr R/3)).  The reference's named
 * actions: LuescherWeisz (2, 1 + 8/12, -1/12), Iwasaki (2, 1 + 8 * 0.331, -0.331), DBW2
 * (2, 1 + 8 * 1.4088, -1.4088) (:273-276).  Radius 2 needs the Checkerboard4 sweeps. */
int lt_set_gauge_action(lt_lattice* h, int stencil_radius, double c_plaq, double c_rect);
int lt_get_gauge_action(lt_lattice* h, int* stencil_radius, double* c_plaq, double* c_rect);

/* ---- local updates: Iterator::Checkerboard (iterators/iterators.hpp:65-87) ------------- */
/* n_sweep sweeps of OverrelaxationSubgroupKernel (updates/overrelaxation.hpp:68-117). */
int lt_overrelax_sweeps(lt_lattice* h, int n_sweep);
/* n_sweep sweeps of HeatbathKernel (updates/heatbath.hpp:30-130) at coupling beta.
 * Random numbers: Philox4x32-10 keyed by seed, one counter value per sweep starting at
 * *counter; *counter is advanced by n_sweep. */
int lt_heatbath_sweeps(lt_lattice* h, double beta, int n_sweep, uint64_t seed, uint64_t* counter);
/* n_sweep rounds of (n_hb heatbath + n_or overrelaxation) sweeps, as the driver's update
 * loop (SU3_main.cpp:381-402); 8 chained launches per sweep on the handle's stream. */
int lt_update_sweeps(lt_lattice* h, double beta, int n_sweep, int n_hb, int n_or, uint64_t seed,
                     uint64_t* counter);
/* The Wilson-action sweeps above refuse a radius-2 action (LT_ERR_ARG): the rectangle staple
 * reaches links that a two-colour checkerboard updates together. */

/* ---- local updates: Iterator::Checkerboard4 (iterators/iterators.hpp:141-166) ----------- */
/* The same sweeps over Checkerboard4: per direction mu four sublattices
 * (t + x + y + z + x_mu) mod 4 = 0..3, one launch each (16 per sweep), with the handle's
 * action; every extent a multiple of 4 (else LT_ERR_ARG, where the reference exits).  The
 * reference driver runs these with every action (SU3_main.cpp:361-362, :594-595). */
int lt_overrelax_sweeps4(lt_lattice* h, int n_sweep);
int lt_heatbath_sweeps4(lt_lattice* h, double beta, int n_sweep, uint64_t seed, uint64_t* counter);
int lt_update_sweeps4(lt_lattice* h, double beta, int n_sweep, int n_hb, int n_or, uint64_t seed,
                      uint64_t* counter);

/* ---- ensembles: independent chains and tempering streams ------------------------------ */
typedef struct lt_ensemble lt_ensemble;
/* n lattices (any even extents, one storage format) advanced together, lattice k at
 * coupling betas[k] with the heatbath stream keyed seed + k.  The reference runs one lattice
 * per process; this packs many into each launch (see lt_ensemble_sweeps). */
int lt_ensemble_create(lt_lattice* const* lattices, const double* betas, int n, uint64_t seed, lt_ensemble** out);
int lt_ensemble_destroy(lt_ensemble* e);
/* n_sweep rounds of (n_hb heatbath + n_or overrelaxation) sweeps on every lattice, one
 * launch per (mu, parity) sub-sweep covering all lattices, the round captured once as a
 * CUDA graph and replayed.  reverse != 0 runs the round's sub-sweeps in reverse order (for
 * a reversible mixture of both orders).  *counter advances by n_sweep * n_hb as in
 * lt_heatbath_sweeps. */
int lt_ensemble_sweeps(lt_ensemble* e, int n_sweep, int n_hb, int n_or, int reverse, uint64_t* counter);
/* Time 64-, 128- and 256-thread blocks for the batched heatbath and overrelaxation on a
 * scratch copy of the links (the chains are not advanced) and keep the fastest. */
int lt_ensemble_autotune(lt_ensemble* e, int* threads_hb, int* threads_or);
/* Fix the block sizes (64, 128 or 256 threads). */
int lt_ensemble_set_block(lt_ensemble* e, int threads_hb, int threads_or);
/* How a round runs (lt_ensemble_autotune picks the faster, with its residency):
 *   LT_ENSEMBLE_GRAPH       one batched launch per (mu, parity) sub-sweep, the round captured
 *                           as a CUDA graph and replayed (the default);
 *   LT_ENSEMBLE_PERSISTENT  one cooperative launch per round: every block resident, the
 *                           sub-sweeps separated by grid barriers whose waits are bounded (a
 *                           barrier that gives up makes lt_ensemble_sweeps return
 *                           LT_ERR_TIMEOUT), blocks_per_sm blocks per SM (0: the occupancy
 *                           limit).
 * The reference runs each sub-sweep as an OpenMP loop with its implicit barrier
 * (iterators.hpp:65-87); the rounds advance every lattice identically in both modes. */
#define LT_ENSEMBLE_GRAPH      0
#define LT_ENSEMBLE_PERSISTENT 1
int lt_ensemble_set_mode(lt_ensemble* e, int mode, int blocks_per_sm);
int lt_ensemble_get_mode(lt_ensemble* e, int* mode, int* blocks_per_sm);
/* The wait bound of the persistent round's grid barriers, in polls of about 100 ns (default
 * 10,000,000: about a second). */
int lt_ensemble_set_barrier_polls(lt_ensemble* e, long long polls);
/* Tempering exchange between streams a and b sampling exp(-S - scale V(Q)) with CVs q_a, q_b
 * (generalises MetadynamicsTemperingKernel::operator(), updates/tempering.hpp:51-72):
 * accepted when u <= exp(-dE), dE = (scale_a - scale_b)(V(q_b) - V(q_a)); on acceptance the
 * link storage of a and b is swapped (lt_swap). */
int lt_tempering_swap(lt_lattice* a, lt_lattice* b, const lt_bias* bias, double scale_a, double scale_b, double q_a,
                      double q_b, double u, int* accepted, double* dE_out);

/* ---- smearing ------------------------------------------------------------------------ */
/* Integrators::GradientFlow (smearing/gradient_flow.hpp:31-168) */
#define LT_FLOW_EULER 0  /* Euler (:31-56), the smoothing of the reference's measurement step */
#define LT_FLOW_RK2   1  /* RK2 (:88-113) */
#define LT_FLOW_RK3   2  /* RK3 (:114-140), Luscher's third-order scheme */
#define LT_FLOW_RK3W7 3  /* RK3W7 (:142-168) */
/* GradientFlowKernel (:252-367) with any of the integrators: out = in flowed by n_step steps
 * of size eps (in == out continues a flow, as GradientFlowKernel::Resume). */
int lt_flow(lt_lattice* in, lt_lattice* out, int integrator, double eps, int n_step);
/* The force of the flows run into a handle (lt_flow, lt_flow_rk3, lt_flow_rk3_measure,
 * lt_flow_t0 with that handle as `out`):
 *   LT_FLOW_ACTION_GAUGE   Z = Algebra(st U^dag) of the handle's gauge action, the reference's
 *                          GradientFlowKernel<IntegratorT, ActionT> (:298-332); the default;
 *   LT_FLOW_ACTION_ZEUTHEN the Zeuthen flow (Ramos and Sint, arXiv:1508.05552): the
 *                          Luescher-Weisz force X acted on by 1 + 1/12 nabla*_mu nabla_mu,
 *                          F_mu(x) = X_mu(x) + [U_mu(x) X_mu(x+mu) U_mu(x)^dag
 *                          + U_mu(x-mu)^dag X_mu(x-mu) U_mu(x-mu) - 2 X_mu(x)] / 12.
 * No counterpart in the reference (it has no Zeuthen flow). */
#define LT_FLOW_ACTION_GAUGE   0
#define LT_FLOW_ACTION_ZEUTHEN 1
int lt_set_flow_action(lt_lattice* h, int flow_action);
int lt_get_flow_action(lt_lattice* h, int* flow_action);
/* GradientFlowKernel<RK3>::operator() (smearing/gradient_flow.hpp:120-168, :339-345):
 * out = in flowed by n_step RK3 steps of size eps.  in == out continues in place
 * (GradientFlowKernel::Resume, :347-351). */
int lt_flow_rk3(lt_lattice* in, lt_lattice* out, double eps, int n_step);
/* Flow with a measurement every `every` steps: plaquette sum, clover Q and clover energy
 * density after steps every, 2*every, ..., n_meas*every (SU3_main.cpp:150-163). */
int lt_flow_rk3_measure(lt_lattice* in, lt_lattice* out, double eps, int n_meas, int every,
                        double* plaq_out, double* q_out, double* e_out);
/* Scale setting: flow `in` into `out` (RK3, step eps) until t^2 E(t) reaches `target`
 * (0.3 defines t0), E the clover energy density measured after every step as the driver
 * measures it (SU3_main.cpp:128-141).  t0 is linearly interpolated between the two steps
 * around the crossing; q_out (may be NULL) receives Q at the last step taken.  Fails with
 * LT_ERR_STATE if the target is not reached within max_steps.  No counterpart in the
 * reference (it measures at fixed flow times only). */
int lt_flow_t0(lt_lattice* in, lt_lattice* out, double eps, double target, int max_steps, double* t0_out,
               double* q_out);
/* n steps of StoutSmearing4D (smearing/stout_smearing.hpp:29-57); in == out allowed. */
int lt_stout(lt_lattice* in, lt_lattice* out, double rho, int n);

/* ---- HMC: GaugeUpdates::HMCKernel (updates/hmc_gauge.hpp:381-600) ---------------------- */
/* beta/6 Algebra(st U^dag) for every link: the momentum kick of UpdateMomenta (:450-464). */
int lt_gauge_force(lt_lattice* h, double beta, double* force_out);
/* The handle's momentum field (full anti-Hermitian 3x3 per link, reference layout). */
int lt_set_momenta(lt_lattice* h, const double* p);
int lt_get_momenta(lt_lattice* h, double* p_out);
/* RandomMomentum (:400-428) from Philox Gaussians keyed by seed at `counter`. */
int lt_random_momenta(lt_lattice* h, uint64_t seed, uint64_t counter);
/* Hamiltonian (:525-541): Wilson action + (-sum ReTr P^2). */
int lt_hamiltonian(lt_lattice* h, double beta, double* out);
/* Integrators::HMC::OMF_2 (:155-190) molecular dynamics from the current links and momenta;
 * H before and after in h_old / h_new (either may be NULL). */
int lt_omf2(lt_lattice* h, double beta, double tau, int n_step, double* h_old, double* h_new);
/* HMCKernel::operator() (:549-583) with OMF_2: momenta, MD, Metropolis (if metropolis != 0)
 * from Philox streams at *counter (advanced by 1); dH and the decision are returned. */
int lt_hmc_trajectory(lt_lattice* h, double beta, double tau, int n_step, uint64_t seed, uint64_t* counter,
                      int metropolis, double* dH, int* accepted);

/* ---- metadynamics: HMCMetaDKernel (updates/hmc_metadynamics.hpp:264-675) ---------------- */
/* CloverDerivative for every link (observables/clover.hpp:279-321) on the handle's links. */
int lt_clover_derivative(lt_lattice* h, double* out);
/* MetaCharge (:302-310): clover Q after n_stout stout steps of parameter rho. */
int lt_metad_charge(lt_lattice* h, double rho, int n_stout, double* q_out);
/* CalculateTopologicalForce (:374-436): dvdq * dQ_stout/dU on the thin links through the
 * hand-written stout-chain adjoint (smearing/stout_smearing.hpp:122-234); the smeared levels
 * are kept, the exponential constants are recomputed.  force_out (may be NULL) in the
 * reference layout; q_out (may be NULL) receives the smeared charge. */
int lt_metad_force(lt_lattice* h, double rho, int n_stout, double dvdq, double* force_out, double* q_out);
/* OMF_2 molecular dynamics with the bias force (UpdateMomenta :441-459); H + V(Q) before/after. */
int lt_metad_omf2(lt_lattice* h, lt_bias* bias, double beta, double tau, int n_step, double rho, int n_stout,
                  double* h_old, double* h_new);
/* HMCMetaDKernel::operator() (:552-655): one MetaD-HMC trajectory, Metropolis, and the
 * symmetric well-tempered bias update from the path samples (:615-643). */
int lt_metad_hmc_trajectory(lt_lattice* h, lt_bias* bias, double beta, double tau, int n_step, double rho,
                            int n_stout, uint64_t seed, uint64_t* counter, int metropolis, double* dH,
                            int* accepted, double* cv_out);

/* ---- molecular-dynamics integrators (updates/hmc_gauge.hpp:19-377,
 *      updates/hmc_metadynamics.hpp:26-238) and parity (updates/parity_update.hpp:22-47) ---- */
#define LT_MD_LEAPFROG_SLOW          0   /* Integrators::HMC::Leapfrog_slow (hmc_gauge.hpp:21-44) */
#define LT_MD_LEAPFROG               1   /* Leapfrog (:47-70) */
#define LT_MD_OMF2_SLOW              2   /* OMF_2_slow (:121-151) */
#define LT_MD_OMF2                   3   /* OMF_2 (:155-190) */
#define LT_MD_OMF4_SLOW              4   /* OMF_4_slow (:195-237) */
#define LT_MD_OMF4                   5   /* OMF_4 (:241-294), the reference driver's choice */
#define LT_MD_LEAPFROG_FRICTION_SLOW 6   /* Leapfrog_friction_slow (:74-116), gauge action only */
#define LT_MD_OMF4_FRICTION_SLOW     7   /* OMF_4_friction_slow (:298-376), gauge action only */
#define LT_MD_LEAPFROG_OMF4          8   /* Leapfrog_OMF_4 (hmc_metadynamics.hpp:28-83), MetaD only */
#define LT_MD_OMF2_OMF4_SLOW         9   /* OMF_2_OMF_4_slow (:85-143), MetaD only */
#define LT_MD_OMF2_OMF4              10  /* OMF_2_OMF_4 (:145-237), MetaD only */
/* Molecular dynamics with any integrator from the current links and momenta, with the bias
 * force (bias != NULL: CV = clover Q after n_stout stout steps of rho) or the gauge action
 * alone; H (+ V(CV)) before and after in h_old / h_new (either may be NULL).  The
 * multiple-timescale integrators evaluate the bias force at the current links at each of
 * their Metadynamics momentum updates (the reference's UpdateMetadynamicsMomenta adds the
 * force it last stored). */
int lt_md_integrate(lt_lattice* h, lt_bias* bias, int integrator, double beta, double tau, int n_step, double rho,
                    int n_stout, double* h_old, double* h_new);
/* HMCKernel::operator() (hmc_gauge.hpp:549-583) or, with a bias, HMCMetaDKernel::operator()
 * (hmc_metadynamics.hpp:552-655) with any integrator: random momenta from Philox at
 * *counter (advanced by 1), MD, Metropolis (if metropolis != 0), and under MetaD the
 * symmetric bias update from the CVs recorded at the submeasurement kicks (the final CV for
 * the multiple-timescale integrators, which record none). */
int lt_md_trajectory(lt_lattice* h, lt_bias* bias, int integrator, double beta, double tau, int n_step, double rho,
                     int n_stout, uint64_t seed, uint64_t* counter, int metropolis, double* dH, int* accepted,
                     double* cv_out);
/* ReverseMomenta (hmc_gauge.hpp:432-446): P <- -P, for reversibility tests. */
int lt_reverse_momenta(lt_lattice* h);
/* ParityUpdate (parity_update.hpp:22-47): the spatial reflection that maps Q to -Q and leaves
 * the action unchanged, in place. */
int lt_parity_update(lt_lattice* h);

/* ---- diagnostics for tests (no counterpart in the reference) ---------------------------- */
#define LT_EXP_DISPATCH     0  /* the branch choice of the flow / stout / HMC kernels            */
#define LT_EXP_CLOSED       1  /* the closed form of ExpConstants (FP64 scalar chain)            */
#define LT_EXP_SERIES_SHORT 2  /* Cayley-Hamilton series, short term count (valid for c1 <= 1/32) */
#define LT_EXP_SERIES_LONG  3  /* Cayley-Hamilton series, long term count (valid for c1 <= 1/2)  */
#define LT_EXP_SERIES_TINY  4  /* Cayley-Hamilton series, tiny term count (valid for c1 <= 1/512) */
/* SU3::exp (math/su3_exp.hpp:419-432) on the device: out[k] = exp(i Q_k) for n traceless
 * Hermitian 3x3 matrices q_in[k] (18 doubles each, row-major, re/im interleaved; host
 * memory), computed in the arithmetic of storage format prec by the branch `path`
 * (LT_EXP_*).  Allocates and synchronises: a test entry point, not a hot path. */
int lt_su3_exp_test(const double* q_in, double* out, int n, int prec, int path);
/* binaryVersion and ptxVersion (cudaFuncGetAttributes) of the library's kernels on the
 * current device: 100 for code built for sm_100a. */
int lt_device_arch(int* binary_version, int* ptx_version);
/* The host packing of lt_upload_links for two-row FP32 storage, on the calling thread and
 * without a device: links (reference layout, V = ext[0] ext[1] ext[2] ext[3] sites) rounded to
 * FP32 and written to out (48 V floats, 16-byte aligned) in the device layout of the two-row
 * storage: chunk c (0..2) of plane (mu, parity) at ((mu * 2 + parity) * 3 + c) * V/2 float4s,
 * checkerboard index s = site / 2, floats 4c .. 4c + 3 of the link's rows 0-1. */
int lt_pack_links_test(const int ext[4], const double* links, float* out);

/* ---- bias potential: MetaBiasPotential (actions/bias_potential/metadynamics.hpp:29-507) -- */
/* Constructor (:60-91); fails with LT_ERR_ARG where the reference throws (:70-77). */
int lt_bias_create(double cv_min, double cv_max, int bin_number, double weight, double width,
                   double well_tempered_parameter, double threshold_weight, lt_bias** out);
int lt_bias_destroy(lt_bias* b);
/* UpdatePotential (:103-131) or UpdatePotentialSymmetric (:134-147) for n CV samples, with
 * the bias's deposit mode (lt_bias_set_update_mode).  The MetaD trajectories deposit through
 * the same mode. */
int lt_bias_update(lt_bias* b, const double* cv, int n, int symmetric);
#define LT_BIAS_GAUSSIAN 0  /* the reference's well-tempered Gaussian deposit (the default) */
#define LT_BIAS_BINNED   1  /* Gaussian-free binned deposit: the weight is split linearly between
                             * the two grid points bracketing the CV, each share well-tempered by
                             * exp(-V_point / well_tempered_parameter); CVs outside [cv_min,
                             * cv_max) deposit nothing and are counted as exceeded */
/* Selects the deposit of lt_bias_update and of the MetaD trajectories.  No counterpart in the
 * reference (its deposits are Gaussians, metadynamics.hpp:103-147). */
int lt_bias_set_update_mode(lt_bias* b, int mode);
int lt_bias_get_update_mode(const lt_bias* b, int* mode);
/* ReturnPotential (:151-179). */
int lt_bias_potential(const lt_bias* b, double cv, double* out);
/* ReturnDerivative (:181-187). */
int lt_bias_derivative(const lt_bias* b, double cv, double* out);
/* The bin_number+1 grid values (read / overwrite). */
int lt_bias_get_grid(const lt_bias* b, double* grid_out, int n);
int lt_bias_set_grid(lt_bias* b, const double* grid, int n);

#ifdef __cplusplus
}
#endif
#endif /* LETTUCE_B200_H */
