/* CPU restatement of the reference (timo-eichhorn/Lettuce) pure-gauge SU(3) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (lettuce_b200/, include/) never links, loads or
 * calls this code; tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py
 * use it as the checker.  Each function cites the reference file:line it follows.
 * Parity pinned against the reference itself: tests/test_oracle_pins.py compares every
 * function with the compiled reference harness (oracle/ref_harness.cpp) and with the
 * committed golden fixtures under tests/golden/.
 *
 * Layout of every field crossing this interface: the reference AoS layout
 * double[V][4][3][3][2] (lattice.hpp:366-382).  Lattice extents are runtime values
 * ext[4] = {Nt, Nx, Ny, Nz}, all even (iterators.hpp:68).
 */
#ifndef LT_ORACLE_H
#define LT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

double or_plaquette_sum(const int ext[4], const double* U);
double or_wilson_action(const int ext[4], const double* U, double beta);
void   or_staples(const int ext[4], const double* U, double* out);
void   or_overrelax_sweeps(const int ext[4], double* U, int n_sweep);
void   or_heatbath_sweeps(const int ext[4], double* U, double beta, int n_sweep,
                          uint64_t seed, uint64_t counter0);
void   or_su3_exp(const double* q_in, double* out, int n);
void   or_flow_rk3(const int ext[4], const double* in, double* out, double eps, int n_step);
void   or_stout(const int ext[4], const double* in, double* out, double rho, int n);
double or_topcharge_clover(const int ext[4], const double* U);
double or_energy_clover(const int ext[4], const double* U);
void   or_gauge_force(const int ext[4], const double* U, double beta, double* out);
void   or_clover_derivative(const int ext[4], const double* U, double* out);
double or_metad_force(const int ext[4], const double* U, double rho, int n_stout, double dvdq,
                      double* out);
double or_metad_charge(const int ext[4], const double* U, double rho, int n_stout);
void   or_omf2(const int ext[4], double* U, double* P, double beta, double tau, int n_step,
               double* h_old, double* h_new);
void   or_random_momenta(const int ext[4], double* P, uint64_t seed, uint64_t counter);
/* any of the eleven MD integrators (ids as LT_MD_* of the C ABI); metad: linear bias slope*Q */
void   or_md_integrate(const int ext[4], double* U, double* P, double beta, double tau, int n_step, int integrator,
                       int metad, double rho, int n_stout, double slope, double* h_old, double* h_new);
void   or_parity_update(const int ext[4], double* U);
/* gauge action of staples, sweeps, HMC forces / energies and the flow (default 1, 1, 0) */
void   or_set_gauge_action(int stencil_radius, double c_plaq, double c_rect);
void   or_overrelax_sweeps4(const int ext[4], double* U, int n_sweep);
void   or_heatbath_sweeps4(const int ext[4], double* U, double beta, int n_sweep, uint64_t seed, uint64_t counter0);
double or_kinetic(const int ext[4], const double* P);

/* MetaBiasPotential (metadynamics.hpp:29-187) */
typedef struct or_bias {
    double cv_min, cv_max, bin_width, bin_width_inv, weight, width, wt, thr;
    int    bins;
    double grid[1];   /* bins + 1 entries (allocated by or_bias_create) */
} or_bias;
or_bias* or_bias_create(double cv_min, double cv_max, int bins, double weight, double width,
                        double wt, double thr);
void     or_bias_destroy(or_bias* b);
void     or_bias_update(or_bias* b, double cv);
void     or_bias_update_symmetric(or_bias* b, double cv);
void     or_bias_update_binned(or_bias* b, double cv);
double   or_bias_potential(const or_bias* b, double cv);
double   or_bias_derivative(const or_bias* b, double cv);

/* Flow with any of the reference's integrators: 0 Euler, 1 RK2, 2 RK3, 3 RK3W7 */
void   or_flow(const int ext[4], const double* in, double* out, double eps, int n_step, int integrator);
/* The Zeuthen flow (not in the reference) with the same integrators */
void   or_flow_zeuthen(const int ext[4], const double* in, double* out, double eps, int n_step, int integrator);

/* The measurement bundle of SU3_main.cpp:89-235 */
void   or_clover_timeslices(const int ext[4], const double* U, double* q_t, double* e_t);
double or_topcharge_plaquette(const int ext[4], const double* U);
double or_rect_action(const int ext[4], const double* U, double beta, double c_plaq, double c_rect);
double or_wilson_loop(const int ext[4], const double* U, int L);
void   or_polyakov_loop(const int ext[4], const double* U, double* re, double* im);

/* BMW configuration payload and its Adler-64 checksum (IO/config_io/bmw_format.hpp:63-97,
 * :131-394, :406-645); full = 1 for the 18-real #18BMW variant.  encode writes the payload when
 * payload is not NULL; both return the checksum. */
uint64_t or_bmw_encode(const int ext[4], const double* U, int full, unsigned char* payload);
uint64_t or_bmw_decode(const int ext[4], const unsigned char* payload, int full, double* U);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) as used by the GPU streams */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

#ifdef __cplusplus
}
#endif
#endif
