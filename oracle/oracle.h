/*
 * ORACLE (test infrastructure only).  CPU restatement of the reference's MP
 * tracking path, used by tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg as the checker.  Never linked into libcetagpu.so.
 *
 * Parity status: the reference's tracking sources need GSL and FFTW, which
 * are absent here, so they cannot be compiled; this restatement of them is
 * therefore "parity unpinned" except for w(z), which is pinned against the
 * reference's own compiled Faddeeva.cpp and its known-answer test.
 */
#ifndef CETASIM_ORACLE_H
#define CETASIM_ORACLE_H
#include <stdint.h>
#include "../include/cetasim_gpu.h"

typedef struct or_state or_state;

void or_faddeeva_w(const double* zr, const double* zi, double* wr, double* wi, int64_t n);
void or_w_fast(double x, double y, double* wr, double* wi);
void or_w_fast_arr(const double* zr, const double* zi, double* wr, double* wi, int64_t n);
void or_gaussian_field(const double* x, const double* y, const double* sx, const double* sy,
                       double* fx, double* fy, int64_t n);
int or_config_derive(cg_config* cfg);
int or_lattice_init(const cg_ring* ring, cg_section* sec, int n);

or_state* or_create(const cg_config* cfg, int n_bunches, const int* n_macro,
                    const int* bunch_harm, const double* n_electrons);
void or_destroy(or_state* s);
const char* or_last_error(or_state* s);
int or_set_bunch(or_state* s, int j, const double* x, const double* px, const double* y,
                 const double* py, const double* z, const double* dp, const uint8_t* surv);
int or_get_bunch(or_state* s, int j, double* x, double* px, double* y, double* py,
                 double* z, double* dp, uint8_t* surv);
int or_beam_rms(or_state* s, int k);
int or_get_moments(or_state* s, cg_bunch_moments* out);
int or_beam_ion_ip(or_state* s, int turn, int k);
int or_section_map(or_state* s, int k);
int or_rf_kick(or_state* s);
int or_resonator_state(or_state* s, int c, double* out);
int or_resonator_set(or_state* s, int c, const double* in);
int or_rf_info(or_state* s, int j, int c, double* out);
int or_longi_drift(or_state* s);
int or_energy_loss(or_state* s);
int or_synrad(or_state* s, int turn);
int or_lr_wake(or_state* s);
int or_sr_wake(or_state* s, int turn);
int or_bbi(or_state* s);
int or_space_charge(or_state* s, int k);
int or_bbi_profile(or_state* s, int j, int* nbins, double* out);
int or_fir(or_state* s, int turn);
int or_mark_lost(or_state* s, double* transmissions);
int or_run_turns(or_state* s, int turn0, int n_turns);
int or_ion_count(or_state* s, int k, int p, int* count);
int or_ion_download(or_state* s, int k, int p, double* x, double* y, double* vx, double* vy,
                    int capacity, int* count);
int or_ion_upload(or_state* s, int k, int p, const double* x, const double* y,
                  const double* vx, const double* vy, int count);
int or_ion_cloud_record(or_state* s, int k, double* out);
int or_sr_bins(or_state* s, int j, double* zlo, double* dz, int* counts);
int or_sr_potentials(or_state* s, int j, double* out);
int or_lr_add_rw(or_state* s, const double* yok);
int or_sr_set_rw(or_state* s, const double* yok);
double or_rw_fz(double u);
int or_lr_table(or_state* s, double* out, int capacity, int* np);
/* counter-based normals shared with the device code (test helper) */
void or_philox_normals(uint64_t seed, uint32_t stream, uint32_t c0, uint32_t c1, uint32_t c2,
                       uint32_t c3, double* out2);
#endif
