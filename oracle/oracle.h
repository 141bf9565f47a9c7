/*
 * oracle.h -- FP64 CPU restatement of the reference's FDTD time step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load liboracle.so, and only as the
 * checker or the timed CPU baseline; the product (libfdtd_b200.so) never
 * links or calls it.
 *
 * Parity pins: the oracle is checked against outputs of the reference
 * program itself (jbaxt089/FDTD-CUDA built unmodified from its sources by
 * oracle/Makefile.ref and run on a B200; fixtures under tests/golden/) and
 * against closed-form coefficient formulas.  The reference ships no tests or
 * golden vectors of its own.
 *
 * State is held in the reference's own layout: dense [i][j][k] arrays with k
 * (z) fastest, index k + NZ*(j + NY*i) (main.cu:16-19).
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H
#include <stddef.h>
#include "../include/fdtd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

void orc_params_default(fdtd_params* p);
int orc_load_input_txt(const char* path, fdtd_params* p);

/* Returns NULL and fills err (256 bytes) on invalid parameters. */
orc_sim* orc_create(const fdtd_params* p, char* err);
void orc_destroy(orc_sim* s);
int orc_set_design(orc_sim* s, const float* rho, size_t count);
/* 1 = DFT accumulators and spectral post emulate the reference's float
 * accumulators and float-complex flux arithmetic (global_var.h:22,
 * Spectral.cu:414-418); 0 = FP64 throughout (default). */
void orc_set_float_dft(orc_sim* s, int on);
/* 0 disables DFT accumulation (CPU-baseline timing of the field update). */
void orc_set_dft_enabled(orc_sim* s, int on);
/* Accumulate the DFT at the listed frequency indices only (n = 0: all);
 * the other frequencies keep zero accumulators.  Each frequency's
 * accumulators are independent, so the listed ones are unchanged: a
 * test-time saving for objectives that read a few frequencies. */
int orc_set_dft_freqs(orc_sim* s, const int* idx, int n);
void orc_set_threads(int n);

/* One full reference time step t (main.cu:2724-2934); advances t. */
void orc_step(orc_sim* s);
void orc_run(orc_sim* s, int nsteps);
int orc_time(const orc_sim* s);

void orc_dims(const orc_sim* s, fdtd_dims* d);
/* comp 0..5 = ex ey ez hx hy hz, reference layout. */
int orc_get_field(const orc_sim* s, int comp, double* out, size_t n);
int orc_set_field(orc_sim* s, int comp, const double* in, size_t n);
/* mat_matrix{X,Y,Z} as the class bits used by the product (bit c set when
 * component c has a dispersive update), plus the raw int class maps. */
int orc_get_material(const orc_sim* s, unsigned char* bits, int* matX,
                     int* matY, int* matZ, size_t n);
int orc_get_dft(const orc_sim* s, int box, int face, int comp, double* re,
                double* im, size_t n);
int orc_spectra(orc_sim* s, double* out19);
/* periodic_xy: lambda, R, T, 1 - R - T, |E_inc|, Re E_inc, Im E_inc per
 * frequency (NUM_freq x 7); -1 for a simulation that is not periodic. */
int orc_reflectance(orc_sim* s, double* out7);
int orc_get_freqs(const orc_sim* s, double* f, size_t n);
int orc_get_incident(const orc_sim* s, double* re, double* im, size_t n);
int orc_get_line(const orc_sim* s, double* e_inc, double* h_inc, size_t n);
/* Dispersive state of component comp, reference layout (n = NX*NY*NZ):
 * which 0 = the Drude polarisation (local model) or current (hydrodynamic)
 * of the last step, P*_d after main.cu:1207 / 2034; 1 = ND* as the
 * reference holds it after its step (the density from before the step,
 * main.cu:1267-1269); 2 = ND*_prev (the density after the step). */
int orc_get_state(const orc_sim* s, int which, int comp, double* out, size_t n);
int orc_get_probe(const orc_sim* s, double* out, size_t n);

/* Coefficient tables for unit tests.  which: 0=kedx 1=kedy 2=kedz
 * 3=khdx 4=khdy 5=khdz 6=be_x_N 7=ce_x_N 8=be_x_F 9=ce_x_F 10=bh_x_N
 * 11=ch_x_N 12=bh_x_F 13=ch_x_F, +8 for y, +16 for z (axis-major:
 * 6+8*axis+slot).  Returns the table length or -1. */
int orc_get_cpml(const orc_sim* s, int which, double* out, size_t n);
/* ADE scalars: C_E, C_E_1, C_E_2, d_1..d_5, d_NL, C_1..C_5 for both CP
 * poles (pole-major), dt, N_EQ: 22 values. */
int orc_get_ade(const orc_sim* s, double* out, size_t n);

#ifdef __cplusplus
}
#endif
#endif
