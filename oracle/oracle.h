/*
 * oracle.h -- FP64 CPU restatement of the cpsFDTD time-stepping loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA product in cpsfdtd_b200/.  It may be loaded only by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg; the product never
 * links, loads or calls it.
 *
 * What it restates (reference file:line, paths inside the cpsFDTD project):
 *   - Yee bulk E/H updates            BasicFDTD.cpp:25-47, 67-84
 *   - per-medium coefficients         Structure.cpp:309-359
 *   - CPML coefficients and updates   CPML.cpp:139-229, 231-527, 529-607, 609-689
 *   - Drude-Lorentz ADE (3-D form of) Drude_Lorentz.cpp:65-108, 153-227
 *   - four-level gain (3-D form of)   FourLevelLaser.cpp:96-105, 202-209, 270-325
 *   - TF/SF Gaussian beam             TF_SF.cpp:29-959 (tables), 966-986 (lookup),
 *                                     988-1089 (E), 1201-1300 (H)
 *   - port sampling                   Ports.cpp:88-99, 342-353
 *   - port DFT accumulators           (no reference; defined here)
 *
 * Storage follows the reference: every field is (nx+1)(ny+1)(nz+1) doubles in
 * [i][j][k] order with k fastest.
 *
 * Parity pins: the dielectric/CPML/TF-SF/port parts are checked against the
 * reference's own code compiled by oracle/Makefile (oracle/_ref/ref_harness);
 * the Drude-Lorentz and gain recursions are checked in 2-D TE form against the
 * reference's 2-D classes compiled with shim headers (oracle/_ref/ref2d_harness).
 * The 3-D extension of those two recursions and the port DFT have no reference
 * counterpart: their parity beyond the 2-D pin is unpinned.
 */
#ifndef CPS_ORACLE_H
#define CPS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/* TF/SF parameters, meaning as TF_SF.cpp:35-97, 898-907.  Angles in degrees.
 * i0,j0 come from xs/dx, ys/dy; k0 is the beam-centre plane (the reference
 * never assigns it, TF_SF.h:65); z0 is the waist offset as the reference uses
 * it (it overwrites the deck value with zs/dz, TF_SF.cpp:57). */
typedef struct orc_tfsf_params {
    double lambda, dlambda, w0, z0;
    int32_t i0, j0, k0;
    double theta_deg, phi_deg, E0, psi_deg;
    int32_t n_x1, n_x2, n_y1, n_y2, n_z1, n_z2;
    int32_t Nt;
    int32_t cwmode;
} orc_tfsf_params;

orc *orc_create(int nx, int ny, int nz, double dx, double dy, double dz, double dt);
void orc_destroy(orc *o);
int orc_set_threads(int n);
int orc_set_media(orc *o, int n, const double *epsR, const double *muR,
                  const double *sig, const double *sigM);
int orc_set_ids(orc *o, const uint8_t *ids);
/* literal = 1: the reference's single psi coefficients dt/eps0 and bH[0]
 * (CPML.cpp:524-525); 0: each cell's own curl coefficient (equal to them in
 * eps_r = mu_r = 1 media, the CFS-PML form in any medium) */
int orc_pml_init(orc *o, const int32_t npml[6], double m, double malp,
                 double kapmax, double sig_ratio, double alpmax, int literal);
/* literal = 1 takes C1 and C5 exactly as Drude_Lorentz.cpp:96,106; 0 (the
 * default of the product) takes the values the ADE discretisation gives;
 * 2 (one Drude pole, no Lorentz pole) is the single-pole Drude class with the
 * coefficients of Drude.cpp:56-60 (fD = omegaP, gD = gamma in Hz). */
int orc_dl_init(orc *o, double sigma, double epsInf,
                int nD, const double *fD, const double *gD,
                int nL, const double *fL, const double *dL, const double *depsL, int literal);
int orc_gain_init(orc *o, int gain_id, double lambda_a, double lambda_b,
                  double gamma_a, double gamma_b, double t30, double t32,
                  double t21, double t10, double N_0, double pump_rate);
int orc_tfsf_init(orc *o, const orc_tfsf_params *p);
int orc_tfsf_set_tables(orc *o, int n, const double *einc, const double *hinc);
int orc_source_add(orc *o, int comp, int i, int j, int k, const double *wave, int nwave);
int orc_port_add(orc *o, int npts, const int32_t *ijk);
int orc_port_set_dft(orc *o, int port, int nfreq, const double *freq_hz, uint32_t comp_mask);
void orc_set_step(orc *o, int64_t n);
int64_t orc_get_step(const orc *o);
void orc_step(orc *o, int nsteps);

/* single reference routines, for call-order tests */
void orc_op_h_bulk(orc *o);
void orc_op_h_pml(orc *o);
void orc_op_e_bulk(orc *o);
void orc_op_e_pml(orc *o);
void orc_op_dl(orc *o);
void orc_op_gain_p(orc *o);
void orc_op_gain_e(orc *o);
void orc_op_gain_n(orc *o);
void orc_op_tfsf_h(orc *o, int n);
void orc_op_tfsf_e(orc *o, int n);
void orc_op_sources(orc *o, int n);
void orc_op_ports(orc *o, int n);

int orc_get_field(const orc *o, int comp, double *out);
int orc_set_field(orc *o, int comp, const double *in);
int orc_get_stretch(const orc *o, int which, double *out);
int orc_port_read(const orc *o, int port, double *out);      /* [npts][6] */
int orc_port_dft_read(const orc *o, int port, double *out);  /* [npts][ncomp][nfreq][2] */
int orc_tfsf_tables(const orc *o, double *einc, double *hinc); /* Nt+1 each */
int orc_gain_populations(const orc *o, double *out);          /* [ncells][4] N0..N3 */
/* three-level gain (ThreeLevel.cpp), "cells" placement on ID gain_id; literal
 * as three_coeffs in cells.h (1: the reference's coefficients as written) */
int orc_three_init(orc *o, int gain_id, double lambda_a, double lambda_b, double gamma_a, double gamma_b,
                   double t20, double t21, double t10, double N_0, int literal);
void orc_op_three_p(orc *o);
void orc_op_three_e(orc *o);
void orc_op_three_n(orc *o);
int orc_three_populations(const orc *o, double *out);
int64_t orc_count_cells(const orc *o, int which); /* 0: DL cells, 1: four-level, 2: three-level gain cells */

/* 2-D TE drivers used to pin the recursions against the reference's 2-D
 * classes.  ids2d is [nx+1][ny+1] (j fastest); the source adds wave[n] to Hz
 * at (si,sj) after the H update of step n.  Outputs are [nx+1][ny+1]. */
int orc2d_run(int nx, int ny, double dx, double dy, double dt,
              const uint8_t *ids2d, int nmedia, const double *epsR, const double *muR,
              const double *sig, const double *sigM,
              int use_dl, double dl_sigma, double dl_epsInf, int nD, const double *fD,
              const double *gD, int nL, const double *fL, const double *dL,
              const double *depsL, int dl_literal,
              int use_gain /* 1: four-level, 2: three-level */,
              const double *gain_params /* four-level: la lb ga gb t30 t32 t21 t10 N_0 pump;
                                           three-level: la lb ga gb t20 t21 t10 N_0 literal */,
              int si, int sj, const double *wave, int nsteps,
              double *Ex, double *Ey, double *Hz);

#ifdef __cplusplus
}
#endif
#endif
