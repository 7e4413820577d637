/*
 * cps_capi.h -- C ABI of the B200 cpsFDTD time-stepping engine.
 *
 * Plain pointers and sizes only.  Every entry point returns a cps_status
 * (0 = success); cps_last_error() returns the message of the last failure on
 * the calling thread.  A cps_grid is one simulation domain resident on one
 * GPU; one grid handle must not be used from two threads at once, distinct
 * grids may be driven concurrently.
 *
 * Host-side arrays use the reference's storage order: a field or ID grid is
 * (nx+1)*(ny+1)*(nz+1) values in [i][j][k] order with k fastest (Fields.cpp:
 * 101-131).  On the device the engine keeps its own layout (x fastest, rows
 * padded to 32 elements); copies convert.
 *
 * Reference interface each call replaces (file:line inside the cpsFDTD tree):
 *   cps_grid_create ........... Structure::generate_mesh grid sizing (Structure.cpp:68-157),
 *                               Field::Field (Fields.cpp:52-186)
 *   cps_grid_set_media ........ Structure::Structure + InitializeBasicFDTDCoefficients
 *                               (Structure.cpp:26-52, 309-359)
 *   cps_grid_upload_ids ....... Structure::ID (Structure.h:36), filled by generate_mesh
 *   cps_mesh_rasterize ........ cuboid/ellipsoid/cylinder/multishape (Structure.cpp:159-307)
 *   cps_pml_init .............. CPML::CPML + InitializeCPML (CPML.cpp:29-68, 231-527);
 *                               CFS_PML::CFS_PML + Initialize_PML (CFS_PML.h:33-36)
 *   cps_dl_init ............... Drude_Lorentz::Drude_Lorentz (Drude_Lorentz.cpp:30-147)
 *   cps_drude_init ............ Drude::Drude (Drude.cpp:29-68); its EFieldUpdate is cps_op_dl
 *   cps_gain_init ............. FourLevelLaser::FourLevelLaser (FourLevelLaser.cpp:30-213)
 *   cps_tfsf_init ............. TF_SF::TF_SF (TF_SF.cpp:29-959)
 *   cps_source_add ............ the field injection of main.cpp:284-286
 *   cps_port_points_plain ..... PlainPort::PlainPort point set (Ports.cpp:201-306)
 *   cps_port_points_spherical . SphericalPort::SphericalPort point set (Ports.cpp:28-86)
 *   cps_port_add .............. a port's Port_Points array (Ports.h:29-36)
 *   cps_op_h_bulk / e_bulk .... BasicHFieldUpdate / BasicEFieldUpdate (BasicFDTD.cpp:67-84, 25-47)
 *   cps_op_h_pml / e_pml ...... CPML::UpdateCPMLHFields / UpdateCPMLEFields (CPML.cpp:609-689,
 *                               529-607); CFS_PML::UpdatePMLHFields / UpdatePMLEFields
 *   cps_op_dl ................. Drude_Lorentz::EFieldUpdate (Drude_Lorentz.cpp:153-227), 3-D form
 *   cps_op_gain_polarization .. FourLevelLaser::UpdatePolarizationDensities (FourLevelLaser.cpp:270-298)
 *   cps_op_gain_efield ........ FourLevelLaser::UpdateElectricField (FourLevelLaser.cpp:300-308)
 *   cps_op_gain_populations ... FourLevelLaser::UpdateStatesPopulations (FourLevelLaser.cpp:310-325)
 *   cps_three_init ............ ThreeLevel::ThreeLevel (ThreeLevel.cpp:29-209)
 *   cps_op_three_* ............ ThreeLevel::UpdatePolarizationDensities / UpdateElectricField /
 *                               UpdateStatesPopulations (ThreeLevel.cpp:216-266), 3-D form
 *   cps_op_tfsf_h / tfsf_e .... TF_SF::UpdateHField / UpdateEField and the face variants
 *                               (TF_SF.cpp:1201-1410, 988-1199)
 *   cps_op_port_sample ........ SphericalPort/PlainPort::Update_Fields_on_Port (Ports.cpp:88-99, 342-353)
 *   cps_deck_load ............. main.cpp:110-262's object construction from the resourses/ decks
 *   cps_step .................. one pass of the loop body of main.cpp:267-344
 *   cps_grid_set_record ....... (no counterpart) runs a step's cps_op_* calls, made in
 *                               main.cpp's order, as one fused step
 *   cps_field_download/upload . direct access to Field::Ex..Hz (Fields.h:28-33)
 *   cps_field_slice, cps_image_png  OutImage (OutImage.h:22-45) without a display
 *   cps_port_read ............. Port_Points::Ex..Hz after Update_Fields_on_Port
 *   cps_port_dft_read / flux .. (no reference counterpart: running FP64 DFT of the port samples)
 */
#ifndef CPS_CAPI_H
#define CPS_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CPS_API __attribute__((visibility("default")))
#else
#define CPS_API
#endif

typedef int32_t cps_status;
typedef struct cps_grid cps_grid;

enum {
    CPS_OK = 0,
    CPS_E_INVALID = 1,   /* bad argument or inconsistent configuration */
    CPS_E_CUDA = 2,      /* a CUDA call failed */
    CPS_E_NOMEM = 3,     /* device or host allocation failed */
    CPS_E_STATE = 4,     /* call not valid in the grid's current state */
    CPS_E_NUMERIC = 5,   /* non-finite field values detected */
    CPS_E_BUDGET = 6,    /* memory footprint exceeds the admission budget */
    CPS_E_TIMEOUT = 7,   /* a bounded device wait gave up */
    CPS_E_CANCELLED = 8, /* job cancelled */
    CPS_E_NOTFOUND = 9   /* unknown handle, port or job */
};

enum { CPS_FP64 = 0, CPS_FP32 = 1 };
enum { CPS_EX = 0, CPS_EY = 1, CPS_EZ = 2, CPS_HX = 3, CPS_HY = 4, CPS_HZ = 5 };
/* cps_step paths: PLAIN launches one kernel per reference routine in the
 * reference order; FUSED runs the fused sweeps, one for H and one for E
 * (same results within the precision's tolerance); ONEPASS runs H and E of
 * a step in one sweep into a second set of field buffers that then becomes
 * current (twice the field memory, about two thirds of FUSED's field traffic;
 * grids the TMA sweeps cannot tile, and sweep mode 1, run FUSED instead). */
enum { CPS_PATH_PLAIN = 0, CPS_PATH_FUSED = 1, CPS_PATH_ONEPASS = 2 };
/* TF/SF face bits for cps_op_tfsf_* (TF_SF.h:41-52 face variants) */
enum { CPS_FACE_X1 = 1, CPS_FACE_X2 = 2, CPS_FACE_Y1 = 4, CPS_FACE_Y2 = 8,
       CPS_FACE_Z1 = 16, CPS_FACE_Z2 = 32, CPS_FACE_ALL = 63 };

/* Material IDs with fixed meaning in the E update (BasicFDTD.cpp:34-38) */
#define CPS_ID_DISPERSIVE 2
#define CPS_ID_PEC 4

typedef struct cps_grid_desc {
    int32_t nx, ny, nz;      /* Structure::Nx..Nz; arrays span indices 0..N */
    double dx, dy, dz;       /* metres */
    double dt;               /* seconds; 0 selects 0.99 of the Courant limit (Structure.cpp:124) */
    int32_t precision;       /* CPS_FP64 or CPS_FP32 */
    int32_t device;          /* CUDA device ordinal */
} cps_grid_desc;

/* CPML deck values (CPML.cpp:37-62).  npml order x1 x2 y1 y2 z1 z2; both ends
 * of an axis must be equal and >= 1, or both 0 to leave that axis open.
 * literal = 0 (default): each cell's psi term takes the cell's own curl
 * coefficient (bE of its medium, the Drude-Lorentz C3 on ID-2 cells, bH of
 * its medium on the H side), the CFS-PML update for any medium; it equals the
 * reference wherever the CPML holds eps_r = mu_r = 1 media.  literal = 1 uses
 * the reference's single dt/eps0 and bH[0] (CPML.cpp:524-525), with which the
 * CPML grows without bound when its medium has eps_r != 1. */
typedef struct cps_pml_params {
    int32_t npml[6];
    double m, malp, kapmax, sig_ratio, alpmax;
    int32_t literal;
} cps_pml_params;

/* Drude-Lorentz deck values (Drude_Lorentz.cpp:37-94); frequencies in Hz.
 * literal = 1 uses C1 and C5 exactly as Drude_Lorentz.cpp:96,106; 0 uses the
 * values the ADE discretisation gives (the literal C5 lacks a factor dt and is
 * unstable with any Lorentz pole); 2, with one Drude pole and no Lorentz pole,
 * uses the single-pole Drude class's coefficients (Drude.cpp:56-60). */
#define CPS_MAX_POLES 8
typedef struct cps_dl_params {
    double sigma, epsInf;
    int32_t nD, nL;
    double fD[CPS_MAX_POLES], gD[CPS_MAX_POLES];
    double fL[CPS_MAX_POLES], dL[CPS_MAX_POLES], depsL[CPS_MAX_POLES];
    int32_t literal;
} cps_dl_params;

/* Single-pole Drude deck values (Drude.cpp:29-52): eps_inf, plasma and
 * collision frequencies in Hz (the class multiplies them by 2 pi) and the
 * conductivity.  The same ID-2 cells and state as the Drude-Lorentz module,
 * with the coefficients of Drude.cpp:56-60; one of the two per grid. */
typedef struct cps_drude_params {
    double epsInf, omegaP_hz, sigma, gamma_hz;
} cps_drude_params;

/* Four-level gain deck values (FourLevelLaser.cpp:37-93).  Gain sites are the
 * cells whose ID equals gain_id (the reference places them on ID==5,
 * FourLevelLaser.cpp:119-140).  pump_rate (1/s) moves population N0 -> N3 and
 * has no reference counterpart; 0 reproduces the reference. */
typedef struct cps_gain_params {
    int32_t gain_id;
    double lambda_a, lambda_b, gamma_a, gamma_b;
    double t30, t32, t21, t10;
    double N_0;
    double pump_rate;
} cps_gain_params;

/* Three-level gain deck values (ThreeLevel.cpp:37-84), "cells" placement on
 * the cells of ID gain_id (the reference's "random" placement compares a char
 * array with a literal and is never taken).  literal = 1 takes the reference's
 * coefficients as written (ThreeLevel.cpp:100-119: its oscillator coefficients
 * make the polarisation double every two steps, and the N0 update applies
 * CN0Ea to the Pbx term); 0 uses the Lorentz-oscillator discretisation
 * (2/dt^2 - w^2)/(1/dt^2 + g/2dt), (g/2dt - 1/dt^2)/(1/dt^2 + g/2dt) and CN0Eb
 * on every b term.  N_1 is read by the reference and unused.  One of the
 * four-level and three-level modules per grid. */
typedef struct cps_three_params {
    int32_t gain_id;
    double lambda_a, lambda_b, gamma_a, gamma_b;
    double t20, t21, t10;
    double N_0, N_1;
    int32_t literal;
} cps_three_params;

/* TF/SF deck values (TF_SF.cpp:35-97, 898-907).  i0 = xs/dx and j0 = ys/dy
 * (truncated), z0 = zs/dz as the reference sets it (TF_SF.cpp:55-57), k0 the
 * beam-centre plane (TF_SF.h:65; the reference never assigns it).  Angles in
 * degrees.  n[] = nTFSF x1 x2 y1 y2 z1 z2.  Nt = incident-table length - 1. */
typedef struct cps_tfsf_params {
    double lambda, dlambda, w0, z0;
    int32_t i0, j0, k0;
    double theta_deg, phi_deg, E0, psi_deg;
    int32_t n[6];
    int32_t Nt;
    int32_t cwmode;
} cps_tfsf_params;

/* One structure.txt shape line (Structure.cpp:88-106); type 0 cuboid,
 * 1 ellipsoid, 2 cylinder, 3 multi (theta/phi/psi = counts, a/b/c = pitch,
 * material_index = index of the template shape). */
enum { CPS_SHAPE_CUBOID = 0, CPS_SHAPE_ELLIPSOID = 1, CPS_SHAPE_CYLINDER = 2, CPS_SHAPE_MULTI = 3 };
typedef struct cps_shape {
    int32_t type;
    int32_t material_index;
    double theta, phi, psi;
    double x0, y0, z0;
    double a, b, c;
} cps_shape;

CPS_API const char *cps_last_error(void);
CPS_API const char *cps_version(void);
CPS_API double cps_courant_dt(double dx, double dy, double dz);

/* ---- grid lifetime ---- */
CPS_API cps_status cps_grid_create(const cps_grid_desc *desc, cps_grid **out);
CPS_API cps_status cps_grid_destroy(cps_grid *g);
CPS_API cps_status cps_grid_info(const cps_grid *g, cps_grid_desc *out);
/* device bytes the grid holds now */
CPS_API cps_status cps_grid_bytes(const cps_grid *g, int64_t *bytes);
/* CUDA stream (cudaStream_t) all work of the grid is enqueued on; NULL = the
 * grid's own stream */
CPS_API cps_status cps_grid_set_stream(cps_grid *g, void *stream);
CPS_API cps_status cps_grid_get_stream(const cps_grid *g, void **stream);
CPS_API cps_status cps_synchronize(cps_grid *g);

/* ---- geometry and media ---- */
CPS_API cps_status cps_grid_set_media(cps_grid *g, int32_t n, const double *epsR, const double *muR,
                                      const double *sig, const double *sigM);
CPS_API cps_status cps_grid_upload_ids(cps_grid *g, const uint8_t *ids);
CPS_API cps_status cps_grid_download_ids(const cps_grid *g, uint8_t *ids);
/* Rasterise shapes into a host ID grid exactly as Structure::generate_mesh does
 * (ids must hold (nx+1)(ny+1)(nz+1) bytes, [i][j][k]; it is overwritten with 0
 * first unless keep != 0). */
CPS_API cps_status cps_mesh_rasterize(int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                      int32_t nshapes, const cps_shape *shapes, uint8_t *ids, int32_t keep);
/* The same rasterisation on the device, straight into the grid's IDs (the
 * grid's cell sizes; the IDs are zeroed first unless keep != 0); the same
 * cells get the same IDs as cps_mesh_rasterize + cps_grid_upload_ids.  Call it
 * where cps_grid_upload_ids would be called. */
CPS_API cps_status cps_grid_rasterize(cps_grid *g, int32_t nshapes, const cps_shape *shapes, int32_t keep);

/* A grid from a directory of the reference's deck files (material.txt,
 * structure.txt; CFS_PML.txt, DrudeLorentz.txt or Drude.txt, FourLevelLaser.txt
 * or ThreeLevel.txt, TF_SF.txt, port0.txt, port1.txt, ... when present), set up
 * through the drop-in classes' parsing (cpsfdtd_classes.hpp).  A malformed or
 * missing required deck gives CPS_E_INVALID with the file named; a failing
 * set-up call gives that call's status.  Port DFTs and sources (main.cpp code
 * in the reference) are added by the caller.  The caller destroys *out. */
CPS_API cps_status cps_deck_load(const char *dir, int32_t precision, cps_grid **out);

/* ---- physics modules (call after media and IDs are set) ---- */
CPS_API cps_status cps_pml_init(cps_grid *g, const cps_pml_params *p);
CPS_API cps_status cps_dl_init(cps_grid *g, const cps_dl_params *p);
CPS_API cps_status cps_drude_init(cps_grid *g, const cps_drude_params *p);
CPS_API cps_status cps_gain_init(cps_grid *g, const cps_gain_params *p);
CPS_API cps_status cps_three_init(cps_grid *g, const cps_three_params *p);
CPS_API cps_status cps_tfsf_init(cps_grid *g, const cps_tfsf_params *p);
/* replace the incident tables Einc/Hinc (n = Nt + 1 values each) */
CPS_API cps_status cps_tfsf_set_tables(cps_grid *g, int32_t n, const double *einc, const double *hinc);
CPS_API cps_status cps_tfsf_get_tables(const cps_grid *g, int32_t n, double *einc, double *hinc);
/* additive source: field comp at (i,j,k) += wave[n] at step n (0 <= n < nwave) */
CPS_API cps_status cps_source_add(cps_grid *g, int32_t comp, int32_t i, int32_t j, int32_t k,
                                  const double *wave, int32_t nwave);

/* ---- ports ---- */
/* point sets of the reference constructors; call with ijk = NULL to get the
 * count, then with room for 3*count int32 */
CPS_API cps_status cps_port_points_plain(int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                         char normal, double position, double w1, double w2, double h1,
                                         double h2, int32_t *count, int32_t *ijk);
CPS_API cps_status cps_port_points_spherical(int32_t nx, int32_t ny, int32_t nz, double dx, double dy,
                                             double dz, double r, double xc, double yc, double zc,
                                             double theta1_deg, double theta2_deg, double phi1_deg,
                                             double phi2_deg, int32_t *count, int32_t *ijk);
CPS_API cps_status cps_port_add(cps_grid *g, int32_t npoints, const int32_t *ijk, int32_t *port_id);
/* running DFT of the samples at nfreq frequencies (Hz) for the components in
 * comp_mask (bit c = component c); FP64 accumulators on the device */
CPS_API cps_status cps_port_set_dft(cps_grid *g, int32_t port_id, int32_t nfreq, const double *freq_hz,
                                    uint32_t comp_mask);
/* last sample, [npoints][6] */
CPS_API cps_status cps_port_read(cps_grid *g, int32_t port_id, double *out);
/* DFT accumulators, [ncomp][nfreq][2][npoints]: for each component (ascending)
 * and frequency a plane of real parts then a plane of imaginary parts */
CPS_API cps_status cps_port_dft_read(cps_grid *g, int32_t port_id, double *out);
/* net Poynting flux 0.5*Re(sum_p (E x conj H) . n dA) per frequency through a
 * planar port whose DFT holds the four tangential components; normal = 'x','y','z' */
CPS_API cps_status cps_port_flux(cps_grid *g, int32_t port_id, char normal, double *out);

/* ---- time stepping ---- */
/* step index n used by TF/SF and sources; main.cpp's loop starts at 1 */
CPS_API cps_status cps_grid_set_step(cps_grid *g, int64_t n);
CPS_API cps_status cps_grid_get_step(const cps_grid *g, int64_t *n);
/* advance nsteps steps, each in the order of main.cpp:267-344: H bulk, TF/SF H,
 * CPML H, E bulk, Drude-Lorentz, gain (P, E, N), TF/SF E, sources, CPML E,
 * port sampling.  Asynchronous on the grid's stream. */
CPS_API cps_status cps_step(cps_grid *g, int32_t nsteps, int32_t path);
/* On (default): cps_step on the fused path runs grids of 4 Mi cells or more
 * as chunks of a one-grid batch (the batch's CUDA-graph-replayed chunks; the
 * results are the direct launches' bit for bit), except while per-step timing
 * (cps_grid_set_timing) is on; off: one launch sequence per step. */
CPS_API cps_status cps_grid_set_chunked(cps_grid *g, int32_t on);

/* ---- single reference routines (one launch each, enqueued on the grid's stream) ---- */
CPS_API cps_status cps_op_h_bulk(cps_grid *g);
CPS_API cps_status cps_op_e_bulk(cps_grid *g);
CPS_API cps_status cps_op_h_pml(cps_grid *g);
CPS_API cps_status cps_op_e_pml(cps_grid *g);
CPS_API cps_status cps_op_dl(cps_grid *g);
CPS_API cps_status cps_op_gain_polarization(cps_grid *g);
CPS_API cps_status cps_op_gain_efield(cps_grid *g);
CPS_API cps_status cps_op_gain_populations(cps_grid *g);
CPS_API cps_status cps_op_tfsf_h(cps_grid *g, int32_t n, uint32_t face_mask);
CPS_API cps_status cps_op_tfsf_e(cps_grid *g, int32_t n, uint32_t face_mask);
CPS_API cps_status cps_op_sources(cps_grid *g, int32_t n);
CPS_API cps_status cps_op_port_sample(cps_grid *g, int32_t port_id, int32_t n);
CPS_API cps_status cps_op_three_polarization(cps_grid *g);
CPS_API cps_status cps_op_three_efield(cps_grid *g);
CPS_API cps_status cps_op_three_populations(cps_grid *g);

/* Record-and-fuse for the calls above (main.cpp:264-330 calls one routine per
 * term each step).  With recording on, cps_op_* calls are validated and queued;
 * a queue that forms one whole step runs as the fused H and E sweeps
 * (CPS_PATH_FUSED's kernels) plus the recorded TF/SF, source and port calls,
 * and any other queue is replayed call by call in its order.  Fusable order:
 * h_bulk first; tfsf_h and h_pml in any order before e_bulk; dl, then gain
 * polarization, efield, populations; then tfsf_e, sources and e_pml in any
 * order; port samples last, each port at most once.  h_pml/e_pml, dl and the
 * gain calls appear exactly once when their module is initialised.  The queue
 * runs at the next h_bulk, at any call that reads or changes the grid (field,
 * port, population reads, cps_synchronize, cps_step, set-up calls,
 * cps_batch_step of a batch holding the grid) and when recording is switched
 * off; a launch error of a recorded call is returned by the call that ran it.
 * Off by default. */
CPS_API cps_status cps_grid_set_record(cps_grid *g, int32_t on);
/* steps run fused, calls replayed one by one, calls queued now; NULL skips */
CPS_API cps_status cps_grid_record_stats(const cps_grid *g, int64_t *fused_steps, int64_t *replayed_calls,
                                         int32_t *pending);

/* ---- field access ---- */
CPS_API cps_status cps_field_download(cps_grid *g, int32_t comp, double *out);
CPS_API cps_status cps_field_upload(cps_grid *g, int32_t comp, const double *in);
CPS_API cps_status cps_field_download_f32(cps_grid *g, int32_t comp, float *out);
/* one plane of a field component (what 0..5) or of |E|^2 (what 6), cut on the
 * device: out[u][v] FP64 with (u, v) = (j, k) for a plane of constant x (axis
 * 0), (i, k) for y (axis 1), (i, j) for z (axis 2) */
CPS_API cps_status cps_field_slice(cps_grid *g, int32_t what, int32_t axis, int32_t index, double *out);
/* Headless stand-in for OutImage::plot_save (OutImage.cpp:140-200): an RGB
 * PNG of values[x][y] (nx x ny) through OutImage's colour map between cmin and
 * cmax (no display, no image library) */
CPS_API cps_status cps_image_png(const char *path, int32_t nx, int32_t ny, const double *values, double cmin,
                                 double cmax);
/* electromagnetic energy in the grid (no reference counterpart): electric
 * 0.5 sum eps0 epsR |E|^2 dV and magnetic 0.5 sum mu0 muR |H|^2 dV over all
 * cells, each cell's medium for both (dispersive and gain polarisation energy
 * not included), summed in FP64 on the device */
CPS_API cps_status cps_grid_energy(cps_grid *g, double *electric, double *magnetic);
/* an 8-bit RGB PNG of rgb[y][x][3] */
CPS_API cps_status cps_png_rgb(const char *path, int32_t nx, int32_t ny, const uint8_t *rgb);
/* reset fields, auxiliary state, port samples and DFT accumulators to zero
 * (initial populations for gain) and the step index to n0; also clears a
 * device timeout (CPS_E_TIMEOUT) recorded by an earlier sweep */
CPS_API cps_status cps_grid_reset(cps_grid *g, int64_t n0);
/* test setting for the bounded device waits (no reference counterpart; the
 * reference has no failure handling, main.cpp:68-85): with extra_bytes > 0
 * (at most 4096) the first plane of every tile of this grid's own TMA sweeps
 * (cps_step FUSED below the chunked size, cps_op_* and recorded steps)
 * expects that many more bytes than its loads bring, so each block's wait
 * runs out after its limit (about a second) and the step reports
 * CPS_E_TIMEOUT at the next synchronisation, with no fault and the context
 * intact.  0 (the default) restores normal operation; cps_grid_reset then
 * makes the grid usable again. */
CPS_API cps_status cps_grid_set_wait_skew(cps_grid *g, int32_t extra_bytes);
/* count of non-finite field values (device reduction) */
CPS_API cps_status cps_grid_check_finite(cps_grid *g, int64_t *nonfinite);
/* FP64 gain populations, [ncells][4] N0..N3, cells in (i,j,k) order */
CPS_API cps_status cps_gain_populations(cps_grid *g, double *out, int64_t *ncells);
/* three-level populations, [ncells][3] N0 N1 N2, cells in (i,j,k) order */
CPS_API cps_status cps_three_populations(cps_grid *g, double *out, int64_t *ncells);
/* number of kernel launches this grid has enqueued since creation */
CPS_API cps_status cps_grid_launch_count(const cps_grid *g, int64_t *launches);
/* fold the port samples still held in the rings into the DFT accumulators
 * (the read-out calls do this themselves) */
CPS_API cps_status cps_ports_flush(cps_grid *g);
/* sweep timing: with stride > 0, cps_step records CUDA events on the grid's
 * stream around the H and E sweeps of every stride-th step (at most 4096
 * samples); cps_grid_timing synchronises and returns their mean durations in
 * milliseconds.  stride 0 turns it off and clears the samples. */
CPS_API cps_status cps_grid_set_timing(cps_grid *g, int32_t stride);
/* tile of the fused sweeps: rows (4, 8 or 16) of 32 columns per block and
 * planes marched per block (>= 1), set for every sweep; the default is 4 rows
 * with 8 planes for the E sweep, 16 for the H sweep and 4 for an FP32 E sweep
 * with gain.  cps_grid_get_tile returns the rows and the E sweep's planes.
 * Tiling does not change results. */
CPS_API cps_status cps_grid_set_tile(cps_grid *g, int32_t rows, int32_t planes);
CPS_API cps_status cps_grid_get_tile(const cps_grid *g, int32_t *rows, int32_t *planes);
/* fused sweep kind: 0 (default) stages x-y tiles of several planes in shared
 * memory with TMA bulk-tensor loads (tiles of 4 or 8 rows); 1 loads through
 * registers.  Both give the same results. */
CPS_API cps_status cps_grid_set_sweep(cps_grid *g, int32_t mode);
CPS_API cps_status cps_grid_timing(cps_grid *g, double *h_sweep_ms, double *e_sweep_ms, int64_t *samples);
/* cps_ports_flush without any device allocation (no reference counterpart):
 * the contraction's phasor scratch is a 512 KiB static device array shared by
 * all grids of a device, so ports may have at most 256 frequencies and calls
 * on one device must not overlap.  For callers that cannot allocate (a fixed
 * admitted memory budget, or a loop that must not enter the allocator).  The
 * first call on a device looks up the array's address.  A grid holding
 * recorded calls not yet run (cps_grid_set_record) is refused with
 * CPS_E_STATE: running them may allocate. */
CPS_API cps_status cps_ports_flush_static(cps_grid *g);
/* host FP64 copies of the per-medium coefficients (Structure::aE, bE, aH,
 * bH, Structure.cpp:309-359), NoMedia entries each; NULL skips an array */
CPS_API cps_status cps_grid_coefficients(const cps_grid *g, double *aE, double *bE, double *aH, double *bH);
/* one stretched-coordinate array (Structure.h:82-83) with the CPML kappa
 * folded in: which = 0..11 for cExy cEyx cEzx cExz cEzy cEyz cHxy cHyx cHzx
 * cHxz cHzy cHyz; *len receives its length (Nz, Ny or Nx); out may be NULL */
CPS_API cps_status cps_grid_stretch(const cps_grid *g, int32_t which, double *out, int32_t *len);

/* ---- batched engine (no reference counterpart: main.cpp runs one grid per
 * process).  A batch advances many independent grids of one precision
 * together: one launch per sweep class over a table of tiles of all member
 * grids, then one launch each for the Drude-Lorentz cells, TF/SF injection,
 * sources and port sampling of all grids; steps run in chunks of at most 64
 * that end with one port-DFT contraction and are captured into CUDA graphs.
 * Members are built and read with the one-grid calls above; results are the
 * same as stepping each grid alone with CPS_PATH_FUSED.  A member changed
 * between batch steps (set-up calls, cps_step, cps_grid_set_step) is picked
 * up by the next cps_batch_step.  Grids need nx >= 32, ny >= 8, nz >= 2. */
typedef struct cps_batch cps_batch;
CPS_API cps_status cps_batch_create(int32_t precision, cps_batch **out);
CPS_API cps_status cps_batch_destroy(cps_batch *b);
CPS_API cps_status cps_batch_add(cps_batch *b, cps_grid *g);
CPS_API cps_status cps_batch_remove(cps_batch *b, cps_grid *g);
CPS_API cps_status cps_batch_info(const cps_batch *b, int32_t *ngrids, int64_t *cells);
/* advance every member by nsteps (asynchronous on the batch stream; member
 * streams are ordered after it) */
CPS_API cps_status cps_batch_step(cps_batch *b, int32_t nsteps);
/* wait for the batch stream; reports a device-side wait that gave up */
CPS_API cps_status cps_batch_synchronize(cps_batch *b);
/* tile rows (4 or 8), planes per tile, sweep launch mode (0: one launch per
 * sweep class over all members' tiles, one block per tile; 1: the same with as
 * many blocks as fit on the device, each walking the table; 2: every member's
 * sweeps as its own one-grid launches, members spread over side streams so
 * that several run at once; the default, with 4 rows and 16 planes).  Results
 * do not depend on the choice. */
CPS_API cps_status cps_batch_set_tile(cps_batch *b, int32_t rows, int32_t planes, int32_t persistent);
CPS_API cps_status cps_batch_get_tile(const cps_batch *b, int32_t *rows, int32_t *planes, int32_t *persistent);
/* CUDA-graph replay of step chunks (default on) */
CPS_API cps_status cps_batch_set_graph(cps_batch *b, int32_t on);
CPS_API cps_status cps_batch_get_stream(const cps_batch *b, void **stream);
CPS_API cps_status cps_batch_launch_count(const cps_batch *b, int64_t *launches);
/* autotuner key of the batch: precision, shape bucket and material mix */
CPS_API cps_status cps_batch_tune_key(const cps_batch *b, char *buf, int32_t len);
/* choose tile rows, planes and persistence: from cache_path when it holds
 * the batch's key, else by timing each candidate over trial_steps live steps
 * (members advance; *steps_run says by how much) and appending the winner */
CPS_API cps_status cps_batch_autotune(cps_batch *b, const char *cache_path, int32_t trial_steps,
                                      int32_t *steps_run);

/* ---- serving loop (no reference counterpart).  Jobs are queued with an
 * admission footprint and a step count; a poll builds the queued jobs that
 * fit (free slot and used + footprint <= budget, first come first served),
 * waits for the chunk in flight, retires finished jobs and launches the next
 * chunk for every live job in one batch (continuous batching).  build creates
 * and sets up the job's grid when it is admitted (a failing build fails that
 * job only); done receives the grid when the job ends -- status CPS_OK,
 * CPS_E_BUDGET (larger than the whole budget), CPS_E_CANCELLED, or the error
 * that ended it -- and must copy out what it needs: the server destroys the
 * grid when done returns.  A job's results do not depend on the other jobs. */
typedef struct cps_server cps_server;
typedef cps_status (*cps_job_build_fn)(void *user, int64_t job_id, cps_grid **out);
typedef void (*cps_job_done_fn)(void *user, int64_t job_id, cps_grid *g, cps_status status);
typedef struct cps_server_config {
    int32_t precision;       /* CPS_FP32 or CPS_FP64: every job's grid */
    int32_t max_jobs;        /* live jobs at most */
    int64_t budget_bytes;    /* device memory admission budget */
    int32_t chunk_steps;     /* steps between scheduling points, 1..64 */
    int32_t tile_rows, tile_planes, tile_persistent;  /* batch tiling; rows 0 keeps the default */
} cps_server_config;
typedef struct cps_server_stats {
    int64_t jobs_done, jobs_failed, jobs_rejected, jobs_cancelled, jobs_live, jobs_queued;
    int64_t bytes_in_use, chunks;
    double latency_p50_ms, latency_p99_ms;   /* submit -> done, finished jobs */
    double wait_p50_ms, wait_p99_ms;         /* submit -> admitted */
    double run_p50_ms;                       /* admitted -> done */
    double cell_updates;                     /* of all chunks completed */
    double span_s;                           /* first submit -> last finished job */
    double gpu_busy_s;                       /* device time of the chunks (events on the batch stream) */
} cps_server_stats;
CPS_API cps_status cps_server_create(const cps_server_config *cfg, cps_server **out);
CPS_API cps_status cps_server_destroy(cps_server *s);   /* cancels what is left */
CPS_API cps_status cps_server_submit(cps_server *s, int64_t footprint_bytes, int32_t nsteps,
                                     cps_job_build_fn build, cps_job_done_fn done, void *user, int64_t *job_id);
CPS_API cps_status cps_server_poll(cps_server *s, int32_t *live, int32_t *queued);
CPS_API cps_status cps_server_drain(cps_server *s);      /* poll until nothing is queued or live */
CPS_API cps_status cps_server_cancel(cps_server *s, int64_t job_id);
CPS_API cps_status cps_server_get_stats(const cps_server *s, cps_server_stats *out);

#ifdef __cplusplus
}
#endif
#endif
