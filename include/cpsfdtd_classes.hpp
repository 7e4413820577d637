// cpsfdtd_classes.hpp -- the cpsFDTD host classes (Structure, Field,
// BasicEFieldUpdate/BasicHFieldUpdate, CPML, CFS_PML, Drude_Lorentz, Drude,
// FourLevelLaser, ThreeLevel, TF_SF, SphericalPort, PlainPort) with the reference's names,
// constructors, public members and update methods, reading the same
// resourses/*.txt decks, over the C ABI of cps_capi.h.  A main.cpp written
// for the reference compiles against this header instead of Structure.h,
// Fields.h, BasicFDTD.h, CPML.h, CFS_PML.h, Drude_Lorentz.h, Drude.h,
// FourLevelLaser.h, ThreeLevel.h, TF_SF.h and Ports.h, and links with -lcpsfdtd.
//
// State lives on the GPU; update calls are recorded on the grid
// (cps_grid_set_record): a step made in main.cpp's order runs as the two
// fused sweeps, any other order routine by routine, on the grid's stream in
// call order.  CPSFDTD_RECORD=0 in the environment runs every call at once.  The Field members Ex..Hz are host mirrors
// in the reference's [i][j][k] layout: Field::sync_to_host() fills them from
// the device and Field::sync_to_device() writes them back (the reference
// reads and writes them directly; here the copies are explicit).
//
// Precision: FP64 by default (the reference's); the environment variable
// CPSFDTD_PRECISION=fp32 or Structure::default_precision selects FP32 grids.
//
// Failures (unreadable deck, rejected parameters, CUDA errors) throw
// std::runtime_error carrying cps_last_error(); the reference reports none.
#pragma once

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cps_capi.h"

namespace cpsfdtd_detail {

// a failed C-ABI call: the message and the call's status
struct call_error : std::runtime_error {
    cps_status code;
    call_error(const std::string &m, cps_status c) : std::runtime_error(m), code(c) {}
};

inline void check(cps_status s, const char *what)
{
    if (s != CPS_OK) throw call_error(std::string(what) + ": " + cps_last_error(), s);
}

// the lines of a deck; a missing file is an error (the reference reads zeros)
inline std::vector<std::string> deck_lines(const char *fileName)
{
    std::ifstream in(fileName);
    if (!in) throw std::runtime_error(std::string("cannot open deck ") + fileName);
    std::vector<std::string> v;
    std::string s;
    while (std::getline(in, s)) v.push_back(s);
    return v;
}

// the values of line n as a stream (a missing line reads as an empty one; a
// value that is not there reads as 0, as the reference's istringstream reads do)
struct LineReader {
    std::vector<std::string> lines;
    explicit LineReader(const char *f) : lines(deck_lines(f)) {}
    std::istringstream line(size_t n) const { return std::istringstream(n < lines.size() ? lines[n] : std::string()); }
};

template <typename T>
T ***alloc3(int n1, int n2, int n3, T init)
{
    T *block = new T[(size_t)n1 * n2 * n3];
    for (size_t q = 0; q < (size_t)n1 * n2 * n3; ++q) block[q] = init;
    T **rows = new T *[(size_t)n1 * n2];
    T ***a = new T **[n1];
    for (int i = 0; i < n1; ++i) {
        a[i] = rows + (size_t)i * n2;
        for (int j = 0; j < n2; ++j) a[i][j] = block + ((size_t)i * n2 + j) * n3;
    }
    return a;
}

template <typename T>
void free3(T ***a)
{
    if (!a) return;
    delete[] a[0][0];
    delete[] a[0];
    delete[] a;
}

}  // namespace cpsfdtd_detail

// Structure.h:20-34
struct shape {
    int index;
    int material_index;
    std::string type;
    double theta, phi, psi;
    double x0, y0, z0;
    double a, b, c;
    int ix0, jy0, kz0;
    int ia, jb, kc;
};

// Structure.h:36-72: material deck in the constructor, mesh deck in
// generate_mesh; the device grid is created by InitializeBasicFDTDCoefficients.
class Structure {
public:
    static int default_precision() {
        const char *p = getenv("CPSFDTD_PRECISION");
        return (p && (strcmp(p, "fp32") == 0 || strcmp(p, "FP32") == 0)) ? CPS_FP32 : CPS_FP64;
    }

    explicit Structure(const char *fileName, int precision = default_precision()) : precision_(precision)
    {
        cpsfdtd_detail::LineReader r(fileName);
        int n = 0;
        r.line(0) >> n;
        if (n < 1 || n > 255) throw std::runtime_error(std::string("bad medium count in ") + fileName);
        NoMedia = (short)n;
        epsR = new double[n]; muR = new double[n]; sig = new double[n]; sigM = new double[n];
        for (int m = 0; m < n; ++m) {
            epsR[m] = 1; muR[m] = 1; sig[m] = 0; sigM[m] = 0;
            r.line(1 + m) >> epsR[m] >> muR[m] >> sig[m] >> sigM[m];
        }
    }
    ~Structure()
    {
        if (grid_) cps_grid_destroy(grid_);
        cpsfdtd_detail::free3(ID);
        delete[] epsR; delete[] muR; delete[] sig; delete[] sigM;
        delete[] shapes;
        delete[] aE; delete[] bE; delete[] aH; delete[] bH;
        for (double *p : {cExy, cEyx, cEzx, cExz, cEzy, cEyz, cHxy, cHyx, cHzx, cHxz, cHzy, cHyz}) delete[] p;
    }
    Structure(const Structure &) = delete;
    Structure &operator=(const Structure &) = delete;

    // Structure.cpp:68-157: sizes (N = L/d, truncated), dt at 0.99 of the
    // Courant limit, IDs rasterised from the shapes
    void generate_mesh(const char *fileName)
    {
        cpsfdtd_detail::LineReader r(fileName);
        r.line(0) >> Lx >> Ly >> Lz;
        r.line(1) >> dx >> dy >> dz;
        int fs = 0;
        r.line(2) >> fs;
        freespace = fs != 0;
        r.line(3) >> NoShapes;
        if (NoShapes < 0) NoShapes = 0;
        delete[] shapes;
        shapes = new shape[NoShapes > 0 ? NoShapes : 1];
        std::vector<cps_shape> cs;
        for (int s = 0; s < NoShapes; ++s) {
            shape &q = shapes[s];
            q = shape{};
            r.line(4 + s) >> q.index >> q.material_index >> q.type >> q.theta >> q.phi >> q.psi >> q.x0 >> q.y0 >>
                q.z0 >> q.a >> q.b >> q.c;
            q.ix0 = (int)(q.x0 / dx); q.jy0 = (int)(q.y0 / dy); q.kz0 = (int)(q.z0 / dz);
            q.ia = (int)(q.a / dx); q.jb = (int)(q.b / dy); q.kc = (int)(q.c / dz);
            cps_shape c{};
            c.type = q.type == "cuboid" ? CPS_SHAPE_CUBOID : q.type == "ellipsoid" ? CPS_SHAPE_ELLIPSOID
                   : q.type == "cylinder" ? CPS_SHAPE_CYLINDER : q.type == "multi" ? CPS_SHAPE_MULTI : -1;
            c.material_index = q.material_index;
            c.theta = q.theta; c.phi = q.phi; c.psi = q.psi;
            c.x0 = q.x0; c.y0 = q.y0; c.z0 = q.z0;
            c.a = q.a; c.b = q.b; c.c = q.c;
            if (c.type >= 0) cs.push_back(c);  // unknown types draw nothing, as in the reference
        }
        Nx = (int)(Lx / dx); Ny = (int)(Ly / dy); Nz = (int)(Lz / dz);
        dt = cps_courant_dt(dx, dy, dz);
        std::vector<uint8_t> ids((size_t)(Nx + 1) * (Ny + 1) * (Nz + 1), 0);
        if (!freespace && !cs.empty())
            cpsfdtd_detail::check(cps_mesh_rasterize(Nx, Ny, Nz, dx, dy, dz, (int)cs.size(), cs.data(), ids.data(), 0),
                                  "generate_mesh");
        cpsfdtd_detail::free3(ID);
        ID = cpsfdtd_detail::alloc3<short>(Nx + 1, Ny + 1, Nz + 1, 0);
        for (size_t q = 0; q < ids.size(); ++q) ID[0][0][q] = ids[q];
    }

    // Structure.cpp:309-359 on the device grid; the host arrays aE..bH and
    // the stretched-coordinate arrays are copies of what the grid uses
    void InitializeBasicFDTDCoefficients()
    {
        if (!ID) throw std::runtime_error("InitializeBasicFDTDCoefficients before generate_mesh");
        if (!grid_) {
            cps_grid_desc d{Nx, Ny, Nz, dx, dy, dz, dt, precision_, 0};
            cpsfdtd_detail::check(cps_grid_create(&d, &grid_), "Structure grid");
            const char *rec = getenv("CPSFDTD_RECORD");
            cpsfdtd_detail::check(cps_grid_set_record(grid_, !(rec && strcmp(rec, "0") == 0)), "record");
        }
        cpsfdtd_detail::check(cps_grid_set_media(grid_, NoMedia, epsR, muR, sig, sigM), "media");
        upload_ids();
        refresh_coefficients();
    }

    // the IDs of ID[][][] to the device again (after editing them on the host)
    void upload_ids()
    {
        std::vector<uint8_t> ids((size_t)(Nx + 1) * (Ny + 1) * (Nz + 1));
        for (size_t q = 0; q < ids.size(); ++q) {
            const short v = ID[0][0][q];
            if (v < 0 || v > 255) throw std::runtime_error("material ID outside 0..255");
            ids[q] = (uint8_t)v;
        }
        cpsfdtd_detail::check(cps_grid_upload_ids(grid_, ids.data()), "IDs");
    }

    void refresh_coefficients()
    {
        if (!aE) { aE = new double[NoMedia]; bE = new double[NoMedia]; aH = new double[NoMedia]; bH = new double[NoMedia]; }
        cpsfdtd_detail::check(cps_grid_coefficients(grid_, aE, bE, aH, bH), "coefficients");
        double **arr[12] = {&cExy, &cEyx, &cEzx, &cExz, &cEzy, &cEyz, &cHxy, &cHyx, &cHzx, &cHxz, &cHzy, &cHyz};
        for (int w = 0; w < 12; ++w) {
            int len = 0;
            cpsfdtd_detail::check(cps_grid_stretch(grid_, w, nullptr, &len), "stretch");
            delete[] *arr[w];
            *arr[w] = new double[len > 0 ? len : 1];
            cpsfdtd_detail::check(cps_grid_stretch(grid_, w, *arr[w], &len), "stretch");
        }
    }

    cps_grid *grid()
    {
        if (!grid_) throw std::runtime_error("the grid exists after InitializeBasicFDTDCoefficients");
        return grid_;
    }

    // hand the device grid to the caller, who destroys it (cps_grid_destroy)
    cps_grid *release_grid()
    {
        cps_grid *g = grid();
        grid_ = nullptr;
        return g;
    }

    double Lx = 0, Ly = 0, Lz = 0;
    double dx = 0, dy = 0, dz = 0;
    double dt = 0;
    int Nx = 0, Ny = 0, Nz = 0;
    short ***ID = nullptr;
    int NoShapes = 0;
    shape *shapes = nullptr;
    bool freespace = false;
    short NoMedia = 0;
    double *epsR = nullptr, *muR = nullptr, *sig = nullptr, *sigM = nullptr;
    double *aE = nullptr, *bE = nullptr, *aH = nullptr, *bH = nullptr;
    double *cExy = nullptr, *cEyx = nullptr, *cEzx = nullptr, *cExz = nullptr, *cEzy = nullptr, *cEyz = nullptr;
    double *cHxy = nullptr, *cHyx = nullptr, *cHzx = nullptr, *cHxz = nullptr, *cHzy = nullptr, *cHyz = nullptr;

private:
    int precision_;
    cps_grid *grid_ = nullptr;
};

// Fields.h:23-45: the six components, host mirrors of the device fields
class Field {
public:
    Field(Structure &sS, const char *smode) : S_(&sS), g_(sS.grid())
    {
        mode = new char[strlen(smode ? smode : "") + 1];
        strcpy(mode, smode ? smode : "");
        xN = sS.Nx + 1; yN = sS.Ny + 1; zN = sS.Nz + 1;
        double ****c[6] = {&Ex, &Ey, &Ez, &Hx, &Hy, &Hz};
        for (int q = 0; q < 6; ++q) *c[q] = cpsfdtd_detail::alloc3<double>(xN, yN, zN, 0.0);
    }
    ~Field()
    {
        for (double ***a : {Ex, Ey, Ez, Hx, Hy, Hz}) cpsfdtd_detail::free3(a);
        delete[] mode;
    }
    Field(const Field &) = delete;
    Field &operator=(const Field &) = delete;

    // device -> Ex..Hz (waits for the enqueued updates)
    void sync_to_host()
    {
        double ***c[6] = {Ex, Ey, Ez, Hx, Hy, Hz};
        for (int q = 0; q < 6; ++q) cpsfdtd_detail::check(cps_field_download(g_, q, c[q][0][0]), "sync_to_host");
    }
    // Ex..Hz -> device
    void sync_to_device()
    {
        double ***c[6] = {Ex, Ey, Ez, Hx, Hy, Hz};
        for (int q = 0; q < 6; ++q) cpsfdtd_detail::check(cps_field_upload(g_, q, c[q][0][0]), "sync_to_device");
    }
    cps_grid *grid() const { return g_; }

    double ***Ex = nullptr, ***Ey = nullptr, ***Ez = nullptr;
    double ***Hx = nullptr, ***Hy = nullptr, ***Hz = nullptr;
    char *mode = nullptr;
    char const *TE_mode = "TE";
    char const *TM_mode = "TM";

private:
    Structure *S_;
    cps_grid *g_;
    int xN = 0, yN = 0, zN = 0;
};

// BasicFDTD.h:8-9
inline void BasicEFieldUpdate(Field &fF, Structure &)
{
    cpsfdtd_detail::check(cps_op_e_bulk(fF.grid()), "BasicEFieldUpdate");
}
inline void BasicHFieldUpdate(Field &fF, Structure &)
{
    cpsfdtd_detail::check(cps_op_h_bulk(fF.grid()), "BasicHFieldUpdate");
}

namespace cpsfdtd_detail {
// CPML.cpp:29-68 and CFS_PML's constructor read the same deck
inline cps_pml_params read_pml(const char *fileName)
{
    LineReader r(fileName);
    cps_pml_params p{};
    r.line(0) >> p.npml[0] >> p.npml[1];
    r.line(1) >> p.npml[2] >> p.npml[3];
    r.line(2) >> p.npml[4] >> p.npml[5];
    r.line(3) >> p.m >> p.malp;
    r.line(4) >> p.kapmax >> p.sig_ratio;
    r.line(5) >> p.alpmax;
    return p;
}
}  // namespace cpsfdtd_detail

// CPML.h:9-38
class CPML {
public:
    CPML(Structure &sS, const char *fileName) : S_(&sS), p_(cpsfdtd_detail::read_pml(fileName)) {}
    void InitializeCPML(Structure &sS)
    {
        cpsfdtd_detail::check(cps_pml_init(sS.grid(), &p_), "InitializeCPML");
        sS.refresh_coefficients();  // kappa folded into the stretched-coordinate arrays
    }
    void UpdateCPMLEFields(Field &fF) { cpsfdtd_detail::check(cps_op_e_pml(fF.grid()), "UpdateCPMLEFields"); }
    void UpdateCPMLHFields(Field &fF) { cpsfdtd_detail::check(cps_op_h_pml(fF.grid()), "UpdateCPMLHFields"); }

private:
    Structure *S_;
    cps_pml_params p_;
};

// CFS_PML.h:27-50: the same CFS-PML, point-list class of the reference
class CFS_PML {
public:
    CFS_PML(Structure &sS, const char *fileName) : p_(cpsfdtd_detail::read_pml(fileName))
    {
        Npmlx1 = p_.npml[0]; Npmlx2 = p_.npml[1]; Npmly1 = p_.npml[2]; Npmly2 = p_.npml[3];
        Npmlz1 = p_.npml[4]; Npmlz2 = p_.npml[5];
        p_order = p_.m; malp = p_.malp; kapmax = p_.kapmax; sig_ratio = p_.sig_ratio; alpmax = p_.alpmax;
        (void)sS;
    }
    void Initialize_PML(Structure &sS)
    {
        cpsfdtd_detail::check(cps_pml_init(sS.grid(), &p_), "Initialize_PML");
        sS.refresh_coefficients();
    }
    void UpdatePMLEFields(Field &fF) { cpsfdtd_detail::check(cps_op_e_pml(fF.grid()), "UpdatePMLEFields"); }
    void UpdatePMLHFields(Field &fF) { cpsfdtd_detail::check(cps_op_h_pml(fF.grid()), "UpdatePMLHFields"); }

    double p_order = 0, kapmax = 0, alpmin = 0, alpmax = 0, malp = 0, sig_ratio = 0, sigmax = 0;
    int Npmlx1 = 0, Npmly1 = 0, Npmlz1 = 0, Npmlx2 = 0, Npmly2 = 0, Npmlz2 = 0;

private:
    cps_pml_params p_;
};

// Drude_Lorentz.h:19-36: deck Drude_Lorentz.cpp:37-94 (frequencies in Hz).
// The default uses the ADE coefficients the discretisation gives; set the
// environment variable CPSFDTD_DL_LITERAL=1 for the reference's literal C1/C5.
class Drude_Lorentz {
public:
    Drude_Lorentz(Structure &sS, const char *fileName)
    {
        cpsfdtd_detail::LineReader r(fileName);
        cps_dl_params p{};
        r.line(0) >> p.nD;
        r.line(1) >> p.nL;
        r.line(2) >> p.sigma;
        r.line(3) >> p.epsInf;
        if (p.nD < 0 || p.nL < 0 || p.nD > CPS_MAX_POLES || p.nL > CPS_MAX_POLES)
            throw std::runtime_error(std::string("bad pole counts in ") + fileName);
        for (int q = 0; q < p.nD; ++q) r.line(4 + q) >> p.fD[q] >> p.gD[q];
        for (int q = 0; q < p.nL; ++q) r.line(4 + p.nD + q) >> p.fL[q] >> p.dL[q] >> p.depsL[q];
        const char *lit = getenv("CPSFDTD_DL_LITERAL");
        p.literal = lit && lit[0] == '1';
        num_of_D_poles = p.nD; num_of_L_poles = p.nL; sigma = p.sigma; epsInf = p.epsInf;
        cpsfdtd_detail::check(cps_dl_init(sS.grid(), &p), "Drude_Lorentz");
    }
    void EFieldUpdate(Field &fF, Structure &) { cpsfdtd_detail::check(cps_op_dl(fF.grid()), "EFieldUpdate"); }

    double sigma = 0, epsInf = 1;
    int num_of_D_poles = 0, num_of_L_poles = 0;
};

// Drude.h:19-35: the single-pole Drude material of the ID-2 cells, deck
// Drude.cpp:29-52 (eps_inf, omega_P and gamma in Hz, sigma); its update
// (Drude.cpp:70-113) is the Drude-Lorentz cell update with Drude.cpp's
// coefficients.  One of Drude and Drude_Lorentz per Structure.
class Drude {
public:
    Drude(Structure &sS, const char *fileName)
    {
        cpsfdtd_detail::LineReader r(fileName);
        cps_drude_params p{};
        r.line(0) >> p.epsInf;
        r.line(1) >> p.omegaP_hz;
        r.line(2) >> p.sigma;
        r.line(3) >> p.gamma_hz;
        epsInf = p.epsInf;
        omegaP = p.omegaP_hz * 2.0 * 3.1415926535897932384626433832795;  // Drude.cpp:40
        sigma = p.sigma;
        gamma = p.gamma_hz * 2.0 * 3.1415926535897932384626433832795;  // Drude.cpp:49
        cpsfdtd_detail::check(cps_drude_init(sS.grid(), &p), "Drude");
    }
    void EFieldUpdate(Field &fF, Structure &) { cpsfdtd_detail::check(cps_op_dl(fF.grid()), "EFieldUpdate"); }

    double epsInf = 1, omegaP = 0, sigma = 0, gamma = 0;
};

// ThreeLevel.h:23-48: deck ThreeLevel.cpp:37-84 (distribution, count, i and j
// ranges, lambda_a, lambda_b, gamma_a, gamma_b, t20, t21, t10, N_0, N_1); the
// sites are the cells of ID 5 (the reference's "cells" placement).  The
// default uses the Lorentz-oscillator coefficients; CPSFDTD_THREE_LITERAL=1
// takes the reference's as written (its polarisation diverges).
class ThreeLevel {
public:
    ThreeLevel(Structure &sS, const char *fileName)
    {
        cpsfdtd_detail::LineReader r(fileName);
        cps_three_params p{};
        r.line(0) >> distri;
        r.line(1) >> NumSources;
        r.line(2) >> i1 >> i2;
        r.line(3) >> j1 >> j2;
        r.line(4) >> p.lambda_a;
        r.line(5) >> p.lambda_b;
        r.line(6) >> p.gamma_a;
        r.line(7) >> p.gamma_b;
        r.line(8) >> p.t20;
        r.line(9) >> p.t21;
        r.line(10) >> p.t10;
        r.line(11) >> p.N_0;
        r.line(12) >> p.N_1;
        p.gain_id = 5;
        const char *lit = getenv("CPSFDTD_THREE_LITERAL");
        p.literal = lit && lit[0] == '1';
        lambda_a = p.lambda_a; lambda_b = p.lambda_b; gamma_a = p.gamma_a; gamma_b = p.gamma_b;
        t20 = p.t20; t21 = p.t21; t10 = p.t10; N_0 = p.N_0; N_1 = p.N_1;
        omega_a = 2.0 * 3.1415926535897932384626433832795 * 2.99792458E8 / lambda_a;  // ThreeLevel.cpp:96
        omega_b = 2.0 * 3.1415926535897932384626433832795 * 2.99792458E8 / lambda_b;
        g_ = sS.grid();
        cpsfdtd_detail::check(cps_three_init(g_, &p), "ThreeLevel");
    }
    void UpdatePolarizationDensities(Field &fF)
    {
        cpsfdtd_detail::check(cps_op_three_polarization(fF.grid()), "UpdatePolarizationDensities");
    }
    void UpdateElectricField(Field &fF) { cpsfdtd_detail::check(cps_op_three_efield(fF.grid()), "UpdateElectricField"); }
    void UpdateStatesPopulations(Field &fF)
    {
        cpsfdtd_detail::check(cps_op_three_populations(fF.grid()), "UpdateStatesPopulations");
    }
    // N0 N1 N2 per site (cells in (i,j,k) order): the reference's N0/N1/N2 arrays
    std::vector<double> populations() const
    {
        int64_t n = 0;
        cpsfdtd_detail::check(cps_three_populations(g_, nullptr, &n), "populations");
        std::vector<double> out((size_t)n * 3);
        cpsfdtd_detail::check(cps_three_populations(g_, out.data(), &n), "populations");
        return out;
    }

    std::string distri;
    int NumSources = 0, i1 = 0, i2 = 0, j1 = 0, j2 = 0;
    double N_0 = 0, N_1 = 0;
    double gamma_a = 0, gamma_b = 0, lambda_a = 0, lambda_b = 0, omega_a = 0, omega_b = 0;
    double t20 = 0, t21 = 0, t10 = 0;

private:
    cps_grid *g_ = nullptr;
};

// FourLevelLaser.h:8-52: deck FourLevelLaser.cpp:37-93; gain sites are the
// cells of ID 5 (the reference's "cells" placement); an extra 15th line, when
// present, is a pump rate in 1/s (no reference counterpart)
class FourLevelLaser {
public:
    FourLevelLaser(Structure &sS, const char *fileName)
    {
        cpsfdtd_detail::LineReader r(fileName);
        std::string dist;
        r.line(0) >> dist;
        strncpy(distri, dist.c_str(), sizeof(distri) - 1);
        r.line(1) >> NumSources;
        r.line(2) >> i1 >> i2;
        r.line(3) >> j1 >> j2;
        double *v[10] = {&lambda_b, &lambda_a, &gamma_a, &gamma_b, &t30, &t32, &t21, &t10, &N_0, &N_1};
        for (int q = 0; q < 10; ++q) r.line(4 + q) >> *v[q];
        double pump = 0;
        r.line(14) >> pump;
        cps_gain_params p{5, lambda_a, lambda_b, gamma_a, gamma_b, t30, t32, t21, t10, N_0, pump};
        cpsfdtd_detail::check(cps_gain_init(sS.grid(), &p), "FourLevelLaser");
        g_ = sS.grid();
    }
    void UpdatePolarizationDensities(Field &fF)
    {
        cpsfdtd_detail::check(cps_op_gain_polarization(fF.grid()), "UpdatePolarizationDensities");
    }
    void UpdateElectricField(Field &fF) { cpsfdtd_detail::check(cps_op_gain_efield(fF.grid()), "UpdateElectricField"); }
    void UpdateStatesPopulations(Field &fF)
    {
        cpsfdtd_detail::check(cps_op_gain_populations(fF.grid()), "UpdateStatesPopulations");
    }
    // FP64 N0..N3 of every gain cell, [cell][4], cells in (i, j, k) order
    std::vector<double> populations()
    {
        int64_t n = 0;
        cpsfdtd_detail::check(cps_gain_populations(g_, nullptr, &n), "populations");
        std::vector<double> out((size_t)n * 4);
        cpsfdtd_detail::check(cps_gain_populations(g_, out.data(), &n), "populations");
        return out;
    }

    int NumSources = 0;
    int i1 = 0, i2 = 0, j1 = 0, j2 = 0;
    double N_0 = 0, N_1 = 0;
    double gamma_a = 0, gamma_b = 0, lambda_a = 0, lambda_b = 0;
    double t30 = 0, t32 = 0, t21 = 0, t10 = 0;
    char distri[40] = {0};

private:
    cps_grid *g_ = nullptr;
};

// TF_SF.h:17-93: deck TF_SF.cpp:35-97, 898-907.  The beam-centre plane k0 is
// never set by the reference (TF_SF.h:65); here it is an optional fourth value
// on the source-position line, default Nz/2.
class TF_SF {
public:
    TF_SF(Structure &sS, const char *fileName)
    {
        cpsfdtd_detail::LineReader r(fileName);
        double z0deck = 0, theta = 0, phi = 0, psi = 0;
        r.line(0) >> lambda;
        r.line(1) >> dlambda;
        r.line(2) >> w0 >> z0deck;
        {
            std::istringstream l3 = r.line(3);
            l3 >> xs >> ys >> zs;
            int kk = 0;
            k0 = (l3 >> kk) ? kk : sS.Nz / 2;
        }
        r.line(4) >> theta >> phi;
        r.line(5) >> E0 >> psi;
        r.line(6) >> nTFSFx1 >> nTFSFx2;
        r.line(7) >> nTFSFy1 >> nTFSFy2;
        r.line(8) >> nTFSFz1 >> nTFSFz2;
        int cw = 0;
        r.line(9) >> Nt;
        r.line(10) >> cw;
        cwmode = cw != 0;
        i0 = (int)(xs / sS.dx);
        j0 = (int)(ys / sS.dy);
        z0 = zs / sS.dz;  // TF_SF.cpp:57 replaces the deck's waist offset by zs/dz
        theta_inc = theta; phi_inc = phi; psi_E = psi;
        nu = 2.99792458E8 / lambda;
        T = 1.0 / nu;
        cps_tfsf_params p{lambda, dlambda, w0, z0, i0, j0, k0, theta, phi, E0, psi,
                          {nTFSFx1, nTFSFx2, nTFSFy1, nTFSFy2, nTFSFz1, nTFSFz2}, Nt, cw};
        g_ = sS.grid();
        cpsfdtd_detail::check(cps_tfsf_init(g_, &p), "TF_SF");
        tab_.assign(2 * (size_t)(Nt + 1), 0.0);
        cpsfdtd_detail::check(cps_tfsf_get_tables(g_, Nt + 1, tab_.data(), tab_.data() + Nt + 1), "TF_SF tables");
        Einc = tab_.data();
        Hinc = tab_.data() + Nt + 1;
    }
    TF_SF(const TF_SF &) = delete;
    TF_SF &operator=(const TF_SF &) = delete;

    void UpdateEField(int n, Field &fF, Structure &) { e(n, fF, CPS_FACE_ALL); }
    void UpdateHField(int n, Field &fF, Structure &) { h(n, fF, CPS_FACE_ALL); }
    void x1UpdateEField(int n, Field &fF, Structure &) { e(n, fF, CPS_FACE_X1); }
    void x1UpdateHField(int n, Field &fF, Structure &) { h(n, fF, CPS_FACE_X1); }
    void x2UpdateEField(int n, Field &fF, Structure &) { e(n, fF, CPS_FACE_X2); }
    void x2UpdateHField(int n, Field &fF, Structure &) { h(n, fF, CPS_FACE_X2); }
    void y1UpdateEField(int n, Field &fF, Structure &) { e(n, fF, CPS_FACE_Y1); }
    void y1UpdateHField(int n, Field &fF, Structure &) { h(n, fF, CPS_FACE_Y1); }
    void y2UpdateEField(int n, Field &fF, Structure &) { e(n, fF, CPS_FACE_Y2); }
    void y2UpdateHField(int n, Field &fF, Structure &) { h(n, fF, CPS_FACE_Y2); }
    void z1UpdateEField(int n, Field &fF, Structure &) { e(n, fF, CPS_FACE_Z1); }
    void z1UpdateHField(int n, Field &fF, Structure &) { h(n, fF, CPS_FACE_Z1); }
    void z2UpdateEField(int n, Field &fF, Structure &) { e(n, fF, CPS_FACE_Z2); }
    void z2UpdateHField(int n, Field &fF, Structure &) { h(n, fF, CPS_FACE_Z2); }

    // TF_SF.cpp:966-986: linear interpolation in the incident tables
    double Einc_onPoint(double retarded) const { return lookup(Einc, retarded); }
    double Hinc_onPoint(double retarded) const { return lookup(Hinc, retarded); }

    double theta_inc = 0, phi_inc = 0;   // degrees here (the reference converts them to radians)
    double psi_E = 0, E0 = 0;
    int nTFSFx1 = 0, nTFSFx2 = 0, nTFSFy1 = 0, nTFSFy2 = 0, nTFSFz1 = 0, nTFSFz2 = 0;
    double *Einc = nullptr, *Hinc = nullptr;
    double lambda = 0, dlambda = 0, nu = 0, T = 0;
    int Nt = 0;
    double w0 = 0, z0 = 0;
    double xs = 0, ys = 0, zs = 0;
    int i0 = 0, j0 = 0, k0 = 0;
    bool cwmode = false;

private:
    void e(int n, Field &fF, uint32_t mask) { cpsfdtd_detail::check(cps_op_tfsf_e(fF.grid(), n, mask), "TF/SF E"); }
    void h(int n, Field &fF, uint32_t mask) { cpsfdtd_detail::check(cps_op_tfsf_h(fF.grid(), n, mask), "TF/SF H"); }
    double lookup(const double *tab, double retarded) const
    {
        if (retarded <= 0) return 0.0;
        const long long m = (long long)retarded;
        const double resid = retarded - (double)m;
        const double a = m <= Nt ? tab[m] : 0.0, b = m + 1 <= Nt ? tab[m + 1] : 0.0;
        return (1.0 - resid) * a + resid * b;
    }
    cps_grid *g_ = nullptr;
    std::vector<double> tab_;
};

// OutImage.h:22-45 without a display: the reference draws through CImg and
// an X11 window; here plot_save and structure_plot_save write the same PNG
// files (OutImage.cpp:140-216) and plot() has nothing to show.
class OutImage {
public:
    OutImage(int N_x, int N_y, int save_modulus, double cmap_min, double cmap_max, const char *file_name_base)
        : savemodulus(save_modulus > 0 ? save_modulus : 1), Nx(N_x), Ny(N_y), cmapmin(cmap_min), cmapmax(cmap_max),
          filenamebase(file_name_base ? file_name_base : "")
    {
        cmapmid = (cmapmax + cmapmin) / 2.0;
        cmapthird = (cmapmax + cmapmin) / 3.0;
        cmap2third = (cmapmax + cmapthird) / 2.0;
        static const short table[10][3] = {{254, 254, 254}, {254, 0, 0},   {0, 0, 254},   {0, 254, 0},   {0, 0, 0},
                                           {254, 254, 0},   {0, 254, 254}, {254, 0, 254}, {127, 0, 254}, {0, 127, 254}};
        for (int q = 0; q < color_table_length; ++q)
            for (int c = 0; c < 3; ++c) color_table[q][c] = table[q][c];
    }
    void plot_save(double **dD, int time_step)
    {
        if (time_step % savemodulus != 0) return;
        std::vector<double> v((size_t)Nx * Ny);
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j) v[(size_t)i * Ny + j] = dD[i][j];
        char name[512];
        snprintf(name, sizeof(name), "%s%06d.png", filenamebase.c_str(), time_step / savemodulus);
        cpsfdtd_detail::check(cps_image_png(name, Nx, Ny, v.data(), cmapmin, cmapmax), "plot_save");
    }
    void structure_plot_save(short **dD)
    {
        std::vector<uint8_t> rgb((size_t)Nx * Ny * 3);
        for (int i = 0; i < Nx; ++i)
            for (int j = 0; j < Ny; ++j) {
                const int id = dD[i][j];
                if (id < 0 || id >= color_table_length) throw std::runtime_error("structure_plot_save: ID without a colour");
                for (int c = 0; c < 3; ++c) rgb[((size_t)j * Nx + i) * 3 + c] = (uint8_t)color_table[id][c];
            }
        const std::string name = filenamebase + "_structure.png";
        cpsfdtd_detail::check(cps_png_rgb(name.c_str(), Nx, Ny, rgb.data()), "structure_plot_save");
    }
    void plot() {}
    void plot(double **, int) {}

    int savemodulus, Nx, Ny, color_table_length = 10;
    double cmapmin, cmapmax, cmapmid, cmapthird, cmap2third;
    short color_table[10][3];
    std::string filenamebase;
};

// Ports.h:20-27
struct Port_Points {
    int i, j, k;
    double Ex, Ey, Ez;
    double Hx, Hy, Hz;
    unsigned short id;
};

namespace cpsfdtd_detail {
// sampling and the text writers shared by both port kinds (Ports.cpp:88-189, 342-522)
class PortBase {
public:
    void Update_Fields_on_Port(Field &fF)
    {
        cpsfdtd_detail::check(cps_op_port_sample(fF.grid(), pid_, ++n_), "Update_Fields_on_Port");
        fresh_ = false;
    }
    void Export_E_onPort(const char *fileName) { std::ofstream o(fileName); Export_E_onPort(o); }
    void Export_E_onPort(std::ofstream &o)
    {
        pull();
        for (int q = 0; q < Num_of_Port_Points; ++q)
            o << port_point[q].Ex << "\t" << port_point[q].Ey << "\t" << port_point[q].Ez << std::endl;
    }
    void Export_Ex_onPort(const char *fileName) { std::ofstream o(fileName); row(o, 0, false); }
    void Export_Ex_onPort(std::ofstream &o) { row(o, 0, true); }
    void Export_Ey_onPort(const char *fileName) { std::ofstream o(fileName); row(o, 1, false); }
    void Export_Ey_onPort(std::ofstream &o) { row(o, 1, true); }
    void Export_Ez_onPort(const char *fileName) { std::ofstream o(fileName); row(o, 2, false); }
    void Export_Ez_onPort(std::ofstream &o) { row(o, 2, true); }
    void Export_EIntensity_onPort(const char *fileName) { std::ofstream o(fileName); row(o, 3, false); }
    void Export_EIntensity_onPort(std::ofstream &o) { row(o, 3, true); }

    Port_Points *port_point = nullptr;
    int Num_of_Port_Points = 0;

protected:
    void attach(Structure &sS, std::vector<int32_t> ijk)
    {
        Num_of_Port_Points = (int)(ijk.size() / 3);
        pts_.assign(Num_of_Port_Points, Port_Points{});
        for (int q = 0; q < Num_of_Port_Points; ++q) {
            Port_Points &p = pts_[q];
            p.i = ijk[3 * q]; p.j = ijk[3 * q + 1]; p.k = ijk[3 * q + 2];
            p.id = (unsigned short)sS.ID[p.i][p.j][p.k];
        }
        port_point = pts_.data();
        g_ = sS.grid();
        cpsfdtd_detail::check(cps_port_add(g_, Num_of_Port_Points, ijk.data(), &pid_), "port");
    }
    // the last sample of the device ring into port_point
    void pull()
    {
        if (fresh_) return;
        std::vector<double> v((size_t)Num_of_Port_Points * 6);
        if (Num_of_Port_Points) cpsfdtd_detail::check(cps_port_read(g_, pid_, v.data()), "port read");
        for (int q = 0; q < Num_of_Port_Points; ++q) {
            Port_Points &p = pts_[q];
            p.Ex = v[6 * q]; p.Ey = v[6 * q + 1]; p.Ez = v[6 * q + 2];
            p.Hx = v[6 * q + 3]; p.Hy = v[6 * q + 4]; p.Hz = v[6 * q + 5];
        }
        fresh_ = true;
    }
    void row(std::ostream &o, int what, bool newline)
    {
        pull();
        for (int q = 0; q < Num_of_Port_Points; ++q) {
            const Port_Points &p = pts_[q];
            const double v = what == 0 ? p.Ex : what == 1 ? p.Ey : what == 2 ? p.Ez
                           : p.Ex * p.Ex + p.Ey * p.Ey + p.Ez * p.Ez;
            o << v << "\t";
        }
        if (newline) o << std::endl;
    }
    cps_grid *g_ = nullptr;
    int32_t pid_ = -1;
    int32_t n_ = 0;
    bool fresh_ = true;
    std::vector<Port_Points> pts_;
};
}  // namespace cpsfdtd_detail

// Ports.h:29-57: deck Ports.cpp:33-58
class SphericalPort : public cpsfdtd_detail::PortBase {
public:
    SphericalPort(Structure &sS, const char *fileName) : dx_(sS.dx), dy_(sS.dy), dz_(sS.dz)
    {
        cpsfdtd_detail::LineReader rd(fileName);
        rd.line(0) >> r;
        rd.line(1) >> xc >> yc >> zc;
        rd.line(2) >> theta1 >> theta2;
        rd.line(3) >> phi1 >> phi2;
        int32_t cnt = 0;
        cpsfdtd_detail::check(cps_port_points_spherical(sS.Nx, sS.Ny, sS.Nz, sS.dx, sS.dy, sS.dz, r, xc, yc, zc, theta1,
                                                        theta2, phi1, phi2, &cnt, nullptr), "SphericalPort");
        std::vector<int32_t> ijk(3 * (size_t)cnt);
        cpsfdtd_detail::check(cps_port_points_spherical(sS.Nx, sS.Ny, sS.Nz, sS.dx, sS.dy, sS.dz, r, xc, yc, zc, theta1,
                                                        theta2, phi1, phi2, &cnt, ijk.data()), "SphericalPort");
        attach(sS, ijk);
    }
    // Ports.cpp:101-109
    void Export_Port(const char *fileName)
    {
        std::ofstream o(fileName);
        o << xc / dx_ << "\t" << yc / dy_ << "\t" << zc / dz_ << std::endl;
        for (int q = 0; q < Num_of_Port_Points; ++q)
            o << port_point[q].i << "\t" << port_point[q].j << "\t" << port_point[q].k << std::endl;
    }
    double r = 0, xc = 0, yc = 0, zc = 0, theta1 = 0, theta2 = 0, phi1 = 0, phi2 = 0;

private:
    double dx_, dy_, dz_;
};

// Ports.h:59-90: deck Ports.cpp:206-237
class PlainPort : public cpsfdtd_detail::PortBase {
public:
    PlainPort(Structure &sS, const char *fileName)
    {
        cpsfdtd_detail::LineReader rd(fileName);
        rd.line(0) >> normal_direction;
        rd.line(1) >> position;
        rd.line(2) >> w1 >> w2;
        rd.line(3) >> h1 >> h2;
        int32_t cnt = 0;
        cpsfdtd_detail::check(cps_port_points_plain(sS.Nx, sS.Ny, sS.Nz, sS.dx, sS.dy, sS.dz, normal_direction,
                                                    position, w1, w2, h1, h2, &cnt, nullptr), "PlainPort");
        std::vector<int32_t> ijk(3 * (size_t)cnt);
        cpsfdtd_detail::check(cps_port_points_plain(sS.Nx, sS.Ny, sS.Nz, sS.dx, sS.dy, sS.dz, normal_direction,
                                                    position, w1, w2, h1, h2, &cnt, ijk.data()), "PlainPort");
        attach(sS, ijk);
    }
    void Export_Port(const char *fileName)
    {
        std::ofstream o(fileName);
        for (int q = 0; q < Num_of_Port_Points; ++q)
            o << port_point[q].i << "\t" << port_point[q].j << "\t" << port_point[q].k << std::endl;
    }
    // the IDs in one row (the reference breaks rows at the port width)
    void Export_ID_onPort(const char *fileName)
    {
        std::ofstream o(fileName);
        for (int q = 0; q < Num_of_Port_Points; ++q) o << port_point[q].id << "\t";
    }
    char normal_direction = 'z';
    double position = 0, w1 = 0, w2 = 0, h1 = 0, h2 = 0;
};
