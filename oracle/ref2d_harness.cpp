// ref2d_harness.cpp -- known-answer generator for the Drude-Lorentz and
// four-level-gain recursions: runs a 2-D TE problem through the reference's
// own Drude_Lorentz and FourLevelLaser classes (compiled unmodified from the
// reference tree against the 2-D stand-in headers in oracle/shim2d/) and dumps
// Ex, Ey, Hz.  oracle.c's orc2d_run runs the same problem through the oracle's
// per-cell recursions; the two must agree to 1e-12.
//
// TEST INFRASTRUCTURE ONLY.
//
// Usage: ref2d_harness <deck_dir> <out_dir>
//   params2d.txt : nx ny dx dy dt nsteps si sj use_dl use_gain [dl_literal [use_drude [use_three]]]
//   With dl_literal 0 the constructed Drude_Lorentz gets C1 and C5 overwritten
//   with the values the ADE discretisation gives (Drude_Lorentz.cpp:96 has the
//   wrong sign on sigma*dt + dt*sum(beta), :106 lacks a factor dt); the update
//   routine itself runs unmodified.
//   media2d.txt  : n, then n lines epsR muR sig sigM
//   ids2d.bin    : uint8 [nx+1][ny+1], j fastest
//   wave.bin     : nsteps doubles, added to Hz[si][sj] after each H update
//   DrudeLorentz.txt / FourLevelLaser.txt / Drude.txt : reference-format decks;
//   use_drude runs the single-pole Drude class (Drude.cpp) as the E update;
//   use_three runs the three-level gain class (ThreeLevel.cpp, deck ThreeLevel.txt)
#include "stdafx.h"
#include "Constants.h"
#include "Structure.h"
#include "Fields.h"
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <new>
#include <sstream>
#include <string>
#include <vector>
#include <unistd.h>

// The coefficient repair below writes private Drude_Lorentz members; the
// access change is confined to this class definition in this file.
#define private public
#include "Drude_Lorentz.h"
#undef private
#include "FourLevelLaser.h"
#include "Drude.h"
#include "ThreeLevel.h"

void *operator new(std::size_t n) { void *p = calloc(n ? n : 1, 1); if (!p) throw std::bad_alloc(); return p; }
void *operator new[](std::size_t n) { void *p = calloc(n ? n : 1, 1); if (!p) throw std::bad_alloc(); return p; }
void operator delete(void *p) noexcept { free(p); }
void operator delete[](void *p) noexcept { free(p); }
void operator delete(void *p, std::size_t) noexcept { free(p); }
void operator delete[](void *p, std::size_t) noexcept { free(p); }

static void die(const char *m) { fprintf(stderr, "ref2d_harness: %s\n", m); _exit(2); }

static double **grid2(int nx, int ny)
{
    double **a = new double *[nx + 1];
    for (int i = 0; i <= nx; ++i) a[i] = new double[ny + 1];
    return a;
}

int main(int argc, char **argv)
{
    if (argc < 3) die("usage");
    const std::string dir = std::string(argv[1]) + "/", out = std::string(argv[2]) + "/";
    int nx, ny, nsteps, si, sj, use_dl, use_gain, dl_literal = 1, use_drude = 0, use_three = 0;
    double dx, dy, dt;
    {
        std::ifstream p(dir + "params2d.txt");
        if (!(p >> nx >> ny >> dx >> dy >> dt >> nsteps >> si >> sj >> use_dl >> use_gain)) die("params");
        if (!(p >> dl_literal)) dl_literal = 1;
        if (!(p >> use_drude)) use_drude = 0;
        if (!(p >> use_three)) use_three = 0;
    }
    int nm;
    std::ifstream mi(dir + "media2d.txt");
    if (!(mi >> nm)) die("media");
    std::vector<double> epsR(nm), muR(nm), sig(nm), sigM(nm);
    for (int m = 0; m < nm; ++m) mi >> epsR[m] >> muR[m] >> sig[m] >> sigM[m];

    Structure S;
    S.Nx = nx; S.Ny = ny; S.dx = dx; S.dy = dy; S.dt = dt;
    S.ID = new short *[nx + 1];
    std::vector<unsigned char> ids((size_t)(nx + 1) * (ny + 1));
    {
        FILE *f = fopen((dir + "ids2d.bin").c_str(), "rb");
        if (!f || fread(ids.data(), 1, ids.size(), f) != ids.size()) die("ids");
        fclose(f);
    }
    for (int i = 0; i <= nx; ++i) {
        S.ID[i] = new short[ny + 1];
        for (int j = 0; j <= ny; ++j) S.ID[i][j] = ids[(size_t)i * (ny + 1) + j];
    }
    S.aE = new double[nm]; S.bE = new double[nm]; S.aH = new double[nm]; S.bH = new double[nm];
    for (int m = 0; m < nm; ++m) {  // the formulas of Structure.cpp:446-451
        S.aE[m] = (2.0 * eps0 * epsR[m] - sig[m] * dt) / (2.0 * eps0 * epsR[m] + sig[m] * dt);
        S.bE[m] = (2.0 * dt) / (2.0 * eps0 * epsR[m] + sig[m] * dt);
        S.aH[m] = (2.0 * mu0 * muR[m] - sigM[m] * dt) / (2.0 * mu0 * muR[m] + sigM[m] * dt);
        S.bH[m] = (2.0 * dt) / (2.0 * mu0 * muR[m] + sigM[m] * dt);
    }
    const double cx = 1.0 / dx, cy = 1.0 / dy;
    S.cExy = new double[ny];
    S.cEyx = new double[nx];
    for (int j = 0; j < ny; ++j) S.cExy[j] = cy;
    for (int i = 0; i < nx; ++i) S.cEyx[i] = cx;
    Field F;
    F.Ex = grid2(nx, ny); F.Ey = grid2(nx, ny); F.Ez = grid2(nx, ny); F.Hz = grid2(nx, ny);
    std::vector<double> wave(nsteps);
    {
        FILE *f = fopen((dir + "wave.bin").c_str(), "rb");
        if (!f || fread(wave.data(), sizeof(double), nsteps, f) != (size_t)nsteps) die("wave");
        fclose(f);
    }
    std::string dlf = dir + "DrudeLorentz.txt", glf = dir + "FourLevelLaser.txt", drf = dir + "Drude.txt";
    std::vector<char> dln(dlf.begin(), dlf.end()), gln(glf.begin(), glf.end()), drn(drf.begin(), drf.end());
    dln.push_back(0); gln.push_back(0); drn.push_back(0);
    Drude *DR = use_drude ? new Drude(S, drn.data()) : nullptr;
    std::string tlf = dir + "ThreeLevel.txt";
    std::vector<char> tln(tlf.begin(), tlf.end());
    tln.push_back(0);
    ThreeLevel *TL = use_three ? new ThreeLevel(S, tln.data()) : nullptr;
    Drude_Lorentz *DL = use_dl ? new Drude_Lorentz(S, dln.data()) : nullptr;
    FourLevelLaser *FL = use_gain ? new FourLevelLaser(S, gln.data()) : nullptr;
    if (DL && !dl_literal) {
        DL->C1 = (2.0 * eps0 * DL->epsInf - DL->sigma * dt - dt * DL->temp1) / DL->denominator;
        for (int p = 0; p < DL->num_of_L_poles; ++p) DL->C5[p] = (1.0 + DL->alpha[p]) * dt / DL->denominator;
    }

    for (int n = 0; n < nsteps; ++n) {
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const int id = S.ID[i][j];
                F.Hz[i][j] = S.aH[id] * F.Hz[i][j] + S.bH[id] * (F.Ex[i][j + 1] - F.Ex[i][j]) * cy - S.bH[id] * (F.Ey[i + 1][j] - F.Ey[i][j]) * cx;
            }
        F.Hz[si][sj] = F.Hz[si][sj] + wave[n];
        if (DR) {
            DR->EFieldUpdate(F, S);
        } else if (DL) {
            DL->EFieldUpdate(F, S);
        } else {
            for (int i = 1; i < nx; ++i)
                for (int j = 1; j < ny; ++j) {
                    const int id = S.ID[i][j];
                    if (id == 4) { F.Ex[i][j] = 0.0; F.Ey[i][j] = 0.0; }
                    else {
                        F.Ex[i][j] = S.aE[id] * F.Ex[i][j] + S.bE[id] * (F.Hz[i][j] - F.Hz[i][j - 1]) * cy;
                        F.Ey[i][j] = S.aE[id] * F.Ey[i][j] - S.bE[id] * (F.Hz[i][j] - F.Hz[i - 1][j]) * cx;
                    }
                }
        }
        if (FL) {
            FL->UpdatePolarizationDensities(F);
            FL->UpdateElectricField(F);
            FL->UpdateStatesPopulations(F);
        }
        if (TL) {
            TL->UpdatePolarizationDensities(F);
            TL->UpdateElectricField(F);
            TL->UpdateStatesPopulations(F);
        }
    }
    std::vector<double> buf((size_t)(nx + 1) * (ny + 1));
    double **arr[3] = {F.Ex, F.Ey, F.Hz};
    const char *names[3] = {"Ex2d.bin", "Ey2d.bin", "Hz2d.bin"};
    for (int a = 0; a < 3; ++a) {
        size_t q = 0;
        for (int i = 0; i <= nx; ++i)
            for (int j = 0; j <= ny; ++j) buf[q++] = arr[a][i][j];
        FILE *f = fopen((out + names[a]).c_str(), "wb");
        if (!f || fwrite(buf.data(), sizeof(double), buf.size(), f) != buf.size()) die("write");
        fclose(f);
    }
    fflush(stdout);
    _exit(0);
}
