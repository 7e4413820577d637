// ref_harness.cpp -- drives the reference's own 3-D code (Structure, Field,
// BasicFDTD, CPML, TF_SF, Ports; compiled in place from the reference tree by
// oracle/Makefile) through a time-stepping loop and dumps the results.
//
// TEST INFRASTRUCTURE ONLY: this is the parity pin for the oracle restatement
// and the CPU baseline of bench.py --impl reference.  It is never linked into
// the product.
//
// Usage: ref_harness <deck_dir> <out_dir>
//   <deck_dir>/harness.txt lists what to build, one directive per line:
//     nsteps N | n0 N | pml FILE | tfsf FILE K0 | ids FILE | dl FILE [LITERAL] | gain FILE
//     source COMP I J K WAVEFILE NWAVE | plainport FILE | sphericalport FILE
//     record_ports 0/1 | bench WARMUP TIMED | threads N
//   material.txt and structure.txt are read by the reference's Structure.
//
// Departures from a literal run of the reference, each forced by undefined
// behaviour in it:
//   * every operator new returns zeroed memory, so members the reference never
//     sets read as zero (the extra port point at Ports.cpp:74,238,259,280; the
//     TFSF_point members its x-face H loops read, TF_SF.cpp:1244-1251);
//   * CPML::H_pml_Coef leaves b/c[npml-1] unset (CPML.cpp:210); they are
//     recomputed here with the formula of the other entries;
//   * TF_SF::k0 is never assigned (TF_SF.h:65); the object is constructed on
//     storage whose k0 already holds the deck's beam-centre plane;
//   * the CPML object is never destroyed (its destructor overruns, CPML.cpp:106)
//     and the harness ends with _exit.
// The 3-D Drude-Lorentz and gain updates are absent from the reference; they
// come from the oracle's per-cell recursions (cells.h), applied to the
// reference's own field arrays.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <new>
#include <sstream>
#include <string>
#include <vector>
#include <unistd.h>
#include <omp.h>

#include "stdafx.h"
#include "Constants.h"
#include "Structure.h"
#include "Fields.h"
#include "BasicFDTD.h"
#include "Ports.h"
// The harness reads and repairs private CPML/TF_SF members (see above); the
// access change is confined to these two class definitions in this file.
#define private public
#include "CPML.h"
#include "TF_SF.h"
#undef private

#include "cells.h"

void *operator new(std::size_t n) { void *p = calloc(n ? n : 1, 1); if (!p) throw std::bad_alloc(); return p; }
void *operator new[](std::size_t n) { void *p = calloc(n ? n : 1, 1); if (!p) throw std::bad_alloc(); return p; }
void operator delete(void *p) noexcept { free(p); }
void operator delete[](void *p) noexcept { free(p); }
void operator delete(void *p, std::size_t) noexcept { free(p); }
void operator delete[](void *p, std::size_t) noexcept { free(p); }

namespace {

struct Source { int comp, i, j, k; std::vector<double> wave; };

double ***field_of(Field &F, int c)
{
    double ***a[6] = {F.Ex, F.Ey, F.Ez, F.Hx, F.Hy, F.Hz};
    return a[c];
}

void die(const char *msg)
{
    fprintf(stderr, "ref_harness: %s\n", msg);
    fflush(stderr);
    _exit(2);
}

std::vector<double> read_doubles(const std::string &path, size_t n)
{
    std::vector<double> v(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f || fread(v.data(), sizeof(double), n, f) != n) die(("cannot read " + path).c_str());
    fclose(f);
    return v;
}

void write_raw(const std::string &path, const void *p, size_t bytes)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f || fwrite(p, 1, bytes, f) != bytes) die(("cannot write " + path).c_str());
    fclose(f);
}

// b/c of H layer npml-1 with the formula of CPML.cpp:191-223
void fill_last_h(double *b, double *c, bool first, int np, double dt, double del, double m,
                 double ma, double sigmax, double kapmax, double alpmax)
{
    const int i = np;  // 1-based index of the last layer
    double ps, pa;
    if (first) { ps = pow(((np - i + 0.5) / np), m); pa = pow(((i - 0.5) / np), ma); }
    else { ps = pow(((i - 0.5) / np), m); pa = pow(((np - i + 0.5) / np), ma); }
    const double sigma = sigmax * ps, kappa = 1.0 + (kapmax - 1.0) * ps, alpha = alpmax * pa;
    b[np - 1] = exp(-(sigma / kappa + alpha) * dt / eps0);
    if ((sigma == 0.0) && (alpha == 0.0)) c[np - 1] = 0.0;
    else c[np - 1] = sigma * (b[np - 1] - 1.0) / (sigma + kappa * alpha) / kappa / del;
}

// Drude-Lorentz deck in the layout Drude_Lorentz.cpp:37-94 parses
void read_dl(const std::string &path, double &sigma, double &epsInf, int &nD, std::vector<double> &fD,
             std::vector<double> &gD, int &nL, std::vector<double> &fL, std::vector<double> &dL,
             std::vector<double> &de)
{
    std::ifstream in(path);
    if (!in) die("cannot open dl deck");
    std::string line;
    std::istringstream iss;
    auto next = [&]() { if (!std::getline(in, line)) die("short dl deck"); iss.clear(); iss.str(line); };
    next(); iss >> nD; next(); iss >> nL; next(); iss >> sigma; next(); iss >> epsInf;
    fD.resize(nD); gD.resize(nD); fL.resize(nL); dL.resize(nL); de.resize(nL);
    for (int p = 0; p < nD; ++p) { next(); iss >> fD[p] >> gD[p]; }
    for (int p = 0; p < nL; ++p) { next(); iss >> fL[p] >> dL[p] >> de[p]; }
}

// Gain deck in the layout FourLevelLaser.cpp:37-93 parses, plus a 15th line
// with the pump rate (read as 0 when absent).
void read_gain(const std::string &path, double v[10])
{
    std::ifstream in(path);
    if (!in) die("cannot open gain deck");
    std::string line;
    std::vector<std::string> lines;
    while (std::getline(in, line)) lines.push_back(line);
    if (lines.size() < 14) die("short gain deck");
    auto num = [&](size_t l) { std::istringstream s(lines[l]); double x = 0; s >> x; return x; };
    // lambda_b(4) lambda_a(5) gamma_a(6) gamma_b(7) t30(8) t32(9) t21(10) t10(11) N_0(12)
    v[0] = num(5); v[1] = num(4); v[2] = num(6); v[3] = num(7);
    v[4] = num(8); v[5] = num(9); v[6] = num(10); v[7] = num(11); v[8] = num(12);
    v[9] = lines.size() > 14 ? num(14) : 0.0;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 3) die("usage: ref_harness <deck_dir> <out_dir>");
    const std::string dir = std::string(argv[1]) + "/", out = std::string(argv[2]) + "/";
    int nsteps = 0, n0 = 1, record_ports = 0, warm = -1, timed = 0, threads = 0;
    std::string pml_file, tfsf_file, ids_file, dl_file, gain_file, drude_file;
    int tfsf_k0 = 0, dl_literal = 0;
    std::vector<Source> sources;
    std::vector<std::pair<int, std::string>> port_files;  // 0 plain, 1 spherical
    {
        std::ifstream in(dir + "harness.txt");
        if (!in) die("no harness.txt");
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream s(line);
            std::string key;
            if (!(s >> key)) continue;
            if (key == "nsteps") s >> nsteps;
            else if (key == "n0") s >> n0;
            else if (key == "pml") s >> pml_file;
            else if (key == "tfsf") s >> tfsf_file >> tfsf_k0;
            else if (key == "ids") s >> ids_file;
            else if (key == "dl") { s >> dl_file; if (!(s >> dl_literal)) dl_literal = 0; }
            else if (key == "gain") s >> gain_file;
            else if (key == "drude") s >> drude_file;
            else if (key == "three") die("the three-level gain runs in the oracle and the engine only (its reference class is 2-D)");
            else if (key == "record_ports") s >> record_ports;
            else if (key == "bench") s >> warm >> timed;
            else if (key == "threads") s >> threads;
            else if (key == "plainport" || key == "sphericalport") {
                std::string f; s >> f; port_files.push_back({key == "plainport" ? 0 : 1, f});
            } else if (key == "source") {
                Source src; std::string wf; int nw = 0;
                s >> src.comp >> src.i >> src.j >> src.k >> wf >> nw;
                src.wave = read_doubles(dir + wf, nw);
                sources.push_back(src);
            } else die(("unknown directive " + key).c_str());
        }
    }
    if (threads > 0) omp_set_num_threads(threads);

    std::string mat = dir + "material.txt", mesh = dir + "structure.txt";
    Structure S(mat.c_str());
    S.generate_mesh(mesh.c_str());
    S.InitializeBasicFDTDCoefficients();
    const int Nx = S.Nx, Ny = S.Ny, Nz = S.Nz;
    const size_t ncell = (size_t)(Nx + 1) * (Ny + 1) * (Nz + 1);
    if (!ids_file.empty()) {
        std::vector<unsigned char> ids(ncell);
        FILE *f = fopen((dir + ids_file).c_str(), "rb");
        if (!f || fread(ids.data(), 1, ncell, f) != ncell) die("cannot read ids");
        fclose(f);
        size_t q = 0;
        for (int i = 0; i <= Nx; ++i)
            for (int j = 0; j <= Ny; ++j)
                for (int k = 0; k <= Nz; ++k) S.ID[i][j][k] = ids[q++];
    }
    char mode[] = "TEM";
    Field F(S, mode);

    CPML *pml = nullptr;
    if (!pml_file.empty()) {
        const std::string path = dir + pml_file;
        std::vector<char> fn(path.begin(), path.end());
        fn.push_back(0);
        pml = new CPML(S, fn.data());
        pml->InitializeCPML(S);
        const double eta0 = sqrt(mu0 / eps0);
        const double sx = pml->sig_ratio * (0.8 * (pml->m + 1) / (S.dx * eta0));
        const double sy = pml->sig_ratio * (0.8 * (pml->m + 1) / (S.dy * eta0));
        const double sz = pml->sig_ratio * (0.8 * (pml->m + 1) / (S.dz * eta0));
        fill_last_h(pml->bxH1, pml->cxH1, true, pml->Npmlx1, S.dt, S.dx, pml->m, pml->malp, sx, pml->kapmax, pml->alpmax);
        fill_last_h(pml->bxH2, pml->cxH2, false, pml->Npmlx2, S.dt, S.dx, pml->m, pml->malp, sx, pml->kapmax, pml->alpmax);
        fill_last_h(pml->byH1, pml->cyH1, true, pml->Npmly1, S.dt, S.dy, pml->m, pml->malp, sy, pml->kapmax, pml->alpmax);
        fill_last_h(pml->byH2, pml->cyH2, false, pml->Npmly2, S.dt, S.dy, pml->m, pml->malp, sy, pml->kapmax, pml->alpmax);
        fill_last_h(pml->bzH1, pml->czH1, true, pml->Npmlz1, S.dt, S.dz, pml->m, pml->malp, sz, pml->kapmax, pml->alpmax);
        fill_last_h(pml->bzH2, pml->czH2, false, pml->Npmlz2, S.dt, S.dz, pml->m, pml->malp, sz, pml->kapmax, pml->alpmax);
    }

    TF_SF *tfsf = nullptr;
    if (!tfsf_file.empty()) {
        const std::string path = dir + tfsf_file;
        std::vector<char> fn(path.begin(), path.end());
        fn.push_back(0);
        void *mem = calloc(1, sizeof(TF_SF));
        static_cast<TF_SF *>(mem)->k0 = tfsf_k0;  // the constructor reads k0 but never sets it
        tfsf = new (mem) TF_SF(S, fn.data());
    }

    // 3-D Drude-Lorentz (oracle recursion) on ID==2 cells of the E range
    dl_t D;
    memset(&D, 0, sizeof(D));
    std::vector<int> dl_cells;
    std::vector<double> dl_state;
    if (!dl_file.empty() || !drude_file.empty()) {
        double sigma, epsInf; int nD, nL;
        std::vector<double> fD, gD, fL, dL, de;
        if (!drude_file.empty()) {  // the single-pole Drude deck, Drude.cpp:29-52
            std::ifstream f(dir + drude_file);
            std::string line;
            double v[4] = {0, 0, 0, 0};
            for (int q = 0; q < 4; ++q) {
                if (!std::getline(f, line)) die("drude deck");
                std::istringstream(line) >> v[q];
            }
            epsInf = v[0]; sigma = v[2]; nD = 1; nL = 0;
            fD = {v[1]}; gD = {v[3]}; fL = {0.0}; dL = {0.0}; de = {0.0};
            dl_literal = 2;
        } else {
            read_dl(dir + dl_file, sigma, epsInf, nD, fD, gD, nL, fL, dL, de);
        }
        dl_coeffs(&D, S.dt, sigma, epsInf, nD, fD.data(), gD.data(), nL, fL.data(), dL.data(), de.data(), dl_literal);
        D.stride = nD + 2 * nL + 1;
        for (int i = 1; i < Nx; ++i)
            for (int j = 1; j < Ny; ++j)
                for (int k = 1; k < Nz; ++k)
                    if (S.ID[i][j][k] == 2) { dl_cells.push_back(i); dl_cells.push_back(j); dl_cells.push_back(k); }
        dl_state.assign(dl_cells.size() / 3 * 3 * D.stride, 0.0);
        D.on = 1;
    }
    gain_t G;
    memset(&G, 0, sizeof(G));
    std::vector<int> g_cells;
    std::vector<double> g_state;
    if (!gain_file.empty()) {
        double v[10];
        read_gain(dir + gain_file, v);
        gain_coeffs(&G, S.dt, S.dx, S.dy, v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9]);
        for (int i = 1; i < Nx; ++i)
            for (int j = 1; j < Ny; ++j)
                for (int k = 1; k < Nz; ++k)
                    if (S.ID[i][j][k] == 5) { g_cells.push_back(i); g_cells.push_back(j); g_cells.push_back(k); }
        g_state.assign(g_cells.size() / 3 * GAIN_WORDS, 0.0);
        for (size_t c = 0; c < g_cells.size() / 3; ++c) gain_site_init(&g_state[c * GAIN_WORDS]);
        G.on = 1;
    }

    std::vector<PlainPort *> pports;
    std::vector<SphericalPort *> sports;
    std::vector<int> port_kind;
    for (auto &pf : port_files) {
        std::string fn = dir + pf.second;
        if (pf.first == 0) { pports.push_back(new PlainPort(S, fn.c_str())); port_kind.push_back(0); }
        else { sports.push_back(new SphericalPort(S, fn.c_str())); port_kind.push_back(1); }
    }
    auto port_points = [&](size_t p, Port_Points *&pts, int &n) {
        size_t a = 0, b = 0;
        for (size_t q = 0; q < p; ++q) (port_kind[q] == 0 ? a : b)++;
        if (port_kind[p] == 0) { pts = pports[a]->port_point; n = pports[a]->Num_of_Port_Points - 1; }
        else { pts = sports[b]->port_point; n = sports[b]->Num_of_Port_Points - 1; }
    };
    std::vector<std::vector<double>> series(port_kind.size());

    const size_t n_dl = dl_cells.size() / 3, n_g = g_cells.size() / 3;
    auto step = [&](int n) {
        BasicHFieldUpdate(F, S);
        if (tfsf) tfsf->UpdateHField(n, F, S);
        if (pml) pml->UpdateCPMLHFields(F);
        BasicEFieldUpdate(F, S);
        if (D.on) {
#pragma omp parallel for schedule(static)
            for (size_t c = 0; c < n_dl; ++c) {
                const int i = dl_cells[3 * c], j = dl_cells[3 * c + 1], k = dl_cells[3 * c + 2];
                double *st = &dl_state[c * 3 * D.stride];
                const double C3 = D.C3;
                const double cx = C3 * (F.Hz[i][j][k] - F.Hz[i][j - 1][k]) * S.cExz[j] - C3 * (F.Hy[i][j][k] - F.Hy[i][j][k - 1]) * S.cExy[k];
                const double cy = C3 * (F.Hx[i][j][k] - F.Hx[i][j][k - 1]) * S.cEyx[k] - C3 * (F.Hz[i][j][k] - F.Hz[i - 1][j][k]) * S.cEyz[i];
                const double cz = C3 * (F.Hy[i][j][k] - F.Hy[i - 1][j][k]) * S.cEzy[i] - C3 * (F.Hx[i][j][k] - F.Hx[i][j - 1][k]) * S.cEzx[j];
                F.Ex[i][j][k] = dl_component(&D, S.dt, F.Ex[i][j][k], cx, st);
                F.Ey[i][j][k] = dl_component(&D, S.dt, F.Ey[i][j][k], cy, st + D.stride);
                F.Ez[i][j][k] = dl_component(&D, S.dt, F.Ez[i][j][k], cz, st + 2 * D.stride);
            }
        }
        if (G.on) {
#pragma omp parallel for schedule(static)
            for (size_t c = 0; c < n_g; ++c) {
                const int i = g_cells[3 * c], j = g_cells[3 * c + 1], k = g_cells[3 * c + 2];
                double E[3] = {F.Ex[i][j][k], F.Ey[i][j][k], F.Ez[i][j][k]};
                gain_site_p(&G, &g_state[c * GAIN_WORDS], E, 3);
            }
#pragma omp parallel for schedule(static)
            for (size_t c = 0; c < n_g; ++c) {
                const int i = g_cells[3 * c], j = g_cells[3 * c + 1], k = g_cells[3 * c + 2];
                double E[3] = {F.Ex[i][j][k], F.Ey[i][j][k], F.Ez[i][j][k]};
                gain_site_e(&G, &g_state[c * GAIN_WORDS], E, 3);
                F.Ex[i][j][k] = E[0]; F.Ey[i][j][k] = E[1]; F.Ez[i][j][k] = E[2];
            }
#pragma omp parallel for schedule(static)
            for (size_t c = 0; c < n_g; ++c) {
                const int i = g_cells[3 * c], j = g_cells[3 * c + 1], k = g_cells[3 * c + 2];
                const double E[3] = {F.Ex[i][j][k], F.Ey[i][j][k], F.Ez[i][j][k]};
                gain_site_n(&G, &g_state[c * GAIN_WORDS], E, 3);
            }
        }
        if (tfsf) tfsf->UpdateEField(n, F, S);
        for (auto &s : sources)
            if (n >= 0 && n < (int)s.wave.size())
                field_of(F, s.comp)[s.i][s.j][s.k] = field_of(F, s.comp)[s.i][s.j][s.k] + s.wave[n];
        if (pml) pml->UpdateCPMLEFields(F);
        for (auto *p : pports) p->Update_Fields_on_Port(F);
        for (auto *p : sports) p->Update_Fields_on_Port(F);
        if (record_ports)
            for (size_t p = 0; p < port_kind.size(); ++p) {
                Port_Points *pts; int np;
                port_points(p, pts, np);
                for (int q = 0; q < np; ++q) {
                    const double v[6] = {pts[q].Ex, pts[q].Ey, pts[q].Ez, pts[q].Hx, pts[q].Hy, pts[q].Hz};
                    series[p].insert(series[p].end(), v, v + 6);
                }
            }
    };

    if (warm >= 0) {
        for (int n = n0; n < n0 + warm; ++n) step(n);
        const double t0 = omp_get_wtime();
        for (int n = n0 + warm; n < n0 + warm + timed; ++n) step(n);
        const double t1 = omp_get_wtime();
        printf("REF_BENCH {\"cells\": %lld, \"steps\": %d, \"seconds\": %.6f, \"threads\": %d}\n",
               (long long)Nx * Ny * Nz, timed, t1 - t0, omp_get_max_threads());
        fflush(stdout);
        _exit(0);
    }
    for (int n = n0; n < n0 + nsteps; ++n) step(n);

    // dumps: ids, fields, stretch arrays, TF/SF tables, ports
    {
        std::vector<unsigned char> ids(ncell);
        std::vector<double> buf(ncell);
        size_t q = 0;
        for (int i = 0; i <= Nx; ++i)
            for (int j = 0; j <= Ny; ++j)
                for (int k = 0; k <= Nz; ++k) ids[q++] = (unsigned char)S.ID[i][j][k];
        write_raw(out + "ids.bin", ids.data(), ncell);
        const char *names[6] = {"Ex", "Ey", "Ez", "Hx", "Hy", "Hz"};
        for (int c = 0; c < 6; ++c) {
            double ***a = field_of(F, c);
            q = 0;
            for (int i = 0; i <= Nx; ++i)
                for (int j = 0; j <= Ny; ++j)
                    for (int k = 0; k <= Nz; ++k) buf[q++] = a[i][j][k];
            write_raw(out + names[c] + ".bin", buf.data(), ncell * sizeof(double));
        }
        std::vector<double> st;
        const double *arrs[12] = {S.cExy, S.cEyx, S.cEzx, S.cExz, S.cEzy, S.cEyz,
                                  S.cHxy, S.cHyx, S.cHzx, S.cHxz, S.cHzy, S.cHyz};
        const int lens[12] = {Nz, Nz, Ny, Ny, Nx, Nx, Nz, Nz, Ny, Ny, Nx, Nx};
        for (int a = 0; a < 12; ++a) st.insert(st.end(), arrs[a], arrs[a] + lens[a]);
        write_raw(out + "stretch.bin", st.data(), st.size() * sizeof(double));
        if (tfsf) {
            std::vector<double> t(tfsf->Einc, tfsf->Einc + tfsf->Nt + 1);
            t.insert(t.end(), tfsf->Hinc, tfsf->Hinc + tfsf->Nt + 1);
            write_raw(out + "tfsf_inc.bin", t.data(), t.size() * sizeof(double));
        }
        for (size_t p = 0; p < port_kind.size(); ++p) {
            Port_Points *pts; int np;
            port_points(p, pts, np);
            std::vector<int> ijk;
            std::vector<double> last;
            for (int r = 0; r < np; ++r) {
                ijk.push_back(pts[r].i); ijk.push_back(pts[r].j); ijk.push_back(pts[r].k);
                const double v[6] = {pts[r].Ex, pts[r].Ey, pts[r].Ez, pts[r].Hx, pts[r].Hy, pts[r].Hz};
                last.insert(last.end(), v, v + 6);
            }
            write_raw(out + "port" + std::to_string(p) + "_points.bin", ijk.data(), ijk.size() * sizeof(int));
            write_raw(out + "port" + std::to_string(p) + "_last.bin", last.data(), last.size() * sizeof(double));
            if (record_ports)
                write_raw(out + "port" + std::to_string(p) + "_series.bin", series[p].data(), series[p].size() * sizeof(double));
        }
        std::ofstream info(out + "info.txt");
        info.precision(17);
        info << "Nx " << Nx << "\nNy " << Ny << "\nNz " << Nz << "\ndx " << S.dx << "\ndy " << S.dy
             << "\ndz " << S.dz << "\ndt " << S.dt << "\nnports " << port_kind.size() << "\n";
    }
    fflush(stdout);
    _exit(0);
}
