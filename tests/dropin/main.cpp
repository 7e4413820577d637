// A main.cpp in the reference's style (main.cpp:110-344 of cpsFDTD), built
// against include/cpsfdtd_classes.hpp instead of the reference headers: reads
// the decks of a directory, runs the reference's call order for nsteps, and
// writes the six fields ([i][j][k] FP64, raw) and the port E exports.
//
//   dropin <deck dir> <nsteps> <out dir>
#include <stdio.h>
#include <sys/stat.h>

#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "cpsfdtd_classes.hpp"

static bool exists(const std::string &f)
{
    struct stat st;
    return stat(f.c_str(), &st) == 0;
}

int main(int argc, char **argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: dropin <deck dir> <nsteps> <out dir>\n");
        return 2;
    }
    const std::string dir = argv[1], out = argv[3];
    const int nsteps = atoi(argv[2]);
    try {
        Structure S((dir + "/material.txt").c_str());
        S.generate_mesh((dir + "/structure.txt").c_str());
        S.InitializeBasicFDTDCoefficients();
        Field F(S, "TEM");
        std::unique_ptr<CPML> pml;
        if (exists(dir + "/CFS_PML.txt")) {
            pml.reset(new CPML(S, (dir + "/CFS_PML.txt").c_str()));
            pml->InitializeCPML(S);
        }
        std::unique_ptr<Drude_Lorentz> DL;
        if (exists(dir + "/DrudeLorentz.txt")) DL.reset(new Drude_Lorentz(S, (dir + "/DrudeLorentz.txt").c_str()));
        std::unique_ptr<Drude> DR;
        if (exists(dir + "/Drude.txt")) DR.reset(new Drude(S, (dir + "/Drude.txt").c_str()));
        std::unique_ptr<FourLevelLaser> FL;
        if (exists(dir + "/FourLevelLaser.txt")) FL.reset(new FourLevelLaser(S, (dir + "/FourLevelLaser.txt").c_str()));
        std::unique_ptr<ThreeLevel> TL;
        if (exists(dir + "/ThreeLevel.txt")) TL.reset(new ThreeLevel(S, (dir + "/ThreeLevel.txt").c_str()));
        std::unique_ptr<TF_SF> tfsf;
        if (exists(dir + "/TF_SF.txt")) tfsf.reset(new TF_SF(S, (dir + "/TF_SF.txt").c_str()));
        std::vector<std::unique_ptr<PlainPort>> ports;
        for (int q = 0; exists(dir + "/port" + std::to_string(q) + ".txt"); ++q) {
            std::ifstream f(dir + "/port" + std::to_string(q) + ".txt");
            std::string first;
            f >> first;
            if (first.size() == 1 && (first[0] == 'x' || first[0] == 'y' || first[0] == 'z'))
                ports.emplace_back(new PlainPort(S, (dir + "/port" + std::to_string(q) + ".txt").c_str()));
        }
        for (int n = 1; n <= nsteps; ++n) {
            BasicHFieldUpdate(F, S);
            if (tfsf) tfsf->UpdateHField(n, F, S);
            if (pml) pml->UpdateCPMLHFields(F);
            BasicEFieldUpdate(F, S);
            if (DL) DL->EFieldUpdate(F, S);
            if (DR) DR->EFieldUpdate(F, S);
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
            if (tfsf) tfsf->UpdateEField(n, F, S);
            if (pml) pml->UpdateCPMLEFields(F);
            for (auto &p : ports) p->Update_Fields_on_Port(F);
        }
        F.sync_to_host();
        double ***c[6] = {F.Ex, F.Ey, F.Ez, F.Hx, F.Hy, F.Hz};
        const size_t cells = (size_t)(S.Nx + 1) * (S.Ny + 1) * (S.Nz + 1);
        for (int q = 0; q < 6; ++q) {
            FILE *f = fopen((out + "/field" + std::to_string(q) + ".bin").c_str(), "wb");
            if (!f || fwrite(c[q][0][0], sizeof(double), cells, f) != cells) return 3;
            fclose(f);
        }
        for (size_t q = 0; q < ports.size(); ++q) {
            ports[q]->Export_E_onPort((out + "/portE" + std::to_string(q) + ".txt").c_str());
            ports[q]->Export_Port((out + "/portP" + std::to_string(q) + ".txt").c_str());
        }
        if (tfsf) {
            std::ofstream t(out + "/tfsf.txt");
            t.precision(17);
            t << tfsf->Nt << "\t" << tfsf->lambda << "\t" << tfsf->nu << "\t" << tfsf->Einc[10] << "\t"
              << tfsf->Einc_onPoint(10.25) << std::endl;
        }
        printf("dropin ok %d %d %d %d\n", S.Nx, S.Ny, S.Nz, (int)ports.size());
    } catch (const std::exception &e) {
        fprintf(stderr, "dropin: %s\n", e.what());
        return 1;
    }
    return 0;
}
