// deck_load.cpp -- cps_deck_load: a grid from a directory of the reference's
// deck files, set up through the drop-in classes of cpsfdtd_classes.hpp (the
// same parsing, validation and set-up calls a main.cpp built on them makes),
// so one front end serves the classes, the served jobs and C callers.
#include <sys/stat.h>

#include <string>

#include "../../include/cpsfdtd_classes.hpp"

namespace cps {
void set_error(const std::string &msg);
}

namespace {
bool exists(const std::string &f)
{
    struct stat st;
    return stat(f.c_str(), &st) == 0;
}
}  // namespace

extern "C" cps_status cps_deck_load(const char *dir, int32_t precision, cps_grid **out)
{
    if (!dir || !out) {
        cps::set_error("cps_deck_load: NULL argument");
        return CPS_E_INVALID;
    }
    *out = nullptr;
    if (precision != CPS_FP64 && precision != CPS_FP32) {
        cps::set_error("cps_deck_load: precision must be CPS_FP64 or CPS_FP32");
        return CPS_E_INVALID;
    }
    const std::string d(dir);
    try {
        Structure S((d + "/material.txt").c_str(), precision);
        S.generate_mesh((d + "/structure.txt").c_str());
        S.InitializeBasicFDTDCoefficients();
        if (exists(d + "/CFS_PML.txt")) {
            CPML pml(S, (d + "/CFS_PML.txt").c_str());
            pml.InitializeCPML(S);
        }
        if (exists(d + "/DrudeLorentz.txt")) Drude_Lorentz dl(S, (d + "/DrudeLorentz.txt").c_str());
        else if (exists(d + "/Drude.txt")) Drude dr(S, (d + "/Drude.txt").c_str());
        if (exists(d + "/FourLevelLaser.txt")) FourLevelLaser fl(S, (d + "/FourLevelLaser.txt").c_str());
        if (exists(d + "/ThreeLevel.txt")) ThreeLevel tl(S, (d + "/ThreeLevel.txt").c_str());
        if (exists(d + "/TF_SF.txt")) TF_SF tf(S, (d + "/TF_SF.txt").c_str());
        // port0.txt, port1.txt, ...: a plain port when the first token is x, y or z
        for (int q = 0; exists(d + "/port" + std::to_string(q) + ".txt"); ++q) {
            const std::string f = d + "/port" + std::to_string(q) + ".txt";
            std::ifstream in(f);
            std::string first;
            in >> first;
            if (first.size() == 1 && (first[0] == 'x' || first[0] == 'y' || first[0] == 'z')) PlainPort p(S, f.c_str());
            else SphericalPort p(S, f.c_str());
        }
        cps_grid *g = S.release_grid();
        cps_grid_set_record(g, 0);  // callers step it with cps_step or a batch
        *out = g;
        return CPS_OK;
    } catch (const cpsfdtd_detail::call_error &e) {
        cps::set_error(std::string("cps_deck_load: ") + e.what());
        return e.code;
    } catch (const std::exception &e) {
        cps::set_error(std::string("cps_deck_load: ") + e.what());
        return CPS_E_INVALID;
    }
}
