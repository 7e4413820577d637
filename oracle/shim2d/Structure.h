// Structure.h (2-D stand-in) -- lets the reference's 2-D TE classes
// Drude_Lorentz and FourLevelLaser compile unmodified for the known-answer
// harness ref2d_harness.cpp.  Only the members those classes read are present.
// TEST INFRASTRUCTURE ONLY.
#ifndef STRUCTURE_H
#define STRUCTURE_H
class Structure
{
public:
    int Nx, Ny;
    double dx, dy, dt;
    short **ID;
    double *aE, *bE, *aH, *bH;
    double *cExy, *cEyx;
};
#endif
