// Fields.h (2-D stand-in) -- 2-D TE field arrays for ref2d_harness.cpp.
// TEST INFRASTRUCTURE ONLY.
#ifndef FIELDS_H
#define FIELDS_H
#include "Structure.h"
class Field
{
public:
    double **Ex, **Ey, **Ez, **Hz;
};
#endif
