// driver.cpp -- registration loop (DUGMA.m) with a quasi-Newton solver.
#include "dugma.h"

extern "C" int dugma_register(const double*, const double*, const double*, const double*, int, int, int,
                              const double*, const double*, int, double, double, double, int, double*, double*,
                              double*)
{
    return DUGMA_ERR_ARG;
}
