/*
 * or_moist.c - oracle restatement of MoistConvection::run (MoistConvection.h:106-1537).
 * TEST INFRASTRUCTURE ONLY, see athad_oracle.h.
 */
#include "or_internal.h"

int or_moist_convection(int im, int jm, int km, const or_params* p, int compat, int iter_n,
                        double* const* f, double* const* f2)
{
    (void)im; (void)jm; (void)km; (void)p; (void)compat; (void)iter_n; (void)f; (void)f2;
    return -1;
}
