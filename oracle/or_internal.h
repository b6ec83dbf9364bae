/*
 * or_internal.h - shared helpers of the oracle (TEST INFRASTRUCTURE ONLY).
 */
#ifndef OR_INTERNAL_H
#define OR_INTERNAL_H

#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include "athad_oracle.h"

#define OR_T_CRIT        647.096            /* MixtureAtm.h:40 */
#define OR_NO_SATURATION (-1.0)             /* SaturationH2O.h:50 */
#define OR_R_STAR        8.314462618        /* MixtureAtm.h:44 */
#define OR_M_H2O         0.018015
#define OR_M_CO2         0.044010
#define OR_R_H2O         (OR_R_STAR / OR_M_H2O)
#define OR_R_CO2         (OR_R_STAR / OR_M_CO2)

/* std::max / std::min / std::clamp semantics exactly: (a < b) ? b : a etc., so NaN and
 * signed zeros propagate the way the reference's C++ does. */
static inline double or_max(double a, double b) { return (a < b) ? b : a; }
static inline double or_min(double a, double b) { return (b < a) ? b : a; }
static inline double or_clamp(double v, double lo, double hi)
{
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
/* IEEE exponent-bit test of lib/Utils.h:121-125 */
static inline int or_is_finite(double v)
{
    uint64_t b;
    memcpy(&b, &v, sizeof b);
    return (b & 0x7FF0000000000000ULL) != 0x7FF0000000000000ULL;
}
/* safe_clamp, RungeKutta_Atm_Turb.cpp:76-81 */
static inline double or_safe_clamp(double v, double lo, double hi)
{
    if (!or_is_finite(v)) return lo;
    return (v < lo) ? lo : (v > hi) ? hi : v;
}

/* Grid geometry.  Coordinates are built by running sums, as Array_1D::Coordinates does
 * (lib/Array_1D.cpp:45-51). */
typedef struct or_geom {
    int im, jm, km;
    double dr, dthe, dphi;
    double* rad; double* the; double* phi;
    double* sin_f;      /* sin(theta), floored at 0.55 (RK4.cpp:92-97, PressureSolverAtm.h:35-39) */
    double* cos_t;      /* cos(theta) */
    double* sin_w;      /* sin(theta), unfloored (level-mean weight, RK4.cpp:31) */
    double* height;     /* get_layer_height(i): float-rounded (cAtmosphereModel.h:441-452) */
    double shell_len;   /* metricShellLength(), cAtmosphereModel.h:465-470 */
} or_geom;

void   or_geom_init(or_geom* g, int im, int jm, int km, const or_params* p, int compat);
void   or_geom_free(or_geom* g);
double or_metric_radius(const or_geom* g, const or_params* p, double rm);

/* thermo (or_thermo.c) */
double or_saturation_pressure_auto(double T);
double or_saturation_mass_fraction_at(double T, double p, double M_other);
double or_latent_heat_sublimation(double T);
double or_latent_heat_auto(double T);
double or_sat_deriv_factor_at(double E, double p, double M_other);
double or_dqsat_dT_from(double E, double L, double T, double p, double M_other);

/* IceSchemeCommon::evaporateWhereImpossible at cell c (or_columns.c) */
void or_evaporate_where_impossible(const or_params* p, double* const* f, size_t c, double t_u);

#define OR_IDX(i, j, k) (((size_t)(i) * (size_t)jm + (size_t)(j)) * (size_t)km + (size_t)(k))

#endif
