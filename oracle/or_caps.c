/*
 * or_caps.c - the moist iteration's bookkeeping after the ice scheme and the moist
 * convection (TEST INFRASTRUCTURE ONLY):
 *
 *   or_moist_caps        UtilsAtm::precipitationSum (UtilsAtm.h:51-65), the caps of the
 *                        microphysics sources at +-1e-3 (cAtmosphereModel.cpp:1277-1297) and
 *                        of cloud + ice at cloud_cap (:1310-1334)
 *   or_vapour_ceiling    c in [0, 1 - co2] with the mass-weighted water it removes
 *                        (:1369-1391); the sums in the reference's serial (i, j, k) order
 *
 * The caps are written inline in run_3D_loop (no callable reference function), so only
 * precipitationSum is pinned against the reference itself.
 */
#include "or_internal.h"

void or_moist_caps(int im, int jm, int km, const or_params* p, double* const* f)
{
    const size_t n = (size_t)im * jm * km;
    for (size_t q = 0; q < n; q++)
        f[OF_PRECIPITATION][q] = f[OF_P_RAIN][q] + f[OF_P_SNOW][q] + f[OF_P_GRAUPEL][q] + f[OF_P_CONV][q];
    const double S_max = 1.0e-3;
    const int caps[7] = { OF_S_V, OF_S_C, OF_S_I, OF_S_R, OF_S_S, OF_S_G, OF_S_C_C };
    for (int s = 0; s < 7; s++) {
        double* S = f[caps[s]];
        for (size_t q = 0; q < n; q++) {
            const double v = S[q];
            if (!or_is_finite(v)) S[q] = 0.0;
            else if (v > S_max) S[q] = S_max;
            else if (v < -S_max) S[q] = -S_max;
        }
    }
    const double cmax = p->cloud_cap;
    for (size_t q = 0; q < n; q++) {
        double cv = f[OF_C][q], cld = f[OF_CLOUD][q], ic = f[OF_ICE][q];
        if (!or_is_finite(cv)) cv = 0.0;
        if (!or_is_finite(cld)) cld = 0.0;
        if (!or_is_finite(ic)) ic = 0.0;
        if (cv < 0.0) cv = 0.0;
        if (cld < 0.0) cld = 0.0;
        if (ic < 0.0) ic = 0.0;
        const double cv_max = or_max(0.0, 1.0 - f[OF_CO2][q]);
        if (cv > cv_max) cv = cv_max;
        const double sum = cld + ic;
        if (sum > cmax) {
            const double scale = cmax / sum;
            cld *= scale;
            ic *= scale;
        }
        f[OF_C][q] = cv; f[OF_CLOUD][q] = cld; f[OF_ICE][q] = ic;
    }
}

void or_vapour_ceiling(int im, int jm, int km, const or_params* p, double* const* f,
                       int64_t* n_ceiling, double* q_clipped, double* w_air)
{
    int64_t nc = 0;
    double qc = 0.0, wa = 0.0;
    double* c = f[OF_C];
    const double* ps = f[OF_P_STAT];
    const double* co2 = f[OF_CO2];
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) {
                const size_t q = OR_IDX(i, j, k);
                if (c[q] < 0.0) c[q] = 0.0;
                const double dp_Pa = (i < im - 1) ? (ps[q] - ps[q + (size_t)jm * km]) * 100.0 : ps[q] * 100.0;
                const double u_air = (dp_Pa > 0.0) ? dp_Pa / p->g : 0.0;
                wa += u_air;
                const double c_ceiling = or_max(0.0, 1.0 - co2[q]);
                if (c[q] > c_ceiling) {
                    qc += (c[q] - c_ceiling) * u_air;
                    c[q] = c_ceiling;
                    nc++;
                }
            }
    *n_ceiling = nc;
    *q_clipped = qc;
    *w_air = wa;
}

/* cAtmosphereModel::searchMinMax_3D (MinMax_Atm.cpp:51-109): the largest and smallest finite
 * value of a field and the first cell, in (i, j, k) order, holding each; 0 where there is
 * none.  out = max, min; idx = imax, jmax, kmax, imin, jmin, kmin. */
void or_min_max(int im, int jm, int km, const double* x, double* out, int* idx)
{
    double mx = -1.7976931348623157e308, mn = 1.7976931348623157e308;
    int a[6] = { 0, 0, 0, 0, 0, 0 };
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) {
                const double v = x[OR_IDX(i, j, k)];
                if (!isfinite(v)) continue;
                if (v > mx) { mx = v; a[0] = i; a[1] = j; a[2] = k; }
                if (v < mn) { mn = v; a[3] = i; a[4] = j; a[5] = k; }
            }
    if (mx == -1.7976931348623157e308) mx = 0.0;
    if (mn == 1.7976931348623157e308) mn = 0.0;
    out[0] = mx; out[1] = mn;
    for (int q = 0; q < 6; q++) idx[q] = a[q];
}
