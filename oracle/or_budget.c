/*
 * or_budget.c - the global mass budgets of the moist iteration (TEST INFRASTRUCTURE ONLY):
 *
 *   or_co2_column     ThermoAtm::co2Column (ThermoAtm.h:1096-1137)
 *   or_water_budget   ThermoAtm::waterBudget (ThermoAtm.h:934-1094), its sums
 *
 * The sums run in the serial order of one OpenMP thread.
 */
#include "or_internal.h"

/* cos((j / (jm - 1) - 0.5) pi), ThermoAtm.h:945, 1105 */
static double coslat_of(int j, int jm) { return cos((j / (double)(jm - 1) - 0.5) * M_PI); }

static double dp_pa(const double* ps, int im, int jm, int km, int i, int j, int k)
{
    return (i < im - 1) ? (ps[OR_IDX(i, j, k)] - ps[OR_IDX(i + 1, j, k)]) * 100.0
                        : ps[OR_IDX(i, j, k)] * 100.0;
}

void or_co2_column(int im, int jm, int km, const or_params* p, double* const* f, double* const* f2,
                   double* out)
{
    double w_num = 0.0, w_den = 0.0;
    const double* ps = f[OF_P_STAT];
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const double coslat = coslat_of(j, jm);
            double col = 0.0;
            for (int i = 0; i < im; i++) {
                const double dp = dp_pa(ps, im, jm, km, i, j, k);
                if (!(dp > 0.0)) continue;
                const double u_air = dp / p->g;
                const double q_c = or_max(0.0, f[OF_CO2][OR_IDX(i, j, k)]);
                col += q_c * u_air;
                w_den += coslat * u_air;
                w_num += coslat * q_c * u_air;
            }
            f2[OF2_CO2_TOTAL][(size_t)j * km + k] = col;
        }
    out[0] = w_num; out[1] = w_den;
}

static double q_water(double* const* f, size_t c)
{
    return or_max(0.0, f[OF_C][c]) + or_max(0.0, f[OF_CLOUD][c]) + or_max(0.0, f[OF_ICE][c])
         + or_max(0.0, f[OF_GR][c]);
}

void or_water_budget(int im, int jm, int km, const or_params* p, double* const* f, double* out,
                     double* qbar, double* abar, double* lev)
{
    const double* ps = f[OF_P_STAT];
    double w_num = 0.0, w_den = 0.0;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const double coslat = coslat_of(j, jm);
            for (int i = 0; i < im; i++) {
                const double dp = dp_pa(ps, im, jm, km, i, j, k);
                if (!(dp > 0.0)) continue;
                const double u_air = dp / p->g;
                const double q_w = q_water(f, OR_IDX(i, j, k));
                w_den += coslat * u_air;
                w_num += coslat * q_w * u_air;
            }
        }
    for (int i = 0; i < im; i++) {
        double qn = 0.0, qd = 0.0, an = 0.0, num = 0.0;
        for (int j = 0; j < jm; j++) {
            const double coslat = coslat_of(j, jm);
            for (int k = 0; k < km; k++) {
                const double dp = dp_pa(ps, im, jm, km, i, j, k);
                const double q_w = q_water(f, OR_IDX(i, j, k));
                qn += coslat * q_w;
                qd += coslat;
                if (dp > 0.0) {
                    an += coslat * dp / p->g;
                    num += coslat * q_w * dp / p->g;
                }
            }
        }
        qbar[i] = (qd > 0.0) ? qn / qd : 0.0;
        abar[i] = an;
        lev[i] = num;          /* divided by w_den by the caller (ThermoAtm.h:1031) */
    }
    out[0] = w_num; out[1] = w_den;
}
