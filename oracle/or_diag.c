/*
 * or_diag.c - the diagnostics of the moist iteration that read the state without changing
 * it (TEST INFRASTRUCTURE ONLY):
 *
 *   or_find_residuum         UtilsAtm::findResiduumAtm (UtilsAtm.h:70-220)
 *   or_stand_atm_dew_point   ThermoAtm::standAtm_DewPoint_HumidRel (ThermoAtm.h:400-516)
 */
#include "or_internal.h"

/* The residual of one cell is the rms of the three normal velocity derivatives
 * (UtilsAtm.h:98-113), with plain rm (no metric radius) and sin(theta) floored at 0.55
 * from the running-sum theta.  The reference's band is i = 10..30; it reads i + 1 = 31, so it
 * needs im >= 32, and the band here stops at im - 2 on smaller grids.  Sums run in the
 * serial (j, k, i) order of one OpenMP thread; the residuum keeps the smallest (i, j, k) on
 * equal values (the tie rule of the reference's reduction, :159-171). */
void or_find_residuum(int im, int jm, int km, double* const* f, double* out, int64_t* cnt, int* idx)
{
    or_geom g;
    or_params p0;
    memset(&p0, 0, sizeof p0);
    p0.zeta = 3.0; p0.L_atm = 1.0;          /* heights unused */
    or_geom_init(&g, im, jm, km, &p0, 1);  /* running-sum theta, plain sin */
    const double* u = f[OF_U];
    const double* v = f[OF_V];
    const double* w = f[OF_W];
    const int i0 = 10, i1 = (im - 2 < 30) ? im - 2 : 30;
    double mx = 0.0, sum = 0.0;
    int mi = 0, mj = 0, mk = 0;
    int64_t n = 0, n_nan = 0;
    int ni = -1, nj = -1, nk = -1;
    const size_t sI = (size_t)jm * km, sJ = (size_t)km;
    for (int j = 1; j < jm - 1; j++)
        for (int k = 1; k < km - 1; k++) {
            double sinthe = sin(g.the[j]);
            if (sinthe < 0.55) sinthe = 0.55;
            for (int i = i0; i <= i1; i++) {
                const size_t c = OR_IDX(i, j, k);
                const double rm = g.rad[i];
                const double exp_rm = 1.0 / (rm + 1.0);
                const double rmsinthe = rm * sinthe;
                const double dudr = (u[c + sI] - u[c - sI]) / (2.0 * g.dr) * exp_rm;
                const double dvdthe = (v[c + sJ] - v[c - sJ]) / (2.0 * rm * g.dthe);
                const double dwdphi = (w[c + 1] - w[c - 1]) / (2.0 * rmsinthe * g.dphi);
                const double res = sqrt((dudr * dudr + dvdthe * dvdthe + dwdphi * dwdphi) / 3.0);
                if (!or_is_finite(res)) {
                    if (n_nan == 0) { ni = i; nj = j; nk = k; }
                    n_nan++;
                    continue;
                }
                sum += res;
                n++;
                const int before = (i < mi) || (i == mi && (j < mj || (j == mj && k < mk)));
                if (res > mx || (res == mx && mx > 0.0 && before)) { mx = res; mi = i; mj = j; mk = k; }
            }
        }
    or_geom_free(&g);
    const double avg = (n > 0) ? sum / (double)n : 0.0;
    out[0] = mx;
    out[1] = avg;
    out[2] = (mx > 0.0) ? avg / mx : 0.0;
    cnt[0] = n; cnt[1] = n_nan;
    idx[0] = mi; idx[1] = mj; idx[2] = mk;
    idx[3] = ni; idx[4] = nj; idx[5] = nk;
}

/* SaturationH2O::dewPoint (SaturationH2O.h:189-202) is or_dew_point; the vapour partial
 * pressure is the exact x_H2O * p (ThermoAtm.h:449-457).  TempStand above the row's
 * tropopause level is the value at that level (:495-500); below-terrain filling is empty on
 * flat terrain. */
void or_stand_atm_dew_point(int im, int jm, int km, const or_params* p, double* const* f,
                            const int* i_trop)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 1);
    const double lapse_rate = 6.5e-3;
    const double t_0 = p->t_0;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const int it = i_trop[j];
            const double ts_surface = f[OF_T][OR_IDX(0, j, k)] * t_0 - t_0;
            f[OF_TEMP_STAND][OR_IDX(0, j, k)] = ts_surface;
            for (int i = 0; i < im; i++) {
                const size_t c = OR_IDX(i, j, k);
                const double t_u = f[OF_T][c] * t_0;
                const double E = (t_u > t_0) ? or_saturation_pressure(t_u) : or_sublimation_pressure(t_u);
                const double x_v = or_x_H2O_of(f[OF_C][c], f[OF_CO2][c], p->M_bg);
                double e = x_v * f[OF_P_STAT][c];
                const int zero_vapour = (e <= 0.0);
                if (zero_vapour) e = 1e-3;
                f[OF_TEMP_STAND][c] = ts_surface - lapse_rate * g.height[i];
                f[OF_TEMP_DEW_POINT][c] = or_dew_point(e) - t_0;
                f[OF_HUMIDITY_REL][c] = (E <= 0.0) ? OR_NO_SATURATION : (zero_vapour ? 0.0 : e / E * 100.0);
            }
            const double ts_trop = f[OF_TEMP_STAND][OR_IDX(it, j, k)];
            for (int i = it + 1; i < im; i++) f[OF_TEMP_STAND][OR_IDX(i, j, k)] = ts_trop;
        }
    or_geom_free(&g);
}
