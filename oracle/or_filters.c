/*
 * or_filters.c - the smoothing filters of the model iteration (TEST INFRASTRUCTURE ONLY),
 * flat terrain (every cell is fluid, so the no-flux substitutions never apply and the
 * orographic, steep-massif and coastal filters flag no column and change nothing):
 *
 *   or_post_rk4_filters: after the RK4 step (cAtmosphereModel.cpp:1507-1520)
 *     AtomUtils::polar_zonal_filter(u|v|w, the.z, 30 deg, 12 passes, gain 3)  lib/Utils.cpp:542-611
 *     AtomUtils::radial_shapiro_filter(u, 2 passes, strength 1)               lib/Utils.cpp:831-873
 *     AtomUtils::radial_shapiro_filter_ho(v|w, 2 passes, strength 1)          lib/Utils.cpp:884-940
 *   or_damp_wiggles: AtomUtils::damp_wiggles(field, along i, j, k, strength 1, 1 pass)
 *     (lib/Utils.cpp:429-531), applied to t, ice, c, cloud after the saturation adjustment
 *     of a moist iteration (cAtmosphereModel.cpp:1225-1228).
 *
 * The polar filter's pass count per row uses sin(theta) from the mirror-exact table, so it
 * is the same for row j and row jm-1-j.
 */
#include "or_internal.h"

/* one periodic 1-2-1 pass along k of row (i, j), from a snapshot of the row */
static void zonal_pass(double* x, double* tmp, int km, double coeff)
{
    memcpy(tmp, x, sizeof(double) * km);
    for (int k = 0; k < km; k++) {
        const int km1 = (k - 1 + km) % km, kp1 = (k + 1) % km;
        x[k] = tmp[k] + coeff * (tmp[km1] - 2.0 * tmp[k] + tmp[kp1]);
    }
}

/* passes of row j, lib/Utils.cpp:559-571 */
int or_polar_passes(int jm, int j, const double* sin_w)
{
    const double sin_ref = cos(30.0 * (M_PI / 180.0));
    const double sin_j = or_max(sin_w[j], 1.0e-6);
    if (sin_j >= sin_ref) return 0;
    const double ratio = sin_ref / sin_j;
    /* (int) of the long, as the reference converts it: on the pole rows (sin guarded to
     * 1e-6) the count overflows an int and wraps before the clamp */
    int p = (int)lround(3.0 * (ratio * ratio - 1.0));
    if (p < 0) p = 0;
    if (p > 12) p = 12;
    (void)jm;
    return p;
}

void or_post_rk4_filters(int im, int jm, int km, const or_params* p, double* const* f)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);
    double* tmp = (double*)malloc(sizeof(double) * (size_t)(km > im ? km : im) * 2);
    const int vel[3] = { OF_U, OF_V, OF_W };
    for (int q = 0; q < 3; q++)                      /* polar zonal filter */
        for (int i = 0; i < im; i++)
            for (int j = 0; j < jm; j++) {
                const int np = or_polar_passes(jm, j, g.sin_w);
                for (int pass = 0; pass < np; pass++) zonal_pass(f[vel[q]] + OR_IDX(i, j, 0), tmp, km, 0.25);
            }
    /* radial filters: per column, two Jacobi passes over i = 1..im-2 */
    for (int q = 0; q < 3; q++) {
        double* x = f[vel[q]];
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++)
                for (int pass = 0; pass < 2; pass++) {
                    for (int i = 0; i < im; i++) tmp[i] = x[OR_IDX(i, j, k)];
                    for (int i = 1; i < im - 1; i++) {
                        const double c = tmp[i];
                        if (q == 0) {                /* 1-2-1, strength 1 */
                            x[OR_IDX(i, j, k)] = c + 0.25 * (tmp[i - 1] - 2.0 * c + tmp[i + 1]);
                        } else if (i - 2 >= 0 && i + 2 <= im - 1) {   /* 4th-order Shapiro */
                            const double d4 = tmp[i + 2] - 4.0 * tmp[i + 1] + 6.0 * c - 4.0 * tmp[i - 1] + tmp[i - 2];
                            x[OR_IDX(i, j, k)] = c - (1.0 / 16.0) * d4;
                        } else {
                            x[OR_IDX(i, j, k)] = c + 0.25 * (tmp[i - 1] - 2.0 * c + tmp[i + 1]);
                        }
                    }
                }
    }
    free(tmp);
    or_geom_free(&g);
}

/* compat = 1: the reference's expression order; 0: the j pass adds the two neighbours first
 * (mirror-exact), as the device does */
void or_damp_wiggles(int im, int jm, int km, double* x, int compat)
{
    const size_t n = (size_t)im * jm * km;
    double* tmp = (double*)malloc(sizeof(double) * n);
    const double coeff = 0.25;
    /* along k, periodic over all km points */
    memcpy(tmp, x, sizeof(double) * n);
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) {
                const int km1 = (k - 1 + km) % km, kp1 = (k + 1) % km;
                x[OR_IDX(i, j, k)] = tmp[OR_IDX(i, j, k)]
                    + coeff * (tmp[OR_IDX(i, j, km1)] - 2.0 * tmp[OR_IDX(i, j, k)] + tmp[OR_IDX(i, j, kp1)]);
            }
    /* along j, clamped at the poles */
    memcpy(tmp, x, sizeof(double) * n);
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            const int jm1 = (j - 1 < 0) ? 0 : j - 1, jp1 = (j + 1 > jm - 1) ? jm - 1 : j + 1;
            for (int k = 0; k < km; k++)
                x[OR_IDX(i, j, k)] = compat
                    ? tmp[OR_IDX(i, j, k)]
                      + coeff * (tmp[OR_IDX(i, jm1, k)] - 2.0 * tmp[OR_IDX(i, j, k)] + tmp[OR_IDX(i, jp1, k)])
                    : tmp[OR_IDX(i, j, k)]
                      + coeff * ((tmp[OR_IDX(i, jm1, k)] + tmp[OR_IDX(i, jp1, k)]) - 2.0 * tmp[OR_IDX(i, j, k)]);
        }
    /* along i, clamped at the surface and the lid */
    memcpy(tmp, x, sizeof(double) * n);
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            for (int i = 0; i < im; i++) {
                const int im1 = (i - 1 < 0) ? 0 : i - 1, ip1 = (i + 1 > im - 1) ? im - 1 : i + 1;
                x[OR_IDX(i, j, k)] = tmp[OR_IDX(i, j, k)]
                    + coeff * (tmp[OR_IDX(im1, j, k)] - 2.0 * tmp[OR_IDX(i, j, k)] + tmp[OR_IDX(ip1, j, k)]);
            }
    free(tmp);
}
