/*
 * or_bc.c - the per-iteration boundary conditions of the atmosphere (TEST INFRASTRUCTURE
 * ONLY): BC_Atm::bcRadius, TurbulenceAtm::apply_wall_bc, BC_Atm::bcTheta, BC_Atm::bcPhi,
 * BC_Atm::bcScalarSurfSur and BC_Atm::bcSolidGround in the order of their call site
 * (cAtmosphereModel.cpp:1439-1446), flat terrain: every cell is air, so the last two keep
 * only bcSolidGround's value limits over every cell (BC_Atm.h:470-545).
 *
 * Only the fields the device context holds are treated: the reference's lists also hold
 * the output-only arrays of ThermoAtm::forces (CentrifugalForce, PresGradForce) and
 * precipitableWater (PrecipitableWaterLocal); the right-hand side's CoriolisForce and
 * BuoyancyForce, the heat diagnostics Q_Latent and Q_Sensible and the radiation flux are
 * treated.  c43 and c13 are `const int` members initialised from 4.0/3.0 and 1.0/3.0
 * (cAtmosphereModel.h:158), i.e. 1 and 0, and are applied as such.
 */
#include "or_internal.h"

static const int bc_both_cubic[] = {            /* BC_Atm.h:567-574, Pattern A */
    OF_S_C_C, OF_S_V, OF_S_C, OF_S_I, OF_S_R, OF_S_S, OF_S_G,
    OF_Q_V_U, OF_Q_C_U, OF_U_U, OF_V_U, OF_W_U,
    OF_MC_S, OF_MC_S_U, OF_MC_S_D,
    OF_M_U, OF_M_D, OF_Q_LATENT, OF_Q_SENSIBLE, OF_CORIOLIS_FORCE, OF_BUOYANCY_FORCE
};
static const int bc_vn_bot[] = { OF_U, OF_V, OF_W, OF_P_CONV };   /* :586-590, Pattern B */
static const int bc_cubic_bot_vn_top[] = {      /* :599-603, Pattern C */
    OF_CLOUD, OF_ICE, OF_GR, OF_CO2,
    OF_C_U, OF_E_DD, OF_E_L, OF_E_P, OF_G_P,
    OF_TKE, OF_DIS, OF_NUE, OF_PROD, OF_TKE_SOURCE, OF_DIS_SOURCE
};
static const int bc_hydro[] = { OF_P_STAT, OF_R_HUMID, OF_R_DRY };  /* :656-665, Pattern D */
static const int bc_theta[] = {                 /* :760-776 */
    OF_T, OF_RADIATION, OF_P_STAT, OF_R_HUMID, OF_R_DRY, OF_U, OF_V, OF_W, OF_C, OF_CLOUD, OF_ICE, OF_GR,
    OF_CO2, OF_TKE, OF_DIS, OF_NUE, OF_PROD, OF_TKE_SOURCE, OF_DIS_SOURCE,
    OF_S_C_C, OF_S_V, OF_S_C, OF_S_I, OF_S_R, OF_S_S, OF_S_G,
    OF_Q_V_U, OF_Q_C_U, OF_U_U, OF_V_U, OF_W_U, OF_MC_S, OF_MC_S_U, OF_MC_S_D,
    OF_C_U, OF_E_DD, OF_E_L, OF_E_P, OF_G_P, OF_Q_LATENT, OF_Q_SENSIBLE,
    OF_CORIOLIS_FORCE, OF_BUOYANCY_FORCE
};
static const int bc_phi_avg[] = {               /* :806-817 */
    OF_T, OF_RADIATION, OF_P_STAT, OF_R_HUMID, OF_R_DRY, OF_U, OF_V, OF_W, OF_C, OF_CLOUD, OF_ICE, OF_GR, OF_CO2,
    OF_S_C_C, OF_S_V, OF_S_C, OF_S_I, OF_S_R, OF_S_S, OF_S_G,
    OF_Q_V_U, OF_Q_C_U, OF_U_U, OF_V_U, OF_W_U, OF_MC_S, OF_MC_S_U, OF_MC_S_D,
    OF_C_U, OF_E_DD, OF_E_L, OF_E_P, OF_G_P, OF_Q_LATENT, OF_Q_SENSIBLE,
    OF_CORIOLIS_FORCE, OF_BUOYANCY_FORCE
};
static const int bc_phi_extrap[] = { OF_TKE, OF_DIS, OF_NUE, OF_PROD, OF_TKE_SOURCE, OF_DIS_SOURCE };  /* :822-825 */

#define NELEM(a) ((int)(sizeof(a) / sizeof((a)[0])))

/* bcPhi's 1-2-1 pass over the three seam cells {km-2, 0 = km-1, 1}, every cell air
 * (BC_Atm.h:869-906) */
static void smooth_seam(double* f, int jm, int km, int i, int j)
{
    const int km2 = km - 2, km3 = km - 3;
    const double c = 0.25;
    double* x = f + OR_IDX(i, j, 0);
    const double f_km2 = x[km2], f_0 = x[0], f_1 = x[1];
    const double w_km2 = x[km3], e_km2 = f_0;
    const double w_0 = f_km2, e_0 = f_1;
    const double w_1 = f_0, e_1 = x[2];
    x[km2] = f_km2 + c * (w_km2 - 2.0 * f_km2 + e_km2);
    x[0] = x[km - 1] = f_0 + c * (w_0 - 2.0 * f_0 + e_0);
    x[1] = f_1 + c * (w_1 - 2.0 * f_1 + e_1);
}

/* TurbulenceAtm::apply_wall_bc, TurbulenceAtm.h:109-147 (C_nue 0.028, nue_air 1.5e-5 of its
 * constructor; y1 = get_layer_height(1), a float) */
void or_turb_wall_bc(int im, int jm, int km, const or_params* p, double* const* f, double* const* f2)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);
    const double y1 = g.height[1];
    const double y1_safe = or_max(y1, 1.0e-6);
    const double nd_omega = p->L_atm / p->u_0;
    const double nue_air = 1.5e-5;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const double vs = f2[OF2_VEL_STAR][(size_t)j * km + k];
            f[OF_TKE][OR_IDX(0, j, k)] = vs * vs / (sqrt(0.028) * p->u_0 * p->u_0);
            f[OF_NUE][OR_IDX(0, j, k)] = 0.0;
            if (p->turb_model == 1) {
                f[OF_DIS][OR_IDX(0, j, k)] = 0.0;
            } else if (p->turb_model == 2) {
                const double om = 6.0 * nue_air / (0.075 * y1_safe * y1_safe);
                f[OF_DIS][OR_IDX(0, j, k)] = om * nd_omega;
            } else if (p->turb_model == 3) {
                const double om = 60.0 * nue_air / (0.0333 * y1_safe * y1_safe);
                f[OF_DIS][OR_IDX(0, j, k)] = om * nd_omega;
            }
        }
    or_geom_free(&g);
}

void or_boundary_conditions(int im, int jm, int km, const or_params* p, double* const* f,
                            double* const* f2)
{
    or_boundary_conditions_ex(im, jm, km, p, f, f2, 1);
}

void or_boundary_conditions_ex(int im, int jm, int km, const or_params* p, double* const* f,
                               double* const* f2, int wall_bc)
{
    const int c43 = 1, c13 = 0;               /* (int)(4.0/3.0), (int)(1.0/3.0) */
    const int iml = im - 1, jml = jm - 1;
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);

    /* ---- bcRadius, BC_Atm.h:556-746 ---- */
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            f[OF_T][OR_IDX(iml, j, k)] = f2[OF2_T_TOP_INIT][(size_t)j * km + k];       /* :613-614 */
            for (int q = 0; q < NELEM(bc_both_cubic); q++) {                            /* :629-633 */
                double* x = f[bc_both_cubic[q]];
                x[OR_IDX(0, j, k)] = x[OR_IDX(3, j, k)] - 3.0 * x[OR_IDX(2, j, k)] + 3.0 * x[OR_IDX(1, j, k)];
                x[OR_IDX(iml, j, k)] = x[OR_IDX(iml - 3, j, k)] - 3.0 * x[OR_IDX(iml - 2, j, k)]
                                     + 3.0 * x[OR_IDX(iml - 1, j, k)];
            }
            for (int q = 0; q < NELEM(bc_hydro); q++) {                                  /* :656-665 */
                double* x = f[bc_hydro[q]];
                x[OR_IDX(0, j, k)] = x[OR_IDX(3, j, k)] - 3.0 * x[OR_IDX(2, j, k)] + 3.0 * x[OR_IDX(1, j, k)];
                const double x1 = x[OR_IDX(iml - 1, j, k)], x2 = x[OR_IDX(iml - 2, j, k)];
                x[OR_IDX(iml, j, k)] = (x1 > 0.0 && x2 > 0.0) ? (x1 * x1 / x2) : x1;
            }
            for (int q = 0; q < NELEM(bc_vn_bot); q++) {                                 /* :671-675 */
                double* x = f[bc_vn_bot[q]];
                x[OR_IDX(0, j, k)] = c43 * x[OR_IDX(1, j, k)] - c13 * x[OR_IDX(2, j, k)];
                x[OR_IDX(iml, j, k)] = x[OR_IDX(iml - 1, j, k)];
            }
            double* V[4] = { f[OF_V], f[OF_W], f[OF_VN], f[OF_WN] };                     /* :685-690 */
            for (int q = 0; q < 4; q++) {
                V[q][OR_IDX(iml, j, k)] = 0.0;
                V[q][OR_IDX(iml - 1, j, k)] *= (1.0 / 3.0);
                V[q][OR_IDX(iml - 2, j, k)] *= (2.0 / 3.0);
            }
            f[OF_U][OR_IDX(iml, j, k)] = 0.0;  f[OF_UN][OR_IDX(iml, j, k)] = 0.0;        /* :704-705 */
            f[OF_U][OR_IDX(0, j, k)] = 0.0;    f[OF_UN][OR_IDX(0, j, k)] = 0.0;          /* :723-724 */
            for (int q = 0; q < NELEM(bc_cubic_bot_vn_top); q++) {                       /* :727-731 */
                double* x = f[bc_cubic_bot_vn_top[q]];
                x[OR_IDX(0, j, k)] = x[OR_IDX(3, j, k)] - 3.0 * x[OR_IDX(2, j, k)] + 3.0 * x[OR_IDX(1, j, k)];
                x[OR_IDX(iml, j, k)] = c43 * x[OR_IDX(iml - 1, j, k)] - c13 * x[OR_IDX(iml - 2, j, k)];
            }
            if (f[OF_Q_V_U][OR_IDX(0, j, k)] < 0.0) f[OF_Q_V_U][OR_IDX(0, j, k)] = 0.0;   /* :734-735 */
            if (f[OF_Q_C_U][OR_IDX(0, j, k)] < 0.0) f[OF_Q_C_U][OR_IDX(0, j, k)] = 0.0;
        }

    /* ---- TurbulenceAtm::apply_wall_bc (the per-iteration sequence only) ---- */
    if (wall_bc) or_turb_wall_bc(im, jm, km, p, f, f2);

    /* ---- bcTheta, BC_Atm.h:750-796: pole copies ---- */
    for (int k = 0; k < km; k++)
        for (int i = 0; i < im; i++)
            for (int q = 0; q < NELEM(bc_theta); q++) {
                double* x = f[bc_theta[q]];
                x[OR_IDX(i, 0, k)] = x[OR_IDX(i, 1, k)];
                x[OR_IDX(i, jml, k)] = x[OR_IDX(i, jml - 1, k)];
            }

    /* ---- bcPhi, BC_Atm.h:803-918: seam average, zero-gradient, seam smoothing ---- */
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            for (int q = 0; q < NELEM(bc_phi_avg); q++) {
                double* x = f[bc_phi_avg[q]] + OR_IDX(i, j, 0);
                const double v0 = c43 * x[1] - c13 * x[2];
                const double vend = c43 * x[km - 2] - c13 * x[km - 3];
                x[0] = x[km - 1] = (v0 + vend) * 0.5;
            }
            for (int q = 0; q < NELEM(bc_phi_extrap); q++) {
                double* x = f[bc_phi_extrap[q]] + OR_IDX(i, j, 0);
                x[0] = c43 * x[1] - c13 * x[2];
                x[km - 1] = c43 * x[km - 2] - c13 * x[km - 3];
            }
        }
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int pass = 0; pass < 2; pass++) {
                smooth_seam(f[OF_U], jm, km, i, j);  smooth_seam(f[OF_UN], jm, km, i, j);
                smooth_seam(f[OF_V], jm, km, i, j);  smooth_seam(f[OF_VN], jm, km, i, j);
                smooth_seam(f[OF_W], jm, km, i, j);  smooth_seam(f[OF_WN], jm, km, i, j);
            }

    /* ---- bcScalarSurfSur (BC_Atm.h:1026-1123) and bcSolidGround (:23-547), flat terrain:
     *      their land branches and the surface copies x[0] := x[i_mount = 0] change nothing;
     *      bcSolidGround's value limits over every cell remain (:470-545) ---- */
    {
        const size_t n = (size_t)im * jm * km;
        const int sign[5] = { OF_C, OF_CLOUD, OF_ICE, OF_TKE, OF_DIS };
        for (int q = 0; q < 5; q++)
            for (size_t e = 0; e < n; e++)
                if (f[sign[q]][e] < 0.0) f[sign[q]][e] = 0.0;
        const double tke_max_nd = 1000.0 / (p->u_0 * p->u_0);
        const double nue_max = 1000.0 / (p->u_0 * p->L_atm);
        const double prod_max = 1.0e4, dis_max = 1.0e6;
        const double vel_max_nd = 100.0 / p->u_0;
        const int vel[6] = { OF_U, OF_UN, OF_V, OF_VN, OF_W, OF_WN };
        for (size_t e = 0; e < n; e++) {
            f[OF_TKE][e] = or_safe_clamp(f[OF_TKE][e], 0.0, tke_max_nd);
            f[OF_TKEN][e] = or_safe_clamp(f[OF_TKEN][e], 0.0, tke_max_nd);
            f[OF_DIS][e] = or_safe_clamp(f[OF_DIS][e], 1.0e-10, dis_max);
            f[OF_DISN][e] = or_safe_clamp(f[OF_DISN][e], 1.0e-10, dis_max);
            f[OF_NUE][e] = or_safe_clamp(f[OF_NUE][e], 0.0, nue_max);
            f[OF_PROD][e] = or_safe_clamp(f[OF_PROD][e], 0.0, prod_max);
            f[OF_TKE_SOURCE][e] = or_safe_clamp(f[OF_TKE_SOURCE][e], -prod_max, prod_max);
            f[OF_DIS_SOURCE][e] = or_safe_clamp(f[OF_DIS_SOURCE][e], -prod_max, prod_max);
            for (int q = 0; q < 6; q++) {
                const double v = f[vel[q]][e];
                f[vel[q]][e] = !or_is_finite(v) ? 0.0 : (v < -vel_max_nd) ? -vel_max_nd
                             : (v > vel_max_nd) ? vel_max_nd : v;
            }
        }
    }
    or_geom_free(&g);
}
