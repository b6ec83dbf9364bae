/*
 * or_turb.c - TurbulenceAtm::run (TEST INFRASTRUCTURE ONLY), flat terrain:
 *
 *   compute_vel_star   TurbulenceAtm.h:88-99
 *   compute_sources    TurbulenceAtm.h:323-476 with compute_k_epsilon (:481-528),
 *                      compute_k_omega (:533-650) or compute_k_omega_SST (:656-772)
 *   zero_land_cells    :301-317 (no land: nothing)
 *   clamp_nue          :271-295
 *
 * The reference's sweep is in place: each cell first floors its own tke/dis, and after its
 * closure raises tke to the column's background value k_bg; later cells of the sweep read
 * those floored values as neighbours.  compat = 1 runs that serial order (j, then k, then
 * i, as one OpenMP thread does); compat = 0 reads every neighbour from the state before
 * the call and floors afterwards, which is order-free and mirror-symmetric (the device
 * form).
 */
#include "or_internal.h"

#define TB_C_NUE   0.028                    /* TurbulenceAtm.h:158 */
#define TB_DIS_MIN 1.0e-10                  /* :161 */
#define TB_NUE_AIR 1.5e-5                   /* constructor default, :28 */

typedef struct turb_cell {
    double tke, dis;                        /* the cell's own values after the entry floors */
    double tke_im1, tke_ip1, tke_jm1, tke_jp1, tke_km1, tke_kp1;
    double dis_im1, dis_ip1, dis_jm1, dis_jp1, dis_km1, dis_kp1;
} turb_cell;

/* the closure of one cell (compute_sources body from the velocity gradients on) */
static void turb_cell_update(int im, int jm, int km, const or_params* p, const or_geom* g,
                             double* const* f, double* const* f2, int i, int j, int k,
                             const turb_cell* tc, double k_bg_nd)
{
    const size_t c = OR_IDX(i, j, k);
    const double* u = f[OF_U];
    const double* v = f[OF_V];
    const double* w = f[OF_W];
    const double rm = g->rad[i];
    const double exp_rm = 1.0 / (rm + 1.0);
    double sinthe = g->sin_w[j];
    if (sinthe == 0.0) sinthe = 1.0e-5;
    const double rmsinthe = rm * sinthe;
    const double inv_2dr = 1.0 / (2.0 * g->dr);
    const double inv_2dthe = 1.0 / (2.0 * g->dthe);
    const double inv_2dphi = 1.0 / (2.0 * g->dphi);
    const double rmet = or_metric_radius(g, p, rm);
    const double inv_rm2dthe = inv_2dthe / rmet;
    const double inv_rmsinthe2dphi = inv_2dphi / (rmet * sinthe);

    const size_t sI = (size_t)jm * km, sJ = (size_t)km;
    const double dudr = (u[c + sI] - u[c - sI]) * inv_2dr * exp_rm;
    const double dvdr = (v[c + sI] - v[c - sI]) * inv_2dr * exp_rm;
    const double dwdr = (w[c + sI] - w[c - sI]) * inv_2dr * exp_rm;
    const double dudthe = (u[c + sJ] - u[c - sJ]) * inv_rm2dthe;
    const double dvdthe = (v[c + sJ] - v[c - sJ]) * inv_rm2dthe;
    const double dwdthe = (w[c + sJ] - w[c - sJ]) * inv_rm2dthe;
    const double dudphi = (u[c + 1] - u[c - 1]) * inv_rmsinthe2dphi;
    const double dvdphi = (v[c + 1] - v[c - 1]) * inv_rmsinthe2dphi;
    const double dwdphi = (w[c + 1] - w[c - 1]) * inv_rmsinthe2dphi;

    const double tke = tc->tke, dis = tc->dis;
    const double dtkedr = (tc->tke_ip1 - tc->tke_im1) * inv_2dr * exp_rm;
    const double ddisdr = (tc->dis_ip1 - tc->dis_im1) * inv_2dr * exp_rm;
    /* compute_sources also forms the theta and phi gradients of tke/dis with 1/rmet; the
     * closures recompute them with 1/rm (:593-596, :722-725) and use only the radial ones */

    const double nue_max = 1000.0 / (p->u_0 * p->L_atm);
    double cnue;
    {
        const double dis_here = or_max(dis, TB_DIS_MIN);
        const double tke_here = or_max(tke, 0.0);
        cnue = (p->turb_model == 1) ? TB_C_NUE * tke_here * tke_here / dis_here : tke_here / dis_here;
        cnue = or_min(cnue, nue_max);
    }
    const double der = 0.66667 * (dudr + dvdthe + dwdphi);
    const double prod = or_max(0.0,
          (cnue * (2.0 * dudr - der) - 0.66667 * tke) * dudr
        + (cnue * (dudthe + dvdr)) * dudthe
        + (cnue * (dudphi + dwdr)) * dudphi
        + (cnue * (2.0 * dvdthe - der) - 0.66667 * tke) * dvdthe
        + (cnue * (dvdr + dudthe)) * dvdr
        + (cnue * (dvdphi + dwdthe)) * dvdphi
        + (cnue * (2.0 * dwdphi - der) - 0.66667 * tke) * dwdphi
        + (cnue * (dwdr + dudphi)) * dwdr
        + (cnue * (dwdthe + dvdphi)) * dwdthe);
    f[OF_PROD][c] = prod;
    const double W12 = dudthe - dvdr;
    const double W13 = dudphi - dwdr;
    const double W23 = dvdphi - dwdthe;
    const double Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);

    const double y_mount = g->height[0];
    double nue, tke_source, dis_source;
    if (p->turb_model == 1) {                 /* compute_k_epsilon, :481-528 */
        const double C_eps_1 = 1.35, C_eps_2 = 1.80;
        const double y_phys = or_max(g->height[i] - y_mount, p->L_atm);
        const double y_star = y_phys / p->L_atm;
        nue = TB_C_NUE * tke * tke / or_max(dis, TB_DIS_MIN);
        const double d_plus = y_phys * f2[OF2_VEL_STAR][(size_t)j * km + k] / TB_NUE_AIR;
        const double f_nue = 1.0 - exp(-0.0115 * d_plus);
        const double Re_T = tke * tke * p->u_0 * p->L_atm
                          / or_max(dis * TB_NUE_AIR, TB_DIS_MIN * TB_NUE_AIR);
        const double f_2 = 1.0 - 0.4 / 1.8 * exp(-Re_T * Re_T / 36.0);
        nue *= f_nue;
        const double y_star2 = y_star * y_star;
        const double L_k = -2.0 * tke / y_star2;
        const double L_w = -2.0 * dis / y_star2 * exp(-d_plus / 2.0);
        const double P_k = prod;
        const double Y_k = dis;
        const double tke_safe = or_max(tke, TB_DIS_MIN);
        const double P_w = C_eps_1 * dis / tke_safe * P_k;
        const double Y_w = C_eps_2 * f_2 * dis * dis / tke_safe;
        tke_source = P_k - Y_k + L_k / p->re_turb;
        dis_source = P_w - Y_w + L_w / p->re_turb;
    } else if (p->turb_model == 2) {          /* compute_k_omega, :533-650 */
        const double bet_star = 0.09, gam = 0.52, C_lim = 0.875, bet_0 = 0.0708;
        const double dtkedthe_neu = (tc->tke_jp1 - tc->tke_jm1) / (rm * 2.0 * g->dthe);
        const double ddisdthe_neu = (tc->dis_jp1 - tc->dis_jm1) / (rm * 2.0 * g->dthe);
        const double dtkedphi_neu = (tc->tke_kp1 - tc->tke_km1) / (rmsinthe * 2.0 * g->dphi);
        const double ddisdphi_neu = (tc->dis_kp1 - tc->dis_km1) / (rmsinthe * 2.0 * g->dphi);
        const double dudr_u = (u[c + sI] - u[c - sI]) / (2.0 * g->dr) / (rm + 1.0);
        const double dvdthe_u = (v[c + sJ] - v[c - sJ]) / (rm * 2.0 * g->dthe);
        const double dwdphi_u = (w[c + 1] - w[c - 1]) / (rmsinthe * 2.0 * g->dphi);
        const double dudthe_u = (u[c + sJ] - u[c - sJ]) / (rm * 2.0 * g->dthe);
        const double dudphi_u = (u[c + 1] - u[c - 1]) / (rmsinthe * 2.0 * g->dphi);
        const double dvdr_u = (v[c + sI] - v[c - sI]) / (2.0 * g->dr) / (rm + 1.0);
        const double dwdr_u = (w[c + sI] - w[c - sI]) / (2.0 * g->dr) / (rm + 1.0);
        const double dvdphi_u = (v[c + 1] - v[c - 1]) / (rmsinthe * 2.0 * g->dphi);
        const double dwdthe_u = (w[c + sJ] - w[c - sJ]) / (rm * 2.0 * g->dthe);
        const double S11 = dudr_u, S22 = dvdthe_u, S33 = dwdphi_u;
        const double S12 = 0.5 * (dudthe_u + dvdr_u);
        const double S13 = 0.5 * (dudphi_u + dwdr_u);
        const double S23 = 0.5 * (dvdphi_u + dwdthe_u);
        const double S_mag = sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33
                                       + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23)));
        const double w_hat = or_max(dis, C_lim * S_mag / sqrt(bet_star));
        const double cross = dtkedr * ddisdr + dtkedthe_neu * ddisdthe_neu + dtkedphi_neu * ddisdphi_neu;
        const double sig_d = (cross <= 0.0) ? 0.0 : 0.125;
        const double chi_w = fabs(Omega * Omega * S_mag / pow(bet_star * or_max(dis, 1.0e-20), 3));
        const double f_bet = (1.0 + 85.0 * chi_w) / (1.0 + 100.0 * chi_w);
        const double bet_wc = bet_0 * f_bet;
        nue = tke / or_max(w_hat, 1.0e-20);
        const double P_k = or_min(prod, 20.0 * bet_star * tke * dis);
        const double Y_k = bet_star * tke * dis;
        const double P_w = gam * dis / or_max(tke, 1.0e-20) * P_k;
        const double Y_w = bet_wc * dis * dis;
        const double D_w = sig_d / or_max(dis, 1.0e-20) * cross;
        tke_source = P_k - Y_k;
        dis_source = P_w - Y_w + D_w;
    } else {                                  /* compute_k_omega_SST, :656-772 */
        const double a1 = 0.31, bet_star = 0.09, bet1 = 0.0333, bet2 = 0.0368;
        const double gam1 = 0.413, gam2 = 0.2, sig_w2 = 1.168;
        const double nue_air_nd = TB_NUE_AIR / (p->u_0 * p->L_atm);
        const double y_phys = or_max(g->height[i] - y_mount, 1.0e-6);
        const double y_star = y_phys / p->L_atm;
        const double dtkedthe_neu = (tc->tke_jp1 - tc->tke_jm1) / (rm * 2.0 * g->dthe);
        const double ddisdthe_neu = (tc->dis_jp1 - tc->dis_jm1) / (rm * 2.0 * g->dthe);
        const double dtkedphi_neu = (tc->tke_kp1 - tc->tke_km1) / (rmsinthe * 2.0 * g->dphi);
        const double ddisdphi_neu = (tc->dis_kp1 - tc->dis_km1) / (rmsinthe * 2.0 * g->dphi);
        const double cross = dtkedr * ddisdr + dtkedthe_neu * ddisdthe_neu + dtkedphi_neu * ddisdphi_neu;
        const double CD_kw = or_max(2.0 * sig_w2 / or_max(dis, 1.0e-20) * cross, 1.0e-20);
        const double dis_safe = or_max(dis, 1.0e-20);
        const double arg1 = or_min(
            or_max(sqrt(tke) / (bet_star * dis_safe * y_star),
                   500.0 * nue_air_nd / (y_star * y_star * dis_safe)),
            4.0 * sig_w2 * tke / (CD_kw * y_star * y_star));
        const double arg2 = or_max(
            2.0 * sqrt(tke) / (bet_star * dis_safe * y_star),
            500.0 * nue_air_nd / (y_star * y_star * dis_safe));
        const double F1 = tanh(pow(arg1, 4));
        const double F2 = tanh(pow(arg2, 2));
        nue = a1 * tke / or_max(a1 * dis_safe, Omega * F2);
        const double tke_safe = or_max(tke, 1.0e-20);
        const double P_k = or_min(prod, 20.0 * bet_star * tke_safe * dis_safe);
        const double Y_k = bet_star * tke_safe * dis_safe;
        const double P_w = (F1 * gam1 + (1.0 - F1) * gam2) * P_k * dis_safe / tke_safe;
        const double Y_w = (F1 * bet1 + (1.0 - F1) * bet2) * dis_safe * dis_safe;
        const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_safe * cross;
        tke_source = P_k - Y_k;
        dis_source = P_w - Y_w + D_w;
    }
    /* the end of the cell, :455-473 */
    const double tke_fin = or_max(k_bg_nd, tke);
    const double dis_fin = or_max(TB_DIS_MIN, dis);
    f[OF_NUE][c] = or_clamp(nue, 0.0, nue_max);
    const double dis_src_max = 20.0 * dis_fin * dis_fin;
    f[OF_DIS_SOURCE][c] = or_clamp(dis_source, -dis_src_max, dis_src_max);
    const double tke_src_max = 20.0 * tke_fin * dis_fin;
    f[OF_TKE_SOURCE][c] = or_clamp(tke_source, -tke_src_max, tke_src_max);
}

static double k_bg_of(const or_params* p, double vs)
{
    return 0.01 * vs * vs / (sqrt(TB_C_NUE) * p->u_0 * p->u_0);
}

void or_turbulence_run(int im, int jm, int km, const or_params* p, int compat,
                       double* const* f, double* const* f2)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    double* tke = f[OF_TKE];
    double* dis = f[OF_DIS];
    double* vs = f2[OF2_VEL_STAR];
    /* compute_vel_star, :88-99: the first air cell above flat ground is i = 1 */
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const int i_surf = (1 < im - 1) ? 1 : im - 1;
            const double v_s = f[OF_V][OR_IDX(i_surf, j, k)];
            const double w_s = f[OF_W][OR_IDX(i_surf, j, k)];
            const double U_horiz = p->u_0 * sqrt(v_s * v_s + w_s * w_s);
            vs[(size_t)j * km + k] = or_max(0.05, sqrt(0.002) * U_horiz);
        }
    const size_t n = (size_t)im * jm * km, sI = (size_t)jm * km, sJ = (size_t)km;
    if (compat) {
        for (int j = 1; j < jm - 1; j++)
            for (int k = 1; k < km - 1; k++) {
                const double k_bg_nd = k_bg_of(p, vs[(size_t)j * km + k]);
                for (int i = 1; i < im - 1; i++) {
                    const size_t c = OR_IDX(i, j, k);
                    tke[c] = or_max(0.0, tke[c]);
                    dis[c] = or_max(TB_DIS_MIN, dis[c]);
                    turb_cell tc;
                    tc.tke = tke[c]; tc.dis = dis[c];
                    tc.tke_im1 = tke[c - sI]; tc.tke_ip1 = tke[c + sI];
                    tc.tke_jm1 = tke[c - sJ]; tc.tke_jp1 = tke[c + sJ];
                    tc.tke_km1 = tke[c - 1];  tc.tke_kp1 = tke[c + 1];
                    tc.dis_im1 = dis[c - sI]; tc.dis_ip1 = dis[c + sI];
                    tc.dis_jm1 = dis[c - sJ]; tc.dis_jp1 = dis[c + sJ];
                    tc.dis_km1 = dis[c - 1];  tc.dis_kp1 = dis[c + 1];
                    turb_cell_update(im, jm, km, p, &g, f, f2, i, j, k, &tc, k_bg_nd);
                    tke[c] = or_max(k_bg_nd, tke[c]);
                    dis[c] = or_max(TB_DIS_MIN, dis[c]);
                }
            }
    } else {
        double* t0 = (double*)malloc(sizeof(double) * n);
        double* d0 = (double*)malloc(sizeof(double) * n);
        memcpy(t0, tke, sizeof(double) * n);
        memcpy(d0, dis, sizeof(double) * n);
        for (int j = 1; j < jm - 1; j++)
            for (int k = 1; k < km - 1; k++) {
                const double k_bg_nd = k_bg_of(p, vs[(size_t)j * km + k]);
                for (int i = 1; i < im - 1; i++) {
                    const size_t c = OR_IDX(i, j, k);
                    turb_cell tc;
                    tc.tke = or_max(0.0, t0[c]); tc.dis = or_max(TB_DIS_MIN, d0[c]);
                    tc.tke_im1 = t0[c - sI]; tc.tke_ip1 = t0[c + sI];
                    tc.tke_jm1 = t0[c - sJ]; tc.tke_jp1 = t0[c + sJ];
                    tc.tke_km1 = t0[c - 1];  tc.tke_kp1 = t0[c + 1];
                    tc.dis_im1 = d0[c - sI]; tc.dis_ip1 = d0[c + sI];
                    tc.dis_jm1 = d0[c - sJ]; tc.dis_jp1 = d0[c + sJ];
                    tc.dis_km1 = d0[c - 1];  tc.dis_kp1 = d0[c + 1];
                    turb_cell_update(im, jm, km, p, &g, f, f2, i, j, k, &tc, k_bg_nd);
                    tke[c] = or_max(k_bg_nd, tc.tke);
                    dis[c] = or_max(TB_DIS_MIN, tc.dis);
                }
            }
        free(t0);
        free(d0);
    }
    /* clamp_nue, :271-295: eddy viscosity tapered to zero over one layer above abl_height */
    const double nue_max = 1000.0 / (p->u_0 * p->L_atm);
    int i_abl = 0;
    while (i_abl < im - 1 && g.height[i_abl] <= p->abl_height) i_abl++;
    const int ia = (i_abl < im - 1) ? i_abl : im - 1;
    const int ib = (i_abl - 1 > 0) ? i_abl - 1 : 0;
    const double taper_dz = or_max(1.0, g.height[ia] - g.height[ib]);
    for (int i = 0; i < im; i++) {
        const double z_agl = g.height[i] - g.height[0];
        const double fac = or_clamp((p->abl_height + taper_dz - z_agl) / taper_dz, 0.0, 1.0);
        for (size_t q = (size_t)i * sI; q < (size_t)(i + 1) * sI; q++)
            f[OF_NUE][q] = or_clamp(f[OF_NUE][q], 0.0, nue_max) * fac;
    }
    or_geom_free(&g);
}
