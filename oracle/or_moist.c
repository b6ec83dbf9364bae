/*
 * or_moist.c - oracle restatement of MoistConvection::run (MoistConvection.h:106-1537).
 * TEST INFRASTRUCTURE ONLY, see athad_oracle.h.
 *
 * Every phase of the reference touches one (j, k) column at a time and reads nothing from
 * other columns except the water vapour c at j+-1 and k+-1, which no phase writes.  The
 * reference runs each phase over all columns before the next; running all phases column by
 * column gives the same result, and that is how this restatement (and the device kernel)
 * is organised.  computeCAPE (:1259-1299) only fills the 1-D diagnostic m.CAPE, written by
 * every column in a serial loop so the last column wins; nothing reads it, and it is not
 * restated.  subTerrainFill (:1487-1533) acts on land columns only and is void on flat
 * terrain.
 */
#include "or_internal.h"

/* AtomMoistConvection constants, MoistConvection.h:20-89 */
#define MC_A_EV 1.0e-3
#define MC_B_EV 5.9
#define MC_T00 236.15
#define MC_T00M2 (MC_T00 - 2.0)
#define MC_B_U 0.33
#define MC_ALF_1 0.05
#define MC_ALF_2 0.05
#define MC_BET_P 2.0e-3
#define MC_EPS_U (0.2 / 100.0)
#define MC_DEL_U MC_EPS_U
#define MC_EPS_D 1.0e-4
#define MC_DEL_D MC_EPS_D
#define MC_GAM_D (-0.3)
#define MC_A_U 3.0e-2
#define MC_A_D 3.0e-2
#define MC_VEL 1.1
#define MC_F_BEG (1000.0 / 1013.25)
#define MC_F_END (970.0 / 1013.25)
#define MC_F_CB (900.0 / 1013.25)
#define MC_F_DIFF (200.0 / 1013.25)
#define MC_F_MID (700.0 / 1013.25)
#define MC_T_ADD_U 0.2
#define MC_Q_V_U_ADD 1.0e-4
#define MC_COEFF_RECURR 0.1
#define MC_SCALE 0.98
#define MC_Q_C_U_MAX 1.0e-2
#define MC_W_CONV_MAX 50.0
#define MC_M_MAX 3.0
#define MC_C_MB 0.003

typedef struct mc_ctx {
    int im, jm, km;
    const or_params* p;
    double* const* f;
    double* const* f2;
    const double* height;   /* float-rounded layer heights */
    const double* step;     /* double differences, step[im-1] = step[im-2] (:300-309) */
    const double* cose;     /* cos(the[equator] - the[j]) (:239) */
} mc_ctx;

#define F3(name, i) (X->f[name][OR_IDX((i), j, k)])

/* clamp_M, MoistConvection.h:216-222 */
static inline double clamp_M(double v)
{
    if (!or_is_finite(v)) return 0.0;
    return (v < -MC_M_MAX) ? -MC_M_MAX : (v > MC_M_MAX) ? MC_M_MAX : v;
}
static inline double safe_r_humid(double r) { return or_max(r, 1e-6); }

/* safe_q_sat, :181-184: the reference CO2 mass fraction co2_0 with the local water */
static inline double safe_q_sat(const mc_ctx* X, double E, double p_u, double q_v)
{
    return or_saturation_mass_fraction(E, p_u, or_M_nonwater(q_v, X->p->co2_0, X->p->M_bg));
}

/* cc_factor, :191-203 */
static double cc_factor(const mc_ctx* X, double T, double p)
{
    const double t_0 = X->p->t_0;
    const double Et = (T >= t_0) ? or_saturation_pressure(T) : or_sublimation_pressure(T);
    const double Er = (288.15 >= t_0) ? or_saturation_pressure(288.15) : or_sublimation_pressure(288.15);
    const double qs_T = safe_q_sat(X, Et, p, X->p->c_0);
    const double qs_ref = safe_q_sat(X, Er, p, X->p->c_0);
    return (qs_ref > 0.0) ? qs_T / qs_ref : 1.0;
}

/* entrainmentGradients, :238-297 (flat terrain: no Neumann substitution) */
static void entrainment_gradients(const mc_ctx* X, int i, int j, int k, double* dcdr,
                                  double* dcdthe, double* dcdphi, double* c_ijk)
{
    const int im = X->im, jm = X->jm, km = X->km;
    const double* c = X->f[OF_C];
    const double costhe = X->cose[j];
    const double height = X->height[i];
    const double r_the_height = (X->p->r_Earth * 1.0e3 + height) * costhe;
    const double U_Earth = r_the_height * 2.0 * M_PI;
    const double step_dr = X->step[i];
    const double inv_step_dr = 0.5 / step_dr;
    const double inv_step_the = 0.5 / (U_Earth / (jm - 1));
    const double inv_step_phi = 1.0 / (U_Earth / (km - 1));
    const int i_p = (i + 1 < im - 1) ? i + 1 : im - 1;
    const int i_m = (i - 1 > 0) ? i - 1 : 0;
    const double c0 = c[OR_IDX(i, j, k)];
    *dcdr = (c[OR_IDX(i_p, j, k)] - c[OR_IDX(i_m, j, k)]) * inv_step_dr;
    *dcdthe = (c[OR_IDX(i, j + 1, k)] - c[OR_IDX(i, j - 1, k)]) * inv_step_the;
    *dcdphi = (c[OR_IDX(i, j, k + 1)] - c[OR_IDX(i, j, k - 1)]) * inv_step_phi;
    *c_ijk = or_max(c0, 1e-4);
}

/* simpsonCxEu, :1426-1455 */
static int simpson_cxeu(const mc_ctx* X, int j, int k, int i_beg, int i_end)
{
    const int jm = X->jm, km = X->km;
    if (i_end <= i_beg) return -1;
    const double* c = X->f[OF_C];
    const double* E_u = X->f[OF_E_U];
    double cumsum = 0.0;
    int i = i_beg;
    for (; i + 2 <= i_end; i += 2) {
        const double h1 = X->step[i], h2 = X->step[i + 1];
        const double f0 = -(c[OR_IDX(i, j, k)] * E_u[OR_IDX(i, j, k)]);
        const double f1 = -(c[OR_IDX(i + 1, j, k)] * E_u[OR_IDX(i + 1, j, k)]);
        const double f2 = -(c[OR_IDX(i + 2, j, k)] * E_u[OR_IDX(i + 2, j, k)]);
        const double pair = (h1 + h2) / 6.0
            * ((2.0 - h2 / h1) * f0 + (h1 + h2) * (h1 + h2) / (h1 * h2) * f1 + (2.0 - h1 / h2) * f2);
        if (cumsum + pair > 0.0) return (cumsum + 0.5 * h1 * (f0 + f1) > 0.0) ? i + 1 : i + 2;
        cumsum += pair;
    }
    if (i + 1 <= i_end) {
        const double f0 = -(c[OR_IDX(i, j, k)] * E_u[OR_IDX(i, j, k)]);
        const double f1 = -(c[OR_IDX(i + 1, j, k)] * E_u[OR_IDX(i + 1, j, k)]);
        if (cumsum + 0.5 * X->step[i] * (f0 + f1) > 0.0) return i + 1;
    }
    return -1;
}

/* CloudBaseUpdate for one column, :1462-1482 */
static void cloud_base_update(const mc_ctx* X, int j, int k, int i_deep_beg, int i_lfs, int* i_base)
{
    const int im = X->im, jm = X->jm, km = X->km;
    if (i_deep_beg < 0 || i_lfs <= i_deep_beg) return;
    const int is = simpson_cxeu(X, j, k, i_deep_beg, i_lfs);
    if (is >= 0 && is < im
        && X->f[OF_P_STAT][OR_IDX(is, j, k)] <= MC_F_CB * X->f[OF_P_STAT][OR_IDX(0, j, k)]
        && (*i_base <= 0 || is <= *i_base)) {
        *i_base = is;
        X->f[OF_CLOUD_BASE][OR_IDX(is, j, k)] = X->height[is];
    }
}

static void mc_column(const mc_ctx* X, int j, int k, int iter_prec_n)
{
    const int im = X->im, jm = X->jm, km = X->km;
    const or_params* p = X->p;
    double* const* f = X->f;
    const int interior = (j >= 1 && j < jm - 1 && k >= 1 && k < km - 1);
    const double t_0 = p->t_0;
    const double p0 = f[OF_P_STAT][OR_IDX(0, j, k)];

    /* precompute, :339-376 */
    for (int i = 0; i < im; i++) {
        const size_t c = OR_IDX(i, j, k);
        f[OF_MC_S][c] = p->cp_l * f[OF_T][c] * t_0 / p->s_0;
        f[OF_M_U][c] = 0.0; f[OF_M_D][c] = 0.0;
        f[OF_MC_S_U][c] = 0.0; f[OF_Q_V_U][c] = 0.0; f[OF_Q_C_U][c] = 0.0;
        f[OF_C_U][c] = 0.0; f[OF_E_L][c] = 0.0; f[OF_E_DD][c] = 0.0; f[OF_E_P][c] = 0.0;
        f[OF_G_P][c] = 0.0; f[OF_MC_S_D][c] = 0.0; f[OF_Q_V_D][c] = 0.0; f[OF_P_CONV][c] = 0.0;
    }
    int i_base = 0, i_lfs = 0, i_deep_beg = -1, i_deep_end = -1;
    double M_d_LFS = 0.0, cape_col = 0.0, dT_sfp = 0.0, dq_sfp = 0.0;

    /* findCloudBaseLFS, :627-777 (every column) */
    for (int i = 0; i < im; i++)
        if (f[OF_P_STAT][OR_IDX(i, j, k)] <= MC_F_BEG * p0) {
            i_deep_beg = i;
            f[OF_DEEP_BEG][OR_IDX(i, j, k)] = X->height[i];
            break;
        }
    for (int i = im - 1; i >= 0; i--)
        if (f[OF_P_STAT][OR_IDX(i, j, k)] >= MC_F_END * p0) {
            i_deep_end = i;
            f[OF_DEEP_END][OR_IDX(i, j, k)] = X->height[i];
            break;
        }
    double* qsc = (double*)malloc(sizeof(double) * im);
    if (i_deep_beg >= 0 && i_deep_end >= 0) {
        for (int i = i_deep_beg; i < im; i++) {
            const double t_u_add = f[OF_T][OR_IDX(i, j, k)] * t_0 + MC_T_ADD_U;
            qsc[i] = safe_q_sat(X, or_saturation_pressure_auto(t_u_add), f[OF_P_STAT][OR_IDX(i, j, k)],
                                f[OF_C][OR_IDX(i, j, k)]);
        }
        for (int i = i_deep_beg; i < im; i++) {
            const size_t c = OR_IDX(i, j, k);
            const double t_u = f[OF_T][c] * t_0;
            const double w = 1.0 / (1.0 + exp(-(t_u - MC_T00) / 2.0));
            f[OF_Q_V_U][c] = f[OF_C][c] + MC_Q_V_U_ADD;
            if (f[OF_Q_V_U][c] >= MC_SCALE * qsc[i] && t_u >= MC_T00)
                f[OF_Q_C_U][c] = f[OF_Q_V_U][c] - MC_SCALE * qsc[i];
            if (f[OF_Q_V_U][c] <= 0.0) f[OF_Q_V_U][c] = 0.0;
            if (f[OF_Q_C_U][c] <= 0.0) f[OF_Q_C_U][c] = 0.0;
            if (f[OF_Q_V_U][c] >= MC_SCALE * qsc[i] && w > 0.01 && f[OF_P_STAT][c] <= MC_F_CB * p0) {
                i_base = i;
                f[OF_CLOUD_BASE][c] = X->height[i] * w;
                break;
            }
        }
        if (i_base > 0) {   /* LNB by theta_e, :711-759 */
            const size_t cb = OR_IDX(i_base, j, k);
            const double T_b = f[OF_T][cb] * t_0 + MC_T_ADD_U;
            const double kappa = or_R_of(f[OF_C][cb], f[OF_CO2][cb], p->R_bg)
                               / or_cp_of(f[OF_C][cb], f[OF_CO2][cb], T_b, p->M_bg);
            const double p_b = f[OF_P_STAT][cb];
            const double qsb = qsc[i_base];
            const double L_b = (T_b >= t_0) ? p->lv : p->ls;
            const double th_p = T_b * pow(p->p_0 / p_b, kappa) * exp(L_b * qsb / (p->cp_l * T_b));
            int became = 0, i_top = i_base;
            double cape = 0.0;
            for (int i = i_base + 1; i < im; i++) {
                const size_t c = OR_IDX(i, j, k);
                const double T_e = f[OF_T][c] * t_0;
                const double p_e = f[OF_P_STAT][c];
                const double L_e = (T_e >= t_0) ? p->lv : p->ls;
                const double th_e = T_e * pow(p->p_0 / p_e, kappa) * exp(L_e * qsc[i] / (p->cp_l * T_e));
                if (th_p - th_e > 0.0) {
                    became = 1;
                    i_top = i;
                    const double dz = X->height[i] - X->height[i - 1];
                    cape += p->g * (th_p - th_e) / th_e * dz;
                } else if (became) {
                    break;
                }
            }
            int i_lnb = (i_top > i_base + 1) ? i_top : i_base + 1;
            if (i_lnb > im - 2) i_lnb = im - 2;
            i_lfs = i_lnb;
            cape_col = or_max(0.0, cape);
            f[OF_LEVEL_FREE_SINKING][OR_IDX(i_lnb, j, k)] = X->height[i_lnb];
        }
    }
    free(qsc);

    /* surfaceFluxPerturbations, :402-485 (interior columns) */
    if (interior) {
        if (p->convection_perturbation == 0) {
            dT_sfp = MC_T_ADD_U;
            dq_sfp = MC_Q_V_U_ADD;
        } else if (!(i_base < 0 || i_lfs <= i_base)) {
            const double T_sfc = f[OF_T][OR_IDX(0, j, k)] * t_0;
            const double rho_sfc = safe_r_humid(f[OF_R_HUMID][OR_IDX(0, j, k)]);
            const double q_cap = MC_Q_V_U_ADD * cc_factor(X, T_sfc, p0);
            const double pb = f[OF_P_STAT][OR_IDX(i_base, j, k)], pl = f[OF_P_STAT][OR_IDX(i_lfs, j, k)];
            if (pb < MC_F_MID * p0) {
                dT_sfp = MC_T_ADD_U;
                dq_sfp = q_cap;
            } else if (!((pb - pl) >= MC_F_DIFF * p0)) {
                const double H_s = X->f2[OF2_Q_SENSIBLE][(size_t)j * km + k];
                const double E = or_max(0.0, X->f2[OF2_EVAPORATION][(size_t)j * km + k]) / 86400.0;
                if (!(E <= 0.0 && H_s <= 0.0)) {
                    const double z_BL = X->height[i_base];
                    if (!(z_BL <= 0.0)) {
                        const double B = (p->g / T_sfc) * (H_s / (rho_sfc * p->cp_l) + 0.61 * T_sfc * E / rho_sfc);
                        const double w_star = cbrt(or_max(0.0, B * z_BL));
                        if (!(w_star <= 0.0)) {
                            const double inv_rho_w = 1.0 / (rho_sfc * w_star);
                            dT_sfp = or_min(0.2 * H_s * inv_rho_w / p->cp_l, MC_T_ADD_U);
                            dq_sfp = or_min(0.2 * E * inv_rho_w, q_cap);
                        }
                    }
                }
            }
        }
    }

    /* initUpdraft, :490-622 (interior columns) */
    if (interior && i_deep_beg != -1 && i_deep_end != -1) {
        const int ib = i_base, il = i_lfs;
        const double pb = f[OF_P_STAT][OR_IDX(ib, j, k)], pl = f[OF_P_STAT][OR_IDX(il, j, k)];
        f[OF_M_U][OR_IDX(i_deep_beg, j, k)] =
            clamp_M(f[OF_R_HUMID][OR_IDX(i_deep_beg, j, k)] * MC_C_MB * sqrt(2.0 * cape_col));
        for (int i = i_deep_beg + 1; i <= i_deep_end; i++) {
            const size_t c = OR_IDX(i, j, k);
            const double t_u = f[OF_T][c] * t_0, t_u_add = t_u + dT_sfp;
            const double r_h_i = f[OF_R_HUMID][c], p_u = f[OF_P_STAT][c];
            const double q_sat_add = safe_q_sat(X, or_saturation_pressure_auto(t_u_add), p_u, f[OF_C][c]);
            f[OF_Q_V_U][c] = f[OF_C][c] + dq_sfp;
            if (f[OF_Q_V_U][c] >= MC_SCALE * q_sat_add && t_u >= MC_T00)
                f[OF_Q_C_U][c] = f[OF_Q_V_U][c] - MC_SCALE * q_sat_add;
            if (f[OF_Q_V_U][c] <= 0.0) f[OF_Q_V_U][c] = 0.0;
            if (f[OF_Q_C_U][c] <= 0.0) f[OF_Q_C_U][c] = 0.0;
            double dcdr, dcdthe, dcdphi, c_ijk;
            entrainment_gradients(X, i, j, k, &dcdr, &dcdthe, &dcdphi, &c_ijk);
            if ((pb - pl) >= MC_F_DIFF * p0)
                f[OF_E_U][c] = -r_h_i / c_ijk * (f[OF_U][c] * dcdr + f[OF_V][c] * dcdthe + f[OF_W][c] * dcdphi);
            else
                f[OF_E_U][c] = 0.0;
            if (t_u <= MC_T00M2) f[OF_E_U][c] = 0.0;
            f[OF_D_U][c] = 0.0;
            const double d_Mu = f[OF_E_U][c] - f[OF_D_U][c];
            f[OF_M_U][c] = clamp_M(f[OF_M_U][OR_IDX(i - 1, j, k)] + d_Mu * X->step[i]);
            f[OF_MC_S][c] = p->cp_l * t_u / p->s_0;
            f[OF_MC_S_U][c] = p->cp_l * t_u_add / p->s_0;
            f[OF_U_U][c] = MC_VEL * f[OF_U][c];
            f[OF_V_U][c] = MC_VEL * f[OF_V][c];
            f[OF_W_U][c] = MC_VEL * f[OF_W][c];
        }
        M_d_LFS = clamp_M(MC_GAM_D * f[OF_M_U][OR_IDX(i_deep_beg, j, k)]);
        f[OF_M_D][OR_IDX(il, j, k)] = M_d_LFS;
        for (int i = i_deep_end + 1; i <= il - 1; i++) {
            const size_t c = OR_IDX(i, j, k);
            const double inv_a_u = 1.0 / (MC_A_U * p->u_0);
            const double t_u = f[OF_T][c] * t_0, r_h_i = f[OF_R_HUMID][c];
            const double t_u_add = t_u + dT_sfp, p_u = f[OF_P_STAT][c];
            const double q_sat_add = safe_q_sat(X, or_saturation_pressure_auto(t_u_add), p_u, f[OF_C][c]);
            if (i == i_deep_end + 1) f[OF_M_U][OR_IDX(i - 1, j, k)] = f[OF_M_U][OR_IDX(i_deep_beg, j, k)];
            f[OF_MC_S][c] = p->cp_l * t_u / p->s_0;
            f[OF_MC_S_U][c] = p->cp_l * t_u / p->s_0;
            f[OF_Q_V_U][c] = f[OF_C][c] + dq_sfp;
            if (f[OF_Q_V_U][c] >= MC_SCALE * q_sat_add && t_u_add >= MC_T00)
                f[OF_Q_C_U][c] = f[OF_Q_V_U][c] - MC_SCALE * q_sat_add;
            double dcdr, dcdthe, dcdphi, c_ijk;
            entrainment_gradients(X, i, j, k, &dcdr, &dcdthe, &dcdphi, &c_ijk);
            if ((pb - pl) >= MC_F_DIFF * p0)
                f[OF_E_U][c] = -r_h_i / c_ijk * (f[OF_U][c] * dcdr + f[OF_V][c] * dcdthe + f[OF_W][c] * dcdphi);
            else
                f[OF_E_U][c] = 0.0;
            if (t_u <= MC_T00M2) f[OF_E_U][c] = 0.0;
            f[OF_D_U][c] = 0.0;
            const double d_Mu = f[OF_E_U][c] - f[OF_D_U][c];
            f[OF_M_U][c] = clamp_M(f[OF_M_U][OR_IDX(i - 1, j, k)] + d_Mu * X->step[i]);
            f[OF_U_U][c] = f[OF_U][c] + f[OF_M_U][c] * inv_a_u / safe_r_humid(r_h_i);
            const double cap = MC_W_CONV_MAX / p->u_0;
            f[OF_U_U][c] = or_max(-cap, or_min(f[OF_U_U][c], cap));
            f[OF_V_U][c] = f[OF_V][c];
            f[OF_W_U][c] = f[OF_W][c];
        }
    }
    if (interior) cloud_base_update(X, j, k, i_deep_beg, i_lfs, &i_base);

    for (int ip = 1; ip <= iter_prec_n; ip++) {
        /* updraftEntrainment, :780-908 (interior columns) */
        if (interior && !(i_base < 0 || i_lfs <= i_base)) {
            const int ib = i_base, il = i_lfs;
            const double pb = f[OF_P_STAT][OR_IDX(ib, j, k)], pl = f[OF_P_STAT][OR_IDX(il, j, k)];
            const int is_shallow = p->convection_mode >= 1 && (pb - pl) < MC_F_DIFF * p0;
            const int is_mid = p->convection_mode >= 2 && pb < MC_F_MID * p0;
            const double delta_i_c = (is_shallow || is_mid) ? 1.0e9 : 500.0;
            const double height_base = X->height[ib];
            for (int ii = 0; ii < ib; ii++) f[OF_M_U][OR_IDX(ii, j, k)] = 0.0;
            f[OF_M_U][OR_IDX(ib, j, k)] = clamp_M(f[OF_R_HUMID][OR_IDX(ib, j, k)] * MC_C_MB * sqrt(2.0 * cape_col));
            {
                const double t_base = f[OF_T][OR_IDX(ib, j, k)] * t_0;
                f[OF_MC_S_U][OR_IDX(ib, j, k)] = p->cp_l * (t_base + dT_sfp) / p->s_0;
                f[OF_Q_V_U][OR_IDX(ib, j, k)] = or_max(f[OF_C][OR_IDX(ib, j, k)] + dq_sfp, 0.0);
            }
            M_d_LFS = clamp_M(MC_GAM_D * f[OF_M_U][OR_IDX(ib, j, k)]);
            for (int i = ib + 1; i <= il; i++) {
                const size_t c = OR_IDX(i, j, k);
                const double height_i = X->height[i];
                const double t_u = f[OF_T][c] * t_0, r_h_i = f[OF_R_HUMID][c];
                double dcdr, dcdthe, dcdphi, c_ijk;
                entrainment_gradients(X, i, j, k, &dcdr, &dcdthe, &dcdphi, &c_ijk);
                if ((pb - pl) >= MC_F_DIFF * p0)
                    f[OF_E_U][c] = -r_h_i / c_ijk * (f[OF_U][c] * dcdr + f[OF_V][c] * dcdthe + f[OF_W][c] * dcdphi)
                                 + MC_EPS_U * f[OF_M_U][c];
                else
                    f[OF_E_U][c] = 0.0;
                if (t_u <= MC_T00M2) f[OF_E_U][c] = 0.0;
                f[OF_D_U][c] = (i <= il) ? MC_EPS_U * f[OF_M_U][c] : 0.0;
                if (ip > 1 && i == il)
                    f[OF_D_U][c] = MC_DEL_U * f[OF_M_U][c] + MC_B_U * f[OF_M_U][c] / X->step[i];
                if (ip > 1 && i == il - 1)
                    f[OF_D_U][c] = MC_DEL_U * f[OF_M_U][c] + (1.0 - MC_B_U) * f[OF_M_U][c] / X->step[i];
                if (t_u <= MC_T00M2) f[OF_D_U][c] = 0.0;
                const double d_Mu = f[OF_E_U][c] - f[OF_D_U][c];
                f[OF_M_U][c] = clamp_M(f[OF_M_U][OR_IDX(i - 1, j, k)] + d_Mu * X->step[i]);
                f[OF_C_U][c] = 0.0;
                if (ip == 1) {
                    f[OF_E_L][c] = 0.0;
                } else {
                    const double r_h_floor = or_max(r_h_i, 0.01);
                    f[OF_E_L][c] = f[OF_D_U][c] * f[OF_Q_C_U][c] / r_h_floor;
                    if (f[OF_E_L][c] <= 0.0) f[OF_E_L][c] = 0.0;
                }
                const double K_p = (height_i > height_base + delta_i_c) ? MC_BET_P : 0.0;
                if (t_u >= t_0) f[OF_G_P][c] = (ip == 1) ? 0.0 : K_p * f[OF_Q_C_U][c];
                else f[OF_G_P][c] = 0.0;
            }
            f[OF_M_U][OR_IDX(il, j, k)] = 0.0;
        }
        if (interior) cloud_base_update(X, j, k, i_deep_beg, i_lfs, &i_base);

        /* updraftRecurrence, :1032-1163 (interior columns) */
        if (interior && !(i_base < 0 || i_lfs <= i_base)) {
            for (int i = i_base + 1; i <= i_lfs - 1; i++) {
                const size_t c = OR_IDX(i, j, k), cm = OR_IDX(i - 1, j, k);
                const double t_u = f[OF_T][cm] * t_0;
                const double r_h_prev = f[OF_R_HUMID][cm];
                const double step_prev = X->step[i - 1];
                const double r_h_i = f[OF_R_HUMID][c];
                const double d_Mu = f[OF_E_U][cm] - f[OF_D_U][cm];
                f[OF_M_U][c] = clamp_M(f[OF_M_U][cm] + d_Mu * step_prev);
                if (t_u <= MC_T00M2) f[OF_M_U][c] = 0.0;
                const double M_u_prev = f[OF_M_U][cm];
                const double dq_v = M_u_prev * f[OF_Q_V_U][cm]
                    + step_prev * (f[OF_E_U][cm] * f[OF_C][cm] - f[OF_D_U][cm] * f[OF_Q_V_U][cm]);
                const double dq_c = M_u_prev * f[OF_Q_C_U][cm]
                    + step_prev * (-f[OF_D_U][cm] * f[OF_CLOUD][cm] - r_h_prev * f[OF_G_P][cm]);
                const double dv = M_u_prev * f[OF_V_U][cm] + step_prev * f[OF_E_U][cm] * f[OF_V][cm];
                const double dw = M_u_prev * f[OF_W_U][cm] + step_prev * f[OF_E_U][cm] * f[OF_W][cm];
                const double ds = (M_u_prev * f[OF_MC_S_U][cm]
                    + step_prev * (f[OF_E_U][cm] * f[OF_MC_S][cm] - f[OF_D_U][cm] * f[OF_MC_S_U][cm])) / p->s_0;
                const double M_u_i = f[OF_M_U][c];
                if (fabs(M_u_i) > MC_COEFF_RECURR) {
                    const double inv = 1.0 / M_u_i;
                    f[OF_Q_V_U][c] = dq_v * inv;
                    f[OF_Q_C_U][c] = dq_c * inv;
                    f[OF_V_U][c] = dv * inv;
                    f[OF_W_U][c] = dw * inv;
                    f[OF_MC_S_U][c] = ds * inv;
                } else {
                    f[OF_MC_S_U][c] = f[OF_MC_S][c];
                    f[OF_Q_V_U][c] = f[OF_C][c];
                    f[OF_Q_C_U][c] = 0.0;
                    f[OF_V_U][c] = f[OF_V][c];
                    f[OF_W_U][c] = f[OF_W][c];
                }
                f[OF_C_U][c] = 0.0;
                if (fabs(f[OF_M_U][c]) > MC_COEFF_RECURR) {
                    double T_u = f[OF_MC_S_U][c] * p->s_0 / p->cp_l;
                    const double p_u = f[OF_P_STAT][c];
                    double dcond_tot = 0.0;
                    for (int it = 0; it < 2; ++it) {
                        const double E_s = or_saturation_pressure_auto(T_u);
                        const double q_sat_u = safe_q_sat(X, E_s, p_u, f[OF_C][c]);
                        const double dq = f[OF_Q_V_U][c] - q_sat_u;
                        if (dq <= 0.0) break;
                        const double L_u = (T_u >= t_0) ? p->lv : p->ls;
                        const double M_o_u = or_M_nonwater(f[OF_C][c], f[OF_CO2][c], p->M_bg);
                        const double dqsdT = or_dqsat_dT(T_u, p_u, M_o_u);
                        const double G = (L_u / p->cp_l) * dqsdT;
                        const double dcond = dq / (1.0 + G);
                        f[OF_Q_V_U][c] -= dcond;
                        f[OF_Q_C_U][c] += dcond;
                        T_u += (L_u / p->cp_l) * dcond;
                        dcond_tot += dcond;
                    }
                    f[OF_MC_S_U][c] = p->cp_l * T_u / p->s_0;
                    f[OF_C_U][c] = dcond_tot * f[OF_M_U][c] / (or_max(r_h_i, 0.01) * X->step[i]);
                }
                const double inv_a_u = 1.0 / (MC_A_U * p->u_0);
                f[OF_U_U][c] = f[OF_U][c] + f[OF_M_U][c] * inv_a_u / safe_r_humid(r_h_i);
                const double cap = MC_W_CONV_MAX / p->u_0;
                f[OF_U_U][c] = or_max(-cap, or_min(f[OF_U_U][c], cap));
                if (f[OF_Q_V_U][c] <= 0.0) f[OF_Q_V_U][c] = 0.0;
                if (f[OF_Q_C_U][c] <= 0.0) f[OF_Q_C_U][c] = 0.0;
                if (f[OF_Q_C_U][c] > MC_Q_C_U_MAX) f[OF_Q_C_U][c] = MC_Q_C_U_MAX;
                if (f[OF_MC_S_U][c] <= 0.0) f[OF_MC_S_U][c] = 0.0;
                if (t_u <= MC_T00) {
                    f[OF_E_U][c] = 0.0; f[OF_D_U][c] = 0.0; f[OF_M_U][c] = 0.0;
                    f[OF_Q_V_U][c] = 0.0; f[OF_Q_C_U][c] = 0.0;
                    f[OF_U_U][c] = 0.0; f[OF_V_U][c] = 0.0; f[OF_W_U][c] = 0.0;
                    f[OF_MC_S_U][c] = 1.0;
                    f[OF_G_P][c] = 0.0; f[OF_C_U][c] = 0.0; f[OF_E_L][c] = 0.0;
                }
            }
        }

        /* downdraftEntrainment, :913-1027 (every column) */
        if (!(i_lfs <= 0 || i_lfs <= i_base)) {
            const int il = i_lfs, ib = i_base;
            const size_t cl = OR_IDX(il, j, k);
            double t_u = f[OF_T][cl] * t_0;
            double p_u = f[OF_P_STAT][cl];
            f[OF_M_D][cl] = clamp_M(M_d_LFS);
            f[OF_E_D][cl] = MC_EPS_D * fabs(f[OF_M_D][cl]);
            f[OF_D_D][cl] = MC_DEL_D * fabs(f[OF_M_D][cl]);
            {
                const double q_sat = safe_q_sat(X, or_saturation_pressure_auto(t_u), p_u, f[OF_C][cl]);
                f[OF_Q_V_D][cl] = 0.5 * (f[OF_CLOUD][cl] + MC_SCALE * q_sat);
            }
            const double r_humid_lfs = 1e2 * p_u / (or_R_of(f[OF_C][cl], f[OF_CO2][cl], p->R_bg) * t_u);
            const double inv_a_d0 = 1.0 / (MC_A_D * p->u_0);
            f[OF_U_D][cl] = f[OF_U][cl] + f[OF_M_D][cl] * inv_a_d0 / safe_r_humid(r_humid_lfs);
            f[OF_V_D][cl] = f[OF_V][cl];
            f[OF_W_D][cl] = f[OF_W][cl];
            f[OF_MC_S_D][cl] = f[OF_MC_S][cl];
            f[OF_P_CONV][cl] = 0.0;
            double sigma_p = 0.0;
            {
                const double w_u_cb = fabs(f[OF_W_U][OR_IDX(ib, j, k)]) * p->u_0;
                if (w_u_cb > 0.0)
                    sigma_p = fabs(f[OF_M_U][OR_IDX(ib, j, k)]) / (safe_r_humid(f[OF_R_HUMID][OR_IDX(ib, j, k)]) * w_u_cb);
                sigma_p = or_min(sigma_p, 1.0);
            }
            for (int i = il - 1; i >= 0; i--) {
                const size_t c = OR_IDX(i, j, k);
                p_u = f[OF_P_STAT][c];
                t_u = f[OF_T][c] * t_0;
                const double r_h_i = f[OF_R_HUMID][c];
                f[OF_MC_S_D][c] = p->cp_l * t_u / p->s_0;
                const double q_sat = safe_q_sat(X, or_saturation_pressure_auto(t_u), p_u, f[OF_C][c]);
                f[OF_Q_V_D][c] = 0.5 * (f[OF_CLOUD][c] + MC_SCALE * q_sat);
                f[OF_E_D][c] = MC_EPS_D * fabs(f[OF_M_D][c]);
                f[OF_D_D][c] = MC_DEL_D * fabs(f[OF_M_D][c]);
                const double d_Md = f[OF_E_D][c] - f[OF_D_D][c];
                f[OF_M_D][c] = clamp_M(f[OF_M_D][OR_IDX(i + 1, j, k)] - d_Md * X->step[i]);
                const double inv_a_d = 1.0 / (MC_A_D * p->u_0);
                f[OF_U_D][c] = f[OF_U][c] + f[OF_M_D][c] * inv_a_d / safe_r_humid(r_h_i);
                f[OF_V_D][c] = f[OF_V][c];
                f[OF_W_D][c] = f[OF_W][c];
                if (i <= ib) {
                    if (ip == 1) {
                        f[OF_E_P][c] = 0.0;
                    } else {
                        const double precip_i = f[OF_P_CONV][c];
                        if (precip_i > 0.0 && sigma_p > 0.0)
                            f[OF_E_P][c] = sigma_p * MC_ALF_1 * (q_sat - f[OF_Q_V_D][c])
                                         * sqrt(1e1 / MC_ALF_2 * precip_i / sigma_p);
                        if (f[OF_E_P][c] <= 0.0) f[OF_E_P][c] = 0.0;
                    }
                }
                if (ip == 1) {
                    f[OF_E_DD][c] = 0.0;
                } else {
                    const double precip_i = f[OF_P_CONV][c];
                    if (precip_i > 0.0) {
                        const double P_16 = pow(precip_i, 1.0 / 6.0);
                        const double P_49 = pow(precip_i, 4.0 / 9.0);
                        f[OF_E_DD][c] = MC_A_EV * (1.0 + MC_B_EV * P_16) * (q_sat - f[OF_Q_V_D][c]) * P_49;
                    } else {
                        f[OF_E_DD][c] = 0.0;
                    }
                    if (f[OF_E_DD][c] <= 0.0) f[OF_E_DD][c] = 0.0;
                }
            }
        }

        /* downdraftRecurrence, :1168-1254 (every column) */
        for (int i = i_lfs - 1; i >= 0; i--) {
            const size_t c = OR_IDX(i, j, k), cp = OR_IDX(i + 1, j, k);
            const double t_u = f[OF_T][c] * t_0;
            const double step_ip1 = X->step[i + 1];
            const double r_h_ip1 = f[OF_R_HUMID][cp], r_h_i = f[OF_R_HUMID][c];
            const double d_Md = f[OF_E_D][c] - f[OF_D_D][c];
            f[OF_M_D][c] = clamp_M(f[OF_M_D][cp] - d_Md * step_ip1);
            if (t_u <= MC_T00M2) f[OF_M_D][c] = 0.0;
            const double L_latent = (t_u >= t_0) ? p->lv : p->ls;
            const double M_d_ip1 = f[OF_M_D][cp];
            const double dq_v = M_d_ip1 * f[OF_Q_V_D][cp]
                - step_ip1 * (f[OF_E_D][cp] * f[OF_C][cp] - f[OF_D_D][cp] * f[OF_Q_V_D][cp]
                              + r_h_ip1 * f[OF_E_DD][cp]);
            const double dv = M_d_ip1 * f[OF_V_D][cp]
                - step_ip1 * (f[OF_E_D][cp] * f[OF_V][cp] - f[OF_D_D][cp] * f[OF_V_D][cp]);
            const double dw = M_d_ip1 * f[OF_W_D][cp]
                - step_ip1 * (f[OF_E_D][cp] * f[OF_W][cp] - f[OF_D_D][cp] * f[OF_W_D][cp]);
            const double ds = (M_d_ip1 * f[OF_MC_S_D][cp]
                - step_ip1 * (f[OF_E_D][cp] * f[OF_MC_S][cp] - f[OF_D_D][cp] * f[OF_MC_S_D][cp]
                              - L_latent * r_h_ip1 * f[OF_E_DD][cp])) / p->s_0;
            const double M_d_i = f[OF_M_D][c];
            if (fabs(M_d_i) > MC_COEFF_RECURR) {
                const double inv = 1.0 / M_d_i;
                f[OF_Q_V_D][c] = dq_v * inv;
                f[OF_V_D][c] = dv * inv;
                f[OF_W_D][c] = dw * inv;
                f[OF_MC_S_D][c] = ds * inv;
            } else {
                f[OF_Q_V_D][c] = f[OF_C][c];
                f[OF_V_D][c] = f[OF_V][c];
                f[OF_W_D][c] = f[OF_W][c];
                f[OF_MC_S_D][c] = f[OF_MC_S][c];
            }
            const double inv_a_d = 1.0 / (MC_A_D * p->u_0);
            f[OF_U_D][c] = f[OF_U][c] + f[OF_M_D][c] * inv_a_d / safe_r_humid(r_h_i);
            if (f[OF_Q_V_D][c] <= 0.0) f[OF_Q_V_D][c] = 0.0;
            if (f[OF_MC_S_D][c] <= 0.0) f[OF_MC_S_D][c] = 0.0;
            if (t_u <= MC_T00) {
                f[OF_E_D][c] = 0.0; f[OF_D_D][c] = 0.0; f[OF_M_D][c] = 0.0;
                f[OF_Q_V_D][c] = 0.0;
                f[OF_U_D][c] = 0.0; f[OF_V_D][c] = 0.0; f[OF_W_D][c] = 0.0;
                f[OF_MC_S_D][c] = 1.0; f[OF_E_DD][c] = 0.0; f[OF_E_P][c] = 0.0;
            }
            if (i > 0)
                f[OF_P_CONV][c] = or_max(0.0, f[OF_P_CONV][cp] + X->step[i] * f[OF_R_HUMID][c]
                                          * (f[OF_G_P][c] - f[OF_E_DD][c] - f[OF_E_P][c]));
        }
        f[OF_P_CONV][OR_IDX(0, j, k)] = f[OF_P_CONV][OR_IDX(1, j, k)];
    }

    /* rhsForcing, :1304-1417 */
    for (int i = 0; i < im; i++) {
        const size_t c = OR_IDX(i, j, k);
        const double vu = f[OF_M_U][c], vd = f[OF_M_D][c];
        f[OF_M_U][c] = !or_is_finite(vu) ? 0.0 : (vu < -3.0) ? -3.0 : (vu > 3.0) ? 3.0 : vu;
        f[OF_M_D][c] = !or_is_finite(vd) ? 0.0 : (vd < -3.0) ? -3.0 : (vd > 3.0) ? 3.0 : vd;
    }
    for (int i = 0; i < im - 1; i++) {
        const size_t c = OR_IDX(i, j, k), cp = OR_IDX(i + 1, j, k);
        const double L_latent = (f[OF_T][c] * t_0 >= t_0) ? p->lv : p->ls;
        const double inv_step_rh = 1.0 / (X->step[i] * or_max(f[OF_R_HUMID][c], 0.01));
        const double Mu1 = f[OF_M_U][cp], Md1 = f[OF_M_D][cp], Mu0 = f[OF_M_U][c], Md0 = f[OF_M_D][c];
        const double fs1 = Mu1 * (f[OF_MC_S_U][cp] - f[OF_MC_S][cp]) + Md1 * (f[OF_MC_S_D][cp] - f[OF_MC_S][cp]);
        const double fs0 = Mu0 * (f[OF_MC_S_U][c] - f[OF_MC_S][c]) + Md0 * (f[OF_MC_S_D][c] - f[OF_MC_S][c]);
        const double conv_src = f[OF_C_U][c] - f[OF_E_DD][c] - f[OF_E_L][c] - f[OF_E_P][c];
        double v = -(fs1 - fs0) * inv_step_rh * t_0 + (L_latent / p->cp_l) * conv_src * t_0;
        f[OF_MC_T][c] = !or_is_finite(v) ? 0.0 : (v < -0.01) ? -0.01 : (v > 0.01) ? 0.01 : v;
        const double fq1 = Mu1 * (f[OF_Q_V_U][cp] - f[OF_C][cp]) + Md1 * (f[OF_Q_V_D][cp] - f[OF_C][cp]);
        const double fq0 = Mu0 * (f[OF_Q_V_U][c] - f[OF_C][c]) + Md0 * (f[OF_Q_V_D][c] - f[OF_C][c]);
        v = -(fq1 - fq0) * inv_step_rh - conv_src;
        f[OF_MC_Q][c] = !or_is_finite(v) ? 0.0 : (v < -2.0e-5) ? -2.0e-5 : (v > 2.0e-5) ? 2.0e-5 : v;
        const double fv1 = Mu1 * (f[OF_V_U][cp] - f[OF_V][cp]) + Md1 * (f[OF_V_D][cp] - f[OF_V][cp]);
        const double fv0 = Mu0 * (f[OF_V_U][c] - f[OF_V][c]) + Md0 * (f[OF_V_D][c] - f[OF_V][c]);
        v = -(fv1 - fv0) * inv_step_rh * p->u_0;
        f[OF_MC_V][c] = !or_is_finite(v) ? 0.0 : (v < -0.01) ? -0.01 : (v > 0.01) ? 0.01 : v;
        const double fw1 = Mu1 * (f[OF_W_U][cp] - f[OF_W][cp]) + Md1 * (f[OF_W_D][cp] - f[OF_W][cp]);
        const double fw0 = Mu0 * (f[OF_W_U][c] - f[OF_W][c]) + Md0 * (f[OF_W_D][c] - f[OF_W][c]);
        v = -(fw1 - fw0) * inv_step_rh * p->u_0;
        f[OF_MC_W][c] = !or_is_finite(v) ? 0.0 : (v < -0.01) ? -0.01 : (v > 0.01) ? 0.01 : v;
    }
}

/* The layer heights, the level steps of MoistConvection::precompute (MoistConvection.h:300-309)
   and cos(theta_equator - theta_j) of entrainmentGradients (:239) */
static void mc_geometry(const or_geom* g, int im, int jm, int compat, double* height, double* step,
                        double* cose)
{
    for (int i = 0; i < im; i++) height[i] = g->height[i];
    for (int i = 0; i < im - 1; i++) step[i] = g->height[i + 1] - g->height[i];
    step[im - 1] = (im >= 2) ? step[im - 2] : 0.0;
    /* the equator row: the.z[90] at the reference's 181 rows (:239), (jm-1)/2 in general */
    const int je = (jm - 1) / 2;
    for (int j = 0; j < jm; j++) {
        if (compat) cose[j] = cos(g->the[je] - g->the[j]);
        else {
            const int jj = (j < jm - 1 - j) ? j : jm - 1 - j;
            cose[j] = cos(g->the[je] - g->the[jj]);
        }
    }
}

int or_moist_geometry(int im, int jm, int km, const or_params* p, int compat, double* height,
                      double* step, double* cose)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    mc_geometry(&g, im, jm, compat, height, step, cose);
    or_geom_free(&g);
    return 0;
}

int or_moist_convection(int im, int jm, int km, const or_params* p, int compat, int iter_n,
                        double* const* f, double* const* f2)
{
    (void)iter_n;
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    double* height = (double*)malloc(sizeof(double) * im);
    double* step = (double*)malloc(sizeof(double) * im);
    double* cose = (double*)malloc(sizeof(double) * jm);
    mc_geometry(&g, im, jm, compat, height, step, cose);
    mc_ctx X = {im, jm, km, p, f, f2, height, step, cose};
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) mc_column(&X, j, k, p->iter_prec);
    free(height);
    free(step);
    free(cose);
    or_geom_free(&g);
    return 0;
}
