// k_moist.cu - deep moist convection of the ATHAD_COND atmosphere on sm_100a.
//
// Replaces MoistConvection::run (MoistConvection.h:106-1537) for flat terrain.  Every phase
// of the reference (precompute, findCloudBaseLFS, surfaceFluxPerturbations, initUpdraft,
// CloudBaseUpdate, iter_prec x {updraftEntrainment, CloudBaseUpdate, updraftRecurrence,
// downdraftEntrainment, downdraftRecurrence}, rhsForcing) works on one (j, k) column and
// reads nothing from other columns except the water vapour c at j+-1 and k+-1, which no
// phase writes.  So one thread runs all phases for its column, k on threadIdx.x for
// coalesced access, the column's indices and mass-flux seeds in registers.  computeCAPE
// (:1259-1299) only fills a diagnostic 1-D vector in a serial last-column-wins loop and is
// not reproduced; subTerrainFill (:1487-1533) acts on land columns only.
#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {

using namespace thermo;

// AtomMoistConvection constants, MoistConvection.h:20-89
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

#define IDX(i, j, k) idx3(d, (i), (j), (k))

// The column code is __host__ __device__: the kernel runs it on the device, and a host build
// of this file runs the same source against the oracle on the CPU (tests/host_moist.cu).

// clamp_M, MoistConvection.h:216-222
__host__ __device__ __forceinline__ double clamp_M(double v)
{
    if (!is_finite_bits(v)) return 0.0;
    return (v < -MC_M_MAX) ? -MC_M_MAX : (v > MC_M_MAX) ? MC_M_MAX : v;
}
__host__ __device__ __forceinline__ double safe_r_humid(double r) { return smax(r, 1e-6); }

// a - b rounded on its own: where the serial order stores a product and subtracts the
// reloaded value, the register form must not fuse the two into one multiply-add
__host__ __device__ __forceinline__ double sub_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}

// safe_q_sat, :181-184: the reference CO2 mass fraction co2_0 with the local water
__host__ __device__ __forceinline__ double safe_q_sat(const MoistArgs& X, double E, double p_u, double q_v)
{
    return saturation_mass_fraction(E, p_u, M_nonwater(q_v, X.co2_0, X.M_bg));
}

// cc_factor, :191-203
__host__ __device__ double cc_factor(const MoistArgs& X, double T, double p)
{
    const double Et = (T >= X.t_0) ? saturation_pressure(T) : sublimation_pressure(T);
    const double Er = (288.15 >= X.t_0) ? saturation_pressure(288.15) : sublimation_pressure(288.15);
    const double qs_T = safe_q_sat(X, Et, p, X.c_0);
    const double qs_ref = safe_q_sat(X, Er, p, X.c_0);
    return (qs_ref > 0.0) ? qs_T / qs_ref : 1.0;
}

// entrainmentGradients, :238-297 (flat terrain)
__host__ __device__ void entrainment_gradients(const MoistArgs& X, int i, int j, int k, double* dcdr,
                                               double* dcdthe, double* dcdphi, double* c_ijk)
{
    const Dims& d = X.d;
    const double* c = X.F[ATHAD_C];
    const double costhe = X.cose[j];
    const double height = X.height[i];
    const double r_the_height = (X.r_Earth * 1.0e3 + height) * costhe;
    const double U_Earth = r_the_height * 2.0 * M_PI;
    const double inv_step_dr = 0.5 / X.step[i];
    const double inv_step_the = 0.5 / (U_Earth / (d.jm - 1));
    const double inv_step_phi = 1.0 / (U_Earth / (d.km - 1));
    const int i_p = (i + 1 < d.im - 1) ? i + 1 : d.im - 1;
    const int i_m = (i - 1 > 0) ? i - 1 : 0;
    *dcdr = (c[IDX(i_p, j, k)] - c[IDX(i_m, j, k)]) * inv_step_dr;
    *dcdthe = (c[IDX(i, j + 1, k)] - c[IDX(i, j - 1, k)]) * inv_step_the;
    *dcdphi = (c[IDX(i, j, k + 1)] - c[IDX(i, j, k - 1)]) * inv_step_phi;
    *c_ijk = smax(c[IDX(i, j, k)], 1e-4);
}

// simpsonCxEu, :1426-1455
__host__ __device__ int simpson_cxeu(const MoistArgs& X, int j, int k, int i_beg, int i_end)
{
    const Dims& d = X.d;
    if (i_end <= i_beg) return -1;
    const double* c = X.F[ATHAD_C];
    const double* E_u = X.F[ATHAD_E_U];
    double cumsum = 0.0;
    int i = i_beg;
    for (; i + 2 <= i_end; i += 2) {
        const double h1 = X.step[i], h2 = X.step[i + 1];
        const double f0 = -(c[IDX(i, j, k)] * E_u[IDX(i, j, k)]);
        const double f1 = -(c[IDX(i + 1, j, k)] * E_u[IDX(i + 1, j, k)]);
        const double f2 = -(c[IDX(i + 2, j, k)] * E_u[IDX(i + 2, j, k)]);
        const double pair = (h1 + h2) / 6.0
            * ((2.0 - h2 / h1) * f0 + (h1 + h2) * (h1 + h2) / (h1 * h2) * f1 + (2.0 - h1 / h2) * f2);
        if (cumsum + pair > 0.0) return (cumsum + 0.5 * h1 * (f0 + f1) > 0.0) ? i + 1 : i + 2;
        cumsum += pair;
    }
    if (i + 1 <= i_end) {
        const double f0 = -(c[IDX(i, j, k)] * E_u[IDX(i, j, k)]);
        const double f1 = -(c[IDX(i + 1, j, k)] * E_u[IDX(i + 1, j, k)]);
        if (cumsum + 0.5 * X.step[i] * (f0 + f1) > 0.0) return i + 1;
    }
    return -1;
}

// CloudBaseUpdate for one column, :1462-1482
__host__ __device__ void cloud_base_update(const MoistArgs& X, int j, int k, int i_deep_beg, int i_lfs, int* i_base)
{
    const Dims& d = X.d;
    if (i_deep_beg < 0 || i_lfs <= i_deep_beg) return;
    const int is = simpson_cxeu(X, j, k, i_deep_beg, i_lfs);
    if (is >= 0 && is < d.im
        && X.F[ATHAD_P_STAT][IDX(is, j, k)] <= MC_F_CB * X.F[ATHAD_P_STAT][IDX(0, j, k)]
        && (*i_base <= 0 || is <= *i_base)) {
        *i_base = is;
        X.F[ATHAD_CLOUD_BASE][IDX(is, j, k)] = X.height[is];
    }
}

// q_sat_col of findCloudBaseLFS (:670-678), evaluated where it is used
#define QSC(ii) safe_q_sat(X, saturation_pressure_auto(p->F[ATHAD_T][IDX((ii), j, k)] * t_0 + MC_T_ADD_U), \
                           p->F[ATHAD_P_STAT][IDX((ii), j, k)], p->F[ATHAD_C][IDX((ii), j, k)])

__host__ __device__ void mc_column(const MoistArgs& X, int j, int k)
{
    const Dims& d = X.d;
    const int im = d.im, jm = d.jm, km = d.km;
    const MoistArgs* p = &X;
    const int interior = (j >= 1 && j < jm - 1 && k >= 1 && k < km - 1);
    const double t_0 = p->t_0;
    const double p0 = p->F[ATHAD_P_STAT][IDX(0, j, k)];

    /* precompute, :339-376.  T is not written here: the next level's value is loaded while
       this level's stores go out. */
    const long long plane_s = (long long)jm * d.pitch;   // IDX(i + 1, j, k) - IDX(i, j, k)
    {
        const double* T = p->F[ATHAD_T];
        double t_cur = T[IDX(0, j, k)];
        for (int i = 0; i < im; i++) {
            const long long c = IDX(i, j, k);
            const double t_nxt = (i + 1 < im) ? T[c + plane_s] : 0.0;
            p->F[ATHAD_MC_S][c] = p->cp_l * t_cur * t_0 / p->s_0;
            p->F[ATHAD_M_U][c] = 0.0; p->F[ATHAD_M_D][c] = 0.0;
            p->F[ATHAD_MC_S_U][c] = 0.0; p->F[ATHAD_Q_V_U][c] = 0.0; p->F[ATHAD_Q_C_U][c] = 0.0;
            p->F[ATHAD_C_U][c] = 0.0; p->F[ATHAD_E_L][c] = 0.0; p->F[ATHAD_E_DD][c] = 0.0; p->F[ATHAD_E_P][c] = 0.0;
            p->F[ATHAD_G_P][c] = 0.0; p->F[ATHAD_MC_S_D][c] = 0.0; p->F[ATHAD_Q_V_D][c] = 0.0; p->F[ATHAD_P_CONV][c] = 0.0;
            t_cur = t_nxt;
        }
    }
    int i_base = 0, i_lfs = 0, i_deep_beg = -1, i_deep_end = -1;
    double M_d_LFS = 0.0, cape_col = 0.0, dT_sfp = 0.0, dq_sfp = 0.0;

    /* findCloudBaseLFS, :627-777 (every column).  Each level's loads are issued before the
       previous level's values are used: the two searches read p_stat four levels at a time,
       the cloud-base search loads the next level while this one computes.  The loops store
       only at the level they are on, so every value is the one the serial order reads. */
    {
        const double* P = p->F[ATHAD_P_STAT];
        for (int i0 = 0; i0 < im && i_deep_beg < 0; i0 += 4) {
            double pv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) pv[q] = (i0 + q < im) ? P[IDX(i0 + q, j, k)] : 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (i_deep_beg < 0 && i0 + q < im && pv[q] <= MC_F_BEG * p0) i_deep_beg = i0 + q;
        }
        if (i_deep_beg >= 0) p->F[ATHAD_DEEP_BEG][IDX(i_deep_beg, j, k)] = p->height[i_deep_beg];
        for (int i0 = im - 1; i0 >= 0 && i_deep_end < 0; i0 -= 4) {
            double pv[4];
#pragma unroll
            for (int q = 0; q < 4; q++) pv[q] = (i0 - q >= 0) ? P[IDX(i0 - q, j, k)] : 0.0;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (i_deep_end < 0 && i0 - q >= 0 && pv[q] >= MC_F_END * p0) i_deep_end = i0 - q;
        }
        if (i_deep_end >= 0) p->F[ATHAD_DEEP_END][IDX(i_deep_end, j, k)] = p->height[i_deep_end];
    }
    if (i_deep_beg >= 0 && i_deep_end >= 0) {
        {
            const long long c0 = IDX(i_deep_beg, j, k);
            double Tn = p->F[ATHAD_T][c0], Pn = p->F[ATHAD_P_STAT][c0];
            double Cn = p->F[ATHAD_C][c0], QCn = p->F[ATHAD_Q_C_U][c0];
            for (int i = i_deep_beg; i < im; i++) {
                const long long c = IDX(i, j, k);
                const double Tc = Tn, Pc = Pn, Cc = Cn;
                double qcu = QCn;
                if (i + 1 < im) {
                    Tn = p->F[ATHAD_T][c + plane_s]; Pn = p->F[ATHAD_P_STAT][c + plane_s];
                    Cn = p->F[ATHAD_C][c + plane_s]; QCn = p->F[ATHAD_Q_C_U][c + plane_s];
                }
                const double t_u = Tc * t_0;
                const double w = 1.0 / (1.0 + exp(-(t_u - MC_T00) / 2.0));
                const double qsc = safe_q_sat(X, saturation_pressure_auto(Tc * t_0 + MC_T_ADD_U), Pc, Cc);
                double qvu = Cc + MC_Q_V_U_ADD;
                if (qvu >= MC_SCALE * qsc && t_u >= MC_T00) qcu = qvu - MC_SCALE * qsc;
                if (qvu <= 0.0) qvu = 0.0;
                if (qcu <= 0.0) qcu = 0.0;
                p->F[ATHAD_Q_V_U][c] = qvu;
                p->F[ATHAD_Q_C_U][c] = qcu;
                if (qvu >= MC_SCALE * qsc && w > 0.01 && Pc <= MC_F_CB * p0) {
                    i_base = i;
                    p->F[ATHAD_CLOUD_BASE][c] = p->height[i] * w;
                    break;
                }
            }
        }
        if (i_base > 0) {   /* LNB by theta_e, :711-759 */
            const long long cb = IDX(i_base, j, k);
            const double T_b = p->F[ATHAD_T][cb] * t_0 + MC_T_ADD_U;
            const double kappa = R_of(p->F[ATHAD_C][cb], p->F[ATHAD_CO2][cb], p->R_bg)
                               / cp_of(p->F[ATHAD_C][cb], p->F[ATHAD_CO2][cb], T_b, p->M_bg);
            const double p_b = p->F[ATHAD_P_STAT][cb];
            const double qsb = QSC(i_base);
            const double L_b = (T_b >= t_0) ? p->lv : p->ls;
            const double th_p = T_b * pow(p->p_0 / p_b, kappa) * exp(L_b * qsb / (p->cp_l * T_b));
            int became = 0, i_top = i_base;
            double cape = 0.0;
            for (int i = i_base + 1; i < im; i++) {
                const long long c = IDX(i, j, k);
                const double T_e = p->F[ATHAD_T][c] * t_0;
                const double p_e = p->F[ATHAD_P_STAT][c];
                const double L_e = (T_e >= t_0) ? p->lv : p->ls;
                const double th_e = T_e * pow(p->p_0 / p_e, kappa) * exp(L_e * QSC(i) / (p->cp_l * T_e));
                if (th_p - th_e > 0.0) {
                    became = 1;
                    i_top = i;
                    const double dz = p->height[i] - p->height[i - 1];
                    cape += p->g * (th_p - th_e) / th_e * dz;
                } else if (became) {
                    break;
                }
            }
            int i_lnb = (i_top > i_base + 1) ? i_top : i_base + 1;
            if (i_lnb > im - 2) i_lnb = im - 2;
            i_lfs = i_lnb;
            cape_col = smax(0.0, cape);
            p->F[ATHAD_LEVEL_FREE_SINKING][IDX(i_lnb, j, k)] = p->height[i_lnb];
        }
    }

    /* surfaceFluxPerturbations, :402-485 (interior columns) */
    if (interior) {
        if (p->convection_perturbation == 0) {
            dT_sfp = MC_T_ADD_U;
            dq_sfp = MC_Q_V_U_ADD;
        } else if (!(i_base < 0 || i_lfs <= i_base)) {
            const double T_sfc = p->F[ATHAD_T][IDX(0, j, k)] * t_0;
            const double rho_sfc = safe_r_humid(p->F[ATHAD_R_HUMID][IDX(0, j, k)]);
            const double q_cap = MC_Q_V_U_ADD * cc_factor(X, T_sfc, p0);
            const double pb = p->F[ATHAD_P_STAT][IDX(i_base, j, k)], pl = p->F[ATHAD_P_STAT][IDX(i_lfs, j, k)];
            if (pb < MC_F_MID * p0) {
                dT_sfp = MC_T_ADD_U;
                dq_sfp = q_cap;
            } else if (!((pb - pl) >= MC_F_DIFF * p0)) {
                const double H_s = p->q_sensible[(long long)j * d.pitch + k];
                const double E = smax(0.0, p->evaporation[(long long)j * d.pitch + k]) / 86400.0;
                if (!(E <= 0.0 && H_s <= 0.0)) {
                    const double z_BL = p->height[i_base];
                    if (!(z_BL <= 0.0)) {
                        const double B = (p->g / T_sfc) * (H_s / (rho_sfc * p->cp_l) + 0.61 * T_sfc * E / rho_sfc);
                        const double w_star = cbrt(smax(0.0, B * z_BL));
                        if (!(w_star <= 0.0)) {
                            const double inv_rho_w = 1.0 / (rho_sfc * w_star);
                            dT_sfp = smin(0.2 * H_s * inv_rho_w / p->cp_l, MC_T_ADD_U);
                            dq_sfp = smin(0.2 * E * inv_rho_w, q_cap);
                        }
                    }
                }
            }
        }
    }

    /* initUpdraft, :490-622 (interior columns).  Every value a level reads is loaded before
       the level stores anything (a level stores only its own cells, and of the fields it
       reads only q_c_u, which it reads first), and the mass flux of the level below is
       carried in a register. */
    if (interior && i_deep_beg != -1 && i_deep_end != -1) {
        const int ib = i_base, il = i_lfs;
        const double pb = p->F[ATHAD_P_STAT][IDX(ib, j, k)], pl_p = p->F[ATHAD_P_STAT][IDX(il, j, k)];
        const double Mu_beg = clamp_M(p->F[ATHAD_R_HUMID][IDX(i_deep_beg, j, k)] * MC_C_MB * sqrt(2.0 * cape_col));
        p->F[ATHAD_M_U][IDX(i_deep_beg, j, k)] = Mu_beg;
        double Mu_m = Mu_beg;
        for (int i = i_deep_beg + 1; i <= i_deep_end; i++) {
            const long long c = IDX(i, j, k);
            const double Tc = p->F[ATHAD_T][c], r_h_i = p->F[ATHAD_R_HUMID][c], p_u = p->F[ATHAD_P_STAT][c];
            const double Cc = p->F[ATHAD_C][c];
            double qcu = p->F[ATHAD_Q_C_U][c];
            const double Uc = p->F[ATHAD_U][c], Vc = p->F[ATHAD_V][c], Wc = p->F[ATHAD_W][c];
            double dcdr, dcdthe, dcdphi, c_ijk;
            entrainment_gradients(X, i, j, k, &dcdr, &dcdthe, &dcdphi, &c_ijk);
            const double t_u = Tc * t_0, t_u_add = t_u + dT_sfp;
            const double q_sat_add = safe_q_sat(X, saturation_pressure_auto(t_u_add), p_u, Cc);
            double qvu = Cc + dq_sfp;
            if (qvu >= MC_SCALE * q_sat_add && t_u >= MC_T00) qcu = qvu - MC_SCALE * q_sat_add;
            if (qvu <= 0.0) qvu = 0.0;
            if (qcu <= 0.0) qcu = 0.0;
            p->F[ATHAD_Q_V_U][c] = qvu;
            p->F[ATHAD_Q_C_U][c] = qcu;
            double eu;
            if ((pb - pl_p) >= MC_F_DIFF * p0)
                eu = -r_h_i / c_ijk * (Uc * dcdr + Vc * dcdthe + Wc * dcdphi);
            else
                eu = 0.0;
            if (t_u <= MC_T00M2) eu = 0.0;
            p->F[ATHAD_E_U][c] = eu;
            p->F[ATHAD_D_U][c] = 0.0;
            const double d_Mu = eu - 0.0;
            const double Mu = clamp_M(Mu_m + d_Mu * p->step[i]);
            p->F[ATHAD_M_U][c] = Mu;
            Mu_m = Mu;
            p->F[ATHAD_MC_S][c] = p->cp_l * t_u / p->s_0;
            p->F[ATHAD_MC_S_U][c] = p->cp_l * t_u_add / p->s_0;
            p->F[ATHAD_U_U][c] = MC_VEL * Uc;
            p->F[ATHAD_V_U][c] = MC_VEL * Vc;
            p->F[ATHAD_W_U][c] = MC_VEL * Wc;
        }
        M_d_LFS = clamp_M(MC_GAM_D * Mu_beg);
        p->F[ATHAD_M_D][IDX(il, j, k)] = M_d_LFS;
        const double inv_a_u = 1.0 / (MC_A_U * p->u_0);
        const double cap = MC_W_CONV_MAX / p->u_0;
        Mu_m = Mu_beg;   // level i_deep_end takes the flux of i_deep_beg below
        for (int i = i_deep_end + 1; i <= il - 1; i++) {
            const long long c = IDX(i, j, k);
            const double Tc = p->F[ATHAD_T][c], r_h_i = p->F[ATHAD_R_HUMID][c], p_u = p->F[ATHAD_P_STAT][c];
            const double Cc = p->F[ATHAD_C][c];
            const double Uc = p->F[ATHAD_U][c], Vc = p->F[ATHAD_V][c], Wc = p->F[ATHAD_W][c];
            double dcdr, dcdthe, dcdphi, c_ijk;
            entrainment_gradients(X, i, j, k, &dcdr, &dcdthe, &dcdphi, &c_ijk);
            const double t_u = Tc * t_0;
            const double t_u_add = t_u + dT_sfp;
            const double q_sat_add = safe_q_sat(X, saturation_pressure_auto(t_u_add), p_u, Cc);
            if (i == i_deep_end + 1) p->F[ATHAD_M_U][IDX(i - 1, j, k)] = Mu_beg;
            p->F[ATHAD_MC_S][c] = p->cp_l * t_u / p->s_0;
            p->F[ATHAD_MC_S_U][c] = p->cp_l * t_u / p->s_0;
            const double qvu = Cc + dq_sfp;
            p->F[ATHAD_Q_V_U][c] = qvu;
            if (qvu >= MC_SCALE * q_sat_add && t_u_add >= MC_T00)
                p->F[ATHAD_Q_C_U][c] = qvu - MC_SCALE * q_sat_add;
            double eu;
            if ((pb - pl_p) >= MC_F_DIFF * p0)
                eu = -r_h_i / c_ijk * (Uc * dcdr + Vc * dcdthe + Wc * dcdphi);
            else
                eu = 0.0;
            if (t_u <= MC_T00M2) eu = 0.0;
            p->F[ATHAD_E_U][c] = eu;
            p->F[ATHAD_D_U][c] = 0.0;
            const double d_Mu = eu - 0.0;
            const double Mu = clamp_M(Mu_m + d_Mu * p->step[i]);
            p->F[ATHAD_M_U][c] = Mu;
            Mu_m = Mu;
            double uu = Uc + Mu * inv_a_u / safe_r_humid(r_h_i);
            uu = smax(-cap, smin(uu, cap));
            p->F[ATHAD_U_U][c] = uu;
            p->F[ATHAD_V_U][c] = Vc;
            p->F[ATHAD_W_U][c] = Wc;
        }
    }
    if (interior) cloud_base_update(X, j, k, i_deep_beg, i_lfs, &i_base);

    for (int ip = 1; ip <= p->iter_prec; ip++) {
        /* updraftEntrainment, :780-908 (interior columns) */
        if (interior && !(i_base < 0 || i_lfs <= i_base)) {
            const int ib = i_base, il = i_lfs;
            const double pb = p->F[ATHAD_P_STAT][IDX(ib, j, k)], pl = p->F[ATHAD_P_STAT][IDX(il, j, k)];
            const int is_shallow = p->convection_mode >= 1 && (pb - pl) < MC_F_DIFF * p0;
            const int is_mid = p->convection_mode >= 2 && pb < MC_F_MID * p0;
            const double delta_i_c = (is_shallow || is_mid) ? 1.0e9 : 500.0;
            const double height_base = p->height[ib];
            for (int ii = 0; ii < ib; ii++) p->F[ATHAD_M_U][IDX(ii, j, k)] = 0.0;
            p->F[ATHAD_M_U][IDX(ib, j, k)] = clamp_M(p->F[ATHAD_R_HUMID][IDX(ib, j, k)] * MC_C_MB * sqrt(2.0 * cape_col));
            {
                const double t_base = p->F[ATHAD_T][IDX(ib, j, k)] * t_0;
                p->F[ATHAD_MC_S_U][IDX(ib, j, k)] = p->cp_l * (t_base + dT_sfp) / p->s_0;
                p->F[ATHAD_Q_V_U][IDX(ib, j, k)] = smax(p->F[ATHAD_C][IDX(ib, j, k)] + dq_sfp, 0.0);
            }
            M_d_LFS = clamp_M(MC_GAM_D * p->F[ATHAD_M_U][IDX(ib, j, k)]);
            double Mu_m = p->F[ATHAD_M_U][IDX(ib, j, k)];   // level i-1 as this loop left it
            for (int i = ib + 1; i <= il; i++) {
                const long long c = IDX(i, j, k);
                const double height_i = p->height[i];
                const double t_u = p->F[ATHAD_T][c] * t_0, r_h_i = p->F[ATHAD_R_HUMID][c];
                double dcdr, dcdthe, dcdphi, c_ijk;
                entrainment_gradients(X, i, j, k, &dcdr, &dcdthe, &dcdphi, &c_ijk);
                const double Mu_c = p->F[ATHAD_M_U][c];   // the previous pass's mass flux here
                const double qcu_c = p->F[ATHAD_Q_C_U][c];  // not written by this loop
                double eu;
                if ((pb - pl) >= MC_F_DIFF * p0)
                    eu = -r_h_i / c_ijk * (p->F[ATHAD_U][c] * dcdr + p->F[ATHAD_V][c] * dcdthe + p->F[ATHAD_W][c] * dcdphi)
                         + MC_EPS_U * Mu_c;
                else
                    eu = 0.0;
                if (t_u <= MC_T00M2) eu = 0.0;
                double du = (i <= il) ? MC_EPS_U * Mu_c : 0.0;
                if (ip > 1 && i == il)
                    du = MC_DEL_U * Mu_c + MC_B_U * Mu_c / p->step[i];
                if (ip > 1 && i == il - 1)
                    du = MC_DEL_U * Mu_c + (1.0 - MC_B_U) * Mu_c / p->step[i];
                if (t_u <= MC_T00M2) du = 0.0;
                const double d_Mu = eu - du;
                const double Mu = clamp_M(Mu_m + d_Mu * p->step[i]);
                p->F[ATHAD_E_U][c] = eu;
                p->F[ATHAD_D_U][c] = du;
                p->F[ATHAD_M_U][c] = Mu;
                Mu_m = Mu;
                p->F[ATHAD_C_U][c] = 0.0;
                if (ip == 1) {
                    p->F[ATHAD_E_L][c] = 0.0;
                } else {
                    const double r_h_floor = smax(r_h_i, 0.01);
                    double el = du * qcu_c / r_h_floor;
                    if (el <= 0.0) el = 0.0;
                    p->F[ATHAD_E_L][c] = el;
                }
                const double K_p = (height_i > height_base + delta_i_c) ? MC_BET_P : 0.0;
                if (t_u >= t_0) p->F[ATHAD_G_P][c] = (ip == 1) ? 0.0 : K_p * qcu_c;
                else p->F[ATHAD_G_P][c] = 0.0;
            }
            p->F[ATHAD_M_U][IDX(il, j, k)] = 0.0;
        }
        if (interior) cloud_base_update(X, j, k, i_deep_beg, i_lfs, &i_base);

        /* updraftRecurrence, :1032-1163 (interior columns).  The updraft values of level i-1
           that level i reads (M_u, q_v_u, q_c_u, v_u, w_u, s_u as this loop left them; E_u,
           D_u, g_p as the entrainment left them or this loop zeroed them) are carried in
           registers from one level to the next instead of being stored and loaded again:
           the same values, so the same results. */
        if (interior && !(i_base < 0 || i_lfs <= i_base)) {
            const long long cb = IDX(i_base, j, k);
            double Mu_m = p->F[ATHAD_M_U][cb], qvu_m = p->F[ATHAD_Q_V_U][cb], qcu_m = p->F[ATHAD_Q_C_U][cb];
            double vu_m = p->F[ATHAD_V_U][cb], wu_m = p->F[ATHAD_W_U][cb], su_m = p->F[ATHAD_MC_S_U][cb];
            double eu_m = p->F[ATHAD_E_U][cb], du_m = p->F[ATHAD_D_U][cb], gp_m = p->F[ATHAD_G_P][cb];
            const double inv_a_u = 1.0 / (MC_A_U * p->u_0);
            const double cap = MC_W_CONV_MAX / p->u_0;
            for (int i = i_base + 1; i <= i_lfs - 1; i++) {
                const long long c = IDX(i, j, k), cm = IDX(i - 1, j, k);
                const double t_u = p->F[ATHAD_T][cm] * t_0;
                const double r_h_prev = p->F[ATHAD_R_HUMID][cm];
                const double step_prev = p->step[i - 1];
                const double r_h_i = p->F[ATHAD_R_HUMID][c];
                const double d_Mu = eu_m - du_m;
                double Mu = clamp_M(Mu_m + d_Mu * step_prev);
                if (t_u <= MC_T00M2) Mu = 0.0;
                const double M_u_prev = Mu_m;
                const double dq_v = M_u_prev * qvu_m
                    + step_prev * (eu_m * p->F[ATHAD_C][cm] - du_m * qvu_m);
                const double dq_c = M_u_prev * qcu_m
                    + step_prev * (-du_m * p->F[ATHAD_CLOUD][cm] - r_h_prev * gp_m);
                const double dv = M_u_prev * vu_m + step_prev * eu_m * p->F[ATHAD_V][cm];
                const double dw = M_u_prev * wu_m + step_prev * eu_m * p->F[ATHAD_W][cm];
                const double ds = (M_u_prev * su_m
                    + step_prev * (eu_m * p->F[ATHAD_MC_S][cm] - du_m * su_m)) / p->s_0;
                double qvu, qcu, vu, wu, su;
                if (fabs(Mu) > MC_COEFF_RECURR) {
                    const double inv = 1.0 / Mu;
                    qvu = dq_v * inv;
                    qcu = dq_c * inv;
                    vu = dv * inv;
                    wu = dw * inv;
                    su = ds * inv;
                } else {
                    su = p->F[ATHAD_MC_S][c];
                    qvu = p->F[ATHAD_C][c];
                    qcu = 0.0;
                    vu = p->F[ATHAD_V][c];
                    wu = p->F[ATHAD_W][c];
                }
                double cu = 0.0;
                if (fabs(Mu) > MC_COEFF_RECURR) {
                    double T_u = su * p->s_0 / p->cp_l;
                    const double p_u = p->F[ATHAD_P_STAT][c];
                    double dcond_tot = 0.0;
                    for (int it = 0; it < 2; ++it) {
                        const double E_s = saturation_pressure_auto(T_u);
                        const double q_sat_u = safe_q_sat(X, E_s, p_u, p->F[ATHAD_C][c]);
                        const double dq = qvu - q_sat_u;
                        if (dq <= 0.0) break;
                        const double L_u = (T_u >= t_0) ? p->lv : p->ls;
                        const double M_o_u = M_nonwater(p->F[ATHAD_C][c], p->F[ATHAD_CO2][c], p->M_bg);
                        const double dqsdT = dqsat_dT_from(E_s, latent_heat_auto(T_u), T_u, p_u, M_o_u);
                        const double G = (L_u / p->cp_l) * dqsdT;
                        const double dcond = dq / (1.0 + G);
                        qvu -= dcond;
                        qcu += dcond;
                        T_u += (L_u / p->cp_l) * dcond;
                        dcond_tot += dcond;
                    }
                    su = p->cp_l * T_u / p->s_0;
                    cu = dcond_tot * Mu / (smax(r_h_i, 0.01) * p->step[i]);
                }
                double uu = p->F[ATHAD_U][c] + Mu * inv_a_u / safe_r_humid(r_h_i);
                uu = smax(-cap, smin(uu, cap));
                if (qvu <= 0.0) qvu = 0.0;
                if (qcu <= 0.0) qcu = 0.0;
                if (qcu > MC_Q_C_U_MAX) qcu = MC_Q_C_U_MAX;
                if (su <= 0.0) su = 0.0;
                double eu = p->F[ATHAD_E_U][c], du = p->F[ATHAD_D_U][c], gp = p->F[ATHAD_G_P][c];
                if (t_u <= MC_T00) {
                    eu = 0.0; du = 0.0; Mu = 0.0;
                    qvu = 0.0; qcu = 0.0;
                    uu = 0.0; vu = 0.0; wu = 0.0;
                    su = 1.0;
                    gp = 0.0; cu = 0.0;
                    p->F[ATHAD_E_U][c] = 0.0; p->F[ATHAD_D_U][c] = 0.0; p->F[ATHAD_G_P][c] = 0.0;
                    p->F[ATHAD_E_L][c] = 0.0;
                }
                p->F[ATHAD_M_U][c] = Mu;
                p->F[ATHAD_Q_V_U][c] = qvu; p->F[ATHAD_Q_C_U][c] = qcu;
                p->F[ATHAD_V_U][c] = vu; p->F[ATHAD_W_U][c] = wu;
                p->F[ATHAD_MC_S_U][c] = su; p->F[ATHAD_C_U][c] = cu; p->F[ATHAD_U_U][c] = uu;
                Mu_m = Mu; qvu_m = qvu; qcu_m = qcu; vu_m = vu; wu_m = wu; su_m = su;
                eu_m = eu; du_m = du; gp_m = gp;
            }
        }

        /* downdraftEntrainment, :913-1027 (every column) */
        if (!(i_lfs <= 0 || i_lfs <= i_base)) {
            const int il = i_lfs, ib = i_base;
            const long long cl = IDX(il, j, k);
            double t_u = p->F[ATHAD_T][cl] * t_0;
            double p_u = p->F[ATHAD_P_STAT][cl];
            p->F[ATHAD_M_D][cl] = clamp_M(M_d_LFS);
            p->F[ATHAD_E_D][cl] = MC_EPS_D * fabs(p->F[ATHAD_M_D][cl]);
            p->F[ATHAD_D_D][cl] = MC_DEL_D * fabs(p->F[ATHAD_M_D][cl]);
            {
                const double q_sat = safe_q_sat(X, saturation_pressure_auto(t_u), p_u, p->F[ATHAD_C][cl]);
                p->F[ATHAD_Q_V_D][cl] = 0.5 * (p->F[ATHAD_CLOUD][cl] + MC_SCALE * q_sat);
            }
            const double r_humid_lfs = 1e2 * p_u / (R_of(p->F[ATHAD_C][cl], p->F[ATHAD_CO2][cl], p->R_bg) * t_u);
            const double inv_a_d0 = 1.0 / (MC_A_D * p->u_0);
            p->F[ATHAD_U_D][cl] = p->F[ATHAD_U][cl] + p->F[ATHAD_M_D][cl] * inv_a_d0 / safe_r_humid(r_humid_lfs);
            p->F[ATHAD_V_D][cl] = p->F[ATHAD_V][cl];
            p->F[ATHAD_W_D][cl] = p->F[ATHAD_W][cl];
            p->F[ATHAD_MC_S_D][cl] = p->F[ATHAD_MC_S][cl];
            p->F[ATHAD_P_CONV][cl] = 0.0;
            double sigma_p = 0.0;
            {
                const double w_u_cb = fabs(p->F[ATHAD_W_U][IDX(ib, j, k)]) * p->u_0;
                if (w_u_cb > 0.0)
                    sigma_p = fabs(p->F[ATHAD_M_U][IDX(ib, j, k)]) / (safe_r_humid(p->F[ATHAD_R_HUMID][IDX(ib, j, k)]) * w_u_cb);
                sigma_p = smin(sigma_p, 1.0);
            }
            // Every value a level reads is loaded before it stores anything (it stores only
            // its own cells and reads nothing it stores); M_d of the level above is carried
            // in a register.  The differences that the serial order forms from stored and
            // reloaded products are formed without contraction into a fused multiply-add.
            double Md_up = p->F[ATHAD_M_D][cl];
            for (int i = il - 1; i >= 0; i--) {
                const long long c = IDX(i, j, k);
                p_u = p->F[ATHAD_P_STAT][c];
                t_u = p->F[ATHAD_T][c] * t_0;
                const double r_h_i = p->F[ATHAD_R_HUMID][c];
                const double Cc = p->F[ATHAD_C][c], CLc = p->F[ATHAD_CLOUD][c];
                const double Md_old = p->F[ATHAD_M_D][c];
                const double Uc = p->F[ATHAD_U][c], Vc = p->F[ATHAD_V][c], Wc = p->F[ATHAD_W][c];
                const double precip_i = p->F[ATHAD_P_CONV][c];
                const double ep_old = p->F[ATHAD_E_P][c];
                p->F[ATHAD_MC_S_D][c] = p->cp_l * t_u / p->s_0;
                const double q_sat = safe_q_sat(X, saturation_pressure_auto(t_u), p_u, Cc);
                const double qvd = 0.5 * (CLc + MC_SCALE * q_sat);
                p->F[ATHAD_Q_V_D][c] = qvd;
                const double ed = MC_EPS_D * fabs(Md_old);
                const double dd = MC_DEL_D * fabs(Md_old);
                p->F[ATHAD_E_D][c] = ed;
                p->F[ATHAD_D_D][c] = dd;
                const double d_Md = sub_rn(ed, dd);
                const double Md = clamp_M(Md_up - d_Md * p->step[i]);
                p->F[ATHAD_M_D][c] = Md;
                Md_up = Md;
                const double inv_a_d = 1.0 / (MC_A_D * p->u_0);
                p->F[ATHAD_U_D][c] = Uc + Md * inv_a_d / safe_r_humid(r_h_i);
                p->F[ATHAD_V_D][c] = Vc;
                p->F[ATHAD_W_D][c] = Wc;
                if (i <= ib) {
                    if (ip == 1) {
                        p->F[ATHAD_E_P][c] = 0.0;
                    } else {
                        double ep = ep_old;
                        if (precip_i > 0.0 && sigma_p > 0.0)
                            ep = sigma_p * MC_ALF_1 * sub_rn(q_sat, qvd)
                                 * sqrt(1e1 / MC_ALF_2 * precip_i / sigma_p);
                        if (ep <= 0.0) ep = 0.0;
                        p->F[ATHAD_E_P][c] = ep;
                    }
                }
                if (ip == 1) {
                    p->F[ATHAD_E_DD][c] = 0.0;
                } else {
                    double edd;
                    if (precip_i > 0.0) {
                        const double P_16 = pow(precip_i, 1.0 / 6.0);
                        const double P_49 = pow(precip_i, 4.0 / 9.0);
                        edd = MC_A_EV * (1.0 + MC_B_EV * P_16) * sub_rn(q_sat, qvd) * P_49;
                    } else {
                        edd = 0.0;
                    }
                    if (edd <= 0.0) edd = 0.0;
                    p->F[ATHAD_E_DD][c] = edd;
                }
            }
        }

        /* downdraftRecurrence, :1168-1254 (every column).  The downdraft values of level
           i+1 that level i reads are carried in registers, as in the updraft recurrence. */
        {
            const long long c0 = IDX(i_lfs, j, k);
            double Md_p = p->F[ATHAD_M_D][c0], qvd_p = p->F[ATHAD_Q_V_D][c0];
            double vd_p = p->F[ATHAD_V_D][c0], wd_p = p->F[ATHAD_W_D][c0], sd_p = p->F[ATHAD_MC_S_D][c0];
            double ed_p = p->F[ATHAD_E_D][c0], dd_p = p->F[ATHAD_D_D][c0], edd_p = p->F[ATHAD_E_DD][c0];
            double pconv_p = p->F[ATHAD_P_CONV][c0], rh_p = p->F[ATHAD_R_HUMID][c0];
            const double inv_a_d = 1.0 / (MC_A_D * p->u_0);
            for (int i = i_lfs - 1; i >= 0; i--) {
                const long long c = IDX(i, j, k), cp = IDX(i + 1, j, k);
                const double t_u = p->F[ATHAD_T][c] * t_0;
                const double gp_c = p->F[ATHAD_G_P][c];   // not written by this loop
                const double step_ip1 = p->step[i + 1];
                const double r_h_ip1 = rh_p, r_h_i = p->F[ATHAD_R_HUMID][c];
                double ed = p->F[ATHAD_E_D][c], dd = p->F[ATHAD_D_D][c];
                const double d_Md = ed - dd;
                double Md = clamp_M(Md_p - d_Md * step_ip1);
                if (t_u <= MC_T00M2) Md = 0.0;
                const double L_latent = (t_u >= t_0) ? p->lv : p->ls;
                const double M_d_ip1 = Md_p;
                const double dq_v = M_d_ip1 * qvd_p
                    - step_ip1 * (ed_p * p->F[ATHAD_C][cp] - dd_p * qvd_p + r_h_ip1 * edd_p);
                const double dv = M_d_ip1 * vd_p - step_ip1 * (ed_p * p->F[ATHAD_V][cp] - dd_p * vd_p);
                const double dw = M_d_ip1 * wd_p - step_ip1 * (ed_p * p->F[ATHAD_W][cp] - dd_p * wd_p);
                const double ds = (M_d_ip1 * sd_p
                    - step_ip1 * (ed_p * p->F[ATHAD_MC_S][cp] - dd_p * sd_p - L_latent * r_h_ip1 * edd_p)) / p->s_0;
                double qvd, vd, wd, sd;
                if (fabs(Md) > MC_COEFF_RECURR) {
                    const double inv = 1.0 / Md;
                    qvd = dq_v * inv;
                    vd = dv * inv;
                    wd = dw * inv;
                    sd = ds * inv;
                } else {
                    qvd = p->F[ATHAD_C][c];
                    vd = p->F[ATHAD_V][c];
                    wd = p->F[ATHAD_W][c];
                    sd = p->F[ATHAD_MC_S][c];
                }
                double ud = p->F[ATHAD_U][c] + Md * inv_a_d / safe_r_humid(r_h_i);
                if (qvd <= 0.0) qvd = 0.0;
                if (sd <= 0.0) sd = 0.0;
                double edd = p->F[ATHAD_E_DD][c], ep = p->F[ATHAD_E_P][c];
                if (t_u <= MC_T00) {
                    ed = 0.0; dd = 0.0; Md = 0.0;
                    qvd = 0.0;
                    ud = 0.0; vd = 0.0; wd = 0.0;
                    sd = 1.0; edd = 0.0; ep = 0.0;
                    p->F[ATHAD_E_D][c] = 0.0; p->F[ATHAD_D_D][c] = 0.0;
                    p->F[ATHAD_E_DD][c] = 0.0; p->F[ATHAD_E_P][c] = 0.0;
                }
                p->F[ATHAD_M_D][c] = Md; p->F[ATHAD_Q_V_D][c] = qvd;
                p->F[ATHAD_U_D][c] = ud; p->F[ATHAD_V_D][c] = vd; p->F[ATHAD_W_D][c] = wd;
                p->F[ATHAD_MC_S_D][c] = sd;
                double pconv = 0.0;
                if (i > 0) {
                    pconv = smax(0.0, pconv_p + p->step[i] * r_h_i * (gp_c - edd - ep));
                    p->F[ATHAD_P_CONV][c] = pconv;
                }
                Md_p = Md; qvd_p = qvd; vd_p = vd; wd_p = wd; sd_p = sd;
                ed_p = ed; dd_p = dd; edd_p = edd; pconv_p = pconv; rh_p = r_h_i;
            }
        }
        p->F[ATHAD_P_CONV][IDX(0, j, k)] = p->F[ATHAD_P_CONV][IDX(1, j, k)];
    }

    /* rhsForcing, :1304-1417.  The clamp of M_u and M_d to [-3, 3] (NaN to 0) is applied
       where the flux of a level first reads them, each level once and before any use, as
       the reference's separate pass leaves them. */
    auto clamp3 = [](double v) { return !is_finite_bits(v) ? 0.0 : (v < -3.0) ? -3.0 : (v > 3.0) ? 3.0 : v; };
    // the four mass fluxes at a level; level i+1's are level i's upper fluxes and the next
    // level's lower ones, so each is formed once and carried (same operands, same values)
    auto flux_at = [&](long long c, double& fs, double& fq, double& fv, double& fw) {
        const double Mu = clamp3(p->F[ATHAD_M_U][c]), Md = clamp3(p->F[ATHAD_M_D][c]);
        const double su = p->F[ATHAD_MC_S_U][c], sm = p->F[ATHAD_MC_S][c], sd = p->F[ATHAD_MC_S_D][c];
        const double qu = p->F[ATHAD_Q_V_U][c], qm = p->F[ATHAD_C][c], qd = p->F[ATHAD_Q_V_D][c];
        const double vu = p->F[ATHAD_V_U][c], vm = p->F[ATHAD_V][c], vd = p->F[ATHAD_V_D][c];
        const double wu = p->F[ATHAD_W_U][c], wm = p->F[ATHAD_W][c], wd = p->F[ATHAD_W_D][c];
        p->F[ATHAD_M_U][c] = Mu;
        p->F[ATHAD_M_D][c] = Md;
        fs = Mu * (su - sm) + Md * (sd - sm);
        fq = Mu * (qu - qm) + Md * (qd - qm);
        fv = Mu * (vu - vm) + Md * (vd - vm);
        fw = Mu * (wu - wm) + Md * (wd - wm);
    };
    double fs0, fq0, fv0, fw0;
    flux_at(IDX(0, j, k), fs0, fq0, fv0, fw0);
    for (int i = 0; i < im - 1; i++) {
        const long long c = IDX(i, j, k), cp = IDX(i + 1, j, k);
        const double Tc = p->F[ATHAD_T][c], Rc = p->F[ATHAD_R_HUMID][c];
        const double cu = p->F[ATHAD_C_U][c], edd = p->F[ATHAD_E_DD][c];
        const double el = p->F[ATHAD_E_L][c], ep = p->F[ATHAD_E_P][c];
        const double L_latent = (Tc * t_0 >= t_0) ? p->lv : p->ls;
        const double inv_step_rh = 1.0 / (p->step[i] * smax(Rc, 0.01));
        double fs1, fq1, fv1, fw1;
        flux_at(cp, fs1, fq1, fv1, fw1);
        const double conv_src = cu - edd - el - ep;
        double v = -(fs1 - fs0) * inv_step_rh * t_0 + (L_latent / p->cp_l) * conv_src * t_0;
        p->F[ATHAD_MC_T][c] = !is_finite_bits(v) ? 0.0 : (v < -0.01) ? -0.01 : (v > 0.01) ? 0.01 : v;
        v = -(fq1 - fq0) * inv_step_rh - conv_src;
        p->F[ATHAD_MC_Q][c] = !is_finite_bits(v) ? 0.0 : (v < -2.0e-5) ? -2.0e-5 : (v > 2.0e-5) ? 2.0e-5 : v;
        v = -(fv1 - fv0) * inv_step_rh * p->u_0;
        p->F[ATHAD_MC_V][c] = !is_finite_bits(v) ? 0.0 : (v < -0.01) ? -0.01 : (v > 0.01) ? 0.01 : v;
        v = -(fw1 - fw0) * inv_step_rh * p->u_0;
        p->F[ATHAD_MC_W][c] = !is_finite_bits(v) ? 0.0 : (v < -0.01) ? -0.01 : (v > 0.01) ? 0.01 : v;
        fs0 = fs1; fq0 = fq1; fv0 = fv1; fw0 = fw1;
    }
}


#ifndef ATHAD_MC_BLOCK
#define ATHAD_MC_BLOCK 128   // columns per CTA
#endif

__global__ void __launch_bounds__(ATHAD_MC_BLOCK) moist_convection_kernel(const MoistArgs X)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= X.d.km || j >= X.d.jm) return;
    mc_column(X, j, k);
}

void launch_moist_convection(const MoistArgs& a, cudaStream_t st)
{
    moist_convection_kernel<<<dim3((a.d.km + ATHAD_MC_BLOCK - 1) / ATHAD_MC_BLOCK, a.d.jm), ATHAD_MC_BLOCK, 0, st>>>(a);
}

}  // namespace athad
