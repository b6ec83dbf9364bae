/*
 * or_dynamics.c - oracle restatement of the RK4 time step, its finite-difference
 * right-hand side and the pressure-Poisson relaxation (TEST INFRASTRUCTURE ONLY, see
 * athad_oracle.h).
 *
 * Terrain is flat (the configured case), so every land branch of the reference is dead:
 * in the interior all derivatives are the central ones (RHS_Atm_Turb.cpp:119-151,
 * 222-255, 326-359), the Poisson source is central (PressureSolverAtm.h:415-420) and the
 * k-omega-SST wall-distance scan reduces to min(i, j, k) (RHS_Atm_Turb.cpp:640-671).
 */
#include "or_internal.h"
#include <stdio.h>

size_t or_params_size(void) { return sizeof(or_params); }
int or_nfields(void) { return OF_NFIELDS; }

void or_geom_init(or_geom* g, int im, int jm, int km, const or_params* p, int compat)
{
    g->im = im; g->jm = jm; g->km = km;
    const double pi180 = 180.0 / M_PI;                       /* cAtmosphereModel.cpp:44 */
    g->dr = 1.0 / (double)(im - 1);                          /* cAtmosphereModel.cpp:57 */
    g->dthe = (180.0 / (double)(jm - 1)) / pi180;            /* :46, :59 generalised */
    g->dphi = (360.0 / (double)(km - 1)) / pi180;            /* :47, :60 generalised */
    g->rad = (double*)malloc(sizeof(double) * im);
    g->the = (double*)malloc(sizeof(double) * jm);
    g->phi = (double*)malloc(sizeof(double) * km);
    g->sin_f = (double*)malloc(sizeof(double) * jm);
    g->cos_t = (double*)malloc(sizeof(double) * jm);
    g->sin_w = (double*)malloc(sizeof(double) * jm);
    g->height = (double*)malloc(sizeof(double) * im);
    g->rad[0] = 1.0;
    for (int i = 1; i < im; i++) g->rad[i] = g->rad[i - 1] + g->dr;
    g->the[0] = 0.0;
    for (int j = 1; j < jm; j++) g->the[j] = g->the[j - 1] + g->dthe;
    g->phi[0] = 0.0;
    for (int k = 1; k < km; k++) g->phi[k] = g->phi[k - 1] + g->dphi;
    for (int j = 0; j < jm; j++) {
        if (compat) {
            g->sin_w[j] = sin(g->the[j]);
            g->cos_t[j] = cos(g->the[j]);
        } else {
            /* mirror-symmetric tables: sin(theta_j) == sin(theta_{jm-1-j}) and
             * cos(theta_j) == -cos(theta_{jm-1-j}) exactly, cos == 0 on the equator row */
            const int jj = (j < jm - 1 - j) ? j : jm - 1 - j;
            g->sin_w[j] = sin(g->the[jj]);
            if (j < jm - 1 - j) g->cos_t[j] = cos(g->the[j]);
            else if (j > jm - 1 - j) g->cos_t[j] = -cos(g->the[jm - 1 - j]);
            else g->cos_t[j] = 0.0;
        }
        g->sin_f[j] = g->sin_w[j];
        if (g->sin_f[j] < 0.55) g->sin_f[j] = 0.55;
    }
    const double span = g->rad[im - 1] - g->rad[0];
    g->shell_len = (span > 0.0) ? (exp(p->zeta * span) - 1.0) * p->L_atm / span : p->L_atm;
    const float hL = (float)p->L_atm;
    for (int i = 0; i < im; i++) {
        const float hf = (float)((exp(p->zeta * (g->rad[i] - g->rad[0])) - 1) * (double)hL);
        g->height[i] = (double)hf;
    }
}

void or_geom_free(or_geom* g)
{
    free(g->rad); free(g->the); free(g->phi); free(g->sin_f); free(g->cos_t);
    free(g->sin_w); free(g->height);
}

/* metricRadius, cAtmosphereModel.h:282-284, with m_metric_r0 from initMetricRadius
 * (cAtmosphereModel.cpp:382-399): metric_r0 < 0 selects the reference default
 * r_Earth * 1e3 / metricShellLength(). */
static double metric_r0_of(const or_geom* g, const or_params* p)
{
    if (p->metric_r0 < 0.0)
        return (g->shell_len > 0.0) ? (p->r_Earth * 1.0e3 / g->shell_len) : 0.0;
    return p->metric_r0;
}
double or_metric_radius(const or_geom* g, const or_params* p, double rm)
{
    const double r0 = metric_r0_of(g, p);
    return (r0 > 0.0) ? (r0 + (rm - g->rad[0])) : rm;
}

/* ---------------------------------------------------------------------------------- */
/* computeLevelMeanTemperature, RungeKutta_Atm_Turb.cpp:24-41.
 * compat: the reference's accumulation order.  Otherwise: per row a 32-way strided
 * partial sum combined by the xor-butterfly order a warp reduction uses, then the rows
 * paired j with jm-1-j, so that the mean of a mirrored field is bit-identical. */
static double row_sum_32(const double* row, int km)
{
    double part[32];
    for (int l = 0; l < 32; l++) {
        double s = 0.0;
        for (int k = l; k < km; k += 32) s += row[k];
        part[l] = s;
    }
    for (int off = 16; off >= 1; off >>= 1) {
        double nxt[32];
        for (int l = 0; l < 32; l++) nxt[l] = part[l] + part[l ^ off];
        memcpy(part, nxt, sizeof part);
    }
    return part[0];
}

static void level_mean_impl(const or_geom* g, const double* t, double* out, int compat)
{
    const int im = g->im, jm = g->jm, km = g->km;
    for (int i = 0; i < im; i++) {
        if (compat) {
            double sum = 0.0, wsum = 0.0;
            for (int j = 0; j < jm; j++) {
                const double w = g->sin_w[j];
                for (int k = 0; k < km; k++) {
                    sum += w * t[OR_IDX(i, j, k)];
                    wsum += w;
                }
            }
            out[i] = (wsum > 0.0) ? sum / wsum : 1.0;
        } else {
            double sum = 0.0, wsum = 0.0;
            const int half = jm / 2;
            for (int j = 0; j < half; j++) {
                const double sj = row_sum_32(&t[OR_IDX(i, j, 0)], km);
                const double sm = row_sum_32(&t[OR_IDX(i, jm - 1 - j, 0)], km);
                sum += g->sin_w[j] * (sj + sm);
                wsum += 2.0 * g->sin_w[j] * (double)km;
            }
            if (jm & 1) {
                sum += g->sin_w[half] * row_sum_32(&t[OR_IDX(i, half, 0)], km);
                wsum += g->sin_w[half] * (double)km;
            }
            out[i] = (wsum > 0.0) ? sum / wsum : 1.0;
        }
    }
}

void or_level_mean(int im, int jm, int km, const or_params* p, int compat,
                   double* const* f, double* const* prof)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    level_mean_impl(&g, f[OF_T], prof[OFP_T_REF_LEVEL], compat);
    or_geom_free(&g);
}

/* ---------------------------------------------------------------------------------- */
/* CellGeometry, cAtmosphereModel.h:170-178, built as RungeKutta_Atm_Turb.cpp:104-135 */
typedef struct cgeo {
    double exp_rm, exp_2_rm, sinthe, sinthe2, costhe;
    double inv_rm, inv_rm2, inv_rmsinthe, inv_rm2sinthe, inv_rm2sinthe2, costhe_inv_rm2sinthe;
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
} cgeo;

static void make_cgeo(const or_geom* g, const or_params* p, int i, int j, cgeo* c)
{
    const double rm = g->rad[i];
    c->exp_rm = 1.0 / (rm + 1.0);
    c->exp_2_rm = c->exp_rm * c->exp_rm;
    c->sinthe = g->sin_f[j];
    c->sinthe2 = c->sinthe * c->sinthe;
    c->costhe = g->cos_t[j];
    const double rmet = or_metric_radius(g, p, rm);
    const double rmet2 = rmet * rmet;
    c->inv_rm = 1.0 / rmet;
    c->inv_rm2 = 1.0 / rmet2;
    c->inv_rmsinthe = 1.0 / (rmet * c->sinthe);
    c->inv_rm2sinthe = c->inv_rm2 / c->sinthe;
    c->inv_rm2sinthe2 = c->inv_rm2 / c->sinthe2;
    c->costhe_inv_rm2sinthe = c->costhe * c->inv_rm2sinthe;
    c->inv_2dr = 1.0 / (2.0 * g->dr);
    c->inv_2dthe = 1.0 / (2.0 * g->dthe);
    c->inv_2dphi = 1.0 / (2.0 * g->dphi);
    c->inv_dr2 = 1.0 / (g->dr * g->dr);
    c->inv_dthe2 = 1.0 / (g->dthe * g->dthe);
    c->inv_dphi2 = 1.0 / (g->dphi * g->dphi);
}

/* minmod, RHS_Atm_Turb.cpp:26-28 */
static inline double minmod(double a, double b)
{
    return (a * b <= 0.0) ? 0.0 : (fabs(a) < fabs(b) ? a : b);
}

enum { Y_T = 0, Y_U, Y_V, Y_W, Y_C, Y_CL, Y_IC, Y_GR, Y_CO, Y_TK, Y_DI, NY };

typedef struct rhs_out {
    double k[NY];
    double aux[3];
    double prod, tke_source, dis_source;
    /* the right-hand side's diagnostic outputs (RHS_Atm_Turb.cpp:448-491, 1031-1057):
     * CoriolisForce, BuoyancyForce, PressureGradientForce, Q_Latent, Q_Sensible and the six
     * terms each of rhs_v and rhs_w (pgf, cor, advv, advh, diff, other) */
    double force[3], q_latent, q_sensible, vbud[6], wbud[6];
} rhs_out;

/* RHS_Atmosphere_Turb for one interior cell, RHS_Atm_Turb.cpp:31-1080, flat terrain.
 * Y[0..10] are the stage fields (t,u,v,w,c,cloud,ice,gr,co2,tke,dis). */
static void rhs_cell(const or_geom* g, const or_params* p, const or_step* s, int compat,
                     int i, int j, int k, const cgeo* G, const double* const* Y,
                     const double* pd, const double* nu, double* const* f,
                     const double* t_ref, const double* dlnrho, rhs_out* o)
{
    const int jm = g->jm, km = g->km;
    const size_t c = OR_IDX(i, j, k);
    const size_t sI = (size_t)jm * km, sJ = (size_t)km;
    double d1r[NY], d2r[NY], d1t[NY], d2t[NY], d1p[NY], d2p[NY];
    for (int n = 0; n < NY; n++) {
        const double* F = Y[n];
        /* radial and zonal: reference expression order (RHS_Atm_Turb.cpp:121-123, 327-329) */
        d1r[n] = (F[c + sI] - F[c - sI]) * G->inv_2dr;
        d2r[n] = (F[c + sI] - 2.0 * F[c] + F[c - sI]) * G->inv_dr2;
        d1p[n] = (F[c + 1] - F[c - 1]) * G->inv_2dphi;
        d2p[n] = (F[c + 1] - 2.0 * F[c] + F[c - 1]) * G->inv_dphi2;
        /* meridional (RHS_Atm_Turb.cpp:223-225); the mirror-symmetric form sums the two
         * neighbours first so that j and jm-1-j round identically */
        d1t[n] = (F[c + sJ] - F[c - sJ]) * G->inv_2dthe;
        if (compat) d2t[n] = (F[c + sJ] - 2.0 * F[c] + F[c - sJ]) * G->inv_dthe2;
        else        d2t[n] = ((F[c + sJ] + F[c - sJ]) - 2.0 * F[c]) * G->inv_dthe2;
    }
    const double dpdr = (pd[c + sI] - pd[c - sI]) * G->inv_2dr;
    const double dpdthe = (pd[c + sJ] - pd[c - sJ]) * G->inv_2dthe;
    const double dpdphi = (pd[c + 1] - pd[c - 1]) * G->inv_2dphi;
    (void)nu;

    const double exp_rm = G->exp_rm, exp_2_rm = G->exp_2_rm;
    const double sinthe = G->sinthe, sinthe2 = G->sinthe2, costhe = G->costhe;
    const double inv_rm = G->inv_rm, inv_rm2 = G->inv_rm2, inv_rmsinthe = G->inv_rmsinthe;
    const double inv_rm2sinthe = G->inv_rm2sinthe, inv_rm2sinthe2 = G->inv_rm2sinthe2;

    const double u_ijk = Y[Y_U][c], v_ijk = Y[Y_V][c], w_ijk = Y[Y_W][c];
    const double t_ijk = Y[Y_T][c], tke_ijk = Y[Y_TK][c], dis_ijk = Y[Y_DI][c];
    const double nue_ijk = nu[c];

    /* coefficients, RHS_Atm_Turb.cpp:363-372 */
    const double coeff_energy_p = p->u_0 * p->u_0 / (p->cp_l * p->t_0);
    const double coeff_energy = 1.0 / (p->c_0 * p->cp_l * p->t_0);
    const double coeff_trans = 1.0;
    const double coeff_MC_vel = p->L_atm / (p->u_0 * p->u_0);
    const double coeff_MC_q = p->L_atm / (p->u_0 * p->c_0);
    const double coeff_MC_t = p->L_atm / (p->u_0 * p->t_0);
    const double coriolis = 1.0;
    /* Coriolis, RHS_Atm_Turb.cpp:392-395 */
    const double nontrad = p->coriolis_nontrad ? 1.0 : 0.0;
    const double coriolis_rad = nontrad * 2.0 * sinthe * w_ijk;
    const double coriolis_the = 2.0 * costhe * w_ijk;
    const double coriolis_phi = -2.0 * (costhe * v_ijk + nontrad * sinthe * u_ijk);
    const double force_nd = p->omega * g->shell_len / p->u_0;   /* :445 */

    /* turbulence, RHS_Atm_Turb.cpp:504-721 */
    double diffusion_t_re = 0.0, diffusion_vel_re = 0.0, diffusion_tke_re = 0.0,
           diffusion_dis_re = 0.0;
    const double diff_prec_re_inv = 1.0 / (p->sc_WaterVapour * p->re_turb);
    const double diff_co2_re_inv = 1.0 / (p->sc_CO2 * p->re_turb);
    const double d_i = (double)i, d_i_mount = 0.0;
    double prod = 0.0, tke_source = 0.0, dis_source = 0.0;
    const int keps = (p->turb_model == 1), kom = (p->turb_model == 2), sst = (p->turb_model == 3);
    {   /* :528-561 */
        const double C_nue_loc = 0.028, dis_min_loc = 1.0e-10;
        const double dudr_s = d1r[Y_U] * exp_rm, dvdr_s = d1r[Y_V] * exp_rm, dwdr_s = d1r[Y_W] * exp_rm;
        const double dudthe_s = d1t[Y_U] * inv_rm, dvdthe_s = d1t[Y_V] * inv_rm, dwdthe_s = d1t[Y_W] * inv_rm;
        const double dudphi_s = d1p[Y_U] * inv_rmsinthe, dvdphi_s = d1p[Y_V] * inv_rmsinthe,
                     dwdphi_s = d1p[Y_W] * inv_rmsinthe;
        const double dis_here = or_max(dis_ijk, dis_min_loc);
        const double tke_here = or_max(tke_ijk, 0.0);
        const double nue_max = 1000.0 / (p->u_0 * p->L_atm);
        double cnue = keps ? C_nue_loc * tke_here * tke_here / dis_here : tke_here / dis_here;
        cnue = or_min(cnue, nue_max);
        const double der = 0.66667 * (dudr_s + dvdthe_s + dwdphi_s);
        prod = or_max(0.0,
              (cnue * (2.0 * dudr_s - der) - 0.66667 * tke_ijk) * dudr_s
            + (cnue * (dudthe_s + dvdr_s)) * dudthe_s
            + (cnue * (dudphi_s + dwdr_s)) * dudphi_s
            + (cnue * (2.0 * dvdthe_s - der) - 0.66667 * tke_ijk) * dvdthe_s
            + (cnue * (dvdr_s + dudthe_s)) * dvdr_s
            + (cnue * (dvdphi_s + dwdthe_s)) * dvdphi_s
            + (cnue * (2.0 * dwdphi_s - der) - 0.66667 * tke_ijk) * dwdphi_s
            + (cnue * (dwdr_s + dudphi_s)) * dwdr_s
            + (cnue * (dwdthe_s + dvdphi_s)) * dwdthe_s);
    }
    const double dtkedr = d1r[Y_TK], dtkedthe = d1t[Y_TK], dtkedphi = d1p[Y_TK];
    const double ddisdr = d1r[Y_DI], ddisdthe = d1t[Y_DI], ddisdphi = d1p[Y_DI];
    if (keps) {   /* :563-599 */
        const double sig_k = 1.0, sig_w = 1.3, C_eps_1 = 1.35, C_eps_2 = 1.80;
        diffusion_t_re = (1.0 / p->re_turb + nue_ijk) / p->pr_turb;
        diffusion_vel_re = 1.0 / p->re_turb + nue_ijk;
        diffusion_tke_re = 1.0 / p->re_turb + nue_ijk / sig_k;
        diffusion_dis_re = 1.0 / p->re_turb + nue_ijk / sig_w;
        const double tke_s = or_max(tke_ijk, 1.0e-10), dis_s = or_max(dis_ijk, 1.0e-10);
        const double P_k = prod, Y_k = dis_s;
        const double P_w = C_eps_1 * (dis_s / tke_s) * P_k;
        const double Y_w = C_eps_2 * dis_s * dis_s / tke_s;
        const double dis_src_max = 20.0 * dis_s * dis_s, tke_src_max = 20.0 * tke_s * dis_s;
        tke_source = or_clamp(P_k - Y_k, -tke_src_max, tke_src_max);
        dis_source = or_clamp(P_w - Y_w, -dis_src_max, dis_src_max);
    }
    if (kom) {    /* :601-631 */
        const double sig_k = 0.6, sig_w = 0.5, bet_star = 0.09, gam = 0.52, bet_0 = 0.0708;
        diffusion_t_re = (1.0 / p->re_turb + nue_ijk) / p->pr_turb;
        diffusion_vel_re = 1.0 / p->re_turb + nue_ijk;
        diffusion_tke_re = 1.0 / p->re_turb + sig_k * nue_ijk;
        diffusion_dis_re = 1.0 / p->re_turb + sig_w * nue_ijk;
        const double tke_s = or_max(tke_ijk, 1.0e-10), dis_s = or_max(dis_ijk, 1.0e-10);
        const double P_k = or_min(prod, 20.0 * bet_star * tke_s * dis_s);
        const double Y_k = bet_star * tke_s * dis_s;
        const double P_w = gam * (dis_s / tke_s) * P_k;
        const double Y_w = bet_0 * dis_s * dis_s;
        const double cross = dtkedr * ddisdr + dtkedthe * inv_rm * ddisdthe * inv_rm
                           + dtkedphi * inv_rmsinthe * ddisdphi * inv_rmsinthe;
        const double sig_d = (cross <= 0.0) ? 0.0 : 0.125;
        const double D_w = sig_d * cross / dis_s;
        const double dis_src_max = 20.0 * dis_s * dis_s, tke_src_max = 20.0 * tke_s * dis_s;
        tke_source = or_clamp(P_k - Y_k, -tke_src_max, tke_src_max);
        dis_source = or_clamp(P_w - Y_w + D_w, -dis_src_max, dis_src_max);
    }
    if (sst) {    /* :633-721 */
        const double bet_star = 0.09, sig_k1 = 1.176, sig_k2 = 1.0, sig_w1 = 2.0, sig_w2 = 1.168;
        double d_j = (double)j;
        if (p->wall_mode == 0) { const int jr = jm - 1 - j; if (jr < j) d_j = (double)jr; }
        const double d_k = (double)k;
        double d_close = d_i - d_i_mount;
        if (d_j <= d_close) d_close = d_j;   /* south and north scans (:648-655) */
        if (d_j <= d_close) d_close = d_j;
        if (d_k <= d_close) d_close = d_k;   /* east and west scans (:657-665) */
        if (d_k <= d_close) d_close = d_k;
        const double CD_kw = or_max(
            (2.0 * sig_w2) / dis_ijk
            * (dtkedr * ddisdr + dtkedthe * inv_rm * ddisdthe * inv_rm
               + dtkedphi * inv_rmsinthe * ddisdphi * inv_rmsinthe),
            1.0e-20);
        const double nue_air_nd = 1.5e-5 / (p->u_0 * p->L_atm);
        const double arg1 = or_min(or_max(
            sqrt(tke_ijk) / (bet_star * dis_ijk * d_close),
            (500.0 * nue_air_nd) / (d_close * d_close * dis_ijk)),
            (4.0 * sig_w2 * tke_ijk) / (CD_kw * d_close * d_close));
        const double F1 = tanh(pow(arg1, 4));
        const double bk = F1 * sig_k1 + (1.0 - F1) * sig_k2;
        const double bw = F1 * sig_w1 + (1.0 - F1) * sig_w2;
        diffusion_t_re = (1.0 / p->re_turb + nue_ijk) / p->pr_turb;
        diffusion_vel_re = 1.0 / p->re_turb + nue_ijk;
        diffusion_tke_re = 1.0 / p->re_turb + nue_ijk / bk;
        diffusion_dis_re = 1.0 / p->re_turb + nue_ijk / bw;
        const double bet1 = 0.0333, bet2 = 0.0368, gam1 = 0.413, gam2 = 0.2;
        const double tke_s = or_max(tke_ijk, 1.0e-10), dis_s = or_max(dis_ijk, 1.0e-10);
        const double P_k = or_min(prod, 20.0 * bet_star * tke_s * dis_s);
        const double Y_k = bet_star * tke_s * dis_s;
        const double P_w = (F1 * gam1 + (1.0 - F1) * gam2) * P_k * dis_s / tke_s;
        const double Y_w = (F1 * bet1 + (1.0 - F1) * bet2) * dis_s * dis_s;
        const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_s
                         * (dtkedr * ddisdr + dtkedthe * inv_rm * ddisdthe * inv_rm
                            + dtkedphi * inv_rmsinthe * ddisdphi * inv_rmsinthe);
        const double dis_src_max = 20.0 * dis_s * dis_s, tke_src_max = 20.0 * tke_s * dis_s;
        tke_source = or_clamp(P_k - Y_k, -tke_src_max, tke_src_max);
        dis_source = or_clamp(P_w - Y_w + D_w, -dis_src_max, dis_src_max);
    }
    diffusion_t_re *= s->diffusion_ramp;     /* :742-745 */
    diffusion_vel_re *= s->diffusion_ramp;
    diffusion_tke_re *= s->diffusion_ramp;
    diffusion_dis_re *= s->diffusion_ramp;

    /* transport, RHS_Atm_Turb.cpp:748-836 */
    const double u_exp = u_ijk * exp_rm, v_invrm = v_ijk * inv_rm, w_invrs = w_ijk * inv_rmsinthe;
    const double pressure_t = coeff_energy_p * (u_exp * dpdr + v_invrm * dpdthe + w_invrs * dpdphi);
    const double inv_dr = 2.0 * G->inv_2dr, inv_dthe = 2.0 * G->inv_2dthe, inv_dphi = 2.0 * G->inv_2dphi;
    double tr[NY], adv_r[NY], adv_t[NY], adv_p[NY];
    for (int n = 0; n < NY; n++) {
        const double* F = Y[n];
        double ar = d1r[n], at = d1t[n], ap = d1p[n];
        if (n <= Y_IC) {  /* minmod-limited for t,u,v,w,c,cloud,ice (:788-814) */
            ar = minmod(F[c] - F[c - sI], F[c + sI] - F[c]) * inv_dr;
            at = minmod(F[c] - F[c - sJ], F[c + sJ] - F[c]) * inv_dthe;
            ap = minmod(F[c] - F[c - 1], F[c + 1] - F[c]) * inv_dphi;
        }
        adv_r[n] = ar; adv_t[n] = at; adv_p[n] = ap;
        tr[n] = u_exp * ar + v_invrm * at + w_invrs * ap;
    }
    if (p->metric_curvature) {   /* :823-828 */
        const double cotanthe = costhe / sinthe;
        tr[Y_U] += -(v_ijk * v_ijk + w_ijk * w_ijk) * inv_rm;
        tr[Y_V] += (u_ijk * v_ijk - w_ijk * w_ijk * cotanthe) * inv_rm;
        tr[Y_W] += (w_ijk * u_ijk + v_ijk * w_ijk * cotanthe) * inv_rm;
    }

    /* diffusion, RHS_Atm_Turb.cpp:858-942 */
    const double two_over_rm_exp = 2.0 * inv_rm * exp_rm;
    const double cos_rm2sin = G->costhe_inv_rm2sinthe;
    const double v_metric = (1.0 + costhe * costhe / sinthe2) * inv_rm2;
    const double diffusion_t = (d2r[Y_T] * exp_2_rm + d1r[Y_T] * two_over_rm_exp
        + d2t[Y_T] * inv_rm2 + d1t[Y_T] * cos_rm2sin + d2p[Y_T] * inv_rm2sinthe2) * diffusion_t_re;
    const double diffusion_u = (d2r[Y_U] * exp_2_rm + 2.0 * u_ijk * inv_rm2
        + d2t[Y_U] * inv_rm2 + 4.0 * d1r[Y_U] * inv_rm * exp_rm
        + d1t[Y_U] * cos_rm2sin + d2p[Y_U] * inv_rm2sinthe2) * diffusion_vel_re;
    const double diffusion_v = (d2r[Y_V] * exp_2_rm + d1r[Y_V] * two_over_rm_exp
        + d2t[Y_V] * inv_rm2 + d1t[Y_V] * cos_rm2sin
        - v_metric * v_ijk + d2p[Y_V] * inv_rm2sinthe2
        + 2.0 * d1t[Y_U] * inv_rm2
        - d1p[Y_W] * 2.0 * costhe * inv_rm2sinthe2) * diffusion_vel_re;
    const double diffusion_w = (d2r[Y_W] * exp_2_rm + d1r[Y_W] * two_over_rm_exp
        + d2t[Y_W] * inv_rm2 + d1t[Y_W] * cos_rm2sin
        - v_metric * w_ijk + d2p[Y_W] * inv_rm2sinthe2
        + 2.0 * d1p[Y_U] * inv_rm2sinthe
        + d1p[Y_V] * 2.0 * costhe * inv_rm2sinthe2) * diffusion_vel_re;
    const double dlnrho_dr_i = (p->tracer_diff_flux && dlnrho) ? dlnrho[i] * exp_2_rm : 0.0;
    double dtr[NY];
    for (int n = Y_C; n <= Y_CO; n++) {
        const double coef = (n == Y_CO) ? diff_co2_re_inv : diff_prec_re_inv;
        dtr[n] = (d2r[n] * exp_2_rm + d1r[n] * two_over_rm_exp
            + d2t[n] * inv_rm2 + d1t[n] * cos_rm2sin
            + d2p[n] * inv_rm2sinthe2
            + d1r[n] * dlnrho_dr_i) * coef;
    }
    const double diffusion_tke = (d2r[Y_TK] * exp_2_rm + dtkedr * two_over_rm_exp
        + d2t[Y_TK] * inv_rm2 + dtkedthe * cos_rm2sin + d2p[Y_TK] * inv_rm2sinthe2) * diffusion_tke_re;
    const double diffusion_dis = (d2r[Y_DI] * exp_2_rm + ddisdr * two_over_rm_exp
        + d2t[Y_DI] * inv_rm2 + ddisdthe * cos_rm2sin + d2p[Y_DI] * inv_rm2sinthe2) * diffusion_dis_re;

    /* assembly, RHS_Atm_Turb.cpp:946-1079 */
    const double dpdr_exp = dpdr * exp_rm, dpdthe_invrm = dpdthe * inv_rm, dpdphi_invrs = dpdphi * inv_rmsinthe;
    const double r_h = f[OF_R_HUMID][c];
    double rhs_t = pressure_t - tr[Y_T] + diffusion_t
        + coeff_MC_t * f[OF_MC_T][c]
        + coeff_energy * (f[OF_S_C][c] + f[OF_S_R][c]) * p->lv * r_h
        + coeff_energy * (f[OF_S_I][c] + f[OF_S_S][c] + f[OF_S_G][c]) * p->ls * r_h;
    {   /* Held-Suarez, :977-992 */
        const double k_a = 1.0 / (4.0 * 86400.0), k_s = 1.0 / (0.4 * 86400.0), sigma_b = 0.7;
        const double p_surf = f[OF_P_STAT][OR_IDX(0, j, k)];
        const double sigma = (p_surf > 0.0) ? f[OF_P_STAT][c] / p_surf : 0.0;
        double bl = (sigma - sigma_b) / (1.0 - sigma_b);
        if (bl < 0.0) bl = 0.0;
        const double cos4lat = sinthe2 * sinthe2;
        const double k_T = k_a + (k_s - k_a) * bl * cos4lat;
        rhs_t -= (k_T * p->L_atm / p->u_0) * (t_ijk - f[OF_T_EQ][c]);
    }
    const double rhs_u = -dpdr_exp - tr[Y_U] + diffusion_u
        + s->buoyancy_ramp * 1.0 * p->g * s->dt / p->u_0 * (t_ijk - t_ref[i])
        + coriolis * force_nd * coriolis_rad;
    const double rayleigh_kf = 1.0 / 86400.0, drag_n_layers = 5.0;
    double drag_profile = 1.0 - (double)(i - 0) / drag_n_layers;
    if (drag_profile < 0.0) drag_profile = 0.0;
    if (drag_profile > 1.0) drag_profile = 1.0;
    const double surf_drag = (rayleigh_kf * p->L_atm / p->u_0 * s->dt) * drag_profile;
    const double rhs_v = -dpdthe_invrm - tr[Y_V] + diffusion_v
        + coriolis * force_nd * coriolis_the
        + coeff_MC_vel * f[OF_MC_V][c]
        - surf_drag * v_ijk;
    const double rhs_w = -dpdphi_invrs - tr[Y_W] + diffusion_w
        + coriolis * force_nd * coriolis_phi
        + coeff_MC_vel * f[OF_MC_W][c]
        - surf_drag * w_ijk;
    o->k[Y_T] = rhs_t;
    o->k[Y_U] = rhs_u;
    o->k[Y_V] = rhs_v;
    o->k[Y_W] = rhs_w;
    o->k[Y_C] = -tr[Y_C] + dtr[Y_C] + coeff_trans * f[OF_S_V][c] * r_h + coeff_MC_q * f[OF_MC_Q][c];
    o->k[Y_CL] = -tr[Y_CL] + dtr[Y_CL] + coeff_trans * f[OF_S_C][c] * r_h;
    o->k[Y_IC] = -tr[Y_IC] + dtr[Y_IC] + coeff_trans * f[OF_S_I][c] * r_h;
    o->k[Y_GR] = -tr[Y_GR] + dtr[Y_GR] + coeff_trans * f[OF_S_G][c] * r_h;
    o->k[Y_CO] = -tr[Y_CO] + dtr[Y_CO];
    o->k[Y_TK] = -tr[Y_TK] + diffusion_tke + tke_source;
    o->k[Y_DI] = -tr[Y_DI] + diffusion_dis + dis_source;
    o->aux[0] = rhs_u + dpdr_exp;
    o->aux[1] = rhs_v + dpdthe_invrm;
    o->aux[2] = rhs_w + dpdphi_invrs;
    o->prod = prod;
    o->tke_source = tke_source;
    o->dis_source = dis_source;

    /* diagnostic outputs: acting forces (:447-456) */
    const double coeff_Coriolis = p->r_air * p->u_0 * p->omega, coeff_buoy = p->r_air * p->g;
    const double coeff_u_p = 0.5 * p->r_air * p->u_0 * p->u_0 / p->L_atm;
    o->force[0] = coriolis * coeff_Coriolis
        * sqrt((pow(coriolis_rad, 2) + pow(coriolis_the, 2) + pow(coriolis_phi, 2)) / 3.0);
    o->force[1] = 1.0 * coeff_buoy * (t_ijk - t_ref[i]);
    o->force[2] = -coeff_u_p
        * sqrt((pow(dpdr, 2) + pow(dpdthe * inv_rm, 2) + pow(dpdphi * inv_rmsinthe, 2)) / 3.0);
    /* latent heat of the advected condensate (:458-488): the thresholds are saturation mass
     * fractions at p_hydro, which nothing writes (0), so the rain branch is on below the
     * critical point (q = 0) and off above it (no saturation: q = 1); the ice branch (the
     * sublimation curve never reports "no saturation") always on */
    const double t_u = t_ijk * p->t_0;
    const double q_rain = or_saturation_mass_fraction(or_saturation_pressure(t_u), 0.0, 0.0);
    const double q_ice = or_saturation_mass_fraction(or_sublimation_pressure(t_u), 0.0, 0.0);
    const double c_ijk = Y[Y_C][c];
    double q_lat = (c_ijk >= 0.85 * q_rain)
        ? u_ijk * d1r[Y_CL] + v_ijk * inv_rm * d1t[Y_CL] + w_ijk * inv_rmsinthe * d1p[Y_CL] : 0.0;
    const double q_lat_ice = (c_ijk >= 0.85 * q_ice)
        ? u_ijk * d1r[Y_IC] + v_ijk * inv_rm * d1t[Y_IC] + w_ijk * inv_rmsinthe * d1p[Y_IC] : 0.0;
    const double coeff_S = p->lamda * p->t_0 / p->L_atm;
    const double coeff_L = p->r_air * p->c_0 * p->lv * p->u_0 / p->L_atm;
    o->q_latent = coeff_L * (q_lat + q_lat_ice);
    o->q_sensible = coeff_S * (d2r[Y_T] + d1r[Y_T] * 2.0 * inv_rm + d2t[Y_T] * inv_rm2
        + d1t[Y_T] * G->costhe_inv_rm2sinthe + d2p[Y_T] * inv_rm2sinthe2);
    /* momentum budget terms of rhs_v and rhs_w (:1031-1057) */
    o->vbud[0] = -dpdthe_invrm;
    o->vbud[1] = coriolis * force_nd * coriolis_the;
    o->vbud[2] = -(u_exp * adv_r[Y_V]);
    o->vbud[3] = -(v_invrm * adv_t[Y_V] + w_invrs * adv_p[Y_V]);
    o->vbud[4] = diffusion_v;
    o->vbud[5] = coeff_MC_vel * f[OF_MC_V][c] - surf_drag * v_ijk;
    o->wbud[0] = -dpdphi_invrs;
    o->wbud[1] = coriolis * force_nd * coriolis_phi;
    o->wbud[2] = -(u_exp * adv_r[Y_W]);
    o->wbud[3] = -(v_invrm * adv_t[Y_W] + w_invrs * adv_p[Y_W]);
    o->wbud[4] = diffusion_w;
    o->wbud[5] = coeff_MC_vel * f[OF_MC_W][c] - surf_drag * w_ijk;
}

/* write_diagnostics: bit 0 the turbulence production and sources, the acting forces and
 * the heat diagnostics; bit 1 the momentum budget terms (the reference's vbudget_capture /
 * wbudget_capture, set on its checkpoint iterations, cAtmosphereModel.cpp:1502-1503) */
static void store_diagnostics(double* const* f, size_t c, const rhs_out* o, int flags)
{
    if (flags & 1) {
        f[OF_PROD][c] = o->prod;
        f[OF_TKE_SOURCE][c] = o->tke_source;
        f[OF_DIS_SOURCE][c] = o->dis_source;
        f[OF_CORIOLIS_FORCE][c] = o->force[0];
        f[OF_BUOYANCY_FORCE][c] = o->force[1];
        f[OF_PRESSURE_GRADIENT_FORCE][c] = o->force[2];
        f[OF_Q_LATENT][c] = o->q_latent;
        f[OF_Q_SENSIBLE][c] = o->q_sensible;
    }
    if (flags & 2)
        for (int q = 0; q < 6; q++) {
            f[OF_VBUD_PGF + q][c] = o->vbud[q];
            f[OF_WBUD_PGF + q][c] = o->wbud[q];
        }
}

/* stage update, RungeKutta_Atm_Turb.cpp:167-182 (and its copies for stages 2-4) */
static void stage_store(double* const* Yo, size_t c, const double* yn, const double* kk,
                        double a, double tke_max_nd)
{
    Yo[Y_T][c] = yn[Y_T] + kk[Y_T] * a;
    Yo[Y_U][c] = yn[Y_U] + kk[Y_U] * a;
    Yo[Y_V][c] = yn[Y_V] + kk[Y_V] * a;
    Yo[Y_W][c] = yn[Y_W] + kk[Y_W] * a;
    Yo[Y_C][c] = or_max(0.0, yn[Y_C] + kk[Y_C] * a);
    Yo[Y_CL][c] = or_max(0.0, yn[Y_CL] + kk[Y_CL] * a);
    Yo[Y_IC][c] = or_max(0.0, yn[Y_IC] + kk[Y_IC] * a);
    Yo[Y_GR][c] = or_max(0.0, yn[Y_GR] + kk[Y_GR] * a);
    Yo[Y_CO][c] = yn[Y_CO] + kk[Y_CO] * a;
    Yo[Y_TK][c] = or_safe_clamp(yn[Y_TK] + kk[Y_TK] * a, 0.0, tke_max_nd);
    Yo[Y_DI][c] = or_max(1.0e-10, yn[Y_DI] + kk[Y_DI] * a);
}

static void final_store(double* const* Yo, size_t c, const double* yn, const double* k1,
                        const double* k2, const double* k3, const double* k4, double dt_sixth,
                        double tke_max_nd)
{
    double kk[NY];
    for (int n = 0; n < NY; n++) kk[n] = (k1[n] + 2.0 * k2[n] + 2.0 * k3[n] + k4[n]);
    stage_store(Yo, c, yn, kk, dt_sixth, tke_max_nd);
}

int or_rk4(int im, int jm, int km, const or_params* p, const or_step* s, int compat,
           double* const* f, double* const* prof)
{
    if (p->turb_model < 1 || p->turb_model > 3) return -1;
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    const size_t n = (size_t)im * jm * km;
    double* t_ref = prof[OFP_T_REF_LEVEL];
    level_mean_impl(&g, f[OF_T], t_ref, compat);
    const double* dlnrho = prof[OFP_DLNRHO_DR];
    const double half_dt = 0.5 * s->dt, dt_sixth = s->dt / 6.0;
    const double tke_max_nd = 1000.0 / (p->u_0 * p->u_0);
    double* Ycur[NY];
    const double* Yn[NY];
    for (int q = 0; q < NY; q++) { Ycur[q] = f[OF_T + q]; Yn[q] = f[OF_TN + q]; }
    const double* pd = f[OF_P_DYN];
    const double* nu = f[OF_NUE];

    if (compat) {
        /* In place, cell by cell: RungeKutta_Atm_Turb.cpp:99-266.  compat = 1 is the serial
         * (i, j, k) order.  compat = T > 1 reproduces the reference run with T OpenMP threads:
         * `collapse(2) schedule(static)` gives thread t one contiguous range of the (i, j)
         * rows, all ranges advance together, so where two ranges meet the later thread's
         * first rows are finished before the earlier thread reaches its last rows.  Running
         * the ranges one after another in reverse order reproduces exactly that. */
        const int T = compat;
        const long nrows = (long)(im - 2) * (jm - 2);
        const long q = nrows / T, rem = nrows % T;
        for (int th = T - 1; th >= 0; th--) {
            const long r0 = th * q + (th < rem ? th : rem);
            const long r1 = r0 + q + (th < rem ? 1 : 0);
            for (long r = r0; r < r1; r++) {
                const int i = 1 + (int)(r / (jm - 2)), j = 1 + (int)(r % (jm - 2));
                cgeo G;
                make_cgeo(&g, p, i, j, &G);
                for (int k = 1; k < km - 1; k++) {
                    const size_t c = OR_IDX(i, j, k);
                    double yn[NY];
                    for (int q = 0; q < NY; q++) yn[q] = Yn[q][c];
                    rhs_out o1, o2, o3, o4;
                    rhs_cell(&g, p, s, 1, i, j, k, &G, (const double* const*)Ycur, pd, nu, f, t_ref, dlnrho, &o1);
                    stage_store(Ycur, c, yn, o1.k, half_dt, tke_max_nd);
                    rhs_cell(&g, p, s, 1, i, j, k, &G, (const double* const*)Ycur, pd, nu, f, t_ref, dlnrho, &o2);
                    stage_store(Ycur, c, yn, o2.k, half_dt, tke_max_nd);
                    rhs_cell(&g, p, s, 1, i, j, k, &G, (const double* const*)Ycur, pd, nu, f, t_ref, dlnrho, &o3);
                    stage_store(Ycur, c, yn, o3.k, s->dt, tke_max_nd);
                    rhs_cell(&g, p, s, 1, i, j, k, &G, (const double* const*)Ycur, pd, nu, f, t_ref, dlnrho, &o4);
                    final_store(Ycur, c, yn, o1.k, o2.k, o3.k, o4.k, dt_sixth, tke_max_nd);
                    f[OF_AUX_U][c] = o4.aux[0];
                    f[OF_AUX_V][c] = o4.aux[1];
                    f[OF_AUX_W][c] = o4.aux[2];
                    store_diagnostics(f, c, &o4, s->write_diagnostics);
                }
            }
        }
        or_geom_free(&g);
        return 0;
    }

    /* Jacobi: every stage reads the previous stage's state everywhere.  Stage buffers
     * start as copies of the current state so boundary cells read their current value. */
    double* A[NY]; double* B[NY]; double* K[NY];
    for (int q = 0; q < NY; q++) {
        A[q] = (double*)malloc(n * sizeof(double));
        B[q] = (double*)malloc(n * sizeof(double));
        K[q] = (double*)calloc(n, sizeof(double));
        memcpy(A[q], Ycur[q], n * sizeof(double));
        memcpy(B[q], Ycur[q], n * sizeof(double));
    }
    for (int stage = 1; stage <= 4; stage++) {
        double* const* Yin = (stage == 1) ? Ycur : (stage == 3) ? B : A;
        double* const* Yout = (stage == 1 || stage == 3) ? A : (stage == 2) ? B : Ycur;
        for (int i = 1; i < im - 1; i++)
            for (int j = 1; j < jm - 1; j++) {
                cgeo G;
                make_cgeo(&g, p, i, j, &G);
                for (int k = 1; k < km - 1; k++) {
                    const size_t c = OR_IDX(i, j, k);
                    double yn[NY];
                    for (int q = 0; q < NY; q++) yn[q] = Yn[q][c];
                    rhs_out o;
                    rhs_cell(&g, p, s, 0, i, j, k, &G, (const double* const*)Yin, pd, nu, f, t_ref, dlnrho, &o);
                    if (stage < 4) {
                        for (int q = 0; q < NY; q++) {
                            const double w = (stage == 1) ? 1.0 : 2.0;
                            K[q][c] = (stage == 1) ? o.k[q] : K[q][c] + w * o.k[q];
                        }
                        stage_store(Yout, c, yn, o.k, (stage == 3) ? s->dt : half_dt, tke_max_nd);
                    } else {
                        double kk[NY];
                        for (int q = 0; q < NY; q++) kk[q] = K[q][c] + o.k[q];
                        stage_store(Yout, c, yn, kk, dt_sixth, tke_max_nd);
                        f[OF_AUX_U][c] = o.aux[0];
                        f[OF_AUX_V][c] = o.aux[1];
                        f[OF_AUX_W][c] = o.aux[2];
                        store_diagnostics(f, c, &o, s->write_diagnostics);
                    }
                }
            }
    }
    for (int q = 0; q < NY; q++) { free(A[q]); free(B[q]); free(K[q]); }
    or_geom_free(&g);
    return 0;
}

/* ---------------------------------------------------------------------------------- */
/* One PressureSolverAtm::run, flat terrain, PressureSolverAtm.h:27-594. */
static void pressure_run(const or_geom* g, const or_params* p, int total_iter_count,
                         double* const* f, const double* dlnrho_in, int64_t* counters)
{
    const int im = g->im, jm = g->jm, km = g->km;
    double* aux_u = f[OF_AUX_U]; double* aux_v = f[OF_AUX_V]; double* aux_w = f[OF_AUX_W];
    double* pd = f[OF_P_DYN];
    const size_t sI = (size_t)jm * km, sJ = (size_t)km;
    const int anelastic = p->anelastic && dlnrho_in != NULL;
    const double* dlnrho = anelastic ? dlnrho_in : NULL;
    /* c43 and c13 are `const int` members initialised from 4.0/3.0 and 1.0/3.0
     * (cAtmosphereModel.h:158), i.e. 1 and 0. */
    const double c43 = 1.0, c13 = 0.0;
    for (int j = 1; j < jm - 1; j++)           /* :106-121 */
        for (int k = 1; k < km - 1; k++) {
            if (anelastic) {
                aux_u[OR_IDX(0, j, k)] = 0.0;
                aux_u[OR_IDX(im - 1, j, k)] = 0.0;
            } else {
                aux_u[OR_IDX(0, j, k)] = c43 * aux_u[OR_IDX(1, j, k)] - c13 * aux_u[OR_IDX(2, j, k)];
                aux_u[OR_IDX(im - 1, j, k)] = c43 * aux_u[OR_IDX(im - 2, j, k)] - c13 * aux_u[OR_IDX(im - 3, j, k)];
            }
            aux_v[OR_IDX(0, j, k)] = c43 * aux_v[OR_IDX(1, j, k)] - c13 * aux_v[OR_IDX(2, j, k)];
            aux_v[OR_IDX(im - 1, j, k)] = c43 * aux_v[OR_IDX(im - 2, j, k)] - c13 * aux_v[OR_IDX(im - 3, j, k)];
            aux_w[OR_IDX(0, j, k)] = c43 * aux_w[OR_IDX(1, j, k)] - c13 * aux_w[OR_IDX(2, j, k)];
            aux_w[OR_IDX(im - 1, j, k)] = c43 * aux_w[OR_IDX(im - 2, j, k)] - c13 * aux_w[OR_IDX(im - 3, j, k)];
        }
    const double inv_2dr = 1.0 / (2.0 * g->dr), inv_2dthe = 1.0 / (2.0 * g->dthe),
                 inv_2dphi = 1.0 / (2.0 * g->dphi);
    const double inv_dr2 = 1.0 / (g->dr * g->dr), inv_dthe2 = 1.0 / (g->dthe * g->dthe),
                 inv_dphi2 = 1.0 / (g->dphi * g->dphi);
    const double p_dyn_cap = 2.0;
    int64_t n_cells = 0, n_clamped = 0;
    for (int colour = 0; colour < 2; colour++)      /* :225-486 */
        for (int i = 1; i < im - 1; i++)
            for (int j = 1; j < jm - 1; j++) {
                const double rm = g->rad[i];
                const double exp_rm = 1.0 / (rm + 1.0);
                const double exp_2_rm = exp_rm * exp_rm;
                const double sinthe = g->sin_f[j];
                const double sinthe2 = sinthe * sinthe;
                const double costhe = g->cos_t[j];
                const double rmet = or_metric_radius(g, p, rm);
                const double rmet2 = rmet * rmet;
                const double inv_rm = 1.0 / rmet;
                const double inv_rm2 = 1.0 / rmet2;
                const double inv_rmsinthe = 1.0 / (rmet * sinthe);
                const double inv_rm2sinthe2 = inv_rm2 / sinthe2;
                const double m_the = p->poisson_metric_fix ? inv_rm2 : inv_rm;
                const double m_phi = p->poisson_metric_fix ? inv_rm2sinthe2 : inv_rmsinthe;
                const double denom = 2.0 * exp_2_rm * inv_dr2 + 2.0 * m_the * inv_dthe2
                                   + 2.0 * m_phi * inv_dphi2;
                const double inv_denom = 1.0 / denom;
                const double num1 = exp_2_rm * inv_dr2, num2 = m_the * inv_dthe2, num3 = m_phi * inv_dphi2;
                const double num_a = anelastic ? exp_2_rm * dlnrho[i] * inv_2dr : 0.0;
                for (int k = 1; k < km - 1; k++) {
                    if (((i + j + k) & 1) != colour) continue;
                    const size_t c = OR_IDX(i, j, k);
                    const double du_dr = (aux_u[c + sI] - aux_u[c - sI]) * inv_2dr;
                    const double dv_dthe = (aux_v[c + sJ] - aux_v[c - sJ]) * inv_2dthe;
                    const double dw_dphi = (aux_w[c + 1] - aux_w[c - 1]) * inv_2dphi;
                    double div_src = du_dr * exp_rm + dv_dthe * inv_rm + dw_dphi * inv_rmsinthe;
                    if (anelastic) div_src += aux_u[c] * dlnrho[i] * exp_rm;
                    if (p->metric_divergence)
                        div_src += (2.0 * aux_u[c] + aux_v[c] * costhe / sinthe) * inv_rm;
                    const double src_max = denom * p_dyn_cap;
                    n_cells++;
                    if (!or_is_finite(div_src)) div_src = 0.0;
                    else if (div_src > src_max) { div_src = src_max; n_clamped++; }
                    else if (div_src < -src_max) { div_src = -src_max; n_clamped++; }
                    pd[c] = ((pd[c + sI] + pd[c - sI]) * num1
                           + (pd[c + sJ] + pd[c - sJ]) * num2
                           + (pd[c + 1] + pd[c - 1]) * num3
                           + (pd[c + sI] - pd[c - sI]) * num_a
                           - div_src) * inv_denom;
                }
            }
    /* radial (:504-526), pole (:535-541), seam (:544-552) */
    for (int k = 0; k < km; k++)
        for (int j = 0; j < jm; j++) {
            pd[OR_IDX(0, j, k)] = c43 * pd[OR_IDX(1, j, k)] - c13 * pd[OR_IDX(2, j, k)];
            pd[OR_IDX(im - 1, j, k)] = pd[OR_IDX(im - 2, j, k)];
        }
    for (int k = 0; k < km; k++)
        for (int i = 0; i < im; i++) {
            pd[OR_IDX(i, 0, k)] = pd[OR_IDX(i, 1, k)];
            pd[OR_IDX(i, jm - 1, k)] = pd[OR_IDX(i, jm - 2, k)];
        }
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            double* row = &pd[OR_IDX(i, j, 0)];
            row[0] = c43 * row[1] - c13 * row[2];
            row[km - 1] = c43 * row[km - 2] - c13 * row[km - 3];
            const double a = (row[0] + row[km - 1]) / 2.0;
            row[0] = a;
            row[km - 1] = a;
        }
    /* ceiling, :583-594 */
    const double ceil_ = (total_iter_count > 300) ? 3.0 : 10.0;
    const size_t n = (size_t)im * jm * km;
    for (size_t q = 0; q < n; q++) {
        const double v = pd[q];
        if (!or_is_finite(v)) pd[q] = 0.0;
        else if (v > ceil_) pd[q] = ceil_;
        else if (v < -ceil_) pd[q] = -ceil_;
    }
    if (counters) { counters[0] += n_cells; counters[1] += n_clamped; }
}

void or_pressure_sweep(int im, int jm, int km, const or_params* p, int compat,
                       int n_sweeps, int total_iter_count, double* const* f,
                       double* const* prof, int64_t* counters)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    if (counters) { counters[0] = 0; counters[1] = 0; }
    for (int s = 0; s < n_sweeps; s++)
        pressure_run(&g, p, total_iter_count, f, prof ? prof[OFP_DLNRHO_DR] : NULL, counters);
    or_geom_free(&g);
}

void or_project_initial_velocity(int im, int jm, int km, const or_params* p, int compat,
                                 int n_sweeps, int total_iter_count, double* const* f,
                                 double* const* prof)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    const size_t n = (size_t)im * jm * km;
    memcpy(f[OF_AUX_U], f[OF_U], n * sizeof(double));   /* :694-704 */
    memcpy(f[OF_AUX_V], f[OF_V], n * sizeof(double));
    memcpy(f[OF_AUX_W], f[OF_W], n * sizeof(double));
    memset(f[OF_P_DYN], 0, n * sizeof(double));
    for (int s = 0; s < n_sweeps; s++)
        pressure_run(&g, p, total_iter_count, f, prof ? prof[OFP_DLNRHO_DR] : NULL, NULL);
    const double inv_2dr = 1.0 / (2.0 * g.dr), inv_2dthe = 1.0 / (2.0 * g.dthe),
                 inv_2dphi = 1.0 / (2.0 * g.dphi);
    const double* pd = f[OF_P_DYN];
    const size_t sI = (size_t)jm * km, sJ = (size_t)km;
    for (int i = 1; i < im - 1; i++)                       /* :728-749 */
        for (int j = 1; j < jm - 1; j++) {
            const double rm = g.rad[i];
            const double exp_rm = 1.0 / (rm + 1.0);
            const double rmet = or_metric_radius(&g, p, rm);
            const double inv_rm = 1.0 / rmet;
            const double inv_rmsinthe = 1.0 / (rmet * g.sin_f[j]);
            for (int k = 1; k < km - 1; k++) {
                const size_t c = OR_IDX(i, j, k);
                const double dpdr = (pd[c + sI] - pd[c - sI]) * inv_2dr;
                const double dpdthe = (pd[c + sJ] - pd[c - sJ]) * inv_2dthe;
                const double dpdphi = (pd[c + 1] - pd[c - 1]) * inv_2dphi;
                f[OF_U][c] -= dpdr * exp_rm;
                f[OF_V][c] -= dpdthe * inv_rm;
                f[OF_W][c] -= dpdphi * inv_rmsinthe;
            }
        }
    memset(f[OF_P_DYN], 0, n * sizeof(double));            /* :752-762 */
    memset(f[OF_AUX_U], 0, n * sizeof(double));
    memset(f[OF_AUX_V], 0, n * sizeof(double));
    memset(f[OF_AUX_W], 0, n * sizeof(double));
    or_geom_free(&g);
}

/* storeIntermediateData3D, UtilsAtm.h:25-49 (coeff 1.0) */
void or_store_n_level(int im, int jm, int km, double* const* f)
{
    const size_t n = (size_t)im * jm * km;
    for (int q = 0; q < 11; q++) memcpy(f[OF_TN + q], f[OF_T + q], n * sizeof(double));
    memcpy(f[OF_P_RAINN], f[OF_P_RAIN], n * sizeof(double));    /* UtilsAtm.h:41-42 */
    memcpy(f[OF_P_SNOWN], f[OF_P_SNOW], n * sizeof(double));
}

/* RHS_Atmosphere_Turb at one interior cell of the current state (t_ref_level taken from
 * prof), with the reference's expression order when compat != 0.  out = rhs_t..rhs_dis,
 * aux_u/v/w, prod, tke_source, dis_source. */
void or_rhs_cell_at(int im, int jm, int km, const or_params* p, const or_step* s, int compat,
                    double* const* f, double* const* prof, int i, int j, int k, double* out)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    cgeo G;
    make_cgeo(&g, p, i, j, &G);
    const double* Y[NY];
    for (int q = 0; q < NY; q++) Y[q] = f[OF_T + q];
    rhs_out o;
    rhs_cell(&g, p, s, compat ? 1 : 0, i, j, k, &G, Y, f[OF_P_DYN], f[OF_NUE], f,
             prof[OFP_T_REF_LEVEL], prof[OFP_DLNRHO_DR], &o);
    for (int q = 0; q < NY; q++) out[q] = o.k[q];
    out[11] = o.aux[0]; out[12] = o.aux[1]; out[13] = o.aux[2];
    out[14] = o.prod; out[15] = o.tke_source; out[16] = o.dis_source;
    or_geom_free(&g);
}
