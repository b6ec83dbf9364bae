/*
 * or_init.c - the reference's deterministic initial state (TEST INFRASTRUCTURE ONLY, see
 * athad_oracle.h): cAtmosphereModel::RunTimeSlice for Ma = 0 (cAtmosphereModel.cpp:468-668)
 * on any grid, flat terrain, followed by run_3D_loop's Held-Suarez snapshot t_eq := t
 * (:750-753).  Its file output, printed diagnostics and the output-only arrays
 * (precipitableWater, forces' centrifugal and pressure-gradient arrays, vegetationLand,
 * standAtm_DewPoint_HumidRel) are left out: no field of the model state reads them.
 *
 * Grid generalisation (the reference fixes 61 x 181 x 361 at 1 degree):
 *   - VelocityInitializer's anchor row of latitude phi, lround(90 - phi)
 *     (VelocityInitializer.h:196-201), is lround((90 - phi) / dlat) with dlat = 180/(jm-1)
 *     degrees per row; its southern-hemisphere test j > 90 (:72) is j > (jm-1)/2.  Both
 *     are the reference's expressions at jm = 181.
 * compat = 0 (the device's semantics) differs from the reference only where the reference
 * breaks north-south mirror symmetry by rounding: the surface temperature parabola and the
 * velocity rows are evaluated on the northern half and mirrored (v negated), the cloud
 * ceiling's level sums run per row then over rows, and every module called on the way uses
 * its own compat = 0 form.  compat = 1 is the reference operation for operation, with its
 * modules in their reference forms on one thread.
 */
#include "or_internal.h"

size_t or_init_cfg_size(void) { return sizeof(or_init_cfg); }

/* AtomUtils::Agnesi (lib/Utils.h:176-179) */
static double agnesi(double a, double x) { return pow(a, 3.0) / (pow(a, 2.0) + pow(x, 2.0)); }

/* cAtmosphereModel::init_tropopause_layers (InitValues_Atm.cpp:330-401): the level of the
 * convective top per row, an Agnesi profile from the equator's height to the poles' */
void or_tropopause_layers(int im, int jm, const or_params* p, const or_init_cfg* c, double* levels)
{
    const int j_max = jm - 1, j_half = j_max / 2;
    const double x_max = c->tropopause_equator * sqrt(c->tropopause_equator / c->tropopause_pole - 1.0);
    const double idx_scale = (double)(im - 1) / p->zeta;
    for (int j = 0; j <= j_half; j++) {
        const double x = x_max * (double)(j_half - j) / (double)j_half;
        const double h = agnesi(c->tropopause_equator, x);
        double lev = 0.0;
        if ((h > 0.0) && (p->L_atm > 0.0) && (p->zeta > 0.0)) {
            lev = round(idx_scale * log(1.0 + h / p->L_atm));
            lev = or_min(or_max(lev, 0.0), (double)(im - 1));
        }
        levels[j] = lev;
        levels[j_max - j] = lev;
    }
}

/* ---- VelocityInitializer::compute (VelocityInitializer.h:23-105) ---------------------- */

typedef struct vel_ctx {
    int im, jm, km, compat;
    const or_params* p;
    const or_init_cfg* c;
    const double* height;      /* get_layer_height(i), float values */
    const double* trop;        /* tropopause_layers[j] */
    double* u; double* v; double* w;   /* (i, j) tables, broadcast along k afterwards */
} vel_ctx;

#define VT(a, i, j) ((a)[(size_t)(i) * V->jm + (j)])

static double edge_lat(const vel_ctx* V, int k)                     /* :185-190 */
{
    const int n = V->c->n_cells_hemisphere;
    if (k <= 0) return 0.0;
    if (n <= 1) return 90.0;
    const double h = 30.0 * V->c->cell_lat_scale;
    return h + (90.0 - h) * (double)(k - 1) / (double)(n - 1);
}
static double centre_lat(const vel_ctx* V, int k) { return 0.5 * (edge_lat(V, k) + edge_lat(V, k + 1)); }
static int j_north(const vel_ctx* V, double phi)                    /* :192-197 */
{
    const double dlat = 180.0 / (double)(V->jm - 1);
    int j = (int)lround((90.0 - phi) / dlat);
    if (j < 0) j = 0;
    if (j > V->jm - 1) j = V->jm - 1;
    return j;
}
static int j_south(const vel_ctx* V, double phi) { return (V->jm - 1) - j_north(V, phi); }
static int trop_layer(const vel_ctx* V, int j) { return (int)V->trop[j]; }   /* cAtmosphereModel.h:222-230 */

typedef struct amp { double v_trop, v_surf, w_trop, w_surf; int has_w; } amp;
static amp edge_amp(int k, int n)                                   /* :210-226 */
{
    const amp eq = { 0.0, 0.0, -3.0, -5.0, 1 }, pole = { 0.5, 0.0, 0.0, 0.0, 1 };
    const amp subtrop = { 0.0, 0.5, 30.0, -1.0, 1 }, subpolar = { -0.2, 0.0, 10.0, 6.0, 1 };
    if (k == 0) return eq;
    if (k == n) return pole;
    if (k == 1) return subtrop;
    return subpolar;
}
static amp centre_amp(int k, int n)                                 /* :211-213, :227-231 */
{
    const amp hadley = { -3.0, 3.5, 5.0, -7.0, 1 }, ferrel = { 4.0, -1.5, 15.0, 10.0, 1 };
    const amp polar = { 0.5, 0.6, 0.0, 0.0, 0 };
    if (k == 0) return hadley;
    if (k == n - 1) return polar;
    return ferrel;
}
static double edge_radial_coeff(int k, double phi)                 /* :236-244 */
{
    double mag;
    if (phi == 0.0) mag = 0.02894;
    else if (phi == 30.0) mag = 0.02315;
    else if (phi == 60.0) mag = 0.01736;
    else if (phi == 90.0) mag = 0.011574;
    else mag = 0.02894 * (1.0 - phi / 150.0);
    return (k % 2 == 0) ? mag : -mag;
}
static double amp_scale(const vel_ctx* V, int is_v)                 /* :309-317 */
{
    const double s = V->c->cell_lat_scale;
    switch (V->c->cell_amp_mode) {
        case 1: return s;
        case 2: return is_v ? s : s * s;
        default: return 1.0;
    }
}
static void init_u_row(vel_ctx* V, int j, double coeff)            /* :341-360 */
{
    const int tl = trop_layer(V, j);
    const double tropo_h = (float)V->height[tl];
    const double half_tropo_h = tropo_h / 3.0;
    const double inv_ascent = 3.0 / half_tropo_h;
    const double inv_descent = 1.0 / half_tropo_h;
    for (int i = 0; i < tl; i++) {
        const double h = (float)V->height[i];
        const double ratio = (h < half_tropo_h) ? h * inv_ascent : (tropo_h - h) * inv_descent;
        VT(V->u, i, j) = coeff * ratio;
    }
}
static void init_v_or_w_row(vel_ctx* V, double* a, int is_v, int j, double coeff_trop, double coeff_sl)
{                                                                   /* :362-402 */
    const int tl = trop_layer(V, j);
    const double inv_tropo_h = 1.0 / (float)V->height[tl];
    const double s = amp_scale(V, is_v);
    coeff_trop *= s;
    coeff_sl *= s;
    const double slope = (coeff_trop - coeff_sl) * inv_tropo_h;
    for (int i = 0; i < tl; i++) VT(a, i, j) = slope * (float)V->height[i] + coeff_sl;
    if (tl >= V->im - 1) return;
    const double h_top = (float)V->height[V->im - 1];
    const double inv_range = 1.0 / (h_top - (float)V->height[tl]);
    for (int i = tl; i < V->im; i++) VT(a, i, j) = coeff_trop * (h_top - (float)V->height[i]) * inv_range;
}
static void set_anchor(vel_ctx* V, double phi, amp a)              /* :246-255 */
{
    const int jn = j_north(V, phi), js = j_south(V, phi);
    init_v_or_w_row(V, V->v, 1, jn, a.v_trop, a.v_surf);
    if (js != jn) init_v_or_w_row(V, V->v, 1, js, a.v_trop, a.v_surf);
    if (a.has_w) {
        init_v_or_w_row(V, V->w, 0, jn, a.w_trop, a.w_surf);
        if (js != jn) init_v_or_w_row(V, V->w, 0, js, a.w_trop, a.w_surf);
    }
}
static int cmp_int(const void* a, const void* b) { return *(const int*)a - *(const int*)b; }
/* sorted, de-duplicated anchor rows, pole to pole (:258-276) */
static int anchor_list(const vel_ctx* V, int with_centres, int skip_polar_centre, int* out)
{
    const int n = V->c->n_cells_hemisphere;
    double phis[64];
    int np = 0, m = 0;
    for (int k = 0; k <= n; k++) phis[np++] = edge_lat(V, k);
    if (with_centres)
        for (int k = 0; k < n; k++) {
            if (skip_polar_centre && k == n - 1) continue;
            phis[np++] = centre_lat(V, k);
        }
    for (int q = 0; q < np; q++) {
        out[m++] = j_north(V, phis[q]);
        if (j_south(V, phis[q]) != j_north(V, phis[q])) out[m++] = j_south(V, phis[q]);
    }
    qsort(out, (size_t)m, sizeof(int), cmp_int);
    int u = 0;
    for (int q = 0; q < m; q++)
        if (u == 0 || out[u - 1] != out[q]) out[u++] = out[q];
    return u;
}
static void form_diagonals(vel_ctx* V, double* a, int start, int end)   /* :404-419 */
{
    const double inv_range = 1.0 / (double)(end - start);
    for (int i = 0; i < V->im; i++) {
        const double a_start = VT(a, i, start);
        const double slope = (VT(a, i, end) - a_start) * inv_range;
        for (int j = start; j < end; j++) VT(a, i, j) = slope * (double)(j - start) + a_start;
    }
}
static void form_chain(vel_ctx* V, double* a, const int* anchors, int n)  /* :278-281 */
{
    for (int q = 0; q + 1 < n; q++)
        if (anchors[q + 1] > anchors[q]) form_diagonals(V, a, anchors[q], anchors[q + 1]);
}

static void velocity_tables(vel_ctx* V)
{
    const int n = V->c->n_cells_hemisphere;
    const int jeq = (V->jm - 1) / 2;
    for (int k = 0; k <= n; k++) {                                  /* :34-39 */
        const double phi = edge_lat(V, k);
        const double coeff = edge_radial_coeff(k, phi);
        init_u_row(V, j_north(V, phi), coeff);
        if (j_south(V, phi) != j_north(V, phi)) init_u_row(V, j_south(V, phi), coeff);
    }
    for (int k = 0; k <= n; k++) set_anchor(V, edge_lat(V, k), edge_amp(k, n));   /* :48-49 */
    for (int k = 0; k < n; k++) set_anchor(V, centre_lat(V, k), centre_amp(k, n));
    int anchors[256];
    int na = anchor_list(V, 0, 0, anchors);                         /* :55-57 */
    form_chain(V, V->u, anchors, na);
    na = anchor_list(V, 1, 0, anchors);
    form_chain(V, V->v, anchors, na);
    na = anchor_list(V, 1, 1, anchors);
    form_chain(V, V->w, anchors, na);
    const double inv_u_0 = 1.0 / V->p->u_0;                         /* :60-79 */
    for (int i = 0; i < V->im; i++)
        for (int j = 0; j < V->jm; j++) {
            VT(V->u, i, j) *= inv_u_0;
            VT(V->w, i, j) *= inv_u_0;
            if (j > jeq) VT(V->v, i, j) = -VT(V->v, i, j) * inv_u_0;
            else VT(V->v, i, j) *= inv_u_0;
        }
    if (!V->compat) {
        /* the southern rows as the mirror of the northern ones: the reference interpolates
         * each hemisphere from its own end, which rounds differently */
        for (int i = 0; i < V->im; i++)
            for (int j = 0; j <= jeq; j++) {
                const int jr = V->jm - 1 - j;
                if (jr == j) continue;
                VT(V->u, i, jr) = VT(V->u, i, j);
                VT(V->w, i, jr) = VT(V->w, i, j);
                VT(V->v, i, jr) = -VT(V->v, i, j);
            }
    }
}

/* ---- initTemperatureData (InitValues_Atm.cpp:466-620), Ma = 0, flat terrain ---------- */

static void init_temperature(int im, int jm, int km, const or_params* p, const or_init_cfg* c, int compat,
                             const double* height, double* const* f, double* const* f2)
{
    const double inv_t0 = 1.0 / p->t_0;
    const double d_j_half = 0.5 * (jm - 1);
    double* Ts = (double*)malloc(sizeof(double) * jm);
    for (int j = 0; j < jm; j++) {
        const double ratio = (double)j / d_j_half;
        const double para = ratio * ratio - 2.0 * ratio;              /* AtomUtils::parabola */
        Ts[j] = (c->t_surf_pole - c->t_surf_equator) * para + c->t_surf_pole;
    }
    if (!compat)
        for (int j = 0; j < jm / 2; j++) Ts[jm - 1 - j] = Ts[j];
    for (int k = 0; k < km; k++)
        for (int j = 0; j < jm; j++) f[OF_T][OR_IDX(0, j, k)] = Ts[j] * inv_t0;
    free(Ts);
    const double R_mix = p->R_mix, R_bg = p->R_bg, M_bg = p->M_bg;
    for (int k = 0; k < km; k++)
        for (int j = 0; j < jm; j++) {
            const double t_u_init = f[OF_T][OR_IDX(0, j, k)] * p->t_0;
            f[OF_P_STAT][OR_IDX(0, j, k)] = 1e-2 * (p->r_air * R_mix * t_u_init);
            f[OF_T][OR_IDX(0, j, k)] = t_u_init;
            double T_prev = or_max(100.0, f[OF_T][OR_IDX(0, j, k)]);
            double p_prev = f[OF_P_STAT][OR_IDX(0, j, k)];
            for (int i = 0; i < im; i++) {
                const size_t q = OR_IDX(i, j, k);
                const double q_v = f[OF_C][q], q_c = f[OF_CO2][q];
                const double R_loc = or_R_of(q_v, q_c, R_bg);
                double T_curr, p_val;
                if (i == 0) {
                    T_curr = T_prev;
                    p_val = p_prev;
                } else {
                    /* get_layer_height(i) - get_layer_height(i-1): a float difference */
                    const double dz = (float)((float)height[i] - (float)height[i - 1]);
                    const double cp_loc = or_cp_of(q_v, q_c, T_prev, M_bg);
                    const double T_ad = T_prev - (p->g / cp_loc) * dz;
                    T_curr = or_max(p->t_skin, T_ad);
                    const double T_mean = 0.5 * (T_prev + T_curr);
                    p_val = p_prev * exp(-p->g * dz / (R_loc * T_mean));
                }
                f[OF_T][q] = T_curr;
                f[OF_P_STAT][q] = p_val;
                const double twf = or_max(0.5, 1.0 - (f[OF_CLOUD][q] + f[OF_ICE][q]));
                const double R_dloc = or_R_of(0.0, q_c, R_bg);
                f[OF_R_DRY][q] = p_val * 100.0 / (R_dloc * T_curr);
                f[OF_R_HUMID][q] = p_val * 100.0 / (R_loc * T_curr * twf);
                T_prev = T_curr;
                p_prev = p_val;
            }
            f2[OF2_P_STAT_LANDSCAPE][(size_t)j * km + k] = f[OF_P_STAT][OR_IDX(0, j, k)];
        }
    for (int j = 0; j < jm; j++)                                    /* Step 9 */
        for (int k = 0; k < km; k++)
            for (int i = 0; i < im; i++) f[OF_T][OR_IDX(i, j, k)] *= inv_t0;
}

/* ---- initWaterWapour (InitValues_Atm.cpp:843-926): the saturation profile over the
 *      dry-top floor, a running minimum up each column ---------------------------------- */
static void init_water_vapour(int im, int jm, int km, const or_params* p, double* const* f)
{
    const double M_nw = or_M_nonwater(p->c_0, p->co2_0, p->M_bg);
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            double q_sat_min = 1.0;
            for (int i = 0; i < im; i++) {
                const size_t q = OR_IDX(i, j, k);
                const double T_i = f[OF_T][q] * p->t_0;
                const double q_s = or_saturation_mass_fraction_at(T_i, f[OF_P_STAT][q], M_nw);
                if (q_s < q_sat_min) q_sat_min = q_s;
                f[OF_C][q] = or_max(q_sat_min, p->c_h2o_dry_top);
                f[OF_CLOUD][q] = 0.0;
            }
        }
}

/* ThermoAtm::co2Atmosphere (ThermoAtm.h:873-918): CO2 well mixed in the dry air */
static void co2_atmosphere(int im, int jm, int km, const or_params* p, const or_init_cfg* c, double* const* f)
{
    const double co2_ref = p->co2_0 * c->co2_scale;
    const double f_CO2 = (c->q_CO2 + c->q_bg > 0.0) ? c->q_CO2 / (c->q_CO2 + c->q_bg) : co2_ref;
    const size_t n = (size_t)im * jm * km;
    for (size_t q = 0; q < n; q++) f[OF_CO2][q] = (1.0 - f[OF_C][q]) * f_CO2 * c->co2_scale;
}

/* ---- initCloudIce (InitValues_Atm.cpp:930-1117) --------------------------------------- */
static double cloud_excess(const or_params* p, double t_u, double p_u, double c, double co2, double factor,
                           double* q_sat_out)
{
    const double E_sat = (t_u >= p->t_0) ? or_saturation_pressure(t_u) : or_sublimation_pressure(t_u);
    const double q_sat = or_saturation_mass_fraction(E_sat, p_u, or_M_nonwater(c, co2, p->M_bg));
    if (q_sat_out) *q_sat_out = q_sat;
    return or_max(0.0, c - factor * q_sat);
}

static void init_cloud_ice(int im, int jm, int km, const or_params* p, int compat, const double* height,
                           double* const* f)
{
    const double alfa_s = 1.5, Hu_cr_max = 1.0, Hu_cr_mid = 0.8;
    const double Hu_diff = Hu_cr_max - Hu_cr_mid;
    const double det_T_0 = p->t_0;
    const double p_crit = p->p_0, p_mid = 0.55 * p->p_0;
    const double x_mid = p_mid / p_crit;
    const double Hu_curv = Hu_diff / (x_mid * (1.0 - x_mid));
    const double inv_p_crit = 1.0 / p_crit;
    double* cloud_max = (double*)calloc(im, sizeof(double));
    double* term = (double*)malloc(sizeof(double) * km);
    for (int i = 0; i < im; i++) {
        double sum = 0.0;
        for (int j = 0; j < jm; j++) {
            for (int k = 0; k < km; k++) {
                const size_t q = OR_IDX(i, j, k);
                const double t_u = f[OF_T][q] * p->t_0;
                term[k] = (t_u >= OR_T_CRIT) ? 0.0
                        : cloud_excess(p, t_u, f[OF_P_STAT][q], f[OF_C][q], f[OF_CO2][q], 0.74, NULL);
                if (compat && t_u < OR_T_CRIT) sum += term[k];
            }
            /* the device's order: a warp's 32 strided partial sums of the row, combined in
             * xor-butterfly order, then the rows one after another */
            if (!compat) {
                double part[32];
                for (int l = 0; l < 32; l++) {
                    double a = 0.0;
                    for (int k = l; k < km; k += 32) a += term[k];
                    part[l] = a;
                }
                for (int off = 16; off >= 1; off >>= 1) {
                    double nxt[32];
                    for (int l = 0; l < 32; l++) nxt[l] = part[l] + part[l ^ off];
                    memcpy(part, nxt, sizeof part);
                }
                sum += part[0];
            }
        }
        cloud_max[i] = sum / ((jm - 1) * (km - 1));
        if (cloud_max[i] <= 1e-4) cloud_max[i] = 1e-4;
    }
    double* step = (double*)calloc(im, sizeof(double));
    double* dt_dim = (double*)calloc(im, sizeof(double));
    double* alfa_over_cmax = (double*)calloc(im, sizeof(double));
    double* two_step = (double*)calloc(im, sizeof(double));
    for (int i = 0; i < im - 1; i++) {
        step[i] = (float)((float)height[i + 1] - (float)height[i]);
        dt_dim[i] = step[i] / 1.6;
        alfa_over_cmax[i] = alfa_s / cloud_max[i];
        two_step[i] = 2.0 * step[i];
    }
    step[im - 1] = step[im - 2];
    dt_dim[im - 1] = dt_dim[im - 2];
    alfa_over_cmax[im - 1] = alfa_over_cmax[im - 2];
    two_step[im - 1] = two_step[im - 2];
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            for (int i = 0; i < im; i++) {
                const size_t q = OR_IDX(i, j, k);
                const double t_u = f[OF_T][q] * p->t_0;
                const double p_u = f[OF_P_STAT][q];
                if (t_u >= OR_T_CRIT) {
                    f[OF_CLOUD][q] = 0.0; f[OF_ICE][q] = 0.0; f[OF_GR][q] = 0.0;
                    continue;
                }
                double q_sat;
                (void)cloud_excess(p, t_u, p_u, f[OF_C][q], f[OF_CO2][q], 0.0, &q_sat);
                const double x_norm = p_u * inv_p_crit;
                double H_crit = Hu_cr_max - Hu_curv * x_norm * (1.0 - x_norm);
                if (H_crit > 1.0) H_crit = 1.0;
                const double del_q_ls = or_max(0.0, f[OF_C][q] - H_crit * q_sat);
                const double cloud_ls = cloud_max[i] * (1.0 - exp(-alfa_over_cmax[i] * del_q_ls));
                double cloud_conv = 0.0;
                if (f[OF_P_RAIN][q] > 0.0 && i < im - 1) {
                    const double del_q_conv = or_max(0.0,
                        (f[OF_P_RAIN][OR_IDX(i + 1, j, k)] - f[OF_P_RAIN][q])
                        / (two_step[i] * f[OF_R_HUMID][q]) * dt_dim[i]);
                    cloud_conv = cloud_max[i] * (1.0 - exp(-alfa_over_cmax[i] * del_q_conv));
                }
                const double cloud_val = cloud_ls + cloud_conv;
                f[OF_CLOUD][q] = cloud_val;
                double h_T = 0.0;
                if (t_u < p->t_0) {
                    const double ratio = (t_u - p->t_0) / det_T_0;
                    h_T = 1.0 - exp(-0.5 * ratio * ratio);
                }
                f[OF_ICE][q] = cloud_val * h_T;
                f[OF_GR][q] = 0.1 * cloud_val * h_T;
                if (t_u <= p->t_00) {
                    f[OF_CLOUD][q] = 0.0; f[OF_ICE][q] = 0.0; f[OF_GR][q] = 0.0;
                }
            }
    free(term); free(cloud_max); free(step); free(dt_dim); free(alfa_over_cmax); free(two_step);
}

/* ---- TurbulenceAtm::init (TurbulenceAtm.h:39-59): compute_vel_star, init_fields
 *      (:193-265), apply_wall_bc; its compute_sources and clamp_nue are or_turbulence_run's */
static void turbulence_init_fields(int im, int jm, int km, const or_params* p, const double* height,
                                   double* const* f, double* const* f2)
{
    const double C_nue = 0.028, Karman = 0.42, dis_min = 1.0e-10;
    double* vs = f2[OF2_VEL_STAR];
    for (int j = 0; j < jm; j++)                                    /* compute_vel_star */
        for (int k = 0; k < km; k++) {
            const int i_surf = (1 < im - 1) ? 1 : im - 1;
            const double v_s = f[OF_V][OR_IDX(i_surf, j, k)], w_s = f[OF_W][OR_IDX(i_surf, j, k)];
            const double U_horiz = p->u_0 * sqrt(v_s * v_s + w_s * w_s);
            vs[(size_t)j * km + k] = or_max(0.05, sqrt(0.002) * U_horiz);
        }
    const double inv_u02 = 1.0 / (p->u_0 * p->u_0);
    const double nd_omega = p->L_atm / p->u_0;
    const double nd_eps = p->L_atm / (p->u_0 * p->u_0 * p->u_0);
    for (int j = 1; j < jm - 1; j++)
        for (int k = 1; k < km - 1; k++) {
            const double v = vs[(size_t)j * km + k];
            const double k_bg = 0.01 * v * v / sqrt(C_nue);
            const double om_bg = pow(C_nue, -0.25) * sqrt(k_bg) / (Karman * p->L_atm);
            const double eps_bg = pow(C_nue, 0.75) * pow(k_bg, 1.5) / (Karman * p->L_atm);
            const double y_mount = (float)height[0];
            for (int i = 1; i < im - 1; i++) {
                const size_t q = OR_IDX(i, j, k);
                const double z_i = (float)height[i] - y_mount;
                const double z_safe = or_max(z_i, 1.0e-6);
                const double z_frac = or_min(z_i, p->abl_height) / p->abl_height;
                const double k_abl = v * v / sqrt(C_nue) * pow(1.0 - z_frac, 2);
                const double k_phys = or_max(k_abl, k_bg);
                double dis_nd;
                if (p->turb_model == 1) {
                    const double eps_phys = pow(C_nue, 0.75) * pow(k_phys, 1.5) / (Karman * z_safe);
                    dis_nd = or_max(eps_phys, eps_bg) * nd_eps;
                } else {
                    const double om_phys = pow(C_nue, -0.25) * sqrt(k_phys) / (Karman * z_safe);
                    dis_nd = or_max(om_phys, om_bg) * nd_omega;
                }
                f[OF_TKE][q] = or_max(0.0, k_phys * inv_u02);
                f[OF_DIS][q] = or_max(dis_min, dis_nd);
                f[OF_TKEN][q] = f[OF_TKE][q];
                f[OF_DISN][q] = f[OF_DIS][q];
            }
        }
    or_turb_wall_bc(im, jm, km, p, f, f2);
}

/* ThermoAtm::forces (ThermoAtm.h:518-614), the two arrays it shares with the right-hand side's
 * outputs: CoriolisForce and BuoyancyForce of the interior cells (its centrifugal and
 * pressure-gradient arrays are output only).  Coriolis and buoyancy are the configuration's
 * 1; the buoyancy reference is the level-mean temperature t_ref, or 1 where none exists yet
 * (t_ref NULL: before the first RK4 step). */
static void forces(int im, int jm, int km, const or_params* p, const or_geom* g, double* const* f,
                   const double* t_ref)
{
    const double two_omega = 2.0 * p->omega;
    const double nontrad_d = p->coriolis_nontrad ? 1.0 : 0.0;
    for (int i = 1; i < im - 1; i++)
        for (int j = 1; j < jm - 1; j++) {
            const double sinthe = g->sin_w[j], costhe = g->cos_t[j];
            for (int k = 1; k < km - 1; k++) {
                const size_t q = OR_IDX(i, j, k);
                const double w_ijk = f[OF_W][q] * p->u_0;
                const double Cor_r = -nontrad_d * two_omega * sinthe * w_ijk;
                const double Cor_the = two_omega * costhe * w_ijk;
                const double Cor_phi = -two_omega * (costhe * f[OF_V][q] + nontrad_d * sinthe * f[OF_U][q]) * p->u_0;
                f[OF_CORIOLIS_FORCE][q] = 1.0 * p->r_air
                    * sqrt(Cor_r * Cor_r + Cor_the * Cor_the + Cor_phi * Cor_phi);
                f[OF_BUOYANCY_FORCE][q] = 1.0e-3 * 1.0 * f[OF_R_HUMID][q] * p->g
                                        * (f[OF_T][q] - (t_ref ? t_ref[i] : 1.0));
            }
        }
}

void or_forces(int im, int jm, int km, const or_params* p, int compat, double* const* f,
               const double* t_ref)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    forces(im, jm, km, p, &g, f, t_ref);
    or_geom_free(&g);
}

static void precipitation_sum(int im, int jm, int km, double* const* f)   /* UtilsAtm.h:51-65 */
{
    const size_t n = (size_t)im * jm * km;
    for (size_t q = 0; q < n; q++)
        f[OF_PRECIPITATION][q] = f[OF_P_RAIN][q] + f[OF_P_SNOW][q] + f[OF_P_GRAUPEL][q] + f[OF_P_CONV][q];
}

/* The reference's sequence, RunTimeSlice (cAtmosphereModel.cpp:468-668), up to stage
 * `upto` (OR_INIT_* of athad_oracle.h; OR_INIT_ALL = everything). */
int or_init_state(int im, int jm, int km, const or_params* p, const or_init_cfg* c, int compat, int upto,
                  double* const* f, double* const* f2, double* const* prof)
{
    if (!c || c->struct_size != sizeof(or_init_cfg) || c->n_cells_hemisphere < 1 || c->n_cells_hemisphere > 30)
        return -1;
    const int cm = compat ? 1 : 0;
    or_geom g;
    or_geom_init(&g, im, jm, km, p, cm);
    const size_t n = (size_t)im * jm * km, n2 = (size_t)jm * km;
    int rc = 0;
    double* trop = (double*)malloc(sizeof(double) * jm);

    /* UtilsAtm::resetArrays (UtilsAtm.h:364-451): zero, except t, tn, t_eq, co2n, s, s_u,
     * s_d = 1, HumidityRel = 100 and vel_star = 0.4 */
    for (int q = 0; q < OF_NFIELDS; q++) memset(f[q], 0, sizeof(double) * n);
    const int ones[] = { OF_T, OF_TN, OF_T_EQ, OF_CO2N, OF_MC_S, OF_MC_S_U, OF_MC_S_D };
    for (int q = 0; q < (int)(sizeof ones / sizeof ones[0]); q++)
        for (size_t e = 0; e < n; e++) f[ones[q]][e] = 1.0;
    for (size_t e = 0; e < n; e++) f[OF_HUMIDITY_REL][e] = 100.0;
    for (int q = 0; q < OF2_N; q++) memset(f2[q], 0, sizeof(double) * n2);
    for (size_t e = 0; e < n2; e++) f2[OF2_VEL_STAR][e] = c->vel_star_init;
    for (int q = 0; q < OFP_N; q++) memset(prof[q], 0, sizeof(double) * im);
    or_tropopause_layers(im, jm, p, c, trop);

    /* VelocityInitializer::compute, then bcVelSurfSur (nothing without land) and the
     * wiggle filter of u, v, w (:512-520) */
    {
        vel_ctx V = { im, jm, km, cm, p, c, g.height, trop, NULL, NULL, NULL };
        V.u = (double*)calloc((size_t)im * jm, sizeof(double));
        V.v = (double*)calloc((size_t)im * jm, sizeof(double));
        V.w = (double*)calloc((size_t)im * jm, sizeof(double));
        velocity_tables(&V);
        for (int i = 0; i < im; i++)
            for (int j = 0; j < jm; j++)
                for (int k = 0; k < km; k++) {
                    f[OF_U][OR_IDX(i, j, k)] = V.u[(size_t)i * jm + j];
                    f[OF_V][OR_IDX(i, j, k)] = V.v[(size_t)i * jm + j];
                    f[OF_W][OR_IDX(i, j, k)] = V.w[(size_t)i * jm + j];
                }
        free(V.u); free(V.v); free(V.w);
        or_damp_wiggles(im, jm, km, f[OF_U], cm);
        or_damp_wiggles(im, jm, km, f[OF_V], cm);
        or_damp_wiggles(im, jm, km, f[OF_W], cm);
    }
    if (upto <= OR_INIT_VELOCITY) goto done;

    init_temperature(im, jm, km, p, c, cm, g.height, f, f2);       /* :524-525 */
    or_damp_wiggles(im, jm, km, f[OF_T], cm);
    for (int j = 0; j < jm; j++)                                    /* :530-536 */
        for (int k = 0; k < km; k++) f2[OF2_T_TOP_INIT][(size_t)j * km + k] = f[OF_T][OR_IDX(im - 1, j, k)];
    if (upto <= OR_INIT_TEMPERATURE) goto done;

    init_water_vapour(im, jm, km, p, f);                            /* :563-567 */
    for (int pass = 0; pass < 2; pass++) {
        co2_atmosphere(im, jm, km, p, c, f);
        or_densities(im, jm, km, p, cm, 1, f, f2, prof);
    }
    if (upto <= OR_INIT_WATER) goto done;

    init_cloud_ice(im, jm, km, p, cm, g.height, f);                 /* :569 */
    if (upto <= OR_INIT_CLOUD) goto done;

    or_saturation_adjust(im, jm, km, p, cm, f, NULL);               /* :574-577 */
    or_damp_wiggles(im, jm, km, f[OF_ICE], cm);
    or_damp_wiggles(im, jm, km, f[OF_C], cm);
    or_damp_wiggles(im, jm, km, f[OF_CLOUD], cm);
    if (upto <= OR_INIT_SATADJ) goto done;

    or_ice_scheme(im, jm, km, p, f);                                /* :581-596 */
    or_damp_wiggles(im, jm, km, f[OF_P_RAIN], cm);
    or_damp_wiggles(im, jm, km, f[OF_P_SNOW], cm);
    if (upto <= OR_INIT_ICE) goto done;

    if (or_moist_convection(im, jm, km, p, cm, 0, f, f2) != 0) { rc = -2; goto done; }   /* :599-608 */
    {
        const int mc[] = { OF_P_CONV, OF_E_U, OF_M_U, OF_Q_V_U, OF_Q_C_U, OF_E_D, OF_M_D, OF_Q_V_D };
        for (int q = 0; q < 8; q++) or_damp_wiggles(im, jm, km, f[mc[q]], cm);
    }
    if (upto <= OR_INIT_MOIST) goto done;

    turbulence_init_fields(im, jm, km, p, g.height, f, f2);         /* :612-624 */
    or_turbulence_run(im, jm, km, p, cm, f, f2);                    /* init's compute_sources, clamp_nue */
    or_turbulence_run(im, jm, km, p, cm, f, f2);                    /* run() */
    {
        const int tb[] = { OF_TKE, OF_DIS, OF_NUE, OF_PROD, OF_TKE_SOURCE, OF_DIS_SOURCE };
        for (int q = 0; q < 6; q++) or_damp_wiggles(im, jm, km, f[tb[q]], cm);
    }
    if (upto <= OR_INIT_TURBULENCE) goto done;

    precipitation_sum(im, jm, km, f);                               /* :627 */
    co2_atmosphere(im, jm, km, p, c, f);                            /* :631 */
    {
        double out[2];
        or_co2_column(im, jm, km, p, f, f2, out);                   /* :632 (co2_total) */
    }
    or_densities(im, jm, km, p, cm, 0, f, f2, prof);                /* :634 */
    forces(im, jm, km, p, &g, f, NULL);                             /* :635 */
    or_water_vapour_evaporation(im, jm, km, p, f, f2);              /* :637 */
    or_latent_sensible_heat(im, jm, km, p, cm, f);                  /* :638 */
    if (upto <= OR_INIT_DIAGNOSE) goto done;

    or_boundary_conditions_ex(im, jm, km, p, f, f2, 0);             /* :651-653, no wall values */
    if (upto <= OR_INIT_BC) goto done;

    or_project_initial_velocity(im, jm, km, p, cm, 200, 0, f, prof);   /* :665 */
    if (upto <= OR_INIT_PROJECT) goto done;

    or_store_n_level(im, jm, km, f);                                /* :667 */
    memcpy(f[OF_T_EQ], f[OF_T], sizeof(double) * n);                /* run_3D_loop :750-753 */

done:
    free(trop);
    or_geom_free(&g);
    return rc;
}
