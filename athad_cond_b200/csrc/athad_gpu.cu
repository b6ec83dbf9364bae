// athad_gpu.cu - the C ABI of include/athad_gpu.h: context lifetime, device-resident
// state, host<->device transfer and the hot-path entry points.
//
// All device memory of a context is one allocation made at creation (fields, RK4 stage
// buffers, the Poisson source, geometry tables, counters), so the hot path allocates
// nothing and a context's HBM footprint is known before it is created.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <new>

#include "ctx.cuh"
#include "thermo.cuh"

extern "C" {

int32_t athad_abi_version(void) { return ATHAD_ABI_VERSION; }
size_t athad_params_size(void) { return sizeof(athad_params); }

// cli/config_cond.xml values; composition resolved as AtmMixture::resolve (MixtureAtm.h:82-109)
void athad_default_params(athad_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->struct_size = sizeof(athad_params);
    p->turb_model = ATHAD_TURB_K_OMEGA_SST;
    p->wall_mode = ATHAD_WALL_MIRROR;
    p->poisson_metric_fix = 1;
    p->convection_perturbation = 1;
    p->convection_mode = 1;
    p->iter_prec = 3;
    p->category_ice_scheme = 2;
    p->metric_r0 = -1.0;                 // derive r_Earth*1e3/metricShellLength()
    p->re_turb = 0.4 * 0.1 / 1.5e-5;     // TurbulenceAtm.h:26-35
    p->r_air = 40.8; p->g = 9.8066; p->u_0 = 8.0; p->cp_l = 1349.0; p->t_0 = 273.15;
    p->c_0 = 0.3464; p->L_atm = 6287.5; p->zeta = 3.0; p->omega = 0.000317; p->lamda = 0.0262;
    p->lv = 2520000.0; p->ls = 2830000.0; p->pr_turb = 0.9; p->sc_WaterVapour = 0.61;
    p->sc_CO2 = 0.96; p->r_Earth = 6370.001; p->p_0 = 60000.0; p->t_00 = 236.15;
    p->t_max_phys = 2000.0; p->cloud_cap = 0.05; p->t_skin = 254.0; p->c_h2o_dry_top = 0.00423;
    p->co2_0 = 0.6233; p->s_0 = 274515.75; p->R_Air = 296.8; p->R_WaterVapour = 461.5;
    p->abl_height = 10000.0;
    p->t_000 = 253.15;
    p->sigma = 5.67028e-08; p->kappa_H2O = 0.01; p->kappa_CO2 = 0.001; p->kappa_bg = 1e-06;
    p->geothermal_flux = 150.0; p->albedo_surface = 0.08; p->albedo_cloud = 0.5;
    p->rad_equator_short = 298.0; p->rad_pole_short = 0.0;
    p->coeff_Dalton = 0.7;
    p->r_0_water = 997.0;
    const double x[8] = {0.5578, 0.4109, 0.0313, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double m_H2O = x[0] * thermo::M_H2O, m_CO2 = x[1] * thermo::M_CO2;
    const double m_bg = x[2] * 0.028014 + x[3] * 0.016043 + x[4] * 0.017031
                      + x[5] * 0.002016 + x[6] * 0.028010 + x[7] * 0.064066;
    const double M_mean = m_H2O + m_CO2 + m_bg;
    p->R_mix = thermo::R_STAR / M_mean;
    const double x_bg = x[2] + x[3] + x[4] + x[5] + x[6] + x[7];
    p->M_bg = (x_bg > 0.0) ? (m_bg / x_bg) : 0.028014;
    p->R_bg = thermo::R_STAR / p->M_bg;
}

size_t athad_footprint_bytes(const athad_grid* grid)
{
    if (!grid || grid->im < 4 || grid->jm < 5 || grid->km < 5) return 0;
    return make_layout(*grid, ATHAD_PRECISION_FP64).bytes;
}

size_t athad_footprint_bytes_params(const athad_grid* grid, const athad_params* params)
{
    if (!grid || !params || grid->im < 4 || grid->jm < 5 || grid->km < 5) return 0;
    if (params->precision != ATHAD_PRECISION_FP64 && params->precision != ATHAD_PRECISION_MIXED) return 0;
    return make_layout(*grid, params->precision).bytes;
}

const char* athad_last_error(const athad_ctx* ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

athad_status athad_create(const athad_grid* grid, const athad_params* params, athad_ctx** out)
{
    if (!out) return ATHAD_ERR_INVALID;
    *out = nullptr;
    if (!grid || !params) return ATHAD_ERR_INVALID;
    if (params->struct_size != sizeof(athad_params)) return ATHAD_ERR_INVALID;
    // im <= 1024 (per-level profiles), jm <= 6144 (the level mean stages a level's row sums
    // in shared memory)
    if (grid->im < 4 || grid->jm < 5 || grid->km < 5 || grid->im > 1024 || grid->jm > 6144)
        return ATHAD_ERR_INVALID;
    if (params->turb_model < ATHAD_TURB_K_EPSILON || params->turb_model > ATHAD_TURB_K_OMEGA_SST)
        return ATHAD_ERR_UNSUPPORTED;
    if (params->precision != ATHAD_PRECISION_FP64 && params->precision != ATHAD_PRECISION_MIXED)
        return ATHAD_ERR_UNSUPPORTED;
    if (params->category_ice_scheme < -1 || params->category_ice_scheme > 3)
        return ATHAD_ERR_UNSUPPORTED;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return ATHAD_ERR_NO_DEVICE; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) { cudaGetLastError(); return ATHAD_ERR_NO_DEVICE; }
    if (prop.major != 10) return ATHAD_ERR_NO_DEVICE;   // built for sm_100a only

    athad_ctx* c = new (std::nothrow) athad_ctx();
    if (!c) return ATHAD_ERR_OOM;
    c->grid = *grid;
    c->p = *params;
    c->L = make_layout(*grid, params->precision);
    const Layout& L = c->L;
    const int im = grid->im, jm = grid->jm, km = grid->km;

    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c; return ATHAD_ERR_CUDA;
    }
    if (cudaEventCreate(&c->ev_step0) != cudaSuccess || cudaEventCreate(&c->ev_step1) != cudaSuccess) {
        cudaGetLastError();
        if (c->ev_step0) cudaEventDestroy(c->ev_step0);
        cudaStreamDestroy(c->own_stream);
        delete c;
        return ATHAD_ERR_CUDA;
    }
    c->stream = c->own_stream;
    if (cudaMalloc((void**)&c->slab, L.bytes) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamDestroy(c->own_stream);
        cudaEventDestroy(c->ev_step0); cudaEventDestroy(c->ev_step1);
        delete c;
        return ATHAD_ERR_OOM;
    }
    // carve the slab
    char* q = c->slab;
    auto take = [&](size_t bytes) { char* r = q; q += round_up(bytes, 256); return r; };
    for (int f = 0; f < ATHAD_NFIELDS; f++) c->field[f] = (double*)take(L.field_elems * sizeof(double));
    for (int n = 0; n < kNY; n++) c->stA[n] = (double*)take(L.field_elems * sizeof(double));
    for (int n = 0; n < kNY; n++) c->stB[n] = (double*)take(L.field_elems * sizeof(double));
    for (int n = 0; n < kNY; n++) c->stK[n] = (double*)take(L.field_elems * sizeof(double));
    c->src = (double*)take(L.field_elems * sizeof(double));
    c->upload_stage = (double*)take(L.field_elems * sizeof(double));
    for (int f = 0; f < ATHAD_NFIELDS2D; f++) c->f2d[f] = (double*)take(L.f2d_elems * sizeof(double));
    for (int f = 0; f < ATHAD_NPROFILES; f++) c->prof[f] = (double*)take(round_up((size_t)im, 64) * sizeof(double));
    c->geo = (GeoIJ*)take((size_t)im * jm * sizeof(GeoIJ));
    c->poi = (PoiIJ*)take((size_t)im * jm * sizeof(PoiIJ));
    const size_t nmax = round_up((size_t)(im > jm ? im : jm), 64) * sizeof(double);
    c->sin_w = (double*)take(nmax);
    c->height = (double*)take(nmax);
    c->step_f = (double*)take(nmax);
    c->coslat = (double*)take(nmax);
    c->step_mc = (double*)take(nmax);
    c->cose = (double*)take(nmax);
    c->res_sin = (double*)take(nmax);
    c->rad_d = (double*)take(nmax);
    c->i_trop = (int*)take((size_t)jm * sizeof(int));
    c->row_sum = (double*)take(round_up((size_t)im * jm, 64) * sizeof(double));
    c->row_cnt = (double*)take(round_up((size_t)im * jm, 64) * sizeof(double));
    c->counters = (unsigned long long*)take(256);
    c->polar_passes = (int*)take((size_t)jm * sizeof(int));
    c->turb_lev = (TurbLevel*)take((size_t)im * sizeof(TurbLevel));
    if (params->precision == ATHAD_PRECISION_MIXED) {
        const size_t fb = L.field_elems * sizeof(float);
        for (int n = 0; n < kNY; n++) c->mA[n] = (float*)take(fb);
        for (int n = 0; n < kNY; n++) c->mB[n] = (float*)take(fb);
        for (int n = 0; n < kNY; n++) c->mK[n] = (float*)take(fb);
        for (int n = 0; n < kNY; n++) c->mYn[n] = (float*)take(fb);
        for (int f = 0; f < ATHAD_MF_COUNT; f++) c->mF[f] = (float*)take(fb);
        c->geof = (GeoF*)take((size_t)im * jm * sizeof(GeoF));
    }
    if ((size_t)(q - c->slab) > L.bytes) {
        cudaFree(c->slab); cudaStreamDestroy(c->own_stream);
        cudaEventDestroy(c->ev_step0); cudaEventDestroy(c->ev_step1); delete c;
        return ATHAD_ERR_INVALID;
    }
    // Every field starts at zero (the reference's Arrays are zero/one-initialised by
    // resetArrays; the caller uploads the state it wants).
    if (cudaMemsetAsync(c->slab, 0, L.bytes, c->stream) != cudaSuccess) {
        cudaFree(c->slab); cudaStreamDestroy(c->own_stream);
        cudaEventDestroy(c->ev_step0); cudaEventDestroy(c->ev_step1); delete c;
        return ATHAD_ERR_CUDA;
    }

    // ---- geometry, built on the host exactly as the reference builds it ----
    const double pi180 = 180.0 / M_PI;                         // cAtmosphereModel.cpp:44
    c->dr = 1.0 / (double)(im - 1);                            // :57
    c->dthe = (180.0 / (double)(jm - 1)) / pi180;              // :46/:59 generalised
    c->dphi = (360.0 / (double)(km - 1)) / pi180;              // :47/:60 generalised
    std::vector<double> rad(im), the(jm);
    rad[0] = 1.0;                                              // Array_1D::Coordinates running sum
    for (int i = 1; i < im; i++) rad[i] = rad[i - 1] + c->dr;
    the[0] = 0.0;
    for (int j = 1; j < jm; j++) the[j] = the[j - 1] + c->dthe;
    c->rad = rad;
    std::vector<double> sin_w(jm), sin_f(jm), cos_t(jm), coslat(jm);
    for (int j = 0; j < jm; j++) {   // mirror-exact tables
        const int jj = (j < jm - 1 - j) ? j : jm - 1 - j;
        sin_w[j] = std::sin(the[jj]);
        if (j < jm - 1 - j) cos_t[j] = std::cos(the[j]);
        else if (j > jm - 1 - j) cos_t[j] = -std::cos(the[jm - 1 - j]);
        else cos_t[j] = 0.0;
        sin_f[j] = sin_w[j] < 0.55 ? 0.55 : sin_w[j];
        coslat[j] = std::cos((jj / (double)(jm - 1) - 0.5) * M_PI);   // ThermoAtm.h:1636
    }
    const double span = rad[im - 1] - rad[0];
    c->shell_len = (span > 0.0) ? (std::exp(params->zeta * span) - 1.0) * params->L_atm / span
                                : params->L_atm;                     // cAtmosphereModel.h:465-470
    c->metric_r0 = (params->metric_r0 < 0.0)
        ? ((c->shell_len > 0.0) ? params->r_Earth * 1.0e3 / c->shell_len : 0.0)
        : params->metric_r0;                                          // cAtmosphereModel.cpp:382-399
    auto rmet_of = [&](double rm) { return (c->metric_r0 > 0.0) ? (c->metric_r0 + (rm - rad[0])) : rm; };
    std::vector<double> height(im), step(im);
    const float hL = (float)params->L_atm;
    for (int i = 0; i < im; i++)
        height[i] = (double)(float)((std::exp(params->zeta * (rad[i] - rad[0])) - 1) * (double)hL);
    c->layer_height1 = height[1];
    c->height_h = height;
    for (int i = 0; i < im; i++) {   // SaturationAdjustment::computeSteps: float difference
        const float h1 = (i + 1 <= im - 1) ? (float)height[i + 1] : -1.0f;
        const float h0 = (float)height[i];
        step[i] = (double)(float)(h1 - h0);
    }
    // MoistConvection::precompute (MoistConvection.h:300-309): double differences of the
    // layer heights; and cos(theta_equator - theta_j) of entrainmentGradients (:239) with
    // the equator row (jm-1)/2, mirror-symmetric
    std::vector<double> step_mc(im), cose(jm);
    for (int i = 0; i < im - 1; i++) step_mc[i] = height[i + 1] - height[i];
    step_mc[im - 1] = step_mc[im - 2];
    for (int j = 0; j < jm; j++) {
        const int jj = (j < jm - 1 - j) ? j : jm - 1 - j;
        cose[j] = std::cos(the[(jm - 1) / 2] - the[jj]);
    }
    // AtomUtils::polar_zonal_filter's passes per row (lib/Utils.cpp:559-571), from the
    // mirror-exact sin table: clamp(lround(3 (sin30/sin_j)^2 - 3), 0, 12) poleward of 30 deg
    std::vector<int> polar(jm, 0);
    for (int j = 0; j < jm; j++) {
        const double sin_ref = std::cos(30.0 * (M_PI / 180.0));
        const double sin_j = (sin_w[j] < 1.0e-6) ? 1.0e-6 : sin_w[j];
        if (sin_j >= sin_ref) continue;
        const double ratio = sin_ref / sin_j;
        // (int) of the long, as lib/Utils.cpp:566 converts it: on the pole rows (sin
        // guarded to 1e-6) the count does not fit an int and wraps before the clamp
        int pp = (int)std::lround(3.0 * (ratio * ratio - 1.0));
        polar[j] = (pp < 0) ? 0 : (pp > 12) ? 12 : pp;
    }
    // TurbulenceAtm's per-level constants; clamp_nue's taper (TurbulenceAtm.h:271-295): the
    // eddy viscosity fades to zero over the grid layer that straddles abl_height
    std::vector<TurbLevel> tlev(im);
    {
        int i_abl = 0;
        while (i_abl < im - 1 && height[i_abl] <= params->abl_height) i_abl++;
        const double taper_dz = std::max(1.0, height[std::min(i_abl, im - 1)] - height[std::max(i_abl - 1, 0)]);
        for (int i = 0; i < im; i++) {
            TurbLevel& T = tlev[i];
            T.rm = rad[i];
            T.exp_rm = 1.0 / (rad[i] + 1.0);
            T.rmet = rmet_of(rad[i]);
            T.height = height[i];
            const double z_agl = height[i] - height[0];
            T.nue_fac = std::clamp((params->abl_height + taper_dz - z_agl) / taper_dz, 0.0, 1.0);
        }
    }
    std::vector<GeoIJ> geo((size_t)im * jm);
    std::vector<PoiIJ> poi((size_t)im * jm);
    const double inv_dr2 = 1.0 / (c->dr * c->dr), inv_dthe2 = 1.0 / (c->dthe * c->dthe),
                 inv_dphi2 = 1.0 / (c->dphi * c->dphi);
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            GeoIJ& G = geo[(size_t)i * jm + j];
            const double rm = rad[i];
            G.exp_rm = 1.0 / (rm + 1.0);
            G.exp_2_rm = G.exp_rm * G.exp_rm;
            G.sinthe = sin_f[j];
            G.sinthe2 = G.sinthe * G.sinthe;
            G.costhe = cos_t[j];
            const double rmet = rmet_of(rm);
            const double rmet2 = rmet * rmet;
            G.inv_rm = 1.0 / rmet;
            G.inv_rm2 = 1.0 / rmet2;
            G.inv_rmsinthe = 1.0 / (rmet * G.sinthe);
            G.inv_rm2sinthe = G.inv_rm2 / G.sinthe;
            G.inv_rm2sinthe2 = G.inv_rm2 / G.sinthe2;
            G.costhe_inv_rm2sinthe = G.costhe * G.inv_rm2sinthe;
            G.two_over_rm_exp = 2.0 * G.inv_rm * G.exp_rm;
            G.v_metric = (1.0 + G.costhe * G.costhe / G.sinthe2) * G.inv_rm2;
            G.cos4lat = G.sinthe2 * G.sinthe2;
            PoiIJ& P = poi[(size_t)i * jm + j];          // PressureSolverAtm.h:236-269
            const double m_the = params->poisson_metric_fix ? G.inv_rm2 : G.inv_rm;
            const double m_phi = params->poisson_metric_fix ? G.inv_rm2sinthe2 : G.inv_rmsinthe;
            P.denom = 2.0 * G.exp_2_rm * inv_dr2 + 2.0 * m_the * inv_dthe2 + 2.0 * m_phi * inv_dphi2;
            P.inv_denom = 1.0 / P.denom;
            P.num1 = G.exp_2_rm * inv_dr2;
            P.num2 = m_the * inv_dthe2;
            P.num3 = m_phi * inv_dphi2;
            P.exp_rm = G.exp_rm; P.exp_2_rm = G.exp_2_rm; P.inv_rm = G.inv_rm;
            P.inv_rmsinthe = G.inv_rmsinthe; P.sinthe = G.sinthe; P.costhe = G.costhe;
        }
    athad_status s = ATHAD_OK;
    s = cuda_check(c, cudaMemcpyAsync(c->geo, geo.data(), geo.size() * sizeof(GeoIJ), cudaMemcpyHostToDevice, c->stream), "geo");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->poi, poi.data(), poi.size() * sizeof(PoiIJ), cudaMemcpyHostToDevice, c->stream), "poi");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->sin_w, sin_w.data(), jm * sizeof(double), cudaMemcpyHostToDevice, c->stream), "sin_w");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->height, height.data(), im * sizeof(double), cudaMemcpyHostToDevice, c->stream), "height");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->step_f, step.data(), im * sizeof(double), cudaMemcpyHostToDevice, c->stream), "step");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->coslat, coslat.data(), jm * sizeof(double), cudaMemcpyHostToDevice, c->stream), "coslat");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->step_mc, step_mc.data(), im * sizeof(double), cudaMemcpyHostToDevice, c->stream), "step_mc");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->cose, cose.data(), jm * sizeof(double), cudaMemcpyHostToDevice, c->stream), "cose");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->polar_passes, polar.data(), jm * sizeof(int), cudaMemcpyHostToDevice, c->stream), "polar passes");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->turb_lev, tlev.data(), im * sizeof(TurbLevel), cudaMemcpyHostToDevice, c->stream), "turbulence levels");
    // findResiduumAtm's sin(theta) of the running-sum theta, floored at 0.55 (UtilsAtm.h:96)
    std::vector<double> res_sin(jm);
    for (int j = 0; j < jm; j++) res_sin[j] = std::max(0.55, std::sin(the[j]));
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->res_sin, res_sin.data(), jm * sizeof(double), cudaMemcpyHostToDevice, c->stream), "res_sin");
    if (s == ATHAD_OK) s = cuda_check(c, cudaMemcpyAsync(c->rad_d, rad.data(), im * sizeof(double), cudaMemcpyHostToDevice, c->stream), "rad");
    std::vector<GeoF> geof;
    if (s == ATHAD_OK && c->geof) {   // FP32 factors rounded from the FP64 ones (mirror-exact)
        geof.resize(geo.size());
        for (size_t q2 = 0; q2 < geo.size(); q2++) {
            const GeoIJ& G = geo[q2];
            GeoF& F = geof[q2];
            F.exp_rm = (float)G.exp_rm; F.exp_2_rm = (float)G.exp_2_rm; F.sinthe = (float)G.sinthe;
            F.costhe = (float)G.costhe; F.inv_rm = (float)G.inv_rm; F.inv_rm2 = (float)G.inv_rm2;
            F.inv_rmsinthe = (float)G.inv_rmsinthe; F.inv_rm2sinthe = (float)G.inv_rm2sinthe;
            F.inv_rm2sinthe2 = (float)G.inv_rm2sinthe2; F.costhe_inv_rm2sinthe = (float)G.costhe_inv_rm2sinthe;
            F.two_over_rm_exp = (float)G.two_over_rm_exp; F.v_metric = (float)G.v_metric;
            F.cos4lat = (float)G.cos4lat; F.pad = 0.0f;
        }
        s = cuda_check(c, cudaMemcpyAsync(c->geof, geof.data(), geof.size() * sizeof(GeoF), cudaMemcpyHostToDevice, c->stream), "geof");
    }
    if (s == ATHAD_OK) s = cuda_check(c, cudaStreamSynchronize(c->stream), "create sync");
    if (s != ATHAD_OK) {
        cudaFree(c->slab); cudaStreamDestroy(c->own_stream);
        cudaEventDestroy(c->ev_step0); cudaEventDestroy(c->ev_step1); delete c;
        return s;
    }
    *out = c;
    return ATHAD_OK;
}

athad_status athad_destroy(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    cudaStreamSynchronize(ctx->stream);
    if (ctx->ckpt_stream) {
        cudaStreamSynchronize(ctx->ckpt_stream);
        cudaStreamDestroy(ctx->ckpt_stream);
        cudaEventDestroy(ctx->ckpt_ready);
        cudaEventDestroy(ctx->ckpt_done);
        cudaFree(ctx->ckpt_buf);
    }
    mg_free(ctx->mg);
    cudaFree(ctx->slab);
    cudaStreamDestroy(ctx->own_stream);
    cudaEventDestroy(ctx->ev_step0);
    cudaEventDestroy(ctx->ev_step1);
    delete ctx;
    return ATHAD_OK;
}

athad_status athad_set_stream(athad_ctx* ctx, void* s)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    ctx->stream = s ? (cudaStream_t)s : ctx->own_stream;
    return ATHAD_OK;
}

athad_status athad_synchronize(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
}

// ---- transfer ---------------------------------------------------------------------------

athad_status athad_upload(athad_ctx* ctx, athad_field f, const double* host, size_t n)
{
    if (!ctx || !host || (int)f < 0 || (int)f >= ATHAD_NFIELDS) return fail(ctx, ATHAD_ERR_INVALID, "upload: bad argument");
    const Dims& d = ctx->L.d;
    if (n != (size_t)d.im * d.jm * d.km) return fail(ctx, ATHAD_ERR_INVALID, "upload: size mismatch");
    // One contiguous copy into the packed staging field, then a device re-pitch: a
    // host-to-device copy of short pitched rows runs at well under half the link's speed.
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(ctx->upload_stage, host, n * sizeof(double),
                                                     cudaMemcpyHostToDevice, ctx->stream), "upload");
    if (s != ATHAD_OK) return s;
    launch_repitch(d, ctx->upload_stage, ctx->field[f], ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "upload repitch");
    return ATHAD_OK;
}

athad_status athad_upload_device(athad_ctx* ctx, athad_field f, const double* device_src, size_t n)
{
    if (!ctx || !device_src || (int)f < 0 || (int)f >= ATHAD_NFIELDS)
        return fail(ctx, ATHAD_ERR_INVALID, "upload_device: bad argument");
    const Dims& d = ctx->L.d;
    if (n != (size_t)d.im * d.jm * d.km) return fail(ctx, ATHAD_ERR_INVALID, "upload_device: size mismatch");
    launch_repitch(d, device_src, ctx->field[f], ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "upload_device repitch");
    return ATHAD_OK;
}

athad_status athad_download(athad_ctx* ctx, athad_field f, double* host, size_t n)
{
    if (!ctx || !host || (int)f < 0 || (int)f >= ATHAD_NFIELDS) return fail(ctx, ATHAD_ERR_INVALID, "download: bad argument");
    const Dims& d = ctx->L.d;
    if (n != (size_t)d.im * d.jm * d.km) return fail(ctx, ATHAD_ERR_INVALID, "download: size mismatch");
    athad_status s = cuda_check(ctx, cudaMemcpy2DAsync(host, d.km * sizeof(double), ctx->field[f], d.pitch * sizeof(double),
                                                       d.km * sizeof(double), (size_t)d.im * d.jm, cudaMemcpyDeviceToHost,
                                                       ctx->stream), "download");
    if (s != ATHAD_OK) return s;
    return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "download sync");
}

athad_status athad_upload_2d(athad_ctx* ctx, athad_field2d f, const double* host, size_t n)
{
    if (!ctx || !host || (int)f < 0 || (int)f >= ATHAD_NFIELDS2D) return fail(ctx, ATHAD_ERR_INVALID, "upload_2d: bad argument");
    const Dims& d = ctx->L.d;
    if (n != (size_t)d.jm * d.km) return fail(ctx, ATHAD_ERR_INVALID, "upload_2d: size mismatch");
    return cuda_check(ctx, cudaMemcpy2DAsync(ctx->f2d[f], d.pitch * sizeof(double), host, d.km * sizeof(double),
                                             d.km * sizeof(double), (size_t)d.jm, cudaMemcpyHostToDevice, ctx->stream),
                      "upload_2d");
}

athad_status athad_download_2d(athad_ctx* ctx, athad_field2d f, double* host, size_t n)
{
    if (!ctx || !host || (int)f < 0 || (int)f >= ATHAD_NFIELDS2D) return fail(ctx, ATHAD_ERR_INVALID, "download_2d: bad argument");
    const Dims& d = ctx->L.d;
    if (n != (size_t)d.jm * d.km) return fail(ctx, ATHAD_ERR_INVALID, "download_2d: size mismatch");
    athad_status s = cuda_check(ctx, cudaMemcpy2DAsync(host, d.km * sizeof(double), ctx->f2d[f], d.pitch * sizeof(double),
                                                       d.km * sizeof(double), (size_t)d.jm, cudaMemcpyDeviceToHost,
                                                       ctx->stream), "download_2d");
    if (s != ATHAD_OK) return s;
    return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "download_2d sync");
}

athad_status athad_upload_profile(athad_ctx* ctx, athad_profile f, const double* host, size_t n)
{
    if (!ctx || !host || (int)f < 0 || (int)f >= ATHAD_NPROFILES) return fail(ctx, ATHAD_ERR_INVALID, "upload_profile: bad argument");
    if (n != (size_t)ctx->grid.im) return fail(ctx, ATHAD_ERR_INVALID, "upload_profile: size mismatch");
    if (f == ATHAD_PROF_T_REF_LEVEL) ctx->level_mean_valid = true;
    return cuda_check(ctx, cudaMemcpyAsync(ctx->prof[f], host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream),
                      "upload_profile");
}

athad_status athad_download_profile(athad_ctx* ctx, athad_profile f, double* host, size_t n)
{
    if (!ctx || !host || (int)f < 0 || (int)f >= ATHAD_NPROFILES) return fail(ctx, ATHAD_ERR_INVALID, "download_profile: bad argument");
    if (n != (size_t)ctx->grid.im) return fail(ctx, ATHAD_ERR_INVALID, "download_profile: size mismatch");
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(host, ctx->prof[f], n * sizeof(double), cudaMemcpyDeviceToHost,
                                                     ctx->stream), "download_profile");
    if (s != ATHAD_OK) return s;
    return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "download_profile sync");
}

athad_status athad_download_profile_async(athad_ctx* ctx, athad_profile f, double* host, size_t n)
{
    if (!ctx || !host || (int)f < 0 || (int)f >= ATHAD_NPROFILES)
        return fail(ctx, ATHAD_ERR_INVALID, "download_profile_async: bad argument");
    if (n != (size_t)ctx->grid.im) return fail(ctx, ATHAD_ERR_INVALID, "download_profile_async: size mismatch");
    return cuda_check(ctx, cudaMemcpyAsync(host, ctx->prof[f], n * sizeof(double), cudaMemcpyDeviceToHost,
                                           ctx->stream), "download_profile_async");
}

athad_status athad_field_device_ptr(athad_ctx* ctx, athad_field f, double** ptr, size_t* pitch)
{
    if (!ctx || !ptr || (int)f < 0 || (int)f >= ATHAD_NFIELDS) return fail(ctx, ATHAD_ERR_INVALID, "field_device_ptr: bad argument");
    *ptr = ctx->field[f];
    if (pitch) *pitch = (size_t)ctx->L.d.pitch;
    return ATHAD_OK;
}

athad_status athad_fill(athad_ctx* ctx, athad_field f, double value)
{
    if (!ctx || (int)f < 0 || (int)f >= ATHAD_NFIELDS) return fail(ctx, ATHAD_ERR_INVALID, "fill: bad argument");
    launch_fill(ctx->L.d, ctx->field[f], value, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "fill");
    return ATHAD_OK;
}

// ---- hot path -----------------------------------------------------------------------------

// P_rain, P_snow -> P_rainn, P_snown (UtilsAtm.h:41-42): consecutive fields, one copy
static athad_status store_precip_n_level(athad_ctx* ctx, cudaStream_t st)
{
    const size_t bytes = ctx->L.field_elems * sizeof(double);
    return cuda_check(ctx, cudaMemcpyAsync(ctx->field[ATHAD_P_RAINN], ctx->field[ATHAD_P_RAIN], 2 * bytes,
                                           cudaMemcpyDeviceToDevice, st), "store_n_level precipitation");
}

athad_status athad_store_n_level(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    // the fields are consecutive in the slab: t..dis -> tn..disn is one copy
    const size_t bytes = ctx->L.field_elems * sizeof(double);
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(ctx->field[ATHAD_TN], ctx->field[ATHAD_T], kNY * bytes,
                                                     cudaMemcpyDeviceToDevice, ctx->stream), "store_n_level");
    if (s != ATHAD_OK) return s;
    return store_precip_n_level(ctx, ctx->stream);
}

athad_status athad_level_mean(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    athad_status s = cuda_check(ctx, cudaMemsetAsync(ctx->counters + kNonfiniteSlot, 0, sizeof(unsigned long long),
                                                     ctx->stream), "level_mean counter");
    if (s != ATHAD_OK) return s;
    launch_level_mean(ctx->L.d, ctx->field[ATHAD_T], ctx->sin_w, ctx->prof[ATHAD_PROF_T_REF_LEVEL], ctx->row_sum,
                      ctx->stream, ctx->counters + kNonfiniteSlot);
    ATHAD_CHECK_LAUNCH(ctx, "level_mean");
    ctx->level_mean_valid = true;
    return ATHAD_OK;
}

static athad_status rk4_step_mixed(athad_ctx* ctx, const athad_step_scalars* s);

static athad_status rk4_step_fp64(athad_ctx* ctx, const athad_step_scalars* s);

// the step between two events on the context's stream: athad_get_report's last_kernel_ms
athad_status athad_rk4_step(athad_ctx* ctx, const athad_step_scalars* s)
{
    if (!ctx || !s) return fail(ctx, ATHAD_ERR_INVALID, "rk4_step: bad argument");
    athad_status st = cuda_check(ctx, cudaEventRecord(ctx->ev_step0, ctx->stream), "rk4_step event");
    if (st != ATHAD_OK) return st;
    st = (ctx->p.precision == ATHAD_PRECISION_MIXED) ? rk4_step_mixed(ctx, s) : rk4_step_fp64(ctx, s);
    if (st != ATHAD_OK) return st;
    if (s->write_diagnostics & 3) {
        // the right-hand side's diagnostic outputs from the last stage's input state (the
        // stage buffer A holds it after the step)
        const athad_params& p = ctx->p;
        RhsDiagArgs g;
        std::memset(&g, 0, sizeof g);
        g.d = ctx->L.d;
        g.geo = ctx->geo;
        g.t_ref = ctx->prof[ATHAD_PROF_T_REF_LEVEL];
        g.p_dyn = ctx->field[ATHAD_P_DYN]; g.nue = ctx->field[ATHAD_NUE];
        g.MC_v = ctx->field[ATHAD_MC_V]; g.MC_w = ctx->field[ATHAD_MC_W];
        const int outs[17] = {ATHAD_CORIOLIS_FORCE, ATHAD_BUOYANCY_FORCE, ATHAD_PRESSURE_GRADIENT_FORCE,
                              ATHAD_Q_LATENT, ATHAD_Q_SENSIBLE,
                              ATHAD_VBUD_PGF, ATHAD_VBUD_COR, ATHAD_VBUD_ADVV, ATHAD_VBUD_ADVH, ATHAD_VBUD_DIFF,
                              ATHAD_VBUD_OTHER, ATHAD_WBUD_PGF, ATHAD_WBUD_COR, ATHAD_WBUD_ADVV, ATHAD_WBUD_ADVH,
                              ATHAD_WBUD_DIFF, ATHAD_WBUD_OTHER};
        for (int q = 0; q < 17; q++) g.out[q] = ctx->field[outs[q]];
        g.inv_2dr = 1.0 / (2.0 * ctx->dr); g.inv_2dthe = 1.0 / (2.0 * ctx->dthe); g.inv_2dphi = 1.0 / (2.0 * ctx->dphi);
        g.inv_dr2 = 1.0 / (ctx->dr * ctx->dr); g.inv_dthe2 = 1.0 / (ctx->dthe * ctx->dthe);
        g.inv_dphi2 = 1.0 / (ctx->dphi * ctx->dphi);
        g.coeff_Coriolis = p.r_air * p.u_0 * p.omega;                 // RHS_Atm_Turb.cpp:365-376
        g.coeff_buoy = p.r_air * p.g;
        g.coeff_u_p = 0.5 * p.r_air * p.u_0 * p.u_0 / p.L_atm;
        g.coeff_L = p.r_air * p.c_0 * p.lv * p.u_0 / p.L_atm;         // :474-475
        g.coeff_S = p.lamda * p.t_0 / p.L_atm;
        g.t_0 = p.t_0;
        g.inv_re = 1.0 / p.re_turb;
        g.diffusion_ramp = s->diffusion_ramp;
        g.drag_pref = 1.0 / 86400.0 * p.L_atm / p.u_0 * s->dt;
        g.force_nd = p.omega * ctx->shell_len / p.u_0;
        g.coeff_MC_vel = p.L_atm / (p.u_0 * p.u_0);
        g.nontrad = p.coriolis_nontrad;
        g.flags = s->write_diagnostics & 3;
        for (int n = 0; n < kNY; n++) {
            if (ctx->p.precision == ATHAD_PRECISION_MIXED) g.Y32[n] = ctx->mA[n];
            else g.Y64[n] = ctx->stA[n];
        }
        launch_rhs_diagnostics(g, ctx->stream);
        ATHAD_CHECK_LAUNCH(ctx, "rhs diagnostics");
    }
    st = cuda_check(ctx, cudaEventRecord(ctx->ev_step1, ctx->stream), "rk4_step event");
    if (st == ATHAD_OK) ctx->step_timed = true;
    return st;
}

static athad_status rk4_step_fp64(athad_ctx* ctx, const athad_step_scalars* s)
{
    const athad_params& p = ctx->p;
    athad_status st = athad_level_mean(ctx);
    if (st != ATHAD_OK) return st;
    RK4Args a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    a.geo = ctx->geo;
    a.t_ref = ctx->prof[ATHAD_PROF_T_REF_LEVEL];
    a.dlnrho = ctx->prof[ATHAD_PROF_DLNRHO_DR];
    for (int n = 0; n < kNY; n++) a.Yn[n] = ctx->field[ATHAD_TN + n];
    for (int n = 0; n < kNY; n++) a.K[n] = ctx->stK[n];
    a.p_dyn = ctx->field[ATHAD_P_DYN]; a.nue = ctx->field[ATHAD_NUE];
    a.t_eq = ctx->field[ATHAD_T_EQ]; a.p_stat = ctx->field[ATHAD_P_STAT]; a.r_humid = ctx->field[ATHAD_R_HUMID];
    a.S_c = ctx->field[ATHAD_S_C]; a.S_r = ctx->field[ATHAD_S_R]; a.S_i = ctx->field[ATHAD_S_I];
    a.S_s = ctx->field[ATHAD_S_S]; a.S_g = ctx->field[ATHAD_S_G]; a.S_v = ctx->field[ATHAD_S_V];
    a.MC_t = ctx->field[ATHAD_MC_T]; a.MC_q = ctx->field[ATHAD_MC_Q];
    a.MC_v = ctx->field[ATHAD_MC_V]; a.MC_w = ctx->field[ATHAD_MC_W];
    a.aux_u = ctx->field[ATHAD_AUX_U]; a.aux_v = ctx->field[ATHAD_AUX_V]; a.aux_w = ctx->field[ATHAD_AUX_W];
    a.prod = ctx->field[ATHAD_PROD]; a.tke_source = ctx->field[ATHAD_TKE_SOURCE];
    a.dis_source = ctx->field[ATHAD_DIS_SOURCE];
    a.inv_2dr = 1.0 / (2.0 * ctx->dr); a.inv_2dthe = 1.0 / (2.0 * ctx->dthe); a.inv_2dphi = 1.0 / (2.0 * ctx->dphi);
    a.inv_dr2 = 1.0 / (ctx->dr * ctx->dr); a.inv_dthe2 = 1.0 / (ctx->dthe * ctx->dthe);
    a.inv_dphi2 = 1.0 / (ctx->dphi * ctx->dphi);
    a.dt = s->dt; a.half_dt = 0.5 * s->dt; a.dt_sixth = s->dt / 6.0;
    a.diffusion_ramp = s->diffusion_ramp; a.buoyancy_ramp = s->buoyancy_ramp;
    a.tke_max_nd = 1000.0 / (p.u_0 * p.u_0);                   // RungeKutta_Atm_Turb.cpp:67-68
    a.force_nd = p.omega * ctx->shell_len / p.u_0;              // RHS_Atm_Turb.cpp:445
    a.coeff_energy_p = p.u_0 * p.u_0 / (p.cp_l * p.t_0);       // RHS_Atm_Turb.cpp:366-372
    a.coeff_energy = 1.0 / (p.c_0 * p.cp_l * p.t_0);
    a.coeff_MC_vel = p.L_atm / (p.u_0 * p.u_0);
    a.coeff_MC_q = p.L_atm / (p.u_0 * p.c_0);
    a.coeff_MC_t = p.L_atm / (p.u_0 * p.t_0);
    a.lv = p.lv; a.ls = p.ls; a.g = p.g; a.u_0 = p.u_0; a.L_atm = p.L_atm; a.re_turb = p.re_turb;
    a.pr_turb = p.pr_turb; a.sc_WaterVapour = p.sc_WaterVapour; a.sc_CO2 = p.sc_CO2;
    a.inv_re = 1.0 / p.re_turb;
    a.nue_max = 1000.0 / (p.u_0 * p.L_atm);
    a.nue_air_nd = 1.5e-5 / (p.u_0 * p.L_atm);
    a.diff_prec_re_inv = 1.0 / (p.sc_WaterVapour * p.re_turb);
    a.diff_co2_re_inv = 1.0 / (p.sc_CO2 * p.re_turb);
    a.buoy_pref = s->buoyancy_ramp * 1.0 * p.g * s->dt / p.u_0;
    a.drag_pref = 1.0 / 86400.0 * p.L_atm / p.u_0 * s->dt;
    a.turb_model = p.turb_model; a.wall_mode = p.wall_mode; a.nontrad = p.coriolis_nontrad;
    a.curvature = p.metric_curvature; a.tracer_diff_flux = p.tracer_diff_flux;
    a.write_diag = s->write_diagnostics & 1;
    a.store_n = s->store_n_level ? 1 : 0;
    for (int n = 0; n < kNY; n++) a.Yn_store[n] = ctx->field[ATHAD_TN + n];
    for (int stage = 1; stage <= 4; stage++) {
        for (int n = 0; n < kNY; n++) {
            double* cur = ctx->field[ATHAD_T + n];
            a.Yin[n] = (stage == 1) ? cur : (stage == 3) ? ctx->stB[n] : ctx->stA[n];
            a.Yout[n] = (stage == 1 || stage == 3) ? ctx->stA[n] : (stage == 2) ? ctx->stB[n] : cur;
            a.Ybnd[n] = ctx->stB[n];
        }
        launch_rk4_stage(stage, a, ctx->stream);
        ATHAD_CHECK_LAUNCH(ctx, "rk4 stage");
    }
    return s->store_n_level ? store_precip_n_level(ctx, ctx->stream) : ATHAD_OK;
}

}  // extern "C"

// Arguments of the mixed-precision stage kernels for one context and step (the stage
// buffers are set per stage by the caller).
void athad::mixed_args(athad_ctx* ctx, const athad_step_scalars* s, RK4MArgs& a)
{
    const athad_params& p = ctx->p;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    a.geo = ctx->geof;
    a.t_ref = ctx->prof[ATHAD_PROF_T_REF_LEVEL];
    a.dlnrho = ctx->prof[ATHAD_PROF_DLNRHO_DR];
    for (int n = 0; n < kNY; n++) {
        a.Y[n] = ctx->field[ATHAD_T + n];
        a.Yn[n] = ctx->field[ATHAD_TN + n];
        a.Yn32[n] = ctx->mYn[n];
        a.K[n] = ctx->mK[n];
    }
    for (int f = 0; f < ATHAD_MF_COUNT; f++) a.F[f] = ctx->mF[f];
    double** F = ctx->field;
    a.p_dyn = F[ATHAD_P_DYN]; a.nue = F[ATHAD_NUE]; a.t_eq = F[ATHAD_T_EQ]; a.p_stat = F[ATHAD_P_STAT];
    a.r_humid = F[ATHAD_R_HUMID];
    a.S_c = F[ATHAD_S_C]; a.S_r = F[ATHAD_S_R]; a.S_i = F[ATHAD_S_I]; a.S_s = F[ATHAD_S_S];
    a.S_g = F[ATHAD_S_G]; a.S_v = F[ATHAD_S_V];
    a.MC_t = F[ATHAD_MC_T]; a.MC_q = F[ATHAD_MC_Q]; a.MC_v = F[ATHAD_MC_V]; a.MC_w = F[ATHAD_MC_W];
    a.aux_u = F[ATHAD_AUX_U]; a.aux_v = F[ATHAD_AUX_V]; a.aux_w = F[ATHAD_AUX_W];
    a.prod = F[ATHAD_PROD]; a.tke_source = F[ATHAD_TKE_SOURCE]; a.dis_source = F[ATHAD_DIS_SOURCE];
    const double inv_2dr = 1.0 / (2.0 * ctx->dr), inv_2dthe = 1.0 / (2.0 * ctx->dthe), inv_2dphi = 1.0 / (2.0 * ctx->dphi);
    a.inv_2dr = (float)inv_2dr; a.inv_2dthe = (float)inv_2dthe; a.inv_2dphi = (float)inv_2dphi;
    a.inv_dr = (float)(2.0 * inv_2dr); a.inv_dthe = (float)(2.0 * inv_2dthe); a.inv_dphi = (float)(2.0 * inv_2dphi);
    a.inv_dr2 = (float)(1.0 / (ctx->dr * ctx->dr)); a.inv_dthe2 = (float)(1.0 / (ctx->dthe * ctx->dthe));
    a.inv_dphi2 = (float)(1.0 / (ctx->dphi * ctx->dphi));
    a.half_dt = 0.5 * s->dt; a.dt_sixth = s->dt / 6.0;
    a.half_dt_f = (float)(0.5 * s->dt); a.dt_f = (float)s->dt;
    a.diffusion_ramp = (float)s->diffusion_ramp;
    a.tke_max_nd = (float)(1000.0 / (p.u_0 * p.u_0));
    a.force_nd = (float)(p.omega * ctx->shell_len / p.u_0);
    a.coeff_energy_p = (float)(p.u_0 * p.u_0 / (p.cp_l * p.t_0));
    a.coeff_energy = 1.0 / (p.c_0 * p.cp_l * p.t_0);
    a.coeff_MC_vel = p.L_atm / (p.u_0 * p.u_0);
    a.coeff_MC_q = p.L_atm / (p.u_0 * p.c_0);
    a.coeff_MC_t = p.L_atm / (p.u_0 * p.t_0);
    a.lv = p.lv; a.ls = p.ls; a.L_atm_over_u0 = p.L_atm / p.u_0;
    a.inv_re = (float)(1.0 / p.re_turb);
    a.inv_pr_turb = (float)(1.0 / p.pr_turb);
    a.nue_max = (float)(1000.0 / (p.u_0 * p.L_atm));
    a.nue_air_nd = (float)(1.5e-5 / (p.u_0 * p.L_atm));
    a.diff_prec_re_inv = (float)(1.0 / (p.sc_WaterVapour * p.re_turb));
    a.diff_co2_re_inv = (float)(1.0 / (p.sc_CO2 * p.re_turb));
    a.buoy_pref = (float)(s->buoyancy_ramp * p.g * s->dt / p.u_0);
    a.drag_pref = (float)(1.0 / 86400.0 * p.L_atm / p.u_0 * s->dt);
    a.turb_model = p.turb_model; a.wall_mode = p.wall_mode; a.nontrad = p.coriolis_nontrad;
    a.curvature = p.metric_curvature; a.tracer_diff_flux = p.tracer_diff_flux;
    a.write_diag = s->write_diagnostics & 1;
    a.store_n = s->store_n_level ? 1 : 0;
    for (int n = 0; n < kNY; n++) a.Yn_store[n] = ctx->field[ATHAD_TN + n];
}

extern "C" {

// The mixed-precision step (k_rk4m.cu): same launches, FP32 private buffers.
static athad_status rk4_step_mixed(athad_ctx* ctx, const athad_step_scalars* s)
{
    athad_status st = athad_level_mean(ctx);
    if (st != ATHAD_OK) return st;
    RK4MArgs a;
    mixed_args(ctx, s, a);
    for (int stage = 1; stage <= 4; stage++) {
        for (int n = 0; n < kNY; n++) {
            a.Yin[n] = (stage == 3) ? ctx->mB[n] : ctx->mA[n];
            a.Yout[n] = (stage == 1 || stage == 3) ? ctx->mA[n] : ctx->mB[n];
            a.Ybnd[n] = ctx->mB[n];
        }
        launch_rk4m_stage(stage, a, ctx->stream);
        ATHAD_CHECK_LAUNCH(ctx, "rk4 mixed stage");
    }
    return s->store_n_level ? store_precip_n_level(ctx, ctx->stream) : ATHAD_OK;
}

static PoissonArgs poisson_args(athad_ctx* ctx, int total_iter_count)
{
    PoissonArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    a.poi = ctx->poi;
    a.dlnrho = ctx->prof[ATHAD_PROF_DLNRHO_DR];
    a.aux_u = ctx->field[ATHAD_AUX_U]; a.aux_v = ctx->field[ATHAD_AUX_V]; a.aux_w = ctx->field[ATHAD_AUX_W];
    a.src = ctx->src;
    a.p = ctx->field[ATHAD_P_DYN];
    a.counters = ctx->counters;
    a.inv_2dr = 1.0 / (2.0 * ctx->dr); a.inv_2dthe = 1.0 / (2.0 * ctx->dthe); a.inv_2dphi = 1.0 / (2.0 * ctx->dphi);
    a.anelastic = ctx->p.anelastic; a.metric_div = ctx->p.metric_divergence;
    a.ceiling = (total_iter_count > 300) ? 3.0 : 10.0;          // PressureSolverAtm.h:583
    return a;
}

athad_status athad_pressure_sweep(athad_ctx* ctx, int32_t n_sweeps, int32_t total_iter_count)
{
    if (!ctx || n_sweeps < 0) return fail(ctx, ATHAD_ERR_INVALID, "pressure_sweep: bad argument");
    if (n_sweeps == 0) return ATHAD_OK;
    PoissonArgs a = poisson_args(ctx, total_iter_count);
    a.aux_lid = 1;
    for (int i = 0; i < n_sweeps; i++) {
        a.first_sweep = (i == 0) ? 1 : 0;
        launch_poisson_sweep(a, ctx->stream);
        ATHAD_CHECK_LAUNCH(ctx, "poisson sweep");
    }
    ctx->poisson_sweeps_since_reset = n_sweeps;
    return ATHAD_OK;
}

athad_status athad_project_initial_velocity(athad_ctx* ctx, int32_t n_sweeps, int32_t total_iter_count)
{
    if (!ctx || n_sweeps < 0) return fail(ctx, ATHAD_ERR_INVALID, "project_initial_velocity: bad argument");
    const size_t bytes = ctx->L.field_elems * sizeof(double);
    athad_status s = ATHAD_OK;
    for (int n = 0; n < 3 && s == ATHAD_OK; n++)               // PressureSolverAtm.h:694-704
        s = cuda_check(ctx, cudaMemcpyAsync(ctx->field[ATHAD_AUX_U + n], ctx->field[ATHAD_U + n], bytes,
                                            cudaMemcpyDeviceToDevice, ctx->stream), "project copy");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaMemsetAsync(ctx->field[ATHAD_P_DYN], 0, bytes, ctx->stream), "project zero");
    if (s != ATHAD_OK) return s;
    s = athad_pressure_sweep(ctx, n_sweeps, total_iter_count);
    if (s != ATHAD_OK) return s;
    PoissonArgs a = poisson_args(ctx, total_iter_count);
    launch_project_correct(a, ctx->field[ATHAD_U], ctx->field[ATHAD_V], ctx->field[ATHAD_W], ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "project correct");
    const int zero_fields[4] = {ATHAD_P_DYN, ATHAD_AUX_U, ATHAD_AUX_V, ATHAD_AUX_W};   // :752-762
    for (int n = 0; n < 4 && s == ATHAD_OK; n++)
        s = cuda_check(ctx, cudaMemsetAsync(ctx->field[zero_fields[n]], 0, bytes, ctx->stream), "project clear");
    return s;
}

static ColumnArgs column_args(athad_ctx* ctx)
{
    ColumnArgs a;
    std::memset(&a, 0, sizeof a);
    const athad_params& p = ctx->p;
    a.d = ctx->L.d;
    a.height = ctx->height; a.step_f = ctx->step_f;
    double** F = ctx->field;
    a.t = F[ATHAD_T]; a.c = F[ATHAD_C]; a.cloud = F[ATHAD_CLOUD]; a.ice = F[ATHAD_ICE]; a.gr = F[ATHAD_GR];
    a.co2 = F[ATHAD_CO2]; a.p_stat = F[ATHAD_P_STAT]; a.r_humid = F[ATHAD_R_HUMID]; a.r_dry = F[ATHAD_R_DRY];
    a.S_c_c = F[ATHAD_S_C_C]; a.P_rain = F[ATHAD_P_RAIN]; a.P_snow = F[ATHAD_P_SNOW];
    a.P_graupel = F[ATHAD_P_GRAUPEL]; a.Precipitation = F[ATHAD_PRECIPITATION];
    a.S_v = F[ATHAD_S_V]; a.S_c = F[ATHAD_S_C]; a.S_i = F[ATHAD_S_I]; a.S_r = F[ATHAD_S_R];
    a.S_s = F[ATHAD_S_S]; a.S_g = F[ATHAD_S_G];
    a.t_top_init = ctx->f2d[ATHAD_2D_T_TOP_INIT]; a.p_stat_landscape = ctx->f2d[ATHAD_2D_P_STAT_LANDSCAPE];
    a.rho_base = ctx->prof[ATHAD_PROF_RHO_BASE]; a.dlnrho = ctx->prof[ATHAD_PROF_DLNRHO_DR];
    a.row_sum = ctx->row_sum; a.row_cnt = ctx->row_cnt; a.coslat = ctx->coslat;
    a.counters = ctx->counters + 2;
    a.t_0 = p.t_0; a.t_00 = p.t_00; a.t_max_phys = p.t_max_phys; a.cloud_cap = p.cloud_cap;
    a.M_bg = p.M_bg; a.R_bg = p.R_bg; a.R_mix = p.R_mix; a.r_air = p.r_air; a.g = p.g; a.t_skin = p.t_skin;
    a.c_h2o_dry_top = p.c_h2o_dry_top;
    a.inv_2dr = 1.0 / (2.0 * ctx->dr); a.inv_dr = 1.0 / ctx->dr;
    return a;
}

athad_status athad_saturation_adjust(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    ColumnArgs a = column_args(ctx);
    athad_status s = cuda_check(ctx, cudaMemsetAsync(ctx->counters + 2, 0, sizeof(unsigned long long), ctx->stream), "counters");
    if (s != ATHAD_OK) return s;
    launch_saturation_adjust(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "saturation_adjust");
    return ATHAD_OK;
}

athad_status athad_densities(athad_ctx* ctx, int32_t set_water_profile)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    ColumnArgs a = column_args(ctx);
    a.set_water_profile = set_water_profile ? 1 : 0;
    launch_densities(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "densities");
    return ATHAD_OK;
}

athad_status athad_moist_convection(athad_ctx* ctx, int32_t iter_n)
{
    (void)iter_n;   // MoistConvection::run keeps it (m.iter_n) but no phase reads it
    if (!ctx) return ATHAD_ERR_INVALID;
    const athad_params& p = ctx->p;
    MoistArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    for (int f = 0; f < ATHAD_NFIELDS; f++) a.F[f] = ctx->field[f];
    a.evaporation = ctx->f2d[ATHAD_2D_EVAPORATION];
    a.q_sensible = ctx->f2d[ATHAD_2D_Q_SENSIBLE];
    a.height = ctx->height; a.step = ctx->step_mc; a.cose = ctx->cose;
    a.t_0 = p.t_0; a.cp_l = p.cp_l; a.s_0 = p.s_0; a.lv = p.lv; a.ls = p.ls; a.g = p.g; a.u_0 = p.u_0;
    a.r_Earth = p.r_Earth; a.p_0 = p.p_0; a.co2_0 = p.co2_0; a.c_0 = p.c_0; a.M_bg = p.M_bg; a.R_bg = p.R_bg;
    a.convection_perturbation = p.convection_perturbation;
    a.convection_mode = p.convection_mode;
    a.iter_prec = p.iter_prec;
    launch_moist_convection(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "moist_convection");
    return ATHAD_OK;
}

athad_status athad_get_report(athad_ctx* ctx, athad_report* out)
{
    if (!ctx || !out) return fail(ctx, ATHAD_ERR_INVALID, "get_report: bad argument");
    unsigned long long h[4] = {0, 0, 0, 0};
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(h, ctx->counters, 3 * sizeof(unsigned long long),
                                                     cudaMemcpyDeviceToHost, ctx->stream), "report");
    if (s == ATHAD_OK)
        s = cuda_check(ctx, cudaMemcpyAsync(h + 3, ctx->counters + kNonfiniteSlot, sizeof(unsigned long long),
                                            cudaMemcpyDeviceToHost, ctx->stream), "report");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "report sync");
    if (s != ATHAD_OK) return s;
    std::memset(out, 0, sizeof *out);
    const int64_t fluid = (int64_t)(ctx->L.d.im - 2) * (ctx->L.d.jm - 2) * (ctx->L.d.km - 2);
    out->poisson_src_cells = fluid * ctx->poisson_sweeps_since_reset;
    out->poisson_src_clamped = (int64_t)h[0];                // counted in every sweep
    out->satadj_ceiling_hits = (int64_t)h[2];
    out->nonfinite_inputs = (int64_t)h[3];
    if (ctx->step_timed) {
        float ms = 0.0f;
        s = cuda_check(ctx, cudaEventElapsedTime(&ms, ctx->ev_step0, ctx->ev_step1), "report step time");
        if (s != ATHAD_OK) return s;
        out->last_kernel_ms = ms;
    }
    return ATHAD_OK;
}

}  // extern "C"

namespace athad {
athad_status boundary_conditions(athad_ctx* ctx, int wall_bc)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    const athad_params& p = ctx->p;
    BcArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    for (int f = 0; f < ATHAD_NFIELDS; f++) a.F[f] = ctx->field[f];
    a.t_top_init = ctx->f2d[ATHAD_2D_T_TOP_INIT];
    a.vel_star = ctx->f2d[ATHAD_2D_VEL_STAR];
    // TurbulenceAtm::apply_wall_bc (TurbulenceAtm.h:109-147): C_nue = 0.028, the
    // constructor's nue_air = 1.5e-5, y1 = get_layer_height(1)
    a.tke_wall_den = std::sqrt(0.028) * p.u_0 * p.u_0;
    const double y1_safe = (ctx->layer_height1 < 1.0e-6) ? 1.0e-6 : ctx->layer_height1;
    const double nd_omega = p.L_atm / p.u_0, nue_air = 1.5e-5;
    if (p.turb_model == ATHAD_TURB_K_EPSILON) {
        a.dis_wall = 0.0; a.set_dis_wall = 1;
    } else if (p.turb_model == ATHAD_TURB_K_OMEGA) {
        a.dis_wall = 6.0 * nue_air / (0.075 * y1_safe * y1_safe) * nd_omega; a.set_dis_wall = 1;
    } else {
        a.dis_wall = 60.0 * nue_air / (0.0333 * y1_safe * y1_safe) * nd_omega; a.set_dis_wall = 1;
    }
    a.wall_bc = wall_bc;
    a.tke_max_nd = 1000.0 / (p.u_0 * p.u_0);
    a.nue_max = 1000.0 / (p.u_0 * p.L_atm);
    a.vel_max_nd = 100.0 / p.u_0;
    launch_boundary_conditions(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "boundary_conditions");
    return ATHAD_OK;
}
}  // namespace athad

extern "C" {

athad_status athad_boundary_conditions(athad_ctx* ctx) { return athad::boundary_conditions(ctx, 1); }

athad_status athad_post_rk4_filters(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    if (ctx->L.d.km > 3072) return fail(ctx, ATHAD_ERR_UNSUPPORTED, "post_rk4_filters: km > 3072");
    FilterArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    a.field[0] = ctx->field[ATHAD_U]; a.field[1] = ctx->field[ATHAD_V]; a.field[2] = ctx->field[ATHAD_W];
    a.polar_passes = ctx->polar_passes;
    launch_post_rk4_filters(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "post_rk4_filters");
    return ATHAD_OK;
}

athad_status athad_damp_wiggles(athad_ctx* ctx, athad_field f)
{
    if (!ctx || (int)f < 0 || (int)f >= ATHAD_NFIELDS) return fail(ctx, ATHAD_ERR_INVALID, "damp_wiggles: bad argument");
    if (ctx->L.d.km > 3072) return fail(ctx, ATHAD_ERR_UNSUPPORTED, "damp_wiggles: km > 3072");
    // the RK4 stage buffer A is free between RK4 steps
    launch_damp_wiggles(ctx->L.d, ctx->field[f], ctx->stA[0], ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "damp_wiggles");
    return ATHAD_OK;
}

static CapsArgs caps_args(athad_ctx* ctx)
{
    CapsArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    double** F = ctx->field;
    a.c = F[ATHAD_C]; a.cloud = F[ATHAD_CLOUD]; a.ice = F[ATHAD_ICE]; a.co2 = F[ATHAD_CO2];
    a.p_stat = F[ATHAD_P_STAT];
    a.P_rain = F[ATHAD_P_RAIN]; a.P_snow = F[ATHAD_P_SNOW]; a.P_graupel = F[ATHAD_P_GRAUPEL];
    a.P_conv = F[ATHAD_P_CONV]; a.Precipitation = F[ATHAD_PRECIPITATION];
    const athad_field S[7] = {ATHAD_S_V, ATHAD_S_C, ATHAD_S_I, ATHAD_S_R, ATHAD_S_S, ATHAD_S_G, ATHAD_S_C_C};
    for (int s = 0; s < 7; s++) a.S[s] = F[S[s]];
    a.cloud_cap = ctx->p.cloud_cap; a.g = ctx->p.g;
    a.row_q = ctx->row_sum; a.row_w = ctx->row_cnt;
    a.count = ctx->counters + 3;
    a.sums = reinterpret_cast<double*>(ctx->counters + 8);
    return a;
}

athad_status athad_moist_caps(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    launch_moist_caps(caps_args(ctx), ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "moist_caps");
    return ATHAD_OK;
}

athad_status athad_vapour_ceiling(athad_ctx* ctx, athad_ceiling_report* out)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    CapsArgs a = caps_args(ctx);
    athad_status s = cuda_check(ctx, cudaMemsetAsync(a.count, 0, sizeof(unsigned long long), ctx->stream),
                                "vapour_ceiling");
    if (s != ATHAD_OK) return s;
    launch_vapour_ceiling(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "vapour_ceiling");
    if (!out) return ATHAD_OK;
    unsigned long long h[11];
    s = cuda_check(ctx, cudaMemcpyAsync(h, ctx->counters, sizeof h, cudaMemcpyDeviceToHost, ctx->stream),
                   "vapour_ceiling report");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "vapour_ceiling sync");
    if (s != ATHAD_OK) return s;
    std::memset(out, 0, sizeof *out);
    out->n_ceiling = (int64_t)h[3];
    std::memcpy(&out->q_clipped, &h[8], sizeof(double));
    std::memcpy(&out->w_air, &h[9], sizeof(double));
    return ATHAD_OK;
}

athad_status athad_min_max(athad_ctx* ctx, athad_field f, athad_min_max_report* out)
{
    if (!ctx || !out || (int)f < 0 || (int)f >= ATHAD_NFIELDS) return fail(ctx, ATHAD_ERR_INVALID, "min_max: bad argument");
    const Dims& d = ctx->L.d;
    double* out_v = reinterpret_cast<double*>(ctx->counters + 12);
    long long* out_a = reinterpret_cast<long long*>(ctx->counters + 14);
    launch_min_max(d, ctx->field[f], ctx->stB[0], out_v, out_a, ctx->stream);   // stage buffer B: scratch
    ATHAD_CHECK_LAUNCH(ctx, "min_max");
    unsigned long long h[4];
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(h, ctx->counters + 12, sizeof h, cudaMemcpyDeviceToHost,
                                                     ctx->stream), "min_max report");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "min_max sync");
    if (s != ATHAD_OK) return s;
    std::memset(out, 0, sizeof *out);
    double v[2];
    long long at[2];
    std::memcpy(v, h, sizeof v);
    std::memcpy(at, h + 2, sizeof at);
    const long long plane = (long long)d.jm * d.km;
    if (at[0] >= 0) {   // MinMax_Atm.cpp:75-76: no finite value -> 0 at (0, 0, 0)
        out->max = v[0];
        out->imax = (int32_t)(at[0] / plane); out->jmax = (int32_t)(at[0] / d.km % d.jm); out->kmax = (int32_t)(at[0] % d.km);
    }
    if (at[1] >= 0) {
        out->min = v[1];
        out->imin = (int32_t)(at[1] / plane); out->jmin = (int32_t)(at[1] / d.km % d.jm); out->kmin = (int32_t)(at[1] % d.km);
    }
    return ATHAD_OK;
}

athad_status athad_find_residuum(athad_ctx* ctx, athad_residuum_report* out)
{
    if (!ctx || !out) return fail(ctx, ATHAD_ERR_INVALID, "find_residuum: bad argument");
    const Dims& d = ctx->L.d;
    ResiduumArgs a;
    a.d = d;
    a.u = ctx->field[ATHAD_U]; a.v = ctx->field[ATHAD_V]; a.w = ctx->field[ATHAD_W];
    a.sinthe = ctx->res_sin;
    a.rad = ctx->rad_d;
    a.dr = ctx->dr; a.dthe = ctx->dthe; a.dphi = ctx->dphi;
    a.i0 = 10;                                     // UtilsAtm.h:99
    a.i1 = std::min(30, d.im - 2);
    a.scratch = ctx->stB[0];                       // stage buffer B: 48 B per band row
    a.out = ctx->counters + 16;
    launch_find_residuum(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "find_residuum");
    unsigned long long h[6];
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(h, ctx->counters + 16, sizeof h, cudaMemcpyDeviceToHost,
                                                     ctx->stream), "find_residuum report");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "find_residuum sync");
    if (s != ATHAD_OK) return s;
    std::memset(out, 0, sizeof *out);
    double mx, sum;
    std::memcpy(&mx, &h[0], sizeof mx);
    std::memcpy(&sum, &h[2], sizeof sum);
    const long long at = (long long)h[1], key = (long long)h[5];
    out->residuum_prev = ctx->residuum_old;
    if (at >= 0) {
        out->residuum = mx;
        out->i_error = (int32_t)(at / ((long long)d.jm * d.km));
        out->j_error = (int32_t)(at / d.km % d.jm);
        out->k_error = (int32_t)(at % d.km);
    }
    out->n_cells = (int64_t)h[3];
    out->n_nonfinite = (int64_t)h[4];
    out->avg_abs = (out->n_cells > 0) ? sum / (double)out->n_cells : 0.0;   // UtilsAtm.h:175-176
    out->avg_rel = (out->residuum > 0.0) ? out->avg_abs / out->residuum : 0.0;
    out->i_nan = out->j_nan = out->k_nan = -1;
    if (out->n_nonfinite > 0) {
        out->i_nan = (int32_t)(key % d.im);
        out->j_nan = (int32_t)(key / d.im / d.km);
        out->k_nan = (int32_t)(key / d.im % d.km);
    }
    ctx->residuum_old = out->residuum;             // set once, after the reduction (:211-213)
    return ATHAD_OK;
}

athad_status athad_set_tropopause_layers(athad_ctx* ctx, const double* layers, int32_t n)
{
    if (!ctx || !layers) return fail(ctx, ATHAD_ERR_INVALID, "set_tropopause_layers: bad argument");
    const int im = ctx->grid.im, jm = ctx->grid.jm;
    if (n != jm) return fail(ctx, ATHAD_ERR_INVALID, "set_tropopause_layers: n must be jm");
    std::vector<int> lev(jm);
    for (int j = 0; j < jm; j++) {
        // ThermoAtm.h:414-419: the equator row takes its northern neighbour's level
        const double v = (j == (jm - 1) / 2 && j > 0) ? layers[j - 1] : layers[j];
        if (!(v >= 0.0) || !(v < (double)im)) return fail(ctx, ATHAD_ERR_INVALID, "set_tropopause_layers: level outside [0, im-1]");
        lev[j] = (int)v;
    }
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(ctx->i_trop, lev.data(), jm * sizeof(int), cudaMemcpyHostToDevice,
                                                     ctx->stream), "tropopause levels");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "tropopause levels sync");
    if (s == ATHAD_OK) ctx->trop_set = true;
    return s;
}

athad_status athad_stand_atm_dew_point(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    if (!ctx->trop_set) return fail(ctx, ATHAD_ERR_INVALID, "stand_atm_dew_point: tropopause layers not set");
    StandAtmArgs a;
    a.d = ctx->L.d;
    a.t = ctx->field[ATHAD_T]; a.c = ctx->field[ATHAD_C]; a.co2 = ctx->field[ATHAD_CO2];
    a.p_stat = ctx->field[ATHAD_P_STAT];
    a.height = ctx->height;
    a.i_trop = ctx->i_trop;
    a.temp_stand = ctx->field[ATHAD_TEMP_STAND];
    a.temp_dew = ctx->field[ATHAD_TEMP_DEW_POINT];
    a.humid_rel = ctx->field[ATHAD_HUMIDITY_REL];
    a.t_0 = ctx->p.t_0;
    a.M_bg = ctx->p.M_bg;
    launch_stand_atm(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "stand_atm_dew_point");
    return ATHAD_OK;
}

athad_status athad_update_skin_temperature(athad_ctx* ctx, double t_skin_relax, double* t_skin)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    const int jm = ctx->grid.jm, km = ctx->grid.km;
    if (t_skin_relax > 0.0) {                                  // cAtmosphereModel.cpp:293
        launch_albedo_rows(ctx->L.d, ctx->f2d[ATHAD_2D_ALBEDO], ctx->stB[0], ctx->stream);
        ATHAD_CHECK_LAUNCH(ctx, "albedo rows");
        std::vector<double> rows(jm);
        athad_status s = cuda_check(ctx, cudaMemcpyAsync(rows.data(), ctx->stB[0], jm * sizeof(double),
                                                         cudaMemcpyDeviceToHost, ctx->stream), "albedo rows");
        if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "albedo rows sync");
        if (s != ATHAD_OK) return s;
        // the insolation profile of MultiLayerRadiation.h:102-108 (AtomUtils::parabola)
        const athad_params& p = ctx->p;
        const int j_max = jm - 1, j_half = j_max / 2;
        std::vector<double> sw(jm, p.rad_pole_short);
        const double eff = p.rad_pole_short - p.rad_equator_short;
        for (int j = j_half; j >= 0; j--) {
            const double x = (double)j / (double)j_half;
            sw[j] = eff * (x * x - 2.0 * x) + p.rad_pole_short;
        }
        for (int j = j_max; j > j_half; j--) sw[j] = sw[j_max - j];
        // planetaryShortWave (:240-264)
        double w_sum = 0.0, abs_w = 0.0, alb_max = 0.0;
        for (int j = 0; j < jm; j++) {
            const double w = std::cos((j / (double)(jm - 1) - 0.5) * M_PI);
            const double alb_k = rows[j] / (double)km;
            alb_max = std::max(alb_max, alb_k);
            w_sum += w;
            abs_w += w * (1.0 - alb_k) * sw[j];
        }
        if (w_sum > 0.0 && alb_max > 0.0) {
            const double in_mean = abs_w / w_sum + p.geothermal_flux;    // :296-297
            if (in_mean > 0.0) {
                const double target = std::pow(in_mean / p.sigma, 0.25);
                ctx->p.t_skin += std::min(1.0, t_skin_relax) * (target - ctx->p.t_skin);
            }
        }
    }
    if (t_skin) *t_skin = ctx->p.t_skin;
    return ATHAD_OK;
}

// the per-level sums of co2Column / waterBudget on the device, read back (6 per level)
static athad_status budget_levels(athad_ctx* ctx, bool co2_total, std::vector<double>& lv)
{
    BudgetArgs a;
    a.d = ctx->L.d;
    a.p_stat = ctx->field[ATHAD_P_STAT];
    a.c = ctx->field[ATHAD_C]; a.cloud = ctx->field[ATHAD_CLOUD]; a.ice = ctx->field[ATHAD_ICE];
    a.gr = ctx->field[ATHAD_GR]; a.co2 = ctx->field[ATHAD_CO2];
    a.coslat = ctx->coslat;
    a.g = ctx->p.g;
    a.rows = ctx->stB[0];                          // stage buffers B: scratch
    a.levels = ctx->stB[1];
    a.co2_total = co2_total ? ctx->f2d[ATHAD_2D_CO2_TOTAL] : nullptr;
    launch_budgets(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "budgets");
    const int im = ctx->grid.im;
    lv.assign(6 * (size_t)im, 0.0);
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(lv.data(), a.levels, lv.size() * sizeof(double),
                                                     cudaMemcpyDeviceToHost, ctx->stream), "budgets report");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "budgets sync");
    return s;
}

static double pct(double now, double ref) { return (ref > 0.0) ? 100.0 * (now / ref - 1.0) : 0.0; }

athad_status athad_co2_column(athad_ctx* ctx, athad_budget_report* out)
{
    if (!ctx || !out) return fail(ctx, ATHAD_ERR_INVALID, "co2_column: bad argument");
    std::vector<double> lv;
    athad_status s = budget_levels(ctx, true, lv);
    if (s != ATHAD_OK) return s;
    double w_num = 0.0, w_den = 0.0;
    for (int i = 0; i < ctx->grid.im; i++) { w_den += lv[6 * i + 0]; w_num += lv[6 * i + 2]; }
    std::memset(out, 0, sizeof *out);
    out->q_mean = (w_den > 0.0) ? w_num / w_den : 0.0;           // ThermoAtm.h:1125-1126
    if (ctx->q_co2_ref <= 0.0) ctx->q_co2_ref = out->q_mean;
    out->q_ref = ctx->q_co2_ref;
    out->drift_pct = pct(out->q_mean, out->q_ref);
    return ATHAD_OK;
}

athad_status athad_water_budget(athad_ctx* ctx, athad_budget_report* out, double* level_drift)
{
    if (!ctx || !out) return fail(ctx, ATHAD_ERR_INVALID, "water_budget: bad argument");
    std::vector<double> lv;
    athad_status s = budget_levels(ctx, false, lv);
    if (s != ATHAD_OK) return s;
    const int im = ctx->grid.im;
    double w_num = 0.0, w_den = 0.0;
    for (int i = 0; i < im; i++) { w_den += lv[6 * i + 0]; w_num += lv[6 * i + 1]; }
    std::memset(out, 0, sizeof *out);
    out->q_mean = (w_den > 0.0) ? w_num / w_den : 0.0;           // ThermoAtm.h:963-964
    if (ctx->q_h2o_ref <= 0.0) ctx->q_h2o_ref = out->q_mean;
    out->q_ref = ctx->q_h2o_ref;
    out->drift_pct = pct(out->q_mean, out->q_ref);
    // level means and air masses (:974-996), frozen weights (:1003-1014), levels (:1020-1033)
    std::vector<double> qbar(im), abar(im), lev(im);
    for (int i = 0; i < im; i++) {
        qbar[i] = (lv[6 * i + 4] > 0.0) ? lv[6 * i + 3] / lv[6 * i + 4] : 0.0;
        abar[i] = lv[6 * i + 0];
        lev[i] = (w_den > 0.0) ? lv[6 * i + 1] / w_den : 0.0;
    }
    if (ctx->air_levels.empty()) ctx->air_levels = abar;
    double qf_num = 0.0, qf_den = 0.0;
    for (int i = 0; i < im; i++) {
        qf_num += ctx->air_levels[i] * qbar[i];
        qf_den += ctx->air_levels[i];
        out->air_now += abar[i];
    }
    out->air_ref = qf_den;
    out->q_fixed = (qf_den > 0.0) ? qf_num / qf_den : 0.0;
    if (ctx->q_h2o_fixed_ref <= 0.0) ctx->q_h2o_fixed_ref = out->q_fixed;
    out->q_fixed_ref = ctx->q_h2o_fixed_ref;
    out->fixed_drift_pct = pct(out->q_fixed, out->q_fixed_ref);
    out->air_drift_pct = pct(out->air_now, out->air_ref);
    if (ctx->h2o_levels.empty()) ctx->h2o_levels = lev;
    if (level_drift)
        for (int i = 0; i < im; i++) level_drift[i] = lev[i] - ctx->h2o_levels[i];
    return ATHAD_OK;
}

static SurfaceArgs surface_args(athad_ctx* ctx)
{
    SurfaceArgs a;
    a.d = ctx->L.d;
    a.c = ctx->field[ATHAD_C]; a.t = ctx->field[ATHAD_T]; a.co2 = ctx->field[ATHAD_CO2];
    a.p_stat = ctx->field[ATHAD_P_STAT];
    a.u = ctx->field[ATHAD_U]; a.v = ctx->field[ATHAD_V]; a.w = ctx->field[ATHAD_W];
    a.evap = ctx->f2d[ATHAD_2D_EVAPORATION];
    a.evap_dalton = ctx->f2d[ATHAD_2D_EVAPORATION_DALTON];
    a.evap_meyer = ctx->f2d[ATHAD_2D_EVAPORATION_MEYER];
    a.evap_rohwer = ctx->f2d[ATHAD_2D_EVAPORATION_ROHWER];
    a.c_fix = ctx->f2d[ATHAD_2D_C_FIX];
    a.q_latent = ctx->field[ATHAD_Q_LATENT];
    a.q_sensible = ctx->field[ATHAD_Q_SENSIBLE];
    a.sin_w = ctx->sin_w;
    a.rad = ctx->rad_d;
    a.t_0 = ctx->p.t_0; a.u_0 = ctx->p.u_0; a.M_bg = ctx->p.M_bg;
    a.coeff_Dalton = ctx->p.coeff_Dalton; a.cp_l = ctx->p.cp_l;
    // the vertical spread of ThermoAtm.h:130-132: r = e^-1 over n_spread = 3 levels
    const double r = std::exp(-1.0);
    a.w_norm = (1.0 - r) / (1.0 - std::pow(r, 3 + 1));
    for (int i = 1; i <= 3; i++) a.weight[i - 1] = std::pow(r, i) * a.w_norm;
    a.dr = ctx->dr; a.dthe = ctx->dthe; a.dphi = ctx->dphi;
    return a;
}

athad_status athad_water_vapour_evaporation(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    launch_water_vapour_evaporation(surface_args(ctx), ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "water_vapour_evaporation");
    return ATHAD_OK;
}

athad_status athad_latent_sensible_heat(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    launch_latent_sensible_heat(surface_args(ctx), ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "latent_sensible_heat");
    return ATHAD_OK;
}

athad_status athad_checkpoint_begin(athad_ctx* ctx, const int32_t* fields, int32_t n, double* const* hosts)
{
    if (!ctx || n < 0 || (n > 0 && (!fields || !hosts))) return fail(ctx, ATHAD_ERR_INVALID, "checkpoint_begin: bad argument");
    for (int q = 0; q < n; q++)
        if (fields[q] < 0 || fields[q] >= ATHAD_NFIELDS || !hosts[q])
            return fail(ctx, ATHAD_ERR_INVALID, "checkpoint_begin: bad field or host buffer");
    const Dims& d = ctx->L.d;
    const size_t fb = ctx->L.field_elems * sizeof(double);
    athad_status s = ATHAD_OK;
    if (!ctx->ckpt_stream) {
        s = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->ckpt_stream, cudaStreamNonBlocking), "checkpoint stream");
        if (s == ATHAD_OK) s = cuda_check(ctx, cudaEventCreateWithFlags(&ctx->ckpt_ready, cudaEventDisableTiming), "checkpoint event");
        if (s == ATHAD_OK) s = cuda_check(ctx, cudaEventCreateWithFlags(&ctx->ckpt_done, cudaEventDisableTiming), "checkpoint event");
        if (s == ATHAD_OK) s = cuda_check(ctx, cudaEventRecord(ctx->ckpt_done, ctx->ckpt_stream), "checkpoint event");
        if (s != ATHAD_OK) return s;
    }
    // the snapshot may still be on its way to the host from the previous checkpoint
    s = cuda_check(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ckpt_done, 0), "checkpoint wait");
    if (s != ATHAD_OK) return s;
    if (n > ctx->ckpt_cap) {
        s = cuda_check(ctx, cudaStreamSynchronize(ctx->ckpt_stream), "checkpoint sync");
        if (s != ATHAD_OK) return s;
        cudaFree(ctx->ckpt_buf);
        ctx->ckpt_buf = nullptr;
        ctx->ckpt_cap = 0;
        s = cuda_check(ctx, cudaMalloc((void**)&ctx->ckpt_buf, (size_t)n * fb), "checkpoint buffer");
        if (s != ATHAD_OK) return s;
        ctx->ckpt_cap = n;
    }
    for (int q = 0; q < n && s == ATHAD_OK; q++)
        s = cuda_check(ctx, cudaMemcpyAsync(ctx->ckpt_buf + (size_t)q * ctx->L.field_elems, ctx->field[fields[q]], fb,
                                            cudaMemcpyDeviceToDevice, ctx->stream), "checkpoint snapshot");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaEventRecord(ctx->ckpt_ready, ctx->stream), "checkpoint event");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaStreamWaitEvent(ctx->ckpt_stream, ctx->ckpt_ready, 0), "checkpoint wait");
    for (int q = 0; q < n && s == ATHAD_OK; q++)
        s = cuda_check(ctx, cudaMemcpy2DAsync(hosts[q], d.km * sizeof(double), ctx->ckpt_buf + (size_t)q * ctx->L.field_elems,
                                              d.pitch * sizeof(double), d.km * sizeof(double), (size_t)d.im * d.jm,
                                              cudaMemcpyDeviceToHost, ctx->ckpt_stream), "checkpoint download");
    if (s == ATHAD_OK) s = cuda_check(ctx, cudaEventRecord(ctx->ckpt_done, ctx->ckpt_stream), "checkpoint event");
    return s;
}

athad_status athad_checkpoint_wait(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    if (!ctx->ckpt_stream) return ATHAD_OK;
    return cuda_check(ctx, cudaEventSynchronize(ctx->ckpt_done), "checkpoint_wait");
}

static athad_status multilayer_radiation(athad_ctx* ctx)
{
    const athad_params& p = ctx->p;
    RadArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    double** F = ctx->field;
    a.t = F[ATHAD_T]; a.c = F[ATHAD_C]; a.co2 = F[ATHAD_CO2]; a.p_stat = F[ATHAD_P_STAT];
    a.cloud = F[ATHAD_CLOUD]; a.ice = F[ATHAD_ICE];
    a.radiation = F[ATHAD_RADIATION]; a.epsilon = F[ATHAD_EPSILON];
    a.epsilon_2D = ctx->f2d[ATHAD_2D_EPSILON]; a.albedo = ctx->f2d[ATHAD_2D_ALBEDO];
    a.T = ctx->stA[1]; a.dn = ctx->stA[2];   // RK4 stage buffers, free between RK4 steps
    a.step_f = ctx->step_f;
    a.t_0 = p.t_0; a.g = p.g; a.R_bg = p.R_bg; a.sigma = p.sigma;
    a.kappa_H2O = p.kappa_H2O; a.kappa_CO2 = p.kappa_CO2; a.kappa_bg = p.kappa_bg;
    a.geothermal_flux = p.geothermal_flux; a.albedo_surface = p.albedo_surface;
    a.albedo_cloud = p.albedo_cloud; a.rad_equator_short = p.rad_equator_short;
    a.rad_pole_short = p.rad_pole_short;
    launch_multilayer_radiation(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "multilayer_radiation");
    return ATHAD_OK;
}

athad_status athad_multilayer_radiation(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    return multilayer_radiation(ctx);
}

athad_status athad_radiative_heating(athad_ctx* ctx, double omega_rad)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    double* t = ctx->field[ATHAD_T];
    double* t_before = ctx->stA[0];
    athad_status s = cuda_check(ctx, cudaMemcpyAsync(t_before, t, ctx->L.field_elems * sizeof(double),
                                                     cudaMemcpyDeviceToDevice, ctx->stream), "radiative_heating");
    if (s == ATHAD_OK) s = multilayer_radiation(ctx);
    if (s != ATHAD_OK) return s;
    launch_rad_blend(ctx->L.d, t_before, t, omega_rad, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "radiative_heating blend");
    return ATHAD_OK;
}

// the fields and constants of the ice / precipitation schemes
static void ice_args(athad_ctx* ctx, IceArgs& a)
{
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    double** F = ctx->field;
    a.t = F[ATHAD_T]; a.c = F[ATHAD_C]; a.cloud = F[ATHAD_CLOUD]; a.ice = F[ATHAD_ICE]; a.gr = F[ATHAD_GR];
    a.co2 = F[ATHAD_CO2]; a.p_stat = F[ATHAD_P_STAT]; a.r_humid = F[ATHAD_R_HUMID];
    a.P_rain = F[ATHAD_P_RAIN]; a.P_snow = F[ATHAD_P_SNOW]; a.P_graupel = F[ATHAD_P_GRAUPEL];
    a.Precipitation = F[ATHAD_PRECIPITATION]; a.P_rainn = F[ATHAD_P_RAINN]; a.P_snown = F[ATHAD_P_SNOWN];
    a.S_v = F[ATHAD_S_V]; a.S_c = F[ATHAD_S_C]; a.S_i = F[ATHAD_S_I]; a.S_r = F[ATHAD_S_R];
    a.S_s = F[ATHAD_S_S]; a.S_g = F[ATHAD_S_G]; a.S_c_c = F[ATHAD_S_C_C];
    a.step_f = ctx->step_f;
    const athad_params& p = ctx->p;
    a.t_0 = p.t_0; a.t_000 = p.t_000; a.M_bg = p.M_bg; a.t_00 = p.t_00; a.ls = p.ls;
}

athad_status athad_two_cat_ice_scheme(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    if (ctx->L.d.im < 3 || ctx->L.d.jm < 3 || ctx->L.d.km < 3)
        return fail(ctx, ATHAD_ERR_UNSUPPORTED, "two_cat_ice_scheme: grid too small");
    IceArgs a;
    ice_args(ctx, a);
    launch_two_cat_ice(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "two_cat_ice_scheme");
    return ATHAD_OK;
}

// ZeroCat, OneCat and ThreeCat read the rain flux at level 23 (P_rain.x[23]) for their
// convergence test
static bool ice_level_23(athad_ctx* ctx, const char* what)
{
    if (ctx->L.d.im >= 24) return true;
    char msg[160];
    std::snprintf(msg, sizeof msg, "%s: the scheme reads level 23, the grid needs im >= 24", what);
    fail(ctx, ATHAD_ERR_UNSUPPORTED, msg);
    return false;
}

athad_status athad_zero_cat_ice_scheme(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    if (!ice_level_23(ctx, "zero_cat_ice_scheme")) return ATHAD_ERR_UNSUPPORTED;
    IceArgs a;
    ice_args(ctx, a);
    launch_zero_cat_ice(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "zero_cat_ice_scheme");
    return ATHAD_OK;
}

athad_status athad_one_cat_ice_scheme(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    if (!ice_level_23(ctx, "one_cat_ice_scheme")) return ATHAD_ERR_UNSUPPORTED;
    IceArgs a;
    ice_args(ctx, a);
    // the carry of S_au across columns, in RK4 stage buffers (free between RK4 steps; one
    // double per interior column each)
    a.sau_exit = ctx->stA[1]; a.sau_has = ctx->stA[2]; a.sau_entry = ctx->stA[3];
    launch_one_cat_ice(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "one_cat_ice_scheme");
    return ATHAD_OK;
}

athad_status athad_three_cat_ice_scheme(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    if (!ice_level_23(ctx, "three_cat_ice_scheme")) return ATHAD_ERR_UNSUPPORTED;
    IceArgs a;
    ice_args(ctx, a);
    // ThreeCatIceScheme.h:147-170, on the host once per call
    const double N_r_0 = 8.0e+6, N_s_0 = 8.0e+5, N_g_0 = 4.0e6, v_s_0 = 130.0, v_r_0 = 4.9;
    const double v_g_0 = 442.0, a_s_m = 0.038, a_g_m = 169.6;
    const double gamma_4_5 = std::tgamma(4.5), gamma_4_0 = std::tgamma(4.0), gamma_3_25 = std::tgamma(3.25);
    const double r0w = ctx->p.r_0_water;
    a.A_r = r0w * M_PI * N_r_0;
    a.A_s = 2.0 * a_s_m * N_s_0;
    a.A_g = 2.0 * a_g_m * N_g_0;
    const double B_rad = r0w * M_PI * N_r_0 * v_r_0 * gamma_4_5 / gamma_4_0;
    const double B_s = N_s_0 * v_s_0 * a_s_m * gamma_3_25;
    const double B_g = N_g_0 * v_g_0 * a_g_m * gamma_3_25;
    a.B_rad_neg89 = std::pow(B_rad, -8.0 / 9.0);
    a.B_s_neg1213 = std::pow(B_s, -12.0 / 13.0);
    a.B_g_neg1213 = std::pow(B_g, -12.0 / 13.0);
    a.E_sat_t_0_Pa = 1e2 * thermo::saturation_pressure(ctx->p.t_0);
    launch_three_cat_ice(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "three_cat_ice_scheme");
    return ATHAD_OK;
}

athad_status athad_ice_scheme(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    switch (ctx->p.category_ice_scheme) {
    case -1: return ATHAD_OK;
    case 0: return athad_zero_cat_ice_scheme(ctx);
    case 1: return athad_one_cat_ice_scheme(ctx);
    case 2: return athad_two_cat_ice_scheme(ctx);
    case 3: return athad_three_cat_ice_scheme(ctx);
    default: return fail(ctx, ATHAD_ERR_UNSUPPORTED, "ice_scheme: category_ice_scheme not in -1..3");
    }
}

athad_status athad_turbulence_run(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    const athad_params& p = ctx->p;
    TurbArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = ctx->L.d;
    double** F = ctx->field;
    a.u = F[ATHAD_U]; a.v = F[ATHAD_V]; a.w = F[ATHAD_W];
    a.tke = F[ATHAD_TKE]; a.dis = F[ATHAD_DIS]; a.prod = F[ATHAD_PROD]; a.nue = F[ATHAD_NUE];
    a.tke_source = F[ATHAD_TKE_SOURCE]; a.dis_source = F[ATHAD_DIS_SOURCE];
    a.vel_star = ctx->f2d[ATHAD_2D_VEL_STAR];
    a.sin_w = ctx->sin_w;
    a.lev = ctx->turb_lev;
    a.inv_2dr = 1.0 / (2.0 * ctx->dr); a.inv_2dthe = 1.0 / (2.0 * ctx->dthe); a.inv_2dphi = 1.0 / (2.0 * ctx->dphi);
    a.dr = ctx->dr; a.dthe = ctx->dthe; a.dphi = ctx->dphi;
    a.u_0 = p.u_0; a.L_atm = p.L_atm; a.re_turb = p.re_turb;
    a.nue_max = 1000.0 / (p.u_0 * p.L_atm);    // TurbulenceAtm.h:272, :454
    a.y_mount = 0.0;                             // get_layer_height(0) of flat terrain
    a.turb_model = p.turb_model;
    launch_turbulence_run(a, ctx->stream);
    ATHAD_CHECK_LAUNCH(ctx, "turbulence_run");
    return ATHAD_OK;
}

}  // extern "C"
