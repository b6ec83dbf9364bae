// Test infrastructure: a host build of the CUDA library's column passes (k_columns.cu) for
// tests/test_columns_host_cpu.py: the fused saturation adjustment and clampAndFade of one
// cell (satadj_cell) and the densities' upward integration of one column
// (densities_column), run over every cell / column of host arrays packed (i, j, k) with
// k fastest, so their logic is checked against the oracle on a machine without a GPU.
#include "../athad_cond_b200/csrc/k_columns.cu"

using namespace athad;

// F: ATHAD_NFIELDS field pointers in the ABI's order; t_top_init, p_stat_landscape: [jm][km];
// height, step_f: [im]; dp: t_0, t_00, t_max_phys, cloud_cap, M_bg, R_bg, R_mix, r_air, g,
// t_skin, c_h2o_dry_top
static ColumnArgs host_args(int im, int jm, int km, double* const* F, double* t_top_init,
                            double* p_stat_landscape, const double* height, const double* step_f,
                            const double* dp)
{
    ColumnArgs a;
    memset(&a, 0, sizeof a);
    a.d.im = im; a.d.jm = jm; a.d.km = km; a.d.pitch = km;
    a.d.plane = (long long)jm * km;
    a.d.fstride = (long long)im * jm * km;
    a.height = height; a.step_f = step_f;
    a.t = F[ATHAD_T]; a.c = F[ATHAD_C]; a.cloud = F[ATHAD_CLOUD]; a.ice = F[ATHAD_ICE]; a.gr = F[ATHAD_GR];
    a.co2 = F[ATHAD_CO2]; a.p_stat = F[ATHAD_P_STAT]; a.r_humid = F[ATHAD_R_HUMID]; a.r_dry = F[ATHAD_R_DRY];
    a.S_c_c = F[ATHAD_S_C_C]; a.P_rain = F[ATHAD_P_RAIN]; a.P_snow = F[ATHAD_P_SNOW];
    a.P_graupel = F[ATHAD_P_GRAUPEL]; a.Precipitation = F[ATHAD_PRECIPITATION];
    a.S_v = F[ATHAD_S_V]; a.S_c = F[ATHAD_S_C]; a.S_i = F[ATHAD_S_I]; a.S_r = F[ATHAD_S_R];
    a.S_s = F[ATHAD_S_S]; a.S_g = F[ATHAD_S_G];
    a.t_top_init = t_top_init; a.p_stat_landscape = p_stat_landscape;
    a.t_0 = dp[0]; a.t_00 = dp[1]; a.t_max_phys = dp[2]; a.cloud_cap = dp[3]; a.M_bg = dp[4];
    a.R_bg = dp[5]; a.R_mix = dp[6]; a.r_air = dp[7]; a.g = dp[8]; a.t_skin = dp[9];
    a.c_h2o_dry_top = dp[10];
    return a;
}

// Returns the number of cells whose vapour hit its 1 - co2 cap (the kernel's counter).
extern "C" long long host_saturation_adjust(int im, int jm, int km, double* const* F, double* t_top_init,
                                            double* p_stat_landscape, const double* height,
                                            const double* step_f, const double* dp)
{
    const ColumnArgs a = host_args(im, jm, km, F, t_top_init, p_stat_landscape, height, step_f, dp);
    long long hits = 0;
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++)
            for (int k = 0; k < km; k++) hits += satadj_cell(a, i, j, k) ? 1 : 0;
    return hits;
}

extern "C" void host_densities_columns(int im, int jm, int km, double* const* F, double* t_top_init,
                                       double* p_stat_landscape, const double* height,
                                       const double* step_f, const double* dp, int set_water_profile)
{
    ColumnArgs a = host_args(im, jm, km, F, t_top_init, p_stat_landscape, height, step_f, dp);
    a.set_water_profile = set_water_profile;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) densities_column(a, j, k);
}
