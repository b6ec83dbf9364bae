// Test infrastructure: a host build of the CUDA library's moist-convection column code
// (athad_cond_b200/csrc/k_moist.cu, mc_column) for tests/test_moist_host_cpu.py.  It runs
// the same source as moist_convection_kernel, one (j, k) column after another, on host
// arrays packed (i, j, k) with k fastest, so the kernel's logic can be checked against the
// oracle on a machine without a GPU.
#include "../athad_cond_b200/csrc/k_moist.cu"

using namespace athad;

// F: ATHAD_NFIELDS field pointers in the ABI's order; evap, q_sensible: [jm][km]; height,
// step: [im]; cose: [jm]; dp: t_0, cp_l, s_0, lv, ls, g, u_0, r_Earth, p_0, co2_0, c_0, M_bg,
// R_bg; ip: convection_perturbation, convection_mode, iter_prec
extern "C" void host_moist_convection(int im, int jm, int km, double* const* F, const double* evap,
                                      const double* q_sensible, const double* height,
                                      const double* step, const double* cose, const double* dp,
                                      const int* ip)
{
    MoistArgs X;
    X.d.im = im; X.d.jm = jm; X.d.km = km; X.d.pitch = km;
    X.d.plane = (long long)jm * km;
    X.d.fstride = (long long)im * jm * km;
    for (int f = 0; f < ATHAD_NFIELDS; f++) X.F[f] = F[f];
    X.evaporation = evap; X.q_sensible = q_sensible;
    X.height = height; X.step = step; X.cose = cose;
    X.t_0 = dp[0]; X.cp_l = dp[1]; X.s_0 = dp[2]; X.lv = dp[3]; X.ls = dp[4]; X.g = dp[5];
    X.u_0 = dp[6]; X.r_Earth = dp[7]; X.p_0 = dp[8]; X.co2_0 = dp[9]; X.c_0 = dp[10];
    X.M_bg = dp[11]; X.R_bg = dp[12];
    X.convection_perturbation = ip[0]; X.convection_mode = ip[1]; X.iter_prec = ip[2];
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) mc_column(X, j, k);
}
