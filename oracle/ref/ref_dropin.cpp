// ref_dropin.cpp - the drop-in demonstrated on the reference itself (test infrastructure).
//
// Compiles the product's C++ adapter (athad_cond_b200/host/athad_dropin.hpp) against the
// reference's own cAtmosphereModel and exposes it to the tests: the reference's hot-path
// calls and their drop-in replacements run on the same model object, so the tests compare
// the reference's CPU results with the device results the reference's call sites would get.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "tinyxml2.h"

#define private public
#define protected public
#include "cAtmosphereModel.h"
#undef private
#undef protected

#include "../../athad_cond_b200/host/athad_dropin.hpp"

using Dev = athad_dropin::Device<cAtmosphereModel>;

extern "C" {

// what: 0 RK4, 1 pressure sweep, 2 saturation adjustment, 3 moist convection,
// 4 densities, 5 densities(set_water_profile), ... 18 the CategoryIceScheme switch with the
// model's CategoryIceScheme set to arg for the call.  wall: 0 mirror, 1 reference.
// Returns 0, or -1 with the message in err.
int dropin_run(void* model, int what, int arg, int wall, char* err, int errlen)
{
    cAtmosphereModel* m = (cAtmosphereModel*)model;
    const int category = m->CategoryIceScheme;
    if (what == 18) m->CategoryIceScheme = arg;
    struct Restore {
        cAtmosphereModel* m; int c;
        ~Restore() { m->CategoryIceScheme = c; }
    } restore{m, category};
    try {
        Dev d(*m, wall ? ATHAD_WALL_REFERENCE : ATHAD_WALL_MIRROR);
        switch (what) {
            case 0: d.SolveRungeKutta(*m); break;
            case 1: d.PressureSolverRun(*m); break;
            case 2: d.SaturationAdjustmentRun(*m); break;
            case 3: d.MoistConvectionRun(*m, arg); break;
            case 4: d.Densities(*m, false); break;
            case 5: d.Densities(*m, true); break;
            case 6: d.BoundaryConditions(*m); break;
            case 7: d.PostRK4Filters(*m); break;
            case 8: d.DampMoistWiggles(*m); break;
            case 9: d.TurbulenceRun(*m); break;
            case 10: d.TwoCatIceSchemeRun(*m); break;
            case 11: d.MultiLayerRadiationRun(*m); break;
            case 12: d.RadiativeHeating(*m, 0.05); break;
            case 13: d.StandAtmDewPointHumidRel(*m); break;
            case 14: d.FindResiduumAtm(*m); break;
            case 15: d.WaterVapourEvaporation(*m); break;
            case 16: d.LatentSensibleHeat(*m); break;
            case 17: {   // first calls of both budgets (the model's references cleared)
                m->m_q_co2_ref = -1.0; m->m_q_h2o_ref = -1.0; m->m_q_h2o_fixed_ref = -1.0;
                d.Co2Column(*m);
                d.WaterBudget(*m);
                break;
            }
            case 18: d.IceSchemeRun(*m); break;
            default: return -1;
        }
    } catch (const std::exception& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return -1;
    }
    return 0;
}

// n iterations of run_3D_loop's body through the device-resident drop-in
// (athad_dropin::ResidentLoop) on the model, with the reference's loop header for each
// (cAtmosphereModel.cpp:1103-1131: total_iter_count, no inviscid spin-up, dt_visc, the
// buoyancy ramp), the state synced back into the model at the end.  residua: n values (the
// residuum of each iteration); t_skin: n values.  Returns 0, or -1 with the message in err.
int dropin_resident(void* model, int n, int first_iter, int wall, double* residua, double* t_skin,
                    char* err, int errlen)
{
    cAtmosphereModel* m = (cAtmosphereModel*)model;
    try {
        Dev d(*m, wall ? ATHAD_WALL_REFERENCE : ATHAD_WALL_MIRROR);
        athad_dropin::ResidentLoop<cAtmosphereModel> loop(d, *m);
        for (int q = 0; q < n; q++) {
            m->iter_n = first_iter + q;
            m->total_iter_count++;
            m->diffusion_ramp = 1.0;
            m->dt = m->dt_visc;
            m->buoyancy_ramp = (m->buoyancy_ramp_iters > 0)
                ? std::min(1.0, (double)m->total_iter_count / m->buoyancy_ramp_iters) : 1.0;
            athad_dropin::IterationReport r = loop.Iteration(*m);
            residua[q] = r.residuum.residuum;
            t_skin[q] = r.t_skin;
        }
        loop.Sync(*m);
    } catch (const std::exception& e) {
        if (err && errlen > 0) { std::strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
        return -1;
    }
    return 0;
}

// the athad_params the adapter builds from the model (athad_dropin::params_from)
void dropin_params(void* model, int wall, athad_params* out)
{
    *out = athad_dropin::params_from(*(cAtmosphereModel*)model, wall ? ATHAD_WALL_REFERENCE : ATHAD_WALL_MIRROR);
}

// the model's loop scalars the resident loop reads: dt_visc, buoyancy_ramp_iters,
// t_skin_relax, checkpoint, total_iter_count, t_skin
void dropin_loop_scalars(void* model, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)model;
    out[0] = m->dt_visc;
    out[1] = (double)m->buoyancy_ramp_iters;
    out[2] = m->t_skin_relax;
    out[3] = (double)m->checkpoint;
    out[4] = (double)m->total_iter_count;
    out[5] = m->t_skin;
}

// the model's budget references: m_q_co2_ref, m_q_h2o_ref, m_q_h2o_fixed_ref
void dropin_budget_refs(void* model, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)model;
    out[0] = m->m_q_co2_ref; out[1] = m->m_q_h2o_ref; out[2] = m->m_q_h2o_fixed_ref;
}

// the model's residuum_old (what findResiduumAtm leaves behind)
double dropin_residuum_old(void* model) { return ((cAtmosphereModel*)model)->residuum_old; }

}  // extern "C"
