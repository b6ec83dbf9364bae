"""A whole model iteration on the device: cAtmosphereModel::run_3D_loop
(atmosphere/cAtmosphereModel.cpp:1101-1700) for the configuration of cli/config_cond.xml
(flat terrain, turb_model k_omega_SST, the ice scheme of the params' category_ice_scheme
(2), radiation_mode 2, no inviscid spin-up), every step through the C ABI on one context, the
state resident in HBM.

Per iteration, in the reference's order:

  :1156  pressure sweep                                   every 4th iteration
  :1162  moist block                                      every 2nd iteration
         :1216 waterBudget("post-RK4"), :1218 SaturationAdjustment,
         :1225 damp_wiggles(t, ice, c, cloud), :1230-1242 the CategoryIceScheme switch,
         :1244 damp_wiggles(P_rain, P_snow), :1247 MoistConvection,
         :1249-1263 damp_wiggles of the convection fields, :1265-1334 precipitationSum and
         the caps, :1369-1391 the vapour ceiling, :1416 co2Column, :1417 waterBudget,
         :1418 densities, :1419 forces, :1420 standAtm_DewPoint_HumidRel,
         :1421 waterVapourEvaporation, :1422 latentSensibleHeat, :1426-1433
         TurbulenceAtm::run and its damp_wiggles
  :1439  boundary conditions (bcRadius, the turbulence wall values, bcTheta, bcPhi,
         bcScalarSurfSur, bcSolidGround)                  every iteration
  :1509  RK4 step, with the right-hand side's diagnostic outputs every iteration (the
         reference writes them in every call) and its momentum-budget terms on checkpoint
         iterations (:1471, 1502); :1524-1575 polar zonal and radial Shapiro filters;
  :1645  findResiduumAtm; :1647 storeIntermediateData3D; :1656 radiative heating;
  :1661  updateSkinTemperature

The orographic, steep-massif and coastal filters act on land cells only and do nothing on
flat terrain; forces' centrifugal and pressure-gradient arrays (output only),
vegetationLand (land only), the zonal-mean momentum-budget differencing of checkpoint
iterations and the file output are not run.  The residuum, the budgets and the skin
temperature each read a few numbers back, so an iteration synchronises with the device four
times.
"""
from __future__ import annotations

import numpy as np

from .context import GpuAtmosphere

MOIST_FIELDS_AFTER_SATADJ = ("t", "ice", "c", "cloud")
ICE_FLUXES = ("P_rain", "P_snow")
CONVECTION_FIELDS = ("P_conv", "E_u", "M_u", "q_v_u", "q_c_u", "E_d", "M_d", "q_v_d",
                     "MC_t", "MC_v", "MC_w")
TURBULENCE_FIELDS = ("tke", "dis", "nue", "prod", "tke_source", "dis_source")


class ModelLoop:
    """run_3D_loop on a GpuAtmosphere whose state is uploaded.

    dt: dt_visc (4e-5); buoyancy_ramp_iters: the buoyancy ramp (300); t_skin_relax: the skin
    temperature's relaxation (0.25); omega_rad: radiation mode 2's blend (0.05);
    tropopause_layers: cAtmosphereModel::tropopause_layers (jm level indices; default the
    configuration's, the tropopause above the 120 km lid on every row, i.e. im - 1);
    first_iter: the first iter_n (iterations counted from 1, as run_3D_loop counts them);
    checkpoint: the output cadence (cli/config_cond.xml: 20), whose iterations capture the
    momentum-budget terms."""

    def __init__(self, g: GpuAtmosphere, dt: float = 4e-5, buoyancy_ramp_iters: int = 300,
                 t_skin_relax: float = 0.25, omega_rad: float = 0.05, tropopause_layers=None,
                 first_iter: int = 1, checkpoint: int = 20):
        self.g = g
        self.checkpoint = checkpoint
        self.dt = dt
        self.ramp_iters = buoyancy_ramp_iters
        self.t_skin_relax = t_skin_relax
        self.omega_rad = omega_rad
        im, jm, _ = g.shape
        layers = np.full(jm, im - 1.0) if tropopause_layers is None else np.asarray(tropopause_layers, float)
        g.set_tropopause_layers(layers)
        self.iter_n = first_iter
        self.total_iter_count = first_iter - 1

    def iteration(self) -> dict:
        """One iteration; returns what the reference prints: the residuum report, the skin
        temperature and, on moist iterations, the CO2 and water budgets."""
        g = self.g
        it = self.iter_n
        self.total_iter_count += 1
        out = {"iter_n": it}
        if it % 4 == 0:
            g.PressureSolverAtm_run(total_iter_count=self.total_iter_count)
        if it % 2 == 0:
            out["h2o_post_rk4"] = g.water_budget()
            g.SaturationAdjustment_run()
            for n in MOIST_FIELDS_AFTER_SATADJ:
                g.damp_wiggles(n)
            g.ice_scheme()
            for n in ICE_FLUXES:
                g.damp_wiggles(n)
            g.MoistConvection_run(it)
            for n in CONVECTION_FIELDS:
                g.damp_wiggles(n)
            g.moist_caps()
            g.vapour_ceiling()
            out["co2"] = g.co2_column()
            out["h2o"] = g.water_budget()
            g.densities()
            g.forces()
            g.stand_atm_dew_point()
            g.water_vapour_evaporation()
            g.latent_sensible_heat()
            g.turbulence_run()
            for n in TURBULENCE_FIELDS:
                g.damp_wiggles(n)
        g.boundary_conditions()
        ramp = min(1.0, self.total_iter_count / self.ramp_iters) if self.ramp_iters > 0 else 1.0
        budget = 2 if (self.checkpoint > 0 and it % self.checkpoint == 0) else 0
        g.solveRungeKutta_Atmosphere_Turb(self.dt, 1.0, ramp, write_diagnostics=1 | budget)
        g.post_rk4_filters()
        out["residuum"] = g.find_residuum()
        g.storeIntermediateData3D()
        g.radiative_heating(self.omega_rad)
        out["t_skin"] = g.update_skin_temperature(self.t_skin_relax)
        self.iter_n += 1
        return out

    def run(self, n: int) -> list:
        return [self.iteration() for _ in range(n)]
