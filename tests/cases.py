"""Input decks used by the parity tests and the benchmark (reference keys)."""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden_cases.json")))


def golden_input(name):
    return GOLDEN[name]["input"]


# small explicit-solver case with a moving, spread beam (exercises beam push, slipping,
# Reflecting plasma boundary and an odd grid -> node-centred multigrid)
EXPLICIT_MOVING = """
amr.n_cell = 33 33 40
hipace.normalized_units = 1
max_step = 2
hipace.dt = 20
hipace.depos_order_xy = 2
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -6. -6. -8.
geometry.prob_hi =  6.  6.  4.
beams.names = beam
beam.injection_type = fixed_weight
beam.num_particles = 20000
beam.position_mean = 0. 0. 0.
beam.position_std = 0.5 0.5 1.0
beam.density = 5.
beam.u_mean = 0. 0. 2000.
beam.u_std = 3. 3. 10.
beam.n_subcycles = 4
random_seed = 7
plasmas.names = plasma
plasma.density(x,y,z) = 1. + 0.05*(x*x+y*y)
plasma.ppc = 1 1
plasma.element = electron
hipace.MG_tolerance_rel = 1e-12
"""

# predictor-corrector solver, 3 fixed iterations (the configuration of the CPU-runnable case)
PC_SMALL = """
amr.n_cell = 32 32 40
hipace.normalized_units = 1
max_step = 2
hipace.dt = 10
hipace.bxby_solver = predictor-corrector
hipace.predcorr_max_iterations = 3
hipace.predcorr_B_error_tolerance = -1
boundary.field = Dirichlet
boundary.particle = Periodic
geometry.prob_lo = -8. -8. -12.
geometry.prob_hi =  8.  8.   6.
beams.names = beam
beam.injection_type = fixed_weight
beam.num_particles = 20000
beam.position_mean = 0. 0. 0.
beam.position_std = 0.5 0.5 1.41
beam.density = 0.5
beam.u_mean = 0. 0. 1000.
beam.u_std = 0. 0. 0.
random_seed = 3
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
"""


# adjoint of one step: driver + witness ("can" profile on [-7, -5]), objective on the witness
# slices, 16 witness-profile knots and 4 plasma-density knots; moderate driver so that no plasma
# particle crosses the QSA filter (the objective is then differentiable in every parameter)
ADJOINT_SMALL = """
amr.n_cell = 32 32 64
hipace.normalized_units = 1
max_step = 0
hipace.dt = 20
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -6. -6. -10.
geometry.prob_hi =  6.  6.  4.
beams.names = driver witness
driver.injection_type = fixed_weight
driver.num_particles = 20000
driver.position_mean = 0. 0. 0.
driver.position_std = 0.3 0.3 1.0
driver.density = 1.
driver.u_mean = 0. 0. 2000.
driver.u_std = 0.0333 0.0333 0.
witness.injection_type = fixed_weight
witness.profile = can
witness.zmin = -7.
witness.zmax = -5.
witness.num_particles = 5000
witness.position_mean = 0. 0. -6.
witness.position_std = 0.1 0.1 1.
witness.density = 5.
witness.u_mean = 0. 0. 2000.
random_seed = 11
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
hipace.MG_tolerance_rel = 1e-13
adjoint.witness = witness
adjoint.profile_zeta = -7. -5.
adjoint.n_profile_knots = 16
adjoint.density_z = -10. 10.
adjoint.n_density_knots = 4
adjoint.objective_zeta = -7. -5.
adjoint.checkpoint_interval = 16
"""


# fixed_weight_pdf witness (BeamParticleContainer.cpp:200-249): trapezoidal current profile on
# [-7, -5], tilted centroid, z-dependent width and energy chirp
PDF_BEAM = """
amr.n_cell = 32 32 64
hipace.normalized_units = 1
max_step = 1
hipace.dt = 20
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -6. -6. -10.
geometry.prob_hi =  6.  6.  4.
beams.names = wit
wit.injection_type = fixed_weight_pdf
wit.pdf = "(z<-5)*(z>-7)*(1+0.3*(z+6))"
wit.position_mean = "0.1*(z+6)" "0."
wit.position_std = "0.1+0.02*(z+6)" "0.1"
wit.u_mean = "0." "0." "2000.*(1+0.01*(z+6))"
wit.u_std = "1." "1." "5."
wit.num_particles = 200000
wit.density = 5.
random_seed = 3
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
hipace.MG_tolerance_rel = 1e-12
"""


def adjoint_beams(seed=1):
    """Seeded driver and witness particles for ADJOINT_SMALL (same arrays for oracle and GPU)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n, m = 20000, 5000
    driver = {"x": rng.normal(0, 0.3, n), "y": rng.normal(0, 0.3, n), "z": rng.normal(0, 1.0, n),
              "w": np.full(n, 0.05), "ux": rng.normal(0, 0.0333, n), "uy": rng.normal(0, 0.0333, n),
              "uz": np.full(n, 2000.), "id": np.arange(1, n + 1, dtype=np.int64)}
    witness = {"x": rng.normal(0, 0.1, m), "y": rng.normal(0, 0.1, m), "z": rng.uniform(-7., -5., m),
               "w": np.full(m, 0.01), "ux": np.zeros(m), "uy": np.zeros(m), "uz": np.full(m, 2000.),
               "id": np.arange(1, m + 1, dtype=np.int64)}
    return driver, witness


def adjoint_knots(seed=4321, n_profile=16, n_density=4):
    """Witness knots 0.5 +- 10 % seeded noise, density knots 1."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return np.concatenate([0.5 * (1 + 0.1 * rng.uniform(-1, 1, n_profile)), np.ones(n_density)])


def config(name):
    """The five benchmark workloads, restated in reference keys (seeded synthetic beams)."""
    if name == "linear_wake_64":
        return """
amr.n_cell = 64 64 100
hipace.normalized_units = 1
max_step = 10
hipace.dt = 10
hipace.bxby_solver = predictor-corrector
hipace.predcorr_max_iterations = 3
hipace.predcorr_B_error_tolerance = -1
boundary.field = Dirichlet
boundary.particle = Periodic
geometry.prob_lo = -8. -8. -12.
geometry.prob_hi =  8.  8.   6.
beams.names = beam
beam.injection_type = fixed_weight
beam.num_particles = 100000
beam.position_mean = 0. 0. 0.
beam.position_std = 0.5 0.5 1.41
beam.density = 0.01
beam.u_mean = 0. 0. 1000.
beam.u_std = 0. 0. 0.
random_seed = 1234
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
"""
    if name == "blowout_255":
        return """
amr.n_cell = 255 255 256
hipace.normalized_units = 1
max_step = 19
hipace.dt = 20
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -6. -6. -8.
geometry.prob_hi =  6.  6.  4.
beams.names = beam
beam.injection_type = fixed_weight
beam.num_particles = 1000000
beam.position_mean = 0. 0. 0.
beam.position_std = 0.3 0.3 1.0
beam.density = 10.
beam.u_mean = 0. 0. 2000.
beam.u_std = 0.0333333333333 0.0333333333333 0.
random_seed = 1234
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
"""
    if name == "channel_1023":
        return """
amr.n_cell = 1023 1023 1024
hipace.normalized_units = 1
max_step = 4
hipace.dt = 20
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -8. -8. -10.
geometry.prob_hi =  8.  8.   4.
beams.names = beam
beam.injection_type = fixed_weight
beam.num_particles = 4000000
beam.position_mean = 0. 0. 0.
beam.position_std = 0.3 0.3 1.0
beam.density = 10.
beam.u_mean = 0. 0. 2000.
beam.u_std = 0.0333333333333 0.0333333333333 0.
random_seed = 1234
plasmas.names = plasma
plasma.density(x,y,z) = 1. + 0.05*(x*x+y*y)
plasma.ppc = 2 2
plasma.element = electron
"""
    if name == "large_2047":
        # large forward (and adjoint) workload: 2047^2 x 2048 slices, 4.2M plasma particles,
        # 1e7 driver and a 2e6 witness with the knot parameterisation of beam_loading_255
        return """
amr.n_cell = 2047 2047 2048
hipace.normalized_units = 1
max_step = 0
hipace.dt = 20
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -10. -10. -12.
geometry.prob_hi =  10.  10.   4.
beams.names = driver witness
driver.injection_type = fixed_weight
driver.num_particles = 10000000
driver.position_mean = 0. 0. 0.
driver.position_std = 0.3 0.3 1.0
driver.density = 10.
driver.u_mean = 0. 0. 2000.
driver.u_std = 0.0333333333333 0.0333333333333 0.
witness.injection_type = fixed_weight
witness.profile = can
witness.zmin = -7.
witness.zmax = -5.
witness.num_particles = 2000000
witness.position_mean = 0. 0. -6.
witness.position_std = 0.1 0.1 1.
witness.density = 5.
witness.u_mean = 0. 0. 2000.
random_seed = 1234
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
adjoint.witness = witness
adjoint.profile_zeta = -7. -5.
adjoint.n_profile_knots = 64
adjoint.density_z = -100. 100.
adjoint.n_density_knots = 8
adjoint.objective_zeta = -7. -5.
adjoint.checkpoint_interval = 64
"""
    if name == "beam_loading_255":
        # adjoint workload: the blowout grid extended to 512 slices, driver plus a witness whose
        # current profile is set by 64 knots on [-7, -5], 8 plasma-density knots, objective on
        # the witness slices, checkpoints every 32 slices
        return """
amr.n_cell = 255 255 512
hipace.normalized_units = 1
max_step = 0
hipace.dt = 20
boundary.field = Dirichlet
boundary.particle = Reflecting
geometry.prob_lo = -6. -6. -10.
geometry.prob_hi =  6.  6.  4.
beams.names = driver witness
driver.injection_type = fixed_weight
driver.num_particles = 1000000
driver.position_mean = 0. 0. 0.
driver.position_std = 0.3 0.3 1.0
driver.density = 10.
driver.u_mean = 0. 0. 2000.
driver.u_std = 0.0333333333333 0.0333333333333 0.
witness.injection_type = fixed_weight
witness.profile = can
witness.zmin = -7.
witness.zmax = -5.
witness.num_particles = 500000
witness.position_mean = 0. 0. -6.
witness.position_std = 0.1 0.1 1.
witness.density = 5.
witness.u_mean = 0. 0. 2000.
random_seed = 1234
plasmas.names = plasma
plasma.density(x,y,z) = 1.
plasma.ppc = 1 1
plasma.element = electron
adjoint.witness = witness
adjoint.profile_zeta = -7. -5.
adjoint.n_profile_knots = 64
adjoint.density_z = -100. 100.
adjoint.n_density_knots = 8
adjoint.objective_zeta = -7. -5.
adjoint.checkpoint_interval = 32
"""
    raise KeyError(name)


# power-of-two-plus-one grids take the FFT path of the Poisson solver (2(n+1) = 128)
EXPLICIT_FFT = EXPLICIT_MOVING.replace("amr.n_cell = 33 33 40", "amr.n_cell = 63 63 48")
PC_FFT = PC_SMALL.replace("amr.n_cell = 32 32 40", "amr.n_cell = 63 63 40")
