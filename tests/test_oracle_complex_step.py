"""The oracle's complex-step residual (the CPU reference of the discrete
adjoint): its real part is the oracle residual, and its derivative matches
central differences of the oracle residual on a smooth state.  CPU only."""
import numpy as np
import pytest

from rhodst_b200 import cases
from tests.oracle_lib import ComplexStep, OracleSolver, conservative_array

SCHEMES = ["Kurganov", "HLL", "HLLC", "HLLCP", "AUSM+", "AUSM+up", "AUSM"]


def step_case(flux, limiter):
    vlim = limiter if limiter in ("Venkatakrishnan", "upwind", "linear") else limiter + "V"
    return cases.forward_step_c1().with_options(**{
        "fluxScheme": flux, "interpolationSchemes.reconstruct(rho)": limiter,
        "interpolationSchemes.reconstruct(T)": limiter, "interpolationSchemes.reconstruct(U)": vlim})


def smooth_state(case, seed=3, amp=0.05):
    rng = np.random.default_rng(seed)
    C = case.mesh.C
    k = rng.uniform(1.0, 4.0, size=(5, 3))
    ph = rng.uniform(0, 2 * np.pi, size=5)
    modes = [np.sin(C @ k[i] * np.pi + ph[i]) for i in range(5)]
    p = case.p * (1 + amp * modes[0])
    T = case.T * (1 + amp * modes[1])
    U = case.U.copy()
    U[:, 0] *= 1 + amp * modes[2]
    U[:, 1] += amp * np.abs(case.U[:, 0]).max() * modes[3]
    U[:, 2] += amp * np.abs(case.U[:, 0]).max() * modes[4]
    g = case.options["thermo"]
    rho = p / (g["R"] * T)
    rhoE = rho * ((g["Cp"] - g["R"]) * T + 0.5 * (U ** 2).sum(1))
    return rho, rho[:, None] * U, rhoE


@pytest.mark.parametrize("flux", SCHEMES)
@pytest.mark.parametrize("limiter", ["OSPRE", "Venkatakrishnan", "upwind"])
def test_complex_step_real_part_is_the_oracle_residual(flux, limiter):
    c = step_case(flux, limiter)
    o = OracleSolver(c.mesh, c.bcs, c.options)
    W = smooth_state(c)
    o.set_conservative(*W)
    R = o.residual()
    Rc, _ = ComplexStep(o).residual(conservative_array(W))
    scale = np.abs(R).max(axis=0)
    assert np.all(np.abs(Rc - R).max(axis=0) <= 1e-12 * scale), (flux, limiter)


@pytest.mark.parametrize("flux", ["HLLC", "AUSM+up"])
def test_complex_step_matches_central_differences(flux):
    c = step_case(flux, "linear")
    o = OracleSolver(c.mesh, c.bcs, c.options)
    W = smooth_state(c)
    Wa = conservative_array(W)
    o.set_conservative(*W)
    o.residual()
    rng = np.random.default_rng(1)
    u = rng.uniform(-1, 1, size=Wa.shape) * np.abs(Wa).max(axis=0).clip(1e-3)
    _, dR = ComplexStep(o).residual(Wa, u)
    h = 1e-6
    Rs = []
    for sgn in (1.0, -1.0):
        Wp = Wa + sgn * h * u
        o.set_conservative(Wp[:, 0], Wp[:, 1:4], Wp[:, 4])
        Rs.append(o.residual())
    fd = (Rs[0] - Rs[1]) / (2 * h)
    assert np.abs(fd - dR).max() <= 1e-6 * np.abs(fd).max()
