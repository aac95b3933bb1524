"""Known answers of the physics, independent of any implementation:

- below the onset of convection (Ra = 1e3 < 1708) a perturbed conduction
  state relaxes to steady conduction: Nu = 1 at both plates and in the bulk
  (to the O(1e-3) offset of the discrete wall rules);
- above it (Ra = 1e5) convection sets in and reaches a statistically steady
  state whose heat flux is the same through both plates and the bulk.

The oracle (CPU) for the first; the engine (GPU) for both, in every storage
format that runs the case."""
import numpy as np
import pytest


def _steady_conduction(obs_a, obs_b, tol, drift=1e-6):
    for k in ("nu_bulk", "nu_top", "nu_bottom"):
        assert abs(obs_b[k] - 1.0) <= tol, (k, obs_b[k])
        assert abs(obs_b[k] - obs_a[k]) <= drift, k    # no longer changing (to storage rounding)


def test_oracle_subcritical_conduction(oracle_mod):
    o = oracle_mod.Oracle(oracle_mod.make_params(16, 16, 8, rayleigh=1e3, prandtl=0.71, periodic_sides=True))
    o.init_conduction(7, 1e-3)
    o.step(4000)
    a = o.observables()
    o.step(1000)
    _steady_conduction(a, o.observables(), 3e-3)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f64", "f32", "f16s", "bf16s"])
def test_subcritical_conduction(lbm, storage):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = lbm.make_params(32, 16, 32, rayleigh=1e3, prandtl=0.71, sides=lbm.SIDES_PERIODIC, storage=storage)
    with lbm.Case(p) as c:
        c.init_conduction(7, 1e-3)
        c.step(4000)
        a = c.observables()
        c.step(1000)
        b = c.observables()
    # 16-bit storage keeps g/w relative to the conduction profile, so the
    # plate gradients of this state are resolved (with one constant shift
    # the plate Nu were off by ~4% in FP16S and ~20% in BF16S here)
    tol, drift = {"f64": (3e-3, 1e-6), "f32": (3e-3, 1e-6), "f16s": (4e-3, 1e-5), "bf16s": (1e-2, 1e-3)}[storage]
    _steady_conduction(a, b, tol, drift)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["f32", "f16s"])
def test_supercritical_convection_balances(lbm, storage):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = lbm.make_params(32, 16, 8, rayleigh=1e5, prandtl=0.71, sides=lbm.SIDES_PERIODIC, storage=storage)
    with lbm.Case(p) as c:
        c.init_conduction(7, 1e-3)
        c.step(14000)
        series = c.step_observed(6000)
    nu = {k: np.mean([s[k] for s in series]) for k in ("nu_bulk", "nu_top", "nu_bottom")}
    assert nu["nu_bulk"] > 3.0, nu                          # convecting
    assert abs(nu["nu_top"] - nu["nu_bottom"]) <= 0.05 * nu["nu_bulk"], nu
    assert abs(nu["nu_bulk"] - 0.5 * (nu["nu_top"] + nu["nu_bottom"])) <= 0.1 * nu["nu_bulk"], nu
