"""The oracle's regularised collision (Latt and Chopard 2006), the checker of
the engine's LBM_COLLISION_REGULARIZED option (the reference has BGK only).

- at tau_f = tau_g = 1 both models are feq + force, so regularised and BGK
  runs agree to rounding;
- total mass is conserved in the closed box (the projection adds no mass);
- away from tau = 1 the two models differ (the option is not a no-op), while
  the conduction state's observables stay close.
"""
import numpy as np
import pytest

from helpers import relerr


def _pair(oracle_mod, lx, ly, lz, ra, pr, periodic, seed=5, amp=1e-2):
    p = oracle_mod.make_params(lx, ly, lz, rayleigh=ra, prandtl=pr, periodic_sides=periodic)
    a, b = oracle_mod.Oracle(p), oracle_mod.Oracle(p)
    b.set_collision("regularized")
    assert a.collision == "bgk" and b.collision == "regularized"
    for o in (a, b):
        o.init_conduction(seed, amp)
    return p, a, b


@pytest.mark.parametrize("periodic", [True, False])
def test_tau_one_equals_bgk(oracle_mod, periodic):
    ly = 12
    ra = (0.6 * ly) ** 2            # nu = u0 LY / sqrt(Ra / Pr) = 1/6 at Pr = 1: tau_f = tau_g = 1
    p, a, b = _pair(oracle_mod, 10, ly, 8, ra, 1.0, periodic)
    assert abs(p.tau - 1.0) < 1e-14 and abs(p.tauc - 1.0) < 1e-14
    for o in (a, b):
        o.step(30)
    for k in ("f", "g", "phi", "uy"):
        assert relerr(b.field(k), a.field(k)) <= 1e-13, k


def test_mass_conserved_closed_box(oracle_mod):
    p, a, b = _pair(oracle_mod, 10, 12, 8, 1e6, 0.71, False)
    m0 = b.field("rho").sum()
    b.step(300)
    assert abs(b.field("rho").sum() - m0) < 1e-13
    assert b.observables()["diverged"] == 0.0


def test_differs_from_bgk_away_from_tau_one(oracle_mod):
    p, a, b = _pair(oracle_mod, 10, 12, 8, 1e6, 0.71, True)
    for o in (a, b):
        o.step(50)
    assert relerr(b.field("f"), a.field("f")) > 1e-6
    oa, ob = a.observables(), b.observables()
    assert abs(oa["phi_mean"] - ob["phi_mean"]) < 1e-3
