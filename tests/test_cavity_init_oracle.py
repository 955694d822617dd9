"""CPU pin of the consistent-initialisation restatement: with the velocity
held at the populations' own velocity, the fixed-velocity MRT collision is
the reference MRT collision (collide_mrt_2d!, via the C oracle) up to the
rounding of rho * (j / rho)."""
import numpy as np

from oracle import cavity_init_oracle as CI
from oracle import oracle as orc

W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def test_fixed_velocity_collision_is_mrt_at_own_velocity():
    rng = np.random.default_rng(0)
    f = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, 13, 17)))
    rho, ux, uy = orc.macroscopic_2d(f)
    ref = f.copy()
    orc.collide_mrt_2d(ref, None, 0.03)
    got = CI.mrt_collide_fixed_u(f, ux, uy, 0.03)
    assert np.max(np.abs(got - ref)) < 1e-15


def test_fixed_velocity_collision_sets_momentum():
    rng = np.random.default_rng(1)
    f = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, 13, 17)))
    ux, uy = 0.05 * rng.standard_normal((2, 13, 17))
    out = CI.mrt_collide_fixed_u(f, ux, uy, 0.03)
    rho, jx, jy = orc.macroscopic_2d(out)
    rho0 = f.sum(axis=0)
    assert np.allclose(rho, rho0, atol=1e-15)
    assert np.allclose(jx, ux, atol=1e-14) and np.allclose(jy, uy, atol=1e-14)
