"""FP64 reductions (mass, steady residual) against numpy and the oracle."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_mass_fp64_and_deviation(cuda, pkg):
    rng = np.random.default_rng(0)
    for shape in ((9, 7, 5), (19, 33, 17, 9), (9, 512, 512)):
        f = rng.random(shape)
        ref = math.fsum(f.ravel().tolist())
        ft = torch.from_numpy(f).cuda()
        assert abs(pkg.mass(ft) - ref) <= 1e-12 * abs(ref)
        Q = shape[0]
        w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4) if Q == 9 else \
            np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
        d = torch.empty(shape, dtype=torch.float32, device="cuda")
        pkg.convert_populations(d, ft, dst_deviation=True)
        assert abs(pkg.mass(d, deviation=True) - ref) <= 1e-6 * abs(ref)
        _ = w


def test_mass_nonfinite_flag(cuda, pkg):
    f = torch.ones((9, 4, 4), dtype=torch.float64, device="cuda")
    f[3, 1, 2] = float("nan")
    with pytest.raises(pkg.KrakenError) as ei:
        pkg.mass(f)
    assert ei.value.code == pkg._lib.KB_ERR_NONFINITE


def test_residual_matches_oracle(cuda, pkg, orc):
    rng = np.random.default_rng(1)
    n = (40, 30)
    ux, uy, uxp, uyp = (rng.standard_normal(n) * 0.01 for _ in range(4))
    solid = (rng.random(n) < 0.2).astype(np.uint8)
    ref = orc.residual(ux, uy, uxp, uyp, solid=solid)
    g = [torch.from_numpy(a).cuda() for a in (ux, uy, uxp, uyp)]
    got = pkg.residual(g[0], g[1], g[2], g[3], is_solid=torch.from_numpy(solid).cuda())
    assert abs(got - ref) <= 1e-13 * ref
    uz, uzp = rng.standard_normal(n) * 0.01, rng.standard_normal(n) * 0.01
    ref3 = orc.residual(ux, uy, uxp, uyp, uz, uzp)
    got3 = pkg.residual(g[0], g[1], g[2], g[3], torch.from_numpy(uz).cuda(),
                        torch.from_numpy(uzp).cuda())
    assert abs(got3 - ref3) <= 1e-13 * ref3
