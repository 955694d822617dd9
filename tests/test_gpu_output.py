"""Asynchronous snapshots of device fields: the files and callbacks carry the
fields of exactly the requested steps, as a synchronous copy would."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _reference_fields(pkg, steps, every, N=48):
    got = {}

    def hook(step, f):
        if step % every == 0:
            torch.cuda.synchronize()
            got[step] = (f["rho"].cpu().numpy().copy(), f["velocity"][0].cpu().numpy().copy(),
                         f["velocity"][1].cpu().numpy().copy())
    cfg = pkg.LBMConfig.d2q9(N, N, 0.05, 0.1, steps)
    pkg.run_cavity_2d(cfg, on_step=hook)
    return got


def test_async_vtk_and_callback_match_sync_copies(cuda, pkg, tmp_path):
    N, steps = 48, 300
    ref = _reference_fields(pkg, steps, 50, N)
    seen = {}

    def cb(step, f):
        seen[step] = (f["rho"].copy(), f["velocity"][0].copy())
    out = pkg.output.StepOutput(N, N, None, 1.0, tmp_path, vtk_every=100, callback=cb,
                                callback_every=50, name="cav")
    cfg = pkg.LBMConfig.d2q9(N, N, 0.05, 0.1, steps)
    pkg.run_cavity_2d(cfg, on_step=out)
    out.close()
    assert sorted(seen) == [50, 100, 150, 200, 250, 300]
    for s, (rho, ux) in seen.items():
        assert np.array_equal(rho, ref[s][0]) and np.array_equal(ux, ref[s][1])
    for s in (100, 200, 300):
        d = pkg.output.read_vtr(tmp_path / f"snapshot_{s:07d}.vtr")
        assert np.array_equal(d["rho"], ref[s][0].reshape(-1))
        assert np.array_equal(d["velocity"][:, 0], ref[s][1].reshape(-1))
        assert np.array_equal(d["velocity"][:, 1], ref[s][2].reshape(-1))
    assert (tmp_path / "cav.pvd").exists()


def test_run_simulation_writes_series(cuda, pkg, tmp_path):
    text = """
Simulation cav D2Q9
Domain L = 1 x 1  N = 32 x 32
Physics nu = 0.05
Boundary north velocity(ux = 0.1)
Boundary south wall
Boundary east wall
Boundary west wall
Run 200 steps
"""
    calls = []
    r = pkg.krk.run_simulation(pkg.krk.parse_kraken(text), output_dir=tmp_path, vtk_every=100,
                               callback=lambda s, f: calls.append(s), callback_every=40)
    assert sorted(calls) == [40, 80, 120, 160, 200]
    d = pkg.output.read_vtr(tmp_path / "snapshot_0000200.vtr")
    assert np.array_equal(d["rho"], r["rho"].reshape(-1))
    assert (tmp_path / "cav.pvd").exists()
