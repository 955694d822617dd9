"""The fused natural-convection step on deviation storage (f - w_q and
g - w_q T_ref, FP32 collision): one step from a perturbed state equals the
oracle's FP64 step within the storage rounding, on walls and ragged grids;
and over a run it stays closer to the FP64 run than the reference-arithmetic
FP32 step, which stores f and g whole."""
import math

import numpy as np
import pytest
import torch

from oracle import thermal_drivers as td

pytestmark = pytest.mark.gpu

W9 = td.W9
PAR = dict(omega_f=1.0 / (3 * 0.05 + 0.5), omega_T=1.0 / (3 * 0.05 / 0.71 + 0.5), beta_g=2e-5,
           T_ref=0.5, T_hot=1.0, T_cold=0.0)


def _state(Nx, Ny, seed):
    rng = np.random.default_rng(seed)
    f = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, Ny, Nx)))
    T = rng.random((Ny, Nx))
    g = W9[:, None, None] * T[None] * (1 + 0.05 * rng.standard_normal((9, Ny, Nx)))
    return f, g


def _dev_run(pkg, f, g, steps, dtype, sr=False, vt=None, par=None):
    PAR = dict(globals()["PAR"], **(par or {}))
    Ny, Nx = f.shape[1:]
    fi = torch.empty((9, Ny, Nx), dtype=dtype, device="cuda")
    gi = torch.empty_like(fi)
    pkg.convert_populations(fi, torch.from_numpy(f).cuda(), dst_deviation=True)
    gi.copy_(pkg.thermal_deviation(torch.from_numpy(g).cuda(), PAR["T_ref"]).to(dtype))
    fo, go = torch.empty_like(fi), torch.empty_like(gi)
    Temp = torch.empty((Ny, Nx), dtype=torch.float32, device="cuda")
    for _ in range(steps):
        if vt is None:
            pkg.fused_natconv_step_(fo, fi, go, gi, Temp, Nx, Ny, PAR["omega_f"], PAR["omega_T"],
                                    PAR["beta_g"], PAR["T_ref"], PAR["T_hot"], PAR["T_cold"],
                                    deviation=True, stochastic_rounding=sr)
        else:
            pkg.fused_natconv_vt_step_(fo, fi, go, gi, Temp, Nx, Ny, vt[0], vt[1], vt[2],
                                       PAR["omega_T"], PAR["beta_g"], PAR["T_ref"], PAR["T_hot"],
                                       PAR["T_cold"], deviation=True, stochastic_rounding=sr)
        fi, fo, gi, go = fo, fi, go, gi
    fb = torch.empty((9, Ny, Nx), dtype=torch.float64, device="cuda")
    pkg.convert_populations(fb, fi, src_deviation=True)
    gb = pkg.thermal_deviation(gi, PAR["T_ref"], to_deviation=False)
    torch.cuda.synchronize()
    return fb.cpu().numpy(), gb.cpu().numpy(), Temp.double().cpu().numpy()


@pytest.mark.parametrize("Nx,Ny", [(1, 1), (2, 3), (17, 13), (130, 9)])
@pytest.mark.parametrize("dtype,tol", [(torch.float32, 3e-7), (torch.float16, 2e-3),
                                       (torch.bfloat16, 1.6e-2)])
def test_natconv_deviation_step_matches_oracle(cuda, pkg, orc, Nx, Ny, dtype, tol):
    f, g = _state(Nx, Ny, 5)
    fr, gr = np.empty_like(f), np.empty_like(g)
    Tr = np.empty((Ny, Nx))
    orc.fused_natconv_2d(fr, f, gr, g, Tr, PAR["omega_f"], PAR["omega_T"], PAR["beta_g"],
                         PAR["T_ref"], PAR["T_hot"], PAR["T_cold"])
    fb, gb, Tb = _dev_run(pkg, f, g, 1, dtype)
    # errors in units of the weights (the storage rounds deviations of O(w))
    wf = W9[:, None, None]
    assert np.max(np.abs(fb - fr) / wf) < tol
    assert np.max(np.abs(gb - gr) / wf) < tol
    assert np.max(np.abs(Tb - Tr)) < 20 * tol


def test_natconv_vt_deviation_step_matches_oracle(cuda, pkg, orc):
    Nx, Ny = 33, 17
    f, g = _state(Nx, Ny, 6)
    fr, gr = np.empty_like(f), np.empty_like(g)
    Tr = np.empty((Ny, Nx))
    vt = (0.05, 0.0, -math.log(3.0))
    orc.fused_natconv_vt_2d(fr, f, gr, g, Tr, vt[0], vt[1], vt[2], PAR["omega_T"], PAR["beta_g"],
                            PAR["T_ref"], PAR["T_hot"], PAR["T_cold"])
    fb, gb, _ = _dev_run(pkg, f, g, 1, torch.float32, vt=vt)
    wf = W9[:, None, None]
    assert np.max(np.abs(fb - fr) / wf) < 3e-7
    assert np.max(np.abs(gb - gr) / wf) < 3e-7


def test_natconv_deviation_storage_beats_whole_fp32(cuda, pkg):
    """64^2 cavity, Ra = 1e4 parameters, 20 000 steps from the reference's
    initial state: velocity and temperature of the FP32 deviation run are
    closer to the FP64 run than those of the FP32 run that stores f and g
    whole, and within stated bounds; FP16 deviations with stochastic
    rounding stay within a looser bound."""
    N, steps = 64, 20000
    p = pkg.drivers.natconv_parameters(N, 1e4, 0.71)
    f0 = np.stack([W9[q] * np.ones((N, N)) for q in range(9)])
    g0 = pkg.drivers.natconv_initial_g(N)
    par = dict(omega_f=p["omega_f"], omega_T=p["omega_T"], beta_g=p["beta_g"], T_ref=p["T_ref"])

    def whole(dtype):
        fi = torch.from_numpy(f0).to("cuda", dtype)
        gi = torch.from_numpy(g0).to("cuda", dtype)
        fo, go = torch.empty_like(fi), torch.empty_like(gi)
        Temp = torch.empty((N, N), dtype=dtype, device="cuda")
        for _ in range(steps):
            pkg.fused_natconv_step_(fo, fi, go, gi, Temp, N, N, par["omega_f"], par["omega_T"],
                                    par["beta_g"], par["T_ref"], 1.0, 0.0)
            fi, fo, gi, go = fo, fi, go, gi
        rho, ux, uy = (torch.empty((N, N), dtype=dtype, device="cuda") for _ in range(3))
        pkg.compute_macroscopic_2d_(rho, ux, uy, fi)
        pkg.compute_temperature_2d_(Temp, gi)
        return (np.stack([ux.double().cpu().numpy(), uy.double().cpu().numpy()]),
                Temp.double().cpu().numpy())

    def dev(dtype, sr=False):
        fb, gb, _ = _dev_run(pkg, f0, g0, steps, dtype, sr, par=par)
        rho = fb.sum(0)
        ux = (fb[1] - fb[3] + fb[5] - fb[6] - fb[7] + fb[8]) / rho
        uy = (fb[2] - fb[4] + fb[5] + fb[6] - fb[7] - fb[8]) / rho
        return np.stack([ux, uy]), gb.sum(0)

    u64, T64 = whole(torch.float64)
    u32, T32 = whole(torch.float32)
    ud, Td = dev(torch.float32)
    uh, Th = dev(torch.float16, sr=True)

    def l2(u):
        return math.sqrt(np.sum((u - u64) ** 2) / np.sum(u64 ** 2))

    # u here is sum(c f) / rho of the stored populations in every run (the
    # moment pass, without the Guo half-force term)
    e32, ed, eh = l2(u32), l2(ud), l2(uh)
    assert ed < e32 and ed < 1e-4, (ed, e32)
    assert np.max(np.abs(Td - T64)) < np.max(np.abs(T32 - T64)) + 1e-7
    assert eh < 5e-3, eh
