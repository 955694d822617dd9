"""A CUDA run resumed from a checkpoint continues bit for bit: D3Q19 TRT on
FP16 deviation storage (the staged kernel at Nx = 256) and on FP64, and the
D2Q9 cavity step on FP64.  The 16-bit populations travel through the file as
float32 values, which round-trips them exactly."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


@pytest.mark.parametrize("dtype,deviation", [(torch.float16, True), (torch.bfloat16, True),
                                             (torch.float64, False)])
def test_resumed_3d_run_is_bit_identical(cuda, pkg, tmp_path, dtype, deviation):
    Nx, Ny, Nz, n1, n2 = 256, 6, 8, 7, 9
    rng = np.random.default_rng(4)
    f = W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19, Nz, Ny, Nx)))
    a = torch.empty((19, Nz, Ny, Nx), dtype=dtype, device="cuda")
    pkg.convert_populations(a, torch.from_numpy(f).cuda(), dst_deviation=deviation)
    start = a.clone()

    def run(x, n):
        y = torch.empty_like(x)
        for _ in range(n):
            pkg.fused_trt_step_3d_(y, x, None, None, None, None, None, Nx, Ny, Nz, 0.02, 0.25,
                                   periodic=(1, 1, 1), deviation=deviation)
            x, y = y, x
        return x

    ref = run(start.clone(), n1 + n2)
    mid = run(start.clone(), n1)
    p = tmp_path / "tgv.ckpt"
    pkg.checkpoint.save_checkpoint_lbm(p, mid, n1, deviation=deviation,
                                       parameters={"nu": 0.02, "Lambda": 0.25})
    g, cycle, _ = pkg.checkpoint.load_checkpoint_lbm(p, torch.empty_like(a), deviation=deviation)
    assert cycle == n1 and g.dtype == dtype and torch.equal(g, mid)
    out = run(g, n2)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)


def test_resumed_2d_cavity_is_bit_identical(cuda, pkg, tmp_path):
    Nx = Ny = 96
    om, u = 1.0 / (3 * 0.02 + 0.5), 0.1
    cfg = pkg.LBMConfig.d2q9(Nx, Ny, 0.02, u, 0)
    st = pkg.initialize_2d(cfg)
    rho, ux, uy = st["rho"], st["ux"], st["uy"]

    def run(x, n):
        y = torch.empty_like(x)
        for _ in range(n):
            pkg.cavity_step_2d_(y, x, rho, ux, uy, None, Nx, Ny, om, u)
            x, y = y, x
        return x

    f0 = st["f_in"].clone()
    ref = run(f0.clone(), 50)
    mid = run(f0.clone(), 20)
    p = tmp_path / "cavity.ckpt"
    pkg.checkpoint.save_checkpoint_lbm(p, mid, 20, moments={"ux": ux, "uy": uy})
    g, cycle, mom = pkg.checkpoint.load_checkpoint_lbm(p, torch.empty_like(f0))
    assert set(mom) == {"ux", "uy"}
    assert torch.equal(run(g, 50 - cycle), ref)


@pytest.mark.parametrize("variant", [0, 2])
def test_resumed_stochastic_rounding_run_is_bit_identical(cuda, pkg, tmp_path, variant):
    """FP16 deviations with stochastic rounding: the checkpoint records the
    rounding-bit counter and the restore sets it back, so the resumed run
    equals the uninterrupted one even after unrelated stochastic-rounding
    launches in between.  Variant 0 is the staged kernel (it advances the
    counter itself), 2 the pair kernel (a counter launch after each step)."""
    Nx, Ny, Nz, n1, n2 = 256, 6, 8, 6, 7
    rng = np.random.default_rng(9)
    f = W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19, Nz, Ny, Nx)))
    a = torch.empty((19, Nz, Ny, Nx), dtype=torch.float16, device="cuda")
    pkg.convert_populations(a, torch.from_numpy(f).cuda(), dst_deviation=True)
    start = a.clone()
    pkg.set_trt3d_variant(variant)
    try:
        def run(x, n):
            y = torch.empty_like(x)
            for _ in range(n):
                pkg.fused_trt_step_3d_(y, x, None, None, None, None, None, Nx, Ny, Nz, 0.02, 0.25,
                                       periodic=(1, 1, 1), deviation=True,
                                       stochastic_rounding=True)
                x, y = y, x
            return x

        pkg.set_stochastic_seed(1234)
        ref = run(start.clone(), n1 + n2)
        pkg.set_stochastic_seed(1234)
        mid = run(start.clone(), n1)
        p = tmp_path / "tgv_sr.ckpt"
        pkg.checkpoint.save_checkpoint_lbm(p, mid, n1, deviation=True, stochastic_rounding=True)
        assert pkg.checkpoint.read_checkpoint(p).run_control["sr_epoch"] == 1234 + n1
        run(start.clone(), 5)  # other stochastic-rounding work moves the counter on
        g, cycle, _ = pkg.checkpoint.load_checkpoint_lbm(p, torch.empty_like(a), deviation=True,
                                                         stochastic_rounding=True)
        assert cycle == n1 and torch.equal(g, mid)
        out = run(g, n2)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        # a round-to-nearest restore of a stochastic-rounding checkpoint is refused
        with pytest.raises(pkg.checkpoint.CheckpointError):
            pkg.checkpoint.load_checkpoint_lbm(p, torch.empty_like(a), deviation=True)
    finally:
        pkg.set_trt3d_variant(0)
