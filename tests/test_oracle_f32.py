"""The single-precision restatement of the fused D3Q19 TRT step (the
reference's T = Float32 path, timed as the FP32 CPU baseline) follows the
FP64 restatement to single-precision rounding, with walls and solids."""
import numpy as np


def test_f32_trt_follows_f64(orc):
    rng = np.random.default_rng(3)
    Nx, Ny, Nz = 11, 7, 9
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    f = w[:, None, None, None] * (1 + 0.02 * rng.standard_normal((19, Nz, Ny, Nx)))
    solid = (rng.random((Nz, Ny, Nx)) < 0.1).astype(np.uint8)
    sp, sm = orc.trt_rates(0.02, 0.25)
    for per in ((0, 0, 0), (1, 1, 1), (1, 0, 1)):
        a, b = f.copy(), np.empty_like(f)
        a32, b32 = f.astype(np.float32), np.empty(f.shape, np.float32)
        m64 = [np.empty((Nz, Ny, Nx)) for _ in range(4)]
        m32 = [np.empty((Nz, Ny, Nx), np.float32) for _ in range(4)]
        for _ in range(20):
            orc.fused_trt_3d(b, a, m64, solid, sp, sm, per)
            orc.fused_trt_3d_f32(b32, a32, m32, solid, sp, sm, per)
            a, b, a32, b32 = b, a, b32, a32
        assert np.abs(a32 - a).max() < 2e-6
        assert all(np.abs(x - y).max() < 2e-6 for x, y in zip(m32, m64))
