"""Snapshots and checkpoint files of the plain LBM (host logic, CPU).

The content rules and the write protocol follow the reference's state
contract (src/platform/state.jl:139-230, src/io/checkpoint_hdf5.jl:111-147):
invalid names, keys, value and element types are refused; non-finite arrays
are refused and leave an existing checkpoint untouched; the previous file
survives as .prev; damaged and truncated files raise CheckpointError; a run
resumed from a checkpoint continues bit for bit (oracle steps)."""
import os
import zipfile

import numpy as np
import pytest
import torch

W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


@pytest.fixture()
def ck(pkg):
    return pkg.checkpoint


def _snap(ck, cycle=3, **kw):
    base = dict(fields={"f": np.arange(12, dtype=np.float64).reshape(3, 4),
                        "block1/mask": np.array([True, False])},
                series={"residual": np.array([1e-3, 1e-4], dtype=np.float32)},
                scalars={"t": 0.5}, identity={"Nx": 4, "lattice": "D2Q9"},
                run_control={"horizon": float("inf"), "backend": None},
                parameters={"nu": 0.02}, derived={"omega": 1.5})
    base.update(kw)
    return ck.StateSnapshot("lbm_plain", 1, cycle, **base)


@pytest.mark.parametrize("kw,what", [
    (dict(fields={"a/": np.zeros(2)}), "invalid name"),
    (dict(fields={"a/../b": np.zeros(2)}), "invalid name"),
    (dict(fields={"a": np.zeros(2), "a/b": np.zeros(2)}), "prefix"),
    (dict(fields={"a": np.zeros(2, dtype=np.float16)}), "element type"),
    (dict(fields={"a": np.zeros((), dtype=np.float64)}), "zero-dimensional"),
    (dict(series={"s": np.zeros((2, 2))}), "vector"),
    (dict(scalars={"a/b": 1}), "invalid key"),
    (dict(scalars={"keys": 1}), "invalid key"),
    (dict(scalars={"x": None}), "not allowed"),
    (dict(derived={"x": [1, 2]}), "not allowed"),
])
def test_invalid_content_is_refused(ck, kw, what):
    with pytest.raises(ck.CheckpointError, match=what):
        _snap(ck, **kw)


def test_negative_cycle_and_empty_solver_are_refused(ck):
    with pytest.raises(ck.CheckpointError, match="cycle"):
        _snap(ck, cycle=-1)
    with pytest.raises(ck.CheckpointError, match="solver"):
        ck.StateSnapshot("", 1, 0)


def test_round_trip_and_previous_generation(ck, tmp_path):
    p = tmp_path / "run.ckpt"
    a = _snap(ck, cycle=10)
    ck.write_checkpoint(p, a)
    b = _snap(ck, cycle=20, fields={"f": np.ones((3, 4))})
    ck.write_checkpoint(p, b)
    got, prev = ck.read_checkpoint(p), ck.read_checkpoint(str(p) + ".prev")
    assert got.cycle == 20 and prev.cycle == 10
    assert np.array_equal(prev.fields["f"], a.fields["f"])
    assert prev.fields["block1/mask"].dtype == np.bool_
    assert np.array_equal(got.series["residual"], a.series["residual"])
    assert got.run_control == {"horizon": float("inf"), "backend": None}
    assert got.identity == a.identity and got.derived == a.derived
    assert ck.checkpoint_info(p)["cycle"] == 20
    assert not os.path.exists(str(p) + ".tmp")


def test_non_finite_state_never_replaces_a_checkpoint(ck, tmp_path):
    p = tmp_path / "run.ckpt"
    ck.write_checkpoint(p, _snap(ck, cycle=5))
    bad = np.ones((3, 4))
    bad[1, 2] = np.nan
    with pytest.raises(ck.CheckpointError, match=r"fields/f: non-finite value nan at index \(1, 2\)"):
        ck.write_checkpoint(p, _snap(ck, cycle=6, fields={"f": bad}))
    assert ck.read_checkpoint(p).cycle == 5
    assert not os.path.exists(str(p) + ".prev")


def test_damaged_and_truncated_files_are_refused(ck, tmp_path):
    p = tmp_path / "run.ckpt"
    ck.write_checkpoint(p, _snap(ck, fields={"f": np.linspace(0, 1, 4096)}))
    raw = bytearray(p.read_bytes())
    with zipfile.ZipFile(p) as z:
        info = z.getinfo("fields/f.npy")
    damaged = tmp_path / "damaged.ckpt"
    raw2 = bytearray(raw)
    raw2[info.header_offset + 200] ^= 0xFF  # inside the stored array bytes
    damaged.write_bytes(bytes(raw2))
    with pytest.raises(ck.CheckpointError):
        ck.read_checkpoint(damaged)
    truncated = tmp_path / "truncated.ckpt"
    truncated.write_bytes(bytes(raw[: len(raw) // 2]))
    with pytest.raises(ck.CheckpointError):
        ck.read_checkpoint(truncated)
    foreign = tmp_path / "foreign.ckpt"
    foreign.write_bytes(b"not a checkpoint")
    with pytest.raises(ck.CheckpointError):
        ck.checkpoint_info(foreign)


def test_check_compatible(ck):
    s = _snap(ck)
    ck.check_compatible(s, solver="lbm_plain", schema_version=1,
                        identity={"Nx": 4, "lattice": "D2Q9"})
    with pytest.raises(ck.CheckpointError, match="solver"):
        ck.check_compatible(s, solver="ehd_ec", schema_version=1, identity={})
    with pytest.raises(ck.CheckpointError, match="schema_version"):
        ck.check_compatible(s, solver="lbm_plain", schema_version=2, identity={})
    with pytest.raises(ck.CheckpointError, match="identity/Nx"):
        ck.check_compatible(s, solver="lbm_plain", schema_version=1,
                            identity={"Nx": 8, "lattice": "D2Q9"})
    with pytest.raises(ck.CheckpointError, match="identity/Nx"):  # type differs
        ck.check_compatible(s, solver="lbm_plain", schema_version=1,
                            identity={"Nx": 4.0, "lattice": "D2Q9"})
    with pytest.raises(ck.CheckpointError, match="not expected"):
        ck.check_compatible(s, solver="lbm_plain", schema_version=1, identity={"Nx": 4})
    ck.check_compatible(s, solver="lbm_plain", schema_version=1,
                        identity={"Nx": 4, "lattice": "D2Q9", "Ny": 3},
                        identity_defaults={"Ny": 3})


def test_resumed_run_continues_bit_for_bit(pkg, orc, ck, tmp_path):
    """Oracle fused BGK on a walled 24 x 17 grid with solids: 30 steps, or 13
    steps + checkpoint + restore into fresh buffers + 17 steps."""
    Nx, Ny, om = 24, 17, 1.0 / (3 * 0.02 + 0.5)
    rng = np.random.default_rng(2)
    f0 = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, Ny, Nx)))
    m = (rng.random((Ny, Nx)) < 0.1).astype(np.uint8)

    def run(f, n):
        g = np.empty_like(f)
        rho, ux, uy = (np.empty((Ny, Nx)) for _ in range(3))
        for _ in range(n):
            orc.fused_bgk_2d(g, f, rho, ux, uy, m, om)
            f, g = g, f
        return f, (rho, ux, uy)

    ref, _ = run(f0.copy(), 30)
    mid, (rho, ux, uy) = run(f0.copy(), 13)
    p = tmp_path / "cavity.ckpt"
    ck.save_checkpoint_lbm(p, torch.from_numpy(mid), 13,
                           moments={"rho": torch.from_numpy(rho)},
                           parameters={"omega": om})
    f, cycle, mom = ck.load_checkpoint_lbm(p, torch.empty((9, Ny, Nx), dtype=torch.float64))
    assert cycle == 13 and np.array_equal(mom["rho"].numpy(), rho)
    out, _ = run(np.ascontiguousarray(f.numpy()), 30 - cycle)
    assert np.array_equal(out, ref)
    with pytest.raises(ck.CheckpointError, match="identity/Nx"):
        ck.load_checkpoint_lbm(p, torch.empty((9, Ny, Nx + 1), dtype=torch.float64))
    with pytest.raises(ck.CheckpointError, match="identity/storage"):
        ck.load_checkpoint_lbm(p, torch.empty((9, Ny, Nx), dtype=torch.float32))
