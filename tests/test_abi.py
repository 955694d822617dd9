"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and rejects bad arguments with KB_ERR_ARG before touching
the device."""
import ctypes as C
import re
import subprocess

import pytest

from conftest import ROOT


def _header_symbols():
    text = (ROOT / "include" / "krakenb200.h").read_text()
    return sorted(set(re.findall(r"^(?:int|const char \*)\s*(kb_\w+)\s*\(", text, re.M)))


def test_header_and_binding_agree(pkg):
    assert _header_symbols() == sorted(pkg._lib.exported_symbols())


def test_library_exports_every_symbol(pkg):
    lib = pkg._lib.load()
    for name in _header_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(pkg._lib.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\s(kb_\w+)$", out, re.M))
    assert set(_header_symbols()) <= exported


def test_library_is_sm100a_and_static_runtime(pkg):
    out = subprocess.run(["cuobjdump", "--list-elf", str(pkg._lib.LIB_PATH)],
                         capture_output=True, text=True)
    if out.returncode == 0:
        assert "sm_100a" in out.stdout
    deps = subprocess.run(["ldd", str(pkg._lib.LIB_PATH)], capture_output=True, text=True).stdout
    assert "libcudart" not in deps  # runtime linked statically
    assert "torch" not in deps


def test_version(pkg):
    assert pkg.version().startswith("krakenb200") and "sm_100a" in pkg.version()


def test_null_pointer_is_arg_error(pkg):
    lib = pkg._lib.load()
    rc = lib.kb_stream_2d(None, None, 4, 4, 0, None)
    assert rc == pkg._lib.KB_ERR_ARG
    assert b"null" in lib.kb_last_error()
    with pytest.raises(pkg.KrakenArgumentError):
        pkg._lib.call("kb_collide_3d", None, None, 4, 4, 4, 1.0, 0, None)


def test_bad_dims_and_dtype(pkg):
    lib = pkg._lib.load()
    fake = C.c_void_p(0x1000)
    assert lib.kb_stream_2d(fake, C.c_void_p(0x2000), 0, 4, 0, None) == pkg._lib.KB_ERR_ARG
    assert lib.kb_stream_2d(fake, C.c_void_p(0x2000), 4, 4, 9, None) == \
        pkg._lib.KB_ERR_UNSUPPORTED
    assert lib.kb_stream_2d(fake, fake, 4, 4, 0, None) == pkg._lib.KB_ERR_ARG
    assert lib.kb_fused_trt_step_3d(fake, C.c_void_p(0x2000), fake, None, None, None, None,
                                    4, 4, 4, 0.1, 0.25, 0, 0, None) == pkg._lib.KB_ERR_ARG
    assert lib.kb_fused_trt_step_3d(fake, C.c_void_p(0x2000), None, None, None, None, None,
                                    4, 4, 4, 0.1, 0.25, 9, 0, None) == pkg._lib.KB_ERR_ARG
    assert lib.kb_apply_zou_he_velocity_3d(fake, 4, 4, 4, 6, 0.0, 0.0, 0.0, 0, None) == \
        pkg._lib.KB_ERR_ARG
    assert lib.kb_apply_bounce_back_wall_2d(fake, 4, 4, 5, 0, None) == pkg._lib.KB_ERR_ARG


def test_trt_rates_host(pkg):
    sp, sm = pkg.trt_rates(1 / 6, 3 / 16)
    assert abs(sp - 1) < 1e-15 and abs(sm - 8 / 7) < 1e-15
    with pytest.raises(pkg.KrakenArgumentError):
        pkg.trt_rates(-0.1)


def test_host_layer_refuses_cpu_tensors(pkg):
    import torch
    f = torch.zeros((9, 4, 4), dtype=torch.float64)
    with pytest.raises(ValueError, match="CUDA"):
        pkg.stream_2d_(f, f.clone(), 4, 4)
    with pytest.raises(ValueError):
        pkg.drivers._require_backend("cpu")


def _field_cases(pkg):
    """Every host entry point that takes macroscopic fields, called with the
    reference's positional arguments, a valid population array and ONE field
    of the wrong element type (float16 where float32/float64 is expected).
    CPU tensors: the argument checks run before anything reaches the device."""
    import torch
    f32, f16 = torch.float32, torch.float16
    N2, N3 = (6, 5), (4, 5, 6)  # (Nx, Ny), (Nx, Ny, Nz)
    Nx, Ny = N2
    X, Y, Z = N3

    def p2(dt=f32):
        return torch.zeros((9, Ny, Nx), dtype=dt)

    def p3(dt=f32):
        return torch.zeros((19, Z, Y, X), dtype=dt)

    def a2(dt=f32):
        return torch.zeros((Ny, Nx), dtype=dt)

    def a3(dt=f32):
        return torch.zeros((Z, Y, X), dtype=dt)

    bad2, bad3 = a2(f16), a3(f16)
    return {
        "compute_macroscopic_2d": lambda: pkg.compute_macroscopic_2d_(a2(), bad2, a2(), p2()),
        "fused_bgk_step": lambda: pkg.fused_bgk_step_(p2(), p2(), bad2, a2(), a2(), None, Nx, Ny, 1.0),
        "fused_trt_step": lambda: pkg.fused_trt_step_(p2(), p2(), a2(), a2(), bad2, None, Nx, Ny, 0.1),
        "compute_macroscopic_forced_2d": lambda: pkg.compute_macroscopic_forced_2d_(bad2, a2(), a2(), p2(), 0.0, 0.0),
        "collide_guo_field_2d": lambda: pkg.collide_guo_field_2d_(p2(), None, bad2, a2(), 1.0),
        "fused_trt_libb_v2_step": lambda: pkg.fused_trt_libb_v2_step_(
            p2(), p2(), a2(), bad2, a2(), None, p2(), p2(), p2(), Nx, Ny, 0.1),
        "aa_stream_step_2d": lambda: pkg.aa_stream_step_2d_(p2(), bad2, a2(), a2(), None, Nx, Ny, 1.0),
        "aa_local_step_2d": lambda: pkg.aa_local_step_2d_(p2(), a2(), a2(), bad2, None, Nx, Ny, 1.0),
        "cavity_step_2d": lambda: pkg.cavity_step_2d_(p2(), p2(), bad2, a2(), a2(), None, Nx, Ny, 1.0, 0.1),
        "cavity_movingwall_step_2d": lambda: pkg.cavity_movingwall_step_2d_(
            p2(), p2(), a2(), bad2, a2(), None, Nx, Ny, 1.0, 0.1),
        "cavity_mrt_step_2d": lambda: pkg.cavity_mrt_step_2d_(p2(), p2(), a2(), a2(), bad2, None, Nx, Ny, 0.1, 0.1),
        "fused_natconv_step": lambda: pkg.fused_natconv_step_(
            p2(), p2(), p2(), p2(), bad2, Nx, Ny, 1.0, 1.0, 1e-4, 0.5, 1.0, 0.0),
        "fused_natconv_vt_step": lambda: pkg.fused_natconv_vt_step_(
            p2(), p2(), p2(), p2(), bad2, Nx, Ny, 0.1, 0.5, 0.0, 1.0, 1e-4, 0.5, 1.0, 0.0),
        "compute_temperature_2d": lambda: pkg.compute_temperature_2d_(bad2, p2()),
        "collide_thermal_2d": lambda: pkg.collide_thermal_2d_(p2(), bad2, a2(), 1.0),
        "collide_thermal_masked_2d": lambda: pkg.collide_thermal_masked_2d_(p2(), a2(), bad2, 1.0, None),
        "collide_boussinesq_2d": lambda: pkg.collide_boussinesq_2d_(p2(), bad2, None, 1.0, 1e-4, 0.5),
        "collide_boussinesq_vt_2d": lambda: pkg.collide_boussinesq_vt_2d_(p2(), bad2, None, 0.1, 0.5, 0.0, 1e-4),
        "compute_macroscopic_3d": lambda: pkg.compute_macroscopic_3d_(a3(), a3(), a3(), bad3, p3()),
        "collide_thermal_3d": lambda: pkg.collide_thermal_3d_(p3(), a3(), bad3, a3(), 1.0),
        "compute_temperature_3d": lambda: pkg.compute_temperature_3d_(bad3, p3()),
        "compute_macroscopic_forced_3d": lambda: pkg.compute_macroscopic_forced_3d_(
            bad3, a3(), a3(), a3(), p3(), 0.0, 0.0, 0.0),
        "collide_guo_field_3d": lambda: pkg.collide_guo_field_3d_(p3(), None, a3(), a3(), bad3, 1.0),
        "collide_boussinesq_3d": lambda: pkg.collide_boussinesq_3d_(p3(), bad3, None, 1.0, 1e-4, 0.5),
        "fused_trt_step_3d": lambda: pkg.fused_trt_step_3d_(
            p3(), p3(), a3(), a3(), a3(), bad3, None, X, Y, Z, 0.1),
        "fused_trt_step_3d deviation": lambda: pkg.fused_trt_step_3d_(
            p3(f16), p3(f16), a3(), bad3, a3(), a3(), None, X, Y, Z, 0.1, deviation=True),
        "fused_trt_libb_v2_step_3d": lambda: pkg.fused_trt_libb_v2_step_3d_(
            p3(), p3(), bad3, a3(), a3(), a3(), None, p3(), p3(), p3(), p3(), X, Y, Z, 0.1),
    }


def test_wrong_eltype_field_is_arg_error(pkg):
    """A field array of the wrong element type never reaches the library: the
    host layer refuses it with the library's own argument error (KB_ERR_ARG),
    as a Julia caller's ArgumentError.  (A float16 moment array where float32
    is written would take 4-byte stores into 2-byte elements.)"""
    for name, call in _field_cases(pkg).items():
        with pytest.raises(pkg.KrakenArgumentError) as err:
            call()
        assert err.value.code == pkg._lib.KB_ERR_ARG, name
        assert "must" in str(err.value), name


def test_float16_populations_need_explicit_deviation(pkg):
    """float16 populations are not taken for deviation storage by default:
    the reference-arithmetic entry points refuse them."""
    import torch
    f = torch.zeros((9, 5, 6), dtype=torch.float16)
    with pytest.raises(pkg.KrakenArgumentError):
        pkg.stream_2d_(f, f.clone(), 6, 5)
    with pytest.raises(pkg.KrakenArgumentError):
        pkg.fused_bgk_step_(f, f.clone(), None, None, None, None, 6, 5, 1.0)
