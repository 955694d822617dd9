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
