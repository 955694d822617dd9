"""kb_mass_static: the mass reduction for callers that cannot let the library
allocate device memory (its partial sums live in a fixed device array).

It must give kb_mass's result (same 1e-12 relative bound as the other
reduction tests) on consecutive calls, since every call reuses the same
array, and refuse inputs larger than that array can serve."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _mass(pkg, name, f, Q, dtype_code):
    out = C.c_double()
    pkg._lib.call(name, C.c_void_p(f.data_ptr()), Q, f.numel() // Q, dtype_code, C.byref(out),
                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return out.value


def test_static_mass_matches_kb_mass_twice(cuda, pkg):
    rng = np.random.default_rng(11)
    lib = pkg._lib
    cases = [
        (torch.from_numpy(rng.random((19, 40, 33, 29))).cuda(), 19, lib.KB_F64),
        (torch.from_numpy(rng.random((9, 700, 513))).cuda(), 9, lib.KB_F64),
        (torch.from_numpy(rng.random((9, 64, 64)).astype(np.float32)).cuda(), 9, lib.KB_F32),
    ]
    for f, Q, code in cases:
        ref = _mass(pkg, "kb_mass", f, Q, code)
        first = _mass(pkg, "kb_mass_static", f, Q, code)
        second = _mass(pkg, "kb_mass_static", f, Q, code)
        assert abs(first - ref) <= 1e-12 * abs(ref)
        assert abs(second - ref) <= 1e-12 * abs(ref)


def test_static_mass_deviation_storages(cuda, pkg):
    """The 16-bit and FP32 deviation storages add w_q back per population;
    the static variant must do the same as kb_mass, twice in a row."""
    rng = np.random.default_rng(12)
    lib = pkg._lib
    d = 0.01 * rng.standard_normal((19, 24, 20, 36))
    for tdt, code in ((torch.float16, lib.KB_F16_DEV), (torch.bfloat16, lib.KB_BF16_DEV),
                      (torch.float16, lib.KB_F16_DEV_SR), (torch.float32, lib.KB_F32_DEV)):
        f = torch.from_numpy(d).to("cuda", tdt)
        ref = _mass(pkg, "kb_mass", f, 19, code)
        assert abs(ref - 24 * 20 * 36) < 0.05 * 24 * 20 * 36  # sum_q w_q = 1 per node
        for _ in range(2):
            got = _mass(pkg, "kb_mass_static", f, 19, code)
            assert abs(got - ref) <= 1e-12 * abs(ref)


def test_static_mass_at_the_limit(cuda, pkg):
    """lattice_q * n_nodes exactly at the static limit uses every partial-sum
    slot of the array; one node more is refused."""
    lib = pkg._lib
    Q, n = 9, 1_073_479_680 // 9
    f = torch.empty((Q, n), dtype=torch.float16, device="cuda")
    f.uniform_(-0.01, 0.01)
    ref = _mass(pkg, "kb_mass", f, Q, lib.KB_F16_DEV)
    for _ in range(2):
        got = _mass(pkg, "kb_mass_static", f, Q, lib.KB_F16_DEV)
        assert abs(got - ref) <= 1e-12 * abs(ref)
    out = C.c_double()
    rc = lib.load().kb_mass_static(C.c_void_p(f.data_ptr()), Q, n + 1, lib.KB_F16_DEV,
                                   C.byref(out), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == lib.KB_ERR_ARG
    del f
    torch.cuda.empty_cache()


def test_static_mass_rejects_size_overflow(cuda, pkg):
    f = torch.zeros((19, 4, 4, 4), dtype=torch.float64, device="cuda")
    out = C.c_double()
    lib = pkg._lib.load()
    rc = lib.kb_mass_static(C.c_void_p(f.data_ptr()), 19, (1 << 64) // 19 + 1, pkg._lib.KB_F64,
                            C.byref(out), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == pkg._lib.KB_ERR_ARG
    assert b"overflow" in lib.kb_last_error()


def test_static_mass_rejects_oversize(cuda, pkg):
    f = torch.zeros((19, 4, 4, 4), dtype=torch.float64, device="cuda")
    out = C.c_double()
    lib = pkg._lib.load()
    too_many_nodes = 1_073_479_680 // 19 + 1
    rc = lib.kb_mass_static(C.c_void_p(f.data_ptr()), 19, too_many_nodes, pkg._lib.KB_F64,
                            C.byref(out), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == pkg._lib.KB_ERR_ARG
    assert b"static scratch" in lib.kb_last_error()
