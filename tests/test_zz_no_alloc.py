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


def test_static_mass_rejects_oversize(cuda, pkg):
    f = torch.zeros((19, 4, 4, 4), dtype=torch.float64, device="cuda")
    out = C.c_double()
    lib = pkg._lib.load()
    too_many_nodes = 1_073_479_680 // 19 + 1
    rc = lib.kb_mass_static(C.c_void_p(f.data_ptr()), 19, too_many_nodes, pkg._lib.KB_F64,
                            C.byref(out), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == pkg._lib.KB_ERR_ARG
    assert b"static scratch" in lib.kb_last_error()
