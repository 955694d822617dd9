"""Batched cavity sweeps and CUDA-graph capture on the C ABI.

`CavityBatch` wraps kb_batch_*: many lid-driven MRT cavities (the loop of
test/test_mrt.jl:19-25) of different sizes advanced by one persistent
kernel until each reaches the steady residual or max_steps.  `sweep_cases`
draws the case table of a sensitivity sweep; `batch_from_sweep` builds one
from `.krk` Sweep setups (src/io/krk/parser.jl:362-420).  `Graph` wraps
kb_graph_* (the device-side form of persistent_fused_bgk!,
src/kernels/persistent_bgk_2d.jl:160).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import KB_BF16_DEV, KB_BF16_DEV_SR, KB_F16_DEV, KB_F16_DEV_SR, KB_F32_DEV, call, load

STORAGE = {"f16": KB_F16_DEV, "bf16": KB_BF16_DEV, "f32": KB_F32_DEV,
           "f16sr": KB_F16_DEV_SR, "bf16sr": KB_BF16_DEV_SR}  # *sr: stochastic rounding
STATE = {0: "live", 1: "converged", 2: "max_steps", 3: "non-finite"}


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def sweep_cases(n_cases=256, seed=0, N_values=tuple(range(64, 513, 32)), Re_range=(100.0, 2000.0),
                u_lid=0.1):
    """Case table of a cavity sensitivity sweep: N uniform on N_values, Re
    log-uniform in Re_range, nu = u_lid * N / Re (seeded numpy PCG64)."""
    rng = np.random.default_rng(seed)
    N = rng.choice(np.asarray(N_values), size=n_cases)
    Re = np.exp(rng.uniform(np.log(Re_range[0]), np.log(Re_range[1]), size=n_cases))
    nu = u_lid * N / Re
    return N.astype(np.int32), nu, np.full(n_cases, u_lid), Re


def batch_from_sweep(setups, storage="f16"):
    """One CavityBatch from `.krk` Sweep setups of a D2Q9 lid-driven cavity."""
    N, nu, u = [], [], []
    for st in setups:
        kinds = {s: b[0] for s, b in st.boundaries.items()}
        if st.lattice != "D2Q9" or kinds.get("north") != "velocity":
            raise ValueError(f"setup '{st.name}' is not a D2Q9 lid-driven cavity")
        n = int(st.sweep_values.get("N", st.N[0]))
        N.append(n)
        nu.append(st.nu)
        u.append(st.boundaries["north"][1].get("ux", 0.1))
    return CavityBatch(np.asarray(N, np.int32), np.asarray(nu), np.asarray(u), storage)


class CavityBatch:
    def __init__(self, N, nu, u_lid, storage="f16"):
        if storage not in STORAGE:
            raise ValueError(f"storage must be one of {sorted(STORAGE)}")
        load()
        self.N = np.ascontiguousarray(N, dtype=np.int32)
        self.nu = np.ascontiguousarray(nu, dtype=np.float64)
        self.u_lid = np.ascontiguousarray(u_lid, dtype=np.float64)
        self.n_cases = len(self.N)
        self.storage = storage
        self._h = C.c_void_p()
        call("kb_batch_create", C.byref(self._h), self.n_cases,
             self.N.ctypes.data_as(C.POINTER(C.c_int)),
             self.nu.ctypes.data_as(C.POINTER(C.c_double)),
             self.u_lid.ctypes.data_as(C.POINTER(C.c_double)), STORAGE[storage], _stream())

    def close(self):
        if self._h:
            call("kb_batch_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        call("kb_batch_reset", self._h, _stream())

    def run(self, max_steps=50000, check_every=100, tol=1e-6, tile_nodes=0, blocks_per_sm=0):
        """Queue the whole sweep (asynchronous)."""
        call("kb_batch_run", self._h, int(max_steps), int(check_every), float(tol),
             int(tile_nodes), int(blocks_per_sm), _stream())

    def capture(self, max_steps=50000, check_every=100, tol=1e-6):
        """The sweep's one cooperative launch (kb_batch_run with the current
        schedule) captured in a CUDA graph.  Each .launch() of the returned
        Graph advances the batch from its state at that moment; reset() first
        to replay the whole sweep.  close() the graph when done."""
        g = Graph()
        with g:
            self.run(max_steps, check_every, tol)
        return g

    def status(self):
        up, live, tout = C.c_longlong(), C.c_int(), C.c_int()
        call("kb_batch_status", self._h, C.byref(up), C.byref(live), C.byref(tout), _stream())
        return dict(updates=up.value, live_tiles=live.value, timed_out=bool(tout.value))

    def case(self, c, fields=True):
        n, steps, st = C.c_int(), C.c_int(), C.c_int()
        res = C.c_double()
        NN = int(self.N[c]) ** 2
        ux = np.empty(NN, np.float32) if fields else None
        uy = np.empty(NN, np.float32) if fields else None
        fp = C.POINTER(C.c_float)
        call("kb_batch_case", self._h, int(c), C.byref(n), C.byref(steps), C.byref(res),
             C.byref(st), ux.ctypes.data_as(fp) if fields else None,
             uy.ctypes.data_as(fp) if fields else None, _stream())
        out = dict(N=n.value, steps=steps.value, residual=res.value, state=STATE[st.value])
        if fields:
            out["ux"] = ux.reshape(n.value, n.value)
            out["uy"] = uy.reshape(n.value, n.value)
        return out

    def autotune(self, trial_steps=200):
        bt, bb = C.c_int(), C.c_int()
        best, fixed = C.c_double(), C.c_double()
        call("kb_batch_autotune", self._h, int(trial_steps), C.byref(bt), C.byref(bb),
             C.byref(best), C.byref(fixed), _stream())
        return dict(tile_nodes=bt.value, blocks_per_sm=bb.value, best_mlups=best.value,
                    fixed_mlups=fixed.value)


class Graph:
    """Capture library calls issued on a side stream, then replay them."""

    def __init__(self):
        self._g = C.c_void_p()
        self.stream = torch.cuda.Stream()

    def __enter__(self):
        self.stream.wait_stream(torch.cuda.current_stream())
        self._ctx = torch.cuda.stream(self.stream)
        self._ctx.__enter__()
        call("kb_graph_begin", C.c_void_p(self.stream.cuda_stream))
        return self

    def __exit__(self, *exc):
        try:
            call("kb_graph_end", C.c_void_p(self.stream.cuda_stream), C.byref(self._g))
        finally:
            self._ctx.__exit__(*exc)
        return False

    def launch(self):
        call("kb_graph_launch", self._g, _stream())

    def close(self):
        if self._g:
            call("kb_graph_destroy", self._g)
            self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def selftest_bounded_wait(limit=100000):
    """Run the bounded-wait self test; returns True when the wait ran out as
    designed (KB_ERR_TIMEOUT with the flag set)."""
    from ._lib import KrakenError, KB_ERR_TIMEOUT
    t = C.c_int()
    try:
        call("kb_selftest_bounded_wait", C.c_longlong(limit), C.byref(t), _stream())
    except KrakenError as e:
        return e.code == KB_ERR_TIMEOUT and t.value == 1
    return False
