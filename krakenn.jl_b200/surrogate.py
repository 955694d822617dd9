"""Learned warm start for lid-driven cavities.

The reference has no learned component; this module adds one beside the plain
method and measures it against the plain method.  A convolutional encoder-decoder
(`kb_surrogate_*`, BF16 tensor-core kernels in libkrakenb200.so) is trained on
steady cavities that the batched LBM kernel produces, then predicts the
steady (rho, ux, uy) of unseen cases.  The populations are initialised
from the predicted field (equilibrium plus a few hundred consistent-
initialisation iterations with the velocity held fixed), then the plain FP64
MRT cavity step (`kb_cavity_mrt_step_2d`, the reference arithmetic) iterates
to the steady residual; the same step from rest is the cold start it is
compared with.

Residual: r_u = ||u^k - u^(k-1)||_2 / ||u^k||_2 over all nodes, the
definition of src/drivers/gnf_periodic_steady.jl:186-194, checked every
`check_every` steps.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import ops
from ._lib import KB_F32, KB_F64, call
from .batch import CavityBatch, Graph
from .drivers import LBMConfig, initialize_2d

IN_CH = 8
# (rho - 1) * 30, u / 0.1: O(1) targets for u_lid = 0.1 cavities
DEFAULT_SCALE = (30.0, 10.0, 10.0)
DEFAULT_OFFSET = (1.0, 0.0, 0.0)


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Surrogate:
    """The encoder-decoder: 4 levels, `base_channels` at the first, inputs of
    H x W cavities, batches of up to `max_batch`."""

    def __init__(self, max_batch, H=256, W=256, base_channels=32, seed=0,
                 scale=DEFAULT_SCALE, offset=DEFAULT_OFFSET):
        self.H, self.W, self.C, self.max_batch = H, W, base_channels, max_batch
        self._h = C.c_void_p()
        call("kb_surrogate_create", C.byref(self._h), int(max_batch), int(H), int(W),
             int(base_channels), C.c_ulonglong(seed), _stream())
        n = C.c_longlong()
        call("kb_surrogate_num_params", self._h, C.byref(n))
        self.n_params = n.value
        self.set_normalisation(scale, offset)
        self._loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.step = 0
        self.grad_weight = 0.0

    def close(self):
        if self._h:
            call("kb_surrogate_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_normalisation(self, scale, offset):
        s = (C.c_float * 3)(*scale)
        o = (C.c_float * 3)(*offset)
        call("kb_surrogate_set_normalisation", self._h, s, o)
        self.scale, self.offset = tuple(scale), tuple(offset)

    def set_grad_weight(self, weight):
        """Weight of the gradient (H1) term of the training loss (0: plain MSE)."""
        call("kb_surrogate_set_grad_weight", self._h, C.c_float(weight))
        self.grad_weight = float(weight)

    def layers(self):
        out = []
        for i in range(15):
            ci, co, lv = C.c_int(), C.c_int(), C.c_int()
            wo, bo = C.c_longlong(), C.c_longlong()
            call("kb_surrogate_layer", self._h, i, C.byref(ci), C.byref(co), C.byref(lv),
                 C.byref(wo), C.byref(bo))
            out.append(dict(cin=ci.value, cout=co.value, level=lv.value, w_off=wo.value,
                            b_off=bo.value))
        return out

    def params(self):
        t = torch.empty(self.n_params, dtype=torch.float32, device="cuda")
        call("kb_surrogate_params", self._h, _p(t), None, _stream())
        return t

    def set_params(self, t):
        t = t.to(device="cuda", dtype=torch.float32).contiguous()
        if t.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {t.numel()}")
        call("kb_surrogate_params", self._h, None, _p(t), _stream())

    def grads(self):
        t = torch.empty(self.n_params, dtype=torch.float32, device="cuda")
        call("kb_surrogate_grads", self._h, _p(t), _stream())
        return t

    def inputs(self, re, n_nodes=None):
        """NHWC BF16 input of cavities with Reynolds numbers `re`."""
        re = torch.as_tensor(re, dtype=torch.float32).to("cuda").contiguous()
        x = torch.empty((re.numel(), self.H, self.W, IN_CH), dtype=torch.bfloat16, device="cuda")
        call("kb_surrogate_cavity_inputs", self._h, _p(x), _p(re), re.numel(),
             int(n_nodes or self.W), _stream())
        return x

    def _check(self, x, n):
        if x.dtype != torch.bfloat16 or not x.is_cuda or not x.is_contiguous():
            raise ValueError("input must be a contiguous CUDA bfloat16 tensor")
        if tuple(x.shape[1:]) != (self.H, self.W, IN_CH) or not 0 < n <= min(x.shape[0],
                                                                                self.max_batch):
            raise ValueError(f"input shape {tuple(x.shape)} does not fit this network")

    def infer(self, x):
        """Physical (rho, ux, uy), planar [n][3][H][W] FP32."""
        n = x.shape[0]
        self._check(x, n)
        out = torch.empty((n, 3, self.H, self.W), dtype=torch.float32, device="cuda")
        call("kb_surrogate_infer", self._h, _p(x), n, _p(out), _stream())
        return out

    def loss_backward(self, x, target):
        n = x.shape[0]
        self._check(x, n)
        target = target.to(device="cuda", dtype=torch.float32).contiguous()
        if tuple(target.shape) != (n, 3, self.H, self.W):
            raise ValueError("target must be [n][3][H][W]")
        call("kb_surrogate_loss_backward", self._h, _p(x), _p(target), n, _p(self._loss),
             _stream())
        return self._loss

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        call("kb_surrogate_adam", self._h, C.c_float(lr), C.c_float(beta1), C.c_float(beta2),
             C.c_float(eps), self.step, _stream())

    def train_step(self, x, target, lr):
        loss = self.loss_backward(x, target)
        self.adam(lr)
        return loss

    def timed_out(self) -> bool:
        t = C.c_int()
        call("kb_surrogate_status", self._h, C.byref(t), _stream())
        return bool(t.value)

    def flops(self, n):
        f, t = C.c_double(), C.c_double()
        call("kb_surrogate_flops", self._h, int(n), C.byref(f), C.byref(t))
        return f.value, t.value


# ----------------------------------------------------------------- data --

def held_out_split(n_train, n_test, re_range=(100.0, 3200.0), seed=0):
    """Reynolds numbers, log-uniform, for disjoint training and held-out sets."""
    rng = np.random.default_rng(seed)
    lo, hi = math.log(re_range[0]), math.log(re_range[1])
    re = np.exp(rng.uniform(lo, hi, n_train + n_test))
    return re[:n_train], re[n_train:]


def steady_cavities(re, N, u_lid=0.1, storage="f32", max_steps=200000, tol=1e-7,
                    check_every=500, tile_nodes=0, blocks_per_sm=0):
    """Steady (rho, ux, uy) of N x N MRT cavities, one per Reynolds number,
    from one persistent batched launch (FP32 collision, `storage`
    deviations).  Returns planar [n][3][N][N] FP32 fields and per-case
    (steps, residual, state)."""
    re = np.asarray(re, dtype=np.float64)
    n = re.size
    Ns = np.full(n, N, dtype=np.int32)
    nu = u_lid * N / re
    b = CavityBatch(Ns, nu, np.full(n, u_lid), storage)
    b.run(max_steps=max_steps, check_every=check_every, tol=tol, tile_nodes=tile_nodes,
          blocks_per_sm=blocks_per_sm)
    out = torch.empty((n, 3, N, N), dtype=torch.float32, device="cuda")
    f64 = torch.empty((9, N, N), dtype=torch.float64, device="cuda")
    m = [torch.empty((N, N), dtype=torch.float64, device="cuda") for _ in range(3)]
    info = []
    for c in range(n):
        ptr, dt = C.c_void_p(), C.c_int()
        call("kb_batch_populations", b._h, c, C.byref(ptr), C.byref(dt), _stream())
        call("kb_convert_populations", _p(f64), KB_F64, ptr, dt.value, 9, N * N, _stream())
        ops.compute_macroscopic_2d_(m[0], m[1], m[2], f64)
        for k in range(3):
            out[c, k].copy_(m[k])
        r = b.case(c, fields=False)
        info.append((r["steps"], r["residual"], r["state"]))
    b.close()
    return out, info


# --------------------------------------------------- plain method to steady --

class PlainCavity:
    """The plain FP64 MRT cavity (kb_cavity_mrt_step_2d) on its own stream,
    advanced `check_every` steps per CUDA-graph replay; the last two steps of
    a replay write the moments the residual compares.

    Cold start: f = w_q (rest).  Warm start from a field `init` = (rho, ux,
    uy): f = equilibrium(rho, u), then `init_iters` consistent-initialisation
    iterations (kb_cavity_mrt_init_step_2d) with u held fixed, which give rho
    and the non-equilibrium populations that go with u.  Without them the
    missing non-equilibrium part excites the slowest Stokes mode of the
    cavity and the warm start loses its lead.  The iterations count as steps."""

    def __init__(self, N, nu, u_lid, check_every=500, init=None, init_iters=500):
        if check_every % 2 or check_every < 2:
            raise ValueError("check_every must be even and >= 2")
        if init_iters % 2:
            raise ValueError("init_iters must be even")
        self.N, self.nu, self.u_lid, self.G = N, nu, u_lid, check_every
        self.stream = torch.cuda.Stream()
        self.steps = 0
        with torch.cuda.stream(self.stream):
            st = initialize_2d(LBMConfig.d2q9(N, N, nu, u_lid, 0))
            self.fa, self.fb = st["f_in"], st["f_out"]
            if init is not None:
                rho, ux, uy = (init[k].contiguous() for k in range(3))
                code = KB_F64 if init.dtype == torch.float64 else KB_F32
                call("kb_init_equilibrium_2d", _p(self.fa), _p(rho), _p(ux), _p(uy), code, N, N,
                     KB_F64, _stream())
                a, b = self.fa, self.fb
                for _ in range(init_iters):
                    call("kb_cavity_mrt_init_step_2d", _p(b), _p(a), _p(ux), _p(uy), code, None, N,
                         N, float(nu), 1.4, 1.4, 1.2, float(u_lid), KB_F64, _stream())
                    a, b = b, a
                self.steps = init_iters
            self.m1 = [torch.zeros((N, N), dtype=torch.float64, device="cuda") for _ in range(3)]
            self.m2 = [torch.zeros((N, N), dtype=torch.float64, device="cuda") for _ in range(3)]
            self.graph = Graph()
            with self.graph:
                x, y = self.fa, self.fb
                for s in range(self.G):
                    m = self.m1 if s == self.G - 2 else (self.m2 if s == self.G - 1 else None)
                    if m is None:
                        ops.cavity_mrt_step_2d_(y, x, None, None, None, None, N, N, nu, u_lid)
                    else:
                        ops.cavity_mrt_step_2d_(y, x, m[0], m[1], m[2], None, N, N, nu, u_lid)
                    x, y = y, x
        self.residual = float("inf")
        self.reached = {}  # residual threshold -> first checked step count at or below it

    def advance(self):
        with torch.cuda.stream(self.stream):
            self.graph.launch()
        self.steps += self.G

    def check(self, thresholds=()):
        with torch.cuda.stream(self.stream):
            self.residual = ops.residual(self.m2[1], self.m2[2], self.m1[1], self.m1[2])
        for t in thresholds:
            if t not in self.reached and self.residual <= t:
                self.reached[t] = self.steps
        return self.residual

    def fields(self):
        self.stream.synchronize()
        return torch.stack(self.m2)

    def close(self):
        self.graph.close()


THRESHOLDS = (1e-4, 1e-5, 1e-6, 1e-7, 1e-8)


def run_to_steady(cases, tol=1e-8, max_steps=2_000_000, check_every=500, thresholds=THRESHOLDS):
    """Advance PlainCavity objects concurrently (one stream each) until each
    reaches r_u <= tol, stops being finite or hits max_steps, recording the
    step count at which each residual threshold is first seen.  Returns the
    wall time in seconds (host clock, the GPU work being synchronised)."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    live = list(cases)
    while live:
        for c in live:
            c.advance()
        nxt = []
        for c in live:
            r = c.check(thresholds)
            if math.isfinite(r) and r > tol and c.steps < max_steps:
                nxt.append(c)
        live = nxt
    torch.cuda.synchronize()
    return time.perf_counter() - t0


# ----------------------------------------------------------------- train --

def train(model, re, targets, epochs=100, batch=16, lr=1e-3, lr_min=1e-5, seed=0,
          n_nodes=None, log_every=0, grad_weight=None):
    """Adam on minibatches of (input from Re, target field), cosine decay of
    the learning rate; grad_weight (if given) sets the loss's gradient term.
    Returns the per-epoch mean loss."""
    if grad_weight is not None:
        model.set_grad_weight(grad_weight)
    re = torch.as_tensor(np.asarray(re), dtype=torch.float32, device="cuda")
    n = re.numel()
    g = torch.Generator(device="cpu").manual_seed(seed)
    steps_per_epoch = max(1, n // batch)
    total = epochs * steps_per_epoch
    hist = []
    k = 0
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to("cuda")
        acc = torch.zeros((), dtype=torch.float64, device="cuda")
        for s in range(steps_per_epoch):
            idx = perm[s * batch:(s + 1) * batch]
            x = model.inputs(re[idx], n_nodes)
            t = targets.index_select(0, idx)
            cur = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * k / max(1, total - 1)))
            acc += model.train_step(x, t, cur).double().sum()
            k += 1
        hist.append(float(acc) / steps_per_epoch)
        if log_every and (ep + 1) % log_every == 0:
            print(f"epoch {ep + 1}: loss {hist[-1]:.3e}", flush=True)
    return hist
