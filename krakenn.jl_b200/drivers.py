"""Drivers: the reference's step loops on the B200 kernels.

`LBMConfig`, `initialize_2d`, `run_cavity_2d`, ... keep the names, arguments
and returned fields of src/drivers/basic.jl and src/drivers/thermal.jl.  The
loops call the C-ABI kernels of `ops`; fields come back as numpy arrays in
(Ny, Nx) / (Nz, Ny, Nx) order (the memory order of the reference's
column-major arrays).  `backend` accepts only "b200": this package has no
CPU path, and asking for one is an error, as in the reference's
_backend_from_krk_symbol (src/simulation_runner.jl:110-149).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import lattice as L
from . import ops


def _require_backend(backend: str):
    if str(backend).lower() != "b200":
        raise ValueError(f"backend '{backend}' is not provided by krakenn.jl_b200 "
                         "(this package implements the 'b200' backend only)")
    if not torch.cuda.is_available():
        raise RuntimeError("backend 'b200' requested but no CUDA device is visible; "
                           "the B200 path never falls back to the CPU")


@dataclass(frozen=True)
class LBMConfig:
    """LBMConfig -- src/drivers/basic.jl:6-23"""
    lattice: str
    Nx: int
    Ny: int
    Nz: int
    nu: float
    u_lid: float = 0.1
    max_steps: int = 10000
    output_interval: int = 1000

    @staticmethod
    def d2q9(Nx, Ny, nu, u_lid=0.1, max_steps=10000, output_interval=1000):
        return LBMConfig("D2Q9", Nx, Ny, 1, nu, u_lid, max_steps, output_interval)

    @staticmethod
    def d3q19(Nx, Ny, Nz, nu, u_lid=0.1, max_steps=10000, output_interval=1000):
        return LBMConfig("D3Q19", Nx, Ny, Nz, nu, u_lid, max_steps, output_interval)


def omega(config: LBMConfig) -> float:
    """omega(config) = 1/(3 nu + 0.5) -- src/drivers/basic.jl:30"""
    return 1.0 / (3.0 * config.nu + 0.5)


def reynolds(config: LBMConfig) -> float:
    """reynolds(config) -- src/drivers/basic.jl:38-41"""
    Ls = config.Ny if config.lattice == "D2Q9" else config.Nz
    return config.u_lid * Ls / config.nu


def _dev(device):
    return torch.device(device if device is not None else "cuda")


def initialize_2d(config: LBMConfig, T=torch.float64, device=None):
    """initialize_2d -- src/drivers/basic.jl:51-73 (f = w_q, rho = 1, u = 0)."""
    d = _dev(device)
    Nx, Ny = config.Nx, config.Ny
    f_host = np.empty((9, Ny, Nx), dtype=np.float64)
    for q in range(9):
        f_host[q] = L.D2Q9_W[q]
    f_in = torch.from_numpy(f_host).to(device=d, dtype=T)
    f_out = f_in.clone()
    return dict(f_in=f_in, f_out=f_out,
                rho=torch.ones((Ny, Nx), dtype=T, device=d),
                ux=torch.zeros((Ny, Nx), dtype=T, device=d),
                uy=torch.zeros((Ny, Nx), dtype=T, device=d),
                is_solid=torch.zeros((Ny, Nx), dtype=torch.bool, device=d))


def initialize_3d(config: LBMConfig, T=torch.float64, device=None):
    """initialize_3d -- src/drivers/basic.jl:80-101"""
    d = _dev(device)
    Nx, Ny, Nz = config.Nx, config.Ny, config.Nz
    f_host = np.empty((19, Nz, Ny, Nx), dtype=np.float64)
    for q in range(19):
        f_host[q] = L.D3Q19_W[q]
    f_in = torch.from_numpy(f_host).to(device=d, dtype=T)
    shape = (Nz, Ny, Nx)
    return dict(f_in=f_in, f_out=f_in.clone(),
                rho=torch.ones(shape, dtype=T, device=d),
                ux=torch.zeros(shape, dtype=T, device=d),
                uy=torch.zeros(shape, dtype=T, device=d),
                uz=torch.zeros(shape, dtype=T, device=d),
                is_solid=torch.zeros(shape, dtype=torch.bool, device=d))


def run_cavity_2d(config: LBMConfig, backend="b200", T=torch.float64, fused=True, state=None,
                  lid="zou_he", on_step=None):
    """run_cavity_2d -- src/drivers/basic.jl:112-144.

    lid="zou_he" (the reference driver): fused=False issues the reference's
    four launches per step (stream_2d!, apply_zou_he_north_2d!, collide_2d!,
    compute_macroscopic_2d!); fused=True issues the single-launch
    kb_cavity_step_2d, which gives the same bits.
    lid="moving_wall": half-way bounce-back on all four walls with the
    moving-wall link rule on the lid (kb_cavity_movingwall_step_2d).
    on_step(step, fields): called after every step with the device moment
    fields (for example an output.StepOutput)."""
    _require_backend(backend)
    if lid not in ("zou_he", "moving_wall"):
        raise ValueError(f"unknown lid '{lid}'")
    st = state if state is not None else initialize_2d(config, T)
    f_in, f_out = st["f_in"], st["f_out"]
    rho, ux, uy, solid = st["rho"], st["ux"], st["uy"], st["is_solid"]
    Nx, Ny = config.Nx, config.Ny
    w = omega(config)
    for step in range(config.max_steps):
        if lid == "moving_wall":
            ops.cavity_movingwall_step_2d_(f_out, f_in, rho, ux, uy, solid, Nx, Ny, w, config.u_lid)
        elif fused:
            ops.cavity_step_2d_(f_out, f_in, rho, ux, uy, solid, Nx, Ny, w, config.u_lid)
        else:
            ops.stream_2d_(f_out, f_in, Nx, Ny)
            ops.apply_zou_he_north_2d_(f_out, config.u_lid, Nx, Ny)
            ops.collide_2d_(f_out, solid, w)
            ops.compute_macroscopic_2d_(rho, ux, uy, f_out)
        f_in, f_out = f_out, f_in
        if on_step is not None:
            on_step(step + 1, {"rho": rho, "velocity": (ux, uy)})
    st["f_in"], st["f_out"] = f_in, f_out
    return dict(rho=rho.cpu().numpy(), ux=ux.cpu().numpy(), uy=uy.cpu().numpy(), config=config,
                state=st)


def run_cavity_3d(config: LBMConfig, backend="b200", T=torch.float64, on_step=None):
    """run_cavity_3d -- src/drivers/basic.jl:153-176 (on_step as run_cavity_2d)"""
    _require_backend(backend)
    st = initialize_3d(config, T)
    f_in, f_out = st["f_in"], st["f_out"]
    Nx, Ny, Nz = config.Nx, config.Ny, config.Nz
    w = omega(config)
    for step in range(config.max_steps):
        ops.stream_3d_(f_out, f_in, Nx, Ny, Nz)
        ops.apply_zou_he_top_3d_(f_out, config.u_lid, Nx, Ny, Nz)
        ops.collide_3d_(f_out, st["is_solid"], w)
        ops.compute_macroscopic_3d_(st["rho"], st["ux"], st["uy"], st["uz"], f_out)
        f_in, f_out = f_out, f_in
        if on_step is not None:
            on_step(step + 1, {"rho": st["rho"], "velocity": (st["ux"], st["uy"], st["uz"])})
    return dict(rho=st["rho"].cpu().numpy(), ux=st["ux"].cpu().numpy(),
                uy=st["uy"].cpu().numpy(), uz=st["uz"].cpu().numpy(), config=config)


def run_poiseuille_2d(Nx=4, Ny=32, nu=0.1, Fx=1e-5, max_steps=10000, backend="b200",
                      T=torch.float64, graph=True):
    """run_poiseuille_2d -- src/drivers/basic.jl:185-203: periodic x, half-way
    bounce-back walls in y, Guo body force Fx."""
    _require_backend(backend)
    cfg = LBMConfig.d2q9(Nx, Ny, nu, 0.0, max_steps)
    st = initialize_2d(cfg, T)
    f = [st["f_in"], st["f_out"]]
    w = omega(cfg)

    def step(par):
        fi, fo = f[par], f[1 - par]
        ops.stream_periodic_x_wall_y_2d_(fo, fi, Nx, Ny)
        ops.collide_guo_2d_(fo, st["is_solid"], w, Fx, 0.0)
        ops.compute_macroscopic_2d_(st["rho"], st["ux"], st["uy"], fo)

    _step_loop(step, max_steps, graph)
    return dict(rho=st["rho"].cpu().numpy(), ux=st["ux"].cpu().numpy(),
                uy=st["uy"].cpu().numpy(), f=f[max_steps & 1], config=cfg)


def run_couette_2d(Nx=4, Ny=32, nu=0.1, u_wall=0.05, max_steps=10000, backend="b200",
                   T=torch.float64, graph=True):
    """run_couette_2d -- src/drivers/basic.jl:213-234: periodic x, Zou-He south
    wall moving at u_wall, resting Zou-He north wall, BGK."""
    _require_backend(backend)
    cfg = LBMConfig.d2q9(Nx, Ny, nu, 0.0, max_steps)
    st = initialize_2d(cfg, T)
    f = [st["f_in"], st["f_out"]]
    w = omega(cfg)

    def step(par):
        fi, fo = f[par], f[1 - par]
        ops.stream_periodic_x_wall_y_2d_(fo, fi, Nx, Ny)
        ops.apply_zou_he_south_2d_(fo, u_wall, Nx)
        ops.apply_zou_he_north_2d_(fo, 0.0, Nx, Ny)
        ops.collide_2d_(fo, st["is_solid"], w)
        ops.compute_macroscopic_2d_(st["rho"], st["ux"], st["uy"], fo)

    _step_loop(step, max_steps, graph)
    return dict(rho=st["rho"].cpu().numpy(), ux=st["ux"].cpu().numpy(),
                uy=st["uy"].cpu().numpy(), f=f[max_steps & 1], config=cfg)


def taylor_green_2d_populations(N, u0):
    """Host FP64 populations of initialize_taylor_green_2d
    (src/drivers/basic.jl:242-273), shape (9, N, N)."""
    k = 2 * math.pi / N
    x = np.arange(N, dtype=np.float64)[None, :]
    y = np.arange(N, dtype=np.float64)[:, None]
    ux = -u0 * np.cos(k * x) * np.sin(k * y)
    uy = u0 * np.sin(k * x) * np.cos(k * y)
    rho = 1.0 - 3.0 * u0 ** 2 / 4.0 * (np.cos(2.0 * k * x) + np.cos(2.0 * k * y))
    return np.stack([L.equilibrium_d2q9(rho, ux, uy, q) for q in range(9)])


def run_taylor_green_2d(N=64, nu=0.01, u0=0.01, max_steps=1000, backend="b200",
                        T=torch.float64):
    """run_taylor_green_2d -- src/drivers/basic.jl:281-299"""
    _require_backend(backend)
    f_in = torch.from_numpy(taylor_green_2d_populations(N, u0)).to("cuda", T)
    f_out = f_in.clone()
    solid = torch.zeros((N, N), dtype=torch.bool, device="cuda")
    w = 1.0 / (3.0 * nu + 0.5)
    for _ in range(max_steps):
        ops.stream_fully_periodic_2d_(f_out, f_in, N, N)
        ops.collide_2d_(f_out, solid, w)
        f_in, f_out = f_out, f_in
    rho = torch.empty((N, N), dtype=T, device="cuda")
    ux, uy = torch.empty_like(rho), torch.empty_like(rho)
    ops.compute_macroscopic_2d_(rho, ux, uy, f_in)
    return dict(rho=rho.cpu().numpy(), ux=ux.cpu().numpy(), uy=uy.cpu().numpy(), u0=u0,
                k=2 * math.pi / N, max_steps=max_steps)


def taylor_green_3d_populations(N, u0, rho0=1.0, Nz=None):
    """Host FP64 equilibrium populations of the z-invariant Taylor-Green
    vortex on an N x N x Nz periodic box: ux = -u0 cos(kx) sin(ky),
    uy = u0 sin(kx) cos(ky), uz = 0, rho = rho0 - 3 u0^2/4 (cos 2kx + cos 2ky)
    (the 2D field of src/drivers/basic.jl:258-263 extruded along z).
    Shape (19, Nz, N, N)."""
    Nz = N if Nz is None else Nz
    k = 2 * math.pi / N
    x = np.arange(N, dtype=np.float64)[None, :]
    y = np.arange(N, dtype=np.float64)[:, None]
    ux = -u0 * np.cos(k * x) * np.sin(k * y)
    uy = u0 * np.sin(k * x) * np.cos(k * y)
    rho = rho0 - 3.0 * u0 ** 2 / 4.0 * (np.cos(2.0 * k * x) + np.cos(2.0 * k * y))
    uz = np.zeros_like(ux)
    plane = np.stack([L.equilibrium_d3q19(rho, ux, uy, uz, q) for q in range(19)])
    return np.ascontiguousarray(np.broadcast_to(plane[:, None, :, :], (19, Nz, N, N)))


def run_taylor_green_3d(N=64, nu=0.01, u0=0.05, Lambda=0.25, max_steps=100, backend="b200",
                        storage=torch.float64, deviation=None, moments_every=0,
                        stochastic_rounding=False):
    """Periodic D3Q19 TRT Taylor-Green vortex (no reference driver: the
    reference has no fully periodic D3Q19 pull).  Returns host fields after
    max_steps.  stochastic_rounding: 16-bit deviation storages round their
    stores stochastically."""
    _require_backend(backend)
    if deviation is None:
        deviation = storage in (torch.float16, torch.bfloat16)
    f64 = torch.from_numpy(taylor_green_3d_populations(N, u0)).to("cuda")
    f_in = torch.empty(f64.shape, dtype=storage, device="cuda")
    if storage == torch.float64 and not deviation:
        f_in.copy_(f64)
    else:
        ops.convert_populations(f_in, f64, dst_deviation=deviation)
    del f64
    f_out = torch.empty_like(f_in)
    fd = torch.float64 if storage == torch.float64 else torch.float32
    shape = (N, N, N)
    rho, ux, uy, uz = (torch.empty(shape, dtype=fd, device="cuda") for _ in range(4))
    for s in range(max_steps):
        last = s == max_steps - 1
        want = last or (moments_every and (s + 1) % moments_every == 0)
        m = (rho, ux, uy, uz) if want else (None, None, None, None)
        ops.fused_trt_step_3d_(f_out, f_in, *m, None, N, N, N, nu, Lambda,
                               periodic=(True, True, True), deviation=deviation,
                               stochastic_rounding=stochastic_rounding)
        f_in, f_out = f_out, f_in
    return dict(rho=rho.cpu().numpy(), ux=ux.cpu().numpy(), uy=uy.cpu().numpy(),
                uz=uz.cpu().numpy(), f=f_in, k=2 * math.pi / N)


def natconv_parameters(N, Ra, Pr, T_hot=1.0, T_cold=0.0):
    """Parameters of run_natural_convection_2d (src/drivers/thermal.jl:161-190)."""
    dT = T_hot - T_cold
    H = float(N)
    nu = 0.05
    alpha = nu / Pr
    beta_g = Ra * nu * alpha / (dT * H ** 3)
    return dict(nu=nu, alpha=alpha, beta_g=beta_g, omega_f=1.0 / (3.0 * nu + 0.5),
                omega_T=1.0 / (3.0 * alpha + 0.5), T_ref=(T_hot + T_cold) / 2)


def natconv_initial_g(N, T_hot=1.0, T_cold=0.0):
    """g = w_q T_init with the linear profile + 1 % seed (thermal.jl:197-206)."""
    dT = T_hot - T_cold
    i = np.arange(1, N + 1, dtype=np.float64)[None, :]
    j = np.arange(1, N + 1, dtype=np.float64)[:, None]
    T0 = T_hot - dT * (i - 0.5) / N
    T0 = T0 + (0.01 * dT) * np.sin(2 * math.pi * i / N) * np.sin(math.pi * j / N)
    return np.stack([L.D2Q9_W[q] * T0 for q in range(9)])


def nusselt_hot_wall(Temp: np.ndarray, T_hot=1.0, T_cold=0.0) -> float:
    """Hot-wall Nusselt number (src/drivers/thermal.jl:225-235); Temp is (Ny, Nx)."""
    Ny, Nx = Temp.shape
    H = float(Nx)
    dT = T_hot - T_cold
    nu_loc = np.zeros(Ny)
    for j in range(1, Ny - 1):
        nu_loc[j] = -H * (-8 * T_hot + 9 * Temp[j, 0] - Temp[j, 1]) / 3.0 / dT
    return float(np.sum(nu_loc[1:-1]) / (Ny - 2))


def run_natural_convection_2d(N=128, Ra=1e4, Pr=0.71, Rc=1.0, T_hot=1.0, T_cold=0.0,
                              max_steps=50000, backend="b200", FT=torch.float64):
    """run_natural_convection_2d -- src/drivers/thermal.jl:161-238"""
    _require_backend(backend)
    p = natconv_parameters(N, Ra, Pr, T_hot, T_cold)
    cfg = LBMConfig.d2q9(N, N, p["nu"], 0.0, max_steps)
    st = initialize_2d(cfg, FT)
    f_in, f_out = st["f_in"], st["f_out"]
    g_in = torch.from_numpy(natconv_initial_g(N, T_hot, T_cold)).to("cuda", FT)
    g_out = g_in.clone()
    Temp = torch.zeros((N, N), dtype=FT, device="cuda")
    a_visc = -math.log(Rc)
    for _ in range(max_steps):
        if Rc == 1.0:
            ops.fused_natconv_step_(f_out, f_in, g_out, g_in, Temp, N, N, p["omega_f"],
                                    p["omega_T"], p["beta_g"], p["T_ref"], T_hot, T_cold)
        else:
            ops.fused_natconv_vt_step_(f_out, f_in, g_out, g_in, Temp, N, N, p["nu"], T_cold,
                                       a_visc, p["omega_T"], p["beta_g"], p["T_ref"], T_hot,
                                       T_cold)
        f_in, f_out = f_out, f_in
        g_in, g_out = g_out, g_in
    ops.compute_macroscopic_2d_(st["rho"], st["ux"], st["uy"], f_in)
    ops.compute_temperature_2d_(Temp, g_in)
    T_cpu = Temp.cpu().numpy()
    return dict(rho=st["rho"].cpu().numpy(), ux=st["ux"].cpu().numpy(),
                uy=st["uy"].cpu().numpy(), Temp=T_cpu, Nu=nusselt_hot_wall(T_cpu, T_hot, T_cold),
                Ra=Ra, Pr=Pr, Rc=Rc, nu=p["nu"], alpha=p["alpha"])


# ------------------------------------------------ unfused thermal DDF drivers

def _step_loop(step, max_steps: int, graph: bool):
    """Run `step(parity)` for parity = 0, 1, 0, ... max_steps times.  With
    `graph`, one two-step cycle (which returns the ping-pong buffers to their
    places) is captured once as a CUDA graph and replayed, so the short
    boundary and collision launches of each step cost one graph launch."""
    if not graph or max_steps < 4:
        for s in range(max_steps):
            step(s & 1)
        return
    from .batch import Graph
    g = Graph()
    with g:
        step(0)
        step(1)
    try:
        for _ in range(max_steps // 2):
            g.launch()
        if max_steps & 1:
            step(0)
    finally:
        g.close()


def rayleigh_benard_initial_g(Nx, Ny, T_hot=1.0, T_cold=0.0, orientation="vertical"):
    """Thermal populations g = w_q T_init of run_rayleigh_benard_2d
    (src/drivers/thermal.jl:79-98): the half-way conduction profile across
    the heated gap, plus the sin-sin seed for the vertical orientation."""
    dT = T_hot - T_cold
    i = np.arange(1, Nx + 1, dtype=np.float64)[None, :]
    j = np.arange(1, Ny + 1, dtype=np.float64)[:, None]
    if orientation == "vertical":
        # the seed is separable: libm sin per row / column value
        si = np.array([math.sin(2 * math.pi * a / Nx) for a in range(1, Nx + 1)])[None, :]
        sj = np.array([math.sin(math.pi * b / Ny) for b in range(1, Ny + 1)])[:, None]
        T0 = (T_hot - dT * (j - 0.5) / Ny) + ((0.01 * dT) * si) * sj
    else:
        T0 = np.broadcast_to(T_hot - dT * (i - 0.5) / Nx, (Ny, Nx))
    return np.stack([L.D2Q9_W[q] * T0 for q in range(9)])


def rayleigh_benard_parameters(Nx, Ny, Ra, Pr, T_hot=1.0, T_cold=0.0, nu=None, alpha=None,
                               orientation="vertical"):
    """Parameters of run_rayleigh_benard_2d (src/drivers/thermal.jl:36-70)."""
    if orientation not in ("vertical", "horizontal"):
        raise ValueError(f"run_rayleigh_benard_2d: orientation '{orientation}' is not supported; "
                         "use 'vertical' (hot south / cold north, periodic x) or 'horizontal' "
                         "(hot west / cold east, solid walls)")
    dT = T_hot - T_cold
    if dT == 0:
        raise ValueError("run_rayleigh_benard_2d: T_hot and T_cold are equal; the buoyancy "
                         "scaling is undefined")
    H = Ny if orientation == "vertical" else Nx
    nu_v = 0.05 if nu is None else float(nu)
    alpha_v = nu_v / Pr if alpha is None else float(alpha)
    if nu_v <= 0 or alpha_v <= 0:
        raise ValueError("run_rayleigh_benard_2d: nu and alpha must be positive")
    Pr_v = Pr if alpha is None else nu_v / alpha_v
    return dict(nu=nu_v, alpha=alpha_v, Pr=Pr_v, H=H,
                beta_g=Ra * nu_v * alpha_v / (dT * H ** 3),
                omega_f=1.0 / (3.0 * nu_v + 0.5), omega_T=1.0 / (3.0 * alpha_v + 0.5),
                T_ref=(T_hot + T_cold) / 2)


def run_rayleigh_benard_2d(Nx=128, Ny=32, Ra=2000.0, Pr=1.0, T_hot=1.0, T_cold=0.0,
                           max_steps=20000, nu=None, alpha=None, orientation="vertical",
                           backend="b200", FT=torch.float64, graph=True):
    """run_rayleigh_benard_2d -- src/drivers/thermal.jl:31-144: the unfused
    DDF loop (stream f and g, fixed-temperature faces, T, moments, thermal
    BGK, Boussinesq BGK) on the B200 kernels."""
    _require_backend(backend)
    p = rayleigh_benard_parameters(Nx, Ny, Ra, Pr, T_hot, T_cold, nu, alpha, orientation)
    cfg = LBMConfig.d2q9(Nx, Ny, p["nu"], 0.0, max_steps)
    st = initialize_2d(cfg, FT)
    f = [st["f_in"], st["f_out"]]
    g0 = torch.from_numpy(rayleigh_benard_initial_g(Nx, Ny, T_hot, T_cold, orientation))
    g = [g0.to("cuda", FT), g0.to("cuda", FT)]
    Temp = torch.zeros((Ny, Nx), dtype=FT, device="cuda")
    rho, ux, uy, solid = st["rho"], st["ux"], st["uy"], st["is_solid"]
    stream = ops.stream_periodic_x_wall_y_2d_ if orientation == "vertical" else ops.stream_2d_

    def step(par):
        fi, fo, gi, go = f[par], f[1 - par], g[par], g[1 - par]
        stream(fo, fi, Nx, Ny)
        stream(go, gi, Nx, Ny)
        if orientation == "vertical":
            ops.apply_fixed_temp_south_2d_(go, T_hot, Nx)
            ops.apply_fixed_temp_north_2d_(go, T_cold, Nx, Ny)
        else:
            ops.apply_fixed_temp_west_2d_(go, T_hot, Ny)
            ops.apply_fixed_temp_east_2d_(go, T_cold, Nx, Ny)
        ops.compute_temperature_2d_(Temp, go)
        ops.compute_macroscopic_2d_(rho, ux, uy, fo)
        ops.collide_thermal_2d_(go, ux, uy, p["omega_T"])
        ops.collide_boussinesq_2d_(fo, Temp, solid, p["omega_f"], p["beta_g"], p["T_ref"])

    _step_loop(step, max_steps, graph)
    fin, gin = f[max_steps & 1], g[max_steps & 1]
    ops.compute_macroscopic_2d_(rho, ux, uy, fin)
    ops.compute_temperature_2d_(Temp, gin)
    return dict(rho=rho.cpu().numpy(), ux=ux.cpu().numpy(), uy=uy.cpu().numpy(),
                Temp=Temp.cpu().numpy(), f=fin, g=gin, Ra=Ra, Pr=p["Pr"], nu=p["nu"],
                alpha=p["alpha"], T_hot=T_hot, T_cold=T_cold, orientation=orientation)


def natconv_3d_initial_g(N, T_hot=1.0, T_cold=0.0):
    """g = w_q T_init, linear in x between the half-way walls
    (src/drivers/thermal.jl:481-490)."""
    dT = T_hot - T_cold
    i = np.arange(1, N + 1, dtype=np.float64)
    T0 = np.broadcast_to(T_hot - dT * (i - 0.5) / N, (N, N, N))
    return np.stack([L.D3Q19_W[q] * T0 for q in range(19)])


def natconv_3d_parameters(N, Ra, Pr, T_hot=1.0, T_cold=0.0):
    """Parameters of run_natural_convection_3d (src/drivers/thermal.jl:458-469)."""
    dT = T_hot - T_cold
    nu = 0.05
    alpha = nu / Pr
    return dict(nu=nu, alpha=alpha, beta_g=Ra * nu * alpha / (dT * float(N) ** 3),
                omega_f=1.0 / (3.0 * nu + 0.5), omega_T=1.0 / (3.0 * alpha + 0.5),
                T_ref=(T_hot + T_cold) / 2)


def nusselt_hot_wall_3d(Temp: np.ndarray, T_hot=1.0, T_cold=0.0) -> float:
    """Hot-wall Nusselt number of run_natural_convection_3d
    (src/drivers/thermal.jl:524-533); Temp is (Nz, Ny, Nx)."""
    Nz, Ny, Nx = Temp.shape
    dT = T_hot - T_cold
    dTdx = (-8 * T_hot + 9 * Temp[:, :, 0] - Temp[:, :, 1]) / 3.0
    nu_arr = -float(Nx) * dTdx / dT
    return float(np.sum(nu_arr[1:-1, 1:-1]) / max((Ny - 2) * (Nz - 2), 1))


def run_natural_convection_3d(N=32, Ra=1e3, Pr=0.71, T_hot=1.0, T_cold=0.0, max_steps=10000,
                              backend="b200", FT=torch.float64, graph=True):
    """run_natural_convection_3d -- src/drivers/thermal.jl:455-537: D3Q19
    flow and thermal DDF, hot west / cold east half-way walls, adiabatic
    bounce-back elsewhere, Boussinesq force along y."""
    _require_backend(backend)
    p = natconv_3d_parameters(N, Ra, Pr, T_hot, T_cold)
    cfg = LBMConfig.d3q19(N, N, N, p["nu"], 0.0, max_steps)
    st = initialize_3d(cfg, FT)
    f = [st["f_in"], st["f_out"]]
    g0 = torch.from_numpy(np.ascontiguousarray(natconv_3d_initial_g(N, T_hot, T_cold)))
    g = [g0.to("cuda", FT), g0.to("cuda", FT)]
    Temp = torch.zeros((N, N, N), dtype=FT, device="cuda")
    rho, ux, uy, uz, solid = st["rho"], st["ux"], st["uy"], st["uz"], st["is_solid"]

    def step(par):
        fi, fo, gi, go = f[par], f[1 - par], g[par], g[1 - par]
        ops.stream_3d_(fo, fi, N, N, N)
        ops.stream_3d_(go, gi, N, N, N)
        ops.apply_fixed_temp_west_3d_(go, T_hot, N, N)
        ops.apply_fixed_temp_east_3d_(go, T_cold, N, N, N)
        ops.compute_temperature_3d_(Temp, go)
        ops.compute_macroscopic_3d_(rho, ux, uy, uz, fo)
        ops.collide_thermal_3d_(go, ux, uy, uz, p["omega_T"])
        ops.collide_boussinesq_3d_(fo, Temp, solid, p["omega_f"], p["beta_g"], p["T_ref"])

    _step_loop(step, max_steps, graph)
    fin, gin = f[max_steps & 1], g[max_steps & 1]
    ops.compute_macroscopic_3d_(rho, ux, uy, uz, fin)
    ops.compute_temperature_3d_(Temp, gin)
    T_cpu = Temp.cpu().numpy()
    return dict(rho=rho.cpu().numpy(), ux=ux.cpu().numpy(), uy=uy.cpu().numpy(),
                uz=uz.cpu().numpy(), Temp=T_cpu, Nu=nusselt_hot_wall_3d(T_cpu, T_hot, T_cold),
                f=fin, g=gin, Ra=Ra, Pr=Pr, nu=p["nu"], alpha=p["alpha"])
