"""`.krk` front end for the b200 backend (the subset that reaches the
stream-collide path).

Directives follow src/io/krk/ (parser.jl, directives.jl): Simulation, Domain,
Physics, Define, Setup reynolds, Boundary, Backend, Sweep (Cartesian
product, diagnostics.jl:435-447 and parser.jl:375-420), Preset
natural_convection_2d, Run.  `Backend` accepts the reference's names
(cpu, cuda, metal) plus `b200`; an unknown name is an error at parse time
(directives.jl:527-535).  `run_simulation` resolves the backend like
src/simulation_runner.jl:156-160 (explicit argument beats the file, which
beats the default) and runs only `b200`: any other backend is an error,
never a silent fallback.
"""
from __future__ import annotations

import ast
import itertools
import re
from dataclasses import dataclass, field, replace
from pathlib import Path

KNOWN_BACKENDS = ("cpu", "cuda", "metal", "b200")


@dataclass
class SimulationSetup:
    name: str = "sim"
    lattice: str = "D2Q9"
    L: tuple = (1.0, 1.0, 1.0)
    N: tuple = (1, 1, 1)
    physics: dict = field(default_factory=dict)
    boundaries: dict = field(default_factory=dict)   # side -> ("wall"|"velocity"|"periodic", params)
    backend: str | None = None
    max_steps: int = 0
    preset: str | None = None
    user_vars: dict = field(default_factory=dict)
    sweep_values: dict = field(default_factory=dict)

    @property
    def nu(self) -> float:
        return float(self.physics["nu"])


_BINOPS = {ast.Add: lambda a, b: a + b, ast.Sub: lambda a, b: a - b,
           ast.Mult: lambda a, b: a * b, ast.Div: lambda a, b: a / b,
           ast.Pow: lambda a, b: a ** b}
_UNOPS = {ast.UAdd: lambda a: +a, ast.USub: lambda a: -a}


def _arith(node, env: dict) -> float:
    """Evaluate a parsed arithmetic expression: numbers, defined names, + - * / ^
    (written **) and parentheses.  Anything else (calls, attributes, indexing)
    is rejected."""
    if isinstance(node, ast.Expression):
        return _arith(node.body, env)
    if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)) \
            and not isinstance(node.value, bool):
        return float(node.value)
    if isinstance(node, ast.Name) and node.id in env:
        return float(env[node.id])
    if isinstance(node, ast.BinOp) and type(node.op) in _BINOPS:
        return _BINOPS[type(node.op)](_arith(node.left, env), _arith(node.right, env))
    if isinstance(node, ast.UnaryOp) and type(node.op) in _UNOPS:
        return _UNOPS[type(node.op)](_arith(node.operand, env))
    raise ValueError("unsupported expression element " + type(node).__name__)


def _num(s: str, user_vars: dict) -> float:
    s = s.strip()
    try:
        return float(s)
    except ValueError:
        pass
    if s in user_vars:
        return float(user_vars[s])
    # tiny arithmetic on numbers and defined names
    if re.fullmatch(r"[\w.eE+\-*/() ]+", s):
        env = {k: float(v) for k, v in user_vars.items() if isinstance(v, (int, float))}
        try:
            return _arith(ast.parse(s, mode="eval"), env)
        except (SyntaxError, ValueError, ZeroDivisionError, OverflowError) as exc:
            raise ValueError(f"cannot evaluate '{s}' in .krk") from exc
    raise ValueError(f"unknown value '{s}' in .krk")


def _parse_backend(line: str) -> str:
    toks = line.split()
    if len(toks) < 2:
        raise ValueError(f"Backend needs a name: {line}")
    name = toks[1].lower()
    if name not in KNOWN_BACKENDS:
        raise ValueError(f"Unknown backend '{toks[1]}' in .krk 'Backend' directive. "
                         f"Supported values: {', '.join(KNOWN_BACKENDS)}.")
    return name


def _parse_sweep(line: str):
    m = re.match(r"^Sweep\s+(\w+)\s*=\s*\[([^\]]+)\]", line)
    if not m:
        raise ValueError(f"Cannot parse Sweep: {line}")
    return m.group(1), [float(t) for t in m.group(2).split(",") if t.strip()]


_PRESETS = {
    # natural_convection_2d: the thermal cavity of run_natural_convection_2d
    "natural_convection_2d": ["Simulation natural_convection D2Q9",
                              "Domain L = 1 x 1 N = 128 x 128",
                              "Physics nu = 0.05 Pr = 0.71 Ra = 10000"],
}


def _lines(text: str) -> list[str]:
    out = []
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if line:
            out.append(line)
    expanded = []
    for line in out:
        if line.split()[0] == "Preset":
            name = line.split()[1] if len(line.split()) > 1 else ""
            if name not in _PRESETS:
                raise ValueError(f"Unknown Preset '{name}'")
            expanded.append(f"__preset {name}")
            expanded.extend(_PRESETS[name])
        else:
            expanded.append(line)
    return expanded


def _parse_single(lines: list[str], overrides: dict) -> SimulationSetup:
    st = SimulationSetup()
    st.user_vars.update(overrides)
    setup_re = None
    for line in lines:
        word = line.split()[0]
        if word == "__preset":
            st.preset = line.split()[1]
        elif word == "Simulation":
            toks = line.split()
            st.name = toks[1] if len(toks) > 1 else "sim"
            st.lattice = toks[2] if len(toks) > 2 else "D2Q9"
        elif word == "Define":
            m = re.match(r"^Define\s+(\w+)\s*=\s*(.+)$", line)
            if not m:
                raise ValueError(f"Cannot parse Define: {line}")
            if m.group(1) not in overrides:
                st.user_vars[m.group(1)] = _num(m.group(2), st.user_vars)
        elif word == "Domain":
            lm = re.search(r"L\s*=\s*([\w.eE+-]+)\s*x\s*([\w.eE+-]+)(?:\s*x\s*([\w.eE+-]+))?", line)
            nm = re.search(r"N\s*=\s*([\w.eE+-]+)\s*x\s*([\w.eE+-]+)(?:\s*x\s*([\w.eE+-]+))?", line)
            if not lm or not nm:
                raise ValueError(f"Cannot parse Domain: {line}")
            st.L = tuple(_num(v, st.user_vars) if v else 1.0 for v in lm.groups())
            st.N = tuple(int(round(_num(v, st.user_vars))) if v else 1 for v in nm.groups())
        elif word == "Physics":
            for m in re.finditer(r"(\w+)\s*=\s*([\w.eE+\-*/()]+)", line):
                key, val = m.group(1), m.group(2)
                try:
                    st.physics[key] = _num(val, st.user_vars)
                except ValueError:
                    st.physics[key] = val
        elif word == "Setup":
            m = re.search(r"reynolds\s*=\s*(\w+)", line)
            if m:
                lref = re.search(r"L_ref\s*=\s*([\w.eE+-]+)", line)
                uref = re.search(r"U_ref\s*=\s*([\w.eE+-]+)", line)
                setup_re = (m.group(1), lref.group(1) if lref else None,
                            uref.group(1) if uref else None)
        elif word == "Boundary":
            toks = line.split(None, 2)
            side, kind = toks[1], toks[2] if len(toks) > 2 else ""
            if kind.startswith("velocity"):
                params = {k: _num(v, st.user_vars)
                          for k, v in re.findall(r"(\w+)\s*=\s*([\w.eE+\-*/]+)", kind)}
                st.boundaries[side] = ("velocity", params)
            elif kind.startswith("periodic"):
                st.boundaries[side] = ("periodic", {})
            elif kind.startswith("wall"):
                st.boundaries[side] = ("wall", {})
            else:
                raise ValueError(f"Boundary kind '{kind}' is not on the b200 path")
        elif word == "Backend":
            st.backend = _parse_backend(line)
        elif word == "Run":
            m = re.match(r"^Run\s+(\d+)\s+steps", line)
            if not m:
                raise ValueError(f"Cannot parse Run: {line}")
            st.max_steps = int(m.group(1))
        elif word in ("Output", "Initial", "Module"):
            continue  # outputs and initial fields are outside the stream-collide path
        else:
            raise ValueError(f"Unknown .krk directive '{word}'")
    if setup_re is not None:
        re_name, lref, uref = setup_re
        Re = _num(re_name, st.user_vars)
        Lr = _num(lref, st.user_vars) if lref else float(st.N[1])
        Ur = _num(uref, st.user_vars) if uref else 0.1
        st.physics["nu"] = Ur * Lr / Re
    st.sweep_values = {k: overrides[k] for k in overrides}
    return st


def parse_kraken_sweep(text: str, **kwargs) -> list[SimulationSetup]:
    """parse_kraken_sweep -- src/io/krk/parser.jl:362-420 (one setup per
    combination, last Sweep varying fastest)."""
    lines = _lines(text)
    sweeps = [_parse_sweep(l) for l in lines if l.split()[0] == "Sweep"]
    rest = [l for l in lines if l.split()[0] != "Sweep"]
    if not sweeps:
        return [_parse_single(rest, dict(kwargs))]
    out = []
    for combo in itertools.product(*[vals for _, vals in sweeps]):
        ov = dict(kwargs)
        ov.update({name: v for (name, _), v in zip(sweeps, combo)})
        out.append(_parse_single(rest, ov))
    return out


def parse_kraken(text: str, **kwargs) -> SimulationSetup:
    setups = parse_kraken_sweep(text, **kwargs)
    if len(setups) != 1:
        raise ValueError("text holds a Sweep; use parse_kraken_sweep")
    return setups[0]


def load_kraken(path: str | Path, **kwargs) -> SimulationSetup:
    return parse_kraken(Path(path).read_text(), **kwargs)


def resolve_backend(setup: SimulationSetup, backend: str | None) -> str:
    """_resolve_run_backend -- src/simulation_runner.jl:156-160."""
    if backend is not None:
        name = str(backend).lower()
    elif setup.backend is not None:
        name = setup.backend
    else:
        name = "b200"
    if name not in KNOWN_BACKENDS:
        raise ValueError(f"Unknown backend '{name}'. Supported values: {', '.join(KNOWN_BACKENDS)}.")
    if name != "b200":
        raise ValueError(f"Backend '{name}' requested, but this package provides only the "
                         "'b200' backend; it never falls back to another device.")
    return name


def run_simulation(setup_or_path, backend: str | None = None, max_steps: int | None = None,
                   T=None, output_dir=None, vtk_every=0, callback=None, callback_every=100,
                   **kwargs):
    """run_simulation -- src/simulation_runner.jl:62-73, 235-443 (dispatch to
    the driver whose stream-collide path this package implements).  For the
    cavity drivers, output_dir + vtk_every write VTK snapshots and a .pvd, and
    callback(step, fields) runs every callback_every steps (:414-426); both
    run asynchronously (output.StepOutput)."""
    import torch

    from . import drivers

    if isinstance(setup_or_path, SimulationSetup):
        setup = setup_or_path
    else:
        setup = load_kraken(setup_or_path, **kwargs)
    resolve_backend(setup, backend)
    steps = max_steps if max_steps is not None else setup.max_steps
    T = T or torch.float64
    if setup.preset == "natural_convection_2d":
        ph = setup.physics
        return drivers.run_natural_convection_2d(N=setup.N[0], Ra=ph.get("Ra", 1e4),
                                                 Pr=ph.get("Pr", 0.71), max_steps=steps, FT=T)
    kinds = {s: b[0] for s, b in setup.boundaries.items()}
    if setup.lattice == "D2Q9":
        Nx, Ny = setup.N[0], setup.N[1]
        if kinds.get("x") == "periodic" and kinds.get("y") == "periodic":
            u0 = float(setup.user_vars.get("u0", 0.01))
            return drivers.run_taylor_green_2d(N=Nx, nu=setup.nu, u0=u0, max_steps=steps, T=T)
        if kinds.get("north") == "velocity" and all(kinds.get(s) == "wall"
                                                     for s in ("south", "east", "west")):
            u = setup.boundaries["north"][1].get("ux", 0.1)
            cfg = drivers.LBMConfig.d2q9(Nx, Ny, setup.nu, u, steps)
            hook = _output_hook(setup, Nx, Ny, None, output_dir, vtk_every, callback,
                                callback_every)
            try:
                return drivers.run_cavity_2d(cfg, T=T, on_step=hook)
            finally:
                if hook is not None:
                    hook.close()
    if setup.lattice == "D3Q19":
        if kinds.get("top") == "velocity":
            u = setup.boundaries["top"][1].get("ux", 0.1)
            cfg = drivers.LBMConfig.d3q19(*setup.N, setup.nu, u, steps)
            hook = _output_hook(setup, *setup.N, output_dir, vtk_every, callback, callback_every)
            try:
                return drivers.run_cavity_3d(cfg, T=T, on_step=hook)
            finally:
                if hook is not None:
                    hook.close()
    raise ValueError(f"setup '{setup.name}' ({setup.lattice}, boundaries {kinds}) is not on the "
                     "b200 stream-collide path")


def _output_hook(setup, Nx, Ny, Nz, output_dir, vtk_every, callback, callback_every):
    if (output_dir is None or not vtk_every) and callback is None:
        return None
    from .output import StepOutput
    dx = setup.L[0] / Nx if setup.L and setup.L[0] else 1.0
    return StepOutput(Nx, Ny, Nz, dx, output_dir, vtk_every, callback, callback_every,
                      name=setup.name)


__all__ = ["SimulationSetup", "parse_kraken", "parse_kraken_sweep", "load_kraken",
           "run_simulation", "resolve_backend", "KNOWN_BACKENDS", "replace"]
