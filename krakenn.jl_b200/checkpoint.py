"""Resumable state of the plain LBM: snapshots and checkpoint files.

Follows the reference's solver-agnostic state contract
(src/platform/state.jl:23-230): a `StateSnapshot` is a plain host-side image
of a solver state -- solver name, schema version, cycle counter, `fields`
and `series` arrays, and five scalar dictionaries (`scalars`, `identity`,
`run_control`, `parameters`, `derived`) -- validated on construction with
the reference's rules (array element types Float32/Float64/Int32/Int64/Bool,
`/`-separated array names, no name both a leaf and a prefix, scalar keys
without `/` or control characters and not `keys`, `None` only in the three
configuration classes).  `write_checkpoint` refuses non-finite arrays, writes
to `path + ".tmp"`, renames an existing file to `path + ".prev"` and moves
the new one into place (src/io/checkpoint_hdf5.jl:111-147);
`check_compatible` compares solver, schema and identity key by key
(src/platform/state.jl:418-442).

The container differs: the reference writes HDF5 with Fletcher32 checksums,
and no HDF5 library is available to this package.  A checkpoint here is a
zip archive (numpy .npz layout) holding one .npy member per array under
`fields/...` and `series/...` plus `meta.json` with the root attributes, the
scalar classes and a CRC-32 of every array; a damaged, truncated or foreign
file raises `CheckpointError` naming the object.

`snapshot_lbm` / `restore_lbm` are the plain LBM client: the populations
(any storage; 16-bit deviation storages are held as float32 values, which
round-trips them exactly), optional moments, the grid and storage as the
identity and the relaxation parameters, so a run resumed from a checkpoint
continues bit for bit.  A stochastic-rounding run also records, in
`run_control`, the device counter that seeds its random rounding bits, and
its identity says so; restoring it sets the counter back, so the resumed run
draws the bits the uninterrupted run would have drawn.

Durability: the archive is closed, then the temporary file and (after the
renames) its directory are fsync'ed, so after a crash `path` is either the
previous complete checkpoint or the new complete one.
"""
from __future__ import annotations

import io
import json
import os
import time
import zipfile
import zlib
from dataclasses import dataclass, field

import numpy as np

CHECKPOINT_CONTAINER_VERSION = 1
SNAPSHOT_ELTYPES = (np.float32, np.float64, np.int32, np.int64, np.bool_)
SNAPSHOT_CONFIG_CLASSES = ("identity", "run_control", "parameters")
SCALAR_CLASSES = ("scalars", "identity", "run_control", "parameters", "derived")
ARRAY_CLASSES = ("fields", "series")
LBM_SOLVER, LBM_SCHEMA = "lbm_plain", 1


class CheckpointError(Exception):
    """A snapshot or checkpoint file refused: invalid content, non-finite
    values, solver / schema / identity mismatch, damaged or truncated file.
    The message names the offending key or object."""


def _check_array_name(cls, name):
    ok = (isinstance(name, str) and name != "" and not any(ord(ch) < 32 or ord(ch) == 127
                                                          for ch in name)
          and all(seg not in ("", ".", "..") for seg in name.split("/")))
    if not ok:
        raise CheckpointError(f"{cls}: invalid name {name!r} (non-empty `/`-separated segments "
                              f"required)")


def _check_scalar_key(cls, key):
    ok = (isinstance(key, str) and key != "" and "/" not in key and key != "keys"
          and not any(ord(ch) < 32 or ord(ch) == 127 for ch in key))
    if not ok:
        raise CheckpointError(f"{cls}: invalid key {key!r} (non-empty, no `/`, no control "
                              f"character, not the reserved name `keys`)")


def _check_arrays(cls, d):
    names = sorted(d)
    for name in names:
        _check_array_name(cls, name)
        a = d[name]
        if not isinstance(a, np.ndarray):
            raise CheckpointError(f"{cls}/{name}: expected a numpy array, got {type(a).__name__}")
        if a.dtype.type not in SNAPSHOT_ELTYPES:
            raise CheckpointError(f"{cls}/{name}: element type {a.dtype} is not allowed (allowed: "
                                  f"float32, float64, int32, int64, bool)")
        if a.ndim < 1:
            raise CheckpointError(f"{cls}/{name}: zero-dimensional arrays are not allowed (use "
                                  f"`scalars`)")
        if cls == "series" and a.ndim != 1:
            raise CheckpointError(f"{cls}/{name}: must be a vector, found shape {a.shape}")
    for name in names:
        for other in names:
            if other.startswith(name + "/"):
                raise CheckpointError(f"{cls}: name {name!r} is also used as a prefix by "
                                      f"{other!r}")


def _check_scalars(cls, d):
    allow_none = cls in SNAPSHOT_CONFIG_CLASSES
    for key, v in d.items():
        _check_scalar_key(cls, key)
        ok = isinstance(v, (str, bool, int, float)) or (allow_none and v is None)
        if not ok:
            raise CheckpointError(f"{cls}/{key}: value of type {type(v).__name__} is not allowed "
                                  f"(allowed: str, bool, int, float{', None' if allow_none else ''})")


@dataclass
class StateSnapshot:
    """Plain host-side image of a solver state (src/platform/state.jl:93-126)."""
    solver: str
    schema_version: int
    cycle: int
    fields: dict = field(default_factory=dict)
    series: dict = field(default_factory=dict)
    scalars: dict = field(default_factory=dict)
    identity: dict = field(default_factory=dict)
    run_control: dict = field(default_factory=dict)
    parameters: dict = field(default_factory=dict)
    derived: dict = field(default_factory=dict)

    def __post_init__(self):
        self.solver, self.schema_version, self.cycle = (str(self.solver), int(self.schema_version),
                                                        int(self.cycle))
        validate_content(self)


def validate_content(snap: StateSnapshot) -> StateSnapshot:
    """Names, keys, value and element types of every entry
    (validate_content, src/platform/state.jl:189-200)."""
    if not snap.solver:
        raise CheckpointError("solver: name must not be empty")
    if snap.cycle < 0:
        raise CheckpointError(f"cycle: must be >= 0, got {snap.cycle}")
    for cls in ARRAY_CLASSES:
        _check_arrays(cls, getattr(snap, cls))
    for cls in SCALAR_CLASSES:
        _check_scalars(cls, getattr(snap, cls))
    return snap


def check_finite(snap: StateSnapshot) -> StateSnapshot:
    """Refuse NaN or Inf in `fields` or `series` (check_finite,
    src/platform/state.jl:222-230); scalars and configuration are not checked."""
    for cls in ARRAY_CLASSES:
        for name, a in getattr(snap, cls).items():
            if a.dtype.kind == "f":
                bad = np.flatnonzero(~np.isfinite(a))
                if bad.size:
                    idx = np.unravel_index(bad[0], a.shape)
                    raise CheckpointError(f"{cls}/{name}: non-finite value {a[idx]} at index "
                                          f"{tuple(int(i) for i in idx)}; snapshot refused")
    return snap


def check_compatible(snap: StateSnapshot, *, solver, schema_version, identity,
                     identity_defaults=None) -> StateSnapshot:
    """Solver, schema and identity compared key by key, type and value
    (check_compatible, src/platform/state.jl:418-442)."""
    defaults = identity_defaults or {}
    if snap.solver != solver:
        raise CheckpointError(f"solver: expected {solver!r}, found {snap.solver!r}")
    if snap.schema_version != schema_version:
        raise CheckpointError(f"schema_version: expected {schema_version}, found "
                              f"{snap.schema_version}")
    for key, expected in identity.items():
        if key in snap.identity:
            found = snap.identity[key]
        elif key in defaults:
            found = defaults[key]
        else:
            raise CheckpointError(f"identity/{key}: expected {expected!r}, key missing from the "
                                  f"snapshot and no default declared")
        if type(found) is not type(expected) or found != expected:
            raise CheckpointError(f"identity/{key}: expected {expected!r}, found {found!r}")
    for key in snap.identity:
        if key not in identity:
            raise CheckpointError(f"identity/{key}: found {snap.identity[key]!r}, key not "
                                  f"expected by the caller")
    return snap


def _npy_bytes(a):
    buf = io.BytesIO()
    np.lib.format.write_array(buf, np.ascontiguousarray(a), allow_pickle=False)
    return buf.getvalue()


def write_checkpoint(path, snap: StateSnapshot, keep_previous=True):
    """Write `snap` to `path` (write_checkpoint, src/io/checkpoint_hdf5.jl:
    111-147): validated, non-finite arrays refused, written to path.tmp,
    then an existing path renamed to path.prev (keep_previous) and path.tmp
    renamed into place, so a complete checkpoint exists at every moment.
    On a refusal or a write failure an existing checkpoint is left as is."""
    validate_content(snap)
    check_finite(snap)
    path = os.fspath(path)
    tmp = path + ".tmp"
    try:
        meta = {"container_version": CHECKPOINT_CONTAINER_VERSION, "solver": snap.solver,
                "schema_version": snap.schema_version, "cycle": snap.cycle,
                "created_unix": time.time(), "crc32": {}}
        for cls in SCALAR_CLASSES:
            meta[cls] = {k: v for k, v in getattr(snap, cls).items()}
        with zipfile.ZipFile(tmp, "w", compression=zipfile.ZIP_STORED) as z:
            for cls in ARRAY_CLASSES:
                for name in sorted(getattr(snap, cls)):
                    data = _npy_bytes(getattr(snap, cls)[name])
                    member = f"{cls}/{name}.npy"
                    meta["crc32"][member] = zlib.crc32(data)
                    z.writestr(member, data)
            z.writestr("meta.json", json.dumps(meta, allow_nan=True))
        # the central directory is written on close: sync the whole file after it
        _fsync_path(tmp)
    except Exception as err:
        if os.path.exists(tmp):
            os.remove(tmp)
        raise CheckpointError(f"{tmp}: write failed, {path!r} left untouched: {err}") from err
    if keep_previous and os.path.exists(path):
        os.replace(path, path + ".prev")
    os.replace(tmp, path)
    _fsync_dir(os.path.dirname(os.path.abspath(path)))
    return path


def _fsync_path(p):
    fd = os.open(p, os.O_RDONLY)
    try:
        os.fsync(fd)
    finally:
        os.close(fd)


def _fsync_dir(d):
    """Make the renames durable (a directory fsync; skipped where the platform
    cannot open a directory)."""
    try:
        fd = os.open(d, os.O_RDONLY)
    except OSError:
        return
    try:
        os.fsync(fd)
    except OSError:
        pass
    finally:
        os.close(fd)


def _open(path):
    try:
        return zipfile.ZipFile(path, "r")
    except Exception as err:
        raise CheckpointError(f"{path}: cannot open (damaged, truncated or foreign file): "
                              f"{err}") from err


def _read_meta(z, path):
    try:
        meta = json.loads(z.read("meta.json"))
    except Exception as err:
        raise CheckpointError(f"{path}: cannot read meta.json (damaged, truncated or foreign "
                              f"file): {err}") from err
    if meta.get("container_version") != CHECKPOINT_CONTAINER_VERSION:
        raise CheckpointError(f"{path}: container version {meta.get('container_version')!r} is "
                              f"not {CHECKPOINT_CONTAINER_VERSION}")
    return meta


def read_checkpoint(path) -> StateSnapshot:
    """The snapshot stored at `path`, every array checked against its CRC-32
    (read_checkpoint, src/io/checkpoint_hdf5.jl:231-255)."""
    path = os.fspath(path)
    with _open(path) as z:
        meta = _read_meta(z, path)
        arrays = {cls: {} for cls in ARRAY_CLASSES}
        names = [n for n in z.namelist() if n != "meta.json"]
        if sorted(names) != sorted(meta.get("crc32", {})):
            raise CheckpointError(f"{path}: the archive's arrays do not match its table")
        for member in names:
            try:
                data = z.read(member)
            except Exception as err:
                raise CheckpointError(f"{path}: cannot read {member} (damaged or truncated): "
                                      f"{err}") from err
            if zlib.crc32(data) != meta["crc32"][member]:
                raise CheckpointError(f"{path}: {member} fails its checksum (damaged file)")
            cls, name = member.split("/", 1)
            if cls not in arrays or not name.endswith(".npy"):
                raise CheckpointError(f"{path}: unexpected object {member}")
            arrays[cls][name[:-4]] = np.lib.format.read_array(io.BytesIO(data),
                                                              allow_pickle=False)
    try:
        return StateSnapshot(meta["solver"], meta["schema_version"], meta["cycle"],
                             arrays["fields"], arrays["series"],
                             **{cls: dict(meta.get(cls, {})) for cls in SCALAR_CLASSES})
    except KeyError as err:
        raise CheckpointError(f"{path}: root attribute {err} missing") from err


def checkpoint_info(path):
    """Root attributes only (checkpoint_info, src/io/checkpoint_hdf5.jl:257-263)."""
    path = os.fspath(path)
    with _open(path) as z:
        meta = _read_meta(z, path)
    return {k: meta[k] for k in ("container_version", "solver", "schema_version", "cycle",
                                 "created_unix")}


# ------------------------------------------------------------- plain LBM

def _host(t):
    import torch
    if t.dtype in (torch.float16, torch.bfloat16):
        t = t.float()
    return t.detach().cpu().numpy().copy()


def lbm_identity(f, deviation=False, stochastic_rounding=False):
    """The identity of a plain LBM state: lattice, grid and storage of its
    populations (Q, [Nz,] Ny, Nx), and whether its stores round
    stochastically."""
    q = int(f.shape[0])
    dims = [int(d) for d in f.shape[1:]][::-1]  # Nx, Ny[, Nz]
    ident = {"lattice": {9: "D2Q9", 19: "D3Q19"}.get(q, f"Q{q}"), "Nx": dims[0], "Ny": dims[1],
             "storage": str(f.dtype).replace("torch.", ""), "deviation": bool(deviation),
             "stochastic_rounding": bool(stochastic_rounding)}
    if len(dims) == 3:
        ident["Nz"] = dims[2]
    return ident


# checkpoints written before the stochastic-rounding key existed
_LBM_IDENTITY_DEFAULTS = {"stochastic_rounding": False}


def snapshot_lbm(f, cycle, moments=None, parameters=None, deviation=False, run_control=None,
                 stochastic_rounding=False):
    """StateSnapshot of a plain LBM state: the populations `f` (any storage),
    optional moments {name: tensor}, the relaxation `parameters` (e.g. nu,
    Lambda, omega, u_lid) and the global `cycle`.  With stochastic_rounding,
    run_control["sr_epoch"] holds the device counter that seeds the rounding
    bits (read from the library; synchronises the current stream)."""
    fields = {"f": _host(f)}
    for name, t in (moments or {}).items():
        fields[f"moments/{name}"] = _host(t)
    rc = dict(run_control or {})
    if stochastic_rounding:
        from . import ops
        rc["sr_epoch"] = ops.get_stochastic_seed()
    return StateSnapshot(LBM_SOLVER, LBM_SCHEMA, cycle, fields=fields,
                         identity=lbm_identity(f, deviation, stochastic_rounding),
                         run_control=rc,
                         parameters=dict(parameters or {}))


def restore_lbm(snap: StateSnapshot, like, deviation=False, stochastic_rounding=False):
    """Populations of `snap` as a tensor with the dtype, device and shape of
    `like`, after check_compatible against `like`'s identity; returns
    (f, cycle, moments {name: tensor on like's device}).  A stochastic-rounding
    state also sets the library's rounding-bit counter back to the recorded
    one, so the resumed run continues bit for bit."""
    import torch
    check_compatible(snap, solver=LBM_SOLVER, schema_version=LBM_SCHEMA,
                     identity=lbm_identity(like, deviation, stochastic_rounding),
                     identity_defaults=_LBM_IDENTITY_DEFAULTS)
    if stochastic_rounding:
        epoch = snap.run_control.get("sr_epoch")
        if not isinstance(epoch, int) or isinstance(epoch, bool):
            raise CheckpointError("run_control/sr_epoch: a stochastic-rounding checkpoint must "
                                  f"record the rounding-bit counter, found {epoch!r}")
    f = torch.from_numpy(snap.fields["f"]).to(like.device).to(like.dtype)
    mom = {k.split("/", 1)[1]: torch.from_numpy(v).to(like.device)
           for k, v in snap.fields.items() if k.startswith("moments/")}
    if stochastic_rounding:
        from . import ops
        ops.set_stochastic_seed(epoch)
    return f, snap.cycle, mom


def save_checkpoint_lbm(path, f, cycle, keep_previous=True, **kw):
    """snapshot_lbm then write_checkpoint (save_checkpoint,
    src/io/checkpoint_hdf5.jl:273-274)."""
    return write_checkpoint(path, snapshot_lbm(f, cycle, **kw), keep_previous=keep_previous)


def load_checkpoint_lbm(path, like, deviation=False, stochastic_rounding=False):
    """read_checkpoint then restore_lbm."""
    return restore_lbm(read_checkpoint(path), like, deviation, stochastic_rounding)


__all__ = ["CheckpointError", "StateSnapshot", "validate_content", "check_finite",
           "check_compatible", "write_checkpoint", "read_checkpoint", "checkpoint_info",
           "snapshot_lbm", "restore_lbm", "save_checkpoint_lbm", "load_checkpoint_lbm",
           "lbm_identity"]
