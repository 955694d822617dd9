"""Output of macroscopic fields without stalling the step loop.

The reference copies the fields to the host and writes each VTK snapshot
inside the time loop (src/simulation_runner.jl:414-426, src/io/vtk_writer.jl).
Here a snapshot costs the loop one device-to-device copy of the fields into a
staging slot, on the compute stream.  The device-to-host copy of that slot
then runs on a separate copy stream, into pinned host memory, while the next
steps compute.  A writer thread waits for the copy and hands the host arrays
to a sink: the VTK writer below, or a user callback.  `depth` staging slots
form a ring; the loop waits only when all of them are still in flight.

VTK format: the files of WriteVTK's `vtk_grid(filename, xs, ys[, zs])` as the
reference calls it (src/io/vtk_writer.jl:8-88): an XML RectilinearGrid with
Nx+1 (Ny+1, Nz+1) points along each axis at spacing dx, so the fields are
cell data, written as raw appended binary; a `.pvd` collection lists the
snapshots with their times.
"""
from __future__ import annotations

import queue
import threading
from pathlib import Path

import numpy as np

_VTK_TYPES = {np.dtype(np.float64): "Float64", np.dtype(np.float32): "Float32"}


def write_vtr(filename, Nx, Ny, Nz, dx, fields: dict):
    """Write one RectilinearGrid snapshot.  `fields` maps a name to an array
    of shape (Ny, Nx) / (Nz, Ny, Nx) (the library's memory order, x fastest)
    or to a tuple of two or three such arrays (a vector field; a missing z
    component is written as zero).  float16 data are written as Float32.
    Returns the path."""
    path = Path(str(filename))
    if path.suffix != ".vtr":
        path = path.with_suffix(".vtr")
    dims3 = Nz is not None
    coords = [np.arange(n + 1, dtype=np.float64) * float(dx) for n in (Nx, Ny)]
    coords.append(np.arange(Nz + 1, dtype=np.float64) * float(dx) if dims3
                  else np.zeros(1, dtype=np.float64))
    blocks, offset = [], 0

    def add(arr, name, ncomp, where):
        nonlocal offset
        a = np.ascontiguousarray(arr)
        if a.dtype == np.float16:
            a = a.astype(np.float32)
        raw = a.tobytes()
        blocks.append(np.uint64(len(raw)).tobytes() + raw)
        where.append(f'        <DataArray type="{_VTK_TYPES[a.dtype]}" Name="{name}" '
                     f'NumberOfComponents="{ncomp}" format="appended" offset="{offset}"/>')
        offset += 8 + len(raw)

    cell = []
    for name, data in fields.items():
        if isinstance(data, (tuple, list)):
            comps = [np.asarray(c).reshape(-1) for c in data]
            if len(comps) == 2:
                comps.append(np.zeros_like(comps[0]))
            add(np.stack(comps, axis=1), name, 3, cell)
        else:
            add(np.asarray(data).reshape(-1), name, 1, cell)
    pts = []
    for n, c in zip("xyz", coords):
        add(c, f"{n}_coordinates", 1, pts)
    extent = f"0 {Nx} 0 {Ny} 0 {Nz if dims3 else 0}"
    head = "\n".join([
        '<?xml version="1.0"?>',
        '<VTKFile type="RectilinearGrid" version="1.0" byte_order="LittleEndian" '
        'header_type="UInt64">',
        f'  <RectilinearGrid WholeExtent="{extent}">',
        f'    <Piece Extent="{extent}">',
        '      <CellData>', *cell, '      </CellData>',
        '      <Coordinates>', *pts, '      </Coordinates>',
        '    </Piece>',
        '  </RectilinearGrid>',
        '  <AppendedData encoding="raw">',
        '_']).encode()
    with open(path, "wb") as fh:
        fh.write(head)
        for b in blocks:
            fh.write(b)
        fh.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return path


def read_vtr(path) -> dict:
    """Read back a file written by write_vtr (inspection and test helper):
    {name: flat array or (n, 3) array}, coordinates included."""
    import xml.etree.ElementTree as ET
    data = Path(path).read_bytes()
    mark = data.index(b"<AppendedData")
    start = data.index(b"_", mark) + 1
    root = ET.fromstring(data[:mark].decode() + "</VTKFile>")
    out = {}
    for arr in root.iter("DataArray"):
        off = start + int(arr.get("offset"))
        n = int(np.frombuffer(data[off:off + 8], dtype=np.uint64)[0])
        dt = np.float64 if arr.get("type") == "Float64" else np.float32
        v = np.frombuffer(data[off + 8:off + 8 + n], dtype=dt)
        k = int(arr.get("NumberOfComponents", "1"))
        out[arr.get("Name")] = v.reshape(-1, k) if k > 1 else v
    return out


class PVDCollection:
    """create_pvd / `pvd[time] = vtk` / vtk_save(pvd) (src/io/vtk_writer.jl:
    39-88): a ParaView collection of snapshot files, rewritten on save."""

    def __init__(self, filename):
        p = Path(str(filename))
        self.path = p if p.suffix == ".pvd" else p.with_suffix(".pvd")
        self.entries: list[tuple[float, str]] = []

    def add(self, time, vtr_path):
        self.entries.append((float(time), Path(vtr_path).name))

    def save(self):
        lines = ['<?xml version="1.0"?>',
                 '<VTKFile type="Collection" version="1.0" byte_order="LittleEndian">',
                 '  <Collection>']
        for t, f in self.entries:
            lines.append(f'    <DataSet timestep="{t!r}" part="0" file="{f}"/>')
        lines += ['  </Collection>', '</VTKFile>', '']
        self.path.write_text("\n".join(lines))
        return self.path


class VTKSeries:
    """Sink of AsyncSnapshots: write_snapshot_2d!/3d! (src/io/vtk_writer.jl:
    150-230), files `snapshot_NNNNNNN.vtr` in `output_dir` registered in
    `<name>.pvd` (written by close())."""

    def __init__(self, output_dir, Nx, Ny, Nz=None, dx=1.0, name="simulation"):
        self.dir = Path(output_dir)
        self.dir.mkdir(parents=True, exist_ok=True)
        self.Nx, self.Ny, self.Nz, self.dx = Nx, Ny, Nz, dx
        self.pvd = PVDCollection(self.dir / name)

    def __call__(self, step, time, fields):
        path = write_vtr(self.dir / f"snapshot_{step:07d}", self.Nx, self.Ny, self.Nz, self.dx,
                         fields)
        self.pvd.add(time, path)

    def close(self):
        self.pvd.save()


class AsyncSnapshots:
    """Snapshots of device fields delivered to `sink(step, time, fields)` on a
    writer thread, as host numpy arrays (views of pinned memory, valid until
    the sink returns).

    submit() orders a device-to-device copy into a staging slot on the current
    stream and returns; the device-to-host copy and the sink run behind the
    next steps.  A slot is reused only after its copy and its sink are done,
    so at most `depth` snapshots are in flight."""

    def __init__(self, sink, depth=2):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("AsyncSnapshots needs a CUDA device (the fields live on the B200)")
        self.sink = sink
        self.depth = int(depth)
        self.copy_stream = torch.cuda.Stream()
        self._slots = [None] * self.depth       # per slot: {name: (device, pinned host)}
        self._free = [threading.Event() for _ in range(self.depth)]
        for e in self._free:
            e.set()
        self._next = 0
        self._q: queue.Queue = queue.Queue()
        self._error = None
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    @staticmethod
    def _flatten(fields):
        out = {}
        for name, v in fields.items():
            if isinstance(v, (tuple, list)):
                for n, c in enumerate(v):
                    out[f"{name}\x00{n}"] = c
            else:
                out[name] = v
        return out

    @staticmethod
    def _regroup(flat):
        out = {}
        for key, arr in flat.items():
            if "\x00" in key:
                name, n = key.split("\x00")
                out.setdefault(name, {})[int(n)] = arr
            else:
                out[key] = arr
        return {k: (tuple(v[i] for i in sorted(v)) if isinstance(v, dict) else v)
                for k, v in out.items()}

    def submit(self, step, fields: dict, time=None):
        import torch
        if self._error is not None:
            raise RuntimeError("snapshot writer failed") from self._error
        k = self._next
        self._next = (k + 1) % self.depth
        self._free[k].wait()             # the slot's previous snapshot is out
        self._free[k].clear()
        flat = self._flatten(fields)
        slot = self._slots[k]
        if slot is None or set(slot) != set(flat) or any(
                slot[n][0].shape != t.shape or slot[n][0].dtype != t.dtype
                for n, t in flat.items()):
            slot = {n: (torch.empty_like(t),
                        torch.empty(t.shape, dtype=t.dtype, pin_memory=True))
                    for n, t in flat.items()}
            self._slots[k] = slot
        compute = torch.cuda.current_stream()
        for n, t in flat.items():
            slot[n][0].copy_(t)          # staging copy, ordered after the step
        staged = torch.cuda.Event()
        staged.record(compute)
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(staged)
            for n in flat:
                slot[n][1].copy_(slot[n][0], non_blocking=True)
            done = torch.cuda.Event()
            done.record(self.copy_stream)
        self._q.put((k, step, float(step if time is None else time), done))

    def _run(self):
        while True:
            item = self._q.get()
            if item is None:
                return
            k, step, time, done = item
            try:
                done.synchronize()
                host = {n: h.numpy() for n, (_, h) in self._slots[k].items()}
                self.sink(step, time, self._regroup(host))
            except BaseException as e:  # reported by the next submit() or close()
                self._error = e
            finally:
                self._free[k].set()

    def close(self):
        """Wait for every snapshot, then close the sink (writes the .pvd)."""
        self._q.put(None)
        self._thread.join()
        if hasattr(self.sink, "close"):
            self.sink.close()
        if self._error is not None:
            raise RuntimeError("snapshot writer failed") from self._error


class StepOutput:
    """The output hook of a step loop: VTK snapshots every `vtk_every` steps
    and `callback(step, fields)` every `callback_every` steps (the `vtk_out`
    interval and `callback` / `callback_every` of run_simulation,
    src/simulation_runner.jl:414-426), both asynchronous.  The fields given to
    the callback are host numpy arrays valid for the duration of the call."""

    def __init__(self, Nx, Ny, Nz=None, dx=1.0, output_dir=None, vtk_every=0, callback=None,
                 callback_every=0, name="simulation", depth=2):
        self.vtk_every = int(vtk_every) if output_dir is not None else 0
        self.callback_every = int(callback_every) if callback is not None else 0
        self.vtk = (AsyncSnapshots(VTKSeries(output_dir, Nx, Ny, Nz, dx, name), depth)
                    if self.vtk_every > 0 else None)
        self.cb = (AsyncSnapshots(lambda step, time, f: callback(step, f), depth)
                   if self.callback_every > 0 else None)

    def __call__(self, step, fields):
        if self.vtk is not None and step % self.vtk_every == 0:
            self.vtk.submit(step, fields)
        if self.cb is not None and step % self.callback_every == 0:
            self.cb.submit(step, fields)

    def close(self):
        for s in (self.vtk, self.cb):
            if s is not None:
                s.close()
