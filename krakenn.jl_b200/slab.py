"""One grid over several GPUs: D3Q19 slabs along z, D2Q9 slabs along y.

The reference runs one grid on one device and has no distributed backend;
this module is the B200 extension for grids larger than one GPU (or to
shorten time to solution).  Rank r of R owns the z-planes [z0, z1) of the
global Nx x Ny x Nz grid, stored in the library's layout f[q][k][j][i] with
one ghost plane below and one above wherever a neighbouring slab exists
(always on a periodic z axis, where the slabs form a ring; not at a global
z wall).

A pull step of node (i, j, k) reads population q from (i, j, k) - c_q, so
the planes next to a slab face need, from the neighbouring slab, only the
five populations that cross that face: c_z = +1 (q = 5, 11, 12, 15, 16)
from the plane below, c_z = -1 (q = 6, 13, 14, 17, 18) from the plane
above.  Each population's plane is contiguous in this layout, so the
exchange after every step sends ten contiguous planes per interior face
(five each way) with no packing: NCCL point-to-point over NVLink on GPUs,
gloo on CPU.

The local step is the library's fused step on the whole local array with a
non-periodic z axis (x and y as on the global grid).  The real planes then
pull across into the ghost planes, which hold exactly the neighbour's
populations; the ghost planes themselves are updated with meaningless
values that nothing reads and the next exchange overwrites; a slab that
ends at a global z wall keeps the step's own half-way bounce-back there.
Every storage and kernel variant of kb_fused_trt_step_3d thus runs
unchanged, and a round-to-nearest storage gives the full-grid result bit
for bit.  The cost is two ghost planes of work per slab.

A D2Q9 grid splits the same way along y (`SlabD2Q9`): `Slab` then counts
rows, the local arrays are (9, ny_alloc, Nx), and three populations cross
each face, c_y = +1 (q = 2, 5, 6) and c_y = -1 (q = 4, 7, 8), each one
contiguous row.  The fused 2D steps wall all four sides, so the split is of
a walled y axis.
"""
from __future__ import annotations

from dataclasses import dataclass

# populations that cross a z face upward (c_z = +1) and downward (c_z = -1)
CZP = (5, 11, 12, 15, 16)
CZM = (6, 13, 14, 17, 18)
# D2Q9 populations that cross a y face upward (c_y = +1) and downward
CYP = (2, 5, 6)
CYM = (4, 7, 8)


@dataclass(frozen=True)
class Slab:
    """Rank `rank`'s part of a grid of `Nz` planes split over `world` ranks."""

    Nz: int
    world: int
    rank: int
    periodic_z: bool

    def __post_init__(self):
        if self.world < 1 or not 0 <= self.rank < self.world:
            raise ValueError(f"bad rank {self.rank} of world {self.world}")
        if self.Nz < self.world:
            raise ValueError(f"{self.Nz} z-planes cannot be split over {self.world} ranks")

    @property
    def z0(self) -> int:
        """First global z-plane of this slab (planes split as evenly as possible)."""
        q, r = divmod(self.Nz, self.world)
        return self.rank * q + min(self.rank, r)

    @property
    def z1(self) -> int:
        q, r = divmod(self.Nz, self.world)
        return self.z0 + q + (1 if self.rank < r else 0)

    @property
    def nz(self) -> int:
        """Real planes of this slab."""
        return self.z1 - self.z0

    @property
    def lo(self) -> bool:
        """A ghost plane below (a neighbouring slab under this one)."""
        return self.periodic_z or self.rank > 0

    @property
    def hi(self) -> bool:
        """A ghost plane above."""
        return self.periodic_z or self.rank < self.world - 1

    @property
    def nz_alloc(self) -> int:
        """Planes of the local arrays: real planes plus ghosts."""
        return self.nz + int(self.lo) + int(self.hi)

    @property
    def k0(self) -> int:
        """Local index of the first real plane."""
        return int(self.lo)

    @property
    def up(self) -> int:
        return (self.rank + 1) % self.world

    @property
    def down(self) -> int:
        return (self.rank - 1) % self.world

    def global_planes(self):
        """Global z index of every local plane (ghosts included, wrapped)."""
        return [(self.z0 - self.k0 + k) % self.Nz for k in range(self.nz_alloc)]

    def local_from_global(self, full, axis=-3):
        """The local array (ghosts filled) cut from a full-grid array whose
        split axis is dimension `axis`: -3 for z in (Q, Nz, Ny, Nx) or
        (Nz, Ny, Nx), -2 for y in the D2Q9 (Q, Ny, Nx) or (Ny, Nx)."""
        idx = (Ellipsis, self.global_planes()) + (slice(None),) * (-axis - 1)
        return full[idx].clone() if hasattr(full, "clone") else full[idx].copy()

    def real(self, local, axis=-3):
        """View of the real planes (rows) of a local array."""
        idx = (Ellipsis, slice(self.k0, self.k0 + self.nz)) + (slice(None),) * (-axis - 1)
        return local[idx]


def exchange(f, slab: Slab, group=None, cross=(CZP, CZM)):
    """Fill the ghost planes of the local populations `f` (19, nz_alloc, Ny,
    Nx) from the neighbouring slabs, after a step wrote `f`.  With one rank
    the ghosts of a periodic z axis are copies of the slab's own end planes.
    Every rank must call this at the same point of its step sequence.
    `cross` names the populations that cross a face upward and downward
    (CZP, CZM for D3Q19 z-slabs; CYP, CYM for D2Q9 y-slabs, f (9, ny_alloc,
    Nx))."""
    if slab.world == 1:
        if not (slab.lo or slab.hi):
            return
        if getattr(f, "is_cuda", False) and f.dim() == 4 and cross == (CZP, CZM):
            # one launch for the ten planes
            import torch
            from . import ops
            ops.slab_fill_ghosts_3d_(f, slab.lo, slab.hi,
                                     deviation=f.dtype in (torch.float16, torch.bfloat16))
            return
        exchange_in_process([f], [slab], cross)
        return
    # one fixed order on every rank (exchange_start): upward sends, upward
    # receives, downward sends, downward receives, each in population order,
    # so the matching per peer pair is the same even when up == down (two
    # ranks)
    for req in exchange_start(f, slab, group, cross):
        req.wait()


def exchange_start(f, slab: Slab, group=None, cross=(CZP, CZM)):
    """`exchange` without the wait: the point-to-point operations are
    posted and their requests returned (an empty list when there is nothing
    in flight, e.g. one rank, where the ghosts are filled at once).  Wait on
    every request before the next step reads `f`'s ghost planes.  On NCCL
    the transfers run on the communicator's stream after the work already
    queued on the current stream, so kernels launched afterwards overlap
    them."""
    if slab.world == 1:
        exchange(f, slab, group, cross)
        return []
    import torch.distributed as dist
    top, bot, ghost_hi = slab.k0 + slab.nz - 1, slab.k0, slab.nz_alloc - 1
    cp, cm = cross
    p2p = []
    if slab.hi:
        p2p += [dist.P2POp(dist.isend, f[q, top], slab.up, group) for q in cp]
    if slab.lo:
        p2p += [dist.P2POp(dist.irecv, f[q, 0], slab.down, group) for q in cp]
    if slab.lo:
        p2p += [dist.P2POp(dist.isend, f[q, bot], slab.down, group) for q in cm]
    if slab.hi:
        p2p += [dist.P2POp(dist.irecv, f[q, ghost_hi], slab.up, group) for q in cm]
    return dist.batch_isend_irecv(p2p) if p2p else []


def exchange_in_process(fs, slabs, cross=(CZP, CZM)):
    """The exchange of `exchange` for all slabs of one grid held by one
    process (a list of local arrays, one per slab, e.g. to run a grid in
    slabs on one GPU or to check the decomposition against the full grid)."""
    R = len(slabs)
    for r, (f, s) in enumerate(zip(fs, slabs)):
        if s.lo:
            below, sb = fs[(r - 1) % R], slabs[(r - 1) % R]
            for q in cross[0]:
                f[q, 0] = below[q, sb.k0 + sb.nz - 1]
        if s.hi:
            above, sa = fs[(r + 1) % R], slabs[(r + 1) % R]
            for q in cross[1]:
                f[q, s.nz_alloc - 1] = above[q, sa.k0]


class SlabTRT3D:
    """The fused D3Q19 TRT step of one slab: kb_fused_trt_step_3d on the
    local array (z non-periodic), then the ghost exchange of its output.

    `step_fn(f_out, f_in, moments, mask)` replaces the library step (a test
    plugs the oracle in here); by default the CUDA step runs with the given
    nu, Lambda, x/y periodicity, storage options.  `moments` is None or four
    local (nz_alloc, Ny, Nx) arrays whose real planes receive rho, ux, uy,
    uz."""

    def __init__(self, slab: Slab, Nx, Ny, nu=None, Lambda=3 / 16, periodic_xy=(False, False),
                 deviation=False, stochastic_rounding=False, mask=None, group=None,
                 step_fn=None, range_fn=None):
        self.slab, self.Nx, self.Ny = slab, Nx, Ny
        self.mask, self.group = mask, group
        if step_fn is None:
            from . import ops
            per = (bool(periodic_xy[0]), bool(periodic_xy[1]), False)

            def step_fn(f_out, f_in, moments, mask):
                m = moments if moments is not None else (None,) * 4
                ops.fused_trt_step_3d_(f_out, f_in, *m, mask, Nx, Ny, slab.nz_alloc, nu, Lambda,
                                       periodic=per, deviation=deviation,
                                       stochastic_rounding=stochastic_rounding)

            def range_fn(f_out, f_in, moments, mask, k_begin, k_end):
                m = moments if moments is not None else (None,) * 4
                ops.fused_trt_step_3d_zrange_(f_out, f_in, *m, mask, Nx, Ny, slab.nz_alloc,
                                              k_begin, k_end, nu, Lambda, periodic_xy=per[:2],
                                              deviation=deviation,
                                              stochastic_rounding=stochastic_rounding)
        self.step_fn, self.range_fn = step_fn, range_fn
        self._side = None  # CUDA side stream of step_overlapped, made on first use

    def shape(self):
        return (19, self.slab.nz_alloc, self.Ny, self.Nx)

    def step(self, f_out, f_in, moments=None):
        """One step f_in -> f_out; afterwards f_out's ghosts are current."""
        self.step_fn(f_out, f_in, moments, self.mask)
        exchange(f_out, self.slab, self.group)

    def overlapped(self) -> bool:
        """True when step_overlapped splits the step: the slab has ghost
        planes on both faces (no global z wall) and a range step exists."""
        return self.range_fn is not None and self.slab.lo and self.slab.hi

    def step_overlapped(self, f_out, f_in, moments=None):
        """`step` with the exchange overlapped: the two real planes next to
        the faces are stepped first, their crossing populations are posted
        to the neighbours, and the interior planes are stepped while they
        travel.  Identical real planes to `step` for round-to-nearest
        storages; the non-crossing populations of f_out's ghost planes are
        left as they were (nothing reads them).  Falls back to `step` on a
        slab that ends at a global z wall."""
        if not self.overlapped():
            return self.step(f_out, f_in, moments)
        s = self.slab
        bot, top = s.k0, s.k0 + s.nz - 1

        def faces():
            self.range_fn(f_out, f_in, moments, self.mask, bot, bot + 1)
            if top > bot:
                self.range_fn(f_out, f_in, moments, self.mask, top, top + 1)
            return exchange_start(f_out, s, self.group)

        if not getattr(f_out, "is_cuda", False):
            reqs = faces()
            if top - bot > 1:
                self.range_fn(f_out, f_in, moments, self.mask, bot + 1, top)
            for req in reqs:
                req.wait()
            return
        # on the GPU the face planes and their exchange run on a side stream
        # beside the interior planes: both read only f_in and write disjoint
        # planes of f_out, and the current stream joins the side stream
        # before anything later reads f_out
        import torch
        main = torch.cuda.current_stream()
        if self._side is None or self._side.device != main.device:
            self._side = torch.cuda.Stream(device=main.device)
        side = self._side
        side.wait_stream(main)
        with torch.cuda.stream(side):
            reqs = faces()
        if top - bot > 1:
            self.range_fn(f_out, f_in, moments, self.mask, bot + 1, top)
        with torch.cuda.stream(side):
            for req in reqs:
                req.wait()
        main.wait_stream(side)


class SlabD2Q9:
    """One y-slab of a walled D2Q9 grid: the library's fused 2D step on the
    local array (9, ny_alloc, Nx), then the exchange of the three crossing
    populations per face (CYP up, CYM down).  The fused 2D steps wall every
    side of their grid, so the real rows pull across into the ghost rows
    (the neighbour's populations) and a slab at a global y wall keeps the
    step's own wall; the real rows equal the full-grid step bit for bit.

    kind: "bgk" (fused_bgk_step!, omega), "trt" (fused_trt_step!, nu and
    Lambda), "cavity" (the one-launch run_cavity_2d step, omega and u_lid;
    the lid is the top slab's top row) or "movingwall" (the moving-wall
    half-way bounce-back lid).  `step_fn(f_out, f_in, moments, mask)`
    replaces the library step (a test plugs the oracle in here).
    `moments` is None or three local (ny_alloc, Nx) arrays rho, ux, uy; the
    2D fused steps always write them, so the slab keeps scratch ones."""

    KINDS = ("bgk", "trt", "cavity", "movingwall")

    def __init__(self, slab: Slab, Nx, kind="bgk", omega=None, nu=None, Lambda=3 / 16,
                 u_lid=0.0, mask=None, group=None, step_fn=None):
        if slab.periodic_z:
            raise ValueError("the fused D2Q9 steps wall the y axis: a y-slab split cannot be "
                             "periodic")
        if kind not in self.KINDS:
            raise ValueError(f"kind must be one of {self.KINDS}")
        self.slab, self.Nx, self.kind = slab, Nx, kind
        self.mask, self.group = mask, group
        self._scratch = None
        if step_fn is None:
            from . import ops
            ny = slab.nz_alloc

            def step_fn(f_out, f_in, moments, mask):
                rho, ux, uy = moments
                if kind == "bgk":
                    ops.fused_bgk_step_(f_out, f_in, rho, ux, uy, mask, Nx, ny, omega)
                elif kind == "trt":
                    ops.fused_trt_step_(f_out, f_in, rho, ux, uy, mask, Nx, ny, nu, Lambda)
                elif kind == "cavity":
                    ops.cavity_step_2d_(f_out, f_in, rho, ux, uy, mask, Nx, ny, omega, u_lid)
                else:
                    ops.cavity_movingwall_step_2d_(f_out, f_in, rho, ux, uy, mask, Nx, ny,
                                                   omega, u_lid)
        self.step_fn = step_fn

    def shape(self):
        return (9, self.slab.nz_alloc, self.Nx)

    def step(self, f_out, f_in, moments=None):
        """One step f_in -> f_out; afterwards f_out's ghost rows are current."""
        if moments is None:
            if self._scratch is None or self._scratch[0].dtype != f_in.dtype:
                import torch
                self._scratch = [torch.empty((self.slab.nz_alloc, self.Nx), dtype=f_in.dtype,
                                             device=f_in.device) for _ in range(3)]
            moments = self._scratch
        self.step_fn(f_out, f_in, moments, self.mask)
        exchange(f_out, self.slab, self.group, (CYP, CYM))
