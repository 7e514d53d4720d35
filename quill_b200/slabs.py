"""One box cut along x into overlapping slab regions: the reference's
multi-process layout (n_sr regions, one per MPI rank), rebuilt on the
library's slab entry points.

* Layout (main.cpp:2232-2262): neighbouring regions overlap by
  ``NX_ICH = 8`` cells; region r covers global cells
  ``[x0[r], x0[r] + nx[r])`` with ``x0[r] = x0[r-1] + nx[r-1] - NX_ICH``.
  The left half of an overlap belongs to the left region, the right half to
  the right one (``NM = NX_ICH / 2``), and each region's diagnostics count
  only the cells it owns: ``[NM*(r>0), nx[r] - NM*(r<n-1))``
  (compute_N / compute_energy with n1, n2, main.cpp:2325-2327).
* Exchange (synchronize_regions, main.cpp:1286-1514): after every step the
  owned cells next to an overlap overwrite the neighbour's copies, fields
  (E, B, J, Bbar) first, then the cell lists.  Region r sends its cells
  ``[nm1, nm1 + nm2)`` to r-1, which puts them in ``[nx - nm2, nx)``, and its
  cells ``[nx - nm2 - nm1, nx - nm2)`` to r+1, which puts them in
  ``[0, nm1)``; nm1 = nm2 = NM, or NM-1, NM+1 after a moving-window shift.
  A particle that changes region moves its x by the offset of the two
  frames, ``x + (x0[src] - x0[dst])`` (plist::xplus, containers.cpp:78-87).
* Load balancing (load_balancing, main.cpp:2155-2184, and balancing.cpp):
  layer weights ``ny*nz + particle_weight * (particles in the layer)``, the
  min-max partition by dynamic programming, clamped so that each new region
  still overlaps its old self, and a resize in which every cell of a new
  region comes from one old region (resize_field / resize_particles,
  main.cpp:1962-2153).

Regions are duck-typed: :class:`quill_b200.api.Region` (one per GPU, or
several on one GPU) or any object with the same slab methods.  Exchange
goes through a communicator: :class:`LocalComm` when one process holds every
region, :class:`TorchComm` (torch.distributed point-to-point, NCCL over
NVLink for device payloads or gloo for host payloads) when each rank holds
one.  The exchange is the path's only data movement between regions; the
diagnostics are summed over regions.
"""
from __future__ import annotations

import numpy as np

NX_ICH = 8
NM = NX_ICH // 2


# ----------------------------------------------------------------------------
# layout
# ----------------------------------------------------------------------------
class SlabLayout:
    """x0 and nx of each region of a box of ``nx_global`` cells."""

    def __init__(self, nx_global: int, x0, nx):
        self.nx_global = int(nx_global)
        self.x0 = [int(v) for v in x0]
        self.nx = [int(v) for v in nx]
        self.n = len(self.x0)
        for r in range(self.n):
            if self.nx[r] < 2 * NX_ICH - (NX_ICH if (r == 0 or r == self.n - 1) else 0):
                raise ValueError(f"region {r} is narrower than its overlaps")
        if self.x0[0] != 0 or self.x0[-1] + self.nx[-1] != self.nx_global:
            raise ValueError("regions do not cover the box")
        for r in range(1, self.n):
            if self.x0[r] != self.x0[r - 1] + self.nx[r - 1] - NX_ICH:
                raise ValueError("neighbouring regions must overlap by NX_ICH cells")

    @classmethod
    def even(cls, nx_global: int, n: int) -> "SlabLayout":
        """The start-up layout (main.cpp:2252-2266)."""
        if n < 1:
            raise ValueError("at least one region")
        if NX_ICH * (n - 1) >= nx_global:
            raise ValueError("too many slices")
        total = nx_global + NX_ICH * (n - 1)
        nx = [total // n] * n
        for i in range(total % n):
            nx[i] += 1
        x0 = [0] * n
        for i in range(1, n):
            x0[i] = x0[i - 1] + nx[i - 1] - NX_ICH
        return cls(nx_global, x0, nx)

    @classmethod
    def from_partition(cls, nx_global: int, partition) -> "SlabLayout":
        """Region sizes for left borders ``partition`` (resize_regions,
        main.cpp:2126-2153)."""
        p = [int(v) for v in partition]
        nx = [p[i + 1] + NX_ICH - p[i] for i in range(len(p) - 1)] + [nx_global - p[-1]]
        return cls(nx_global, p, nx)

    def diag_range(self, r: int):
        """Owned cells of region r, local indices [lo, hi)."""
        return (NM if r > 0 else 0, self.nx[r] - (NM if r < self.n - 1 else 0))

    def owned(self, r: int):
        """Owned cells of region r, global indices [lo, hi)."""
        lo, hi = self.diag_range(r)
        return self.x0[r] + lo, self.x0[r] + hi


# ----------------------------------------------------------------------------
# load balancing (balancing.cpp)
# ----------------------------------------------------------------------------
def _acc(w, a: int, b: int) -> float:
    """std::accumulate over w[a:b] from 0.0, left to right (Python's sum()
    compensates, which would change the last bits)."""
    s = 0.0
    for i in range(a, b):
        s += w[i]
    return s


def optimal_partition(weights, regions: int, overlap: int = NX_ICH) -> list:
    """Left borders of ``regions`` regions that minimise the heaviest region
    (calculate_optimal_partition, balancing.cpp:54-115): max_weight[k][i] is
    the least possible heaviest region when regions 0..k cover layers
    [0, i], side regions at least ``overlap`` layers, middle ones at least
    2*overlap, and a region's weight includes the overlap it shares with
    the next region."""
    if regions == 1:
        return [0]
    w = [float(v) for v in weights]
    size = len(w)
    mw = [[0.0] * size for _ in range(regions)]
    lb = [[0] * size for _ in range(regions)]
    side, middle = overlap, 2 * overlap

    def best(k, i, initial_left, minimum_left):
        cw = _acc(w, initial_left, i + 1)
        mw[k][i] = max(cw, mw[k - 1][initial_left + overlap - 1])
        lb[k][i] = initial_left + overlap - 1
        for left in range(initial_left - 1, minimum_left - 1, -1):
            cw += w[left]
            cm = max(cw, mw[k - 1][left + overlap - 1])
            if cm < mw[k][i]:
                mw[k][i] = cm
                lb[k][i] = left + overlap - 1
            if cw > mw[k][i]:
                break

    mw[0][side - 1] = _acc(w, 0, side)
    for i in range(side, size):
        mw[0][i] = mw[0][i - 1] + w[i]
        for k in range(1, regions - 1):
            if i < (k + 1) * overlap - 1:
                break
            best(k, i, i - middle + 1, (k - 1) * overlap)
    k, i = regions - 1, size - 1
    best(k, i, size - side, (regions - 2) * overlap)
    # retrieve_partition (balancing.cpp:42-52)
    out = []
    border = lb[k][i]
    while k > 0:
        out.append(border - overlap + 1)
        border = lb[k - 1][border]
        k -= 1
    out.append(border)
    return out[::-1]


def partition_weights(weights, partition, overlap: int = NX_ICH) -> list:
    """calculate_partition_weights (balancing.cpp:117-126)."""
    w = [float(v) for v in weights]
    n = len(partition)
    out = [_acc(w, partition[i], partition[i + 1] + overlap) for i in range(n - 1)]
    out.append(_acc(w, partition[-1], len(w)))
    return out


def partition_imbalance(weights, partition, overlap: int = NX_ICH) -> float:
    """max / min - 1 of the region weights (balancing.cpp:128-134)."""
    pw = partition_weights(weights, partition, overlap)
    return max(pw) / min(pw) - 1.0


def normalize_partition(old, new, overlap: int = NX_ICH) -> list:
    """Clamp a new partition so that each new region overlaps its old self
    and regions stay ``overlap`` apart (normalize_new_partition,
    balancing.cpp:136-175)."""
    if old[0] != 0 or new[0] != 0 or len(old) != len(new):
        raise ValueError("partitions must start at 0 and have the same length")
    n = len(old)
    if n == 1:
        return list(new)
    out = [0] * n
    out[0] = new[0]
    for i in range(1, n - 1):
        out[i] = new[i]
        if new[i] < old[i - 1]:
            out[i] = old[i - 1]
        if new[i] > old[i + 1]:
            out[i] = old[i + 1]
        if out[i] < out[i - 1] + overlap:
            out[i] = out[i - 1] + overlap
    i = n - 1
    out[i] = new[i]
    if new[i] < old[i - 1]:
        out[i] = old[i - 1]
    if out[i] < out[i - 1] + overlap:
        out[i] = out[i - 1] + overlap
    return out


# ----------------------------------------------------------------------------
# communicators
# ----------------------------------------------------------------------------
class LocalComm:
    """Every region in this process: messages are handed over directly.
    With a CUDA ``device`` the library regions exchange device buffers
    (several regions on one GPU, or on the GPUs of one process)."""

    n_ranks = 1

    def __init__(self, device=None):
        if device is None:
            self.device = None
        else:
            import torch
            self.device = torch.device(device)

    def local_regions(self, n: int):
        return list(range(n))

    def route(self, out: dict, n: int) -> dict:
        return dict(out)

    def allsum(self, v: np.ndarray) -> np.ndarray:
        return v


class TorchComm:
    """One region per rank of the default torch.distributed process group;
    messages go point to point between neighbouring ranks.  ``device`` is
    where payloads travel: a CUDA device for NCCL, "cpu" for gloo."""

    def __init__(self, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.rank = dist.get_rank()
        self.n_ranks = dist.get_world_size()
        if device is None:
            device = f"cuda:{torch.cuda.current_device()}" if dist.get_backend() == "nccl" else "cpu"
        self.device = torch.device(device)

    def local_regions(self, n: int):
        if n != self.n_ranks:
            raise ValueError(f"{n} regions on {self.n_ranks} ranks: one region per rank")
        return [self.rank]

    def _t(self, a):
        torch = self.torch
        if isinstance(a, torch.Tensor):
            return a.reshape(-1).to(self.device, torch.float64)
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).reshape(-1)).to(self.device)

    def route(self, out: dict, n: int) -> dict:
        """``out[(src, dst)]`` = list of float64 arrays from this rank to a
        neighbour.  Every neighbour pair exchanges a message both ways (an
        empty list if there is nothing to send), lengths first."""
        torch, dist = self.torch, self.dist
        me = self.rank
        nbrs = [p for p in (me - 1, me + 1) if 0 <= p < n]
        metas_out, metas_in = {}, {}
        MAXA = 64
        for p in nbrs:
            arrs = out.get((me, p), [])
            if len(arrs) >= MAXA:
                raise ValueError("too many arrays in one message")
            m = torch.zeros(MAXA, dtype=torch.int64)
            m[0] = len(arrs)
            for i, a in enumerate(arrs):
                m[1 + i] = int(np.prod(a.shape)) if not isinstance(a, torch.Tensor) else a.numel()
            metas_out[p] = m.to(self.device)
            metas_in[p] = torch.zeros(MAXA, dtype=torch.int64, device=self.device)
        self._exchange({p: metas_out[p] for p in nbrs}, metas_in)
        # the received lengths size the receive buffers: one copy to the host
        # for both neighbours
        host = torch.stack([metas_in[p] for p in nbrs]).cpu() if nbrs else None
        data_out, data_in, lens_in = {}, {}, {}
        for q, p in enumerate(nbrs):
            arrs = out.get((me, p), [])
            flat = [self._t(a) for a in arrs]
            data_out[p] = torch.cat(flat) if flat else torch.zeros(0, dtype=torch.float64, device=self.device)
            mi = host[q]
            lens = [int(v) for v in mi[1:1 + int(mi[0])]]
            lens_in[p] = lens
            data_in[p] = torch.empty(sum(lens), dtype=torch.float64, device=self.device)
        self._exchange(data_out, data_in)
        res = {}
        for p in nbrs:
            parts, o = [], 0
            for ln in lens_in[p]:
                parts.append(data_in[p][o:o + ln])
                o += ln
            res[(p, me)] = parts
        return res

    def _exchange(self, send: dict, recv: dict):
        dist = self.dist
        ops = []
        for p, t in send.items():
            if t.numel():
                ops.append(dist.P2POp(dist.isend, t, p))
        for p, t in recv.items():
            if t.numel():
                ops.append(dist.P2POp(dist.irecv, t, p))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def allsum(self, v: np.ndarray) -> np.ndarray:
        """Sum over ranks in rank order (the in-process order, so that both
        exchanges give the same bits)."""
        t = self.torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).to(self.device)
        parts = [self.torch.empty_like(t) for _ in range(self.n_ranks)]
        self.dist.all_gather(parts, t)
        acc = parts[0].cpu().numpy().copy()
        for p in parts[1:]:
            acc = acc + p.cpu().numpy()
        return acc


# ----------------------------------------------------------------------------
# a box of slab regions
# ----------------------------------------------------------------------------
def _payload(a, comm):
    """Arrays as the communicator wants them: torch tensors on its device
    when it has one, numpy arrays otherwise."""
    if comm.device is None or comm.device.type == "cpu":
        return a.cpu().numpy() if hasattr(a, "cpu") else a
    return a


def _for_region(a, reg):
    """A received array as the region takes it: library regions take numpy
    or torch (host or device); other regions take numpy."""
    if hasattr(reg, "lib") or not hasattr(a, "cpu"):
        return a
    return a.cpu().numpy()


class SlabBox:
    """A box of ``layout.n`` slab regions; this process holds
    ``comm.local_regions(n)`` of them.

    ``make_region(r, nx_local)`` returns an empty region (zero fields, no
    particles) of ``nx_local`` x-cells for slot r; it is called again when
    load balancing resizes a region.  Every region must expose
    ``species_ids`` and the slab methods of :class:`quill_b200.api.Region`.
    """

    def __init__(self, layout: SlabLayout, make_region, comm=None):
        self.layout = layout
        self.make_region = make_region
        self.comm = comm or LocalComm()
        self.local = self.comm.local_regions(layout.n)
        self.regions = {r: make_region(r, layout.nx[r]) for r in self.local}
        for r in self.local:
            self.regions[r].set_diag_range(*layout.diag_range(r))
        self.species_ids = self.regions[self.local[0]].species_ids

    # --- loading ------------------------------------------------------------
    def set_fields(self, planes6):
        """Global E, B planes (6, nx_global, ny, nz): each region takes its
        cells."""
        for r in self.local:
            a, b = self.layout.x0[r], self.layout.x0[r] + self.layout.nx[r]
            self.regions[r].set_fields(*[np.ascontiguousarray(p[a:b]) for p in planes6])

    def init_boundaries(self):
        for r in self.local:
            self.regions[r].init_boundaries()

    def add_particles(self, species, parts: dict):
        """Global particles (x in global cell units): each region takes
        those inside its cells, x shifted to its frame."""
        x = np.asarray(parts["x"])
        for r in self.local:
            a, b = self.layout.x0[r], self.layout.x0[r] + self.layout.nx[r]
            sel = (x >= a) & (x < b)
            if not sel.any():
                continue
            p = {k: np.asarray(v)[sel] for k, v in parts.items() if v is not None}
            p["x"] = p["x"] - float(a)
            reg = self.regions[r]
            if species is None:
                reg.add_particles(p)
            else:
                reg.add_particles(species, p)

    # --- the time loop --------------------------------------------------------
    def _step_region(self, reg, external_bz) -> np.ndarray:
        d = reg.step(1, external_bz)
        row = d[0]
        return row.as_array() if hasattr(row, "as_array") else np.asarray(row, dtype=np.float64)

    def step(self, nsteps: int = 1, external_bz: float = 0.0, moving_window: bool = False) -> np.ndarray:
        """``nsteps`` steps of every region, each followed by the exchange
        (main.cpp:2319-2342).  With ``moving_window`` every step also shifts
        the box by one cell before its exchange.  Returns the diagnostics
        summed over regions, one row per step."""
        rows = []
        for _ in range(nsteps):
            acc = None
            for r in self.local:
                d = self._step_region(self.regions[r], external_bz)
                acc = d if acc is None else acc + d
            rows.append(self.comm.allsum(acc))
            if moving_window:
                for r in self.local:
                    self.regions[r].moving_window()
                self.synchronize(NM - 1, NM + 1)
            else:
                self.synchronize(NM, NM)
        return np.array(rows)

    def synchronize(self, nm1: int = NM, nm2: int = NM):
        """synchronize_regions (main.cpp:1493-1506): fields, then particles."""
        L = self.layout
        n = L.n
        out = {}
        for r in self.local:
            reg = self.regions[r]
            if r > 0:
                out[(r, r - 1)] = [_payload(reg.get_field_slab(nm1, nm2, **self._dev_kw(reg, nm2)), self.comm)]
            if r < n - 1:
                out[(r, r + 1)] = [_payload(reg.get_field_slab(L.nx[r] - nm2 - nm1, nm1, **self._dev_kw(reg, nm1)),
                                            self.comm)]
        for (src, dst), arrs in self.comm.route(out, n).items():
            if dst not in self.regions:
                continue
            i0 = L.nx[dst] - nm2 if src == dst + 1 else 0
            self.regions[dst].set_field_slab(i0, _for_region(arrs[0], self.regions[dst]))
        self._move_particles(
            {(r, r - 1): (nm1, nm2) for r in self.local if r > 0} |
            {(r, r + 1): (L.nx[r] - nm2 - nm1, nm1) for r in self.local if r < n - 1},
            lambda src, dst: (L.nx[dst] - nm2, nm2) if src == dst + 1 else (0, nm1),
            L, L)

    def _dev_kw(self, reg, width):
        """Device output buffer for a field slab when payloads travel on a
        GPU and the region is a library region."""
        dev = self.comm.device
        if dev is None or dev.type == "cpu" or not hasattr(reg, "lib"):
            return {}
        import torch
        return {"out": torch.empty((12, width) + tuple(reg.shape[1:]), dtype=torch.float64, device=dev)}

    def _get_particles(self, reg, species, i0, width):
        dev = self.comm.device
        if dev is not None and dev.type != "cpu" and hasattr(reg, "lib"):
            return reg.get_particle_slab(species, i0, width, device=dev)
        return reg.get_particle_slab(species, i0, width)

    def _move_particles(self, sends: dict, recv_slab, old: SlabLayout, new: SlabLayout, regions_new=None):
        """Send the particles of slab ``sends[(src, dst)] = (i0, width)`` of
        each local region to region dst, which replaces its slab
        ``recv_slab(src, dst)`` with them, x moved from the frame of
        old.x0[src] to that of new.x0[dst]."""
        keys = None
        out = {}
        for (src, dst), (i0, width) in sends.items():
            reg = self.regions[src]
            arrs = []
            for s in self.species_ids:
                p = self._get_particles(reg, s, i0, width)
                keys = [k for k in p]
                arrs += [_payload(p[k], self.comm) for k in keys]
            out[(src, dst)] = arrs
        if keys is None:
            # every rank needs the key order of its region type
            reg = self.regions[self.local[0]]
            keys = list(self._get_particles(reg, self.species_ids[0], 0, 0).keys())
        nk = len(keys)
        dst_regions = regions_new if regions_new is not None else self.regions
        for (src, dst), arrs in self.comm.route(out, old.n).items():
            if dst not in dst_regions or not arrs:
                continue
            i0, width = recv_slab(src, dst)
            shift = float(old.x0[src] - new.x0[dst])
            reg = dst_regions[dst]
            for si, s in enumerate(self.species_ids):
                p = {k: _for_region(arrs[si * nk + j], reg) for j, k in enumerate(keys)}
                p["x"] = p["x"] + shift  # plist::xplus
                reg.replace_particle_slab(s, i0, width, p)

    # --- load balancing -------------------------------------------------------
    def layer_weights(self, particle_weight: float = 1.0) -> np.ndarray:
        """Weights of the box's x-layers (calculate_global_layer_weights,
        main.cpp:997-1024): each region reports the layers it owns."""
        L = self.layout
        g = np.zeros(L.nx_global)
        for r in self.local:
            reg = self.regions[r]
            ny, nz = reg.shape[1], reg.shape[2]
            w = float(ny * nz) + particle_weight * reg.layer_counts().astype(np.float64)
            left = 0 if r == 0 else NX_ICH // 2
            right = L.nx[r] if r == L.n - 1 else L.nx[r] - NX_ICH // 2
            g[L.x0[r] + left:L.x0[r] + right] = w[left:right]
        return self.comm.allsum(g)

    def balance(self, threshold: float, particle_weight: float = 1.0):
        """load_balancing (main.cpp:2155-2184): repartition when the
        imbalance exceeds ``threshold``.  Returns (imbalance before, after
        or None)."""
        w = self.layer_weights(particle_weight)
        before = partition_imbalance(w, self.layout.x0)
        if not before > threshold:
            return before, None
        new = normalize_partition(self.layout.x0, optimal_partition(w, self.layout.n), NX_ICH)
        self.resize(new)
        return before, partition_imbalance(w, new)

    def resize(self, partition):
        """resize_regions (main.cpp:2126-2153).  A region whose x0 and nx
        stay is kept; any other is rebuilt: E, B and Bbar and the cell lists
        of each of its cells come from one old region (its own old range,
        the left neighbour's cells left of it, the right neighbour's right
        of it), J starts at zero."""
        old = self.layout
        new = SlabLayout.from_partition(old.nx_global, partition)
        n = old.n
        changed = {r: (new.x0[r] != old.x0[r] or new.nx[r] != old.nx[r]) for r in range(n)}

        def ranges(src, dst):
            """Global cells region dst takes from old region src."""
            if src == dst:
                lo, hi = old.x0[src], old.x0[src] + old.nx[src]
            elif src == dst - 1:
                lo, hi = old.x0[src], old.x0[src] + old.nx[src] - NX_ICH
            else:
                lo, hi = old.x0[src] + NX_ICH, old.x0[src] + old.nx[src]
            lo, hi = max(lo, new.x0[dst]), min(hi, new.x0[dst] + new.nx[dst])
            return (lo, hi) if lo < hi else None

        for dst in range(n):
            if not changed[dst]:
                continue
            cover = np.zeros(new.nx[dst], dtype=bool)
            for src in (dst - 1, dst, dst + 1):
                if 0 <= src < n and (rg := ranges(src, dst)):
                    cover[rg[0] - new.x0[dst]:rg[1] - new.x0[dst]] = True
            if not cover.all():
                raise ValueError("new partition reaches beyond the neighbouring regions")

        fresh = {}
        for r in self.local:
            if changed[r]:
                fresh[r] = self.make_region(r, new.nx[r])
                fresh[r].set_diag_range(*new.diag_range(r))
        # fields
        out = {}
        for src in self.local:
            for dst in (src - 1, src + 1):
                if 0 <= dst < n and changed[dst] and (rg := ranges(src, dst)):
                    out[(src, dst)] = [_payload(self._field_cells(self.regions[src], rg[0] - old.x0[src],
                                                                  rg[1] - rg[0]), self.comm)]
        routed = self.comm.route(out, n)
        for dst in fresh:
            if rg := ranges(dst, dst):
                routed[(dst, dst)] = [self._field_cells(self.regions[dst], rg[0] - old.x0[dst], rg[1] - rg[0])]
        for (src, dst), arrs in routed.items():
            if dst in fresh and arrs:
                rg = ranges(src, dst)
                fresh[dst].set_field_slab(rg[0] - new.x0[dst], _for_region(arrs[0], fresh[dst]))
        # particles
        sends = {}
        for src in self.local:
            for dst in (src - 1, src, src + 1):
                if 0 <= dst < n and changed[dst] and (rg := ranges(src, dst)):
                    sends[(src, dst)] = (rg[0] - old.x0[src], rg[1] - rg[0])
        remote = {k: v for k, v in sends.items() if k[0] != k[1]}
        own = {k: v for k, v in sends.items() if k[0] == k[1]}

        def recv_slab(src, dst):
            rg = ranges(src, dst)
            return rg[0] - new.x0[dst], rg[1] - rg[0]

        self._move_particles(remote, recv_slab, old, new, regions_new=fresh)
        self._move_particles_local(own, recv_slab, old, new, fresh)
        for r, reg in fresh.items():
            self.regions[r].close() if hasattr(self.regions[r], "close") else None
            self.regions[r] = reg
        self.layout = new

    def _field_cells(self, reg, i0, width):
        """E, B, Bbar of a slab with J zeroed (a resized region's cj is a
        fresh array)."""
        f = reg.get_field_slab(i0, width)
        f = np.array(f.cpu() if hasattr(f, "cpu") else f, dtype=np.float64, copy=True)
        f[6:9] = 0.0
        return f

    def _move_particles_local(self, sends, recv_slab, old, new, fresh):
        for (src, dst), (i0, width) in sends.items():
            reg = self.regions[src]
            j0, w = recv_slab(src, dst)
            shift = float(old.x0[src] - new.x0[dst])
            for s in self.species_ids:
                p = reg.get_particle_slab(s, i0, width)
                p["x"] = p["x"] + shift
                fresh[dst].replace_particle_slab(s, j0, w, p)

    # --- reading back -----------------------------------------------------------
    def global_fields(self) -> np.ndarray:
        """(12, nx_global, ny, nz): each cell from the region that owns it
        (in-process boxes only)."""
        if set(self.local) != set(range(self.layout.n)):
            raise ValueError("global_fields needs every region in this process")
        parts = []
        for r in range(self.layout.n):
            lo, hi = self.layout.diag_range(r)
            parts.append(self.regions[r].get_fields()[:, lo:hi])
        return np.concatenate(parts, axis=1)

    def global_particles(self, species) -> dict:
        """The particles of the owned cells in global traversal order, x in
        global cell units (in-process boxes only)."""
        if set(self.local) != set(range(self.layout.n)):
            raise ValueError("global_particles needs every region in this process")
        out = {}
        for r in range(self.layout.n):
            lo, hi = self.layout.diag_range(r)
            p = self.regions[r].get_particle_slab(species, lo, hi - lo)
            p = {k: np.asarray(v.cpu() if hasattr(v, "cpu") else v) for k, v in p.items()}
            p["x"] = p["x"] + float(self.layout.x0[r])
            for k, v in p.items():
                out.setdefault(k, []).append(v)
        return {k: np.concatenate(v) for k, v in out.items()}

    def close(self):
        for reg in self.regions.values():
            if hasattr(reg, "close"):
                reg.close()
