"""Element partitions with halo faces for the multi-GPU form of the element update.

EDGE partitions the mesh (METIS in EDGE-V, mesh/Partition.cpp), splits every partition into inner
and send elements, and exchanges the face-projected time-integrated DOFs of the send faces once
per time step (AderDg.hpp:419-473 packs them in the local step, 675-684 reads the received ones in
the neighbour step; setup.inc:337-399). Here a partition is a contiguous range of the mesh's
element order (Z-order for ingested meshes, z-slabs for boxes). Each part numbers its owned
elements first and appends the remote face neighbours as ghost elements; the device kernels run on
the owned range only, and a ghost's face buffer entry is filled by the exchange: per step, after
the local kernel, every part packs the face rows of its send faces, sends them to the owning
neighbours, and unpacks what it receives into its ghosts' face slots before the neighbour kernel.

plan(mesh, n_parts) builds the per-part index tables.
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Part:
    rank: int
    lo: int                       # owned elements are the global range [lo, hi)
    hi: int
    owned: np.ndarray             # global ids of the owned elements in local order: send elements first
    n_send: int                   # owned elements with a face neighbour in another part (local 0 .. n_send)
    ghosts: np.ndarray            # global ids of the ghost elements (local ids n_owned ...)
    el_fa_el: np.ndarray          # [n_local][4] local neighbour ids (-1 none; ghost rows all -1)
    fid: np.ndarray               # [n_local][4]
    vid: np.ndarray               # [n_local][4]
    el_fa_type: np.ndarray        # [n_local][4] (ghost rows: outflow)
    send: dict = field(default_factory=dict)   # peer -> [n][2] (local owned element, face)
    recv: dict = field(default_factory=dict)   # peer -> [n][2] (local ghost element, face)

    @property
    def n_owned(self):
        return self.hi - self.lo

    @property
    def n_local(self):
        return self.n_owned + len(self.ghosts)

    def global_ids(self):
        return np.concatenate([self.owned, self.ghosts]).astype(np.int64)


def ranges(n_el, n_parts):
    """Contiguous, balanced element ranges: bounds [n_parts + 1]."""
    return np.linspace(0, n_el, n_parts + 1).round().astype(np.int64)


def plan(mesh, n_parts):
    """Per-part tables for a partition of the mesh's elements into contiguous ranges. Within a part
    the send elements (a face neighbour in another part) come first, as EDGE's send region follows
    its inner region in a separate range (setup.inc:337-399), so that their local step can run, and
    their face rows leave, before the inner elements' local step."""
    from .host import FACE_INNER, FACE_OUTFLOW
    bounds = ranges(mesh.n_el, n_parts)
    ne = mesh.el_fa_el.astype(np.int64)
    inner = (mesh.el_fa_type == FACE_INNER) & (ne >= 0)
    parts = []
    for p in range(n_parts):
        lo, hi = int(bounds[p]), int(bounds[p + 1])
        nb = ne[lo:hi]
        remote = inner[lo:hi] & ((nb < lo) | (nb >= hi))
        is_send = remote.any(axis=1)
        owned = np.concatenate([np.flatnonzero(is_send), np.flatnonzero(~is_send)]) + lo
        n_own = hi - lo
        loc_of = np.empty(n_own, np.int64)
        loc_of[owned - lo] = np.arange(n_own)
        ghosts = np.unique(nb[remote])
        g2l = {int(g): n_own + i for i, g in enumerate(ghosts)}
        n_local = n_own + len(ghosts)
        rows = owned - lo
        nbo, rmo, ino = nb[rows], remote[rows], inner[lo:hi][rows]
        el_fa_el = np.full((n_local, 4), -1, np.int32)
        mapped = np.where(ino & ~rmo, loc_of[np.clip(nbo - lo, 0, n_own - 1)], -1)
        for i, f in zip(*np.nonzero(rmo)):
            mapped[i, f] = g2l[int(nbo[i, f])]
        el_fa_el[:n_own] = mapped
        fid = np.zeros((n_local, 4), np.uint8)
        vid = np.zeros((n_local, 4), np.uint8)
        ty = np.full((n_local, 4), FACE_OUTFLOW, np.uint8)
        fid[:n_own] = mesh.fid[owned]
        vid[:n_own] = mesh.vid[owned]
        ty[:n_own] = mesh.el_fa_type[owned]
        part = Part(p, lo, hi, owned.astype(np.int64), int(is_send.sum()), ghosts.astype(np.int64), el_fa_el,
                    fid, vid, ty)
        # A neighbour reads face (element, its own face id) of this element's face buffer, so the
        # send list holds (owned element, face) pairs whose face neighbour lives in the peer, and the
        # peer stores them at (its ghost copy of the element, the same face). Both sides list the
        # pairs in ascending (global element, face) order.
        for q in range(n_parts):
            if q == p:
                continue
            qlo, qhi = int(bounds[q]), int(bounds[q + 1])
            i, f = np.nonzero(inner[lo:hi] & (nb >= qlo) & (nb < qhi))
            if len(i):
                order = np.lexsort((f, i))
                part.send[q] = np.stack([loc_of[i[order]], f[order]], 1).astype(np.int32)
            j, g = np.nonzero(inner[qlo:qhi] & (ne[qlo:qhi] >= lo) & (ne[qlo:qhi] < hi))
            if len(j):
                order = np.lexsort((g, j))
                ge = j[order] + qlo
                part.recv[q] = np.stack([[g2l[int(x)] for x in ge], g[order]], 1).astype(np.int32)
        parts.append(part)
    return parts


class PartSolver:
    """One part of a partition on a device: its solver (owned elements + ghosts), the device index
    lists of its send and receive faces, and packed face buffers per peer.

    Per step: phase0 (receivers, local, sources of the owned elements), pack() -> {peer: buffer},
    the transport moves each buffer to the peer (exchange_nccl between GPUs), unpack({peer: buffer})
    into the ghosts' face slots, phase1 (neighbour)."""

    def __init__(self, prob, part, precision=64, device=0, stream=None):
        import types

        import torch
        from . import host
        from ._lib import lib
        from .solver import Solver
        ids = part.global_ids()
        mesh = types.SimpleNamespace(n_el=part.n_local, el_fa_el=part.el_fa_el, fid=part.fid, vid=part.vid,
                                     el_fa_type=part.el_fa_type)
        take = lambda a, ax=0: None if a is None else np.ascontiguousarray(np.take(a, ids, axis=ax))
        local = host.Problem(order=prob.order, runs=prob.runs, rm=prob.rm, mesh=mesh, rho=take(prob.rho),
                             lam=take(prob.lam), mu=take(prob.mu), starE=take(prob.starE), fsE=take(prob.fsE, 1),
                             dt=prob.dt, starA=take(prob.starA), srcA=take(prob.srcA), fsA=take(prob.fsA, 1),
                             omega=prob.omega, name=f"part{part.rank}")
        self.part, self.prob = part, local
        self.solver = Solver(local, precision=precision, stream=stream, device=device)
        self.solver._chk(lib().edge_b200_set_owned(self.solver._h, part.n_owned), "set_owned")
        self.solver._chk(lib().edge_b200_set_send_count(self.solver._h, part.n_send), "set_send_count")
        self.block = lib().edge_b200_face_block_bytes(self.solver._h)
        dev = torch.device("cuda", device)
        slots = lambda lst: torch.from_numpy((lst[:, 0].astype(np.int64) * 4 + lst[:, 1]).astype(np.int32)).to(dev)
        self.send_slots = {q: slots(v) for q, v in part.send.items()}
        self.recv_slots = {q: slots(v) for q, v in part.recv.items()}
        self.send_buf = {q: torch.empty(len(v) * self.block, dtype=torch.uint8, device=dev) for q, v in part.send.items()}
        self.recv_buf = {q: torch.empty(len(v) * self.block, dtype=torch.uint8, device=dev) for q, v in part.recv.items()}

    def upload_owned(self, dofs_e_global):
        e = np.zeros((self.part.n_local,) + dofs_e_global.shape[1:], dofs_e_global.dtype)
        e[:self.part.n_owned] = dofs_e_global[self.part.owned]
        self.solver.upload_dofs(e)

    def download_owned(self):
        """DOFs of the owned elements in global order (elements lo .. hi)."""
        e, a = self.solver.download_dofs()
        idx = self.part.owned - self.part.lo
        out_e = np.empty_like(e[:self.part.n_owned])
        out_e[idx] = e[:self.part.n_owned]
        out_a = None
        if a is not None:
            out_a = np.empty_like(a[:self.part.n_owned])
            out_a[idx] = a[:self.part.n_owned]
        return out_e, out_a

    def phase0(self, t, dt):
        from ._lib import lib
        self.solver._chk(lib().edge_b200_step_phase(self.solver._h, t, dt, 0), "step_phase 0")

    def phase_send(self, t, dt):
        """Receivers and the local step of the send elements (their face rows can then be packed)."""
        from ._lib import lib
        self.solver._chk(lib().edge_b200_step_phase(self.solver._h, t, dt, 2), "step_phase 2")

    def phase_inner(self, t, dt):
        """The local step of the other owned elements and the sources (overlapping the exchange)."""
        from ._lib import lib
        self.solver._chk(lib().edge_b200_step_phase(self.solver._h, t, dt, 3), "step_phase 3")

    def phase1(self, t, dt):
        from ._lib import lib
        self.solver._chk(lib().edge_b200_step_phase(self.solver._h, t, dt, 1), "step_phase 1")

    def pack(self):
        from ._lib import lib
        for q, sl in self.send_slots.items():
            self.solver._chk(lib().edge_b200_pack_faces(self.solver._h, len(sl), sl.data_ptr(),
                                                        self.send_buf[q].data_ptr()), "pack_faces")
        return self.send_buf

    def unpack(self):
        from ._lib import lib
        for q, sl in self.recv_slots.items():
            self.solver._chk(lib().edge_b200_unpack_faces(self.solver._h, len(sl), sl.data_ptr(),
                                                          self.recv_buf[q].data_ptr()), "unpack_faces")

    def close(self):
        self.solver.close()


def exchange_nccl(ps, wait=True):
    """Moves this rank's packed send buffers to their peers' receive buffers (torch.distributed
    send / recv, NCCL between GPUs); every rank calls it once per step after pack(). The part's
    solver must run on torch's current stream (stream=None), which NCCL orders its copies after.
    wait=False returns the pending works: work queued on the stream after this call (the inner
    elements' local step) overlaps the transfer; wait on them before unpack()."""
    import torch.distributed as dist
    ops = [dist.P2POp(dist.isend, b, q) for q, b in sorted(ps.send_buf.items())]
    ops += [dist.P2POp(dist.irecv, b, q) for q, b in sorted(ps.recv_buf.items())]
    works = dist.batch_isend_irecv(ops) if ops else []
    if wait:
        for r in works:
            r.wait()
        return []
    return works


def step_overlapped(ps, t, dt):
    """One GTS step of a part with the halo exchange behind the inner elements' local step: send
    elements' local step, pack, NCCL transfer started, inner elements' local step (and sources),
    wait for the transfer, unpack into the ghosts' face slots, neighbour step."""
    ps.phase_send(t, dt)
    ps.pack()
    works = exchange_nccl(ps, wait=False)
    ps.phase_inner(t, dt)
    for r in works:
        r.wait()
    ps.unpack()
    ps.phase1(t, dt)
