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
        return np.concatenate([np.arange(self.lo, self.hi), self.ghosts]).astype(np.int64)


def ranges(n_el, n_parts):
    """Contiguous, balanced element ranges: bounds [n_parts + 1]."""
    return np.linspace(0, n_el, n_parts + 1).round().astype(np.int64)


def plan(mesh, n_parts):
    """Per-part tables for a partition of the mesh's elements into contiguous ranges."""
    from .host import FACE_INNER, FACE_OUTFLOW
    bounds = ranges(mesh.n_el, n_parts)
    ne = mesh.el_fa_el.astype(np.int64)
    inner = (mesh.el_fa_type == FACE_INNER) & (ne >= 0)
    parts = []
    for p in range(n_parts):
        lo, hi = int(bounds[p]), int(bounds[p + 1])
        nb = ne[lo:hi]
        remote = inner[lo:hi] & ((nb < lo) | (nb >= hi))
        ghosts = np.unique(nb[remote])
        g2l = {int(g): (hi - lo) + i for i, g in enumerate(ghosts)}
        n_local = (hi - lo) + len(ghosts)
        el_fa_el = np.full((n_local, 4), -1, np.int32)
        loc = np.where(inner[lo:hi], nb, -1)
        mapped = np.where((loc >= lo) & (loc < hi), loc - lo, -1)
        for i, f in zip(*np.nonzero(remote)):
            mapped[i, f] = g2l[int(nb[i, f])]
        el_fa_el[:hi - lo] = mapped
        fid = np.zeros((n_local, 4), np.uint8)
        vid = np.zeros((n_local, 4), np.uint8)
        ty = np.full((n_local, 4), FACE_OUTFLOW, np.uint8)
        fid[:hi - lo] = mesh.fid[lo:hi]
        vid[:hi - lo] = mesh.vid[lo:hi]
        ty[:hi - lo] = mesh.el_fa_type[lo:hi]
        part = Part(p, lo, hi, ghosts.astype(np.int64), el_fa_el, fid, vid, ty)
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
                part.send[q] = np.stack([i[order], f[order]], 1).astype(np.int32)
            j, g = np.nonzero(inner[qlo:qhi] & (ne[qlo:qhi] >= lo) & (ne[qlo:qhi] < hi))
            if len(j):
                order = np.lexsort((g, j))
                ge = j[order] + qlo
                part.recv[q] = np.stack([[g2l[int(x)] for x in ge], g[order]], 1).astype(np.int32)
        parts.append(part)
    return parts
