"""Halo partitions (edge_b200.shard): index tables on one process, and multi-rank gloo runs of the
oracle's local / neighbour work regions with the per-step exchange, against the one-domain run.

The ranks exchange what the device form exchanges: the face rows of the send faces, projected on
the face and pre-mixed with the reading element's flux solver (oracle.face_rows_premixed), sent
after the send elements' local step and before the inner elements' one, and lifted by the
reader with the face orientation and fluxT. So the partition, the local numbering (send elements
first), the ghost mapping, the exchange format and the overlapped step order are checked on the
CPU against the one-domain oracle.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from edge_b200 import host, shard


def _prob(order=3, n=4, runs=1):
    return host.build_problem(n, order, runs, jitter=0.15, seed=8, n_receivers=0, source=None)


@pytest.mark.parametrize("n_parts", [2, 3, 5])
def test_plan_covers_every_inner_face_once(n_parts):
    p = _prob()
    m = p.mesh
    parts = shard.plan(m, n_parts)
    assert sum(q.n_owned for q in parts) == m.n_el
    sent = {}
    for q in parts:
        gid = q.global_ids()
        # local connectivity maps back to the global one on owned rows
        loc = q.el_fa_el[:q.n_owned]
        glob = np.where(loc >= 0, gid[np.maximum(loc, 0)], -1)
        expect = np.where(m.el_fa_type[q.owned] == host.FACE_INNER, m.el_fa_el[q.owned], -1)
        assert np.array_equal(glob, expect)
        assert sorted(q.owned) == list(range(q.lo, q.hi))
        # send elements first: exactly the owned elements with a face neighbour in another part
        remote = (loc >= q.n_owned).any(axis=1)
        assert remote[:q.n_send].all() and not remote[q.n_send:].any()
        for peer, lst in q.send.items():
            rec = parts[peer].recv[q.rank]
            assert len(rec) == len(lst)
            assert (lst[:, 0] < q.n_send).all()
            # the receiver's ghost is the sender's element, at the same face
            assert np.array_equal(parts[peer].global_ids()[rec[:, 0]], q.owned[lst[:, 0]])
            assert np.array_equal(rec[:, 1], lst[:, 1])
            for e, f in lst:
                key = (int(q.owned[e]), int(f))
                assert key not in sent
                sent[key] = peer
    # every face between two parts is sent exactly once, to the part of the neighbour
    bounds = shard.ranges(m.n_el, n_parts)
    owner = np.searchsorted(bounds, np.arange(m.n_el), side="right") - 1
    for e in range(m.n_el):
        for f in range(4):
            ne = m.el_fa_el[e, f]
            if m.el_fa_type[e, f] == host.FACE_INNER and ne >= 0 and owner[ne] != owner[e]:
                assert sent.pop((e, f)) == owner[ne]
    assert not sent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, order, n_steps, out_dir):
    """One rank: the oracle's local step of the send elements, the pre-mixed face rows of the send
    faces to the peers (gloo), the local step of the inner elements, the neighbour step with the
    received rows for the ghost faces -- the device form's step order and exchange format."""
    import torch

    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = _prob(order=order)
        rng = np.random.default_rng(1)
        e0 = rng.normal(size=(p.n_el, 9, p.B, 1)) * 1e-3
        part = shard.plan(p.mesh, world)[rank]
        ids = part.global_ids()
        full = p.oracle_dict()
        O, _ = oracle.face_orientations(full["fluxL"], full["fluxN"])
        d = dict(full)
        d.update(nEl=part.n_local, starE=np.ascontiguousarray(full["starE"][ids]),
                 fsE=np.ascontiguousarray(full["fsE"][:, ids]),
                 elFaEl=np.ascontiguousarray(part.el_fa_el), fIdElFaEl=np.ascontiguousarray(part.fid),
                 vIdElFaEl=np.ascontiguousarray(part.vid), faType=np.ascontiguousarray(part.el_fa_type))
        # the neighbour step skips the ghost faces; their rows come from the peers
        ghost_face = (part.el_fa_el >= part.n_owned)
        dn = dict(d, faType=np.ascontiguousarray(np.where(ghost_face, 2, part.el_fa_type).astype(np.uint8)))
        ghost_faces = [(int(e), int(f)) for e, f in zip(*np.nonzero(ghost_face[:part.n_owned]))]
        st = dict(dofsE=np.ascontiguousarray(e0[ids]), dofsA=None,
                  tDofs=np.zeros((part.n_local, 9, p.B, 1)))
        t = 0.0
        for _ in range(n_steps):
            oracle.lts_local(d, st, 0, part.n_send, True, t, p.dt, None)
            reqs, got = [], {}
            for peer in sorted(set(part.send) | set(part.recv)):
                if peer in part.send:
                    rows = oracle.face_rows_premixed(d, st["tDofs"], part.send[peer])
                    reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(rows)), peer))
                if peer in part.recv:
                    b = torch.zeros((len(part.recv[peer]), 9, p.order * (p.order + 1) // 2, 1), dtype=torch.float64)
                    reqs.append(dist.irecv(b, peer))
                    got[peer] = b
            # the inner elements' local step while the rows travel
            oracle.lts_local(d, st, part.n_send, part.n_owned - part.n_send, True, t, p.dt, None)
            for r in reqs:
                r.wait()
            slot = {}
            for peer, b in got.items():
                for (g, f), row in zip(part.recv[peer], b.numpy()):
                    slot[(int(g), int(f))] = row
            oracle.lts_neigh(dn, st, 0, part.n_owned, True, None)
            rows = [slot[(int(part.el_fa_el[e, f]), int(part.fid[e, f]))] for e, f in ghost_faces]
            oracle.neigh_premixed_faces(d, st["dofsE"], ghost_faces, rows, O)
            t += p.dt
        out = np.empty_like(st["dofsE"][:part.n_owned])
        out[part.owned - part.lo] = st["dofsE"][:part.n_owned]
        np.save(os.path.join(out_dir, f"part{rank}.npy"), out)
    finally:
        dist.destroy_process_group()


def test_face_orientation_factorisation():
    import oracle
    for order in (2, 3, 4, 5):
        d = _prob(order=order, n=2).oracle_dict()
        _, res = oracle.face_orientations(d["fluxL"], d["fluxN"])
        assert res < 1e-12, (order, res)


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_with_exchange_match_one_domain(tmp_path, world):
    from helpers import OracleRun
    order, n_steps = 3, 4
    mp.spawn(_rank_main, args=(world, _free_port(), order, n_steps, str(tmp_path)), nprocs=world, join=True)
    p = _prob(order=order)
    rng = np.random.default_rng(1)
    e0 = rng.normal(size=(p.n_el, 9, p.B, 1)) * 1e-3
    ref = OracleRun(p, e0)
    ref.step(n_steps)
    got = np.concatenate([np.load(os.path.join(tmp_path, f"part{r}.npy")) for r in range(world)])
    # (the ghost faces' fluxes are added after the other faces, with fluxL . O for fluxN: the same
    # sums in another order)
    rel = np.linalg.norm(got - ref.state["dofsE"]) / np.linalg.norm(ref.state["dofsE"])
    assert rel < 1e-12, rel
