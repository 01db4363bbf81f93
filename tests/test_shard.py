"""Halo partitions (edge_b200.shard): index tables on one process, and multi-rank gloo runs of the
oracle's local / neighbour work regions with the per-step exchange, against the one-domain run.

The device form exchanges face projections of the send faces between GPUs; this CPU test
exchanges the whole time-integrated DOFs of the same send elements (what the oracle's neighbour
step reads), so the partition, the local numbering, the ghost mapping and the step order are
checked bit for bit without a GPU.
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
        expect = np.where(m.el_fa_type[q.lo:q.hi] == host.FACE_INNER, m.el_fa_el[q.lo:q.hi], -1)
        assert np.array_equal(glob, expect)
        for peer, lst in q.send.items():
            rec = parts[peer].recv[q.rank]
            assert len(rec) == len(lst)
            # the receiver's ghost is the sender's element, at the same face
            assert np.array_equal(parts[peer].global_ids()[rec[:, 0]], lst[:, 0] + q.lo)
            assert np.array_equal(rec[:, 1], lst[:, 1])
            for e, f in lst:
                key = (int(e) + q.lo, int(f))
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
        d = dict(full)
        d.update(nEl=part.n_local, starE=np.ascontiguousarray(full["starE"][ids]),
                 fsE=np.ascontiguousarray(full["fsE"][:, ids]),
                 elFaEl=np.ascontiguousarray(part.el_fa_el), fIdElFaEl=np.ascontiguousarray(part.fid),
                 vIdElFaEl=np.ascontiguousarray(part.vid), faType=np.ascontiguousarray(part.el_fa_type))
        st = dict(dofsE=np.ascontiguousarray(e0[ids]), dofsA=None,
                  tDofs=np.zeros((part.n_local, 9, p.B, 1)))
        t = 0.0
        for _ in range(n_steps):
            oracle.lts_local(d, st, 0, part.n_owned, True, t, p.dt, None)
            # exchange: the send elements' time integrals into the peers' ghost rows
            reqs, bufs = [], []
            for peer in sorted(set(part.send) | set(part.recv)):
                if peer in part.send:
                    el = np.unique(part.send[peer][:, 0])
                    reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(st["tDofs"][el])), peer))
                if peer in part.recv:
                    el = np.unique(part.recv[peer][:, 0])
                    b = torch.zeros((len(el), 9, p.B, 1), dtype=torch.float64)
                    reqs.append(dist.irecv(b, peer))
                    bufs.append((el, b))
            for r in reqs:
                r.wait()
            for el, b in bufs:
                st["tDofs"][el] = b.numpy()
            oracle.lts_neigh(d, st, 0, part.n_owned, True, None)
            t += p.dt
        np.save(os.path.join(out_dir, f"part{rank}.npy"), st["dofsE"][:part.n_owned])
    finally:
        dist.destroy_process_group()


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
    assert np.array_equal(got, ref.state["dofsE"])
