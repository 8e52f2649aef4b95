"""Multi-rank plumbing on CPU: two gloo ranks (world size 2) on 127.0.0.1.

* the walker shards cover every walker once, uneven counts included;
* max over ranks of a per-rank time;
* the sharded adjoint (one all-reduce of the coefficient and nuclear
  gradients) equals the single-process gradients; the per-rank adjoint is the
  CPU oracle's restatement of the reference's orbital forces.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from qmckl_b200 import replicas


def test_shards_cover_every_walker():
    for n in (0, 1, 5, 64, 513):
        for world in (1, 2, 3, 8):
            got = [replicas.shard(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    from oracle import pyoracle as O
    from qmckl_b200 import gen
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = replicas.max_over_ranks(1.5 + rank)
        d = gen.config(0, walk_num=3)
        W, E = d["elec_coord"].shape[:2]
        basis = O.Basis(d)
        w = np.random.default_rng(5).standard_normal((W * E, 5, d["mo_num"]))

        def local(w0, w1):
            pts = d["elec_coord"][w0:w1].reshape(-1, 3)
            if pts.shape[0] == 0:
                return (torch.zeros(d["mo_num"], d["ao_num"], dtype=torch.float64),
                        torch.zeros(d["nucl_num"], 3, dtype=torch.float64), torch.zeros(3, 0, dtype=torch.float64))
            gc, gn, gr = O.mo_vgl_adjoint(basis, pts, d["nucl_coord"], d["mo_coef"], w[w0 * E:w1 * E])
            return torch.from_numpy(gc), torch.from_numpy(gn), torch.from_numpy(np.ascontiguousarray(gr.T))

        gc, gn, gr, (w0, w1) = replicas.sharded_adjoint(W, E, rank, world, local)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), t=t, gc=gc.numpy(), gn=gn.numpy(), gr=gr.numpy(),
                 w=np.array([w0, w1]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    from oracle import pyoracle as O
    from qmckl_b200 import gen
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    res = [dict(np.load(tmp_path / f"r{r}.npz")) for r in range(world)]
    assert all(float(r["t"]) == 2.5 for r in res)
    d = gen.config(0, walk_num=3)
    E = d["elec_coord"].shape[1]
    w = np.random.default_rng(5).standard_normal((3 * E, 5, d["mo_num"]))
    gc, gn, gr = O.mo_vgl_adjoint(O.Basis(d), gen.points(d), d["nucl_coord"], d["mo_coef"], w)
    for r in res:
        assert np.abs(r["gc"] - gc).max() <= 1e-12 * np.abs(gc).max()
        assert np.abs(r["gn"] - gn).max() <= 1e-12 * np.abs(gn).max()
    got_r = np.concatenate([r["gr"].T for r in sorted(res, key=lambda x: int(x["w"][0]))])
    assert got_r.shape == gr.shape
    assert np.abs(got_r - gr).max() <= 1e-12 * np.abs(gr).max()
    assert [tuple(r["w"]) for r in res] == [(0, 2), (2, 3)]
