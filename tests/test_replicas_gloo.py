"""Multi-process path of bench.py (replicas) with world size 2 on the gloo backend (no GPU):
barrier, max-over-ranks device time, whole-job rate, independent per-rank scenes."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from turbospharticles_b200 import replicas, scene
    from turbospharticles_b200.params import dam_params
    ws, r, _ = replicas.dist_env()
    dist = replicas.init("gloo", ws, timeout_s=60)
    replicas.barrier(dist)
    ms = 10.0 + 5.0 * r  # the slower rank defines the job time
    mx = replicas.max_over_ranks(dist, ms)
    p = dam_params(0.02, 1e-3)
    p.jitterFracF = 0.01
    p.jitterSeedF = replicas.replica_seed(42, r)
    st, _, _ = scene.dam_scene(4, 0.02, (0.2, 0.2, 0.2), p, seed=replicas.replica_seed(42, r))
    out[r] = (mx, replicas.aggregate_rate(1000, ws, mx), float(st.xPosF.sum()))
    dist.destroy_process_group()


def test_two_rank_replicas():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert out[0][0] == out[1][0] == 15.0
    assert out[0][1] == pytest.approx(2 * 1000 / 0.015)
    assert out[0][2] != out[1][2], "replica scenes must be independently seeded"
