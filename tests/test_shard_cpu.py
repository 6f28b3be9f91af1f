"""Multi-process (gloo, world size 2) tests of the analyzer sharding: the
partition covers every configuration once, and the gathered ensemble equals
the single-process result, real and complex outputs, even and uneven splits.
The per-configuration measurement is a deterministic stand-in (no GPU)."""
import os
import socket

import numpy as np
import pytest

from three_part_dwf_study_b200.shard import partition, gather_outputs, sharded_measure


def fake_measure(thetas):
    # deterministic per configuration: depends only on its own links
    s = thetas.sum(axis=1)
    cpp = np.stack([np.cos(s + k) for k in range(6)], axis=1)
    loop = np.exp(1j * np.outer(s, np.arange(5)))
    return {"cpp": cpp, "loop": loop}


def test_partition_covers_once():
    for nconf in (0, 1, 5, 8, 64, 65):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                a, b = partition(nconf, world, r)
                assert 0 <= a <= b <= nconf
                seen.extend(range(a, b))
            assert seen == list(range(nconf))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nconf, q):
    import torch.distributed as dist
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        thetas = np.random.default_rng(7).uniform(-np.pi, np.pi, (nconf, 32))
        out = sharded_measure(fake_measure, thetas, world, rank)
        q.put((rank, {k: v.tolist() if not np.iscomplexobj(v) else (v.real.tolist(), v.imag.tolist())
                      for k, v in out.items()}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nconf", [6, 5])
def test_sharded_measure_matches_single_process(nconf):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nconf, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    thetas = np.random.default_rng(7).uniform(-np.pi, np.pi, (nconf, 32))
    ref = fake_measure(thetas)
    for rank in (0, 1):
        got = res[rank]
        np.testing.assert_array_equal(np.array(got["cpp"]), ref["cpp"])
        re, im = got["loop"]
        np.testing.assert_array_equal(np.array(re) + 1j * np.array(im), ref["loop"])
