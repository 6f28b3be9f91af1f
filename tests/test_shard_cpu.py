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


class _FakeDomainWall:
    """Stand-in for DomainWall in the analyzer test: measure() returns outputs
    that depend on each configuration's links and on its Z4 digits, so a rank
    that drew the digits of the wrong configuration index changes the result."""

    def __init__(self, Nt, Nx, Ls, M5, mf, beta=0.0, device=0):
        self.Nt, self.Nx = Nt, Nx

    def measure(self, thetas, z4=None, n_noise=0, max_momentum=0, **kw):
        n, V = thetas.shape[0], self.Nt * self.Nx
        zz = np.asarray(z4, np.float64).reshape(n, -1) if z4 is not None else np.zeros((n, 1))
        s = thetas.sum(axis=1) + 0.01 * zz.sum(axis=1)
        t = np.arange(self.Nt)
        cpp = 1.0 + np.exp(-0.3 * t)[None, :] * (1.5 + np.cos(s))[:, None]
        cj5 = 0.01 * cpp * (1.0 + 0.1 * np.sin(s))[:, None]
        loop = np.exp(1j * (s[:, None] + np.arange(V)[None, :] * 0.1 + zz[:, :1]))
        mom = np.stack([cpp * (k + 1) for k in range(max_momentum + 1)], axis=1)
        return {"cpp": cpp, "cj5": cj5, "loop": loop, "mom_cpp": mom}

    def close(self):
        pass


def _analyzer_worker(rank, world, port, workdir, q):
    import datetime
    import torch.distributed as dist
    from three_part_dwf_study_b200 import analyzer, dwf
    dwf.DomainWall = _FakeDomainWall
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        red = analyzer.analyze(workdir, world, rank, write=False)
        q.put((rank, {k: np.asarray(red[k]).tolist()
                      for k in ("cpp", "cj5", "m_res", "disconnected", "eta")}))
    finally:
        dist.destroy_process_group()


def test_sharded_analyzer_matches_single_process(tmp_path, monkeypatch):
    """analyzer.analyze on two gloo ranks (3 and 2 configurations of the
    reference's own 5-configuration ensemble) gives the single-process
    reductions: the blocks, the global Z4 seeds and the gather line up."""
    import shutil
    import torch.multiprocessing as mp
    from conftest import GOLDEN
    from three_part_dwf_study_b200 import analyzer, dwf
    g = GOLDEN / "dwf_hmc_8x8x4"
    shutil.copy2(g / "parameters.txt", tmp_path / "parameters.txt")
    (tmp_path / "output" / "domain_wall").mkdir(parents=True)
    cfg = np.load(g / "analysis_configs.npy")
    assert cfg.shape[0] >= 3
    shutil.copy2(g / "analysis_configs.npy", tmp_path / "output" / "domain_wall" / "analysis_configs.npy")
    monkeypatch.setattr(dwf, "DomainWall", _FakeDomainWall)
    ref = analyzer.analyze(str(tmp_path), 1, 0, write=False)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_analyzer_worker, args=(r, 2, port, str(tmp_path), q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        for k in ("cpp", "cj5", "m_res", "disconnected", "eta"):
            np.testing.assert_allclose(np.array(res[rank][k]), np.asarray(ref[k]), rtol=1e-14,
                                       atol=1e-300, err_msg=f"rank {rank} {k}")
