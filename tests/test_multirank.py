"""Multi-rank host logic (aurora_b200.shard) with gloo ranks on the CPU: sample-range
splitting, the film combine and the max-over-ranks timing. The per-rank renders are
the oracle's CPU renders of the rank's sample range (the device renderer is the same
function of (pixel, sample index), so the combine logic is what is under test)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sample_range_partitions():
    from aurora_b200.shard import sample_range
    for world in (1, 2, 3, 4, 8):
        for spp in (0, 1, 7, 16, 64, 65):
            ranges = [sample_range(r, world, spp) for r in range(world)]
            covered = [s for first, n in ranges for s in range(first, first + n)]
            assert covered == list(range(spp))
            assert max(n for _, n in ranges) - min(n for _, n in ranges) <= 1
        assert [sample_range(r, world, 16, "weak") for r in range(world)] == [(16 * r, 16) for r in range(world)]
    with pytest.raises(ValueError):
        sample_range(2, 2, 16)
    with pytest.raises(ValueError):
        sample_range(0, 1, 16, "diagonal")


def _worker(rank, world, port, spp, result_path):
    import torch
    import torch.distributed as dist
    import datetime
    from aurora_b200 import scenes
    from aurora_b200.shard import combine_films, max_over_ranks, sample_range
    from oracle import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        data = scenes.box_scene(32, 32, spp=spp)
        osc = oracle.OracleScene(data, np.zeros((21, 64, 32), np.float32))
        first, count = sample_range(rank, world, spp)
        mean, _, _ = osc.render(count, 5, 5, 1, sample_offset=first, threads=1, want_m2=False)
        film = torch.tensor(mean, dtype=torch.float32)
        combine_films(film, count)
        t = max_over_ranks(10.0 + rank)
        if rank == 0:
            np.save(result_path, film.numpy())
            assert t == 10.0 + (world - 1)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,spp", [(2, 8), (3, 7)])
def test_sharded_render_equals_single_render(tmp_path, oracle_lib, world, spp):
    import torch.multiprocessing as mp
    from aurora_b200 import scenes
    path = str(tmp_path / "film.npy")
    mp.start_processes(_worker, args=(world, _free_port(), spp, path), nprocs=world, join=True,
                       start_method="spawn")
    combined = np.load(path)
    data = scenes.box_scene(32, 32, spp=spp)
    osc = oracle_lib.OracleScene(data, np.zeros((21, 64, 32), np.float32))
    whole, _, _ = osc.render(spp, 5, 5, 1, threads=1, want_m2=False)
    np.testing.assert_allclose(combined, whole, rtol=1e-6, atol=1e-6)


def _adjoint_worker(rank, world, port, spp, result_path):
    import datetime
    import torch.distributed as dist
    from aurora_b200 import scenes
    from aurora_b200.shard import combine_gradients, sample_range
    from oracle import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        data = scenes.texture_scene(24, 24)
        osc = oracle.OracleScene(data, np.zeros((21, 64, 32), np.float32))
        w = np.random.default_rng(3).normal(size=(24, 24, 4)).astype(np.float32)
        first, count = sample_range(rank, world, spp)
        gm, gt = osc.adjoint(count, 6, 6, 2, w, sample_offset=first, threads=1)
        combine_gradients((gm, gt), count, spp)
        if rank == 0:
            np.save(result_path, np.concatenate([gm.ravel(), gt.ravel()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,spp", [(2, 6), (3, 7)])
def test_sharded_adjoint_equals_single_adjoint(tmp_path, oracle_lib, world, spp):
    """Each rank's adjoint over its sample range, combined by combine_gradients (one sum
    all-reduce of the count-weighted gradients), equals the adjoint over all samples."""
    import torch.multiprocessing as mp
    from aurora_b200 import scenes
    path = str(tmp_path / "grad.npy")
    mp.start_processes(_adjoint_worker, args=(world, _free_port(), spp, path), nprocs=world, join=True,
                       start_method="spawn")
    combined = np.load(path)
    data = scenes.texture_scene(24, 24)
    osc = oracle_lib.OracleScene(data, np.zeros((21, 64, 32), np.float32))
    w = np.random.default_rng(3).normal(size=(24, 24, 4)).astype(np.float32)
    gm, gt = osc.adjoint(spp, 6, 6, 2, w, threads=1)
    whole = np.concatenate([gm.ravel(), gt.ravel()])
    assert np.any(whole != 0)
    np.testing.assert_allclose(combined, whole, rtol=1e-9, atol=1e-12)
