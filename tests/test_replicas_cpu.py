"""bench.py under torchrun runs one independent replica per rank (the step does not
shard); the only collective is the max over ranks of the timed region. Two gloo ranks
on the CPU check that reduction and that every rank sees the same value."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
        assert dict(out) == {0: 15.0, 1: 15.0}


def test_reference_arm_uses_every_core():
    """The CPU reference arm runs one spawned process per core, each its own sample,
    and reports their aggregate over the common timed interval."""
    from oracle import numpy_ref
    r = numpy_ref.time_rain_on_terrain_parallel(n=48, steps=2, warm=1, procs=2)
    assert r["cores"] == 2 and r["value"] > 0 and r["seconds"] > 0
    one = numpy_ref.time_rain_on_terrain(n=48, steps=2, warm=1)
    assert one["cores"] == 1 and one["value"] > 0


def test_tuner_cache_writes_from_many_processes(tmp_path, monkeypatch):
    """Ranks that tune at the same time write the cache without failing."""
    import multiprocessing as mp
    monkeypatch.setenv("GSW_TUNE_CACHE", str(tmp_path / "autotune.json"))
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_store_many, args=(str(tmp_path / "autotune.json"), r)) for r in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    import json
    json.loads((tmp_path / "autotune.json").read_text())


def _store_many(path, rank):
    import os
    os.environ["GSW_TUNE_CACHE"] = path
    from geoswe_b200 import autotune
    autotune._key = lambda kind, cells: f"{kind}|{cells}"      # no device query on the CPU
    for k in range(50):
        autotune._store("dense", rank * 1000 + k, {"tile_rows": 32, "warps": 4, "min_blocks": 4, "ms": 1.0})
