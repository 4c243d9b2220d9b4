"""The multi-process path on CPU: scene partitioning for sharded batches, the
measurement reductions over two gloo ranks, and a rank that leaves early
(the survivor must get an error, not hang)."""
import json
import multiprocessing as mp
import os
import socket
import time

import numpy as np
import pytest

from warpsph_b200 import ranks


def _sizes(count=64, seed=3):
    rng = np.random.default_rng(seed)
    return [int(np.exp(rng.uniform(np.log(5e3), np.log(2e5)))) for _ in range(count)]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_every_scene_once_and_balances(world):
    sizes = _sizes()
    parts = ranks.partition_scenes(sizes, world)
    assert len(parts) == world
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(sizes)))
    for p in parts:
        assert p == sorted(p)
    loads = [sum(sizes[k] for k in p) for p in parts]
    # LPT bound: no rank exceeds the mean by more than the largest scene
    assert max(loads) <= sum(sizes) / world + max(sizes)
    assert ranks.partition_scenes(sizes, world) == parts  # deterministic


def test_partition_edge_cases():
    assert ranks.partition_scenes([], 2) == [[], []]
    assert ranks.partition_scenes([5], 3) == [[0], [], []]
    assert ranks.partition_scenes([1, 1, 1, 1], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        ranks.partition_scenes([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, leave_early):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    res = {"rank": rank}
    try:
        dist = ranks.init("gloo", timeout_s=10.0)
        sizes = _sizes()
        mine = ranks.partition_scenes(sizes, world)[rank]
        load = sum(sizes[k] for k in mine)
        fake_ms = 1e-3 * load  # a rank's time grows with its particles
        res["load"] = load
        res["max_ms"] = ranks.max_over_ranks(fake_ms, dist)
        res["total"] = ranks.sum_over_ranks(load, dist)
        if leave_early and rank == 1:
            os._exit(0)  # leaves between steps, no collective in flight
        t0 = time.time()
        try:
            ranks.max_over_ranks(1.0, dist)
            res["second"] = "ok"
        except Exception as e:  # the peer is gone: an error, not a hang
            res["second"] = f"error: {type(e).__name__}"
        res["second_s"] = time.time() - t0
        dist.destroy_process_group()
    except Exception as e:
        res["fatal"] = repr(e)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def _run(tmp_path, leave_early):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path), leave_early)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=90)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
    out = {}
    for r in range(2):
        f = tmp_path / f"rank{r}.json"
        if f.exists():
            out[r] = json.loads(f.read_text())
    return out


def test_two_gloo_ranks_reduce_the_measurement(tmp_path):
    out = _run(tmp_path, leave_early=False)
    assert set(out) == {0, 1}
    sizes = _sizes()
    loads = [out[r]["load"] for r in range(2)]
    assert sum(loads) == sum(sizes)
    for r in range(2):
        assert "fatal" not in out[r], out[r]
        assert out[r]["max_ms"] == pytest.approx(1e-3 * max(loads))
        assert out[r]["total"] == pytest.approx(sum(sizes))
        assert out[r]["second"] == "ok"


def test_rank_leaving_early_is_an_error_for_the_other(tmp_path):
    out = _run(tmp_path, leave_early=True)
    assert 0 in out and "fatal" not in out[0], out
    assert out[0]["second"].startswith("error"), out[0]
    assert out[0]["second_s"] < 60
