"""Host-side logic without a GPU: the bench's multi-rank timing (max over
ranks, whole-job throughput) on two gloo ranks, and the batch tuner's
record/replay of per-resolution settings."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    assert bench.dist_env() == (rank, world, rank)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(times[rank], "cpu", world)
        out.put((rank, ms, bench.aggregate_value(3, world, ms)))
    finally:
        dist.destroy_process_group()


def test_bench_timing_is_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [120.0, 250.0]  # ms per rank: the job takes the slower one
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [250.0, 250.0]
    # 3 steps per rank, 2 ranks, 0.25 s -> 24 units/s
    assert res[0][2] == pytest.approx(24.0)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(42.0, "cpu", 1) == 42.0
    assert bench.aggregate_value(3, 1, 1500.0) == pytest.approx(2.0)


class _Desc:
    def __init__(self, nr, nt, pressure):
        self.nr_cells, self.ntheta_cells, self.pressure_space = nr, nt, pressure


class _Ctx:
    def __init__(self, nr, nt, pressure=1):
        self.desc = _Desc(nr, nt, pressure)


def test_tuning_record_replays(tmp_path):
    sys.path.insert(0, ROOT)
    from dimspers_b200 import batch
    table = {"64x512/discontinuous": dict(apply_warps=8, apply_warps_t=2, cheb_degree=2, coarse_max=1024,
                                          ms_per_outer=1.0, trials=4, default=None)}
    path = tmp_path / "t.json"
    path.write_text(json.dumps(table))
    loaded = batch.load_tuning(str(path))
    o = batch.tuned_opts(_Ctx(64, 512), loaded)
    assert (o["apply_warps"], o["apply_warps_t"], o["cheb_degree"], o["coarse_max"]) == (8, 2, 2, 1024)
    assert o["precision"] == batch.FAST["precision"]
    # a resolution without a record keeps the base options
    o2 = batch.tuned_opts(_Ctx(32, 256), loaded)
    assert o2 == batch.FAST
    assert batch.tuning_key(_Ctx(16, 128, 0)) == "16x128/continuous"


def test_solve_bytes_model():
    """The per-solve byte model is linear in the iteration counts, and its
    V-cycle stops at the dense coarsest level (4x32 under coarse_max 1536)."""
    sys.path.insert(0, ROOT)
    import bench
    m = bench.solve_bytes_model
    base = m(128, 1024, 0, 0)
    assert base == 0.0
    one_in, one_out = m(128, 1024, 0, 1), m(128, 1024, 1, 0)
    assert m(128, 1024, 904, 2949) == pytest.approx(904 * one_out + 2949 * one_in)
    # the fine-level FP32 applies alone: 6 per V-cycle of 90.2 MB
    assert one_in > 6 * (312 * 262144 + 16 * 526336)
    # the dense coarsest (1,152 DOFs) is part of every V-cycle, and a mesh that
    # is its own coarsest level is the dense apply plus the Krylov work
    assert m(4, 32, 0, 1) == pytest.approx(1152 ** 2 * 8 + 624 * 256 + 48 * 576 + 108 * 1152)
