"""The multi-GPU plumbing of bench.py on CPU: ranks as gloo processes (world size 2), each with its
own timing; every rank must see the slowest rank's time, and the whole-job figure divides it over
all ranks' units (replicas: weak scaling, no data-path collective).  Also the bench helper that
reads the roofline's DRAM traffic from the committed ncu summaries."""
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


def _rank_main(rank, world, port, times, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(times[rank], dist, "cpu")
        out[rank] = (slowest, bench.whole_job_ms_per_unit(slowest, 10, world))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("times", [(12.5, 40.0), (33.0, 7.25)])
def test_max_over_ranks_and_whole_job(times):
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, _free_port(), list(times), out), nprocs=world, join=True)
    slowest = max(times)
    for r in range(world):
        assert out[r][0] == slowest
        assert out[r][1] == pytest.approx(slowest / (10 * world))


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_ms_per_unit(40.0, 10, 1) == 4.0


def test_roofline_traffic_comes_from_committed_profiles():
    """The bench's roofline lines read `traffic` (DRAM bytes per launch) from the committed ncu
    summaries of the kernels they time; both summaries carry the figure."""
    import bench
    fold = bench.profiled_traffic("bivariate_fold_eval_kernel_log20.md")
    ntt = bench.profiled_traffic("ntt_pass_kernel_log20_b4.md")
    assert isinstance(fold, int) and isinstance(ntt, int)
    # the fold reads its two 2^20-element operands (32 MiB) once: traffic near the read bytes
    assert 32 << 20 <= fold <= 48 << 20
    assert ntt > 0
