"""The multi-rank plumbing of bench.py on CPU (two gloo ranks): the timed
region's job time is the slowest rank's, the whole-job throughput counts every
rank's units, and under torchrun the reference arm runs on rank 0 only.

Ranks are independent replicas (the path has no exchange step), so these are
the only cross-rank steps the benchmark takes."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = [bench.max_over_ranks(t, dist, device="cpu") for t in times[rank]]
        q.put((rank, got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    world = 2
    # three timed regions (batched, per-op, end-to-end) as bench.py runs them,
    # a different rank the slowest in each
    times = {0: [5.0, 1.0, 7.5], 1: [3.0, 2.5, 7.25]}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [max(times[0][i], times[1][i]) for i in range(3)]
    assert res[0] == want and res[1] == want


def test_job_throughput_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(4.0, None) == 4.0
    # 32 pairs x 20 steps per rank on 2 ranks in 160 ms
    assert bench.job_throughput(32 * 20, 2, 160.0) == pytest.approx(8000.0)
    assert bench.job_throughput(32 * 20, 1, 160.0) == pytest.approx(4000.0)


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_ntt_traffic_from_ncu_csv(tmp_path):
    """roofline.traffic from a capture: the last cols + rows pair's DRAM
    read + write bytes, units converted."""
    import bench

    hdr = '"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size","Grid Size",' \
          '"Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"\n'
    rows = []
    for i, (k, rd, wr) in enumerate([("k_ntt_fwd_cols<8, 8, 3, 0, 1, 1>", "1.0", "2.0"),
                                     ("k_ntt_fwd_rows<8, 8, 3, 0, 1, 1, 1>", "3.0", "4.0"),
                                     ("k_ntt_fwd_cols<8, 8, 3, 0, 1, 1>", "503.5", "443.6"),
                                     ("k_ntt_fwd_rows<8, 8, 3, 0, 1, 1, 1>", "534,800", "444.6")]):
        unit_r = "Kbyte" if "," in rd else "Mbyte"
        for m, u, v in (("dram__bytes_read.sum", unit_r, rd), ("dram__bytes_write.sum", "Mbyte", wr)):
            rows.append('"%d","1","python3","h","void %s(DevCtx, LimbMap)","1","7","(256, 1, 1)","(16, 32, 30)",'
                        '"0","10.0","Command line profiler metrics","%s","%s","%s"\n' % (i, k, m, u, v))
    p = tmp_path / "t.csv"
    p.write_text("==PROF== Connected\n" + hdr + "".join(rows))
    assert abs(bench.ntt_traffic_from_csv(str(p)) - 1926.5e6) < 1.0
