"""bench.py's multi-process path on CPU: two ranks over gloo (the GPU box runs the same code over NCCL).

The step has no exchange between replicas; what ranks share is the timing protocol: a barrier on both sides of
the timed region and the maximum of the ranks' times.  The reference arm runs on rank 0 only.
"""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank), "CUDA_VISIBLE_DEVICES": ""})
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, pg = bench.dist_setup()
    try:
        bench.barrier(pg)
        m = bench.reduce_max(pg, 10.0 * (rank + 1) + 0.5)
        bench.barrier(pg)
        q.put((r, w, m))
    finally:
        pg.destroy_process_group()


def test_max_over_ranks_and_barrier_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2, 20.5), (1, 2, 20.5)]


def test_reference_arm_under_torchrun_prints_one_line_from_rank_zero():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "3", "--ref-sample-cells", "1"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
