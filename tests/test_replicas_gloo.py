"""Multi-rank bookkeeping of the replica runs (cheddar-fhe_b200/replicas.py,
used by bench.py under torchrun) with two gloo ranks on the CPU: the slowest
rank's time reaches every rank, the whole-job throughput counts every
rank's units, ranks get distinct input seeds, a missing peer ends the wait
with an error instead of a hang, and the reference arm of bench.py runs on
rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))


def _worker(rank, world, port, q):
    _env(rank, world, port)
    import replicas as rp
    dist = rp.init_group(world, "gloo", timeout_s=60)
    r, w, _ = rp.env_rank()
    rp.barrier(dist)
    ms = rp.max_over_ranks(dist, 10.0 * (r + 1))
    q.put((r, w, ms, rp.job_throughput(w, 8, 5, ms), rp.rank_seed(1234, r)))
    rp.finish(dist)


def _lonely_worker(rank, world, port, q):
    # rank 1 of 2 whose peer never joins: the group's short timeout turns the
    # wait into an error
    _env(rank, world, port)
    import replicas as rp
    try:
        dist = rp.init_group(world, "gloo", timeout_s=3)
        rp.barrier(dist)
        q.put("joined")
    except Exception as e:  # noqa: BLE001
        q.put(f"error: {type(e).__name__}")


def _run(target, ranks, world, timeout):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=target, args=(r, world, port, q)) for r in ranks]
    for p in ps:
        p.start()
    out = [q.get(timeout=timeout) for _ in ps]
    for p in ps:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return out, [p.exitcode for p in ps]


def test_two_gloo_ranks():
    out, codes = _run(_worker, [0, 1], 2, 120)
    assert codes == [0, 0]
    out.sort()
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 20.0 for o in out)             # max over ranks
    assert all(abs(o[3] - 2 * 8 * 5 / 0.020) < 1e-6 for o in out)
    assert out[0][4] != out[1][4]                     # distinct input seeds


def test_missing_peer_times_out():
    out, codes = _run(_lonely_worker, [1], 2, 120)
    assert out[0].startswith("error"), out


def test_single_rank_needs_no_group():
    import replicas as rp
    assert rp.init_group(1) is None
    assert rp.max_over_ranks(None, 3.5) == 3.5
    assert rp.job_throughput(1, 8, 10, 100.0) == 800.0


def test_reference_arm_rank0_only():
    # under torchrun every rank starts the reference arm; ranks above 0 exit
    # at once without output
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "", (r.stdout, r.stderr)


def test_reference_arm_line():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
