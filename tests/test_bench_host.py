"""bench.py's multi-rank arithmetic: the job time is the slowest rank's and
the value is the units all ranks processed over it (two gloo ranks on CPU)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rank(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 10.0 * (rank + 1)
    t = bench.max_over_ranks(dist, ms)
    q.put((rank, t, bench.job_rate(1000, world, t)))
    dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
    for rank, t, v in res:
        assert t == 20.0 and v == pytest.approx(1000 * 2 / 0.020)


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(None, 3.5) == 3.5


def test_launcher_starts_the_ranks_itself():
    # bench.py --gpus 2 without a torchrun environment starts its two ranks
    # (here a gloo self-test instead of the GPU work) and rank 0 prints the line
    import json
    import subprocess
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "MASTER_PORT")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dist-check"],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["ms_max"] == 20.0


def test_gpus_must_match_the_launch():
    import subprocess
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="1", MASTER_ADDR="127.0.0.1", MASTER_PORT="29999")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dist-check"],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode != 0 and "WORLD_SIZE 1" in out.stderr


def test_slab_initial_state_is_the_global_field_on_the_slab_planes():
    import numpy as np
    import bench
    from isothermal_mhd_b200 import forcing, slabs
    n, ws = 16, 2
    dec = slabs.Decomposition(n, ws, slabs.halo_width("plm", 2))
    f = forcing.OUForcing(n, seed=7)
    v = f.field(rms=2.0)
    f.advance(0.05)
    d = f.field(rms=1.0)
    for r in range(ws):
        q, b, p, delv = bench.slab_initial_state(dec, r, 2.0, 2, 7, 0.5)
        np.testing.assert_allclose(q[1:4], dec.scatter(v, r), rtol=0, atol=1e-12)
        np.testing.assert_allclose(delv, dec.scatter(d, r), rtol=0, atol=1e-12)
        assert q.shape == (7, dec.local_nz(r), n, n) and np.all(b[0] == 0.5)


def test_step_roofline_binds_on_the_slower_bound():
    import bench
    rl = bench.step_roofline(4.75e9, "roe", "plm", 2, 4, 6553.6, 1965.0)
    assert rl["bound"] == "fp32" and rl["bytes_per_cell"] == 72
    peak = 148 * 128 * 2 * 1965e6
    assert abs(rl["fp32_frac"] - 4.75e9 * rl["ops_per_cell"] / peak) < 1e-12
    assert abs(rl["frac"] - rl["fp32_frac"]) < 1e-12


def test_op_count_table_matches_the_oracle_tally():
    # bench.py's per-cell op table is the committed output of the op-counting
    # oracle, and one configuration recounted now agrees with it
    import json
    import bench
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import count_ops
    with open(os.path.join(ROOT, "oracle", "op_counts.json")) as fh:
        table = json.load(fh)["configs"]
    for (r, rc, npass), ops in bench.ALG_OPS_PER_CELL.items():
        assert abs(table[f"{r}-{rc}-np{npass}"]["ops"] - ops) < 0.1
    now = count_ops.per_cell("roe", "plm", 2)
    assert abs(now["ops"] - bench.ALG_OPS_PER_CELL[("roe", "plm", 2)]) < 0.1
