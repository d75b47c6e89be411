"""The replica harness of a multi-GPU run (sigmasph_b200.replicas), on CPU: world size 2
over gloo, each rank stepping its own copy of a small dam break with the CPU restatement
in place of the GPU path (the harness is the same code bench.py runs over NCCL).

Checks: the ranks' copies stay identical (replicas, not shards), every rank sees the same
maximum time, the whole-job throughput counts both ranks' particles over that maximum,
only rank 0 reports, and a rank that never joins makes the other's first collective fail
within the group timeout instead of hanging."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})


def _replica_rank(rank, world, port, out_dir):
    _env(rank, world, port)
    import time
    from sigmasph_b200 import abi
    from sigmasph_b200.config import SimConfig
    from sigmasph_b200.particle_system import ParticleSystem
    from sigmasph_b200.replicas import Replicas
    from sigmasph_b200.scenes import dambreak3d, dx_for_particles
    from sigmasph_b200.solver import build_params
    from oracle.oracle import Oracle, state_from_sets

    rep = Replicas("gloo", timeout_s=60)
    ps = ParticleSystem(SimConfig(dambreak3d(dx=dx_for_particles(600))), device="cpu")
    o = Oracle(build_params(ps), ps.particle_max_num, fp64=False)
    o.set_state(state_from_sets(ps.state_numpy()), 1e-4)
    o.stage(abi.STAGE_SORT)
    rep.barrier()
    t0 = time.perf_counter()
    o.step(3)
    own = time.perf_counter() - t0 + 0.05 * rank     # the ranks' times differ
    rep.barrier()
    t_max = rep.max_over_ranks(own)
    s = o.get_state()
    x = s["x"][np.argsort(s["pid"])]
    sums = rep.gather(float(np.sum(x, dtype=np.float64)))
    value = rep.throughput(ps.particle_max_num * 3, t_max)
    np.save(os.path.join(out_dir, f"r{rank}.npy"),
            np.array([own, t_max, value, ps.particle_max_num, float(rep.reporter)] + sums))
    rep.close()


def _lonely_rank(rank, world, port, out_dir):
    _env(rank, world, port)
    if rank == 1:
        return                       # never joins
    from sigmasph_b200.replicas import Replicas
    ok = "joined"
    try:
        rep = Replicas("gloo", timeout_s=3)
        rep.barrier()
    except Exception as e:           # the rendezvous or the barrier times out
        ok = type(e).__name__
    with open(os.path.join(out_dir, "r0.txt"), "w") as f:
        f.write(ok)


def test_two_replicas_on_gloo():
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_replica_rank, args=(2, _free_port(), d), nprocs=2, join=True,
                           start_method="spawn")
        r = [np.load(os.path.join(d, f"r{k}.npy")) for k in range(2)]
    own = [x[0] for x in r]
    assert r[0][1] == r[1][1] == pytest.approx(max(own))
    n = r[0][3]
    assert r[0][2] == r[1][2] == pytest.approx(2 * n * 3 / max(own))
    assert (r[0][4], r[1][4]) == (1.0, 0.0)
    sums0, sums1 = r[0][5:], r[1][5:]
    assert list(sums0) == list(sums1) and sums0[0] == sums0[1]


def test_missing_rank_fails_within_timeout():
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_lonely_rank, args=(2, _free_port(), d), nprocs=2, join=True,
                           start_method="spawn")
        with open(os.path.join(d, "r0.txt")) as f:
            assert f.read() != "joined"


def test_shard_balances_the_strips():
    """Largest first to the least-loaded rank: disjoint, complete, and the ranks' particle
    counts differ by at most one strip (the 256-strip ensemble's specs, no GPU)."""
    from sigmasph_b200.ensemble import shard, strip_specs
    specs = strip_specs(256)
    biggest = max(s.particles for s in specs)
    for world in (1, 2, 3, 4, 8):
        parts = [shard(specs, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(specs)))
        loads = [sum(specs[k].particles for k in p) for p in parts]
        assert max(loads) - min(loads) <= biggest, (world, loads)
        assert all(p == sorted(p) for p in parts)


def _shard_rank(rank, world, port, out_dir):
    _env(rank, world, port)
    from sigmasph_b200.ensemble import shard, strip_specs, state_row, STATE_COLUMNS
    from sigmasph_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    specs = strip_specs(256)
    own = shard(specs, world, rank)
    # stand-in states: what a strip reports, made from its index so the table is checkable
    rows = [state_row({"sim_time": 0.5 + k, "dt": 1e-5 * (k + 1), "load_s": -0.0 if k == 3 else k / 256,
                       "sts_stages": k % 7, "force": np.full((2, 3), -1.25 * k),
                       "disp": np.arange(6.0).reshape(2, 3) * k}) for k in own]
    table = rep.gather_rows(np.array(rows), own, len(specs))
    total = rep.sum_over_ranks(sum(specs[k].particles for k in own))
    np.save(os.path.join(out_dir, f"t{rank}.npy"), np.concatenate([[total], table.ravel()]))
    # rank 1 also claims rank 0's first strip: that one unit is owned twice
    other = shard(specs, world, 0)[0]
    idx = own if rank == 0 else own + [other]
    extra = rows if rank == 0 else rows + [rows[0]]
    try:
        rep.gather_rows(np.array(extra), idx, len(specs))
        twice = "accepted"
    except RuntimeError:
        twice = "refused"
    with open(os.path.join(out_dir, f"t{rank}.txt"), "w") as f:
        f.write(twice + " " + str(len(STATE_COLUMNS)))
    rep.close()


def test_sharded_ensemble_gather_on_gloo():
    """Two ranks each own half the strips; the float64 gather rebuilds the full table
    exactly on both ranks, the particle total counts every strip once, and a strip that
    two ranks claim is an error rather than a sum."""
    from sigmasph_b200.ensemble import strip_specs, state_row
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_shard_rank, args=(2, _free_port(), d), nprocs=2, join=True,
                           start_method="spawn")
        out = [np.load(os.path.join(d, f"t{r}.npy")) for r in range(2)]
        notes = [open(os.path.join(d, f"t{r}.txt")).read().split() for r in range(2)]
    specs = strip_specs(256)
    want = np.array([state_row({"sim_time": 0.5 + k, "dt": 1e-5 * (k + 1),
                                "load_s": -0.0 if k == 3 else k / 256, "sts_stages": k % 7,
                                "force": np.full((2, 3), -1.25 * k),
                                "disp": np.arange(6.0).reshape(2, 3) * k}) for k in range(256)])
    for o in out:
        assert o[0] == sum(s.particles for s in specs)
        assert np.array_equal(o[1:].reshape(want.shape), want)
    assert notes[0][0] == notes[1][0] == "refused" and int(notes[0][1]) == want.shape[1]
