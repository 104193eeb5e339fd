"""Ensemble sharding (magnumaf/ensemble.py) on CPU: the static cost-balanced
assignment, and the gather of member results over a world-size-2 gloo group,
including a member that fails on one rank (every rank then raises, none hangs)."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PY = os.path.join(os.path.dirname(HERE), "magnum.af_b200", "python")


def _ensemble():
    sys.path.insert(0, PY)
    from magnumaf import ensemble
    return ensemble


def test_assignment_covers_every_member_once_and_balances():
    E = _ensemble()
    rng = np.random.default_rng(5)
    sides = [64, 96, 128, 192, 256, 384, 512]
    members = [(int(rng.choice(sides)), int(rng.choice(sides)), 1, 10000) for _ in range(64)]
    costs = [E.member_cost(*m) for m in members]
    for world in (1, 2, 4, 8):
        parts = E.assign(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= 1.1 * (sum(costs) / world) or world == 1
        assert parts == E.assign(costs, world)  # a pure function: the same on every rank


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, fail_member, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, PY)
    from magnumaf import ensemble

    members = [(8 * (i % 3 + 1), 8, 1, 100 + i, i) for i in range(7)]
    costs = [ensemble.member_cost(*m[:4]) for m in members]

    def run(m):
        if m[4] == fail_member:
            raise ValueError("member %d diverged" % m[4])
        rng = np.random.default_rng(m[4])
        return {"member": m[4], "rank": rank, "value": float(rng.normal())}

    try:
        res = ensemble.run_sharded(members, costs, run)
        out.put((rank, "ok", res))
    except RuntimeError as e:
        out.put((rank, "err", str(e)))
    dist.destroy_process_group()


def _run_two_ranks(fail_member):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, fail_member, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(got)


def test_gather_over_two_gloo_ranks():
    got = _run_two_ranks(fail_member=-1)
    (r0, s0, res0), (r1, s1, res1) = got
    assert (r0, r1) == (0, 1) and s0 == s1 == "ok"
    assert res0 == res1
    assert [r["member"] for r in res0] == list(range(7))
    for r in res0:
        assert r["value"] == float(np.random.default_rng(r["member"]).normal())
    assert {r["rank"] for r in res0} == {0, 1}  # both ranks did work


def test_failed_member_raises_on_every_rank():
    got = _run_two_ranks(fail_member=4)
    assert [g[1] for g in got] == ["err", "err"]
    assert all("member 4" in g[2] and "diverged" in g[2] for g in got)
