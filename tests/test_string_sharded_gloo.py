"""Sharded string method (magnumaf/string_sharded.py) on CPU ranks (gloo):
images integrated by the oracle, arc lengths and re-interpolation through the
point-to-point exchanges.  One rank and two ranks give bit-identical strings,
equal (to summation order) to the serial oracle string method run with one
integrator per image — the sharded method's policy; the reference instead passes
one controller state from image to image, which changes how far each image
overshoots t0 + dt and so cannot be sharded."""
import copy
import datetime
import os
import socket
import sys

import numpy as np

import maf_oracle as O
import maf_string_oracle as SO

HERE = os.path.dirname(os.path.abspath(__file__))
PY = os.path.join(os.path.dirname(HERE), "magnum.af_b200", "python")

SHAPE = (8, 8, 1)
MS = 1.1e6
N_INTERP = 5
DT = 5e-14
STEPS = 2


def _setup():
    mesh = O.Mesh(*SHAPE, 1e-9, 1e-9, 1e-9)
    terms = [O.ExchangeField(1.6e-11), O.DmiField(4e-3), O.UniaxialAnisotropyField(1e6),
             O.ExternalField(np.array([0.0, 0.0, 0.01 / O.mu0]))]
    a = np.zeros(SHAPE + (3,))
    a[..., 2] = 1.0
    a[2:6, 2:6, 0, 2] = -1.0
    a[..., 0] += 0.1
    b = np.zeros(SHAPE + (3,))
    b[..., 0] = 0.1
    b[..., 2] = 1.0
    return mesh, terms, O.normalize(a), O.normalize(b)


def _soa(m):
    return np.transpose(m, (3, 2, 1, 0)).reshape(-1).copy()


def _aos(v):
    return np.transpose(v.reshape(3, SHAPE[2], SHAPE[1], SHAPE[0]), (3, 2, 1, 0))


class OracleImages:
    def __init__(self, mesh, terms, indices):
        self.size = 3 * int(np.prod(SHAPE))
        proto = O.LLGIntegrator(1.0, terms)
        self.states = {i: O.State(mesh, MS, np.ones(SHAPE + (3,))) for i in indices}
        self.llgs = {i: copy.deepcopy(proto) for i in indices}

    def step(self, i, dt):
        s = self.states[i]
        t0 = s.t
        while s.t < t0 + dt:
            self.llgs[i].step(s)

    def get(self, i):
        return _soa(self.states[i].m)

    def set(self, i, m):
        self.states[i].m = _aos(m)

    def energy(self, i):
        return self.llgs[i].E(self.states[i])


def _run(rank, world):
    sys.path.insert(0, PY)
    from magnumaf import string_sharded as SS

    mesh, terms, a, b = _setup()
    mine = SS.blocks(N_INTERP, world)[rank]
    sm = SS.ShardedStringMethod(OracleImages(mesh, terms, mine), N_INTERP, DT, [_soa(a), _soa(b)])
    for _ in range(STEPS):
        sm.step()
    E = sm.calc_E()
    return sm.x, E, {i: sm.img.get(i) for i in mine}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    q.put((rank,) + _run(rank, world))
    dist.destroy_process_group()


def _two_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted([q.get(timeout=300) for _ in ps], key=lambda g: g[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return got


def test_blocks_partition_the_images():
    sys.path.insert(0, PY)
    from magnumaf import string_sharded as SS

    for n in (1, 2, 5, 32):
        for w in (1, 2, 3, 8):
            bl = SS.blocks(n, w)
            assert [i for b in bl for i in b] == list(range(n))
            assert max(len(b) for b in bl) - min(len(b) for b in bl) <= 1


def test_two_ranks_equal_one_rank_and_follow_the_serial_reference():
    x1, E1, imgs1 = _run(0, 1)
    got = _two_ranks()
    for _, x, E, _imgs in got:
        assert x == x1 and E == E1  # bit-identical on every rank
    imgs2 = {}
    for g in got:
        imgs2.update(g[3])
    for i in range(N_INTERP):
        assert np.array_equal(imgs1[i], imgs2[i])
    # the serial oracle string method with the same per-image integrator policy
    mesh, terms, a, b = _setup()
    ref = SO.StringMethod(O.State(mesh, MS, a), [a, b], N_INTERP, DT, O.LLGIntegrator(1.0, terms),
                          per_image_integrators=True)
    for _ in range(STEPS):
        ref.step()
    np.testing.assert_allclose(x1, ref.x, rtol=1e-12)
    np.testing.assert_allclose(E1, ref.calc_E(), rtol=1e-12)
    for i in range(N_INTERP):
        np.testing.assert_allclose(_aos(imgs1[i]), ref.images[i].m, atol=1e-12)
