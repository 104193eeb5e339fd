"""String method with its images sharded over the ranks of a torch.distributed
process group (one GPU per rank).

Rank r owns a contiguous block of images.  Per string step:
  1. every rank integrates its own images for dt;
  2. arc lengths: each rank sends its last image to the next rank (one
     point-to-point exchange), computes the lengths of the segments that end in
     its images, and all ranks all-gather those lengths, so every rank forms the
     same prefix sums x[i] = x[i-1] + |m_i - m_{i-1}|_F in the same order;
  3. re-interpolation: each rank requests the images j, j+1 its own images
     need (normally on itself or a neighbour), the owners send them point to
     point, and the new images are normalised;
  4. energies are all-gathered.
The interpolation, bracket search and abort rules are those of
magnumaf/src/solvers/string_method.cpp (see the single-GPU maf_string_* path).

Difference to the reference, on purpose: the reference steps all images with
one integrator, so its step-size controller state passes from image to image in
order — an inherently serial chain.  Here every image keeps its own integrator
state, which makes the result independent of how many ranks share the work.

The per-image work goes through an adapter with three methods:
  ``step(i, dt)``   integrate image i for dt (until t >= t0 + dt),
  ``get(i)``        image i's m as a float64 array [3*N],
  ``set(i, m)``     replace image i's m (normalised by the caller),
  ``energy(i)``     image i's total energy;
``DeviceImages`` is the GPU adapter (one State and one LLGIntegrator per image).
"""
from __future__ import annotations

import math
from typing import Callable, List, Sequence

import numpy as np


def blocks(n: int, world: int) -> List[range]:
    """Contiguous image blocks per rank, sizes differing by at most one."""
    q, r = divmod(n, world)
    out, s = [], 0
    for k in range(world):
        e = s + q + (1 if k < r else 0)
        out.append(range(s, e))
        s = e
    return out


def frob(a: np.ndarray, b: np.ndarray) -> float:
    d = a - b
    return math.sqrt(float(np.mean(d * d)))


def normalize_soa(m: np.ndarray) -> np.ndarray:
    """Zero-safe normalisation of a [3*N] structure-of-arrays field."""
    v = m.reshape(3, -1)
    n = np.sqrt(np.sum(v * v, axis=0))
    with np.errstate(invalid="ignore", divide="ignore"):
        out = np.where(n > 0, v / np.where(n > 0, n, 1.0), 0.0)
    return out.reshape(-1)


class ShardedStringMethod:
    def __init__(self, images, n_interp: int, dt: float, inputimages: Sequence[np.ndarray], group=None):
        """images: adapter over this rank's images (global indices of its block);
        inputimages: the initial path, [3*N] float64 arrays (every rank passes all)."""
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.n = int(n_interp)
        self.dt = float(dt)
        self.img = images
        self.blocks = blocks(self.n, self.world)
        self.mine = self.blocks[self.rank]
        ins = [np.asarray(m, dtype=np.float64) for m in inputimages]
        x = [0.0]
        for i in range(1, len(ins)):
            x.append(x[-1] + frob(ins[i], ins[i - 1]))
        self.x = x
        self.x_interp = [i / (self.n - 1) * x[-1] for i in range(self.n)]
        for i in self.mine:
            j = self._bracket(i)
            if j < self.n - 1:
                a, b = ins[j], ins[j + 1]
                m = a + ((self.x_interp[i] - x[j]) * (b - a)) / (x[j + 1] - x[j])
            else:
                m = ins[j]
            self.img.set(i, normalize_soa(m))
        self.E: List[float] = []

    # string_method.cpp:22-28 / :86-92
    def _bracket(self, i: int) -> int:
        j = 0
        while j < min(self.n, len(self.x)) and self.x[j] < self.x_interp[i]:
            j += 1
        return j - 1 if j > 0 else j

    def _owner(self, i: int) -> int:
        for r, b in enumerate(self.blocks):
            if i in b:
                return r
        raise IndexError(i)

    def _allgather(self, obj):
        if self.world == 1:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj, group=self.group)
        return out

    def _exchange(self, want: List[int]) -> dict:
        """Images of other ranks by global index: every rank lists what it needs,
        owners send, requesters receive (point to point, in a fixed order)."""
        import torch

        lists = self._allgather(sorted(set(want)))
        # NCCL moves device buffers, gloo host buffers
        dev = "cuda" if self.world > 1 and self.dist.get_backend(self.group) == "nccl" else "cpu"
        got = {}
        reqs = []
        for r in range(self.world):
            for i in lists[r]:
                o = self._owner(i)
                if o == r:
                    continue
                if o == self.rank:
                    t = torch.from_numpy(self.img.get(i)).to(dev)
                    reqs.append(self.dist.isend(t, dst=r, group=self.group))
                elif r == self.rank:
                    buf = torch.empty(self.img.size, dtype=torch.float64, device=dev)
                    reqs.append(self.dist.irecv(buf, src=o, group=self.group))
                    got[i] = buf
        for q in reqs:
            q.wait()
        return {i: b.cpu().numpy() for i, b in got.items()}

    def step(self):
        for i in self.mine:
            self.img.step(i, self.dt)
        cur = {i: self.img.get(i) for i in self.mine}
        prev = self._exchange([self.mine.start - 1] if self.mine.start > 0 and len(self.mine) else [])
        seg = {}
        for i in self.mine:
            if i == 0:
                continue
            a = cur[i - 1] if (i - 1) in cur else prev[i - 1]
            seg[i] = frob(cur[i], a)
        allseg = {}
        for part in self._allgather(seg):
            allseg.update(part)
        x = [0.0]
        for i in range(1, self.n):
            x.append(x[-1] + allseg[i])
        self.x = x
        self.x_interp = [i / (self.n - 1) * x[-1] for i in range(self.n)]
        need = set()
        plan = {}
        for i in self.mine:
            j = self._bracket(i)
            plan[i] = j
            need.update([j, j + 1] if j < self.n - 1 else [j])
        remote = self._exchange([k for k in need if k not in cur])
        src = dict(cur)
        src.update(remote)
        for i in self.mine:
            j = plan[i]
            if j < self.n - 1:
                a, b = src[j], src[j + 1]
                m = a + ((self.x_interp[i] - x[j]) * (b - a)) / (x[j + 1] - x[j])
            else:
                m = src[j]
            self.img.set(i, normalize_soa(m))

    def calc_E(self) -> List[float]:
        local = {i: self.img.energy(i) for i in self.mine}
        allE = {}
        for part in self._allgather(local):
            allE.update(part)
        self.E = [allE[i] for i in range(self.n)]
        return list(self.E)

    def run(self, string_abort_rel_diff=1e-12, string_abort_abs_diff=1e-27, string_steps=10000):
        """The iteration and abort rules of string_method.cpp:174-233; returns
        (lowest barrier, iterations)."""
        max_lowest, max_prev, it = 1e100, 1e100, 0
        for i in range(string_steps):
            it = i + 1
            self.step()
            E = self.calc_E()
            barrier = max(E) - E[0]
            max_lowest = min(max_lowest, barrier)
            abs_diff = abs(barrier - max_prev)
            with np.errstate(divide="ignore", invalid="ignore"):
                rel_diff = abs(np.float64(2.0 * abs_diff) / np.float64(barrier + max_prev))
            if i > 25 and (rel_diff < string_abort_rel_diff or abs_diff < string_abort_abs_diff):
                break
            max_prev = barrier
        return max_lowest, it


class DeviceImages:
    """GPU adapter: one State and one LLGIntegrator per owned image.
    make_llg() returns a fresh magnumaf.LLGIntegrator (its own controller)."""

    def __init__(self, mesh, Ms, indices: Sequence[int], make_llg: Callable, precision="fp64"):
        import magnumaf as M

        self.M = M
        self.mesh = mesh
        self.size = 3 * mesh.nx * mesh.ny * mesh.nz
        self.states = {}
        self.llgs = {}
        m0 = np.zeros((mesh.nx, mesh.ny, mesh.nz, 3))
        m0[..., 2] = 1.0
        for i in indices:
            self.states[i] = M.State(mesh, Ms, m0, precision=precision)
            self.llgs[i] = make_llg()

    def _to_soa(self, m):
        return np.asarray(m, order="F").reshape(-1, order="F")

    def _from_soa(self, v):
        mesh = self.mesh
        return v.reshape((mesh.nx, mesh.ny, mesh.nz, 3), order="F")

    def step(self, i, dt):
        s = self.states[i]
        t0 = s.t
        while s.t < t0 + dt:
            self.llgs[i].step(s)

    def get(self, i):
        return self._to_soa(self.states[i].m).copy()

    def set(self, i, m):
        self.states[i].m = self._from_soa(m)

    def energy(self, i):
        return self.llgs[i].Eeff_in_J(self.states[i])
