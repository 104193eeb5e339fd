"""Oracle (test infrastructure, CPU, FP64 NumPy) for the string method.

Restates magnumaf/src/solvers/string_method.cpp:12-127 and :174-314 (the
iteration logic of ``run``; its output files are not restated).  Only tests
and the benchmark's CPU baseline import this module; the library never does.

Semantics kept from the reference:
  * x[i] = x[i-1] + FrobeniusNorm(m_i - m_{i-1}), FrobeniusNorm(a) =
    sqrt(mean(a*a)) over all 3N values (util.cpp:53-55); x_interp[i] =
    i / (n_interp - 1) * x[-1]  (:57-81).
  * linear re-interpolation with the reference's bracket search, including
    its "copy image j" branch when j >= n_interp - 1 (:83-106), followed by
    the zero-safe normalisation of every image (:134-140).
  * integrate(): every image is stepped with the one shared LLGIntegrator
    until image.t >= t_start + dt, so the controller state (h, errold) carries
    over from image to image (:108-121).
  * run(): barrier max(E) - E[0] per iteration, lowest barrier kept, stop
    after iteration 25 on a relative or absolute change below the thresholds
    (:174-233).
"""
import numpy as np

import maf_oracle as O


class StringMethod:
    def __init__(self, state, inputimages, n_interp, dt, llg, per_image_integrators=False):
        """state: template State (mesh, Ms / Ms_field); inputimages: list of
        States or m arrays (nx, ny, nz, 3).  per_image_integrators: every image
        gets its own copy of llg (its own controller state) instead of the
        reference's one integrator shared in image order; the sharded string
        method (magnumaf/string_sharded.py) uses that policy."""
        if not inputimages or len(inputimages) < 2:
            raise RuntimeError("StringMethod: at least two input images are needed")
        self.llg = llg
        self.per_image = per_image_integrators
        self.n_interp = int(n_interp)
        self.dt = float(dt)
        inputs = []
        for a in inputimages:
            if isinstance(a, O.State):
                inputs.append(a.copy())
            else:
                s = state.copy()
                s.m = O.normalize(np.asarray(a, dtype=np.float64))
                s.t = 0.0
                inputs.append(s)
        self._calc_x([s.m for s in inputs])
        self.images = []
        for i in range(self.n_interp):
            j = self._bracket(i)
            if j < self.n_interp - 1:
                img = state.copy()
                img.t = 0.0
                a, b = inputs[j].m, inputs[j + 1].m
                img.m = a + ((self.x_interp[i] - self.x[j]) * (b - a)) / (self.x[j + 1] - self.x[j])
            else:
                img = inputs[j].copy()
            self.images.append(img)
        self._normalize()
        self.E = []
        import copy
        self.llgs = [copy.deepcopy(llg) for _ in range(self.n_interp)] if per_image_integrators else None

    def _calc_x(self, ms):
        self.x = [0.0]
        for i in range(1, len(ms)):
            self.x.append(self.x[i - 1] + O.FrobeniusNorm(ms[i] - ms[i - 1]))
        self.x_interp = [i / (self.n_interp - 1) * self.x[-1] for i in range(self.n_interp)]

    def _bracket(self, i):
        j = 0
        while j < min(self.n_interp, len(self.x)) and self.x[j] < self.x_interp[i]:
            j += 1
        if j > 0:
            j -= 1
        return j

    def _normalize(self):
        for img in self.images:
            img.m = O.normalize(img.m)

    rk4_substeps = 0  # > 0: the batched integration of the device string (maf_string_set_batched)

    def integrate(self):
        if self.rk4_substeps:
            # every image: rk4_substeps deterministic RK4 steps of dt / rk4_substeps
            # (stochastic_integrator.cpp:34-40) with the llg's alpha and terms
            h = self.dt / self.rk4_substeps
            for img in self.images:
                for _ in range(self.rk4_substeps):
                    O.det_rk4_step(img, self.llg.terms, self.llg.alpha, h)
            return
        for i, img in enumerate(self.images):
            llg = self.llgs[i] if self.per_image else self.llg
            t0 = img.t
            while img.t < t0 + self.dt:
                llg.step(img)

    def lin_interpolate(self):
        tmp = [img.copy() for img in self.images]
        for i in range(self.n_interp):
            j = self._bracket(i)
            if j < self.n_interp - 1:
                a, b = tmp[j].m, tmp[j + 1].m
                self.images[i].m = a + ((self.x_interp[i] - self.x[j]) * (b - a)) / (self.x[j + 1] - self.x[j])
            else:
                self.images[i] = tmp[j].copy()
        self._normalize()

    def step(self):
        self.integrate()
        self._calc_x([img.m for img in self.images])
        self.lin_interpolate()

    def calc_E(self):
        self.E = [self.llg.E(img) for img in self.images]
        return list(self.E)

    def run(self, string_abort_rel_diff=1e-12, string_abort_abs_diff=1e-27, string_steps=10000):
        """Returns (lowest barrier, iterations run, barrier per iteration)."""
        max_lowest = 1e100
        max_prev = 1e100
        barriers = []
        it = 0
        for i in range(string_steps):
            it = i + 1
            self.step()
            self.calc_E()
            emax = max(self.E)
            barrier = emax - self.E[0]
            barriers.append(barrier)
            if barrier < max_lowest:
                max_lowest = barrier
            abs_diff = abs(barrier - max_prev)
            with np.errstate(divide="ignore", invalid="ignore"):  # IEEE like the reference: 0/0 -> NaN
                rel_diff = abs(np.float64(2.0 * abs_diff) / np.float64(barrier + max_prev))
            if i > 25 and rel_diff < string_abort_rel_diff:
                break
            if i > 25 and abs_diff < string_abort_abs_diff:
                break
            max_prev = barrier
        return max_lowest, it, barriers
