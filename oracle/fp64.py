"""FP64 restatement of the phasing iteration -- TEST INFRASTRUCTURE ONLY.

A NumPy float64/complex128 statement of the reference CPU engine's steps, for
stating the rounding error of a float32 result (the GPU library's, or the
reference engine's) against exact-as-possible arithmetic.  It follows the
same algorithm and cadence as ``oracle/sporacle.c`` but evaluates every step
in double precision with NumPy's FFT:

* iteration dispatch and support-update cadence: src/phasing.c:895-1024 (an
  update consumes one iteration slot);
* ER / HIO / RAAR: src/phasing.c:1111-1219; difference map with its f1
  transform: src/phasing.c:1222-1274;
* Fourier constraints, modulus projection (with the error-margin mode) and
  phased-amplitude projection: src/phasing.c:1061-1109;
* real-space constraints: src/phasing.c:1026-1059;
* area and threshold support updates: src/support_update.c:124-179 with the
  Fourier-domain Gaussian blur of src/image_filter.c:80-90 and
  dist_to_top_left (src/image_util.c:1012-1032), area index (int)(N*area) of
  |blur| sorted descending, strict ``>``.

Schedule values (beta, blur radius, area) are host inputs, taken as the
reference evaluates them (float Bezier schedule, ``oracle.bezier``).  The
starting model is an input too (``set_model``): a float32 run's start is
given to both, so the error measured is that of the iterations alone.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module.
"""
from __future__ import annotations

import numpy as np

HIO, RAAR, DIFFMAP, ER = 1, 2, 3, 4
SUP_THRESHOLD, SUP_AREA, SUP_STATIC = 1, 2, 5
REAL, POS_REAL, POS_COMPLEX, FLIP, CENTROSYM, MARGIN = 1, 2, 4, 8, 16, 32
INSIDE, MEASURED = 1, 2


def _sched(s):
    return s if isinstance(s, dict) else {0: float(s)}


def schedule_value(s, iteration):
    from oracle import bezier

    return float(np.float32(bezier(_sched(s), float(iteration))))


class Fp64Phaser:
    """One reconstruction in float64 (arrays (nz, ny, nx) or (ny, nx))."""

    def __init__(self, shape):
        shape = tuple(int(s) for s in shape)
        self.out_shape = shape
        self.shape3 = shape if len(shape) == 3 else (1,) + shape
        self.nz, self.ny, self.nx = self.shape3
        self.n = self.nx * self.ny * self.nz
        self.flags_ = np.zeros(self.shape3, np.int32)
        self.sup = []
        self.period = 0
        self.iteration = 0
        self.objective = 0
        self.amp = self.amin = self.amax = self.pamp = None
        self.g0 = self.g1 = self.gp = None

    # -- configuration --
    def set_algorithm(self, alg, beta=0.9, constraints=0, gamma1=float("inf"), gamma2=float("inf")):
        self.alg, self.beta, self.constraints = alg, beta, constraints
        if alg == DIFFMAP:
            if np.isinf(gamma1):
                # sp_phasing_diff_map_alloc defaults (src/phasing.c:50-76), sigma 0.1
                b, s = schedule_value(beta, 0), 0.1
                gamma1 = -(4 + (2 + b) * s + b * s * s) / (b * (4 - s + s * s))
                gamma2 = (3 - b) / (2 * b)
            self.gamma1, self.gamma2 = float(gamma1), float(gamma2)

    def add_support_update(self, kind, period, blur, sel):
        self.sup.append((kind, blur, sel))
        self.period = period

    def set_amplitudes(self, amp, mask):
        self.amp = np.asarray(amp, np.float64).reshape(self.shape3)
        m = np.asarray(mask).reshape(self.shape3) != 0
        self.flags_ = np.where(m, self.flags_ | MEASURED, self.flags_ & ~MEASURED)

    def set_amplitudes_margins(self, amin, amax):
        self.amin = np.asarray(amin, np.float64).reshape(self.shape3)
        self.amax = np.asarray(amax, np.float64).reshape(self.shape3)

    def set_phased_amplitudes(self, pa, mask):
        self.pamp = np.asarray(pa, np.complex128).reshape(self.shape3)
        m = np.asarray(mask).reshape(self.shape3) != 0
        self.flags_ = np.where(m, self.flags_ | MEASURED, self.flags_ & ~MEASURED)

    def set_objective(self, obj):
        self.objective = obj

    def set_support(self, support):
        s = np.real(np.asarray(support)).reshape(self.shape3) != 0
        self.flags_ = np.where(s, self.flags_ | INSIDE, self.flags_ & ~INSIDE)

    def set_flags(self, flags):
        self.flags_ = np.asarray(flags, np.int32).reshape(self.shape3).copy()

    def set_model(self, model, iteration=0):
        """g1 = model (a float32 run's start), g0 = gp = 0."""
        self.g1 = np.asarray(model, np.complex128).reshape(self.shape3).copy()
        self.g0 = np.zeros_like(self.g1)
        self.gp = np.zeros_like(self.g1)
        self.iteration = iteration

    # -- steps --
    def _constraints(self, g):
        c, ins = self.constraints, (self.flags_ & INSIDE) != 0
        re, im = g.real.copy(), g.imag.copy()
        if c & REAL:
            im[ins] = 0
        elif c & POS_REAL:
            neg = ins & (re < 0)
            re[neg] = np.abs(re[neg]) if c & FLIP else 0
            im[ins] = 0
        elif c & POS_COMPLEX:
            neg = ins & (re < 0)
            re[neg] = np.abs(re[neg]) if c & FLIP else 0
            neg = ins & (im < 0)
            im[neg] = np.abs(im[neg]) if c & FLIP else 0
        return re + 1j * im

    def _fourier_constraints(self, G):
        if self.constraints & CENTROSYM:
            return G.real + 0j
        return G

    def _module_projection(self, G):
        meas = (self.flags_ & MEASURED) != 0
        a = np.abs(G)
        with np.errstate(divide="ignore", invalid="ignore"):
            if not self.constraints & MARGIN:
                m = self.amp / a
            else:
                m = np.ones_like(a)
                lo, hi = a < self.amin, a > self.amax
                m[lo] = self.amin[lo] / a[lo]
                m[hi & ~lo] = self.amax[hi & ~lo] / a[hi & ~lo]
        fin = np.isfinite(m)
        out = G.copy()
        out[meas & fin] = G[meas & fin] * m[meas & fin]
        bad = meas & ~fin
        out[bad] = self.amp[bad]
        return out

    def _project(self, G):
        if self.objective == 0:
            return self._module_projection(G)
        meas = (self.flags_ & MEASURED) != 0
        return np.where(meas, self.pamp, G)

    def _step_simple(self):
        beta = 0.0 if self.alg == ER else schedule_value(self.beta, self.iteration)
        self.g0, self.g1 = self.g1, self.g0
        G = self._project(self._fourier_constraints(np.fft.fftn(self.g0)))
        self.gp = np.fft.ifftn(G)
        ins = (self.flags_ & INSIDE) != 0
        if self.alg == HIO:
            out = self.g0 - self.gp * beta
        elif self.alg == RAAR:
            out = self.gp * (1 - 2 * beta) + self.g0 * beta
        else:
            out = np.zeros_like(self.gp)
        self.g1 = self._constraints(np.where(ins, self.gp, out))
        self.iteration += 1

    def _step_diff_map(self):
        beta = schedule_value(self.beta, self.iteration)
        g1c, g2c = self.gamma1, self.gamma2
        self.g0, self.g1 = self.g1, self.g0
        ins = (self.flags_ & INSIDE) != 0
        G = self._fourier_constraints(np.fft.fftn(self.g0))
        f1 = np.where(ins, self.g0, -g1c * self.g0)
        f1 = np.fft.ifftn(self._module_projection(np.fft.fftn(f1)))
        rho = np.fft.ifftn(self._module_projection(G))
        self.gp = rho * self.n  # the reference keeps the unnormalised backward transform here
        g = np.where(ins, self.g0 + beta * ((1 + g2c) * rho - g2c * self.g0), self.g0)
        self.g1 = self._constraints(g - beta * f1)
        self.iteration += 1

    def _blur(self, x, radius):
        """sp_gaussian_blur in float64 (src/image_filter.c:80-90): the radius
        is measured in units of nx on every axis."""
        def d(n):
            i = np.arange(n, dtype=np.float64)
            return np.minimum(i, n - i)

        dz, dy, dx = np.meshgrid(d(self.nz), d(self.ny), d(self.nx), indexing="ij")
        cr = np.sqrt(dx * dx + dy * dy + dz * dz) / self.nx
        return np.fft.ifftn(np.fft.fftn(x) * np.exp(-2.0 * np.pi ** 2 * cr ** 2 * float(radius) ** 2))

    def _support_update(self):
        for kind, blur, sel in self.sup:
            if kind not in (SUP_AREA, SUP_THRESHOLD):
                continue
            b = np.abs(self._blur(np.abs(self.g1), schedule_value(blur, self.iteration)))
            v = schedule_value(sel, self.iteration)
            if kind == SUP_AREA:
                idx = int(np.float32(self.n) * np.float32(v))
                t = np.sort(b.ravel())[::-1][min(idx, self.n - 1)]
            else:
                t = b.max() * v
            self.flags_ = np.where(b > t, self.flags_ | INSIDE, self.flags_ & ~INSIDE)

    def iterate(self, iterations):
        step = self._step_diff_map if self.alg == DIFFMAP else self._step_simple
        if not self.sup:
            for _ in range(iterations):
                step()
            return 0
        while iterations:
            to_update = self.period - 1 - self.iteration % self.period
            k = min(iterations, to_update)
            for _ in range(k):
                step()
            iterations -= k
            to_update -= k
            if to_update == 0 and iterations > 0:
                self._support_update()
                self.iteration += 1
                iterations -= 1
        return 0

    # -- results --
    def _out(self, a):
        return a.reshape(self.out_shape)

    def get(self, which):
        return self._out((self.g0, self.g1, self.gp)[which])

    def model(self):
        return self.get(1)

    def flags(self):
        return self._out(self.flags_)

    def support(self):
        return self._out((self.flags_ & INSIDE).astype(np.int32))

    def efourier(self):
        """(E_F, FcFo) of the model, src/phasing.c:852-891, in float64."""
        return efourier64(self.g1, self.amp, self.flags_)


def efourier64(model, amp, flags):
    """(E_F, FcFo) of a model (src/phasing.c:852-891) evaluated in float64:
    for stating the Fourier error of a float32 model without the rounding of
    the reference's float accumulation."""
    model = np.asarray(model, np.complex128)
    F = np.abs(np.fft.fftn(model))
    meas = (np.asarray(flags).reshape(model.shape) & MEASURED) != 0
    A = np.abs(np.asarray(amp, np.float64).reshape(model.shape))
    nom = ((F - A) ** 2)[meas].sum()
    den = (A ** 2)[meas].sum() + (F ** 2)[~meas].sum()
    return float(np.sqrt(nom / den)), float(A[meas].sum() / F[meas].sum())


def rel_l2(a, b):
    """||a - b|| / ||b|| in float64."""
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
