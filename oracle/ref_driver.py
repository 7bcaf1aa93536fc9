"""TEST INFRASTRUCTURE ONLY -- the reference's kernels run on the host CPU.

Used by ``bench.py`` as the CPU baseline ("reference" kind): the
reference's own kernels (PyFWI src/PyFWI/elastic.cl, elastic_surface.cl,
compiled for the CPU by ``ref_build``/``ref_programs`` and recorded in
oracle/_ref/manifest.json) driven in the order of the reference's host loops
(wave_propagation.py:699-733 forward, :751-848 gradient with every step
stored as chpr = 100 does).  One ``run_shot`` call models one shot over the
first ``nsteps`` steps and back-propagates over them.

Buffers keep zero guard bands (the reference kernels read up to four rows
past either end of a field)."""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
import ref_build  # noqa: E402


class _Buf:
    GUARD = 1 << 16

    def __init__(self, n, init=None):
        self.store = np.zeros(n + 2 * self.GUARD, np.float32)
        self.v = self.store[self.GUARD:self.GUARD + n]
        if init is not None:
            self.v[:] = np.asarray(init, np.float32).reshape(-1)

    @property
    def a(self):
        return self.v.ctypes.data


def available(name):
    man = ref_build.load_manifest()
    if name not in man:
        return False
    return all(os.path.exists(os.path.join(HERE, man[name][k]["so"])) for k in ("main", "surface"))


class RefRunner:
    """Reference kernels for the geometry recorded under ``name``."""

    def __init__(self, name, W):
        """W: an oracle.OracleWavePropagator of the same survey (set-up values
        and materials)."""
        self.progs = ref_build.load_programs(name)
        self.W = W
        self.main = self.progs["main"]
        acq = int(W.acq_type)
        self.inj = self.progs["surface"] if acq == 1 else (self.progs["crosswell"] if acq == 0 else self.main)
        n = int(W.tnz) * int(W.tnx)
        self.n = n
        self.g = (int(W.tnz), int(W.tnx))
        self.lam = _Buf(n, W.lam)
        self.mu = _Buf(n, W.mu)
        self.rho_b = _Buf(n, W.rho_b)
        self.vdx = _Buf(n, W.vdx)
        self.vdz = _Buf(n, W.vdz)
        self.f = [_Buf(n) for _ in range(5)]
        self.af = [_Buf(n) for _ in range(5)]
        self.G = [_Buf(n) for _ in range(6)]
        self.seis = [_Buf(int(W.nt_ext) * int(W.nr)) for _ in range(5)]
        self.res = [_Buf(int(W.nr)) for _ in range(5)]

    def _fwd4(self, coeff):
        m, g, f = self.main, self.g, self.f
        m.launch("update_velx", g, [coeff, f[0].a, f[2].a, f[4].a, self.rho_b.a, self.vdx.a, self.vdz.a])
        m.launch("update_velz", g, [coeff, f[1].a, f[3].a, f[4].a, self.rho_b.a, self.vdx.a, self.vdz.a])
        m.launch("update_tauz", g, [coeff, f[0].a, f[1].a, f[2].a, f[3].a, self.lam.a, self.mu.a, self.vdx.a,
                                    self.vdz.a])
        m.launch("update_tauxz", g, [coeff, f[0].a, f[1].a, f[4].a, self.mu.a, self.vdx.a, self.vdz.a])

    def run_shot(self, s, nsteps, residual=None):
        """Forward over steps [0, nsteps) storing every state, then the
        backward loop over t = nsteps-1 .. 1.  Returns seconds spent."""
        W, g = self.W, self.g
        if not 0 < nsteps <= int(W.nt):
            # the reference's trace buffers hold nt_ext rows: more steps would
            # write past them
            raise ValueError("nsteps must be in [1, %d], not %d" % (int(W.nt), nsteps))
        t0 = time.perf_counter()
        for b in self.f:
            b.v[:] = 0
        store = np.zeros((nsteps, 5, self.n), np.float32)
        t_src = 0
        for t in range(nsteps):
            if t % int(W.dt_scale) == 0:
                v = W.src_vals[t_src] if t_src < len(W.src_vals) else np.zeros(4, np.float32)
                self.inj.launch("injSrc", g, [b.a for b in self.f] + [b.a for b in self.seis] +
                                [int(W.dxr), int(W.srcx[s]), int(W.srcz[s]), v[0], v[1], v[2], v[3], t_src])
                t_src += 1
            self._fwd4(1)
            for k in range(5):
                store[t, k] = self.f[k].v
        for b in self.af + self.G:
            b.v[:] = 0
        nr = int(W.nr)
        t_src = nsteps // int(W.dt_scale)
        for t in range(nsteps - 1, 0, -1):
            for k in range(5):
                self.f[k].v[:] = store[t, k]
            if t % int(W.dt_scale) == 0:
                for k in range(5):
                    row = residual[k][t_src - 1, s * nr:(s + 1) * nr] if residual is not None else 0.0
                    self.res[k].v[:] = row
                self.inj.launch("Adj_injSrc", g, [b.a for b in self.af] + [b.a for b in self.res] + [int(W.dxr)])
                t_src -= 1
            self.main.launch("Adj_update_tau", g, [b.a for b in self.af] + [self.rho_b.a, self.vdx.a, self.vdz.a])
            self.main.launch("Adj_update_v", g, [b.a for b in self.af] + [self.lam.a, self.mu.a, self.vdx.a,
                                                                          self.vdz.a])
            Gp = self.G
            self.main.launch("Grad", g, [b.a for b in self.f] + [b.a for b in self.af] +
                             [self.lam.a, self.mu.a, self.rho_b.a, Gp[0].a, Gp[3].a, Gp[1].a, Gp[4].a, Gp[2].a,
                              Gp[5].a])
        return time.perf_counter() - t0
