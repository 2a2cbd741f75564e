"""Independent numpy restatement of the reference GPE stepper (test-only).

TEST INFRASTRUCTURE ONLY -- a second, vectorised restatement used to
cross-check ``liboracle.so`` on small grids.  Boundary handling is written
differently from the C oracle on purpose: ``np.pad`` with mode ``wrap``
(periodic, src/variables.f90:186-358 single-rank exchange and the x wrap of
src/derivs.f90:290-301) or ``reflect`` (mirror about the end nodes,
src/derivs.f90:302-313, 365-394).  Arrays are complex128 shaped (nz, ny, nx).
"""
from __future__ import annotations

import numpy as np

CK_B = [
    [],
    [0.2],
    [0.075, 0.225],
    [0.3, -0.9, 1.2],
    [-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0],
    [1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0],
]
CK_C = [37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0]
CK_CS = [2825.0 / 27648.0, 0.0, 18575.0 / 48384.0, 13525.0 / 55296.0, 277.0 / 14336.0, 0.25]


class NumpyGPE:
    def __init__(self, nx, ny, nz, xr, yr, zr, *, eqn=4, bcs=1, order=2,
                 g=1.0, mu=1.0, omx=0.0, omy=0.0, omz=0.0, Urhs=0.0,
                 diss_amp=0.0, nn=1.0, real_time=True):
        self.n = (nx, ny, nz)
        self.h = tuple(2.0 * r / (n - 1) for r, n in zip((xr, yr, zr), self.n))
        self.x = -xr + np.arange(nx) * self.h[0]
        self.y = -yr + np.arange(ny) * self.h[1]
        self.z = -zr + np.arange(nz) * self.h[2]
        self.eqn, self.bcs, self.order = eqn, bcs, order
        self.g, self.mu, self.Urhs, self.diss_amp, self.nn = g, mu, Urhs, diss_amp, nn
        self.real_time = real_time
        Z, Y, X = np.meshgrid(self.z, self.y, self.x, indexing="ij")
        self.V = 0.5 * (omx ** 2 * X ** 2 + omy ** 2 * Y ** 2 + omz ** 2 * Z ** 2)
        a, b, c = self.x[-3], self.y[-3], self.z[-3]
        self.diss = diss_amp * ((1 + np.tanh(X - a) * np.tanh(X + a))
                                + (1 + np.tanh(Y - b) * np.tanh(Y + b))
                                + (1 + np.tanh(Z - c) * np.tanh(Z + c)))
        self.sphere = 0.5 * (1 + np.tanh(np.sqrt(X ** 2 + Y ** 2 + Z ** 2) - 12.0))

    def _pad(self, f):
        return np.pad(f, 2, mode="wrap" if self.bcs == 1 else "reflect")

    def d2(self, f, axis):
        """Second derivative along numpy axis (2 = x, 1 = y, 0 = z)."""
        p = self._pad(f)
        h = self.h[2 - axis]
        sl = lambda o: p[tuple(slice(2 + (o if a == axis else 0),
                                     2 + (o if a == axis else 0) + f.shape[a])
                               for a in range(3))]
        if self.order == 2:
            return (sl(1) - 2 * sl(0) + sl(-1)) / h ** 2
        return (-sl(2) + 16 * sl(1) - 30 * sl(0) + 16 * sl(-1) - sl(-2)) / (12 * h ** 2)

    def d1(self, f, axis):
        p = self._pad(f)
        h = self.h[2 - axis]
        sl = lambda o: p[tuple(slice(2 + (o if a == axis else 0),
                                     2 + (o if a == axis else 0) + f.shape[a])
                               for a in range(3))]
        if self.order == 2:
            return (sl(1) - sl(-1)) / (2 * h)
        return (-sl(2) + 8 * sl(1) - 8 * sl(-1) + sl(-2)) / (12 * h)

    def lap(self, f):
        return self.d2(f, 2) + self.d2(f, 1) + self.d2(f, 0)

    def rhs(self, f):
        L = self.lap(f)
        a2 = np.abs(f) ** 2
        if self.eqn in (1, 3):
            r = 0.5 * (1j + self.diss) * (L + (1 - a2) * f) + self.Urhs * self.d1(f, 2)
            return r * self.sphere if self.eqn == 3 else r
        if self.eqn == 2:
            return 1j * (L - a2 * f) + self.Urhs * self.d1(f, 2)
        return -1j * (-0.5 * L + self.V * f + self.g * a2 * f - self.mu * f)

    def step(self, f, dt, scheme):
        if scheme == "euler":
            return f + dt * self.rhs(f)
        if scheme == "rk2":
            return f + dt * self.rhs(f + 0.5 * dt * self.rhs(f))
        if scheme == "rk4":
            k1 = self.rhs(f)
            k2 = self.rhs(f + 0.5 * dt * k1)
            k3 = self.rhs(f + 0.5 * dt * k2)
            k4 = self.rhs(f + dt * k3)
            return f + dt * (k1 / 6 + k2 / 3 + k3 / 3 + k4 / 6)
        raise ValueError(scheme)

    def rkck(self, f, dt):
        ks = []
        for s in range(6):
            u = f + sum(b * k for b, k in zip(CK_B[s], ks))
            ks.append(dt * self.rhs(u))
        new = f + sum(c * k for c, k in zip(CK_C, ks))
        err = sum((c - cs) * k for c, cs, k in zip(CK_C, CK_CS, ks))
        return new, err

    def rkqs(self, f, dt):
        """Returns (new, dt_did, dt_next, errmax)."""
        safety, eps = 0.9, 1e-6
        errcon = (5.0 / safety) ** (1.0 / -0.2)
        psi_scal = np.abs(f) + dt * np.abs(self.rhs(f)) + 1e-30
        while True:
            new, err = self.rkck(f, dt)
            errmax = np.max(np.abs(err / psi_scal)) / eps
            if errmax <= 1.0:
                break
            mag = max(abs(safety * dt * errmax ** -0.25), 0.1 * abs(dt))
            dt = complex(mag, 0.0) if self.real_time else complex(0.0, -mag)
        dt_next = safety * dt * errmax ** -0.2 if errmax > errcon else 5.0 * dt
        return new, dt, dt_next, errmax

    def weights(self, n):
        w = np.ones(n)
        w[[0, -1]] = 3.0 / 8.0
        w[[1, -2]] = 7.0 / 6.0
        w[[2, -3]] = 23.0 / 24.0
        return w

    def norm(self, f):
        nx, ny, nz = self.n
        w = (self.weights(nz)[:, None, None] * self.weights(ny)[None, :, None]
             * self.weights(nx)[None, None, :])
        return float(np.sum(w * np.abs(f) ** 2) * self.h[0] * self.h[1] * self.h[2])

    def energy(self, f):
        e = np.real(-self.lap(f) * np.conj(f) + 0.5 * np.abs(f) ** 4)
        return float(np.sum(e) * self.h[0] * self.h[1] * self.h[2])
