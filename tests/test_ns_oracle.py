"""The Navier-Stokes oracle against properties of the continuous problem
(no GPU): the Taylor-Green vortex's kinetic energy is (lx pi)^3 v0^2 / 8
exactly; the projected right-hand side is divergence free; with nu = 0 the
dealiased advection term conserves energy; over a short time the energy of
the vortex decays as exp(-2 nu |k|^2 t) with |k|^2 = 3."""
import numpy as np
import pytest

import ns_oracle as N


@pytest.mark.parametrize("n,lx,v0", [(16, 2.0, 1.0), (24, 2.0, 0.5), (16, 4.0, 2.0)])
def test_taylor_green_energy(n, lx, v0):
    _, uk = N.taylor_green(n, n, n, lx, v0)
    e = N.energy(uk, lx, (n, n, n))
    assert abs(e / ((lx * np.pi) ** 3 * v0 * v0 / 8.0) - 1.0) < 1e-13


def _random_spectrum(shape, seed):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((3,) + shape)
    return np.fft.rfftn(u, axes=(1, 2, 3))


def test_rhs_divergence_free_and_energy_conserving():
    # extents not divisible by 3: the reference's cutoff int(n / 2 * 2 / 3) is
    # inclusive, so for n = 3 m products of kept modes alias onto |k| = m
    shape, lx = (16, 14, 20), 2.0
    k, _, inv_ksq = N.wavenumbers(*shape, lx)
    uk = N.projection(_random_spectrum(shape, 3), k, inv_ksq)  # u . grad u conserves energy if div u = 0
    ukd, r = N.rhs(uk, 0.0, lx, shape)
    div = k[0] * r[0] + k[1] * r[1] + k[2] * r[2]
    assert np.abs(div).max() < 1e-12 * np.abs(r).max() * np.abs(np.asarray(k[2])).max()
    factor = np.full(shape[2] // 2 + 1, 2.0)
    factor[0] = 1.0
    # d/dt of the energy from advection alone
    de = np.sum(factor * np.real(np.conj(ukd) * r))
    assert abs(de) < 1e-12 * np.sqrt(np.sum(factor * np.abs(ukd) ** 2) * np.sum(factor * np.abs(r) ** 2))


def test_taylor_green_decay():
    n, lx, nu, dt = 16, 2.0, 0.01, 0.01
    _, uk = N.taylor_green(n, n, n, lx)
    e0 = N.energy(uk, lx, (n, n, n))
    y = uk
    for _ in range(5):
        y = N.rk4_step(y, nu, dt, lx, (n, n, n))
    ratio = N.energy(y, lx, (n, n, n)) / e0
    assert abs(ratio / np.exp(-6.0 * nu * 5 * dt) - 1.0) < 1e-5
