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


@pytest.mark.parametrize("n,lx,v0", [(16, 2.0, 1.0), (24, 2.0, 0.5), (16, 4.0, 2.0)])
def test_taylor_green_diagnostics(n, lx, v0):
    """Vorticity of the vortex is v0 (-cos x sin y sin z, -sin x cos y sin z,
    2 sin x sin y cos z) on x = lx pi i / n, so the enstrophy is 3 times the
    energy; the field is divergence free; all its energy sits in the spectrum
    bin of |k| = sqrt(3)."""
    shape = (n, n, n)
    _, uk = N.taylor_green(n, n, n, lx, v0)
    e = N.energy(uk, lx, shape)
    assert abs(N.enstrophy(uk, lx, shape) / (3.0 * e) - 1.0) < 1e-12
    assert N.divergence_l2(uk, lx, shape) < 1e-12 * np.sqrt(e)
    x = np.arange(n) * lx * np.pi / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    w = v0 * np.stack([-np.cos(X) * np.sin(Y) * np.sin(Z), -np.sin(X) * np.cos(Y) * np.sin(Z),
                                    2.0 * np.sin(X) * np.sin(Y) * np.cos(Z)])
    assert np.max(np.abs(N.vorticity(uk, lx, shape) - w)) < 1e-12 * v0
    spec, kv = N.spectrum(uk, lx, shape, 50)
    coef = (lx * np.pi) ** 3 / float(n ** 3) ** 2
    assert abs(float(np.sum(spec)) * coef / e - 1.0) < 1e-12
    kk = np.sqrt(3.0)
    i = int(np.argmax(spec))
    half = (kv[1] - kv[0]) / 2.0
    assert kv[i] - half <= kk < kv[i] + half + 1e-12


def test_spectrum_bins_follow_the_reference():
    """Bins linspace(0, k_max, nb + 1) with the strict upper edge: the mode(s)
    at |k| = k_max fall outside every bin, as in diag_energy."""
    shape, lx = (8, 6, 10), 2.0
    rng = np.random.default_rng(5)
    uk = rng.standard_normal((3, 8, 6, 6)) + 1j * rng.standard_normal((3, 8, 6, 6))
    spec, kv = N.spectrum(uk, lx, shape, 7)
    _, ksq, _ = N.wavenumbers(*shape, lx)
    km = np.sqrt(ksq)
    f = np.full(6, 2.0)
    f[0] = 1.0
    ek = 0.5 * f[None, None, :] * np.sum(np.abs(uk) ** 2, axis=0)
    assert abs(float(np.sum(spec)) - float(np.sum(ek[km < km.max()]))) < 1e-9 * float(np.sum(ek))
    assert np.allclose(kv, (np.arange(7) + 0.5) * km.max() / 7, rtol=0, atol=1e-12)


def test_energy_factor_at_the_reference_decomposition():
    """The example takes the Hermitian factor of its energy by the local z
    index of each rank's output block; at out_topology (1, 1, px, 1) (z not
    split) that is the global kz = 0 plane and the two sums agree exactly; with
    z split (py > 1) the example weights the first plane of every z block by 1
    instead of 2, so its diagnostic differs from the energy by that plane's
    share (the solver itself is unaffected)."""
    shape, lx = (16, 16, 16), 2.0
    rng = np.random.default_rng(9)
    k, _, inv_ksq = N.wavenumbers(*shape, lx)
    uk = N.projection(np.fft.rfftn(rng.standard_normal((3,) + shape), axes=(1, 2, 3)), k, inv_ksq)
    e = N.energy(uk, lx, shape)
    assert N.energy_with_block_local_factor(uk, lx, shape, [(0, 9)]) == e
    z_split = [(0, 5), (5, 4)]  # 9 half-spectrum planes over py = 2 (first n % P bins larger)
    e_blocks = N.energy_with_block_local_factor(uk, lx, shape, z_split)
    plane = 0.5 * np.sum(np.abs(uk[..., 5]) ** 2) * (lx * np.pi) ** 3 / float(16 ** 3) ** 2
    assert abs((e - e_blocks) - plane) <= 1e-12 * e
