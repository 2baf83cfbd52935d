"""CPU oracle for the pseudo-spectral Navier-Stokes step (test infrastructure).

Only the tests and ``bench.py``'s CPU legs use this module, as the checker or
as the timed CPU baseline; the library never calls it.

It restates, in numpy float64 on global arrays, the reference's batched
example (``examples/navier-stokes-MPI-batched/main.cpp``) and its RK4 solver
(``examples/utils/math_utils.hpp``):

* ``wavenumbers``   Grid: fftfreq(n, lx / (2 n)) and rfftfreq (main.cpp:123-137),
                    k^2 and 1 / k^2 with 0 at the origin (main.cpp:146-162)
* ``alias_mask``    2/3 rule, keep |m| <= int(n / 2 * 2 / 3) (main.cpp:165-192)
* ``taylor_green``  x = linspace(0, lx pi, n, endpoint=False) (main.cpp:103-105),
                    u = (v0 sin x cos y cos z, -v0 cos x sin y cos z, 0) (main.cpp:322-337),
                    forward transform, dealias, projection (main.cpp:355-363)
* ``rhs``           dealias uk in place, i k uk, four backward transforms, u . grad u,
                    one forward transform, dealias, -adv - nu k^2 uk, projection
                    (main.cpp:536-586 with derivative :596-616, advection :629-645,
                    combine :655-669, dealias :220-233, projection :241-260)
* ``rk4_step``      low-storage RK4 stages 0..3 (math_utils.hpp:90-141), each stage after
                    one ``rhs`` (main.cpp:518-528)
* ``energy``        coef * sum 0.5 * factor * |uk|^2, factor 1 on the kz = 0 plane, else 2,
                    coef = (lx pi)^3 / N^2 (main.cpp:511-513, :746-766)
* ``vorticity``     i k x uk with the full wavenumbers, backward transform (main.cpp:677-698)
* ``spectrum``      radial bins linspace(0, k_max, nb + 1) over |k| (main.cpp:471-500), per bin
                    sum 0.5 * factor * |uk|^2 with bins[i] <= |k| < bins[i + 1] (main.cpp:741-794)
* ``enstrophy``, ``divergence_l2``  coef * sum 0.5 * factor * |k x uk|^2 and
                    (coef * sum factor * |k . uk|^2)^(1/2): (1/2) int |curl u|^2 and (int |div u|^2)^(1/2)

Transforms are numpy's pocketfft with the reference's default ``backward``
normalisation (forward unscaled, backward scaled by 1 / N), the same
convention as ``dfft_oracle.global_fft``.  Arrays are the global
(3, nx, ny, nz) real field and the (3, nx, ny, nz / 2 + 1) half spectrum.
"""
import numpy as np


def wavenumbers(nx, ny, nz, lx):
    """(kx, ky, kz) broadcastable to (nx, ny, nz // 2 + 1), ksq, inv_ksq."""
    kx = np.fft.fftfreq(nx, lx / (2.0 * nx))[:, None, None]
    ky = np.fft.fftfreq(ny, lx / (2.0 * ny))[None, :, None]
    kz = np.fft.rfftfreq(nz, lx / (2.0 * nz))[None, None, :]
    ksq = kx * kx + ky * ky + kz * kz
    with np.errstate(divide="ignore"):
        inv_ksq = np.where(ksq == 0.0, 0.0, 1.0 / np.where(ksq == 0.0, 1.0, ksq))
    return (kx, ky, kz), ksq, inv_ksq


def alias_mask(nx, ny, nz):
    mx = np.rint(np.fft.fftfreq(nx) * nx).astype(np.int64)[:, None, None]
    my = np.rint(np.fft.fftfreq(ny) * ny).astype(np.int64)[None, :, None]
    mz = np.arange(nz // 2 + 1)[None, None, :]
    cx, cy, cz = (nx // 2) * 2 // 3, (ny // 2) * 2 // 3, (nz // 2) * 2 // 3
    keep = (np.abs(mx) <= cx) & (np.abs(my) <= cy) & (mz <= cz)
    return keep.astype(np.float64)


def _fwd(u):
    return np.fft.rfftn(u, axes=(1, 2, 3))


def _bwd(uk, shape):
    return np.fft.irfftn(uk, s=shape, axes=(1, 2, 3))


def projection(uk, k, inv_ksq):
    div = (k[0] * uk[0] + k[1] * uk[1] + k[2] * uk[2]) * inv_ksq
    return np.stack([uk[d] - k[d] * div for d in range(3)])


def taylor_green(nx, ny, nz, lx, v0=1.0):
    """(u, uk): the physical field and its dealiased, projected spectrum."""
    x = lx * np.pi * np.arange(nx) / nx
    y = lx * np.pi * np.arange(ny) / ny
    z = lx * np.pi * np.arange(nz) / nz
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    u = np.stack([v0 * np.sin(X) * np.cos(Y) * np.cos(Z), -v0 * np.cos(X) * np.sin(Y) * np.cos(Z),
                  np.zeros_like(X)])
    k, _, inv_ksq = wavenumbers(nx, ny, nz, lx)
    uk = _fwd(u) * alias_mask(nx, ny, nz)
    return u, projection(uk, k, inv_ksq)


def rhs(uk, nu, lx, shape):
    """Returns (dealiased uk, dukdt); ``uk`` itself is not modified."""
    nx, ny, nz = shape
    k, ksq, inv_ksq = wavenumbers(nx, ny, nz, lx)
    mask = alias_mask(nx, ny, nz)
    uk = uk * mask
    u = _bwd(uk, shape)
    du = [_bwd(1j * k[a] * uk, shape) for a in range(3)]
    adv = np.stack([u[0] * du[0][d] + u[1] * du[1][d] + u[2] * du[2][d] for d in range(3)])
    advk = _fwd(adv) * mask
    r = -advk + (-nu * ksq) * uk
    return uk, projection(r, k, inv_ksq)


def rk4_step(uk, nu, dt, lx, shape):
    """One time step (four right-hand sides) of the reference's RK4 solver."""
    y = uk
    y, f = rhs(y, nu, lx, shape)
    y0 = y
    k1 = f * dt
    y = y0 + k1 / 2.0
    y, f = rhs(y, nu, lx, shape)
    k2 = f * dt
    y = y0 + k2 / 2.0
    y, f = rhs(y, nu, lx, shape)
    k3 = f * dt
    y = y0 + k3
    y, f = rhs(y, nu, lx, shape)
    return y0 + (k1 + 2.0 * k2 + 2.0 * k3 + f * dt) / 6.0


def energy(uk, lx, shape):
    nx, ny, nz = shape
    n = float(nx) * ny * nz
    factor = np.full(uk.shape[-1], 2.0)
    factor[0] = 1.0
    e = 0.5 * factor[None, None, None, :] * (uk.real ** 2 + uk.imag ** 2)
    return float(np.sum(e) * (lx * np.pi) ** 3 / (n * n))


def _factor(nzh):
    f = np.full(nzh, 2.0)
    f[0] = 1.0
    return f[None, None, :]


def vorticity(uk, lx, shape):
    """Physical vorticity (3, nx, ny, nz) of the spectrum uk (compute_vorticity)."""
    k, _, _ = wavenumbers(*shape, lx)
    kx, ky, kz = k
    w = np.stack([1j * (ky * uk[2] - kz * uk[1]), 1j * (kz * uk[0] - kx * uk[2]), 1j * (kx * uk[1] - ky * uk[0])])
    return _bwd(w, shape)


def enstrophy(uk, lx, shape):
    nx, ny, nz = shape
    n = float(nx) * ny * nz
    k, _, _ = wavenumbers(*shape, lx)
    kx, ky, kz = k
    c = [ky * uk[2] - kz * uk[1], kz * uk[0] - kx * uk[2], kx * uk[1] - ky * uk[0]]
    s = sum(np.abs(ci) ** 2 for ci in c)
    return float(np.sum(0.5 * _factor(uk.shape[-1]) * s) * (lx * np.pi) ** 3 / (n * n))


def divergence_l2(uk, lx, shape):
    nx, ny, nz = shape
    n = float(nx) * ny * nz
    k, _, _ = wavenumbers(*shape, lx)
    d = k[0] * uk[0] + k[1] * uk[1] + k[2] * uk[2]
    return float(np.sqrt(np.sum(_factor(uk.shape[-1]) * np.abs(d) ** 2) * (lx * np.pi) ** 3 / (n * n)))


def spectrum(uk, lx, shape, num_bins=50):
    """(e_spec, k_vals) of diag_energy: bin edges linspace(0, k_max, nb + 1),
    k_max the largest |k| of the grid, midpoints as k values."""
    _, ksq, _ = wavenumbers(*shape, lx)
    k_mag = np.sqrt(ksq)
    k_max = float(np.max(k_mag))
    delta = (k_max - 0.0) / num_bins
    bins = np.array([0.0 + delta * i for i in range(num_bins)] + [k_max])
    ek = 0.5 * _factor(uk.shape[-1]) * np.sum(np.abs(uk) ** 2, axis=0)
    spec = np.zeros(num_bins)
    for i in range(num_bins):
        m = (k_mag >= bins[i]) & (k_mag < bins[i + 1])
        spec[i] = float(np.sum(ek[m]))
    return spec, 0.5 * (bins[:-1] + bins[1:])


def energy_with_block_local_factor(uk, lx, shape, z_blocks):
    """The example's diag_energy sum with its factor taken by the local z
    index of each output block (main.cpp:741-766: factor 1 where the block's
    local i2 == 0): z_blocks lists the (start, extent) of the z bins of the
    output topology.  Equal to ``energy`` when z is not split."""
    nx, ny, nz = shape
    n = float(nx) * ny * nz
    factor = np.full(uk.shape[-1], 2.0)
    for start, _ in z_blocks:
        factor[start] = 1.0
    e = 0.5 * factor[None, None, None, :] * (uk.real ** 2 + uk.imag ** 2)
    return float(np.sum(e) * (lx * np.pi) ** 3 / (n * n))
