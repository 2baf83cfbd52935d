"""Navier-Stokes step of the reference's batched example on the GPU plan,
against the numpy oracle (ns_oracle) on the same inputs.

The plan is the example's: R2C over LayoutRight 4D views (3, nx, ny, nz),
axes (1, 2, 3), in_topology (1, px, py, 1), out_topology (1, 1, px, py)
(examples/navier-stokes-MPI-batched/main.cpp:96-102, 476-479).  Checked:
the Taylor-Green initial spectrum, one right-hand side (and the in-place
dealiasing of uk), two RK4 steps, the kinetic energy, and the energy decay
of the vortex against exp(-6 nu t).  Tolerances: relative L2 <= 1e-12 for
float64, <= 1e-5 for float32."""
import numpy as np
import pytest

import dfft
import ns_oracle as N

pytestmark = pytest.mark.gpu

CASES = [
    ((16, 16, 16), (1, 2, 1, 1), (1, 1, 2, 1)),   # slab, px = 2 (the example's default split)
    ((16, 16, 16), (1, 2, 2, 1), (1, 1, 2, 2)),   # pencil 2 x 2
    ((24, 20, 18), (1, 3, 2, 1), (1, 1, 3, 2)),   # ragged pencil 3 x 2
    ((16, 14, 20), (1, 1, 1, 1), (1, 1, 1, 1)),   # one rank
]


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b)))


def _setup(shape, tin, tout, precision):
    import torch
    nx, ny, nz = shape
    plan = dfft.Plan((3, nx, ny, nz), (3, nx, ny, nz // 2 + 1), (1, 2, 3), tin, tout, real_input=True,
                     precision=precision)
    cdt = torch.complex128 if precision == "float64" else torch.complex64
    return plan, cdt


def _to_dev(plan, a, cdt):
    import torch
    np_c = np.complex128 if cdt == torch.complex128 else np.complex64
    return torch.from_numpy(np.ascontiguousarray(dfft.scatter_blocks(plan, a.astype(np_c), "out"))).cuda()


def _to_host(plan, t):
    import torch
    torch.cuda.synchronize()
    return dfft.gather_blocks(plan, t.cpu().numpy(), "out").astype(np.complex128)


def _random_spectrum(shape, seed, lx):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((3,) + shape)
    k, _, inv_ksq = N.wavenumbers(*shape, lx)
    return N.projection(np.fft.rfftn(u, axes=(1, 2, 3)), k, inv_ksq)


@pytest.mark.parametrize("shape,tin,tout", CASES)
@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_ns_matches_oracle(shape, tin, tout, precision):
    import torch
    lx, nu, dt = 2.0, 0.01, 0.01
    tol = 1e-12 if precision == "float64" else 1e-5
    plan, cdt = _setup(shape, tin, tout, precision)
    ns = dfft.NavierStokes(plan, nu=nu, dt=dt, lx=lx)
    nout = plan.buffer_elements("out")

    # Taylor-Green initial condition and its energy
    uk = torch.empty(nout, dtype=cdt, device="cuda")
    ns.init_taylor_green(uk, v0=1.0)
    _, ref_tg = N.taylor_green(*shape, lx)
    assert _rel(_to_host(plan, uk), ref_tg) <= tol
    e = ns.energy(uk)
    assert abs(e / N.energy(ref_tg, lx, shape) - 1.0) <= tol

    # one right-hand side of a random divergence-free field (not dealiased:
    # rhs dealiases uk in place, as the reference does)
    y = _random_spectrum(shape, 7, lx)
    uk = _to_dev(plan, y, cdt)
    dukdt = torch.empty_like(uk)
    ns.rhs(uk, dukdt)
    ref_ukd, ref_r = N.rhs(y, nu, lx, shape)
    assert _rel(_to_host(plan, uk), ref_ukd) <= tol
    assert _rel(_to_host(plan, dukdt), ref_r) <= tol

    # two RK4 steps
    uk = _to_dev(plan, y, cdt)
    ref = y
    for _ in range(2):
        ns.step(uk)
        ref = N.rk4_step(ref, nu, dt, lx, shape)
    assert _rel(_to_host(plan, uk), ref) <= tol * 10
    assert abs(ns.energy(uk) / N.energy(ref, lx, shape) - 1.0) <= tol * 10


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_taylor_green_decay(precision):
    """E(t) / E(0) of the vortex follows exp(-2 nu |k|^2 t), |k|^2 = 3, over
    short times; E(0) = (lx pi)^3 / 8."""
    import torch
    n, lx, nu, dt, steps = 32, 2.0, 0.01, 0.01, 10
    plan, cdt = _setup((n, n, n), (1, 2, 2, 1), (1, 1, 2, 2), precision)
    ns = dfft.NavierStokes(plan, nu=nu, dt=dt, lx=lx)
    uk = torch.empty(plan.buffer_elements("out"), dtype=cdt, device="cuda")
    ns.init_taylor_green(uk)
    e0 = ns.energy(uk)
    assert abs(e0 / np.pi ** 3 - 1.0) < (1e-13 if precision == "float64" else 1e-6)
    prev = e0
    for _ in range(steps):
        ns.step(uk)
        e = ns.energy(uk)
        assert e < prev
        prev = e
    ratio = prev / e0
    assert abs(ratio / np.exp(-6.0 * nu * steps * dt) - 1.0) < (1e-5 if precision == "float64" else 1e-4)


def test_ns_rejects_wrong_plan():
    plan = dfft.Plan((16, 16, 16), (16, 16, 9), (0, 1, 2), (2, 1, 1), (1, 2, 1), real_input=True)
    with pytest.raises(dfft.DistributedFFTError):
        dfft.NavierStokes(plan)
    plan = dfft.Plan((3, 16, 16, 16), (3, 16, 16, 16), (1, 2, 3), (1, 2, 1, 1), (1, 1, 2, 1))
    with pytest.raises(dfft.DistributedFFTError):
        dfft.NavierStokes(plan)
    # component axis split across ranks
    plan = dfft.Plan((3, 16, 16, 16), (3, 16, 16, 9), (1, 2, 3), (3, 1, 1, 1), (3, 1, 1, 1), real_input=True)
    with pytest.raises(dfft.DistributedFFTError):
        dfft.NavierStokes(plan)


@pytest.mark.parametrize("shape,tin,tout", CASES)
@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_ns_diagnostics_match_oracle(shape, tin, tout, precision):
    """Velocity and vorticity in physical space, FP64 energy / enstrophy /
    divergence and the 50-bin energy spectrum of a random (not projected)
    spectrum against the oracle's restatement of main.cpp:677-794."""
    import torch
    lx = 2.0
    tol = 1e-12 if precision == "float64" else 1e-5
    plan, cdt = _setup(shape, tin, tout, precision)
    ns = dfft.NavierStokes(plan, nu=0.01, dt=0.01, lx=lx)
    rng = np.random.default_rng(11)
    y = np.fft.rfftn(rng.standard_normal((3,) + shape), axes=(1, 2, 3))
    uk = _to_dev(plan, y, cdt)
    rdt = torch.float64 if precision == "float64" else torch.float32
    u = torch.empty(plan.buffer_elements("in"), dtype=rdt, device="cuda")
    ns.velocity(uk, u)
    torch.cuda.synchronize()
    assert _rel(dfft.gather_blocks(plan, u.cpu().numpy(), "in"), np.fft.irfftn(y, s=shape, axes=(1, 2, 3))) <= tol
    ns.vorticity(uk, u)
    torch.cuda.synchronize()
    assert _rel(dfft.gather_blocks(plan, u.cpu().numpy(), "in"), N.vorticity(y, lx, shape)) <= tol
    assert _rel(_to_host(plan, uk), y) <= (0.0 if precision == "float64" else 1e-7)  # uk not modified
    d = ns.diagnostics(uk, num_bins=50)
    yq = _to_host(plan, uk)  # the values the GPU saw (FP32-rounded for float32)
    dtol = 1e-12
    assert abs(d["energy"] / N.energy(yq, lx, shape) - 1.0) <= dtol
    assert abs(d["enstrophy"] / N.enstrophy(yq, lx, shape) - 1.0) <= dtol
    assert abs(d["divergence_l2"] / N.divergence_l2(yq, lx, shape) - 1.0) <= dtol
    spec, kv = N.spectrum(yq, lx, shape, 50)
    assert np.allclose(d["e_spec"], spec, rtol=dtol, atol=0.0)
    assert np.array_equal(np.array(d["k_vals"]), kv)
    # a projected field is divergence free to rounding
    k, _, inv_ksq = N.wavenumbers(*shape, lx)
    uk = _to_dev(plan, N.projection(y, k, inv_ksq), cdt)
    d = ns.diagnostics(uk, num_bins=0)
    assert d["divergence_l2"] <= (1e-12 if precision == "float64" else 1e-5) * np.sqrt(2.0 * d["enstrophy"])


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_ns_write_diagnostics_files(tmp_path, precision):
    """The example's files: per rank (rx, ry) of in_topology (1, px, py, 1) the
    local block of each velocity / vorticity component in C order, and the
    spectrum under rank 0's coordinates, named label_rxNNN_ryNNN_NNNNNNNNNN.dat."""
    import torch
    shape, tin, tout, lx = (24, 20, 18), (1, 3, 2, 1), (1, 1, 3, 2), 2.0
    plan, cdt = _setup(shape, tin, tout, precision)
    ns = dfft.NavierStokes(plan, nu=0.01, dt=0.01, lx=lx)
    uk = torch.empty(plan.buffer_elements("out"), dtype=cdt, device="cuda")
    ns.init_taylor_green(uk)
    d = ns.write_diagnostics(uk, tmp_path, 7, num_bins=50)
    y = _to_host(plan, uk)
    vel = np.fft.irfftn(y, s=shape, axes=(1, 2, 3))
    vor = N.vorticity(y, lx, shape)
    rdt = np.float64 if precision == "float64" else np.float32
    tol = 1e-12 if precision == "float64" else 1e-5
    names = set()
    for r in range(plan.nprocs):
        ext, st = plan.local_extents(r, "in")
        rx, ry = r // 2, r % 2  # rank_to_coord((px, py), r), LayoutRight
        assert (st[1], st[2]) == (sum(plan.local_extents(q * 2, "in")[0][1] for q in range(rx)),
                                  sum(plan.local_extents(q, "in")[0][2] for q in range(ry)))
        for field, labels in ((vel, ("u", "v", "w")), (vor, ("vor_x", "vor_y", "vor_z"))):
            for c, lab in enumerate(labels):
                fn = tmp_path / f"{lab}_rx{rx:03d}_ry{ry:03d}_{7:010d}.dat"
                names.add(fn.name)
                got = np.fromfile(fn, dtype=rdt).reshape(ext[1:])
                ref = field[c][st[1]:st[1] + ext[1], st[2]:st[2] + ext[2], st[3]:st[3] + ext[3]]
                assert np.max(np.abs(got - ref)) <= tol * max(1.0, np.max(np.abs(field[c])))
    spec, kv = N.spectrum(y, lx, shape, 50)
    assert np.allclose(np.fromfile(tmp_path / f"E_spec_rx000_ry000_{7:010d}.dat"), spec, rtol=1e-12, atol=0.0)
    assert np.array_equal(np.fromfile(tmp_path / f"k_vals_rx000_ry000_{7:010d}.dat"), kv)
    names |= {f"E_spec_rx000_ry000_{7:010d}.dat", f"k_vals_rx000_ry000_{7:010d}.dat"}
    assert {p.name for p in tmp_path.iterdir()} == names
    assert abs(d["energy"] / N.energy(y, lx, shape) - 1.0) <= 1e-12
    assert abs(d["enstrophy"] / (3.0 * d["energy"]) - 1.0) <= tol


@pytest.mark.parametrize("n,tin,tout", [
    (64, (1, 2, 2, 1), (1, 1, 2, 2)),   # the example's decomposition, px = py = 2
    (96, (1, 4, 1, 1), (1, 1, 4, 1)),   # its slab form (py = 1)
    (96, (1, 2, 3, 1), (1, 1, 2, 3)),
])
def test_ns_at_the_reference_decomposition(n, tin, tout):
    """The solver on the example's own decomposition (1, px, py, 1) ->
    (1, 1, px, py) at cfg3 grid sizes, FP64, against the oracle: one
    right-hand side and one RK4 step of a random divergence-free field."""
    import torch
    shape, lx, nu, dt = (n, n, n), 2.0, 1.0 / 1600.0, 1e-3
    plan, cdt = _setup(shape, tin, tout, "float64")
    ns = dfft.NavierStokes(plan, nu=nu, dt=dt, lx=lx)
    y = _random_spectrum(shape, 12, lx) / n ** 1.5
    uk = _to_dev(plan, y, cdt)
    dukdt = torch.empty_like(uk)
    ns.rhs(uk, dukdt)
    _, ref_r = N.rhs(y, nu, lx, shape)
    assert _rel(_to_host(plan, dukdt), ref_r) <= 1e-12
    uk = _to_dev(plan, y, cdt)
    ns.step(uk)
    assert _rel(_to_host(plan, uk), N.rk4_step(y, nu, dt, lx, shape)) <= 1e-12
