"""Pseudo-spectral Navier-Stokes step of the reference's batched example
(``examples/navier-stokes-MPI-batched/main.cpp``) on a distributed R2C plan.

The plan transforms the velocity field, a LayoutRight 4D view (3, nx, ny, nz),
over axes (1, 2, 3); ``uk`` is the plan's output (spectral) buffer.  The
reference builds the same plan with in_topology (1, px, py, 1) and
out_topology (1, 1, px, py) (main.cpp:96-102).
"""
import ctypes

from ._lib import NS_MAX_BINS, NsDiag, lib
from .plan import Graph, _check, _ptr


class NavierStokes:
    """``NavierStokes(plan, nu, dt, lx)``: nu = 1 / Re, dt the time step, the
    domain [0, lx pi)^3.  Methods mirror the example's NavierStokes / RK4th
    members: ``init_taylor_green`` (Variables constructor, main.cpp:322-363),
    ``rhs`` (main.cpp:536-586), ``step`` (solve, main.cpp:518-528),
    ``energy`` (diag_energy, main.cpp:746-766), ``velocity`` / ``vorticity``
    (diag_fields / compute_vorticity, main.cpp:677-724), ``diagnostics``
    (FP64 energy, enstrophy, divergence and the energy spectrum of
    diag_energy, main.cpp:741-794) and ``write_diagnostics`` (the example's
    binary files, main.cpp:705-818)."""

    def __init__(self, plan, nu=0.01, dt=0.01, lx=2.0):
        self._plan = plan  # the plan must outlive the state
        self._h = ctypes.c_void_p()
        _check(lib.dfft_ns_create(ctypes.byref(self._h), plan._h, float(nu), float(dt), float(lx)))

    @staticmethod
    def _stream(stream):
        return ctypes.c_void_p(int(stream)) if stream else None

    def init_taylor_green(self, uk, v0=1.0, stream=None):
        _check(lib.dfft_ns_init_taylor_green(self._h, _ptr(uk), float(v0), self._stream(stream)))

    def rhs(self, uk, dukdt, stream=None):
        _check(lib.dfft_ns_rhs(self._h, _ptr(uk), _ptr(dukdt), self._stream(stream)))

    def step(self, uk, stream=None):
        _check(lib.dfft_ns_step(self._h, _ptr(uk), self._stream(stream)))

    def energy(self, uk, stream=None):
        e = ctypes.c_double(0.0)
        _check(lib.dfft_ns_energy(self._h, _ptr(uk), ctypes.byref(e), self._stream(stream)))
        return e.value

    def rhs_adjoint(self, uk, lam, grad, stream=None):
        """grad = (d rhs / d uk)^T lam (real inner product of the half spectrum)."""
        _check(lib.dfft_ns_rhs_adjoint(self._h, _ptr(uk), _ptr(lam), _ptr(grad), self._stream(stream)))

    def step_adjoint(self, uk, lam, stream=None):
        """lam <- (d step / d uk)^T lam for one RK4 step from state uk."""
        _check(lib.dfft_ns_step_adjoint(self._h, _ptr(uk), _ptr(lam), self._stream(stream)))

    def velocity(self, uk, u, stream=None):
        _check(lib.dfft_ns_velocity(self._h, _ptr(uk), _ptr(u), self._stream(stream)))

    def vorticity(self, uk, vor, stream=None):
        _check(lib.dfft_ns_vorticity(self._h, _ptr(uk), _ptr(vor), self._stream(stream)))

    def diagnostics(self, uk, num_bins=50, stream=None):
        """dict(energy, enstrophy, divergence_l2, e_spec, k_vals); the sums are FP64."""
        if not 0 <= num_bins <= NS_MAX_BINS:
            raise ValueError(f"num_bins must be in [0, {NS_MAX_BINS}]")
        spec = (ctypes.c_double * max(num_bins, 1))()
        kv = (ctypes.c_double * max(num_bins, 1))()
        d = NsDiag()
        _check(lib.dfft_ns_diagnostics(self._h, _ptr(uk), int(num_bins), spec, kv, ctypes.byref(d),
                                       self._stream(stream)))
        return {"energy": d.energy, "enstrophy": d.enstrophy, "divergence_l2": d.divergence_l2,
                "e_spec": list(spec)[:num_bins], "k_vals": list(kv)[:num_bins]}

    def write_diagnostics(self, uk, out_dir, iteration, num_bins=50, stream=None):
        """The example's per-rank velocity / vorticity files and the spectrum files of one iteration."""
        d = NsDiag()
        _check(lib.dfft_ns_write_diagnostics(self._h, _ptr(uk), str(out_dir).encode(), int(iteration),
                                             int(num_bins), ctypes.byref(d), self._stream(stream)))
        return {"energy": d.energy, "enstrophy": d.enstrophy, "divergence_l2": d.divergence_l2}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.dfft_ns_destroy(h)
            self._h = None


def step_graph(states, uks, batched=True):
    """A library-owned CUDA graph of one RK4 step of every field (states[i]
    advances uks[i]); ``batched``: each transform of all fields batched into
    one launch per stage, else each field's step on one of up to four
    concurrent branches.  ``launch(stream)`` advances all fields by one step."""
    n = len(states)
    if len(uks) != n or n == 0:
        raise ValueError("one spectral buffer per state")
    st = (ctypes.c_void_p * n)(*[s._h.value for s in states])
    bufs = (ctypes.c_void_p * n)(*[_ptr(u).value for u in uks])
    h = ctypes.c_void_p()
    _check(lib.dfft_ns_graph_create(ctypes.byref(h), st, bufs, n, 1 if batched else 0))
    return Graph._from_handle(h, list(states) + [s._plan for s in states])
