"""ORACLE / TEST INFRASTRUCTURE: ctypes front end of liboracle.so and oracle/_ref."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .cf import cf_poles_residues

HERE = os.path.dirname(os.path.abspath(__file__))
SOLVERS = {"radau2a": 0, "exprb43": 1, "exp4": 2, "rkc": 3}
STAT_NAMES = ["steps", "accept", "reject", "jac", "decomp", "newton", "rhs", "errsolve",
              "krylov", "arnoldi"]
NSTATS = 16
NRA = 10
NMAX = 64

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class _Mech(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n", ctypes.c_int), ("n_species", ctypes.c_int),
                ("n_reactions", ctypes.c_int), ("mw", _dp), ("cp", _dp), ("h_form", _dp),
                ("s_ref", _dp), ("log_a", _dp), ("beta", _dp), ("ta", _dp), ("reac", _ip),
                ("prod", _ip), ("jac_fd", ctypes.c_int), ("fd_atol", ctypes.c_double),
                ("fd_rtol", ctypes.c_double)]


class _Config(ctypes.Structure):
    _fields_ = [("atol", ctypes.c_double), ("rtol", ctypes.c_double),
                ("poles_re", ctypes.c_double * NRA), ("poles_im", ctypes.c_double * NRA),
                ("res_re", ctypes.c_double * NRA), ("res_im", ctypes.c_double * NRA),
                ("max_steps", ctypes.c_int), ("stage_extrap", ctypes.c_int)]


_POLES = None


def cf_poles(atol: float = 1e-10):
    """Poles and residues of the (10,10) CF approximant (numpy restatement of cf.c)."""
    global _POLES
    if _POLES is None or _POLES[0] != atol:
        _POLES = (atol, cf_poles_residues(NRA, atol))
    return _POLES[1]


def _lib_path():
    return os.path.join(HERE, "_build", "liboracle.so")


def oracle_available() -> bool:
    return os.path.exists(_lib_path())


def reference_available(solver: str = "radau2a", n: int = 2) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libref_{solver}_n{n}.so"))


def _mech_struct(mech, keep, fd=None):
    """fd: (atol, rtol) for a finite-difference Jacobian (generic/fd_jacob.c), else None."""
    from accelerint_b200.mechanism import MECH_VAN_DER_POL
    m = _Mech()
    m.n = mech.n_state
    if fd is not None:
        m.jac_fd, m.fd_atol, m.fd_rtol = 1, fd[0], fd[1]
    if mech.kind == MECH_VAN_DER_POL:
        m.kind = 0
        return m
    m.kind = 1
    m.n_species = mech.n_species
    m.n_reactions = mech.n_reactions
    for name in ("mw", "cp", "h_form", "s_ref", "log_a", "beta", "ta"):
        a = np.ascontiguousarray(getattr(mech, name), dtype=np.float64)
        keep.append(a)
        setattr(m, name, a.ctypes.data_as(_dp))
    for name in ("reac", "prod"):
        a = np.ascontiguousarray(getattr(mech, name), dtype=np.int32).reshape(-1)
        keep.append(a)
        setattr(m, name, a.ctypes.data_as(_ip))
    return m


def global_steps(t0: float, t_end: float, dt: float):
    """The reference CLI loop (generic/solver_main.c:196-209): t_next = min(t_end, (k+1) dt)."""
    eps = np.finfo(float).eps
    t, k, out = t0, 0, []
    t_next = min(t_end, t0 + dt)
    while t + eps < t_end:
        k += 1
        out.append((t, t_next))
        t = t_next
        t_next = min(t_end, t0 + (k + 1) * dt)
    return out


class Oracle:
    """The plain-C restatement; integrates a column-major batch y[N, num] in place (copy returned)."""

    def __init__(self):
        self.lib = ctypes.CDLL(_lib_path())
        f = self.lib.or_integrate_batch
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, ctypes.POINTER(_Config), ctypes.POINTER(_Mech), ctypes.c_int,
                      ctypes.c_double, ctypes.c_double, _dp, _dp, _ip, _dp, ctypes.c_int]
        self.lib.or_dydt.argtypes = [ctypes.POINTER(_Mech), ctypes.c_double, ctypes.c_double, _dp, _dp]
        self.lib.or_jacob.argtypes = [ctypes.POINTER(_Mech), ctypes.c_double, ctypes.c_double, _dp, _dp]
        self.lib.or_phi_ac.argtypes = [ctypes.POINTER(_Config), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       _dp, ctypes.c_double, _dp]
        self.lib.or_phi_ac.restype = ctypes.c_int
        self.lib.or_hessenberg_lu.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, _ip]
        self.lib.or_hessenberg_lu.restype = ctypes.c_int
        self.lib.or_complex_inverse_hessenberg.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, _ip]
        self.lib.or_complex_inverse_hessenberg.restype = ctypes.c_int

    def config(self, atol=1e-10, rtol=1e-6, poles=None, max_steps=0, stage_extrapolation=0):
        c = _Config()
        c.atol, c.rtol = atol, rtol
        c.max_steps = max_steps
        c.stage_extrap = stage_extrapolation
        p, r = poles if poles is not None else cf_poles(1e-10)
        for i in range(NRA):
            c.poles_re[i], c.poles_im[i] = p[i].real, p[i].imag
            c.res_re[i], c.res_im[i] = r[i].real, r[i].imag
        return c

    def integrate(self, solver, mech, y, var, t0, t1, atol=1e-10, rtol=1e-6, nthreads=0, poles=None,
                  fd_jacobian=False, max_steps=0, stage_extrapolation=0):
        """One global step [t0, t1] for every system.  Returns (y_new, codes, stats[num, NSTATS]).
        max_steps: Radau step limit (0: the reference's 200000).  stage_extrapolation: Radau
        starting values, 0 the reference's, 1 the collocation polynomial at all three nodes."""
        keep = []
        m = _mech_struct(mech, keep, (atol, rtol) if fd_jacobian else None)
        c = self.config(atol, rtol, poles, max_steps, stage_extrapolation)
        y = np.array(y, dtype=np.float64, order="C", copy=True)
        num = y.shape[1]
        var = np.ascontiguousarray(var, dtype=np.float64)
        codes = np.zeros(num, dtype=np.int32)
        stats = np.zeros((num, NSTATS))
        self.lib.or_integrate_batch(SOLVERS[solver], ctypes.byref(c), ctypes.byref(m), num, t0, t1,
                                    var.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                    codes.ctypes.data_as(_ip), stats.ctypes.data_as(_dp), nthreads)
        return y, codes, stats

    def run(self, solver, mech, y, var, t0, t_end, dt, **kw):
        """The CLI loop over global steps; stats accumulate over steps."""
        stats = None
        codes = None
        for (a, b) in global_steps(t0, t_end, dt):
            y, c, s = self.integrate(solver, mech, y, var, a, b, **kw)
            stats = s if stats is None else stats + s
            codes = c if codes is None else np.maximum(codes, c)
        return y, codes, stats

    def dydt(self, mech, y, var, t=0.0):
        keep = []
        m = _mech_struct(mech, keep)
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros_like(y)
        self.lib.or_dydt(ctypes.byref(m), t, var, y.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        return out

    def jacob(self, mech, y, var, t=0.0, fd=None):
        """Column-major Jacobian returned as an [N, N] array J[i, j] = d f_i / d y_j
        (fd = (atol, rtol): by finite differences, generic/fd_jacob.c)."""
        keep = []
        m = _mech_struct(mech, keep, fd)
        y = np.ascontiguousarray(y, dtype=np.float64)
        n = y.shape[0]
        out = np.zeros(n * n)
        self.lib.or_jacob(ctypes.byref(m), t, var, y.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        return out.reshape(n, n, order="F")

    def phi(self, order, H, c, poles=None):
        """phi_order(c H) of an m x m matrix by the rational approximant (phiAHessenberg.c)."""
        m = H.shape[0]
        A = np.asfortranarray(H, dtype=np.float64).reshape(-1, order="F").copy()
        out = np.zeros(m * m)
        cfg = self.config(poles=poles)
        info = self.lib.or_phi_ac(ctypes.byref(cfg), order, m, m, A.ctypes.data_as(_dp), c,
                                  out.ctypes.data_as(_dp))
        return info, out.reshape(m, m, order="F")

    def hessenberg_lu(self, A):
        m = A.shape[0]
        a = np.asfortranarray(A, dtype=np.complex128).reshape(-1, order="F").copy()
        piv = np.zeros(m, dtype=np.int32)
        info = self.lib.or_hessenberg_lu(m, m, a.ctypes.data, piv.ctypes.data_as(_ip))
        return info, a.reshape(m, m, order="F"), piv

    def inverse_hessenberg(self, A):
        m = A.shape[0]
        a = np.asfortranarray(A, dtype=np.complex128).reshape(-1, order="F").copy()
        piv = np.zeros(m, dtype=np.int32)
        info = self.lib.or_complex_inverse_hessenberg(m, m, a.ctypes.data, piv.ctypes.data_as(_ip))
        return info, a.reshape(m, m, order="F")


class Reference:
    """The reference's own CPU integrator compiled for one (solver, state length)."""

    def __init__(self, solver: str, n: int):
        self.solver, self.n = solver, n
        self.lib = ctypes.CDLL(os.path.join(HERE, "_ref", f"libref_{solver}_n{n}.so"))
        self.lib.ref_integrate_batch.restype = ctypes.c_int
        self.lib.ref_integrate_batch.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp,
                                                 _ip, ctypes.c_int]
        self.lib.ref_int_driver.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp,
                                            ctypes.c_int]
        self.lib.ref_poles.argtypes = [_dp, _dp, _dp, _dp]
        if solver == "radau2a":
            self.lib.ref_fd_eval_jacob.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp]
        self._keep = []
        # the exponential methods' CF poles and residues (rational_approximant.c:23-44)
        self.lib.ref_init()

    def fd_jacob(self, y, pres, t=0.0):
        """The reference's generic/fd_jacob.c (ATOL 1e-10, RTOL 1e-6) at one state: [N, N]."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(self.n * self.n)
        self.lib.ref_fd_eval_jacob(t, pres, y.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
        return out.reshape(self.n, self.n, order="F")

    def set_mechanism(self, mech):
        if self.n == 2:
            return
        keep = []
        arrs = [np.ascontiguousarray(getattr(mech, k), dtype=np.float64)
                for k in ("mw", "cp", "h_form", "s_ref")]
        ints = [np.ascontiguousarray(getattr(mech, k), dtype=np.int32).reshape(-1) for k in ("reac", "prod")]
        rates = [np.ascontiguousarray(getattr(mech, k), dtype=np.float64) for k in ("log_a", "beta", "ta")]
        keep += arrs + ints + rates
        self._keep = keep
        f = self.lib.refshim_set_mass_action
        f.argtypes = [ctypes.c_int, ctypes.c_int] + [_dp] * 4 + [_ip] * 2 + [_dp] * 3
        f(mech.n_species, mech.n_reactions, *[a.ctypes.data_as(_dp) for a in arrs],
          *[a.ctypes.data_as(_ip) for a in ints], *[a.ctypes.data_as(_dp) for a in rates])

    def poles(self):
        a = [np.zeros(NRA) for _ in range(4)]
        k = self.lib.ref_poles(*[x.ctypes.data_as(_dp) for x in a])
        if k == 0:
            return None
        return a[0] + 1j * a[1], a[2] + 1j * a[3]

    def integrate(self, y, var, t0, t1, nthreads=0):
        y = np.array(y, dtype=np.float64, order="C", copy=True)
        num = y.shape[1]
        var = np.ascontiguousarray(var, dtype=np.float64)
        codes = np.zeros(num, dtype=np.int32)
        self.lib.ref_integrate_batch(num, t0, t1, var.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                     codes.ctypes.data_as(_ip), nthreads)
        return y, codes

    def int_driver(self, y, var, t0, t1, nthreads=0):
        """The reference's stock intDriver (exits the process on a failed system)."""
        var = np.ascontiguousarray(var, dtype=np.float64)
        self.lib.ref_int_driver(y.shape[1], t0, t1, var.ctypes.data_as(_dp), y.ctypes.data_as(_dp), nthreads)
        return y

    def run(self, y, var, t0, t_end, dt, nthreads=0):
        codes = None
        for (a, b) in global_steps(t0, t_end, dt):
            y, c = self.integrate(y, var, a, b, nthreads)
            codes = c if codes is None else np.maximum(codes, c)
        return y, codes


def reference_gpu_available(n: int, q3_fix: bool = False) -> bool:
    tag = "_q3fix" if q3_fix else ""
    return os.path.exists(os.path.join(HERE, "_ref", f"libref_gpu_radau2a{tag}_n{n}.so"))


class ReferenceGPU:
    """The reference's own GPU Radau IIA (radau2a/radau2a.cu under generic/solver_generic.cu's
    intDriver, one thread per system), compiled unmodified by oracle/build.py with the
    mechanism callbacks for state length n (2: the reference's van der Pol example; 54: the
    synthetic mass-action mechanism, oracle/refshim/ma_gpu) and the host entry
    oracle/refshim/ref_gpu_entry.cu.  q3_fix: the build whose error estimate solves with
    the factored E1 (oracle/build.py: Q3_FIX) instead of the raw Jacobian.  Needs a GPU."""

    def __init__(self, n: int, q3_fix: bool = False):
        self.n = n
        tag = "_q3fix" if q3_fix else ""
        self.lib = ctypes.CDLL(os.path.join(HERE, "_ref", f"libref_gpu_radau2a{tag}_n{n}.so"))
        self.lib.refgpu_run.restype = ctypes.c_int
        self.lib.refgpu_run.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp,
                                        _ip, _dp]
        self._keep = []

    def set_mechanism(self, mech):
        if self.n == 2:
            return
        arrs = [np.ascontiguousarray(getattr(mech, k), dtype=np.float64) for k in ("mw", "cp", "h_form", "s_ref")]
        ints = [np.ascontiguousarray(getattr(mech, k), dtype=np.int32).reshape(-1) for k in ("reac", "prod")]
        rates = [np.ascontiguousarray(getattr(mech, k), dtype=np.float64) for k in ("log_a", "beta", "ta")]
        self._keep = arrs + ints + rates
        f = self.lib.refgpu_set_mass_action
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, ctypes.c_int] + [_dp] * 4 + [_ip] * 2 + [_dp] * 3
        rc = f(mech.n_species, mech.n_reactions, *[a.ctypes.data_as(_dp) for a in arrs],
               *[a.ctypes.data_as(_ip) for a in ints], *[a.ctypes.data_as(_dp) for a in rates])
        if rc != 0:
            raise RuntimeError(f"refgpu_set_mass_action failed ({rc})")

    def run(self, y, var, t0, t_end, dt):
        """Global steps t0 -> t_end of dt; returns (y_out, codes (max over steps), summed kernel ms)."""
        y = np.array(y, dtype=np.float64, order="C", copy=True)
        num = y.shape[1]
        var = np.ascontiguousarray(var, dtype=np.float64)
        codes = np.zeros(num, dtype=np.int32)
        ms = ctypes.c_double(0.0)
        rc = self.lib.refgpu_run(num, t0, t_end, dt, y.ctypes.data_as(_dp), var.ctypes.data_as(_dp),
                                 codes.ctypes.data_as(_ip), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"refgpu_run failed ({rc})")
        return y, codes, ms.value
