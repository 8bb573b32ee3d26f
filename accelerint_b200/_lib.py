"""ctypes binding of libaccelerint_b200.so (include/accelerint_b200.h)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .mechanism import MECH_VAN_DER_POL, MassActionDesc

HERE = os.path.dirname(os.path.abspath(__file__))

ACCELERINT_OK = 0
ACCELERINT_ERR_ARGUMENT = -1
ACCELERINT_ERR_CUDA = -2
ACCELERINT_ERR_STATE = -3
ACCELERINT_ERR_UNSUPPORTED = -4
ACCELERINT_ERR_SYSTEMS = -5
ACCELERINT_EC_NONFINITE = 5   # per-system code: success reported but the final state is not finite
SOLVERS = {"radau2a": 0, "exprb43": 1, "exp4": 2, "rkc": 3}
LU_FP64, LU_FP32, LU_FP32_ALL = 0, 1, 2
NSTATS = 10
STAT_NAMES = ["steps", "accept", "reject", "jac", "decomp", "newton", "rhs", "aux", "krylov", "arnoldi"]

# Every symbol include/accelerint_b200.h declares.
EXPORTED_SYMBOLS = [
    "accelerInt_initialize", "accelerInt_integrate", "accelerInt_cleanup",
    "accelerInt_set_solver", "accelerInt_set_mechanism_van_der_pol",
    "accelerInt_set_mechanism_mass_action", "accelerInt_set_tolerances",
    "accelerInt_set_lu_precision", "accelerInt_integrate_status", "accelerInt_integrate_device",
    "accelerInt_last_status", "accelerInt_get_codes", "accelerInt_get_poles", "accelerInt_version",
    "accelerInt_measure_fma_peak", "accelerInt_integrate_device_noalloc", "accelerInt_kernel_launches",
    "accelerInt_mlp_sizes", "accelerInt_mlp_forward", "accelerInt_mlp_loss_grad", "accelerInt_mlp_adam_step",
    "accelerInt_set_learned", "accelerInt_set_step_recording", "accelerInt_set_graph_launch",
    "accelerInt_set_launch_config", "accelerInt_autotune", "accelerInt_set_persistent",
    "accelerInt_set_queue_order", "accelerInt_set_cost_model", "accelerInt_set_learned_growth_floor",
    "accelerInt_set_jacobian", "accelerInt_radau_decomp", "accelerInt_set_mapping", "accelerInt_get_mapping",
    "accelerInt_set_stage_extrapolation",
]

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_LIB = None


def library_path() -> str:
    return os.path.join(HERE, "libaccelerint_b200.so")


def load_library():
    """Load the in-tree C-ABI library; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m accelerint_b200.build`")
    lib = ctypes.CDLL(path)
    lib.accelerInt_initialize.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.accelerInt_initialize.restype = None
    lib.accelerInt_integrate.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         _dp, _dp]
    lib.accelerInt_integrate.restype = None
    lib.accelerInt_cleanup.argtypes = []
    lib.accelerInt_cleanup.restype = None
    lib.accelerInt_set_solver.argtypes = [ctypes.c_int]
    vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    lib.accelerInt_mlp_sizes.argtypes = [vp, vp, vp, vp]
    lib.accelerInt_mlp_forward.argtypes = [vp, vp, vp, i, vp, vp]
    lib.accelerInt_mlp_loss_grad.argtypes = [vp, vp, vp, vp, i, vp, vp, vp]
    lib.accelerInt_mlp_adam_step.argtypes = [vp, vp, vp, vp, i, f, f, f, f, vp]
    lib.accelerInt_set_learned.argtypes = [vp, vp, i]
    lib.accelerInt_set_step_recording.argtypes = [vp, vp, i]
    lib.accelerInt_set_graph_launch.argtypes = [i]
    lib.accelerInt_set_persistent.argtypes = [i]
    lib.accelerInt_set_jacobian.argtypes = [i]
    lib.accelerInt_set_queue_order.argtypes = [i]
    lib.accelerInt_set_cost_model.argtypes = [vp, vp]
    lib.accelerInt_set_learned_growth_floor.argtypes = [ctypes.c_double]
    lib.accelerInt_set_launch_config.argtypes = [i, i]
    lib.accelerInt_set_mapping.argtypes = [i, i]
    lib.accelerInt_set_stage_extrapolation.argtypes = [i]
    lib.accelerInt_get_mapping.argtypes = [vp, vp, vp]
    lib.accelerInt_autotune.argtypes = [i, ctypes.c_double, ctypes.c_double, ctypes.c_double, vp, vp, i, vp, vp, vp]
    lib.accelerInt_radau_decomp.argtypes = [i, i, i, vp, vp, vp, vp, vp, vp, vp]
    lib.accelerInt_kernel_launches.argtypes = []
    lib.accelerInt_kernel_launches.restype = ctypes.c_longlong
    lib.accelerInt_set_mechanism_van_der_pol.argtypes = []
    lib.accelerInt_set_mechanism_mass_action.argtypes = [ctypes.POINTER(MassActionDesc)]
    lib.accelerInt_set_tolerances.argtypes = [ctypes.c_double, ctypes.c_double]
    lib.accelerInt_set_lu_precision.argtypes = [ctypes.c_int]
    lib.accelerInt_integrate_status.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, _dp, _dp]
    lib.accelerInt_integrate_device.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.accelerInt_integrate_device_noalloc.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                        ctypes.c_void_p, ctypes.c_void_p]
    lib.accelerInt_last_status.argtypes = []
    lib.accelerInt_get_codes.argtypes = [_ip, ctypes.c_int]
    lib.accelerInt_get_poles.argtypes = [_dp, _dp, _dp, _dp]
    lib.accelerInt_version.restype = ctypes.c_char_p
    _LIB = lib
    return lib


class Integrator:
    """One configured integrator instance over the process-wide C-ABI state.

    Mirrors the reference's library use: configure (solver, mechanism,
    tolerances) -> accelerInt_initialize(NUM, device) -> accelerInt_integrate
    -> accelerInt_cleanup.
    """

    def __init__(self, num: int, mechanism, solver: str = "radau2a", device: int = 0,
                 atol: float = 1e-10, rtol: float = 1e-6, lu: int = LU_FP64, stage_extrapolation: int = 0):
        self.lib = load_library()
        self.mechanism = mechanism
        self.n = mechanism.n_state
        self._check(self.lib.accelerInt_set_solver(SOLVERS[solver]))
        self._check(self.lib.accelerInt_set_tolerances(atol, rtol))
        self._check(self.lib.accelerInt_set_lu_precision(lu))
        self._check(self.lib.accelerInt_set_stage_extrapolation(int(stage_extrapolation)))
        if mechanism.kind == MECH_VAN_DER_POL:
            self._check(self.lib.accelerInt_set_mechanism_van_der_pol())
        else:
            self._desc = mechanism.as_struct()
            self._check(self.lib.accelerInt_set_mechanism_mass_action(ctypes.byref(self._desc)))
        self.lib.accelerInt_initialize(int(num), int(device))
        self._check(self.lib.accelerInt_last_status())
        self.num = num

    @staticmethod
    def _check(rc):
        if rc not in (ACCELERINT_OK, ACCELERINT_ERR_SYSTEMS):
            raise RuntimeError(f"accelerint_b200 call failed with status {rc}")
        return rc

    def integrate(self, t_start, t_end, stepsize, y, var):
        """Host-buffer path (accelerInt_integrate_status).  y[N, NUM] is not modified; returns
        (y_out, codes, status)."""
        y = np.array(y, dtype=np.float64, order="C", copy=True)
        var = np.ascontiguousarray(var, dtype=np.float64)
        num = y.shape[1]
        rc = self.lib.accelerInt_integrate_status(num, t_start, t_end, stepsize, y.ctypes.data_as(_dp),
                                                  var.ctypes.data_as(_dp))
        self._check(rc)
        codes = np.zeros(num, dtype=np.int32)
        self._check(self.lib.accelerInt_get_codes(codes.ctypes.data_as(_ip), num))
        return y, codes, rc

    def integrate_device(self, t_start, t_end, stepsize, y_dev, var_dev, codes_dev=None, stats_dev=None,
                         stream=None):
        """Device-buffer path on torch CUDA tensors (y_dev [N, NUM] float64, in place)."""
        num = y_dev.shape[1]
        s = stream.cuda_stream if stream is not None else None
        return self._check(self.lib.accelerInt_integrate_device(
            num, t_start, t_end, stepsize, y_dev.data_ptr(), var_dev.data_ptr(),
            codes_dev.data_ptr() if codes_dev is not None else None,
            stats_dev.data_ptr() if stats_dev is not None else None, s))

    def autotune(self, t_start, t_end, stepsize, y_dev, var_dev, sample: int):
        """Pick the launch mapping by timing candidates on a copy of the first `sample` systems.
        Returns (occupancy cap, queue order, thread-per-system block size, best ms)."""
        occ, blk, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.accelerInt_autotune(y_dev.shape[1], t_start, t_end, stepsize, y_dev.data_ptr(),
                                                 var_dev.data_ptr(), int(sample), ctypes.byref(occ),
                                                 ctypes.byref(blk), ctypes.byref(ms)))
        return occ.value & 0xffff, occ.value >> 16, blk.value, ms.value

    def set_mapping(self, team_lanes: int = 0, grain: int = 1):
        """team_lanes 0: the default team; 16: two systems per warp (state length <= 16).
        grain: work-queue slots a team claims per atomic."""
        self._check(self.lib.accelerInt_set_mapping(int(team_lanes), int(grain)))

    def mapping(self):
        """(team_lanes, grain, resident blocks per SM of the last persistent launch)."""
        tl, gr, oc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.accelerInt_get_mapping(ctypes.byref(tl), ctypes.byref(gr), ctypes.byref(oc)))
        return tl.value, gr.value, oc.value

    def set_stage_extrapolation(self, mode: int):
        """Radau starting values after an accepted step: 0 the reference's (default), 1 the
        collocation polynomial at all three nodes."""
        self._check(self.lib.accelerInt_set_stage_extrapolation(int(mode)))

    def set_queue_order(self, mode: int):
        self._check(self.lib.accelerInt_set_queue_order(int(mode)))

    def set_jacobian(self, finite_difference: bool):
        self._check(self.lib.accelerInt_set_jacobian(1 if finite_difference else 0))

    def set_persistent(self, enable: bool = True):
        self._check(self.lib.accelerInt_set_persistent(1 if enable else 0))

    def set_graph_launch(self, enable: bool = True):
        self._check(self.lib.accelerInt_set_graph_launch(1 if enable else 0))

    def kernel_launches(self) -> int:
        """Kernels the library has launched in this process (all entry points)."""
        return int(self.lib.accelerInt_kernel_launches())

    def poles(self):
        a = [np.zeros(10) for _ in range(4)]
        self._check(self.lib.accelerInt_get_poles(*[x.ctypes.data_as(_dp) for x in a]))
        return a[0] + 1j * a[1], a[2] + 1j * a[3]

    def close(self):
        self.lib.accelerInt_cleanup()
