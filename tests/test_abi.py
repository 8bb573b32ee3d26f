"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU needed)."""
import glob
import os
import re

import accelerint_b200 as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(accelerInt_\w+)\s*\(", src))
    return names


def _lib():
    if not os.path.exists(A.library_path()):
        from accelerint_b200.build import build
        build()
    return A.load_library()


def test_header_and_binding_agree():
    assert declared_symbols() == set(A.EXPORTED_SYMBOLS)


def test_library_exports_declared_symbols():
    lib = _lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.accelerInt_version()


def test_setters_validate_without_a_device():
    lib = _lib()
    assert lib.accelerInt_set_solver(99) == -1
    assert lib.accelerInt_set_tolerances(-1.0, 1e-6) == -1
    assert lib.accelerInt_set_lu_precision(7) == -1


def test_host_cf_poles_match_reference():
    """accelerInt_get_poles runs the library's own C++ CF solver on the host (no GPU):
    its poles and residues match the reference's cf() output stored with the fixtures
    (to the conditioning of the Hankel SVD and the polynomial roots), in the same
    conjugate-pair order."""
    import ctypes
    import numpy as np
    lib = _lib()
    lib.accelerInt_set_tolerances(1e-10, 1e-6)
    a = [np.zeros(10) for _ in range(4)]
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.accelerInt_get_poles(*[x.ctypes.data_as(dp) for x in a]) == 0
    p, r = a[0] + 1j * a[1], a[2] + 1j * a[3]
    g = np.load(os.path.join(ROOT, "tests", "golden", "vdp_exprb43.npz"))
    assert np.max(np.abs(p - g["poles"]) / np.abs(g["poles"])) < 1e-7
    assert np.max(np.abs(r - g["res"]) / np.abs(g["res"])) < 1e-6
    assert np.allclose(p[0::2], np.conj(p[1::2]), rtol=0, atol=0)


def test_kernel_launch_counter_is_exported():
    import ctypes
    lib = _lib()
    lib.accelerInt_kernel_launches.restype = ctypes.c_longlong
    assert lib.accelerInt_kernel_launches() >= 0


def test_extension_setters_validate_without_a_device():
    import ctypes
    lib = _lib()
    # queue order 3 needs a cost model; orders outside 0..3 are rejected
    lib.accelerInt_set_cost_model(None, None)
    assert lib.accelerInt_set_queue_order(3) == -3
    assert lib.accelerInt_set_queue_order(4) == -1
    assert lib.accelerInt_set_queue_order(0) == 0
    # growth floor bounds, Jacobian modes, launch configuration
    lib.accelerInt_set_learned_growth_floor.argtypes = [ctypes.c_double]
    assert lib.accelerInt_set_learned_growth_floor(1.0) == -1
    assert lib.accelerInt_set_learned_growth_floor(9.0) == -1
    assert lib.accelerInt_set_learned_growth_floor(2.0) == 0
    assert lib.accelerInt_set_jacobian(2) == -1
    assert lib.accelerInt_set_jacobian(0) == 0
    assert lib.accelerInt_set_launch_config(-1, 0) == -1
    assert lib.accelerInt_set_launch_config(0, 48) == -1
    # mapping: team lanes 0 or 16, queue grain 1..64
    assert lib.accelerInt_set_mapping(8, 1) == -1
    assert lib.accelerInt_set_mapping(0, 0) == -1
    assert lib.accelerInt_set_mapping(0, 65) == -1
    assert lib.accelerInt_set_mapping(16, 4) == 0
    tl, gr = ctypes.c_int(), ctypes.c_int()
    assert lib.accelerInt_get_mapping(ctypes.byref(tl), ctypes.byref(gr), None) == 0
    assert (tl.value, gr.value) == (16, 4)
    assert lib.accelerInt_set_mapping(0, 1) == 0
    # Radau starting values: 0 the reference's, 1 collocation
    assert lib.accelerInt_set_stage_extrapolation(2) == -1
    assert lib.accelerInt_set_stage_extrapolation(-1) == -1
    assert lib.accelerInt_set_stage_extrapolation(1) == 0
    assert lib.accelerInt_set_stage_extrapolation(0) == 0
    # learned proposals: unknown flags, missing buffers, not initialised
    assert lib.accelerInt_set_learned(None, None, 4) == -1
    assert lib.accelerInt_set_learned(None, None, 1) == -1
    assert lib.accelerInt_set_learned(None, None, 0) == 0
    assert lib.accelerInt_set_step_recording(ctypes.c_void_p(16), None, 10) == -1
    assert lib.accelerInt_set_step_recording(None, None, 0) == 0


def test_entry_points_refuse_before_initialize():
    import ctypes
    lib = _lib()
    lib.accelerInt_cleanup()
    dp = ctypes.POINTER(ctypes.c_double)
    import numpy as np
    y = np.zeros((2, 4))
    var = np.ones(4)
    assert lib.accelerInt_integrate_status(4, 0.0, 1.0, 0.1, y.ctypes.data_as(dp), var.ctypes.data_as(dp)) == -3
    vp = ctypes.c_void_p
    lib.accelerInt_integrate_device.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                vp, vp, vp, vp, vp]
    assert lib.accelerInt_integrate_device(4, 0.0, 1.0, 0.1, vp(16), vp(16), None, None, None) == -3
    lib.accelerInt_integrate_device_noalloc.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_double, vp, vp, vp, vp]
    assert lib.accelerInt_integrate_device_noalloc(4, 0.0, 1.0, 0.1, vp(16), vp(16), None, None) == -3
    lib.accelerInt_autotune.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, vp, vp,
                                        ctypes.c_int, vp, vp, vp]
    assert lib.accelerInt_autotune(4, 0.0, 1.0, 0.1, vp(16), vp(16), 4, None, None, None) == -3


def test_mlp_sizes_match_the_python_layout():
    import ctypes
    from accelerint_b200 import learned as L
    lib = _lib()
    a = [ctypes.c_int() for _ in range(4)]
    lib.accelerInt_mlp_sizes.argtypes = [ctypes.c_void_p] * 4
    assert lib.accelerInt_mlp_sizes(*[ctypes.byref(x) for x in a]) == 0
    assert [x.value for x in a] == [L.n_params(), 2 * L.D_IN + 2 * L.D_OUT, L.D_IN, L.D_OUT]
