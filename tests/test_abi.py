"""The C-ABI library loads and exports every entry point its headers declare (no GPU needed).

include/dugma.h declares the extern "C" surface; include/dugma_mex.hpp declares
the reference's four C++ entry points (init, cpd x2, fr_m) with their exact
signatures, which must be exported under their C++ mangled names so that the
reference's MEX gateways (init.cpp:9-19, update_sig.cpp:7, compi.cpp:7,
fr_m.cpp:7) link against the library unchanged."""
import os
import re
import subprocess

from dugma_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _exported():
    path = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_c_symbols_exported_and_bound():
    hdr = open(os.path.join(ROOT, "include", "dugma.h")).read()
    declared = set(re.findall(r"^\s*(?:int|const char\*)\s+(dugma_\w+)\s*\(", hdr, re.M))
    assert len(declared) >= 20
    syms = _exported()
    missing = declared - syms
    assert not missing, missing
    # every declared function has a ctypes binding with an argtypes list
    assert declared <= set(_lib.EXPORTS)
    L = _lib.load()
    for name in declared:
        assert getattr(L, name).argtypes is not None


def test_reference_cpp_signatures_exported():
    syms = _exported()
    # Itanium mangling of the reference's four functions
    want = {
        "_Z4initPdS_S_S_S_iiiPPf",          # void init(double*, double*, double*, double*, double*, int, int, int, float**)
        "_Z3cpdPPfPdS1_S1_S1_S1_S_",        # void cpd(float**, double*, double*, double*, double*, double*, float*)
        "_Z3cpdPPfPdS1_S1_S1_S1_S1_S1_",    # void cpd(float**, double* x7)
        "_Z4fr_mPPf",                       # void fr_m(float**)
    }
    assert want <= syms, want - syms


def test_version_string():
    assert b"sm_100a" in _lib.load().dugma_version()


def test_errors_are_returned_not_fatal():
    """Bad arguments come back as status codes with a message (the reference exit()s)."""
    import ctypes
    L = _lib.load()
    ptrs = _lib.PtrArray()
    rc = L.dugma_fr_m(ptrs)
    assert rc == _lib.ERR_ARG
    assert b"context" in L.dugma_last_error()
    coef = ctypes.c_double(5)
    rc = L.dugma_init(None, None, None, None, ctypes.byref(coef), 10, 10, 3, ptrs)
    assert rc == _lib.ERR_ARG and coef.value == 0


def test_argument_errors_before_any_device_work():
    """Entry points check their arguments before touching the device: each bad call returns
    the argument status and a message (no GPU needed)."""
    import ctypes

    import numpy as np
    L = _lib.load()
    pts = np.zeros((8, 3))
    cov = np.zeros((8, 3, 3))
    dp = _lib.dp
    for k, n, D in [(0, 8, 3), (16, 8, 3), (8, 8, 3), (3, 1, 3), (3, 8, 4)]:
        rc = L.dugma_knn_covariance(pts.ctypes.data_as(dp), n, D, k, 1e-6, 1e-2, cov.ctypes.data_as(dp))
        assert rc == _lib.ERR_ARG, (k, n, D)
        assert b"knn_covariance" in L.dugma_last_error()
    rc = L.dugma_knn_covariance(pts.ctypes.data_as(dp), 8, 3, 3, 0.0, 1e-2, cov.ctypes.data_as(dp))
    assert rc == _lib.ERR_ARG   # lo must be positive
    A = np.zeros(640)
    out = np.zeros(9)
    assert L.dugma_minimise_surrogate(4, A.ctypes.data_as(dp), out.ctypes.data_as(dp),
                                      out.ctypes.data_as(dp), None, None) == _lib.ERR_ARG
    buf = (ctypes.c_int * 64)()
    assert L.dugma_shapes(7, buf, 16) < 0
    eye = np.eye(3).reshape(-1)
    R_out = np.zeros(9)
    t_out = np.zeros(3)
    rc = L.dugma_register(pts.ctypes.data_as(dp), cov.ctypes.data_as(dp), pts.ctypes.data_as(dp),
                          cov.ctypes.data_as(dp), 8, 8, 3, eye.ctypes.data_as(dp), t_out.ctypes.data_as(dp),
                          10, 1e-5, 1e-5, 1e-5, 99, R_out.ctypes.data_as(dp), t_out.ctypes.data_as(dp), None)
    assert rc == _lib.ERR_ARG and b"mode" in L.dugma_last_error()


def build_mex_harness(out_dir):
    """Compile tests/abi/mex_harness.cpp against include/dugma_mex.hpp and link it to the
    library: the reference's C++ signatures resolve against the exported symbols."""
    lib = build.build()
    exe = os.path.join(str(out_dir), "mex_harness")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi", "mex_harness.cpp"), "-o", exe,
                    "-L", os.path.dirname(lib), "-ldugma_b200", "-Wl,-rpath," + os.path.dirname(lib)],
                   check=True, capture_output=True)
    return exe


def test_reference_gateway_calls_link(tmp_path):
    exe = build_mex_harness(tmp_path)
    assert os.access(exe, os.X_OK)


def test_default_kernel_shapes_are_compiled():
    """The shapes a new context uses by default (adjoint, energy, nearest neighbours, CONV
    adjoint, CONV energy) are among the compiled ones, and every listed shape is unique (the
    host tables only: no GPU needed)."""
    from dugma_b200 import api
    defaults = {0: (4, 64, 64, 2), 1: (4, 128, 32, 2), 2: (4, 128, 64, 1), 3: (2, 64, 32, 2), 4: (1, 128, 32, 2)}
    for what, shape in defaults.items():
        listed = api.shapes(what)
        assert shape in listed, (what, shape, listed)
        assert len(set(listed)) == len(listed), what
