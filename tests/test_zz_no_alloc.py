"""fin_construct_l_noalloc: ConstructL for callers that cannot allocate
device memory (their own allocator owns the device, or they run where
allocation is forbidden).  It keeps its scratch in a static device array, so
the caller passes device buffers it already owns.  This file is collected
last so a failure here never hides another test.

The checks:
* calls in a row on different inputs, each against the existing entry point
  fin_construct_l and against the oracle, at the 1e-12 relative L-infinity
  the ConstructL parity tests use; a later call must not see an earlier
  call's scratch contents.  The cases cover WENO-Z and WENO-JS with the
  global alpha, FD5 with the local (per-face) alpha, and JS with a WENO power
  other than 2 (the kernels' general-power instantiation);
* a repeated call changes the device's free memory by nothing (the first
  call on a device may load the library's module, which holds the array);
* with check != 0 a non-finite input is reported as FIN_ERR_NONFINITE;
* grids beyond the array's size are refused with FIN_ERR_SIZE."""
import ctypes as C

import numpy as np
import pytest

from conftest import interior, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import (FIN_ERR_NONFINITE, FIN_ERR_SIZE, FIN_OK, FIN_WENO_FD, FIN_WENO_JS, FIN_WENO_Z,
                              ghosted_shape)

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _lib():
    from finess_b200.solver import load_library
    lib = load_library()
    lib.fin_construct_l_noalloc.argtypes = [C.POINTER(type(P.riemann_params(n=8))), C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_int]
    lib.fin_construct_l_noalloc.restype = C.c_int
    return lib


def _call(lib, p, qd, Ld, check):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    return lib.fin_construct_l_noalloc(C.byref(p), C.c_void_p(qd.data_ptr()), C.c_void_p(Ld.data_ptr()),
                                       C.c_void_p(stream), check)


def _noalloc_construct_l(lib, p, q, check=0):
    import torch
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    Ld = torch.zeros(ghosted_shape(p), dtype=torch.float64, device="cuda")
    rc = _call(lib, p, qd, Ld, check)
    assert rc == FIN_OK, rc
    torch.cuda.synchronize()
    return Ld.cpu().numpy()


def _cases(oracle):
    rng = np.random.default_rng(123)
    cases = []
    p = P.riemann_params(n=96, weno=FIN_WENO_Z)
    p.my = 80
    cases.append((p, oracle.set_bnd(p, P.random_riemann_state(p, rng))))
    p = P.vortex_params(n=64, weno=FIN_WENO_JS)
    p.my = 40
    cases.append((p, oracle.set_bnd(p, P.random_smooth_state(p, rng))))
    p = P.vortex_params(n=30, weno=FIN_WENO_FD, global_alpha=0)
    p.my = 21
    cases.append((p, oracle.set_bnd(p, P.random_smooth_state(p, rng))))
    p = P.riemann_params(n=33, weno=FIN_WENO_JS, power_param=1.0)
    p.my = 19
    cases.append((p, oracle.set_bnd(p, P.random_riemann_state(p, rng))))
    return cases


def test_noalloc_matches_construct_l_and_oracle_calls_in_a_row(oracle):
    from finess_b200.solver import Solver
    lib = _lib()
    for k, (p, q) in enumerate(_cases(oracle)):
        L_new = _noalloc_construct_l(lib, p, q, check=k % 2)
        with Solver(p) as s:
            L_api, _ = s.ConstructL(q)
        L_orc, _ = oracle.construct_l(p, q)
        assert rel_linf(interior(p, L_new), interior(p, L_api)) <= TOL, k
        assert rel_linf(interior(p, L_new), interior(p, L_orc)) <= TOL, k


def test_noalloc_repeated_call_allocates_nothing(oracle):
    import torch
    lib = _lib()
    p, q = _cases(oracle)[0]
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    Ld = torch.zeros(ghosted_shape(p), dtype=torch.float64, device="cuda")
    assert _call(lib, p, qd, Ld, 1) == FIN_OK       # may load the module (first call on this device)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for check in (0, 1):
        assert _call(lib, p, qd, Ld, check) == FIN_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_reports_nonfinite_when_asked(oracle):
    import torch
    lib = _lib()
    p, q = _cases(oracle)[0]
    q = q.copy()
    mb = p.mbc
    q[mb + 10, mb + 7, 4] = np.nan
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    Ld = torch.zeros(ghosted_shape(p), dtype=torch.float64, device="cuda")
    assert _call(lib, p, qd, Ld, 1) == FIN_ERR_NONFINITE
    # the next call on finite data starts from cleared slots
    p2, q2 = _cases(oracle)[1]
    L2 = _noalloc_construct_l(lib, p2, q2, check=1)
    L2o, _ = oracle.construct_l(p2, q2)
    assert rel_linf(interior(p2, L2), interior(p2, L2o)) <= TOL


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = _lib()
    p = P.riemann_params(n=1024, weno=FIN_WENO_Z)    # 1,048,576 cells > 262,144
    rc = lib.fin_construct_l_noalloc(C.byref(p), C.c_void_p(16), C.c_void_p(16), None, 0)
    assert rc == FIN_ERR_SIZE
