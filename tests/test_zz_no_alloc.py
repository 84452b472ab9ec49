"""fin_construct_l_noalloc: ConstructL for callers that cannot allocate
device memory (their own allocator owns the device, or they run where
allocation is forbidden).  It keeps its scratch in a static device array, so
the caller passes device buffers it already owns.  This file is collected
last so a failure here never hides another test.

The check: two calls in a row on different inputs, each against the
existing entry point fin_construct_l, at the 1e-12 relative L-infinity the
ConstructL parity tests use; the second call must not see the first call's
scratch contents."""
import ctypes as C

import numpy as np
import pytest

from conftest import interior, rel_linf
from finess_b200 import problems as P
from finess_b200._abi import FIN_ERR_SIZE, FIN_OK, FIN_WENO_JS, FIN_WENO_Z, ghosted_shape

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _lib():
    from finess_b200.solver import load_library
    lib = load_library()
    lib.fin_construct_l_noalloc.argtypes = [C.POINTER(type(P.riemann_params(n=8))), C.c_void_p, C.c_void_p,
                                            C.c_void_p]
    lib.fin_construct_l_noalloc.restype = C.c_int
    return lib


def _noalloc_construct_l(lib, p, q):
    import torch
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    Ld = torch.zeros(ghosted_shape(p), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.fin_construct_l_noalloc(C.byref(p), C.c_void_p(qd.data_ptr()), C.c_void_p(Ld.data_ptr()),
                                     C.c_void_p(stream))
    assert rc == FIN_OK, rc
    torch.cuda.synchronize()
    return Ld.cpu().numpy()


def test_noalloc_matches_construct_l_two_calls():
    from finess_b200.solver import Solver
    lib = _lib()
    rng = np.random.default_rng(123)
    cases = []
    p1 = P.riemann_params(n=96, weno=FIN_WENO_Z)
    p1.my = 80
    cases.append((p1, P.random_riemann_state(p1, rng)))
    p2 = P.vortex_params(n=64, weno=FIN_WENO_JS)
    p2.my = 40
    cases.append((p2, P.random_smooth_state(p2, rng)))
    for p, q in cases:
        L_new = _noalloc_construct_l(lib, p, q)
        with Solver(p) as s:
            L_ref, _ = s.ConstructL(q)
        assert rel_linf(interior(p, L_new), interior(p, L_ref)) <= TOL


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = _lib()
    p = P.riemann_params(n=1024, weno=FIN_WENO_Z)    # 1,048,576 cells > 262,144
    rc = lib.fin_construct_l_noalloc(C.byref(p), C.c_void_p(16), C.c_void_p(16), None)
    assert rc == FIN_ERR_SIZE
