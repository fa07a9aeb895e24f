"""Argument and call-order errors of the solver's C ABI: each returns its
status code with a message instead of running (the reference throws in the
same places: KMatrixExtractor for E <= 0, the setup for an l_cont outside the
prepared channel set)."""
import ctypes as C

import numpy as np
import pytest

from scatt_b200 import _lib, synth
from scatt_b200 import solver as S

pytestmark = pytest.mark.gpu

ARG, STATE = 1, 8


@pytest.fixture(scope="module")
def solver():
    sol = S.ScanSolver(synth.h2_like(Nr=201, dr=0.05, l_cont=11))
    yield sol
    sol.close()


def _code(fn):
    with pytest.raises(_lib.ScattError) as ex:
        fn()
    return ex.value.code, str(ex.value)


def test_empty_energy_list_is_a_no_op(solver):
    assert solver.solve([]) == []


@pytest.mark.parametrize("E", [0.0, -0.3, float("nan")])
def test_energy_must_be_positive(solver, E):
    code, msg = _code(lambda: solver.solve([0.5, E]))
    assert code == ARG and "energy must be > 0" in msg


def test_l_cont_outside_the_uploaded_scan(solver):
    code, msg = _code(lambda: solver.solve([0.5], l_cont=[12]))
    assert code == ARG and "l_cont 12" in msg
    # l_cont 9 would change the exchange cutoff min(l_cont, 10) of the scan
    code, msg = _code(lambda: solver.solve([0.5], l_cont=[9]))
    assert code == ARG and "exchange cutoff" in msg


def test_solve_before_upload_is_a_state_error():
    L = _lib.lib()
    S._bind()
    ctx = C.c_void_p()
    _lib.check(L.scatt_ctx_create(0, C.byref(ctx)))
    try:
        E = np.array([0.5])
        out = S.Outputs()
        st = np.zeros(1, dtype=np.int32)
        out.status = st.ctypes.data_as(_lib.iptr)
        rc = L.scatt_solve_batch(ctx, 1, _lib.as_dptr(E), None, None, C.byref(out))
        assert rc == STATE
        assert b"scatt_upload_static" in L.scatt_last_error()
    finally:
        L.scatt_ctx_destroy(ctx)
