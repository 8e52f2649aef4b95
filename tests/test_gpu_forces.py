"""Orbital forces getters (qmckl_get_forces_*) on the GPU against the oracle's
restatement of the reference's forces (pinned to nuclear finite differences in
tests/test_oracle_derivatives.py), FP64, parity metric <= 1e-12."""
import numpy as np
import pytest

from conftest import parity_error
from oracle import pyoracle as O
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["chbrclf", "config0"])
def test_forces_match_oracle(which, chbrclf):
    d = chbrclf if which == "chbrclf" else gen.config(0, walk_num=3)
    ctx = make_context(d, form=pq.FORM_FP64)
    pts = gen.points(d)
    P, N, A, M = pts.shape[0], d["nucl_num"], d["ao_num"], d["mo_num"]
    fao, fmv, fmg, fml = O.forces(O.Basis(d), pts, d["nucl_coord"], d["mo_coef"])
    got_ao = pq.get_forces_ao_value(ctx, N * P * 3 * A).reshape(N, P, 3, A)
    got_v = pq.get_forces_mo_value(ctx, N * P * 3 * M).reshape(N, P, 3, M)
    got_g = pq.get_forces_mo_g(ctx, N * 9 * P * M).reshape(N, 3, P, 3, M)
    got_l = pq.get_forces_mo_l(ctx, N * 3 * P * M).reshape(N, 3, P, M)
    inpl = pq.get_forces_mo_value_inplace(ctx, N * P * 3 * M).reshape(N, P, 3, M)
    inpl_g = pq.get_forces_mo_g_inplace(ctx, N * 9 * P * M).reshape(N, 3, P, 3, M)
    pq.context_destroy(ctx)
    assert parity_error(got_ao, fao) <= 1e-12
    assert parity_error(got_v, fmv) <= 1e-12
    assert parity_error(got_g, fmg) <= 1e-12
    assert parity_error(got_l, fml) <= 1e-12
    assert np.array_equal(inpl, got_v) and np.array_equal(inpl_g, got_g)


def test_forces_size_checks(chbrclf):
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    with pytest.raises(RuntimeError):
        pq.get_forces_mo_value(ctx, 10)
    with pytest.raises(RuntimeError):
        pq.get_forces_mo_g(ctx, 10)
    pq.context_destroy(ctx)
