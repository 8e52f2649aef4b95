"""The oracle against the reference's own C code (CPU only).

oracle/build_ref.py extracts the reference's HPC kernels and basis
finalization verbatim from its org sources and compiles them
(oracle/_ref/libqmckl_ref.so, built where the reference's sources are
present).  Built the same way (no fused multiply-add contraction), the
oracle's restatement reproduces them to the last bit for AO VGL, MO VGL and
MO value; AO value differs by at most 1e-17 absolute where the reference's
value kernel leaves out the 1e-20 shift of some polynomial terms
(org/qmckl_ao.org:7919-7935).  The reference's golden vectors pass through
its own compiled code as well.  Skipped where the library was not built.
"""
import numpy as np
import pytest

from conftest import parity_error
from oracle import pyoracle as O
from oracle import refpath
from qmckl_b200 import gen

pytestmark = pytest.mark.skipif(not refpath.available(), reason="oracle/_ref not built (no reference sources)")


def _systems(chbrclf):
    return [("chbrclf", chbrclf), ("config0", gen.config(0, walk_num=16)), ("high_l", gen.high_l_config(4)),
            ("config1", gen.config(1, walk_num=2))]


@pytest.mark.parametrize("k", range(4))
def test_oracle_is_the_reference_bit_for_bit(chbrclf, k):
    name, d = _systems(chbrclf)[k]
    pts = gen.points(d)
    ref = refpath.RefSystem(d, num_threads=4)
    b = O.Basis(d)
    ao = O.ao_vgl(b, pts, d["nucl_coord"])
    assert np.array_equal(ao, ref.ao_vgl(pts)), name
    assert np.array_equal(O.mo_vgl(d["mo_coef"], ao), ref.mo_vgl(pts)), name
    av = O.ao_value(b, pts, d["nucl_coord"])
    rv = ref.ao_value(pts)
    assert np.abs(av - rv).max() <= 1e-17 and parity_error(av, rv) < 1e-14, name
    assert np.array_equal(O.mo_value(d["mo_coef"], rv), ref.mo_value(pts)), name


def test_single_precision_exponentials_bit_for_bit(chbrclf):
    """precision 23: FP32 exponentials in both (org/qmckl_ao.org:8775-8796)."""
    pts = gen.points(chbrclf)
    ref = refpath.RefSystem(chbrclf, precision=23)
    ao = O.ao_vgl(O.Basis(chbrclf), pts, chbrclf["nucl_coord"], precision=23)
    assert np.array_equal(ao, ref.ao_vgl(pts))


def test_golden_vectors_through_the_reference_build(chbrclf):
    """The golden ao_vgl / ao_value of the reference's own tests
    (org/qmckl_ao.org:9355-9384, 8399-8405), 68 points of walker 1."""
    ref = refpath.RefSystem(chbrclf)
    pts = chbrclf["elec_coord"][0]
    for name, arr in (("ao_vgl", ref.ao_vgl(pts)), ("ao_value", ref.ao_value(pts))):
        idx = chbrclf[f"golden_{name}_index"]
        got = np.array([arr[tuple(i)] for i in idx])
        assert np.all(np.abs(got - chbrclf[f"golden_{name}_value"]) < chbrclf[f"golden_{name}_tol"]), name


def test_threads_do_not_change_the_result(chbrclf):
    pts = gen.points(chbrclf)
    ref = refpath.RefSystem(chbrclf)
    assert np.array_equal(ref.mo_vgl(pts, nthreads=1), ref.mo_vgl(pts, nthreads=4))
