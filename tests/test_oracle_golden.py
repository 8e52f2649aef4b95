"""Pin the CPU oracle to the reference's own golden vectors (CPU only)."""
import numpy as np
import pytest

from conftest import parity_error
from oracle import pyoracle as O


@pytest.fixture(scope="module")
def basis(chbrclf):
    return O.Basis(chbrclf)


def _walker1(chbrclf):
    return chbrclf["elec_coord"][0]   # the 68 points of walker 1 used by the reference tests


@pytest.mark.parametrize("name", ["prim_vgl", "shell_vgl"])
def test_radial_golden(chbrclf, basis, name):
    fn = O.primitive_vgl if name == "prim_vgl" else O.shell_vgl
    arr = fn(basis, _walker1(chbrclf), chbrclf["nucl_coord"])
    idx = chbrclf[f"golden_{name}_index"]
    val = chbrclf[f"golden_{name}_value"]
    tol = chbrclf[f"golden_{name}_tol"]
    got = np.array([arr[tuple(i)] for i in idx])
    assert np.all(np.abs(got - val) < tol)


@pytest.mark.parametrize("path", ["hpc", "doc"])
def test_ao_vgl_golden(chbrclf, basis, path):
    arr = O.ao_vgl(basis, _walker1(chbrclf), chbrclf["nucl_coord"], path=path)
    idx = chbrclf["golden_ao_vgl_index"]
    got = np.array([arr[tuple(i)] for i in idx])
    assert np.all(np.abs(got - chbrclf["golden_ao_vgl_value"]) < chbrclf["golden_ao_vgl_tol"])


def test_ao_value_golden(chbrclf, basis):
    arr = O.ao_value(basis, _walker1(chbrclf), chbrclf["nucl_coord"])
    idx = chbrclf["golden_ao_value_index"]
    got = np.array([arr[tuple(i)] for i in idx])
    assert np.all(np.abs(got - chbrclf["golden_ao_value_value"]) < chbrclf["golden_ao_value_tol"])


def test_hpc_and_doc_paths_agree(chbrclf, basis):
    """The two reference algorithms restated here agree under the parity metric."""
    pts = chbrclf["elec_coord"].reshape(-1, 3)
    h = O.ao_vgl(basis, pts, chbrclf["nucl_coord"], path="hpc")
    d = O.ao_vgl(basis, pts, chbrclf["nucl_coord"], path="doc")
    assert parity_error(h, d) < 1e-13
    mh = O.mo_vgl(chbrclf["mo_coef"], h)
    md = O.mo_vgl(chbrclf["mo_coef"], d)
    assert parity_error(mh, md) < 1e-12


def test_mo_consistency(chbrclf, basis):
    """mo_vgl[:,0,:] == mo_value (org/qmckl_mo.org:3745-3761) and rescale x2 linearity."""
    pts = chbrclf["elec_coord"].reshape(-1, 3)
    av = O.ao_vgl(basis, pts, chbrclf["nucl_coord"])
    aval = O.ao_value(basis, pts, chbrclf["nucl_coord"])
    mv = O.mo_vgl(chbrclf["mo_coef"], av)
    mval = O.mo_value(chbrclf["mo_coef"], aval)
    assert np.abs(mv[:, 0, :] - mval).max() < 1e-12
    m2 = O.mo_value(2.0 * chbrclf["mo_coef"], aval)
    assert np.abs(2.0 * mv[:, 0, :] - m2).max() < 1e-12


def test_precision_cutoff():
    assert abs(O.cutoff(53) - 52 * np.log(2.0)) < 1e-12
    assert abs(O.cutoff(24) - 23 * np.log(2.0)) < 1e-12


def test_single_precision_exponentials(chbrclf, basis):
    """precision <= 23 switches the reference's exponentials to FP32 (org/qmckl_ao.org:8775-8796)."""
    pts = chbrclf["elec_coord"][0]
    d = O.ao_vgl(basis, pts, chbrclf["nucl_coord"], precision=53)
    s = O.ao_vgl(basis, pts, chbrclf["nucl_coord"], precision=23)
    err = np.abs(s - d).max() / np.abs(d).max()
    assert 0 < err < 1e-4
