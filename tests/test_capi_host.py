"""Host-side behaviour of the C-ABI library (CPU only, no kernel launches)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context


def _declared_symbols():
    names = set()
    for h in ("qmckl.h", "qmckl_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(qmckl_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = pq.lib()
    missing = [n for n in _declared_symbols() if not hasattr(L, n)]
    assert not missing, missing
    assert len(_declared_symbols()) > 90


def test_context_lifecycle():
    ctx = pq.context_create()
    assert pq.context_check(ctx) == ctx
    assert pq.context_check(0) == 0
    ctx2 = pq.context_copy(ctx)
    assert ctx2 != 0 and pq.context_check(ctx2) == ctx2
    pq.context_destroy(ctx2)
    pq.context_destroy(ctx)


def test_numprec():
    ctx = pq.context_create()
    assert pq.get_numprec_precision(ctx) == 53
    assert pq.get_numprec_range(ctx) == 11
    assert pq.get_numprec_epsilon(ctx) == 2.0 ** -52
    pq.set_numprec_precision(ctx, 24)
    assert pq.get_numprec_epsilon(ctx) == 2.0 ** -23
    with pytest.raises(RuntimeError, match="Invalid argument 2"):
        pq.set_numprec_precision(ctx, 54)
    with pytest.raises(RuntimeError, match="Invalid argument 2"):
        pq.set_numprec_range(ctx, 1)
    pq.context_destroy(ctx)


def test_error_strings():
    assert pq.string_of_error(0) == "Success"
    assert pq.string_of_error(108) == "Already set"
    assert pq.string_of_error(106) == "Not provided"


def test_setters_masks_and_finalize(chbrclf):
    """Set-up sequence of the reference AO test (org/qmckl_ao.org:2459-2545)."""
    d = chbrclf
    ctx = pq.context_create()
    pq.set_nucleus_num(ctx, 5)
    pq.set_nucleus_coord(ctx, "T", d["nucl_coord"].reshape(-1))
    pq.set_nucleus_charge(ctx, d["charge"])
    assert pq.nucleus_provided(ctx)
    with pytest.raises(RuntimeError, match="Already set"):
        pq.set_nucleus_num(ctx, 5)
    pq.set_ao_basis_type(ctx, "G")
    with pytest.raises(RuntimeError, match="Already set"):
        pq.set_ao_basis_cartesian(ctx, True)      # shares mask bit 1 with the type
    pq.set_ao_basis_shell_num(ctx, 72)
    pq.set_ao_basis_prim_num(ctx, 297)
    pq.set_ao_basis_nucleus_index(ctx, d["nucleus_index"])
    with pytest.raises(RuntimeError, match="Already set"):
        pq.set_ao_basis_nucleus_index(ctx, d["nucleus_index"])
    pq.set_ao_basis_nucleus_shell_num(ctx, d["nucleus_shell_num"])
    pq.set_ao_basis_shell_ang_mom(ctx, d["shell_ang_mom"])
    pq.set_ao_basis_shell_factor(ctx, d["shell_factor"])
    pq.set_ao_basis_shell_prim_num(ctx, d["shell_prim_num"])
    pq.set_ao_basis_shell_prim_index(ctx, d["shell_prim_index"])
    pq.set_ao_basis_exponent(ctx, d["exponent"])
    pq.set_ao_basis_coefficient(ctx, d["coefficient"])
    assert not pq.ao_basis_provided(ctx)
    pq.set_ao_basis_prim_factor(ctx, d["prim_factor"])
    pq.set_ao_basis_ao_num(ctx, 263)
    pq.set_ao_basis_ao_factor(ctx, d["ao_factor"])
    assert pq.ao_basis_provided(ctx)
    assert pq.get_ao_basis_type(ctx) == "G"
    assert pq.get_ao_basis_shell_num(ctx) == 72
    assert pq.get_ao_basis_ao_num(ctx) == 263
    assert np.array_equal(pq.get_ao_basis_nucleus_index(ctx, 5), d["nucleus_index"])
    assert np.array_equal(pq.get_ao_basis_shell_ang_mom(ctx, 72), d["shell_ang_mom"])
    assert np.array_equal(pq.get_ao_basis_exponent(ctx, 297), d["exponent"])
    assert np.array_equal(pq.get_ao_basis_r_power(ctx, 72), np.zeros(72, dtype=np.int32))
    with pytest.raises(RuntimeError, match="Invalid argument 3"):
        pq.get_ao_basis_exponent(ctx, 10)
    pq.set_mo_basis_mo_num(ctx, 224)
    assert not pq.mo_basis_provided(ctx)
    pq.set_mo_basis_coefficient(ctx, d["mo_coef"].reshape(-1))
    assert pq.mo_basis_provided(ctx)
    assert np.array_equal(pq.get_mo_basis_coefficient(ctx, 224 * 263), d["mo_coef"].reshape(-1))
    pq.set_mo_basis_coefficient(ctx, d["mo_coef"].reshape(-1))   # may be replaced
    with pytest.raises(RuntimeError, match="Already set"):
        pq.set_mo_basis_mo_num(ctx, 224)
    keep = np.zeros(224, dtype=np.int32)
    keep[:10] = 1
    pq.mo_basis_select_mo(ctx, keep)
    assert pq.get_mo_basis_mo_num(ctx) == 10
    with pytest.raises(RuntimeError, match="Invalid argument 2"):
        pq.mo_basis_rescale(ctx, 0.0)
    pq.context_destroy(ctx)


def test_points_and_electrons(chbrclf):
    ctx = pq.context_create()
    with pytest.raises(RuntimeError):
        pq.set_electron_coord(ctx, "N", 2, chbrclf["elec_coord"].reshape(-1))   # electrons not set
    pq.set_electron_num(ctx, 34, 34)
    assert pq.electron_provided(ctx)
    pq.set_electron_coord(ctx, "N", 2, chbrclf["elec_coord"].reshape(-1))
    assert pq.get_point_num(ctx) == 136
    assert pq.get_electron_walk_num(ctx) == 2
    back = pq.get_point(ctx, "N", 3 * 136)
    assert np.array_equal(back, chbrclf["elec_coord"].reshape(-1))
    t = pq.get_point(ctx, "T", 3 * 136)
    assert np.array_equal(t.reshape(3, -1).T, chbrclf["elec_coord"].reshape(-1, 3))
    with pytest.raises(RuntimeError, match="Invalid argument 2"):
        pq.set_point(ctx, "X", 2, np.zeros(6))
    with pytest.raises(RuntimeError, match="Invalid argument 4"):
        pq.set_point(ctx, "N", 3, np.zeros(6))
    pq.context_destroy(ctx)


def test_inconsistent_basis_is_rejected(chbrclf):
    d = dict(chbrclf)
    d["ao_factor"] = np.ones(262)
    with pytest.raises(RuntimeError, match="Failure"):
        make_context(d, points=False)


def test_allocation_failure_injection(chbrclf):
    ctx = pq.context_create()
    pq.set_nucleus_num(ctx, 5)
    pq.b200_inject_alloc_failure(0)
    with pytest.raises(RuntimeError, match="Allocation failed"):
        pq.set_nucleus_charge(ctx, chbrclf["charge"])
    # the context stays usable and the field stays unset
    assert not pq.nucleus_provided(ctx)
    pq.set_nucleus_charge(ctx, chbrclf["charge"])
    pq.context_destroy(ctx)


def test_compute_without_gpu_fails_loudly(chbrclf):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    ctx = make_context(chbrclf)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        pq.get_mo_basis_mo_vgl(ctx, 136 * 5 * 224)
    pq.context_destroy(ctx)


def test_trexio_read_rejects_a_file_no_backend_opens():
    """qmckl_trexio_read on a path that is not a TREXIO text-backend directory
    fails with QMCKL_INVALID_ARG_2, as the reference does when none of its
    backends opens the file (org/qmckl_trexio.org:1148-1155)."""
    ctx = pq.context_create()
    with pytest.raises(RuntimeError, match="Invalid argument 2"):
        pq.trexio_read(ctx, "fake.h5")
    pq.context_destroy(ctx)
