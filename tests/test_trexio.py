"""qmckl_trexio_read on TREXIO text-backend directories.

The reference's test (org/qmckl_trexio.org:1192-1404) reads its CHBrClF dump
(share/qmckl/test_data/chbrclf, written by TREXIO 2.2.0) and compares every
array with the fixture header include/chbrclf.h; the same comparison runs
here against tests/golden/chbrclf.npz (made from that header) on

* a dump of the fixture written by write_text_dump below in the text
  backend's layout (CPU, always), and
* the reference's own dump when the reference tree is present (CPU), and
* on the GPU, the golden ao_vgl values of the reference's AO tests through
  the C ABI after the read.
"""
import os

import numpy as np
import pytest

from oracle import build_ref
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq


def _fmt(x):
    return f"{x: .16e}"


def write_text_dump(d, path):
    """The arrays of a system dict as a TREXIO text-backend directory (one
    file per group: scalars as "<name> <value>" with "<name>_isSet 1",
    arrays as "rank_" / "dims_" lines then their values one per line)."""
    os.makedirs(path, exist_ok=True)
    N, A = int(d["nucl_num"]), int(d["ao_num"])
    S, P, M = d["shell_ang_mom"].size, d["exponent"].size, int(d["mo_coef"].shape[0])
    shell_nucl = np.repeat(np.arange(N), d["nucleus_shell_num"])
    prim_shell = np.repeat(np.arange(S), d["shell_prim_num"])

    def arrays(f, specs):
        for name, dims, _ in specs:
            f.write(f"rank_{name} {len(dims)}\n")
            for i, e in enumerate(dims):
                f.write(f"dims_{name} {i} {e}\n")
        return specs

    def values(f, specs):
        for name, _, vals in specs:
            f.write(f"{name}\n")
            for v in np.asarray(vals).ravel():
                f.write((_fmt(v) if np.issubdtype(np.asarray(vals).dtype, np.floating) else str(int(v))) + "\n")

    with open(os.path.join(path, "electron.txt"), "w") as f:
        f.write(f"electron_up_num_isSet 1 \nelectron_up_num {int(d['elec_up_num'])} \n")
        f.write(f"electron_dn_num_isSet 1 \nelectron_dn_num {int(d['elec_dn_num'])} \n")
    with open(os.path.join(path, "nucleus.txt"), "w") as f:
        sp = arrays(f, [("nucleus_charge", [N], d["charge"]),
                        ("nucleus_coord", [N, 3], np.asarray(d["nucl_coord"]).T)])
        f.write(f"nucleus_num_isSet 1 \nnucleus_num {N} \n")
        values(f, sp)
    with open(os.path.join(path, "basis.txt"), "w") as f:
        sp = arrays(f, [("basis_nucleus_index", [S], shell_nucl), ("basis_shell_ang_mom", [S], d["shell_ang_mom"]),
                        ("basis_shell_factor", [S], d["shell_factor"]), ("basis_shell_index", [P], prim_shell),
                        ("basis_exponent", [P], d["exponent"]), ("basis_coefficient", [P], d["coefficient"]),
                        ("basis_prim_factor", [P], d["prim_factor"])])
        f.write(f"basis_prim_num_isSet 1 \nbasis_prim_num {P} \nbasis_shell_num_isSet 1 \nbasis_shell_num {S} \n")
        f.write("len_basis_type 9\nbasis_type\nGaussian\n")
        values(f, sp)
    with open(os.path.join(path, "ao.txt"), "w") as f:
        sp = arrays(f, [("ao_normalization", [A], d["ao_factor"])])
        f.write(f"ao_cartesian_isSet 1 \nao_cartesian 1 \nao_num_isSet 1 \nao_num {A} \n")
        values(f, sp)
    with open(os.path.join(path, "mo.txt"), "w") as f:
        sp = arrays(f, [("mo_coefficient", [M, A], d["mo_coef"])])
        f.write(f"mo_num_isSet 1 \nmo_num {M} \nlen_mo_type 0\nmo_type\n")
        values(f, sp)


def check_against_fixture(ctx, d, reference_tolerances=False):
    """The reference's TREXIO test: every array read equals the fixture's,
    exactly for a dump written from the fixture; for the reference's own dump
    (written by another program) with the reference test's bounds: shell
    factors within 1e-6, exponents, coefficients and primitive factors within
    1e-7 relative, MO coefficients within 1e-12 relative."""
    N, A = int(d["nucl_num"]), int(d["ao_num"])
    S, P, M = d["shell_ang_mom"].size, d["exponent"].size, int(d["mo_coef"].shape[0])
    assert pq.get_electron_up_num(ctx) == int(d["elec_up_num"])
    assert pq.get_electron_down_num(ctx) == int(d["elec_dn_num"])
    assert pq.get_nucleus_num(ctx) == N
    assert np.array_equal(pq.get_nucleus_charge(ctx, N), d["charge"])
    assert np.array_equal(pq.get_nucleus_coord(ctx, "T", 3 * N), np.asarray(d["nucl_coord"]).ravel())
    assert pq.get_ao_basis_type(ctx) == "G"
    assert pq.get_ao_basis_shell_num(ctx) == S
    assert pq.get_ao_basis_prim_num(ctx) == P
    assert pq.get_ao_basis_ao_num(ctx) == A
    assert not pq.get_ao_basis_r_power(ctx, S).any()
    for name, n in (("nucleus_index", N), ("nucleus_shell_num", N), ("shell_ang_mom", S), ("shell_prim_num", S),
                    ("shell_prim_index", S), ("shell_factor", S), ("exponent", P), ("coefficient", P),
                    ("prim_factor", P), ("ao_factor", A)):
        got = getattr(pq, f"get_ao_basis_{name}")(ctx, n)
        want = np.asarray(d[name]).ravel()
        if not reference_tolerances:
            assert np.array_equal(got, want), name
        elif name == "shell_factor":
            assert np.all(np.abs(got - want) < 1e-6), name
        elif name in ("exponent", "coefficient", "prim_factor"):
            assert np.all(np.abs((got - want) / want) < 1e-7), name
        elif name != "ao_factor":   # not compared by the reference's test
            assert np.array_equal(got, want), name
    assert pq.get_mo_basis_mo_num(ctx) == M
    got = pq.get_mo_basis_coefficient(ctx, M * A)
    want = np.asarray(d["mo_coef"]).ravel()
    if reference_tolerances:
        assert np.all(np.abs(got - want) <= 1e-12 * np.abs(got))
    else:
        assert np.array_equal(got, want)


def test_trexio_text_dump_round_trip(chbrclf, tmp_path):
    path = str(tmp_path / "chbrclf")
    write_text_dump(chbrclf, path)
    ctx = pq.context_create()
    pq.trexio_read(ctx, path)
    check_against_fixture(ctx, chbrclf)
    assert pq.ao_basis_provided(ctx) and pq.mo_basis_provided(ctx)
    pq.context_destroy(ctx)


def test_trexio_high_l_round_trip(tmp_path):
    d = gen.high_l_config(walk_num=1)
    path = str(tmp_path / "high_l")
    write_text_dump(d, path)
    ctx = pq.context_create()
    pq.trexio_read(ctx, path)
    check_against_fixture(ctx, d)
    pq.context_destroy(ctx)


def _reference_dump():
    root = os.environ.get("QMCKL_REFERENCE_ROOT") or build_ref.DEFAULT_ROOT
    p = os.path.join(root, "share", "qmckl", "test_data", "chbrclf")
    return p if os.path.isdir(p) else None


@pytest.mark.skipif(_reference_dump() is None, reason="the reference's TREXIO test data is not present")
def test_trexio_reads_the_reference_dump(chbrclf):
    """The reference's own CHBrClF dump (TREXIO 2.2.0, text backend) gives the
    arrays of include/chbrclf.h, as the reference's test checks."""
    ctx = pq.context_create()
    pq.trexio_read(ctx, _reference_dump())
    check_against_fixture(ctx, chbrclf, reference_tolerances=True)
    pq.context_destroy(ctx)


def test_trexio_rejects_what_it_cannot_open(tmp_path):
    ctx = pq.context_create()
    with pytest.raises(RuntimeError, match="not a TREXIO text-backend directory"):
        pq.trexio_read(ctx, str(tmp_path / "missing.h5"))
    bad = tmp_path / "bad"
    bad.mkdir()
    (bad / "nucleus.txt").write_text("nucleus_num_isSet 0 \n")
    (bad / "electron.txt").write_text("electron_up_num_isSet 1 \nelectron_up_num 1 \nelectron_dn_num_isSet 1 \n"
                                      "electron_dn_num 0 \n")
    with pytest.raises(RuntimeError, match="trexio_read_nucleus_num"):
        pq.trexio_read(ctx, str(bad))
    pq.context_destroy(ctx)


@pytest.mark.gpu
def test_trexio_golden_ao_vgl_through_capi(chbrclf, tmp_path):
    """After the read, the golden ao_vgl of the reference's AO test
    (org/qmckl_ao.org:9355-9384) at the 68 points of walker 1."""
    path = str(tmp_path / "chbrclf")
    write_text_dump(chbrclf, path)
    ctx = pq.context_create()
    pq.b200_set_form(ctx, pq.FORM_FP64)
    pq.trexio_read(ctx, path)
    pq.set_electron_coord(ctx, "N", 1, np.asarray(chbrclf["elec_coord"][:1]).ravel())
    P, A = 68, int(chbrclf["ao_num"])
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    idx = chbrclf["golden_ao_vgl_index"]
    got = np.array([ao[tuple(i)] for i in idx])
    assert np.all(np.abs(got - chbrclf["golden_ao_vgl_value"]) < chbrclf["golden_ao_vgl_tol"])
    pq.context_destroy(ctx)
