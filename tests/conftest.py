import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "chbrclf.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def chbrclf():
    from qmckl_b200 import gen
    return gen.chbrclf(GOLDEN)


def parity_error(got, ref, floor=1e-2):
    """Relative error with a floor of `floor` times the (point, component) row maximum.

    max over elements of |got - ref| / max(|ref|, floor * max_k |ref[p, c, k]|).
    The reference's own two CPU paths (doc and HPC) agree to 2e-14 (AO) and
    2e-13 (MO) under this metric on CHBrClF, while element-wise they differ
    by up to 1e-9 where a value is dominated by cancellation.
    """
    got = np.asarray(got)
    ref = np.asarray(ref)
    scale = np.abs(ref).max(axis=-1, keepdims=True)
    den = np.maximum(np.abs(ref), floor * scale)
    den = np.where(den == 0, 1.0, den)
    return float((np.abs(got - ref) / den).max())


COMPONENTS = ("value", "grad_x", "grad_y", "grad_z", "laplacian")


def elementwise_rel_error(got, ref, floor=1e-8):
    """Per component of [P][5][n] arrays: max |got - ref| / |ref| over the
    elements with |ref| > floor * max |ref| of that component; 5 floats."""
    out = []
    for c in range(ref.shape[1]):
        r = ref[:, c, :]
        g = got[:, c, :]
        s = np.abs(r).max()
        m = np.abs(r) > floor * s
        out.append(float((np.abs(g[m] - r[m]) / np.abs(r[m])).max()) if m.any() else 0.0)
    return out


def row_floored_error(got, ref, floor=1e-2):
    """Per component of [P][5][n] arrays: parity_error restricted to that component; 5 floats."""
    return [parity_error(got[:, c, :], ref[:, c, :], floor) for c in range(ref.shape[1])]


def bits_of_agreement(a, b):
    """Bits two FP64 arrays agree on, element-wise: the reference's
    qmckl_test_precision_64 (org/qmckl_numprec.org:384-430).  The distance in
    units in the last place is the difference of the two bit patterns (0 bits
    when the signs differ and neither value is zero); the result is 53 minus
    the bit length of that distance, at least 0."""
    af = np.ascontiguousarray(a, dtype=np.float64).ravel()
    bf = np.ascontiguousarray(b, dtype=np.float64).ravel()
    x, y = af.view(np.int64), bf.view(np.int64)
    same = (x < 0) == (y < 0)
    d = np.zeros(x.size, dtype=np.int64)
    d[same] = np.abs(x[same] - y[same])          # same sign: no overflow
    out = 53 - np.minimum(53, np.frexp(d.astype(np.float64))[1])   # frexp exponent = bit length
    for i in np.flatnonzero(~same):
        if af[i] != 0.0 and bf[i] != 0.0:
            out[i] = 0
        else:   # one of them is +-0: the plain difference of the bit patterns
            out[i] = 53 - min(53, abs(int(x[i]) - int(y[i])).bit_length())
    return out.astype(np.int32).reshape(np.shape(a))


def mixed_error_report(got, ref):
    """The three error measures of the mixed form against an FP64 reference,
    per component: max|diff| / max|ref|, the row-floored relative error and
    the element-wise relative error (|ref| > 1e-8 max|ref|)."""
    return {"max_abs_over_max_ref": dict(zip(COMPONENTS, comp_error(got, ref))),
            "row_floored_rel": dict(zip(COMPONENTS, row_floored_error(got, ref))),
            "elementwise_rel": dict(zip(COMPONENTS, elementwise_rel_error(got, ref)))}


def comp_error(got, ref):
    """Per-component max|got - ref| / max|ref| for arrays [P][5][n]; returns 5 floats."""
    out = []
    for c in range(ref.shape[1]):
        s = np.abs(ref[:, c, :]).max()
        out.append(float(np.abs(got[:, c, :] - ref[:, c, :]).max() / (s if s > 0 else 1.0)))
    return out
