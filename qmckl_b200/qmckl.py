"""Python face of libqmckl_b200.so, mirroring the reference's SWIG module.

The reference's Python module ``qmckl`` (python/src/qmckl.i) strips the
``qmckl_`` prefix, turns every ``(array, size_max)`` input pair into one numpy
argument, every ``(array, size_max)`` output pair into a ``size_max`` argument
and a returned numpy array, scalar output pointers into return values, and a
non-zero exit code into ``RuntimeError(qmckl_string_of_error(rc))``
(python/src/qmckl.i:15, 59-95; python/src/process_header.py:44-70).  The same
conventions hold here, so the reference's own Python test
(python/test/test_api.py) reads unchanged apart from the import:

    from qmckl_b200 import qmckl as pq
    ctx = pq.context_create()
    pq.set_electron_coord(ctx, 'T', walk_num, coord)
    mo_vgl = pq.get_mo_basis_mo_vgl(ctx, size_max)
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libqmckl_b200.so")

_lib = None


def lib():
    """The loaded product library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libqmckl_b200.so is not built ({LIB_PATH}); run python -m qmckl_b200.build")
        L = C.CDLL(LIB_PATH)
        L.qmckl_string_of_error.restype = C.c_char_p
        L.qmckl_string_of_error.argtypes = [C.c_int32]
        L.qmckl_context_create.restype = C.c_int64
        L.qmckl_context_create.argtypes = []
        L.qmckl_context_copy.restype = C.c_int64
        L.qmckl_context_copy.argtypes = [C.c_int64]
        L.qmckl_context_check.restype = C.c_int64
        L.qmckl_context_check.argtypes = [C.c_int64]
        L.qmckl_get_numprec_epsilon.restype = C.c_double
        L.qmckl_get_numprec_epsilon.argtypes = [C.c_int64]
        L.qmckl_get_numprec_precision.restype = C.c_int32
        L.qmckl_get_numprec_precision.argtypes = [C.c_int64]
        L.qmckl_get_numprec_range.restype = C.c_int32
        L.qmckl_get_numprec_range.argtypes = [C.c_int64]
        L.qmckl_b200_kernel_launch_count.restype = C.c_int64
        L.qmckl_b200_kernel_launch_count.argtypes = []
        L.qmckl_b200_inject_alloc_failure.restype = None
        L.qmckl_b200_inject_alloc_failure.argtypes = [C.c_int64]
        for name in ("qmckl_nucleus_provided", "qmckl_electron_provided", "qmckl_ao_basis_provided",
                     "qmckl_mo_basis_provided"):
            getattr(L, name).restype = C.c_bool
            getattr(L, name).argtypes = [C.c_int64]
        _lib = L
    return _lib


def string_of_error(rc):
    return lib().qmckl_string_of_error(int(rc)).decode()


def _check(rc, ctx=None):
    if rc != 0:
        msg = string_of_error(rc)
        if ctx is not None:
            buf = C.create_string_buffer(1024)
            if lib().qmckl_last_error(C.c_int64(ctx), buf) == 0:
                msg = msg + " | " + buf.value.decode(errors="replace")
        raise RuntimeError(msg)


def _call(name, ctx, *args, restype=C.c_int32):
    f = getattr(lib(), name)
    f.restype = restype
    rc = f(C.c_int64(ctx), *args)
    _check(rc, ctx)


def _arr(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, a.ctypes.data_as(C.c_void_p), C.c_int64(a.size)


# ---------------------------------------------------------------- context

def context_create():
    ctx = lib().qmckl_context_create()
    if ctx == 0:
        raise RuntimeError("qmckl_context_create failed")
    return ctx


def context_copy(ctx):
    return lib().qmckl_context_copy(C.c_int64(ctx))


def context_check(ctx):
    return lib().qmckl_context_check(C.c_int64(ctx))


def context_destroy(ctx):
    _call("qmckl_context_destroy", ctx)


def context_touch(ctx):
    _call("qmckl_context_touch", ctx)


def context_set_num_threads(ctx, n):
    _call("qmckl_context_set_num_threads", ctx, C.c_int32(n))


def context_get_num_threads(ctx):
    v = C.c_int32()
    _call("qmckl_context_get_num_threads", ctx, C.byref(v))
    return v.value


def last_error(ctx):
    buf = C.create_string_buffer(1024)
    lib().qmckl_last_error(C.c_int64(ctx), buf)
    return buf.value.decode(errors="replace")


def set_numprec_precision(ctx, p):
    _call("qmckl_set_numprec_precision", ctx, C.c_int(p))


def get_numprec_precision(ctx):
    return lib().qmckl_get_numprec_precision(C.c_int64(ctx))


def set_numprec_range(ctx, r):
    _call("qmckl_set_numprec_range", ctx, C.c_int(r))


def get_numprec_range(ctx):
    return lib().qmckl_get_numprec_range(C.c_int64(ctx))


def get_numprec_epsilon(ctx):
    return lib().qmckl_get_numprec_epsilon(C.c_int64(ctx))


# ------------------------------------------------------------ nuclei

def set_nucleus_num(ctx, n):
    _call("qmckl_set_nucleus_num", ctx, C.c_int64(n))


def set_nucleus_charge(ctx, charge):
    a, p, n = _arr(charge, np.float64)
    _call("qmckl_set_nucleus_charge", ctx, p, n)


def set_nucleus_coord(ctx, transp, coord):
    a, p, n = _arr(coord, np.float64)
    _call("qmckl_set_nucleus_coord", ctx, C.c_char(transp.encode()), p, n)


def get_nucleus_num(ctx):
    v = C.c_int64()
    _call("qmckl_get_nucleus_num", ctx, C.byref(v))
    return v.value


def get_nucleus_charge(ctx, size_max):
    out = np.zeros(size_max, dtype=np.float64)
    _call("qmckl_get_nucleus_charge", ctx, out.ctypes.data_as(C.c_void_p), C.c_int64(size_max))
    return out


def get_nucleus_coord(ctx, transp, size_max):
    out = np.zeros(size_max, dtype=np.float64)
    _call("qmckl_get_nucleus_coord", ctx, C.c_char(transp.encode()), out.ctypes.data_as(C.c_void_p), C.c_int64(size_max))
    return out


def nucleus_provided(ctx):
    return bool(lib().qmckl_nucleus_provided(C.c_int64(ctx)))


# ------------------------------------------------------ electrons / points

def set_electron_num(ctx, up, dn):
    _call("qmckl_set_electron_num", ctx, C.c_int64(up), C.c_int64(dn))


def set_electron_coord(ctx, transp, walk_num, coord):
    a, p, n = _arr(coord, np.float64)
    _call("qmckl_set_electron_coord", ctx, C.c_char(transp.encode()), C.c_int64(walk_num), p, n)


def get_electron_num(ctx):
    v = C.c_int64()
    _call("qmckl_get_electron_num", ctx, C.byref(v))
    return v.value


def get_electron_up_num(ctx):
    v = C.c_int64()
    _call("qmckl_get_electron_up_num", ctx, C.byref(v))
    return v.value


def get_electron_down_num(ctx):
    v = C.c_int64()
    _call("qmckl_get_electron_down_num", ctx, C.byref(v))
    return v.value


def get_electron_walk_num(ctx):
    v = C.c_int64()
    _call("qmckl_get_electron_walk_num", ctx, C.byref(v))
    return v.value


def get_electron_coord(ctx, transp, size_max):
    out = np.zeros(size_max, dtype=np.float64)
    _call("qmckl_get_electron_coord", ctx, C.c_char(transp.encode()), out.ctypes.data_as(C.c_void_p), C.c_int64(size_max))
    return out


def electron_provided(ctx):
    return bool(lib().qmckl_electron_provided(C.c_int64(ctx)))


def set_point(ctx, transp, num, coord):
    a, p, n = _arr(coord, np.float64)
    _call("qmckl_set_point", ctx, C.c_char(transp.encode()), C.c_int64(num), p, n)


def get_point_num(ctx):
    v = C.c_int64()
    _call("qmckl_get_point_num", ctx, C.byref(v))
    return v.value


def get_point(ctx, transp, size_max):
    out = np.zeros(size_max, dtype=np.float64)
    _call("qmckl_get_point", ctx, C.c_char(transp.encode()), out.ctypes.data_as(C.c_void_p), C.c_int64(size_max))
    return out


# ------------------------------------------------------------- AO basis

def set_ao_basis_type(ctx, t):
    _call("qmckl_set_ao_basis_type", ctx, C.c_char(t.encode()))


def get_ao_basis_type(ctx):
    v = C.c_char()
    _call("qmckl_get_ao_basis_type", ctx, C.byref(v))
    return v.value.decode()


for _name in ("shell_num", "prim_num", "ao_num"):
    def _mk(name):
        def setter(ctx, n):
            _call(f"qmckl_set_ao_basis_{name}", ctx, C.c_int64(n))

        def getter(ctx):
            v = C.c_int64()
            _call(f"qmckl_get_ao_basis_{name}", ctx, C.byref(v))
            return v.value
        return setter, getter
    globals()[f"set_ao_basis_{_name}"], globals()[f"get_ao_basis_{_name}"] = _mk(_name)

_AO_ARRAYS = {
    "nucleus_shell_num": np.int64, "nucleus_index": np.int64, "shell_ang_mom": np.int32,
    "shell_prim_num": np.int64, "shell_prim_index": np.int64, "shell_factor": np.float64,
    "exponent": np.float64, "coefficient": np.float64, "prim_factor": np.float64,
    "ao_factor": np.float64, "r_power": np.int32,
}
for _name, _dt in _AO_ARRAYS.items():
    def _mk(name, dt):
        def setter(ctx, arr):
            a, p, n = _arr(arr, dt)
            _call(f"qmckl_set_ao_basis_{name}", ctx, p, n)

        def getter(ctx, size_max):
            out = np.zeros(size_max, dtype=dt)
            _call(f"qmckl_get_ao_basis_{name}", ctx, out.ctypes.data_as(C.c_void_p), C.c_int64(size_max))
            return out
        return setter, getter
    globals()[f"set_ao_basis_{_name}"], globals()[f"get_ao_basis_{_name}"] = _mk(_name, _dt)


def set_ao_basis_cartesian(ctx, cartesian):
    _call("qmckl_set_ao_basis_cartesian", ctx, C.c_bool(cartesian))


def get_ao_basis_cartesian(ctx):
    v = C.c_bool()
    _call("qmckl_get_ao_basis_cartesian", ctx, C.byref(v))
    return bool(v.value)


def ao_basis_provided(ctx):
    return bool(lib().qmckl_ao_basis_provided(C.c_int64(ctx)))


def _array_getter(cname):
    def getter(ctx, size_max):
        out = np.empty(size_max, dtype=np.float64)
        _call(cname, ctx, out.ctypes.data_as(C.c_void_p), C.c_int64(size_max))
        return out
    getter.__name__ = cname[len("qmckl_"):]
    return getter


get_ao_basis_primitive_vgl = _array_getter("qmckl_get_ao_basis_primitive_vgl")
get_ao_basis_shell_vgl = _array_getter("qmckl_get_ao_basis_shell_vgl")
get_ao_basis_ao_vgl = _array_getter("qmckl_get_ao_basis_ao_vgl")
get_ao_basis_ao_vgl_inplace = _array_getter("qmckl_get_ao_basis_ao_vgl_inplace")
get_ao_basis_ao_value = _array_getter("qmckl_get_ao_basis_ao_value")
get_ao_basis_ao_value_inplace = _array_getter("qmckl_get_ao_basis_ao_value_inplace")
get_ao_basis_ao_hessian = _array_getter("qmckl_get_ao_basis_ao_hessian")
get_forces_ao_value = _array_getter("qmckl_get_forces_ao_value")
get_forces_mo_value = _array_getter("qmckl_get_forces_mo_value")
get_forces_mo_value_inplace = _array_getter("qmckl_get_forces_mo_value_inplace")
get_forces_mo_g = _array_getter("qmckl_get_forces_mo_g")
get_forces_mo_g_inplace = _array_getter("qmckl_get_forces_mo_g_inplace")
get_forces_mo_l = _array_getter("qmckl_get_forces_mo_l")

# ----------------------------------------------- standalone AO helpers


def ao_power(ctx, X, LMAX, ldp):
    """P[n][ldp], P[i][k-1] = X[i]**k for k = 1..LMAX[i] (entries past LMAX[i] are 0)."""
    x, xp, n = _arr(X, np.float64)
    lm, lp, _ = _arr(LMAX, np.int32)
    P = np.zeros((x.size, ldp), dtype=np.float64)
    _check(lib().qmckl_ao_power(C.c_int64(ctx), n, xp, lp, P.ctypes.data_as(C.c_void_p), C.c_int64(ldp)))
    return P


def ao_gaussian_vgl(ctx, X, R, A, ldv=None):
    """VGL[5][ldv] of exp(-A[i] |X-R|^2): value, gradient, Laplacian."""
    x, xp, _ = _arr(X, np.float64)
    r, rp, _ = _arr(R, np.float64)
    a, ap, n = _arr(A, np.float64)
    ldv = a.size if ldv is None else ldv
    VGL = np.zeros((5, max(ldv, 0)), dtype=np.float64)
    _check(lib().qmckl_ao_gaussian_vgl(C.c_int64(ctx), xp, rp, n, ap, VGL.ctypes.data_as(C.c_void_p),
                                       C.c_int64(ldv)))
    return VGL


def _polynomial(cname, transposed):
    def f(ctx, X, R, lmax, ldl=3, ldv=None):
        x, xp, _ = _arr(X, np.float64)
        r, rp, _ = _arr(R, np.float64)
        npoly = max(lmax + 1, 0) * (lmax + 2) * (lmax + 3) // 6
        if ldv is None:
            ldv = npoly if transposed else 5
        L = np.zeros((max(npoly, 1), max(ldl, 0)), dtype=np.int32)
        VGL = np.zeros((5, max(ldv, 0)) if transposed else (max(npoly, 1), max(ldv, 0)), dtype=np.float64)
        n = C.c_int64(0)
        _check(getattr(lib(), cname)(C.c_int64(ctx), xp, rp, C.c_int32(lmax), C.byref(n),
                                     L.ctypes.data_as(C.c_void_p), C.c_int64(ldl),
                                     VGL.ctypes.data_as(C.c_void_p), C.c_int64(ldv)))
        return n.value, L, VGL
    f.__name__ = cname[len("qmckl_"):]
    f.__doc__ = (f"{cname}: (n, L[n][ldl], VGL) with VGL[5][ldv] (monomial m in column m)" if transposed else
                 f"{cname}: (n, L[n][ldl], VGL) with VGL[n][ldv] (component c in column c)")
    return f


ao_polynomial_vgl = _polynomial("qmckl_ao_polynomial_vgl", False)
ao_polynomial_vgl_doc = _polynomial("qmckl_ao_polynomial_vgl_doc", False)
ao_polynomial_transp_vgl = _polynomial("qmckl_ao_polynomial_transp_vgl", True)
ao_polynomial_transp_vgl_doc = _polynomial("qmckl_ao_polynomial_transp_vgl_doc", True)
ao_polynomial_transp_vgl_hpc = _polynomial("qmckl_ao_polynomial_transp_vgl_hpc", True)

# ------------------------------------------------------------- MO basis


def set_mo_basis_mo_num(ctx, n):
    _call("qmckl_set_mo_basis_mo_num", ctx, C.c_int64(n))


def get_mo_basis_mo_num(ctx):
    v = C.c_int64()
    _call("qmckl_get_mo_basis_mo_num", ctx, C.byref(v))
    return v.value


def set_mo_basis_coefficient(ctx, coef):
    a, p, n = _arr(coef, np.float64)
    _call("qmckl_set_mo_basis_coefficient", ctx, p, n)


def get_mo_basis_coefficient(ctx, size_max):
    out = np.zeros(size_max, dtype=np.float64)
    _call("qmckl_get_mo_basis_coefficient", ctx, out.ctypes.data_as(C.c_void_p), C.c_int64(size_max))
    return out


def mo_basis_provided(ctx):
    return bool(lib().qmckl_mo_basis_provided(C.c_int64(ctx)))


def mo_basis_select_mo(ctx, keep):
    a, p, n = _arr(keep, np.int32)
    _call("qmckl_mo_basis_select_mo", ctx, p, n)


def mo_basis_rescale(ctx, factor):
    _call("qmckl_mo_basis_rescale", ctx, C.c_double(factor))


def b200_get_kblock_stats(ctx, reset=False):
    """(issued, dense) 16-AO k-steps of the fused kernel's launches since the last reset."""
    ev, tot = C.c_int64(0), C.c_int64(0)
    _call("qmckl_b200_get_kblock_stats", ctx, C.byref(ev), C.byref(tot), C.c_int32(1 if reset else 0))
    return ev.value, tot.value


def trexio_read(ctx, file_name):
    """qmckl_trexio_read: electrons, nuclei, AO basis and MO coefficients of a
    TREXIO text-backend directory into the context (RuntimeError otherwise)."""
    b = file_name.encode()
    _call("qmckl_trexio_read", ctx, C.c_char_p(b), C.c_int64(len(b)))


def set_mo_basis_r_cusp(ctx, r_cusp):
    a, p, n = _arr(r_cusp, np.float64)
    _call("qmckl_set_mo_basis_r_cusp", ctx, p, n)


get_mo_basis_mo_vgl = _array_getter("qmckl_get_mo_basis_mo_vgl")
get_mo_basis_mo_vgl_inplace = _array_getter("qmckl_get_mo_basis_mo_vgl_inplace")
get_mo_basis_mo_value = _array_getter("qmckl_get_mo_basis_mo_value")
get_mo_basis_mo_value_inplace = _array_getter("qmckl_get_mo_basis_mo_value_inplace")
get_mo_basis_mo_hessian = _array_getter("qmckl_get_mo_basis_mo_hessian")
get_electron_en_distance = _array_getter("qmckl_get_electron_en_distance")

# -------------------------------------------------- B200 extensions

FORM_AUTO, FORM_FP64, FORM_MIXED = 0, 1, 2


def b200_set_form(ctx, form):
    _call("qmckl_b200_set_form", ctx, C.c_int32(form))


def b200_get_form(ctx):
    v = C.c_int32()
    _call("qmckl_b200_get_form", ctx, C.byref(v))
    return v.value


def b200_set_split_terms(ctx, pieces):
    _call("qmckl_b200_set_split_terms", ctx, C.c_int32(pieces))


def b200_set_mixed_kernel(ctx, fused):
    _call("qmckl_b200_set_mixed_kernel", ctx, C.c_int32(1 if fused else 0))


def b200_set_stream(ctx, stream_ptr):
    _call("qmckl_b200_set_stream", ctx, C.c_void_p(stream_ptr))


def b200_synchronize(ctx):
    _call("qmckl_b200_synchronize", ctx)


def _device_entry(cname):
    def f(ctx, point_num, d_coord_ptr, d_out_ptr):
        _call(cname, ctx, C.c_int64(point_num), C.c_void_p(d_coord_ptr), C.c_void_p(d_out_ptr))
    f.__name__ = cname[len("qmckl_"):]
    return f


b200_ao_vgl_device = _device_entry("qmckl_b200_ao_vgl_device")
b200_ao_value_device = _device_entry("qmckl_b200_ao_value_device")
b200_mo_vgl_device = _device_entry("qmckl_b200_mo_vgl_device")
b200_mo_value_device = _device_entry("qmckl_b200_mo_value_device")
b200_ao_hessian_device = _device_entry("qmckl_b200_ao_hessian_device")


def b200_mo_vgl_adjoint_device(ctx, point_num, d_coord_ptr, d_weight_ptr, d_grad_coef_ptr=0, d_grad_nucl_ptr=0,
                               d_grad_coord_ptr=0):
    """Gradient of sum(weight * mo_vgl); pointers of device buffers, 0 for an output not wanted."""
    _call("qmckl_b200_mo_vgl_adjoint_device", ctx, C.c_int64(point_num), C.c_void_p(d_coord_ptr),
          C.c_void_p(d_weight_ptr), C.c_void_p(d_grad_coef_ptr or None), C.c_void_p(d_grad_nucl_ptr or None),
          C.c_void_p(d_grad_coord_ptr or None))


def b200_kernel_launch_count():
    return int(lib().qmckl_b200_kernel_launch_count())


def b200_inject_alloc_failure(n):
    lib().qmckl_b200_inject_alloc_failure(C.c_int64(n))


def b200_get_fused_plan(ao_num, mo_num, pieces=3):
    """(n_tile, n_tiles, accumulators, stages) of the fused kernel's MO tiling."""
    v = [C.c_int32() for _ in range(4)]
    f = lib().qmckl_b200_get_fused_plan
    f.restype = C.c_int32
    _check(f(C.c_int64(ao_num), C.c_int64(mo_num), C.c_int32(pieces), *[C.byref(x) for x in v]))
    return tuple(x.value for x in v)


def b200_inject_late_warps(ns):
    f = lib().qmckl_b200_inject_late_warps
    f.restype = C.c_int32
    _check(f(C.c_int64(ns)))


def b200_inject_wait_failure(ctx, code):
    """Test hook: mark the context's tensor-core error word as a bounded wait that gave up."""
    _call("qmckl_b200_inject_wait_failure", ctx, C.c_int32(code))


# ------------------------------------------------------ batched systems


def _bcall(name, *args, ctx=None):
    f = getattr(lib(), name)
    f.restype = C.c_int32
    _check(f(*args), ctx)


def b200_batch_create(contexts, point_num):
    """One batch over `contexts` with point_num[s] points for system s; returns the handle."""
    ctxs = np.ascontiguousarray(contexts, dtype=np.int64)
    pn = np.ascontiguousarray(point_num, dtype=np.int64)
    if ctxs.size != pn.size:
        raise ValueError("one point count per context")
    h = C.c_int64(0)
    _bcall("qmckl_b200_batch_create", ctxs.ctypes.data_as(C.c_void_p), pn.ctypes.data_as(C.c_void_p),
           C.c_int64(ctxs.size), C.byref(h), ctx=int(ctxs[0]) if ctxs.size else None)
    return h.value


def b200_batch_destroy(batch):
    _bcall("qmckl_b200_batch_destroy", C.c_int64(batch))


def b200_batch_layout(batch, num):
    """(coord_offset[num], out_offset[num], (coord_total, out_total)) in doubles."""
    co = np.zeros(num, dtype=np.int64)
    oo = np.zeros(num, dtype=np.int64)
    tot = np.zeros(2, dtype=np.int64)
    _bcall("qmckl_b200_batch_layout", C.c_int64(batch), co.ctypes.data_as(C.c_void_p),
           oo.ctypes.data_as(C.c_void_p), tot.ctypes.data_as(C.c_void_p))
    return co, oo, (int(tot[0]), int(tot[1]))


def b200_batch_set_stream(batch, stream_ptr):
    _bcall("qmckl_b200_batch_set_stream", C.c_int64(batch), C.c_void_p(stream_ptr))


def b200_batch_set_graph(batch, enable):
    _bcall("qmckl_b200_batch_set_graph", C.c_int64(batch), C.c_int32(1 if enable else 0))


def b200_batch_mo_vgl_device(batch, d_coord_ptr, d_out_ptr):
    _bcall("qmckl_b200_batch_mo_vgl_device", C.c_int64(batch), C.c_void_p(d_coord_ptr), C.c_void_p(d_out_ptr))


def b200_batch_mo_vgl_loop_device(batch, d_coord_ptr, d_out_ptr):
    _bcall("qmckl_b200_batch_mo_vgl_loop_device", C.c_int64(batch), C.c_void_p(d_coord_ptr), C.c_void_p(d_out_ptr))


def b200_batch_synchronize(batch, raise_on_error=True):
    """Wait for the batch; returns the launch's error word (0 = success)."""
    st = C.c_int32(0)
    f = lib().qmckl_b200_batch_synchronize
    f.restype = C.c_int32
    rc = f(C.c_int64(batch), C.byref(st))
    if rc != 0 and raise_on_error:
        _check(rc)
    return st.value


def b200_batch_tune(batch, d_coord_ptr, d_out_ptr, reps=3):
    best = C.c_double(0.0)
    _bcall("qmckl_b200_batch_tune", C.c_int64(batch), C.c_void_p(d_coord_ptr), C.c_void_p(d_out_ptr),
           C.c_int32(reps), C.byref(best))
    return best.value


def b200_batch_set_tuning(batch, producer_warps, order):
    _bcall("qmckl_b200_batch_set_tuning", C.c_int64(batch), C.c_int32(producer_warps), C.c_int32(order))


def b200_batch_get_tuning(batch):
    pw, od = C.c_int32(0), C.c_int32(0)
    _bcall("qmckl_b200_batch_get_tuning", C.c_int64(batch), C.byref(pw), C.byref(od))
    return pw.value, od.value


def b200_batch_set_wait_limit(batch, polls, publish=True):
    _bcall("qmckl_b200_batch_set_wait_limit", C.c_int64(batch), C.c_int64(polls), C.c_int32(1 if publish else 0))
