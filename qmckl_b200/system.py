"""Load a system dict (qmckl_b200.gen) into a context through the qmckl API.

The call sequence is the reference's own test set-up sequence
(org/qmckl_ao.org:2459-2545, org/qmckl_mo.org:3620-3700).
"""
import numpy as np

from . import qmckl as pq


def make_context(sysd, points=True, form=None, precision=None):
    ctx = pq.context_create()
    if precision is not None:
        pq.set_numprec_precision(ctx, precision)
    if form is not None:
        pq.b200_set_form(ctx, form)
    n = int(sysd["nucl_num"])
    pq.set_nucleus_num(ctx, n)
    pq.set_nucleus_coord(ctx, "T", np.asarray(sysd["nucl_coord"]).reshape(-1))
    pq.set_nucleus_charge(ctx, sysd["charge"])
    pq.set_ao_basis_type(ctx, "G")
    pq.set_ao_basis_shell_num(ctx, int(sysd["shell_ang_mom"].size))
    pq.set_ao_basis_prim_num(ctx, int(sysd["exponent"].size))
    pq.set_ao_basis_nucleus_index(ctx, sysd["nucleus_index"])
    pq.set_ao_basis_nucleus_shell_num(ctx, sysd["nucleus_shell_num"])
    pq.set_ao_basis_shell_ang_mom(ctx, sysd["shell_ang_mom"])
    pq.set_ao_basis_shell_factor(ctx, sysd["shell_factor"])
    pq.set_ao_basis_shell_prim_num(ctx, sysd["shell_prim_num"])
    pq.set_ao_basis_shell_prim_index(ctx, sysd["shell_prim_index"])
    pq.set_ao_basis_exponent(ctx, sysd["exponent"])
    pq.set_ao_basis_coefficient(ctx, sysd["coefficient"])
    pq.set_ao_basis_prim_factor(ctx, sysd["prim_factor"])
    pq.set_ao_basis_ao_num(ctx, int(sysd["ao_factor"].size))
    pq.set_ao_basis_ao_factor(ctx, sysd["ao_factor"])
    pq.set_mo_basis_mo_num(ctx, int(sysd["mo_coef"].shape[0]))
    pq.set_mo_basis_coefficient(ctx, np.asarray(sysd["mo_coef"]).reshape(-1))
    if points:
        pq.set_electron_num(ctx, int(sysd["elec_up_num"]), int(sysd["elec_dn_num"]))
        walk = int(sysd["elec_coord"].shape[0])
        pq.set_electron_coord(ctx, "N", walk, np.asarray(sysd["elec_coord"]).reshape(-1))
    return ctx
