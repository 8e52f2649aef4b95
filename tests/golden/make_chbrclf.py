#!/usr/bin/env python3
"""Build tests/golden/chbrclf.npz from the reference's CHBrClF test fixture.

Reads, as text, the reference's C fixture header ``include/chbrclf.h``
(CHBrClF / aug-cc-pVTZ: 5 nuclei, 72 shells, 297 primitives, 263 cartesian
AOs, 224 MOs, 68 electrons x 2 walkers) and the golden values asserted by the
reference's own unit tests in ``org/qmckl_ao.org`` (primitive_vgl 4697-4712,
shell_vgl 5248-5252, ao_vgl 9355-9384, ao_value 8399-8405).  The result is a
small numpy archive that the tests read on any machine; the reference tree is
only needed to regenerate it:

    python tests/golden/make_chbrclf.py /path/to/qmckl
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _c_array(text, name):
    m = re.search(r"\b" + re.escape(name) + r"\s*\[[^=]*=\s*\{", text)
    if m is None:
        raise KeyError(name)
    depth, i = 1, m.end()
    while depth:
        ch = text[i]
        depth += ch == "{"
        depth -= ch == "}"
        i += 1
    body = text[m.end():i - 1].replace("{", " ").replace("}", " ")
    body = re.sub(r"//[^\n]*", " ", body)
    return [t for t in (s.strip() for s in body.split(",")) if t]


def _floats(text, name):
    return np.array([float(t) for t in _c_array(text, name)], dtype=np.float64)


def _ints(text, name, dtype):
    return np.array([int(t) for t in _c_array(text, name)], dtype=dtype)


def _asserts(org, array):
    """All `assert( fabs(<array>[i][j]...[k] - (value)) < tol )` lines."""
    pat = re.compile(r"assert\(\s*fabs\(\s*" + array + r"((?:\[\d+\])+)\s*-\s*\(\s*([-+0-9.eE]+)\s*\)\)\s*<\s*([0-9.eE+-]+)\s*\)")
    out = []
    for m in pat.finditer(org):
        idx = tuple(int(t) for t in re.findall(r"\d+", m.group(1)))
        out.append((idx, float(m.group(2)), float(m.group(3))))
    return out


def main(ref_root):
    hdr = open(os.path.join(ref_root, "include", "chbrclf.h")).read()
    org = open(os.path.join(ref_root, "org", "qmckl_ao.org")).read()
    d = {}
    d["charge"] = _floats(hdr, "chbrclf_charge")
    d["nucl_coord"] = _floats(hdr, "chbrclf_nucl_coord").reshape(3, -1)          # [3][nucl]
    d["nucleus_index"] = _ints(hdr, "chbrclf_basis_nucleus_index", np.int64)
    d["nucleus_shell_num"] = _ints(hdr, "chbrclf_basis_nucleus_shell_num", np.int64)
    d["shell_ang_mom"] = _ints(hdr, "chbrclf_basis_shell_ang_mom", np.int32)
    d["shell_prim_num"] = _ints(hdr, "chbrclf_basis_shell_prim_num", np.int64)
    d["shell_prim_index"] = _ints(hdr, "chbrclf_basis_shell_prim_index", np.int64)
    d["shell_factor"] = _floats(hdr, "chbrclf_basis_shell_factor")
    d["ao_factor"] = _floats(hdr, "chbrclf_basis_ao_factor")
    d["exponent"] = _floats(hdr, "chbrclf_basis_exponent")
    d["coefficient"] = _floats(hdr, "chbrclf_basis_coefficient")
    d["prim_factor"] = _floats(hdr, "chbrclf_basis_prim_factor")
    mo = _floats(hdr, "chbrclf_mo_coef")
    ao_num = d["ao_factor"].size
    d["mo_coef"] = mo.reshape(-1, ao_num)                                          # [mo][ao]
    d["elec_coord"] = _floats(hdr, "chbrclf_elec_coord").reshape(2, 68, 3)        # [walk][elec][3]
    d["elec_up_num"] = np.array(34, dtype=np.int64)
    d["elec_dn_num"] = np.array(34, dtype=np.int64)
    for name in ("prim_vgl", "shell_vgl", "ao_vgl", "ao_value"):
        rows = _asserts(org, name)
        if not rows:
            raise RuntimeError(f"no golden asserts found for {name}")
        d[f"golden_{name}_index"] = np.array([r[0] for r in rows], dtype=np.int64)
        d[f"golden_{name}_value"] = np.array([r[1] for r in rows], dtype=np.float64)
        d[f"golden_{name}_tol"] = np.array([r[2] for r in rows], dtype=np.float64)
    out = os.path.join(HERE, "chbrclf.npz")
    np.savez_compressed(out, **d)
    print("wrote", out, {k: v.shape for k, v in d.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_chbrclf.py <reference source root>")
    main(sys.argv[1])
