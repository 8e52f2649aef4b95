"""Build recipe: the reference's own C kernels of the orbital path, compiled
from its sources into oracle/_ref/libqmckl_ref.so (test infrastructure only).

    python -m oracle.build_ref [REFERENCE_ROOT]

The reference keeps its C code inside literate org files (org/*.org, blocks
``#+begin_src c ... :tangle (eval c)``) and tangles them with emacs, which is
not installed here.  This recipe is a minimal tangler: it takes, verbatim,
the C blocks that define the functions listed in WANTED, expands their noweb
references (``<<name>>`` -> the block named ``#+NAME: name``), and compiles
them with gcc against ``oracle/ref_shim.h`` / ``oracle/ref_shim.c``, a small
stand-in for the parts of the reference's context, memory and matrix modules
those functions touch.  The extracted source and the library are written to
oracle/_ref/ only (git-ignored); nothing of the reference is committed.

The reference root comes from the argument, else $QMCKL_REFERENCE_ROOT, else
/root/reference; without it the recipe does nothing.  Flags: -O3, HAVE_HPC and
HAVE_OPENMP (the reference's production configuration), x86-64-v3 so that the
library built here also runs on the GPU host, and no contraction of a*b+c
into fused multiply-adds (-ffp-contract=off: the reference's default build
for x86-64 has no FMA instructions, and the oracle is built the same way, so
that the two agree to the last bit).
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libqmckl_ref.so")
SRC = os.path.join(OUT_DIR, "qmckl_ref_extracted.c")
DEFAULT_ROOT = "/root/reference"

# (org file, function defined in the block) -- the reference's HPC path of
# AO VGL / AO value and MO VGL / MO value, and the basis finalization
WANTED = [
    ("org/qmckl_ao.org", "qmckl_finalize_basis"),
    ("org/qmckl_ao.org", "qmckl_finalize_basis_hpc"),
    ("org/qmckl_ao.org", "qmckl_ao_polynomial_transp_vgl_hpc_inline"),
    ("org/qmckl_ao.org", "qmckl_compute_ao_vgl_hpc_gaussian"),
    ("org/qmckl_ao.org", "qmckl_compute_ao_value_hpc_gaussian"),
    ("org/qmckl_mo.org", "qmckl_compute_mo_basis_mo_vgl_hpc"),
    ("org/qmckl_mo.org", "qmckl_compute_mo_basis_mo_vgl_hpc_sp"),
    ("org/qmckl_mo.org", "qmckl_compute_mo_basis_mo_value_hpc"),
    ("org/qmckl_mo.org", "qmckl_compute_mo_basis_mo_value_hpc_sp"),
]

_BEGIN = re.compile(r"^\s*#\+begin_src\s+(\S+)(.*)$", re.IGNORECASE)
_END = re.compile(r"^\s*#\+end_src\s*$", re.IGNORECASE)
_NAME = re.compile(r"^\s*#\+NAME:\s*(\S+)\s*$", re.IGNORECASE)
_NOWEB = re.compile(r"^(\s*)<<([^>\s]+)>>\s*$")
# org escapes a line of a source block that starts with "*" or "#+" (after
# optional blanks) by a leading comma; tangling removes it
_ESCAPED = re.compile(r"^(\s*),(?=\*|#\+|,\*|,#\+)")


def org_blocks(path):
    """[(language, header, name or None, text, first line number)] of an org file."""
    blocks = []
    lines = open(path, encoding="utf-8").read().split("\n")
    name = None
    i = 0
    while i < len(lines):
        m = _NAME.match(lines[i])
        if m:
            name = m.group(1)
            i += 1
            continue
        m = _BEGIN.match(lines[i])
        if m:
            j = i + 1
            while j < len(lines) and not _END.match(lines[j]):
                j += 1
            body = [_ESCAPED.sub(r"\1", line) for line in lines[i + 1:j]]
            blocks.append((m.group(1).lower(), m.group(2), name, "\n".join(body), i + 2))
            name = None
            i = j + 1
            continue
        if lines[i].strip():
            name = None
        i += 1
    return blocks


def expand(text, named, depth=0):
    if depth > 8:
        raise RuntimeError("noweb references nest too deeply")
    out = []
    for line in text.split("\n"):
        m = _NOWEB.match(line)
        if m and m.group(2) in named:
            out.append(expand(named[m.group(2)], named, depth + 1))
        else:
            out.append(line)
    return "\n".join(out)


def _defines(text, fn):
    return re.search(r"\b" + re.escape(fn) + r"\s*\(([^;{}]*)\)\s*\{", text, re.DOTALL) is not None


def extract(root):
    """The C source of the WANTED functions, in their org order, noweb expanded."""
    pieces = []
    by_file = {}
    for org, fn in WANTED:
        by_file.setdefault(org, []).append(fn)
    for org, fns in by_file.items():
        path = os.path.join(root, org)
        blocks = org_blocks(path)
        named = {b[2]: b[3] for b in blocks if b[2]}
        taken = set()
        for fn in fns:
            hits = [k for k, b in enumerate(blocks)
                    if b[0] == "c" and "(eval c)" in b[1] and _defines(b[3], fn)]
            if len(hits) != 1:
                raise RuntimeError(f"{org}: {len(hits)} C blocks define {fn}")
            taken.add(hits[0])
        for k in sorted(taken):
            lang, header, name, text, line = blocks[k]
            pieces.append(f"/* ---- {org}:{line} */\n" + expand(text, named))
    return "\n\n".join(pieces) + "\n"


def build(root=None, force=False, verbose=False):
    root = root or os.environ.get("QMCKL_REFERENCE_ROOT") or DEFAULT_ROOT
    if not os.path.isdir(os.path.join(root, "org")):
        if verbose:
            print(f"oracle/_ref: no reference sources at {root}; skipped")
        return None
    deps = [os.path.join(HERE, f) for f in ("ref_shim.h", "ref_shim.c", "build_ref.py")]
    deps += [os.path.join(root, org) for org, _ in WANTED]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    src = '#include "ref_shim.h"\n\n' + extract(root)
    with open(SRC, "w") as f:
        f.write(src)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=gnu11",
           "-DHAVE_HPC",
           "-DHAVE_OPENMP", "-I" + HERE, SRC, os.path.join(HERE, "ref_shim.c"), "-o", LIB, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else None, force=True, verbose=True))
