"""Seeded synthetic molecules for the orbital-evaluation workloads.

Every workload is generated from numpy's default_rng(seed) with
seed = 20260000 + config id, so the same inputs are produced on any machine.
There is no public dataset behind these workloads; the shapes follow the
benchmark definitions:

  0  small molecule: 4 C + 6 H in an 8-bohr cube, C 3s2p1d / H 2s1p
     (90 AOs), 90 MOs, 30 electrons x 64 walkers (1,920 points)
  1  mid-size: 40 heavy (Z in {6,7,8}) + 40 H in a 20-bohr cube,
     cc-pVTZ-shaped cartesian basis (heavy 4s3p2d1f = 35 AOs, H 3s2p1d = 15),
     2,000 AOs, 160 MOs, ~320 electrons x 512 walkers
  2  batch: 256 systems, 5..80 nuclei, DZ or TZ shape, MOs = electrons/2,
     16..256 walkers
  3  adjoint: the config-1 molecule with 128 walkers
  4  large: 100 heavy + 100 H in a 32-bohr cube, TZ shape (5,000 AOs),
     350 MOs, 700 electrons x 256 walkers (179,200 points)

Basis conventions (all cartesian, Gaussian):
  * nuclei placed uniformly, rejecting any pair closer than 1.8 bohr;
  * the first s shell of a heavy atom has 8 primitives, other shells 1-3;
  * exponents log-uniform in [0.1, 5000] (heavy) or [0.1, 50] (H);
  * contraction coefficients N(0,1), rescaled so each contracted shell is
    normalised; prim_factor is the normalisation of a primitive of angular
    momentum l, shell_factor = 1, ao_factor = 1/sqrt((2a-1)!!(2b-1)!!(2c-1)!!/(2l-1)!!);
  * MO coefficients: Q of the QR factorisation of a Gaussian ao_num x mo_num;
  * electrons: count = sum of Z, each assigned to a nucleus with probability
    proportional to Z and displaced by N(0, 1 bohr) per axis, per walker; the
    points are ordered walker by walker, up-spin electrons first.
"""
import math

import numpy as np

SHAPES = {
    "c0_heavy": [0, 0, 0, 1, 1, 2],
    "c0_h": [0, 0, 1],
    "dz_heavy": [0, 0, 0, 1, 1, 2],
    "dz_h": [0, 0, 1],
    "tz_heavy": [0, 0, 0, 0, 1, 1, 1, 2, 2, 3],
    "tz_h": [0, 0, 0, 1, 1, 2],
    # high angular momentum: g, h shells on one kind of atom, g, i, k on the other
    "hl_a": [0, 0, 1, 2, 3, 4, 5],
    "hl_b": [0, 1, 2, 4, 6, 7],
}


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def ncart(l):
    return (l + 1) * (l + 2) // 2


def place_nuclei(rng, n, side, min_sep=1.8, max_tries=200000):
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place nuclei with the requested separation")
        p = rng.uniform(0.0, side, size=3)
        if all(np.linalg.norm(p - q) >= min_sep for q in pts):
            pts.append(p)
    return np.array(pts)


def prim_norm(a, l):
    """Normalisation of x^l exp(-a r^2) (axis-aligned component)."""
    return (2.0 * a / math.pi) ** 0.75 * (4.0 * a) ** (l / 2.0) / math.sqrt(_dfact(2 * l - 1))


def _shell(rng, l, heavy, first_s):
    nprim = 8 if (heavy and first_s) else int(rng.integers(1, 4))
    hi = 5000.0 if heavy else 50.0
    expo = np.exp(rng.uniform(math.log(0.1), math.log(hi), size=nprim))
    coef = rng.standard_normal(nprim)
    pf = np.array([prim_norm(a, l) for a in expo])
    # overlap of normalised primitives of equal l on one centre
    s = np.empty((nprim, nprim))
    for i in range(nprim):
        for j in range(nprim):
            s[i, j] = (2.0 * math.sqrt(expo[i] * expo[j]) / (expo[i] + expo[j])) ** (l + 1.5)
    norm2 = coef @ s @ coef
    coef = coef / math.sqrt(norm2)
    return expo, coef, pf


def build_system(rng, charges, coords, shape_heavy, shape_h, mo_num, walk_num, elec_num=None, shapes=None):
    """Assemble every array of the qmckl setters for one molecule (shapes:
    optional list of shell angular momenta per nucleus, replacing the
    heavy / H shapes)."""
    nucl_num = len(charges)
    nucleus_index, nucleus_shell_num = [], []
    shell_ang_mom, shell_prim_num, shell_prim_index = [], [], []
    exponent, coefficient, prim_factor, ao_factor = [], [], [], []
    for n, z in enumerate(charges):
        heavy = z > 1
        shape = shapes[n] if shapes is not None else (shape_heavy if heavy else shape_h)
        nucleus_index.append(len(shell_ang_mom))
        nucleus_shell_num.append(len(shape))
        first_s = True
        for l in shape:
            expo, coef, pf = _shell(rng, l, heavy, first_s and l == 0)
            if l == 0:
                first_s = False
            shell_ang_mom.append(l)
            shell_prim_index.append(len(exponent))
            shell_prim_num.append(len(expo))
            exponent += list(expo)
            coefficient += list(coef)
            prim_factor += list(pf)
            for a in range(l, -1, -1):
                for b in range(l - a, -1, -1):
                    c = l - a - b
                    ao_factor.append(1.0 / math.sqrt(_dfact(2 * a - 1) * _dfact(2 * b - 1) * _dfact(2 * c - 1)
                                                     / _dfact(2 * l - 1)))
    ao_num = len(ao_factor)
    mo_num = min(mo_num, ao_num)
    q, _ = np.linalg.qr(rng.standard_normal((ao_num, mo_num)))
    mo_coef = np.ascontiguousarray(q.T)                       # [mo][ao]
    zsum = int(round(sum(charges)))
    if elec_num is None:
        elec_num = zsum
    up = (elec_num + 1) // 2
    dn = elec_num - up
    prob = np.asarray(charges, dtype=np.float64) / sum(charges)
    owner = rng.choice(nucl_num, size=(walk_num, elec_num), p=prob)
    elec = coords[owner] + rng.standard_normal((walk_num, elec_num, 3))
    return {
        "nucl_num": nucl_num,
        "charge": np.asarray(charges, dtype=np.float64),
        "nucl_coord": np.ascontiguousarray(coords.T),              # [3][nucl]
        "nucleus_index": np.array(nucleus_index, dtype=np.int64),
        "nucleus_shell_num": np.array(nucleus_shell_num, dtype=np.int64),
        "shell_ang_mom": np.array(shell_ang_mom, dtype=np.int32),
        "shell_prim_num": np.array(shell_prim_num, dtype=np.int64),
        "shell_prim_index": np.array(shell_prim_index, dtype=np.int64),
        "shell_factor": np.ones(len(shell_ang_mom), dtype=np.float64),
        "exponent": np.array(exponent, dtype=np.float64),
        "coefficient": np.array(coefficient, dtype=np.float64),
        "prim_factor": np.array(prim_factor, dtype=np.float64),
        "ao_factor": np.array(ao_factor, dtype=np.float64),
        "ao_num": ao_num,
        "mo_num": mo_num,
        "mo_coef": mo_coef,
        "elec_up_num": up,
        "elec_dn_num": dn,
        "walk_num": walk_num,
        "elec_coord": elec,                                         # [walk][elec][3]
    }


def config(cid, walk_num=None, seed=None):
    """One of the benchmark molecules (cid 0, 1, 3, 4); see the module docstring."""
    rng = np.random.default_rng(20260000 + cid if seed is None else seed)
    if cid == 0:
        charges = [6.0] * 4 + [1.0] * 6
        coords = place_nuclei(rng, 10, 8.0)
        return build_system(rng, charges, coords, SHAPES["c0_heavy"], SHAPES["c0_h"], 90,
                            walk_num or 64)
    if cid in (1, 3):
        rng = np.random.default_rng(20260001 if seed is None else seed)   # config 3 reuses the config-1 molecule
        charges = list(rng.choice([6.0, 7.0, 8.0], size=40)) + [1.0] * 40
        coords = place_nuclei(rng, 80, 20.0)
        return build_system(rng, charges, coords, SHAPES["tz_heavy"], SHAPES["tz_h"], 160,
                            walk_num or (512 if cid == 1 else 128))
    if cid == 4:
        charges = list(rng.choice([6.0, 7.0, 8.0], size=100)) + [1.0] * 100
        coords = place_nuclei(rng, 200, 32.0)
        return build_system(rng, charges, coords, SHAPES["tz_heavy"], SHAPES["tz_h"], 350,
                            walk_num or 256, elec_num=700)
    raise ValueError(f"no single-molecule config {cid}")


def high_l_config(walk_num=16, seed=20260007):
    """A small molecule whose basis reaches l = 7: 3 atoms (Z = 6) with
    s s p d f g h shells (57 AOs each) and 3 atoms (Z = 8) with s p d g i k
    shells (89 AOs each) in a 6-bohr cube; 438 AOs, 120 MOs, 42 electrons."""
    rng = np.random.default_rng(seed)
    charges = [6.0, 8.0, 6.0, 8.0, 6.0, 8.0]
    coords = place_nuclei(rng, 6, 6.0)
    nucleus_shapes = [SHAPES["hl_a"] if z == 6.0 else SHAPES["hl_b"] for z in charges]
    return build_system(rng, charges, coords, None, None, 120, walk_num, shapes=nucleus_shapes)


def batch_config(num_systems=256, seed=20260002, max_walkers=256):
    """Config 2: many independent molecules of uneven size."""
    rng = np.random.default_rng(seed)
    systems = []
    for _ in range(num_systems):
        nn = int(rng.integers(5, 81))
        nh = nn // 2
        charges = list(rng.choice([6.0, 7.0, 8.0], size=nn - nh)) + [1.0] * nh
        side = 8.0 * (nn / 10.0) ** (1.0 / 3.0)
        coords = place_nuclei(rng, nn, side)
        tz = bool(rng.integers(0, 2))
        sh = (SHAPES["tz_heavy"], SHAPES["tz_h"]) if tz else (SHAPES["dz_heavy"], SHAPES["dz_h"])
        ne = int(round(sum(charges)))
        walkers = int(rng.integers(16, max_walkers + 1))
        systems.append(build_system(rng, charges, coords, sh[0], sh[1], max(1, ne // 2), walkers))
    return systems


def points(sysd):
    """Electron coordinates as points [P][3] (walker-major, reference order)."""
    return np.ascontiguousarray(sysd["elec_coord"].reshape(-1, 3))


def chbrclf(path):
    """The reference's CHBrClF fixture (tests/golden/chbrclf.npz) as a system dict."""
    d = dict(np.load(path))
    d["nucl_num"] = int(d["nucleus_index"].size)
    d["ao_num"] = int(d["ao_factor"].size)
    d["mo_num"] = int(d["mo_coef"].shape[0])
    d["walk_num"] = int(d["elec_coord"].shape[0])
    d["elec_up_num"] = int(d["elec_up_num"])
    d["elec_dn_num"] = int(d["elec_dn_num"])
    return d
