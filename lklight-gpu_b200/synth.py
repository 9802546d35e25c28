"""Synthetic complexes and setup poses for the benchmark configurations.

The reference measures on PDB systems that are not shipped (an RNA complex,
1AZP); these seeded generators stand in for them with the shapes, sizes and
value distributions of the five benchmark configurations:

* receptor: self-avoiding random chain (1.5 A bonds, >= 3.0 A from atoms more
  than two bonds back) confined to a sphere that starts at 30 A and grows by
  0.5 A when the chain end is stuck at the boundary (``lkg_synth_chain``);
  AMBER types drawn uniformly from the DNA family's 54-type vdW table
  (src/dna.rs:88-105), heavy = type name does not start with 'H'
  (src/dna.rs:397); charges U[-0.8, 0.8] shifted so the net charge is +10.
* ligand: B-DNA-like duplex (rise 3.38 A, 36 deg per base pair, phosphates at
  ~8.9 A) whose pseudo-atoms carry the DA/DC/DG/DT atom names and AMBER types
  (src/dna.rs:117-132); q = -1 on each P, 0 elsewhere.
* both centred at their centre of mass and rounded to f32, as LKlight's setup
  centres them (src/bin/lightdock.rs:443-445) and the configs ask for fp32.
* poses: ``setup_poses`` reproduces ``LKlight setup`` (src/bin/lightdock.rs:
  396-548): Fibonacci-sphere swarm centres at avg_r(receptor) + 3 A,
  +-1 A jitter and a random quaternion per glowworm from StdRng(seed), written
  with 6 decimals.

Random streams: the chain uses std::mt19937_64(seed) in C++; types, charges
and sequences use numpy's PCG64(seed); poses use the reference's StdRng.

``gen``: the generators of the chain and of StdRng.  None uses liblkg's
(``lkg_synth_chain``, ``lkg_rng_*``); a caller that must not load the library
passes an object with the same ``chain(n, seed, r0=...)`` and ``Rng(seed)``
(the benchmark's CPU reference arm passes the oracle's).
"""
import functools
import json
import math
import os

import numpy as np

from . import C, _check, lib, lr_sasa, ptr, Rng

HERE = os.path.dirname(os.path.abspath(__file__))


@functools.lru_cache(maxsize=1)
def tables():
    with open(os.path.join(HERE, "data", "amber_types.json")) as f:
        return json.load(f)


# cpydock desolvation coefficient by AMBER type, the fallback branch of
# des_energy (src/cpydock.rs:123-134), and radius_per_asp (src/cpydock.rs:59-70)
_DES = {}
for names, v in ((("CT", "C", "CD", "CZ", "CY"), 0.01918),
                 (("CA", "CB", "CC", "CK", "CM", "CN", "CQ", "CR", "CV", "CW", "C*"), 0.1108),
                 (("N", "N*", "NA", "NB", "NC", "NY", "NT", "N2"), -0.0391), (("N3",), -0.12604),
                 (("O",), -0.03128), (("O2", "O3"), -0.06877), (("OH", "OW", "OS"), -0.04255),
                 (("S",), 0.00506), (("SH",), 0.02576)):
    for n in names:
        _DES[n] = v
_RASP = {}
for names, v in ((("C", "CD", "CT", "CY", "CZ"), 1.95),
                 (("C*", "CA", "CB", "CC", "CK", "CM", "CN", "CQ", "CR", "CV", "CW"), 1.8),
                 (("N", "N*", "N2", "N3", "NA", "NB", "NC", "NT", "NY"), 1.7), (("O", "O2", "O3"), 1.4),
                 (("OH", "OS", "OW"), 1.6), (("S",), 1.85), (("SH",), 2.0)):
    for n in names:
        _RASP[n] = v


def chain(n, seed, r0=30.0, bond=1.5, min_sep=3.0, patience=10000, gen=None):
    if gen is not None:
        return gen.chain(n, seed, r0=r0, bond=bond, min_sep=min_sep, patience=patience)
    out = np.zeros((n, 3))
    rf = C.c_double()
    _check(lib().lkg_synth_chain(seed, n, r0, bond, min_sep, patience, ptr(out), C.byref(rf)))
    return out, rf.value


def _params(type_names):
    t = {k: (e, r) for k, e, r in tables()["types"]}
    eps = np.array([t[n][0] for n in type_names])
    rad = np.array([t[n][1] for n in type_names])
    heavy = np.array([0 if n.startswith("H") else 1 for n in type_names], np.uint8)
    return eps, rad, heavy


def _f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def globule(n, seed, r0=30.0, net_charge=10.0, shift=True, gen=None):
    """Random-chain globule receptor with uniform DNA-table types."""
    coords, radius = chain(n, seed, r0=r0, gen=gen)
    rng = np.random.default_rng(seed)
    names = [tables()["types"][i][0] for i in rng.integers(0, len(tables()["types"]), n)]
    eps, rad, heavy = _params(names)
    q = rng.uniform(-0.8, 0.8, n)
    if shift:
        q = q + (net_charge - q.sum()) / n
    coords = coords - coords.mean(axis=0)
    return dict(coords=_f32(coords), ele=q, vdw=eps, radius=rad, heavy=heavy, types=names,
                chain_radius=radius, density=n / (4.0 / 3.0 * math.pi * radius ** 3))


_BACKBONE = {"P", "O1P", "O2P", "OP1", "OP2"}


def duplex(n_bp, seed):
    """B-DNA-like duplex of pseudo-atoms with nucleotide atom names/types."""
    nuc = tables()["nucleotides"]
    rng = np.random.default_rng(seed + 7919)
    seq = [("DA", "DC", "DG", "DT")[i] for i in rng.integers(0, 4, n_bp)]
    comp = {"DA": "DT", "DT": "DA", "DC": "DG", "DG": "DC"}
    coords, names, types = [], [], []
    for i in range(n_bp):
        z0 = i * 3.38
        th = math.radians(36.0 * i)
        for strand, res in ((0, seq[i]), (1, comp[seq[i]])):
            phi0 = th + (math.pi if strand else 0.0)
            atoms = nuc[res]
            shells = {"bb": [a for a in atoms if a[0] in _BACKBONE],
                      "sugar": [a for a in atoms if a[0] not in _BACKBONE and "'" in a[0]],
                      "base": [a for a in atoms if a[0] not in _BACKBONE and "'" not in a[0]]}
            for shell, lst in shells.items():
                m = len(lst)
                for k, (name, typ) in enumerate(lst):
                    f = (k + 0.5) / m
                    if shell == "bb":
                        r = 8.9 if name == "P" else 9.6
                        ph = phi0 + (f - 0.5) * 0.30
                        z = z0 + (f - 0.5) * 2.0
                    elif shell == "sugar":
                        r = 8.2 - 2.4 * f
                        ph = phi0 + 0.18 + (f - 0.5) * 0.35
                        z = z0 + 0.6 + (f - 0.5) * 1.6
                    else:
                        r = 5.4 - 4.8 * f
                        ph = phi0 + 0.35 + (f - 0.5) * 0.5
                        z = z0 + (f - 0.5) * 0.8
                    j = rng.uniform(-0.2, 0.2, 3)
                    coords.append((r * math.cos(ph) + j[0], r * math.sin(ph) + j[1], z + j[2]))
                    names.append(name)
                    types.append(typ)
    coords = np.array(coords)
    eps, rad, _ = _params(types)
    heavy = np.array([0 if n.startswith("H") else 1 for n in names], np.uint8)
    q = np.array([-1.0 if n == "P" else 0.0 for n in names])
    coords = coords - coords.mean(axis=0)
    return dict(coords=_f32(coords), ele=q, vdw=eps, radius=rad, heavy=heavy, types=types, names=names)


def add_cpydock(m):
    """cpydock side arrays: des by AMBER type, reference ASA by Lee-Richards
    over heavy atoms with radius_per_asp radii (hydrogens get -1), hyd = heavy."""
    types = m["types"]
    heavy = np.asarray(m["heavy"]).astype(bool)
    des = np.array([0.0 if not h else _DES.get(t, 0.0) for t, h in zip(types, heavy)])
    asa = np.full(len(types), -1.0)
    hidx = np.nonzero(heavy)[0]
    rad = np.array([_RASP.get(types[i], 0.0) for i in hidx])
    asa[hidx] = lr_sasa(np.asarray(m["coords"])[hidx], rad)
    out = dict(m)
    out.update(hyd=heavy.astype(np.int32), des=des, asa=asa)
    return out


def fib_sphere(n, r):
    """src/bin/lightdock.rs:406-414."""
    g = math.pi * (3.0 - math.sqrt(5.0))
    out = []
    for i in range(n):
        y = 1.0 - (i / max(n - 1.0, 1.0)) * 2.0
        rr = math.sqrt(max(1.0 - y * y, 0.0))
        th = g * i
        out.append((r * rr * math.cos(th), r * y, r * rr * math.sin(th)))
    return out


def setup_poses(rec_coords, n_swarms, n_glow, seed, swarm_radius=3.0, gen=None):
    """``LKlight setup`` initial positions: (n_swarms * n_glow) x 7 rows of
    (tx, ty, tz, qw, qx, qy, qz), 6-decimal text precision."""
    c = np.asarray(rec_coords, np.float64)
    avg_r = float(np.mean(np.sqrt((c * c).sum(axis=1))))
    centers = fib_sphere(max(n_swarms * 5, 2000), avg_r + swarm_radius)[:n_swarms]
    rng = (gen.Rng if gen is not None else Rng)(seed)
    rows = []
    two_pi = 2.0 * math.pi
    for cx, cy, cz in centers:
        for _ in range(n_glow):
            dx = (rng.f64() - 0.5) * 2.0
            dy = (rng.f64() - 0.5) * 2.0
            dz = (rng.f64() - 0.5) * 2.0
            u1 = rng.f64()
            u2 = rng.f64() * 2.0 * math.pi
            u3 = rng.f64() * two_pi
            s1, s2 = math.sqrt(1.0 - u1), math.sqrt(u1)
            q = (s1 * math.sin(u2), s1 * math.cos(u2), s2 * math.sin(u3), s2 * math.cos(u3))
            row = (cx + dx, cy + dy, cz + dz, q[3], q[0], q[1], q[2])
            rows.append([float("%.6f" % v) for v in row])
    return np.array(rows)


def to_kernel_poses(positions):
    """(tx, ty, tz, qw, qx, qy, qz) rows -> kernel layout (w, x, y, z, tx, ty, tz)."""
    p = np.asarray(positions, np.float64).reshape(-1, 7)
    return np.ascontiguousarray(np.hstack([p[:, 3:7], p[:, 0:3]]))


# ---------------------------------------------------------------------------
# benchmark configurations
# ---------------------------------------------------------------------------
def config0(n_rec=12625, n_bp=20, seed=42, gen=None):
    """Plain scorer, dna: 12,625-atom globule + 20 bp duplex; 1 x 200, seed 42."""
    rec = globule(n_rec, seed, gen=gen)
    lig = duplex(n_bp, seed)
    return dict(rec=rec, lig=lig, family="dna", swarms=1, glowworms=200, steps=100, seed=seed)


def config1(family, seed=7, base=None):
    """config-0 complex with vdw / pydock / cpydock; 6 x 300, seed 7."""
    b = base or config0()
    rec, lig = b["rec"], b["lig"]
    if family == "cpydock":
        rec, lig = add_cpydock(rec), add_cpydock(lig)
    return dict(rec=rec, lig=lig, family=family, swarms=6, glowworms=300, steps=100, seed=seed)


def config2(n_complex=64, seed=11, swarms=20, glowworms=300, gen=None):
    """64 complexes, receptors log-uniform 2k-40k atoms, ligands 300-5k atoms;
    first half dna, second half pydock."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_complex):
        nr = int(round(math.exp(rng.uniform(math.log(2000), math.log(40000)))))
        nl = int(round(math.exp(rng.uniform(math.log(300), math.log(5000)))))
        n_bp = max(2, int(round(nl / 62.0)))
        rec = globule(nr, seed * 1000 + k, r0=30.0 * (nr / 12625.0) ** (1.0 / 3.0), gen=gen)
        lig = duplex(n_bp, seed * 1000 + k)
        out.append(dict(rec=rec, lig=lig, family="dna" if k < n_complex // 2 else "pydock",
                        swarms=swarms, glowworms=glowworms, steps=100, seed=seed))
    return out


def config4(seed=19, n_glob=12625, n_lig=12000):
    """cpydock, 8 globules edge to edge (~100k atoms) + 12k-atom globule ligand."""
    globs = [globule(n_glob, seed * 100 + i) for i in range(8)]
    R = max(g["chain_radius"] for g in globs)
    parts = []
    for i, g in enumerate(globs):
        off = np.array([(i & 1) * 2 - 1, ((i >> 1) & 1) * 2 - 1, ((i >> 2) & 1) * 2 - 1], float) * R
        parts.append(g["coords"] + off)
    rec = dict(coords=_f32(np.vstack(parts) - np.vstack(parts).mean(axis=0)),
               ele=np.concatenate([g["ele"] for g in globs]), vdw=np.concatenate([g["vdw"] for g in globs]),
               radius=np.concatenate([g["radius"] for g in globs]),
               heavy=np.concatenate([g["heavy"] for g in globs]), types=sum((g["types"] for g in globs), []))
    lig = globule(n_lig, seed, shift=False)
    return dict(rec=add_cpydock(rec), lig=add_cpydock(lig), family="cpydock", swarms=50, glowworms=500,
                steps=100, seed=seed)


def restraints(rec_coords, n_lig, centres, seed, n_rec_res=20, n_lig_res=6, n_membrane=300,
               rec_res_atoms=10, lig_res_atoms=30, reach=20.0):
    """Synthetic active restraints and membrane for a complex whose atoms
    carry no residues: receptor residues are blocks of `rec_res_atoms`
    consecutive chain atoms, ligand residues blocks of `lig_res_atoms`
    (about one nucleotide).  Restraint residues and membrane beads are drawn
    among receptor atoms within `reach` A of the swarm centres, so that the
    poses touch some of them.  Returns per-atom receptor / ligand restraint
    residue indices (-1 = none) and the membrane atom indices."""
    rng = np.random.default_rng(seed)
    rc = np.asarray(rec_coords, np.float64)
    near = np.zeros(len(rc), bool)
    for c in np.asarray(centres, np.float64).reshape(-1, 3):
        near |= np.linalg.norm(rc - c, axis=1) < reach
    idx = np.nonzero(near)[0]
    rres = np.minimum(np.arange(len(rc)) // rec_res_atoms, len(rc) // rec_res_atoms - 1)
    cand = np.unique(rres[idx])
    ract = rng.choice(cand, min(n_rec_res, len(cand)), replace=False)
    pos = {int(r): k for k, r in enumerate(ract)}
    rr = np.array([pos.get(int(r), -1) for r in rres], np.int32)
    lres = np.arange(n_lig) // lig_res_atoms
    lact = rng.choice(lres.max() + 1, min(n_lig_res, lres.max() + 1), replace=False)
    lpos = {int(r): k for k, r in enumerate(lact)}
    lr = np.array([lpos.get(int(r), -1) for r in lres], np.int32)
    mem = np.sort(rng.choice(idx, min(n_membrane, len(idx)), replace=False)).astype(np.int32)
    return rr, lr, mem
