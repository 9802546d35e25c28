"""ctypes binding of the oracle (CPU restatement of LKlight's CPU grid path).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by ``bench.py`` for the timed CPU baseline.  The product
library never loads it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liblkg_oracle.so")

DNA, VDW, PYDOCK, CPYDOCK = 0, 1, 2, 3
FAMILIES = {"dna": DNA, "vdw": VDW, "pydock": PYDOCK, "cpydock": CPYDOCK}

_lib = None


def build(force=False):
    """Compile the oracle with its Makefile (g++, OpenMP, no FMA contraction)."""
    src = [os.path.join(HERE, f) for f in ("oracle.cpp", "oracle.h", "Makefile")]
    if (force or not os.path.exists(LIB_PATH)
            or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(s) for s in src)):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P, D, I64, I32, U64, V = C.c_void_p, C.c_double, C.c_int64, C.c_int32, C.c_uint64, None
        sig = {
            "orc_rng_new": (P, [U64]), "orc_rng_free": (V, [P]), "orc_rng_f64": (D, [P]),
            "orc_rng_u64": (U64, [P]),
            "orc_quat_random": (V, [P, P]), "orc_quat_slerp": (V, [P, P, D, P]),
            "orc_quat_normalize": (V, [P]),
            "orc_field_new": (P, [P, P, I64, C.c_int]), "orc_field_new_scatter": (P, [P, P, I64, C.c_int]),
            "orc_field_info": (V, [P, P, P, P]),
            "orc_field_phi32": (P, [P]), "orc_field_phi64": (P, [P]),
            "orc_field_sample": (D, [P, D, D, D]), "orc_field_free": (V, [P]),
            "orc_crec_build": (I64, [P, I64, P, P, P, P, P]),
            "orc_nearcell_pair_count": (I64, [P, I64, D]), "orc_allpairs_count": (I64, [P, I64, D]),
            "orc_model_new": (P, [C.c_int, I64, P, P, P, P, P, P, P, P, I64, P, P, P, P, P, P, P, P]),
            "orc_model_free": (V, [P]), "orc_model_field": (P, [P, C.c_int]),
            "orc_energy_grid": (D, [P, P, P, C.c_int, P]), "orc_energy_exact": (D, [P, P, P]),
            "orc_batch_energy_grid": (V, [P, I64, P, C.c_int, C.c_int, P, P]),
            "orc_model_set_restraints": (V, [P, P, C.c_int, P, C.c_int, P, I64]),
            "orc_batch_energy_grid_iface": (V, [P, I64, P, C.c_int, C.c_int, P, P]),
            "orc_gso_new": (P, [P, I64, P, U64, C.c_int, C.c_int]), "orc_gso_run": (V, [P, C.c_int]),
            "orc_gso_state": (V, [P, P, P, P, P, P, P, P]), "orc_gso_scored": (I64, [P]),
            "orc_gso_free": (V, [P]),
            "orc_synth_chain": (C.c_int, [U64, I32, D, D, D, I32, P, P]),
            "orc_lr_sasa": (V, [P, P, I32, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Rng:
    """rand 0.7.3 ``StdRng::seed_from_u64`` stream."""

    def __init__(self, seed):
        self.h = lib().orc_rng_new(seed)

    def f64(self):
        return lib().orc_rng_f64(self.h)

    def u64(self):
        return lib().orc_rng_u64(self.h)

    def quat(self):
        out = np.zeros(4)
        lib().orc_quat_random(self.h, _p(out))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_rng_free(self.h)


def lr_sasa(coords, radii):
    """Lee & Richards per-atom SASA (src/lr_sasa.rs: probe 1.4 A, 20 slices)."""
    c, r = _f64(coords).reshape(-1, 3), _f64(radii)
    out = np.zeros(len(r))
    lib().orc_lr_sasa(_p(c), _p(r), len(r), _p(out))
    return out


def synth_chain(n, seed, r0=30.0, bond=1.5, min_sep=3.0, patience=10000):
    """The benchmark's synthetic receptor chain (liblkg's generator, restated
    here): n x 3 coordinates and the final confinement radius."""
    out, rf = np.zeros((n, 3)), C.c_double()
    if lib().orc_synth_chain(seed, n, r0, bond, min_sep, patience, _p(out), C.byref(rf)) != 0:
        raise ValueError("random chain did not fit (%d atoms, r0 %.1f)" % (n, r0))
    return out, rf.value


class Generators:
    """Input generators for the CPU reference arm: the synthetic chain and
    StdRng from the oracle, so that its complexes and poses are made without
    loading the product library (``synth`` functions take ``gen=``)."""
    chain = staticmethod(synth_chain)
    Rng = None   # set below


def slerp(a, b, t):
    a, b, out = _f64(a), _f64(b), np.zeros(4)
    lib().orc_quat_slerp(_p(a), _p(b), t, _p(out))
    return out


class Field:
    """``ReceptorField`` (grid_dna.rs); fp64 keeps phi in double.  scatter:
    build by the plain single-threaded per-atom scatter instead of the
    parallel brick order (the same bits; a check of the brick order)."""

    def __init__(self, coords, charges, fp64=False, _handle=None, _owner=None, scatter=False):
        if _handle is not None:
            self.h, self._owner = _handle, _owner
        else:
            c, q = _f64(coords), _f64(charges)
            new = lib().orc_field_new_scatter if scatter else lib().orc_field_new
            self.h, self._owner = new(_p(c), _p(q), len(q), int(fp64)), None
        o, d, s = np.zeros(3), np.zeros(3, np.int64), C.c_double()
        lib().orc_field_info(self.h, _p(o), _p(d), C.byref(s))
        self.origin, self.dims, self.spacing, self.fp64 = o, d, s.value, fp64

    @property
    def phi(self):
        n = int(np.prod(self.dims))
        if self.fp64:
            ptr = lib().orc_field_phi64(self.h)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), (n,)).copy()
        ptr = lib().orc_field_phi32(self.h)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), (n,)).copy()

    def phi_view(self):
        """The f32 grid in place (no copy): valid while this field (or the
        model that owns it) lives."""
        n = int(np.prod(self.dims))
        ptr = lib().orc_field_phi32(self.h)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), (n,))

    def sample(self, x, y, z):
        return lib().orc_field_sample(self.h, x, y, z)

    def __del__(self):
        if getattr(self, "h", None) and self._owner is None:
            lib().orc_field_free(self.h)


Generators.Rng = Rng


def crec_build(coords):
    """``CudaReceptor::build`` cell list: returns dict of the C-ABI fields."""
    c = _f64(coords)
    nc, org, sp = np.zeros(3, np.int32), np.zeros(3, np.float32), C.c_float()
    ncs = lib().orc_crec_build(_p(c), len(c), _p(nc), _p(org), C.byref(sp), None, None)
    cs, ca = np.zeros(ncs, np.int32), np.zeros(len(c), np.int32)
    lib().orc_crec_build(_p(c), len(c), _p(nc), _p(org), C.byref(sp), _p(cs), _p(ca))
    return dict(cell_start=cs, cell_atoms=ca, nc=nc, origin=org, sp=sp.value)


class Model:
    """Scoring model of one family over one receptor/ligand pair (f64 arrays)."""

    def __init__(self, family, rec, lig):
        self.family = FAMILIES[family] if isinstance(family, str) else family
        self._keep = []

        def side(m):
            c = _f64(m["coords"]).reshape(-1, 3)
            q, v, r = _f64(m["ele"]), _f64(m["vdw"]), _f64(m["radius"])
            h = None if m.get("heavy") is None else np.ascontiguousarray(m["heavy"], np.uint8)
            hy = None if m.get("hyd") is None else np.ascontiguousarray(m["hyd"], np.int32)
            de, a = _f64(m.get("des")), _f64(m.get("asa"))
            self._keep += [c, q, v, r, h, hy, de, a]
            return [len(c), _p(c), _p(q), _p(v), _p(r), _p(h), _p(hy), _p(de), _p(a)]

        self.h = lib().orc_model_new(self.family, *side(rec), *side(lig))

    def field(self, fp64=False):
        return Field(None, None, fp64, _handle=lib().orc_model_field(self.h, int(fp64)), _owner=self)

    def energy_grid(self, t, q, fp64=False, parts=False):
        t, q, pa = _f64(t), _f64(q), np.zeros(5)
        e = lib().orc_energy_grid(self.h, _p(t), _p(q), int(fp64), _p(pa))
        return (e, pa) if parts else e

    def energy_exact(self, t, q):
        t, q = _f64(t), _f64(q)
        return lib().orc_energy_exact(self.h, _p(t), _p(q))

    def batch_energy_grid(self, poses, fp64=False, threads=0, parts=False):
        """poses: N x 7 (w, x, y, z, tx, ty, tz), the kernel's pose layout."""
        poses = _f64(poses).reshape(-1, 7)
        out = np.zeros(len(poses))
        pa = np.zeros((len(poses), 5)) if parts else None
        lib().orc_batch_energy_grid(self.h, len(poses), _p(poses), int(fp64), threads, _p(out), _p(pa))
        return (out, pa) if parts else out

    def set_restraints(self, rec_res=None, nres_r=0, lig_res=None, nres_l=0, membrane=None):
        """Active restraints (restraint residue index per atom, -1 = none)
        and receptor membrane bead atom indices."""
        rr = None if not nres_r else np.ascontiguousarray(rec_res, np.int32)
        lr = None if not nres_l else np.ascontiguousarray(lig_res, np.int32)
        mm = None if membrane is None or len(membrane) == 0 else np.ascontiguousarray(membrane, np.int32)
        self._keep += [rr, lr, mm]
        lib().orc_model_set_restraints(self.h, _p(rr), int(nres_r), _p(lr), int(nres_l), _p(mm),
                                       0 if mm is None else len(mm))

    def batch_energy_grid_iface(self, poses, fp64=False, threads=0):
        """Scores and per-pose (pr, pl, membrane intersection)."""
        poses = _f64(poses).reshape(-1, 7)
        out = np.zeros(len(poses))
        f = np.zeros((len(poses), 3))
        lib().orc_batch_energy_grid_iface(self.h, len(poses), _p(poses), int(fp64), threads, _p(out), _p(f))
        return out, f

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_model_free(self.h)


class GSO:
    """Glowworm swarm optimisation over an oracle model (lib.rs / swarm.rs)."""

    def __init__(self, model, positions, seed, fp64=False, threads=0):
        self.model = model
        self.pos = _f64(positions).reshape(-1, 7)
        self.n = len(self.pos)
        self.h = lib().orc_gso_new(model.h, self.n, _p(self.pos), seed, int(fp64), threads)

    def run(self, steps):
        lib().orc_gso_run(self.h, steps)

    def state(self):
        n = self.n
        t, r, luc, sc, vis = np.zeros((n, 3)), np.zeros((n, 4)), np.zeros(n), np.zeros(n), np.zeros(n)
        nn, mv = np.zeros(n, np.int32), np.zeros(n, np.uint8)
        lib().orc_gso_state(self.h, _p(t), _p(r), _p(luc), _p(sc), _p(vis), _p(nn), _p(mv))
        return dict(translation=t, rotation=r, luciferin=luc, scoring=sc, vision=vis,
                    neighbors=nn, moved=mv)

    @property
    def scored(self):
        return lib().orc_gso_scored(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_gso_free(self.h)
