"""lkg: B200-native batched pose scoring for LKlight GSO docking.

Python binding of liblkg.so (built in-tree by ``build.py``).  The compute
path is the CUDA library; this module only marshals arrays.  There is no CPU
fallback: if the library or a CUDA device is missing, calls raise.

The ``Scorer`` class mirrors the reference's ``Score`` trait
(src/scoring.rs:20-81: ``energy``, ``supports_batch``, ``batch_energy``) for
the dna / vdw / pydock / cpydock families; ``compat`` exposes the
reference-compatible C entry points (``cuda_batch_score`` ...).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liblkg.so")

DNA, VDW, PYDOCK, CPYDOCK = 0, 1, 2, 3
FAMILIES = {"dna": DNA, "vdw": VDW, "pydock": PYDOCK, "cpydock": CPYDOCK}
FLAGS = {"dna": 7, "pydock": 3, "cpydock": 3, "vdw": 0}   # gpu_family.rs:187-194
PREC_FAST, PREC_EXACT = 0, 1

STATUS = {0: "ok", 1: "invalid argument", 2: "device out of memory", 3: "kernel launch failed",
          4: "timed out", 5: "device error", 6: "device capacity exceeded", 7: "no CUDA device",
          8: "invalid state"}


class LkgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("lkg status %d (%s): %s" % (status, STATUS.get(status, "?"), msg))
        self.status = status


class Mol(C.Structure):
    _fields_ = [("n", C.c_int32), ("coords", C.c_void_p), ("ele", C.c_void_p), ("vdw", C.c_void_p),
                ("radius", C.c_void_p), ("heavy", C.c_void_p), ("hyd", C.c_void_p), ("des", C.c_void_p),
                ("asa", C.c_void_p)]


class Field(C.Structure):
    _fields_ = [("phi", C.c_void_p), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("ox", C.c_double), ("oy", C.c_double), ("oz", C.c_double), ("spacing", C.c_double)]


_lib = None


def build(force=False):
    from importlib import util
    spec = util.spec_from_file_location("_lkg_build", os.path.join(HERE, "build.py"))
    mod = util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


def lib():
    """Load liblkg.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError("liblkg.so not built (%s); run lklight-gpu_b200/build.py" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    P, I, I64, U64, D, F = C.c_void_p, C.c_int, C.c_int64, C.c_uint64, C.c_double, C.c_float
    I32 = C.c_int32
    sig = {
        "lkg_status_string": (C.c_char_p, [I]), "lkg_last_status": (I, []),
        "lkg_last_error": (C.c_char_p, []), "lkg_device_available": (I, []),
        "lkg_version": (C.c_char_p, []),
        "lkg_ctx_create": (I, [I, P]), "lkg_ctx_destroy": (I, [P]),
        "lkg_ctx_set_precision": (I, [P, I]), "lkg_ctx_set_tiles": (I, [P, I, I]),
        "lkg_ctx_set_stream": (I, [P, P]), "lkg_ctx_set_setup": (I, [P, I]), "lkg_ctx_set_staging": (I, [P, I]), "lkg_ctx_set_group": (I, [P, I]), "lkg_ctx_set_xsub": (I, [P, I]), "lkg_ctx_stream": (P, [P]), "lkg_ctx_launches": (I64, [P]),
        "lkg_complex_add": (I, [P, I, P, P, P, P]), "lkg_complex_info": (I, [P, I, P, P, P]),
        "lkg_score": (I, [P, I, I, P, P, P]), "lkg_score_device": (I, [P, I, I, P, P, P]),
        "lkg_score_interface": (I, [P, I, I, P, P, P]),
        "lkg_complex_set_restraints": (I, [P, I, P, I, P, I, P, I]),
        "lkg_surrogate_reserve": (I, [P, I, I]),
        "lkg_score_multi_device": (I, [P, I, P, P, P, P, P]),
        "lkg_score_multi": (I, [P, I, P, P, P, P, P]),
        "lkg_ctx_sync": (I, [P]),
        "lkg_surrogate_create": (I, [P, I, U64, P]), "lkg_surrogate_destroy": (I, [P]),
        "lkg_surrogate_set_target_scale": (I, [P, I, P]), "lkg_surrogate_predict": (I, [P, I, P, P]),
        "lkg_surrogate_train": (I, [P, I, P, P, I, I, C.c_float, P]), "lkg_surrogate_nparams": (I64, []),
        "lkg_surrogate_get_params": (I, [P, P]), "lkg_surrogate_set_params": (I, [P, P]),
        "lkg_surrogate_grad": (I, [P, I, P, P, P, P, P]), "lkg_surrogate_features": (I, [P, I, P, P]),
        "lkg_plan_create": (I, [P, I, P, P, P]), "lkg_plan_launch": (I, [P, P, P, P]),
        "lkg_plan_capture": (I, [P, P, P, P, I]), "lkg_plan_replay": (I, [P]),
        "lkg_plan_sync": (I, [P]), "lkg_plan_destroy": (I, [P]),
        "lkg_field_build": (I, [P, P, I32, P, P, P, P]), "lkg_lr_sasa": (I, [P, P, I32, P]),
        "lkg_receptor_distance_bound": (I, [P, I32, P, I32, P]),
        "lkg_synth_chain": (I, [U64, I32, D, D, D, I32, P, P]),
        "lkg_rng_new": (P, [U64]), "lkg_rng_f64": (D, [P]), "lkg_rng_free": (None, [P]),
        "lkg_gso_create": (I, [P, I, P, P, P, P, P, P]), "lkg_gso_run": (I, [P, I]),
        "lkg_gso_state": (I, [P, P, P, P, P, P, P]), "lkg_gso_scored": (I64, [P]),
        "lkg_gso_save": (I, [P, I, I, C.c_char_p]),
        "lkg_gso_destroy": (I, [P]), "lkg_compat_cache_clear": (None, []),
        "lkg_gso_set_screen": (I, [P, P]), "lkg_gso_finalize": (I, [P]), "lkg_gso_predicted": (I64, [P]), "lkg_gso_timing": (I, [P, P]), "lkg_surrogate_set_backend": (I, [P, I]), "lkg_surrogate_status": (I, [P, P]), "lkg_gso_run_device": (I, [P, I]),
        "cuda_batch_score": (I, [P, I, I, I, F, F, F, F, P, P, P, P, P, I, P, P, I, I, I, F, F, F, F,
                                 P, P, P, P, P, P, I, I, C.c_uint, P]),
        "cuda_cpydock_solv": (I, [P, P, I, P, P, I, I, I, F, F, F, F, P, P, P, P, I, I, P, P, P, P, P]),
        "cuda_full_score": (I, [P, I, I, I, F, F, F, F, P, P, P, P, P, I, P, P, I, I, I, F, F, F, F,
                                P, P, P, P, P, I, P, P]),
        "cuda_far_field": (I, [P, I, I, I, F, F, F, F, P, P, I, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _addr(a):
    """Address of a contiguous numpy array or a (CPU, possibly pinned) torch tensor."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _check(status):
    if status != 0:
        raise LkgError(status, lib().lkg_last_error().decode())


def ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _arr(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def device_available():
    return bool(lib().lkg_device_available())


def make_mol(m, keep):
    """Build an lkg_mol from a dict of per-atom arrays (coords n x 3, ele,
    vdw (well depth), radius, optional heavy / hyd / des / asa)."""
    c = _arr(m["coords"], np.float64).reshape(-1, 3)
    arrs = dict(coords=c, ele=_arr(m["ele"], np.float64), vdw=_arr(m["vdw"], np.float64),
                radius=_arr(m["radius"], np.float64), heavy=_arr(m.get("heavy"), np.uint8),
                hyd=_arr(m.get("hyd"), np.int32), des=_arr(m.get("des"), np.float64),
                asa=_arr(m.get("asa"), np.float64))
    keep.append(arrs)
    return Mol(len(c), *[None if arrs[k] is None else arrs[k].ctypes.data
                         for k in ("coords", "ele", "vdw", "radius", "heavy", "hyd", "des", "asa")])


class Screen(C.Structure):
    """``lkg_screen``: surrogate screening of GSO moves."""
    _fields_ = [("candidates", C.c_int32), ("exact_fraction", C.c_double), ("rescore_every", C.c_int32),
                ("train_steps", C.c_int32), ("train_epochs", C.c_int32), ("finetune_epochs", C.c_int32),
                ("lr", C.c_float), ("seed", C.c_uint64), ("random_rank", C.c_int32), ("batch", C.c_int32),
                ("carry_prediction", C.c_int32)]


class Context:
    """A device context: resident complexes, a stream, scratch buffers."""

    def __init__(self, device=0, precision="fast", tile=0, cell=0.0, group=0, xsub=0, host_setup=False,
                 stage="l1"):
        """host_setup: sort and pack receptors on the host instead of the
        GPU (the same arrays; the check of the GPU set-up).  stage: "l1"
        (default) or "tma": how the plain kernel loads candidate receptor
        atoms (lkg_ctx_set_staging)."""
        h = C.c_void_p()
        _check(lib().lkg_ctx_create(device, C.byref(h)))
        self.h = h
        self._keep = []
        if host_setup:
            _check(lib().lkg_ctx_set_setup(self.h, 0))
        if stage != "l1":
            _check(lib().lkg_ctx_set_staging(self.h, 1 if stage == "tma" else 0))
        if precision != "fast":
            _check(lib().lkg_ctx_set_precision(self.h, PREC_EXACT if precision == "exact" else PREC_FAST))
        if tile or cell:
            _check(lib().lkg_ctx_set_tiles(self.h, int(tile), int(round(cell * 1000))))
        if group:
            _check(lib().lkg_ctx_set_group(self.h, int(group)))
        if xsub:
            _check(lib().lkg_ctx_set_xsub(self.h, int(xsub)))

    def set_precision(self, precision):
        _check(lib().lkg_ctx_set_precision(self.h, PREC_EXACT if precision == "exact" else PREC_FAST))

    def add_complex(self, family, rec, lig, field=None):
        keep = []
        r, l = make_mol(rec, keep), make_mol(lig, keep)
        f = None
        if field is not None:
            phi = _arr(field["phi"], np.float32)
            keep.append(phi)
            nx, ny, nz = (int(v) for v in field["dims"])
            f = Field(phi.ctypes.data, nx, ny, nz, *[float(v) for v in field["origin"]], float(field["spacing"]))
        cid = C.c_int()
        fam = FAMILIES[family] if isinstance(family, str) else family
        _check(lib().lkg_complex_add(self.h, fam, C.byref(r), C.byref(l),
                                     None if f is None else C.byref(f), C.byref(cid)))
        return cid.value

    def info(self, cid):
        nr, nl, nc = C.c_int(), C.c_int(), C.c_int()
        _check(lib().lkg_complex_info(self.h, cid, C.byref(nr), C.byref(nl), C.byref(nc)))
        return nr.value, nl.value, nc.value

    def score(self, cid, poses, parts=False):
        """poses: N x 7 (w, x, y, z, tx, ty, tz) host array -> N scores
        (and N x 4 parts: raw electrostatics, LJ, desolvation, near pairs)."""
        p = _arr(poses, np.float64).reshape(-1, 7)
        out = np.zeros(len(p))
        pa = np.zeros((len(p), 4)) if parts else None
        _check(lib().lkg_score(self.h, cid, len(p), ptr(p), ptr(out), ptr(pa)))
        return (out, pa) if parts else out

    def set_restraints(self, cid, rec_residue=None, lig_residue=None, membrane=None):
        """Active restraints and membrane of complex cid: rec_residue /
        lig_residue give each atom's restraint residue index (-1 = none;
        the count is max + 1), membrane the receptor atom indices of the
        membrane beads.  No arguments clears them."""
        def res(a):
            if a is None:
                return None, 0
            a = np.ascontiguousarray(a, np.int32)
            return a, (int(a.max()) + 1 if len(a) and a.max() >= 0 else 0)
        rr, nr = res(rec_residue)
        lr, nl = res(lig_residue)
        mm = None if membrane is None else np.ascontiguousarray(membrane, np.int32)
        nm = 0 if mm is None else len(mm)
        _check(lib().lkg_complex_set_restraints(self.h, cid, ptr(rr) if nr else None, nr, ptr(lr) if nl else None,
                                                nl, ptr(mm) if nm else None, nm))

    def score_interface(self, cid, poses):
        """Scores with the restraint / membrane terms, and per pose the
        receptor and ligand restraint fractions and the membrane
        intersection (N x 3)."""
        p = _arr(poses, np.float64).reshape(-1, 7)
        out = np.zeros(len(p))
        f = np.zeros((len(p), 3))
        _check(lib().lkg_score_interface(self.h, cid, len(p), ptr(p), ptr(out), ptr(f)))
        return out, f

    def score_device(self, cid, n, d_poses, d_scores, d_parts=0):
        _check(lib().lkg_score_device(self.h, cid, n, C.c_void_p(d_poses), C.c_void_p(d_scores),
                                      C.c_void_p(d_parts) if d_parts else None))

    def score_multi_device(self, ids, counts, d_poses, d_scores, d_parts=0):
        ids = np.ascontiguousarray(ids, np.int32)
        counts = np.ascontiguousarray(counts, np.int32)
        _check(lib().lkg_score_multi_device(self.h, len(ids), ptr(ids), ptr(counts), C.c_void_p(d_poses),
                                            C.c_void_p(d_scores), C.c_void_p(d_parts) if d_parts else None))

    def score_multi(self, ids, counts, poses, scores=None, parts=None):
        """Host-buffer batch over many complexes (one launch group); poses is
        sum(counts) x 7.  Page-locked arrays are DMA'd without staging."""
        ids = np.ascontiguousarray(ids, np.int32)
        counts = np.ascontiguousarray(counts, np.int32)
        n = int(counts.sum())
        if scores is None:
            scores = np.zeros(n)
        _check(lib().lkg_score_multi(self.h, len(ids), ptr(ids), ptr(counts), C.c_void_p(_addr(poses)),
                                     C.c_void_p(_addr(scores)), C.c_void_p(_addr(parts)) if parts is not None
                                     else None))
        return scores

    def sync(self):
        """Bounded wait for the context stream + device status check."""
        _check(lib().lkg_ctx_sync(self.h))

    def plan(self, ids, counts):
        return Plan(self, ids, counts)

    @property
    def stream(self):
        return lib().lkg_ctx_stream(self.h)

    def set_stream(self, stream_ptr):
        _check(lib().lkg_ctx_set_stream(self.h, C.c_void_p(stream_ptr)))

    @property
    def launches(self):
        return lib().lkg_ctx_launches(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().lkg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """A batch prepared once; launches are capturable in a CUDA graph."""

    def __init__(self, ctx, ids, counts):
        self.ctx = ctx
        ids = np.ascontiguousarray(ids, np.int32)
        counts = np.ascontiguousarray(counts, np.int32)
        h = C.c_void_p()
        _check(lib().lkg_plan_create(ctx.h, len(ids), ptr(ids), ptr(counts), C.byref(h)))
        self.h = h

    def launch(self, d_poses, d_scores, d_parts=0):
        _check(lib().lkg_plan_launch(self.h, C.c_void_p(d_poses), C.c_void_p(d_scores),
                                     C.c_void_p(d_parts) if d_parts else None))

    def capture(self, d_poses, d_scores, d_parts=0, n_launches=1):
        _check(lib().lkg_plan_capture(self.h, C.c_void_p(d_poses), C.c_void_p(d_scores),
                                      C.c_void_p(d_parts) if d_parts else None, n_launches))

    def replay(self):
        _check(lib().lkg_plan_replay(self.h))

    def sync(self):
        _check(lib().lkg_plan_sync(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().lkg_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Surrogate:
    """BF16 tensor-core MLP surrogate of the pose energy of one complex."""

    def __init__(self, ctx, cid, seed=0):
        self.ctx = ctx
        h = C.c_void_p()
        _check(lib().lkg_surrogate_create(ctx.h, cid, seed, C.byref(h)))
        self.h = h

    @staticmethod
    def nparams():
        return lib().lkg_surrogate_nparams()

    def set_target_scale(self, scores):
        s = _arr(scores, np.float64)
        _check(lib().lkg_surrogate_set_target_scale(self.h, len(s), ptr(s)))

    def predict_device(self, n, d_poses, d_pred):
        _check(lib().lkg_surrogate_predict(self.h, n, C.c_void_p(d_poses), C.c_void_p(d_pred)))

    def train_device(self, n, d_poses, d_scores, epochs=1, batch=1024, lr=1e-3):
        loss = C.c_float()
        _check(lib().lkg_surrogate_train(self.h, n, C.c_void_p(d_poses), C.c_void_p(d_scores), epochs, batch,
                                         lr, C.byref(loss)))
        return loss.value

    def params(self):
        out = np.zeros(self.nparams(), np.float32)
        _check(lib().lkg_surrogate_get_params(self.h, ptr(out)))
        return out

    def set_params(self, p):
        p = _arr(p, np.float32)
        _check(lib().lkg_surrogate_set_params(self.h, ptr(p)))

    def grad(self, feats_bf16, targets):
        f = np.ascontiguousarray(feats_bf16, np.uint16)
        t = _arr(targets, np.float32)
        n = len(t)
        y, g, l = np.zeros(n, np.float32), np.zeros(self.nparams(), np.float32), C.c_float()
        _check(lib().lkg_surrogate_grad(self.h, n, ptr(f), ptr(t), ptr(y), ptr(g), C.byref(l)))
        return y, g, l.value

    def set_backend(self, tcgen05):
        """Forward layers on tcgen05 (True) or mma.sync (False)."""
        _check(lib().lkg_surrogate_set_backend(self.h, 1 if tcgen05 else 0))

    def status(self):
        b = C.c_int()
        _check(lib().lkg_surrogate_status(self.h, C.byref(b)))
        return b.value

    def features_device(self, n, d_poses):
        out = np.zeros((n, 64), np.uint16)
        _check(lib().lkg_surrogate_features(self.h, n, C.c_void_p(d_poses), ptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().lkg_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scorer:
    """The reference ``Score`` trait for one complex (src/scoring.rs:20-81)."""

    def __init__(self, family, rec, lig, ctx=None, precision="fast"):
        self.ctx = ctx or Context(precision=precision)
        self.family = family
        self.cid = self.ctx.add_complex(family, rec, lig)

    def supports_batch(self):
        return device_available()

    def energy(self, translation, rotation):
        """Score::energy for one pose: translation (3), rotation (w, x, y, z)."""
        return float(self.batch_energy([translation], [rotation])[0])

    def batch_energy(self, translations, rotations):
        t = np.asarray(translations, np.float64).reshape(-1, 3)
        q = np.asarray(rotations, np.float64).reshape(-1, 4)
        return self.ctx.score(self.cid, np.hstack([q, t]))


class GSO:
    """Batched GSO over groups of (complex, swarms x glowworms)."""

    def __init__(self, ctx, groups, positions, seeds):
        self.ctx = ctx
        ids = np.array([g[0] for g in groups], np.int32)
        ns = np.array([g[1] for g in groups], np.int32)
        ng = np.array([g[2] for g in groups], np.int32)
        self.n = int((ns * ng).sum())
        self._pos = _arr(positions, np.float64).reshape(-1, 7)
        assert len(self._pos) == self.n
        sd = np.ascontiguousarray(seeds, np.uint64)
        h = C.c_void_p()
        _check(lib().lkg_gso_create(ctx.h, len(ids), ptr(ids), ptr(ns), ptr(ng), ptr(self._pos), ptr(sd),
                                    C.byref(h)))
        self.h = h

    def run(self, steps, device=False):
        """steps of the plain GSO; device=True runs whole steps on the GPU
        (graph-replayed; not bitwise equal to the host GSO, see lkg.h)."""
        _check((lib().lkg_gso_run_device if device else lib().lkg_gso_run)(self.h, steps))

    def state(self):
        n = self.n
        t, r, luc, sc, vis = np.zeros((n, 3)), np.zeros((n, 4)), np.zeros(n), np.zeros(n), np.zeros(n)
        nn = np.zeros(n, np.int32)
        _check(lib().lkg_gso_state(self.h, ptr(t), ptr(r), ptr(luc), ptr(sc), ptr(vis), ptr(nn)))
        return dict(translation=t, rotation=r, luciferin=luc, scoring=sc, vision=vis, neighbors=nn)

    def set_screen(self, candidates=4, exact_fraction=0.25, rescore_every=10, train_steps=20, train_epochs=20,
                   finetune_epochs=2, lr=1e-3, seed=0, random_rank=False, batch=1024, carry_prediction=False):
        """Screen moves with the surrogate (random_rank: the same search with
        random candidate ranks instead of the network, for ablations;
        carry_prediction: unscored moves score current + predicted gain
        instead of keeping their last exact score)."""
        cfg = Screen(candidates, exact_fraction, rescore_every, train_steps, train_epochs, finetune_epochs, lr, seed,
                     1 if random_rank else 0, batch, 1 if carry_prediction else 0)
        _check(lib().lkg_gso_set_screen(self.h, C.byref(cfg)))

    def finalize(self):
        """Exact rescoring of every glowworm."""
        _check(lib().lkg_gso_finalize(self.h))

    @property
    def scored(self):
        return lib().lkg_gso_scored(self.h)

    @property
    def predicted(self):
        return lib().lkg_gso_predicted(self.h)

    def save(self, swarm, step, directory):
        """Swarm `swarm` as <directory>/gso_<step>.out (swarm.rs:232-271)."""
        _check(lib().lkg_gso_save(self.h, swarm, step, os.fsencode(directory)))

    def timing(self):
        """Wall seconds in exact scoring, host movement, surrogate inference
        and surrogate training."""
        t = np.zeros(4)
        _check(lib().lkg_gso_timing(self.h, ptr(t)))
        return dict(exact=t[0], movement=t[1], inference=t[2], training=t[3])

    def __del__(self):
        h, self.h = getattr(self, "h", None), None
        if h:
            try:
                lib().lkg_gso_destroy(h)
            except Exception:   # interpreter shutdown: the module's globals are gone
                pass


class Rng:
    """rand 0.7.3 ``StdRng::seed_from_u64`` (the product's copy)."""

    def __init__(self, seed):
        self.h = lib().lkg_rng_new(seed)

    def f64(self):
        return lib().lkg_rng_f64(self.h)

    def __del__(self):
        h, self.h = getattr(self, "h", None), None
        if h:
            try:
                lib().lkg_rng_free(h)
            except Exception:   # interpreter shutdown: the module's globals are gone
                pass


def field_build(coords, charges):
    """Receptor far field on the GPU, bit-identical to ReceptorField::build."""
    c, q = _arr(coords, np.float64).reshape(-1, 3), _arr(charges, np.float64)
    o, d, s = np.zeros(3), np.zeros(3, np.int32), C.c_double()
    _check(lib().lkg_field_build(ptr(c), ptr(q), len(q), ptr(o), ptr(d), C.byref(s), None))
    phi = np.zeros(int(np.prod(d.astype(np.int64))), np.float32)
    _check(lib().lkg_field_build(ptr(c), ptr(q), len(q), ptr(o), ptr(d), C.byref(s), ptr(phi)))
    return dict(phi=phi, dims=d, origin=o, spacing=s.value)


def receptor_distance_bound(coords, points):
    """Lower bound of each point's distance to the nearest receptor atom, as
    the warp kernels use it to skip ligand groups out of reach (host)."""
    c, q = _arr(coords, np.float64).reshape(-1, 3), _arr(points, np.float64).reshape(-1, 3)
    out = np.zeros(len(q), np.float32)
    _check(lib().lkg_receptor_distance_bound(ptr(c), len(c), ptr(q), len(q), ptr(out)))
    return out


def lr_sasa(coords, radii):
    c, r = _arr(coords, np.float64).reshape(-1, 3), _arr(radii, np.float64)
    out = np.zeros(len(r))
    _check(lib().lkg_lr_sasa(ptr(c), ptr(r), len(r), ptr(out)))
    return out
