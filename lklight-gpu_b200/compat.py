"""The reference's GPU bridge, restated over liblkg's compatible C entry points.

``CudaReceptor`` / ``CudaLigand`` pack f32 arrays and the 10 A receptor cell
list exactly as src/gpu_score.rs:38-144 and src/gpu_family.rs:82-182 do, and
``batch_scores`` / ``cpydock_solv`` call ``cuda_batch_score`` /
``cuda_cpydock_solv`` with the reference's argument order, so a Python caller
(or a test) sees the same contract the Rust bridge sees.
"""
import ctypes as C
import math

import numpy as np

from . import lib, ptr, LkgError

FACTOR, EPSILON = 332.0, 4.0


class CudaReceptor:
    """gpu_score.rs:75-144: f32 receptor arrays + 10 A cell list (origin
    floor(min - 0.01), cells = floor((hi - lo)/10) + 1 per axis)."""

    def __init__(self, coords, ele, svdw, vdwr, heavy=None):
        c = np.asarray(coords, np.float64).reshape(-1, 3)
        cell = 10.0
        lo = np.floor(c.min(axis=0) - 0.01)
        hi = c.max(axis=0)
        n = [max(int(math.floor((hi[a] - lo[a]) / cell)) + 1, 1) for a in range(3)]
        ncells = (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
        idx = [np.clip(np.floor((c[:, a] - lo[a]) / cell).astype(np.int64), 0, n[a] - 1) for a in range(3)]
        cell_of = (idx[2] * n[1] + idx[1]) * n[0] + idx[0]
        counts = np.bincount(cell_of, minlength=ncells)
        cs = np.zeros(ncells + 1, np.int32)
        cs[1:] = np.cumsum(counts)
        self.cell_start = cs
        self.cell_atoms = np.argsort(cell_of, kind="stable").astype(np.int32)
        self.ncx, self.ncy, self.ncz = n
        self.c_o = [float(np.float32(v)) for v in lo]
        self.c_sp = 10.0
        self.r_coords = np.ascontiguousarray(c, np.float32).reshape(-1)
        self.r_ele = np.ascontiguousarray(ele, np.float32)
        self.r_svdw = np.ascontiguousarray(svdw, np.float32)
        self.r_vdwr = np.ascontiguousarray(vdwr, np.float32)
        self.r_heavy = np.ascontiguousarray(np.zeros(len(c)) if heavy is None else heavy, np.uint8)
        self.nr = len(c)


class CudaLigand:
    """gpu_score.rs:38-52: f32 ligand reference coordinates and parameters."""

    def __init__(self, coords, ele, svdw, vdwr, heavy=None):
        c = np.asarray(coords, np.float64).reshape(-1, 3)
        self.base = np.ascontiguousarray(c, np.float32).reshape(-1)
        self.ele = np.ascontiguousarray(ele, np.float32)
        self.svdw = np.ascontiguousarray(svdw, np.float32)
        self.vdw = np.ascontiguousarray(vdwr, np.float32)
        self.heavy = np.ascontiguousarray(np.zeros(len(c)) if heavy is None else heavy, np.uint8)
        self.nl = len(c)


def pack_poses(translations, rotations):
    """gpu_score.rs:292-301: N x 7 (w, x, y, z, tx, ty, tz)."""
    t = np.asarray(translations, np.float64).reshape(-1, 3)
    q = np.asarray(rotations, np.float64).reshape(-1, 4)
    return np.ascontiguousarray(np.hstack([q, t]))


def batch_raw(field, rec, lig, poses, flags, library=None):
    """cuda_batch_score: returns N x 2 (raw electrostatics, LJ[+clash]).
    ``library``: another ctypes library exporting the same symbol (the
    reference's own kernels, in tests); liblkg by default."""
    poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 7)
    n = len(poses)
    out = np.zeros(2 * n)
    dummy = np.zeros(1, np.float32)
    if field is not None:
        phi = np.ascontiguousarray(field["phi"], np.float32)
        nx, ny, nz = (int(v) for v in field["dims"])
        ox, oy, oz = (float(np.float32(v)) for v in field["origin"])
        sp = float(field["spacing"])
    else:
        phi, nx, ny, nz, ox, oy, oz, sp = dummy, 0, 0, 0, 0.0, 0.0, 0.0, 0.0
    L = library if library is not None else lib()
    r = L.cuda_batch_score(ptr(phi), nx, ny, nz, ox, oy, oz, sp,
                               ptr(rec.r_coords), ptr(rec.r_ele), ptr(rec.r_svdw), ptr(rec.r_vdwr),
                               ptr(rec.r_heavy), rec.nr, ptr(rec.cell_start), ptr(rec.cell_atoms),
                               rec.ncx, rec.ncy, rec.ncz, rec.c_o[0], rec.c_o[1], rec.c_o[2], rec.c_sp,
                               ptr(lig.base), ptr(poses), ptr(lig.ele), ptr(lig.svdw), ptr(lig.vdw),
                               ptr(lig.heavy), lig.nl, n, flags, ptr(out))
    if r != 0:
        if library is not None:
            raise RuntimeError("cuda_batch_score returned %d" % r)
        raise LkgError(lib().lkg_last_status(), lib().lkg_last_error().decode())
    return out.reshape(n, 2)


def batch_scores(field, rec, lig, poses, flags):
    """gpu_score.rs:326-331 / gpu_family.rs:283-288: -(E*332/4 + V)."""
    raw = batch_raw(field, rec, lig, poses, flags)
    return -(raw[:, 0] * FACTOR / EPSILON + raw[:, 1])


def cpy_flag(hyd):
    """cpydock.rs:808-819: flag(i) = i even and hydrogens[i/2] != 0."""
    hyd = np.asarray(hyd)
    f = np.zeros(len(hyd), np.uint8)
    f[0::2] = (hyd[: (len(hyd) + 1) // 2] != 0)
    return f


def cpydock_solv(rec, lig, poses, r_flag, l_flag, r_des, r_asa, l_des, l_asa, library=None):
    """cuda_cpydock_solv: per-pose desolvation S.  ``library``: another
    ctypes library exporting the same symbol (as for batch_raw)."""
    poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 7)
    n = len(poses)
    out = np.zeros(n)
    a = [np.ascontiguousarray(x, dt) for x, dt in ((r_flag, np.uint8), (l_flag, np.uint8), (r_des, np.float32),
                                                   (r_asa, np.float32), (l_des, np.float32), (l_asa, np.float32))]
    L = library if library is not None else lib()
    r = L.cuda_cpydock_solv(ptr(rec.r_coords), ptr(a[0]), rec.nr, ptr(rec.cell_start), ptr(rec.cell_atoms),
                            rec.ncx, rec.ncy, rec.ncz, rec.c_o[0], rec.c_o[1], rec.c_o[2], rec.c_sp,
                            ptr(lig.base), ptr(poses), ptr(a[1]), ptr(lig.ele), lig.nl, n,
                            ptr(a[2]), ptr(a[3]), ptr(a[4]), ptr(a[5]), ptr(out))
    if r != 0:
        if library is not None:
            raise RuntimeError("cuda_cpydock_solv returned %d" % r)
        raise LkgError(lib().lkg_last_status(), lib().lkg_last_error().decode())
    return out


def full_score(field, rec, lig_coords, lig):
    """cuda_full_score: per-atom (elec_raw, vdw) for pre-transformed coords."""
    lc = np.ascontiguousarray(lig_coords, np.float32).reshape(-1)
    nl = len(lc) // 3
    oe, ov = np.zeros(nl, np.float32), np.zeros(nl, np.float32)
    phi = np.ascontiguousarray(field["phi"], np.float32)
    nx, ny, nz = (int(v) for v in field["dims"])
    ox, oy, oz = (float(np.float32(v)) for v in field["origin"])
    r = lib().cuda_full_score(ptr(phi), nx, ny, nz, ox, oy, oz, float(field["spacing"]),
                              ptr(rec.r_coords), ptr(rec.r_ele), ptr(rec.r_svdw), ptr(rec.r_vdwr),
                              ptr(rec.r_heavy), rec.nr, ptr(rec.cell_start), ptr(rec.cell_atoms),
                              rec.ncx, rec.ncy, rec.ncz, rec.c_o[0], rec.c_o[1], rec.c_o[2], rec.c_sp,
                              ptr(lc), ptr(lig.ele), ptr(lig.svdw), ptr(lig.vdw), ptr(lig.heavy), nl,
                              ptr(oe), ptr(ov))
    if r != 0:
        raise LkgError(lib().lkg_last_status(), lib().lkg_last_error().decode())
    return oe, ov


def far_field(field, coords, charges):
    """cuda_far_field: sum_j q_j * phi(x_j)."""
    c = np.ascontiguousarray(coords, np.float32).reshape(-1)
    q = np.ascontiguousarray(charges, np.float32)
    phi = np.ascontiguousarray(field["phi"], np.float32)
    nx, ny, nz = (int(v) for v in field["dims"])
    ox, oy, oz = (float(np.float32(v)) for v in field["origin"])
    res = C.c_double()
    r = lib().cuda_far_field(ptr(phi), nx, ny, nz, ox, oy, oz, float(field["spacing"]), ptr(c), ptr(q),
                             len(q), C.byref(res))
    if r != 0:
        raise LkgError(lib().lkg_last_status(), lib().lkg_last_error().decode())
    return res.value
