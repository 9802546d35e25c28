"""The scoring entry point that allocates no device memory.

Some callers cannot let a library call cudaMalloc while they score: a host
framework that hands out the whole GPU heap through its own pool or caching
allocator, a latency-bound docking loop that cannot take an allocation's
implicit synchronisation, or code running where allocation is not permitted.
``lkg_score_device_noalloc`` serves them: it runs the fast tile-scoring
kernel with its scratch (per-tile partial sums, per-pose counters, work
counter) in a fixed 8 MiB device array compiled into liblkg.

The test calls it through the C ABI twice in a row on the same inputs and
checks each result against the regular entry point (``lkg_score_device``):
scores on both calls, the per-pose parts (raw electrostatics, LJ, near
pairs) on the second, the kernel's status word (read by ``lkg_ctx_sync``),
and once against the oracle (the reference's CPU grid path).  Then it
checks that a batch too large for the fixed array is refused up front.
This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import oracle
from tests.lkg_helpers import azp_model, lkg, random_poses, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the fast path's parity tolerance


def _entry():
    f = lkg.lib().lkg_score_device_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_noalloc_matches_regular_entry_point_on_two_calls():
    import torch
    noalloc = _entry()
    ctx = lkg.Context()
    stream = torch.cuda.ExternalStream(ctx.stream)
    rec, lig = azp_model("dna")
    cid = ctx.add_complex("dna", rec, lig)
    n = 300
    poses = random_poses(n, [0, 0, 0], 6.0, 21)
    d_poses = torch.tensor(poses, dtype=torch.float64, device="cuda")
    ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    ref_parts = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    # the regular entry point (also puts the complex descriptor on the device)
    ctx.score_device(cid, n, d_poses.data_ptr(), ref.data_ptr(), ref_parts.data_ptr())
    stream.synchronize()
    ref_h, ref_parts_h = ref.cpu().numpy(), ref_parts.cpu().numpy()
    for call in range(2):
        out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        parts = torch.full((n, 4), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = noalloc(ctx.h, cid, n, d_poses.data_ptr(), out.data_ptr(), parts.data_ptr() if call else None)
        assert rc == 0, lkg.lib().lkg_last_error().decode()
        ctx.sync()   # waits for the call and checks its status word (raises if set)
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, ref_h).max() < TOL
        if call:
            # the parts are the score's terms (score = -(83 elec + vdW)): each
            # must agree within the fast path's budget of the score
            p = parts.cpu().numpy()
            scale = np.maximum(np.abs(ref_h), 1.0)
            assert (np.abs(p[:, 0] - ref_parts_h[:, 0]) * 83.0 / scale).max() < TOL   # raw electrostatics
            assert (np.abs(p[:, 1] - ref_parts_h[:, 1]) / scale).max() < TOL          # LJ + clash
            assert np.all(np.abs(p[:, 3] - ref_parts_h[:, 3]) <= 2)                 # near pairs
        else:
            # the reference's CPU grid path on the same poses
            assert rel_err(got, oracle.Model("dna", rec, lig).batch_energy_grid(poses)).max() < TOL
    ctx.close()


def test_noalloc_rejects_batches_beyond_the_fixed_scratch():
    import torch
    noalloc = _entry()
    ctx = lkg.Context()
    rec, lig = azp_model("dna")
    cid = ctx.add_complex("dna", rec, lig)
    d_poses = torch.zeros((8, 7), dtype=torch.float64, device="cuda")
    d_poses[:, 0] = 1.0
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.score_device(cid, 8, d_poses.data_ptr(), out.data_ptr())
    torch.cuda.Stream(stream_ptr=ctx.stream).synchronize()
    # 10^6 poses x 4 ligand tiles needs far more than 8 MiB: refused before any work
    rc = noalloc(ctx.h, cid, 1000000, d_poses.data_ptr(), out.data_ptr(), None)
    assert rc == 6  # LKG_ERR_CAPACITY
    assert b"scratch" in lkg.lib().lkg_last_error()
    ctx.close()
