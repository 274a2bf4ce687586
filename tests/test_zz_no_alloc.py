"""The allocation-free Green's function entry point, relax_op_green_noalloc.

It exists for callers that cannot allocate device memory themselves or let
the library do it (a host whose pool allocator owns the device, code where
cudaMalloc/cudaFree are not allowed): its scratch is a fixed device array in
the library.  Checked through the C ABI against relax_op_green on two calls
in a row with different inputs (the second call must not see the first
call's scratch), and for the size limit.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from relax_b200 import _lib

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _inputs(seed, sx1, sx2, sx3):
    rng = np.random.default_rng(seed)
    c = np.zeros((3, sx3, sx2, sx1 + 2), np.float32)
    c[:, : sx3 // 2, :, :sx1] = rng.standard_normal((3, sx3 // 2, sx2, sx1))
    t = np.zeros((3, sx2, sx1 + 2), np.float32)
    t[:, :, :sx1] = 0.1 * rng.standard_normal((3, sx2, sx1))
    return c, t


def _green(fn, c, t, sx1, sx2, sx3, gam):
    dc = [torch.from_numpy(c[k].copy()).cuda() for k in range(3)]
    dt = [torch.from_numpy(t[k].copy()).cuda() for k in range(3)]
    _lib.check(fn(*[C.c_void_p(x.data_ptr()) for x in dc], *[C.c_void_p(x.data_ptr()) for x in dt],
                  sx1, sx2, sx3, 0.5, 0.4, 0.25, 1.0, 1.0, gam, None))
    torch.cuda.synchronize()
    return np.stack([x.cpu().numpy() for x in dc])[..., :sx1]


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


# 128 x 128 x 64 needs 13 MB of the 16 MiB scratch (the twiddle tables sit
# near the end of the array) and takes the register passes in relax_op_green
@pytest.mark.parametrize("sx1,sx2,sx3", [(64, 48, 32), (32, 32, 32), (128, 128, 64)])
def test_noalloc_green_matches_allocating_green_twice(sx1, sx2, sx3):
    lib = _lib.load()
    for call, (seed, gam) in enumerate(((1, 8.3e-4), (2, 0.0))):
        c, t = _inputs(seed, sx1, sx2, sx3)
        ref = _green(lib.relax_op_green, c, t, sx1, sx2, sx3, gam)
        got = _green(lib.relax_op_green_noalloc, c, t, sx1, sx2, sx3, gam)
        assert _rel(got, ref) < 1e-6, (call, _rel(got, ref))


def test_noalloc_green_rejects_grids_beyond_its_scratch():
    lib = _lib.load()
    sx1, sx2, sx3 = 256, 256, 64        # needs ~25 MB of scratch
    c = torch.zeros((3, sx3, sx2, sx1 + 2), device="cuda")
    t = torch.zeros((3, sx2, sx1 + 2), device="cuda")
    rc = lib.relax_op_green_noalloc(*[C.c_void_p(c[k].data_ptr()) for k in range(3)],
                                    *[C.c_void_p(t[k].data_ptr()) for k in range(3)],
                                    sx1, sx2, sx3, 1.0, 1.0, 1.0, 1.0, 1.0, 0.0, None)
    assert rc == 1
    assert b"scratch" in lib.relax_last_error()


def test_noalloc_green_rejects_a_grid_just_over_its_scratch():
    """48 x 384 x 72 needs 16 MiB + 46 KB; 48 x 384 x 64 fits."""
    lib = _lib.load()
    for sx3, want in ((72, 1), (64, 0)):
        sx1, sx2 = 48, 384
        c = torch.zeros((3, sx3, sx2, sx1 + 2), device="cuda")
        t = torch.zeros((3, sx2, sx1 + 2), device="cuda")
        rc = lib.relax_op_green_noalloc(*[C.c_void_p(c[k].data_ptr()) for k in range(3)],
                                        *[C.c_void_p(t[k].data_ptr()) for k in range(3)],
                                        sx1, sx2, sx3, 1.0, 1.0, 1.0, 1.0, 1.0, 0.0, None)
        torch.cuda.synchronize()
        assert rc == want, (sx3, rc, lib.relax_last_error())


@pytest.mark.parametrize("sx1,sx2,sx3", [(32, 8, 16), (8, 12, 8)])
def test_noalloc_green_small_grid_matches_oracle(oracle32, sx1, sx2, sx3):
    """Small grids (sx2 = 8 or 12, sx1 = 8 with the generic x passes) and a
    box shallower than a context takes (sx3/2 = 4: the step's
    differentiators stop at 5, the Green's function alone does not), against
    the oracle's greenfunctioncowling."""
    lib = _lib.load()
    c, t = _inputs(5, sx1, sx2, sx3)
    cr, tr = c.copy(), t.copy()
    oracle32.green(cr, tr, sx1, sx2, sx3, (0.5, 0.4, 0.25), 1.0, 1.0, 8.3e-4)
    for call in range(2):
        got = _green(lib.relax_op_green_noalloc, c, t, sx1, sx2, sx3, 8.3e-4)
        assert _rel(got, cr[..., :sx1]) < 1e-5, (call, _rel(got, cr[..., :sx1]))
