"""The mixed-precision form: the x3 transform's length-64 DFT sub-transforms
as tensor-core products (tcgen05, split BF16 hi/lo operands, FP32
accumulation), k_zspec_tc.

* relax_op_dft64_tc, the product alone, against numpy's FFT (relative L2
  <= 3e-5: two BF16 parts keep about 16 bits of each operand).
* relax_op_green_mixed against the oracle's greenfunctioncowling on 128-deep
  boxes with the time step's pruning (lower half of the body force zero,
  upper half of the displacement compared), full and partial tiles of 64
  columns, with and without gravity: relative L2 <= 1e-4.
* Time steps in the mixed form against the FP64 oracle (and the FP32
  oracle) with the GPU's Dt sequence replayed: <= 1e-4 after the run, the
  bound of the mixed form; runs are deterministic.
"""
import ctypes as C

import numpy as np
import pytest

from relax_b200 import _lib
from relax_b200.api import Relax
from relax_b200.config import powerlaw_thrust

from cases import powerlaw_small, rel_l2
from test_gpu_step import compare

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dft64(x, inverse):
    lib = _lib.load()
    xi = np.ascontiguousarray(np.stack([x.real, x.imag], axis=-1).astype(np.float32))
    d_in = torch.from_numpy(xi).cuda()
    d_out = torch.zeros_like(d_in)
    _lib.check(lib.relax_op_dft64_tc(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), inverse, None))
    o = d_out.cpu().numpy().astype(np.float64)
    return o[..., 0] + 1j * o[..., 1]


@pytest.mark.parametrize("inverse", [0, 1])
def test_dft64_tensor_core_product_matches_numpy(inverse):
    rng = np.random.default_rng(3 + inverse)
    x = rng.standard_normal((128, 64)) + 1j * rng.standard_normal((128, 64))
    x[5] *= 1e3           # rows of very different scale: the split is relative
    x[9] *= 1e-3
    got = _dft64(x, inverse)
    want = np.fft.fft(x, axis=1) if inverse == 0 else 64.0 * np.fft.ifft(x, axis=1)
    for r in range(128):
        e = rel_l2(np.stack([got[r].real, got[r].imag]), np.stack([want[r].real, want[r].imag]))
        assert e < 3e-5, (r, e)


def _green_inputs(seed, sx1, sx2, sx3):
    rng = np.random.default_rng(seed)
    c = np.zeros((3, sx3, sx2, sx1 + 2), np.float32)
    c[:, : sx3 // 2, :, :sx1] = rng.standard_normal((3, sx3 // 2, sx2, sx1))
    t = np.zeros((3, sx2, sx1 + 2), np.float32)
    t[:, :, :sx1] = 0.1 * rng.standard_normal((3, sx2, sx1))
    return c, t


def _green_gpu(fn, c, t, sx1, sx2, sx3, dx, gam):
    dc = [torch.from_numpy(c[k].copy()).cuda() for k in range(3)]
    dt = [torch.from_numpy(t[k].copy()).cuda() for k in range(3)]
    _lib.check(fn(*[C.c_void_p(x.data_ptr()) for x in dc], *[C.c_void_p(x.data_ptr()) for x in dt],
                  sx1, sx2, sx3, *dx, 1.0, 1.0, gam, None))
    torch.cuda.synchronize()
    return np.stack([x.cpu().numpy() for x in dc])


# 64 x 32: 33 x 32 = 1056 columns, 16 full tiles and a partial one;
# 256 x 32 and 128 x 128: whole tiles only
@pytest.mark.parametrize("sx1,sx2", [(64, 32), (256, 32), (128, 128)])
@pytest.mark.parametrize("gam", [0.0, 8.3e-4])
def test_green_mixed_matches_oracle(oracle32, sx1, sx2, gam):
    lib = _lib.load()
    sx3, dx = 128, (0.5, 0.4, 0.25)
    c, t = _green_inputs(21, sx1, sx2, sx3)
    cr, tr = c.copy(), t.copy()
    oracle32.green(cr, tr, sx1, sx2, sx3, dx, 1.0, 1.0, gam)
    got = _green_gpu(lib.relax_op_green_mixed, c, t, sx1, sx2, sx3, dx, gam)
    h = sx3 // 2
    err = rel_l2(got[:, :h, :, :sx1], cr[:, :h, :, :sx1])
    assert err < 1e-4, err
    # and the plain FP32 operator on the same input
    plain = _green_gpu(lib.relax_op_green, c, t, sx1, sx2, sx3, dx, gam)
    assert rel_l2(got[:, :h, :, :sx1], plain[:, :h, :, :sx1]) < 1e-4


def test_green_mixed_rejects_other_depths():
    lib = _lib.load()
    c = torch.zeros((3, 64, 32, 66), device="cuda")
    t = torch.zeros((3, 32, 66), device="cuda")
    rc = lib.relax_op_green_mixed(*[C.c_void_p(c[k].data_ptr()) for k in range(3)],
                                  *[C.c_void_p(t[k].data_ptr()) for k in range(3)],
                                  64, 32, 64, 1.0, 1.0, 1.0, 1.0, 1.0, 0.0, None)
    assert rc == 4


def _mixed_run(sim, nsteps):
    with Relax(sim) as r:
        r.set_precision("mixed")
        logs = [r.coseismic()]
        for _ in range(nsteps):
            logs.append(r.step())
        fields = {k: r.field(k) for k in ("u", "sig", "tau", "gamma")}
    return logs, fields


@pytest.mark.parametrize("builder,nsteps", [(lambda: powerlaw_small(sx=32, sz=128), 1),
                                            (lambda: powerlaw_small(sx=32, sz=128), 6),
                                            (lambda: powerlaw_thrust(sx=256, sz=128, dx=0.5), 4)])
def test_mixed_steps_match_oracles(oracle32, oracle64, builder, nsteps):
    sim = builder()
    glogs, gf = _mixed_run(sim, nsteps)
    dts = [lg[1] for lg in glogs[1:]]
    _, df = oracle64.run(sim, nsteps, dt_schedule=dts)
    compare(gf, df, 1e-4)
    rlogs, rf = oracle32.run(sim, nsteps, dt_schedule=dts)
    compare(gf, rf, 1e-4)
    # logs: Dt, t, power and C:E^i to 1e-3; the Maxwell times (minima over the
    # grid of 1/gammadot ~ stress^(1 - n)) carry (n - 1) times the stress
    # error of the mixed form, hence 2e-4
    assert len(glogs) == len(rlogs)
    for g, o in zip(glogs, rlogs):
        assert g[0] == o[0]
        for c in (1, 5, 6, 7):
            assert abs(g[c] - o[c]) <= 1e-3 * max(abs(o[c]), 1e-30), (g, o, c)
        for c in (2, 3, 4):
            assert abs(g[c] - o[c]) <= 2e-4 * abs(o[c]), (g, o, c)


def test_mixed_runs_are_deterministic_and_replay_as_a_graph():
    """No atomics on the data path: two mixed runs are bitwise identical
    (the later steps of each are replayed from a captured graph)."""
    sim = powerlaw_small(sx=32, sz=128)
    a = _mixed_run(sim, 4)
    b = _mixed_run(sim, 4)
    assert a[0] == b[0]
    for k in a[1]:
        assert np.array_equal(a[1][k].view(np.uint8), b[1][k].view(np.uint8)), k


def test_precision_mode_is_checked():
    sim = powerlaw_small()          # 32 deep
    with Relax(sim) as r:
        with pytest.raises(_lib.RelaxError) as e:
            r.set_precision("mixed")
        assert e.value.code == 4
        r.set_precision("fp32")
