"""The C ABI on a machine without a GPU: the library loads, exports what
include/relax_b200.h declares, its host helpers agree with the oracle, and
the compute path fails loudly instead of falling back to the CPU."""
import ctypes as C
import math

import pytest

from relax_b200 import _lib
from relax_b200.config import (powerlaw_thrust, reference_output2, relax_layer, wang_convention)


def test_library_exports_every_declared_function():
    lib = _lib.load()
    names = _lib.header_functions()
    assert "relax_create" in names and "calfftnelasic_" in names and "custressupdatewrapper_" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []
    assert lib.relax_version().startswith(b"relax_b200")


@pytest.mark.parametrize("builder", [powerlaw_thrust, reference_output2])
def test_structure_expansion_matches_oracle(oracle32, builder):
    sim = builder()
    lin, non, fc = sim.layer_lists()
    for layers in (non, fc):
        if not layers:
            continue
        a = _lib.structure_fn(layers, sim.dx3, sim.sx3h)
        b = oracle32.structure_fn(layers, sim.dx3, sim.sx3h)
        for k in range(sim.sx3h):
            for f, _ in relax_layer._fields_:
                assert getattr(a[k], f) == getattr(b[k], f), (k, f)


def test_structure_rejects_decreasing_depths():
    layers = [relax_layer(z=5.0, gammadot0=1, stressexponent=1), relax_layer(z=1.0, gammadot0=1, stressexponent=1)]
    with pytest.raises(_lib.RelaxError) as e:
        _lib.structure_fn(layers, 0.5, 32)
    assert e.value.code == 1


def test_wang_convention_matches_input_semantics():
    lib = _lib.load()
    args = (1.5, -3.0, 2.0, 0.5, 20.0, 8.0, 30.0, 60.0, 90.0)
    ref = wang_convention(*args, 1.0, -2.0, 15.0)
    vals = [C.c_double(v) for v in (args[0], args[1], args[2], args[3])]
    strike, dip, rake = C.c_double(args[6]), C.c_double(args[7]), C.c_double(args[8])
    lib.relax_wang_convention.restype = None
    lib.relax_wang_convention(C.byref(vals[0]), C.byref(vals[1]), C.byref(vals[2]), C.byref(vals[3]),
                              C.c_double(args[4]), C.c_double(args[5]), C.byref(strike), C.byref(dip),
                              C.byref(rake), C.c_double(1.0), C.c_double(-2.0), C.c_double(15.0))
    got = (vals[0].value, vals[1].value, vals[2].value, vals[3].value, strike.value, dip.value, rake.value)
    for a, b in zip(got, ref):
        assert math.isclose(a, b, rel_tol=1e-15, abs_tol=1e-15)


def test_no_cpu_fallback_without_a_gpu():
    """relax_create on a host without a usable CUDA device returns an error
    (no silent CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    sim = powerlaw_thrust(sx=32, sz=32, dx=2.0)
    cfg, keep = sim.to_c(_lib.structure_fn)
    h = C.c_void_p()
    rc = lib.relax_create(C.byref(cfg), 0, C.byref(h))
    assert rc == 2 and not h.value
    assert b"cuda" in lib.relax_last_error().lower() or len(lib.relax_last_error()) > 0
