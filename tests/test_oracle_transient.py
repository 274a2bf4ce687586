"""The oracle's transient (Burgers) rheology, transienteigenstress
(src/viscoelastic3d.f90:123-202) in the RK2 loop (src/relax.f90:614-645,
:693-695, :764-790), pinned where it has a closed form: with a linear
transient layer (exponent 1) the strain rate is gammadot0 whatever the
stress, so tm(transient) = 1/gammadot0 and Dt = tm/10 * tscale exactly."""
import numpy as np

from cases import rel_l2, tensor_array, transient_small


def test_linear_transient_maxwell_time_is_exact(oracle32):
    sim = transient_small(linear=True)
    logs, out = oracle32.run(sim, 2, fields=False)
    for (tl, tnl), lg in zip(out["tm_transient"][1:], logs[1:]):
        assert tl == 1.0
        assert lg[1] == 0.5            # Dt = 1/10 * tscale(5)


def test_transient_fp32_and_fp64_oracles_agree(oracle32, oracle64):
    sim = transient_small(linear=True, nonlinear=True, viscous=True)
    l32, f32 = oracle32.run(sim, 3)
    dts = [l[1] for l in l32[1:]]
    l64, f64 = oracle64.run(sim, 3, dt_schedule=dts)
    assert rel_l2(f32["u"][..., :-2], f64["u"][..., :-2]) < 1e-5
    assert rel_l2(tensor_array(f32["tau"]), tensor_array(f64["tau"])) < 1e-5


def test_transient_strain_relaxes_stress(oracle32):
    """the transient creep changes the stress field relative to the elastic run"""
    el = transient_small(linear=False)
    tr = transient_small(linear=True)
    _, fe = oracle32.run(el, 2)
    _, ft = oracle32.run(tr, 2)
    d = rel_l2(tensor_array(ft["tau"]), tensor_array(fe["tau"]))
    assert d > 1e-4
