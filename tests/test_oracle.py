"""The CPU oracle against analytic known answers and numpy.fft.

The oracle restates the reference CPU path; these checks pin its pieces
independently of the captured reference logs (tests/test_oracle_pins.py).
"""
import math

import numpy as np
import pytest

from relax_b200.config import relax_layer


@pytest.mark.parametrize("n", [2, 3, 4, 8, 12, 64, 96, 128, 192, 256, 512, 10, 7])
def test_complex_fft_matches_numpy(oracle64, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign, ref in ((-1, np.fft.fft(x)), (+1, np.fft.ifft(x) * n)):
        got = oracle64.fft_c(x, sign)
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("prec,tol", [(32, 3e-7), (64, 1e-14)])
@pytest.mark.parametrize("shape", [(16, 12, 8), (32, 32, 16), (24, 8, 12)])
def test_fft3_normalisation_and_layout(prec, tol, shape):
    """fft3 = numpy rfftn x dx1 dx2 dx3 in the in-place (sx1+2) layout
    (src/fourier.f90:177-201); inverse divides by sx1 dx1 sx2 dx2 sx3 dx3."""
    from oracle.oracle import Oracle
    o = Oracle(prec)
    sx1, sx2, sx3 = shape
    dx = (0.5, 0.7, 0.3)
    rng = np.random.default_rng(1)
    a = np.zeros((sx3, sx2, sx1 + 2), o.real)
    a[:, :, :sx1] = rng.standard_normal((sx3, sx2, sx1))
    ref = np.fft.rfftn(a[:, :, :sx1].astype(np.float64), axes=(0, 1, 2)) * (dx[0] * dx[1] * dx[2])
    b = a.copy()
    o.fft3(b, sx1, sx2, sx3, *dx, -1)
    got = b.view(np.complex64 if prec == 32 else np.complex128)
    assert np.abs(got - ref).max() <= tol * 10 * np.abs(ref).max()
    o.fft3(b, sx1, sx2, sx3, *dx, +1)
    assert np.abs(b[:, :, :sx1] - a[:, :, :sx1]).max() <= tol * 10 * np.abs(a).max()


def _tensor_field(o, shape, rng, const=None):
    t = np.zeros(shape, o.tensor)
    for n in o.tensor.names:
        t[n] = const if const is not None else rng.standard_normal(shape)
    return t


def test_divergence_of_constant_tensor_is_zero(oracle64):
    o = oracle64
    sx1, sx2, sx3h = 16, 16, 8
    sig = _tensor_field(o, (sx3h, sx2, sx1), None, const=0.7)
    c = np.zeros((3, sx3h, sx2, sx1 + 2), o.real)
    t = np.zeros((3, sx2, sx1 + 2), o.real)
    o.bodyforce(sig, (0.5, 0.5, 0.5), sx1, sx2, sx3h, c, t)
    assert np.abs(c).max() == 0.0
    assert np.allclose(t[:, :, :sx1], 0.7)


def test_linear_maxwell_time_is_inverse_fluidity(oracle32):
    """Linear viscosity: tm = 1/gammadot0 exactly (src/viscoelastic3d.f90:303)."""
    o = oracle32
    sx1, sx2, sx3h = 16, 16, 8
    rng = np.random.default_rng(3)
    sig = _tensor_field(o, (sx3h, sx2, sx1), rng)
    layers = [relax_layer(z=0.0, gammadot0=4.0, stressexponent=1.0, cohesion=0.0, friction=0.0,
                          Gk=0.0)]
    st = o.structure_fn(layers, 0.5, sx3h)
    mom = np.zeros_like(sig)
    rc, tm = o.viscouseigenstress(1.0, st, None, sig, sx1, sx2, sx3h, mom, maxwell=1e7)
    assert rc == 0 and tm == np.float32(0.25)
    # moment = 2 gammadot0 dev(sig) for n = 1
    tr = (sig["s11"] + sig["s22"] + sig["s33"]) / 3
    assert np.allclose(mom["s11"], 8.0 * (sig["s11"] - tr), rtol=1e-5, atol=1e-5)
    assert np.allclose(mom["s12"], 8.0 * sig["s12"], rtol=1e-6)


def test_elastic_response_solves_navier(oracle64):
    """elasticresponse (src/green.f90:51-101) inverts the Navier operator:
    4 pi^2 [mu k^2 u + (lambda+mu) k (k.u)] = f for every k != 0."""
    from oracle.oracle import ptr
    o = oracle64
    sx1, sx2, sx3 = 16, 8, 12
    dx = (0.5, 0.25, 0.4)
    lam, mu = 1.7, 0.9
    rng = np.random.default_rng(4)
    f = [np.ascontiguousarray(rng.standard_normal((sx3, sx2, sx1 + 2))) for _ in range(3)]
    u = [a.copy() for a in f]
    o.lib.orc_elasticresponse(lam, mu, ptr(u[0]), ptr(u[1]), ptr(u[2]), sx1, sx2, sx3, *dx)
    fc = [a.view(np.complex128) for a in f]
    uc = [a.view(np.complex128) for a in u]
    k1 = np.arange(sx1 // 2 + 1) / (sx1 * dx[0])
    k2 = np.fft.fftfreq(sx2, dx[1])
    k3 = np.fft.fftfreq(sx3, dx[2])
    K3, K2, K1 = np.meshgrid(k3, k2, k1, indexing="ij")
    k = [K1, K2, K3]
    kk = K1 ** 2 + K2 ** 2 + K3 ** 2
    kdotu = sum(k[i] * uc[i] for i in range(3))
    for i in range(3):
        lhs = 4 * math.pi ** 2 * (mu * kk * uc[i] + (lam + mu) * k[i] * kdotu)
        mask = kk > 0
        assert np.abs(lhs[mask] - fc[i][mask]).max() < 1e-10 * np.abs(fc[i]).max()
        assert uc[i][0, 0, 0] == 0


def test_green_function_free_surface(oracle64):
    """Body force only, no gravity: the surface-traction correction
    (surfacetractioncowling + cerrutimodified, src/green.f90:327-612) at
    least halves the traction sigma_i3(x3=0) the full-space solution leaves
    on a shallow source (the periodic-in-x3 Cerruti kernel and the one-sided
    finite difference at the surface, src/elastic3d.f90:977-1002, bound how
    close to zero it gets)."""
    from oracle.oracle import ptr
    o = oracle64
    sx1 = sx2 = 64
    sx3 = 64
    dx = (1.0, 1.0, 1.0)
    x = (np.arange(sx1) - sx1 / 2) * dx[0]
    X3, X2, X1 = np.meshgrid(np.arange(sx3) * dx[2], x, x, indexing="ij")
    blob = np.exp(-((X1) ** 2 + (X2) ** 2 + (X3 - 8.0) ** 2) / 8.0)
    blob[sx3 // 2:] = 0
    c0 = np.zeros((3, sx3, sx2, sx1 + 2))
    c0[0, :, :, :sx1] = np.fft.ifftshift(blob, axes=(1, 2))
    c0[2, :, :, :sx1] = 0.5 * np.fft.ifftshift(blob, axes=(1, 2))

    def surface_traction(c):
        u = np.ascontiguousarray(c[:, : sx3 // 2])
        sig = np.zeros((sx3 // 2, sx2, sx1), o.tensor)
        o.stressupdate(u, 1.0, 1.0, dx, sx1, sx2, sx3 // 2, sig)
        scale = max(np.abs(sig[n]).max() for n in o.tensor.names)
        return max(np.abs(sig[n][0]).max() for n in ("s13", "s23", "s33")) / scale

    c = c0.copy()
    t = np.zeros((3, sx2, sx1 + 2))
    o.green(c, t, sx1, sx2, sx3, dx, 1.0, 1.0, 0.0)
    full = c0.copy()
    for k in range(3):
        o.fft3(full[k], sx1, sx2, sx3, *dx, -1)
    o.lib.orc_elasticresponse(1.0, 1.0, ptr(full[0]), ptr(full[1]), ptr(full[2]), sx1, sx2, sx3,
                              *dx)
    for k in range(3):
        o.fft3(full[k], sx1, sx2, sx3, *dx, +1)
    assert surface_traction(c) < 0.55 * surface_traction(full)
