"""The MIXED adjoint writes its pair terms with the unit offset u = d / r
(walk.cu, pair_adjoint for FP32) so that no factor overflows FP32; the FP64
form keeps the textbook expression with h = g'(r) / r. Both must be the same
function of (d, G m, dL/da): checked here in FP64 over nine decades of r."""
import numpy as np

G = 6.67384e-11


def textbook(d, gm, la, damp):
    r2 = (d * d).sum(1)
    inv = 1.0 / np.sqrt(r2)
    inv2 = inv * inv
    if damp:
        r = r2 * inv
        e = np.exp(-r)
        den = r2 + e
        g = inv / den
        h = -(3 * r2 + e - r * e) * inv2 * inv / (den * den)
    else:
        g = inv * inv2
        h = -3 * g * inv2
    s = (d * la).sum(1)
    v = gm[:, None] * (g[:, None] * la + (h * s)[:, None] * d)
    return v, G * g * s


def unit_offset(d, gm, la, damp):
    r2 = (d * d).sum(1)
    inv = 1.0 / np.sqrt(r2)
    u = d * inv[:, None]
    sh = (u * la).sum(1)
    if damp:
        r = r2 * inv
        e = np.exp(-r)
        den = r2 + e
        g = inv / den
        gr = 1.0 / den
        hr2 = -(3 * r2 + e - r * e) * inv / (den * den)
    else:
        gr = inv * inv
        g = gr * inv
        hr2 = -3 * g
    v = gm[:, None] * (g[:, None] * la + (hr2 * sh)[:, None] * u)
    return v, G * gr * sh


def test_unit_offset_form_equals_textbook_form():
    rng = np.random.default_rng(0xDEADBEEF)
    k = 4000
    d = rng.normal(size=(k, 3)) * 10.0 ** rng.uniform(-4, 5, size=(k, 1))
    gm = G * rng.uniform(5e10, 5e11, size=k)
    la = rng.normal(size=(k, 3))
    for damp in (False, True):
        v0, m0 = textbook(d, gm, la, damp)
        v1, m1 = unit_offset(d, gm, la, damp)
        scale = np.linalg.norm(v0, axis=1)
        assert (np.linalg.norm(v1 - v0, axis=1) <= 1e-12 * scale).all()
        assert (np.abs(m1 - m0) <= 1e-12 * np.abs(m0) + 1e-300).all()
