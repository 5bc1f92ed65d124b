"""GPU image rendering against the reference's own write_image
(src/main.cpp:556-678), run in-process through the oracle harness. With an
integer brightness every per-pixel sum is exact, so the bitmaps must be equal
byte for byte."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [  # projection, color, adaptive, nonlinear, scale, brightness
    (3, 0, False, False, 1.0, 255.0),   # the reference's defaults
    (0, 0, False, False, 1.0, 40.0),
    (1, 1, False, False, 1.5, 60.0),
    (2, 1, True, False, 0.75, 1.0),
    (3, 0, True, True, 2.0, 3.0),
    (0, 1, True, True, 1.0, 7.0),
    (2, 0, False, True, 1.0, 20.0),
    (3, 1, True, False, 1.0, 1.0),
]


@pytest.fixture(scope="module")
def cloud(nb):
    pos, vel, mass = nb.generate(20000, gen_type=1, size=400.0)  # sphere; some particles land off-image
    return pos, vel, mass


@pytest.mark.parametrize("w,h", [(320, 200), (200, 320)])  # y is bounded by the width in the reference
@pytest.mark.parametrize("case", CASES)
def test_render_matches_reference(nb, ref, cloud, w, h, case):
    proj, color, adaptive, nonlinear, scale, brightness = case
    pos, vel, mass = cloud
    want = ref.write_image(pos, w, h, proj, color, adaptive, nonlinear, scale, brightness)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        got = e.render(width=w, height=h, projection=proj, color=color, adaptive=int(adaptive),
                       nonlinear=int(nonlinear), scale=scale, brightness=brightness)
    assert got.shape == want.shape
    assert np.array_equal(got, want), np.argwhere(got != want)[:5]


def test_render_after_steps_and_empty_image(nb, ref):
    pos, vel, mass = nb.generate(3000, gen_type=0, size=100.0)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        e.step(3)
        p, _ = e.get_particles()
        got = e.render(width=64, height=48, projection=0, brightness=9.0)
        assert np.array_equal(got, ref.write_image(p, 64, 48, 0, 0, False, False, 1.0, 9.0))
        # everything off-image: adaptive divides 0 by a zero maximum (NaN), as the reference does
        e.set_particles(pos + 1e6, vel, mass)
        for color in (0, 1):
            got = e.render(width=32, height=32, projection=2, color=color, adaptive=1, nonlinear=1)
            assert np.array_equal(got, ref.write_image(pos + 1e6, 32, 32, 2, color, True, True, 1.0, 255.0))


def test_render_rejects_bad_params(nb):
    pos, vel, mass = nb.generate(100)
    with nb.Engine() as e:
        with pytest.raises(nb.NBodyError):
            e.render(width=16, height=16)  # no particles set yet
        e.set_particles(pos, vel, mass)
        for bad in (dict(width=0), dict(projection=4), dict(color=2)):
            with pytest.raises(nb.NBodyError):
                e.render(**{"width": 16, "height": 16, **bad})
