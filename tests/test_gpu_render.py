"""Headless rasterizer on the GPU (lima_render, lima_render_image) against
the oracle's restatement of Rasterizer.cu and the display's shaded discs:
ball lists and images bit-identical, in both semantics.  The restatement's
ball list is itself pinned to the reference's Rasterizer run on the host
(tests/test_render_pin.py); here the GPU list is also compared with that
reference run directly, on a box where most depths are tied."""
import numpy as np
import pytest

from oracle import pyoracle as po
from quantom_b200 import systems as S

pytestmark = pytest.mark.gpu


def _params(E, s, semantics):
    if semantics == "physics":
        return E.default_params(box_len=s.spec.box_len, cutoff=s.spec.cutoff, dt=s.spec.dt,
                                semantics=E.SEMANTICS_PHYSICS, skin=0.1, switch_on=1.0, nlist_period=0)
    return E.default_params(box_len=s.spec.box_len, cutoff=s.spec.cutoff, dt=s.spec.dt)


@pytest.mark.parametrize("semantics", ["physics", "reference"])
@pytest.mark.parametrize("name", ["tiny_chains", "small_bridged"])
def test_balls_and_image_match_oracle(gpu, name, semantics):
    E = gpu
    s = S.make_system(name, seed=11)
    with E.Engine(s, _params(E, s, semantics)) as eng:
        eng.step(13)
        balls = eng.render()
        img = eng.render_image(320, 240)
        img2 = eng.render_image(1080, 1080)
        st, _ = eng.compound_states()
        sol = eng.solvents()["pos"]
    pos, kind = po.render_slots(s, [st[c]["positions"] for c in range(s.n_compounds)], sol)
    ref = po.render_balls(pos, kind, s.spec.box_len)
    assert balls.tobytes() == ref.tobytes()
    np.testing.assert_array_equal(img, po.render_image(ref, 320, 240))
    np.testing.assert_array_equal(img2, po.render_image(ref, 1080, 1080))
    assert img2.any(2).mean() > 0.05


def test_ppm_file(gpu, tmp_path):
    E = gpu
    s = S.make_system("tiny_chains", seed=11)
    with E.Engine(s, _params(E, s, "physics")) as eng:
        img = eng.render_image(64, 48)
    E.save_ppm(tmp_path / "frame.ppm", img)
    data = (tmp_path / "frame.ppm").read_bytes()
    assert data.startswith(b"P6\n64 48\n255\n") and data[len(b"P6\n64 48\n255\n"):] == img.tobytes()


def test_balls_match_reference_rasterizer(gpu):
    """Reference semantics, the state as loaded and after 3 steps, and a
    lattice box of tied depths: the GPU ball list equals the one the
    reference's own Rasterizer kernels and merge sort make (oracle/_ref)."""
    from test_render_pin import _lattice_box, FIELDS
    if not po.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    E = gpu
    for s, steps in ((S.make_system("tiny_chains", seed=11), 0), (S.make_system("small_bridged", seed=11), 3),
                     (_lattice_box(8, 4.0), 0)):
        ref = po.RefEngine(s, n_threads=4)
        if steps:
            ref.update_nlists()
            ref.step(steps)
        want = ref.render()
        ref.close()
        with E.Engine(s, _params(E, s, "reference")) as eng:
            eng.step(steps)
            got = eng.render()
        for f in FIELDS:
            a, b = got[f], want[f]
            if a.dtype.kind == "f":
                a, b = a.view(np.uint32), b.view(np.uint32)
            assert np.array_equal(a, b), (s.spec.name, f)
