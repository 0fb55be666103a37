"""Progressive photon mapping (caustic mode 1, configuration 2's extension of
the reference's single kNN pass): sample s uses photon pass
min(s / spp_per_pass, passes - 1), emitted from its own streams and gathered
within radius * shrink^(2 pass) (the radius option is compared against
squared distances, get_caustic.c:45).

 * the image does not depend on how the samples are split into calls, nor on
   their order (passes are re-emitted deterministically);
 * the fixed-radius estimate of a pass equals the direct sum over that
   pass's photons (read back from the device) within its radius, / (pi r^2)
   / norm, at query points on the caustic.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_c2p(scenes):
    return scenes.make_c2(width=64, height=48, spp=8, depth=6, grid=64, photons=20000, passes=4,
                          mode=1, spp_per_pass=2)


@pytest.fixture(scope="module")
def built(mrt, scenes, oracle):
    lib = mrt.load()
    assert lib.mrt_device_count() > 0, "gpu tests need a CUDA device"
    sc = small_c2p(scenes)
    return sc, oracle.canonical_scene(sc)


def _ctx(mrt, sc, cs):
    c = mrt.Context(sc.width, sc.height)
    c.build(cs)
    return c


def test_split_and_order_do_not_change_the_image(mrt, built):
    sc, cs = built
    a = _ctx(mrt, sc, cs)
    a.render(8, seed=3, sample_base=0, form=mrt.FORM_MEGAKERNEL)
    img_a, n_a = a.read_accum()
    b = _ctx(mrt, sc, cs)
    for s in reversed(range(8)):
        b.render(1, seed=3, sample_base=s, form=mrt.FORM_MEGAKERNEL)
    img_b, n_b = b.read_accum()
    assert n_a == n_b == 8
    np.testing.assert_allclose(img_a, img_b, rtol=1e-5, atol=1e-6)
    # the wavefront form follows the same pass schedule
    c = _ctx(mrt, sc, cs)
    c.render(8, seed=3, sample_base=0, form=mrt.FORM_WAVEFRONT)
    img_c, _ = c.read_accum()
    np.testing.assert_allclose(img_c, img_a, rtol=1e-4, atol=1e-5)
    assert np.abs(img_a).sum() > 0


@pytest.mark.parametrize("q", [0, 3])
def test_pass_estimate_is_the_fixed_radius_sum(mrt, built, q):
    sc, cs = built
    c = _ctx(mrt, sc, cs)
    c.render(1, seed=3, sample_base=q * 2, form=mrt.FORM_MEGAKERNEL)   # builds pass q
    pos, pw = c.photons()
    assert len(pos) > 1000
    r2 = sc.caustic["radius"] * sc.caustic["shrink"] ** (2 * q)
    rng = np.random.default_rng(q)
    pts = pos[rng.choice(len(pos), 200, replace=False)].astype(np.float64)
    pts += rng.normal(scale=0.3 * np.sqrt(r2), size=pts.shape)
    got = c.caustic_query(pts)
    d2 = ((pos[None, :, :].astype(np.float64) - pts[:, None, :]) ** 2).sum(-1)
    want = (d2 <= r2).astype(np.float64) @ pw.astype(np.float64) / (np.pi * r2) / sc.caustic["norm"]
    # photons within float rounding of the radius may fall either side
    close = np.abs(np.sqrt(d2) - np.sqrt(r2)) < 1e-5
    ok = ~close.any(axis=1)
    assert ok.mean() > 0.9
    np.testing.assert_allclose(got[ok], want[ok], rtol=1e-4, atol=1e-6)
    if q:
        # the pass really is a different photon set from pass 0
        c.render(1, seed=3, sample_base=0, form=mrt.FORM_MEGAKERNEL)
        pos0, _ = c.photons()
        assert not np.array_equal(np.sort(pos0[:, 0]), np.sort(pos[:, 0]))
