"""render_state.rts checkpoints (export_render_state.c:15-51): the file
layout on the host, and save / load of the device accumulator."""
from __future__ import annotations

import numpy as np
import pytest


def test_rts_layout_roundtrip(mrt, tmp_path):
    rng = np.random.default_rng(0)
    fr = rng.uniform(0, 40, (6, 10, 3))
    p = tmp_path / "render_state.rts"
    mrt.write_rts(p, fr, 37)
    raw = p.read_bytes()
    assert len(raw) == 12 + 6 * 10 * 3 * 8
    assert tuple(np.frombuffer(raw[:12], "<i4")) == (10, 6, 37)
    back, sample = mrt.read_rts(p)
    assert sample == 37
    np.testing.assert_array_equal(back, fr)
    p.write_bytes(raw[:-8])
    with pytest.raises(ValueError):
        mrt.read_rts(p)


@pytest.mark.gpu
def test_save_load_continues_the_render(mrt, oracle, scenes, tmp_path):
    """Render 4 spp, save, load into a fresh context, render 4 more from
    sample 4: the same as 8 spp in one context (float sums, up to the order
    of the atomic additions)."""
    sc = scenes.make_c0(0, 40, 30, depth=6)
    a = mrt.Context(40, 30)
    a.build(sc)
    a.render(4, seed=9)
    p = tmp_path / "render_state.rts"
    a.save_state(p)
    fr, sample = mrt.read_rts(p)
    img, n = a.read_accum()
    assert sample == n == 4
    np.testing.assert_array_equal(fr.astype(np.float32), img)
    b = mrt.Context(40, 30)
    b.build(sc)
    b.load_state(p)
    b.render(4, seed=9, sample_base=4)
    cont, m = b.read_accum()
    assert m == 8
    a.render(4, seed=9, sample_base=4)
    ref, _ = a.read_accum()
    np.testing.assert_allclose(cont, ref, rtol=1e-5, atol=1e-5)
    c = mrt.Context(20, 30)
    c.build(scenes.make_c0(0, 20, 30, depth=6))
    with pytest.raises(mrt.MRTError, match="40x30"):
        c.load_state(p)
