"""Host-side pieces of the inverse-rendering fit (no GPU): the per-pixel
image-gradient clip that fit(grad_quantile=...) applies."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import inverse


def test_clip_quantile_caps_only_the_tail():
    rng = np.random.default_rng(0)
    g = rng.normal(size=(64, 64, 3)).astype(np.float32)
    g[3, 5, 1] = 1e4          # a firefly's residual
    g[10, 2, 0] = -2e4
    t = torch.tensor(g)
    c = inverse.clip_quantile(t, 0.999)
    thr = float(torch.quantile(t.abs().flatten(), 0.999))
    assert c.shape == t.shape
    assert float(c.abs().max()) <= thr * 1.01
    assert float(c[3, 5, 1]) > 0 > float(c[10, 2, 0])
    # entries below the threshold are untouched
    small = t.abs() < 0.5 * thr
    assert torch.equal(c[small], t[small])


def test_clip_quantile_subsamples_large_images():
    t = torch.linspace(-1.0, 1.0, 3 * 1024 * 1024).reshape(1024, 1024, 3)
    c = inverse.clip_quantile(t, 0.99)
    assert abs(float(c.max()) - 0.99) < 0.01 and abs(float(c.min()) + 0.99) < 0.01
