"""Multi-GPU sample sharding through the C-ABI (mrt_comm_* and
mrt_reduce_frame over NCCL) on the one GPU a test run has.

Two ranks cannot share one GPU in an NCCL communicator, and kernels of
different ranks must not wait on one another on one device, so the
multi-rank reduce itself is not exercised here: the tests check (a) that
shards rendered separately sum to the single render of all their samples
(the arithmetic every rank relies on), and (b) a world-size-1 communicator
end to end (unique id, init, reduce, destroy) through libmrt."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def require_device(mrt):
    lib = mrt.load()
    assert lib.mrt_device_count() > 0, "gpu tests need a CUDA device"


def test_sample_shards_sum_to_the_single_render(mrt, oracle, scenes):
    sc = scenes.make_c0(0, 64, 48, depth=6)
    total, world = 12, 3
    full = mrt.Context(sc.width, sc.height)
    full.build(oracle.canonical_scene(sc))
    full.render(total, seed=5, sample_base=0, form=mrt.FORM_WAVEFRONT)
    ref, n = full.read_accum()
    assert n == total
    parts = []
    for r in range(world):
        first, count = mrt.shard_samples(total, world, r)
        ctx = mrt.Context(sc.width, sc.height)
        ctx.build(oracle.canonical_scene(sc))
        ctx.render(count, seed=5, sample_base=first, form=mrt.FORM_WAVEFRONT)
        img, k = ctx.read_accum()
        assert k == count
        parts.append(img.astype(np.float64))
        ctx.close()
    summed = np.sum(parts, axis=0)
    # same paths, different float summation order (per-shard atomics)
    np.testing.assert_allclose(summed, ref, rtol=2e-5, atol=1e-5 * float(np.abs(ref).max()))
    full.close()


def test_world_one_communicator_reduce(mrt, oracle, scenes):
    sc = scenes.make_c0(0, 48, 32, depth=4)
    ctx = mrt.Context(sc.width, sc.height)
    ctx.build(oracle.canonical_scene(sc))
    cid = mrt.comm_unique_id()
    assert len(cid) == mrt.COMM_ID_BYTES
    ctx.comm_init(cid, 0, 1)
    with pytest.raises(mrt.MRTError):
        ctx.comm_init(cid, 0, 1)          # one communicator per context
    ctx.render(4, seed=3)
    before, n0 = ctx.read_accum()
    ctx.reduce_frame(0)
    after, n1 = ctx.read_accum()
    assert n0 == n1 == 4
    np.testing.assert_array_equal(before, after)
    with pytest.raises(mrt.MRTError):
        ctx.reduce_frame(1)               # root outside the world
    ctx.comm_destroy()
    with pytest.raises(mrt.MRTError):
        ctx.reduce_frame(0)               # no communicator any more
    ctx.close()
