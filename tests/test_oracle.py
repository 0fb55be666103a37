"""Pins the FP64 oracle restatement (oracle/mrt_oracle.c) against the
reference's own outputs: the committed golden fixtures (made by
tests/golden/make_golden.py from the compiled reference) and, where the
reference is built here, the live reference on fresh seeds. All comparisons
are bit-exact: the restatement reproduces the reference's arithmetic."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden



@pytest.fixture(scope="module")
def mg():
    import sys
    from conftest import GOLDEN
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    return make_golden


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "q0", "t0"])
def test_scene_generator_is_deterministic(mg, name):
    g = golden(f"{name}_pins.npz")
    sc = mg.CASES[name]["make"]()
    assert mg.scene_digest(sc) == str(g["digest"])


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "q0", "t0"])
def test_first_hits_match_reference_golden(mg, oracle, name):
    g = golden(f"{name}_pins.npz")
    sc = mg.CASES[name]["make"]()
    oracle.Restatement.set_seed(4242)
    ro = oracle.Restatement(sc)
    h = ro.first_hit(g["rays_o"], g["rays_d"])
    for f in ("prim", "front_face", "depth", "t", "u", "v", "point", "normal", "color"):
        np.testing.assert_array_equal(h[f], g["hit_" + f], err_msg=f)
    assert (g["hit_prim"] >= 0).sum() > 100


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "q0", "t0"])
def test_render_matches_reference_golden_bit_exact(mg, oracle, name):
    g = golden(f"{name}_pins.npz")
    sc = mg.CASES[name]["make"]()
    oracle.Restatement.set_seed(4242)
    ro = oracle.Restatement(sc)
    oracle.Restatement.set_seed(int(g["render_seed"]))
    acc = ro.render_reference(int(g["render_spp"]))
    np.testing.assert_array_equal(acc, g["render"])


def test_env_tables_match_reference_golden(mg, oracle):
    g = golden("c1_pins.npz")
    ro = oracle.Restatement(mg.CASES["c1"]["make"]())
    pdf, cm, cc, avg = ro.env_tables()
    np.testing.assert_array_equal(pdf, g["pdf_joint"])
    np.testing.assert_array_equal(cm, g["cdf_m_inv"])
    np.testing.assert_array_equal(cc, g["cdf_c_inv"])
    assert avg == float(g["column_average"])


def test_photon_map_and_caustics_match_reference_golden(mg, oracle):
    g = golden("c2_pins.npz")
    oracle.Restatement.set_seed(4242)
    ro = oracle.Restatement(mg.CASES["c2"]["make"]())
    pos, pw, leaf = ro.photons()
    np.testing.assert_array_equal(pos, g["photon_pos"])
    np.testing.assert_array_equal(pw, g["photon_pow"])
    np.testing.assert_array_equal(leaf, g["photon_in_leaf"])
    np.testing.assert_array_equal(ro.caustic_query(g["caustic_q"], 15), g["caustic_rgb"])


def test_mesh_retransform_matches_reference_golden(mg, oracle):
    g = golden("c1_pins.npz")
    ro = oracle.Restatement(mg.CASES["c1"]["make"]())
    np.testing.assert_array_equal(ro.triangle_positions(), g["tri_positions"])


def test_pcg_stream_matches_python_restatement(oracle):
    """The counter RNG shared with the kernels: splitmix64 seeding + PCG32."""
    M = (1 << 64) - 1

    def splitmix(z):
        z = (z + 0x9E3779B97F4A7C15) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    def stream(seed, pixel, sample, n):
        s = splitmix(seed ^ splitmix((sample << 32) | pixel))
        out = []
        for _ in range(n):
            old = s
            s = (old * 6364136223846793005 + 1442695040888963407) & M
            xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
            rot = old >> 59
            v = ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF
            out.append((v >> 8) / 16777216.0)
        return np.array(out, np.float32)

    for args in [(1, 0, 0), (7, 12345, 3), (2**40 + 3, 2**31 - 1, 4095)]:
        np.testing.assert_array_equal(oracle.pcg_stream(*args, 16), stream(*args, 16))


@pytest.mark.parametrize("name,seed", [("c0", 11), ("c1", 12), ("c2", 13), ("q0", 14), ("t0", 15)])
def test_restatement_matches_live_reference(mg, oracle, has_reference, name, seed):
    if not has_reference:
        pytest.skip("reference not built here (oracle/_ref)")
    sc = mg.CASES[name]["make"]()
    oracle.ref_lib().refh_set_seed(seed)
    ref = oracle.RefOracle(sc)
    oracle.Restatement.set_seed(seed)
    ro = oracle.Restatement(sc)
    o, d = mg.rays_for(ref, 2048, seed)
    a, b = ref.first_hit(o, d), ro.first_hit(o, d)
    for f in ("prim", "t", "point", "normal", "depth"):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)
    ref.set_seed(seed * 7 + 1)
    ref.render(2)
    oracle.Restatement.set_seed(seed * 7 + 1)
    np.testing.assert_array_equal(ro.render_reference(2), ref.accum())


def test_restatement_counter_mode_is_deterministic(mg, oracle):
    ro = oracle.Restatement(mg.CASES["c0"]["make"]())
    a, _ = ro.render_counter(99, 2)
    b, _ = ro.render_counter(99, 2)
    np.testing.assert_array_equal(a, b)
    c, _ = ro.render_counter(100, 2)
    assert not np.array_equal(a, c)
