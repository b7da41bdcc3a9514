"""Host logic of the bench's closest-hit roofline (no GPU): the launch-shape key of ncu's
per-query instruction counts, and their lookup with the nearest-shape fallback named in the
result."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _launch(spec, bps=8, block=128, wave=1 << 25):
    return {"speculate": spec, "blocks_per_sm": bps, "block_extend": block, "wave_paths": wave}


def test_shape_key():
    assert bench.extend_shape_key(4, 2, _launch(2)) == "w4_l2_s0_b8x128_q25"
    assert bench.extend_shape_key(8, 3, _launch(1, 16, 256, 1 << 24)) == "w8_l3_s1_b16x256_q24"
    assert bench.extend_shape_key(4, 8, _launch(3)).startswith("w4_l8_s1_")
    assert bench.extend_shape_key(2, 1, _launch(4)).startswith("w2_l1_s0_")  # shadow-only speculation
    assert bench.extend_shape_key(4, 2, _launch(2), 2) == "w4_l2_s0_b8x128_q25_ploc"
    assert bench.extend_shape_key(4, 2, _launch(2), 1) == "w4_l2_s0_b8x128_q25_lbvh"


def test_instruction_counts_by_shape(tmp_path, monkeypatch):
    prof = tmp_path / "profiles"
    prof.mkdir()
    (prof / "k_extend_issue.txt").write_text(
        "# comment line\n"
        "scene-a@w4_l2_s1_b8x128_q25 warp_inst_per_query: 100.0\n"
        "scene-a@w4_l2_s1_b16x128_q24 warp_inst_per_query: 90.0\n"
        "scene-a@w4_l8_s1_b8x128_q25 warp_inst_per_query: 80.0\n"
        "scene-a@w8_l2_s1_b8x128_q25 warp_inst_per_query: 70.0\n"
        "scene-a@w4_l2_s0_b8x128_q25 warp_inst_per_query: 120.0\n"
        "scene-a@w4_l2_s1_b8x128_q25 fp32_flop_per_query: 300.0\n"
        "scene-a@w4_l2_s1_b8x128_q25_ploc warp_inst_per_query: 60.0\n"
        "scene-b@w4_l2_s0_b8x128_q25 warp_inst_per_query: 50.0\n")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    f = bench._ncu_shape_per_query
    k = "warp_inst_per_query"
    assert f("scene-a", "w4_l2_s1_b8x128_q25", k) == (100.0, "w4_l2_s1_b8x128_q25")  # exact
    assert f("scene-a", "w4_l2_s1_b16x128_q24", k) == (90.0, "w4_l2_s1_b16x128_q24")
    # width, then speculation, then the closest leaf, then the grid, then the wave
    assert f("scene-a", "w4_l2_s1_b16x128_q25", k) == (90.0, "w4_l2_s1_b16x128_q24")
    assert f("scene-a", "w4_l2_s1_b8x256_q24", k) == (90.0, "w4_l2_s1_b16x128_q24")
    assert f("scene-a", "w4_l2_s1_b8x128_q24", k) == (100.0, "w4_l2_s1_b8x128_q25")
    assert f("scene-a", "w4_l3_s1_b8x128_q25", k) == (100.0, "w4_l2_s1_b8x128_q25")
    assert f("scene-a", "w4_l6_s1_b8x128_q25", k) == (80.0, "w4_l8_s1_b8x128_q25")
    assert f("scene-a", "w8_l4_s1_b8x128_q25", k) == (70.0, "w8_l2_s1_b8x128_q25")
    assert f("scene-a", "w4_l4_s0_b8x128_q25", k) == (120.0, "w4_l2_s0_b8x128_q25")
    assert f("scene-a", "w4_l8_s1_b8x128_q25", "fp32_flop_per_query") == (300.0, "w4_l2_s1_b8x128_q25")
    # a tree built by another builder is matched first by its builder
    assert f("scene-a", "w4_l2_s1_b8x128_q25_ploc", k) == (60.0, "w4_l2_s1_b8x128_q25_ploc")
    assert f("scene-a", "w8_l4_s0_b16x256_q24_ploc", k) == (60.0, "w4_l2_s1_b8x128_q25_ploc")
    assert f("scene-a", "w4_l2_s1_b8x128_q25_lbvh", k) == (100.0, "w4_l2_s1_b8x128_q25")
    # a workload or field without a capture gives nothing
    assert f("scene-c", "w4_l2_s0_b8x128_q25", k) == (None, None)
    assert f("scene-b", "w4_l2_s0_b8x128_q25", "fp32_flop_per_query") == (None, None)
    assert f("scene-a", None, k) == (None, None)


def test_committed_counts_cover_every_headline_workload():
    """each single-scene configuration has at least one capture, so every bench line carries
    an issue figure"""
    for cfg in (0, 1, 2, 3):
        wl = bench.WORKLOADS[cfg]["name"]
        v, shape = bench._ncu_shape_per_query(wl, "w4_l2_s0_b8x128_q25", "warp_inst_per_query")
        assert v is not None and v > 0, wl
