"""Host checks of the synthetic workload generators and the bench's byte
model (no GPU): seeded, with the shapes, fractions and statistics the
workload definitions state."""
import numpy as np

import bench
from janus_b200 import microstructures as micro


def test_random_spheres_are_disjoint_and_reach_the_fraction():
    phase, centres = micro.random_spheres(48, radius=4, volume_fraction=0.3, seed=5)
    assert phase.shape == (48, 48, 48) and phase.dtype == np.uint8
    assert 0.3 <= phase.mean() < 0.33
    d = centres[:, None, :] - centres[None, :, :]
    d -= 48 * np.round(d / 48)
    dist2 = (d * d).sum(-1) + np.eye(len(centres)) * 1e9
    assert dist2.min() >= (2 * 4) ** 2
    again, _ = micro.random_spheres(48, radius=4, volume_fraction=0.3, seed=5)
    assert np.array_equal(phase, again)


def test_voronoi_partition_is_two_phase_and_seeded():
    a = micro.voronoi(24, cells=40, seed=3)
    b = micro.voronoi(24, cells=40, seed=3)
    assert a.shape == (24, 24, 24) and np.array_equal(a, b)
    assert set(np.unique(a)) == {0, 1}
    assert 0.1 < a.mean() < 0.9


def test_gaussian_field_statistics():
    g = micro.gaussian_field(64, dim=3, corr_len=8.0, std=1.5, seed=2)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.5) < 1e-12
    # squared-exponential correlation: neighbours nearly equal, far voxels not
    c1 = np.mean(g * np.roll(g, 1, axis=0)) / g.var()
    c16 = np.mean(g * np.roll(g, 16, axis=0)) / g.var()
    assert c1 > 0.9 and abs(c16) < 0.4


def test_ellipses_and_square_inclusion():
    e = micro.ellipses(64, 5, seed=1)
    assert e.shape == (64, 64) and e.max() <= 5 and (e > 0).any()
    sq = micro.square_inclusion(64, side=32)
    assert sq.sum() == 32 * 32


def test_bench_byte_model_is_the_algorithmic_one():
    # 11 s p + m per 3D voxel-iteration (FP64: 529 B, FP32: 265 B)
    assert sum(bench.pass_bytes(6, 8).values()) == 529
    assert sum(bench.pass_bytes(6, 4).values()) == 265


def test_clock_summary_from_nvidia_smi_lines():
    lines = ["1965, 1965, 812.3, 0x0000000000000000, Not Active, Not Active, Not Active, "
             "Not Active",
             "1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
             "1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
             "[N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
             "garbage"]
    s = bench.ClockSampler.summarise(lines)
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                 "samples": 3}
    assert bench.ClockSampler.summarise([]) is None


def test_measured_peak_reads_the_file_or_falls_back(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.measured_peak() == (bench.FALLBACK_HBM_GBS, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6558.4, "bf16_tflops": 1590}')
    assert bench.measured_peak() == (6558.4, "measured")


def test_reference_arm_line_on_a_small_cell():
    """The reference arm (the reference's own CPU path, one process per load
    case) prints the contract's JSON line; run here on a 16^3 cell."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.abspath(bench.__file__))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", "--n", "16"],
                         capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["unit"] == "voxel-iter/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
