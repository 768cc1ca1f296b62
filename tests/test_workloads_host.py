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
