"""Synthetic workloads are seeded, shaped and classed as specified."""
import numpy as np

from floodca_b200 import synth


def test_terrain_is_deterministic():
    a = synth.make_terrain(synth.TerrainSpec(64, 80, seed=5))
    b = synth.make_terrain(synth.TerrainSpec(64, 80, seed=5))
    assert np.array_equal(a.z, b.z) and np.array_equal(a.n, b.n)


def test_terrain_slopes_south_and_has_channel():
    d = synth.make_terrain(synth.TerrainSpec(128, 128, amplitude=0.0, seed=1))
    assert d.z[0].mean() > d.z[-1].mean()
    assert np.isclose(d.z[0, 0] - d.z[-1, 0], 0.005 * 90.0 * 127, rtol=1e-5)
    c = 128 // 2 - 1
    assert np.allclose(d.z[:, 0] - d.z[:, c], 2.0, atol=1e-4)


def test_fbm_amplitude_and_classes():
    d = synth.make_terrain(synth.TerrainSpec(96, 96, amplitude=20.0, seed=2, slope=0.0,
                                             channel_depth=0.0))
    relief = d.z - 10.0
    assert np.isclose(np.abs(relief).max(), 20.0, rtol=1e-5)
    assert set(np.unique(d.n).tolist()) <= {float(np.float32(v)) for v in synth.MANNING_CLASSES}
    assert len(np.unique(d.n)) >= 4


def test_configs_shapes_and_forcing():
    d, p = synth.config1(n=32)
    assert d.shape == (32, 32) and p.T_sim == 7200.0 and p.rain_end == 3600.0
    assert np.allclose(d.Rday, 50 * 24 / 1000.0) and p.edges == (0, 1, 0, 0)
    d2, p2 = synth.config2(n=64)
    assert p2.inflow_cell == 32 and p2.inflow_peak == 500.0 and p2.rain_end == 7200.0
