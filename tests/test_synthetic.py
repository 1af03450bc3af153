"""The seeded synthetic inputs the benchmark and the tests use: sizes of the configured
trajectories, coordinates within [-pi, pi] (radial spokes end on the boundary, which the
NUFFT treats periodically), determinism, and the normalisations of the coil maps and the
density compensation."""
import math

import numpy as np
import pytest

from hastycucompute_b200 import synthetic


PI32 = float(np.float32(math.pi))  # float32 rounds pi up


def _in_range(k):
    return float(k.min()) >= -PI32 and float(k.max()) <= PI32


@pytest.mark.parametrize("gen,args,shape", [
    (synthetic.golden_means_radial, (1024, 128), (3, 131072)),            # 64^3 radial, 8 coils
    (synthetic.golden_means_radial, (16384, 128), (3, 2097152)),          # 128^3 radial volumes
    (synthetic.variable_density_spiral_2d, (32, 2048), (2, 65536)),       # 2-D spirals
    (synthetic.golden_angle_radial_2d, (64, 256), (2, 16384)),
])
def test_trajectory_sizes_and_range(gen, args, shape):
    k = gen(*args)
    assert k.shape == shape and k.dtype == np.float32
    assert _in_range(k)


def test_cones_spiral_full_size_is_deterministic_and_in_range():
    """160^3 cones workload: 24000 interleaves x 256 samples = 6,144,000 points."""
    k = synthetic.cones_spiral(24000, 256)
    assert k.shape == (3, 6144000) and k.dtype == np.float32 and k.flags.c_contiguous
    assert _in_range(k)
    small = synthetic.cones_spiral(100, 64)
    assert np.array_equal(small, synthetic.cones_spiral(100, 64))
    # samples start at the centre of k-space and reach the edge
    r = np.sqrt((k.astype(np.float64) ** 2).sum(0)).reshape(24000, 256)
    assert r[:, 0].max() == 0.0 and r[:, -1].min() > 0.95 * math.pi


def test_radial_spokes_differ_by_offset():
    """Frames draw consecutive golden-means spokes (offset), so their trajectories differ."""
    a = synthetic.golden_means_radial(300, 128, offset=0)
    b = synthetic.golden_means_radial(300, 128, offset=300)
    assert not np.allclose(a, b)
    assert np.array_equal(a, synthetic.golden_means_radial(300, 128, offset=0))


@pytest.mark.parametrize("C,shape", [(8, (16, 16, 16)), (12, (32, 32)), (32, (8, 10, 12))])
def test_coil_maps_are_rss_normalised(C, shape):
    s = synthetic.coil_maps(C, shape)
    assert s.shape == (C, *shape) and s.dtype == np.complex64
    rss = np.sqrt((np.abs(s.astype(np.complex128)) ** 2).sum(0))
    assert np.allclose(rss, 1.0, atol=1e-5)
    assert np.array_equal(s, synthetic.coil_maps(C, shape))


def test_dcf_has_mean_one():
    k = synthetic.golden_means_radial(256, 64)
    w = synthetic.dcf_k2(k)
    assert w.shape == (k.shape[1],) and abs(float(w.astype(np.float64).mean()) - 1.0) < 1e-6
    assert float(w.min()) >= 0.0
