"""The Jones time map on the device (ddfg_jones_time_map) against the reference's
ClassJones.GiveTimeMapping (tests/golden/maps_golden.npz) and the host restatement at scale."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "maps_golden.npz"))


def test_jones_time_map_gpu_matches_reference():
    import torch

    from ddfacet_b200 import maps

    t = torch.from_numpy(G["times"]).cuda()
    got = maps.jones_time_map_gpu(t, G["t0"], G["t1"]).cpu().numpy()
    np.testing.assert_array_equal(got, G["time_map"])


def test_jones_time_map_gpu_large():
    import torch

    from ddfacet_b200 import maps

    rng = np.random.default_rng(5)
    times = rng.uniform(0, 8 * 3600.0, 3_000_000)
    t0 = np.arange(0, 8 * 3600.0, 300.0)
    t1 = t0 + 300.0
    got = maps.jones_time_map_gpu(torch.from_numpy(times).cuda(), t0, t1).cpu().numpy()
    np.testing.assert_array_equal(got, maps.jones_time_map(times, t0, t1))
