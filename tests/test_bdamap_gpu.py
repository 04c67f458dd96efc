"""Mode-1 BDA maps built on the GPU (ddfg_bda_mode1_*, bda.smear_mapping_gpu) are word-for-word
the reference's maps (tests/golden/bda_golden.npz, made by ClassSmearMapping itself) and the host
builder's on larger and edge cases (one-row baselines, two bands, coarse and fine decorrelation)."""
import os

import numpy as np
import pytest

from ddfacet_b200 import bda, synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("which", ["a", "b"])
def test_against_reference_maps(which):
    g = dict(np.load(os.path.join(HERE, "golden", "bda_golden.npz")))
    m = bda.smear_mapping_gpu(g["A0"], g["A1"], g["uvw"], g["freqs"], float(g["dfreq"]), float(g[f"dphi_{which}"]),
                              float(g["l"]), g["chan_map"])
    np.testing.assert_array_equal(m.cpu().numpy(), g[f"map_mode1_{which}"])


@pytest.mark.parametrize("nchan,decorr,bands", [(64, 0.02, 1), (64, 0.002, 2), (16, 0.2, 1), (7, 0.05, 3)])
def test_against_host_builder(nchan, decorr, bands):
    obs = synth.make_observation(5, 16, 3000.0, 34.0, 40.0, 1.0, 8.0, nchan, 0.9e9, 1.67e9)
    chan_map = (np.arange(nchan) * bands // nchan).astype(np.int32)
    dfreq = float(obs.freqs[1] - obs.freqs[0])
    dphi = np.sqrt(6 * decorr)
    l = 0.02
    want = bda.smear_mapping(obs.A0, obs.A1, obs.uvw, obs.freqs, dfreq, dphi, l, chan_map, mode=1)
    got = bda.smear_mapping_gpu(obs.A0, obs.A1, obs.uvw, obs.freqs, dfreq, dphi, l, chan_map).cpu().numpy()
    np.testing.assert_array_equal(got, want)


def test_one_row_baselines_and_autocorrelations():
    obs = synth.make_observation(9, 6, 1000.0, 34.0, 40.0, 30.0 / 3600, 30.0, 8, 1.3e9, 1.4e9)  # one dump
    A0 = np.concatenate([obs.A0, [0, 1]]).astype(np.int32)          # plus two autocorrelation rows
    A1 = np.concatenate([obs.A1, [0, 1]]).astype(np.int32)
    uvw = np.concatenate([obs.uvw, np.zeros((2, 3))])
    chan_map = np.zeros(8, np.int32)
    args = (A0, A1, uvw, obs.freqs, float(obs.freqs[1] - obs.freqs[0]), np.sqrt(6 * 0.02), 0.01, chan_map)
    np.testing.assert_array_equal(bda.smear_mapping_gpu(*args).cpu().numpy(), bda.smear_mapping(*args, mode=1))


@pytest.mark.parametrize("which", ["a", "b"])
def test_mode2_against_reference_maps(which):
    """Mode 2 (GiveBlocksRowsListBL) built on the GPU equals the reference's own map word for word."""
    g = dict(np.load(os.path.join(HERE, "golden", "bda_golden.npz")))
    m = bda.smear_mapping_gpu(g["A0"], g["A1"], g["uvw"], g["freqs"], float(g["dfreq"]), float(g[f"dphi_{which}"]),
                              float(g["l"]), g["chan_map"], mode=2)
    np.testing.assert_array_equal(m.cpu().numpy(), g[f"map_mode2_{which}"])


@pytest.mark.parametrize("nchan,decorr,bands", [(64, 0.02, 1), (64, 0.002, 2), (16, 0.2, 1), (7, 0.05, 3),
                                                (32, 0.0, 1)])
def test_mode2_against_host_builder(nchan, decorr, bands):
    obs = synth.make_observation(5, 16, 3000.0, 34.0, 40.0, 1.0, 8.0, nchan, 0.9e9, 1.67e9)
    chan_map = (np.arange(nchan) * bands // nchan).astype(np.int32)
    dfreq = float(obs.freqs[1] - obs.freqs[0])
    dphi = np.sqrt(6 * decorr)
    want = bda.smear_mapping(obs.A0, obs.A1, obs.uvw, obs.freqs, dfreq, dphi, 0.02, chan_map, mode=2)
    got = bda.smear_mapping_gpu(obs.A0, obs.A1, obs.uvw, obs.freqs, dfreq, dphi, 0.02, chan_map, mode=2)
    np.testing.assert_array_equal(got.cpu().numpy(), want)


def test_mode2_single_row_baseline_is_refused():
    obs = synth.make_observation(9, 6, 1000.0, 34.0, 40.0, 30.0 / 3600, 30.0, 8, 1.3e9, 1.4e9)  # one dump
    with pytest.raises(IndexError):
        bda.smear_mapping_gpu(obs.A0, obs.A1, obs.uvw, obs.freqs, float(obs.freqs[1] - obs.freqs[0]),
                              np.sqrt(6 * 0.02), 0.01, np.zeros(8, np.int32), mode=2)
    with pytest.raises(IndexError):
        bda.smear_mapping(obs.A0, obs.A1, obs.uvw, obs.freqs, float(obs.freqs[1] - obs.freqs[0]),
                          np.sqrt(6 * 0.02), 0.01, np.zeros(8, np.int32), mode=2)
