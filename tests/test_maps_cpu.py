"""The integer maps that feed the kernels (ddfacet_b200.maps) against the reference's own functions
run on the same inputs (tests/golden/maps_golden.npz, made by tests/golden/make_golden.py):
ClassJones.GiveTimeMapping and GiveVisToJonesChanMapping, and the grid / degrid channel maps that
ClassVisServer.Init builds for two measurement sets under four frequency settings -- word for word."""
import os

import numpy as np

from ddfacet_b200 import maps

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "maps_golden.npz"))


def test_jones_time_map_matches_reference():
    got = maps.jones_time_map(G["times"], G["t0"], G["t1"])
    assert got.dtype == np.int32
    np.testing.assert_array_equal(got, G["time_map"])
    # the fixture covers rows outside every slot, a gap and overlapping slots
    assert (G["times"] < G["t0"].min()).any() and (G["times"] >= G["t1"].max()).any()


def test_jones_chan_map_matches_reference():
    np.testing.assert_array_equal(maps.jones_chan_map(G["jchan_freqs"], G["jchan_domains"]), G["jchan_map"])


def test_channel_maps_match_reference():
    ms = [maps.MSChannels(G["ms_a_freq"], G["ms_a_width"]), maps.MSChannels(G["ms_b_freq"], G["ms_b_width"])]
    for k in range(int(G["nsettings"])):
        band_mhz, nband, dband_mhz, ndband = G[f"s{k}_settings"]
        cm = maps.ChannelMaps.build(ms, band_mhz=band_mhz, nband=int(nband), degrid_band_mhz=dband_mhz,
                                    ndegrid_band=int(ndband))
        assert cm.nbands == int(G[f"s{k}_nbands"])
        np.testing.assert_array_equal(cm.band_centers, G[f"s{k}_centers"])
        for ims in (0, 1):
            np.testing.assert_array_equal(cm.chan_mapping[ims], G[f"s{k}_ms{ims}_map"])
            np.testing.assert_array_equal(cm.chan_mapping_chan[ims], G[f"s{k}_ms{ims}_mapchan"])
            np.testing.assert_array_equal(cm.chan_mapping_degrid[ims], G[f"s{k}_ms{ims}_degrid"])
            np.testing.assert_array_equal(cm.degrid_freqs[ims], G[f"s{k}_ms{ims}_degrid_freqs"])
