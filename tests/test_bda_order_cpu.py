"""Block reordering of packed BDA maps (bda.uv_locality_order, bda.reorder_blocks) on the host:
the rewritten map holds exactly the original blocks, in the requested order, with their sizes."""
import numpy as np
import torch

import cases
from ddfacet_b200 import bda


def _blocks(m):
    nb = int(np.uint32(m[0]))
    sizes = m[2:2 + nb]
    out, p = [], 2 + nb
    for s in sizes:
        out.append(tuple(int(x) for x in m[p:p + s]))
        p += s
    return out


def _starts(m):
    nb = int(np.uint32(m[0]))
    sizes = m[2:2 + nb].astype(np.int64)
    return torch.from_numpy(2 + nb + np.concatenate([[0], np.cumsum(sizes)[:-1]]))


def test_reorder_blocks_is_the_permutation():
    c = cases.make_case(seed=3, bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=8, ncorr=4)
    m = torch.from_numpy(c.bda)
    starts = _starts(c.bda)
    nb = starts.numel()
    rng = np.random.default_rng(0)
    order = torch.from_numpy(rng.permutation(nb))
    new = bda.reorder_blocks(m, starts, order).numpy()
    a, b = _blocks(c.bda), _blocks(new)
    assert new.size == c.bda.size and new[0] == c.bda[0] and new[1] == c.bda[1]
    assert b == [a[i] for i in order.tolist()]


def test_uv_locality_order():
    c = cases.make_case(seed=4, bda_mode=1, dphi=np.sqrt(6 * 0.05), nchan=8, ncorr=4)
    m = torch.from_numpy(c.bda)
    starts = _starts(c.bda)
    nb = starts.numel()
    uvw = torch.from_numpy(c.uvw)
    fr = torch.from_numpy(c.freqs)
    tile = 150.0
    order = bda.uv_locality_order(m, starts, uvw, fr, tile)
    assert sorted(order.tolist()) == list(range(nb))
    # tiles are visited in Z order: the interleaved tile key never decreases along the order
    blocks = _blocks(c.bda)
    lam = np.array([c.freqs[b[0]] / 299792458.0 for b in blocks])
    rows = np.array([b[2] for b in blocks])
    iu = np.floor(c.uvw[rows, 0] * lam / tile).astype(np.int64)
    iv = np.floor(c.uvw[rows, 1] * lam / tile).astype(np.int64)
    iu -= iu.min()
    iv -= iv.min()

    def z(x, y):
        k = 0
        for bit in range(16):
            k |= ((int(x) >> bit) & 1) << (2 * bit) | ((int(y) >> bit) & 1) << (2 * bit + 1)
        return k

    keys = np.array([z(x, y) for x, y in zip(iu, iv)])[order.numpy()]
    assert np.all(np.diff(keys) >= 0)
    # within a tile the map order is kept (stable)
    o = order.numpy()
    same = np.diff(keys) == 0
    assert np.all(o[1:][same] > o[:-1][same])
    # with W planes as the second key, planes never decrease inside a tile
    ow = bda.uv_locality_order(m, starts, uvw, fr, tile, w_planes=(4, float(np.abs(c.uvw[:, 2]).max()) * 1.01))
    assert sorted(ow.tolist()) == list(range(nb))


def test_large_block_list_rule():
    """VisData.with_large_blocks lists exactly the blocks of more than min_vis visibilities (the
    rule the kernels use to leave them out of the one-lane walks); block reordering rebuilds it."""
    from ddfacet_b200 import device as D

    c = cases.make_case(seed=5, bda_mode=1, dphi=np.sqrt(6 * 1.0), nchan=16, ntimes=60, ncorr=4)
    m = torch.from_numpy(c.bda)
    starts = _starts(c.bda)
    nb = starts.numel()
    blocks = _blocks(c.bda)
    nv = np.array([(len(b) - 2) * (b[1] - b[0]) for b in blocks])
    vs = D.VisData(vis=torch.zeros((c.nrow, c.nchan, 4), dtype=torch.complex64), uvw=torch.from_numpy(c.uvw),
                   flags=torch.zeros((c.nrow, c.nchan, 4), dtype=torch.uint8),
                   weights=torch.ones((c.nrow, c.nchan)), freqs=torch.from_numpy(c.freqs), freqs_host=c.freqs,
                   recip_wvl=torch.from_numpy(c.freqs / 299792458.0), chan_map=torch.zeros(c.nchan, dtype=torch.int32),
                   bda_map=m, block_start=starts, nblocks=nb, chan_equidistant=1)
    big = vs.with_large_blocks(128)
    np.testing.assert_array_equal(big.large_blocks.numpy(), np.flatnonzero(nv > 128))
    assert big.large_min_vis == 128 and big.struct().nlarge == int((nv > 128).sum())
    assert vs.with_large_blocks(10 ** 6).large_blocks is None
