"""Baseline-dependent averaging (BDA) block maps, integer-exact.

Restates DDFacet's block-map builders (DDFacet/Data/ClassSmearMapping.py):

* ``blocks_mode1``  -- ``GiveBlocksRowsListBL_old`` (:496-625), the default (``[Comp] BDAMode=1``):
                       accumulate |delta uvw| along a baseline until it exceeds
                       Duv = C dPhi / (pi l nu_max), channel blocks from the smallest
                       (C/pi) dPhi / (|uvw| l) / dFreq of the time block, cut again wherever the
                       grid band changes.
* ``blocks_mode2``  -- ``GiveBlocksRowsListBL`` (:348-491).
* ``pack``          -- ``collectSmearMapping`` (:83-135): baselines in the order of their
                       "a0:a1" key strings, header [NB_lo, NB_hi], the block sizes, then the
                       blocks [ch0, ch1, rows...].
* ``plain_map``     -- the map mode 1 produces with dPhi = 0 (every row and channel its own
                       block), built directly with array operations.

Like the reference, the builders use C = 3e8 (ClassSmearMapping.py:356, :509) and a scalar
channel width.  ``smear_mapping`` drives all baselines.
"""
from __future__ import annotations

import itertools
import math

import numpy as np
import torch

C_BDA = 3e8


def _baseline_rows(A0, A1):
    """{(a0, a1): rows} for every ordered pair present, rows ascending."""
    A0 = np.asarray(A0)
    A1 = np.asarray(A1)
    key = A0.astype(np.int64) * (1 << 32) + A1.astype(np.int64)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    cuts = np.flatnonzero(np.diff(ks)) + 1
    out = {}
    for grp in np.split(order, cuts):
        if grp.size == 0:
            continue
        a0, a1 = int(A0[grp[0]]), int(A1[grp[0]])
        if a0 == a1:
            continue
        out[(a0, a1)] = grp
    return out


def blocks_mode1(rows, uvw, freqs, dfreq, dPhi, l, chan_map):
    """``GiveBlocksRowsListBL_old`` for one baseline: (flat list, block sizes)."""
    ind = rows
    nchan = freqs.size
    nu0 = np.max(freqs)
    u, v, w = uvw[ind, :].T
    nchan_block_max = 1e3
    du = u[1::] - u[0:-1]
    dv = v[1::] - v[0:-1]
    dw = w[1::] - w[0:-1]
    if du.size < 1:
        du = np.concatenate((du, [1e-30]))
        dv = np.concatenate((dv, [1e-30]))
        dw = np.concatenate((dw, [1e-30]))
    du = np.concatenate((du, [du[-1]]))
    dv = np.concatenate((dv, [dv[-1]]))
    dw = np.concatenate((dw, [dw[-1]]))
    Duv = C_BDA * dPhi / (np.pi * l * nu0)
    duvtot = 0
    current = []
    flat, sizes = [], []
    for irow in range(ind.size):
        current.append(int(ind[irow]))
        uv = np.sqrt(u[irow] ** 2 + v[irow] ** 2 + w[irow] ** 2)
        uv = max(uv, 1e-10)
        dnu = (C_BDA / np.pi) * dPhi / (uv * l)
        nchan_block = dnu / dfreq
        if nchan_block < nchan_block_max:
            nchan_block_max = nchan_block
        duvtot += np.sqrt(du[irow] ** 2 + dv[irow] ** 2 + dw[irow] ** 2)
        if (duvtot > Duv) | (irow == (ind.size - 1)):
            nchan_block_max = np.max([nchan_block_max, 1])
            ch = np.arange(0, nchan, nchan_block_max).tolist()
            if not (nchan in ch):
                ch.append(nchan)
            nchblocks = len(ch)
            chblock = np.int32(np.linspace(0, nchan, nchblocks))
            rampe = np.zeros((nchan,), np.int32)
            for ib in range(chblock.size - 1):
                rampe[chblock[ib]:chblock[ib + 1]] = ib
            prev = (-1, -1)
            cuts = []
            for ic in range(nchan):
                cur = (rampe[ic], chan_map[ic])
                if cur != prev:
                    cuts.append(ic)
                prev = cur
            if not (chblock[-1] in cuts):
                cuts.append(chblock[-1])
            cuts = np.array(cuts, np.int32)
            for ib in range(cuts.size - 1):
                desc = [int(cuts[ib]), int(cuts[ib + 1])] + current
                sizes.append(len(desc))
                flat += desc
            nchan_block_max = 1e3
            current = []
            duvtot = 0
    return flat, sizes


def blocks_mode2(rows, uvw_all, freqs, dfreq, dPhi, l_max, chan_map):
    """``GiveBlocksRowsListBL`` for one baseline: (flat list, block sizes)."""
    row_index = rows
    nrows = row_index.size
    uvw = uvw_all[row_index]
    nchan = freqs.size
    nu0 = np.max(freqs)
    Duv = C_BDA * dPhi / (2 * np.pi * nu0)
    duvw = np.zeros_like(uvw)
    duvw[:-1, :] = uvw[:-1, :] - uvw[1:, :]
    duvw[-1, :] = duvw[-2, :]
    n_max = abs(math.sqrt(1 - l_max ** 2) - 1)
    delta_phase = (2 * np.pi * nu0 / C_BDA) * (np.sqrt((duvw[:, :2] ** 2).sum(1)) * l_max + abs(duvw[:, 2]) * n_max)
    uv = np.sqrt((uvw[:, :2] ** 2).sum(1)) * l_max + abs(uvw[:, 2]) * n_max
    dnu = (C_BDA / (2 * np.pi)) * dPhi / uv
    frac = dnu / dfreq
    if Duv:
        rowblock = np.zeros(nrows + 1)
        rowblock[:nrows] = np.int32(delta_phase.cumsum() / dPhi)
        rowblock[nrows] = -1
        blockcut = np.where(np.roll(rowblock, 1) != rowblock)[0]
        nblocks = len(blockcut)
        slices = [slice(blockcut[i], blockcut[i + 1]) for i in range(nblocks - 1)]
    else:
        slices = [slice(i, i + 1) for i in range(nrows)]
    frac_min = np.array([max(frac[s].min(), 1) for s in slices])
    num_chan_blocks = np.ceil(nchan / frac_min)
    size_chan_block = np.int32(np.ceil(nchan / num_chan_blocks))
    uniq = np.array(list(set(size_chan_block)))
    num_bs = uniq.size
    cnum = dict([(sz, i) for i, sz in enumerate(uniq)])
    chanrange = np.arange(0, nchan, dtype=np.int32)
    chanpairs = np.zeros((num_bs, nchan + 1, 2), np.int32)
    chanpairs[:, :-1, 0] = chanrange[np.newaxis, :] / uniq[:, np.newaxis]
    chanpairs[:, :-1, 1] = np.asarray(chan_map)[np.newaxis, :]
    chanpairs[:, -1, :] = -1
    changes = (chanpairs != np.roll(chanpairs, 1, axis=1)).any(axis=2)
    where = [np.where(changes[bs, :])[0] for bs in range(num_bs)]
    cuts = [[(w[i], w[i + 1]) for i in range(len(w) - 1)] for w in where]
    blocklists = [[int(c0), int(c1)] + [int(r) for r in row_index[slices[ib]]]
                  for ib, sz in enumerate(size_chan_block) for c0, c1 in cuts[cnum[sz]]]
    sizes = [len(b) for b in blocklists]
    flat = list(itertools.chain(*blocklists))
    return flat, sizes


def _header(nb):
    """The two header words: NB's low 32 bits (as stored in an int32) and NB >> 32."""
    return np.array([nb & 0xFFFFFFFF, nb >> 32], np.uint32).view(np.int32)


def pack(per_baseline):
    """``collectSmearMapping`` (ClassSmearMapping.py:83-135): {"a0:a1": (flat, sizes)} -> int32 map."""
    keys = sorted(per_baseline.keys())
    nb = sum(len(per_baseline[k][1]) for k in keys)
    nrows = sum(int(np.sum(per_baseline[k][1])) for k in keys)
    m = np.zeros((2 + nb + nrows,), np.int32)
    m[0:2] = _header(nb)
    sizes_out = m[2:2 + nb]
    body = m[2 + nb:]
    i = j = 0
    for k in keys:
        flat, sizes = per_baseline[k]
        body[i:i + len(flat)] = flat
        i += len(flat)
        sizes_out[j:j + len(sizes)] = sizes
        j += len(sizes)
    return m


def smear_mapping(A0, A1, uvw, freqs, dfreq, dPhi, l, chan_map, mode=1):
    """All baselines' blocks packed into one map (``computeSmearMappingInBackground`` +
    ``collectSmearMapping``).  ``dPhi`` is sqrt(6 (1 - Decorr)) (ClassSmearMapping.py:66)."""
    freqs = np.asarray(freqs, np.float64)
    uvw = np.asarray(uvw, np.float64)
    chan_map = np.asarray(chan_map)
    per = {}
    for (a0, a1), rows in _baseline_rows(A0, A1).items():
        if mode == 1:
            per["%d:%d" % (a0, a1)] = blocks_mode1(rows, uvw, freqs, dfreq, dPhi, l, chan_map)
        elif mode == 2:
            per["%d:%d" % (a0, a1)] = blocks_mode2(rows, uvw, freqs, dfreq, dPhi, l, chan_map)
        else:
            raise ValueError("unknown BDAMode setting %d" % mode)
    return pack(per)


def plain_map(A0, A1, nchan, uvw=None):
    """Mode-1 map for dPhi = 0: every (row, channel) its own block, baselines in key-string
    order, rows ascending, channels ascending.  Identical to ``smear_mapping(..., dPhi=0)`` when
    consecutive rows of a baseline have distinct uvw (checked by the tests)."""
    A0 = np.asarray(A0)
    A1 = np.asarray(A1)
    groups = _baseline_rows(A0, A1)
    keys = sorted(groups.keys(), key=lambda k: "%d:%d" % k)
    rows = np.concatenate([groups[k] for k in keys]) if keys else np.zeros(0, np.int64)
    nb = rows.size * nchan
    m = np.empty(2 + nb + 3 * nb, np.int32)
    m[0:2] = _header(nb)
    m[2:2 + nb] = 3
    body = m[2 + nb:].reshape(nb, 3)
    ch = np.tile(np.arange(nchan, dtype=np.int32), rows.size)
    body[:, 0] = ch
    body[:, 1] = ch + 1
    body[:, 2] = np.repeat(rows.astype(np.int32), nchan)
    return m


def smear_mapping_gpu(A0, A1, uvw, freqs, dfreq, dPhi, l, chan_map, device=None, mode=1):
    """The block map of every baseline, packed as ``collectSmearMapping`` does, built on the GPU:
    mode 1 (``GiveBlocksRowsListBL_old``, ddfg_bda_mode1_count / _write) or mode 2
    (``GiveBlocksRowsListBL``, ddfg_bda_mode2_count / _write, ``l`` being l_max): the same words as
    ``smear_mapping(..., mode=mode)``.  Returns an int32 device tensor."""
    from . import _abi, device as D

    dev = D._dev(device)
    A0 = np.asarray(A0)
    A1 = np.asarray(A1)
    freqs = np.asarray(freqs, np.float64)
    nchan = freqs.size
    # baselines in the order of their "a0:a1" key strings (autocorrelations excluded)
    na = int(max(A0.max(), A1.max())) + 1 if A0.size else 1
    pairs = np.unique(A0.astype(np.int64) * na + A1.astype(np.int64))
    pairs = pairs[(pairs // na) != (pairs % na)]
    order = sorted(range(pairs.size), key=lambda i: "%d:%d" % (pairs[i] // na, pairs[i] % na))
    rank = np.full(na * na, -1, np.int64)
    rank[pairs[order]] = np.arange(pairs.size)
    a0 = torch.from_numpy(A0.astype(np.int64)).to(dev)
    a1 = torch.from_numpy(A1.astype(np.int64)).to(dev)
    key = torch.from_numpy(rank).to(dev)[a0 * na + a1]
    srt, perm = torch.sort(key, stable=True)
    keep = srt >= 0
    rows = perm[keep].to(torch.int32).contiguous()
    nbl = int(pairs.size)
    counts = torch.bincount(srt[keep], minlength=nbl)
    bl_off = torch.zeros(nbl + 1, dtype=torch.int64, device=dev)
    bl_off[1:] = torch.cumsum(counts, 0)
    uvw_d = D.to_device(uvw, torch.float64, dev)
    cmap = D.to_device(np.asarray(chan_map, np.int32), torch.int32, dev)
    nblk = torch.zeros(max(nbl, 1), dtype=torch.int64, device=dev)
    nwords = torch.zeros(max(nbl, 1), dtype=torch.int64, device=dev)
    lib = _abi.lib()
    st = D._stream_ptr()
    nu0 = float(np.max(freqs))
    args = (uvw_d.data_ptr(), rows.data_ptr(), bl_off.data_ptr(), nbl, nchan, cmap.data_ptr(), float(dfreq),
            float(dPhi), float(l), nu0)
    count, write = ((lib.ddfg_bda_mode1_count, lib.ddfg_bda_mode1_write) if mode == 1 else
                    (lib.ddfg_bda_mode2_count, lib.ddfg_bda_mode2_write))
    _abi.check(count(*args, nblk.data_ptr(), nwords.data_ptr(), st))
    if mode != 1 and bool((nblk[:nbl] < 0).any()):
        raise IndexError("BDA mode 2: a baseline has a single row (GiveBlocksRowsListBL reads the row "
                         "difference before the last)")
    blk_off = torch.cumsum(nblk, 0) - nblk
    word_off = torch.cumsum(nwords, 0) - nwords
    nb = int(nblk[:nbl].sum().item())
    nw = int(nwords[:nbl].sum().item())
    m = torch.empty(2 + nb + nw, dtype=torch.int32, device=dev)
    m[0:2] = torch.from_numpy(_header(nb)).to(dev)
    _abi.check(write(*args, blk_off.data_ptr(), word_off.data_ptr(), m[2:].data_ptr(), m[2 + nb:].data_ptr(), st))
    return m


def _spread_bits16(x: torch.Tensor) -> torch.Tensor:
    """Bits 0..15 of x moved to the even bit positions 0..30."""
    x = (x | (x << 8)) & 0x00FF00FF
    x = (x | (x << 4)) & 0x0F0F0F0F
    x = (x | (x << 2)) & 0x33333333
    return (x | (x << 1)) & 0x55555555


def uv_locality_order(bda_map: torch.Tensor, block_start: torch.Tensor, uvw: torch.Tensor, freqs: torch.Tensor,
                      tile_wavelengths: float, w_planes=None) -> torch.Tensor:
    """A permutation of a packed map's blocks (int64 [nblocks]) that visits them in Z order of
    uv tiles: each block's first row and first channel give (u, v) in wavelengths, cut into
    tiles of ``tile_wavelengths``.  The same order suits every facet, whose grid positions are
    the uv coordinates scaled by the facet's size (plus a small w shift).  With ``w_planes`` =
    (Nw, wmax), blocks of a tile are further ordered by their W plane, lrint((Nw-1) |w| nu /
    (nu_max wmax)) (gridder.h:324 with RefWave = c / nu_max), which every facet shares: runs of
    equal support."""
    nb = block_start.numel()
    if nb == 0:
        return torch.zeros(0, dtype=torch.int64, device=bda_map.device)
    ch0 = bda_map[block_start].to(torch.int64)
    row = bda_map[block_start + 2].to(torch.int64)
    lam = freqs.to(torch.float64)[ch0] / 299792458.0
    u = uvw[row, 0] * lam
    v = uvw[row, 1] * lam
    t = float(tile_wavelengths)
    iu = torch.floor(u / t).to(torch.int64)
    iv = torch.floor(v / t).to(torch.int64)
    iu = (iu - iu.min()).clamp_(0, 0xFFFF)
    iv = (iv - iv.min()).clamp_(0, 0xFFFF)
    key = _spread_bits16(iu) | (_spread_bits16(iv) << 1)
    if w_planes is not None:
        nw, wmax = int(w_planes[0]), float(w_planes[1])
        fr = freqs.to(torch.float64)
        iw = torch.round((nw - 1) * uvw[row, 2].abs() * fr[ch0] / (fr.max() * wmax)).to(torch.int64)
        key = (key << 8) | iw.clamp_(0, 255)
    return torch.sort(key, stable=True)[1]


def reorder_blocks(bda_map: torch.Tensor, block_start: torch.Tensor, order: torch.Tensor) -> torch.Tensor:
    """The packed map (int32, on the map's device) with its blocks in ``order`` (a permutation of
    block indices): the same blocks, so the degridder's result is unchanged and the gridder's
    differs only by the order of its floating-point sums."""
    nb = block_start.numel()
    if nb == 0:
        return bda_map.clone()
    sizes = bda_map[2:2 + nb].to(torch.int64)
    s = sizes[order]
    starts = block_start[order]
    new_off = torch.cumsum(s, 0) - s
    total = int(s.sum().item())
    base = 2 + nb
    idx = torch.repeat_interleave(starts - new_off, s) + torch.arange(total, device=bda_map.device)
    out = torch.empty(base + total, dtype=torch.int32, device=bda_map.device)
    out[:2] = bda_map[:2]
    out[2:base] = s.to(torch.int32)
    out[base:] = bda_map[idx]
    return out
