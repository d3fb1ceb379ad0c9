"""Host logic of the int8-sliced FP64 product (no device): the tile lists that
ptbgpu_oz_tiles returns for each kernel variant cover every output block that
the product must write exactly once, with K ranges (whole 128-column blocks)
that contain every nonzero slice pair of a triangular operand, and the default
variant is resolved from the slice count and the K block as documented."""
import itertools

import pytest

from ptb_b200 import PtbGpuError
from ptb_b200.api import oz_tiles

BM = 128


def required_blocks(n, bn, symmetric):
    ldp = -(-n // BM) * BM
    nbi, nbj = ldp // BM, -(-ldp // bn)
    return ldp, {(bi, bj) for bi in range(nbi) for bj in range(nbj)
                 if not symmetric or bj * bn + bn - 1 >= bi * BM}


def nonzero_k(bi, bj, bn, ldp, a_tri, b_tri):
    """K range [lo, hi) outside which the block's slice products vanish."""
    lo, hi = 0, ldp
    if a_tri == 1:   # A(i, k) = 0 for k > i
        hi = min(hi, (bi + 1) * BM)
    if a_tri == 2:   # A(i, k) = 0 for k < i
        lo = max(lo, bi * BM)
    if b_tri == 1:
        hi = min(hi, min(ldp, bj * bn + bn))
    if b_tri == 2:
        lo = max(lo, bj * bn)
    return lo, hi


def check(n, slices, kblock, variant, a_tri, b_tri, symmetric):
    tiles, info = oz_tiles(n, slices, kblock, variant, a_tri, b_tri, symmetric)
    bn, pair = info["tile_n"], info["rows"] == 2 * BM
    ldp, need = required_blocks(n, bn, symmetric)
    nbi = ldp // BM
    assert info["ctas"] == len(tiles) * (2 if pair else 1)
    lengths = [int(t[3] - t[2]) for t in tiles]
    assert lengths == sorted(lengths, reverse=True), "longest K ranges first"
    seen = {}
    for x, bj, k0, k1 in tiles.tolist():
        assert 0 <= k0 < k1 <= ldp and k0 % BM == 0 and k1 % BM == 0
        halves = [2 * x, 2 * x + 1] if pair else [x]
        kept = [bi for bi in halves if bi < nbi and (bi, bj) in need]
        assert kept, "a tile entry with nothing to write"
        for bi in kept:
            assert (bi, bj) not in seen, "output block listed twice"
            seen[(bi, bj)] = (k0, k1)
            lo, hi = nonzero_k(bi, bj, bn, ldp, a_tri, b_tri)
            if lo < hi:
                assert k0 <= lo and k1 >= hi, (bi, bj, k0, k1, lo, hi)
    assert set(seen) == need
    return info


@pytest.mark.parametrize("n", [100, 128, 300, 700, 1000, 2944])
@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5])
def test_tiles_cover_every_block_once(n, variant):
    kblock = 32 if variant in (4, 5) else 64
    bn = oz_tiles(n, 8, kblock, variant)[1]["tile_n"]
    for a_tri, b_tri, symmetric in itertools.product((0, 1, 2), (0, 1, 2), (False, True)):
        ldp, need = required_blocks(n, bn, symmetric)
        if any(lo >= hi for lo, hi in (nonzero_k(bi, bj, bn, ldp, a_tri, b_tri) for bi, bj in need)):
            # a block whose product vanishes identically (A lower and B^T upper, or the
            # reverse, below the diagonal) is refused, not listed with an empty K range
            with pytest.raises(PtbGpuError):
                oz_tiles(n, 8, kblock, variant, a_tri, b_tri, symmetric)
            continue
        info = check(n, 8, kblock, variant, a_tri, b_tri, symmetric)
        assert info["variant"] == variant


@pytest.mark.parametrize("slices", [4, 6, 7, 8])
@pytest.mark.parametrize("kblock", [0, 32, 64])
def test_default_variant(slices, kblock):
    info = check(1000, slices, kblock, 0, 0, 0, True)
    expected = 5 if slices >= 6 and kblock != 64 else 1
    assert info["variant"] == expected
    assert info["tile_n"] == (128 if expected == 5 else 64)
    assert info["rows"] == (256 if expected == 5 else 128)


def test_variant_tile_widths():
    assert oz_tiles(700, 8, 0, 2)[1]["tile_n"] == 48   # A in tensor memory, 7 or 8 slices
    assert oz_tiles(700, 6, 0, 2)[1]["tile_n"] == 64
    assert oz_tiles(700, 8, 0, 4)[1]["tile_n"] == 128


def test_bad_arguments():
    for kw in ({"variant": 6}, {"kblock": 48}, {"slices": 5}, {"a_tri": 3}):
        args = dict(n=300, slices=8, kblock=0, variant=0, a_tri=0, b_tri=0, symmetric=False)
        args.update(kw)
        with pytest.raises(PtbGpuError):
            oz_tiles(**args)
    with pytest.raises(PtbGpuError):   # the 128-column kernels take 32-byte K blocks
        oz_tiles(300, 8, 64, 5)
