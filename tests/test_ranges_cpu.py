"""Host logic of the streamed gradient pass (no GPU): the slice ranges that
the index columns are uploaded, factorised and marched in, and that the
adjoint runs backwards, cover slices 1..L once, in order, for every depth the
streamed path takes (L >= 64); the first range is short and the later ones
double, so each block's upload and factorisation fit under the march before
it."""

from types import SimpleNamespace

import pytest

from thick_ptycho_b200.gradient import PWEGradient2D


def _ranges(L):
    holder = SimpleNamespace(engine=SimpleNamespace(L=L), _RANGE_FRACTIONS=PWEGradient2D._RANGE_FRACTIONS)
    return PWEGradient2D._slice_ranges(holder)


@pytest.mark.parametrize("L", [64, 65, 100, 127, 199, 255, 511, 1023, 1024, 2047, 4095])
def test_slice_ranges_cover_every_slice_once(L):
    r = _ranges(L)
    assert r[0][0] == 1 and r[-1][1] == L
    for (a0, a1), (b0, b1) in zip(r, r[1:]):
        assert a0 <= a1 and b0 == a1 + 1
    assert sum(b - a + 1 for a, b in r) == L
    # a short first range, then (up to rounding) doubling lengths
    lengths = [b - a + 1 for a, b in r]
    assert lengths[0] <= max(2, L // 16)
    for x, y in zip(lengths[1:], lengths[2:]):
        assert y >= x


def test_slice_ranges_at_the_headline_depth():
    assert _ranges(1023) == [(1, 32), (33, 64), (65, 128), (129, 256), (257, 512), (513, 1023)]
