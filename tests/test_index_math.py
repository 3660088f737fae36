"""Index arithmetic of the spread's range path, checked exhaustively on the CPU.

A spread tile covers grid points [lo, lo + ext) of a dimension of extent K; a
sample's taps are (k0 + j) mod K, j < J.  When K >= T + J (T the tile extent),
the taps that land in the tile are one index range of j whose tile-local
coordinates are l + j, with l = k0 - lo, or k0 - lo - K when the taps reach
the tile only after the periodic wrap.  The kernel relies on this to serve
wrapping samples on its fast path.
"""
import pytest


def _range_path(k0, lo, ext, K, J):
    l = k0 - lo
    if l >= ext:
        l -= K
    return {l + j for j in range(max(0, -l), min(J, ext - l))}


def _truth(k0, lo, ext, K, J):
    return {(k0 + j) % K - lo for j in range(J) if 0 <= (k0 + j) % K - lo < ext}


@pytest.mark.parametrize("T", [4, 8, 16, 32])
def test_wrapped_taps_form_one_range(T):
    for K in range(6, 72):
        for J in range(1, 17):
            if J > K or K < T + J:
                continue
            for lo in range(0, K, T):
                ext = min(T, K - lo)
                for k0 in range(K):
                    assert _range_path(k0, lo, ext, K, J) == _truth(k0, lo, ext, K, J)
