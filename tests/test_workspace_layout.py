"""Workspace sizing without a GPU: every allocation that backs the stage kernels' scratch
(solver slots, the autotune bench, the allocation-free entry point) is sized by
sbg_workspace_bytes(n, precision, pairs), which must cover the seven 256-byte-aligned regions
the kernels address, for every order and capacity."""
from __future__ import annotations

import numpy as np


def _align(x, a=256):
    return (x + a - 1) // a * a


def carve_end(n, pairs):
    """End of the last region: LV (n*n complex), tau (n complex), d, e (n real), the QL rotation
    log ((3n^2)/2 + 8n + 16 entries of 16 B, or the mixed form's stash of C, NP (NP + 4) entries
    with NP = n rounded up to a multiple of 8, if that is larger), perm (n int), flag (1 int), per
    pair, each region rounded up to 256 bytes."""
    np_ = (n + 7) // 8 * 8
    cap = max((3 * n * n) // 2 + 8 * n + 16, np_ * (np_ + 4))
    regions = [16 * n * n * pairs, 16 * n * pairs, 8 * n * pairs, 8 * n * pairs, 16 * cap * pairs,
               4 * n * pairs, 4 * pairs]
    return sum(_align(r) for r in regions)


def test_workspace_bytes_covers_the_carve_for_every_n_and_capacity(monkeypatch):
    monkeypatch.delenv("SBG_QL_LOG_CAPACITY", raising=False)
    import sbg
    lib = sbg.load()
    pairs = np.arange(1, 4097)
    for n in range(1, 257):
        per = lib.sbg_workspace_bytes_per_pair(n, 0)
        got = np.array([lib.sbg_workspace_bytes(n, 0, int(p)) for p in pairs], dtype=np.int64)
        want = np.array([carve_end(n, int(p)) for p in pairs], dtype=np.int64)
        assert (got >= want).all(), (n, pairs[got < want][:5])
        assert (got <= per * pairs + 7 * 256).all(), n
    assert lib.sbg_workspace_bytes(0, 0, 10) == 0 and lib.sbg_workspace_bytes(54, 0, 0) == 0


def carve_end_mixed(n, pairs):
    """The mixed form's layout: above n = 63 six more regions follow the seven of carve_end -- five
    n x n complex matrices per pair (the refinement's C, second Y buffer, P / E, G, S) and one int
    per pair (its status); at n <= 63 the layout is the plain one."""
    end = carve_end(n, pairs)
    if n > 63:
        end += 5 * _align(16 * n * n * pairs) + _align(4 * pairs)
    return end


def test_mixed_workspace_bytes_cover_the_carve(monkeypatch):
    monkeypatch.delenv("SBG_QL_LOG_CAPACITY", raising=False)
    import sbg
    lib = sbg.load()
    pairs = np.arange(1, 2049)
    for n in range(1, 257):
        per = lib.sbg_workspace_bytes_per_pair(n, 1)
        got = np.array([lib.sbg_workspace_bytes(n, 1, int(p)) for p in pairs], dtype=np.int64)
        want = np.array([carve_end_mixed(n, int(p)) for p in pairs], dtype=np.int64)
        assert (got >= want).all(), (n, pairs[got < want][:5])
        assert (got <= per * pairs + 13 * 256).all(), n
        if n <= 63:
            assert lib.sbg_workspace_bytes_per_pair(n, 1) == lib.sbg_workspace_bytes_per_pair(n, 0)
        else:
            assert per == lib.sbg_workspace_bytes_per_pair(n, 0) + 80 * n * n + 4


def test_old_slack_was_short_somewhere():
    """The sizing this replaced (per-pair bytes x pairs + 5 x 256) fell short of the carve for
    some orders and capacities: the exact size matters."""
    short = 0
    for n in (1, 3, 9, 27, 49, 57, 249):
        for p in range(1, 4097):
            cap = (3 * n * n) // 2 + 8 * n + 16
            per = 16 * n * n + 16 * n + 16 * n + 16 * cap + 4 * n + 4
            if carve_end(n, p) > per * p + 5 * 256:
                short += 1
                break
    assert short > 0
