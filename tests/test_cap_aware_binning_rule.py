"""The rule behind the splat path's cap-aware binning (compat_splat.cu:
k_bin_diff / k_bin_rows / k_bin_cols / k_bin_cutoff / k_bin_pairs), checked in
numpy on random tile rectangles: per (tile, block of splat indices) counts from
2D difference grids equal brute-force counts, and keeping only the blocks up
to the one in which a tile's running count reaches the cap keeps every tile
list's first `cap` entries in index order (and at most one block more).  The
kernels themselves are checked against the oracle on the GPU."""
import numpy as np


def _rects(n, tx, ty, rng):
    x0 = rng.integers(0, tx, n)
    y0 = rng.integers(0, ty, n)
    x1 = np.minimum(tx, x0 + rng.integers(1, 6, n))
    y1 = np.minimum(ty, y0 + rng.integers(1, 6, n))
    live = rng.random(n) > 0.1  # some splats are culled (no rectangle)
    return x0, y0, x1, y1, live


def _block_counts(x0, y0, x1, y1, live, tx, ty, bs):
    n = len(x0)
    nb = -(-n // bs)
    grid = np.zeros((nb, ty + 1, tx + 1), np.int64)
    for i in np.nonzero(live)[0]:
        b = i // bs
        grid[b, y0[i], x0[i]] += 1
        grid[b, y0[i], x1[i]] -= 1
        grid[b, y1[i], x0[i]] -= 1
        grid[b, y1[i], x1[i]] += 1
    grid = np.cumsum(np.cumsum(grid, axis=2), axis=1)  # rows, then columns
    return grid[:, :ty, :tx]


def test_difference_grids_count_every_rectangle():
    rng = np.random.default_rng(1)
    tx, ty, n, bs = 7, 5, 400, 64
    x0, y0, x1, y1, live = _rects(n, tx, ty, rng)
    cnt = _block_counts(x0, y0, x1, y1, live, tx, ty, bs)
    brute = np.zeros_like(cnt)
    for i in np.nonzero(live)[0]:
        brute[i // bs, y0[i]:y1[i], x0[i]:x1[i]] += 1
    np.testing.assert_array_equal(cnt, brute)


def test_cutoff_keeps_the_first_cap_entries_of_every_list():
    rng = np.random.default_rng(2)
    for tx, ty, n, bs, cap in ((6, 4, 3000, 100, 64), (9, 9, 5000, 250, 128), (3, 2, 800, 17, 40)):
        x0, y0, x1, y1, live = _rects(n, tx, ty, rng)
        cnt = _block_counts(x0, y0, x1, y1, live, tx, ty, bs)
        run = np.cumsum(cnt, axis=0)
        nb = cnt.shape[0]
        reach = run >= cap
        cutoff = np.where(reach.any(axis=0), reach.argmax(axis=0), nb - 1)
        for yy in range(ty):
            for xx in range(tx):
                full = [i for i in range(n) if live[i] and x0[i] <= xx < x1[i] and y0[i] <= yy < y1[i]]
                kept = [i for i in full if i // bs <= cutoff[yy, xx]]
                assert kept[:cap] == full[:cap]
                assert len(kept) <= max(cap, 0) + bs
                assert run[-1, yy, xx] == len(full)
