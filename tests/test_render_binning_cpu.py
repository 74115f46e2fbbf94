"""The renderer's binning (csrc/render.cu) as a model on the CPU: the
(tile, particle) pair list built by scan and expand, and the stable LSD
radix sort whose scatter ranks entries per warp with __match_any_sync and
places them from digit-major block offsets.  The model follows the kernels'
index arithmetic (2048 entries a block, 8 warps of 256, 32 lanes a step) and
must give exactly the stable sort by tile, with every write inside the pair
buffer; the pair count must be what the vertex kernel's tile ranges give."""
import numpy as np
import pytest

from oracle import render as O

SORT_BLOCK, WARPS, RADIX = 2048, 8, 256


def radix_pass(keys, vals, shift):
    """One pass of sort_hist_kernel + exclusive scan + sort_scatter_kernel."""
    m = len(keys)
    nblocks = -(-m // SORT_BLOCK)
    digit = (keys >> shift) & (RADIX - 1)
    counts = np.zeros((RADIX, nblocks), np.int64)
    for b in range(nblocks):
        seg = digit[b * SORT_BLOCK:(b + 1) * SORT_BLOCK]
        counts[:, b] = np.bincount(seg, minlength=RADIX)
    offsets = (np.cumsum(counts.reshape(-1)) - counts.reshape(-1)).reshape(RADIX, nblocks)
    out_k = np.full(m, -1, np.int64)
    out_v = np.full(m, -1, np.int64)
    for b in range(nblocks):
        wcount = np.zeros((WARPS, RADIX), np.int64)
        for w in range(WARPS):
            first = b * SORT_BLOCK + w * (SORT_BLOCK // WARPS)
            seg = digit[first:min(m, first + SORT_BLOCK // WARPS)]
            if len(seg):
                wcount[w] = np.bincount(seg, minlength=RADIX)
        base = offsets[:, b] + np.concatenate([np.zeros((1, RADIX), np.int64),
                                               np.cumsum(wcount, axis=0)[:-1]])
        for w in range(WARPS):
            first = b * SORT_BLOCK + w * (SORT_BLOCK // WARPS)
            run = base[w].copy()
            for step in range(SORT_BLOCK // WARPS // 32):
                lo = first + 32 * step
                idx = np.arange(lo, min(m, lo + 32))
                for i in idx:  # a lane's rank: equal digits on lower lanes
                    d = digit[i]
                    rank = int(np.count_nonzero(digit[lo:i] == d))
                    dst = run[d] + rank
                    assert 0 <= dst < m and out_k[dst] == -1
                    out_k[dst], out_v[dst] = keys[i], vals[i]
                for d, c in zip(*np.unique(digit[idx], return_counts=True)):
                    run[d] += c
    assert (out_k >= 0).all()
    return out_k, out_v


@pytest.mark.parametrize("m,tiles,seed", [(1, 1, 0), (2047, 12, 1), (2049, 300, 2), (9000, 14400, 3),
                                          (5000, 70000, 4)])
def test_radix_sort_is_the_stable_sort_by_tile(m, tiles, seed):
    rng = np.random.default_rng(seed)
    # long runs of one tile next to scattered ones, as dense and sparse screen regions give
    keys = np.where(rng.random(m) < 0.5, rng.integers(0, min(tiles, 4), m), rng.integers(0, tiles, m))
    vals = np.arange(m)
    bits = 0
    while (1 << bits) < tiles:
        bits += 1
    k, v = keys.copy(), vals.copy()
    for shift in range(0, bits, 8):
        k, v = radix_pass(k, v, shift)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])


def test_pairs_cover_every_drawn_pixel_in_particle_order():
    """Expanding each visible point over the 16 x 16 tiles of its pixel box
    (one pixel of margin) lists, for every pixel a fragment lands on, that
    point in the pixel's tile; the stable sort keeps the particles of a tile
    in index order."""
    from mog_solver_b200.render import camera_matrices

    rng = np.random.default_rng(7)
    n, W, H = 3000, 97, 53
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-10, 110, (n, 3))
    vel = np.zeros_like(pos)
    v, p = camera_matrices(20.0, 10.0, 2.5, W / H)
    clip, _, _ = O.vertex_stage(pos, vel, v, p, 100.0, 0.0)
    x, y, z, w = (clip[:, i] for i in range(4))
    keep = (w > 0) & (x >= -w) & (x <= w) & (y >= -w) & (y <= w) & (z >= -w) & (z <= w)
    F = np.float32
    xw = (x / w) * F(W * 0.5) + F(W * 0.5)
    yw = (y / w) * F(H * 0.5) + F(H * 0.5)
    tiles_x = -(-W // 16)
    pairs = []
    for q in np.nonzero(keep)[0]:
        h = F(1.0) * F(0.5)
        i0, i1 = max(int(np.floor(xw[q] - h)) - 1, 0), min(int(np.floor(xw[q] + h)) + 1, W - 1)
        j0, j1 = max(int(np.floor(yw[q] - h)) - 1, 0), min(int(np.floor(yw[q] + h)) + 1, H - 1)
        if i0 > i1 or j0 > j1:
            continue
        for ty in range(j0 // 16, j1 // 16 + 1):
            for tx in range(i0 // 16, i1 // 16 + 1):
                pairs.append((ty * tiles_x + tx, q))
        # the pixel a 1-pixel point covers (if any) lies in the listed tiles
        for j in range(j0, j1 + 1):
            for i in range(i0, i1 + 1):
                xc, yc = F(i) + F(0.5), F(j) + F(0.5)
                if xw[q] - h <= xc < xw[q] + h and yw[q] - h <= yc < yw[q] + h:
                    assert (j // 16) * tiles_x + i // 16 in {t for t, pq in pairs if pq == q}
    keys = np.array([t for t, _ in pairs])
    vals = np.array([pq for _, pq in pairs])
    k, v = keys, vals
    for shift in (0, 8):
        k, v = radix_pass(k, v, shift)
    for t in np.unique(k):
        seg = v[k == t]
        assert (np.diff(seg) > 0).all()  # particle order within the tile
