"""Generates the golden fixtures of tests/golden/ (run: python tests/golden/make_golden.py).

The reference (dimforge/slosh) has no runnable CPU path here and no golden
vectors of its own, so the fixtures are built from its published rules by an
implementation independent of the oracle (pure Python / numpy):

* prefix_sum.npz — the input recipe of the reference's (commented-out)
  prefix-sum test, src/grid/prefix_sum.rs:219-270: length 15071, values
  `random % 10000` (seeded here), expected output = exclusive scan with the
  total dropped (eval_cpu, src/grid/prefix_sum.rs:97-110).
* grid_small.json — a small hand-built particle set (negative coordinates,
  block boundaries, exact round-half ties) and its sparse-grid layout in
  canonical order: packed keys (shaders/slosh/grid/grid.slang:77-91), per
  block bucket counts of primaries and extras (shaders/slosh/grid/sort.slang:
  15-42, 208-246), first_particle (exclusive scan) and the sorted ids
  (sort.slang:304-357) with each bucket ordered by particle id.
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def pack_key(b, dim):
    if dim == 3:
        return ((b[0] + 0x3FF) & 0x7FF) | (((b[1] + 0x1FF) & 0x3FF) << 11) | (((b[2] + 0x3FF) & 0x7FF) << 21)
    return ((b[0] + 0x7FFF) & 0xFFFF) | (((b[1] + 0x7FFF) & 0xFFFF) << 16)


def cell_of(x, h, dim):
    bw = 4 if dim == 3 else 8
    blk, loc = [], []
    for k in range(dim):
        q = np.float32(np.float32(x[k]) / np.float32(h))
        assoc = float(np.rint(q)) - 1.0  # half-to-even
        b = int(np.floor(assoc / bw))
        blk.append(b)
        loc.append(int(assoc - b * bw))
    return blk, loc


def assoc_offsets(dim):
    if dim == 3:
        return [(0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)]
    return [(0, 0), (0, 1), (1, 0), (1, 1)]


def layout(positions, h, dim):
    bw = 4 if dim == 3 else 8
    npb = 4 if dim == 3 else 8
    nb_buckets = 10 if dim == 3 else 18
    min_shift = 2 if dim == 3 else 6
    info = []
    active = set()
    for i, x in enumerate(positions):
        blk, loc = cell_of(x, h, dim)
        info.append((blk, loc))
        active.add(tuple(blk))
    prim = list(active)
    for b in prim:
        for o in assoc_offsets(dim)[1:]:
            active.add(tuple(b[k] + o[k] for k in range(dim)))
    keys = sorted(pack_key(b, dim) for b in active)
    rank = {k: r for r, k in enumerate(keys)}
    buckets = [[[] for _ in range(nb_buckets)] for _ in keys]
    for i, (blk, loc) in enumerate(info):
        r0 = rank[pack_key(blk, dim)]
        # primaries are ordered by (cell, id); cell = x + BW y (+ BW^2 z)
        cell = sum(loc[k] * bw**k for k in range(dim))
        buckets[r0][loc[dim - 1]].append((cell, i))
        for o in assoc_offsets(dim)[1:]:
            if all(loc[k] >= min_shift for k in range(dim) if o[k] == 1):
                nbk = [blk[k] + o[k] for k in range(dim)]
                local = loc[dim - 1] - o[dim - 1] * bw
                eb = npb + (max(local, -2) + 2)
                buckets[rank[pack_key(nbk, dim)]][eb].append(i)
    first, np_, npe, counts, sorted_ids = [], [], [], [], []
    run = 0
    for r in range(len(keys)):
        first.append(run)
        c = [len(buckets[r][b]) for b in range(nb_buckets)]
        counts.append(c)
        np_.append(sum(c[:npb]))
        npe.append(sum(c))
        for b in range(nb_buckets):
            if b < npb:
                sorted_ids.extend(i for _, i in sorted(buckets[r][b]))
            else:
                sorted_ids.extend(sorted(buckets[r][b]))
        run += sum(c)
    return {
        "keys": keys,
        "first_particle": first,
        "num_particles": np_,
        "num_particles_with_extras": npe,
        "bucket_counts": counts,
        "sorted_ids": sorted_ids,
    }


def small_positions_3d(h):
    rng = np.random.default_rng(11)
    pts = [
        # exact half-cell ties: x/h = k + 0.5 rounds to the even neighbour
        (2.5 * h, 3.5 * h, 4.5 * h),
        (-2.5 * h, -3.5 * h, -0.5 * h),
        # block boundaries and negative coordinates
        (0.0, 0.0, 0.0),
        (-h, -h, -h),
        (4 * h - 1e-6, 4 * h, 5 * h),
        (-4 * h, 7 * h, -9 * h),
    ]
    pts += [tuple(p) for p in rng.uniform(-10 * h, 10 * h, size=(60, 3))]
    # a dense clump sharing cells (duplicate keys within warps)
    pts += [tuple(p) for p in 3 * h + rng.uniform(0, 2 * h, size=(40, 3))]
    return [tuple(float(np.float32(c)) for c in p) for p in pts]


def small_positions_2d(h):
    rng = np.random.default_rng(12)
    pts = [(2.5 * h, 3.5 * h), (-0.5 * h, -1.5 * h), (0.0, 0.0), (8 * h, -8 * h), (7.9 * h, 15.5 * h)]
    pts += [tuple(p) for p in rng.uniform(-20 * h, 20 * h, size=(60, 2))]
    return [tuple(float(np.float32(c)) for c in p) for p in pts]


def main():
    rng = np.random.default_rng(0)
    v = (rng.integers(0, 2**32, size=15071, dtype=np.uint64) % 10000).astype(np.uint32)
    expected = np.zeros_like(v)
    expected[1:] = np.cumsum(v.astype(np.uint64))[:-1].astype(np.uint32)
    np.savez_compressed(os.path.join(HERE, "prefix_sum.npz"), input=v, expected=expected)

    out = {}
    h3 = float(np.float32(1.0 / 16.0))
    p3 = small_positions_3d(h3)
    out["grid3"] = {"dim": 3, "h": h3, "positions": p3, "layout": layout(p3, h3, 3)}
    h2 = float(np.float32(1.0 / 32.0))
    p2 = small_positions_2d(h2)
    out["grid2"] = {"dim": 2, "h": h2, "positions": p2, "layout": layout(p2, h2, 2)}
    with open(os.path.join(HERE, "grid_small.json"), "w") as f:
        json.dump(out, f)
    print("wrote prefix_sum.npz and grid_small.json")


if __name__ == "__main__":
    main()
