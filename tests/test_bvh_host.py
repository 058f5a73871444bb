"""The host BVH builder (cupbr_b200/csrc/bvh_build.cpp) on the CPU, through
a small harness compiled here (tests/bvh_host_harness.cpp).

The device builder reproduces this builder's arrays byte for byte (GPU
tests); that rests on the host tree depending only on which primitives a
node holds, not on the order they sit in or on thread timing.  Checked
here: two builds of the same boxes (large enough for the builder's
threads) are byte-identical; every leaf lists its primitives in ascending
id order; every child box holds its leaf's primitive boxes; every
primitive appears once; leaves respect max_leaf; boxes with one common
centroid (no SAH split) are split by id, so the leaf order is 0, 1, 2, ...
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "cupbr_b200", "csrc")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("bvh") / "bvh_host_harness")
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-ffp-contract=off", "-I", CSRC,
           os.path.join(HERE, "bvh_host_harness.cpp"), os.path.join(CSRC, "bvh_build.cpp"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def build(exe, tmp_path, boxes, max_leaf=4, tag="a"):
    src, dst = tmp_path / f"boxes_{tag}.bin", tmp_path / f"out_{tag}.bin"
    np.ascontiguousarray(boxes, dtype=np.float32).tofile(src)
    subprocess.run([exe, str(src), str(dst), str(max_leaf)], check=True)
    raw = dst.read_bytes()
    n_nodes, leaves, depth = np.frombuffer(raw[:12], np.uint32)
    sah = np.frombuffer(raw[12:20], np.float64)[0]
    nodes = np.frombuffer(raw[20:20 + 128 * int(n_nodes)], np.float32).reshape(-1, 32)
    perm = np.frombuffer(raw[20 + 128 * int(n_nodes):], np.uint32)
    return raw, nodes, perm, int(leaves), int(depth), sah


def leaf_ranges(nodes):
    """(slot start, count, child box) of every leaf child in the node array."""
    refs = nodes[:, 24:28].view(np.int32)
    out = []
    for i in range(len(nodes)):
        for k in range(4):
            r = int(refs[i, k])
            if r >= 0 or r == np.iinfo(np.int32).min:  # inner node or empty slot
                continue
            v = ~r & 0xFFFFFFFF
            lo = nodes[i, [0 + k, 8 + k, 16 + k]]
            hi = nodes[i, [4 + k, 12 + k, 20 + k]]
            out.append((v >> 3, (v & 7) + 1, lo, hi))
    return out


def random_boxes(n, seed):
    rng = np.random.default_rng(seed)
    c = np.concatenate([rng.normal(size=(n // 2, 3)) * 0.3 + rng.integers(-4, 4, size=(n // 2, 3)),
                        rng.uniform(-5, 5, size=(n - n // 2, 3))]).astype(np.float32)
    half = rng.uniform(0.001, 0.05, size=(n, 3)).astype(np.float32)
    dup = rng.choice(n, n // 50, replace=False)  # some boxes repeated exactly
    c[dup[1:]] = c[dup[0]]
    half[dup[1:]] = half[dup[0]]
    return np.concatenate([c - half, c + half], axis=1)


def test_deterministic_and_well_formed(harness, tmp_path):
    boxes = random_boxes(200_000, 7)  # above the builder's threading threshold
    raw1, nodes, perm, leaves, depth, sah = build(harness, tmp_path, boxes, tag="a")
    raw2, *_ = build(harness, tmp_path, boxes, tag="b")
    assert raw1 == raw2                                                # byte-identical rebuild
    assert np.array_equal(np.sort(perm), np.arange(len(boxes)))        # every primitive once
    lr = leaf_ranges(nodes)
    assert len(lr) == leaves and 0 < depth < 48 and sah > 0
    for start, cnt, lo, hi in lr:
        ids = perm[start:start + cnt]
        assert cnt <= 4
        assert np.all(np.diff(ids.astype(np.int64)) > 0)               # ascending ids
        assert np.all(boxes[ids, :3] >= lo) and np.all(boxes[ids, 3:] <= hi)


def test_identical_centroids_split_by_id(harness, tmp_path):
    box = np.array([0.0, 0.0, 0.0, 1.0, 1.0, 1.0], np.float32)
    for n, max_leaf in ((64, 4), (1000, 3), (5, 8)):
        _, nodes, perm, leaves, _, _ = build(harness, tmp_path, np.tile(box, (n, 1)), max_leaf=max_leaf,
                                             tag=f"same{n}")
        assert np.array_equal(perm, np.arange(n))                      # median by id: order kept
        assert all(cnt <= max_leaf for _, cnt, _, _ in leaf_ranges(nodes))
