"""Path-traced targets on the CPU: the BVH builders and the scalar path tracer
restatement against tests/golden/path_trace.npz (outputs of the reference's
own path_trace.wgsl / path_trace_resolve.wgsl run on the host).

* BVH: the library's host builder (nps_bvh_build) and the bvh.ts
  restatement (oracle/bvh.py) give the fixture's nodes and triangle order bit
  for bit, and the tree is well formed.
* Path tracer: oracle/path_trace.py reproduces the reference's per-pixel
  radiance within 1e-5 on a grid of pixels (float32 arithmetic in the same
  order; the transcendental functions come from numpy rather than the C
  library, which can differ in the last place).
* With the reference checkout present, the shaders are run again and must
  reproduce the fixtures bit for bit.
"""
from pathlib import Path

import numpy as np
import pytest

import bvh as obvh
import path_trace as opt
from conftest import requires_reference

GOLD = Path(__file__).resolve().parent / "golden" / "path_trace.npz"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def lib_bvh():
    from nprush_b200 import build
    build.build()
    from nprush_b200.path_trace import build_bvh
    return build_bvh


def test_bvh_restatement_matches_fixture(gold):
    nodes, tris = obvh.build_bvh(gold["vertices"], gold["indices"])
    np.testing.assert_array_equal(nodes.view(np.uint32), gold["nodes"].view(np.uint32))
    np.testing.assert_array_equal(tris, gold["tris"])


def test_library_bvh_builder_matches_fixture(gold, lib_bvh):
    nodes, tris = lib_bvh(gold["vertices"], gold["indices"])
    np.testing.assert_array_equal(nodes.view(np.uint32), gold["nodes"].view(np.uint32))
    np.testing.assert_array_equal(tris, gold["tris"])
    nodes, tris = lib_bvh(np.zeros((0, 12), np.float32), np.zeros(0, np.uint32))
    np.testing.assert_array_equal(nodes.view(np.uint32), gold["empty_nodes"].view(np.uint32))
    assert tris.shape == (0, 3)


@pytest.mark.parametrize("n_tris,seed", [(1, 0), (4, 1), (5, 2), (37, 3), (600, 4)])
def test_library_bvh_builder_matches_restatement_random(n_tris, seed, lib_bvh):
    """Random soups with repeated coordinates and identical triangles (the
    median-split and empty-bin paths)."""
    rng = np.random.default_rng(seed)
    v = np.zeros((max(3, n_tris), 12), np.float32)
    v[:, :3] = np.round(rng.normal(size=(v.shape[0], 3)) * 4) / 4
    idx = rng.integers(0, v.shape[0], n_tris * 3).astype(np.uint32)
    idx[: 3 * min(n_tris, 6)] = np.tile(idx[:3], min(n_tris, 6))
    a = lib_bvh(v, idx)
    b = obvh.build_bvh(v, idx)
    np.testing.assert_array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
    np.testing.assert_array_equal(a[1], b[1])


def test_bvh_is_well_formed(gold):
    nodes, tris = gold["nodes"], gold["tris"]
    bits = nodes.view(np.uint32)
    seen = np.zeros(len(tris), np.int32)
    stack, visited = [0], 0
    while stack:
        k = stack.pop()
        visited += 1
        if bits[k, 7] & obvh.LEAF_FLAG:
            first, count = int(bits[k, 3]), int(bits[k, 7] & 0x7FFFFFFF)
            assert 1 <= count <= obvh.MAX_LEAF_TRIS
            seen[first:first + count] += 1
            v = gold["vertices"][tris[first:first + count].reshape(-1), :3]
            assert np.all(v >= nodes[k, 0:3]) and np.all(v <= nodes[k, 4:7])
        else:
            for c in (int(bits[k, 3]), int(bits[k, 7])):
                assert c > k  # pre-order
                assert np.all(nodes[c, 0:3] >= nodes[k, 0:3]) and np.all(nodes[c, 4:7] <= nodes[k, 4:7])
                stack.append(c)
    assert visited == len(nodes)
    assert np.all(seen == 1)
    np.testing.assert_array_equal(np.sort(tris, axis=0), np.sort(gold["indices"].reshape(-1, 3), axis=0))


def test_library_bvh_builder_rejects_bad_input(lib_bvh):
    from nprush_b200 import _lib
    v = np.zeros((3, 12), np.float32)
    with pytest.raises(_lib.NpsError):
        lib_bvh(v, np.array([0, 1, 3], np.uint32))
    v[1, 0] = np.nan
    with pytest.raises(_lib.NpsError):
        lib_bvh(v, np.array([0, 1, 2], np.uint32))


@pytest.mark.parametrize("case", ["diffuse", "mirror", "empty"])
def test_restatement_matches_reference_radiance(gold, case):
    verts = {"diffuse": gold["vertices"], "mirror": gold["mirror_vertices"], "empty": np.zeros((0, 12), np.float32)}
    nodes = gold["empty_nodes"] if case == "empty" else gold["nodes"]
    tris = np.zeros((0, 3), np.uint32) if case == "empty" else gold["tris"]
    key, frame = {"diffuse": ("accum_f0", 0), "mirror": ("mirror_accum_f5", 5), "empty": ("empty_accum_f0", 0)}[case]
    sc = opt.Scene(verts[case], nodes, tris, gold["env"])
    want = gold[key]
    h, w = want.shape[:2]
    for y in range(0, h, 4):
        for x in range(0, w, 5):
            got = opt.trace_pixel(sc, gold["inv_view_proj"], x, y, w, h, frame)
            np.testing.assert_allclose(got, want[y, x, :3], atol=1e-5, rtol=0, err_msg=f"pixel {x},{y}")
    assert np.all(want[..., 3] == 1.0)


def test_restatement_matches_every_mirror_pixel(gold):
    """All 45 x 37 pixels of the all-mirror fixture (paths of up to 8 mirror
    bounces, no random directions) from the scalar restatement."""
    sc = opt.Scene(gold["mirror_vertices"], gold["nodes"], gold["tris"], gold["env"])
    want = gold["mirror_accum_f5"]
    h, w = want.shape[:2]
    got = np.array([[opt.trace_pixel(sc, gold["inv_view_proj"], x, y, w, h, 5) for x in range(w)]
                    for y in range(h)], np.float32)
    np.testing.assert_allclose(got, want[..., :3], atol=1e-5, rtol=0)


def test_restatement_resolve(gold):
    np.testing.assert_array_equal(opt.resolve(gold["accum_f012"]), gold["resolved_f012"])


def test_fixture_sanity(gold):
    acc = gold["accum_f012"]
    assert np.all(acc[..., 3] == 3.0)
    assert acc[..., :3].mean() > 0.1 and acc[..., :3].std() > 0.05  # not blank
    m = gold["mirror_accum_f5"][..., :3]
    assert (m.sum(-1) > 0).mean() > 0.9  # most mirror paths escape to the sky


@requires_reference
def test_reference_shaders_reproduce_the_fixtures(tmp_path, monkeypatch):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", GOLD.parent / "make_path_trace_golden.py")
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    monkeypatch.setattr(mk, "HERE", tmp_path)
    mk.main()
    a, b = np.load(GOLD), np.load(tmp_path / "path_trace.npz")
    for k in a.files:
        np.testing.assert_array_equal(a[k], b[k])


@requires_reference
@pytest.mark.parametrize("case", ["soups", "degenerate", "same_centroid", "scene", "empty"])
def test_reference_bvh_builder_equals_restatement(case):
    """The reference's own buildBvh (bvh.ts, translated by oracle/ts2py.py)
    and the restatement in oracle/bvh.py give the same bytes."""
    import refrun
    from nprush_b200 import meshes
    rng = np.random.default_rng(11)
    if case == "soups":  # coordinates rounded to repeat, so centroid ties and equal bounds occur
        inputs = []
        for k in range(8):
            nv, nt = int(rng.integers(3, 80)), int(rng.integers(1, 120))
            v = np.zeros((nv, 12), np.float32)
            v[:, :3] = np.round(rng.normal(size=(nv, 3)) * 3, k % 3)
            inputs.append((v, rng.integers(0, nv, size=(nt, 3)).astype(np.uint32)))
    elif case == "degenerate":  # repeated vertex indices and flat (zero-extent) triangles
        v = np.zeros((10, 12), np.float32)
        v[:, 0] = np.arange(10)
        idx = np.array([[0, 0, 0], [1, 1, 2], [2, 3, 4], [5, 6, 7], [7, 8, 9], [0, 9, 5]] * 3, np.uint32)
        inputs = [(v, idx)]
    elif case == "same_centroid":  # every centroid equal: the split falls back to halves
        v = np.zeros((3 * 40, 12), np.float32)
        for t in range(40):
            s = 0.1 + 0.05 * t
            v[3 * t:3 * t + 3, :3] = [[-s, -s, 0], [s, -s, 0], [0, 2 * s, 0]]
        inputs = [(v, np.arange(120, dtype=np.uint32).reshape(-1, 3))]
    elif case == "scene":
        sc = meshes.demo_scene(5, seed=9, mirror_fraction=0.2, sphere_detail=8)
        inputs = [(sc.vertices, sc.indices)]
    else:
        inputs = [(np.zeros((3, 12), np.float32), np.zeros((0, 3), np.uint32))]
    for v, idx in inputs:
        n_ref, t_ref = refrun.build_bvh(v, idx)
        n_res, t_res = obvh.build_bvh(v, idx)
        np.testing.assert_array_equal(n_ref.view(np.uint32), np.asarray(n_res, np.float32).view(np.uint32))
        np.testing.assert_array_equal(t_ref, t_res)


@requires_reference
def test_library_bvh_builder_equals_reference_on_the_benchmark_scene(lib_bvh):
    """The library's host builder against the reference's own buildBvh on the
    path-tracer benchmark's 12k-triangle scene: the same bytes."""
    import importlib.util

    import refrun
    spec = importlib.util.spec_from_file_location("bench", Path(__file__).resolve().parent.parent / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    sc, _, _ = bench.pt_scene()
    n_ref, t_ref = refrun.build_bvh(sc.vertices, sc.indices)
    n_lib, t_lib = lib_bvh(sc.vertices, sc.indices)
    assert t_ref.shape[0] > 10_000
    np.testing.assert_array_equal(n_lib.view(np.uint32), n_ref.view(np.uint32))
    np.testing.assert_array_equal(t_lib, t_ref)
