"""CPU tests of the GPU per-ray code: traverse.cuh and shading.cuh are built
for the host (tests/hostemu, with the device self-checks on) over the same
packed tree the kernels read, and compared bit for bit with the oracle.

This checks the packer (8-byte nodes, re-inserted empty slabs, ropes, leaf
records), the stackless traversal with start-leaf hints and the shared-memory
node prefix, the mailbox and the tie ranks, without a GPU. The GPU tests run
the same functions compiled for sm_100a."""
import numpy as np
import pytest

import oracle as O
from tests import scenes as S

emu = pytest.importorskip("tests.hostemu")


@pytest.fixture(scope="module", params=[(0, {}), (1, dict(seed=1, texture_size=32))],
                ids=["room", "spheres"])
def pair(request):
    cfg, kw = request.param
    mesh, nodes, leaf = S.make_scene(cfg, **kw)
    return O.CpuScene(mesh, nodes, leaf), emu.EmuScene(mesh, nodes, leaf)


def _same_hits(ref, got):
    ok = ref["overflow"] == 0
    assert ok.mean() > 0.999
    for k in ("tri", "t", "u", "v"):
        a, b = ref[k][ok], got[k][ok]
        bad = np.flatnonzero(a.view(np.int32) != b.view(np.int32))
        assert bad.size == 0, (k, bad[:5], a[bad[:5]], b[bad[:5]])


def _rays(kind):
    if kind == "camera":
        return O.raygen(S.ROOM_CAM, 96, 64, 1, 1)
    if kind == "pano":
        return O.raygen(S.PANO_CAM, 64, 32, 1, 1)
    return S.random_rays(8000, seed=3)


@pytest.mark.parametrize("kind", ["camera", "pano", "random"])
@pytest.mark.parametrize("smem", [0, 2048])
def test_traversal_matches_oracle(pair, kind, smem):
    cs, em = pair
    o, d = _rays(kind)
    got = em.intersect(o, d, smem_nodes=smem)
    assert got["err"][0] == 0, got["err"]
    _same_hits(cs.intersect(o, d), got)


@pytest.mark.parametrize("kind", ["camera", "pano", "random"])
def test_step_traversal_matches_leaf_traversal(pair, kind):
    """trav_step (one unit of work per call) gives the oracle's hits and the
    same per-ray work as trav_leaf."""
    cs, em = pair
    o, d = _rays(kind)
    a = em.intersect(o, d, smem_nodes=2048)
    b = em.intersect(o, d, smem_nodes=2048, step=True)
    assert b["err"][0] == 0, b["err"]
    _same_hits(cs.intersect(o, d), b)
    assert np.array_equal(a["node"], b["node"])
    assert np.array_equal(a["counts"], b["counts"])


@pytest.mark.parametrize("step", [False, True])
def test_edge_rays_match_oracle(pair, step):
    """Axis-parallel directions, rays lying in split planes (walked once per
    side), rays aimed at vertices and shared edges, degenerate rays: the
    oracle's hits under the contract of scenes.check_edge_hits, in both
    traversal forms."""
    cs, em = pair
    for name, (o, d) in S.edge_rays(cs, cs.nodes).items():
        got = em.intersect(o, d, step=step)
        assert got["err"][0] == 0, (name, got["err"])
        S.check_edge_hits(name, o, d, cs.intersect(o, d), got["tri"], got["t"], got["u"],
                          got["v"])


def test_edge_rays_same_walks_in_both_forms(pair):
    """On the edge-ray sets (split-plane walks included) trav_step and
    trav_leaf report the same hits, the same hit leaves and the same work."""
    cs, em = pair
    for name, (o, d) in S.edge_rays(cs, cs.nodes, seed=3).items():
        a = em.intersect(o, d)
        b = em.intersect(o, d, step=True)
        for k in ("tri", "t", "u", "v", "node"):
            assert np.array_equal(a[k].view(np.int32), b[k].view(np.int32)), (name, k)
        assert np.array_equal(a["counts"], b["counts"]), name


def test_hinted_secondary_rays_match_oracle(pair):
    """Secondary rays started from the leaf of the previous hit (the kernels'
    start-leaf hint) find the same closest hit as a traversal from the root."""
    cs, em = pair
    o, d = S.random_rays(8000, seed=7)
    first = em.intersect(o, d)
    h = first["tri"] >= 0
    p = o[h] + first["t"][h, None] * d[h]
    rng = np.random.default_rng(5)
    nd = rng.normal(size=p.shape).astype(np.float32)
    nd /= np.linalg.norm(nd, axis=1, keepdims=True)
    for eps in (0.0, 1e-5, 1e-3):
        o2 = (p + np.float32(eps) * nd).astype(np.float32)
        ref = cs.intersect(o2, nd)
        hinted = em.intersect(o2, nd, hints=first["node"][h], smem_nodes=2048)
        assert hinted["err"][0] == 0, hinted["err"]
        _same_hits(ref, hinted)
        stepped = em.intersect(o2, nd, hints=first["node"][h], smem_nodes=2048, step=True)
        assert stepped["err"][0] == 0, stepped["err"]
        _same_hits(ref, stepped)
        plain = em.intersect(o2, nd)
        # a hint never costs more node visits than starting at the root
        assert hinted["counts"][0] <= plain["counts"][0]


def test_hints_on_a_split_plane_do_not_hide_the_other_side(pair):
    """Rays lying in a split plane, each hinted with a leaf that contains its
    origin, chosen on either side of the plane: a hint whose leaf has the
    origin on a face along a zero direction component must not be taken (the
    walk would skip the split planes that need both sides), so the hits stay
    those of the unhinted walks, under the edge-ray contract."""
    cs, em = pair
    o, d = S.edge_rays(cs, cs.nodes, n=500, seed=21)["in_split"]
    meta, _, leaves = em.tree()
    leaf_nodes = np.flatnonzero((meta >> 30) == 3)
    lo = leaves[meta[leaf_nodes] & 0x3FFFFFFF][:, 0:3].view(np.float32)
    hi = leaves[meta[leaf_nodes] & 0x3FFFFFFF][:, 4:7].view(np.float32)
    ref = cs.intersect(o, d)
    for pick in (0, -1):  # first / last leaf (in node order) containing the origin
        hints = np.full(len(o), -1, np.int32)
        for i in range(len(o)):
            inside = np.flatnonzero(((o[i] >= lo) & (o[i] <= hi)).all(axis=1))
            if inside.size:
                hints[i] = leaf_nodes[inside[pick]]
        assert (hints >= 0).mean() > 0.9
        for step in (False, True):
            got = em.intersect(o, d, hints=hints, step=step)
            assert got["err"][0] == 0, got["err"]
            S.check_edge_hits("in_split", o, d, ref, got["tri"], got["t"], got["u"], got["v"])


def test_bad_hints_fall_back_to_root(pair):
    """A hint that is not a leaf node of this tree is ignored."""
    cs, em = pair
    o, d = S.random_rays(2000, seed=11)
    n = em.counts()["nodes"]
    hints = np.random.default_rng(2).integers(-5, n + 5, len(o)).astype(np.int32)
    got = em.intersect(o, d, hints=hints)
    assert got["err"][0] == 0, got["err"]
    _same_hits(cs.intersect(o, d), got)


def test_packed_tree_structure(pair):
    """Children sit side by side, every leaf record's ref range is inside
    leaf_refs, and every rope names a node of the tree (the smallest one that
    covers that face, Popov et al. 2007) or -1 on the scene boundary."""
    cs, em = pair
    c = em.counts()
    meta, split, leaves = em.tree()
    tag = meta >> 30
    child = (meta & 0x3FFFFFFF).astype(np.int64)
    inner = tag != 3
    assert (child[inner] + 1 < c["nodes"]).all()
    assert (child[inner] > np.flatnonzero(inner)).all()
    lf = child[~inner]
    assert ((lf >= 0) & (lf < c["leaves"])).all()
    assert len(np.unique(lf)) == c["leaves"]
    first, count = leaves[:, 3], leaves[:, 7]
    assert ((first >= 0) & (count >= 0) & (first + count <= c["refs"])).all()
    ropes = leaves[:, 8:14]
    assert ((ropes == -1) | ((ropes > 0) & (ropes < c["nodes"]))).all()
    assert (ropes >= 0).any()


def test_shade_and_next_dir_match_oracle(pair):
    cs, em = pair
    o, d = S.random_rays(4000, seed=13)
    hit = cs.intersect(o, d)
    m = hit["tri"] >= 0
    o, d = o[m], d[m]
    rng = np.random.default_rng(1)
    strength = rng.uniform(0.1, 1.0, size=(len(o), 3)).astype(np.float32)
    seeds = rng.integers(0, 2 ** 48, size=len(o), dtype=np.int64)
    for dd in (0, 1):
        ref = cs.shade(o, d, strength, hit["tri"][m], hit["t"][m], seeds, disable_diffuse=dd)
        got = em.shade(o, d, strength, hit["tri"][m], hit["t"][m], seeds.view(np.uint64),
                       disable_diffuse=dd)
        for k in ("contrib", "hit_p", "normal", "strength", "param", "branch"):
            assert np.array_equal(np.asarray(ref[k]).view(np.int32),
                                  np.asarray(got[k]).view(np.int32)), k
        assert np.array_equal(ref["seeds"].view(np.uint64), got["seeds"])
        nref = cs.next_dir(ref["branch"], d, ref["hit_p"], ref["normal"], ref["strength"],
                           ref["param"], ref["seeds"])
        ngot = em.next_dir(got["branch"], d, got["hit_p"], got["normal"], got["strength"],
                           got["param"], got["seeds"])
        alive = nref["alive"] != 0
        assert np.array_equal(nref["alive"], ngot["alive"])
        for k in ("origins", "directions", "strength"):
            assert np.array_equal(nref[k][alive].view(np.int32), ngot[k][alive].view(np.int32)), k
