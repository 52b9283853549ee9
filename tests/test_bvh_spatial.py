"""The spatial-split BVH built on the host (no GPU): every triangle is
referenced by some leaf, the tree's clipped leaf bounds are conservative
(the closest hit of random rays through the tree equals brute force over
all triangles, for the binned and the spatial-split trees alike), the SAH
cost drops on a soup of small overlapping triangles, and the records grow
within the 4x budget."""
import numpy as np

from oxideav_render_b200 import native, testscenes as ts


def soup_positions(scene):
    return np.ascontiguousarray(np.concatenate([it.positions.reshape(-1, 9) for it in scene.items]).astype(np.float32))


def build(pos, spatial):
    lib = native.load()
    n = pos.shape[0]
    st = np.zeros(6)
    nodes = np.zeros((10 * n + 16, 16), np.float32)
    recs = np.zeros((5 * n + 16, 12), np.float32)
    rc = lib.pt_debug_build_bvh(pos.ctypes.data_as(native.fp), n, spatial, st.ctypes.data_as(native.dp),
                                nodes.ctypes.data, nodes.shape[0], recs.ctypes.data, recs.shape[0])
    assert rc == 0
    return st, nodes[:int(st[0])], recs[:int(st[5])]


def hit_t(o, d, v0, v1, v2):
    """Moller-Trumbore in float64 over arrays of triangles: t or inf."""
    e1, e2 = v1 - v0, v2 - v0
    p = np.cross(d, e2)
    det = np.einsum("ij,ij->i", e1, p)
    ok = np.abs(det) > 1e-12
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    tv = o - v0
    u = np.einsum("ij,ij->i", tv, p) * inv
    q = np.cross(tv, e1)
    v = (q @ d) * inv
    t = np.einsum("ij,ij->i", e2, q) * inv
    good = ok & (u >= 0) & (v >= 0) & (u + v <= 1) & (t > 0)
    return np.where(good, t, np.inf)


def trace(nodes, recs, o, d):
    """Closest hit through the two-child tree (slab tests, nearest first)."""
    ints = nodes.view(np.int32)
    inv = 1.0 / np.where(d == 0, 1e-30, d)
    best, stack = np.inf, [0]
    while stack:
        ni = stack.pop()
        if ni < 0:
            first = ~ni
            cnt = (first >> 27) & 0xF
            first &= (1 << 27) - 1
            r = recs[first:first + cnt].astype(np.float64)
            t = hit_t(o, d, r[:, 0:3], r[:, 4:7], r[:, 8:11])
            best = min(best, float(t.min()) if t.size else np.inf)
            continue
        a, b, c, dd = nodes[ni, 0:4], nodes[ni, 4:8], nodes[ni, 8:12], ints[ni, 12:16]
        hits = []
        for lo, hi, ch in (((a[0], a[2], c[0]), (a[1], a[3], c[1]), dd[0]),
                           ((b[0], b[2], c[2]), (b[1], b[3], c[3]), dd[1])):
            t0 = (np.array(lo) - o) * inv
            t1 = (np.array(hi) - o) * inv
            tn = max(np.minimum(t0, t1).max(), 0.0)
            tf = min(np.maximum(t0, t1).min() * (1 + 1e-6), best)
            if tn <= tf:
                hits.append((tn, int(ch)))
        for _, ch in sorted(hits, reverse=True):
            stack.append(ch)
    return best


def check_tree(pos, spatial, rays):
    st, nodes, recs = build(pos, spatial)
    n = pos.shape[0]
    gids = recs[:, 3].view(np.uint32)
    assert np.array_equal(np.unique(gids), np.arange(n, dtype=np.uint32))  # every triangle referenced
    assert n <= st[5] <= 4 * n + 2
    if not spatial:
        assert st[5] == n
    tri = pos.astype(np.float64).reshape(-1, 3, 3)
    hits = 0
    for o, d in rays:
        want = hit_t(o, d, tri[:, 0], tri[:, 1], tri[:, 2]).min()
        assert trace(nodes, recs, o, d) == want
        hits += np.isfinite(want)
    assert hits >= 0.6 * len(rays)  # the rays do find triangles
    return st


def test_spatial_split_tree_is_conservative_and_better_on_a_soup():
    scene = ts.random_soup(20000, seed=5)
    pos = soup_positions(scene)
    rng = np.random.default_rng(2)
    idx = rng.integers(0, pos.shape[0], 60)
    w = rng.dirichlet([1, 1, 1], 60)
    org = (pos[idx].reshape(-1, 3, 3).astype(np.float64) * w[:, :, None]).sum(1)
    dirs = rng.normal(size=(60, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    rays = list(zip(org + 1e-4 * dirs, dirs))
    # Camera-like rays from outside the cube as well.
    cam = np.array([0.5, 0.5, 2.2])
    for _ in range(20):
        tgt = rng.random(3)
        d = tgt - cam
        rays.append((cam, d / np.linalg.norm(d)))
    binned = check_tree(pos, 0, rays)
    spatial = check_tree(pos, 1, rays)
    assert spatial[3] < binned[3]  # SAH cost
    assert spatial[5] > binned[5]  # triangles cut by split planes are referenced twice


def test_spatial_split_tree_on_a_mesh_is_conservative():
    scene, _ = ts.sphere_grid_c1(32, 1)
    pos = soup_positions(scene)[:20000]
    rng = np.random.default_rng(3)
    # Rays from random points on the spheres' triangles toward other
    # triangles' centres: each ray's target lies on a triangle.
    tri = pos.astype(np.float64).reshape(-1, 3, 3)
    rays = []
    for _ in range(40):
        a, b = rng.integers(0, len(tri), 2)
        o = tri[a].mean(0) + rng.normal(size=3) * 0.5
        d = tri[b].mean(0) - o
        rays.append((o, d / np.linalg.norm(d)))
    check_tree(pos, 1, rays)
