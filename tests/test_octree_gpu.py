"""The device octree builder (snog_scene_create_ex with OCTREE_DEVICE) against
the host builder and the reference's golden octrees.

Both builders must give the same tree: the node arrays in breadth-first order,
the child masks, every surface list in last-in first-out order, the root cube
and the statistics (space/octree-builder.cc:173-650).  The cases cover root
growth in every direction (surfaces far outside the current root, ties), forced
insertion of small straddling surfaces, degenerate triangles left out, trees
deeper than 21 levels (keys wider than 64 bits), and the full-size
intersection-only (1M triangles) and terrain (2M triangles) scenes.
"""

import hashlib

import numpy as np
import pytest

from gen_golden import TRACE_CASES
import snogray_b200 as sb
from snogray_b200 import Scene, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _device():
    sb.init(0)


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def growth_scene(seed=5):
    """Triangles whose boxes fall ever further outside the root, on alternating
    sides of every axis, some exactly on the cube's faces (ties grow down), with
    small ones between that straddle midplanes."""
    rng = np.random.default_rng(seed)
    tris = []
    for k in range(60):
        scale = 2.0 ** (k % 23 - 6)
        sign = np.array([1 if (k >> a) & 1 else -1 for a in range(3)], np.float64)
        c = sign * scale * rng.uniform(0.5, 1.5, 3)
        if k % 7 == 3:
            c = np.round(c)                      # on lattice points: boxes touch faces
        e = rng.normal(size=(2, 3)) * scale * 0.05
        tris.append([c, c + e[0], c + e[1]])
        for _ in range(3):                       # small straddlers near the origin
            c2 = rng.uniform(-1, 1, 3) * 0.01
            e2 = rng.normal(size=(2, 3)) * 1e-3
            tris.append([c2, c2 + e2[0], c2 + e2[1]])
    v = np.asarray(tris, np.float32).reshape(-1, 3)
    n = len(tris)
    return sb.SceneData(materials=scenes.random_triangles(1).materials, vertices=v,
                        triangles=np.arange(3 * n, dtype=np.uint32).reshape(n, 3),
                        tri_mat=np.zeros(n, np.uint32), name="growth")


def deep_scene():
    """Sizes from 1 down to 1e-7: a tree 27 levels deep, so node keys use more
    than 64 bits (21 digits fit in the high word)."""
    rng = np.random.default_rng(9)
    tris = []
    for k in range(400):
        s = 10.0 ** rng.uniform(-7, 0)
        c = rng.uniform(0, 1, 3)
        e = rng.normal(size=(2, 3)) * s
        tris.append([c, c + e[0], c + e[1]])
    v = np.asarray(tris, np.float32).reshape(-1, 3)
    n = len(tris)
    return sb.SceneData(materials=scenes.random_triangles(1).materials, vertices=v,
                        triangles=np.arange(3 * n, dtype=np.uint32).reshape(n, 3),
                        tri_mat=np.zeros(n, np.uint32), name="deep")


def degenerate_scene():
    sd = scenes.random_triangles(2000, seed=1)
    v = sd.vertices.copy()
    v[5] = v[3]                                   # triangle 1 collapses to a segment
    v[3 * 700 + 2] = v[3 * 700]                   # and triangle 700
    sd.vertices = v
    return sd


CASES = {
    "cornell": lambda: scenes.cornell_box(),
    "soup_wide": lambda: scenes.random_triangles(3000, seed=17, edge_lo=0.0, edge_hi=0.3),
    "mixed": lambda: scenes.mixed_scene(500, 500, 500, seed=23),
    "soup_scene": lambda: scenes.soup_scene(5000, 4),
    "terrain_small": lambda: scenes.terrain_scene(n=48, n_spheres=10, seed=3, env_w=32, env_h=16),
    "growth": growth_scene,
    "deep": deep_scene,
    "degenerate": degenerate_scene,
}

INFO_KEYS = ("n_nodes", "n_plist", "max_depth", "n_leaf_nodes", "n_list_surfaces", "origin", "size")


def _both(sd):
    with Scene(sd, octree=Scene.OCTREE_HOST) as h, Scene(sd, octree=Scene.OCTREE_DEVICE) as d:
        return (h.info(), h.octree()), (d.info(), d.octree())


def _same_tree(host, dev):
    (hi, ho), (di, do) = host, dev
    for k in INFO_KEYS:
        assert hi[k] == di[k], k
    for k in ("children", "heads", "list", "origin"):
        assert np.array_equal(ho[k], do[k]), k
    assert np.float32(ho["size"]) == np.float32(do["size"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_octree_equals_host_octree(name):
    _same_tree(*_both(CASES[name]()))


def test_deep_case_is_deeper_than_64_bit_keys():
    with Scene(deep_scene(), octree=Scene.OCTREE_DEVICE) as d:
        assert d.info()["max_depth"] > 22


@pytest.mark.parametrize("name", sorted(TRACE_CASES))
def test_device_octree_matches_reference_fixture(name, golden):
    g = golden(f"trace_{name}.npz")
    sd = TRACE_CASES[name][0]()
    with Scene(sd, octree=Scene.OCTREE_DEVICE) as sc:
        oc = sc.octree()
    assert len(oc["heads"]) == int(g["oct_nodes"])
    assert np.array_equal(oc["origin"], g["oct_origin"])
    assert np.float32(oc["size"]) == np.float32(g["oct_size"])
    assert _digest(oc["children"]) == str(g["oct_children_digest"])
    assert _digest(oc["heads"]) == str(g["oct_heads_digest"])
    assert _digest(oc["list"]) == str(g["oct_list_digest"])


def test_traces_agree_across_builders():
    sd = scenes.mixed_scene(3000, 200, 200, seed=41)
    rays = scenes.random_rays(20000, seed=42)
    with Scene(sd, octree=Scene.OCTREE_HOST) as h, Scene(sd, octree=Scene.OCTREE_DEVICE) as d:
        ph, th, _, ch = h.trace(rays, 10000)
        pd, td, _, cd = d.trace(rays, 10000)
    assert np.array_equal(ph, pd) and np.array_equal(th, td)
    assert ch == cd


@pytest.mark.parametrize("make", [lambda: scenes.random_triangles(1 << 20, seed=2),
                                  lambda: scenes.terrain_scene()], ids=["soup_1M", "terrain_2M"])
def test_full_size_device_octree_equals_host(make):
    _same_tree(*_both(make()))


def test_auto_mode_gives_the_same_tree():
    sd = scenes.random_triangles(70000, seed=3)      # above the device threshold
    with Scene(sd) as a, Scene(sd, octree=Scene.OCTREE_HOST) as h:
        for k in ("children", "heads", "list"):
            assert np.array_equal(a.octree()[k], h.octree()[k]), k


def test_unknown_octree_mode_rejected():
    with pytest.raises(sb.SnogError) as e:
        Scene(scenes.cornell_box(), octree=7)
    assert e.value.code == sb.SNOG_EINVAL
