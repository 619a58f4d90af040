"""Near-pair topology built on the GPU against the host build.

Meshes of at least eb_set_device_topology_min triangles build the Sauter-Schwab
near-pair lists on the device (topology.cu), the others on the host
(mesh_host.cpp). Both must give the same lists: the operators of a mesh built
either way are compared bit for bit, in both precisions, on the golden meshes
(closed, open, the reference's shaft meshes), on one with a repeated
triangle, on a perturbed icosphere, and on a fan whose centre vertex is shared by more
triangles than the device pass takes (it falls back to the host).
"""
import os

import numpy as np
import pytest

from easybem_b200 import meshes

pytestmark = pytest.mark.gpu

NEVER = 2**31 - 1


@pytest.fixture(scope="module")
def golden_orders():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_orders.npz"))


@pytest.fixture
def threshold(gpu_lib):
    old = gpu_lib.device_topology_min()
    yield gpu_lib
    gpu_lib.set_device_topology_min(old)


def _fan(n):
    ang = np.linspace(0.0, 2.0 * np.pi, n, endpoint=False)
    nodes = np.vstack([[0.0, 0.0, 0.2], np.c_[np.cos(ang), np.sin(ang), 0.05 * np.sin(3 * ang)]])
    elems = np.array([[1, 2 + k, 2 + (k + 1) % n] for k in range(n)], dtype=np.int32)
    return nodes, elems


def _operators(gpu_lib, nodes, elems, t, u):
    with gpu_lib.Mesh(nodes, elems) as m:
        out = {
            "on_device": m.topology_on_device,
            "near_pairs": m.near_pairs,
            "far_quad_pairs": m.far_quad_pairs,
            "near_bytes": m.near_field_bytes(),
            "fp64": m.apply_sl_dl(t, u),
            "mixed": m.apply_sl_dl(t, u, precision="mixed"),
            "p1": m.apply_sl_p1(u),
        }
    return out


def _cases(golden_ops, golden_orders):
    z, zo = golden_ops, golden_orders
    out = [(n, z[f"{n}_nodes"], z[f"{n}_elems"]) for n in ("cube", "ico2", "torus16", "cap", "pair")]
    out += [(n, zo[f"{n}_nodes"], zo[f"{n}_elems"]) for n in ("shaft0", "shafttxt")]
    # a repeated triangle (the first one again, reversed): its pairs with the
    # original are skipped on both paths
    out.append(("pico2_repeat", z["pico2_nodes"], np.vstack([z["pico2_elems"], z["pico2_elems"][:1, ::-1]])))
    out.append(("pico4",) + meshes.perturbed_icosphere(4, seed=5))
    return out


def test_device_topology_equals_host(threshold, golden_ops, golden_orders):
    gpu_lib = threshold
    for name, nodes, elems in _cases(golden_ops, golden_orders):
        rng = np.random.default_rng(len(name))
        t = rng.normal(size=elems.shape[0])
        u = rng.normal(size=nodes.shape[0])
        gpu_lib.set_device_topology_min(NEVER)
        host = _operators(gpu_lib, nodes, elems, t, u)
        gpu_lib.set_device_topology_min(0)
        dev = _operators(gpu_lib, nodes, elems, t, u)
        assert not host["on_device"] and dev["on_device"], name
        for key in ("near_pairs", "far_quad_pairs", "near_bytes"):
            assert host[key] == dev[key], (name, key)
        for key in ("fp64", "mixed"):
            for a, b in zip(host[key], dev[key]):
                assert np.array_equal(a, b), (name, key)
        assert np.array_equal(host["p1"], dev["p1"]), name


def test_device_topology_falls_back_for_high_valence(threshold):
    gpu_lib = threshold
    nodes, elems = _fan(60)  # the centre vertex is in 60 triangles
    rng = np.random.default_rng(1)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    gpu_lib.set_device_topology_min(NEVER)
    host = _operators(gpu_lib, nodes, elems, t, u)
    gpu_lib.set_device_topology_min(0)
    dev = _operators(gpu_lib, nodes, elems, t, u)
    assert not dev["on_device"]
    assert dev["near_pairs"] == host["near_pairs"] == 60 * 60
    for a, b in zip(host["fp64"], dev["fp64"]):
        assert np.array_equal(a, b)


def test_default_threshold_puts_large_meshes_on_the_device(gpu_lib):
    assert gpu_lib.device_topology_min() == 65536
    with gpu_lib.Mesh(*meshes.perturbed_icosphere(1, seed=0)) as m:
        assert not m.topology_on_device
    with gpu_lib.Mesh(*meshes.perturbed_icosphere(6, seed=1)) as m:  # 81,920 triangles
        assert m.topology_on_device and m.near_pairs == 1064900
    with pytest.raises(Exception):
        gpu_lib.set_device_topology_min(-1)
