"""The C-ABI library on the CPU: it loads, exports every declared symbol, and
its host-side parts (hierarchy builder, ray caster, argument checks) work
without a GPU. No kernel runs here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import kat
from continuum_b200 import _lib, host_scene, scenes
from continuum_b200.kernel import MaskConeKernel, flatten_meshes
from oracle.oracle import OracleScene

HEADER = Path(__file__).resolve().parent.parent / "include" / "continuum_cuda.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"CC_API\s+[\w\s\*]+?\b(cc_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(_lib.EXPORTS) == names


def test_options_defaults():
    o = _lib.default_options()
    assert (o.hierarchy, o.wide_extent, o.light_cone_cap, o.wide_cone_cap, o.points_per_warp, o.flags) == \
        (2, 8.0, 4096, 512, 32, 0)


def _gpu_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-device path")
def test_no_device_gives_none():
    """MaskConeKernel::new returns None without an adapter (lib.rs:1155-1175)."""
    assert MaskConeKernel.new() is None
    h = C.c_void_p()
    assert _lib.load().cc_context_create(0, C.byref(h)) == _lib.CC_ERR_NO_DEVICE
    assert b"device" in _lib.load().cc_last_error()


def _same_arrays(a, b):
    for k in ("ranges", "blas", "blas_items", "nodes", "items"):
        assert a[k].shape == b[k].shape, k
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k


@pytest.mark.parametrize("name", ["box_field", "four_boxes", "rubble", "spheres", "single", "with_empty"])
def test_host_builder_matches_the_oracle_builder(name):
    """The library's hierarchy builder reproduces the reference's layouts
    (hierarchy.rs) bit for bit, as restated independently by the oracle."""
    if name == "box_field":
        meshes = scenes.box_field(grid=4).meshes
    elif name == "four_boxes":
        meshes = kat.four_boxes()
    elif name == "rubble":
        meshes = kat.with_rubble(500)
    elif name == "spheres":
        meshes = [scenes.ground_quad(500.0)] + [scenes.displaced_icosphere((3.0 * i, 1.0, 0.0), 1.0, seed=i,
                                                                           subdivisions=3) for i in range(6)]
    elif name == "single":
        meshes = [np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32)]
    else:
        meshes = [kat.box_mesh((0, 0, 0), (1, 1, 1)), np.zeros((0, 3, 3), np.float32), kat.box_mesh((2, 0, 0), (3, 1, 1))]
    a = host_scene(meshes).arrays()
    b = OracleScene(meshes).arrays()
    _same_arrays(a, b)


def test_parallel_build_of_a_large_mesh_matches():
    """A mesh above a million triangles builds its top levels on several
    threads; the tree is the serial one."""
    unit = scenes.unit_icosphere(5).astype(np.float32)  # 20,480 triangles
    offsets = np.arange(52, dtype=np.float32)[:, None, None, None] * np.array([3.0, 0, 0], np.float32)
    big = (unit[None] + offsets).reshape(-1, 3, 3)  # 1,064,960 triangles in one mesh
    tri9, counts = flatten_meshes([big])
    a = host_scene(tri9=tri9, counts=counts).arrays()
    b = OracleScene(tri9=tri9, counts=counts).arrays()
    _same_arrays(a, b)


def test_oversized_meshes_get_their_own_subtree():
    """object_hierarchy (hierarchy.rs:219-252): a ground 64x larger than the
    median object sits under its own child of the root."""
    meshes = [scenes.ground_quad(1000.0)] + [kat.box_mesh((i, 0, 0), (i + 0.5, 0.5, 0.5)) for i in range(9)]
    a = host_scene(meshes).arrays()
    assert a["nodes"][0]["info"][0] == 1 and a["nodes"][0]["info"][1] == 0
    assert a["items"][0] == 0  # the ground is the first item, in the big subtree
    _same_arrays(a, OracleScene(meshes).arrays())


def test_primary_hits_face_the_camera():
    w = scenes.icosphere_field(n_spheres=10, subdivisions=3, width=96, height=54, with_receivers=False)
    s = host_scene(w.meshes)
    rec, hit = s.primary_hits(w.camera, 96, 54)
    assert hit.all()  # the ground fills the view
    eye = w.camera[:3]
    to_eye = eye[None, :] - rec[:, :3]
    assert np.all(np.einsum("ij,ij->i", rec[:, 4:7], to_eye) > 0)
    assert np.allclose(np.linalg.norm(rec[:, 4:7], axis=1), 1.0, atol=1e-5)


def test_pcg32_known_answers():
    """O'Neill's pcg32 demo sequence for (seed 42, stream 54), the generator
    the reference seeds as Pcg32::new(seed, stream) (flatland rng.rs:9-18)."""
    r = scenes.Pcg32(42, 54)
    got = [r.next_u32() for _ in range(6)]
    assert got == [0xA15C02B7, 0x7B47F409, 0xBA1D3330, 0x83D2F293, 0xBFA4784B, 0xCBED606E]


def test_icosphere_is_closed_and_outward():
    t = scenes.unit_icosphere(5)
    assert t.shape == (20480, 3, 3)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    assert np.all(np.einsum("ij,ij->i", n, t.sum(axis=1)) > 0)
    d = scenes.displaced_icosphere((0, 2, 0), 2.0, seed=3, subdivisions=2)
    r = np.linalg.norm(d.reshape(-1, 3) - np.array([0, 2, 0], np.float32), axis=1)
    assert r.min() >= 2.0 * 0.85 - 1e-4 and r.max() <= 2.0 * 1.15 + 1e-4


def test_invalid_arguments_are_errors_not_crashes():
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.cc_scene_build(None, None, None, 1, C.byref(h)) == _lib.CC_ERR_INVALID
    assert lib.cc_scene_sizes(None, None) == _lib.CC_ERR_INVALID
    # A host-only scene cannot be used for visibility.
    s = host_scene([kat.box_mesh((0, 0, 0), (1, 1, 1))])
    out = _lib.Outputs()
    assert lib.cc_visibility(None, s.handle, None, 0, None, 0, None, C.byref(out), None) == _lib.CC_ERR_INVALID
    # Nor for the entry point without allocation, nor in a batch.
    assert lib.cc_visibility_static(s.handle, None, 0, None, 0, None, C.byref(out), None) == _lib.CC_ERR_INVALID
    assert lib.cc_batch_create(None, C.byref(h)) == _lib.CC_ERR_INVALID
    assert lib.cc_batch_add(None, s.handle, None, 0, None, 0, None, C.byref(out), None) == _lib.CC_ERR_INVALID
    assert lib.cc_batch_submit(None, None, None) == _lib.CC_ERR_INVALID
    assert lib.cc_batch_wait(None, 0) == _lib.CC_ERR_INVALID
    assert lib.cc_batch_tune(None, None, 1, None, None, 0) == -_lib.CC_ERR_INVALID
    s.close()


def test_batch_options_defaults():
    o = _lib.BatchOptions()
    _lib.load().cc_batch_options_default(C.byref(o))
    assert (o.points_per_warp, o.blocks_per_sm, o.flags) == (32, 8, _lib.CC_BATCH_GRAPH)


def test_server_options_and_invalid_arguments():
    lib = _lib.load()
    o = _lib.ServerOptions()
    lib.cc_server_options_default(C.byref(o))
    assert (o.hbm_budget, o.max_inflight, o.max_queue, o.max_launch_cones, o.points_per_warp, o.blocks_per_sm,
            o.deadline_ns_per_cone) == (8 << 30, 4, 256, 2 << 20, 32, 8, 12)
    h = C.c_void_p()
    assert lib.cc_server_create(None, C.byref(o), C.byref(h)) == _lib.CC_ERR_INVALID
    assert lib.cc_server_submit(None, None, None) == _lib.CC_ERR_INVALID
    assert lib.cc_server_wait(None, 1, 0, None) == _lib.CC_ERR_INVALID
    assert lib.cc_server_destroy(None) == _lib.CC_OK
