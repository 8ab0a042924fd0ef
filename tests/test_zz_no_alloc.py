"""cc_visibility_static, the entry point that allocates nothing, against
cc_visibility with device pointers on a B200.

Its scratch is one fixed device array per device, shared by every call, so
this file is collected last: it must pass alone and after every other test
has run its own calls on the same device.
"""
import numpy as np
import pytest

from continuum_b200 import Light, RectLight, _lib, light_gpu, scenes

pytestmark = pytest.mark.gpu

KEYS = ("full", "any", "partial", "irradiance", "fraction", "work")


def device_outputs(torch, n):
    dev = torch.device("cuda:0")
    return {"full": torch.zeros(n, dtype=torch.int64, device=dev), "any": torch.zeros(n, dtype=torch.int64, device=dev),
            "partial": torch.zeros(n, 64, device=dev), "irradiance": torch.zeros(n, device=dev),
            "fraction": torch.zeros(n, device=dev), "work": torch.zeros(n, 4, dtype=torch.int32, device=dev)}


def host(outs):
    return {k: v.cpu().numpy().copy() for k, v in outs.items()}


def run(kernel, entry, scene, rec, lig, outs, stream):
    fn = kernel.visibility_device if entry == "device" else kernel.visibility_static
    fn(scene, rec.data_ptr(), rec.shape[0], lig.data_ptr(), lig.shape[0], {k: v.data_ptr() for k, v in outs.items()},
       stream=stream.cuda_stream)


def assert_same(a, b):
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k


def second_light():
    return light_gpu(Light.rect(RectLight((2.0, 5.0, -1.0), (0.0, 0.0, 1.5), (1.0, 0.0, 0.0), one_sided=False)))


def test_two_calls_in_a_row_equal_cc_visibility(kernel):
    """Two workloads of different sizes, each through cc_visibility and then
    twice in a row through cc_visibility_static on one stream: identical."""
    import torch

    stream = torch.cuda.Stream()
    for w in (scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=4, width=160, height=90),
              scenes.box_field(grid=128)):
        scene = kernel.scene(w.meshes)
        rec = torch.from_numpy(w.receivers).cuda()
        lig = torch.from_numpy(w.lights).cuda()
        n = rec.shape[0] * lig.shape[0]
        ref, a, b = device_outputs(torch, n), device_outputs(torch, n), device_outputs(torch, n)
        with torch.cuda.stream(stream):
            run(kernel, "device", scene, rec, lig, ref, stream)
            run(kernel, "static", scene, rec, lig, a, stream)
            run(kernel, "static", scene, rec, lig, b, stream)
        stream.synchronize()
        r = host(ref)
        assert_same(r, host(a))
        assert_same(r, host(b))
        scene.close()


def test_at_the_limit_without_allocating(kernel):
    """CC_STATIC_MAX_CONES cones (65,536 points x 2 lights) give cc_visibility's
    results, the device's free memory does not move across the calls, and one
    cone (or one point) more is rejected before any work."""
    import torch

    w = scenes.box_field(grid=256)
    lights = np.stack([w.lights[0], second_light()])
    scene = kernel.scene(w.meshes)
    rec = torch.from_numpy(w.receivers).cuda()
    lig = torch.from_numpy(lights).cuda()
    n = rec.shape[0] * lig.shape[0]
    assert n == _lib.CC_STATIC_MAX_CONES
    stream = torch.cuda.Stream()
    ref, a, b = device_outputs(torch, n), device_outputs(torch, n), device_outputs(torch, n)
    with torch.cuda.stream(stream):
        run(kernel, "device", scene, rec, lig, ref, stream)
        run(kernel, "static", scene, rec[:64], lig[:1], a, stream)  # first call on the device: setup
    stream.synchronize()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    with torch.cuda.stream(stream):
        run(kernel, "static", scene, rec, lig, a, stream)
        run(kernel, "static", scene, rec, lig, b, stream)
    stream.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    r = host(ref)
    assert_same(r, host(a))
    assert_same(r, host(b))

    three = torch.cat([lig, lig[:1]])
    more = torch.cat([rec, rec, rec[:1]])
    for rr, ll in ((rec, three), (more, lig[:1])):
        with pytest.raises(_lib.CCError) as e:
            run(kernel, "static", scene, rr, ll, a, stream)
        assert e.value.code == _lib.CC_ERR_INVALID
    scene.close()
