"""The benchmark's CPU legs, without a GPU: the oracle's camera pass gives the
library's receivers bit for bit (so the reference arm can build its inputs
alone), the reference arm loads nothing of the library, and the reference
CPU path's BVH gives the same results as its brute-force form."""
import subprocess
import sys
from pathlib import Path

import numpy as np

from continuum_b200 import scenes
from oracle.oracle import OracleScene

ROOT = Path(__file__).resolve().parent.parent


def test_oracle_camera_pass_equals_the_library_caster():
    w = scenes.icosphere_field(seed=3, n_spheres=16, subdivisions=3, width=200, height=120, with_receivers=False)
    lib = scenes.primary_hits(w, 200, 120)
    osc = OracleScene(w.meshes)
    rec, hit = osc.primary_hits(w.camera, 200, 120)
    osc.close()
    assert np.array_equal(lib.view(np.uint32), rec[hit.astype(bool)].view(np.uint32))
    assert lib.shape[0] > 1000


def test_oracle_camera_pass_equals_the_library_caster_instanced():
    world = scenes.instanced_world(seed=3, n_instances=300, n_boulders=3, half=40.0, n_lights=2, width=96, height=54,
                                   segments=24, rings=13)
    osc = OracleScene.instanced(world.geometries, world.instances)
    rec, hit = osc.primary_hits(world.camera, 96, 54)
    osc.close()
    assert np.array_equal(world.receivers.view(np.uint32), rec[hit.astype(bool)].view(np.uint32))


def test_cpu_path_bvh_equals_brute_force():
    w = scenes.box_field(grid=32)
    osc = OracleScene(w.meshes)
    L = w.lights[0]
    l9 = np.concatenate([L[0:3], L[4:7], L[8:11]])
    bvh = osc.cpu_bvh()
    a, ta = osc.cpu_masked_with(bvh, w.receivers, l9, threads=2)
    b, tb = osc.cpu_masked_with(None, w.receivers, l9, threads=1)
    c, tc = osc.cpu_masked(w.receivers, l9, use_bvh=True)
    bvh.close()
    osc.close()
    assert np.array_equal(ta, tb)
    assert np.max(np.abs(a - b) / tb) <= 2.5e-6  # M1 gate 2's hierarchy = brute force bound
    assert np.array_equal(a, c)


def test_reference_arm_loads_no_library():
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--reference-seconds', "
        "'0.2', '--cpu-path-points', '256']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LIBRARY', 'libcontinuum_cuda' in maps, 'ORACLE', 'libcone_oracle' in maps)\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert "LIBRARY False ORACLE True" in out.stdout, out.stdout
    import json

    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][0])
    assert line["impl"] == "reference" and line["unit"] == "cones/s" and line["value"] > 0
    assert line["cpu_path"]["threads_1"]["value"] > 0 and line["cpu_path"]["bvh_build_ms"] > 0
