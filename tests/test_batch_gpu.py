"""The batched form (cc_batch_*) on a B200: every job's results equal the
plain call's for that job alone, on the first (direct) submission, on graph
replays, and under every configuration the autotuner tries."""
import numpy as np
import pytest

from continuum_b200 import Batch, _lib, scenes

pytestmark = pytest.mark.gpu

KEYS = ("full", "any", "partial", "irradiance", "fraction", "work")


def outputs(torch, n):
    dev = torch.device("cuda:0")
    return {"full": torch.zeros(n, dtype=torch.int64, device=dev), "any": torch.zeros(n, dtype=torch.int64, device=dev),
            "partial": torch.zeros(n, 64, device=dev), "irradiance": torch.zeros(n, device=dev),
            "fraction": torch.zeros(n, device=dev), "work": torch.zeros(n, 4, dtype=torch.int32, device=dev)}


def ptrs(outs):
    return {k: v.data_ptr() for k, v in outs.items()}


def host(outs):
    return {k: v.cpu().numpy().copy() for k, v in outs.items()}


def same(a, b, keys=KEYS):
    for k in keys:
        assert np.array_equal(a[k], b[k]), k


class Jobs:
    """Uneven jobs: different scenes, point and light counts, an empty job,
    a job with another hierarchy mode, and a scene shared by two jobs."""

    def __init__(self, kernel, torch):
        ico_a = scenes.icosphere_field(seed=5, n_spheres=12, subdivisions=4, width=160, height=90)
        ico_b = scenes.icosphere_field(seed=8, n_spheres=6, subdivisions=3, width=64, height=36)
        box = scenes.box_field(grid=64)
        self.scenes = [kernel.scene(w.meshes) for w in (ico_a, ico_b, box)]
        specs = [(0, ico_a.receivers, ico_a.lights, 2), (1, ico_b.receivers, ico_b.lights[:1], 2),
                 (2, box.receivers, box.lights, 1), (2, box.receivers[:0], box.lights, 2),
                 (0, ico_a.receivers[::7], ico_a.lights[1:3], 2)]
        self.jobs = []
        for si, rec, lig, h in specs:
            r = torch.from_numpy(np.ascontiguousarray(rec)).cuda()
            l = torch.from_numpy(np.ascontiguousarray(lig)).cuda()
            n = r.shape[0] * l.shape[0]
            self.jobs.append((self.scenes[si], r, l, h, outputs(torch, max(n, 1))))

    def alone(self, kernel, stream):
        import torch

        res = []
        for scene, r, l, h, outs in self.jobs:
            ref = {k: torch.zeros_like(v) for k, v in outs.items()}
            kernel.visibility_device(scene, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], ptrs(ref),
                                     stream=stream.cuda_stream, hierarchy=h)
            res.append(ref)
        stream.synchronize()
        return [host(x) for x in res]

    def batch(self, kernel):
        b = Batch(kernel)
        for scene, r, l, h, outs in self.jobs:
            b.add(scene, r.data_ptr(), r.shape[0], l.data_ptr(), l.shape[0], ptrs(outs), hierarchy=h)
        return b

    def check(self, alone, keys=KEYS):
        for (_, r, l, _, outs), ref in zip(self.jobs, alone):
            n = r.shape[0] * l.shape[0]
            same({k: v[:n] for k, v in host(outs).items()}, {k: v[:n] for k, v in ref.items()}, keys)

    def zero(self):
        for *_, outs in self.jobs:
            for v in outs.values():
                v.zero_()

    def close(self):
        for s in self.scenes:
            s.close()


def test_batch_equals_each_job_alone_and_graph_replays(kernel):
    import torch

    stream = torch.cuda.Stream()
    jobs = Jobs(kernel, torch)
    alone = jobs.alone(kernel, stream)
    b = jobs.batch(kernel)
    sizes = b.sizes()
    assert sizes["jobs"] == 5
    assert sizes["cones"] == sum(r.shape[0] * l.shape[0] for _, r, l, _, _ in jobs.jobs)
    for submission in range(3):  # direct + capture, then two graph replays
        jobs.zero()
        torch.cuda.synchronize()
        b.submit(stream=stream.cuda_stream)
        b.wait()
        jobs.check(alone)
    b.close()
    jobs.close()


def test_every_tuned_configuration_gives_the_same_results(kernel):
    import torch

    stream = torch.cuda.Stream()
    jobs = Jobs(kernel, torch)
    alone = jobs.alone(kernel, stream)
    b = jobs.batch(kernel)
    best, ms = b.tune(reps=1)
    assert len(ms) == 12 and np.all(ms > 0)
    assert best.points_per_warp in (8, 16, 32) and best.blocks_per_sm in (4, 8)
    assert best.flags & _lib.CC_BATCH_GRAPH
    for opt in (best, Batch.options(1, 1, 0), Batch.options(32, 5, _lib.CC_KEEP_ORDER)):
        jobs.zero()
        torch.cuda.synchronize()
        b.submit(opt, stream=stream.cuda_stream)
        b.wait()
        # Work counters depend on which cones share a packet; the results do not.
        jobs.check(alone, KEYS[:5])
    b.close()
    jobs.close()


def test_small_split_chunks_give_the_same_results(kernel):
    """A batch split into chunks of whole packets that end inside jobs (and
    jobs spread over several chunks) gives every job's results alone."""
    import torch

    stream = torch.cuda.Stream()
    jobs = Jobs(kernel, torch)
    alone = jobs.alone(kernel, stream)
    b = jobs.batch(kernel)
    try:
        for chunk in (1000, 20000):
            kernel.set_split_chunk(chunk)
            for opt in (Batch.options(32, 5, _lib.CC_BATCH_GRAPH), Batch.options(8, 3, 0)):
                jobs.zero()
                torch.cuda.synchronize()
                b.submit(opt, stream=stream.cuda_stream)
                b.wait()
                jobs.check(alone, KEYS[:5])
    finally:
        kernel.set_split_chunk(1 << 25)
        b.close()
        jobs.close()


def test_batch_rejects_bad_jobs_and_options(kernel):
    import torch

    w = scenes.box_field(grid=16)
    scene = kernel.scene(w.meshes)
    r = torch.from_numpy(w.receivers).cuda()
    l = torch.from_numpy(w.lights).cuda()
    outs = outputs(torch, r.shape[0])
    b = Batch(kernel)
    with pytest.raises(_lib.CCError) as e:
        b.add(scene, r.data_ptr() + 4, r.shape[0], l.data_ptr(), 1, ptrs(outs))
    assert e.value.code == _lib.CC_ERR_INVALID
    b.add(scene, r.data_ptr(), r.shape[0], l.data_ptr(), 1, ptrs(outs))
    for bad in (Batch.options(0, 4), Batch.options(33, 4), Batch.options(32, 9), Batch.options(32, 4, 1 << 10)):
        with pytest.raises(_lib.CCError) as e:
            b.submit(bad)
        assert e.value.code == _lib.CC_ERR_INVALID
    b.submit()
    b.wait()
    b.clear()
    assert b.sizes()["jobs"] == 0
    b.submit()  # an empty batch is no work
    b.wait()
    b.close()
    scene.close()
