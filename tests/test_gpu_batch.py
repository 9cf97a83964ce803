"""Multi-scene probe batches: one persistent launch over the probe sets of
several scenes of uneven size equals baking each scene on its own, bit for
bit. That holds for direct frames, for frames replayed from the captured CUDA
graph, and after the autotuner has changed the launch shape; and the same
for the multi-scene wavefront mode."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _probe_set(device, node, count, seed, compensated=False):
    import nan_b200
    from nan_b200 import scenes

    scene = nan_b200.Scene(device, node)
    probes, pinst = scenes.surface_sites(node, count, seed=seed, radius=0.2)
    layout = type("L", (), {})()
    layout.probes, layout.instance_gpu_data = probes, pinst
    layout.nodes = np.zeros((1, 4), np.uint32)
    layout.triangle_vertex_probes = np.zeros((1, 4), np.uint32)
    layout.total_probe_count = probes.shape[0]
    layout.instance_infos = list(range(pinst.shape[0]))
    geometry = nan_b200.SurfaceProbeGpuGeometry.create(device, layout)
    baker = nan_b200.SurfaceProbeDiffuseIrradianceBaker(device, scene, geometry, samples_per_probe=4,
                                                        compensated=compensated)
    return scene, baker


def _buffers(device, baker):
    import nan_b200

    rt = nan_b200.SurfaceProbeRuntimeBuffers.acquire(nan_b200.RenderData(device), baker.geometry.probe_count)
    return rt.field, rt.attachments


def _snapshot(field, attachments, baker):
    out = [field.values.cpu().numpy().copy(), field.sample_counts.cpu().numpy().copy(),
           attachments.self_hit_counts.cpu().numpy().copy(), attachments.radial_moments.cpu().numpy().copy()]
    if baker.compensation is not None:
        out.append(baker.compensation.cpu().numpy().copy())
    return out


@pytest.fixture(scope="module")
def sets(device):
    from nan_b200 import scenes

    items = [
        _probe_set(device, scenes.cornell_box(32, 32), 300, seed=3),
        _probe_set(device, scenes.terrain_boxes(seed=2, grid=65, boxes=30), 1000, seed=4, compensated=True),
        _probe_set(device, scenes.terrain_boxes(seed=3, grid=97, boxes=60), 517, seed=5),
    ]
    for scene, _ in items:
        scene.configure("megakernel")
    return items


def _reference(device, sets, frames):
    refs = []
    for scene, baker in sets:
        field, att = _buffers(device, baker)
        if baker.compensation is not None:
            baker.compensation.zero_()
        for it in range(frames):
            baker.execute(None, field, att, it, reset=(it == 0))
        refs.append(_snapshot(field, att, baker))
    return refs


def _bake_batch(device, sets, run, **mode):
    import nan_b200

    bufs = [_buffers(device, b) for _, b in sets]
    for _, b in sets:
        if b.compensation is not None:
            b.compensation.zero_()
    batch = nan_b200.ProbeBatch(device, [(b, f, a) for (_, b), (f, a) in zip(sets, bufs)], **mode)
    run(batch)
    return batch, [_snapshot(f, a, b) for (_, b), (f, a) in zip(sets, bufs)]


def test_batch_equals_per_scene_bakes(device, sets):
    refs = _reference(device, sets, 3)

    def run(batch):
        # double-sided walls carry a back record per site as well
        assert batch.info()["total_probes"] == sum(int(b.geometry.probe_count) for _, b in sets)
        for it in range(3):
            batch.execute(None, it, 4, 3, reset=(it == 0))

    _, got = _bake_batch(device, sets, run)
    for g, ref in zip(got, refs):
        for a, b in zip(g, ref):
            np.testing.assert_array_equal(a, b)
    device.check()


def test_batch_graph_replay_and_autotune(device, sets):
    from nan_b200._native import NanError

    refs = _reference(device, sets, 3)
    state = {}

    def run(batch):
        tuned = batch.autotune(4, 3)
        print("autotune", tuned, batch.info())
        assert tuned["stack_depth"] >= batch.info()["min_stack_depth"] and tuned["frame_ms"] > 0.0
        for _, b in sets:
            if b.compensation is not None:
                b.compensation.zero_()
        batch.capture(0, True, 4, 3)
        batch.replay(3)
        state["batch"] = batch

    batch, got = _bake_batch(device, sets, run)
    for g, ref in zip(got, refs):
        for a, b in zip(g, ref):
            np.testing.assert_array_equal(a, b)
    # a shallower stack than the BVHs need is refused
    with pytest.raises(NanError):
        batch.set_tuning(16, 4, 1)
    device.check()


def test_batch_independent_samples_match_oracle(device):
    """Independent-sample mode (one RNG stream per sample, a warp per probe)
    against the oracle's same mode, over two scenes and three iterations:
    >= 99.9 % of probes exact, sample counts equal."""
    import nan_b200
    from nan_b200 import scenes
    from oracle.oracle import OracleScene

    sets = [_probe_set(device, scenes.cornell_box(32, 32), 300, seed=7),
            _probe_set(device, scenes.terrain_boxes(seed=3, grid=97, boxes=60), 700, seed=8)]
    spp = 40  # more than one warp of samples per probe
    bufs = [_buffers(device, b) for _, b in sets]
    batch = nan_b200.ProbeBatch(device, [(b, f, a) for (_, b), (f, a) in zip(sets, bufs)], independent_samples=True)
    for it in range(3):
        batch.execute(None, it, spp, 3, reset=(it == 0))
    for (scene, baker), (field, att) in zip(sets, bufs):
        orc = OracleScene(**scene.host)
        n = int(baker.geometry.probe_count)
        probes = baker.geometry.probes.cpu().numpy().view(np.uint8).reshape(n, 48)
        pinst = baker.geometry.instances.cpu().numpy().view(np.uint8).reshape(-1, 48)
        values = np.zeros((n, 3), np.float32)
        counts = np.zeros(n, np.uint32)
        self_hits = np.zeros(n, np.uint32)
        radial = np.zeros((n, 16), np.uint32)
        units = np.arange(n, dtype=np.uint32)
        for it in range(3):
            orc.trace_probes(scene.lighting, values, counts, self_hits, radial, probes, pinst, units, it, spp, 3,
                             it == 0, independent_samples=True)
        g_values = field.values.cpu().numpy().view(np.float32).reshape(n, 3)
        g_counts = field.sample_counts.cpu().numpy().view(np.uint32)
        g_self = att.self_hit_counts.cpu().numpy().view(np.uint32)
        g_radial = att.radial_moments.cpu().numpy().view(np.uint32).reshape(n, 16)
        np.testing.assert_array_equal(g_counts, counts)
        exact = np.all(g_values == values, axis=1) & (g_self == self_hits) & np.all(g_radial == radial, axis=1)
        print("independent samples vs oracle exact", exact.mean())
        assert exact.mean() >= 0.999, exact.mean()
    device.check()


def test_batch_wavefront_equals_per_scene_bakes(device, sets):
    """The multi-scene wavefront (every probe of every scene a path in
    flight) keeps the reference's sample sequence: direct frames, autotuned
    and graph-replayed frames equal the per-scene bakes bit for bit."""
    refs = _reference(device, sets, 3)

    def direct(batch):
        for it in range(3):
            batch.execute(None, it, 4, 3, reset=(it == 0))

    _, got = _bake_batch(device, sets, direct, wavefront=True)
    for g, ref in zip(got, refs):
        for a, b in zip(g, ref):
            np.testing.assert_array_equal(a, b)

    def tuned_graph(batch):
        tuned = batch.autotune(4, 3)
        print("wavefront autotune", tuned)
        for _, b in sets:
            if b.compensation is not None:
                b.compensation.zero_()
        batch.capture(0, True, 4, 3)
        batch.replay(3)

    _, got = _bake_batch(device, sets, tuned_graph, wavefront=True)
    for g, ref in zip(got, refs):
        for a, b in zip(g, ref):
            np.testing.assert_array_equal(a, b)
    device.check()


def test_batch_wavefront_independent_equals_persistent_independent(device):
    """Independent samples on the wavefront (one path per probe and sample,
    samples folded in order afterwards) equal the persistent independent
    kernel bit for bit; with 2 spp x 3 bounces and 70 spp (more than one warp
    of samples per probe)."""
    import nan_b200
    from nan_b200 import scenes

    sets = [_probe_set(device, scenes.cornell_box(32, 32), 300, seed=7),
            _probe_set(device, scenes.terrain_boxes(seed=3, grid=97, boxes=60), 700, seed=8, compensated=True)]
    for spp in (2, 70):
        results = []
        for wavefront in (False, True):
            bufs = [_buffers(device, b) for _, b in sets]
            for _, b in sets:
                if b.compensation is not None:
                    b.compensation.zero_()
            batch = nan_b200.ProbeBatch(device, [(b, f, a) for (_, b), (f, a) in zip(sets, bufs)],
                                        independent_samples=True, wavefront=wavefront)
            for it in range(3):
                batch.execute(None, it, spp, 3, reset=(it == 0))
            results.append([_snapshot(f, a, b) for (_, b), (f, a) in zip(sets, bufs)])
            batch.close()
        for g, ref in zip(*results):
            for a, b in zip(g, ref):
                np.testing.assert_array_equal(a, b)
    device.check()
