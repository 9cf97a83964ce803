"""Surface-probe baking of many scenes in one persistent launch (no
counterpart in the reference, which dispatches once per scene:
surface_probe_path_tracer.py:49-83).

    batch = ProbeBatch(device, [(baker, field, attachments), ...])
    batch.autotune(samples_per_probe=64, max_bounces=3)     # picks the launch shape
    batch.execute(stream, iteration, 64, 3, reset=(iteration == 0))
    # or: batch.capture(0, True, 64, 3); batch.replay(frames)   (CUDA graph)

Each item is a SurfaceProbeDiffuseIrradianceBaker with the field and
attachments it would be executed with; the results equal those of
baker.execute(...) per scene, bit for bit. With independent_samples=True
each sample of a probe draws from its own RNG stream and a warp traces 32
samples of one probe at once (a different, equally valid sample set). With
wavefront=True the reference's sample sequence runs as one multi-scene
wavefront: every probe of every scene is a path in flight and each
extend / shade / shadow / finalize round covers all scenes (results equal
the per-scene bakes bit for bit); with both flags every (probe, sample) is
a path and the samples are folded in order afterwards (results equal the
independent-sample persistent kernel's).
"""

from __future__ import annotations

import ctypes

from ._native import NanBatchTuning, NanProbeSet, check, lib, ptr, stream_handle


class ProbeBatch:
    def __init__(self, device, items, *, independent_samples: bool = False, wavefront: bool = False):

        self.device = device
        self._keep = []
        sets = (NanProbeSet * max(len(items), 1))()
        for i, (baker, field, attachments) in enumerate(items):
            g = baker.geometry
            s = sets[i]
            s.scene = baker.scene.context.handle
            s.probes = ptr(g.probes)
            s.probe_count = int(g.probe_count)
            s.probe_instances = ptr(g.instances)
            s.probe_instance_count = int(g.instance_count)
            s.values = ptr(field.values)
            s.sample_counts = ptr(field.sample_counts)
            s.self_hits = ptr(attachments.self_hit_counts)
            s.radial = ptr(attachments.radial_moments)
            s.compensation = ptr(baker.compensation)
            s.lighting = baker.scene.lighting.to_struct()
            self._keep.append((baker, field, attachments))
        self._context = device.new_context()
        handle = ctypes.c_void_p()
        check(lib().nan_batch_create(self._context.handle, sets, len(items), ctypes.byref(handle)))
        self.handle = handle
        mode = (3 if wavefront else 1) if independent_samples else (2 if wavefront else 0)
        if mode:
            check(lib().nan_batch_set_mode(self.handle, mode))

    @property
    def context(self):
        return self._context

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().nan_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        depth, total = ctypes.c_uint32(), ctypes.c_uint32()
        t = NanBatchTuning()
        check(lib().nan_batch_info(self.handle, ctypes.byref(depth), ctypes.byref(total), ctypes.byref(t)))
        return {"min_stack_depth": depth.value, "total_probes": total.value, "stack_depth": t.stack_depth,
                "blocks_per_sm": t.blocks_per_sm, "units_per_grab": t.units_per_grab,
                "min_blocks_per_sm": t.min_blocks_per_sm}

    def set_tuning(self, stack_depth: int, blocks_per_sm: int, units_per_grab: int, min_blocks_per_sm: int = 0) -> None:
        t = NanBatchTuning()
        t.stack_depth, t.blocks_per_sm, t.units_per_grab = int(stack_depth), int(blocks_per_sm), int(units_per_grab)
        t.min_blocks_per_sm = int(min_blocks_per_sm)
        check(lib().nan_batch_set_tuning(self.handle, ctypes.byref(t)))

    def autotune(self, samples_per_probe: int, max_bounces: int = 3, stream=None) -> dict:
        t = NanBatchTuning()
        ms = ctypes.c_float()
        check(lib().nan_batch_autotune(self.handle, int(samples_per_probe), int(max_bounces), stream_handle(stream),
                                       ctypes.byref(t), ctypes.byref(ms)))
        return {"stack_depth": t.stack_depth, "blocks_per_sm": t.blocks_per_sm, "units_per_grab": t.units_per_grab,
                "min_blocks_per_sm": t.min_blocks_per_sm, "frame_ms": ms.value}

    def execute(self, command_encoder, iteration: int, samples_per_probe: int, max_bounces: int = 3, *,
                reset: bool = False) -> None:
        check(lib().nan_batch_trace_probes(self.handle, int(iteration) & 0xFFFFFFFF, int(samples_per_probe),
                                           int(max_bounces), int(bool(reset)), stream_handle(command_encoder)))

    def capture(self, first_iteration: int, reset_first: bool, samples_per_probe: int, max_bounces: int = 3,
                stream=None) -> None:
        check(lib().nan_batch_capture(self.handle, int(first_iteration) & 0xFFFFFFFF, int(bool(reset_first)),
                                      int(samples_per_probe), int(max_bounces), stream_handle(stream)))

    def replay(self, frames: int = 1, stream=None) -> None:
        check(lib().nan_batch_replay(self.handle, int(frames), stream_handle(stream)))
