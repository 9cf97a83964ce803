"""Host-side logic and the C-ABI surface (no GPU needed).

Covers the reference's CPU-only tests for the parts of the path that live on
the host -- the Mesh Colors layout (test_mesh_colors.py:16-163), the probe
field strides and runtime buffers (test_surface_probe_fields.py:39-86) -- and
checks that libnan_b200.so loads and exports every entry point declared in
include/nan_b200.h. No kernel is launched.
"""

import ctypes
import re
import types
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


# ---- C ABI ------------------------------------------------------------------

def _declared_functions():
    text = (ROOT / "include" / "nan_b200.h").read_text()
    return sorted(set(re.findall(r"NAN_B200_API\s+[\w\s\*]+?\b(nan_\w+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    from nan_b200 import _native

    declared = _declared_functions()
    assert len(declared) >= 20
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing
    # and the binding declares a prototype for each of them
    assert sorted(_native.EXPORTS) == declared


def test_binding_loads_and_reports_version():
    from nan_b200 import _native

    assert _native.lib().nan_version() >= 1
    assert _native.lib().nan_wavefront_bytes_per_path() > 0


def test_struct_layouts_match_header():
    from nan_b200 import _native

    assert ctypes.sizeof(_native.NanLighting) == 96
    assert ctypes.sizeof(_native.NanCamera) == 64
    assert ctypes.sizeof(_native.NanCounters) == 32
    assert ctypes.sizeof(_native.NanTuning) == 32
    assert ctypes.sizeof(_native.NanKernelTimes) == 48
    assert ctypes.sizeof(_native.NanCacheConfig) == 72
    assert ctypes.sizeof(_native.NanCachedFrame) == 64
    assert ctypes.sizeof(_native.NanProbeSet) == 176
    assert ctypes.sizeof(_native.NanBatchTuning) == 16


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """sizeof and every field offset of the ABI structs, as gcc lays them out
    from include/nan_b200.h, equal the ctypes mirrors."""
    import shutil
    import subprocess

    from nan_b200 import _native

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    structs = ["NanLighting", "NanCamera", "NanCounters", "NanTuning", "NanKernelTimes", "NanCacheConfig",
               "NanCachedFrame", "NanProbeSet", "NanBatchTuning", "NanProbeLayoutDesc", "NanProbeResolveOptions",
               "NanWseOptions", "NanSceneDesc", "NanMeshColorsDesc", "NanSceneInfo"]
    structs = [s for s in structs if hasattr(_native, s)]
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "nan_b200.h"', "int main(void) {"]
    expect = []
    for name in structs:
        cls = getattr(_native, name)
        lines.append(f'printf("%zu\\n", sizeof({name}));')
        expect.append(ctypes.sizeof(cls))
        for field, *_ in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({name}, {field}));')
            expect.append(getattr(cls, field).offset)
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    include = Path(_native.__file__).resolve().parents[1] / "include"
    subprocess.run(["gcc", "-std=c11", "-I", str(include), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect


def test_null_arguments_are_rejected_without_a_device():
    from nan_b200 import _native

    lib = _native.lib()
    assert lib.nan_ctx_create(0, None) == _native.NAN_ERR_INVALID_ARGUMENT
    assert b"null" in lib.nan_last_error()
    assert lib.nan_ctx_configure(None, None) == _native.NAN_ERR_INVALID_ARGUMENT


def test_product_package_does_not_import_the_oracle():
    for path in (ROOT / "nan_b200").rglob("*.py"):
        text = path.read_text()
        assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\w+)", text, re.M), path


# ---- Mesh Colors layout (mesh_colors.py:147-297) ------------------------------

def test_layout_address_round_trip():
    from nan_b200.mesh_colors import address_to_ij, barycentric_at, colors_per_patch, ij_to_address

    for resolution in (1, 2, 4, 8, 16):
        for address in range(colors_per_patch(resolution)):
            i, j = address_to_ij(address, resolution)
            assert ij_to_address(i, j, resolution) == address
            b = barycentric_at(i, j, resolution)
            assert abs(sum(b) - 1.0) < 1e-12 and min(b) >= 0.0


def test_layout_demo_counts_and_budget():
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED, MeshColorsLayout

    demo = scenes.reference_demo()
    layout = MeshColorsLayout.build(demo, texels_per_unit=1.0, min_resolution=2, max_resolution=2,
                                    max_total_texels=276)
    assert layout.total_surface_texels == 216
    assert layout.total_payload_count == 276
    two_sided = sum(int(i.texel_count) for i, s in zip(layout.instance_infos, layout.side_infos)
                    if s.flags & MESH_COLORS_SIDE_FLAG_DOUBLE_SIDED)
    assert two_sided == 60
    with pytest.raises(ValueError, match="texel budget exceeded"):
        MeshColorsLayout.build(demo, texels_per_unit=1.0, min_resolution=2, max_resolution=2, max_total_texels=275)
    with pytest.raises(ValueError, match="texel budget exceeded"):
        MeshColorsLayout.build(demo, min_resolution=4, max_resolution=4, max_total_texels=1)


def test_layout_offsets_are_contiguous():
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MESH_COLORS_INVALID_OFFSET, MeshColorsLayout, colors_per_patch

    demo = scenes.reference_demo()
    layout = MeshColorsLayout.build(demo, texels_per_unit=64.0, min_resolution=2, max_resolution=8,
                                    max_total_texels=100_000)
    expected = 0
    ranges = []
    for inst, side in zip(layout.instance_infos, layout.side_infos):
        assert inst.texel_offset == expected
        local = 0
        for f in range(inst.face_count):
            face = layout.face_infos[inst.face_offset + f]
            assert face.address == local and 2 <= face.resolution <= 8
            local += colors_per_patch(face.resolution)
        assert inst.texel_count == local
        ranges.append((inst.texel_offset, inst.texel_offset + local))
        if side.is_double_sided:
            assert side.back_texel_offset == inst.texel_offset + local
            ranges.append((side.back_texel_offset, side.back_texel_offset + local))
            expected += 2 * local
        else:
            assert side.back_texel_offset == MESH_COLORS_INVALID_OFFSET
            expected += local
    for a, b in zip(ranges, ranges[1:]):
        assert a[1] == b[0]
    assert expected == layout.total_payload_count
    assert layout.surface_prefix[-1] == layout.total_surface_texels


def test_layout_resolution_limits_normalize_inward():
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout

    layout = MeshColorsLayout.build(scenes.reference_demo(), min_resolution=3, max_resolution=7,
                                    max_total_texels=100_000)
    assert layout.min_resolution == 4 and layout.max_resolution == 4
    with pytest.raises(ValueError, match="min_resolution"):
        MeshColorsLayout.build(scenes.reference_demo(), min_resolution=5, max_resolution=7)


def test_greedy_halving_gives_early_triangles_full_resolution():
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout, colors_per_patch

    demo = scenes.reference_demo()
    full = MeshColorsLayout.build(demo, texels_per_unit=64.0, min_resolution=2, max_resolution=8,
                                  max_total_texels=100_000)
    budget = full.total_payload_count - 30  # one R=8 patch (45) halved to R=4 (15)
    halved = MeshColorsLayout.build(demo, texels_per_unit=64.0, min_resolution=2, max_resolution=8,
                                    max_total_texels=budget)
    assert halved.total_payload_count <= budget
    r_full, r_half = full.face_array[:, 1], halved.face_array[:, 1]
    changed = np.nonzero(r_full != r_half)[0]
    assert changed.size > 0 and np.all(r_half[changed] < r_full[changed])
    assert np.all(r_half[: changed[0]] == r_full[: changed[0]])
    assert colors_per_patch(int(r_half[changed[0]])) < colors_per_patch(int(r_full[changed[0]]))


def test_bench_scene_layout_fits_budget_without_halving():
    from nan_b200 import scenes
    from nan_b200.mesh_colors import MeshColorsLayout

    node = scenes.terrain_boxes()
    assert node.triangle_count == 200_688
    layout = MeshColorsLayout.build(node)
    assert layout.total_payload_count <= 16_777_216
    r = layout.face_array[:, 1]
    assert r.min() >= 4 and r.max() <= 64


# ---- surface-probe fields (surface_probe_fields.py) ---------------------------

class _FakeRenderData:
    def __init__(self):
        self.requests = []

    def get_buffer(self, name, **kwargs):
        buffer = object()
        self.requests.append((name, kwargs, buffer))
        return buffer


class _FakeDevice:
    def __init__(self):
        self.requests = []

    def create_buffer(self, **kwargs):
        buffer = object()
        self.requests.append((kwargs, buffer))
        return buffer


def test_field_strides():
    from nan_b200.surface_probe_fields import DIFFUSE_IRRADIANCE_RGB_FIELD, DIFFUSE_PRT_L2_RGB_FIELD

    assert DIFFUSE_IRRADIANCE_RGB_FIELD.value_stride == 12
    assert DIFFUSE_IRRADIANCE_RGB_FIELD.bytes_per_probe == 16
    assert DIFFUSE_PRT_L2_RGB_FIELD.value_stride == 108
    assert DIFFUSE_PRT_L2_RGB_FIELD.bytes_per_probe == 112


def test_runtime_buffers_separate_values_counts_and_attachments():
    from nan_b200.surface_probe_fields import (DIFFUSE_IRRADIANCE_RGB_FIELD, DIFFUSE_PRT_ATTACHMENTS,
                                               DIFFUSE_PRT_L2_RGB_FIELD, SurfaceProbeRuntimeBuffers)

    rd = _FakeRenderData()
    runtime = SurfaceProbeRuntimeBuffers.acquire(rd, 7)
    requests = {name: kw for name, kw, _ in rd.requests}
    values = next(kw for name, kw in requests.items() if name.endswith(".values"))
    counts = requests["surface_probe_renderer.field.diffuse_irradiance_rgb.v1.sample_counts"]
    assert values["size"] == 7 * 12
    assert counts["struct_size"] == 4 and counts["element_count"] == 7
    assert runtime.field.desc is DIFFUSE_IRRADIANCE_RGB_FIELD
    assert runtime.field.values is not runtime.field.sample_counts
    assert len(rd.requests) == 4
    rd2 = _FakeRenderData()
    SurfaceProbeRuntimeBuffers.acquire(rd2, 11, field_desc=DIFFUSE_PRT_L2_RGB_FIELD,
                                       attachment_descs=DIFFUSE_PRT_ATTACHMENTS)
    assert len(rd2.requests) == 5


def test_invalid_field_shape_is_rejected():
    from nan_b200.surface_probe_fields import (SurfaceProbeFieldDesc, SurfaceProbeFieldSemantic,
                                               SurfaceProbeFieldStorage)

    with pytest.raises(ValueError):
        SurfaceProbeFieldDesc(SurfaceProbeFieldSemantic.DIFFUSE_PRT_L2_RGB, 0, 1, SurfaceProbeFieldStorage.FLOAT32)


def test_geometry_upload_contains_no_field_buffers():
    from nan_b200.surface_probe_resources import SurfaceProbeGpuGeometry

    layout = types.SimpleNamespace(
        probes=np.zeros((3, 48), np.uint8), nodes=np.zeros((2, 4), np.uint32),
        instance_gpu_data=np.zeros((1, 48), np.uint8), triangle_vertex_probes=np.zeros((4, 4), np.uint32),
        total_probe_count=3, instance_infos=(object(),))
    device = _FakeDevice()
    geometry = SurfaceProbeGpuGeometry.create(device, layout)
    labels = {kw["label"] for kw, _ in device.requests}
    assert geometry.probe_count == 3 and geometry.instance_count == 1
    assert labels == {"surface_probe_metadata", "surface_probe_nodes", "surface_probe_instances",
                      "surface_probe_triangle_vertex_map"}


def test_baker_rejects_wrong_field_before_any_launch():
    from nan_b200.surface_probe_fields import DIFFUSE_PRT_L2_RGB_FIELD, SurfaceProbeFieldBuffers
    from nan_b200.surface_probe_path_tracer import SurfaceProbeDiffuseIrradianceBaker

    baker = SurfaceProbeDiffuseIrradianceBaker.__new__(SurfaceProbeDiffuseIrradianceBaker)
    with pytest.raises(ValueError, match="diffuse irradiance"):
        baker.execute(None, SurfaceProbeFieldBuffers(DIFFUSE_PRT_L2_RGB_FIELD, None, None), None, 0)


# ---- camera host math (camera.py:4-96) -----------------------------------------

def test_halton_matches_reference(golden):
    from nan_b200.camera import halton

    got2 = np.asarray([halton(int(i), 2) for i in golden["halton_index"]])
    got3 = np.asarray([halton(int(i), 3) for i in golden["halton_index"]])
    np.testing.assert_array_equal(got2, golden["halton_base2"])
    np.testing.assert_array_equal(got3, golden["halton_base3"])


def test_camera_jitter_sequence_matches_reference(golden):
    """Camera.begin_frame's jitter over 40 frames (two cycles of the 16-point
    Halton(2,3) pattern) at four image sizes, bit for bit against the
    reference's camera.py:87-96 run on the same frames."""
    from nan_b200.camera import Camera

    for (w, h), expect in zip(golden["camera_sizes"], golden["camera_jitter"]):
        cam = Camera()
        got = np.zeros_like(expect)
        for f in range(expect.shape[0]):
            cam.begin_frame(int(w), int(h))
            got[f] = cam.jitter
        np.testing.assert_array_equal(got.view(np.uint32), expect.view(np.uint32))


def test_mesh_factories_match_reference(golden):
    """Vertex records (position, normal, uv; 32 B) and triangle order of the
    reference's mesh factories (mesh.py:31-189)."""
    from nan_b200.scene_node import Mesh

    made = {
        "cube_1": Mesh.cube((1.0, 1.0, 1.0)), "cube_a": Mesh.cube((0.6, 1.2, 0.6)),
        "cube_b": Mesh.cube((2.5, 0.3, 1.1)), "quad": Mesh.quad((2.0, 3.0)),
        "quad_yz_pos": Mesh.quad_yz((2.0, 3.0), True), "quad_yz_neg": Mesh.quad_yz((2.0, 3.0), False),
        "quad_xy_pos": Mesh.quad_xy((2.0, 3.0), True), "quad_xy_neg": Mesh.quad_xy((2.0, 3.0), False),
    }
    for key, m in made.items():
        np.testing.assert_array_equal(m.vertices, golden[f"mesh_{key}_vertices"], err_msg=key)
        np.testing.assert_array_equal(m.indices, golden[f"mesh_{key}_indices"], err_msg=key)


def test_descriptor_records_match_reference(golden):
    """SceneNode.pack's mesh and instance descriptors are the reference's
    16-byte MeshDesc / InstanceDesc records (scene.py:85-108): fields in the
    same order, one u32 each."""
    from nan_b200.scene_node import Material, Mesh, SceneNode, make_transform

    np.testing.assert_array_equal(golden["desc_mesh_packed"], golden["desc_mesh_fields"])
    np.testing.assert_array_equal(golden["desc_instance_packed"], golden["desc_instance_fields"])
    node = SceneNode()
    a = node.add_mesh(Mesh.cube((1.0, 1.0, 1.0)))
    b = node.add_mesh(Mesh.quad((2.0, 3.0)))
    mat = node.add_material(Material())
    node.add_instance(a, mat, node.add_transform(make_transform()))
    node.add_instance(b, mat, node.add_transform(make_transform(scaling=(-1.0, 1.0, 1.0))))
    packed = node.pack()
    np.testing.assert_array_equal(packed["mesh_descs"], [[24, 36, 0, 0], [4, 6, 24, 36]])
    np.testing.assert_array_equal(packed["instance_descs"], [[0, 0, 0, 0], [1, 0, 1, 1]])


def test_camera_basis_is_orthogonal_and_scaled():
    from nan_b200.camera import Camera

    cam = Camera()
    cam.position = np.array([0, 1, 3], np.float32)
    cam.target = np.array([0, 1, 0], np.float32)
    cam.fov = 60.0
    cam.width, cam.height = 200, 100
    cam.recompute()
    u, v, w = (x.astype(np.float64) for x in (cam.image_u, cam.image_v, cam.image_w))
    assert abs(np.dot(u, v)) < 1e-3 * np.linalg.norm(u) * np.linalg.norm(v)
    assert abs(np.linalg.norm(v) / np.linalg.norm(w) - np.tan(np.radians(30))) < 1e-5
    assert abs(np.linalg.norm(u) / np.linalg.norm(v) - 2.0) < 1e-5
