"""Area-light NEE with MIS (an option of the screen tracer, not in the
reference) estimates the same image as the reference's BSDF-only path
tracer: checked on the FP64 oracle (CPU), Cornell box, 5 path vertices."""

import numpy as np


def _table(node):
    import nan_b200.scene as sc

    stand_in = type("S", (), {})()
    stand_in.scene_node = node
    return sc.Scene.area_light_table(stand_in)


def test_area_nee_is_unbiased_against_bsdf_sampling():
    from nan_b200 import scenes
    from nan_b200.scene import Lighting
    from oracle.oracle import F64, OracleScene

    node = scenes.cornell_box(8, 8)
    orc = OracleScene(**node.pack())
    table, power = _table(node)
    assert table.shape[0] == 2 and abs(float(table[:, 7].sum()) - 0.25) < 1e-6 and table[-1, 3] == 1.0
    orc.set_area_lights(table, power)
    w = h = 8
    px = np.stack(np.meshgrid(np.arange(w), np.arange(h), indexing="xy"), -1).reshape(-1, 2)
    stats = {}
    for area, frames in ((False, 4096), (True, 1024)):
        light = Lighting(sun_intensity=0.0, sky_radiance=(0, 0, 0), sun_disk=False, area_nee=area)
        acc = np.zeros((w * h, 3))
        acc2 = np.zeros((w * h, 3))
        for f in range(frames):
            node.camera.begin_frame(w, h)
            r, _ = orc.trace_screen(light, node.camera, w, h, f + (500000 if area else 0), 5, px, precision=F64)
            acc += r[:, :3]
            acc2 += r[:, :3] ** 2
        m = acc / frames
        stats[area] = (m, acc2 / frames - m * m, frames)
    (mp, vp, fp), (ma, va, fa) = stats[False], stats[True]
    z = (ma - mp) / np.sqrt(va / fa + vp / fp + 1e-12)
    print("image means", mp.mean(0), ma.mean(0), "variance per sample", vp.mean(), va.mean(), "z", z.mean(), z.std())
    assert np.all(np.abs(ma.mean(0) - mp.mean(0)) <= 0.02 * mp.mean(0))
    assert abs(z.mean()) < 0.3 and z.std() < 1.5
    assert va.mean() < vp.mean()
