"""bench.py's derived fields, checked on CPU with synthetic kernel times and traversal counts:
the roofline's algorithmic bytes follow the traversal model (32 B ray + 8 B hit + 80 B per node +
48 B per triangle for a closest-hit ray, 48 B + the same per node and triangle for a shadow ray),
the merged traversal launch counts both queues, and the fraction is achieved / peak."""

import bench


def _counts(rays, shadow, nodes, tris, s_nodes, s_tris):
    return {"rays": rays, "shadow_rays": shadow, "nodes_closest": nodes * rays, "tris_closest": tris * rays,
            "nodes_any": s_nodes * shadow, "tris_any": s_tris * shadow}


def test_roofline_of_merged_trace_launch():
    kernel_ms = {"prepare_ms": 1.0, "regen_ms": 2.0, "extend_ms": 100.0, "shade_ms": 30.0, "shadow_ms": 0.5}
    c = _counts(1e6, 5e5, 7.0, 4.0, 5.0, 3.0)
    r = bench.roofline_of(kernel_ms, 1e6, 5e5, 10, c)
    closest = 40.0 + 80.0 * 7.0 + 48.0 * 4.0
    shadow = 48.0 + 80.0 * 5.0 + 48.0 * 3.0
    assert r["kernel"] == "trace (closest + any hit)"
    assert abs(r["achieved"] - (closest * 1e6 + shadow * 5e5) / 0.1 / 1e9) < 1e-9
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert abs(r["algorithmic_bytes_per_launch"] - (closest * 1e6 + shadow * 5e5) / 10) < 1e-6
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"


def test_roofline_of_separate_launches_and_shade():
    c = _counts(1e6, 5e5, 7.0, 4.0, 5.0, 3.0)
    split = bench.roofline_of({"prepare_ms": 1, "regen_ms": 1, "extend_ms": 50, "shade_ms": 20, "shadow_ms": 30},
                              1e6, 5e5, 10, c)
    assert split["kernel"] == "extend (closest hit)"
    shade = bench.roofline_of({"prepare_ms": 1, "regen_ms": 1, "extend_ms": 10, "shade_ms": 40, "shadow_ms": 5},
                              1e6, 5e5, 10, c)
    assert shade["kernel"] == "shade"
    assert abs(shade["achieved"] - 328 * 1e6 / 0.04 / 1e9) < 1e-9
