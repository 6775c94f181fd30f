"""The library loads without a GPU and exports every entry point the public headers declare."""

import os
import re

import pytest
from conftest import ROOT

import photon_gpu


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return set(re.findall(r"\b((?:pgpu|ph)[A-Za-z_0-9]*)\s*\(", text))


def test_library_exports_all_declared_symbols():
    lib = photon_gpu.load()
    names = _declared("photon_gpu.h") | _declared("ph_c_core.h")
    assert len(names) > 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_python_binding_declares_every_export():
    names = _declared("photon_gpu.h") | _declared("ph_c_core.h")
    bound = {n for n, _, _ in photon_gpu.PGPU_SIGNATURES} | {n for n, _, _ in photon_gpu.PH_SIGNATURES}
    assert names == bound, f"header-only {sorted(names - bound)}, binding-only {sorted(bound - names)}"


def test_calls_without_device_fail_loudly():
    # no compute call runs here; creating GPU objects without a device must fail with a status
    if photon_gpu.device_count() > 0:
        return
    import numpy as np
    try:
        photon_gpu.Geometry(np.zeros((1, 3, 3), np.float32) + np.eye(3, dtype=np.float32))
    except photon_gpu.PhotonGpuError as e:
        assert "no CUDA device" in str(e)
    else:
        raise AssertionError("geometry creation succeeded without a device")


def _create_status(tris, tri_mat, tri_em, mats, ems, cam, emitters_null=False):
    import ctypes

    import numpy as np

    lib = photon_gpu.load()
    sid = ctypes.c_uint64(0)

    def ptr(a, t):
        return a.ctypes.data_as(ctypes.POINTER(t))

    em_ptr = None if emitters_null else ptr(ems, ctypes.c_float)
    status = lib.pgpu_scene_create_ex(ptr(tris, ctypes.c_float), ptr(tri_mat, ctypes.c_uint32),
                                      ptr(tri_em, ctypes.c_uint32), tris.shape[0], ptr(mats, ctypes.c_float),
                                      mats.shape[0], em_ptr, ems.shape[0], ptr(cam, ctypes.c_float), 0,
                                      ctypes.byref(sid))
    assert sid.value == 0
    return status, lib.pgpu_last_error().decode()


@pytest.mark.parametrize("case, message", [
    ("width0", "resolution"), ("height_negative", "resolution"), ("width_nan", "resolution"),
    ("width_fraction", "resolution"), ("too_many_pixels", "resolution"), ("emitters_null", "missing input"),
    ("emitter_type", "unknown emitter type"), ("material_type", "unknown material type"),
    ("material_type_nan", "unknown material type"), ("material_index", "material index out of range"),
])
def test_scene_create_rejects_bad_input_before_device_work(case, message):
    # every check runs before the library touches a device, so these need no GPU
    import numpy as np

    import scenes

    tris, tri_mat, tri_em, mats, ems, cam = photon_gpu.flatten_scene(scenes.cornell(8, 8, 1))
    tris, tri_mat, tri_em, mats, ems, cam = (a.copy() for a in (tris, tri_mat, tri_em, mats, ems, cam))
    assert ems.shape[0] > 0
    emitters_null = False
    if case == "width0":
        cam[10] = 0
    elif case == "height_negative":
        cam[11] = -8
    elif case == "width_nan":
        cam[10] = np.nan
    elif case == "width_fraction":
        cam[10] = 8.5
    elif case == "too_many_pixels":
        cam[10], cam[11] = 65536, 65537
    elif case == "emitters_null":
        emitters_null = True
    elif case == "emitter_type":
        ems[0, 3] = 7
    elif case == "material_type":
        mats[0, 0] = 3
    elif case == "material_type_nan":
        mats[0, 0] = np.nan
    elif case == "material_index":
        tri_mat[0] = mats.shape[0]
    status, text = _create_status(tris, tri_mat, tri_em, mats, ems, cam, emitters_null)
    assert status == 1, (status, text)   # PG_ERR_INVALID_ARGUMENT
    assert message in text, text


def test_frames_load_and_save_pfm_without_a_device(tmp_path):
    # frames live on the host: phCreateFrame / phLoadFrame / phSaveFrame / phGetFrameRgbData
    import ctypes

    import numpy as np

    lib = photon_gpu.load()
    fid = ctypes.c_uint64(0)
    lib.phCreateFrame(ctypes.byref(fid), 2, 2)
    assert fid.value != 0
    try:
        rgb = np.arange(12, dtype=np.float32).reshape(2, 2, 3) / 7.0
        good = tmp_path / "a.pfm"
        good.write_bytes(b"PF\n2 2\n-1.0\n" + rgb.astype("<f4").tobytes())
        assert lib.phLoadFrame(fid.value, str(good).encode()) == 1
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        lib.phGetFrameDimension(fid.value, ctypes.byref(w), ctypes.byref(h))
        assert (w.value, h.value) == (2, 2)
        data = ctypes.POINTER(ctypes.c_float)()
        lib.phGetFrameRgbData(fid.value, ctypes.byref(data))
        assert np.array_equal(np.ctypeslib.as_array(data, (12,)), rgb.reshape(-1))
        out = tmp_path / "b.pfm"
        assert lib.phSaveFrame(fid.value, str(out).encode(), None) == 1
        assert out.read_bytes() == good.read_bytes()
        huge = tmp_path / "huge.pfm"
        huge.write_bytes(b"PF\n100000 100000\n-1.0\n" + bytes(48))
        assert lib.phLoadFrame(fid.value, str(huge).encode()) == 0
        short = tmp_path / "short.pfm"
        short.write_bytes(b"PF\n2 2\n-1.0\n" + bytes(44))
        assert lib.phLoadFrame(fid.value, str(short).encode()) == 0
        assert lib.phLoadFrame(fid.value, str(tmp_path / "missing.pfm").encode()) == 0
    finally:
        lib.phDeleteFrame(fid.value)


@pytest.mark.parametrize("filt, width, height, n, null_samples, message", [
    (0, 4, 4, 1, False, "not one of the 4 x 4 filters"),        # box: its samples are not splatted
    (7, 4, 4, 1, False, "not one of the 4 x 4 filters"),
    (1, 0, 4, 1, False, "1 to 2^24 pixels"),
    (1, 4097, 4097, 1, False, "1 to 2^24 pixels"),
    (1, 4, 4, (1 << 26) + 1, False, "more than 2^26 samples"),
    (1, 4, 4, 3, True, "null pointer"),
])
def test_film_splat_rejects_bad_input_before_device_work(filt, width, height, n, null_samples, message):
    """pgpu_film_splat checks its filter, film size, sample count and pointers on the host, so these
    calls fail with status 1 and the reason also on a machine without a GPU."""
    import ctypes

    import numpy as np

    lib = photon_gpu.load()
    smp = np.zeros((1, 5), np.float32)   # never read: every case is rejected first
    sums = np.zeros(4, np.float64)
    p_smp = None if null_samples else smp.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    status = lib.pgpu_film_splat(filt, width, height, p_smp, n, sums.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert status == 1
    assert message in lib.pgpu_last_error().decode()


def test_noalloc_rejects_oversized_batches_before_device_work():
    """pgpu_trace_closest_noalloc refuses more rays than its static staging holds (65,536) before it
    looks at the geometry or the device."""
    import ctypes

    import numpy as np

    lib = photon_gpu.load()
    rays = np.zeros((1, 8), np.float32)   # never read: the count is rejected first
    status = lib.pgpu_trace_closest_noalloc(0, rays.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 65537,
                                            None, None, None)
    assert status == 1
    assert "exceed the static scratch capacity" in lib.pgpu_last_error().decode()
