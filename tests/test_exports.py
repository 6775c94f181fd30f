"""The library loads without a GPU and exports every entry point the public headers declare."""

import os
import re

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
