"""The C ABI library: it loads, exports exactly what include/terawarp_b200.h
declares, and its host-only functions (parameter surface, sizes) behave.
CPU only: no compute call is made here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from terawarp_b200 import _lib as L
from terawarp_b200 import api

HEADER = Path(__file__).resolve().parents[1] / "include" / "terawarp_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"typedef[^;]*;", "", text)
    names = set(re.findall(r"\b(tw_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    lib = L.load()
    decl = declared_functions()
    assert len(decl) >= 30
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes signature table covers exactly the declared functions
    assert sorted(L.SIGNATURES) == decl


def test_abi_version_and_status_strings():
    lib = L.load()
    assert lib.tw_abi_version() == 1
    for s in range(9):
        assert lib.tw_status_string(s)


def test_params_default_matches_reference_constants():
    p = api.params()
    assert p.grid_spacing == 4 and abs(p.lambda_ - 0.2) < 1e-15 and p.device_mode == 1
    assert api.output_size(p, (10, 20, 30)) == (10, 20, 30)
    p2 = api.params(resize_mode=1, newsize=(5, 6, 7))
    assert api.output_size(p2, (10, 20, 30)) == (5, 6, 7)


def test_grid_size_rule():
    # gsz = ceil(sz / g) + 1 + 2  (q_imgwarp_tps_quicksmallmemory.cpp:592)
    for sz, g in [(256, 16), (255, 16), (257, 16), (2048, 8), (7, 4)]:
        assert api.grid_size(sz, g) == int(np.ceil(sz / g)) + 3


def test_downsample_factor_rule():
    assert api.downsample_factor((600, 10, 10)) == 1
    assert api.downsample_factor((900, 10, 10)) == 2
    assert api.downsample_factor((100, 100, 100)) == 1  # never 0


def test_translation_matrix():
    M = api.make_affine(1, 1, (3.0, -2.0, 5.5), (10, 10, 10))
    ref = np.eye(4)
    ref[:3, 3] = [-3.0, 2.0, -5.5]
    np.testing.assert_allclose(M, ref)


def test_scaling_matrix():
    M = api.make_affine(0, 2, (2.0, 0.5, 4.0), (10, 10, 10))
    np.testing.assert_allclose(M, np.diag([0.5, 2.0, 0.25, 1.0]))


def test_rotation_matrix_maps_centre_to_centre_and_is_orthonormal():
    in_sz, out_sz = (101, 81, 61), (121, 101, 81)
    M = api.make_affine(1, 0, (30.0, -20.0, 45.0), in_sz, out_sz)
    co = (np.array(out_sz) - 1) / 2
    ci = (np.array(in_sz) - 1) / 2
    np.testing.assert_allclose(M[:3, :3] @ co + M[:3, 3], ci, atol=1e-12)
    np.testing.assert_allclose(M[:3, :3] @ M[:3, :3].T, np.eye(3), atol=1e-12)
    # forward map p_out = c_out + Rz Ry Rx (p_in - c_in); M is its inverse
    ax, ay, az = np.deg2rad([30.0, -20.0, 45.0])
    Rx = np.array([[1, 0, 0], [0, np.cos(ax), -np.sin(ax)], [0, np.sin(ax), np.cos(ax)]])
    Ry = np.array([[np.cos(ay), 0, np.sin(ay)], [0, 1, 0], [-np.sin(ay), 0, np.cos(ay)]])
    Rz = np.array([[np.cos(az), -np.sin(az), 0], [np.sin(az), np.cos(az), 0], [0, 0, 1]])
    np.testing.assert_allclose(M[:3, :3], (Rz @ Ry @ Rx).T, atol=1e-12)


def test_invalid_parameter_combinations_rejected():
    with pytest.raises(api.TeraWarpError):
        api.make_affine(1, 2, (1, 1, 1), (4, 4, 4))
    with pytest.raises(api.TeraWarpError):
        api.make_affine(0, 2, (0.0, 1, 1), (4, 4, 4))


def test_context_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(api.TeraWarpError):
        api.Context(0)
