"""The oracle's FFT against numpy, and the synthetic-input generator."""
import ctypes

import numpy as np
import pytest

from molmodel_b200.water import box_length, water_box
from oracle.oracle import PORT_LIB, port


@pytest.mark.parametrize("shape", [(6, 10, 14), (18, 18, 18), (7, 5, 9), (48, 48, 48), (12, 20, 21)])
def test_fft_matches_numpy(shape):
    port()
    lib = ctypes.CDLL(PORT_LIB)
    nx, ny, nz = shape
    a = np.random.default_rng(0).random(shape)
    out = np.zeros((nx, ny, nz // 2 + 1), dtype=np.complex128)
    lib.fft235_r2c_3d(nx, ny, nz, a.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    ref = np.fft.rfftn(a)
    assert np.abs(out - ref).max() <= 1e-14 * np.abs(ref).max()
    back = np.zeros(shape)
    lib.fft235_c2r_3d(nx, ny, nz, ref.ctypes.data_as(ctypes.c_void_p), back.ctypes.data_as(ctypes.c_void_p))
    assert np.abs(back / a.size - a).max() < 1e-14


def test_box_lengths_match_workloads():
    assert abs(box_length(216) - 18.644) < 1e-3
    assert abs(box_length(4096) - 49.719) < 1e-3
    assert abs(box_length(32768) - 99.437) < 1e-3
    assert abs(box_length(512) - 24.859) < 1e-3


def test_water_geometry_and_determinism():
    a, b = water_box(4, seed=3), water_box(4, seed=3)
    assert np.array_equal(a.positions, b.positions)
    assert not np.array_equal(a.positions, water_box(4, seed=4).positions)
    r = a.positions.reshape(-1, 3, 3)
    d1 = np.linalg.norm(r[:, 1] - r[:, 0], axis=1)
    d2 = np.linalg.norm(r[:, 2] - r[:, 0], axis=1)
    ang = np.degrees(np.arccos(((r[:, 1] - r[:, 0]) * (r[:, 2] - r[:, 0])).sum(1) / (d1 * d2)))
    assert np.allclose(d1, 1.0, atol=1e-12) and np.allclose(d2, 1.0, atol=1e-12)
    assert np.allclose(ang, 109.47, atol=1e-9)
    assert abs(a.q.sum()) < 1e-12
