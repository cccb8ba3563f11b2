"""mmnb_kspace_field_noalloc: the ordinary Ewald k-sum for callers that cannot
allocate device memory (a host that has reserved all of it for its own pool,
or a loop that must not let cudaMalloc/cudaFree synchronise the device).

It is called here through the C ABI with device arrays the test owns, twice in
a row, and must give what the allocating path (mmnb_create + mmnb_compute with
only the k-space term switched on) gives, within the FP64 parity tolerance.
The file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_max
from molmodel_b200 import ElecLJ, load_library, water_box

pytestmark = pytest.mark.gpu

TOL = 1e-10


def test_noalloc_kspace_matches_allocating_path_twice():
    import torch
    wb = water_box(6, seed=1)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, kspace_cutoff=7.0, include_rspace=False,
               include_self=False, include_lj_correction=False)
    ref = ElecLJ(**cfg).init(wb).compute(wb.positions, want_fields=True)
    lib = load_library()
    dev = torch.device("cuda", 0)
    d_r = torch.tensor(wb.positions.reshape(-1), dtype=torch.float64, device=dev)
    d_q = torch.tensor(wb.q, dtype=torch.float64, device=dev)
    box = (ctypes.c_double * 3)(wb.box, wb.box, wb.box)
    for _ in range(2):
        d_phi = torch.zeros(wb.nsite, dtype=torch.float64, device=dev)
        d_evec = torch.zeros(3 * wb.nsite, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        st = lib.mmnb_kspace_field_noalloc(wb.nsite, d_r.data_ptr(), d_q.data_ptr(), 1, box, 0.35, 7.0,
                                           d_phi.data_ptr(), d_evec.data_ptr(), None)
        assert st == 0, lib.mmnb_last_error(None)
        torch.cuda.synchronize(dev)
        assert rel_max(d_phi.cpu().numpy(), ref["phi"]) < TOL
        assert rel_max(d_evec.cpu().numpy().reshape(-1, 3), ref["evec"]) < TOL


def test_noalloc_rejects_more_wave_vectors_than_it_holds():
    import torch
    lib = load_library()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    box = (ctypes.c_double * 3)(20.0, 20.0, 20.0)
    st = lib.mmnb_kspace_field_noalloc(3, buf.data_ptr(), buf.data_ptr(), 1, box, 0.35, 14.0,
                                       buf.data_ptr(), buf.data_ptr(), None)
    assert st == 1
    assert b"at most 4096" in lib.mmnb_last_error(None)
