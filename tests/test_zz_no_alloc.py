"""mmnb_kspace_field_noalloc: the ordinary Ewald k-sum for callers that cannot
allocate device memory (a host that has reserved all of it for its own pool,
or a loop that must not let cudaMalloc/cudaFree synchronise the device).

It is called here through the C ABI with device arrays the test owns, twice in
a row, and must give what the allocating path (mmnb_create + mmnb_compute with
only the k-space term switched on) gives, and what the oracle's restatement of
kspace_field (src/kspace.c:87-174) gives, within the FP64 parity tolerance, on
a cubic and an orthorhombic box.  The file is named to be collected last, so a
run that stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_max
from molmodel_b200 import ElecLJ, load_library, water_box

pytestmark = pytest.mark.gpu

TOL = 1e-10
CUBIC, ORTHORHOMBIC = 1, 2


def _noalloc(lib, r, q, bctype, box, eta, kc):
    import torch
    dev = torch.device("cuda", 0)
    d_r = torch.tensor(np.ascontiguousarray(r).reshape(-1), dtype=torch.float64, device=dev)
    d_q = torch.tensor(q, dtype=torch.float64, device=dev)
    d_phi = torch.zeros(len(q), dtype=torch.float64, device=dev)
    d_evec = torch.zeros(3 * len(q), dtype=torch.float64, device=dev)
    b = (ctypes.c_double * 3)(*box)
    torch.cuda.synchronize(dev)
    st = lib.mmnb_kspace_field_noalloc(len(q), d_r.data_ptr(), d_q.data_ptr(), bctype, b, eta, kc,
                                       d_phi.data_ptr(), d_evec.data_ptr(), None)
    assert st == 0, lib.mmnb_last_error(None)
    torch.cuda.synchronize(dev)
    return d_phi.cpu().numpy(), d_evec.cpu().numpy().reshape(-1, 3)


def test_noalloc_kspace_matches_allocating_path_twice():
    wb = water_box(6, seed=1)
    cfg = dict(rspace_cutoff=9.0, ewald_screening=0.35, kspace_cutoff=7.0, include_rspace=False,
               include_self=False, include_lj_correction=False)
    ref = ElecLJ(**cfg).init(wb).compute(wb.positions, want_fields=True)
    lib = load_library()
    for _ in range(2):
        phi, evec = _noalloc(lib, wb.positions, wb.q, CUBIC, (wb.box,) * 3, 0.35, 7.0)
        assert rel_max(phi, ref["phi"]) < TOL
        assert rel_max(evec, ref["evec"]) < TOL


def test_noalloc_kspace_matches_oracle_cubic_and_orthorhombic():
    from oracle.oracle import port
    wb = water_box(6, seed=3)
    lib = load_library()
    # the cubic box, then the same sites in an orthorhombic box with three different edges
    for bctype, box, kc in [(CUBIC, (wb.box,) * 3, 9.3), (ORTHORHOMBIC, (wb.box, 1.1 * wb.box, 1.25 * wb.box), 8.0)]:
        phi_o, evec_o, nk = port().kspace_field(kc, wb.positions, wb.q, np.diag(box), 0.31)
        assert nk > 0
        for _ in range(2):
            phi, evec = _noalloc(lib, wb.positions, wb.q, bctype, box, 0.31, kc)
            assert rel_max(phi, phi_o) < TOL
            assert rel_max(evec, evec_o) < TOL


def test_noalloc_rejects_more_wave_vectors_than_it_holds():
    import torch
    lib = load_library()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    box = (ctypes.c_double * 3)(20.0, 20.0, 20.0)
    # 12.5 is counted (4108 wave vectors); 14, 1e300 and inf are refused before counting
    for kc in (12.5, 14.0, 1e300, float("inf"), float("nan")):
        st = lib.mmnb_kspace_field_noalloc(3, buf.data_ptr(), buf.data_ptr(), 1, box, 0.35, kc,
                                           buf.data_ptr(), buf.data_ptr(), None)
        assert st == 1
        if kc == kc:  # NaN is refused as a cutoff that is not > 0
            assert b"at most 4096" in lib.mmnb_last_error(None)
