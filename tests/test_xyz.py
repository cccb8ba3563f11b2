"""xyz format of the reference (src/msys.cpp:823-941): round trip and a
hand-written frame in the layout MSys::write_as_xyz produces."""
import io

import numpy as np

from molmodel_b200 import maxwell_boltzmann, water_box
from molmodel_b200.xyz import read_xyz, water_symbols, write_xyz


def test_round_trip_keeps_every_double():
    wb = water_box(3, seed=2)
    v = maxwell_boltzmann(wb, 300.0, seed=1)
    buf = io.StringIO()
    write_xyz(buf, water_symbols(wb.nwater), wb.positions, v, box=wb.box, comment="Time elapsed: 0.500000 psec")
    buf.seek(0)
    d = read_xyz(buf)
    assert d["symbols"] == water_symbols(wb.nwater)
    assert np.array_equal(d["positions"], wb.positions) and np.array_equal(d["velocities"], v)
    assert d["bctype"] == "cubic" and d["box"] == wb.box
    assert d["comment"] == "Time elapsed: 0.500000 psec"


def test_reads_the_reference_layouts():
    text = ("3\nboundary_conditions orthorhombic 10 11 12  Time elapsed: 1.000000 psec\n"
            "O  1 2 3 OW  0.1 0.2 0.3\n"
            "H  1.5 2 3 *\n"
            "H  0.5 2 3\n")
    d = read_xyz(io.StringIO(text))
    assert d["bctype"] == "orthorhombic" and np.allclose(d["box"], [10, 11, 12])
    assert d["types"] == ["OW", "*", "*"]
    assert np.allclose(d["positions"][1], [1.5, 2, 3])
    assert np.allclose(d["velocities"][0], [0.1, 0.2, 0.3]) and np.allclose(d["velocities"][2], 0)
