"""The reference's SIC file formats (publicrelease_2020_b200/files.py):
Fortran edit descriptors as gfortran writes them, and the unformatted record
layout (4-byte length, payload, 4-byte length)."""
import os

import numpy as np

from publicrelease_2020_b200 import files as F


def test_fortran_edit_descriptors():
    assert F.fortran_f(1.0, 4, 0) == "  1."
    assert F.fortran_f(12.0, 4, 0) == " 12."
    assert F.fortran_f(-0.5, 11, 6) == "  -0.500000"
    assert F.fortran_f(0.123456789, 12, 5) == "     0.12346"
    assert F.fortran_f(-1e-9, 12, 5) == "    -0.00000"
    assert F.fortran_f(1.0e12, 12, 5) == "************"
    assert F.fortran_f(-0.25, 5, 3) == "-.250"
    assert F.fortran_f(3.0, 20, 12) == "      3.000000000000"


def test_format_reversion_of_sicd_rows():
    lines = F.format_line(np.arange(20) * 0.5, 12, 5, 15)
    assert len(lines) == 2 and lines[0].startswith(" ") and len(lines[0]) == 1 + 15 * 12
    assert len(lines[1]) == 1 + 5 * 12


def test_unformatted_records_roundtrip(tmp_path):
    pot = np.linspace(-1, 1, 7)
    p = F.write_zpot(str(tmp_path), 3, pot)
    assert os.path.basename(p) == "ZPOT0003" and os.path.getsize(p) == 16 * 7
    recs = F.read_unformatted(p)
    assert len(recs) == 7 and np.array_equal(np.concatenate(recs), pot)
    mix = np.arange(24, dtype=float).reshape(6, 4)
    p = F.write_mgga(str(tmp_path), 12, mix)
    recs = F.read_unformatted(p)
    assert os.path.basename(p) == "MGGA0012" and len(recs) == 6 and np.array_equal(np.stack(recs), mix)


def test_sic_energy_and_fforce_layout(tmp_path):
    res = np.zeros((2, 3, 13))
    for k in range(3):
        res[0, k] = np.arange(13) * 0.1 + k
        res[0, k, 0] = k + 1
    F.write_sic_energy(str(tmp_path / "SIC_ENERGY"), res, [3])
    lines = open(tmp_path / "SIC_ENERGY").read().splitlines()
    assert lines[0] == F.SIC_ENERGY_HEADER and len(lines) == 4
    assert lines[1][:4] == "  1." and len(lines[1]) == 4 + 8 * 11
    vals = [float(lines[2][4 + 11 * i: 15 + 11 * i]) for i in range(8)]
    assert np.allclose(vals, [res[0, 1, i - 1] for i in F.IRES[1:]], atol=5e-7)
    deb = np.arange(18, dtype=float).reshape(2, 3, 3) / 7
    F.write_fforce(str(tmp_path / "fforce.dat"), deb, [3, 2])
    lines = open(tmp_path / "fforce.dat").read().splitlines()
    assert len(lines) == 5 and all(len(x) == 61 for x in lines)
    assert abs(float(lines[4].split()[2]) - deb[1, 1, 2]) < 1e-12
