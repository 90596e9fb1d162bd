"""parsec.dat writer / reader (library C++, no GPU): round trip, the record
sequence of shared/parsec_wfn.F90, loading a synthetic molecule back, and
unsupported / damaged files reported as errors."""
import struct

import numpy as np
import pytest

from nanogw_b200 import NGWError, parsec
from nanogw_b200._lib import NGW_ERR_ARG


def _records(path):
    recs = []
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        (n,) = struct.unpack_from("<i", data, i)
        payload = data[i + 4:i + 4 + n]
        (m,) = struct.unpack_from("<i", data, i + 4 + n)
        assert m == n
        recs.append(payload)
        i += 8 + n
    return recs


def test_round_trip_and_record_order(small_system, tmp_path):
    mol = small_system.mol
    d = parsec.from_molecule(mol)
    p = tmp_path / "parsec.dat"
    parsec.write(p, d)
    r = parsec.read(p)
    for name in ("gtable", "rho", "irep", "e0", "occ", "iord", "wfn", "trans", "chi", "shift"):
        assert np.array_equal(getattr(r, name), getattr(d, name)), name
    assert r.step == d.step and r.ndim == d.ndim and r.datelabel == d.datelabel.rstrip()
    recs = _records(p)
    ng, ns = mol.psi.shape
    # the reader's sequence: header, symmetry, grid, states, density, wavefunctions
    assert len(recs[0]) == 26
    assert struct.unpack("<3i", recs[1]) == (1, 0, 0)
    assert struct.unpack("<d", recs[2])[0] == mol.h
    assert struct.unpack("<2i", recs[5]) == (ng, 1)
    assert len(recs[7]) == 72 and len(recs[10]) == 4
    assert np.array_equal(np.frombuffer(recs[11], dtype="<i4").reshape(ng, 3), mol.grid_idx)
    assert struct.unpack("<i", recs[12])[0] == ns
    assert np.array_equal(np.frombuffer(recs[14], dtype="<f8"), mol.e1)
    assert np.array_equal(np.frombuffer(recs[17], dtype="<f8"), mol.rho)
    assert struct.unpack("<i", recs[25])[0] == ns
    assert len(recs) == 27 + ns
    assert np.array_equal(np.frombuffer(recs[27], dtype="<f8"), mol.psi[:, 0])


def test_load_molecule(small_system, tmp_path):
    mol = small_system.mol
    p = tmp_path / "parsec.dat"
    parsec.write(p, parsec.from_molecule(mol))
    m = parsec.load_molecule(p)
    assert np.array_equal(m.grid_idx, mol.grid_idx)      # already in descending density
    assert np.array_equal(m.psi, mol.psi) and np.array_equal(m.rho, mol.rho)
    assert m.nval == mol.nval and np.array_equal(m.e1, mol.e1)
    r = np.sqrt((mol.grid.astype(np.float64) ** 2).sum(axis=1)).max()
    assert abs(m.rmax - r) < 1e-12 and m.rmax <= mol.rmax


def test_unsupported_and_damaged_files(small_system, tmp_path):
    mol = small_system.mol
    p = tmp_path / "parsec.dat"
    parsec.write(p, parsec.from_molecule(mol))
    data = bytearray(open(p, "rb").read())
    # nspin = 2 in record 2 (payload starts after record 1: 4 + 26 + 4 + 4 bytes)
    spin = bytearray(data)
    struct.pack_into("<i", spin, 38, 2)
    q = tmp_path / "spin.dat"
    q.write_bytes(bytes(spin))
    with pytest.raises(NGWError) as e:
        parsec.read(q)
    assert e.value.code == NGW_ERR_ARG
    t = tmp_path / "trunc.dat"
    t.write_bytes(bytes(data[: len(data) // 2]))
    with pytest.raises(NGWError):
        parsec.read(t)
