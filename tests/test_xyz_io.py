"""CPU: structure file input through the C ABI (tb_read_xyz, host only):
an XYZ file written from a generated structure reads back as the same atomic
numbers and coordinates (Bohr), element symbols in any case and atomic
numbers are accepted, the cap = 0 call sizes the buffers, and malformed
files give TB_BAD_INPUT."""
import numpy as np
import pytest

from tblite_b200 import capi, geometry as g


def test_round_trip(tmp_path):
    mol = g.water_clusters(1, seed=61, nmin=7, nmax=7)[0]
    p = tmp_path / "w7.xyz"
    g.write_xyz(mol, str(p))
    z, xyz, comment = capi.read_xyz(str(p))
    np.testing.assert_array_equal(z, np.array([1, 6, 8])[mol.id])
    np.testing.assert_allclose(xyz, mol.xyz, rtol=0, atol=1e-12)
    assert comment == mol.label


def test_symbols_and_numbers(tmp_path):
    p = tmp_path / "mix.xyz"
    p.write_text("3\ncomment here\n o 0 0 0\nH 0.96 0 0\n1 -0.24 0.93 0\n")
    z, xyz, comment = capi.read_xyz(str(p))
    assert z.tolist() == [8, 1, 1] and comment == "comment here"
    np.testing.assert_allclose(xyz[1], [0.96 / 0.529177210903, 0, 0], rtol=1e-15)


@pytest.mark.parametrize("text", ["x\n\nH 0 0 0\n", "2\n\nH 0 0 0\n", "1\n\nQq 0 0 0\n", "1\n\nH 0 0\n"])
def test_malformed(tmp_path, text):
    p = tmp_path / "bad.xyz"
    p.write_text(text)
    with pytest.raises(capi.TBError) as e:
        capi.read_xyz(str(p))
    assert e.value.status == capi.TB_BAD_INPUT


@pytest.mark.gpu
def test_singlepoint_from_xyz(gpu_calc, tmp_path):
    mol = g.octane()
    p = tmp_path / "octane.xyz"
    g.write_xyz(mol, str(p))
    m2 = gpu_calc.molecule_from_xyz(str(p))
    assert m2.id.tolist() == mol.id.tolist()
    a, b = gpu_calc.singlepoint_batch([mol])[0], gpu_calc.singlepoint_batch([m2])[0]
    assert abs(a["energy"] - b["energy"]) < 1e-11
