"""Host-side logic that needs no GPU: the force-field container, the golden fixtures' integrity, the options mapping."""
import numpy as np

from caps_b200 import DynamicsOptions, EnergyOptions, ForceField, cell_array
from tests.fixtures import NAMES, load, rel_rms


def test_fixtures_are_whole():
    for name in NAMES:
        fx = load(name)
        n = fx.ff.natoms
        assert fx.x.shape == (n, 3)
        assert fx.cell.shape == (12,)
        assert fx.ff.excl_offset.size == n + 1
        for (k, prec), f in fx.forces.items():
            assert f.shape == (n, 3) and np.all(np.isfinite(f))


def test_reference_mixed_error_is_small():
    """The reference's own mixed kernel against its FP64 path on the fixtures: the level the device mixed path must meet."""
    for name in ("ps_small", "ps_medium", "lj_triclinic"):
        fx = load(name)
        for k, _ in fx.cases():
            assert rel_rms(fx.forces[(k, "mixed")], fx.forces[(k, "double")]) < 1e-5


def test_forcefield_struct_round_trip():
    fx = load("ps_small")
    ff = fx.ff
    s, keep = ff.to_struct()
    assert s.natoms == ff.natoms and s.ntypes == ff.ntypes
    assert s.nbonds == len(ff.bond_ij) and s.ndihedrals == len(ff.dihedral_ijkl)
    ff2 = ForceField.from_arrays(ff.arrays())
    assert np.array_equal(ff2.excl_list, ff.excl_list) and ff2.lj14 == ff.lj14


def test_options_map_to_the_c_struct():
    o = EnergyOptions(cutoff=12.0, electrostatics="pme", precision="double", pme_order=4).to_struct()
    assert o.cutoff == 12.0 and o.electrostatics == 1 and o.precision == 1 and o.pme_order == 4
    m = DynamicsOptions(thermostat="nose-hoover", constraints="h-bonds").to_struct(load("ps_small").ff, [])
    assert m.thermostat == 3 and m.constraints == 1


def test_cell_array_forms():
    assert cell_array(np.eye(3) * 10).tolist() == [0, 0, 0, 10, 0, 0, 0, 10, 0, 0, 0, 10]
    assert cell_array(list(range(12))).size == 12


def test_constraint_algorithm_and_barostat_names():
    """constraint_algorithm maps shake / lincs onto the C struct (constraint_algorithm_from_string, constraints.hpp:22),
    the barostat names as barostat_from_string does (dynamics.cpp:36-42); unknown names are refused before any call."""
    import pytest
    fx = load("ps_small")
    keep: list = []
    assert DynamicsOptions(constraints="h-bonds", constraint_algorithm="LINCS").to_struct(fx.ff, keep).constraint_algorithm == 1
    assert DynamicsOptions(constraints="h-bonds").to_struct(fx.ff, keep).constraint_algorithm == 0
    with pytest.raises(ValueError, match="unknown constraint algorithm"):
        DynamicsOptions(constraint_algorithm="p-lincs").to_struct(fx.ff, keep)
    assert DynamicsOptions(barostat="mtk").to_struct(fx.ff, keep).barostat == 3
    with pytest.raises(ValueError, match="unknown barostat"):
        DynamicsOptions(barostat="andersen").to_struct(fx.ff, keep)
