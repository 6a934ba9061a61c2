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


def test_pair_forms_and_tables_map_to_the_c_struct():
    """ForceField.pair_func and tables flatten into the ABI 5 fields: type pairs as (a <= b), the reference's form codes
    (field.hpp:61-75), (form, a, b, c, rc) per entry, and the tables one after another."""
    import ctypes as C
    import dataclasses
    import numpy as np
    fx = load("ps_small")
    tab = (1.5, 0.01, np.linspace(1.0, 0.0, 5), np.linspace(2.0, 0.0, 5))
    ff = dataclasses.replace(fx.ff, pair_func={(1, 0): ("buckingham", 1.0, 0.3, 2.0), (2, 2): ("morse", 0.1, 1.2, 3.8, 6.5),
                                               (3, 3): ("table", 0, 0, 0), (0, 3): (20, 0.03, 2.6, 0.0)},
                             lj_inner=6.0, lj_fsw=True, tables=[tab, tab])
    s, keep = ff.to_struct()
    assert s.npair_func == 4 and s.ntables == 2 and s.lj_fsw == 1 and s.lj_inner == 6.0
    ab = np.ctypeslib.as_array(C.cast(s.pair_func_ab, C.POINTER(C.c_int32)), shape=(8,)).reshape(4, 2)
    p = np.ctypeslib.as_array(C.cast(s.pair_func_p, C.POINTER(C.c_double)), shape=(20,)).reshape(4, 5)
    assert ab.tolist() == [[0, 1], [0, 3], [2, 2], [3, 3]]
    assert p[:, 0].tolist() == [1.0, 20.0, 2.0, 40.0] and p[2, 4] == 6.5 and p[0, 4] == 0.0
    n = np.ctypeslib.as_array(C.cast(s.table_n, C.POINTER(C.c_int32)), shape=(2,))
    e = np.ctypeslib.as_array(C.cast(s.table_e, C.POINTER(C.c_double)), shape=(10,))
    assert n.tolist() == [5, 5] and np.allclose(e[:5], tab[2]) and np.allclose(e[5:], tab[2])
