"""Equilibration protocols as data (core/src/equilibrate.cpp:43-164): the 21-step table, annealing and push-off
lists, and the plain-text protocol format. Needs no GPU."""
import pytest

from caps_b200 import ProtocolParams, parse_protocol, protocol_by_name
from caps_b200.equilibrate import protocol_ps


def test_larsen21_table():
    s = protocol_by_name("larsen21", ProtocolParams())
    assert len(s) == 21
    assert abs(protocol_ps(s) - 1560.0) < 1e-9          # 1.56 ns at time_scale 1 (equilibrate.hpp:40-42)
    assert [g.ensemble for g in s].count("npt") == 7
    assert s[8].pressure == pytest.approx(49346.2) and s[20].pressure == 1.0 and s[20].ps == 800
    half = protocol_by_name("21-step", ProtocolParams(time_scale=0.5))
    assert abs(protocol_ps(half) - 780.0) < 1e-9


def test_annealing_and_pushoff():
    a = protocol_by_name("annealing", ProtocolParams(cycles=2))
    assert len(a) == 1 + 4 * 2 and a[1].t_end == 600 and a[3].t_end == 300
    p = protocol_by_name("push-off", ProtocolParams())
    assert [g.force_cap for g in p[:7]] == [5, 10, 20, 50, 100, 200, 500] and p[-1].ensemble == "npt"
    with pytest.raises(ValueError):
        protocol_by_name("nonsense", ProtocolParams())
    with pytest.raises(ValueError):
        protocol_by_name("larsen21", ProtocolParams(time_scale=0))


def test_parse_protocol():
    s = parse_protocol("nvt 50 ps T 600   # heat\nnpt 0.05 ns T 300 P 987 bar\n\nnvt 20 ps T 300 to 600\nnvt 5000 fs T 300 cap 20\nnve 10 ps\n")
    assert [g.ensemble for g in s] == ["nvt", "npt", "nvt", "nvt", "nve"]
    assert s[0].label == "heat" and s[1].label == "2 · npt"
    assert s[1].ps == 50 and s[1].pressure == pytest.approx(987 / 1.01325)
    assert s[2].t_start == 300 and s[2].t_end == 600
    assert s[3].ps == 5 and s[3].force_cap == 20
    for bad in ("xyz 10 ps", "npt 10 ps T 300", "nvt T 300", "nvt 10 ps T", "nvt 10 ps Q 3", ""):
        with pytest.raises(ValueError):
            parse_protocol(bad)
