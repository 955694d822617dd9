"""`.krk` front end: Backend directive and Sweep expansion
(test/test_simulation_runner.jl:327-400, test/test_kraken_parser.jl:543-580)."""
import pytest

CAVITY = """
Simulation backend_dispatch_test D2Q9
Domain L = 1 x 1  N = 8 x 8
Physics nu = 0.1
{backend}
Boundary north velocity(ux = 0.1, uy = 0)
Boundary south wall
Boundary east  wall
Boundary west  wall
Run 5 steps
"""


def test_backend_parsed(pkg):
    st = pkg.krk.parse_kraken(CAVITY.format(backend="Backend b200"))
    assert st.backend == "b200" and st.N[:2] == (8, 8) and st.max_steps == 5
    assert st.boundaries["north"] == ("velocity", {"ux": 0.1, "uy": 0.0})
    assert pkg.krk.parse_kraken(CAVITY.format(backend="")).backend is None


def test_unknown_backend_is_parse_error(pkg):
    with pytest.raises(ValueError, match="tpu"):
        pkg.krk.parse_kraken(CAVITY.format(backend="Backend tpu"))


def test_non_b200_backend_never_falls_back(pkg):
    st = pkg.krk.parse_kraken(CAVITY.format(backend="Backend cuda"))
    with pytest.raises(ValueError, match="cuda"):
        pkg.krk.resolve_backend(st, None)
    # the explicit argument wins over the file
    assert pkg.krk.resolve_backend(st, "b200") == "b200"
    st2 = pkg.krk.parse_kraken(CAVITY.format(backend="Backend b200"))
    with pytest.raises(ValueError, match="cpu"):
        pkg.krk.resolve_backend(st2, "cpu")


def test_sweep_cartesian_product(pkg):
    text = """
Simulation sweep_re D2Q9
Domain L = 1 x 1 N = 64 x 64
Setup reynolds = Re L_ref = 64 U_ref = 0.1
Boundary north velocity(ux = 0.1, uy = 0)
Boundary south wall
Boundary east wall
Boundary west wall
Sweep Re = [100, 200, 500]
Sweep N = [64, 96]
Run 100 steps
"""
    setups = pkg.krk.parse_kraken_sweep(text)
    assert len(setups) == 6
    assert [s.sweep_values["Re"] for s in setups[:2]] == [100.0, 100.0]
    assert [s.sweep_values["N"] for s in setups[:2]] == [64.0, 96.0]
    assert abs(setups[0].nu - 0.1 * 64 / 100) < 1e-15
    assert abs(setups[2].nu - 0.1 * 64 / 200) < 1e-15


def test_examples_parse(pkg):
    st = pkg.krk.parse_kraken("""
Simulation taylor_green D2Q9
Domain  L = 64 x 64  N = 64 x 64
Define u0 = 0.01
Physics nu = 0.01
Boundary x periodic
Boundary y periodic
Run 1000 steps
""")
    assert st.boundaries["x"][0] == "periodic" and st.user_vars["u0"] == 0.01


def test_krk_arithmetic_rejects_code(pkg):
    """Values in a .krk file are numbers, defined names and + - * / ( );
    anything else (calls, attributes) is an error, never executed."""
    k = pkg.krk
    assert k._num("2*nu+1", {"nu": 0.5}) == 2.0
    assert k._num("-(3/4)", {}) == -0.75
    for bad in ("__import__('os')", "nu.real", "f(1)", "1/0"):
        with pytest.raises(ValueError):
            k._num(bad, {"nu": 0.5})
