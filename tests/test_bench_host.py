"""CPU tests of bench.py's host-side bookkeeping: the byte model behind the
roofline, the forward kinds of the transform leg, and the parsing of the
clock samples taken during the timed region (no GPU needed)."""
import bench
from oracle import emulation as E


def test_solve_bytes_512_bc340():
    """512^3, codes (3, 4, 0): each of the five passes moves 2.15 GB and a
    solve 10.76 GB (80 B per point), the figures the roofline divides by."""
    b = bench.solve_pass_bytes(512, 512, 512, 3, 4, 0)
    assert list(b) == ["solve_x_fwd", "solve_y_fwd", "solve_z_fwd_div_inv", "solve_y_inv", "solve_x_inv"]
    assert all(v == 2151677952 for v in b.values())
    assert sum(b.values()) == 10758389760
    assert abs(sum(b.values()) / 512 ** 3 - 80.15) < 0.01


def test_solve_bytes_windows_follow_the_solver():
    """Windows per code match the solver's (the oracle's solver_windows), and
    a periodic axis adds the N+1 spectral entry."""
    for bc in range(5):
        s, e, sp0, sp1 = bench._windows(bc, 64)
        assert (s, e) == E.solver_windows(bc, 64)
        assert sp0 == s and sp1 == (65 if bc == 0 else e)
    b = bench.solve_pass_bytes(32, 16, 8, 1, 2, 0)
    X, Y, Z = 31, 16, 8            # code 1: 1..31, code 2: 1..16, code 0: 0..7
    Xs, Zs = 31, 9                 # spectral: x as its window, z 0..8
    assert b["solve_x_fwd"] == Y * Z * (X + Xs) * 8
    assert b["solve_z_fwd_div_inv"] == Xs * Y * 2 * Z * 8


def test_transform_leg_kinds():
    """The transform leg uses the solver's forward kind of each code, and the
    128^3 configuration's stated DST-I / DST-II / DFT."""
    for bc in range(5):
        assert bench.FORWARD_KIND[bc] == E.solver_kinds(bc)[0]
    assert bench.TRANSFORM_KINDS["helmholtz_fp64_128"] == (E.DST_1, E.DST_2, E.DFT_R2C)


def test_clock_sampler_parses_reasons_and_median():
    s = bench.ClockSampler(["0"])
    s.proc = type("P", (), {"terminate": lambda self: None, "wait": lambda self, timeout=None: 0})()
    s._t = type("T", (), {"join": lambda self, timeout=None: None})()
    s.lines = [
        "1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "1950, 1965, 980.4, 0x4, Not Active, Not Active, Not Active, Active",
        "1965, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "garbage line",
    ]
    c = s.stop()
    assert c["samples"] == 3
    assert c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]


def test_clock_sampler_without_nvidia_smi():
    c = bench.ClockSampler(["0"]).stop()
    assert c["reasons"] == ["unsampled"] and c["samples"] == 0
