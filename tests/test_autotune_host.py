"""The autotuner's search (thruster_cx_code_b200/autotune.py) on the host, with a made-up
cost in place of timed GPU steps."""
from thruster_cx_code_b200 import autotune as A

SPACE = {"a": (1, 2, 3), "b": ("x", "y"), "c": (10, 20, 40)}


def _cost(k):
    # separable, minimum at a=3, b="y", c=20
    return {1: 5.0, 2: 4.0, 3: 3.0}[k["a"]] + {"x": 2.0, "y": 1.0}[k["b"]] + {10: 1.5, 20: 1.0, 40: 1.2}[k["c"]]


def test_finds_separable_minimum():
    calls = []

    def measure(k):
        calls.append(dict(k))
        return _cost(k)

    best, table = A.coordinate_descent({"a": 1, "b": "x", "c": 10}, SPACE, measure)
    assert best == {"a": 3, "b": "y", "c": 20}
    # each distinct setting measured once: start + 2 + 1 + 2 candidates
    assert len(calls) == len(table) == 6


def test_min_gain_keeps_incumbent():
    # b = "y" is only 0.5% faster than the incumbent: not taken at a 1% threshold
    def measure(k):
        return 100.0 - (0.5 if k["b"] == "y" else 0.0)

    best, _ = A.coordinate_descent({"a": 1, "b": "x", "c": 10}, SPACE, measure, min_gain=0.01)
    assert best["b"] == "x"
    best, _ = A.coordinate_descent({"a": 1, "b": "x", "c": 10}, SPACE, measure, min_gain=0.001)
    assert best["b"] == "y"


def test_second_pass_uses_new_incumbent():
    # a = 3 wins at c = 10, then c = 40 wins at a = 3; only a second pass finds that a = 1
    # is better again at c = 40
    table = {(1, 10): 10.0, (3, 10): 9.0, (3, 40): 5.0, (1, 40): 2.0}

    def measure(k):
        return table[(k["a"], k["c"])]

    space = {"a": (1, 3), "c": (10, 40)}
    best1, _ = A.coordinate_descent({"a": 1, "c": 10}, space, measure, passes=1)
    best2, _ = A.coordinate_descent({"a": 1, "c": 10}, space, measure, passes=2)
    assert best1 == {"a": 3, "c": 40}
    assert best2 == {"a": 1, "c": 40}


def test_knob_space_matches_the_library():
    assert set(A.KNOBS) == {"max_coarse", "tol_inner", "sort_every", "particle_blocks_per_sm", "solve_blocks",
                            "deposit_hist", "ion_tma_window", "electron_kernel", "particles_per_block",
                            "smoother_sweeps"}
    assert max(A.KNOBS["max_coarse"]) <= 4096 and min(A.KNOBS["max_coarse"]) >= 4


def test_kernel_variant_knobs_round_trip():
    from thruster_cx_code_b200 import _lib
    for bits in (0, _lib.PB_OPT_SMEM_HIST, _lib.PB_OPT_TMA_TILE | _lib.PB_OPT_ELE_PAIRS,
                 _lib.PB_OPT_SMEM_HIST | _lib.PB_OPT_ELE_SPLIT):
        assert A.options_bits(A.options_knobs(bits)) == bits
    assert A.options_bits({"electron_kernel": "split"}, _lib.PB_OPT_SMEM_HIST) == \
        _lib.PB_OPT_SMEM_HIST | _lib.PB_OPT_ELE_SPLIT
