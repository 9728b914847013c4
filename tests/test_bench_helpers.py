"""Host-side helpers of bench.py that need no GPU."""
import bench


def test_mt19937_64_known_answer():
    # C++ [rand.predef]: the 10000th draw of a default-constructed std::mt19937_64 (seed 5489)
    g = bench.MT19937_64(5489)
    x = 0
    for _ in range(10000):
        x = g()
    assert x == 9981545732273789042


def test_seeded_nodes_distinct_and_deterministic():
    cand = list(range(100, 700, 3))
    a = bench.seeded_nodes(cand, 20, 20261203)
    assert len(a) == 20 and len(set(a)) == 20 and all(c in cand for c in a)
    assert a == bench.seeded_nodes(cand, 20, 20261203)


def test_cpu_section_parity_and_baseline_on_a_small_mesh():
    """The oracle leg of the GPU arm on a tiny cylinder: fed with the oracle's own step-1 and
    step-3 states as the 'GPU' fields it reports bit-exact parity, and the timed CPU baseline
    (reference algorithm) produces a rate."""
    from types import SimpleNamespace

    import numpy as np

    args = SimpleNamespace(rings=2, layers=6, no_cpu_baseline=False)
    _, o = bench.oracle_cylinder(2, 6, pressure_solver=3)
    o.set_momentum_solver(1 if bench.MOMENTUM_SOLVER == "cg" else 0)  # the headline's method
    states = {}
    for k in (1, 2, 3):
        assert o.piso_step() == 0
        if k in (1, 3):
            st = o.state()
            states[k] = (st["u"].copy(), st["p"].copy())
    parity, mixed_cpu, cpu = bench.cpu_section(args, states, {"fp64": (np.zeros((o.N2, 3)), np.zeros(o.nv))})
    assert parity["ok"] and set(parity["at_step"]) == {"1", "3"}
    assert all(v["bit_exact"] and v["u"] == 0.0 for v in parity["at_step"].values())
    assert mixed_cpu["fp64"]["u"] == 1.0  # zero field against the oracle's step 1
    assert cpu["kind"] == "port" and cpu["value"] > 0 and cpu["cores"] >= 1
