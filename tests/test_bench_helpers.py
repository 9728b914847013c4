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
