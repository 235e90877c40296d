"""Host logic of the batched ensemble: the seeded box draw (no GPU)."""
from compact_schemes_b200.ensemble import MT19937_64, SIZES, draw_boxes, ensemble_points


def test_mt19937_64_known_answer():
    # 10000th output of the 64-bit Mersenne Twister with the default seed 5489
    # (the value the C++ standard requires of std::mt19937_64)
    g = MT19937_64(5489)
    for _ in range(9999):
        g.next_u64()
    assert g.next_u64() == 9981545732273789042


def test_draw_boxes_seeded_and_in_range():
    a = draw_boxes(64, 0)
    assert a == draw_boxes(64, 0)
    assert a != draw_boxes(64, 1)
    assert len(a) == 64
    for dims, mach, re in a:
        assert all(n in SIZES for n in dims)
        assert 0.05 <= mach < 0.3 and 400.0 <= re < 3200.0
    # every size and both ends of the ranges are represented in 192 draws
    assert {n for d, _, _ in a for n in d} == set(SIZES)
    assert 10_000_000 < ensemble_points(a) < 64 * 128 ** 3
