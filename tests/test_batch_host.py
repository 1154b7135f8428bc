"""Host side of the batched workload: seeded descriptors and size classes (no GPU)."""
from distorteddustydiscanalysistoolkits_b200 import batch


def test_c4_descriptors_are_seeded_and_in_range():
    a = batch.c4_discs(64)
    b = batch.c4_discs(64)
    assert a == b and len(a) == 64
    assert all(50_000 <= d["particles"] <= 4_000_000 for d in a)
    assert {d["edge"] for d in a} <= {32, 64, 128, 256}
    assert all(0.0 <= d["tilt"] <= 30.0 for d in a)
    assert len({d["particles"] for d in a}) == 64


def test_size_classes():
    assert batch.size_class(4 ** 5, 4 ** 7) == (5, 7)
    assert batch.size_class(1, 1) == (0, 0)
