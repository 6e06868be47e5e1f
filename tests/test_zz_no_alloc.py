"""kd_count_radii_static: the count for callers that cannot allocate device
memory while they count (a fixed-budget memory pool owns the device, or a
cudaMalloc would synchronize the device and stall other work).  Its buffers
come from one static device array; its counts must equal kd_count_radii's
exactly, call after call, with the shared array's leftover contents from the
previous call never leaking into the next one.

Kept in its own file, collected last, so a failure here never hides the rest
of the suite; it passes alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

from corruscant_b200 import _native as N

pytestmark = pytest.mark.gpu


def _catalog(seed, n, nparents, sigma, nf):
    rs = np.random.RandomState(seed)
    c = rs.rand(nparents, 3)
    p = (c[rs.randint(0, nparents, n)] + rs.normal(0, sigma, (n, 3))) % 1.0
    f = (p[:, 0] * nf).astype(np.int32).clip(0, nf - 1)
    return N.build_tree(np.ascontiguousarray(p), f, nf)


def test_static_scratch_count_matches_allocating_count_on_consecutive_calls():
    # a 2M-point tree queried with itself needs several batches of tile
    # records in the 32 MiB array; a small clustered pair runs in one
    big = N.build_tree(np.random.RandomState(7).rand(2_000_000, 3), None, 1)
    a = _catalog(8, 40_000, 400, 0.01, 4)
    b = _catalog(9, 60_000, 600, 0.02, 4)
    radii_big = np.logspace(-3, -1.3, 9)
    radii_ab = np.array([0.0, 0.004, np.nan, 0.01, 0.03, 0.06, 0.06, np.inf])
    try:
        want_big = N.count_radii(big, big, radii_big)
        want_ab = N.count_radii(a, b, radii_ab)
        want_ba = N.count_radii(b, a, radii_ab, mode=N.KD_MODE_FP64)
        for _ in range(2):
            assert np.array_equal(N.count_radii_static(big, big, radii_big), want_big)
            assert np.array_equal(N.count_radii_static(a, b, radii_ab), want_ab)
            assert np.array_equal(N.count_radii_static(b, a, radii_ab, mode=N.KD_MODE_FP64),
                                  want_ba)
    finally:
        for t in (big, a, b):
            N.destroy(t)


def _fields_catalog(seed, n, ids, num_fields, axis):
    """Clustered points whose field ids run over 0 .. ids-1 in slabs along
    one axis, declared with num_fields fields (the reference's counter is
    qfield * Fq + tfield, so with Fq != Ft several (qfield, tfield) pairs
    share one slot)."""
    rs = np.random.RandomState(seed)
    c = rs.rand(n // 100, 3)
    p = (c[rs.randint(0, len(c), n)] + rs.normal(0, 0.01, (n, 3))) % 1.0
    f = np.minimum((p[:, axis] * ids).astype(np.int32), ids - 1)
    return N.build_tree(np.ascontiguousarray(p), f, num_fields)


def test_static_scratch_count_with_unequal_field_counts():
    # query 2 fields / tree 3 fields: slots qf*2 + tf, (0,2) and (1,0) share
    # slot 2; query declared with 3 fields but ids 0..1 against a 2-field tree
    # query fields in slabs along x, tree fields along y: every (qfield,
    # tfield) combination has close pairs
    q2 = _fields_catalog(21, 30_000, 2, 2, 0)
    t3 = _fields_catalog(22, 50_000, 3, 3, 1)
    q3 = _fields_catalog(23, 30_000, 2, 3, 0)
    t2 = _fields_catalog(24, 50_000, 2, 2, 1)
    radii = np.array([0.002, 0.01, 0.02, 0.05])
    try:
        cases = [(t3, q2), (t2, q3)]
        want = [N.count_radii(t, q, radii) for t, q in cases]
        for _ in range(2):
            for (t, q), w in zip(cases, want):
                for mode in (N.KD_MODE_MIXED, N.KD_MODE_FP64):
                    assert np.array_equal(N.count_radii_static(t, q, radii, mode=mode), w)
        # slot 2 of the 2 x 3 layout really holds two field pairs
        assert want[0][:, 2].sum() > 0
    finally:
        for t in (q2, t3, q3, t2):
            N.destroy(t)


def test_static_scratch_count_rejects_what_does_not_fit():
    t = _catalog(10, 5000, 50, 0.01, 2)
    try:
        with pytest.raises(N.NativeError):
            N.count_radii_static(t, t, np.linspace(0.01, 0.2, 65))  # more than 64 radii
        with pytest.raises(N.NativeError):
            N.count_radii_static(t, t, [-0.1])
    finally:
        N.destroy(t)
