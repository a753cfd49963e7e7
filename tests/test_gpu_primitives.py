"""The primitive bindings of riptide.libcpp -- rollback, fused_rollback_add,
circular_prefix_sum (python_bindings.cpp:44-81), benchmark_ffa2 (:99-118) and snr1
(:121-138) -- through the C ABI, bit for bit against the reference's own module built from its
sources (the C restatement where it is absent). circular_prefix_sum with nsum > size is
compared with the C restatement only: the reference's binding sizes its output like the
input and writes past it."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import riptide_b200

    return riptide_b200


@pytest.fixture(scope="module")
def ref():
    return O.ref_libcpp()


SIZES = [1, 2, 7, 240, 257, 4096, 100003]


def test_rollback(rb, ref):
    rng = np.random.default_rng(1)
    for size in SIZES:
        x = rng.standard_normal(size).astype(np.float32)
        for shift in sorted({0, 1, 5, size - 1, size, size + 3, 3 * size + 11}):
            want = ref.rollback(x, shift) if ref is not None else np.roll(x, -shift)
            assert np.array_equal(rb.libcpp.rollback(x, shift), want), (size, shift)
    with pytest.raises(ValueError, match="contiguous"):
        rb.libcpp.rollback(np.zeros(8, np.float32)[::2], 1)


def test_fused_rollback_add(rb, ref):
    rng = np.random.default_rng(2)
    for size in SIZES:
        x = rng.standard_normal(size).astype(np.float32)
        y = rng.standard_normal(size).astype(np.float32)
        for shift in sorted({0, 1, 5, size - 1, size, 2 * size + 7}):
            got = rb.libcpp.fused_rollback_add(x, y, shift)
            if ref is not None:
                want = ref.fused_rollback_add(x, y, shift)
            else:
                want = (x + np.roll(y, -shift)).astype(np.float32)
            assert np.array_equal(got, want), (size, shift)
    with pytest.raises(ValueError, match="same number of elements"):
        rb.libcpp.fused_rollback_add(np.zeros(4, np.float32), np.zeros(5, np.float32), 1)


@pytest.mark.parametrize("size,nsum", [(1, 1), (10, 3), (10, 10), (257, 257), (260, 140),
                                       (300000, 300000), (1000003, 999999)])
def test_circular_prefix_sum_first_wrap(rb, ref, size, nsum):
    # nsum <= size: the double accumulator in the reference's order. Random data of this
    # length needs more than 53 bits for some partial sums, so the rounding order matters.
    x = (np.random.default_rng(size).standard_normal(size) * 3).astype(np.float32)
    got = rb.libcpp.circular_prefix_sum(x, nsum)
    assert got.shape == (nsum,)
    want = ref.circular_prefix_sum(x, nsum)[:nsum] if ref is not None else O.C().circular_prefix_sum(x, nsum)
    assert np.array_equal(got, want)
    assert np.array_equal(got, O.C().circular_prefix_sum(x, nsum))


@pytest.mark.parametrize("size,nsum", [(240, 282), (260, 302), (100, 1050), (7, 100), (1, 5),
                                       (4096, 3 * 4096 + 5)])
def test_circular_prefix_sum_wraps(rb, size, nsum):
    # several wraps: out[i*size + j] = out[j] + float(i) * float(total)
    x = np.random.default_rng(nsum).standard_normal(size).astype(np.float32)
    assert np.array_equal(rb.libcpp.circular_prefix_sum(x, nsum), O.C().circular_prefix_sum(x, nsum))


def test_circular_prefix_sum_edge_cases(rb):
    assert rb.libcpp.circular_prefix_sum(np.ones(5, np.float32), 0).shape == (0,)
    with pytest.raises(ValueError):
        rb.libcpp.circular_prefix_sum(np.zeros(0, np.float32), 3)


def test_snr1(rb, ref):
    rng = np.random.default_rng(3)
    for b, widths in [(240, O.generate_width_trials(240)), (257, O.generate_width_trials(257)),
                      (64, np.arange(1, 64)), (33, [1, 5, 7, 32]), (1000, [3, 30, 300])]:
        x = (rng.standard_normal(b) * 2).astype(np.float32)
        w = np.asarray(widths, dtype=np.uint64)
        for stdnoise in (1.0, 0.37):
            got = rb.libcpp.snr1(x, w, stdnoise)
            want = (ref.snr1(x, w, stdnoise) if ref is not None
                    else O.C().snr2(x.reshape(1, -1), w, stdnoise)[0])
            assert np.array_equal(got, want), (b, stdnoise)
    with pytest.raises(ValueError):
        rb.libcpp.snr1(np.zeros(32, np.float32), np.asarray([1, 32], np.uint64))
    with pytest.raises(ValueError):
        rb.libcpp.snr1(np.zeros(32, np.float32), np.asarray([1, 2], np.uint64), -1.0)


def test_benchmark_ffa2(rb, ref):
    # seconds per transform of a zero block, as the reference's benchmark reports
    for rows, cols in [(1024, 256), (2684, 250), (37, 240)]:
        t = rb.libcpp.benchmark_ffa2(rows, cols, 10)
        assert isinstance(t, float) and 0.0 < t < 1.0
        if ref is not None:
            assert ref.benchmark_ffa2(rows, cols, 2) > 0.0
    assert rb.libcpp.benchmark_ffa2(0, 256, 3) == 0.0
