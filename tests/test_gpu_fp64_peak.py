"""tcs_measure_fp64_peak: the FP64 FMA throughput that the bench divides the
line kernels' FP64 arithmetic by (needs a B200)."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp64_peak_is_measured():
    import pascal_tcs_b200 as P
    P.load()
    v = P.measure_fp64_peak(0)
    # B200: about 33 TFLOP/s measured (37-40 nominal); the bounds only catch a broken timing
    assert 5.0 < v < 100.0, v
    assert P.launch_count() > 0


def test_fp64_peak_rejects_bad_device():
    import pascal_tcs_b200 as P
    with pytest.raises(P.TcsError):
        P.measure_fp64_peak(9999)


def test_line_solver_reciprocal_within_an_ulp():
    # qrcp (approximate reciprocal + two Newton-Raphson steps) against the
    # correctly rounded quotient over 10^-6 .. 10^6, both signs
    import pascal_tcs_b200 as P
    P.load()
    err = P.check_reciprocal(1 << 16)
    assert 0.0 <= err <= 1.0, err


def test_fp32_line_solver_reciprocal_within_an_ulp():
    # the FP32 form's reciprocal (approximate + one Newton-Raphson step)
    import pascal_tcs_b200 as P
    P.load()
    err = P.check_reciprocal(1 << 16, fp32=True)
    assert 0.0 <= err <= 1.0, err
