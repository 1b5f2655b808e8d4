"""Real transforms on the CPU: the post-process (R2C) and pre-process (C2R) formulas of
sycl-fft_b200/csrc/real_kernel.cu restated in numpy and checked against numpy.fft.rfft /
irfft in FP64, pair by pair as the kernel walks them (k, H - k); plus the plan API's
argument checks that need no device."""
import numpy as np
import pytest

import syclfft_b200 as sf


def r2c_post(z_spec, n):
    """X[k] = 1/2 [(Z[k] + conj Z[H-k]) - i W_N^k (Z[k] - conj Z[H-k])], k = 0..H, per pair."""
    h = n // 2
    w = np.exp(-2j * np.pi * np.arange(h + 1) / n)
    x = np.zeros(h + 1, np.complex128)

    def post(a, c, wk):
        e = a + np.conj(c)
        d = a - np.conj(c)
        return 0.5 * (e - 1j * wk * d)

    for k in range(h // 2 + 1):
        kk = h - k
        a, c = z_spec[k], z_spec[kk % h]
        x[k] = post(a, c, w[k])
        if kk != k:
            x[kk] = post(c, a, w[kk])
    return x


def c2r_pre(x_spec, n):
    """Z[k] = (X[k] + conj X[H-k]) + i conj(W_N^k) (X[k] - conj X[H-k]), k = 0..H-1."""
    h = n // 2
    w = np.exp(-2j * np.pi * np.arange(h + 1) / n)
    z = np.zeros(h, np.complex128)

    def pre(a, c, wk):
        return (a + np.conj(c)) + 1j * np.conj(wk) * (a - np.conj(c))

    for k in range(h // 2 + 1):
        kk = h - k
        a, c = x_spec[k], x_spec[kk]
        if k == 0:
            z[0] = pre(a.real, c.real, w[0])
        else:
            z[k] = pre(a, c, w[k])
            if kk != k:
                z[kk] = pre(c, a, w[kk])
    return z


@pytest.mark.parametrize("n", [2, 4, 6, 8, 10, 30, 256, 1000, 2018])
def test_r2c_post_process_matches_rfft(n):
    rng = np.random.default_rng(n)
    x = rng.uniform(-1, 1, n)
    z = x[0::2] + 1j * x[1::2]
    got = r2c_post(np.fft.fft(z), n)
    ref = np.fft.rfft(x)
    assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("n", [2, 4, 6, 8, 10, 30, 256, 1000, 2018])
def test_c2r_pre_process_is_the_unnormalized_inverse(n):
    rng = np.random.default_rng(n + 1)
    h = n // 2
    spec = rng.uniform(-1, 1, h + 1) + 1j * rng.uniform(-1, 1, h + 1)
    z = np.fft.ifft(c2r_pre(spec, n)) * h          # unnormalized inverse of length H
    got = np.empty(n)
    got[0::2], got[1::2] = z.real, z.imag
    clean = spec.copy()
    clean[0] = clean[0].real                        # imaginary parts of DC and Nyquist ignored
    clean[h] = clean[h].real
    ref = np.fft.irfft(clean, n) * n
    assert np.max(np.abs(got - ref)) <= 1e-12 * n
    # and numpy's irfft ignores them too, so the results agree on the raw spectrum
    assert np.max(np.abs(got - np.fft.irfft(spec, n) * n)) <= 1e-12 * n


def test_real_plan_argument_checks_need_no_device():
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_r2c_1d("float", 7)
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_c2r_1d("half", 8)
    assert e.value.code == sf.error_code.unsupported_precision
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_r2c_1d("float", 8, 0)
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_r2c_1d("float", 8, 1, sf.plan_options(placement=sf.placement.in_place))
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        sf.RealPlan("float", 8, 1, "r2r")
    assert e.value.code == sf.error_code.invalid_argument


def _catalog(path, macro):
    """Entries X(...) of a catalog macro, as tuples of ints."""
    import os
    import re
    src = open(os.path.join(os.path.dirname(__file__), "..", "sycl-fft_b200", "csrc", path)).read()
    body = src[src.index("#define " + macro):]
    body = body[: body.index("\n\n")]
    return [tuple(int(v) for v in m.split(",")) for m in re.findall(r"X\(([-0-9, ]+)\)", body)]


def test_fused_real_catalog_matches_the_line_kernels():
    """Each one-pass real kernel (real_kernel.cu) is the size-specialised line kernel of its half
    length (fixed_catalog.h, contiguous lines, plain feature): same threads per line, same
    radices, radices multiplying to the length; its lines per CTA fit the CTA-size bound."""
    fixed = {(e[1], e[4]): e for e in _catalog("fixed_catalog.h", "SFB_FIXED_CATALOG") if e[2] == 0 and e[3] == 0}
    fused = _catalog("real_kernel.cu", "SFB_REAL_FUSED_CATALOG")
    assert fused
    for e in fused:
        _, dbl, h, tpl, maxt, *radices = e
        f = fixed[(dbl, h)]
        assert (f[5], list(f[8:])) == (tpl, radices), e
        prod = 1
        for r in radices:
            prod *= r
        assert prod == h and maxt % tpl == 0 and maxt // tpl >= 1


def test_multidimensional_real_plan_argument_checks():
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_r2c("float", [4, 7])            # odd last length
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_c2r("double", [2, 2, 2, 2])     # rank 4
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_r2c("float", [0, 8])
    assert e.value.code == sf.error_code.invalid_argument
