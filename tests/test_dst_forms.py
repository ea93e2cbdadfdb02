"""The two DST-I forms of the transform kernels, restated in numpy and checked on the CPU.

The reference takes every line's DST-I from FFTW's RODFT00 (src/EllipticSolver2d.cc:57-85):
y_k = 2 sum_{j=1}^{N-1} f_j sin(pi j k / N), k = 1 .. N-1.  The kernels (ibpm_b200/csrc/elliptic.cu)
pack two real lines a, b into one complex FFT and take the DST in one of two forms:

* odd extension (k_dst_rows / k_dst_cols with H = false): the FFT of length 2N of
  [0, f_1 .. f_{N-1}, 0, -f_{N-1} .. -f_1] is -2i times the sine sums, so line a's DST is -Im and
  line b's is Re of outputs 1 .. N-1;
* half length (H = true, FP64 plans; dst_pre, dst_post): the FFT of length N of
  y_j = s_j (f_j + f_{N-j}) + (f_j - f_{N-j}) / 2, s_j = sin(pi j / N).  Its imaginary parts give
  the even outputs directly (2 S_k = y_{2k}); its real parts R_k satisfy
  y_{2k+1} - y_{2k-1} = 2 R_k (from 2 sin(a) cos(b) = sin(a + b) - sin(b - a)), so the odd outputs are
  the prefix sum R_0, R_0 + 2 R_1, ...

These tests hold both restatements, in the kernels' index arithmetic (the unpacking of the two lines
from Z_k and Z_{N-k}, the k ranges for odd and even N), to scipy's DST-I; they need no GPU.
"""
import numpy as np
import pytest
import scipy.fft


def dst1_odd_pair(a, b):
    """k_dst_rows / k_dst_cols, odd extension: two lines of n = N - 1 values -> their DST-I."""
    n = a.size
    N = n + 1
    z = np.zeros(2 * N, complex)
    z[1:N] = a + 1j * b
    z[N + 1:] = -(a + 1j * b)[::-1]
    G = np.fft.fft(z)[1:N]
    return -G.imag, G.real


def dst1_half_pair(a, b):
    """k_dst_rows / k_dst_cols, half length: dst_pre, one FFT of length N, dst_post."""
    n = a.size
    N = n + 1
    f = np.zeros(N + 1, complex)  # f_0 = f_N = 0
    f[1:N] = a + 1j * b
    j = np.arange(1, N)
    s = np.sin(np.pi * j / N)
    # dst_pre on each line (real and imaginary parts separately, as the kernel does)
    fj, fn = f[j], f[N - j]
    y = np.zeros(N, complex)
    y[1:] = s * (fj.real + fn.real) + 0.5 * (fj.real - fn.real) + 1j * (s * (fj.imag + fn.imag) + 0.5 * (fj.imag - fn.imag))
    Z = np.fft.fft(y)
    half, kh = N // 2, (N + 1) // 2
    out_a = np.zeros(n)
    out_b = np.zeros(n)
    terms_a, terms_b = [], []
    for k in range(kh):
        zk, zn = Z[k], Z[0 if k == 0 else N - k]
        ca, cb = 0.5 * (zk.real + zn.real), 0.5 * (zk.imag + zn.imag)
        if k >= 1:  # output 2k (1-based) at 2k - 1
            out_a[2 * k - 1] = zn.imag - zk.imag
            out_b[2 * k - 1] = zk.real - zn.real
        if k < half:
            terms_a.append(ca if k == 0 else 2 * ca)
            terms_b.append(cb if k == 0 else 2 * cb)
    # output 2k + 1 (1-based) at 2k: the prefix sums (the kernel scans them in 32-wide segments)
    out_a[0:2 * half:2] = np.cumsum(terms_a)
    out_b[0:2 * half:2] = np.cumsum(terms_b)
    return out_a, out_b


# every line length of the benchmark grids' FFT lengths, odd and even N, and small and prime cases
LENGTHS = list(range(1, 70)) + [99, 127, 128, 191, 199, 249, 255, 383, 399, 499, 511, 767, 799, 999, 1023]


@pytest.mark.parametrize("form", [dst1_odd_pair, dst1_half_pair], ids=["odd_extension", "half_length"])
@pytest.mark.parametrize("n", LENGTHS)
def test_dst_form_matches_rodft00(form, n):
    rng = np.random.default_rng(n)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    ya, yb = form(a, b)
    ra, rb = scipy.fft.dst(a, type=1), scipy.fft.dst(b, type=1)
    scale = max(np.abs(ra).max(), np.abs(rb).max(), 1.0)
    assert np.abs(ya - ra).max() <= 1e-12 * scale * max(1.0, np.log2(n + 1))
    assert np.abs(yb - rb).max() <= 1e-12 * scale * max(1.0, np.log2(n + 1))


def test_half_length_is_its_own_inverse_up_to_scale():
    """DST-I applied twice is 2N times the identity; the solves rely on it (the inverse pass is the
    forward pass with the eigenvalue scaling and 1 / 2N folded in)."""
    rng = np.random.default_rng(7)
    for n in (127, 199, 255):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        ya, yb = dst1_half_pair(a, b)
        za, zb = dst1_half_pair(ya, yb)
        assert np.allclose(za / (2 * (n + 1)), a, atol=1e-12)
        assert np.allclose(zb / (2 * (n + 1)), b, atol=1e-12)
