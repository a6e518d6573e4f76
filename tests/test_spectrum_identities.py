"""The algebra the refresh kernel's FFT stages rely on, checked in FP64 with
numpy on the CPU: the residue split of the packed transform, the unpacking of
the real spectrum from Z[k] and Z[Nh - k] (with the mirror bin's twiddle), and
the folding of a pair's W_L factor into its twist.  The kernel itself is
checked against the oracle by the GPU parity tests; these pin the identities
that its index and twiddle arithmetic encode."""
import numpy as np
import pytest


def _w(n, e):
    """exp(-2 pi i e / n)"""
    return np.exp(-2j * np.pi * np.asarray(e, dtype=np.float64) / n)


@pytest.mark.parametrize("nfft,L", [(64, 8), (256, 16), (1024, 128), (4096, 4096), (8192, 256)])
def test_residue_split_of_the_packed_transform(nfft, L):
    # a window of up to 2L real samples, zero-padded to nfft, packed two per
    # complex point: Z[Mq + r] = FFT_L(y_r)[q], y_r[n] = z[n] W_Nh^{rn}
    rng = np.random.default_rng(nfft + L)
    nh = nfft // 2
    L = min(L, nh)
    m_res = nh // L
    x = np.zeros(nfft)
    x[: min(2 * L, nfft)] = rng.standard_normal(min(2 * L, nfft))
    z = x[0::2] + 1j * x[1::2]
    zfull = np.fft.fft(z)
    n = np.arange(L)
    for r in range(m_res):
        y = z[:L] * _w(nh, r * n)
        assert np.allclose(np.fft.fft(y), zfull[r::m_res], atol=1e-9)


@pytest.mark.parametrize("nfft", [16, 128, 2048, 1 << 14])
def test_real_spectrum_unpacked_from_mirrored_pair(nfft):
    # X[k] = E + W D and X[Nh - k] = conj(E - W D), W = W_Nfft^k,
    # E = (Z[k] + conj Z[Nh-k]) / 2, D = (Z[k] - conj Z[Nh-k]) / 2i
    rng = np.random.default_rng(nfft)
    x = rng.standard_normal(nfft)
    nh = nfft // 2
    big_x = np.fft.fft(x)
    zf = np.fft.fft(x[0::2] + 1j * x[1::2])
    k = np.arange(1, nh)
    a, b = zf[k], zf[nh - k]
    e = (a + np.conj(b)) / 2
    d = (a - np.conj(b)) / 2j
    wk = _w(nfft, k)
    assert np.allclose(e + wk * d, big_x[k], atol=1e-8)
    assert np.allclose(np.conj(e - wk * d), big_x[nh - k], atol=1e-8)
    # the same with the partner bin's own twiddle, -conj(W_Nfft^k)
    wm = _w(nfft, nh - k)
    assert np.allclose(wm, -np.conj(wk), atol=1e-12)
    dm = (b - np.conj(a)) / 2j
    assert np.allclose((np.conj(a) + b) / 2 + wm * dm, big_x[nh - k], atol=1e-8)
    # k = 0 gives the DC and Nyquist bins: X[0] = Re Z0 + Im Z0, X[Nh] = Re Z0 - Im Z0
    assert np.isclose(zf[0].real + zf[0].imag, big_x[0])
    assert np.isclose(zf[0].real - zf[0].imag, big_x[nh])


@pytest.mark.parametrize("m_res,L", [(8, 16), (32, 8), (4, 1024)])
def test_mirror_twiddle_of_partner_residue(m_res, L):
    # residues r and M - r: W_Nfft^{M - r} W_2L^{L-1-q} = -conj(W_Nfft^r W_2L^q)
    nfft = 2 * m_res * L
    q = np.arange(L)
    for r in range(1, m_res // 2 + 1):
        w0 = _w(nfft, r) * _w(2 * L, q)
        w1 = _w(nfft, m_res - r) * _w(2 * L, L - 1 - q)
        assert np.allclose(w1, -np.conj(w0), atol=1e-12)
    # the rotation by W_2L from q to q + 1 is the step of W_Nfft^k from k to k + M
    assert np.isclose(_w(nfft, m_res), _w(2 * L, 1))


def test_pair_twist_folds_the_w_l_factor():
    # z conj(W_Nh^{rn}) W_L^n = z conj(t2) with t2 = W_Nh^{rn} conj(W_L^n),
    # and t2 steps by the same product of the two steps
    rng = np.random.default_rng(7)
    nh, L, r = 512, 64, 3
    n = np.arange(0, L, 4)
    z = rng.standard_normal(n.size) + 1j * rng.standard_normal(n.size)
    t = _w(nh, r * n)
    pf = _w(L, n)
    t2 = t * np.conj(pf)
    assert np.allclose(z * np.conj(t) * pf, z * np.conj(t2))
    step = _w(nh, r * 4) * np.conj(_w(L, 4))
    assert np.allclose(t2[1:], t2[:-1] * step)
