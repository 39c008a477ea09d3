"""The oracle's FFT and convolution against the reference's own known-answer tests
(crates/sr-physics/src/reference/fft.rs:285-548): each case here restates one of those tests with its tolerance."""
import numpy as np
import pytest

import oracle as O

MASK = (1 << 64) - 1


def pseudo_random(count, seed):
    """The reference tests' 64-bit LCG in [-1, 1) (fft.rs:290-300)."""
    s = seed
    out = np.empty(count)
    for i in range(count):
        s = (s * 6364136223846793005 + 1442695040888963407) & MASK
        out[i] = ((s >> 11) / float(1 << 53)) * 2.0 - 1.0
    return out


def pseudo_complex(count, seed):
    v = pseudo_random(2 * count, seed)
    return v[0::2] + 1j * v[1::2]


def direct_dft(x, inverse):
    n = len(x)
    sign = 1.0 if inverse else -1.0
    k = np.arange(n)
    ang = sign * 2.0 * np.pi * ((np.outer(k, k)) % n) / n
    out = (np.exp(1j * ang) * x[None, :]).sum(axis=1)
    return out / n if inverse else out


def rel_err(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 32, 64, 128])
def test_fft_matches_the_direct_dft(n):
    x = pseudo_complex(n, 7 + n)
    for inverse in (False, True):
        assert rel_err(O.fft(x, inverse), direct_dft(x, inverse)) < 1e-12


def test_fft_of_a_delta_and_a_wave_are_exact():
    d = np.zeros(16, complex)
    d[0] = 1.0
    y = O.fft(d)
    assert np.all(np.abs(y.real - 1.0) < 1e-15) and np.all(np.abs(y.imag) < 1e-15)
    wave = np.exp(2j * np.pi * 3.0 * np.arange(16) / 16.0)
    y = O.fft(wave)
    want = np.where(np.arange(16) == 3, 16.0, 0.0)
    assert np.all(np.abs(y.real - want) < 1e-12) and np.all(np.abs(y.imag) < 1e-12)


def test_inverse_undoes_forward_in_1d_and_2d():
    for n in (32, 256, 2048):
        x = pseudo_complex(n, 3)
        assert rel_err(O.fft(O.fft(x), True), x) < 1e-13
    x = pseudo_complex(64 * 32, 5).reshape(32, 64)
    assert rel_err(O.fft2(O.fft2(x), True), x) < 1e-13


def test_fft2_matches_the_direct_2d_dft_and_obeys_parseval():
    nx, ny = 16, 8
    x = pseudo_complex(nx * ny, 11).reshape(ny, nx)
    y = O.fft2(x)
    direct = np.zeros((ny, nx), complex)
    jy, jx = np.mgrid[0:ny, 0:nx]
    for ky in range(ny):
        for kx in range(nx):
            phase = ((kx * jx) % nx) / nx + ((ky * jy) % ny) / ny
            direct[ky, kx] = (x * np.exp(-2j * np.pi * phase)).sum()
    assert rel_err(y, direct) < 1e-12
    space = (np.abs(x) ** 2).sum()
    freq = (np.abs(y) ** 2).sum() / (nx * ny)
    assert abs((space - freq) / space) < 1e-13


def test_parseval_holds_at_the_largest_size():
    x = pseudo_complex(2048, 17)
    y = O.fft(x)
    space = (np.abs(x) ** 2).sum()
    freq = (np.abs(y) ** 2).sum() / 2048.0
    assert abs((space - freq) / space) < 1e-13


def asymmetric_kernel(dx, dy):
    """The reference tests' kernel with no symmetry in either axis (fft.rs:432-437)."""
    x, y = float(dx), float(dy)
    return (1.0 + 0.5 * np.tanh(0.2 * x) + 0.3 * np.tanh(0.1 * y)) / np.sqrt(1.0 + x * x + 2.0 * y * y)


def ktab_for(w, h, kernel):
    px, py = O.padded_size(w), O.padded_size(h)
    t = np.zeros((py, px))
    for j in range(py):
        for i in range(px):
            dx = i if i < px // 2 else i - px
            dy = j if j < py // 2 else j - py
            t[j, i] = kernel(dx, dy)
    return t


def direct_convolution(field, kernel):
    h, w = field.shape
    out = np.zeros((h, w))
    for ty in range(h):
        for tx in range(w):
            s = 0.0
            for sy in range(h):
                dy = ty - sy
                s += sum(kernel(tx - sx, dy) * field[sy, sx] for sx in range(w) if field[sy, sx] != 0.0)
            out[ty, tx] = s
    return out


def direct_convolution_fast(field, kernel):
    h, w = field.shape
    dx = np.arange(-(w - 1), w)
    dy = np.arange(-(h - 1), h)
    K = np.array([[kernel(a, b) for a in dx] for b in dy])
    out = np.zeros((h, w))
    for ty in range(h):
        for tx in range(w):
            sub = K[ty - np.arange(h)[:, None] + h - 1, tx - np.arange(w)[None, :] + w - 1]
            out[ty, tx] = (sub * field).sum()
    return out


def test_convolution_matches_direct_summation_on_48_by_40_with_an_asymmetric_kernel():
    w, h = 48, 40
    assert asymmetric_kernel(5, 3) != asymmetric_kernel(-5, 3)
    field = (pseudo_random(w * h, 29) + 1.0).reshape(h, w)
    fast = O.convolve_ringed(field, ktab_for(w, h, asymmetric_kernel))
    direct = direct_convolution_fast(field, asymmetric_kernel)
    assert np.abs(fast - direct).max() / np.abs(direct).max() < 1e-10
    for x in range(w):
        for y in (0, h - 1):
            assert abs((fast[y, x] - direct[y, x]) / direct[y, x]) < 1e-10
    for y in range(h):
        for x in (0, w - 1):
            assert abs((fast[y, x] - direct[y, x]) / direct[y, x]) < 1e-10


def test_mass_in_the_corners_does_not_wrap_around():
    w, h = 40, 33
    field = np.zeros((h, w))
    for x, y in ((0, 0), (w - 1, 0), (0, h - 1), (w - 1, h - 1)):
        field[y, x] = 1.0
    fast = O.convolve_ringed(field, ktab_for(w, h, asymmetric_kernel))
    direct = direct_convolution_fast(field, asymmetric_kernel)
    assert np.abs(fast - direct).max() / np.abs(direct).max() < 1e-10


def test_a_single_source_reproduces_the_kernel_shifted():
    w, h, sx, sy = 20, 17, 6, 11
    field = np.zeros((h, w))
    field[sy, sx] = 2.5
    out = O.convolve_ringed(field, ktab_for(w, h, asymmetric_kernel))
    for y in range(h):
        for x in range(w):
            want = 2.5 * asymmetric_kernel(x - sx, y - sy)
            assert abs(out[y, x] - want) < 1e-12 * max(abs(want), 1.0)


def test_padded_sizes_follow_the_box_rule_and_refuse_out_of_range_boxes():
    for n, want in ((1, 32), (16, 32), (17, 64), (32, 64), (48, 128), (64, 128), (300, 1024), (1024, 2048)):
        assert O.padded_size(n) == want
    assert O.padded_size(0) == 0
    assert O.padded_size(1025) == 0
    # this build lifts the cap: a 2048 axis pads to 4096
    assert O.padded_size(2048, 4096) == 4096
    with pytest.raises(ValueError):
        O.fft(np.zeros(48, complex))
