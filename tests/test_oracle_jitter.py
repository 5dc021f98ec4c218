"""The oracle's restatement of the reference's jitter generator (randGPU, Utils.cu:1002-1044):
cuRAND's scrambled Sobol64 points (direction numbers from cuRAND's host API), mapped to
N(0,1) / 4 * radius.  Checked here against an independent statement of the same
mathematics (Gray-code Sobol points in numpy, the normal quantile from scipy) and against
the reference's own quirks; the GPU suite pins it to the reference's kernels."""
import numpy as np
import pytest

import orc

pytest.importorskip("scipy")


def _points_numpy(dirs, scramble32, n_states, first, length):
    """Point (k % 20000) + first + k // 20000 of dimension k % 20000, Gray-code form."""
    out = np.zeros(length, np.uint64)
    for k in range(length):
        i = k % 20000
        n = np.uint64(i + first + k // 20000)
        g = int(n ^ (n >> np.uint64(1)))
        x = np.uint64(scramble32[i])
        b = 0
        while g:
            if g & 1:
                x ^= dirs[i, b]
            g >>= 1
            b += 1
        out[k] = x
    return out


def test_offsets_match_sobol_points_and_normal_quantile():
    from scipy.special import ndtri

    n = orc.max_sample_point(64, 64, 64, 0.5)
    first = 1804289383
    radius = np.float32(0.25)
    got = orc.sobol_offsets(n, first, radius)
    dirs, scr = orc.sobol_tables(n)
    x = _points_numpy(dirs, scr, n, first, n)
    upper = (x >> np.uint64(63)) == 1
    m = np.where(upper, ~x, x)
    q = (m.astype(np.float64) + 0.5) * 2.0 ** -64
    z = np.where(upper, -ndtri(q), ndtri(q))
    want = z / 4.0 * np.float64(radius)
    assert np.abs(got - want).max() <= 1e-12 * np.float64(radius)


def test_offsets_are_normal_with_the_reference_scale():
    n = orc.max_sample_point(512, 512, 512, 0.5)
    got = orc.sobol_offsets(n, 12345, 0.25)
    sigma = 0.25 / 4
    assert abs(got.mean()) < 4 * sigma / np.sqrt(n)
    assert abs(got.std() / sigma - 1) < 0.05


def test_square_launch_grid_leaves_the_tail_unwritten():
    """randGPU's grid of ((round(sqrt(len)) + 31) / 32)^2 blocks of 1024 threads reaches 1024
    of 1050 entries: the last 26 keep their previous values."""
    prev = np.full(1050, 7.0)
    got = orc.sobol_offsets(1050, 3, 0.25, out=prev)
    assert np.all(got[1024:] == 7.0) and np.all(got[:1024] != 7.0)
    got = orc.sobol_offsets(1100, 3, 0.25)  # round(sqrt(1100)) = 33 -> 4 blocks
    assert np.all(got != 0.0)


def test_scramble_words_are_the_32_bit_halves():
    """randGPU copies n * 4 bytes of the 64-bit scramble table into a 32-bit array: state 2k
    takes the low word of constant k and state 2k + 1 its high word."""
    _, s = orc.sobol_tables(8)
    lib_ptr = orc._sobol_tables[2]
    import ctypes as C

    full = np.ctypeslib.as_array(C.cast(lib_ptr, C.POINTER(C.c_uint64)), shape=(4,))
    assert s[0] == (int(full[0]) & 0xFFFFFFFF) and s[1] == (int(full[0]) >> 32)
    assert s[6] == (int(full[3]) & 0xFFFFFFFF) and s[7] == (int(full[3]) >> 32)
