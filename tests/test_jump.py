"""Jumps in the xoshiro256** stream (dpd_xoshiro_jump, host code of libdpd.so;
no GPU): n draws ahead by the characteristic polynomial equals n serial steps
of the reference's generator (cel/engine/oercel.c:143-174)."""
import numpy as np
import pytest

from oercel_b200._capi import check, load, ptr

M64 = (1 << 64) - 1


def serial(state, n):
    s = [int(v) for v in state]
    for _ in range(n):
        t = (s[1] << 17) & M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = ((s[3] << 45) | (s[3] >> 19)) & M64
    return np.array(s, np.uint64)


@pytest.mark.parametrize("n", [0, 1, 2, 63, 64, 65, 1000, 4097, 12345])
def test_jump_equals_serial_steps(n):
    s0 = np.array([0x0123456789ABCDEF, 0xFEDCBA9876543210, 0x0F1E2D3C4B5A6978, 0x1122334455667788], np.uint64)
    out = np.zeros(4, np.uint64)
    check(load().dpd_xoshiro_jump(ptr(s0), n, ptr(out)))
    assert np.array_equal(out, serial(s0, n))


def test_jumps_compose():
    s0 = np.array([1, 2, 3, 4], np.uint64)
    a, b, c = (np.zeros(4, np.uint64) for _ in range(3))
    lib = load()
    check(lib.dpd_xoshiro_jump(ptr(s0), 2**40 + 17, ptr(a)))
    check(lib.dpd_xoshiro_jump(ptr(a), 2**41 + 5, ptr(b)))
    check(lib.dpd_xoshiro_jump(ptr(s0), 2**40 + 17 + 2**41 + 5, ptr(c)))
    assert np.array_equal(b, c)
