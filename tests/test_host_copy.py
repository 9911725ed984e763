"""Host-side copy routines of the library (csrc/jfg_host.cpp), on the CPU.

copy_stream must equal memcpy for every length and alignment (its AVX-512
body uses non-temporal stores between an unaligned head and tail), and
expand_stream must place each live value of a compacted stream at its masked
position with +0.0 elsewhere, for whole and partial 32-entry words, with the
vector path and the scalar tail.  The routines are compiled here with g++
into a small test library with C entry points.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "jf_2026_05_19_b200", "csrc")

WRAP = r'''
#include "jfg_host.h"
extern "C" {
void t_copy(void *d, const void *s, size_t n) { jfg_host::copy_stream(d, s, n); }
void t_expand(double *d, const double *s, const uint32_t *m, int64_t n) { jfg_host::expand_stream(d, s, m, n); }
int t_avx512() { return jfg_host::have_avx512() ? 1 : 0; }
}
'''


@pytest.fixture(scope="module", params=["vector", "scalar"])
def lib(tmp_path_factory, request):
    """The routines as the library builds them (AVX-512 where the CPU has it) and
    with the portable path forced."""
    d = tmp_path_factory.mktemp("hostcopy_" + request.param)
    w = d / "wrap.cpp"
    w.write_text(WRAP)
    so = d / "libt.so"
    flags = ["-DJFG_HOST_SCALAR"] if request.param == "scalar" else []
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", *flags, "-I", CSRC, str(w),
                    os.path.join(CSRC, "jfg_host.cpp"), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    L.t_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    L.t_expand.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
    return L


def test_copy_stream_equals_memcpy(lib):
    rng = np.random.default_rng(0)
    src = rng.integers(0, 256, 1 << 20, dtype=np.uint8)
    for n in (0, 1, 63, 4095, 4096, 4097, 65536 + 17, (1 << 20) - 200):
        for off_d in (0, 8, 13, 64):
            for off_s in (0, 3):
                dst = np.zeros((1 << 20) + 256, np.uint8)
                lib.t_copy(dst.ctypes.data + off_d, src.ctypes.data + off_s, n)
                assert np.array_equal(dst[off_d:off_d + n], src[off_s:off_s + n]), (n, off_d, off_s)
                assert not dst[:off_d].any() and not dst[off_d + n:].any()


@pytest.mark.parametrize("n", [1, 31, 32, 33, 96, 1000, 4096 + 7])
@pytest.mark.parametrize("off", [0, 1, 8])
def test_expand_stream_places_live_values(lib, n, off):
    rng = np.random.default_rng(n + off)
    # a shell-like pattern (three live, three dead) mixed with random words and whole live/dead words
    live = np.tile([1, 1, 1, 0, 0, 0], n // 6 + 1)[:n].astype(bool)
    live ^= rng.random(n) < 0.1
    if n > 200:
        live[64:96] = True
        live[128:160] = False
    words = np.zeros((n + 31) // 32, np.uint32)
    for i in np.nonzero(live)[0]:
        words[i >> 5] |= np.uint32(1) << np.uint32(i & 31)
    vals = rng.standard_normal(int(live.sum()))
    vals[vals == 0.0] = 1.0
    buf = np.full(n + off + 8, np.nan)
    lib.t_expand(buf.ctypes.data + 8 * off, vals.ctypes.data, words.ctypes.data, n)
    out = buf[off:off + n]
    want = np.zeros(n)
    want[live] = vals
    assert np.array_equal(out, want)
    assert not np.signbit(out[~live]).any()                       # dead entries are +0.0
    assert np.isnan(buf[:off]).all() and np.isnan(buf[off + n:]).all()   # nothing outside the range
