// jfg_host.cpp -- host-side copies of device results into caller memory.
#include "jfg_host.h"

#include <cstring>
#include <immintrin.h>

namespace jfg_host {

bool have_avx512() {
#ifdef JFG_HOST_SCALAR  // test builds of the portable path
    return false;
#else
    static const bool v = __builtin_cpu_supports("avx512f");
    return v;
#endif
}

namespace {

// n a multiple of 64 bytes, d 64-byte aligned.
__attribute__((target("avx512f"))) void copy_nt(char *d, const char *s, size_t n) {
    size_t i = 0;
    for (; i + 256 <= n; i += 256) {
        const __m512i a = _mm512_loadu_si512(s + i), b = _mm512_loadu_si512(s + i + 64);
        const __m512i c = _mm512_loadu_si512(s + i + 128), e = _mm512_loadu_si512(s + i + 192);
        _mm512_stream_si512(reinterpret_cast<__m512i *>(d + i), a);
        _mm512_stream_si512(reinterpret_cast<__m512i *>(d + i + 64), b);
        _mm512_stream_si512(reinterpret_cast<__m512i *>(d + i + 128), c);
        _mm512_stream_si512(reinterpret_cast<__m512i *>(d + i + 192), e);
    }
    for (; i < n; i += 64) _mm512_stream_si512(reinterpret_cast<__m512i *>(d + i), _mm512_loadu_si512(s + i));
    _mm_sfence();
}

// Whole 32-entry words; returns the source position after them.  Each word
// is 256 bytes of dst, so a 64-byte-aligned dst stays aligned.
__attribute__((target("avx512f"))) const double *expand_words(double *dst, const double *src, const uint32_t *mask,
                                                               int64_t nw, bool nt) {
    for (int64_t w = 0; w < nw; ++w) {
        const uint32_t m = mask[w];
        for (int g = 0; g < 4; ++g) {
            const __mmask8 k = (__mmask8)(m >> (8 * g));
            const __m512d v = _mm512_maskz_expandloadu_pd(k, src);
            if (nt)
                _mm512_stream_pd(dst, v);
            else
                _mm512_storeu_pd(dst, v);
            src += __builtin_popcount((unsigned)k);
            dst += 8;
        }
    }
    if (nt) _mm_sfence();
    return src;
}

void expand_scalar(double *dst, const double *src, const uint32_t *mask, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        const bool live = (mask[i >> 5] >> (i & 31)) & 1u;
        dst[i] = live ? *src : 0.0;
        src += live ? 1 : 0;
    }
}

}  // namespace

void copy_stream(void *dst, const void *src, size_t bytes) {
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    if (!have_avx512() || bytes < 4096) {
        std::memcpy(d, s, bytes);
        return;
    }
    const size_t head = (64 - (reinterpret_cast<uintptr_t>(d) & 63)) & 63;
    std::memcpy(d, s, head);
    d += head;
    s += head;
    bytes -= head;
    const size_t body = bytes & ~size_t(63);
    copy_nt(d, s, body);
    std::memcpy(d + body, s + body, bytes - body);
}

void expand_stream(double *dst, const double *src, const uint32_t *mask, int64_t n) {
    int64_t done = 0;
    if (have_avx512() && n >= 32) {
        const int64_t nw = n / 32;
        src = expand_words(dst, src, mask, nw, (reinterpret_cast<uintptr_t>(dst) & 63) == 0);
        done = 32 * nw;
    }
    expand_scalar(dst + done, src, mask + done / 32, n - done);
}

}  // namespace jfg_host
