// jfg_host.h -- host-side copies of device results into caller memory
// (compiled by the host compiler from jfg_host.cpp).
#pragma once
#include <cstddef>
#include <cstdint>

namespace jfg_host {

// True when the CPU executes AVX-512F (checked once).
bool have_avx512();

// memcpy of a large block whose destination the caller reads later: with
// AVX-512 the 64-byte-aligned body is written with non-temporal stores (no
// read-for-ownership of the destination lines, which halves the memory
// traffic of a pageable destination), followed by a store fence.
void copy_stream(void *dst, const void *src, size_t bytes);

// Expansion of a compacted value stream: mask bit l of word w says whether
// entry 32 w + l is live.  Writes entries [32 w0, 32 w0 + n) of dst: live
// entries take the next value of src (in order), the others +0.0.  dst points
// at entry 32 w0, mask at word w0, src at the first value of word w0.
void expand_stream(double *dst, const double *src, const uint32_t *mask, int64_t n);

}  // namespace jfg_host
