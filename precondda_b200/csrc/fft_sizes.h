// FFT lengths with compiled transform kernels.  Every entry is even and
// factors into 2, 3 and 5; the engine pads each box axis n to the
// smallest listed L >= 2n (or to any listed L the caller picks).
#pragma once

#define DDA_FFT_SIZES(X) \
  X(8) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(72) X(80) X(96) X(128) X(144) X(160) X(192) X(256) \
  X(288) X(320) X(384) X(512)

namespace dda {
inline bool fft_size_compiled(int L) {
  switch (L) {
#define DDA_CASE(n) case n:
    DDA_FFT_SIZES(DDA_CASE)
#undef DDA_CASE
    return true;
    default: return false;
  }
}
}  // namespace dda
