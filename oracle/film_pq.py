"""ORACLE — test infrastructure only (the checker, never the product).

sundog's HDR output encoding of a film, restated in numpy so that a film
rendered here can be compared with sundog's own golden images (12-bit PQ
BT.2020 lossless AVIF, decoded to 8 bits per channel):

  exposure (x 2^exposure) -> BT.709 -> BT.2020 primaries -> linear 1.0 at
  203 cd/m^2 (BT.2408 reference white) -> SMPTE ST 2084 PQ -> 12-bit code
  (src/film.cpp:96-115 `Film::writeAvif`; src/transfer.h:14-50),

then the 12-bit codes scaled to 8 bits as a decoder does for an 8-bit RGB
request (code * 255 / 4095, rounded). The AVIF itself is lossless with an
identity matrix and full range (src/film.cpp:35-48), so its decoded samples
are these codes. Arithmetic in float32 with rounding half away from zero
(lroundf), as the reference's host loop.
"""

import numpy as np

PQ_WHITE_NITS = 203.0
PQ_PEAK_NITS = 10000.0

# SMPTE ST 2084 constants.
M1 = np.float32(2610.0 / 16384.0)
M2 = np.float32(2523.0 / 4096.0 * 128.0)
C1 = np.float32(3424.0 / 4096.0)
C2 = np.float32(2413.0 / 4096.0 * 32.0)
C3 = np.float32(2392.0 / 4096.0 * 32.0)

# Linear BT.709 -> BT.2020 (both D65), ITU-R BT.2087.
BT709_TO_2020 = np.array([[0.627404, 0.329283, 0.043313],
                          [0.069097, 0.919540, 0.011362],
                          [0.016391, 0.088013, 0.895595]], np.float32)


def pq_oetf(lin):
    """Display luminance / 10000 cd/m^2 (clamped to [0, 1]) -> PQ signal."""
    y = np.power(np.clip(lin, 0.0, 1.0).astype(np.float32), M1)
    return np.power((C1 + C2 * y) / (np.float32(1.0) + C3 * y), M2)


def pq_codes12(film, exposure=0.0):
    """12-bit PQ BT.2020 codes of a linear BT.709 film (H x W x >=3)."""
    c = film[..., :3].astype(np.float32) * np.float32(2.0 ** exposure)
    c = c @ BT709_TO_2020.T
    e = pq_oetf(c * np.float32(PQ_WHITE_NITS / PQ_PEAK_NITS))
    return np.floor(e * np.float32(4095.0) + np.float32(0.5)).astype(np.int32)


def codes12_to_8(codes):
    return np.floor(codes.astype(np.float64) * 255.0 / 4095.0 + 0.5).astype(np.uint8)


def pq8(film, exposure=0.0):
    """The film as the 8-bit decode of sundog's HDR AVIF output."""
    return codes12_to_8(pq_codes12(film, exposure))


def psnr(a, b):
    """PSNR in dB of two 8-bit images."""
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(255.0 * 255.0 / mse)
