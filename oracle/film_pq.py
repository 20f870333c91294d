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
    """12-bit PQ BT.2020 codes of a linear BT.709 film (H x W x >=3), each
    FP32 operation in the reference's order (no fused multiply-adds)."""
    f = np.float32
    c = film[..., :3].astype(np.float32) * f(2.0 ** exposure)
    x, y, z = c[..., 0], c[..., 1], c[..., 2]
    m = BT709_TO_2020
    rgb = np.stack([(m[r, 0] * x + m[r, 1] * y) + m[r, 2] * z for r in range(3)], -1)
    e = pq_oetf(rgb * f(PQ_WHITE_NITS / PQ_PEAK_NITS)) * f(4095.0)
    # lroundf: the FP32 value widened exactly to FP64, half away from zero.
    return np.floor(e.astype(np.float64) + 0.5).astype(np.int32)


def read_pq16_png(path):
    """(codes, cicp) of a 16-bit RGB PNG written by the renderer: the 12-bit
    codes (top 12 bits of each sample) as (H, W, 3) int32, and the cICP chunk
    bytes (None if absent). Reads only what that writer emits: non-interlaced
    RGB16 with filter type 0 rows."""
    import struct
    import zlib
    with open(path, "rb") as fh:
        data = fh.read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n", "not a PNG"
    return _read_png_chunks(data, struct, zlib)


def _read_png_chunks(data, struct, zlib):
    pos, idat, cicp, w, h = 8, b"", None, 0, 0
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if kind == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 16 and ctype == 2, "expected 16-bit RGB"
        elif kind == b"cICP":
            cicp = tuple(body)
        elif kind == b"IDAT":
            idat += body
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + w * 6)
    assert np.all(raw[:, 0] == 0), "expected filter type 0 rows"
    px = raw[:, 1:].reshape(h, w * 3, 2).astype(np.int32)
    v = (px[..., 0] << 8) | px[..., 1]
    return (v >> 4).reshape(h, w, 3), cicp


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
