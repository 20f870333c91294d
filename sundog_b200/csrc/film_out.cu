// HDR output encoding of a film on the device, and its lossless container.
//
// sundog writes its beauty film as 12-bit PQ BT.2020 (src/film.cpp:96-115,
// src/transfer.h:14-50): linear radiance x 2^exposure -> BT.709 to BT.2020
// primaries -> linear 1.0 at 203 cd/m^2 -> SMPTE ST 2084 PQ -> 12-bit code
// (round half away from zero). pqEncode12 runs that chain per pixel with the
// FP32 operations in the reference's order written as round-to-nearest
// intrinsics (no FMA contraction) and powf for the two PQ powers; the codes
// go to the host as uint16 RGB.
//
// The reference wraps the codes in a lossless AVIF through libavif, which is
// not part of this build. writePq16Png stores them instead in a 16-bit RGB
// PNG (deflated with zlib) whose cICP chunk declares BT.2020
// primaries, the PQ transfer and full-range RGB, so HDR-aware viewers show
// it as sundog's AVIF would be shown; each 12-bit code c is widened to 16 bits
// by bit replication (c << 4 | c >> 8), which maps 0 and 4095 to 0 and 65535;
// the top 12 bits of a sample (v >> 4) are the code again.
#include <cuda_runtime.h>
#include <zlib.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "film_out.h"
#include "render_session.h"

namespace sdb {

__device__ __forceinline__ float pqOetfDevice(float lin) {
  const float m1 = 2610.0f / 16384.0f;
  const float m2 = 2523.0f / 4096.0f * 128.0f;
  const float c1 = 3424.0f / 4096.0f;
  const float c2 = 2413.0f / 4096.0f * 32.0f;
  const float c3 = 2392.0f / 4096.0f * 32.0f;
  float y = powf(fminf(fmaxf(lin, 0.0f), 1.0f), m1);
  float num = __fadd_rn(c1, __fmul_rn(c2, y));
  float den = __fadd_rn(1.0f, __fmul_rn(c3, y));
  return powf(__fdiv_rn(num, den), m2);
}

__device__ __forceinline__ unsigned short code12(float lin) {
  const float toPq = 203.0f / 10000.0f;
  float e = pqOetfDevice(__fmul_rn(lin, toPq));
  return (unsigned short)lroundf(__fmul_rn(e, 4095.0f));
}

__global__ void pqEncode12(const float4* __restrict__ film, int n, float scale,
                           unsigned short* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 f = film[i];
    float x = __fmul_rn(f.x, scale), y = __fmul_rn(f.y, scale), z = __fmul_rn(f.z, scale);
    float r = __fadd_rn(__fadd_rn(__fmul_rn(0.627404f, x), __fmul_rn(0.329283f, y)),
                        __fmul_rn(0.043313f, z));
    float g = __fadd_rn(__fadd_rn(__fmul_rn(0.069097f, x), __fmul_rn(0.919540f, y)),
                        __fmul_rn(0.011362f, z));
    float b = __fadd_rn(__fadd_rn(__fmul_rn(0.016391f, x), __fmul_rn(0.088013f, y)),
                        __fmul_rn(0.895595f, z));
    out[3 * (size_t)i + 0] = code12(r);
    out[3 * (size_t)i + 1] = code12(g);
    out[3 * (size_t)i + 2] = code12(b);
  }
}

void encodePq12(const float4* film, int width, int height, float exposure,
                unsigned short* hostOut, cudaStream_t st) {
  const int n = width * height;
  if (n <= 0) return;
  DevBuf d;
  d.alloc((size_t)n * 3 * sizeof(unsigned short));
  const float scale = exp2f(exposure);
  int grid = (n + 255) / 256;
  if (grid > 148 * 16) grid = 148 * 16;
  pqEncode12<<<grid, 256, 0, st>>>(film, n, scale, (unsigned short*)d.ptr);
  cudaCheck(cudaGetLastError(), "PQ encode launch");
  cudaCheck(cudaMemcpyAsync(hostOut, d.ptr, d.bytes, cudaMemcpyDeviceToHost, st), "PQ download");
  cudaCheck(cudaStreamSynchronize(st), "PQ encode");
}

namespace {

void put32(std::vector<unsigned char>& v, uint32_t x) {
  v.push_back((unsigned char)(x >> 24));
  v.push_back((unsigned char)(x >> 16));
  v.push_back((unsigned char)(x >> 8));
  v.push_back((unsigned char)x);
}

void chunk(FILE* f, const char* type, const std::vector<unsigned char>& data) {
  std::vector<unsigned char> buf;
  put32(buf, (uint32_t)data.size());
  buf.insert(buf.end(), type, type + 4);
  buf.insert(buf.end(), data.begin(), data.end());
  uint32_t crc = (uint32_t)crc32(0L, buf.data() + 4, (uInt)(buf.size() - 4));
  put32(buf, crc);
  if (std::fwrite(buf.data(), 1, buf.size(), f) != buf.size())
    throw std::runtime_error("PNG write failed");
}

}  // namespace

void writePq16Png(const std::string& path, const unsigned short* codes, int width, int height) {
  // Raw scanlines: filter byte 0, then big-endian 16-bit R G B samples.
  const size_t rowBytes = 1 + (size_t)width * 6;
  std::vector<unsigned char> raw(rowBytes * height);
  for (int y = 0; y < height; y++) {
    unsigned char* r = &raw[rowBytes * y];
    r[0] = 0;
    for (int x = 0; x < width * 3; x++) {
      unsigned c = codes[(size_t)y * width * 3 + x] & 0xFFFu;
      unsigned v = (c << 4) | (c >> 8);
      r[1 + 2 * x] = (unsigned char)(v >> 8);
      r[2 + 2 * x] = (unsigned char)v;
    }
  }
  uLongf zcap = compressBound((uLong)raw.size());
  std::vector<unsigned char> z(zcap);
  if (compress2(z.data(), &zcap, raw.data(), (uLong)raw.size(), 1) != Z_OK)
    throw std::runtime_error("PNG deflate failed");
  z.resize(zcap);
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("failed to write " + path);
  try {
    static const unsigned char sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    if (std::fwrite(sig, 1, 8, f) != 8) throw std::runtime_error("PNG write failed");
    std::vector<unsigned char> ihdr;
    put32(ihdr, (uint32_t)width);
    put32(ihdr, (uint32_t)height);
    ihdr.push_back(16);  // bit depth
    ihdr.push_back(2);   // colour type: RGB
    ihdr.push_back(0);   // deflate
    ihdr.push_back(0);   // adaptive filtering
    ihdr.push_back(0);   // no interlace
    chunk(f, "IHDR", ihdr);
    // cICP (PNG third edition): BT.2020 primaries (9), SMPTE ST 2084 (16),
    // RGB (matrix 0), full range.
    chunk(f, "cICP", std::vector<unsigned char>{9, 16, 0, 1});
    chunk(f, "IDAT", z);
    chunk(f, "IEND", {});
  } catch (...) {
    std::fclose(f);
    throw;
  }
  if (std::fclose(f) != 0) throw std::runtime_error("failed to write " + path);
}

}  // namespace sdb
