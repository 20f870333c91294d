// HDR output encoding of a film (film_out.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace sdb {

// 12-bit PQ BT.2020 codes (RGB, width*height*3 uint16 in host memory) of a
// device film of linear BT.709 running means, exposure in EV; waits for the
// stream.
void encodePq12(const float4* film, int width, int height, float exposure,
                unsigned short* hostOut, cudaStream_t st);

// 16-bit RGB PNG of 12-bit codes (bit-replicated to 16 bits) with a cICP
// chunk declaring BT.2020 / PQ / full-range RGB.
void writePq16Png(const std::string& path, const unsigned short* codes, int width, int height);

}  // namespace sdb
