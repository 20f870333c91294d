// Load-time asset readers: Wavefront OBJ meshes and Radiance RGBE (.hdr)
// environment maps, plus small image readers for textures.
#pragma once

#include <string>
#include <vector>

#include "sd_vec.h"

namespace sdb {

struct HostMesh {
  std::vector<float3> pos;      // seam-duplicated when uvs are present
  std::vector<uint3> idx;
  std::vector<float3> nrm;      // empty: faceted (geometric normals)
  std::vector<float2> uv;       // empty: barycentric uv
};

// OBJ -> triangle mesh with the reference loader's conventions
// (src/mesh_obj.cpp:13-145): n-gons triangulated as fans, optional usemtl
// group filter (names from the mtllib), uv-seam vertex duplication by unique
// (position, texcoord) pair in first-use order, area-weighted smooth normals
// aggregated per original position, OBJ normals ignored.
HostMesh loadObj(const std::string& path, bool smooth, const std::string& usemtl);

// Radiance RGBE file -> linear float RGBA (alpha 1), row 0 = top. Flat and
// run-length-encoded scanlines; only the standard "-Y H +X W" orientation.
// Texel value = mantissa * 2^(exponent - 136), 0 when the exponent is 0.
bool loadHdr(const std::string& path, int& w, int& h, std::vector<float>& rgba, std::string& err);

// 8-bit RGBA textures: binary PPM (P6), PAM (P7 RGB/RGBA) or PNG-free
// formats only; AVIF needs libavif, which this build does not link.
bool loadImageRgba8(const std::string& path, int& w, int& h, std::vector<unsigned char>& rgba,
                    std::string& err);

}  // namespace sdb
