#include "assets.h"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace sdb {

namespace {

std::string dirOf(const std::string& p) {
  size_t k = p.find_last_of('/');
  return k == std::string::npos ? std::string(".") : p.substr(0, k);
}

// OBJ index token "v", "v/vt", "v//vn", "v/vt/vn" -> (v, vt) zero-based;
// negative indices count back from the current end; vt = -1 when absent.
bool parseCorner(const char* tok, long nv, long nt, long& v, long& vt) {
  char* end = nullptr;
  long a = std::strtol(tok, &end, 10);
  if (end == tok) return false;
  v = a > 0 ? a - 1 : nv + a;
  vt = -1;
  if (*end == '/') {
    const char* q = end + 1;
    if (*q != '/') {
      char* e2 = nullptr;
      long b = std::strtol(q, &e2, 10);
      if (e2 != q) vt = b > 0 ? b - 1 : nt + b;
    }
  }
  return true;
}

}  // namespace

HostMesh loadObj(const std::string& path, bool smooth, const std::string& usemtl) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("OBJ load failed: " + path + ": cannot open file");
  std::vector<float3> P;
  std::vector<float2> T;
  std::vector<std::pair<long, long>> corners;  // (position, texcoord)
  std::vector<std::string> mtlNames;
  std::string curMtl;
  bool filtering = !usemtl.empty();
  bool anyVtMissing = false;
  std::string line;
  std::vector<std::pair<long, long>> poly;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    const char* s = line.c_str();
    while (*s == ' ' || *s == '\t') s++;
    if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
      float x = 0, y = 0, z = 0;
      std::sscanf(s + 2, "%f %f %f", &x, &y, &z);
      P.push_back(make_float3(x, y, z));
    } else if (s[0] == 'v' && s[1] == 't' && (s[2] == ' ' || s[2] == '\t')) {
      float u = 0, v = 0;
      std::sscanf(s + 3, "%f %f", &u, &v);
      T.push_back(make_float2(u, v));
    } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
      poly.clear();
      std::istringstream ss(s + 2);
      std::string tok;
      while (ss >> tok) {
        long v, vt;
        if (!parseCorner(tok.c_str(), (long)P.size(), (long)T.size(), v, vt))
          throw std::runtime_error("OBJ has a malformed face: " + path);
        if (v < 0 || v >= (long)P.size())
          throw std::runtime_error("OBJ has out-of-range vertex index: " + path);
        if (vt >= (long)T.size() || vt < -1)
          throw std::runtime_error("OBJ has out-of-range texcoord index: " + path);
        poly.push_back({v, vt});
      }
      if (filtering && curMtl != usemtl) continue;
      for (size_t k = 1; k + 1 < poly.size(); k++) {
        const std::pair<long, long> tri[3] = {poly[0], poly[k], poly[k + 1]};
        for (const auto& c : tri) {
          if (c.second < 0) anyVtMissing = true;
          corners.push_back(c);
        }
      }
    } else if (std::strncmp(s, "usemtl", 6) == 0 && (s[6] == ' ' || s[6] == '\t')) {
      std::istringstream ss(s + 7);
      ss >> curMtl;
    } else if (std::strncmp(s, "mtllib", 6) == 0 && (s[6] == ' ' || s[6] == '\t')) {
      std::istringstream ss(s + 7);
      std::string lib;
      ss >> lib;
      std::ifstream mf(dirOf(path) + "/" + lib);
      std::string ml;
      while (std::getline(mf, ml)) {
        std::istringstream ms(ml);
        std::string key, name;
        ms >> key;
        if (key == "newmtl" && (ms >> name)) mtlNames.push_back(name);
      }
    }
  }
  if (filtering) {
    bool known = false;
    for (const std::string& n : mtlNames) known = known || n == usemtl;
    if (!known) throw std::runtime_error("OBJ usemtl group not found: " + usemtl + " in " + path);
  }
  if (corners.empty())
    throw std::runtime_error(filtering ? "OBJ usemtl group has no triangles: " + usemtl + " in " + path
                                       : "OBJ has no triangles: " + path);
  bool allUv = !T.empty() && !anyVtMissing;
  if (!T.empty() && anyVtMissing)
    std::fprintf(stderr, "[mesh] %s: some faces lack vt — ignoring texture coords\n", path.c_str());

  HostMesh m;
  std::vector<unsigned> posOf;
  m.idx.resize(corners.size() / 3);
  if (allUv) {
    std::unordered_map<unsigned long long, unsigned> remap;
    remap.reserve(P.size() * 2);
    for (size_t c = 0; c < corners.size(); c++) {
      unsigned long long key = ((unsigned long long)corners[c].first << 32) |
                               (unsigned long long)(unsigned)corners[c].second;
      auto it = remap.find(key);
      unsigned id;
      if (it == remap.end()) {
        id = (unsigned)m.pos.size();
        remap.emplace(key, id);
        m.pos.push_back(P[corners[c].first]);
        m.uv.push_back(T[corners[c].second]);
        posOf.push_back((unsigned)corners[c].first);
      } else {
        id = it->second;
      }
      (&m.idx[c / 3].x)[c % 3] = id;
    }
  } else {
    m.pos = P;
    posOf.resize(P.size());
    for (size_t i = 0; i < P.size(); i++) posOf[i] = (unsigned)i;
    for (size_t c = 0; c < corners.size(); c++) (&m.idx[c / 3].x)[c % 3] = (unsigned)corners[c].first;
  }
  if (smooth) {
    std::vector<float3> acc(P.size(), v3(0.0f));
    for (const uint3& t : m.idx) {
      float3 n = cross(m.pos[t.y] - m.pos[t.x], m.pos[t.z] - m.pos[t.x]);
      acc[posOf[t.x]] += n;
      acc[posOf[t.y]] += n;
      acc[posOf[t.z]] += n;
    }
    m.nrm.resize(m.pos.size());
    for (size_t i = 0; i < m.pos.size(); i++) {
      float3 n = acc[posOf[i]];
      float l = len(n);
      m.nrm[i] = l > 1e-12f ? n / l : v3(0.0f, 1.0f, 0.0f);
    }
  }
  return m;
}

bool loadHdr(const std::string& path, int& w, int& h, std::vector<float>& rgba, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open";
    return false;
  }
  auto fail = [&](const char* m) {
    err = m;
    std::fclose(f);
    return false;
  };
  char line[512];
  if (!std::fgets(line, sizeof line, f)) return fail("empty file");
  if (std::strncmp(line, "#?RADIANCE", 10) != 0 && std::strncmp(line, "#?RGBE", 6) != 0)
    return fail("not a Radiance HDR file");
  bool fmtOk = false;
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '\n' || (line[0] == '\r' && line[1] == '\n')) break;
    if (std::strncmp(line, "FORMAT=32-bit_rle_rgbe", 22) == 0) fmtOk = true;
  }
  if (!fmtOk) return fail("unsupported HDR format");
  if (!std::fgets(line, sizeof line, f)) return fail("missing resolution line");
  if (std::sscanf(line, "-Y %d +X %d", &h, &w) != 2 || w <= 0 || h <= 0 || w > (1 << 16) ||
      h > (1 << 16))
    return fail("unsupported HDR orientation (only -Y H +X W)");
  rgba.assign((size_t)w * h * 4, 0.0f);
  std::vector<unsigned char> scan((size_t)w * 4);
  auto emit = [&](int row) {
    for (int x = 0; x < w; x++) {
      const unsigned char* p = &scan[(size_t)x * 4];
      float* o = &rgba[((size_t)row * w + x) * 4];
      if (p[3]) {
        float s = (float)std::ldexp(1.0f, (int)p[3] - (128 + 8));
        o[0] = p[0] * s;
        o[1] = p[1] * s;
        o[2] = p[2] * s;
      } else {
        o[0] = o[1] = o[2] = 0.0f;
      }
      o[3] = 1.0f;
    }
  };
  for (int row = 0; row < h; row++) {
    unsigned char hd[4];
    if (std::fread(hd, 1, 4, f) != 4) return fail("truncated HDR data");
    bool rle = w >= 8 && w < 32768 && hd[0] == 2 && hd[1] == 2 && !(hd[2] & 0x80) &&
               ((hd[2] << 8) | hd[3]) == w;
    if (!rle) {
      // flat pixels: this header was the first pixel
      std::memcpy(&scan[0], hd, 4);
      if (w > 1 && std::fread(&scan[4], 1, (size_t)(w - 1) * 4, f) != (size_t)(w - 1) * 4)
        return fail("truncated HDR data");
      emit(row);
      continue;
    }
    for (int c = 0; c < 4; c++) {
      int x = 0;
      while (x < w) {
        int cnt = std::fgetc(f);
        if (cnt == EOF) return fail("truncated HDR data");
        if (cnt > 128) {
          cnt -= 128;
          int val = std::fgetc(f);
          if (val == EOF || x + cnt > w) return fail("bad HDR run");
          for (int k = 0; k < cnt; k++) scan[(size_t)(x++) * 4 + c] = (unsigned char)val;
        } else {
          if (cnt == 0 || x + cnt > w) return fail("bad HDR run");
          for (int k = 0; k < cnt; k++) {
            int val = std::fgetc(f);
            if (val == EOF) return fail("truncated HDR data");
            scan[(size_t)(x++) * 4 + c] = (unsigned char)val;
          }
        }
      }
    }
    emit(row);
  }
  std::fclose(f);
  return true;
}

bool loadImageRgba8(const std::string& path, int& w, int& h, std::vector<unsigned char>& rgba,
                    std::string& err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open";
    return false;
  }
  char magic[3] = {0, 0, 0};
  if (std::fread(magic, 1, 2, f) != 2) {
    std::fclose(f);
    err = "empty file";
    return false;
  }
  auto readTok = [&](std::string& t) {
    t.clear();
    int c = std::fgetc(f);
    while (c != EOF) {
      if (c == '#') {
        while (c != EOF && c != '\n') c = std::fgetc(f);
      } else if (std::isspace(c)) {
        if (!t.empty()) return true;
      } else {
        t.push_back((char)c);
      }
      c = std::fgetc(f);
    }
    return !t.empty();
  };
  if (magic[0] == 'P' && magic[1] == '6') {
    std::string a, b, c;
    if (!readTok(a) || !readTok(b) || !readTok(c) || std::atoi(c.c_str()) != 255) {
      std::fclose(f);
      err = "unsupported PPM header";
      return false;
    }
    w = std::atoi(a.c_str());
    h = std::atoi(b.c_str());
    std::vector<unsigned char> rgb((size_t)w * h * 3);
    if (w <= 0 || h <= 0 || std::fread(rgb.data(), 1, rgb.size(), f) != rgb.size()) {
      std::fclose(f);
      err = "truncated PPM";
      return false;
    }
    rgba.resize((size_t)w * h * 4);
    for (size_t i = 0; i < (size_t)w * h; i++) {
      rgba[4 * i] = rgb[3 * i];
      rgba[4 * i + 1] = rgb[3 * i + 1];
      rgba[4 * i + 2] = rgb[3 * i + 2];
      rgba[4 * i + 3] = 255;
    }
    std::fclose(f);
    return true;
  }
  if (magic[0] == 'P' && magic[1] == '7') {
    std::string k, v;
    int depth = 0;
    w = h = 0;
    while (readTok(k)) {
      if (k == "ENDHDR") break;
      if (!readTok(v)) break;
      if (k == "WIDTH") w = std::atoi(v.c_str());
      if (k == "HEIGHT") h = std::atoi(v.c_str());
      if (k == "DEPTH") depth = std::atoi(v.c_str());
    }
    if (w <= 0 || h <= 0 || (depth != 3 && depth != 4)) {
      std::fclose(f);
      err = "unsupported PAM header";
      return false;
    }
    std::vector<unsigned char> px((size_t)w * h * depth);
    if (std::fread(px.data(), 1, px.size(), f) != px.size()) {
      std::fclose(f);
      err = "truncated PAM";
      return false;
    }
    rgba.resize((size_t)w * h * 4);
    for (size_t i = 0; i < (size_t)w * h; i++)
      for (int c = 0; c < 4; c++) rgba[4 * i + c] = c < depth ? px[depth * i + c] : 255;
    std::fclose(f);
    return true;
  }
  std::fclose(f);
  err = "unsupported image format (AVIF needs libavif; use PPM/PAM)";
  return false;
}

}  // namespace sdb
