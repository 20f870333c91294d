// ORACLE — test infrastructure only (the checker, never the product).
//
// CPU path tracer restating sundog's render path: scene assets and tables as
// src/capi_render.cpp:74-221 builds them (mesh-light CDFs 126-172, env CDFs
// src/env_light.cpp:27-56, camera src/scene_build.cpp:13-29), the per-pixel
// estimator of device/programs.cu:311-572, and the hit semantics OptiX gives
// the reference (closest accepted hit with any-hit filtering for radiance
// rays, exactly-once crossing bookkeeping for shadow rays; programs.cu:49-302,
// src/accel.cpp:54-58, 105-107). Device math comes from sdo/sdo.h.
//
// Independent of the CUDA product by construction: own median-split BVH, own
// OBJ / RGBE readers, triangles intersected in double precision
// (Moller-Trumbore), instance inverses in double.
//
// Scene input is a line-oriented text description (written by
// oracle/oracle.py from the parse-time scene state); see sdo_scene_load.
#include <algorithm>
#include <cctype>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "sdo/sdo.h"

using namespace sdo;

namespace {

struct Camera { float3 origin, lowerLeft, horizontal, vertical, u, v, w; float lensRadius; };

struct Mesh {
  std::vector<float3> pos, nrm;
  std::vector<float2> uv;
  std::vector<uint3> idx;
  std::vector<int> bvhPrim;   // leaf order -> triangle
  struct Node { float lo[3], hi[3]; int left, right, start, count; };
  std::vector<Node> nodes;
};

struct Instance {
  int kind, mesh;
  uint16_t matF, matB;
  int cutout, lightId;
  double m[12];      // object -> world
  float w2o[12];     // world -> object (rounded from double)
  float lo[3], hi[3];
};

struct Scene {
  int W = 0, H = 0, spp = 1, maxDepth = 16, transparentShadows = 1;
  float clampVal = 0;
  unsigned seed = 7;
  Camera cam;
  int bgKind = 0;
  float3 bgA{0, 0, 0}, bgB{0, 0, 0};
  EnvDesc env{};
  std::vector<float> envTexels, envMarg, envCond;
  std::vector<TextureDesc> tex;
  std::vector<std::vector<unsigned char>> texImg;
  std::vector<MaterialDesc> mats;
  std::vector<Mesh> meshes;
  std::vector<Instance> inst;
  std::vector<Mesh::Node> tlas;
  std::vector<int> tlasPrim;
  std::vector<LightDesc> lights;
  std::vector<std::vector<float3>> lightPos;
  std::vector<std::vector<float>> lightCdf;
  std::vector<FlameDesc> flames;
};

// ---- assets ---------------------------------------------------------------------

// Binary PPM (P6, maxval 255) or PAM (P7, DEPTH 3 or 4, MAXVAL 255) as RGBA8,
// row 0 = top; alpha 255 where the file has none. The oracle's own reader of
// the uncompressed formats the tests write (the reference decodes AVIF with
// libavif into the same RGBA8 layout, src/textures.cpp:22-64).
std::vector<unsigned char> loadImageRgba8(const std::string& path, int& w, int& h) {
  std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "rb"), &std::fclose);
  if (!f) throw std::runtime_error("oracle: cannot open " + path);
  // Next whitespace-separated header token, skipping '#' comments.
  auto token = [&]() {
    std::string t;
    int c;
    while ((c = std::fgetc(f.get())) != EOF) {
      if (c == '#' && t.empty()) {
        while (c != EOF && c != '\n') c = std::fgetc(f.get());
      } else if (std::isspace(c)) {
        if (!t.empty()) return t;
      } else {
        t.push_back((char)c);
      }
    }
    if (t.empty()) throw std::runtime_error("oracle: truncated header in " + path);
    return t;
  };
  std::string magic = token();
  int depth = 0;
  w = h = 0;
  if (magic == "P6") {
    w = std::atoi(token().c_str());
    h = std::atoi(token().c_str());
    if (std::atoi(token().c_str()) != 255) throw std::runtime_error("oracle: PPM maxval must be 255");
    depth = 3;
  } else if (magic == "P7") {
    for (std::string k = token(); k != "ENDHDR"; k = token()) {
      std::string v = token();
      if (k == "WIDTH") w = std::atoi(v.c_str());
      else if (k == "HEIGHT") h = std::atoi(v.c_str());
      else if (k == "DEPTH") depth = std::atoi(v.c_str());
      else if (k == "MAXVAL" && v != "255") throw std::runtime_error("oracle: PAM maxval must be 255");
    }
  } else {
    throw std::runtime_error("oracle: unsupported image " + path);
  }
  if (w <= 0 || h <= 0 || (depth != 3 && depth != 4))
    throw std::runtime_error("oracle: unsupported image header in " + path);
  // token() consumed the one whitespace byte that ends the header.
  std::vector<unsigned char> raw((size_t)w * h * depth);
  if (std::fread(raw.data(), 1, raw.size(), f.get()) != raw.size())
    throw std::runtime_error("oracle: truncated pixels in " + path);
  std::vector<unsigned char> rgba((size_t)w * h * 4);
  for (size_t i = 0; i < (size_t)w * h; i++)
    for (int c = 0; c < 4; c++) rgba[4 * i + c] = c < depth ? raw[depth * i + c] : 255;
  return rgba;
}

// OBJ reader with the reference loader's conventions (src/mesh_obj.cpp:13-145).
void loadObj(const std::string& path, bool smooth, const std::string& usemtl, Mesh& out) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("oracle: cannot open " + path);
  std::vector<float3> P;
  std::vector<float2> T;
  std::vector<std::pair<long, long>> corners;
  std::string cur, line;
  bool anyNoVt = false;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string key;
    if (!(ss >> key)) continue;
    if (key == "v") {
      float x, y, z;
      ss >> x >> y >> z;
      P.push_back(f3(x, y, z));
    } else if (key == "vt") {
      float a, b;
      ss >> a >> b;
      T.push_back({a, b});
    } else if (key == "usemtl") {
      ss >> cur;
    } else if (key == "f") {
      std::vector<std::pair<long, long>> poly;
      std::string tok;
      while (ss >> tok) {
        long v = std::strtol(tok.c_str(), nullptr, 10);
        long vt = -1;
        size_t sl = tok.find('/');
        if (sl != std::string::npos && sl + 1 < tok.size() && tok[sl + 1] != '/')
          vt = std::strtol(tok.c_str() + sl + 1, nullptr, 10);
        v = v > 0 ? v - 1 : (long)P.size() + v;
        if (vt != -1) vt = vt > 0 ? vt - 1 : (long)T.size() + vt;
        poly.push_back({v, vt});
      }
      if (!usemtl.empty() && cur != usemtl) continue;
      for (size_t k = 1; k + 1 < poly.size(); k++)
        for (auto c : {poly[0], poly[k], poly[k + 1]}) {
          if (c.second < 0) anyNoVt = true;
          corners.push_back(c);
        }
    }
  }
  if (corners.empty()) throw std::runtime_error("oracle: no triangles in " + path);
  bool allUv = !T.empty() && !anyNoVt;
  std::vector<unsigned> posOf;
  out.idx.resize(corners.size() / 3);
  if (allUv) {
    std::unordered_map<uint64_t, unsigned> remap;
    for (size_t c = 0; c < corners.size(); c++) {
      uint64_t key = ((uint64_t)corners[c].first << 32) | (uint32_t)corners[c].second;
      auto it = remap.find(key);
      unsigned id;
      if (it == remap.end()) {
        id = (unsigned)out.pos.size();
        remap[key] = id;
        out.pos.push_back(P[corners[c].first]);
        out.uv.push_back(T[corners[c].second]);
        posOf.push_back((unsigned)corners[c].first);
      } else {
        id = it->second;
      }
      (&out.idx[c / 3].x)[c % 3] = id;
    }
  } else {
    out.pos = P;
    for (size_t i = 0; i < P.size(); i++) posOf.push_back((unsigned)i);
    for (size_t c = 0; c < corners.size(); c++) (&out.idx[c / 3].x)[c % 3] = (unsigned)corners[c].first;
  }
  if (smooth) {
    std::vector<float3> acc(P.size(), f3(0.0f));
    for (const uint3& t : out.idx) {
      float3 n = cross(out.pos[t.y] - out.pos[t.x], out.pos[t.z] - out.pos[t.x]);
      acc[posOf[t.x]] += n;
      acc[posOf[t.y]] += n;
      acc[posOf[t.z]] += n;
    }
    out.nrm.resize(out.pos.size());
    for (size_t i = 0; i < out.pos.size(); i++) {
      float3 n = acc[posOf[i]];
      float l = length(n);
      out.nrm[i] = l > 1e-12f ? n / l : f3(0.0f, 1.0f, 0.0f);
    }
  }
}

// Radiance RGBE reader; texel = mantissa * 2^(e - 136) (the conversion of
// extern/stb_image.h's HDR loader the reference uses).
void loadHdr(const std::string& path, int& w, int& h, std::vector<float>& px) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("oracle: cannot open " + path);
  char line[512];
  bool ok = std::fgets(line, sizeof line, f) && std::strncmp(line, "#?", 2) == 0;
  while (ok && std::fgets(line, sizeof line, f) && line[0] != '\n') {
  }
  if (!ok || !std::fgets(line, sizeof line, f) || std::sscanf(line, "-Y %d +X %d", &h, &w) != 2) {
    std::fclose(f);
    throw std::runtime_error("oracle: bad HDR header " + path);
  }
  px.assign((size_t)w * h * 4, 0.0f);
  std::vector<unsigned char> row((size_t)w * 4);
  for (int y = 0; y < h; y++) {
    unsigned char q[4];
    if (std::fread(q, 1, 4, f) != 4) break;
    if (w >= 8 && w < 32768 && q[0] == 2 && q[1] == 2 && ((q[2] << 8) | q[3]) == w) {
      for (int c = 0; c < 4; c++) {
        int x = 0;
        while (x < w) {
          int n = std::fgetc(f);
          if (n > 128) {
            int v = std::fgetc(f);
            for (int k = 0; k < n - 128 && x < w; k++) row[(size_t)(x++) * 4 + c] = (unsigned char)v;
          } else {
            for (int k = 0; k < n && x < w; k++) row[(size_t)(x++) * 4 + c] = (unsigned char)std::fgetc(f);
          }
        }
      }
    } else {
      std::memcpy(row.data(), q, 4);
      if (w > 1 && std::fread(row.data() + 4, 1, (size_t)(w - 1) * 4, f) != (size_t)(w - 1) * 4) break;
    }
    for (int x = 0; x < w; x++) {
      const unsigned char* p = &row[(size_t)x * 4];
      float* o = &px[((size_t)y * w + x) * 4];
      if (p[3]) {
        float s = (float)std::ldexp(1.0f, (int)p[3] - (128 + 8));
        o[0] = p[0] * s;
        o[1] = p[1] * s;
        o[2] = p[2] * s;
      }
      o[3] = 1.0f;
    }
  }
  std::fclose(f);
}

// ---- simple median-split BVH ----------------------------------------------------------
template <class BoxOf>
void buildTree(int n, BoxOf boxOf, std::vector<Mesh::Node>& nodes, std::vector<int>& prim, int leafMax) {
  prim.resize(n);
  for (int i = 0; i < n; i++) prim[i] = i;
  std::vector<float> lo(3 * (size_t)n), hi(3 * (size_t)n);
  for (int i = 0; i < n; i++) boxOf(i, &lo[3 * (size_t)i], &hi[3 * (size_t)i]);
  nodes.clear();
  struct Job { int node, b, e; };
  nodes.push_back({});
  std::vector<Job> st{{0, 0, n}};
  while (!st.empty()) {
    Job j = st.back();
    st.pop_back();
    Mesh::Node nd;
    for (int a = 0; a < 3; a++) { nd.lo[a] = 1e30f; nd.hi[a] = -1e30f; }
    for (int i = j.b; i < j.e; i++)
      for (int a = 0; a < 3; a++) {
        nd.lo[a] = std::min(nd.lo[a], lo[3 * (size_t)prim[i] + a]);
        nd.hi[a] = std::max(nd.hi[a], hi[3 * (size_t)prim[i] + a]);
      }
    nd.left = nd.right = -1;
    nd.start = j.b;
    nd.count = j.e - j.b;
    if (j.e - j.b > leafMax) {
      int ax = 0;
      float best = -1;
      for (int a = 0; a < 3; a++)
        if (nd.hi[a] - nd.lo[a] > best) { best = nd.hi[a] - nd.lo[a]; ax = a; }
      int mid = (j.b + j.e) / 2;
      std::nth_element(prim.begin() + j.b, prim.begin() + mid, prim.begin() + j.e, [&](int x, int y) {
        return lo[3 * (size_t)x + ax] + hi[3 * (size_t)x + ax] < lo[3 * (size_t)y + ax] + hi[3 * (size_t)y + ax];
      });
      nd.left = (int)nodes.size();
      nodes.push_back({});
      nd.right = (int)nodes.size();
      nodes.push_back({});
      nd.count = 0;
      st.push_back({nd.left, j.b, mid});
      st.push_back({nd.right, mid, j.e});
    }
    nodes[j.node] = nd;
  }
}

bool boxHit(const Mesh::Node& nd, const double o[3], const double inv[3], double tmax) {
  double t0 = 0.0, t1 = tmax;
  for (int a = 0; a < 3; a++) {
    double ta = ((double)nd.lo[a] - o[a]) * inv[a], tb = ((double)nd.hi[a] - o[a]) * inv[a];
    if (ta > tb) std::swap(ta, tb);
    t0 = std::max(t0, ta);
    t1 = std::min(t1, tb * (1.0 + 1e-9));
    if (t0 > t1) return false;
  }
  return true;
}

// ---- scene loading --------------------------------------------------------------------------

Camera makeCamera(float3 lf, float3 la, float3 up, float vfov, float aperture, float focusDist, int W, int H) {
  Camera c;
  float aspect = (float)W / (float)H;
  float theta = vfov * SD_PI / 180.0f;
  float halfH = std::tan(theta / 2.0f);
  float halfW = aspect * halfH;
  float focus = focusDist > 0.0f ? focusDist : length(lf - la);
  c.w = normalize(lf - la);
  c.u = normalize(cross(up, c.w));
  c.v = cross(c.w, c.u);
  c.origin = lf;
  c.lowerLeft = c.origin - halfW * focus * c.u - halfH * focus * c.v - focus * c.w;
  c.horizontal = 2.0f * halfW * focus * c.u;
  c.vertical = 2.0f * halfH * focus * c.v;
  c.lensRadius = aperture / 2.0f;
  return c;
}

void invert(const double* m, float* out) {
  double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
  double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  double r[9] = {(e * i - f * h) / det, (c * h - b * i) / det, (b * f - c * e) / det,
                 (f * g - d * i) / det, (a * i - c * g) / det, (c * d - a * f) / det,
                 (d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det};
  for (int row = 0; row < 3; row++) {
    double t = -(r[3 * row] * m[3] + r[3 * row + 1] * m[7] + r[3 * row + 2] * m[11]);
    out[4 * row] = (float)r[3 * row];
    out[4 * row + 1] = (float)r[3 * row + 1];
    out[4 * row + 2] = (float)r[3 * row + 2];
    out[4 * row + 3] = (float)t;
  }
}

float3 apply(const float* m, float3 p, bool point) {
  return f3(m[0] * p.x + m[1] * p.y + m[2] * p.z + (point ? m[3] : 0.0f),
            m[4] * p.x + m[5] * p.y + m[6] * p.z + (point ? m[7] : 0.0f),
            m[8] * p.x + m[9] * p.y + m[10] * p.z + (point ? m[11] : 0.0f));
}
float3 normalToWorld(const float* w2o, float3 n) {
  return f3(w2o[0] * n.x + w2o[4] * n.y + w2o[8] * n.z, w2o[1] * n.x + w2o[5] * n.y + w2o[9] * n.z,
            w2o[2] * n.x + w2o[6] * n.y + w2o[10] * n.z);
}

std::unique_ptr<Scene> parseScene(const std::string& text) {
  std::unique_ptr<Scene> S(new Scene());
  std::istringstream in(text);
  std::string line;
  std::vector<std::string> meshFiles, meshMtl;
  std::vector<int> meshSmooth;
  std::string envFile;
  float envRot = 0, envInt = 1;
  int envImp = 1;
  float3 lf{0, 2, 8}, la{0, 0, 0}, up{0, 1, 0};
  float vfov = 40, aperture = 0, focus = 0;
  std::vector<float> objXf;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string k;
    if (!(ss >> k)) continue;
    if (k == "render") {
      ss >> S->W >> S->H >> S->spp >> S->maxDepth >> S->clampVal >> S->seed >> S->transparentShadows;
    } else if (k == "camera") {
      ss >> lf.x >> lf.y >> lf.z >> la.x >> la.y >> la.z >> up.x >> up.y >> up.z >> vfov >> aperture >> focus;
    } else if (k == "bg") {
      ss >> S->bgKind >> S->bgA.x >> S->bgA.y >> S->bgA.z >> S->bgB.x >> S->bgB.y >> S->bgB.z;
    } else if (k == "env") {
      ss >> envFile >> envRot >> envInt >> envImp;
    } else if (k == "texture") {
      TextureDesc t{};
      std::string file;
      ss >> t.kind >> t.a.x >> t.a.y >> t.a.z >> t.b.x >> t.b.y >> t.b.z >> t.scale.x >> t.scale.y >> t.width >>
          t.srgb >> file;
      if (t.kind == TX_IMAGE) {
        S->texImg.push_back(loadImageRgba8(file, t.imgW, t.imgH));
      } else {
        S->texImg.emplace_back();
      }
      S->tex.push_back(t);
    } else if (k == "material") {
      MaterialDesc m{};
      ss >> m.kind >> m.texId >> m.color.x >> m.color.y >> m.color.z >> m.roughness >> m.ior >> m.intensity >>
          m.twoSided >> m.absorb.x >> m.absorb.y >> m.absorb.z >> m.waveAmp >> m.waveFreq;
      S->mats.push_back(m);
    } else if (k == "mesh") {
      int sm;
      std::string f, mtl;
      ss >> sm >> f >> mtl;
      meshSmooth.push_back(sm);
      meshFiles.push_back(f);
      meshMtl.push_back(mtl == "-" ? "" : mtl);
    } else if (k == "object") {
      Instance o{};
      int mf, mb;
      ss >> o.kind >> o.mesh >> mf >> mb >> o.cutout >> o.lightId;
      o.matF = (uint16_t)mf;
      o.matB = (uint16_t)mb;
      for (int i = 0; i < 12; i++) {
        float v;
        ss >> v;
        o.m[i] = v;
      }
      S->inst.push_back(o);
    } else if (k == "light") {
      LightDesc l{};
      ss >> l.kind >> l.p.x >> l.p.y >> l.p.z >> l.u.x >> l.u.y >> l.u.z >> l.v.x >> l.v.y >> l.v.z >> l.n.x >>
          l.n.y >> l.n.z >> l.L.x >> l.L.y >> l.L.z >> l.radius >> l.area >> l.dir.x >> l.dir.y >> l.dir.z >>
          l.twoSided >> l.texId >> l.flameId;
      S->lights.push_back(l);
    } else if (k == "flame") {
      FlameDesc f{};
      ss >> f.base.x >> f.base.y >> f.base.z >> f.height >> f.radius >> f.intensity >> f.sigma >> f.noiseScale >>
          f.seed >> f.steps;
      S->flames.push_back(f);
    }
  }
  if (S->W <= 0 || S->H <= 0) throw std::runtime_error("oracle: missing render line");
  S->cam = makeCamera(lf, la, up, vfov, aperture, focus, S->W, S->H);
  for (size_t i = 0; i < S->tex.size(); i++)
    S->tex[i].img = S->tex[i].kind == TX_IMAGE ? S->texImg[i].data() : nullptr;
  // meshes
  S->meshes.resize(meshFiles.size());
  for (size_t i = 0; i < meshFiles.size(); i++) {
    Mesh& m = S->meshes[i];
    loadObj(meshFiles[i], meshSmooth[i] != 0, meshMtl[i], m);
    buildTree((int)m.idx.size(), [&](int t, float* lo, float* hi) {
      const uint3& tr = m.idx[t];
      for (int a = 0; a < 3; a++) {
        float v0 = (&m.pos[tr.x].x)[a], v1 = (&m.pos[tr.y].x)[a], v2 = (&m.pos[tr.z].x)[a];
        lo[a] = std::min(v0, std::min(v1, v2));
        hi[a] = std::max(v0, std::max(v1, v2));
      }
    }, m.nodes, m.bvhPrim, 4);
  }
  // instances: inverses and world boxes
  for (Instance& o : S->inst) {
    invert(o.m, o.w2o);
    float fm[12];
    for (int i = 0; i < 12; i++) fm[i] = (float)o.m[i];
    for (int a = 0; a < 3; a++) { o.lo[a] = 1e30f; o.hi[a] = -1e30f; }
    auto grow = [&](float3 p) {
      float3 w = apply(fm, p, true);
      for (int a = 0; a < 3; a++) {
        o.lo[a] = std::min(o.lo[a], (&w.x)[a]);
        o.hi[a] = std::max(o.hi[a], (&w.x)[a]);
      }
    };
    if (o.kind == GK_MESH) {
      for (const float3& p : S->meshes[o.mesh].pos) grow(p);
    } else {
      float lo[3] = {-1, -1, -1}, hi[3] = {1, 1, 1};
      if (o.kind == GK_RECT || o.kind == GK_DISK) { lo[1] = -1e-4f; hi[1] = 1e-4f; }
      if (o.kind == GK_PARABOLA) { lo[1] = -1e-4f; hi[1] = 0.5f + 1e-4f; }
      for (int c = 0; c < 8; c++) grow(f3(c & 1 ? hi[0] : lo[0], c & 2 ? hi[1] : lo[1], c & 4 ? hi[2] : lo[2]));
    }
    for (int a = 0; a < 3; a++) {  // pad: world boxes come from rounded corners
      float e = 1e-5f * (1.0f + std::fabs(o.lo[a]) + std::fabs(o.hi[a]));
      o.lo[a] -= e;
      o.hi[a] += e;
    }
  }
  buildTree((int)S->inst.size(), [&](int i, float* lo, float* hi) {
    for (int a = 0; a < 3; a++) { lo[a] = S->inst[i].lo[a]; hi[a] = S->inst[i].hi[a]; }
  }, S->tlas, S->tlasPrim, 1);
  // mesh lights (src/capi_render.cpp:126-172)
  S->lightPos.resize(S->lights.size());
  S->lightCdf.resize(S->lights.size());
  for (const Instance& o : S->inst) {
    if (o.kind != GK_MESH || o.lightId < 0) continue;
    const Mesh& m = S->meshes[o.mesh];
    float fm[12];
    for (int i = 0; i < 12; i++) fm[i] = (float)o.m[i];
    std::vector<float3>& wp = S->lightPos[o.lightId];
    wp.resize(m.pos.size());
    for (size_t i = 0; i < wp.size(); i++) wp[i] = apply(fm, m.pos[i], true);
    std::vector<float>& cdf = S->lightCdf[o.lightId];
    cdf.assign(m.idx.size() + 1, 0.0f);
    double total = 0.0;
    for (size_t t = 0; t < m.idx.size(); t++) {
      const uint3& tr = m.idx[t];
      total += 0.5 * (double)length(cross(wp[tr.y] - wp[tr.x], wp[tr.z] - wp[tr.x]));
      cdf[t + 1] = (float)total;
    }
    for (size_t t = 1; t < m.idx.size(); t++) cdf[t] = (float)(cdf[t] / total);
    cdf[m.idx.size()] = 1.0f;
    LightDesc& l = S->lights[o.lightId];
    l.mPositions = wp.data();
    l.mIndices = m.idx.data();
    l.mUvs = m.uv.empty() ? nullptr : m.uv.data();
    l.mCdf = cdf.data();
    l.mNumTris = (int)m.idx.size();
    l.area = (float)total;
    float3 ux = apply(fm, f3(1, 0, 0), false), uy = apply(fm, f3(0, 1, 0), false), uz = apply(fm, f3(0, 0, 1), false);
    l.mNgSign = dot(uy, cross(uz, ux)) < 0.0f ? -1.0f : 1.0f;
  }
  // environment (src/env_light.cpp:12-97)
  if (S->bgKind == 2) {
    int w, h;
    loadHdr(envFile, w, h, S->envTexels);
    S->envMarg.assign(h + 1, 0.0f);
    S->envCond.assign((size_t)h * (w + 1), 0.0f);
    double total = 0.0;
    for (int row = 0; row < h; row++) {
      float sinT = std::sin(SD_PI * (row + 0.5f) / h);
      float* cdf = &S->envCond[(size_t)row * (w + 1)];
      double sum = 0.0;
      for (int col = 0; col < w; col++) {
        const float* p = &S->envTexels[4 * ((size_t)row * w + col)];
        float lum = 0.2126f * p[0] + 0.7152f * p[1] + 0.0722f * p[2];
        sum += (double)std::fmax(lum, 0.0f) * sinT;
        cdf[col + 1] = (float)sum;
      }
      if (sum > 0.0) {
        for (int c = 1; c <= w; c++) cdf[c] = (float)(cdf[c] / sum);
      } else {
        for (int c = 0; c <= w; c++) cdf[c] = (float)c / w;
      }
      cdf[w] = 1.0f;
      total += sum;
      S->envMarg[row + 1] = (float)total;
    }
    bool degenerate = total <= 0.0;
    if (!degenerate) {
      for (int r = 1; r <= h; r++) S->envMarg[r] = (float)(S->envMarg[r] / total);
    } else {
      for (int r = 0; r <= h; r++) S->envMarg[r] = (float)r / h;
    }
    S->envMarg[h] = 1.0f;
    S->env.texels = S->envTexels.data();
    S->env.margCdf = S->envMarg.data();
    S->env.condCdf = S->envCond.data();
    S->env.width = w;
    S->env.height = h;
    S->env.rotate = envRot * SD_PI / 180.0f;
    S->env.intensity = envInt;
    S->env.importance = (envImp && !degenerate) ? 1 : 0;
  }
  return S;
}

// ---- traversal --------------------------------------------------------------------------------

struct ShadePoint { float3 nFront; float u, v; bool frontface; };
struct Hit { bool hit; float t; int inst; int prim; float u, v; float3 nq; bool front; };

ShadePoint triShade(const Scene& S, const Instance& o, int prim, float b1, float b2, float3 D) {
  const Mesh& m = S.meshes[o.mesh];
  uint3 tri = m.idx[prim];
  float3 p0 = m.pos[tri.x], p1 = m.pos[tri.y], p2 = m.pos[tri.z];
  float3 ng = normalize(normalToWorld(o.w2o, cross(p1 - p0, p2 - p0)));
  float3 ns = ng;
  if (!m.nrm.empty()) {
    float3 n = m.nrm[tri.x] * (1.0f - b1 - b2) + m.nrm[tri.y] * b1 + m.nrm[tri.z] * b2;
    ns = normalize(normalToWorld(o.w2o, n));
    if (dot(ns, ng) < 0.0f) ns = -ns;
  }
  ShadePoint sp;
  sp.nFront = ns;
  if (!m.uv.empty()) {
    float2 t = m.uv[tri.x] * (1.0f - b1 - b2) + m.uv[tri.y] * b1 + m.uv[tri.z] * b2;
    sp.u = t.x;
    sp.v = t.y;
  } else {
    sp.u = b1;
    sp.v = b2;
  }
  sp.frontface = dot(ng, D) < 0.0f;
  if (o.lightId >= 0) {
    uint16_t side = sp.frontface ? o.matF : o.matB;
    if (side != MAT_NONE && S.mats[side].kind == MT_EMISSIVE) sp.nFront = ng;
  }
  return sp;
}

ShadePoint quadShade(const Instance& o, float3 nq, float u, float v, float3 D) {
  ShadePoint sp;
  sp.nFront = normalize(normalToWorld(o.w2o, nq));
  sp.u = u;
  sp.v = v;
  sp.frontface = dot(sp.nFront, D) < 0.0f;
  return sp;
}

bool accepts(const Scene& S, const Instance& o, bool front, float u, float v) {
  uint16_t m = front ? o.matF : o.matB;
  if (m == MAT_NONE) return false;
  if (o.cutout >= 0 && evalTexture(S.tex[o.cutout], u, v).w < 0.5f) return false;
  return true;
}

// Double-precision Moller-Trumbore (the FP64 triangle oracle).
bool triHit(const double o[3], const double d[3], float3 a, float3 b, float3 c, double tmax, double& t,
            double& b1, double& b2) {
  double e1[3] = {(double)b.x - a.x, (double)b.y - a.y, (double)b.z - a.z};
  double e2[3] = {(double)c.x - a.x, (double)c.y - a.y, (double)c.z - a.z};
  double p[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
  double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
  if (det == 0.0) return false;
  double inv = 1.0 / det;
  double s[3] = {o[0] - a.x, o[1] - a.y, o[2] - a.z};
  b1 = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv;
  if (b1 < 0.0 || b1 > 1.0) return false;
  double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
  b2 = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
  if (b2 < 0.0 || b1 + b2 > 1.0) return false;
  t = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * inv;
  return t > 0.0 && t < tmax;
}

// Visits every candidate (instance, primitive, root) in (0, tmax). For
// radiance keeps the closest accepted one; for shadows returns false on an
// occluder and accumulates transparent crossings.
template <bool SHADOW>
bool trace(const Scene& S, float3 O, float3 D, float tmaxIn, Hit& best, float& trProd, float3& tau) {
  double tmax = tmaxIn;
  best.hit = false;
  if (S.inst.empty()) return true;
  double Od[3] = {O.x, O.y, O.z}, invD[3] = {1.0 / D.x, 1.0 / D.y, 1.0 / D.z};
  std::vector<int> st{0};
  while (!st.empty()) {
    const Mesh::Node& nd = S.tlas[st.back()];
    st.pop_back();
    if (!boxHit(nd, Od, invD, tmax)) continue;
    if (nd.left >= 0) {
      st.push_back(nd.left);
      st.push_back(nd.right);
      continue;
    }
    for (int k = 0; k < nd.count; k++) {
      int ii = S.tlasPrim[nd.start + k];
      const Instance& o = S.inst[ii];
      bool masked = o.matF == MAT_NONE || o.matB == MAT_NONE || o.cutout >= 0;
      bool trans = (o.matF != MAT_NONE && (S.mats[o.matF].kind == MT_DIELECTRIC || S.mats[o.matF].kind == MT_WATER)) ||
                   (o.matB != MAT_NONE && (S.mats[o.matB].kind == MT_DIELECTRIC || S.mats[o.matB].kind == MT_WATER));
      float3 oo = apply(o.w2o, O, true), dd = apply(o.w2o, D, false);
      auto consider = [&](float t, int prim, float u, float v, float3 nq, ShadePoint sp) -> bool {
        // returns false when a shadow ray is occluded
        if (masked && !accepts(S, o, sp.frontface, sp.u, sp.v)) return true;
        if (SHADOW) {
          if (!trans) return false;
          uint16_t mid = sp.frontface ? o.matF : o.matB;
          const MaterialDesc& m = S.mats[mid];
          if (m.kind != MT_DIELECTRIC && m.kind != MT_WATER) return false;
          if (!S.transparentShadows) return false;
          float3 n = sp.frontface ? sp.nFront : -sp.nFront;
          float eta = sp.frontface ? 1.0f / m.ior : m.ior;
          float3 refr;
          if (!refract(D, n, eta, refr)) return false;
          float f0 = (1.0f - eta) / (1.0f + eta);
          f0 = f0 * f0;
          float c = sp.frontface ? -dot(D, n) : -dot(refr, n);
          trProd *= (1.0f - schlick(c, f0));
          float s = sp.frontface ? -t : t;
          tau = f3(tau.x + m.absorb.x * s, tau.y + m.absorb.y * s, tau.z + m.absorb.z * s);
          return true;
        }
        if (!best.hit || t < best.t) {
          best.hit = true;
          best.t = t;
          best.inst = ii;
          best.prim = prim;
          best.u = u;
          best.v = v;
          best.nq = nq;
          best.front = sp.frontface;
          tmax = t;
        }
        return true;
      };
      if (o.kind != GK_MESH) {
        QuadricHits qh = intersectQuadric(o.kind, oo, dd, 0.0f, (float)tmax);
        for (int r = 0; r < qh.count; r++) {
          if (qh.hits[r].t >= tmax) continue;
          ShadePoint sp = quadShade(o, qh.hits[r].n, qh.hits[r].u, qh.hits[r].v, D);
          if (!consider(qh.hits[r].t, 0, qh.hits[r].u, qh.hits[r].v, qh.hits[r].n, sp)) return false;
        }
        continue;
      }
      const Mesh& m = S.meshes[o.mesh];
      double od[3] = {oo.x, oo.y, oo.z}, ddd[3] = {dd.x, dd.y, dd.z};
      double inv2[3] = {1.0 / ddd[0], 1.0 / ddd[1], 1.0 / ddd[2]};
      std::vector<int> st2{0};
      while (!st2.empty()) {
        const Mesh::Node& n2 = m.nodes[st2.back()];
        st2.pop_back();
        if (!boxHit(n2, od, inv2, tmax)) continue;
        if (n2.left >= 0) {
          st2.push_back(n2.left);
          st2.push_back(n2.right);
          continue;
        }
        for (int q = 0; q < n2.count; q++) {
          int tri = m.bvhPrim[n2.start + q];
          const uint3& ix = m.idx[tri];
          double t, b1, b2;
          if (!triHit(od, ddd, m.pos[ix.x], m.pos[ix.y], m.pos[ix.z], tmax, t, b1, b2)) continue;
          ShadePoint sp = triShade(S, o, tri, (float)b1, (float)b2, D);
          if (!consider((float)t, tri, (float)b1, (float)b2, f3(0.0f), sp)) return false;
        }
      }
    }
  }
  return true;
}

float3 traceShadow(const Scene& S, float3 o, float3 d, float tmax) {
  Hit h;
  float trProd = 1.0f;
  float3 tau = f3(0.0f);
  if (!trace<true>(S, o, d, tmax, h, trProd, tau)) return f3(0.0f);
  tau = f3(std::fmax(0.0f, tau.x), std::fmax(0.0f, tau.y), std::fmax(0.0f, tau.z));
  float3 tr = f3(trProd);
  if (maxComp(tau) > 0.0f) tr = tr * exp3(-tau);
  return tr;
}

float3 sanitize(float3 c) {
  if (!std::isfinite(c.x) || !std::isfinite(c.y) || !std::isfinite(c.z)) return f3(0.0f);
  return c;
}

// One camera sample of one pixel (device/programs.cu:327-563). Returns L and
// the first-hit AOVs; counts radiance and shadow traces.
void samplePixel(const Scene& S, int px, int py, int s, int nStrata, float3& Lout, float3& alb, float3& nrmOut,
                 unsigned long long& rays) {
  int pixel = py * S.W + px;
  const Camera& cam = S.cam;
  Pcg32 rng = Pcg32::init(((unsigned long long)pixel << 32) ^ (unsigned long long)s, (unsigned long long)S.seed);
  float jx, jy;
  if (s < nStrata * nStrata) {
    jx = ((s % nStrata) + rng.rnd()) / nStrata;
    jy = ((s / nStrata) + rng.rnd()) / nStrata;
  } else {
    jx = rng.rnd();
    jy = rng.rnd();
  }
  float u = (px + jx) / S.W;
  float v = ((S.H - 1 - py) + jy) / S.H;
  float3 org = cam.origin;
  if (cam.lensRadius > 0.0f) {
    float2 rd = concentricDisk(rng.rnd2()) * cam.lensRadius;
    org = org + cam.u * rd.x + cam.v * rd.y;
  }
  float3 dir = normalize(cam.lowerLeft + u * cam.horizontal + v * cam.vertical - org);
  float3 L = f3(0.0f), beta = f3(1.0f);
  float prevPdf = 0.0f;
  bool specular = true;
  float3 prevX = org, o = org, d = dir;
  bool aovDone = false;
  const int MED_MAX = 4;
  float3 medSigma[MED_MAX];
  float medIor[MED_MAX];
  int medDepth = 0;
  const bool hasEnv = S.bgKind == 2;
  const int nStrat = (int)S.lights.size() + (hasEnv ? 1 : 0);
  const int numFlames = (int)S.flames.size();
  alb = f3(0.0f);
  nrmOut = f3(0.0f);
  for (int depth = 0; depth < S.maxDepth; depth++) {
    Hit hit;
    float dummyTr = 1.0f;
    float3 dummyTau = f3(0.0f);
    trace<false>(S, o, d, 1e16f, hit, dummyTr, dummyTau);
    rays++;
    if (medDepth > 0) {
      float3 sigma = medSigma[std::min(medDepth, MED_MAX) - 1];
      if (maxComp(sigma) > 0.0f) beta *= exp3(-sigma * (hit.hit ? hit.t : 1e4f));
    }
    if (numFlames > 0) {
      float3 trans = f3(1.0f);
      float3 Lv = marchFlames(S.flames.data(), numFlames, o, d, hit.hit ? hit.t : 1e16f, rng, trans);
      float3 cv = beta * Lv;
      if (depth >= 1 && S.clampVal > 0.0f) cv = min3(cv, f3(S.clampVal));
      L += cv;
      beta *= trans;
    }
    if (!hit.hit) {
      float3 bg;
      if (S.bgKind == 2) bg = envEval(S.env, d);
      else if (S.bgKind == 1) bg = lerp3(S.bgA, S.bgB, 0.5f * (d.y + 1.0f));
      else bg = S.bgA;
      float w = 1.0f;
      if (hasEnv && !specular) {
        float pdfE = envPdfSolidAngle(S.env, d) / nStrat;
        w = prevPdf / (prevPdf + pdfE);
      }
      float3 c = beta * bg * w;
      if (depth >= 1 && S.clampVal > 0.0f) c = min3(c, f3(S.clampVal));
      L += c;
      if (!aovDone) {
        alb = f3(std::fmin(bg.x, 1.0f), std::fmin(bg.y, 1.0f), std::fmin(bg.z, 1.0f));
        nrmOut = f3(0.0f);
        aovDone = true;
      }
      break;
    }
    const Instance& ins = S.inst[hit.inst];
    ShadePoint sp = ins.kind == GK_MESH ? triShade(S, ins, hit.prim, hit.u, hit.v, d)
                                        : quadShade(ins, hit.nq, hit.u, hit.v, d);
    bool front = hit.front;
    int matId = front ? ins.matF : ins.matB;
    float3 x = o + hit.t * d;
    float3 ns = front ? sp.nFront : -sp.nFront;
    const MaterialDesc& mat = S.mats[matId];
    float3 albedo = materialAlbedo(mat, S.tex.data(), sp.u, sp.v);
    if (mat.kind == MT_WATER && mat.waveAmp > 0.0f) ns = waterNormal(x, ns, -d, mat.waveAmp, mat.waveFreq);
    if (!aovDone) {
      alb = albedo;
      nrmOut = f3(dot(ns, cam.u), dot(ns, cam.v), dot(ns, cam.w));
      aovDone = true;
    }
    if (mat.kind == MT_EMISSIVE) {
      if (front || mat.twoSided) {
        float3 Le = albedo * mat.intensity;
        float w = 1.0f;
        if (!specular && ins.lightId >= 0 && !S.lights.empty()) {
          float pdfL = lightPdfSolidAngle(S.lights[ins.lightId], prevX, x, ns) / nStrat;
          w = prevPdf / (prevPdf + pdfL);
        }
        float3 c = beta * Le * w;
        if (depth >= 1 && S.clampVal > 0.0f) c = min3(c, f3(S.clampVal));
        L += c;
      }
      break;
    }
    float etaExt = 1.0f;
    if (mat.kind == MT_DIELECTRIC || mat.kind == MT_WATER) {
      int outer = std::min(front ? medDepth : medDepth - 1, MED_MAX);
      if (outer > 0) etaExt = medIor[outer - 1];
    }
    float etaRel = front ? etaExt / mat.ior : mat.ior / etaExt;
    if (nStrat > 0 && !bsdfIsDelta(mat)) {
      int k = std::min((int)(rng.rnd() * nStrat), nStrat - 1);
      LightSample ls = k < (int)S.lights.size() ? sampleLight(S.lights[k], x, rng, S.tex.data()) : sampleEnv(S.env, rng);
      float cosS = ls.valid ? dot(ls.wi, ns) : 0.0f;
      bool transmitNee = cosS < 0.0f && mat.kind == MT_DIELECTRIC;
      if (ls.valid && (cosS > 0.0f || transmitNee)) {
        rays++;
        float3 so = offsetRay(x, transmitNee ? -ns : ns);
        float tmaxS = ls.dist * 0.999f;
        float3 tr = traceShadow(S, so, ls.wi, tmaxS);
        if (maxComp(tr) > 0.0f) {
          if (numFlames > 0 && S.transparentShadows) {
            int skip = k < (int)S.lights.size() ? S.lights[k].flameId : -1;
            tr = tr * flameTransmittance(S.flames.data(), numFlames, so, ls.wi, tmaxS, rng, skip);
          }
          float pdfLe = (ls.isDelta ? 1.0f : ls.pdf) / nStrat;
          float3 f = bsdfEval(mat, albedo, -d, ls.wi, ns, etaRel);
          float w = 1.0f;
          if (!ls.isDelta) {
            float pdfB = bsdfPdf(mat, -d, ls.wi, ns, etaRel);
            w = pdfLe / (pdfLe + pdfB);
          }
          float3 c = beta * f * std::fabs(cosS) * ls.Li * w / pdfLe;
          c = c * tr;
          if (depth >= 1 && S.clampVal > 0.0f) c = min3(c, f3(S.clampVal));
          L += sanitize(c);
        }
      }
    }
    BsdfSample bs = bsdfSample(mat, albedo, d, ns, front, etaExt, rng);
    if (!bs.valid) break;
    if ((mat.kind == MT_WATER || mat.kind == MT_DIELECTRIC) && dot(bs.wi, ns) < 0.0f) {
      if (front) {
        if (medDepth < MED_MAX) {
          medSigma[medDepth] = mat.absorb;
          medIor[medDepth] = mat.ior;
        }
        medDepth++;
      } else if (medDepth > 0) {
        medDepth--;
      }
    }
    beta *= bs.weight;
    specular = bs.isDelta;
    prevPdf = bs.isDelta ? 0.0f : bs.pdf;
    prevX = x;
    float3 offN = dot(bs.wi, ns) >= 0.0f ? ns : -ns;
    o = offsetRay(x, offN);
    d = bs.wi;
    if (depth >= 4) {
      float q = clampf(maxComp(beta), 0.05f, 0.95f);
      if (rng.rnd() >= q) break;
      beta *= 1.0f / q;
    }
    if (maxComp(beta) <= 0.0f) break;
  }
  Lout = sanitize(L);
}

int strata(int spp) {
  int n = (int)std::floor(std::sqrt((float)spp) + 0.5f);
  if (n * n > spp) n--;
  return n < 1 ? 1 : n;
}

thread_local std::string t_err;

}  // namespace

// ---- C API --------------------------------------------------------------------------------------

// Parse + load + build. Returns NULL and fills err on failure.
extern "C" void* sdo_scene_load(const char* text, char* err, int errcap) {
  try {
    return parseScene(text).release();
  } catch (const std::exception& e) {
    if (err && errcap > 0) std::snprintf(err, (size_t)errcap, "%s", e.what());
    return nullptr;
  }
}

extern "C" void sdo_scene_free(void* s) { delete (Scene*)s; }

// Renders samples [s0, s1) of the pixel rectangle (x0, y0, w, h), folding
// them in sample order into rgba (w*h float4 running means, caller-owned and
// holding the previous samples' means). alb / nrm may be NULL. Returns the
// radiance + shadow trace count.
extern "C" unsigned long long sdo_render(void* sp, int x0, int y0, int w, int h, int s0, int s1, int threads,
                                         float* rgba, float* alb, float* nrm) {
  const Scene& S = *(const Scene*)sp;
  int nStrata = strata(S.spp);
  std::atomic<int> nextRow(0);
  std::atomic<unsigned long long> total(0);
  auto worker = [&]() {
    unsigned long long rays = 0;
    for (int r = nextRow++; r < h; r = nextRow++) {
      for (int c = 0; c < w; c++) {
        int px = x0 + c, py = y0 + r;
        float* acc = rgba + 4 * ((size_t)r * w + c);
        float* aa = alb ? alb + 4 * ((size_t)r * w + c) : nullptr;
        float* na = nrm ? nrm + 4 * ((size_t)r * w + c) : nullptr;
        for (int s = s0; s < s1; s++) {
          float3 L, A, N;
          samplePixel(S, px, py, s, nStrata, L, A, N, rays);
          acc[0] = acc[0] + (L.x - acc[0]) / (s + 1);
          acc[1] = acc[1] + (L.y - acc[1]) / (s + 1);
          acc[2] = acc[2] + (L.z - acc[2]) / (s + 1);
          acc[3] = 1.0f;
          if (aa) {
            aa[0] = aa[0] + (A.x - aa[0]) / (s + 1);
            aa[1] = aa[1] + (A.y - aa[1]) / (s + 1);
            aa[2] = aa[2] + (A.z - aa[2]) / (s + 1);
            aa[3] = 1.0f;
          }
          if (na) {
            na[0] = na[0] + (N.x - na[0]) / (s + 1);
            na[1] = na[1] + (N.y - na[1]) / (s + 1);
            na[2] = na[2] + (N.z - na[2]) / (s + 1);
            na[3] = 1.0f;
          }
        }
      }
    }
    total += rays;
  };
  if (threads <= 1) {
    worker();
  } else {
    std::vector<std::thread> ts;
    for (int i = 0; i < threads; i++) ts.emplace_back(worker);
    for (auto& t : ts) t.join();
  }
  return total.load();
}

// Scene tables for parity checks: which 0 = env marginal CDF, 1 = env
// conditional CDF, 2.. = mesh-light CDF of light (which - 2). Returns the
// number of floats (copies at most cap into out).
extern "C" long sdo_scene_table(void* sp, int which, float* out, long cap) {
  const Scene& S = *(const Scene*)sp;
  const std::vector<float>* v = nullptr;
  if (which == 0) v = &S.envMarg;
  else if (which == 1) v = &S.envCond;
  else if (which - 2 < (int)S.lightCdf.size()) v = &S.lightCdf[which - 2];
  if (!v) return -1;
  long n = (long)v->size();
  if (out) std::memcpy(out, v->data(), sizeof(float) * (size_t)std::min(n, cap));
  return n;
}

// FP64 quadric roots for the intersection-t parity check: same canonical
// shapes, evaluated in double. out: count, t0, t1.
extern "C" void sdo_quadric_fp64(int kind, const double* o, const double* d, double tmin, double tmax, double* out) {
  double ts[2];
  int n = 0;
  auto push = [&](double t, bool ok) {
    if (ok && t > tmin && t < tmax) ts[n++] = t;
  };
  if (kind == GK_SPHERE || kind == GK_CYLINDER) {
    bool cyl = kind == GK_CYLINDER;
    double a = d[0] * d[0] + (cyl ? 0.0 : d[1] * d[1]) + d[2] * d[2];
    double b = o[0] * d[0] + (cyl ? 0.0 : o[1] * d[1]) + o[2] * d[2];
    double c = o[0] * o[0] + (cyl ? 0.0 : o[1] * o[1]) + o[2] * o[2] - 1.0;
    double disc = b * b - a * c;
    if (a != 0.0 && disc > 0.0) {
      double s = std::sqrt(disc);
      for (double t : {(-b - s) / a, (-b + s) / a}) push(t, !cyl || std::fabs(o[1] + t * d[1]) <= 1.0);
    }
  } else if (kind == GK_RECT || kind == GK_DISK) {
    if (d[1] != 0.0) {
      double t = -o[1] / d[1], x = o[0] + t * d[0], z = o[2] + t * d[2];
      push(t, kind == GK_RECT ? (std::fabs(x) <= 1.0 && std::fabs(z) <= 1.0) : (x * x + z * z <= 1.0));
    }
  } else if (kind == GK_PARABOLA) {
    double A = 0.5 * (d[0] * d[0] + d[2] * d[2]), B = o[0] * d[0] + o[2] * d[2] - d[1];
    double C = 0.5 * (o[0] * o[0] + o[2] * o[2]) - o[1];
    auto inside = [&](double t) {
      double x = o[0] + t * d[0], z = o[2] + t * d[2];
      return x * x + z * z <= 1.0;
    };
    if (std::fabs(A) < 1e-12) {
      if (B != 0.0) push(-C / B, inside(-C / B));
    } else {
      double disc = B * B - 4 * A * C;
      if (disc > 0.0) {
        double s = std::sqrt(disc);
        double t0 = (-B - s) / (2 * A), t1 = (-B + s) / (2 * A);
        push(t0, inside(t0));
        push(t1, inside(t1));
      }
    }
  }
  out[0] = n;
  out[1] = n > 0 ? ts[0] : 0.0;
  out[2] = n > 1 ? ts[1] : 0.0;
}
