// ORACLE — test infrastructure only (the checker, never the product).
//
// Scene derivation by the reference itself: this file is compiled together
// with sundog's own src/capi_scene.cpp and src/scene_build.cpp, read in place
// from the reference tree by oracle/Makefile (`make ref`), into
// oracle/_ref/libsdref_scene.so. That library therefore exports the
// reference's scene-construction C ABI (sundog_scene_create ...
// sundog_scene_validate, src/sundog_api.h:30-150) with the reference's own
// defaults, light registration (scene_build.cpp:31-153), flame lights
// (scene_build.cpp:155-181) and transform composition (scene_build.cpp:
// 48-70). This file adds two oracle-side entry points:
//
//   sundog_set_flame_steps   ray-march steps of one flame (the reference
//                            hard-codes 32 in device/volume.cuh:92,132; the
//                            volumes workload asks for 64), kept here in a
//                            side table because the reference's FlameDesc
//                            has no such field;
//   sdo_ref_scene_text       the derived sd::Scene written as the CPU
//                            oracle's line-oriented scene description (the
//                            format sdo_scene_load in oracle/integrator.cpp
//                            parses), so the oracle renders what the
//                            reference would have built from the same calls.
//
// Nothing of the CUDA product is linked or loaded.
#include "capi_internal.h"
#include "scene.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

namespace {

std::mutex g_stepsMu;
std::map<const sundog_scene*, std::map<int, int>> g_steps;

void put(std::string& o, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void put(std::string& o, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  int n = std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (n > 0) o.append(buf, (size_t)std::min(n, (int)sizeof buf - 1));
}

void f1(std::string& o, float v) { put(o, " %.9g", (double)v); }
void v3(std::string& o, float3 v) {
  f1(o, v.x);
  f1(o, v.y);
  f1(o, v.z);
}
std::string path(const std::string& base, const std::string& p) {
  if (p.empty() || p[0] == '/') return p;
  return base + "/" + p;
}

std::string sceneText(const sundog_scene* h) {
  const sd::Scene& s = h->scene;
  std::string o;
  const sd::RenderSettings& r = s.render;
  put(o, "render %d %d %d %d", r.width, r.height, r.spp, r.maxDepth);
  f1(o, r.clampVal);
  put(o, " %u %d\n", r.seed, r.transparentShadows ? 1 : 0);
  const sd::CameraSettings& c = s.camera;
  o += "camera";
  v3(o, c.lookfrom);
  v3(o, c.lookat);
  v3(o, c.up);
  f1(o, c.vfov);
  f1(o, c.aperture);
  f1(o, c.focusDist);
  o += "\n";
  put(o, "bg %d", s.bg.kind);
  v3(o, s.bg.a);
  v3(o, s.bg.b);
  o += "\n";
  if (s.bg.kind == sd::BG_ENVMAP) {
    put(o, "env %s", path(s.baseDir, s.env.file).c_str());
    f1(o, s.env.rotateDeg);
    f1(o, s.env.intensity);
    put(o, " %d\n", s.env.importance ? 1 : 0);
  }
  for (const sd::SceneTexture& t : s.textures) {
    put(o, "texture %d", t.desc.kind);
    v3(o, t.desc.a);
    v3(o, t.desc.b);
    f1(o, t.desc.scale.x);
    f1(o, t.desc.scale.y);
    f1(o, t.desc.width);
    put(o, " %d %s\n", t.srgb ? 1 : 0,
        t.imageFile.empty() ? "-" : path(s.baseDir, t.imageFile).c_str());
  }
  for (const sd::MaterialDesc& m : s.materials) {
    put(o, "material %d %d", m.kind, m.texId);
    v3(o, m.color);
    f1(o, m.roughness);
    f1(o, m.ior);
    f1(o, m.intensity);
    put(o, " %d", m.twoSided);
    v3(o, m.absorb);
    f1(o, m.waveAmp);
    f1(o, m.waveFreq);
    o += "\n";
  }
  for (const sd::SceneMesh& m : s.meshes)
    put(o, "mesh %d %s %s\n", m.smoothNormals ? 1 : 0, path(s.baseDir, m.objFile).c_str(),
        m.usemtl.empty() ? "-" : m.usemtl.c_str());
  for (const sd::SceneObject& ob : s.objects) {
    put(o, "object %d %d %d %d %d %d", ob.geomKind, ob.meshId, (int)ob.matFront,
        (int)ob.matBack, ob.cutoutTexId, ob.lightId);
    for (int k = 0; k < 12; k++) f1(o, ob.xform.m[k]);
    o += "\n";
  }
  for (const sd::LightDesc& l : s.lights) {
    put(o, "light %d", l.kind);
    v3(o, l.p);
    v3(o, l.u);
    v3(o, l.v);
    v3(o, l.n);
    v3(o, l.L);
    f1(o, l.radius);
    f1(o, l.area);
    v3(o, l.dir);
    put(o, " %d %d %d\n", l.twoSided, l.texId, l.flameId);
  }
  std::map<int, int> steps;
  {
    std::lock_guard<std::mutex> lock(g_stepsMu);
    auto it = g_steps.find(h);
    if (it != g_steps.end()) steps = it->second;
  }
  for (size_t i = 0; i < s.flames.size(); i++) {
    const sd::FlameDesc& f = s.flames[i];
    o += "flame";
    v3(o, f.base);
    f1(o, f.height);
    f1(o, f.radius);
    f1(o, f.intensity);
    f1(o, f.sigma);
    f1(o, f.noiseScale);
    auto st = steps.find((int)i);
    put(o, " %u %d\n", f.seed, st == steps.end() ? 32 : st->second);
  }
  return o;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int sundog_set_flame_steps(sundog_scene* h,
                                                                           int flame, int steps) {
  if (!h || flame < 0 || flame >= (int)h->scene.flames.size() || steps < 1 || steps > 4096)
    return 1;
  std::lock_guard<std::mutex> lock(g_stepsMu);
  g_steps[h][flame] = steps;
  return 0;
}

// Writes the oracle description of the scene behind `h` into buf (cap bytes,
// NUL-terminated); *needed receives the full size. 0 = OK, 1 = bad handle.
extern "C" __attribute__((visibility("default"))) int sdo_ref_scene_text(const sundog_scene* h,
                                                                       char* buf, size_t cap,
                                                                       size_t* needed) {
  if (!h) return 1;
  std::string t = sceneText(h);
  if (needed) *needed = t.size() + 1;
  if (buf && cap > 0) {
    size_t n = std::min(cap - 1, t.size());
    std::memcpy(buf, t.data(), n);
    buf[n] = '\0';
  }
  return 0;
}

// Forgets the side table of a handle about to be destroyed.
extern "C" __attribute__((visibility("default"))) void sdo_ref_scene_forget(const sundog_scene* h) {
  std::lock_guard<std::mutex> lock(g_stepsMu);
  g_steps.erase(h);
}
