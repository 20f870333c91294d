// Scene-construction half of the C ABI (no CUDA calls; testable without a
// GPU). Each entry narrows its doubles to float once, applies the reference
// renderer's defaults and checks, and records the result in the handle.
// Semantics follow src/capi_scene.cpp (cited per function); error messages
// keep the reference's wording so callers that match on them keep working.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sundog_api.h"
#include "abi_util.h"
#include "scene_model.h"

using namespace sdb;

namespace sdb {
static thread_local std::string t_error;
void setError(const std::string& m) { t_error = m; }
}  // namespace sdb

namespace {

bool isSet(double v) { return !std::isnan(v); }
float nf(double v, float dflt) { return std::isnan(v) ? dflt : (float)v; }
float3 nf3(const double* p, float3 dflt) {
  return p ? v3((float)p[0], (float)p[1], (float)p[2]) : dflt;
}

// Call-order guard (src/capi_internal.h:36-42).
void enterPhase(sundog_scene* h, int needed, const char* what) {
  if (!h) throw std::runtime_error("scene: null handle");
  if (h->phase > needed)
    throw std::runtime_error(std::string("scene: ") + what +
                             " must come before objects/flames/lights "
                             "(call order: config, objects, flames, lights)");
  h->phase = needed;
}

SdMaterial baseMaterial() {  // src/capi_scene.cpp:197-206
  SdMaterial m{};
  m.texId = -1;
  m.color = v3(0.8f);
  m.ior = 1.5f;
  m.roughness = 0.0f;
  m.intensity = 1.0f;
  m.twoSided = 0;
  return m;
}

int pushMaterial(sundog_scene* h, const SdMaterial& m, int tex) {
  enterPhase(h, 0, "materials");
  if (tex != -1 && (tex < 0 || tex >= (int)h->scene.textures.size()))
    sceneError("material: texture id out of range");
  if (h->scene.materials.size() >= kMatNone) sceneError("too many materials");
  int id = (int)h->scene.materials.size();
  h->scene.materials.push_back(m);
  return id;
}

int pushTexture(sundog_scene* h, const TextureCfg& t) {
  enterPhase(h, 0, "textures");
  int id = (int)h->scene.textures.size();
  h->scene.textures.push_back(t);
  return id;
}

}  // namespace

extern "C" const char* sundog_last_error(void) { return t_error.c_str(); }

// src/capi_scene.cpp:23-31
extern "C" sundog_scene* sundog_scene_create(const char* base_dir) {
  SDB_TRY
  sundog_scene* h = new sundog_scene();
  h->scene.baseDir = (base_dir && *base_dir) ? base_dir : ".";
  return h;
  SDB_CATCH(nullptr)
}

extern "C" void sundog_scene_destroy(sundog_scene* h) { delete h; }

// src/capi_scene.cpp:33-49
extern "C" int sundog_set_render(sundog_scene* h, int width, int height, int spp, int max_depth,
                                 double clamp, int64_t seed, double exposure,
                                 int transparent_shadows) {
  SDB_TRY
  enterPhase(h, 0, "render settings");
  RenderCfg& r = h->scene.render;
  if (width > 0) r.width = width;
  if (height > 0) r.height = height;
  if (spp > 0) r.spp = spp;
  if (max_depth > 0) r.maxDepth = max_depth;
  if (isSet(clamp)) r.clampVal = (float)clamp;
  if (seed >= 0) r.seed = (unsigned)seed;
  if (isSet(exposure)) r.exposure = (float)exposure;
  if (transparent_shadows >= 0) r.transparentShadows = transparent_shadows == 1;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

// src/capi_scene.cpp:51-67
extern "C" int sundog_set_camera(sundog_scene* h, const double lookfrom[3], const double lookat[3],
                                 const double up[3], double vfov, double aperture,
                                 double focus_dist) {
  SDB_TRY
  enterPhase(h, 0, "camera");
  if (!lookfrom || !lookat) sceneError("camera: lookfrom and lookat are required");
  CameraCfg& c = h->scene.camera;
  c.lookfrom = nf3(lookfrom, c.lookfrom);
  c.lookat = nf3(lookat, c.lookat);
  c.up = nf3(up, c.up);
  c.vfov = nf(vfov, 40.0f);
  c.aperture = nf(aperture, 0.0f);
  c.focusDist = nf(focus_dist, 0.0f);
  h->hasCamera = true;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

// src/capi_scene.cpp:69-106
extern "C" int sundog_set_background_solid(sundog_scene* h, const double color[3]) {
  SDB_TRY
  enterPhase(h, 0, "background");
  if (!color) sceneError("background: color is required");
  h->scene.bgKind = BG_SOLID;
  h->scene.bgA = nf3(color, v3(0.0f));
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_set_background_gradient(sundog_scene* h, const double horizon[3],
                                              const double zenith[3]) {
  SDB_TRY
  enterPhase(h, 0, "background");
  if (!horizon || !zenith) sceneError("background: horizon and zenith are required");
  h->scene.bgKind = BG_GRADIENT;
  h->scene.bgA = nf3(horizon, v3(0.0f));
  h->scene.bgB = nf3(zenith, v3(0.0f));
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_set_background_envmap(sundog_scene* h, const char* file, double rotate_deg,
                                            double intensity, int importance) {
  SDB_TRY
  enterPhase(h, 0, "background");
  if (!file || !*file) sceneError("envmap: file is required");
  h->scene.bgKind = BG_ENVMAP;
  h->scene.env.file = file;
  h->scene.env.rotateDeg = nf(rotate_deg, 0.0f);
  h->scene.env.intensity = nf(intensity, 1.0f);
  h->scene.env.importance = importance != 0;
  if (h->scene.env.intensity < 0.0f) sceneError("envmap: intensity must be >= 0");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

// src/capi_scene.cpp:108-132
extern "C" int sundog_set_physics(sundog_scene* h, const double gravity[3], double timestep,
                                  double max_time, double friction, double restitution,
                                  int pos_iters, int vel_iters, double sleep_threshold,
                                  double stop_time) {
  SDB_TRY
  enterPhase(h, 0, "physics settings");
  PhysicsCfg& p = h->scene.physics;
  p.enabled = true;
  p.gravity = nf3(gravity, p.gravity);
  p.timestep = nf(timestep, p.timestep);
  p.maxTime = nf(max_time, p.maxTime);
  p.friction = nf(friction, p.friction);
  p.restitution = nf(restitution, p.restitution);
  if (pos_iters >= 0) p.posIters = pos_iters;
  if (vel_iters >= 0) p.velIters = vel_iters;
  p.sleepThreshold = nf(sleep_threshold, p.sleepThreshold);
  p.stopTime = nf(stop_time, p.stopTime);
  if (p.timestep <= 0.0f || p.maxTime <= 0.0f)
    sceneError("physics: timestep and max_time must be positive");
  if (p.stopTime < 0.0f) sceneError("physics: stop_time must be >= 0 (0 = settle to sleep)");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

// src/capi_scene.cpp:143-195
extern "C" int sundog_add_texture_solid(sundog_scene* h, const double color[3]) {
  SDB_TRY
  if (!color) sceneError("texture: color is required");
  TextureCfg t;
  t.desc.width = 0.05f;
  t.desc.kind = TX_SOLID;
  t.desc.a = nf3(color, v3(0.0f));
  return pushTexture(h, t);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_texture_checker(sundog_scene* h, const double a[3], const double b[3],
                                          const double scale[2]) {
  SDB_TRY
  if (!a || !b) sceneError("texture: a and b are required");
  TextureCfg t;
  t.desc.width = 0.05f;
  t.desc.kind = TX_CHECKER;
  t.desc.a = nf3(a, v3(0.0f));
  t.desc.b = nf3(b, v3(0.0f));
  t.desc.scale = scale ? make_float2((float)scale[0], (float)scale[1]) : make_float2(8.0f, 8.0f);
  return pushTexture(h, t);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_texture_grid(sundog_scene* h, const double a[3], const double b[3],
                                       const double scale[2], double width) {
  SDB_TRY
  if (!a || !b) sceneError("texture: a and b are required");
  TextureCfg t;
  t.desc.kind = TX_GRID;
  t.desc.a = nf3(a, v3(0.0f));
  t.desc.b = nf3(b, v3(0.0f));
  t.desc.scale = scale ? make_float2((float)scale[0], (float)scale[1]) : make_float2(8.0f, 8.0f);
  t.desc.width = nf(width, 0.05f);
  return pushTexture(h, t);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_texture_image(sundog_scene* h, const char* file, int srgb) {
  SDB_TRY
  if (!file || !*file) sceneError("texture: file is required");
  TextureCfg t;
  t.desc.width = 0.05f;
  t.desc.kind = TX_IMAGE;
  t.file = file;
  t.srgb = srgb != 0;
  return pushTexture(h, t);
  SDB_CATCH(-1)
}

// src/capi_scene.cpp:218-314
extern "C" int sundog_add_material_lambert(sundog_scene* h, const double color[3], int tex_id) {
  SDB_TRY
  SdMaterial m = baseMaterial();
  m.kind = MT_LAMBERT;
  m.color = nf3(color, m.color);
  m.texId = tex_id;
  return pushMaterial(h, m, tex_id);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_material_metal(sundog_scene* h, const double color[3], int tex_id,
                                         double roughness) {
  SDB_TRY
  SdMaterial m = baseMaterial();
  m.kind = MT_METAL;
  m.color = nf3(color, m.color);
  m.texId = tex_id;
  m.roughness = nf(roughness, m.roughness);
  return pushMaterial(h, m, tex_id);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_material_dielectric(sundog_scene* h, double ior, const double absorb[3],
                                              const double color[3], int tex_id,
                                              double roughness) {
  SDB_TRY
  SdMaterial m = baseMaterial();
  m.kind = MT_DIELECTRIC;
  m.color = nf3(color, m.color);
  m.texId = tex_id;
  m.ior = nf(ior, m.ior);
  m.roughness = nf(roughness, m.roughness);
  if (absorb) {
    m.absorb = nf3(absorb, v3(0.0f));
    if (m.absorb.x < 0.0f || m.absorb.y < 0.0f || m.absorb.z < 0.0f)
      sceneError("dielectric: absorb components must be >= 0");
  }
  return pushMaterial(h, m, tex_id);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_material_emissive(sundog_scene* h, const double color[3], int tex_id,
                                            double intensity, int two_sided) {
  SDB_TRY
  SdMaterial m = baseMaterial();
  m.kind = MT_EMISSIVE;
  m.color = nf3(color, m.color);
  m.texId = tex_id;
  m.intensity = nf(intensity, m.intensity);
  if (m.intensity < 0.0f) sceneError("emissive: intensity must be >= 0");
  m.twoSided = two_sided == 1 ? 1 : 0;
  return pushMaterial(h, m, tex_id);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_material_water(sundog_scene* h, double ior, const double absorb[3],
                                         double wave_amp, double wave_freq,
                                         const double color[3]) {
  SDB_TRY
  SdMaterial m = baseMaterial();
  m.kind = MT_WATER;
  m.ior = nf(ior, 1.33f);
  m.absorb = nf3(absorb, v3(0.45f, 0.08f, 0.035f));
  m.waveAmp = nf(wave_amp, 0.05f);
  m.waveFreq = nf(wave_freq, 2.0f);
  m.color = nf3(color, v3(1.0f));
  m.texId = -1;
  if (m.waveAmp < 0.0f || m.waveFreq < 0.0f)
    sceneError("water: wave_amp and wave_freq must be >= 0");
  if (m.absorb.x < 0.0f || m.absorb.y < 0.0f || m.absorb.z < 0.0f)
    sceneError("water: absorb components must be >= 0");
  return pushMaterial(h, m, -1);
  SDB_CATCH(-1)
}

extern "C" int sundog_add_material_plastic(sundog_scene* h, const double color[3], int tex_id,
                                           double roughness) {
  SDB_TRY
  SdMaterial m = baseMaterial();
  m.kind = MT_PLASTIC;
  m.color = nf3(color, m.color);
  m.texId = tex_id;
  m.roughness = nf(roughness, 0.15f);
  return pushMaterial(h, m, tex_id);
  SDB_CATCH(-1)
}

// src/capi_scene.cpp:316-329
extern "C" int sundog_add_mesh(sundog_scene* h, const char* obj_file, int smooth_normals,
                               const char* usemtl) {
  SDB_TRY
  enterPhase(h, 0, "meshes");
  if (!obj_file || !*obj_file) sceneError("mesh: obj file is required");
  MeshCfg m;
  m.file = obj_file;
  m.usemtl = usemtl ? usemtl : "";
  m.smooth = smooth_normals != 0;
  int id = (int)h->scene.meshes.size();
  h->scene.meshes.push_back(m);
  return id;
  SDB_CATCH(-1)
}

// src/capi_scene.cpp:333-390
extern "C" int sundog_add_object(sundog_scene* h, int geom_kind, int mesh_id, int mat_front,
                                 int mat_back, int cutout_tex_id, const sundog_xform_step* steps,
                                 int num_steps, int nee, const sundog_physics_body* physics) {
  SDB_TRY
  enterPhase(h, 1, "objects");
  SceneDesc& s = h->scene;
  ObjectCfg o;
  if (geom_kind < 0 || geom_kind > GK_MESH) sceneError("object: unknown shape");
  o.kind = geom_kind;
  if (geom_kind == GK_MESH) {
    if (mesh_id < 0 || mesh_id >= (int)s.meshes.size()) sceneError("object: mesh id out of range");
    o.mesh = mesh_id;
  }
  auto matOf = [&](int id) -> uint16_t {
    if (id == SUNDOG_MAT_NONE) return kMatNone;
    if (id < 0 || id >= (int)s.materials.size()) sceneError("object: material id out of range");
    return (uint16_t)id;
  };
  o.matFront = matOf(mat_front);
  o.matBack = mat_back == SUNDOG_MAT_DEFAULT ? o.matFront : matOf(mat_back);
  if (cutout_tex_id != -1) {
    if (cutout_tex_id < 0 || cutout_tex_id >= (int)s.textures.size())
      sceneError("object: cutout texture id out of range");
    o.cutoutTex = cutout_tex_id;
  }
  if (num_steps > 0 && !steps) sceneError("object: transform steps missing");
  std::vector<XformStepF> xs((size_t)std::max(num_steps, 0));
  for (int i = 0; i < num_steps; i++) {
    xs[i].kind = steps[i].kind;
    xs[i].a = (float)steps[i].a;
    xs[i].b = (float)steps[i].b;
    xs[i].c = (float)steps[i].c;
  }
  o.xform = composeSteps(xs.data(), num_steps);
  o.nee = nee != 0;
  if (physics) {
    o.body.enabled = true;
    o.body.dynamic = physics->dynamic == 1;
    o.body.density = nf(physics->density, o.body.density);
    if (physics->has_velocity) o.body.velocity = nf3(physics->velocity, o.body.velocity);
    if (physics->has_angular_velocity)
      o.body.angularVelocity = nf3(physics->angular_velocity, o.body.angularVelocity);
    o.body.friction = nf(physics->friction, o.body.friction);
    o.body.restitution = nf(physics->restitution, o.body.restitution);
    o.body.thickness = nf(physics->thickness, o.body.thickness);
  }
  int id = (int)s.objects.size();
  registerObject(s, o);
  return id;
  SDB_CATCH(-1)
}

// src/capi_scene.cpp:392-412
extern "C" int sundog_add_flame(sundog_scene* h, const double base[3], double height,
                                double radius, double intensity, double sigma, double noise_scale,
                                int64_t seed, double light_intensity) {
  SDB_TRY
  enterPhase(h, 2, "flames");
  if (!base) sceneError("flame: base is required");
  SdFlame f{};
  f.base = nf3(base, v3(0.0f));
  f.height = (float)height;
  f.radius = (float)radius;
  f.intensity = nf(intensity, 20.0f);
  f.sigma = nf(sigma, 4.0f);
  f.noiseScale = nf(noise_scale, 3.0f);
  f.seed = seed >= 0 ? (unsigned)seed : 0u;
  f.steps = 32;
  float li = nf(light_intensity, 12.0f);
  int id = (int)h->scene.flames.size();
  registerFlame(h->scene, f, li);
  return id;
  SDB_CATCH(-1)
}

// src/capi_scene.cpp:414-451
extern "C" int sundog_add_point_light(sundog_scene* h, const double position[3],
                                      const double intensity[3], double radius) {
  SDB_TRY
  enterPhase(h, 3, "lights");
  if (!position || !intensity) sceneError("point light: position and intensity are required");
  SdLight l{};
  l.texId = -1;
  l.flameId = -1;
  l.kind = LT_POINT;
  l.p = nf3(position, v3(0.0f));
  l.radius = nf(radius, 0.0f);
  l.L = nf3(intensity, v3(0.0f));
  if (l.L.x < 0.0f || l.L.y < 0.0f || l.L.z < 0.0f)
    sceneError("point light: intensity components must be >= 0");
  int id = (int)h->scene.lights.size();
  h->scene.lights.push_back(l);
  return id;
  SDB_CATCH(-1)
}

extern "C" int sundog_add_distant_light(sundog_scene* h, const double direction[3],
                                        const double radiance[3]) {
  SDB_TRY
  enterPhase(h, 3, "lights");
  if (!direction || !radiance) sceneError("distant light: direction and radiance are required");
  SdLight l{};
  l.texId = -1;
  l.flameId = -1;
  l.kind = LT_DISTANT;
  l.dir = unit(nf3(direction, v3(0.0f)));
  l.L = nf3(radiance, v3(0.0f));
  if (l.L.x < 0.0f || l.L.y < 0.0f || l.L.z < 0.0f)
    sceneError("distant light: radiance components must be >= 0");
  int id = (int)h->scene.lights.size();
  h->scene.lights.push_back(l);
  return id;
  SDB_CATCH(-1)
}

// src/capi_scene.cpp:453-458
extern "C" int sundog_scene_validate(sundog_scene* h) {
  SDB_TRY
  if (!h) throw std::runtime_error("scene: null handle");
  if (!h->hasCamera) sceneError("missing camera");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

// ---- additive entry points ------------------------------------------------------

extern "C" int sundog_set_flame_steps(sundog_scene* h, int flame_id, int steps) {
  SDB_TRY
  if (!h) throw std::runtime_error("scene: null handle");
  if (flame_id < 0 || flame_id >= (int)h->scene.flames.size())
    sceneError("flame steps: flame id out of range");
  if (steps < 1 || steps > 1024) sceneError("flame steps: must be in 1..1024");
  h->scene.flames[flame_id].steps = steps;
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

namespace {
void jf(std::ostringstream& o, float v) {
  if (std::isfinite(v)) {
    char b[48];
    std::snprintf(b, sizeof b, "%.9g", (double)v);
    o << b;
  } else {
    o << "null";
  }
}
void jv(std::ostringstream& o, float3 v) {
  o << "[";
  jf(o, v.x);
  o << ",";
  jf(o, v.y);
  o << ",";
  jf(o, v.z);
  o << "]";
}
std::string jstr(const std::string& s) {
  std::string r = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') {
      r += '\\';
      r += c;
    } else if ((unsigned char)c < 0x20) {
      char b[8];
      std::snprintf(b, sizeof b, "\\u%04x", c);
      r += b;
    } else {
      r += c;
    }
  }
  return r + "\"";
}
}  // namespace

extern "C" int sundog_scene_debug_json(sundog_scene* h, char* buf, size_t cap, size_t* needed) {
  SDB_TRY
  if (!h) throw std::runtime_error("scene: null handle");
  const SceneDesc& s = h->scene;
  std::ostringstream o;
  const RenderCfg& r = s.render;
  o << "{\"render\":{\"width\":" << r.width << ",\"height\":" << r.height << ",\"spp\":" << r.spp
    << ",\"max_depth\":" << r.maxDepth << ",\"clamp\":";
  jf(o, r.clampVal);
  o << ",\"seed\":" << r.seed << ",\"exposure\":";
  jf(o, r.exposure);
  o << ",\"transparent_shadows\":" << (r.transparentShadows ? 1 : 0) << "},";
  const CameraCfg& c = s.camera;
  o << "\"camera\":{\"lookfrom\":";
  jv(o, c.lookfrom);
  o << ",\"lookat\":";
  jv(o, c.lookat);
  o << ",\"up\":";
  jv(o, c.up);
  o << ",\"vfov\":";
  jf(o, c.vfov);
  o << ",\"aperture\":";
  jf(o, c.aperture);
  o << ",\"focus_dist\":";
  jf(o, c.focusDist);
  SdCamera cd = buildCamera(c, r.width, r.height);
  o << ",\"frame\":{\"origin\":";
  jv(o, cd.origin);
  o << ",\"lower_left\":";
  jv(o, cd.lowerLeft);
  o << ",\"horizontal\":";
  jv(o, cd.horizontal);
  o << ",\"vertical\":";
  jv(o, cd.vertical);
  o << ",\"u\":";
  jv(o, cd.u);
  o << ",\"v\":";
  jv(o, cd.v);
  o << ",\"w\":";
  jv(o, cd.w);
  o << ",\"lens_radius\":";
  jf(o, cd.lensRadius);
  o << "}},\"has_camera\":" << (h->hasCamera ? 1 : 0) << ",\"phase\":" << h->phase;
  o << ",\"base_dir\":" << jstr(s.baseDir);
  o << ",\"background\":{\"kind\":" << s.bgKind << ",\"a\":";
  jv(o, s.bgA);
  o << ",\"b\":";
  jv(o, s.bgB);
  o << ",\"env_file\":" << jstr(s.env.file) << ",\"env_rotate_deg\":";
  jf(o, s.env.rotateDeg);
  o << ",\"env_intensity\":";
  jf(o, s.env.intensity);
  o << ",\"env_importance\":" << (s.env.importance ? 1 : 0) << "}";
  o << ",\"textures\":[";
  for (size_t i = 0; i < s.textures.size(); i++) {
    const TextureCfg& t = s.textures[i];
    if (i) o << ",";
    o << "{\"kind\":" << t.desc.kind << ",\"a\":";
    jv(o, t.desc.a);
    o << ",\"b\":";
    jv(o, t.desc.b);
    o << ",\"scale\":[";
    jf(o, t.desc.scale.x);
    o << ",";
    jf(o, t.desc.scale.y);
    o << "],\"width\":";
    jf(o, t.desc.width);
    o << ",\"file\":" << jstr(t.file) << ",\"srgb\":" << (t.srgb ? 1 : 0) << "}";
  }
  o << "],\"materials\":[";
  for (size_t i = 0; i < s.materials.size(); i++) {
    const SdMaterial& m = s.materials[i];
    if (i) o << ",";
    o << "{\"kind\":" << m.kind << ",\"tex\":" << m.texId << ",\"color\":";
    jv(o, m.color);
    o << ",\"roughness\":";
    jf(o, m.roughness);
    o << ",\"ior\":";
    jf(o, m.ior);
    o << ",\"intensity\":";
    jf(o, m.intensity);
    o << ",\"two_sided\":" << m.twoSided << ",\"absorb\":";
    jv(o, m.absorb);
    o << ",\"wave_amp\":";
    jf(o, m.waveAmp);
    o << ",\"wave_freq\":";
    jf(o, m.waveFreq);
    o << "}";
  }
  o << "],\"meshes\":[";
  for (size_t i = 0; i < s.meshes.size(); i++) {
    if (i) o << ",";
    o << "{\"file\":" << jstr(s.meshes[i].file) << ",\"usemtl\":" << jstr(s.meshes[i].usemtl)
      << ",\"smooth\":" << (s.meshes[i].smooth ? 1 : 0) << "}";
  }
  o << "],\"objects\":[";
  for (size_t i = 0; i < s.objects.size(); i++) {
    const ObjectCfg& ob = s.objects[i];
    if (i) o << ",";
    o << "{\"kind\":" << ob.kind << ",\"mesh\":" << ob.mesh << ",\"mat_front\":" << ob.matFront
      << ",\"mat_back\":" << ob.matBack << ",\"cutout\":" << ob.cutoutTex
      << ",\"light\":" << ob.lightId << ",\"nee\":" << (ob.nee ? 1 : 0) << ",\"xform\":[";
    for (int k = 0; k < 12; k++) {
      if (k) o << ",";
      jf(o, ob.xform.m[k]);
    }
    o << "],\"physics\":" << (ob.body.enabled ? 1 : 0) << ",\"dynamic\":" << (ob.body.dynamic ? 1 : 0)
      << ",\"density\":";
    jf(o, ob.body.density);
    o << ",\"thickness\":";
    jf(o, ob.body.thickness);
    o << "}";
  }
  o << "],\"lights\":[";
  for (size_t i = 0; i < s.lights.size(); i++) {
    const SdLight& l = s.lights[i];
    if (i) o << ",";
    o << "{\"kind\":" << l.kind << ",\"p\":";
    jv(o, l.p);
    o << ",\"u\":";
    jv(o, l.u);
    o << ",\"v\":";
    jv(o, l.v);
    o << ",\"n\":";
    jv(o, l.n);
    o << ",\"L\":";
    jv(o, l.L);
    o << ",\"radius\":";
    jf(o, l.radius);
    o << ",\"area\":";
    jf(o, l.area);
    o << ",\"dir\":";
    jv(o, l.dir);
    o << ",\"two_sided\":" << l.twoSided << ",\"tex\":" << l.texId << ",\"flame\":" << l.flameId
      << "}";
  }
  o << "],\"flames\":[";
  for (size_t i = 0; i < s.flames.size(); i++) {
    const SdFlame& f = s.flames[i];
    if (i) o << ",";
    o << "{\"base\":";
    jv(o, f.base);
    o << ",\"height\":";
    jf(o, f.height);
    o << ",\"radius\":";
    jf(o, f.radius);
    o << ",\"intensity\":";
    jf(o, f.intensity);
    o << ",\"sigma\":";
    jf(o, f.sigma);
    o << ",\"noise_scale\":";
    jf(o, f.noiseScale);
    o << ",\"seed\":" << f.seed << ",\"steps\":" << f.steps << "}";
  }
  const PhysicsCfg& p = s.physics;
  o << "],\"physics\":{\"enabled\":" << (p.enabled ? 1 : 0) << ",\"gravity\":";
  jv(o, p.gravity);
  o << ",\"timestep\":";
  jf(o, p.timestep);
  o << ",\"max_time\":";
  jf(o, p.maxTime);
  o << ",\"stop_time\":";
  jf(o, p.stopTime);
  o << ",\"friction\":";
  jf(o, p.friction);
  o << ",\"restitution\":";
  jf(o, p.restitution);
  o << ",\"pos_iters\":" << p.posIters << ",\"vel_iters\":" << p.velIters << "}}";
  std::string js = o.str();
  if (needed) *needed = js.size() + 1;
  if (buf && cap > 0) {
    size_t n = std::min(cap - 1, js.size());
    std::memcpy(buf, js.data(), n);
    buf[n] = '\0';
  }
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}
