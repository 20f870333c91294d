// Scene derivation shared by the scene-construction ABI: camera frame,
// transform composition, automatic NEE light registration for emissive
// objects, flame point lights. The float arithmetic follows
// src/scene_build.cpp operation for operation (same narrowing point, same
// order) because light frames and transforms feed the sampled image directly.
#include <cmath>
#include <stdexcept>

#include "scene_model.h"

namespace sdb {

void sceneError(const std::string& msg) { throw std::runtime_error("scene: " + msg); }

SdCamera buildCamera(const CameraCfg& cs, int width, int height) {
  SdCamera c{};
  float aspect = (float)width / (float)height;
  float theta = cs.vfov * kPi / 180.0f;
  float halfH = tanf(theta / 2.0f);
  float halfW = aspect * halfH;
  float focus = cs.focusDist > 0.0f ? cs.focusDist : len(cs.lookfrom - cs.lookat);
  c.w = unit(cs.lookfrom - cs.lookat);
  c.u = unit(cross(cs.up, c.w));
  c.v = cross(c.w, c.u);
  c.origin = cs.lookfrom;
  c.lowerLeft = c.origin - halfW * focus * c.u - halfH * focus * c.v - focus * c.w;
  c.horizontal = 2.0f * halfW * focus * c.u;
  c.vertical = 2.0f * halfH * focus * c.v;
  c.lensRadius = cs.aperture / 2.0f;
  return c;
}

static Xform xfScale(float3 s) {
  Xform x = {{s.x, 0, 0, 0, 0, s.y, 0, 0, 0, 0, s.z, 0}};
  return x;
}
static Xform xfTranslate(float3 t) {
  Xform x = {{1, 0, 0, t.x, 0, 1, 0, t.y, 0, 0, 1, t.z}};
  return x;
}
static Xform xfRotX(float r) {
  float c = cosf(r), s = sinf(r);
  Xform x = {{1, 0, 0, 0, 0, c, -s, 0, 0, s, c, 0}};
  return x;
}
static Xform xfRotY(float r) {
  float c = cosf(r), s = sinf(r);
  Xform x = {{c, 0, s, 0, 0, 1, 0, 0, -s, 0, c, 0}};
  return x;
}
static Xform xfRotZ(float r) {
  float c = cosf(r), s = sinf(r);
  Xform x = {{c, -s, 0, 0, s, c, 0, 0, 0, 0, 1, 0}};
  return x;
}

Xform composeSteps(const XformStepF* steps, int n) {
  Xform m = Xform::ident();
  const float d2r = kPi / 180.0f;
  for (int i = 0; i < n; i++) {
    const XformStepF& st = steps[i];
    Xform step;
    switch (st.kind) {
      case 0: step = xfScale(v3(st.a, st.b, st.c)); break;
      case 1: step = xfTranslate(v3(st.a, st.b, st.c)); break;
      case 2: step = xfRotX(st.a * d2r); break;
      case 3: step = xfRotY(st.a * d2r); break;
      case 4: step = xfRotZ(st.a * d2r); break;
      default: sceneError("unknown transform step kind");
    }
    m = compose(step, m);
  }
  return m;
}

static const char* kindName(int k) {
  switch (k) {
    case GK_SPHERE: return "sphere";
    case GK_RECT: return "rect";
    case GK_DISK: return "disk";
    case GK_CYLINDER: return "cylinder";
    case GK_PARABOLA: return "parabola";
    default: return "mesh";
  }
}

void registerObject(SceneDesc& s, ObjectCfg& o) {
  if (o.matFront == kMatNone && o.matBack == kMatNone)
    sceneError("object has no material on either face");
  if (o.body.enabled) {
    if (!s.physics.enabled)
      sceneError("physics: object opts in but the scene has no top-level physics block");
    if (o.kind == GK_DISK || o.kind == GK_CYLINDER || o.kind == GK_PARABOLA)
      sceneError(std::string("physics: shape '") + kindName(o.kind) +
                 "' is not supported as a collider (use sphere, rect, or mesh)");
    if (o.kind == GK_RECT && o.body.dynamic)
      sceneError("physics: rect colliders are static-only (zero-thickness plates tunnel)");
    if (o.body.dynamic && o.body.density <= 0.0f)
      sceneError("physics: dynamic body needs positive density");
    if (o.body.thickness <= 0.0f) sceneError("physics: thickness must be positive");
  }

  uint16_t em = kMatNone;
  if (o.matFront != kMatNone && s.materials[o.matFront].kind == MT_EMISSIVE) em = o.matFront;
  bool light = em != kMatNone && o.nee &&
               (o.kind == GK_RECT || o.kind == GK_DISK || o.kind == GK_SPHERE || o.kind == GK_MESH);
  if (o.body.dynamic && light)
    sceneError("physics: a dynamic object cannot be an NEE area light (the light frame is "
               "baked at parse time); set nee:false or keep it static");
  if (o.cutoutTex >= 0 && light)
    sceneError("an alpha-cutout object cannot be an NEE area light (NEE would sample "
               "emission inside the holes); set nee:false");
  if (light) {
    const SdMaterial& m = s.materials[em];
    SdLight ld{};
    ld.texId = -1;
    ld.flameId = -1;
    ld.p = o.xform.point(v3(0, 0, 0));
    float3 ux = o.xform.vec(v3(1, 0, 0));
    float3 uy = o.xform.vec(v3(0, 1, 0));
    float3 uz = o.xform.vec(v3(0, 0, 1));
    float sg = orientSign(ux, uy, uz);
    ld.L = m.color * m.intensity;
    ld.twoSided = m.twoSided;
    if (m.texId >= 0) {
      if (o.kind == GK_SPHERE)
        sceneError("textured emissive sphere cannot be an NEE light (uv frame is "
                   "object-space); use a solid color or set nee:false");
      ld.texId = m.texId;
      ld.L = v3(m.intensity);
    }
    if (o.kind == GK_RECT) {
      ld.kind = LT_RECT;
      ld.u = ux;
      ld.v = uz;
      ld.n = unit(cross(uz, ux)) * sg;
      ld.area = 4.0f * len(cross(ux, uz));
    } else if (o.kind == GK_DISK) {
      float ru = len(ux), rz = len(uz);
      if (fabsf(ru - rz) > 1e-3f * fmaxf(ru, rz))
        sceneError("disk NEE light requires uniform XZ scale (pdf would be wrong); set nee:false");
      ld.kind = LT_DISK;
      ld.u = ux;
      ld.v = uz;
      ld.n = unit(cross(uz, ux)) * sg;
      ld.area = kPi * ru * rz;
    } else if (o.kind == GK_SPHERE) {
      float rx = len(ux), rz = len(uz);
      float ry = len(o.xform.vec(v3(0, 1, 0)));
      if (fabsf(rx - ry) > 1e-3f * rx || fabsf(rx - rz) > 1e-3f * rx)
        sceneError("sphere NEE light requires uniform scale; set nee:false");
      ld.kind = LT_SPHERE;
      ld.radius = rx;
    } else {
      // Mesh light: geometry, CDF and area are filled in at render time once
      // the OBJ is loaded; the light-list slot is fixed now.
      ld.kind = LT_MESH;
    }
    o.lightId = (int)s.lights.size();
    s.lights.push_back(ld);
  }
  s.objects.push_back(o);
}

void registerFlame(SceneDesc& s, const SdFlame& f, float lightIntensity) {
  if (f.height <= 0.0f || f.radius <= 0.0f) sceneError("flame: height and radius must be positive");
  if (f.intensity < 0.0f || f.sigma < 0.0f) sceneError("flame: intensity and sigma must be >= 0");
  const float frac[2] = {0.65f, 0.35f};
  const float hfac[2] = {0.35f, 0.70f};
  const float3 warm[2] = {v3(1.0f, 0.50f, 0.15f), v3(1.0f, 0.62f, 0.25f)};
  for (int k = 0; k < 2; k++) {
    SdLight ld{};
    ld.texId = -1;
    ld.flameId = (int)s.flames.size();
    ld.kind = LT_POINT;
    ld.p = f.base + v3(0.0f, hfac[k] * f.height, 0.0f);
    ld.radius = 0.3f * f.radius;
    ld.L = warm[k] * (lightIntensity * frac[k]);
    s.lights.push_back(ld);
  }
  s.flames.push_back(f);
}

}  // namespace sdb
