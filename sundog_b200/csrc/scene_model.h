// Host-side scene state behind a sundog_scene handle, as built by the C ABI
// scene-construction calls (scene_api.cpp) and consumed by the render
// orchestration (render.cpp). Defaults are the reference renderer's
// (src/scene.h:11-21, src/capi_scene.cpp:197-314).
#pragma once

#include <string>
#include <vector>

#include "sd_types.h"

namespace sdb {

struct RenderCfg {
  int width = 1280, height = 720;
  int spp = 64;
  int maxDepth = 16;
  float clampVal = 50.0f;
  unsigned seed = 7;
  float exposure = 0.0f;
  bool transparentShadows = true;
  bool denoise = false;
};

struct CameraCfg {
  float3 lookfrom{0, 2, 8}, lookat{0, 0, 0}, up{0, 1, 0};
  float vfov = 40.0f;
  float aperture = 0.0f;
  float focusDist = 0.0f;  // 0: |lookfrom - lookat|
};

struct TextureCfg {
  SdTexture desc{};
  std::string file;  // TX_IMAGE
  bool srgb = true;
};

struct EnvCfg {
  std::string file;
  float rotateDeg = 0.0f;
  float intensity = 1.0f;
  bool importance = true;
};

struct MeshCfg {
  std::string file;
  std::string usemtl;
  bool smooth = true;
};

struct BodyCfg {
  bool enabled = false;
  bool dynamic = false;
  float density = 250.0f;
  float3 velocity{0, 0, 0}, angularVelocity{0, 0, 0};
  float friction = -1.0f, restitution = -1.0f;
  float thickness = 0.2f;
};

struct PhysicsCfg {
  bool enabled = false;
  float3 gravity{0.0f, -9.81f, 0.0f};
  float timestep = 1.0f / 240.0f;
  float maxTime = 15.0f;
  float stopTime = 0.0f;
  float friction = 0.6f, restitution = 0.1f;
  int posIters = 8, velIters = 2;
  float sleepThreshold = -1.0f;
};

struct ObjectCfg {
  int kind = GK_SPHERE;
  int mesh = -1;
  uint16_t matFront = kMatNone, matBack = kMatNone;
  int cutoutTex = -1;
  Xform xform = Xform::ident();
  int lightId = -1;
  bool nee = true;
  BodyCfg body;
};

struct SceneDesc {
  RenderCfg render;
  CameraCfg camera;
  int bgKind = BG_SOLID;
  float3 bgA{0, 0, 0}, bgB{0, 0, 0};
  EnvCfg env;
  std::vector<TextureCfg> textures;
  std::vector<SdMaterial> materials;
  std::vector<MeshCfg> meshes;
  std::vector<ObjectCfg> objects;
  std::vector<SdLight> lights;
  std::vector<SdFlame> flames;
  PhysicsCfg physics;
  std::string baseDir;
};

// Glass and water faces transmit shadow rays (src/scene.h:100-107).
inline bool matTransmissive(const SceneDesc& s, uint16_t m) {
  return m != kMatNone &&
         (s.materials[m].kind == MT_DIELECTRIC || s.materials[m].kind == MT_WATER);
}

// Thin-lens look-at camera (src/scene_build.cpp:13-29).
SdCamera buildCamera(const CameraCfg& c, int width, int height);

// Step-by-step transform composition, later steps wrapping earlier ones
// (src/scene_build.cpp:31-48).
struct XformStepF {
  int kind;
  float a, b, c;
};
Xform composeSteps(const XformStepF* steps, int n);

// NEE light registration and physics-collider checks for a new object
// (src/scene_build.cpp:61-153); throws std::runtime_error("scene: ...").
void registerObject(SceneDesc& s, ObjectCfg& o);

// Domain checks, the two embedded point lights, append
// (src/scene_build.cpp:155-181).
void registerFlame(SceneDesc& s, const SdFlame& f, float lightIntensity);

[[noreturn]] void sceneError(const std::string& msg);

}  // namespace sdb

// The opaque ABI handle: scene plus the call-order phase
// (0 config/registries, 1 objects, 2 flames, 3 explicit lights).
struct sundog_scene {
  sdb::SceneDesc scene;
  int phase = 0;
  bool hasCamera = false;
};
