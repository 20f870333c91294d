// ORACLE — test infrastructure only (the checker, never the product).
//
// Function-vector harness: evaluates one hot-path function of the device
// math over a batch of packed items. Compiled two ways by oracle/Makefile:
//   * against the oracle's restatement (oracle/sdo/sdo.h) into
//     libsdoracle.so as sdo_fn(), and
//   * with -DSDO_USE_REFERENCE against sundog's own device headers
//     (device/rng.cuh, bsdf.cuh, intersect.cuh, light_sample.cuh,
//     env_light.cuh, noise.cuh, volume.cuh, read in place) into the
//     oracle/_ref/fnvec_ref executable, whose outputs become the golden
//     vectors in tests/golden/.
// Item layouts are byte-identical to the device self-test items in
// sundog_b200/csrc/selftest.cu, so one packed input feeds the reference, the
// oracle and the GPU.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef SDO_USE_REFERENCE
#include <algorithm>
using std::min;
#include "rng.cuh"
#include "bsdf.cuh"
#include "intersect.cuh"
#include "light_sample.cuh"
#include "env_light.cuh"
#include "noise.cuh"
#include "volume.cuh"
namespace M = sd;
#else
#include "sdo/sdo.h"
namespace M = sdo;
#endif

namespace {

struct V3 { float x, y, z; };
struct PMat { int kind, texId; V3 color; float roughness, ior, intensity; int twoSided; V3 absorb; float waveAmp, waveFreq; };
struct PLight { int kind; V3 p, u, v, n, L; float radius, area; V3 dir; int twoSided, texId, flameId; uint64_t ptr[4]; int numTris; float ngSign; };
struct PFlame { V3 base; float height, radius, intensity, sigma, noiseScale; unsigned seed; int steps; };

struct PcgIn { uint64_t seed, seq; };
struct PcgOut { uint32_t next[8]; float uni[4]; };
struct EvalIn { PMat m; V3 albedo, wo, wi, n; float eta; };
struct EvalOut { V3 f; float pdf; };
struct DrawIn { PMat m; V3 albedo, d, n; int front; float etaExt; uint64_t state, inc; };
struct DrawOut { V3 wi, weight; float pdf; int delta, ok; uint32_t pad; uint64_t state; };
struct QuadIn { int kind; V3 o, d; float tmin, tmax; };
struct QuadOut { int count; float t0; V3 n0; float u0, v0, t1; V3 n1; float u1, v1; };
struct LightIn { PLight l; V3 x; uint64_t state, inc; };
struct LightOut { V3 wi, Li; float dist, pdf; int delta, ok; uint64_t state; float density, pad; };
struct FlameIn { PFlame f; V3 o, d; float tEnd; int skip; uint64_t state, inc; };
struct FlameOut { V3 Lv, trans; float tr; int pad; uint64_t stateMarch, stateShadow; };
struct NoiseIn { V3 p; unsigned seed; V3 ns, wo; float amp, freq; };
struct NoiseOut { float fbm, vnoise; V3 wave; };

static_assert(sizeof(PMat) == 56, "material item layout");
static_assert(sizeof(PLight) == 136, "light item layout");
static_assert(sizeof(PFlame) == 40, "flame item layout");
static_assert(sizeof(EvalIn) == 108 && sizeof(DrawIn) == 120 && sizeof(DrawOut) == 48, "bsdf items");
static_assert(sizeof(QuadIn) == 36 && sizeof(QuadOut) == 52, "quadric items");
static_assert(sizeof(LightIn) == 168 && sizeof(LightOut) == 56, "light items");
static_assert(sizeof(FlameIn) == 88 && sizeof(FlameOut) == 48, "flame items");
static_assert(sizeof(NoiseIn) == 48 && sizeof(NoiseOut) == 20, "noise items");

template <class T> T f3(const V3& v) { T r; r.x = v.x; r.y = v.y; r.z = v.z; return r; }
template <class T> V3 v3(const T& v) { return V3{v.x, v.y, v.z}; }

M::MaterialDesc mat(const PMat& p) {
  M::MaterialDesc m;
  std::memset(&m, 0, sizeof m);
  m.kind = p.kind;
  m.texId = p.texId;
  m.color = f3<decltype(m.color)>(p.color);
  m.roughness = p.roughness;
  m.ior = p.ior;
  m.intensity = p.intensity;
  m.twoSided = p.twoSided;
  m.absorb = f3<decltype(m.absorb)>(p.absorb);
  m.waveAmp = p.waveAmp;
  m.waveFreq = p.waveFreq;
  return m;
}
M::LightDesc light(const PLight& p) {
  M::LightDesc l;
  std::memset(&l, 0, sizeof l);
  l.kind = p.kind;
  l.p = f3<decltype(l.p)>(p.p);
  l.u = f3<decltype(l.u)>(p.u);
  l.v = f3<decltype(l.v)>(p.v);
  l.n = f3<decltype(l.n)>(p.n);
  l.L = f3<decltype(l.L)>(p.L);
  l.radius = p.radius;
  l.area = p.area;
  l.dir = f3<decltype(l.dir)>(p.dir);
  l.twoSided = p.twoSided;
  l.texId = -1;
  l.flameId = p.flameId;
  return l;
}
template <class F> auto setSteps(F& f, int s, int) -> decltype(f.steps = s, void()) { f.steps = s; }
template <class F> void setSteps(F&, int, long) {}
M::FlameDesc flame(const PFlame& p) {
  M::FlameDesc f;
  std::memset(&f, 0, sizeof f);
  f.base = f3<decltype(f.base)>(p.base);
  f.height = p.height;
  f.radius = p.radius;
  f.intensity = p.intensity;
  f.sigma = p.sigma;
  f.noiseScale = p.noiseScale;
  f.seed = p.seed;
  setSteps(f, p.steps, 0);
  return f;
}
M::Pcg32 pcg(uint64_t state, uint64_t inc) {
  M::Pcg32 g;
  g.state = state;
  g.inc = inc;
  return g;
}

}  // namespace

// Returns 0 on success; 1 for an unknown function id. `in` for which 9
// (cdf search) carries int count + floats after the items.
extern "C" int sdo_fn(int which, const void* in, int n, void* out) {
  using namespace M;
  for (int i = 0; i < n; i++) {
    switch (which) {
      case 1: {
        const PcgIn& a = ((const PcgIn*)in)[i];
        PcgOut& o = ((PcgOut*)out)[i];
        M::Pcg32 g = M::Pcg32::init(a.seed, a.seq);
        for (int k = 0; k < 8; k++) o.next[k] = g.next();
        for (int k = 0; k < 4; k++) o.uni[k] = g.rnd();
        break;
      }
      case 2: {
        const EvalIn& a = ((const EvalIn*)in)[i];
        EvalOut& o = ((EvalOut*)out)[i];
        M::MaterialDesc m = mat(a.m);
        using F3 = decltype(m.color);
        o.f = v3(M::bsdfEval(m, f3<F3>(a.albedo), f3<F3>(a.wo), f3<F3>(a.wi), f3<F3>(a.n), a.eta));
        o.pdf = M::bsdfPdf(m, f3<F3>(a.wo), f3<F3>(a.wi), f3<F3>(a.n), a.eta);
        break;
      }
      case 3: {
        const DrawIn& a = ((const DrawIn*)in)[i];
        DrawOut& o = ((DrawOut*)out)[i];
        M::MaterialDesc m = mat(a.m);
        using F3 = decltype(m.color);
        M::Pcg32 g = pcg(a.state, a.inc);
        M::BsdfSample s = M::bsdfSample(m, f3<F3>(a.albedo), f3<F3>(a.d), f3<F3>(a.n), a.front != 0,
                                        a.etaExt, g);
        o.ok = s.valid;
        o.delta = s.isDelta;
        // Fields a failed draw leaves unset are reported as 0.
        o.wi = s.valid ? v3(s.wi) : V3{0, 0, 0};
        o.weight = s.valid ? v3(s.weight) : V3{0, 0, 0};
        o.pdf = s.valid ? s.pdf : 0.0f;
        o.pad = 0;
        o.state = g.state;
        break;
      }
      case 4: {
        const QuadIn& a = ((const QuadIn*)in)[i];
        QuadOut& o = ((QuadOut*)out)[i];
        using F3 = decltype(M::QuadricHit().n);
        M::QuadricHits h = M::intersectQuadric(a.kind, f3<F3>(a.o), f3<F3>(a.d), a.tmin, a.tmax);
        std::memset(&o, 0, sizeof o);
        o.count = h.count;
        if (h.count > 0) { o.t0 = h.hits[0].t; o.n0 = v3(h.hits[0].n); o.u0 = h.hits[0].u; o.v0 = h.hits[0].v; }
        if (h.count > 1) { o.t1 = h.hits[1].t; o.n1 = v3(h.hits[1].n); o.u1 = h.hits[1].u; o.v1 = h.hits[1].v; }
        break;
      }
      case 6: {
        const LightIn& a = ((const LightIn*)in)[i];
        LightOut& o = ((LightOut*)out)[i];
        M::LightDesc l = light(a.l);
        using F3 = decltype(l.p);
        M::Pcg32 g = pcg(a.state, a.inc);
        F3 x = f3<F3>(a.x);
        M::LightSample s = M::sampleLight(l, x, g, nullptr);
        std::memset(&o, 0, sizeof o);
        o.ok = s.valid;
        o.delta = s.isDelta;
        if (s.valid) {
          o.wi = v3(s.wi);
          o.Li = v3(s.Li);
          o.dist = s.dist;
          o.pdf = s.pdf;
          F3 hp = x + s.wi * s.dist;
          o.density = M::lightPdfSolidAngle(l, x, hp, l.n);
        }
        o.state = g.state;
        break;
      }
      case 7: {
        const FlameIn& a = ((const FlameIn*)in)[i];
        FlameOut& o = ((FlameOut*)out)[i];
        M::FlameDesc f = flame(a.f);
        using F3 = decltype(f.base);
        M::Pcg32 g1 = pcg(a.state, a.inc), g2 = pcg(a.state, a.inc);
        F3 trans = M::f3(1.0f);
        o.Lv = v3(M::marchFlames(&f, 1, f3<F3>(a.o), f3<F3>(a.d), a.tEnd, g1, trans));
        o.trans = v3(trans);
        o.tr = M::flameTransmittance(&f, 1, f3<F3>(a.o), f3<F3>(a.d), a.tEnd, g2, a.skip);
        o.pad = 0;
        o.stateMarch = g1.state;
        o.stateShadow = g2.state;
        break;
      }
      case 8: {
        const NoiseIn& a = ((const NoiseIn*)in)[i];
        NoiseOut& o = ((NoiseOut*)out)[i];
        using F3 = decltype(M::f3(0.0f));
        o.fbm = M::fbm3(f3<F3>(a.p), a.seed);
        o.vnoise = M::vnoise(f3<F3>(a.p), a.seed);
        o.wave = v3(M::waterNormal(f3<F3>(a.p), f3<F3>(a.ns), f3<F3>(a.wo), a.amp, a.freq));
        break;
      }
      case 9: {
        const float* us = (const float*)in;
        const char* tail = (const char*)in + sizeof(float) * n;
        int cnt;
        std::memcpy(&cnt, tail, sizeof cnt);
        const float* cdf = (const float*)(tail + sizeof(int));
        ((int*)out)[i] = M::findInterval(cdf, cnt, us[i]);
        break;
      }
      default:
        return 1;
    }
  }
  return 0;
}

#ifdef SDO_USE_REFERENCE
// fnvec_ref WHICH N IN OUT OUTBYTES: run sdo_fn over a packed input file.
int main(int argc, char** argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s which n in.bin out.bin out_item_bytes\n", argv[0]);
    return 2;
  }
  int which = std::atoi(argv[1]), n = std::atoi(argv[2]);
  size_t ob = (size_t)std::atol(argv[5]);
  FILE* f = std::fopen(argv[3], "rb");
  if (!f) return 3;
  std::vector<char> in;
  char buf[1 << 16];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) in.insert(in.end(), buf, buf + k);
  std::fclose(f);
  std::vector<char> out(ob * (size_t)n);
  if (sdo_fn(which, in.data(), n, out.data()) != 0) return 4;
  f = std::fopen(argv[4], "wb");
  if (!f) return 5;
  std::fwrite(out.data(), 1, out.size(), f);
  std::fclose(f);
  return 0;
}
#endif
