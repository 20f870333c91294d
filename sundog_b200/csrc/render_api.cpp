// sundog_render / sundog_render_ex: one resident session, one render, film
// download, image + stats output. Progress and notices go to stderr as in
// src/capi_render.cpp:224-245 (stdout belongs to the calling program).
//
// Output: the reference encodes a 12-bit PQ BT.2020 AVIF through libavif
// (src/film.cpp:96-115), which this build does not link. The same 12-bit PQ
// codes are encoded on the device (film_out.cu) and written losslessly as a
// 16-bit PNG with a BT.2020 / PQ cICP chunk: for a ".png" out_path there, for
// an ".avif" out_path beside it (".png" replacing the extension) with a
// notice. A ".pfm" or ".hdr" out_path is written as linear float (exposure
// applied); any other extension gets a ".pfm" file beside it and a notice.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sundog_api.h"
#include "abi_util.h"
#include "denoise.h"
#include "film_out.h"
#include "guide.h"
#include "render_session.h"
#include "wavefront.h"

using namespace sdb;

namespace {

bool endsWith(const std::string& s, const char* suf) {
  size_t n = std::strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

void writePfm(const std::string& path, const float* rgba, int w, int h, float scale) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("failed to write " + path);
  std::fprintf(f, "PF\n%d %d\n-1.0\n", w, h);
  std::vector<float> row((size_t)w * 3);
  for (int y = h - 1; y >= 0; y--) {  // PFM rows run bottom to top
    for (int x = 0; x < w; x++)
      for (int c = 0; c < 3; c++) row[(size_t)x * 3 + c] = rgba[((size_t)y * w + x) * 4 + c] * scale;
    std::fwrite(row.data(), sizeof(float), row.size(), f);
  }
  if (std::fclose(f) != 0) throw std::runtime_error("failed to write " + path);
}

void writeRgbe(const std::string& path, const float* rgba, int w, int h, float scale) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("failed to write " + path);
  std::fprintf(f, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n", h, w);
  std::vector<unsigned char> px((size_t)w * 4);
  for (int y = 0; y < h; y++) {
    for (int x = 0; x < w; x++) {
      const float* p = rgba + ((size_t)y * w + x) * 4;
      float r = p[0] * scale, g = p[1] * scale, b = p[2] * scale;
      float m = std::fmax(r, std::fmax(g, b));
      unsigned char* o = &px[(size_t)x * 4];
      if (m < 1e-32f) {
        o[0] = o[1] = o[2] = o[3] = 0;
      } else {
        int e;
        float fr = std::frexp(m, &e) * 256.0f / m;
        o[0] = (unsigned char)(r * fr);
        o[1] = (unsigned char)(g * fr);
        o[2] = (unsigned char)(b * fr);
        o[3] = (unsigned char)(e + 128);
      }
    }
    std::fwrite(px.data(), 1, px.size(), f);
  }
  if (std::fclose(f) != 0) throw std::runtime_error("failed to write " + path);
}

std::string writeImage(const std::string& path, const float* rgba, int w, int h, float scale) {
  if (endsWith(path, ".hdr")) {
    writeRgbe(path, rgba, w, h, scale);
    return path;
  }
  if (endsWith(path, ".pfm")) {
    writePfm(path, rgba, w, h, scale);
    return path;
  }
  std::string p = path + ".pfm";
  writePfm(p, rgba, w, h, scale);
  return p;
}

std::string jesc(const std::string& s) {
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

// Same keys as the reference's stats sidecar (src/stats.cpp:26-61), plus
// samples_per_sec, the device-timed kernel milliseconds and BVH figures.
void writeStats(const std::string& path, const char* sceneName, const RenderSession& s,
                const sundog_render_result& r, double totalMs, double denoiseMs, size_t peakMB) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw std::runtime_error("cannot write " + path);
  cudaDeviceProp p;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaGetDeviceProperties(&p, dev);
  int dv = 0, rv = 0;
  cudaDriverGetVersion(&dv);
  cudaRuntimeGetVersion(&rv);
  const RenderCfg& rs = s.scene.render;
  std::fprintf(f, "{\n  \"scene\": %s,\n", jesc(sceneName).c_str());
  std::fprintf(f, "  \"width\": %d,\n  \"height\": %d,\n  \"spp\": %d,\n", rs.width, rs.height, rs.spp);
  std::fprintf(f, "  \"max_depth\": %d,\n  \"seed\": %u,\n  \"denoised\": %s,\n", rs.maxDepth,
               rs.seed, rs.denoise ? "true" : "false");
  std::fprintf(f,
               "  \"timings_ms\": {\n    \"scene_load\": %.17g,\n    \"physics\": 0,\n"
               "    \"gas_build\": %.17g,\n    \"render\": %.17g,\n    \"denoise\": %.17g,\n"
               "    \"total\": %.17g\n  },\n",
               s.loadMs, s.buildMs, r.render_ms, denoiseMs, totalMs);
  std::fprintf(f, "  \"rays_traced\": %llu,\n  \"mrays_per_sec\": %.17g,\n",
               (unsigned long long)r.rays_traced, r.mrays_per_sec);
  std::fprintf(f, "  \"samples_per_sec\": %.17g,\n  \"kernel_ms\": %.17g,\n", r.samples_per_sec,
               r.kernel_ms);
  std::fprintf(f, "  \"peak_vram_mb\": %zu,\n", peakMB);
  std::fprintf(f,
               "  \"scene_stats\": {\n    \"objects\": %zu,\n    \"lights\": %zu,\n"
               "    \"meshes\": %zu,\n    \"mesh_triangles\": %zu\n  },\n",
               s.scene.objects.size(), s.scene.lights.size(), s.scene.meshes.size(),
               s.meshTriangles);
  std::fprintf(f, "  \"bvh\": {\"nodes\": %zu, \"triangles\": %zu, \"tlas_depth\": %d, \"blas_depth\": %d},\n",
               s.numNodes, s.numTris, s.tlasDepth, s.blasDepth);
  std::fprintf(f,
               "  \"device\": {\n    \"name\": %s,\n    \"compute\": \"sm_%d%d\",\n"
               "    \"vram_mb\": %zu,\n    \"cuda_driver\": %d,\n    \"cuda_runtime\": %d,\n"
               "    \"optix_header\": 0\n  }\n}\n",
               jesc(p.name).c_str(), p.major, p.minor, (size_t)(p.totalGlobalMem >> 20), dv, rv);
  std::fclose(f);
}

int renderImpl(sundog_scene* h, const sundog_render_options* opt, const sundog_render_ext* ext,
               sundog_render_result* res, bool requireOut) {
  if (!opt) throw std::runtime_error("render: options are required");
  if (requireOut && (!opt->out_path || !*opt->out_path))
    throw std::runtime_error("render: out_path is required");
  if (!h) throw std::runtime_error("render: null scene");
  if (sundog_scene_validate(h) != SUNDOG_OK) throw std::runtime_error(sundog_last_error());
  const char* sceneName = opt->scene_name ? opt->scene_name : "(scene)";
  auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<RenderSession> s(new RenderSession());
  s->build(h, opt, ext);
  const RenderCfg& rs = s->scene.render;
  bool quiet = s->quiet;
  if (!quiet) {
    cudaDeviceProp p;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaGetDeviceProperties(&p, dev);
    std::fprintf(stderr, "sundog: %s %dx%d, %d spp, depth %d on %s\n", sceneName, rs.width,
                 rs.height, rs.spp, rs.maxDepth, p.name);

  }
  sundog_render_result r{};
  int reps = ext && ext->repeat > 1 ? ext->repeat : 1;
  double best = 1e300;
  sundog_render_result bestR{};
  for (int i = 0; i < reps; i++) {
    s->render(nullptr, true, &r);
    if (r.render_ms < best) {
      best = r.render_ms;
      bestR = r;
    }
  }
  r = bestR;
  size_t npix = (size_t)rs.width * rs.height;
  // Optional post-process (src/capi_render.cpp:247-256): the denoised film
  // replaces the raw one as the call's output.
  double denoiseMs = 0.0;
  DevBuf denoised;
  if (rs.denoise) {
    auto tDen = std::chrono::steady_clock::now();
    denoised.alloc(npix * sizeof(float4));
    denoiseFilm((const float4*)s->accum.ptr, (const float4*)s->aovAlb.ptr,
                (const float4*)s->aovNrm.ptr, rs.width, rs.height, denoiseDefaults(),
                (float4*)denoised.ptr, s->stream);
    denoiseMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tDen).count();
  }
  // The film goes straight into the caller's buffer when there is one.
  std::vector<float> own;
  float* film = ext && ext->film_rgba ? ext->film_rgba : nullptr;
  if (!film) {
    own.resize(npix * 4);
    film = own.data();
  }
  if (rs.denoise) {
    cudaCheck(cudaMemcpy(film, denoised.ptr, npix * sizeof(float4), cudaMemcpyDeviceToHost),
              "denoised film download");
    countDownload(npix * sizeof(float4));
  } else {
    s->read(film, nullptr, nullptr);
  }
  std::vector<float> alb, nrm;
  if (s->aov) {
    alb.resize(npix * 4);
    nrm.resize(npix * 4);
    s->read(nullptr, alb.data(), nrm.data());
    if (ext && ext->aov_albedo) std::memcpy(ext->aov_albedo, alb.data(), alb.size() * sizeof(float));
    if (ext && ext->aov_normal) std::memcpy(ext->aov_normal, nrm.data(), nrm.size() * sizeof(float));
  }
  float scale = exp2f(rs.exposure);
  if (opt->out_path && *opt->out_path) {
    std::string out = opt->out_path, wrote;
    const bool avif = endsWith(out, ".avif");
    if (avif || endsWith(out, ".png")) {
      if (avif) out = out.substr(0, out.size() - 5) + ".png";
      std::vector<unsigned short> codes(npix * 3);
      encodePq12((const float4*)(rs.denoise ? denoised.ptr : s->accum.ptr), rs.width, rs.height,
                 rs.exposure, codes.data(), s->stream);
      writePq16Png(out, codes.data(), rs.width, rs.height);
      wrote = out;
    } else {
      wrote = writeImage(opt->out_path, film, rs.width, rs.height, scale);
    }
    if (opt->aov_albedo_path) writeImage(opt->aov_albedo_path, alb.data(), rs.width, rs.height, 1.0f);
    if (opt->aov_normal_path) writeImage(opt->aov_normal_path, nrm.data(), rs.width, rs.height, 1.0f);
    if (!quiet) {
      std::fprintf(stderr, "Rendering elapsed time: %f seconds (%.0f Mrays/s)\nwrote %s\n",
                   r.render_ms / 1000.0, r.mrays_per_sec, wrote.c_str());
      if (wrote != opt->out_path)
        std::fprintf(stderr, "sundog: no AVIF encoder in this build; wrote %s instead\n",
                     wrote.c_str());
    }
  }
  size_t freeAfter = 0, tot = 0;
  cudaMemGetInfo(&freeAfter, &tot);
  double totalMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  r.total_ms = totalMs;
  if (opt->stats_path) {
    size_t peak = s->freeBefore > freeAfter ? (s->freeBefore - freeAfter) >> 20 : 0;
    writeStats(opt->stats_path, sceneName, *s, r, totalMs, denoiseMs, peak);
  }
  if (res) *res = r;
  return SUNDOG_OK;
}

}  // namespace

extern "C" int sundog_session_denoise(sundog_session* sh, float* out) {
  SDB_TRY
  if (!sh || !out) throw std::runtime_error("denoise: null argument");
  RenderSession& s = *reinterpret_cast<RenderSession*>(sh);
  if (!s.aov) throw std::runtime_error("denoise: the session renders no AOVs (create it with AOVs)");
  size_t npix = (size_t)s.lp.width * s.lp.height;
  DevBuf d;
  d.alloc(npix * sizeof(float4));
  denoiseFilm((const float4*)s.accum.ptr, (const float4*)s.aovAlb.ptr, (const float4*)s.aovNrm.ptr,
              s.lp.width, s.lp.height, denoiseDefaults(), (float4*)d.ptr, s.stream);
  cudaCheck(cudaMemcpy(out, d.ptr, npix * sizeof(float4), cudaMemcpyDeviceToHost), "denoise read");
  countDownload(npix * sizeof(float4));
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_session_read_pq12(sundog_session* sh, double exposure, uint16_t* out) {
  SDB_TRY
  if (!sh || !out) throw std::runtime_error("read pq12: null argument");
  RenderSession& s = *reinterpret_cast<RenderSession*>(sh);
  float ev = std::isnan(exposure) ? s.scene.render.exposure : (float)exposure;
  encodePq12((const float4*)s.accum.ptr, s.lp.width, s.lp.height, ev, out, s.stream);
  countDownload((size_t)s.lp.width * s.lp.height * 3 * sizeof(uint16_t));
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

// src/capi_render.cpp:280-307
extern "C" int sundog_render(sundog_scene* h, const sundog_render_options* opt) {
  SDB_TRY
  return renderImpl(h, opt, nullptr, nullptr, true);
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_render_ex(sundog_scene* h, const sundog_render_options* opt,
                                const sundog_render_ext* ext, sundog_render_result* res) {
  SDB_TRY
  return renderImpl(h, opt, ext, res, false);
  SDB_CATCH(SUNDOG_ERROR)
}
