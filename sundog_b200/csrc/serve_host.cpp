// Render server: admission by free device memory, resident shared scenes,
// continuous batching of tile-passes across jobs (serve.cu).
//
// The server thread loops: admit queued jobs (arrival order; a job that does
// not fit lets later ones that do pass), build one batch of tile-passes from
// the active jobs, run it (one persistent launch + one fold), retire the
// jobs whose tiles have all their samples (film to the host, memory back).
//
// Batch policy: every active job gets at least one tile-pass per iteration
// (no starvation); the remaining path budget goes to jobs in order of least
// remaining work (short jobs finish early, which keeps median latency low).
// Within a job, tiles take turns; a tile appears at most once per batch, so
// its samples fold in order.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sundog_api.h"
#include "abi_util.h"
#include "kernels.h"
#include "render_session.h"
#include "scene_model.h"
#include "serve.h"
#include "wavefront.h"

namespace sdb {

using Clock = std::chrono::steady_clock;

static double msBetween(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Key of a scene's device data: its description without render settings and
// camera (those are per film), plus the directory assets resolve against.
static std::string sceneKey(const sundog_scene* h) {
  size_t need = 0;
  if (sundog_scene_debug_json(const_cast<sundog_scene*>(h), nullptr, 0, &need) != SUNDOG_OK)
    throw std::runtime_error(sundog_last_error());
  std::string js(need, '\0');
  if (sundog_scene_debug_json(const_cast<sundog_scene*>(h), &js[0], need, &need) != SUNDOG_OK)
    throw std::runtime_error(sundog_last_error());
  size_t c = js.find("\"camera\":{");
  if (c != std::string::npos) {
    int depth = 0;
    size_t i = js.find('{', c);
    for (; i < js.size(); i++) {
      if (js[i] == '{') depth++;
      if (js[i] == '}' && --depth == 0) break;
    }
    js = js.substr(i + 1);
  }
  return h->scene.baseDir + "\n" + js;
}

struct ServeJob {
  int64_t id = 0;
  SceneDesc desc;
  std::string key;
  float* hostFilm = nullptr;
  int width = 0, height = 0, spp = 0;
  int state = SUNDOG_JOB_QUEUED;
  bool cancel = false;
  bool admitted = false;
  std::string error;
  Clock::time_point tSubmit, tAdmit, tEnd;
  // device side (server thread only)
  std::shared_ptr<const DeviceScene> dev;
  DevBuf film;  // the device film (a pooled buffer may be larger than filmBytes)
  uint64_t filmBytes = 0;
  SdLaunch lp{};
  int slot = -1;
  int tilesX = 0, tilesY = 0;
  std::vector<int> tileNext;  // next sample of each tile
  int cursor = 0;
  uint64_t pathsTotal = 0, pathsDone = 0;
};

struct CachedScene {
  std::shared_ptr<DeviceScene> dev;
  int users = 0;
  uint64_t lastUse = 0;
};

class Server {
 public:
  explicit Server(const sundog_server_config& c) : cfg(c) {
    t0 = Clock::now();
    cudaCheck(cudaFree(nullptr), "CUDA context");
    cudaCheck(cudaGetDevice(&device), "cudaGetDevice");
    cudaCheck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    cudaCheck(cudaEventCreate(&ev0), "event");
    cudaCheck(cudaEventCreate(&ev1), "event");
    int t = cfg.tile;
    maxItemPaths = (uint64_t)((t + 7) / 8) * ((t + 7) / 8) * 64 * cfg.pass_spp;
    // The budget, plus the one tile-pass every job gets even past it.
    scratch.alloc((cfg.iteration_paths + (uint64_t)kMaxServeJobs * maxItemPaths) * sizeof(float4));
    maxItems = (int)std::min<uint64_t>(1u << 20, cfg.iteration_paths / 64 + 2 * kMaxServeJobs);
    dItems.alloc((size_t)maxItems * sizeof(ServeItem));
    cudaCheck(cudaMallocHost((void**)&hItems, (size_t)maxItems * sizeof(ServeItem)), "pinned items");
    counters.alloc(2 * sizeof(unsigned long long));
    grid = serveGridSize();
    if (cfg.engine != 1) {  // the wavefront engine's slot pool, sized for a batch
      wf = wfAcquire();
      uint64_t batchPaths = cfg.iteration_paths + (uint64_t)kMaxServeJobs * maxItemPaths;
      wf->ensure((int)std::min<uint64_t>(batchPaths, 1ull << 26));
    }
    slots.assign(kMaxServeJobs, nullptr);
    thread = std::thread([this] { loop(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> g(mu);
      stopping = true;
      for (auto& kv : jobs)
        if (kv.second->state == SUNDOG_JOB_QUEUED || kv.second->state == SUNDOG_JOB_RUNNING)
          kv.second->cancel = true;
    }
    cv.notify_all();
    if (thread.joinable()) thread.join();
    wfRelease(std::move(wf));
    for (auto& j : slots)
      if (j) j->film.release();
    dropFilmPool();
    sceneCache.clear();
    if (hItems) cudaFreeHost(hItems);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (st) cudaStreamDestroy(st);
  }

  int64_t submit(const sundog_scene* h, const sundog_render_options* opt, float* film) {
    std::shared_ptr<ServeJob> j(new ServeJob());
    j->desc = h->scene;
    applyRenderOverrides(j->desc, opt);
    j->key = sceneKey(h);
    j->width = j->desc.render.width;
    j->height = j->desc.render.height;
    j->spp = j->desc.render.spp;
    j->hostFilm = film;
    j->tSubmit = Clock::now();
    {
      std::lock_guard<std::mutex> g(mu);
      if (stopping) throw std::runtime_error("server: shutting down");
      j->id = nextId++;
      jobs[j->id] = j;
      queue.push_back(j);
      submitted++;
    }
    cv.notify_all();
    return j->id;
  }

  void status(int64_t id, sundog_job_status* out) {
    std::lock_guard<std::mutex> g(mu);
    fillStatus(find(id), out);
  }

  bool wait(int64_t id, double timeoutMs, sundog_job_status* out) {
    std::unique_lock<std::mutex> g(mu);
    std::shared_ptr<ServeJob> j = find(id);
    auto done = [&] { return j->state >= SUNDOG_JOB_DONE; };
    bool ok = true;
    if (timeoutMs < 0) cvDone.wait(g, done);
    else ok = cvDone.wait_for(g, std::chrono::duration<double, std::milli>(timeoutMs), done);
    if (out) fillStatus(j, out);
    return ok;
  }

  bool cancel(int64_t id) {
    std::lock_guard<std::mutex> g(mu);
    std::shared_ptr<ServeJob> j = find(id);
    if (j->state >= SUNDOG_JOB_DONE) return false;
    j->cancel = true;
    cv.notify_all();
    return true;
  }

  void stats(sundog_server_statistics* s) {
    std::lock_guard<std::mutex> g(mu);
    std::memset(s, 0, sizeof *s);
    s->jobs_submitted = submitted;
    s->jobs_done = nDone;
    s->jobs_failed = nFailed;
    s->jobs_cancelled = nCancelled;
    s->iterations = iterations;
    s->rays = rays;
    s->paths = paths;
    s->busy_ms = busyMs;
    s->wall_ms = msBetween(t0, Clock::now());
    s->active_jobs = activeCount;
    s->queued_jobs = (int32_t)queue.size();
    s->scenes_resident = residentScenes;
    s->scene_bytes = residentBytes;
  }

 private:
  sundog_server_config cfg;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf scratch, dItems, counters;
  std::unique_ptr<WfBuffers> wf;  // engine 0: the wavefront engine's slot pool
  ServeItem* hItems = nullptr;
  int maxItems = 0;
  uint64_t maxItemPaths = 0;
  int grid = 0;
  std::thread thread;
  std::mutex mu;
  std::condition_variable cv, cvDone;
  bool stopping = false;
  int64_t nextId = 0;
  std::map<int64_t, std::shared_ptr<ServeJob>> jobs;
  std::deque<std::shared_ptr<ServeJob>> queue;
  // server-thread state
  std::vector<std::shared_ptr<ServeJob>> slots;
  std::map<std::string, CachedScene> sceneCache;
  uint64_t useClock = 0;
  // statistics (under mu)
  Clock::time_point t0;
  uint64_t submitted = 0, nDone = 0, nFailed = 0, nCancelled = 0, iterations = 0, rays = 0,
           paths = 0, residentScenes = 0, residentBytes = 0;
  double busyMs = 0.0;
  int activeCount = 0;

  std::shared_ptr<ServeJob> find(int64_t id) {
    auto it = jobs.find(id);
    if (it == jobs.end()) throw std::runtime_error("server: unknown job id");
    return it->second;
  }

  void fillStatus(const std::shared_ptr<ServeJob>& j, sundog_job_status* out) {
    std::memset(out, 0, sizeof *out);
    out->state = j->state;
    out->width = j->width;
    out->height = j->height;
    out->spp = j->spp;
    out->paths_done = j->pathsDone;
    out->paths_total = j->pathsTotal;
    Clock::time_point now = Clock::now();
    if (j->admitted) out->queued_ms = msBetween(j->tSubmit, j->tAdmit);
    else out->queued_ms = msBetween(j->tSubmit, j->state >= SUNDOG_JOB_DONE ? j->tEnd : now);
    out->latency_ms = j->state >= SUNDOG_JOB_DONE ? msBetween(j->tSubmit, j->tEnd)
                                                  : msBetween(j->tSubmit, now);
    std::snprintf(out->error, sizeof out->error, "%s", j->error.c_str());
  }

  // Final state of a job (server thread; takes the lock).
  void finish(const std::shared_ptr<ServeJob>& j, int state, const std::string& err) {
    {
      std::lock_guard<std::mutex> g(mu);
      j->state = state;
      j->error = err;
      j->tEnd = Clock::now();
      if (state == SUNDOG_JOB_DONE) nDone++;
      if (state == SUNDOG_JOB_FAILED) nFailed++;
      if (state == SUNDOG_JOB_CANCELLED) nCancelled++;
    }
    cvDone.notify_all();
  }

  // Films of finished jobs are kept for later jobs (up to kFilmPoolBytes):
  // a job's admission then allocates no device memory, and a finished job
  // frees none, so neither waits on the driver's allocator.
  static constexpr uint64_t kFilmPoolBytes = 1ull << 30;
  std::vector<DevBuf> filmPool;
  uint64_t filmPoolBytes = 0;

  void takeFilm(DevBuf& film, uint64_t bytes) {
    int best = -1;
    for (int k = 0; k < (int)filmPool.size(); k++)
      if (filmPool[k].bytes >= bytes && (best < 0 || filmPool[k].bytes < filmPool[best].bytes))
        best = k;
    if (best < 0) {
      film.alloc(bytes);
      return;
    }
    filmPoolBytes -= filmPool[best].bytes;
    film = std::move(filmPool[best]);
    filmPool.erase(filmPool.begin() + best);
  }

  void returnFilm(DevBuf& film) {
    if (!film.ptr) return;
    if (filmPoolBytes + film.bytes > kFilmPoolBytes) {
      film.release();
      return;
    }
    filmPoolBytes += film.bytes;
    filmPool.push_back(std::move(film));
  }

  void dropFilmPool() {
    filmPool.clear();
    filmPoolBytes = 0;
  }

  void releaseJob(const std::shared_ptr<ServeJob>& j) {
    returnFilm(j->film);
    if (j->slot >= 0) slots[j->slot] = nullptr;
    j->slot = -1;
    if (j->dev) {
      auto it = sceneCache.find(j->key);
      if (it != sceneCache.end()) it->second.users--;
      j->dev.reset();
    }
  }

  // Drops unused scenes, least recently used first, until `need` more bytes
  // fit or nothing is left to drop; also trims to the cache budget.
  void evictScenes(uint64_t need, uint64_t freeBytes) {
    for (;;) {
      uint64_t held = 0;
      for (auto& kv : sceneCache) held += kv.second.dev->deviceBytes;
      bool overBudget = held > cfg.scene_cache_bytes;
      bool short_ = need > 0 && freeBytes < need + cfg.reserve_bytes;
      if (!overBudget && !short_) return;
      auto victim = sceneCache.end();
      for (auto it = sceneCache.begin(); it != sceneCache.end(); ++it)
        if (it->second.users == 0 && (victim == sceneCache.end() ||
                                      it->second.lastUse < victim->second.lastUse))
          victim = it;
      if (victim == sceneCache.end()) return;
      freeBytes += victim->second.dev->deviceBytes;
      sceneCache.erase(victim);
    }
  }

  void updateSceneStats() {
    uint64_t n = sceneCache.size(), b = 0;
    for (auto& kv : sceneCache) b += kv.second.dev->deviceBytes;
    std::lock_guard<std::mutex> g(mu);
    residentScenes = n;
    residentBytes = b;
  }

  // Tries to place job j on the device. Returns false to leave it queued.
  bool admit(const std::shared_ptr<ServeJob>& j) {
    int slot = -1;
    for (int s = 0; s < std::min(cfg.max_jobs, kMaxServeJobs); s++)
      if (!slots[s]) {
        slot = s;
        break;
      }
    if (slot < 0) return false;
    size_t freeB = 0, totB = 0;
    cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
    uint64_t filmBytes = (uint64_t)j->width * j->height * sizeof(float4);
    if (filmBytes + cfg.reserve_bytes > totB)
      throw std::runtime_error("job needs more device memory than the device has");
    auto it = sceneCache.find(j->key);
    if (it == sceneCache.end()) {
      dropFilmPool();
      evictScenes(filmBytes, freeB);
      cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
      if (freeB < filmBytes + cfg.reserve_bytes) return false;
      std::shared_ptr<DeviceScene> ds(new DeviceScene());
      ds->build(j->desc);
      it = sceneCache.emplace(j->key, CachedScene{ds, 0, 0}).first;
      cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
    }
    if (freeB < filmBytes + cfg.reserve_bytes) {
      dropFilmPool();
      evictScenes(filmBytes, freeB);
      cudaCheck(cudaMemGetInfo(&freeB, &totB), "cudaMemGetInfo");
      if (freeB < filmBytes + cfg.reserve_bytes) {
        bool othersRunning = false;
        for (auto& s : slots) othersRunning |= (s != nullptr);
        if (!othersRunning && it->second.users == 0)
          throw std::runtime_error("job does not fit in free device memory");
        return false;  // wait for running jobs to free memory
      }
    }
    it->second.users++;
    it->second.lastUse = ++useClock;
    j->dev = it->second.dev;
    takeFilm(j->film, filmBytes);
    j->filmBytes = filmBytes;
    cudaCheck(cudaMemsetAsync(j->film.ptr, 0, filmBytes, st), "film reset");
    std::memset(&j->lp, 0, sizeof j->lp);
    fillRenderLaunch(j->lp, j->desc, j->desc.render);
    j->dev->fillLaunch(j->lp);
    j->lp.accum = (float4*)j->film.ptr;
    j->lp.sampleOffset = 0;
    j->lp.sppThisLaunch = j->spp;
    j->slot = slot;  // its launch block is uploaded with every batch
    slots[slot] = j;
    j->tilesX = (j->width + cfg.tile - 1) / cfg.tile;
    j->tilesY = (j->height + cfg.tile - 1) / cfg.tile;
    j->tileNext.assign((size_t)j->tilesX * j->tilesY, 0);
    j->pathsTotal = (uint64_t)j->width * j->height * j->spp;
    {
      std::lock_guard<std::mutex> g(mu);
      j->state = SUNDOG_JOB_RUNNING;
      j->tAdmit = Clock::now();
      j->admitted = true;
    }
    return true;
  }

  void admitQueued() {
    std::vector<std::shared_ptr<ServeJob>> pending;
    {
      std::lock_guard<std::mutex> g(mu);
      pending.assign(queue.begin(), queue.end());
    }
    for (auto& j : pending) {
      bool cancelled;
      {
        std::lock_guard<std::mutex> g(mu);
        cancelled = j->cancel;
      }
      bool leaveQueue = false;
      if (cancelled) {
        finish(j, SUNDOG_JOB_CANCELLED, "");
        leaveQueue = true;
      } else {
        try {
          leaveQueue = admit(j);
        } catch (const std::exception& e) {
          releaseJob(j);
          finish(j, SUNDOG_JOB_FAILED, e.what());
          leaveQueue = true;
        }
      }
      if (leaveQueue) {
        std::lock_guard<std::mutex> g(mu);
        queue.erase(std::find(queue.begin(), queue.end(), j));
      }
    }
    updateSceneStats();
  }

  // Next tile-pass of job j not yet in this batch; false when none is left.
  int tileNpad(const ServeJob& j, int t) const {
    int x0 = (t % j.tilesX) * cfg.tile, y0 = (t / j.tilesX) * cfg.tile;
    int w = std::min(cfg.tile, j.width - x0), h = std::min(cfg.tile, j.height - y0);
    return ((w + 7) / 8) * ((h + 7) / 8) * 64;
  }

  bool nextTilePass(ServeJob& j, std::vector<char>& used, int chunk, ServeItem& it) {
    int nt = (int)j.tileNext.size();
    for (int k = 0; k < nt; k++) {
      int t = (j.cursor + k) % nt;
      if (used[t] || j.tileNext[t] >= j.spp) continue;
      j.cursor = (t + 1) % nt;
      used[t] = 1;
      int tx = t % j.tilesX, ty = t / j.tilesX;
      it.job = j.slot;
      it.x0 = tx * cfg.tile;
      it.y0 = ty * cfg.tile;
      it.w = std::min(cfg.tile, j.width - it.x0);
      it.h = std::min(cfg.tile, j.height - it.y0);
      it.bw = (it.w + 7) / 8;
      it.npad = it.bw * ((it.h + 7) / 8) * 64;
      it.sampleBegin = j.tileNext[t];
      it.sampleCount = std::min(chunk, j.spp - j.tileNext[t]);
      it.pad0 = t;  // tile index, for the host's bookkeeping
      return true;
    }
    return false;
  }

  void runIteration() {
    std::vector<std::shared_ptr<ServeJob>> act;
    for (auto& s : slots)
      if (s) act.push_back(s);
    std::sort(act.begin(), act.end(), [](const std::shared_ptr<ServeJob>& a,
                                         const std::shared_ptr<ServeJob>& b) {
      uint64_t ra = a->pathsTotal - a->pathsDone, rb = b->pathsTotal - b->pathsDone;
      return ra != rb ? ra < rb : a->id < b->id;
    });
    std::vector<std::vector<char>> used(act.size());
    for (size_t i = 0; i < act.size(); i++) used[i].assign(act[i]->tileNext.size(), 0);
    // Samples per tile-pass: pass_spp, or more when every remaining tile at
    // pass_spp would not fill the path budget (few or small jobs left), so
    // the launch stays full. The batch stays within the budget: each item is
    // at most `factor` times its tile's share of `demand`.
    uint64_t demand = 0;
    for (auto& j : act)
      for (int t = 0; t < (int)j->tileNext.size(); t++)
        if (j->tileNext[t] < j->spp)
          demand += (uint64_t)tileNpad(*j, t) * std::min(cfg.pass_spp, j->spp - j->tileNext[t]);
    int chunk = cfg.pass_spp;
    if (demand > 0 && demand < cfg.iteration_paths)
      chunk = (int)std::min<uint64_t>((uint64_t)cfg.pass_spp * (cfg.iteration_paths / demand), 4096);
    const uint64_t itemMax = (uint64_t)((cfg.tile + 7) / 8) * ((cfg.tile + 7) / 8) * 64 * chunk;
    int n = 0;
    uint64_t total = 0;
    auto add = [&](size_t i) {
      ServeItem it;
      if (n >= maxItems || !nextTilePass(*act[i], used[i], chunk, it)) return false;
      it.pathBegin = total;
      total += (uint64_t)it.npad * it.sampleCount;
      hItems[n++] = it;
      return true;
    };
    // Shortest remaining work first: a job whose whole remaining work fits
    // the budget, with room kept for one tile-pass of every job, goes in
    // whole (every open tile with all its remaining samples as one item), so
    // a small job finishes in this batch instead of taking one pass_spp pass
    // of each tile per batch. The batch stays within iteration_paths.
    std::vector<char> whole(act.size(), 0);
    const uint64_t reserve = (uint64_t)act.size() * itemMax;
    for (size_t i = 0; reserve < cfg.iteration_paths && i < act.size(); i++) {
      ServeJob& j = *act[i];
      uint64_t rem = 0;
      int open = 0;
      for (int t = 0; t < (int)j.tileNext.size(); t++)
        if (j.tileNext[t] < j.spp) {
          rem += (uint64_t)tileNpad(j, t) * (uint64_t)(j.spp - j.tileNext[t]);
          open++;
        }
      if (rem == 0 || total + rem > cfg.iteration_paths - reserve || n + open > maxItems) continue;
      ServeItem it;
      while (nextTilePass(j, used[i], j.spp, it)) {
        it.pathBegin = total;
        total += (uint64_t)it.npad * it.sampleCount;
        hItems[n++] = it;
      }
      whole[i] = 1;
    }
    for (size_t i = 0; i < act.size(); i++)  // one tile-pass each
      if (!whole[i]) add(i);
    for (size_t i = 0; i < act.size(); i++)
      while (!whole[i] && total + itemMax <= cfg.iteration_paths && add(i)) {
      }
    if (n == 0) return;
    // The job table and batch block live in per-device constant memory,
    // shared with sessions and other servers on the device: upload them and
    // run the batch to completion under the device's launch lock.
    std::lock_guard<std::mutex> launchLock(deviceLaunchLock());
    std::vector<SdLaunch> table(kMaxServeJobs);
    std::memset(table.data(), 0, table.size() * sizeof(SdLaunch));
    int maxInstances = 0;
    for (size_t k = 0; k < slots.size(); k++)
      if (slots[k]) {
        table[k] = slots[k]->lp;
        maxInstances = std::max(maxInstances, slots[k]->lp.numInstances);
      }
    // Both engines fold through ptServeFold, which reads the megakernel's
    // table; the wavefront stages read their own.
    cudaCheck(serveSetJobs(table.data(), st), "job table");
    if (wf) cudaCheck(wfSetJobs(table.data(), st), "job table");
    cudaCheck(cudaMemcpyAsync(dItems.ptr, hItems, (size_t)n * sizeof(ServeItem),
                              cudaMemcpyHostToDevice, st),
              "batch items");
    cudaCheck(cudaMemsetAsync(counters.ptr, 0, counters.bytes, st), "batch counters");
    ServeBatch b;
    b.items = (const ServeItem*)dItems.ptr;
    b.numItems = n;
    b.numPaths = total;
    b.pathCounter = (unsigned long long*)counters.ptr;
    b.rayCounter = (unsigned long long*)counters.ptr + 1;
    b.sampleL = (float4*)scratch.ptr;
    cudaCheck(cudaEventRecord(ev0, st), "event");
    if (wf) {
      wfRenderBatch(b, *wf, st, maxInstances);
      cudaCheck(serveFold(b, st), "serve fold");
    } else {
      cudaCheck(serveLaunch(b, grid, st), "serve launch");
    }
    cudaCheck(cudaEventRecord(ev1, st), "event");
    unsigned long long r = 0;
    cudaCheck(cudaMemcpyAsync(&r, b.rayCounter, sizeof r, cudaMemcpyDeviceToHost, st), "rays");
    cudaCheck(cudaStreamSynchronize(st), "serve iteration");
    float ms = 0.0f;
    cudaCheck(cudaEventElapsedTime(&ms, ev0, ev1), "event time");
    uint64_t camPaths = 0;
    for (int k = 0; k < n; k++) {
      const ServeItem& it = hItems[k];
      std::shared_ptr<ServeJob>& j = slots[it.job];
      j->tileNext[it.pad0] += it.sampleCount;
      uint64_t p = (uint64_t)it.w * it.h * it.sampleCount;
      j->pathsDone += p;
      camPaths += p;
    }
    {
      std::lock_guard<std::mutex> g(mu);
      iterations++;
      rays += r;
      paths += camPaths;
      busyMs += ms;
    }
    for (auto& j : act) {
      if (j->pathsDone < j->pathsTotal) continue;
      if (j->hostFilm)
        cudaCheck(cudaMemcpy(j->hostFilm, j->film.ptr, j->filmBytes, cudaMemcpyDeviceToHost),
                  "film download");
      releaseJob(j);
      finish(j, SUNDOG_JOB_DONE, "");
    }
  }

  void dropCancelledActive() {
    for (auto& s : slots) {
      if (!s) continue;
      bool c;
      {
        std::lock_guard<std::mutex> g(mu);
        c = s->cancel;
      }
      if (c) {
        std::shared_ptr<ServeJob> j = s;
        releaseJob(j);
        finish(j, SUNDOG_JOB_CANCELLED, "");
      }
    }
  }

  void loop() {
    cudaSetDevice(device);
    for (;;) {
      try {
        dropCancelledActive();
        admitQueued();
        int nact = 0;
        for (auto& s : slots) nact += s ? 1 : 0;
        {
          std::lock_guard<std::mutex> g(mu);
          activeCount = nact;
        }
        if (nact == 0) {
          std::unique_lock<std::mutex> g(mu);
          if (stopping && queue.empty()) break;
          cv.wait_for(g, std::chrono::milliseconds(20));
          continue;
        }
        runIteration();
        evictScenes(0, 0);
        updateSceneStats();
      } catch (const std::exception& e) {
        // A device error ends every job on the device; queued jobs stay.
        for (auto& s : slots) {
          if (!s) continue;
          std::shared_ptr<ServeJob> j = s;
          releaseJob(j);
          finish(j, SUNDOG_JOB_FAILED, std::string("device error: ") + e.what());
        }
        std::unique_lock<std::mutex> g(mu);
        if (stopping) break;
        cv.wait_for(g, std::chrono::milliseconds(20));
      }
    }
    // Shutdown: whatever is left is cancelled.
    for (auto& s : slots)
      if (s) {
        std::shared_ptr<ServeJob> j = s;
        releaseJob(j);
        finish(j, SUNDOG_JOB_CANCELLED, "server stopped");
      }
    std::vector<std::shared_ptr<ServeJob>> rest;
    {
      std::lock_guard<std::mutex> g(mu);
      rest.assign(queue.begin(), queue.end());
      queue.clear();
    }
    for (auto& j : rest) finish(j, SUNDOG_JOB_CANCELLED, "server stopped");
  }
};

sundog_server_config serverDefaults() {
  sundog_server_config c;
  std::memset(&c, 0, sizeof c);
  c.max_jobs = 16;
  c.tile = 64;
  c.pass_spp = 8;
  c.iteration_paths = 1ull << 23;
  c.reserve_bytes = 1ull << 30;
  c.scene_cache_bytes = 8ull << 30;
  return c;
}

}  // namespace sdb

using namespace sdb;

extern "C" void sundog_server_defaults(sundog_server_config* c) {
  if (c) *c = serverDefaults();
}

extern "C" sundog_server* sundog_server_create(const sundog_server_config* c) {
  SDB_TRY
  sundog_server_config cfg = c ? *c : serverDefaults();
  if (cfg.max_jobs < 1 || cfg.max_jobs > kMaxServeJobs)
    throw std::runtime_error("server: max_jobs must be 1..32");
  if (cfg.tile < 8 || cfg.tile % 8 != 0 || cfg.tile > 1024)
    throw std::runtime_error("server: tile must be a multiple of 8 in 8..1024");
  if (cfg.pass_spp < 1) throw std::runtime_error("server: pass_spp must be positive");
  if (cfg.engine < 0 || cfg.engine > 2) throw std::runtime_error("server: engine must be 0, 1 or 2");
  uint64_t itemPaths = (uint64_t)(cfg.tile / 8) * (cfg.tile / 8) * 64 * cfg.pass_spp;
  if (cfg.iteration_paths < itemPaths)
    throw std::runtime_error("server: iteration_paths is smaller than one tile-pass");
  return reinterpret_cast<sundog_server*>(new Server(cfg));
  SDB_CATCH(nullptr)
}

extern "C" sundog_server* sundog_server_create_on_device(const sundog_server_config* c,
                                                        int device) {
  SDB_TRY
  int count = 0;
  cudaCheck(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
  if (device < 0 || device >= count) throw std::runtime_error("server: no such device");
  int prev = 0;
  cudaCheck(cudaGetDevice(&prev), "cudaGetDevice");
  cudaCheck(cudaSetDevice(device), "cudaSetDevice");
  sundog_server* sv = sundog_server_create(c);  // the server keeps the device current then
  cudaSetDevice(prev);
  return sv;
  SDB_CATCH(nullptr)
}

extern "C" int sundog_device_count(void) {
  int n = 0;
  return cudaGetDeviceCount(&n) == cudaSuccess ? n : -1;
}

extern "C" int64_t sundog_server_submit(sundog_server* sv, sundog_scene* h,
                                        const sundog_render_options* opt, float* film) {
  SDB_TRY
  if (!sv || !h) throw std::runtime_error("server: null argument");
  if (sundog_scene_validate(h) != SUNDOG_OK) throw std::runtime_error(sundog_last_error());
  return reinterpret_cast<Server*>(sv)->submit(h, opt, film);
  SDB_CATCH(-1)
}

extern "C" int sundog_server_status(sundog_server* sv, int64_t job, sundog_job_status* out) {
  SDB_TRY
  if (!sv || !out) throw std::runtime_error("server: null argument");
  reinterpret_cast<Server*>(sv)->status(job, out);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_server_wait(sundog_server* sv, int64_t job, double timeoutMs,
                                  sundog_job_status* out) {
  SDB_TRY
  if (!sv) throw std::runtime_error("server: null argument");
  if (!reinterpret_cast<Server*>(sv)->wait(job, timeoutMs, out))
    throw std::runtime_error("server: wait timed out");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_server_cancel(sundog_server* sv, int64_t job) {
  SDB_TRY
  if (!sv) throw std::runtime_error("server: null argument");
  if (!reinterpret_cast<Server*>(sv)->cancel(job))
    throw std::runtime_error("server: job already finished");
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" int sundog_server_stats(sundog_server* sv, sundog_server_statistics* out) {
  SDB_TRY
  if (!sv || !out) throw std::runtime_error("server: null argument");
  reinterpret_cast<Server*>(sv)->stats(out);
  return SUNDOG_OK;
  SDB_CATCH(SUNDOG_ERROR)
}

extern "C" void sundog_server_destroy(sundog_server* sv) {
  delete reinterpret_cast<Server*>(sv);
}
