// bn_server.cpp -- continuous-batching render server (bnxServer*, no
// reference counterpart).
//
// Requests name a resident volume (a built BNModel), a renderer (its
// parameters are copied at submission), a camera, an image size and a wave
// count.  One worker thread owns the context's stream and loops:
//
//   1. admit queued requests, in arrival order, while their per-request
//      device buffers (accumulation, compensation, colour) fit the HBM budget
//      and a batch slot is free;
//   2. render one slice -- at most sliceWaves waves of every admitted request
//      -- in one persistent launch of the batch kernel (renderBatch);
//   3. requests whose waves are all done keep only their resolved colour
//      buffer (counted against the budget until the client reads it); their
//      other device buffers return to the pool and waiters are woken.
//
// Requests that arrive while a slice is on the GPU join the next slice, so
// their work overlaps with every other admitted request's on the device.
// A request's result does not depend on what it was batched with: its pixels
// are accumulated in wave order by one lane each, with per-pixel RNG streams
// keyed by (pixel, accumID), never by queue position.
#include "bn_objects.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <map>
#include <thread>

namespace bnb {

using Clock = std::chrono::steady_clock;

struct ServerRequest {
  long long id = 0;
  std::shared_ptr<Model> model;
  std::shared_ptr<Renderer> renderer;  // private copy of the submitted renderer's parameters
  std::shared_ptr<Camera> camera;
  std::shared_ptr<FrameBuffer> fb;     // device buffers while admitted
  int spp = 1, wavesDone = 0;
  size_t deviceBytes = 0;
  Clock::time_point submitted, admitted, finished;
  bool done = false, failed = false;
  std::string error;
  void *result = nullptr;   // device colour channel, held until the client reads it
  size_t resultBytes = 0;
};

// Device buffers of admitted requests.  Buffers are carved out of large
// chunks (one cudaMalloc per kChunkBytes, 256-byte aligned) and, once
// released, kept on a free list keyed by size for the next request of that
// size: a cudaMalloc per request measured several milliseconds each inside a
// serving process, and admitting a burst of requests stalled the GPU for
// hundreds of milliseconds.  The worker takes buffers; client threads return
// colour buffers after reading them.  Chunks are freed with the server.
struct BufferPool {
  static constexpr size_t kChunkBytes = (size_t)256 << 20;
  struct Chunk {
    unsigned char *base;
    size_t size, used;
  };
  std::mutex m;
  std::multimap<size_t, void *> freeDevice;
  std::vector<Chunk> chunks;
  size_t deviceBytesHeld = 0;
  ~BufferPool() {
    for (auto &c : chunks) cudaFree(c.base);
  }
  void *getDevice(size_t n) {
    const size_t need = (n + 255) & ~(size_t)255;
    {
      std::lock_guard<std::mutex> l(m);
      auto it = freeDevice.find(n);
      if (it != freeDevice.end()) { void *p = it->second; freeDevice.erase(it); return p; }
      for (auto &c : chunks)  // first chunk with room at its end
        if (c.size - c.used >= need) {
          void *p = c.base + c.used;
          c.used += need;
          return p;
        }
    }
    // a new chunk, not under the lock: cudaMalloc can take milliseconds
    const size_t size = std::max(kChunkBytes, need);
    void *base = nullptr;
    ck(deviceMalloc(&base, size), "server buffer chunk");
    std::lock_guard<std::mutex> l(m);
    chunks.push_back({(unsigned char *)base, size, need});
    deviceBytesHeld += size;
    return base;
  }
  void putDevice(void *p, size_t n) {
    if (!p) return;
    std::lock_guard<std::mutex> l(m);
    freeDevice.emplace(n, p);
  }
  // chunks until at least `bytes` are held, so that serving allocates nothing
  void reserve(size_t bytes) {
    while (true) {
      {
        std::lock_guard<std::mutex> l(m);
        if (deviceBytesHeld >= bytes) return;
      }
      void *base = nullptr;
      ck(deviceMalloc(&base, kChunkBytes), "server buffer chunk");
      std::lock_guard<std::mutex> l(m);
      chunks.push_back({(unsigned char *)base, kChunkBytes, 0});
      deviceBytesHeld += kChunkBytes;
    }
  }
};

struct Server {
  Context *ctx;
  BNXServerConfig cfg;
  std::mutex m;
  std::condition_variable cvWork, cvDone;
  std::deque<std::shared_ptr<ServerRequest>> queue;
  std::vector<std::shared_ptr<ServerRequest>> active;
  std::unordered_map<long long, std::shared_ptr<ServerRequest>> finished;
  long long nextId = 0;
  size_t bytesInUse = 0, peakBytes = 0;
  bool stop = false;
  BufferPool pool;
  std::thread worker;
  // statistics
  std::vector<double> latenciesMs, queueWaitsMs;
  double maxSliceMs = 0.0;
  FILE *trace = nullptr;  // BNX_SERVER_TRACE: one line per launch
  Clock::time_point created = Clock::now(), lastSliceEnd = Clock::now();
  unsigned long long submittedCount = 0, completedCount = 0, rejectedCount = 0, launches = 0;
  double busySeconds = 0.0;
  Clock::time_point statsStart = Clock::now();
  unsigned long long samples = 0;

  cudaStream_t copyStream = nullptr;  // client read-back, off the render stream

  Server(Context *c, const BNXServerConfig &config) : ctx(c), cfg(config) {
    ck(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking), "server copy stream");
    reserveBatch(ctx, cfg.maxSlots);  // no pinned-table growth while serving
    if (const char *path = std::getenv("BNX_SERVER_TRACE")) {
      trace = std::fopen(path, "a");
      if (trace)
        std::fprintf(trace,
                     "# start_ms gap_ms admit_ms dur_ms requests admitted retired queued waves pixel_waves\n");
    }
    worker = std::thread([this] { loop(); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> l(m);
      stop = true;
    }
    cvWork.notify_all();
    if (worker.joinable()) worker.join();
    for (auto &r : active) releaseDevice(*r);
    for (auto &kv : finished) releaseResult(*kv.second);
    if (copyStream) cudaStreamDestroy(copyStream);
    if (trace) std::fclose(trace);
    cudaGetLastError();
  }

  void releaseResult(ServerRequest &r) {
    if (!r.result) return;
    pool.putDevice(r.result, r.resultBytes);
    bytesInUse -= r.resultBytes;
    r.result = nullptr;
  }

  static size_t bytesFor(int w, int h, int fmt, bool comp) {
    const size_t px = (size_t)w * h;
    return px * 16 + (comp ? px * 16 : 0) + px * (fmt == FMT_FLOAT4 ? 16 : 4);
  }

  // Returns the request's accumulation buffers to the pool; the colour buffer
  // moves to r.result when keepColor (completed requests), else it is freed too.
  void releaseDevice(ServerRequest &r, bool keepColor = false) {
    if (!r.fb) return;
    const size_t px = (size_t)r.fb->width * r.fb->height;
    pool.putDevice(r.fb->accum.ptr, px * 16);
    if (r.fb->comp.ptr) pool.putDevice(r.fb->comp.ptr, px * 16);
    if (keepColor) {
      r.result = r.fb->color.ptr;
      r.resultBytes = r.fb->color.bytes;
    } else {
      pool.putDevice(r.fb->color.ptr, r.fb->color.bytes);
    }
    bytesInUse -= r.deviceBytes - (keepColor ? r.fb->color.bytes : 0);
    r.fb->accum.ptr = r.fb->comp.ptr = r.fb->color.ptr = nullptr;  // owned by the pool / result now
    r.fb->accum.bytes = r.fb->comp.bytes = r.fb->color.bytes = 0;
    r.fb.reset();
  }

  // device buffers of an admitted request (from the pool); its bytes were
  // reserved against the budget when it was picked for admission
  void acquireDevice(ServerRequest &r) {
    auto fb = std::make_shared<FrameBuffer>(ctx);
    const int w = r.fb ? r.fb->width : 0, h = r.fb ? r.fb->height : 0;
    const int fmt = r.fb ? r.fb->colorFormat : FMT_RGBA8;
    fb->width = w;
    fb->height = h;
    fb->colorFormat = fmt;
    const size_t px = (size_t)w * h;
    const size_t cb = px * (fmt == FMT_FLOAT4 ? 16 : 4);
    try {
      fb->accum.ptr = pool.getDevice(px * 16);
      fb->accum.bytes = px * 16;
      if (r.renderer->p.compensatedAccum) {
        fb->comp.ptr = pool.getDevice(px * 16);
        fb->comp.bytes = px * 16;
        ck(cudaMemsetAsync(fb->comp.ptr, 0, px * 16, ctx->stream), "compensation clear");
      }
      fb->color.ptr = pool.getDevice(cb);
      fb->color.bytes = cb;
    } catch (...) {  // give back what was taken; the pool owns the buffers
      pool.putDevice(fb->accum.ptr, fb->accum.bytes);
      pool.putDevice(fb->comp.ptr, fb->comp.bytes);
      fb->accum.ptr = fb->comp.ptr = nullptr;
      throw;
    }
    fb->accumID = 0;
    r.fb = fb;
  }

  void loop() {
    cudaSetDevice(ctx->device);
    while (true) {
      std::vector<std::shared_ptr<ServerRequest>> slice, admit;
      int admittedNow = 0;
      size_t queuedNow = 0;
      double admitMs = 0.0;
      {
        std::unique_lock<std::mutex> l(m);
        cvWork.wait(l, [&] { return stop || !queue.empty() || !active.empty(); });
        if (stop) return;
        // 1. admission, in arrival order, by HBM budget and slots: the
        //    bytes are reserved here, the buffers taken below without the lock
        while (!queue.empty() && (int)(active.size() + admit.size()) < cfg.maxSlots) {
          auto r = queue.front();
          if (r->deviceBytes > cfg.hbmBudgetBytes) {  // can never fit: reject
            queue.pop_front();
            r->failed = true;
            r->error = "request needs more device memory than the server's budget";
            r->done = true;
            rejectedCount++;
            finished[r->id] = r;
            cvDone.notify_all();
            continue;
          }
          if (bytesInUse + r->deviceBytes > cfg.hbmBudgetBytes) break;
          queue.pop_front();
          bytesInUse += r->deviceBytes;
          peakBytes = std::max(peakBytes, bytesInUse);
          admit.push_back(r);
        }
      }
      const auto ta = Clock::now();
      std::vector<std::shared_ptr<ServerRequest>> noMemory;
      for (auto &r : admit) {
        try {
          acquireDevice(*r);
        } catch (const Error &) {  // out of device memory: retry once others finish
          noMemory.push_back(r);
        }
      }
      admitMs = std::chrono::duration<double, std::milli>(Clock::now() - ta).count();
      {
        std::lock_guard<std::mutex> l(m);
        for (auto &r : admit) {
          if (std::find(noMemory.begin(), noMemory.end(), r) != noMemory.end()) continue;
          r->admitted = Clock::now();
          queueWaitsMs.push_back(std::chrono::duration<double, std::milli>(r->admitted - r->submitted).count());
          active.push_back(r);
          admittedNow++;
        }
        for (auto it = noMemory.rbegin(); it != noMemory.rend(); ++it) {
          bytesInUse -= (*it)->deviceBytes;
          if (active.empty()) {  // nothing will free memory: the request cannot run
            auto &r = *it;
            r->failed = true;
            r->error = "out of device memory for the request's buffers";
            r->done = true;
            rejectedCount++;
            finished[r->id] = r;
            cvDone.notify_all();
          } else {
            queue.push_front(*it);
          }
        }
        slice = active;
        queuedNow = queue.size();
      }
      if (slice.empty()) {
        std::this_thread::sleep_for(std::chrono::microseconds(200));
        continue;
      }
      // 2. one slice of waves for every admitted request, one launch
      std::vector<BatchEntry> entries;
      std::vector<int> waves;
      long long sliceWaves = 0, pixelWaves = 0;
      {
        // oldest first (active is in admission order) while the slice's
        // pixel-waves fit cfg.slicePixelWaves; the others wait for the next
        // launch, so that no slice holds the GPU for long
        std::vector<std::shared_ptr<ServerRequest>> inSlice;
        for (auto &r : slice) {
          const int n = std::min(cfg.sliceWaves, r->spp - r->wavesDone);
          const long long pw = (long long)n * r->fb->width * r->fb->height;
          if (!inSlice.empty() && cfg.slicePixelWaves > 0 && pixelWaves + pw > cfg.slicePixelWaves) continue;
          sliceWaves += n;
          pixelWaves += pw;
          r->renderer->p.pathsPerPixel = n;
          waves.push_back(n);
          entries.push_back({r->renderer.get(), r->model.get(), r->camera.get(), r->fb.get()});
          inSlice.push_back(r);
        }
        slice.swap(inSlice);
      }
      const auto t0 = Clock::now();
      NvtxRange range("server slice");
      std::string err;
      const bool graphs = ctx->useGraphs;
      ctx->useGraphs = false;  // the batch changes every slice: plain launches
      try {
        renderBatch(ctx, entries);
      } catch (const std::exception &e) {
        err = e.what();
      }
      ctx->useGraphs = graphs;
      const auto t1 = Clock::now();
      // 3. completions
      std::lock_guard<std::mutex> l(m);
      const double durMs = std::chrono::duration<double, std::milli>(t1 - t0).count();
      busySeconds += durMs * 1e-3;
      maxSliceMs = std::max(maxSliceMs, durMs);
      launches++;
      samples += ctx->stats.samples;
      int retiredNow = 0;
      std::vector<std::shared_ptr<ServerRequest>> still;
      for (size_t i = 0; i < slice.size(); i++) {
        auto &r = slice[i];
        r->wavesDone += waves[i];
        if (err.empty() && r->wavesDone < r->spp) { still.push_back(r); continue; }
        if (!err.empty()) {
          r->failed = true;
          r->error = err;
        }
        r->finished = Clock::now();
        r->done = true;
        retiredNow++;
        releaseDevice(*r, !r->failed);
        if (!r->failed) {
          latenciesMs.push_back(std::chrono::duration<double, std::milli>(r->finished - r->submitted).count());
          completedCount++;
        }
        finished[r->id] = r;
      }
      // requests left out of this slice stay active, in admission order
      {
        std::vector<std::shared_ptr<ServerRequest>> next;
        size_t si = 0;
        for (auto &r : active) {
          if (si < slice.size() && slice[si] == r) {
            si++;
            if (!r->done) next.push_back(r);
          } else {
            next.push_back(r);
          }
        }
        active.swap(next);
      }
      (void)still;
      if (trace) {
        std::fprintf(trace, "%.3f %.3f %.3f %.3f %zu %d %d %zu %lld %lld\n",
                     std::chrono::duration<double, std::milli>(t0 - created).count(),
                     std::chrono::duration<double, std::milli>(t0 - lastSliceEnd).count(), admitMs, durMs,
                     slice.size(),
                     admittedNow, retiredNow, queuedNow, sliceWaves, pixelWaves);
        std::fflush(trace);
      }
      lastSliceEnd = t1;
      cvDone.notify_all();
    }
  }
};

static std::mutex g_serverMutex;
static std::unordered_map<Server *, std::unique_ptr<Server>> g_servers;

static Server *getServer(BNXServer h) {
  std::lock_guard<std::mutex> l(g_serverMutex);
  auto it = g_servers.find((Server *)h);
  if (it == g_servers.end()) throw Error(E_INVALID_HANDLE, "invalid BNXServer handle");
  return it->second.get();
}

}  // namespace bnb

using namespace bnb;

extern "C" {

BN_API BNXServer bnxServerCreate(BNContext context, const BNXServerConfig *config) {
  BN_TRY
  Context *c = getContext(context);
  BNXServerConfig cfg{(size_t)150 << 30, 256, 4};
  if (config) cfg = *config;
  if (cfg.maxSlots < 1 || cfg.sliceWaves < 1) throw Error(E_INVALID_ARG, "maxSlots and sliceWaves must be >= 1");
  if (cfg.slicePixelWaves < 0) throw Error(E_INVALID_ARG, "slicePixelWaves must be >= 0");
  c->activate();
  auto s = std::make_unique<Server>(c, cfg);
  Server *raw = s.get();
  std::lock_guard<std::mutex> l(g_serverMutex);
  g_servers[raw] = std::move(s);
  return (BNXServer)raw;
  BN_CATCH(nullptr)
}

BN_API void bnxServerDestroy(BNXServer server) {
  BN_TRY
  Server *s = getServer(server);
  std::unique_ptr<Server> owned;
  {
    std::lock_guard<std::mutex> l(g_serverMutex);
    owned = std::move(g_servers[s]);
    g_servers.erase(s);
  }
  BN_CATCH()
}

BN_API void bnxServerReserve(BNXServer server, size_t bytes) {
  BN_TRY
  Server *s = getServer(server);
  if (bytes > s->cfg.hbmBudgetBytes) throw Error(E_INVALID_ARG, "reservation exceeds the server's HBM budget");
  s->ctx->activate();
  s->pool.reserve(bytes);
  BN_CATCH()
}

BN_API long long bnxServerSubmit(BNXServer server, const BNXRequest *q) {
  BN_TRY
  Server *s = getServer(server);
  if (!q) throw Error(E_INVALID_ARG, "request is null");
  auto r = std::make_shared<ServerRequest>();
  r->submitted = Clock::now();
  r->model = getAs<Model>(q->model, Object::K_MODEL, "BNModel");
  if (!r->model->built) throw Error(E_STATE, "the request's model has not been built");
  auto tmpl = getAs<Renderer>(q->renderer, Object::K_RENDERER, "BNRenderer");
  r->renderer = std::make_shared<Renderer>(s->ctx);
  r->renderer->p = tmpl->p;
  auto cam = std::make_shared<Camera>(s->ctx);
  cam->set3f("position", q->position.x, q->position.y, q->position.z);
  cam->set3f("direction", q->direction.x, q->direction.y, q->direction.z);
  cam->set3f("up", q->up.x, q->up.y, q->up.z);
  cam->set1f("fovy", q->fovy);
  cam->commit();
  r->camera = cam;
  if (q->width <= 0 || q->height <= 0 || q->spp <= 0) throw Error(E_INVALID_ARG, "width, height, spp must be > 0");
  if ((long long)q->width * q->height > kMaxFramePixels) throw Error(E_INVALID_ARG, "frame larger than 2^31 - 1 pixels");
  const int fmt = q->colorFormat == BN_FLOAT4 ? FMT_FLOAT4 : q->colorFormat == BN_UFIXED8_RGBA ? FMT_RGBA8
                : q->colorFormat == BN_UFIXED8_RGBA_SRGB ? FMT_RGBA8_SRGB : -1;
  if (fmt < 0) throw Error(E_UNSUPPORTED, "unsupported colour format");
  auto fb = std::make_shared<FrameBuffer>(s->ctx);  // size holder until admission
  fb->width = q->width;
  fb->height = q->height;
  fb->colorFormat = fmt;
  r->fb = fb;
  r->spp = q->spp;
  r->deviceBytes = Server::bytesFor(q->width, q->height, fmt, r->renderer->p.compensatedAccum != 0);
  {
    std::lock_guard<std::mutex> l(s->m);
    r->id = s->nextId++;
    s->submittedCount++;
    s->queue.push_back(r);
  }
  s->cvWork.notify_one();
  return r->id;
  BN_CATCH(-1)
}

BN_API int bnxServerWait(BNXServer server, long long id, int timeoutMs, void *hostPixels) {
  BN_TRY
  Server *s = getServer(server);
  std::unique_lock<std::mutex> l(s->m);
  auto ready = [&] { return s->finished.count(id) > 0; };
  if (timeoutMs < 0) s->cvDone.wait(l, ready);
  else if (!s->cvDone.wait_for(l, std::chrono::milliseconds(timeoutMs), ready)) return 0;
  auto r = s->finished[id];
  s->finished.erase(id);
  if (r->failed) throw Error(E_CUDA, "request failed: " + r->error);
  void *src = r->result;
  const size_t n = r->resultBytes;
  l.unlock();
  cudaError_t e = cudaSuccess;
  if (hostPixels && src) {
    cudaSetDevice(s->ctx->device);
    e = cudaMemcpyAsync(hostPixels, src, n, cudaMemcpyDefault, s->copyStream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->copyStream);
  }
  l.lock();
  s->releaseResult(*r);
  l.unlock();
  s->cvWork.notify_one();  // freed budget may admit queued requests
  ck(e, "result copy");
  return 1;
  BN_CATCH(-g_lastError)
}

BN_API void bnxServerGetStats(BNXServer server, BNXServerStats *out) {
  BN_TRY
  Server *s = getServer(server);
  if (!out) return;
  std::lock_guard<std::mutex> l(s->m);
  BNXServerStats st{};
  st.submitted = s->submittedCount;
  st.completed = s->completedCount;
  st.rejected = s->rejectedCount;
  st.launches = s->launches;
  st.busySeconds = s->busySeconds;
  st.samples = s->samples;
  st.peakBytes = s->peakBytes;
  st.queued = (unsigned long long)s->queue.size();
  st.active = (unsigned long long)s->active.size();
  const double wall = std::chrono::duration<double>(Clock::now() - s->statsStart).count();
  st.wallSeconds = wall;
  st.framesPerSecond = wall > 0 ? s->completedCount / wall : 0.0;
  if (!s->latenciesMs.empty()) {
    std::vector<double> v = s->latenciesMs;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
    st.p50Ms = pct(0.50);
    st.p99Ms = pct(0.99);
    double sum = 0;
    for (double x : v) sum += x;
    st.meanMs = sum / v.size();
    st.maxMs = v.back();
  }
  if (!s->queueWaitsMs.empty()) {
    std::vector<double> q = s->queueWaitsMs;
    std::sort(q.begin(), q.end());
    st.queueP99Ms = q[std::min(q.size() - 1, (size_t)(0.99 * (q.size() - 1) + 0.5))];
  }
  st.maxSliceMs = s->maxSliceMs;
  *out = st;
  BN_CATCH()
}

BN_API void bnxServerResetStats(BNXServer server) {
  BN_TRY
  Server *s = getServer(server);
  std::lock_guard<std::mutex> l(s->m);
  s->latenciesMs.clear();
  s->queueWaitsMs.clear();
  s->maxSliceMs = 0;
  s->submittedCount = s->completedCount = s->rejectedCount = s->launches = 0;
  s->busySeconds = 0;
  s->samples = 0;
  s->statsStart = Clock::now();
  BN_CATCH()
}

}  // extern "C"
