// server.cu -- a frame-serving loop over the grid builder and the map.
//
// The reference renders one scene at a time from a host program
// (BT/BlackTracer.cpp main: grids, then Distorter::drawBlocks / makeImage per
// frame).  This is the serving form of that path: requests (resolution,
// camera, spin) arrive from any thread; one worker thread owns all device
// work and runs continuous batching --
//   * admission: a request enters when a render slot of its resolution and
//     the HBM for its grid are available (grid cache budget, render budget,
//     in-flight cap); otherwise it waits, in arrival order;
//   * grids: resident in a cache keyed by the exact camera and spin (a
//     request for a resident pose reuses it), evicted least recently used
//     when the budget is full and no in-flight frame uses them; the grids
//     missing at an admission round are built together as one grid set
//     (bt_batch), one set build in flight at a time;
//   * frames: every admitted request renders on its slot's own stream, after
//     an event that marks its grid ready, so frames of different requests
//     and the next grid build overlap on the device; the frame is copied to
//     the caller's host buffer on the same stream.
// Completions carry submit / admit / done times for latency statistics.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bt_internal.h"
#include "map_internal.h"

using bt::clear_error;
using bt::set_error;

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct PoseKey {
  double v[13];  // the 12 camera fields and the spin
  bool operator==(const PoseKey& o) const { return std::memcmp(v, o.v, sizeof(v)) == 0; }
};

struct PoseHash {
  size_t operator()(const PoseKey& k) const {
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the bytes
    const unsigned char* p = (const unsigned char*)k.v;
    for (size_t i = 0; i < sizeof(k.v); i++) h = (h ^ p[i]) * 1099511628211ull;
    return (size_t)h;
  }
};

struct Entry {
  PoseKey key;
  bt_camera cam;
  double a;
  float2* grid = nullptr;  // resident map grid (rows x cols float2)
  cudaEvent_t ready = nullptr;
  int state = 0;           // 0 waiting for a build, 1 build enqueued
  int pins = 0;            // admitted requests using it
  std::list<Entry*>::iterator lru;
};

struct Request {
  bt_request r;
  double t_submit = 0, t_admit = 0;
  int reused = 0;  // its grid came from the cache
};

struct Slot {
  int W = 0, H = 0;
  size_t bytes = 0;
  bt_map* map = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  uint8_t* dev_out = nullptr;
  bool busy = false;
  bool rendered = false;  // render enqueued (else waiting for its grid's build)
  Request req;
  Entry* entry = nullptr;
};

// Device bytes of a renderer of W x H (bt_map_create + star cells of step s).
size_t map_bytes(int W, int H, int step) {
  const size_t np = (size_t)W * H, nc = (size_t)(W + 1) * (H + 1);
  const size_t fw = 2 * (size_t)step + 1;
  return nc * (8 + 4) + np * (1 + 4 + 4 + 12 + 12 + 4 + 1 + 4 + 4 + 4 + 4 + 4) +
         np * fw * fw * 12 + np * 4 /* frame */ + bt::map_star_scratch_bytes(np, (int)fw) +
         (1 << 16);
}

}  // namespace

struct bt_server {
  bt_server_config cfg{};
  int device = 0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;       // new work or stop
  std::condition_variable done_cv;  // new completions
  bool stop = false;
  std::deque<Request> incoming;
  std::deque<bt_completion> done;
  bt_server_stats stats{};
  // worker-owned
  std::deque<Request> pending;
  std::unordered_map<PoseKey, Entry*, PoseHash> cache;
  std::list<Entry*> lru;  // front = most recently used
  size_t grid_bytes_used = 0;
  size_t grid_bytes = 0;  // one map grid
  int32_t grid_rows = 0, grid_cols = 0;
  std::vector<Slot> slots;
  size_t slot_bytes_used = 0;
  std::map<std::pair<int, int>, float*> views;
  bt_batch* set = nullptr;
  // Stream priorities: grid builds first (a build is a chain of short
  // latency-bound launches that frames of other requests wait for), then
  // frames by size, smaller first (slot_priority).
  cudaStream_t build_stream = nullptr;
  int prio_least = 0, prio_greatest = 0;
  char* arena = nullptr;                // the grid cache's memory
  std::vector<float2*> free_grids;      // unused grid slices of the arena
  cudaEvent_t build_done = nullptr;
  bool building = false;
  std::vector<Entry*> to_build;
  bt_integ_opts opts{};
};

namespace {

void complete(bt_server* S, const Request& q, int status, int reused) {
  bt_completion c;
  std::memset(&c, 0, sizeof(c));
  c.id = q.r.id;
  c.status = status;
  c.grid_reused = reused;
  c.t_submit = q.t_submit;
  c.t_admit = q.t_admit;
  c.t_done = now_s();
  std::lock_guard<std::mutex> lk(S->mu);
  S->done.push_back(c);
  if (status == BT_OK) S->stats.completed++;
  else S->stats.failed++;
  S->done_cv.notify_all();
}

// Grid buffers are slices of one arena of the whole grid-cache budget,
// reserved when the server is created: growing device memory while frames
// run (cudaMalloc, or a stream-ordered pool that has to map more memory)
// blocked the worker thread for up to hundreds of milliseconds.
void entry_free(bt_server* S, Entry* e);

void entry_free(bt_server* S, Entry* e) {
  if (e->grid) S->free_grids.push_back(e->grid);
  if (e->ready) cudaEventDestroy(e->ready);
  delete e;
}

// Makes room for `bytes` of grids by evicting unpinned, built entries.
bool grid_room(bt_server* S, size_t bytes) {
  while (S->grid_bytes_used + bytes > S->cfg.grid_cache_bytes) {
    Entry* victim = nullptr;
    for (auto it = S->lru.rbegin(); it != S->lru.rend(); ++it)
      if ((*it)->pins == 0 && (*it)->state == 1) {
        victim = *it;
        break;
      }
    if (!victim) return false;
    if (cudaEventQuery(victim->ready) != cudaSuccess) return false;  // still building
    S->lru.erase(victim->lru);
    S->cache.erase(victim->key);
    S->grid_bytes_used -= S->grid_bytes;
    entry_free(S, victim);
    std::lock_guard<std::mutex> lk(S->mu);
    S->stats.evictions++;
  }
  return true;
}

float* view_for(bt_server* S, int W, int H) {
  auto it = S->views.find({W, H});
  if (it != S->views.end()) return it->second;
  float* v = nullptr;
  if (cudaMalloc((void**)&v, (size_t)2 * (W + 1) * (H + 1) * sizeof(float)) != cudaSuccess)
    return nullptr;
  if (bt_view_sphere(v, W, H, S->build_stream) != BT_OK) {
    cudaFree(v);
    return nullptr;
  }
  cudaStreamSynchronize(S->build_stream);
  S->views[{W, H}] = v;
  return v;
}

// Priority of the stream of a W x H frame: one level below builds for
// frames up to 1 MP, two up to 4 MP, the least above (clamped to the
// device's range; numerically lower is higher priority).
int slot_priority(const bt_server* S, int W, int H) {
  const double mp = (double)W * H / 1e6;
  const int p = S->prio_greatest + (mp <= 1.0 ? 1 : mp <= 4.0 ? 2 : 3);
  return std::min(std::max(p, S->prio_greatest), S->prio_least);
}

// An idle slot for W x H: reuse one of that size, else create one within
// the render budget (freeing idle slots of other sizes if needed).
Slot* slot_for(bt_server* S, int W, int H) {
  for (Slot& s : S->slots)
    if (!s.busy && s.W == W && s.H == H) return &s;
  int busy = 0;
  for (Slot& s : S->slots) busy += s.busy ? 1 : 0;
  if (busy >= S->cfg.max_inflight) return nullptr;
  const size_t need = map_bytes(W, H, S->cfg.step);
  while (S->slot_bytes_used + need > S->cfg.render_bytes) {
    auto it = std::find_if(S->slots.begin(), S->slots.end(),
                           [](const Slot& s) { return !s.busy; });
    if (it == S->slots.end()) return nullptr;
    bt_map_destroy(it->map);
    cudaFree(it->dev_out);
    cudaStreamDestroy(it->stream);
    cudaEventDestroy(it->done);
    S->slot_bytes_used -= it->bytes;
    S->slots.erase(it);
  }
  Slot s;
  s.W = W;
  s.H = H;
  s.bytes = need;
  if (bt_map_create(W, H, &s.map) != BT_OK) return nullptr;
  if (cudaMalloc((void**)&s.dev_out, (size_t)W * H * 4) != cudaSuccess ||
      cudaStreamCreateWithPriority(&s.stream, cudaStreamNonBlocking,
                                   slot_priority(S, W, H)) != cudaSuccess ||
      cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
    bt_map_destroy(s.map);
    if (s.dev_out) cudaFree(s.dev_out);
    return nullptr;
  }
  S->slot_bytes_used += need;
  S->slots.push_back(s);
  return &S->slots.back();
}

// Enqueues the frame of an admitted slot whose grid build is enqueued.
int render(bt_server* S, Slot& sl) {
  const bt_request& r = sl.req.r;
  float* view = view_for(S, sl.W, sl.H);
  if (!view) return BT_ERR_NOMEM;
  BT_CUDA_TRY(cudaStreamWaitEvent(sl.stream, sl.entry->ready, 0));
  bt_frame f;
  std::memset(&f, 0, sizeof(f));
  f.grid = (const float*)sl.entry->grid;
  f.grid_rows = S->grid_rows;
  f.grid_cols = S->grid_cols;
  f.grid_level = S->cfg.maxlevel;
  f.view = view;
  if (int rc = bt_camera_params(&sl.entry->cam, f.cam)) return rc;
  f.env = S->cfg.env;
  f.stars = S->cfg.stars;
  f.map = S->cfg.env ? 1 : 0;
  f.star = S->cfg.stars ? 1 : 0;
  f.lr = S->cfg.lr;
  f.step = S->cfg.step;
  f.out = sl.dev_out;
  if (int rc = bt_map_render(sl.map, &f, sl.stream)) return rc;
  BT_CUDA_TRY(cudaMemcpyAsync(r.out, sl.dev_out, (size_t)sl.W * sl.H * 4, cudaMemcpyDefault,
                              sl.stream));
  BT_CUDA_TRY(cudaEventRecord(sl.done, sl.stream));
  sl.rendered = true;
  return BT_OK;
}

// One grid-set build of up to the set size of the waiting entries.
int launch_builds(bt_server* S) {
  if (S->to_build.empty() || S->building) return BT_OK;
  const int n = std::min((int)S->to_build.size(), S->cfg.max_build_batch);
  std::vector<bt_camera> cams(n);
  std::vector<double> spins(n);
  for (int k = 0; k < n; k++) {
    cams[k] = S->to_build[k]->cam;
    spins[k] = S->to_build[k]->a;
  }
  if (int rc = bt_batch_build_first(S->set, n, cams.data(), spins.data(), S->cfg.startlevel,
                                    &S->opts, S->build_stream))
    return rc;
  for (int k = 0; k < n; k++) {
    Entry* e = S->to_build[k];
    if (int rc = bt::grid_map_export_into(bt_batch_grid(S->set, k), (float*)e->grid,
                                          S->build_stream))
      return rc;
    BT_CUDA_TRY(cudaEventRecord(e->ready, S->build_stream));
    e->state = 1;
  }
  BT_CUDA_TRY(cudaEventRecord(S->build_done, S->build_stream));
  S->building = true;
  S->to_build.erase(S->to_build.begin(), S->to_build.begin() + n);
  std::lock_guard<std::mutex> lk(S->mu);
  S->stats.grids_built += n;
  S->stats.build_sets++;
  return BT_OK;
}

// Admits waiting requests in arrival order while resources allow.
void admit(bt_server* S) {
  while (!S->pending.empty()) {
    Request& q = S->pending.front();
    const bt_request& r = q.r;
    PoseKey key;
    std::memcpy(key.v, &r.cam, sizeof(bt_camera));
    key.v[12] = r.a;
    auto it = S->cache.find(key);
    Entry* e = it == S->cache.end() ? nullptr : it->second;
    if (map_bytes(r.width, r.height, S->cfg.step) > S->cfg.render_bytes) {
      // its frame can never fit the render budget: fail it instead of
      // holding it (and every request behind it) forever
      Request fail = q;
      S->pending.pop_front();
      complete(S, fail, BT_ERR_NOMEM, 0);
      continue;
    }
    if (!e && !grid_room(S, S->grid_bytes)) return;  // wait for grids to unpin
    Slot* sl = slot_for(S, r.width, r.height);
    if (!sl) return;  // wait for a slot
    int reused = 1;
    if (!e) {
      reused = 0;
      e = new (std::nothrow) Entry;
      if (e && !S->free_grids.empty()) {
        e->grid = S->free_grids.back();
        S->free_grids.pop_back();
      }
      if (!e || !e->grid ||
          cudaEventCreateWithFlags(&e->ready, cudaEventDisableTiming) != cudaSuccess) {
        if (e) entry_free(S, e);
        Request fail = q;
        S->pending.pop_front();
        complete(S, fail, BT_ERR_NOMEM, 0);
        continue;
      }
      e->key = key;
      e->cam = r.cam;
      e->a = r.a;
      S->cache[key] = e;
      S->lru.push_front(e);
      e->lru = S->lru.begin();
      S->grid_bytes_used += S->grid_bytes;
      S->to_build.push_back(e);
    } else {
      S->lru.erase(e->lru);
      S->lru.push_front(e);
      e->lru = S->lru.begin();
    }
    e->pins++;
    sl->busy = true;
    sl->rendered = false;
    sl->entry = e;
    sl->req = q;
    sl->req.t_admit = now_s();
    sl->req.reused = reused;
    S->pending.pop_front();
    std::lock_guard<std::mutex> lk(S->mu);
    if (reused) S->stats.grid_hits++;
    else S->stats.grid_misses++;
  }
}

void worker_main(bt_server* S) {
  cudaSetDevice(S->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      bool idle = S->incoming.empty() && S->pending.empty() && !S->building;
      for (Slot& s : S->slots) idle = idle && !s.busy;
      if (idle) {
        if (S->stop) break;
        S->cv.wait_for(lk, std::chrono::milliseconds(50));
      }
      while (!S->incoming.empty()) {
        S->pending.push_back(S->incoming.front());
        S->incoming.pop_front();
      }
    }
    // retire finished frames
    for (Slot& s : S->slots) {
      if (!s.busy || !s.rendered) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) continue;
      s.entry->pins--;
      s.busy = false;
      complete(S, s.req, q == cudaSuccess ? BT_OK : BT_ERR_CUDA, s.req.reused);
    }
    if (S->building && cudaEventQuery(S->build_done) != cudaErrorNotReady) S->building = false;
    admit(S);
    if (int rc = launch_builds(S)) {
      // fail every request waiting for a build that could not be enqueued
      for (Slot& s : S->slots)
        if (s.busy && !s.rendered && s.entry->state == 0) {
          s.entry->pins--;
          s.busy = false;
          complete(S, s.req, rc, 0);
        }
    }
    for (Slot& s : S->slots)
      if (s.busy && !s.rendered && s.entry->state == 1) {
        if (int rc = render(S, s)) {
          s.entry->pins--;
          s.busy = false;
          complete(S, s.req, rc, 0);
        }
      }
    // short sleep while work is on the device
    std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
}

}  // namespace

extern "C" {

void bt_server_config_default(bt_server_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->maxlevel = 11;
  c->startlevel = 6;
  c->angle = 1;
  c->precision = BT_PRECISION_FAST;
  c->grid_cache_bytes = (size_t)40 << 30;
  c->render_bytes = (size_t)40 << 30;
  c->max_inflight = 16;
  c->max_build_batch = 8;
  c->step = 1;
  c->lr = 1;
}

int bt_server_create(const bt_server_config* cfg, bt_server** out) {
  clear_error();
  BT_ARG_CHECK(cfg && out, "NULL pointer");
  BT_ARG_CHECK(cfg->max_inflight >= 1 && cfg->max_build_batch >= 1 &&
                   cfg->max_build_batch <= 1024,
               "max_inflight and max_build_batch must be positive (batch <= 1024)");
  BT_ARG_CHECK(cfg->step >= 0 && cfg->step <= 2, "step out of [0, 2]");
  *out = nullptr;
  int32_t N, M;
  if (int rc = bt_grid_dims(cfg->maxlevel, cfg->angle, &N, &M)) return rc;
  bt_server* S = new (std::nothrow) bt_server;
  if (!S) return BT_ERR_NOMEM;
  S->cfg = *cfg;
  cudaGetDevice(&S->device);
  bt_integ_opts_default(&S->opts);
  S->opts.precision = cfg->precision;
  // map grid shape (bt_grid_map_export): half grids are mirrored to 2N-1 rows
  const int sym = (float)M / (float)N > 3 ? 1 : 0;
  S->grid_rows = sym ? 2 * N - 1 : N;
  S->grid_cols = M;
  S->grid_bytes = (size_t)S->grid_rows * S->grid_cols * sizeof(float2);
  BT_ARG_CHECK(S->grid_bytes <= cfg->grid_cache_bytes, "grid cache smaller than one grid");
  int rc = bt_batch_create(cfg->maxlevel, cfg->angle, cfg->max_build_batch, &S->set);
  // the T-vertex fix as a launch per pass: builds share the device with
  // frames on other streams, and a cooperative launch must wait until all of
  // its blocks fit at once (p99 at 120 requests/s: 56-58 ms against 79-84)
  if (rc == BT_OK) rc = bt_grid_set_tfix_launch(bt_batch_grid(S->set, 0), 0);
  cudaDeviceGetStreamPriorityRange(&S->prio_least, &S->prio_greatest);
  if (rc == BT_OK) {
    const size_t n = cfg->grid_cache_bytes / S->grid_bytes;
    if (cudaMalloc((void**)&S->arena, n * S->grid_bytes) != cudaSuccess) {
      set_error("grid cache of %zu bytes could not be reserved", n * S->grid_bytes);
      rc = BT_ERR_NOMEM;
    } else {
      S->free_grids.reserve(n);
      for (size_t k = n; k-- > 0;)
        S->free_grids.push_back((float2*)(S->arena + k * S->grid_bytes));
    }
  }
  if (rc == BT_OK && (cudaStreamCreateWithPriority(&S->build_stream, cudaStreamNonBlocking,
                                                   S->prio_greatest) != cudaSuccess ||
                      cudaEventCreateWithFlags(&S->build_done, cudaEventDisableTiming) !=
                          cudaSuccess))
    rc = BT_ERR_CUDA;
  if (rc) {
    if (S->set) bt_batch_destroy(S->set);
    if (S->arena) cudaFree(S->arena);
    delete S;
    return rc;
  }
  S->worker = std::thread(worker_main, S);
  *out = S;
  return BT_OK;
}

int bt_server_submit(bt_server* S, const bt_request* r) {
  clear_error();
  BT_ARG_CHECK(S && r && r->out, "NULL pointer");
  BT_ARG_CHECK(r->width > 0 && r->height > 0 && (size_t)r->width * r->height <= ((size_t)1 << 28),
               "image size out of range");
  Request q;
  q.r = *r;
  q.t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) {
      set_error("server is shutting down");
      return BT_ERR_STATE;
    }
    S->incoming.push_back(q);
    S->stats.submitted++;
  }
  S->cv.notify_one();
  return BT_OK;
}

int bt_server_poll(bt_server* S, bt_completion* out, int cap, int* n, int wait_ms) {
  clear_error();
  BT_ARG_CHECK(S && out && n && cap > 0, "invalid arguments");
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->done.empty() && wait_ms > 0)
    S->done_cv.wait_for(lk, std::chrono::milliseconds(wait_ms),
                        [&] { return !S->done.empty(); });
  int k = 0;
  while (k < cap && !S->done.empty()) {
    out[k++] = S->done.front();
    S->done.pop_front();
  }
  *n = k;
  return BT_OK;
}

int bt_server_stats_get(bt_server* S, bt_server_stats* st) {
  BT_ARG_CHECK(S && st, "NULL pointer");
  std::lock_guard<std::mutex> lk(S->mu);
  *st = S->stats;
  st->grids_resident = (int64_t)(S->grid_bytes_used / (S->grid_bytes ? S->grid_bytes : 1));
  st->grid_cache_bytes_used = S->grid_bytes_used;
  st->render_bytes_used = S->slot_bytes_used;
  return BT_OK;
}

void bt_server_destroy(bt_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  if (S->worker.joinable()) S->worker.join();  // drains: returns once idle
  cudaStreamSynchronize(S->build_stream);
  for (Slot& s : S->slots) {
    cudaStreamSynchronize(s.stream);
    bt_map_destroy(s.map);
    cudaFree(s.dev_out);
    cudaStreamDestroy(s.stream);
    cudaEventDestroy(s.done);
  }
  for (auto& kv : S->cache) entry_free(S, kv.second);
  if (S->arena) cudaFree(S->arena);
  for (auto& kv : S->views) cudaFree(kv.second);
  bt_batch_destroy(S->set);
  cudaEventDestroy(S->build_done);
  cudaStreamDestroy(S->build_stream);
  delete S;
}

}  // extern "C"
