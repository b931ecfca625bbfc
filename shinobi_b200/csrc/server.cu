// Ray-query server: resident grids, admission by memory budget, continuous
// batching.
//
// A worker thread takes requests from a FIFO queue and packs consecutive ray
// requests -- for any resident scenes, closest-hit or any-hit -- into ONE
// launch of a mixed-scene persistent trace kernel (each lane looks up its
// request's grid in a segment table), up to the staging capacity.  Two
// launch slots alternate, so requests that arrive while one launch is on the
// GPU are packed and copied in for the next one (continuous batching); a
// completer thread finishes launches in order, copies results out and
// records per-request latency.  Scene-update requests rebuild a slot's grid
// on the device after the launches queued before them have finished, so
// every request sees the scene as of its submission order.  With coalescing
// off, every request gets its own launch and nothing overlaps: the plain
// one-launch-per-request path, same kernel.
//
// The reference's closest analogue is DynamicRTEngine's two-stream
// rebuild/render overlap (src/Engine/DynamicRTEngine.h:91-147).
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

#include "internal.h"
#include "trace_coop.cuh"

namespace shn {
namespace {

constexpr int kServeBlock = 128;
constexpr int kUpdaters = 16;  // concurrent scene replacements (distinct slots)
// launches in flight: the uploads of one overlap the trace of the other (3 or
// 4 measured no faster at saturation: 904-1012 against 1000-1033 Mrays/s)
constexpr int kLaunchSlots = 2;

struct ServeSeg {
  uint32_t ray_begin;
  uint32_t anyhit;
  GridView g;
};

struct ServeAcc {
  static constexpr bool kIndirect = false;
  const ServeSeg* __restrict__ segs;
  SHN_D const Geom& geom(uint32_t s) const { return segs[s].g.g; }
  SHN_D const uint2* cells(uint32_t s) const { return segs[s].g.cells; }
  SHN_D const uint2* leaves(uint32_t s) const { return segs[s].g.leaves; }
  SHN_D Refs refs(uint32_t s) const { return Refs{segs[s].g.rv0, segs[s].g.rv1, segs[s].g.rv2}; }
};

// Rays are AoS records of 8 floats: ox, oy, oz, dx, dy, dz, tmax, unused.
__global__ void __launch_bounds__(kServeBlock, 8) k_serve_trace(const ServeSeg* __restrict__ segs, uint32_t nseg,
                                                            const float4* __restrict__ rays, uint32_t n,
                                                            uint32_t* counter, uint32_t* __restrict__ otri,
                                                            float* __restrict__ ot) {
  // incoherent request rays rarely share a cell range: no grouping
  warp_trace_acc<0, false, false>(
      ServeAcc{segs}, n, counter,
      [&](uint32_t i, V3& o, V3& d, float& tmax, uint32_t& seg, uint32_t& anyhit) {
        uint32_t lo = 0, hi = nseg;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (segs[mid].ray_begin <= i) lo = mid; else hi = mid;
        }
        seg = lo;
        anyhit = segs[lo].anyhit;
        const float4 a = rays[2 * (size_t)i], b = rays[2 * (size_t)i + 1];
        o = mk(a.x, a.y, a.z);
        d = mk(a.w, b.x, b.y);
        tmax = b.z;
      },
      [&](uint32_t i, const Hit& h, uint32_t, uint32_t, uint32_t) {
        otri[i] = h.tri;
        ot[i] = h.t;
      });
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace shn

using namespace shn;

struct ServeReq {
  shn_request r;
  uint64_t ticket = 0;
  double t_submit = 0.0, t_done = 0.0;
  shn_status result = SHN_OK;
  bool done = false;
};

struct ServeLaunch {
  cudaStream_t st = nullptr;
  cudaEvent_t ev_done = nullptr;
  float4* d_rays = nullptr;
  uint32_t* d_tri = nullptr;
  float* d_t = nullptr;
  ServeSeg* d_segs = nullptr;
  ServeSeg* h_segs = nullptr;   // pinned
  uint32_t* d_counter = nullptr;
  std::vector<ServeReq*> reqs;
  std::vector<uint32_t> begin;
  uint32_t nrays = 0;
  uint64_t seq = 0;             // launch number (launches complete in issue order)
  bool busy = false;
};

struct ServeSlot {
  shn_scene* scene = nullptr;
  shn_grid* grid = nullptr;
  uint32_t pending = 0;         // updates of this slot handed to the updater, not yet applied
};

// A replaced scene/grid pair, released once every launch issued before the
// replacement (seq <= after_seq) has completed: it becomes its slot's spare,
// whose buffers the slot's next replacement is built into, or is freed.
struct ServeRetired {
  ServeSlot pair;
  uint32_t slot = 0;
  uint64_t after_seq = 0;
};

struct shn_server {
  shn_ctx* ctx = nullptr;
  shn_server_config cfg{};
  std::vector<ServeSlot> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_launch;
  std::deque<ServeReq*> queue;
  std::unordered_map<uint64_t, ServeReq*> reqs;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread worker, completer;
  std::vector<std::thread> updaters;     // scene replacements of different slots run concurrently
  std::vector<cudaStream_t> upd_streams;
  ServeLaunch L[kLaunchSlots];
  std::deque<int> inflight;
  int blocks = 0;
  cudaStream_t update_st = nullptr;
  // asynchronous scene updates (continuous-batching mode)
  std::condition_variable cv_upd;
  std::deque<ServeReq*> upd_q;
  bool stop_upd = false;
  std::vector<ServeRetired> retired;
  // per slot, one released pair kept for the next replacement: rebuilding
  // into its buffers avoids allocating and freeing gigabytes of pool memory
  // per replacement (pool calls of that size block the host for 30-500 ms and
  // hold up every other thread's CUDA calls meanwhile)
  std::vector<ServeSlot> spares;
  std::vector<uint8_t> blocked;  // per slot, scratch of one queue scan
  uint64_t work_gen = 0;         // bumped when a request arrives or an update is applied
  uint32_t upd_outstanding = 0;  // updates handed to the updater and not yet applied
  uint64_t launch_seq = 0, done_seq = 0;
  // stats
  std::vector<double> lat_us;
  std::vector<shn_request_record> records;  // per request, completion order
  uint64_t rays_done = 0, launches = 0, requests_done = 0, updates_done = 0;
  double t_first = 0.0, t_last = 0.0;
  uint64_t max_requests_per_launch = 0;
};

namespace {

void complete(shn_server* s, ServeReq* r, shn_status st) {
  // caller holds s->mu
  r->result = st;
  r->done = true;
  r->t_done = now_s();
  s->lat_us.push_back((r->t_done - r->t_submit) * 1e6);
  shn_request_record rec;
  rec.submit_s = r->t_submit;
  rec.latency_us = (r->t_done - r->t_submit) * 1e6;
  rec.kind = r->r.kind;
  rec.scene = r->r.scene;
  rec.num_rays = r->r.kind == SHN_REQ_UPDATE ? 0u : r->r.num_rays;
  rec.status = st;
  s->records.push_back(rec);
  s->requests_done++;
  if (r->r.kind != SHN_REQ_UPDATE) s->rays_done += r->r.num_rays;
  s->t_last = r->t_done;
  s->cv_done.notify_all();
}

void free_pair(const ServeSlot& p) {
  if (p.grid) shn_grid_destroy(p.grid);
  if (p.scene) shn_scene_destroy(p.scene);
}

// New scene + uniform grid for a slot, built and synchronised on st, into the
// buffers of spare (a released pair of this slot, may be empty) where they
// are large enough.  The spare is consumed either way.
shn_status build_slot(shn_server* s, ServeSlot spare, const float* vtx, uint32_t nv, const uint32_t* idx,
                      uint32_t nt, float lambda, cudaStream_t st, ServeSlot* out) {
  shn_scene* sc = spare.scene;
  shn_status rc = sc ? scene_reload(sc, vtx, nv, idx, nt, st)
                     : shn_scene_create(s->ctx, vtx, nv, idx, nt, SHN_MEM_HOST, st, &sc);
  if (rc) {
    free_pair(spare);
    return rc;
  }
  shn_grid* g = spare.grid;
  if (!g) shn_grid_create(s->ctx, &g);
  shn_grid_params p;
  shn_grid_params_default(SHN_GRID_UNIFORM, &p);
  p.lambda = lambda > 0.f ? lambda : 5.f;
  rc = shn_grid_build(g, sc, &p, st);
  if (rc) {
    shn_grid_destroy(g);
    shn_scene_destroy(sc);
    return rc;
  }
  rc = shn_grid_sync_status(g, st);  // the build's last stage, then its error word
  if (rc) {
    shn_grid_destroy(g);
    shn_scene_destroy(sc);
    return rc;
  }
  out->scene = sc;
  out->grid = g;
  return SHN_OK;
}

// Takes the slot's spare pair (caller holds s->mu).
ServeSlot take_spare(shn_server* s, uint32_t slot) {
  ServeSlot p = s->spares[slot];
  s->spares[slot] = ServeSlot{};
  return p;
}

// Keeps a released pair as the slot's spare if it has none; otherwise
// returns it to be freed (caller holds s->mu; frees after unlocking).
void release_pair(shn_server* s, uint32_t slot, const ServeSlot& p, std::vector<ServeSlot>* dead) {
  if (!p.scene && !p.grid) return;
  ServeSlot& sp = s->spares[slot];
  if (!sp.scene && !sp.grid) {
    sp.scene = p.scene;
    sp.grid = p.grid;
  } else {
    dead->push_back(p);
  }
}

// Every spare, to be freed (caller holds s->mu): an allocation that the HBM
// budget or the device refused is retried once without them.
std::vector<ServeSlot> take_all_spares(shn_server* s) {
  std::vector<ServeSlot> out;
  for (ServeSlot& sp : s->spares)
    if (sp.scene || sp.grid) {
      out.push_back(sp);
      sp = ServeSlot{};
    }
  return out;
}

// build_slot with the slot's spare, retried once from scratch after freeing
// every spare when the budget or the device refused memory.
shn_status build_slot_retry(shn_server* s, uint32_t slot, ServeSlot spare, const float* vtx, uint32_t nv,
                            const uint32_t* idx, uint32_t nt, float lambda, cudaStream_t st, ServeSlot* out) {
  shn_status rc = build_slot(s, spare, vtx, nv, idx, nt, lambda, st, out);
  if (rc != SHN_ERR_BUDGET && rc != SHN_ERR_OOM) return rc;
  std::vector<ServeSlot> all;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    all = take_all_spares(s);
  }
  if (all.empty()) return rc;
  for (const ServeSlot& p : all) free_pair(p);
  return build_slot(s, ServeSlot{}, vtx, nv, idx, nt, lambda, st, out);
}

// Replaces the slot's pair immediately (no launch may be using it); the old
// pair becomes the slot's spare.  Caller holds s->mu.
shn_status load_slot(shn_server* s, uint32_t slot, const float* vtx, uint32_t nv, const uint32_t* idx,
                     uint32_t nt, float lambda, cudaStream_t st) {
  ServeSlot fresh;
  const ServeSlot spare = take_spare(s, slot);
  shn_status rc = build_slot(s, spare, vtx, nv, idx, nt, lambda, st, &fresh);
  if (rc == SHN_ERR_BUDGET || rc == SHN_ERR_OOM) {
    std::vector<ServeSlot> all = take_all_spares(s);
    if (!all.empty()) {
      for (const ServeSlot& p : all) free_pair(p);
      rc = build_slot(s, ServeSlot{}, vtx, nv, idx, nt, lambda, st, &fresh);
    }
  }
  if (rc) return rc;
  ServeSlot old = s->slots[slot];
  s->slots[slot].scene = fresh.scene;
  s->slots[slot].grid = fresh.grid;
  std::vector<ServeSlot> dead;
  release_pair(s, slot, ServeSlot{old.scene, old.grid, 0}, &dead);
  for (const ServeSlot& p : dead) free_pair(p);
  return SHN_OK;
}

// Releases the retired pairs whose launches have all completed (caller
// holds s->mu): spares where the slot has none, the rest returned to be
// freed after unlocking.
std::vector<ServeSlot> take_retired(shn_server* s) {
  std::vector<ServeSlot> out;
  size_t w = 0;
  for (size_t i = 0; i < s->retired.size(); ++i) {
    if (s->retired[i].after_seq <= s->done_seq) release_pair(s, s->retired[i].slot, s->retired[i].pair, &out);
    else s->retired[w++] = s->retired[i];
  }
  s->retired.resize(w);
  return out;
}

// Continuous-batching mode: scene replacements run here, off the launch
// path.  The new pair is built while launches continue; it replaces the old
// one at once for every request of that slot behind the update, and the old
// pair is retired until the launches that captured it have completed.
void updater_main(shn_server* s, int index) {
  cudaSetDevice(s->ctx->device);
  const cudaStream_t ust = s->upd_streams[index];
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_upd.wait(lk, [&] { return s->stop_upd || !s->upd_q.empty(); });
    if (s->upd_q.empty()) {
      if (s->stop_upd) break;
      continue;
    }
    ServeReq* r = s->upd_q.front();
    s->upd_q.pop_front();
    const shn_request q = r->r;
    const ServeSlot spare = take_spare(s, q.scene);
    lk.unlock();
    ServeSlot fresh;
    const shn_status rc = build_slot_retry(s, q.scene, spare, q.vtx, q.nv, q.idx, q.nt, q.lambda, ust, &fresh);
    lk.lock();
    ServeSlot& sl = s->slots[q.scene];
    if (rc == SHN_OK) {
      ServeRetired old;
      old.pair.scene = sl.scene;
      old.pair.grid = sl.grid;
      old.slot = q.scene;
      old.after_seq = s->launch_seq;
      s->retired.push_back(old);
      sl.scene = fresh.scene;
      sl.grid = fresh.grid;
    }
    sl.pending--;
    s->upd_outstanding--;
    s->updates_done++;
    complete(s, r, rc);
    s->work_gen++;
    s->cv_work.notify_all();
    std::vector<ServeSlot> dead = take_retired(s);
    lk.unlock();
    for (const ServeSlot& p : dead) free_pair(p);
    lk.lock();
  }
}

// Issues one launch for the requests in la (segment table, ray uploads, the
// trace, result read-backs, completion event).  Caller holds the lock; it
// is released while the copies and the launch are enqueued.
void issue_launch(shn_server* s, ServeLaunch& la, int slot_index, std::unique_lock<std::mutex>& lk) {
  for (size_t k = 0; k < la.reqs.size(); ++k) {
    const ServeReq* r = la.reqs[k];
    const shn_grid* g = s->slots[r->r.scene].grid;
    ServeSeg& sg = la.h_segs[k];
    sg.ray_begin = la.begin[k];
    sg.anyhit = r->r.kind == SHN_REQ_ANY ? 1u : 0u;
    sg.g.g = g->geom;
    sg.g.kind = g->kind;
    sg.g.cells = g->cells;
    sg.g.leaves = g->leaves;
    sg.g.rv0 = g->rtri;
    sg.g.rv1 = g->rtri + g->num_refs;
    sg.g.rv2 = g->rtri + 2 * g->num_refs;
    sg.g.src = g->src_tri;
    sg.g.cbox = g->num_blocks ? (const float4*)g->cbox.ptr : nullptr;
    sg.g.sbox = g->num_blocks ? (const float4*)g->sbox.ptr : nullptr;
    sg.g.ridx = nullptr;
  }
  s->max_requests_per_launch = std::max<uint64_t>(s->max_requests_per_launch, la.reqs.size());
  la.busy = true;
  la.seq = ++s->launch_seq;
  const uint32_t nseg = (uint32_t)la.reqs.size();
  const uint32_t total = la.nrays;
  lk.unlock();
  cudaMemcpyAsync(la.d_segs, la.h_segs, sizeof(ServeSeg) * nseg, cudaMemcpyHostToDevice, la.st);
  for (size_t k = 0; k < la.reqs.size(); ++k) {
    const shn_request& q = la.reqs[k]->r;
    cudaMemcpyAsync(la.d_rays + 2 * (size_t)la.begin[k], q.rays, 32 * (size_t)q.num_rays,
                    cudaMemcpyHostToDevice, la.st);
  }
  cudaMemsetAsync(la.d_counter, 0, 4, la.st);
  k_serve_trace<<<s->blocks, kServeBlock, 0, la.st>>>(la.d_segs, nseg, la.d_rays, total, la.d_counter,
                                                      la.d_tri, la.d_t);
  for (size_t k = 0; k < la.reqs.size(); ++k) {
    const shn_request& q = la.reqs[k]->r;
    if (q.out_tri)
      cudaMemcpyAsync(q.out_tri, la.d_tri + la.begin[k], 4 * (size_t)q.num_rays, cudaMemcpyDeviceToHost, la.st);
    if (q.out_t)
      cudaMemcpyAsync(q.out_t, la.d_t + la.begin[k], 4 * (size_t)q.num_rays, cudaMemcpyDeviceToHost, la.st);
  }
  cudaEventRecord(la.ev_done, la.st);
  lk.lock();
  s->launches++;
  s->inflight.push_back(slot_index);
  s->cv_done.notify_all();
}

// Plain path: requests one at a time in arrival order, one launch each,
// nothing overlaps; an update waits for the launch before it and runs inline.
void worker_plain(shn_server* s, std::unique_lock<std::mutex>& lk) {
  while (true) {
    s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
    if (s->queue.empty() && s->stop) break;
    ServeReq* head = s->queue.front();
    s->queue.pop_front();
    if (head->r.scene >= s->slots.size()) {
      complete(s, head, SHN_ERR_INVALID);
      continue;
    }
    if (head->r.kind == SHN_REQ_UPDATE) {
      const shn_request& q = head->r;
      const ServeSlot spare = take_spare(s, q.scene);
      lk.unlock();
      ServeSlot fresh;
      const shn_status rc =
          build_slot_retry(s, q.scene, spare, q.vtx, q.nv, q.idx, q.nt, q.lambda, s->update_st, &fresh);
      lk.lock();
      if (rc == SHN_OK) {
        ServeSlot& sl = s->slots[q.scene];
        const ServeSlot old{sl.scene, sl.grid, 0};
        sl.scene = fresh.scene;
        sl.grid = fresh.grid;
        std::vector<ServeSlot> dead;
        release_pair(s, q.scene, old, &dead);
        if (!dead.empty()) {
          lk.unlock();
          for (const ServeSlot& p : dead) free_pair(p);
          lk.lock();
        }
      }
      s->updates_done++;
      complete(s, head, rc);
      continue;
    }
    if (!s->slots[head->r.scene].grid) {
      complete(s, head, SHN_ERR_INVALID);
      continue;
    }
    ServeLaunch& la = s->L[0];
    la.reqs.assign(1, head);
    la.begin.assign(1, 0u);
    la.nrays = head->r.num_rays;
    issue_launch(s, la, 0, lk);
    s->cv_launch.wait(lk, [&] { return s->inflight.empty(); });
  }
}

// Continuous batching: every pass packs the queued requests that may run now
// into the next free launch slot (up to max_batch_rays / max_requests_per_launch),
// across scenes, in arrival order.  Requests of a slot with an update in
// progress wait for it (and keep their order); an update is handed to the
// updater only once every earlier request of its slot has been packed, and
// after the launch holding them captured the slot's current grid.
void worker_coalesced(shn_server* s, std::unique_lock<std::mutex>& lk) {
  int next_slot = 0;
  uint64_t idle_gen = ~0ull;
  std::vector<uint32_t> touched;
  std::vector<ServeReq*> dispatch;
  while (true) {
    s->cv_work.wait(lk, [&] {
      return (s->stop && s->queue.empty()) || (!s->queue.empty() && s->work_gen != idle_gen);
    });
    if (s->queue.empty()) break;  // stop requested and nothing left
    const uint64_t gen = s->work_gen;
    s->cv_launch.wait(lk, [&] { return !s->L[next_slot].busy; });
    ServeLaunch& la = s->L[next_slot];
    la.reqs.clear();
    la.begin.clear();
    dispatch.clear();
    touched.clear();
    uint32_t total = 0;
    for (auto it = s->queue.begin(); it != s->queue.end();) {
      ServeReq* r = *it;
      const uint32_t k = r->r.scene;
      if (k >= s->slots.size()) {
        complete(s, r, SHN_ERR_INVALID);
        it = s->queue.erase(it);
        continue;
      }
      if (r->r.kind == SHN_REQ_UPDATE) {
        const bool go = !s->blocked[k] && s->slots[k].pending == 0;
        if (!s->blocked[k]) {
          s->blocked[k] = 1;
          touched.push_back(k);
        }
        if (go) {
          s->slots[k].pending++;
          s->upd_outstanding++;
          dispatch.push_back(r);
          it = s->queue.erase(it);
        } else {
          ++it;
        }
        continue;
      }
      if (s->blocked[k] || s->slots[k].pending) {
        if (!s->blocked[k]) {
          s->blocked[k] = 1;
          touched.push_back(k);
        }
        ++it;
        continue;
      }
      if (!s->slots[k].grid) {
        complete(s, r, SHN_ERR_INVALID);
        it = s->queue.erase(it);
        continue;
      }
      if (!la.reqs.empty() && (total + r->r.num_rays > s->cfg.max_batch_rays ||
                               la.reqs.size() >= s->cfg.max_requests_per_launch))
        break;
      la.begin.push_back(total);
      la.reqs.push_back(r);
      total += r->r.num_rays;
      it = s->queue.erase(it);
    }
    for (uint32_t k : touched) s->blocked[k] = 0;
    if (!la.reqs.empty()) {
      la.nrays = total;
      issue_launch(s, la, next_slot, lk);
      next_slot = (next_slot + 1) % kLaunchSlots;
    }
    if (!dispatch.empty()) {
      for (ServeReq* r : dispatch) s->upd_q.push_back(r);
      s->cv_upd.notify_all();
    }
    if (la.reqs.empty() && dispatch.empty()) idle_gen = gen;  // nothing can run until something changes
  }
}

void worker_main(shn_server* s) {
  cudaSetDevice(s->ctx->device);
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->cfg.coalesce) worker_coalesced(s, lk);
  else worker_plain(s, lk);
}

void completer_main(shn_server* s) {
  cudaSetDevice(s->ctx->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_done.wait(lk, [&] { return !s->inflight.empty() || (s->stop && s->queue.empty() && s->inflight.empty()); });
    if (s->inflight.empty()) {
      if (s->stop && s->queue.empty()) break;
      continue;
    }
    const int li = s->inflight.front();
    ServeLaunch& la = s->L[li];
    lk.unlock();
    const cudaError_t e = cudaEventSynchronize(la.ev_done);
    lk.lock();
    const shn_status st = e == cudaSuccess ? SHN_OK : SHN_ERR_CUDA;
    for (ServeReq* r : la.reqs) complete(s, r, st);
    la.reqs.clear();
    la.busy = false;
    s->done_seq = la.seq;
    s->inflight.pop_front();
    s->cv_launch.notify_all();
    s->cv_work.notify_all();
    std::vector<ServeSlot> dead = take_retired(s);
    if (!dead.empty()) {
      lk.unlock();
      for (const ServeSlot& p : dead) free_pair(p);
      lk.lock();
    }
  }
}

}  // namespace

extern "C" {

void shn_server_config_default(shn_server_config* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->num_slots = 64;
  c->max_batch_rays = 4u << 20;
  c->max_requests_per_launch = 4096;
  c->coalesce = 1;
}

shn_status shn_server_create(shn_ctx* ctx, const shn_server_config* cfg, shn_server** out) {
  if (!ctx || !cfg || !out || cfg->num_slots == 0 || cfg->max_batch_rays == 0 || cfg->max_requests_per_launch == 0)
    return SHN_ERR_INVALID;
  *out = nullptr;
  shn_server* s = new shn_server();
  s->ctx = ctx;
  ctx_retain(ctx);
  s->cfg = *cfg;
  s->slots.resize(cfg->num_slots);
  s->blocked.assign(cfg->num_slots, 0);
  s->spares.resize(cfg->num_slots);
  cudaStreamCreateWithFlags(&s->update_st, cudaStreamNonBlocking);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_serve_trace, kServeBlock, 0);
  s->blocks = std::max(1, per_sm) * ctx->num_sms;
  const size_t cap = cfg->max_batch_rays;
  for (int i = 0; i < kLaunchSlots; ++i) {
    ServeLaunch& la = s->L[i];
    cudaStreamCreateWithFlags(&la.st, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&la.ev_done, cudaEventDisableTiming);
    cudaError_t e = dev_alloc(ctx, (void**)&la.d_rays, 32 * cap, la.st);
    if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&la.d_tri, 4 * cap, la.st);
    if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&la.d_t, 4 * cap, la.st);
    if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&la.d_segs, sizeof(ServeSeg) * cfg->max_requests_per_launch, la.st);
    if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&la.d_counter, 64, la.st);
    if (e == cudaSuccess) e = cudaMallocHost(&la.h_segs, sizeof(ServeSeg) * cfg->max_requests_per_launch);
    if (e != cudaSuccess) {
      shn_server_destroy(s);
      return set_error(ctx, e == cudaErrorNotPermitted ? SHN_ERR_BUDGET : SHN_ERR_OOM, "server staging");
    }
  }
  s->worker = std::thread(worker_main, s);
  s->completer = std::thread(completer_main, s);
  for (int i = 0; i < kUpdaters; ++i) {
    cudaStream_t us = nullptr;
    cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking);
    s->upd_streams.push_back(us);
  }
  for (int i = 0; i < kUpdaters; ++i) s->updaters.emplace_back(updater_main, s, i);
  *out = s;
  return SHN_OK;
}

shn_status shn_server_load_scene(shn_server* s, uint32_t slot, const float* vtx_xyz, uint32_t nv,
                                 const uint32_t* idx, uint32_t nt, float lambda) {
  if (!s || slot >= s->slots.size()) return SHN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->inflight.empty() || !s->queue.empty())
    return set_error(s->ctx, SHN_ERR_BUSY, "load_scene while requests are pending; submit an update request");
  return load_slot(s, slot, vtx_xyz, nv, idx, nt, lambda, s->update_st);
}

shn_status shn_server_submit(shn_server* s, const shn_request* r, uint64_t* ticket) {
  if (!s || !r || !ticket) return SHN_ERR_INVALID;
  if (r->kind > SHN_REQ_UPDATE) return SHN_ERR_INVALID;
  if (r->kind != SHN_REQ_UPDATE) {
    if (r->num_rays == 0 || !r->rays || r->num_rays > s->cfg.max_batch_rays)
      return set_error(s->ctx, SHN_ERR_INVALID, "request rays empty or above max_batch_rays");
  }
  ServeReq* q = new ServeReq();
  q->r = *r;
  q->t_submit = now_s();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    delete q;
    return SHN_ERR_CANCELLED;
  }
  if (s->cfg.max_queue && s->queue.size() >= s->cfg.max_queue) {
    delete q;
    return SHN_ERR_BUSY;
  }
  q->ticket = s->next_ticket++;
  if (s->t_first == 0.0) s->t_first = q->t_submit;
  s->reqs[q->ticket] = q;
  s->queue.push_back(q);
  s->work_gen++;
  *ticket = q->ticket;
  s->cv_work.notify_one();
  return SHN_OK;
}

shn_status shn_server_wait(shn_server* s, uint64_t ticket, uint32_t timeout_ms, shn_status* result) {
  if (!s) return SHN_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return SHN_ERR_INVALID;
  ServeReq* q = it->second;
  const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return q->done; });
  if (!ok) return SHN_ERR_BUSY;
  if (result) *result = q->result;
  s->reqs.erase(it);
  delete q;
  return SHN_OK;
}

shn_status shn_server_poll(shn_server* s, uint64_t ticket, shn_status* result) {
  return shn_server_wait(s, ticket, 0, result);
}

shn_status shn_server_drain(shn_server* s, uint32_t timeout_ms) {
  if (!s) return SHN_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                      [&] { return s->queue.empty() && s->inflight.empty() && s->upd_outstanding == 0; });
  return ok ? SHN_OK : SHN_ERR_BUSY;
}

shn_status shn_server_get_stats(shn_server* s, shn_server_stats* out, int reset) {
  if (!s || !out) return SHN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof(*out));
  out->requests = s->requests_done;
  out->updates = s->updates_done;
  out->rays = s->rays_done;
  out->launches = s->launches;
  out->max_requests_per_launch = s->max_requests_per_launch;
  std::vector<double> v = s->lat_us;
  std::sort(v.begin(), v.end());
  if (!v.empty()) {
    out->p50_us = v[(size_t)(0.50 * (v.size() - 1))];
    out->p99_us = v[(size_t)(0.99 * (v.size() - 1))];
    out->max_us = v.back();
    double sum = 0;
    for (double x : v) sum += x;
    out->mean_us = sum / v.size();
  }
  out->wall_s = s->t_last > s->t_first ? s->t_last - s->t_first : 0.0;
  out->mrays_per_s = out->wall_s > 0 ? s->rays_done / out->wall_s / 1e6 : 0.0;
  if (reset) {
    s->lat_us.clear();
    s->records.clear();
    s->rays_done = s->launches = s->requests_done = s->updates_done = 0;
    s->t_first = s->t_last = 0.0;
    s->max_requests_per_launch = 0;
  }
  return SHN_OK;
}

shn_status shn_server_get_records(shn_server* s, uint32_t max_records, shn_request_record* out,
                                  uint32_t* count) {
  if (!s || !count || (max_records && !out)) return SHN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  const uint32_t n = (uint32_t)std::min<size_t>(max_records, s->records.size());
  if (n) memcpy(out, s->records.data(), n * sizeof(shn_request_record));
  *count = (uint32_t)s->records.size();
  return SHN_OK;
}

shn_status shn_server_run_schedule(shn_server* s, uint32_t n, const shn_request* reqs,
                                   const double* arrival_s, shn_status* results) {
  if (!s || (n && (!reqs || !arrival_s))) return SHN_ERR_INVALID;
  std::vector<uint64_t> tickets(n, 0);
  std::vector<shn_status> sub(n, SHN_OK);
  const double t0 = now_s();
  for (uint32_t i = 0; i < n; ++i) {
    const double due = t0 + arrival_s[i];
    while (true) {
      const double t = now_s();
      if (t >= due) break;
      if (due - t > 2e-4) std::this_thread::sleep_for(std::chrono::microseconds((long)((due - t - 1e-4) * 1e6)));
    }
    sub[i] = shn_server_submit(s, &reqs[i], &tickets[i]);
  }
  shn_status rc = SHN_OK;
  for (uint32_t i = 0; i < n; ++i) {
    shn_status r = sub[i];
    if (r == SHN_OK) {
      shn_status w = shn_server_wait(s, tickets[i], 600000, &r);
      if (w != SHN_OK) r = w;
    }
    if (results) results[i] = r;
    if (r != SHN_OK && rc == SHN_OK) rc = r;
  }
  return rc;
}

void shn_server_destroy(shn_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  s->cv_launch.notify_all();
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop_upd = true;
  }
  s->cv_upd.notify_all();
  for (std::thread& t : s->updaters)
    if (t.joinable()) t.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->cv_done.notify_all();
  }
  if (s->completer.joinable()) s->completer.join();
  cudaDeviceSynchronize();
  for (auto& kv : s->reqs) delete kv.second;
  for (auto& r : s->retired) free_pair(r.pair);
  for (auto& sl : s->slots) free_pair(sl);
  for (auto& sl : s->spares) free_pair(sl);
  for (int i = 0; i < kLaunchSlots; ++i) {
    ServeLaunch& la = s->L[i];
    dev_free(s->ctx, la.d_rays, 32 * (size_t)s->cfg.max_batch_rays, la.st);
    dev_free(s->ctx, la.d_tri, 4 * (size_t)s->cfg.max_batch_rays, la.st);
    dev_free(s->ctx, la.d_t, 4 * (size_t)s->cfg.max_batch_rays, la.st);
    dev_free(s->ctx, la.d_segs, sizeof(ServeSeg) * s->cfg.max_requests_per_launch, la.st);
    dev_free(s->ctx, la.d_counter, 64, la.st);
    if (la.h_segs) cudaFreeHost(la.h_segs);
    if (la.ev_done) cudaEventDestroy(la.ev_done);
    if (la.st) {
      cudaStreamSynchronize(la.st);
      cudaStreamDestroy(la.st);
    }
  }
  if (s->update_st) cudaStreamDestroy(s->update_st);
  for (cudaStream_t us : s->upd_streams) cudaStreamDestroy(us);
  shn_ctx* c = s->ctx;
  delete s;
  ctx_release(c);
}

}  // extern "C"
