// capi_server.cu — serving: continuous batching of scenes under an HBM budget.
//
// Requests (scenes with a lifetime in ticks) queue in FIFO order. Each tick
// the server
//  1. swaps in a cohort whose build finished: the cohort's world was built
//     from the requests' specs on a host worker thread while earlier ticks
//     ran; scenes folded in from older cohorts get their current state by a
//     device-to-device import (World::import_scene), so state never leaves
//     HBM between admission and retirement;
//  2. admits the longest FIFO prefix of the queue that fits the budget (the
//     admission estimate is the scene's own planned world size) and starts
//     that cohort's build, folding the smallest cohort into it when there
//     are already max_cohorts, and any cohort that is more than half retired;
//  3. steps every cohort once (each cohort is one world on its own stream,
//     one CUDA graph per tick), the cohorts' work overlapping on the GPU;
//  4. retires the scenes whose lifetime is over: their final state is read
//     back once, their slots stop being stepped; a cohort with no live
//     scene is freed and its bytes return to the budget.
// Scenes are independent and every stage is per-scene deterministic, so a
// scene's result is the same alone and inside any cohort.
//
// PLAIN mode gives each request its own world (no graph, no folding) and
// steps the scenes one after another, waiting for each (the reference's
// `await simulation.step()` per scene): the per-scene loop the batched mode
// is measured against, on the same stream of requests and admission rule.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <deque>
#include <future>
#include <memory>
#include <string>
#include <vector>

#include "capi_handles.cuh"
#include "common.cuh"
#include "world.cuh"

using namespace pf;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  // Read by cohort builds on the worker thread; after submission the main
  // thread writes it only through a world's first step (never concurrently
  // with a build that holds it: folded scenes have stepped before).
  std::unique_ptr<SceneSpec> spec;
  std::unique_ptr<SceneSpec> result;  // final state, once retired
  uint32_t lifetime = 0, done = 0;
  uint64_t est_bytes = 0;
  uint64_t ps_per_step = 0;  // particles x substeps
  uint32_t state = PF_REQ_QUEUED;
  struct Cohort* cohort = nullptr;
  uint32_t index = 0;
};

struct Cohort {
  std::unique_ptr<World> world;
  std::vector<Request*> members;
  uint32_t live = 0;
  uint64_t bytes = 0;
  uint64_t live_particles = 0;
  bool folding = false;  // its live members move into the build in flight
};

struct Build {
  std::unique_ptr<Cohort> cohort;
  std::vector<Request*> members;  // in world order: folded members first, then fresh ones
  std::vector<Cohort*> folded;
  uint64_t reserved = 0;
  std::future<std::pair<pf_status, std::string>> result;
};

double ms_since(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }

}  // namespace

struct pf_server {
  pf_server_opts opts{};
  int device = 0;
  std::vector<std::unique_ptr<Request>> reqs;  // ticket - 1
  std::deque<Request*> queue;
  std::vector<std::unique_ptr<Cohort>> cohorts;
  std::unique_ptr<Build> build;
  uint64_t used = 0;  // bytes of cohorts + the reservation of the build in flight
  uint64_t ticks = 0, particle_substeps = 0, rebuilds = 0;
  uint32_t finished = 0;
  double busy_ms = 0;
  std::vector<float> tick_ms;
  float max_swap_ms = 0, max_admit_ms = 0;
  float max_step_ms = 0, max_free_ms = 0;
  float last_admit_ms = 0;  // admission (and synchronous builds) inside the last tick
  bool blocked = false;  // the last build ran out of memory: wait for a cohort to free
  std::string last_error;
  bool have_tuning = false;  // the first cohort's autotuned neighbour path, reused by later cohorts
  World::Tuning tuning{};

  ~pf_server() {
    if (build && build->result.valid()) build->result.wait();
  }
};

namespace {

uint32_t live_count(const pf_server* s) {
  uint32_t n = 0;
  for (auto& c : s->cohorts) n += c->live;
  return n;
}

pf_status plan_bytes(SceneSpec* spec, uint64_t* bytes) {
  World w;
  PF_TRY(w.build({spec}, false, true));
  *bytes = w.device_bytes();
  return PF_OK;
}

// Swap a finished build in: import the folded members' current state, then
// retire the folded cohorts.
pf_status swap_in(pf_server* S) {
  Build& B = *S->build;
  auto [st, err] = B.result.get();
  if (st != PF_OK) {
    // back to the queue head in their original order; folded cohorts go on
    for (auto it = B.members.rbegin(); it != B.members.rend(); ++it) {
      Request* r = *it;
      if (r->state == PF_REQ_BUILDING) {
        r->state = PF_REQ_QUEUED;
        S->queue.push_front(r);
      }
    }
    for (Cohort* f : B.folded) f->folding = false;
    S->used -= B.reserved;
    S->build.reset();
    S->last_error = err;
    if (st == PF_ERR_OOM && !S->cohorts.empty()) {
      S->blocked = true;  // retried once a live cohort retires and frees its memory
      return PF_OK;
    }
    return fail(st, "server: cohort build failed: " + err);
  }
  Cohort& C = *B.cohort;
  World& W = *C.world;
  if (S->have_tuning) W.set_tuning(S->tuning);
  for (uint32_t j = 0; j < B.members.size(); ++j) {
    Request* r = B.members[j];
    if (r->state == PF_REQ_LIVE) {
      // folded: bring its current state over, device to device
      PF_CUDA(cudaStreamSynchronize(r->cohort->world->stream()));
      PF_TRY(W.import_scene(j, *r->cohort->world, r->index));
    }
  }
  PF_CUDA(cudaStreamSynchronize(W.stream()));
  for (uint32_t j = 0; j < B.members.size(); ++j) {
    Request* r = B.members[j];
    if (r->state == PF_REQ_DONE) {
      W.retire(j);  // finished in its old cohort while this one was built
      continue;
    }
    if (r->state == PF_REQ_LIVE) {
      r->cohort->live--;
      r->cohort->live_particles -= r->spec->cap;
    }
    r->state = PF_REQ_LIVE;
    r->cohort = &C;
    r->index = j;
    C.live++;
    C.live_particles += r->spec->cap;
  }
  C.members = B.members;
  S->used -= B.reserved;
  S->used += C.bytes;
  for (Cohort* f : B.folded) f->folding = false;
  S->cohorts.push_back(std::move(B.cohort));
  S->build.reset();
  S->rebuilds++;
  // folded cohorts now have no live member
  for (size_t i = 0; i < S->cohorts.size();) {
    if (S->cohorts[i]->live == 0) {
      S->used -= S->cohorts[i]->bytes;
      S->cohorts.erase(S->cohorts.begin() + i);
      S->blocked = false;
    } else {
      ++i;
    }
  }
  return PF_OK;
}

pf_status start_build(pf_server* S, std::vector<Request*> fresh, std::vector<Cohort*> folded, uint64_t reserve) {
  auto B = std::make_unique<Build>();
  for (Cohort* f : folded) {
    f->folding = true;
    for (Request* r : f->members)
      if (r->state == PF_REQ_LIVE) B->members.push_back(r);
  }
  for (Request* r : fresh) {
    r->state = PF_REQ_BUILDING;
    B->members.push_back(r);
  }
  B->folded = std::move(folded);
  B->reserved = reserve;
  B->cohort = std::make_unique<Cohort>();
  B->cohort->world = std::make_unique<World>();
  S->used += reserve;
  std::vector<SceneSpec*> specs;
  std::vector<uint8_t> imported;  // folded scenes get their state by import at the swap
  for (Request* r : B->members) {
    specs.push_back(r->spec.get());
    imported.push_back(r->state == PF_REQ_LIVE ? 1 : 0);
  }
  World* W = B->cohort->world.get();
  Cohort* C = B->cohort.get();
  const bool graph = S->opts.mode == PF_SERVER_BATCHED && S->opts.use_graph;
  const int dev = S->device;
  auto job = [W, C, specs, imported, graph, dev]() -> std::pair<pf_status, std::string> {
    cudaSetDevice(dev);
    const pf_status st = W->build(specs, graph, false, &imported);
    if (st != PF_OK) return {st, get_error()};
    C->bytes = W->device_bytes();
    return {PF_OK, std::string()};
  };
  if (S->opts.async_build) {
    B->result = std::async(std::launch::async, job);
  } else {
    std::promise<std::pair<pf_status, std::string>> p;
    p.set_value(job());
    B->result = p.get_future();
  }
  S->build = std::move(B);
  return PF_OK;
}

// Admit the FIFO prefix that fits; in PLAIN mode each request is a cohort of
// its own (built one after another, synchronously like a caller building
// its Simulation).
pf_status admit(pf_server* S) {
  if (S->build || S->queue.empty() || S->blocked) return PF_OK;
  const uint64_t budget = S->opts.hbm_budget_bytes;
  uint32_t slots = S->opts.max_scenes > live_count(S) ? S->opts.max_scenes - live_count(S) : 0;
  if (S->opts.mode == PF_SERVER_PLAIN) {
    while (!S->queue.empty() && slots > 0) {
      Request* r = S->queue.front();
      if (S->used + r->est_bytes > budget) break;
      S->queue.pop_front();
      PF_TRY(start_build(S, {r}, {}, r->est_bytes));
      PF_TRY(swap_in(S));
      --slots;
      if (S->blocked) break;
    }
    return PF_OK;
  }
  // folds: cohorts more than half retired, and the smallest when at the cap
  std::vector<Cohort*> folded;
  uint64_t fold_bytes = 0;
  for (auto& c : S->cohorts) {
    if (c->folding) continue;
    const uint64_t cap_particles = [&] {
      uint64_t t = 0;
      for (Request* r : c->members) t += r->spec->cap;
      return t;
    }();
    if (c->live_particles * 2 < cap_particles) folded.push_back(c.get());
  }
  const uint32_t max_cohorts = std::max<uint32_t>(1, S->opts.max_cohorts);
  while (S->cohorts.size() + 1 - folded.size() > max_cohorts) {
    Cohort* best = nullptr;
    for (auto& c : S->cohorts)
      if (std::find(folded.begin(), folded.end(), c.get()) == folded.end() &&
          (!best || c->live_particles < best->live_particles))
        best = c.get();
    if (!best) break;
    folded.push_back(best);
  }
  for (Cohort* f : folded)
    for (Request* r : f->members)
      if (r->state == PF_REQ_LIVE) fold_bytes += r->est_bytes;
  std::vector<Request*> fresh;
  uint64_t add = fold_bytes;
  while (!S->queue.empty() && slots > 0) {
    Request* r = S->queue.front();
    if (S->used + add + r->est_bytes > budget) break;
    add += r->est_bytes;
    fresh.push_back(r);
    S->queue.pop_front();
    --slots;
  }
  if (fresh.empty()) return PF_OK;
  return start_build(S, std::move(fresh), std::move(folded), add);
}

bool build_ready(const pf_server* S) {
  return S->build && S->build->result.wait_for(std::chrono::seconds(0)) == std::future_status::ready;
}

}  // namespace

extern "C" {

pf_status pf_server_create(const pf_server_opts* opts, pf_server** out) {
  if (!out) return fail(PF_ERR_INVALID, "server: out is NULL");
  auto s = std::make_unique<pf_server>();
  if (opts) s->opts = *opts;
  if (!s->opts.hbm_budget_bytes) s->opts.hbm_budget_bytes = 150ull * 1000 * 1000 * 1000;
  if (!s->opts.max_scenes) s->opts.max_scenes = 65536;
  if (!s->opts.max_cohorts) s->opts.max_cohorts = 4;
  if (s->opts.mode != PF_SERVER_BATCHED && s->opts.mode != PF_SERVER_PLAIN)
    return fail(PF_ERR_INVALID, "server: unknown mode " + std::to_string(s->opts.mode));
  PF_CUDA(cudaGetDevice(&s->device));
  *out = s.release();
  return PF_OK;
}

void pf_server_destroy(pf_server* s) { delete s; }

pf_status pf_server_estimate_bytes(pf_scene* scene, const pf_loop_desc* loop, uint64_t* bytes) {
  if (!scene || !bytes) return fail(PF_ERR_INVALID, "server: NULL argument");
  SceneSpec spec = scene->spec;
  if (loop) spec.loop = *loop;
  else if (!scene->world) return fail(PF_ERR_STATE, "server: scene has no SimLoop and no loop options were given");
  return plan_bytes(&spec, bytes);
}

pf_status pf_server_submit(pf_server* S, pf_scene* scene, const pf_loop_desc* loop, uint32_t lifetime,
                           uint64_t* ticket) {
  if (!S || !scene) return fail(PF_ERR_INVALID, "server: NULL argument");
  if (lifetime == 0) return fail(PF_ERR_INVALID, "server: lifetime must be at least one step");
  auto r = std::make_unique<Request>();
  r->spec = std::make_unique<SceneSpec>(scene->spec);
  if (scene->world) {
    PF_TRY(scene->world->pull_state(0, r->spec.get()));
  } else if (!loop) {
    return fail(PF_ERR_STATE, "server: scene has no SimLoop and no loop options were given");
  }
  if (loop) {
    if (loop->substeps < 1) return fail(PF_ERR_INVALID, "SimLoop: substeps must be an integer >= 1, got 0");
    r->spec->loop = *loop;
  }
  if (!scene->world) PF_TRY(allocate_collision_groups(*r->spec));
  r->spec->built = true;
  PF_TRY(plan_bytes(r->spec.get(), &r->est_bytes));
  if (r->est_bytes > S->opts.hbm_budget_bytes)
    return fail(PF_ERR_BUDGET, "server: scene needs " + std::to_string(r->est_bytes) + " bytes, over the budget of " +
                                   std::to_string(S->opts.hbm_budget_bytes));
  r->lifetime = lifetime;
  r->ps_per_step = (uint64_t)r->spec->cap * r->spec->loop.substeps;
  r->ticket = S->reqs.size() + 1;
  S->queue.push_back(r.get());
  if (ticket) *ticket = r->ticket;
  S->reqs.push_back(std::move(r));
  return PF_OK;
}

pf_status pf_server_drain_build(pf_server* S) {
  if (!S) return fail(PF_ERR_INVALID, "server: NULL");
  if (S->build) {
    S->build->result.wait();
    PF_TRY(swap_in(S));
  }
  return PF_OK;
}

pf_status pf_server_tick(pf_server* S, double dt) {
  if (!S) return fail(PF_ERR_INVALID, "server: NULL");
  if (!(dt > 0)) return fail(PF_ERR_INVALID, "server: dt must be positive");
  const auto t0 = Clock::now();
  double swap_ms = 0;
  if (build_ready(S)) {
    PF_TRY(swap_in(S));
    swap_ms = ms_since(t0);
    S->max_swap_ms = std::max(S->max_swap_ms, (float)swap_ms);
  }
  S->last_admit_ms = 0;
  if (!S->opts.async_build || S->opts.mode == PF_SERVER_PLAIN) {
    const auto ta = Clock::now();
    PF_TRY(admit(S));
    if (S->build) PF_TRY(swap_in(S));
    S->last_admit_ms = (float)ms_since(ta);
    S->max_admit_ms = std::max(S->max_admit_ms, S->last_admit_ms);
  }
  bool stepped = false;
  const bool plain = S->opts.mode == PF_SERVER_PLAIN;
  const auto ts = Clock::now();
  std::vector<float> host_ms(S->cohorts.size(), 0.0f);  // per cohort, for the verbose log
  for (size_t ci = 0; ci < S->cohorts.size(); ++ci) {
    auto& c = S->cohorts[ci];
    if (c->live) {
      const auto th = Clock::now();
      PF_TRY(c->world->step(dt));
      host_ms[ci] = (float)ms_since(th);
      if (!S->have_tuning && c->world->tuned() && c->world->has_fluid()) {
        S->tuning = c->world->tuning_all();
        S->have_tuning = true;
      }
      // the per-scene loop steps one scene and waits for it
      if (plain) PF_CUDA(cudaStreamSynchronize(c->world->stream()));
      stepped = true;
    }
  }
  if (!plain)
    for (auto& c : S->cohorts)
      if (c->live) PF_CUDA(cudaStreamSynchronize(c->world->stream()));
  const double step_ms = ms_since(ts);
  S->max_step_ms = std::max(S->max_step_ms, (float)step_ms);
  if (verbose() && !plain)
    // each stepped cohort: its step call on the host and its step on the
    // device (the cohorts' steps overlap there); printed before this tick's
    // line
    for (size_t ci = 0; ci < S->cohorts.size(); ++ci) {
      float gpu = 0;
      if (host_ms[ci] > 0 && S->cohorts[ci]->world->elapsed_ms(&gpu) == PF_OK)
        std::fprintf(stderr, "pfsim:   cohort %zu: %u live, step call %.2f ms, device %.2f ms\n", ci,
                     S->cohorts[ci]->live, host_ms[ci], gpu);
    }
  const auto tr = Clock::now();
  bool freed = false;
  for (auto& c : S->cohorts) {
    for (uint32_t j = 0; j < c->members.size(); ++j) {
      Request* r = c->members[j];
      if (r->state != PF_REQ_LIVE || r->cohort != c.get()) continue;
      r->done++;
      S->particle_substeps += r->ps_per_step;
      if (r->done >= r->lifetime) {
        auto res = std::make_unique<SceneSpec>();
        res->cap = r->spec->cap;
        res->pos4.assign(4ull * res->cap, 0.0f);
        res->vel4.assign(4ull * res->cap, 0.0f);
        res->inv_mass.assign(res->cap, 0.0f);
        res->bvol.assign(res->cap, 0.0f);
        PF_TRY(c->world->pull_state(j, res.get()));
        r->result = std::move(res);
        c->world->retire(j);
        r->state = PF_REQ_DONE;
        c->live--;
        c->live_particles -= r->spec->cap;
        S->finished++;
      }
    }
  }
  const double retire_ms = ms_since(tr);
  const auto tf = Clock::now();
  for (size_t i = 0; i < S->cohorts.size();) {
    Cohort* c = S->cohorts[i].get();
    if (c->live == 0 && !c->folding) {
      S->used -= c->bytes;
      S->cohorts.erase(S->cohorts.begin() + i);
      freed = true;
    } else {
      ++i;
    }
  }
  if (freed) S->blocked = false;
  const double free_ms = ms_since(tf);
  S->max_free_ms = std::max(S->max_free_ms, (float)free_ms);
  // An asynchronous build starts after this tick's steps (and their first-step
  // graph captures), and runs on the worker thread while the next ticks go on.
  if (S->opts.async_build && S->opts.mode != PF_SERVER_PLAIN) {
    const auto ta = Clock::now();
    PF_TRY(admit(S));
    const float ms = (float)ms_since(ta);
    S->last_admit_ms += ms;
    S->max_admit_ms = std::max(S->max_admit_ms, ms);
  }
  S->ticks++;
  const double ms = ms_since(t0);
  if (stepped) {  // latency statistics cover ticks that stepped at least one scene
    S->busy_ms += ms;
    S->tick_ms.push_back((float)ms);
  }
  if (verbose()) {
    std::fprintf(stderr,
                 "pfsim: tick %llu %.2f ms: swap %.2f, admit %.2f, step %.2f, retire %.2f, free %.2f; %zu cohorts, "
                 "%u live\n",
                 (unsigned long long)S->ticks, ms, swap_ms, (double)S->last_admit_ms, step_ms, retire_ms, free_ms,
                 S->cohorts.size(), live_count(S));
  }
  return PF_OK;
}

pf_status pf_server_request_state(pf_server* S, uint64_t ticket, uint32_t* state, uint32_t* steps_done) {
  if (!S || ticket == 0 || ticket > S->reqs.size()) return fail(PF_ERR_INVALID, "server: no such ticket");
  const Request& r = *S->reqs[ticket - 1];
  if (state) *state = r.state;
  if (steps_done) *steps_done = r.done;
  return PF_OK;
}

pf_status pf_server_readback(pf_server* S, uint64_t ticket, uint32_t field, void* dst, size_t bytes) {
  if (!S || !dst || ticket == 0 || ticket > S->reqs.size()) return fail(PF_ERR_INVALID, "server: no such ticket");
  const Request& r = *S->reqs[ticket - 1];
  if (r.state == PF_REQ_DONE) return spec_readback(*r.result, field, dst, bytes);
  if (r.state == PF_REQ_LIVE) return r.cohort->world->readback(r.index, field, dst, bytes);
  return fail(PF_ERR_STATE, "server: request " + std::to_string(ticket) + " is not admitted yet");
}

pf_status pf_server_stats_read(pf_server* S, pf_server_stats* o) {
  if (!S || !o) return fail(PF_ERR_INVALID, "server: NULL");
  std::memset(o, 0, sizeof(*o));
  o->live = live_count(S);
  o->queued = (uint32_t)S->queue.size();
  if (S->build)
    for (Request* r : S->build->members) o->building += r->state == PF_REQ_BUILDING;
  o->finished = S->finished;
  o->cohorts = (uint32_t)S->cohorts.size();
  o->ticks = S->ticks;
  o->particle_substeps = S->particle_substeps;
  o->state_bytes = S->used;
  o->rebuilds = S->rebuilds;
  o->busy_ms = S->busy_ms;
  if (!S->tick_ms.empty()) {
    std::vector<float> t = S->tick_ms;
    std::sort(t.begin(), t.end());
    auto pct = [&](double p) { return t[std::min(t.size() - 1, (size_t)(p * (t.size() - 1) + 0.5))]; };
    o->last_tick_ms = S->tick_ms.back();
    o->p50_tick_ms = pct(0.50);
    o->p99_tick_ms = pct(0.99);
    o->max_tick_ms = t.back();
  }
  o->max_swap_ms = S->max_swap_ms;
  o->max_admit_ms = S->max_admit_ms;
  o->last_admit_ms = S->last_admit_ms;
  o->max_step_ms = S->max_step_ms;
  o->max_free_ms = S->max_free_ms;
  return PF_OK;
}

}  // extern "C"
