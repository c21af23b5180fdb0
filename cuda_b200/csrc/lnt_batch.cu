// Batch engine: many independent LL / PRP tests of mixed lengths on one GPU.
//
// The reference runs one exponent per process (main_process.cu:64-149 builds
// one MainProcess, lucas_prp.cu drives one residue).  Here tests are grouped
// by length and every group advances with batched launches: each kernel of
// the squaring takes a device array of test descriptors and blockIdx.y picks
// the test, so one launch per kernel covers all tests of a length.  The
// SMEM-resident plan (n <= 4096) runs all its tests, of any lengths, in one
// launch with one CTA per test and a per-test iteration count.  Groups run on
// their own streams so small groups overlap.  Tests are admitted against an
// HBM budget and retired (Res64 and verdict recorded, memory released) as they
// finish, so a caller can keep the engine full: continuous batching.
//
// Each group's launches of `kGraphChunk` squarings are captured once per group
// membership into a CUDA graph on the group's stream and replayed, so a batch
// step costs one graph launch per group and chunk instead of 3 x chunk kernel
// launches.  Without a time budget every group advances by the same count per
// call (lockstep); with one (lnt_batch_step_seconds) each group and resident
// test runs as many squarings as fit in it at its measured pace.  Optionally
// (lnt_batch_autotune) each length's plan (split, column tile, pass radix,
// column fusion) is picked by timing the candidates once per length -- alone or
// on a group of copies (lnt_batch_autotune_group) -- the analogue of the
// reference's per-run autotune (process.cu:45-127), and kept in a JSON cache
// (lnt_batch_plan_cache).  Res64 checkpoints every K squarings
// (lnt_batch_checkpoint_every) record each test's intermediate residues.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/lucasntt.h"
#include "lnt_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Entry {
  uint64_t id;
  lnt_test* t;
  uint32_t q, n;
  int prp;
  uint64_t target, done;
  uint64_t bytes;
  Clock::time_point submitted;
  uint64_t last_checkpoint = 0;  // squaring count of the last recorded checkpoint
};

struct Pending {
  uint64_t id;
  uint32_t q, n;
  int prp;
  uint64_t iterations;
  Clock::time_point enqueued;
};

// Tests share launches when their kernels see the same geometry: length,
// split, tile, pass radix (the pass tables differ) and column fusion.
struct GroupKey {
  uint32_t n, log2n2, tile, radix;
  bool fused;
  bool operator<(const GroupKey& o) const {
    if (n != o.n) return n < o.n;
    if (log2n2 != o.log2n2) return log2n2 < o.log2n2;
    if (tile != o.tile) return tile < o.tile;
    if (radix != o.radix) return radix < o.radix;
    return fused < o.fused;
  }
};

constexpr uint64_t kGraphChunk = 8;  // squarings per captured graph

struct Group {
  uint32_t n = 0;
  bool fused = false;  // the plan's steady squarings use the carry-fused column kernel
  std::vector<size_t> members;  // indices into active
  lnt::TwoPassDesc geometry{};
  lnt::TwoPassDesc* d_descs = nullptr;
  size_t cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t join = nullptr;  // recorded on `stream` after the group's launches
  cudaEvent_t t0 = nullptr, t1 = nullptr;  // around the group's squarings of a call
  cudaGraphExec_t graph = nullptr;  // kGraphChunk squarings, captured on `stream`
  uint64_t k = 0;                   // squarings of the current call
};

int berr(int status, const std::string& msg) {
  lnt::set_last_error(msg);
  return status;
}

}  // namespace

struct lnt_batch {
  int device = 0;
  uint64_t budget = 0, used = 0;
  uint64_t next_id = 1;
  cudaStream_t stream = nullptr;
  std::vector<Entry> active;
  std::deque<Pending> pending;  // enqueued, waiting for budget
  std::deque<lnt_batch_result> finished;
  // launch groups, rebuilt when membership changes
  bool dirty = true;
  std::map<GroupKey, Group> groups;  // fast two-pass tests by geometry
  std::vector<size_t> resident;      // SMEM-resident tests
  std::vector<size_t> singles;       // tests iterated one by one
  lnt::ResidentDesc* d_rdescs = nullptr;
  size_t rcap = 0;
  std::vector<cudaStream_t> spare_streams;
  cudaStream_t rstream = nullptr;    // the resident launch, beside the groups
  cudaEvent_t fork = nullptr;        // recorded on `stream` before the group launches
  cudaEvent_t r0 = nullptr, r1 = nullptr;  // around the resident launch
  bool use_graphs = true;
  bool short_lengths = false;  // n = 0 requests take lnt_smallest_length (2^k or 5 * 2^k)
  // per-call time budget (lnt_batch_step_seconds; 0: every group advances in lockstep) and the
  // measured seconds per squaring per test of each group geometry, and per word-squaring of
  // the resident launch, that it is split by
  double step_seconds = 0;
  std::map<GroupKey, double> group_rate;
  double resident_rate = 0;
  // autotuned plans: (n, shortest valid run) -> plan; loops = 0: policy plans
  uint32_t tune_loops = 0;
  uint32_t tune_group = 1;  // tests timed together per candidate plan (1: one test alone)
  std::map<uint64_t, lnt_plan_options> tuned;
  std::map<uint64_t, float> tuned_ms;  // time of `tune_loops` squarings of the chosen plan
  std::string cache_path;              // JSON plan cache ("" = none)
  // Res64 checkpoints every `checkpoint_every` squarings (0 = none)
  uint64_t checkpoint_every = 0;
  std::deque<lnt_batch_checkpoint> checkpoints;
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

#define BCUDA(call, what)                                                          \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) return berr(LNT_ERR_CUDA, std::string(what) + ": " +    \
                                                         cudaGetErrorString(e_)); \
  } while (0)

cudaStream_t take_stream(lnt_batch* b) {
  if (!b->spare_streams.empty()) {
    cudaStream_t s = b->spare_streams.back();
    b->spare_streams.pop_back();
    return s;
  }
  cudaStream_t s = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  return s;
}

void drop_graphs(lnt_batch* b) {
  for (auto& kv : b->groups) {
    if (kv.second.graph) cudaGraphExecDestroy(kv.second.graph);
    kv.second.graph = nullptr;
  }
}

// k squarings of one group on its stream.
int group_launches(Group& g, uint64_t k) {
  const uint32_t cnt = (uint32_t)g.members.size();
  if (!g.fused) {
    for (uint64_t it = 0; it < k; ++it) {
      BCUDA(lnt::launch_col_forward_r16(g.geometry, g.d_descs, cnt, true, g.stream), "col_forward");
      BCUDA(lnt::launch_row_square_r16(g.geometry, g.d_descs, cnt, g.stream), "row_square");
      BCUDA(lnt::launch_col_inverse_r16(g.geometry, g.d_descs, cnt, false, g.stream), "col_inverse");
    }
  } else if (k > 0) {
    // col_forward, row, (fused col_inverse + col_forward, row) x (k - 1), col_inverse
    BCUDA(lnt::launch_col_forward_r16(g.geometry, g.d_descs, cnt, true, g.stream), "col_forward");
    BCUDA(lnt::launch_row_square_r16(g.geometry, g.d_descs, cnt, g.stream), "row_square");
    for (uint64_t it = 1; it < k; ++it) {
      BCUDA(lnt::launch_col_fused_r16(g.geometry, g.d_descs, cnt, g.stream), "col_fused");
      BCUDA(lnt::launch_row_square_r16(g.geometry, g.d_descs, cnt, g.stream), "row_square");
    }
    BCUDA(lnt::launch_col_inverse_r16(g.geometry, g.d_descs, cnt, false, g.stream), "col_inverse");
  }
  return LNT_OK;
}

// The group's kGraphChunk squarings captured once per membership and replayed.
int build_group_graph(Group& g) {
  BCUDA(cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  const int st = group_launches(g, kGraphChunk);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(g.stream, &graph);
  if (st != LNT_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (e != cudaSuccess) return berr(LNT_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
  const cudaError_t ie = cudaGraphInstantiate(&g.graph, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    g.graph = nullptr;
    return berr(LNT_ERR_CUDA, std::string("instantiate graph: ") + cudaGetErrorString(ie));
  }
  return LNT_OK;
}

// Every group's g.k squarings, forked from b->stream onto the group streams
// (graph replays of kGraphChunk squarings, the remainder as plain launches)
// and joined back; events around each group's work time it.
int launch_groups(lnt_batch* b) {
  BCUDA(cudaEventRecord(b->fork, b->stream), "fork");
  for (auto& kv : b->groups) {
    Group& g = kv.second;
    BCUDA(cudaStreamWaitEvent(g.stream, b->fork, 0), "fork wait");
    BCUDA(cudaEventRecord(g.t0, g.stream), "group timer");
    uint64_t left = g.k;
    if (b->use_graphs && left >= kGraphChunk) {
      if (!g.graph) {
        const int st = build_group_graph(g);
        if (st != LNT_OK) return st;
      }
      for (; left >= kGraphChunk; left -= kGraphChunk) BCUDA(cudaGraphLaunch(g.graph, g.stream), "graph launch");
    }
    const int st = group_launches(g, left);
    if (st != LNT_OK) return st;
    BCUDA(cudaEventRecord(g.t1, g.stream), "group timer");
    BCUDA(cudaEventRecord(g.join, g.stream), "join");
    BCUDA(cudaStreamWaitEvent(b->stream, g.join, 0), "join wait");
  }
  return LNT_OK;
}

void free_group(lnt_batch* b, Group& g, bool keep_stream) {
  if (g.graph) cudaGraphExecDestroy(g.graph);
  if (g.d_descs) cudaFree(g.d_descs);
  for (cudaEvent_t e : {g.join, g.t0, g.t1})
    if (e) cudaEventDestroy(e);
  if (keep_stream) b->spare_streams.push_back(g.stream);
  else if (g.stream) cudaStreamDestroy(g.stream);
  g = Group();
}

int rebuild(lnt_batch* b) {
  for (auto& kv : b->groups) free_group(b, kv.second, true);
  b->groups.clear();
  b->resident.clear();
  b->singles.clear();
  for (size_t i = 0; i < b->active.size(); ++i) {
    const lnt::Plan& p = lnt::test_plan(b->active[i].t);
    if (p.kind == lnt::PlanKind::Resident) {
      b->resident.push_back(i);
    } else if (p.fast && lnt::test_ready_for_group(b->active[i].t)) {
      // one launch serves tests of identical geometry
      Group& g = b->groups[GroupKey{p.n, p.log2n2, p.tile, p.radix, p.fused}];
      g.n = p.n;
      g.fused = p.fused;
      g.members.push_back(i);
    } else {
      b->singles.push_back(i);
    }
  }
  for (auto& kv : b->groups) {
    Group& g = kv.second;
    std::vector<lnt::TwoPassDesc> h;
    for (size_t i : g.members) h.push_back(lnt::test_twopass_desc(b->active[i].t));
    g.geometry = h[0];
    BCUDA(cudaMalloc((void**)&g.d_descs, h.size() * sizeof(lnt::TwoPassDesc)), "group descriptors");
    g.cap = h.size();
    BCUDA(cudaMemcpy(g.d_descs, h.data(), h.size() * sizeof(lnt::TwoPassDesc), cudaMemcpyHostToDevice),
          "upload descriptors");
    // a copy from pageable memory may return before its DMA lands, and the
    // group's kernels run on non-blocking streams that do not wait for it
    BCUDA(cudaDeviceSynchronize(), "synchronize");
    g.stream = take_stream(b);
    BCUDA(cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming), "group event");
    BCUDA(cudaEventCreate(&g.t0), "group event");
    BCUDA(cudaEventCreate(&g.t1), "group event");
  }
  if (b->resident.size() > b->rcap) {
    if (b->d_rdescs) cudaFree(b->d_rdescs);
    b->rcap = std::max<size_t>(b->resident.size(), 2 * b->rcap);
    BCUDA(cudaMalloc((void**)&b->d_rdescs, b->rcap * sizeof(lnt::ResidentDesc)), "resident descriptors");
  }
  b->dirty = false;
  return LNT_OK;
}

int retire_finished(lnt_batch* b) {
  bool any = false;
  for (size_t i = 0; i < b->active.size();) {
    Entry& e = b->active[i];
    if (e.done < e.target) {
      ++i;
      continue;
    }
    lnt_batch_result r{};
    r.id = e.id;
    r.exponent = e.q;
    r.n = e.n;
    r.prp = e.prp;
    r.iterations = e.done;
    int st = lnt_res64(e.t, &r.res64);
    if (st == LNT_OK) st = lnt_is_prime(e.t, &r.is_prime);
    r.status = st;
    r.seconds = std::chrono::duration<double>(Clock::now() - e.submitted).count();
    b->finished.push_back(r);
    lnt_destroy(e.t);
    b->used -= e.bytes;
    b->active.erase(b->active.begin() + (long)i);
    any = true;
  }
  if (any) b->dirty = true;
  return LNT_OK;
}

}  // namespace

extern "C" {

uint64_t lnt_test_device_bytes(uint32_t exponent, uint32_t n) {
  if (n == 0) n = 1u << lnt_secured_log2_length(exponent);
  return lnt::test_device_bytes(n);
}

int lnt_batch_create(int device, uint64_t hbm_budget_bytes, lnt_batch** out) {
  if (!out) return berr(LNT_ERR_INVALID_ARGUMENT, "null output pointer");
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return berr(LNT_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= count) return berr(LNT_ERR_INVALID_ARGUMENT, "bad device index");
  DeviceGuard guard(device);
  lnt_batch* b = new lnt_batch();
  b->device = device;
  b->budget = hbm_budget_bytes;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->rstream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&b->r0) != cudaSuccess || cudaEventCreate(&b->r1) != cudaSuccess) {
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->rstream) cudaStreamDestroy(b->rstream);
    for (cudaEvent_t e : {b->fork, b->r0, b->r1})
      if (e) cudaEventDestroy(e);
    delete b;
    return berr(LNT_ERR_CUDA, "cudaStreamCreate");
  }
  *out = b;
  return LNT_OK;
}

int lnt_batch_destroy(lnt_batch* b) {
  if (!b) return LNT_OK;
  DeviceGuard guard(b->device);
  cudaDeviceSynchronize();
  for (auto& e : b->active) lnt_destroy(e.t);
  for (auto& kv : b->groups) free_group(b, kv.second, false);
  for (cudaEvent_t e : {b->fork, b->r0, b->r1})
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : b->spare_streams)
    if (s) cudaStreamDestroy(s);
  if (b->d_rdescs) cudaFree(b->d_rdescs);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->rstream) cudaStreamDestroy(b->rstream);
  delete b;
  return LNT_OK;
}

}  // extern "C"

namespace {

// ---- JSON plan cache: {"device": NAME, "plans": [{"n": .., "run": .., "kind": ..,
// "log2_rows": .., "tile": .., "radix": .., "fused": .., "ms": .., "loops": ..}, ...]}

std::string device_name(int device) {
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return "unknown";
  return prop.name;
}

void save_plan_cache(const lnt_batch* b) {
  std::ostringstream o;
  o << "{\n \"device\": \"" << device_name(b->device) << "\",\n \"plans\": [";
  bool first = true;
  for (const auto& kv : b->tuned) {
    const lnt_plan_options& p = kv.second;
    if (p.kind == 0) continue;  // tuning failed: nothing to keep
    auto ms = b->tuned_ms.find(kv.first);
    o << (first ? "\n" : ",\n") << "  {\"n\": " << (kv.first >> 8) << ", \"run\": " << (kv.first & 0xFF)
      << ", \"kind\": " << p.kind << ", \"log2_rows\": " << p.log2_rows << ", \"tile\": " << p.tile
      << ", \"radix\": " << p.radix << ", \"fused\": " << p.fused
      << ", \"ms\": " << (ms == b->tuned_ms.end() ? -1.0f : ms->second) << ", \"loops\": " << b->tune_loops
      << "}";
    first = false;
  }
  o << "\n ]\n}\n";
  const std::string tmp = b->cache_path + ".tmp";
  {
    std::ofstream f(tmp, std::ios::trunc);
    if (!f) return;
    f << o.str();
  }
  std::rename(tmp.c_str(), b->cache_path.c_str());
}

// The number after "key": inside one plan object (text between braces).
bool json_number(const std::string& obj, const char* key, double& out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t pos = obj.find(k);
  if (pos == std::string::npos) return false;
  pos = obj.find(':', pos + k.size());
  if (pos == std::string::npos) return false;
  char* end = nullptr;
  out = std::strtod(obj.c_str() + pos + 1, &end);
  return end != obj.c_str() + pos + 1;
}

// Loads the plans measured on a device of this batch's device name.
void load_plan_cache(lnt_batch* b) {
  std::ifstream f(b->cache_path);
  if (!f) return;
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  const size_t dk = text.find("\"device\"");
  if (dk == std::string::npos) return;
  const size_t q0 = text.find('"', text.find(':', dk) + 1);
  const size_t q1 = q0 == std::string::npos ? q0 : text.find('"', q0 + 1);
  if (q1 == std::string::npos || text.substr(q0 + 1, q1 - q0 - 1) != device_name(b->device)) return;
  size_t pos = text.find("\"plans\"");
  while (pos != std::string::npos) {
    const size_t o0 = text.find('{', pos);
    if (o0 == std::string::npos) break;
    const size_t o1 = text.find('}', o0);
    if (o1 == std::string::npos) break;
    const std::string obj = text.substr(o0, o1 - o0 + 1);
    double n, run, kind, rows, tile, radix, fused, ms = -1;
    if (json_number(obj, "n", n) && json_number(obj, "run", run) && json_number(obj, "kind", kind) &&
        json_number(obj, "log2_rows", rows) && json_number(obj, "tile", tile) &&
        json_number(obj, "radix", radix) && json_number(obj, "fused", fused)) {
      json_number(obj, "ms", ms);
      const uint64_t key = ((uint64_t)n << 8) | ((uint64_t)run & 0xFF);
      lnt_plan_options p{(uint32_t)kind, (uint32_t)rows, (uint32_t)tile, (uint32_t)radix, (uint32_t)fused};
      b->tuned[key] = p;
      b->tuned_ms[key] = (float)ms;
    }
    pos = o1 + 1;
  }
}

int admit(lnt_batch* b, uint64_t id, uint32_t exponent, uint32_t n, int prp, uint64_t iterations,
          Clock::time_point since);

// Batch-aware tuning: every candidate plan of (n, exponent's run class) timed
// on `tune_group` copies of the test advancing together in a scratch batch
// (graph replay, as the real groups run), `tune_loops` squarings after a
// warm-up; the fastest is kept.  A plan that fails is skipped.
void tune_in_group(lnt_batch* b, uint32_t exponent, uint32_t n, int prp, uint64_t key,
                   lnt_plan_options& chosen, float& best_ms) {
  lnt_plan_options cands[128];
  int count = 0;
  if (lnt_plan_candidates(exponent, n, cands, 128, &count) != LNT_OK) return;
  for (int c = 0; c < count && c < 128; ++c) {
    lnt_batch* tb = nullptr;
    if (lnt_batch_create(b->device, 0, &tb) != LNT_OK) return;
    tb->tune_loops = 1;  // admissions take the plan below, no timing of their own
    tb->tuned[key] = cands[c];
    bool ok = true;
    for (uint32_t g = 0; g < b->tune_group && ok; ++g)
      ok = admit(tb, tb->next_id++, exponent, n, prp, 0, Clock::now()) == LNT_OK;
    ok = ok && lnt_batch_run(tb, kGraphChunk) == LNT_OK;  // graph capture, kernel loading
    const Clock::time_point t0 = Clock::now();
    ok = ok && lnt_batch_run(tb, b->tune_loops) == LNT_OK;  // ends with a device synchronisation
    const float ms = std::chrono::duration<float, std::milli>(Clock::now() - t0).count();
    lnt_batch_destroy(tb);
    if (ok && (best_ms < 0 || ms < best_ms)) {
      best_ms = ms;
      chosen = cands[c];
    }
  }
}

// Create the test's state on the device and add it to the active set.
int admit(lnt_batch* b, uint64_t id, uint32_t exponent, uint32_t n, int prp, uint64_t iterations,
          Clock::time_point since) {
  const uint64_t bytes = lnt::test_device_bytes(n);
  lnt_test* t = nullptr;
  const lnt_plan_options* plan = nullptr;
  int st;
  if (b->tune_loops && n > 4096) {
    // one timing per (length, shortest carry run the exponent allows)
    const uint32_t run = lnt::r16_run_words_needed(exponent, n) <= 4 ? 4 : 8;
    const uint64_t key = ((uint64_t)n << 8) | run;
    auto it = b->tuned.find(key);
    if (it == b->tuned.end()) {
      lnt_plan_options chosen{};
      float best_ms = -1.0f;
      if (b->tune_group > 1) {
        tune_in_group(b, exponent, n, prp, key, chosen, best_ms);
      } else {
        lnt_plan_options tried[128];
        float ms[128];
        int count = 0, best = -1;
        st = lnt_autotune(exponent, n, prp, b->device, b->tune_loops, tried, ms, 128, &count, &best);
        if (st == LNT_OK && best >= 0 && best < 128) {
          chosen = tried[best];
          best_ms = ms[best];
        }
      }
      if (chosen.kind) b->tuned_ms[key] = best_ms;
      it = b->tuned.emplace(key, chosen).first;
      if (!b->cache_path.empty()) save_plan_cache(b);
    }
    plan = &it->second;
  }
  st = lnt_create_with_plan(exponent, n, prp, b->device, plan, &t);
  if (st != LNT_OK) return st;
  Entry e{};
  e.id = id;
  e.t = t;
  e.q = exponent;
  e.n = n;
  e.prp = prp ? 1 : 0;
  e.target = iterations ? iterations : (prp ? (uint64_t)exponent : (uint64_t)exponent - 2);
  e.done = 0;
  e.bytes = bytes;
  e.submitted = since;
  const lnt::Plan& p = lnt::test_plan(t);
  if (p.kind == lnt::PlanKind::TwoPass && e.target > 0) {
    // the first squaring reads non-negative digits (unsigned outputs): run it
    // alone, after which the test joins its length group
    if ((st = lnt_iterate(t, 1)) != LNT_OK || (st = lnt_synchronize(t)) != LNT_OK) {
      lnt_destroy(t);
      return st;
    }
    e.done = 1;
  }
  b->used += bytes;
  b->active.push_back(e);
  b->dirty = true;
  return LNT_OK;
}

// Admit queued tests first-fit while the budget allows.
int admit_pending(lnt_batch* b) {
  for (auto it = b->pending.begin(); it != b->pending.end();) {
    const uint64_t bytes = lnt::test_device_bytes(it->n);
    if (b->budget && b->used + bytes > b->budget) {
      ++it;
      continue;
    }
    const int st = admit(b, it->id, it->q, it->n, it->prp, it->iterations, it->enqueued);
    if (st != LNT_OK) return st;
    it = b->pending.erase(it);
  }
  return LNT_OK;
}

// Squarings a test may run before its target or its next checkpoint.
uint64_t steps_left(const lnt_batch* b, const Entry& e) {
  uint64_t r = e.target - e.done;
  if (b->checkpoint_every) r = std::min(r, b->checkpoint_every - e.done % b->checkpoint_every);
  return r;
}

// Res64 of every test that has just reached a checkpoint below its target.
void record_checkpoints(lnt_batch* b) {
  if (!b->checkpoint_every) return;
  for (Entry& e : b->active) {
    if (e.done == 0 || e.done >= e.target || e.done % b->checkpoint_every || e.last_checkpoint == e.done)
      continue;
    lnt_batch_checkpoint c{};
    c.id = e.id;
    c.iteration = e.done;
    c.status = lnt_res64(e.t, &c.res64);
    b->checkpoints.push_back(c);
    e.last_checkpoint = e.done;
  }
}

int check_request(const lnt_batch* b, uint32_t exponent, uint32_t& n) {
  if (n == 0 && !(b->short_lengths && lnt_smallest_length(exponent, &n) == LNT_OK))
    n = 1u << lnt_secured_log2_length(exponent);
  if (lnt::test_device_bytes(n) == 0) return berr(LNT_ERR_UNSUPPORTED_LENGTH, "unsupported length");
  return LNT_OK;
}

}  // namespace

extern "C" {

int lnt_batch_submit(lnt_batch* b, uint32_t exponent, uint32_t n, int prp, uint64_t iterations,
                     uint64_t* id) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  DeviceGuard guard(b->device);
  int st = check_request(b, exponent, n);
  if (st != LNT_OK) return st;
  if (b->budget && b->used + lnt::test_device_bytes(n) > b->budget)
    return berr(LNT_ERR_BUDGET, "test does not fit the HBM budget");
  const uint64_t new_id = b->next_id++;
  if ((st = admit(b, new_id, exponent, n, prp, iterations, Clock::now())) != LNT_OK) return st;
  if (id) *id = new_id;
  return retire_finished(b);
}

int lnt_batch_enqueue(lnt_batch* b, uint32_t exponent, uint32_t n, int prp, uint64_t iterations,
                      uint64_t* id) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  DeviceGuard guard(b->device);
  int st = check_request(b, exponent, n);
  if (st != LNT_OK) return st;
  if (b->budget && lnt::test_device_bytes(n) > b->budget)
    return berr(LNT_ERR_BUDGET, "test larger than the whole HBM budget");
  Pending p{b->next_id++, exponent, n, prp ? 1 : 0, iterations, Clock::now()};
  b->pending.push_back(p);
  if (id) *id = p.id;
  return admit_pending(b);
}

int lnt_batch_run(lnt_batch* b, uint64_t iterations) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  DeviceGuard guard(b->device);
  int st = admit_pending(b);
  if (st != LNT_OK) return st;
  record_checkpoints(b);  // tests admitted at a checkpoint (their first squaring runs at admission)
  if (b->active.empty() || iterations == 0) return LNT_OK;
  if (b->dirty && (st = rebuild(b)) != LNT_OK) return st;
  const bool budget = b->step_seconds > 0;
  // squarings test i may run in this call: up to its target and its next checkpoint
  std::vector<uint64_t> step(b->active.size());
  for (size_t i = 0; i < b->active.size(); ++i) step[i] = std::min(iterations, steps_left(b, b->active[i]));
  // a group's tests advance together, none past its target or checkpoint.  Without a
  // time budget every group runs the same count (lockstep); with one, each group runs
  // as many squarings as fit in the budget at its measured (at first, modelled) pace
  uint64_t lockstep = iterations;
  for (auto& kv : b->groups)
    for (size_t i : kv.second.members) lockstep = std::min(lockstep, step[i]);
  for (auto& kv : b->groups) {
    Group& g = kv.second;
    uint64_t k = iterations;
    for (size_t i : g.members) k = std::min(k, step[i]);
    if (!budget) {
      k = lockstep;
    } else {
      auto r = b->group_rate.find(kv.first);
      const double per_test = r != b->group_rate.end() ? r->second : 60e-12 * g.n + 2e-6;
      const double sq = per_test * (double)g.members.size() + 10e-6;
      k = std::min<uint64_t>(k, std::max<uint64_t>(1, (uint64_t)(b->step_seconds / sq)));
    }
    g.k = k;
    for (size_t i : g.members) step[i] = k;
  }
  // SMEM-resident tests: one launch, per-test counts, beside the groups
  uint64_t resident_work = 0;  // word-squarings of the slowest CTA
  if (!b->resident.empty()) {
    std::vector<lnt::ResidentDesc> h;
    uint32_t max_n = 0;
    const double rate = b->resident_rate > 0 ? b->resident_rate : 5e-9;
    for (size_t i : b->resident) {
      Entry& e = b->active[i];
      if (budget)
        step[i] = std::min<uint64_t>(step[i], std::max<uint64_t>(1, (uint64_t)(b->step_seconds / (rate * e.n))));
      h.push_back(lnt::test_resident_desc(e.t, step[i]));
      max_n = std::max(max_n, e.n);
      resident_work = std::max<uint64_t>(resident_work, step[i] * e.n);
    }
    BCUDA(cudaMemcpyAsync(b->d_rdescs, h.data(), h.size() * sizeof(lnt::ResidentDesc),
                          cudaMemcpyHostToDevice, b->rstream),
          "upload resident descriptors");
    BCUDA(cudaEventRecord(b->r0, b->rstream), "resident timer");
    BCUDA(lnt::launch_resident(b->d_rdescs, (uint32_t)h.size(), max_n, b->rstream), "resident kernel");
    BCUDA(cudaEventRecord(b->r1, b->rstream), "resident timer");
  }
  if (!b->groups.empty() && (st = launch_groups(b)) != LNT_OK) return st;
  for (size_t i : b->singles) {
    if ((st = lnt_iterate(b->active[i].t, step[i])) != LNT_OK) return st;
  }
  BCUDA(cudaDeviceSynchronize(), "synchronize");
  // paces for the next budgeted call (smoothed)
  for (auto& kv : b->groups) {
    Group& g = kv.second;
    float ms = 0;
    if (g.k >= kGraphChunk && cudaEventElapsedTime(&ms, g.t0, g.t1) == cudaSuccess && ms > 0) {
      const double per_test = ms * 1e-3 / ((double)g.k * (double)g.members.size());
      auto r = b->group_rate.find(kv.first);
      b->group_rate[kv.first] = r == b->group_rate.end() ? per_test : 0.5 * (r->second + per_test);
    }
  }
  if (!b->resident.empty() && resident_work >= 8 * 512) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, b->r0, b->r1) == cudaSuccess && ms > 0) {
      const double rate = ms * 1e-3 / (double)resident_work;
      b->resident_rate = b->resident_rate > 0 ? 0.5 * (b->resident_rate + rate) : rate;
    }
  }
  for (size_t i : b->resident) {
    b->active[i].done += step[i];
    lnt::test_mark_iterated(b->active[i].t);
  }
  for (auto& kv : b->groups)
    for (size_t i : kv.second.members) {
      b->active[i].done += step[i];
      lnt::test_mark_iterated(b->active[i].t);
    }
  for (size_t i : b->singles) b->active[i].done += step[i];
  record_checkpoints(b);
  if ((st = retire_finished(b)) != LNT_OK) return st;
  return admit_pending(b);
}

int lnt_batch_step_seconds(lnt_batch* b, double seconds) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  if (!(seconds >= 0)) return berr(LNT_ERR_INVALID_ARGUMENT, "seconds must be >= 0");
  b->step_seconds = seconds;
  return LNT_OK;
}

int lnt_batch_autotune(lnt_batch* b, uint32_t loops) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  b->tune_loops = loops;
  return LNT_OK;
}

int lnt_batch_autotune_group(lnt_batch* b, uint32_t tests) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  if (tests == 0 || tests > 1024) return berr(LNT_ERR_INVALID_ARGUMENT, "tests must be in [1, 1024]");
  b->tune_group = tests;
  return LNT_OK;
}

int lnt_batch_checkpoint_every(lnt_batch* b, uint64_t every) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  b->checkpoint_every = every;
  return LNT_OK;
}

int lnt_batch_poll_checkpoints(lnt_batch* b, lnt_batch_checkpoint* out, int cap, int* count) {
  if (!b || !count || (cap > 0 && !out)) return berr(LNT_ERR_INVALID_ARGUMENT, "null argument");
  int k = 0;
  while (k < cap && !b->checkpoints.empty()) {
    out[k++] = b->checkpoints.front();
    b->checkpoints.pop_front();
  }
  *count = k;
  return LNT_OK;
}

int lnt_batch_plan_cache(lnt_batch* b, const char* path) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  b->cache_path = path ? path : "";
  if (!b->cache_path.empty()) load_plan_cache(b);
  return LNT_OK;
}

int lnt_batch_short_lengths(lnt_batch* b, int enable) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  b->short_lengths = enable != 0;
  return LNT_OK;
}

int lnt_batch_use_graphs(lnt_batch* b, int enable) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  DeviceGuard guard(b->device);
  b->use_graphs = enable != 0;
  if (!b->use_graphs) drop_graphs(b);
  return LNT_OK;
}

int lnt_batch_poll(lnt_batch* b, lnt_batch_result* out, int cap, int* count) {
  if (!b || !count || (cap > 0 && !out)) return berr(LNT_ERR_INVALID_ARGUMENT, "null argument");
  int k = 0;
  while (k < cap && !b->finished.empty()) {
    out[k++] = b->finished.front();
    b->finished.pop_front();
  }
  *count = k;
  return LNT_OK;
}

int lnt_batch_status(lnt_batch* b, uint32_t* active, uint64_t* bytes_in_use) {
  if (!b) return berr(LNT_ERR_INVALID_ARGUMENT, "null batch");
  if (active) *active = (uint32_t)b->active.size();
  if (bytes_in_use) *bytes_in_use = b->used;
  return LNT_OK;
}

int lnt_batch_pending(lnt_batch* b, uint32_t* pending) {
  if (!b || !pending) return berr(LNT_ERR_INVALID_ARGUMENT, "null argument");
  *pending = (uint32_t)b->pending.size();
  return LNT_OK;
}

}  // extern "C"
