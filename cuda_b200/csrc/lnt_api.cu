// C ABI of the single-test path: context lifetime, residue I/O, iteration.
//
// Mirrors LucasPRP (lucas_prp.cu:24-346): Initialize allocates the residue and
// the IBDWT tables, InitializeTest writes the start value, MainLoop queues
// `iterations` squarings, and readout copies the canonical digits back.
// Errors are status codes (the reference throws std::runtime_error from
// cudaCheckErrors, common/common.cuh:23-29).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lucasntt.h"
#include "goldilocks.cuh"
#include "lnt_internal.h"

namespace lnt {
struct Gerbicz;
struct Jacobi;
bool jacobi_available(std::string* why);
int jacobi_of_ll_residue(const uint64_t* digits, const uint8_t* widths, uint32_t n, uint32_t q,
                         std::string* why);
}

struct lnt_test {
  uint32_t q = 0, n = 0;
  int prp = 0;
  int device = 0;
  lnt::Plan plan;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  int64_t* x = nullptr;
  uint64_t* w = nullptr;
  uint64_t* uw = nullptr;
  uint8_t* widths = nullptr;
  uint32_t* status = nullptr;
  // resident plan
  uint64_t* rt = nullptr;
  uint64_t* irt = nullptr;
  lnt::ResidentDesc* rdesc = nullptr;
  lnt::TwoPassDesc* tdesc = nullptr;  // device copy of the two-pass descriptor
  // two-pass plan
  uint64_t *twf = nullptr, *twi = nullptr;
  uint64_t *rt1 = nullptr, *irt1 = nullptr, *rt2 = nullptr, *irt2 = nullptr;
  uint64_t *itw1 = nullptr, *iitw1 = nullptr, *itw2 = nullptr, *iitw2 = nullptr;
  uint64_t *tw5 = nullptr, *itw5 = nullptr;  // n = 5 * 2^k: the radix-5 step's twiddles
  uint64_t c5[4] = {};                        // and its constants
  uint64_t *wt = nullptr, *uwt = nullptr;
  uint8_t* widt = nullptr;
  int64_t* carry = nullptr;
  uint32_t* fuse = nullptr;  // carry-fused column kernel: ticket, epoch, tile flags
  // canonical readout
  uint64_t* canon = nullptr;
  int64_t* blk_carry = nullptr;
  uint8_t* blk_fn = nullptr;
  int8_t* blk_cin = nullptr;
  uint32_t* cflags = nullptr;
  uint32_t* h_pinned = nullptr;  // 2 words: status, canon flags

  std::vector<uint8_t> h_widths;
  bool canonical_input = true;  // digits non-negative: next squaring reads outputs unsigned
  bool pending_carries = false; // two-pass: carry buffer holds carries not yet applied
  bool pristine = true;         // no squaring since the digits were set
  bool zero_start = false;      // digits were set to all zero
  bool canon_valid = false;     // `canon` holds the canonical digits of the current state
  // steady-state squarings of the pass-kernel plan, captured once and replayed
  cudaGraphExec_t graph = nullptr;
  bool graph_failed = false;    // capture unavailable on this stream: plain launches
  lnt::Gerbicz* gz = nullptr;   // PRP error check (lnt_gerbicz_enable), or none
  lnt::Jacobi* jc = nullptr;    // LL error check (lnt_jacobi_enable), or none
};

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? LNT_ERR_OUT_OF_MEMORY : LNT_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define LNT_CUDA(call, what)                          \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

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

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, count * sizeof(T));
}

void free_gerbicz(lnt_test* t);
void free_jacobi(lnt_test* t);

void free_all(lnt_test* t) {
  free_gerbicz(t);
  free_jacobi(t);
  void* ptrs[] = {t->x, t->w, t->uw, t->widths, t->status, t->rt, t->irt, t->rdesc, t->tdesc,
                  t->twf, t->twi, t->rt1, t->irt1, t->rt2, t->irt2, t->itw1, t->iitw1,
                  t->itw2, t->iitw2, t->tw5, t->itw5, t->wt, t->uwt, t->widt, t->carry, t->fuse, t->canon,
                  t->blk_carry, t->blk_fn, t->blk_cin, t->cflags};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (t->h_pinned) cudaFreeHost(t->h_pinned);
  if (t->graph) cudaGraphExecDestroy(t->graph);
  if (t->own_stream && t->stream) cudaStreamDestroy(t->stream);
}

// omega_n^k for k < max(n/2, 1), generator 554 (pre_calculation.cu:61-66).
void root_table(uint32_t n, bool inverse, std::vector<uint64_t>& out) {
  uint64_t r = gl::pow(554, (gl::P - 1) / n);
  if (inverse) r = gl::inv(r);
  size_t half = n > 1 ? n / 2 : 1;
  out.resize(half);
  out[0] = 1;
  for (size_t k = 1; k < half; ++k) out[k] = gl::mul(out[k - 1], r);
}

// omega_n^e for all e < n (the radix-16 kernels index it with t * k * span_scale < n).
void power_table(uint32_t n, bool inverse, std::vector<uint64_t>& out) {
  uint64_t r = gl::pow(554, (gl::P - 1) / n);
  if (inverse) r = gl::inv(r);
  out.resize(n);
  out[0] = 1;
  for (size_t k = 1; k < n; ++k) out[k] = gl::mul(out[k - 1], r);
}

// Inter-pass twiddles of a length-n radix-16 transform in pass order: pass j
// (span s, radix R, q = s / R) holds, for each task t < q, the run
// omega_n^(t brev_R(r) n / s), r < R.  The last pass (q = 1) has none.
void pass_table(uint32_t n, uint32_t max_radix, bool inverse, std::vector<uint64_t>& out) {
  uint32_t log2n = 0;
  while ((1u << log2n) < n) ++log2n;
  std::vector<uint64_t> pw;
  power_table(n, inverse, pw);
  const std::vector<uint32_t> radix = lnt::r16_pass_radices(log2n, max_radix);
  out.clear();
  uint32_t span = n;
  for (size_t j = 0; j + 1 < radix.size(); ++j) {
    const uint32_t R = radix[j], q = span / R, scale = n / span;
    uint32_t bits = 0;
    while ((1u << bits) < R) ++bits;
    for (uint32_t t = 0; t < q; ++t)
      for (uint32_t r = 0; r < R; ++r) {
        uint32_t b = 0;
        for (uint32_t i = 0; i < bits; ++i) b |= ((r >> i) & 1u) << (bits - 1 - i);
        out.push_back(pw[(size_t)t * b * scale]);
      }
    span /= R;
  }
  if (out.empty()) out.push_back(1);  // keep the pointer valid
}

// max_radix = 0: root_table (n/2 entries); 8 or 16: pass_table of passes of
// at most that radix
int upload_roots(lnt_test* t, uint32_t n, uint64_t** rt, uint64_t** irt, uint32_t max_radix = 0) {
  std::vector<uint64_t> a, b;
  if (max_radix) {
    pass_table(n, max_radix, false, a);
    pass_table(n, max_radix, true, b);
  } else {
    root_table(n, false, a);
    root_table(n, true, b);
  }
  LNT_CUDA(dalloc(rt, a.size()), "cudaMalloc roots");
  LNT_CUDA(dalloc(irt, b.size()), "cudaMalloc roots");
  // host-to-device copies go on the test's (non-blocking) stream, ahead of the
  // kernels that read them: a plain cudaMemcpy from pageable memory may return
  // before its DMA lands, and it is not ordered with work on that stream
  LNT_CUDA(cudaMemcpyAsync(*rt, a.data(), a.size() * 8, cudaMemcpyHostToDevice, t->stream), "copy roots");
  LNT_CUDA(cudaMemcpyAsync(*irt, b.data(), b.size() * 8, cudaMemcpyHostToDevice, t->stream), "copy roots");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  return LNT_OK;
}

lnt::TwoPassDesc twopass_desc(const lnt_test* t) {
  lnt::TwoPassDesc d{};
  d.x = t->x;
  d.carry = t->carry;
  d.w = t->w;
  d.uw = t->uw;
  d.widths = t->widths;
  d.twf = t->twf;
  d.twi = t->twi;
  d.rt1 = t->rt1;
  d.irt1 = t->irt1;
  d.rt2 = t->rt2;
  d.irt2 = t->irt2;
  d.fuse = t->fuse;
  d.itw1 = t->itw1;
  d.iitw1 = t->iitw1;
  d.itw2 = t->itw2;
  d.iitw2 = t->iitw2;
  d.wt = t->wt;
  d.uwt = t->uwt;
  d.widt = t->widt;
  d.status = t->status;
  d.n1 = t->plan.n1;
  d.n2 = t->plan.n2;
  d.log2n1 = t->plan.log2n1;
  d.log2n2 = t->plan.log2n2;
  d.tile = t->plan.tile;
  d.ntiles = t->plan.ntiles;
  d.prp = (uint32_t)t->prp;
  d.radix = t->plan.radix;
  d.five = t->plan.five ? 1 : 0;
  d.tw5 = t->tw5;
  d.itw5 = t->itw5;
  for (int k = 0; k < 4; ++k) d.c5[k] = t->c5[k];
  return d;
}

// Exact cyclic normalisation on the host: the fallback of the device readout.
void canonicalize_host(const std::vector<int64_t>& x, const std::vector<int64_t>& carries,
                       const lnt_test* t, std::vector<uint64_t>& out) {
  const uint32_t n = t->n;
  std::vector<int64_t> v(x);
  if (!carries.empty()) {
    const lnt::Plan& P = t->plan;
    for (uint32_t tt = 0; tt < P.ntiles; ++tt)
      for (uint32_t r = 0; r < P.n2; ++r) {
        // carry of run (tt, r) lands at the start of the next run
        uint32_t nt = tt + 1, nr = r;
        if (nt == P.ntiles) { nt = 0; nr = (r + 1) % P.n2; }
        v[(size_t)nr * P.n1 + (size_t)nt * P.tile] += carries[(size_t)tt * P.n2 + r];
      }
  }
  int64_t carry = 0;
  uint32_t j = 0;
  bool wrapped = false;
  for (;;) {
    int64_t s = v[j] + carry;
    unsigned w = t->h_widths[j];
    v[j] = s & ((int64_t(1) << w) - 1);
    carry = s >> w;
    if (++j == n) { j = 0; wrapped = true; }
    if (wrapped && carry == 0) break;
  }
  out.assign(v.begin(), v.end());
}

// Apply the reference's choice between the two representations of 0 mod M:
// LL residues are in [0, M-1]; PRP residues in [1, M] unless the test started
// from an all-zero residue.
void fix_zero_representation(const lnt_test* t, std::vector<uint64_t>& d) {
  bool all_max = true, all_zero = true;
  for (uint32_t j = 0; j < t->n; ++j) {
    uint64_t mask = (1ull << t->h_widths[j]) - 1;
    all_max &= d[j] == mask;
    all_zero &= d[j] == 0;
  }
  if (!t->prp && all_max) std::fill(d.begin(), d.end(), 0);
  if (t->prp && all_zero && !t->zero_start)
    for (uint32_t j = 0; j < t->n; ++j) d[j] = (1ull << t->h_widths[j]) - 1;
}

int check_status(lnt_test* t) {
  LNT_CUDA(cudaMemcpyAsync(t->h_pinned, t->status, 4, cudaMemcpyDeviceToHost, t->stream),
           "read status");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  if (t->h_pinned[0] & lnt::kStatusCarryOverflow)
    return fail(LNT_ERR_NUMERIC, "carry exceeded the balanced-digit headroom");
  if (t->h_pinned[0] & lnt::kStatusFuseTimeout)
    return fail(LNT_ERR_CUDA, "a carry-fused column CTA timed out waiting for its neighbour");
  return LNT_OK;
}

// Bring `canon` up to date with the current residue.
int canonicalize(lnt_test* t) {
  if (t->canon_valid) return LNT_OK;
  int st = check_status(t);
  if (st != LNT_OK) return st;
  if (t->pristine) {
    LNT_CUDA(cudaMemcpyAsync(t->canon, t->x, (size_t)t->n * 8, cudaMemcpyDeviceToDevice, t->stream),
             "copy digits");
    LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
    t->canon_valid = true;
    return LNT_OK;
  }
  lnt::CanonDesc c{};
  c.x = t->x;
  c.carry = (t->plan.kind == lnt::PlanKind::TwoPass && t->pending_carries) ? t->carry : nullptr;
  c.widths = t->widths;
  c.out = t->canon;
  c.blk_carry = t->blk_carry;
  c.blk_fn = t->blk_fn;
  c.blk_cin = t->blk_cin;
  c.flags = t->cflags;
  c.n = t->n;
  c.block = lnt::canon_block_size(t->n);
  c.nblocks = t->n / c.block;
  c.n1 = t->plan.n1;
  c.n2 = t->plan.n2;
  c.tile = t->plan.tile;
  c.ntiles = t->plan.ntiles;
  LNT_CUDA(cudaMemsetAsync(t->cflags, 0, 4, t->stream), "memset flags");
  LNT_CUDA(lnt::launch_canonicalize(c, t->stream), "canonical readout");
  LNT_CUDA(cudaMemcpyAsync(t->h_pinned + 1, t->cflags, 4, cudaMemcpyDeviceToHost, t->stream),
           "read flags");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  uint32_t flags = t->h_pinned[1];
  if (flags & lnt::kCanonError) {
    // host fallback: exact sequential carry
    std::vector<int64_t> x(t->n), carries;
    LNT_CUDA(cudaMemcpy(x.data(), t->x, (size_t)t->n * 8, cudaMemcpyDeviceToHost), "copy digits");
    if (c.carry) {
      carries.resize((size_t)t->plan.ntiles * t->plan.n2);
      LNT_CUDA(cudaMemcpy(carries.data(), t->carry, carries.size() * 8, cudaMemcpyDeviceToHost),
               "copy carries");
    }
    std::vector<uint64_t> out;
    canonicalize_host(x, carries, t, out);
    fix_zero_representation(t, out);
    LNT_CUDA(cudaMemcpyAsync(t->canon, out.data(), (size_t)t->n * 8, cudaMemcpyHostToDevice, t->stream),
             "upload digits");
    LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
    t->canon_valid = true;
    return LNT_OK;
  }
  const bool all_max = !(flags & lnt::kCanonNotAllMax);
  if (!t->prp && all_max) {
    LNT_CUDA(cudaMemsetAsync(t->canon, 0, (size_t)t->n * 8, t->stream), "zero residue");
  } else if (t->prp && !t->zero_start && !(flags & lnt::kCanonHighNonZero)) {
    uint64_t d0 = 0;
    LNT_CUDA(cudaMemcpy(&d0, t->canon, 8, cudaMemcpyDeviceToHost), "read digit");
    if (d0 == 0) LNT_CUDA(lnt::launch_fill_max(t->canon, t->widths, t->n, t->stream), "fill");
  }
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  t->canon_valid = true;
  return LNT_OK;
}

int upload_digits(lnt_test* t, const uint64_t* digits) {
  LNT_CUDA(cudaMemcpyAsync(t->x, digits, (size_t)t->n * 8, cudaMemcpyHostToDevice, t->stream),
           "upload digits");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  bool zero = true;
  for (uint32_t j = 0; j < t->n && zero; ++j) zero = digits[j] == 0;
  t->zero_start = zero;
  t->canonical_input = true;
  t->pending_carries = false;
  t->pristine = true;
  t->canon_valid = false;
  return LNT_OK;
}

// CUDA events recorded between kernel launches (lnt_profile_iterations).
struct LaunchTimer {
  std::vector<cudaEvent_t> events;
  std::vector<const char*> kinds;  // kinds[i] ran between events[i] and events[i + 1]
  ~LaunchTimer() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
  }
  cudaError_t mark(cudaStream_t s) {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return r;
    events.push_back(e);
    return cudaEventRecord(e, s);
  }
};

#define LNT_LAUNCH(call, kind)                                   \
  do {                                                           \
    if (timer && timer->events.empty())                          \
      LNT_CUDA(timer->mark(t->stream), "event");                 \
    LNT_CUDA(call, kind);                                        \
    if (timer) {                                                 \
      timer->kinds.push_back(kind);                              \
      LNT_CUDA(timer->mark(t->stream), "event");                 \
    }                                                            \
  } while (0)

// Queue `iterations` squarings on the test's stream (LucasPRP::MainLoop).
// Squarings per captured graph: launch overhead amortised over 3 x 16 kernels.
constexpr uint64_t kGraphSquarings = 16;

// Capture kGraphSquarings steady-state squarings on the test's stream: each a
// fused column launch (the inverse half of one squaring and the forward half of
// the next) and a row launch, or, without fusion, the three launches of a
// squaring.  On any failure the test keeps plain launches (graph_failed).
void capture_graph(lnt_test* t, const lnt::TwoPassDesc& d) {
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(t->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    t->graph_failed = true;
    return;
  }
  bool ok = true;
  for (uint64_t k = 0; k < kGraphSquarings && ok; ++k)
    ok = t->plan.fused
             ? lnt::launch_col_fused_r16(d, t->tdesc, 1, t->stream) == cudaSuccess &&
                   lnt::launch_row_square_r16(d, t->tdesc, 1, t->stream) == cudaSuccess
             : lnt::launch_col_forward_r16(d, t->tdesc, 1, true, t->stream) == cudaSuccess &&
                   lnt::launch_row_square_r16(d, t->tdesc, 1, t->stream) == cudaSuccess &&
                   lnt::launch_col_inverse_r16(d, t->tdesc, 1, false, t->stream) == cudaSuccess;
  const cudaError_t e = cudaStreamEndCapture(t->stream, &g);
  if (ok && e == cudaSuccess && g && cudaGraphInstantiate(&t->graph, g, 0) != cudaSuccess) t->graph = nullptr;
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();  // a failed capture leaves no error behind for the next launch
  if (!t->graph) t->graph_failed = true;
}

int queue_iterations(lnt_test* t, uint64_t iterations, LaunchTimer* timer) {
  if (t->plan.kind == lnt::PlanKind::Resident) {
    lnt::ResidentDesc d{};
    d.digits = t->x;
    d.w = t->w;
    d.uw = t->uw;
    d.widths = t->widths;
    d.rt = t->rt;
    d.irt = t->irt;
    d.status = t->status;
    d.n = t->n;
    d.log2n = t->plan.log2n;
    d.prp = (uint32_t)t->prp;
    d.unsigned_first = t->canonical_input ? 1 : 0;
    d.iterations = iterations;
    d.short_runs = lnt::r16_run_words_needed(t->q, t->n) <= 4 ? 1 : 0;
    LNT_CUDA(cudaMemcpyAsync(t->rdesc, &d, sizeof(d), cudaMemcpyHostToDevice, t->stream),
             "upload descriptor");
    LNT_LAUNCH(lnt::launch_resident(t->rdesc, 1, t->n, t->stream), "resident_square_loop");
    // the descriptor copy is staged from pageable memory: wait so `d` may go
    LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  } else {
    lnt::TwoPassDesc d = twopass_desc(t);
    if (t->plan.fast) {
      uint64_t left = iterations;
      if (t->canonical_input) {
        // the first squaring of non-negative digits reads its outputs unsigned
        LNT_LAUNCH(lnt::launch_col_forward_r16(d, t->tdesc, 1, t->pending_carries, t->stream),
                   "col_forward");
        LNT_LAUNCH(lnt::launch_row_square_r16(d, t->tdesc, 1, t->stream), "row_square");
        LNT_LAUNCH(lnt::launch_col_inverse_r16(d, t->tdesc, 1, true, t->stream), "col_inverse");
        t->pending_carries = true;
        t->canonical_input = false;
        --left;
      }
      if (left && t->plan.fused) {
        // col_forward, then (row, fused col_inverse + col_forward) x (left - 1),
        // row, col_inverse: between calls the state stays digits + carries
        LNT_LAUNCH(lnt::launch_col_forward_r16(d, t->tdesc, 1, true, t->stream), "col_forward");
        LNT_LAUNCH(lnt::launch_row_square_r16(d, t->tdesc, 1, t->stream), "row_square");
        uint64_t mid = left - 1;
        if (!timer && mid >= kGraphSquarings && !t->graph_failed && !t->graph) capture_graph(t, d);
        if (!timer && t->graph)
          for (; mid >= kGraphSquarings; mid -= kGraphSquarings)
            LNT_CUDA(cudaGraphLaunch(t->graph, t->stream), "graph launch");
        for (; mid > 0; --mid) {
          LNT_LAUNCH(lnt::launch_col_fused_r16(d, t->tdesc, 1, t->stream), "col_fused");
          LNT_LAUNCH(lnt::launch_row_square_r16(d, t->tdesc, 1, t->stream), "row_square");
        }
        LNT_LAUNCH(lnt::launch_col_inverse_r16(d, t->tdesc, 1, false, t->stream), "col_inverse");
      } else if (left) {
        // three launches per squaring; whole graphs of kGraphSquarings squarings
        if (!timer && left >= kGraphSquarings && !t->graph_failed && !t->graph) capture_graph(t, d);
        if (!timer && t->graph)
          for (; left >= kGraphSquarings; left -= kGraphSquarings)
            LNT_CUDA(cudaGraphLaunch(t->graph, t->stream), "graph launch");
        for (; left > 0; --left) {
          LNT_LAUNCH(lnt::launch_col_forward_r16(d, t->tdesc, 1, true, t->stream), "col_forward");
          LNT_LAUNCH(lnt::launch_row_square_r16(d, t->tdesc, 1, t->stream), "row_square");
          LNT_LAUNCH(lnt::launch_col_inverse_r16(d, t->tdesc, 1, false, t->stream), "col_inverse");
        }
      }
      t->pending_carries = true;
    } else {
      for (uint64_t i = 0; i < iterations; ++i) {
        LNT_LAUNCH(lnt::launch_col_forward(d, t->pending_carries, t->stream), "col_forward");
        LNT_LAUNCH(lnt::launch_row_square(d, t->stream), "row_square");
        LNT_LAUNCH(lnt::launch_col_inverse(d, t->canonical_input, t->stream), "col_inverse");
        t->pending_carries = true;
        t->canonical_input = false;
      }
    }
  }
  t->canonical_input = false;
  t->pristine = false;
  t->canon_valid = false;
  return LNT_OK;
}

// ---- Gerbicz-Li check for PRP tests ---------------------------------------
//
// No counterpart in the reference, which checks nothing during a test
// (lucas_prp.cu:137-195).  With x_i = x_0^(2^i) (the PRP residue after i
// squarings) and checkpoints c_k = x_{kB} every B squarings, the products
// D_k = c_0 c_1 ... c_k satisfy D_k = c_0 * D_{k-1}^(2^B).  Every B squarings
// the engine folds the current residue into D (one residue product); every
// B^2 squarings it verifies the identity (B squarings of D_{k-1}, one product
// with c_0, a digit compare).  An error anywhere since the last verification
// breaks it: the test then returns to the last verified residue and product
// and redoes the work.  Cost: about 2.5 squarings per B squarings plus B per
// B^2, under 0.5 % at B = 1000.

}  // namespace

namespace lnt {

// A residue state sharing its test's tables: digits and pending run carries.
struct StateBuf {
  int64_t* x = nullptr;
  int64_t* carry = nullptr;
  bool canonical_input = true, pending_carries = false, pristine = true, zero_start = false;
};

struct Gerbicz {
  uint32_t block = 0;
  StateBuf c0, d, dprev, v, xok, dok;
  StateBuf f;                        // scratch: the transformed operand of a product
  TwoPassDesc* fdesc = nullptr;      // device descriptor of `f`
  uint64_t done = 0, verified = 0, checks = 0, errors = 0;
  uint32_t failed_in_a_row = 0;  // recoveries since the last passed verification
  bool have_prev = false;
};

}  // namespace lnt

namespace {

size_t carry_words(const lnt_test* t) { return (size_t)t->plan.ntiles * t->plan.n2; }

void free_state(lnt::StateBuf& s) {
  if (s.x) cudaFree(s.x);
  if (s.carry) cudaFree(s.carry);
  s.x = nullptr;
  s.carry = nullptr;
}

void free_gerbicz(lnt_test* t) {
  if (!t->gz) return;
  lnt::Gerbicz& g = *t->gz;
  for (lnt::StateBuf* s : {&g.c0, &g.d, &g.dprev, &g.v, &g.xok, &g.dok, &g.f}) free_state(*s);
  if (g.fdesc) cudaFree(g.fdesc);
  delete t->gz;
  t->gz = nullptr;
}

lnt::StateBuf main_state(const lnt_test* t) {
  lnt::StateBuf s;
  s.x = t->x;
  s.carry = t->carry;
  s.canonical_input = t->canonical_input;
  s.pending_carries = t->pending_carries;
  s.pristine = t->pristine;
  s.zero_start = t->zero_start;
  return s;
}

// Make `s` the test's current state (and the test's state `s`); the device
// descriptor follows.  Kernels already queued read the descriptor, so the
// stream is drained first.
int swap_state(lnt_test* t, lnt::StateBuf& s) {
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  std::swap(t->x, s.x);
  std::swap(t->carry, s.carry);
  std::swap(t->canonical_input, s.canonical_input);
  std::swap(t->pending_carries, s.pending_carries);
  std::swap(t->pristine, s.pristine);
  std::swap(t->zero_start, s.zero_start);
  t->canon_valid = false;
  const lnt::TwoPassDesc hd = twopass_desc(t);
  // on the test's stream, so the next kernel cannot read the previous state's descriptor
  LNT_CUDA(cudaMemcpyAsync(t->tdesc, &hd, sizeof(hd), cudaMemcpyHostToDevice, t->stream), "descriptor");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  return LNT_OK;
}

int copy_state(lnt_test* t, lnt::StateBuf& dst, const lnt::StateBuf& src) {
  LNT_CUDA(cudaMemcpyAsync(dst.x, src.x, (size_t)t->n * 8, cudaMemcpyDeviceToDevice, t->stream), "copy state");
  LNT_CUDA(cudaMemcpyAsync(dst.carry, src.carry, carry_words(t) * 8, cudaMemcpyDeviceToDevice, t->stream),
           "copy carries");
  dst.canonical_input = src.canonical_input;
  dst.pending_carries = src.pending_carries;
  dst.pristine = src.pristine;
  dst.zero_start = src.zero_start;
  return LNT_OK;
}

// Copy the test's own state into / out of a buffer.
int save_main(lnt_test* t, lnt::StateBuf& dst) { return copy_state(t, dst, main_state(t)); }
int load_main(lnt_test* t, const lnt::StateBuf& src) {
  lnt::StateBuf m = main_state(t);
  int st = copy_state(t, m, src);
  t->canonical_input = src.canonical_input;
  t->pending_carries = src.pending_carries;
  t->pristine = src.pristine;
  t->zero_start = src.zero_start;
  t->canon_valid = false;
  return st;
}

// a <- a * b (a, b: states of this test; b may be the test's own state)
int mul_state(lnt_test* t, lnt::StateBuf& a, const lnt::StateBuf& b) {
  lnt::Gerbicz& g = *t->gz;
  int st;
  if ((st = copy_state(t, g.f, b)) != LNT_OK) return st;
  const lnt::TwoPassDesc geo = twopass_desc(t);
  lnt::TwoPassDesc fd = geo;
  fd.x = g.f.x;
  fd.carry = g.f.carry;
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  LNT_CUDA(cudaMemcpyAsync(g.fdesc, &fd, sizeof(fd), cudaMemcpyHostToDevice, t->stream), "descriptor");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  // the operand's full transform, in place in f
  LNT_CUDA(lnt::launch_col_forward_r16(geo, g.fdesc, 1, b.pending_carries, t->stream), "col_forward");
  LNT_CUDA(lnt::launch_row_forward_r16(geo, g.fdesc, t->stream), "row_forward");
  // a: forward, product with f, inverse, carries
  const bool both_canonical = a.canonical_input && b.canonical_input;
  if ((st = swap_state(t, a)) != LNT_OK) return st;
  const lnt::TwoPassDesc d = twopass_desc(t);
  cudaError_t e = lnt::launch_col_forward_r16(d, t->tdesc, 1, t->pending_carries, t->stream);
  if (e == cudaSuccess) e = lnt::launch_row_mul_r16(d, t->tdesc, reinterpret_cast<const uint64_t*>(g.f.x), t->stream);
  if (e == cudaSuccess) e = lnt::launch_col_inverse_r16(d, t->tdesc, 1, both_canonical, t->stream);
  t->pending_carries = true;
  t->canonical_input = false;
  t->pristine = false;
  t->zero_start = false;
  st = swap_state(t, a);
  if (e != cudaSuccess) return cuda_fail(e, "residue product");
  return st;
}

// canonical digits of a state
int state_digits(lnt_test* t, lnt::StateBuf& s, std::vector<uint64_t>& out) {
  int st = swap_state(t, s);
  if (st != LNT_OK) return st;
  out.resize(t->n);
  st = canonicalize(t);
  if (st == LNT_OK) {
    cudaError_t e = cudaMemcpyAsync(out.data(), t->canon, (size_t)t->n * 8, cudaMemcpyDeviceToHost, t->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
    if (e != cudaSuccess) st = cuda_fail(e, "read digits");
  }
  const int st2 = swap_state(t, s);
  return st != LNT_OK ? st : st2;
}

// B squarings of a state
int square_state(lnt_test* t, lnt::StateBuf& s, uint64_t k) {
  int st = swap_state(t, s);
  if (st != LNT_OK) return st;
  st = queue_iterations(t, k, nullptr);
  const int st2 = swap_state(t, s);
  return st != LNT_OK ? st : st2;
}

// Recoveries in a row without a passed verification before the error is
// returned: a fault that repeats on the same squarings is not transient.
constexpr uint32_t kGerbiczRetries = 3;

// The kernels' status word (sticky bits, lnt::kStatus*), read on the stream.
int read_status(lnt_test* t, uint32_t& flags) {
  LNT_CUDA(cudaMemcpyAsync(t->h_pinned, t->status, 4, cudaMemcpyDeviceToHost, t->stream), "read status");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  flags = t->h_pinned[0];
  return LNT_OK;
}

// A detected error (a failed comparison, or a carry that left the
// balanced-digit headroom, which only corrupted data produces): back to the
// last verified residue and product, with the carry flag cleared.
int gerbicz_recover(lnt_test* t) {
  lnt::Gerbicz& g = *t->gz;
  ++g.errors;
  if (++g.failed_in_a_row > kGerbiczRetries)
    return fail(LNT_ERR_NUMERIC, "Gerbicz check: the same squarings failed " +
                                     std::to_string(kGerbiczRetries) + " times in a row");
  int st;
  if ((st = load_main(t, g.xok)) != LNT_OK || (st = copy_state(t, g.d, g.dok)) != LNT_OK) return st;
  LNT_CUDA(cudaMemsetAsync(t->status, 0, 4, t->stream), "clear status");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  g.done = g.verified;
  g.have_prev = false;
  return LNT_OK;
}

// Start (or restart) the chain at the test's current residue.
int gerbicz_rebase(lnt_test* t) {
  lnt::Gerbicz& g = *t->gz;
  int st;
  for (lnt::StateBuf* s : {&g.c0, &g.d, &g.xok, &g.dok})
    if ((st = save_main(t, *s)) != LNT_OK) return st;
  g.done = g.verified = 0;
  g.failed_in_a_row = 0;
  g.have_prev = false;
  return LNT_OK;
}

// D_k = c_0 * D_{k-1}^(2^B)?  On success the current residue and product become
// the verified ones; on failure the test returns to them.
int gerbicz_verify(lnt_test* t, bool& ok) {
  lnt::Gerbicz& g = *t->gz;
  int st;
  if ((st = copy_state(t, g.v, g.dprev)) != LNT_OK) return st;
  if ((st = square_state(t, g.v, g.block)) != LNT_OK) return st;
  if ((st = mul_state(t, g.v, g.c0)) != LNT_OK) return st;
  // a carry flagged anywhere since the last look fails the check without a readout
  uint32_t flags = 0;
  if ((st = read_status(t, flags)) != LNT_OK) return st;
  ok = false;
  if (!(flags & lnt::kStatusCarryOverflow)) {
    std::vector<uint64_t> lhs, rhs;
    if ((st = state_digits(t, g.d, lhs)) != LNT_OK) return st;
    if ((st = state_digits(t, g.v, rhs)) != LNT_OK) return st;
    ok = lhs == rhs;
  }
  if (ok) {
    if ((st = save_main(t, g.xok)) != LNT_OK || (st = copy_state(t, g.dok, g.d)) != LNT_OK) return st;
    g.verified = g.done;
    g.failed_in_a_row = 0;
    ++g.checks;
  } else if ((st = gerbicz_recover(t)) != LNT_OK) {
    return st;
  }
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  return LNT_OK;
}

// A carry flagged by the kernels since the last look: recover (and redo the
// squarings since the last verification).  Called where the stream is about to
// be drained anyway.
int gerbicz_check_carries(lnt_test* t, uint64_t& left, bool& recovered) {
  lnt::Gerbicz& g = *t->gz;
  uint32_t flags = 0;
  int st = read_status(t, flags);
  recovered = false;
  if (st != LNT_OK || !(flags & lnt::kStatusCarryOverflow)) return st;
  const uint64_t before = g.done;
  if ((st = gerbicz_recover(t)) != LNT_OK) return st;
  left += before - g.done;
  recovered = true;
  return LNT_OK;
}

// lnt_iterate with the check: `iterations` squarings that are (up to the last
// B^2 boundary) verified, redoing blocks that fail a comparison or raise the
// carry flag.
int gerbicz_iterate(lnt_test* t, uint64_t iterations) {
  lnt::Gerbicz& g = *t->gz;
  const uint64_t B = g.block;
  uint64_t left = iterations;
  int st;
  for (bool recovered = true; recovered;) {
    while (left) {
      const uint64_t step = std::min<uint64_t>(left, B - g.done % B);
      if ((st = queue_iterations(t, step, nullptr)) != LNT_OK) return st;
      g.done += step;
      left -= step;
      if (g.done % B != 0) continue;
      if ((st = gerbicz_check_carries(t, left, recovered)) != LNT_OK) return st;
      if (recovered) continue;
      // checkpoint: D_{k-1} kept, D_k = D_{k-1} * x
      lnt::StateBuf x = main_state(t);
      if ((st = copy_state(t, g.dprev, g.d)) != LNT_OK) return st;
      if ((st = mul_state(t, g.d, x)) != LNT_OK) return st;
      g.have_prev = true;
      if ((g.done / B) % B == 0) {
        const uint64_t before = g.done;
        bool ok = false;
        if ((st = gerbicz_verify(t, ok)) != LNT_OK) return st;
        if (!ok) left += before - g.done;  // redo what the failed block covered
      }
    }
    // no carry flag may reach the caller: a last look, and a redo if needed
    if ((st = gerbicz_check_carries(t, left, recovered)) != LNT_OK) return st;
  }
  return LNT_OK;
}

// ---- Jacobi check for LL tests (lnt_jacobi.cpp has the symbol) ----------
//
// Every `interval` squarings the residue's symbol (s - 2 | M_q) must be -1; a
// residue that passes becomes the verified one, a residue that fails (or a
// carry flag raised by the kernels) sends the test back to the last verified
// residue, and the squarings since are redone.

}  // namespace

namespace lnt {
struct Jacobi {
  uint64_t interval = 0;
  StateBuf ok;  // the last residue whose symbol was -1 (or the state when the check began)
  uint64_t done = 0, verified = 0, checks = 0, errors = 0;
  uint32_t failed_in_a_row = 0;
};
}  // namespace lnt

namespace {

void free_jacobi(lnt_test* t) {
  if (!t->jc) return;
  free_state(t->jc->ok);
  delete t->jc;
  t->jc = nullptr;
}

int save_state_buf(lnt_test* t, lnt::StateBuf& dst) {
  LNT_CUDA(cudaMemcpyAsync(dst.x, t->x, (size_t)t->n * 8, cudaMemcpyDeviceToDevice, t->stream), "copy state");
  if (carry_words(t))
    LNT_CUDA(cudaMemcpyAsync(dst.carry, t->carry, carry_words(t) * 8, cudaMemcpyDeviceToDevice, t->stream),
             "copy carries");
  dst.canonical_input = t->canonical_input;
  dst.pending_carries = t->pending_carries;
  dst.pristine = t->pristine;
  dst.zero_start = t->zero_start;
  return LNT_OK;
}

int load_state_buf(lnt_test* t, const lnt::StateBuf& src) {
  LNT_CUDA(cudaMemcpyAsync(t->x, src.x, (size_t)t->n * 8, cudaMemcpyDeviceToDevice, t->stream), "copy state");
  if (carry_words(t))
    LNT_CUDA(cudaMemcpyAsync(t->carry, src.carry, carry_words(t) * 8, cudaMemcpyDeviceToDevice, t->stream),
             "copy carries");
  t->canonical_input = src.canonical_input;
  t->pending_carries = src.pending_carries;
  t->pristine = src.pristine;
  t->zero_start = src.zero_start;
  t->canon_valid = false;
  return LNT_OK;
}

int jacobi_rebase(lnt_test* t) {
  lnt::Jacobi& j = *t->jc;
  const int st = save_state_buf(t, j.ok);
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  j.done = j.verified = 0;
  j.failed_in_a_row = 0;
  return st;
}

// The symbol (s - 2 | M_q) of the current residue; a raised carry flag counts
// as a failed check (symbol 0).
int jacobi_symbol(lnt_test* t, int& symbol) {
  uint32_t flags = 0;
  int st = read_status(t, flags);
  if (st != LNT_OK) return st;
  if (flags & lnt::kStatusCarryOverflow) {
    symbol = 0;
    return LNT_OK;
  }
  if ((st = canonicalize(t)) != LNT_OK) return st;
  std::vector<uint64_t> d(t->n);
  LNT_CUDA(cudaMemcpyAsync(d.data(), t->canon, (size_t)t->n * 8, cudaMemcpyDeviceToHost, t->stream),
           "download digits");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  std::string why;
  symbol = lnt::jacobi_of_ll_residue(d.data(), t->h_widths.data(), t->n, t->q, &why);
  if (symbol == 2) return fail(LNT_ERR_UNSUPPORTED_LENGTH, "Jacobi check: " + why);
  return LNT_OK;
}

int jacobi_iterate(lnt_test* t, uint64_t iterations) {
  lnt::Jacobi& j = *t->jc;
  uint64_t left = iterations;
  while (left) {
    const uint64_t step = std::min<uint64_t>(left, j.interval - j.done % j.interval);
    int st = queue_iterations(t, step, nullptr);
    if (st != LNT_OK) return st;
    j.done += step;
    left -= step;
    if (j.done % j.interval != 0) continue;
    int symbol = 0;
    if ((st = jacobi_symbol(t, symbol)) != LNT_OK) return st;
    if (symbol == -1) {
      if ((st = save_state_buf(t, j.ok)) != LNT_OK) return st;
      LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
      j.verified = j.done;
      j.failed_in_a_row = 0;
      ++j.checks;
      continue;
    }
    ++j.errors;
    if (++j.failed_in_a_row > kGerbiczRetries)
      return fail(LNT_ERR_NUMERIC, "Jacobi check: the same squarings failed " +
                                       std::to_string(kGerbiczRetries) + " times in a row");
    if ((st = load_state_buf(t, j.ok)) != LNT_OK) return st;
    LNT_CUDA(cudaMemsetAsync(t->status, 0, 4, t->stream), "clear status");
    LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
    left += j.done - j.verified;
    j.done = j.verified;
  }
  return LNT_OK;
}

}  // namespace

namespace lnt {
// Lets other translation units of the library report a failure detail.
void set_last_error(const std::string& msg) { g_last_error = msg; }

// ---- hooks for the batch engine (lnt_batch.cu) -----------------------------
const Plan& test_plan(const lnt_test* t) { return t->plan; }
int test_prp(const lnt_test* t) { return t->prp; }
const TwoPassDesc* test_twopass_device_desc(const lnt_test* t) { return t->tdesc; }
TwoPassDesc test_twopass_desc(const lnt_test* t) { return twopass_desc(t); }
bool test_ready_for_group(const lnt_test* t) {
  // batched two-pass launches assume the steady state: carries pending, signed outputs
  return t->plan.kind == PlanKind::Resident || (t->pending_carries && !t->canonical_input);
}
ResidentDesc test_resident_desc(const lnt_test* t, uint64_t iterations) {
  ResidentDesc d{};
  d.digits = t->x;
  d.w = t->w;
  d.uw = t->uw;
  d.widths = t->widths;
  d.rt = t->rt;
  d.irt = t->irt;
  d.status = t->status;
  d.n = t->n;
  d.log2n = t->plan.log2n;
  d.prp = (uint32_t)t->prp;
  d.unsigned_first = t->canonical_input ? 1 : 0;
  d.iterations = iterations;
  d.short_runs = r16_run_words_needed(t->q, t->n) <= 4 ? 1 : 0;
  return d;
}
// bookkeeping after squarings were launched outside lnt_iterate
void test_mark_iterated(lnt_test* t) {
  if (t->plan.kind == PlanKind::TwoPass) t->pending_carries = true;
  t->canonical_input = false;
  t->pristine = false;
  t->canon_valid = false;
}

// Device bytes lnt_create allocates for a test (the batch engine's budget unit).
uint64_t test_device_bytes(uint32_t n) {
  Plan plan;
  if (!make_plan(n, 0, nullptr, plan)) return 0;
  const uint64_t nb = n / canon_block_size(n);
  uint64_t b = 8ull * n * 4 + n + 4 + nb * 10 + 4;  // x, w, uw, canon, widths, status, readout
  if (plan.kind == PlanKind::Resident) {
    b += 8ull * n + sizeof(ResidentDesc);  // root tables
  } else {
    // carry buffer: one word per run, at most n / 4 runs (the narrowest tile)
    b += 16ull * n + 8ull * (plan.n1 + plan.n2) + 2ull * n + sizeof(TwoPassDesc) +
         4ull * (plan.n1 + 2);  // fused-kernel flags
    if (plan.fast) b += 16ull * (plan.n1 + plan.n2) + 17ull * n;  // inner twiddles, tile-major tables
    if (plan.five) b += 64ull * (plan.n1 / 5);                      // radix-5 twiddles
  }
  return b;
}
}  // namespace lnt

namespace {
lnt::PlanOptions from_abi(const lnt_plan_options& o) {
  lnt::PlanOptions p;
  p.kind = o.kind;
  p.log2_rows = o.log2_rows;
  p.tile = o.tile;
  p.radix = o.radix;
  p.fused = o.fused;
  return p;
}

lnt_plan_options to_abi(const lnt::PlanOptions& p) {
  return {p.kind, p.log2_rows, p.tile, p.radix, p.fused};
}
}  // namespace

extern "C" {

const char* lnt_status_string(int status) {
  switch (status) {
    case LNT_OK: return "ok";
    case LNT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case LNT_ERR_UNSUPPORTED_LENGTH: return "unsupported NTT length";
    case LNT_ERR_CUDA: return "CUDA error";
    case LNT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case LNT_ERR_NUMERIC: return "carry headroom exceeded";
    case LNT_ERR_NO_DEVICE: return "no CUDA device";
    case LNT_ERR_BUDGET: return "does not fit the memory budget";
    default: return "unknown status";
  }
}

const char* lnt_last_error(void) { return g_last_error.c_str(); }

int lnt_create(uint32_t exponent, uint32_t n, int prp, int device, lnt_test** out) {
  return lnt_create_with_plan(exponent, n, prp, device, nullptr, out);
}

int lnt_create_with_plan(uint32_t exponent, uint32_t n, int prp, int device,
                         const lnt_plan_options* options, lnt_test** out) {
  if (!out) return fail(LNT_ERR_INVALID_ARGUMENT, "null output pointer");
  *out = nullptr;
  if (exponent < 3) return fail(LNT_ERR_INVALID_ARGUMENT, "exponent must be >= 3");
  if (n == 0) {
    uint32_t l = lnt_secured_log2_length(exponent);
    if (l < 1 || l > lnt::kMaxLog2) return fail(LNT_ERR_UNSUPPORTED_LENGTH, "exponent out of range");
    n = 1u << l;
  }
  lnt::Plan plan;
  lnt::PlanOptions opt;
  if (options) opt = from_abi(*options);
  std::string why;
  if (!lnt::make_plan(n, exponent, &opt, plan, &why)) return fail(LNT_ERR_UNSUPPORTED_LENGTH, why);
  if (n > exponent) return fail(LNT_ERR_UNSUPPORTED_LENGTH, "length exceeds the exponent");
  if ((exponent + n - 1) / n > 30) return fail(LNT_ERR_UNSUPPORTED_LENGTH, "more than 30 bits per word");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(LNT_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= count) return fail(LNT_ERR_INVALID_ARGUMENT, "bad device index");
  DeviceGuard guard(device);

  lnt_test* t = new lnt_test();
  t->q = exponent;
  t->n = n;
  t->prp = prp ? 1 : 0;
  t->device = device;
  t->plan = plan;
  auto bail = [&](int st) {
    free_all(t);
    delete t;
    return st;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(cuda_fail(e, "cudaStreamCreate"));
  t->own_stream = true;

  // widths: ceil(q(j+1)/n) - ceil(qj/n), pre_calculation.cu:35 in exact integers
  t->h_widths.resize(n);
  lnt::word_widths(exponent, n, t->h_widths.data());

  const uint32_t cb = lnt::canon_block_size(n), nb = n / cb;
  if ((e = dalloc(&t->x, n)) || (e = dalloc(&t->w, n)) || (e = dalloc(&t->uw, n)) ||
      (e = dalloc(&t->widths, n)) || (e = dalloc(&t->status, 1)) || (e = dalloc(&t->canon, n)) ||
      (e = dalloc(&t->blk_carry, nb)) || (e = dalloc(&t->blk_fn, nb)) ||
      (e = dalloc(&t->blk_cin, nb)) || (e = dalloc(&t->cflags, 1)) ||
      (e = cudaMallocHost((void**)&t->h_pinned, 16)))
    return bail(cuda_fail(e, "allocate residue"));
  if ((e = cudaMemcpyAsync(t->widths, t->h_widths.data(), n, cudaMemcpyHostToDevice, t->stream)) ||
      (e = cudaMemsetAsync(t->status, 0, 4, t->stream)))
    return bail(cuda_fail(e, "upload widths"));
  if ((e = lnt::launch_weights(exponent, n, t->w, t->uw, t->stream)))
    return bail(cuda_fail(e, "weights"));

  int st;
  if (plan.kind == lnt::PlanKind::Resident) {
    if ((st = upload_roots(t, n, &t->rt, &t->irt, 8)) != LNT_OK) return bail(st);  // the resident kernel's passes
    if ((e = dalloc(&t->rdesc, 1))) return bail(cuda_fail(e, "allocate descriptor"));
  } else {
    if ((st = upload_roots(t, plan.n1, &t->rt1, &t->irt1)) != LNT_OK) return bail(st);
    if ((st = upload_roots(t, plan.n2, &t->rt2, &t->irt2)) != LNT_OK) return bail(st);
    if (plan.fast) {
      // pass tables of the row transform: n1 points, or L = n1 / 5 for each plane of a 5 * 2^k row
      const uint32_t row_points = plan.five ? plan.n1 / 5 : plan.n1;
      if ((st = upload_roots(t, row_points, &t->itw1, &t->iitw1, plan.radix)) != LNT_OK) return bail(st);
      if (plan.five &&
          ((e = dalloc(&t->tw5, 4 * (size_t)row_points)) || (e = dalloc(&t->itw5, 4 * (size_t)row_points)) ||
           (e = lnt::launch_five_twiddles(row_points, t->tw5, t->itw5, t->c5, t->stream))))
        return bail(cuda_fail(e, "radix-5 twiddles"));
      if ((st = upload_roots(t, plan.n2, &t->itw2, &t->iitw2, plan.radix)) != LNT_OK) return bail(st);
      if ((e = dalloc(&t->wt, n)) || (e = dalloc(&t->uwt, n)) || (e = dalloc(&t->widt, n)) ||
          (e = lnt::launch_tile_major(t->w, t->uw, t->widths, plan.n1, plan.n2, plan.tile, t->wt,
                                      t->uwt, t->widt, t->stream)))
        return bail(cuda_fail(e, "tile-major tables"));
    }
    if ((e = dalloc(&t->twf, n)) || (e = dalloc(&t->twi, n)) ||
        (e = dalloc(&t->carry, (size_t)plan.ntiles * plan.n2)) ||
        (e = dalloc(&t->fuse, (size_t)plan.ntiles + 2)) ||
        (e = cudaMemsetAsync(t->fuse, 0, ((size_t)plan.ntiles + 2) * 4, t->stream)))
      return bail(cuda_fail(e, "allocate twiddles"));
    if ((e = lnt::launch_twiddles(plan.n1, plan.n2, plan.log2n2, t->twf, t->twi, t->stream)))
      return bail(cuda_fail(e, "twiddles"));
    // the device copy of the descriptor, built once every buffer it names exists
    const lnt::TwoPassDesc hd = twopass_desc(t);
    const void* needed[] = {hd.x, hd.carry, hd.w, hd.uw, hd.widths, hd.twf, hd.twi, hd.rt1,
                            hd.irt1, hd.rt2, hd.irt2, hd.status};
    for (const void* ptr : needed)
      if (!ptr) return bail(fail(LNT_ERR_CUDA, "internal: descriptor built before its buffers"));
    if (plan.fast && (!hd.itw1 || !hd.iitw1 || !hd.itw2 || !hd.iitw2 || !hd.wt || !hd.uwt || !hd.widt ||
                      (plan.five && (!hd.tw5 || !hd.itw5))))
      return bail(fail(LNT_ERR_CUDA, "internal: descriptor built before its buffers"));
    if ((e = dalloc(&t->tdesc, 1)) ||
        (e = cudaMemcpyAsync(t->tdesc, &hd, sizeof(hd), cudaMemcpyHostToDevice, t->stream)) ||
        (e = cudaStreamSynchronize(t->stream)))
      return bail(cuda_fail(e, "descriptor"));
  }
  if ((e = cudaStreamSynchronize(t->stream))) return bail(cuda_fail(e, "initialize"));
  if ((st = lnt_init_test(t)) != LNT_OK) return bail(st);
  *out = t;
  return LNT_OK;
}

int lnt_destroy(lnt_test* t) {
  if (!t) return LNT_OK;
  DeviceGuard guard(t->device);
  if (t->stream) cudaStreamSynchronize(t->stream);
  free_all(t);
  delete t;
  return LNT_OK;
}

int lnt_init_test(lnt_test* t) {
  if (!t) return fail(LNT_ERR_INVALID_ARGUMENT, "null test");
  DeviceGuard guard(t->device);
  std::vector<uint64_t> d(t->n, 0);
  d[0] = t->prp ? 3 : 4;
  int st = upload_digits(t, d.data());
  if (st == LNT_OK && t->gz) st = gerbicz_rebase(t);
  if (st == LNT_OK && t->jc) st = jacobi_rebase(t);
  return st;
}

int lnt_set_digits(lnt_test* t, const uint64_t* digits, size_t n) {
  if (!t || !digits || n != t->n) return fail(LNT_ERR_INVALID_ARGUMENT, "digits/length mismatch");
  DeviceGuard guard(t->device);
  int st = upload_digits(t, digits);
  if (st == LNT_OK && t->gz) st = gerbicz_rebase(t);
  if (st == LNT_OK && t->jc) st = jacobi_rebase(t);
  return st;
}

int lnt_iterate(lnt_test* t, uint64_t iterations) {
  if (!t) return fail(LNT_ERR_INVALID_ARGUMENT, "null test");
  if (iterations == 0) return LNT_OK;
  DeviceGuard guard(t->device);
  if (t->gz) return gerbicz_iterate(t, iterations);
  if (t->jc) return jacobi_iterate(t, iterations);
  return queue_iterations(t, iterations, nullptr);
}

int lnt_jacobi_of_digits(const uint64_t* digits, const uint8_t* widths, uint32_t n, uint32_t exponent,
                         int* symbol) {
  if (!digits || !widths || !symbol || n == 0 || exponent < 3)
    return fail(LNT_ERR_INVALID_ARGUMENT, "null argument or bad size");
  std::string why;
  const int r = lnt::jacobi_of_ll_residue(digits, widths, n, exponent, &why);
  if (r == 2) return fail(LNT_ERR_UNSUPPORTED_LENGTH, "Jacobi symbol: " + why);
  *symbol = r;
  return LNT_OK;
}

int lnt_jacobi_check(lnt_test* t, int* symbol) {
  if (!t || !symbol) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  if (t->prp) return fail(LNT_ERR_INVALID_ARGUMENT, "the Jacobi check applies to LL tests");
  DeviceGuard guard(t->device);
  return jacobi_symbol(t, *symbol);
}

int lnt_jacobi_enable(lnt_test* t, uint64_t interval) {
  if (!t) return fail(LNT_ERR_INVALID_ARGUMENT, "null test");
  DeviceGuard guard(t->device);
  if (interval == 0) {
    free_jacobi(t);
    return LNT_OK;
  }
  if (t->prp) return fail(LNT_ERR_INVALID_ARGUMENT, "the Jacobi check applies to LL tests");
  std::string why;
  if (!lnt::jacobi_available(&why)) return fail(LNT_ERR_UNSUPPORTED_LENGTH, "Jacobi check: " + why);
  free_jacobi(t);
  t->jc = new lnt::Jacobi();
  t->jc->interval = interval;
  cudaError_t e = dalloc(&t->jc->ok.x, t->n);
  if (e == cudaSuccess && carry_words(t)) e = dalloc(&t->jc->ok.carry, carry_words(t));
  if (e != cudaSuccess) {
    free_jacobi(t);
    return cuda_fail(e, "allocate the Jacobi check's state");
  }
  const int st = jacobi_rebase(t);
  if (st != LNT_OK) free_jacobi(t);
  return st;
}

int lnt_jacobi_stats(lnt_test* t, uint64_t* verified_iterations, uint64_t* checks, uint64_t* errors) {
  if (!t || !t->jc) return fail(LNT_ERR_INVALID_ARGUMENT, "no Jacobi check on this test");
  if (verified_iterations) *verified_iterations = t->jc->verified;
  if (checks) *checks = t->jc->checks;
  if (errors) *errors = t->jc->errors;
  return LNT_OK;
}

int lnt_gerbicz_enable(lnt_test* t, uint32_t block) {
  if (!t) return fail(LNT_ERR_INVALID_ARGUMENT, "null test");
  DeviceGuard guard(t->device);
  if (block == 0) {
    free_gerbicz(t);
    return LNT_OK;
  }
  if (!t->prp) return fail(LNT_ERR_INVALID_ARGUMENT, "the Gerbicz check applies to PRP tests");
  if (block < 2) return fail(LNT_ERR_INVALID_ARGUMENT, "block must be >= 2");
  if (t->plan.kind != lnt::PlanKind::TwoPass || !t->plan.fast)
    return fail(LNT_ERR_UNSUPPORTED_LENGTH, "the Gerbicz check needs a two-pass register-pass plan (n >= 8192)");
  free_gerbicz(t);
  t->gz = new lnt::Gerbicz();
  lnt::Gerbicz& g = *t->gz;
  g.block = block;
  cudaError_t e = cudaSuccess;
  for (lnt::StateBuf* s : {&g.c0, &g.d, &g.dprev, &g.v, &g.xok, &g.dok, &g.f})
    if (e == cudaSuccess && ((e = dalloc(&s->x, t->n)) == cudaSuccess)) e = dalloc(&s->carry, carry_words(t));
  if (e == cudaSuccess) e = dalloc(&g.fdesc, 1);
  if (e != cudaSuccess) {
    free_gerbicz(t);
    return cuda_fail(e, "allocate Gerbicz states");
  }
  const int st = gerbicz_rebase(t);
  if (st != LNT_OK) free_gerbicz(t);
  return st;
}

int lnt_gerbicz_stats(lnt_test* t, uint64_t* verified_iterations, uint64_t* checks, uint64_t* errors) {
  if (!t || !t->gz) return fail(LNT_ERR_INVALID_ARGUMENT, "no Gerbicz check on this test");
  if (verified_iterations) *verified_iterations = t->gz->verified;
  if (checks) *checks = t->gz->checks;
  if (errors) *errors = t->gz->errors;
  return LNT_OK;
}

int lnt_debug_corrupt(lnt_test* t, uint32_t word) { return lnt_debug_corrupt_add(t, word, 1); }

int lnt_debug_corrupt_add(lnt_test* t, uint32_t word, int64_t delta) {
  if (!t || word >= t->n) return fail(LNT_ERR_INVALID_ARGUMENT, "word out of range");
  DeviceGuard guard(t->device);
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  int64_t v = 0;
  LNT_CUDA(cudaMemcpy(&v, t->x + word, 8, cudaMemcpyDeviceToHost), "read word");
  v += delta;
  LNT_CUDA(cudaMemcpyAsync(t->x + word, &v, 8, cudaMemcpyHostToDevice, t->stream), "write word");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  t->canon_valid = false;
  return LNT_OK;
}

int lnt_profile_iterations(lnt_test* t, uint64_t iterations, lnt_kernel_time* out, int cap,
                           int* count) {
  if (!t || !count || (cap > 0 && !out)) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  DeviceGuard guard(t->device);
  LaunchTimer timer;
  int st = queue_iterations(t, iterations, &timer);
  if (st != LNT_OK) return st;
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  std::vector<lnt_kernel_time> kinds;
  for (size_t i = 0; i < timer.kinds.size(); ++i) {
    float ms = 0;
    LNT_CUDA(cudaEventElapsedTime(&ms, timer.events[i], timer.events[i + 1]), "event time");
    auto it = std::find_if(kinds.begin(), kinds.end(), [&](const lnt_kernel_time& k) {
      return std::strcmp(k.name, timer.kinds[i]) == 0;
    });
    if (it == kinds.end()) {
      lnt_kernel_time k{};
      std::snprintf(k.name, sizeof(k.name), "%s", timer.kinds[i]);
      kinds.push_back(k);
      it = kinds.end() - 1;
    }
    it->launches++;
    it->total_ms += ms;
  }
  *count = (int)kinds.size();
  for (int i = 0; i < cap && i < (int)kinds.size(); ++i) out[i] = kinds[i];
  return check_status(t);
}

int lnt_get_digits(lnt_test* t, uint64_t* digits, size_t n) {
  if (!t || !digits || n != t->n) return fail(LNT_ERR_INVALID_ARGUMENT, "digits/length mismatch");
  DeviceGuard guard(t->device);
  int st = canonicalize(t);
  if (st != LNT_OK) return st;
  LNT_CUDA(cudaMemcpyAsync(digits, t->canon, (size_t)t->n * 8, cudaMemcpyDeviceToHost, t->stream),
           "download digits");
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  return LNT_OK;
}

int lnt_res64(lnt_test* t, uint64_t* res64) {
  if (!t || !res64) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  DeviceGuard guard(t->device);
  int st = canonicalize(t);
  if (st != LNT_OK) return st;
  uint64_t head[64];
  const uint32_t k = t->n < 64 ? t->n : 64;
  LNT_CUDA(cudaMemcpy(head, t->canon, k * 8, cudaMemcpyDeviceToHost), "download digits");
  uint64_t r = 0;
  uint32_t pos = 0;
  for (uint32_t j = 0; j < k && pos < 64; ++j) {
    r += head[j] << pos;
    pos += t->h_widths[j];
  }
  *res64 = r;
  return LNT_OK;
}

int lnt_is_prime(lnt_test* t, int* is_prime) {
  if (!t || !is_prime) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  DeviceGuard guard(t->device);
  std::vector<uint64_t> d(t->n);
  int st = lnt_get_digits(t, d.data(), d.size());
  if (st != LNT_OK) return st;
  bool prime = d[0] == (uint64_t)(t->prp ? 9 : 0);
  for (uint32_t j = 1; j < t->n && prime; ++j) prime = d[j] == 0;
  *is_prime = prime ? 1 : 0;
  return LNT_OK;
}

int lnt_get_raw_state(lnt_test* t, int64_t* words, size_t n) {
  if (!t || !words || n != t->n) return fail(LNT_ERR_INVALID_ARGUMENT, "words/length mismatch");
  DeviceGuard guard(t->device);
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  LNT_CUDA(cudaMemcpy(words, t->x, (size_t)t->n * 8, cudaMemcpyDeviceToHost), "download state");
  return LNT_OK;
}

int lnt_get_length(lnt_test* t, uint32_t* n) {
  if (!t || !n) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  *n = t->n;
  return LNT_OK;
}

int lnt_get_widths(lnt_test* t, uint8_t* widths, size_t n) {
  if (!t || !widths || n != t->n) return fail(LNT_ERR_INVALID_ARGUMENT, "widths/length mismatch");
  std::memcpy(widths, t->h_widths.data(), n);
  return LNT_OK;
}

int lnt_get_plan(lnt_test* t, lnt_plan_options* out) {
  if (!t || !out) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  const lnt::Plan& p = t->plan;
  out->kind = p.kind == lnt::PlanKind::Resident ? LNT_PLAN_RESIDENT
                                                : (p.fast ? LNT_PLAN_RADIX16 : LNT_PLAN_RADIX2);
  out->log2_rows = p.kind == lnt::PlanKind::Resident ? 0 : p.log2n2;
  out->tile = p.kind == lnt::PlanKind::Resident ? 0 : p.tile;
  out->radix = p.fast ? p.radix : 0;
  out->fused = p.fast ? (p.fused ? 1 : 2) : 0;
  return LNT_OK;
}

int lnt_plan_candidates(uint32_t exponent, uint32_t n, lnt_plan_options* out, int cap, int* count) {
  if (!count || (cap > 0 && !out)) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0) n = 1u << lnt_secured_log2_length(exponent);
  const std::vector<lnt::PlanOptions> c = lnt::plan_candidates(n, exponent);
  *count = (int)c.size();
  for (int i = 0; i < cap && i < (int)c.size(); ++i) out[i] = to_abi(c[i]);
  return c.empty() ? fail(LNT_ERR_UNSUPPORTED_LENGTH, "no plan for this length") : LNT_OK;
}

int lnt_plan_describe(const lnt_plan_options* o, uint32_t exponent, uint32_t n, char* out,
                      size_t outlen) {
  if (!o || !out || outlen == 0) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0) n = 1u << lnt_secured_log2_length(exponent);
  lnt::Plan plan;
  const lnt::PlanOptions opt = from_abi(*o);
  std::string why;
  if (!lnt::make_plan(n, exponent, &opt, plan, &why)) return fail(LNT_ERR_UNSUPPORTED_LENGTH, why);
  std::snprintf(out, outlen, "%s", plan.name.c_str());
  return LNT_OK;
}

// Process::GetBestPerformers (process.cu:45-127) over this library's plans:
// every candidate runs `loops` squarings after a short warm-up, timed with CUDA
// events on its stream; the fastest wins.
int lnt_time_plans(uint32_t exponent, uint32_t n, int prp, int device, uint32_t loops,
                   const lnt_plan_options* plans, int count, float* ms) {
  if ((count > 0 && (!plans || !ms)) || count < 0) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  if (loops == 0) return fail(LNT_ERR_INVALID_ARGUMENT, "loops must be > 0");
  if (n == 0) n = 1u << lnt_secured_log2_length(exponent);
  int ok = 0, last_status = LNT_ERR_UNSUPPORTED_LENGTH;
  for (int i = 0; i < count; ++i) {
    lnt_test* t = nullptr;
    float elapsed = -1;
    int st = lnt_create_with_plan(exponent, n, prp, device, &plans[i], &t);
    if (st == LNT_OK) {
      DeviceGuard guard(t->device);
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      // the warm-up is the timed call itself, untimed: it captures the CUDA
      // graphs and loads the kernels that call uses (the first candidate also
      // pays the per-device set-up there), so the timed call replays only
      if ((st = lnt_iterate(t, loops)) == LNT_OK && (st = lnt_synchronize(t)) == LNT_OK) {
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
            cudaEventRecord(e0, t->stream) != cudaSuccess)
          st = fail(LNT_ERR_CUDA, "autotune events");
        else if ((st = lnt_iterate(t, loops)) == LNT_OK &&
                 cudaEventRecord(e1, t->stream) == cudaSuccess &&
                 cudaEventSynchronize(e1) == cudaSuccess &&
                 (st = lnt_synchronize(t)) == LNT_OK)
          cudaEventElapsedTime(&elapsed, e0, e1);
      }
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      lnt_destroy(t);
    }
    if (st == LNT_ERR_NO_DEVICE || st == LNT_ERR_CUDA) return st;
    if (st != LNT_OK) last_status = st;
    ms[i] = st == LNT_OK ? elapsed : -1.0f;
    ok += st == LNT_OK;
  }
  return ok ? LNT_OK : last_status;
}

int lnt_autotune(uint32_t exponent, uint32_t n, int prp, int device, uint32_t loops,
                 lnt_plan_options* tried, float* ms, int cap, int* count, int* best) {
  if (!count || !best || (cap > 0 && (!tried || !ms))) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0) n = 1u << lnt_secured_log2_length(exponent);
  const std::vector<lnt::PlanOptions> c = lnt::plan_candidates(n, exponent);
  std::vector<lnt_plan_options> plans;
  for (const auto& o : c) plans.push_back(to_abi(o));
  std::vector<float> t(plans.size(), -1.0f);
  *count = (int)plans.size();
  *best = -1;
  const int st = lnt_time_plans(exponent, n, prp, device, loops, plans.data(), (int)plans.size(), t.data());
  for (size_t i = 0; i < plans.size(); ++i) {
    if ((int)i < cap) {
      tried[i] = plans[i];
      ms[i] = t[i];
    }
    if (t[i] >= 0 && (*best < 0 || t[i] < t[(size_t)*best])) *best = (int)i;
  }
  if (plans.empty()) return fail(LNT_ERR_UNSUPPORTED_LENGTH, "no plan for this length");
  return st;
}

// LucasPRP::DumpEnvironment (lucas_prp.cu:265-291): the same lines, for the
// host program, which has no CUDA headers of its own.
int lnt_environment(char* out, size_t outlen) {
  if (!out || outlen == 0) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  std::string s;
  char line[512];
  int rt = 0;
  cudaRuntimeGetVersion(&rt);
  std::snprintf(line, sizeof line, "CUDA Version = %d\n", rt);
  s += line;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) count = 0;
  std::snprintf(line, sizeof line, "CUDA devices = %d\n", count);
  s += line;
  const int kb = 1024, mb = kb * kb;
  for (int i = 0; i < count; ++i) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, i) != cudaSuccess) continue;
    std::snprintf(line, sizeof line, "Device %d = %s\n", i, p.name);
    s += line;
    std::snprintf(line, sizeof line, "  Revision = %d.%d\n", p.major, p.minor);
    s += line;
    std::snprintf(line, sizeof line, "  Multiprocessors = %d\n", p.multiProcessorCount);
    s += line;
    std::snprintf(line, sizeof line, "  Global memory (mb) = %d\n", (int)(p.totalGlobalMem / mb));
    s += line;
    std::snprintf(line, sizeof line, "  Shared memory (kb) = %d\n", (int)(p.sharedMemPerBlock / kb));
    s += line;
    std::snprintf(line, sizeof line, "  Constant memory (kb) = %d\n", (int)(p.totalConstMem / kb));
    s += line;
    std::snprintf(line, sizeof line, "  Block registers = %d\n", p.regsPerBlock);
    s += line;
    std::snprintf(line, sizeof line, "  Warp size = %d\n", p.warpSize);
    s += line;
    std::snprintf(line, sizeof line, "  Threads per block = %d\n", p.maxThreadsPerBlock);
    s += line;
    std::snprintf(line, sizeof line, "  Max block dimensions = [%d, %d, %d]\n", p.maxThreadsDim[0],
                  p.maxThreadsDim[1], p.maxThreadsDim[2]);
    s += line;
    std::snprintf(line, sizeof line, "  Max grid dimensions = [%d, %d, %d]\n", p.maxGridSize[0],
                  p.maxGridSize[1], p.maxGridSize[2]);
    s += line;
  }
  std::snprintf(out, outlen, "%s", s.c_str());
  return s.size() < outlen ? LNT_OK : fail(LNT_ERR_INVALID_ARGUMENT, "buffer too small");
}

int lnt_plan_name(lnt_test* t, char* out, size_t outlen) {
  if (!t || !out || outlen == 0) return fail(LNT_ERR_INVALID_ARGUMENT, "null argument");
  std::snprintf(out, outlen, "%s", t->plan.name.c_str());
  return LNT_OK;
}

int lnt_set_stream(lnt_test* t, void* cuda_stream) {
  if (!t) return fail(LNT_ERR_INVALID_ARGUMENT, "null test");
  DeviceGuard guard(t->device);
  LNT_CUDA(cudaStreamSynchronize(t->stream), "synchronize");
  if (cuda_stream) {
    if (t->own_stream) cudaStreamDestroy(t->stream);
    t->stream = (cudaStream_t)cuda_stream;
    t->own_stream = false;
  } else if (!t->own_stream) {
    LNT_CUDA(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    t->own_stream = true;
  }
  return LNT_OK;
}

int lnt_synchronize(lnt_test* t) {
  if (!t) return fail(LNT_ERR_INVALID_ARGUMENT, "null test");
  DeviceGuard guard(t->device);
  return check_status(t);
}

}  // extern "C"
