// Internal declarations of the LucasNTT B200 library: plan, kernel descriptors
// and launchers.  Nothing here is part of the C ABI (include/lucasntt.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

namespace lnt {

// Status bits a kernel may raise in its status word.
enum : uint32_t {
  kStatusCarryOverflow = 1u << 0,  // a run absorbed a carry above kAbsorbLimit
  kStatusCanonFallback = 1u << 1,  // canonical readout needs the host fallback
  kStatusFuseTimeout = 1u << 2,    // a carry-fused column CTA gave up waiting for its neighbour
};

// ---------------------------------------------------------------- plans ----
// How one squaring of an n-word residue is laid out on the GPU.  Replaces the
// reference's pool/length choice (kernel_pool.cu:17-142, lucas_prp.cu:36-70).
enum class PlanKind { Resident, TwoPass };

struct Plan {
  PlanKind kind = PlanKind::Resident;
  uint32_t n = 0, log2n = 0;
  // TwoPass: natural index j = j1 + n1 * j2 is stored row-major (row j2,
  // column j1).  Columns (stride n1, length n2) are transformed by the column
  // passes, rows (contiguous, length n1) by the row pass.
  uint32_t n1 = 0, n2 = 0, log2n1 = 0, log2n2 = 0;
  uint32_t tile = 0;    // columns per column-pass CTA = words per carry run
  uint32_t ntiles = 0;  // n1 / tile
  bool fast = false;    // register-pass kernels (lnt_radix16.cu) instead of radix-2
  uint32_t radix = 8;   // register-pass kernels: largest pass radix, 8 or 16
  // steady squarings use the carry-fused column kernel (col_inverse of one
  // squaring + col_forward of the next): from 2^19 words, where its tiles fill
  // the GPU (at n = 2^23: 244.6 us for the pair that takes 270.1 us as two
  // launches); below, where a squaring is latency-bound, two plain launches win
  bool fused = false;
  // n = 5 * 2^k: rows of n1 = 5 L words, each row transform a radix-5 step over
  // the words c + L j5 followed by an L-point NTT of each of the five planes
  // (register-pass plans only; log2n1 is then log2 L)
  bool five = false;
  std::string name;
};

// Largest length handled by the SMEM-resident single-CTA kernel.
constexpr uint32_t kResidentMaxLog2 = 12;
constexpr uint32_t kMaxLog2 = 26;  // (p - 1) / 192 holds 2^26: the largest IBDWT length

// Explicit choices for make_plan (the C ABI's lnt_plan_options); 0 = policy.
struct PlanOptions {
  uint32_t kind = 0;       // 0 policy, 1 resident, 2 two-pass register passes, 3 two-pass radix-2
  uint32_t log2_rows = 0;  // two-pass: log2 n2 (column length)
  uint32_t tile = 0;       // two-pass: words per carry run (4 or 8)
  uint32_t radix = 0;      // register passes: largest pass radix, 8 or 16
  uint32_t fused = 0;      // register passes: 1 carry-fused column kernel, 2 two plain launches
};

// The plan for an n-word residue of exponent q.  With opt == nullptr (or all
// zero) the policy chooses; otherwise every non-zero field is honoured or the
// call fails with the reason in *why.
// n = 5 * 2^k
bool five_length(uint32_t n);
bool make_plan(uint32_t n, uint32_t exponent, const PlanOptions* opt, Plan& plan,
               std::string* why = nullptr);
// Every valid explicit plan for (n, q): the autotuner's candidates.
std::vector<PlanOptions> plan_candidates(uint32_t n, uint32_t exponent);

// Digit widths ceil(q(j+1)/n) - ceil(qj/n) in exact integer arithmetic: word j
// starts at bit ceil(qj/n), the bit its IBDWT weight 2^(ceil(qj/n) - qj/n) assumes.
void word_widths(uint32_t exponent, uint32_t n, uint8_t* widths);
// The words j whose start bit in the reference's table (pre_calculation.cu:35, the
// same expression in double) is below ceil(qj/n): possible once q*j passes 2^53.
// Its widths of j - 1 and j are then swapped against these, its weights still
// assume the exact bit, and its squaring is not that of the number its digits hold.
std::vector<uint32_t> shifted_words(uint32_t exponent, uint32_t n);

// ------------------------------------------------------------ device ----
struct DeviceInfo {
  int sms = 0;                   // streaming multiprocessors
  int smem_per_sm = 0;           // shared memory per SM, bytes
  int smem_per_block_optin = 0;  // largest dynamic shared memory a CTA may ask for
};
// The current device's properties (queried once per device, then cached).
cudaError_t device_info(DeviceInfo& out);
// Its SM count (148 on B200 if the query fails).
uint32_t device_sms();

// ------------------------------------------------------ resident kernel ----
// One residue per CTA, state kept in shared memory for all iterations.
struct ResidentDesc {
  int64_t* digits;        // n words, natural order (balanced or canonical)
  const uint64_t* w;      // IBDWT weights
  const uint64_t* uw;     // unweights with 1/n folded in
  const uint8_t* widths;  // digit widths
  const uint64_t* rt;     // pass table of the length-n transform (smem_passes.cuh)
  const uint64_t* irt;    // and of its inverse
  uint32_t* status;
  uint32_t n, log2n;
  uint32_t prp;
  uint32_t unsigned_first;  // the first squaring reads its outputs as non-negative
  uint64_t iterations;      // squarings this CTA performs in the launch
  uint32_t short_runs;      // carry runs of 4 words suffice for this exponent (else 8)
};

size_t resident_smem_bytes(uint32_t n, uint32_t threads);
// threads per CTA: one per 4 words when the launch has fewer tests than the
// device has SMs (latency), one per 8 otherwise (throughput)
uint32_t resident_threads(uint32_t n, uint32_t count, uint32_t sms);
cudaError_t launch_resident(const ResidentDesc* d_descs, uint32_t count, uint32_t max_n,
                            cudaStream_t stream);

// ------------------------------------------------------ two-pass kernels ----
struct TwoPassDesc {
  int64_t* x;             // n words: digits, or the column-transformed residue
  int64_t* carry;         // pending run carries, index tile * n2 + row
  const uint64_t* w;
  const uint64_t* uw;
  const uint8_t* widths;
  const uint64_t* twf;    // 4-step twiddles omega_n^(j1 * brev(row)), n2 x n1
  const uint64_t* twi;    // their inverses
  const uint64_t* rt1;    // row roots omega_n1^k, k < n1/2
  const uint64_t* irt1;
  const uint64_t* rt2;    // column roots omega_n2^k, k < n2/2
  const uint64_t* irt2;
  // radix-16 kernels: inter-pass twiddles of the row (1) and column (2)
  // transforms, and their inverses.  Pass j of a length-L transform (span s_j,
  // radix R_j, q_j = s_j / R_j) owns s_j words at offset s_0 + ... + s_{j-1};
  // task t reads its R_j twiddles omega_L^(t brev(r) L / s_j) as one run.
  const uint64_t* itw1;
  const uint64_t* iitw1;
  const uint64_t* itw2;
  const uint64_t* iitw2;
  // radix-16 column kernels: w, uw, widths in tile-major order, index
  // (tile * n2 + row) * tile_width + column-in-tile, so a row's run is contiguous
  const uint64_t* wt;
  const uint64_t* uwt;
  const uint8_t* widt;
  uint32_t* status;
  // carry-fused column kernel: [0] ticket, [1] epoch, [2 + t] flag of tile t (zeroed at creation)
  uint32_t* fuse;
  uint32_t n1, n2, log2n1, log2n2, tile, ntiles;
  uint32_t prp;
  uint32_t radix;  // largest pass radix of the row and column transforms: 8 or 16
  // n = 5 * 2^k (five != 0): n1 = 5 L and log2n1 = log2 L.  tw5[(k5 - 1) L + c] =
  // omega_{5L}^(k5 c) for plane k5 = 1..4 and plane position c, itw5 its
  // inverse; c5 = the radix-5 constants (w + w^4)/2, (w^2 + w^3)/2, (w - w^4)/2,
  // (w^2 - w^3)/2 of w = omega_5 = omega_{5L}^L
  uint32_t five;
  const uint64_t* tw5;
  const uint64_t* itw5;
  uint64_t c5[4];
};

cudaError_t launch_col_forward(const TwoPassDesc& d, bool apply_carries, cudaStream_t s);
cudaError_t launch_row_square(const TwoPassDesc& d, cudaStream_t s);
cudaError_t launch_col_inverse(const TwoPassDesc& d, bool unsigned_mode, cudaStream_t s);

// register-pass kernels (lnt_radix16.cu, passes of radix up to 8 or 16): n2 in [2^6, 2^12],
// n1 in [2^7, 2^14], n1 >= n2
bool r16_supported(uint32_t log2n1, uint32_t log2n2);
// radices of the passes of a length-2^log2L transform whose passes take at most
// `radix` (8 or 16) points, first (largest span) first
std::vector<uint32_t> r16_pass_radices(uint32_t log2L, uint32_t radix);
uint32_t r16_tile(uint32_t log2n2);
uint32_t r16_run_words_needed(uint32_t exponent, uint32_t n);
// `d` gives the geometry (shared by every test of the launch); `dd` is a device
// array of `count` descriptors of tests with that geometry (blockIdx.y picks one).
cudaError_t launch_col_forward_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                   bool apply_carries, cudaStream_t s);
cudaError_t launch_row_square_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                  cudaStream_t s);
cudaError_t launch_col_inverse_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                   bool unsigned_mode, cudaStream_t s);
// product of two residues (one test each, count 1): row_forward_r16 turns a
// col_forward'ed residue into its full transform F (in place); row_mul_r16 is
// row_square_r16 with the square replaced by the pointwise product with F
cudaError_t launch_row_forward_r16(const TwoPassDesc& d, const TwoPassDesc* dd, cudaStream_t s);
cudaError_t launch_row_mul_r16(const TwoPassDesc& d, const TwoPassDesc* dd, const uint64_t* F,
                               cudaStream_t s);
// col_inverse of one squaring and col_forward of the next (steady state: carries
// pending, signed outputs) in one launch
cudaError_t launch_col_fused_r16(const TwoPassDesc& d, const TwoPassDesc* dd, uint32_t count,
                                 cudaStream_t s);

// ------------------------------------------------------------- tables ----
cudaError_t launch_weights(uint32_t exponent, uint32_t n, uint64_t* w, uint64_t* uw,
                           cudaStream_t s);
cudaError_t launch_twiddles(uint32_t n1, uint32_t n2, uint32_t log2n2, uint64_t* twf,
                            uint64_t* twi, cudaStream_t s);
// n = 5 * 2^k rows: the radix-5 step's twiddles for planes of L points (4 L words
// each) and its constants c5 (TwoPassDesc)
cudaError_t launch_five_twiddles(uint32_t L, uint64_t* tw5, uint64_t* itw5, uint64_t c5[4],
                                 cudaStream_t s);
cudaError_t launch_tile_major(const uint64_t* w, const uint64_t* uw, const uint8_t* widths,
                              uint32_t n1, uint32_t n2, uint32_t tile, uint64_t* wt, uint64_t* uwt,
                              uint8_t* widt, cudaStream_t s);

// --------------------------------------------------- canonical readout ----
struct CanonDesc {
  const int64_t* x;        // balanced digits
  const int64_t* carry;    // pending run carries or nullptr
  const uint8_t* widths;
  uint64_t* out;           // canonical non-negative digits
  int64_t* blk_carry;      // per block
  uint8_t* blk_fn;         // per block carry transfer function
  int8_t* blk_cin;         // per block resolved carry-in
  uint32_t* flags;         // kCanon* bits
  uint32_t n, block, nblocks;
  uint32_t n1, n2, tile, ntiles;  // run geometry when carry != nullptr
};

enum : uint32_t {
  kCanonNotAllMax = 1u << 0,
  kCanonHighNonZero = 1u << 1,  // some digit j >= 1 is non-zero
  kCanonError = 1u << 2,        // needs the host fallback
};

uint32_t canon_block_size(uint32_t n);
cudaError_t launch_canonicalize(const CanonDesc& d, cudaStream_t s);
cudaError_t launch_fill_max(uint64_t* out, const uint8_t* widths, uint32_t n, cudaStream_t s);

// ------------------------------------------- hooks for the batch engine ----
}  // namespace lnt

struct lnt_test;

namespace lnt {
const Plan& test_plan(const lnt_test* t);
int test_prp(const lnt_test* t);
const TwoPassDesc* test_twopass_device_desc(const lnt_test* t);
TwoPassDesc test_twopass_desc(const lnt_test* t);
bool test_ready_for_group(const lnt_test* t);
ResidentDesc test_resident_desc(const lnt_test* t, uint64_t iterations);
void test_mark_iterated(lnt_test* t);
uint64_t test_device_bytes(uint32_t n);
void set_last_error(const std::string& msg);
}  // namespace lnt
