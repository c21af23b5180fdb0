/*
 * lucasntt.h -- C ABI of the B200 LucasNTT squaring loop (liblucasntt.so).
 *
 * The reference LucasNTT program is a monolithic binary with no plugin or FFI;
 * its internal seam for this path is the Process interface
 * (process.cuh:16-35) implemented by LucasPRP (lucas_prp.cu) over a KernelPool
 * (kernel_pool.cu), with the length policy in NttLengths (ntt_lengths.cu).
 * Each entry point below names the reference function it replaces.
 *
 * Conventions: plain C types only; every call returns an lnt_status (0 = ok)
 * and never throws; the context owns its device memory.  Digits are the
 * reference's residue words: one uint64 per word, natural order, each word
 * d_j in [0, 2^w_j) with w_j = ceil(q(j+1)/n) - ceil(qj/n), exactly the vector
 * the reference dumps to LucasNTT_results.dat (lucas_prp.cu:254-263).  The
 * widths are exact integers; the reference's double-precision table differs from
 * them only at the words lnt_shifted_words lists (some q at n = 2^25, 2^26).
 */
#ifndef LUCASNTT_H
#define LUCASNTT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum lnt_status {
  LNT_OK = 0,
  LNT_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size or exponent */
  LNT_ERR_UNSUPPORTED_LENGTH = 2, /* n not a power of two in [2, 2^26] or n > q */
  LNT_ERR_CUDA = 3,             /* a CUDA call failed; see lnt_last_error() */
  LNT_ERR_OUT_OF_MEMORY = 4,    /* device allocation failed */
  LNT_ERR_NUMERIC = 5,          /* carry headroom exceeded: the residue is not trustworthy */
  LNT_ERR_NO_DEVICE = 6,        /* no CUDA device */
  LNT_ERR_BUDGET = 7            /* batch/serving: request does not fit the HBM budget */
} lnt_status;

typedef struct lnt_test lnt_test;

/* Text of a status code. */
const char* lnt_status_string(int status);

/* Detail of the last failure on the calling thread ("" if none). */
const char* lnt_last_error(void);

/* ---- length policy --------------------------------------------------------- */

/* NttLengths::GetNttSecuredLength (ntt_lengths.cu:88-98): log2 of the NTT
 * length the reference picks for exponent q. */
uint32_t lnt_secured_log2_length(uint32_t exponent);

/* NttLengths::GetCandidates (ntt_lengths.cu:100-128): writes the candidate
 * length strings, ';'-terminated, exactly as the reference spells them
 * ("8388608.000000;2048.000000:4096.000000;..."). Returns the count. */
int lnt_length_candidates(uint32_t exponent, char* out, size_t outlen);

/* NttLengths::StringToLengths + GetTotalLength (ntt_lengths.cu:32-75,
 * :130-142): total length of an "fft" description such as "4096", "8M",
 * "2048:4096".  Returns LNT_ERR_INVALID_ARGUMENT for lengths the reference
 * rejects (factors other than 2, 3, 5) and LNT_ERR_UNSUPPORTED_LENGTH for
 * totals other than 2^k and 5 * 2^k (the reference has no kernel for any
 * non-power-of-two total; this library runs 5 * 2^k, 13 <= k <= 24, on its
 * register-pass plan, and no IBDWT of length 3 * 2^k exists modulo p). */
int lnt_parse_length(const char* description, uint32_t* n_out);

/* The smallest length with a plan here that meets the reference's bound
 * 2n(2^W - 1)^2 < p, W = ceil(q/n) (ntt_lengths.cu:94), among 2^k and 5 * 2^k
 * (13 <= k <= 24).  Where it is 5 * 2^k it lies between 2^(k+2), which fails
 * the bound, and the reference's 2^(k+3): 37.5 % fewer words.  Otherwise it is
 * the power of two the reference picks. */
int lnt_smallest_length(uint32_t exponent, uint32_t* n_out);

/* NttLengths::CheckProvidedLength (ntt_lengths.cu:77-86): secured log2 length
 * minus log2 of the provided description (> 0: too small, < 0: larger than
 * needed).  Writes the difference to *diff. */
int lnt_check_provided_length(uint32_t exponent, const char* description, int* diff);

/* ---- one test ---------------------------------------------------------------- */

/* LucasPRP::LucasPRP + LucasPRP::Initialize (lucas_prp.cu:24-72, :82-111):
 * allocate the residue and its tables for exponent q on CUDA device `device`,
 * NTT length n (0 = the reference's policy), PRP (prp != 0) or Lucas-Lehmer,
 * and set the start value (InitializeTest, lucas_prp.cu:127-134). */
int lnt_create(uint32_t exponent, uint32_t n, int prp, int device, lnt_test** out);

/* ---- plans and autotuning ---------------------------------------------------
 * The reference picks, per run, the fastest of its candidate lengths, pools
 * and kernels by timing PerformanceLoops iterations of each
 * (Process::GetBestPerformers, process.cu:45-127; KernelPool, kernel_pool.cu:17-142;
 * LucasPRP::LucasPRP, lucas_prp.cu:36-70).  Here a plan is the kernel family,
 * the 4-step split, the column tile, the pass radix and the fusion depth of one
 * NTT length (the reference's kernel choice, butterflies per thread and
 * transpose tile, kernel.cu:157-192, :257-287). */
typedef enum lnt_plan_kind {
  LNT_PLAN_AUTO = 0,     /* the policy's choice */
  LNT_PLAN_RESIDENT = 1, /* n <= 4096: one CTA per residue, state in shared memory (FFT_1SMEM) */
  LNT_PLAN_RADIX16 = 2,  /* 4-step columns x rows, register passes of radix <= 16 (FFT_2SMEM family) */
  LNT_PLAN_RADIX2 = 3    /* 4-step columns x rows, radix-2 stages (the first kernels; an explicit plan) */
} lnt_plan_kind;

typedef struct lnt_plan_options {
  uint32_t kind;      /* lnt_plan_kind */
  uint32_t log2_rows; /* two-pass: log2 of the column length n2 (n = n2 x n1); 0 = policy */
  uint32_t tile;      /* two-pass: columns per column CTA = words per carry run, 4 or 8; 0 = policy */
  uint32_t radix;     /* LNT_PLAN_RADIX16: largest pass radix, 8 or 16; 0 = policy (8) */
  uint32_t fused;     /* LNT_PLAN_RADIX16: 1 = the inverse column pass of a squaring and the
                         forward one of the next in one carry-fused launch, 2 = two launches;
                         0 = policy (fused from 2^19 words) */
} lnt_plan_options;

/* lnt_create with an explicit plan (NULL = policy): the analogue of forcing
 * the reference's Pool / Kernels / fft options (LucasNTT.ini).  Returns
 * LNT_ERR_UNSUPPORTED_LENGTH with the reason in lnt_last_error() for a plan the
 * kernels cannot run, or whose carry runs are too short for the exponent. */
int lnt_create_with_plan(uint32_t exponent, uint32_t n, int prp, int device,
                         const lnt_plan_options* plan, lnt_test** out);

/* The plan a test runs. */
int lnt_get_plan(lnt_test* t, lnt_plan_options* out);

/* KernelFactory::GetCandidates analogue (kernel_factory.cu:45-141): every valid
 * plan for (q, n) (n = 0: policy length).  Writes min(count, cap) entries. */
int lnt_plan_candidates(uint32_t exponent, uint32_t n, lnt_plan_options* out, int cap, int* count);

/* Name of a plan ("TWOPASS_2048x4096_R8_T4": n2 x n1, pass radix, tile), the
 * stats file's Pool line. */
int lnt_plan_describe(const lnt_plan_options* plan, uint32_t exponent, uint32_t n, char* out,
                      size_t outlen);

/* Process::GetBestPerformers (process.cu:45-127): times `loops` squarings of
 * every candidate plan on `device` (as lnt_time_plans).  tried[i] / ms[i]
 * (ms = -1: the candidate failed) for i < min(count, cap); *best indexes the
 * fastest.  Allocates and frees one test at a time. */
int lnt_autotune(uint32_t exponent, uint32_t n, int prp, int device, uint32_t loops,
                 lnt_plan_options* tried, float* ms, int cap, int* count, int* best);

/* Process::EvaluatePerformance (process.cu:129-149) for a given list of plans:
 * ms[i] = time of `loops` squarings with plans[i], or -1 if it failed.  Each
 * plan runs `loops` squarings untimed first (graph capture, kernel loading),
 * then the same call timed. */
int lnt_time_plans(uint32_t exponent, uint32_t n, int prp, int device, uint32_t loops,
                   const lnt_plan_options* plans, int count, float* ms);

/* LucasPRP::Finalize + ~LucasPRP (lucas_prp.cu:113-125, :74-80). NULL is ok. */
int lnt_destroy(lnt_test* t);

/* LucasPRP::InitializeTest (lucas_prp.cu:127-134): residue := 4 (LL) or 3 (PRP). */
int lnt_init_test(lnt_test* t);

/* LucasPRP::MainLoop / OneIteration (lucas_prp.cu:197-229): `iterations`
 * squarings, each followed by minus two for LL.  Asynchronous on the test's
 * stream; errors raised by the kernels are reported by the next readout. */
int lnt_iterate(lnt_test* t, uint64_t iterations);

/* LucasPRP::LoadResidue (lucas_prp.cu:326-346): replace the residue with the
 * n digits at `digits` (host memory, natural order, as dumped). */
int lnt_set_digits(lnt_test* t, const uint64_t* digits, size_t n);

/* The device-to-host copy of lucas_prp.cu:164 + DumpResidue's word order
 * (lucas_prp.cu:254-263): write the residue's n digits to host memory. */
int lnt_get_digits(lnt_test* t, uint64_t* digits, size_t n);

/* Low 64 bits of the residue value sum d_j 2^ceil(qj/n) (Res64, derived from
 * the dumped digits; the reference prints no Res64 itself). */
int lnt_res64(lnt_test* t, uint64_t* res64);

/* Verdict of LucasPRP::Run (lucas_prp.cu:167-184): *is_prime = 1 when the
 * residue is 0 (LL) or 9 (PRP). Meaningful after the full test. */
int lnt_is_prime(lnt_test* t, int* is_prime);

/* ---- Gerbicz-Li error check (PRP) --------------------------------------------
 * No counterpart in the reference, which checks nothing during a test
 * (lucas_prp.cu:137-195).  For PRP tests on two-pass plans (n >= 8192):
 * every `block` squarings lnt_iterate folds the residue into a running
 * product D of checkpoint residues, and every block^2 squarings it verifies
 * D_k = x_0 * D_{k-1}^(2^block); on a mismatch, or when the kernels flag a
 * carry outside the balanced-digit headroom (which only corrupted data
 * produces), it returns to the last verified residue and redoes the work, so
 * the residues it returns are the error-free ones up to the last verification.
 * After 3 such recoveries in a row without a passed verification it returns
 * LNT_ERR_NUMERIC: the fault is not transient.  Costs about 2.5 squarings per block plus
 * `block` per block^2 (under 0.5 % at block = 1000) and 7 residue-sized
 * buffers.  lnt_set_digits / lnt_init_test restart the chain.
 * block = 0 turns the check off.  LNT_ERR_INVALID_ARGUMENT for LL tests,
 * LNT_ERR_UNSUPPORTED_LENGTH for the SMEM-resident and radix-2 plans. */
int lnt_gerbicz_enable(lnt_test* t, uint32_t block);

/* Squarings verified so far (since enable / the last set_digits), checks
 * passed and errors detected (each followed by a rollback). */
int lnt_gerbicz_stats(lnt_test* t, uint64_t* verified_iterations, uint64_t* checks, uint64_t* errors);

/* ---- Jacobi error check (LL) ------------------------------------------------
 * No counterpart in the reference (lucas_prp.cu:137-195 checks nothing).  For
 * an LL sequence u_0 = 4, u_{k+1} = u_k^2 - 2, the Jacobi symbol
 * (u_k - 2 | 2^q - 1) is -1 for every k >= 1; a residue whose symbol is not -1
 * is wrong (an error leaves it at -1 about half of the time).  The symbol of a
 * q-bit number needs GMP's subquadratic mpz_jacobi, loaded at run time from
 * libgmp.so.10: LNT_ERR_UNSUPPORTED_LENGTH when it is not installed.  A host
 * computation: seconds at q ~ 10^8, so checks belong at long intervals. */

/* (s - 2 | 2^exponent - 1) for the residue s given by canonical digits (the
 * dump order and widths of lnt_get_digits / lnt_get_widths): *symbol = -1, 0
 * or +1.  No GPU needed. */
int lnt_jacobi_of_digits(const uint64_t* digits, const uint8_t* widths, uint32_t n, uint32_t exponent,
                         int* symbol);

/* The symbol of a test's current residue (0 when the kernels flagged a carry
 * outside the balanced-digit headroom).  Valid from the first squaring after
 * lnt_init_test on: the start value 4 itself has symbol +1. */
int lnt_jacobi_check(lnt_test* t, int* symbol);

/* interval > 0: every `interval` squarings lnt_iterate checks the symbol; a
 * residue with symbol -1 becomes the verified one, any other (or a carry flag)
 * sends the test back to the last verified residue and the squarings since are
 * redone; after 3 failures in a row without a pass it returns LNT_ERR_NUMERIC.
 * Assumes the residue is an LL term u_k with k >= 1 at every check (tests
 * started by lnt_init_test, or resumed from such a residue).  One residue-sized
 * buffer.  interval = 0 turns it off; LNT_ERR_INVALID_ARGUMENT for PRP tests. */
int lnt_jacobi_enable(lnt_test* t, uint64_t interval);

/* Squarings verified, checks passed and errors detected (each followed by a
 * rollback) since enable / the last set_digits. */
int lnt_jacobi_stats(lnt_test* t, uint64_t* verified_iterations, uint64_t* checks, uint64_t* errors);

/* Diagnostic without a reference counterpart, for tests of the check: adds 1
 * to word `word` of the device state, as a hardware error would corrupt it. */
int lnt_debug_corrupt(lnt_test* t, uint32_t word);

/* The same with any amount: a large `delta` (say 2^40) makes the next squarings
 * raise the kernels' carry flag, which the check also treats as an error. */
int lnt_debug_corrupt_add(lnt_test* t, uint32_t word, int64_t delta);

/* Length, widths (n bytes: ceil(q(j+1)/n) - ceil(qj/n), pre_calculation.cu:35
 * in exact integers) and plan name of a test. */
int lnt_get_length(lnt_test* t, uint32_t* n);
int lnt_get_widths(lnt_test* t, uint8_t* widths, size_t n);
int lnt_plan_name(lnt_test* t, char* out, size_t outlen);

/* Words j where the reference's widths differ from this library's.  The
 * reference evaluates ceil(q(j+1)/n) - ceil(qj/n) in double
 * (pre_calculation.cu:35); once q*j passes 2^53 (n = 2^25 and 2^26) the double
 * ceil(qj/n) can land one bit low, so word j starts one bit below the bit its
 * weight (pre_calculation.cu:30-31) assumes and the reference's squaring is not
 * that of the number its digits hold: its LL/PRP residues for such (q, n) are not
 * those of M_q.  This library uses the exact integers (the widths of j - 1 and j
 * are swapped against the reference's).  *count = how many such j, *first = the
 * lowest (0 if none; `first` may be NULL).  Host only, no device. */
int lnt_shifted_words(uint32_t exponent, uint32_t n, uint32_t* count, uint32_t* first);

/* LucasPRP::DumpEnvironment (lucas_prp.cu:265-291): the text of the
 * reference's .env file (CUDA version, devices and their properties). */
int lnt_environment(char* out, size_t outlen);

/* Self-test without a reference counterpart: the device modular arithmetic
 * (multiply, add, subtract, power-of-two shifts, digit products) on edge and
 * seeded random operands, each result compared with the host implementation.
 * LNT_ERR_NUMERIC (first mismatch in lnt_last_error) if any differs. */
int lnt_arith_selftest(int device, uint64_t* checked, uint64_t* mismatches);

/* Run the test's work on a caller-owned cudaStream_t (NULL = the test's own
 * stream), the analogue of common::stream (common/common.cu:118). */
int lnt_set_stream(lnt_test* t, void* cuda_stream);

/* Wait for queued work; reports kernel-raised errors (LNT_ERR_NUMERIC). */
int lnt_synchronize(lnt_test* t);

/* Diagnostic without a reference counterpart: the internal representation,
 * n signed words (balanced digits, or the reference's digits right after a
 * set), before pending carries are applied and before canonicalisation. */
int lnt_get_raw_state(lnt_test* t, int64_t* words, size_t n);

/* Per-kernel device time of a run of squarings. */
typedef struct lnt_kernel_time {
  char name[32];     /* kernel kind, e.g. "col_forward" */
  uint32_t launches; /* launches of that kind */
  float total_ms;    /* summed CUDA-event time of those launches */
} lnt_kernel_time;

/* Process::EvaluatePerformance (process.cu:133-149), which times a candidate
 * with cudaEvents: performs `iterations` squarings exactly as lnt_iterate, with
 * a CUDA event recorded on the test's stream between consecutive kernel
 * launches, then waits and writes up to `cap` per-kind totals to `out`
 * (count in *count).  The residue advances as with lnt_iterate. */
int lnt_profile_iterations(lnt_test* t, uint64_t iterations, lnt_kernel_time* out, int cap,
                           int* count);

/* ---- batches of tests ------------------------------------------------------ */

/* The reference runs one exponent per process (main_process.cu:64-149); per
 * test it is LucasPRP (lucas_prp.cu:24-229).  A batch runs many independent
 * LL / PRP tests of mixed lengths on one GPU: tests of a length share batched
 * launches, tests are admitted against an HBM budget and retired as they
 * finish (continuous batching).  Results are bit-identical to running each
 * test alone. */
typedef struct lnt_batch lnt_batch;

typedef struct lnt_batch_result {
  uint64_t id;         /* as returned by lnt_batch_submit */
  uint64_t iterations; /* squarings performed */
  uint64_t res64;      /* Res64 of the final residue */
  double seconds;      /* submission to completion, host clock */
  uint32_t exponent;
  uint32_t n;
  int prp;
  int is_prime;        /* residue 0 (LL) / 9 (PRP): meaningful for full tests */
  int status;          /* LNT_OK, or the readout's error */
} lnt_batch_result;

/* Device bytes one test of exponent q at length n (0 = policy) occupies. */
uint64_t lnt_test_device_bytes(uint32_t exponent, uint32_t n);

/* hbm_budget_bytes = 0: no budget. */
int lnt_batch_create(int device, uint64_t hbm_budget_bytes, lnt_batch** out);
int lnt_batch_destroy(lnt_batch* b);

/* Admit a test (n = 0: policy length; iterations = 0: the full test, q - 2
 * squarings for LL and q for PRP as lucas_prp.cu:167).  LNT_ERR_BUDGET when it
 * does not fit the budget now. */
int lnt_batch_submit(lnt_batch* b, uint32_t exponent, uint32_t n, int prp, uint64_t iterations,
                     uint64_t* id);

/* Like lnt_batch_submit, but a test that does not fit the budget now waits in
 * a queue and is admitted (first fit) as soon as retired tests free memory;
 * its result's `seconds` count from this call.  LNT_ERR_BUDGET only for a
 * test larger than the whole budget. */
int lnt_batch_enqueue(lnt_batch* b, uint32_t exponent, uint32_t n, int prp, uint64_t iterations,
                      uint64_t* id);

/* Advance every admitted test by up to `iterations` squarings (none passes its
 * own count); finished tests are retired into the result queue and queued
 * tests admitted. */
int lnt_batch_run(lnt_batch* b, uint64_t iterations);

/* seconds > 0: each lnt_batch_run call gives every launch group (tests of one
 * geometry) and every resident test as many squarings, up to `iterations`, as
 * fit in about `seconds` at its measured pace, so a call takes about that long
 * and small tests are not held to the pace of large ones (the serving loop's
 * iteration-level scheduling); 0 (default): every test advances by the same
 * count.  Results do not depend on it. */
int lnt_batch_step_seconds(lnt_batch* b, double seconds);

/* Move up to `cap` finished results to `out` (count in *count). */
int lnt_batch_poll(lnt_batch* b, lnt_batch_result* out, int cap, int* count);

/* Tests in flight and device bytes they hold; tests waiting in the queue. */
int lnt_batch_status(lnt_batch* b, uint32_t* active, uint64_t* bytes_in_use);
int lnt_batch_pending(lnt_batch* b, uint32_t* pending);

/* loops > 0: the plan of every length admitted from now on is chosen by
 * lnt_autotune with `loops` squarings per candidate, once per length (and
 * carry-run class) for the batch's lifetime; 0 (default): policy plans. */
int lnt_batch_autotune(lnt_batch* b, uint32_t loops);

/* tests > 1: the autotuner times each candidate plan on `tests` copies of the
 * test advancing together in a scratch batch (the batched launches the real
 * groups run) instead of one test alone; 1 (default): alone. */
int lnt_batch_autotune_group(lnt_batch* b, uint32_t tests);

/* enable != 0 (default): grouped squarings replay a captured CUDA graph of
 * 8 squarings of every group; 0: plain stream launches. */
int lnt_batch_use_graphs(lnt_batch* b, int enable);

/* enable != 0: requests with n = 0 take lnt_smallest_length (5 * 2^k where that
 * meets the bound, 37.5 % fewer words) instead of the reference's power of two
 * (the default).  Residues do not depend on the length. */
int lnt_batch_short_lengths(lnt_batch* b, int enable);

/* Per-test Res64 checkpoints (no counterpart in the reference, which reports
 * Res64 only at the end of a run, lucas_prp.cu:254-263, so its intermediate
 * residues come from separate runs of k iterations): with every > 0 each test
 * records the Res64 of its residue whenever its squaring count reaches a
 * multiple of `every` below its target; 0 (default) turns this off.  Batched
 * launches stop at the checkpoints, so they cost one readout per test each. */
typedef struct lnt_batch_checkpoint {
  uint64_t id;        /* as returned by lnt_batch_submit / lnt_batch_enqueue */
  uint64_t iteration; /* squarings performed when the Res64 was taken */
  uint64_t res64;
  int status;         /* LNT_OK, or the readout's error */
} lnt_batch_checkpoint;
int lnt_batch_checkpoint_every(lnt_batch* b, uint64_t every);
/* Move up to `cap` recorded checkpoints to `out` (count in *count). */
int lnt_batch_poll_checkpoints(lnt_batch* b, lnt_batch_checkpoint* out, int cap, int* count);

/* Autotuned plans cached in a JSON file (the analogue of the reference's
 * per-run autotune summary, main_process.cu:160-190, kept across runs): plans
 * in `path` measured on a GPU of this device's name are used instead of timing
 * again, and every plan the batch tunes from now on is written back.  Takes
 * effect with lnt_batch_autotune(b, loops > 0).  NULL turns the cache off. */
int lnt_batch_plan_cache(lnt_batch* b, const char* path);

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory when they need a residue in the reference's digit format (a serving
 * process whose HBM is all handed to its own pool or budget, a latency-critical
 * step that must not pay cudaMalloc's implicit device synchronisation, a
 * checkpoint written by a path that must not allocate): turns n signed words
 * `words` (widths `widths`) into the reference's canonical digits, written to
 * `digits`.  The words must be the whole residue: any digits, balanced or
 * non-negative, whose weighted sum is the value, with no carry pending
 * elsewhere (lnt_get_raw_state of a RESIDENT-plan test qualifies; that of a
 * two-pass test does not, since its run carries are held apart).  All three are
 * DEVICE pointers owned by the caller; nothing is allocated.  The scratch lives
 * in one library-owned array of device memory sized for n <= 2^24 (about
 * 2.5 MiB, held by every GPU that loads the library until exit); larger n is
 * rejected with LNT_ERR_INVALID_ARGUMENT.  prp / zero_start select the
 * reference's representation of 0 mod M (LL: 0; PRP: M unless the test started
 * from zero).  The first call on a device sets up the scratch address, so make
 * it before any stream capture; a device reset invalidates that address (do not
 * call this after cudaDeviceReset).  Every call shares the one array: calls
 * that overlap on the GPU (other streams, other threads) race.  Runs on
 * `cuda_stream` (NULL = legacy default stream; a stream must belong to the
 * current device, else LNT_ERR_INVALID_ARGUMENT) and returns after it
 * finished.  LNT_ERR_NUMERIC: the words were too far from normalised digits
 * (a carry that does not settle within one block of 64 words); `digits` is
 * then undefined, although lnt_get_digits of a test may still read such words
 * (it falls back to an exact carry on the host). */
int lnt_canonicalize_noalloc(const int64_t* words, const uint8_t* widths, uint32_t n, int prp,
                             int zero_start, uint64_t* digits, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* LUCASNTT_H */
