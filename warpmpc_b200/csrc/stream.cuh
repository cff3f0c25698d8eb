// Streaming (TMA-fed) persistent OSQP path: host-built schedule tables and
// the device helpers shared by its kernels.
//
// Per instance tile (32 instances, one per lane) the LDL^T factor is stored
// twice, each copy in the order one sweep reads it: a forward stream (rows in
// order, a row's entries by ascending column) and a backward stream (columns
// in reverse order of use, a column's entries by ascending row, then D^-1 of
// the chunk's columns).  Both are cut into chunks; every chunk is one
// contiguous bulk copy (cp.async.bulk) into a shared-memory ring stage.
//
// ADMM state (x or z, y) and parameters (q or l, u) are stored per tile as
// records per (index, lane) -- the iterates, written every iteration, and the
// parameters, only read; 4 bytes for a primal index, 8 for a constraint --
// in "release order" U: the order in which
// the backward sweep finishes with a KKT index (after the smallest column
// whose correction reads it), so each chunk of the backward sweep updates one
// contiguous U range.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace wmpc {

// Sweeps run over "units" of 4 L entries of one row (forward) or one column
// (backward), stored per tile as [unit][lane][4] floats (512 bytes).  Unit
// meta (8 int32 words): byte offsets (row * 128) of the 4 work-vector rows the
// slots read; the target row's byte offset (read: right-hand side / x_j);
// flags | D^-1 byte offset << kUnitDoffShift (backward; relative to the
// stage's L area); the unit's L byte offset in the stage; the byte offset the
// result is stored to (the target on a row's / column's last unit, the trash
// row n + 1 otherwise).
constexpr int kUnitFirst = 1;  // first unit of its row/column: start the sum
constexpr int kUnitLast = 2;   // last unit: the stored result is final
constexpr int kUnitFwd = 4;    // the forwarding slot (3 forward, 0 backward) reads the previous unit's result
constexpr int kUnitDoffShift = 8;
constexpr int kUnitWords = 8;
constexpr int kUnitGroup = 3;      // units computed per loop trip
constexpr int kUnitSentinels = 4;  // sentinel units after a chunk's last unit
constexpr int kChunkHeader = 8;
// Backward chunk meta block (int32 words, 16-byte padded):
//   [0] nunits [1] ncols [2] nrel [3] c0 [4] u0 [5] nprim [6..7] 0
//   units (8 words each), then kUnitSentinels sentinel units
//   one record per release (4 words: byte offset of the released row, rho and
//   rho^-1 float bits, the index's unscale factor); the nprim primal indices first
// Forward chunk meta block: [0] nunits [1..7] 0, units, sentinels.
// Stage L area: units (512 B each), then D^-1 of the chunk's columns (128 B each).
// Work vector rows: 0..n-1 the KKT indices, n a zero row, n + 1 a trash row.
// Frontier form (frontier_slots > 0): the work vector rows are slots (zero
// slot frontier_slots, trash slot + 1); a forward header carries its rows
// [r0, r1) in words 1-2 and in word 3 the number of (stage offset, slot
// offset) copy pairs after the sentinels, and its stage the rows' right-hand
// sides after the units; a backward stage carries its columns' forward results after the
// D^-1 rows; unit targets are stage offsets and release records carry the
// released index in word 3.

struct StreamPlan {
  int n;              // KKT dimension
  int nnz_l;
  // forward sweep (row-gather form)
  int n_fchunks, flen, max_funits, max_fmeta_words;
  const int* fchunk_off;    // [n_fchunks + 1] float offset (lane 0) in the forward stream
  const int* fchunk_units;  // [n_fchunks]
  const int* fmeta_off;     // [n_fchunks]
  const int* fmeta_words;   // [n_fchunks]
  const int* fmeta;
  // backward sweep (column form) + releases
  int n_chunks, blen, max_units, max_cols, max_rel, max_meta_words;
  int max_meta_lead;        // backward meta words before the release records (the last 4 nrel words), at most
  const int* chunk_off;     // [n_chunks + 1] float offset (lane 0) in the backward stream
  const int* chunk_units;   // [n_chunks]
  const int* chunk_cols;    // [n_chunks]
  const int* chunk_u0;      // [n_chunks] first U index released
  const int* chunk_nrel;    // [n_chunks]
  const int* chunk_nprim;   // [n_chunks] primal releases (the chunk's first)
  const int* chunk_pre_u0;     // [n_chunks] stage position of the releaser's forward units
  const int* chunk_pre_units;  // [n_chunks] their count (copied in the first-right-hand-side pass too)
  const int* meta_off;      // [n_chunks]
  const int* meta_words;    // [n_chunks]
  const int* meta;
  // factorization (compact accumulator) tables and stream offsets
  const int* init_slot;     // [init_ptr[n]] slot of each init row in reach(k)
  const int* upd_ptr;       // [nnz_l + 1]
  const int* upd_slot;      // [upd_ptr[nnz_l]]
  const int* col_uoff;      // [n] backward-stream float offset of column c's first unit
  const int* dinv_off;      // [n] backward-stream float offset of D^-1_c (lane stride 1)
  const int* proc_boff;     // [nnz_l] backward-stream float offset of the entry each program step writes
  const int* proc_foff;     // [nnz_l] forward-stream float offset of that entry
  const int* upd_pos;       // [upd_ptr[nnz_l]] backward-stream float offset of the L entry each update reads
  const int* step_doff;     // [nnz_l] backward-stream float offset of D^-1 of each program step's column
  int max_row_kv;           // KKT values a factor row reads (diagonal + init entries), at most
  const int* pad_boff;      // [n_pad_b] padding slots (L = 0) of the backward stream
  const int* pad_foff;      // [n_pad_f] padding slots of the forward stream
  int n_pad_b, n_pad_f;
  // release order
  const int* u_perm;        // [n] U index -> permuted KKT index
  const int* u_orig;        // [n] U index -> original KKT index
  int max_row_nnz;
  int max_lstages, max_sstages;  // ring depth limits (tuning; defaults 12 and 6)
  // frontier form: slots (0: the plain form), the release lag the slots
  // assume (the L ring may be no deeper), the longest forward chunk in rows
  int frontier_slots, frontier_lag, max_frows;
  const int* chunk_c0;  // [n_chunks] first column of a backward chunk (its forward-result block)
  const int* frow0;     // [n_fchunks] first row of a forward chunk (its right-hand-side block)
  const int* frows;     // [n_fchunks] its rows
  // frontier form with termination checks: the unscale factor of each
  // permuted KKT index (the plain form's records carry it in their last word)
  const float* unscale_perm;  // [n]
  // factorization rows read ahead: per row {p0, p1, i0, i1} (program steps,
  // initial entries), {ub, uend, doff, kin base} (updates, D^-1 offset,
  // first KKT input descriptor of the row in Osqp::kin_desc)
  const int4* row_info;  // [2 n]
  // rho class of each U index's constraint (-1 loose, 0 inequality, 1
  // equality; 0 for primal indices): per-instance rho, when it adapts
  const int* u_cls;  // [n] (null: the problem has no rho classes)
};

// ---- PTX helpers -----------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait that may suspend the thread until the phase completes (or the
// hinted time passes), instead of returning at once.
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up (returns false) after `limit_ns` or when *abort is set.
// Waiting threads are suspended in the barrier between checks.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int* abort,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t start = global_timer_ns();
  // suspend for at most 20 us between checks, or the whole limit when shorter
  const uint32_t hint = limit_ns < 20000ull ? (uint32_t)limit_ns : 20000u;
  for (;;) {
    if (mbar_try_wait_suspend(bar, parity, hint)) return true;
    if (abort && *abort) return false;
    if (global_timer_ns() - start > limit_ns) return false;
  }
}

// Bulk copy global -> this CTA's shared memory, completion on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Shared-memory counters between warps of one CTA: release store / acquire load.
__device__ __forceinline__ void st_release_cta(unsigned* p, unsigned v) {
  asm volatile("st.release.cta.shared.u32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire_cta(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.cta.shared.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}

// Bounded wait until *ctr >= target: gives up (false) after `limit_ns` or
// when *abort is set.  Polls with a short sleep so that a waiting warp does
// not compete for the shared-memory pipe.
__device__ __forceinline__ bool wait_counter_bounded(const unsigned* ctr, unsigned target, const volatile int* abort,
                                                     uint64_t limit_ns) {
  if (ld_acquire_cta(ctr) >= target) return true;
  const uint64_t start = global_timer_ns();
  for (uint32_t it = 1;; ++it) {
    __nanosleep(64);
    if (ld_acquire_cta(ctr) >= target) return true;
    if ((it & 63u) == 0) {
      if (abort && *abort) return false;
      if (global_timer_ns() - start > limit_ns) return false;
    }
  }
}

// 4-byte asynchronous global -> shared copy (this thread's), and the wait for
// all of this thread's outstanding copies.
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// wait until at most N of this thread's committed cp.async groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_mbarrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Build the schedule on the host from the ragged pattern (called once per
// plan).  Returns false (and sets *why) when the pattern cannot use the
// streaming path.
struct HostPattern {
  int n, nnz_a, nnz_l;
  std::vector<int> init_ptr, init_rows, proc_ptr, proc_cols, proc_offsets, proc_lidx, lp, li, p;
};

struct StreamTargets {
  // chunk targets: 24-unit chunks are the largest whose ring still lets two
  // frontier-form CTAs share an SM on the quadrotor pattern, and measured
  // fastest there (59.8 ms per ADMM launch at 65,536 instances against 62.9
  // with 16) and chosen by the tuner for every benchmarked class
  int units = 24, cols = 24, rel = 16;  // backward chunks
  int funits = 24;                      // forward chunks
  int offload = 0;                      // also give the releaser warp: 1 leaf columns, 2 pre rows (bits)
  int frontier = 0;                     // frontier slots (see build_frontier_slots); needs offload 0
  int frontier_lag = 4;                 // chunks a release may trail the sweep (bounds the L ring depth)
  int frontier_copies = 0;              // frontier: rows without entries copied into slots, not swept as units
};

// Host result: every array of StreamPlan, to be uploaded by the plan.
struct HostStream {
  int n_chunks = 0, blen = 0, max_units = 0, max_cols = 0, max_rel = 0, max_meta_words = 0;
  int max_meta_lead = 0;  // backward meta words before the release records, at most
  std::vector<int> chunk_off, chunk_units, chunk_cols, chunk_u0, chunk_nrel, meta_off, meta_words, meta;
  std::vector<int> chunk_pre_u0, chunk_pre_units;
  int n_fchunks = 0, flen = 0, max_funits = 0, max_fmeta_words = 0;
  std::vector<int> fchunk_off, fchunk_units, fmeta_off, fmeta_words, fmeta;
  std::vector<int> col_uoff, dinv_off, proc_boff, proc_foff, pad_boff, pad_foff, upd_pos, step_doff;
  int max_row_kv = 0;
  std::vector<int> u_perm, u_orig;
  int dummy_units = 0;
  // frontier mode: work-vector slots (zero slot = frontier_slots, trash slot
  // + 1), the release lag the slot reservations assume, the longest forward
  // chunk in rows (its right-hand-side block in the stage)
  int frontier_slots = 0, frontier_lag = 0, max_frows = 0;
  std::vector<int> chunk_c0, frow0, frows;  // first column of a backward chunk; first row, rows of a forward chunk
  // host copies used by the OSQP side to lay out the state
  std::vector<int> u_of_perm;  // permuted index -> U index
};

// unscale_by_index (optional, original KKT order): the factor turning a scaled
// iterate change into an unscaled one (D_j for a primal index, max(E^-1, E/c)
// for a constraint), kept in the release records for early termination.
bool build_stream_schedule(const HostPattern& hp, const StreamTargets& t, const float* rho_by_constraint,
                           const float* rhoinv_by_constraint, int n_primal, HostStream* out, std::string* why,
                           const float* unscale_by_index = nullptr);
bool build_factor_tables(const HostPattern& hp, std::vector<int>* init_slot, std::vector<int>* upd_ptr,
                         std::vector<unsigned short>* upd_slot, int* max_row_nnz, std::string* why);

struct StreamLaunch {
  int stages, sstages, meta_bytes, lbytes, sbytes, pres_off;
  size_t smem;
};
bool stream_launch_config(const StreamPlan& sp, StreamLaunch* cfg);
// most CTAs of a fixed-iteration launch of this plan that fit one SM of `device`
// (within the launch limit: 2 unless WMPC_STREAM_MAX_CTAS allows up to 4)
// (track: a launch that checks termination, whose S stages also carry residuals)
int stream_max_ctas(const StreamPlan& sp, int device, int limit, bool track = false);
// the CTAs-per-SM limit of the environment (WMPC_STREAM_CTAS=1: one;
// WMPC_STREAM_MAX_CTAS: 2 to 4; default 2), fixed per problem at creation
int stream_ctas_limit_setting();
// CTAs per SM a fixed-iteration launch of `tiles` tiles of this plan runs
// with (k only when there are more than k - 1 tiles per SM)
int stream_ctas_for(const StreamPlan& sp, int device, int tiles, int num_sms, int limit, bool track = false);
size_t stream_workspace_floats(const StreamPlan& sp, int batch);

// One class of a streaming launch (host view): its plan, stream buffers and
// iteration settings.  stream_begin fills the buffers and sizes; the caller
// sets max_iter, check_every, chg_eps and iters.
struct StreamJobDesc {
  StreamPlan sp;
  const float* bstream = nullptr;
  const float* fstream = nullptr;
  float2* state = nullptr;        // [tile][U][lane] constraint iterate records (z, y)
  const float2* param = nullptr;  // [tile][U][lane] constraint parameter records (l, u)
  float* state_p = nullptr;       // [tile][U][lane] primal iterate records x
  const float* param_p = nullptr; // [tile][U][lane] primal parameter records (sigma-scaled q)
  float* pres = nullptr;
  float* rhs = nullptr;   // frontier form: [tile][n][lane] right-hand sides
  float* fwd = nullptr;   // frontier form: [tile][n][lane] forward results
  int* iters = nullptr;
  int n_tiles = 0, max_iter = 0, batch = 0, check_every = 0;
  float chg_eps = 0.0f, sigma = 0.0f, alpha = 0.0f, one_minus_alpha = 0.0f;
  int ctas_limit = 2;  // most CTAs per SM this class's problem allows (a launch takes the smallest)
  // per-instance rho (adaptation): an instance whose rho changed (count > 0)
  // takes its rows' rho from its scalar rho_b by the rows' classes; null: the
  // schedule's rho vector for every instance
  const float* rho_b = nullptr;
  const int* rho_count = nullptr;
};

}  // namespace wmpc
