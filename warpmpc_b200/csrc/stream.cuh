// Streaming (TMA-fed) persistent OSQP path: host-built schedule tables and
// the device helpers shared by its kernels.
//
// Per instance tile (32 instances, one per lane) the LDL^T factor is stored
// "stream-major": [tile][stream position][lane], where the stream visits the
// columns of L in chunks of whole columns and stores, per chunk, the L entries
// of its columns (CSC order) followed by D^-1 of those columns.  The forward
// sweep reads the chunks' L parts in ascending order, the backward sweep reads
// L + D^-1 of every chunk in descending order: each read is one contiguous
// bulk copy (cp.async.bulk, 128 bytes per stream position).
//
// ADMM state (x or z, y) and parameters (q or l, u) are stored per tile in
// "release order" U: the order in which the backward sweep finishes with a KKT
// index (after the smallest column whose correction reads it), so each chunk
// of the backward sweep updates one contiguous U range.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "common.cuh"

namespace wmpc {

// Meta block of one chunk (int32 words, 16-byte padded), copied into the
// shared-memory stage together with the chunk's L data:
//   [0] ncols  [1] nent  [2] nrel  [3] c0 (first column)  [4] u0 (first U index)
//   [5 .. 5+ncols]           col_start (entry offset of each column, ncols+1)
//   [.. + nent]              row offset (32 * L row index of each entry)
//   [.. + nrel]              rel_i (permuted KKT index released)
//   [.. + nrel]              rel_kind (0 primal, 1 constraint)
//   [.. + nrel]              rel_rho (float bits)
//   [.. + nrel]              rel_rhoinv (float bits)
constexpr int kMetaHeader = 5;

struct StreamPlan {
  int n;              // KKT dimension
  int nnz_l;
  // forward sweep (row-gather form): L in CSR order, chunks of whole rows
  int n_fchunks;
  int max_fent, max_frows, max_fmeta_words;
  const int* fchunk_pos;    // [n_fchunks + 1] position in the forward stream (= CSR entry index)
  const int* fmeta_off;     // [n_fchunks]
  const int* fmeta_words;   // [n_fchunks]
  const int* fmeta;         // forward meta blocks:
                            //   [0] nrows [1] nent [2] r0 [3] 0 | row_start[nrows+1] | col offset (32*c)[nent]
  const int* proc_fpos;     // [nnz_l] forward-stream position of the L entry each program step writes
  // backward sweep (column form): L in CSC order + D^-1, chunks of whole columns
  int n_chunks;
  int stream_len;     // nnz_l + n
  int max_ent, max_cols, max_rel, max_meta_words;
  const int* chunk_pos;     // [n_chunks + 1] stream position of chunk start
  const int* chunk_ent;     // [n_chunks] entries in the chunk
  const int* chunk_cols;    // [n_chunks] columns in the chunk
  const int* meta_off;      // [n_chunks] word offset of the chunk's meta block
  const int* meta_words;    // [n_chunks] words (multiple of 4)
  const int* meta;          // all meta blocks
  // factor (compact accumulator) tables
  const int* init_slot;     // [init_ptr[n]] slot of each init row in reach(k)
  const int* upd_ptr;       // [nnz_l + 1]
  const int* upd_slot;      // [upd_ptr[nnz_l]]
  const int* col_spos;      // [n] stream position of column c's first L entry
  const int* dinv_spos;     // [n] stream position of D^-1_c
  const int* proc_spos;     // [nnz_l] stream position of the L entry each program step writes
  // release order
  const int* u_perm;        // [n] U index -> permuted KKT index
  const int* u_orig;        // [n] U index -> original KKT index
  int max_row_nnz;
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

// Bounded wait: gives up (returns false) after `limit_ns` or when *abort is set.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int* abort,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t start = global_timer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0) {
      if (abort && *abort) return false;
      if (global_timer_ns() - start > limit_ns) return false;
    }
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
  int ent = 32, cols = 12, rel = 8;  // backward chunks
  int fent = 32, frows = 12;         // forward chunks
};

// Host result: every array of StreamPlan, to be uploaded by the plan.
struct HostStream {
  int n_chunks = 0, stream_len = 0, max_ent = 0, max_cols = 0, max_rel = 0, max_meta_words = 0, max_row_nnz = 0;
  std::vector<int> chunk_pos, chunk_ent, chunk_cols, meta_off, meta_words, meta;
  int n_fchunks = 0, max_fent = 0, max_frows = 0, max_fmeta_words = 0;
  std::vector<int> fchunk_pos, fmeta_off, fmeta_words, fmeta, proc_fpos;
  std::vector<int> init_slot, upd_ptr, col_spos, dinv_spos, proc_spos, u_perm, u_orig;
  std::vector<unsigned short> upd_slot;
  // host copies used by the OSQP side to lay out the state
  std::vector<int> u_of_perm;  // permuted index -> U index
};

bool build_stream_schedule(const HostPattern& hp, const StreamTargets& t, const float* rho_by_constraint,
                           const float* rhoinv_by_constraint, int n_primal, HostStream* out, std::string* why);
bool build_factor_tables(const HostPattern& hp, std::vector<int>* init_slot, std::vector<int>* upd_ptr,
                         std::vector<unsigned short>* upd_slot, int* max_row_nnz, std::string* why);

struct StreamLaunch {
  int stages, sstages, meta_bytes, lbytes, sbytes;
  size_t smem;
};
constexpr int kFMetaHeader = 4;
bool stream_launch_config(const StreamPlan& sp, StreamLaunch* cfg);
size_t stream_workspace_floats(const StreamPlan& sp, int batch);

}  // namespace wmpc
