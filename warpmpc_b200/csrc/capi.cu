// extern "C" entry points of libwarpmpc_b200.so (declared in
// include/warpmpc_b200.h).  Argument validation, table upload, error
// reporting; all numerics live in qdldl.cu / osqp.cu.
#include <atomic>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "osqp.cuh"
#include "qdldl.cuh"

namespace wmpc {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

// ---- profiling ------------------------------------------------------------
namespace {
std::mutex g_prof_mu;
bool g_prof_on = false;
std::atomic<long long> g_launches{0};
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_prof_events;
size_t g_prof_used = 0;
bool g_prof_open = false;
int g_prof_channel = kProfileDominant;
std::mutex g_launch_mu;
int g_last_launch[4] = {0, 0, 0, 0};
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void profile_mark_begin(cudaStream_t s, int channel) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on || channel != g_prof_channel) return;
  if (g_prof_used == g_prof_events.size()) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return;
    if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return; }
    g_prof_events.push_back({a, b});
  }
  cudaEventRecord(g_prof_events[g_prof_used].first, s);
  g_prof_open = true;
}

void profile_mark_end(cudaStream_t s, int channel) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on || !g_prof_open || channel != g_prof_channel) return;
  cudaEventRecord(g_prof_events[g_prof_used].second, s);
  ++g_prof_used;
  g_prof_open = false;
}

void record_stream_launch(int form, int ctas_per_sm, int grid, int smem_bytes) {
  std::lock_guard<std::mutex> lk(g_launch_mu);
  g_last_launch[0] = form;
  g_last_launch[1] = ctas_per_sm;
  g_last_launch[2] = grid;
  g_last_launch[3] = smem_bytes;
}

size_t osqp_workspace_bytes(const wmpc_osqp& q, int batch, int pb, int ab, int mode, bool external);
size_t osqp_factor_workspace_bytes(const Osqp& o, const Pattern& pat, int pb, int ab);
size_t osqp_adjoint_extra_bytes(const Osqp& o, int batch);
int osqp_adjoint(const wmpc_osqp& q, const wmpc_osqp_options& opt, const wmpc_osqp_adjoint_batch& a, int mode,
                 void* ws, size_t ws_bytes, cudaStream_t s);
int osqp_factor(const Osqp& o, const wmpc_plan& plan, const float* p_values, int pb, const float* a_values, int ab,
                float* lx, float* d, float* dinv, void* ws, size_t ws_bytes, cudaStream_t s);
int osqp_solve(const wmpc_osqp& q, const wmpc_osqp_options& opt, const wmpc_osqp_batch& d,
               const float* lx_ext, const float* dinv_ext, int fb_ext, int mode, void* ws, size_t ws_bytes,
               cudaStream_t s);
int osqp_solve_multi(const wmpc_osqp* const* qs, const wmpc_osqp_options* opts, const wmpc_osqp_batch* ds, int n,
                     void* const* ws, const size_t* ws_bytes, cudaStream_t s);

namespace {

// Scoped device switch: compute entry points run on the plan's device.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; return; }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) ok = false;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

bool valid_perm(const int32_t* p, int n) {
  std::vector<char> seen(n, 0);
  for (int i = 0; i < n; ++i) {
    if (p[i] < 0 || p[i] >= n || seen[p[i]]) return false;
    seen[p[i]] = 1;
  }
  return true;
}

bool in_range(const int32_t* v, size_t count, int lo, int hi) {
  for (size_t i = 0; i < count; ++i)
    if (v[i] < lo || v[i] >= hi) return false;
  return true;
}

bool monotone_ptr(const int32_t* ptr, int n, int total) {
  if (ptr[0] != 0 || ptr[n] != total) return false;
  for (int i = 0; i < n; ++i)
    if (ptr[i + 1] < ptr[i]) return false;
  return true;
}

// Pack host arrays into one pinned-free staging vector and upload once.
struct Packer {
  std::vector<int32_t> ints;
  std::vector<std::pair<size_t, const int**>> fixups;
  void add(const int32_t* src, size_t count, const int** dst) {
    size_t off = (ints.size() + 31) / 32 * 32;  // 128-byte aligned sub-arrays
    ints.resize(off + count);
    if (count) std::memcpy(ints.data() + off, src, count * sizeof(int32_t));
    fixups.push_back({off, dst});
  }
  void addf(const float* src, size_t count, const float** dst) {
    static_assert(sizeof(float) == sizeof(int32_t), "float size");
    add(reinterpret_cast<const int32_t*>(src), count, reinterpret_cast<const int**>(dst));
  }
  int upload(int** block) {
    const size_t bytes = (ints.size() ? ints.size() : 1) * sizeof(int32_t);
    WMPC_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(block), bytes));
    if (!ints.empty()) {
      cudaError_t e = cudaMemcpy(*block, ints.data(), ints.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        cudaFree(*block);
        *block = nullptr;
        return fail(WMPC_ERR_CUDA, "table upload failed: %s", cudaGetErrorString(e));
      }
    }
    for (auto& f : fixups) *f.second = *block + f.first;
    return WMPC_OK;
  }
};


// One streaming schedule of an OSQP problem: compact factor tables, chunk
// schedule and launch check, uploaded in one block.  False (why set) when the
// pattern cannot use the streaming kernel in this form.
bool build_stream_plan(const HostPattern& hp, const StreamTargets& targets, const wmpc_osqp_desc* desc,
                       const std::vector<float>& unscale, StreamPlan* out, void** block, std::string* why) {
  HostStream hs;
  std::vector<int> init_slot, upd_ptr;
  std::vector<unsigned short> upd_slot16;
  int max_row = 0;
  if (!build_factor_tables(hp, &init_slot, &upd_ptr, &upd_slot16, &max_row, why) ||
      !build_stream_schedule(hp, targets, desc->rho_vec, desc->rho_inv_vec, desc->n, &hs, why, unscale.data()))
    return false;
  StreamPlan sp{};
  sp.n = hp.n;
  sp.nnz_l = hp.nnz_l;
  sp.n_chunks = hs.n_chunks;
  sp.blen = hs.blen;
  sp.max_units = hs.max_units;
  sp.max_cols = hs.max_cols;
  sp.max_rel = hs.max_rel;
  sp.max_meta_words = hs.max_meta_words;
  sp.max_meta_lead = hs.max_meta_lead;
  sp.max_row_nnz = max_row;
  sp.n_fchunks = hs.n_fchunks;
  sp.flen = hs.flen;
  sp.max_funits = hs.max_funits;
  sp.max_fmeta_words = hs.max_fmeta_words;
  sp.n_pad_b = static_cast<int>(hs.pad_boff.size());
  sp.n_pad_f = static_cast<int>(hs.pad_foff.size());
  sp.max_row_kv = hs.max_row_kv;
  sp.frontier_slots = hs.frontier_slots;
  sp.frontier_lag = hs.frontier_lag;
  sp.max_frows = hs.max_frows;
  sp.max_lstages = 12;
  sp.max_sstages = 6;
  if (const char* v = getenv("WMPC_STREAM_LSTAGES")) sp.max_lstages = atoi(v);
  if (const char* v = getenv("WMPC_STREAM_SSTAGES")) sp.max_sstages = atoi(v);
  StreamLaunch cfg;
  if (!stream_launch_config(sp, &cfg)) {
    *why = "work vector and ring do not fit in shared memory";
    return false;
  }
  std::vector<int> upd_slot(upd_slot16.begin(), upd_slot16.end());
  // factorization rows: {p0, p1, i0, i1}, {first update, update end, D^-1 offset, first KKT input}
  std::vector<int> row_info;
  row_info.reserve(8 * (size_t)hp.n);
  for (int k = 0; k < hp.n; ++k) {
    const int p0 = hp.proc_ptr[k], p1 = hp.proc_ptr[k + 1], i0 = hp.init_ptr[k], i1 = hp.init_ptr[k + 1];
    row_info.insert(row_info.end(), {p0, p1, i0, i1, upd_ptr[p0], upd_ptr[p1], hs.dinv_off[k], k + i0});
  }
  std::vector<float> unscale_perm(hp.n, 1.0f);
  for (int i = 0; i < hp.n; ++i) unscale_perm[i] = unscale[hp.p[i]];
  // rho class of each U index's constraint (per-instance rho)
  std::vector<int> u_cls;
  if (desc->rho_type) {
    u_cls.assign(hp.n, 0);
    for (int u = 0; u < hp.n; ++u) {
      const int orig = hs.u_orig[u];
      if (orig >= desc->n) u_cls[u] = desc->rho_type[orig - desc->n];
    }
  }
  Packer sk;
  if (!u_cls.empty()) sk.add(u_cls.data(), u_cls.size(), &sp.u_cls);
  sk.addf(unscale_perm.data(), unscale_perm.size(), &sp.unscale_perm);
  sk.add(hs.chunk_off.data(), hs.chunk_off.size(), &sp.chunk_off);
  sk.add(hs.chunk_units.data(), hs.chunk_units.size(), &sp.chunk_units);
  sk.add(hs.chunk_cols.data(), hs.chunk_cols.size(), &sp.chunk_cols);
  sk.add(hs.chunk_u0.data(), hs.chunk_u0.size(), &sp.chunk_u0);
  sk.add(hs.chunk_c0.data(), hs.chunk_c0.size(), &sp.chunk_c0);
  sk.add(hs.frow0.data(), hs.frow0.size(), &sp.frow0);
  sk.add(hs.frows.data(), hs.frows.size(), &sp.frows);
  sk.add(hs.chunk_nrel.data(), hs.chunk_nrel.size(), &sp.chunk_nrel);
  // primal releases per backward chunk (chunk header word 5)
  std::vector<int> chunk_nprim(hs.n_chunks, 0);
  for (int c = 0; c < hs.n_chunks; ++c) chunk_nprim[c] = hs.meta[hs.meta_off[c] + 5];
  sk.add(chunk_nprim.data(), chunk_nprim.size(), &sp.chunk_nprim);
  sk.add(hs.chunk_pre_u0.data(), hs.chunk_pre_u0.size(), &sp.chunk_pre_u0);
  sk.add(hs.chunk_pre_units.data(), hs.chunk_pre_units.size(), &sp.chunk_pre_units);
  sk.add(hs.meta_off.data(), hs.meta_off.size(), &sp.meta_off);
  sk.add(hs.meta_words.data(), hs.meta_words.size(), &sp.meta_words);
  sk.add(hs.meta.data(), hs.meta.size(), &sp.meta);
  sk.add(row_info.data(), row_info.size(), reinterpret_cast<const int**>(&sp.row_info));
  sk.add(init_slot.data(), init_slot.size(), &sp.init_slot);
  sk.add(upd_ptr.data(), upd_ptr.size(), &sp.upd_ptr);
  sk.add(upd_slot.data(), upd_slot.size(), &sp.upd_slot);
  sk.add(hs.col_uoff.data(), hs.col_uoff.size(), &sp.col_uoff);
  sk.add(hs.dinv_off.data(), hs.dinv_off.size(), &sp.dinv_off);
  sk.add(hs.proc_boff.data(), hs.proc_boff.size(), &sp.proc_boff);
  sk.add(hs.proc_foff.data(), hs.proc_foff.size(), &sp.proc_foff);
  sk.add(hs.upd_pos.data(), hs.upd_pos.size(), &sp.upd_pos);
  sk.add(hs.step_doff.data(), hs.step_doff.size(), &sp.step_doff);
  sk.add(hs.pad_boff.data(), hs.pad_boff.size(), &sp.pad_boff);
  sk.add(hs.pad_foff.data(), hs.pad_foff.size(), &sp.pad_foff);
  sk.add(hs.u_perm.data(), hs.u_perm.size(), &sp.u_perm);
  sk.add(hs.u_orig.data(), hs.u_orig.size(), &sp.u_orig);
  sk.add(hs.fchunk_off.data(), hs.fchunk_off.size(), &sp.fchunk_off);
  sk.add(hs.fchunk_units.data(), hs.fchunk_units.size(), &sp.fchunk_units);
  sk.add(hs.fmeta_off.data(), hs.fmeta_off.size(), &sp.fmeta_off);
  sk.add(hs.fmeta_words.data(), hs.fmeta_words.size(), &sp.fmeta_words);
  sk.add(hs.fmeta.data(), hs.fmeta.size(), &sp.fmeta);
  int* sblock = nullptr;
  if (sk.upload(&sblock) != WMPC_OK) {
    *why = g_last_error;
    return false;
  }
  *block = sblock;
  *out = sp;
  return true;
}
}  // namespace
}  // namespace wmpc

using namespace wmpc;

extern "C" {

const char* wmpc_last_error_string(void) { return g_last_error.c_str(); }

const char* wmpc_version(void) { return "0.1.0 sm_100a"; }

int wmpc_profile_begin(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = true;
  g_prof_used = 0;
  g_prof_open = false;
  g_launches.store(0);
  return WMPC_OK;
}

int wmpc_profile_select(int32_t channel) {
  if (channel < 0 || channel > 1) return fail(WMPC_ERR_INVALID_ARGUMENT, "profile channel %d (0 or 1)", channel);
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_channel = channel;
  return WMPC_OK;
}

int wmpc_stream_last_launch(int32_t info[4]) {
  if (!info) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(g_launch_mu);
  for (int i = 0; i < 4; ++i) info[i] = g_last_launch[i];
  return WMPC_OK;
}

int wmpc_profile_end(float* dominant_ms, int32_t* dominant_launches, int64_t* total_launches) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  double total = 0.0;
  for (size_t i = 0; i < g_prof_used; ++i) {
    cudaError_t e = cudaEventSynchronize(g_prof_events[i].second);
    if (e != cudaSuccess) {
      g_prof_on = false;
      return fail(WMPC_ERR_CUDA, "profile event sync failed: %s", cudaGetErrorString(e));
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g_prof_events[i].first, g_prof_events[i].second);
    total += ms;
  }
  if (dominant_ms) *dominant_ms = static_cast<float>(total);
  if (dominant_launches) *dominant_launches = static_cast<int32_t>(g_prof_used);
  if (total_launches) *total_launches = g_launches.load();
  g_prof_on = false;
  g_prof_used = 0;
  return WMPC_OK;
}

int64_t wmpc_launch_count(void) { return g_launches.load(); }

int wmpc_solve_tables_host(const wmpc_pattern_desc* desc, int32_t* out, int64_t out_capacity, int64_t* out_words) {
  if (!desc || !out_words || !desc->lp || (desc->nnz_l > 0 && !desc->li))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  const int n = desc->n, nnz_l = desc->nnz_l;
  if (n <= 0 || nnz_l <= 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "bad sizes");
  std::vector<int> tables, sdesc;
  if (!build_solve_tables(n, std::vector<int>(desc->lp, desc->lp + n + 1), std::vector<int>(desc->li, desc->li + nnz_l),
                          &tables, &sdesc))
    return fail(WMPC_ERR_UNSUPPORTED, "a column has more entries than a solve chunk holds");
  std::vector<int> w{static_cast<int>(sdesc.size() / 8), static_cast<int>(tables.size())};
  w.insert(w.end(), tables.begin(), tables.end());
  w.insert(w.end(), sdesc.begin(), sdesc.end());
  *out_words = static_cast<int64_t>(w.size());
  if (out) {
    if (out_capacity < *out_words) return fail(WMPC_ERR_INVALID_ARGUMENT, "output capacity too small");
    std::memcpy(out, w.data(), w.size() * sizeof(int32_t));
  }
  return WMPC_OK;
}

int wmpc_stream_schedule_host(const wmpc_pattern_desc* desc, const float* rho, const float* rhoinv, int32_t n_primal,
                              int32_t units, int32_t cols, int32_t rel, int32_t funits, int32_t offload,
                              int32_t* out, int64_t out_capacity, int64_t* out_words) {
  if (!desc || !out_words) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  const int n = desc->n, nnz_l = desc->nnz_l;
  if (n <= 0 || nnz_l < 0 || n_primal < 0 || n_primal > n || units <= 0 || cols <= 0 || rel <= 0 || funits <= 0)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "bad sizes");
  HostPattern hp;
  hp.n = n;
  hp.nnz_a = desc->nnz_a;
  hp.nnz_l = nnz_l;
  hp.init_ptr.assign(desc->init_ptr, desc->init_ptr + n + 1);
  const int n_init = desc->init_ptr[n];
  hp.init_rows.assign(desc->init_rows, desc->init_rows + n_init);
  hp.proc_ptr.assign(desc->proc_ptr, desc->proc_ptr + n + 1);
  hp.proc_cols.assign(desc->proc_cols, desc->proc_cols + nnz_l);
  hp.proc_offsets.assign(desc->proc_offsets, desc->proc_offsets + nnz_l);
  hp.proc_lidx.assign(desc->proc_lidx, desc->proc_lidx + nnz_l);
  hp.lp.assign(desc->lp, desc->lp + n + 1);
  hp.li.assign(desc->li, desc->li + nnz_l);
  hp.p.assign(desc->p, desc->p + n);
  std::string why;
  std::vector<int> init_slot, upd_ptr;
  std::vector<unsigned short> upd_slot;
  int max_row = 0;
  HostStream hs;
  StreamTargets t;
  t.units = units;
  t.cols = cols;
  t.rel = rel;
  t.funits = funits;
  t.offload = offload & 3;
  t.frontier = (offload >> 2) & 1;  // bit 2: frontier-slot schedule
  t.frontier_copies = (offload >> 3) & 1;  // bit 3: with chunk-start copies of rows without entries
  if (offload >> 8) t.frontier_lag = offload >> 8;  // bits 8+: its release lag
  if (!build_factor_tables(hp, &init_slot, &upd_ptr, &upd_slot, &max_row, &why) ||
      !build_stream_schedule(hp, t, rho, rhoinv, n_primal, &hs, &why))
    return fail(WMPC_ERR_UNSUPPORTED, "%s", why.c_str());
  std::vector<int> w{hs.n_chunks, hs.blen, hs.max_units, hs.max_cols, hs.max_rel, hs.max_meta_words, max_row,
                     static_cast<int>(hs.meta.size())};
  auto app = [&](const std::vector<int>& v) { w.insert(w.end(), v.begin(), v.end()); };
  app(hs.chunk_off); app(hs.chunk_units); app(hs.chunk_cols); app(hs.chunk_u0); app(hs.chunk_nrel);
  app(hs.meta_off); app(hs.meta_words); app(hs.meta);
  app(hs.col_uoff); app(hs.dinv_off); app(hs.proc_boff); app(hs.u_perm); app(hs.u_orig);
  app(init_slot); app(upd_ptr);
  for (unsigned short v : upd_slot) w.push_back(v);
  w.push_back(hs.n_fchunks); w.push_back(hs.flen); w.push_back(hs.max_funits); w.push_back(hs.max_fmeta_words);
  w.push_back(static_cast<int>(hs.fmeta.size()));
  app(hs.fchunk_off); app(hs.fchunk_units); app(hs.fmeta_off); app(hs.fmeta_words); app(hs.fmeta); app(hs.proc_foff);
  w.push_back(static_cast<int>(hs.pad_boff.size())); w.push_back(static_cast<int>(hs.pad_foff.size()));
  w.push_back(hs.dummy_units);
  app(hs.pad_boff); app(hs.pad_foff);
  app(hs.chunk_pre_u0); app(hs.chunk_pre_units);
  w.push_back(hs.frontier_slots); w.push_back(hs.frontier_lag); w.push_back(hs.max_frows);
  *out_words = static_cast<int64_t>(w.size());
  if (!out) return WMPC_OK;
  if (out_capacity < static_cast<int64_t>(w.size())) return fail(WMPC_ERR_INVALID_ARGUMENT, "output buffer too small");
  std::memcpy(out, w.data(), w.size() * sizeof(int32_t));
  return WMPC_OK;
}

int wmpc_plan_create(const wmpc_pattern_desc* desc, int device, wmpc_plan** out) {
  if (!desc || !out) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  const int n = desc->n, nnz_a = desc->nnz_a, nnz_l = desc->nnz_l;
  if (n <= 0 || nnz_a < n || nnz_l < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "bad sizes n=%d nnz_a=%d nnz_l=%d", n, nnz_a, nnz_l);
  if (!desc->perm_to_orig || !desc->diag_pos || !desc->init_ptr || !desc->proc_ptr || !desc->lp || !desc->p ||
      !desc->pinv || (nnz_l && (!desc->proc_cols || !desc->proc_lidx || !desc->proc_offsets || !desc->li)))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "null table pointer");
  const int n_init = desc->init_ptr[n];
  // structural validation: every index the kernels dereference is in range
  if (!valid_perm(desc->p, n) || !valid_perm(desc->pinv, n)) return fail(WMPC_ERR_INVALID_ARGUMENT, "p/pinv are not permutations");
  for (int i = 0; i < n; ++i)
    if (desc->pinv[desc->p[i]] != i) return fail(WMPC_ERR_INVALID_ARGUMENT, "pinv is not the inverse of p");
  if (!valid_perm(desc->perm_to_orig, nnz_a)) return fail(WMPC_ERR_INVALID_ARGUMENT, "perm_to_orig is not a permutation");
  if (!in_range(desc->diag_pos, n, 0, nnz_a)) return fail(WMPC_ERR_INVALID_ARGUMENT, "diag_pos out of range");
  if (!monotone_ptr(desc->init_ptr, n, n_init) || n_init > nnz_a) return fail(WMPC_ERR_INVALID_ARGUMENT, "bad init_ptr");
  if (n_init && (!desc->init_rows || !desc->init_pos)) return fail(WMPC_ERR_INVALID_ARGUMENT, "null init tables");
  if (!in_range(desc->init_rows, n_init, 0, n) || !in_range(desc->init_pos, n_init, 0, nnz_a))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "init tables out of range");
  if (!monotone_ptr(desc->proc_ptr, n, nnz_l) || !monotone_ptr(desc->lp, n, nnz_l))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "bad proc_ptr/lp");
  if (!in_range(desc->proc_cols, nnz_l, 0, n) || !in_range(desc->proc_lidx, nnz_l, 0, nnz_l) ||
      !in_range(desc->li, nnz_l, 0, n))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "L tables out of range");
  int max_row = 0, max_col = 0;
  for (int k = 0; k < n; ++k) {
    max_row = std::max(max_row, desc->proc_ptr[k + 1] - desc->proc_ptr[k]);
    max_col = std::max(max_col, desc->lp[k + 1] - desc->lp[k]);
    for (int e = desc->proc_ptr[k]; e < desc->proc_ptr[k + 1]; ++e) {
      const int c = desc->proc_cols[e];
      if (c >= k || desc->proc_offsets[e] < 0 || desc->proc_offsets[e] > desc->lp[c + 1] - desc->lp[c] ||
          desc->proc_lidx[e] != desc->lp[c] + desc->proc_offsets[e])
        return fail(WMPC_ERR_INVALID_ARGUMENT, "inconsistent row program at row %d", k);
    }
    for (int e = desc->lp[k]; e < desc->lp[k + 1]; ++e)
      if (desc->li[e] <= k) return fail(WMPC_ERR_INVALID_ARGUMENT, "L is not strictly lower triangular");
  }
  DeviceGuard guard(device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", device);
  auto* plan = new wmpc_plan();
  plan->device = device;
  Pattern& pat = plan->pat;
  pat.n = n;
  pat.nnz_a = nnz_a;
  pat.nnz_l = nnz_l;
  pat.max_row_nnz = max_row;
  pat.max_col_nnz = max_col;
  Packer pk;
  pk.add(desc->perm_to_orig, nnz_a, &pat.perm_to_orig);
  pk.add(desc->diag_pos, n, &pat.diag_pos);
  pk.add(desc->init_ptr, n + 1, &pat.init_ptr);
  pk.add(desc->init_rows, n_init, &pat.init_rows);
  pk.add(desc->init_pos, n_init, &pat.init_pos);
  pk.add(desc->proc_ptr, n + 1, &pat.proc_ptr);
  pk.add(desc->proc_cols, nnz_l, &pat.proc_cols);
  pk.add(desc->proc_lidx, nnz_l, &pat.proc_lidx);
  pk.add(desc->proc_offsets, nnz_l, &pat.proc_offsets);
  pk.add(desc->lp, n + 1, &pat.lp);
  pk.add(desc->li, nnz_l, &pat.li);
  pk.add(desc->p, n, &pat.p);
  pk.add(desc->pinv, n, &pat.pinv);
  // compact-accumulator tables of the staged per-call factorization
  std::vector<int> fac_init_slot, fac_upd_ptr, fac_upd_slot, fac_upd_lidx;
  {
    HostPattern hp;
    hp.n = n;
    hp.nnz_a = nnz_a;
    hp.nnz_l = nnz_l;
    hp.init_ptr.assign(desc->init_ptr, desc->init_ptr + n + 1);
    hp.init_rows.assign(desc->init_rows, desc->init_rows + n_init);
    hp.proc_ptr.assign(desc->proc_ptr, desc->proc_ptr + n + 1);
    hp.proc_cols.assign(desc->proc_cols, desc->proc_cols + nnz_l);
    hp.proc_offsets.assign(desc->proc_offsets, desc->proc_offsets + nnz_l);
    hp.proc_lidx.assign(desc->proc_lidx, desc->proc_lidx + nnz_l);
    hp.lp.assign(desc->lp, desc->lp + n + 1);
    hp.li.assign(desc->li, desc->li + nnz_l);
    std::vector<unsigned short> slot16;
    std::string why;
    int max_row = 0;
    if (nnz_l > 0 && build_factor_tables(hp, &fac_init_slot, &fac_upd_ptr, &slot16, &max_row, &why)) {
      fac_upd_slot.assign(slot16.begin(), slot16.end());
      for (int k = 0; k < n; ++k)
        for (int e = hp.proc_ptr[k]; e < hp.proc_ptr[k + 1]; ++e)
          for (int q = 0; q < hp.proc_offsets[e]; ++q) fac_upd_lidx.push_back(hp.lp[hp.proc_cols[e]] + q);
      int max_kv = 0;
      for (int k = 0; k < n; ++k) max_kv = std::max(max_kv, 1 + hp.init_ptr[k + 1] - hp.init_ptr[k]);
      pk.add(fac_init_slot.data(), fac_init_slot.size(), &plan->fac_init_slot);
      pk.add(fac_upd_ptr.data(), fac_upd_ptr.size(), &plan->fac_upd_ptr);
      pk.add(fac_upd_slot.data(), fac_upd_slot.size(), &plan->fac_upd_slot);
      pk.add(fac_upd_lidx.data(), fac_upd_lidx.size(), &plan->fac_upd_lidx);
      // rows read ahead: {p0, p1, i0, i1}, {first update, update end, first input, 0}; per input its KKT slot
      std::vector<int> row_info, kin_slot;
      row_info.reserve(8 * (size_t)n);
      kin_slot.reserve((size_t)n + n_init);
      for (int k = 0; k < n; ++k) {
        const int p0 = hp.proc_ptr[k], p1 = hp.proc_ptr[k + 1], i0 = hp.init_ptr[k], i1 = hp.init_ptr[k + 1];
        row_info.insert(row_info.end(), {p0, p1, i0, i1, fac_upd_ptr[p0], fac_upd_ptr[p1], k + i0, 0});
        kin_slot.push_back(desc->perm_to_orig[desc->diag_pos[k]]);
        for (int e = i0; e < i1; ++e) kin_slot.push_back(desc->perm_to_orig[desc->init_pos[e]]);
      }
      pk.add(row_info.data(), row_info.size(), reinterpret_cast<const int**>(&plan->fac_row_info));
      pk.add(kin_slot.data(), kin_slot.size(), &plan->fac_kin_slot);
      plan->fac_max_row = std::max(max_row, 1);
      plan->fac_max_kv = max_kv;
    }
  }
  // chunk tables of the TMA-fed per-call solve (when every column fits a chunk)
  std::vector<int> solve_tables, solve_desc;
  if (nnz_l > 0 && build_solve_tables(n, std::vector<int>(desc->lp, desc->lp + n + 1),
                                      std::vector<int>(desc->li, desc->li + nnz_l), &solve_tables, &solve_desc)) {
    pk.add(solve_tables.data(), solve_tables.size(), &plan->solve_tables);
    pk.add(solve_desc.data(), solve_desc.size(), &plan->solve_desc);
    plan->solve_chunks = (int)solve_desc.size() / 8;
  }
  int rc = pk.upload(&plan->table_block);
  if (rc) {
    delete plan;
    return rc;
  }
  plan->table_ints = pk.ints.size();
  plan->h_init_ptr.assign(desc->init_ptr, desc->init_ptr + n + 1);
  plan->h_init_rows.assign(desc->init_rows, desc->init_rows + n_init);
  plan->h_proc_ptr.assign(desc->proc_ptr, desc->proc_ptr + n + 1);
  plan->h_proc_cols.assign(desc->proc_cols, desc->proc_cols + nnz_l);
  plan->h_proc_offsets.assign(desc->proc_offsets, desc->proc_offsets + nnz_l);
  plan->h_proc_lidx.assign(desc->proc_lidx, desc->proc_lidx + nnz_l);
  plan->h_lp.assign(desc->lp, desc->lp + n + 1);
  plan->h_li.assign(desc->li, desc->li + nnz_l);
  plan->h_p.assign(desc->p, desc->p + n);
  plan->h_perm_to_orig.assign(desc->perm_to_orig, desc->perm_to_orig + nnz_a);
  plan->h_diag_pos.assign(desc->diag_pos, desc->diag_pos + n);
  plan->h_init_pos.assign(desc->init_pos, desc->init_pos + n_init);
  *out = plan;
  return WMPC_OK;
}

int wmpc_plan_destroy(wmpc_plan* plan) {
  if (!plan) return WMPC_OK;
  DeviceGuard guard(plan->device);
  if (plan->table_block) cudaFree(plan->table_block);
  delete plan;
  return WMPC_OK;
}

int wmpc_plan_info(const wmpc_plan* plan, int32_t* n, int32_t* nnz_a, int32_t* nnz_l, int32_t* max_row_nnz,
                   int32_t* max_col_nnz) {
  if (!plan) return fail(WMPC_ERR_INVALID_ARGUMENT, "null plan");
  if (n) *n = plan->pat.n;
  if (nnz_a) *nnz_a = plan->pat.nnz_a;
  if (nnz_l) *nnz_l = plan->pat.nnz_l;
  if (max_row_nnz) *max_row_nnz = plan->pat.max_row_nnz;
  if (max_col_nnz) *max_col_nnz = plan->pat.max_col_nnz;
  return WMPC_OK;
}

size_t wmpc_factor_workspace_bytes(const wmpc_plan* plan, int32_t batch) {
  return plan ? factor_workspace_bytes(plan->pat, batch) : 0;
}

size_t wmpc_solve_workspace_bytes(const wmpc_plan* plan, int32_t batch) {
  return plan ? solve_workspace_bytes(plan->pat, batch) : 0;
}

int wmpc_factor(const wmpc_plan* plan, const float* values, int64_t values_ld, int32_t values_bstride, float* lx,
                float* d, float* dinv, int32_t batch, void* workspace, size_t workspace_bytes,
                wmpc_stream_t stream) {
  if (!plan || batch < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "bad plan or batch");
  if (batch == 0) return WMPC_OK;
  if (!values || (!lx && plan->pat.nnz_l > 0) || !d || !dinv) return fail(WMPC_ERR_INVALID_ARGUMENT, "null buffer");
  if ((values_bstride != 0 && values_bstride != 1) || (values_bstride == 1 && values_ld < batch))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "values_ld/values_bstride inconsistent with batch");
  DeviceGuard guard(plan->device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", plan->device);
  return launch_factor_plan(*plan, values, values_ld, values_bstride, lx, d, dinv, batch, workspace,
                       workspace_bytes, static_cast<cudaStream_t>(stream));
}

int wmpc_solve(const wmpc_plan* plan, const float* lx, const float* dinv, int32_t factor_bstride,
               const float* rhs, float* x, int32_t batch, void* workspace, size_t workspace_bytes,
               wmpc_stream_t stream) {
  if (!plan || batch < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "bad plan or batch");
  if (batch == 0) return WMPC_OK;
  if ((!lx && plan->pat.nnz_l > 0) || !dinv || !rhs || !x) return fail(WMPC_ERR_INVALID_ARGUMENT, "null buffer");
  if (factor_bstride != 0 && factor_bstride != 1) return fail(WMPC_ERR_INVALID_ARGUMENT, "factor_bstride must be 0 or 1");
  DeviceGuard guard(plan->device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", plan->device);
  return launch_solve_plan(*plan, lx, dinv, factor_bstride, rhs, x, batch, workspace, workspace_bytes,
                           static_cast<cudaStream_t>(stream));
}

int wmpc_factor_solve(const wmpc_plan* plan, const float* values, int64_t values_ld, int32_t values_bstride,
                      const float* rhs, float* x, float* lx, float* d, float* dinv, int32_t batch, void* workspace,
                      size_t workspace_bytes, wmpc_stream_t stream) {
  const int kb = values_bstride ? batch : 1;
  int rc = wmpc_factor(plan, values, values_ld, values_bstride, lx, d, dinv, kb, workspace, workspace_bytes, stream);
  if (rc) return rc;
  return wmpc_solve(plan, lx, dinv, values_bstride ? 1 : 0, rhs, x, batch, workspace, workspace_bytes, stream);
}

int wmpc_osqp_create(const wmpc_osqp_desc* desc, const wmpc_plan* kkt_plan, wmpc_osqp** out) {
  if (!desc || !kkt_plan || !out) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  const int n = desc->n, m = desc->m, np = desc->nnz_p, na = desc->nnz_a, nk = desc->nnz_kkt, npf = desc->nnz_p_full;
  if (n <= 0 || m < 0 || np < 0 || na < 0 || nk <= 0 || npf < 0)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "bad OSQP sizes");
  if (kkt_plan->pat.n != n + m || kkt_plan->pat.nnz_a != nk)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "KKT plan (n=%d nnz=%d) does not match OSQP problem (n+m=%d nnz_kkt=%d)",
                kkt_plan->pat.n, kkt_plan->pat.nnz_a, n + m, nk);
  if (!in_range(desc->p_to_kkt, np, 0, nk) || !in_range(desc->a_to_kkt, na, 0, nk) ||
      !in_range(desc->a_rows, na, 0, m) || !in_range(desc->a_cols, na, 0, n) ||
      !in_range(desc->p_full_rows, npf, 0, n) || !in_range(desc->p_full_cols, npf, 0, n) ||
      !in_range(desc->p_full_value_map, npf, 0, np > 0 ? np : 1))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "OSQP index tables out of range");
  for (int e = 1; e < na; ++e)
    if (desc->a_cols[e] < desc->a_cols[e - 1]) return fail(WMPC_ERR_INVALID_ARGUMENT, "A entries must be in CSC order");

  // KKT slot sources
  std::vector<int32_t> kkt_src(nk, -1);
  for (int j = 0; j < np; ++j) {
    if (kkt_src[desc->p_to_kkt[j]] != -1) return fail(WMPC_ERR_INVALID_ARGUMENT, "duplicate KKT slot");
    kkt_src[desc->p_to_kkt[j]] = j;
  }
  for (int j = 0; j < na; ++j) {
    if (kkt_src[desc->a_to_kkt[j]] != -1) return fail(WMPC_ERR_INVALID_ARGUMENT, "duplicate KKT slot");
    kkt_src[desc->a_to_kkt[j]] = np + j;
  }
  // A by rows (stable: ascending entry index within each row)
  std::vector<int32_t> a_row_ptr(m + 1, 0), a_row_ent(na), a_col_ptr(n + 1, 0);
  for (int e = 0; e < na; ++e) a_row_ptr[desc->a_rows[e] + 1]++;
  for (int r = 0; r < m; ++r) a_row_ptr[r + 1] += a_row_ptr[r];
  {
    std::vector<int32_t> fillp(a_row_ptr.begin(), a_row_ptr.end() - 1);
    for (int e = 0; e < na; ++e) a_row_ent[fillp[desc->a_rows[e]]++] = e;
  }
  for (int e = 0; e < na; ++e) a_col_ptr[desc->a_cols[e] + 1]++;
  for (int j = 0; j < n; ++j) a_col_ptr[j + 1] += a_col_ptr[j];
  // upper entries of P: first occurrence of each entry in the full pattern
  std::vector<int32_t> p_up_rows(np, 0), p_up_cols(np, 0);
  {
    std::vector<char> seen(np, 0);
    for (int t = 0; t < npf; ++t) {
      const int k = desc->p_full_value_map[t];
      if (!seen[k]) {
        seen[k] = 1;
        p_up_rows[k] = desc->p_full_rows[t];
        p_up_cols[k] = desc->p_full_cols[t];
      }
    }
  }
  // both triangles of P grouped by row, stable in the reference's entry order
  std::vector<int32_t> pf_row_ptr(n + 1, 0), pf_val(npf), pf_col(npf);
  for (int t = 0; t < npf; ++t) pf_row_ptr[desc->p_full_rows[t] + 1]++;
  for (int j = 0; j < n; ++j) pf_row_ptr[j + 1] += pf_row_ptr[j];
  {
    std::vector<int32_t> fillp(pf_row_ptr.begin(), pf_row_ptr.end() - 1);
    for (int t = 0; t < npf; ++t) {
      const int pos = fillp[desc->p_full_rows[t]]++;
      pf_val[pos] = desc->p_full_value_map[t];
      pf_col[pos] = desc->p_full_cols[t];
    }
  }

  DeviceGuard guard(kkt_plan->device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", kkt_plan->device);
  auto* q = new wmpc_osqp();
  q->device = kkt_plan->device;
  q->ctas_limit = stream_ctas_limit_setting();
  q->kkt_plan = kkt_plan;
  Osqp& o = q->dev;
  o.n = n;
  o.m = m;
  o.nk = n + m;
  o.nnz_p = np;
  o.nnz_a = na;
  o.nnz_kkt = nk;
  o.nnz_pf = npf;
  o.sigma = desc->sigma;
  o.alpha = desc->alpha;
  o.one_minus_alpha = 1.0f - desc->alpha;
  Packer pk;
  pk.addf(desc->kkt_base, nk, &o.kkt_base);
  pk.add(kkt_src.data(), nk, &o.kkt_src);
  pk.addf(desc->p_scale, np, &o.p_scale);
  pk.addf(desc->p_diag_sigma, np, &o.p_diag_sigma);
  pk.addf(desc->a_scale, na, &o.a_scale);
  pk.add(a_row_ptr.data(), m + 1, &o.a_row_ptr);
  pk.add(a_row_ent.data(), na, &o.a_row_ent);
  pk.add(desc->a_cols, na, &o.a_cols);
  pk.add(desc->a_rows, na, &o.a_rows);
  pk.add(a_col_ptr.data(), n + 1, &o.a_col_ptr);
  pk.add(pf_row_ptr.data(), n + 1, &o.pf_row_ptr);
  pk.add(pf_val.data(), npf, &o.pf_val);
  pk.add(pf_col.data(), npf, &o.pf_col);
  pk.addf(desc->rho_vec, m, &o.rho);
  pk.addf(desc->rho_inv_vec, m, &o.rho_inv);
  pk.addf(desc->q_scale, n, &o.q_scale);
  pk.addf(desc->scaling_d, n, &o.scaling_d);
  pk.addf(desc->scaling_dinv, n, &o.scaling_dinv);
  pk.addf(desc->scaling_e, m, &o.scaling_e);
  pk.addf(desc->scaling_einv, m, &o.scaling_einv);
  pk.addf(desc->y_scale, m, &o.y_scale);
  pk.addf(desc->y_unscale, m, &o.y_unscale);
  pk.add(p_up_rows.data(), np, &q->p_upper_rows);
  pk.add(p_up_cols.data(), np, &q->p_upper_cols);
  // the factorization rows' KKT inputs in row-program order, resolved
  {
    const wmpc_plan& kp = *kkt_plan;
    const int nkkt = n + m;
    std::vector<int32_t> kin;
    kin.reserve(4 * ((size_t)nkkt + kp.h_init_pos.size()));
    auto put = [&](int slot) {
      const int idx = kp.h_perm_to_orig[slot];
      const int src = kkt_src[idx];
      float scale = 0.0f, add = 0.0f;
      int kind = 0;
      if (src < 0) {
        add = desc->kkt_base[idx];
      } else if (src < np) {
        kind = 1;
        scale = desc->p_scale[src];
        add = desc->p_diag_sigma[src];
      } else {
        kind = 2;
        scale = desc->a_scale[src - np];
      }
      int32_t sb, ab;
      std::memcpy(&sb, &scale, 4);
      std::memcpy(&ab, &add, 4);
      kin.insert(kin.end(), {src < 0 ? -1 : src, kind, sb, ab});
    };
    for (int k = 0; k < nkkt; ++k) {
      put(kp.h_diag_pos[k]);
      for (int e = kp.h_init_ptr[k]; e < kp.h_init_ptr[k + 1]; ++e) put(kp.h_init_pos[e]);
    }
    pk.add(kin.data(), kin.size(), reinterpret_cast<const int**>(&o.kin_desc));
  }
  // rho adaptation: each constraint's rho class and, per KKT slot, the
  // constraint whose -1/rho it holds (-1: none)
  std::vector<int32_t> kkt_rho_row;
  if (desc->rho_type && desc->rho_to_kkt && m > 0) {
    kkt_rho_row.assign(nk, -1);
    for (int r = 0; r < m; ++r) {
      const int slot = desc->rho_to_kkt[r];
      const int t = desc->rho_type[r];
      if (slot < 0 || slot >= nk || kkt_src[slot] >= 0 || kkt_rho_row[slot] >= 0 || t < -1 || t > 1) {
        delete q;
        return fail(WMPC_ERR_INVALID_ARGUMENT, "bad rho_to_kkt/rho_type entry for constraint %d", r);
      }
      kkt_rho_row[slot] = r;
    }
    pk.add(desc->rho_type, m, &o.rho_type);
    pk.add(kkt_rho_row.data(), nk, &o.kkt_rho_row);
    o.rho0 = desc->rho;
    // the factorization rows' inputs with every -1/rho slot read from the
    // instance's 1/rho row (constraint r: source nnz_p + nnz_a + r, kind 3)
    const wmpc_plan& kp = *kkt_plan;
    std::vector<int32_t> kin;
    kin.reserve(4 * ((size_t)(n + m) + kp.h_init_pos.size()));
    auto put = [&](int slot) {
      const int idx = kp.h_perm_to_orig[slot];
      const int r = kkt_rho_row[idx];
      const int src = kkt_src[idx];
      float scale = 0.0f, add = 0.0f;
      int kind = 0, s = -1;
      if (r >= 0) {
        kind = 3;
        s = np + na + r;
      } else if (src < 0) {
        add = desc->kkt_base[idx];
      } else if (src < np) {
        kind = 1;
        s = src;
        scale = desc->p_scale[src];
        add = desc->p_diag_sigma[src];
      } else {
        kind = 2;
        s = src;
        scale = desc->a_scale[src - np];
      }
      int32_t sb, ab;
      std::memcpy(&sb, &scale, 4);
      std::memcpy(&ab, &add, 4);
      kin.insert(kin.end(), {s, kind, sb, ab});
    };
    for (int k = 0; k < n + m; ++k) {
      put(kp.h_diag_pos[k]);
      for (int e = kp.h_init_ptr[k]; e < kp.h_init_ptr[k + 1]; ++e) put(kp.h_init_pos[e]);
    }
    pk.add(kin.data(), kin.size(), reinterpret_cast<const int**>(&o.kin_desc_rho));
  }
  int* block = nullptr;
  int rc = pk.upload(&block);
  if (rc) {
    delete q;
    return rc;
  }
  q->block = block;
  cudaDeviceGetAttribute(&q->num_sms, cudaDevAttrMultiProcessorCount, kkt_plan->device);
  // streaming persistent path: schedule + compact factor tables
  {
    HostPattern hp;
    hp.n = kkt_plan->pat.n;
    hp.nnz_a = kkt_plan->pat.nnz_a;
    hp.nnz_l = kkt_plan->pat.nnz_l;
    hp.init_ptr = kkt_plan->h_init_ptr;
    hp.init_rows = kkt_plan->h_init_rows;
    hp.proc_ptr = kkt_plan->h_proc_ptr;
    hp.proc_cols = kkt_plan->h_proc_cols;
    hp.proc_offsets = kkt_plan->h_proc_offsets;
    hp.proc_lidx = kkt_plan->h_proc_lidx;
    hp.lp = kkt_plan->h_lp;
    hp.li = kkt_plan->h_li;
    hp.p = kkt_plan->h_p;
    StreamTargets targets;
    if (const char* v = getenv("WMPC_STREAM_UNITS")) targets.units = atoi(v);
    if (const char* v = getenv("WMPC_STREAM_COLS")) targets.cols = atoi(v);
    if (const char* v = getenv("WMPC_STREAM_REL")) targets.rel = atoi(v);
    if (const char* v = getenv("WMPC_STREAM_FUNITS")) targets.funits = atoi(v);
    if (const char* v = getenv("WMPC_STREAM_OFFLOAD")) targets.offload = atoi(v) & 3;
    if (targets.units <= 0 || targets.cols <= 0 || targets.rel <= 0 || targets.funits <= 0) targets = StreamTargets();
    // the frontier-slot form (fixed-iteration solves only; no releaser offload):
    // 0 none, 1 the only schedule, 2 (default) a second schedule beside the plain one
    int frontier_mode = 2;
    if (const char* v = getenv("WMPC_STREAM_FRONTIER")) frontier_mode = atoi(v);
    StreamTargets ftargets = targets;
    ftargets.frontier = 1;
    ftargets.offload = 0;
    if (const char* lag = getenv("WMPC_STREAM_FRONTIER_LAG")) ftargets.frontier_lag = atoi(lag);
    if (const char* v = getenv("WMPC_STREAM_FRONTIER_COPIES")) ftargets.frontier_copies = atoi(v) > 0 ? 1 : 0;
    // iterate-change unscale factors (original KKT order) for early termination
    std::vector<float> unscale(hp.n, 1.0f);
    for (int j = 0; j < n; ++j) unscale[j] = desc->scaling_d[j];
    for (int r = 0; r < m; ++r) unscale[n + r] = std::max(desc->scaling_einv[r], desc->y_unscale[r]);
    q->has_stream = build_stream_plan(hp, frontier_mode == 1 ? ftargets : targets, desc, unscale, &q->sp,
                                      &q->stream_block, &q->stream_why);
    if (q->has_stream && frontier_mode == 2) {
      std::string why;
      q->has_frontier = build_stream_plan(hp, ftargets, desc, unscale, &q->spf, &q->stream_block_f, &why);
      // worth it where it lets more CTAs share an SM than the plain form
      q->frontier_pays = q->has_frontier &&
                         stream_max_ctas(q->spf, kkt_plan->device, q->ctas_limit) >
                             stream_max_ctas(q->sp, kkt_plan->device, q->ctas_limit);
    }
  }
  *out = q;
  return WMPC_OK;
}

int wmpc_osqp_destroy(wmpc_osqp* osqp) {
  if (!osqp) return WMPC_OK;
  DeviceGuard guard(osqp->device);
  if (osqp->block) cudaFree(osqp->block);
  if (osqp->stream_block) cudaFree(osqp->stream_block);
  if (osqp->stream_block_f) cudaFree(osqp->stream_block_f);
  delete osqp;
  return WMPC_OK;
}

int wmpc_osqp_stream_info(const wmpc_osqp* osqp, int32_t info[4]) {
  if (!osqp || !info) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  // (the schedule a fixed-iteration solve of more tiles than SMs runs)
  const wmpc::StreamPlan& sp = osqp->frontier_pays ? osqp->spf : osqp->sp;
  info[0] = osqp->has_stream ? 1 : 0;
  info[1] = osqp->has_stream ? sp.frontier_slots : 0;
  info[2] = osqp->has_stream ? sp.n : 0;
  info[3] = osqp->has_stream ? sp.frontier_lag : 0;
  return WMPC_OK;
}

size_t wmpc_osqp_workspace_bytes(const wmpc_osqp* osqp, int32_t batch, int32_t mode, int32_t external_factor) {
  if (!osqp || batch <= 0) return 0;
  // P/A value batches may be 1 or `batch`; size for the larger case, and
  // for the factorization-only call as well
  const size_t solve = osqp_workspace_bytes(*osqp, batch, batch, batch, mode, external_factor != 0);
  const size_t fac = osqp_factor_workspace_bytes(osqp->dev, osqp->kkt_plan->pat, batch, batch);
  return solve > fac ? solve : fac;
}

size_t wmpc_osqp_adjoint_workspace_bytes(const wmpc_osqp* osqp, int32_t batch, int32_t mode) {
  if (!osqp || batch <= 0) return 0;
  return osqp_workspace_bytes(*osqp, batch, batch, batch, mode, false) + osqp_adjoint_extra_bytes(osqp->dev, batch);
}

int wmpc_osqp_adjoint(const wmpc_osqp* osqp, const wmpc_osqp_options* options, const wmpc_osqp_adjoint_batch* data,
                      int32_t mode, void* workspace, size_t workspace_bytes, wmpc_stream_t stream) {
  if (!osqp || !options || !data) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  if (mode != WMPC_OSQP_PLAIN && mode != WMPC_OSQP_PERSISTENT) return fail(WMPC_ERR_INVALID_ARGUMENT, "unknown mode %d", mode);
  const wmpc_osqp_adjoint_batch& a = *data;
  if (a.batch < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "negative batch");
  if (a.batch == 0) return WMPC_OK;
  if ((a.p_batch != 1 && a.p_batch != a.batch) || (a.a_batch != 1 && a.a_batch != a.batch))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "p_batch/a_batch must be 1 or batch");
  if (!a.p_values || !a.a_values || !a.l || !a.u || !a.x || !a.z || !a.y || !a.dx || !a.dq || !a.dl || !a.du)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "null buffer");
  if (options->max_iter < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "max_iter must be nonnegative");
  DeviceGuard guard(osqp->device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", osqp->device);
  return osqp_adjoint(*osqp, *options, a, mode, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

int wmpc_osqp_factor(const wmpc_osqp* osqp, const float* p_values, int32_t p_batch, const float* a_values,
                     int32_t a_batch, float* lx, float* d, float* dinv, void* workspace, size_t workspace_bytes,
                     wmpc_stream_t stream) {
  if (!osqp || !p_values || !a_values || (!lx && osqp->kkt_plan->pat.nnz_l > 0) || !d || !dinv)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  if (p_batch <= 0 || a_batch <= 0 || (p_batch != 1 && a_batch != 1 && p_batch != a_batch))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "p_batch/a_batch must be positive and equal unless one is 1");
  DeviceGuard guard(osqp->device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", osqp->device);
  return osqp_factor(osqp->dev, *osqp->kkt_plan, p_values, p_batch, a_values, a_batch, lx, d, dinv, workspace,
                     workspace_bytes, static_cast<cudaStream_t>(stream));
}

int wmpc_osqp_solve(const wmpc_osqp* osqp, const wmpc_osqp_options* options, const wmpc_osqp_batch* data,
                    const float* lx, const float* dinv, int32_t factor_batch, int32_t mode, void* workspace,
                    size_t workspace_bytes, wmpc_stream_t stream) {
  if (!osqp || !options || !data) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  if (mode != WMPC_OSQP_PLAIN && mode != WMPC_OSQP_PERSISTENT) return fail(WMPC_ERR_INVALID_ARGUMENT, "unknown mode %d", mode);
  const wmpc_osqp_batch& d = *data;
  if (d.batch < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "negative batch");
  if (d.batch == 0) return WMPC_OK;
  if ((d.p_batch != 1 && d.p_batch != d.batch) || (d.a_batch != 1 && d.a_batch != d.batch))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "p_batch/a_batch must be 1 or batch");
  if (!d.p_values || !d.a_values || !d.q || !d.l || !d.u || !d.x || !d.z || !d.y || !d.prim_res || !d.dual_res || !d.obj)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "null buffer");
  if ((lx == nullptr) != (dinv == nullptr)) return fail(WMPC_ERR_INVALID_ARGUMENT, "lx and dinv go together");
  if (lx && factor_batch != 1 && factor_batch != d.batch)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "factor_batch must be 1 or batch");
  if (options->max_iter < 0 || options->check_termination < 0)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "max_iter and check_termination must be nonnegative");
  if (mode == WMPC_OSQP_PLAIN && options->check_termination > 0)
    return fail(WMPC_ERR_UNSUPPORTED, "the per-call path runs exactly max_iter iterations (check_termination=0)");
  DeviceGuard guard(osqp->device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", osqp->device);
  return osqp_solve(*osqp, *options, d, lx, dinv, factor_batch, mode, workspace, workspace_bytes,
                    static_cast<cudaStream_t>(stream));
}

int wmpc_osqp_solve_persistent(const wmpc_osqp* const* osqps, const wmpc_osqp_options* options,
                               const wmpc_osqp_batch* data, int32_t n_classes, void* const* workspaces,
                               const size_t* workspace_bytes, wmpc_stream_t stream) {
  if (!osqps || !options || !data || !workspaces || !workspace_bytes) return fail(WMPC_ERR_INVALID_ARGUMENT, "null argument");
  if (n_classes < 1 || n_classes > 6) return fail(WMPC_ERR_INVALID_ARGUMENT, "n_classes must be 1..6, got %d", n_classes);
  for (int i = 0; i < n_classes; ++i) {
    const wmpc_osqp_batch& d = data[i];
    if (!osqps[i]) return fail(WMPC_ERR_INVALID_ARGUMENT, "null handle for class %d", i);
    if (d.batch < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "negative batch (class %d)", i);
    if (d.batch == 0) continue;
    if ((d.p_batch != 1 && d.p_batch != d.batch) || (d.a_batch != 1 && d.a_batch != d.batch))
      return fail(WMPC_ERR_INVALID_ARGUMENT, "p_batch/a_batch must be 1 or batch (class %d)", i);
    if (!d.p_values || !d.a_values || !d.q || !d.l || !d.u || !d.x || !d.z || !d.y || !d.prim_res || !d.dual_res ||
        !d.obj)
      return fail(WMPC_ERR_INVALID_ARGUMENT, "null buffer (class %d)", i);
    if (options[i].max_iter < 0 || options[i].check_termination < 0)
      return fail(WMPC_ERR_INVALID_ARGUMENT, "max_iter and check_termination must be nonnegative (class %d)", i);
    if (options[i].reuse_factor) return fail(WMPC_ERR_UNSUPPORTED, "multi-class solves factor every class");
  }
  DeviceGuard guard(osqps[0]->device);
  if (!guard.ok) return fail(WMPC_ERR_CUDA, "cannot select device %d", osqps[0]->device);
  return osqp_solve_multi(osqps, options, data, n_classes, workspaces, workspace_bytes,
                          static_cast<cudaStream_t>(stream));
}

}  // extern "C"
