// Host construction of the factorization's compact-accumulator tables and of
// the streaming sweep schedule (chunks, stream positions, release order).
#include <algorithm>
#include <cstring>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include "stream.cuh"

namespace wmpc {

// Compact accumulator: row k of the factorization only touches the entries of
// its etree reach (the columns visited by its row program), so the dense work
// vector y can be replaced by one slot per reach position.  init_slot[e] and
// upd_slot[u] give, for every scattered update of the row program, the slot
// of its target row.
bool build_factor_tables(const HostPattern& hp, std::vector<int>* init_slot, std::vector<int>* upd_ptr,
                         std::vector<unsigned short>* upd_slot, int* max_row_nnz, std::string* why) {
  const int n = hp.n;
  std::vector<int> slot_of(n, -1);
  init_slot->assign(hp.init_rows.size(), 0);
  upd_ptr->assign(hp.nnz_l + 1, 0);
  upd_slot->clear();
  *max_row_nnz = 0;
  for (int k = 0; k < n; ++k) {
    const int p0 = hp.proc_ptr[k], p1 = hp.proc_ptr[k + 1];
    *max_row_nnz = std::max(*max_row_nnz, p1 - p0);
    if (p1 - p0 > 65535) {
      *why = "row reach exceeds 65535 entries";
      return false;
    }
    for (int e = p0; e < p1; ++e) slot_of[hp.proc_cols[e]] = e - p0;
    for (int e = hp.init_ptr[k]; e < hp.init_ptr[k + 1]; ++e) {
      const int s = slot_of[hp.init_rows[e]];
      if (s < 0) {
        *why = "init row outside the etree reach";
        return false;
      }
      (*init_slot)[e] = s;
    }
    for (int e = p0; e < p1; ++e) {
      const int c = hp.proc_cols[e];
      (*upd_ptr)[e] = static_cast<int>(upd_slot->size());
      for (int q = 0; q < hp.proc_offsets[e]; ++q) {
        const int s = slot_of[hp.li[hp.lp[c] + q]];
        if (s < 0) {
          *why = "update row outside the etree reach";
          return false;
        }
        upd_slot->push_back(static_cast<unsigned short>(s));
      }
    }
    for (int e = p0; e < p1; ++e) slot_of[hp.proc_cols[e]] = -1;
  }
  (*upd_ptr)[hp.nnz_l] = static_cast<int>(upd_slot->size());
  return true;
}

// Units: the sweeps are cut into units of 4 L entries of one row (forward) or
// one column (backward), stored [unit][lane][4 entries] so a lane loads its 4
// values with one 16-byte access.  Forward rows are right-aligned (padding
// first, so a row's last entry -- the one that may read the row just before
// it -- is always slot 3); backward columns are left-aligned (padding last, so
// a column's first entry -- the one that may read the column just after it --
// is always slot 0).  Padding slots hold L = 0 and read the zero row n of the
// work vector, which leaves the running sum bit-for-bit unchanged.
//
// The consumer loads unit u+1 before it stores unit u's result, so a slot of
// unit u+1 that reads unit u's target sees a stale value: the builder marks
// such a read in the designated slot (kUnitFwd: the consumer substitutes the
// register result) and separates the units by a no-op unit otherwise.
namespace {

struct UnitBuild {
  int src[4];
  int target;
  int flags;
  int doff;
};

// Cut one row (forward, right-aligned) or column (backward, left-aligned)
// with `cnt` entries into units; entry q (in accumulation order) reads
// work-vector row entry_src(q).  Returns the units; slot_of[q] receives
// (unit index within the returned vector) * 4 + slot.
template <typename Src>
std::vector<UnitBuild> cut_units(int cnt, bool right_aligned, int target, int zero_row, Src entry_src,
                                 std::vector<int>* slot_of) {
  const int nu = cnt == 0 ? 1 : (cnt + 3) / 4;
  const int pad = nu * 4 - cnt;
  std::vector<UnitBuild> units(nu);
  slot_of->assign(cnt, -1);
  for (int k = 0; k < nu; ++k) {
    UnitBuild& ub = units[k];
    ub.target = target;
    ub.flags = (k == 0 ? kUnitFirst : 0) | (k == nu - 1 ? kUnitLast : 0);
    ub.doff = 0;
    for (int s = 0; s < 4; ++s) {
      const int q = right_aligned ? k * 4 + s - pad : k * 4 + s;
      if (q < 0 || q >= cnt) {
        ub.src[s] = zero_row;
      } else {
        ub.src[s] = entry_src(q);
        (*slot_of)[q] = k * 4 + s;
      }
    }
  }
  return units;
}

// Append one row's / column's units to a chunk.  The consumer loads a unit
// before the previous unit's result is stored, so if the first new unit reads
// the previous unit's target it must do so in the forwarding slot (flag
// kUnitFwd); any other slot gets a no-op unit (flags 0, zero slots) in
// between.  Returns the index of the first appended unit.
int append_units(std::vector<UnitBuild>* chunk, std::vector<UnitBuild> add, int fwd_slot, int zero_row,
                 int* dummies) {
  if (!chunk->empty() && (chunk->back().flags & kUnitLast)) {
    const int prev_target = chunk->back().target;
    bool other = false, fwd = false;
    for (int s = 0; s < 4; ++s)
      if (add[0].src[s] == prev_target) (s == fwd_slot ? fwd : other) = true;
    if (other) {
      UnitBuild d;
      for (int s = 0; s < 4; ++s) d.src[s] = zero_row;
      d.target = zero_row;
      d.flags = 0;
      d.doff = 0;
      chunk->push_back(d);
      ++*dummies;
    } else if (fwd) {
      add[0].flags |= kUnitFwd;
    }
  }
  const int first = static_cast<int>(chunk->size());
  chunk->insert(chunk->end(), add.begin(), add.end());
  return first;
}

// Meta of unit `u` of its chunk (see stream.cuh for the word layout).
void push_unit_meta(const UnitBuild& ub, int u, int trash_row, std::vector<int>* m) {
  for (int s = 0; s < 4; ++s) m->push_back(ub.src[s] * 128);
  m->push_back(ub.target * 128);
  m->push_back(ub.flags | (ub.doff << kUnitDoffShift));
  m->push_back(u * 512);
  m->push_back(((ub.flags & kUnitLast) ? ub.target : trash_row) * 128);
}

// Meta of the sentinel units after a chunk's last unit.  The consumer
// computes units in groups of kUnitGroup and loads operands one unit and meta
// two units ahead, so up to kUnitSentinels units past the last one are read
// and some computed: they read the zero row and unit 0's L values, and store
// to the trash row.
void push_sentinels(int zero_row, int trash_row, std::vector<int>* m) {
  for (int k = 0; k < kUnitSentinels; ++k) {
    for (int s = 0; s < 4; ++s) m->push_back(zero_row * 128);
    m->push_back(zero_row * 128);
    m->push_back(0);
    m->push_back(0);
    m->push_back(trash_row * 128);
  }
}

// Units of one chunk kept for the frontier pass: where the chunk's unit meta
// starts, its units in stage order, and its row (forward) or column
// (backward) range.
struct ChunkUnits {
  int word0;  // first word of unit 0 in the meta vector
  int lo, hi; // rows [lo, hi) (forward) or columns [lo, hi) (backward)
  int nu;     // units (= meta words / kUnitWords before the sentinels)
  int rel_word0 = -1, u0 = 0, nrel = 0;  // backward: release records
  std::vector<UnitBuild> units;
  std::vector<int> copies;  // forward: rows without entries copied into their slots at chunk start
  int copy_word0 = -1;      // their (stage offset, slot offset) pairs in the meta vector
};

// Slots for the values of one sweep phase.  A value gets a slot when the unit
// that finishes it stores it and keeps it through its last read; the slot is
// reusable `gap` time steps later (two units: a unit's operands are loaded
// before the previous unit stores).  Values nothing reads later go to the
// trash slot.  Returns the slot of every value (-1: none) and the number of
// slots used.
std::vector<int> assign_slots(int n_values, const std::vector<int>& write_t, const std::vector<int>& free_after,
                              int* n_slots, int gap = 2) {
  std::vector<int> by_time(n_values);
  std::iota(by_time.begin(), by_time.end(), 0);
  std::sort(by_time.begin(), by_time.end(), [&](int a, int b) { return write_t[a] < write_t[b]; });
  std::vector<int> slot(n_values, -1);
  std::priority_queue<int, std::vector<int>, std::greater<int>> free_slots;
  using Pending = std::pair<int, int>;  // (reusable from time, slot)
  std::priority_queue<Pending, std::vector<Pending>, std::greater<Pending>> pending;
  int used = 0;
  for (int v : by_time) {
    if (write_t[v] < 0 || free_after[v] < 0) continue;  // never written, or never read after its store
    while (!pending.empty() && pending.top().first <= write_t[v]) {
      free_slots.push(pending.top().second);
      pending.pop();
    }
    int sl;
    if (free_slots.empty()) {
      sl = used++;
    } else {
      sl = free_slots.top();
      free_slots.pop();
    }
    slot[v] = sl;
    pending.push({free_after[v] + gap, sl});
  }
  *n_slots = used;
  return slot;
}

// Frontier mode: rename the work-vector rows of every unit and release record
// to slots, so the work vector holds only what a sweep still reads.  The
// right-hand sides move to a per-tile vector R read through each forward
// chunk's stage (block of rows [lo, hi) after its units, where the units also
// leave the rows' forward results); the forward results to a vector Y read
// through each backward chunk's stage (block of columns [lo, hi) after the
// D^-1 rows).  Unit words: sources and store become slot offsets, the target
// becomes the byte offset of `t` in the stage's L area (a forward unit has no
// D^-1 offset: its flags word is the flags alone); release records carry the
// released index's slot and, in place of the unscale factor, the index (its R
// entry).  Sentinels and no-op units read stage offset 0.
bool build_frontier_slots(int n, int lag, const std::vector<ChunkUnits>& fwd, const std::vector<ChunkUnits>& bwd,
                          const std::vector<int>& order, HostStream* S, std::string* why) {
  const int zero_row = n;
  // ---- forward phase: values y_i, written by the last unit of row i, or (a
  // row without entries) copied from the stage before its chunk's first unit.
  // Time: unit k at 2k + 2, a chunk's copies at 2k + 1 (k its first unit).
  std::vector<int> f_write(n, -1), f_read(n, -1);
  int tau = 0;
  for (const ChunkUnits& c : fwd) {
    for (int row : c.copies) f_write[row] = 2 * tau + 1;
    for (const UnitBuild& ub : c.units) {
      for (int s2 = 0; s2 < 4; ++s2)
        if (ub.src[s2] != zero_row) f_read[ub.src[s2]] = std::max(f_read[ub.src[s2]], 2 * tau + 2);
      if ((ub.flags & kUnitLast) && ub.target != zero_row) f_write[ub.target] = 2 * tau + 2;
      ++tau;
    }
  }
  std::vector<int> f_free(n, -1);
  for (int v = 0; v < n; ++v)
    if (f_read[v] > f_write[v] && f_write[v] >= 0) f_free[v] = f_read[v];
  int f_slots = 0;
  const std::vector<int> fslot = assign_slots(n, f_write, f_free, &f_slots, 4);
  // ---- backward phase (chunks in sweep order: last chunk first): values x_j
  std::vector<int> b_write(n, -1), b_read(n, -1), chunk_end;
  tau = 0;
  for (int k = static_cast<int>(bwd.size()) - 1; k >= 0; --k) {
    for (const UnitBuild& ub : bwd[k].units) {
      for (int s2 = 0; s2 < 4; ++s2)
        if (ub.src[s2] != zero_row) b_read[ub.src[s2]] = std::max(b_read[ub.src[s2]], tau);
      if ((ub.flags & kUnitLast) && ub.target != zero_row) b_write[ub.target] = tau;
      ++tau;
    }
    chunk_end.push_back(tau - 1);
  }
  // a release may run until the sweep is `lag` chunks further (ring depth)
  const int nb = static_cast<int>(bwd.size());
  for (int p = 0; p < nb; ++p) {
    const ChunkUnits& c = bwd[nb - 1 - p];
    const int t_rel = chunk_end[std::min(nb - 1, p + lag - 1)];
    for (int k = 0; k < c.nrel; ++k) {
      const int i = order[c.u0 + k];
      if (b_write[i] < 0 || b_write[i] > t_rel) {
        *why = "frontier: a release precedes its column";
        return false;
      }
      b_read[i] = std::max(b_read[i], t_rel);
    }
  }
  std::vector<int> b_free(n, -1);
  for (int v = 0; v < n; ++v)
    if (b_write[v] >= 0) b_free[v] = std::max(b_read[v], b_write[v] + 1);
  int b_slots = 0;
  const std::vector<int> bslot = assign_slots(n, b_write, b_free, &b_slots);
  const int F = std::max(f_slots, b_slots);
  const int zs = F, ts = F + 1;
  if (F + 2 > (1 << 20)) {
    *why = "frontier: too many slots";
    return false;
  }
  auto sentinel_words = [&](std::vector<int>& m, int w0) {
    for (int k = 0; k < kUnitSentinels; ++k) {
      int* w = &m[w0 + k * kUnitWords];
      for (int s2 = 0; s2 < 4; ++s2) w[s2] = zs * 128;
      w[4] = 0;
      w[5] = 0;
      w[6] = 0;
      w[7] = ts * 128;
    }
  };
  // ---- rewrite the forward meta
  for (const ChunkUnits& c : fwd) {
    for (int u = 0; u < c.nu; ++u) {
      const UnitBuild& ub = c.units[u];
      int* w = &S->fmeta[c.word0 + u * kUnitWords];
      for (int s2 = 0; s2 < 4; ++s2) {
        const int r = ub.src[s2];
        if (r != zero_row && fslot[r] < 0) {
          *why = "frontier: a forward read without a slot";
          return false;
        }
        w[s2] = (r == zero_row ? zs : fslot[r]) * 128;
      }
      const bool real = ub.target != zero_row;
      w[4] = real ? c.nu * 512 + (ub.target - c.lo) * 128 : 0;
      w[5] = ub.flags;
      const bool keep = (ub.flags & kUnitLast) && real && fslot[ub.target] >= 0;
      w[7] = (keep ? fslot[ub.target] : ts) * 128;
    }
    sentinel_words(S->fmeta, c.word0 + c.nu * kUnitWords);
    for (size_t k = 0; k < c.copies.size(); ++k) {
      const int row = c.copies[k];
      S->fmeta[c.copy_word0 + 2 * k] = c.nu * 512 + (row - c.lo) * 128;
      S->fmeta[c.copy_word0 + 2 * k + 1] = (fslot[row] >= 0 ? fslot[row] : ts) * 128;
    }
  }
  // ---- rewrite the backward meta and release records
  for (const ChunkUnits& c : bwd) {
    const int ncols = c.hi - c.lo;
    for (int u = 0; u < c.nu; ++u) {
      const UnitBuild& ub = c.units[u];
      int* w = &S->meta[c.word0 + u * kUnitWords];
      for (int s2 = 0; s2 < 4; ++s2) {
        const int r = ub.src[s2];
        if (r != zero_row && bslot[r] < 0) {
          *why = "frontier: a backward read without a slot";
          return false;
        }
        w[s2] = (r == zero_row ? zs : bslot[r]) * 128;
      }
      const bool real = ub.target != zero_row;
      w[4] = real ? c.nu * 512 + ncols * 128 + (ub.target - c.lo) * 128 : 0;
      w[7] = ((ub.flags & kUnitLast) && real ? bslot[ub.target] : ts) * 128;
    }
    for (int l = 0; l < 3; ++l) sentinel_words(S->meta, c.word0 + (c.nu + l * kUnitSentinels) * kUnitWords);
    for (int k = 0; k < c.nrel; ++k) {
      const int i = order[c.u0 + k];
      S->meta[c.rel_word0 + 4 * k] = bslot[i] * 128;
      S->meta[c.rel_word0 + 4 * k + 3] = i;
    }
  }
  S->frontier_slots = F;
  S->frontier_lag = lag;
  return true;
}

// Every word the streaming kernel reads in the frontier form, checked against
// what it addresses: slots inside the work vector (zero and trash slot
// included), stage offsets inside the chunk's L area plus its right-hand-side
// or forward-result block, rows, columns and released indices inside [0, n).
bool check_frontier_tables(const HostStream& S, int n, std::string* why) {
  const int F = S.frontier_slots;
  auto bad = [&](const char* what, int ch) {
    *why = std::string("frontier table check: ") + what + " (chunk " + std::to_string(ch) + ")";
    return false;
  };
  auto slot_ok = [&](int w, int top) { return w >= 0 && w % 128 == 0 && w / 128 <= top; };
  for (int ch = 0; ch < S.n_fchunks; ++ch) {
    const int* m = &S.fmeta[S.fmeta_off[ch]];
    const int nu = m[0], r0 = m[1], r1 = m[2], ncopy = m[3];
    if (nu != S.fchunk_units[ch] || nu < 0 || nu > S.max_funits || ncopy < 0 || nu + ncopy < 1)
      return bad("forward units", ch);
    if (r0 < 0 || r1 <= r0 || r1 > n || r1 - r0 > S.max_frows) return bad("forward rows", ch);
    if (S.frow0[ch] != r0 || S.frows[ch] != r1 - r0) return bad("forward row table", ch);
    const int copy0 = kChunkHeader + (nu + kUnitSentinels) * kUnitWords;
    if (S.fmeta_words[ch] < copy0 + 2 * ncopy) return bad("forward meta size", ch);
    const int area = nu * 512 + (r1 - r0) * 128;
    for (int k = 0; k < ncopy; ++k) {
      const int src = m[copy0 + 2 * k], dst = m[copy0 + 2 * k + 1];
      if (src < nu * 512 || src % 128 != 0 || src + 128 > area || !slot_ok(dst, F + 1)) return bad("forward copy", ch);
    }
    for (int u = 0; u < (nu > 0 ? nu + kUnitSentinels : 0); ++u) {
      const int* w = m + kChunkHeader + u * kUnitWords;
      for (int s2 = 0; s2 < 4; ++s2)
        if (!slot_ok(w[s2], F)) return bad("forward source slot", ch);
      if (w[4] < 0 || w[4] % 128 != 0 || w[4] + 128 > area) return bad("forward right-hand-side offset", ch);
      if ((w[5] >> kUnitDoffShift) != 0 || (u >= nu && (w[5] & kUnitLast))) return bad("forward flags", ch);
      if (w[6] < 0 || w[6] % 512 != 0 || w[6] + 512 > nu * 512) return bad("forward L offset", ch);
      if (!slot_ok(w[7], F + 1)) return bad("forward store slot", ch);
    }
  }
  for (int ch = 0; ch < S.n_chunks; ++ch) {
    const int* m = &S.meta[S.meta_off[ch]];
    const int ns = m[0], ncols = m[1], nrel = m[2], c0 = m[3], u0 = m[4];
    if (m[6] != 0 || m[7] != 0) return bad("releaser units", ch);
    if (ns != S.chunk_units[ch] || ns < 0 || ns > S.max_units) return bad("backward units", ch);
    if (ncols != S.chunk_cols[ch] || ncols < 0 || ncols > S.max_cols || c0 < 0 || c0 + ncols > n ||
        S.chunk_c0[ch] != c0)
      return bad("backward columns", ch);
    if (nrel < 0 || nrel > S.max_rel || u0 < 0 || u0 + nrel > n) return bad("releases", ch);
    const int rel0 = kChunkHeader + (ns + 3 * kUnitSentinels) * kUnitWords;
    if (S.meta_words[ch] < rel0 + 4 * nrel) return bad("backward meta size", ch);
    const int dend = ns * 512 + ncols * 128, area = dend + ncols * 128;
    for (int u = 0; u < ns + kUnitSentinels; ++u) {
      const int* w = m + kChunkHeader + u * kUnitWords;
      for (int s2 = 0; s2 < 4; ++s2)
        if (!slot_ok(w[s2], F)) return bad("backward source slot", ch);
      if (w[4] < 0 || w[4] % 128 != 0 || (u < ns && w[4] + 128 > area)) return bad("backward forward-result offset", ch);
      const int doff = w[5] >> kUnitDoffShift;
      if (doff < 0 || doff % 128 != 0 || doff + 128 > (u < ns ? dend : 128)) return bad("backward D^-1 offset", ch);
      if (w[6] < 0 || w[6] % 512 != 0 || (u < ns && w[6] + 512 > ns * 512)) return bad("backward L offset", ch);
      if (!slot_ok(w[7], F + 1)) return bad("backward store slot", ch);
    }
    for (int k = 0; k < nrel; ++k) {
      const int* r = m + rel0 + 4 * k;
      if (!slot_ok(r[0], F - 1) || r[3] < 0 || r[3] >= n) return bad("release record", ch);
    }
  }
  return true;
}

}  // namespace

bool build_stream_schedule(const HostPattern& hp, const StreamTargets& t, const float* rho_by_constraint,
                           const float* rhoinv_by_constraint, int n_primal, HostStream* out, std::string* why,
                           const float* unscale_by_index) {
  const int n = hp.n;
  const int zero_row = n, trash_row = n + 1;
  HostStream& S = *out;
  S = HostStream();
  if (t.units <= 0 || t.cols <= 0 || t.rel <= 0 || t.funits <= 0) {
    *why = "bad stream targets";
    return false;
  }
  if (t.frontier_copies && !t.frontier) {
    *why = "frontier copies need the frontier form";
    return false;
  }
  if (t.frontier && (t.offload || t.frontier_lag < 1)) {
    *why = "frontier mode needs offload 0 and a release lag of at least one chunk";
    return false;
  }
  std::vector<ChunkUnits> fwd_units, bwd_units;  // frontier mode only
  // release column of every index: smallest column whose L entry lies in row i
  std::vector<int> rel_col(n);
  for (int i = 0; i < n; ++i) rel_col[i] = i;
  for (int c = 0; c < n; ++c)
    for (int e = hp.lp[c]; e < hp.lp[c + 1]; ++e) rel_col[hp.li[e]] = std::min(rel_col[hp.li[e]], c);
  // U order: release column descending, then index descending
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    if (rel_col[a] != rel_col[b]) return rel_col[a] > rel_col[b];
    return a > b;
  });
  std::vector<int> rel_count(n, 0);
  for (int i = 0; i < n; ++i) rel_count[rel_col[i]]++;
  std::vector<int> rel_first(n + 1, 0);
  {
    int u = 0;
    for (int c = n - 1; c >= 0; --c) {
      rel_first[c] = u;
      u += rel_count[c];
    }
  }
  // Rows of L.  A leaf row (no entries) is read by no column of the backward
  // sweep, so its column can be solved by the releaser right before its own
  // release, and its forward value is its right-hand side.  A row whose entries
  // all read leaf rows ("pre row") can be solved forward by the releaser as
  // soon as it and its leaves are released (all in the chunk of its release
  // column).  The sweeper walks everything else.
  std::vector<int> rcount(n, 0);
  std::vector<std::vector<int>> row_entries(n);  // CSC entry indices of each row, columns ascending
  std::vector<int> col_of(hp.nnz_l);
  for (int c = 0; c < n; ++c)
    for (int e = hp.lp[c]; e < hp.lp[c + 1]; ++e) {
      rcount[hp.li[e]]++;
      row_entries[hp.li[e]].push_back(e);
      col_of[e] = c;
    }
  std::vector<char> pre_row(n, 0), leaf_col(n, 0);
  for (int i = 0; i < n; ++i) leaf_col[i] = (t.offload & 1) && rcount[i] == 0;
  for (int i = 0; i < n && (t.offload & 2); ++i) {
    if (rcount[i] == 0) continue;
    bool all_leaf = true;
    for (int e : row_entries[i]) all_leaf = all_leaf && rcount[col_of[e]] == 0;
    pre_row[i] = all_leaf ? 1 : 0;
  }
  auto col_units = [&](int c) { const int ce = hp.lp[c + 1] - hp.lp[c]; return ce == 0 ? 1 : (ce + 3) / 4; };
  std::vector<int> pre_units_at(n, 0);  // pre-row units run in the chunk of the row's release column
  for (int i = 0; i < n; ++i)
    if (pre_row[i]) pre_units_at[rel_col[i]] += (rcount[i] + 3) / 4;
  // ---- backward chunks: whole columns, units <= t.units, columns <= t.cols, releases <= t.rel
  std::vector<int> bounds{0};
  {
    int units = 0, cols = 0, rel = 0;
    for (int c = 0; c < n; ++c) {
      const int cu = col_units(c) + pre_units_at[c], cr = rel_count[c];
      if (cols > 0 && (units + cu > t.units || cols + 1 > t.cols || rel + cr > t.rel)) {
        bounds.push_back(c);
        units = cols = rel = 0;
      }
      units += cu;
      cols += 1;
      rel += cr;
    }
    bounds.push_back(n);
  }
  S.n_chunks = static_cast<int>(bounds.size()) - 1;
  S.chunk_off.resize(S.n_chunks + 1);
  S.chunk_units.resize(S.n_chunks);
  S.chunk_cols.resize(S.n_chunks);
  S.chunk_u0.resize(S.n_chunks);
  S.chunk_c0.resize(S.n_chunks);
  S.chunk_nrel.resize(S.n_chunks);
  S.meta_off.resize(S.n_chunks);
  S.meta_words.resize(S.n_chunks);
  S.col_uoff.assign(n, 0);
  S.dinv_off.assign(n, 0);
  std::vector<int> entry_boff(hp.nnz_l, -1);  // CSC entry -> backward stream float offset (lane 0)
  std::vector<int> entry_foff(hp.nnz_l, -1);  // CSC entry -> forward position; -1 - offset: a pre unit slot
  int boff = 0;                                // running float offset in the backward stream
  for (int ch = 0; ch < S.n_chunks; ++ch) {
    const int c0 = bounds[ch], c1 = bounds[ch + 1];
    // three unit lists: sweeper columns, leaf columns, pre rows; placement is (list, index, slot)
    std::vector<UnitBuild> lists[3];
    std::vector<int> col_list(c1 - c0), col_first(c1 - c0), col_last(c1 - c0);
    struct Placed { int entry, list, pos; };  // pos = unit * 4 + slot within its list
    std::vector<Placed> placed, placed_pre;
    for (int c = c1 - 1; c >= c0; --c) {  // the order the backward sweep visits the columns
      const int e0 = hp.lp[c], cnt = hp.lp[c + 1] - e0;
      const int li = leaf_col[c] ? 1 : 0;
      std::vector<int> slot_of;
      std::vector<UnitBuild> add = cut_units(cnt, false, c, zero_row, [&](int q) { return hp.li[e0 + q]; }, &slot_of);
      const int nadd = static_cast<int>(add.size());
      const int first = append_units(&lists[li], std::move(add), 0, zero_row, &S.dummy_units);
      col_list[c - c0] = li;
      col_first[c - c0] = first;
      col_last[c - c0] = first + nadd - 1;
      for (int q = 0; q < cnt; ++q) placed.push_back({e0 + q, li, first * 4 + slot_of[q]});
    }
    for (int v = 0; v < n; ++v) {
      if (!pre_row[v] || rel_col[v] < c0 || rel_col[v] >= c1) continue;
      const std::vector<int>& re = row_entries[v];
      const int cnt = static_cast<int>(re.size());
      std::vector<int> slot_of;
      std::vector<UnitBuild> add = cut_units(cnt, true, v, zero_row, [&](int q) { return col_of[re[q]]; }, &slot_of);
      const int first = append_units(&lists[2], std::move(add), 3, zero_row, &S.dummy_units);
      for (int q = 0; q < cnt; ++q) placed_pre.push_back({re[q], 2, first * 4 + slot_of[q]});
    }
    const int ns = static_cast<int>(lists[0].size()), nl = static_cast<int>(lists[1].size());
    const int np = static_cast<int>(lists[2].size());
    const int base[3] = {0, ns, ns + nl};  // unit index of each list in the stage
    const int nu = ns + nl + np;
    const int units_floats = nu * 128;
    auto stream_pos = [&](const Placed& pl) {
      const int u = base[pl.list] + (pl.pos >> 2);
      return boff + u * 128 + (pl.pos & 3);
    };
    for (const Placed& pl : placed) entry_boff[pl.entry] = stream_pos(pl);
    for (const Placed& pl : placed_pre) entry_foff[pl.entry] = -1 - stream_pos(pl);
    for (int c = c0; c < c1; ++c) {
      const int li = col_list[c - c0];
      S.col_uoff[c] = boff + (base[li] + col_first[c - c0]) * 128;
      S.dinv_off[c] = boff + units_floats + (c - c0) * 32;
      // D^-1 offset (bytes, relative to the stage's L area) on the column's last unit
      lists[li][col_last[c - c0]].doff = (units_floats + (c - c0) * 32) * 4;
    }
    int nrel = 0;
    for (int c = c0; c < c1; ++c) nrel += rel_count[c];
    const int u0 = rel_first[c1 - 1];
    S.chunk_off[ch] = boff;
    S.chunk_pre_u0.push_back(ns + nl);
    S.chunk_pre_units.push_back(np);
    S.chunk_units[ch] = nu;
    S.chunk_cols[ch] = c1 - c0;
    S.chunk_c0[ch] = c0;
    S.chunk_u0[ch] = u0;
    S.chunk_nrel[ch] = nrel;
    S.max_units = std::max(S.max_units, nu);
    S.max_cols = std::max(S.max_cols, c1 - c0);
    S.max_rel = std::max(S.max_rel, nrel);
    boff += units_floats + (c1 - c0) * 32;
    // meta block: header, the three unit lists (each followed by its sentinels), releases
    // the chunk's releases: primal indices first, then constraints (two branch-free loops)
    for (int u = u0; u < u0 + nrel; ++u)
      if (rel_col[order[u]] < c0 || rel_col[order[u]] >= c1) {
        *why = "release order does not match the chunking";
        return false;
      }
    std::stable_partition(order.begin() + u0, order.begin() + u0 + nrel,
                          [&](int i) { return hp.p[i] < n_primal; });
    int nprim = 0;
    for (int u = u0; u < u0 + nrel; ++u) nprim += hp.p[order[u]] < n_primal ? 1 : 0;
    std::vector<int> m{ns, c1 - c0, nrel, c0, u0, nprim, nl, np};
    for (int li = 0; li < 3; ++li) {
      for (int u = 0; u < static_cast<int>(lists[li].size()); ++u) push_unit_meta(lists[li][u], base[li] + u, trash_row, &m);
      push_sentinels(zero_row, trash_row, &m);
    }
    std::vector<int> rel_i, rel_rho, rel_rinv, rel_unscale;
    for (int u = u0; u < u0 + nrel; ++u) {
      const int i = order[u];
      const int o = hp.p[i];
      rel_i.push_back(i * 128);
      {
        const float f = unscale_by_index ? unscale_by_index[o] : 1.0f;
        int fb;
        memcpy(&fb, &f, 4);
        rel_unscale.push_back(fb);
      }
      const bool cons = o >= n_primal;
      float rho = 0.f, rinv = 0.f;
      if (cons && rho_by_constraint) {
        rho = rho_by_constraint[o - n_primal];
        rinv = rhoinv_by_constraint[o - n_primal];
      }
      int rb, ib;
      memcpy(&rb, &rho, 4);
      memcpy(&ib, &rinv, 4);
      rel_rho.push_back(rb);
      rel_rinv.push_back(ib);
    }
    for (int k = 0; k < nrel; ++k) {  // one 16-byte record per release
      m.push_back(rel_i[k]);
      m.push_back(rel_rho[k]);
      m.push_back(rel_rinv[k]);
      m.push_back(rel_unscale[k]);
    }
    while (m.size() % 4) m.push_back(0);
    S.meta_off[ch] = static_cast<int>(S.meta.size());
    S.meta_words[ch] = static_cast<int>(m.size());
    if (t.frontier) {
      ChunkUnits cu;
      cu.word0 = S.meta_off[ch] + kChunkHeader;
      cu.lo = c0;
      cu.hi = c1;
      cu.nu = ns;
      cu.rel_word0 = S.meta_off[ch] + kChunkHeader + (ns + nl + np + 3 * kUnitSentinels) * kUnitWords;
      cu.u0 = u0;
      cu.nrel = nrel;
      cu.units = lists[0];
      bwd_units.push_back(std::move(cu));
    }
    S.max_meta_words = std::max(S.max_meta_words, static_cast<int>(m.size()));
    S.max_meta_lead = std::max(S.max_meta_lead, static_cast<int>(m.size()) - 4 * nrel);
    S.meta.insert(S.meta.end(), m.begin(), m.end());
    for (int li = 0; li < 3; ++li)
      for (int u = 0; u < static_cast<int>(lists[li].size()); ++u)
        for (int s2 = 0; s2 < 4; ++s2)
          if (lists[li][u].src[s2] == zero_row) S.pad_boff.push_back(S.chunk_off[ch] + (base[li] + u) * 128 + s2);
  }
  S.chunk_off[S.n_chunks] = boff;
  S.blen = boff;
  S.u_perm = order;
  S.u_orig.resize(n);
  S.u_of_perm.resize(n);
  for (int u = 0; u < n; ++u) {
    S.u_orig[u] = hp.p[order[u]];
    S.u_of_perm[order[u]] = u;
  }
  for (int e = 0; e < hp.nnz_l; ++e)
    if (entry_boff[e] < 0) {
      *why = "backward stream misses an entry";
      return false;
    }
  // ---- forward sweep (sweeper): rows in order (row-gather form), columns ascending in a row; pre rows excluded
  {
    // (frontier mode: a row without entries gets one no-op unit that carries
    // its right-hand side into its forward value, or with frontier_copies a
    // copy from the stage into its slot at chunk start, sized here as a unit)
    auto row_units = [&](int i) { return pre_row[i] ? 0 : t.frontier && rcount[i] == 0 ? 1 : (rcount[i] + 3) / 4; };
    std::vector<int> fb{0};
    {
      int units = 0;
      for (int i = 0; i < n; ++i) {
        const int ru = row_units(i);
        if (units > 0 && units + ru > t.funits) {
          fb.push_back(i);
          units = 0;
        }
        units += ru;
      }
      fb.push_back(n);
    }
    // drop empty chunks (rows without sweeper work only)
    int foff = 0;
    for (size_t k = 0; k + 1 < fb.size(); ++k) {
      const int r0 = fb[k], r1 = fb[k + 1];
      std::vector<UnitBuild> units;
      std::vector<std::pair<int, int>> placed;
      std::vector<int> copies;
      for (int i = r0; i < r1; ++i) {
        const std::vector<int>& re = row_entries[i];
        const int cnt = static_cast<int>(re.size());
        if ((cnt == 0 && !t.frontier) || pre_row[i]) continue;
        if (cnt == 0 && t.frontier_copies) {
          copies.push_back(i);
          continue;
        }
        std::vector<int> slot_of;
        std::vector<UnitBuild> add = cut_units(cnt, true, i, zero_row, [&](int q) { return col_of[re[q]]; }, &slot_of);
        const int first = append_units(&units, std::move(add), 3, zero_row, &S.dummy_units);
        for (int q = 0; q < cnt; ++q) placed.emplace_back(re[q], first * 4 + slot_of[q]);
      }
      const int nu = static_cast<int>(units.size());
      const int ncopy = static_cast<int>(copies.size());
      if (nu == 0 && ncopy == 0) continue;
      for (const auto& pe : placed) entry_foff[pe.first] = foff + (pe.second >> 2) * 128 + (pe.second & 3);
      std::vector<int> m{nu, t.frontier ? r0 : 0, t.frontier ? r1 : 0, ncopy, 0, 0, 0, 0};
      for (int u = 0; u < nu; ++u) push_unit_meta(units[u], u, trash_row, &m);
      push_sentinels(zero_row, trash_row, &m);
      // frontier copies: (stage offset of the row's right-hand side, slot offset) pairs
      const int copy_word0 = static_cast<int>(S.fmeta.size() + m.size());
      for (int k = 0; k < 2 * ncopy; ++k) m.push_back(0);
      while (m.size() % 4) m.push_back(0);
      if (t.frontier) {
        ChunkUnits cu;
        cu.word0 = static_cast<int>(S.fmeta.size()) + kChunkHeader;
        cu.lo = r0;
        cu.hi = r1;
        cu.nu = nu;
        cu.units = units;
        cu.copies = copies;
        cu.copy_word0 = copy_word0;
        fwd_units.push_back(std::move(cu));
        S.max_frows = std::max(S.max_frows, r1 - r0);
      }
      S.fchunk_off.push_back(foff);
      S.fchunk_units.push_back(nu);
      S.frow0.push_back(r0);
      S.frows.push_back(r1 - r0);
      S.fmeta_off.push_back(static_cast<int>(S.fmeta.size()));
      S.fmeta_words.push_back(static_cast<int>(m.size()));
      S.max_fmeta_words = std::max(S.max_fmeta_words, static_cast<int>(m.size()));
      S.max_funits = std::max(S.max_funits, nu);
      S.fmeta.insert(S.fmeta.end(), m.begin(), m.end());
      for (int u = 0; u < nu; ++u)
        for (int s2 = 0; s2 < 4; ++s2)
          if (units[u].src[s2] == zero_row) S.pad_foff.push_back(foff + u * 128 + s2);
      foff += nu * 128;
    }
    S.n_fchunks = static_cast<int>(S.fchunk_units.size());
    S.fchunk_off.push_back(foff);
    S.flen = foff;
  }
  for (int e = 0; e < hp.nnz_l; ++e)
    if (entry_foff[e] == -1 && !pre_row[hp.li[e]]) {
      *why = "forward stream misses an entry";
      return false;
    }
  if (t.frontier && !build_frontier_slots(n, t.frontier_lag, fwd_units, bwd_units, order, &S, why)) return false;
  if (t.frontier && !check_frontier_tables(S, n, why)) return false;
  // factorization re-reads: the L entry every update reads, D^-1 of every step's column
  S.upd_pos.clear();
  S.step_doff.resize(hp.nnz_l);
  for (int k = 0; k < n; ++k) {
    S.max_row_kv = std::max(S.max_row_kv, 1 + hp.init_ptr[k + 1] - hp.init_ptr[k]);
    for (int e = hp.proc_ptr[k]; e < hp.proc_ptr[k + 1]; ++e) {
      const int c = hp.proc_cols[e];
      S.step_doff[e] = S.dinv_off[c];
      for (int q = 0; q < hp.proc_offsets[e]; ++q) S.upd_pos.push_back(S.col_uoff[c] + (q >> 2) * 128 + (q & 3));
    }
  }
  // factor program step -> stream offsets of the L entry it writes
  S.proc_boff.resize(hp.nnz_l);
  S.proc_foff.resize(hp.nnz_l);
  for (int k = 0; k < n; ++k)
    for (int e = hp.proc_ptr[k]; e < hp.proc_ptr[k + 1]; ++e) {
      S.proc_boff[e] = entry_boff[hp.proc_lidx[e]];
      S.proc_foff[e] = entry_foff[hp.proc_lidx[e]];
    }
  return true;
}

}  // namespace wmpc
