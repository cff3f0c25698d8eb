// Host construction of the factorization's compact-accumulator tables and of
// the streaming sweep schedule (chunks, stream positions, release order).
#include <algorithm>
#include <cstring>
#include <numeric>
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

bool build_stream_schedule(const HostPattern& hp, const StreamTargets& t, const float* rho_by_constraint,
                           const float* rhoinv_by_constraint, int n_primal, HostStream* out, std::string* why) {
  const int n = hp.n;
  HostStream& S = *out;
  S = HostStream();
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
  S.u_perm = order;
  S.u_orig.resize(n);
  S.u_of_perm.resize(n);
  for (int u = 0; u < n; ++u) {
    S.u_orig[u] = hp.p[order[u]];
    S.u_of_perm[order[u]] = u;
  }
  std::vector<int> rel_count(n, 0);
  for (int i = 0; i < n; ++i) rel_count[rel_col[i]]++;
  // U start of the releases of column c (U is ordered by column descending)
  std::vector<int> rel_first(n + 1, 0);
  {
    int u = 0;
    for (int c = n - 1; c >= 0; --c) {
      rel_first[c] = u;
      u += rel_count[c];
    }
  }
  // chunk columns: whole columns, entries <= t.ent, columns <= t.cols, releases <= t.rel
  std::vector<int> bounds{0};
  {
    int ent = 0, cols = 0, rel = 0;
    for (int c = 0; c < n; ++c) {
      const int ce = hp.lp[c + 1] - hp.lp[c];
      const int cr = rel_count[c];
      if (cols > 0 && (ent + ce > t.ent || cols + 1 > t.cols || rel + cr > t.rel)) {
        bounds.push_back(c);
        ent = cols = rel = 0;
      }
      ent += ce;
      cols += 1;
      rel += cr;
    }
    bounds.push_back(n);
  }
  S.n_chunks = static_cast<int>(bounds.size()) - 1;
  S.stream_len = hp.nnz_l + n;
  S.col_spos.resize(n);
  S.dinv_spos.resize(n);
  S.chunk_pos.resize(S.n_chunks + 1);
  S.chunk_ent.resize(S.n_chunks);
  S.chunk_cols.resize(S.n_chunks);
  S.meta_off.resize(S.n_chunks);
  S.meta_words.resize(S.n_chunks);
  std::vector<int> chunk_of_col(n);
  for (int ch = 0; ch < S.n_chunks; ++ch) {
    const int c0 = bounds[ch], c1 = bounds[ch + 1];
    const int e0 = hp.lp[c0], e1 = hp.lp[c1];
    S.chunk_pos[ch] = e0 + c0;
    S.chunk_ent[ch] = e1 - e0;
    S.chunk_cols[ch] = c1 - c0;
    S.max_ent = std::max(S.max_ent, e1 - e0);
    S.max_cols = std::max(S.max_cols, c1 - c0);
    int nrel = 0;
    for (int c = c0; c < c1; ++c) {
      chunk_of_col[c] = ch;
      S.col_spos[c] = hp.lp[c] + c0;
      S.dinv_spos[c] = e1 + c;
      nrel += rel_count[c];
    }
    S.max_rel = std::max(S.max_rel, nrel);
    // meta block
    const int ncols = c1 - c0, nent = e1 - e0;
    const int u0 = rel_first[c1 - 1];  // releases of the chunk start at its highest column
    S.meta_off[ch] = static_cast<int>(S.meta.size());
    std::vector<int> m;
    m.push_back(ncols);
    m.push_back(nent);
    m.push_back(nrel);
    m.push_back(c0);
    m.push_back(u0);
    for (int c = c0; c <= c1; ++c) m.push_back((c < c1 ? hp.lp[c] : e1) - e0);  // col_start
    for (int e = e0; e < e1; ++e) m.push_back(hp.li[e] * 32);  // word offset of row li[e] in the work vector
    std::vector<int> rel_i, rel_kind, rel_rho, rel_rinv;
    for (int u = u0; u < u0 + nrel; ++u) {
      const int i = order[u];
      const int o = hp.p[i];
      rel_i.push_back(i);
      const bool cons = o >= n_primal;
      rel_kind.push_back(cons ? 1 : 0);
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
    for (int v : rel_i) m.push_back(v);
    for (int v : rel_kind) m.push_back(v);
    for (int v : rel_rho) m.push_back(v);
    for (int v : rel_rinv) m.push_back(v);
    while (m.size() % 4) m.push_back(0);
    S.meta_words[ch] = static_cast<int>(m.size());
    S.max_meta_words = std::max(S.max_meta_words, static_cast<int>(m.size()));
    S.meta.insert(S.meta.end(), m.begin(), m.end());
  }
  S.chunk_pos[S.n_chunks] = S.stream_len;
  // sanity: every chunk's releases are exactly its columns' releases
  for (int ch = 0; ch < S.n_chunks; ++ch) {
    const int c0 = bounds[ch], c1 = bounds[ch + 1];
    int nrel = 0;
    for (int c = c0; c < c1; ++c) nrel += rel_count[c];
    const int u0 = rel_first[c1 - 1];
    for (int u = u0; u < u0 + nrel; ++u) {
      const int rc = rel_col[order[u]];
      if (rc < c0 || rc >= c1) {
        *why = "release order does not match the chunking";
        return false;
      }
    }
  }
  // ---- forward sweep: L in CSR order (row-gather form), chunks of whole rows
  {
    std::vector<int> rcount(n, 0);
    for (int e = 0; e < hp.nnz_l; ++e) rcount[hp.li[e]]++;
    std::vector<int> rowptr(n + 1, 0);
    for (int i = 0; i < n; ++i) rowptr[i + 1] = rowptr[i] + rcount[i];
    // CSR position of each CSC entry: within a row, columns ascending (the
    // reference's accumulation order for that row)
    std::vector<int> csr_of_csc(hp.nnz_l);
    std::vector<int> csr_col(hp.nnz_l);
    {
      std::vector<int> fillp(rowptr.begin(), rowptr.end() - 1);
      for (int c = 0; c < n; ++c)
        for (int e = hp.lp[c]; e < hp.lp[c + 1]; ++e) {
          const int pos = fillp[hp.li[e]]++;
          csr_of_csc[e] = pos;
          csr_col[pos] = c;
        }
    }
    std::vector<int> fb{0};
    int ent = 0, rows = 0;
    for (int i = 0; i < n; ++i) {
      const int re = rcount[i];
      if (rows > 0 && (ent + re > t.fent || rows + 1 > t.frows)) {
        fb.push_back(i);
        ent = rows = 0;
      }
      ent += re;
      rows += 1;
    }
    fb.push_back(n);
    S.n_fchunks = static_cast<int>(fb.size()) - 1;
    S.fchunk_pos.resize(S.n_fchunks + 1);
    S.fmeta_off.resize(S.n_fchunks);
    S.fmeta_words.resize(S.n_fchunks);
    for (int ch = 0; ch < S.n_fchunks; ++ch) {
      const int r0 = fb[ch], r1 = fb[ch + 1];
      const int e0 = rowptr[r0], e1 = rowptr[r1];
      S.fchunk_pos[ch] = e0;
      S.max_fent = std::max(S.max_fent, e1 - e0);
      S.max_frows = std::max(S.max_frows, r1 - r0);
      std::vector<int> m{r1 - r0, e1 - e0, r0, 0};
      for (int i = r0; i <= r1; ++i) m.push_back(rowptr[i] - e0);
      for (int e = e0; e < e1; ++e) m.push_back(csr_col[e] * 32);
      while (m.size() % 4) m.push_back(0);
      S.fmeta_off[ch] = static_cast<int>(S.fmeta.size());
      S.fmeta_words[ch] = static_cast<int>(m.size());
      S.max_fmeta_words = std::max(S.max_fmeta_words, static_cast<int>(m.size()));
      S.fmeta.insert(S.fmeta.end(), m.begin(), m.end());
    }
    S.fchunk_pos[S.n_fchunks] = rowptr[n];
    S.proc_fpos.resize(hp.nnz_l);
    for (int k = 0; k < n; ++k)
      for (int e = hp.proc_ptr[k]; e < hp.proc_ptr[k + 1]; ++e) S.proc_fpos[e] = csr_of_csc[hp.proc_lidx[e]];
  }
  S.proc_spos.resize(hp.nnz_l);
  for (int k = 0; k < n; ++k)
    for (int e = hp.proc_ptr[k]; e < hp.proc_ptr[k + 1]; ++e) {
      const int c = hp.proc_cols[e];
      S.proc_spos[e] = hp.proc_lidx[e] + bounds[chunk_of_col[c]];
    }
  return true;
}

}  // namespace wmpc
