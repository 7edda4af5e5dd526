// Host-side symbolic analysis for the chordal multifrontal sweeps.
//
// Each routine restates one step of the reference's pure-Python symbolic
// factorisation (chompack src/python/symbolic.py) over plain int64 arrays so
// that every output array is identical to the reference's for the same
// pattern, permutation and merge rule, while running in O(nnz) time instead
// of interpreted loops (the reference's `amalgamate` renumbering is O(Nsn^2),
// symbolic.py:322-324).  Roots of a forest carry parent[k] == k, as in the
// reference.  All routines return 0 on success and a negative code when an
// internal consistency check fails (never expected for valid input).
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../../include/chompack_b200.h"

typedef int64_t i64;

namespace {

// Depth-first postorder of the tree rooted at j (symbolic.py:6-24).
i64 tdfs(i64 j, i64 k, i64* head, const i64* next, i64* post, i64* stack) {
  i64 top = 0;
  stack[0] = j;
  while (top >= 0) {
    i64 p = stack[top];
    i64 i = head[p];
    if (i == -1) {
      top -= 1;
      post[k++] = p;
    } else {
      head[p] = next[i];
      stack[++top] = i;
    }
  }
  return k;
}

// Sorted-set union of left[offl:offl+nl] and right[offr:offr+nr], written back
// into left at offl; returns the merged length (cbase.c:64-101 / misc.py
// lmerge).  `tmp` must hold nl+nr entries.
i64 lmerge(i64* left, const i64* right, i64 offl, i64 offr, i64 nl, i64 nr, std::vector<i64>& tmp) {
  tmp.resize((size_t)(nl + nr));
  i64 il = 0, ir = 0, k = 0;
  while (il < nl && ir < nr) {
    i64 a = left[offl + il], b = right[offr + ir];
    if (a < b) { tmp[k] = a; il++; }
    else if (a > b) { tmp[k] = b; ir++; }
    else { tmp[k] = a; il++; ir++; }
    k++;
  }
  while (il < nl) tmp[k++] = left[offl + il++];
  while (ir < nr) tmp[k++] = right[offr + ir++];
  for (i64 i = 0; i < k; i++) left[offl + i] = tmp[i];
  return k;
}

}  // namespace

extern "C" {

// Elimination tree from the upper triangle of a symmetric CCS pattern
// (symbolic.py:49-72).
int chb_sym_etree(i64 n, const i64* cp, const i64* ri, i64* parent) {
  std::vector<i64> w((size_t)n);
  for (i64 k = 0; k < n; k++) {
    parent[k] = k;
    w[k] = -1;
    for (i64 p = cp[k]; p < cp[k + 1]; p++) {
      i64 i = ri[p];
      while (i != -1 && i < k) {
        i64 inext = w[i];
        w[i] = k;
        if (inext == -1) parent[i] = k;
        i = inext;
      }
    }
  }
  return 0;
}

// Postorder of a forest given by parent (roots: parent[j] == j)
// (symbolic.py:26-47).
int chb_sym_post_order(i64 n, const i64* parent, i64* post) {
  std::vector<i64> head((size_t)n, -1), next((size_t)n, 0), stack((size_t)n, 0);
  for (i64 j = n - 1; j >= 0; j--) {
    if (parent[j] == j) continue;
    if (parent[j] < 0 || parent[j] >= n) return -1;
    next[j] = head[parent[j]];
    head[parent[j]] = j;
  }
  i64 k = 0;
  for (i64 j = 0; j < n; j++) {
    if (parent[j] != j) continue;
    k = tdfs(j, k, head.data(), next.data(), post, stack.data());
  }
  return k == n ? 0 : -2;
}

// Column counts of the Cholesky factor (symbolic.py:74-131).
int chb_sym_counts(i64 n, const i64* cp, const i64* ri, const i64* parent, const i64* post, i64* colcount) {
  std::vector<i64> ancestor((size_t)n), maxfirst((size_t)n, -1), prevleaf((size_t)n, -1), first((size_t)n, -1);
  for (i64 i = 0; i < n; i++) ancestor[i] = i;
  for (i64 k = 0; k < n; k++) {
    i64 j = post[k];
    colcount[j] = (first[j] == -1) ? 1 : 0;
    while (j != -1 && first[j] == -1) {
      first[j] = k;
      // a root's parent is itself; the reference loop then sees first[j]
      // already set and stops, which the same test reproduces here
      j = parent[j];
    }
  }
  for (i64 k = 0; k < n; k++) {
    i64 j = post[k];
    if (parent[j] != j) colcount[parent[j]] -= 1;
    for (i64 p = cp[j]; p < cp[j + 1]; p++) {
      i64 i = ri[p];
      if (i <= j) continue;
      // __leaf(i, j, first, maxfirst, prevleaf, ancestor)  (symbolic.py:74-93)
      i64 q = -1;
      int jleaf = 0;
      if (!(i <= j || first[j] <= maxfirst[i])) {
        maxfirst[i] = first[j];
        i64 jprev = prevleaf[i];
        prevleaf[i] = j;
        jleaf = (jprev == -1) ? 1 : 2;
        if (jleaf == 1) {
          q = i;
        } else {
          q = jprev;
          while (q != ancestor[q]) q = ancestor[q];
          i64 s = jprev;
          while (s != q) {
            i64 sparent = ancestor[s];
            ancestor[s] = q;
            s = sparent;
          }
        }
      }
      if (jleaf >= 1) colcount[j] += 1;
      if (jleaf == 2) colcount[q] -= 1;
    }
    if (parent[j] != j) ancestor[j] = parent[j];
  }
  for (i64 j = 0; j < n; j++)
    if (parent[j] != j) colcount[parent[j]] += colcount[j];
  return 0;
}

// Fundamental supernodes and the supernodal elimination tree
// (pothen_sun + supernodes, symbolic.py:133-244).  Outputs: snode[n],
// snptr[N+1], snpar[N]; *nsn receives N.  snptr/snpar need room for n+1/n.
int chb_sym_supernodes(i64 n, const i64* par, const i64* post, const i64* colcount,
                       i64* snode, i64* snptr, i64* snpar, i64* nsn) {
  std::vector<i64> flag((size_t)n, -1), sp((size_t)n, -1);
  // children lists in the order the reference appends them (postorder)
  std::vector<i64> chhead((size_t)n, -1), chtail((size_t)n, -1), chnext((size_t)n, -1);
  for (i64 t = 0; t < n; t++) {
    i64 j = post[t];
    i64 pj = par[j];
    // ch[par[j]].append(j)
    if (chhead[pj] == -1) chhead[pj] = j; else chnext[chtail[pj]] = j;
    chtail[pj] = j;
    i64 mdeg = colcount[j] - 1;
    if (pj != j) {
      if (mdeg == colcount[pj] && flag[pj] == -1) {
        if (flag[j] < 0) {
          flag[pj] = j;
          flag[j] -= 1;
        } else {
          flag[pj] = flag[j];
          flag[flag[j]] -= 1;
        }
      }
    } else {
      if (flag[j] < 0) sp[j] = j;
      else sp[flag[j]] = flag[j];
    }
    i64 k = flag[j] < 0 ? j : flag[j];
    for (i64 i = chhead[j]; i != -1; i = chnext[i]) {
      i64 l = flag[i] < 0 ? i : flag[i];
      if (l != k) sp[l] = k;
    }
  }
  // renumber supernodes by representative vertex
  std::vector<i64> sn((size_t)n + 1, -1);
  i64 N = 0;
  for (i64 i = 0; i < n; i++)
    if (flag[i] < 0) sn[i] = N++;
  i64 m = 0;
  for (i64 i = 0; i < n; i++) {
    if (flag[i] < 0) {
      i64 v = sp[i];
      snpar[m++] = (v < 0) ? sn[n] : sn[v];
    }
  }
  // snode/snptr: vertices grouped by representative, increasing order
  std::vector<i64> cnt((size_t)n, 0);
  for (i64 i = 0; i < n; i++) cnt[flag[i] < 0 ? i : flag[i]] += 1;
  std::vector<i64> start((size_t)n, 0);
  snptr[0] = 0;
  i64 j = 0, acc = 0;
  for (i64 i = 0; i < n; i++) {
    if (cnt[i] > 0) {
      start[i] = acc;
      acc += cnt[i];
      snptr[j + 1] = acc;
      j++;
    }
  }
  if (j != N) return -1;
  std::vector<i64> fill((size_t)n, 0);
  for (i64 i = 0; i < n; i++) {
    i64 r = flag[i] < 0 ? i : flag[i];
    snode[start[r] + fill[r]++] = i;
  }
  *nsn = N;
  return 0;
}

// Supernodal amalgamation with the merge_size_fill rule (symbolic.py:246-326
// and :486-496).  In/out: colcount[n] (updated in place); snode[n] and
// snptr[N+1] in/out; snpar[N] in/out (renumbered); snpost[N] output.  *nsn
// in/out.  Merges supernode k into its parent when
//   fill = (|J_p| - (|J_k| - |N_k|)) * |N_k| <= tfill  or
//   (|N_k| <= tsize and |N_p| <= tsize).
// When `merge_fn` is non-null it replaces the rule above: it is called as
// merge_fn(|J_p|, |J_k|, |N_p|, |N_k|) and a non-zero return merges (this is
// how an arbitrary Python merge callable is honoured, symbolic.py:527-528).
int chb_sym_amalgamate(i64 n, i64* colcount, i64* snode, i64* snptr, i64* snpar, const i64* snpost_in,
                       i64* snpost_out, i64* nsn, i64 tsize, i64 tfill, chb_merge_fn merge_fn) {
  i64 N = *nsn;
  std::vector<std::vector<i64>> snlist((size_t)N);
  std::vector<char> alive((size_t)N, 1);
  for (i64 k = 0; k < N; k++) snlist[k].assign(snode + snptr[k], snode + snptr[k + 1]);
  // ch[snpar[j]].append(j) for j in snpost
  std::vector<std::vector<i64>> ch((size_t)N);
  for (i64 t = 0; t < N; t++) {
    i64 j = snpost_in[t];
    ch[snpar[j]].push_back(j);
  }
  std::vector<i64> spar(snpar, snpar + N);
  std::vector<i64> merged;
  for (i64 t = 0; t < N; t++) {
    i64 k = snpost_in[t];
    if (spar[k] == k) continue;
    i64 pk = spar[k];
    i64 colk = colcount[snlist[k][0]];
    i64 colp = colcount[snlist[pk][0]];
    i64 nk = (i64)snlist[k].size();
    i64 np = (i64)snlist[pk].size();
    bool doit;
    if (merge_fn) {
      doit = merge_fn(colp, colk, np, nk) != 0;
    } else {
      i64 fillv = (colp - (colk - nk)) * nk;
      doit = (fillv <= tfill) || (nk <= tsize && np <= tsize);
    }
    if (doit) {
      merged.clear();
      merged.reserve(snlist[k].size() + snlist[pk].size());
      std::merge(snlist[k].begin(), snlist[k].end(), snlist[pk].begin(), snlist[pk].end(),
                 std::back_inserter(merged));
      snlist[pk].swap(merged);
      snlist[k].clear();
      alive[k] = 0;
      colcount[snlist[pk][0]] = colp + nk;
      for (i64 c : ch[k]) spar[c] = pk;
      ch[pk].insert(ch[pk].end(), ch[k].begin(), ch[k].end());
      spar[k] = k;
    }
  }
  std::vector<i64> newid((size_t)N, -1);
  i64 M = 0;
  for (i64 k = 0; k < N; k++)
    if (alive[k]) newid[k] = M++;
  snptr[0] = 0;
  i64 i = 0;
  for (i64 k = 0; k < N; k++) {
    if (!alive[k]) continue;
    snptr[i + 1] = snptr[i] + (i64)snlist[k].size();
    std::copy(snlist[k].begin(), snlist[k].end(), snode + snptr[i]);
    i++;
  }
  i = 0;
  for (i64 k = 0; k < N; k++) {
    if (!alive[k]) continue;
    i64 v = newid[spar[k]];
    if (v < 0) return -1;
    snpar[i++] = v;
  }
  *nsn = M;
  return chb_sym_post_order(M, snpar, snpost_out);
}

// Filled pattern of the representative columns (symbolic.py:328-384).
// cp/ri: CCS of tril(Ap) of the permuted pattern.  colptr[N+1] output;
// rowidx output with capacity colptr[N] (query with rowidx == NULL first:
// then only colptr is written).
int chb_sym_embed(i64 n, const i64* cp, const i64* ri, const i64* colcount, const i64* snode, const i64* snptr,
                  const i64* snpar, const i64* snpost, i64 N, i64* colptr, i64* rowidx) {
  colptr[0] = 0;
  for (i64 k = 0; k < N; k++) colptr[k + 1] = colptr[k] + colcount[snode[snptr[k]]];
  if (!rowidx) return 0;
  for (i64 t = 0; t < colptr[N]; t++) rowidx[t] = -1;
  std::vector<i64> cnnz((size_t)N, 0), tmp;
  for (i64 k = 0; k < N; k++) {
    i64 p = snptr[k];
    i64 Nk = snptr[k + 1] - p;
    i64 c0 = snode[p];
    i64 nk = cp[c0 + 1] - cp[c0];
    if (nk > colptr[k + 1] - colptr[k]) return -1;
    for (i64 t = 0; t < nk; t++) rowidx[colptr[k] + t] = ri[cp[c0] + t];
    cnnz[k] = nk;
    for (i64 i = 1; i < Nk; i++) {
      i64 c = snode[p + i];
      i64 nc = cp[c + 1] - cp[c];
      cnnz[k] = lmerge(rowidx, ri, colptr[k], cp[c], cnnz[k], nc, tmp);
      if (cnnz[k] > colptr[k + 1] - colptr[k]) return -2;
    }
  }
  for (i64 t = 0; t < N; t++) {
    i64 k = snpost[t];
    i64 Nk = snptr[k + 1] - snptr[k];
    i64 pk = snpar[k];
    if (pk != k) {
      cnnz[pk] = lmerge(rowidx, rowidx, colptr[pk], colptr[k] + Nk, cnnz[pk], cnnz[k] - Nk, tmp);
      if (cnnz[pk] > colptr[pk + 1] - colptr[pk]) return -3;
    }
  }
  return 0;
}

// Relative indices of each supernode's separator within its parent's clique
// (symbolic.py:386-411).  relptr[N+1] output; relidx output with capacity
// colptr[N] (the reference allocates that much and returns the prefix of
// length relptr[N]).
int chb_sym_relative_idx(i64 N, const i64* colptr, const i64* rowidx, const i64* snptr, const i64* snpar,
                         i64* relptr, i64* relidx) {
  relptr[0] = 0;
  for (i64 k = 0; k < N; k++) {
    i64 p = snpar[k];
    relptr[k + 1] = relptr[k];
    i64 nk = snptr[k + 1] - snptr[k];
    relptr[k + 1] += colptr[k + 1] - colptr[k] - nk;
    // lfind(a, b): positions of the sorted entries of a within sorted b
    const i64* a = rowidx + colptr[k] + nk;
    i64 na = colptr[k + 1] - colptr[k] - nk;
    const i64* b = rowidx + colptr[p];
    i64 nb = colptr[p + 1] - colptr[p];
    i64 i = 0;
    for (i64 t = 0; t < na; t++) {
      while (i < nb && a[t] != b[i]) i++;
      if (i >= nb) return -1;
      relidx[relptr[k] + t] = i;
      i++;
    }
  }
  return 0;
}

}  // extern "C"
