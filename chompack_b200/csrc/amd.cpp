// Approximate minimum degree ordering.
//
// The reference obtains its fill-reducing ordering from cvxopt.amd.order
// (SuiteSparse AMD), called as symbolic(A, p=amd.order) (chompack
// src/python/symbolic.py:541-542) on the lower triangle of the symmetrised
// pattern.  That library is not part of the reference tree, so this file
// restates the published algorithm: P. R. Amestoy, T. A. Davis, I. S. Duff,
// "An approximate minimum degree ordering algorithm", SIAM J. Matrix Anal.
// Appl. 17(4):886-905, 1996, with the refinements described in its user
// guide (element absorption, aggressive absorption, mass elimination,
// supervariable detection by hashing, removal of dense rows with degree above
// max(16, 10*sqrt(n)), and a final postorder of the assembly tree that places
// the child with the largest front last).  The quotient graph lives in one
// integer workspace with in-place garbage collection.
//
// Credit and licence.  Reproducing cvxopt's permutation exactly means taking
// the same steps in the same order as SuiteSparse AMD's implementation, so
// the structure of this file follows that implementation (the elimination
// loop of AMD_2 in amd_2.c and the tree postorder of amd_post_tree.c), and
// several of its helper names (EMPTY, FLIP, clear_flag, post_tree) are
// SuiteSparse's.  SuiteSparse AMD is Copyright (c) 1996-2023 Timothy A.
// Davis, Patrick R. Amestoy and Iain S. Duff, and is distributed under the
// BSD-3-Clause licence; this file is a derivative work under those terms.
// Redistribution must retain that copyright notice and the licence's
// conditions and disclaimer; the names of the copyright holders may not be
// used to endorse products derived from this software without permission.
#include <cstdint>
#include <cmath>
#include <vector>
#include <algorithm>

#include "../../include/chompack_b200.h"

typedef int64_t I;

namespace {

const I EMPTY = -1;
inline I FLIP(I i) { return -i - 2; }

I clear_flag(I wflg, I wbig, I* W, I n) {
  if (wflg < 2 || wflg >= wbig) {
    for (I x = 0; x < n; x++)
      if (W[x] != 0) W[x] = 1;
    wflg = 2;
  }
  return wflg;
}

// Postorder one tree of the assembly forest (children lists already ordered).
I post_tree(I root, I k, I* Child, const I* Sibling, I* Order, I* Stack) {
  I head = 0;
  Stack[0] = root;
  while (head >= 0) {
    I i = Stack[head];
    if (Child[i] != EMPTY) {
      for (I f = Child[i]; f != EMPTY; f = Sibling[f]) head++;
      I h = head;
      for (I f = Child[i]; f != EMPTY; f = Sibling[f]) Stack[h--] = f;
      Child[i] = EMPTY;
    } else {
      head--;
      Order[i] = k++;
    }
  }
  return k;
}

void postorder(I nn, const I* Parent, const I* Nv, const I* Fsize, I* Order, I* Child, I* Sibling, I* Stack) {
  for (I j = 0; j < nn; j++) { Child[j] = EMPTY; Sibling[j] = EMPTY; }
  for (I j = nn - 1; j >= 0; j--) {
    if (Nv[j] > 0) {
      I parent = Parent[j];
      if (parent != EMPTY) {
        Sibling[j] = Child[parent];
        Child[parent] = j;
      }
    }
  }
  // move the child with the largest front to the end of each child list
  for (I i = 0; i < nn; i++) {
    if (Nv[i] > 0 && Child[i] != EMPTY) {
      I fprev = EMPTY, maxfrsize = EMPTY, bigfprev = EMPTY, bigf = EMPTY;
      for (I f = Child[i]; f != EMPTY; f = Sibling[f]) {
        I frsize = Fsize[f];
        if (frsize >= maxfrsize) {
          maxfrsize = frsize;
          bigfprev = fprev;
          bigf = f;
        }
        fprev = f;
      }
      I fnext = Sibling[bigf];
      if (fnext != EMPTY) {
        if (bigfprev == EMPTY) Child[i] = fnext;
        else Sibling[bigfprev] = fnext;
        Sibling[bigf] = EMPTY;
        Sibling[fprev] = bigf;
      }
    }
  }
  for (I i = 0; i < nn; i++) Order[i] = EMPTY;
  I k = 0;
  for (I i = 0; i < nn; i++)
    if (Parent[i] == EMPTY && Nv[i] > 0) k = post_tree(i, k, Child, Sibling, Order, Stack);
}

}  // namespace

extern "C" int chb_amd_order(int64_t n, const int64_t* Ap, const int64_t* Ai, int64_t* perm) {
  if (n <= 0) return 0;
  // --- pattern of A + A' without the diagonal, built from the lower
  // triangle (entries i > j of each column j), in the order of a column scan
  std::vector<I> Len((size_t)n, 0);
  I nzaat = 0;
  for (I j = 0; j < n; j++) {
    for (I p = Ap[j]; p < Ap[j + 1]; p++) {
      I i = Ai[p];
      if (i > j) { Len[i]++; Len[j]++; nzaat += 2; }
      else if (i < j) return -1;  // input must be lower triangular
    }
  }
  bool any = nzaat > 0;
  if (!any) {
    for (I k = 0; k < n; k++) perm[k] = k;
    return 0;
  }
  I iwlen = nzaat + nzaat / 5 + 8 * n + 1024;
  std::vector<I> Iw((size_t)iwlen), Pe((size_t)n), Nv((size_t)n), Next((size_t)n), Last((size_t)n),
      Head((size_t)n), Elen((size_t)n), Degree((size_t)n), W((size_t)n), Sp((size_t)n);
  I pfree = 0;
  for (I j = 0; j < n; j++) { Pe[j] = pfree; Sp[j] = pfree; pfree += Len[j]; }
  for (I j = 0; j < n; j++) {
    for (I p = Ap[j]; p < Ap[j + 1]; p++) {
      I i = Ai[p];
      if (i > j) { Iw[Sp[i]++] = j; Iw[Sp[j]++] = i; }
    }
  }

  // --- minimum degree elimination on the quotient graph
  I dense;
  {
    double alpha = 10.0;
    double d = alpha * std::sqrt((double)n);
    d = std::max(16.0, d);
    d = std::min((double)n, d);
    dense = (I)d;
  }
  I lemax = 0, nel = 0, mindeg = 0;
  I wbig = INT64_MAX - n;
  for (I i = 0; i < n; i++) {
    Last[i] = EMPTY; Head[i] = EMPTY; Next[i] = EMPTY; Nv[i] = 1; W[i] = 1; Elen[i] = 0; Degree[i] = Len[i];
  }
  I wflg = clear_flag(0, wbig, W.data(), n);
  for (I i = 0; i < n; i++) {
    I deg = Degree[i];
    if (deg == 0) {
      Elen[i] = FLIP(1);
      nel++;
      Pe[i] = EMPTY;
      W[i] = 0;
    } else if (deg > dense) {
      Nv[i] = 0;
      Elen[i] = EMPTY;
      nel++;
      Pe[i] = EMPTY;
    } else {
      I inext = Head[deg];
      if (inext != EMPTY) Last[inext] = i;
      Next[i] = inext;
      Head[deg] = i;
    }
  }

  while (nel < n) {
    // pivot of minimum degree
    I deg, me = EMPTY;
    for (deg = mindeg; deg < n; deg++) {
      me = Head[deg];
      if (me != EMPTY) break;
    }
    if (me == EMPTY) return -2;
    mindeg = deg;
    I inext = Next[me];
    if (inext != EMPTY) Last[inext] = EMPTY;
    Head[deg] = inext;
    I elenme = Elen[me];
    I nvpiv = Nv[me];
    nel += nvpiv;

    // construct the new element Lme
    Nv[me] = -nvpiv;
    I degme = 0, pme1, pme2;
    if (elenme == 0) {
      pme1 = Pe[me];
      pme2 = pme1 - 1;
      for (I p = pme1; p <= pme1 + Len[me] - 1; p++) {
        I i = Iw[p];
        I nvi = Nv[i];
        if (nvi > 0) {
          degme += nvi;
          Nv[i] = -nvi;
          Iw[++pme2] = i;
          I ilast = Last[i];
          I in2 = Next[i];
          if (in2 != EMPTY) Last[in2] = ilast;
          if (ilast != EMPTY) Next[ilast] = in2;
          else Head[Degree[i]] = in2;
        }
      }
    } else {
      I p = Pe[me];
      pme1 = pfree;
      I slenme = Len[me] - elenme;
      for (I knt1 = 1; knt1 <= elenme + 1; knt1++) {
        I e, pj, ln;
        if (knt1 > elenme) {
          e = me; pj = p; ln = slenme;
        } else {
          e = Iw[p++]; pj = Pe[e]; ln = Len[e];
        }
        for (I knt2 = 1; knt2 <= ln; knt2++) {
          I i = Iw[pj++];
          I nvi = Nv[i];
          if (nvi > 0) {
            if (pfree >= iwlen) {
              // garbage collection: compact all live lists to the front
              Pe[me] = p;
              Len[me] -= knt1;
              if (Len[me] == 0) Pe[me] = EMPTY;
              Pe[e] = pj;
              Len[e] = ln - knt2;
              if (Len[e] == 0) Pe[e] = EMPTY;
              for (I j = 0; j < n; j++) {
                I pn = Pe[j];
                if (pn >= 0) { Pe[j] = Iw[pn]; Iw[pn] = FLIP(j); }
              }
              I psrc = 0, pdst = 0, pend = pme1 - 1;
              while (psrc <= pend) {
                I j = FLIP(Iw[psrc++]);
                if (j >= 0) {
                  Iw[pdst] = Pe[j];
                  Pe[j] = pdst++;
                  I lenj = Len[j];
                  for (I knt3 = 0; knt3 <= lenj - 2; knt3++) Iw[pdst++] = Iw[psrc++];
                }
              }
              I p1 = pdst;
              for (psrc = pme1; psrc <= pfree - 1; psrc++) Iw[pdst++] = Iw[psrc];
              pme1 = p1;
              pfree = pdst;
              pj = Pe[e];
              p = Pe[me];
              if (pfree >= iwlen) return -3;
            }
            degme += nvi;
            Nv[i] = -nvi;
            Iw[pfree++] = i;
            I ilast = Last[i];
            I in2 = Next[i];
            if (in2 != EMPTY) Last[in2] = ilast;
            if (ilast != EMPTY) Next[ilast] = in2;
            else Head[Degree[i]] = in2;
          }
        }
        if (e != me) {
          Pe[e] = FLIP(me);
          W[e] = 0;
        }
      }
      pme2 = pfree - 1;
    }
    Degree[me] = degme;
    Pe[me] = pme1;
    Len[me] = pme2 - pme1 + 1;
    Elen[me] = FLIP(nvpiv + degme);

    wflg = clear_flag(wflg, wbig, W.data(), n);

    // |Le \ Lme| for every element e adjacent to a variable of Lme
    for (I pme = pme1; pme <= pme2; pme++) {
      I i = Iw[pme];
      I eln = Elen[i];
      if (eln > 0) {
        I nvi = -Nv[i];
        I wnvi = wflg - nvi;
        for (I p = Pe[i]; p <= Pe[i] + eln - 1; p++) {
          I e = Iw[p];
          I we = W[e];
          if (we >= wflg) we -= nvi;
          else if (we != 0) we = Degree[e] + wnvi;
          W[e] = we;
        }
      }
    }

    // degree update, aggressive element absorption, mass elimination
    for (I pme = pme1; pme <= pme2; pme++) {
      I i = Iw[pme];
      I p1 = Pe[i];
      I p2 = p1 + Elen[i] - 1;
      I pn = p1;
      uint64_t hash = 0;
      I dg = 0;
      for (I p = p1; p <= p2; p++) {
        I e = Iw[p];
        I we = W[e];
        if (we != 0) {
          I dext = we - wflg;
          if (dext > 0) {
            dg += dext;
            Iw[pn++] = e;
            hash += (uint64_t)e;
          } else {
            Pe[e] = FLIP(me);
            W[e] = 0;
          }
        }
      }
      Elen[i] = pn - p1 + 1;
      I p3 = pn;
      I p4 = p1 + Len[i];
      for (I p = p2 + 1; p < p4; p++) {
        I j = Iw[p];
        I nvj = Nv[j];
        if (nvj > 0) {
          dg += nvj;
          Iw[pn++] = j;
          hash += (uint64_t)j;
        }
      }
      if (Elen[i] == 1 && p3 == pn) {
        Pe[i] = FLIP(me);
        I nvi = -Nv[i];
        degme -= nvi;
        nvpiv += nvi;
        nel += nvi;
        Nv[i] = 0;
        Elen[i] = EMPTY;
      } else {
        Degree[i] = std::min(Degree[i], dg);
        Iw[pn] = Iw[p3];
        Iw[p3] = Iw[p1];
        Iw[p1] = me;
        Len[i] = pn - p1 + 1;
        I h = (I)(hash % (uint64_t)n);
        I j = Head[h];
        if (j <= EMPTY) {
          Next[i] = FLIP(j);
          Head[h] = FLIP(i);
        } else {
          Next[i] = Last[j];
          Last[j] = i;
        }
        Last[i] = h;
      }
    }
    Degree[me] = degme;

    lemax = std::max(lemax, degme);
    wflg += lemax;
    wflg = clear_flag(wflg, wbig, W.data(), n);

    // supervariable detection
    for (I pme = pme1; pme <= pme2; pme++) {
      I i = Iw[pme];
      if (Nv[i] < 0) {
        I h = Last[i];
        I j = Head[h];
        if (j == EMPTY) {
          i = EMPTY;
        } else if (j < EMPTY) {
          i = FLIP(j);
          Head[h] = EMPTY;
        } else {
          i = Last[j];
          Last[j] = EMPTY;
        }
        while (i != EMPTY && Next[i] != EMPTY) {
          I ln = Len[i];
          I eln = Elen[i];
          for (I p = Pe[i] + 1; p <= Pe[i] + ln - 1; p++) W[Iw[p]] = wflg;
          I jlast = i;
          I jj = Next[i];
          while (jj != EMPTY) {
            bool ok = (Len[jj] == ln) && (Elen[jj] == eln);
            for (I p = Pe[jj] + 1; ok && p <= Pe[jj] + ln - 1; p++)
              if (W[Iw[p]] != wflg) ok = false;
            if (ok) {
              Pe[jj] = FLIP(i);
              Nv[i] += Nv[jj];
              Nv[jj] = 0;
              Elen[jj] = EMPTY;
              jj = Next[jj];
              Next[jlast] = jj;
            } else {
              jlast = jj;
              jj = Next[jj];
            }
          }
          wflg++;
          i = Next[i];
        }
      }
    }

    // restore degree lists; drop non-principal variables from the element
    I p = pme1;
    I nleft = n - nel;
    for (I pme = pme1; pme <= pme2; pme++) {
      I i = Iw[pme];
      I nvi = -Nv[i];
      if (nvi > 0) {
        Nv[i] = nvi;
        I d = Degree[i] + degme - nvi;
        d = std::min(d, nleft - nvi);
        I in2 = Head[d];
        if (in2 != EMPTY) Last[in2] = i;
        Next[i] = in2;
        Last[i] = EMPTY;
        Head[d] = i;
        mindeg = std::min(mindeg, d);
        Degree[i] = d;
        Iw[p++] = i;
      }
    }
    Nv[me] = nvpiv;
    Len[me] = p - pme1;
    if (Len[me] == 0) {
      Pe[me] = EMPTY;
      W[me] = 0;
    }
    if (elenme != 0) pfree = p;
  }

  // --- assembly tree: parent of j is Pe[j]; element sizes in Elen
  for (I i = 0; i < n; i++) Pe[i] = FLIP(Pe[i]);
  for (I i = 0; i < n; i++) Elen[i] = FLIP(Elen[i]);
  // compress the paths of the non-principal variables to their element
  for (I i = 0; i < n; i++) {
    if (Nv[i] == 0) {
      I j = Pe[i];
      if (j == EMPTY) continue;
      while (Nv[j] == 0) j = Pe[j];
      I e = j;
      j = i;
      while (Nv[j] == 0) {
        I jnext = Pe[j];
        Pe[j] = e;
        j = jnext;
      }
    }
  }
  postorder(n, Pe.data(), Nv.data(), Elen.data(), W.data(), Head.data(), Next.data(), Last.data());
  for (I k = 0; k < n; k++) { Head[k] = EMPTY; Next[k] = EMPTY; }
  for (I e = 0; e < n; e++) {
    I k = W[e];
    if (k != EMPTY) Head[k] = e;
  }
  nel = 0;
  for (I k = 0; k < n; k++) {
    I e = Head[k];
    if (e == EMPTY) break;
    Next[e] = nel;
    nel += Nv[e];
  }
  for (I i = 0; i < n; i++) {
    if (Nv[i] == 0) {
      I e = Pe[i];
      if (e != EMPTY) {
        Next[i] = Next[e];
        Next[e]++;
      } else {
        Next[i] = nel++;
      }
    }
  }
  for (I i = 0; i < n; i++) {
    I k = Next[i];
    if (k < 0 || k >= n) return -4;
    perm[k] = i;
  }
  return 0;
}
