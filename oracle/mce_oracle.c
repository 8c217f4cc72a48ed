/*
 * mce_oracle.c - CPU oracle for maximal-clique counting.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load this library, and only as
 * the checker or as the timed CPU baseline; the product path (libmce.so)
 * never links or calls it.
 *
 * It restates, in plain C, the algorithm of yen-hsiang-chang/mce-gpu for the
 * hot path (reference paths are relative to that project's root):
 *
 *   oracle_peel    - synchronous k-core peeling with the reference's round
 *                    numbering (include/kcore.cuh:233-316, kernels :21-143)
 *   oracle_orient  - orientation + stable split of every row into
 *                    [earlier | later] neighbours
 *                    (include/main_support.cuh:6-84, src/main.cu:102-146)
 *   oracle_mce     - per-root Bron-Kerbosch with Tomita pivoting over the
 *                    bitmap of the root's later neighbours, the L1 + IP
 *                    scheme (mce/mce_kernel_nowl.cuh:9-109 with the helpers
 *                    of mce/mce_utils.cuh cited inline)
 *
 * and adds two independent checkers that share no code with the above:
 *
 *   oracle_brute   - enumerates every clique of a graph with <= 64 vertices
 *   oracle_tomita  - textbook whole-graph Tomita-Tanaka-Takahashi search
 *
 * Counting convention (mce/mce_kernel_wl.cuh:70-79, mce/mce_utils.cuh:507-524):
 * maximal cliques with at least 2 vertices; isolated vertices never count.
 */
#include <alloca.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_OK 0
#define ORACLE_EINVAL (-1)
#define ORACLE_ENOMEM (-2)
#define ORACLE_ELIMIT (-6)

/* ------------------------------------------------------------------------ */
/* Degeneracy order.                                                        */
/*                                                                          */
/* Follows SingleGPU_Kcore::findKcoreIncremental_async                      */
/* (include/kcore.cuh:233-316): levels k = 0, 1, 2, ...; at each level the  */
/* vertices whose remaining degree equals k form round 0 (filter_window +   */
/* filter_with_random_append, :21-48, :179-197); removing a round's         */
/* vertices lowers their neighbours' degrees and every neighbour whose      */
/* degree falls to k joins the next round (process_degree /                 */
/* kernel_partition_level_next, :80-95, :107-143).  Rounds are numbered     */
/* consecutively over all levels (`priority++`, :297); a vertex's priority  */
/* is its round number (:130, :284); the final round, which empties the     */
/* graph, is never processed (`if (0 == todo) break;`, :276) so its         */
/* vertices keep the initial value numEdges (:258).  The degeneracy is the  */
/* last level (printed as k - 1, :313-315).                                 */
/* ------------------------------------------------------------------------ */
int oracle_peel(int64_t n, const int32_t *row_ptr, const int32_t *col, uint32_t *prio,
                int32_t *core, int32_t *degeneracy) {
  if (n < 0 || (n > 0 && (!row_ptr || !prio))) return ORACLE_EINVAL;
  const int64_t m = n ? row_ptr[n] : 0;
  int32_t *deg = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t *cr = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t *rem = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t *cur = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t *nxt = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
  if (!deg || !cr || !rem || !cur || !nxt) {
    free(deg); free(cr); free(rem); free(cur); free(nxt);
    return ORACLE_ENOMEM;
  }
  int64_t nrem = n;
  for (int64_t v = 0; v < n; ++v) {
    deg[v] = row_ptr[v + 1] - row_ptr[v];
    prio[v] = (uint32_t)m;
    cr[v] = -1;
    rem[v] = (int32_t)v;
  }
  int64_t todo = n;
  int32_t level = 0;
  uint32_t priority = 0;
  int32_t last_level = -1;
  while (todo > 0) {
    /* round 0 of this level: remaining vertices of degree == level, in id order */
    int64_t ncur = 0, keep = 0;
    for (int64_t i = 0; i < nrem; ++i) {
      const int32_t v = rem[i];
      if (cr[v] >= 0) continue;
      if (deg[v] == level) {
        cur[ncur++] = v;
        cr[v] = level;
      } else {
        rem[keep++] = v;
      }
    }
    nrem = keep;
    while (ncur > 0) {
      last_level = level;
      todo -= ncur;
      if (todo == 0) break;
      int64_t nn = 0;
      for (int64_t i = 0; i < ncur; ++i) prio[cur[i]] = priority;
      for (int64_t i = 0; i < ncur; ++i) {
        const int32_t v = cur[i];
        for (int64_t j = row_ptr[v]; j < row_ptr[v + 1]; ++j) {
          const int32_t u = col[j];
          if (cr[u] >= 0) continue; /* in this round, already queued, or removed */
          if (--deg[u] == level) {
            cr[u] = level;
            nxt[nn++] = u;
          }
        }
      }
      int32_t *t = cur;
      cur = nxt;
      nxt = t;
      ncur = nn;
      ++priority;
    }
    ++level;
  }
  if (core)
    for (int64_t v = 0; v < n; ++v) core[v] = cr[v];
  if (degeneracy) *degeneracy = last_level < 0 ? 0 : last_level;
  free(deg); free(cr); free(rem); free(cur); free(nxt);
  return ORACLE_OK;
}

/* ------------------------------------------------------------------------ */
/* Orientation.  keep(src -> dst) = prio[src] == prio[dst] ? src < dst      */
/*                                : prio[src] < prio[dst]                   */
/* (include/main_support.cuh:14): dst is later than src.  Each row becomes  */
/* [earlier | later], both parts in the original (sorted) order, and        */
/* split[v] is where the later part starts (split_data, :31-84).            */
/* ------------------------------------------------------------------------ */
int oracle_orient(int64_t n, const int32_t *row_ptr, const int32_t *col, const uint32_t *prio,
                  int32_t *split, int32_t *col_out) {
  if (n < 0 || (n > 0 && (!row_ptr || !prio || !split || !col_out))) return ORACLE_EINVAL;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < n; ++v) {
    int64_t e = row_ptr[v];
    for (int64_t j = row_ptr[v]; j < row_ptr[v + 1]; ++j) {
      const int32_t u = col[j];
      const int later = prio[v] == prio[u] ? (v < u) : (prio[v] < prio[u]);
      if (!later) col_out[e++] = u;
    }
    split[v] = (int32_t)e;
    for (int64_t j = row_ptr[v]; j < row_ptr[v + 1]; ++j) {
      const int32_t u = col[j];
      const int later = prio[v] == prio[u] ? (v < u) : (prio[v] < prio[u]);
      if (later) col_out[e++] = u;
    }
  }
  return ORACLE_OK;
}

/* ------------------------------------------------------------------------ */
/* Per-root search (L1 + IP).                                               */
/* ------------------------------------------------------------------------ */
static int bsearch_i32(const int32_t *a, int64_t lo, int64_t hi, int32_t key) {
  /* graph::binary_search (mce/mce_utils.cuh:63-88) */
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (a[mid] == key) return 1;
    if (a[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return 0;
}

static inline int popc64(uint64_t x) { return __builtin_popcountll(x); }

typedef struct {
  int64_t maxd, maxu, W;
  uint64_t *enc;   /* maxd x W     : adjacency rows inside P(root)        */
  uint64_t *pl;    /* (maxd+2) x W : branch set of each level              */
  uint64_t *cl;    /* (maxd+2) x W : candidate set P of each level         */
  uint64_t *xl;    /* (maxd+2) x W : in-subgraph X of each level           */
  int64_t *ptr;    /* (maxd+2)     : next bit to branch on at each level   */
  int32_t *cnode;  /* (maxd+2)     : vertex chosen at each level           */
  int32_t *xx;     /* maxu         : earlier neighbours of the root (Xx)   */
  int32_t *xaux;   /* maxu                                                  */
  int64_t *xsz;    /* (maxd+3)     : |Xx| at each level                    */
  uint64_t *xo;    /* (maxd+2) x W : L2 outside rows of the root's later nbrs */
} bk_ws;

static void ws_free(bk_ws *w) {
  free(w->enc); free(w->pl); free(w->cl); free(w->xl); free(w->ptr);
  free(w->cnode); free(w->xx); free(w->xaux); free(w->xsz); free(w->xo);
}

static int ws_alloc(bk_ws *w, int64_t maxd, int64_t maxu) {
  memset(w, 0, sizeof(*w));
  w->maxd = maxd;
  w->maxu = maxu;
  w->W = (maxd + 63) / 64;
  if (w->W == 0) w->W = 1;
  const size_t L = (size_t)(maxd + 3);
  w->enc = (uint64_t *)calloc((size_t)(maxd ? maxd : 1) * w->W, 8);
  w->pl = (uint64_t *)calloc(L * w->W, 8);
  w->cl = (uint64_t *)calloc(L * w->W, 8);
  w->xl = (uint64_t *)calloc(L * w->W, 8);
  w->ptr = (int64_t *)calloc(L, 8);
  w->cnode = (int32_t *)calloc(L, 4);
  w->xx = (int32_t *)calloc((size_t)(maxu ? maxu : 1), 4);
  w->xaux = (int32_t *)calloc((size_t)(maxu ? maxu : 1), 4);
  w->xsz = (int64_t *)calloc(L + 1, 8);
  w->xo = (uint64_t *)calloc(L * w->W, 8);
  if (!w->enc || !w->pl || !w->cl || !w->xl || !w->ptr || !w->cnode || !w->xx || !w->xaux ||
      !w->xsz || !w->xo) {
    ws_free(w);
    return ORACLE_ENOMEM;
  }
  return ORACLE_OK;
}

/* The walk below level 0 of one search tree (L1: the root's; L2: a unit's),
   the reference's state machine of mce/mce_kernel_nowl.cuh:9-109 over the
   bitmaps of the workspace.  Level 0 (pl, cl, xl, ptr, xx/xsz, and for L2
   the outside rows xo) is set up by the caller.  base = the clique's size
   before level 0's branch (1: the root; 2: root and L2 edge). */
static void bk_walk(bk_ws *w, int64_t d, int64_t W, uint64_t W32, const int32_t *row_ptr,
                    const int32_t *split, const int32_t *cs, int64_t sb, int64_t ub, int l2,
                    int64_t base, uint64_t *hist, int hist_len, uint64_t *cnt, uint64_t *nodes,
                    uint64_t *ops) {
  uint64_t *enc = w->enc, *pl = w->pl, *cl = w->cl, *xl = w->xl, *xo = w->xo;
  uint64_t *tcl = (uint64_t *)alloca(sizeof(uint64_t) * (size_t)W);
  uint64_t *txl = (uint64_t *)alloca(sizeof(uint64_t) * (size_t)W);
  uint64_t *txo = (uint64_t *)alloca(sizeof(uint64_t) * (size_t)W);
  int64_t l = 0; /* level index (the reference's l - 2) */
  while (l >= 0) {
    /* get_next_candidate (mce/mce_utils.cuh:526-563): next set bit of the
       level's branch set at or after ptr[l]; none left -> backtrack. */
    int64_t v = -1;
    for (int64_t b = w->ptr[l]; b < d;) {
      const uint64_t word = pl[l * W + b / 64] & (~0ull << (b % 64));
      if (word) {
        v = (b / 64) * 64 + __builtin_ctzll(word);
        break;
      }
      b = (b / 64 + 1) * 64;
    }
    if (v < 0 || v >= d) {
      --l;
      continue;
    }
    ++*nodes;
    w->ptr[l] = v + 1; /* clean_level_L1_IP (:786-805) */
    const int32_t cn = cs[sb + v];
    /* Xx_compaction_for_IP (mce/mce_utils.cuh:265-292): the root's earlier
       neighbours adjacent to the chosen vertex (binary search in its
       earlier list) move to the front; their count is the next level's |Xx|. */
    {
      const int64_t lim = w->xsz[l];
      int64_t f = 0, b2 = lim;
      const int64_t cb = row_ptr[cn], ce = split[cn];
      for (int64_t k = 0; k < lim; ++k) {
        const int32_t cur = w->xx[k];
        if (bsearch_i32(cs, cb, ce, cs[ub + cur]))
          w->xaux[f++] = cur;
        else
          w->xaux[--b2] = cur;
      }
      memcpy(w->xx, w->xaux, sizeof(int32_t) * (size_t)lim);
      w->xsz[l + 1] = f;
    }
    /* populate_xl_and_cl (mce/mce_utils.cuh:321-336): branch bits before v
       move from P to X; child P' = P & N(v), X' = X & N(v); L2's outside
       rows of the root's later neighbours keep those adjacent to v. */
    int64_t curSZ = 0;
    int xo_any = 0;
    for (int64_t k = 0; k < W; ++k) {
      uint64_t before;
      if (k < v / 64)
        before = ~0ull;
      else if (k > v / 64)
        before = 0;
      else
        before = (1ull << (v % 64)) - 1;
      const uint64_t done = pl[l * W + k] & before;
      txl[k] = (xl[l * W + k] | done) & enc[v * W + k];
      tcl[k] = (cl[l * W + k] & ~done) & enc[v * W + k];
      txo[k] = l2 ? (xo[l * W + k] & enc[v * W + k]) : 0;
      xo_any |= txo[k] != 0;
      curSZ += popc64(tcl[k]);
    }
    /* select_pivot_from_P_and_Xp (mce/mce_utils.cuh:366-402): pivot over
       P' u X'; an X' vertex adjacent to all of P' eliminates the path. */
    int more = 0, elim = 0;
    int64_t pv = -1, pbest = -1, cand = 0;
    for (int64_t j = 0; j < d; ++j) {
      const uint64_t bit = 1ull << (j % 64);
      const int inP = (tcl[j / 64] & bit) != 0, inX = (txl[j / 64] & bit) != 0;
      if (!inP && !inX) continue;
      ++cand;
      int64_t c = 0;
      for (int64_t k = 0; k < W; ++k) c += popc64(tcl[k] & enc[j * W + k]);
      if (c == curSZ) elim = 1; /* only possible for j in X' */
      more = 1;
      if (c > pbest) {
        pbest = c;
        pv = j;
      }
    }
    *ops += 2 * W32 * (uint64_t)cand + 4 * W32;
    if (!more || elim) {
      /* test_maximality (mce/mce_utils.cuh:507-524) */
      if (w->xsz[l + 1] == 0 && !xo_any) {
        int xe = 1;
        for (int64_t k = 0; k < W; ++k) xe &= (txl[k] == 0);
        if (xe && curSZ == 0) {
          ++*cnt;
          const int64_t size = base + l + 1; /* one vertex per level */
          if (hist && size < hist_len) hist[size]++;
        }
      }
      continue;
    }
    /* apply_pivot_to_next_level (mce/mce_utils.cuh:218-239) + go_to_next_level */
    for (int64_t k = 0; k < W; ++k) {
      pl[(l + 1) * W + k] = ~enc[pv * W + k] & tcl[k];
      cl[(l + 1) * W + k] = tcl[k];
      xl[(l + 1) * W + k] = txl[k];
      if (l2) xo[(l + 1) * W + k] = txo[k];
    }
    w->ptr[l + 1] = 0;
    ++l;
  }
}

/* Count the maximal cliques whose first vertex in the order is r.
   *ops_out: the walk's algorithmic 32-bit word operations, W32 =
   ceil(d / 32) words per row: 2 W32 per row scored by a pivot selection
   (AND + POPC; the root's over all d rows, select_pivot_from_P,
   mce/mce_utils.cuh:338-364, a node's over P' | X',
   select_pivot_from_P_and_Xp, :366-402) and 4 W32 per node for the child
   sets (populate_xl_and_cl, :321-336).

   l2prio != NULL: the L2 scheme (mce/mce_kernel_wl.cuh:307-485 with
   setup_stack_original_L2_IP, mce/mce_utils.cuh:664-712): every oriented
   edge (r, v), v a later neighbour, is a unit whose candidates are the
   triangle list P = N+(r) & N+(v) (block_count_and_set_tri, :151-171) and
   whose outside list holds the neighbours of r earlier than v and adjacent
   to it (the reference's Xx over r's whole row); an empty P counts the edge
   when that list is empty; otherwise the unit's pivot is taken from P alone
   and the walk below is the L1 one.  Units are not tree nodes (the
   reference's traversed_nodes counts branches inside a unit,
   mce/mce_kernel_wl_lb.cuh:445). */
static void root_search(bk_ws *w, int32_t r, const int32_t *row_ptr, const int32_t *split,
                        const int32_t *cs, uint64_t *hist, int hist_len, uint64_t *cnt_out,
                        uint64_t *nodes_out, uint64_t *ops_out, const uint32_t *l2prio) {
  const int64_t sb = split[r], d = row_ptr[r + 1] - sb; /* later neighbours: P */
  const int64_t ub = row_ptr[r], u = sb - ub;          /* earlier neighbours: Xx */
  uint64_t cnt = 0, nodes = 0, ops = 0;
  *cnt_out = 0;
  *nodes_out = 0;
  *ops_out = 0;
  if (d == 0) return; /* a root without later neighbours yields nothing */
  const int64_t W = (d + 63) / 64;
  const uint64_t W32 = (uint64_t)((d + 31) / 32);
  uint64_t *enc = w->enc;
  memset(enc, 0, sizeof(uint64_t) * (size_t)(d * W));
  /* warp_sorted_count_and_encode_full (mce/mce_utils.cuh:90-117): for every
     j, search each P[i] in N+(P[j]); a hit sets bits (j, i) and (i, j). */
  for (int64_t j = 0; j < d; ++j) {
    const int32_t v = cs[sb + j];
    const int64_t vb = split[v], ve = row_ptr[v + 1];
    for (int64_t i = 0; i < d; ++i)
      if (bsearch_i32(cs, vb, ve, cs[sb + i])) {
        enc[j * W + i / 64] |= 1ull << (i % 64);
        enc[i * W + j / 64] |= 1ull << (j % 64);
      }
  }
  uint64_t *pl = w->pl, *cl = w->cl, *xl = w->xl, *xo = w->xo;
  const uint64_t lastmask = (d % 64) ? ((1ull << (d % 64)) - 1) : ~0ull;
  if (!l2prio) {
    /* setup_stack_original_L1_IP (mce/mce_utils.cuh:565-611): Xx = all
       earlier neighbours, level 0 holds P = all of N+(r), X = 0;
       select_pivot_from_P (:338-364): the row with the most bits,
       finalize_pivot (:191-202), ties: the first row;
       apply_pivot_to_first_level (:204-216). */
    for (int64_t k = 0; k < u; ++k) w->xx[k] = (int32_t)k;
    w->xsz[0] = u;
    int64_t piv = 0, best = -1;
    ops += 2 * W32 * (uint64_t)d;
    for (int64_t j = 0; j < d; ++j) {
      int64_t c = 0;
      for (int64_t k = 0; k < W; ++k) c += popc64(enc[j * W + k]);
      if (c > best) {
        best = c;
        piv = j;
      }
    }
    for (int64_t k = 0; k < W; ++k) {
      const uint64_t m = (k == W - 1) ? lastmask : ~0ull;
      pl[k] = ~enc[piv * W + k] & m;
      cl[k] = m;
      xl[k] = 0;
    }
    w->ptr[0] = 0;
    bk_walk(w, d, W, W32, row_ptr, split, cs, sb, ub, 0, 1, hist, hist_len, &cnt, &nodes, &ops);
  } else {
    for (int64_t vj = 0; vj < d; ++vj) { /* unit (r, v) */
      const int32_t v = cs[sb + vj];
      const uint32_t pv = l2prio[v];
      /* the triangle list (later than v) and r's later neighbours earlier
         than v and adjacent to it (outside rows) */
      int tri_any = 0, xo_any = 0;
      for (int64_t k = 0; k < W; ++k) pl[k] = cl[k] = xl[k] = xo[k] = 0;
      for (int64_t j = 0; j < d; ++j) {
        if (!(enc[vj * W + j / 64] >> (j % 64) & 1ull)) continue;
        const int32_t x = cs[sb + j];
        const uint32_t px = l2prio[x];
        const int later = px == pv ? v < x : pv < px; /* include/main_support.cuh:14 */
        if (later) {
          cl[j / 64] |= 1ull << (j % 64);
          tri_any = 1;
        } else {
          xo[j / 64] |= 1ull << (j % 64);
          xo_any = 1;
        }
      }
      /* the root's earlier neighbours adjacent to v (earlier than v too) */
      int64_t f = 0;
      const int64_t cb = row_ptr[v], ce = split[v];
      for (int64_t k = 0; k < u; ++k)
        if (bsearch_i32(cs, cb, ce, cs[ub + k])) w->xx[f++] = (int32_t)k;
      w->xsz[0] = f;
      if (!tri_any) { /* the edge alone: maximal unless its outside list is not empty */
        if (f == 0 && !xo_any) {
          ++cnt;
          if (hist && 2 < hist_len) hist[2]++;
        }
        continue;
      }
      /* select_pivot_from_P over the triangle list alone */
      int64_t piv = -1, best = -1;
      for (int64_t j = 0; j < d; ++j) {
        if (!(cl[j / 64] >> (j % 64) & 1ull)) continue;
        int64_t c = 0;
        for (int64_t k = 0; k < W; ++k) c += popc64(cl[k] & enc[j * W + k]);
        if (c > best) {
          best = c;
          piv = j;
        }
      }
      for (int64_t k = 0; k < W; ++k) pl[k] = cl[k] & ~enc[piv * W + k];
      w->ptr[0] = 0;
      bk_walk(w, d, W, W32, row_ptr, split, cs, sb, ub, 1, 2, hist, hist_len, &cnt, &nodes, &ops);
    }
  }
  *cnt_out = cnt;
  *nodes_out = nodes;
  *ops_out = ops;
}

/*
 * Search the roots begin, begin + stride, ... < end (all roots: 0, n, 1).
 * total: maximal cliques found; hist (nullable, hist_len entries) by size;
 * root_count / root_nodes / root_ops (nullable, n entries) per root.
 */
static int mce_roots(int64_t n, const int32_t *row_ptr, const int32_t *split, const int32_t *cs,
                     int64_t begin, int64_t end, int64_t stride, int nthreads, uint64_t *total,
                     uint64_t *hist, int hist_len, uint64_t *root_count, uint64_t *root_nodes,
                     uint64_t *root_ops, const uint32_t *l2prio) {
  if (n < 0 || stride < 1 || !total || (n > 0 && (!row_ptr || !split || !cs)))
    return ORACLE_EINVAL;
  if (end > n) end = n;
  if (begin < 0) begin = 0;
  int64_t maxd = 0, maxu = 0;
  for (int64_t v = 0; v < n; ++v) {
    const int64_t d = row_ptr[v + 1] - split[v], u = split[v] - row_ptr[v];
    if (d > maxd) maxd = d;
    if (u > maxu) maxu = u;
  }
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  uint64_t tot = 0;
  int err = 0;
  if (hist)
    for (int i = 0; i < hist_len; ++i) hist[i] = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : tot)
  {
    bk_ws w;
    uint64_t *lh = hist ? (uint64_t *)calloc((size_t)hist_len, 8) : NULL;
    const int ok = ws_alloc(&w, maxd, maxu) == ORACLE_OK && (!hist || lh);
    if (!ok) {
#pragma omp atomic write
      err = 1;
    }
#pragma omp for schedule(dynamic, 64)
    for (int64_t r = begin; r < end; r += stride) {
      if (!ok) continue;
      uint64_t c, nd, op;
      root_search(&w, (int32_t)r, row_ptr, split, cs, lh, hist_len, &c, &nd, &op, l2prio);
      tot += c;
      if (root_count) root_count[r] = c;
      if (root_nodes) root_nodes[r] = nd;
      if (root_ops) root_ops[r] = op;
    }
    if (ok) {
      if (hist) {
#pragma omp critical
        for (int i = 0; i < hist_len; ++i) hist[i] += lh[i];
      }
      ws_free(&w);
    }
    free(lh);
  }
  if (err) return ORACLE_ENOMEM;
  *total = tot;
  return ORACLE_OK;
}

int oracle_mce_ops(int64_t n, const int32_t *row_ptr, const int32_t *split, const int32_t *cs,
                   int64_t begin, int64_t end, int64_t stride, int nthreads, uint64_t *total,
                   uint64_t *hist, int hist_len, uint64_t *root_count, uint64_t *root_nodes,
                   uint64_t *root_ops) {
  return mce_roots(n, row_ptr, split, cs, begin, end, stride, nthreads, total, hist, hist_len,
                   root_count, root_nodes, root_ops, NULL);
}

int oracle_mce(int64_t n, const int32_t *row_ptr, const int32_t *split, const int32_t *cs,
               int64_t begin, int64_t end, int64_t stride, int nthreads, uint64_t *total,
               uint64_t *hist, int hist_len, uint64_t *root_count, uint64_t *root_nodes) {
  return mce_roots(n, row_ptr, split, cs, begin, end, stride, nthreads, total, hist, hist_len,
                   root_count, root_nodes, NULL, NULL);
}

/* The L2 (edge-rooted) scheme over every root; prio = the peel's priorities. */
int oracle_mce_l2(int64_t n, const int32_t *row_ptr, const int32_t *split, const int32_t *cs,
                  const uint32_t *prio, int nthreads, uint64_t *total, uint64_t *hist,
                  int hist_len, uint64_t *root_count, uint64_t *root_nodes) {
  if (!prio && n > 0) return ORACLE_EINVAL;
  return mce_roots(n, row_ptr, split, cs, 0, n, 1, nthreads, total, hist, hist_len, root_count,
                   root_nodes, NULL, prio);
}

/* Peel + orient + search in one call (all roots). */
int oracle_count(int64_t n, const int32_t *row_ptr, const int32_t *col, int nthreads,
                 uint64_t *total, uint64_t *hist, int hist_len, int32_t *degeneracy) {
  if (n < 0 || !total) return ORACLE_EINVAL;
  if (n == 0) {
    *total = 0;
    if (hist)
      for (int i = 0; i < hist_len; ++i) hist[i] = 0;
    if (degeneracy) *degeneracy = 0;
    return ORACLE_OK;
  }
  const int64_t m = row_ptr[n];
  uint32_t *prio = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)n);
  int32_t *split = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
  int32_t *cs = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m ? m : 1));
  int rc = ORACLE_ENOMEM;
  if (prio && split && cs) {
    rc = oracle_peel(n, row_ptr, col, prio, NULL, degeneracy);
    if (!rc) rc = oracle_orient(n, row_ptr, col, prio, split, cs);
    if (!rc)
      rc = oracle_mce(n, row_ptr, split, cs, 0, n, 1, nthreads, total, hist, hist_len, NULL,
                      NULL);
  }
  free(prio); free(split); free(cs);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Independent checker 1: all cliques of a graph with n <= 64 vertices.     */
/* A clique C is maximal iff no vertex outside C is adjacent to all of C.   */
/* ------------------------------------------------------------------------ */
static void brute_rec(const uint64_t *adj, uint64_t clique, int size, uint64_t common,
                      int last, int n, uint64_t *total, uint64_t *hist, int hist_len) {
  if (size >= 2 && common == 0) {
    ++*total;
    if (hist && size < hist_len) hist[size]++;
  }
  for (int v = last + 1; v < n; ++v)
    if ((common >> v) & 1) brute_rec(adj, clique | (1ull << v), size + 1, common & adj[v], v, n, total, hist, hist_len);
}

int oracle_brute(int64_t n, const int32_t *row_ptr, const int32_t *col, uint64_t *total,
                 uint64_t *hist, int hist_len) {
  if (n < 0 || n > 64 || !total) return ORACLE_ELIMIT;
  uint64_t adj[64] = {0};
  for (int64_t v = 0; v < n; ++v)
    for (int64_t j = row_ptr[v]; j < row_ptr[v + 1]; ++j) adj[v] |= 1ull << col[j];
  if (hist)
    for (int i = 0; i < hist_len; ++i) hist[i] = 0;
  *total = 0;
  /* start from each single vertex; `common` = vertices adjacent to all of C */
  for (int v = 0; v < n; ++v) {
    /* a clique is generated from its smallest vertex; maximality needs every
       outside vertex, so pass adjacency including vertices below v */
    uint64_t common = adj[v];
    /* recursion only extends with larger vertices but tests all of common */
    brute_rec(adj, 1ull << v, 1, common, v, (int)n, total, hist, hist_len);
  }
  return ORACLE_OK;
}

/* ------------------------------------------------------------------------ */
/* Independent checker 2: textbook Tomita pivoting on the whole graph       */
/* (Tomita, Tanaka, Takahashi 2006), pivot from P u X, bitsets over all n.  */
/* Size-1 cliques are dropped to match the counting convention.             */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t n, W;
  const uint64_t *adj;
  uint64_t *total, *hist;
  int hist_len;
} tt_ctx;

static void tt_rec(tt_ctx *c, uint64_t *P, uint64_t *X, int size, uint64_t *buf) {
  const int64_t W = c->W;
  int emptyP = 1, emptyX = 1;
  for (int64_t k = 0; k < W; ++k) {
    emptyP &= P[k] == 0;
    emptyX &= X[k] == 0;
  }
  if (emptyP) {
    if (emptyX && size >= 2) {
      ++*c->total;
      if (c->hist && size < c->hist_len) c->hist[size]++;
    }
    return;
  }
  int64_t piv = -1, best = -1;
  for (int64_t k = 0; k < W; ++k) {
    uint64_t cand = P[k] | X[k];
    while (cand) {
      const int64_t u = k * 64 + __builtin_ctzll(cand);
      cand &= cand - 1;
      int64_t s = 0;
      for (int64_t q = 0; q < W; ++q) s += popc64(P[q] & c->adj[u * W + q]);
      if (s > best) {
        best = s;
        piv = u;
      }
    }
  }
  uint64_t *np = buf, *nx = buf + W, *ext = buf + 2 * W;
  for (int64_t k = 0; k < W; ++k) ext[k] = P[k] & ~c->adj[piv * W + k];
  for (int64_t k = 0; k < W; ++k) {
    while (ext[k]) {
      const int64_t v = k * 64 + __builtin_ctzll(ext[k]);
      ext[k] &= ext[k] - 1;
      for (int64_t q = 0; q < W; ++q) {
        np[q] = P[q] & c->adj[v * W + q];
        nx[q] = X[q] & c->adj[v * W + q];
      }
      tt_rec(c, np, nx, size + 1, buf + 3 * W);
      P[k] &= ~(1ull << (v % 64));
      X[k] |= 1ull << (v % 64);
    }
  }
}

int oracle_tomita(int64_t n, const int32_t *row_ptr, const int32_t *col, uint64_t *total,
                  uint64_t *hist, int hist_len) {
  if (n < 0 || n > 8192 || !total) return ORACLE_ELIMIT;
  const int64_t W = n ? (n + 63) / 64 : 1;
  uint64_t *adj = (uint64_t *)calloc((size_t)(n ? n : 1) * W, 8);
  uint64_t *P = (uint64_t *)calloc((size_t)W, 8), *X = (uint64_t *)calloc((size_t)W, 8);
  uint64_t *buf = (uint64_t *)calloc((size_t)(3 * W) * (size_t)(n + 2), 8);
  if (!adj || !P || !X || !buf) {
    free(adj); free(P); free(X); free(buf);
    return ORACLE_ENOMEM;
  }
  for (int64_t v = 0; v < n; ++v) {
    P[v / 64] |= 1ull << (v % 64);
    for (int64_t j = row_ptr[v]; j < row_ptr[v + 1]; ++j)
      adj[v * W + col[j] / 64] |= 1ull << (col[j] % 64);
  }
  if (hist)
    for (int i = 0; i < hist_len; ++i) hist[i] = 0;
  *total = 0;
  tt_ctx c = {n, W, adj, total, hist, hist_len};
  if (n) tt_rec(&c, P, X, 0, buf);
  free(adj); free(P); free(X); free(buf);
  return ORACLE_OK;
}

/* ------------------------------------------------------------------------ */
/* Cost-model reference in double precision (checks the GPU MLP kernels).    */
/* Layout: W1[64][8], b1[64], W2[64][64], b2[64], W3[64], b3; ReLU;          */
/* loss = mean (out - y)^2.  The caller passes the weights the GPU uses       */
/* (its FP16 copy, widened), so only the accumulation precision differs.     */
/* ------------------------------------------------------------------------ */
#define MLP_F 8
#define MLP_H 64
#define MLP_NP (MLP_H * MLP_F + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1)

static double mlp_fwd(const double *w, const float *x, double *h1, double *h2) {
  const double *W1 = w, *b1 = W1 + MLP_H * MLP_F, *W2 = b1 + MLP_H, *b2 = W2 + MLP_H * MLP_H;
  const double *W3 = b2 + MLP_H, *b3 = W3 + MLP_H;
  for (int j = 0; j < MLP_H; ++j) {
    double a = b1[j];
    for (int i = 0; i < MLP_F; ++i) a += W1[j * MLP_F + i] * x[i];
    h1[j] = a > 0 ? a : 0;
  }
  double out = b3[0];
  for (int k = 0; k < MLP_H; ++k) {
    double a = b2[k];
    for (int j = 0; j < MLP_H; ++j) a += W2[k * MLP_H + j] * h1[j];
    h2[k] = a > 0 ? a : 0;
    out += W3[k] * h2[k];
  }
  return out;
}

int oracle_mlp_forward(const float *params, const float *X, int64_t count, double *out) {
  double w[MLP_NP], h1[MLP_H], h2[MLP_H];
  for (int p = 0; p < MLP_NP; ++p) w[p] = params[p];
  for (int64_t s = 0; s < count; ++s) out[s] = mlp_fwd(w, X + s * MLP_F, h1, h2);
  return ORACLE_OK;
}

int oracle_mlp_grad(const float *params, const float *X, const float *Y, int64_t count,
                    double *grad, double *loss) {
  if (count < 1) return ORACLE_EINVAL;
  double w[MLP_NP], h1[MLP_H], h2[MLP_H], d2[MLP_H], a1;
  for (int p = 0; p < MLP_NP; ++p) {
    w[p] = params[p];
    grad[p] = 0;
  }
  const double *W2 = w + MLP_H * MLP_F + MLP_H, *W3 = W2 + MLP_H * MLP_H + MLP_H;
  double *gW1 = grad, *gb1 = gW1 + MLP_H * MLP_F, *gW2 = gb1 + MLP_H, *gb2 = gW2 + MLP_H * MLP_H;
  double *gW3 = gb2 + MLP_H, *gb3 = gW3 + MLP_H;
  double L = 0;
  for (int64_t s = 0; s < count; ++s) {
    const float *x = X + s * MLP_F;
    const double e = mlp_fwd(w, x, h1, h2) - Y[s];
    L += e * e;
    const double g = 2 * e / (double)count;
    gb3[0] += g;
    for (int k = 0; k < MLP_H; ++k) {
      gW3[k] += g * h2[k];
      d2[k] = h2[k] > 0 ? g * W3[k] : 0;
      gb2[k] += d2[k];
      for (int j = 0; j < MLP_H; ++j) gW2[k * MLP_H + j] += d2[k] * h1[j];
    }
    for (int j = 0; j < MLP_H; ++j) {
      double a = 0;
      if (h1[j] > 0)
        for (int k = 0; k < MLP_H; ++k) a += W2[k * MLP_H + j] * d2[k];
      a1 = a;
      gb1[j] += a1;
      for (int i = 0; i < MLP_F; ++i) gW1[j * MLP_F + i] += a * x[i];
    }
  }
  *loss = L / (double)count;
  return ORACLE_OK;
}
