/*
 * TEST INFRASTRUCTURE ONLY — the oracle (see tamm_oracle.h).
 *
 * Plain-C restatement of TAMM's CPU block-contraction path.  Paths in citations are
 * relative to the TAMM source tree.  Build: oracle/Makefile (liboracle_port.so).
 */
#include "tamm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- helpers */

static int find_label(const int* v, int n, int x) {
  for(int i = 0; i < n; i++)
    if(v[i] == x) return i;
  return -1;
}

static int64_t prod64(const int64_t* d, int n) {
  int64_t p = 1;
  for(int i = 0; i < n; i++) p *= d[i];
  return p;
}

/* internal::are_permutations (src/tamm/perm.hpp:36-47). */
static int are_permutations(const int* v1, int n1, const int* v2, int n2) {
  if(n1 != n2) return 0;
  int taken[OR_MAXR] = {0};
  for(int i = 0; i < n1; i++) {
    int p = find_label(v2, n2, v1[i]); /* std::find: first occurrence */
    if(p < 0) return 0;
    if(taken[p]) return 0;
    taken[p] = 1;
  }
  return 1;
}

/* hptt::create_plan(perm, ndim, alpha, A, sizeA, NULL, beta, B, NULL, ESTIMATE, 1,
 * NULL, rowMajor=true)->execute() as called at src/tamm/kernels/assign.hpp:396-400:
 * row-major B with sizeB[j] = sizeA[perm[j]] and B = alpha*perm(A) + beta*B (B is
 * not read when beta == 0).  HPTT itself is a third-party library absent from the
 * TAMM tree; this is its documented transposition semantics. */
static void hptt_permute(const int* perm, int ndim, double alpha, const double* A,
                         const int64_t* sizeA, double beta, double* B) {
  int64_t sizeB[OR_MAXR], strideA[OR_MAXR], ia[OR_MAXR];
  int64_t n = prod64(sizeA, ndim);
  for(int j = 0; j < ndim; j++) sizeB[j] = sizeA[perm[j]];
  int64_t s = 1;
  for(int i = ndim - 1; i >= 0; i--) {
    strideA[i] = s;
    s *= sizeA[i];
  }
  (void) strideA;
  for(int i = 0; i < ndim; i++) ia[i] = 0;
  for(int64_t lin = 0; lin < n; lin++) {
    int64_t ob = 0;
    for(int j = 0; j < ndim; j++) ob = ob * sizeB[j] + ia[perm[j]];
    B[ob] = (beta == 0.0) ? alpha * A[lin] : alpha * A[lin] + beta * B[ob];
    for(int q = ndim - 1; q >= 0; q--) {
      if(++ia[q] < sizeA[q]) break;
      ia[q] = 0;
    }
  }
}

/* internal::ip_gen_loop (src/tamm/kernels/assign.hpp:312-373): loop over the unique
 * dst labels then the src-only labels, strides from the row-major layouts, and run
 * the ndim(dst)-deep loop (ip0..ip4 / ipacc0..ipacc4, assign.hpp:19-169). */
static int ip_gen_loop(double* dst, const int64_t* ddims, const int* dlabels, int nd, double scale,
                       const double* src, const int64_t* sdims, const int* slabels, int ns,
                       int is_assign) {
  int64_t sld[OR_MAXR + 1], dld[OR_MAXR + 1];
  sld[ns] = 1;
  for(int i = ns - 1; i >= 0; i--) sld[i] = sld[i + 1] * sdims[i];
  dld[nd] = 1;
  for(int i = nd - 1; i >= 0; i--) dld[i] = dld[i + 1] * ddims[i];

  int loop_labels[2 * OR_MAXR];
  int nl = 0;
  for(int i = 0; i < nd; i++)
    if(find_label(loop_labels, nl, dlabels[i]) < 0) loop_labels[nl++] = dlabels[i];
  for(int i = 0; i < ns; i++)
    if(find_label(loop_labels, nl, slabels[i]) < 0) loop_labels[nl++] = slabels[i];

  int64_t loop_dims[2 * OR_MAXR] = {0}, loop_sld[2 * OR_MAXR] = {0}, loop_dld[2 * OR_MAXR] = {0};
  for(int i = 0; i < nl; i++) {
    int p = find_label(slabels, ns, loop_labels[i]);
    if(p >= 0) {
      loop_sld[i]  = sld[p + 1];
      loop_dims[i] = sdims[p];
    }
  }
  for(int i = 0; i < nl; i++) {
    int p = find_label(dlabels, nd, loop_labels[i]);
    if(p >= 0) {
      loop_dld[i]  = dld[p + 1];
      loop_dims[i] = ddims[p];
    }
  }
  if(nd > 4) return OR_ENOTIMPL;
  if(nl < nd) return OR_EINVAL; /* repeated dst labels read past loop_dims in the reference */

  int64_t it[4] = {0, 0, 0, 0};
  int64_t total = 1;
  for(int k = 0; k < nd; k++) total *= loop_dims[k];
  for(int64_t lin = 0; lin < total; lin++) {
    int64_t so = 0, doff = 0;
    for(int k = 0; k < nd; k++) {
      so += it[k] * loop_sld[k];
      doff += it[k] * loop_dld[k];
    }
    if(is_assign) dst[doff] = scale * src[so];
    else dst[doff] += scale * src[so];
    for(int k = nd - 1; k >= 0; k--) {
      if(++it[k] < loop_dims[k]) break;
      it[k] = 0;
    }
  }
  return OR_OK;
}

int or_assign(double* dst, const int64_t* ddims, const int* dlabels, int nd, double scale,
              const double* src, const int64_t* sdims, const int* slabels, int ns, int is_assign) {
  if(nd > OR_MAXR || ns > OR_MAXR || nd < 0 || ns < 0) return OR_EINVAL;
  if(dst == NULL || src == NULL) return OR_EINVAL;
  if(are_permutations(slabels, ns, dlabels, nd)) {
    if(nd == 0) {
      /* internal::index_permute / index_permute_acc, ndim 0 (assign.hpp:187,239) */
      if(is_assign) dst[0] = scale * src[0];
      else dst[0] += scale * src[0];
      return OR_OK;
    }
    /* internal::ip_hptt (assign.hpp:375-401) */
    int perm[OR_MAXR];
    for(int i = 0; i < nd; i++) {
      int p = find_label(slabels, ns, dlabels[i]);
      if(p < 0) return OR_EINVAL;
      perm[i] = p;
    }
    hptt_permute(perm, nd, scale, src, sdims, is_assign ? 0.0 : 1.0, dst);
    return OR_OK;
  }
  return ip_gen_loop(dst, ddims, dlabels, nd, scale, src, sdims, slabels, ns, is_assign);
}

/* blas::gemm(RowMajor, NoTrans, NoTrans, ...) as called by kernels::cpu::gemm
 * (src/tamm/kernels/cpu_blas.cpp:5-10): C = alpha*A*B + beta*C, C not read when
 * beta == 0 (BLAS convention). */
static void gemm_rm(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t lda,
                    const double* B, int64_t ldb, double beta, double* C, int64_t ldc) {
  double* acc = (double*) malloc(sizeof(double) * (size_t) (n > 0 ? n : 1));
  for(int64_t i = 0; i < m; i++) {
    for(int64_t j = 0; j < n; j++) acc[j] = 0.0;
    for(int64_t p = 0; p < k; p++) {
      const double  a  = A[i * lda + p];
      const double* bp = B + p * ldb;
      for(int64_t j = 0; j < n; j++) acc[j] += a * bp[j];
    }
    double* cp = C + i * ldc;
    for(int64_t j = 0; j < n; j++) cp[j] = (beta == 0.0) ? alpha * acc[j] : alpha * acc[j] + beta * cp[j];
  }
  free(acc);
}

int or_block_multiply(double alpha, const double* abuf, const int64_t* adims, const int* alabels,
                      int na, const double* bbuf, const int64_t* bdims, const int* blabels, int nb,
                      double beta, double* cbuf, const int64_t* cdims, const int* clabels, int nc,
                      int is_assign) {
  if(abuf == NULL || bbuf == NULL || cbuf == NULL) return OR_EINVAL; /* multiply.hpp:226 */
  if(na > OR_MAXR || nb > OR_MAXR || nc > OR_MAXR) return OR_EINVAL;

  /* label classification (multiply.hpp:237-302) */
  int     batch_l[OR_MAXR], aouter_l[OR_MAXR], bouter_l[OR_MAXR], inner_l[OR_MAXR], ared_l[OR_MAXR],
    bred_l[OR_MAXR];
  int64_t batch_d[OR_MAXR], aouter_d[OR_MAXR], bouter_d[OR_MAXR], inner_d[OR_MAXR], ared_d[OR_MAXR],
    bred_d[OR_MAXR];
  int     nbt = 0, nao = 0, nbo = 0, nin = 0, nar = 0, nbr = 0;
  int64_t B = 1, M = 1, N = 1, K = 1, AR = 1, BR = 1;
  for(int i = 0; i < nc; i++) {
    int l = clabels[i], ina = find_label(alabels, na, l) >= 0, inb = find_label(blabels, nb, l) >= 0;
    if(ina && inb) {
      batch_l[nbt] = l;
      batch_d[nbt++] = cdims[i];
      B *= cdims[i];
    }
    else if(ina) {
      aouter_l[nao] = l;
      aouter_d[nao++] = cdims[i];
      M *= cdims[i];
    }
    else if(inb) {
      bouter_l[nbo] = l;
      bouter_d[nbo++] = cdims[i];
      N *= cdims[i];
    }
  }
  for(int i = 0; i < na; i++) {
    int l = alabels[i], inb = find_label(blabels, nb, l) >= 0, inc = find_label(clabels, nc, l) >= 0;
    if(inb && inc) {}
    else if(inb) {
      inner_l[nin] = l;
      inner_d[nin++] = adims[i];
      K *= adims[i];
    }
    else if(inc) {}
    else {
      AR *= adims[i];
      ared_l[nar] = l;
      ared_d[nar++] = adims[i];
    }
  }
  for(int i = 0; i < nb; i++) {
    int l = blabels[i], ina = find_label(alabels, na, l) >= 0, inc = find_label(clabels, nc, l) >= 0;
    if(ina && inc) {}
    else if(ina) {}
    else if(inc) {}
    else {
      BR *= bdims[i];
      bred_l[nbr] = l;
      bred_d[nbr++] = bdims[i];
    }
  }

  /* intermediate layouts (multiply.hpp:304-330) */
  int     ail[OR_MAXR * 2], bil[OR_MAXR * 2], cil[OR_MAXR * 2];
  int64_t aid[OR_MAXR * 2], bid[OR_MAXR * 2], cid[OR_MAXR * 2];
  int     nai = 0, nbi = 0, nci = 0;
#define APP(L, D, n, srcl, srcd, cnt)   \
  for(int q = 0; q < (cnt); q++) {     \
    L[n]   = srcl[q];                  \
    D[n++] = srcd[q];                  \
  }
  APP(ail, aid, nai, ared_l, ared_d, nar);
  APP(ail, aid, nai, batch_l, batch_d, nbt);
  APP(ail, aid, nai, aouter_l, aouter_d, nao);
  APP(ail, aid, nai, inner_l, inner_d, nin);
  APP(bil, bid, nbi, bred_l, bred_d, nbr);
  APP(bil, bid, nbi, batch_l, batch_d, nbt);
  APP(bil, bid, nbi, inner_l, inner_d, nin);
  APP(bil, bid, nbi, bouter_l, bouter_d, nbo);
  APP(cil, cid, nci, batch_l, batch_d, nbt);
  APP(cil, cid, nci, aouter_l, aouter_d, nao);
  APP(cil, cid, nci, bouter_l, bouter_d, nbo);
#undef APP
  if(nai > OR_MAXR || nbi > OR_MAXR || nci > OR_MAXR) return OR_EINVAL;

  const int64_t asize = prod64(adims, na), bsize = prod64(bdims, nb), csize = prod64(cdims, nc);
  double*       cinter = (double*) calloc((size_t) csize, sizeof(double)); /* :344-348 */
  double*       ainter = (double*) malloc(sizeof(double) * (size_t) asize);
  double*       binter = (double*) malloc(sizeof(double) * (size_t) bsize);
  int           rc     = OR_OK;

  /* transpose_inputs, CPU branch (multiply.hpp:191-192) */
  rc = or_assign(ainter, aid, ail, nai, 1.0, abuf, adims, alabels, na, 1);
  if(rc == OR_OK) rc = or_assign(binter, bid, bil, nbi, 1.0, bbuf, bdims, blabels, nb, 1);

  /* gemm_wrapper (multiply.hpp:42-74) */
  if(rc == OR_OK) {
    const int64_t abatch_ld = M * K, bbatch_ld = K * N, cbatch_ld = M * N;
    const int64_t areduce_ld = B * abatch_ld, breduce_ld = B * bbatch_ld;
    for(int64_t ari = 0; ari < AR; ari++)
      for(int64_t bri = 0; bri < BR; bri++)
        for(int64_t i = 0; i < B; i++)
          gemm_rm(M, N, K, alpha, ainter + ari * areduce_ld + i * abatch_ld, K,
                  binter + bri * breduce_ld + i * bbatch_ld, N, beta, cinter + i * cbatch_ld, N);
    /* transpose_output, CPU branch (multiply.hpp:209) */
    rc = or_assign(cbuf, cdims, clabels, nc, 1.0, cinter, cid, cil, nci, is_assign);
  }
  free(cinter);
  free(ainter);
  free(binter);
  return rc;
}

/* ------------------------------------------------------------ tiling / sparsity */

static int cmp_i64(const void* a, const void* b) {
  int64_t x = *(const int64_t*) a, y = *(const int64_t*) b;
  return (x > y) - (x < y);
}

static int64_t sort_unique(int64_t* v, int64_t n) {
  qsort(v, (size_t) n, sizeof(int64_t), cmp_i64);
  int64_t m = 0;
  for(int64_t i = 0; i < n; i++)
    if(m == 0 || v[m - 1] != v[i]) v[m++] = v[i];
  return m;
}

int64_t or_tile_offsets_uniform(int64_t n, const int64_t* bounds, int nbounds, int64_t tile,
                                int64_t* out, int64_t cap) {
  int64_t cnt = 0;
  if(tile <= 0) return -1;
  if(n == 0) {
    if(cap < 1) return -1;
    out[0] = 0;
    return 1;
  }
  if(nbounds == 0) {
    for(int64_t i = 0; i < n; i += tile) {
      if(cnt >= cap) return -1;
      out[cnt++] = i;
    }
  }
  else {
    int64_t* b = (int64_t*) malloc(sizeof(int64_t) * (size_t) nbounds);
    memcpy(b, bounds, sizeof(int64_t) * (size_t) nbounds);
    int64_t nb = sort_unique(b, nbounds);
    int64_t i = 0, j = (i == b[0]) ? 1 : 0;
    while(i < n) {
      if(cnt >= cap) {
        free(b);
        return -1;
      }
      out[cnt++] = i;
      /* tiled_index_space.hpp:1187: jump to the next boundary when the tile would
       * reach or cross it */
      if(j < nb && i + tile >= b[j]) i = b[j++];
      else i = i + tile;
    }
    free(b);
  }
  if(cnt >= cap) return -1;
  out[cnt++] = n;
  return cnt;
}

int64_t or_tile_offsets_list(int64_t n, const int64_t* bounds, int nbounds, const int64_t* tiles,
                             int64_t ntiles, int64_t* out) {
  if(n == 0) {
    out[0] = 0;
    return 1;
  }
  int64_t s = 0;
  for(int64_t t = 0; t < ntiles; t++) s += tiles[t];
  if(s != n) return -1; /* tiled_index_space.hpp:1211-1215 */
  int64_t cnt = 0, j = 0;
  for(int64_t i = 0; i < n; i += tiles[j++]) out[cnt++] = i;
  out[cnt++] = n;
  if(nbounds > 0) {
    int64_t* b = (int64_t*) malloc(sizeof(int64_t) * (size_t) nbounds);
    memcpy(b, bounds, sizeof(int64_t) * (size_t) nbounds);
    int64_t nb = sort_unique(b, nbounds);
    for(int64_t q = 0; q < nb; q++) {
      /* binary_search of every boundary among the tile starts (:1252-1257) */
      int found = 0;
      for(int64_t r = 0; r < cnt; r++)
        if(out[r] == b[q]) {
          found = 1;
          break;
        }
      if(!found) {
        free(b);
        return -1;
      }
    }
    free(b);
  }
  return cnt;
}

int or_is_non_zero(int nmodes, const int* spins, const int* mask, int has_spin) {
  if(!has_spin) return 1;
  int upper = 0, lower = 0;
  for(int i = 0; i < nmodes; i++) {
    if(mask[i] == 0) upper += spins[i];
    else if(mask[i] == 1) lower += spins[i];
  }
  return upper == lower;
}

static int block_admitted(const or_tensor* t, const int64_t* blockid) {
  int spins[OR_MAXR];
  for(int i = 0; i < t->nmodes; i++) spins[i] = t->tile_spin[i] ? t->tile_spin[i][blockid[i]] : 0;
  return or_is_non_zero(t->nmodes, spins, t->spin_mask, t->has_spin);
}

static int64_t block_key(const or_tensor* t, const int64_t* blockid) {
  /* Distribution_NW::compute_key_offsets / compute_key (distribution.hpp:334-355) */
  int64_t key = 0, stride = 1;
  for(int i = t->nmodes - 1; i >= 0; i--) {
    key += blockid[i] * stride;
    stride *= t->ntiles[i];
  }
  return key;
}

static int64_t block_elems(const or_tensor* t, const int64_t* blockid) {
  int64_t s = 1;
  for(int i = 0; i < t->nmodes; i++) s *= t->tile_size[i][blockid[i]];
  return s;
}

typedef struct {
  int64_t key, size;
} key_size;

static int cmp_key(const void* a, const void* b) {
  int64_t x = ((const key_size*) a)->key, y = ((const key_size*) b)->key;
  return (x > y) - (x < y);
}

int64_t or_nw_pack(or_tensor* t, int64_t* keys_out, int64_t* offsets_out, int64_t* total_out) {
  int64_t nall = 1;
  for(int i = 0; i < t->nmodes; i++) nall *= t->ntiles[i];
  key_size* h  = (key_size*) malloc(sizeof(key_size) * (size_t) (nall > 0 ? nall : 1));
  int64_t   nb = 0;
  int64_t   id[OR_MAXR] = {0};
  for(int64_t lin = 0; lin < nall; lin++) {
    if(block_admitted(t, id)) {
      h[nb].key    = block_key(t, id);
      h[nb++].size = block_elems(t, id);
    }
    for(int q = t->nmodes - 1; q >= 0; q--) {
      if(++id[q] < t->ntiles[q]) break;
      id[q] = 0;
    }
  }
  qsort(h, (size_t) nb, sizeof(key_size), cmp_key);
  int64_t off = 0;
  for(int64_t i = 0; i < nb; i++) {
    keys_out[i]    = h[i].key;
    offsets_out[i] = off;
    off += h[i].size;
  }
  free(h);
  *total_out = off;
  return nb;
}

int64_t or_nw_locate(const or_tensor* t, const int64_t* blockid) {
  int64_t key = block_key(t, blockid);
  int64_t lo = 0, hi = t->nblocks;
  while(lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if(t->keys[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  if(lo < t->nblocks && t->keys[lo] == key) return t->offsets[lo];
  return -1;
}

/* ---------------------------------------------------------------- MultOp bufacc */

static void translate(const or_operand* op, const int64_t* labelid, int64_t* blockid) {
  for(int i = 0; i < op->t->nmodes; i++)
    blockid[i] = op->tmap[i] ? op->tmap[i][labelid[i]] : labelid[i];
}

typedef struct {
  int     nred;
  int     red[2 * OR_MAXR];
  int64_t red_nt[2 * OR_MAXR];
  int     a_out[OR_MAXR], a_red[OR_MAXR], b_out[OR_MAXR], b_red[OR_MAXR];
} mult_maps;

static int cmp_int(const void* a, const void* b) {
  int x = *(const int*) a, y = *(const int*) b;
  return (x > y) - (x < y);
}

/* reduction labels and rhs->output/reduction maps (multop.hpp:593-629) */
static void build_maps(const or_operand* c, const or_operand* a, const or_operand* b,
                       mult_maps* mm) {
  const int nc = c->t->nmodes, na = a->t->nmodes, nb = b->t->nmodes;
  int       allr[2 * OR_MAXR];
  int64_t   allnt[2 * OR_MAXR];
  int       nall = 0;
  for(int i = 0; i < na; i++)
    if(find_label(allr, nall, a->labels[i]) < 0) {
      allr[nall]    = a->labels[i];
      allnt[nall++] = a->lntiles[i];
    }
  for(int i = 0; i < nb; i++)
    if(find_label(allr, nall, b->labels[i]) < 0) {
      allr[nall]    = b->labels[i];
      allnt[nall++] = b->lntiles[i];
    }
  int sorted[2 * OR_MAXR];
  memcpy(sorted, allr, sizeof(int) * (size_t) nall);
  qsort(sorted, (size_t) nall, sizeof(int), cmp_int);
  mm->nred = 0;
  for(int i = 0; i < nall; i++) {
    if(find_label(c->labels, nc, sorted[i]) >= 0) continue;
    mm->red[mm->nred]      = sorted[i];
    mm->red_nt[mm->nred++] = allnt[find_label(allr, nall, sorted[i])];
  }
  for(int i = 0; i < na; i++) {
    mm->a_out[i] = find_label(c->labels, nc, a->labels[i]);
    mm->a_red[i] = find_label(mm->red, mm->nred, a->labels[i]);
  }
  for(int i = 0; i < nb; i++) {
    mm->b_out[i] = find_label(c->labels, nc, b->labels[i]);
    mm->b_red[i] = find_label(mm->red, mm->nred, b->labels[i]);
  }
}

static void fill_rhs_id(const or_operand* op, const int* out, const int* red, const int64_t* itval,
                        const int64_t* inner, int64_t* labelid) {
  for(int i = 0; i < op->t->nmodes; i++) {
    labelid[i] = 0;
    if(out[i] != -1) labelid[i] = itval[out[i]];
    if(red[i] != -1) labelid[i] = inner[red[i]];
  }
}

static int next_tuple(int64_t* it, const int64_t* nt, int n) {
  for(int q = n - 1; q >= 0; q--) {
    if(++it[q] < nt[q]) return 1;
    it[q] = 0;
  }
  return 0;
}

static int mult_loop(or_operand* c, double alpha, const or_operand* a, const or_operand* b,
                     int compute, int64_t* ntriples, double* flops, or_block_fn fn) {
  const or_tensor *C = c->t, *A = a->t, *Bt = b->t;
  mult_maps        mm;
  build_maps(c, a, b, &mm);
  int64_t itval[OR_MAXR] = {0}, inner[2 * OR_MAXR] = {0};
  int64_t cid[OR_MAXR], aid_l[OR_MAXR], aid[OR_MAXR], bid_l[OR_MAXR], bid[OR_MAXR];
  int64_t cd[OR_MAXR], ad[OR_MAXR], bd[OR_MAXR];
  int64_t ncomb = 1;
  for(int i = 0; i < C->nmodes; i++) ncomb *= c->lntiles[i];
  if(ncomb == 0) return OR_OK;
  int rc = OR_OK;
  do { /* LHS LabelLoopNest, row-major, last label fastest */
    translate(c, itval, cid);
    if(!block_admitted(C, cid)) continue; /* multop.hpp:888-889 (single owner) */
    int64_t csize = block_elems(C, cid);
    for(int i = 0; i < C->nmodes; i++) cd[i] = C->tile_size[i][cid[i]];
    double* cbuf = compute ? (double*) calloc((size_t) csize, sizeof(double)) : NULL;
    for(int i = 0; i < mm.nred; i++) inner[i] = 0;
    int more = 1;
    while(more) { /* reduction LabelLoopNest (multop.hpp:704) */
      int ok = 1;
      for(int i = 0; i < mm.nred; i++)
        if(mm.red_nt[i] == 0) ok = 0;
      if(ok) {
        fill_rhs_id(a, mm.a_out, mm.a_red, itval, inner, aid_l);
        translate(a, aid_l, aid);
        fill_rhs_id(b, mm.b_out, mm.b_red, itval, inner, bid_l);
        translate(b, bid_l, bid);
        if(block_admitted(A, aid) && block_admitted(Bt, bid)) {
          if(ntriples) (*ntriples)++;
          if(flops) {
            double k = 1;
            for(int i = 0; i < mm.nred; i++) {
              int p = -1;
              for(int q = 0; q < A->nmodes; q++)
                if(a->labels[q] == mm.red[i]) p = q;
              if(p >= 0) k *= (double) A->tile_size[p][aid[p]];
              else
                for(int q = 0; q < Bt->nmodes; q++)
                  if(b->labels[q] == mm.red[i]) k *= (double) Bt->tile_size[q][bid[q]];
            }
            *flops += 2.0 * (double) csize * k;
          }
          if(compute) {
            int64_t ao = or_nw_locate(A, aid), bo = or_nw_locate(Bt, bid);
            if(ao < 0 || bo < 0) {
              rc = OR_EINVAL;
              free(cbuf);
              return rc;
            }
            for(int i = 0; i < A->nmodes; i++) ad[i] = A->tile_size[i][aid[i]];
            for(int i = 0; i < Bt->nmodes; i++) bd[i] = Bt->tile_size[i][bid[i]];
            /* kernels::block_multiply(..., cscale=1, is_assign=false) (multop.hpp:793-798) */
            rc = fn(alpha, A->data + ao, ad, a->labels, A->nmodes, Bt->data + bo, bd, b->labels,
                    Bt->nmodes, 1.0, cbuf, cd, c->labels, C->nmodes, 0);
            if(rc != OR_OK) {
              free(cbuf);
              return rc;
            }
          }
        }
      }
      more = mm.nred > 0 ? next_tuple(inner, mm.red_nt, mm.nred) : 0;
    }
    if(compute) { /* ctensor.add (multop.hpp:835-838) */
      int64_t co = or_nw_locate(C, cid);
      if(co < 0) {
        free(cbuf);
        return OR_EINVAL;
      }
      for(int64_t q = 0; q < csize; q++) C->data[co + q] += cbuf[q];
      free(cbuf);
    }
  } while(C->nmodes > 0 ? next_tuple(itval, c->lntiles, C->nmodes) : 0);
  return rc;
}

int or_mult_bufacc(or_operand* c, double alpha, const or_operand* a, const or_operand* b) {
  return mult_loop(c, alpha, a, b, 1, NULL, NULL, or_block_multiply);
}

int or_mult_bufacc_fn(or_operand* c, double alpha, const or_operand* a, const or_operand* b,
                      or_block_fn fn) {
  return mult_loop(c, alpha, a, b, 1, NULL, NULL, fn ? fn : or_block_multiply);
}

int or_mult_count(const or_operand* c, const or_operand* a, const or_operand* b,
                  int64_t* ntriples, double* flops) {
  *ntriples = 0;
  *flops    = 0.0;
  return mult_loop((or_operand*) c, 1.0, a, b, 0, ntriples, flops, or_block_multiply);
}

/* Elements stored = offset of the last (largest-key) block + its size. */
static int64_t stored_elems(const or_tensor* t) {
  if(t->nblocks == 0) return 0;
  int64_t id[OR_MAXR], key = t->keys[t->nblocks - 1];
  for(int i = t->nmodes - 1; i >= 0; i--) {
    id[i] = key % t->ntiles[i];
    key /= t->ntiles[i];
  }
  return t->offsets[t->nblocks - 1] + block_elems(t, id);
}

void or_set(or_tensor* t, double value, int is_assign) {
  int64_t total = stored_elems(t);
  for(int64_t q = 0; q < total; q++) t->data[q] = is_assign ? value : t->data[q] + value;
}

double or_norm(const or_tensor* t) {
  int64_t total = stored_elems(t);
  double  s     = 0.0;
  for(int64_t q = 0; q < total; q++) s += t->data[q] * t->data[q];
  return sqrt(s);
}

/* ------------------------------------------------------------- seeded inputs */

static uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static double u01(uint64_t seed, uint64_t i) {
  uint64_t h = splitmix64(splitmix64(seed) ^ (i * 0xD1B54A32D192ED03ull));
  return (double) (h >> 11) * (1.0 / 9007199254740992.0);
}

double or_uniform(uint64_t seed, uint64_t i, double lo, double hi) {
  return lo + (hi - lo) * u01(seed, i);
}

double or_normal(uint64_t seed, uint64_t i, double mean, double sd) {
  double u1 = u01(seed, 2 * i), u2 = u01(seed, 2 * i + 1);
  if(u1 < 1e-300) u1 = 1e-300;
  return mean + sd * sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

void or_fill_uniform(double* x, int64_t n, uint64_t seed, uint64_t first, double lo, double hi) {
  for(int64_t q = 0; q < n; q++) x[q] = or_uniform(seed, first + (uint64_t) q, lo, hi);
}

void or_fill_normal(double* x, int64_t n, uint64_t seed, uint64_t first, double mean, double sd) {
  for(int64_t q = 0; q < n; q++) x[q] = or_normal(seed, first + (uint64_t) q, mean, sd);
}
