/*
 * pfgt_oracle.c -- CPU restatement (FP64, plain C, single thread) of the
 * reference discrete point fast Gauss transform `pfgt`.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it.  The product library never links or calls it.
 *
 * Parity status: the reference (Fortran 77 + finufft) cannot be compiled in
 * this environment (no Fortran compiler, finufft and FFTW absent), and its
 * test suite holds no golden vectors or fixtures.  The restatement is pinned
 * instead (a) to the mathematical definition through an independent exact
 * FP64 direct sum (oracle_direct_exact, periodic images included) and (b) to
 * the reference test's own accuracy criterion (test/pfgt/test_pfgt_all.f:
 * 437-512, relative l2 `derr`).  Golden fixtures generated from this file are
 * committed under tests/golden/ with their generating script.
 *
 * Each function names the reference routine (file:line, paths relative to the
 * reference project root) whose behaviour it restates.  The finufft calls of
 * the reference (pfgt.f:752-802, 853-1069; pfgt_nufftrouts.f:138-150,
 * 282-298) are replaced by exact separable non-uniform DFTs, i.e. the
 * infinitely accurate limit of the NUFFT the reference requests.
 *
 * Known reference defects are reproduced only when `quirks` != 0:
 *   bit 0: ifpgh == ifpghtarg far-field skip of the multi-threaded branch
 *          (pfgt.f:918-948).
 *   bit 1: nd > 1 index-order scramble of the potential coefficients in the
 *          evaluation (pfgt_nufftrouts.f:252-258).
 * The OpenMP list-1 race (tree_routs_nd.f:1171-1253) cannot occur here
 * (serial code).
 *
 * Conventions: all arrays are 0-based; box ids are 0-based (the reference is
 * 1-based).  Point/field layouts follow the reference's column-major layout:
 * sources[i*dim+k], charge[i*nd+id], grad[(i*dim+k)*nd+id],
 * hess[(i*nhess+m)*nd+id].
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double complex zcplx;

#define MAXDIM 3

/* ------------------------------------------------------------------------ */
/* small helpers                                                            */
/* ------------------------------------------------------------------------ */

static void *xmalloc(size_t n) {
  void *p = malloc(n ? n : 1);
  if (!p) {
    fprintf(stderr, "oracle: out of memory (%zu bytes)\n", n);
    abort();
  }
  return p;
}
static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s ? s : 1);
  if (!p) {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}
static int ipow(int b, int e) {
  int r = 1;
  while (e-- > 0) r *= b;
  return r;
}

/* Child sign convention, pts_tree_nd.f:1418-1464 (get_child_box_sign):
 * child j (0-based) has coordinate k on the + side iff bit k of j is set. */
static int child_sign(int j, int k) { return ((j >> k) & 1) ? 1 : -1; }

/* find_childbox_ind, pts_tree_nd.f:713-741: bit k set iff x_k - c_k >= 0. */
static int child_index(int dim, const double *x, const double *c) {
  int k, idx = 0;
  for (k = 0; k < dim; k++)
    if (x[k] - c[k] >= 0) idx |= (1 << k);
  return idx;
}

/* Fortran single-precision literal 1.05 promoted to double, as used in the
 * colleague tests of tree_routs_nd.f:224 and pts_tree_nd.f:1020. */
static double f105(void) { return (double)1.05f; }

/* ------------------------------------------------------------------------ */
/* tree                                                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
  int dim, mc, mnbors;
  int nlevels, nboxes, cap;
  int *laddr;      /* 2*(nlevels+1): first,last box of each level (-1 empty) */
  int *ilevel, *iparent, *nchild, *ichild; /* ichild[b*mc+j] */
  int *nnbors, *nbors;                     /* nbors[b*mnbors+j] */
  double *centers;                         /* centers[b*dim+k] */
  double *boxsize;                         /* 0..nlevels */
  int *iflag;
} otree;

static void tree_reserve(otree *t, int need) {
  if (need <= t->cap) return;
  int nc = t->cap ? t->cap : 1024;
  while (nc < need) nc *= 2;
  t->ilevel = realloc(t->ilevel, sizeof(int) * nc);
  t->iparent = realloc(t->iparent, sizeof(int) * nc);
  t->nchild = realloc(t->nchild, sizeof(int) * nc);
  t->ichild = realloc(t->ichild, sizeof(int) * nc * t->mc);
  t->nnbors = realloc(t->nnbors, sizeof(int) * nc);
  t->nbors = realloc(t->nbors, sizeof(int) * nc * t->mnbors);
  t->centers = realloc(t->centers, sizeof(double) * nc * t->dim);
  t->iflag = realloc(t->iflag, sizeof(int) * nc);
  if (!t->ilevel || !t->iparent || !t->nchild || !t->ichild || !t->nnbors ||
      !t->nbors || !t->centers || !t->iflag) {
    fprintf(stderr, "oracle: out of memory (tree)\n");
    abort();
  }
  t->cap = nc;
}

static void tree_free(otree *t) {
  free(t->laddr); free(t->ilevel); free(t->iparent); free(t->nchild);
  free(t->ichild); free(t->nnbors); free(t->nbors); free(t->centers);
  free(t->boxsize); free(t->iflag);
  memset(t, 0, sizeof(*t));
}

/* Append the mc children of box `ib` at level `lev`+1 with child-box size
 * `bs`; tree_refine_boxes, tree_routs_nd.f:9-62 (children centre =
 * parent centre + sign*bs/2). */
static void make_children(otree *t, int ib, double bs, int childlev) {
  int j, k, l, dim = t->dim, mc = t->mc;
  double bsh = bs / 2;
  tree_reserve(t, t->nboxes + mc);
  t->nchild[ib] = mc;
  for (j = 0; j < mc; j++) {
    int jb = t->nboxes + j;
    for (k = 0; k < dim; k++)
      t->centers[jb * dim + k] = t->centers[ib * dim + k] + child_sign(j, k) * bsh;
    t->iparent[jb] = ib;
    t->nchild[jb] = 0;
    for (l = 0; l < mc; l++) t->ichild[jb * mc + l] = -1;
    t->ichild[ib * mc + j] = jb;
    t->ilevel[jb] = childlev;
    t->nnbors[jb] = 0;
    t->iflag[jb] = 0;
  }
  t->nboxes += mc;
}

/* Stable bin sort of the points of box ib into its children;
 * sort_pts_to_children, pts_tree_nd.f:650-708. se[2*b] = first, se[2*b+1] =
 * last (inclusive, 0-based; empty = first > last). */
static void sort_to_children(const otree *t, int ib, const double *x, int n,
                             int *iperm, int *se, int *tmp, int *bin) {
  int mc = t->mc, dim = t->dim, i, j;
  if (n == 0) {
    for (j = 0; j < mc; j++) {
      int jb = t->ichild[ib * mc + j];
      se[2 * jb] = 0;
      se[2 * jb + 1] = -1;
    }
    return;
  }
  int is = se[2 * ib], ie = se[2 * ib + 1];
  int cnt[8] = {0}, ip[9];
  for (i = is; i <= ie; i++) {
    int c = child_index(dim, &x[(size_t)iperm[i] * dim], &t->centers[ib * dim]);
    bin[i - is] = c;
    cnt[c]++;
  }
  ip[0] = 0;
  for (j = 0; j < mc; j++) ip[j + 1] = ip[j] + cnt[j];
  for (j = 0; j < mc; j++) {
    int jb = t->ichild[ib * mc + j];
    se[2 * jb] = is + ip[j];
    se[2 * jb + 1] = is + ip[j + 1] - 1;
  }
  for (i = is; i <= ie; i++) tmp[ip[bin[i - is]]++] = iperm[i];
  for (i = is; i <= ie; i++) iperm[i] = tmp[i - is];
}

/* computecoll, tree_routs_nd.f:106-242. */
static void compute_colleagues(otree *t, int iperiod) {
  int dim = t->dim, mc = t->mc, mnb = t->mnbors;
  double bs0 = t->boxsize[0];
  int b, ilev, i, j, k;
  for (b = 0; b < t->nboxes; b++) {
    t->nnbors[b] = 0;
    for (j = 0; j < mnb; j++) t->nbors[b * mnb + j] = -1;
  }
  t->nnbors[0] = 1;
  t->nbors[0] = 0;
  for (ilev = 1; ilev <= t->nlevels; ilev++) {
    int f = t->laddr[2 * ilev], l = t->laddr[2 * ilev + 1];
    double tol = f105() * t->boxsize[ilev];
    for (b = f; b <= l; b++) {
      int dad = t->iparent[b];
      for (i = 0; i < t->nnbors[dad]; i++) {
        int jb = t->nbors[dad * mnb + i];
        for (j = 0; j < mc; j++) {
          int kb = t->ichild[jb * mc + j];
          if (kb < 0) continue;
          int ok = 1;
          for (k = 0; k < dim; k++) {
            double dis = fabs(t->centers[kb * dim + k] - t->centers[b * dim + k]);
            if (iperiod == 1) {
              double dp1 = bs0 - dis;
              if (dp1 < dis) dis = dp1;
            }
            if (dis > tol) { ok = 0; break; }
          }
          if (ok) t->nbors[b * mnb + t->nnbors[b]++] = kb;
        }
      }
    }
  }
}

/* tree_refine_boxes_flag, tree_routs_nd.f:365-424: refine every box of
 * [first, first+nbloc) with iflag > 0; children of flag-1 boxes get flag 3,
 * children of flag-2 boxes get flag 0. */
static void refine_flagged(otree *t, int first, int nbloc, double bs, int lev) {
  int i;
  for (i = 0; i < nbloc; i++) {
    int ib = first + i;
    if (t->iflag[ib] > 0) {
      int fl = t->iflag[ib], j, c0 = t->nboxes;
      make_children(t, ib, bs, lev + 1);
      for (j = 0; j < t->mc; j++) t->iflag[c0 + j] = (fl == 1) ? 3 : 0;
    }
  }
}

/* updateflags, tree_routs_nd.f:248-357. */
static void update_flags(otree *t, int curlev, int first, int last) {
  int dim = t->dim, mc = t->mc, mnb = t->mnbors;
  double distest = 1.05 * (t->boxsize[curlev] + t->boxsize[curlev + 1]) / 2.0;
  int b, i, j, k;
  for (b = first; b <= last; b++) {
    if (t->iflag[b] != 3) continue;
    t->iflag[b] = 0;
    for (i = 0; i < t->nnbors[b] && t->iflag[b] == 0; i++) {
      int jb = t->nbors[b * mnb + i];
      for (j = 0; j < mc; j++) {
        int kb = t->ichild[jb * mc + j];
        if (kb >= 0 && t->nchild[kb] > 0) {
          int ict = 0;
          for (k = 0; k < dim; k++)
            if (fabs(t->centers[kb * dim + k] - t->centers[b * dim + k]) <= distest)
              ict++;
          if (ict == dim) { t->iflag[b] = 1; break; }
        }
      }
    }
  }
}

/* pts_tree_reorg, pts_tree_nd.f:1063-1219: renumber so that each level holds
 * its original boxes followed by its tail boxes. */
static void tree_reorg(otree *t, const int *tail) {
  int nb = t->nboxes, dim = t->dim, mc = t->mc, nl = t->nlevels;
  int *map = xmalloc(sizeof(int) * nb);
  int *lev = xmalloc(sizeof(int) * nb), *par = xmalloc(sizeof(int) * nb);
  int *nch = xmalloc(sizeof(int) * nb), *chi = xmalloc(sizeof(int) * nb * mc);
  int *flg = xmalloc(sizeof(int) * nb);
  double *cen = xmalloc(sizeof(double) * nb * dim);
  int *newladdr = xmalloc(sizeof(int) * 2 * (nl + 1));
  int b, ilev, k, cur;
  memcpy(lev, t->ilevel, sizeof(int) * nb);
  memcpy(par, t->iparent, sizeof(int) * nb);
  memcpy(nch, t->nchild, sizeof(int) * nb);
  memcpy(chi, t->ichild, sizeof(int) * nb * mc);
  memcpy(flg, t->iflag, sizeof(int) * nb);
  memcpy(cen, t->centers, sizeof(double) * nb * dim);
  memcpy(newladdr, t->laddr, sizeof(int) * 2 * (nl + 1));
  for (ilev = 0; ilev <= 1 && ilev <= nl; ilev++)
    for (b = t->laddr[2 * ilev]; b <= t->laddr[2 * ilev + 1]; b++) map[b] = b;
  cur = (nl >= 2) ? t->laddr[4] : 0;
  for (ilev = 2; ilev <= nl; ilev++) {
    int pass, f, l;
    newladdr[2 * ilev] = cur;
    for (pass = 0; pass < 2; pass++) {
      f = pass ? tail[2 * ilev] : t->laddr[2 * ilev];
      l = pass ? tail[2 * ilev + 1] : t->laddr[2 * ilev + 1];
      for (b = f; b <= l; b++) {
        t->ilevel[cur] = lev[b];
        t->nchild[cur] = nch[b];
        for (k = 0; k < dim; k++) t->centers[cur * dim + k] = cen[b * dim + k];
        t->iflag[cur] = flg[b];
        map[b] = cur;
        cur++;
      }
    }
    newladdr[2 * ilev + 1] = cur - 1;
  }
  for (b = 0; b < nb; b++) {
    int nbx = map[b];
    t->iparent[nbx] = (par[b] < 0) ? -1 : map[par[b]];
    for (k = 0; k < mc; k++)
      t->ichild[nbx * mc + k] = (chi[b * mc + k] < 0) ? -1 : map[chi[b * mc + k]];
  }
  memcpy(t->laddr, newladdr, sizeof(int) * 2 * (nl + 1));
  free(map); free(lev); free(par); free(nch); free(chi); free(flg); free(cen);
  free(newladdr);
}

/* pts_tree_fix_lr, pts_tree_nd.f:746-1058. */
static void fix_level_restriction(otree *t, int iperiod) {
  int dim = t->dim, mc = t->mc, mnb = t->mnbors, nl = t->nlevels;
  int *tail = xmalloc(sizeof(int) * 2 * (nl + 1));
  int b, i, k, ilev;
  for (b = 0; b < t->nboxes; b++) t->iflag[b] = 0;
  /* flag: leaf colleagues of the grandparent touching the parent */
  for (ilev = nl; ilev >= 2; ilev--) {
    double distest = 1.05 * (t->boxsize[ilev - 1] + t->boxsize[ilev - 2]) / 2.0;
    for (b = t->laddr[2 * ilev]; b <= t->laddr[2 * ilev + 1]; b++) {
      int dad = t->iparent[b], gd = t->iparent[dad];
      for (i = 0; i < t->nnbors[gd]; i++) {
        int jb = t->nbors[gd * mnb + i];
        if (t->nchild[jb] == 0 && t->iflag[jb] == 0) {
          int ict = 0;
          for (k = 0; k < dim; k++)
            if (fabs(t->centers[jb * dim + k] - t->centers[dad * dim + k]) <= distest)
              ict++;
          if (ict == dim) t->iflag[jb] = 1;
        }
      }
    }
  }
  /* flag+: leaf colleagues of the parent touching a flagged box */
  for (ilev = nl; ilev >= 1; ilev--) {
    double distest = 1.05 * (t->boxsize[ilev] + t->boxsize[ilev - 1]) / 2.0;
    for (b = t->laddr[2 * ilev]; b <= t->laddr[2 * ilev + 1]; b++) {
      if (t->iflag[b] != 1 && t->iflag[b] != 2) continue;
      int dad = t->iparent[b];
      for (i = 0; i < t->nnbors[dad]; i++) {
        int jb = t->nbors[dad * mnb + i];
        if (t->nchild[jb] == 0 && t->iflag[jb] == 0) {
          int ict = 0;
          for (k = 0; k < dim; k++)
            if (fabs(t->centers[jb * dim + k] - t->centers[b * dim + k]) <= distest)
              ict++;
          if (ict == dim) t->iflag[jb] = 2;
        }
      }
    }
  }
  for (ilev = 0; ilev <= nl; ilev++) { tail[2 * ilev] = 0; tail[2 * ilev + 1] = -1; }
  for (ilev = 1; ilev <= nl - 2; ilev++) {
    tail[2 * (ilev + 1)] = t->nboxes;
    int f = t->laddr[2 * ilev], nbloc = t->laddr[2 * ilev + 1] - f + 1;
    refine_flagged(t, f, nbloc, t->boxsize[ilev + 1], ilev);
    tail[2 * (ilev + 1) + 1] = t->nboxes - 1;
  }
  tree_reorg(t, tail);
  compute_colleagues(t, iperiod);
  /* flag++ processing */
  for (b = 0; b < t->nboxes; b++)
    if (t->iflag[b] != 3) t->iflag[b] = 0;
  for (ilev = 0; ilev <= nl; ilev++) { tail[2 * ilev] = 0; tail[2 * ilev + 1] = -1; }
  for (ilev = 2; ilev <= nl - 2; ilev++) {
    update_flags(t, ilev, t->laddr[2 * ilev], t->laddr[2 * ilev + 1]);
    update_flags(t, ilev, tail[2 * ilev], tail[2 * ilev + 1]);
    tail[2 * (ilev + 1)] = t->nboxes;
    int f = t->laddr[2 * ilev], nbloc = t->laddr[2 * ilev + 1] - f + 1;
    refine_flagged(t, f, nbloc, t->boxsize[ilev + 1], ilev);
    f = tail[2 * ilev];
    nbloc = tail[2 * ilev + 1] - f + 1;
    if (nbloc > 0) refine_flagged(t, f, nbloc, t->boxsize[ilev + 1], ilev);
    tail[2 * (ilev + 1) + 1] = t->nboxes - 1;
    /* colleagues of the new boxes (free-space test, pts_tree_nd.f:1003-1034) */
    double tol = f105() * t->boxsize[ilev + 1];
    for (b = tail[2 * (ilev + 1)]; b <= tail[2 * (ilev + 1) + 1]; b++) {
      int dad = t->iparent[b], j;
      t->nnbors[b] = 0;
      for (i = 0; i < t->nnbors[dad]; i++) {
        int jb = t->nbors[dad * mnb + i];
        for (j = 0; j < mc; j++) {
          int kb = t->ichild[jb * mc + j];
          if (kb < 0) continue;
          int ok = 1;
          for (k = 0; k < dim; k++)
            if (fabs(t->centers[kb * dim + k] - t->centers[b * dim + k]) > tol) { ok = 0; break; }
          if (ok) t->nbors[b * mnb + t->nnbors[b]++] = kb;
        }
      }
    }
  }
  tree_reorg(t, tail);
  compute_colleagues(t, iperiod);
  free(tail);
}

/* pts_tree_build (pts_tree_nd.f:393-644) with idivflag=0 (divide on
 * sources), nlmin=0, ifunif=0, followed by pts_tree_sort (:1226-1256) of
 * sources and targets on the final tree.  Output se arrays hold, per box,
 * first/last sorted index (inclusive). */
static void tree_build(otree *t, int dim, const double *src, int ns,
                       const double *trg, int nt, int ndiv, int nlmax,
                       int iperiod, double bs0, const double *cen0) {
  int k, ilev, b;
  memset(t, 0, sizeof(*t));
  t->dim = dim;
  t->mc = 1 << dim;
  t->mnbors = ipow(3, dim);
  tree_reserve(t, 1);
  t->boxsize = xmalloc(sizeof(double) * (nlmax + 1));
  t->laddr = xmalloc(sizeof(int) * 2 * (nlmax + 1));
  t->boxsize[0] = bs0;
  for (k = 0; k < dim; k++) t->centers[k] = cen0[k];
  t->laddr[0] = 0; t->laddr[1] = 0;
  t->ilevel[0] = 0; t->iparent[0] = -1; t->nchild[0] = 0;
  for (k = 0; k < t->mc; k++) t->ichild[k] = -1;
  t->iflag[0] = 0;
  t->nboxes = 1;
  int *isrc = xmalloc(sizeof(int) * (ns + 1)), *itrg = xmalloc(sizeof(int) * (nt + 1));
  int *tmp = xmalloc(sizeof(int) * ((ns > nt ? ns : nt) + 1));
  int *bin = xmalloc(sizeof(int) * ((ns > nt ? ns : nt) + 1));
  int secap = 1024;
  int *sse = xmalloc(sizeof(int) * 2 * secap), *tse = xmalloc(sizeof(int) * 2 * secap);
  for (k = 0; k < ns; k++) isrc[k] = k;
  for (k = 0; k < nt; k++) itrg[k] = k;
  sse[0] = 0; sse[1] = ns - 1; tse[0] = 0; tse[1] = nt - 1;
  for (ilev = 0; ilev < nlmax; ilev++) {
    int f = t->laddr[2 * ilev], l = t->laddr[2 * ilev + 1], any = 0;
    for (b = f; b <= l; b++)
      if (sse[2 * b + 1] - sse[2 * b] + 1 > ndiv) any = 1;
    if (!any) break;
    t->boxsize[ilev + 1] = t->boxsize[ilev] / 2;
    t->laddr[2 * (ilev + 1)] = t->nboxes;
    for (b = f; b <= l; b++) {
      if (sse[2 * b + 1] - sse[2 * b] + 1 > ndiv) {
        make_children(t, b, t->boxsize[ilev + 1], ilev + 1);
        if (t->nboxes > secap) {
          while (secap < t->nboxes) secap *= 2;
          sse = realloc(sse, sizeof(int) * 2 * secap);
          tse = realloc(tse, sizeof(int) * 2 * secap);
        }
        sort_to_children(t, b, src, ns, isrc, sse, tmp, bin);
        sort_to_children(t, b, trg, nt, itrg, tse, tmp, bin);
      }
    }
    t->laddr[2 * (ilev + 1) + 1] = t->nboxes - 1;
  }
  t->nlevels = ilev;
  compute_colleagues(t, iperiod);
  if (t->nlevels >= 2) fix_level_restriction(t, iperiod);
  free(isrc); free(itrg); free(tmp); free(bin); free(sse); free(tse);
}

/* pts_tree_sort, pts_tree_nd.f:1226-1256. */
static void tree_sort_points(const otree *t, const double *x, int n, int *iperm,
                             int *se) {
  int i, ilev, b;
  int *tmp = xmalloc(sizeof(int) * (n + 1)), *bin = xmalloc(sizeof(int) * (n + 1));
  for (i = 0; i < n; i++) iperm[i] = i;
  se[0] = 0;
  se[1] = n - 1;
  for (ilev = 0; ilev < t->nlevels; ilev++)
    for (b = t->laddr[2 * ilev]; b <= t->laddr[2 * ilev + 1]; b++)
      if (t->nchild[b] > 0) sort_to_children(t, b, x, n, iperm, se, tmp, bin);
  free(tmp);
  free(bin);
}

/* ------------------------------------------------------------------------ */
/* scalar set-up                                                            */
/* ------------------------------------------------------------------------ */

/* pts_tree_boxsize0, pts_tree_nd.f:1330-1414. */
static void boxsize0(int dim, double delta, double eps, int iperiod,
                     const double *src, int ns, const double *trg, int nt,
                     int *levcut, double *bs0, double *cen0) {
  int i, k;
  if (iperiod != 1) {
    double lo[MAXDIM], hi[MAXDIM];
    for (k = 0; k < dim; k++) lo[k] = hi[k] = src[k];
    for (i = 0; i < ns; i++)
      for (k = 0; k < dim; k++) {
        double v = src[(size_t)i * dim + k];
        if (v < lo[k]) lo[k] = v;
        if (v > hi[k]) hi[k] = v;
      }
    for (i = 0; i < nt; i++)
      for (k = 0; k < dim; k++) {
        double v = trg[(size_t)i * dim + k];
        if (v < lo[k]) lo[k] = v;
        if (v > hi[k]) hi[k] = v;
      }
    *bs0 = hi[0] - lo[0];
    for (k = 1; k < dim; k++)
      if (hi[k] - lo[k] > *bs0) *bs0 = hi[k] - lo[k];
    for (k = 0; k < dim; k++) cen0[k] = (lo[k] + hi[k]) / 2;
  }
  double dc = sqrt(delta * log(1.0 / eps));
  double dl = log(*bs0 / dc) / log(2.0);
  *levcut = (int)dl; /* Fortran int(): truncation toward zero */
  if (iperiod == 1) return;
  if (*bs0 < dc) return;
  *levcut = *levcut + 1;
  *bs0 = (double)ipow(2, *levcut) * dc;
}

/* fgtpwterms, fgtterms.f:72-141. */
static void pw_terms(double bsize, double delta, double eps, int iperiod,
                     double *pmax, int *npw) {
  double pi = 4.0 * atan(1.0);
  if (iperiod == 0) {
    double rmax = bsize / sqrt(delta);
    double d = sqrt(log(1.0 / eps));
    *pmax = 2.0 * d;
    double h = 2 * pi / (rmax + d);
    *npw = 2 * ((int)(*pmax / h) + 1);
  } else {
    *npw = 2 * ((int)(bsize * sqrt(log(1.0 / eps) / delta) / pi) + 1) + 1;
  }
}

/* get_pwnodes (itype=1, trapezoid), fgtterms.f:151-179; arrays hold
 * j = -npw/2 .. npw/2-1 at offset j+npw/2. */
static void pw_nodes(double pmax, int npw, double *ws, double *ts) {
  double pi = 4.0 * atan(1.0);
  int npw2 = npw / 2, j;
  double h = pmax / npw2, w = h / (2.0 * sqrt(pi));
  for (j = -npw2; j <= npw2 - 1; j++) {
    ts[j + npw2] = j * h;
    ws[j + npw2] = w * exp(-ts[j + npw2] * ts[j + npw2] / 4);
  }
}

/* get_periodic_pwnodes, fgtterms.f:191-211; j = -npw/2 .. (npw-1)/2. */
static void pw_nodes_periodic(double bsize0, double delta, int npw, double *ws,
                              double *ts) {
  double pi = 4.0 * atan(1.0);
  int npw2 = npw / 2, j;
  double h = 2 * pi / bsize0, w = sqrt(pi * delta) / bsize0, hw = h * sqrt(delta) / 2;
  for (j = -npw2; j <= (npw - 1) / 2; j++) {
    ts[j + npw2] = j * h;
    ws[j + npw2] = w * exp(-(hw * j) * (hw * j));
  }
}

/* ------------------------------------------------------------------------ */
/* direct kernels, pfgt_direct.f:47-615                                     */
/* ------------------------------------------------------------------------ */

/* One source/target pair of the gnd_direct{c,d,cd}{p,g,h} kernels
 * (pfgt_direct.f:47-615).  dr = t - s.  Output increments.
 *
 * One departure: with charges AND dipoles and ifpgh = 3, the reference's
 * gnd_directcdh (pfgt_direct.f:510-598) forms the dipole Hessian from
 * dg = (-2/delta) dr (the charge kernel's factor) in the formula written for
 * dg = (+2/delta) dr, so the signs of its rinc and rincg terms are flipped
 * and its dipole Hessian is not the Hessian of its dipole potential (the
 * finite-difference test in tests/test_oracle.py shows it).  Here the dipole
 * part always uses the gnd_directdh formulas (pfgt_direct.f:309-384), the
 * true Hessian, as the reference's own dipole-only kernel and its
 * plane-wave far field do. */
static void direct_pair(int nd, int dim, double delta, double dmax,
                        const double *dr, int ifcharge, const double *q,
                        int ifdipole, const double *rn, const double *ds,
                        int ifpgh, double *pot, double *grad, double *hess) {
  int k, j, m, ii, nhess = dim * (dim + 1) / 2;
  double rr = 0;
  for (k = 0; k < dim; k++) rr += dr[k] * dr[k];
  if (!(rr < dmax)) return;
  double e = exp(-rr / delta);
  if (ifcharge) {
    double rfac = -2.0 / delta, dg[MAXDIM], dh[6];
    for (k = 0; k < dim; k++) dg[k] = rfac * dr[k];
    if (ifpgh >= 3) {
      if (dim != 2) {
        for (k = 0; k < dim; k++) dh[k] = rfac + dg[k] * dg[k];
        m = dim;
        for (k = 0; k < dim - 1; k++)
          for (j = k + 1; j < dim; j++) dh[m++] = dg[k] * dg[j];
      } else {
        dh[0] = rfac + dg[0] * dg[0];
        dh[1] = dg[0] * dg[1];
        dh[2] = rfac + dg[1] * dg[1];
      }
    }
    for (ii = 0; ii < nd; ii++) {
      double r = e * q[ii];
      if (ifpgh >= 1) pot[ii] += r;
      if (ifpgh >= 2)
        for (k = 0; k < dim; k++) grad[k * nd + ii] += dg[k] * r;
      if (ifpgh >= 3)
        for (k = 0; k < nhess; k++) hess[k * nd + ii] += dh[k] * r;
    }
  }
  if (ifdipole) {
    /* formulas of gnd_directdh, pfgt_direct.f:309-384 (rfac = +2/delta) */
    double rfac = 2.0 / delta, d[MAXDIM], rinc = 0, rg[MAXDIM], rh[6];
    for (k = 0; k < dim; k++) d[k] = rfac * dr[k];
    for (k = 0; k < dim; k++) rinc += d[k] * rn[k];
    for (k = 0; k < dim; k++) rg[k] = rn[k] * rfac - rinc * d[k];
    if (ifpgh >= 3) {
      if (dim != 2) {
        for (k = 0; k < dim; k++) rh[k] = -rfac * (d[k] * rn[k] + rinc) - rg[k] * d[k];
        m = dim;
        for (k = 0; k < dim - 1; k++)
          for (j = k + 1; j < dim; j++) rh[m++] = -rfac * d[k] * rn[j] - rg[k] * d[j];
      } else {
        rh[0] = -rfac * (d[0] * rn[0] + rinc) - rg[0] * d[0];
        rh[1] = -rfac * d[0] * rn[1] - rg[0] * d[1];
        rh[2] = -rfac * (d[1] * rn[1] + rinc) - rg[1] * d[1];
      }
    }
    for (ii = 0; ii < nd; ii++) {
      double r = e * ds[ii];
      if (ifpgh >= 1) pot[ii] += rinc * r;
      if (ifpgh >= 2)
        for (k = 0; k < dim; k++) grad[k * nd + ii] += rg[k] * r;
      if (ifpgh >= 3)
        for (k = 0; k < nhess; k++) hess[k * nd + ii] += rh[k] * r;
    }
  }
}

/* pfgt_direct, pfgt.f:1156-1382: sources [is,ie] (sorted arrays, shifted by
 * `shift` when iperiod0 == 1) onto targets [js,je]. */
static void direct_block(int nd, int dim, double delta, double dmax,
                         const double *shift, int is, int ie, const double *src,
                         int ifcharge, const double *q, int ifdipole,
                         const double *rn, const double *ds, int js, int je,
                         const double *trg, int ifpgh, double *pot, double *grad,
                         double *hess) {
  int nhess = dim * (dim + 1) / 2, i, j, k;
  if (ifpgh <= 0) return;
  for (j = js; j <= je; j++) {
    for (i = is; i <= ie; i++) {
      double dr[MAXDIM];
      for (k = 0; k < dim; k++)
        dr[k] = trg[(size_t)j * dim + k] - (src[(size_t)i * dim + k] + (shift ? shift[k] : 0.0));
      direct_pair(nd, dim, delta, dmax, dr, ifcharge, q ? &q[(size_t)i * nd] : NULL,
                  ifdipole, rn ? &rn[(size_t)i * dim] : NULL,
                  ds ? &ds[(size_t)i * nd] : NULL, ifpgh, &pot[(size_t)j * nd],
                  grad ? &grad[(size_t)j * dim * nd] : NULL,
                  hess ? &hess[(size_t)j * nhess * nd] : NULL);
    }
  }
}

/* pfgt_find_local_shift, pfgt_direct.f:620-651. */
static void local_shift(int dim, const double *tc, const double *sc, double bs0,
                        double *shift) {
  int i;
  for (i = 0; i < dim; i++) {
    double dx = tc[i] - sc[i], dxp1 = dx - bs0, dxm1 = dx + bs0;
    shift[i] = 0;
    if (fabs(dx) > fabs(dxp1)) { dx = dxp1; shift[i] = bs0; }
    if (fabs(dx) > fabs(dxm1)) shift[i] = -bs0;
  }
}

/* ------------------------------------------------------------------------ */
/* plane-wave machinery (exact NUDFT in place of finufft)                   */
/* ------------------------------------------------------------------------ */

/* Mode index layout: x fastest, modes m_d = 0..npw-1 <-> j = m_d - npw/2. */

/* gnd_formpw, pfgt_nufftrouts.f:21-163, with the type-1 NUFFT
 * fk(k) = sum_j cj exp(-i k . xj) evaluated exactly. */
static void form_pw(int nd, int dim, double delta0, const double *src, int n,
                    int ifcharge, const double *q, int ifdipole, const double *rn,
                    const double *ds, const double *cen, double hpw, int npw,
                    const double *ws, const double *ts, zcplx *ffexp) {
  int nexp = ipow(npw, dim), j, k, id, m;
  double dsq0 = 1 / sqrt(delta0), dsq = hpw / sqrt(delta0);
  int npw2 = npw / 2;
  zcplx *e1 = xmalloc(sizeof(zcplx) * npw * dim);
  for (m = 0; m < nexp * nd; m++) ffexp[m] = 0;
  for (j = 0; j < n; j++) {
    for (k = 0; k < dim; k++) {
      double xj = (src[(size_t)j * dim + k] - cen[k]) * dsq;
      int mm;
      for (mm = 0; mm < npw; mm++) e1[k * npw + mm] = cexp(-I * (double)(mm - npw2) * xj);
    }
    for (m = 0; m < nexp; m++) {
      int r = m, mi[MAXDIM];
      zcplx ex = 1.0;
      double wsum = 1.0;
      for (k = 0; k < dim; k++) {
        mi[k] = r % npw;
        r /= npw;
        ex *= e1[k * npw + mi[k]];
        wsum *= ws[mi[k]];
      }
      for (id = 0; id < nd; id++) {
        zcplx c = 0;
        if (ifcharge) c += wsum * q[(size_t)j * nd + id];
        if (ifdipole) {
          zcplx z = -I * ds[(size_t)j * nd + id] * dsq0;
          for (k = 0; k < dim; k++) c += wsum * ts[mi[k]] * z * rn[(size_t)j * dim + k];
        }
        ffexp[(size_t)id * nexp + m] += c * ex;
      }
    }
  }
  free(e1);
}

/* gnd_pweval, pfgt_nufftrouts.f:169-327, type-2 NUFFT evaluated exactly.
 * quirk_scramble reproduces the nd>1 coefficient index bug (:252-258). */
static void eval_pw(int nd, int dim, double delta0, const double *cen, double hpw,
                    int npw, const double *ts, const zcplx *pwexp, const double *x,
                    int n, int ifpgh, double *pot, double *grad, double *hess,
                    int quirk_scramble) {
  int nexp = ipow(npw, dim), j, k, id, m, l, nhess = dim * (dim + 1) / 2;
  int kend = (ifpgh == 1) ? 0 : (ifpgh == 2 ? dim : dim + nhess);
  double dsq = hpw / sqrt(delta0);
  zcplx z = I / sqrt(delta0), z2 = z * z;
  int npw2 = npw / 2;
  /* coefficient sets fk[(c*nd+id)*nexp+m], c = 0 pot, 1..dim grad, rest hess */
  zcplx *fk = xcalloc((size_t)(kend + 1) * nd * nexp, sizeof(zcplx));
  /* potential coefficients first (pfgt_nufftrouts.f:252-256) */
  for (id = 0; id < nd; id++)
    for (m = 0; m < nexp; m++) {
      zcplx p = pwexp[(size_t)id * nexp + m];
      if (ifpgh >= 2 && quirk_scramble && nd > 1) {
        /* fk(j,0,ind) written into an fk(nexp,nd,0:kend) array lands at the
         * linear offset j - nexp + nexp*nd*ind (1-based j, ind); the slots
         * it never reaches are uninitialised in the reference (zero here). */
        long lin = (long)m - nexp + (long)nexp * nd * (id + 1);
        if (lin >= 0 && lin < (long)(kend + 1) * nd * nexp) fk[lin] = p;
      } else {
        fk[(size_t)id * nexp + m] = p;
      }
    }
  /* then gradient and hessian coefficients (:259-276) */
  for (id = 0; id < nd && ifpgh >= 2; id++)
    for (m = 0; m < nexp; m++) {
      int r = m, mi[MAXDIM];
      for (k = 0; k < dim; k++) { mi[k] = r % npw; r /= npw; }
      zcplx p = pwexp[(size_t)id * nexp + m];
      for (k = 0; k < dim; k++) fk[(size_t)((1 + k) * nd + id) * nexp + m] = p * ts[mi[k]] * z;
      if (ifpgh >= 3) {
        /* wnufftgh hessian weights, pfgt_nufftrouts.f:483-528 */
        double wh[6];
        if (dim == 1) wh[0] = ts[mi[0]] * ts[mi[0]];
        else if (dim == 2) {
          wh[0] = ts[mi[0]] * ts[mi[0]];
          wh[1] = ts[mi[0]] * ts[mi[1]];
          wh[2] = ts[mi[1]] * ts[mi[1]];
        } else {
          wh[0] = ts[mi[0]] * ts[mi[0]];
          wh[1] = ts[mi[1]] * ts[mi[1]];
          wh[2] = ts[mi[2]] * ts[mi[2]];
          wh[3] = ts[mi[0]] * ts[mi[1]];
          wh[4] = ts[mi[0]] * ts[mi[2]];
          wh[5] = ts[mi[1]] * ts[mi[2]];
        }
        for (k = 0; k < nhess; k++)
          fk[(size_t)((1 + dim + k) * nd + id) * nexp + m] = p * wh[k] * z2;
      }
    }
  zcplx *e1 = xmalloc(sizeof(zcplx) * npw * dim);
  for (j = 0; j < n; j++) {
    for (k = 0; k < dim; k++) {
      double xj = (x[(size_t)j * dim + k] - cen[k]) * dsq;
      int mm;
      for (mm = 0; mm < npw; mm++) e1[k * npw + mm] = cexp(I * (double)(mm - npw2) * xj);
    }
    for (l = 0; l <= kend; l++)
      for (id = 0; id < nd; id++) {
        zcplx acc = 0;
        const zcplx *f = &fk[(size_t)(l * nd + id) * nexp];
        for (m = 0; m < nexp; m++) {
          int r = m;
          zcplx ex = 1.0;
          for (k = 0; k < dim; k++) { ex *= e1[k * npw + r % npw]; r /= npw; }
          acc += f[m] * ex;
        }
        double v = creal(acc);
        if (l == 0) pot[(size_t)j * nd + id] += v;
        else if (l <= dim) grad[((size_t)j * dim + (l - 1)) * nd + id] += v;
        else hess[((size_t)j * nhess + (l - 1 - dim)) * nd + id] += v;
      }
  }
  free(e1);
  free(fk);
}

/* ------------------------------------------------------------------------ */
/* fast NUFFT (timed CPU baseline): exponential-of-semicircle spreading on  */
/* the sub-grid the box's points reach, separable DFT passes, FP64.         */
/* ------------------------------------------------------------------------ */

typedef struct {
  int npw, nf, w, G, l0, wrap;
  double dx, halfw, beta;
  double *phihat; /* modes j = -npw/2 .. npw/2-1 */
  zcplx *tw;      /* tw[l*npw + m] = exp(-i (m-npw/2) x_l), x_l = (l0+l) dx */
} fastnufft;

static void fast_setup(fastnufft *F, int npw, double eps, double xmax) {
  const double pi = 4.0 * atan(1.0);
  int w = (int)ceil(log10(1.0 / eps)) + 2, i, m, l;
  if (w < 4) w = 4;
  if (w > 16) w = 16;
  F->npw = npw;
  F->nf = 2 * (npw + 1);
  F->w = w;
  F->dx = 2 * pi / F->nf;
  F->halfw = w * F->dx / 2;
  F->beta = 0.97 * pi * 0.75 * w;
  xmax = xmax * (1 + 1e-6) + 1e-12;
  int lmin = (int)ceil((-xmax - F->halfw) / F->dx);
  int lmax = (int)ceil((xmax - F->halfw) / F->dx) + w - 1;
  F->l0 = lmin;
  F->G = lmax - lmin + 1;
  F->wrap = 0;
  if (F->G >= F->nf) { F->wrap = 1; F->G = F->nf; F->l0 = 0; }
  F->phihat = xmalloc(sizeof(double) * npw);
  /* midpoint quadrature of the kernel transform (smooth, compact) */
  const int nq = 400;
  for (m = 0; m < npw; m++) {
    double k = m - npw / 2, acc = 0;
    for (i = 0; i < nq; i++) {
      double z = -1 + (i + 0.5) * 2.0 / nq;
      acc += exp(F->beta * (sqrt(1 - z * z) - 1)) * cos(k * z * F->halfw);
    }
    F->phihat[m] = acc * F->halfw * 2.0 / nq;
  }
  F->tw = xmalloc(sizeof(zcplx) * F->G * npw);
  for (l = 0; l < F->G; l++)
    for (m = 0; m < npw; m++)
      F->tw[l * npw + m] = cexp(-I * (double)(m - npw / 2) * (F->l0 + l) * F->dx);
}
static void fast_free(fastnufft *F) { free(F->phihat); free(F->tw); }

/* cells and kernel values of one coordinate */
static void fast_row(const fastnufft *F, double x, int *idx, double *phi) {
  double u = x / F->dx;
  int i0 = (int)ceil(u - F->halfw / F->dx), j;
  for (j = 0; j < F->w; j++) {
    double z = ((i0 + j) - u) * F->dx / F->halfw, v = 1 - z * z;
    phi[j] = exp(F->beta * (sqrt(v > 0 ? v : 0) - 1));
    int c = i0 + j;
    if (F->wrap) { c %= F->nf; if (c < 0) c += F->nf; }
    else {
      c -= F->l0;
      if (c < 0) c = 0;
      if (c >= F->G) c = F->G - 1;
    }
    idx[j] = c;
  }
}

/* separable transform of a dim-D array along every axis: in[G..] -> out[npw..]
 * (forward, sign -) or out[G..] from in[npw..] (inverse, sign +). */
static void fast_dft(const fastnufft *F, int dim, const zcplx *in, zcplx *out, int inverse) {
  int G = F->G, P = F->npw, d, nin = inverse ? P : G, nout = inverse ? G : P;
  size_t tot = 1;
  for (d = 0; d < dim; d++) tot *= (size_t)(nin > nout ? nin : nout);
  zcplx *a = xcalloc(tot, sizeof(zcplx)), *b = xcalloc(tot, sizeof(zcplx));
  int ext[MAXDIM];
  for (d = 0; d < dim; d++) ext[d] = nin;
  size_t n0 = 1;
  for (d = 0; d < dim; d++) n0 *= nin;
  memcpy(a, in, sizeof(zcplx) * n0);
  for (d = 0; d < dim; d++) { /* transform axis d (axis 0 fastest) */
    size_t inner = 1, outer = 1, i, o, j;
    int k;
    for (k = 0; k < d; k++) inner *= ext[k];
    for (k = d + 1; k < dim; k++) outer *= ext[k];
    for (o = 0; o < outer; o++)
      for (i = 0; i < inner; i++)
        for (j = 0; j < (size_t)nout; j++) {
          zcplx acc = 0;
          int l;
          for (l = 0; l < nin; l++) {
            zcplx t = inverse ? conj(F->tw[(size_t)j * P + l]) : F->tw[(size_t)l * P + j];
            acc += a[(o * nin + l) * inner + i] * t;
          }
          b[(o * nout + j) * inner + i] = acc;
        }
    ext[d] = nout;
    zcplx *t = a; a = b; b = t;
  }
  size_t nres = 1;
  for (d = 0; d < dim; d++) nres *= nout;
  memcpy(out, a, sizeof(zcplx) * nres);
  free(a);
  free(b);
}

/* type-1 sums fk(k) = sum_j c_j exp(-i k.x_j), modes -npw/2..npw/2-1 (x fastest) */
static void fast_type1(const fastnufft *F, int dim, int n, const double *x /* scaled, n*dim */,
                       const double *c, zcplx *fk) {
  int G = F->G, P = F->npw, w = F->w, j, a, b2, e;
  size_t ng = 1, m, nexp = 1;
  int d;
  for (d = 0; d < dim; d++) { ng *= G; nexp *= P; }
  zcplx *g = xcalloc(ng, sizeof(zcplx));
  int idx[MAXDIM][16];
  double ph[MAXDIM][16];
  for (j = 0; j < n; j++) {
    for (d = 0; d < dim; d++) fast_row(F, x[(size_t)j * dim + d], idx[d], ph[d]);
    if (dim == 1) {
      for (a = 0; a < w; a++) g[idx[0][a]] += c[j] * ph[0][a];
    } else if (dim == 2) {
      for (b2 = 0; b2 < w; b2++)
        for (a = 0; a < w; a++) g[(size_t)idx[1][b2] * G + idx[0][a]] += c[j] * ph[0][a] * ph[1][b2];
    } else {
      for (e = 0; e < w; e++)
        for (b2 = 0; b2 < w; b2++)
          for (a = 0; a < w; a++)
            g[((size_t)idx[2][e] * G + idx[1][b2]) * G + idx[0][a]] +=
                c[j] * ph[0][a] * ph[1][b2] * ph[2][e];
    }
  }
  fast_dft(F, dim, g, fk, 0);
  for (m = 0; m < nexp; m++) {
    size_t r = m;
    double f = 1;
    for (d = 0; d < dim; d++) { f *= F->dx / F->phihat[r % P]; r /= P; }
    fk[m] *= f;
  }
  free(g);
}

/* type-2 values Re sum_k fk(k) exp(+i k.x_j) at n scaled points */
static void fast_type2(const fastnufft *F, int dim, const zcplx *fk, int n, const double *x,
                       double *out) {
  int G = F->G, P = F->npw, w = F->w, j, a, b2, e, d;
  size_t ng = 1, m, nexp = 1;
  for (d = 0; d < dim; d++) { ng *= G; nexp *= P; }
  zcplx *h = xmalloc(sizeof(zcplx) * nexp), *g = xmalloc(sizeof(zcplx) * ng);
  for (m = 0; m < nexp; m++) {
    size_t r = m;
    double f = 1;
    for (d = 0; d < dim; d++) { f *= F->dx / F->phihat[r % P]; r /= P; }
    h[m] = fk[m] * f;
  }
  fast_dft(F, dim, h, g, 1);
  int idx[MAXDIM][16];
  double ph[MAXDIM][16];
  for (j = 0; j < n; j++) {
    double acc = 0;
    for (d = 0; d < dim; d++) fast_row(F, x[(size_t)j * dim + d], idx[d], ph[d]);
    if (dim == 1) {
      for (a = 0; a < w; a++) acc += creal(g[idx[0][a]]) * ph[0][a];
    } else if (dim == 2) {
      for (b2 = 0; b2 < w; b2++)
        for (a = 0; a < w; a++) acc += creal(g[(size_t)idx[1][b2] * G + idx[0][a]]) * ph[0][a] * ph[1][b2];
    } else {
      for (e = 0; e < w; e++)
        for (b2 = 0; b2 < w; b2++)
          for (a = 0; a < w; a++)
            acc += creal(g[((size_t)idx[2][e] * G + idx[1][b2]) * G + idx[0][a]]) * ph[0][a] *
                   ph[1][b2] * ph[2][e];
    }
    out[j] = acc;
  }
  free(h);
  free(g);
}

/* gnd_formpw with the fast type-1 transform */
static void form_pw_fast(const fastnufft *F, int nd, int dim, double delta0, const double *src,
                         int n, int ifcharge, const double *q, int ifdipole, const double *rn,
                         const double *ds, const double *cen, double hpw, int npw,
                         const double *ws, const double *ts, zcplx *ffexp) {
  int nexp = ipow(npw, dim), j, k, id, m;
  double dsq = hpw / sqrt(delta0), dsq0 = 1 / sqrt(delta0);
  double *x = xmalloc(sizeof(double) * (size_t)n * dim + 8), *c = xmalloc(sizeof(double) * (n + 1));
  zcplx *fk = xmalloc(sizeof(zcplx) * nexp);
  for (j = 0; j < n; j++)
    for (k = 0; k < dim; k++) x[(size_t)j * dim + k] = (src[(size_t)j * dim + k] - cen[k]) * dsq;
  for (m = 0; m < nexp * nd; m++) ffexp[m] = 0;
  for (id = 0; id < nd; id++) {
    int comp;
    for (comp = 0; comp <= dim; comp++) {
      if (comp == 0 && !ifcharge) continue;
      if (comp > 0 && !ifdipole) break;
      for (j = 0; j < n; j++)
        c[j] = comp == 0 ? q[(size_t)j * nd + id]
                         : ds[(size_t)j * nd + id] * rn[(size_t)j * dim + comp - 1];
      fast_type1(F, dim, n, x, c, fk);
      for (m = 0; m < nexp; m++) {
        int r = m, mi[MAXDIM];
        double wsum = 1;
        for (k = 0; k < dim; k++) { mi[k] = r % npw; r /= npw; wsum *= ws[mi[k]]; }
        zcplx f = comp == 0 ? wsum : wsum * ts[mi[comp - 1]] * (-I * dsq0);
        ffexp[(size_t)id * nexp + m] += f * fk[m];
      }
    }
  }
  free(x); free(c); free(fk);
}

/* gnd_pweval with the fast type-2 transform (no quirks) */
static void eval_pw_fast(const fastnufft *F, int nd, int dim, double delta0, const double *cen,
                         double hpw, int npw, const double *ts, const zcplx *pwexp,
                         const double *xin, int n, int ifpgh, double *pot, double *grad,
                         double *hess) {
  int nexp = ipow(npw, dim), j, k, id, m, l, nhess = dim * (dim + 1) / 2;
  int kend = (ifpgh == 1) ? 0 : (ifpgh == 2 ? dim : dim + nhess);
  double dsq = hpw / sqrt(delta0), z = 1 / sqrt(delta0);
  double *x = xmalloc(sizeof(double) * (size_t)n * dim + 8), *v = xmalloc(sizeof(double) * (n + 1));
  zcplx *fk = xmalloc(sizeof(zcplx) * nexp);
  for (j = 0; j < n; j++)
    for (k = 0; k < dim; k++) x[(size_t)j * dim + k] = (xin[(size_t)j * dim + k] - cen[k]) * dsq;
  for (id = 0; id < nd; id++)
    for (l = 0; l <= kend; l++) {
      int pa = 0, pb = 0;
      if (l > dim) {
        int hm = l - 1 - dim;
        if (dim == 2) { pa = hm == 2 ? 1 : 0; pb = hm == 0 ? 0 : 1; }
        else if (dim == 3) { pa = hm < 3 ? hm : (hm < 5 ? 0 : 1); pb = hm < 3 ? hm : (hm == 3 ? 1 : 2); }
      }
      for (m = 0; m < nexp; m++) {
        int r = m, mi[MAXDIM];
        for (k = 0; k < dim; k++) { mi[k] = r % npw; r /= npw; }
        zcplx p = pwexp[(size_t)id * nexp + m];
        if (l == 0) fk[m] = p;
        else if (l <= dim) fk[m] = p * ts[mi[l - 1]] * (I * z);
        else fk[m] = -p * ts[mi[pa]] * ts[mi[pb]] * z * z;
      }
      fast_type2(F, dim, fk, n, x, v);
      for (j = 0; j < n; j++) {
        if (l == 0) pot[(size_t)j * nd + id] += v[j];
        else if (l <= dim) grad[((size_t)j * dim + (l - 1)) * nd + id] += v[j];
        else hess[((size_t)j * nhess + (l - 1 - dim)) * nd + id] += v[j];
      }
    }
  free(x); free(v); free(fk);
}

/* gnd_mk_full_translation_matrices, pfgt_nufftrouts.f:336-424 (nmax = 1):
 * W[s][m] = prod_d exp(i ts(m_d) xmin s_d), shift index s = sum_d
 * (s_d+1) 3^d with dimension 0 fastest (gnd_find_pwshift_ind order). */
static void shift_tables(int dim, double xmin, int npw, const double *ts, zcplx *W) {
  int nexp = ipow(npw, dim), ns = ipow(3, dim), s, m, k;
  for (s = 0; s < ns; s++)
    for (m = 0; m < nexp; m++) {
      int r = m, rs = s;
      zcplx w = 1.0;
      for (k = 0; k < dim; k++) {
        int mi = r % npw, si = rs % 3 - 1;
        r /= npw;
        rs /= 3;
        if (si != 0) w *= cexp(I * ts[mi] * xmin * (double)si);
      }
      W[(size_t)s * nexp + m] = w;
    }
}

/* Fortran nint(): round half away from zero. */
static int fnint(double x) { return (int)(x >= 0 ? floor(x + 0.5) : -floor(-x + 0.5)); }

/* gnd_find_pwshift_ind, bfgt_pwrouts.f:1592-1636 (nmax = 1), 0-based. */
static int shift_index(int dim, int iperiod, const double *tc, const double *sc,
                       double bs0, double xmin) {
  int i, ind = 0, inc = 1;
  for (i = 0; i < dim; i++) {
    int jx = fnint((tc[i] - sc[i]) / xmin);
    if (iperiod == 1) {
      int jxp1 = fnint((tc[i] - sc[i] - bs0) / xmin);
      int jxm1 = fnint((tc[i] - sc[i] + bs0) / xmin);
      if (abs(jx) > abs(jxp1)) jx = jxp1;
      if (abs(jx) > abs(jxm1)) jx = jxm1;
    }
    ind += (jx + 1) * inc;
    inc *= 3;
  }
  return ind;
}

/* ------------------------------------------------------------------------ */
/* lists                                                                    */
/* ------------------------------------------------------------------------ */

/* pfgt_find_pwexp_boxes, tree_routs_nd.f:1373-1460. */
static void find_pwexp_boxes(const otree *t, int npwlevel, int *ifpwexp) {
  int b, j;
  for (b = 0; b < t->nboxes; b++) ifpwexp[b] = 0;
  if (npwlevel <= 0) { ifpwexp[0] = 1; return; }
  if (npwlevel > t->nlevels) return;
  for (b = t->laddr[2 * npwlevel]; b <= t->laddr[2 * npwlevel + 1]; b++)
    for (j = 0; j < t->nnbors[b]; j++)
      if (t->nchild[t->nbors[b * t->mnbors + j]] > 0) { ifpwexp[b] = 1; break; }
}

typedef struct { int *n, *l, cap; } olist; /* l[b*cap + i] */

static void list_add(olist *L, int b, int v) {
  if (L->n[b] >= L->cap) {
    fprintf(stderr, "oracle: list overflow\n");
    abort();
  }
  L->l[(size_t)b * L->cap + L->n[b]++] = v;
}

/* pfgt_compute_listpw, tree_routs_nd.f:1487-1555. */
static void compute_listpw(const otree *t, int npwlevel, olist *L) {
  int b, i;
  for (b = 0; b < t->nboxes; b++) L->n[b] = 0;
  if (npwlevel > t->nlevels) return;
  int nc = npwlevel > 0 ? npwlevel : 0;
  for (b = t->laddr[2 * nc]; b <= t->laddr[2 * nc + 1]; b++)
    for (i = 0; i < t->nnbors[b]; i++) {
      int jb = t->nbors[b * t->mnbors + i];
      if (jb != b && t->nchild[b] > 0) list_add(L, jb, b);
    }
}

/* pfgt_compute_modified_list1, tree_routs_nd.f:1063-1257 (serial). */
static void compute_list1(const otree *t, int npwlevel, int iperiod, olist *L) {
  int dim = t->dim, mc = t->mc, mnb = t->mnbors;
  double bs0 = t->boxsize[0];
  int b, i, j, k, ilev;
  for (b = 0; b < t->nboxes; b++) L->n[b] = 0;
  if (t->nchild[0] == 0) list_add(L, 0, 0);
  int nlevend = t->nlevels;
  if (npwlevel < t->nlevels) nlevend = npwlevel;
  for (ilev = 1; ilev <= nlevend; ilev++) {
    for (b = t->laddr[2 * ilev]; b <= t->laddr[2 * ilev + 1]; b++) {
      if (t->nchild[b] != 0) continue;
      int dad = t->iparent[b];
      for (i = 0; i < t->nnbors[b]; i++) {
        int jb = t->nbors[b * mnb + i];
        if (t->nchild[jb] == 0 || ilev == npwlevel) {
          list_add(L, jb, b);
        } else if (ilev < npwlevel) {
          double distest = 1.05 * (t->boxsize[ilev] + t->boxsize[ilev + 1]) / 2.0;
          for (j = 0; j < mc; j++) {
            int kb = t->ichild[jb * mc + j];
            if (t->nchild[kb] != 0) continue;
            int ok = 1;
            for (k = 0; k < dim; k++) {
              double dis = fabs(t->centers[kb * dim + k] - t->centers[b * dim + k]);
              if (iperiod == 1) { double dp1 = bs0 - dis; if (dp1 < dis) dis = dp1; }
              if (dis >= distest) { ok = 0; break; }
            }
            if (ok) list_add(L, kb, b);
          }
        }
      }
      double distest = 1.05 * (t->boxsize[ilev] + t->boxsize[ilev - 1]) / 2.0;
      for (i = 0; i < t->nnbors[dad]; i++) {
        int jb = t->nbors[dad * mnb + i];
        if (t->nchild[jb] != 0) continue;
        int ok = 1;
        for (k = 0; k < dim; k++) {
          double dis = fabs(t->centers[jb * dim + k] - t->centers[b * dim + k]);
          if (iperiod == 1) { double dp1 = bs0 - dis; if (dp1 < dis) dis = dp1; }
          if (dis >= distest) { ok = 0; break; }
        }
        if (ok) list_add(L, jb, b);
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* exported: tree introspection                                             */
/* ------------------------------------------------------------------------ */

/* Result of a tree build, exposed to the tests through ctypes. */
typedef struct {
  int dim, nlevels, nboxes, npwlevel, ndiv;
  double bs0, cen0[MAXDIM];
  int *ilevel, *iparent, *nchild, *nnbors, *nbors, *laddr;
  double *centers, *boxsize;
  int *isrc, *isrcse, *itrg, *itrgse; /* se: first,last inclusive */
  int *ifpwexp, *nlistpw, *listpw, *nlist1, *list1;
  int mnbors, mlistpw, mlist1;
  int npw;
  double pmax;
} oracle_tree_t;

void oracle_tree_free(oracle_tree_t *r) {
  if (!r) return;
  free(r->ilevel); free(r->iparent); free(r->nchild); free(r->nnbors);
  free(r->nbors); free(r->laddr); free(r->centers); free(r->boxsize);
  free(r->isrc); free(r->isrcse); free(r->itrg); free(r->itrgse);
  free(r->ifpwexp); free(r->nlistpw); free(r->listpw); free(r->nlist1);
  free(r->list1);
  free(r);
}

static int ndiv_for_dim(int dim) { return dim == 1 ? 20 : (dim == 2 ? 80 : 250); }

/* Fixed root box in free space (>= 0): bs0/cen0 are inputs and the cut-off
 * level is this value, as a shard of a larger point set uses the geometry
 * pts_tree_boxsize0 computed on the whole set.  -1: the reference's own
 * computation from the points. */
static int g_root_level = -1;
void oracle_set_root_level(int level) { g_root_level = level; }

/* Build the tree and lists exactly as pfgt/pfgtmain do (pfgt.f:110-200,
 * 611-674) and return them.  bs0/cen0 are inputs when iperiod == 1. */
oracle_tree_t *oracle_tree_build(int dim, double delta, double eps, int iperiod,
                                 double bs0_in, const double *cen0_in, int ns,
                                 const double *src, int nt, const double *trg,
                                 int ndiv_override) {
  oracle_tree_t *r = xcalloc(1, sizeof(oracle_tree_t));
  otree t;
  int k, b;
  double bs0 = bs0_in, cen0[MAXDIM] = {0, 0, 0};
  for (k = 0; k < dim; k++) cen0[k] = cen0_in ? cen0_in[k] : 0.0;
  int npwlevel;
  if (g_root_level >= 0 && iperiod != 1)
    npwlevel = g_root_level;
  else
    boxsize0(dim, delta, eps, iperiod, src, ns, trg, nt, &npwlevel, &bs0, cen0);
  int ndiv = ndiv_override > 0 ? ndiv_override : ndiv_for_dim(dim);
  int nlmax = npwlevel >= 0 ? npwlevel + 1 : 0;
  tree_build(&t, dim, src, ns, trg, nt, ndiv, nlmax, iperiod, bs0, cen0);
  r->dim = dim; r->nlevels = t.nlevels; r->nboxes = t.nboxes;
  r->npwlevel = npwlevel; r->ndiv = ndiv; r->bs0 = bs0;
  for (k = 0; k < dim; k++) r->cen0[k] = cen0[k];
  r->mnbors = t.mnbors;
  int nb = t.nboxes;
  r->isrc = xmalloc(sizeof(int) * (ns + 1));
  r->itrg = xmalloc(sizeof(int) * (nt + 1));
  r->isrcse = xmalloc(sizeof(int) * 2 * nb);
  r->itrgse = xmalloc(sizeof(int) * 2 * nb);
  tree_sort_points(&t, src, ns, r->isrc, r->isrcse);
  tree_sort_points(&t, trg, nt, r->itrg, r->itrgse);
  /* npw, pfgt.f:321-334 */
  int npw = 0;
  double pmax = 0;
  if (npwlevel <= t.nlevels) {
    if (npwlevel <= 1) {
      double bsize = 2 * t.boxsize[npwlevel > 0 ? npwlevel : 0];
      pw_terms(bsize, delta, eps, iperiod, &pmax, &npw);
      if (iperiod == 1) npw = npw + 1;
    } else {
      pw_terms(2 * t.boxsize[npwlevel], delta, eps, 0, &pmax, &npw);
    }
  }
  if (npw < 4) npw = 4;
  r->npw = npw; r->pmax = pmax;
  /* lists with the colleague fix-up of pfgt.f:620-628 */
  int iperiod0 = iperiod;
  if (npwlevel <= 1 && iperiod == 1) {
    iperiod0 = 0;
    compute_colleagues(&t, 0);
  }
  r->ifpwexp = xmalloc(sizeof(int) * nb);
  find_pwexp_boxes(&t, npwlevel, r->ifpwexp);
  olist Lpw = {xmalloc(sizeof(int) * nb), NULL, t.mnbors - 1};
  Lpw.l = xmalloc(sizeof(int) * nb * (size_t)(Lpw.cap > 0 ? Lpw.cap : 1));
  compute_listpw(&t, npwlevel, &Lpw);
  int cap1 = 8 * t.mnbors + 8;
  olist L1 = {xmalloc(sizeof(int) * nb), xmalloc(sizeof(int) * (size_t)nb * cap1), cap1};
  compute_list1(&t, npwlevel, iperiod0, &L1);
  r->nlistpw = Lpw.n; r->listpw = Lpw.l; r->mlistpw = Lpw.cap;
  r->nlist1 = L1.n; r->list1 = L1.l; r->mlist1 = L1.cap;
  r->ilevel = xmalloc(sizeof(int) * nb);
  r->iparent = xmalloc(sizeof(int) * nb);
  r->nchild = xmalloc(sizeof(int) * nb);
  r->nnbors = xmalloc(sizeof(int) * nb);
  r->nbors = xmalloc(sizeof(int) * nb * t.mnbors);
  r->centers = xmalloc(sizeof(double) * nb * dim);
  r->laddr = xmalloc(sizeof(int) * 2 * (t.nlevels + 1));
  r->boxsize = xmalloc(sizeof(double) * (t.nlevels + 1));
  memcpy(r->ilevel, t.ilevel, sizeof(int) * nb);
  memcpy(r->iparent, t.iparent, sizeof(int) * nb);
  memcpy(r->nchild, t.nchild, sizeof(int) * nb);
  memcpy(r->nnbors, t.nnbors, sizeof(int) * nb);
  memcpy(r->nbors, t.nbors, sizeof(int) * nb * t.mnbors);
  memcpy(r->centers, t.centers, sizeof(double) * nb * dim);
  memcpy(r->laddr, t.laddr, sizeof(int) * 2 * (t.nlevels + 1));
  memcpy(r->boxsize, t.boxsize, sizeof(double) * (t.nlevels + 1));
  (void)b;
  tree_free(&t);
  return r;
}

/* ------------------------------------------------------------------------ */
/* exported: full pfgt                                                      */
/* ------------------------------------------------------------------------ */

/* Restatement of pfgt (pfgt.f:6-409) + pfgtmain (pfgt.f:415-1150).
 * Returns 0.  Output arrays are overwritten for the requested fields only. */
int oracle_pfgt(int nd, int dim, double delta, double eps, int iperiod,
                double *bs0_io, double *cen0_io, int ns, const double *sources,
                int ifcharge, const double *charge, int ifdipole,
                const double *rnormal, const double *dipstr, int ifpgh,
                double *pot, double *grad, double *hess, int nt,
                const double *targ, int ifpghtarg, double *pottarg,
                double *gradtarg, double *hesstarg, int quirks, int nufft_mode) {
  int k, i, b, id, nhess = dim * (dim + 1) / 2;
  double cen0[MAXDIM] = {0, 0, 0};
  for (k = 0; k < dim; k++) cen0[k] = cen0_io[k];
  oracle_tree_t *r = oracle_tree_build(dim, delta, eps, iperiod, *bs0_io, cen0, ns,
                                       sources, nt, targ, 0);
  *bs0_io = r->bs0;
  for (k = 0; k < dim; k++) cen0_io[k] = r->cen0[k];
  int npwlevel = r->npwlevel, nlevels = r->nlevels, npw = r->npw;
  int ndiv = r->ndiv, nb = r->nboxes;
  double bs0 = r->boxsize[0];
  /* sorted copies, dreorderf fmmcommon2d.f:3-27 */
  double *ss = xmalloc(sizeof(double) * (size_t)ns * dim + 8);
  double *ts_ = xmalloc(sizeof(double) * (size_t)nt * dim + 8);
  double *qs = ifcharge ? xmalloc(sizeof(double) * (size_t)ns * nd + 8) : NULL;
  double *dss = ifdipole ? xmalloc(sizeof(double) * (size_t)ns * nd + 8) : NULL;
  double *rns = ifdipole ? xmalloc(sizeof(double) * (size_t)ns * dim + 8) : NULL;
  for (i = 0; i < ns; i++) {
    int o = r->isrc[i];
    for (k = 0; k < dim; k++) ss[(size_t)i * dim + k] = sources[(size_t)o * dim + k];
    for (id = 0; id < nd; id++) {
      if (ifcharge) qs[(size_t)i * nd + id] = charge[(size_t)o * nd + id];
      if (ifdipole) dss[(size_t)i * nd + id] = dipstr[(size_t)o * nd + id];
    }
    if (ifdipole)
      for (k = 0; k < dim; k++) rns[(size_t)i * dim + k] = rnormal[(size_t)o * dim + k];
  }
  for (i = 0; i < nt; i++) {
    int o = r->itrg[i];
    for (k = 0; k < dim; k++) ts_[(size_t)i * dim + k] = targ[(size_t)o * dim + k];
  }
  double *ps = xcalloc((size_t)ns * nd + 1, sizeof(double));
  double *gs = xcalloc((size_t)ns * nd * dim + 1, sizeof(double));
  double *hs = xcalloc((size_t)ns * nd * nhess + 1, sizeof(double));
  double *pt = xcalloc((size_t)nt * nd + 1, sizeof(double));
  double *gt = xcalloc((size_t)nt * nd * dim + 1, sizeof(double));
  double *ht = xcalloc((size_t)nt * nd * nhess + 1, sizeof(double));

  /* pfgtmain set-up, pfgt.f:611-636 */
  int ncutoff = npwlevel > 0 ? npwlevel : 0;
  double *ws = xmalloc(sizeof(double) * (npw + 1)), *tsn = xmalloc(sizeof(double) * (npw + 1));
  int iperiod0 = iperiod;
  double delta0 = delta;
  if (npwlevel <= 1 && iperiod == 1) {
    pw_nodes_periodic(bs0, delta, npw, ws, tsn);
    iperiod0 = 0;
    delta0 = 1.0;
  } else {
    pw_nodes(r->pmax, npw, ws, tsn);
  }
  double hpw = tsn[npw / 2 + 1];
  int nlevend = nlevels;
  if (npwlevel <= nlevels) nlevend = npwlevel;
  int do_pw = npwlevel < nlevels;
  /* A root smaller than half the cut-off with ns <= ndiv forms no expansion
   * and the reference returns zeros (pfgt.f:649-650, 779); unless that quirk
   * is requested, compute its direct self interaction. */
  if (!(quirks & 4) && npwlevel < 0 && ns <= ndiv) {
    do_pw = 0;
    nlevend = 0;
    r->nlist1[0] = 1;
    r->list1[0] = 0;
  }
  fastnufft FN;
  if (nufft_mode == 1 && do_pw) {
    double xmax = (r->boxsize[ncutoff] / 2) * hpw / sqrt(delta0);
    fast_setup(&FN, npw, eps, xmax);
  }

  if (do_pw) {
    int nexp = ipow(npw, dim);
    int nshift = ipow(3, dim);
    zcplx *W = xmalloc(sizeof(zcplx) * (size_t)nexp * nshift);
    shift_tables(dim, r->boxsize[ncutoff] / sqrt(delta0), npw, tsn, W);
    double xmin = r->boxsize[ncutoff];
    zcplx **mp = xcalloc(nb, sizeof(zcplx *)), **loc = xcalloc(nb, sizeof(zcplx *));
    int f = r->laddr[2 * ncutoff], l = r->laddr[2 * ncutoff + 1];
    for (b = f; b <= l; b++)
      if (r->ifpwexp[b]) {
        mp[b] = xcalloc((size_t)nexp * nd, sizeof(zcplx));
        loc[b] = xcalloc((size_t)nexp * nd, sizeof(zcplx));
      }
    /* step 1: form, pfgt.f:764-798 */
#pragma omp parallel for schedule(dynamic)
    for (b = f; b <= l; b++) {
      int is = r->isrcse[2 * b], npts = r->isrcse[2 * b + 1] - is + 1;
      if (npts > ndiv && nufft_mode == 1) {
        form_pw_fast(&FN, nd, dim, delta0, &ss[(size_t)is * dim], npts, ifcharge,
                     ifcharge ? &qs[(size_t)is * nd] : NULL, ifdipole,
                     ifdipole ? &rns[(size_t)is * dim] : NULL,
                     ifdipole ? &dss[(size_t)is * nd] : NULL, &r->centers[b * dim], hpw,
                     npw, ws, tsn, mp[b]);
        memcpy(loc[b], mp[b], sizeof(zcplx) * (size_t)nexp * nd);
      } else if (npts > ndiv) {
        form_pw(nd, dim, delta0, &ss[(size_t)is * dim], npts, ifcharge,
                ifcharge ? &qs[(size_t)is * nd] : NULL, ifdipole,
                ifdipole ? &rns[(size_t)is * dim] : NULL,
                ifdipole ? &dss[(size_t)is * nd] : NULL, &r->centers[b * dim], hpw,
                npw, ws, tsn, mp[b]);
        memcpy(loc[b], mp[b], sizeof(zcplx) * (size_t)nexp * nd);
      }
    }
    /* step 2: mp -> loc, pfgt.f:818-835 */
#pragma omp parallel for schedule(dynamic) private(i)
    for (b = f; b <= l; b++)
      for (i = 0; i < r->nlistpw[b]; i++) {
        int jb = r->listpw[(size_t)b * r->mlistpw + i];
        int ind = shift_index(dim, iperiod0, &r->centers[b * dim], &r->centers[jb * dim],
                              bs0, xmin);
        size_t m;
        for (m = 0; m < (size_t)nexp * nd; m++)
          loc[b][m] += mp[jb][m] * W[(size_t)ind * nexp + m % nexp];
      }
    /* step 3: eval, pfgt.f:880-1062 */
#pragma omp parallel for schedule(dynamic)
    for (b = f; b <= l; b++) {
      if (!r->ifpwexp[b]) continue;
      int its = r->itrgse[2 * b], nts = r->itrgse[2 * b + 1] - its + 1;
      int iss = r->isrcse[2 * b], nss = r->isrcse[2 * b + 1] - iss + 1;
      int do_t = 1, do_s = 1;
      if ((quirks & 1) && ifpgh == ifpghtarg) {
        /* multi-threaded branch of pfgt.f:938-958 */
        do_t = (nts > 0 && nss == 0);
        do_s = (nss > 0 && nts == 0);
      }
      if (nufft_mode == 1 && !(quirks & 2)) {
        if (do_t && nts > 0 && ifpghtarg > 0)
          eval_pw_fast(&FN, nd, dim, delta0, &r->centers[b * dim], hpw, npw, tsn, loc[b],
                       &ts_[(size_t)its * dim], nts, ifpghtarg, &pt[(size_t)its * nd],
                       &gt[(size_t)its * nd * dim], &ht[(size_t)its * nd * nhess]);
        if (do_s && nss > 0 && ifpgh > 0)
          eval_pw_fast(&FN, nd, dim, delta0, &r->centers[b * dim], hpw, npw, tsn, loc[b],
                       &ss[(size_t)iss * dim], nss, ifpgh, &ps[(size_t)iss * nd],
                       &gs[(size_t)iss * nd * dim], &hs[(size_t)iss * nd * nhess]);
        continue;
      }
      if (do_t && nts > 0 && ifpghtarg > 0)
        eval_pw(nd, dim, delta0, &r->centers[b * dim], hpw, npw, tsn, loc[b],
                &ts_[(size_t)its * dim], nts, ifpghtarg, &pt[(size_t)its * nd],
                &gt[(size_t)its * nd * dim], &ht[(size_t)its * nd * nhess], quirks & 2);
      if (do_s && nss > 0 && ifpgh > 0)
        eval_pw(nd, dim, delta0, &r->centers[b * dim], hpw, npw, tsn, loc[b],
                &ss[(size_t)iss * dim], nss, ifpgh, &ps[(size_t)iss * nd],
                &gs[(size_t)iss * nd * dim], &hs[(size_t)iss * nd * nhess], quirks & 2);
    }
    for (b = 0; b < nb; b++) { free(mp[b]); free(loc[b]); }
    free(mp); free(loc); free(W);
    if (nufft_mode == 1) fast_free(&FN);
  }
  /* step 4: direct, pfgt.f:1082-1136 */
  double dmax = log(1.0 / eps) * delta;
  int ilev;
  for (ilev = 0; ilev <= nlevend; ilev++) {
#pragma omp parallel for schedule(dynamic) private(i)
    for (b = r->laddr[2 * ilev]; b <= r->laddr[2 * ilev + 1]; b++) {
      int jss = r->isrcse[2 * b], jse = r->isrcse[2 * b + 1];
      int jts = r->itrgse[2 * b], jte = r->itrgse[2 * b + 1];
      int nps = jse - jss + 1, npt = jte - jts + 1;
      if (nps + npt <= 0) continue;
      for (i = 0; i < r->nlist1[b]; i++) {
        int ib = r->list1[(size_t)b * r->mlist1 + i];
        double shift[MAXDIM] = {0, 0, 0};
        if (iperiod0 == 1)
          local_shift(dim, &r->centers[b * dim], &r->centers[ib * dim], bs0, shift);
        int is = r->isrcse[2 * ib], ie = r->isrcse[2 * ib + 1];
        if (npt > 0)
          direct_block(nd, dim, delta, dmax, iperiod0 == 1 ? shift : NULL, is, ie, ss,
                       ifcharge, qs, ifdipole, rns, dss, jts, jte, ts_, ifpghtarg, pt, gt,
                       ht);
        if (nps > 0)
          direct_block(nd, dim, delta, dmax, iperiod0 == 1 ? shift : NULL, is, ie, ss,
                       ifcharge, qs, ifdipole, rns, dss, jss, jse, ss, ifpgh, ps, gs, hs);
      }
    }
  }
  /* unsort, dreorderi/dreorderiv fmmcommon2d.f:29-90 */
  for (i = 0; i < ns; i++) {
    int o = r->isrc[i];
    if (ifpgh >= 1)
      for (id = 0; id < nd; id++) pot[(size_t)o * nd + id] = ps[(size_t)i * nd + id];
    if (ifpgh >= 2)
      for (k = 0; k < dim * nd; k++) grad[(size_t)o * dim * nd + k] = gs[(size_t)i * dim * nd + k];
    if (ifpgh >= 3)
      for (k = 0; k < nhess * nd; k++)
        hess[(size_t)o * nhess * nd + k] = hs[(size_t)i * nhess * nd + k];
  }
  for (i = 0; i < nt; i++) {
    int o = r->itrg[i];
    if (ifpghtarg >= 1)
      for (id = 0; id < nd; id++) pottarg[(size_t)o * nd + id] = pt[(size_t)i * nd + id];
    if (ifpghtarg >= 2)
      for (k = 0; k < dim * nd; k++)
        gradtarg[(size_t)o * dim * nd + k] = gt[(size_t)i * dim * nd + k];
    if (ifpghtarg >= 3)
      for (k = 0; k < nhess * nd; k++)
        hesstarg[(size_t)o * nhess * nd + k] = ht[(size_t)i * nhess * nd + k];
  }
  free(ss); free(ts_); free(qs); free(dss); free(rns);
  free(ps); free(gs); free(hs); free(pt); free(gt); free(ht); free(ws); free(tsn);
  oracle_tree_free(r);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* exported: exact FP64 direct sum                                          */
/* ------------------------------------------------------------------------ */

/* Exact Gauss transform at `nt` evaluation points: sum over all sources
 * (self included) of the pfgt_direct.f kernels without truncation; periodic:
 * images |n_d| <= nimg of period bs0 in every dimension. */
void oracle_direct_exact(int nd, int dim, double delta, int iperiod, double bs0,
                         int nimg, int ns, const double *src, int ifcharge,
                         const double *charge, int ifdipole, const double *rnormal,
                         const double *dipstr, int nt, const double *targ, int ifpgh,
                         double *pot, double *grad, double *hess) {
  int nhess = dim * (dim + 1) / 2, j;
  int ni = iperiod ? nimg : 0, span = 2 * ni + 1, nimgs = ipow(span, dim);
  memset(pot, 0, sizeof(double) * (size_t)nt * nd);
  if (ifpgh >= 2) memset(grad, 0, sizeof(double) * (size_t)nt * nd * dim);
  if (ifpgh >= 3) memset(hess, 0, sizeof(double) * (size_t)nt * nd * nhess);
  /* evaluation points are independent (each writes its own outputs) */
#pragma omp parallel for schedule(dynamic, 1)
  for (j = 0; j < nt; j++)
    for (int i = 0; i < ns; i++) {
      int im, k;
      for (im = 0; im < nimgs; im++) {
        double dr[MAXDIM];
        int r = im;
        for (k = 0; k < dim; k++) {
          int o = r % span - ni;
          r /= span;
          dr[k] = targ[(size_t)j * dim + k] - (src[(size_t)i * dim + k] + o * bs0);
        }
        direct_pair(nd, dim, delta, INFINITY, dr, ifcharge,
                    ifcharge ? &charge[(size_t)i * nd] : NULL, ifdipole,
                    ifdipole ? &rnormal[(size_t)i * dim] : NULL,
                    ifdipole ? &dipstr[(size_t)i * nd] : NULL, ifpgh,
                    &pot[(size_t)j * nd], ifpgh >= 2 ? &grad[(size_t)j * dim * nd] : NULL,
                    ifpgh >= 3 ? &hess[(size_t)j * nhess * nd] : NULL);
      }
    }
}

/* Truncated direct sum of the reference's pfgt_direct (pfgt.f:1156-1382)
 * over all source/target pairs, free space, cut-off rr < dmax. */
void oracle_direct_truncated(int nd, int dim, double delta, double dmax, int ns,
                             const double *src, int ifcharge, const double *charge,
                             int ifdipole, const double *rnormal, const double *dipstr,
                             int nt, const double *targ, int ifpgh, double *pot,
                             double *grad, double *hess) {
  int nhess = dim * (dim + 1) / 2;
  memset(pot, 0, sizeof(double) * (size_t)nt * nd);
  if (ifpgh >= 2) memset(grad, 0, sizeof(double) * (size_t)nt * nd * dim);
  if (ifpgh >= 3) memset(hess, 0, sizeof(double) * (size_t)nt * nd * nhess);
  direct_block(nd, dim, delta, dmax, NULL, 0, ns - 1, src, ifcharge, charge, ifdipole,
               rnormal, dipstr, 0, nt - 1, targ, ifpgh, pot, grad, hess);
}

#ifdef _OPENMP
#include <omp.h>
int oracle_threads(void) { return omp_get_max_threads(); }
#else
int oracle_threads(void) { return 1; }
#endif

/* Scalar set-up only (pts_tree_boxsize0 + fgtpwterms) for host-logic tests. */
void oracle_setup_scalars(int dim, double delta, double eps, int iperiod,
                          int ns, const double *src, int nt, const double *trg,
                          int *levcut, double *bs0, double *cen0) {
  boxsize0(dim, delta, eps, iperiod, src, ns, trg, nt, levcut, bs0, cen0);
}

void oracle_pwterms(double bsize, double delta, double eps, int iperiod,
                    double *pmax, int *npw) {
  pw_terms(bsize, delta, eps, iperiod, pmax, npw);
}
