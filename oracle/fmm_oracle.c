/*
 * fmm_oracle.c -- CPU restatement of the reference's fast marching method
 * for the signed distance function (test infrastructure only: the tests and
 * bench.py's CPU leg call it to check and time the GPU distance solver).
 *
 * It follows, step by step:
 *   - computeDistanceFunction3d -> computeExtensionFields3d with no fields
 *     (src/serial/lsm_FMM_field_extension.c:203-395): every value starts at
 *     -1, points with mask < 0 are OUTSIDE_DOMAIN and hold LSMLIB_REAL_MAX;
 *   - the first-order front initialisation, used at both orders
 *     (:397-668): a point on the zero level set (|phi| < 1e-11) gets
 *     +-1e-11, a point whose neighbour along an axis has phi of the other
 *     sign (or zero) gets +-sqrt(1 / sum_axes 1/d_axis^2) with d_axis the
 *     nearer linear-interpolated crossing; both become KNOWN;
 *   - FMM_Core_initializeFront (src/toolbox/fast_marching_method/
 *     FMM_Core.c:176-246): the front points, in a heap keyed on their signed
 *     values, are popped in order and each updates its non-KNOWN neighbours;
 *   - FMM_Core_advanceFront / FMM_Core_updateNeighbors (FMM_Core.c:321-451):
 *     the TRIAL point of smallest |d| becomes KNOWN and recomputes the trial
 *     value of each non-KNOWN neighbour (x-, x+, y-, y+, z-, z+);
 *   - the trial update (lsm_FMM_field_extension.c:966-1176 first order,
 *     :1180-1400 second order): per axis the KNOWN neighbour of smaller |d|
 *     (minus first, plus when strictly smaller), at second order with the
 *     next point in that direction when KNOWN and not larger in |d|; the
 *     upwind quadratic with coefficients accumulated over x, y, z; a
 *     negative discriminant keeps the current value;
 *   - extension fields (computeExtensionFields3d, :203-370): at the front
 *     the source fields interpolated linearly to the crossing along each
 *     axis (or taken from one side where extension_mask < 0) and averaged
 *     with weights 1/d_axis^2 (:524-660); at every trial update the weighted
 *     average over the axes in the update of the upwind neighbour's field,
 *     weights (dist - phi_upwind)/dx^2 (first order, :1135-1168) or
 *     (1.5 dist - 2 phi_upwind1 + 0.5 phi_upwind2)/dx^2 where the
 *     second-order stencil is used (:1400-1460);
 *   - the Eikonal solver (solveEikonalEquation3d, lsm_FMM_eikonal.c:140-652):
 *     points with mask < 0 or speed < 1e-11 are outside (LSMLIB_REAL_MAX),
 *     points with phi > -1e-11 are the KNOWN front with their own values,
 *     the update's constant term is 1/speed^2 and its root always
 *     0.5 (-B + sqrt(disc)) / A; points never updated keep their input;
 *   - the binary heap of FMM_Heap.c:118-470 (insert with sift-up, extract
 *     moving the last node into the root's slot and sifting down, update
 *     sifting up when below the parent and down otherwise), with the same
 *     comparisons so that ties are broken the same way.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>

typedef double real;

#define ZERO_TOL 1.0e-11
#define REAL_MAX DBL_MAX

enum { FAR = 0, TRIAL = 1, KNOWN = 2, OUTSIDE = 3 };

/* ---- indexed binary heap (FMM_Heap.c) --------------------------------- */
typedef struct {
  long idx;   /* linear grid index */
  real value;
  int pos;    /* position in the heap order */
} hnode;

/* Acceptance time of a point in the ordered march (below): lexicographic
 * (a, b, c). */
typedef struct {
  real a, b, c;
} time3;

typedef struct {
  hnode *nodes; /* by handle */
  int *heap;    /* position -> handle */
  int size, cap;
  const time3 *tm; /* NULL: keyed on the value, as the reference's heap;
                      else keyed on (tm[idx], idx), a total order */
} fheap;

static int t3_less(const time3 *x, const time3 *y) {
  return x->a < y->a || (x->a == y->a && (x->b < y->b || (x->b == y->b && x->c < y->c)));
}

/* node of handle ha before node of handle hb */
static int h_less(const fheap *h, int ha, int hb) {
  const hnode *x = &h->nodes[ha], *y = &h->nodes[hb];
  if (!h->tm) return x->value < y->value;
  const time3 *tx = &h->tm[x->idx], *ty = &h->tm[y->idx];
  if (t3_less(tx, ty)) return 1;
  if (t3_less(ty, tx)) return 0;
  return x->idx < y->idx;
}

static void h_init(fheap *h, int cap) {
  h->cap = cap > 16 ? cap : 16;
  h->size = 0;
  h->nodes = (hnode *)malloc(sizeof(hnode) * h->cap);
  h->heap = (int *)malloc(sizeof(int) * h->cap);
  h->tm = NULL;
}

static void h_free(fheap *h) {
  free(h->nodes);
  free(h->heap);
}

static void h_grow(fheap *h) {
  h->cap *= 2;
  h->nodes = (hnode *)realloc(h->nodes, sizeof(hnode) * h->cap);
  h->heap = (int *)realloc(h->heap, sizeof(int) * h->cap);
}

static inline int parent_pos(int p) { return (p + 1) / 2 - 1; }
static inline int left_pos(int p) { return 2 * (p + 1) - 1; }
static inline int right_pos(int p) { return 2 * (p + 1); }

static void h_swap(fheap *h, int a, int b) {
  h->nodes[h->heap[a]].pos = b;
  h->nodes[h->heap[b]].pos = a;
  int t = h->heap[a];
  h->heap[a] = h->heap[b];
  h->heap[b] = t;
}

static void h_up(fheap *h, int p) {
  while (p > 0 && h_less(h, h->heap[p], h->heap[parent_pos(p)])) {
    h_swap(h, p, parent_pos(p));
    p = parent_pos(p);
  }
}

static void h_down(fheap *h, int p) {
  for (;;) {
    int l = left_pos(p), r = right_pos(p);
    if (l >= h->size) return;
    if (h->tm) {
      /* total order: the smaller child moves up while it is before p */
      int c = (r < h->size && h_less(h, h->heap[r], h->heap[l])) ? r : l;
      if (!h_less(h, h->heap[c], h->heap[p])) return;
      h_swap(h, p, c);
      p = c;
      continue;
    }
    real cur = h->nodes[h->heap[p]].value;
    real lv = h->nodes[h->heap[l]].value;
    real rv = r < h->size ? h->nodes[h->heap[r]].value : REAL_MAX;
    if (cur <= lv && cur <= rv) return;
    if (lv < cur && lv <= rv) {
      h_swap(h, p, l);
      p = l;
    } else if (r < h->size) {
      h_swap(h, p, r);
      p = r;
    } else {
      return;
    }
  }
}

static int h_insert(fheap *h, long idx, real value) {
  int n = h->size;
  h->heap[n] = n;
  h->nodes[n].idx = idx;
  h->nodes[n].value = value;
  h->nodes[n].pos = n;
  h_up(h, n);
  h->size++;
  if (h->size == h->cap) h_grow(h);
  return h->size - 1;
}

/* Removes the root.  The node in the last handle slot moves into the root's
 * slot; *moved_idx / *moved_handle say where it went (-1 when none moved). */
static hnode h_extract(fheap *h, long *moved_idx, int *moved_handle) {
  int n = h->size;
  int root = h->heap[0];
  hnode min = h->nodes[root];
  *moved_idx = -1;
  *moved_handle = -1;
  if (root != n - 1) {
    hnode mv = h->nodes[n - 1];
    h->nodes[root] = mv;
    h->heap[mv.pos] = root;
    h->nodes[n - 1].value = REAL_MAX;
    *moved_idx = mv.idx;
    *moved_handle = root;
  } else {
    h->nodes[root].value = REAL_MAX;
  }
  /* the last position's node goes to the root and sifts down while the
   * last position still counts (as FMM_Heap_extractMin does) */
  h->nodes[h->heap[n - 1]].pos = 0;
  h->heap[0] = h->heap[n - 1];
  h_down(h, 0);
  h->heap[n - 1] = -1;
  h->size--;
  return min;
}

static void h_update(fheap *h, int handle, real value) {
  h->nodes[handle].value = value;
  int p = h->nodes[handle].pos;
  if (p > 0 && h_less(h, handle, h->heap[parent_pos(p)]))
    h_up(h, p);
  else
    h_down(h, p);
}

/* ---- the march ---------------------------------------------------------- */
typedef struct {
  real *d;
  const real *phi;
  unsigned char *st;
  int *handle;
  int n[3];
  long s[3];
  real dx[3];
  int order;
  int nf;            /* extension fields */
  real **ext;
  real **src;
  const real *emask;
  const real *speed; /* the Eikonal solver's speed (NULL: distance function) */
  time3 *tm;         /* the ordered march only: acceptance times */
  fheap trial;
} march_t;

/* The acceptance time of a point whose last update came from the acceptance
 * of a point of time x (has_trigger: a free point; else the front), for a
 * value of magnitude a: a new first level when a is above x's first level;
 * otherwise one level under x's, right after x (the heap pops a point an
 * update has lowered below the key just popped next).  Past the third level
 * the point keeps x's time. */
static time3 t3_after(const time3 *x, real a, int has_trigger) {
  time3 t = {a, -1.0, -1.0};
  if (!has_trigger || a > x->a) return t;
  t.a = x->a;
  if (x->b < 0 || a > x->b) {
    t.b = a;
    return t;
  }
  t.b = x->b;
  if (x->c < 0 || a > x->c) {
    t.c = a;
    return t;
  }
  return *x;
}

static real trial_update(march_t *m, long o, const int c[3]) {
  real A = 0, B = 0, C = 0;
  int used[3], plus[3], sws[3];
  real up1[3], up2[3];
  for (int dir = 0; dir < 3; dir++) {
    real u1 = REAL_MAX, u2 = REAL_MAX;
    int sw = 0;
    used[dir] = 0;
    plus[dir] = 0;
    for (int sg = -1; sg <= 1; sg += 2) {
      int c1 = c[dir] + sg;
      if (c1 < 0 || c1 >= m->n[dir]) continue;
      long o1 = o + sg * m->s[dir];
      if (m->st[o1] != KNOWN) continue;
      if (sg == 1 && !(fabs(m->d[o1]) < fabs(u1))) continue;
      u1 = m->d[o1];
      u2 = REAL_MAX;
      sw = 0;
      used[dir] = 1;
      plus[dir] = sg == 1;
      if (m->order == 2) {
        int c2 = c1 + sg;
        if (c2 >= 0 && c2 < m->n[dir]) {
          long o2 = o1 + sg * m->s[dir];
          if (m->st[o2] == KNOWN && fabs(m->d[o2]) <= fabs(u1)) {
            u2 = m->d[o2];
            sw = 1;
          }
        }
      }
    }
    up1[dir] = u1;
    up2[dir] = u2;
    sws[dir] = sw;
    if (u1 < REAL_MAX) {
      real inv = 1 / m->dx[dir];
      inv *= inv;
      if (m->order == 1) {
        A += inv;
        B += inv * u1;
        C += inv * u1 * u1;
      } else {
        real s = 1.0 + 0.5 * sw;
        real contrib = sw == 1 ? 2.0 * u1 - 0.5 * u2 : u1;
        A += inv * s * s;
        B += inv * s * contrib;
        C += inv * contrib * contrib;
      }
    }
  }
  if (fabs(A) == 0) return REAL_MAX;
  B *= -2.0;
  if (m->speed)
    C -= 1 / m->speed[o] / m->speed[o];
  else
    C -= 1.0;
  real disc = B * B - 4.0 * A * C;
  real out;
  if (disc >= 0) {
    if (m->speed)
      out = 0.5 * (-B + sqrt(disc)) / A;
    else if (B == 0)
      out = 0;
    else if (B < ZERO_TOL)
      out = 0.5 * (-B + sqrt(disc)) / A;
    else
      out = 0.5 * (-B - sqrt(disc)) / A;
  } else {
    out = m->d[o];
  }
  /* extension fields: weighted average over the axes in the update */
  for (int k = 0; k < m->nf; k++) {
    real num = 0, den = 0;
    for (int dir = 0; dir < 3; dir++) {
      if (!used[dir]) continue;
      long o1 = o + (plus[dir] ? 1 : -1) * m->s[dir];
      real inv = 1 / m->dx[dir];
      inv *= inv;
      real g = (m->order == 2 && sws[dir] == 1)
                   ? 1.5 * out - 2.0 * up1[dir] + 0.5 * up2[dir]
                   : out - up1[dir];
      num += inv * g * m->ext[k][o1];
      den += inv * g;
    }
    m->ext[k][o] = num / den;
  }
  m->d[o] = out;
  return out;
}

static void update_neighbors(march_t *m, long o, int from_free) {
  int c[3];
  c[0] = (int)(o % m->n[0]);
  c[1] = (int)((o / m->n[0]) % m->n[1]);
  c[2] = (int)(o / ((long)m->n[0] * m->n[1]));
  for (int dir = 0; dir < 3; dir++) {
    for (int sg = -1; sg <= 1; sg += 2) {
      int q[3] = {c[0], c[1], c[2]};
      q[dir] += sg;
      if (q[dir] < 0 || q[dir] >= m->n[dir]) continue;
      long oq = o + sg * m->s[dir];
      if (m->st[oq] == KNOWN || m->st[oq] == OUTSIDE) continue;
      real v = trial_update(m, oq, q);
      if (v < 0) v = -v;
      if (m->tm) m->tm[oq] = t3_after(&m->tm[o], v, from_free);
      if (m->st[oq] == FAR) {
        m->st[oq] = TRIAL;
        m->handle[oq] = h_insert(&m->trial, oq, v);
      } else {
        h_update(&m->trial, m->handle[oq], v);
      }
    }
  }
}

/* orc_computeExtensionFields3d: the reference's computeExtensionFields3d
 * (distance function and extension fields together); arrays x fastest,
 * grid_dims and dx in x, y, z order.  Returns 0, or 2 for an order other
 * than 1 and 2. */
static int extension_march(real *distance, real **ext, const real *phi, const real *mask,
                           real **src, const real *emask, int nf, int order,
                           const int *grid_dims, const real *dx, int ordered) {
  if (order != 1 && order != 2) return 2;
  march_t m;
  m.d = distance;
  m.phi = phi;
  m.order = order;
  m.nf = nf;
  m.ext = ext;
  m.src = src;
  m.emask = emask;
  m.speed = NULL;
  m.tm = NULL;
  for (int q = 0; q < 3; q++) {
    m.n[q] = grid_dims[q];
    m.dx[q] = dx[q];
  }
  m.s[0] = 1;
  m.s[1] = m.n[0];
  m.s[2] = (long)m.n[0] * m.n[1];
  long np = m.s[2] * m.n[2];
  m.st = (unsigned char *)calloc((size_t)np, 1);
  m.handle = (int *)malloc(sizeof(int) * (size_t)np);
  if (ordered) m.tm = (time3 *)calloc((size_t)np, sizeof(time3));
  for (long o = 0; o < np; o++) {
    distance[o] = -1;
    for (int k = 0; k < nf; k++) ext[k][o] = -1;
    m.handle[o] = -1;
    if (mask && mask[o] < 0) {
      m.st[o] = OUTSIDE;
      distance[o] = REAL_MAX;
      for (int k = 0; k < nf; k++) ext[k][o] = REAL_MAX;
    }
  }
  fheap known;
  h_init(&known, m.n[0] + m.n[1] + m.n[2]);
  h_init(&m.trial, m.n[0] + m.n[1] + m.n[2]);
  m.trial.tm = m.tm;

  /* the front (first-order initialisation at both orders) */
  real *fsum = nf ? (real *)malloc(sizeof(real) * nf) : NULL;
  real *fdir = nf ? (real *)malloc(sizeof(real) * 2 * nf) : NULL;
  for (long o = 0; o < np; o++) {
    if (m.st[o] == OUTSIDE) continue;
    int c[3] = {(int)(o % m.n[0]), (int)((o / m.n[0]) % m.n[1]),
                (int)(o / ((long)m.n[0] * m.n[1]))};
    real pc = phi[o];
    if (fabs(pc) < ZERO_TOL) {
      distance[o] = pc > 0 ? ZERO_TOL : -ZERO_TOL;
      for (int k = 0; k < nf; k++) ext[k][o] = src[k][o];
      m.st[o] = KNOWN;
      h_insert(&known, o, distance[o]);
      continue;
    }
    int borders = 0;
    real sum = 0;
    for (int k = 0; k < nf; k++) fsum[k] = 0;
    for (int dir = 0; dir < 3; dir++) {
      real dp = REAL_MAX, dm = REAL_MAX;
      for (int k = 0; k < 2 * nf; k++) fdir[k] = 0;   /* [minus k, plus k] */
      for (int sg = -1; sg <= 1; sg += 2) {
        if (c[dir] + sg < 0 || c[dir] + sg >= m.n[dir]) continue;
        long on = o + sg * m.s[dir];
        real p = phi[on];
        if (!(p * pc <= 0)) continue;
        real frac = pc / (pc - p);
        for (int k = 0; k < nf; k++) {
          real v;
          if (emask && emask[o] < 0)
            v = src[k][on];
          else if (emask && emask[on] < 0)
            v = src[k][o];
          else
            v = src[k][o] + frac * (src[k][on] - src[k][o]);
          fdir[(sg == 1 ? nf : 0) + k] = v;
        }
        frac *= m.dx[dir];
        if (sg == 1) dp = frac; else dm = frac;
      }
      if (dp < REAL_MAX || dm < REAL_MAX) {
        borders = 1;
        int use_plus = dp < dm;
        real dd = use_plus ? dp : dm;
        real w = 1 / dd / dd;
        sum += w;
        for (int k = 0; k < nf; k++) fsum[k] += fdir[(use_plus ? nf : 0) + k] * w;
      }
    }
    if (borders) {
      distance[o] = pc > 0 ? sqrt(1.0 / sum) : -sqrt(1.0 / sum);
      for (int k = 0; k < nf; k++) ext[k][o] = fsum[k] / sum;
      m.st[o] = KNOWN;
      h_insert(&known, o, distance[o]);
    }
  }
  free(fsum);
  free(fdir);
  /* the front's neighbours become trial points */
  while (known.size > 0) {
    long mi;
    int mh;
    hnode nd = h_extract(&known, &mi, &mh);
    if (nd.value < REAL_MAX) update_neighbors(&m, nd.idx, 0);
  }
  /* the march */
  while (m.trial.size > 0) {
    long mi;
    int mh;
    hnode nd = h_extract(&m.trial, &mi, &mh);
    if (mh != -1) m.handle[mi] = mh;
    m.st[nd.idx] = KNOWN;
    update_neighbors(&m, nd.idx, 1);
  }
  h_free(&known);
  h_free(&m.trial);
  free(m.st);
  free(m.handle);
  free(m.tm);
  return 0;
}

int orc_computeExtensionFields3d(real *distance, real **ext, const real *phi, const real *mask,
                                 real **src, const real *emask, int nf, int order,
                                 const int *grid_dims, const real *dx) {
  return extension_march(distance, ext, phi, mask, src, emask, nf, order, grid_dims, dx, 0);
}

/* orc_computeDistanceFunction3d: the distance function alone. */
int orc_computeDistanceFunction3d(real *distance, const real *phi, const real *mask, int order,
                                  const int *grid_dims, const real *dx) {
  return orc_computeExtensionFields3d(distance, NULL, phi, mask, NULL, NULL, 0, order,
                                      grid_dims, dx);
}

/* orc_solveEikonalEquation3d: the reference's solveEikonalEquation3d; phi is
 * the boundary data on input (the front: phi > -1e-11) and the solution on
 * output.  Returns 0, or 2 for an order other than 1 and 2. */
static int eikonal_march(real *phi, const real *speed, const real *mask, int order,
                         const int *grid_dims, const real *dx, int ordered) {
  if (order != 1 && order != 2) return 2;
  march_t m;
  m.d = phi;
  m.phi = phi;
  m.order = order;
  m.nf = 0;
  m.ext = NULL;
  m.src = NULL;
  m.emask = NULL;
  m.speed = speed;
  m.tm = NULL;
  for (int q = 0; q < 3; q++) {
    m.n[q] = grid_dims[q];
    m.dx[q] = dx[q];
  }
  m.s[0] = 1;
  m.s[1] = m.n[0];
  m.s[2] = (long)m.n[0] * m.n[1];
  long np = m.s[2] * m.n[2];
  m.st = (unsigned char *)calloc((size_t)np, 1);
  m.handle = (int *)malloc(sizeof(int) * (size_t)np);
  if (ordered) m.tm = (time3 *)calloc((size_t)np, sizeof(time3));
  for (long o = 0; o < np; o++) {
    m.handle[o] = -1;
    if ((mask && mask[o] < 0) || speed[o] < ZERO_TOL) {
      m.st[o] = OUTSIDE;
      phi[o] = REAL_MAX;
    }
  }
  fheap known;
  h_init(&known, m.n[0] + m.n[1] + m.n[2]);
  h_init(&m.trial, m.n[0] + m.n[1] + m.n[2]);
  m.trial.tm = m.tm;
  for (long o = 0; o < np; o++)
    if (phi[o] > -ZERO_TOL && m.st[o] != OUTSIDE) {
      m.st[o] = KNOWN;
      h_insert(&known, o, phi[o]);
    }
  while (known.size > 0) {
    long mi;
    int mh;
    hnode nd = h_extract(&known, &mi, &mh);
    if (nd.value < REAL_MAX) update_neighbors(&m, nd.idx, 0);
  }
  while (m.trial.size > 0) {
    long mi;
    int mh;
    hnode nd = h_extract(&m.trial, &mi, &mh);
    if (mh != -1) m.handle[mi] = mh;
    m.st[nd.idx] = KNOWN;
    update_neighbors(&m, nd.idx, 1);
  }
  h_free(&known);
  h_free(&m.trial);
  free(m.st);
  free(m.handle);
  free(m.tm);
  return 0;
}

int orc_solveEikonalEquation3d(real *phi, const real *speed, const real *mask, int order,
                               const int *grid_dims, const real *dx) {
  return eikonal_march(phi, speed, mask, order, grid_dims, dx, 0);
}

/* ---- the ordered march ----------------------------------------------------
 * The same march with the trial heap keyed on a total order instead of the
 * value: (acceptance time, linear index), the time set at every update by
 * t3_after from the time of the point whose acceptance made the update.
 * Where no two keys tie, this pops in the reference's order and the results
 * are the reference's bit for bit.  Where keys tie exactly (symmetric
 * inputs, flat fronts, quantised data), the reference's binary heap pops the
 * tied points in an order set by its whole history of insertions and
 * removals; this march pops them by time and then by index.  The GPU solver
 * computes this march's result, except where updates among exactly equal
 * values lower points more than three levels deep (t3_after keeps the
 * trigger's time there); that has been seen at first order only, with
 * differences of a few ulps. */
int orc_computeExtensionFields3d_ordered(real *distance, real **ext, const real *phi,
                                         const real *mask, real **src, const real *emask,
                                         int nf, int order, const int *grid_dims,
                                         const real *dx) {
  return extension_march(distance, ext, phi, mask, src, emask, nf, order, grid_dims, dx, 1);
}

int orc_computeDistanceFunction3d_ordered(real *distance, const real *phi, const real *mask,
                                          int order, const int *grid_dims, const real *dx) {
  return extension_march(distance, NULL, phi, mask, NULL, NULL, 0, order, grid_dims, dx, 1);
}

int orc_solveEikonalEquation3d_ordered(real *phi, const real *speed, const real *mask, int order,
                                       const int *grid_dims, const real *dx) {
  return eikonal_march(phi, speed, mask, order, grid_dims, dx, 1);
}
