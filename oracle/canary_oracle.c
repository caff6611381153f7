/*
 * CPU oracle: a plain-C restatement of the CPU code path of CliMA/Canary.jl
 * for the nodal-DG hot path.  TEST INFRASTRUCTURE ONLY (see canary_oracle.h).
 *
 * Every function follows the cited Julia lines operation by operation, in the
 * same evaluation order (Julia folds `a*b*c` and `a+b+c` left to right), and
 * is compiled with -ffp-contract=off so that no multiply-add is fused.
 * Deviations that are unavoidable in C are listed where they occur:
 *   - Julia's 2-argument `hypot` is replaced by C99 hypot (both are within one
 *     ulp of the correctly rounded value).
 *   - Julia's n-argument `hypot` (used for 3-D face normals) is restated as
 *     maxabs * sqrt(sum((v/maxabs)^2)), which is how Julia Base defines it.
 *   - `sortperm`/`sortslices` are replaced by a stable sort; ties only occur
 *     for equal keys, whose order the reference leaves unspecified.
 */
#include "canary_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OMP_THREADS(nt) num_threads((nt) > 0 ? (nt) : 1)

/* ===================================================================== */
/* src/GaussQuadrature/quadrature.jl                                     */
/* ===================================================================== */

/* legendre_coefs, quadrature.jl:140-148 */
int or_legendre_coefs(int n, double *a, double *b) {
  for (int i = 0; i < n; i++) a[i] = 0.0;
  b[0] = sqrt(2.0);
  for (int k = 2; k <= n + 1; k++)
    b[k - 1] = (double)(k - 1) / sqrt((double)((2 * k - 1) * (2 * k - 3)));
  return 0;
}

/* solve, quadrature.jl:216-233 (1-based a[i] -> a[i-1]) */
static double qsolve(int n, double shift, const double *a, const double *b) {
  double t = a[0] - shift;
  for (int i = 2; i <= n - 1; i++)
    t = (a[i - 1] - shift) - (b[i - 1] * b[i - 1]) / t;
  return 1.0 / t;
}

/* special_eigenproblem!, quadrature.jl:235-326.  Returns 0, or the iteration
 * count at which the reference raises "No convergence after j iterations". */
static int special_eigenproblem(int n, double *d, double *e, double *z,
                                int maxits) {
  /* 1-based views: D(i) = d[i-1], E(i) = e[i-1], Z(i) = z[i-1] */
#define D_(i) d[(i)-1]
#define E_(i) e[(i)-1]
#define Z_(i) z[(i)-1]
  Z_(1) = 1.0;
  for (int i = 2; i <= n; i++) Z_(i) = 0.0;
  E_(n + 1) = 0.0;
  if (n == 1) return 0;
  for (int l = 1; l <= n; l++) {
    for (int j = 1; j <= maxits; j++) {
      int m = n;
      for (int i = l; i <= n - 1; i++) {
        if (fabs(E_(i + 1)) <= DBL_EPSILON * (fabs(D_(i)) + fabs(D_(i + 1)))) {
          m = i;
          break;
        }
      }
      double p = D_(l);
      if (m == l) continue;
      if (j == maxits) return j;
      double g = (D_(l + 1) - p) / (2.0 * E_(l + 1));
      double r = hypot(g, 1.0);
      g = (D_(m) - p) + E_(l + 1) / (g + copysign(r, g));
      double s = 1.0, c = 1.0;
      p = 0.0;
      for (int i = m - 1; i >= l; i--) {
        double f = s * E_(i + 1);
        double b = c * E_(i + 1);
        if (fabs(f) < fabs(g)) {
          s = f / g;
          r = hypot(s, 1.0);
          E_(i + 2) = g * r;
          c = 1.0 / r;
          s *= c;
        } else {
          c = g / f;
          r = hypot(c, 1.0);
          E_(i + 2) = f * r;
          s = 1.0 / r;
          c *= s;
        }
        g = D_(i + 1) - p;
        r = (D_(i) - g) * s + (2.0 * c) * b;
        p = s * r;
        D_(i + 1) = g + p;
        g = c * r - b;
        f = Z_(i + 1);
        Z_(i + 1) = s * Z_(i) + c * f;
        Z_(i) = c * Z_(i) - s * f;
      }
      D_(l) -= p;
      E_(l + 1) = g;
      E_(m + 1) = 0.0;
    }
  }
#undef D_
#undef E_
#undef Z_
  return 0;
}

/* custom_gauss_rule, quadrature.jl:175-214.  endpt is 'N','L','R','B'.
 * Returns 0; 1 for "Must have at least two points for both ends."; 2 for
 * "No convergence after *err_iter iterations". a (n) and b (n+1) are
 * overwritten as in the reference. */
int or_custom_gauss_rule(double lo, double hi, int n, double *a, double *b,
                         char endpt, int maxits, double *x, double *w,
                         int *err_iter) {
  if (endpt == 'L') {
    if (n == 1) a[0] = lo;
    else a[n - 1] = qsolve(n, lo, a, b) * (b[n - 1] * b[n - 1]) + lo;
  } else if (endpt == 'R') {
    if (n == 1) a[0] = hi;
    else a[n - 1] = qsolve(n, hi, a, b) * (b[n - 1] * b[n - 1]) + hi;
  } else if (endpt == 'B') {
    if (n == 1) return 1;
    double g = qsolve(n, lo, a, b);
    double t1 = (hi - lo) / (g - qsolve(n, hi, a, b));
    b[n - 1] = sqrt(t1);
    a[n - 1] = lo + g * t1;
  }
  double *wz = (double *)calloc((size_t)n, sizeof(double));
  int it = special_eigenproblem(n, a, b, wz, maxits);
  if (it) {
    if (err_iter) *err_iter = it;
    free(wz);
    return 2;
  }
  for (int i = 0; i < n; i++) {
    double t = b[0] * wz[i];
    wz[i] = t * t;
  }
  /* idx = sortperm(a): stable insertion sort of indices by value */
  int *idx = (int *)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; i++) idx[i] = i;
  for (int i = 1; i < n; i++) {
    int v = idx[i], j = i - 1;
    while (j >= 0 && a[idx[j]] > a[v]) {
      idx[j + 1] = idx[j];
      j--;
    }
    idx[j + 1] = v;
  }
  /* "Ensure end point values are exact": `both` only pins the left end
   * (quadrature.jl:208-212). */
  if (endpt == 'L' || endpt == 'B') a[idx[0]] = lo;
  else if (endpt == 'R') a[idx[n - 1]] = hi;
  for (int i = 0; i < n; i++) {
    x[i] = a[idx[i]];
    w[i] = wz[idx[i]];
  }
  free(idx);
  free(wz);
  return 0;
}

/* legendre, quadrature.jl:126-131 (maxiterations[Float64] = 30, :115) */
int or_legendre(int n, char endpt, double *x, double *w) {
  if (n < 1) return 3;
  double *a = (double *)malloc(sizeof(double) * (size_t)n);
  double *b = (double *)malloc(sizeof(double) * (size_t)(n + 1));
  or_legendre_coefs(n, a, b);
  int it = 0;
  int rc = or_custom_gauss_rule(-1.0, 1.0, n, a, b, endpt, 30, x, w, &it);
  free(a);
  free(b);
  return rc;
}

/* ===================================================================== */
/* src/operators.jl                                                      */
/* ===================================================================== */

/* lglpoints, operators.jl:10-13 */
int or_lglpoints(int N, double *r, double *w) {
  if (N < 1) return 3;
  return or_legendre(N + 1, 'B', r, w);
}

/* lgpoints, operators.jl:21-24 */
int or_lgpoints(int N, double *r, double *w) {
  if (N < 1) return 3;
  return or_legendre(N + 1, 'N', r, w);
}

/* baryweights, operators.jl:36-49 */
void or_baryweights(int n, const double *r, double *wb) {
  for (int j = 0; j < n; j++) wb[j] = 1.0;
  for (int j = 0; j < n; j++) {
    for (int i = 0; i < n; i++)
      if (i != j) wb[j] = wb[j] * (r[j] - r[i]);
    wb[j] = 1.0 / wb[j];
  }
}

/* spectralderivative, operators.jl:64-84.  D is n x n column-major. */
void or_spectralderivative(int n, const double *r, double *D) {
  double *wb = (double *)malloc(sizeof(double) * (size_t)n);
  or_baryweights(n, r, wb);
  for (int i = 0; i < n * n; i++) D[i] = 0.0;
  for (int k = 0; k < n; k++) {
    for (int j = 0; j < n; j++) {
      if (k == j) {
        for (int l = 0; l < n; l++)
          if (l != k) D[j + n * k] = D[j + n * k] + 1.0 / (r[k] - r[l]);
      } else {
        D[j + n * k] = (wb[k] / wb[j]) / (r[j] - r[k]);
      }
    }
  }
  free(wb);
}

/* interpolationmatrix, operators.jl:98-117.  I is ndst x nsrc. */
void or_interpolationmatrix(int nsrc, const double *rsrc, int ndst,
                            const double *rdst, double *I) {
  double *wb = (double *)malloc(sizeof(double) * (size_t)nsrc);
  or_baryweights(nsrc, rsrc, wb);
  for (int k = 0; k < ndst; k++) {
    for (int j = 0; j < nsrc; j++) {
      I[k + ndst * j] = wb[j] / (rdst[k] - rsrc[j]);
      if (!isfinite(I[k + ndst * j])) {
        for (int jj = 0; jj < nsrc; jj++) I[k + ndst * jj] = 0.0;
        I[k + ndst * j] = 1.0;
        break;
      }
    }
    double d = 0.0;
    for (int j = 0; j < nsrc; j++) d += I[k + ndst * j];
    for (int j = 0; j < nsrc; j++) I[k + ndst * j] = I[k + ndst * j] / d;
  }
  free(wb);
}

/* ===================================================================== */
/* src/mesh.jl                                                           */
/* ===================================================================== */

/* hilbertcode, mesh.jl:35-88 (Skilling's AxestoTranspose + bit transpose) */
void or_hilbertcode(int n, const uint64_t *Y, int bits, uint64_t *H) {
  uint64_t X[16];
  for (int i = 0; i < n; i++) X[i] = Y[i];
  uint64_t M = (uint64_t)1 << (bits - 1);
  uint64_t Qb = M;
  for (int j = 1; j <= bits - 1; j++) {
    uint64_t P = Qb - 1;
    for (int i = 0; i < n; i++) {
      if ((X[i] & Qb) != 0) {
        X[0] ^= P;
      } else {
        uint64_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
    Qb >>= 1;
  }
  for (int i = 1; i < n; i++) X[i] ^= X[i - 1];
  uint64_t t = 0;
  Qb = M;
  for (int j = 1; j <= bits - 1; j++) {
    if ((X[n - 1] & Qb) != 0) t ^= Qb - 1;
    Qb >>= 1;
  }
  for (int i = 0; i < n; i++) X[i] ^= t;
  for (int i = 0; i < n; i++) H[i] = 0;
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < bits; j++) {
      int k = i * bits + j;
      uint64_t bit = (X[(n - (k % n)) - 1] >> (k / n)) & 1u;
      H[(n - i) - 1] |= bit << j;
    }
  }
}

/* floor((2^64-1) * c) evaluated exactly, c in [0, 1] (mesh.jl:136 computes it
 * in 128-bit BigFloat, where the product of the 64-bit and 53-bit
 * significands is exact). */
static uint64_t scaled_floor_u64(double c) {
  if (!(c > 0.0)) return 0;
  int ex;
  double f = frexp(c, &ex); /* c = f * 2^ex, f in [0.5, 1) */
  uint64_t m = (uint64_t)ldexp(f, 53);
  unsigned __int128 P = (unsigned __int128)UINT64_MAX * m;
  int sh = 53 - ex;
  if (sh <= 0) return UINT64_MAX;
  if (sh >= 128) return 0;
  return (uint64_t)(P >> sh);
}

/* centroidtocode, mesh.jl:107-141 (single rank: Allreduce is the identity) */
void or_centroidtocode(int d, int nvert, int64_t nelem,
                       const double *elemtocoord, uint64_t *code) {
  double *cen = (double *)malloc(sizeof(double) * (size_t)(d * (nelem > 0 ? nelem : 1)));
  double cmin[8], cmax[8], csize[8];
  for (int i = 0; i < d; i++) {
    cmin[i] = DBL_MAX;
    cmax[i] = -DBL_MAX;
  }
  for (int64_t e = 0; e < nelem; e++) {
    for (int i = 0; i < d; i++) {
      double s = 0.0;
      for (int v = 0; v < nvert; v++) s += elemtocoord[i + d * (v + nvert * e)];
      cen[i + d * e] = s / (double)nvert;
      if (cen[i + d * e] < cmin[i]) cmin[i] = cen[i + d * e];
      if (cen[i + d * e] > cmax[i]) cmax[i] = cen[i + d * e];
    }
  }
  int allzero = 1;
  double maxsize = -DBL_MAX;
  for (int i = 0; i < d; i++) {
    csize[i] = cmax[i] - cmin[i];
    if (csize[i] != 0.0) allzero = 0;
    if (csize[i] > maxsize) maxsize = csize[i];
  }
  if (allzero) {
    for (int i = 0; i < d; i++) csize[i] = 1.0;
  } else {
    for (int i = 0; i < d; i++)
      if (csize[i] == 0.0) csize[i] = maxsize;
  }
  for (int64_t e = 0; e < nelem; e++) {
    uint64_t X[8];
    for (int i = 0; i < d; i++) {
      double c = (cen[i + d * e] - cmin[i]) / csize[i];
      X[i] = scaled_floor_u64(c);
    }
    or_hilbertcode(d, X, 64, code + d * e);
  }
  free(cen);
}

/* vertsortandorder, mesh.jl:595-719.  Returns 0, or 1 when the reference
 * raises "Problem finding vertex ordering". flips (if non-NULL) receives the
 * swap flags s1..s5. */
int or_vertsortandorder(int nv, const int64_t *vin, int64_t *v, int *o,
                        int *flips) {
  for (int i = 0; i < nv; i++) v[i] = vin[i];
#define MMF(x, y, s)                                                         \
  do {                                                                       \
    if (v[y] < v[x]) {                                                       \
      int64_t t_ = v[x];                                                     \
      v[x] = v[y];                                                           \
      v[y] = t_;                                                             \
      s = 1;                                                                 \
    } else                                                                   \
      s = 0;                                                                 \
  } while (0)
  if (nv == 1) {
    *o = 1;
    return 0;
  }
  if (nv == 2) {
    int s1;
    MMF(0, 1, s1);
    *o = s1 ? 2 : 1;
    if (flips) flips[0] = s1;
    return 0;
  }
  if (nv == 3) {
    int s1, s2, s3;
    MMF(1, 2, s1);
    MMF(0, 2, s2);
    MMF(0, 1, s3);
    if (flips) {
      flips[0] = s1;
      flips[1] = s2;
      flips[2] = s3;
    }
    if (!s1 && !s2 && !s3) *o = 1;
    else if (!s1 && s2 && s3) *o = 2;
    else if (s1 && !s2 && s3) *o = 3;
    else if (!s1 && !s2 && s3) *o = 4;
    else if (s1 && s2 && s3) *o = 5;
    else if (s1 && !s2 && !s3) *o = 6;
    else return 1;
    return 0;
  }
  if (nv == 4) {
    int s1, s2, s3, s4, s5;
    MMF(0, 1, s1);
    MMF(2, 3, s2);
    MMF(0, 2, s3);
    MMF(1, 3, s4);
    MMF(1, 2, s5);
    if (flips) {
      flips[0] = s1;
      flips[1] = s2;
      flips[2] = s3;
      flips[3] = s4;
      flips[4] = s5;
    }
    if (!s1 && !s2 && !s3 && !s4 && !s5) *o = 1;
    else if (!s1 && !s2 && !s3 && !s4 && s5) *o = 2;
    else if (s1 && !s2 && !s3 && !s4 && !s5) *o = 3;
    else if (!s1 && !s2 && s3 && s4 && s5) *o = 4;
    else if (s1 && s2 && !s3 && !s4 && s5) *o = 5;
    else if (!s1 && !s2 && s3 && s4 && !s5) *o = 6;
    else if (s1 && s2 && s3 && s4 && s5) *o = 7;
    else if (s1 && s2 && s3 && s4 && !s5) *o = 8;
    else return 1;
    return 0;
  }
#undef MMF
  return 2;
}

/* face corner mask of brickmesh/connectmesh (mesh.jl:281-284, :757-760):
 * corners of the 2^d reference element whose coordinate in dimension
 * div(f,2) is f%2, listed column-major.  Zero-based corner ids. */
static void corner_fmask(int d, int f, int *out) {
  int fd = f / 2, side = f % 2, c = 0;
  for (int v = 0; v < (1 << d); v++)
    if (((v >> fd) & 1) == side) out[c++] = v;
}

/* brickmesh, mesh.jl:259-317.  x holds the concatenated coordinate vectors
 * (nx[i] entries for dimension i); boundary is 2 x d column-major.  Outputs
 * are sized for the local part; faceconnections rows are (2 + 2^(d-1))
 * int64 [e, f, verts...] with 1-based values.  Returns the number of local
 * elements (or -1 on bad arguments). */
int64_t or_brickmesh(int d, const double *x, const int64_t *nx,
                     const int *periodic, int64_t part, int64_t numparts,
                     const int64_t *boundary, int64_t *elemtovert,
                     double *elemtocoord, int64_t *elemtobndy,
                     int64_t *faceconnections, int64_t *nfc) {
  if (d < 1 || d > 3 || part < 1 || part > numparts) return -1;
  int nvert = 1 << d, nface = 2 * d, nfv = 1 << (d - 1);
  int64_t nelemdim[3], off[3];
  int64_t total = 1, o = 0;
  for (int i = 0; i < d; i++) {
    nelemdim[i] = nx[i] - 1;
    total *= nelemdim[i];
    off[i] = o;
    o += nx[i];
  }
  int64_t lo = ((part - 1) * total) / numparts + 1;
  int64_t hi = (part * total) / numparts;
  int64_t nloc = hi - lo + 1;
  int fmask[6][4];
  for (int f = 0; f < nface; f++) corner_fmask(d, f, fmask[f]);
  int64_t cfc = 0;
  for (int64_t el = 0; el < nloc; el++) {
    int64_t g = lo - 1 + el; /* zero-based global element, column-major */
    int64_t ec[3];
    for (int i = 0; i < d; i++) {
      ec[i] = g % nelemdim[i] + 1;
      g /= nelemdim[i];
    }
    for (int v = 0; v < nvert; v++) {
      int64_t vid = 0, stride = 1;
      for (int j = 0; j < d; j++) {
        int64_t vc = ec[j] + ((v >> j) & 1);
        vid += (vc - 1) * stride;
        stride *= nx[j];
        elemtocoord[j + d * (v + nvert * el)] = x[off[j] + vc - 1];
      }
      elemtovert[v + nvert * el] = vid + 1;
    }
    for (int f = 0; f < nface; f++) elemtobndy[f + nface * el] = 0;
    for (int i = 0; i < d; i++) {
      if (!periodic[i] && ec[i] == 1)
        elemtobndy[2 * i + nface * el] = boundary[0 + 2 * i];
      if (!periodic[i] && ec[i] == nelemdim[i])
        elemtobndy[2 * i + 1 + nface * el] = boundary[1 + 2 * i];
    }
    for (int i = 0; i < d; i++) {
      if (periodic[i] && ec[i] == nelemdim[i]) {
        int64_t *row = faceconnections + (2 + nfv) * cfc;
        row[0] = el + 1;
        row[1] = 2 * (i + 1);
        for (int q = 0; q < nfv; q++) {
          int v = fmask[2 * i][q];
          int64_t vid = 0, stride = 1;
          for (int j = 0; j < d; j++) {
            int64_t base = (j == i) ? 1 : ec[j];
            int64_t vc = base + ((v >> j) & 1);
            vid += (vc - 1) * stride;
            stride *= nx[j];
          }
          row[2 + q] = vid + 1;
        }
        cfc++;
      }
    }
  }
  *nfc = cfc;
  return nloc;
}

/* lexicographic comparison of Hilbert codes with the element number as the
 * final key (the columns [code; e] of getpartition, mesh.jl:413-420) */
static const uint64_t *g_codes;
static int g_d;
static int cmp_code(const void *pa, const void *pb) {
  int64_t a = *(const int64_t *)pa, b = *(const int64_t *)pb;
  for (int i = 0; i < g_d; i++) {
    uint64_t ca = g_codes[i + g_d * a], cb = g_codes[i + g_d * b];
    if (ca < cb) return -1;
    if (ca > cb) return 1;
  }
  return (a > b) - (a < b);
}

/* partition, mesh.jl:499-580, on a single rank: elements are reordered by
 * Hilbert code of their centroids; face connections follow their elements.
 * Arrays are permuted in place. */
int or_partition(int d, int64_t nelem, int64_t *elemtovert,
                 double *elemtocoord, int64_t *elemtobndy,
                 int64_t *faceconnections, int64_t *nfc) {
  int nvert = 1 << d, nface = 2 * d, nfv = 1 << (d - 1);
  uint64_t *code = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(d * (nelem > 0 ? nelem : 1)));
  or_centroidtocode(d, nvert, nelem, elemtocoord, code);
  int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nelem > 0 ? nelem : 1));
  for (int64_t e = 0; e < nelem; e++) order[e] = e;
  g_codes = code;
  g_d = d;
  qsort(order, (size_t)nelem, sizeof(int64_t), cmp_code);
  /* elemtofaceconnect (nfv, nface, nelem), mesh.jl:513-517 */
  int64_t *e2fc = (int64_t *)calloc((size_t)(nfv * nface * (nelem > 0 ? nelem : 1)), sizeof(int64_t));
  for (int64_t c = 0; c < *nfc; c++) {
    const int64_t *row = faceconnections + (2 + nfv) * c;
    for (int q = 0; q < nfv; q++)
      e2fc[q + nfv * ((row[1] - 1) + nface * (row[0] - 1))] = row[2 + q];
  }
  int64_t *tv = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nvert * nelem + 1));
  double *tc = (double *)malloc(sizeof(double) * (size_t)(d * nvert * nelem + 1));
  int64_t *tb = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nface * nelem + 1));
  int64_t *tf = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nfv * nface * nelem + 1));
  for (int64_t e = 0; e < nelem; e++) {
    int64_t s = order[e];
    memcpy(tv + nvert * e, elemtovert + nvert * s, sizeof(int64_t) * nvert);
    memcpy(tc + d * nvert * e, elemtocoord + d * nvert * s, sizeof(double) * d * nvert);
    memcpy(tb + nface * e, elemtobndy + nface * s, sizeof(int64_t) * nface);
    memcpy(tf + nfv * nface * e, e2fc + nfv * nface * s, sizeof(int64_t) * nfv * nface);
  }
  memcpy(elemtovert, tv, sizeof(int64_t) * nvert * nelem);
  memcpy(elemtocoord, tc, sizeof(double) * d * nvert * nelem);
  memcpy(elemtobndy, tb, sizeof(int64_t) * nface * nelem);
  /* the second, local code sort of mesh.jl:562-570 is the identity here */
  int64_t c = 0;
  for (int64_t e = 0; e < nelem; e++) {
    for (int f = 0; f < nface; f++) {
      if (tf[0 + nfv * (f + nface * e)] > 0) {
        int64_t *row = faceconnections + (2 + nfv) * c;
        row[0] = e + 1;
        row[1] = f + 1;
        for (int q = 0; q < nfv; q++) row[2 + q] = tf[q + nfv * (f + nface * e)];
        c++;
      }
    }
  }
  *nfc = c;
  free(code);
  free(order);
  free(e2fc);
  free(tv);
  free(tc);
  free(tb);
  free(tf);
  return 0;
}

typedef struct {
  int64_t v[4];
  int64_t col; /* (e-1)*nface + f - 1 */
  int o;
} face_key;
static int g_nfv;
static int cmp_face(const void *pa, const void *pb) {
  const face_key *a = (const face_key *)pa, *b = (const face_key *)pb;
  for (int i = 0; i < g_nfv; i++) {
    if (a->v[i] < b->v[i]) return -1;
    if (a->v[i] > b->v[i]) return 1;
  }
  return (a->col > b->col) - (a->col < b->col);
}

/* connectmesh, mesh.jl:751-956, on a single rank (no ghosts).  Returns 0,
 * 1 on a vertex-ordering error, 2 on an unsupported 3-D orientation
 * ("TODO add support for other orientations", :913-915). */
int or_connectmesh(int d, int64_t nelem, const int64_t *elemtovert,
                   const int64_t *elemtobndy_in,
                   const int64_t *faceconnections, int64_t nfc,
                   int64_t *elemtoelem, int64_t *elemtoface,
                   int64_t *elemtoordr, int64_t *elemtobndy) {
  int nvert = 1 << d, nface = 2 * d, nfv = 1 << (d - 1);
  int fmask[6][4];
  for (int f = 0; f < nface; f++) corner_fmask(d, f, fmask[f]);
  int64_t ncol = nface * nelem;
  face_key *A = (face_key *)malloc(sizeof(face_key) * (size_t)(ncol > 0 ? ncol : 1));
  for (int64_t e = 0; e < nelem; e++) {
    for (int f = 0; f < nface; f++) {
      int64_t j = e * nface + f, fvin[4];
      for (int q = 0; q < nfv; q++) fvin[q] = elemtovert[fmask[f][q] + nvert * e];
      face_key *k = &A[j];
      if (or_vertsortandorder(nfv, fvin, k->v, &k->o, NULL)) {
        free(A);
        return 1;
      }
      k->col = j;
    }
  }
  for (int64_t c = 0; c < nfc; c++) {
    const int64_t *row = faceconnections + (2 + nfv) * c;
    int64_t j = (row[0] - 1) * nface + (row[1] - 1);
    if (or_vertsortandorder(nfv, row + 2, A[j].v, &A[j].o, NULL)) {
      free(A);
      return 1;
    }
  }
  g_nfv = nfv;
  qsort(A, (size_t)ncol, sizeof(face_key), cmp_face);
  for (int64_t e = 0; e < nelem; e++) {
    for (int f = 0; f < nface; f++) {
      elemtoelem[f + nface * e] = e + 1;
      elemtoface[f + nface * e] = f + 1;
      elemtoordr[f + nface * e] = 1;
      elemtobndy[f + nface * e] = elemtobndy_in[f + nface * e];
    }
  }
  int64_t j = 0;
  while (j < ncol) {
    int same = 0;
    if (j + 1 < ncol) {
      same = 1;
      for (int q = 0; q < nfv; q++)
        if (A[j].v[q] != A[j + 1].v[q]) same = 0;
    }
    if (same) {
      for (int s = 0; s < 2; s++) {
        face_key *m = &A[j + s], *n = &A[j + 1 - s];
        int64_t me = m->col / nface, mf = m->col % nface;
        int64_t ne = n->col / nface, nf = n->col % nface;
        elemtoelem[mf + nface * me] = ne + 1;
        elemtoface[mf + nface * me] = nf + 1;
        if (d == 2) {
          elemtoordr[mf + nface * me] = (n->o == m->o) ? 1 : 2;
        } else if (d == 3) {
          if (n->o != 1 || m->o != 1) {
            free(A);
            return 2;
          }
          elemtoordr[mf + nface * me] = 1;
        }
      }
      j += 2;
    } else {
      j += 1;
    }
  }
  free(A);
  return 0;
}

/* mappings, mesh.jl:973-1001.  Returns 1 if an orientation other than 1 is
 * met (the reference asserts o2 == 1). */
int or_mappings(int d, int N, int64_t nelem, const int64_t *elemtoelem,
                const int64_t *elemtoface, const int64_t *elemtoordr,
                int64_t *vmapM, int64_t *vmapP) {
  int nface = 2 * d, Nq = N + 1;
  int64_t Np = 1, Nfp = 1;
  for (int i = 0; i < d; i++) Np *= Nq;
  for (int i = 0; i < d - 1; i++) Nfp *= Nq;
  int64_t *fm = (int64_t *)malloc(sizeof(int64_t) * (size_t)(Nfp * nface));
  for (int f = 0; f < nface; f++) {
    int fd = f / 2, fe = N * (f % 2);
    int64_t c = 0;
    for (int64_t n = 0; n < Np; n++) {
      int64_t t = n;
      int ok = 1;
      for (int j = 0; j < d; j++) {
        int64_t ij = t % Nq;
        t /= Nq;
        if (j == fd && ij != fe) ok = 0;
      }
      if (ok) fm[c++ + Nfp * f] = n + 1;
    }
  }
  for (int64_t e1 = 0; e1 < nelem; e1++) {
    for (int f1 = 0; f1 < nface; f1++) {
      int64_t e2 = elemtoelem[f1 + nface * e1];
      int64_t f2 = elemtoface[f1 + nface * e1];
      int64_t o2 = elemtoordr[f1 + nface * e1];
      if (o2 != 1) {
        free(fm);
        return 1;
      }
      for (int64_t n = 0; n < Nfp; n++) {
        vmapM[n + Nfp * (f1 + nface * e1)] = Np * e1 + fm[n + Nfp * f1];
        vmapP[n + Nfp * (f1 + nface * e1)] = Np * (e2 - 1) + fm[n + Nfp * (f2 - 1)];
      }
    }
  }
  free(fm);
  return 0;
}

/* ===================================================================== */
/* src/metric.jl                                                         */
/* ===================================================================== */

/* creategrid! 1-D :11-24, 2-D :36-57, 3-D :70-107 */
void or_creategrid(int d, int Nq, int64_t nelem, const double *e2c,
                   const double *r, double *x, double *y, double *z) {
  int nvert = 1 << d;
  if (d == 1) {
    for (int64_t e = 0; e < nelem; e++)
      for (int i = 0; i < Nq; i++)
        x[i + Nq * e] = ((1.0 - r[i]) * e2c[0 + nvert * e] +
                         (1.0 + r[i]) * e2c[1 + nvert * e]) / 2.0;
    return;
  }
  if (d == 2) {
    double *F[2] = {x, y};
    for (int n = 0; n < 2; n++)
      for (int64_t e = 0; e < nelem; e++)
        for (int j = 0; j < Nq; j++)
          for (int i = 0; i < Nq; i++) {
#define C2(v) e2c[n + 2 * ((v) + 4 * e)]
            double t = (1.0 - r[i]) * (1.0 - r[j]) * C2(0);
            t = t + (1.0 + r[i]) * (1.0 - r[j]) * C2(1);
            t = t + (1.0 - r[i]) * (1.0 + r[j]) * C2(2);
            t = t + (1.0 + r[i]) * (1.0 + r[j]) * C2(3);
            F[n][i + Nq * (j + Nq * e)] = t / 4.0;
#undef C2
          }
    return;
  }
  double *F[3] = {x, y, z};
  for (int n = 0; n < 3; n++)
    for (int64_t e = 0; e < nelem; e++)
      for (int k = 0; k < Nq; k++)
        for (int j = 0; j < Nq; j++)
          for (int i = 0; i < Nq; i++) {
#define C3(v) e2c[n + 3 * ((v) + 8 * e)]
            double a = 1.0 - r[i], b = 1.0 + r[i];
            double c = 1.0 - r[j], dd = 1.0 + r[j];
            double g = 1.0 - r[k], h = 1.0 + r[k];
            double t = a * c * g * C3(0);
            t = t + b * c * g * C3(1);
            t = t + a * dd * g * C3(2);
            t = t + b * dd * g * C3(3);
            t = t + a * c * h * C3(4);
            t = t + b * c * h * C3(5);
            t = t + a * dd * h * C3(6);
            t = t + b * dd * h * C3(7);
            F[n][i + Nq * (j + Nq * (k + Nq * e))] = t / 8.0;
#undef C3
          }
}

static double sgn(double v) { return (v > 0) - (v < 0); }

/* computemetric! 1-D, metric.jl:120-141 */
void or_computemetric1d(int Nq, int64_t nelem, const double *x, double *J,
                        double *xix, double *sJ, double *nx, const double *D) {
  for (int64_t e = 0; e < nelem; e++) {
    for (int i = 0; i < Nq; i++) {
      double s = 0.0;
      for (int n = 0; n < Nq; n++) s += D[i + Nq * n] * x[n + Nq * e];
      J[i + Nq * e] = s;
    }
    for (int i = 0; i < Nq; i++) xix[i + Nq * e] = 1.0 / J[i + Nq * e];
    nx[0 + 2 * e] = -sgn(J[0 + Nq * e]);
    nx[1 + 2 * e] = sgn(J[Nq - 1 + Nq * e]);
    sJ[0 + 2 * e] = 1.0;
    sJ[1 + 2 * e] = 1.0;
  }
}

/* computemetric! 2-D, metric.jl:155-208 */
void or_computemetric2d(int Nq, int64_t nelem, const double *x,
                        const double *y, double *J, double *xix, double *etax,
                        double *xiy, double *etay, double *sJ, double *nx,
                        double *ny, const double *Dm) {
#define V2(a, i, j) a[(i) + Nq * ((j) + Nq * e)]
#define S2(a, i, f) a[(i) + Nq * ((f) + 4 * e)]
#define DD(i, n) Dm[(i) + Nq * (n)]
  for (int64_t e = 0; e < nelem; e++) {
    for (int j = 0; j < Nq; j++)
      for (int i = 0; i < Nq; i++) {
        double xr = 0, xs = 0, yr = 0, ys = 0;
        for (int n = 0; n < Nq; n++) {
          xr += DD(i, n) * V2(x, n, j);
          xs += DD(j, n) * V2(x, i, n);
          yr += DD(i, n) * V2(y, n, j);
          ys += DD(j, n) * V2(y, i, n);
        }
        double Jv = xr * ys - yr * xs;
        V2(J, i, j) = Jv;
        V2(xix, i, j) = ys / Jv;
        V2(etax, i, j) = -yr / Jv;
        V2(xiy, i, j) = -xs / Jv;
        V2(etay, i, j) = xr / Jv;
      }
    for (int i = 0; i < Nq; i++) {
      S2(nx, i, 0) = -V2(J, 0, i) * V2(xix, 0, i);
      S2(ny, i, 0) = -V2(J, 0, i) * V2(xiy, 0, i);
      S2(nx, i, 1) = V2(J, Nq - 1, i) * V2(xix, Nq - 1, i);
      S2(ny, i, 1) = V2(J, Nq - 1, i) * V2(xiy, Nq - 1, i);
      S2(nx, i, 2) = -V2(J, i, 0) * V2(etax, i, 0);
      S2(ny, i, 2) = -V2(J, i, 0) * V2(etay, i, 0);
      S2(nx, i, 3) = V2(J, i, Nq - 1) * V2(etax, i, Nq - 1);
      S2(ny, i, 3) = V2(J, i, Nq - 1) * V2(etay, i, Nq - 1);
      for (int f = 0; f < 4; f++) {
        S2(sJ, i, f) = hypot(S2(nx, i, f), S2(ny, i, f));
        S2(nx, i, f) /= S2(sJ, i, f);
        S2(ny, i, f) /= S2(sJ, i, f);
      }
    }
  }
#undef V2
#undef S2
#undef DD
}

/* Julia Base n-argument hypot: maxabs * sqrt(sum(abs2(v / maxabs))) */
static double hypot3(double a, double b, double c) {
  double m = fabs(a);
  if (fabs(b) > m) m = fabs(b);
  if (fabs(c) > m) m = fabs(c);
  if (m == 0.0 || isinf(m)) return m;
  double p = a / m, q = b / m, s = c / m;
  return m * sqrt((p * p + q * q) + s * s);
}

/* computemetric! 3-D (curl-invariant form), metric.jl:230-400 */
void or_computemetric3d(int Nq, int64_t nelem, const double *x,
                        const double *y, const double *z, double *J,
                        double *xix, double *etax, double *zetax, double *xiy,
                        double *etay, double *zetay, double *xiz,
                        double *etaz, double *zetaz, double *sJ, double *nx,
                        double *ny, double *nz, const double *Dm) {
  int64_t Np = (int64_t)Nq * Nq * Nq;
  int nface = 6;
  double *JI2 = (double *)malloc(sizeof(double) * (size_t)Np);
  double *yzr = (double *)malloc(sizeof(double) * 9 * (size_t)Np);
  double *yzs = yzr + Np, *yzt = yzr + 2 * Np, *zxr = yzr + 3 * Np,
         *zxs = yzr + 4 * Np, *zxt = yzr + 5 * Np, *xyr = yzr + 6 * Np,
         *xys = yzr + 7 * Np, *xyt = yzr + 8 * Np;
#define L3(i, j, k) ((i) + Nq * ((j) + Nq * (k)))
#define V3(a, i, j, k) a[L3(i, j, k) + Np * e]
#define DD(i, n) Dm[(i) + Nq * (n)]
  for (int64_t q = 0; q < Np * nelem; q++) {
    xix[q] = 0; etax[q] = 0; zetax[q] = 0;
    xiy[q] = 0; etay[q] = 0; zetay[q] = 0;
    xiz[q] = 0; etaz[q] = 0; zetaz[q] = 0;
  }
  for (int64_t e = 0; e < nelem; e++) {
    for (int k = 0; k < Nq; k++)
      for (int j = 0; j < Nq; j++)
        for (int i = 0; i < Nq; i++) {
          double xr = 0, xs = 0, xt = 0, yr = 0, ys = 0, yt = 0, zr = 0, zs = 0, zt = 0;
          for (int n = 0; n < Nq; n++) {
            xr += DD(i, n) * V3(x, n, j, k);
            xs += DD(j, n) * V3(x, i, n, k);
            xt += DD(k, n) * V3(x, i, j, n);
            yr += DD(i, n) * V3(y, n, j, k);
            ys += DD(j, n) * V3(y, i, n, k);
            yt += DD(k, n) * V3(y, i, j, n);
            zr += DD(i, n) * V3(z, n, j, k);
            zs += DD(j, n) * V3(z, i, n, k);
            zt += DD(k, n) * V3(z, i, j, n);
          }
          double Jv = (xr * (ys * zt - zs * yt) + yr * (zs * xt - xs * zt)) +
                      zr * (xs * yt - ys * xt);
          V3(J, i, j, k) = Jv;
          int64_t l = L3(i, j, k);
          JI2[l] = 1.0 / (2.0 * Jv);
          double X = V3(x, i, j, k), Y = V3(y, i, j, k), Z = V3(z, i, j, k);
          yzr[l] = Y * zr - Z * yr;
          yzs[l] = Y * zs - Z * ys;
          yzt[l] = Y * zt - Z * yt;
          zxr[l] = Z * xr - X * zr;
          zxs[l] = Z * xs - X * zs;
          zxt[l] = Z * xt - X * zt;
          xyr[l] = X * yr - Y * xr;
          xys[l] = X * ys - Y * xs;
          xyt[l] = X * yt - Y * xt;
        }
    for (int k = 0; k < Nq; k++)
      for (int j = 0; j < Nq; j++)
        for (int i = 0; i < Nq; i++) {
          int64_t l = L3(i, j, k), g = l + Np * e;
          for (int n = 0; n < Nq; n++) {
            xix[g] += DD(j, n) * yzt[L3(i, n, k)];
            xix[g] -= DD(k, n) * yzs[L3(i, j, n)];
            etax[g] += DD(k, n) * yzr[L3(i, j, n)];
            etax[g] -= DD(i, n) * yzt[L3(n, j, k)];
            zetax[g] += DD(i, n) * yzs[L3(n, j, k)];
            zetax[g] -= DD(j, n) * yzr[L3(i, n, k)];
            xiy[g] += DD(j, n) * zxt[L3(i, n, k)];
            xiy[g] -= DD(k, n) * zxs[L3(i, j, n)];
            etay[g] += DD(k, n) * zxr[L3(i, j, n)];
            etay[g] -= DD(i, n) * zxt[L3(n, j, k)];
            zetay[g] += DD(i, n) * zxs[L3(n, j, k)];
            zetay[g] -= DD(j, n) * zxr[L3(i, n, k)];
            xiz[g] += DD(j, n) * xyt[L3(i, n, k)];
            xiz[g] -= DD(k, n) * xys[L3(i, j, n)];
            etaz[g] += DD(k, n) * xyr[L3(i, j, n)];
            etaz[g] -= DD(i, n) * xyt[L3(n, j, k)];
            zetaz[g] += DD(i, n) * xys[L3(n, j, k)];
            zetaz[g] -= DD(j, n) * xyr[L3(i, n, k)];
          }
          xix[g] *= JI2[l];
          etax[g] *= JI2[l];
          zetax[g] *= JI2[l];
          xiy[g] *= JI2[l];
          etay[g] *= JI2[l];
          zetay[g] *= JI2[l];
          xiz[g] *= JI2[l];
          etaz[g] *= JI2[l];
          zetaz[g] *= JI2[l];
        }
    int64_t Nq2 = (int64_t)Nq * Nq;
    for (int j = 0; j < Nq; j++)
      for (int i = 0; i < Nq; i++) {
        int64_t ije = i + Nq * j + e * nface * Nq2;
        int N1 = Nq - 1;
        nx[ije + 0 * Nq2] = -V3(J, 0, i, j) * V3(xix, 0, i, j);
        nx[ije + 1 * Nq2] = V3(J, N1, i, j) * V3(xix, N1, i, j);
        nx[ije + 2 * Nq2] = -V3(J, i, 0, j) * V3(etax, i, 0, j);
        nx[ije + 3 * Nq2] = V3(J, i, N1, j) * V3(etax, i, N1, j);
        nx[ije + 4 * Nq2] = -V3(J, i, j, 0) * V3(zetax, i, j, 0);
        nx[ije + 5 * Nq2] = V3(J, i, j, N1) * V3(zetax, i, j, N1);
        ny[ije + 0 * Nq2] = -V3(J, 0, i, j) * V3(xiy, 0, i, j);
        ny[ije + 1 * Nq2] = V3(J, N1, i, j) * V3(xiy, N1, i, j);
        ny[ije + 2 * Nq2] = -V3(J, i, 0, j) * V3(etay, i, 0, j);
        ny[ije + 3 * Nq2] = V3(J, i, N1, j) * V3(etay, i, N1, j);
        ny[ije + 4 * Nq2] = -V3(J, i, j, 0) * V3(zetay, i, j, 0);
        ny[ije + 5 * Nq2] = V3(J, i, j, N1) * V3(zetay, i, j, N1);
        nz[ije + 0 * Nq2] = -V3(J, 0, i, j) * V3(xiz, 0, i, j);
        nz[ije + 1 * Nq2] = V3(J, N1, i, j) * V3(xiz, N1, i, j);
        nz[ije + 2 * Nq2] = -V3(J, i, 0, j) * V3(etaz, i, 0, j);
        nz[ije + 3 * Nq2] = V3(J, i, N1, j) * V3(etaz, i, N1, j);
        nz[ije + 4 * Nq2] = -V3(J, i, j, 0) * V3(zetaz, i, j, 0);
        nz[ije + 5 * Nq2] = V3(J, i, j, N1) * V3(zetaz, i, j, N1);
        for (int n = 0; n < 6; n++) {
          int64_t q = ije + n * Nq2;
          sJ[q] = hypot3(nx[q], ny[q], nz[q]);
          nx[q] /= sJ[q];
          ny[q] /= sJ[q];
          nz[q] /= sJ[q];
        }
      }
  }
#undef L3
#undef V3
#undef DD
  free(JI2);
  free(yzr);
}

/* computegeometry of the set3c drivers: euler3d_set3c.jl:210-248 (3-D) and
 * euler2d_set3c.jl:171-208 (2-D).  vgeo is (Np, nvgeo, nelem), sgeo is
 * (nsgeo, Nfp, nface, nelem) with the field orders of :100-111. */
int or_computegeometry(int d, int N, int64_t nelem, const double *elemtocoord,
                       const int64_t *vmapM, int warp, double warp_amp,
                       double *vgeo, double *sgeo) {
  if (d != 2 && d != 3) return 1;
  int Nq = N + 1, nface = 2 * d;
  int64_t Np = d == 2 ? (int64_t)Nq * Nq : (int64_t)Nq * Nq * Nq;
  int64_t Nfp = d == 2 ? Nq : (int64_t)Nq * Nq;
  int nvgeo = d == 2 ? 8 : 14, nsgeo = d == 2 ? 4 : 5;
  double *r = (double *)malloc(sizeof(double) * Nq);
  double *w = (double *)malloc(sizeof(double) * Nq);
  double *Dm = (double *)malloc(sizeof(double) * Nq * Nq);
  if (or_lglpoints(N, r, w)) return 2;
  or_spectralderivative(Nq, r, Dm);
  int64_t nv = Np * nelem, ns = Nfp * nface * nelem;
  double *buf = (double *)calloc((size_t)(16 * nv + 5 * ns + 1), sizeof(double));
  double *X = buf, *Y = buf + nv, *Z = buf + 2 * nv, *J = buf + 3 * nv;
  double *m[9];
  for (int i = 0; i < 9; i++) m[i] = buf + (4 + i) * nv;
  double *sJ = buf + 16 * nv, *NX = sJ + ns, *NY = sJ + 2 * ns, *NZ = sJ + 3 * ns;
  or_creategrid(d, Nq, nelem, elemtocoord, r, X, Y, Z);
  for (int64_t q = 0; q < nv; q++) {
    if (warp == 1) {
      if (d == 3) {
        double s = sin(X[q]) * sin(Y[q]) * sin(Z[q]);
        double dx = warp_amp * s;
        X[q] = X[q] + dx;
        Y[q] = Y[q] + dx;
        Z[q] = Z[q] + dx;
      } else {
        double s = sin(X[q]) * sin(Y[q]);
        double dx = warp_amp * s;
        X[q] = X[q] + dx;
        Y[q] = Y[q] + dx;
      }
    }
  }
  if (d == 3)
    or_computemetric3d(Nq, nelem, X, Y, Z, J, m[0], m[1], m[2], m[3], m[4],
                       m[5], m[6], m[7], m[8], sJ, NX, NY, NZ, Dm);
  else
    or_computemetric2d(Nq, nelem, X, Y, J, m[0], m[1], m[2], m[3], sJ, NX, NY,
                       Dm);
  /* M = kron(1, ω, ω[, ω]) : M[p,q,r] = (ω[r]*ω[q])*ω[p] */
  double *M = (double *)malloc(sizeof(double) * Np);
  for (int64_t n = 0; n < Np; n++) {
    int p = n % Nq, q = (n / Nq) % Nq, rr = (int)(n / (Nq * Nq));
    M[n] = d == 3 ? (w[rr] * w[q]) * w[p] : w[q] * w[p];
  }
  int nmet = d == 2 ? 4 : 9;
  int fMJ = nmet, fMJI = nmet + 1, fx = nmet + 2;
  for (int64_t e = 0; e < nelem; e++)
    for (int64_t n = 0; n < Np; n++) {
      int64_t q = n + Np * e;
      double *vg = vgeo + Np * nvgeo * e;
      for (int f = 0; f < nmet; f++) vg[n + Np * f] = m[f][q];
      vg[n + Np * fMJ] = M[n] * J[q];
      vg[n + Np * fMJI] = 1.0 / vg[n + Np * fMJ];
      vg[n + Np * fx] = X[q];
      vg[n + Np * (fx + 1)] = Y[q];
      if (d == 3) vg[n + Np * (fx + 2)] = Z[q];
    }
  /* sM = kron(1, ω[, ω]) */
  for (int64_t e = 0; e < nelem; e++)
    for (int f = 0; f < nface; f++)
      for (int64_t n = 0; n < Nfp; n++) {
        int64_t q = n + Nfp * (f + nface * e);
        double sM = d == 3 ? w[n / Nq] * w[n % Nq] : w[n];
        double *sg = sgeo + nsgeo * q;
        sg[0] = NX[q];
        sg[1] = NY[q];
        if (d == 3) sg[2] = NZ[q];
        sg[d] = sM * sJ[q];
        int64_t idM = vmapM[q] - 1;
        int64_t eM = idM / Np, vM = idM % Np;
        sg[d + 1] = vgeo[vM + Np * (fMJI + nvgeo * eM)];
      }
  free(M);
  free(buf);
  free(r);
  free(w);
  free(Dm);
  return 0;
}

/* ===================================================================== */
/* set3c Euler: volumerhs!, fluxrhs!, updatesolution!                    */
/* ===================================================================== */

#define EOS(p) ((p)->R_gas / (p)->c_v)

/* volumerhs! 3-D (euler3d_set3c.jl:253-339) and 2-D (euler2d_set3c.jl:214-279) */
void or_volumerhs(int d, int N, double *rhs, const double *Q,
                  const double *vgeo, const double *Dm, int64_t nelem,
                  const or_phys *p, int nthreads) {
  const int Nq = N + 1;
  const double gam = p->gamma, eos = EOS(p), grav = p->gravity;
  (void)gam;
  if (d == 3) {
    const int64_t Np = (int64_t)Nq * Nq * Nq;
    const int ns = 5, nvg = 14;
#pragma omp parallel OMP_THREADS(nthreads)
    {
      double *sF = (double *)malloc(sizeof(double) * 3 * ns * Np);
      double *sG = sF + ns * Np, *sH = sG + ns * Np;
#pragma omp for schedule(static)
      for (int64_t e = 0; e < nelem; e++) {
        const double *q = Q + Np * ns * e;
        const double *vg = vgeo + Np * nvg * e;
        double *r = rhs + Np * ns * e;
        for (int64_t n = 0; n < Np; n++) {
          double MJ = vg[n + Np * 9];
          double xx = vg[n], ex = vg[n + Np], zx = vg[n + 2 * Np];
          double xy = vg[n + 3 * Np], ey = vg[n + 4 * Np], zy = vg[n + 5 * Np];
          double xz = vg[n + 6 * Np], ez = vg[n + 7 * Np], zz = vg[n + 8 * Np];
          double zc = vg[n + 13 * Np];
          double U = q[n], V = q[n + Np], W = q[n + 2 * Np];
          double rho = q[n + 3 * Np], E = q[n + 4 * Np];
          double P = eos * ((E - ((U * U + V * V) + W * W) / (2.0 * rho)) - rho * grav * zc);
          double ri = 1.0 / rho;
          double fr[3] = {U, V, W};
          double fU[3] = {ri * U * U + P, ri * U * V, ri * U * W};
          double fV[3] = {ri * V * U, ri * V * V + P, ri * V * W};
          double fW[3] = {ri * W * U, ri * W * V, ri * W * W + P};
          double fE[3] = {ri * U * (E + P), ri * V * (E + P), ri * W * (E + P)};
          const double *fl[5] = {fU, fV, fW, fr, fE}; /* state order U,V,W,ρ,E */
          for (int s = 0; s < ns; s++) {
            const double *f = fl[s];
            sF[n + Np * s] = MJ * ((xx * f[0] + xy * f[1]) + xz * f[2]);
            sG[n + Np * s] = MJ * ((ex * f[0] + ey * f[1]) + ez * f[2]);
            sH[n + Np * s] = MJ * ((zx * f[0] + zy * f[1]) + zz * f[2]);
          }
          r[n + Np * 2] -= MJ * rho * grav;
        }
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  r[i + Nq * (j + Nq * k) + Np * s] +=
                      Dm[n + Nq * i] * sF[n + Nq * (j + Nq * k) + Np * s];
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  r[i + Nq * (j + Nq * k) + Np * s] +=
                      Dm[n + Nq * j] * sG[i + Nq * (n + Nq * k) + Np * s];
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  r[i + Nq * (j + Nq * k) + Np * s] +=
                      Dm[n + Nq * k] * sH[i + Nq * (j + Nq * n) + Np * s];
      }
      free(sF);
    }
  } else {
    const int64_t Np = (int64_t)Nq * Nq;
    const int ns = 4, nvg = 8;
#pragma omp parallel OMP_THREADS(nthreads)
    {
      double *sF = (double *)malloc(sizeof(double) * 2 * ns * Np);
      double *sG = sF + ns * Np;
#pragma omp for schedule(static)
      for (int64_t e = 0; e < nelem; e++) {
        const double *q = Q + Np * ns * e;
        const double *vg = vgeo + Np * nvg * e;
        double *r = rhs + Np * ns * e;
        for (int64_t n = 0; n < Np; n++) {
          double MJ = vg[n + Np * 4];
          double xx = vg[n], ex = vg[n + Np], xy = vg[n + 2 * Np], ey = vg[n + 3 * Np];
          double yc = vg[n + 7 * Np];
          double U = q[n], V = q[n + Np], rho = q[n + 2 * Np], E = q[n + 3 * Np];
          double P = eos * ((E - (U * U + V * V) / (2.0 * rho)) - rho * grav * yc);
          double ri = 1.0 / rho;
          double fr[2] = {U, V};
          double fU[2] = {ri * U * U + P, ri * U * V};
          double fV[2] = {ri * V * U, ri * V * V + P};
          double fE[2] = {ri * U * (E + P), ri * V * (E + P)};
          const double *fl[4] = {fU, fV, fr, fE}; /* state order U,V,ρ,E */
          for (int s = 0; s < ns; s++) {
            const double *f = fl[s];
            sF[n + Np * s] = MJ * (xx * f[0] + xy * f[1]);
            sG[n + Np * s] = MJ * (ex * f[0] + ey * f[1]);
          }
          r[n + Np * 1] -= MJ * rho * grav;
        }
        for (int s = 0; s < ns; s++)
          for (int j = 0; j < Nq; j++)
            for (int i = 0; i < Nq; i++)
              for (int k = 0; k < Nq; k++)
                r[i + Nq * j + Np * s] += Dm[k + Nq * i] * sF[k + Nq * j + Np * s];
        for (int s = 0; s < ns; s++)
          for (int j = 0; j < Nq; j++)
            for (int i = 0; i < Nq; i++)
              for (int k = 0; k < Nq; k++)
                r[i + Nq * j + Np * s] += Dm[k + Nq * j] * sG[i + Nq * k + Np * s];
      }
      free(sF);
    }
  }
}

/* Euler flux components of the set3c formulation for one state.
 * f[s][c]: state s (reference order), direction c. */
static void euler_flux3(double U, double V, double W, double rho, double E,
                        double P, double f[5][3]) {
  double ri = 1.0 / rho;
  f[3][0] = U; f[3][1] = V; f[3][2] = W;
  f[0][0] = ri * U * U + P; f[0][1] = ri * U * V; f[0][2] = ri * U * W;
  f[1][0] = ri * V * U; f[1][1] = ri * V * V + P; f[1][2] = ri * V * W;
  f[2][0] = ri * W * U; f[2][1] = ri * W * V; f[2][2] = ri * W * W + P;
  f[4][0] = ri * U * (E + P); f[4][1] = ri * V * (E + P); f[4][2] = ri * W * (E + P);
}

/* fluxrhs! 3-D (euler3d_set3c.jl:342-458) and 2-D (euler2d_set3c.jl:282-377).
 * Returns 0, or 1 if a face carries a boundary code other than 0 or 1. */
int or_fluxrhs(int d, int N, double *rhs, const double *Q, const double *sgeo,
               const double *vgeo, int64_t nelem, const int64_t *vmapM,
               const int64_t *vmapP, const int64_t *elemtobndy,
               const or_phys *p, int nthreads) {
  const int Nq = N + 1, nface = 2 * d;
  const double gam = p->gamma, eos = EOS(p), grav = p->gravity;
  int bad = 0;
  if (d == 3) {
    const int64_t Np = (int64_t)Nq * Nq * Nq, Nfp = (int64_t)Nq * Nq;
    const int ns = 5, nvg = 14, nsg = 5;
#pragma omp parallel for schedule(static) OMP_THREADS(nthreads) reduction(| : bad)
    for (int64_t e = 0; e < nelem; e++) {
      for (int f = 0; f < nface; f++) {
        for (int64_t n = 0; n < Nfp; n++) {
          const double *sg = sgeo + nsg * (n + Nfp * (f + nface * e));
          double nxM = sg[0], nyM = sg[1], nzM = sg[2], sMJ = sg[3];
          int64_t idM = vmapM[n + Nfp * (f + nface * e)];
          int64_t idP = vmapP[n + Nfp * (f + nface * e)];
          int64_t eM = e, eP = (idP - 1) / Np;
          int64_t vM = (idM - 1) % Np, vP = (idP - 1) % Np;
          const double *qM = Q + Np * ns * eM, *qP = Q + Np * ns * eP;
          double rhoM = qM[vM + 3 * Np], UM = qM[vM], VM = qM[vM + Np],
                 WM = qM[vM + 2 * Np], EM = qM[vM + 4 * Np];
          double zM = vgeo[vM + Np * (13 + nvg * eM)];
          int64_t bc = elemtobndy[f + nface * e];
          double PM = eos * ((EM - ((UM * UM + VM * VM) + WM * WM) / (2.0 * rhoM)) - rhoM * grav * zM);
          double rhoP, UP, VP, WP, EP, PP;
          if (bc == 0) {
            rhoP = qP[vP + 3 * Np]; UP = qP[vP]; VP = qP[vP + Np];
            WP = qP[vP + 2 * Np]; EP = qP[vP + 4 * Np];
            double zP = vgeo[vP + Np * (13 + nvg * eP)];
            PP = eos * ((EP - ((UP * UP + VP * VP) + WP * WP) / (2.0 * rhoP)) - rhoP * grav * zP);
          } else if (bc == 1) {
            double UnM = (nxM * UM + nyM * VM) + nzM * WM;
            UP = UM - 2.0 * UnM * nxM;
            VP = VM - 2.0 * UnM * nyM;
            WP = WM - 2.0 * UnM * nzM;
            rhoP = rhoM; EP = EM; PP = PM;
          } else {
            bad = 1;
            continue;
          }
          double fM[5][3], fP[5][3];
          euler_flux3(UM, VM, WM, rhoM, EM, PM, fM);
          euler_flux3(UP, VP, WP, rhoP, EP, PP, fP);
          double rMi = 1.0 / rhoM, rPi = 1.0 / rhoP;
          double lM = rMi * fabs((nxM * UM + nyM * VM) + nzM * WM) + sqrt(rMi * gam * PM);
          double lP = rPi * fabs((nxM * UP + nyM * VP) + nzM * WP) + sqrt(rPi * gam * PP);
          double lam = lM > lP ? lM : lP;
          if (isnan(lM) || isnan(lP)) lam = NAN;
          double qMv[5] = {UM, VM, WM, rhoM, EM}, qPv[5] = {UP, VP, WP, rhoP, EP};
          double *r = rhs + Np * ns * eM;
          for (int s = 0; s < ns; s++) {
            double fs = (((nxM * (fM[s][0] + fP[s][0]) + nyM * (fM[s][1] + fP[s][1])) +
                          nzM * (fM[s][2] + fP[s][2])) -
                         lam * (qPv[s] - qMv[s])) / 2.0;
            r[vM + Np * s] -= sMJ * fs;
          }
        }
      }
    }
  } else {
    const int64_t Np = (int64_t)Nq * Nq, Nfp = Nq;
    const int ns = 4, nvg = 8, nsg = 4;
#pragma omp parallel for schedule(static) OMP_THREADS(nthreads) reduction(| : bad)
    for (int64_t e = 0; e < nelem; e++) {
      for (int f = 0; f < nface; f++) {
        for (int64_t n = 0; n < Nfp; n++) {
          const double *sg = sgeo + nsg * (n + Nfp * (f + nface * e));
          double nxM = sg[0], nyM = sg[1], sMJ = sg[2];
          int64_t idM = vmapM[n + Nfp * (f + nface * e)];
          int64_t idP = vmapP[n + Nfp * (f + nface * e)];
          int64_t eM = e, eP = (idP - 1) / Np;
          int64_t vM = (idM - 1) % Np, vP = (idP - 1) % Np;
          const double *qM = Q + Np * ns * eM, *qP = Q + Np * ns * eP;
          double rhoM = qM[vM + 2 * Np], UM = qM[vM], VM = qM[vM + Np], EM = qM[vM + 3 * Np];
          double yM = vgeo[vM + Np * (7 + nvg * eM)];
          double PM = eos * ((EM - (UM * UM + VM * VM) / (2.0 * rhoM)) - rhoM * grav * yM);
          int64_t bc = elemtobndy[f + nface * e];
          double rhoP, UP, VP, EP, PP;
          if (bc == 0) {
            rhoP = qP[vP + 2 * Np]; UP = qP[vP]; VP = qP[vP + Np]; EP = qP[vP + 3 * Np];
            double yP = vgeo[vP + Np * (7 + nvg * eP)];
            PP = eos * ((EP - (UP * UP + VP * VP) / (2.0 * rhoP)) - rhoP * grav * yP);
          } else if (bc == 1) {
            double UnM = nxM * UM + nyM * VM;
            UP = UM - 2.0 * UnM * nxM;
            VP = VM - 2.0 * UnM * nyM;
            rhoP = rhoM; EP = EM; PP = PM;
          } else {
            bad = 1;
            continue;
          }
          double rMi = 1.0 / rhoM, rPi = 1.0 / rhoP;
          double fM[4][2] = {{rMi * UM * UM + PM, rMi * UM * VM},
                             {rMi * VM * UM, rMi * VM * VM + PM},
                             {UM, VM},
                             {rMi * UM * (EM + PM), rMi * VM * (EM + PM)}};
          double fP[4][2] = {{rPi * UP * UP + PP, rPi * UP * VP},
                             {rPi * VP * UP, rPi * VP * VP + PP},
                             {UP, VP},
                             {rPi * UP * (EP + PP), rPi * VP * (EP + PP)}};
          double lM = rMi * fabs(nxM * UM + nyM * VM) + sqrt(rMi * gam * PM);
          double lP = rPi * fabs(nxM * UP + nyM * VP) + sqrt(rPi * gam * PP);
          double lam = lM > lP ? lM : lP;
          if (isnan(lM) || isnan(lP)) lam = NAN;
          double qMv[4] = {UM, VM, rhoM, EM}, qPv[4] = {UP, VP, rhoP, EP};
          double *r = rhs + Np * ns * eM;
          for (int s = 0; s < ns; s++) {
            double fs = ((nxM * (fM[s][0] + fP[s][0]) + nyM * (fM[s][1] + fP[s][1])) -
                         lam * (qPv[s] - qMv[s])) / 2.0;
            r[vM + Np * s] -= sMJ * fs;
          }
        }
      }
    }
  }
  return bad;
}

/* updatesolution!, euler3d_set3c.jl:862-872 / nse2d.jl:806-814.
 * rhs_gradQ (Np, nstate, dim, nelem) may be NULL for the inviscid form, in
 * which case the `visc*rhs_gradQ` term (zero in the reference) is skipped. */
void or_updatesolution(int d, int N, double *rhs, const double *rhs_gradQ,
                       double *Q, const double *vgeo, int64_t nelem,
                       double rka, double rkb, double dt, double visc,
                       int nthreads) {
  const int Nq = N + 1;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int ns = d == 3 ? 5 : 4, nvg = d == 3 ? 14 : 8, fMJI = d == 3 ? 10 : 5;
#pragma omp parallel for schedule(static) OMP_THREADS(nthreads)
  for (int64_t e = 0; e < nelem; e++)
    for (int s = 0; s < ns; s++)
      for (int64_t i = 0; i < Np; i++) {
        int64_t q = i + Np * (s + ns * e);
        if (rhs_gradQ) rhs[q] += visc * rhs_gradQ[i + Np * (s + ns * d * e)];
        Q[q] += rkb * dt * rhs[q] * vgeo[i + Np * (fMJI + nvg * e)];
        rhs[q] *= rka;
      }
}

/* ===================================================================== */
/* nse LDG viscous passes                                                */
/* ===================================================================== */

/* volume_grad!, nse2d.jl:396-463 / nse3d.jl:475-562.
 * rhs is (Np, nstate, dim, nelem) and is zeroed first. */
void or_volume_grad(int d, int N, double *rhs, const double *Q,
                    const double *vgeo, const double *Dm, int64_t nelem,
                    const or_phys *p, int nthreads) {
  const int Nq = N + 1;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int ns = d == 3 ? 5 : 4, nvg = d == 3 ? 14 : 8;
  const double eos = EOS(p), grav = p->gravity, Rg = p->R_gas;
  for (int64_t q = 0; q < Np * ns * d * nelem; q++) rhs[q] = 0.0;
#pragma omp parallel OMP_THREADS(nthreads)
  {
    /* s_X[n, s, c] for reference direction X and physical component c */
    double *sF = (double *)malloc(sizeof(double) * 3 * ns * 3 * Np);
    double *sG = sF + ns * 3 * Np, *sH = sG + ns * 3 * Np;
#pragma omp for schedule(static)
    for (int64_t e = 0; e < nelem; e++) {
      const double *q = Q + Np * ns * e;
      const double *vg = vgeo + Np * nvg * e;
      double *r = rhs + Np * ns * d * e;
      for (int64_t n = 0; n < Np; n++) {
        double flux[5];
        double met[3][3]; /* met[dir][comp] */
        double MJ;
        if (d == 3) {
          MJ = vg[n + Np * 9];
          met[0][0] = vg[n]; met[1][0] = vg[n + Np]; met[2][0] = vg[n + 2 * Np];
          met[0][1] = vg[n + 3 * Np]; met[1][1] = vg[n + 4 * Np]; met[2][1] = vg[n + 5 * Np];
          met[0][2] = vg[n + 6 * Np]; met[1][2] = vg[n + 7 * Np]; met[2][2] = vg[n + 8 * Np];
          double zc = vg[n + 13 * Np];
          double U = q[n], V = q[n + Np], W = q[n + 2 * Np], rho = q[n + 3 * Np], E = q[n + 4 * Np];
          double P = eos * ((E - ((U * U + V * V) + W * W) / (2.0 * rho)) - rho * grav * zc);
          flux[3] = rho; flux[0] = U / rho; flux[1] = V / rho; flux[2] = W / rho;
          flux[4] = P / (Rg * rho);
        } else {
          MJ = vg[n + Np * 4];
          met[0][0] = vg[n]; met[1][0] = vg[n + Np];
          met[0][1] = vg[n + 2 * Np]; met[1][1] = vg[n + 3 * Np];
          double yc = vg[n + 7 * Np];
          double U = q[n], V = q[n + Np], rho = q[n + 2 * Np], E = q[n + 3 * Np];
          double P = eos * ((E - (U * U + V * V) / (2.0 * rho)) - rho * grav * yc);
          flux[2] = rho; flux[0] = U / rho; flux[1] = V / rho; flux[3] = P / (Rg * rho);
        }
        for (int s = 0; s < ns; s++)
          for (int c = 0; c < d; c++) {
            sF[n + Np * (s + ns * c)] = MJ * (met[0][c] * flux[s]);
            sG[n + Np * (s + ns * c)] = MJ * (met[1][c] * flux[s]);
            if (d == 3) sH[n + Np * (s + ns * c)] = MJ * (met[2][c] * flux[s]);
          }
      }
      if (d == 3) {
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  for (int c = 0; c < 3; c++)
                    r[i + Nq * (j + Nq * k) + Np * (s + ns * c)] -=
                        Dm[n + Nq * i] * sF[n + Nq * (j + Nq * k) + Np * (s + ns * c)];
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  for (int c = 0; c < 3; c++)
                    r[i + Nq * (j + Nq * k) + Np * (s + ns * c)] -=
                        Dm[n + Nq * j] * sG[i + Nq * (n + Nq * k) + Np * (s + ns * c)];
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  for (int c = 0; c < 3; c++)
                    r[i + Nq * (j + Nq * k) + Np * (s + ns * c)] -=
                        Dm[n + Nq * k] * sH[i + Nq * (j + Nq * n) + Np * (s + ns * c)];
      } else {
        for (int s = 0; s < ns; s++)
          for (int j = 0; j < Nq; j++)
            for (int i = 0; i < Nq; i++)
              for (int n = 0; n < Nq; n++)
                for (int c = 0; c < 2; c++)
                  r[i + Nq * j + Np * (s + ns * c)] -=
                      Dm[n + Nq * i] * sF[n + Nq * j + Np * (s + ns * c)];
        for (int s = 0; s < ns; s++)
          for (int j = 0; j < Nq; j++)
            for (int i = 0; i < Nq; i++)
              for (int n = 0; n < Nq; n++)
                for (int c = 0; c < 2; c++)
                  r[i + Nq * j + Np * (s + ns * c)] -=
                      Dm[n + Nq * j] * sG[i + Nq * n + Np * (s + ns * c)];
      }
    }
    free(sF);
  }
}

/* flux_grad!, nse2d.jl:467-557 / nse3d.jl:566-672 */
int or_flux_grad(int d, int N, double *rhs, const double *Q,
                 const double *sgeo, const double *vgeo, int64_t nelem,
                 const int64_t *vmapM, const int64_t *vmapP,
                 const int64_t *elemtobndy, const or_phys *p, int nthreads) {
  const int Nq = N + 1, nface = 2 * d;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int64_t Nfp = d == 3 ? (int64_t)Nq * Nq : Nq;
  const int ns = d == 3 ? 5 : 4, nvg = d == 3 ? 14 : 8, nsg = d == 3 ? 5 : 4;
  const double eos = EOS(p), grav = p->gravity, Rg = p->R_gas;
  const int irho = d == 3 ? 3 : 2, iE = d == 3 ? 4 : 3, igc = d == 3 ? 13 : 7;
  int bad = 0;
#pragma omp parallel for schedule(static) OMP_THREADS(nthreads) reduction(| : bad)
  for (int64_t e = 0; e < nelem; e++)
    for (int f = 0; f < nface; f++)
      for (int64_t n = 0; n < Nfp; n++) {
        const double *sg = sgeo + nsg * (n + Nfp * (f + nface * e));
        double nrm[3] = {sg[0], sg[1], d == 3 ? sg[2] : 0.0};
        double sMJ = sg[d];
        int64_t idM = vmapM[n + Nfp * (f + nface * e)];
        int64_t idP = vmapP[n + Nfp * (f + nface * e)];
        int64_t eP = (idP - 1) / Np, vM = (idM - 1) % Np, vP = (idP - 1) % Np;
        const double *qM = Q + Np * ns * e, *qP = Q + Np * ns * eP;
        double mom[3] = {qM[vM], qM[vM + Np], d == 3 ? qM[vM + 2 * Np] : 0.0};
        double rhoM = qM[vM + irho * Np], EM = qM[vM + iE * Np];
        double gcM = vgeo[vM + Np * (igc + nvg * e)];
        double ke = d == 3 ? (mom[0] * mom[0] + mom[1] * mom[1]) + mom[2] * mom[2]
                           : mom[0] * mom[0] + mom[1] * mom[1];
        double PM = eos * ((EM - ke / (2.0 * rhoM)) - rhoM * grav * gcM);
        double fluxM[5], fluxP[5];
        /* primitive (u, v, [w], ρ, T) in state slots */
        for (int c = 0; c < d; c++) fluxM[c] = mom[c] / rhoM;
        fluxM[irho] = rhoM;
        double TM = PM / (Rg * rhoM);
        fluxM[iE] = TM;
        int64_t bc = elemtobndy[f + nface * e];
        if (bc == 0) {
          double momP[3] = {qP[vP], qP[vP + Np], d == 3 ? qP[vP + 2 * Np] : 0.0};
          double rhoP = qP[vP + irho * Np], EP = qP[vP + iE * Np];
          double gcP = vgeo[vP + Np * (igc + nvg * eP)];
          double keP = d == 3 ? (momP[0] * momP[0] + momP[1] * momP[1]) + momP[2] * momP[2]
                              : momP[0] * momP[0] + momP[1] * momP[1];
          double PP = eos * ((EP - keP / (2.0 * rhoP)) - rhoP * grav * gcP);
          for (int c = 0; c < d; c++) fluxP[c] = momP[c] / rhoP;
          fluxP[irho] = rhoP;
          fluxP[iE] = PP / (Rg * rhoP);
        } else if (bc == 1) {
          double UnM = d == 3 ? (nrm[0] * mom[0] + nrm[1] * mom[1]) + nrm[2] * mom[2]
                              : nrm[0] * mom[0] + nrm[1] * mom[1];
          for (int c = 0; c < d; c++) fluxP[c] = (mom[c] - 2.0 * UnM * nrm[c]) / rhoM;
          fluxP[irho] = rhoM;
          fluxP[iE] = TM;
        } else {
          bad = 1;
          continue;
        }
        double *r = rhs + Np * ns * d * e;
        for (int s = 0; s < ns; s++) {
          double fs = 0.5 * (fluxM[s] + fluxP[s]);
          for (int c = 0; c < d; c++) r[vM + Np * (s + ns * c)] += sMJ * nrm[c] * fs;
        }
      }
  return bad;
}

/* update_gradQ!, nse2d.jl:769-778 */
void or_update_gradQ(int d, int N, double *gradQ, const double *rhs,
                     const double *vgeo, int64_t nelem, int nthreads) {
  const int Nq = N + 1;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int ns = d == 3 ? 5 : 4, nvg = d == 3 ? 14 : 8, fMJI = d == 3 ? 10 : 5;
#pragma omp parallel for schedule(static) OMP_THREADS(nthreads)
  for (int64_t e = 0; e < nelem; e++)
    for (int s = 0; s < ns; s++)
      for (int64_t i = 0; i < Np; i++)
        for (int c = 0; c < d; c++) {
          int64_t q = i + Np * (s + ns * (c + d * e));
          gradQ[q] = rhs[q] * vgeo[i + Np * (fMJI + nvg * e)];
        }
}

/* Viscous flux of the nse drivers for one node (nse3d.jl:717-742,
 * nse2d.jl:598-614).  g[s][c] is gradQ (state slot s, component c) holding
 * grad(u, v, [w], ρ, T); vel = (u, v, [w]).  out[s][c]. */
static void visc_flux(int d, const double g[5][3], const double *vel,
                      const or_phys *p, double out[5][3]) {
  const double lam = p->lambda, cpPr = p->c_p / p->Pr;
  if (d == 3) {
    double ux = g[0][0], uy = g[0][1], uz = g[0][2];
    double vx = g[1][0], vy = g[1][1], vz = g[1][2];
    double wx = g[2][0], wy = g[2][1], wz = g[2][2];
    double Tx = g[4][0], Ty = g[4][1], Tz = g[4][2];
    double div_u = (ux + vy) + wz;
    double u = vel[0], v = vel[1], w = vel[2];
    out[3][0] = 0.0 * g[3][0]; out[3][1] = 0.0 * g[3][1]; out[3][2] = 0.0 * g[3][2];
    out[0][0] = 2.0 * ux + lam * div_u; out[0][1] = uy + vx; out[0][2] = uz + wx;
    out[1][0] = vx + uy; out[1][1] = 2.0 * vy + lam * div_u; out[1][2] = vz + wy;
    out[2][0] = wx + uz; out[2][1] = wy + vz; out[2][2] = 2.0 * wz + lam * div_u;
    out[4][0] = ((u * (2.0 * ux + lam * div_u) + v * (uy + vx)) + w * (uz + wx)) + cpPr * Tx;
    out[4][1] = ((u * (vx + uy) + v * (2.0 * vy + lam * div_u)) + w * (vz + wy)) + cpPr * Ty;
    out[4][2] = ((u * (wx + uz) + v * (wy + vz)) + w * (2.0 * wz + lam * div_u)) + cpPr * Tz;
  } else {
    double ux = g[0][0], uy = g[0][1], vx = g[1][0], vy = g[1][1];
    double Tx = g[3][0], Ty = g[3][1];
    double div_u = ux + vy;
    double u = vel[0], v = vel[1];
    out[2][0] = 0.0 * g[2][0]; out[2][1] = 0.0 * g[2][1];
    out[0][0] = 2.0 * ux + lam * div_u; out[0][1] = uy + vx;
    out[1][0] = vx + uy; out[1][1] = 2.0 * vy + lam * div_u;
    out[3][0] = (u * (2.0 * ux + lam * div_u) + v * (uy + vx)) + cpPr * Tx;
    out[3][1] = (u * (vx + uy) + v * (2.0 * vy + lam * div_u)) + cpPr * Ty;
  }
}

/* volume_div!, nse2d.jl:561-636 / nse3d.jl:676-776.  rhs (Np,ns,dim,nelem)
 * is zeroed; only component slot 1 is written. */
void or_volume_div(int d, int N, double *rhs, const double *gradQ,
                   const double *Q, const double *vgeo, const double *Dm,
                   int64_t nelem, const or_phys *p, int nthreads) {
  const int Nq = N + 1;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int ns = d == 3 ? 5 : 4, nvg = d == 3 ? 14 : 8;
  const int irho = d == 3 ? 3 : 2;
  for (int64_t q = 0; q < Np * ns * d * nelem; q++) rhs[q] = 0.0;
#pragma omp parallel OMP_THREADS(nthreads)
  {
    double *sF = (double *)malloc(sizeof(double) * 3 * ns * Np);
    double *sG = sF + ns * Np, *sH = sG + ns * Np;
#pragma omp for schedule(static)
    for (int64_t e = 0; e < nelem; e++) {
      const double *vg = vgeo + Np * nvg * e;
      const double *gq = gradQ + Np * ns * d * e;
      const double *q = Q + Np * ns * e;
      double *r = rhs + Np * ns * d * e;
      for (int64_t n = 0; n < Np; n++) {
        double g[5][3], out[5][3], vel[3], met[3][3], MJ;
        for (int s = 0; s < ns; s++)
          for (int c = 0; c < d; c++) g[s][c] = gq[n + Np * (s + ns * c)];
        double rho = q[n + irho * Np];
        for (int c = 0; c < d; c++) vel[c] = q[n + c * Np] / rho;
        if (d == 3) {
          MJ = vg[n + Np * 9];
          met[0][0] = vg[n]; met[1][0] = vg[n + Np]; met[2][0] = vg[n + 2 * Np];
          met[0][1] = vg[n + 3 * Np]; met[1][1] = vg[n + 4 * Np]; met[2][1] = vg[n + 5 * Np];
          met[0][2] = vg[n + 6 * Np]; met[1][2] = vg[n + 7 * Np]; met[2][2] = vg[n + 8 * Np];
        } else {
          MJ = vg[n + Np * 4];
          met[0][0] = vg[n]; met[1][0] = vg[n + Np];
          met[0][1] = vg[n + 2 * Np]; met[1][1] = vg[n + 3 * Np];
        }
        visc_flux(d, g, vel, p, out);
        for (int s = 0; s < ns; s++) {
          if (d == 3) {
            sF[n + Np * s] = MJ * ((met[0][0] * out[s][0] + met[0][1] * out[s][1]) + met[0][2] * out[s][2]);
            sG[n + Np * s] = MJ * ((met[1][0] * out[s][0] + met[1][1] * out[s][1]) + met[1][2] * out[s][2]);
            sH[n + Np * s] = MJ * ((met[2][0] * out[s][0] + met[2][1] * out[s][1]) + met[2][2] * out[s][2]);
          } else {
            sF[n + Np * s] = MJ * (met[0][0] * out[s][0] + met[0][1] * out[s][1]);
            sG[n + Np * s] = MJ * (met[1][0] * out[s][0] + met[1][1] * out[s][1]);
          }
        }
      }
      if (d == 3) {
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  r[i + Nq * (j + Nq * k) + Np * s] -= Dm[n + Nq * i] * sF[n + Nq * (j + Nq * k) + Np * s];
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  r[i + Nq * (j + Nq * k) + Np * s] -= Dm[n + Nq * j] * sG[i + Nq * (n + Nq * k) + Np * s];
        for (int s = 0; s < ns; s++)
          for (int k = 0; k < Nq; k++)
            for (int j = 0; j < Nq; j++)
              for (int i = 0; i < Nq; i++)
                for (int n = 0; n < Nq; n++)
                  r[i + Nq * (j + Nq * k) + Np * s] -= Dm[n + Nq * k] * sH[i + Nq * (j + Nq * n) + Np * s];
      } else {
        for (int s = 0; s < ns; s++)
          for (int j = 0; j < Nq; j++)
            for (int i = 0; i < Nq; i++)
              for (int n = 0; n < Nq; n++)
                r[i + Nq * j + Np * s] -= Dm[n + Nq * i] * sF[n + Nq * j + Np * s];
        for (int s = 0; s < ns; s++)
          for (int j = 0; j < Nq; j++)
            for (int i = 0; i < Nq; i++)
              for (int n = 0; n < Nq; n++)
                r[i + Nq * j + Np * s] -= Dm[n + Nq * j] * sG[i + Nq * n + Np * s];
      }
    }
    free(sF);
  }
}

/* flux_div!, nse2d.jl:640-765 / nse3d.jl:780-955 */
int or_flux_div(int d, int N, double *rhs, const double *gradQ,
                const double *Q, const double *sgeo, int64_t nelem,
                const int64_t *vmapM, const int64_t *vmapP,
                const int64_t *elemtobndy, const or_phys *p, int nthreads) {
  const int Nq = N + 1, nface = 2 * d;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int64_t Nfp = d == 3 ? (int64_t)Nq * Nq : Nq;
  const int ns = d == 3 ? 5 : 4, nsg = d == 3 ? 5 : 4;
  const int irho = d == 3 ? 3 : 2;
  int bad = 0;
#pragma omp parallel for schedule(static) OMP_THREADS(nthreads) reduction(| : bad)
  for (int64_t e = 0; e < nelem; e++)
    for (int f = 0; f < nface; f++)
      for (int64_t n = 0; n < Nfp; n++) {
        const double *sg = sgeo + nsg * (n + Nfp * (f + nface * e));
        double nrm[3] = {sg[0], sg[1], d == 3 ? sg[2] : 0.0};
        double sMJ = sg[d];
        int64_t idM = vmapM[n + Nfp * (f + nface * e)];
        int64_t idP = vmapP[n + Nfp * (f + nface * e)];
        int64_t eP = (idP - 1) / Np, vM = (idM - 1) % Np, vP = (idP - 1) % Np;
        const double *gM = gradQ + Np * ns * d * e, *gP = gradQ + Np * ns * d * eP;
        const double *qM = Q + Np * ns * e, *qP = Q + Np * ns * eP;
        double gm[5][3], gp[5][3], velM[3], velP[3];
        for (int s = 0; s < ns; s++)
          for (int c = 0; c < d; c++) gm[s][c] = gM[vM + Np * (s + ns * c)];
        double rhoM = qM[vM + irho * Np];
        for (int c = 0; c < d; c++) velM[c] = qM[vM + c * Np] / rhoM;
        int64_t bc = elemtobndy[f + nface * e];
        if (bc == 0) {
          for (int s = 0; s < ns; s++)
            for (int c = 0; c < d; c++) gp[s][c] = gP[vP + Np * (s + ns * c)];
          double rhoP = qP[vP + irho * Np];
          for (int c = 0; c < d; c++) velP[c] = qP[vP + c * Np] / rhoP;
        } else if (bc == 1) {
          for (int s = 0; s < ns; s++) {
            double sn = d == 3 ? (nrm[0] * gm[s][0] + nrm[1] * gm[s][1]) + nrm[2] * gm[s][2]
                               : nrm[0] * gm[s][0] + nrm[1] * gm[s][1];
            for (int c = 0; c < d; c++) gp[s][c] = gm[s][c] - 2.0 * sn * nrm[c];
          }
          double un = d == 3 ? (nrm[0] * velM[0] + nrm[1] * velM[1]) + nrm[2] * velM[2]
                             : nrm[0] * velM[0] + nrm[1] * velM[1];
          for (int c = 0; c < d; c++) velP[c] = velM[c] - 2.0 * un * nrm[c];
          /* temperature gradient copied from the interior (nse3d.jl:898) */
          for (int c = 0; c < d; c++) gp[ns - 1][c] = gm[ns - 1][c];
        } else {
          bad = 1;
          continue;
        }
        double fM[5][3], fP[5][3];
        visc_flux(d, gm, velM, p, fM);
        visc_flux(d, gp, velP, p, fP);
        double *r = rhs + Np * ns * d * e;
        for (int s = 0; s < ns; s++) {
          double a = nrm[0] * (fM[s][0] + fP[s][0]) + nrm[1] * (fM[s][1] + fP[s][1]);
          if (d == 3) a = a + nrm[2] * (fM[s][2] + fP[s][2]);
          r[vM + Np * s] += sMJ * (0.5 * a);
        }
      }
  return bad;
}

/* lowstorageRK, euler3d_set3c.jl:1361-1523 with the nse viscous branch of
 * nse2d.jl:1826-1849: Carpenter-Kennedy LSRK(5,4) 2N-storage; rhs carries
 * the residual scaled by the next stage's A coefficient. */
int or_lowstorageRK(int d, int N, int64_t nelem, const double *vgeo,
                    const double *sgeo, double *Q, double *rhs,
                    const double *Dm, double dt, int64_t nsteps,
                    const int64_t *vmapM, const int64_t *vmapP,
                    const int64_t *elemtobndy, const or_phys *p,
                    int nthreads) {
  const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0,
                         -2404267990393.0 / 2016746695238.0,
                         -3550918686646.0 / 2091501179385.0,
                         -1275806237668.0 / 842570457699.0};
  const double RKB[5] = {1432997174477.0 / 9575080441755.0,
                         5161836677717.0 / 13612068292357.0,
                         1720146321549.0 / 2090206949498.0,
                         3134564353537.0 / 4481467310338.0,
                         2277821191437.0 / 14882151754819.0};
  const int Nq = N + 1;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int ns = d == 3 ? 5 : 4;
  double *gradQ = NULL, *rhs_gradQ = NULL;
  int visc = p->visc > 0;
  if (visc) {
    gradQ = (double *)calloc((size_t)(Np * ns * d * nelem), sizeof(double));
    rhs_gradQ = (double *)calloc((size_t)(Np * ns * d * nelem), sizeof(double));
  }
  int rc = 0;
  for (int64_t step = 0; step < nsteps && !rc; step++) {
    for (int s = 0; s < 5; s++) {
      or_volumerhs(d, N, rhs, Q, vgeo, Dm, nelem, p, nthreads);
      rc |= or_fluxrhs(d, N, rhs, Q, sgeo, vgeo, nelem, vmapM, vmapP, elemtobndy, p, nthreads);
      if (visc) {
        or_volume_grad(d, N, rhs_gradQ, Q, vgeo, Dm, nelem, p, nthreads);
        rc |= or_flux_grad(d, N, rhs_gradQ, Q, sgeo, vgeo, nelem, vmapM, vmapP, elemtobndy, p, nthreads);
        or_update_gradQ(d, N, gradQ, rhs_gradQ, vgeo, nelem, nthreads);
        or_volume_div(d, N, rhs_gradQ, gradQ, Q, vgeo, Dm, nelem, p, nthreads);
        rc |= or_flux_div(d, N, rhs_gradQ, gradQ, Q, sgeo, nelem, vmapM, vmapP, elemtobndy, p, nthreads);
      }
      or_updatesolution(d, N, rhs, rhs_gradQ, Q, vgeo, nelem, RKA[(s + 1) % 5],
                        RKB[s], dt, p->visc, nthreads);
    }
  }
  free(gradQ);
  free(rhs_gradQ);
  return rc;
}

/* L2energysquared, euler3d_set3c.jl:1252-1264 */
double or_L2energysquared(int d, int N, int nstate, const double *Q,
                          const double *vgeo, int64_t nelem) {
  const int Nq = N + 1;
  const int64_t Np = d == 3 ? (int64_t)Nq * Nq * Nq : (int64_t)Nq * Nq;
  const int nvg = d == 3 ? 14 : 8, fMJ = d == 3 ? 9 : 4;
  double energy = 0.0;
  for (int64_t e = 0; e < nelem; e++)
    for (int q = 0; q < nstate; q++)
      for (int64_t i = 0; i < Np; i++) {
        double v = Q[i + Np * (q + nstate * e)];
        energy += vgeo[i + Np * (fMJ + nvg * e)] * (v * v);
      }
  return energy;
}
