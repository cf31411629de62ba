/* CPU oracle for the ERI / Fock-build path.  TEST INFRASTRUCTURE ONLY (see
 * eri_oracle.h): a plain-C restatement of the reference's algorithm, kept
 * deliberately close to the reference's loop structure so each block can be
 * read against the cited lines.  Pinned against the reference compiled
 * headless (oracle/_ref/ref_driver) and the golden fixtures it wrote.
 */
#include "eri_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ */
/* Quantum-number arithmetic, QuantumNumbers.h:40-87                   */
/* ------------------------------------------------------------------ */
typedef struct {
  int l, m, n;
} qn;

static int qL(qn q) { return q.l + q.m + q.n; }
/* GetCanonicalIndex, QuantumNumbers.h:46-49 */
static int qci(qn q) { return (q.m + q.n + 1) * (q.m + q.n + 2) / 2 - q.m - 1; }
/* GetTotalCanonicalIndex, QuantumNumbers.h:51-58 */
static int qtci(qn q) {
  const int L = qL(q);
  return L * (L * (L + 3) + 2) / 6 + qci(q);
}
static int nfunc(int L) { return (L + 1) * (L + 2) / 2; }
/* CanonicalIncrement, QuantumNumbers.h:60-80 */
static void qinc(qn *q) {
  const int L = qL(*q);
  if (q->n == L) {
    q->l = L + 1;
    q->m = q->n = 0;
  } else if (q->m > 0) {
    --q->m;
    ++q->n;
  } else if (q->l > 0) {
    --q->l;
    q->m = L - q->l;
    q->n = 0;
  }
}
static qn mkqn(int l, int m, int n) {
  qn q = {l, m, n};
  return q;
}
static int qmax(qn q) {
  int a = q.l > q.m ? q.l : q.m;
  return a > q.n ? a : q.n;
}
/* direction picked by the reference's recursions: x if l is the largest
 * component, else y if m is, else z (GaussianTwoElectrons.h:40-73) */
static int qdir(qn q) {
  const int mx = qmax(q);
  if (q.l == mx) return 0;
  if (q.m == mx) return 1;
  return 2;
}
static int *qcomp(qn *q, int d) { return d == 0 ? &q->l : (d == 1 ? &q->m : &q->n); }

/* ------------------------------------------------------------------ */
/* Boys function                                                       */
/* ------------------------------------------------------------------ */
static double double_factorial(long n) {
  /* MathUtils::DoubleFactorial (MathUtils.h:35-45); the table of
   * MathUtils.cpp:16-38 holds n!! for n <= 20 */
  double r = 1;
  if (n <= 1) return 1;
  for (; n > 1; n -= 2) r *= (double)n;
  return r;
}

/* MathUtils::IncompleteGamma (MathUtils.h:163-200): series for x <= 1+a,
 * else an 80-term continued fraction for the upper function and
 * gamma(a) - Gamma(a,x). */
static int incomplete_gamma(double a, double x, double *gin) {
  *gin = 0;
  if (a < 0.0 || x < 0) return 0;
  if (x == 0.0) return 1;
  const double xam = -x + a * log(x);
  if (xam > 600 || a > 160.0) return 0;
  if (x <= 1.0 + a) {
    double sum = 1.0 / a, r = sum;
    for (int k = 1; k <= 80; ++k) {
      r *= x / (a + k);
      sum += r;
      if (fabs(r / sum) <= DBL_EPSILON) break;
    }
    *gin = exp(xam) * sum;
  } else {
    double t0 = 0.0;
    for (int k = 80; k >= 1; --k) t0 = (k - a) / (1.0 + k / (x + t0));
    const double gim = exp(xam) / (x + t0);
    *gin = tgamma(a) - gim;
  }
  return 1;
}

/* BoysFunction::operator() (BoysFunction.cpp:7-25) */
double orc_boys_single(double m, double x) {
  if (0. == m && 0. == x) return 1.;
  double res = 0;
  const double t = 1E-10;
  if (fabs(x) < t) x = t;
  if (x > 160) return double_factorial((long)(2 * m - 1)) / pow(2, m + 1) * sqrt(M_PI / pow(x, 2 * m + 1));
  incomplete_gamma(m + 0.5, x, &res);
  return res / (2. * pow(x, m + 0.5));
}

/* BoysFunctions::GenerateBoysFunctions (BoysFunctions.cpp:10-25) */
void orc_boys(int max_m, double T, double *out) {
  out[max_m] = orc_boys_single(max_m, T);
  for (int m = max_m - 1; m >= 0; --m) out[m] = (2. * T * out[m + 1] + exp(-T)) / (2. * m + 1.);
}

/* ------------------------------------------------------------------ */
/* Primitive quartet: GaussianTwoElectrons::Reset + VRR + ET           */
/* (GaussianTwoElectrons.cpp:15-188)                                   */
/* ------------------------------------------------------------------ */
typedef struct {
  int rows, cols;
  double *v; /* row-major */
} mat;
static double *at(mat *M, int r, int c) { return &M->v[(size_t)r * M->cols + c]; }

/* Returns the cropped (L1..L1+L2) x (L3..L3+L4) block in `out`
 * (rows = #cart in [L1, L1+L2], cols = #cart in [L3, L3+L4]). */
static void primitive_vrr_et(double a1, double a2, double a3, double a4, const double *c1, const double *c2,
                             const double *c3, const double *c4, int L1, int L2, int L3, int L4, int max_boys_m,
                             int exact_et, mat *out) {
  const double alpha12 = a1 + a2, alpha34 = a3 + a4;
  const double alphaProd = alpha12 * alpha34, alphaSum = alpha12 + alpha34;
  const double alpha = alphaProd / alphaSum;
  const int maxL12 = L1 + L2, maxL34 = L3 + L4, maxL = maxL12 + maxL34, size = maxL + 1;
  const int maxIndex = qtci(mkqn(0, 0, maxL));
  double R12[3], R34[3], Rp[3], Rq[3], Rpq[3];
  for (int d = 0; d < 3; ++d) {
    R12[d] = c1[d] - c2[d];
    R34[d] = c3[d] - c4[d];
    Rp[d] = (a1 * c1[d] + a2 * c2[d]) / alpha12;
    Rq[d] = (a3 * c3[d] + a4 * c4[d]) / alpha34;
    Rpq[d] = Rp[d] - Rq[d];
  }
  const double r12 = R12[0] * R12[0] + R12[1] * R12[1] + R12[2] * R12[2];
  const double r34 = R34[0] * R34[0] + R34[1] * R34[1] + R34[2] * R34[2];
  const double rpq = Rpq[0] * Rpq[0] + Rpq[1] * Rpq[1] + Rpq[2] * Rpq[2];
  const double exponent = -a1 * a2 / alpha12 * r12 - a3 * a4 / alpha34 * r34;
  const double factor = 2. * pow(M_PI, 5. / 2.) / (alphaProd * sqrt(alphaSum)) * exp(exponent);
  const double T = alpha * rpq;

  /* VRR matrix: (maxIndex+1) x size, Reset lines 48-53 */
  mat V = {maxIndex + 1, size, calloc((size_t)(maxIndex + 1) * size, sizeof(double))};
  double *boys = calloc((size_t)max_boys_m + 1, sizeof(double));
  orc_boys(max_boys_m, T, boys);
  for (int i = 0; i < size; ++i) *at(&V, 0, i) = factor * boys[i];
  free(boys);

  /* VerticalRecursion (GaussianTwoElectrons.cpp:98-134) */
  {
    double Rpa[3], Rwp[3];
    for (int d = 0; d < 3; ++d) {
      Rpa[d] = Rp[d] - c1[d];
      Rwp[d] = -alpha / alpha12 * Rpq[d];
    }
    const double oneDiv2alpha12 = 1. / (2. * alpha12);
    const double alphaDivAlpha12 = alpha / alpha12;
    for (qn cur = mkqn(1, 0, 0); qL(cur) < size; qinc(&cur)) {
      const int d = qdir(cur);
      qn prev = cur, pprev = cur;
      --*qcomp(&prev, d);
      int addPrevPrev = 0;
      double N = 0;
      if (*qcomp(&prev, d) > 0) {
        N = *qcomp(&prev, d);
        *qcomp(&pprev, d) -= 2;
        addPrevPrev = 1;
      }
      const int ci = qtci(cur), pi = qtci(prev);
      for (int m = 0; m < size - qL(cur); ++m) {
        double v = Rpa[d] * *at(&V, pi, m) + Rwp[d] * *at(&V, pi, m + 1);
        if (addPrevPrev) {
          const int ppi = qtci(pprev);
          v += N * oneDiv2alpha12 * (*at(&V, ppi, m) - alphaDivAlpha12 * *at(&V, ppi, m + 1));
        }
        *at(&V, ci, m) = v;
      }
    }
  }

  /* ElectronTransfer (GaussianTwoElectrons.cpp:137-188) */
  const int maxIndex12 = qtci(mkqn(0, 0, maxL12));
  const int maxIndex34 = qtci(mkqn(0, 0, maxL34));
  const int indexL1 = qtci(mkqn(L1, 0, 0));
  const int indexL3 = qtci(mkqn(L3, 0, 0));
  mat E = {maxIndex + 1, maxIndex34 + 1, calloc((size_t)(maxIndex + 1) * (maxIndex34 + 1), sizeof(double))};
  for (int r = 0; r <= maxIndex; ++r) *at(&E, r, 0) = *at(&V, r, 0);
  free(V.v);
  {
    double delta[3];
    for (int d = 0; d < 3; ++d) delta[d] = -(a2 * R12[d] + a4 * R34[d]) / alpha34;
    const double alpha12DivAlpha34 = alpha12 / alpha34;
    const double oneDiv2alpha34 = 1. / (2. * alpha34);
    for (qn q2 = mkqn(1, 0, 0); qL(q2) <= maxL34; qinc(&q2)) {
      const int curL = qL(q2);
      const int d = qdir(q2);
      qn p2 = q2, pp2 = q2;
      --*qcomp(&p2, d);
      int addPrevPrev = 0;
      double Ny = 0;
      if (*qcomp(&p2, d) > 0) {
        Ny = *qcomp(&p2, d);
        *qcomp(&pp2, d) -= 2;
        addPrevPrev = 1;
      }
      const int ci2 = qtci(q2), pi2 = qtci(p2), ppi2 = addPrevPrev ? qtci(pp2) : 0;
      /* the reference starts each column at total L = curL - 1
       * (GaussianTwoElectrons.cpp:162); the exact variant starts at 0 */
      for (qn q1 = exact_et ? mkqn(0, 0, 0) : mkqn(curL - 1, 0, 0); qL(q1) <= maxL - curL; qinc(&q1)) {
        const int ci1 = qtci(q1);
        qn next = q1, prev1 = q1;
        ++*qcomp(&next, d);
        int addPrev = 0;
        double Nx = 0;
        if (*qcomp(&prev1, d) > 0) {
          Nx = *qcomp(&prev1, d);
          --*qcomp(&prev1, d);
          addPrev = 1;
        }
        double v = delta[d] * *at(&E, ci1, pi2) - alpha12DivAlpha34 * *at(&E, qtci(next), pi2);
        if (addPrev) v += Nx * oneDiv2alpha34 * *at(&E, qtci(prev1), pi2);
        if (addPrevPrev) v += Ny * oneDiv2alpha34 * *at(&E, ci1, ppi2);
        *at(&E, ci1, ci2) = v;
      }
    }
  }
  /* crop, Reset line 95 */
  out->rows = maxIndex12 - indexL1 + 1;
  out->cols = maxIndex34 - indexL3 + 1;
  out->v = malloc((size_t)out->rows * out->cols * sizeof(double));
  for (int r = 0; r < out->rows; ++r)
    for (int c = 0; c < out->cols; ++c) *at(out, r, c) = *at(&E, indexL1 + r, indexL3 + c);
  free(E.v);
}

/* ------------------------------------------------------------------ */
/* Contracted quartet: IntegralsRepository::getElectronElectron        */
/* (IntegralsRepository.cpp:344-433) + HorizontalRecursion1/2          */
/* (GaussianTwoElectrons.cpp:198-359)                                  */
/* ------------------------------------------------------------------ */
static int fL(const orc_function *f) { return f->l + f->m + f->n; }

double orc_eri(const orc_function *fn, const orc_primitive *pr, int i, int j, int k, int l, int max_boys_m,
               int exact_et) {
  const orc_function *o1 = &fn[i], *o2 = &fn[j], *o3 = &fn[k], *o4 = &fn[l], *t;
  /* SwapOrbitals (IntegralsRepository.cpp:344-370) */
  if (fL(o1) < fL(o2) || (fL(o1) == fL(o2) && o1->id < o2->id)) { t = o1; o1 = o2; o2 = t; }
  if (fL(o3) < fL(o4) || (fL(o3) == fL(o4) && o3->id < o4->id)) { t = o3; o3 = o4; o4 = t; }
  if (fL(o1) + fL(o2) < fL(o3) + fL(o4) ||
      (fL(o1) + fL(o2) == fL(o3) + fL(o4) && (o1->id < o3->id || (o1->id == o3->id && o2->id < o4->id)))) {
    t = o1; o1 = o3; o3 = t;
    t = o2; o2 = o4; o4 = t;
  }
  const int L1 = fL(o1), L2 = fL(o2), L3 = fL(o3), L4 = fL(o4);
  const int rows = qtci(mkqn(0, 0, L1 + L2)) - qtci(mkqn(L1, 0, 0)) + 1;
  const int cols = qtci(mkqn(0, 0, L3 + L4)) - qtci(mkqn(L3, 0, 0)) + 1;
  double *acc = calloc((size_t)rows * cols, sizeof(double));

  /* primitive IDs run over all primitives in function order (Molecule.cpp:64-69) */
  for (int p1 = 0; p1 < o1->nprim; ++p1)
    for (int p2 = 0; p2 < o2->nprim; ++p2)
      for (int p3 = 0; p3 < o3->nprim; ++p3)
        for (int p4 = 0; p4 < o4->nprim; ++p4) {
          const orc_primitive *g[4] = {&pr[o1->prim_offset + p1], &pr[o2->prim_offset + p2],
                                       &pr[o3->prim_offset + p3], &pr[o4->prim_offset + p4]};
          const orc_function *gf[4] = {o1, o2, o3, o4};
          int gid[4] = {o1->prim_offset + p1, o2->prim_offset + p2, o3->prim_offset + p3, o4->prim_offset + p4};
          const double factor = g[0]->norm * g[1]->norm * g[2]->norm * g[3]->norm * g[0]->coef * g[1]->coef *
                                g[2]->coef * g[3]->coef;
          /* getElectronElectronVerticalAndTransfer (IntegralsRepository.cpp:436-475) */
          int ord[4] = {0, 1, 2, 3}, tt;
          if (L1 == L2 && gid[ord[0]] < gid[ord[1]]) { tt = ord[0]; ord[0] = ord[1]; ord[1] = tt; }
          if (L3 == L4 && gid[ord[2]] < gid[ord[3]]) { tt = ord[2]; ord[2] = ord[3]; ord[3] = tt; }
          int swapped = 0;
          if (L1 + L2 == L3 + L4 && (gid[ord[0]] < gid[ord[2]] || (gid[ord[0]] == gid[ord[2]] && gid[ord[1]] < gid[ord[3]]))) {
            tt = ord[0]; ord[0] = ord[2]; ord[2] = tt;
            tt = ord[1]; ord[1] = ord[3]; ord[3] = tt;
            swapped = 1;
          }
          const int Ls[4] = {L1, L2, L3, L4};
          mat blk;
          primitive_vrr_et(g[ord[0]]->alpha, g[ord[1]]->alpha, g[ord[2]]->alpha, g[ord[3]]->alpha,
                           gf[ord[0]]->center, gf[ord[1]]->center, gf[ord[2]]->center, gf[ord[3]]->center,
                           Ls[ord[0]], Ls[ord[1]], Ls[ord[2]], Ls[ord[3]], max_boys_m, exact_et, &blk);
          for (int r = 0; r < rows; ++r)
            for (int c = 0; c < cols; ++c) acc[r * cols + c] += factor * (swapped ? *at(&blk, c, r) : *at(&blk, r, c));
          free(blk.v);
        }

  /* HorizontalRecursion1 (GaussianTwoElectrons.cpp:198-272): (L1+L2,s|..) -> (L1,L2|..) */
  const int ind2Limit = qtci(mkqn(0, 0, L2)) + 1;
  const int ind3Limit = cols;
  const int QN1Base = qtci(mkqn(L1, 0, 0));
  double *w3 = calloc((size_t)rows * ind2Limit * ind3Limit, sizeof(double));
#define W3(a, b, c) w3[((size_t)(a) * ind2Limit + (b)) * ind3Limit + (c)]
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) W3(r, 0, c) = acc[r * cols + c];
  free(acc);
  {
    double dif[3];
    for (int d = 0; d < 3; ++d) dif[d] = o1->center[d] - o2->center[d];
    int L12 = L1 + L2;
    for (qn q2 = mkqn(1, 0, 0); qL(q2) <= L2;) {
      for (qn q1 = mkqn(L1, 0, 0); qL(q1) < L12; qinc(&q1)) {
        const int d = qdir(q2);
        qn next = q1, prev2 = q2;
        ++*qcomp(&next, d);
        --*qcomp(&prev2, d);
        const int cur1 = qtci(q1) - QN1Base, next1 = qtci(next) - QN1Base;
        const int cur2 = qtci(q2), p2 = qtci(prev2);
        for (int c = 0; c < ind3Limit; ++c) W3(cur1, cur2, c) = W3(next1, p2, c) + dif[d] * W3(cur1, p2, c);
      }
      /* IncrementQNandDecrementLimitIfNeeded (GaussianTwoElectrons.h:109-117) */
      const int oldL = qL(q2);
      qinc(&q2);
      if (qL(q2) != oldL) --L12;
    }
  }
  const int n1 = nfunc(L1), n2 = nfunc(L2), n3 = nfunc(L3), n4 = nfunc(L4);
  const int QN2Base = qtci(mkqn(L2, 0, 0));
  const int limit3 = cols, limit4 = qtci(mkqn(0, 0, L4)) + 1;
  const int QN3Base = qtci(mkqn(L3, 0, 0)), QN4Base = qtci(mkqn(L4, 0, 0));
  /* HorizontalRecursion2 (GaussianTwoElectrons.cpp:278-359): (..|L3+L4,s) -> (..|L3,L4) */
  double *w4 = calloc((size_t)n1 * n2 * limit3 * limit4, sizeof(double));
#define W4(a, b, c, e) w4[(((size_t)(a) * n2 + (b)) * limit3 + (c)) * limit4 + (e)]
  for (int a = 0; a < n1; ++a)
    for (int b = 0; b < n2; ++b)
      for (int c = 0; c < limit3; ++c) W4(a, b, c, 0) = W3(a, QN2Base + b, c);
  free(w3);
  {
    double dif[3];
    for (int d = 0; d < 3; ++d) dif[d] = o3->center[d] - o4->center[d];
    int L34 = L3 + L4;
    for (qn q4 = mkqn(1, 0, 0); qL(q4) <= L4;) {
      for (qn q3 = mkqn(L3, 0, 0); qL(q3) < L34; qinc(&q3)) {
        const int d = qdir(q4);
        qn next = q3, prev4 = q4;
        ++*qcomp(&next, d);
        --*qcomp(&prev4, d);
        const int cur3 = qtci(q3) - QN3Base, next3 = qtci(next) - QN3Base;
        const int cur4 = qtci(q4), p4 = qtci(prev4);
        for (int a = 0; a < n1; ++a)
          for (int b = 0; b < n2; ++b) W4(a, b, cur3, cur4) = W4(a, b, next3, p4) + dif[d] * W4(a, b, cur3, p4);
      }
      const int oldL = qL(q4);
      qinc(&q4);
      if (qL(q4) != oldL) --L34;
    }
  }
  /* getValue (GaussianTwoElectrons.cpp:9-12) */
  const qn Q1 = mkqn(o1->l, o1->m, o1->n), Q2 = mkqn(o2->l, o2->m, o2->n);
  const qn Q3 = mkqn(o3->l, o3->m, o3->n), Q4 = mkqn(o4->l, o4->m, o4->n);
  (void)n3;
  const double val = W4(qci(Q1), qci(Q2), qci(Q3), QN4Base + qci(Q4));
  free(w4);
#undef W3
#undef W4
  return val;
}

/* ------------------------------------------------------------------ */
/* Packed table and Fock two-electron parts                            */
/* ------------------------------------------------------------------ */
static int64_t two_index(int64_t i, int64_t j) { return i < j ? j * (j + 1) / 2 + i : i * (i + 1) / 2 + j; }
static int64_t ee_index(int i, int j, int k, int l) { return two_index(two_index(i, j), two_index(k, l)); }

int64_t orc_packed_size(int n) { return ee_index(n - 1, n - 1, n - 1, n - 1) + 1; }

/* CalculateElectronElectronIntegrals (IntegralsRepository.cpp:484-584):
 * i, j <= i, k, l <= k with ij <= kl */
void orc_eri_packed(int n, const orc_function *f, const orc_primitive *p, int max_boys_m, int exact_et,
                    double *out) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      const int64_t ij = two_index(i, j);
      for (int k = 0; k < n; ++k)
        for (int l = 0; l <= k; ++l) {
          if (ij <= two_index(k, l)) out[ee_index(i, j, k, l)] = orc_eri(f, p, i, j, k, l, max_boys_m, exact_et);
        }
    }
}

/* Diagonal quartets (ij|ij), i >= j, at index i(i+1)/2 + j: the Schwarz
 * bounds of the function pairs.  OpenMP over i. */
void orc_eri_diagonal(int n, const orc_function *f, const orc_primitive *p, int max_boys_m, int exact_et,
                      double *out) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) out[two_index(i, j)] = orc_eri(f, p, i, j, i, j, max_boys_m, exact_et);
}

void orc_g_rhf(int n, const double *packed, const double *P, double *G) {
#pragma omp parallel for
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double g = 0;
      for (int k = 0; k < n; ++k)
        for (int l = 0; l < n; ++l) {
          const double coulomb = packed[ee_index(i, j, k, l)];
          const double exchange = packed[ee_index(i, l, k, j)];
          g += P[k * n + l] * (coulomb - 0.5 * exchange);
        }
      G[i * n + j] = g;
    }
}

/* Rows of RestrictedHartreeFock::InitFockMatrix's two-electron part
 * (RestrictedHartreeFock.cpp:189-200) straight from the contracted accessor,
 * no stored table, for molecules whose packed table does not fit:
 * G_ij = sum_kl P_kl [(ij|kl) - 1/2 (il|kj)] for i in rows[0..nrows), all j.
 * The J sum uses the symmetry of P (kl and lk together).  OpenMP over j. */
void orc_g_rhf_rows(int n, const orc_function *f, const orc_primitive *p, int max_boys_m, int exact_et,
                    const double *P, const int *rows, int nrows, double *out) {
  for (int r = 0; r < nrows; ++r) {
    const int i = rows[r];
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < n; ++j) {
      double coulomb = 0, exchange = 0;
      for (int k = 0; k < n; ++k) {
        for (int l = 0; l < k; ++l) coulomb += 2.0 * P[k * n + l] * orc_eri(f, p, i, j, k, l, max_boys_m, exact_et);
        coulomb += P[k * n + k] * orc_eri(f, p, i, j, k, k, max_boys_m, exact_et);
        for (int l = 0; l < n; ++l) exchange += P[k * n + l] * orc_eri(f, p, i, l, k, j, max_boys_m, exact_et);
      }
      out[(size_t)r * n + j] = coulomb - 0.5 * exchange;
    }
  }
}

void orc_g_uhf(int n, const double *packed, const double *Pa, const double *Pb, double *Ga, double *Gb) {
#pragma omp parallel for
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double ga = 0, gb = 0;
      for (int k = 0; k < n; ++k)
        for (int l = 0; l < n; ++l) {
          const double coulomb = packed[ee_index(i, j, k, l)];
          const double exchange = packed[ee_index(i, l, k, j)];
          ga += Pa[k * n + l] * (coulomb - exchange) + Pb[k * n + l] * coulomb;
          gb += Pb[k * n + l] * (coulomb - exchange) + Pa[k * n + l] * coulomb;
        }
      Ga[i * n + j] = ga;
      Gb[i * n + j] = gb;
    }
}

/* ------------------------------------------------------------------ */
/* One-electron integrals                                              */
/* ------------------------------------------------------------------ */
/* 1D overlap table by the reference's vertical + transfer recurrences
 * (GaussianOverlap.cpp:34-65 / GaussianMoment.cpp:44-90):
 * s[i][j], i <= imax, j <= jmax. */
static void overlap_1d(double a1, double a2, double A, double B, int imax, int jmax, double s[8][8]) {
  const double alpha = a1 + a2;
  const double P = (a1 * A + a2 * B) / alpha;
  const double dif = A - B, difCenter = P - A, oneDiv2alpha = 1. / (2. * alpha);
  double m[16][8];
  memset(m, 0, sizeof m);
  m[0][0] = 1;
  m[1][0] = difCenter;
  int limit = imax + jmax + 1;
  for (int i = 2; i <= limit; ++i) m[i][0] = difCenter * m[i - 1][0] + (i - 1) * oneDiv2alpha * m[i - 2][0];
  --limit;
  for (int j = 1; j <= jmax; ++j, --limit)
    for (int i = 0; i <= limit; ++i) m[i][j] = m[i + 1][j - 1] + dif * m[i][j - 1];
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) s[i][j] = m[i][j];
}

/* GaussianKinetic::CalculateKinetic (GaussianKinetic.cpp:60-84) on the 1D
 * overlaps extended by one in each index */
static double kinetic_1d(double a1, double a2, int i, int j, double s[8][8]) {
  const double tp = 2 * a1 * a2;
  if (i == 0 && j == 0) return tp * s[1][1];
  if (j == 0) return -i * a2 * s[i - 1][1] + tp * s[i + 1][1];
  if (i == 0) return -j * a1 * s[1][j - 1] + tp * s[1][j + 1];
  return (double)i * j * s[i - 1][j - 1] * 0.5 - j * a1 * s[i + 1][j - 1] - i * a2 * s[i - 1][j + 1] +
         tp * s[i + 1][j + 1];
}

/* Nuclear attraction of one contracted pair to one nucleus:
 * GaussianNuclear::Reset/VerticalRecursion (GaussianNuclear.cpp:11-72)
 * per primitive pair, contraction (IntegralsRepository.cpp:250-286), then
 * HorizontalRecursion (GaussianNuclear.cpp:75-108). */
static double nuclear_pair(const orc_function *o1, const orc_function *o2, const orc_primitive *pr,
                           const double *nuc, int max_boys_m) {
  const orc_function *t;
  if (fL(o1) < fL(o2) || (fL(o1) == fL(o2) && o1->id > o2->id)) { t = o1; o1 = o2; o2 = t; }
  const int L1 = fL(o1), L2 = fL(o2), maxL = L1 + L2, size = maxL + 1;
  const int rowsN = qtci(mkqn(0, 0, maxL)) + 1;
  double *acc = calloc((size_t)rowsN, sizeof(double));
  double *M = malloc((size_t)rowsN * size * sizeof(double));
  double *boys = calloc((size_t)max_boys_m + 1, sizeof(double));
  for (int p1 = 0; p1 < o1->nprim; ++p1)
    for (int p2 = 0; p2 < o2->nprim; ++p2) {
      const orc_primitive *g1 = &pr[o1->prim_offset + p1], *g2 = &pr[o2->prim_offset + p2];
      const double alpha = g1->alpha + g2->alpha;
      double Rp[3], difN[3], dif[3], difRp[3];
      for (int d = 0; d < 3; ++d) {
        Rp[d] = (g1->alpha * o1->center[d] + g2->alpha * o2->center[d]) / alpha;
        difN[d] = nuc[d] - Rp[d];
        dif[d] = o1->center[d] - o2->center[d];
        difRp[d] = Rp[d] - o1->center[d];
      }
      const double dn2 = difN[0] * difN[0] + difN[1] * difN[1] + difN[2] * difN[2];
      const double d2 = dif[0] * dif[0] + dif[1] * dif[1] + dif[2] * dif[2];
      orc_boys(max_boys_m, alpha * dn2, boys);
      const double factor = 2. * M_PI / alpha * exp(-g1->alpha * g2->alpha / alpha * d2);
      memset(M, 0, (size_t)rowsN * size * sizeof(double));
      for (int i = 0; i < size; ++i) M[i] = factor * boys[i];
      const double oneDiv2alpha = 1. / (2. * alpha);
      for (qn cur = mkqn(1, 0, 0); qL(cur) < size; qinc(&cur)) {
        const int d = qdir(cur);
        qn prev = cur, pprev = cur;
        --*qcomp(&prev, d);
        int addPrevPrev = 0;
        double N = 0;
        if (*qcomp(&prev, d) > 0) {
          N = *qcomp(&prev, d);
          *qcomp(&pprev, d) -= 2;
          addPrevPrev = 1;
        }
        const int ci = qtci(cur), pi = qtci(prev);
        for (int m = 0; m < size - qL(cur); ++m) {
          double v = difRp[d] * M[pi * size + m] + difN[d] * M[pi * size + m + 1];
          if (addPrevPrev) {
            const int ppi = qtci(pprev);
            v += N * oneDiv2alpha * (M[ppi * size + m] - M[ppi * size + m + 1]);
          }
          M[ci * size + m] = v;
        }
      }
      /* IntegralsRepository.cpp:273 */
      const double f = g1->norm * g2->norm * g1->coef * g2->coef;
      for (int r = 0; r < rowsN; ++r) acc[r] += f * M[r * size];
    }
  free(M);
  free(boys);
  /* horizontal recursion on the contracted column */
  const int limit = qtci(mkqn(0, 0, L2)) + 1;
  double *H = calloc((size_t)rowsN * limit, sizeof(double));
  for (int r = 0; r < rowsN; ++r) H[r * limit] = acc[r];
  free(acc);
  double dif[3];
  for (int d = 0; d < 3; ++d) dif[d] = o1->center[d] - o2->center[d];
  int mL = maxL;
  for (qn qj = mkqn(1, 0, 0); qL(qj) <= L2;) {
    for (qn q = mkqn(0, 0, 0); qL(q) < mL; qinc(&q)) {
      const int d = qdir(qj);
      qn next = q, prevj = qj;
      ++*qcomp(&next, d);
      --*qcomp(&prevj, d);
      H[qtci(q) * limit + qtci(qj)] = H[qtci(next) * limit + qtci(prevj)] + dif[d] * H[qtci(q) * limit + qtci(prevj)];
    }
    const int oldL = qL(qj);
    qinc(&qj);
    if (qL(qj) != oldL) --mL;
  }
  const double v = H[qtci(mkqn(o1->l, o1->m, o1->n)) * limit + qtci(mkqn(o2->l, o2->m, o2->n))];
  free(H);
  return v;
}

void orc_one_electron(int n, const orc_function *f, const orc_primitive *p, int natoms, const double *atom_xyz,
                      const int *atom_z, int max_boys_m, double *S, double *T, double *V) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      const orc_function *o1 = &f[i], *o2 = &f[j];
      double s = 0, t = 0;
      for (int p1 = 0; p1 < o1->nprim; ++p1)
        for (int p2 = 0; p2 < o2->nprim; ++p2) {
          const orc_primitive *g1 = &p[o1->prim_offset + p1], *g2 = &p[o2->prim_offset + p2];
          double sx[8][8], sy[8][8], sz[8][8];
          overlap_1d(g1->alpha, g2->alpha, o1->center[0], o2->center[0], o1->l + 1, o2->l + 1, sx);
          overlap_1d(g1->alpha, g2->alpha, o1->center[1], o2->center[1], o1->m + 1, o2->m + 1, sy);
          overlap_1d(g1->alpha, g2->alpha, o1->center[2], o2->center[2], o1->n + 1, o2->n + 1, sz);
          double d2 = 0;
          for (int d = 0; d < 3; ++d) d2 += (o1->center[d] - o2->center[d]) * (o1->center[d] - o2->center[d]);
          const double inv = 1. / (g1->alpha + g2->alpha);
          const double factor = exp(-g1->alpha * g2->alpha * inv * d2) * pow(M_PI * inv, 1.5);
          /* IntegralsRepository.cpp:96-106, 182-192 */
          const double cc = g1->norm * g2->norm * g1->coef * g2->coef;
          s += cc * (factor * sx[o1->l][o2->l] * sy[o1->m][o2->m] * sz[o1->n][o2->n]);
          /* GaussianKinetic::getKinetic (GaussianKinetic.cpp:42-57) */
          t += cc * factor *
               (kinetic_1d(g1->alpha, g2->alpha, o1->l, o2->l, sx) * sy[o1->m][o2->m] * sz[o1->n][o2->n] +
                sx[o1->l][o2->l] * kinetic_1d(g1->alpha, g2->alpha, o1->m, o2->m, sy) * sz[o1->n][o2->n] +
                sx[o1->l][o2->l] * sy[o1->m][o2->m] * kinetic_1d(g1->alpha, g2->alpha, o1->n, o2->n, sz));
        }
      double v = 0;
      /* NuclearMatrix::Calculate (QuantumMatrix.cpp:128-155) */
      for (int a = 0; a < natoms; ++a) v -= atom_z[a] * nuclear_pair(o1, o2, p, &atom_xyz[3 * a], max_boys_m);
      S[i * n + j] = S[j * n + i] = s;
      T[i * n + j] = T[j * n + i] = t;
      V[i * n + j] = V[j * n + i] = v;
    }
}
