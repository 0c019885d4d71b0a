// Level-symmetric (LQn) discrete-ordinates sets for 2D (XY) and 3D.
//
// Restates the published construction that UBOLT's generator
// (src/sn_lqn_table.py, module docstring and build_order) derives its table
// from, and the ordinate expansion of src/sn_quadraturek.kokkos.cxx:286-427:
//
//   * n = N/2 levels with mu_l^2 in arithmetic progression,
//     mu_l^2 = mu_1^2 + (l - 1) delta, delta = (1 - 3 mu_1^2) / (n - 1);
//   * one octant holds every ORDERED level triple (i, j, k) with
//     i + j + k = n + 2, listed lexicographically;
//   * a point's weight depends only on its sorted triple (permutation class);
//   * the level sums y_l solve the even axis moments m = 0, 2..n exactly, and
//     mu_1 is the root of sum_l (3 l - (n + 2)) y_l = 0;
//   * class weights come from the level sums through the integer
//     class-to-level map; where that map has a null space (S14 and up) the
//     member minimising the relative error of the mixed even moments
//     <mu^2a eta^2b xi^2c>, a + b + c <= n, is taken (least squares).
//
// Everything is computed in long double and rounded to double on output.
// Parity with the reference generator's emitted constants is pinned by
// tests/golden/lqn_reference.json (made by running the reference script).
//
// Ordinate order (sn_quadraturek.kokkos.cxx:319-330 for 2D, 379-392 for 3D):
// octant point slowest, then the sign combinations with x fastest. 2D keeps
// the xi > 0 half and doubles the weights; both sum to 4 pi.
#include "ubolt_internal.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <numeric>
#include <vector>

namespace {

using LD = long double;

// Exact rational on 64-bit integers: the class map entries are tiny counts,
// so nothing here comes near overflow.
struct Frac {
   int64_t num = 0, den = 1;
   Frac() = default;
   Frac(int64_t n, int64_t d = 1) : num(n), den(d) { norm(); }
   void norm()
   {
      if (den < 0) { num = -num; den = -den; }
      const int64_t g = std::gcd(num < 0 ? -num : num, den);
      if (g > 1) { num /= g; den /= g; }
   }
   bool zero() const { return num == 0; }
   Frac operator-(const Frac &o) const { return Frac(num * o.den - o.num * den, den * o.den); }
   Frac operator*(const Frac &o) const { return Frac(num * o.num, den * o.den); }
   Frac operator/(const Frac &o) const { return Frac(num * o.den, den * o.num); }
   LD value() const { return (LD)num / (LD)den; }
};

// Solve a small dense system in place by partial pivoting (long double).
bool SolveDense(std::vector<std::vector<LD>> A, std::vector<LD> b, std::vector<LD> &x)
{
   const size_t n = b.size();
   for (size_t k = 0; k < n; k++) {
      size_t p = k;
      for (size_t i = k + 1; i < n; i++) if (fabsl(A[i][k]) > fabsl(A[p][k])) p = i;
      if (A[p][k] == 0.0L) return false;
      std::swap(A[k], A[p]);
      std::swap(b[k], b[p]);
      for (size_t i = k + 1; i < n; i++) {
         const LD f = A[i][k] / A[k][k];
         for (size_t j = k; j < n; j++) A[i][j] -= f * A[k][j];
         b[i] -= f * b[k];
      }
   }
   x.assign(n, 0.0L);
   for (size_t k = n; k-- > 0;) {
      LD s = b[k];
      for (size_t j = k + 1; j < n; j++) s -= A[k][j] * x[j];
      x[k] = s / A[k][k];
   }
   return true;
}

using Triple = std::array<int, 3>;

std::vector<Triple> OctantTriples(int n)
{
   std::vector<Triple> out;
   for (int i = 1; i <= n; i++)
      for (int j = 1; j <= n; j++) {
         const int k = n + 2 - i - j;
         if (k >= 1 && k <= n) out.push_back({i, j, k});
      }
   return out;
}

Triple Sorted(Triple t)
{
   std::sort(t.begin(), t.end());
   return t;
}

std::vector<LD> LevelSquares(int n, LD mu1)
{
   if (n == 1) return {1.0L / 3.0L};
   const LD x1 = mu1 * mu1;
   const LD delta = (1.0L - 3.0L * x1) / (LD)(n - 1);
   std::vector<LD> x(n);
   for (int i = 0; i < n; i++) x[i] = x1 + (LD)i * delta;
   return x;
}

// y_l: total octant weight of the points whose first level index is l, from
// the even axis moments m = 0, 2, .., n (m = 1 is a multiple of m = 0).
std::vector<LD> LevelSums(int n, LD mu1)
{
   const std::vector<LD> x = LevelSquares(n, mu1);
   std::vector<int> moments = {0};
   for (int m = 2; m <= n; m++) moments.push_back(m);
   std::vector<std::vector<LD>> V(n, std::vector<LD>(n));
   std::vector<LD> rhs(n), y;
   for (int r = 0; r < n; r++) {
      for (int l = 0; l < n; l++) V[r][l] = powl(x[l], (LD)moments[r]);
      rhs[r] = 1.0L / (8.0L * (2.0L * moments[r] + 1.0L));
   }
   SolveDense(V, rhs, y);
   return y;
}

LD Mu1Residual(int n, LD mu1)
{
   const std::vector<LD> y = LevelSums(n, mu1);
   LD s = 0.0L;
   for (int l = 0; l < n; l++) s += (LD)(3 * (l + 1) - (n + 2)) * y[l];
   return s;
}

// Seeds for the mu_1 root-find: the 7-digit textbook values of the
// level-symmetric first cosine (Lewis & Miller, Table 4-1). Only seeds; the
// root is refined to working precision.
LD Mu1Seed(int sn_order)
{
   switch (sn_order) {
   case 4: return 0.3500212L;
   case 6: return 0.2666355L;
   case 8: return 0.2182179L;
   case 10: return 0.1893213L;
   case 12: return 0.1672126L;
   case 14: return 0.1519859L;
   case 16: return 0.1389568L;
   case 18: return 0.1293445L;
   default: return 0.0L;
   }
}

LD SolveMu1(int n)
{
   if (n == 1) return sqrtl(1.0L / 3.0L);
   const LD seed = Mu1Seed(2 * n);
   LD a = seed * 0.999L, b = seed * 1.001L;
   LD fa = Mu1Residual(n, a), fb = Mu1Residual(n, b);
   for (int it = 0; it < 200 && fb != fa; it++) {
      const LD c = b - fb * (b - a) / (fb - fa);
      a = b;
      fa = fb;
      b = c;
      fb = Mu1Residual(n, b);
      if (fabsl(b - a) <= 1e-19L * fabsl(b)) break;
   }
   return b;
}

int64_t DoubleFactorial(int k)
{
   int64_t out = 1;
   while (k > 1) { out *= k; k -= 2; }
   return out;
}

// <mu^2a eta^2b xi^2c> over the unit sphere, exactly.
LD SphereMoment(int a, int b, int c)
{
   return (LD)(DoubleFactorial(2 * a - 1) * DoubleFactorial(2 * b - 1) * DoubleFactorial(2 * c - 1)) /
          (LD)DoubleFactorial(2 * (a + b + c) + 1);
}

}  // namespace

namespace ubolt {

// One order's octant: level cosines and per-point weights (fractions of the
// whole sphere), the points in lexicographic triple order.
int LqnOctant(int sn_order, std::vector<double> &mu, std::vector<std::array<int, 3>> &points,
              std::vector<double> &weight)
{
   if (sn_order < 2 || sn_order > 18 || sn_order % 2) return -1;
   const int n = sn_order / 2;
   const LD mu1 = SolveMu1(n);
   const std::vector<LD> x = LevelSquares(n, mu1);
   const std::vector<Triple> triples = OctantTriples(n);

   std::vector<Triple> classes;
   for (const Triple &t : triples) classes.push_back(Sorted(t));
   std::sort(classes.begin(), classes.end());
   classes.erase(std::unique(classes.begin(), classes.end()), classes.end());
   std::map<Triple, int> cls_of;
   for (size_t c = 0; c < classes.size(); c++) cls_of[classes[c]] = (int)c;
   const int n_cls = (int)classes.size();

   const std::vector<LD> y = LevelSums(n, mu1);

   // Class weights -> level sums, an integer map; exact RREF with the row
   // transform so a particular solution and the null space fall out.
   std::vector<std::vector<Frac>> A(n, std::vector<Frac>(n_cls, Frac(0)));
   for (const Triple &t : triples) {
      Frac &e = A[t[0] - 1][cls_of[Sorted(t)]];
      e = Frac(e.num + e.den, e.den);
   }
   std::vector<std::vector<Frac>> T(n, std::vector<Frac>(n, Frac(0)));
   for (int i = 0; i < n; i++) T[i][i] = Frac(1);
   std::vector<int> pivots;
   int r = 0;
   for (int c = 0; c < n_cls && r < n; c++) {
      int pr = -1;
      for (int k = r; k < n; k++) if (!A[k][c].zero()) { pr = k; break; }
      if (pr < 0) continue;
      std::swap(A[r], A[pr]);
      std::swap(T[r], T[pr]);
      const Frac inv = A[r][c];
      for (auto &v : A[r]) v = v / inv;
      for (auto &v : T[r]) v = v / inv;
      for (int k = 0; k < n; k++) {
         if (k == r || A[k][c].zero()) continue;
         const Frac f = A[k][c];
         for (int j = 0; j < n_cls; j++) A[k][j] = A[k][j] - f * A[r][j];
         for (int j = 0; j < n; j++) T[k][j] = T[k][j] - f * T[r][j];
      }
      pivots.push_back(c);
      r++;
   }
   std::vector<LD> base(n_cls, 0.0L);
   for (size_t row = 0; row < pivots.size(); row++) {
      LD ty = 0.0L;
      for (int k = 0; k < n; k++) ty += T[row][k].value() * y[k];
      base[pivots[row]] = ty;
   }
   std::vector<std::vector<LD>> null_basis;
   for (int fc = 0; fc < n_cls; fc++) {
      if (std::find(pivots.begin(), pivots.end(), fc) != pivots.end()) continue;
      std::vector<LD> v(n_cls, 0.0L);
      v[fc] = 1.0L;
      for (size_t row = 0; row < pivots.size(); row++) v[pivots[row]] = -A[row][fc].value();
      null_basis.push_back(v);
   }

   auto moment = [&](const std::vector<LD> &w, int a, int b, int c) {
      LD s = 0.0L;
      for (const Triple &t : triples)
         s += w[cls_of[Sorted(t)]] * powl(x[t[0] - 1], (LD)a) * powl(x[t[1] - 1], (LD)b) *
              powl(x[t[2] - 1], (LD)c);
      return s;
   };

   std::vector<LD> w_cls = base;
   if (!null_basis.empty()) {
      std::vector<std::array<int, 3>> keys;
      for (int a = 0; a <= n; a++)
         for (int b = 0; b <= std::min(a, n - a); b++)
            for (int c = 0; c <= std::min(b, n - a - b); c++)
               if (b > 0) keys.push_back({a, b, c});
      const size_t nk = keys.size(), nn = null_basis.size();
      std::vector<std::vector<LD>> G(nk, std::vector<LD>(nn));
      std::vector<LD> r0(nk);
      for (size_t row = 0; row < nk; row++) {
         const auto &k = keys[row];
         const LD want = SphereMoment(k[0], k[1], k[2]) / 8.0L;
         r0[row] = (moment(base, k[0], k[1], k[2]) - want) / want;
         for (size_t col = 0; col < nn; col++) G[row][col] = moment(null_basis[col], k[0], k[1], k[2]) / want;
      }
      std::vector<std::vector<LD>> GtG(nn, std::vector<LD>(nn, 0.0L));
      std::vector<LD> rhs(nn, 0.0L), t;
      for (size_t i = 0; i < nn; i++) {
         for (size_t j = 0; j < nn; j++)
            for (size_t row = 0; row < nk; row++) GtG[i][j] += G[row][i] * G[row][j];
         for (size_t row = 0; row < nk; row++) rhs[i] -= G[row][i] * r0[row];
      }
      SolveDense(GtG, rhs, t);
      for (int k = 0; k < n_cls; k++)
         for (size_t j = 0; j < nn; j++) w_cls[k] += t[j] * null_basis[j][k];
   }
   for (LD v : w_cls) if (!(v > 0.0L)) return -2;

   mu.resize(n);
   for (int l = 0; l < n; l++) mu[l] = (double)sqrtl(x[l]);
   points.clear();
   weight.clear();
   for (const Triple &t : triples) {
      points.push_back({t[0], t[1], t[2]});
      weight.push_back((double)w_cls[cls_of[Sorted(t)]]);
   }
   return 0;
}

}  // namespace ubolt

// ~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~

extern "C" int ubolt_lqn_octant(int sn_order, double *mu, int *points, double *weight, int *n_levels,
                                int *n_points)
{
   std::vector<double> m, w;
   std::vector<std::array<int, 3>> p;
   const int rc = ubolt::LqnOctant(sn_order, m, p, w);
   if (rc) return ubolt::SetError(UBOLT_ERR_ARG, "no level-symmetric set for S%d (even orders 2..18 only)",
                                  sn_order);
   if (n_levels) *n_levels = (int)m.size();
   if (n_points) *n_points = (int)p.size();
   if (mu) for (size_t i = 0; i < m.size(); i++) mu[i] = m[i];
   if (points) for (size_t i = 0; i < p.size(); i++) for (int d = 0; d < 3; d++) points[3 * i + d] = p[i][d];
   if (weight) for (size_t i = 0; i < w.size(); i++) weight[i] = w[i];
   return UBOLT_OK;
}

extern "C" int ubolt_quadrature_lqn(int dim, int sn_order, double *omega, double *w, int *reflect,
                                    int *n_angles, double *sum_weights)
{
   if (dim != 2 && dim != 3) return ubolt::SetError(UBOLT_ERR_ARG, "LQn sets are 2D or 3D, was given %dD", dim);
   std::vector<double> mu, frac;
   std::vector<std::array<int, 3>> pts;
   if (ubolt::LqnOctant(sn_order, mu, pts, frac))
      return ubolt::SetError(UBOLT_ERR_ARG, "no level-symmetric set for S%d (even orders 2..18 only)", sn_order);
   const int per = (dim == 2) ? 4 : 8;
   const int na = (int)pts.size() * per;
   if (n_angles) *n_angles = na;
   if (sum_weights) *sum_weights = 4.0 * M_PI;
   if (!omega && !w && !reflect) return UBOLT_OK;

   std::vector<double> om(3 * na, 0.0), wt(na);
   int a = 0;
   for (size_t p = 0; p < pts.size(); p++) {
      const double bx = mu[pts[p][0] - 1], by = mu[pts[p][1] - 1], bz = mu[pts[p][2] - 1];
      if (dim == 2) {
         const double wp = 2.0 * frac[p] * (4.0 * M_PI);
         for (int sy = -1; sy <= 1; sy += 2)
            for (int sx = -1; sx <= 1; sx += 2) {
               om[3 * a] = sx * bx;
               om[3 * a + 1] = sy * by;
               wt[a++] = wp;
            }
      } else {
         const double wp = frac[p] * (4.0 * M_PI);
         for (int sz = -1; sz <= 1; sz += 2)
            for (int sy = -1; sy <= 1; sy += 2)
               for (int sx = -1; sx <= 1; sx += 2) {
                  om[3 * a] = sx * bx;
                  om[3 * a + 1] = sy * by;
                  om[3 * a + 2] = sz * bz;
                  wt[a++] = wp;
               }
      }
   }
   // Reflection maps by exact search (sn_quadraturek.kokkos.cxx:60-115): the
   // mirrored ordinate is built from the same cosine value, so == holds.
   std::vector<int> refl(3 * na, -1);
   for (int d = 0; d < dim; d++)
      for (int b = 0; b < na; b++) {
         for (int c = 0; c < na; c++) {
            bool match = true;
            for (int e = 0; e < dim; e++) {
               const double want = (e == d) ? -om[3 * b + e] : om[3 * b + e];
               if (om[3 * c + e] != want) { match = false; break; }
            }
            if (match) { refl[d * na + b] = c; break; }
         }
         if (refl[d * na + b] < 0 || wt[refl[d * na + b]] != wt[b])
            return ubolt::SetError(UBOLT_ERR_STATE, "quadrature set is not reflection symmetric");
      }
   double wsum = 0.0;
   for (int b = 0; b < na; b++) wsum += wt[b];
   if (std::fabs(wsum - 4.0 * M_PI) > 1e-12 * 4.0 * M_PI * na)
      return ubolt::SetError(UBOLT_ERR_STATE, "quadrature weights sum to %.17g, not 4 pi", wsum);
   if (omega) std::copy(om.begin(), om.end(), omega);
   if (w) std::copy(wt.begin(), wt.end(), w);
   if (reflect) std::copy(refl.begin(), refl.end(), reflect);
   return UBOLT_OK;
}
