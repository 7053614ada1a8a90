#include "multilevel.hpp"

#include <algorithm>
#include <cmath>

namespace dpm {
namespace {

// Compressed rows with ascending columns (diagonal included).
struct Csr {
  int n = 0;
  std::vector<int64_t> off;
  std::vector<int> col;
  std::vector<double> val;
};

// Rows are independent: counted in parallel, then filled in parallel at their prefix offsets.
Csr csr_from_ell(int n, int WA, const int* col, const double* val) {
  Csr A;
  A.n = n;
  A.off.assign(n + 1, 0);
  auto row_entries = [&](int i, int* cj, double* vj) {  // sorted, equal columns summed
    int m = 0;
    for (int s = 0; s < WA; ++s) {
      const int j = col[(size_t)s * n + i];
      const double v = val[(size_t)s * n + i];
      if (!(j == i || v != 0.0)) continue;
      int t = m++;
      while (t > 0 && cj[t - 1] > j) { cj[t] = cj[t - 1]; vj[t] = vj[t - 1]; --t; }  // stable
      cj[t] = j;
      vj[t] = v;
    }
    int u = 0;
    for (int k = 0; k < m; ++k) {
      if (u > 0 && cj[u - 1] == cj[k]) {  // padding slots share the own column
        vj[u - 1] += vj[k];
        continue;
      }
      cj[u] = cj[k];
      vj[u] = vj[k];
      ++u;
    }
    return u;
  };
  std::vector<int> cnt(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    int cj[64];
    double vj[64];
    cnt[i] = row_entries(i, cj, vj);
  }
  for (int i = 0; i < n; ++i) A.off[i + 1] = A.off[i] + cnt[i];
  A.col.resize(A.off[n]);
  A.val.resize(A.off[n]);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    int cj[64];
    double vj[64];
    const int u = row_entries(i, cj, vj);
    for (int k = 0; k < u; ++k) {
      A.col[A.off[i] + k] = cj[k];
      A.val[A.off[i] + k] = vj[k];
    }
  }
  return A;
}

// One pass of pairwise aggregation: rows in order; an unpaired row takes its strongest unpaired
// neighbour j (largest -a_ij, first in column order on ties) if -a_ij >= beta * max_k(-a_ik).
int pairwise(const Csr& A, double beta, std::vector<int>& agg) {
  agg.assign(A.n, -1);
  int na = 0;
  for (int i = 0; i < A.n; ++i) {
    if (agg[i] >= 0) continue;
    double mx = 0.0;
    for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k)
      if (A.col[k] != i) mx = std::max(mx, -A.val[k]);
    int best = -1;
    double bv = 0.0;
    for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k) {
      const int j = A.col[k];
      if (j == i || agg[j] >= 0) continue;
      const double s = -A.val[k];
      if (s >= beta * mx && s > bv) {
        bv = s;
        best = j;
      }
    }
    agg[i] = na;
    if (best >= 0) agg[best] = na;
    ++na;
  }
  // A row left alone (its strong neighbours were all taken, typically around one strongly
  // coupled row) joins the aggregate of its strongest neighbour if that holds fewer than 3 rows,
  // so that a pass keeps coarsening on irregular meshes; 3 passes then give at most 27 rows.
  std::vector<int> size(na, 0);
  for (int i = 0; i < A.n; ++i) size[agg[i]]++;
  for (int i = 0; i < A.n; ++i) {
    if (size[agg[i]] != 1) continue;
    int best = -1;
    double bv = 0.0;
    for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k) {
      const int j = A.col[k];
      if (j == i || size[agg[j]] >= 3 || -A.val[k] <= bv) continue;
      bv = -A.val[k];
      best = j;
    }
    if (best < 0) continue;
    size[agg[i]] = 0;
    agg[i] = agg[best];
    size[agg[best]]++;
  }
  // renumber the aggregates densely, in order of first appearance
  std::vector<int> remap(na, -1);
  int m = 0;
  for (int i = 0; i < A.n; ++i) {
    if (remap[agg[i]] < 0) remap[agg[i]] = m++;
    agg[i] = remap[agg[i]];
  }
  return m;
}

// Member rows of every aggregate, ascending.
void members(const std::vector<int>& agg, int na, std::vector<int64_t>& moff, std::vector<int>& mrow) {
  moff.assign(na + 1, 0);
  for (int a : agg) moff[a + 1]++;
  for (int a = 0; a < na; ++a) moff[a + 1] += moff[a];
  mrow.assign(agg.size(), 0);
  std::vector<int64_t> fill(moff.begin(), moff.end() - 1);
  for (size_t i = 0; i < agg.size(); ++i) mrow[fill[agg[i]]++] = (int)i;
}

// A_c = T^T A T for the aggregation T (row i -> column agg[i]); entries summed in the order
// (aggregate member ascending, fine column ascending), so the result is reproducible.
Csr galerkin(const Csr& A, const std::vector<int>& agg, int na) {
  std::vector<int64_t> moff;
  std::vector<int> mrow;
  members(agg, na, moff, mrow);
  Csr C;
  C.n = na;
  C.off.assign(na + 1, 0);
  // one aggregate's row: columns in order of first appearance, summed, then sorted by column
  auto agg_row = [&](int a, std::vector<int64_t>& pos, std::vector<int>& cols, std::vector<double>& vals,
                     std::vector<int>& order) {
    cols.clear();
    vals.clear();
    for (int64_t m = moff[a]; m < moff[a + 1]; ++m) {
      const int i = mrow[m];
      for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k) {
        const int c = agg[A.col[k]];
        if (pos[c] < 0) {
          pos[c] = (int64_t)cols.size();
          cols.push_back(c);
          vals.push_back(0.0);
        }
        vals[pos[c]] += A.val[k];
      }
    }
    order.resize(cols.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
    std::sort(order.begin(), order.end(), [&](int x, int y) { return cols[x] < cols[y]; });
    for (int c : cols) pos[c] = -1;
  };
  std::vector<int64_t> cnt(na);
#pragma omp parallel
  {
    std::vector<int64_t> pos(na, -1);
    std::vector<int> cols, order;
    std::vector<double> vals;
#pragma omp for schedule(static)
    for (int a = 0; a < na; ++a) {
      agg_row(a, pos, cols, vals, order);
      cnt[a] = (int64_t)cols.size();
    }
  }
  for (int a = 0; a < na; ++a) C.off[a + 1] = C.off[a] + cnt[a];
  C.col.resize(C.off[na]);
  C.val.resize(C.off[na]);
#pragma omp parallel
  {
    std::vector<int64_t> pos(na, -1);
    std::vector<int> cols, order;
    std::vector<double> vals;
#pragma omp for schedule(static)
    for (int a = 0; a < na; ++a) {
      agg_row(a, pos, cols, vals, order);
      int64_t o = C.off[a];
      for (int k : order) {
        C.col[o] = cols[k];
        C.val[o] = vals[k];
        ++o;
      }
    }
  }
  return C;
}

// Largest eigenvalue of D^-1 A by 30 power steps from a fixed start vector.  The norms are summed
// over fixed chunks of rows, then the chunks in order: the same value on any number of threads.
double lambda_max(const Csr& A, const std::vector<double>& dinv) {
  constexpr int CH = 16384;
  const int n = A.n, nch = (n + CH - 1) / CH;
  std::vector<double> v(n), w(n), pv(nch), pw(nch);
  for (int i = 0; i < n; ++i) v[i] = 1.0 + 0.5 * std::sin(0.7 * i + 0.3);
  double lam = 0.0;
  for (int it = 0; it < 30; ++it) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nch; ++c) {
      double nv = 0.0, nw = 0.0;
      const int i1 = std::min(n, (c + 1) * CH);
      for (int i = c * CH; i < i1; ++i) {
        double s = 0.0;
        for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k) s += A.val[k] * v[A.col[k]];
        w[i] = dinv[i] * s;
        nv += v[i] * v[i];
        nw += w[i] * w[i];
      }
      pv[c] = nv;
      pw[c] = nw;
    }
    double nv = 0.0, nw = 0.0;
    for (int c = 0; c < nch; ++c) { nv += pv[c]; nw += pw[c]; }
    if (!(nw > 0.0)) return 1.0;
    lam = std::sqrt(nw / nv);
    const double sc = 1.0 / std::sqrt(nw);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) v[i] = w[i] * sc;
  }
  return lam;
}

bool cholesky_lower(std::vector<double>& a, int n) {
  for (int j = 0; j < n; ++j) {
    double d = a[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= a[(size_t)j * n + k] * a[(size_t)j * n + k];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    a[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = a[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= a[(size_t)i * n + k] * a[(size_t)j * n + k];
      a[(size_t)i * n + j] = s / d;
    }
  }
  return true;
}

int dense_inverse(const Csr& A, bool nullsp, std::vector<float>& out) {
  const int n = A.n;
  std::vector<double> a((size_t)n * n, 0.0);
  double tr = 0.0;
  for (int i = 0; i < n; ++i)
    for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k) {
      a[(size_t)i * n + A.col[k]] += A.val[k];
      if (A.col[k] == i) tr += A.val[k];
    }
  if (nullsp) {  // constant mode lifted to the mean diagonal: (A + s 1 1^T) 1 = (tr / n) 1
    const double s = tr / ((double)n * n);
    for (auto& x : a) x += s;
  }
  if (!cholesky_lower(a, n)) return -4;
  out.assign((size_t)n * n, 0.0f);
  std::vector<double> y(n);
  for (int c = 0; c < n; ++c) {  // column c of the inverse: L L^T y = e_c
    for (int i = 0; i < n; ++i) {
      double s = i == c ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) s -= a[(size_t)i * n + k] * y[k];
      y[i] = s / a[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < n; ++k) s -= a[(size_t)k * n + i] * y[k];
      y[i] = s / a[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i) out[(size_t)i * n + c] = (float)y[i];
  }
  return 0;
}

// IEEE binary16 bits of a finite double, round to nearest even (subnormals included; values
// beyond the largest finite half saturate to it).
unsigned short half_bits(double v) {
  const unsigned short sign = std::signbit(v) ? 0x8000 : 0;
  double a = std::fabs(v);
  if (a >= 65504.0) return sign | 0x7bff;
  if (a < std::ldexp(1.0, -24) * 0.5) return sign;
  int e;
  std::frexp(a, &e);  // a = m 2^e, m in [0.5, 1)
  int ex = e - 1;     // a = (1.f) 2^ex
  if (ex < -14) ex = -14;  // subnormal range: fixed exponent, 10-bit fraction of 2^-24 units
  const double q = std::ldexp(a, 10 - ex);  // value in units of the last place
  double r = std::nearbyint(q);             // round half to even (default rounding mode)
  unsigned mant = (unsigned)r;
  if (mant >= 2048) { mant >>= 1; ex += 1; }  // rounding carried into the next binade
  if (ex > 15) return sign | 0x7bff;
  if (mant < 1024) return sign | (unsigned short)mant;  // subnormal (ex == -14)
  return sign | (unsigned short)(((ex + 15) << 10) | (mant - 1024));
}

double half_value(unsigned short h) {
  const int e = (h >> 10) & 0x1f, f = h & 0x3ff;
  const double m = e == 0 ? std::ldexp((double)f, -24) : std::ldexp(1024.0 + f, e - 25);
  return (h & 0x8000) ? -m : m;
}

MlLevel make_level(const Csr& A, const std::vector<int>& agg, int na, int& rc) {
  MlLevel L;
  rc = 0;
  L.n = A.n;
  for (int i = 0; i < A.n; ++i) L.W = std::max<int>(L.W, (int)(A.off[i + 1] - A.off[i]));
  L.dinv.resize(A.n);
  std::vector<double> dinv(A.n, 0.0);
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (int i = 0; i < A.n; ++i) {
    double dg = 0.0;
    for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k)
      if (A.col[k] == i) dg = A.val[k];
    if (!(dg > 0.0)) bad = 1;
    dinv[i] = dg > 0.0 ? 1.0 / dg : 0.0;
    L.dinv[i] = (float)dinv[i];
  }
  if (bad) rc = -5;
  L.lmax = lambda_max(A, dinv);
  // scaled off-diagonal form of the smoother
  for (int i = 0; i < A.n; ++i) L.Wo = std::max<int>(L.Wo, (int)(A.off[i + 1] - A.off[i]) - 1);
  L.Wo = std::max(L.Wo, 1);
  L.ocol.resize((size_t)L.Wo * A.n);
  L.sv32.assign((size_t)L.Wo * A.n, 0.0f);
  L.sv16.assign((size_t)L.Wo * A.n, 0);
  L.g32.resize(A.n);
  L.g16.resize(A.n);
  L.diag.resize(A.n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A.n; ++i) {
    int s = 0;
    double d32 = 1.0, d16 = 1.0;
    for (int64_t k = A.off[i]; k < A.off[i + 1]; ++k) {
      if (A.col[k] == i) continue;
      const double sij = A.val[k] * dinv[i];
      const float f = (float)sij;
      const unsigned short h = half_bits(sij);
      L.ocol[(size_t)s * A.n + i] = A.col[k];
      L.sv32[(size_t)s * A.n + i] = f;
      L.sv16[(size_t)s * A.n + i] = h;
      d32 += sij - (double)f;
      d16 += sij - half_value(h);
      ++s;
    }
    for (; s < L.Wo; ++s) L.ocol[(size_t)s * A.n + i] = i;
    L.g32[i] = (float)d32;
    L.g16[i] = (float)d16;
    L.diag[i] = (float)(dinv[i] > 0.0 ? 1.0 / dinv[i] : 0.0);
  }
  L.agg = agg;
  std::vector<int64_t> moff;
  std::vector<int> mrow;
  members(agg, na, moff, mrow);
  for (int a = 0; a < na; ++a) L.M = std::max<int>(L.M, (int)(moff[a + 1] - moff[a]));
  L.mem.assign((size_t)L.M * na, -1);
  for (int a = 0; a < na; ++a)
    for (int64_t m = moff[a]; m < moff[a + 1]; ++m) L.mem[(size_t)(m - moff[a]) * na + a] = mrow[m];
  return L;
}

}  // namespace

int build_multilevel(int n, int WA, const int* A_col, const double* A_val, bool nullsp, int passes, double beta,
                     int ncoarse, int max_dense, Multilevel& M) {
  if (n < 1 || WA < 1 || WA > 64 || passes < 1 || ncoarse < 1) return -1;
  M = Multilevel{};
  Csr A = csr_from_ell(n, WA, A_col, A_val);
  for (;;) {
    M.sizes.push_back(A.n);
    M.nnz.push_back((int64_t)A.col.size());
    if (A.n <= ncoarse) break;
    if ((int)M.lv.size() >= ML_MAX_LEVELS) {
      if (A.n > max_dense) return -3;
      break;
    }
    std::vector<int> agg_tot;
    Csr Ac;
    for (int p = 0; p < passes; ++p) {
      std::vector<int> agg;
      const Csr& from = p == 0 ? A : Ac;
      const int na = pairwise(from, beta, agg);
      Csr next = galerkin(from, agg, na);
      if (p == 0) agg_tot = agg;
      else
        for (int i = 0; i < A.n; ++i) agg_tot[i] = agg[agg_tot[i]];
      Ac = std::move(next);
    }
    if (Ac.n > 0.85 * A.n) {  // coarsening stalled: solve this level directly if it is small enough
      if (A.n > max_dense) return -2;
      break;
    }
    int rc = 0;
    M.lv.push_back(make_level(A, agg_tot, Ac.n, rc));
    if (rc) return rc;
    A = std::move(Ac);
  }
  M.nC = A.n;
  return dense_inverse(A, nullsp, M.cinv);
}

}  // namespace dpm
