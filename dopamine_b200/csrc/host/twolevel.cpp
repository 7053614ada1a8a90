#include "twolevel.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace dpm {
namespace {

// Split ids (cell indices) into parts [p0, p0+np) whose sizes are given by `size`, cutting
// along the axis of largest extent each time.  Ties are broken by cell index, so the result
// does not depend on the sort implementation.
void rcb(std::vector<int>& ids, size_t lo, size_t hi, int p0, int np, const std::vector<int64_t>& start,
         const double* xyz, std::vector<int>& part) {
  if (np == 1) {
    for (size_t k = lo; k < hi; ++k) part[ids[k]] = p0;
    return;
  }
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (size_t k = lo; k < hi; ++k)
    for (int a = 0; a < 3; ++a) {
      double v = xyz[3 * (size_t)ids[k] + a];
      mn[a] = std::min(mn[a], v);
      mx[a] = std::max(mx[a], v);
    }
  int ax = 0;
  for (int a = 1; a < 3; ++a)
    if (mx[a] - mn[a] > mx[ax] - mn[ax]) ax = a;
  const int nl = np / 2;
  const size_t cut = lo + (size_t)(start[p0 + nl] - start[p0]);
  auto less = [&](int a, int b) {
    double va = xyz[3 * (size_t)a + ax], vb = xyz[3 * (size_t)b + ax];
    return va < vb || (va == vb && a < b);
  };
  std::nth_element(ids.begin() + lo, ids.begin() + cut, ids.begin() + hi, less);
  rcb(ids, lo, cut, p0, nl, start, xyz, part);
  rcb(ids, cut, hi, p0 + nl, np - nl, start, xyz, part);
}

// bfloat16 bits of a float, round to nearest even (finite inputs).
unsigned bf16_bits(double v) {
  float f = (float)v;
  unsigned u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return u >> 16;
}

// In-place Cholesky of an SPD matrix (row-major n x n, lower factor); false if not SPD.
bool cholesky(std::vector<double>& a, int n) {
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

}  // namespace

int build_two_level(int n, int WA, const int* A_col, const double* A_val, const double* xyz, int P, bool nullsp,
                    TwoLevel& T, bool coarse) {
  if (n < 1 || WA < 1 || P < 1) return -1;
  int C = (n + P - 1) / P;
  P = (n + C - 1) / C;  // every part non-empty
  if (C > 32767) return -2;  // local columns are 16-bit
  T = TwoLevel{};
  T.n = n;
  T.P = P;
  T.C = C;
  T.WA = WA;
  std::vector<int64_t> start(P + 1);
  for (int b = 0; b <= P; ++b) start[b] = std::min<int64_t>((int64_t)b * C, n);
  std::vector<int> ids(n), part(n);
  std::iota(ids.begin(), ids.end(), 0);
  rcb(ids, 0, (size_t)n, 0, P, start, xyz, part);
  // new numbering: parts in order, original index order inside a part
  T.perm.resize(n);
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int i = 0; i < n; ++i) T.perm[fill[part[i]]++] = i;
  }
  std::vector<int> iperm(n);
  for (int i = 0; i < n; ++i) iperm[T.perm[i]] = i;

  T.col.assign((size_t)WA * n, 0);
  T.val.assign((size_t)WA * n, 0.0);
  T.dinv.assign(n, 1.0);
  std::vector<std::vector<std::pair<int, double>>> loc(n);
  std::vector<double> E(coarse ? (size_t)P * P : 0, 0.0);
  int WL = 0;
  for (int i = 0; i < n; ++i) {
    const int o = T.perm[i];
    const int b = i / C;
    std::vector<std::pair<int, double>> row;
    double dg = 0.0;
    for (int w = 0; w < WA; ++w) {
      int c = A_col[(size_t)w * n + o];
      double v = A_val[(size_t)w * n + o];
      if (v == 0.0) continue;
      int j = iperm[c];
      row.push_back({j, v});
      if (j == i) dg += v;
      if (coarse) E[(size_t)b * P + j / C] += v;
    }
    std::sort(row.begin(), row.end());
    for (size_t s = 0; s < row.size(); ++s) {
      T.col[s * n + i] = row[s].first;
      T.val[s * n + i] = row[s].second;
    }
    for (size_t s = row.size(); s < (size_t)WA; ++s) T.col[s * n + i] = i;
    T.dinv[i] = dg != 0.0 ? 1.0 / dg : 1.0;
    for (auto& e : row)
      if (e.first != i && e.first / C == b) loc[i].push_back({e.first - b * C, e.second});
    WL = std::max<int>(WL, (int)loc[i].size());
  }
  if (WL > 16) return -3;
  T.WL = std::max(WL, 1);
  T.lpk.assign((size_t)T.WL * n, 0u);
  for (int i = 0; i < n; ++i) {
    const unsigned self = (unsigned)(i % C);
    for (int s = 0; s < T.WL; ++s) {
      unsigned colv = self, hi = 0u;
      if (s < (int)loc[i].size()) {
        colv = (unsigned)loc[i][s].first;
        hi = bf16_bits(loc[i][s].second * T.dinv[i]);
      }
      T.lpk[(size_t)s * n + i] = colv | (hi << 16);
    }
  }
  if (!coarse) {  // intra-part row sums only
    T.srow.assign(n, 0.0f);
    T.xoff.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
      double sr = 0.0;
      for (int w = 0; w < WA; ++w) {
        const double v = T.val[(size_t)w * n + i];
        if (v != 0.0 && T.col[(size_t)w * n + i] / C == i / C) sr += v;
      }
      T.srow[i] = (float)sr;
    }
    T.xval.assign(1, 0.0f);
    T.xslot.assign(1, 0);
    return 0;
  }
  // coarse operator: with the constant null space, E is singular along the constant vector;
  // adding (mean diag / P) 1 1^T makes it SPD and leaves E^-1 unchanged on the complement.
  if (nullsp) {
    double s = 0.0;
    for (int b = 0; b < P; ++b) s += E[(size_t)b * P + b];
    s /= (double)P * P;
    for (auto& e : E) e += s;
  }
  std::vector<double> L = E;
  if (!cholesky(L, P)) return -4;
  T.einv.assign((size_t)P * P, 0.0);
  std::vector<double> y(P);
  for (int k = 0; k < P; ++k) {
    for (int i = 0; i < P; ++i) {
      double s = (i == k) ? 1.0 : 0.0;
      for (int j = 0; j < i; ++j) s -= L[(size_t)i * P + j] * y[j];
      y[i] = s / L[(size_t)i * P + i];
    }
    for (int i = P - 1; i >= 0; --i) {
      double s = y[i];
      for (int j = i + 1; j < P; ++j) s -= L[(size_t)j * P + i] * y[j];
      y[i] = s / L[(size_t)i * P + i];
    }
    for (int i = 0; i < P; ++i) T.einv[(size_t)i * P + k] = y[i];
  }
  // ---- deflation data
  std::vector<std::vector<int>> nb_of(P);
  for (int i = 0; i < n; ++i) {
    const int b = i / C;
    for (int w = 0; w < WA; ++w) {
      const double v = T.val[(size_t)w * n + i];
      const int j = T.col[(size_t)w * n + i];
      if (v != 0.0 && j / C != b) nb_of[b].push_back(j / C);
    }
  }
  int NB = 1;
  for (int b = 0; b < P; ++b) {
    auto& l = nb_of[b];
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
    NB = std::max<int>(NB, 1 + (int)l.size());
  }
  T.srow.assign(n, 0.0f);
  T.xoff.assign(n + 1, 0);
  if (NB <= 32) {
    T.deflate = 1;
    T.NB = NB;
    T.nbr.assign((size_t)P * NB, -1);
    T.einv_nb.assign((size_t)P * NB * P, 0.0);
    for (int b = 0; b < P; ++b) {
      T.nbr[(size_t)b * NB] = b;
      for (size_t s = 0; s < nb_of[b].size(); ++s) T.nbr[(size_t)b * NB + 1 + s] = nb_of[b][s];
      for (int s = 0; s < NB; ++s) {
        const int q = T.nbr[(size_t)b * NB + s];
        if (q >= 0)
          std::copy(T.einv.begin() + (size_t)q * P, T.einv.begin() + (size_t)(q + 1) * P,
                    T.einv_nb.begin() + ((size_t)b * NB + s) * P);
      }
    }
    for (int i = 0; i < n; ++i) {
      const int b = i / C;
      double sr = 0.0;
      for (int w = 0; w < WA; ++w) {
        const double v = T.val[(size_t)w * n + i];
        const int j = T.col[(size_t)w * n + i];
        if (v == 0.0) continue;
        if (j / C == b) {
          sr += v;
        } else {
          const auto& l = nb_of[b];
          const int s = 1 + (int)(std::lower_bound(l.begin(), l.end(), j / C) - l.begin());
          T.xslot.push_back((unsigned char)s);
          T.xval.push_back((float)v);
        }
      }
      T.srow[i] = (float)sr;
      T.xoff[i + 1] = (int)T.xval.size();
    }
  } else {
    T.deflate = 0;
    T.NB = 1;
    T.nbr.assign(P, 0);
    T.einv_nb = T.einv;
    for (int b = 0; b < P; ++b) T.nbr[b] = b;
  }
  if (T.xval.empty()) {  // keep device arrays non-empty
    T.xval.push_back(0.0f);
    T.xslot.push_back(0);
  }
  return 0;
}

}  // namespace dpm
