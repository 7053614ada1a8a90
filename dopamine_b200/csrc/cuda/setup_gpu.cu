// Device builder of the mesh and the static operator data; see setup_gpu.hpp.
//
// The translation unit is compiled with -fmad=false: every product and sum below is rounded as
// the host builder (csrc/host/mesh.cpp, ops.cpp, plain IEEE double on x86-64) rounds it, and
// every per-cell accumulation walks its terms in the host builder's order, so that the two
// builders agree value for value.  Layout of the work:
//   * cells: one thread per cell (centroid and volume by the tet decomposition);
//   * face matching: every element face becomes a record with its canonical node key (the
//     sorted node ids, padded with -1), packed into two 64-bit words; two stable LSD radix sorts
//     (low word, then high word) order the records by (key, cell, local face) exactly as the
//     host's comparison sort does, because records are generated in (cell, local face) order;
//     an interior face is created at the second record of each run of equal keys, and numbering
//     interior faces by that record's generation order reproduces the reference's numbering
//     (a face is created when its second cell reaches it);
//   * boundary faces: one thread per face, lower_bound of its key in the sorted records;
//   * per-cell lists (cell -> faces, vertex -> cells): counts by atomics, offsets by a scan,
//     slots by atomics, then each list sorted, which makes the result independent of the order
//     in which the atomics landed;
//   * LS stencil and per-cell operators: one thread per cell over its sorted lists.
//   * face-based (OpenFOAM) meshes skip the matching: their faces come in the file's order, and
//     polygon face geometry, polyhedron moments and face-ordered cell vertices (the reference's
//     OpenFOAM path) are one thread per face or cell before the shared stages.
// Periodic pairing (per patch, a sort of the patch's face centres) and the outlet rows stay on
// the host; they touch boundary faces only.  Per-cell work arrays have fixed capacities (16
// pressure-solver entries, 64 vertices): a cell beyond them makes the builder stop with
// SETUP_DEVICE_LIMIT before any kernel reads an incomplete list, and the caller uses the host
// builder.
#include "setup_gpu.hpp"

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace dpm {
namespace {

constexpr int STPB = 256;
constexpr int CPS_CAP = 16;   // pressure-solver entries per cell kept in registers
constexpr int AROW_CAP = 17;  // diagonal + CPS_CAP
constexpr double DBL_BIG = 1.7976931348623157e308;
constexpr int NONE_PAD = -2147483647 - 1;

inline unsigned nblocks(int64_t n) { return (unsigned)((n + STPB - 1) / STPB); }

__device__ __forceinline__ int64_t gtid() { return blockIdx.x * (int64_t)blockDim.x + threadIdx.x; }
// std::max / std::min semantics
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

// Element tables (src/mesh/mod_gmsh_reader.f90:get_element_faces; tet decomposition of
// hex_geometry, prism_geometry, pyramid_geometry), slots tet, hex, prism, pyramid.
__constant__ signed char c_ef[4][6][4] = {
    {{0, 1, 2, -1}, {0, 1, 3, -1}, {1, 2, 3, -1}, {0, 2, 3, -1}, {-1, -1, -1, -1}, {-1, -1, -1, -1}},
    {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {2, 3, 7, 6}, {0, 3, 7, 4}, {1, 2, 6, 5}},
    {{0, 1, 2, -1}, {3, 4, 5, -1}, {0, 1, 4, 3}, {1, 2, 5, 4}, {0, 2, 5, 3}, {-1, -1, -1, -1}},
    {{0, 1, 2, 3}, {0, 1, 4, -1}, {1, 2, 4, -1}, {2, 3, 4, -1}, {0, 3, 4, -1}, {-1, -1, -1, -1}}};
__constant__ signed char c_efn[4][6] = {{3, 3, 3, 3, 0, 0}, {4, 4, 4, 4, 4, 4}, {3, 3, 4, 4, 4, 0}, {4, 3, 3, 3, 3, 0}};
__constant__ signed char c_nface[4] = {4, 6, 5, 5};
__constant__ signed char c_tet[4][5][4] = {
    {{0, 1, 2, 3}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    {{0, 1, 3, 4}, {1, 2, 3, 6}, {3, 4, 6, 7}, {1, 4, 5, 6}, {1, 3, 4, 6}},
    {{0, 1, 2, 3}, {1, 3, 4, 2}, {2, 3, 4, 5}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    {{0, 1, 3, 4}, {1, 2, 3, 4}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}}};
__constant__ signed char c_ntet[4] = {1, 5, 3, 2};

__device__ __forceinline__ int tslot(int type) { return (type >= EL_TET4 && type <= EL_PYR5) ? type - EL_TET4 : -1; }

// ---- geometry --------------------------------------------------------------------------------

__device__ void d_tet(const double* p1, const double* p2, const double* p3, const double* p4, double c[3], double& v) {
  double a[3], b[3], d[3];
  for (int k = 0; k < 3; ++k) { a[k] = p2[k] - p1[k]; b[k] = p3[k] - p1[k]; d[k] = p4[k] - p1[k]; }
  v = fabs(a[0] * (b[1] * d[2] - b[2] * d[1]) - a[1] * (b[0] * d[2] - b[2] * d[0]) +
           a[2] * (b[0] * d[1] - b[1] * d[0])) / 6.0;
  for (int k = 0; k < 3; ++k) c[k] = (((p1[k] + p2[k]) + p3[k]) + p4[k]) / 4.0;
}

__device__ void d_face_geom(const int* fn, int nn, const double* xyz, double ce[3], double nr[3], double& area) {
  ce[0] = ce[1] = ce[2] = 0.0;
  for (int i = 0; i < nn; ++i)
    for (int k = 0; k < 3; ++k) ce[k] += xyz[3 * (int64_t)fn[i] + k];
  for (int k = 0; k < 3; ++k) ce[k] /= (double)nn;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < nn; ++i) {
    const double* pi = xyz + 3 * (int64_t)fn[i];
    const double* pj = xyz + 3 * (int64_t)fn[(i + 1) % nn];
    double a[3], b[3];
    for (int k = 0; k < 3; ++k) { a[k] = pi[k] - ce[k]; b[k] = pj[k] - ce[k]; }
    double cr0 = a[1] * b[2] - a[2] * b[1], cr1 = a[2] * b[0] - a[0] * b[2], cr2 = a[0] * b[1] - a[1] * b[0];
    acc[0] += 0.5 * cr0;
    acc[1] += 0.5 * cr1;
    acc[2] += 0.5 * cr2;
  }
  area = sqrt(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2]);
  for (int k = 0; k < 3; ++k) nr[k] = acc[k] / (area + SMALL);
}

__device__ __forceinline__ double ddot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__device__ void d_invert3x3(const double A[3][3], double Ai[3][3], double& det) {
  double c11 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  double c12 = -(A[1][0] * A[2][2] - A[1][2] * A[2][0]);
  double c13 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  double c21 = -(A[0][1] * A[2][2] - A[0][2] * A[2][1]);
  double c22 = A[0][0] * A[2][2] - A[0][2] * A[2][0];
  double c23 = -(A[0][0] * A[2][1] - A[0][1] * A[2][0]);
  double c31 = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  double c32 = -(A[0][0] * A[1][2] - A[0][2] * A[1][0]);
  double c33 = A[0][0] * A[1][1] - A[0][1] * A[1][0];
  det = A[0][0] * c11 + A[0][1] * c12 + A[0][2] * c13;
  double m = dmax(fabs(det), SMALL);
  double idet = 1.0 / (det < 0 ? -m : m);
  Ai[0][0] = c11 * idet; Ai[0][1] = c21 * idet; Ai[0][2] = c31 * idet;
  Ai[1][0] = c12 * idet; Ai[1][1] = c22 * idet; Ai[1][2] = c32 * idet;
  Ai[2][0] = c13 * idet; Ai[2][1] = c23 * idet; Ai[2][2] = c33 * idet;
}

// Canonical face key: node ids sorted ascending, padded with -1; packed (k0+1, k1+1) into the
// high word and (k2+1, k3+1) into the low word, B bits per id.
__device__ __forceinline__ void d_key(const int* fn, int nn, int B, unsigned long long& hi, unsigned long long& lo) {
  int k[4] = {-1, -1, -1, -1};
  for (int i = 0; i < nn; ++i) k[i] = fn[i];
  for (int i = 1; i < nn; ++i) {
    int t = k[i], j = i - 1;
    while (j >= 0 && k[j] > t) { k[j + 1] = k[j]; --j; }
    k[j + 1] = t;
  }
  hi = ((unsigned long long)(unsigned)(k[0] + 1) << B) | (unsigned long long)(unsigned)(k[1] + 1);
  lo = ((unsigned long long)(unsigned)(k[2] + 1) << B) | (unsigned long long)(unsigned)(k[3] + 1);
}

__device__ __forceinline__ void elem_face(int s, const int* n, int fi, int fn[4], int& nn) {
  nn = c_efn[s][fi];
  for (int j = 0; j < nn; ++j) fn[j] = n[c_ef[s][fi][j]];
}

// ---- kernels: cells and face matching --------------------------------------------------------

__global__ void k_cells(int64_t nc, const int* type, const int64_t* coff, const int* cn, const double* xyz, double* cen,
                        double* vol, long long* nfc, int* bad) {
  int64_t c = gtid();
  if (c >= nc) return;
  int s = tslot(type[c]);
  if (s < 0) {
    nfc[c] = 0;
    atomicOr(bad, 1);
    return;
  }
  nfc[c] = c_nface[s];
  const int* n = cn + coff[c];
  double cc[3], v;
  if (s == 0) {
    d_tet(xyz + 3 * (int64_t)n[0], xyz + 3 * (int64_t)n[1], xyz + 3 * (int64_t)n[2], xyz + 3 * (int64_t)n[3], cc, v);
  } else {
    v = 0.0;
    cc[0] = cc[1] = cc[2] = 0.0;
    for (int i = 0; i < c_ntet[s]; ++i) {
      double tc[3], tv;
      d_tet(xyz + 3 * (int64_t)n[c_tet[s][i][0]], xyz + 3 * (int64_t)n[c_tet[s][i][1]],
            xyz + 3 * (int64_t)n[c_tet[s][i][2]], xyz + 3 * (int64_t)n[c_tet[s][i][3]], tc, tv);
      v += tv;
      for (int k = 0; k < 3; ++k) cc[k] += tv * tc[k];
    }
    if (v > SMALL)
      for (int k = 0; k < 3; ++k) cc[k] /= v;
  }
  for (int k = 0; k < 3; ++k) cen[3 * c + k] = cc[k];
  vol[c] = v;
}

__global__ void k_records(int64_t nc, const int* type, const int64_t* coff, const int* cn, const long long* roff, int B,
                          unsigned long long* hi, unsigned long long* lo, int* rcell, unsigned char* rfi, int* rid) {
  int64_t c = gtid();
  if (c >= nc) return;
  int s = tslot(type[c]);
  if (s < 0) return;
  const int* n = cn + coff[c];
  const long long base = roff[c];
  for (int i = 0; i < c_nface[s]; ++i) {
    int fn[4], nn;
    elem_face(s, n, i, fn, nn);
    d_key(fn, nn, B, hi[base + i], lo[base + i]);
    rcell[base + i] = (int)c;
    rfi[base + i] = (unsigned char)i;
    rid[base + i] = (int)(base + i);
  }
}

__global__ void k_gather64(int64_t n, const unsigned long long* src, const int* perm, unsigned long long* dst) {
  int64_t i = gtid();
  if (i < n) dst[i] = src[perm[i]];
}

// Runs of equal keys: every member is matched; the run's second record creates an interior face
// owned by the first record's cell.
__global__ void k_match(int64_t n, const unsigned long long* hs, const unsigned long long* ls, const int* perm,
                        const int* rcell, unsigned char* matched, int* sflag, int* sowner) {
  int64_t i = gtid();
  if (i >= n) return;
  bool eqp = i > 0 && hs[i] == hs[i - 1] && ls[i] == ls[i - 1];
  bool eqn = i + 1 < n && hs[i + 1] == hs[i] && ls[i + 1] == ls[i];
  matched[i] = (eqp || eqn) ? 1 : 0;
  if (!eqp && eqn) {
    int r2 = perm[i + 1];
    sflag[r2] = 1;
    sowner[r2] = rcell[perm[i]];
  }
}

__global__ void k_int_faces(int64_t nrec, const int* sflag, const int* sidx, const int* sowner, const int* rcell,
                            const unsigned char* rfi, const int* type, const int64_t* coff, const int* cn,
                            const double* xyz, const double* cen, int* owner, int* nbr, int* patch, double* area,
                            double* centre, double* normal) {
  int64_t r = gtid();
  if (r >= nrec || !sflag[r]) return;
  const int f = sidx[r], c2 = rcell[r], o = sowner[r];
  int fn[4], nn;
  elem_face(tslot(type[c2]), cn + coff[c2], rfi[r], fn, nn);
  double ce[3], nr[3], a;
  d_face_geom(fn, nn, xyz, ce, nr, a);
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = cen[3 * (int64_t)c2 + k] - cen[3 * (int64_t)o + k];
  if (ddot(nr, d) < 0.0)
    for (int k = 0; k < 3; ++k) nr[k] = -nr[k];
  owner[f] = o;
  nbr[f] = c2;
  patch[f] = -1;
  area[f] = a;
  for (int k = 0; k < 3; ++k) {
    centre[3 * (int64_t)f + k] = ce[k];
    normal[3 * (int64_t)f + k] = nr[k];
  }
}

__global__ void k_bnd_faces(int64_t nfb, const int64_t* boff, const int* bnodes, const int* bpatch, const long long* bpos,
                            int64_t nfi, int B, int64_t nrec, const unsigned long long* hs, const unsigned long long* ls,
                            const int* perm, const int* rcell, const double* xyz, const double* cen,
                            unsigned char* matched, int* bad, int* owner, int* nbr, int* patch, double* area,
                            double* centre, double* normal) {
  int64_t b = gtid();
  if (b >= nfb) return;
  const int* fn = bnodes + boff[b];
  const int nn = (int)(boff[b + 1] - boff[b]);
  if (nn < 3 || nn > 4) {
    atomicOr(bad, 4);
    return;
  }
  unsigned long long kh, kl;
  d_key(fn, nn, B, kh, kl);
  int64_t lo = 0, hi = nrec;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (hs[mid] < kh || (hs[mid] == kh && ls[mid] < kl)) lo = mid + 1;
    else hi = mid;
  }
  if (lo == nrec || hs[lo] != kh || ls[lo] != kl) {
    atomicOr(bad, 2);
    return;
  }
  matched[lo] = 1;
  const int o = rcell[perm[lo]];
  double ce[3], nr[3], a;
  d_face_geom(fn, nn, xyz, ce, nr, a);
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = ce[k] - cen[3 * (int64_t)o + k];
  if (ddot(nr, d) < 0.0)
    for (int k = 0; k < 3; ++k) nr[k] = -nr[k];
  const int64_t f = nfi + bpos[b];
  owner[f] = o;
  nbr[f] = -1;
  patch[f] = bpatch[b];
  area[f] = a;
  for (int k = 0; k < 3; ++k) {
    centre[3 * f + k] = ce[k];
    normal[3 * f + k] = nr[k];
  }
}

__global__ void k_count_zero(int64_t n, const unsigned char* v, unsigned long long* cnt) {
  int64_t i = gtid();
  if (i < n && !v[i]) atomicAdd(cnt, 1ULL);
}

// Face geometry (mod_mesh.f90:mesh_compute_geometry, mesh_tag_refinement_faces).
__global__ void k_face_metrics(int64_t nf, const int* owner, const int* nbr, const double* area, const double* normal,
                               const double* centre, const double* cen, double* sf, double* dcf, double* gc,
                               double* eps, double* skew, unsigned char* isref) {
  int64_t f = gtid();
  if (f >= nf) return;
  for (int k = 0; k < 3; ++k) sf[3 * f + k] = area[f] * normal[3 * f + k];
  const double* co = cen + 3 * (int64_t)owner[f];
  const double* ce = centre + 3 * f;
  if (nbr[f] >= 0) {
    const double* cn = cen + 3 * (int64_t)nbr[f];
    double d_on[3], d_oc[3];
    for (int k = 0; k < 3; ++k) { d_on[k] = cn[k] - co[k]; d_oc[k] = ce[k] - co[k]; }
    double d_on2 = d_on[0] * d_on[0] + d_on[1] * d_on[1] + d_on[2] * d_on[2];
    double dc = dmax(sqrt(d_on2), 1.0e-30);
    double w = ddot(d_oc, d_on) / (d_on2 + SMALL);
    double g = dmax(0.0, dmin(1.0, 1.0 - w));
    double s2 = 0.0;
    for (int k = 0; k < 3; ++k) {
      eps[3 * f + k] = ce[k] - (co[k] + (1.0 - g) * (cn[k] - co[k]));
      double em = ce[k] - 0.5 * (co[k] + cn[k]);
      s2 += em * em;
    }
    double sk = sqrt(s2) / dmax(dc, 1.0e-30);
    dcf[f] = dc;
    gc[f] = g;
    skew[f] = sk;
    isref[f] = sk > REFINE_SKEW_TOL ? 1 : 0;
  } else {
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = ce[k] - co[k];
    dcf[f] = dmax(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), 1.0e-30);
    gc[f] = 1.0;
    for (int k = 0; k < 3; ++k) eps[3 * f + k] = 0.0;
    skew[f] = 0.0;
    isref[f] = 0;
  }
}

// ---- kernels: CSR lists ----------------------------------------------------------------------

__global__ void k_cf_count(int64_t nf, const int* owner, const int* nbr, unsigned long long* cnt) {
  int64_t f = gtid();
  if (f >= nf) return;
  atomicAdd(&cnt[owner[f]], 1ULL);
  if (nbr[f] >= 0) atomicAdd(&cnt[nbr[f]], 1ULL);
}

__global__ void k_cf_fill(int64_t nf, const int* owner, const int* nbr, unsigned long long* cur, int* list) {
  int64_t f = gtid();
  if (f >= nf) return;
  list[atomicAdd(&cur[owner[f]], 1ULL)] = (int)f;
  if (nbr[f] >= 0) list[atomicAdd(&cur[nbr[f]], 1ULL)] = (int)f;
}

__global__ void k_vc_count(int64_t nc, const int64_t* coff, const int* cn, unsigned long long* cnt) {
  int64_t c = gtid();
  if (c >= nc) return;
  for (int64_t k = coff[c]; k < coff[c + 1]; ++k) atomicAdd(&cnt[cn[k]], 1ULL);
}

__global__ void k_vc_fill(int64_t nc, const int64_t* coff, const int* cn, unsigned long long* cur, int* list) {
  int64_t c = gtid();
  if (c >= nc) return;
  for (int64_t k = coff[c]; k < coff[c + 1]; ++k) list[atomicAdd(&cur[cn[k]], 1ULL)] = (int)c;
}

// Sorts every CSR row ascending (rows are short: faces of a cell, cells of a vertex).
__global__ void k_sort_rows(int64_t n, const long long* off, int* list) {
  int64_t r = gtid();
  if (r >= n) return;
  int* a = list + off[r];
  const int64_t len = off[r + 1] - off[r];
  for (int64_t i = 1; i < len; ++i) {
    int t = a[i];
    int64_t j = i - 1;
    while (j >= 0 && a[j] > t) { a[j + 1] = a[j]; --j; }
    a[j + 1] = t;
  }
}

// ---- kernels: LS stencil (mod_mesh.f90:mesh_build_ls_stencil) --------------------------------

__global__ void k_ls_neigh(int64_t nc, int max_st, const long long* cfo, const int* cfl, const int* owner,
                           const int* nbr, const int* patch, const int* pbc, int64_t nfi, const int* ppair,
                           const int64_t* coff, const int* cn, const long long* voff, const int* vcell, int* tnb,
                           int* tface, unsigned char* tper, long long* cnt_out) {
  int64_t i = gtid();
  if (i >= nc) return;
  int cnt = 0;
  for (long long idx = cfo[i]; idx < cfo[i + 1]; ++idx) {
    int f = cfl[idx];
    int nb = owner[f];
    if (nb == i) nb = nbr[f];
    bool is_per = false;
    if (nb < 0) {
      int64_t fb = f - nfi;
      int p = patch[f];
      if (p >= 0 && pbc[p] == BC_PERIODIC) {
        int pb = ppair[fb];
        if (pb >= 0) nb = owner[nfi + pb];
        if (nb >= 0) is_per = true;
      }
      if (nb < 0) nb = -1;
    }
    int64_t s = (int64_t)cnt * nc + i;
    tnb[s] = nb;
    tper[s] = is_per ? 1 : 0;
    tface[s] = nb == -1 ? f : -1;
    ++cnt;
  }
  for (int64_t k = coff[i]; k < coff[i + 1]; ++k) {
    int v = cn[k];
    for (long long kk = voff[v]; kk < voff[v + 1]; ++kk) {
      int cnb = vcell[kk];
      if (cnb == i) continue;
      bool found = false;
      for (int j = 0; j < cnt; ++j)
        if (tnb[(int64_t)j * nc + i] == cnb) { found = true; break; }
      if (found) continue;
      if (cnt < max_st) {
        int64_t s = (int64_t)cnt * nc + i;
        tnb[s] = cnb;
        tper[s] = 0;
        tface[s] = -1;
        ++cnt;
      }
    }
  }
  cnt_out[i] = cnt;
}

struct LsArgs {
  int64_t nc, nfi, nfb;
  const long long *ls_off, *cfo;
  const int *tnb, *tface, *cfl;
  const unsigned char* tper;
  const double *cen, *dcf, *normal, *centre, *ppdcf;
  int *ls_cell, *ls_face;
  double* ls_w;
  unsigned long long* ndeg;
};

__device__ __forceinline__ void ls_offset(const LsArgs& a, int64_t i, int idx, double d[3]) {
  int64_t s = (int64_t)idx * a.nc + i;
  int nb = a.tnb[s];
  const double* ci = a.cen + 3 * i;
  if (nb >= 0 && a.tper[s]) {
    int f = a.cfl[a.cfo[i] + idx];
    double dpo = a.dcf[f], dpn = dpo;
    int64_t fb = f - a.nfi;
    if (fb >= 0 && fb < a.nfb && a.ppdcf[fb] > 0.0) dpn = a.ppdcf[fb];
    for (int k = 0; k < 3; ++k) d[k] = (dpo + dpn) * a.normal[3 * (int64_t)f + k];
  } else if (nb >= 0) {
    for (int k = 0; k < 3; ++k) d[k] = a.cen[3 * (int64_t)nb + k] - ci[k];
  } else {
    int f = a.cfl[a.cfo[i] + idx];
    for (int k = 0; k < 3; ++k) d[k] = a.centre[3 * (int64_t)f + k] - ci[k];
  }
}

__global__ void k_ls_weights(LsArgs a) {
  int64_t i = gtid();
  if (i >= a.nc) return;
  const long long off = a.ls_off[i];
  const int cnt = (int)(a.ls_off[i + 1] - off);
  double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int idx = 0; idx < cnt; ++idx) {
    int64_t s = (int64_t)idx * a.nc + i;
    a.ls_cell[off + idx] = a.tnb[s];
    a.ls_face[off + idx] = a.tface[s];
    double d[3];
    ls_offset(a, i, idx, d);
    double w = 1.0 / (sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + SMALL);
    double ww = w * w;
    A[0][0] += ww * d[0] * d[0]; A[0][1] += ww * d[0] * d[1];
    A[0][2] += ww * d[0] * d[2]; A[1][1] += ww * d[1] * d[1];
    A[1][2] += ww * d[1] * d[2]; A[2][2] += ww * d[2] * d[2];
  }
  A[1][0] = A[0][1]; A[2][0] = A[0][2]; A[2][1] = A[1][2];
  double scale = (A[0][0] + A[1][1] + A[2][2]) / 3.0;
  double Ai[3][3], det;
  d_invert3x3(A, Ai, det);
  if (scale <= 0.0 || fabs(det) < LS_DET_TOL * (scale * scale * scale)) {
    for (int k = 0; k < 3; ++k) A[k][k] += LS_REG_FRAC * dmax(scale, SMALL);
    d_invert3x3(A, Ai, det);
    atomicAdd(a.ndeg, 1ULL);
  }
  for (int idx = 0; idx < cnt; ++idx) {
    double d[3];
    ls_offset(a, i, idx, d);
    double w = 1.0 / (sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + SMALL);
    double r[3] = {w * w * d[0], w * w * d[1], w * w * d[2]};
    for (int k = 0; k < 3; ++k) a.ls_w[3 * (off + idx) + k] = Ai[k][0] * r[0] + Ai[k][1] * r[1] + Ai[k][2] * r[2];
  }
}

// ---- kernels: static operators (ops.cpp) -------------------------------------------------------

// Interior pressure-solver faces (mod_pressure_solver.f90:pressure_solver_init).
__global__ void k_ps_interior(int64_t nfi, const int* owner, const int* nbr, const double* cen, const double* normal,
                              const double* area, const double* dcf, double cfl, int* pso, int* psn, int* psf,
                              double* psc, int* bad) {
  int64_t f = gtid();
  if (f >= nfi) return;
  int o = owner[f], n = nbr[f];
  pso[f] = o;
  psn[f] = n;
  psf[f] = (int)f;
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = cen[3 * (int64_t)n + k] - cen[3 * (int64_t)o + k];
  double dor = ddot(d, normal + 3 * f);
  if (cfl > 0.0 && dor < cfl * dcf[f]) dor = cfl * dcf[f];
  double coeff = dor > SMALL ? area[f] / dor : area[f] / (dcf[f] + SMALL);
  if (!(fabs(coeff) <= DBL_BIG) || coeff <= SMALL) atomicOr(bad, 1);
  psc[f] = coeff;
}

// Over-relaxed Jasak k-vector (mod_nonortho.f90:65-99) of every pressure-solver face, kept where
// the face is non-orthogonal; [3][nfp].
__global__ void k_ps_jasak(int64_t nfp, const int* pso, const int* psn, const int* psf, const double* sf,
                           const double* cen, double cfl, double* kk, unsigned long long* n_active) {
  int64_t i = gtid();
  if (i >= nfp) return;
  const int o = pso[i], n = psn[i];
  const double* s = sf + 3 * (int64_t)psf[i];
  double d[3], k[3];
  for (int j = 0; j < 3; ++j) d[j] = cen[3 * (int64_t)n + j] - cen[3 * (int64_t)o + j];
  double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (len < 1.0e-30) {
    k[0] = k[1] = k[2] = 0.0;
  } else {
    double inv = 1.0 / len, sdd = ddot(s, d) * inv, dl = sdd * len, s2 = ddot(s, s);
    if (cfl > 0.0) dl = dmax(dl, cfl * sqrt(s2) * len);
    if (dl > 1.0e-30)
      for (int j = 0; j < 3; ++j) k[j] = s[j] - (s2 / dl) * d[j];
    else
      for (int j = 0; j < 3; ++j) k[j] = s[j] - (sdd * inv) * d[j];
  }
  const double NONORTHO_SIN2_TOL = 1.0e-10;
  bool act = ddot(k, k) >= NONORTHO_SIN2_TOL * ddot(s, s);
  for (int j = 0; j < 3; ++j) kk[j * nfp + i] = act ? k[j] : 0.0;
  if (act) atomicAdd(n_active, 1ULL);
}

// Per-cell pressure-solver list: ps idx (owner side) or ~idx (neighbour side), ascending idx;
// boundary-face list; [slot][nc] with PAD.
__global__ void k_cell_lists(int64_t nc, int64_t nfi, const long long* cfo, const int* cfl, const int* owner,
                             const int* bps, const unsigned char* bcanon, int* cf_ell, int S, int* cps_ell, int* cb_ell,
                             int SB, int* widths, int* bad) {
  // S and SB: allocated widths (at least 1), padded with PAD
  int64_t c = gtid();
  if (c >= nc) return;
  int e[CPS_CAP];
  int ne = 0, nbd = 0, s = 0;
  for (long long k = cfo[c]; k < cfo[c + 1]; ++k, ++s) {
    int f = cfl[k];
    cf_ell[(int64_t)s * nc + c] = f;
    int entry;
    bool has = true;
    if (f < nfi) {
      entry = owner[f] == c ? f : ~f;
    } else {
      int64_t b = f - nfi;
      cb_ell[(int64_t)nbd * nc + c] = (int)b;
      ++nbd;
      int i = bps[b];
      has = i >= 0;
      entry = bcanon[b] ? i : ~i;
    }
    if (has) {
      if (ne == CPS_CAP) atomicOr(bad, 2);  // the host stops before any kernel reads this cell's list
      else e[ne++] = entry;
    }
  }
  for (; s < S; ++s) cf_ell[(int64_t)s * nc + c] = NONE_PAD;
  for (int q = nbd; q < SB; ++q) cb_ell[(int64_t)q * nc + c] = NONE_PAD;
  for (int i = 1; i < ne; ++i) {
    int t = e[i], kt = t >= 0 ? t : ~t, j = i - 1;
    while (j >= 0 && (e[j] >= 0 ? e[j] : ~e[j]) > kt) { e[j + 1] = e[j]; --j; }
    e[j + 1] = t;
  }
  for (int i = 0; i < ne; ++i) cps_ell[(int64_t)i * nc + c] = e[i];
  for (int i = ne; i < CPS_CAP; ++i) cps_ell[(int64_t)i * nc + c] = NONE_PAD;
  atomicMax(&widths[0], ne);
}

// Diagonal: periodic pairs first, then interior faces, then outlet rows, each in list order
// (the host builder's accumulation order).
__global__ void k_diag(int64_t nc, int64_t nfi, int SB, const int* cps_ell, const int* cb_ell, const double* psc,
                       const double* bdiag, const unsigned char* bdiag_on, double* diag) {
  int64_t c = gtid();
  if (c >= nc) return;
  double s = 0.0;
  for (int pass = 0; pass < 2; ++pass)
    for (int q = 0; q < CPS_CAP; ++q) {
      int e = cps_ell[(int64_t)q * nc + c];
      if (e == NONE_PAD) break;
      int i = e >= 0 ? e : ~e;
      if ((pass == 0) == (i >= nfi)) s += psc[i];
    }
  for (int q = 0; q < SB; ++q) {
    int b = cb_ell[(int64_t)q * nc + c];
    if (b == NONE_PAD) break;
    if (bdiag_on[b]) s += bdiag[b];
  }
  if (!(s > SMALL) || !(s <= DBL_BIG)) s = 1.0;
  diag[c] = s;
}

// Assembled row: (self, diag) then one entry per pressure-solver face in idx order, stable-sorted
// by column, equal columns summed in that order; pass 0 counts, pass 1 writes ELL [WA][nc].
__global__ void k_arow(int64_t nc, const int* cps_ell, const int* pso, const int* psn, const double* psc,
                       const double* diag, int WA, int* Acol, double* Aval, int* width) {
  int64_t c = gtid();
  if (c >= nc) return;
  int col[AROW_CAP];
  double val[AROW_CAP];
  int n = 0;
  col[n] = (int)c;
  val[n] = diag[c];
  ++n;
  for (int q = 0; q < CPS_CAP; ++q) {
    int e = cps_ell[(int64_t)q * nc + c];
    if (e == NONE_PAD) break;
    int i = e >= 0 ? e : ~e;
    if (psc[i] == 0.0) continue;
    col[n] = e >= 0 ? psn[i] : pso[i];
    val[n] = -psc[i];
    ++n;
  }
  for (int i = 1; i < n; ++i) {
    int tc = col[i];
    double tv = val[i];
    int j = i - 1;
    while (j >= 0 && col[j] > tc) { col[j + 1] = col[j]; val[j + 1] = val[j]; --j; }
    col[j + 1] = tc;
    val[j + 1] = tv;
  }
  int m = 0;
  for (int i = 0; i < n; ++i) {
    if (m > 0 && col[m - 1] == col[i]) val[m - 1] += val[i];
    else { col[m] = col[i]; val[m] = val[i]; ++m; }
  }
  if (!Acol) {
    atomicMax(width, m);
    return;
  }
  for (int w = 0; w < WA; ++w) {
    Acol[(int64_t)w * nc + c] = w < m ? col[w] : (int)c;
    Aval[(int64_t)w * nc + c] = w < m ? val[w] : 0.0;
  }
}

// LS stencil as ELL: [W][nc] indices (cell, -(b+1) boundary entry, -(nb+1) cell value, PAD) and
// [3][W][nc] weights.
__global__ void k_ls_ell(int64_t nc, int64_t nfi, int64_t nb, int W, const long long* ls_off, const int* ls_cell,
                         const int* ls_face, const double* ls_w, int* idx, double* w) {
  int64_t c = gtid();
  if (c >= nc) return;
  const long long off = ls_off[c];
  const int cnt = (int)(ls_off[c + 1] - off);
  for (int s = 0; s < W; ++s) {
    if (s < cnt) {
      int n = ls_cell[off + s];
      int v;
      if (n >= 0) v = n;
      else {
        int f = ls_face[off + s];
        int64_t b = f >= 0 ? f - nfi : -1;
        v = (b >= 0 && b < nb) ? -(int)(b + 1) : -(int)(nb + 1);
      }
      idx[(int64_t)s * nc + c] = v;
      for (int j = 0; j < 3; ++j) w[((int64_t)j * W + s) * nc + c] = ls_w[3 * (off + s) + j];
    } else {
      idx[(int64_t)s * nc + c] = NONE_PAD;
      for (int j = 0; j < 3; ++j) w[((int64_t)j * W + s) * nc + c] = 0.0;
    }
  }
}

// Reconstruction operator T^-1 (mod_fv_solver.f90:build_reconstruct_operator): pressure-solver
// faces in idx order, then non-periodic boundary faces in boundary order; [nc][9].
__global__ void k_tinv(int64_t nc, int64_t nfi, int SB, const int* cps_ell, const int* cb_ell, const int* psf,
                       const int* bbc, const double* area, const double* normal, double* Tinv) {
  int64_t c = gtid();
  if (c >= nc) return;
  double T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  auto add = [&](int64_t f) {
    const double* n = normal + 3 * f;
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) T[i + 3 * j] += area[f] * n[i] * n[j];
  };
  for (int q = 0; q < CPS_CAP; ++q) {
    int e = cps_ell[(int64_t)q * nc + c];
    if (e == NONE_PAD) break;
    add(psf[e >= 0 ? e : ~e]);
  }
  for (int q = 0; q < SB; ++q) {
    int b = cb_ell[(int64_t)q * nc + c];
    if (b == NONE_PAD) break;
    if (bbc[b] != BC_PERIODIC) add(nfi + b);
  }
  double a11 = T[0], a21 = T[1], a31 = T[2], a12 = T[3], a22 = T[4], a32 = T[5], a13 = T[6], a23 = T[7], a33 = T[8];
  double c11 = a22 * a33 - a23 * a32, c12 = a13 * a32 - a12 * a33, c13 = a12 * a23 - a13 * a22;
  double c22 = a11 * a33 - a13 * a31, c23 = a13 * a21 - a11 * a23, c33 = a11 * a22 - a12 * a21;
  double det = a11 * c11 + a12 * (a23 * a31 - a21 * a33) + a13 * (a21 * a32 - a22 * a31);
  double tr = a11 + a22 + a33, mt = dmax(tr, SMALL);
  double* Ti = Tinv + 9 * c;
  if (fabs(det) <= 1.0e-12 * mt * mt * mt) {
    for (int k = 0; k < 9; ++k) Ti[k] = 0.0;
    Ti[0] = Ti[4] = Ti[8] = 3.0 / mt;
    return;
  }
  Ti[0] = c11 / det; Ti[3] = c12 / det; Ti[6] = c13 / det;
  Ti[1] = c12 / det; Ti[4] = c22 / det; Ti[7] = c23 / det;
  Ti[2] = c13 / det; Ti[5] = c23 / det; Ti[8] = c33 / det;
}

// SGS filter tensor with det G = V^2 (src/sgs/mod_vreman.f90:build_filter_tensor); [nc][9].
__global__ void k_filter(int64_t nc, const long long* cfo, const int* cfl, const double* centre, const double* cen,
                         const double* area, const double* vol, double* G) {
  int64_t c = gtid();
  if (c >= nc) return;
  double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long k = cfo[c]; k < cfo[c + 1]; ++k) {
    int64_t f = cfl[k];
    double dx[3];
    for (int j = 0; j < 3; ++j) dx[j] = centre[3 * f + j] - cen[3 * c + j];
    for (int n = 0; n < 3; ++n)
      for (int i = 0; i < 3; ++i) g[i + 3 * n] += area[f] * dx[i] * dx[n];
  }
  double dt = g[0] * (g[4] * g[8] - g[7] * g[5]) - g[3] * (g[1] * g[8] - g[7] * g[2]) + g[6] * (g[1] * g[5] - g[4] * g[2]);
  double t = (g[0] + g[4] + g[8]) / 3.0, t3 = t * t * t;
  double* Gc = G + 9 * c;
  if (t3 > 0.0 && dt > 1.0e-12 * t3) {
    double s = pow(vol[c] * vol[c] / dt, 1.0 / 3.0);
    for (int j = 0; j < 9; ++j) Gc[j] = s * g[j];
  } else {
    double d2 = pow(vol[c], 2.0 / 3.0);
    for (int j = 0; j < 9; ++j) Gc[j] = 0.0;
    Gc[0] = Gc[4] = Gc[8] = d2;
  }
}

// One face-area smoothing pass (src/sgs/mod_vreman.f90:smooth_filter_tensor): interior faces of
// the cell in face order.
__global__ void k_filter_smooth(int64_t nc, int64_t nfi, const long long* cfo, const int* cfl, const int* owner,
                                const int* nbr, const double* area, const double* Gin, double* Gout) {
  int64_t c = gtid();
  if (c >= nc) return;
  double gn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, ws = 0.0;
  for (long long k = cfo[c]; k < cfo[c + 1]; ++k) {
    int f = cfl[k];
    if (f >= nfi) continue;
    int other = owner[f] == c ? nbr[f] : owner[f];
    double a = area[f];
    for (int j = 0; j < 9; ++j) gn[j] += a * Gin[9 * (int64_t)other + j];
    ws += a;
  }
  for (int j = 0; j < 9; ++j)
    Gout[9 * c + j] = ws > SMALL ? 0.5 * Gin[9 * c + j] + 0.5 * gn[j] / ws : Gin[9 * c + j];
}

__global__ void k_wblend(int64_t nf, int64_t nfi, const double* skew, double* wbl) {
  int64_t f = gtid();
  if (f >= nf) return;
  if (f >= nfi) {
    wbl[f] = 1.0;
    return;
  }
  double t = (skew[f] - SKEW_BLEND_LO) / (SKEW_BLEND_HI - SKEW_BLEND_LO);
  t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
  wbl[f] = 1.0 - t * t * (3.0 - 2.0 * t);
}

// ---- kernels: face-based (polyhedral) meshes ---------------------------------------------------

// Polygon face geometry (src/mesh/mod_mesh.f90:compute_polygon_face_geometry), as build_mesh_poly.
__global__ void k_poly_faces(int64_t nf, const int64_t* foff, const int* fnodes, const double* xyz, double* area,
                             double* centre, double* normal) {
  int64_t f = gtid();
  if (f >= nf) return;
  const int* fn = fnodes + foff[f];
  const int nn = (int)(foff[f + 1] - foff[f]);
  double ce[3] = {0.0, 0.0, 0.0}, nr[3] = {0.0, 0.0, 0.0}, a = SMALL;
  if (nn >= 3) {
    const double* pref = xyz + 3 * (int64_t)fn[0];
    double nacc[3] = {0.0, 0.0, 0.0};
    for (int i = 1; i < nn - 1; ++i) {
      const double* pi = xyz + 3 * (int64_t)fn[i];
      const double* pj = xyz + 3 * (int64_t)fn[i + 1];
      double u[3], v[3];
      for (int k = 0; k < 3; ++k) { u[k] = pi[k] - pref[k]; v[k] = pj[k] - pref[k]; }
      const double c0 = u[1] * v[2] - u[2] * v[1], c1 = u[2] * v[0] - u[0] * v[2], c2 = u[0] * v[1] - u[1] * v[0];
      nacc[0] = nacc[0] + 0.5 * c0;
      nacc[1] = nacc[1] + 0.5 * c1;
      nacc[2] = nacc[2] + 0.5 * c2;
    }
    a = sqrt(nacc[0] * nacc[0] + nacc[1] * nacc[1] + nacc[2] * nacc[2]) + SMALL;
    for (int k = 0; k < 3; ++k) nr[k] = nacc[k] / a;
    double asum = 0.0;
    for (int i = 1; i < nn - 1; ++i) {
      const double* pi = xyz + 3 * (int64_t)fn[i];
      const double* pj = xyz + 3 * (int64_t)fn[i + 1];
      double u[3], v[3];
      for (int k = 0; k < 3; ++k) { u[k] = pi[k] - pref[k]; v[k] = pj[k] - pref[k]; }
      const double tv[3] = {0.5 * (u[1] * v[2] - u[2] * v[1]), 0.5 * (u[2] * v[0] - u[0] * v[2]),
                            0.5 * (u[0] * v[1] - u[1] * v[0])};
      const double ta = ddot(tv, nr);
      for (int k = 0; k < 3; ++k) ce[k] = ce[k] + ta * ((pref[k] + pi[k]) + pj[k]) / 3.0;
      asum = asum + ta;
    }
    if (fabs(asum) > SMALL)
      for (int k = 0; k < 3; ++k) ce[k] = ce[k] / asum;
    else
      for (int k = 0; k < 3; ++k) ce[k] = pref[k];
  }
  area[f] = a;
  for (int k = 0; k < 3; ++k) {
    centre[3 * f + k] = ce[k];
    normal[3 * f + k] = nr[k];
  }
}

// Cell volume and centroid from the faces (mod_mesh.f90:compute_polyhedron_cell_moments): fan
// tetrahedra about the first vertex of the cell's first face, signed by the face's side, summed in
// face order.
__global__ void k_poly_cells(int64_t nc, const long long* cfo, const int* cfl, const int* owner, const int64_t* foff,
                             const int* fnodes, const double* xyz, double* cen, double* vol) {
  int64_t c = gtid();
  if (c >= nc) return;
  double r[3] = {0.0, 0.0, 0.0};
  for (long long q = cfo[c]; q < cfo[c + 1]; ++q) {
    const int f = cfl[q];
    if (foff[f + 1] - foff[f] < 3) continue;
    for (int k = 0; k < 3; ++k) r[k] = xyz[3 * (int64_t)fnodes[foff[f]] + k];
    break;
  }
  double v = 0.0, mo[3] = {0.0, 0.0, 0.0};
  for (long long q = cfo[c]; q < cfo[c + 1]; ++q) {
    const int f = cfl[q];
    const int64_t s0 = foff[f], s1 = foff[f + 1];
    if (s1 - s0 < 3) continue;
    const bool own = owner[f] == c;
    double v0[3];
    for (int k = 0; k < 3; ++k) v0[k] = xyz[3 * (int64_t)fnodes[s0] + k] - r[k];
    for (int64_t i = s0 + 1; i < s1 - 1; ++i) {
      double v1[3], v2[3];
      for (int k = 0; k < 3; ++k) {
        v1[k] = xyz[3 * (int64_t)fnodes[i] + k] - r[k];
        v2[k] = xyz[3 * (int64_t)fnodes[i + 1] + k] - r[k];
      }
      const double cr[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
      const double sv = ddot(v0, cr) / 6.0;
      double sm[3];
      for (int k = 0; k < 3; ++k) sm[k] = sv * ((v0[k] + v1[k]) + v2[k]) / 4.0;
      if (own) {
        v = v + sv;
        for (int k = 0; k < 3; ++k) mo[k] = mo[k] + sm[k];
      } else {
        v = v - sv;
        for (int k = 0; k < 3; ++k) mo[k] = mo[k] - sm[k];
      }
    }
  }
  for (int k = 0; k < 3; ++k) cen[3 * c + k] = fabs(v) > SMALL ? r[k] + mo[k] / v : 0.0;
  vol[c] = fabs(v);
}

// Cell vertex lists (mod_foam_reader.f90:build_cell_topology_metadata): the cell's owner faces in
// face order, then its neighbour faces, each vertex once at its first appearance.  coff == null:
// count into cnt; else write at coff[c].
constexpr int CV_CAP = 64;
__global__ void k_poly_cellverts(int64_t nc, const long long* cfo, const int* cfl, const int* owner,
                                 const int64_t* foff, const int* fnodes, const int64_t* coff, long long* cnt, int* cn,
                                 int* bad) {
  int64_t c = gtid();
  if (c >= nc) return;
  int vs[CV_CAP];
  int n = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (long long q = cfo[c]; q < cfo[c + 1]; ++q) {
      const int f = cfl[q];
      if ((owner[f] == c) != (pass == 0)) continue;
      for (int64_t k = foff[f]; k < foff[f + 1]; ++k) {
        const int v = fnodes[k];
        bool seen = false;
        for (int j = 0; j < n; ++j)
          if (vs[j] == v) { seen = true; break; }
        if (seen) continue;
        if (n == CV_CAP) {  // the host stops after the counting pass
          atomicOr(bad, 8);
          if (!coff) cnt[c] = n;
          return;
        }
        vs[n++] = v;
      }
    }
  if (!coff) {
    cnt[c] = n;
    return;
  }
  for (int j = 0; j < n; ++j) cn[coff[c] + j] = vs[j];
}

// Per-cell list widths: [0] faces, [1] boundary faces (atomicMax over cells).
__global__ void k_cell_widths(int64_t nc, int64_t nfi, const long long* cfo, const int* cfl, int* w) {
  int64_t c = gtid();
  if (c >= nc) return;
  int nbd = 0;
  for (long long k = cfo[c]; k < cfo[c + 1]; ++k) nbd += cfl[k] >= nfi;
  atomicMax(&w[0], (int)(cfo[c + 1] - cfo[c]));
  atomicMax(&w[1], nbd);
}

__global__ void k_ls_width(int64_t nc, const long long* cnt, int* w) {
  int64_t c = gtid();
  if (c < nc) atomicMax(w, (int)cnt[c]);
}

__global__ void k_any(int64_t n, const unsigned char* v, int* flag) {
  int64_t i = gtid();
  if (i < n && v[i]) atomicOr(flag, 1);
}

// [n][K] -> [K][n]
__global__ void k_to_soa(int64_t n, int K, const double* src, double* dst) {
  int64_t i = gtid();
  if (i >= n) return;
  for (int k = 0; k < K; ++k) dst[(int64_t)k * n + i] = src[(int64_t)K * i + k];
}

__global__ void k_inv_floor(int64_t n, const double* v, double floor_, double* out) {
  int64_t i = gtid();
  if (i < n) out[i] = 1.0 / dmax(v[i], floor_);
}

__global__ void k_recip(int64_t n, const double* v, double* out) {
  int64_t i = gtid();
  if (i < n) out[i] = 1.0 / v[i];
}

// ---- host side -------------------------------------------------------------------------------

struct Arena {
  std::vector<void*> ptrs;
  bool ok = true;
  ~Arena() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* put(const T* h, size_t n, cudaStream_t st) {
    T* p = get<T>(n);
    if (p && n) ok = ok && cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, st) == cudaSuccess;
    return p;
  }
  void drop(void* p) {
    for (auto& q : ptrs)
      if (q == p) {
        cudaFree(q);
        q = nullptr;
      }
  }
  // hands p over to `to` (no longer freed here)
  void give(void* p, std::vector<void*>& to) {
    if (!p) return;
    for (auto& q : ptrs)
      if (q == p) {
        q = nullptr;
        to.push_back(p);
        return;
      }
  }
};

template <class T>
bool fetch(std::vector<T>& h, const T* d, size_t n, cudaStream_t st) {
  h.resize(n);
  if (!n) return true;
  return cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, st) == cudaSuccess;
}

// Exclusive scan of n counts into n + 1 offsets (off[n] = total).
bool scan_counts(Arena& ar, const unsigned long long* cnt, long long* off, int64_t n, cudaStream_t st) {
  if (n == 0) return cudaMemsetAsync(off, 0, sizeof(long long), st) == cudaSuccess;
  size_t tb = 0;
  const long long* in = reinterpret_cast<const long long*>(cnt);
  if (cub::DeviceScan::InclusiveSum(nullptr, tb, in, off + 1, n, st) != cudaSuccess) return false;
  void* tmp = ar.get<unsigned char>(tb);
  if (!tmp) return false;
  bool ok = cub::DeviceScan::InclusiveSum(tmp, tb, in, off + 1, n, st) == cudaSuccess &&
            cudaMemsetAsync(off, 0, sizeof(long long), st) == cudaSuccess;
  ar.drop(tmp);
  return ok;
}

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t0) { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

struct Stream {
  cudaStream_t s = nullptr;
  ~Stream() {
    if (s) cudaStreamDestroy(s);
  }
};

}  // namespace

SetupDeviceArrays::~SetupDeviceArrays() {
  for (void* p : owned) cudaFree(p);
}

namespace {
int setup_device_impl(const RawMesh* rawp, const PolyMesh* polyp, const dpm_patch_cfg_t* pc, const dpm_params_t& P,
                      int device, Mesh& m, StaticOps& S, std::string* err, SetupTimes* times, SetupDeviceArrays* dev) {
  const bool full = dev == nullptr;  // every array to the host, as the host builder fills them
  auto fail = [&](int code, const char* msg) {
    if (err) *err = msg;
    return code;
  };
  SetupTimes tloc;
  SetupTimes& T = times ? *times : tloc;
  T = SetupTimes();
  if (cudaSetDevice(device) != cudaSuccess) return fail(DPM_ERR_CUDA, "cudaSetDevice failed");
  Stream stream;
  if (cudaStreamCreateWithFlags(&stream.s, cudaStreamNonBlocking) != cudaSuccess) return fail(DPM_ERR_CUDA, "stream");
  cudaStream_t st = stream.s;
  Arena ar;
#define SCK(x)                                                                        \
  do {                                                                                \
    if ((x) != cudaSuccess || !ar.ok) return fail(DPM_ERR_CUDA, "CUDA call failed: " #x); \
  } while (0)
#define SLAUNCH(n, kern, ...)                                        \
  do {                                                               \
    if ((n) > 0) kern<<<nblocks(n), STPB, 0, st>>>(__VA_ARGS__);     \
    SCK(cudaGetLastError());                                         \
  } while (0)

  int64_t nc = 0, nv = 0, nfb = 0, ncn = 0, nfi = 0, nf = 0;
  double *d_xyz = nullptr, *d_cen = nullptr, *d_vol = nullptr, *d_area = nullptr, *d_centre = nullptr,
         *d_normal = nullptr;
  int64_t* d_coff = nullptr;
  int *d_cn = nullptr, *d_owner = nullptr, *d_nbr = nullptr, *d_patch = nullptr, *d_bad = nullptr, *d_cfl = nullptr;
  unsigned long long *d_cnt1 = nullptr, *d_ccnt = nullptr;
  long long* d_cfo = nullptr;
  long long ncf = 0;
  int bad = 0;
  bool csr_done = false;  // the face-based path builds the cell -> face lists with its geometry
  auto t_all = Clock::now();
  auto t0 = Clock::now();
  if (rawp) {
    const RawMesh& raw = *rawp;
    nc = raw.n_cells; nv = raw.n_nodes; nfb = raw.n_bfaces;
    if (nc <= 0 || nc > 2000000000LL || nv > 2000000000LL) return fail(DPM_ERR_UNSUPPORTED, "mesh size out of range");
    m = Mesh();
    m.n_cells = nc;
    m.n_patches = raw.n_patches;
    m.n_vertices = nv;
    m.vertices.assign(raw.xyz, raw.xyz + 3 * nv);
    m.cell_vert_off.assign(raw.cell_off, raw.cell_off + nc + 1);
    m.cell_vertices.assign(raw.cell_nodes, raw.cell_nodes + raw.cell_off[nc]);
    ncn = raw.cell_off[nc];
    d_xyz = ar.put(raw.xyz, 3 * nv, st);
    int* d_type = ar.put(raw.cell_type, nc, st);
    d_coff = ar.put(raw.cell_off, nc + 1, st);
    d_cn = ar.put(raw.cell_nodes, ncn, st);
    int64_t* d_boff = ar.put(raw.bface_off, nfb + 1, st);
    int* d_bnodes = ar.put(raw.bface_nodes, raw.bface_off[nfb], st);
    int* d_bpatch = ar.put(raw.bface_patch, nfb, st);
    SCK(cudaStreamSynchronize(st));
    T.stage_ms[0] = ms_since(t0);

    // cells and face matching
    t0 = Clock::now();
    d_bad = ar.get<int>(4);
    d_cnt1 = ar.get<unsigned long long>(2);
    d_cen = ar.get<double>(3 * nc);
    d_vol = ar.get<double>(nc);
    long long* d_nfc = ar.get<long long>(nc);
    long long* d_roff = ar.get<long long>(nc + 1);
    SCK(cudaMemsetAsync(d_bad, 0, 4 * sizeof(int), st));
    SCK(cudaMemsetAsync(d_cnt1, 0, 2 * sizeof(unsigned long long), st));
    SLAUNCH(nc, k_cells, nc, d_type, d_coff, d_cn, d_xyz, d_cen, d_vol, d_nfc, d_bad);
    if (!scan_counts(ar, reinterpret_cast<unsigned long long*>(d_nfc), d_roff, nc, st)) return fail(DPM_ERR_CUDA, "scan");
    long long nrec_ll = 0;
    bad = 0;
    SCK(cudaMemcpyAsync(&nrec_ll, d_roff + nc, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (bad & 1) return fail(-1, "unsupported element type");
    if (nrec_ll > 2147483647LL) return fail(SETUP_DEVICE_LIMIT, "too many element faces for the device set-up");
    const int64_t nrec = nrec_ll;
    ar.drop(d_nfc);
    int B = 1;
    while (B < 32 && (1LL << B) <= nv) ++B;  // ids + 1 in [0, nv] fit in B bits
    unsigned long long* d_hi = ar.get<unsigned long long>(nrec);
    unsigned long long* d_lo = ar.get<unsigned long long>(nrec);
    unsigned long long* d_k1 = ar.get<unsigned long long>(nrec);
    unsigned long long* d_hs = ar.get<unsigned long long>(nrec);
    int* d_rcell = ar.get<int>(nrec);
    unsigned char* d_rfi = ar.get<unsigned char>(nrec);
    int* d_rid = ar.get<int>(nrec);
    int* d_p1 = ar.get<int>(nrec);
    int* d_perm = ar.get<int>(nrec);
    SCK(cudaGetLastError());
    SLAUNCH(nc, k_records, nc, d_type, d_coff, d_cn, d_roff, B, d_hi, d_lo, d_rcell, d_rfi, d_rid);
    {
      size_t tb1 = 0, tb2 = 0;
      SCK(cub::DeviceRadixSort::SortPairs(nullptr, tb1, d_lo, d_k1, d_rid, d_p1, (int)nrec, 0, 2 * B, st));
      SCK(cub::DeviceRadixSort::SortPairs(nullptr, tb2, d_k1, d_hs, d_p1, d_perm, (int)nrec, 0, 2 * B, st));
      void* tmp = ar.get<unsigned char>(std::max(tb1, tb2));
      SCK(cudaGetLastError());
      // stable LSD: low word first, then the high word (carrying the low-word order)
      SCK(cub::DeviceRadixSort::SortPairs(tmp, tb1, d_lo, d_k1, d_rid, d_p1, (int)nrec, 0, 2 * B, st));
      SLAUNCH(nrec, k_gather64, nrec, d_hi, d_p1, d_k1);
      SCK(cub::DeviceRadixSort::SortPairs(tmp, tb2, d_k1, d_hs, d_p1, d_perm, (int)nrec, 0, 2 * B, st));
      ar.drop(tmp);
    }
    unsigned long long* d_ls = d_k1;  // low words in sorted order
    SLAUNCH(nrec, k_gather64, nrec, d_lo, d_perm, d_ls);
    ar.drop(d_hi);
    ar.drop(d_lo);
    ar.drop(d_rid);
    ar.drop(d_p1);
    unsigned char* d_matched = ar.get<unsigned char>(nrec);
    int* d_sflag = ar.get<int>(nrec);
    int* d_sowner = ar.get<int>(nrec);
    int* d_sidx = ar.get<int>(nrec);
    SCK(cudaGetLastError());
    SCK(cudaMemsetAsync(d_sflag, 0, nrec * sizeof(int), st));
    SLAUNCH(nrec, k_match, nrec, d_hs, d_ls, d_perm, d_rcell, d_matched, d_sflag, d_sowner);
    {
      size_t tb = 0;
      SCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_sflag, d_sidx, (int)nrec, st));
      void* tmp = ar.get<unsigned char>(tb);
      SCK(cudaGetLastError());
      SCK(cub::DeviceScan::ExclusiveSum(tmp, tb, d_sflag, d_sidx, (int)nrec, st));
      ar.drop(tmp);
    }
    int last_idx = 0, last_flag = 0;
    SCK(cudaMemcpyAsync(&last_idx, d_sidx + nrec - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&last_flag, d_sflag + nrec - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    T.stage_ms[1] = ms_since(t0);

    // faces: interior in creation order, boundary regrouped by patch
    t0 = Clock::now();
    nfi = (int64_t)last_idx + last_flag;
    nf = nfi + nfb;
    if (nf > 2000000000LL) return fail(DPM_ERR_UNSUPPORTED, "too many faces");
    m.n_int_faces = nfi;
    m.n_bnd_faces = nfb;
    m.n_faces = nf;
    m.patch_start.assign(m.n_patches, 0);
    m.patch_nfaces.assign(m.n_patches, 0);
    std::vector<long long> bpos(nfb);
    for (int64_t b = 0; b < nfb; ++b) {
      int p = raw.bface_patch[b];
      if (p < 0 || p >= m.n_patches) return fail(DPM_ERR_ARG, "boundary face with a patch index out of range");
      m.patch_nfaces[p]++;
    }
    for (int p = 1; p < m.n_patches; ++p) m.patch_start[p] = m.patch_start[p - 1] + m.patch_nfaces[p - 1];
    {
      std::vector<int64_t> cursor(m.patch_start);
      for (int64_t b = 0; b < nfb; ++b) bpos[b] = cursor[raw.bface_patch[b]]++;
    }
    m.patch_bc.resize(m.n_patches);
    for (int p = 0; p < m.n_patches; ++p) m.patch_bc[p] = pc[p].bc_id;
    long long* d_bpos = ar.put(bpos.data(), nfb, st);
    d_owner = ar.get<int>(nf);
    d_nbr = ar.get<int>(nf);
    d_patch = ar.get<int>(nf);
    d_area = ar.get<double>(nf);
    d_centre = ar.get<double>(3 * nf);
    d_normal = ar.get<double>(3 * nf);
    SCK(cudaGetLastError());
    SLAUNCH(nrec, k_int_faces, nrec, d_sflag, d_sidx, d_sowner, d_rcell, d_rfi, d_type, d_coff, d_cn, d_xyz, d_cen,
            d_owner, d_nbr, d_patch, d_area, d_centre, d_normal);
    SLAUNCH(nfb, k_bnd_faces, nfb, d_boff, d_bnodes, d_bpatch, d_bpos, nfi, B, nrec, d_hs, d_ls, d_perm, d_rcell, d_xyz,
            d_cen, d_matched, d_bad, d_owner, d_nbr, d_patch, d_area, d_centre, d_normal);
    SLAUNCH(nrec, k_count_zero, nrec, d_matched, d_cnt1);
    unsigned long long unmatched = 0;
    SCK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&unmatched, d_cnt1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (bad & 4) return fail(-2, "boundary face with other than 3 or 4 nodes");
    if (bad & 2) return fail(-2, "boundary face has no owner cell");
    if (unmatched) return fail(-3, "unlabelled boundary faces (open cells)");
    for (void* p : {(void*)d_hs, (void*)d_ls, (void*)d_perm, (void*)d_rcell, (void*)d_rfi, (void*)d_matched,
                    (void*)d_sflag, (void*)d_sowner, (void*)d_sidx, (void*)d_roff, (void*)d_bpos})
      ar.drop(p);

  } else {
    // face-based mesh: faces, owners and patches as given (build_mesh_poly's checks), the
    // reference's polygon face geometry and polyhedron moments, cell vertices in face order
    const PolyMesh& pm = *polyp;
    nf = pm.n_faces;
    nfi = pm.n_int_faces;
    nfb = nf - nfi;
    nv = pm.n_points;
    if (nf < 1 || nfi < 0 || nfi > nf || nf > 2000000000LL || nv > 2000000000LL)
      return fail(-5, "face counts out of range");
    int64_t mx = -1;
    for (int64_t f = 0; f < nf; ++f) {
      if (pm.owner[f] < 0) return fail(-5, "negative cell index in owner/neighbour (corrupt polyMesh files)");
      mx = std::max<int64_t>(mx, pm.owner[f]);
    }
    for (int64_t f = 0; f < nfi; ++f) {
      if (pm.neighbour[f] < 0) return fail(-5, "negative cell index in owner/neighbour (corrupt polyMesh files)");
      mx = std::max<int64_t>(mx, pm.neighbour[f]);
    }
    for (int64_t f = 0; f < nfi; ++f)
      if (pm.owner[f] >= pm.neighbour[f]) return fail(-6, "OpenFOAM upper-triangular convention violated");
    for (int64_t k = 0; k < pm.face_off[nf]; ++k)
      if (pm.face_nodes[k] < 0 || pm.face_nodes[k] >= nv) return fail(-5, "face node index out of range");
    nc = mx + 1;
    if (nc <= 0 || nc > 2000000000LL) return fail(DPM_ERR_UNSUPPORTED, "mesh size out of range");
    m = Mesh();
    m.n_cells = nc;
    m.n_faces = nf;
    m.n_int_faces = nfi;
    m.n_bnd_faces = nfb;
    m.n_patches = pm.n_patches;
    m.n_vertices = nv;
    m.vertices.assign(pm.xyz, pm.xyz + 3 * nv);
    m.patch_start.assign(m.n_patches, 0);
    m.patch_nfaces.assign(m.n_patches, 0);
    m.patch_bc.resize(m.n_patches);
    std::vector<int> fpatch(nf, -1), fnbr(nf, -1);
    int n_periodic = 0;
    for (int p = 0; p < m.n_patches; ++p) {
      const int64_t s0 = pm.patch_start[p] - nfi, n = pm.patch_nfaces[p];
      if (s0 < 0 || n < 0) return fail(-7, "boundary connectivity invalid (patch has invalid start_face/n_faces)");
      if (s0 + n > nfb) return fail(-7, "patch face range exceeds boundary faces");
      m.patch_start[p] = s0;
      m.patch_nfaces[p] = n;
      m.patch_bc[p] = pc[p].bc_id;
      for (int64_t f = nfi + s0; f < nfi + s0 + n; ++f) fpatch[f] = p;
      if (pc[p].bc_id == BC_PERIODIC) n_periodic++;
    }
    for (int64_t f = nfi; f < nf; ++f)
      if (fpatch[f] < 0) return fail(-7, "boundary faces not mapped to a patch");
    if (n_periodic % 2) return fail(-8, "odd number of periodic patches");
    for (int64_t f = 0; f < nfi; ++f) fnbr[f] = pm.neighbour[f];
    d_xyz = ar.put(pm.xyz, 3 * nv, st);
    int64_t* d_foff = ar.put(pm.face_off, nf + 1, st);
    int* d_fnodes = ar.put(pm.face_nodes, pm.face_off[nf], st);
    d_owner = ar.put(pm.owner, nf, st);
    d_nbr = ar.put(fnbr.data(), nf, st);
    d_patch = ar.put(fpatch.data(), nf, st);
    SCK(cudaStreamSynchronize(st));
    T.stage_ms[0] = ms_since(t0);
    t0 = Clock::now();
    d_bad = ar.get<int>(4);
    d_cnt1 = ar.get<unsigned long long>(2);
    d_cen = ar.get<double>(3 * nc);
    d_vol = ar.get<double>(nc);
    d_area = ar.get<double>(nf);
    d_centre = ar.get<double>(3 * nf);
    d_normal = ar.get<double>(3 * nf);
    d_ccnt = ar.get<unsigned long long>(nc);
    d_cfo = ar.get<long long>(nc + 1);
    long long* d_cvn = ar.get<long long>(nc);
    SCK(cudaGetLastError());
    SCK(cudaMemsetAsync(d_bad, 0, 4 * sizeof(int), st));
    SCK(cudaMemsetAsync(d_cnt1, 0, 2 * sizeof(unsigned long long), st));
    SLAUNCH(nf, k_poly_faces, nf, d_foff, d_fnodes, d_xyz, d_area, d_centre, d_normal);
    SCK(cudaMemsetAsync(d_ccnt, 0, nc * sizeof(unsigned long long), st));
    SLAUNCH(nf, k_cf_count, nf, d_owner, d_nbr, d_ccnt);
    if (!scan_counts(ar, d_ccnt, d_cfo, nc, st)) return fail(DPM_ERR_CUDA, "scan");
    SCK(cudaMemcpyAsync(&ncf, d_cfo + nc, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    d_cfl = ar.get<int>(ncf);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(d_ccnt, d_cfo, nc * sizeof(long long), cudaMemcpyDeviceToDevice, st));
    SLAUNCH(nf, k_cf_fill, nf, d_owner, d_nbr, d_ccnt, d_cfl);
    SLAUNCH(nc, k_sort_rows, nc, d_cfo, d_cfl);
    csr_done = true;
    SLAUNCH(nc, k_poly_cells, nc, d_cfo, d_cfl, d_owner, d_foff, d_fnodes, d_xyz, d_cen, d_vol);
    // cell vertex lists: count, offsets, fill
    SLAUNCH(nc, k_poly_cellverts, nc, d_cfo, d_cfl, d_owner, d_foff, d_fnodes, (const int64_t*)nullptr, d_cvn,
            (int*)nullptr, d_bad);
    d_coff = ar.get<int64_t>(nc + 1);
    SCK(cudaGetLastError());
    if (!scan_counts(ar, reinterpret_cast<unsigned long long*>(d_cvn), reinterpret_cast<long long*>(d_coff), nc, st))
      return fail(DPM_ERR_CUDA, "scan");
    long long ncn_ll = 0;
    SCK(cudaMemcpyAsync(&ncn_ll, d_coff + nc, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (bad & 8) return fail(SETUP_DEVICE_LIMIT, "a cell with more vertices than the device set-up holds");
    ncn = ncn_ll;
    d_cn = ar.get<int>(ncn);
    SCK(cudaGetLastError());
    SLAUNCH(nc, k_poly_cellverts, nc, d_cfo, d_cfl, d_owner, d_foff, d_fnodes, d_coff, d_cvn, d_cn, d_bad);
    if (full) {
      SCK(fetch(m.cell_vert_off, d_coff, nc + 1, st) ? cudaSuccess : cudaErrorUnknown);
      SCK(fetch(m.cell_vertices, d_cn, ncn, st) ? cudaSuccess : cudaErrorUnknown);
    }
    SCK(cudaStreamSynchronize(st));
    ar.drop(d_cvn);
    T.stage_ms[1] = ms_since(t0);
    t0 = Clock::now();
  }
  double* d_sf = ar.get<double>(3 * nf);
  double* d_dcf = ar.get<double>(nf);
  double* d_gc = ar.get<double>(nf);
  double* d_eps = ar.get<double>(3 * nf);
  double* d_skew = ar.get<double>(nf);
  unsigned char* d_isref = ar.get<unsigned char>(nf);
  if (!csr_done) {
    d_ccnt = ar.get<unsigned long long>(nc);
    d_cfo = ar.get<long long>(nc + 1);
  }
  SCK(cudaGetLastError());
  SLAUNCH(nf, k_face_metrics, nf, d_owner, d_nbr, d_area, d_normal, d_centre, d_cen, d_sf, d_dcf, d_gc, d_eps, d_skew,
          d_isref);
  // cell -> face lists (mod_mesh.f90:mesh_build_connectivity), faces ascending
  if (!csr_done) {
    SCK(cudaMemsetAsync(d_ccnt, 0, nc * sizeof(unsigned long long), st));
    SLAUNCH(nf, k_cf_count, nf, d_owner, d_nbr, d_ccnt);
    if (!scan_counts(ar, d_ccnt, d_cfo, nc, st)) return fail(DPM_ERR_CUDA, "scan");
    SCK(cudaMemcpyAsync(&ncf, d_cfo + nc, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    d_cfl = ar.get<int>(ncf);
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(d_ccnt, d_cfo, nc * sizeof(long long), cudaMemcpyDeviceToDevice, st));
    SLAUNCH(nf, k_cf_fill, nf, d_owner, d_nbr, d_ccnt, d_cfl);
    SLAUNCH(nc, k_sort_rows, nc, d_cfo, d_cfl);
  }
  // the host needs the boundary faces for the periodic pairing and the outlet rows, and the
  // whole mesh for the rest of the solver set-up
  int widths[2] = {0, 0}, refine_any = 0;
  int* d_widths = ar.get<int>(4);
  SCK(cudaGetLastError());
  SCK(cudaMemsetAsync(d_widths, 0, 4 * sizeof(int), st));
  SLAUNCH(nc, k_cell_widths, nc, nfi, d_cfo, d_cfl, d_widths);
  SLAUNCH(nfi, k_any, nfi, d_isref, d_widths + 2);
  SCK(cudaMemcpyAsync(widths, d_widths, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaMemcpyAsync(&refine_any, d_widths + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(fetch(m.centroid, d_cen, 3 * nc, st) ? cudaSuccess : cudaErrorUnknown);
  SCK(fetch(m.volume, d_vol, nc, st) ? cudaSuccess : cudaErrorUnknown);
  SCK(fetch(m.owner, d_owner, nf, st) ? cudaSuccess : cudaErrorUnknown);
  SCK(fetch(m.patch, d_patch, nf, st) ? cudaSuccess : cudaErrorUnknown);
  SCK(fetch(m.area, d_area, nf, st) ? cudaSuccess : cudaErrorUnknown);
  SCK(fetch(m.centre, d_centre, 3 * nf, st) ? cudaSuccess : cudaErrorUnknown);
  SCK(fetch(m.normal, d_normal, 3 * nf, st) ? cudaSuccess : cudaErrorUnknown);
  SCK(fetch(m.d_cf, d_dcf, nf, st) ? cudaSuccess : cudaErrorUnknown);
  if (full) {
    std::vector<long long> cfo_h;
    SCK(fetch(m.neighbour, d_nbr, nf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.sf, d_sf, 3 * nf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.gc, d_gc, nf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.eps, d_eps, 3 * nf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.skew, d_skew, nf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.is_refine, d_isref, nf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(cfo_h, d_cfo, nc + 1, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.cell_faces, d_cfl, ncf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(cudaStreamSynchronize(st));
    m.cell_face_off.assign(cfo_h.begin(), cfo_h.end());
  }
  SCK(cudaStreamSynchronize(st));
  T.stage_ms[2] = ms_since(t0);

  // periodic pairing (host, boundary faces only)
  t0 = Clock::now();
  {
    int rc = build_periodic(m, err);
    if (rc) return rc;
  }
  T.stage_ms[3] = ms_since(t0);

  // LS stencil: face neighbours (periodic partners across seams), then vertex-sharing cells
  t0 = Clock::now();
  const int max_faces = std::max(1, widths[0]);
  const int max_st = std::max(32, 4 * max_faces);
  int* d_pbc = ar.put(m.patch_bc.data(), (size_t)m.n_patches, st);
  int* d_ppair = ar.put(m.periodic_pair.data(), nfb, st);
  double* d_ppdcf = ar.put(m.periodic_pair_dcf.data(), nfb, st);
  unsigned long long* d_vcnt = ar.get<unsigned long long>(nv);
  long long* d_voff = ar.get<long long>(nv + 1);
  int* d_vcell = ar.get<int>(ncn);
  int* d_tnb = ar.get<int>((size_t)max_st * nc);
  int* d_tface = ar.get<int>((size_t)max_st * nc);
  unsigned char* d_tper = ar.get<unsigned char>((size_t)max_st * nc);
  long long* d_lcnt = ar.get<long long>(nc);
  long long* d_lsoff = ar.get<long long>(nc + 1);
  SCK(cudaGetLastError());
  SCK(cudaMemsetAsync(d_vcnt, 0, nv * sizeof(unsigned long long), st));
  SLAUNCH(nc, k_vc_count, nc, d_coff, d_cn, d_vcnt);
  if (!scan_counts(ar, d_vcnt, d_voff, nv, st)) return fail(DPM_ERR_CUDA, "scan");
  SCK(cudaMemcpyAsync(d_vcnt, d_voff, nv * sizeof(long long), cudaMemcpyDeviceToDevice, st));
  SLAUNCH(nc, k_vc_fill, nc, d_coff, d_cn, d_vcnt, d_vcell);
  SLAUNCH(nv, k_sort_rows, nv, d_voff, d_vcell);
  SLAUNCH(nc, k_ls_neigh, nc, max_st, d_cfo, d_cfl, d_owner, d_nbr, d_patch, d_pbc, nfi, d_ppair, d_coff, d_cn, d_voff,
          d_vcell, d_tnb, d_tface, d_tper, d_lcnt);
  if (!scan_counts(ar, reinterpret_cast<unsigned long long*>(d_lcnt), d_lsoff, nc, st))
    return fail(DPM_ERR_CUDA, "scan");
  long long ns = 0;
  SCK(cudaMemcpyAsync(&ns, d_lsoff + nc, sizeof(long long), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  int* d_lscell = ar.get<int>(ns);
  int* d_lsface = ar.get<int>(ns);
  double* d_lsw = ar.get<double>(3 * ns);
  SCK(cudaGetLastError());
  SCK(cudaMemsetAsync(d_cnt1, 0, sizeof(unsigned long long), st));
  {
    LsArgs a{nc, nfi, nfb, d_lsoff, d_cfo, d_tnb, d_tface, d_cfl, d_tper, d_cen, d_dcf, d_normal, d_centre, d_ppdcf,
             d_lscell, d_lsface, d_lsw, d_cnt1};
    SLAUNCH(nc, k_ls_weights, a);
  }
  unsigned long long ndeg = 0;
  SCK(cudaMemsetAsync(d_widths + 3, 0, sizeof(int), st));
  SLAUNCH(nc, k_ls_width, nc, d_lcnt, d_widths + 3);
  int W = 0;
  SCK(cudaMemcpyAsync(&W, d_widths + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (full) {
    std::vector<long long> lsoff_h;
    SCK(fetch(lsoff_h, d_lsoff, nc + 1, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.ls_cell, d_lscell, ns, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.ls_face, d_lsface, ns, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(m.ls_w, d_lsw, 3 * ns, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(cudaStreamSynchronize(st));
    m.ls_off.assign(lsoff_h.begin(), lsoff_h.end());
  }
  SCK(cudaMemcpyAsync(&ndeg, d_cnt1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  m.ls_degenerate = (int64_t)ndeg;
  for (void* p : {(void*)d_vcnt, (void*)d_voff, (void*)d_vcell, (void*)d_tnb, (void*)d_tface, (void*)d_tper,
                  (void*)d_lcnt})
    ar.drop(p);
  T.stage_ms[4] = ms_since(t0);
  T.mesh_ms = ms_since(t_all);

  // ---- static operators (ops.cpp, build_static_ops) --------------------------------------------
  auto t_ops = Clock::now();
  t0 = Clock::now();
  S = StaticOps();
  S.nc = nc; S.nf = nf; S.nfi = nfi; S.nb = nfb;
  S.bnd_bc.assign(nfb, BC_ZEROGRADIENT);
  S.bnd_pnb.assign(nfb, -1);
  for (int64_t b = 0; b < nfb; ++b) {
    int p = m.patch[nfi + b];
    if (p >= 0) S.bnd_bc[b] = pc[p].bc_id;
    if (S.bnd_bc[b] == BC_PERIODIC) {
      int n = m.periodic_partner_cell(b);
      S.bnd_pnb[b] = (n == m.owner[nfi + b]) ? -1 : n;
    }
  }
  std::vector<int64_t> per_canon;
  for (int q = 0; q < m.n_patches; ++q) {
    if (pc[q].bc_id != BC_PERIODIC) continue;
    for (int64_t k = 0; k < m.patch_nfaces[q]; ++k) {
      int64_t b = m.patch_start[q] + k;
      int o = m.owner[nfi + b], n = m.periodic_partner_cell(b);
      if (n < 0 || n <= o) continue;
      per_canon.push_back(b);
    }
  }
  S.nfp = nfi + (int64_t)per_canon.size();
  const int64_t nfp = S.nfp;
  const int64_t npc = (int64_t)per_canon.size();
  // periodic pairs (host): coefficients and face-velocity weights
  std::vector<int> tp_o(npc), tp_n(npc), tp_f(npc);
  std::vector<double> tp_c(npc), tp_gcf(npc), tp_gcw(npc);
  std::vector<int> bps(nfb, -1);
  std::vector<unsigned char> bcanon(nfb, 0);
  for (int64_t k = 0; k < npc; ++k) {
    int64_t b = per_canon[k], f = nfi + b;
    int o = m.owner[f], n = m.periodic_partner_cell(b);
    int pb = m.periodic_pair[b];
    int64_t pf = pb >= 0 ? nfi + pb : -1;
    double pdcf = m.periodic_pair_dcf[b];
    if (pdcf <= SMALL && pf >= 0) pdcf = m.d_cf[pf];
    if (pdcf <= SMALL) pdcf = m.d_cf[f];
    double area = m.area[f];
    if (pf >= 0) area = 0.5 * (area + m.area[pf]);
    tp_o[k] = o; tp_n[k] = n; tp_f[k] = (int)f;
    tp_c[k] = area / (m.d_cf[f] + pdcf + SMALL);
    double d_o = m.d_cf[f], d_n = d_o;
    if (m.periodic_pair_dcf[b] > SMALL) d_n = m.periodic_pair_dcf[b];
    if (d_n <= SMALL && pf >= 0) d_n = m.d_cf[pf];
    double dt_ = d_o + d_n;
    tp_gcf[k] = dt_ > SMALL ? d_n / dt_ : 0.5;
    tp_gcw[k] = m.periodic_gc[b];
    bps[b] = (int)(nfi + k);
    bcanon[b] = 1;
    if (pb >= 0) bps[pb] = (int)(nfi + k);
  }
  // outlet rows (host)
  const double cfl = P.pressure_min_cos_theta;
  S.bnd_cb.assign(nfb, 0.0);
  S.bnd_kout.assign(3 * nfb, 0.0);
  S.n_outlet = 0;
  std::vector<double> bdiag(nfb, 0.0);
  std::vector<unsigned char> bdiag_on(nfb, 0);
  for (int q = 0; q < m.n_patches; ++q) {
    if (pc[q].bc_id != BC_OUTLET) continue;
    for (int64_t k = 0; k < m.patch_nfaces[q]; ++k) {
      int64_t b = m.patch_start[q] + k, f = nfi + b;
      int o = m.owner[f];
      double d[3];
      for (int j = 0; j < 3; ++j) d[j] = m.centre[3 * f + j] - m.centroid[3 * o + j];
      double dpb = std::fabs(d[0] * m.normal[3 * f] + d[1] * m.normal[3 * f + 1] + d[2] * m.normal[3 * f + 2]);
      S.n_outlet++;
      S.bnd_cb[b] = m.area[f] / std::max(dpb, SMALL);
      if (dpb <= SMALL) dpb = m.d_cf[f];
      if (cfl > 0.0) dpb = std::max(dpb, cfl * m.d_cf[f]);
      if (dpb <= SMALL) continue;
      double cb = m.area[f] / dpb;
      bdiag[b] = cb;
      bdiag_on[b] = 1;
      S.dir_rows.push_back(o);
      S.dir_vals.push_back(cb * pc[q].p_val);
    }
  }
  // outlet k-vectors (host)
  int64_t n_active_b = 0;
  std::vector<double> kb(3 * nfb, 0.0);
  for (int64_t b = 0; b < nfb; ++b) {
    if (S.bnd_bc[b] != BC_OUTLET) continue;
    int64_t f = nfi + b;
    int o = m.owner[f];
    const double s[3] = {m.area[f] * m.normal[3 * f], m.area[f] * m.normal[3 * f + 1], m.area[f] * m.normal[3 * f + 2]};
    double d[3], k[3];
    for (int j = 0; j < 3; ++j) d[j] = m.centre[3 * f + j] - m.centroid[3 * o + j];
    double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len < 1.0e-30) {
      k[0] = k[1] = k[2] = 0.0;
    } else {
      double inv = 1.0 / len, sdd = (s[0] * d[0] + s[1] * d[1] + s[2] * d[2]) * inv, dl = sdd * len,
             s2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
      if (cfl > 0.0) dl = std::max(dl, cfl * std::sqrt(s2) * len);
      if (dl > 1.0e-30)
        for (int j = 0; j < 3; ++j) k[j] = s[j] - (s2 / dl) * d[j];
      else
        for (int j = 0; j < 3; ++j) k[j] = s[j] - (sdd * inv) * d[j];
    }
    if (k[0] * k[0] + k[1] * k[1] + k[2] * k[2] >= 1.0e-10 * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2])) {
      n_active_b++;
      for (int j = 0; j < 3; ++j) kb[3 * b + j] = k[j];
    }
  }
  // device: pressure-solver faces, lists, diagonal, k-vectors
  int* d_pso = ar.get<int>(nfp);
  int* d_psn = ar.get<int>(nfp);
  int* d_psf = ar.get<int>(nfp);
  double* d_psc = ar.get<double>(nfp);
  double* d_kk = ar.get<double>(3 * nfp);
  int* d_bps = ar.put(bps.data(), nfb, st);
  unsigned char* d_bcanon = ar.put(bcanon.data(), nfb, st);
  double* d_bdiag = ar.put(bdiag.data(), nfb, st);
  unsigned char* d_bdiag_on = ar.put(bdiag_on.data(), nfb, st);
  int* d_bbc = ar.put(S.bnd_bc.data(), nfb, st);
  SCK(cudaGetLastError());
  if (npc) {
    SCK(cudaMemcpyAsync(d_pso + nfi, tp_o.data(), npc * sizeof(int), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_psn + nfi, tp_n.data(), npc * sizeof(int), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_psf + nfi, tp_f.data(), npc * sizeof(int), cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_psc + nfi, tp_c.data(), npc * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  SCK(cudaMemsetAsync(d_bad, 0, 4 * sizeof(int), st));
  SCK(cudaMemsetAsync(d_cnt1, 0, 2 * sizeof(unsigned long long), st));
  SLAUNCH(nfi, k_ps_interior, nfi, d_owner, d_nbr, d_cen, d_normal, d_area, d_dcf, cfl, d_pso, d_psn, d_psf, d_psc,
          d_bad);
  SLAUNCH(nfp, k_ps_jasak, nfp, d_pso, d_psn, d_psf, d_sf, d_cen, cfl, d_kk, d_cnt1);
  const int Sw = widths[0], SB = widths[1];
  S.S = Sw;
  S.SB = SB;
  int* d_cfell = ar.get<int>((size_t)std::max(Sw, 1) * nc);
  int* d_cbell = ar.get<int>((size_t)std::max(SB, 1) * nc);
  int* d_cpsell = ar.get<int>((size_t)CPS_CAP * nc);
  double* d_diag = ar.get<double>(nc);
  SCK(cudaGetLastError());
  SCK(cudaMemsetAsync(d_widths, 0, 2 * sizeof(int), st));
  SLAUNCH(nc, k_cell_lists, nc, nfi, d_cfo, d_cfl, d_owner, d_bps, d_bcanon, d_cfell, std::max(Sw, 1), d_cpsell,
          d_cbell, std::max(SB, 1), d_widths, d_bad);
  // a cell whose pressure-solver list overflowed has an incomplete list: stop before reading it
  SCK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  if (bad & 2)
    return fail(SETUP_DEVICE_LIMIT, "more pressure-solver faces per cell than the device set-up holds");
  SLAUNCH(nc, k_diag, nc, nfi, SB, d_cpsell, d_cbell, d_psc, d_bdiag, d_bdiag_on, d_diag);
  SLAUNCH(nc, k_arow, nc, d_cpsell, d_pso, d_psn, d_psc, d_diag, 0, (int*)nullptr, (double*)nullptr, d_widths + 1);
  unsigned long long n_active_i = 0;
  SCK(cudaMemcpyAsync(widths, d_widths, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaMemcpyAsync(&n_active_i, d_cnt1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  if (bad & 1) return fail(DPM_ERR_MESH, "non-finite or non-positive pressure coefficient");
  if (bad & 2) return fail(SETUP_DEVICE_LIMIT, "more pressure-solver faces per cell than the device set-up holds");
  S.SP = widths[0];
  S.WA = widths[1];
  if (S.WA > 16) return fail(DPM_ERR_UNSUPPORTED, "matrix row wider than 16");
  int* d_acol = ar.get<int>((size_t)S.WA * nc);
  double* d_aval = ar.get<double>((size_t)S.WA * nc);
  SCK(cudaGetLastError());
  SLAUNCH(nc, k_arow, nc, d_cpsell, d_pso, d_psn, d_psc, d_diag, S.WA, d_acol, d_aval, d_widths + 1);
  T.stage_ms[5] = ms_since(t0);
  // LS stencil as ELL, T^-1, filter tensor, blend weights
  t0 = Clock::now();
  S.W = W;
  const int Wc = std::max(W, 1);
  int* d_lsidx = ar.get<int>((size_t)Wc * nc);
  double* d_lswell = ar.get<double>((size_t)3 * Wc * nc);
  double* d_tinv = ar.get<double>(9 * (size_t)nc);
  double* d_G0 = ar.get<double>(9 * (size_t)nc);
  double* d_G1 = ar.get<double>(9 * (size_t)nc);
  double* d_wbl = ar.get<double>(nf);
  SCK(cudaGetLastError());
  if (W == 0) {
    SCK(cudaMemsetAsync(d_lswell, 0, 3 * nc * sizeof(double), st));
    std::vector<int> pad(nc, NONE_PAD);
    SCK(cudaMemcpyAsync(d_lsidx, pad.data(), nc * sizeof(int), cudaMemcpyHostToDevice, st));
    SCK(cudaStreamSynchronize(st));
  } else {
    SLAUNCH(nc, k_ls_ell, nc, nfi, nfb, W, d_lsoff, d_lscell, d_lsface, d_lsw, d_lsidx, d_lswell);
  }
  if (!full) {  // the ELL copy is what the step reads
    SCK(cudaStreamSynchronize(st));
    for (void* q : {(void*)d_lscell, (void*)d_lsface, (void*)d_lsw}) ar.drop(q);
  }
  SLAUNCH(nc, k_tinv, nc, nfi, SB, d_cpsell, d_cbell, d_psf, d_bbc, d_area, d_normal, d_tinv);
  SLAUNCH(nc, k_filter, nc, d_cfo, d_cfl, d_centre, d_cen, d_area, d_vol, d_G0);
  SLAUNCH(nc, k_filter_smooth, nc, nfi, d_cfo, d_cfl, d_owner, d_nbr, d_area, d_G0, d_G1);
  SLAUNCH(nc, k_filter_smooth, nc, nfi, d_cfo, d_cfl, d_owner, d_nbr, d_area, d_G1, d_G0);
  SLAUNCH(nf, k_wblend, nf, nfi, d_skew, d_wbl);
  const int64_t n_active = (int64_t)n_active_i + n_active_b;
  S.skip_nonortho = (n_active == 0);
  if (full) {
    std::vector<int> cps_full;
    std::vector<double> kk_h;
    SCK(fetch(S.ps_o, d_pso, nfp, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.ps_n, d_psn, nfp, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.ps_f, d_psf, nfp, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.ps_coeff, d_psc, nfp, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(kk_h, d_kk, 3 * nfp, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.diag, d_diag, nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.A_col, d_acol, (size_t)S.WA * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.A_val, d_aval, (size_t)S.WA * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.cell_face, d_cfell, (size_t)std::max(Sw, 1) * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.cell_bnd, d_cbell, (size_t)std::max(SB, 1) * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(cps_full, d_cpsell, (size_t)std::max(S.SP, 1) * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.ls_idx, d_lsidx, (size_t)Wc * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.ls_w, d_lswell, (size_t)3 * Wc * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.Tinv, d_tinv, 9 * (size_t)nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.G, d_G0, 9 * (size_t)nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.wblend, d_wbl, nf, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(cudaStreamSynchronize(st));
    S.cell_ps.swap(cps_full);
    S.ps_gcf.resize(nfp);
    S.ps_gcw.resize(nfp);
    std::memcpy(S.ps_gcf.data(), m.gc.data(), nfi * sizeof(double));
    std::memcpy(S.ps_gcw.data(), m.gc.data(), nfi * sizeof(double));
    for (int64_t k = 0; k < npc; ++k) {
      S.ps_gcf[nfi + k] = tp_gcf[k];
      S.ps_gcw[nfi + k] = tp_gcw[k];
    }
    S.ps_k.assign(3 * nfp, 0.0);
    S.ps_krc.assign(3 * nfp, 0.0);
    if (!S.skip_nonortho) {
      S.ps_k = kk_h;
      if (!P.rhie_chow_dual) S.ps_krc = kk_h;
    }
  } else {
    // the time step's layouts, in HBM; the host keeps the matrix for the hierarchy set-ups
    SCK(fetch(S.A_col, d_acol, (size_t)S.WA * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SCK(fetch(S.A_val, d_aval, (size_t)S.WA * nc, st) ? cudaSuccess : cudaErrorUnknown);
    SetupDeviceArrays& o = *dev;
    auto soa = [&](const double* src, int64_t n, int K) {
      double* dst = ar.get<double>((size_t)K * n);
      if (dst && n > 0) k_to_soa<<<nblocks(n), STPB, 0, st>>>(n, K, src, dst);
      return dst;
    };
    o.cen = soa(d_cen, nc, 3);
    o.Tinv = soa(d_tinv, nc, 9);
    o.G = soa(d_G0, nc, 9);
    o.sf = soa(d_sf, nf, 3);
    o.nrm = soa(d_normal, nf, 3);
    o.fcen = soa(d_centre, nf, 3);
    o.eps = soa(d_eps, nf, 3);
    o.ivol = ar.get<double>(nc);
    o.Adinv = ar.get<double>(nc);
    o.psgcf = ar.get<double>(nfp);
    o.psgcw = ar.get<double>(nfp);
    SCK(cudaGetLastError());
    SLAUNCH(nc, k_inv_floor, nc, d_vol, SMALL, o.ivol);
    SLAUNCH(nc, k_recip, nc, d_diag, o.Adinv);
    SCK(cudaMemcpyAsync(o.psgcf, d_gc, nfi * sizeof(double), cudaMemcpyDeviceToDevice, st));
    SCK(cudaMemcpyAsync(o.psgcw, d_gc, nfi * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (npc) {
      SCK(cudaMemcpyAsync(o.psgcf + nfi, tp_gcf.data(), npc * sizeof(double), cudaMemcpyHostToDevice, st));
      SCK(cudaMemcpyAsync(o.psgcw + nfi, tp_gcw.data(), npc * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    if (S.skip_nonortho) {  // both k-vectors zero
      SCK(cudaMemsetAsync(d_kk, 0, 3 * nfp * sizeof(double), st));
      o.psk = o.pskrc = d_kk;
    } else {
      o.psk = d_kk;
      if (P.rhie_chow_dual) {
        o.pskrc = ar.get<double>(3 * nfp);
        SCK(cudaGetLastError());
        SCK(cudaMemsetAsync(o.pskrc, 0, 3 * nfp * sizeof(double), st));
      } else {
        o.pskrc = d_kk;  // the same vector, read-only
      }
    }
    o.vol = d_vol; o.area = d_area; o.gc = d_gc; o.wbl = d_wbl; o.dcf = d_dcf;
    o.fo = d_owner; o.fn = d_nbr;
    o.cf = d_cfell; o.cps = d_cpsell; o.cbn = d_cbell; o.ls_idx = d_lsidx; o.ls_w = d_lswell;
    o.pso = d_pso; o.psn = d_psn; o.psf = d_psf; o.psc = d_psc; o.Acol = d_acol; o.Aval = d_aval;
    o.bps = bps;
    o.bcanon.assign(bcanon.begin(), bcanon.end());
    SCK(cudaStreamSynchronize(st));
    for (void* q : {(void*)o.cen, (void*)o.Tinv, (void*)o.G, (void*)o.sf, (void*)o.nrm, (void*)o.fcen, (void*)o.eps,
                    (void*)o.ivol, (void*)o.Adinv, (void*)o.psgcf, (void*)o.psgcw, (void*)o.psk, (void*)o.vol,
                    (void*)o.area, (void*)o.gc, (void*)o.wbl, (void*)o.dcf, (void*)o.fo, (void*)o.fn, (void*)o.cf,
                    (void*)o.cps, (void*)o.cbn, (void*)o.ls_idx, (void*)o.ls_w, (void*)o.pso, (void*)o.psn,
                    (void*)o.psf, (void*)o.psc, (void*)o.Acol, (void*)o.Aval})
      ar.give(q, o.owned);
    if (o.pskrc != o.psk) ar.give(o.pskrc, o.owned);
  }
  T.stage_ms[6] = ms_since(t0);
  // host remainder: non-orthogonal switches, volumes, wall distance
  int n_gradbc = 0;
  for (int q = 0; q < m.n_patches; ++q) {
    int b = pc[q].bc_id;
    if (!(b == BC_OUTLET || b == BC_PERIODIC || b == BC_WALL_NOSLIP || b == BC_WALL_VELOCITY ||
          b == BC_WALL_MODEL || b == BC_SLIP || b == BC_SYMMETRY))
      n_gradbc++;
  }
  S.skip_grad_p = S.skip_nonortho && n_gradbc == 0;
  S.n_nonortho_corr = P.n_nonortho_corr > 0 ? P.n_nonortho_corr : (S.skip_nonortho ? 1 : 2);
  if (!S.skip_nonortho)
    for (int64_t b = 0; b < nfb; ++b)
      for (int j = 0; j < 3; ++j) S.bnd_kout[j * nfb + b] = kb[3 * b + j];
  S.diag_interface = refine_any != 0;
  S.V_min = 1e300;
  S.V_total = 0.0;
  for (int64_t c = 0; c < nc; ++c) { S.V_min = std::min(S.V_min, m.volume[c]); S.V_total += m.volume[c]; }
  S.y_w.assign(nfb, 0.0);
  for (int64_t b = 0; b < nfb; ++b) {
    if (S.bnd_bc[b] != BC_WALL_MODEL) continue;
    int64_t f = nfi + b;
    int o = m.owner[f];
    double d[3], nin[3];
    for (int j = 0; j < 3; ++j) { d[j] = m.centroid[3 * o + j] - m.centre[3 * f + j]; nin[j] = -m.normal[3 * f + j]; }
    S.y_w[b] = std::fabs(d[0] * nin[0] + d[1] * nin[1] + d[2] * nin[2]) + SMALL;
  }
  T.ops_ms = ms_since(t_ops);
#undef SCK
#undef SLAUNCH
  return 0;
}
}  // namespace

int build_setup_device(const RawMesh& raw, const dpm_patch_cfg_t* pc, const dpm_params_t& P, int device, Mesh& m,
                       StaticOps& S, std::string* err, SetupTimes* times, SetupDeviceArrays* dev) {
  return setup_device_impl(&raw, nullptr, pc, P, device, m, S, err, times, dev);
}

int build_setup_device_poly(const PolyMesh& pm, const dpm_patch_cfg_t* pc, const dpm_params_t& P, int device,
                            Mesh& m, StaticOps& S, std::string* err, SetupTimes* times, SetupDeviceArrays* dev) {
  return setup_device_impl(nullptr, &pm, pc, P, device, m, S, err, times, dev);
}

}  // namespace dpm

// ---- builder comparison (C-ABI) ----------------------------------------------------------------

namespace dpm {
namespace {

const char* const kSetupArrays[] = {
    "centroid", "volume", "cell_face_off", "cell_faces", "owner", "neighbour", "patch", "area", "centre", "normal",
    "sf", "d_cf", "gc", "eps", "skew", "is_refine", "patch_start", "patch_nfaces", "periodic_pair",
    "periodic_pair_dcf", "periodic_gc", "ls_off", "ls_cell", "ls_face", "ls_w", "mesh_scalars", "ps_o", "ps_n",
    "ps_f", "ps_coeff", "ps_gcf", "ps_gcw", "ps_k", "ps_krc", "diag", "bnd_kout", "bnd_cb", "bnd_bc", "bnd_pnb",
    "dir_rows", "dir_vals", "A_col", "A_val", "cell_face", "cell_ps", "cell_bnd", "ls_idx", "ls_w_ell", "Tinv",
    "y_w", "wblend", "ops_scalars"};
constexpr int kNSetupArrays = (int)(sizeof(kSetupArrays) / sizeof(kSetupArrays[0]));

template <class T>
int64_t n_diff(const std::vector<T>& a, const std::vector<T>& b) {
  if (a.size() != b.size()) return (int64_t)std::max(a.size(), b.size()) + 1;
  int64_t n = 0;
  for (size_t i = 0; i < a.size(); ++i) n += std::memcmp(&a[i], &b[i], sizeof(T)) != 0;
  return n;
}

void compare_meshes(const Mesh& mh, const StaticOps& Sh, const Mesh& md, const StaticOps& Sd, int64_t* mismatches,
                    double* G_max_rel) {
  for (int k = 0; k < DPM_SETUP_N_ARRAYS; ++k) mismatches[k] = 0;
  int k = 0;
  auto put = [&](int64_t v) { mismatches[k++] = v; };
  put(n_diff(mh.centroid, md.centroid)); put(n_diff(mh.volume, md.volume));
  put(n_diff(mh.cell_face_off, md.cell_face_off)); put(n_diff(mh.cell_faces, md.cell_faces));
  put(n_diff(mh.owner, md.owner)); put(n_diff(mh.neighbour, md.neighbour)); put(n_diff(mh.patch, md.patch));
  put(n_diff(mh.area, md.area)); put(n_diff(mh.centre, md.centre)); put(n_diff(mh.normal, md.normal));
  put(n_diff(mh.sf, md.sf)); put(n_diff(mh.d_cf, md.d_cf)); put(n_diff(mh.gc, md.gc)); put(n_diff(mh.eps, md.eps));
  put(n_diff(mh.skew, md.skew)); put(n_diff(mh.is_refine, md.is_refine));
  put(n_diff(mh.patch_start, md.patch_start)); put(n_diff(mh.patch_nfaces, md.patch_nfaces));
  put(n_diff(mh.periodic_pair, md.periodic_pair)); put(n_diff(mh.periodic_pair_dcf, md.periodic_pair_dcf));
  put(n_diff(mh.periodic_gc, md.periodic_gc)); put(n_diff(mh.ls_off, md.ls_off));
  put(n_diff(mh.ls_cell, md.ls_cell)); put(n_diff(mh.ls_face, md.ls_face)); put(n_diff(mh.ls_w, md.ls_w));
  put((mh.n_cells != md.n_cells) + (mh.n_faces != md.n_faces) + (mh.n_int_faces != md.n_int_faces) +
      (mh.n_bnd_faces != md.n_bnd_faces) + (mh.ls_degenerate != md.ls_degenerate) +
      n_diff(mh.vertices, md.vertices) + n_diff(mh.cell_vert_off, md.cell_vert_off) +
      n_diff(mh.cell_vertices, md.cell_vertices) + n_diff(mh.patch_bc, md.patch_bc));
  put(n_diff(Sh.ps_o, Sd.ps_o)); put(n_diff(Sh.ps_n, Sd.ps_n)); put(n_diff(Sh.ps_f, Sd.ps_f));
  put(n_diff(Sh.ps_coeff, Sd.ps_coeff)); put(n_diff(Sh.ps_gcf, Sd.ps_gcf)); put(n_diff(Sh.ps_gcw, Sd.ps_gcw));
  put(n_diff(Sh.ps_k, Sd.ps_k)); put(n_diff(Sh.ps_krc, Sd.ps_krc)); put(n_diff(Sh.diag, Sd.diag));
  put(n_diff(Sh.bnd_kout, Sd.bnd_kout)); put(n_diff(Sh.bnd_cb, Sd.bnd_cb)); put(n_diff(Sh.bnd_bc, Sd.bnd_bc));
  put(n_diff(Sh.bnd_pnb, Sd.bnd_pnb)); put(n_diff(Sh.dir_rows, Sd.dir_rows)); put(n_diff(Sh.dir_vals, Sd.dir_vals));
  put(n_diff(Sh.A_col, Sd.A_col)); put(n_diff(Sh.A_val, Sd.A_val)); put(n_diff(Sh.cell_face, Sd.cell_face));
  put(n_diff(Sh.cell_ps, Sd.cell_ps)); put(n_diff(Sh.cell_bnd, Sd.cell_bnd)); put(n_diff(Sh.ls_idx, Sd.ls_idx));
  put(n_diff(Sh.ls_w, Sd.ls_w)); put(n_diff(Sh.Tinv, Sd.Tinv)); put(n_diff(Sh.y_w, Sd.y_w));
  put(n_diff(Sh.wblend, Sd.wblend));
  put((Sh.nc != Sd.nc) + (Sh.nf != Sd.nf) + (Sh.nfi != Sd.nfi) + (Sh.nb != Sd.nb) + (Sh.nfp != Sd.nfp) +
      (Sh.S != Sd.S) + (Sh.SP != Sd.SP) + (Sh.SB != Sd.SB) + (Sh.W != Sd.W) + (Sh.WA != Sd.WA) +
      (Sh.skip_nonortho != Sd.skip_nonortho) + (Sh.skip_grad_p != Sd.skip_grad_p) +
      (Sh.diag_interface != Sd.diag_interface) + (Sh.n_nonortho_corr != Sd.n_nonortho_corr) +
      (Sh.n_outlet != Sd.n_outlet) + (std::memcmp(&Sh.V_min, &Sd.V_min, sizeof(double)) != 0) +
      (std::memcmp(&Sh.V_total, &Sd.V_total, sizeof(double)) != 0));
  // per cell: largest entry difference relative to the tensor's scale |G_11| + |G_22| + |G_33|
  // (off-diagonal entries near zero come from cancellation, so entry-wise ratios mean nothing)
  double gmax = Sh.G.size() == Sd.G.size() ? 0.0 : 1e300;
  if (Sh.G.size() == Sd.G.size())
    for (size_t c = 0; c + 9 <= Sh.G.size(); c += 9) {
      const double* a = &Sh.G[c];
      const double* b = &Sd.G[c];
      const double scale = std::fabs(a[0]) + std::fabs(a[4]) + std::fabs(a[8]);
      for (int j = 0; j < 9; ++j) {
        double e = a[j] == b[j] ? 0.0 : std::fabs(a[j] - b[j]) / std::max(scale, 1e-300);
        if (!(e <= gmax)) gmax = e;
      }
    }
  *G_max_rel = gmax;
}

}  // namespace

}  // namespace dpm

extern "C" int dpm_setup_compare(const dpm_raw_mesh_t* raw, const dpm_patch_cfg_t* patches, const dpm_params_t* params,
                                 int device, int64_t* mismatches, double* G_max_rel, double* ms) {
  using namespace dpm;
  if (!raw || !patches || !params || !mismatches || !G_max_rel) return DPM_ERR_ARG;
  static_assert(kNSetupArrays <= DPM_SETUP_N_ARRAYS, "array table");
  RawMesh r;
  r.n_nodes = raw->n_nodes; r.xyz = raw->xyz; r.n_cells = raw->n_cells; r.cell_type = raw->cell_type;
  r.cell_off = raw->cell_off; r.cell_nodes = raw->cell_nodes; r.n_bfaces = raw->n_bfaces;
  r.bface_off = raw->bface_off; r.bface_nodes = raw->bface_nodes; r.bface_patch = raw->bface_patch;
  r.n_patches = raw->n_patches;
  std::vector<int> pbc(raw->n_patches);
  for (int i = 0; i < raw->n_patches; ++i) pbc[i] = patches[i].bc_id;
  Mesh mh, md;
  StaticOps Sh, Sd;
  std::string err;
  auto t0 = std::chrono::steady_clock::now();
  if (build_mesh(r, pbc.data(), mh, &err)) return DPM_ERR_MESH;
  auto t1 = std::chrono::steady_clock::now();
  if (build_static_ops(mh, patches, *params, Sh)) return DPM_ERR_MESH;
  auto t2 = std::chrono::steady_clock::now();
  SetupTimes tt;
  int rc = build_setup_device(r, patches, *params, device, md, Sd, &err, &tt);
  if (rc) {
    std::fprintf(stderr, "dopamine_b200: device set-up failed: %s\n", err.c_str());
    return rc == SETUP_DEVICE_LIMIT ? DPM_ERR_UNSUPPORTED : (rc < 0 && rc >= -4 ? DPM_ERR_MESH : rc);
  }
  if (ms) {
    ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    ms[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
    ms[2] = tt.mesh_ms;
    ms[3] = tt.ops_ms;
  }
  compare_meshes(mh, Sh, md, Sd, mismatches, G_max_rel);
  return 0;
}

extern "C" const char* dpm_setup_array_name(int k) {
  return (k >= 0 && k < dpm::kNSetupArrays) ? dpm::kSetupArrays[k] : nullptr;
}

extern "C" int dpm_setup_compare_poly(const dpm_poly_mesh_t* pmsh, const dpm_patch_cfg_t* patches,
                                      const dpm_params_t* params, int device, int64_t* mismatches, double* G_max_rel,
                                      double* ms) {
  using namespace dpm;
  if (!pmsh || !patches || !params || !mismatches || !G_max_rel) return DPM_ERR_ARG;
  PolyMesh pm;
  pm.n_points = pmsh->n_points; pm.xyz = pmsh->xyz; pm.n_faces = pmsh->n_faces; pm.face_off = pmsh->face_off;
  pm.face_nodes = pmsh->face_nodes; pm.owner = pmsh->owner; pm.n_int_faces = pmsh->n_int_faces;
  pm.neighbour = pmsh->neighbour; pm.n_patches = pmsh->n_patches; pm.patch_start = pmsh->patch_start;
  pm.patch_nfaces = pmsh->patch_nfaces;
  std::vector<int> pbc(pmsh->n_patches);
  for (int i = 0; i < pmsh->n_patches; ++i) pbc[i] = patches[i].bc_id;
  Mesh mh, md;
  StaticOps Sh, Sd;
  std::string err;
  auto t0 = std::chrono::steady_clock::now();
  if (build_mesh_poly(pm, pbc.data(), mh, &err)) return DPM_ERR_MESH;
  auto t1 = std::chrono::steady_clock::now();
  if (build_static_ops(mh, patches, *params, Sh)) return DPM_ERR_MESH;
  auto t2 = std::chrono::steady_clock::now();
  SetupTimes tt;
  int rc = build_setup_device_poly(pm, patches, *params, device, md, Sd, &err, &tt);
  if (rc) {
    std::fprintf(stderr, "dopamine_b200: device set-up failed: %s\n", err.c_str());
    return rc == SETUP_DEVICE_LIMIT ? DPM_ERR_UNSUPPORTED : (rc < 0 && rc >= -8 ? DPM_ERR_MESH : rc);
  }
  if (ms) {
    ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    ms[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
    ms[2] = tt.mesh_ms;
    ms[3] = tt.ops_ms;
  }
  compare_meshes(mh, Sh, md, Sd, mismatches, G_max_rel);
  return 0;
}

// ---- host builder digests (C-ABI, no device) ---------------------------------------------------

namespace dpm {
namespace {

// 64-bit FNV-1a over the bytes, seeded with the element count.
struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void bytes(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
  }
  void i64(int64_t v) { bytes(&v, sizeof(v)); }
  template <class T> void vec(const std::vector<T>& v) {
    i64((int64_t)v.size());
    bytes(v.data(), v.size() * sizeof(T));
  }
};

template <class T> uint64_t digest(const std::vector<T>& v) {
  Fnv f;
  f.vec(v);
  return f.h;
}

// One digest per array, in kSetupArrays order; returns how many were written.
int digest_setup(const Mesh& m, const StaticOps& S, uint64_t* out) {
  int k = 0;
  auto put = [&](uint64_t v) { out[k++] = v; };
  put(digest(m.centroid)); put(digest(m.volume)); put(digest(m.cell_face_off)); put(digest(m.cell_faces));
  put(digest(m.owner)); put(digest(m.neighbour)); put(digest(m.patch)); put(digest(m.area));
  put(digest(m.centre)); put(digest(m.normal)); put(digest(m.sf)); put(digest(m.d_cf)); put(digest(m.gc));
  put(digest(m.eps)); put(digest(m.skew)); put(digest(m.is_refine)); put(digest(m.patch_start));
  put(digest(m.patch_nfaces)); put(digest(m.periodic_pair)); put(digest(m.periodic_pair_dcf));
  put(digest(m.periodic_gc)); put(digest(m.ls_off)); put(digest(m.ls_cell)); put(digest(m.ls_face));
  put(digest(m.ls_w));
  {
    Fnv f;
    f.i64(m.n_cells); f.i64(m.n_faces); f.i64(m.n_int_faces); f.i64(m.n_bnd_faces); f.i64(m.ls_degenerate);
    f.vec(m.vertices); f.vec(m.cell_vert_off); f.vec(m.cell_vertices); f.vec(m.patch_bc);
    put(f.h);
  }
  put(digest(S.ps_o)); put(digest(S.ps_n)); put(digest(S.ps_f)); put(digest(S.ps_coeff)); put(digest(S.ps_gcf));
  put(digest(S.ps_gcw)); put(digest(S.ps_k)); put(digest(S.ps_krc)); put(digest(S.diag)); put(digest(S.bnd_kout));
  put(digest(S.bnd_cb)); put(digest(S.bnd_bc)); put(digest(S.bnd_pnb)); put(digest(S.dir_rows));
  put(digest(S.dir_vals)); put(digest(S.A_col)); put(digest(S.A_val)); put(digest(S.cell_face));
  put(digest(S.cell_ps)); put(digest(S.cell_bnd)); put(digest(S.ls_idx)); put(digest(S.ls_w)); put(digest(S.Tinv));
  put(digest(S.y_w)); put(digest(S.wblend));
  {
    Fnv f;
    for (int64_t v : {(int64_t)S.nc, (int64_t)S.nf, (int64_t)S.nfi, (int64_t)S.nb, (int64_t)S.nfp, (int64_t)S.S,
                      (int64_t)S.SP, (int64_t)S.SB, (int64_t)S.W, (int64_t)S.WA, (int64_t)S.skip_nonortho,
                      (int64_t)S.skip_grad_p, (int64_t)S.diag_interface, (int64_t)S.n_nonortho_corr,
                      (int64_t)S.n_outlet})
      f.i64(v);
    f.bytes(&S.V_min, sizeof(double));
    f.bytes(&S.V_total, sizeof(double));
    put(f.h);
  }
  return k;
}

int host_digest(const RawMesh* raw, const PolyMesh* poly, int n_patches, const dpm_patch_cfg_t* patches,
                const dpm_params_t& P, uint64_t* digests, int* n_arrays, uint64_t* G_digest, char* errbuf,
                int errlen) {
  std::vector<int> pbc(n_patches);
  for (int i = 0; i < n_patches; ++i) pbc[i] = patches[i].bc_id;
  Mesh m;
  StaticOps S;
  std::string err;
  int rc = raw ? build_mesh(*raw, pbc.data(), m, &err) : build_mesh_poly(*poly, pbc.data(), m, &err);
  if (rc) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", err.c_str());
    return DPM_ERR_MESH;
  }
  rc = build_static_ops(m, patches, P, S);
  if (rc) {
    if (errbuf && errlen > 0)
      std::snprintf(errbuf, (size_t)errlen, "%s",
                    rc == DPM_ERR_UNSUPPORTED ? "a matrix row wider than 16 entries" : "static operators refused the mesh");
    return rc;
  }
  const int n = digest_setup(m, S, digests);
  if (n_arrays) *n_arrays = n;
  if (G_digest) *G_digest = digest(S.G);
  return n == kNSetupArrays ? DPM_OK : DPM_ERR_ARG;
}

}  // namespace
}  // namespace dpm

extern "C" int dpm_setup_host_digest(const dpm_raw_mesh_t* raw, const dpm_patch_cfg_t* patches,
                                     const dpm_params_t* params, uint64_t* digests, int* n_arrays, uint64_t* G_digest,
                                     char* errbuf, int errlen) {
  using namespace dpm;
  if (!raw || (raw->n_patches > 0 && !patches) || !params || !digests) return DPM_ERR_ARG;
  RawMesh r;
  r.n_nodes = raw->n_nodes; r.xyz = raw->xyz; r.n_cells = raw->n_cells; r.cell_type = raw->cell_type;
  r.cell_off = raw->cell_off; r.cell_nodes = raw->cell_nodes; r.n_bfaces = raw->n_bfaces;
  r.bface_off = raw->bface_off; r.bface_nodes = raw->bface_nodes; r.bface_patch = raw->bface_patch;
  r.n_patches = raw->n_patches;
  return host_digest(&r, nullptr, raw->n_patches, patches, *params, digests, n_arrays, G_digest, errbuf, errlen);
}

extern "C" int dpm_setup_host_digest_poly(const dpm_poly_mesh_t* pmsh, const dpm_patch_cfg_t* patches,
                                          const dpm_params_t* params, uint64_t* digests, int* n_arrays,
                                          uint64_t* G_digest, char* errbuf, int errlen) {
  using namespace dpm;
  if (!pmsh || (pmsh->n_patches > 0 && !patches) || !params || !digests) return DPM_ERR_ARG;
  PolyMesh pm;
  pm.n_points = pmsh->n_points; pm.xyz = pmsh->xyz; pm.n_faces = pmsh->n_faces; pm.face_off = pmsh->face_off;
  pm.face_nodes = pmsh->face_nodes; pm.owner = pmsh->owner; pm.n_int_faces = pmsh->n_int_faces;
  pm.neighbour = pmsh->neighbour; pm.n_patches = pmsh->n_patches; pm.patch_start = pmsh->patch_start;
  pm.patch_nfaces = pmsh->patch_nfaces;
  return host_digest(nullptr, &pm, pmsh->n_patches, patches, *params, digests, n_arrays, G_digest, errbuf, errlen);
}
