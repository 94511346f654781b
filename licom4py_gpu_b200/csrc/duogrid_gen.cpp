// duogrid_gen.cpp - cubed-sphere duogrid geometry generator (host C++).
//
// Restates the reference's Fortran library src/duogrid_c/chtholly/global_grid/*
// (built there with -fdefault-real-8, so every real is IEEE double) for
// grid_type 0 (equal-edge gnomonic), ng = 3, and the Python post-processing
// of src/initial_field/main.py (transpose, truncation to res+6, stacking of
// the six tiles).  Each routine below cites the Fortran it follows.
//
// Arithmetic follows the Fortran expression order term by term and the file
// is compiled with -ffp-contract=off (no FMA), so that glibc libm plus IEEE
// double reproduce what gfortran (x86-64, no -march) would compute.
//
// Storage differs from the Fortran: the quantities that are identical on all
// six tiles (ext_x/ext_y/kik_x/kik_y, ext_dx/ext_dy/ext_da, k2e tables) are
// stored once, and the per-point vector/matrix quantities (e1co, e2co, sina,
// g_co, c2l, ...) are evaluated on demand at the sampled super-grid points
// instead of being stored on the whole 2x super-grid.  The kinked-grid vector
// quantities of global_grid_gen_vec.F90 (kik_e1co, kik_sina, kik_c2l, ...) feed
// no exported field and are not computed.

#include "../../include/licom_duogrid.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;     // lib_grid.F90:17
constexpr double kRadius = 6.3712e+6;              // lib_grid.F90:16
constexpr double kOmega = 7.292e-5;                // lib_grid.F90:19
constexpr int kNg = 3;                             // halo width (initial_field/main.py:107)
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

struct V3 {
  double x, y, z;
};

// lib_grid.F90:80-95
inline V3 lonlat2cart(double lon, double lat) {
  return {std::cos(lat) * std::cos(lon), std::cos(lat) * std::sin(lon), std::sin(lat)};
}

// lib_grid.F90:191-199
inline V3 cross(const V3& a, const V3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// gfortran dot_product: sequential sum a1*b1 + a2*b2 + a3*b3
inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// lib_grid.F90:178-189
inline V3 normv(const V3& r) {
  double d = std::sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
  return {r.x / d, r.y / d, r.z / d};
}

// lib_grid.F90:55-78
inline void cart2lonlat(const V3& c, double* lon, double* lat) {
  double n = std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
  V3 p{c.x / n, c.y / n, c.z / n};
  const double esl = 1.e-5;
  double lo;
  if ((std::fabs(p.x) + std::fabs(p.y)) < esl) {
    lo = 0.;
  } else {
    lo = std::atan2(p.y, p.x);
  }
  if (lo < 0.) lo = 2. * kPi + lo;
  *lon = lo;
  *lat = std::asin(p.z);
}

// lib_grid.F90:161-176
inline V3 unit_vec_2pt(double lon1, double lat1, double lon2, double lat2) {
  V3 p1 = lonlat2cart(lon1, lat1);
  V3 p2 = lonlat2cart(lon2, lat2);
  V3 p12 = cross(p1, p2);
  V3 e = cross(p12, p1);
  return normv(e);
}

// lib_grid.F90:123-159
inline double area_4pt(const double* q1, const double* q2, const double* q3, const double* q4,
                       double r) {
  V3 p1 = lonlat2cart(q1[0], q1[1]);
  V3 p2 = lonlat2cart(q2[0], q2[1]);
  V3 p3 = lonlat2cart(q3[0], q3[1]);
  V3 p4 = lonlat2cart(q4[0], q4[1]);
  V3 p12 = normv(cross(p1, p2));
  V3 p23 = normv(cross(p2, p3));
  V3 p34 = normv(cross(p3, p4));
  V3 p41 = normv(cross(p4, p1));
  double c123 = dot(p12, p23);
  double c234 = dot(p23, p34);
  double c341 = dot(p34, p41);
  double c412 = dot(p41, p12);
  double a123 = std::acos(-c123);
  double a234 = std::acos(-c234);
  double a341 = std::acos(-c341);
  double a412 = std::acos(-c412);
  return (a123 + a234 + a341 + a412 - 2 * kPi) * (r * r);
}

struct M2 {
  double m[2][2];  // m[a][b] = Fortran (a+1, b+1)
};

// 2x2 matmul in the order gfortran's inline matmul uses: C(a,b) = A(a,1)B(1,b) + A(a,2)B(2,b)
inline M2 matmul2(const M2& A, const M2& B) {
  M2 C;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) C.m[a][b] = A.m[a][0] * B.m[0][b] + A.m[a][1] * B.m[1][b];
  return C;
}

}  // namespace

struct ldg_grid {
  int res = 0;
  // super grid (2x resolution) index range, global_grid_alloc.F90:205-208
  int s_lo = 0, s_hi = 0, sw = 0;
  // A-grid index range of the k2e tables, global_grid_alloc.F90:267-270
  int a_lo = 0, a_hi = 0, aw = 0;
  // output A-grid range isd..ied (initial_field/main.py:54-55) and width M
  int isd = -2, ied = 0, M = 0;

  std::vector<double> pt_ext;  // [n][j][i][2] lon, lat
  std::vector<double> pt_kik;  // [n][j][i][2]
  // tile-independent super-grid quantities [j][i]
  std::vector<double> ext_x, ext_y, kik_x, kik_y, ext_dx, ext_dy, ext_da;
  // tile-independent k2e tables on the A grid [j][i] and [j][i][2]
  std::vector<int> k2e_loc;
  std::vector<double> k2e_coef;

  size_t sidx(int i, int j) const { return (size_t)(j - s_lo) * sw + (i - s_lo); }
  size_t pidx(int i, int j, int n) const { return (((size_t)(n - 1) * sw + (j - s_lo)) * sw + (i - s_lo)) * 2; }
  size_t aidx(int i, int j) const { return (size_t)(j - a_lo) * aw + (i - a_lo); }

  double lon(int i, int j, int n) const { return pt_ext[pidx(i, j, n)]; }
  double lat(int i, int j, int n) const { return pt_ext[pidx(i, j, n) + 1]; }

  // ---- per-point ext quantities (global_grid_gen_vec.F90) -------------------
  // e1co / e2co, global_grid_gen_vec.F90:54-82
  V3 e1co(int i, int j, int n) const {
    if (i == s_hi) {
      V3 e = unit_vec_2pt(lon(i, j, n), lat(i, j, n), lon(i - 1, j, n), lat(i - 1, j, n));
      return {-e.x, -e.y, -e.z};
    }
    return unit_vec_2pt(lon(i, j, n), lat(i, j, n), lon(i + 1, j, n), lat(i + 1, j, n));
  }
  V3 e2co(int i, int j, int n) const {
    if (j == s_hi) {
      V3 e = unit_vec_2pt(lon(i, j, n), lat(i, j, n), lon(i, j - 1, n), lat(i, j - 1, n));
      return {-e.x, -e.y, -e.z};
    }
    return unit_vec_2pt(lon(i, j, n), lat(i, j, n), lon(i, j + 1, n), lat(i, j + 1, n));
  }
  // global_grid_gen_vec.F90:265-280
  V3 elon(int i, int j, int n) const {
    double lo = lon(i, j, n);
    return {-std::sin(lo), std::cos(lo), 0.};
  }
  V3 elat(int i, int j, int n) const {
    double lo = lon(i, j, n), la = lat(i, j, n);
    return {-std::sin(la) * std::cos(lo), -std::sin(la) * std::sin(lo), std::cos(la)};
  }
  // global_grid_gen_vec.F90:334-345
  void sincos_a(int i, int j, int n, double* sina, double* cosa) const {
    double c = dot(e1co(i, j, n), e2co(i, j, n));
    *cosa = c;
    *sina = std::sqrt(1. - c * c);
  }

  struct Mats {
    double sina, cosa;
    M2 g_co, g_ctr, ct2ort_x, ort2ct_x, ct2ort_y, ort2ct_y, ct2rll, rll2ct, c2l, l2c;
  };

  // global_grid_gen_vec.F90:413-489 (the ext branch of global_grid_gen_mat)
  Mats mats(int i, int j, int n) const {
    Mats r;
    double sina, cosa;
    sincos_a(i, j, n, &sina, &cosa);
    r.sina = sina;
    r.cosa = cosa;
    r.g_co.m[0][0] = 1.;
    r.g_co.m[0][1] = cosa;
    r.g_co.m[1][0] = cosa;
    r.g_co.m[1][1] = 1.;
    double coef = 1. / sina / sina;
    r.g_ctr.m[0][0] = coef;
    r.g_ctr.m[0][1] = -(coef * cosa);
    r.g_ctr.m[1][0] = -(coef * cosa);
    r.g_ctr.m[1][1] = coef;
    double gct11 = r.g_ctr.m[0][0], gco12 = r.g_co.m[0][1], gco22 = r.g_co.m[1][1];
    double gct22 = r.g_ctr.m[1][1], gco11 = r.g_co.m[0][0], gco21 = r.g_co.m[1][0];
    r.ct2ort_x.m[0][0] = 1. / std::sqrt(gct11);
    r.ct2ort_x.m[0][1] = 0.;
    r.ct2ort_x.m[1][0] = gco12 / std::sqrt(gco22);
    r.ct2ort_x.m[1][1] = std::sqrt(gco22);
    r.ort2ct_x.m[0][0] = std::sqrt(gct11);
    r.ort2ct_x.m[0][1] = 0.;
    r.ort2ct_x.m[1][0] = -((gco12 / gco22) * std::sqrt(gct11));
    r.ort2ct_x.m[1][1] = 1. / std::sqrt(gco22);
    r.ct2ort_y.m[0][0] = 0.;
    r.ct2ort_y.m[0][1] = 1. / std::sqrt(gct22);
    r.ct2ort_y.m[1][0] = std::sqrt(gco11);
    r.ct2ort_y.m[1][1] = gco21 / std::sqrt(gco11);
    r.ort2ct_y.m[0][0] = -((gco21 / gco11) * std::sqrt(gct22));
    r.ort2ct_y.m[0][1] = 1. / std::sqrt(gco11);
    r.ort2ct_y.m[1][0] = std::sqrt(gct22);
    r.ort2ct_y.m[1][1] = 0.;
    V3 e1 = e1co(i, j, n), e2 = e2co(i, j, n), el = elon(i, j, n), et = elat(i, j, n);
    M2 mat;
    mat.m[0][0] = dot(e1, el);
    mat.m[0][1] = dot(e2, el);
    mat.m[1][0] = dot(e1, et);
    mat.m[1][1] = dot(e2, et);
    r.ct2rll = mat;
    double c2 = 1. / (mat.m[0][0] * mat.m[1][1] - mat.m[0][1] * mat.m[1][0]);
    r.rll2ct.m[0][0] = c2 * mat.m[1][1];
    r.rll2ct.m[0][1] = -(c2 * mat.m[0][1]);
    r.rll2ct.m[1][0] = -(c2 * mat.m[1][0]);
    r.rll2ct.m[1][1] = c2 * mat.m[0][0];
    r.c2l = matmul2(r.ct2rll, r.g_ctr);
    r.l2c = matmul2(r.g_co, r.rll2ct);
    return r;
  }

  double sx(const std::vector<double>& a, int i, int j) const { return a[sidx(i, j)]; }
};

namespace {

// Fortran get_neighbor_tile_num, global_grid_util.F90:127-146 (1-based tiles)
void neighbor_tiles(int n, int* nw, int* ne, int* ns, int* nn) {
  if (n % 2 == 0) {
    *nn = (n + 0) % 6 + 1;
    *ne = (n + 1) % 6 + 1;
    *ns = (n + 3) % 6 + 1;
    *nw = (n + 4) % 6 + 1;
  } else {
    *ne = (n + 0) % 6 + 1;
    *nn = (n + 1) % 6 + 1;
    *nw = (n + 3) % 6 + 1;
    *ns = (n + 4) % 6 + 1;
  }
}

// get_neighbor_index, global_grid_util.F90:53-101
void neighbor_index(int* ii, int* jj, int i, int j, int n, int n_src, int npx, int npy) {
  const int isc = 1, jsc = 1, iec = npx, jec = npy;
  int nw, ne, ns, nn;
  neighbor_tiles(n, &nw, &ne, &ns, &nn);
  if (n % 2 != 0) {
    if (n_src == nw) { *ii = iec - (j - jsc); *jj = jec + (i - isc); }
    if (n_src == ne) { *ii = isc + (i - iec); *jj = jsc + (j - jsc); }
    if (n_src == ns) { *ii = isc + (i - isc); *jj = jec + (j - jsc); }
    if (n_src == nn) { *ii = isc + (j - jec); *jj = jec - (i - isc); }
  } else {
    if (n_src == nw) { *ii = iec + (i - isc); *jj = jsc + (j - jsc); }
    if (n_src == ne) { *ii = iec - (j - jsc); *jj = jsc + (i - iec); }
    if (n_src == ns) { *ii = iec + (j - jsc); *jj = jec - (i - isc); }
    if (n_src == nn) { *ii = isc + (i - isc); *jj = jsc + (j - jec); }
  }
}

// get_neighbor_bounds, global_grid_util.F90:103-125
void neighbor_bounds(int* is, int* ie, int* js, int* je, int n, int n_src, int npx, int npy, int ng) {
  const int isc = 1, jsc = 1, iec = npx, jec = npy;
  int nw, ne, ns, nn;
  neighbor_tiles(n, &nw, &ne, &ns, &nn);
  if (n_src == nw) { *is = isc - ng; *ie = isc - 1; *js = jsc; *je = jec; }
  if (n_src == ne) { *is = iec + 1; *ie = iec + ng; *js = jsc; *je = jec; }
  if (n_src == ns) { *is = isc; *ie = iec; *js = jsc - ng; *je = jsc - 1; }
  if (n_src == nn) { *is = isc; *ie = iec; *js = jec + 1; *je = jec + ng; }
}

// global_grid_gen_lonlat.F90:18-150 (grid_type 0) and global_grid_update_kik
// (global_grid_util.F90:23-51) for the lon/lat points.
void gen_lonlat(ldg_grid& g) {
  const int is = 1, ie = 2 * g.res + 1, js = is, je = ie;
  const int ng = 2 * kNg;
  const int isd = is - ng, ied = ie + ng, jsd = isd, jed = ied;
  const int nc = 1 + g.res;
  std::vector<double> line(ied - isd + 1, -999.);
  auto L = [&](int k) -> double& { return line[k - isd]; };

  const double rsq3 = 1.0 / std::sqrt(3.0);
  const double alpha = std::asin(rsq3);
  const double dela = 2.0 * alpha / (double)(ie - is);
  L(js) = -1.;
  L(nc) = 0.;
  for (int j = js + 1; j <= nc - 1; ++j) {
    double angl_y = (double)(j - 1) * dela - alpha;
    L(j) = std::tan(angl_y) * std::sqrt(2.0);
  }
  for (int j = jsd; j <= js - 1; ++j) {
    int jj = 2 * js - j;
    double angl_g = -0.5 * kPi - std::atan(L(jj));
    L(j) = std::tan(angl_g);
  }
  for (int j = jsd; j <= nc - 1; ++j) {
    int jj = je - j + 1;
    L(jj) = -L(j);
  }
  for (int n = 1; n <= 6; ++n) {
    for (int j = jsd; j <= jed; ++j) {
      for (int i = isd; i <= ied; ++i) {
        double x = L(i), y = L(j);
        V3 c;
        switch (n) {
          case 1: c = {1.0, x, y}; break;
          case 2: c = {-x, 1.0, y}; break;
          case 3: c = {-x, -y, 1.0}; break;
          case 4: c = {-1.0, -y, -x}; break;
          case 5: c = {y, -1.0, -x}; break;
          default: c = {y, x, -1.0}; break;
        }
        size_t p = g.pidx(i, j, n);
        cart2lonlat(c, &g.pt_ext[p], &g.pt_ext[p + 1]);
      }
    }
  }
  // global_grid_update_kik with np = 2
  std::fill(g.pt_kik.begin(), g.pt_kik.end(), -999.);
  const int ks = isd + ng, ke = ied - ng;  // = is, ie
  for (int n = 1; n <= 6; ++n)
    for (int j = ks; j <= ke; ++j)
      for (int i = ks; i <= ke; ++i) {
        size_t p = g.pidx(i, j, n);
        g.pt_kik[p] = g.pt_ext[p];
        g.pt_kik[p + 1] = g.pt_ext[p + 1];
      }
  for (int n = 1; n <= 6; ++n) {
    int nb[4];
    neighbor_tiles(n, &nb[0], &nb[1], &nb[2], &nb[3]);  // nw, ne, ns, nn
    for (int k = 0; k < 4; ++k) {
      int n_src = nb[k];
      int isk = 0, iek = -1, jsk = 0, jek = -1;
      neighbor_bounds(&isk, &iek, &jsk, &jek, n, n_src, ke, ke, ng);
      for (int j = jsk; j <= jek; ++j)
        for (int i = isk; i <= iek; ++i) {
          int ii = 0, jj = 0;
          neighbor_index(&ii, &jj, i, j, n, n_src, ke, ke);
          size_t d = g.pidx(i, j, n), s = g.pidx(ii, jj, n_src);
          g.pt_kik[d] = g.pt_kik[s];
          g.pt_kik[d + 1] = g.pt_kik[s + 1];
        }
    }
  }
}

// global_grid_gen_coords.F90:27-117
void gen_coords(ldg_grid& g) {
  const int is = 1, ie = 2 * g.res + 1, js = is, je = ie;
  const int ng = 2 * kNg;
  const int jsd = is - ng, jed = ie + ng;
  const int nc = 1 + g.res;
  std::vector<double> line(jed - jsd + 1, -999.);
  auto L = [&](int k) -> double& { return line[k - jsd]; };
  for (int k = 1; k <= ng; ++k) {
    // kinked points of tile 1, column is-k
    L(nc) = 0.;
    for (int j = js; j <= nc - 1; ++j) {
      L(j) = g.pt_kik[g.pidx(is - k, j, 1) + 1] - g.pt_kik[g.pidx(is - k, nc, 1) + 1];
      L(je - j + 1) = -L(j);
    }
    for (int j = js; j <= je; ++j) {
      g.kik_y[g.sidx(is - k, j)] = L(j);
      g.kik_x[g.sidx(j, is - k)] = L(j);
      g.kik_y[g.sidx(ie + k, j)] = L(j);
      g.kik_x[g.sidx(j, ie + k)] = L(j);
    }
    // extended points of tile 1, column is-k
    L(nc) = 0.;
    for (int j = jsd; j <= nc - 1; ++j) {
      L(j) = g.pt_ext[g.pidx(is - k, j, 1) + 1] - g.pt_ext[g.pidx(is - k, nc, 1) + 1];
      L(je - j + 1) = -L(j);
    }
    for (int j = jsd; j <= jed; ++j) {
      g.ext_y[g.sidx(is - k, j)] = L(j);
      g.ext_x[g.sidx(j, is - k)] = L(j);
      g.ext_y[g.sidx(ie + k, j)] = L(j);
      g.ext_x[g.sidx(j, ie + k)] = L(j);
    }
  }
}

// global_grid_gen_cell.F90:28-128 (ext part of gen_ds; kik halo ds feeds no output)
void gen_ds(ldg_grid& g) {
  const int is = 1, ie = 2 * g.res + 1, je = ie;
  const int ng = 2 * kNg;
  const int isd = is - ng, jsd = isd;
  const int nc = 1 + g.res;
  for (int j = jsd; j <= nc - 1; ++j)
    for (int i = isd; i <= nc; ++i) {
      double dy = (g.lat(i, j + 1, 1) - g.lat(i, j, 1)) * kRadius;
      int ii = ie - i + 1, jj = je - j;
      g.ext_dy[g.sidx(i, j)] = dy;
      g.ext_dy[g.sidx(ii, j)] = dy;
      g.ext_dy[g.sidx(i, jj)] = dy;
      g.ext_dy[g.sidx(ii, jj)] = dy;
      g.ext_dx[g.sidx(j, i)] = dy;
      g.ext_dx[g.sidx(j, ii)] = dy;
      g.ext_dx[g.sidx(jj, i)] = dy;
      g.ext_dx[g.sidx(jj, ii)] = dy;
    }
}

// global_grid_gen_cell.F90:130-225 (ext part of gen_da)
void gen_da(ldg_grid& g) {
  const int is = 1, ie = 2 * g.res + 1, je = ie;
  const int ng = 2 * kNg;
  const int isd = is - ng, jsd = isd;
  const int nc = 1 + g.res;
  for (int j = jsd; j <= nc - 1; ++j)
    for (int i = isd; i <= nc - 1; ++i) {
      const double* p1 = &g.pt_ext[g.pidx(i, j, 1)];
      const double* p2 = &g.pt_ext[g.pidx(i + 1, j, 1)];
      const double* p3 = &g.pt_ext[g.pidx(i + 1, j + 1, 1)];
      const double* p4 = &g.pt_ext[g.pidx(i, j + 1, 1)];
      double da = area_4pt(p1, p2, p3, p4, kRadius);
      int ii = ie - i, jj = je - j;
      g.ext_da[g.sidx(i, j)] = da;
      g.ext_da[g.sidx(ii, j)] = da;
      g.ext_da[g.sidx(i, jj)] = da;
      g.ext_da[g.sidx(ii, jj)] = da;
    }
}

// global_grid_gen_k2e.F90:28-172, k2e_nord = 2 (linear Lagrange), np = 0.
void gen_k2e(ldg_grid& g) {
  const int is = 1, ie = g.res, js = is, je = ie;
  const int ng = kNg;
  const int isd = is - ng, ied = ie + ng, jsd = isd, jed = ied;
  const int np = 2 / 2 - 1;
  std::fill(g.k2e_loc.begin(), g.k2e_loc.end(), -999);
  std::fill(g.k2e_coef.begin(), g.k2e_coef.end(), -999.);
  auto ext_xa = [&](int i, int j) { return g.ext_x[g.sidx(2 * i, 2 * j)]; };
  auto ext_ya = [&](int i, int j) { return g.ext_y[g.sidx(2 * i, 2 * j)]; };
  auto kik_xa = [&](int i, int j) { return g.kik_x[g.sidx(2 * i, 2 * j)]; };
  auto kik_ya = [&](int i, int j) { return g.kik_y[g.sidx(2 * i, 2 * j)]; };
  std::vector<double> x(ie - is + 1), y(ied - isd + 1);
  auto X = [&](int k) { return x[k - is]; };
  auto set = [&](int i, int j, double yy) {
    int klo = is, khi = ie;
    while (khi - klo > 1) {
      int k = (khi + klo) / 2;
      if (X(k) > yy)
        khi = k;
      else
        klo = k;
    }
    klo = std::max(klo, is + np);
    klo = std::min(klo, ie - np - 1);
    khi = klo + 1;
    g.k2e_loc[g.aidx(i, j)] = klo;
    // lib_interp_lag_get_coef (lib_grid.F90:213-231) on (x(klo), x(khi))
    double x0 = X(klo), x1 = X(khi);
    double c0 = 1.;
    c0 = c0 * (yy - x1) / (x0 - x1);
    double c1 = 1.;
    c1 = c1 * (yy - x0) / (x1 - x0);
    g.k2e_coef[g.aidx(i, j) * 2 + 0] = c0;
    g.k2e_coef[g.aidx(i, j) * 2 + 1] = c1;
  };
  // k2e tables are identical for all six tiles (ext_x etc. are tile independent)
  for (int ii = 1; ii <= ng; ++ii) {
    // get_loc_x for rows j = js-ii and j = je+ii
    for (int j : {js - ii, je + ii}) {
      for (int k = is; k <= ie; ++k) x[k - is] = kik_xa(k, j);
      for (int k = isd; k <= ied; ++k) y[k - isd] = ext_xa(k, j);
      for (int i = is - ii + 1; i <= ie + ii - 1; ++i) set(i, j, y[i - isd]);
    }
    // get_loc_y for columns i = is-ii and i = ie+ii
    for (int i : {is - ii, ie + ii}) {
      for (int k = js; k <= je; ++k) x[k - js] = kik_ya(i, k);
      for (int k = jsd; k <= jed; ++k) y[k - jsd] = ext_ya(i, k);
      for (int j = js - ii + 1; j <= je + ii - 1; ++j) set(i, j, y[j - jsd]);
    }
  }
}

enum Kind { A2, A3, A4, B3, C2, C4, D2, D4, AI };

struct FieldDef {
  const char* name;
  Kind kind;
};

// Field names and layouts of the reference NPZ (src/licom/duogrid/duogrid.py:97-151,
// src/initial_field/_c_duogrid_function.py:216-307).
const FieldDef kFields[] = {
    {"a_x", A2},        {"a_y", A2},          {"a_kik_x", A2},      {"a_kik_y", A2},
    {"a_sina", A2},     {"a_cosa", A2},       {"a_dx", A2},         {"a_dy", A2},
    {"a_da", A2},       {"rda", A2},          {"rdx", A2},          {"rdy", A2},
    {"a_f", A2},        {"ub", A2},           {"vb", A2},           {"a_pt", A3},
    {"k2e_coef", A3},   {"a_gco", A4},        {"a_gct", A4},        {"a_c2l", A4},
    {"a_l2c", A4},      {"k2e_loc", AI},      {"k2e_loc_i", AI},    {"k2e_loc_j", AI},
    {"b_pt", B3},       {"c_gco", C4},        {"c_gct", C4},        {"c_ct2ort_x", C4},
    {"c_ort2ct_x", C4}, {"c_sina", C2},       {"c_cosa", C2},       {"c_dy", C2},
    {"c_dx", C2},       {"d_gco", D4},        {"d_gct", D4},        {"d_ct2ort_y", D4},
    {"d_ort2ct_y", D4}, {"d_sina", D2},       {"d_cosa", D2},       {"d_dx", D2},
    {"d_dy", D2},
};
constexpr int kNumFields = sizeof(kFields) / sizeof(kFields[0]);

const FieldDef* find_field(const char* name) {
  if (!name) return nullptr;
  for (const auto& f : kFields)
    if (std::strcmp(f.name, name) == 0) return &f;
  return nullptr;
}

int ncomp(Kind k) {
  switch (k) {
    case A3:
    case B3: return 2;
    case A4:
    case C4:
    case D4: return 4;
    default: return 1;
  }
}

const M2& pick(const ldg_grid::Mats& m, const char* name) {
  const char* s = std::strchr(name, '_') + 1;  // strip "a_", "c_", "d_"
  if (!std::strcmp(s, "gco")) return m.g_co;
  if (!std::strcmp(s, "gct")) return m.g_ctr;
  if (!std::strcmp(s, "c2l")) return m.c2l;
  if (!std::strcmp(s, "l2c")) return m.l2c;
  if (!std::strcmp(s, "ct2ort_x")) return m.ct2ort_x;
  if (!std::strcmp(s, "ort2ct_x")) return m.ort2ct_x;
  if (!std::strcmp(s, "ct2ort_y")) return m.ct2ort_y;
  return m.ort2ct_y;
}

// Value of a scalar float64 field at output point (Fortran i, j) of tile n,
// global_grid_base.F90:106-214.
double scalar_at(const ldg_grid& g, const char* name, int i, int j, int n) {
  const int ii = 2 * i, jj = 2 * j;
  if (!std::strcmp(name, "a_x")) return g.sx(g.ext_x, ii, jj);
  if (!std::strcmp(name, "a_y")) return g.sx(g.ext_y, ii, jj);
  if (!std::strcmp(name, "a_kik_x")) return g.sx(g.kik_x, ii, jj);
  if (!std::strcmp(name, "a_kik_y")) return g.sx(g.kik_y, ii, jj);
  if (!std::strcmp(name, "a_sina") || !std::strcmp(name, "a_cosa")) {
    double s, c;
    g.sincos_a(ii, jj, n, &s, &c);
    return name[2] == 's' ? s : c;
  }
  auto a_dx = [&]() { return g.sx(g.ext_dx, ii - 1, jj) + g.sx(g.ext_dx, ii, jj); };
  auto a_dy = [&]() { return g.sx(g.ext_dy, ii, jj - 1) + g.sx(g.ext_dy, ii, jj); };
  auto a_da = [&]() {
    return g.sx(g.ext_da, ii - 1, jj - 1) + g.sx(g.ext_da, ii - 1, jj) + g.sx(g.ext_da, ii, jj - 1) +
           g.sx(g.ext_da, ii, jj);
  };
  if (!std::strcmp(name, "a_dx")) return a_dx();
  if (!std::strcmp(name, "a_dy")) return a_dy();
  if (!std::strcmp(name, "a_da")) return a_da();
  if (!std::strcmp(name, "rda")) return 1.0 / a_da();
  if (!std::strcmp(name, "rdx")) return 1.0 / a_dx();
  if (!std::strcmp(name, "rdy")) return 1.0 / a_dy();
  if (!std::strcmp(name, "a_f") || !std::strcmp(name, "ub") || !std::strcmp(name, "vb")) {
    const double alpha = 0.0, ubar = 1.0;
    double lo = g.lon(ii, jj, n), la = g.lat(ii, jj, n);
    if (name[0] == 'a')
      return 2. * kOmega * (-1. * std::cos(lo) * std::cos(la) * std::sin(alpha) + std::sin(la) * std::cos(alpha));
    double u0 = ubar * (std::cos(alpha) * std::cos(la) + std::sin(alpha) * std::cos(lo) * std::sin(la));
    double u1 = -ubar * std::sin(alpha) * std::sin(lo);
    ldg_grid::Mats m = g.mats(ii, jj, n);
    if (name[0] == 'u') return m.l2c.m[0][0] * u0 + m.l2c.m[0][1] * u1;
    return m.l2c.m[1][0] * u0 + m.l2c.m[1][1] * u1;
  }
  // C grid (west faces): super point (2i-1, 2j)
  if (!std::strcmp(name, "c_sina") || !std::strcmp(name, "c_cosa")) {
    double s, c;
    g.sincos_a(ii - 1, jj, n, &s, &c);
    return name[2] == 's' ? s : c;
  }
  if (!std::strcmp(name, "c_dy")) return g.sx(g.ext_dy, ii - 1, jj - 1) + g.sx(g.ext_dy, ii - 1, jj);
  if (!std::strcmp(name, "c_dx")) {
    if (i < g.isd + 1) return kNaN;  // not assigned by the reference (global_grid_base.F90:179-184)
    return g.sx(g.ext_dx, ii - 2, jj) + g.sx(g.ext_dx, ii - 1, jj);
  }
  // D grid (south faces): super point (2i, 2j-1)
  if (!std::strcmp(name, "d_sina") || !std::strcmp(name, "d_cosa")) {
    double s, c;
    g.sincos_a(ii, jj - 1, n, &s, &c);
    return name[2] == 's' ? s : c;
  }
  if (!std::strcmp(name, "d_dx")) return g.sx(g.ext_dx, ii - 1, jj - 1) + g.sx(g.ext_dx, ii, jj - 1);
  if (!std::strcmp(name, "d_dy")) {
    if (j < g.isd + 1) return kNaN;  // not assigned by the reference (global_grid_base.F90:186-191)
    return g.sx(g.ext_dy, ii, jj - 2) + g.sx(g.ext_dy, ii, jj - 1);
  }
  return kNaN;
}

}  // namespace

extern "C" {

int ldg_create(int res, ldg_grid** out) {
  if (!out) return fail(LDG_EINVAL, "ldg_create: out is NULL");
  *out = nullptr;
  if (res < 6) return fail(LDG_EINVAL, "ldg_create: res must be >= 6 (equal-edge ghost line needs 7 points)");
  if (res > 4096) return fail(LDG_EINVAL, "ldg_create: res must be <= 4096");
  ldg_grid* g = new (std::nothrow) ldg_grid;
  if (!g) return fail(LDG_ENOMEM, "ldg_create: out of memory");
  try {
    g->res = res;
    g->s_lo = 1 - 2 * kNg;
    g->s_hi = 2 * res + 1 + 2 * kNg;
    g->sw = g->s_hi - g->s_lo + 1;
    g->a_lo = 1 - kNg;
    g->a_hi = res + kNg;
    g->aw = g->a_hi - g->a_lo + 1;
    g->isd = -2;
    g->ied = res + 3;
    g->M = res + 6;
    size_t s2 = (size_t)g->sw * g->sw;
    g->pt_ext.assign(s2 * 6 * 2, kNaN);
    g->pt_kik.assign(s2 * 6 * 2, kNaN);
    for (auto* v : {&g->ext_x, &g->ext_y, &g->kik_x, &g->kik_y, &g->ext_dx, &g->ext_dy, &g->ext_da})
      v->assign(s2, kNaN);
    g->k2e_loc.assign((size_t)g->aw * g->aw, -999);
    g->k2e_coef.assign((size_t)g->aw * g->aw * 2, -999.);
    gen_lonlat(*g);
    gen_coords(*g);
    gen_ds(*g);
    gen_da(*g);
    gen_k2e(*g);
  } catch (const std::bad_alloc&) {
    delete g;
    return fail(LDG_ENOMEM, "ldg_create: out of memory");
  }
  *out = g;
  return LDG_OK;
}

void ldg_destroy(ldg_grid* g) { delete g; }

int ldg_num_fields(void) { return kNumFields; }

const char* ldg_field_name(int i) {
  if (i < 0 || i >= kNumFields) return nullptr;
  return kFields[i].name;
}

int ldg_field_is_int(const char* name) {
  const FieldDef* f = find_field(name);
  return f && f->kind == AI;
}

int ldg_field_shape(const ldg_grid* g, const char* name, int* ndim, long* shape) {
  if (!g || !ndim || !shape) return fail(LDG_EINVAL, "ldg_field_shape: NULL argument");
  const FieldDef* f = find_field(name);
  if (!f) return fail(LDG_ENOFIELD, std::string("ldg_field_shape: unknown field ") + (name ? name : "(null)"));
  shape[0] = 6;
  shape[1] = g->M;
  shape[2] = g->M;
  int nd = 3;
  int nc = ncomp(f->kind);
  if (nc == 2) shape[nd++] = 2;
  if (nc == 4) {
    shape[nd++] = 2;
    shape[nd++] = 2;
  }
  *ndim = nd;
  return LDG_OK;
}

int ldg_get_f64(const ldg_grid* g, const char* name, double* out) {
  if (!g || !out) return fail(LDG_EINVAL, "ldg_get_f64: NULL argument");
  const FieldDef* f = find_field(name);
  if (!f) return fail(LDG_ENOFIELD, std::string("ldg_get_f64: unknown field ") + (name ? name : "(null)"));
  if (f->kind == AI) return fail(LDG_EINVAL, std::string("ldg_get_f64: ") + name + " is an int32 field");
  const int M = g->M, nc = ncomp(f->kind);
  for (int n = 1; n <= 6; ++n)
    for (int pi = 0; pi < M; ++pi)
      for (int pj = 0; pj < M; ++pj) {
        const int i = pi + g->isd, j = pj + g->isd;
        double* o = out + (((size_t)(n - 1) * M + pi) * M + pj) * nc;
        switch (f->kind) {
          case A3:
            if (!std::strcmp(name, "a_pt")) {
              size_t p = g->pidx(2 * i, 2 * j, n);
              o[0] = g->pt_ext[p];
              o[1] = g->pt_ext[p + 1];
            } else {  // k2e_coef
              size_t a = g->aidx(i, j) * 2;
              o[0] = g->k2e_coef[a];
              o[1] = g->k2e_coef[a + 1];
            }
            break;
          case B3: {
            size_t p = g->pidx(2 * i - 1, 2 * j - 1, n);
            o[0] = g->pt_ext[p];
            o[1] = g->pt_ext[p + 1];
            break;
          }
          case A4:
          case C4:
          case D4: {
            int si = 2 * i, sj = 2 * j;
            if (f->kind == C4) si -= 1;
            if (f->kind == D4) sj -= 1;
            ldg_grid::Mats m = g->mats(si, sj, n);
            const M2& r = pick(m, name);
            o[0] = r.m[0][0];
            o[1] = r.m[0][1];
            o[2] = r.m[1][0];
            o[3] = r.m[1][1];
            break;
          }
          default:
            o[0] = scalar_at(*g, name, i, j, n);
        }
      }
  return LDG_OK;
}

int ldg_get_i32(const ldg_grid* g, const char* name, int* out) {
  if (!g || !out) return fail(LDG_EINVAL, "ldg_get_i32: NULL argument");
  const FieldDef* f = find_field(name);
  if (!f || f->kind != AI)
    return fail(LDG_ENOFIELD, std::string("ldg_get_i32: not an int32 field: ") + (name ? name : "(null)"));
  // k2e_loc_i = k2e_loc - isd, k2e_loc_j = k2e_loc - jsd (chtholly_get_global_grid.F90:146-157)
  const int shift = !std::strcmp(name, "k2e_loc") ? 0 : -g->isd;
  const int M = g->M;
  for (int n = 1; n <= 6; ++n)
    for (int pi = 0; pi < M; ++pi)
      for (int pj = 0; pj < M; ++pj) {
        const int i = pi + g->isd, j = pj + g->isd;
        out[((size_t)(n - 1) * M + pi) * M + pj] = g->k2e_loc[g->aidx(i, j)] + shift;
      }
  return LDG_OK;
}

const char* ldg_last_error(void) { return g_err.c_str(); }

}  // extern "C"
