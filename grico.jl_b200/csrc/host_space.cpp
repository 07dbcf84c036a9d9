// Native host compile of an hp space on a dyadically refined Cartesian grid.
//
// This is the product's replacement for the host setup that Grico.jl performs in Julia
// before the matrix-free runtime runs: Morton ordering of the active leaves
// (topology.jl:250-268, 451-463), boundary/interface enumeration (topology.jl:1502-1545),
// and the continuity algebra that turns leaf-local modes into sparse expansions in global
// scalar dofs (continuity.jl phases 1-6, :153-1227).  DOF numbering, hanging-node
// coefficients and mode tables follow the reference exactly: boundary dofs are numbered by
// the smallest provisional variable of each merged class (union-find with the smaller root
// kept, continuity.jl:1053-1065), free roots before interior modes, interior modes leaf by
// leaf in Morton order (continuity.jl:264-350, 934-945).
//
// Unlike the reference, leaves are addressed through flat arrays (no per-leaf dictionaries)
// and face partners are found through a hash of face lower corners, so a 64^3 grid with
// p = 4 (25.7 M provisional variables) compiles in seconds.

#include "grico_host.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <set>
#include <unordered_set>
#include <vector>

namespace grico {

thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

namespace {

constexpr int kMaxDim = 3;

// ---------------------------------------------------------------------------
// 1-D numerics (polynomials.jl:294-434, quadrature.jl:342-410)
// ---------------------------------------------------------------------------

void legendre_vd(double x, int n, double* v, double* d) {
  v[0] = 1.0;
  d[0] = 0.0;
  if (n >= 1) { v[1] = x; d[1] = 1.0; }
  for (int k = 2; k <= n; ++k) {
    double inv_k = 1.0 / double(k);
    double first = double(2 * k - 1) * inv_k;
    double second = double(k - 1) * inv_k;
    v[k] = first * x * v[k - 1] - second * v[k - 2];
    d[k] = first * (v[k - 1] + x * d[k - 1]) - second * d[k - 2];
  }
}

}  // namespace

void fe_basis(double x, int p, double* v, double* d) {
  if (p == 0) { v[0] = 1.0; if (d) d[0] = 0.0; return; }
  double leg[64];
  leg[0] = 1.0;
  leg[1] = x;
  for (int k = 2; k <= p; ++k) {
    double inv_k = 1.0 / double(k);
    leg[k] = double(2 * k - 1) * inv_k * x * leg[k - 1] - double(k - 1) * inv_k * leg[k - 2];
  }
  if (d) {
    for (int k = p; k >= 2; --k) d[k] = std::sqrt(double(2 * k - 1) / 2.0) * leg[k - 1];
    d[0] = -0.5;
    d[1] = 0.5;
  }
  for (int k = p; k >= 2; --k) v[k] = (leg[k] - leg[k - 2]) / std::sqrt(double(4 * k - 2));
  v[0] = 0.5 * (1.0 - x);
  v[1] = 0.5 * (1.0 + x);
}

void gauss_legendre(int count, double* pts, double* wts) {
  const double tol = 1.0e3 * 2.220446049250313e-16;
  std::vector<double> v(count + 1), d(count + 1);
  int half = (count + 1) / 2;
  for (int i = 1; i <= half; ++i) {
    double x = std::cos(M_PI * (double(i) - 0.25) / (double(count) + 0.5));
    bool ok = false;
    for (int it = 0; it < 32; ++it) {
      legendre_vd(x, count, v.data(), d.data());
      double delta = v[count] / d[count];
      x -= delta;
      if (std::fabs(delta) <= tol) {
        legendre_vd(x, count, v.data(), d.data());
        ok = true;
        break;
      }
    }
    if (!ok) throw std::runtime_error("Gauss-Legendre root did not converge");
    double w = 2.0 / ((1.0 - x * x) * d[count] * d[count]);
    pts[i - 1] = -x;
    wts[i - 1] = w;
    pts[count - i] = x;
    wts[count - i] = w;
  }
}

namespace {

// Small dense LU with partial pivoting (unblocked; same pivot rule as LAPACK getf2).
void lu_solve_inplace(int n, std::vector<double>& a, std::vector<double>& b, int nrhs) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::fabs(a[k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = std::fabs(a[i * n + k]);
      if (v > best) { best = v; p = i; }
    }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(a[k * n + j], a[p * n + j]);
    double inv = 1.0 / a[k * n + k];
    for (int i = k + 1; i < n; ++i) a[i * n + k] *= inv;
    for (int i = k + 1; i < n; ++i)
      for (int j = k + 1; j < n; ++j) a[i * n + j] -= a[i * n + k] * a[k * n + j];
  }
  for (int k = 0; k < n; ++k)
    if (piv[k] != k)
      for (int j = 0; j < nrhs; ++j) std::swap(b[k * nrhs + j], b[piv[k] * nrhs + j]);
  // column-oriented substitutions in the order of the reference BLAS dtrsm used by getrs:
  // forward with unit L (k ascending), backward with U (k descending, divide before use)
  for (int j = 0; j < nrhs; ++j) {
    for (int k = 0; k < n; ++k) {
      const double bk = b[k * nrhs + j];
      if (bk != 0.0)
        for (int i = k + 1; i < n; ++i) b[i * nrhs + j] -= bk * a[i * n + k];
    }
    for (int k = n - 1; k >= 0; --k) {
      if (b[k * nrhs + j] != 0.0) {
        b[k * nrhs + j] /= a[k * n + k];
        const double bk = b[k * nrhs + j];
        for (int i = 0; i < k; ++i) b[i * nrhs + j] -= bk * a[i * n + k];
      }
    }
  }
}

}  // namespace

// Restriction of a source 1-D basis on an interval to a target basis on a dyadic subinterval
// (continuity.jl:1158-1198).  Returns a (target_degree+1) x (source_degree+1) row-major matrix.
std::vector<double> affine_restriction_matrix(int src_deg, int tgt_deg, int delta, long long rel) {
  if (delta == 0) {
    // Same interval: the hierarchical family is nested (psi_0..psi_p are shared by every degree
    // >= p), so the collocation solve reproduces the identity embedding; state it exactly.
    std::vector<double> e((tgt_deg + 1) * (src_deg + 1), 0.0);
    for (int i = 0; i <= src_deg && i <= tgt_deg; ++i) e[i * (src_deg + 1) + i] = 1.0;
    return e;
  }
  double scale = std::ldexp(1.0, -delta);
  double shift = delta == 0 ? 0.0 : scale * (2.0 * double(rel) + 1.0) - 1.0;
  int n = tgt_deg + 1;
  std::vector<double> pts(n), wts(n);
  gauss_legendre(n, pts.data(), wts.data());
  std::vector<double> a(n * n), b(n * (src_deg + 1));
  std::vector<double> v(n + 1), sv(src_deg + 2);
  for (int i = 0; i < n; ++i) {
    fe_basis(pts[i], tgt_deg, v.data(), nullptr);
    for (int j = 0; j < n; ++j) a[i * n + j] = v[j];
    fe_basis(scale * pts[i] + shift, src_deg, sv.data(), nullptr);
    for (int j = 0; j <= src_deg; ++j) b[i * (src_deg + 1) + j] = sv[j];
  }
  lu_solve_inplace(n, a, b, src_deg + 1);
  return b;
}

namespace {

// ---------------------------------------------------------------------------
// Mode patterns (basis.jl:150-330)
// ---------------------------------------------------------------------------

struct Pattern {
  int deg[kMaxDim];
  int shape[kMaxDim];
  int box;                         // prod(shape)
  std::vector<int> modes;          // active box indices in enumeration order
  std::vector<int> boundary_rank;  // box index -> rank among boundary modes, -1 otherwise
  std::vector<int> boundary_box;   // rank -> box index
  std::vector<int> face_rank[kMaxDim][2];  // ranks of boundary modes with m[a] == side
};

int mode_digit(int box_index, const int* shape, int a) {
  for (int b = 0; b < a; ++b) box_index /= shape[b];
  return box_index % shape[a];
}

Pattern make_pattern(int dim, const int* deg, int basis) {
  Pattern p;
  p.box = 1;
  int limit = 0;
  for (int a = 0; a < kMaxDim; ++a) {
    p.deg[a] = a < dim ? deg[a] : 0;
    p.shape[a] = p.deg[a] + 1;
    if (a < dim) { p.box *= p.shape[a]; limit = std::max(limit, p.deg[a]); }
  }
  p.boundary_rank.assign(p.box, -1);
  for (int i = 0; i < p.box; ++i) {
    int m[kMaxDim];
    int order = 0;
    bool boundary = false;
    for (int a = 0; a < dim; ++a) {
      m[a] = mode_digit(i, p.shape, a);
      order += m[a] <= 1 ? 0 : m[a];
      boundary |= m[a] <= 1;
    }
    if (basis == GRICO_BASIS_TRUNK && order > limit) continue;
    p.modes.push_back(i);
    if (boundary) {
      int r = int(p.boundary_box.size());
      p.boundary_rank[i] = r;
      p.boundary_box.push_back(i);
      for (int a = 0; a < dim; ++a)
        if (m[a] <= 1) p.face_rank[a][m[a]].push_back(r);
    }
  }
  return p;
}

struct Row {
  std::vector<int64_t> vars;
  std::vector<double> coefs;
  void add(int64_t v, double c) {
    for (size_t i = 0; i < vars.size(); ++i)
      if (vars[i] == v) { coefs[i] += c; return; }
    vars.push_back(v);
    coefs.push_back(c);
  }
  void remove_at(size_t i) {
    vars.erase(vars.begin() + i);
    coefs.erase(coefs.begin() + i);
  }
  void cleanup() {  // continuity.jl:681-700, 1213-1223
    double scale = 0.0;
    for (double c : coefs) scale = std::max(scale, std::fabs(c));
    double tol = 4.0 * 2.220446049250313e-16 * std::max(scale, 1.0);
    size_t i = 0;
    while (i < vars.size()) {
      if (std::fabs(coefs[i]) <= tol) remove_at(i); else ++i;
    }
  }
  void accumulate(const Row& src, double factor) {
    for (size_t i = 0; i < src.vars.size(); ++i) add(src.vars[i], factor * src.coefs[i]);
  }
};

int64_t uf_root(std::vector<int64_t>& parent, int64_t v) {
  int64_t r = v;
  while (parent[r] != r) r = parent[r];
  while (parent[v] != v) { int64_t n = parent[v]; parent[v] = r; v = n; }
  return r;
}

void uf_union(std::vector<int64_t>& parent, int64_t a, int64_t b) {
  int64_t ra = uf_root(parent, a), rb = uf_root(parent, b);
  if (ra == rb) return;
  if (ra < rb) parent[rb] = ra; else parent[ra] = rb;
}

struct KeyHash {
  size_t operator()(const std::array<int64_t, 4>& k) const {
    uint64_t h = 1469598103934665603ull;
    for (int64_t v : k) { h ^= uint64_t(v) + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2); }
    return size_t(h);
  }
};

}  // namespace

struct Space {
  int dim = 0;
  int basis = GRICO_BASIS_FULL;
  int continuity = GRICO_CONTINUITY_CG;
  int64_t nleaves = 0;
  int64_t root_counts[kMaxDim] = {1, 1, 1};
  int finest[kMaxDim] = {0, 0, 0};
  std::vector<int64_t> order;      // Morton position -> input leaf index
  std::vector<int> levels;         // [leaf(morton) * dim + a]
  std::vector<int64_t> coords;
  std::vector<int64_t> lower, upper;  // finest lattice
  std::vector<int> pattern_of;     // leaf -> pattern index
  std::vector<Pattern> patterns;
  std::vector<int> qshape;         // leaf * dim
  // faces
  std::vector<int64_t> bnd_leaf;
  std::vector<int> bnd_axis, bnd_side;
  std::vector<int64_t> if_minus, if_plus;
  std::vector<int> if_axis;
  // compiled terms: per leaf, per box mode: CSR (box modes absent from the active table have
  // an empty range)
  std::vector<int64_t> term_offsets;  // [nleaves * box_max + 1] addressed via leaf_box_offset
  std::vector<int64_t> leaf_box_offset;
  std::vector<int64_t> term_index;    // 0-based global dof
  std::vector<double> term_coef;
  int64_t ndofs = 0;
  double min_pivot = 1e300;  // smallest |pivot coefficient| met in the elimination
  int64_t noise_rows = 0;    // redundant continuity rows dropped at rounding-noise level
};

namespace {

void morton_sort(Space& s) {
  const int D = s.dim;
  int bit_count = 0;
  for (int a = 0; a < D; ++a) {
    int64_t value = (s.root_counts[a] << s.finest[a]) - 1;
    int bits = 0;
    while (value > 0) { ++bits; value >>= 1; }
    bit_count = std::max(bit_count, bits);
  }
  std::vector<int64_t> lower0(s.nleaves * D);
  for (int64_t l = 0; l < s.nleaves; ++l)
    for (int a = 0; a < D; ++a)
      lower0[l * D + a] = s.coords[l * D + a] << (s.finest[a] - s.levels[l * D + a]);
  s.order.resize(s.nleaves);
  for (int64_t l = 0; l < s.nleaves; ++l) s.order[l] = l;
  auto less = [&](int64_t x, int64_t y) {
    for (int bit = bit_count - 1; bit >= 0; --bit)
      for (int a = D - 1; a >= 0; --a) {
        int bx = int((lower0[x * D + a] >> bit) & 1), by = int((lower0[y * D + a] >> bit) & 1);
        if (bx != by) return bx < by;
      }
    for (int a = 0; a < D; ++a)
      if (s.levels[x * D + a] != s.levels[y * D + a]) return s.levels[x * D + a] < s.levels[y * D + a];
    return x < y;
  };
  std::sort(s.order.begin(), s.order.end(), less);
  std::vector<int> lev(s.nleaves * D);
  std::vector<int64_t> crd(s.nleaves * D);
  s.lower.resize(s.nleaves * D);
  s.upper.resize(s.nleaves * D);
  for (int64_t i = 0; i < s.nleaves; ++i) {
    int64_t l = s.order[i];
    for (int a = 0; a < D; ++a) {
      lev[i * D + a] = s.levels[l * D + a];
      crd[i * D + a] = s.coords[l * D + a];
      s.lower[i * D + a] = crd[i * D + a] << (s.finest[a] - lev[i * D + a]);
      s.upper[i * D + a] = (crd[i * D + a] + 1) << (s.finest[a] - lev[i * D + a]);
    }
  }
  s.levels.swap(lev);
  s.coords.swap(crd);
}

// Boundary faces and interfaces in the reference enumeration order (topology.jl:1502-1545):
// leaves in Morton order, axes ascending; boundary sides LOWER then UPPER; interface partners
// on the UPPER side sorted by their tangential lower corner (axis 1 first).
void enumerate_faces(Space& s) {
  const int D = s.dim;
  int64_t extent[kMaxDim];
  for (int a = 0; a < D; ++a) extent[a] = s.root_counts[a] << s.finest[a];
  // hash: (axis, lower corner) -> leaf
  std::unordered_map<std::array<int64_t, 4>, int64_t, KeyHash> by_lower;
  by_lower.reserve(size_t(s.nleaves) * 2);
  for (int64_t l = 0; l < s.nleaves; ++l) {
    std::array<int64_t, 4> k = {0, 0, 0, 0};
    for (int a = 0; a < D; ++a) k[a] = s.lower[l * D + a];
    by_lower[k] = l;
  }
  auto find_lower = [&](const int64_t* corner) -> int64_t {
    std::array<int64_t, 4> k = {0, 0, 0, 0};
    for (int a = 0; a < D; ++a) k[a] = corner[a];
    auto it = by_lower.find(k);
    return it == by_lower.end() ? -1 : it->second;
  };
  // Locate the leaf containing the finest-lattice cell at `p` by trying every coarser
  // dyadic alignment of p per axis (at most prod(levels) lookups; 1 in conforming meshes).
  auto containing = [&](const int64_t* p) -> int64_t {
    int maxlev[kMaxDim];
    for (int a = 0; a < D; ++a) maxlev[a] = s.finest[a];
    int sh[kMaxDim] = {0, 0, 0};
    while (true) {
      int64_t c[kMaxDim];
      for (int a = 0; a < D; ++a) c[a] = (p[a] >> sh[a]) << sh[a];
      int64_t l = find_lower(c);
      if (l >= 0) {
        bool ok = true;
        for (int a = 0; a < D; ++a) ok &= s.upper[l * D + a] > p[a];
        if (ok) return l;
      }
      int a = 0;
      while (a < D) {
        if (sh[a] < maxlev[a]) { ++sh[a]; break; }
        sh[a] = 0;
        ++a;
      }
      if (a == D) return -1;
    }
  };
  for (int64_t l = 0; l < s.nleaves; ++l)
    for (int a = 0; a < D; ++a)
      for (int side = 0; side < 2; ++side) {
        int64_t c = side == 0 ? s.lower[l * D + a] : s.upper[l * D + a];
        bool boundary = (c == 0 || c == extent[a]);
        if (!boundary) {
          int64_t p[kMaxDim];
          for (int b = 0; b < D; ++b) p[b] = s.lower[l * D + b];
          p[a] = side == 0 ? c - 1 : c;
          boundary = containing(p) < 0;
        }
        if (boundary) {
          s.bnd_leaf.push_back(l);
          s.bnd_axis.push_back(a);
          s.bnd_side.push_back(side);
        }
      }
  std::vector<int64_t> partners;
  for (int64_t l = 0; l < s.nleaves; ++l)
    for (int a = 0; a < D; ++a) {
      int64_t U = s.upper[l * D + a];
      if (U == extent[a]) continue;
      partners.clear();
      int64_t p[kMaxDim];
      for (int b = 0; b < D; ++b) p[b] = s.lower[l * D + b];
      p[a] = U;
      int64_t first = containing(p);
      bool covers = first >= 0 && s.lower[first * D + a] == U;
      for (int b = 0; covers && b < D; ++b)
        if (b != a) covers &= s.lower[first * D + b] <= s.lower[l * D + b] && s.upper[first * D + b] >= s.upper[l * D + b];
      if (covers) {
        partners.push_back(first);
      } else {
        // Finer partners, possibly with gaps (leaves removed from a physical domain): flood
        // the face from its lower corner, jumping across every leaf found and stepping one
        // finest-lattice unit across holes, so every leaf touching the face is reached.
        std::vector<std::array<int64_t, kMaxDim>> stack;
        std::unordered_set<int64_t> seen;
        std::set<std::array<int64_t, kMaxDim>> probed;
        std::array<int64_t, kMaxDim> c0 = {0, 0, 0};
        for (int b = 0; b < D; ++b) c0[b] = p[b];
        stack.push_back(c0);
        while (!stack.empty()) {
          auto c = stack.back();
          stack.pop_back();
          if (!probed.insert(c).second) continue;
          int64_t q = containing(c.data());
          if (q >= 0 && !seen.count(q)) {
            seen.insert(q);
            partners.push_back(q);
          }
          for (int b = 0; b < D; ++b) {
            if (b == a) continue;
            auto n = c;
            n[b] = q >= 0 ? s.upper[q * D + b] : c[b] + 1;
            if (n[b] < s.upper[l * D + b]) stack.push_back(n);
          }
        }
      }
      std::sort(partners.begin(), partners.end(), [&](int64_t x, int64_t y) {
        for (int b = 0; b < D; ++b) {
          if (b == a) continue;
          if (s.lower[x * D + b] != s.lower[y * D + b]) return s.lower[x * D + b] < s.lower[y * D + b];
        }
        return false;
      });
      for (int64_t q : partners) {
        s.if_minus.push_back(l);
        s.if_plus.push_back(q);
        s.if_axis.push_back(a);
      }
    }
}

struct RestrictionCache {
  std::unordered_map<uint64_t, std::vector<double>> cache;
  double coefficient(const Space& s, int axis, int64_t src_lo, int64_t src_hi, int64_t tgt_lo, int64_t tgt_hi,
                     int src_index, int src_deg, int tgt_deg, int tgt_index) {
    auto level_coord = [&](int64_t lo, int64_t hi, int& level, int64_t& coord) {
      int64_t len = hi - lo;
      int shift = 0;
      while ((int64_t(1) << shift) < len) ++shift;
      level = s.finest[axis] - shift;
      coord = lo >> shift;
    };
    int sl, tl;
    int64_t sc, tc;
    level_coord(src_lo, src_hi, sl, sc);
    level_coord(tgt_lo, tgt_hi, tl, tc);
    int delta = tl - sl;
    int64_t rel = tc - (sc << delta);
    uint64_t key = (uint64_t(src_deg) << 56) | (uint64_t(tgt_deg) << 48) | (uint64_t(delta) << 40) | uint64_t(rel);
    auto it = cache.find(key);
    if (it == cache.end()) it = cache.emplace(key, affine_restriction_matrix(src_deg, tgt_deg, delta, rel)).first;
    return it->second[tgt_index * (src_deg + 1) + src_index];
  }
};

void compile_continuity(Space& s) {
  const int D = s.dim;
  const int64_t L = s.nleaves;
  std::vector<int64_t> var_base(L + 1, 0);
  for (int64_t l = 0; l < L; ++l)
    var_base[l + 1] = var_base[l] + (s.continuity == GRICO_CONTINUITY_CG ? int64_t(s.patterns[s.pattern_of[l]].boundary_box.size()) : 0);
  const int64_t nvars = var_base[L];
  std::vector<std::vector<std::pair<int64_t, double>>> bterms_sparse;  // only for constrained roots
  std::vector<int64_t> roots;
  std::vector<int64_t> free_dof;   // per root variable: assigned dof or -1
  std::vector<char> is_pivot;
  std::unordered_map<int64_t, std::vector<std::pair<int64_t, double>>> pivot_terms;
  int64_t next_dof = 0;
  if (s.continuity == GRICO_CONTINUITY_CG && nvars > 0) {
    std::vector<int64_t> parent(nvars);
    for (int64_t v = 0; v < nvars; ++v) parent[v] = v;
    std::vector<size_t> constraint_faces;
    for (size_t f = 0; f < s.if_minus.size(); ++f) {
      int64_t a = s.if_minus[f], b = s.if_plus[f];
      int ax = s.if_axis[f];
      bool matching = true;
      for (int e = 0; e < D; ++e)
        if (e != ax) matching &= s.lower[a * D + e] == s.lower[b * D + e] && s.upper[a * D + e] == s.upper[b * D + e];
      const Pattern& pa = s.patterns[s.pattern_of[a]];
      const Pattern& pb = s.patterns[s.pattern_of[b]];
      bool same = matching && pa.face_rank[ax][1].size() == pb.face_rank[ax][0].size();
      if (same) {
        for (int r : pa.face_rank[ax][1]) {
          int box = pa.boundary_box[r];
          int m2 = 0, stride = 1;
          bool inside = true;
          for (int e = 0; e < D; ++e) {
            int m = mode_digit(box, pa.shape, e);
            if (e == ax) m = 0;
            if (m >= pb.shape[e]) inside = false;
            m2 += m * stride;
            stride *= pb.shape[e];
          }
          if (!inside || pb.boundary_rank[m2] < 0) { same = false; break; }
        }
      }
      if (!same) { constraint_faces.push_back(f); continue; }
      for (int r : pa.face_rank[ax][1]) {
        int box = pa.boundary_box[r];
        int m2 = 0, stride = 1;
        for (int e = 0; e < D; ++e) {
          int m = e == ax ? 0 : mode_digit(box, pa.shape, e);
          m2 += m * stride;
          stride *= pb.shape[e];
        }
        uf_union(parent, var_base[a] + r, var_base[b] + pb.boundary_rank[m2]);
      }
    }
    roots.resize(nvars);
    for (int64_t v = 0; v < nvars; ++v) roots[v] = uf_root(parent, v);
    // hanging / p-mismatch rows (continuity.jl:470-530)
    std::vector<Row> rows;
    RestrictionCache rc;
    for (size_t f : constraint_faces) {
      int64_t a = s.if_minus[f], b = s.if_plus[f];
      int ax = s.if_axis[f];
      const Pattern& pa = s.patterns[s.pattern_of[a]];
      const Pattern& pb = s.patterns[s.pattern_of[b]];
      int cdeg[kMaxDim] = {0, 0, 0}, cshape[kMaxDim] = {1, 1, 1};
      int64_t plo[kMaxDim], phi[kMaxDim];
      int ccount = 1;
      for (int e = 0; e < D; ++e) {
        cdeg[e] = e == ax ? 0 : std::max(pa.deg[e], pb.deg[e]);
        cshape[e] = cdeg[e] + 1;
        ccount *= cshape[e];
        plo[e] = e == ax ? s.upper[a * D + e] : std::max(s.lower[a * D + e], s.lower[b * D + e]);
        phi[e] = e == ax ? s.upper[a * D + e] : std::min(s.upper[a * D + e], s.upper[b * D + e]);
      }
      for (int cm = 0; cm < ccount; ++cm) {
        Row row;
        for (int sidx = 0; sidx < 2; ++sidx) {
          int64_t leaf = sidx == 0 ? a : b;
          const Pattern& pp = sidx == 0 ? pa : pb;
          double sign = sidx == 0 ? 1.0 : -1.0;
          for (int r : pp.face_rank[ax][sidx == 0 ? 1 : 0]) {
            int box = pp.boundary_box[r];
            double coef = 1.0;
            for (int e = 0; e < D; ++e) {
              if (e == ax) continue;
              coef *= rc.coefficient(s, e, s.lower[leaf * D + e], s.upper[leaf * D + e], plo[e], phi[e],
                                     mode_digit(box, pp.shape, e), pp.deg[e], cdeg[e], mode_digit(cm, cshape, e));
              if (coef == 0.0) break;
            }
            if (coef == 0.0) continue;
            row.add(roots[var_base[leaf] + r], sign * coef);
          }
        }
        row.cleanup();
        if (!row.vars.empty()) rows.push_back(std::move(row));
      }
    }

    is_pivot.assign(nvars, 0);
    std::vector<std::vector<int64_t>> orders;
    std::unordered_map<int64_t, Row> pivots;
    if (!rows.empty()) {
      std::unordered_map<int64_t, int64_t> cparent_map;
      auto cfind = [&](int64_t v) {
        auto it = cparent_map.find(v);
        if (it == cparent_map.end()) { cparent_map[v] = v; return v; }
        int64_t r = v;
        while (cparent_map[r] != r) r = cparent_map[r];
        int64_t x = v;
        while (cparent_map[x] != x) { int64_t n = cparent_map[x]; cparent_map[x] = r; x = n; }
        return r;
      };
      auto cunion = [&](int64_t x, int64_t y) {
        int64_t rx = cfind(x), ry = cfind(y);
        if (rx == ry) return;
        if (rx < ry) cparent_map[ry] = rx; else cparent_map[rx] = ry;
      };
      for (auto& row : rows)
        for (size_t i = 1; i < row.vars.size(); ++i) cunion(row.vars[0], row.vars[i]);
      std::map<int64_t, std::vector<size_t>> comps;
      for (size_t i = 0; i < rows.size(); ++i) comps[cfind(rows[i].vars[0])].push_back(i);
      for (auto& kv : comps) {
        std::unordered_map<int64_t, const Row*> local;
        std::vector<int64_t> order;
        for (size_t ri : kv.second) {
          Row& row = rows[ri];
          // largest magnitude that entered the row: the scale of its rounding noise
          double seen = 0.0;
          for (double c : row.coefs) seen = std::max(seen, std::fabs(c));
          while (true) {
            bool changed = false;
            for (size_t i = 0; i < row.vars.size(); ++i) {
              auto it = local.find(row.vars[i]);
              if (it == local.end()) continue;
              double factor = row.coefs[i];
              row.remove_at(i);
              for (double c : it->second->coefs) seen = std::max(seen, std::fabs(factor * c));
              row.accumulate(*it->second, factor);
              changed = true;
              break;
            }
            row.cleanup();
            if (!changed) break;
          }
          if (row.vars.empty()) continue;
          // A redundant row (its constraint already implied by earlier pivots) cancels to
          // rounding noise; the reference's cleanup (4 eps against max(scale, 1)) can keep such
          // a residue and would then eliminate a free variable.  Rows whose every remaining
          // coefficient is at noise level relative to what was summed into them are dropped.
          double left = 0.0;
          for (double c : row.coefs) left = std::max(left, std::fabs(c));
          if (left <= 256.0 * 2.220446049250313e-16 * seen) { ++s.noise_rows; continue; }
          // Pivot: the largest variable id (continuity.jl:995-998) among the terms whose
          // coefficient is at least kPivotFloor of the row's largest.  Restriction coefficients
          // of high modes onto half faces are ~2^-p; pivoting on one divides the row by it, and on
          // deep hp meshes such steps chain (the 3-D L-shape graded to level 7, degrees 2..7:
          // expansion coefficients up to 9.8e5 with the plain rule, 25 with the floor, and Jacobi
          // CG stalls on the former).  Where every coefficient is within the floor of the
          // largest, which covers the meshes the maps are pinned on, the choice is the
          // reference's.
          constexpr double kPivotFloor = 0.1;
          size_t pidx = row.vars.size();
          for (size_t i = 0; i < row.vars.size(); ++i)
            if (std::fabs(row.coefs[i]) >= kPivotFloor * left &&
                (pidx == row.vars.size() || row.vars[i] > row.vars[pidx]))
              pidx = i;
          int64_t pivot = row.vars[pidx];
          double pcoef = row.coefs[pidx];
          row.remove_at(pidx);
          double scale = -(1.0 / pcoef);
          Row expr;
          expr.accumulate(row, scale);
          expr.cleanup();
          auto& stored = pivots[pivot];
          stored = std::move(expr);
          local[pivot] = &stored;
          is_pivot[pivot] = 1;
          order.push_back(pivot);
          s.min_pivot = std::min(s.min_pivot, std::fabs(pcoef));
        }
        orders.push_back(std::move(order));
      }
    }
    free_dof.assign(nvars, -1);
    for (int64_t v = 0; v < nvars; ++v)
      if (roots[v] == v && !is_pivot[v]) free_dof[v] = next_dof++;
    for (auto& order : orders)
      for (auto it = order.rbegin(); it != order.rend(); ++it) {
        const Row& expr = pivots[*it];
        Row acc;
        for (size_t i = 0; i < expr.vars.size(); ++i) {
          int64_t v = expr.vars[i];
          double factor = expr.coefs[i];
          if (factor == 0.0) continue;
          if (free_dof[v] >= 0) {
            acc.add(free_dof[v], factor * 1.0);
          } else {
            auto pt = pivot_terms.find(v);
            if (pt == pivot_terms.end()) continue;  // constrained to zero
            for (auto& t : pt->second) acc.add(t.first, factor * t.second);
          }
        }
        acc.cleanup();
        std::vector<std::pair<int64_t, double>> terms;
        for (size_t i = 0; i < acc.vars.size(); ++i) terms.emplace_back(acc.vars[i], acc.coefs[i]);
        std::sort(terms.begin(), terms.end(), [](auto& x, auto& y) { return x.first < y.first; });
        pivot_terms[*it] = std::move(terms);
      }
  }
  // phase 6: per leaf, per box mode term lists
  int box_max = 0;
  for (auto& p : s.patterns) box_max = std::max(box_max, p.box);
  s.leaf_box_offset.resize(L + 1);
  s.leaf_box_offset[0] = 0;
  for (int64_t l = 0; l < L; ++l) s.leaf_box_offset[l + 1] = s.leaf_box_offset[l] + s.patterns[s.pattern_of[l]].box;
  s.term_offsets.assign(s.leaf_box_offset[L] + 1, 0);
  s.term_index.clear();
  s.term_coef.clear();
  s.term_index.reserve(s.leaf_box_offset[L]);
  s.term_coef.reserve(s.leaf_box_offset[L]);
  std::vector<int64_t> counts(s.leaf_box_offset[L], 0);
  // First pass writes terms in leaf/mode order; interior dofs are numbered as encountered.
  std::vector<std::vector<std::pair<int64_t, double>>> dummy;
  std::vector<int64_t> tmp_index;
  std::vector<double> tmp_coef;
  std::vector<int64_t> entry_start(s.leaf_box_offset[L], -1), entry_len(s.leaf_box_offset[L], 0);
  for (int64_t l = 0; l < L; ++l) {
    const Pattern& p = s.patterns[s.pattern_of[l]];
    for (int box : p.modes) {
      int64_t e = s.leaf_box_offset[l] + box;
      int r = s.continuity == GRICO_CONTINUITY_CG ? p.boundary_rank[box] : -1;
      entry_start[e] = int64_t(tmp_index.size());
      if (r >= 0) {
        int64_t v = var_base[l] + r;
        int64_t root = roots[v];
        if (free_dof[root] >= 0) {
          tmp_index.push_back(free_dof[root]);
          tmp_coef.push_back(1.0);
        } else {
          auto pt = pivot_terms.find(root);
          if (pt != pivot_terms.end())
            for (auto& t : pt->second)
              if (t.second != 0.0) { tmp_index.push_back(t.first); tmp_coef.push_back(t.second); }
        }
      } else {
        tmp_index.push_back(next_dof++);
        tmp_coef.push_back(1.0);
      }
      entry_len[e] = int64_t(tmp_index.size()) - entry_start[e];
    }
  }
  for (int64_t e = 0; e < s.leaf_box_offset[L]; ++e) s.term_offsets[e + 1] = s.term_offsets[e] + entry_len[e];
  s.term_index.resize(s.term_offsets.back());
  s.term_coef.resize(s.term_offsets.back());
  for (int64_t e = 0; e < s.leaf_box_offset[L]; ++e)
    for (int64_t k = 0; k < entry_len[e]; ++k) {
      s.term_index[s.term_offsets[e] + k] = tmp_index[entry_start[e] + k];
      s.term_coef[s.term_offsets[e] + k] = tmp_coef[entry_start[e] + k];
    }
  s.ndofs = next_dof;
}

}  // namespace
}  // namespace grico

using grico::Space;

extern "C" {

const char* grico_last_error(void) { return grico::g_last_error.c_str(); }

int grico_space_build(int dim, const int64_t* root_counts, int64_t nleaves, const int32_t* leaf_levels,
                      const int64_t* leaf_coords, const int32_t* leaf_degrees, int basis, int continuity,
                      int quadrature_extra, GricoSpace** out) {
  try {
    if (!out || dim < 1 || dim > 3 || nleaves < 1) { grico::set_error("grico_space_build: invalid arguments"); return GRICO_ERR_INVALID; }
    auto* s = new Space();
    s->dim = dim;
    s->basis = basis;
    s->continuity = continuity;
    s->nleaves = nleaves;
    for (int a = 0; a < dim; ++a) s->root_counts[a] = root_counts[a];
    s->levels.assign(leaf_levels, leaf_levels + nleaves * dim);
    s->coords.assign(leaf_coords, leaf_coords + nleaves * dim);
    for (int a = 0; a < dim; ++a) {
      s->finest[a] = 0;
      for (int64_t l = 0; l < nleaves; ++l) s->finest[a] = std::max(s->finest[a], s->levels[l * dim + a]);
    }
    grico::morton_sort(*s);
    // degrees follow the Morton permutation
    std::unordered_map<uint64_t, int> pattern_index;
    s->pattern_of.resize(nleaves);
    s->qshape.resize(nleaves * dim);
    for (int64_t i = 0; i < nleaves; ++i) {
      int64_t l = s->order[i];
      int deg[3] = {0, 0, 0};
      uint64_t key = 0;
      for (int a = 0; a < dim; ++a) {
        deg[a] = leaf_degrees[l * dim + a];
        if (deg[a] < 0 || deg[a] > 15) { delete s; grico::set_error("degree out of range 0..15"); return GRICO_ERR_INVALID; }
        if (continuity == GRICO_CONTINUITY_CG && deg[a] == 0) { delete s; grico::set_error("degree must be at least 1 on :cg axes"); return GRICO_ERR_INVALID; }
        key = key * 16 + uint64_t(deg[a]);
        s->qshape[i * dim + a] = std::max(deg[a] + quadrature_extra, 1);
      }
      auto it = pattern_index.find(key);
      if (it == pattern_index.end()) {
        it = pattern_index.emplace(key, int(s->patterns.size())).first;
        s->patterns.push_back(grico::make_pattern(dim, deg, basis));
      }
      s->pattern_of[i] = it->second;
    }
    grico::enumerate_faces(*s);
    grico::compile_continuity(*s);
    *out = reinterpret_cast<GricoSpace*>(s);
    return GRICO_OK;
  } catch (const std::exception& e) {
    grico::set_error(std::string("grico_space_build: ") + e.what());
    return GRICO_ERR_INVALID;
  }
}

int grico_space_destroy(GricoSpace* space) {
  delete reinterpret_cast<Space*>(space);
  return GRICO_OK;
}

int grico_space_sizes(const GricoSpace* space, int64_t* ndofs, int64_t* nterms, int64_t* nboxes,
                      int64_t* nboundary, int64_t* ninterfaces) {
  auto* s = reinterpret_cast<const Space*>(space);
  if (!s) return GRICO_ERR_INVALID;
  if (ndofs) *ndofs = s->ndofs;
  if (nterms) *nterms = int64_t(s->term_index.size());
  if (nboxes) *nboxes = s->leaf_box_offset.back();
  if (nboundary) *nboundary = int64_t(s->bnd_leaf.size());
  if (ninterfaces) *ninterfaces = int64_t(s->if_minus.size());
  return GRICO_OK;
}

int grico_space_export(const GricoSpace* space, int64_t* morton_order, int64_t* leaf_box_offset,
                       int64_t* term_offsets, int64_t* term_index, double* term_coef, int32_t* qshape,
                       int64_t* bnd_leaf, int32_t* bnd_axis, int32_t* bnd_side, int64_t* if_minus,
                       int64_t* if_plus, int32_t* if_axis) {
  auto* s = reinterpret_cast<const Space*>(space);
  if (!s) return GRICO_ERR_INVALID;
  auto cp = [](auto* dst, const auto& src) { if (dst) std::copy(src.begin(), src.end(), dst); };
  cp(morton_order, s->order);
  cp(leaf_box_offset, s->leaf_box_offset);
  cp(term_offsets, s->term_offsets);
  cp(term_index, s->term_index);
  cp(term_coef, s->term_coef);
  cp(qshape, s->qshape);
  cp(bnd_leaf, s->bnd_leaf);
  cp(bnd_axis, s->bnd_axis);
  cp(bnd_side, s->bnd_side);
  cp(if_minus, s->if_minus);
  cp(if_plus, s->if_plus);
  cp(if_axis, s->if_axis);
  return GRICO_OK;
}

int grico_gauss_legendre(int count, double* points, double* weights) {
  if (count < 1 || count > 64) return GRICO_ERR_INVALID;
  try { grico::gauss_legendre(count, points, weights); } catch (...) { return GRICO_ERR_INVALID; }
  return GRICO_OK;
}

int grico_fe_basis(double x, int degree, double* values, double* derivatives) {
  if (degree < 0 || degree > 60) return GRICO_ERR_INVALID;
  grico::fe_basis(x, degree, values, derivatives);
  return GRICO_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Multigrid transfer between two compiled spaces on the same grid (multigrid.jl:614-848).
//
// Every coarse leaf is either a leaf of the fine space (p-coarsening) or the parent of two fine
// leaves (one h-coarsening split).  Local entries are tensor products of 1-D restriction
// matrices (coarse degree -> fine degree on the child interval); the reduced transfer follows
// _append_field_reduced_transfer_entries!: coarse modes are expanded through the coarse term
// map and reduced map, accumulated per fine (leaf, mode), then mapped to the fine reduced dof of
// single-term fine modes with the inverse term coefficient.  Duplicate (coarse, fine) pairs
// must agree (multigrid.jl:837-848); the first value is kept.
struct Transfer {
  int64_t n_fine = 0, n_coarse = 0;
  std::vector<int64_t> row_off, col;
  std::vector<double> val;
};

namespace grico {
namespace {

struct LeafKey {
  std::array<int64_t, 6> k;
  bool operator==(const LeafKey& o) const { return k == o.k; }
};
struct LeafKeyHash {
  size_t operator()(const LeafKey& x) const {
    uint64_t h = 1469598103934665603ull;
    for (int64_t v : x.k) h ^= uint64_t(v) + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    return size_t(h);
  }
};

LeafKey leaf_key(const Space& s, int64_t leaf) {
  LeafKey key;
  key.k.fill(0);
  for (int a = 0; a < s.dim; ++a) {
    key.k[a] = s.levels[leaf * s.dim + a];
    key.k[3 + a] = s.coords[leaf * s.dim + a];
  }
  return key;
}

}  // namespace
}  // namespace grico

extern "C" int grico_transfer_build(const GricoSpace* coarse_space, const GricoSpace* fine_space,
                                    const int64_t* coarse_red_offsets, const int64_t* coarse_red_index,
                                    const double* coarse_red_coef, int64_t n_coarse_reduced,
                                    const int64_t* fine_reduced_index, int64_t n_fine_reduced,
                                    GricoTransfer** out) {
  using namespace grico;
  try {
    auto* C = reinterpret_cast<const Space*>(coarse_space);
    auto* F = reinterpret_cast<const Space*>(fine_space);
    if (!C || !F || !out || C->dim != F->dim) { set_error("grico_transfer_build: invalid arguments"); return GRICO_ERR_INVALID; }
    const int D = C->dim;
    std::unordered_map<LeafKey, int64_t, LeafKeyHash> fine_pos;
    fine_pos.reserve(size_t(F->nleaves) * 2);
    for (int64_t l = 0; l < F->nleaves; ++l) fine_pos[leaf_key(*F, l)] = l;
    std::unordered_map<uint64_t, std::vector<double>> mats;
    auto matrix = [&](int sdeg, int tdeg, int delta, int64_t rel) -> const std::vector<double>& {
      uint64_t key = (uint64_t(sdeg) << 56) | (uint64_t(tdeg) << 48) | (uint64_t(delta) << 40) | uint64_t(rel);
      auto it = mats.find(key);
      if (it == mats.end()) it = mats.emplace(key, affine_restriction_matrix(sdeg, tdeg, delta, rel)).first;
      return it->second;
    };
    // Every fine leaf lies under exactly one coarse leaf, so the target expansion of a fine
    // (leaf, mode) is complete once its coarse leaf has been processed.
    struct Triple { int64_t fine, coarse; double v; };
    std::vector<Triple> triples;
    std::vector<std::pair<int64_t, double>> source;
    std::vector<std::vector<std::pair<int64_t, double>>> local;
    std::vector<std::pair<int, double>> nz[3][17];
    std::vector<char> active;
    std::vector<int> touched;
    auto add_to = [](std::vector<std::pair<int64_t, double>>& v, int64_t k, double x) {
      if (x == 0.0) return;
      for (auto& t : v)
        if (t.first == k) { t.second += x; return; }
      v.emplace_back(k, x);
    };
    for (int64_t cl = 0; cl < C->nleaves; ++cl) {
      std::vector<int64_t> fines;
      auto same = fine_pos.find(leaf_key(*C, cl));
      if (same != fine_pos.end()) {
        fines.push_back(same->second);
      } else {
        for (int a = 0; a < D && fines.size() != 2; ++a) {
          fines.clear();
          for (int off = 0; off < 2; ++off) {
            LeafKey k = leaf_key(*C, cl);
            k.k[a] += 1;
            k.k[3 + a] = 2 * k.k[3 + a] + off;
            auto it = fine_pos.find(k);
            if (it != fine_pos.end()) fines.push_back(it->second);
          }
        }
        if (fines.size() != 2) {
          set_error("fine multigrid space does not contain the coarse leaf or its two children");
          return GRICO_ERR_INVALID;
        }
      }
      const Pattern& cp = C->patterns[C->pattern_of[cl]];
      for (int64_t fl : fines) {
        const Pattern& fp = F->patterns[F->pattern_of[fl]];
        const std::vector<double>* M[3] = {nullptr, nullptr, nullptr};
        for (int a = 0; a < D; ++a) {
          int delta = F->levels[fl * D + a] - C->levels[cl * D + a];
          int64_t rel = F->coords[fl * D + a] - (C->coords[cl * D + a] << delta);
          if (fp.deg[a] < cp.deg[a]) { set_error("fine multigrid level must represent every coarse mode exactly"); return GRICO_ERR_INVALID; }
          M[a] = &matrix(cp.deg[a], fp.deg[a], delta, rel);
        }
        // nonzero 1-D restriction entries per axis and coarse digit: (fine digit, value); entries
        // of O(eps) are rounding residues of exact zeros
        for (int a = 0; a < D; ++a)
          for (int c = 0; c <= cp.deg[a]; ++c) {
            nz[a][c].clear();
            for (int f = 0; f <= fp.deg[a]; ++f) {
              const double m = (*M[a])[f * (cp.deg[a] + 1) + c];
              if (std::fabs(m) > 4.0 * 2.220446049250313e-16) nz[a][c].emplace_back(f, m);
            }
          }
        if (int(local.size()) < fp.box) local.resize(size_t(fp.box));
        active.assign(size_t(fp.box), 0);
        for (int fbox : fp.modes) active[size_t(fbox)] = 1;
        touched.clear();
        for (int cbox : cp.modes) {
          int64_t ce = C->leaf_box_offset[cl] + cbox;
          if (C->term_offsets[ce] == C->term_offsets[ce + 1]) continue;
          source.clear();
          for (int64_t t = C->term_offsets[ce]; t < C->term_offsets[ce + 1]; ++t) {
            int64_t g = C->term_index[t];
            for (int64_t p = coarse_red_offsets[g]; p < coarse_red_offsets[g + 1]; ++p)
              add_to(source, coarse_red_index[p], C->term_coef[t] * coarse_red_coef[p]);
          }
          if (source.empty()) continue;
          int cm[3] = {0, 0, 0};
          for (int a = 0; a < D; ++a) cm[a] = mode_digit(cbox, cp.shape, a);
          static const std::vector<std::pair<int, double>> one{{0, 1.0}};
          const auto& n0 = nz[0][cm[0]];
          const auto& n1 = D > 1 ? nz[1][cm[1]] : one;
          const auto& n2 = D > 2 ? nz[2][cm[2]] : one;
          // fine modes in box order (axis 1 fastest), as the dense loop visited them
          for (const auto& e2 : n2)
            for (const auto& e1 : n1)
              for (const auto& e0 : n0) {
                const int fbox = e0.first + fp.shape[0] * (e1.first + (D > 1 ? fp.shape[1] : 1) * e2.first);
                if (!active[size_t(fbox)]) continue;
                double coef = e0.second;
                if (D > 1) coef *= e1.second;
                if (D > 2) coef *= e2.second;
                if (coef == 0.0) continue;
                if (!std::isfinite(coef)) { set_error("multigrid transfer coefficient must be finite"); return GRICO_ERR_INVALID; }
                auto& lf = local[size_t(fbox)];
                if (active[size_t(fbox)] == 1) {  // first contribution to this fine mode
                  active[size_t(fbox)] = 2;
                  touched.push_back(fbox);
                }
                for (auto& sp : source) add_to(lf, sp.first, coef * sp.second);
              }
        }
        std::sort(touched.begin(), touched.end());
        for (int fbox : touched) {
          if (local[fbox].empty()) continue;
          int64_t fe = F->leaf_box_offset[fl] + fbox;
          if (F->term_offsets[fe + 1] - F->term_offsets[fe] != 1) continue;
          int64_t t = F->term_offsets[fe];
          int64_t r = fine_reduced_index[F->term_index[t]];
          if (r < 0) continue;
          double inv = 1.0 / F->term_coef[t];
          for (auto& sp : local[fbox]) {
            double c = inv * sp.second;
            if (c != 0.0) triples.push_back({r, sp.first, c});
          }
        }
        for (int fbox : touched) local[size_t(fbox)].clear();
      }
    }
    // stable order by (fine, coarse): a counting sort by fine row keeps the emission order inside
    // each row, then a stable sort of each (short) row by coarse column
    {
      std::vector<int64_t> start(size_t(n_fine_reduced) + 1, 0);
      for (const Triple& t : triples) {
        if (t.fine < 0 || t.fine >= n_fine_reduced) { set_error("multigrid transfer row out of range"); return GRICO_ERR_INVALID; }
        ++start[size_t(t.fine) + 1];
      }
      for (int64_t r = 0; r < n_fine_reduced; ++r) start[size_t(r) + 1] += start[size_t(r)];
      std::vector<Triple> sorted(triples.size());
      std::vector<int64_t> fill(start.begin(), start.end() - 1);
      for (const Triple& t : triples) sorted[size_t(fill[size_t(t.fine)]++)] = t;
      for (int64_t r = 0; r < n_fine_reduced; ++r)
        std::stable_sort(sorted.begin() + start[size_t(r)], sorted.begin() + start[size_t(r) + 1],
                         [](const Triple& a, const Triple& b) { return a.coarse < b.coarse; });
      triples.swap(sorted);
    }
    std::vector<int64_t> row_count(n_fine_reduced, 0);
    std::vector<int64_t> cols;
    std::vector<double> vals;
    cols.reserve(triples.size());
    vals.reserve(triples.size());
    for (size_t i = 0; i < triples.size();) {
      size_t j = i + 1;
      while (j < triples.size() && triples[j].fine == triples[i].fine && triples[j].coarse == triples[i].coarse) {
        double a = triples[i].v, c = triples[j].v;
        double scale = std::max({1.0, std::fabs(a), std::fabs(c)});
        if (std::fabs(a - c) > 10000 * 2.220446049250313e-16 * scale) {
          set_error("inconsistent duplicate multigrid transfer entry");
          return GRICO_ERR_INVALID;
        }
        ++j;
      }
      cols.push_back(triples[i].coarse);
      vals.push_back(triples[i].v);
      row_count[triples[i].fine]++;
      i = j;
    }
    auto* T = new Transfer();
    T->n_fine = n_fine_reduced;
    T->n_coarse = n_coarse_reduced;
    T->row_off.assign(n_fine_reduced + 1, 0);
    for (int64_t r = 0; r < n_fine_reduced; ++r) T->row_off[r + 1] = T->row_off[r] + row_count[r];
    T->col.swap(cols);
    T->val.swap(vals);
    *out = reinterpret_cast<GricoTransfer*>(T);
    return GRICO_OK;
  } catch (const std::exception& e) {
    set_error(std::string("grico_transfer_build: ") + e.what());
    return GRICO_ERR_INVALID;
  }
}

extern "C" int grico_transfer_export(const GricoTransfer* transfer, int64_t* nnz, int64_t* row_offsets,
                                     int64_t* col_index, double* values) {
  auto* T = reinterpret_cast<const Transfer*>(transfer);
  if (!T) return GRICO_ERR_INVALID;
  if (nnz) *nnz = T->row_off.back();
  if (row_offsets) std::copy(T->row_off.begin(), T->row_off.end(), row_offsets);
  if (col_index) std::copy(T->col.begin(), T->col.end(), col_index);
  if (values) std::copy(T->val.begin(), T->val.end(), values);
  return GRICO_OK;
}

extern "C" int grico_transfer_destroy(GricoTransfer* transfer) {
  delete reinterpret_cast<Transfer*>(transfer);
  return GRICO_OK;
}
