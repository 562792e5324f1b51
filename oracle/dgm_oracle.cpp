// dgm_oracle.cpp -- CPU FP64 restatement of DGM_in_rust's DG residual + SSP-RK3 time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: it is loaded by
// tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and by nothing
// else.  The product (dgm_in_rust_b200/) never links, imports or calls it.
//
// Parity status: UNPINNED by reference outputs.  The reference is a Rust crate (Cargo, rayon,
// ndarray) that cannot be built in this environment (no rustc/cargo, no vendored crates) and it
// ships no tests, golden vectors or usable output (its only output file holds NaN).  This
// restatement is therefore checked against known answers derived from the mathematics
// (tests/test_oracle.py) and against the reference's own input fixture (airfoil.msh).
//
// Every function cites the reference file:line it restates.  The arithmetic is written in the
// same operation order as the reference so that, compiled with -ffp-contract=off, each scalar
// expression rounds like the Rust code does.  Three places can differ at the ulp level from the
// Rust binary: (a) rayon's fold/reduce summation order of the edge pass
// (src/spatial_disc.rs:167,210), which is run-dependent in the reference itself; (b) ndarray's
// 2-D .dot (matrixmultiply dgemm, possibly FMA) in src/spatial_disc/limiter/weno.rs:124,155,195
// and src/spatial_disc/boundary_condition.rs:67, restated here as plain sequential sums;
// (c) libm pow in HLLC (src/spatial_disc/flux.rs:77).
//
// Layout: states are the reference's Array<f64, Ix3> [element][variable][basis], C order.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int NEQ = 4;
constexpr double F64_EPSILON = 2.220446049250313e-16;  // f64::EPSILON (weno.rs:1)

enum Status {
  ORC_OK = 0,
  ORC_NEG_DENSITY = 1,   // flux.rs:56-57
  ORC_NEG_PRESSURE = 2,  // flux.rs:59-60
  ORC_TOO_MANY_BOUNDARY_EDGES = 4,  // weno.rs:107
  ORC_BAD_ARG = 7,
  ORC_PARSE = 8,
};

// Rust's f64::powi lowers to compiler-rt __powidf2 (square-and-multiply).
double powi(double a, int b) {
  double r = 1.0;
  while (true) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return r;
}

// ------------------------------------------------------------------------------------------
// Quadrature: src/gauss_point.rs:13-95.  Interval rules 3/4/5 and triangle rules 4/6 are the
// reference's tables; the 2-point interval rule and the 3- and 12-point triangle rules are
// extensions (the reference panics for them, gauss_point.rs:57,91) needed for p=1 and p=3.
// Triangle weights are normalised to sum 1 over the reference triangle, like the 6-point rule.
// ------------------------------------------------------------------------------------------
struct Gauss {
  int nq = 0, ng = 0;
  std::vector<double> cell_pts;   // [nq][2]
  std::vector<double> cell_w;     // [nq]
  std::vector<double> edge_pts;   // [3][ng][2]
  std::vector<double> edge_w;     // [ng]
};

bool interval_rule(int n, std::vector<double>& x, std::vector<double>& w) {
  switch (n) {
    case 2:
      x = {-0.5773502691896257, 0.5773502691896257};
      w = {1.0, 1.0};
      return true;
    case 3:
      x = {-0.7745966692414834, 0.0, 0.7745966692414834};
      w = {0.5555555555555556, 0.8888888888888889, 0.5555555555555556};
      return true;
    case 4:
      x = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
      w = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
      return true;
    case 5:
      x = {-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831, 0.9061798459386640};
      w = {0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665,
           0.2369268850561891};
      return true;
    default:
      return false;
  }
}

bool triangle_rule(int n, std::vector<double>& p, std::vector<double>& w) {
  switch (n) {
    case 3:  // degree-2 rule (extension)
      p = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
      w = {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0};
      return true;
    case 4:  // gauss_point.rs:63-69 (weights sum to 0.5 -- kept as the reference has it)
      p = {1.0 / 3.0, 1.0 / 3.0, 2.0 / 15.0, 11.0 / 15.0, 2.0 / 15.0, 2.0 / 15.0, 11.0 / 15.0,
           2.0 / 15.0};
      w = {-27.0 / 96.0, 25.0 / 96.0, 25.0 / 96.0, 25.0 / 96.0};
      return true;
    case 6:  // gauss_point.rs:71-89 (degree-4 rule, 14 significant digits as tabulated)
      p = {0.44594849091597, 0.44594849091597, 0.44594849091597, 0.10810301816807,
           0.10810301816807, 0.44594849091597, 0.09157621350977, 0.09157621350977,
           0.09157621350977, 0.81684757298046, 0.81684757298046, 0.09157621350977};
      w = {0.22338158967801, 0.22338158967801, 0.22338158967801,
           0.10995174365532, 0.10995174365532, 0.10995174365532};
      return true;
    case 12: {  // degree-6 Dunavant rule (extension)
      const double a = 0.063089014491502, wa = 0.050844906370207;
      const double b = 0.249286745170910, wb = 0.116786275726379;
      const double c = 0.053145049844817, d = 0.310352451033784, wc = 0.082851075618374;
      const double e = 1.0 - c - d;
      p = {a, a, 1.0 - 2.0 * a, a, a, 1.0 - 2.0 * a,
           b, b, 1.0 - 2.0 * b, b, b, 1.0 - 2.0 * b,
           c, d, d, c, c, e, e, c, d, e, e, d};
      w = {wa, wa, wa, wb, wb, wb, wc, wc, wc, wc, wc, wc};
      return true;
    }
    default:
      return false;
  }
}

// GaussPoints::new, gauss_point.rs:13-37: edge 0 -> ((x+1)/2, 0), edge 1 -> ((1-x)/2, (1+x)/2),
// edge 2 -> (0, (x_rev+1)/2) with the interval points reversed.
bool make_gauss(int nq, int ng, Gauss& g) {
  std::vector<double> x;
  if (!triangle_rule(nq, g.cell_pts, g.cell_w)) return false;
  if (!interval_rule(ng, x, g.edge_w)) return false;
  g.nq = nq;
  g.ng = ng;
  g.edge_pts.assign(3 * ng * 2, 0.0);
  for (int i = 0; i < ng; ++i) {
    g.edge_pts[(0 * ng + i) * 2 + 0] = (x[i] + 1.0) / 2.0;
    g.edge_pts[(0 * ng + i) * 2 + 1] = 0.0;
    g.edge_pts[(1 * ng + i) * 2 + 0] = (1.0 - x[i]) / 2.0;
    g.edge_pts[(1 * ng + i) * 2 + 1] = (1.0 + x[i]) / 2.0;
    g.edge_pts[(2 * ng + i) * 2 + 0] = 0.0;
    g.edge_pts[(2 * ng + i) * 2 + 1] = (x[ng - 1 - i] + 1.0) / 2.0;
  }
  return true;
}

// ------------------------------------------------------------------------------------------
// Dubiner basis: src/basis_function.rs:56-203.
// ------------------------------------------------------------------------------------------

// basis_function.rs:56-74
double jacobi_poly(int n, double alpha, double beta, double x) {
  if (n == 0) return 1.0;
  if (n == 1) return (alpha + 1.0) + (alpha + beta + 2.0) * (x - 1.0) / 2.0;
  const double nn = (double)n;
  const double a1 = 2.0 * nn * (nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0);
  const double a2 = 2.0 * nn + alpha + beta - 1.0;
  const double a3 = (2.0 * nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0) * x + alpha * alpha -
                    beta * beta;
  const double a4 = 2.0 * (nn + alpha - 1.0) * (nn + beta - 1.0) * (2.0 * nn + alpha + beta);
  const double pn_1 = jacobi_poly(n - 1, alpha, beta, x);
  const double pn_2 = jacobi_poly(n - 2, alpha, beta, x);
  return (a2 * a3 * pn_1 - a4 * pn_2) / a1;
}

// basis_function.rs:75-79
double dubiner_basis(int l, int k, double xi, double eta) {
  const double legendre = jacobi_poly(k, 0.0, 0.0, 2.0 * xi / (1.0 - eta) - 1.0);
  const double jacobi = jacobi_poly(l, 2.0 * (double)k + 1.0, 0.0, 2.0 * eta - 1.0);
  return powi(2.0, k) * legendre * powi(1.0 - eta, k) * jacobi;
}

// Mode ordering of compute_phi_cell (basis_function.rs:86-93): by total degree d, l = 0..d,
// k = d - l, i.e. (l,k) = (0,0),(0,1),(1,0),(0,2),(1,1),(2,0),(0,3),(1,2),(2,1),(3,0).
void mode_lk(int b, int& l, int& k) {
  int d = 0, start = 0;
  while (start + d + 1 <= b) {
    start += d + 1;
    ++d;
  }
  l = b - start;
  k = d - l;
}

// Derivative keys (a,b) = d^a/dx^a d^b/dy^b, index = l(l+1)/2 - 1 + b for order l = a+b:
// (1,0),(0,1),(2,0),(1,1),(0,2),(3,0),(2,1),(1,2),(0,3).
inline int key_index(int a, int b) {
  const int l = a + b;
  return l * (l + 1) / 2 - 1 + b;
}
inline int n_keys(int max_order) { return (max_order + 1) * (max_order + 2) / 2 - 1; }

// Bivariate polynomials in (xi, eta) up to degree 3, used only for the derivatives that the
// reference does not tabulate (modes 6..9 and third derivatives, p=3 extension).
struct Poly {
  double c[4][4] = {};  // c[i][j] * xi^i * eta^j
};
Poly pmul(const Poly& a, const Poly& b) {
  Poly r;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      if (a.c[i][j] != 0.0)
        for (int k = 0; i + k < 4; ++k)
          for (int m = 0; j + m < 4; ++m) r.c[i + k][j + m] += a.c[i][j] * b.c[k][m];
  return r;
}
Poly padd(const Poly& a, const Poly& b, double sa = 1.0, double sb = 1.0) {
  Poly r;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r.c[i][j] = sa * a.c[i][j] + sb * b.c[i][j];
  return r;
}
Poly pconst(double v) {
  Poly r;
  r.c[0][0] = v;
  return r;
}
// Jacobi polynomial P_n^{(alpha,0)}(2 eta - 1) as a polynomial in eta (same recursion as
// jacobi_poly, basis_function.rs:56-74, carried out on coefficients).
Poly jacobi_eta(int n, double alpha) {
  Poly y;  // 2 eta - 1
  y.c[0][0] = -1.0;
  y.c[0][1] = 2.0;
  Poly p0 = pconst(1.0);
  if (n == 0) return p0;
  Poly p1 = padd(pconst(alpha + 1.0), padd(y, pconst(-1.0)), 1.0, (alpha + 2.0) / 2.0);
  if (n == 1) return p1;
  Poly pm2 = p0, pm1 = p1;
  for (int m = 2; m <= n; ++m) {
    const double nn = m, beta = 0.0;
    const double a1 = 2.0 * nn * (nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0);
    const double a2 = 2.0 * nn + alpha + beta - 1.0;
    const double a3s = (2.0 * nn + alpha + beta) * (2.0 * nn + alpha + beta - 2.0);
    const double a3c = alpha * alpha - beta * beta;
    const double a4 = 2.0 * (nn + alpha - 1.0) * (nn + beta - 1.0) * (2.0 * nn + alpha + beta);
    Poly a3 = padd(y, pconst(a3c), a3s, 1.0);
    Poly cur = padd(pmul(a3, pm1), pm2, a2 / a1, -a4 / a1);
    pm2 = pm1;
    pm1 = cur;
  }
  return pm1;
}
Poly dubiner_poly(int l, int k) {
  // (1-eta)^k P_k(x) with x = (2 xi - 1 + eta)/(1 - eta): sum_m a_m (2xi-1+eta)^m (1-eta)^(k-m)
  static const double leg[4][4] = {
      {1.0, 0, 0, 0}, {0, 1.0, 0, 0}, {-0.5, 0, 1.5, 0}, {0, -1.5, 0, 2.5}};
  Poly s;  // 2 xi - 1 + eta
  s.c[0][0] = -1.0;
  s.c[1][0] = 2.0;
  s.c[0][1] = 1.0;
  Poly om;  // 1 - eta
  om.c[0][0] = 1.0;
  om.c[0][1] = -1.0;
  Poly q;
  for (int m = 0; m <= k; ++m) {
    if (leg[k][m] == 0.0) continue;
    Poly t = pconst(leg[k][m]);
    for (int r = 0; r < m; ++r) t = pmul(t, s);
    for (int r = 0; r < k - m; ++r) t = pmul(t, om);
    q = padd(q, t);
  }
  Poly r = pmul(q, jacobi_eta(l, 2.0 * k + 1.0));
  const double two_k = powi(2.0, k);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r.c[i][j] *= two_k;
  return r;
}
double poly_deriv_eval(const Poly& p, int da, int db, double xi, double eta) {
  double sum = 0.0;
  for (int i = da; i < 4; ++i)
    for (int j = db; j < 4; ++j) {
      if (p.c[i][j] == 0.0) continue;
      double f = p.c[i][j];
      for (int t = 0; t < da; ++t) f *= (double)(i - t);
      for (int t = 0; t < db; ++t) f *= (double)(j - t);
      sum += f * powi(xi, i - da) * powi(eta, j - db);
    }
  return sum;
}

// Reference-space derivative of mode b, key (a, c) = d^a/dxi^a d^c/deta^c, at (xi, eta).
// Modes 0..5 up to second order are the reference's closed forms (basis_function.rs:114-193);
// everything else comes from the polynomial expansion above.
double ref_deriv(int b, int a, int c, double xi, double eta) {
  const int order = a + c;
  if (b < 6 && order <= 2) {
    switch (b) {
      case 0:
        return 0.0;
      case 1:
        if (a == 1 && c == 0) return 4.0;
        if (a == 0 && c == 1) return 2.0;
        return 0.0;
      case 2:
        if (a == 0 && c == 1) return 3.0;
        return 0.0;
      case 3:
        if (a == 1 && c == 0) return 48.0 * xi + 24.0 * eta - 24.0;
        if (a == 0 && c == 1) return 24.0 * xi + 8.0 * eta - 8.0;
        if (a == 2) return 48.0;
        if (a == 1 && c == 1) return 24.0;
        return 8.0;
      case 4:
        if (a == 1 && c == 0) return 20.0 * eta - 4.0;
        if (a == 0 && c == 1) return 20.0 * xi + 20.0 * eta - 12.0;
        if (a == 2) return 0.0;
        if (a == 1 && c == 1) return 20.0;
        return 20.0;
      case 5:
        if (a == 1 && c == 0) return 0.0;
        if (a == 0 && c == 1) return 20.0 * eta - 8.0;
        if (a == 2) return 0.0;
        if (a == 1 && c == 1) return 0.0;
        return 20.0;
    }
  }
  int l, k;
  mode_lk(b, l, k);
  if (l + k < order) return 0.0;
  return poly_deriv_eval(dubiner_poly(l, k), a, c, xi, eta);
}

struct Basis {
  int p = 0, nb = 0, nkeys = 0, max_order = 0;
  std::vector<double> phi_cell;   // [nq][nb]          basis_function.rs:80-95
  std::vector<double> phi_edge;   // [3][ng][nb]       basis_function.rs:96-113
  std::vector<double> dphi_cell;  // [nq][nb][nkeys]   reference-space derivatives
  std::vector<double> dphi_edge;  // [3][ng][nb][2]    d/dxi, d/deta at the edge points (basis_function.rs:152-193)
  std::vector<double> mass;       // [nb]              basis_function.rs:194-203
};

void make_basis(int p, const Gauss& g, Basis& B) {
  B.p = p;
  B.nb = (p + 1) * (p + 2) / 2;
  B.max_order = std::max(p, 2);  // the reference always tabulates up to second order
  B.nkeys = n_keys(B.max_order);
  const int nb = B.nb, nq = g.nq, ng = g.ng;
  B.phi_cell.assign((size_t)nq * nb, 0.0);
  B.phi_edge.assign((size_t)3 * ng * nb, 0.0);
  B.dphi_cell.assign((size_t)nq * nb * B.nkeys, 0.0);
  B.mass.assign(nb, 0.0);
  for (int i = 0; i < nq; ++i) {
    const double xi = g.cell_pts[i * 2], eta = g.cell_pts[i * 2 + 1];
    for (int b = 0; b < nb; ++b) {
      int l, k;
      mode_lk(b, l, k);
      B.phi_cell[i * nb + b] = dubiner_basis(l, k, xi, eta);
    }
  }
  for (int e = 0; e < 3; ++e)
    for (int i = 0; i < ng; ++i) {
      const double xi = g.edge_pts[(e * ng + i) * 2], eta = g.edge_pts[(e * ng + i) * 2 + 1];
      for (int b = 0; b < nb; ++b) {
        int l, k;
        mode_lk(b, l, k);
        B.phi_edge[(e * ng + i) * nb + b] = dubiner_basis(l, k, xi, eta);
      }
    }
  for (int i = 0; i < nq; ++i) {
    const double xi = g.cell_pts[i * 2], eta = g.cell_pts[i * 2 + 1];
    for (int b = 0; b < nb; ++b)
      for (int o = 1; o <= B.max_order; ++o)
        for (int c = 0; c <= o; ++c) {
          const int a = o - c;
          B.dphi_cell[((size_t)i * nb + b) * B.nkeys + key_index(a, c)] = ref_deriv(b, a, c, xi, eta);
        }
  }
  // compute_dphi_edge, basis_function.rs:152-193 (first derivatives, the keys the viscous terms use)
  B.dphi_edge.assign((size_t)3 * ng * nb * 2, 0.0);
  for (int e = 0; e < 3; ++e)
    for (int i = 0; i < ng; ++i) {
      const double xi = g.edge_pts[(e * ng + i) * 2], eta = g.edge_pts[(e * ng + i) * 2 + 1];
      for (int b = 0; b < nb; ++b) {
        B.dphi_edge[(((size_t)e * ng + i) * nb + b) * 2 + 0] = ref_deriv(b, 1, 0, xi, eta);
        B.dphi_edge[(((size_t)e * ng + i) * nb + b) * 2 + 1] = ref_deriv(b, 0, 1, xi, eta);
      }
    }
  // compute_mass_mat, basis_function.rs:194-203
  for (int b = 0; b < nb; ++b)
    for (int i = 0; i < nq; ++i) {
      const double ph = B.phi_cell[i * nb + b];
      B.mass[b] += g.cell_w[i] * (ph * ph);
    }
}

// ------------------------------------------------------------------------------------------
// Mesh: src/mesh.rs:5-189, src/initialization.rs:112-261, src/io/mesh_parser.rs:28-158.
// ------------------------------------------------------------------------------------------
struct EdgeBlock {
  std::vector<int64_t> pairs;  // [n][2], 0-based node ids
  std::string name;
};
struct RawMesh {
  std::vector<double> xy;                  // [nv][2]
  std::vector<EdgeBlock> edge_blocks;
  std::vector<std::vector<int64_t>> tri_blocks;  // each [n][3], 0-based
};

enum BoundaryType { WALL = 0, FARFIELD = 1 };

struct Mesh {
  int64_t nv = 0, ne = 0, ned = 0, np = 0;
  std::vector<double> xy;
  // elements (mesh.rs:154-163)
  std::vector<int64_t> e_vert, e_edge, e_nbr;  // [ne][3]
  std::vector<double> e_jac, e_circ, e_hmin;   // [ne]
  std::vector<double> e_dinv;                  // [ne][4] dxi_dx, dxi_dy, deta_dx, deta_dy
  // edges (mesh.rs:164-173)
  std::vector<int64_t> d_elem, d_vert, d_icell;  // [ned][2]
  std::vector<double> d_jac, d_normal;           // [ned], [ned][2]
  std::vector<int64_t> d_patch;                  // [ned]
  // patches (mesh.rs:185-189)
  std::vector<int> p_type;
  std::vector<double> p_q;  // [np][4] rho, u, v, p
  std::vector<int64_t> internal_edges, internal_elements, boundary_elements;
};

std::vector<std::string> split_ws(const std::string& s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string t;
  while (is >> t) out.push_back(t);
  return out;
}

// GmshParser::parse, mesh_parser.rs:28-158 -- the same line state machine.
int parse_gmsh(const char* path, RawMesh& raw, std::string& err) {
  std::ifstream f(path);
  if (!f) {
    err = "Failed to open file";
    return ORC_PARSE;
  }
  enum St {
    StandingBy, PhysNames, FirstPhys, Entities, FirstEnt, Nodes, FirstNodes, FirstElems,
    EdgeBlocks, ElemBlocks, FirstBlocks
  } st = StandingBy;
  std::map<long, std::string> physical_names;
  std::map<long, long> ent_to_phys;
  long line_count = 0, max_line_count = 0;
  std::string line;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.rfind("$End", 0) == 0) { st = StandingBy; continue; }
    if (line.rfind("$PhysicalNames", 0) == 0) { st = FirstPhys; continue; }
    if (line.rfind("$Entities", 0) == 0) { st = FirstEnt; continue; }
    if (line.rfind("$Nodes", 0) == 0) { st = FirstNodes; continue; }
    if (line.rfind("$Elements", 0) == 0) { st = FirstElems; continue; }
    auto v = split_ws(line);
    switch (st) {
      case StandingBy: break;
      case FirstPhys: st = PhysNames; break;
      case PhysNames:
        if (v.size() == 3) {
          std::string name = v[2];
          while (!name.empty() && name.front() == '"') name.erase(name.begin());
          while (!name.empty() && name.back() == '"') name.pop_back();
          physical_names[std::stol(v[1])] = name;
        }
        break;
      case FirstEnt: st = Entities; break;
      case Entities:
        if (v.size() >= 11) ent_to_phys[std::stol(v[0])] = std::stol(v[8]);
        break;
      case FirstNodes:
        raw.xy.reserve(2 * std::stol(v[1]));
        st = Nodes;
        break;
      case Nodes:
        if (v.size() == 3) {
          raw.xy.push_back(std::stod(v[0]));
          raw.xy.push_back(std::stod(v[1]));
        }
        break;
      case FirstElems: st = FirstBlocks; break;
      case FirstBlocks: {
        const long dim = std::stol(v[0]);
        const long tag = std::stol(v[1]);
        const long num = std::stol(v[3]);
        auto it = ent_to_phys.find(tag);
        if (it == ent_to_phys.end() || !physical_names.count(it->second)) {
          err = "entity without physical name";
          return ORC_PARSE;
        }
        if (dim == 1) {
          raw.edge_blocks.push_back(EdgeBlock{{}, physical_names[it->second]});
          st = EdgeBlocks;
        }
        if (dim == 2) {
          raw.tri_blocks.emplace_back();
          st = ElemBlocks;
        }
        line_count = 0;
        max_line_count = num;
        break;
      }
      case EdgeBlocks:
        ++line_count;
        raw.edge_blocks.back().pairs.push_back(std::stol(v[1]) - 1);
        raw.edge_blocks.back().pairs.push_back(std::stol(v[2]) - 1);
        if (line_count == max_line_count) st = FirstBlocks;
        break;
      case ElemBlocks:
        ++line_count;
        raw.tri_blocks.back().push_back(std::stol(v[1]) - 1);
        raw.tri_blocks.back().push_back(std::stol(v[2]) - 1);
        raw.tri_blocks.back().push_back(std::stol(v[3]) - 1);
        if (line_count == max_line_count) st = FirstBlocks;
        break;
    }
  }
  return ORC_OK;
}

struct FreeStream {  // io/boundary_condition_parser.rs:4-12, io/initial_solution_parser.rs:4-10
  double aoa_deg, mach, rho, p;
};

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

struct PairHash {
  size_t operator()(const std::pair<int64_t, int64_t>& p) const {
    return std::hash<int64_t>()(p.first * 1000003 + p.second);
  }
};

// process_mesh, initialization.rs:112-261
int process_mesh(const RawMesh& raw, const FreeStream& fs, double hcr, Mesh& m, std::string& err) {
  m.xy = raw.xy;
  m.nv = (int64_t)raw.xy.size() / 2;
  std::unordered_map<std::pair<int64_t, int64_t>, int64_t, PairHash> edge_map;
  std::vector<int64_t> d_elem, d_vert, d_icell, d_patch;
  for (const auto& blk : raw.edge_blocks) {
    const std::string nm = lower(blk.name);
    int type;
    double q[4] = {0, 0, 0, 0};
    if (nm == "wall") {
      type = WALL;
    } else if (nm == "farfield") {
      type = FARFIELD;
      const double c = std::sqrt(hcr * fs.p / fs.rho);
      const double a = fs.aoa_deg * (M_PI / 180.0);  // f64::to_radians
      q[0] = fs.rho;
      q[1] = fs.mach * c * std::cos(a);
      q[2] = fs.mach * c * std::sin(a);
      q[3] = fs.p;
    } else {
      err = "Boundary type not implemented";
      return ORC_BAD_ARG;
    }
    const int64_t np = (int64_t)blk.pairs.size() / 2;
    for (int64_t i = 0; i < np; ++i) {
      const int64_t n1 = blk.pairs[2 * i], n2 = blk.pairs[2 * i + 1];
      d_vert.push_back(n1);
      d_vert.push_back(n2);
      d_elem.push_back(0);
      d_elem.push_back(-1);
      d_icell.push_back(0);
      d_icell.push_back(-1);
      d_patch.push_back((int64_t)m.p_type.size());
      edge_map[{n1, n2}] = (int64_t)d_patch.size() - 1;
    }
    m.p_type.push_back(type);
    for (int k = 0; k < 4; ++k) m.p_q.push_back(q[k]);
  }
  auto find_edge = [&](int64_t a, int64_t b) -> int64_t {
    auto it = edge_map.find({a, b});
    if (it != edge_map.end()) return it->second;
    it = edge_map.find({b, a});
    if (it != edge_map.end()) return it->second;
    return -1;
  };
  int64_t ne = 0;
  for (const auto& blk : raw.tri_blocks) {
    const int64_t nt = (int64_t)blk.size() / 3;
    for (int64_t t = 0; t < nt; ++t)
      for (int i = 0; i < 3; ++i) {
        const int64_t a = blk[3 * t + i], b = blk[3 * t + (i + 1) % 3];
        if (find_edge(a, b) < 0) {
          d_vert.push_back(a);
          d_vert.push_back(b);
          d_elem.push_back(0);
          d_elem.push_back(0);
          d_icell.push_back(0);
          d_icell.push_back(0);
          d_patch.push_back(-1);
          m.internal_edges.push_back((int64_t)d_patch.size() - 1);
          edge_map[{a, b}] = (int64_t)d_patch.size() - 1;
        }
      }
    for (int64_t t = 0; t < nt; ++t) {
      int64_t iv[3], ie[3];
      bool internal = true;
      for (int i = 0; i < 3; ++i) {
        iv[i] = blk[3 * t + i];
        ie[i] = find_edge(blk[3 * t + i], blk[3 * t + (i + 1) % 3]);
      }
      for (int k = 0; k < 3; ++k) {
        const int64_t ed = ie[k];
        if (d_elem[2 * ed + 1] == -1) {
          d_elem[2 * ed] = ne;
          d_icell[2 * ed] = k;
          internal = false;
        } else if (iv[k] == d_vert[2 * ed]) {
          d_elem[2 * ed] = ne;
          d_icell[2 * ed] = k;
        } else {
          d_elem[2 * ed + 1] = ne;
          d_icell[2 * ed + 1] = k;
        }
      }
      for (int k = 0; k < 3; ++k) {
        m.e_vert.push_back(iv[k]);
        m.e_edge.push_back(ie[k]);
        m.e_nbr.push_back(-1);
      }
      if (internal) m.internal_elements.push_back(ne);
      else m.boundary_elements.push_back(ne);
      ++ne;
    }
  }
  m.ne = ne;
  m.ned = (int64_t)d_patch.size();
  m.np = (int64_t)m.p_type.size();
  m.d_elem = d_elem;
  m.d_vert = d_vert;
  m.d_icell = d_icell;
  m.d_patch = d_patch;

  const auto X = [&](int64_t v) { return m.xy[2 * v]; };
  const auto Y = [&](int64_t v) { return m.xy[2 * v + 1]; };
  // compute_jacob_det, mesh.rs:25-42
  m.d_jac.assign(m.ned, 0.0);
  m.d_normal.assign(2 * m.ned, 0.0);
  for (int64_t d = 0; d < m.ned; ++d) {
    const double x1 = X(m.d_vert[2 * d]), x2 = X(m.d_vert[2 * d + 1]);
    const double y1 = Y(m.d_vert[2 * d]), y2 = Y(m.d_vert[2 * d + 1]);
    m.d_jac[d] = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
  }
  m.e_jac.assign(ne, 0.0);
  m.e_circ.assign(ne, 0.0);
  m.e_hmin.assign(ne, 0.0);
  m.e_dinv.assign(4 * ne, 0.0);
  for (int64_t e = 0; e < ne; ++e) {
    const double x1 = X(m.e_vert[3 * e]), x2 = X(m.e_vert[3 * e + 1]), x3 = X(m.e_vert[3 * e + 2]);
    const double y1 = Y(m.e_vert[3 * e]), y2 = Y(m.e_vert[3 * e + 1]), y3 = Y(m.e_vert[3 * e + 2]);
    m.e_jac[e] = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
  }
  // compute_normal, mesh.rs:15-24
  for (int64_t d = 0; d < m.ned; ++d) {
    const double x1 = X(m.d_vert[2 * d]), x2 = X(m.d_vert[2 * d + 1]);
    const double y1 = Y(m.d_vert[2 * d]), y2 = Y(m.d_vert[2 * d + 1]);
    m.d_normal[2 * d] = (y2 - y1) / m.d_jac[d];
    m.d_normal[2 * d + 1] = -(x2 - x1) / m.d_jac[d];
  }
  for (int64_t e = 0; e < ne; ++e) {
    const double x1 = X(m.e_vert[3 * e]), x2 = X(m.e_vert[3 * e + 1]), x3 = X(m.e_vert[3 * e + 2]);
    const double y1 = Y(m.e_vert[3 * e]), y2 = Y(m.e_vert[3 * e + 1]), y3 = Y(m.e_vert[3 * e + 2]);
    // compute_dphi inverse Jacobian, mesh.rs:93-100
    const double J = m.e_jac[e];
    m.e_dinv[4 * e + 0] = (y3 - y1) / J;
    m.e_dinv[4 * e + 1] = -(x3 - x1) / J;
    m.e_dinv[4 * e + 2] = -(y2 - y1) / J;
    m.e_dinv[4 * e + 3] = (x2 - x1) / J;
    // compute_circumradius, mesh.rs:43-57
    const double a = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    const double b = std::sqrt((x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2));
    const double c = std::sqrt((x1 - x3) * (x1 - x3) + (y1 - y3) * (y1 - y3));
    const double s = (a + b + c) / 2.0;
    m.e_circ[e] = a * b * c / (4.0 * std::sqrt(s * (s - a) * (s - b) * (s - c)));
    // compute_minimum_height, mesh.rs:58-84 (Rust f64::min ignores a NaN operand)
    const double surface = 0.5 * J;
    auto fmin_rs = [](double p, double q) { return std::isnan(p) ? q : (std::isnan(q) ? p : std::min(p, q)); };
    m.e_hmin[e] = fmin_rs(fmin_rs(2.0 * surface / a, 2.0 * surface / b), 2.0 * surface / c);
  }
  // set_neighbours, mesh.rs:133-147
  for (int64_t e = 0; e < ne; ++e)
    for (int k = 0; k < 3; ++k) {
      const int64_t d = m.e_edge[3 * e + k];
      if (m.d_elem[2 * d + 1] == -1) continue;
      if (m.e_vert[3 * e + k] == m.d_vert[2 * d]) m.e_nbr[3 * e + k] = m.d_elem[2 * d + 1];
      else m.e_nbr[3 * e + k] = m.d_elem[2 * d];
    }
  return ORC_OK;
}

// Physical derivative of mode b at cell GP q, key index kk (compute_dphi, mesh.rs:101-114).
// dinv = (dxi_dx, dxi_dy, deta_dx, deta_dy).
double phys_deriv(const Basis& B, const double* dinv, int q, int b, int kk) {
  const double* r = &B.dphi_cell[((size_t)q * B.nb + b) * B.nkeys];
  const double xx = dinv[0], xy = dinv[1], ex = dinv[2], ey = dinv[3];
  switch (kk) {
    case 0: return xx * r[0] + ex * r[1];  // (1,0)
    case 1: return xy * r[0] + ey * r[1];  // (0,1)
    case 2: return (xx * xx) * r[2] + 2.0 * xx * ex * r[3] + (ex * ex) * r[4];                     // (2,0)
    case 3: return xx * xy * r[2] + (xx * ey + ex * xy) * r[3] + ex * ey * r[4];                   // (1,1)
    case 4: return (xy * xy) * r[2] + 2.0 * xy * ey * r[3] + (ey * ey) * r[4];                     // (0,2)
    default: {
      // third order (p=3 extension): expand (xx Dxi + ex Deta)^a (xy Dxi + ey Deta)^c
      const int o = 3, c = kk - 5, a = o - c;
      double coef[4] = {0, 0, 0, 0};  // coefficient of Dxi^(3-j) Deta^j
      coef[0] = 1.0;
      int deg = 0;
      auto mul = [&](double s, double t) {  // multiply by (s Dxi + t Deta)
        double nc[4] = {0, 0, 0, 0};
        for (int j = 0; j <= deg; ++j) {
          nc[j] += coef[j] * s;
          nc[j + 1] += coef[j] * t;
        }
        ++deg;
        for (int j = 0; j < 4; ++j) coef[j] = nc[j];
      };
      for (int i = 0; i < a; ++i) mul(xx, ex);
      for (int i = 0; i < c; ++i) mul(xy, ey);
      double s = 0.0;
      for (int j = 0; j <= 3; ++j) s += coef[j] * r[5 + j];
      return s;
    }
  }
}

// ------------------------------------------------------------------------------------------
// Fluxes: src/spatial_disc/flux.rs:28-169, local_characteristics.rs:4-50.
// ------------------------------------------------------------------------------------------

// flux::flux, flux.rs:154-169
inline void euler_flux(const double* q, double hcr, double* f, double* g) {
  const double u = q[1] / q[0];
  const double v = q[2] / q[0];
  const double p = (hcr - 1.0) * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
  f[0] = q[1];
  f[1] = q[1] * u + p;
  f[2] = q[2] * u;
  f[3] = u * (q[3] + p);
  g[0] = q[2];
  g[1] = q[1] * v;
  g[2] = q[2] * v + p;
  g[3] = v * (q[3] + p);
}

// flux::hllc, flux.rs:28-153
int hllc(const double* lv, const double* rv, double nx, double ny, double hcr, double* flux) {
  const double ql[4] = {lv[0], lv[1] * nx + lv[2] * ny, -lv[1] * ny + lv[2] * nx, lv[3]};
  const double qr[4] = {rv[0], rv[1] * nx + rv[2] * ny, -rv[1] * ny + rv[2] * nx, rv[3]};
  const double ul = ql[1] / ql[0];
  const double ur = qr[1] / qr[0];
  const double vl = ql[2] / ql[0];
  const double vr = qr[2] / qr[0];
  const double pl = (hcr - 1.0) * (ql[3] - 0.5 * (ql[1] * ql[1] + ql[2] * ql[2]) / ql[0]);
  const double pr = (hcr - 1.0) * (qr[3] - 0.5 * (qr[1] * qr[1] + qr[2] * qr[2]) / qr[0]);
  if (ql[0] < 0.0 || qr[0] < 0.0) return ORC_NEG_DENSITY;
  if (pl < 0.0 || pr < 0.0) return ORC_NEG_PRESSURE;
  const double cl = std::sqrt(hcr * pl / ql[0]);
  const double cr = std::sqrt(hcr * pr / qr[0]);
  double fl[4], fr[4];
  fl[0] = ql[1];
  fl[1] = ql[1] * ul + pl;
  fl[2] = ql[2] * ul;
  fl[3] = ul * (ql[3] + pl);
  fr[0] = qr[1];
  fr[1] = qr[1] * ur + pr;
  fr[2] = qr[2] * ur;
  fr[3] = ur * (qr[3] + pr);
  const double zeta = (hcr - 1.0) / (2.0 * hcr);
  const double p_star =
      std::pow((cl + cr - (zeta - 1.0) / 2.0 * (ur - ul)) / (cl / std::pow(pl, zeta) + cr / std::pow(pr, zeta)),
               1.0 / zeta);
  const double ql_lower = (p_star <= pl) ? 1.0 : std::sqrt(1.0 + (hcr + 1.0) / (2.0 * hcr) * (p_star / pl - 1.0));
  const double sl = ul - cl * ql_lower;
  const double qr_lower = (p_star <= pr) ? 1.0 : std::sqrt(1.0 + (hcr + 1.0) / (2.0 * hcr) * (p_star / pr - 1.0));
  const double sr = ur + cr * qr_lower;
  if (sl >= 0.0) {
    flux[0] = fl[0];
    flux[1] = fl[1] * nx - fl[2] * ny;
    flux[2] = fl[1] * ny + fl[2] * nx;
    flux[3] = fl[3];
  } else if (sr <= 0.0) {
    flux[0] = fr[0];
    flux[1] = fr[1] * nx - fr[2] * ny;
    flux[2] = fr[1] * ny + fr[2] * nx;
    flux[3] = fr[3];
  } else {
    const double s_star = (pr - pl + ql[0] * ul * (sl - ul) - qr[0] * ur * (sr - ur)) /
                          (ql[0] * (sl - ul) - qr[0] * (sr - ur));
    if (s_star >= 0.0) {
      double qs[4];
      qs[0] = ql[0] * (sl - ul) / (sl - s_star);
      qs[1] = ql[0] * (sl - ul) / (sl - s_star) * s_star;
      qs[2] = ql[0] * (sl - ul) / (sl - s_star) * vl;
      qs[3] = ql[0] * (sl - ul) / (sl - s_star) * (ql[3] / ql[0] + (s_star - ul) * (s_star + pl / (ql[0] * (sl - ul))));
      flux[0] = fl[0] + sl * (qs[0] - ql[0]);
      const double fn = fl[1] + sl * (qs[1] - ql[1]);
      const double ft = fl[2] + sl * (qs[2] - ql[2]);
      flux[1] = fn * nx - ft * ny;
      flux[2] = fn * ny + ft * nx;
      flux[3] = fl[3] + sl * (qs[3] - ql[3]);
    } else {
      double qs[4];
      qs[0] = qr[0] * (sr - ur) / (sr - s_star);
      qs[1] = qr[0] * (sr - ur) / (sr - s_star) * s_star;
      qs[2] = qr[0] * (sr - ur) / (sr - s_star) * vr;
      qs[3] = qr[0] * (sr - ur) / (sr - s_star) * (qr[3] / qr[0] + (s_star - ur) * (s_star + pr / (qr[0] * (sr - ur))));
      flux[0] = fr[0] + sr * (qs[0] - qr[0]);
      const double fn = fr[1] + sr * (qs[1] - qr[1]);
      const double ft = fr[2] + sr * (qs[2] - qr[2]);
      flux[1] = fn * nx - ft * ny;
      flux[2] = fn * ny + ft * nx;
      flux[3] = fr[3] + sr * (qs[3] - qr[3]);
    }
  }
  return ORC_OK;
}

// compute_eigenmatrix, local_characteristics.rs:4-50
void eigenmatrix(const double* q, double nx, double ny, double hcr, double L[4][4], double R[4][4]) {
  const double u = q[1] / q[0];
  const double v = q[2] / q[0];
  const double p = (hcr - 1.0) * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
  const double c = std::sqrt(hcr * p / q[0]);
  const double h = (q[3] + p) / q[0];
  const double b1 = (hcr - 1.0) / (c * c);
  const double b2 = b1 * (u * u + v * v) / 2.0;
  L[0][0] = (b2 + (u * nx + v * ny) / c) / 2.0;
  L[0][1] = -(b1 * u + nx / c) / 2.0;
  L[0][2] = -(b1 * v + ny / c) / 2.0;
  L[0][3] = b1 / 2.0;
  L[1][0] = ny * u - nx * v;
  L[1][1] = -ny;
  L[1][2] = nx;
  L[1][3] = 0.0;
  L[2][0] = 1.0 - b2;
  L[2][1] = b1 * u;
  L[2][2] = b1 * v;
  L[2][3] = -b1;
  L[3][0] = (b2 - (u * nx + v * ny) / c) / 2.0;
  L[3][1] = -(b1 * u - nx / c) / 2.0;
  L[3][2] = -(b1 * v - ny / c) / 2.0;
  L[3][3] = b1 / 2.0;
  R[0][0] = 1.0;
  R[0][1] = 0.0;
  R[0][2] = 1.0;
  R[0][3] = 1.0;
  R[1][0] = u - c * nx;
  R[1][1] = -ny;
  R[1][2] = u;
  R[1][3] = u + c * nx;
  R[2][0] = v - c * ny;
  R[2][1] = nx;
  R[2][2] = v;
  R[2][3] = v + c * ny;
  R[3][0] = h - c * (u * nx + v * ny);
  R[3][1] = -u * ny + v * nx;
  R[3][2] = (u * u + v * v) / 2.0;
  R[3][3] = h + c * (u * nx + v * ny);
}

// ------------------------------------------------------------------------------------------
// Solver
// ------------------------------------------------------------------------------------------
struct Solver {
  Gauss g;
  Basis B;
  Mesh m;
  double hcr = 1.4;
  double cfl = 0.0;
  double final_time = 0.0;
  int64_t final_step = 0;
  FreeStream init{};
  int threads = 1;
  int limiter = 1;  // 1 = reference sequential in-place WENO, 0 = off
  // Navier-Stokes (BR2) residual in place of the Euler one: the reference's integrate_over_cell_ns,
  // integrate_over_edges_ns and apply_bc_ns (spatial_disc.rs:70-160,212-348,
  // boundary_condition.rs:121-413), which it keeps disabled (spatial_disc.rs:34-36)
  int viscous = 0;
  double prandtl_number = 0.72;  // parameters.json
  double gas_constant = 287.0;
  // time_march state (temporal_disc.rs:8-19)
  double current_time = 0.0;
  int64_t current_step = 0;
  std::vector<double> tmp0, tmp1;
  // diagnostics of the last failure
  int64_t err_where = -1;
  int64_t last_troubled = 0;
};

inline size_t SZ(const Solver& s) { return (size_t)s.m.ne * NEQ * s.B.nb; }

int nthreads(const Solver& s) {
#ifdef _OPENMP
  return std::max(1, s.threads);
#else
  (void)s;
  return 1;
#endif
}

// integrate_over_cell_euler, spatial_disc.rs:40-69 (one element, accumulated into acc[e])
void volume_element(const Solver& s, int64_t e, const double* U, double* acc) {
  const int nb = s.B.nb, nq = s.g.nq;
  const double* dinv = &s.m.e_dinv[4 * e];
  const double J = s.m.e_jac[e];
  for (int q = 0; q < nq; ++q) {
    double sol[4] = {0, 0, 0, 0};
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b) sol[v] += U[(e * NEQ + v) * nb + b] * s.B.phi_cell[q * nb + b];
    double f[4], gg[4];
    euler_flux(sol, s.hcr, f, gg);
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b) {
        const double dx = phys_deriv(s.B, dinv, q, b, 0);
        const double dy = phys_deriv(s.B, dinv, q, b, 1);
        acc[(e * NEQ + v) * nb + b] += (f[v] * dx + gg[v] * dy) * s.g.cell_w[q] * 0.5 * J;
      }
  }
}

// Parallel fold/reduce like the rayon sites (spatial_disc.rs:46,68 and :167,210,
// boundary_condition.rs:17,119): one zeroed accumulator per thread, then a sum.
template <class F>
int fold_reduce(const Solver& s, const std::vector<int64_t>& items, double* residuals, F&& body) {
  const size_t n = SZ(s);
  const int T = nthreads(s);
  std::vector<std::vector<double>> acc(T);
  int status = ORC_OK;
  int64_t where = -1;
#pragma omp parallel num_threads(T)
  {
#ifdef _OPENMP
    const int t = omp_get_thread_num();
#else
    const int t = 0;
#endif
    acc[t].assign(n, 0.0);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < (int64_t)items.size(); ++i) {
      const int st = body(items[i], acc[t].data());
      if (st != ORC_OK) {
#pragma omp critical
        {
          if (status == ORC_OK) {
            status = st;
            where = items[i];
          }
        }
      }
    }
  }
  std::vector<double> sum(n, 0.0);
  for (int t = 0; t < T; ++t)
    for (size_t i = 0; i < n; ++i) sum[i] = sum[i] + acc[t][i];
  for (size_t i = 0; i < n; ++i) residuals[i] = residuals[i] + sum[i];
  const_cast<Solver&>(s).err_where = where;
  return status;
}

// compute_boundary_edges_values, boundary_condition.rs:496-509
void boundary_trace(const Solver& s, int64_t d, const double* U, int g, double* out) {
  const int nb = s.B.nb, ng = s.g.ng;
  const int64_t e = s.m.d_elem[2 * d];
  const int ic = (int)s.m.d_icell[2 * d];
  for (int v = 0; v < NEQ; ++v) {
    out[v] = 0.0;
    for (int b = 0; b < nb; ++b) out[v] += U[(e * NEQ + v) * nb + b] * s.B.phi_edge[(ic * ng + g) * nb + b];
  }
}

int compute_residuals_ns(Solver& s, double* R, const double* U);

// compute_residuals, spatial_disc.rs:27-39
int compute_residuals(Solver& s, double* R, const double* U) {
  if (s.viscous) return compute_residuals_ns(s, R, U);
  const int nb = s.B.nb, ng = s.g.ng;
  // integrate_over_cell_euler (spatial_disc.rs:40-69)
  int st = fold_reduce(s, s.m.internal_elements, R, [&](int64_t e, double* acc) {
    volume_element(s, e, U, acc);
    return (int)ORC_OK;
  });
  if (st) return st;
  // integrate_over_edges_euler (spatial_disc.rs:161-211)
  st = fold_reduce(s, s.m.internal_edges, R, [&](int64_t d, double* acc) {
    const int ilic = (int)s.m.d_icell[2 * d], iric = (int)s.m.d_icell[2 * d + 1];
    const int64_t L = s.m.d_elem[2 * d], Rr = s.m.d_elem[2 * d + 1];
    const double nx = s.m.d_normal[2 * d], ny = s.m.d_normal[2 * d + 1];
    const double jd = s.m.d_jac[d];
    for (int g = 0; g < ng; ++g) {
      double lv[4] = {0, 0, 0, 0}, rv[4] = {0, 0, 0, 0};
      for (int v = 0; v < NEQ; ++v)
        for (int b = 0; b < nb; ++b) {
          lv[v] += U[(L * NEQ + v) * nb + b] * s.B.phi_edge[(ilic * ng + g) * nb + b];
          rv[v] += U[(Rr * NEQ + v) * nb + b] * s.B.phi_edge[(iric * ng + (ng - 1 - g)) * nb + b];
        }
      double fl[4];
      const int hs = hllc(lv, rv, nx, ny, s.hcr, fl);
      if (hs != ORC_OK) return hs;
      for (int v = 0; v < NEQ; ++v)
        for (int b = 0; b < nb; ++b) {
          acc[(L * NEQ + v) * nb + b] -= s.g.edge_w[g] * fl[v] * s.B.phi_edge[(ilic * ng + g) * nb + b] * 0.5 * jd;
          acc[(Rr * NEQ + v) * nb + b] +=
              s.g.edge_w[ng - 1 - g] * fl[v] * s.B.phi_edge[(iric * ng + (ng - 1 - g)) * nb + b] * 0.5 * jd;
        }
    }
    return (int)ORC_OK;
  });
  if (st) return st;
  // apply_bc_euler (boundary_condition.rs:9-120)
  st = fold_reduce(s, s.m.boundary_elements, R, [&](int64_t e, double* acc) {
    for (int k = 0; k < 3; ++k) {
      const int64_t d = s.m.e_edge[3 * e + k];
      const int64_t patch = s.m.d_patch[d];
      if (patch == -1) continue;
      double nx, ny;
      if (s.m.e_vert[3 * e + k] == s.m.d_vert[2 * d]) {
        nx = s.m.d_normal[2 * d];
        ny = s.m.d_normal[2 * d + 1];
      } else {
        nx = -s.m.d_normal[2 * d];
        ny = -s.m.d_normal[2 * d + 1];
      }
      const double jd = s.m.d_jac[d];
      if (s.m.p_type[patch] == WALL) {
        for (int g = 0; g < ng; ++g) {
          double lv[4];
          boundary_trace(s, d, U, g, lv);
          const double pressure = (s.hcr - 1.0) * (lv[3] - 0.5 * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
          const double bf[4] = {0.0, pressure * nx, pressure * ny, 0.0};
          for (int v = 0; v < NEQ; ++v)
            for (int b = 0; b < nb; ++b)
              acc[(e * NEQ + v) * nb + b] -= s.g.edge_w[g] * bf[v] * s.B.phi_edge[(k * ng + g) * nb + b] * 0.5 * jd;
        }
      } else {
        const double* bq = &s.m.p_q[4 * patch];
        const double bc[4] = {bq[0], bq[0] * bq[1], bq[0] * bq[2],
                              bq[3] / (s.hcr - 1.0) + 0.5 * bq[0] * (bq[1] * bq[1] + bq[2] * bq[2])};
        std::vector<double> qn(ng * 4);
        for (int g = 0; g < ng; ++g) {
          double lv[4];
          boundary_trace(s, d, U, g, lv);
          const double u = lv[1] / lv[0];
          const double v = lv[2] / lv[0];
          const double p = (s.hcr - 1.0) * (lv[3] - 0.5 * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
          const double c = std::sqrt(s.hcr * p / lv[0]);
          const double vn = u * nx + v * ny;
          double Lm[4][4], Rm[4][4];
          eigenmatrix(lv, nx, ny, s.hcr, Lm, Rm);
          const double lam[4] = {vn - c, vn, vn, vn + c};
          double mix[4];
          for (int i = 0; i < 4; ++i) {
            double alpha = 0.0, beta = 0.0;
            for (int j = 0; j < 4; ++j) {
              alpha = alpha + Lm[i][j] * lv[j];
              beta = beta + Lm[i][j] * bc[j];
            }
            mix[i] = lam[i] >= 0.0 ? alpha : beta;
          }
          for (int i = 0; i < 4; ++i) {
            double sum = 0.0;
            for (int j = 0; j < 4; ++j) sum = sum + Rm[i][j] * mix[j];
            qn[g * 4 + i] = sum;
          }
        }
        for (int g = 0; g < ng; ++g) {
          const double* q = &qn[g * 4];
          const double un = q[1] / q[0];
          const double vv = q[2] / q[0];
          const double vn_new = un * nx + vv * ny;
          const double p_new = (s.hcr - 1.0) * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
          const double h_new = q[3] + p_new;
          const double bf[4] = {q[0] * vn_new, q[1] * vn_new + p_new * nx, q[2] * vn_new + p_new * ny,
                                h_new * vn_new};
          for (int v = 0; v < NEQ; ++v)
            for (int b = 0; b < nb; ++b)
              acc[(e * NEQ + v) * nb + b] -= s.g.edge_w[g] * bf[v] * s.B.phi_edge[(k * ng + g) * nb + b] * 0.5 * jd;
        }
      }
    }
    volume_element(s, e, U, acc);
    return (int)ORC_OK;
  });
  if (st) return st;
  // divide_residual_by_mass_mat_diag, spatial_disc.rs:349-357
  const int64_t ne = s.m.ne;
  for (int64_t e = 0; e < ne; ++e)
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b) R[(e * NEQ + v) * nb + b] /= s.B.mass[b] * 0.5 * s.m.e_jac[e];
  return ORC_OK;
}

// ------------------------------------------------------------------------------------------
// Navier-Stokes terms (BR2 lifting), kept disabled by the reference (spatial_disc.rs:34-36).
// ------------------------------------------------------------------------------------------

// compute_dynamic_viscosity, viscous.rs:6-12 (Sutherland's law)
double dynamic_viscosity(double temperature) {
  const double mu_ref = 1.716e-5;
  const double sutherland_constant = 110.4;
  const double t_ref = 273.15;
  return mu_ref * std::pow(temperature / t_ref, 1.5) * (t_ref + sutherland_constant) /
         (temperature + sutherland_constant);
}

// viscous_jacobian, viscous.rs:13-64: G[0..3] = g11, g12, g21, g22, each [4][4], times mu / rho.
void viscous_jacobian(const Solver& s, const double* q, double mu, double G[4][4][4]) {
  const double hcr = s.hcr, pr = s.prandtl_number;
  const double u = q[1] / q[0];
  const double v = q[2] / q[0];
  const double e = q[3] / q[0];
  for (int m = 0; m < 4; ++m)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) G[m][i][j] = 0.0;
  double(&g11)[4][4] = G[0];
  double(&g12)[4][4] = G[1];
  double(&g21)[4][4] = G[2];
  double(&g22)[4][4] = G[3];
  g11[1][0] = -4.0 / 3.0 * u;
  g11[1][1] = 4.0 / 3.0;
  g11[2][0] = -v;
  g11[2][2] = 1.0;
  g11[3][0] = -(4.0 / 3.0 * std::pow(u, 2.0) + std::pow(v, 2.0) + hcr / pr * (e - std::pow(u, 2.0) - std::pow(v, 2.0)));
  g11[3][1] = (4.0 / 3.0 - hcr / pr) * u;
  g11[3][2] = (1.0 - hcr / pr) * v;
  g11[3][3] = hcr / pr;
  g12[1][0] = 2.0 / 3.0 * v;
  g12[1][2] = -2.0 / 3.0;
  g12[2][0] = -u;
  g12[2][1] = 1.0;
  g12[3][0] = -1.0 / 3.0 * u * v;
  g12[3][1] = v;
  g12[3][2] = -2.0 / 3.0 * u;
  g21[1][0] = -v;
  g21[1][2] = 1.0;
  g21[2][0] = 2.0 / 3.0 * u;
  g21[2][1] = -2.0 / 3.0;
  g21[3][0] = -1.0 / 3.0 * u * v;
  g21[3][1] = -2.0 / 3.0 * v;
  g21[3][2] = u;
  g22[1][0] = -u;
  g22[1][1] = 1.0;
  g22[2][0] = -4.0 / 3.0 * v;
  g22[2][2] = 4.0 / 3.0;
  g22[3][0] = -(std::pow(u, 2.0) + 4.0 / 3.0 * std::pow(v, 2.0) + hcr / pr * (e - std::pow(u, 2.0) - std::pow(v, 2.0)));
  g22[3][1] = (1.0 - hcr / pr) * u;
  g22[3][2] = (4.0 / 3.0 - hcr / pr) * v;
  g22[3][3] = hcr / pr;
  const double scale = mu / q[0];  // g11 *= mu / q[0], ... (viscous.rs:58-61)
  for (int m = 0; m < 4; ++m)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) G[m][i][j] *= scale;
}

// The viscosity of a state (the `viscosity` blocks of spatial_disc.rs:125-129 and the other
// NS sites): pressure, T = p / (R rho), Sutherland.
double state_viscosity(const Solver& s, const double* q) {
  const double pressure = (s.hcr - 1.0) * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
  const double temperature = pressure / (s.gas_constant * q[0]);
  return dynamic_viscosity(temperature);
}

// Physical first derivative of mode b at point g of local edge k of an element (the
// dphis_edge_gps of mesh.rs:115-127), kk = 0: d/dx, 1: d/dy.
double phys_deriv_edge(const Basis& B, int ng, const double* dinv, int k, int g, int b, int kk) {
  const double* r = &B.dphi_edge[(((size_t)k * ng + g) * B.nb + b) * 2];
  return kk == 0 ? dinv[0] * r[0] + dinv[2] * r[1] : dinv[1] * r[0] + dinv[3] * r[1];
}

// fv, gv of spatial_disc.rs:131-146 and the other NS sites: G times (gradient + lift), with the
// gradient of dofs and the lift evaluated by the callbacks for (ivar, ibasis).
template <class DX, class DY, class LX, class LY>
void viscous_flux(const double G[4][4][4], const double* dofs, int nb, DX dphi_dx, DY dphi_dy, LX lift_x, LY lift_y,
                  double* fv, double* gv) {
  for (int i = 0; i < 4; ++i) fv[i] = gv[i] = 0.0;
  for (int iflux = 0; iflux < NEQ; ++iflux)
    for (int ivar = 0; ivar < NEQ; ++ivar) {
      double dsol_dx = 0.0, dsol_dy = 0.0, lx = 0.0, ly = 0.0;
      for (int b = 0; b < nb; ++b) {
        dsol_dx += dofs[ivar * nb + b] * dphi_dx(b);
        dsol_dy += dofs[ivar * nb + b] * dphi_dy(b);
        lx += lift_x(ivar, b);
        ly += lift_y(ivar, b);
      }
      fv[iflux] += G[0][iflux][ivar] * (dsol_dx + lx) + G[1][iflux][ivar] * (dsol_dy + ly);
      gv[iflux] += G[2][iflux][ivar] * (dsol_dx + lx) + G[3][iflux][ivar] * (dsol_dy + ly);
    }
}

// The neighbour an element's lifting operator takes across its local edge k (spatial_disc.rs:86-93,
// boundary_condition.rs:145-152), with the reference's test: the edge's first in-cell index equal
// to k selects the edge's second element and the edge normal, else its first element and the
// negated normal -- whichever side e is on.
void lift_neighbour(const Solver& s, int64_t d, int k, int& iric, int64_t& irelem, double& nx, double& ny) {
  if (s.m.d_icell[2 * d] == k) {
    iric = (int)s.m.d_icell[2 * d + 1];
    irelem = s.m.d_elem[2 * d + 1];
    nx = s.m.d_normal[2 * d];
    ny = s.m.d_normal[2 * d + 1];
  } else {
    iric = (int)s.m.d_icell[2 * d];
    irelem = s.m.d_elem[2 * d];
    nx = -s.m.d_normal[2 * d];
    ny = -s.m.d_normal[2 * d + 1];
  }
}

// The jump terms of variable ivar, mode ibasis across local edge k into lift[ivar][ibasis]
// (spatial_disc.rs:95-108, boundary_condition.rs:156-167).
void lift_edge_terms(const Solver& s, int64_t e, int k, const double* U, int ivar, int ibasis, double* lx, double* ly) {
  const int nb = s.B.nb, ng = s.g.ng;
  const int64_t d = s.m.e_edge[3 * e + k];
  int iric;
  int64_t irelem;
  double nx, ny;
  lift_neighbour(s, d, k, iric, irelem, nx, ny);
  for (int g = 0; g < ng; ++g) {
    double left_value = 0.0, right_value = 0.0;
    for (int b = 0; b < nb; ++b) {
      left_value += U[(e * NEQ + ivar) * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b];
      right_value += U[(irelem * NEQ + ivar) * nb + b] * s.B.phi_edge[(iric * ng + (ng - 1 - g)) * nb + b];
    }
    const double jump_x = (left_value - right_value) * nx;
    const double jump_y = (left_value - right_value) * ny;
    *lx -= 0.5 * jump_x * s.B.phi_edge[(k * ng + g) * nb + ibasis] * s.g.edge_w[g] * 0.5 * s.m.d_jac[d];
    *ly -= 0.5 * jump_y * s.B.phi_edge[(k * ng + g) * nb + ibasis] * s.g.edge_w[g] * 0.5 * s.m.d_jac[d];
  }
}

// The cell term with the element's global lift (spatial_disc.rs:114-155, boundary_condition.rs:373-407).
void ns_volume(const Solver& s, int64_t e, const double* U, const double* glx, const double* gly, double* acc) {
  const int nb = s.B.nb, nq = s.g.nq;
  const double* dinv = &s.m.e_dinv[4 * e];
  const double J = s.m.e_jac[e];
  for (int q = 0; q < nq; ++q) {
    double sol[4] = {0, 0, 0, 0};
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b) sol[v] += U[(e * NEQ + v) * nb + b] * s.B.phi_cell[q * nb + b];
    double f[4], gg[4];
    euler_flux(sol, s.hcr, f, gg);
    double G[4][4][4];
    viscous_jacobian(s, sol, state_viscosity(s, sol), G);
    double fv[4], gv[4];
    viscous_flux(
        G, &U[e * NEQ * nb], nb, [&](int b) { return phys_deriv(s.B, dinv, q, b, 0); },
        [&](int b) { return phys_deriv(s.B, dinv, q, b, 1); },
        [&](int ivar, int b) { return glx[ivar * nb + b] * s.B.phi_cell[q * nb + b]; },
        [&](int ivar, int b) { return gly[ivar * nb + b] * s.B.phi_cell[q * nb + b]; }, fv, gv);
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b) {
        const double dx = phys_deriv(s.B, dinv, q, b, 0);
        const double dy = phys_deriv(s.B, dinv, q, b, 1);
        acc[(e * NEQ + v) * nb + b] += ((f[v] - fv[v]) * dx + (gg[v] - gv[v]) * dy) * s.g.cell_w[q] * 0.5 * J;
      }
  }
}

// compute_residuals with the Navier-Stokes terms (spatial_disc.rs:27-39 with the NS calls of
// :34-36 in place of the Euler ones).
int compute_residuals_ns(Solver& s, double* R, const double* U) {
  const int nb = s.B.nb, ng = s.g.ng;
  // integrate_over_cell_ns, spatial_disc.rs:70-160
  int st = fold_reduce(s, s.m.internal_elements, R, [&](int64_t e, double* acc) {
    std::vector<double> glx(NEQ * nb, 0.0), gly(NEQ * nb, 0.0);
    for (int ivar = 0; ivar < NEQ; ++ivar)
      for (int ibasis = 0; ibasis < nb; ++ibasis) {
        for (int k = 0; k < 3; ++k) lift_edge_terms(s, e, k, U, ivar, ibasis, &glx[ivar * nb + ibasis], &gly[ivar * nb + ibasis]);
        glx[ivar * nb + ibasis] /= s.B.mass[ibasis] * 0.5 * s.m.e_jac[e];
        gly[ivar * nb + ibasis] /= s.B.mass[ibasis] * 0.5 * s.m.e_jac[e];
      }
    ns_volume(s, e, U, glx.data(), gly.data(), acc);
    return (int)ORC_OK;
  });
  if (st) return st;
  // integrate_over_edges_ns, spatial_disc.rs:212-348
  st = fold_reduce(s, s.m.internal_edges, R, [&](int64_t d, double* acc) {
    const int ilic = (int)s.m.d_icell[2 * d], iric = (int)s.m.d_icell[2 * d + 1];
    const int64_t L = s.m.d_elem[2 * d], Rr = s.m.d_elem[2 * d + 1];
    const double nx = s.m.d_normal[2 * d], ny = s.m.d_normal[2 * d + 1];
    const double jd = s.m.d_jac[d];
    const double* ldofs = &U[L * NEQ * nb];
    const double* rdofs = &U[Rr * NEQ * nb];
    std::vector<double> llx(NEQ * nb, 0.0), lly(NEQ * nb, 0.0), rlx(NEQ * nb, 0.0), rly(NEQ * nb, 0.0);
    for (int ivar = 0; ivar < NEQ; ++ivar)
      for (int ibasis = 0; ibasis < nb; ++ibasis) {
        const int i = ivar * nb + ibasis;
        for (int g = 0; g < ng; ++g) {
          double left_value = 0.0, right_value = 0.0;
          for (int b = 0; b < nb; ++b) {
            left_value += ldofs[ivar * nb + b] * s.B.phi_edge[(ilic * ng + g) * nb + b];
            right_value += rdofs[ivar * nb + b] * s.B.phi_edge[(iric * ng + (ng - 1 - g)) * nb + b];
          }
          const double jump_x = (left_value - right_value) * nx;
          const double jump_y = (left_value - right_value) * ny;
          llx[i] -= 0.5 * jump_x * s.B.phi_edge[(ilic * ng + g) * nb + ibasis] * s.g.edge_w[g] * 0.5 * jd;
          lly[i] -= 0.5 * jump_y * s.B.phi_edge[(ilic * ng + g) * nb + ibasis] * s.g.edge_w[g] * 0.5 * jd;
          rlx[i] += 0.5 * jump_x * s.B.phi_edge[(iric * ng + (ng - 1 - g)) * nb + ibasis] * s.g.edge_w[ng - 1 - g] * 0.5 * jd;
          rly[i] += 0.5 * jump_y * s.B.phi_edge[(iric * ng + (ng - 1 - g)) * nb + ibasis] * s.g.edge_w[ng - 1 - g] * 0.5 * jd;
        }
        llx[i] /= s.B.mass[ibasis] * 0.5 * s.m.e_jac[L];
        lly[i] /= s.B.mass[ibasis] * 0.5 * s.m.e_jac[L];
        rlx[i] /= s.B.mass[ibasis] * 0.5 * s.m.e_jac[Rr];
        rly[i] /= s.B.mass[ibasis] * 0.5 * s.m.e_jac[Rr];
      }
    const double* ldinv = &s.m.e_dinv[4 * L];
    const double* rdinv = &s.m.e_dinv[4 * Rr];
    for (int g = 0; g < ng; ++g) {
      const int gr = ng - 1 - g;
      double lv[4] = {0, 0, 0, 0}, rv[4] = {0, 0, 0, 0};
      for (int v = 0; v < NEQ; ++v)
        for (int b = 0; b < nb; ++b) {
          lv[v] += ldofs[v * nb + b] * s.B.phi_edge[(ilic * ng + g) * nb + b];
          rv[v] += rdofs[v * nb + b] * s.B.phi_edge[(iric * ng + gr) * nb + b];
        }
      double num_flux[4];
      const int hs = hllc(lv, rv, nx, ny, s.hcr, num_flux);
      if (hs != ORC_OK) return hs;
      double num_visc[4] = {0, 0, 0, 0};
      double G[4][4][4], fv[4], gv[4];
      // left contribution (spatial_disc.rs:281-307): lifts scaled by 3
      viscous_jacobian(s, lv, state_viscosity(s, lv), G);
      viscous_flux(
          G, ldofs, nb, [&](int b) { return phys_deriv_edge(s.B, ng, ldinv, ilic, g, b, 0); },
          [&](int b) { return phys_deriv_edge(s.B, ng, ldinv, ilic, g, b, 1); },
          [&](int ivar, int b) { return 3.0 * llx[ivar * nb + b] * s.B.phi_edge[(ilic * ng + g) * nb + b]; },
          [&](int ivar, int b) { return 3.0 * lly[ivar * nb + b] * s.B.phi_edge[(ilic * ng + g) * nb + b]; }, fv, gv);
      for (int v = 0; v < NEQ; ++v) num_visc[v] = num_visc[v] + 0.5 * (nx * fv[v] + ny * gv[v]);
      // right contribution (spatial_disc.rs:309-335): lifts not scaled
      viscous_jacobian(s, rv, state_viscosity(s, rv), G);
      viscous_flux(
          G, rdofs, nb, [&](int b) { return phys_deriv_edge(s.B, ng, rdinv, iric, gr, b, 0); },
          [&](int b) { return phys_deriv_edge(s.B, ng, rdinv, iric, gr, b, 1); },
          [&](int ivar, int b) { return rlx[ivar * nb + b] * s.B.phi_edge[(iric * ng + gr) * nb + b]; },
          [&](int ivar, int b) { return rly[ivar * nb + b] * s.B.phi_edge[(iric * ng + gr) * nb + b]; }, fv, gv);
      for (int v = 0; v < NEQ; ++v) num_visc[v] = num_visc[v] + 0.5 * (nx * fv[v] + ny * gv[v]);
      for (int v = 0; v < NEQ; ++v)
        for (int b = 0; b < nb; ++b) {
          acc[(L * NEQ + v) * nb + b] -=
              s.g.edge_w[g] * (num_flux[v] - num_visc[v]) * s.B.phi_edge[(ilic * ng + g) * nb + b] * 0.5 * jd;
          acc[(Rr * NEQ + v) * nb + b] +=
              s.g.edge_w[gr] * (num_flux[v] - num_visc[v]) * s.B.phi_edge[(iric * ng + gr) * nb + b] * 0.5 * jd;
        }
    }
    return (int)ORC_OK;
  });
  if (st) return st;
  // apply_bc_ns, boundary_condition.rs:121-413
  st = fold_reduce(s, s.m.boundary_elements, R, [&](int64_t e, double* acc) {
    std::vector<double> glx(NEQ * nb, 0.0), gly(NEQ * nb, 0.0);
    const double J = s.m.e_jac[e];
    const double* dofs = &U[e * NEQ * nb];
    const double* dinv = &s.m.e_dinv[4 * e];
    for (int k = 0; k < 3; ++k) {
      const int64_t d = s.m.e_edge[3 * e + k];
      const int64_t patch = s.m.d_patch[d];
      if (patch == -1) {  // boundary_condition.rs:144-168
        for (int ivar = 0; ivar < NEQ; ++ivar)
          for (int ibasis = 0; ibasis < nb; ++ibasis)
            lift_edge_terms(s, e, k, U, ivar, ibasis, &glx[ivar * nb + ibasis], &gly[ivar * nb + ibasis]);
        continue;
      }
      double nx, ny;
      if (s.m.e_vert[3 * e + k] == s.m.d_vert[2 * d]) {
        nx = s.m.d_normal[2 * d];
        ny = s.m.d_normal[2 * d + 1];
      } else {
        nx = -s.m.d_normal[2 * d];
        ny = -s.m.d_normal[2 * d + 1];
      }
      const double jd = s.m.d_jac[d];
      std::vector<double> llx(NEQ * nb, 0.0), lly(NEQ * nb, 0.0);
      if (s.m.p_type[patch] == WALL) {  // boundary_condition.rs:181-246
        for (int g = 0; g < ng; ++g) {
          double lv[4];
          boundary_trace(s, d, U, g, lv);
          const double pressure = (s.hcr - 1.0) * (lv[3] - 0.5 * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
          const double boundary_energy = pressure / (s.hcr - 1.0);
          const double jx[4] = {0.0, lv[1] * nx, lv[2] * nx, (lv[3] - boundary_energy) * nx};
          const double jy[4] = {0.0, lv[1] * ny, lv[2] * ny, (lv[3] - boundary_energy) * ny};
          // the cell table and cell weights at index g, as the reference writes them (:193-200)
          for (int b = 0; b < nb; ++b)
            for (int v = 1; v < NEQ; ++v) {
              llx[v * nb + b] -= 0.5 * jx[v] * s.B.phi_cell[g * nb + b] * s.g.cell_w[g] * 0.5 * J;
              lly[v * nb + b] -= 0.5 * jy[v] * s.B.phi_cell[g * nb + b] * s.g.cell_w[g] * 0.5 * J;
            }
        }
        for (int i = 0; i < NEQ * nb; ++i) {
          glx[i] = glx[i] + llx[i];
          gly[i] = gly[i] + lly[i];
        }
        for (int v = 1; v < NEQ; ++v)
          for (int b = 0; b < nb; ++b) {
            llx[v * nb + b] /= s.B.mass[b] * 0.5 * J;
            lly[v * nb + b] /= s.B.mass[b] * 0.5 * J;
          }
        for (int g = 0; g < ng; ++g) {
          double lv[4];
          boundary_trace(s, d, U, g, lv);
          const double pressure = (s.hcr - 1.0) * (lv[3] - 0.5 * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
          const double inv[4] = {0.0, pressure * nx, pressure * ny, 0.0};
          const double temperature = pressure / (s.gas_constant * lv[0]);
          double G[4][4][4], fv[4], gv[4];
          viscous_jacobian(s, lv, dynamic_viscosity(temperature), G);
          viscous_flux(
              G, dofs, nb, [&](int b) { return phys_deriv_edge(s.B, ng, dinv, k, g, b, 0); },
              [&](int b) { return phys_deriv_edge(s.B, ng, dinv, k, g, b, 1); },
              [&](int ivar, int b) { return 3.0 * llx[ivar * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b]; },
              [&](int ivar, int b) { return 3.0 * lly[ivar * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b]; }, fv, gv);
          for (int v = 0; v < NEQ; ++v) {
            const double visc = nx * fv[v] + ny * gv[v];
            for (int b = 0; b < nb; ++b)
              acc[(e * NEQ + v) * nb + b] -= s.g.edge_w[g] * (inv[v] - visc) * s.B.phi_edge[(k * ng + g) * nb + b] * 0.5 * jd;
          }
        }
      } else {  // far field, boundary_condition.rs:248-370
        const double* bq = &s.m.p_q[4 * patch];
        const double bc[4] = {bq[0], bq[0] * bq[1], bq[0] * bq[2],
                              bq[3] / (s.hcr - 1.0) + 0.5 * bq[0] * (bq[1] * bq[1] + bq[2] * bq[2])};
        std::vector<double> qn(ng * 4);
        for (int g = 0; g < ng; ++g) {
          double lv[4];
          boundary_trace(s, d, U, g, lv);
          const double u = lv[1] / lv[0];
          const double v = lv[2] / lv[0];
          const double p = (s.hcr - 1.0) * (lv[3] - 0.5 * (lv[1] * lv[1] + lv[2] * lv[2]) / lv[0]);
          const double c = std::sqrt(s.hcr * p / lv[0]);
          const double vn = u * nx + v * ny;
          double Lm[4][4], Rm[4][4];
          eigenmatrix(lv, nx, ny, s.hcr, Lm, Rm);
          const double lam[4] = {vn - c, vn, vn, vn + c};
          double mix[4];
          for (int i = 0; i < 4; ++i) {
            double alpha = 0.0, beta = 0.0;
            for (int j = 0; j < 4; ++j) {
              alpha = alpha + Lm[i][j] * lv[j];
              beta = beta + Lm[i][j] * bc[j];
            }
            mix[i] = lam[i] >= 0.0 ? alpha : beta;
          }
          double* q = &qn[g * 4];
          for (int i = 0; i < 4; ++i) {
            double sum = 0.0;
            for (int j = 0; j < 4; ++j) sum = sum + Rm[i][j] * mix[j];
            q[i] = sum;
          }
          for (int b = 0; b < nb; ++b)
            for (int w = 0; w < NEQ; ++w) {
              llx[w * nb + b] -= 0.5 * ((lv[w] - q[w]) * nx) * s.B.phi_edge[(k * ng + g) * nb + b] * s.g.edge_w[g] * 0.5 * jd;
              lly[w * nb + b] -= 0.5 * ((lv[w] - q[w]) * ny) * s.B.phi_edge[(k * ng + g) * nb + b] * s.g.edge_w[g] * 0.5 * jd;
            }
        }
        for (int i = 0; i < NEQ * nb; ++i) {
          glx[i] = glx[i] + llx[i];
          gly[i] = gly[i] + lly[i];
        }
        for (int w = 0; w < NEQ; ++w)
          for (int b = 0; b < nb; ++b) {
            llx[w * nb + b] /= s.B.mass[b] * 0.5 * J;
            lly[w * nb + b] /= s.B.mass[b] * 0.5 * J;
          }
        for (int g = 0; g < ng; ++g) {
          const double* q = &qn[g * 4];
          const double u_new = q[1] / q[0];
          const double v_new = q[2] / q[0];
          const double vn_new = u_new * nx + v_new * ny;
          const double p_new = (s.hcr - 1.0) * (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0]);
          const double h_new = q[3] + p_new;
          const double inv[4] = {q[0] * vn_new, q[1] * vn_new + p_new * nx, q[2] * vn_new + p_new * ny,
                                 h_new * vn_new};
          double lv[4];
          boundary_trace(s, d, U, g, lv);
          double G[4][4][4], fv[4], gv[4];
          viscous_jacobian(s, lv, state_viscosity(s, lv), G);
          viscous_flux(
              G, dofs, nb, [&](int b) { return phys_deriv_edge(s.B, ng, dinv, k, g, b, 0); },
              [&](int b) { return phys_deriv_edge(s.B, ng, dinv, k, g, b, 1); },
              [&](int ivar, int b) { return 3.0 * llx[ivar * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b]; },
              [&](int ivar, int b) { return 3.0 * lly[ivar * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b]; }, fv, gv);
          for (int v = 0; v < NEQ; ++v) {
            const double visc = nx * fv[v] + ny * gv[v];
            for (int b = 0; b < nb; ++b)
              acc[(e * NEQ + v) * nb + b] -= s.g.edge_w[g] * (inv[v] - visc) * s.B.phi_edge[(k * ng + g) * nb + b] * 0.5 * jd;
          }
        }
      }
    }
    for (int i = 0; i < NEQ * nb; ++i) {
      glx[i] /= s.B.mass[i % nb] * 0.5 * J;
      gly[i] /= s.B.mass[i % nb] * 0.5 * J;
    }
    ns_volume(s, e, U, glx.data(), gly.data(), acc);
    return (int)ORC_OK;
  });
  if (st) return st;
  const int64_t ne = s.m.ne;
  for (int64_t e = 0; e < ne; ++e)
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b) R[(e * NEQ + v) * nb + b] /= s.B.mass[b] * 0.5 * s.m.e_jac[e];
  return ORC_OK;
}

// modified_kxrcf, weno.rs:7-85
bool modified_kxrcf(const Solver& s, const double* U, int64_t e) {
  const int nb = s.B.nb, ng = s.g.ng;
  double density_jump = 0.0, total_energy_jump = 0.0, surface = 0.0;
  double min_density = 1.0e10, min_total_energy = 1.0e10;
  for (int k = 0; k < 3; ++k) {
    const int64_t d = s.m.e_edge[3 * e + k];
    if (s.m.d_elem[2 * d + 1] == -1) continue;
    const int64_t nbr = s.m.e_nbr[3 * e + k];
    double nx, ny;
    int nic;
    if (s.m.e_vert[3 * e + k] == s.m.d_vert[2 * d]) {
      nx = s.m.d_normal[2 * d];
      ny = s.m.d_normal[2 * d + 1];
      nic = (int)s.m.d_icell[2 * d];
    } else {
      nx = -s.m.d_normal[2 * d];
      ny = -s.m.d_normal[2 * d + 1];
      nic = (int)s.m.d_icell[2 * d + 1];
    }
    for (int g = 0; g < ng; ++g) {
      double rho = 0.0, rho_e = 0.0;
      for (int b = 0; b < nb; ++b) {
        rho += U[(e * NEQ + 0) * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b];
        rho_e += U[(e * NEQ + 3) * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b];
      }
      if (rho < min_density) min_density = rho;
      if (rho_e < min_total_energy) min_total_energy = rho_e;
    }
    const int cg = ng / 2;
    double rho_u = 0.0, rho_v = 0.0;
    for (int b = 0; b < nb; ++b) {
      rho_u += U[(e * NEQ + 1) * nb + b] * s.B.phi_edge[(k * ng + cg) * nb + b];
      rho_v += U[(e * NEQ + 2) * nb + b] * s.B.phi_edge[(k * ng + cg) * nb + b];
    }
    const double center = rho_u * nx + rho_v * ny;
    if (center < 0.0) {
      double rho_jump = 0.0, rho_e_jump = 0.0;
      const double jd = s.m.d_jac[d];
      for (int g = 0; g < ng; ++g) {
        double ir = 0.0, ire = 0.0, er = 0.0, ere = 0.0;
        for (int b = 0; b < nb; ++b) {
          ir += U[(e * NEQ + 0) * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b];
          ire += U[(e * NEQ + 3) * nb + b] * s.B.phi_edge[(k * ng + g) * nb + b];
          er += U[(nbr * NEQ + 0) * nb + b] * s.B.phi_edge[(nic * ng + (ng - 1 - g)) * nb + b];
          ere += U[(nbr * NEQ + 3) * nb + b] * s.B.phi_edge[(nic * ng + (ng - 1 - g)) * nb + b];
        }
        rho_jump += 0.5 * jd * s.g.edge_w[g] * (ir - er);
        rho_e_jump += 0.5 * jd * s.g.edge_w[g] * (ire - ere);
      }
      density_jump += rho_jump;
      total_energy_jump += rho_e_jump;
      surface += jd;
    }
  }
  const double h = s.m.e_circ[e];
  const double h15 = std::pow(h, 1.5);
  const double ind_d = std::fabs(density_jump) / (h15 * surface * min_density);
  const double ind_e = std::fabs(total_energy_jump) / (h15 * surface * min_total_energy);
  return (ind_d >= 1.0) || (ind_e >= 1.0);
}

// beta of one projected polynomial (weno.rs:125-142 and :156-173)
double smoothness(const Solver& s, const double* dinv, double J, const double* pol) {
  const int nb = s.B.nb, nq = s.g.nq;
  double beta = 0.0;
  for (int l = 1; l <= s.B.p; ++l)
    for (int l1 = 0; l1 <= l; ++l1) {
      const int l2 = l - l1;
      const int kk = key_index(l1, l2);
      double integral = 0.0;
      for (int q = 0; q < nq; ++q) {
        double value = 0.0;
        for (int b = 0; b < nb; ++b) value += pol[b] * phys_deriv(s.B, dinv, q, b, kk);
        integral += 0.5 * J * s.g.cell_w[q] * (value * value);
      }
      beta += std::pow(J, (double)(l - 1)) * integral;
    }
  return beta;
}


// weno, weno.rs:86-269.  Sequential over elements in index order, in place: later elements see
// the already-limited values of earlier ones, exactly like the reference.
int weno(Solver& s, double* U) {
  const int nb = s.B.nb;
  const int64_t ne = s.m.ne;
  int64_t troubled = 0;
  std::vector<double> proj(4 * NEQ * nb), recon(NEQ * nb), pol_new(NEQ * nb), tmp(NEQ * nb),
      nbpol(NEQ * nb);
  for (int64_t e = 0; e < ne; ++e) {
    if (!modified_kxrcf(s, U, e)) continue;
    ++troubled;
    // linear weights (weno.rs:93-110), including the reference's indexing
    double lw[4] = {0.997, 0.001, 0.001, 0.001};
    int nbd = 0;
    for (int i = 0; i < 3; ++i) {
      const int64_t d = s.m.e_edge[3 * e + i];
      if (s.m.d_elem[2 * d + 1] == -1) {
        ++nbd;
        lw[i] = 0.0;
      }
    }
    if (nbd == 0) lw[0] = 0.997;
    else if (nbd == 1) lw[1] = 0.998;
    else if (nbd == 2) lw[2] = 0.999;
    else {
      s.err_where = e;
      return ORC_TOO_MANY_BOUNDARY_EDGES;
    }
    const double* dinv = &s.m.e_dinv[4 * e];
    const double J = s.m.e_jac[e];
    const double* tgt = &U[e * NEQ * nb];
    double neighbour_area = 0.0;
    std::fill(recon.begin(), recon.end(), 0.0);
    for (int i = 0; i < 3; ++i) {
      const int64_t di = s.m.e_edge[3 * e + i];
      if (s.m.d_elem[2 * di + 1] == -1) continue;
      const int64_t inb = s.m.e_nbr[3 * e + i];
      neighbour_area += s.m.e_jac[inb] * 0.5;
      double nlw[4][NEQ] = {};
      std::fill(proj.begin(), proj.end(), 0.0);
      const double nx = s.m.d_normal[2 * di], ny = s.m.d_normal[2 * di + 1];
      double mean[4];
      for (int v = 0; v < NEQ; ++v) mean[v] = tgt[v * nb + 0];
      double Lm[4][4], Rm[4][4];
      eigenmatrix(mean, nx, ny, s.hcr, Lm, Rm);
      // proj_pols[0] = L . tgt_pol (weno.rs:124)
      for (int r = 0; r < NEQ; ++r)
        for (int b = 0; b < nb; ++b) {
          double sum = 0.0;
          for (int k = 0; k < NEQ; ++k) sum = sum + Lm[r][k] * tgt[k * nb + b];
          proj[(0 * NEQ + r) * nb + b] = sum;
        }
      for (int v = 0; v < NEQ; ++v) {
        const double beta = smoothness(s, dinv, J, &proj[(0 * NEQ + v) * nb]);
        nlw[0][v] = lw[0] / ((beta + F64_EPSILON) * (beta + F64_EPSILON));
      }
      for (int j = 0; j < 3; ++j) {
        const int64_t dj = s.m.e_edge[3 * e + j];
        if (s.m.d_elem[2 * dj + 1] == -1) continue;
        const int64_t jnb = s.m.e_nbr[3 * e + j];
        for (int v = 0; v < NEQ; ++v)
          for (int b = 0; b < nb; ++b) nbpol[v * nb + b] = U[(jnb * NEQ + v) * nb + b];
        for (int v = 0; v < NEQ; ++v) nbpol[v * nb + 0] = tgt[v * nb + 0];
        for (int r = 0; r < NEQ; ++r)
          for (int b = 0; b < nb; ++b) {
            double sum = 0.0;
            for (int k = 0; k < NEQ; ++k) sum = sum + Lm[r][k] * nbpol[k * nb + b];
            proj[((j + 1) * NEQ + r) * nb + b] = sum;
          }
        for (int v = 0; v < NEQ; ++v) {
          const double beta = smoothness(s, dinv, J, &proj[((j + 1) * NEQ + v) * nb]);
          nlw[j + 1][v] = lw[j + 1] / ((beta + F64_EPSILON) * (beta + F64_EPSILON));
        }
      }
      // normalise (weno.rs:180-186), combine (weno.rs:187-194)
      double den[NEQ];
      for (int v = 0; v < NEQ; ++v) {
        double sum = 0.0;
        for (int j = 0; j < 4; ++j) sum = sum + nlw[j][v];
        den[v] = sum;
      }
      std::fill(pol_new.begin(), pol_new.end(), 0.0);
      for (int v = 0; v < NEQ; ++v)
        for (int j = 0; j < 4; ++j) {
          const double w = nlw[j][v] / den[v];
          for (int b = 0; b < nb; ++b) pol_new[v * nb + b] += w * proj[(j * NEQ + v) * nb + b];
        }
      // back to conserved variables (weno.rs:195) and area weighting (weno.rs:196)
      const double anb = s.m.e_jac[inb];
      for (int r = 0; r < NEQ; ++r)
        for (int b = 0; b < nb; ++b) {
          double sum = 0.0;
          for (int k = 0; k < NEQ; ++k) sum = sum + Rm[r][k] * pol_new[k * nb + b];
          recon[r * nb + b] = recon[r * nb + b] + sum * anb * 0.5;
        }
    }
    for (int r = 0; r < NEQ * nb; ++r) recon[r] /= neighbour_area;
    std::memcpy(&U[e * NEQ * nb], recon.data(), sizeof(double) * NEQ * nb);  // weno.rs:263
  }
  s.last_troubled = troubled;
  return ORC_OK;
}

// compute_time_step, temporal_disc.rs:58-88
double compute_time_step(const Solver& s, const double* U) {
  const int nb = s.B.nb;
  double time_step = 1.0e10;
  for (int64_t e = 0; e < s.m.ne; ++e) {
    double rho = 0.0, rho_u = 0.0, rho_v = 0.0, rho_e = 0.0;
    for (int b = 0; b < nb; ++b) {
      rho += U[(e * NEQ + 0) * nb + b];
      rho_u += U[(e * NEQ + 1) * nb + b];
      rho_v += U[(e * NEQ + 2) * nb + b];
      rho_e += U[(e * NEQ + 3) * nb + b];
    }
    const double u = rho_u / rho;
    const double v = rho_v / rho;
    const double p = (s.hcr - 1.0) * (rho_e - 0.5 * rho * (u * u + v * v));
    const double c = std::sqrt(s.hcr * p / rho);
    const double speed = std::sqrt(u * u + v * v) + c;
    const double dx = s.m.e_hmin[e];
    const double dt = s.cfl * dx / speed;
    if (dt < time_step) time_step = dt;
  }
  return time_step;
}

int apply_limiter(Solver& s, double* U) {
  if (!s.limiter) {
    s.last_troubled = 0;
    return ORC_OK;
  }
  return weno(s, U);
}

// rk3, rk3.rs:7-26
int rk3(Solver& s, double* R, double* U, double dt) {
  const size_t n = SZ(s);
  s.tmp0.resize(n);
  s.tmp1.resize(n);
  int st;
  std::fill(R, R + n, 0.0);
  if ((st = compute_residuals(s, R, U))) return st;
  for (size_t i = 0; i < n; ++i) s.tmp0[i] = U[i] + dt * R[i];
  if ((st = apply_limiter(s, s.tmp0.data()))) return st;
  std::fill(R, R + n, 0.0);
  if ((st = compute_residuals(s, R, s.tmp0.data()))) return st;
  for (size_t i = 0; i < n; ++i) s.tmp1[i] = 0.75 * U[i] + 0.25 * (s.tmp0[i] + dt * R[i]);
  if ((st = apply_limiter(s, s.tmp1.data()))) return st;
  std::fill(R, R + n, 0.0);
  if ((st = compute_residuals(s, R, s.tmp1.data()))) return st;
  const double third = 1.0 / 3.0, two_thirds = 2.0 / 3.0;
  for (size_t i = 0; i < n; ++i) U[i] = third * U[i] + two_thirds * (s.tmp1[i] + dt * R[i]);
  return apply_limiter(s, U);
}

// Solver::set_initial_solution, solver.rs:45-79 (L2 projection of a uniform state)
void set_initial_solution(const Solver& s, const FreeStream& in, double* U) {
  const int nb = s.B.nb, nq = s.g.nq;
  const double sound_speed = std::sqrt(s.hcr * in.p / in.rho);
  const double a = in.aoa_deg * (M_PI / 180.0);
  const double xm = in.mach * std::cos(a), ym = in.mach * std::sin(a);
  const double xv = xm * sound_speed, yv = ym * sound_speed;
  const double te = in.p / (s.hcr - 1.0) + 0.5 * in.rho * (xv * xv + yv * yv);
  const double q[4] = {in.rho, in.rho * xv, in.rho * yv, te};
  std::fill(U, U + SZ(s), 0.0);
  for (int64_t e = 0; e < s.m.ne; ++e)
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b)
        for (int g = 0; g < nq; ++g)
          U[(e * NEQ + v) * nb + b] += 0.5 * s.m.e_jac[e] * s.g.cell_w[g] * q[v] * s.B.phi_cell[g * nb + b];
  for (int64_t e = 0; e < s.m.ne; ++e)
    for (int v = 0; v < NEQ; ++v)
      for (int b = 0; b < nb; ++b) U[(e * NEQ + v) * nb + b] /= s.B.mass[b] * 0.5 * s.m.e_jac[e];
}

}  // namespace

// ==========================================================================================
// C API (ctypes).  Test infrastructure only.
// ==========================================================================================
extern "C" {

struct orc_config {
  int32_t order;         // polynomial order p (reference: 2)
  int32_t ncell_gp;      // triangle rule size
  int32_t nedge_gp;      // interval rule size
  int32_t limiter;       // 1 = reference WENO, 0 = off
  int32_t threads;       // OpenMP threads for the parallel passes
  int32_t _pad;
  double hcr;            // ratio of specific heats
  double cfl;            // > 0: explicit; <= 0: initialization.rs:29-33 formula
  double final_time;
  int64_t final_step;
  double fs_aoa_deg, fs_mach, fs_rho, fs_p;      // freestream.json
  double in_aoa_deg, in_mach, in_rho, in_p;      // initial_solution.json
};

struct orc_raw_mesh {
  int64_t n_vertices;
  const double* xy;            // [nv][2]
  int32_t n_edge_blocks;
  const int64_t* edge_block_sizes;
  const int32_t* edge_block_types;  // 0 wall, 1 farfield
  const int64_t* edge_pairs;        // concatenated [n][2], 0-based
  int32_t n_tri_blocks;
  const int64_t* tri_block_sizes;
  const int64_t* tris;              // concatenated [n][3], 0-based
};

static int setup(Solver* s, const orc_config* c) {
  s->hcr = c->hcr;
  s->threads = c->threads;
  s->limiter = c->limiter;
  s->final_time = c->final_time;
  s->final_step = c->final_step;
  if (c->cfl > 0.0) {
    s->cfl = c->cfl;
  } else {  // initialization.rs:29-33
    const double vc = 1.0, p = (double)c->order;
    s->cfl = vc * 1.0 / ((2.0 * p + 1.0) * (1.0 + 4.0 / std::pow(p + 2.0, 2.0)));
  }
  s->init = FreeStream{c->in_aoa_deg, c->in_mach, c->in_rho, c->in_p};
  if (!make_gauss(c->ncell_gp, c->nedge_gp, s->g)) return ORC_BAD_ARG;
  if (c->order < 1 || c->order > 3) return ORC_BAD_ARG;
  make_basis(c->order, s->g, s->B);
  return ORC_OK;
}

void* orc_create_from_msh(const char* path, const orc_config* c, int32_t* status) {
  auto* s = new Solver();
  int st = setup(s, c);
  RawMesh raw;
  std::string err;
  if (!st) st = parse_gmsh(path, raw, err);
  if (!st) st = process_mesh(raw, FreeStream{c->fs_aoa_deg, c->fs_mach, c->fs_rho, c->fs_p}, c->hcr, s->m, err);
  if (st) {
    if (!err.empty()) std::fprintf(stderr, "oracle: %s\n", err.c_str());
    delete s;
    *status = st;
    return nullptr;
  }
  *status = ORC_OK;
  return s;
}

void* orc_create_from_raw(const orc_raw_mesh* r, const orc_config* c, int32_t* status) {
  auto* s = new Solver();
  int st = setup(s, c);
  RawMesh raw;
  raw.xy.assign(r->xy, r->xy + 2 * r->n_vertices);
  int64_t off = 0;
  for (int b = 0; b < r->n_edge_blocks; ++b) {
    EdgeBlock eb;
    eb.name = r->edge_block_types[b] == WALL ? "Wall" : "Farfield";
    eb.pairs.assign(r->edge_pairs + 2 * off, r->edge_pairs + 2 * (off + r->edge_block_sizes[b]));
    off += r->edge_block_sizes[b];
    raw.edge_blocks.push_back(eb);
  }
  off = 0;
  for (int b = 0; b < r->n_tri_blocks; ++b) {
    raw.tri_blocks.emplace_back(r->tris + 3 * off, r->tris + 3 * (off + r->tri_block_sizes[b]));
    off += r->tri_block_sizes[b];
  }
  std::string err;
  if (!st) st = process_mesh(raw, FreeStream{c->fs_aoa_deg, c->fs_mach, c->fs_rho, c->fs_p}, c->hcr, s->m, err);
  if (st) {
    delete s;
    *status = st;
    return nullptr;
  }
  *status = ORC_OK;
  return s;
}

void orc_destroy(void* h) { delete static_cast<Solver*>(h); }

// The Navier-Stokes residual (the reference's disabled NS calls, spatial_disc.rs:34-36) on or off.
void orc_set_viscous(void* h, int32_t enable, double prandtl_number, double gas_constant) {
  auto* s = static_cast<Solver*>(h);
  s->viscous = enable ? 1 : 0;
  s->prandtl_number = prandtl_number;
  s->gas_constant = gas_constant;
}

// sizes: ne, ned, nv, np, nb, nq, ng, n_internal_edges, n_internal_elements,
// n_boundary_elements, nkeys, max_order
void orc_sizes(void* h, int64_t* out) {
  auto* s = static_cast<Solver*>(h);
  out[0] = s->m.ne;
  out[1] = s->m.ned;
  out[2] = s->m.nv;
  out[3] = s->m.np;
  out[4] = s->B.nb;
  out[5] = s->g.nq;
  out[6] = s->g.ng;
  out[7] = (int64_t)s->m.internal_edges.size();
  out[8] = (int64_t)s->m.internal_elements.size();
  out[9] = (int64_t)s->m.boundary_elements.size();
  out[10] = s->B.nkeys;
  out[11] = s->B.max_order;
}

double orc_cfl(void* h) { return static_cast<Solver*>(h)->cfl; }

// Copy out a named array of the processed mesh or tables (for cross-checks in tests).
int32_t orc_get_array(void* h, const char* name, void* out) {
  auto* s = static_cast<Solver*>(h);
  const std::string n(name);
  auto cp_d = [&](const std::vector<double>& v) { std::memcpy(out, v.data(), v.size() * sizeof(double)); return 0; };
  auto cp_i = [&](const std::vector<int64_t>& v) { std::memcpy(out, v.data(), v.size() * sizeof(int64_t)); return 0; };
  if (n == "xy") return cp_d(s->m.xy);
  if (n == "elem_vertices") return cp_i(s->m.e_vert);
  if (n == "elem_edges") return cp_i(s->m.e_edge);
  if (n == "elem_neighbours") return cp_i(s->m.e_nbr);
  if (n == "elem_jacob_det") return cp_d(s->m.e_jac);
  if (n == "elem_circumradius") return cp_d(s->m.e_circ);
  if (n == "elem_minimum_height") return cp_d(s->m.e_hmin);
  if (n == "elem_dinv") return cp_d(s->m.e_dinv);
  if (n == "edge_elements") return cp_i(s->m.d_elem);
  if (n == "edge_vertices") return cp_i(s->m.d_vert);
  if (n == "edge_in_cell") return cp_i(s->m.d_icell);
  if (n == "edge_jacob_det") return cp_d(s->m.d_jac);
  if (n == "edge_normal") return cp_d(s->m.d_normal);
  if (n == "edge_patch") return cp_i(s->m.d_patch);
  if (n == "patch_quantity") return cp_d(s->m.p_q);
  if (n == "patch_type") {
    std::vector<int64_t> t(s->m.p_type.begin(), s->m.p_type.end());
    return cp_i(t);
  }
  if (n == "internal_edges") return cp_i(s->m.internal_edges);
  if (n == "internal_elements") return cp_i(s->m.internal_elements);
  if (n == "boundary_elements") return cp_i(s->m.boundary_elements);
  if (n == "cell_points") return cp_d(s->g.cell_pts);
  if (n == "cell_weights") return cp_d(s->g.cell_w);
  if (n == "edge_points") return cp_d(s->g.edge_pts);
  if (n == "edge_weights") return cp_d(s->g.edge_w);
  if (n == "phi_cell") return cp_d(s->B.phi_cell);
  if (n == "phi_edge") return cp_d(s->B.phi_edge);
  if (n == "dphi_cell") return cp_d(s->B.dphi_cell);
  if (n == "mass") return cp_d(s->B.mass);
  return ORC_BAD_ARG;
}

// Physical derivative table of one element, [nq][nb][nkeys] (mesh.rs:85-114).
void orc_element_dphi(void* h, int64_t e, double* out) {
  auto* s = static_cast<Solver*>(h);
  const int nq = s->g.nq, nb = s->B.nb, nk = s->B.nkeys;
  for (int q = 0; q < nq; ++q)
    for (int b = 0; b < nb; ++b)
      for (int k = 0; k < nk; ++k) out[((size_t)q * nb + b) * nk + k] = phys_deriv(s->B, &s->m.e_dinv[4 * e], q, b, k);
}

void orc_set_initial_solution(void* h, double* U) {
  auto* s = static_cast<Solver*>(h);
  set_initial_solution(*s, s->init, U);
}

int32_t orc_compute_residuals(void* h, double* R, const double* U) {
  return compute_residuals(*static_cast<Solver*>(h), R, U);
}

int32_t orc_apply_limiter(void* h, double* U, int64_t* troubled) {
  auto* s = static_cast<Solver*>(h);
  const int st = apply_limiter(*s, U);
  if (troubled) *troubled = s->last_troubled;
  return st;
}

// Jacobi (parallel-order) KXRCF flags of every element, without modifying U.
void orc_troubled_flags(void* h, const double* U, int8_t* flags) {
  auto* s = static_cast<Solver*>(h);
  for (int64_t e = 0; e < s->m.ne; ++e) flags[e] = modified_kxrcf(*s, U, e) ? 1 : 0;
}

double orc_compute_time_step(void* h, const double* U) { return compute_time_step(*static_cast<Solver*>(h), U); }

int32_t orc_rk3(void* h, double* R, double* U, double dt) { return rk3(*static_cast<Solver*>(h), R, U, dt); }

int64_t orc_err_where(void* h) { return static_cast<Solver*>(h)->err_where; }

// time_march, temporal_disc.rs:21-57 (without the per-step print and the VTK write).
// Advances from the solver's current time/step; returns the status of the first failure.
int32_t orc_time_march(void* h, double* R, double* U, double* t_out, int64_t* step_out) {
  auto* s = static_cast<Solver*>(h);
  while (s->current_step < s->final_step && s->current_time < s->final_time) {
    double dt = compute_time_step(*s, U);
    if (s->current_time + dt > s->final_time) dt = s->final_time - s->current_time;
    const int st = rk3(*s, R, U, dt);
    if (st) return st;
    s->current_time += dt;
    s->current_step += 1;
  }
  if (t_out) *t_out = s->current_time;
  if (step_out) *step_out = s->current_step;
  return ORC_OK;
}

void orc_reset_clock(void* h) {
  auto* s = static_cast<Solver*>(h);
  s->current_time = 0.0;
  s->current_step = 0;
}

void orc_set_threads(void* h, int32_t threads) { static_cast<Solver*>(h)->threads = threads; }

// Single-state kernels of the flux module, for known-answer tests.
int32_t orc_hllc(const double* lv, const double* rv, double nx, double ny, double hcr, double* flux) {
  return hllc(lv, rv, nx, ny, hcr, flux);
}
void orc_flux(const double* q, double hcr, double* f, double* g) { euler_flux(q, hcr, f, g); }
void orc_eigenmatrix(const double* q, double nx, double ny, double hcr, double* L, double* R) {
  double Lm[4][4], Rm[4][4];
  eigenmatrix(q, nx, ny, hcr, Lm, Rm);
  std::memcpy(L, Lm, sizeof(Lm));
  std::memcpy(R, Rm, sizeof(Rm));
}

}  // extern "C"
