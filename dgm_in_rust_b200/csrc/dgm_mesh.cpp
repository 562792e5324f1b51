// Host mesh ingest, native: the gmsh 4.1 ASCII reader GmshParser::parse
// (src/io/mesh_parser.rs:28-158), and process_mesh (src/initialization.rs:112-261) followed by the
// Mesh::compute_* geometry (src/mesh.rs:15-147), in passes linear in the mesh size.
//
// Conventions (all the reference's; the device kernels rely on them):
//   * boundary edges are numbered first, in the order of the line blocks' node pairs; internal
//     edges follow in order of first appearance over elements and their local edges, the local
//     edge k of a triangle being the node pair (v_k, v_{k+1 mod 3});
//   * a node pair is looked up unordered; among repeated boundary pairs the last one is found
//     (the reference's HashMap insert overwrites);
//   * element -> edge assignment (initialization.rs:181-201): a boundary edge takes the element
//     as ielements[0] and keeps ielements[1] = -1 (the element is then a boundary element); an
//     internal edge takes it as ielements[0] when the element's local vertex k is the edge's
//     first vertex, else as ielements[1]; in_cell_indices follow the same sides;
//   * geometry with the reference's expressions in its operation order (no contraction into
//     fused multiply-adds; the library is compiled with -ffp-contract=off), so the arrays are bit
//     for bit those of the reference's f64 code.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "dgm_b200.h"

struct dgm_gmsh;

struct dgm_mesh_build {
  int64_t ne = 0, ned = 0;
  std::vector<int64_t> elem_edges, elem_neighbours, edge_elements, edge_vertices, edge_in_cell;
  std::vector<int64_t> internal_edges, internal_elements, boundary_elements;
  std::vector<double> elem_jac, elem_circ, elem_hmin, edge_jac, edge_normal;
};

namespace {

// Unordered node pair -> edge id, bucketed by the pair's lower node: every node's bucket holds
// (higher node, edge id) of the pairs whose lower node it is.  Buckets are sized by counting
// beforehand and are scanned linearly (a few entries each); neighbouring elements touch nearby
// buckets, so the lookups stay cache friendly.
class EdgeMap {
 public:
  EdgeMap(int64_t nv, int64_t nbd, const int64_t* bpairs, int64_t ne, const int64_t* tris) : bucket_((size_t)nv) {
    for (int64_t d = 0; d < nbd; ++d) ++bucket_[(size_t)lo(bpairs[2 * d], bpairs[2 * d + 1])].fill;
    for (int64_t t = 0; t < ne; ++t)
      for (int k = 0; k < 3; ++k) ++bucket_[(size_t)lo(tris[3 * t + k], tris[3 * t + (k + 1) % 3])].fill;
    int64_t total = 0;
    for (Bucket& b : bucket_) {
      b.start = total;
      total += b.fill;
      b.fill = 0;
    }
    entry_.resize((size_t)total);
  }
  int64_t find(int64_t a, int64_t b) const {
    const Bucket& bk = bucket_[(size_t)lo(a, b)];
    const int64_t h = a < b ? b : a;
    for (int64_t i = bk.start, e = bk.start + bk.fill; i < e; ++i)
      if (entry_[(size_t)i].hi == h) return entry_[(size_t)i].id;
    return -1;
  }
  void put(int64_t a, int64_t b, int64_t id) {  // insert or overwrite
    Bucket& bk = bucket_[(size_t)lo(a, b)];
    const int64_t h = a < b ? b : a;
    for (int64_t i = bk.start, e = bk.start + bk.fill; i < e; ++i)
      if (entry_[(size_t)i].hi == h) {
        entry_[(size_t)i].id = id;
        return;
      }
    entry_[(size_t)(bk.start + bk.fill++)] = Entry{h, id};
  }

 private:
  struct Bucket {
    int64_t start = 0, fill = 0;
  };
  struct Entry {
    int64_t hi, id;
  };
  static int64_t lo(int64_t a, int64_t b) { return a < b ? a : b; }
  std::vector<Bucket> bucket_;
  std::vector<Entry> entry_;
};

int build(dgm_mesh_build& m, int64_t nv, const double* xy, int64_t nbd, const int64_t* bpairs, int64_t ne,
          const int64_t* tris) {
  for (int64_t i = 0; i < 2 * nbd; ++i)
    if (bpairs[i] < 0 || bpairs[i] >= nv) return DGM_BAD_ARG;
  for (int64_t i = 0; i < 3 * ne; ++i)
    if (tris[i] < 0 || tris[i] >= nv) return DGM_BAD_ARG;

  // ---- edge numbering (initialization.rs:139-180) ----
  EdgeMap map(nv, nbd, bpairs, ne, tris);
  m.edge_vertices.reserve((size_t)(2 * (nbd + 2 * ne)));
  for (int64_t d = 0; d < nbd; ++d) {
    m.edge_vertices.push_back(bpairs[2 * d]);
    m.edge_vertices.push_back(bpairs[2 * d + 1]);
    map.put(bpairs[2 * d], bpairs[2 * d + 1], d);
  }
  int64_t ned = nbd;
  m.ne = ne;
  m.elem_edges.resize((size_t)(3 * ne));
  for (int64_t t = 0; t < ne; ++t)
    for (int k = 0; k < 3; ++k) {
      const int64_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
      int64_t d = map.find(a, b);
      if (d < 0) {
        d = ned++;
        map.put(a, b, d);
        m.edge_vertices.push_back(a);
        m.edge_vertices.push_back(b);
        m.internal_edges.push_back(d);
      }
      m.elem_edges[3 * t + k] = d;
    }
  m.ned = ned;

  // ---- element -> edge assignment (initialization.rs:181-201) ----
  m.edge_elements.assign((size_t)(2 * ned), 0);
  m.edge_in_cell.assign((size_t)(2 * ned), 0);
  for (int64_t d = 0; d < nbd; ++d) {
    m.edge_elements[2 * d + 1] = -1;
    m.edge_in_cell[2 * d + 1] = -1;
  }
  std::vector<char> internal((size_t)ne, 1);
  for (int64_t t = 0; t < ne; ++t)
    for (int k = 0; k < 3; ++k) {
      const int64_t d = m.elem_edges[3 * t + k];
      int side;
      if (m.edge_elements[2 * d + 1] == -1) {
        side = 0;
        internal[t] = 0;
      } else {
        side = tris[3 * t + k] == m.edge_vertices[2 * d] ? 0 : 1;
      }
      m.edge_elements[2 * d + side] = t;
      m.edge_in_cell[2 * d + side] = k;
    }
  for (int64_t t = 0; t < ne; ++t) (internal[t] ? m.internal_elements : m.boundary_elements).push_back(t);

  // ---- edge geometry, mesh.rs:15-30 ----
  m.edge_jac.resize((size_t)ned);
  m.edge_normal.resize((size_t)(2 * ned));
  for (int64_t d = 0; d < ned; ++d) {
    const int64_t p = m.edge_vertices[2 * d], q = m.edge_vertices[2 * d + 1];
    const double edx = xy[2 * q] - xy[2 * p], edy = xy[2 * q + 1] - xy[2 * p + 1];
    const double len = std::sqrt(edx * edx + edy * edy);
    m.edge_jac[d] = len;
    m.edge_normal[2 * d] = edy / len;
    m.edge_normal[2 * d + 1] = -edx / len;
  }
  // ---- element geometry, mesh.rs:31-84 ----
  m.elem_jac.resize((size_t)ne);
  m.elem_circ.resize((size_t)ne);
  m.elem_hmin.resize((size_t)ne);
  for (int64_t t = 0; t < ne; ++t) {
    const int64_t i1 = tris[3 * t], i2 = tris[3 * t + 1], i3 = tris[3 * t + 2];
    const double x1 = xy[2 * i1], y1 = xy[2 * i1 + 1];
    const double x2 = xy[2 * i2], y2 = xy[2 * i2 + 1];
    const double x3 = xy[2 * i3], y3 = xy[2 * i3 + 1];
    const double jac = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
    const double a = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    const double b = std::sqrt((x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2));
    const double c = std::sqrt((x1 - x3) * (x1 - x3) + (y1 - y3) * (y1 - y3));
    const double s = (a + b + c) / 2.0;
    const double surface = 0.5 * jac;
    m.elem_jac[t] = jac;
    m.elem_circ[t] = a * b * c / (4.0 * std::sqrt(s * (s - a) * (s - b) * (s - c)));
    m.elem_hmin[t] = std::fmin(std::fmin(2.0 * surface / a, 2.0 * surface / b), 2.0 * surface / c);
  }
  // ---- set_neighbours, mesh.rs:133-147 ----
  m.elem_neighbours.assign((size_t)(3 * ne), -1);
  for (int64_t t = 0; t < ne; ++t)
    for (int k = 0; k < 3; ++k) {
      const int64_t d = m.elem_edges[3 * t + k];
      if (m.edge_elements[2 * d + 1] == -1) continue;
      const bool first = tris[3 * t + k] == m.edge_vertices[2 * d];
      m.elem_neighbours[3 * t + k] = first ? m.edge_elements[2 * d + 1] : m.edge_elements[2 * d];
    }
  return DGM_OK;
}

// ---- GmshParser::parse (mesh_parser.rs:28-158): the reference's line state machine ----
// Lines end at '\n' with one '\r' before it dropped (BufRead::lines); tokens are split at ASCII
// white space; integers are unsigned decimals (an optional '+'), reals whatever f64::from_str
// reads.  Where the reference unwraps a failed parse or lookup (a panic), this returns
// DGM_BAD_ARG.
struct GmshData {
  std::vector<double> xy;
  std::vector<std::string> edge_names;
  std::vector<std::vector<int64_t>> edge_pairs, elem_nodes;
};

bool parse_usize(const char* t, int64_t& out) {
  if (*t == '+') ++t;
  if (!*t) return false;
  uint64_t v = 0;
  for (; *t; ++t) {
    if (*t < '0' || *t > '9') return false;
    if (v > (UINT64_MAX - 9) / 10) return false;
    v = 10 * v + (uint64_t)(*t - '0');
  }
  if (v > (uint64_t)INT64_MAX) return false;
  out = (int64_t)v;
  return true;
}

bool parse_f64(const char* t, double& out) {
  // f64::from_str takes decimal and exponent forms, inf/infinity/nan, an optional sign; strtod
  // also reads hexadecimal forms, which f64::from_str rejects
  const char* u = (*t == '+' || *t == '-') ? t + 1 : t;
  if (u[0] == '0' && (u[1] == 'x' || u[1] == 'X')) return false;
  char* end = nullptr;
  out = std::strtod(t, &end);
  return end != t && *end == '\0';
}

bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

int parse_gmsh(const char* path, GmshData& g) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return DGM_BAD_ARG;
  std::vector<char> buf;
  if (std::fseek(f, 0, SEEK_END) == 0) {
    const long n = std::ftell(f);
    if (n > 0) buf.resize((size_t)n);
    std::fseek(f, 0, SEEK_SET);
  }
  const size_t got = buf.empty() ? 0 : std::fread(buf.data(), 1, buf.size(), f);
  std::fclose(f);
  if (got != buf.size()) return DGM_BAD_ARG;
  if (buf.empty() || buf.back() != '\n') buf.push_back('\n');  // a last line without a newline
  enum St { Standby, FirstPhys, Phys, FirstEnt, Ent, FirstNodes, Nodes, FirstElems, FirstBlock, EdgeBlock, ElemBlock };
  St st = Standby;
  std::map<int64_t, std::string> phys_names;
  std::map<int64_t, int64_t> ent_to_phys;
  int64_t line_count = 0, max_line_count = 0;
  std::vector<char*> tok;
  char* p = buf.data();
  char* const end = buf.data() + buf.size();
  while (p < end) {
    char* nl = static_cast<char*>(std::memchr(p, '\n', (size_t)(end - p)));
    if (!nl) break;
    char* line = p;
    char* lend = nl;
    p = nl + 1;
    if (lend > line && lend[-1] == '\r') --lend;
    *lend = '\0';
    const size_t len = (size_t)(lend - line);
    auto starts = [&](const char* pre) { const size_t n = std::strlen(pre); return len >= n && std::memcmp(line, pre, n) == 0; };
    if (starts("$End")) { st = Standby; continue; }
    if (starts("$PhysicalNames")) { st = FirstPhys; continue; }
    if (starts("$Entities")) { st = FirstEnt; continue; }
    if (starts("$Nodes")) { st = FirstNodes; continue; }
    if (starts("$Elements")) { st = FirstElems; continue; }
    if (st == Standby) continue;
    if (st == FirstPhys) { st = Phys; continue; }
    if (st == FirstEnt) { st = Ent; continue; }
    if (st == FirstElems) { st = FirstBlock; continue; }
    tok.clear();
    for (char* c = line; c < lend;) {
      while (c < lend && is_ws(*c)) ++c;
      if (c >= lend) break;
      tok.push_back(c);
      while (c < lend && !is_ws(*c)) ++c;
      *c = '\0';
      ++c;
    }
    int64_t a = 0, b = 0, c3 = 0;
    switch (st) {
      case Phys:
        if (tok.size() == 3) {
          if (!parse_usize(tok[1], a)) return DGM_BAD_ARG;
          const char* s0 = tok[2];
          const char* s1 = s0 + std::strlen(s0);
          while (s0 < s1 && *s0 == '"') ++s0;
          while (s1 > s0 && s1[-1] == '"') --s1;
          phys_names[a] = std::string(s0, s1);
        }
        break;
      case Ent:
        if (tok.size() >= 11) {
          if (!parse_usize(tok[0], a) || !parse_usize(tok[8], b)) return DGM_BAD_ARG;
          ent_to_phys[a] = b;
        }
        break;
      case FirstNodes:
        if (tok.size() < 2 || !parse_usize(tok[1], a)) return DGM_BAD_ARG;
        g.xy.reserve((size_t)(2 * std::min<int64_t>(a, (int64_t)1 << 24)));  // a hint only
        st = Nodes;
        break;
      case Nodes:
        if (tok.size() == 3) {
          double x, y;
          if (!parse_f64(tok[0], x) || !parse_f64(tok[1], y)) return DGM_BAD_ARG;
          g.xy.push_back(x);
          g.xy.push_back(y);
        }
        break;
      case FirstBlock: {
        int64_t dim, tag, num;
        if (tok.size() < 4 || !parse_usize(tok[0], dim) || !parse_usize(tok[1], tag) || !parse_usize(tok[3], num))
          return DGM_BAD_ARG;
        auto ip = ent_to_phys.find(tag);
        if (ip == ent_to_phys.end()) return DGM_BAD_ARG;
        auto in = phys_names.find(ip->second);
        if (in == phys_names.end()) return DGM_BAD_ARG;
        if (dim == 1) {
          g.edge_names.push_back(in->second);
          g.edge_pairs.emplace_back();
          g.edge_pairs.back().reserve((size_t)(2 * std::min<int64_t>(num, (int64_t)1 << 24)));
          st = EdgeBlock;
        }
        if (dim == 2) {
          g.elem_nodes.emplace_back();
          g.elem_nodes.back().reserve((size_t)(3 * std::min<int64_t>(num, (int64_t)1 << 24)));
          st = ElemBlock;
        }
        line_count = 0;
        max_line_count = num;
        break;
      }
      case EdgeBlock:
        ++line_count;
        if (tok.size() < 3 || !parse_usize(tok[1], a) || !parse_usize(tok[2], b) || a < 1 || b < 1) return DGM_BAD_ARG;
        g.edge_pairs.back().push_back(a - 1);
        g.edge_pairs.back().push_back(b - 1);
        if (line_count == max_line_count) st = FirstBlock;
        break;
      case ElemBlock:
        ++line_count;
        if (tok.size() < 4 || !parse_usize(tok[1], a) || !parse_usize(tok[2], b) || !parse_usize(tok[3], c3) ||
            a < 1 || b < 1 || c3 < 1)
          return DGM_BAD_ARG;
        g.elem_nodes.back().push_back(a - 1);
        g.elem_nodes.back().push_back(b - 1);
        g.elem_nodes.back().push_back(c3 - 1);
        if (line_count == max_line_count) st = FirstBlock;
        break;
      default:
        break;
    }
  }
  return DGM_OK;
}

}  // namespace

extern "C" {

dgm_mesh_build* dgm_mesh_process(int64_t n_vertices, const double* vertex_xy, int64_t n_boundary_edges,
                                 const int64_t* boundary_pairs, int64_t n_elements, const int64_t* elem_vertices,
                                 int32_t* status) {
  int32_t st = DGM_OK;
  dgm_mesh_build* m = nullptr;
  if (n_vertices < 1 || n_boundary_edges < 0 || n_elements < 1 || !vertex_xy || !elem_vertices ||
      (n_boundary_edges > 0 && !boundary_pairs) || n_vertices > (int64_t)1 << 31) {
    st = DGM_BAD_ARG;
  } else {
    m = new (std::nothrow) dgm_mesh_build();
    if (!m) {
      st = DGM_OOM;
    } else {
      try {
        st = build(*m, n_vertices, vertex_xy, n_boundary_edges, boundary_pairs, n_elements, elem_vertices);
      } catch (const std::bad_alloc&) {
        st = DGM_OOM;
      }
      if (st != DGM_OK) {
        delete m;
        m = nullptr;
      }
    }
  }
  if (status) *status = st;
  return m;
}

int32_t dgm_mesh_counts(const dgm_mesh_build* m, int64_t* n_edges, int64_t* n_internal_edges,
                        int64_t* n_internal_elements) {
  if (!m) return DGM_BAD_ARG;
  if (n_edges) *n_edges = m->ned;
  if (n_internal_edges) *n_internal_edges = (int64_t)m->internal_edges.size();
  if (n_internal_elements) *n_internal_elements = (int64_t)m->internal_elements.size();
  return DGM_OK;
}

int32_t dgm_mesh_fetch(const dgm_mesh_build* m, int64_t* elem_edges, int64_t* elem_neighbours,
                       double* elem_jacob_det, double* elem_circumradius, double* elem_minimum_height,
                       int64_t* edge_elements, int64_t* edge_vertices, int64_t* edge_in_cell, double* edge_jacob_det,
                       double* edge_normal, int64_t* internal_edges, int64_t* internal_elements,
                       int64_t* boundary_elements) {
  if (!m) return DGM_BAD_ARG;
  auto put = [](void* dst, const auto& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
  };
  put(elem_edges, m->elem_edges);
  put(elem_neighbours, m->elem_neighbours);
  put(elem_jacob_det, m->elem_jac);
  put(elem_circumradius, m->elem_circ);
  put(elem_minimum_height, m->elem_hmin);
  put(edge_elements, m->edge_elements);
  put(edge_vertices, m->edge_vertices);
  put(edge_in_cell, m->edge_in_cell);
  put(edge_jacob_det, m->edge_jac);
  put(edge_normal, m->edge_normal);
  put(internal_edges, m->internal_edges);
  put(internal_elements, m->internal_elements);
  put(boundary_elements, m->boundary_elements);
  return DGM_OK;
}

void dgm_mesh_free(dgm_mesh_build* m) { delete m; }

dgm_gmsh* dgm_gmsh_parse(const char* path, int32_t* status) {
  int32_t st = DGM_BAD_ARG;
  dgm_gmsh* g = nullptr;
  if (path) {
    auto* d = new (std::nothrow) GmshData();
    if (!d) {
      st = DGM_OOM;
    } else {
      try {
        st = parse_gmsh(path, *d);
      } catch (const std::bad_alloc&) {
        st = DGM_OOM;
      }
      if (st == DGM_OK) g = reinterpret_cast<dgm_gmsh*>(d);
      else delete d;
    }
  }
  if (status) *status = st;
  return g;
}

int32_t dgm_gmsh_counts(const dgm_gmsh* h, int64_t* n_vertices, int32_t* n_edge_blocks, int32_t* n_elem_blocks) {
  if (!h) return DGM_BAD_ARG;
  const GmshData& g = *reinterpret_cast<const GmshData*>(h);
  if (n_vertices) *n_vertices = (int64_t)(g.xy.size() / 2);
  if (n_edge_blocks) *n_edge_blocks = (int32_t)g.edge_pairs.size();
  if (n_elem_blocks) *n_elem_blocks = (int32_t)g.elem_nodes.size();
  return DGM_OK;
}

int32_t dgm_gmsh_vertices(const dgm_gmsh* h, double* xy) {
  if (!h || !xy) return DGM_BAD_ARG;
  const GmshData& g = *reinterpret_cast<const GmshData*>(h);
  if (!g.xy.empty()) std::memcpy(xy, g.xy.data(), g.xy.size() * sizeof(double));
  return DGM_OK;
}

int64_t dgm_gmsh_block_size(const dgm_gmsh* h, int32_t dim, int32_t i) {
  if (!h) return -1;
  const GmshData& g = *reinterpret_cast<const GmshData*>(h);
  if (dim == 1 && i >= 0 && (size_t)i < g.edge_pairs.size()) return (int64_t)(g.edge_pairs[(size_t)i].size() / 2);
  if (dim == 2 && i >= 0 && (size_t)i < g.elem_nodes.size()) return (int64_t)(g.elem_nodes[(size_t)i].size() / 3);
  return -1;
}

const char* dgm_gmsh_block_name(const dgm_gmsh* h, int32_t i) {
  if (!h) return nullptr;
  const GmshData& g = *reinterpret_cast<const GmshData*>(h);
  return (i >= 0 && (size_t)i < g.edge_names.size()) ? g.edge_names[(size_t)i].c_str() : nullptr;
}

int32_t dgm_gmsh_block(const dgm_gmsh* h, int32_t dim, int32_t i, int64_t* nodes) {
  if (!h || !nodes || dgm_gmsh_block_size(h, dim, i) < 0) return DGM_BAD_ARG;
  const GmshData& g = *reinterpret_cast<const GmshData*>(h);
  const std::vector<int64_t>& v = dim == 1 ? g.edge_pairs[(size_t)i] : g.elem_nodes[(size_t)i];
  if (!v.empty()) std::memcpy(nodes, v.data(), v.size() * sizeof(int64_t));
  return DGM_OK;
}

void dgm_gmsh_free(dgm_gmsh* h) { delete reinterpret_cast<GmshData*>(h); }

}  // extern "C"
