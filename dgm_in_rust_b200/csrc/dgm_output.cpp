// Result output in the reference's format, native: write_to_vtk (src/io/write_results.rs:8-93).
//
// The reference writes one legacy ASCII VTK file through the vtkio crate: the vertices as points
// (z = 0), the triangles, and three cell attributes from each element's mode-0 coefficients --
// Density, Velocity (u, v, 0) and Pressure.  The text follows vtkio's legacy writer: an empty
// title, each data block on one line, one cell type per line, an empty POINT_DATA block.  Numbers
// are printed as Rust's `{}` prints an f64: the shortest digits that read back to the same value,
// in positional notation (never an exponent), without a trailing ".0", and "NaN", "inf", "-inf".
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "dgm_b200.h"

namespace {

// Rust's Display of an f64 appended to out.
void put_f64(std::string& out, double x) {
  if (x != x) {
    out += "NaN";
    return;
  }
  if (x == __builtin_inf()) {
    out += "inf";
    return;
  }
  if (x == -__builtin_inf()) {
    out += "-inf";
    return;
  }
  char buf[64];
  // shortest round-trip digits, scientific: [-]d[.ddd]e(+|-)XX
  const std::to_chars_result r = std::to_chars(buf, buf + sizeof(buf), x, std::chars_format::scientific);
  const char* p = buf;
  if (*p == '-') {
    out += '-';
    ++p;
  }
  char digits[32];
  int nd = 0;
  const char* q = p;
  for (; q < r.ptr && *q != 'e'; ++q)
    if (*q != '.') digits[nd++] = *q;
  int exp10 = 0;
  std::from_chars(q + 1 + (q[1] == '+' ? 1 : 0), r.ptr, exp10);
  // value = 0.d1 d2 ... dn * 10^(exp10 + 1)
  if (exp10 >= 0) {
    const int int_digits = exp10 + 1;
    for (int i = 0; i < int_digits; ++i) out += i < nd ? digits[i] : '0';
    if (nd > int_digits) {
      out += '.';
      out.append(digits + int_digits, (size_t)(nd - int_digits));
    }
  } else {
    out += "0.";
    out.append((size_t)(-exp10 - 1), '0');
    out.append(digits, (size_t)nd);
  }
}

void put_i64(std::string& out, int64_t v) {
  char buf[32];
  const std::to_chars_result r = std::to_chars(buf, buf + sizeof(buf), v);
  out.append(buf, (size_t)(r.ptr - buf));
}

}  // namespace

extern "C" int32_t dgm_vtk_write(const char* path, int64_t n_vertices, const double* vertex_xy, int64_t n_elements,
                                 const int64_t* elem_vertices, const double* fields) {
  if (!path || n_vertices < 0 || n_elements < 0 || (n_vertices > 0 && !vertex_xy) ||
      (n_elements > 0 && (!elem_vertices || !fields)))
    return DGM_BAD_ARG;
  std::string s;
  try {
    s.reserve((size_t)(60 * n_vertices + 150 * n_elements + 512));
    auto line = [&s](const char* t) {
      s += t;
      s += '\n';
    };
    auto join = [&s](int64_t n, int stride, const double* a, int width, bool pad_zero) {
      // n rows of `width` values taken from rows of `stride` doubles, a trailing 0 when pad_zero
      bool first = true;
      for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < width + (pad_zero ? 1 : 0); ++k) {
          if (!first) s += ' ';
          first = false;
          put_f64(s, k < width ? a[i * stride + k] : 0.0);
        }
      }
      s += '\n';
    };
    line("# vtk DataFile Version 2.0");
    line("");
    line("ASCII");
    line("");
    line("DATASET UNSTRUCTURED_GRID");
    s += "POINTS ";
    put_i64(s, n_vertices);
    line(" double");
    join(n_vertices, 2, vertex_xy, 2, true);
    line("");
    s += "CELLS ";
    put_i64(s, n_elements);
    s += ' ';
    put_i64(s, 4 * n_elements);
    s += '\n';
    for (int64_t e = 0; e < n_elements; ++e) {
      if (e) s += ' ';
      s += "3 ";
      put_i64(s, elem_vertices[3 * e]);
      s += ' ';
      put_i64(s, elem_vertices[3 * e + 1]);
      s += ' ';
      put_i64(s, elem_vertices[3 * e + 2]);
    }
    s += '\n';
    line("");
    s += "CELL_TYPES ";
    put_i64(s, n_elements);
    s += '\n';
    for (int64_t e = 0; e < n_elements; ++e) line("5");  // VTK_TRIANGLE
    line("");
    line("");
    s += "POINT_DATA ";
    put_i64(s, n_vertices);
    s += '\n';
    line("");
    s += "CELL_DATA ";
    put_i64(s, n_elements);
    s += '\n';
    line("");
    line("SCALARS Density double 1");
    line("LOOKUP_TABLE default");
    join(n_elements, 4, fields, 1, false);
    line("");
    line("VECTORS Velocity double");
    join(n_elements, 4, fields + 1, 2, true);
    line("");
    line("SCALARS Pressure double 1");
    line("LOOKUP_TABLE default");
    join(n_elements, 4, fields + 3, 1, false);
    line("");
  } catch (...) {
    return DGM_OOM;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return DGM_BAD_ARG;
  const size_t w = std::fwrite(s.data(), 1, s.size(), f);
  const int c = std::fclose(f);
  return (w == s.size() && c == 0) ? DGM_OK : DGM_BAD_ARG;
}
