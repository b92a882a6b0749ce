// Value-preserving Matrix-Market reader (spgemm_read_mtx). The reference's
// readMTX (src/coo.cpp:110-173, kept behaviour-identical in host_coo.cpp)
// forces every value to 1.1, takes the first size token as the column count
// and misparses pattern files; this reader follows the format instead:
// "%%MatrixMarket matrix coordinate <field> <symmetry>", comment lines, a
// "rows cols entries" line, then one "row col [value]" line per entry with
// 1-based indices.
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/coo.h"
#include "../../include/spgemm_b200.h"

namespace {

std::string lower(std::string s) {
  for (char& ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}

// Reads one line of any length into `out` (without the newline); false at EOF.
bool read_line(FILE* f, std::string* out) {
  out->clear();
  int ch;
  bool any = false;
  while ((ch = fgetc(f)) != EOF) {
    any = true;
    if (ch == '\n') break;
    out->push_back((char)ch);
  }
  return any;
}

bool only_space(const std::string& s) {
  for (char ch : s)
    if (!std::isspace((unsigned char)ch)) return false;
  return true;
}

}  // namespace

extern "C" int spgemm_read_mtx(coo* out, const char* path) {
  if (!out || !path) return SPGEMM_ERR_INVALID;
  out->data = nullptr;
  out->nnz = out->num_rows = out->num_cols = 0;
  FILE* f = fopen(path, "r");
  if (!f) return SPGEMM_ERR_INVALID;
  std::string line;
  int status = SPGEMM_ERR_INVALID;
  triplet* data = nullptr;
  do {
    if (!read_line(f, &line)) break;
    char banner[64] = {0}, object[64] = {0}, format[64] = {0}, field[64] = {0}, symmetry[64] = {0};
    if (sscanf(line.c_str(), "%63s %63s %63s %63s %63s", banner, object, format, field, symmetry) != 5)
      break;
    if (lower(banner) != "%%matrixmarket" || lower(object) != "matrix" ||
        lower(format) != "coordinate")
      break;
    const std::string fld = lower(field), sym = lower(symmetry);
    const bool pattern = fld == "pattern";
    if (!pattern && fld != "real" && fld != "double" && fld != "integer") break;
    const bool general = sym == "general";
    const bool symmetric = sym == "symmetric" || sym == "hermitian";
    const bool skew = sym == "skew-symmetric";
    if (!general && !symmetric && !skew) break;
    // size line (after comments and blank lines)
    bool have_size = false;
    while (read_line(f, &line)) {
      if (line.empty() || line[0] == '%' || only_space(line)) continue;
      have_size = true;
      break;
    }
    if (!have_size) break;
    long long rows = -1, cols = -1, entries = -1;
    if (sscanf(line.c_str(), "%lld %lld %lld", &rows, &cols, &entries) != 3) break;
    if (rows < 0 || cols < 0 || entries < 0 || rows > 2147483647ll || cols > 2147483647ll) break;
    if (!general && rows != cols) break;
    const long long cap = entries * (general ? 1 : 2);
    if (cap > 2147483647ll) {
      status = SPGEMM_ERR_TOO_LARGE;
      break;
    }
    data = static_cast<triplet*>(malloc(sizeof(triplet) * (size_t)(cap > 0 ? cap : 1)));
    if (!data) {
      status = SPGEMM_ERR_ALLOC;
      break;
    }
    long long n = 0, read = 0;
    bool bad = false;
    while (read < entries && read_line(f, &line)) {
      if (line.empty() || line[0] == '%' || only_space(line)) continue;
      const char* p = line.c_str();
      char* end = nullptr;
      errno = 0;
      const long long r = strtoll(p, &end, 10);
      if (end == p) { bad = true; break; }
      p = end;
      const long long c = strtoll(p, &end, 10);
      if (end == p) { bad = true; break; }
      p = end;
      double v = 1.0;
      if (!pattern) {
        v = strtod(p, &end);
        if (end == p) { bad = true; break; }
      }
      if (errno == ERANGE || r < 1 || r > rows || c < 1 || c > cols) { bad = true; break; }
      data[n].ridx = (int)(r - 1);
      data[n].cidx = (int)(c - 1);
      data[n].val = (float)v;
      ++n;
      ++read;
      if (!general && r != c) {
        data[n].ridx = (int)(c - 1);
        data[n].cidx = (int)(r - 1);
        data[n].val = skew ? -(float)v : (float)v;
        ++n;
      } else if (skew && r == c) {
        bad = true;  // a skew-symmetric matrix has a zero diagonal, which is not stored
        break;
      }
    }
    if (bad || read != entries) break;  // malformed or truncated
    out->data = data;
    out->nnz = (int)n;
    out->num_rows = (int)rows;
    out->num_cols = (int)cols;
    data = nullptr;
    status = SPGEMM_OK;
  } while (false);
  free(data);
  fclose(f);
  return status;
}
