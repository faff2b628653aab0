// Matrix Market reader for the solver's inputs: the reference drivers read
// their matrices and right-hand sides with cusp::io::read_matrix_market_file
// (examples/driver_mm.cu); this is the host-side replacement behind the C ABI.
//
// Matrices: "coordinate" with real / integer / pattern values and general /
// symmetric / skew-symmetric storage, returned as CSR with rows and the
// columns inside every row sorted; duplicate entries are summed.  Vectors:
// "array" (one column) or "coordinate" real / integer.
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sap_b200.h"

namespace {

std::string g_mm_error;

struct MMFile {
  std::vector<char> buf;
  size_t pos = 0;
  bool load(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize((size_t)std::max(len, 0L) + 1);
    const size_t got = len > 0 ? std::fread(buf.data(), 1, (size_t)len, f) : 0;
    std::fclose(f);
    buf[got] = 0;
    buf.resize(got + 1);
    return true;
  }
  // next line (without the newline); false at the end
  bool line(std::string& out) {
    if (pos + 1 >= buf.size()) return false;
    const size_t s = pos;
    while (pos + 1 < buf.size() && buf[pos] != '\n') pos++;
    out.assign(buf.data() + s, pos - s);
    if (pos + 1 < buf.size()) pos++;
    if (!out.empty() && out.back() == '\r') out.pop_back();
    return true;
  }
};

struct Header {
  bool coordinate = true, pattern = false, complex_ = false, symmetric = false, skew = false, hermitian = false;
  bool matrix = true;
};

std::string lower(std::string s) {
  for (char& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

bool parse_header(MMFile& f, Header& h, std::string& sizeline) {
  std::string ln;
  if (!f.line(ln)) { g_mm_error = "empty file"; return false; }
  ln = lower(ln);
  if (ln.rfind("%%matrixmarket", 0) != 0) { g_mm_error = "missing %%MatrixMarket banner"; return false; }
  char obj[64] = {0}, fmt[64] = {0}, field[64] = {0}, sym[64] = {0};
  if (std::sscanf(ln.c_str(), "%%%%matrixmarket %63s %63s %63s %63s", obj, fmt, field, sym) < 3) {
    g_mm_error = "malformed banner";
    return false;
  }
  h.matrix = std::string(obj) == "matrix" || std::string(obj) == "vector";
  h.coordinate = std::string(fmt) == "coordinate";
  if (!h.coordinate && std::string(fmt) != "array") { g_mm_error = "unknown format"; return false; }
  const std::string fl(field), sy(sym);
  h.pattern = fl == "pattern";
  h.complex_ = fl == "complex";
  if (h.complex_) { g_mm_error = "complex matrices are not supported"; return false; }
  if (!(fl == "real" || fl == "integer" || fl == "double" || h.pattern)) { g_mm_error = "unknown field"; return false; }
  h.symmetric = sy == "symmetric";
  h.skew = sy == "skew-symmetric";
  h.hermitian = sy == "hermitian";
  while (f.line(ln)) {
    size_t i = 0;
    while (i < ln.size() && std::isspace((unsigned char)ln[i])) i++;
    if (i == ln.size() || ln[i] == '%') continue;
    sizeline = ln;
    return true;
  }
  g_mm_error = "missing size line";
  return false;
}

struct Triplet {
  int r, c;
  double v;
};

}  // namespace

extern "C" {

const char* sap_mm_last_error(void) { return g_mm_error.c_str(); }

int sap_mm_read_csr(const char* path, int* n_rows, int* n_cols, int64_t* nnz, int* row_offsets, int* col_indices,
                    double* values) {
  if (!path || !n_rows || !n_cols || !nnz) { g_mm_error = "null argument"; return SAP_ERR_INVALID_ARGUMENT; }
  MMFile f;
  if (!f.load(path)) { g_mm_error = std::string("cannot open ") + path; return SAP_ERR_INVALID_ARGUMENT; }
  Header h;
  std::string sizeline;
  if (!parse_header(f, h, sizeline)) return SAP_ERR_INVALID_ARGUMENT;
  if (!h.coordinate) { g_mm_error = "a matrix must be in coordinate format"; return SAP_ERR_INVALID_ARGUMENT; }
  long long m = 0, n = 0, ne = 0;
  if (std::sscanf(sizeline.c_str(), "%lld %lld %lld", &m, &n, &ne) != 3 || m <= 0 || n <= 0 || ne < 0 ||
      m > 2147483647LL || n > 2147483647LL) {
    g_mm_error = "malformed size line";
    return SAP_ERR_INVALID_ARGUMENT;
  }
  std::vector<Triplet> t;
  t.reserve((size_t)ne * ((h.symmetric || h.skew || h.hermitian) ? 2 : 1));
  const char* p = f.buf.data() + f.pos;
  char* end = nullptr;
  for (long long k = 0; k < ne; k++) {
    const long long r = std::strtoll(p, &end, 10);
    if (end == p) { g_mm_error = "truncated entry list"; return SAP_ERR_INVALID_ARGUMENT; }
    p = end;
    const long long c = std::strtoll(p, &end, 10);
    if (end == p) { g_mm_error = "truncated entry list"; return SAP_ERR_INVALID_ARGUMENT; }
    p = end;
    double v = 1.0;
    if (!h.pattern) {
      v = std::strtod(p, &end);
      if (end == p) { g_mm_error = "missing value"; return SAP_ERR_INVALID_ARGUMENT; }
      p = end;
    }
    if (r < 1 || r > m || c < 1 || c > n) { g_mm_error = "entry index out of range"; return SAP_ERR_INVALID_ARGUMENT; }
    t.push_back({(int)(r - 1), (int)(c - 1), v});
    if ((h.symmetric || h.skew || h.hermitian) && r != c) t.push_back({(int)(c - 1), (int)(r - 1), h.skew ? -v : v});
  }
  std::sort(t.begin(), t.end(), [](const Triplet& a, const Triplet& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
  // sum duplicates
  size_t w = 0;
  for (size_t k = 0; k < t.size(); k++) {
    if (w > 0 && t[w - 1].r == t[k].r && t[w - 1].c == t[k].c) t[w - 1].v += t[k].v;
    else t[w++] = t[k];
  }
  t.resize(w);
  if (t.size() > 2147483647ULL) { g_mm_error = "too many entries for int32 indices"; return SAP_ERR_INVALID_ARGUMENT; }
  *n_rows = (int)m;
  *n_cols = (int)n;
  *nnz = (int64_t)t.size();
  if (row_offsets) {
    std::fill(row_offsets, row_offsets + m + 1, 0);
    for (const auto& e : t) row_offsets[e.r + 1]++;
    for (long long i = 0; i < m; i++) row_offsets[i + 1] += row_offsets[i];
  }
  if (col_indices)
    for (size_t k = 0; k < t.size(); k++) col_indices[k] = t[k].c;
  if (values)
    for (size_t k = 0; k < t.size(); k++) values[k] = t[k].v;
  return SAP_OK;
}

int sap_mm_read_vector(const char* path, int64_t* n, double* values) {
  if (!path || !n) { g_mm_error = "null argument"; return SAP_ERR_INVALID_ARGUMENT; }
  MMFile f;
  if (!f.load(path)) { g_mm_error = std::string("cannot open ") + path; return SAP_ERR_INVALID_ARGUMENT; }
  Header h;
  std::string sizeline;
  if (!parse_header(f, h, sizeline)) return SAP_ERR_INVALID_ARGUMENT;
  long long m = 0, cols = 0, ne = 0;
  const int got = std::sscanf(sizeline.c_str(), "%lld %lld %lld", &m, &cols, &ne);
  if (got < 2 || m <= 0 || cols != 1) { g_mm_error = "a vector must have one column"; return SAP_ERR_INVALID_ARGUMENT; }
  *n = m;
  if (!values) return SAP_OK;
  const char* p = f.buf.data() + f.pos;
  char* end = nullptr;
  if (!h.coordinate) {
    for (long long i = 0; i < m; i++) {
      values[i] = std::strtod(p, &end);
      if (end == p) { g_mm_error = "truncated vector"; return SAP_ERR_INVALID_ARGUMENT; }
      p = end;
    }
    return SAP_OK;
  }
  if (got != 3) { g_mm_error = "malformed size line"; return SAP_ERR_INVALID_ARGUMENT; }
  std::fill(values, values + m, 0.0);
  for (long long k = 0; k < ne; k++) {
    const long long r = std::strtoll(p, &end, 10);
    if (end == p) { g_mm_error = "truncated entry list"; return SAP_ERR_INVALID_ARGUMENT; }
    p = end;
    const long long c = std::strtoll(p, &end, 10);
    p = end;
    const double v = h.pattern ? 1.0 : std::strtod(p, &end);
    p = end;
    if (r < 1 || r > m || c != 1) { g_mm_error = "entry index out of range"; return SAP_ERR_INVALID_ARGUMENT; }
    values[r - 1] += v;
  }
  return SAP_OK;
}

}  // extern "C"
