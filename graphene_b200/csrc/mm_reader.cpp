// MatrixMarket coordinate reader, written from the public format description
// (NIST MatrixMarket exchange format). Replaces the reference's use of
// fast_matrix_market 1.7.6 (matrix/host/details/MatrixMarket.cpp:31-65):
// 1-based indices become 0-based, "pattern" entries get value 1, and
// symmetric / skew-symmetric files are expanded to general form (the mirror
// of an off-diagonal entry is appended), as fast_matrix_market's triplet
// reader does by default.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "host_matrix.hpp"

namespace gr {

namespace {

std::string lower(std::string s) {
  for (auto& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}

}  // namespace

Coo readMatrixMarket(const std::string& path, DType valueType) {
  std::ifstream in(path);
  if (!in.is_open()) fail(GR_EIO, "Failed to open file " + path);
  std::string line;
  if (!std::getline(in, line)) fail(GR_EPARSE, "empty MatrixMarket file");
  std::istringstream hs(line);
  std::string banner, object, format, field, symmetry;
  hs >> banner >> object >> format >> field >> symmetry;
  if (banner != "%%MatrixMarket") fail(GR_EPARSE, "missing %%MatrixMarket banner");
  object = lower(object);
  format = lower(format);
  field = lower(field);
  symmetry = lower(symmetry);
  if (object != "matrix") fail(GR_EPARSE, "unsupported MatrixMarket object " + object);
  if (format != "coordinate") fail(GR_EPARSE, "only coordinate MatrixMarket files are supported");
  if (field != "real" && field != "integer" && field != "pattern" && field != "double")
    fail(GR_EPARSE, "unsupported MatrixMarket field " + field);
  if (symmetry != "general" && symmetry != "symmetric" && symmetry != "skew-symmetric")
    fail(GR_EPARSE, "unsupported MatrixMarket symmetry " + symmetry);
  const bool pattern = field == "pattern";
  const bool sym = symmetry == "symmetric";
  const bool skew = symmetry == "skew-symmetric";
  // Size line (after comments).
  i64 nr = -1, nc = -1, nnz = -1;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '%') continue;
    std::istringstream ss(line);
    if (!(ss >> nr >> nc >> nnz)) fail(GR_EPARSE, "malformed MatrixMarket size line");
    break;
  }
  if (nr < 0 || nc < 0 || nnz < 0) fail(GR_EPARSE, "missing MatrixMarket size line");
  Coo coo;
  coo.nrows = nr;
  coo.ncols = nc;
  coo.row.reserve(sym || skew ? 2 * nnz : nnz);
  coo.col.reserve(coo.row.capacity());
  coo.val.reserve(coo.row.capacity());
  i64 read = 0;
  while (read < nnz && std::getline(in, line)) {
    if (line.empty() || line[0] == '%') continue;
    const char* p = line.c_str();
    char* end = nullptr;
    long long i = std::strtoll(p, &end, 10);
    if (end == p) fail(GR_EPARSE, "malformed MatrixMarket entry: " + line);
    p = end;
    long long j = std::strtoll(p, &end, 10);
    if (end == p) fail(GR_EPARSE, "malformed MatrixMarket entry: " + line);
    p = end;
    double v = 1.0;
    if (!pattern) {
      if (valueType == DType::F32) {
        float f = std::strtof(p, &end);
        v = static_cast<double>(f);
      } else {
        v = std::strtod(p, &end);
      }
      if (end == p) fail(GR_EPARSE, "malformed MatrixMarket value: " + line);
    }
    if (i < 1 || i > nr || j < 1 || j > nc) fail(GR_EPARSE, "MatrixMarket index out of range: " + line);
    coo.row.push_back(i - 1);
    coo.col.push_back(j - 1);
    coo.val.push_back(v);
    if ((sym || skew) && i != j) {
      coo.row.push_back(j - 1);
      coo.col.push_back(i - 1);
      coo.val.push_back(skew ? -v : v);
    }
    ++read;
  }
  if (read != nnz) fail(GR_EPARSE, "MatrixMarket file ends after " + std::to_string(read) + " of " +
                                       std::to_string(nnz) + " entries");
  return coo;
}

std::vector<double> readMatrixMarketVector(const std::string& path, DType valueType) {
  std::ifstream in(path);
  if (!in.is_open()) fail(GR_EIO, "Failed to open file " + path);
  std::string line;
  if (!std::getline(in, line)) fail(GR_EPARSE, "empty MatrixMarket file");
  std::istringstream hs(line);
  std::string banner, object, format, field;
  hs >> banner >> object >> format >> field;
  if (banner != "%%MatrixMarket") fail(GR_EPARSE, "missing %%MatrixMarket banner");
  object = lower(object);
  format = lower(format);
  field = lower(field);
  if (object != "matrix" && object != "vector") fail(GR_EPARSE, "unsupported MatrixMarket object " + object);
  if (format != "coordinate" && format != "array") fail(GR_EPARSE, "unsupported MatrixMarket format " + format);
  if (field != "real" && field != "integer" && field != "double")
    fail(GR_EPARSE, "unsupported MatrixMarket field for a vector: " + field);
  if (object == "matrix" && format == "coordinate") {
    // The first column of a coordinate matrix.
    in.close();
    const Coo coo = readMatrixMarket(path, valueType);
    std::vector<double> v(static_cast<size_t>(coo.nrows), 0.0);
    for (size_t k = 0; k < coo.val.size(); ++k)
      if (coo.col[k] == 0) v[static_cast<size_t>(coo.row[k])] = coo.val[k];
    return v;
  }
  auto parseValue = [&](const char*& p) {
    char* end = nullptr;
    double v;
    if (valueType == DType::F32) v = static_cast<double>(std::strtof(p, &end));
    else v = std::strtod(p, &end);
    if (end == p) fail(GR_EPARSE, "malformed MatrixMarket value: " + line);
    p = end;
    return v;
  };
  // Size line: "rows [cols]" (array), "rows entries" (vector coordinate).
  i64 a = -1, b = -1;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '%') continue;
    std::istringstream ss(line);
    if (!(ss >> a)) fail(GR_EPARSE, "malformed MatrixMarket size line");
    if (!(ss >> b)) b = -1;
    break;
  }
  if (a < 0) fail(GR_EPARSE, "missing MatrixMarket size line");
  const bool coordinate = format == "coordinate";
  if (coordinate && b < 0) fail(GR_EPARSE, "MatrixMarket vector coordinate file needs rows and entries");
  std::vector<double> v(static_cast<size_t>(a), 0.0);
  // Entries to read: coordinate, b (index value) pairs; array, the first
  // column of a rows x cols matrix (column-major) or the rows of a vector.
  const i64 count = coordinate ? b : a;
  i64 read = 0;
  while (read < count && std::getline(in, line)) {
    if (line.empty() || line[0] == '%') continue;
    const char* p = line.c_str();
    if (coordinate) {
      char* end = nullptr;
      const long long i = std::strtoll(p, &end, 10);
      if (end == p) fail(GR_EPARSE, "malformed MatrixMarket entry: " + line);
      p = end;
      const double val = parseValue(p);
      if (i < 1 || i > a) fail(GR_EPARSE, "MatrixMarket index out of range: " + line);
      v[static_cast<size_t>(i - 1)] = val;
    } else {
      v[static_cast<size_t>(read)] = parseValue(p);
    }
    ++read;
  }
  if (read != count) fail(GR_EPARSE, "MatrixMarket file ends after " + std::to_string(read) + " of " +
                                       std::to_string(count) + " entries");
  return v;
}

}  // namespace gr
