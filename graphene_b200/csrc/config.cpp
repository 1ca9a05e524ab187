// JSON(C) reader and solver configuration tree. See config.hpp.
#include "config.hpp"

#include <cctype>
#include <cstdlib>
#include <set>

namespace gr {

namespace {

class Reader {
 public:
  explicit Reader(const std::string& s) : s_(s) {}

  Json document() {
    Json v = value();
    skip();
    if (i_ != s_.size()) error("trailing characters");
    return v;
  }

 private:
  const std::string& s_;
  size_t i_ = 0;

  [[noreturn]] void error(const std::string& what) const {
    fail(GR_EPARSE, "JSON parse error at offset " + std::to_string(i_) + ": " + what);
  }
  void skip() {
    for (;;) {
      while (i_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[i_]))) ++i_;
      if (i_ + 1 < s_.size() && s_[i_] == '/' && s_[i_ + 1] == '/') {
        while (i_ < s_.size() && s_[i_] != '\n') ++i_;
      } else if (i_ + 1 < s_.size() && s_[i_] == '/' && s_[i_ + 1] == '*') {
        size_t e = s_.find("*/", i_ + 2);
        if (e == std::string::npos) error("unterminated comment");
        i_ = e + 2;
      } else {
        return;
      }
    }
  }
  bool match(const char* lit) {
    size_t n = std::char_traits<char>::length(lit);
    if (s_.compare(i_, n, lit) == 0) {
      i_ += n;
      return true;
    }
    return false;
  }
  std::string str() {
    if (s_[i_] != '"') error("expected string");
    ++i_;
    std::string out;
    while (i_ < s_.size() && s_[i_] != '"') {
      char c = s_[i_++];
      if (c == '\\') {
        if (i_ >= s_.size()) error("bad escape");
        char e = s_[i_++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': {
            if (i_ + 4 > s_.size()) error("bad \\u escape");
            unsigned cp = std::strtoul(s_.substr(i_, 4).c_str(), nullptr, 16);
            i_ += 4;
            if (cp < 0x80) out += static_cast<char>(cp);
            else if (cp < 0x800) { out += static_cast<char>(0xC0 | (cp >> 6)); out += static_cast<char>(0x80 | (cp & 0x3F)); }
            else { out += static_cast<char>(0xE0 | (cp >> 12)); out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F)); out += static_cast<char>(0x80 | (cp & 0x3F)); }
            break;
          }
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (i_ >= s_.size()) error("unterminated string");
    ++i_;
    return out;
  }
  Json value() {
    skip();
    if (i_ >= s_.size()) error("unexpected end of input");
    Json v;
    char c = s_[i_];
    if (c == '{') {
      v.kind = Json::Object;
      ++i_;
      skip();
      if (i_ < s_.size() && s_[i_] == '}') { ++i_; return v; }
      for (;;) {
        skip();
        std::string k = str();
        skip();
        if (i_ >= s_.size() || s_[i_] != ':') error("expected ':'");
        ++i_;
        v.members.emplace_back(std::move(k), value());
        skip();
        if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
        if (i_ < s_.size() && s_[i_] == '}') { ++i_; break; }
        error("expected ',' or '}'");
      }
    } else if (c == '[') {
      v.kind = Json::Array;
      ++i_;
      skip();
      if (i_ < s_.size() && s_[i_] == ']') { ++i_; return v; }
      for (;;) {
        v.items.push_back(value());
        skip();
        if (i_ < s_.size() && s_[i_] == ',') { ++i_; continue; }
        if (i_ < s_.size() && s_[i_] == ']') { ++i_; break; }
        error("expected ',' or ']'");
      }
    } else if (c == '"') {
      v.kind = Json::String;
      v.text = str();
    } else if (match("true")) {
      v.kind = Json::Bool;
      v.text = "true";
    } else if (match("false")) {
      v.kind = Json::Bool;
      v.text = "false";
    } else if (match("null")) {
      v.kind = Json::Null;
    } else {
      size_t b = i_;
      while (i_ < s_.size() && (std::isdigit(static_cast<unsigned char>(s_[i_])) || s_[i_] == '-' ||
                                s_[i_] == '+' || s_[i_] == '.' || s_[i_] == 'e' || s_[i_] == 'E'))
        ++i_;
      if (b == i_) error("unexpected character");
      v.kind = Json::Number;
      v.text = s_.substr(b, i_ - b);
    }
    return v;
  }
};

// Typed field readers in the manner of boost::property_tree::get_optional:
// the value's text is converted; an unconvertible value is an error.
bool readFloat(const Json& j, const char* key, float& dst) {
  const Json* v = j.find(key);
  if (!v) return false;
  char* end = nullptr;
  float f = std::strtof(v->text.c_str(), &end);
  if (v->text.empty() || *end != '\0') fail(GR_EPARSE, std::string("field ") + key + " is not a number");
  dst = f;
  return true;
}
bool readInt(const Json& j, const char* key, int& dst) {
  const Json* v = j.find(key);
  if (!v) return false;
  char* end = nullptr;
  long x = std::strtol(v->text.c_str(), &end, 10);
  if (v->text.empty() || *end != '\0') fail(GR_EPARSE, std::string("field ") + key + " is not an integer");
  dst = static_cast<int>(x);
  return true;
}
bool readBool(const Json& j, const char* key, bool& dst) {
  const Json* v = j.find(key);
  if (!v) return false;
  if (v->text == "true" || v->text == "1") dst = true;
  else if (v->text == "false" || v->text == "0") dst = false;
  else fail(GR_EPARSE, std::string("field ") + key + " is not a boolean");
  return true;
}
// solver/Configuration.cpp:52-78
void readMultiColor(const Json& j, const char* key, MultiColorMode& dst) {
  const Json* v = j.find(key);
  if (!v) return;
  const std::string& s = v->text;
  if (s == "true" || s == "on") dst = MultiColorMode::On;
  else if (s == "false" || s == "off") dst = MultiColorMode::Off;
  else if (s == "auto") dst = MultiColorMode::Auto;
  else
    fail(GR_EPARSE, std::string("Invalid value for MultiColorMode field ") + key + ": " + s +
                        ". Allowed values are true, false, on, off or \"auto\"");
}
// common/Type.cpp parseType
int parseTypeName(const std::string& s) {
  if (s == "float32" || s == "float") return GR_FLOAT32;
  if (s == "float64" || s == "double") return GR_FLOAT64;
  if (s == "twofloat32") return GR_TWOFLOAT32;
  fail(GR_EPARSE, "Unknown type in config: " + s);
}
// matrix/Norm.cpp:24-47
int parseNorm(const std::string& s) {
  if (s == "L1") return GR_NORM_L1;
  if (s == "LINF") return GR_NORM_LINF;
  if (s == "L2") return GR_NORM_L2;
  fail(GR_EPARSE, "Invalid norm: " + s);
}

}  // namespace

const Json* Json::find(const std::string& key) const {
  for (auto& [k, v] : members)
    if (k == key) return &v;
  return nullptr;
}

Json Json::parse(const std::string& src) { return Reader(src).document(); }

std::string SolverConfig::solverName() const {
  if (type == "PBiCGStab") return preconditioner ? "PBiCGStab(" + preconditioner->solverName() + ")" : "BiCGStab";
  if (type == "ILU") return diagonalBased ? "DILU" : "ILU(0)";
  if (type == "GaussSeidel") return "GaussSeidel";
  if (type == "IterativeRefinement") return "IterativeRefinement(" + innerSolver->solverName() + ")";
  if (type == "restarter") return "Restarter of " + innerSolver->solverName();
  return type;
}

std::unique_ptr<SolverConfig> SolverConfig::fromJson(const Json& j) {
  if (j.kind != Json::Object) fail(GR_EPARSE, "a solver configuration must be a JSON object");
  const Json* t = j.find("type");
  if (!t) fail(GR_EPARSE, "No solver type specified in configuration");
  auto c = std::make_unique<SolverConfig>();
  c->type = t->text;
  std::set<std::string> known = {"type"};
  auto mark = [&](const char* k) { known.insert(k); };
  const std::string& ty = c->type;
  const bool stats = ty == "PBiCGStab" || ty == "GaussSeidel" || ty == "IterativeRefinement";
  if (stats) {
    for (const char* k : {"absTolerance", "relTolerance", "relResidual", "maxIterations", "minIterations",
                          "printPerformanceAfterSolve", "printPerformanceEachIteration", "norm"})
      mark(k);
    readFloat(j, "absTolerance", c->absTolerance);
    readFloat(j, "relTolerance", c->relTolerance);
    readFloat(j, "relResidual", c->relResidual);
    readInt(j, "maxIterations", c->maxIterations);
    readInt(j, "minIterations", c->minIterations);
    readBool(j, "printPerformanceAfterSolve", c->printPerformanceAfterSolve);
    readBool(j, "printPerformanceEachIteration", c->printPerformanceEachIteration);
    if (const Json* v = j.find("norm")) c->norm = parseNorm(v->text);
  }
  if (ty == "PBiCGStab") {
    mark("verbose"); mark("workingType"); mark("preconditioner"); mark("reduce");
    if (const Json* v = j.find("reduce")) {
      if (v->text == "float64") c->reduceRef = false;
      else if (v->text == "f32_ref_order") c->reduceRef = true;
      else fail(GR_EPARSE, "PBiCGStab reduce must be \"float64\" or \"f32_ref_order\"");
    }
    readBool(j, "verbose", c->verbose);
    if (const Json* v = j.find("workingType")) c->workingType = parseTypeName(v->text);
    if (const Json* v = j.find("preconditioner")) c->preconditioner = fromJson(*v);
  } else if (ty == "ILU") {
    mark("solveMulticolor"); mark("factorizeMulticolor"); mark("diagonalBased"); mark("kernel");
    mark("ringLog2"); mark("prefetch"); mark("unroll"); mark("ringBytes"); mark("l2Ahead"); mark("tilesPerBlock");
    mark("compactRing"); mark("recordLevels"); mark("pairRows"); mark("warpsPerBlock"); mark("computeWarps");
    readInt(j, "warpsPerBlock", c->warpsPerBlock);
    readInt(j, "computeWarps", c->computeWarps);
    mark("waitingWarp");
    readBool(j, "waitingWarp", c->waitingWarp);
    mark("producerWarp");
    readBool(j, "producerWarp", c->producerWarp);
    if (c->computeWarps != 0 && c->computeWarps != 1 && c->computeWarps != 2 && c->computeWarps != 4 &&
        c->computeWarps != 8)
      fail(GR_EINVAL, "computeWarps must be 1, 2, 4 or 8");
    if (c->warpsPerBlock < 1 || c->warpsPerBlock > 8) fail(GR_EINVAL, "warpsPerBlock must be 1..8");
    readBool(j, "compactRing", c->compactRing);
    readBool(j, "pairRows", c->pairRows);
    readBool(j, "recordLevels", c->ringRecords);
    readInt(j, "tilesPerBlock", c->tilesPerBlock);
    if (c->tilesPerBlock < 0 || c->tilesPerBlock > 64) fail(GR_EINVAL, "tilesPerBlock must be 0 (default) or 1..64");
    readInt(j, "l2Ahead", c->l2Ahead);
    if (c->l2Ahead < -1 || c->l2Ahead > (1 << 24)) fail(GR_EINVAL, "l2Ahead must be -1 (default) or 0..16 MiB");
    if (const Json* v = j.find("ringBytes")) {
      c->ringBytes = std::stoll(v->text);
      if (c->ringBytes < 0 || c->ringBytes > 200 * 1024) fail(GR_EINVAL, "ringBytes must be 0 (default) or up to 204800");
    }
    readInt(j, "ringLog2", c->ringLog2);
    readInt(j, "prefetch", c->prefetchChunks);
    if (c->prefetchChunks < -1 || c->prefetchChunks > 64) fail(GR_EINVAL, "prefetch must be -1 (default) or 0..64");
    if (j.find("unroll")) {
      bool u = false;
      readBool(j, "unroll", u);
      c->unrollRows = u ? 1 : 0;
    }
    if (c->ringLog2 != 0 && (c->ringLog2 < 13 || c->ringLog2 > 17))
      fail(GR_EINVAL, "ringLog2 must be 0 (automatic) or between 13 and 17");
    readMultiColor(j, "solveMulticolor", c->solveMulticolor);
    readMultiColor(j, "factorizeMulticolor", c->factorizeMulticolor);
    readBool(j, "diagonalBased", c->diagonalBased);
    if (const Json* v = j.find("kernel")) {
      if (v->text == "auto") c->iluKernel = 0;
      else if (v->text == "tma") c->iluKernel = 1;
      else if (v->text == "levels") c->iluKernel = 2;
      else if (v->text == "warp") c->iluKernel = 3;
      else if (v->text == "ring") c->iluKernel = 4;
      else if (v->text == "wring") c->iluKernel = 5;
      else fail(GR_EPARSE, "ILU kernel must be \"auto\", \"ring\", \"wring\", \"warp\", \"tma\" or \"levels\"");
    }
  } else if (ty == "GaussSeidel") {
    mark("numSweeps"); mark("numFixedIterations"); mark("solveMulticolor"); mark("workingType");
    mark("seed"); mark("kernel"); mark("recordLevels"); mark("warpsPerBlock"); mark("halo"); mark("pairRows");
    readBool(j, "recordLevels", c->ringRecords);
    readBool(j, "pairRows", c->gsPairRows);
    if (const Json* v = j.find("halo")) {
      if (v->text == "stale") c->gsDropHalo = false;
      else if (v->text == "drop") c->gsDropHalo = true;
      else fail(GR_EPARSE, "GaussSeidel halo must be \"stale\" or \"drop\"");
    }
    readInt(j, "warpsPerBlock", c->warpsPerBlock);
    if (c->warpsPerBlock < 1 || c->warpsPerBlock > 8) fail(GR_EINVAL, "warpsPerBlock must be 1..8");
    if (const Json* v = j.find("kernel")) {
      if (v->text == "auto") c->gsKernel = 0;
      else if (v->text == "ring") c->gsKernel = 1;
      else if (v->text == "levels") c->gsKernel = 2;
      else if (v->text == "wring") c->gsKernel = 3;
      else fail(GR_EPARSE, "GaussSeidel kernel must be \"auto\", \"ring\", \"wring\" or \"levels\"");
    }
    readInt(j, "numSweeps", c->numSweeps);
    readInt(j, "numFixedIterations", c->numFixedIterations);
    readMultiColor(j, "solveMulticolor", c->solveMulticolor);
    if (const Json* v = j.find("workingType")) c->workingType = parseTypeName(v->text);
    if (const Json* v = j.find("seed")) {
      if (v->text == "b") c->gsSeedB = true;
      else if (v->text == "diag") c->gsSeedB = false;
      else fail(GR_EPARSE, "GaussSeidel seed must be \"b\" or \"diag\"");
    }
    if (c->numSweeps < 1) fail(GR_EINVAL, "numSweeps must be at least 1");
  } else if (ty == "IterativeRefinement") {
    mark("extendedPrecisionType"); mark("innerSolver");
    if (const Json* v = j.find("extendedPrecisionType")) c->extendedPrecisionType = parseTypeName(v->text);
    const Json* in = j.find("innerSolver");
    if (!in) fail(GR_EPARSE, "IterativeRefinement requires an innerSolver configuration");
    c->innerSolver = fromJson(*in);
  } else if (ty == "restarter") {
    mark("maxRestarts"); mark("innerSolver");
    readInt(j, "maxRestarts", c->maxRestarts);
    const Json* in = j.find("innerSolver");
    if (!in) fail(GR_EPARSE, "Restarter requires an innerSolver configuration");
    c->innerSolver = fromJson(*in);
  } else {
    fail(GR_EPARSE, "Unknown solver: " + ty);
  }
  for (auto& [k, v] : j.members)
    if (!known.count(k)) c->unknownKeys.push_back(k);
  return c;
}

std::unique_ptr<SolverConfig> SolverConfig::fromText(const std::string& text) {
  return fromJson(Json::parse(text));
}

}  // namespace gr
