// CPU oracle for the graphene_b200 hot path -- TEST INFRASTRUCTURE ONLY.
//
// A plain restatement of the reference (esa-tu-darmstadt/graphene,
// libgraphene/matrix). Each function cites the reference file:line it
// follows. Compiled with -ffp-contract=off: every arithmetic operator rounds
// once, in the type the reference's expression has.
//
// Differences from the reference, all deliberate and shared with the GPU
// path:
//  - METIS is unavailable: row_to_tile is an input (raw part ids).
//  - Halo regions of a tile are ordered as a sequential run of the
//    reference's parallel tile loop produces them (source tile ascending,
//    then the source's region creation order); the reference's own order is
//    thread-timing dependent (CRSHostMatrix.cpp:310-346).
//  - No dummy 0 entries for tiles without off-diagonals (an IPU artefact of
//    empty tensors, CRSHostMatrix.cpp:423-428 and :508-512).
//  - Dot products and norms accumulate in FP64 (the reference reduces in the
//    vector type, dsl/tensor/Expression.cpp:729-769); scalars derived from
//    them (alpha, beta, omega) are rounded to the working type where a
//    vector update uses them.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <queue>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

thread_local std::string g_err;
int g_threads = 1;

struct OErr : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Runs f(t) for every tile, on g_threads host threads.
template <class F>
void forTiles(size_t P, F&& f) {
  if (g_threads <= 1 || P <= 1) {
    for (size_t t = 0; t < P; ++t) f(t);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  int nt = std::min<int>(g_threads, static_cast<int>(P));
  for (int i = 0; i < nt; ++i)
    pool.emplace_back([&] {
      for (;;) {
        size_t t = next.fetch_add(1);
        if (t >= P) break;
        f(t);
      }
    });
  for (auto& th : pool) th.join();
}

// ---- double-word arithmetic (Joldes, Muller, Popescu, ACM TOMS 2017) ----
struct DW {
  float h, l;
};
DW twoSum(float a, float b) {
  float s = a + b;
  float ap = s - b;
  float bp = s - ap;
  float da = a - ap;
  float db = b - bp;
  return {s, da + db};
}
DW fastTwoSum(float a, float b) {
  float s = a + b;
  float z = s - a;
  return {s, b - z};
}
DW twoProd(float a, float b) {
  float p = a * b;
  return {p, std::fmaf(a, b, -p)};
}
DW dwPlusFp(DW x, float y) {
  DW s = twoSum(x.h, y);
  float v = x.l + s.l;
  return fastTwoSum(s.h, v);
}
DW dwPlusDw(DW x, DW y) {
  DW s = twoSum(x.h, y.h);
  DW t = twoSum(x.l, y.l);
  float c = s.l + t.h;
  DW v = fastTwoSum(s.h, c);
  float w = t.l + v.l;
  return fastTwoSum(v.h, w);
}
DW dwTimesFp(DW x, float y) {
  DW c = twoProd(x.h, y);
  float cl3 = std::fmaf(x.l, y, c.l);
  return fastTwoSum(c.h, cl3);
}

// ---- minimal JSON(C) reader -------------------------------------------------
struct JVal {
  enum Kind { Null, Bool, Num, Str, Obj, Arr } kind = Null;
  bool b = false;
  std::string s;  // numbers keep their text, as a property tree does
  std::vector<std::pair<std::string, JVal>> obj;
  std::vector<JVal> arr;
  const JVal* get(const std::string& k) const {
    for (auto& [kk, v] : obj)
      if (kk == k) return &v;
    return nullptr;
  }
};

struct JParser {
  const char* p;
  const char* e;
  void ws() {
    for (;;) {
      while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
      if (p + 1 < e && p[0] == '/' && p[1] == '/') {
        while (p < e && *p != '\n') ++p;
      } else if (p + 1 < e && p[0] == '/' && p[1] == '*') {
        p += 2;
        while (p + 1 < e && !(p[0] == '*' && p[1] == '/')) ++p;
        p += 2;
      } else {
        break;
      }
    }
  }
  JVal parse() {
    ws();
    if (p >= e) throw OErr("json: unexpected end");
    JVal v;
    if (*p == '{') {
      v.kind = JVal::Obj;
      ++p;
      ws();
      if (*p == '}') { ++p; return v; }
      for (;;) {
        ws();
        JVal k = parse();
        if (k.kind != JVal::Str) throw OErr("json: key must be a string");
        ws();
        if (*p != ':') throw OErr("json: expected ':'");
        ++p;
        JVal val = parse();
        v.obj.emplace_back(k.s, std::move(val));
        ws();
        if (*p == ',') { ++p; continue; }
        if (*p == '}') { ++p; break; }
        throw OErr("json: expected ',' or '}'");
      }
    } else if (*p == '[') {
      v.kind = JVal::Arr;
      ++p;
      ws();
      if (*p == ']') { ++p; return v; }
      for (;;) {
        v.arr.push_back(parse());
        ws();
        if (*p == ',') { ++p; continue; }
        if (*p == ']') { ++p; break; }
        throw OErr("json: expected ',' or ']'");
      }
    } else if (*p == '"') {
      v.kind = JVal::Str;
      ++p;
      while (p < e && *p != '"') {
        if (*p == '\\') ++p;
        v.s += *p++;
      }
      ++p;
    } else if (!strncmp(p, "true", 4)) {
      v.kind = JVal::Bool; v.b = true; v.s = "true"; p += 4;
    } else if (!strncmp(p, "false", 5)) {
      v.kind = JVal::Bool; v.b = false; v.s = "false"; p += 5;
    } else if (!strncmp(p, "null", 4)) {
      p += 4;
    } else {
      v.kind = JVal::Num;
      const char* s = p;
      while (p < e && (isdigit(static_cast<unsigned char>(*p)) || *p == '-' || *p == '+' || *p == '.' ||
                       *p == 'e' || *p == 'E'))
        ++p;
      v.s.assign(s, p);
      if (v.s.empty()) throw OErr("json: bad value");
    }
    return v;
  }
};

// ---- solver configuration (matrix/solver/*/Configuration.cpp) -------------
struct Conf {
  std::string type;
  float absTolerance = 0, relTolerance = 0, relResidual = 0;
  int maxIterations = 2147483647, minIterations = 0;
  int norm = 1;             // L2
  int workingType = -1;     // -1: x.type()
  bool diagonalBased = false;
  int numSweeps = 1, numFixedIterations = 0;
  int extendedType = -1;    // -1: x.type(); 0 f32, 1 f64, 2 dw
  int maxRestarts = 1;
  int gsSeedB = 1;          // extension: 1 seeds Gauss-Seidel rows with b
  int gsDropHalo = 0;       // extension: 1 takes halo values as 0 ("halo": "drop")
  // extension: PBiCGStab dot products and norms in the reference's own
  // reduction order and operand type ("reduce": "f32_ref_order") instead of
  // FP64 accumulation ("float64", the default).
  bool reduceRef = false;
  std::unique_ptr<Conf> pre, inner;
};

int parseTypeName(const std::string& s) {
  if (s == "float32" || s == "float") return 0;
  if (s == "float64" || s == "double") return 1;
  if (s == "twofloat32") return 2;
  throw OErr("Unknown type in config: " + s);
}

std::unique_ptr<Conf> parseConf(const JVal& j) {
  if (j.kind != JVal::Obj) throw OErr("solver config must be an object");
  auto c = std::make_unique<Conf>();
  const JVal* t = j.get("type");
  if (!t) throw OErr("No solver type specified in configuration");
  c->type = t->s;
  auto f = [&](const char* k, float& dst) { if (auto v = j.get(k)) dst = std::stof(v->s); };
  auto i = [&](const char* k, int& dst) { if (auto v = j.get(k)) dst = std::stoi(v->s); };
  auto b = [&](const char* k, bool& dst) { if (auto v = j.get(k)) dst = (v->s == "true" || v->s == "1"); };
  f("absTolerance", c->absTolerance);
  f("relTolerance", c->relTolerance);
  f("relResidual", c->relResidual);
  i("maxIterations", c->maxIterations);
  i("minIterations", c->minIterations);
  i("numSweeps", c->numSweeps);
  i("numFixedIterations", c->numFixedIterations);
  i("maxRestarts", c->maxRestarts);
  b("diagonalBased", c->diagonalBased);
  if (auto v = j.get("norm")) {
    if (v->s == "L1") c->norm = 0;
    else if (v->s == "L2") c->norm = 1;
    else if (v->s == "LINF") c->norm = 2;
    else throw OErr("Invalid norm: " + v->s);
  }
  if (auto v = j.get("workingType")) c->workingType = parseTypeName(v->s);
  if (auto v = j.get("extendedPrecisionType")) c->extendedType = parseTypeName(v->s);
  if (auto v = j.get("seed")) c->gsSeedB = (v->s == "b") ? 1 : 0;
  if (auto v = j.get("halo")) c->gsDropHalo = (v->s == "drop") ? 1 : 0;
  if (auto v = j.get("reduce")) {
    if (v->s == "f32_ref_order") c->reduceRef = true;
    else if (v->s == "float64") c->reduceRef = false;
    else throw OErr("reduce must be \"float64\" or \"f32_ref_order\"");
  }
  if (auto v = j.get("preconditioner")) c->pre = parseConf(*v);
  if (auto v = j.get("innerSolver")) c->inner = parseConf(*v);
  if (c->type == "IterativeRefinement" && !c->inner)
    throw OErr("IterativeRefinement requires an innerSolver configuration");
  if (c->type == "restarter" && !c->inner) throw OErr("Restarter requires an innerSolver configuration");
  if (c->type != "PBiCGStab" && c->type != "ILU" && c->type != "GaussSeidel" &&
      c->type != "IterativeRefinement" && c->type != "restarter")
    throw OErr("Unknown solver: " + c->type);
  return c;
}

// ---- tile layout (DistributedTileLayout.hpp / .cpp) -----------------------
struct SepRegion {
  std::set<size_t> dst;
  size_t proc;
  std::vector<size_t> cells;
};
struct HaloRegion {
  SepRegion* src;
  std::vector<size_t> cells;
};
struct Tile {
  size_t id = 0;
  std::vector<size_t> interior;
  std::vector<std::unique_ptr<SepRegion>> sep;
  std::vector<std::unique_ptr<HaloRegion>> halo;
  std::vector<size_t> l2g;
  std::unordered_map<size_t, size_t> g2l;
  size_t nInterior() const { return interior.size(); }
  size_t nSep() const {
    size_t s = 0;
    for (auto& r : sep) s += r->cells.size();
    return s;
  }
  size_t nHalo() const {
    size_t s = 0;
    for (auto& r : halo) s += r->cells.size();
    return s;
  }
  // TilePartition::getSeperatorRegionTo (DistributedTileLayout.cpp:63-75)
  SepRegion& sepTo(const std::set<size_t>& d) {
    for (auto& r : sep)
      if (r->dst == d) return *r;
    sep.push_back(std::make_unique<SepRegion>(SepRegion{d, id, {}}));
    return *sep.back();
  }
  // TilePartition::getHaloRegionFrom (DistributedTileLayout.cpp:77-89)
  HaloRegion& haloFrom(SepRegion& s) {
    for (auto& r : halo)
      if (r->src == &s) return *r;
    halo.push_back(std::make_unique<HaloRegion>(HaloRegion{&s, {}}));
    return *halo.back();
  }
  // TilePartition::calculateRowMapping (DistributedTileLayout.cpp:91-126)
  void mapping() {
    for (size_t r : interior) l2g.push_back(r);
    for (auto& s : sep)
      for (size_t r : s->cells) l2g.push_back(r);
    for (auto& h : halo)
      for (size_t r : h->cells) l2g.push_back(r);
    for (size_t i = 0; i < l2g.size(); ++i) g2l[l2g[i]] = i;
  }
};

struct Local {
  std::vector<size_t> rowPtr, colInd;
  std::vector<double> off, diag;
  std::vector<size_t> color;
  size_t nColors = 0;
};

// A tile's LDU addressing in the reference's terms (LDUAddressing.hpp:42-91),
// over tile-local cell ids (halo cells included): local row c owns the faces
// [ownerStart[c], ownerStart[c+1]) (upper coefficient, x at upperAddr) and
// neighbours the faces neighbourColInd[s] for s in
// [neighbourStart[c], neighbourStart[c+1]) (lower coefficient lowerLosort[s],
// x at lowerAddr[face]). Faces owned by a halo cell are appended after the
// owned ones so that lowerAddr covers every face a row needs.
struct LocalLdu {
  std::vector<size_t> ownerStart, upperAddr, neighbourStart, neighbourColInd, lowerAddr;
  std::vector<double> upper, lowerLosort;
};

}  // namespace

struct or_matrix {
  int vt = 0;
  size_t n = 0, P = 0;
  std::vector<size_t> gRowPtr, gCol;
  std::vector<double> gOff, gDiag;
  std::vector<size_t> rowToTile;
  std::vector<Tile> tiles;
  std::vector<Local> loc;
  std::vector<size_t> tileStart;  // tile order without halo
  std::vector<size_t> haloStart;  // layout with halo
  size_t nWithHalo = 0;
  bool multicolor = false;
  bool ldu = false;
  std::vector<LocalLdu> lloc;
};

namespace {

double roundVT(int vt, double v) { return vt == 0 ? static_cast<double>(static_cast<float>(v)) : v; }

void buildMatrix(or_matrix& A, std::vector<std::tuple<size_t, size_t, double>> ent, size_t n,
                 size_t numTiles, const int32_t* raw) {
  A.n = n;
  // sortTripletMatrx (CoordinateFormat.cpp:29-40)
  std::sort(ent.begin(), ent.end(), [](const auto& a, const auto& b) {
    return std::tie(std::get<0>(a), std::get<1>(a)) < std::tie(std::get<0>(b), std::get<1>(b));
  });
  for (size_t i = 1; i < ent.size(); ++i)
    if (std::get<0>(ent[i]) == std::get<0>(ent[i - 1]) && std::get<1>(ent[i]) == std::get<1>(ent[i - 1]))
      throw OErr("duplicate entries");
  // convertToCRS (CRSHostMatrix.cpp:88-137)
  A.gDiag.assign(n, 0.0);
  for (auto& [r, c, v] : ent)
    if (r == c) A.gDiag[r] = v;
  A.gRowPtr.push_back(0);
  size_t lastRow = 0;
  for (auto& [r, c, v] : ent) {
    if (r == c) continue;
    while (lastRow != r) {
      A.gRowPtr.push_back(A.gCol.size());
      lastRow++;
    }
    A.gCol.push_back(c);
    A.gOff.push_back(v);
  }
  while (A.gRowPtr.size() <= n) A.gRowPtr.push_back(A.gCol.size());

  // Partitioning: single tile short-circuit (CRSHostMatrix.cpp:151-158),
  // otherwise empty-part removal (CRSHostMatrix.cpp:235-270).
  if (numTiles == 1) {
    A.P = 1;
    A.rowToTile.assign(n, 0);
  } else {
    std::vector<size_t> per(numTiles, 0);
    for (size_t i = 0; i < n; ++i) {
      if (raw[i] < 0 || static_cast<size_t>(raw[i]) >= numTiles) throw OErr("row_to_tile out of range");
      per[raw[i]]++;
    }
    size_t empty = 0;
    std::vector<long long> shift(numTiles);
    for (size_t i = 0; i < numTiles; ++i) {
      if (per[i] == 0) { ++empty; shift[i] = -1; continue; }
      shift[i] = static_cast<long long>(i - empty);
    }
    A.P = numTiles - empty;
    A.rowToTile.resize(n);
    for (size_t i = 0; i < n; ++i) A.rowToTile[i] = static_cast<size_t>(shift[raw[i]]);
  }

  // calculateTileLayouts (CRSHostMatrix.cpp:273-354), tiles processed in
  // order; each tile's rows in ascending order.
  const size_t P = A.P;
  A.tiles.resize(P);
  for (size_t t = 0; t < P; ++t) A.tiles[t].id = t;
  std::vector<std::vector<size_t>> rowsOf(P);
  for (size_t r = 0; r < n; ++r) rowsOf[A.rowToTile[r]].push_back(r);
  for (size_t t = 0; t < P; ++t) {
    Tile& tile = A.tiles[t];
    for (size_t row : rowsOf[t]) {
      std::set<size_t> nb;
      for (size_t i = A.gRowPtr[row]; i < A.gRowPtr[row + 1]; ++i)
        if (A.rowToTile[A.gCol[i]] != t) nb.insert(A.rowToTile[A.gCol[i]]);
      if (nb.empty()) {
        tile.interior.push_back(row);
      } else {
        SepRegion& own = tile.sepTo(nb);
        own.cells.push_back(row);
        for (size_t nt : nb) A.tiles[nt].haloFrom(own).cells.push_back(row);
      }
    }
  }
  for (auto& tile : A.tiles) tile.mapping();

  // calculateLocalAddressings (CRSHostMatrix.cpp:379-432) and the value
  // decomposition (CRSHostMatrix.cpp:434-525).
  A.loc.resize(P);
  for (size_t t = 0; t < P; ++t) {
    const Tile& tile = A.tiles[t];
    Local& L = A.loc[t];
    size_t nRows = tile.nInterior() + tile.nSep();
    for (size_t lr = 0; lr < nRows; ++lr) {
      L.rowPtr.push_back(L.colInd.size());
      size_t g = tile.l2g[lr];
      std::set<size_t> cols;
      std::set<std::pair<size_t, double>> vals;
      for (size_t i = A.gRowPtr[g]; i < A.gRowPtr[g + 1]; ++i) {
        size_t lc = tile.g2l.at(A.gCol[i]);
        cols.insert(lc);
        vals.insert({lc, A.gOff[i]});
      }
      L.colInd.insert(L.colInd.end(), cols.begin(), cols.end());
      for (auto& pv : vals) L.off.push_back(pv.second);
      L.diag.push_back(A.gDiag[g]);
    }
    L.rowPtr.push_back(L.colInd.size());
  }

  // calculateRowColors (CRSHostMatrix.cpp:527-614)
  for (size_t t = 0; t < P; ++t) {
    const Tile& tile = A.tiles[t];
    Local& L = A.loc[t];
    size_t numRows = tile.nInterior() + tile.nSep();
    L.color.assign(numRows, SIZE_MAX);
    std::queue<size_t> cur, next;
    std::vector<size_t> pending(numRows, 0);
    for (size_t lr = 0; lr < numRows; ++lr)
      for (size_t i = L.rowPtr[lr]; i < L.rowPtr[lr + 1]; ++i) {
        size_t lc = L.colInd[i];
        if (lc > lr) break;
        if (lc >= numRows) continue;
        ++pending[lr];
      }
    for (size_t lr = 0; lr < numRows; ++lr)
      if (pending[lr] == 0) next.push(lr);
    size_t color = 0;
    while (!next.empty()) {
      std::swap(cur, next);
      next = std::queue<size_t>();
      while (!cur.empty()) {
        size_t lr = cur.front();
        cur.pop();
        L.color[lr] = color;
        for (long long i = static_cast<long long>(L.rowPtr[lr + 1]) - 1;
             i >= static_cast<long long>(L.rowPtr[lr]); --i) {
          size_t lc = L.colInd[i];
          if (lc < lr) break;
          if (lc >= numRows) continue;
          if (--pending[lc] == 0) next.push(lc);
        }
      }
      ++color;
    }
    L.nColors = color;
  }
  // calculateColorAddressings recommendation (CRSHostMatrix.cpp:648-669)
  size_t par = 0, total = 0;
  for (size_t t = 0; t < P; ++t) {
    std::vector<size_t> sz(A.loc[t].nColors, 0);
    for (size_t c : A.loc[t].color)
      if (c != SIZE_MAX) sz[c]++;
    for (size_t s : sz) {
      total += s;
      if (s > 12) par += s;
    }
  }
  A.multicolor = par > 0.9 * total;

  A.tileStart.assign(P + 1, 0);
  A.haloStart.assign(P + 1, 0);
  for (size_t t = 0; t < P; ++t) {
    size_t nr = A.tiles[t].nInterior() + A.tiles[t].nSep();
    A.tileStart[t + 1] = A.tileStart[t] + nr;
    A.haloStart[t + 1] = A.haloStart[t] + nr + A.tiles[t].nHalo();
  }
  A.nWithHalo = A.haloStart[P];
}

// ---- vectors with halo ------------------------------------------------------
template <class T>
std::vector<T> withHalo(const or_matrix& A, const T* tileOrdered) {
  std::vector<T> v(A.nWithHalo, T());
  for (size_t t = 0; t < A.P; ++t) {
    size_t nr = A.tileStart[t + 1] - A.tileStart[t];
    for (size_t i = 0; i < nr; ++i) v[A.haloStart[t] + i] = tileOrdered[A.tileStart[t] + i];
  }
  return v;
}

template <class T>
void stripHalo(const or_matrix& A, const std::vector<T>& v, T* tileOrdered) {
  for (size_t t = 0; t < A.P; ++t) {
    size_t nr = A.tileStart[t + 1] - A.tileStart[t];
    for (size_t i = 0; i < nr; ++i) tileOrdered[A.tileStart[t] + i] = v[A.haloStart[t] + i];
  }
}

// MatrixBase::exchangeHaloCells (MatrixBase.cpp:36-109): each halo region
// receives the owner's current values.
template <class T>
void exchange(const or_matrix& A, std::vector<T>& v) {
  // Destination tiles write disjoint halo slots and read owned slots only.
  forTiles(A.P, [&](size_t t) {
    const Tile& dst = A.tiles[t];
    for (auto& h : dst.halo) {
      const Tile& src = A.tiles[h->src->proc];
      for (size_t g : h->cells)
        v[A.haloStart[t] + dst.g2l.at(g)] = v[A.haloStart[src.id] + src.g2l.at(g)];
    }
  });
}

// Conversion helpers mirroring Value::cast.
template <class T> T conv(double v) { return static_cast<T>(v); }

// CRSMatrix::spmv / residual (CRSMatrix.cpp:42-128): per tile, per row
// sum = diag * x[i], then sum += offDiag[j] * x[colInd[j]], in type I.
template <class V, class X, class I>
I rowSum(const Local& L, const std::vector<V>& off, const std::vector<V>& dg, const std::vector<X>& x,
         size_t hb, size_t i) {
  I sum = static_cast<I>(dg[i]) * static_cast<I>(x[hb + i]);
  for (size_t j = L.rowPtr[i]; j < L.rowPtr[i + 1]; ++j)
    sum += static_cast<I>(off[j]) * static_cast<I>(x[hb + L.colInd[j]]);
  return sum;
}

// Coefficients of each tile in the stored type (and, for LDU matrices, the
// upper and losort-ordered lower coefficients).
template <class V>
struct TileValues {
  std::vector<std::vector<V>> off, diag, up, lo;
  explicit TileValues(const or_matrix& A) : off(A.P), diag(A.P), up(A.P), lo(A.P) {
    for (size_t t = 0; t < A.P; ++t) {
      off[t].assign(A.loc[t].off.begin(), A.loc[t].off.end());
      diag[t].assign(A.loc[t].diag.begin(), A.loc[t].diag.end());
      if (A.ldu) {
        up[t].assign(A.lloc[t].upper.begin(), A.lloc[t].upper.end());
        lo[t].assign(A.lloc[t].lowerLosort.begin(), A.lloc[t].lowerLosort.end());
      }
    }
  }
};

// LDUMatrix::spmv / residual row loop (LDUMatrix.cpp:64-86, 128-152):
// sum = diag * x[c], then the owned faces in face order, then the
// neighbouring faces in losort order, in type I.
template <class V, class X, class I>
I rowSumLdu(const LocalLdu& L, const std::vector<V>& up, const std::vector<V>& lo, const std::vector<V>& dg,
            const std::vector<X>& x, size_t hb, size_t c) {
  I sum = static_cast<I>(dg[c]) * static_cast<I>(x[hb + c]);
  for (size_t f = L.ownerStart[c]; f < L.ownerStart[c + 1]; ++f)
    sum += static_cast<I>(up[f]) * static_cast<I>(x[hb + L.upperAddr[f]]);
  for (size_t s = L.neighbourStart[c]; s < L.neighbourStart[c + 1]; ++s) {
    const size_t face = L.neighbourColInd[s];
    sum += static_cast<I>(lo[s]) * static_cast<I>(x[hb + L.lowerAddr[face]]);
  }
  return sum;
}

template <class V, class X, class I>
I rowTotal(const or_matrix& A, const TileValues<V>& tv, size_t t, const std::vector<X>& x, size_t hb, size_t i) {
  if (A.ldu) return rowSumLdu<V, X, I>(A.lloc[t], tv.up[t], tv.lo[t], tv.diag[t], x, hb, i);
  return rowSum<V, X, I>(A.loc[t], tv.off[t], tv.diag[t], x, hb, i);
}

template <class V, class T>
void spmvT(const or_matrix& A, const TileValues<V>& tv, std::vector<T>& x, std::vector<T>& y) {
  exchange(A, x);
  forTiles(A.P, [&](size_t t) {
    size_t nr = A.tileStart[t + 1] - A.tileStart[t];
    for (size_t i = 0; i < nr; ++i)
      y[A.haloStart[t] + i] = rowTotal<V, T, T>(A, tv, t, x, A.haloStart[t], i);
  });
}

template <class V, class X, class B, class R, class I>
void residualT(const or_matrix& A, const TileValues<V>& tv, std::vector<X>& x, const std::vector<B>& b,
               std::vector<R>& r) {
  exchange(A, x);
  forTiles(A.P, [&](size_t t) {
    size_t nr = A.tileStart[t + 1] - A.tileStart[t];
    size_t hb = A.haloStart[t];
    for (size_t i = 0; i < nr; ++i) {
      I sum = rowTotal<V, X, I>(A, tv, t, x, hb, i);
      r[hb + i] = static_cast<R>(static_cast<I>(b[hb + i]) - sum);
    }
  });
}

// Residual with double-word intermediate (x double-word or float).
template <class X>
void residualDw(const or_matrix& A, const TileValues<float>& tv, std::vector<X>& x,
                const std::vector<float>& b, std::vector<float>& r) {
  exchange(A, x);
  auto asDw = [](const X& v) -> DW {
    if constexpr (std::is_same_v<X, DW>) return v;
    else return DW{static_cast<float>(v), 0.0f};
  };
  forTiles(A.P, [&](size_t t) {
    const Local& L = A.loc[t];
    size_t nr = A.tileStart[t + 1] - A.tileStart[t];
    size_t hb = A.haloStart[t];
    for (size_t i = 0; i < nr; ++i) {
      DW sum = dwTimesFp(asDw(x[hb + i]), tv.diag[t][i]);
      if (A.ldu) {
        const LocalLdu& D = A.lloc[t];
        for (size_t f = D.ownerStart[i]; f < D.ownerStart[i + 1]; ++f)
          sum = dwPlusDw(sum, dwTimesFp(asDw(x[hb + D.upperAddr[f]]), tv.up[t][f]));
        for (size_t s = D.neighbourStart[i]; s < D.neighbourStart[i + 1]; ++s)
          sum = dwPlusDw(sum, dwTimesFp(asDw(x[hb + D.lowerAddr[D.neighbourColInd[s]]]), tv.lo[t][s]));
      } else {
        for (size_t j = L.rowPtr[i]; j < L.rowPtr[i + 1]; ++j)
          sum = dwPlusDw(sum, dwTimesFp(asDw(x[hb + L.colInd[j]]), tv.off[t][j]));
      }
      DW res = dwPlusDw(DW{b[hb + i], 0.0f}, DW{-sum.h, -sum.l});
      r[hb + i] = res.h + res.l;
    }
  });
}

// Matrix::vectorNorm (MatrixBase.cpp:149-152, Tensor.cpp:425-439) on the
// non-halo cells, FP64 accumulation: a partial per tile (tiles in parallel),
// then the partials in tile order, so the result does not depend on the
// number of threads.
template <class T>
double normT(const or_matrix& A, const std::vector<T>& v, int norm) {
  std::vector<double> part(A.P);
  forTiles(A.P, [&](size_t t) {
    double acc = norm == 2 ? -INFINITY : 0.0;
    size_t nr = A.tileStart[t + 1] - A.tileStart[t];
    for (size_t i = 0; i < nr; ++i) {
      double x = static_cast<double>(v[A.haloStart[t] + i]);
      if (norm == 1) acc += x * x;
      else if (norm == 2) acc = std::max(acc, x);
      else acc += x;
    }
    part[t] = acc;
  });
  double acc = norm == 2 ? -INFINITY : 0.0;
  for (double p : part) acc = norm == 2 ? std::max(acc, p) : acc + p;
  return norm == 1 ? std::sqrt(acc) : acc;
}

template <class T>
double dotT(const or_matrix& A, const std::vector<T>& a, const std::vector<T>& b) {
  std::vector<double> part(A.P);
  forTiles(A.P, [&](size_t t) {
    double acc = 0.0;
    size_t nr = A.tileStart[t + 1] - A.tileStart[t];
    for (size_t i = 0; i < nr; ++i)
      acc += static_cast<double>(a[A.haloStart[t] + i]) * static_cast<double>(b[A.haloStart[t] + i]);
    part[t] = acc;
  });
  double acc = 0.0;
  for (double p : part) acc += p;
  return acc;
}

// Expression::reduce in the reference's own order, accumulating in the
// operand type R (dsl/tensor/Expression.cpp:472-481, :597-769), for a value
// per non-halo row (value(i), i an index of the with-halo layout):
//  stage 1 (more than 6 rows in all, :735-740): each tile's rows split over
//    6 workers, chunks of floor(n_t / 6 / 4) * 4 rows with the rest on worker
//    5 (:472-481), each chunk summed in row order from 0 (out = out + v, or
//    out + v * v for a squared sum, :522-533);
//  stage 2 (:743, reducePerTile :597-646): the tile's 6 partials summed in
//    worker order from 0 (with 6 rows or fewer in all: the tile's rows);
//  stages 2.1-4 (:749-752, reduceGrouped :680-727): the values of each run
//    of 368, then 736, then 1472 consecutive tiles, then of all, collected
//    on the run's first tile (common/Shape.hpp:336-351) and summed in tile
//    order - per worker first, as in stage 1, when some run holds more than
//    6 values. A run holding one value passes it on unchanged.
template <class R, class F>
R refReduce(const or_matrix& A, F value, bool square) {
  size_t total = 0;
  for (size_t t = 0; t < A.P; ++t) total += A.tileStart[t + 1] - A.tileStart[t];
  auto seqSum = [&](auto get, size_t b, size_t e, bool sq) {
    R acc = R(0);
    for (size_t i = b; i < e; ++i) {
      const R v = get(i);
      acc = sq ? acc + v * v : acc + v;
    }
    return acc;
  };
  // Per worker (6 chunks), then the 6 partials.
  auto workers = [&](auto get, size_t cnt, bool sq) {
    const size_t chunk = (cnt / 6 / 4) * 4;
    R part[6];
    for (size_t w = 0; w < 6; ++w) {
      const size_t s = chunk * w, e = w == 5 ? cnt : s + chunk;
      part[w] = seqSum(get, s, e, sq);
    }
    return seqSum([&](size_t w) { return part[w]; }, 0, 6, false);
  };
  std::vector<R> vals(A.P);
  forTiles(A.P, [&](size_t t) {
    const size_t nt = A.tileStart[t + 1] - A.tileStart[t], hb = A.haloStart[t];
    auto get = [&](size_t i) { return static_cast<R>(value(hb + i)); };
    vals[t] = total > 6 ? workers(get, nt, square) : seqSum(get, 0, nt, square);
  });
  std::vector<size_t> at(A.P);  // tile holding each value
  for (size_t t = 0; t < A.P; ++t) at[t] = t;
  const size_t groups[4] = {1472 / 4, 1472 / 2, 1472, static_cast<size_t>(-1)};
  for (size_t G : groups) {
    if (vals.size() <= 1) break;
    std::vector<size_t> key, start;
    for (size_t k = 0; k < vals.size(); ++k) {
      const size_t g = G == static_cast<size_t>(-1) ? 0 : at[k] / G * G;
      if (key.empty() || key.back() != g) {
        key.push_back(g);
        start.push_back(k);
      }
    }
    start.push_back(vals.size());
    bool perWorker = false;
    for (size_t q = 0; q + 1 < start.size(); ++q) perWorker = perWorker || start[q + 1] - start[q] > 6;
    std::vector<R> next(key.size());
    for (size_t q = 0; q < key.size(); ++q) {
      auto get = [&](size_t i) { return vals[start[q] + i]; };
      const size_t cnt = start[q + 1] - start[q];
      next[q] = perWorker ? workers(get, cnt, false) : seqSum(get, 0, cnt, false);
    }
    vals.swap(next);
    at.swap(key);
  }
  return vals.empty() ? R(0) : vals[0];
}

// Tensor::norm (dsl/tensor/Tensor.cpp:425-439) of the non-halo cells in the
// reference's reduction order and the vector's type.
template <class T>
T refNorm(const or_matrix& A, const std::vector<T>& v, int norm) {
  if (norm == 2) {
    T m = -std::numeric_limits<T>::infinity();
    for (size_t t = 0; t < A.P; ++t)
      for (size_t i = 0; i < A.tileStart[t + 1] - A.tileStart[t]; ++i) m = std::max(m, v[A.haloStart[t] + i]);
    return m;
  }
  const T s = refReduce<T>(A, [&](size_t i) { return v[i]; }, norm == 1);
  return norm == 1 ? std::sqrt(s) : s;
}

template <class T>
T refDot(const or_matrix& A, const std::vector<T>& a, const std::vector<T>& b) {
  return refReduce<T>(A, [&](size_t i) { return static_cast<T>(a[i] * b[i]); }, false);
}

// ---- ILU(0) / DILU (ilu/Solver.cpp) -----------------------------------------
template <class V>
struct IluFactors {
  std::vector<std::vector<V>> off, inv;
};

// ilu::Solver::factorizeCRS, sequential branch (ilu/Solver.cpp:134-292).
template <class V>
IluFactors<V> factorize(const or_matrix& A, const TileValues<V>& tv, bool dilu) {
  IluFactors<V> F;
  F.off = tv.off;
  F.inv = tv.diag;
  forTiles(A.P, [&](size_t t) {
    const Local& L = A.loc[t];
    const size_t nRows = L.diag.size();
    std::vector<V>& off = F.off[t];
    const std::vector<V>& aOff = tv.off[t];
    std::vector<V>& d = F.inv[t];
    // getOffDiagValue (ilu/Solver.cpp:150-161): linear search of row i for
    // column j, 0 when absent.
    auto get = [&](size_t i, size_t j, const std::vector<V>& vals) -> V {
      V r = 0;
      for (size_t a = L.rowPtr[i]; a < L.rowPtr[i + 1]; ++a)
        if (L.colInd[a] == j) r = vals[a];
      return r;
    };
    for (size_t i = 1; i < nRows; ++i) {
      const size_t iStart = L.rowPtr[i], iEnd = L.rowPtr[i + 1];
      for (size_t ik = iStart; ik < iEnd; ++ik) {
        size_t k = L.colInd[ik];
        if (k >= i) break;
        V a_kk = d[k];
        if (!dilu) {
          off[ik] = off[ik] / a_kk;
          for (size_t ij = ik + 1; ij < iEnd; ++ij) {
            size_t j = L.colInd[ij];
            if (j >= nRows) break;
            V a_kj = get(k, j, off);
            off[ij] = off[ij] - off[ik] * a_kj;
          }
          V a_ki = get(k, i, off);
          d[i] = d[i] - off[ik] * a_ki;
        } else {
          V a_ki = get(k, i, aOff);
          d[i] = d[i] - aOff[ik] * a_ki / a_kk;
        }
      }
    }
    for (size_t i = 0; i < nRows; ++i) d[i] = V(1) / d[i];
  });
  return F;
}

// ilu::Solver::solveCRS, sequential branch (ilu/Solver.cpp:380-443,
// :526-543). x and b are vectors with halo; halo entries are ignored.
template <class V, class T>
void iluSolve(const or_matrix& A, const std::vector<std::vector<V>>& off,
              const std::vector<std::vector<V>>& inv, bool dilu, const std::vector<T>& b,
              std::vector<T>& x) {
  forTiles(A.P, [&](size_t t) {
    const Local& L = A.loc[t];
    const size_t nRows = L.diag.size();
    const size_t hb = A.haloStart[t];
    for (size_t i = 0; i < nRows; ++i) {
      T temp = b[hb + i];
      for (size_t a = L.rowPtr[i]; a < L.rowPtr[i + 1]; ++a) {
        size_t j = L.colInd[a];
        if (i < j) break;
        if (j >= nRows) break;
        temp -= static_cast<T>(off[t][a]) * x[hb + j];
      }
      x[hb + i] = dilu ? temp * static_cast<T>(inv[t][i]) : temp;
    }
    for (size_t ii = nRows; ii-- > 0;) {
      T temp = 0;
      for (size_t a = L.rowPtr[ii + 1]; a-- > L.rowPtr[ii];) {
        size_t j = L.colInd[a];
        if (j < ii) break;
        if (j >= nRows) continue;
        temp -= static_cast<T>(off[t][a]) * x[hb + j];
      }
      if (dilu) x[hb + ii] = x[hb + ii] + temp * static_cast<T>(inv[t][ii]);
      else x[hb + ii] = (x[hb + ii] + temp) * static_cast<T>(inv[t][ii]);
    }
  });
}

// gaussseidel::Solver::solveIterationCSR (gauss-seidel/Solver.cpp:45-86):
// each row computed in the working type W (:76-82, every operand cast to
// it) and stored in x's type T (:83).
template <class V, class T, class W = T>
// dropHalo: the halo cells read as 0 (a block Gauss-Seidel that drops the
// couplings between tiles) instead of the values the exchange brings.
void gsSweep(const or_matrix& A, const TileValues<V>& tv, std::vector<T>& x, const std::vector<T>& b,
             bool seedB, bool dropHalo = false) {
  exchange(A, x);
  forTiles(A.P, [&](size_t t) {
    const Local& L = A.loc[t];
    const size_t nRows = L.diag.size();
    const size_t hb = A.haloStart[t];
    if (dropHalo)
      for (size_t h = hb + nRows; h < A.haloStart[t + 1]; ++h) x[h] = static_cast<T>(0);
    for (size_t i = 0; i < nRows; ++i) {
      W sum = seedB ? static_cast<W>(b[hb + i]) : static_cast<W>(tv.diag[t][i]);
      for (size_t j = L.rowPtr[i]; j < L.rowPtr[i + 1]; ++j)
        sum -= static_cast<W>(tv.off[t][j]) * static_cast<W>(x[hb + L.colInd[j]]);
      x[hb + i] = static_cast<T>(sum / static_cast<W>(tv.diag[t][i]));
    }
  });
}

// ---- solvers -----------------------------------------------------------------
struct Stats {
  double init = INFINITY, fin = INFINITY, bNorm = 0;
  int iterations = 0, inner = 0;
  bool converged = false, singular = false;
  // SolverStats::checkConvergence (SolverStats.cpp:33-56)
  void check(const Conf& c) {
    if (c.relTolerance > 0)
      converged = fin < c.absTolerance || fin < init * c.relResidual || fin < bNorm * c.relTolerance;
    else
      converged = fin < c.absTolerance || fin < init * c.relResidual;
  }
};

const double kVsmall = 1e-37;  // Traits<float>::vsmall (common/Traits.hpp:43)

template <class V>
struct Ctx {
  const or_matrix& A;
  TileValues<V> tv;
  std::vector<double>* history = nullptr;
  const void* root = nullptr;  // the top-level node records the history
  explicit Ctx(const or_matrix& a) : A(a), tv(a) {}
};

template <class V, class T>
struct SolverNode {
  virtual ~SolverNode() = default;
  virtual Stats solve(std::vector<T>& x, const std::vector<T>& b) = 0;
  virtual bool usesInitialGuess() const = 0;
};

template <class V, class T>
std::unique_ptr<SolverNode<V, T>> makeNode(Ctx<V>& C, const Conf& c);

template <class V, class T>
struct IluNode : SolverNode<V, T> {
  Ctx<V>& C;
  bool dilu;
  IluFactors<V> F;
  IluNode(Ctx<V>& c, const Conf& conf) : C(c), dilu(conf.diagonalBased), F(factorize(c.A, c.tv, conf.diagonalBased)) {}
  Stats solve(std::vector<T>& x, const std::vector<T>& b) override {
    iluSolve<V, T>(C.A, dilu ? C.tv.off : F.off, F.inv, dilu, b, x);
    Stats s;
    s.iterations = 1;
    return s;
  }
  bool usesInitialGuess() const override { return false; }
};

// gaussseidel::Solver::solve (gauss-seidel/Solver.cpp:98-160)
template <class V, class T>
struct GsNode : SolverNode<V, T> {
  Ctx<V>& C;
  const Conf& c;
  GsNode(Ctx<V>& ctx, const Conf& conf) : C(ctx), c(conf) {}
  Stats solve(std::vector<T>& x, const std::vector<T>& b) override {
    // workingType (gauss-seidel/Solver.cpp:65, :114): the sweeps and the
    // residual in W, x kept in its own type.
    const int wt = c.workingType < 0 ? (std::is_same_v<T, float> ? 0 : 1) : c.workingType;
    if (wt == 1) return solveIn<double>(x, b);
    if (wt == 0) return solveIn<float>(x, b);
    throw OErr("GaussSeidel workingType must be float32 or float64");
  }
  template <class W>
  Stats solveIn(std::vector<T>& x, const std::vector<T>& b) {
    Stats s;
    if (c.numFixedIterations > 0) {
      for (int k = 0; k < c.numFixedIterations; ++k) gsSweep<V, T, W>(C.A, C.tv, x, b, c.gsSeedB, c.gsDropHalo);
      s.iterations = c.numFixedIterations;
      return s;
    }
    if (c.relTolerance > 0) s.bNorm = normT(C.A, b, c.norm);
    std::vector<W> r(C.A.nWithHalo);
    residualT<V, T, T, W, W>(C.A, C.tv, x, b, r);
    s.init = s.fin = normT(C.A, r, c.norm);
    while (!((s.converged && s.iterations >= c.minIterations) || s.iterations >= c.maxIterations)) {
      for (int k = 0; k < c.numSweeps; ++k) {
        gsSweep<V, T, W>(C.A, C.tv, x, b, c.gsSeedB, c.gsDropHalo);
        s.iterations++;
      }
      residualT<V, T, T, W, W>(C.A, C.tv, x, b, r);
      s.fin = normT(C.A, r, c.norm);
      s.check(c);
    }
    return s;
  }
  bool usesInitialGuess() const override { return true; }
};

template <class T> T rnd(double v) { return static_cast<T>(v); }

// pbicgstab::Solver::solve (pbicgstab/Solver.cpp:48-194). With a
// workingType other than x's type (:63), every vector but x is in the
// working type W, the residual is computed in W (:66), the preconditioner
// runs on W vectors, and x = x + alpha y + omega z is evaluated in W and
// rounded to x's type each iteration (:164).
template <class V, class T>
struct PbicgstabNode : SolverNode<V, T> {
  using O = std::conditional_t<std::is_same_v<T, float>, double, float>;
  Ctx<V>& C;
  const Conf& c;
  std::unique_ptr<SolverNode<V, T>> pre;
  std::unique_ptr<SolverNode<V, O>> preO;  // the preconditioner on working-type vectors
  bool other = false;                       // working type differs from x's type
  PbicgstabNode(Ctx<V>& ctx, const Conf& conf) : C(ctx), c(conf) {
    if (conf.workingType == 2) throw OErr("PBiCGStab workingType twofloat32 is not supported");
    other = conf.workingType >= 0 && conf.workingType != (std::is_same_v<T, float> ? 0 : 1);
    if (conf.pre) {
      if (other) preO = makeNode<V, O>(ctx, *conf.pre);
      else pre = makeNode<V, T>(ctx, *conf.pre);
    }
  }
  Stats solve(std::vector<T>& x, const std::vector<T>& b) override {
    if (c.reduceRef) {
      if (other) throw OErr("reduce f32_ref_order needs the working type of x");
      return solveRef(x, b);
    }
    if (other) return core<O>(x, b, preO.get());
    return core<T>(x, b, pre.get());
  }
  template <class W>
  Stats core(std::vector<T>& x, const std::vector<T>& b, SolverNode<V, W>* pre) {
    const or_matrix& A = C.A;
    const size_t N = A.nWithHalo;
    Stats s;
    std::vector<W> r(N), r0, p, v(N), y(N), z(N), sv(N), tv(N);
    residualT<V, T, T, W, W>(A, C.tv, x, b, r);
    if (c.relTolerance > 0) s.bNorm = normT(A, b, c.norm);  // the reference uses x here (:70)
    s.init = s.fin = normT(A, r, c.norm);
    r0 = r;
    p = r;
    double rhoOld = 0, alpha = 0, omega = 0;
    while (!((s.converged && s.iterations >= c.minIterations) || s.iterations >= c.maxIterations ||
             s.singular)) {
      double rho = dotT(A, r0, r);
      s.singular = s.singular || std::fabs(rho) < kVsmall;
      if (s.singular) break;
      if (s.iterations != 0) {
        W beta = rnd<W>((rho / rhoOld) * (alpha / omega));
        W om = rnd<W>(omega);
        forTiles(A.P, [&](size_t t) {
          for (size_t i = A.haloStart[t]; i < A.haloStart[t] + A.tileStart[t + 1] - A.tileStart[t]; ++i)
            p[i] = r[i] + beta * (p[i] - om * v[i]);
        });
      }
      if (pre) {
        if (pre->usesInitialGuess()) std::fill(y.begin(), y.end(), W(0));
        pre->solve(y, p);
      } else {
        y = p;
      }
      spmvT<V, W>(A, C.tv, y, v);
      alpha = rho / dotT(A, r0, v);
      W al = rnd<W>(alpha);
      forTiles(A.P, [&](size_t t) {
        for (size_t i = A.haloStart[t]; i < A.haloStart[t] + A.tileStart[t + 1] - A.tileStart[t]; ++i)
          sv[i] = r[i] - al * v[i];
      });
      if (pre) {
        if (pre->usesInitialGuess()) std::fill(z.begin(), z.end(), W(0));
        pre->solve(z, sv);
      } else {
        z = sv;
      }
      spmvT<V, W>(A, C.tv, z, tv);
      double tt = dotT(A, tv, tv);
      omega = dotT(A, tv, sv) / tt;
      s.singular = s.singular || std::fabs(omega) < kVsmall;
      if (s.singular) break;
      W om = rnd<W>(omega);
      forTiles(A.P, [&](size_t t) {
        for (size_t i = A.haloStart[t]; i < A.haloStart[t] + A.tileStart[t + 1] - A.tileStart[t]; ++i) {
          x[i] = static_cast<T>(static_cast<W>(x[i]) + al * y[i] + om * z[i]);
          r[i] = sv[i] - om * tv[i];
        }
      });
      s.fin = normT(A, r, c.norm);
      s.check(c);
      rhoOld = rho;
      s.iterations++;
      if (C.history && C.root == this) C.history->push_back(s.fin);
    }
    return s;
  }

  // The same iteration with every scalar in the vector type T: dot products
  // and norms in the reference's reduction order (refReduce), alpha, beta,
  // omega in T, the residual norms stored as float and compared in float
  // (SolverStats.hpp:33-36, SolverStats.cpp:33-63).
  Stats solveRef(std::vector<T>& x, const std::vector<T>& b) {
    const or_matrix& A = C.A;
    const size_t N = A.nWithHalo;
    Stats s;
    std::vector<T> r(N), r0, p, v(N), y(N), z(N), sv(N), tv(N);
    residualT<V, T, T, T, T>(A, C.tv, x, b, r);
    float bNorm = 0;
    if (c.relTolerance > 0) bNorm = static_cast<float>(refNorm(A, b, c.norm));
    const float init = static_cast<float>(refNorm(A, r, c.norm));
    float fin = init;
    s.init = s.fin = init;
    s.bNorm = bNorm;
    r0 = r;
    p = r;
    T rhoOld = 0, alpha = 0, omega = 0;
    const float vsmall = 1e-37f;
    auto rows = [&](auto&& f) {
      forTiles(A.P, [&](size_t t) {
        for (size_t i = A.haloStart[t]; i < A.haloStart[t] + A.tileStart[t + 1] - A.tileStart[t]; ++i) f(i);
      });
    };
    while (!((s.converged && s.iterations >= c.minIterations) || s.iterations >= c.maxIterations ||
             s.singular)) {
      const T rho = refDot(A, r0, r);
      s.singular = s.singular || std::fabs(rho) < static_cast<T>(vsmall);
      if (s.singular) break;
      if (s.iterations != 0) {
        const T beta = (rho / rhoOld) * (alpha / omega);
        rows([&](size_t i) { p[i] = r[i] + beta * (p[i] - omega * v[i]); });
      }
      if (pre) {
        if (pre->usesInitialGuess()) std::fill(y.begin(), y.end(), T(0));
        pre->solve(y, p);
      } else {
        y = p;
      }
      spmvT<V, T>(A, C.tv, y, v);
      alpha = rho / refDot(A, r0, v);
      rows([&](size_t i) { sv[i] = r[i] - alpha * v[i]; });
      if (pre) {
        if (pre->usesInitialGuess()) std::fill(z.begin(), z.end(), T(0));
        pre->solve(z, sv);
      } else {
        z = sv;
      }
      spmvT<V, T>(A, C.tv, z, tv);
      const T tt = refDot(A, tv, tv);
      omega = refDot(A, tv, sv) / tt;
      s.singular = s.singular || std::fabs(omega) < static_cast<T>(vsmall);
      if (s.singular) break;
      rows([&](size_t i) {
        x[i] = x[i] + alpha * y[i] + omega * z[i];
        r[i] = sv[i] - omega * tv[i];
      });
      fin = static_cast<float>(refNorm(A, r, c.norm));
      s.fin = fin;
      if (c.relTolerance > 0)
        s.converged = fin < c.absTolerance || fin < init * c.relResidual || fin < bNorm * c.relTolerance;
      else
        s.converged = fin < c.absTolerance || fin < init * c.relResidual;
      rhoOld = rho;
      s.iterations++;
      if (C.history && C.root == this) C.history->push_back(s.fin);
    }
    return s;
  }
  bool usesInitialGuess() const override { return true; }
};

// restarter::Solver::solve (restarter/Solver.cpp:40-56)
template <class V, class T>
struct RestarterNode : SolverNode<V, T> {
  Ctx<V>& C;
  const Conf& c;
  std::unique_ptr<SolverNode<V, T>> inner;
  RestarterNode(Ctx<V>& ctx, const Conf& conf) : C(ctx), c(conf), inner(makeNode<V, T>(ctx, *conf.inner)) {}
  Stats solve(std::vector<T>& x, const std::vector<T>& b) override {
    int restarts = 0;
    Stats s = inner->solve(x, b);
    int total = s.iterations;
    while (restarts < c.maxRestarts && !s.converged) {
      restarts++;
      s = inner->solve(x, b);
      total += s.iterations;
    }
    s.inner = total;
    return s;
  }
  bool usesInitialGuess() const override { return inner->usesInitialGuess(); }
};

template <class V, class T>
std::unique_ptr<SolverNode<V, T>> makeNode(Ctx<V>& C, const Conf& c) {
  if (c.type == "ILU") return std::make_unique<IluNode<V, T>>(C, c);
  if (c.type == "GaussSeidel") return std::make_unique<GsNode<V, T>>(C, c);
  if (c.type == "PBiCGStab") return std::make_unique<PbicgstabNode<V, T>>(C, c);
  if (c.type == "restarter") return std::make_unique<RestarterNode<V, T>>(C, c);
  throw OErr("solver " + c.type + " cannot be nested here");
}

// iterativerefinement::Solver::solve (iterative-refinement/Solver.cpp:48-123)
// with working precision float (x) and extended precision E.
template <class V, class E>
Stats mpirT(Ctx<V>& C, const Conf& c, std::vector<float>& x, const std::vector<float>& b,
            double* phiOut) {
  const or_matrix& A = C.A;
  Stats s;
  auto inner = makeNode<V, float>(C, *c.inner);
  if (c.relTolerance > 0) s.bNorm = normT(A, b, c.norm);
  std::vector<float> r(A.nWithHalo);
  auto resid = [&](std::vector<E>& phi) {
    if constexpr (std::is_same_v<E, DW>) residualDw<DW>(A, C.tv, phi, b, r);
    else residualT<V, E, float, float, E>(A, C.tv, phi, b, r);
  };
  std::vector<E> phi(A.nWithHalo);
  for (size_t i = 0; i < A.nWithHalo; ++i) {
    if constexpr (std::is_same_v<E, DW>) phi[i] = DW{x[i], 0.0f};
    else phi[i] = static_cast<E>(x[i]);
  }
  {
    // The initial residual uses x itself (in E arithmetic).
    std::vector<E> xe = phi;
    resid(xe);
  }
  s.init = s.fin = normT(A, r, c.norm);
  std::vector<float>& corr = x;
  while (!((s.converged && s.iterations >= c.minIterations) || s.iterations >= c.maxIterations)) {
    s.iterations++;
    if (inner->usesInitialGuess()) std::fill(corr.begin(), corr.end(), 0.0f);
    Stats is = inner->solve(corr, r);
    s.inner += is.inner ? is.inner : is.iterations;
    for (size_t i = 0; i < A.nWithHalo; ++i) {
      if constexpr (std::is_same_v<E, DW>) phi[i] = dwPlusFp(phi[i], corr[i]);
      else phi[i] = phi[i] + static_cast<E>(corr[i]);
    }
    resid(phi);
    s.fin = normT(A, r, c.norm);
    s.check(c);
    if (C.history) C.history->push_back(s.fin);
  }
  for (size_t i = 0; i < A.nWithHalo; ++i) {
    if constexpr (std::is_same_v<E, DW>) x[i] = phi[i].h + phi[i].l;
    else x[i] = static_cast<float>(phi[i]);
  }
  if (phiOut) {
    for (size_t t = 0; t < A.P; ++t) {
      size_t nr = A.tileStart[t + 1] - A.tileStart[t];
      for (size_t i = 0; i < nr; ++i) {
        const E& e = phi[A.haloStart[t] + i];
        if constexpr (std::is_same_v<E, DW>) phiOut[A.tileStart[t] + i] = static_cast<double>(e.h) + static_cast<double>(e.l);
        else phiOut[A.tileStart[t] + i] = static_cast<double>(e);
      }
    }
  }
  return s;
}

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

template <class V>
int solveWithValues(const or_matrix* A, const Conf& c, void* x, int xt, const void* b, int bt,
                    or_stats* st, double* phiOut, std::vector<double>* hist) {
  Ctx<V> C(*A);
  C.history = hist;
  Stats s;
  if (c.type == "IterativeRefinement") {
    if (xt != 0 || bt != 0) throw OErr("IterativeRefinement needs float32 x and b");
    auto xv = withHalo(*A, static_cast<float*>(x));
    auto bv = withHalo(*A, static_cast<const float*>(b));
    int E = c.extendedType < 0 ? 0 : c.extendedType;
    if (E == 0) s = mpirT<V, float>(C, c, xv, bv, phiOut);
    else if (E == 1) s = mpirT<V, double>(C, c, xv, bv, phiOut);
    else {
      if constexpr (std::is_same_v<V, float>) s = mpirT<V, DW>(C, c, xv, bv, phiOut);
      else throw OErr("twofloat32 needs float32 coefficients");
    }
    stripHalo(*A, xv, static_cast<float*>(x));
  } else if (xt == 0) {
    if (bt != 0) throw OErr("b must have the type of x");
    auto xv = withHalo(*A, static_cast<float*>(x));
    auto bv = withHalo(*A, static_cast<const float*>(b));
    auto node = makeNode<V, float>(C, c);
    C.root = node.get();
    s = node->solve(xv, bv);
    stripHalo(*A, xv, static_cast<float*>(x));
  } else {
    if (bt != 1) throw OErr("b must have the type of x");
    auto xv = withHalo(*A, static_cast<double*>(x));
    auto bv = withHalo(*A, static_cast<const double*>(b));
    auto node = makeNode<V, double>(C, c);
    C.root = node.get();
    s = node->solve(xv, bv);
    stripHalo(*A, xv, static_cast<double*>(x));
  }
  st->initial_residual = s.init;
  st->final_residual = s.fin;
  st->b_norm = s.bNorm;
  st->iterations = s.iterations;
  st->converged = s.converged;
  st->singular = s.singular;
  st->inner_iterations = s.inner;
  return 0;
}

}  // namespace

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

void or_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }

or_matrix* or_build(int64_t n, int64_t nnz, const int64_t* rows, const int64_t* cols, const double* vals,
                    int64_t num_tiles, const int32_t* row_to_tile, int value_type) {
  or_matrix* A = new or_matrix();
  if (guard([&] {
        A->vt = value_type;
        std::vector<std::tuple<size_t, size_t, double>> ent(nnz);
        for (int64_t i = 0; i < nnz; ++i) {
          if (rows[i] < 0 || rows[i] >= n || cols[i] < 0 || cols[i] >= n) throw OErr("index out of range");
          ent[i] = {static_cast<size_t>(rows[i]), static_cast<size_t>(cols[i]), roundVT(value_type, vals[i])};
        }
        buildMatrix(*A, std::move(ent), n, num_tiles, row_to_tile);
      })) {
    delete A;
    return nullptr;
  }
  return A;
}

or_matrix* or_build_ldu(int64_t n, int64_t num_faces, const int64_t* owner, const int64_t* neighbour,
                        const double* diag, const double* lower, const double* upper, int64_t num_tiles,
                        const int32_t* row_to_tile, int value_type) {
  or_matrix* A = new or_matrix();
  if (guard([&] {
        A->vt = value_type;
        const double* up = upper ? upper : lower;
        std::vector<std::tuple<size_t, size_t, double>> ent;
        ent.reserve(n + 2 * num_faces);
        for (int64_t c = 0; c < n; ++c) ent.emplace_back(c, c, roundVT(value_type, diag[c]));
        for (int64_t f = 0; f < num_faces; ++f) {
          if (owner[f] < 0 || owner[f] >= neighbour[f] || neighbour[f] >= n) throw OErr("bad face");
          ent.emplace_back(owner[f], neighbour[f], roundVT(value_type, up[f]));
          ent.emplace_back(neighbour[f], owner[f], roundVT(value_type, lower[f]));
        }
        buildMatrix(*A, std::move(ent), n, num_tiles, row_to_tile);
        // Global addressing: owned faces per cell (faces are sorted by
        // owner) and losort (faces by neighbour, then face index).
        std::vector<size_t> ownerStart(n + 1, 0), losortStart(n + 1, 0), losort(num_faces);
        for (int64_t f = 0; f < num_faces; ++f) {
          ownerStart[owner[f] + 1]++;
          losortStart[neighbour[f] + 1]++;
        }
        for (int64_t c = 0; c < n; ++c) {
          ownerStart[c + 1] += ownerStart[c];
          losortStart[c + 1] += losortStart[c];
        }
        std::vector<size_t> fill(losortStart.begin(), losortStart.end() - 1);
        for (int64_t f = 0; f < num_faces; ++f) losort[fill[neighbour[f]]++] = f;
        A->ldu = true;
        A->lloc.resize(A->P);
        for (size_t t = 0; t < A->P; ++t) {
          const Tile& T = A->tiles[t];
          LocalLdu& L = A->lloc[t];
          const size_t nr = A->tileStart[t + 1] - A->tileStart[t];
          std::unordered_map<size_t, size_t> localFace;
          std::vector<size_t> faceOwner;
          L.ownerStart.push_back(0);
          for (size_t c = 0; c < nr; ++c) {
            const size_t gc = T.l2g[c];
            for (size_t f = ownerStart[gc]; f < ownerStart[gc + 1]; ++f) {
              localFace[f] = L.upperAddr.size();
              L.upperAddr.push_back(T.g2l.at(neighbour[f]));
              L.upper.push_back(roundVT(value_type, up[f]));
              faceOwner.push_back(c);
            }
            L.ownerStart.push_back(L.upperAddr.size());
          }
          L.neighbourStart.push_back(0);
          for (size_t c = 0; c < nr; ++c) {
            const size_t gc = T.l2g[c];
            for (size_t s = losortStart[gc]; s < losortStart[gc + 1]; ++s) {
              const size_t f = losort[s];
              auto it = localFace.find(f);
              size_t lf;
              if (it != localFace.end()) {
                lf = it->second;
              } else {  // owned by a halo cell
                lf = faceOwner.size();
                localFace[f] = lf;
                faceOwner.push_back(T.g2l.at(owner[f]));
              }
              L.neighbourColInd.push_back(lf);
              L.lowerLosort.push_back(roundVT(value_type, lower[f]));
            }
            L.neighbourStart.push_back(L.neighbourColInd.size());
          }
          L.lowerAddr = faceOwner;
        }
      })) {
    delete A;
    return nullptr;
  }
  return A;
}

or_matrix* or_poisson(int64_t nx, int64_t ny, int64_t nz, int64_t num_tiles, const int32_t* row_to_tile,
                      int value_type) {
  // generate3DPoissonTripletMatrix (Poisson.cpp:26-69)
  std::vector<int64_t> r, c;
  std::vector<double> v;
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        int64_t row = k * nx * ny + j * nx + i;
        auto put = [&](int64_t col, double val) { r.push_back(row); c.push_back(col); v.push_back(val); };
        put(row, 6.0);
        if (i > 0) put(row - 1, -1.0);
        if (i < nx - 1) put(row + 1, -1.0);
        if (j > 0) put(row - nx, -1.0);
        if (j < ny - 1) put(row + nx, -1.0);
        if (k > 0) put(row - nx * ny, -1.0);
        if (k < nz - 1) put(row + nx * ny, -1.0);
      }
  return or_build(nx * ny * nz, static_cast<int64_t>(r.size()), r.data(), c.data(), v.data(), num_tiles,
                  row_to_tile, value_type);
}

void or_free(or_matrix* A) { delete A; }

int64_t or_num_rows(const or_matrix* A) { return static_cast<int64_t>(A->n); }
int64_t or_num_tiles(const or_matrix* A) { return static_cast<int64_t>(A->P); }
int64_t or_num_off_diag(const or_matrix* A) { return static_cast<int64_t>(A->gCol.size()); }
int64_t or_num_halo(const or_matrix* A) { return static_cast<int64_t>(A->nWithHalo - A->n); }

int or_row_to_tile(const or_matrix* A, int32_t* out) {
  for (size_t i = 0; i < A->n; ++i) out[i] = static_cast<int32_t>(A->rowToTile[i]);
  return 0;
}

int or_tile_sizes(const or_matrix* A, int64_t* out) {
  for (size_t t = 0; t < A->P; ++t) {
    out[3 * t] = static_cast<int64_t>(A->tiles[t].nInterior());
    out[3 * t + 1] = static_cast<int64_t>(A->tiles[t].nSep());
    out[3 * t + 2] = static_cast<int64_t>(A->tiles[t].nHalo());
  }
  return 0;
}

int or_local_to_global(const or_matrix* A, int64_t* out) {
  size_t o = 0;
  for (auto& t : A->tiles)
    for (size_t g : t.l2g) out[o++] = static_cast<int64_t>(g);
  return 0;
}

int or_local_crs(const or_matrix* A, int64_t* row_ptr, int32_t* col_ind, double* off_diag, double* diag) {
  size_t orow = 0, oc = 0, od = 0;
  for (auto& L : A->loc) {
    for (size_t v : L.rowPtr)
      if (row_ptr) row_ptr[orow++] = static_cast<int64_t>(v);
    for (size_t i = 0; i < L.colInd.size(); ++i) {
      if (col_ind) col_ind[oc] = static_cast<int32_t>(L.colInd[i]);
      if (off_diag) off_diag[oc] = L.off[i];
      ++oc;
    }
    for (double d : L.diag)
      if (diag) diag[od++] = d;
  }
  return 0;
}

int or_colors(const or_matrix* A, int32_t* color) {
  size_t o = 0;
  for (auto& L : A->loc)
    for (size_t c : L.color) color[o++] = c == SIZE_MAX ? -1 : static_cast<int32_t>(c);
  return 0;
}

int or_multicolor_recommended(const or_matrix* A) { return A->multicolor ? 1 : 0; }

int or_spmv(const or_matrix* A, const void* x, void* y, int t) {
  return guard([&] {
    if (t == 0) {
      auto xv = withHalo(*A, static_cast<const float*>(x));
      std::vector<float> yv(A->nWithHalo);
      if (A->vt == 0) spmvT<float, float>(*A, TileValues<float>(*A), xv, yv);
      else throw OErr("float32 vectors with float64 coefficients");
      stripHalo(*A, yv, static_cast<float*>(y));
    } else {
      auto xv = withHalo(*A, static_cast<const double*>(x));
      std::vector<double> yv(A->nWithHalo);
      if (A->vt == 0) spmvT<float, double>(*A, TileValues<float>(*A), xv, yv);
      else spmvT<double, double>(*A, TileValues<double>(*A), xv, yv);
      stripHalo(*A, yv, static_cast<double*>(y));
    }
  });
}

int or_residual(const or_matrix* A, const void* x, int xt, const void* b, int bt, void* r, int rt, int it) {
  return guard([&] {
    if (it == 2) {
      if (A->vt != 0 || bt != 0 || rt != 0) throw OErr("double-word residual needs float32 data");
      auto bv = withHalo(*A, static_cast<const float*>(b));
      std::vector<float> rv(A->nWithHalo);
      TileValues<float> tv(*A);
      if (xt == 2) {
        auto xv = withHalo(*A, static_cast<const DW*>(x));
        residualDw<DW>(*A, tv, xv, bv, rv);
      } else {
        auto xv = withHalo(*A, static_cast<const float*>(x));
        residualDw<float>(*A, tv, xv, bv, rv);
      }
      stripHalo(*A, rv, static_cast<float*>(r));
      return;
    }
    auto run = [&](auto vtag, auto xtag, auto btag, auto rtag, auto itag) {
      using V = decltype(vtag);
      using X = decltype(xtag);
      using B = decltype(btag);
      using R = decltype(rtag);
      using I = decltype(itag);
      auto xv = withHalo(*A, static_cast<const X*>(x));
      auto bv = withHalo(*A, static_cast<const B*>(b));
      std::vector<R> rv(A->nWithHalo);
      residualT<V, X, B, R, I>(*A, TileValues<V>(*A), xv, bv, rv);
      stripHalo(*A, rv, static_cast<R*>(r));
    };
    auto withI = [&](auto v, auto xx, auto bb, auto rr) {
      if (it == 0) run(v, xx, bb, rr, float());
      else run(v, xx, bb, rr, double());
    };
    auto withR = [&](auto v, auto xx, auto bb) {
      if (rt == 0) withI(v, xx, bb, float());
      else withI(v, xx, bb, double());
    };
    auto withB = [&](auto v, auto xx) {
      if (bt == 0) withR(v, xx, float());
      else withR(v, xx, double());
    };
    auto withX = [&](auto v) {
      if (xt == 0) withB(v, float());
      else withB(v, double());
    };
    if (A->vt == 0) withX(float());
    else withX(double());
  });
}

double or_norm(const or_matrix* A, const void* x, int t, int norm) {
  if (t == 0) return normT(*A, withHalo(*A, static_cast<const float*>(x)), norm);
  return normT(*A, withHalo(*A, static_cast<const double*>(x)), norm);
}

// Expression::reduce on one tile (Expression.cpp:472-481, :729-769): 6
// worker chunks of floor(n/6/4)*4 elements, worker 5 takes the rest; each
// worker sums its chunk in order, then the 6 partials are summed in worker
// order.
double or_reduce_sum(const float* x, int64_t n, int f32) {
  if (!f32) {
    double acc = 0;
    for (int64_t i = 0; i < n; ++i) acc += x[i];
    return acc;
  }
  if (n <= 6) {
    float acc = 0;
    for (int64_t i = 0; i < n; ++i) acc += x[i];
    return acc;
  }
  int64_t chunk = (n / 6 / 4) * 4;
  float tot = 0;
  for (int w = 0; w < 6; ++w) {
    int64_t s = chunk * w, e = (w == 5) ? n : s + chunk;
    float acc = 0;
    for (int64_t i = s; i < e; ++i) acc += x[i];
    tot += acc;
  }
  return tot;
}

double or_ref_dot(const or_matrix* A, const void* a, const void* b, int t) {
  if (t == 0)
    return refDot(*A, withHalo(*A, static_cast<const float*>(a)), withHalo(*A, static_cast<const float*>(b)));
  return refDot(*A, withHalo(*A, static_cast<const double*>(a)), withHalo(*A, static_cast<const double*>(b)));
}

double or_ref_norm(const or_matrix* A, const void* x, int t, int norm) {
  if (t == 0) return refNorm(*A, withHalo(*A, static_cast<const float*>(x)), norm);
  return refNorm(*A, withHalo(*A, static_cast<const double*>(x)), norm);
}

int or_ilu_factorize(const or_matrix* A, int dilu, double* off_out, double* inv_out) {
  return guard([&] {
    auto emit = [&](auto F) {
      size_t o = 0, d = 0;
      for (size_t t = 0; t < A->P; ++t) {
        for (auto v : F.off[t]) off_out[o++] = static_cast<double>(v);
        for (auto v : F.inv[t]) inv_out[d++] = static_cast<double>(v);
      }
    };
    if (A->vt == 0) emit(factorize<float>(*A, TileValues<float>(*A), dilu != 0));
    else emit(factorize<double>(*A, TileValues<double>(*A), dilu != 0));
  });
}

int or_ilu_solve(const or_matrix* A, int dilu, const double* factor_off, const double* inv_diag,
                 const void* b, void* x, int t) {
  return guard([&] {
    auto run = [&](auto vtag, auto ttag) {
      using V = decltype(vtag);
      using T = decltype(ttag);
      std::vector<std::vector<V>> off(A->P), inv(A->P);
      size_t o = 0, d = 0;
      for (size_t tt = 0; tt < A->P; ++tt) {
        for (size_t i = 0; i < A->loc[tt].off.size(); ++i) off[tt].push_back(static_cast<V>(factor_off[o++]));
        for (size_t i = 0; i < A->loc[tt].diag.size(); ++i) inv[tt].push_back(static_cast<V>(inv_diag[d++]));
      }
      auto bv = withHalo(*A, static_cast<const T*>(b));
      std::vector<T> xv(A->nWithHalo, T(0));
      iluSolve<V, T>(*A, off, inv, dilu != 0, bv, xv);
      stripHalo(*A, xv, static_cast<T*>(x));
    };
    if (A->vt == 0 && t == 0) run(float(), float());
    else if (A->vt == 0) run(float(), double());
    else run(double(), double());
  });
}

int or_gs_sweep(const or_matrix* A, void* x, const void* b, int t, int seed_b, int drop_halo) {
  return guard([&] {
    auto run = [&](auto vtag, auto ttag) {
      using V = decltype(vtag);
      using T = decltype(ttag);
      auto xv = withHalo(*A, static_cast<const T*>(x));
      auto bv = withHalo(*A, static_cast<const T*>(b));
      gsSweep<V, T>(*A, TileValues<V>(*A), xv, bv, seed_b != 0, drop_halo != 0);
      stripHalo(*A, xv, static_cast<T*>(x));
    };
    if (A->vt == 0 && t == 0) run(float(), float());
    else if (A->vt == 0) run(float(), double());
    else run(double(), double());
  });
}

int or_solve(const or_matrix* A, const char* json, void* x, int xt, const void* b, int bt, or_stats* stats,
             double* phi_out, double* history, int history_len) {
  return guard([&] {
    JParser jp{json, json + std::strlen(json)};
    JVal root = jp.parse();
    auto conf = parseConf(root);
    std::vector<double> hist;
    if (A->vt == 0) solveWithValues<float>(A, *conf, x, xt, b, bt, stats, phi_out, history ? &hist : nullptr);
    else solveWithValues<double>(A, *conf, x, xt, b, bt, stats, phi_out, history ? &hist : nullptr);
    if (history)
      for (int i = 0; i < history_len; ++i) history[i] = i < static_cast<int>(hist.size()) ? hist[i] : NAN;
  });
}

}  // extern "C"
