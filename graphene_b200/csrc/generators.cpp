// Synthetic 3-D test matrices beyond the reference's constant Poisson
// stencil (matrix/host/details/Poisson.cpp:26-69). All use the reference's
// natural row order row = k*nx*ny + j*nx + i and drop neighbours outside the
// grid; rows are emitted sorted by column. Random numbers come from a
// counter-based splitmix64 stream, so a matrix depends only on its seed.
#include <algorithm>
#include <atomic>
#include <cmath>

#include "host_matrix.hpp"

namespace gr {

namespace {

// splitmix64 finaliser (Steele, Lea, Flood 2014).
inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform in [0, 1): the 53 high bits of the i-th output of stream `seed`.
inline double uniform(uint64_t seed, uint64_t i) {
  uint64_t z = mix64(mix64(seed) ^ (i * 0xD1B54A32D192ED03ull));
  return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);
}

// Standard normal by Box-Muller on outputs 2i and 2i+1.
inline double normal(uint64_t seed, uint64_t i) {
  const double u1 = 1.0 - uniform(seed, 2 * i);  // (0, 1]
  const double u2 = uniform(seed, 2 * i + 1);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
}

// Fills a 7-point CRS given per-row neighbour weights. coef(r, dir) returns
// the off-diagonal value towards direction dir (0:-z 1:-y 2:-x 3:+x 4:+y
// 5:+z); diag(r) the diagonal.
template <class Coef, class Diag>
GeneratedCsr sevenPoint(i64 nx, i64 ny, i64 nz, Coef coef, Diag diag) {
  if (nx <= 0 || ny <= 0 || nz <= 0) fail(GR_EINVAL, "grid dimensions must be positive");
  GeneratedCsr g;
  g.n = nx * ny * nz;
  const i64 n = g.n;
  g.rowPtr.assign(n + 1, 0);
  for (i64 r = 0; r < n; ++r) {
    i64 i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
    g.rowPtr[r + 1] = g.rowPtr[r] + 1 + (k > 0) + (j > 0) + (i > 0) + (i < nx - 1) + (j < ny - 1) + (k < nz - 1);
  }
  g.col.resize(g.rowPtr[n]);
  g.val.resize(g.rowPtr[n]);
  g.coords.resize(3 * n);
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 r = b; r < e; ++r) {
      i64 i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
      i64 o = g.rowPtr[r];
      auto put = [&](i64 c, double v) { g.col[o] = c; g.val[o] = v; ++o; };
      if (k > 0) put(r - nx * ny, coef(r, 0));
      if (j > 0) put(r - nx, coef(r, 1));
      if (i > 0) put(r - 1, coef(r, 2));
      put(r, diag(r));
      if (i < nx - 1) put(r + 1, coef(r, 3));
      if (j < ny - 1) put(r + nx, coef(r, 4));
      if (k < nz - 1) put(r + nx * ny, coef(r, 5));
      g.coords[3 * r] = static_cast<double>(i);
      g.coords[3 * r + 1] = static_cast<double>(j);
      g.coords[3 * r + 2] = static_cast<double>(k);
    }
  });
  return g;
}

// The values of a 7-point matrix only, in the order sevenPoint emits them:
// each row's off-diagonals (-z, -y, -x, +x, +y, +z, present ones) at
// gVal[gRowPtr[r]..], its diagonal at gDiag[r]. False if gRowPtr is not
// this grid's pattern.
template <class Coef, class Diag>
bool sevenPointValues(i64 nx, i64 ny, i64 nz, Coef coef, Diag diag, const std::vector<i64>& gRowPtr, double* gVal,
                      double* gDiag) {
  const i64 n = nx * ny * nz;
  if (static_cast<i64>(gRowPtr.size()) != n + 1) return false;
  std::atomic<bool> ok{true};
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 r = b; r < e; ++r) {
      const i64 i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
      const bool has[6] = {k > 0, j > 0, i > 0, i < nx - 1, j < ny - 1, k < nz - 1};
      i64 o = gRowPtr[r];
      for (int d = 0; d < 6; ++d)
        if (has[d]) {
          if (o >= gRowPtr[r + 1]) {
            ok = false;
            return;
          }
          gVal[o++] = coef(r, d);
        }
      if (o != gRowPtr[r + 1]) ok = false;
      gDiag[r] = diag(r);
    }
  });
  return ok;
}

// Variable-coefficient Poisson stencil: cell conductivity k = exp(sigma *
// N(0,1)); face coefficient = harmonic mean 2 k_a k_b / (k_a + k_b);
// off-diagonal = -face coefficient; diagonal = sum of face coefficients
// plus 2 k for every boundary face (Dirichlet condition at the face).
// Computed in FP64.
struct VarPoissonStencil {
  i64 nx, ny, nz;
  std::vector<double> kc;
  i64 off[6];
  VarPoissonStencil(i64 x, i64 y, i64 z, double sigma, uint64_t seed) : nx(x), ny(y), nz(z), kc(x * y * z) {
    const i64 n = nx * ny * nz;
    parallelChunks(n, [&](i64 b, i64 e) {
      for (i64 r = b; r < e; ++r) kc[r] = std::exp(sigma * normal(seed, static_cast<uint64_t>(r)));
    });
    const i64 o[6] = {-nx * ny, -nx, -1, 1, nx, nx * ny};
    std::copy(o, o + 6, off);
  }
  double face(i64 r, int d) const {
    const double a = kc[r], bb = kc[r + off[d]];
    return 2.0 * a * bb / (a + bb);
  }
  double coef(i64 r, int d) const { return -face(r, d); }
  double diag(i64 r) const {
    i64 i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
    const bool has[6] = {k > 0, j > 0, i > 0, i < nx - 1, j < ny - 1, k < nz - 1};
    double s = 0;
    for (int d = 0; d < 6; ++d) s += has[d] ? face(r, d) : 2.0 * kc[r];
    return s;
  }
};

// Upwind convection-diffusion with unit diffusion and grid spacing and
// velocity (vx, vy, vz) >= 0: neighbour coefficients -(1 + v_d) upstream,
// -1 downstream; diagonal 6 + vx + vy + vz, kept at the boundary.
struct ConvDiffStencil {
  double up[6], dg;
  ConvDiffStencil(double vx, double vy, double vz)
      : up{-(1.0 + vz), -(1.0 + vy), -(1.0 + vx), -1.0, -1.0, -1.0}, dg(6.0 + vx + vy + vz) {}
  double coef(i64, int d) const { return up[d]; }
  double diag(i64) const { return dg; }
};

}  // namespace

GeneratedCsr generateVarPoisson(i64 nx, i64 ny, i64 nz, double sigma, uint64_t seed) {
  const VarPoissonStencil S(nx, ny, nz, sigma, seed);
  return sevenPoint(nx, ny, nz, [&](i64 r, int d) { return S.coef(r, d); }, [&](i64 r) { return S.diag(r); });
}

GeneratedCsr generateConvDiff(i64 nx, i64 ny, i64 nz, double vx, double vy, double vz) {
  const ConvDiffStencil S(vx, vy, vz);
  return sevenPoint(nx, ny, nz, [&](i64 r, int d) { return S.coef(r, d); }, [&](i64 r) { return S.diag(r); });
}

bool generateValues(int kind, i64 nx, i64 ny, i64 nz, const double* params, uint64_t seed,
                    const std::vector<i64>& gRowPtr, double* gVal, double* gDiag) {
  if (nx <= 0 || ny <= 0 || nz <= 0) fail(GR_EINVAL, "grid dimensions must be positive");
  if (kind == 0)
    return sevenPointValues(nx, ny, nz, [](i64, int) { return -1.0; }, [](i64) { return 6.0; }, gRowPtr, gVal, gDiag);
  if (kind == 1) {
    const VarPoissonStencil S(nx, ny, nz, params[0], seed);
    return sevenPointValues(nx, ny, nz, [&](i64 r, int d) { return S.coef(r, d); },
                            [&](i64 r) { return S.diag(r); }, gRowPtr, gVal, gDiag);
  }
  if (kind == 2) {
    if (params[0] < 0 || params[1] < 0 || params[2] < 0) fail(GR_EINVAL, "velocity must be >= 0");
    const ConvDiffStencil S(params[0], params[1], params[2]);
    return sevenPointValues(nx, ny, nz, [&](i64 r, int d) { return S.coef(r, d); },
                            [&](i64 r) { return S.diag(r); }, gRowPtr, gVal, gDiag);
  }
  fail(GR_EINVAL, "unknown generator");
}

// Uniform [lo, hi) values of stream `seed` (used for seeded right-hand sides).
void generateUniform(uint64_t seed, i64 n, double lo, double hi, double* out) {
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 i = b; i < e; ++i) out[i] = lo + (hi - lo) * uniform(seed, static_cast<uint64_t>(i));
  });
}

void generateNormal(uint64_t seed, i64 n, double* out) {
  parallelChunks(n, [&](i64 b, i64 e) {
    for (i64 i = b; i < e; ++i) out[i] = normal(seed, static_cast<uint64_t>(i));
  });
}

}  // namespace gr
