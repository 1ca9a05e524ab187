// Seeded benchmark inputs for the oracle -- TEST INFRASTRUCTURE ONLY.
//
// The reference arm of the benchmark runs the oracle alone, so the oracle
// needs its own copy of the benchmark's synthetic inputs: the 7-point
// matrices (constant, variable-coefficient and convection-diffusion), the
// seeded vectors and the coordinate bisection that partitions a generated
// grid into tiles. Each is written here from its definition, not taken from
// the product library; tests/test_generators.py pins both against the numpy
// restatement in tests/generators_ref.py.
//
// Definitions:
//  - stream: splitmix64 finaliser (Steele, Lea, Flood 2014) applied to
//    mix(seed) ^ (i * 0xD1B54A32D192ED03); uniform [0,1) from the top 53
//    bits; normals by Box-Muller over outputs 2i, 2i+1.
//  - natural row order r = i + nx (j + ny k); each row's entries by column:
//    -z, -y, -x, diagonal, +x, +y, +z; neighbours outside the grid dropped
//    (as generate3DPoissonTripletMatrix does, matrix/host/details/Poisson.cpp:26-69).
//  - variable coefficients: k = exp(sigma N(0,1)) per cell, face value
//    2 k_row k_nb / (k_row + k_nb), off-diagonal -face, diagonal the six
//    face terms summed in direction order with 2 k_row at a boundary face.
//  - convection-diffusion: -(1 + v_d) towards -x, -y, -z, -1 towards +x, +y,
//    +z, diagonal 6 + vx + vy + vz.
//  - bisection: the partitioner of the benchmark's tile maps (METIS 5.2.1,
//    which the reference calls at CRSHostMatrix.cpp:214-231, is not
//    available). Split the longest axis of the rows' bounding box; order
//    rows by (coordinate, row); cut at the first prefix whose weight (row
//    off-diagonals + 1, the reference's vertex weight, CRSHostMatrix.cpp:185-194)
//    reaches total * p1 / parts, p1 = parts / 2; move the cut to the nearer
//    (by weight) coordinate-plane boundary; recurse.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

uint64_t smix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double unit(uint64_t seed, uint64_t i) {
  const uint64_t z = smix(smix(seed) ^ (i * 0xD1B54A32D192ED03ull));
  return static_cast<double>(z >> 11) / 9007199254740992.0;
}

double gauss(uint64_t seed, uint64_t i) {
  const double a = 1.0 - unit(seed, 2 * i);
  const double b = unit(seed, 2 * i + 1);
  return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586476925 * b);
}

struct Rcb {
  const double* xyz;
  const int64_t* wt;
  int32_t* part;

  void run(int64_t* rows, int64_t cnt, int32_t parts, int32_t first, int depth) {
    if (parts == 1) {
      for (int64_t q = 0; q < cnt; ++q) part[rows[q]] = first;
      return;
    }
    if (cnt == 0) return;
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = xyz[3 * rows[0] + d];
    for (int64_t q = 1; q < cnt; ++q)
      for (int d = 0; d < 3; ++d) {
        const double v = xyz[3 * rows[q] + d];
        if (v < lo[d]) lo[d] = v;
        if (v > hi[d]) hi[d] = v;
      }
    int ax = 0;
    if (hi[1] - lo[1] > hi[ax] - lo[ax]) ax = 1;
    if (hi[2] - lo[2] > hi[ax] - lo[ax]) ax = 2;
    std::sort(rows, rows + cnt, [&](int64_t a, int64_t b) {
      const double ca = xyz[3 * a + ax], cb = xyz[3 * b + ax];
      return ca < cb || (ca == cb && a < b);
    });
    const int32_t p1 = parts / 2;
    int64_t total = 0;
    for (int64_t q = 0; q < cnt; ++q) total += wt[rows[q]];
    int64_t cut = cnt, acc = 0;
    for (int64_t q = 0; q < cnt; ++q) {
      if (acc * parts >= total * p1) {
        cut = q;
        break;
      }
      acc += wt[rows[q]];
    }
    auto onPlane = [&](int64_t q) {
      return q == 0 || q == cnt || xyz[3 * rows[q - 1] + ax] != xyz[3 * rows[q] + ax];
    };
    if (!onPlane(cut)) {
      int64_t left = cut, right = cut;
      while (!onPlane(left)) --left;
      while (!onPlane(right)) ++right;
      int64_t wl = 0, wr = 0;
      for (int64_t q = 0; q < right; ++q) {
        if (q < left) wl += wt[rows[q]];
        wr += wt[rows[q]];
      }
      const double target = static_cast<double>(total) * p1 / parts;
      const int64_t pick = std::fabs(static_cast<double>(wl) - target) <= std::fabs(static_cast<double>(wr) - target)
                               ? left
                               : right;
      if (pick > 0 && pick < cnt) cut = pick;
    }
    if (depth < 4 && cnt > 100000) {
      std::thread t([&] { run(rows, cut, p1, first, depth + 1); });
      run(rows + cut, cnt - cut, parts - p1, first + p1, depth + 1);
      t.join();
    } else {
      run(rows, cut, p1, first, depth + 1);
      run(rows + cut, cnt - cut, parts - p1, first + p1, depth + 1);
    }
  }
};

}  // namespace

extern "C" {

int64_t or_generate_nnz(int64_t nx, int64_t ny, int64_t nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return -1;
  // 7 per cell minus one per missing neighbour on each face of the box.
  return 7 * nx * ny * nz - 2 * (ny * nz + nx * nz + nx * ny);
}

int or_generate(int kind, int64_t nx, int64_t ny, int64_t nz, const double* params, uint64_t seed,
                int64_t* rows, int64_t* cols, double* vals, double* coords) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || kind < 0 || kind > 2) return 1;
  const int64_t n = nx * ny * nz;
  const int64_t step[6] = {-nx * ny, -nx, -1, 1, nx, nx * ny};
  std::vector<double> k;
  if (kind == 1) {
    k.resize(n);
    for (int64_t r = 0; r < n; ++r) k[r] = std::exp(params[0] * gauss(seed, static_cast<uint64_t>(r)));
  }
  double cd[6] = {0, 0, 0, 0, 0, 0}, cdDiag = 0;
  if (kind == 2) {
    cd[0] = -(1.0 + params[2]);
    cd[1] = -(1.0 + params[1]);
    cd[2] = -(1.0 + params[0]);
    cd[3] = cd[4] = cd[5] = -1.0;
    cdDiag = 6.0 + params[0] + params[1] + params[2];
  }
  int64_t o = 0;
  for (int64_t r = 0; r < n; ++r) {
    const int64_t i = r % nx, j = (r / nx) % ny, kk = r / (nx * ny);
    const bool in[6] = {kk > 0, j > 0, i > 0, i + 1 < nx, j + 1 < ny, kk + 1 < nz};
    double off[6], diag = 0;
    for (int d = 0; d < 6; ++d) {
      if (kind == 0) {
        off[d] = -1.0;
      } else if (kind == 2) {
        off[d] = cd[d];
      } else {
        const double a = k[r];
        const double f = in[d] ? 2.0 * a * k[r + step[d]] / (a + k[r + step[d]]) : 2.0 * a;
        off[d] = -f;
        diag += f;
      }
    }
    if (kind == 0) diag = 6.0;
    if (kind == 2) diag = cdDiag;
    for (int s = 0; s < 7; ++s) {
      const int d = s < 3 ? s : s - 1;
      if (s == 3) {
        rows[o] = r;
        cols[o] = r;
        vals[o] = diag;
        ++o;
      } else if (in[d]) {
        rows[o] = r;
        cols[o] = r + step[d];
        vals[o] = off[d];
        ++o;
      }
    }
    if (coords) {
      coords[3 * r] = static_cast<double>(i);
      coords[3 * r + 1] = static_cast<double>(j);
      coords[3 * r + 2] = static_cast<double>(kk);
    }
  }
  return o == or_generate_nnz(nx, ny, nz) ? 0 : 1;
}

int or_random_vector(uint64_t seed, int64_t n, int dist, double lo, double hi, double* out) {
  if (n < 0) return 1;
  for (int64_t i = 0; i < n; ++i)
    out[i] = dist == 0 ? lo + (hi - lo) * unit(seed, static_cast<uint64_t>(i)) : gauss(seed, static_cast<uint64_t>(i));
  return 0;
}

int or_partition_rcb(int64_t n, const double* coords, const int64_t* weights, int32_t parts, int32_t* out) {
  if (n < 0 || parts < 1) return 1;
  std::vector<int64_t> rows(static_cast<size_t>(n));
  std::iota(rows.begin(), rows.end(), int64_t(0));
  std::fill(out, out + n, 0);
  Rcb rcb{coords, weights, out};
  rcb.run(rows.data(), n, parts, 0, 0);
  return 0;
}

}  // extern "C"
