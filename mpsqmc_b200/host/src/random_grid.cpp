// Random (one 32-bit Mersenne Twister, uniforms x / 2^32) and GridGenerator.
#include <cmath>
#include <cstdlib>
#include <ctime>
#include <vector>

#include "GridGenerator.h"
#include "Random.h"

Random::Random() {
  const char *s = getenv("MPSQMC_SEED");
  seed = s ? (uint32_t)strtoul(s, nullptr, 10) : (uint32_t)time(0);
  gen.seed(seed);
  draws = 0;
}
Random::~Random() {}
double Random::rand() {
  ++draws;
  return (double)gen() / 4294967296.0;
}
void Random::test() {
  for (int k = 0; k < 10; ++k) cout << "tID = 0 and RN = " << rand() << endl;
}
uint32_t Random::gSeed() const { return seed; }
unsigned long long Random::gDraws() const { return draws; }
void Random::discard(unsigned long long n) {
  gen.discard(n);
  draws += n;
}

GridGenerator::GridGenerator(const int d) : dim(d), gridFilled(false), nStates(0), grid(nullptr) {}
GridGenerator::~GridGenerator() { delete[] grid; }
int GridGenerator::gDim() const { return dim; }
int GridGenerator::gNPoints() const { return nStates; }
double GridGenerator::gCoOfPoint(const int point, const int index) const { return grid[index + dim * point]; }

namespace {
// inverse error function: bisection to a bracket, then Newton on erf
double erf_inverse(double z) {
  if (z == 0.0) return 0.0;
  const double sgn = z < 0 ? -1.0 : 1.0, t = std::fabs(z);
  double lo = 0.0, hi = 6.0;
  for (int it = 0; it < 60; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (std::erf(mid) < t) lo = mid; else hi = mid;
  }
  double x = 0.5 * (lo + hi);
  for (int it = 0; it < 4; ++it) x -= (std::erf(x) - t) / (1.1283791670955126 * std::exp(-x * x));
  return sgn * x;
}
}  // namespace

// Points from inverse-normal quantiles of pointsPerCo equally spaced levels in every
// coordinate, normalised, duplicates (distance^2 < 1e-16) dropped (GridGenerator.cpp:167-225).
void GridGenerator::FillMarsaglia(const int pointsPerCo) {
  std::vector<double> one(pointsPerCo);
  for (int c = 0; c < pointsPerCo; ++c) one[c] = erf_inverse(2 * (c + 0.5) / pointsPerCo - 1.0);
  long total = 1;
  for (int k = 0; k < dim; ++k) total *= pointsPerCo;
  std::vector<double> pts;
  std::vector<double> x(dim);
  for (long cnt = 0; cnt < total; ++cnt) {
    long cc = cnt;
    double nrm = 0.0;
    for (int k = 0; k < dim; ++k) {
      x[k] = one[cc % pointsPerCo];
      cc /= pointsPerCo;
      nrm += x[k] * x[k];
    }
    if (nrm <= 1e-16) continue;
    nrm = 1.0 / std::sqrt(nrm);
    for (int k = 0; k < dim; ++k) x[k] *= nrm;
    bool fresh = true;
    for (size_t p = 0; p < pts.size() / dim && fresh; ++p) {
      double d2 = 0.0;
      for (int k = 0; k < dim; ++k) d2 += (x[k] - pts[p * dim + k]) * (x[k] - pts[p * dim + k]);
      if (d2 < 1e-16) fresh = false;
    }
    if (fresh) pts.insert(pts.end(), x.begin(), x.end());
  }
  delete[] grid;
  nStates = (int)(pts.size() / dim);
  grid = new double[pts.size()];
  for (size_t q = 0; q < pts.size(); ++q) grid[q] = pts[q];
  gridFilled = true;
}

bool GridGenerator::GenerateNextSimple(int *state, const int denominator) {
  if (state[dim - 1] == denominator) return false;
  int index = dim - 2;
  while (state[index] == 0) --index;
  if (state[dim - 1] == 0) {
    state[index] -= 1;
    state[index + 1] += 1;
  } else {
    const int last = state[dim - 1];
    state[dim - 1] = 0;
    state[index + 1] += 1 + last;
    state[index] -= 1;
  }
  return true;
}

// Points +-sqrt(n_k / denominator) over all compositions n of the denominator, every sign
// pattern of the nonzero entries (GridGenerator.cpp:227-308).
void GridGenerator::FillSimple(const int denominator) {
  std::vector<int> st(dim, 0);
  std::vector<double> pts;
  st[0] = denominator;
  for (int sgn = 0; sgn < 2; ++sgn) {
    for (int k = 0; k < dim; ++k) pts.push_back(k == 0 ? (sgn ? -1.0 : 1.0) : 0.0);
  }
  while (GenerateNextSimple(st.data(), denominator)) {
    std::vector<int> nz;
    for (int k = 0; k < dim; ++k)
      if (st[k] > 0) nz.push_back(k);
    const int factor = 1 << nz.size();
    for (int c = 0; c < factor; ++c) {
      std::vector<double> p(dim, 0.0);
      for (size_t q = 0; q < nz.size(); ++q)
        p[nz[q]] = ((c >> q) & 1 ? -1.0 : 1.0) * std::sqrt((double)st[nz[q]] / denominator);
      pts.insert(pts.end(), p.begin(), p.end());
    }
  }
  delete[] grid;
  nStates = (int)(pts.size() / dim);
  grid = new double[pts.size()];
  for (size_t q = 0; q < pts.size(); ++q) grid[q] = pts[q];
  gridFilled = true;
}

ostream &operator<<(ostream &os, const GridGenerator &g) {
  const int D = g.gDim(), N = g.gNPoints();
  os << "GridGenerator print for Dim = " << D << endl << "The points:" << endl;
  std::vector<double> outer(D * D, 0.0);
  for (int p = 0; p < N; ++p) {
    os << "      Point " << p + 1 << "\t [";
    double n2 = 0.0;
    for (int a = 0; a < D; ++a) {
      const double v = g.gCoOfPoint(p, a);
      os << v << "\t";
      n2 += v * v;
      for (int b = 0; b < D; ++b) outer[a + D * b] += v * g.gCoOfPoint(p, b);
    }
    os << "] \t\t with 2-norm " << std::sqrt(n2) << endl;
  }
  os << "#vectors / dim = " << (double)N / D << " vs. sum over the outer product of the vectors:" << endl;
  for (int a = 0; a < D; ++a) {
    os << "      [ ";
    for (int b = 0; b < D; ++b) os << outer[a + D * b] << "\t";
    os << "]" << endl;
  }
  return os;
}
