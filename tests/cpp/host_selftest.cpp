// Drives the reference-compatible host classes (mpsqmc_b200/host) and prints JSON, so that
// tests/test_host_classes.py can compare them with the reference's golden outputs.
//   host_selftest grid
//   host_selftest trotter <dtau> <J>
//   host_selftest mpsops <trial.mps> <DW>
//   host_selftest dmrg <L> <D>
//   host_selftest energy <trial.mps>
//   host_selftest setup <trial.mps> <DW> <Nwalkers> <dtau>   (uniforms drawn by the set-up)
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "DMRG.h"
#include "GridGenerator.h"
#include "HeisenbergMPO.h"
#include "MPSQMC2.h"
#include "MPSstate.h"
#include "TrotterHeisenberg.h"
#include "Walker.h"

static void arr(const char *name, const double *v, size_t n, bool last = false) {
  printf("\"%s\": [", name);
  for (size_t i = 0; i < n; ++i) printf("%s%.17g", i ? ", " : "", v[i]);
  printf("]%s\n", last ? "" : ",");
}

static std::vector<double> flat(MPSstate &m, std::vector<double> *dims = nullptr) {
  std::vector<double> out;
  if (dims) dims->clear();
  for (int b = 0; b <= m.gLength(); ++b)
    if (dims) dims->push_back(m.gDimAtBound(b));
  for (int s = 0; s < m.gLength(); ++s) {
    const int n = m.gDimAtBound(s) * m.gDimAtBound(s + 1) * m.gPhys_d();
    out.insert(out.end(), m.gMPStensor(s)->gStorage(), m.gMPStensor(s)->gStorage() + n);
  }
  return out;
}

static void chain(HeisenbergMPO &mpo, int L) {
  for (int i = 0; i < L - 1; ++i) mpo.sCoupling(i, i + 1, 1.0);
  mpo.sField(0.0);
}

int main(int argc, char **argv) {
  std::streambuf *old = std::cout.rdbuf();
  std::stringstream sink;
  std::cout.rdbuf(sink.rdbuf());  // the classes' own progress lines are not part of the JSON
  const std::string mode = argc > 1 ? argv[1] : "";
  std::string json;
  if (mode == "grid") {
    GridGenerator a(4), b(4);
    a.FillMarsaglia(4);
    b.FillSimple(4);
    std::vector<double> pa, pb;
    for (int p = 0; p < a.gNPoints(); ++p)
      for (int k = 0; k < 4; ++k) pa.push_back(a.gCoOfPoint(p, k));
    for (int p = 0; p < b.gNPoints(); ++p)
      for (int k = 0; k < 4; ++k) pb.push_back(b.gCoOfPoint(p, k));
    std::cout.rdbuf(old);
    printf("{\n");
    arr("marsaglia", pa.data(), pa.size());
    arr("simple", pb.data(), pb.size(), true);
    printf("}\n");
  } else if (mode == "trotter") {
    const double dt = atof(argv[2]), J = atof(argv[3]);
    HeisenbergMPO mpo(4, 2, false);
    for (int i = 0; i < 3; ++i) mpo.sCoupling(i, i + 1, J);
    TrotterHeisenberg t(&mpo, dt);
    double U[16], S[4], VT[16];
    for (int k = 0; k < 4; ++k) {
      S[k] = t.gTwoSitePropSVD_Sing(J, k);
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
          U[i + 2 * (j + 2 * k)] = t.gTwoSitePropSVD_Left(J, k, i, j);
          VT[k + 4 * (i + 2 * j)] = t.gTwoSitePropSVD_Right(J, k, i, j);
        }
    }
    std::cout.rdbuf(old);
    printf("{\n");
    arr("U", U, 16);
    arr("S", S, 4);
    arr("VT", VT, 16, true);
    printf("}\n");
  } else if (mode == "mpsops") {
    Random RN;
    MPSstate psi(argv[2], &RN);
    const int DW = atoi(argv[3]);
    std::vector<double> sc;
    sc.push_back(psi.InnerProduct(&psi));
    MPSstate ln(&psi);
    sc.push_back(ln.LeftNormalize());
    MPSstate comp(&ln);
    comp.CompressState(DW);
    sc.push_back(ln.InnerProduct(&comp));
    sc.push_back(comp.InnerProduct(&comp));
    MPSstate rn(&psi);
    rn.RightNormalize();
    sc.push_back(rn.InnerProduct(&psi));
    std::vector<double> lnd = flat(ln), cdims, cd = flat(comp, &cdims);
    std::cout.rdbuf(old);
    printf("{\n");
    arr("scalars", sc.data(), sc.size());
    arr("leftnorm", lnd.data(), lnd.size());
    arr("compressed_dims", cdims.data(), cdims.size());
    arr("compressed", cd.data(), cd.size(), true);
    printf("}\n");
  } else if (mode == "dmrg") {
    const int L = atoi(argv[2]), D = atoi(argv[3]);
    HeisenbergMPO mpo(L, 2, false);
    chain(mpo, L);
    Random RN;
    MPSstate psi(L, D, 2, &RN);
    DMRG solver(&psi, &mpo);
    double E = solver.Solve();
    // <psi|H|psi> through ApplyMPO + InnerProduct
    psi.LeftNormalize();
    MPSstate hpsi(&psi);
    hpsi.ApplyMPO(&mpo, &psi);
    double E2 = hpsi.InnerProduct(&psi);
    hpsi.CompressState();
    double E3 = hpsi.InnerProduct(&psi);
    std::cout.rdbuf(old);
    double v[3] = {E, E2, E3};
    printf("{\n");
    arr("energies", v, 3, true);
    printf("}\n");
  } else if (mode == "energy") {
    Random RN;
    MPSstate psi(argv[2], &RN);
    const int L = psi.gLength();
    HeisenbergMPO mpo(L, 2, false);
    chain(mpo, L);
    psi.LeftNormalize();
    MPSstate hpsi(&psi);
    hpsi.ApplyMPO(&mpo, &psi);
    const double E = hpsi.InnerProduct(&psi);
    Walker w(&psi, 1.0, 1.0, 0.0);
    w.setOverlap(&psi);
    const double Ew = w.calcIndividualProjectedEnergy(&hpsi);
    std::cout.rdbuf(old);
    double v[2] = {E, Ew};
    printf("{\n");
    arr("energies", v, 2, true);
    printf("}\n");
  } else if (mode == "setup") {
    Random RN;
    MPSstate psi(argv[2], &RN);
    const int L = psi.gLength();
    HeisenbergMPO mpo(L, 2, false);
    chain(mpo, L);
    GridGenerator grid(4);
    grid.FillMarsaglia(4);
    std::streambuf *olderr = std::cerr.rdbuf();
    std::cerr.rdbuf(sink.rdbuf());  // no device here is not an error for this mode
    {
      MPSQMC2 q(&mpo, &grid, &RN, &psi, atoi(argv[3]), atoi(argv[4]), atof(argv[5]));
    }
    std::cerr.rdbuf(olderr);
    std::cout.rdbuf(old);
    printf("{\"draws\": %llu, \"seed\": %u}\n", (unsigned long long)RN.gDraws(), RN.gSeed());
  } else {
    std::cout.rdbuf(old);
    fprintf(stderr, "unknown mode\n");
    return 2;
  }
  return 0;
}
