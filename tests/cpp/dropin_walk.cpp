// The call sequence of the reference's main.cpp:36-57 (chain of L sites, J = 1, h = 0; trial
// read from a file; Marsaglia(4) grid; MPSQMC2(...).Walk(n)) with the sizes taken from the
// command line:  dropin_walk <trial.mps> <DW> <Nwalkers> <dtau> <steps>
#include <cstdlib>
#include <iostream>

#include "GridGenerator.h"
#include "HeisenbergMPO.h"
#include "MPSQMC2.h"
#include "MPSstate.h"
#include "Random.h"

using namespace std;

int main(int argc, char **argv) {
  if (argc < 6) return 2;
  cout.precision(15);
  Random RN;
  MPSstate Psi0(argv[1], &RN);
  const int L = Psi0.gLength();
  HeisenbergMPO theMPO(L, 2, false);
  for (int cnt = 0; cnt < L - 1; cnt++) theMPO.sCoupling(cnt, cnt + 1, 1.0);
  theMPO.sField(0.0);
  GridGenerator theGrid(4);
  theGrid.FillMarsaglia(4);
  MPSQMC2 thePopulation(&theMPO, &theGrid, &RN, &Psi0, atoi(argv[2]), atoi(argv[3]), atof(argv[4]));
  thePopulation.Walk(atoi(argv[5]));
  return 0;
}
