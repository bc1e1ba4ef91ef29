// The reference's MPO-term projector driven as its sources allow (MPSQMC.h:15-31, main.cpp:136-144):
// chain of L sites, J = 1, h from the command line, term list built, MPSQMC(...).Walk(n).
//   dropin_legacy <L> <D> <Nwalkers> <dtau> <steps> <h>
#include <cstdlib>
#include <iostream>

#include "HeisenbergMPO.h"
#include "MPSQMC.h"
#include "Random.h"

using namespace std;

int main(int argc, char **argv) {
  if (argc < 7) return 2;
  cout.precision(15);
  const int L = atoi(argv[1]);
  HeisenbergMPO theMPO(L, 2, false);
  for (int cnt = 0; cnt < L - 1; cnt++) theMPO.sCoupling(cnt, cnt + 1, 1.0);
  theMPO.sField(atof(argv[6]));
  theMPO.findNonZeroContributions();
  Random RN;
  MPSQMC thePopulation(&theMPO, &RN, atoi(argv[2]), atoi(argv[3]), atof(argv[4]));
  thePopulation.Walk(atoi(argv[5]));
  return 0;
}
