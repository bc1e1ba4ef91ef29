// Test infrastructure (oracle side): a driver that links the UNMODIFIED reference sources
// (compiled in place from the reference tree by oracle/Makefile) and dumps what they compute,
// so the CPU restatement (oracle/mpsqmc_oracle.cpp) and the CUDA path can be checked against
// the reference itself.  Nothing in the product links or runs this file; only tests, the
// golden-fixture generator and bench.py's CPU-baseline leg execute the binary it builds.
//
// Modes (all write .npy / .json into <outdir>):
//   dmrg    <L> <D> <out.mps>                     two-site DMRG trial, DMRG.cpp:50-68
//   trotter <dtau> <J> <outdir>                   U,S,VT tables, TrotterHeisenberg.cpp:102-285
//   grid    <marsaglia|simple> <n> <outdir>       GridGenerator.cpp:167-308
//   mpsops  <trial.mps> <DW> <outdir>             InnerProduct / LeftNormalize / CompressState /
//                                                 ApplyTwoSiteTrotterTerm, MPSstate.cpp
//   walk    <trial.mps> <DW> <Nw> <dtau> <steps> <outdir> [trace] [tensors]
//                                                 MPSQMC2::Walk body (MPSQMC2.cpp:443-513),
//                                                 with per-coupling trace of 518-611
//   time    <trial.mps> <DW> <Nw> <dtau> <steps>  wall clock of MPSQMC2::Walk (stdout muted)
//   propagate <trial.mps> <DW> <Nw> <dtau> <steps>
//                                                 propagation-only timing for sizes whose
//                                                 H*Psi_T MPS and trial-term copies do not fit
// All runs use a 1D open Heisenberg chain J=1, h=0, d=2, as main.cpp:36-41 builds it.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include <chrono>
#include <sys/stat.h>
#include <omp.h>

// The walk driver needs MPSQMC2's private members (MPSQMC2.h:29-164) to replay the body of
// Walk step by step.  Access specifiers do not change the layout g++ gives these classes.
#define private public
#include "MPSQMC2.h"
#include "MPSQMC.h"
#undef private
#include "HeisenbergMPO.h"
#include "GridGenerator.h"
#include "TrotterHeisenberg.h"
#include "MPSstate.h"
#include "Random.h"
#include "DMRG.h"

namespace {

struct NullBuf : public std::streambuf {
  int overflow(int c) { return c; }
};
NullBuf g_nullbuf;

void save_npy(const std::string &path, const char *descr, const void *data, size_t elem,
              const std::vector<size_t> &shape) {
  std::ostringstream hdr;
  hdr << "{'descr': '" << descr << "', 'fortran_order': False, 'shape': (";
  size_t n = 1;
  for (size_t i = 0; i < shape.size(); ++i) {
    hdr << shape[i] << (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
    n *= shape[i];
  }
  hdr << "), }";
  std::string h = hdr.str();
  size_t total = 10 + h.size() + 1;
  size_t pad = (64 - total % 64) % 64;
  h.append(pad, ' ');
  h.push_back('\n');
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
  const char magic[] = "\x93NUMPY";
  fwrite(magic, 1, 6, f);
  unsigned char ver[2] = {1, 0};
  fwrite(ver, 1, 2, f);
  unsigned short hl = (unsigned short)h.size();
  fwrite(&hl, 2, 1, f);
  fwrite(h.data(), 1, h.size(), f);
  if (n) fwrite(data, elem, n, f);
  fclose(f);
}
void save_d(const std::string &p, const std::vector<double> &v) {
  save_npy(p, "<f8", v.data(), 8, std::vector<size_t>(1, v.size()));
}
void save_d2(const std::string &p, const std::vector<double> &v, size_t r, size_t c) {
  std::vector<size_t> s; s.push_back(r); s.push_back(c);
  save_npy(p, "<f8", v.data(), 8, s);
}
void save_i(const std::string &p, const std::vector<int> &v) {
  save_npy(p, "<i4", v.data(), 4, std::vector<size_t>(1, v.size()));
}
void save_i2(const std::string &p, const std::vector<int> &v, size_t r, size_t c) {
  std::vector<size_t> s; s.push_back(r); s.push_back(c);
  save_npy(p, "<i4", v.data(), 4, s);
}

// Flatten an MPS: bond dims (L+1) and the concatenated site storages (MPStensor.cpp:91-96).
void flatten(MPSstate *m, std::vector<int> &dims, std::vector<double> &data) {
  const int L = m->gLength(), d = m->gPhys_d();
  dims.assign(L + 1, 0);
  for (int b = 0; b <= L; ++b) dims[b] = m->gDimAtBound(b);
  data.clear();
  for (int s = 0; s < L; ++s) {
    const int n = dims[s] * dims[s + 1] * d;
    const double *st = m->gMPStensor(s)->gStorage();
    data.insert(data.end(), st, st + n);
  }
}
void save_mps(const std::string &prefix, MPSstate *m) {
  std::vector<int> dims; std::vector<double> data;
  flatten(m, dims, data);
  save_i(prefix + "_dims.npy", dims);
  save_d(prefix + "_data.npy", data);
}

// Chain of main.cpp:36-41; the field h comes from $MPSQMC_REF_FIELD (default 0, as main.cpp).
double field_from_env() {
  const char *f = getenv("MPSQMC_REF_FIELD");
  return f ? atof(f) : 0.0;
}

// Couplings: the chain of main.cpp:36-41 by default; $MPSQMC_REF_LATTICE = "snake:WxH" gives
// the open W x H square lattice along the snake path (even rows left to right, odd rows right
// to left), J = 1 on every nearest-neighbour pair, set through HeisenbergMPO::sCoupling as
// main.cpp:66-95 sets its periodic J1-J2 square lattice.
int snake_site(int W, int r, int c) { return r * W + ((r % 2 == 0) ? c : W - 1 - c); }

void build_chain(HeisenbergMPO &mpo, int L) {
  const char *lat = getenv("MPSQMC_REF_LATTICE");
  int W = 0, H = 0;
  if (lat && sscanf(lat, "snake:%dx%d", &W, &H) == 2 && W * H == L) {
    for (int r = 0; r < H; ++r)
      for (int c = 0; c < W; ++c) {
        const int s = snake_site(W, r, c);
        if (c + 1 < W) {
          const int t = snake_site(W, r, c + 1);
          mpo.sCoupling(std::min(s, t), std::max(s, t), 1.0);
        }
        if (r + 1 < H) {
          const int t = snake_site(W, r + 1, c);
          mpo.sCoupling(std::min(s, t), std::max(s, t), 1.0);
        }
      }
  } else {
    for (int i = 0; i < L - 1; ++i) mpo.sCoupling(i, i + 1, 1.0);
  }
  mpo.sField(field_from_env());
}

int trial_length(const char *file) {
  std::ifstream in(file);
  int L = 0;
  in >> L;
  return L;
}

void write_json(const std::string &path, const std::string &body) {
  std::ofstream o(path.c_str());
  o << body << std::endl;
}

std::string fmt17(double x) {
  char buf[64];
  snprintf(buf, sizeof buf, "%.17g", x);
  return buf;
}

int mode_dmrg(int argc, char **argv) {
  if (argc < 5) return 2;
  const int L = atoi(argv[2]), D = atoi(argv[3]);
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  HeisenbergMPO mpo(L, 2, false);
  build_chain(mpo, L);
  Random RN;
  MPSstate psi(L, D, 2, &RN);
  DMRG solver(&psi, &mpo);
  const double E = solver.Solve();
  std::cout.rdbuf(old);
  std::ofstream out(argv[4]);
  out.precision(17);
  out << psi << std::endl;
  printf("{\"energy\": %.17g, \"draws\": %llu, \"seed\": %u}\n", E,
         mpsqmc_compat::mt_draw_count(), mpsqmc_compat::mt_last_seed());
  return 0;
}

int mode_trotter(int argc, char **argv) {
  if (argc < 5) return 2;
  const double dtau = atof(argv[2]), J = atof(argv[3]);
  std::string out = argv[4];
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  HeisenbergMPO mpo(4, 2, false);
  for (int i = 0; i < 3; ++i) mpo.sCoupling(i, i + 1, J);
  mpo.sField(0.0);
  TrotterHeisenberg tr(&mpo, dtau);
  std::cout.rdbuf(old);
  const int d = 2, n = d * d;
  std::vector<double> U(n * n), S(n), VT(n * n);
  for (int k = 0; k < n; ++k) {
    S[k] = tr.gTwoSitePropSVD_Sing(J, k);
    for (int i = 0; i < d; ++i)
      for (int j = 0; j < d; ++j) {
        U[i + d * (j + d * k)] = tr.gTwoSitePropSVD_Left(J, k, i, j);
        VT[k + n * (i + d * j)] = tr.gTwoSitePropSVD_Right(J, k, i, j);
      }
  }
  save_d(out + "/U.npy", U);
  save_d(out + "/S.npy", S);
  save_d(out + "/VT.npy", VT);
  return 0;
}

int mode_grid(int argc, char **argv) {
  if (argc < 5) return 2;
  const int n = atoi(argv[3]);
  std::string out = argv[4];
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  GridGenerator g(4);
  if (std::string(argv[2]) == "marsaglia") g.FillMarsaglia(n); else g.FillSimple(n);
  std::cout.rdbuf(old);
  std::vector<double> pts(g.gNPoints() * 4);
  for (int p = 0; p < g.gNPoints(); ++p)
    for (int k = 0; k < 4; ++k) pts[k + 4 * p] = g.gCoOfPoint(p, k);
  save_d2(out + "/grid.npy", pts, g.gNPoints(), 4);
  return 0;
}

int mode_mpsops(int argc, char **argv) {
  if (argc < 5) return 2;
  const char *file = argv[2];
  const int DW = atoi(argv[3]);
  std::string out = argv[4];
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  Random RN;
  MPSstate psi(file, &RN);
  const int L = psi.gLength();
  save_mps(out + "/trial", &psi);
  std::vector<double> scal;
  // InnerProduct of the file state with itself, then LeftNormalize (MPSstate.cpp:216-229,248-284).
  scal.push_back(psi.InnerProduct(&psi));
  MPSstate ln(&psi);
  scal.push_back(ln.LeftNormalize());
  save_mps(out + "/leftnorm", &ln);
  // A second, random state of bond dimension DW (MPStensor.cpp:75-79 fills it).
  MPSstate other(L, DW, 2, &RN);
  save_mps(out + "/other", &other);
  scal.push_back(psi.InnerProduct(&other));
  scal.push_back(other.InnerProduct(&psi));
  MPSstate otherln(&other);
  scal.push_back(otherln.LeftNormalize());
  save_mps(out + "/other_leftnorm", &otherln);
  scal.push_back(ln.InnerProduct(&otherln));
  // Lossy two-sweep SVD compression to DW (MPSstate.cpp:379-404, TwoSiteObject.cpp:71-184).
  MPSstate comp(&ln);
  comp.CompressState(DW);
  save_mps(out + "/compressed", &comp);
  scal.push_back(ln.InnerProduct(&comp));
  // Site operators of the two-site propagator (MPSstate.cpp:505-633).
  HeisenbergMPO mpo(L, 2, false);
  build_chain(mpo, L);
  TrotterHeisenberg tr(&mpo, 0.01);
  GridGenerator g(4);
  g.FillMarsaglia(4);
  MPSstate gridop(&ln);
  gridop.ApplyTwoSiteTrotterTerm(&tr, 1, 2, &g, 37);
  save_mps(out + "/gridop_1_2_37", &gridop);
  MPSstate svdop(&ln);
  svdop.ApplyTwoSiteTrotterTerm(&tr, 2, 3, 1, 3, true);
  save_mps(out + "/svdop_2_3_1_3_hc", &svdop);
  scal.push_back(gridop.InnerProduct(&otherln));
  MPSstate ph(&ln);
  ph.ChangePhase();
  scal.push_back(ph.InnerProduct(&ln));
  std::cout.rdbuf(old);
  save_d(out + "/scalars.npy", scal);
  return 0;
}

// Per-walker trace of one PropagateSeparately pass, replaying MPSQMC2.cpp:533-598 with the
// reference objects so every intermediate (C_kl, PDF norm, uniform, grid index, weight,
// overlap) can be recorded.  Called with OMP_NUM_THREADS=1, thread id 0.
struct Trace {
  std::vector<double> C, pdfnorm, u, weight, overlap;
  std::vector<int> index;
};

double propagate_traced(MPSQMC2 &q, Trace &tr) {
  const int myID = 0;
  double sum = 0.0;
  for (int walker = 0; walker < q.NCurrentWalkersPerRank[q.MPIrank]; ++walker) {
    Walker *W = q.theWalkers[walker];
    W->gState()->ApplyOneSiteTrotterTermEverywhere(q.theTrotter);
    W->setOverlap(q.Psi0[myID]);
    for (int t = 0; t < q.nCouplings; ++t) {
      for (int a = 0; a < q.trotterSVDsize; ++a)
        for (int b = 0; b < q.trotterSVDsize; ++b) {
          const int ci = a + q.trotterSVDsize * b;
          q.theOperatorCombos[myID][ci] =
              q.TrotterTermsTimesPsi0[myID][t][ci]->InnerProduct(W->gState());
        }
      // stored in combined-index order C[firstOp + d^2*secondOp] (MPSQMC2.cpp:543)
      for (int ci = 0; ci < q.trotterSVDsize * q.trotterSVDsize; ++ci)
        tr.C.push_back(q.theOperatorCombos[myID][ci]);
      double norm = 0.0;
      const int G = q.theGrid->gNPoints();
      for (int p = 0; p < G; ++p) {
        double v = 0.0;
        for (int l = 0; l < q.trotterSVDsize; ++l)
          for (int r = 0; r < q.trotterSVDsize; ++r)
            v += q.theOperatorCombos[myID][l + q.trotterSVDsize * r] * q.theGrid->gCoOfPoint(p, l) *
                 q.theGrid->gCoOfPoint(p, r);
        v = std::max(0.0, v);
        v *= q.trotterSVDsize / (W->gOverlap() * G);
        q.thePDF[myID][p] = v;
        norm += v;
      }
      const double inv = 1.0 / norm;
      for (int p = 0; p < G; ++p) q.thePDF[myID][p] *= inv;
      W->multiplyWeight(norm);
      const double u = q.RN->rand();
      int count = 0;
      double cum = q.thePDF[myID][0];
      while ((cum <= u) && (count < G - 1)) {
        count += 1;
        cum += q.thePDF[myID][count];
      }
      W->gState()->ApplyTwoSiteTrotterTerm(q.theTrotter, q.firstIndexCoupling[t],
                                           q.secondIndexCoupling[t], q.theGrid, count);
      W->setOverlap(q.Psi0[myID]);
      tr.pdfnorm.push_back(norm);
      tr.u.push_back(u);
      tr.index.push_back(count);
      tr.weight.push_back(W->gWeight());
      tr.overlap.push_back(W->gOverlap());
    }
    W->gState()->ApplyOneSiteTrotterTermEverywhere(q.theTrotter);
    W->setOverlap(q.Psi0[myID]);
    sum += W->gWeight();
  }
  return sum;
}

int mode_walk(int argc, char **argv) {
  if (argc < 8) return 2;
  const char *file = argv[2];
  const int DW = atoi(argv[3]), Nw = atoi(argv[4]);
  const double dtau = atof(argv[5]);
  const int steps = atoi(argv[6]);
  std::string out = argv[7];
  bool trace = false, tensors = false;
  for (int i = 8; i < argc; ++i) {
    if (std::string(argv[i]) == "trace") trace = true;
    if (std::string(argv[i]) == "tensors") tensors = true;
  }
  const int L = trial_length(file);
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  HeisenbergMPO mpo(L, 2, false);
  build_chain(mpo, L);
  Random RN;
  MPSstate psi(file, &RN);
  GridGenerator grid(4);
  grid.FillMarsaglia(4);
  MPSQMC2 q(&mpo, &grid, &RN, &psi, DW, Nw, dtau);
  const unsigned long long setup_draws = mpsqmc_compat::mt_draw_count();
  std::cout.rdbuf(old);

  // Static inputs the other implementations need to replay this run.
  save_mps(out + "/trial_ln", q.Psi0[0]);
  save_mps(out + "/walker0_init", q.theWalkers[0]->gState());
  {
    // the coupling list in the order PropagateSeparately walks it (MPSQMC2.cpp:286-299)
    std::vector<int> ci(q.nCouplings), cj(q.nCouplings);
    std::vector<double> cJ(q.nCouplings);
    for (int c = 0; c < q.nCouplings; ++c) {
      ci[c] = q.firstIndexCoupling[c];
      cj[c] = q.secondIndexCoupling[c];
      cJ[c] = q.theTrotter->gCoupling(ci[c], cj[c]);
    }
    save_i(out + "/coup_i.npy", ci);
    save_i(out + "/coup_j.npy", cj);
    save_d(out + "/coup_J.npy", cJ);
  }
  {
    const int d = 2, n = 4;
    std::vector<double> U(16), S(4), VT(16);
    const double J = 1.0;
    for (int k = 0; k < n; ++k) {
      S[k] = q.theTrotter->gTwoSitePropSVD_Sing(J, k);
      for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
          U[i + d * (j + d * k)] = q.theTrotter->gTwoSitePropSVD_Left(J, k, i, j);
          VT[k + n * (i + d * j)] = q.theTrotter->gTwoSitePropSVD_Right(J, k, i, j);
        }
    }
    save_d(out + "/U.npy", U);
    save_d(out + "/S.npy", S);
    save_d(out + "/VT.npy", VT);
    std::vector<double> pts(grid.gNPoints() * 4);
    for (int p = 0; p < grid.gNPoints(); ++p)
      for (int k = 0; k < 4; ++k) pts[k + 4 * p] = grid.gCoOfPoint(p, k);
    save_d2(out + "/grid.npy", pts, grid.gNPoints(), 4);
  }
  double E0 = 0.0;
  q.EnergyFunctionAndHistory(1, &E0, false);
  {
    std::vector<double> ov0, w0;
    for (int w = 0; w < q.NCurrentWalkersPerRank[0]; ++w) {
      ov0.push_back(q.theWalkers[w]->gOverlap());
      w0.push_back(q.theWalkers[w]->gWeight());
    }
    save_d(out + "/init_overlap.npy", ov0);
    save_d(out + "/init_weight.npy", w0);
  }

  std::vector<double> stat_sumw, stat_EP, stat_ET, stat_omega, stat_scaling;
  std::vector<int> stat_n, stat_draws;
  for (int step = 1; step <= steps; ++step) {
    char pre[256];
    snprintf(pre, sizeof pre, "%s/step%03d_", out.c_str(), step);
    const unsigned long long d0 = mpsqmc_compat::mt_draw_count();
    Trace tr;
    std::cout.rdbuf(&g_nullbuf);
    const double sumw = trace ? propagate_traced(q, tr) : q.PropagateSeparately();
    std::cout.rdbuf(old);
    const int N = q.totalNCurrentWalkers;
    const double avgW = sumw / N;
    const double scaling = q.totalNDesiredWalkers / (N * avgW);
    const double ET = std::log(scaling) / q.dtau;
    std::vector<double> wts, ovs, ens;
    for (int w = 0; w < N; ++w) {
      Walker *W = q.theWalkers[w];
      wts.push_back(W->gWeight());
      ovs.push_back(W->gOverlap());
      ens.push_back(W->calcIndividualProjectedEnergy(q.HPsi0[0]));
      if (tensors) {
        char nm[64];
        snprintf(nm, sizeof nm, "walker%04d", w);
        save_mps(std::string(pre) + nm, W->gState());
      }
    }
    double EP = 0.0;
    const double omega = q.EnergyFunctionAndHistory(step, &EP, true);
    std::vector<double> hist;
    for (int w = 0; w < N; ++w) hist.push_back(q.theWalkers[w]->gEnergyHistory());
    // Threshold branching (MPSQMC2.cpp:613-686); parents recovered from pointer identity,
    // since copies are appended directly after their original (660-665).
    std::vector<Walker *> before(q.theWalkers, q.theWalkers + N);
    const unsigned long long d1 = mpsqmc_compat::mt_draw_count();
    std::cout.rdbuf(&g_nullbuf);
    q.SeparatePopulationControl(scaling);
    std::cout.rdbuf(old);
    const unsigned long long d2 = mpsqmc_compat::mt_draw_count();
    const int Nn = q.totalNCurrentWalkers;
    std::vector<int> parent(Nn, -1);
    std::vector<double> newW(Nn);
    int last = -1;
    for (int k = 0; k < Nn; ++k) {
      for (int w = 0; w < N; ++w)
        if (q.theWalkers[k] == before[w]) { last = w; break; }
      parent[k] = last;
      newW[k] = q.theWalkers[k]->gWeight();
    }
    save_d(std::string(pre) + "weight.npy", wts);
    save_d(std::string(pre) + "overlap.npy", ovs);
    save_d(std::string(pre) + "energy.npy", ens);
    save_d(std::string(pre) + "ehist.npy", hist);
    save_i(std::string(pre) + "parent.npy", parent);
    save_d(std::string(pre) + "newweight.npy", newW);
    if (trace) {
      save_d2(std::string(pre) + "trace_C.npy", tr.C, tr.C.size() / 16, 16);
      save_d(std::string(pre) + "trace_pdfnorm.npy", tr.pdfnorm);
      save_d(std::string(pre) + "trace_u.npy", tr.u);
      save_i(std::string(pre) + "trace_index.npy", tr.index);
      save_d(std::string(pre) + "trace_weight.npy", tr.weight);
      save_d(std::string(pre) + "trace_overlap.npy", tr.overlap);
    }
    stat_sumw.push_back(sumw);
    stat_EP.push_back(EP);
    stat_ET.push_back(ET);
    stat_omega.push_back(omega);
    stat_scaling.push_back(scaling);
    stat_n.push_back(N);
    stat_draws.push_back((int)(d1 - d0));
    stat_draws.push_back((int)(d2 - d1));
  }
  save_d(out + "/stat_sumw.npy", stat_sumw);
  save_d(out + "/stat_EP.npy", stat_EP);
  save_d(out + "/stat_ET.npy", stat_ET);
  save_d(out + "/stat_omega.npy", stat_omega);
  save_d(out + "/stat_scaling.npy", stat_scaling);
  save_i(out + "/stat_n.npy", stat_n);
  save_i2(out + "/stat_draws.npy", stat_draws, stat_draws.size() / 2, 2);
  std::ostringstream js;
  js << "{\"L\": " << L << ", \"DW\": " << DW << ", \"DT\": " << q.DT << ", \"Nw\": " << Nw
     << ", \"dtau\": " << fmt17(dtau) << ", \"steps\": " << steps
     << ", \"seed\": " << mpsqmc_compat::mt_last_seed() << ", \"setup_draws\": " << setup_draws
     << ", \"E0\": " << fmt17(E0) << ", \"nCouplings\": " << q.nCouplings
     << ", \"G\": " << grid.gNPoints() << ", \"h\": " << fmt17(field_from_env())
     << ", \"lattice\": \"" << (getenv("MPSQMC_REF_LATTICE") ? getenv("MPSQMC_REF_LATTICE") : "chain") << "\"}";
  write_json(out + "/meta.json", js.str());
  return 0;
}

int mode_time(int argc, char **argv) {
  if (argc < 7) return 2;
  const char *file = argv[2];
  const int DW = atoi(argv[3]), Nw = atoi(argv[4]);
  const double dtau = atof(argv[5]);
  const int steps = atoi(argv[6]);
  char tmpl[] = "/tmp/mpsqmc_ref_XXXXXX";
  if (!mkdtemp(tmpl)) return 3;
  std::string trial_abs = file;
  if (file[0] != '/') {
    char cwd[4096];
    if (getcwd(cwd, sizeof cwd)) trial_abs = std::string(cwd) + "/" + file;
  }
  if (chdir(tmpl) != 0) return 3;
  mkdir("output", 0755);
  mkdir("output/Heisenberg1D", 0755);
  const int L = trial_length(trial_abs.c_str());
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  HeisenbergMPO mpo(L, 2, false);
  build_chain(mpo, L);
  Random RN;
  MPSstate psi(trial_abs.c_str(), &RN);
  GridGenerator grid(4);
  grid.FillMarsaglia(4);
  MPSQMC2 q(&mpo, &grid, &RN, &psi, DW, Nw, dtau);
  const auto t0 = std::chrono::steady_clock::now();
  q.Walk(steps);
  const auto t1 = std::chrono::steady_clock::now();
  std::cout.rdbuf(old);
  const double sec = std::chrono::duration<double>(t1 - t0).count();
  printf("{\"walker_steps\": %lld, \"seconds\": %.6f, \"walker_steps_per_s\": %.6f, \"threads\": %d, "
         "\"kind\": \"reference MPSQMC2::Walk\"}\n",
         (long long)Nw * steps, sec, (double)Nw * steps / sec, omp_get_max_threads());
  return 0;
}

// Propagation-only timing over the reference classes: the reference's MPSQMC2 ctor keeps
// nC*16 trial-term copies per thread and builds H*Psi_T with bond up to MPOdim*D_T, neither
// of which fits for L=64, D_T=64.  This mode builds the 16 trial terms of one coupling at a
// time per thread (same objects, MPSQMC2.cpp:303-330) and runs the per-walker body of
// PropagateSeparately (533-598) coupling-major; energy is not computed.
int mode_propagate(int argc, char **argv) {
  if (argc < 7) return 2;
  const char *file = argv[2];
  const int DW = atoi(argv[3]), Nw = atoi(argv[4]);
  const double dtau = atof(argv[5]);
  const int steps = atoi(argv[6]);
  const int L = trial_length(file);
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  HeisenbergMPO mpo(L, 2, false);
  build_chain(mpo, L);
  Random RN;
  MPSstate psi(file, &RN);
  psi.LeftNormalize();
  GridGenerator grid(4);
  grid.FillMarsaglia(4);
  TrotterHeisenberg trot(&mpo, dtau);
  Walker w0(&psi, 1.0, 1.0, 0.0);
  if (DW < psi.gDtrunc()) {
    w0.gState()->CompressState(DW);
    w0.setOverlap(&psi);
  }
  std::vector<Walker *> walkers;
  for (int i = 0; i < Nw; ++i) walkers.push_back(new Walker(&w0));
  const int nth = omp_get_max_threads();
  std::vector<MPSstate *> trials(nth);
  for (int t = 0; t < nth; ++t) trials[t] = new MPSstate(&psi);
  const int G = grid.gNPoints();
  // the non-zero couplings in the order MPSQMC2.cpp:286-299 lists them
  std::vector<int> ci, cj;
  for (int i = 0; i < L - 1; ++i)
    for (int j = i + 1; j < L; ++j)
      if (trot.gCoupling(i, j) != 0.0) {
        ci.push_back(i);
        cj.push_back(j);
      }
  const int nC = (int)ci.size();
  // $MPSQMC_REF_MAX_COUPLINGS = k: time the first k couplings of each walker-step only (large
  // lattices); the rate is then extrapolated to all nC couplings
  const char *mk = getenv("MPSQMC_REF_MAX_COUPLINGS");
  const int ntime = (mk && atoi(mk) > 0) ? std::min(nC, atoi(mk)) : nC;
  std::cout.rdbuf(old);
  const auto t0 = std::chrono::steady_clock::now();
  for (int step = 0; step < steps; ++step) {
#pragma omp parallel
    {
      const int tid = omp_get_thread_num();
      std::vector<double> C(16), pdf(G);
      std::vector<MPSstate *> terms(16, (MPSstate *)0);
      for (int w = tid; w < Nw; w += nth) {
        Walker *W = walkers[w];
        W->gState()->ApplyOneSiteTrotterTermEverywhere(&trot);
        W->setOverlap(trials[tid]);
        for (int c = 0; c < ntime; ++c) {
          for (int k = 0; k < 16; ++k) {
            delete terms[k];
            terms[k] = new MPSstate(trials[tid]);
            terms[k]->ApplyTwoSiteTrotterTerm(&trot, ci[c], cj[c], k % 4, k / 4, true);
            C[k] = terms[k]->InnerProduct(W->gState());
          }
          double norm = 0.0;
          for (int p = 0; p < G; ++p) {
            double v = 0.0;
            for (int l = 0; l < 4; ++l)
              for (int r = 0; r < 4; ++r)
                v += C[l + 4 * r] * grid.gCoOfPoint(p, l) * grid.gCoOfPoint(p, r);
            v = std::max(0.0, v) * 4.0 / (W->gOverlap() * G);
            pdf[p] = v;
            norm += v;
          }
          for (int p = 0; p < G; ++p) pdf[p] /= norm;
          W->multiplyWeight(norm);
          const double u = RN.rand();
          int count = 0;
          double cum = pdf[0];
          while (cum <= u && count < G - 1) cum += pdf[++count];
          W->gState()->ApplyTwoSiteTrotterTerm(&trot, ci[c], cj[c], &grid, count);
          W->setOverlap(trials[tid]);
        }
        W->gState()->ApplyOneSiteTrotterTermEverywhere(&trot);
        W->setOverlap(trials[tid]);
      }
      for (int k = 0; k < 16; ++k) delete terms[k];
    }
  }
  const auto t1 = std::chrono::steady_clock::now();
  const double sec = std::chrono::duration<double>(t1 - t0).count();
  const double full = sec * (double)nC / (double)ntime;  // all couplings (extrapolated when ntime < nC)
  printf("{\"walker_steps\": %lld, \"seconds\": %.6f, \"walker_steps_per_s\": %.6f, \"threads\": %d, "
         "\"couplings_timed\": %d, \"couplings\": %d, \"measured_seconds\": %.6f, "
         "\"kind\": \"reference classes, propagation only (no energy)\"}\n",
         (long long)Nw * steps, full, (double)Nw * steps / full, nth, ntime, nC, sec);
  for (size_t i = 0; i < walkers.size(); ++i) delete walkers[i];
  for (int t = 0; t < nth; ++t) delete trials[t];
  return 0;
}

}  // namespace

// OpenBLAS (the LAPACK/BLAS these sources link against) runs its own thread pool; the
// reference's parallelism is OpenMP over walkers, so BLAS calls stay single-threaded.
extern "C" void openblas_set_num_threads(int);

// Legacy MPO-term projector (MPSQMC.cpp): MPSQMC(mpo, RN, D, Nw, dtau) builds its own DMRG trial
// and walkers; the body of MPSQMC::Walk (MPSQMC.cpp:236-318) is replayed step by step so that
// per-walker quantities can be saved:
//   legacy <L> <D> <Nw> <dtau> <steps> <outdir>
int mode_legacy(int argc, char **argv) {
  if (argc < 8) return 2;
  const int L = atoi(argv[2]), D = atoi(argv[3]), Nw = atoi(argv[4]);
  const double dtau = atof(argv[5]);
  const int steps = atoi(argv[6]);
  const std::string out = argv[7];
  std::streambuf *old = std::cout.rdbuf(&g_nullbuf);
  HeisenbergMPO mpo(L, 2, false);
  build_chain(mpo, L);
  mpo.findNonZeroContributions();  // the terms MPSQMC samples (main.cpp:144)
  Random RN;
  MPSQMC q(&mpo, &RN, D, Nw, dtau);
  const unsigned long long setup_draws = mpsqmc_compat::mt_draw_count();
  std::cout.rdbuf(old);
  save_mps(out + "/trial_ln", q.Psi0[0]);
  {  // the MPO terms the projector samples (HeisenbergMPO.cpp:456-553): prefactor, sites, ops
    std::vector<double> pref;
    std::vector<int> sites, ops;
    for (int t = 0; t < mpo.gRN_nTerms(); ++t) {
      pref.push_back(mpo.gRN_prefactor(t));
      int s0 = -1, s1 = -1, o0 = -1, o1 = -1;
      for (int k = 0; k < L; ++k) {
        Operator *op = mpo.gRN_operator(t, k);
        if (op->AmIOpI()) continue;
        const int code = (op == mpo.gRN_operator(t, k) && (*op)(0, 1) != 0.0) ? (((*op)(0, 1) == (*op)(1, 0)) ? 1 : 2) : 3;
        if (s0 < 0) { s0 = k; o0 = code; } else { s1 = k; o1 = code; }
      }
      sites.push_back(s0); sites.push_back(s1); ops.push_back(o0); ops.push_back(o1);
    }
    save_d(out + "/terms_prefactor.npy", pref);
    save_i2(out + "/terms_sites.npy", sites, pref.size(), 2);
    save_i2(out + "/terms_ops.npy", ops, pref.size(), 2);  // 1 Sx, 2 iSy, 3 Sz
  }
  std::vector<double> stat_sum, stat_EP, stat_ET, stat_omega, stat_scaling;
  std::vector<int> stat_n, stat_draws;
  const double E0 = q.EnergyFunction();
  for (int step = 1; step <= steps; ++step) {
    const unsigned long long d0 = mpsqmc_compat::mt_draw_count();
    std::cout.rdbuf(&g_nullbuf);
    const double sum = q.PropagateSeparately();
    std::cout.rdbuf(old);
    const int N = q.myNCurrentWalkers;
    std::vector<double> coeff(q.walkerCoeff, q.walkerCoeff + N), ov(q.walkerOverlap, q.walkerOverlap + N), en(N);
    for (int w = 0; w < N; ++w) en[w] = q.HPsi0[0]->InnerProduct(q.theWalkers[w]) / q.walkerOverlap[w];
    char pre[64];
    snprintf(pre, sizeof pre, "%s/step%03d_", out.c_str(), step);
    save_d(std::string(pre) + "weight.npy", coeff);
    save_d(std::string(pre) + "overlap.npy", ov);
    save_d(std::string(pre) + "energy.npy", en);
    const double avgCoeff = sum / q.totalNCurrentWalkers;
    const double omega = q.updateEnergyHistory(step);
    const double EP = q.EnergyFunction();
    const double scaling = q.totalNDesiredWalkers / (q.totalNCurrentWalkers * avgCoeff);
    const double ET = std::log(scaling) / dtau;
    const unsigned long long d1 = mpsqmc_compat::mt_draw_count();
    std::cout.rdbuf(&g_nullbuf);
    q.SeparatePopulationControl(scaling);
    std::cout.rdbuf(old);
    q.totalNCurrentWalkers = q.myNCurrentWalkers;
    const unsigned long long d2 = mpsqmc_compat::mt_draw_count();
    const int Nn = q.myNCurrentWalkers;
    std::vector<double> ov2(q.walkerOverlap, q.walkerOverlap + Nn), eh2(q.walkerEnergyHistorySum,
                                                                     q.walkerEnergyHistorySum + Nn);
    save_d(std::string(pre) + "newoverlap.npy", ov2);
    save_d(std::string(pre) + "newehist.npy", eh2);
    if (step == steps) {
      for (int w = 0; w < Nn; ++w) {
        char nm[96];
        snprintf(nm, sizeof nm, "%swalker%04d", pre, w);
        save_mps(nm, q.theWalkers[w]);
      }
    }
    stat_sum.push_back(sum);
    stat_EP.push_back(EP);
    stat_ET.push_back(ET);
    stat_omega.push_back(omega);
    stat_scaling.push_back(scaling);
    stat_n.push_back(N);
    stat_draws.push_back((int)(d1 - d0));
    stat_draws.push_back((int)(d2 - d1));
  }
  save_d(out + "/stat_sum.npy", stat_sum);
  save_d(out + "/stat_EP.npy", stat_EP);
  save_d(out + "/stat_ET.npy", stat_ET);
  save_d(out + "/stat_omega.npy", stat_omega);
  save_d(out + "/stat_scaling.npy", stat_scaling);
  save_i(out + "/stat_n.npy", stat_n);
  save_i2(out + "/stat_draws.npy", stat_draws, stat_draws.size() / 2, 2);
  std::ostringstream js;
  js << "{\"L\": " << L << ", \"D\": " << D << ", \"Nw\": " << Nw << ", \"dtau\": " << fmt17(dtau)
     << ", \"steps\": " << steps << ", \"seed\": " << mpsqmc_compat::mt_last_seed()
     << ", \"setup_draws\": " << setup_draws << ", \"E0\": " << fmt17(E0)
     << ", \"nTerms\": " << mpo.gRN_nTerms() << ", \"h\": " << fmt17(field_from_env()) << "}";
  write_json(out + "/meta.json", js.str());
  return 0;
}

int main(int argc, char **argv) {
  openblas_set_num_threads(1);
  if (argc < 2) {
    fprintf(stderr, "usage: ref_harness <dmrg|trotter|grid|mpsops|walk|time|propagate|legacy> ...\n");
    return 2;
  }
  std::cout.precision(17);
  const std::string m = argv[1];
  int rc = 2;
  if (m == "dmrg") rc = mode_dmrg(argc, argv);
  else if (m == "trotter") rc = mode_trotter(argc, argv);
  else if (m == "grid") rc = mode_grid(argc, argv);
  else if (m == "mpsops") rc = mode_mpsops(argc, argv);
  else if (m == "walk") rc = mode_walk(argc, argv);
  else if (m == "time") rc = mode_time(argc, argv);
  else if (m == "propagate") rc = mode_propagate(argc, argv);
  else if (m == "legacy") rc = mode_legacy(argc, argv);
  if (rc == 2) fprintf(stderr, "bad arguments for mode %s\n", m.c_str());
  return rc;
}
