// Test-oracle harness around the UNMODIFIED reference program (compiled from
// its own sources by oracle/Makefile into oracle/_ref/).  It is test
// infrastructure: only tests/, the smoke check and bench.py's CPU-baseline
// leg run it.
//
// It builds a Meamzilla object exactly as src/main.cpp does (parameter file,
// potential file, configuration file, pair/triplet lists) and then drives the
// objective through the reference's own public interface:
//   Potential::compute(const Comm&, ErrorVec*)    src/potential.h:67
//   Potential::coeff(int)                          src/potential.h:60
//   PotEAM::compute_densities                      src/pots/pot_eam/pot_eam.h:45
//
// Usage:
//   mzref -p <param> [-x <coeff.bin>] [-o <prefix>] [-reps K] [-fd h] [-q]
//     -x     raw float64 file with get_ncoeff() values, applied via coeff(i)
//     -o     write <prefix>.{obj,errvec,energy,stress,force,dens,coeff}.bin
//            (raw little-endian float64; forces in configuration order)
//     -reps  time K back-to-back compute() calls (no ErrorVec) after one
//            warm-up; prints "seconds_per_eval <t>"
//     -fd    central finite-difference gradient of the objective with step h
//            for every coefficient -> <prefix>.fdgrad.bin
//     -write P  Potential::write_data(comm, P, -1) (src/potential.cpp:325-342):
//            P.rho/.energy/.stress/.force/.error/.punish, after -x / -rescale
//     -rescale F  call Potential::rescale(comm, out, F) (src/potential.h:68)
//            after -x, then dump every spline -> <prefix>.rescale.bin:
//            [returned value, nsplines, per spline: n, x[n], y[n], grad[2],
//            natural[2], step] (function groups in file order)
//     -powell K  the reference's own Powell optimizer (OptPowell::compute_pot,
//            src/opt_powell.cpp:96-315) from the -x start, for k = 1..K
//            outer steps each from that same start -> <prefix>.powell.bin:
//            per k the objective of the returned potential and its
//            get_ncoeff() coefficients
#define protected public
#include "meamzilla.h"
#include "universe.h"
#include "config.h"
#include "cell.h"
#include "atom.h"
#include "pot_list.h"
#include "potential.h"
#include "pots/pot_eam/pot_eam.h"
#include "pot_fns.h"
#include "spline3eq.h"
#include "opt_powell.h"
#undef protected

#include <chrono>
#include <fcntl.h>
#include <iostream>
#include <unistd.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace MEAMZ_NS;

static void dump(const std::string &path, const std::vector<double> &v) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) { std::fprintf(stderr, "mzref: cannot write %s\n", path.c_str()); std::exit(2); }
  if (!v.empty()) std::fwrite(v.data(), sizeof(double), v.size(), f);
  std::fclose(f);
}

int main(int argc, char **argv) {
  std::string param, xfile, prefix, write_prefix;
  int reps = 0, quiet = 0, rescale_flag = 0, powell_steps = 0;
  bool do_rescale = false;
  double fd_h = 0.0;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "-p" && i + 1 < argc) param = argv[++i];
    else if (a == "-x" && i + 1 < argc) xfile = argv[++i];
    else if (a == "-o" && i + 1 < argc) prefix = argv[++i];
    else if (a == "-reps" && i + 1 < argc) reps = std::atoi(argv[++i]);
    else if (a == "-fd" && i + 1 < argc) fd_h = std::atof(argv[++i]);
    else if (a == "-write" && i + 1 < argc) write_prefix = argv[++i];
    else if (a == "-rescale" && i + 1 < argc) rescale_flag = std::atoi(argv[++i]), do_rescale = true;
    else if (a == "-q") quiet = 1;
    else if (a == "-powell" && i + 1 < argc) powell_steps = std::atoi(argv[++i]);
    else { std::fprintf(stderr, "mzref: bad argument %s\n", a.c_str()); return 2; }
  }
  if (param.empty()) { std::fprintf(stderr, "mzref: -p <param> required\n"); return 2; }

  MPI_Init(&argc, &argv);
  // Silence the reference's progress prints when asked (they go to stdout).
  int saved_stdout = -1;
  if (quiet) {
    std::fflush(stdout);
    saved_stdout = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    dup2(devnull, 1);
    close(devnull);
  }
  char *margv[3] = {argv[0], (char *)"-p", (char *)param.c_str()};
  Meamzilla *mmz = new Meamzilla(3, margv, MPI_COMM_WORLD);
  if (quiet) {
    std::cout.flush();
    std::fflush(stdout);
    dup2(saved_stdout, 1);
    close(saved_stdout);
  }

  const Comm &comm = mmz->universe->comm_inter;
  Potential *pot = mmz->potlist->at(0);
  const int ncoeff = pot->get_ncoeff();

  if (!xfile.empty()) {
    std::vector<double> x(ncoeff);
    FILE *f = std::fopen(xfile.c_str(), "rb");
    if (!f || std::fread(x.data(), sizeof(double), ncoeff, f) != (size_t)ncoeff) {
      std::fprintf(stderr, "mzref: cannot read %d coefficients from %s\n", ncoeff, xfile.c_str());
      return 2;
    }
    std::fclose(f);
    for (int i = 0; i < ncoeff; ++i) pot->coeff(i) = x[i];
  }

  if (do_rescale) {
    const int ret = pot->rescale(comm, &std::cerr, rescale_flag);
    std::vector<double> out{(double)ret, 0.0};
    int nspl = 0;
    for (PotFns &pf : pot->pot_fns_)
      for (Basis *b : pf.fns) {
        Spline3Eq *sp = dynamic_cast<Spline3Eq *>(b);
        if (!sp) { std::fprintf(stderr, "mzref: rescale dump supports spline3eq only\n"); return 2; }
        out.push_back((double)sp->nknots_);
        out.insert(out.end(), sp->x_.begin(), sp->x_.end());
        out.insert(out.end(), sp->y_.begin(), sp->y_.end());
        out.push_back(sp->grad_[0]);
        out.push_back(sp->grad_[1]);
        out.push_back((double)sp->is_nat_[0]);
        out.push_back((double)sp->is_nat_[1]);
        out.push_back(sp->step_);
        ++nspl;
      }
    out[1] = (double)nspl;
    if (!prefix.empty()) dump(prefix + ".rescale.bin", out);
  }

  if (!write_prefix.empty()) pot->write_data(comm, write_prefix, -1);

  if (powell_steps > 0) {
    OptPowell opt(mmz, nullptr);
    std::vector<double> out;
    for (int k = 1; k <= powell_steps; ++k) {
      Potential *p = opt.compute_pot(pot, k);
      out.push_back(p->compute(comm));
      for (int i = 0; i < ncoeff; ++i) out.push_back(p->coeff(i));
      delete p;
    }
    if (!prefix.empty()) dump(prefix + ".powell.bin", out);
  }

  ErrorVec evec;
  double obj = pot->compute(comm, &evec);
  std::fprintf(stderr, "objective %.17g ncoeff %d esize %zu natoms %d ncells %d\n", obj, ncoeff,
               evec.size(), mmz->config->total_natoms, mmz->config->ncells);

  if (!prefix.empty()) {
    dump(prefix + ".obj.bin", std::vector<double>{obj});
    dump(prefix + ".errvec.bin", evec);
    std::vector<double> en, st, fo, co(ncoeff);
    for (Cell *c : mmz->config->cells) {
      en.push_back(c->energy);
      st.push_back(c->stress.xx); st.push_back(c->stress.yy); st.push_back(c->stress.zz);
      st.push_back(c->stress.xy); st.push_back(c->stress.yz); st.push_back(c->stress.zx);
      for (Atom *a : c->atoms) { fo.push_back(a->force.x); fo.push_back(a->force.y); fo.push_back(a->force.z); }
    }
    for (int i = 0; i < ncoeff; ++i) co[i] = pot->coeff(i);
    dump(prefix + ".energy.bin", en);
    dump(prefix + ".stress.bin", st);
    dump(prefix + ".force.bin", fo);
    dump(prefix + ".coeff.bin", co);
    PotEAM *eam = dynamic_cast<PotEAM *>(pot);
    if (eam) {
      std::vector<double> dens;
      eam->compute_densities(comm, &dens);
      dump(prefix + ".dens.bin", dens);
    }
  }

  if (fd_h > 0.0) {
    std::vector<double> g(ncoeff);
    for (int i = 0; i < ncoeff; ++i) {
      double keep = pot->coeff(i);
      pot->coeff(i) = keep + fd_h;
      double fp = pot->compute(comm);
      pot->coeff(i) = keep - fd_h;
      double fm = pot->compute(comm);
      pot->coeff(i) = keep;
      g[i] = (fp - fm) / (2.0 * fd_h);
    }
    if (!prefix.empty()) dump(prefix + ".fdgrad.bin", g);
  }

  if (reps > 0) {
    pot->compute(comm);
    auto t0 = std::chrono::steady_clock::now();
    for (int r = 0; r < reps; ++r) pot->compute(comm);
    auto t1 = std::chrono::steady_clock::now();
    double s = std::chrono::duration<double>(t1 - t0).count() / reps;
    std::printf("seconds_per_eval %.9g\n", s);
    std::fflush(stdout);
  }

  delete mmz;
  MPI_Finalize();
  return 0;
}
