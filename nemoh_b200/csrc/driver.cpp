// nemoh_solver_b200: drop-in for the reference Solver executable
// (Solver/NEMOH.f90:30-176). Reads the case named by ID.dat exactly as the
// reference does -- ID.dat (Common/Identification.f90:30-37), mesh/L10.dat and
// mesh/L12.dat (Common/Mesh.f90:81-132), Normalvelocities.dat
// (Solver/Core/Bodyconditions.f90:65-89), Nemoh.cal lines 2-5 and input.txt
// (Solver/Core/INITIALIZATION.f90:44-53), mesh/Integration.dat, mesh/Kochin.dat,
// mesh/Freesurface.dat (NEMOH.f90:88-118) -- solves every problem on the GPU
// through the C-ABI and writes results/Forces.dat in the reference's layout
// (NEMOH.f90:152-166).
//
// Problems are solved a frequency at a time: consecutive problems that share
// a frequency go to one nemoh_b200_solve_frequencies call (one assembly and
// one factorization for all of them, as the reference's w_previous cache).
// Problems whose Kochin or free-surface switch is set are also solved through
// nemoh_b200_solve_problem for their source strengths; their Kochin functions
// go to results/Kochin.<I5>.dat (SOLVE_BEM.f90:98-102, OUTPUT.f90:25-40) and
// their free-surface elevations at the points of mesh/Freesurface.dat to
// results/freesurface.<I5>.dat (SOLVE_BEM.f90:104-109, OUTPUT.f90:42-64).
// Pressure outputs (Switch_Potential) are not produced.
//
// usage: nemoh_solver_b200 [case-root] [--mixed] [--device N]
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "case_io.h"
#include "nemoh_b200.h"

namespace {

using nb200io::IoError;
using nb200io::Records;

void check(nemoh_ctx* ctx, int st, const char* what) {
  if (st) {
    std::fprintf(stderr, "nemoh_solver_b200: %s failed (status %d): %s\n", what, st,
                 ctx ? nemoh_b200_last_error(ctx) : "");
    std::exit(st);
  }
}

}  // namespace

int main(int argc, char** argv) {
  std::string root;
  int mode = NEMOH_B200_FP64, device = 0;
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--mixed")) mode = NEMOH_B200_MIXED;
    else if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
    else root = argv[a];
  }
  const std::string pre = root.empty() ? "" : root + "/";
  try {
    Records idr(pre + "ID.dat");
    const int lid = idr.integer();
    const std::string dir = pre + idr.read(1)[0].substr(0, lid);
    Records l10(dir + "/mesh/L10.dat");
    l10.skip();
    const auto h = l10.read(4);
    const int np = std::stoi(h[1]), nfa = std::stoi(h[2]);
    Records l12(dir + "/mesh/L12.dat");
    const auto h2 = l12.read(2);
    if (std::stoi(h2[0]) != 2) throw IoError("The mesh file format is not correct.");
    const int isym = std::stoi(h2[1]) == 1 ? 1 : 0;
    std::vector<double> xyz(3 * (size_t)np);
    for (int i = 0; i < np; ++i) {
      const auto v = l12.read(4);
      for (int k = 0; k < 3; ++k) xyz[3 * i + k] = std::stod(v[1 + k]);
    }
    l12.skip();
    std::vector<int> m(4 * (size_t)nfa);
    for (int i = 0; i < nfa; ++i) {
      const auto v = l12.read(4);
      for (int k = 0; k < 4; ++k) m[4 * i + k] = std::stoi(v[k]);
    }
    const int nc = nfa * (isym ? 2 : 1);
    Records bc(dir + "/Normalvelocities.dat");
    const int npb = bc.integer();
    std::vector<double> omega(npb), stype(npb);
    auto vo = bc.read(npb);
    for (int j = 0; j < npb; ++j) omega[j] = std::stod(vo[j]);
    auto vt = bc.read(npb);
    for (int j = 0; j < npb; ++j) stype[j] = std::stod(vt[j]);
    bool extra_outputs = false;
    for (const auto& t : bc.read(npb)) extra_outputs |= std::stoi(t) != 0;   // Switch_Potential
    std::vector<int> fs_switch(npb);
    {
      const auto v = bc.read(npb);
      for (int j = 0; j < npb; ++j) fs_switch[j] = std::stoi(v[j]);
    }
    std::vector<int> kochin_switch(npb);
    {
      const auto v = bc.read(npb);
      for (int j = 0; j < npb; ++j) kochin_switch[j] = std::stoi(v[j]);
    }
    std::vector<std::complex<double>> nvel((size_t)nc * npb);
    for (int c = 0; c < nc; ++c) {
      const auto v = bc.read(2 * (size_t)npb);
      for (int j = 0; j < npb; ++j) nvel[c + (size_t)nc * j] = {std::stod(v[2 * j]), std::stod(v[2 * j + 1])};
    }
    Records cal(dir + "/Nemoh.cal");
    cal.skip();
    const double rho = cal.real(), g = cal.real(), depth = cal.real();
    const auto xy = cal.read(2);
    const double xeff = std::stod(xy[0]), yeff = std::stod(xy[1]);
    {
      Records inp(dir + "/input.txt");
      inp.skip();
    }
    Records ig(dir + "/mesh/Integration.dat");
    const int nint = ig.integer();
    std::vector<double> nds((size_t)nint * nc);   // column-major nint x nc
    for (int i = 0; i < nint; ++i) {
      const auto v = ig.read(nc);
      for (int c = 0; c < nc; ++c) nds[i + (size_t)nint * c] = std::stod(v[c]);
    }
    std::vector<double> theta;
    {
      Records kr(dir + "/mesh/Kochin.dat");
      const int nth = kr.integer();
      for (int j = 0; j < nth; ++j) theta.push_back(kr.real());
    }
    std::vector<double> fs_xy;   // 2 x npts
    std::vector<int> fs_quads;   // 4 x nquads
    {
      Records fr(dir + "/mesh/Freesurface.dat");
      const auto v = fr.read(2);
      const int npts = std::stoi(v[0]), nquads = std::stoi(v[1]);
      for (int q = 0; q < npts; ++q)
        for (const auto& t : fr.read(2)) fs_xy.push_back(std::stod(t));
      for (int q = 0; q < nquads; ++q)
        for (const auto& t : fr.read(4)) fs_quads.push_back(std::stoi(t));
    }
    const int fs_npts = (int)fs_xy.size() / 2;
    if (extra_outputs) std::fprintf(stderr, "nemoh_solver_b200: pressure outputs are not produced\n");

    nemoh_ctx* ctx = nullptr;
    check(nullptr, nemoh_b200_create(&ctx, device, mode), "create");
    check(ctx, nemoh_b200_set_mesh(ctx, np, nfa, isym, xyz.data(), m.data(), rho, g, depth), "set_mesh");

    std::vector<std::complex<double>> force((size_t)nint * npb);
    int j = 0;
    while (j < npb) {
      int e = j;
      while (e < npb && omega[e] == omega[j] && e - j < 16) ++e;
      const int nrhs = e - j;
      std::vector<std::complex<double>> f((size_t)nint * nrhs);
      check(ctx,
            nemoh_b200_solve_frequencies(ctx, 1, &omega[j], nrhs, reinterpret_cast<const double*>(&nvel[(size_t)nc * j]),
                                         nint, nds.data(), reinterpret_cast<double*>(f.data())),
            "solve_frequencies");
      for (int p = 0; p < nrhs; ++p)
        for (int i = 0; i < nint; ++i) force[i + (size_t)nint * (j + p)] = f[i + (size_t)nint * p];
      j = e;
    }
    // Kochin functions and free-surface elevations of the problems that ask for them
    {
      std::vector<std::complex<double>> zigb(nfa), zigs(nfa), h(theta.size()), eta(fs_npts);
      const double PI = 4. * std::atan(1.);
      for (int p = 0; p < npb; ++p) {
        const bool want_fs = fs_switch[p] == 1 && fs_npts > 0, want_k = kochin_switch[p] == 1 && !theta.empty();
        if (!want_fs && !want_k) continue;
        const double period = 2. * PI / omega[p];
        int nexp = 0;
        check(ctx,
              nemoh_b200_solve_problem(ctx, period, reinterpret_cast<const double*>(&nvel[(size_t)nc * p]),
                                       reinterpret_cast<double*>(zigb.data()), reinterpret_cast<double*>(zigs.data()),
                                       nullptr, nullptr, &nexp),
              "solve_problem");
        char name[40];
        if (want_fs) {
          check(ctx,
                nemoh_b200_free_surface(ctx, period, fs_npts, fs_xy.data(), 1,
                                        reinterpret_cast<const double*>(zigb.data()),
                                        reinterpret_cast<const double*>(zigs.data()),
                                        reinterpret_cast<double*>(eta.data())),
                "free_surface");
          std::snprintf(name, sizeof name, "freesurface.%5d.dat", p + 1);
          std::ofstream ff(dir + "/results/" + name);
          if (!ff) throw IoError("cannot write " + dir + "/results/" + name);
          ff << " VARIABLES=\"X\" \"Y\" \"abs(eta) (m)\" \"angle(phi) (rad)\" \"PRE1\" \"PRE2\"\n";
          char line[160];
          std::snprintf(line, sizeof line, "ZONE N=%7d ,E = %7d ,F=FEPOINT,ET=QUADRILATERAL\n", fs_npts,
                        (int)fs_quads.size() / 4);
          ff << line;
          for (int q = 0; q < fs_npts; ++q) {
            const std::complex<double> e = eta[q];
            std::snprintf(line, sizeof line, " %.17E %.17E %.17E %.17E %.17E %.17E\n", fs_xy[2 * q], fs_xy[2 * q + 1],
                          std::abs(e), std::atan2(e.imag(), e.real()), e.real(), e.imag());
            ff << line;
          }
          for (size_t q = 0; q < fs_quads.size(); q += 4) {
            std::snprintf(line, sizeof line, " %d %d %d %d\n", fs_quads[q], fs_quads[q + 1], fs_quads[q + 2],
                          fs_quads[q + 3]);
            ff << line;
          }
        }
        if (want_k) {
          check(ctx,
                nemoh_b200_kochin(ctx, period, xeff, yeff, (int)theta.size(), theta.data(), 1,
                                  reinterpret_cast<const double*>(zigb.data()),
                                  reinterpret_cast<const double*>(zigs.data()), reinterpret_cast<double*>(h.data())),
                "kochin");
          std::snprintf(name, sizeof name, "Kochin.%5d.dat", p + 1);
          std::ofstream kf(dir + "/results/" + name);
          if (!kf) throw IoError("cannot write " + dir + "/results/" + name);
          char line[96];
          for (size_t t = 0; t < theta.size(); ++t) {
            std::snprintf(line, sizeof line, " %.17E %.17E %.17E\n", theta[t], std::abs(h[t]),
                          std::atan2(h[t].imag(), h[t].real()));
            kf << line;
          }
        }
      }
    }
    nemoh_b200_destroy(ctx);

    std::ofstream out(dir + "/results/Forces.dat");
    if (!out) throw IoError("cannot write " + dir + "/results/Forces.dat");
    char buf[80];
    for (int c = 0; c < nint; ++c) {
      for (int q = 0; q < npb; ++q) {
        const std::complex<double> F = force[c + (size_t)nint * q];
        double a, b;
        if (stype[q] != -1.) {
          a = std::abs(F);
          b = std::atan2(F.imag(), F.real());
        } else {
          a = F.imag() / omega[q];
          b = -F.real();
        }
        std::snprintf(buf, sizeof buf, " %.17E %.17E", a, b);
        out << buf;
      }
      out << "\n";
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "nemoh_solver_b200: %s\n", e.what());
    return NEMOH_B200_EIO;
  }
  return 0;
}
