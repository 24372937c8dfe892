// nemoh_postproc_b200: drop-in for the reference postProcessor executable
// (postProcessor/Main.f90:26-101). Reads the case named by ID.dat --
// results/index.dat, results/Forces.dat and results/FKForce.tec
// (ReadTResults, Common/Results.f90:104-165) and the IRF line of Nemoh.cal
// (Initialize_IRF, postProcessor/IRF.f90:72-98) -- and writes
// RadiationCoefficients.tec, DiffractionForce.tec, ExcitationForce.tec, CA.dat,
// CM.dat, Fe.dat (SaveTResults, Results.f90:167-251) and, when the IRF switch is
// set, IRF.tec (Save_IRF, IRF.f90:129-145) with the impulse response functions
// and the infinite-frequency added mass computed on the GPU (nemoh_b200_irf).
// Compute_RAOs only zeroes its array and Plot_WaveElevation never runs (its
// switch is never set, Plot_WaveElevation.f90:121-135): neither writes a file.
// Reals are written with 17 significant digits in place of E14.7 / E13.6.
//
// usage: nemoh_postproc_b200 [case-root] [--device N]
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "case_io.h"
#include "nemoh_b200.h"

namespace {

using nb200io::IoError;
using nb200io::Records;
using cplx = std::complex<double>;

class Text {
 public:
  explicit Text(const std::string& path) : f_(path) {
    if (!f_) throw IoError("cannot write " + path);
  }
  Text& operator()(const char* fmt, ...) __attribute__((format(printf, 2, 3))) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    f_ << buf;
    return *this;
  }

 private:
  std::ofstream f_;
};

// TResults (Common/Results.f90:23-38); arrays with w fastest
struct Results {
  int nw = 0, nbeta = 0, nrad = 0, nint = 0, ntheta = 0;
  std::vector<double> w, beta;
  std::vector<int> fbody, fmode, rbody, rmode;
  std::vector<cplx> diffraction, froude_krylov;   // (nw, nbeta, nint)
  std::vector<double> added_mass, damping;        // (nw, nrad, nint)
  size_t b(int i, int j, int k) const { return i + (size_t)nw * (j + (size_t)nbeta * k); }
  size_t r(int i, int j, int k) const { return i + (size_t)nw * (j + (size_t)nrad * k); }
};

Results read_results(const std::string& dir) {
  Results R;
  Records ix(dir + "/results/index.dat");
  const auto h = ix.read(5);
  R.nw = std::stoi(h[0]);
  R.nbeta = std::stoi(h[1]);
  R.nrad = std::stoi(h[2]);
  R.nint = std::stoi(h[3]);
  R.ntheta = std::stoi(h[4]);
  ix.skip();
  for (int k = 0; k < R.nint; ++k) {
    const auto v = ix.read(3);
    R.fbody.push_back(std::stoi(v[1]));
    R.fmode.push_back(std::stoi(v[2]));
  }
  ix.skip();
  for (int k = 0; k < R.nrad; ++k) {
    const auto v = ix.read(3);
    R.rbody.push_back(std::stoi(v[1]));
    R.rmode.push_back(std::stoi(v[2]));
  }
  for (const auto& t : ix.read(R.nbeta)) R.beta.push_back(std::stod(t));
  for (const auto& t : ix.read(R.nw)) R.w.push_back(std::stod(t));
  R.diffraction.assign((size_t)R.nw * R.nbeta * R.nint, 0.);
  R.froude_krylov = R.diffraction;
  R.added_mass.assign((size_t)R.nw * R.nrad * R.nint, 0.);
  R.damping = R.added_mass;
  const cplx II(0., 1.);
  Records fr(dir + "/results/Forces.dat");
  for (int k = 0; k < R.nint; ++k) {
    const auto v = fr.read(2 * (size_t)R.nw * (R.nbeta + R.nrad));
    size_t c = 0;
    for (int i = 0; i < R.nw; ++i) {
      for (int j = 0; j < R.nbeta; ++j, c += 2)
        R.diffraction[R.b(i, j, k)] = std::stod(v[c]) * std::exp(II * std::stod(v[c + 1]));
      for (int j = 0; j < R.nrad; ++j, c += 2) {
        R.added_mass[R.r(i, j, k)] = std::stod(v[c]);
        R.damping[R.r(i, j, k)] = std::stod(v[c + 1]);
      }
    }
  }
  Records fk(dir + "/results/FKForce.tec");
  for (int k = 0; k <= R.nint; ++k) fk.skip();
  for (int j = 0; j < R.nbeta; ++j) {
    fk.skip();
    for (int i = 0; i < R.nw; ++i) {
      const auto v = fk.read(1 + 2 * (size_t)R.nint);
      for (int k = 0; k < R.nint; ++k)
        R.froude_krylov[R.b(i, j, k)] = std::stod(v[1 + 2 * k]) * std::exp(II * std::stod(v[2 + 2 * k]));
    }
  }
  return R;
}

void save_results(const Results& R, const std::string& rd) {
  const double PI = 4. * std::atan(1.0);
  {
    Text t(rd + "RadiationCoefficients.tec");
    t("VARIABLES=\"w (rad/s)\"\n");
    for (int k = 0; k < R.nint; ++k) t("\"A%4d%4d\" \"B%4d%4d\"\n", R.fbody[k], R.fmode[k], R.fbody[k], R.fmode[k]);
    for (int j = 0; j < R.nrad; ++j) {
      t("Zone t=\"Motion of body %4d in DoF%4d\",I=%6d,F=POINT\n", R.rbody[j], R.rmode[j], R.nw);
      for (int i = 0; i < R.nw; ++i) {
        t(" %.17E", R.w[i]);
        for (int k = 0; k < R.nint; ++k) t(" %.17E %.17E", R.added_mass[R.r(i, j, k)], R.damping[R.r(i, j, k)]);
        t("\n");
      }
    }
  }
  for (int excitation = 0; excitation < 2; ++excitation) {
    Text t(rd + (excitation ? "ExcitationForce.tec" : "DiffractionForce.tec"));
    t("VARIABLES=\"w (rad/s)\"\n");
    for (int k = 0; k < R.nint; ++k)
      t("\"abs(F%4d%4d)\" \"angle(F%4d%4d)\"\n", R.fbody[k], R.fmode[k], R.fbody[k], R.fmode[k]);
    for (int j = 0; j < R.nbeta; ++j) {
      t("Zone t=\"Diffraction force - beta = %7.3f deg\",I=%6d,F=POINT\n", R.beta[j] * 180. / PI, R.nw);
      for (int i = 0; i < R.nw; ++i) {
        t(" %.17E", R.w[i]);
        for (int k = 0; k < R.nint; ++k) {
          const cplx F = excitation ? R.diffraction[R.b(i, j, k)] + R.froude_krylov[R.b(i, j, k)]
                                    : R.diffraction[R.b(i, j, k)];
          t(" %.17E %.17E", std::abs(F), std::atan2(F.imag(), F.real()));
        }
        t("\n");
      }
    }
  }
  for (int mass = 0; mass < 2; ++mass) {   // CA.dat: damping, CM.dat: added mass (Aquaplus layout)
    Text t(rd + (mass ? "CM.dat" : "CA.dat"));
    t("Nb de periode : %5d\n", R.nw);
    const std::vector<double>& X = mass ? R.added_mass : R.damping;
    for (int l = 0; l < R.nw; ++l) {
      t(" %.17E\n", R.w[l]);
      for (int j = 0; j < R.nrad; ++j)
        for (int k = 0; k < R.nrad; ++k)   // six values per record
          t(" %.17E%s", X[R.r(l, j, k)], (k % 6 == 5 || k == R.nrad - 1) ? "\n" : "");
    }
  }
  {
    Text t(rd + "Fe.dat");
    t("VARIABLES=\"Period (s)\" \"|Fx| (N/m)\" \"|Fy| (N/m)\" \"|Fz| (N/m)\" \"|Cx| (N)\" \"|Cy| (N)\" \"|Cz| (N)\" "
      "\"ang(Fx) (\xb0)\" \"ang(Fy) (\xb0)\" \"ang(Fz) (\xb0)\" \"ang(Cx) (\xb0)\" \"ang(Cy) (\xb0)\" \"ang(Cz) (\xb0)\"\n");
    t("Zone t=\"Corps %2d\"\n", 1);
    for (int j = 0; j < R.nbeta; ++j) {
      t("Zone t=\"Diffraction force - beta = %7.3f deg\",I=%6d,F=POINT\n", R.beta[j] * 180. / PI, R.nw);
      for (int l = 0; l < R.nw; ++l) {
        t(" %.17E", R.w[l]);
        for (int k = 0; k < R.nint; ++k) t(" %.17E", std::abs(R.diffraction[R.b(l, j, k)] + R.froude_krylov[R.b(l, j, k)]));
        for (int k = 0; k < R.nint; ++k) {
          const cplx F = R.diffraction[R.b(l, j, k)] + R.froude_krylov[R.b(l, j, k)];
          t(" %.17E", 180. / PI * std::atan2(F.imag(), F.real()));
        }
        t("\n");
      }
    }
  }
}

void check(nemoh_ctx* ctx, int st, const char* what) {
  if (st) {
    std::fprintf(stderr, "nemoh_postproc_b200: %s failed (status %d): %s\n", what, st,
                 ctx ? nemoh_b200_last_error(ctx) : "");
    std::exit(st);
  }
}

}  // namespace

int main(int argc, char** argv) {
  std::string root;
  int device = 0;
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
    else root = argv[a];
  }
  try {
    const std::string dir = nb200io::case_dir(root);
    const Results R = read_results(dir);
    const std::string rd = dir + "/results/";
    save_results(R, rd);
    // Initialize_IRF: the record after the "--- Post processing " line
    Records cal(dir + "/Nemoh.cal");
    std::string s;
    bool found = false;
    while (!found && cal.next_line(s)) found = s.compare(0, 20, "--- Post processing ") == 0;
    if (!found) throw IoError("Nemoh.cal: no post-processing section");
    const auto irf = cal.read(3);
    if (std::stoi(irf[0]) == 1) {
      const double dt = std::stod(irf[1]), tf = std::stod(irf[2]);
      const int ntime = (int)(tf / dt);
      const int npair = R.nrad * R.nint;
      std::vector<double> K((size_t)ntime * npair), ainf(npair);
      nemoh_ctx* ctx = nullptr;
      check(nullptr, nemoh_b200_create(&ctx, device, NEMOH_B200_FP64), "create");
      check(ctx,
            nemoh_b200_irf(ctx, R.nw, R.w.data(), R.nrad, R.nint, R.damping.data(), R.added_mass.data(), ntime, dt,
                           K.data(), ainf.data()),
            "irf");
      nemoh_b200_destroy(ctx);
      Text t(rd + "IRF.tec");
      t(" VARIABLES=\"Time (s)\"\n");
      for (int k = 0; k < R.nint; ++k) t("\"AddedMass %4d\" \"IRF %4d\"\n", k + 1, k + 1);
      for (int j = 0; j < R.nrad; ++j) {
        t("Zone t=\"DoF %4d\",I=%6d,F=POINT\n", j + 1, ntime);
        for (int i = 0; i < ntime; ++i) {
          t(" %.17E", i * dt);
          for (int k = 0; k < R.nint; ++k)
            t(" %.17E %.17E", ainf[j + (size_t)R.nrad * k], K[i + (size_t)ntime * (j + (size_t)R.nrad * k)]);
          t("\n");
        }
      }
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "nemoh_postproc_b200: %s\n", e.what());
    return NEMOH_B200_EIO;
  }
  return 0;
}
