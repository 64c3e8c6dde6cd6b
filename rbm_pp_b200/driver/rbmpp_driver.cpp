// rbmpp_driver.cpp -- the C++ host program that mirrors main.f90 on top of the C ABI (include/rbmpp.h).
//
// It reads the reference's input files from the working directory (or --dir):
//   RBM.input                 main.f90:75-84
//   sym_info.txt              main.f90:89-124 (permutation checks :110-119)
//   orbitalidx.def            parameter.f90:81-101, main.f90:126-129
//   zqp_orbital_initial.dat   parameter.f90:114-141 (rescaled to mean |f| = 0.25)
//   W.input (optional)        parameter.f90:42-75
// and runs the optimisation loop of main.f90:300-455 through rbmpp_iteration, averaging the parameters
// of the last Nav iterations (:410-422, :455-485), writes optimized_W.txt and zqp_orbital_opt.dat
// (write_optimized_parameters, parameter.f90:238-277), then measures the final energy (:486-575) into
// energy_after_opt.txt and Average_Energy.txt.  Energy_vs_Iteration.txt follows main.f90:310,406.
//
// MPI ranks are the library's walkers: --walkers W emulates Nmpi = W ranks on one GPU, each with
// Nsample/Nmpi stored samples and the seeding rule of main.f90:224-235.
//
// With --correlation the final measurement follows the Calc_Correlation program instead
// (Calc_Correlation/main.f90:498-600): shift = 0 for a first make_sample, shift = 1e-5 times the mean |psi|
// of its samples, 7 more make_samples, then Nav rounds of make_sample + rbmpp_measure_correlation, each
// writing Chi_sp / norm to fort.<60000+it> and Chi_vbs / norm to fort.<70000+it> in the reference's formats.
//
// With --transverse it runs the transverse code instead (transverse_code/main.f90): spin projection at
// beta = -pi/2, pi/2 with sqrt(2)-scaled weights (transverse_code/spin_projection.f90:30-38) and the shift
// schedule of transverse_code/main.f90:451; the library then carries the full skew Pfaffian matrix.
//
// Usage: rbmpp_driver [--dir D] [--walkers W] [--seed S] [--precision fp64|split] [--device G]
//                     [--nstep N] [--correlation | --transverse] [--check-inputs]
// --check-inputs parses and validates the inputs, prints a summary and exits without touching a GPU.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rbmpp.h"

namespace {

[[noreturn]] void die(const std::string& m) {
  std::fprintf(stderr, "rbmpp_driver: %s\n", m.c_str());
  std::exit(1);
}

std::vector<std::string> read_lines(const std::string& path) {
  std::ifstream f(path);
  if (!f) die("cannot open " + path);
  std::vector<std::string> out;
  std::string ln;
  while (std::getline(f, ln)) out.push_back(ln);
  return out;
}

// list-directed tokens: blanks, commas and the parentheses of complex literals separate values;
// Fortran exponents (1.0d-3) are accepted
std::vector<std::string> toks(std::string s) {
  for (char& ch : s)
    if (ch == ',' || ch == '(' || ch == ')') ch = ' ';
  std::istringstream is(s);
  std::vector<std::string> t;
  std::string w;
  while (is >> w) t.push_back(w);
  return t;
}

double fnum(std::string s) {
  for (char& ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';
  return std::strtod(s.c_str(), nullptr);
}

const std::vector<std::string>& line_at(const std::vector<std::string>& L, size_t i, const std::string& file) {
  if (i >= L.size()) die(file + ": unexpected end of file");
  return L;
}

struct Inputs {
  int L = 0, Nsample = 0, spin_parity = 1, alphac = 0, alphar = 0, Nstep = 0, Nav = 0;
  double delta_tau = 0, s_factor0 = 0, s_factor_scale = 1, s_cut = 0, J1 = 1, J2 = 0;
  int N = 0, n_mp = 0, n_slater = 0;
  std::vector<double> para;      // (re, im) per projection
  std::vector<int> W_map;        // (N, n_mp) column-major, 1-based
  std::vector<int> orbital_idx;  // (N, N) column-major, 1-based
  std::vector<double> slater;    // N_Slater
  bool have_W = false;
  std::vector<double> Wr, br;    // (N, alphar) column-major, alphar
  std::vector<double> Wc, bc;    // complex units as (re, im) pairs: (N, alphac) column-major, alphac
};

std::vector<std::string> tk(const std::vector<std::string>& L, size_t i, const std::string& file) {
  line_at(L, i, file);
  return toks(L[i]);
}

void read_rbm_input(const std::string& dir, Inputs& in) {  // main.f90:75-84
  const std::string fn = dir + "/RBM.input";
  auto L = read_lines(fn);
  auto a = tk(L, 1, fn), b = tk(L, 3, fn), c = tk(L, 5, fn), d = tk(L, 7, fn);
  if (a.size() < 3 || b.size() < 5 || c.size() < 3 || d.size() < 2) die(fn + ": malformed");
  in.L = std::atoi(a[0].c_str());
  in.Nsample = std::atoi(a[1].c_str());
  in.spin_parity = std::atoi(a[2].c_str());
  in.alphac = std::atoi(b[0].c_str());
  in.alphar = std::atoi(b[1].c_str());
  in.Nstep = std::atoi(b[2].c_str());
  in.Nav = std::atoi(b[3].c_str());
  in.delta_tau = fnum(b[4]);
  in.s_factor0 = fnum(c[0]);
  in.s_factor_scale = fnum(c[1]);
  in.s_cut = fnum(c[2]);
  in.J1 = fnum(d[0]);
  in.J2 = fnum(d[1]);
  in.N = in.L * in.L;
}

void read_sym_info(const std::string& dir, Inputs& in) {  // main.f90:89-124
  const std::string fn = dir + "/sym_info.txt";
  auto L = read_lines(fn);
  auto t = tk(L, 1, fn);
  in.n_mp = std::atoi(t[0].c_str());
  if (t.size() < 2 || std::atoi(t[1].c_str()) != 1) die("i1/=Ncopy (sym_info.txt)");
  in.para.assign(2 * (size_t)in.n_mp, 0.0);
  size_t pos = 3;
  for (int mp = 0; mp < in.n_mp; mp++) {
    auto u = tk(L, pos++, fn);
    if (u.size() < 2 || std::atoi(u[0].c_str()) != mp + 1) die("i1/=mpidx (sym_info.txt)");
    in.para[2 * mp] = fnum(u[1]);
    in.para[2 * mp + 1] = u.size() > 2 ? fnum(u[2]) : 0.0;
  }
  pos++;
  const int N = in.N;
  in.W_map.assign((size_t)N * in.n_mp, 0);
  for (int mp = 0; mp < in.n_mp; mp++) {
    std::vector<char> seen(N, 0);
    for (int i = 0; i < N; i++) {
      auto u = tk(L, pos++, fn);
      if (u.size() < 4 || std::atoi(u[0].c_str()) != mp + 1 || std::atoi(u[1].c_str()) != 1 ||
          std::atoi(u[2].c_str()) != i + 1)
        die("index mismatch (sym_info.txt)");
      const int w = std::atoi(u[3].c_str());
      if (w < 1 || w > N) die("W_map wrong 1 (sym_info.txt)");
      if (seen[w - 1]) die("W_map wrong 2 (sym_info.txt)");
      seen[w - 1] = 1;
      in.W_map[i + (size_t)N * mp] = w;
    }
  }
}

void read_orbital_idx(const std::string& dir, Inputs& in) {  // parameter.f90:81-101
  const std::string fn = dir + "/orbitalidx.def";
  auto L = read_lines(fn);
  auto t = tk(L, 1, fn);
  if (t.size() < 2) die(fn + ": malformed");
  in.n_slater = std::atoi(t[1].c_str());
  const int N = in.N;
  in.orbital_idx.assign((size_t)N * N, 0);
  size_t pos = 5;
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      auto u = tk(L, pos++, fn);
      if (u.size() < 3 || std::atoi(u[0].c_str()) != i || std::atoi(u[1].c_str()) != j) die("error2/3, orbitalidx");
      const int v = std::atoi(u[2].c_str()) + 1;
      if (v < 1 || v > in.n_slater) die("error4, orbitalidx");
      in.orbital_idx[i + (size_t)N * j] = v;
    }
}

void read_zqp(const std::string& dir, Inputs& in) {  // parameter.f90:114-141
  const std::string fn = dir + "/zqp_orbital_initial.dat";
  auto L = read_lines(fn);
  auto t = tk(L, 1, fn);
  if (t.size() < 2 || std::atoi(t[1].c_str()) != in.n_slater) die("error in zqp_orbital_initial 1");
  in.slater.assign(in.n_slater, 0.0);
  double r3 = 0.0;
  for (int k = 0; k < in.n_slater; k++) {
    auto u = tk(L, 5 + (size_t)k, fn);
    if (u.size() < 2 || std::atoi(u[0].c_str()) != k) die("error in zqp_orbital_initial 2");
    in.slater[k] = fnum(u[1]);
    r3 += std::fabs(in.slater[k]);
    if (u.size() > 2 && std::fabs(fnum(u[2])) > 1e-10) die("imaginary zqp_orbital_initial, not implemented");
  }
  r3 /= (double)in.n_slater;
  for (double& v : in.slater) v = v * 0.25 / r3;  // slater_abs_av, module.f90:66
}

void read_W(const std::string& dir, Inputs& in) {  // parameter.f90:42-75: complex units, then real ones
  const std::string fn = dir + "/W.input";
  std::ifstream probe(fn);
  if (!probe) return;
  auto L = read_lines(fn);
  const int N = in.N;
  in.Wr.assign((size_t)N * in.alphar, 0.0);
  in.br.assign(in.alphar, 0.0);
  in.Wc.assign((size_t)2 * N * in.alphac, 0.0);
  in.bc.assign((size_t)2 * in.alphac, 0.0);
  size_t pos = 1;
  for (int f = 0; f < in.alphac; f++) {
    auto u = tk(L, pos++, fn);  // "# bias f re im"
    if (u.size() < 5 || std::atoi(u[2].c_str()) != f + 1) die("i1/=f (W.input)");
    in.bc[2 * f] = fnum(u[3]);
    in.bc[2 * f + 1] = fnum(u[4]);
    for (int iw = 0; iw < N; iw++) {
      auto v = tk(L, pos++, fn);
      if (v.size() < 4 || std::atoi(v[0].c_str()) != f + 1 || std::atoi(v[1].c_str()) != iw + 1)
        die("index mismatch (W.input)");
      in.Wc[2 * (iw + (size_t)N * f)] = fnum(v[2]);
      in.Wc[2 * (iw + (size_t)N * f) + 1] = fnum(v[3]);
    }
    pos++;
  }
  for (int f = 0; f < in.alphar; f++) {
    auto u = tk(L, pos++, fn);  // "# bias f b 0"
    if (u.size() < 5 || std::atoi(u[2].c_str()) != f + 1) die("i1/=f (W.input)");
    in.br[f] = fnum(u[3]);
    if (std::fabs(fnum(u[4])) > 1e-15) die("r2 /= 0 (W.input)");
    for (int iw = 0; iw < N; iw++) {
      auto v = tk(L, pos++, fn);
      if (v.size() < 4 || std::atoi(v[0].c_str()) != f + 1 || std::atoi(v[1].c_str()) != iw + 1)
        die("index mismatch (W.input)");
      in.Wr[iw + (size_t)N * f] = fnum(v[2]);
      if (std::fabs(fnum(v[3])) > 1e-15) die("r2 /= 0 (W.input)");
    }
    pos++;
  }
  in.have_W = true;
}

void write_W(const std::string& path, int N, int alphar, const std::vector<double>& br, const std::vector<double>& Wr,
             int alphac = 0, const std::vector<double>& bc = {}, const std::vector<double>& Wc = {}) {
  FILE* f = std::fopen(path.c_str(), "w");  // parameter.f90:159-175, 248-262
  if (!f) die("cannot write " + path);
  std::fprintf(f, "# index for independent neurons (f), index for interaction (iw), irreducible interaction Wirr(iw,f)\n");
  for (int fi = 0; fi < alphac; fi++) {
    std::fprintf(f, "# bias%6d%22.15f%22.15f\n", fi + 1, bc[2 * fi], bc[2 * fi + 1]);
    for (int iw = 0; iw < N; iw++)
      std::fprintf(f, "%6d%6d%22.15f%22.15f\n", fi + 1, iw + 1, Wc[2 * (iw + (size_t)N * fi)],
                   Wc[2 * (iw + (size_t)N * fi) + 1]);
    std::fprintf(f, "\n");
  }
  for (int fi = 0; fi < alphar; fi++) {
    std::fprintf(f, "# bias%6d%22.15f%22.15f\n", fi + 1, br[fi], 0.0);
    for (int iw = 0; iw < N; iw++) std::fprintf(f, "%6d%6d%22.15f%22.15f\n", fi + 1, iw + 1, Wr[iw + (size_t)N * fi], 0.0);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
}

// Fortran edit descriptor Ew.d: a sign, "0.", d significant digits, then E+xx (or +xxx without the E for
// exponents beyond 99), right-justified in w columns.
std::string fort_e(double v, int w, int d) {
  char m[64];
  std::snprintf(m, sizeof(m), "%.*E", d - 1, v);  // [-]D.DDDE[+-]XX with d significant digits
  std::string s(m);
  const bool neg = s[0] == '-';
  if (neg) s = s.substr(1);
  const size_t ep = s.find('E');
  std::string digits = s.substr(0, 1) + s.substr(2, ep - 2);
  int e = std::atoi(s.c_str() + ep + 1);
  if (v != 0.0) e += 1;
  char ex[16];
  if (std::abs(e) <= 99)
    std::snprintf(ex, sizeof(ex), "E%c%02d", e < 0 ? '-' : '+', std::abs(e));
  else
    std::snprintf(ex, sizeof(ex), "%c%03d", e < 0 ? '-' : '+', std::abs(e));
  std::string out = std::string(neg ? "-" : "") + "0." + digits + ex;
  if ((int)out.size() < w) out = std::string(w - out.size(), ' ') + out;
  return out;
}

void write_zqp(const std::string& path, const std::vector<double>& sl) {  // parameter.f90:266-275
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) die("cannot write " + path);
  std::fprintf(f, "\n Slater%10d\n\n\n\n", (int)sl.size());
  for (size_t k = 0; k < sl.size(); k++)
    std::fprintf(f, "%5d%s%s\n", (int)k, fort_e(sl[k], 25, 15).c_str(), fort_e(0.0, 25, 15).c_str());
  std::fclose(f);
}

// The input echoes of write_initial_parameters (parameter.f90:177-207): chk_orbitalidx.def,
// chk_qptransidx.def (MP_Trans_Idx = W_map, parameter.f90:107) and chk_zqp_orbital_opt.dat.
// The list-directed integers are written in a 12-column field.
void write_input_checks(const std::string& dir, const Inputs& in) {
  const int N = in.N;
  FILE* f = std::fopen((dir + "/chk_orbitalidx.def").c_str(), "w");
  if (!f) die("cannot write chk_orbitalidx.def");
  std::fprintf(f, "%12d\n", in.n_slater);
  for (int i1 = 0; i1 < N; i1++)
    for (int i2 = 0; i2 < N; i2++)
      std::fprintf(f, "%5d%7d%7d\n", i1, i2, in.orbital_idx[i1 + (size_t)N * i2] - 1);
  std::fclose(f);
  f = std::fopen((dir + "/chk_qptransidx.def").c_str(), "w");
  if (!f) die("cannot write chk_qptransidx.def");
  std::fprintf(f, "%12d\n", in.n_mp);
  for (int mp = 0; mp < in.n_mp; mp++) std::fprintf(f, "%3d%20.12f%20.12f\n", mp + 1, in.para[2 * mp], in.para[2 * mp + 1]);
  for (int mp = 0; mp < in.n_mp; mp++)
    for (int i = 0; i < N; i++) std::fprintf(f, "%5d%7d%7d\n", mp + 1, i + 1, in.W_map[i + (size_t)N * mp]);
  std::fclose(f);
  f = std::fopen((dir + "/chk_zqp_orbital_opt.dat").c_str(), "w");
  if (!f) die("cannot write chk_zqp_orbital_opt.dat");
  std::fprintf(f, "# N_Slater%10d\n", in.n_slater);
  for (int k = 0; k < in.n_slater; k++) std::fprintf(f, "%4d%s\n", k, fort_e(in.slater[k], 25, 15).c_str());
  std::fclose(f);
}

void av_er(const std::vector<double>& x, double& av, double& er) {  // calc_av_er, sub.f90:93-114
  av = 0.0;
  for (double v : x) av += v;
  av /= (double)x.size();
  er = 0.0;
  for (double v : x) er += (v - av) * (v - av);
  er = std::sqrt(er / (double)x.size());
}

struct Lib {
  rbmpp_ctx* c = nullptr;
  void ck(int rc, const char* what) const {
    if (rc) die(std::string(what) + ": error " + std::to_string(rc) + ": " + rbmpp_last_error(c));
  }
};

}  // namespace

int main(int argc, char** argv) {
  std::string dir = ".", prec = "fp64";
  int walkers = 1, device = 0, nstep_override = -1;
  long long seed = -1;
  bool check_only = false, correlation = false, transverse = false;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) die("missing value after " + a);
      return argv[++i];
    };
    if (a == "--dir") dir = next();
    else if (a == "--walkers") walkers = std::atoi(next().c_str());
    else if (a == "--seed") seed = std::atoll(next().c_str());
    else if (a == "--precision") prec = next();
    else if (a == "--device") device = std::atoi(next().c_str());
    else if (a == "--nstep") nstep_override = std::atoi(next().c_str());
    else if (a == "--check-inputs") check_only = true;
    else if (a == "--correlation") correlation = true;
    else if (a == "--transverse") transverse = true;
    else die("unknown argument " + a);
  }
  if (correlation && transverse) die("--correlation and --transverse: the Calc_Correlation program has no transverse form");
  Inputs in;
  read_rbm_input(dir, in);
  read_sym_info(dir, in);
  read_orbital_idx(dir, in);
  read_zqp(dir, in);
  read_W(dir, in);
  if (nstep_override >= 0) in.Nstep = nstep_override;
  if (walkers < 1 || in.Nsample % walkers) die("Nsample must be a multiple of --walkers (main.f90:138)");
  const int N = in.N, ns = in.Nsample / walkers;
  if (check_only) {
    double fabs_av = 0.0;
    for (double v : in.slater) fabs_av += std::fabs(v);
    fabs_av /= (double)in.n_slater;
    std::printf("L %d N %d Nsample %d walkers %d ns %d alphar %d Nstep %d Nav %d n_mp %d n_slater %d W.input %d "
                "mean|f| %.15f W_map(1,last) %d orbital_idx(N,N) %d\n",
                in.L, N, in.Nsample, walkers, ns, in.alphar, in.Nstep, in.Nav, in.n_mp, in.n_slater, in.have_W ? 1 : 0,
                fabs_av, in.W_map[(size_t)N * (in.n_mp - 1)], in.orbital_idx[(size_t)N * N - 1]);
    write_input_checks(dir, in);
    return 0;
  }
  const int precision = prec == "split" ? RBMPP_SR_SPLIT_BF16 : RBMPP_SR_FP64;
  if (prec != "split" && prec != "fp64") die("--precision fp64|split");
  if (seed < 0) {  // main.f90:222-225: iseed from the clock
    const long long j = std::chrono::steady_clock::now().time_since_epoch().count() / 1000;
    seed = j % 10000000 + 1;
  }
  std::printf("iseed (initial) =%12lld\n", seed);

  rbmpp_dims d;
  std::memset(&d, 0, sizeof(d));
  d.L = in.L;
  d.n_mp_trans = in.n_mp;
  d.alphac = in.alphac;
  d.alphar = in.alphar;
  d.n_slater = in.n_slater;
  d.nsample = ns;
  d.n_walkers = walkers;
  d.spin_parity = in.spin_parity;
  d.J1 = in.J1;
  d.J2 = in.J2;
  d.device = device;
  d.walker_offset = 0;
  Lib lib;
  lib.ck(rbmpp_create(&d, &lib.c), "rbmpp_create");
  // InitSPWeight: SP_GL_Cos, SP_GL_Sin, para_spin_proj per point (spin_projection.f90:25-63; transverse:
  // transverse_code/spin_projection.f90:30-38)
  std::vector<double> spw(6);
  {
    const double pi = std::acos(-1.0);
    const double beta[2] = {transverse ? -0.5 * pi : 0.0, transverse ? 0.5 * pi : pi};
    const double scale = transverse ? std::sqrt(2.0) : 1.0;
    for (int sp = 0; sp < 2; sp++) {
      spw[3 * sp] = scale * std::cos(0.5 * beta[sp]);
      spw[3 * sp + 1] = scale * std::sin(0.5 * beta[sp]);
      spw[3 * sp + 2] = (sp == 0 || in.spin_parity == 1) ? 1.0 : -1.0;
    }
  }
  lib.ck(rbmpp_set_tables(lib.c, in.W_map.data(), in.para.data(), in.orbital_idx.data(), nullptr, nullptr,
                          spw.data()),
         "set_tables");
  lib.ck(rbmpp_seed_walkers(lib.c, (int)seed), "seed_walkers");
  // initialize_parameters (parameter.f90:21-41): rank 0 draws U(-0.05, 0.05), complex units first as (re, im)
  // pairs; W.input overrides
  std::vector<double> u((size_t)2 * in.alphac * (N + 1) + (size_t)in.alphar * (N + 1));
  lib.ck(rbmpp_rank0_grnd(lib.c, (int)u.size(), u.data()), "rank0_grnd");
  std::vector<double> br(in.alphar), Wr((size_t)N * in.alphar), bc((size_t)2 * in.alphac), Wc((size_t)2 * N * in.alphac);
  size_t k = 0;
  for (int f = 0; f < in.alphac; f++) {
    bc[2 * f] = 0.1 * (u[k++] - 0.5);
    bc[2 * f + 1] = 0.1 * (u[k++] - 0.5);
    if (in.spin_parity == -1) {
      bc[2 * f] *= 10.0;
      bc[2 * f + 1] *= 10.0;
    }
    for (int iw = 0; iw < N; iw++) {
      Wc[2 * (iw + (size_t)N * f)] = 0.1 * (u[k++] - 0.5);
      Wc[2 * (iw + (size_t)N * f) + 1] = 0.1 * (u[k++] - 0.5);
    }
  }
  for (int f = 0; f < in.alphar; f++) {
    br[f] = 0.1 * (u[k++] - 0.5);
    if (in.spin_parity == -1) br[f] *= 10.0;
    for (int iw = 0; iw < N; iw++) Wr[iw + (size_t)N * f] = 0.1 * (u[k++] - 0.5);
  }
  if (in.have_W) {
    br = in.br;
    Wr = in.Wr;
    bc = in.bc;
    Wc = in.Wc;
  }
  // write_initial_parameters (parameter.f90:148-234); rank 4's sub_initial_W.txt is the same content
  write_W(dir + "/initial_W.txt", N, in.alphar, br, Wr, in.alphac, bc, Wc);
  write_W(dir + "/sub_initial_W.txt", N, in.alphar, br, Wr, in.alphac, bc, Wc);
  write_input_checks(dir, in);
  std::vector<double> sl = in.slater;
  lib.ck(rbmpp_set_params(lib.c, Wr.data(), br.data(), in.alphac ? Wc.data() : nullptr,
                          in.alphac ? bc.data() : nullptr, sl.data(), 0.0),
         "set_params");

  // optimisation loop, main.f90:300-455
  FILE* fe = std::fopen((dir + "/Energy_vs_Iteration.txt").c_str(), "w");
  if (!fe) die("cannot write Energy_vs_Iteration.txt");
  std::vector<double> br_av(in.alphar, 0.0), Wr_av(Wr.size(), 0.0), sl_av(sl.size(), 0.0);
  std::vector<double> bc_av(bc.size(), 0.0), Wc_av(Wc.size(), 0.0);
  double shift_av = 0.0;
  int nav_chk = 0;
  for (int it = 1; it <= in.Nstep; it++) {
    double shift_now = 0.0;
    lib.ck(rbmpp_get_params(lib.c, nullptr, nullptr, nullptr, &shift_now), "get_params");
    rbmpp_sr_out o;
    lib.ck(rbmpp_iteration(lib.c, precision, in.delta_tau, in.s_factor_scale, in.s_cut, in.s_factor0, &o), "iteration");
    const double var = (o.Etot2 - o.Etot * o.Etot) / (o.Etot * o.Etot);
    std::printf("Iteration :%6d\n   Total Energy         :%20.10f\n   Energy Variance      :%20.10f\n"
                "   Acceptance Ratio     :%20.10f\n   Stabilization Factor :%20.10f%20.10f\n"
                "   wf_av, shift         :%s%s\n   Maximum change in W  :%20.10f%20.10f%8d\n",
                it, o.Etot, var, o.accept_ratio, o.s_factor, in.s_cut, fort_e(o.wf_av, 20, 5).c_str(),
                fort_e(shift_now, 20, 5).c_str(),
                std::fmin(o.delW_max, 0.04), o.delW_max / 0.04, o.kmax);
    std::fprintf(fe, "%12d %25.16E %25.16E\n", it, o.Etot, var);
    if (it > in.Nstep - in.Nav) {  // :410-422
      nav_chk++;
      shift_av += shift_now;
      lib.ck(rbmpp_get_params(lib.c, Wr.data(), br.data(), sl.data(), nullptr), "get_params");
      if (in.alphac) lib.ck(rbmpp_get_params_c(lib.c, Wc.data(), bc.data()), "get_params_c");
      for (size_t q = 0; q < bc.size(); q++) bc_av[q] += bc[q];
      for (size_t q = 0; q < Wc.size(); q++) Wc_av[q] += Wc[q];
      for (size_t q = 0; q < br.size(); q++) br_av[q] += br[q];
      for (size_t q = 0; q < Wr.size(); q++) Wr_av[q] += Wr[q];
      for (size_t q = 0; q < sl.size(); q++) sl_av[q] += sl[q];
    }
  }
  std::fclose(fe);
  if (in.Nav < 1 || nav_chk != in.Nav) die("Nav_chk /= Nav");
  // averaged parameters (:455-485) and write_optimized_parameters (parameter.f90:238-277)
  for (double& v : bc_av) v /= (double)in.Nav;
  for (double& v : Wc_av) v /= (double)in.Nav;
  for (double& v : br_av) v /= (double)in.Nav;
  for (double& v : Wr_av) v /= (double)in.Nav;
  for (double& v : sl_av) v /= (double)in.Nav;
  shift_av /= (double)in.Nav;
  lib.ck(rbmpp_set_params(lib.c, Wr_av.data(), br_av.data(), in.alphac ? Wc_av.data() : nullptr,
                          in.alphac ? bc_av.data() : nullptr, sl_av.data(), shift_av),
         "set_params");
  write_W(dir + "/optimized_W.txt", N, in.alphar, br_av, Wr_av, in.alphac, bc_av, Wc_av);
  write_zqp(dir + "/zqp_orbital_opt.dat", sl_av);
  // rank 3's copies (parameter.f90:280-311)
  write_W(dir + "/sub_optimized_W.txt", N, in.alphar, br_av, Wr_av, in.alphac, bc_av, Wc_av);
  write_zqp(dir + "/sub_zqp_orbital_opt.dat", sl_av);

  // final energy (:486-575): warm up, then Nav measurements
  const size_t nchi = (size_t)N * (N + 1) / 2;
  std::vector<double> chi_sp, chi_vbs;
  double shift_meas = shift_av;  // mod_main's shift during the measurements
  if (correlation) {  // Calc_Correlation/main.f90:498-527
    chi_sp.resize(2 * nchi);
    chi_vbs.resize(4 * nchi);
    lib.ck(rbmpp_set_shift(lib.c, 0.0), "set_shift");
    lib.ck(rbmpp_make_sample(lib.c, 1, nullptr, nullptr), "make_sample");
    std::vector<double> psi((size_t)2 * (in.n_mp * 2 + 1) * ns * walkers);
    lib.ck(rbmpp_get_samples(lib.c, nullptr, psi.data(), nullptr), "get_samples");
    double wf = 0.0;
    for (long long k = 0; k < (long long)ns * walkers; k++) {
      const double* q = psi.data() + (size_t)2 * (in.n_mp * 2 + 1) * k;
      wf += std::hypot(q[0], q[1]);
    }
    wf /= (double)ns * walkers;
    shift_meas = wf * 1e-5;
    lib.ck(rbmpp_set_shift(lib.c, shift_meas), "set_shift");
    std::printf("wf_av, shift =%15.5E%15.5E\n", wf, wf * 1e-5);
    for (int it = 0; it < 7; it++) lib.ck(rbmpp_make_sample(lib.c, 0, nullptr, nullptr), "make_sample");
  } else {
    lib.ck(rbmpp_make_sample(lib.c, 1, nullptr, nullptr), "make_sample");
    for (int it = 0; it < 2; it++) lib.ck(rbmpp_make_sample(lib.c, 0, nullptr, nullptr), "make_sample");
  }
  FILE* fa = std::fopen((dir + "/energy_after_opt.txt").c_str(), "w");
  if (!fa) die("cannot write energy_after_opt.txt");
  std::vector<double> e1, e2;
  for (int it = 1; it <= in.Nav; it++) {
    long long nacc = 0;
    lib.ck(rbmpp_make_sample(lib.c, 0, nullptr, &nacc), "make_sample");
    double sc[5];
    if (correlation) {
      lib.ck(rbmpp_measure_correlation(lib.c, sc, chi_sp.data(), chi_vbs.data()), "measure_correlation");
      // Calc_Correlation/main.f90:572-581 (divided by norm) and :596-607 (unit 60000+it, 70000+it)
      FILE* f6 = std::fopen((dir + "/fort." + std::to_string(60000 + it)).c_str(), "w");
      FILE* f7 = std::fopen((dir + "/fort." + std::to_string(70000 + it)).c_str(), "w");
      if (!f6 || !f7) die("cannot write the correlation files");
      std::fprintf(f6, "# chi index,  SzSz,  SpSm\n");
      for (size_t i = 0; i < nchi; i++)
        std::fprintf(f6, "%6zu%25.15f%25.15f\n", i + 1, chi_sp[2 * i] / sc[2], chi_sp[2 * i + 1] / sc[2]);
      std::fprintf(f7, "# chi index, <SSSS> for (1,0), (0,1), (1,1), (1,-1)\n");
      for (size_t i = 0; i < nchi; i++)
        std::fprintf(f7, "%6zu%25.15f%25.15f%25.15f%25.15f\n", i + 1, chi_vbs[i] / sc[2], chi_vbs[i + nchi] / sc[2],
                     chi_vbs[i + 2 * nchi] / sc[2], chi_vbs[i + 3 * nchi] / sc[2]);
      std::fclose(f6);
      std::fclose(f7);
    } else {
      lib.ck(rbmpp_measure_energy(lib.c, sc), "measure_energy");
    }
    const double E = sc[0] / sc[2], E2 = sc[1] / sc[2];
    const double nst = (double)ns * walkers;
    const double acc = (double)nacc / nst / (double)N;
    // main.f90:548-554; Calc_Correlation/main.f90:587-594 adds wf_sgn (abs, re, im; the real path has im = 0)
    std::printf("Iteration (Energy Measuement) :%6d\n   total energy         :%20.10f\n"
                "   energy variance      :%20.10f\n   acceptance ratio     :%20.10f\n"
                "   wf_av, shift         :%s%s\n   norm                 :%20.10f\n",
                it, E, (E2 - E * E) / (E * E), acc, fort_e(sc[3] / nst, 20, 5).c_str(),
                fort_e(shift_meas, 20, 5).c_str(), sc[2] / nst);
    if (correlation) {
      const double sg = sc[4] / nst;
      std::printf("   wf_sgn               :%20.10f%20.10f%20.10f\n", std::fabs(sg), sg, 0.0);
    }
    std::fprintf(fa, "%12d %25.16E %25.16E\n", it, E, (E2 - E * E) / (E * E));
    e1.push_back(E);
    e2.push_back(E2 - E * E);
  }
  std::fclose(fa);
  double E, Eer, V, Ver;
  av_er(e1, E, Eer);
  av_er(e2, V, Ver);
  V /= E * E;
  Ver /= E * E;
  FILE* fv = std::fopen((dir + "/Average_Energy.txt").c_str(), "w");
  if (!fv) die("cannot write Average_Energy.txt");
  const double sq = in.Nav > 1 ? std::sqrt((double)(in.Nav - 1)) : 1.0;
  std::fprintf(fv, "%25.15f%25.15f%25.15f\n", E, Eer / sq, Eer);
  std::fprintf(fv, "%25.15E%25.15E%25.15E\n", V, Ver / sq, Ver);
  std::fprintf(fv, "%20.12f%20.12f%20.12f%20.12f\n", E, Eer / sq, V, Ver / sq);
  std::fclose(fv);
  rbmpp_destroy(lib.c);
  return 0;
}
