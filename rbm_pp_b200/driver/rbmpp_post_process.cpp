// rbmpp_post_process.cpp -- the correlation post-processing program of the Calc_Correlation code
// (Calc_Correlation/post_process/post_process.f90 with calc_av_er and bond_map of post_process/sub.f90), a
// host-only C++ program over the files that `rbmpp_driver --correlation` writes.
//
// It reads L, Nav and J1, J2 from RBM.input and, for it = 1..Nav, fort.<60000+it> (Chi_sp / norm per site
// pair) and fort.<70000+it> (Chi_vbs / norm), then writes the reference's outputs in its formats:
//   m2_SS_vs_iteration.txt, Chi_VBS_vs_iteration.txt, sub_Chi_VBS_vs_iteration.txt (per iteration)
//   Chi_SS_R.txt, Chi_SS_q.txt, total_S.txt, m2_SS_{pipi,pi0,0pi}.txt
//   Chi_VBS_R.txt, sub_Chi_VBS_R.txt, Chi_VBS_q.txt, sub_Chi_VBS_q.txt, [sub_]m2_VBS_{pipi,pi0,0pi}.txt
//   SS_correlation_{ratio,length}_{1,2}.txt, VBS_correlation_{ratio,length}_{0,1,2}.txt
//   Chi_SS_10.txt, Chi_SS_01.txt, Chi_SS_11.txt, E_chk.txt (4 x the bond sum of the averaged Chi_R).
// The reference's consistency stops (onsite correlation 1/4, Fourier symmetry, zero-distance rows) become
// an error message and exit status 1.
//
// Usage: rbmpp_post_process [--dir D]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

[[noreturn]] void die(const std::string& m) {
  std::fprintf(stderr, "rbmpp_post_process: %s\n", m.c_str());
  std::exit(1);
}

// calc_av_er of post_process/sub.f90:4-25: the mean and sqrt(sum (d - av)^2 / (N (N - 1)))
void av_er(const std::vector<double>& d, double& av, double& er) {
  const int n = (int)d.size();
  av = 0.0;
  for (double v : d) av += v;
  av /= (double)n;
  er = 0.0;
  for (double v : d) er += (v - av) * (v - av);
  er = er / (double)n / (double)(n - 1);
  er = std::sqrt(er);
}

// bond_map of post_process/sub.f90:29-74, 1-based sites
int bond_map(int L, int i0, int i1) {
  int ix = (i1 - 1) / L, iy = (i1 - 1) - ix * L;
  if (i0 == 1) {
    ix = (ix + 1) % L;
  } else if (i0 == 2) {
    iy = (iy + 1) % L;
  } else if (i0 == 3) {
    ix = (ix + 1) % L;
    iy = (iy + 1) % L;
  } else {
    ix = (ix + 1) % L;
    iy = (iy - 1 + L) % L;
  }
  return ix * L + iy + 1;
}

// Fortran Fw.d: the field of asterisks when the number does not fit, NaN right-justified
std::string ff(double v, int w, int d) {
  char b[64];
  if (std::isnan(v)) {
    std::snprintf(b, sizeof(b), "%*s", w, "NaN");
    return b;
  }
  std::snprintf(b, sizeof(b), "%*.*f", w, d, v);
  std::string s(b);
  if ((int)s.size() > w) return std::string(w, '*');
  return s;
}

struct Out {
  FILE* f;
  Out(const std::string& path) : f(std::fopen(path.c_str(), "w")) {
    if (!f) die("cannot write " + path);
  }
  ~Out() { std::fclose(f); }
  void line(const std::string& s) { std::fprintf(f, "%s\n", s.c_str()); }
};

std::string ints(std::initializer_list<int> v, int w) {
  std::string s;
  char b[32];
  for (int x : v) {
    std::snprintf(b, sizeof(b), "%*d", w, x);
    s += b;
  }
  return s;
}

std::string reals(std::initializer_list<double> v, int w = 20, int d = 10) {
  std::string s;
  for (double x : v) s += ff(x, w, d);
  return s;
}

std::vector<std::string> read_lines(const std::string& path) {
  std::ifstream in(path);
  if (!in) die("cannot read " + path);
  std::vector<std::string> out;
  std::string s;
  while (std::getline(in, s)) out.push_back(s);
  return out;
}

std::vector<double> nums(const std::string& s) {
  std::vector<double> v;
  std::string t = s;
  for (char& c : t)
    if (c == ',') c = ' ';
  std::istringstream is(t);
  std::string w;
  while (is >> w) {
    for (char& c : w)
      if (c == 'd' || c == 'D') c = 'e';
    v.push_back(std::strtod(w.c_str(), nullptr));
  }
  return v;
}

}  // namespace

int main(int argc, char** argv) {
  std::string dir = ".";
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--dir" && i + 1 < argc)
      dir = argv[++i];
    else
      die("usage: rbmpp_post_process [--dir D]");
  }
  // RBM.input (post_process.f90:38-47): line 2 L, line 4 (alphac alphar Nstep Nav ...), line 8 J1 J2
  const auto R = read_lines(dir + "/RBM.input");
  if (R.size() < 8) die("RBM.input: malformed");
  const int L = (int)nums(R[1]).at(0);
  const auto l4 = nums(R[3]);
  if (l4.size() < 4) die("RBM.input: malformed line 4");
  const int Nav = (int)l4[3];
  const auto l8 = nums(R[7]);
  if (l8.size() < 2) die("RBM.input: malformed line 8");
  const double J1 = l8[0], J2 = l8[1];
  const int N = L * L;
  const int Nchi = N * (N + 1) / 2;
  const double tpi = 2.0 * std::acos(-1.0);
  if (Nav < 1) die("Nav < 1");
  // map1(i) = (x, y) of site i = x L + y + 1 (post_process.f90:49-64)
  std::vector<int> mx(N + 1), my(N + 1);
  for (int i = 1; i <= N; i++) {
    mx[i] = (i - 1) / L;
    my[i] = (i - 1) % L;
  }
  auto map2 = [&](int x, int y) { return x * L + y + 1; };
  // arrays indexed [it][x][y] (L x L) or [it][kx][ky] ((L+1) x (L+1))
  const int LL = L * L, KK = (L + 1) * (L + 1);
  std::vector<double> RSz((size_t)Nav * LL, 0.0), RSp((size_t)Nav * LL, 0.0), RV((size_t)Nav * LL * 4, 0.0);
  std::vector<double> QSz((size_t)Nav * KK, 0.0), QSp((size_t)Nav * KK, 0.0), QV((size_t)Nav * KK * 4, 0.0);
  // Chi_{SzSz,SpSm}_{10,01,11}(it, x, k) for k = 1..N
  auto dirarr = [&]() { return std::vector<double>((size_t)Nav * L * (N + 1), 0.0); };
  std::vector<double> Sz10 = dirarr(), Sz01 = dirarr(), Sz11 = dirarr(), Sp10 = dirarr(), Sp01 = dirarr(),
                      Sp11 = dirarr();
  auto R2 = [&](std::vector<double>& a, int it, int x, int y) -> double& { return a[((size_t)it * L + x) * L + y]; };
  auto RV4 = [&](int it, int x, int y, int t) -> double& { return RV[(((size_t)it * L + x) * L + y) * 4 + t]; };
  auto Q2 = [&](std::vector<double>& a, int it, int kx, int ky) -> double& {
    return a[((size_t)it * (L + 1) + kx) * (L + 1) + ky];
  };
  auto QV4 = [&](int it, int kx, int ky, int t) -> double& {
    return QV[(((size_t)it * (L + 1) + kx) * (L + 1) + ky) * 4 + t];
  };
  auto D3 = [&](std::vector<double>& a, int it, int x, int k) -> double& {
    return a[((size_t)it * L + x) * (N + 1) + k];
  };
  std::vector<double> tmp1((size_t)(N + 1) * (N + 1), 0.0);
  Out f300(dir + "/m2_SS_vs_iteration.txt"), f301(dir + "/Chi_VBS_vs_iteration.txt"),
      f302(dir + "/sub_Chi_VBS_vs_iteration.txt");
  for (int it = 0; it < Nav; it++) {
    const auto A = read_lines(dir + "/fort." + std::to_string(60001 + it));
    const auto B = read_lines(dir + "/fort." + std::to_string(70001 + it));
    if ((int)A.size() < Nchi + 1 || (int)B.size() < Nchi + 1) die("fort.6xxxx/7xxxx: too few records");
    std::vector<int> chk(LL, 0);
    int i0 = 0;
    for (int i2 = 1; i2 <= N; i2++)
      for (int i1 = 1; i1 <= i2; i1++) {
        const auto a = nums(A[1 + i0]), b = nums(B[1 + i0]);
        i0++;
        if (a.size() < 3 || b.size() < 5) die("fort.6xxxx/7xxxx: malformed record");
        const double r1 = a[1], r2 = a[2], r3 = b[1], r4 = b[2], r5 = b[3], r6 = b[4];
        tmp1[(size_t)i1 * (N + 1) + i2] = 0.25 * (r1 + 2.0 * r2);
        tmp1[(size_t)i2 * (N + 1) + i1] = tmp1[(size_t)i1 * (N + 1) + i2];
        for (int sgn = 1; sgn >= -1; sgn -= 2) {  // displacement d and -d (post_process.f90:124-192)
          int x = sgn * (mx[i2] - mx[i1]), y = sgn * (my[i2] - my[i1]);
          if (x < 0) x += L;
          if (y < 0) y += L;
          R2(RSz, it, x, y) += r1;
          R2(RSp, it, x, y) += r2;
          RV4(it, x, y, 0) += r3;
          RV4(it, x, y, 1) += r4;
          RV4(it, x, y, 2) += r5;
          RV4(it, x, y, 3) += r6;
          const int c = ++chk[x * L + y];  // at most N off the origin when the records are consistent
          if (c > N && !(x == 0 && y == 0)) die("chk(x,y) /= N");
          if (y == 0 && x != 0) {
            D3(Sz10, it, x, c) = r1;
            D3(Sp10, it, x, c) = r2;
          }
          if (x == 0 && y != 0) {
            D3(Sz01, it, y, c) = r1;
            D3(Sp01, it, y, c) = r2;
          }
          if (x == y && x != 0) {
            D3(Sz11, it, x, c) = r1;
            D3(Sp11, it, x, c) = r2;
          }
        }
      }
    // translation average (post_process.f90:196-226)
    for (int y = 0; y < L; y++)
      for (int x = 0; x < L; x++) {
        const double nn = (x == 0 && y == 0) ? 2.0 * N : (double)N;
        if (chk[x * L + y] != (int)nn) die(x == 0 && y == 0 ? "chk(x,y) /= 2*N" : "chk(x,y) /= N");
        R2(RSz, it, x, y) *= 0.25 / nn;
        R2(RSp, it, x, y) *= 0.25 / nn;
        for (int t = 0; t < 4; t++) RV4(it, x, y, t) *= 0.25 * 0.25 / nn;
        if (x == 0 && y == 0) {
          if (std::fabs(R2(RSz, it, 0, 0) - 0.25) > 1e-5) die("onsite Chi_R wrong 1");
          if (std::fabs(R2(RSp, it, 0, 0) - 0.25) > 1e-5) die("onsite Chi_R wrong 2");
          R2(RSz, it, 0, 0) = 0.25;
          R2(RSp, it, 0, 0) = 0.25;
        }
      }
    // <B_i B_j> - <B_i><B_j> (post_process.f90:230-250)
    for (int t = 1; t <= 4; t++)
      for (int y = 0; y < L; y++)
        for (int x = 0; x < L; x++)
          for (int i1 = 1; i1 <= N; i1++) {
            const int i2 = map2((mx[i1] + x) % L, (my[i1] + y) % L);
            const int i3 = bond_map(L, t, i1), i4 = bond_map(L, t, i2);
            RV4(it, x, y, t - 1) -= tmp1[(size_t)i1 * (N + 1) + i3] * tmp1[(size_t)i2 * (N + 1) + i4] / (double)N;
          }
    // Fourier transform (post_process.f90:254-268)
    for (int ky = 0; ky <= L; ky++)
      for (int kx = 0; kx <= L; kx++)
        for (int y = 0; y < L; y++)
          for (int x = 0; x < L; x++) {
            const double c = std::cos((double)(kx * x + ky * y) * tpi / (double)L);
            Q2(QSz, it, kx, ky) += R2(RSz, it, x, y) * c;
            Q2(QSp, it, kx, ky) += R2(RSp, it, x, y) * c;
            for (int t = 0; t < 4; t++) QV4(it, kx, ky, t) += RV4(it, x, y, t) * c;
          }
    const int h = L / 2;
    const double a1 = Q2(QSz, it, h, h) + 2.0 * Q2(QSp, it, h, h);
    const double a2 = Q2(QSz, it, h, 0) + 2.0 * Q2(QSp, it, h, 0);
    const double a3 = Q2(QSz, it, 0, h) + 2.0 * Q2(QSp, it, 0, h);
    f300.line(ints({it + 1}, 5) + reals({a1 / N, a2 / N, a3 / N}));
    f301.line(ints({it + 1}, 5) + reals({QV4(it, h, 0, 0), QV4(it, h, 0, 1), QV4(it, 0, h, 0), QV4(it, 0, h, 1),
                                         QV4(it, h, h, 0), QV4(it, h, h, 1)}));
    f302.line(ints({it + 1}, 5) + reals({QV4(it, h, 0, 2), QV4(it, h, 0, 3), QV4(it, 0, h, 2), QV4(it, 0, h, 3),
                                         QV4(it, h, h, 2), QV4(it, h, h, 3)}));
  }
  auto series = [&](auto get) {
    std::vector<double> v(Nav);
    for (int it = 0; it < Nav; it++) v[it] = get(it);
    return v;
  };
  double r1, r2, r3, r4, r5, r6, r7, r8;
  // spin correlation in real space (post_process.f90:265-278)
  std::vector<double> RSz_av(LL), RSp_av(LL);
  {
    Out f(dir + "/Chi_SS_R.txt");
    for (int y = 0; y < L; y++) {
      for (int x = 0; x < L; x++) {
        av_er(series([&](int it) { return R2(RSz, it, x, y); }), r1, r2);
        av_er(series([&](int it) { return R2(RSp, it, x, y); }), r3, r4);
        av_er(series([&](int it) { return R2(RSz, it, x, y) + 2.0 * R2(RSp, it, x, y); }), r5, r6);
        f.line(ints({x, y}, 5) + reals({r5, r6, r1, r2, r3, r4}));
        RSz_av[x * L + y] = r1;
        RSp_av[x * L + y] = r3;
      }
      f.line("");
    }
  }
  {  // (post_process.f90:280-316)
    Out f101(dir + "/Chi_SS_q.txt"), f200(dir + "/total_S.txt"), f201(dir + "/m2_SS_pipi.txt"),
        f202(dir + "/m2_SS_pi0.txt"), f203(dir + "/m2_SS_0pi.txt");
    f200.line("#  total  SzSz  SpSm");
    for (int ky = 0; ky <= L; ky++) {
      for (int kx = 0; kx <= L; kx++) {
        av_er(series([&](int it) { return Q2(QSz, it, kx, ky); }), r1, r2);
        av_er(series([&](int it) { return Q2(QSp, it, kx, ky); }), r3, r4);
        av_er(series([&](int it) { return Q2(QSz, it, kx, ky) + 2.0 * Q2(QSp, it, kx, ky); }), r5, r6);
        f101.line(ints({kx, ky}, 5) + reals({r5, r6, r1, r2, r3, r4}));
        if (kx == 0 && ky == 0)
          f200.line(reals({r5 * N, r6 * N, r1 * N, r2 * N, r3 * N, r4 * N}));
        else if (kx == L / 2 && ky == L / 2)
          f201.line(reals({r5 / N, r6 / N, r1 / N, r2 / N, r3 / N, r4 / N}));
        else if (kx == L / 2 && ky == 0)
          f202.line(reals({r5 / N, r6 / N, r1 / N, r2 / N, r3 / N, r4 / N}));
        else if (kx == 0 && ky == L / 2)
          f203.line(reals({r5 / N, r6 / N, r1 / N, r2 / N, r3 / N, r4 / N}));
      }
      f101.line("");
    }
  }
  // VBS correlation in real and momentum space, bond types (1,2) and, as sub_*, (3,4) (:321-389)
  for (int part = 0; part < 2; part++) {
    const int t0 = 2 * part;
    const std::string pre = part ? "sub_" : "";
    {
      Out f(dir + "/" + pre + "Chi_VBS_R.txt");
      for (int y = 0; y < L; y++) {
        for (int x = 0; x < L; x++) {
          av_er(series([&](int it) { return RV4(it, x, y, t0); }), r1, r2);
          av_er(series([&](int it) { return RV4(it, x, y, t0 + 1); }), r3, r4);
          f.line(ints({x, y}, 5) + reals({r1, r2, r3, r4}));
        }
        f.line("");
      }
    }
    Out f401(dir + "/" + pre + "Chi_VBS_q.txt"), f501(dir + "/" + pre + "m2_VBS_pipi.txt"),
        f502(dir + "/" + pre + "m2_VBS_pi0.txt"), f503(dir + "/" + pre + "m2_VBS_0pi.txt");
    for (int ky = 0; ky <= L; ky++) {
      for (int kx = 0; kx <= L; kx++) {
        av_er(series([&](int it) { return QV4(it, kx, ky, t0); }), r1, r2);
        av_er(series([&](int it) { return QV4(it, kx, ky, t0 + 1); }), r3, r4);
        f401.line(ints({kx, ky}, 5) + reals({r1, r2, r3, r4}));
        r1 /= N;
        r2 /= N;
        r3 /= N;
        r4 /= N;
        if (kx == L / 2 && ky == L / 2) f501.line(reals({r1, r2, r3, r4}));
        if (kx == L / 2 && ky == 0) f502.line(reals({r1, r2, r3, r4}));
        if (kx == 0 && ky == L / 2) f503.line(reals({r1, r2, r3, r4}));
      }
      f401.line("");
    }
  }
  const int h = L / 2;
  const double pi = std::acos(-1.0);
  auto S = [&](int it, int kx, int ky) { return Q2(QSz, it, kx, ky) + 2.0 * Q2(QSp, it, kx, ky); };
  // spin correlation ratios and lengths (:393-429)
  for (int variant = 1; variant <= 2; variant++) {
    std::vector<double> c2(Nav), c3(Nav);
    for (int it = 0; it < Nav; it++) {
      const double s1 = S(it, h, h);
      const double s6 = variant == 1
                            ? 0.25 * (S(it, h + 1, h) + S(it, h, h + 1) + S(it, h - 1, h) + S(it, h, h - 1))
                            : 0.25 * (S(it, h - 1, h - 1) + S(it, h + 1, h - 1) + S(it, h - 1, h + 1) +
                                      S(it, h + 1, h + 1));
      c2[it] = 1.0 - s6 / s1;
      c3[it] = std::sqrt(s1 / s6 - 1.0) / 2.0 / pi;
    }
    av_er(c2, r1, r2);
    av_er(c3, r3, r4);
    Out fr(dir + "/SS_correlation_ratio_" + std::to_string(variant) + ".txt");
    Out fl(dir + "/SS_correlation_length_" + std::to_string(variant) + ".txt");
    fr.line(reals({r1, r2}));
    fl.line(ints({L}, 5) + ff(J2, 10, 5) + reals({r3, r4}));
  }
  // VBS correlation ratios and lengths: variants 1, 2 (:432-503) and 0 (:505-543)
  auto sym = [&](double a, double b, int n) {
    if (std::fabs(a - b) > 1e-4) die("Chi_q_VBS symmetry wrong " + std::to_string(n));
  };
  auto V = [&](int it, int kx, int ky, int t) { return QV4(it, kx, ky, t); };
  for (int variant : {1, 2, 0}) {
    std::vector<double> c2(Nav), c3(Nav), c4(Nav), c5(Nav);
    const int nb = variant == 1 ? 1 : (variant == 2 ? 4 : 7);
    for (int it = 0; it < Nav; it++) {
      // one bond type: along x (type 1) with k = (L/2, 0), along y (type 2) with k = (0, L/2)
      auto ratio = [&](int t, bool xdir, int chk0) {
        auto q = [&](int a, int b) { return xdir ? V(it, a, b, t) : V(it, b, a, t); };
        const double s1 = q(h, 0);
        if (variant == 1) {
          const double s2 = q(h + 1, 0), s3 = q(h - 1, 0);
          sym(s2, s3, chk0);
          return 1.0 - 0.5 * (s2 + s3) / s1;
        }
        if (variant == 2) {
          const double s2 = q(h, 1), s3 = q(h, L - 1);
          sym(s2, s3, chk0);
          return 1.0 - 0.5 * (s2 + s3) / s1;
        }
        const double s2 = q(h + 1, 0), s3 = q(h - 1, 0), s4 = q(h, 1), s5 = q(h, L - 1);
        sym(s2, s3, chk0);
        sym(s4, s5, chk0 + 1);
        return 1.0 - 0.25 * (s2 + s3 + s4 + s5) / s1;
      };
      c2[it] = ratio(0, true, nb);
      c3[it] = ratio(1, false, variant == 0 ? nb + 2 : nb + 1);
      auto tot = [&](int a, int b) { return V(it, a, b, 0) + V(it, b, a, 1); };
      const double s1 = tot(h, 0);
      double s6;
      if (variant == 1) {
        const double s2 = tot(h + 1, 0), s3 = tot(h - 1, 0);
        sym(s2, s3, nb + 2);
        s6 = 0.5 * (s2 + s3);
      } else if (variant == 2) {
        const double s2 = tot(h, 1), s3 = tot(h, L - 1);
        sym(s2, s3, nb + 2);
        s6 = 0.5 * (s2 + s3);
      } else {
        const double s2 = tot(h + 1, 0), s3 = tot(h - 1, 0), s4 = tot(h, 1), s5 = tot(h, L - 1);
        sym(s2, s3, nb + 4);
        sym(s4, s5, nb + 5);
        s6 = 0.25 * (s2 + s3 + s4 + s5);
      }
      c4[it] = 1.0 - s6 / s1;
      c5[it] = std::sqrt(s1 / s6 - 1.0) / 2.0 / pi;
    }
    av_er(c2, r1, r2);
    av_er(c3, r3, r4);
    av_er(c4, r5, r6);
    av_er(c5, r7, r8);
    Out fr(dir + "/VBS_correlation_ratio_" + std::to_string(variant) + ".txt");
    Out fl(dir + "/VBS_correlation_length_" + std::to_string(variant) + ".txt");
    fr.line(reals({r5, r6, r1, r2, r3, r4}));
    fl.line(ints({L}, 5) + ff(J2, 10, 5) + reals({r7, r8}));
  }
  // spin correlation along (1,0), (0,1), (1,1) (:547-621); entries are 1/4 of the Chi_sp records
  {
    Out f102(dir + "/Chi_SS_10.txt"), f103(dir + "/Chi_SS_01.txt"), f104(dir + "/Chi_SS_11.txt");
    auto emit = [&](Out& f, std::vector<double>& Sz, std::vector<double>& Sp, int x, int k, const char* nm) {
      av_er(series([&](int it) { return 0.25 * D3(Sz, it, x, k); }), r1, r2);
      av_er(series([&](int it) { return 0.25 * D3(Sp, it, x, k); }), r3, r4);
      av_er(series([&](int it) { return 0.25 * D3(Sz, it, x, k) + 2.0 * 0.25 * D3(Sp, it, x, k); }), r5, r6);
      if (x == 0) {
        for (double v : {r1, r2, r3, r4, r5, r6})
          if (std::fabs(v) > 1e-5) die(std::string(nm) + " wrong");
        r1 = 0.25;
        r3 = 0.25;
        r5 = 0.75;
      }
      f.line(ints({x, k}, 5) + reals({r5, r6, r1, r2, r3, r4}));
    };
    for (int k = 1; k <= N; k++) {
      for (int x = 0; x < L; x++) {
        emit(f102, Sz10, Sp10, x, k, "Chi_SS_10");
        emit(f103, Sz01, Sp01, x, k, "Chi_SS_01");
        emit(f104, Sz11, Sp11, x, k, "Chi_SS_11");
      }
      f102.line("");
      f103.line("");
      f104.line("");
    }
  }
  // energy check (:623-644): 4 x the bond sum of the averaged Chi_R
  double E = 0.0;
  for (int t = 1; t <= 4; t++)
    for (int i1 = 1; i1 <= N; i1++) {
      const int i2 = bond_map(L, t, i1);
      int x = mx[i2] - mx[i1], y = my[i2] - my[i1];
      if (x < 0) x += L;
      if (y < 0) y += L;
      if (x == 0 && y == 0) die("x == 0 .and. y == 0");
      E += (t <= 2 ? J1 : J2) * (RSz_av[x * L + y] + 2.0 * RSp_av[x * L + y]);
    }
  Out f105(dir + "/E_chk.txt");
  f105.line(ff(E * 4.0, 20, 12));
  return 0;
}
