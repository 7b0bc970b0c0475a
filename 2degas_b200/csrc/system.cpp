// system.cpp - host-side reader of the reference's run directory: the
// keyword file <runid>.sy, the spline tables it names, the k-vector file and
// the walker configuration files. Restates `input` (reptation.f:12-710),
// `readwords` (:4790), `t_read` (:4689), `kread` (:4740), `read_conf`
// (:2452) and the orbital wave-vector builds of `input` (:674-708) and
// `tabc`/`twistg` (:9559, :9818) with the heapsort SORTTF (:9514).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/qmc2d.h"
#include "common.h"

namespace {

// Split one record of a table or k-vector file into blank-separated words.
// List-directed reads see the whole record (only the keyword file's
// readwords is limited to 80 columns).
std::vector<std::string> words_of(const std::string &rec) {
  std::vector<std::string> w;
  std::istringstream is(rec);
  std::string s;
  while (is >> s) w.push_back(s);
  return w;
}

// Fortran list-directed real: accepts d/D exponents.
bool fnum(const std::string &s, double *v) {
  std::string t = s;
  for (auto &c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  *v = std::strtod(t.c_str(), &end);
  return end != t.c_str() && (*end == 0 || *end == ',');
}

// Sequential record reader with Fortran list-directed semantics: every read
// starts on a fresh record and consumes as many records as its item list
// needs; what is left on the last record is discarded.
struct Records {
  std::vector<std::string> lines;
  size_t pos = 0;
  bool eof() const { return pos >= lines.size(); }
  bool read_reals(int n, double *out) {
    int got = 0;
    while (got < n) {
      if (eof()) return false;
      auto w = words_of(lines[pos++] + std::string(""));
      for (auto &s : w) {
        if (got == n) break;
        if (!fnum(s, &out[got])) return false;
        got++;
      }
    }
    return true;
  }
  bool read_word(std::string *s) {
    while (!eof()) {
      auto w = words_of(lines[pos++]);
      if (!w.empty()) {
        *s = w[0];
        return true;
      }
    }
    return false;
  }
  void skip(int n) { pos += n; }
};

bool load_lines(const std::string &path, std::vector<std::string> *lines) {
  std::ifstream f(path);
  if (!f) return false;
  std::string l;
  while (std::getline(f, l)) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    lines->push_back(l);
  }
  return true;
}

std::string join(const std::string &dir, const std::string &name) {
  if (dir.empty() || name.empty() || name[0] == '/') return name;
  return dir + "/" + name;
}

// t_read (reptation.f:4689-4738): returns the table index, deduplicated by
// file name; sets the shared knot spacing.
int t_read(qmc2d_system *sys, const std::string &dir, const std::string &file) {
  for (int i = 0; i < sys->ntables; i++)
    if (file == sys->tables[i].name) return i;
  if (sys->ntables >= QMC2D_MAX_TABLES) {
    q2d::set_error("too many tables");
    return -QMC2D_ERR_LIMIT;
  }
  Records rec;
  if (!load_lines(join(dir, file), &rec.lines)) {
    q2d::set_error("cannot open table " + join(dir, file));
    return -QMC2D_ERR_IO;
  }
  qmc2d_table *t = &sys->tables[sys->ntables];
  std::memset(t, 0, sizeof(*t));
  std::snprintf(t->name, sizeof(t->name), "%s", file.c_str());
  double hdr[2];
  if (!rec.read_reals(2, hdr)) {
    q2d::set_error("bad table header in " + file);
    return -QMC2D_ERR_PARSE;
  }
  t->ngrid = (int)hdr[0];
  if (t->ngrid < 1 || t->ngrid > 100000) {
    q2d::set_error("bad knot count in " + file);
    return -QMC2D_ERR_PARSE;
  }
  sys->drt = hdr[1];
  t->ut = (double *)std::calloc((size_t)4 * (t->ngrid + 1), sizeof(double));
  for (int i = 0; i <= t->ngrid; i++)
    if (!rec.read_reals(4, t->ut + 4 * i)) {
      q2d::set_error("short table " + file);
      return -QMC2D_ERR_PARSE;
    }
  std::string routine;
  if (rec.read_word(&routine)) {
    double np_;
    if (rec.read_reals(1, &np_)) {
      rec.skip((int)np_);
      std::string kw;
      if (rec.read_word(&kw) && kw == "kspace") {
        double nk;
        if (!rec.read_reals(1, &nk)) return -QMC2D_ERR_PARSE;
        t->nk_ewald = (int)nk;
        t->vk = (double *)std::calloc((size_t)t->nk_ewald + 1, sizeof(double));
        for (int k = 0; k <= t->nk_ewald; k++)
          if (!rec.read_reals(1, &t->vk[k])) {
            q2d::set_error("short k-space block in " + file);
            return -QMC2D_ERR_PARSE;
          }
      }
    }
  }
  sys->drti = 1.0 / sys->drt;
  sys->drti2 = 2.0 * sys->drti * sys->drti;
  return sys->ntables++;
}

// kread (reptation.f:4740-4769)
int kread(qmc2d_system *sys, const std::string &dir, const std::string &file) {
  Records rec;
  if (!load_lines(join(dir, file), &rec.lines)) {
    q2d::set_error("cannot open k-vector file " + join(dir, file));
    return QMC2D_ERR_IO;
  }
  std::vector<double> k;
  double v[2];
  while (!rec.eof()) {
    size_t save = rec.pos;
    if (words_of(rec.lines[rec.pos]).empty()) {
      rec.pos++;
      continue;
    }
    rec.pos = save;
    if (!rec.read_reals(2, v)) break;
    k.push_back(v[0]);
    k.push_back(v[1]);
  }
  sys->nk = (int)(k.size() / 2);
  if (sys->nk > QMC2D_MAX_NK) {
    q2d::set_error("too many k vectors");
    return QMC2D_ERR_LIMIT;
  }
  std::free(sys->kvec);
  sys->kvec = (double *)std::malloc(sizeof(double) * (k.size() + 2));
  std::memcpy(sys->kvec, k.data(), sizeof(double) * k.size());
  return QMC2D_OK;
}

}  // namespace

int q2d_t_read(qmc2d_system *sys, const std::string &dir, const std::string &file) {
  return t_read(sys, dir, file);
}
int q2d_kread(qmc2d_system *sys, const std::string &dir, const std::string &file) {
  return kread(sys, dir, file);
}

// SORTTF (reptation.f:9514-9557): heapsort of an index vector by a(.),
// 1-based arrays as in the original so ties fall out the same way.
void q2d::sorttf(int n1, const double *a1, int *index1) {
  const double *A = a1 - 1;
  int *INDEX = index1 - 1;
  int N = n1, I1, I2, I3, I22, I33, I222;
  double AI;
  for (I1 = 2; I1 <= N; I1++) {
    I3 = I1;
    I33 = INDEX[I3];
    AI = A[I33];
  L1:
    I2 = I3 / 2;
    if (I2 <= 0) goto L3;
    I22 = INDEX[I2];
    if (AI <= A[I22]) goto L3;
    INDEX[I3] = I22;
    I3 = I2;
    goto L1;
  L3:
    INDEX[I3] = I33;
  }
L4:
  I3 = INDEX[N];
  INDEX[N] = INDEX[1];
  AI = A[I3];
  N = N - 1;
  if (N - 1 <= 0) goto L12;
  I1 = 1;
L6:
  I2 = I1 + I1;
  if (I2 <= N) I22 = INDEX[I2];
  if (I2 - N < 0) goto L7;
  if (I2 - N == 0) goto L9;
  goto L11;
L7:
  I222 = INDEX[I2 + 1];
  if (A[I22] - A[I222] < 0) goto L8;
  goto L9;
L8:
  I2 = I2 + 1;
  I22 = I222;
L9:
  if (AI - A[I22] < 0) goto L10;
  goto L11;
L10:
  INDEX[I1] = I22;
  I1 = I2;
  goto L6;
L11:
  INDEX[I1] = I3;
  goto L4;
L12:
  INDEX[1] = I3;
}

extern "C" int qmc2d_system_set_twist(qmc2d_system *sys, int ith, int jth) {
  if (!sys || sys->nk <= 0) return QMC2D_ERR_ARG;
  int ng = 2 * sys->nk + 1;
  std::vector<double> gvec(2 * ng), gnorm2(ng);
  const double pi = std::acos(-1.0);
  if (ith == 0 && jth == 0) {
    // Gamma point (input, reptation.f:674-708): 0, then +k_i, -k_i.
    gvec[0] = gvec[1] = 0.0;
    int j = 1;
    for (int i = 0; i < sys->nk; i++) {
      for (int d = 0; d < 2; d++) {
        gvec[2 * j + d] = sys->kvec[2 * i + d];
        gvec[2 * (j + 1) + d] = -sys->kvec[2 * i + d];
      }
      j += 2;
    }
  } else {
    // twistg (reptation.f:9818-9861)
    double theta[2];
    theta[0] = ith * 2.0 * pi * sys->eli[0] / sys->ntheta;
    theta[1] = jth * 2.0 * pi * sys->eli[1] / sys->ntheta;
    std::vector<double> gv(2 * ng);
    std::vector<int> igvec(ng);
    gnorm2[0] = 0.0;
    for (int d = 0; d < 2; d++) {
      gv[d] = theta[d];
      gnorm2[0] = gnorm2[0] + gv[d] * gv[d];
    }
    igvec[0] = 1;
    for (int k = sys->nk; k >= 1; k--) {
      int a = 2 * k, b = 2 * k + 1;  // 1-based slots
      gnorm2[b - 1] = 0.0;
      gnorm2[a - 1] = 0.0;
      for (int d = 0; d < 2; d++) {
        gv[2 * (b - 1) + d] = -sys->kvec[2 * (k - 1) + d] + theta[d];
        gv[2 * (a - 1) + d] = sys->kvec[2 * (k - 1) + d] + theta[d];
        gnorm2[b - 1] = gnorm2[b - 1] + gv[2 * (b - 1) + d] * gv[2 * (b - 1) + d];
        gnorm2[a - 1] = gnorm2[a - 1] + gv[2 * (a - 1) + d] * gv[2 * (a - 1) + d];
      }
      igvec[a - 1] = a;
      igvec[b - 1] = b;
    }
    q2d::sorttf(ng, gnorm2.data(), igvec.data());
    for (int k = 0; k < ng; k++)
      for (int d = 0; d < 2; d++) gvec[2 * k + d] = gv[2 * (igvec[k] - 1) + d];
  }
  std::free(sys->gvec);
  sys->gvec = (double *)std::malloc(sizeof(double) * 2 * ng);
  std::memcpy(sys->gvec, gvec.data(), sizeof(double) * 2 * ng);
  sys->ngvec = ng;
  sys->ith = ith;
  sys->jth = jth;
  return QMC2D_OK;
}

extern "C" void qmc2d_system_free(qmc2d_system *sys) {
  if (!sys) return;
  for (int i = 0; i < sys->ntables; i++) {
    std::free(sys->tables[i].ut);
    std::free(sys->tables[i].vk);
  }
  std::free(sys->kvec);
  std::free(sys->gvec);
  std::free(sys);
}
