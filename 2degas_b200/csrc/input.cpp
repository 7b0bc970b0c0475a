// input.cpp - the keyword pass of `input` (reptation.f:12-710) for the
// walker path, and read_conf's configuration reader (reptation.f:2452-2491).
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
thread_local std::string g_error;
}

void q2d::set_error(const std::string &msg) { g_error = msg; }
extern "C" const char *qmc2d_last_error(void) { return g_error.c_str(); }
extern "C" const char *qmc2d_version(void) { return "qmc2d-b200 1.0 (sm_100a)"; }

// Defined in system.cpp (file-local there); re-declared for the pass below.
int q2d_t_read(qmc2d_system *sys, const std::string &dir, const std::string &file);
int q2d_kread(qmc2d_system *sys, const std::string &dir, const std::string &file);

namespace {

std::vector<std::string> words_of(const std::string &rec) {
  std::string r = rec.substr(0, 80);  // character*80 record
  std::vector<std::string> w;
  std::istringstream is(r);
  std::string s;
  while (is >> s) w.push_back(s);
  return w;
}

bool fnum(const std::string &s, double *v) {
  std::string t = s;
  for (auto &c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  *v = std::strtod(t.c_str(), &end);
  return end != t.c_str() && *end == 0;
}

bool fint(const std::string &s, int *v) {
  double d;
  if (!fnum(s, &d)) return false;
  *v = (int)d;
  return true;
}

std::string join(const std::string &dir, const std::string &name) {
  if (dir.empty() || name.empty() || name[0] == '/') return name;
  return dir + "/" + name;
}

int fail(int code, const std::string &msg) {
  q2d::set_error(msg);
  return code;
}

// Table-kind consistency: the reference walks one shared pair list and each
// pair term advances its own pair counter only for type pairs that have a
// table, so a kind set for some type pairs but not others would misalign
// the pair arrays. Accept a kind only for all type pairs or for none.
int check_all_or_none(const qmc2d_system *s, const int tab[QMC2D_MAX_TYPES][QMC2D_MAX_TYPES],
                      const char *kind) {
  int set = 0, tot = 0;
  for (int a = 0; a < s->ntypes; a++)
    for (int b = a; b < s->ntypes; b++) {
      tot++;
      set += tab[a][b] >= 0;
    }
  if (set != 0 && set != tot)
    return fail(QMC2D_ERR_UNSUPPORTED,
                std::string(kind) + " must be given for every pair of types or for none");
  return QMC2D_OK;
}

int finish(qmc2d_system *s) {
  if (s->ndim != 2) return fail(QMC2D_ERR_UNSUPPORTED, "ndim must be 2");
  if (s->ntypes < 1) return fail(QMC2D_ERR_PARSE, "no particle types");
  s->nptot = 0;
  s->npnorm = 0;
  for (int it = 0; it < s->ntypes; it++) {
    if (s->hbs2m[it] == 0.0)
      return fail(QMC2D_ERR_UNSUPPORTED, "static particle types (hbs2m = 0) are not supported");
    s->ipfrst[it] = s->nptot;
    s->nptot += s->np[it];
    s->npnorm += s->np[it];
  }
  if (s->nptot > QMC2D_MAX_NP) return fail(QMC2D_ERR_LIMIT, "too many particles");
  int st;
  if ((st = check_all_or_none(s, s->iu2, "u2"))) return st;
  if ((st = check_all_or_none(s, s->iu3, "u3"))) return st;
  if ((st = check_all_or_none(s, s->iub, "backflow"))) return st;
  if ((st = check_all_or_none(s, s->iv2, "v2"))) return st;
  if (s->el[0] <= 0.0 || s->el[1] <= 0.0) return fail(QMC2D_ERR_UNSUPPORTED, "pbc is required");
  // property layout (reptation.f:577-637)
  s->n_scalar_props = QMC2D_NSCALAR(s->ntypes);
  s->jrhok = s->n_scalar_props;
  s->n_props = s->n_scalar_props + 2 * s->nk * s->nrhok;
  // k-space potential reads rho_k of every type (reptation.f:4034-4052)
  for (int a = 0; a < s->ntypes; a++)
    for (int b = 0; b < s->ntypes; b++) {
      int iv = s->iv2[a][b];
      if (iv >= 0 && s->tables[iv].nk_ewald > 0) {
        if (s->tables[iv].nk_ewald > s->nk)
          return fail(QMC2D_ERR_PARSE, "v2 table has more k points than kspace");
        for (int t = 0; t < s->ntypes; t++)
          if (s->irhok[t] != t + 1)
            return fail(QMC2D_ERR_UNSUPPORTED,
                        "a k-space pair potential needs 'rhok' for every type, in type order");
      }
    }
  bool backflow = s->iub[0][0] >= 0;
  if (backflow) {
    if (s->nk <= 0) return fail(QMC2D_ERR_PARSE, "backflow needs kspace");
    // input builds the Gamma-point wave vectors only when ibckf != 0
    // (reptation.f:679): with ibckf 0 and no twists every orbital would be
    // the k = 0 constant and the determinant singular
    if (s->ntheta == 0 && s->ibckf == 0)
      return fail(QMC2D_ERR_UNSUPPORTED,
                  "backflow with ibckf 0 at the Gamma point: no orbital wave vectors");
    for (int it = 0; it < s->ntypes; it++)
      if (s->np[it] > QMC2D_MAX_ORB || s->np[it] > 2 * s->nk + 1)
        return fail(QMC2D_ERR_LIMIT, "not enough orbitals for the determinant");
    int st2 = s->ntheta == 0 ? qmc2d_system_set_twist(s, 0, 0)
                             : qmc2d_system_set_twist(s, 1, 1);  // first twist of tabc
    if (st2) return st2;
  }
  return QMC2D_OK;
}

}  // namespace

extern "C" int qmc2d_system_read(const char *dir_c, const char *runid_c, qmc2d_system **out) {
  if (!out || !runid_c) return fail(QMC2D_ERR_ARG, "null argument");
  *out = nullptr;
  std::string dir = dir_c ? dir_c : "";
  std::string runid = runid_c;
  qmc2d_system *s = (qmc2d_system *)std::calloc(1, sizeof(qmc2d_system));
  if (!s) return fail(QMC2D_ERR_NOMEM, "out of host memory");
  s->ndim = 2;
  for (int a = 0; a < QMC2D_MAX_TYPES; a++)
    for (int b = 0; b < QMC2D_MAX_TYPES; b++)
      s->iu2[a][b] = s->iu3[a][b] = s->iub[a][b] = s->iv2[a][b] = -1;
  s->rejection = 1;
  s->seed[0] = s->seed[1] = s->seed[2] = 0;
  s->seed[3] = 1;
  s->ref_underflow_return = 1;
  // 'seed' file of the run directory (reptation.f:31-33)
  {
    std::ifstream f(join(dir, "seed"));
    int v[4];
    if (f && (f >> v[0] >> v[1] >> v[2] >> v[3]))
      for (int i = 0; i < 4; i++) s->seed[i] = v[i];
  }
  std::ifstream f(join(dir, runid + ".sy"));
  if (!f) {
    qmc2d_system_free(s);
    return fail(QMC2D_ERR_IO, "cannot open " + join(dir, runid + ".sy"));
  }
  std::string line;
  int st = QMC2D_OK;
  bool ended = false;
  auto ty = [&](const std::string &n) {
    for (int i = 0; i < s->ntypes; i++)
      if (n == s->type_name[i]) return i;
    return -1;
  };
  while (!ended && st == QMC2D_OK && std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    auto w = words_of(line);
    if (w.empty()) {
      st = fail(QMC2D_ERR_PARSE, "blank record: not a keyword");
      break;
    }
    const std::string &k = w[0];
    auto need = [&](size_t n) {
      if (w.size() < n) st = fail(QMC2D_ERR_PARSE, "too few words in '" + k + "' record");
      return st == QMC2D_OK;
    };
    if (k == "end") {
      ended = true;
    } else if (k == "ndim") {
      if (need(2) && !fint(w[1], &s->ndim)) st = fail(QMC2D_ERR_PARSE, "ndim");
    } else if (k == "v0") {
      if (need(2) && !fnum(w[1], &s->v0)) st = fail(QMC2D_ERR_PARSE, "v0");
    } else if (k == "adrift") {
      if (need(2) && !fnum(w[1], &s->adrift)) st = fail(QMC2D_ERR_PARSE, "adrift");
    } else if (k == "gstorto") {
      if (need(2)) fint(w[1], &s->gstorto);
    } else if (k == "wpiu") {
      if (need(2)) fint(w[1], &s->wpiu);
    } else if (k == "nodalaction") {
      if (need(2)) fint(w[1], &s->nodalaction);
    } else if (k == "rejection") {
      if (need(2)) fint(w[1], &s->rejection);
    } else if (k == "fullprop") {
      // only used by the rmc energy-derivative estimators (out of scope)
    } else if (k == "ecut") {
      if (need(2)) {
        fint(w[1], &s->ecut);
        if (s->ecut != 0 && need(3)) fnum(w[2], &s->value_ecut);
      }
    } else if (k == "seed") {
      if (need(5))
        for (int i = 0; i < 4; i++) fint(w[i + 1], &s->seed[i]);
    } else if (k == "pbc") {
      if (need(3))
        for (int i = 0; i < 2; i++) {
          fnum(w[i + 1], &s->el[i]);
          s->eli[i] = 1.0 / s->el[i];
        }
    } else if (k == "kspace") {
      if (need(2)) st = q2d_kread(s, dir, w[1]);
    } else if (k == "rhok") {
      if (need(2)) {
        int it = ty(w[1]);
        if (it < 0) st = fail(QMC2D_ERR_PARSE, "rhok: unknown type " + w[1]);
        else s->irhok[it] = ++s->nrhok;
      }
    } else if (k == "type") {
      if (need(5)) {
        if (s->ntypes >= QMC2D_MAX_TYPES) {
          st = fail(QMC2D_ERR_LIMIT, "at most two particle types");
        } else {
          int it = s->ntypes++;
          std::snprintf(s->type_name[it], QMC2D_NAME_LEN, "%s", w[1].c_str());
          fint(w[2], &s->np[it]);
          fnum(w[3], &s->hbs2m[it]);
          std::snprintf(s->x_file[it], QMC2D_NAME_LEN, "%s", w[4].c_str());
        }
      }
    } else if (k == "v2" || k == "u2" || k == "u3" || k == "backflow") {
      size_t tw = k == "backflow" ? 5 : 4;  // backflow it jt ibckf table
      if (need(tw)) {
        int it = ty(w[1]), jt = ty(w[2]);
        if (it < 0 || jt < 0) {
          st = fail(QMC2D_ERR_PARSE, k + ": unknown type");
        } else {
          if (k == "backflow") fint(w[3], &s->ibckf);
          int i = q2d_t_read(s, dir, w[tw - 1]);
          if (i < 0) {
            st = -i;
          } else {
            int(*tab)[QMC2D_MAX_TYPES] =
                k == "v2" ? s->iv2 : k == "u2" ? s->iu2 : k == "u3" ? s->iu3 : s->iub;
            tab[it][jt] = tab[jt][it] = i;
            if (k == "v2") {
              if (need(6)) {
                fnum(w[4], &s->tables[i].tail);
                fint(w[5], &s->tables[i].iexp);
              }
            }
          }
        }
      }
    } else if (k == "ntwists") {
      if (need(2)) fint(w[1], &s->ntheta);
    } else if (k == "mstar" || k == "cmass" || k == "itc") {
      // path-estimator records, set up when reptation starts
      int *n = k == "mstar" ? &s->nmstar : k == "cmass" ? &s->ncmass : &s->nitc;
      char(*rec)[QMC2D_RECORD_LEN] =
          k == "mstar" ? s->mstar_record : k == "cmass" ? s->cmass_record : s->itc_record;
      if (*n >= QMC2D_MAX_EST) {
        st = fail(QMC2D_ERR_LIMIT, "too many '" + k + "' records");
      } else {
        std::string r;
        for (size_t i = 1; i < w.size(); i++) r += (i > 1 ? " " : "") + w[i];
        if (r.size() >= QMC2D_RECORD_LEN) st = fail(QMC2D_ERR_LIMIT, "'" + k + "' record too long");
        else std::snprintf(rec[(*n)++], QMC2D_RECORD_LEN, "%s", r.c_str());
      }
    } else {
      st = fail(QMC2D_ERR_UNSUPPORTED, "keyword outside the walker path: " + k);
    }
  }
  if (st == QMC2D_OK) st = finish(s);
  if (st != QMC2D_OK) {
    qmc2d_system_free(s);
    return st;
  }
  *out = s;
  return QMC2D_OK;
}

extern "C" int qmc2d_read_configs(const qmc2d_system *sys, const char *dir_c, const char *suffix,
                                  int first, int count, double *x, int *nread) {
  if (!sys || !x || count < 0 || first < 0) return fail(QMC2D_ERR_ARG, "bad argument");
  std::string dir = dir_c ? dir_c : "";
  int N = sys->nptot;
  int got = count;
  for (int it = 0; it < sys->ntypes; it++) {
    std::string path = join(dir, std::string(sys->x_file[it]) + (suffix ? suffix : ""));
    std::ifstream f(path);
    if (!f) return fail(QMC2D_ERR_IO, "cannot open " + path);
    std::string line;
    int c = 0, ip = 0;
    long skip = (long)first * sys->np[it];
    while (c < got && std::getline(f, line)) {
      auto w = words_of(line);
      if (w.empty()) continue;
      if (skip > 0) {
        skip--;
        continue;
      }
      double v[2];
      if (w.size() < 2 || !fnum(w[0], &v[0]) || !fnum(w[1], &v[1]))
        return fail(QMC2D_ERR_PARSE, "bad coordinate line in " + path);
      int p = sys->ipfrst[it] + ip;
      x[(size_t)2 * N * c + 2 * p] = v[0];
      x[(size_t)2 * N * c + 2 * p + 1] = v[1];
      if (++ip == sys->np[it]) {
        ip = 0;
        c++;
      }
    }
    if (c < got) got = c;
  }
  if (nread) *nread = got;
  return QMC2D_OK;
}
