// io.cpp - host-side block statistics and checkpoints: averages(3) and
// write_nonscalar_props (reptation.f:4305-4352, 4582-4616), write_conf
// (:2504) and restart (:4439-4541), in the reference's file formats.
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
#include "handle.h"

struct qmc2d_stats {
  int n_props = 0, iblk = 0;
  double cml_norm = 0.0;
  std::vector<double> cml_av, cml2;
};

namespace {

int fail(int code, const std::string &msg) {
  q2d::set_error(msg);
  return code;
}

std::string join(const std::string &dir, const std::string &name) {
  if (dir.empty()) return name;
  return dir.back() == '/' ? dir + name : dir + "/" + name;
}

// Fortran Ew.d output: 0.<d digits>E+xx (sign-magnitude exponent, no E for
// three-digit exponents), right-justified in w columns, asterisks if too
// wide. The digits are C's correctly rounded %e digits.
std::string fe(double v, int w, int d) {
  std::string s;
  if (std::isnan(v)) {
    s = "NaN";
  } else if (std::isinf(v)) {
    s = v < 0 ? "-Infinity" : "Infinity";
  } else if (v == 0.0) {
    s = "0." + std::string(d, '0') + "E+00";
  } else {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(v));
    std::string digs(1, buf[0]);
    const char *p = buf + 1;
    if (*p == '.')
      for (p++; *p && *p != 'e'; p++) digs += *p;
    while (*p && *p != 'e') p++;
    const int ex = std::atoi(p + 1) + 1;
    char eb[16];
    if (std::abs(ex) <= 99)
      std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else
      std::snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    s = std::string(v < 0 ? "-" : "") + "0." + digs + eb;
  }
  if ((int)s.size() < w) return std::string(w - s.size(), ' ') + s;
  if ((int)s.size() > w) return std::string(w, '*');
  return s;
}

std::string fa(const std::string &t, int w) {  // Fortran Aw output
  if ((int)t.size() >= w) return t.substr(0, w);
  return t + std::string(w - t.size(), ' ');
}

std::string fi(long v, int w) {  // Fortran Iw output
  std::string s = std::to_string(v);
  if ((int)s.size() > w) return std::string(w, '*');
  return std::string(w - s.size(), ' ') + s;
}

// The scalar property names of the reference (reptation.f:577-615).
std::string scalar_name(const qmc2d_system *sys, int i) {
  static const char *fixed[] = {"elocal", "-log tf", "acc.rate", "epot", "ekin", "e2", "gg"};
  const int nt = sys->ntypes;
  if (i < 7) return fixed[i];
  i -= 7;
  if (i < nt) return std::string("pot_") + sys->type_name[i];
  i -= nt;
  if (i < nt) return std::string("kin_") + sys->type_name[i];
  i -= nt;
  if (i < nt) return std::string("un_") + sys->type_name[i];
  return "efp";
}

double err_of(const qmc2d_stats *st, int i) {
  if (st->iblk <= 1 || st->cml_norm == 0.0) return 0.0;
  const double m = st->cml_av[i] / st->cml_norm;
  return std::sqrt(std::fabs((st->cml2[i] / st->cml_norm - m * m) / (st->iblk - 1)));
}

// A list-directed REAL*8 the way this library writes it (readable by any
// Fortran list-directed read).
std::string ld(double v) {
  char buf[40];
  std::snprintf(buf, sizeof buf, "  %.17E", v);
  return buf;
}

bool write_coords(const std::string &path, const std::vector<double> &x, int nw, int N,
                  int first, int count) {
  std::FILE *f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  for (int w = 0; w < nw; w++)
    for (int p = first; p < first + count; p++)
      std::fprintf(f, "%s%s\n", ld(x[(size_t)2 * N * w + 2 * p]).c_str(),
                   ld(x[(size_t)2 * N * w + 2 * p + 1]).c_str());
  return std::fclose(f) == 0;
}

}  // namespace

extern "C" int qmc2d_stats_create(int n_props, qmc2d_stats **out) {
  if (!out || n_props <= 0) return fail(QMC2D_ERR_ARG, "qmc2d_stats_create: bad argument");
  qmc2d_stats *st = new qmc2d_stats;
  st->n_props = n_props;
  st->cml_av.assign(n_props, 0.0);
  st->cml2.assign(n_props, 0.0);
  *out = st;
  return QMC2D_OK;
}

extern "C" int qmc2d_stats_destroy(qmc2d_stats *st) {
  delete st;
  return QMC2D_OK;
}

extern "C" int qmc2d_stats_add_block(qmc2d_stats *st, const double *blk, double blk_norm) {
  if (!st || !blk) return fail(QMC2D_ERR_ARG, "qmc2d_stats_add_block: bad argument");
  if (!(blk_norm > 0.0)) return fail(QMC2D_ERR_ARG, "qmc2d_stats_add_block: blk_norm <= 0");
  for (int i = 0; i < st->n_props; i++) {
    st->cml_av[i] += blk[i];
    st->cml2[i] += blk[i] * blk[i] / blk_norm;
  }
  st->cml_norm += blk_norm;
  st->iblk++;
  return QMC2D_OK;
}

extern "C" int qmc2d_stats_get(const qmc2d_stats *st, double *mean, double *err,
                               double *cml_norm, int *iblk) {
  if (!st) return fail(QMC2D_ERR_ARG, "qmc2d_stats_get: bad argument");
  for (int i = 0; i < st->n_props; i++) {
    if (mean) mean[i] = st->cml_norm != 0.0 ? st->cml_av[i] / st->cml_norm : 0.0;
    if (err) err[i] = err_of(st, i);
  }
  if (cml_norm) *cml_norm = st->cml_norm;
  if (iblk) *iblk = st->iblk;
  return QMC2D_OK;
}

extern "C" int qmc2d_stats_report(const qmc2d_stats *st, const qmc2d_system *sys,
                                  const double *blk, double blk_norm, const char *who,
                                  char *buf, size_t len, size_t *needed) {
  if (!st || !sys || !blk || !who || st->n_props != sys->n_props)
    return fail(QMC2D_ERR_ARG, "qmc2d_stats_report: bad argument");
  std::string out = " ===>> " + std::string(who) + " block " + std::to_string(st->iblk) + "\n";
  for (int i = 0; i < sys->n_scalar_props; i++) {
    out += fe(blk[i] / blk_norm, 19, 11) + fe(st->cml_av[i] / st->cml_norm, 19, 11) +
           fe(err_of(st, i), 9, 2) + fe(blk_norm, 10, 3) + "  " + fa(scalar_name(sys, i), 20) +
           "\n";
  }
  if (needed) *needed = out.size() + 1;
  if (buf && len > 0) {
    const size_t n = out.size() < len - 1 ? out.size() : len - 1;
    std::memcpy(buf, out.data(), n);
    buf[n] = '\0';
    if (n < out.size()) return fail(QMC2D_ERR_LIMIT, "qmc2d_stats_report: buffer too small");
  }
  return QMC2D_OK;
}

extern "C" int qmc2d_stats_write_rhok(const qmc2d_stats *st, const qmc2d_system *sys,
                                      const double *blk, double blk_norm, const char *dir,
                                      const char *runid) {
  if (!st || !sys || !blk || !runid || st->n_props != sys->n_props)
    return fail(QMC2D_ERR_ARG, "qmc2d_stats_write_rhok: bad argument");
  int i = sys->jrhok;
  for (int t = 0; t < sys->ntypes; t++) {
    if (sys->irhok[t] == 0) continue;
    const std::string path =
        join(dir ? dir : "", std::string(runid) + ".rhok_" + sys->type_name[t]);
    std::FILE *f = std::fopen(path.c_str(), "w");
    if (!f) return fail(QMC2D_ERR_IO, "cannot write " + path);
    for (int j = 1; j <= 2 * sys->nk; j++, i++)
      std::fprintf(f, "%s%s%s%s %s%s\n", fe(blk[i] / blk_norm, 19, 11).c_str(),
                   fe(st->cml_av[i] / st->cml_norm, 19, 11).c_str(), fe(err_of(st, i), 9, 2).c_str(),
                   fe(blk_norm, 10, 3).c_str(), fa(" merea ", 7).c_str(), fi(j, 5).c_str());
    if (std::fclose(f) != 0) return fail(QMC2D_ERR_IO, "cannot write " + path);
  }
  return QMC2D_OK;
}

std::string q2d_itc_filename(const qmc2d_system *sys, int i, const std::string &runid);

extern "C" int qmc2d_stats_write_estimators(const qmc2d_stats *st, const qmc2d_system *sys,
                                           const qmc2d_rmc_estimators *est, const double *blk,
                                           double blk_norm, const char *dir, const char *runid) {
  if (!st || !sys || !est || !blk || !runid || st->n_props != est->nvalues || !(blk_norm > 0.0))
    return fail(QMC2D_ERR_ARG, "qmc2d_stats_write_estimators: bad argument");
  const std::string d = dir ? dir : "", rid = runid;
  // write_nonscalar_props: n lines from index i of the estimator vector
  auto put = [&](const std::string &name, int i, int n, const char *mode) {
    const std::string path = join(d, name);
    std::FILE *f = std::fopen(path.c_str(), mode);
    if (!f) return fail(QMC2D_ERR_IO, "cannot write " + path);
    for (int j = 1; j <= n; j++, i++)
      std::fprintf(f, "%s%s%s%s %s%s\n", fe(blk[i] / blk_norm, 19, 11).c_str(),
                   fe(st->cml_av[i] / st->cml_norm, 19, 11).c_str(),
                   fe(err_of(st, i), 9, 2).c_str(), fe(blk_norm, 10, 3).c_str(),
                   fa(" merea ", 7).c_str(), fi(j, 5).c_str());
    if (std::fclose(f) != 0) return fail(QMC2D_ERR_IO, "cannot write " + path);
    return (int)QMC2D_OK;
  };
  const int nb = est->ntau - 2 * est->ntauskip;
  int st2;
  int i = est->jmstar;
  for (int j = 0; j < est->nmstar; j++) {
    const int n = nb / est->mstar_tau_skip[j];
    if ((st2 = put(rid + ".mstar_" + sys->type_name[est->mstar_type[j]], i, n, "w"))) return st2;
    i += n;
  }
  // z_cmass: the reference leaves the unit open, so each block's lines follow
  // the previous block's (the first block starts the file)
  i = est->jcmass_z;
  for (int j = 0; j < est->ncmass; j++, i += 4)
    if ((st2 = put(rid + ".z_cmass_" + sys->type_name[est->cmass_type[j]], i, 4,
                   st->iblk <= 1 ? "w" : "a")))
      return st2;
  i = est->jcmass_d;
  for (int j = 0; j < est->ncmass; j++) {
    int n = 0;
    for (int k = 0; k < est->cmass_nskip; k++)
      n += (est->ntau - 2 * est->cmass_ntauskip[j][k]) / est->cmass_tau_skip[j];
    if ((st2 = put(rid + ".cmass_" + sys->type_name[est->cmass_type[j]], i, n, "w"))) return st2;
    i += n;
  }
  i = est->jitc;
  for (int j = 0; j < est->nitc; j++) {
    const int n = (nb / est->itc_tau_skip[j]) * est->itc_count[j];
    const std::string name = q2d_itc_filename(sys, j, rid);
    if (name.empty()) return fail(QMC2D_ERR_PARSE, "qmc2d_stats_write_estimators: itc record");
    if ((st2 = put(name, i, n, "w"))) return st2;
    i += n;
  }
  return QMC2D_OK;
}

extern "C" int qmc2d_write_conf(qmc2d_handle *h, const qmc2d_system *sys, const char *dir,
                                int rank) {
  if (!h || !sys || sys->nptot != h->N) return fail(QMC2D_ERR_ARG, "qmc2d_write_conf: bad argument");
  int nw = 0;
  int st = qmc2d_population_size(h, &nw);
  if (st) return st;
  std::vector<double> x((size_t)nw * 2 * sys->nptot);
  if (nw > 0 && (st = qmc2d_population_get(h, x.data(), nullptr, nullptr, nullptr, nullptr,
                                           nullptr)))
    return st;
  for (int t = 0; t < sys->ntypes; t++) {
    const std::string path =
        join(dir ? dir : "", std::string(sys->x_file[t]) + "." + std::to_string(rank));
    if (!write_coords(path, x, nw, sys->nptot, sys->ipfrst[t], sys->np[t]))
      return fail(QMC2D_ERR_IO, "cannot write " + path);
  }
  return QMC2D_OK;
}

extern "C" int qmc2d_restart_write(qmc2d_handle *h, const qmc2d_system *sys,
                                   const qmc2d_stats *st, int iblk, const char *who,
                                   const char *dir, const char *runid, int rank) {
  if (!h || !sys || !st || !who || !runid || st->n_props != sys->n_props)
    return fail(QMC2D_ERR_ARG, "qmc2d_restart_write: bad argument");
  const std::string w(who);
  if (w != "vmc" && w != "dmc" && w != "rmc")
    return fail(QMC2D_ERR_ARG, "qmc2d_restart_write: who must be vmc, dmc or rmc");
  const std::string d = dir ? dir : "";
  const std::string res = join(d, std::string(runid) + ".res");
  std::FILE *f = std::fopen(res.c_str(), "w");
  if (!f) return fail(QMC2D_ERR_IO, "cannot write " + res);
  std::fprintf(f, " %12d %s\n", iblk, who);
  std::fprintf(f, "%s\n", ld(st->cml_norm).c_str());
  for (int i = 0; i < st->n_props; i++)
    std::fprintf(f, "%s%s\n", ld(st->cml_av[i]).c_str(), ld(st->cml2[i]).c_str());
  // the random-stream state in place of the eight rannyu/rannyu2 seed words
  std::fprintf(f, " %12u %12u %12u %12u %12u %12d %12d %12d\n",
               (unsigned)(h->seed & 0xFFFFFFFFu), (unsigned)(h->seed >> 32),
               (unsigned)h->move_counter, (unsigned)h->gen_counter, (unsigned)h->rmc.step, 0, 0, 0);
  if (sys->ntheta != 0) std::fprintf(f, " %12d %12d\n", sys->ith, sys->jth);
  if (std::fclose(f) != 0) return fail(QMC2D_ERR_IO, "cannot write " + res);
  // configurations: every walker (vmc, dmc) or every reptile's path (rmc)
  std::vector<double> x;
  int nconf = 0;
  if (w == "rmc") {
    if (h->rmc.nrep <= 0) return fail(QMC2D_ERR_ARG, "qmc2d_restart_write: no reptiles");
    const int ntau = h->rmc.ntau;
    x.resize((size_t)h->rmc.nrep * ntau * 2 * sys->nptot);
    for (int r = 0; r < h->rmc.nrep; r++) {
      int s2 = qmc2d_rmc_get_path(h, r, x.data() + (size_t)r * ntau * 2 * sys->nptot, nullptr);
      if (s2) return s2;
    }
    nconf = h->rmc.nrep * ntau;
  } else {
    int s2 = qmc2d_population_size(h, &nconf);
    if (s2) return s2;
    x.resize((size_t)nconf * 2 * sys->nptot);
    if (nconf > 0 && (s2 = qmc2d_population_get(h, x.data(), nullptr, nullptr, nullptr, nullptr,
                                                nullptr)))
      return s2;
  }
  for (int t = 0; t < sys->ntypes; t++) {
    const std::string path =
        join(d, std::string(sys->x_file[t]) + ".res." + std::to_string(rank));
    if (!write_coords(path, x, nconf, sys->nptot, sys->ipfrst[t], sys->np[t]))
      return fail(QMC2D_ERR_IO, "cannot write " + path);
  }
  return QMC2D_OK;
}

namespace {

// restart(0) of who's .res file: the block, the cumulative sums into st and
// the stream state into the handle; then every stored configuration (all
// types' <x_file>.res.<rank> files) into *x, their count into *nconf.
int read_res(qmc2d_handle *h, const qmc2d_system *sys, qmc2d_stats *st, const char *dir,
             const char *runid, int rank, int *iblk, double *etrial, std::vector<double> *x,
             int *nconf_out) {
  const std::string d = dir ? dir : "";
  const std::string res = join(d, std::string(runid) + ".res");
  std::ifstream f(res);
  if (!f) return fail(QMC2D_ERR_IO, "cannot open " + res);
  std::string tag;
  int ib = 0;
  double norm = 0.0;
  if (!(f >> ib >> tag >> norm)) return fail(QMC2D_ERR_PARSE, "bad header in " + res);
  std::vector<double> av(st->n_props), c2(st->n_props);
  for (int i = 0; i < st->n_props; i++)
    if (!(f >> av[i] >> c2[i])) return fail(QMC2D_ERR_PARSE, "short property list in " + res);
  unsigned long long s[8];
  for (int i = 0; i < 8; i++)
    if (!(f >> s[i])) return fail(QMC2D_ERR_PARSE, "bad stream state in " + res);
  st->iblk = ib;
  st->cml_norm = norm;
  st->cml_av = av;
  st->cml2 = c2;
  h->seed = (s[0] & 0xFFFFFFFFull) | ((s[1] & 0xFFFFFFFFull) << 32);
  h->move_counter = (uint32_t)s[2];
  h->gen_counter = (uint32_t)s[3];
  h->rmc.step = (uint32_t)s[4];
  if (iblk) *iblk = ib;
  if (etrial) *etrial = norm != 0.0 ? av[QMC2D_JETOT] / norm : 0.0;
  // configurations: count the first type's lines, then read them all
  const std::string suffix = ".res." + std::to_string(rank);
  std::ifstream c(join(d, std::string(sys->x_file[0]) + suffix));
  if (!c) return fail(QMC2D_ERR_IO, "cannot open " + join(d, std::string(sys->x_file[0]) + suffix));
  long lines = 0;
  std::string line;
  while (std::getline(c, line))
    if (line.find_first_not_of(" \t\r") != std::string::npos) lines++;
  const int nconf = (int)(lines / sys->np[0]);
  if (nconf <= 0) return fail(QMC2D_ERR_PARSE, "no configurations in " + res);
  x->assign((size_t)nconf * 2 * sys->nptot, 0.0);
  int got = 0;
  int s2 = qmc2d_read_configs(sys, d.c_str(), suffix.c_str(), 0, nconf, x->data(), &got);
  if (s2) return s2;
  if (got != nconf) return fail(QMC2D_ERR_PARSE, "configuration files of unequal length");
  *nconf_out = nconf;
  return QMC2D_OK;
}

}  // namespace

extern "C" int qmc2d_restart_read(qmc2d_handle *h, const qmc2d_system *sys, qmc2d_stats *st,
                                  const char *who, const char *dir, const char *runid, int rank,
                                  int *iblk, double *etrial) {
  if (!h || !sys || !st || !who || !runid || st->n_props != sys->n_props)
    return fail(QMC2D_ERR_ARG, "qmc2d_restart_read: bad argument");
  const std::string w(who);
  if (w != "vmc" && w != "dmc")
    return fail(QMC2D_ERR_ARG, "qmc2d_restart_read: who must be vmc or dmc");
  std::vector<double> x;
  int nconf = 0;
  int s2 = read_res(h, sys, st, dir, runid, rank, iblk, etrial, &x, &nconf);
  if (s2) return s2;
  return qmc2d_population_set(h, nconf, x.data());
}

extern "C" int qmc2d_restart_read_rmc(qmc2d_handle *h, const qmc2d_system *sys,
                                      qmc2d_stats *st, const qmc2d_rmc_params *prm,
                                      const char *dir, const char *runid, int rank, int *iblk) {
  if (!h || !sys || !st || !prm || !runid || st->n_props != sys->n_props || prm->ntau < 2)
    return fail(QMC2D_ERR_ARG, "qmc2d_restart_read_rmc: bad argument");
  std::vector<double> x;
  int nconf = 0;
  int s2 = read_res(h, sys, st, dir, runid, rank, iblk, nullptr, &x, &nconf);
  if (s2) return s2;
  if (nconf % prm->ntau != 0)
    return fail(QMC2D_ERR_PARSE, "qmc2d_restart_read_rmc: " + std::to_string(nconf) +
                                     " stored configurations are not whole paths of " +
                                     std::to_string(prm->ntau) + " beads");
  const uint32_t step = h->rmc.step;  // qmc2d_rmc_init starts the reptation counter at 0
  if ((s2 = qmc2d_rmc_init(h, nconf / prm->ntau, prm, x.data()))) return s2;
  h->rmc.step = step;
  return QMC2D_OK;
}
