// estimators.cpp - setup of the reptation path estimators: mstar_setup,
// cmass_setup and itc_setup (reptation.f:1378-1553) on the deck's 'mstar',
// 'cmass' and 'itc' records, host side. The device evaluation is in rmc.cu.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../../include/qmc2d.h"
#include "common.h"

namespace {

int efail(int code, const std::string &msg) {
  q2d::set_error("qmc2d_rmc_estimators_setup: " + msg);
  return code;
}

std::vector<std::string> words(const char *rec) {
  std::istringstream in(rec);
  std::vector<std::string> w;
  std::string t;
  while (in >> t) w.push_back(t);
  return w;
}

bool to_int(const std::string &s, int *v) {
  char *end = nullptr;
  long x = std::strtol(s.c_str(), &end, 10);
  if (end == s.c_str() || *end != '\0') return false;
  *v = (int)x;
  return true;
}

int type_index(const qmc2d_system *sys, const std::string &n) {
  for (int t = 0; t < sys->ntypes; t++)
    if (n == sys->type_name[t]) return t;
  return -1;
}

// The names of the stored bead properties with their start and count (the
// name table of input, reptation.f:577-628; rhok, :630-639).
std::map<std::string, std::pair<int, int>> prop_names(const qmc2d_system *sys) {
  std::map<std::string, std::pair<int, int>> m;
  const int nt = sys->ntypes;
  m["elocal"] = {QMC2D_JETOT, 1};
  m["acc.rate"] = {QMC2D_JACC, 1};
  m["epot"] = {QMC2D_JPOT0, 1};
  m["ekin"] = {QMC2D_JKIN0, 1};
  m["e2"] = {QMC2D_JE2, 1};
  m["gg"] = {QMC2D_JGG, 1};
  for (int t = 0; t < nt; t++) {
    const std::string tn = sys->type_name[t];
    m["pot_" + tn] = {QMC2D_JPOT(nt, t), 1};
    m["kin_" + tn] = {QMC2D_JKIN(nt, t), 1};
    m["un_" + tn] = {QMC2D_JUN(nt, t), 1};
  }
  m["efp"] = {QMC2D_JEFP(nt), 1};
  for (int t = 0; t < nt; t++)
    if (sys->irhok[t] > 0)
      m["rhok_" + std::string(sys->type_name[t])] = {
          sys->jrhok + 2 * sys->nk * (sys->irhok[t] - 1), 2 * sys->nk};
  return m;
}

int complex_flag(const std::string &s) {
  return s == "complex" ? 1 : s == "conjg" ? -1 : 0;
}

}  // namespace

// The file name itc_setup builds for itc record i: runid, then the first
// factor's names joined by '.', '+', then the second's by '_', '+'
// (reptation.f:1474-1530); empty if the record does not parse.
std::string q2d_itc_filename(const qmc2d_system *sys, int i, const std::string &runid) {
  const auto names = prop_names(sys);
  auto w = words(sys->itc_record[i]);
  std::string f = runid;
  size_t iw = 0;
  for (int sidx = 0; sidx < 2; sidx++) {
    int add = 0;
    if (iw >= w.size() || !to_int(w[iw++], &add)) return "";
    for (int j = 0; j < add; j++) {
      if (iw >= w.size() || names.find(w[iw]) == names.end()) return "";
      f += (j == 0 ? (sidx == 0 ? "." : "_") : "+") + w[iw++];
    }
    if (iw < w.size() && complex_flag(w[iw]) != 0) iw++;
  }
  return f;
}

extern "C" int qmc2d_rmc_estimators_setup(const qmc2d_system *sys, int ntau, int ntauskip,
                                          qmc2d_rmc_estimators *est) {
  if (!sys || !est || ntau < 2 || ntauskip < 0 || ntau - 2 * ntauskip < 1)
    return efail(QMC2D_ERR_ARG, "bad argument");
  qmc2d_rmc_estimators e{};
  e.ntau = ntau;
  e.ntauskip = ntauskip;
  const int nb = ntau - 2 * ntauskip;
  // cmass_setup: <type> <tau skip> <n skips> [skip ...] (n = 1: ntauskip)
  e.ncmass = sys->ncmass;
  e.cmass_nskip = 0;
  for (int i = 0; i < sys->ncmass; i++) {
    auto w = words(sys->cmass_record[i]);
    int n = 0;
    if (w.size() < 3 || (e.cmass_type[i] = type_index(sys, w[0])) < 0 ||
        !to_int(w[1], &e.cmass_tau_skip[i]) || !to_int(w[2], &n) || n < 1 ||
        n > QMC2D_MAX_CMSKIP || e.cmass_tau_skip[i] < 1)
      return efail(QMC2D_ERR_PARSE, std::string("cmass record '") + sys->cmass_record[i] + "'");
    // the reference keeps one count for every record (ncm_ntauskip)
    if (i > 0 && n != e.cmass_nskip)
      return efail(QMC2D_ERR_UNSUPPORTED, "cmass records with different numbers of bead skips");
    e.cmass_nskip = n;
    if (n == 1) {
      e.cmass_ntauskip[i][0] = ntauskip;
    } else {
      if ((int)w.size() < 3 + n)
        return efail(QMC2D_ERR_PARSE, std::string("cmass record '") + sys->cmass_record[i] + "'");
      for (int k = 0; k < n; k++)
        if (!to_int(w[3 + k], &e.cmass_ntauskip[i][k]) || e.cmass_ntauskip[i][k] < 0 ||
            ntau - 2 * e.cmass_ntauskip[i][k] < e.cmass_tau_skip[i])
          return efail(QMC2D_ERR_PARSE, std::string("cmass skip in '") + sys->cmass_record[i] + "'");
    }
    if (nb < e.cmass_tau_skip[i]) return efail(QMC2D_ERR_PARSE, "cmass tau skip beyond the path");
  }
  // mstar_setup: <type> <tau skip>
  e.nmstar = sys->nmstar;
  for (int i = 0; i < sys->nmstar; i++) {
    auto w = words(sys->mstar_record[i]);
    if (w.size() < 2 || (e.mstar_type[i] = type_index(sys, w[0])) < 0 ||
        !to_int(w[1], &e.mstar_tau_skip[i]) || e.mstar_tau_skip[i] < 1 ||
        e.mstar_tau_skip[i] > nb)
      return efail(QMC2D_ERR_PARSE, std::string("mstar record '") + sys->mstar_record[i] + "'");
  }
  // itc_setup: <n> <name>... [complex|conjg] <n> <name>... [complex|conjg] <tau skip>
  const auto names = prop_names(sys);
  e.nitc = sys->nitc;
  for (int i = 0; i < sys->nitc; i++) {
    auto w = words(sys->itc_record[i]);
    const std::string rec = sys->itc_record[i];
    size_t iw = 0;
    auto next = [&](std::string *s) {
      if (iw >= w.size()) return false;
      *s = w[iw++];
      return true;
    };
    std::string t;
    auto side = [&](int *add, int(*start), int *count, int *cflag) {
      if (!next(&t) || !to_int(t, add) || *add < 1 || *add > QMC2D_MAX_ADD) return false;
      for (int j = 0; j < *add; j++) {
        if (!next(&t)) return false;
        auto it = names.find(t);
        if (it == names.end()) return false;
        start[j] = it->second.first;
        if (count) *count = it->second.second;
      }
      if (!next(&t)) return false;
      *cflag = complex_flag(t);
      if (*cflag == 0) iw--;  // not a flag: the next field
      return true;
    };
    if (!side(&e.itc_add[i], e.itc_start[i], &e.itc_count[i], &e.itc_complex[i]) ||
        !side(&e.jtc_add[i], e.jtc_start[i], nullptr, &e.jtc_complex[i]) || !next(&t) ||
        !to_int(t, &e.itc_tau_skip[i]) || e.itc_tau_skip[i] < 1 || e.itc_tau_skip[i] > nb)
      return efail(QMC2D_ERR_PARSE, "itc record '" + rec + "' (names: stored bead properties)");
    if (e.itc_complex[i] != 0 && e.itc_count[i] % 2 != 0)
      return efail(QMC2D_ERR_PARSE, "itc record '" + rec + "': complex needs pairs");
  }
  // offsets: cmass z, cmass diffusion, mstar, itc (the reference's order)
  int off = 0;
  e.jcmass_z = off;
  off += 2 * 2 * e.ncmass;
  e.jcmass_d = off;
  for (int i = 0; i < e.ncmass; i++)
    for (int k = 0; k < e.cmass_nskip; k++)
      off += (ntau - 2 * e.cmass_ntauskip[i][k]) / e.cmass_tau_skip[i];
  e.jmstar = off;
  for (int i = 0; i < e.nmstar; i++) off += nb / e.mstar_tau_skip[i];
  e.jitc = off;
  for (int i = 0; i < e.nitc; i++) off += (nb / e.itc_tau_skip[i]) * e.itc_count[i];
  e.nvalues = off;
  *est = e;
  return QMC2D_OK;
}
