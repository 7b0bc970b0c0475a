/*
 * oracle_input.c - the oracle's own reader of a reference run directory
 * (TEST INFRASTRUCTURE ONLY). It fills a qmc2d_system (the data layout of
 * include/qmc2d.h) from <runid>.sy, the tables and the k-vector file, so
 * that the oracle and the product library read every deck independently: a
 * misread keyword, table trailer, k list or v0 on either side shows up as a
 * parity failure instead of hitting both sides alike.
 *
 * Restated from reptation.f:
 *   readwords  :4790-4842  80-column records, blank-separated words of at
 *                          most 48 characters, '\' continues on the next
 *                          record;
 *   input      :12-515     the keyword pass (the walker-path keywords only;
 *                          every other keyword is refused), :516-637 the
 *                          particle counts and the property layout, :674-708
 *                          the Gamma-point orbital wave vectors;
 *   t_read     :4689-4738  spline tables, deduplicated by file name, the
 *                          shared knot spacing and the k-space trailer;
 *   kread      :4740-4769  the k vectors;
 *   twistg     :9818-9861  twisted wave vectors, ordered by SORTTF (:9514);
 *   read_conf  :2452-2491  configuration files.
 * Written in plain C with its own list-directed number reader; it shares no
 * code with the product's reader (2degas_b200/csrc/input.cpp, system.cpp).
 */
#include "qmc2d_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define REC_LEN 80   /* character*80 record */
#define WORD_LEN 48  /* character*48 word */
#define MAX_WORDS 32 /* mword */

/* ------------------------------------------------------------ file text */

typedef struct text {
  char **line;
  int n, pos;
} text;

static void text_free(text *t) {
  for (int i = 0; i < t->n; i++) free(t->line[i]);
  free(t->line);
  t->line = NULL;
  t->n = t->pos = 0;
}

static int text_load(const char *path, text *t) {
  memset(t, 0, sizeof *t);
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  int cap = 0;
  char *buf = NULL;
  size_t bcap = 0;
  ssize_t len;
  while ((len = getline(&buf, &bcap, f)) >= 0) {
    while (len > 0 && (buf[len - 1] == '\n' || buf[len - 1] == '\r')) buf[--len] = 0;
    if (t->n == cap) {
      cap = cap ? 2 * cap : 256;
      t->line = realloc(t->line, sizeof(char *) * cap);
    }
    t->line[t->n++] = strdup(buf);
  }
  free(buf);
  fclose(f);
  return 0;
}

static void path_join(char *out, size_t n, const char *dir, const char *name) {
  if (!dir || !*dir || name[0] == '/')
    snprintf(out, n, "%s", name);
  else
    snprintf(out, n, "%s/%s", dir, name);
}

/* A Fortran list-directed real: digits with an optional d/D/e/E exponent,
 * ended by a blank, a comma or the end of the record. */
static int list_real(const char *s, double *v) {
  char tmp[64];
  size_t k = 0;
  while (s[k] && s[k] != ' ' && s[k] != ',' && s[k] != '\t' && k < sizeof tmp - 1) {
    tmp[k] = (s[k] == 'd' || s[k] == 'D') ? 'e' : s[k];
    k++;
  }
  tmp[k] = 0;
  if (k == 0) return -1;
  char *end = NULL;
  *v = strtod(tmp, &end);
  return (end && *end == 0) ? 0 : -1;
}

static int list_int(const char *s, int *v) {
  double d;
  if (list_real(s, &d)) return -1;
  *v = (int)d;
  return 0;
}

/* List-directed READ of n reals: starts on the next record, takes values
 * across as many records as needed, drops the rest of the last record. */
static int read_reals(text *t, int n, double *out) {
  int got = 0;
  while (got < n) {
    if (t->pos >= t->n) return -1;
    const char *p = t->line[t->pos++];
    while (*p && got < n) {
      while (*p == ' ' || *p == '\t' || *p == ',') p++;
      if (!*p) break;
      if (list_real(p, &out[got])) return -1;
      got++;
      while (*p && *p != ' ' && *p != '\t' && *p != ',') p++;
    }
  }
  return 0;
}

/* List-directed READ of one character item: the first word of the next
 * non-blank record. */
static int read_word(text *t, char *w, size_t n) {
  while (t->pos < t->n) {
    const char *p = t->line[t->pos++];
    while (*p == ' ' || *p == '\t') p++;
    if (!*p) continue;
    size_t k = 0;
    while (p[k] && p[k] != ' ' && p[k] != '\t' && p[k] != ',' && k < n - 1) {
      w[k] = p[k];
      k++;
    }
    w[k] = 0;
    return 0;
  }
  return -1;
}

/* readwords (reptation.f:4790-4842): the words of the next keyword record.
 * Returns the number of words, or -1 at end of file. */
static int readwords(text *t, char word[MAX_WORDS][WORD_LEN + 1]) {
  int nw = 0;
  for (int i = 0; i < MAX_WORDS; i++) word[i][0] = 0;
  for (;;) {
    if (t->pos >= t->n) return nw ? nw : -1;
    char rec[REC_LEN + 1];
    snprintf(rec, sizeof rec, "%s", t->line[t->pos++]);
    size_t L = strlen(rec);
    int cont = 0;
    for (size_t i = 0; i < L; i++) {
      if (rec[i] == '\\') {
        cont = 1;
        break;
      }
      if (rec[i] == ' ') continue;
      size_t k = 0;
      char w[WORD_LEN + 1];
      while (i < L && rec[i] != ' ') {
        if (k < WORD_LEN) w[k++] = rec[i];
        i++;
      }
      w[k] = 0;
      if (nw < MAX_WORDS) snprintf(word[nw++], WORD_LEN + 1, "%s", w);
    }
    if (!cont) return nw;
  }
}

/* ------------------------------------------------------------ t_read */

/* t_read (reptation.f:4689-4738). Returns the 0-based table index, or a
 * negative status. */
static int t_read(qmc2d_system *s, const char *dir, const char *file) {
  for (int i = 0; i < s->ntables; i++)
    if (strcmp(s->tables[i].name, file) == 0) return i;
  if (s->ntables >= QMC2D_MAX_TABLES) return -QMC2D_ERR_LIMIT;
  char path[1024];
  path_join(path, sizeof path, dir, file);
  text t;
  if (text_load(path, &t)) return -QMC2D_ERR_IO;
  qmc2d_table *tb = &s->tables[s->ntables];
  memset(tb, 0, sizeof *tb);
  snprintf(tb->name, sizeof tb->name, "%s", file);
  double hdr[2];
  int st = 0;
  if (read_reals(&t, 2, hdr)) {
    st = -QMC2D_ERR_PARSE;
    goto out;
  }
  tb->ngrid = (int)hdr[0];
  if (tb->ngrid < 1) {
    st = -QMC2D_ERR_PARSE;
    goto out;
  }
  s->drt = hdr[1];
  tb->ut = calloc((size_t)4 * (tb->ngrid + 1), sizeof(double));
  for (int it = 0; it <= tb->ngrid; it++)
    if (read_reals(&t, 4, tb->ut + 4 * it)) {
      st = -QMC2D_ERR_PARSE;
      goto out;
    }
  {
    char name[WORD_LEN + 1];
    double npar;
    /* routine name, the parameter count, the parameter records */
    if (read_word(&t, name, sizeof name) == 0 && read_reals(&t, 1, &npar) == 0) {
      t.pos += (int)npar;
      char kw[WORD_LEN + 1];
      if (read_word(&t, kw, sizeof kw) == 0 && strcmp(kw, "kspace") == 0) {
        double nk;
        if (read_reals(&t, 1, &nk)) {
          st = -QMC2D_ERR_PARSE;
          goto out;
        }
        tb->nk_ewald = (int)nk;
        tb->vk = calloc((size_t)tb->nk_ewald + 1, sizeof(double));
        for (int k = 0; k <= tb->nk_ewald; k++) /* v_k, k = 1..nk, then v_k0 */
          if (read_reals(&t, 1, &tb->vk[k])) {
            st = -QMC2D_ERR_PARSE;
            goto out;
          }
      }
    }
  }
  s->drti = 1.0 / s->drt;
  s->drti2 = 2.0 * s->drti * s->drti;
  s->ntables++;
out:
  if (st) {
    free(tb->ut);
    free(tb->vk);
    memset(tb, 0, sizeof *tb);
  }
  text_free(&t);
  return st ? st : s->ntables - 1;
}

/* kread (reptation.f:4740-4769): k vectors until the end of the file. */
static int kread(qmc2d_system *s, const char *dir, const char *file) {
  char path[1024];
  path_join(path, sizeof path, dir, file);
  text t;
  if (text_load(path, &t)) return QMC2D_ERR_IO;
  free(s->kvec);
  s->kvec = calloc(2 * (size_t)QMC2D_MAX_NK, sizeof(double));
  int ik = 0;
  while (ik < QMC2D_MAX_NK && read_reals(&t, 2, s->kvec + 2 * ik) == 0) ik++;
  s->nk = ik;
  text_free(&t);
  return QMC2D_OK;
}

/* ------------------------------------------------- orbital wave vectors */

/* SORTTF (reptation.f:9514-9557): heapsort of the 1-based index vector idx
 * by a(idx(.)), ascending; a is 1-based (a[1..n]). */
static void sorttf(int n1, const double *a, int *idx) {
  int n = n1;
  for (int i1 = 2; i1 <= n; i1++) { /* build the heap */
    int i3 = i1, i33 = idx[i3];
    double ai = a[i33];
    while (i3 / 2 > 0) {
      int i2 = i3 / 2, i22 = idx[i2];
      if (ai <= a[i22]) break;
      idx[i3] = i22;
      i3 = i2;
    }
    idx[i3] = i33;
  }
  for (;;) { /* pop the largest to the end */
    int i3 = idx[n];
    idx[n] = idx[1];
    double ai = a[i3];
    n--;
    if (n - 1 <= 0) {
      idx[1] = i3;
      return;
    }
    int i1 = 1;
    for (;;) {
      int i2 = i1 + i1, i22 = 0;
      if (i2 <= n) i22 = idx[i2];
      if (i2 > n) break;
      if (i2 < n) {
        int i222 = idx[i2 + 1];
        if (a[i22] - a[i222] < 0) {
          i2 = i2 + 1;
          i22 = i222;
        }
      }
      if (ai - a[i22] < 0) {
        idx[i1] = i22;
        i1 = i2;
      } else {
        break;
      }
    }
    idx[i1] = i3;
  }
}

int oracle_system_set_twist(qmc2d_system *s, int ith, int jth) {
  if (!s || s->nk <= 0 || ith < 0 || jth < 0 || (ith == 0) != (jth == 0) ||
      (ith > 0 && (s->ntheta <= 0 || ith > s->ntheta || jth > s->ntheta)))
    return QMC2D_ERR_ARG;
  const int ng = 2 * s->nk + 1;
  free(s->gvec);
  s->gvec = calloc(2 * (size_t)ng, sizeof(double));
  s->ngvec = ng;
  s->ith = ith;
  s->jth = jth;
  if (ith == 0) { /* Gamma point (input, reptation.f:680-698): 0, then +-k */
    for (int i = 0; i < s->nk; i++)
      for (int d = 0; d < 2; d++) {
        s->gvec[2 * (2 * i + 1) + d] = s->kvec[2 * i + d];
        s->gvec[2 * (2 * i + 2) + d] = -s->kvec[2 * i + d];
      }
    return QMC2D_OK;
  }
  /* twistg (reptation.f:9818-9861), 1-based arrays as in the Fortran */
  const double pi = acos(-1.0);
  double theta[2] = {ith * 2.0 * pi * s->eli[0] / s->ntheta,
                     jth * 2.0 * pi * s->eli[1] / s->ntheta};
  double *gv = calloc(2 * (size_t)(ng + 1), sizeof(double));
  double *gn = calloc((size_t)ng + 1, sizeof(double));
  int *ig = calloc((size_t)ng + 1, sizeof(int));
  gn[1] = 0.0;
  for (int d = 0; d < 2; d++) {
    gv[2 * 1 + d] = theta[d];
    gn[1] += theta[d] * theta[d];
  }
  ig[1] = 1;
  for (int k = s->nk; k >= 1; k--) {
    gn[2 * k + 1] = gn[2 * k] = 0.0;
    for (int d = 0; d < 2; d++) {
      gv[2 * (2 * k + 1) + d] = -s->kvec[2 * (k - 1) + d] + theta[d];
      gv[2 * (2 * k) + d] = s->kvec[2 * (k - 1) + d] + theta[d];
      gn[2 * k + 1] += gv[2 * (2 * k + 1) + d] * gv[2 * (2 * k + 1) + d];
      gn[2 * k] += gv[2 * (2 * k) + d] * gv[2 * (2 * k) + d];
    }
    ig[2 * k] = 2 * k;
    ig[2 * k + 1] = 2 * k + 1;
  }
  sorttf(ng, gn, ig);
  for (int k = 1; k <= ng; k++)
    for (int d = 0; d < 2; d++) s->gvec[2 * (k - 1) + d] = gv[2 * ig[k] + d];
  free(gv);
  free(gn);
  free(ig);
  return QMC2D_OK;
}

/* ------------------------------------------------------------ input */

void oracle_system_free(qmc2d_system *s) {
  if (!s) return;
  for (int i = 0; i < s->ntables; i++) {
    free(s->tables[i].ut);
    free(s->tables[i].vk);
  }
  free(s->kvec);
  free(s->gvec);
  free(s);
}

static int type_of(const qmc2d_system *s, const char *name) {
  for (int i = 0; i < s->ntypes; i++)
    if (strcmp(s->type_name[i], name) == 0) return i;
  return -1;
}

/* The words after the keyword, one blank apart (mstar/cmass/itc records,
 * reptation.f:210-224, parsed again when reptation starts). */
static int keep_record(char rec[QMC2D_RECORD_LEN], char word[MAX_WORDS][WORD_LEN + 1], int nw) {
  size_t k = 0;
  rec[0] = 0;
  for (int i = 1; i < nw; i++) {
    size_t l = strlen(word[i]);
    if (k + l + 2 > QMC2D_RECORD_LEN) return QMC2D_ERR_LIMIT;
    if (i > 1) rec[k++] = ' ';
    memcpy(rec + k, word[i], l);
    k += l;
    rec[k] = 0;
  }
  return QMC2D_OK;
}

static int keyword(qmc2d_system *s, const char *dir, char w[MAX_WORDS][WORD_LEN + 1], int nw,
                   int *ended) {
#define NEED(n) \
  if (nw < (n)) return QMC2D_ERR_PARSE
#define INT(i, v) \
  if (list_int(w[i], &(v))) return QMC2D_ERR_PARSE
#define REAL(i, v) \
  if (list_real(w[i], &(v))) return QMC2D_ERR_PARSE
  const char *k = w[0];
  if (!strcmp(k, "end")) {
    *ended = 1;
  } else if (!strcmp(k, "ndim")) {
    NEED(2);
    INT(1, s->ndim);
  } else if (!strcmp(k, "v0")) {
    NEED(2);
    REAL(1, s->v0);
  } else if (!strcmp(k, "adrift")) {
    NEED(2);
    REAL(1, s->adrift);
  } else if (!strcmp(k, "gstorto")) {
    NEED(2);
    INT(1, s->gstorto);
  } else if (!strcmp(k, "wpiu")) {
    NEED(2);
    INT(1, s->wpiu);
  } else if (!strcmp(k, "nodalaction")) {
    NEED(2);
    INT(1, s->nodalaction);
  } else if (!strcmp(k, "rejection")) {
    NEED(2);
    INT(1, s->rejection);
  } else if (!strcmp(k, "fullprop")) {
    /* read by the energy-derivative estimators only */
  } else if (!strcmp(k, "ecut")) {
    NEED(2);
    INT(1, s->ecut);
    if (s->ecut != 0) {
      NEED(3);
      REAL(2, s->value_ecut);
    }
  } else if (!strcmp(k, "seed")) {
    NEED(5);
    for (int i = 0; i < 4; i++) INT(i + 1, s->seed[i]);
  } else if (!strcmp(k, "pbc")) {
    NEED(3);
    for (int i = 0; i < 2; i++) {
      REAL(i + 1, s->el[i]);
      s->eli[i] = 1.0 / s->el[i];
    }
  } else if (!strcmp(k, "kspace")) {
    NEED(2);
    return kread(s, dir, w[1]);
  } else if (!strcmp(k, "rhok")) {
    NEED(2);
    int it = type_of(s, w[1]);
    if (it < 0) return QMC2D_ERR_PARSE;
    s->irhok[it] = ++s->nrhok;
  } else if (!strcmp(k, "mstar") || !strcmp(k, "cmass") || !strcmp(k, "itc")) {
    int *n = k[0] == 'm' ? &s->nmstar : k[0] == 'c' ? &s->ncmass : &s->nitc;
    char(*rec)[QMC2D_RECORD_LEN] =
        k[0] == 'm' ? s->mstar_record : k[0] == 'c' ? s->cmass_record : s->itc_record;
    if (*n >= QMC2D_MAX_EST) return QMC2D_ERR_LIMIT;
    int st = keep_record(rec[*n], w, nw);
    if (st) return st;
    (*n)++;
  } else if (!strcmp(k, "type")) {
    NEED(5);
    if (s->ntypes >= QMC2D_MAX_TYPES) return QMC2D_ERR_LIMIT;
    int it = s->ntypes++;
    snprintf(s->type_name[it], QMC2D_NAME_LEN, "%s", w[1]);
    INT(2, s->np[it]);
    REAL(3, s->hbs2m[it]);
    snprintf(s->x_file[it], QMC2D_NAME_LEN, "%s", w[4]);
  } else if (!strcmp(k, "v2") || !strcmp(k, "u2") || !strcmp(k, "u3") ||
             !strcmp(k, "backflow")) {
    const int bf = !strcmp(k, "backflow");
    NEED(bf ? 5 : 4);
    int it = type_of(s, w[1]), jt = type_of(s, w[2]);
    if (it < 0 || jt < 0) return QMC2D_ERR_PARSE;
    if (bf) INT(3, s->ibckf);
    int i = t_read(s, dir, w[bf ? 4 : 3]);
    if (i < 0) return -i;
    int(*tab)[QMC2D_MAX_TYPES] = !strcmp(k, "v2")   ? s->iv2
                                 : !strcmp(k, "u2") ? s->iu2
                                 : !strcmp(k, "u3") ? s->iu3
                                                    : s->iub;
    tab[it][jt] = tab[jt][it] = i;
    if (!strcmp(k, "v2")) {
      NEED(6);
      REAL(4, s->tables[i].tail);
      INT(5, s->tables[i].iexp);
    }
  } else if (!strcmp(k, "ntwists")) {
    NEED(2);
    INT(1, s->ntheta);
  } else {
    /* sites, vext, vps, plane-wave, lcao, inc, der, gofr, ... are not
     * restated here; unknown words stop the reference (:511-514) */
    return QMC2D_ERR_UNSUPPORTED;
  }
  return QMC2D_OK;
#undef NEED
#undef INT
#undef REAL
}

int oracle_system_read(const char *dir, const char *runid, qmc2d_system **out) {
  if (!runid || !out) return QMC2D_ERR_ARG;
  *out = NULL;
  qmc2d_system *s = calloc(1, sizeof *s);
  /* defaults of input (reptation.f:24, 40-130) */
  s->ndim = 2;
  s->rejection = 1;
  s->seed[3] = 1;
  s->ref_underflow_return = 1;
  for (int a = 0; a < QMC2D_MAX_TYPES; a++)
    for (int b = 0; b < QMC2D_MAX_TYPES; b++)
      s->iu2[a][b] = s->iu3[a][b] = s->iub[a][b] = s->iv2[a][b] = -1;
  char path[1024];
  /* the 'seed' file (reptation.f:31-33): four integers, if present */
  path_join(path, sizeof path, dir, "seed");
  {
    text t;
    if (text_load(path, &t) == 0) {
      double v[4];
      if (read_reals(&t, 4, v) == 0)
        for (int i = 0; i < 4; i++) s->seed[i] = (int)v[i];
      text_free(&t);
    }
  }
  char name[256];
  snprintf(name, sizeof name, "%s.sy", runid);
  path_join(path, sizeof path, dir, name);
  text t;
  if (text_load(path, &t)) {
    oracle_system_free(s);
    return QMC2D_ERR_IO;
  }
  int st = QMC2D_OK, ended = 0;
  char w[MAX_WORDS][WORD_LEN + 1];
  while (!ended && st == QMC2D_OK) {
    int nw = readwords(&t, w);
    if (nw < 0) break;                  /* end of file ends the pass */
    if (nw == 0) st = QMC2D_ERR_PARSE;  /* blank record: not a keyword */
    else st = keyword(s, dir, w, nw, &ended);
  }
  text_free(&t);
  /* particle counts (reptation.f:516-528); every type here moves */
  if (st == QMC2D_OK && (s->ndim != 2 || s->ntypes < 1)) st = QMC2D_ERR_UNSUPPORTED;
  for (int it = 0; st == QMC2D_OK && it < s->ntypes; it++) {
    if (s->hbs2m[it] == 0.0) st = QMC2D_ERR_UNSUPPORTED;
    s->ipfrst[it] = s->nptot;
    s->nptot += s->np[it];
    s->npnorm += s->np[it];
  }
  if (st == QMC2D_OK && (s->nptot > QMC2D_MAX_NP || s->el[0] <= 0.0)) st = QMC2D_ERR_LIMIT;
  /* property layout (reptation.f:577-637) */
  s->n_scalar_props = QMC2D_NSCALAR(s->ntypes);
  s->jrhok = s->n_scalar_props;
  s->n_props = s->n_scalar_props + 2 * s->nk * s->nrhok;
  /* orbital wave vectors: only the backflow determinant uses them. input
   * builds them at Gamma when ibckf != 0 (:674-708); with ntwists the run
   * starts at tabc's first twist (1,1) */
  if (st == QMC2D_OK && s->iub[0][0] >= 0) {
    if (s->nk <= 0) st = QMC2D_ERR_PARSE;
    else if (s->ntheta == 0 && s->ibckf == 0) st = QMC2D_ERR_UNSUPPORTED;
    else st = oracle_system_set_twist(s, s->ntheta ? 1 : 0, s->ntheta ? 1 : 0);
  }
  if (st != QMC2D_OK) {
    oracle_system_free(s);
    return st;
  }
  *out = s;
  return QMC2D_OK;
}

/* read_conf (reptation.f:2452-2491): configuration `first` onwards from the
 * per-type files <x_file><suffix>, np(type) coordinate records each. */
int oracle_read_configs(const qmc2d_system *s, const char *dir, const char *suffix, int first,
                        int count, double *x, int *nread) {
  if (!s || !x || first < 0 || count < 0) return QMC2D_ERR_ARG;
  const int N = s->nptot;
  int got = count;
  for (int it = 0; it < s->ntypes; it++) {
    char name[256], path[1024];
    snprintf(name, sizeof name, "%s%s", s->x_file[it], suffix ? suffix : "");
    path_join(path, sizeof path, dir, name);
    text t;
    if (text_load(path, &t)) return QMC2D_ERR_IO;
    double skip[2];
    for (long k = 0; k < (long)first * s->np[it]; k++)
      if (read_reals(&t, 2, skip)) break;
    int c = 0;
    for (; c < got; c++) {
      int ok = 1;
      for (int ip = 0; ip < s->np[it] && ok; ip++)
        ok = read_reals(&t, 2, x + (size_t)2 * N * c + 2 * (s->ipfrst[it] + ip)) == 0;
      if (!ok) break;
    }
    if (c < got) got = c;
    text_free(&t);
  }
  if (nread) *nread = got;
  return QMC2D_OK;
}

void oracle_system_sizes(const qmc2d_system *s, int *nptot, int *ntypes, int *n_props) {
  *nptot = s->nptot;
  *ntypes = s->ntypes;
  *n_props = s->n_props;
}
