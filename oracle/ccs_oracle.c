/*
 * ccs_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 CPU restatement of the reference's trajectory-method CCS path
 * (cces-cepid/massccs).  Written from the reference's mathematics, in plain C,
 * keeping the reference's operation order so that its shipped logs replay.
 * Citations are file:line within the reference project (src/...).
 *
 * Where the reference has undefined behaviour the oracle picks the
 * well-defined reading and says so at the spot:
 *   - all-pairs dipole routines read uninitialised accumulators
 *     (Force.cpp:517-522, 836-889, 1658-1663): zero-initialised here;
 *   - coulomb_LC's bounds test is always false (Force.cpp:753): an out-of-grid
 *     site gets zero force here, as every other *_LC routine does.
 */
#define _GNU_SOURCE
#include "ccs_oracle.h"

#include <ctype.h>
#include <math.h>
#include <omp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ---- constants: src/headers/Constants.h:22-83 ---------------------------- */
#define AMU_TO_KG (1.66053904E-27)
#define BOLTZMANN_K (1.38064E-23)
#define ANG_TO_M (1.0E-10)
#define FS_TO_S (1.0E-15)
#define KCALMOLANGAMU_TO_ANGFS2 (1.0 / 48.88821291 / 48.88821291)
#define ALPHA_TO_KCAL_MOL (331.842254885)
#define OMEGA_TO_FS_INV (2.45400505E8)
#define KCOUL (332.06348078020324)
#define AMUANGFS2_TO_KCAL_MOL (2390.07)
#define PI_D 3.14159265358979323846

/* ---- small helpers ------------------------------------------------------- */
static void set_err(char *err, int errlen, const char *fmt, ...) {
  if (!err || errlen <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(err, (size_t)errlen, fmt, ap);
  va_end(ap);
}
static double wall_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
/* Math::dotProduct / vecModulus accumulate left to right from 0 (Math.h:58-74). */
static double dot3(const double *a, const double *b) {
  double r = 0.0;
  r += a[0] * b[0];
  r += a[1] * b[1];
  r += a[2] * b[2];
  return r;
}
static double mod3(const double *a) { return sqrt(dot3(a, a)); }
static void cross3(const double *a, const double *b, double *o) { /* Math.h:77-91 */
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

/* ---- MT19937 (Matsumoto & Nishimura 1998), as std::mt19937 ---------------- */
typedef struct {
  uint32_t s[624];
  int i;
} mt_t;
static void mt_seed(mt_t *m, uint32_t seed) {
  m->s[0] = seed;
  for (int k = 1; k < 624; k++)
    m->s[k] = 1812433253u * (m->s[k - 1] ^ (m->s[k - 1] >> 30)) + (uint32_t)k;
  m->i = 624;
}
static uint32_t mt_next(mt_t *m) {
  if (m->i >= 624) {
    for (int k = 0; k < 624; k++) {
      uint32_t y = (m->s[k] & 0x80000000u) | (m->s[(k + 1) % 624] & 0x7fffffffu);
      uint32_t v = m->s[(k + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      m->s[k] = v;
    }
    m->i = 0;
  }
  uint32_t y = m->s[m->i++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}
/* RandomNumber::getRandomNumber: (r - min)/max with min=0, max=2^32-1, so [0,1]
 * inclusive (RandomNumber.cpp:27-29). */
static double mt_uniform(mt_t *m) { return ((double)mt_next(m) - 0.0) / 4294967295.0; }

void orc_mt19937(unsigned seed, size_t n, uint32_t *out) {
  mt_t m;
  mt_seed(&m, seed);
  for (size_t k = 0; k < n; k++) out[k] = mt_next(&m);
}

/* ---- input.json (Input.cpp:49-263) --------------------------------------- */
typedef struct {
  char target[1024], ff[1024];
  unsigned nprobe, niter, seed, nthreads;
  double dt, temp, skin, lj_cutoff, coul_cutoff, alpha;
  int gas_flag, equip, short_cut, long_flag, long_cut, polar, user_ff;
  char gas_str[16], equip_str[8], short_str[8], long_str[8], long_cut_str[8], polar_str[8];
} orc_input;

/* Minimal reader for the flat JSON object the reference accepts: string and
 * number values only.  Returns the raw text of key's value or NULL. */
typedef struct {
  char key[64];
  char val[1024];
  int is_str;
} jkv;
static int json_parse_flat(const char *txt, jkv *kv, int maxkv, char *err, int errlen) {
  const char *p = txt;
  int n = 0;
  while (*p && isspace((unsigned char)*p)) p++;
  if (*p != '{') {
    set_err(err, errlen, "input.json: not a JSON object");
    return -1;
  }
  p++;
  for (;;) {
    while (*p && (isspace((unsigned char)*p) || *p == ',')) p++;
    if (*p == '}') break;
    if (*p != '"') {
      set_err(err, errlen, "input.json: expected a key");
      return -1;
    }
    p++;
    int k = 0;
    while (*p && *p != '"' && k < 63) kv[n].key[k++] = *p++;
    kv[n].key[k] = 0;
    if (*p != '"') {
      set_err(err, errlen, "input.json: bad key");
      return -1;
    }
    p++;
    while (*p && isspace((unsigned char)*p)) p++;
    if (*p != ':') {
      set_err(err, errlen, "input.json: expected ':'");
      return -1;
    }
    p++;
    while (*p && isspace((unsigned char)*p)) p++;
    int v = 0;
    if (*p == '"') {
      p++;
      while (*p && *p != '"' && v < 1023) kv[n].val[v++] = *p++;
      if (*p != '"') {
        set_err(err, errlen, "input.json: unterminated string");
        return -1;
      }
      p++;
      kv[n].is_str = 1;
    } else {
      while (*p && *p != ',' && *p != '}' && !isspace((unsigned char)*p) && v < 1023)
        kv[n].val[v++] = *p++;
      kv[n].is_str = 0;
    }
    kv[n].val[v] = 0;
    if (n + 1 < maxkv) n++;
  }
  return n;
}
static const jkv *jget(const jkv *kv, int n, const char *key) {
  const jkv *hit = NULL;
  for (int i = 0; i < n; i++)
    if (!strcmp(kv[i].key, key)) hit = &kv[i];
  return hit;
}

static int read_input(const char *path, orc_input *in, char *err, int errlen) {
  FILE *f = fopen(path, "rb");
  if (!f) {
    set_err(err, errlen, "cannot open %s", path);
    return -1;
  }
  fseek(f, 0, SEEK_END);
  long len = ftell(f);
  fseek(f, 0, SEEK_SET);
  char *txt = (char *)malloc((size_t)len + 1);
  size_t got = fread(txt, 1, (size_t)len, f);
  txt[got] = 0;
  fclose(f);
  jkv kv[64];
  int n = json_parse_flat(txt, kv, 64, err, errlen);
  free(txt);
  if (n < 0) return -1;
  const jkv *e;
  memset(in, 0, sizeof(*in));
  /* required (Input.cpp:62-70) */
  if (!(e = jget(kv, n, "targetFileName")) || !e->is_str) {
    set_err(err, errlen, "Error input.json: targetFileName not found");
    return -1;
  }
  snprintf(in->target, sizeof in->target, "%s", e->val);
  in->nprobe = (e = jget(kv, n, "numberProbe")) ? (unsigned)strtoul(e->val, 0, 10) : 10000;
  in->niter = (e = jget(kv, n, "nIter")) ? (unsigned)strtoul(e->val, 0, 10) : 10;
  in->seed = (e = jget(kv, n, "seed")) ? (unsigned)strtoul(e->val, 0, 10) : 20162104u;
  in->nthreads = (e = jget(kv, n, "nthreads")) ? (unsigned)strtoul(e->val, 0, 10)
                                               : (unsigned)omp_get_max_threads();
  in->dt = (e = jget(kv, n, "dt")) ? strtod(e->val, 0) : 10.0;
  in->temp = (e = jget(kv, n, "Temp")) ? strtod(e->val, 0) : 298.0;
  in->skin = (e = jget(kv, n, "skin")) ? strtod(e->val, 0) : 0.01;
  /* gas (Input.cpp:131-155) */
  if ((e = jget(kv, n, "GasBuffer"))) {
    snprintf(in->gas_str, sizeof in->gas_str, "%s", e->val);
    if (!strcmp(e->val, "He")) in->gas_flag = 1;
    else if (!strcmp(e->val, "N2")) in->gas_flag = 2;
    else if (!strcmp(e->val, "CO2")) in->gas_flag = 3;
    else if (!strcmp(e->val, "Ar")) in->gas_flag = 4;
    else if (!strcmp(e->val, "co2")) in->gas_flag = 5;
    else {
      set_err(err, errlen, "only available the follow gas buffer types: He Ar N2 CO2");
      return -1;
    }
  } else {
    strcpy(in->gas_str, "He");
    in->gas_flag = 1;
  }
#define YESNO(KEY, STR, FLAG, DEF_STR, DEF_FLAG)                                   \
  if ((e = jget(kv, n, KEY))) {                                                  \
    if (!strcmp(e->val, "yes")) { strcpy(STR, "yes"); FLAG = 1; }                \
    else if (!strcmp(e->val, "no")) { strcpy(STR, "no"); FLAG = 0; }             \
    else { set_err(err, errlen, "need to choice " KEY ": yes or no"); return -1; } \
  } else { strcpy(STR, DEF_STR); FLAG = DEF_FLAG; }
  YESNO("Equipotential", in->equip_str, in->equip, "no", 0)
  YESNO("Short-range cutoff", in->short_str, in->short_cut, "yes", 1)
  in->lj_cutoff = (e = jget(kv, n, "LJ-cutoff")) ? strtod(e->val, 0) : 12.0;
  YESNO("Long-range forces", in->long_str, in->long_flag, "no", 0)
  YESNO("Long-range cutoff", in->long_cut_str, in->long_cut, "yes", 1)
  in->coul_cutoff = (e = jget(kv, n, "Coul-cutoff")) ? strtod(e->val, 0) : 25.0;
  if (in->gas_flag == 1) {
    YESNO("polarizability", in->polar_str, in->polar, "yes", 1)
  } else {
    YESNO("polarizability", in->polar_str, in->polar, "no", 0)
  }
#undef YESNO
  /* alpha (Input.cpp:236-248); left 0 when polarizability is off and unset */
  if ((e = jget(kv, n, "alpha"))) in->alpha = strtod(e->val, 0);
  else if (in->polar) {
    const double tab[6] = {0.0, 0.204956, 1.710, 2.911, 1.6411, 2.911};
    in->alpha = tab[in->gas_flag];
  }
  if ((e = jget(kv, n, "force-field"))) {
    snprintf(in->ff, sizeof in->ff, "%s", e->val);
    in->user_ff = 1;
  }
  return 0;
}

/* ---- gas probe models (GasBuffer.cpp:58-192) ------------------------------ */
typedef struct {
  int natoms;
  double x[3], y[3], z[3], q[3], m[3], eps[3], sig[3];
  double mass, d;
  const char *type;
} orc_gas;

static void gas_init(orc_gas *g, int flag) {
  memset(g, 0, sizeof(*g));
  if (flag == 1) {
    g->natoms = 1; g->type = "He";
    g->m[0] = 4.0026; g->eps[0] = 0.0309008; g->sig[0] = 3.043;
    g->mass = g->m[0]; g->d = 0.0;
  } else if (flag == 2) {
    g->natoms = 3; g->type = "N2";
    g->z[0] = 0.5488; g->z[1] = -0.5488; g->z[2] = 0.0;
    g->q[0] = -0.4825; g->q[1] = -0.4825; g->q[2] = 0.965;
    g->m[0] = 14.007; g->m[1] = 14.007; g->m[2] = 0.0;
    g->eps[0] = 1.0; g->eps[1] = 1.0;
    g->mass = g->m[0] + g->m[1];
    g->d = fabs(g->z[0] - g->z[1]);
  } else if (flag == 3) {
    g->natoms = 3; g->type = "CO2";
    g->z[0] = -1.149; g->z[1] = 0.0; g->z[2] = 1.149;
    g->q[0] = -0.3256; g->q[1] = 0.6512; g->q[2] = -0.3256;
    g->m[0] = 15.999; g->m[1] = 12.011; g->m[2] = 15.999;
    g->eps[0] = 0.159; g->eps[1] = 0.055; g->eps[2] = 0.159;
    g->sig[0] = 3.033; g->sig[1] = 2.757; g->sig[2] = 3.033;
    g->mass = g->m[0] + g->m[1] + g->m[2];
    g->d = fabs(g->z[0] - g->z[2]);
  } else if (flag == 4) {
    g->natoms = 1; g->type = "Ar";
    g->m[0] = 39.948; g->eps[0] = 0.185; g->sig[0] = 3.446;
    g->mass = g->m[0]; g->d = 0.0;
  } else {
    g->natoms = 1; g->type = "co2";
    g->m[0] = 44.0098; g->eps[0] = 0.4008; g->sig[0] = 4.444;
    g->mass = g->m[0]; g->d = 0.0;
  }
}

/* ---- target molecule (MoleculeTarget.cpp) -------------------------------- */
#define NAMELEN 16
typedef struct {
  int natoms;
  double *x, *y, *z, *q, *m, *eps, *sig, *eps_c, *sig_c;
  char (*name)[NAMELEN];
  double mass, Q, maxX, maxY, maxZ, radius;
  double inertia[3][3], ivals[3], ivecs[3][3];
  int diagonal;
  int nparam;
  char pname[64][NAMELEN];
  double pm[64], peps[64], psig[64];
} orc_target;

static void target_free(orc_target *t) {
  free(t->x); free(t->y); free(t->z); free(t->q); free(t->m);
  free(t->eps); free(t->sig); free(t->eps_c); free(t->sig_c); free(t->name);
}
static void target_alloc(orc_target *t, int n) {
  t->natoms = n;
  size_t sz = (size_t)(n > 0 ? n : 1) * sizeof(double);
  t->x = malloc(sz); t->y = malloc(sz); t->z = malloc(sz); t->q = malloc(sz);
  t->m = malloc(sz); t->eps = malloc(sz); t->sig = malloc(sz);
  t->eps_c = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  t->sig_c = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  t->name = calloc((size_t)(n > 0 ? n : 1), NAMELEN);
}

/* defaultFF (MoleculeTarget.cpp:372-538): built-in per-gas parameter tables. */
static void default_ff(orc_target *t, int gas) {
  typedef struct { const char *s; double m, e, g; } row;
  static const row he[] = {{"C", 12.011, 0.0309, 3.043}, {"N", 14.007, 0.0309, 3.043},
                           {"H", 1.008, 0.0150, 2.38},   {"O", 15.999, 0.0309, 3.043},
                           {"S", 32.06, 0.0311, 3.5}};
  static const row n2[] = {{"C", 12.011, 0.0824736, 3.2255}, {"N", 14.007, 0.0758527, 3.5719},
                           {"H", 1.008, 0.0362711, 1.8986},  {"O", 15.999, 0.062323, 3.0750},
                           {"S", 32.06, 0.138032, 3.4237},   {"P", 30.9738, 0.145372, 3.47},
                           {"F", 18.9984, 0.04649, 3.1285}};
  static const row uff[] = {{"C", 12.011, 0.10499, 3.43085},  {"N", 14.007, 0.06899, 3.26069},
                            {"H", 1.008, 0.04399, 2.57113},   {"O", 15.999, 0.05999, 3.11815},
                            {"S", 32.06, 0.27399, 3.59478},   {"P", 30.9738, 0.30499, 3.69456}};
  static const row imos[] = {{"C", 12.011, 0.09759, 3.58140}, {"N", 14.007, 0.05579, 3.25500},
                             {"H", 1.008, 0.01892, 1.24090},  {"O", 15.999, 0.08279, 4.39200},
                             {"S", 32.06, 0.05999, 3.50000},  {"P", 30.9738, 0.05999, 3.50000},
                             {"K", 39.0983, 0.05999, 3.50000}};
  const row *r;
  int n;
  if (gas == 1) { r = he; n = 5; }
  else if (gas == 2) { r = n2; n = 7; }
  else if (gas == 3 || gas == 4) { r = uff; n = 6; }
  else { r = imos; n = 7; }
  t->nparam = n;
  for (int i = 0; i < n; i++) {
    snprintf(t->pname[i], NAMELEN, "%s", r[i].s);
    t->pm[i] = r[i].m; t->peps[i] = r[i].e; t->psig[i] = r[i].g;
  }
}

/* readUserFF (MoleculeTarget.cpp:321-370): count line, comment, then "Sym m eps sig". */
static int read_user_ff(orc_target *t, const char *path, char *err, int errlen) {
  FILE *f = fopen(path, "r");
  if (!f) {
    set_err(err, errlen, "Error: reading force-field parameters file %s", path);
    return -1;
  }
  char line[4096];
  int n = 0;
  if (!fgets(line, sizeof line, f) || sscanf(line, "%d", &n) != 1 || n < 0 || n > 64) {
    fclose(f);
    set_err(err, errlen, "Error: reading force-field parameters file");
    return -1;
  }
  if (!fgets(line, sizeof line, f)) n = 0;
  for (int i = 0; i < n; i++) {
    char sym[NAMELEN];
    double m, e, s;
    if (!fgets(line, sizeof line, f) || sscanf(line, "%15s %lf %lf %lf", sym, &m, &e, &s) != 4) {
      fclose(f);
      set_err(err, errlen, "Error: reading force-field parameters file");
      return -1;
    }
    snprintf(t->pname[i], NAMELEN, "%s", sym);
    t->pm[i] = m; t->peps[i] = e; t->psig[i] = s;
  }
  t->nparam = n;
  fclose(f);
  return 0;
}

/* assignedParameter (MoleculeTarget.cpp:540-570): per-gas pair parameters;
 * Lorentz-Berthelot mixing only for CO2 (O and C sites) and Ar. */
static int assign_param(const orc_target *t, int gas, const char *sym, double *m, double *e,
                        double *s, double *ec, double *sc) {
  for (int i = 0; i < t->nparam; i++) {
    if (!strcmp(sym, t->pname[i])) {
      *m = t->pm[i];
      if (gas == 3) {
        *e = sqrt(t->peps[i] * 0.159);
        *s = 0.5 * (t->psig[i] + 3.033);
        *ec = sqrt(t->peps[i] * 0.055);
        *sc = 0.5 * (t->psig[i] + 2.757);
      } else if (gas == 4) {
        *e = sqrt(t->peps[i] * 0.185);
        *s = 0.5 * (t->psig[i] + 3.446);
      } else {
        *e = t->peps[i];
        *s = t->psig[i];
      }
      return 0;
    }
  }
  return -1;
}

/* readXYZfile (MoleculeTarget.cpp:148-319).  4 columns: no charges.  Any other
 * consistent column count is read as "Sym x y z q" (the reference's checks at
 * :199 and :217 accept it); charges are zeroed for force_type 1/2. */
static int read_xyz(orc_target *t, const char *path, int gas, int force_type, int user_ff,
                    char *err, int errlen) {
  FILE *f = fopen(path, "r");
  if (!f) {
    set_err(err, errlen, "Error: reading xyz file %s", path);
    return -1;
  }
  char line[4096];
  int n = 0;
  if (!fgets(line, sizeof line, f) || sscanf(line, "%d", &n) != 1 || n < 0) {
    fclose(f);
    set_err(err, errlen, "Error: missing number ot atoms in xyz file");
    return -1;
  }
  if (!fgets(line, sizeof line, f)) line[0] = 0; /* comment */
  /* count items per remaining line */
  long pos = ftell(f);
  int nlines = 0, items0 = -1;
  while (fgets(line, sizeof line, f)) {
    int items = 0, in_tok = 0;
    for (char *c = line; *c; c++) {
      if (isspace((unsigned char)*c)) in_tok = 0;
      else if (!in_tok) { in_tok = 1; items++; }
    }
    if (items0 < 0) items0 = items;
    else if (items != items0) {
      fclose(f);
      set_err(err, errlen, "Error: numbers of items by lines in the xyz file");
      return -1;
    }
    nlines++;
  }
  if (nlines != n) {
    fclose(f);
    set_err(err, errlen, "Error: numbers of lines and natoms are differens in the xyz file");
    return -1;
  }
  int cond = (items0 == 4) ? 0 : 1;
  fseek(f, pos, SEEK_SET);
  target_alloc(t, n);
  t->mass = 0.0;
  t->Q = 0.0;
  for (int i = 0; i < n; i++) {
    char sym[NAMELEN] = {0};
    double xi = 0, yi = 0, zi = 0, qi = 0;
    if (!fgets(line, sizeof line, f)) line[0] = 0;
    if (cond == 0) sscanf(line, "%15s %lf %lf %lf", sym, &xi, &yi, &zi);
    else sscanf(line, "%15s %lf %lf %lf %lf", sym, &xi, &yi, &zi, &qi);
    if (cond == 0 || force_type == 1 || force_type == 2) qi = 0.0;
    snprintf(t->name[i], NAMELEN, "%s", sym);
    double m, e, s, ec = 0, sc = 0;
    if (assign_param(t, gas, sym, &m, &e, &s, &ec, &sc)) {
      fclose(f);
      set_err(err, errlen, user_ff ? "Atom type not found in the file user force field"
                                   : "Atom type not found in the default data base ");
      return -1;
    }
    t->x[i] = xi; t->y[i] = yi; t->z[i] = zi; t->q[i] = qi;
    t->m[i] = m; t->eps[i] = e; t->sig[i] = s; t->eps_c[i] = ec; t->sig_c[i] = sc;
    t->mass += m;
    t->Q += qi;
  }
  fclose(f);
  return 0;
}

/* readPQRfile (MoleculeTarget.cpp:60-146): whitespace fields
 * "ATOM serial name resName resSeq x y z q r"; element = first letter of the
 * atom name unless a user force field is given. */
static int read_pqr(orc_target *t, const char *path, int gas, int user_ff, char *err, int errlen) {
  FILE *f = fopen(path, "r");
  if (!f) {
    set_err(err, errlen, "Error: reading pqr file %s", path);
    return -1;
  }
  char line[4096];
  int n = 0;
  while (fgets(line, sizeof line, f)) {
    char rec[32] = {0};
    if (sscanf(line, "%31s", rec) == 1 && !strcmp(rec, "ATOM")) n++;
  }
  rewind(f);
  target_alloc(t, n);
  t->mass = 0.0;
  t->Q = 0.0;
  int i = 0;
  while (fgets(line, sizeof line, f) && i < n) {
    char rec[32] = {0}, aname[64] = {0}, res[64] = {0};
    int serial = 0, chain = 0;
    double xi, yi, zi, qi, ri;
    int got = sscanf(line, "%31s %d %63s %63s %d %lf %lf %lf %lf %lf", rec, &serial, aname, res,
                     &chain, &xi, &yi, &zi, &qi, &ri);
    if (got < 1 || strcmp(rec, "ATOM")) continue;
    if (got < 9) {
      fclose(f);
      set_err(err, errlen, "Error: unsupported PQR ATOM record: %s", line);
      return -1;
    }
    char sym[NAMELEN];
    if (user_ff) snprintf(sym, NAMELEN, "%s", aname);
    else { sym[0] = aname[0]; sym[1] = 0; }
    snprintf(t->name[i], NAMELEN, "%s", sym);
    double m, e, s, ec = 0, sc = 0;
    if (assign_param(t, gas, sym, &m, &e, &s, &ec, &sc)) {
      fclose(f);
      set_err(err, errlen, user_ff ? "Atom type not found in the file user force field"
                                   : "Atom type not found in the default data base ");
      return -1;
    }
    t->x[i] = xi; t->y[i] = yi; t->z[i] = zi; t->q[i] = qi;
    t->m[i] = m; t->eps[i] = e; t->sig[i] = s; t->eps_c[i] = ec; t->sig_c[i] = sc;
    t->mass += m;
    t->Q += qi;
    i++;
  }
  fclose(f);
  return 0;
}

/* calculateCenterOfMass + moveToCenterOfMass (MoleculeTarget.cpp:596-620) */
static void move_to_com(orc_target *t) {
  double r[3] = {0, 0, 0};
  for (int i = 0; i < t->natoms; i++) {
    r[0] += t->m[i] * t->x[i];
    r[1] += t->m[i] * t->y[i];
    r[2] += t->m[i] * t->z[i];
  }
  r[0] /= t->mass; r[1] /= t->mass; r[2] /= t->mass;
  for (int i = 0; i < t->natoms; i++) {
    t->x[i] -= r[0]; t->y[i] -= r[1]; t->z[i] -= r[2];
  }
}

/* calculateMoleculeRadius (MoleculeTarget.cpp:905-931) */
static void molecule_radius(orc_target *t) {
  double rmax = 0.0;
  int id = 0;
  for (int i = 0; i < t->natoms; i++) {
    double r = sqrt(t->x[i] * t->x[i] + t->y[i] * t->y[i] + t->z[i] * t->z[i]);
    if (r > rmax) { id = i; rmax = r; }
  }
  t->radius = sqrt(t->x[id] * t->x[id] + t->y[id] * t->y[id] + t->z[id] * t->z[id]);
}

/* orientateMolecule (MoleculeTarget.cpp:623-698).  The reference leaves theta
 * unset when the farthest atom has x==0 or y==0; 0 is used here. */
static void orientate(orc_target *t) {
  double rmax = 0.0, theta = 0.0, phi, gamma;
  int id = 0;
  for (int i = 0; i < t->natoms; i++) {
    double r = sqrt(t->x[i] * t->x[i] + t->y[i] * t->y[i] + t->z[i] * t->z[i]);
    if (r > rmax) { id = i; rmax = r; }
  }
  double xi = t->x[id], yi = t->y[id], zi = t->z[id];
  if ((xi != 0.0) & (yi != 0.0)) theta = atan2(yi, xi);
  phi = acos(zi / rmax);
  theta *= -1.0;
  for (int i = 0; i < t->natoms; i++) {
    xi = t->x[i]; yi = t->y[i];
    t->x[i] = cos(theta) * xi - sin(theta) * yi;
    t->y[i] = sin(theta) * xi + cos(theta) * yi;
  }
  phi *= -1.0;
  for (int i = 0; i < t->natoms; i++) {
    xi = t->x[i]; zi = t->z[i];
    t->x[i] = sin(phi) * zi + cos(phi) * xi;
    t->z[i] = cos(phi) * zi - sin(phi) * xi;
  }
  rmax = 0.0;
  for (int i = 0; i < t->natoms; i++) {
    double r = sqrt(t->x[i] * t->x[i] + t->y[i] * t->y[i]);
    if (r > rmax) { id = i; rmax = r; }
  }
  gamma = atan2(t->y[id], t->x[id]);
  gamma *= -1.0;
  for (int i = 0; i < t->natoms; i++) {
    xi = t->x[i]; yi = t->y[i];
    t->x[i] = cos(gamma) * xi - sin(gamma) * yi;
    t->y[i] = sin(gamma) * xi + cos(gamma) * yi;
  }
}

/* getEigenvalues: closed-form cubic roots (MoleculeTarget.cpp:812-850) */
static void eigenvalues(double A[3][3], double ev[3]) {
  double a0, a1, a2, p, q, R, Q, D, a, b, phase, mag;
  a0 = A[0][0] * A[1][1] * A[2][2] - A[0][0] * A[1][2] * A[2][1] - A[1][1] * A[0][2] * A[2][0] -
       A[2][2] * A[0][1] * A[1][0] + A[0][1] * A[1][2] * A[2][0] + A[0][2] * A[2][1] * A[1][0];
  a1 = A[0][1] * A[1][0] + A[0][2] * A[2][0] + A[1][2] * A[2][1] - A[0][0] * A[1][1] -
       A[1][1] * A[2][2] - A[2][2] * A[0][0];
  a2 = A[0][0] + A[1][1] + A[2][2];
  a0 = -a0; a1 = -a1; a2 = -a2;
  p = (3 * a1 - a2 * a2) / 3;
  q = (9 * a1 * a2 - 27 * a0 - 2 * a2 * a2 * a2) / 27;
  Q = p / 3; R = q / 2; D = Q * Q * Q + R * R;
  if (D < 0) { a = R; b = sqrt(-D); }
  else { a = R + sqrt(D); b = 0; }
  phase = atan2(b, a);
  mag = pow(a * a + b * b, 1.0 / 6.0);
  ev[0] = -(a2 / 3) + mag * 2 * cos(phase / 3.0);
  ev[1] = -(a2 / 3) - mag * (cos(phase / 3.0) + sqrt(3.0) * sin(phase / 3.0));
  ev[2] = -(a2 / 3) - mag * (cos(phase / 3.0) - sqrt(3.0) * sin(phase / 3.0));
}

/* getEigenvectors (MoleculeTarget.cpp:852-878) */
static void eigenvectors(double A[3][3], const double l[3], double V[3][3]) {
  double det, x, y, z, nf;
  det = l[0] * l[0] - l[0] * A[1][1] - A[1][2] * A[1][2] - l[0] * A[2][2] + A[1][1] * A[2][2];
  y = (l[0] * A[1][0] - A[2][2] * A[1][0] + A[1][2] * A[2][0]) / det;
  z = (A[2][1] * A[1][0] + l[0] * A[2][0] - A[1][1] * A[2][0]) / det;
  nf = sqrt(1 + y * y + z * z);
  V[0][0] = 1.0 / nf; V[0][1] = y / nf; V[0][2] = z / nf;
  det = l[1] * l[1] - l[1] * A[0][0] - A[0][2] * A[0][2] - l[1] * A[2][2] + A[0][0] * A[2][2];
  x = (l[1] * A[0][1] + A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
  z = (A[0][1] * A[0][2] + (l[1] - A[0][0]) * A[2][1]) / det;
  nf = sqrt(1 + x * x + z * z);
  V[1][0] = x / nf; V[1][1] = 1 / nf; V[1][2] = z / nf;
  V[2][0] = V[0][1] * V[1][2] - V[0][2] * V[1][1];
  V[2][1] = V[0][2] * V[1][0] - V[0][0] * V[1][2];
  V[2][2] = V[0][0] * V[1][1] - V[0][1] * V[1][0];
}

/* setInertia (MoleculeTarget.cpp:701-805): principal-axis frame, longest extent on z. */
static void set_inertia(orc_target *t) {
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) t->inertia[a][b] = 0.0;
  for (int i = 0; i < t->natoms; i++) {
    double r[3] = {t->x[i], t->y[i], t->z[i]}, mi = t->m[i];
    double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        t->inertia[a][b] += mi * (r2 * (a == b ? 1.0 : 0.0) - r[a] * r[b]);
  }
  double (*I)[3] = t->inertia;
  t->diagonal = 0;
  if (fabs(I[0][1]) < 1.e-12 && fabs(I[1][0]) < 1.e-12 && fabs(I[1][2]) < 1.e-12 &&
      fabs(I[2][1]) < 1.e-12 && fabs(I[2][0]) < 1.e-12 && fabs(I[0][2]) < 1.e-12) {
    orientate(t);
    t->diagonal = 1;
  } else {
    eigenvalues(I, t->ivals);
    eigenvectors(I, t->ivals, t->ivecs);
    double (*V)[3] = t->ivecs;
    double d = sqrt(pow(dot3(V[0], V[1]), 2.0));
    d = fmax(sqrt(pow(dot3(V[0], V[2]), 2.0)), d);
    d = fmax(sqrt(pow(dot3(V[1], V[2]), 2.0)), d);
    if (d > 1e-6) {
      orientate(t);
    } else {
      for (int i = 0; i < t->natoms; i++) {
        double xi = t->x[i], yi = t->y[i], zi = t->z[i];
        t->x[i] = xi * V[0][0] + yi * V[0][1] + zi * V[0][2];
        t->y[i] = xi * V[1][0] + yi * V[1][1] + zi * V[1][2];
        t->z[i] = xi * V[2][0] + yi * V[2][1] + zi * V[2][2];
      }
    }
  }
  double mx = 0, my = 0, mz = 0;
  for (int i = 0; i < t->natoms; i++) {
    if (fabs(t->x[i]) > fabs(mx)) mx = fabs(t->x[i]);
    if (fabs(t->y[i]) > fabs(my)) my = fabs(t->y[i]);
    if (fabs(t->z[i]) > fabs(mz)) mz = fabs(t->z[i]);
  }
  if (mx > my && mx > mz) {
    for (int i = 0; i < t->natoms; i++) {
      double xi = t->x[i], zi = t->z[i];
      t->x[i] = -zi; t->z[i] = xi;
    }
  } else if (my > mx && my > mz) {
    for (int i = 0; i < t->natoms; i++) {
      double yi = t->y[i], zi = t->z[i];
      t->y[i] = zi; t->z[i] = -yi;
    }
  }
  mx = 0; my = 0; mz = 0; /* signed extremes, as the reference keeps them (:795-803) */
  for (int i = 0; i < t->natoms; i++) {
    if (fabs(t->x[i]) > fabs(mx)) mx = t->x[i];
    if (fabs(t->y[i]) > fabs(my)) my = t->y[i];
    if (fabs(t->z[i]) > fabs(mz)) mz = t->z[i];
  }
  t->maxX = mx; t->maxY = my; t->maxZ = mz;
}

/* ---- linked cells (LinkedCell.cpp) ---------------------------------------- */
typedef struct {
  int Nx, Ny, Nz, Ncells, next;
  double lx, ly, lz, corner[3], h;
  int *count, *start;
  int *nb1_start, *nb1; /* CSR over cells */
  int *nb2_start, *nb2;
} orc_cells;

static void cells_free(orc_cells *c) {
  free(c->count); free(c->start); free(c->nb1_start); free(c->nb1);
  free(c->nb2_start); free(c->nb2);
}

/* calculateIndex (LinkedCell.cpp:117-129): flat index k + Nz*j + Nz*Ny*i. */
static int cell_index(const orc_cells *c, const double pos[3]) {
  int i = (int)floor((pos[0] - c->corner[0]) / c->h);
  int j = (int)floor((pos[1] - c->corner[1]) / c->h);
  int k = (int)floor((pos[2] - c->corner[2]) / c->h);
  return k + c->Nz * j + c->Nz * c->Ny * i;
}

typedef struct { int i, j, k; } off3;

/* Stencil classification of LinkedCell::calculateCellsNeighbors (LinkedCell.cpp:228-400).
 * Returns 1 (neighbors1), 2 (neighbors2) or 0 (not a neighbour). */
static int stencil_class(int i, int j, int k, int n1, double R1, double R2, int next) {
  double R1s = R1 * R1, R2s = R2 * R2;
  if (i == 0 && j == 0 && k == 0) return 1;
  int ai = abs(i), aj = abs(j), ak = abs(k);
  double dij, dm; /* squared distance in cell units, and with each |.|-1 */
  if (i != 0 && j == 0 && k == 0) return ai <= n1 ? 1 : (next ? 2 : 0);
  if (i == 0 && j != 0 && k == 0) return aj <= n1 ? 1 : (next ? 2 : 0);
  if (i == 0 && j == 0 && k != 0) return ak <= n1 ? 1 : (next ? 2 : 0);
  if (i == 0) { dij = (double)(j * j + k * k); dm = pow(aj - 1, 2) + pow(ak - 1, 2); }
  else if (j == 0) { dij = (double)(i * i + k * k); dm = pow(ai - 1, 2) + pow(ak - 1, 2); }
  else if (k == 0) { dij = (double)(i * i + j * j); dm = pow(ai - 1, 2) + pow(aj - 1, 2); }
  else { dij = (double)(i * i + j * j + k * k); dm = pow(ai - 1, 2) + pow(aj - 1, 2) + pow(ak - 1, 2); }
  if (next) {
    if (dij < R2s || dm < R2s) {
      if (dij < R1s) return 1;
      if (dm < R1s) return 1;
      return 2;
    }
    return 0;
  }
  if (dij < R1s || dm < R1s) return 1;
  return 0;
}

/* LinkedCell::LinkedCell (LinkedCell.cpp:19-42): grid, binning, in-place sort of
 * the target arrays by cell, neighbour lists of non-empty cells. */
static void build_cells(orc_cells *c, orc_target *t, int gas, double a, double b, double cc,
                        double lj_cutoff, double skin, int long_flag, double coul_cutoff) {
  memset(c, 0, sizeof(*c));
  c->h = lj_cutoff + skin;
  c->lx = 2.0 * a; c->ly = 2.0 * b; c->lz = 2.0 * cc;
  c->Nx = (int)ceil(c->lx / c->h);
  c->Ny = (int)ceil(c->ly / c->h);
  c->Nz = (int)ceil(c->lz / c->h);
  c->lx = ((double)c->Nx) * c->h;
  c->ly = ((double)c->Ny) * c->h;
  c->lz = ((double)c->Nz) * c->h;
  c->Ncells = c->Nx * c->Ny * c->Nz;
  c->next = long_flag == 1;
  c->corner[0] = -0.5 * c->lx; c->corner[1] = -0.5 * c->ly; c->corner[2] = -0.5 * c->lz;
  int N = t->natoms, NC = c->Ncells;
  c->count = calloc((size_t)NC, sizeof(int));
  c->start = calloc((size_t)NC + 1, sizeof(int));
  int *cell_of = malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  for (int i = 0; i < N; i++) {
    double p[3] = {t->x[i], t->y[i], t->z[i]};
    cell_of[i] = cell_index(c, p);
    c->count[cell_of[i]]++;
  }
  for (int k = 0; k < NC; k++) c->start[k + 1] = c->start[k] + c->count[k];
  /* stable bucket order: cells ascending, original atom order within a cell (:161-180) */
  int *fill = malloc(sizeof(int) * (size_t)NC), *perm = malloc(sizeof(int) * (size_t)(N > 0 ? N : 1));
  memcpy(fill, c->start, sizeof(int) * (size_t)NC);
  for (int i = 0; i < N; i++) perm[fill[cell_of[i]]++] = i;
  orc_target tmp;
  memset(&tmp, 0, sizeof tmp);
  target_alloc(&tmp, N);
  for (int s = 0; s < N; s++) {
    int i = perm[s];
    tmp.x[s] = t->x[i]; tmp.y[s] = t->y[i]; tmp.z[s] = t->z[i]; tmp.q[s] = t->q[i];
    tmp.m[s] = t->m[i]; tmp.eps[s] = t->eps[i]; tmp.sig[s] = t->sig[i];
    tmp.eps_c[s] = t->eps_c[i]; tmp.sig_c[s] = t->sig_c[i];
    memcpy(tmp.name[s], t->name[i], NAMELEN);
  }
#define SWAPF(F) { void *sw = t->F; t->F = tmp.F; tmp.F = sw; }
  SWAPF(x) SWAPF(y) SWAPF(z) SWAPF(q) SWAPF(m) SWAPF(eps) SWAPF(sig) SWAPF(eps_c) SWAPF(sig_c) SWAPF(name)
#undef SWAPF
  target_free(&tmp);
  free(fill); free(perm); free(cell_of);
  (void)gas;

  /* stencils (:228-400), enumerated in the reference's i,j,k loop order */
  double R1 = lj_cutoff / c->h, R2 = c->next ? coul_cutoff / c->h : 0.0;
  int n1 = (int)ceil(R1), ncl = n1;
  if (c->next) ncl = (int)ceil(R2);
  int side = 2 * ncl + 1;
  off3 *s1 = malloc(sizeof(off3) * (size_t)side * side * side);
  off3 *s2 = malloc(sizeof(off3) * (size_t)side * side * side);
  int ns1 = 0, ns2 = 0;
  for (int i = -ncl; i < ncl + 1; i++)
    for (int j = -ncl; j < ncl + 1; j++)
      for (int k = -ncl; k < ncl + 1; k++) {
        int cls = stencil_class(i, j, k, n1, R1, R2, c->next);
        if (cls == 1) s1[ns1++] = (off3){i, j, k};
        else if (cls == 2) s2[ns2++] = (off3){i, j, k};
      }
  /* neighbour lists keep only in-grid, non-empty cells (:405-433) */
  c->nb1_start = calloc((size_t)NC + 1, sizeof(int));
  c->nb2_start = calloc((size_t)NC + 1, sizeof(int));
  for (int pass = 0; pass < 2; pass++) {
    int n1tot = 0, n2tot = 0;
    for (int i = 0; i < c->Nx; i++)
      for (int j = 0; j < c->Ny; j++)
        for (int k = 0; k < c->Nz; k++) {
          int idx = k + c->Nz * j + c->Nz * c->Ny * i;
          if (pass == 1) { c->nb1_start[idx] = n1tot; c->nb2_start[idx] = n2tot; }
          for (int m = 0; m < ns1; m++) {
            int ii = i + s1[m].i, jj = j + s1[m].j, kk = k + s1[m].k;
            if (-1 < ii && ii < c->Nx && -1 < jj && jj < c->Ny && -1 < kk && kk < c->Nz) {
              int nb = kk + c->Nz * jj + c->Nz * c->Ny * ii;
              if (c->count[nb] != 0) {
                if (pass == 1) c->nb1[n1tot] = nb;
                n1tot++;
              }
            }
          }
          if (c->next)
            for (int m = 0; m < ns2; m++) {
              int ii = i + s2[m].i, jj = j + s2[m].j, kk = k + s2[m].k;
              if (-1 < ii && ii < c->Nx && -1 < jj && jj < c->Ny && -1 < kk && kk < c->Nz) {
                int nb = kk + c->Nz * jj + c->Nz * c->Ny * ii;
                if (c->count[nb] != 0) {
                  if (pass == 1) c->nb2[n2tot] = nb;
                  n2tot++;
                }
              }
            }
        }
    if (pass == 0) {
      c->nb1 = malloc(sizeof(int) * (size_t)(n1tot > 0 ? n1tot : 1));
      c->nb2 = malloc(sizeof(int) * (size_t)(n2tot > 0 ? n2tot : 1));
    } else {
      c->nb1_start[NC] = n1tot;
      c->nb2_start[NC] = n2tot;
    }
  }
  free(s1);
  free(s2);
}

/* ---- the system ------------------------------------------------------------ */
struct orc_system {
  orc_input in;
  orc_target t;
  orc_gas gas;
  orc_cells lc;
  int force_type;
  double mu, alpha, inertia_gas, d_bond, a, b, c, bmax, lx, ly, lz;
  double t_orient, t_ellip, t_lc;
};

/* force_type selection (System.cpp:49-87) */
static int select_force_type(const orc_input *in) {
  int g = in->gas_flag, s = in->short_cut, l = in->long_flag, lc = in->long_cut, p = in->polar;
  if (g == 1 || g == 4 || g == 5) {
    if (s == 0 && l == 0) return 1;
    if (s == 1 && l == 0) return 2;
    if (s == 0 && p == 1 && lc == 0) return 3;
    if (s == 1 && p == 1 && lc == 1) return 4;
    return 2;
  }
  if (s == 0 && l == 0 && p == 0) return 1;
  if (s == 1 && l == 0 && p == 0) return 2;
  if (s == 0 && l == 1 && lc == 0 && p == 0) return 3;
  if (s == 1 && l == 1 && lc == 1 && p == 0) return 4;
  if (s == 0 && l == 1 && lc == 0 && p == 1) return 5;
  if (s == 1 && l == 1 && lc == 1 && p == 1) return 6;
  return 2;
}

/* geometric_ellipsoid (System.cpp:1640-1698) */
static void geometric_ellipsoid(orc_system *S, int print) {
  orc_target *t = &S->t;
  double maxX = fabs(t->maxX), maxY = fabs(t->maxY), maxZ = fabs(t->maxZ);
  double d = S->gas.d;
  double radius = S->in.long_flag == 1 ? 2.0 * S->in.coul_cutoff : 2.0 * S->in.lj_cutoff;
  if (print) {
    printf("*********************************************************\n");
    printf("Geometric Ellipsoid: \n");
    printf("*********************************************************\n");
    printf("maximal distances: %g  %g  %g  Ang\n", maxX, maxY, maxZ);
  }
  double a = maxX + radius + S->in.skin + d;
  double b = maxY + radius + S->in.skin + d;
  double c = maxZ + radius + S->in.skin + d;
  if (print) printf("Initial axis length: %g  %g  %g  Ang\n", a, b, c);
  const double delta = 0.01;
  for (int i = 0; i < t->natoms; i++) {
    double xi = t->x[i], yi = t->y[i], zi = t->z[i];
    double ri = sqrt(xi * xi + yi * yi + zi * zi);
    double ux = xi / ri, uy = yi / ri, uz = zi / ri;
    double x = xi + (radius + d) * ux, y = yi + (radius + d) * uy, z = zi + (radius + d) * uz;
    for (;;) {
      double e = pow(x / a, 2) + pow(y / b, 2) + pow(z / c, 2);
      if (e > 1.0) { a += delta; b += delta; c += delta; }
      else break;
    }
  }
  if (print) printf("Ellipsoid axis length: %g  %g  %g  Ang\n", a, b, c);
  S->a = a; S->b = b; S->c = c;
}

static void print_input(const orc_input *in) { /* Input.cpp:313-345 */
  printf("*********************************************************\n");
  printf("INPUT:: Simulation Parameters \n");
  printf("*********************************************************\n");
  printf("target filename                  : %s\n", in->target);
  printf("number of probe                  : %u\n", in->nprobe);
  printf("number of iterarions             : %u\n", in->niter);
  printf("number of threads                : %u\n", in->nthreads);
  printf("seed number                      : %u\n", in->seed);
  printf("gas buffer                       : %s\n", in->gas_str);
  printf("Target Temperature (K)           : %g\n", in->temp);
  printf("timestep (fs)                    : %g\n", in->dt);
  printf("Skin cell size (Ang)             : %g\n", in->skin);
  printf("Equipotential                    : %s\n", in->equip_str);
  printf("Cut short-range interaction      : %s\n", in->short_str);
  if (in->short_cut == 1) printf("LJ cutoff (Ang)                  : %g\n", in->lj_cutoff);
  printf("Apply long-range interaction     : %s\n", in->long_str);
  printf("Cut long-range interaction       : %s\n", in->long_cut_str);
  if (in->long_cut == 1) printf("Coulomb cutoff (Ang)             : %g\n", in->coul_cutoff);
  printf("Apply induced-dipole interaction : %s\n", in->polar_str);
  if (in->polar == 1) printf("alpha (Ang^3)                    : %g\n", in->alpha);
  if (in->user_ff == 1) printf("force-field                      : %s\n", in->ff);
}

static void resolve_relative(char *dst, size_t n, const char *json_path, const char *file) {
  if (file[0] == '/') { snprintf(dst, n, "%s", file); return; }
  const char *slash = strrchr(json_path, '/');
  if (!slash) { snprintf(dst, n, "%s", file); return; }
  snprintf(dst, n, "%.*s/%s", (int)(slash - json_path), json_path, file);
}

orc_system *orc_open(const char *json_path, int print, char *err, int errlen) {
  orc_system *S = calloc(1, sizeof(orc_system));
  if (read_input(json_path, &S->in, err, errlen)) { free(S); return NULL; }
  if (print) print_input(&S->in);
  S->force_type = select_force_type(&S->in);
  gas_init(&S->gas, S->in.gas_flag);
  /* paths in input.json are taken relative to the json file's directory here
   * (the reference resolves them against the working directory) */
  char tpath[2048], fpath[2048];
  resolve_relative(tpath, sizeof tpath, json_path, S->in.target);
  double t0 = wall_s();
  if (S->in.user_ff) {
    resolve_relative(fpath, sizeof fpath, json_path, S->in.ff);
    if (read_user_ff(&S->t, fpath, err, errlen)) { free(S); return NULL; }
  } else default_ff(&S->t, S->in.gas_flag);
  if (print) { /* printFF (MoleculeTarget.cpp:572-594) */
    printf("*********************************************************\n");
    printf("Force Field parameters: \n");
    printf("*********************************************************\n");
    printf("Symbol  mass (amu)  epsilon (kcal/mol)  sigma(Angstroms) \n");
    for (int i = 0; i < S->t.nparam; i++)
      printf("%s   %g   %g   %g\n", S->t.pname[i], S->t.pm[i], S->t.peps[i], S->t.psig[i]);
  }
  const char *ext = strrchr(S->in.target, '.');
  int rc;
  if (ext && !strcmp(ext, ".pqr")) rc = read_pqr(&S->t, tpath, S->in.gas_flag, S->in.user_ff, err, errlen);
  else if (ext && !strcmp(ext, ".xyz"))
    rc = read_xyz(&S->t, tpath, S->in.gas_flag, S->force_type, S->in.user_ff, err, errlen);
  else { set_err(err, errlen, "Error: only acceptable PQR or XYZ or XYZ-Q format"); rc = -1; }
  if (rc) { free(S); return NULL; }
  move_to_com(&S->t);
  molecule_radius(&S->t);
  set_inertia(&S->t);
  S->t_orient = wall_s() - t0;
  if (print) {
    printf("*********************************************************\n");
    printf("MOLECULE:: orientation around the inertia principal axis \n");
    printf("*********************************************************\n");
    printf("Inertia matrix a.u. Ang^2: \n");
    for (int a = 0; a < 3; a++)
      printf("{  %g  %g  %g  }\n", S->t.inertia[a][0], S->t.inertia[a][1], S->t.inertia[a][2]);
    if (!S->t.diagonal) {
      printf("Rotation matrix applied to molecule: \n");
      for (int a = 0; a < 3; a++)
        printf("{  %g  %g  %g  }\n", S->t.ivecs[a][0], S->t.ivecs[a][1], S->t.ivecs[a][2]);
    }
    printf("Molecule radius: %g Ang \n", S->t.radius);
    printf("orientation time of molecule target: %g s\n", S->t_orient);
  }
  /* reduced mass / molecular inertia (System.cpp:97-114) */
  int g = S->in.gas_flag;
  if (g == 1 || g == 4 || g == 5) S->mu = S->t.mass * S->gas.mass / (S->t.mass + S->gas.mass);
  else {
    S->mu = S->gas.mass;
    S->inertia_gas = 0.0;
    for (int i = 0; i < S->gas.natoms; i++) S->inertia_gas += S->gas.m[i] * pow(S->gas.z[i], 2);
    S->d_bond = S->gas.d;
  }
  if (print) {
    printf("target mass: %g amu\n", S->t.mass);
    printf("gas mass: %g amu\n", S->gas.mass);
    printf("reduce mass: %g amu\n", S->mu);
    printf("charge state: %g e\n", S->t.Q);
  }
  S->alpha = S->in.alpha * ALPHA_TO_KCAL_MOL;
  t0 = wall_s();
  if (S->in.equip) { /* the Equipotential boundary is outside this path */
    set_err(err, errlen, "Equipotential ellipsoid is not part of this oracle");
    target_free(&S->t);
    free(S);
    return NULL;
  }
  geometric_ellipsoid(S, print);
  S->t_ellip = wall_s() - t0;
  if (print) printf("ellipsoid calculation time: %gs\n", S->t_ellip);
  S->bmax = fmax(fmax(S->a, S->b), S->c);
  if (print) printf("maximal impact parameter: %g Ang\n", S->bmax);
  t0 = wall_s();
  build_cells(&S->lc, &S->t, g, S->a, S->b, S->c, S->in.lj_cutoff, S->in.skin, S->in.long_flag,
              S->in.coul_cutoff);
  S->t_lc = wall_s() - t0;
  if (print) { /* LinkedCell::print (LinkedCell.cpp:443-480) */
    int filled = 0, empty = 0, avg = 0, mx = 0, mn = S->t.natoms;
    for (int i = 0; i < S->lc.Ncells; i++) {
      int n = S->lc.count[i];
      if (n == 0) empty++;
      else { avg += n; filled++; if (n > mx) mx = n; if (n < mn) mn = n; }
    }
    printf("*********************************************************\n");
    printf("Linked-cell: \n");
    printf("Numbers of cells: %d\n", S->lc.Ncells);
    printf("Nx: %d Ny: %d Nz: %d\n", S->lc.Nx, S->lc.Ny, S->lc.Nz);
    printf("Filled cells: %d\n", filled);
    printf("Empty cells: %d\n", empty);
    printf("Average atoms per cell: %g\n", (double)((float)avg / (float)filled));
    printf("Maximum atoms per cell: %d\n", mx);
    printf("Minimum atoms per cell: %d\n", mn);
    printf("Simulation box: \n");
    printf("lx: %g Ang\nly: %g Ang\nlz: %g Ang\n", S->lc.lx, S->lc.ly, S->lc.lz);
    printf("linked-cell calculation time: %g s\n", S->t_lc);
  }
  S->lx = 0.5 * S->lc.lx;
  S->ly = 0.5 * S->lc.ly;
  S->lz = 0.5 * S->lc.lz;
  return S;
}

void orc_close(orc_system *S) {
  if (!S) return;
  target_free(&S->t);
  cells_free(&S->lc);
  free(S);
}

void orc_get_params(const orc_system *S, orc_params *p) {
  memset(p, 0, sizeof(*p));
  p->gas_flag = S->in.gas_flag;
  p->force_type = S->force_type;
  p->natoms = S->t.natoms;
  p->gas_natoms = S->gas.natoms;
  p->nprobe = S->in.nprobe; p->niter = S->in.niter; p->seed = S->in.seed; p->nthreads = S->in.nthreads;
  p->short_range_cutoff = S->in.short_cut; p->long_range_flag = S->in.long_flag;
  p->long_range_cutoff = S->in.long_cut; p->polarizability_flag = S->in.polar;
  p->equipotential_flag = S->in.equip; p->user_ff_flag = S->in.user_ff;
  p->dt = S->in.dt; p->temperature = S->in.temp; p->skin = S->in.skin;
  p->lj_cutoff = S->in.lj_cutoff; p->coul_cutoff = S->in.coul_cutoff;
  p->alpha = S->alpha;
  p->mu = S->mu; p->target_mass = S->t.mass; p->target_charge = S->t.Q;
  p->gas_mass = S->gas.mass; p->gas_inertia = S->inertia_gas; p->d_bond = S->d_bond;
  p->a = S->a; p->b = S->b; p->c = S->c; p->bmax = S->bmax;
  p->lx = S->lx; p->ly = S->ly; p->lz = S->lz;
  p->Nx = S->lc.Nx; p->Ny = S->lc.Ny; p->Nz = S->lc.Nz; p->Ncells = S->lc.Ncells;
  p->cell_size = S->lc.h;
  p->max_x = S->t.maxX; p->max_y = S->t.maxY; p->max_z = S->t.maxZ; p->radius = S->t.radius;
}

void orc_get_target(const orc_system *S, double *x, double *y, double *z, double *q, double *m,
                    double *eps, double *sig, double *eps_c, double *sig_c) {
  size_t n = (size_t)S->t.natoms * sizeof(double);
  if (x) memcpy(x, S->t.x, n);
  if (y) memcpy(y, S->t.y, n);
  if (z) memcpy(z, S->t.z, n);
  if (q) memcpy(q, S->t.q, n);
  if (m) memcpy(m, S->t.m, n);
  if (eps) memcpy(eps, S->t.eps, n);
  if (sig) memcpy(sig, S->t.sig, n);
  if (eps_c) memcpy(eps_c, S->t.eps_c, n);
  if (sig_c) memcpy(sig_c, S->t.sig_c, n);
}

/* ---- forces (Force.cpp) ------------------------------------------------------
 * Accumulator block shared by the routines; visits counts every atom of every
 * stencil cell walked (the instrumented reference's unit of work). */
typedef struct {
  double U, fx, fy, fz;
  double Ex, Ey, Ez, Exx, Eyy, Ezz, Exy, Exz, Eyz;
  uint64_t visits;
} facc;

#define LJ_BLOCK(EPS, SIG)                                                         \
  {                                                                                \
    double epsilon = (EPS), sigma = (SIG);                                         \
    double r6inv = r2inv * r2inv * r2inv;                                          \
    double lj1 = 4.0 * epsilon * pow(sigma, 6.0);                                  \
    double lj2 = lj1 * pow(sigma, 6.0);                                            \
    double Ulj = r6inv * (lj2 * r6inv - lj1);                                      \
    double rc6inv = 1.0 / pow(lj_cutoff, 6);                                       \
    double Ulj_cut = rc6inv * (lj2 * rc6inv - lj1);                                \
    double lj3 = 6.0 * lj1, lj4 = 12.0 * lj2;                                      \
    double flj = r6inv * (lj4 * r6inv - lj3) * r2inv;                              \
    A->U += Ulj - Ulj_cut;                                                         \
    A->fx += flj * dx; A->fy += flj * dy; A->fz += flj * dz;                       \
  }
#define COUL_BLOCK(QI, QJ)                                                         \
  {                                                                                \
    double qi_ = (QI), qj_ = (QJ);                                                 \
    double rinv = 1.0 / r;                                                         \
    double Ucoul = qi_ * qj_ * rinv * KCOUL;                                       \
    double Ushift = -1.5 * qi_ * qj_ * KCOUL / coul_cutoff +                      \
                    0.5 * qi_ * qj_ * KCOUL * r2 / pow(coul_cutoff, 3);            \
    double r2inv_c = 1.0 / r2;                                                     \
    double fcoul = Ucoul * r2inv_c * (1.0 - pow(r / coul_cutoff, 3));              \
    A->U += Ucoul + Ushift;                                                        \
    A->fx += fcoul * dx; A->fy += fcoul * dy; A->fz += fcoul * dz;                 \
  }
/* smoothed field and gradient, Force.cpp:393-426 (R3 is 1/r^3 as the routine forms it) */
#define DIPOLE_LC_BLOCK(QA, R3)                                                    \
  {                                                                                \
    double q_ = (QA);                                                              \
    double r3inv = (R3);                                                           \
    double r5inv = r3inv * r2inv;                                                  \
    double rc3inv = 1.0 / pow(coul_cutoff, 3);                                     \
    double smooth = (1.0 - r * r2 * rc3inv);                                       \
    double qr3inv = q_ * r3inv * smooth;                                           \
    double qr5inv = -3.0 * q_ * r5inv * smooth;                                    \
    double qrc = -3.0 * q_ * rc3inv * r2inv;                                       \
    A->Ex += dx * qr3inv; A->Ey += dy * qr3inv; A->Ez += dz * qr3inv;              \
    A->Exx += qr3inv + dx * dx * qr5inv + dx * dx * qrc;                           \
    A->Eyy += qr3inv + dy * dy * qr5inv + dy * dy * qrc;                           \
    A->Ezz += qr3inv + dz * dz * qr5inv + dz * dz * qrc;                           \
    A->Exy += dx * dy * qr5inv + dx * dy * qrc;                                    \
    A->Exz += dx * dz * qr5inv + dx * dz * qrc;                                    \
    A->Eyz += dy * dz * qr5inv + dy * dz * qrc;                                    \
  }

enum { LC_LJ = 1, LC_COUL = 2, LC_DIP = 4 };

/* One linked-cell routine covering Force.cpp's *_LC family.  mode picks the
 * terms: LJ on neighbors1 (r < lj_cutoff), Coulomb and/or the smoothed dipole
 * field on neighbors1+2 (r < coul_cutoff).  dipole_r3_from_rinv selects how
 * the routine forms 1/r^3 (1.0/r*r2inv vs rinv*r2inv; both equal 1/r/r^2). */
static int force_lc(const orc_system *S, const double p[3], double qi, const double *eps,
                    const double *sig, int mode, int r2inv_first, facc *A) {
  const orc_cells *c = &S->lc;
  const orc_target *t = &S->t;
  const double lj_cutoff = S->in.lj_cutoff, coul_cutoff = S->in.coul_cutoff;
  int index = cell_index(c, p);
  if (index >= c->Ncells || index < 0) return 0; /* Force.cpp:58-66 */
  for (int pass = 0; pass < 2; pass++) {
    if (pass == 1 && !c->next) break;
    const int *nb = pass == 0 ? c->nb1 : c->nb2;
    int b = pass == 0 ? c->nb1_start[index] : c->nb2_start[index];
    int e = pass == 0 ? c->nb1_start[index + 1] : c->nb2_start[index + 1];
    for (int ci = b; ci < e; ci++) {
      int cell = nb[ci];
      int a0 = c->start[cell], a1 = a0 + c->count[cell];
      A->visits += (uint64_t)(a1 - a0);
      for (int j = a0; j < a1; j++) {
        double dx = p[0] - t->x[j], dy = p[1] - t->y[j], dz = p[2] - t->z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double r2inv = r2inv_first ? 1.0 / r2 : 0.0;
        if (pass == 0 && (mode & LC_LJ) && r < lj_cutoff) {
          if (!r2inv_first) r2inv = 1.0 / r2;
          LJ_BLOCK(eps[j], sig[j])
        }
        if ((mode & (LC_COUL | LC_DIP)) && r < coul_cutoff) {
          if (mode & LC_COUL) COUL_BLOCK(qi, t->q[j])
          if (mode & LC_DIP) {
            if (!r2inv_first) r2inv = 1.0 / r2;
            DIPOLE_LC_BLOCK(t->q[j], 1.0 / r * r2inv)
          }
        }
      }
    }
  }
  return 1;
}

/* All-pairs routines (Force.cpp:117-300, 495-574, 836-897, 1169-1219,
 * 1352-1415, 1637-1725): no cutoffs, no shifts, unsmoothed field. */
static void force_all(const orc_system *S, const double p[3], double qi, const double *eps,
                      const double *sig, int lj, int coul, int dip, facc *A) {
  const orc_target *t = &S->t;
  for (int i = 0; i < t->natoms; i++) {
    double dx = p[0] - t->x[i], dy = p[1] - t->y[i], dz = p[2] - t->z[i];
    double r2 = dx * dx + dy * dy + dz * dz;
    double r = sqrt(r2);
    if (lj) {
      double epsilon = eps[i], sigma = sig[i];
      double r2inv = 1.0 / r2;
      double r6inv = r2inv * r2inv * r2inv;
      double lj1 = 4.0 * epsilon * pow(sigma, 6.0);
      double lj2 = lj1 * pow(sigma, 6.0);
      A->U += r6inv * (lj2 * r6inv - lj1);
      double lj3 = 6.0 * lj1, lj4 = 12.0 * lj2;
      double flj = r6inv * (lj4 * r6inv - lj3) * r2inv;
      A->fx += flj * dx; A->fy += flj * dy; A->fz += flj * dz;
    }
    double rinv = 1.0 / r, r2inv = 1.0 / r2;
    if (coul) {
      double Ucoul = qi * t->q[i] * rinv * KCOUL;
      double fcoul = Ucoul * r2inv;
      A->U += Ucoul;
      A->fx += fcoul * dx; A->fy += fcoul * dy; A->fz += fcoul * dz;
    }
    if (dip) {
      double q = t->q[i];
      double r3inv = rinv * r2inv;
      double r5inv = r3inv * r2inv;
      double qr3inv = q * r3inv, qr5inv = q * r5inv;
      A->Ex += dx * qr3inv; A->Ey += dy * qr3inv; A->Ez += dz * qr3inv;
      A->Exx += qr3inv - 3.0 * dx * dx * qr5inv;
      A->Eyy += qr3inv - 3.0 * dy * dy * qr5inv;
      A->Ezz += qr3inv - 3.0 * dz * dz * qr5inv;
      A->Exy += -3.0 * dx * dy * qr5inv;
      A->Exz += -3.0 * dx * dz * qr5inv;
      A->Eyz += -3.0 * dy * dz * qr5inv;
    }
  }
  A->visits += (uint64_t)t->natoms;
}

static void finish(const facc *A, double alpha, int dip, double f[3], double *U) {
  if (dip) { /* Force.cpp:483-487 */
    f[0] = A->fx + alpha * (A->Ex * A->Exx + A->Ey * A->Exy + A->Ez * A->Exz);
    f[1] = A->fy + alpha * (A->Ex * A->Exy + A->Ey * A->Eyy + A->Ez * A->Eyz);
    f[2] = A->fz + alpha * (A->Ex * A->Exz + A->Ey * A->Eyz + A->Ez * A->Ezz);
    *U = A->U - 0.5 * alpha * (A->Ex * A->Ex + A->Ey * A->Ey + A->Ez * A->Ez);
  } else {
    f[0] = A->fx; f[1] = A->fy; f[2] = A->fz;
    *U = A->U;
  }
}

/* The reference's per-site force dispatch (System.cpp:371-379, 594-637,
 * 1028-1065, repeated inside the step loops). */
static void site_force(const orc_system *S, int iatom, const double p[3], double f[3], double *U,
                       uint64_t *visits) {
  facc A;
  memset(&A, 0, sizeof A);
  const orc_target *t = &S->t;
  int g = S->in.gas_flag, ft = S->force_type;
  double qi = S->gas.q[iatom];
  int dip = 0, inside = 1;
  if (g == 1 || g == 4 || g == 5) {
    switch (ft) {
      case 1: force_all(S, p, 0.0, t->eps, t->sig, 1, 0, 0, &A); break;
      case 2: inside = force_lc(S, p, 0.0, t->eps, t->sig, LC_LJ, 0, &A); break;
      case 3: force_all(S, p, 0.0, t->eps, t->sig, 1, 0, 1, &A); dip = 1; break;
      case 4: inside = force_lc(S, p, 0.0, t->eps, t->sig, LC_LJ | LC_DIP, 1, &A); dip = 1; break;
    }
  } else if (g == 2) {
    if (iatom == 2) {
      switch (ft) {
        case 1: case 2: break;
        case 3: force_all(S, p, qi, t->eps, t->sig, 0, 1, 0, &A); break;
        case 4: inside = force_lc(S, p, qi, t->eps, t->sig, LC_COUL, 0, &A); break;
        case 5: force_all(S, p, qi, t->eps, t->sig, 0, 1, 1, &A); dip = 1; break;
        case 6: inside = force_lc(S, p, qi, t->eps, t->sig, LC_COUL | LC_DIP, 0, &A); dip = 1; break;
      }
    } else {
      switch (ft) {
        case 1: force_all(S, p, qi, t->eps, t->sig, 1, 0, 0, &A); break;
        case 2: inside = force_lc(S, p, qi, t->eps, t->sig, LC_LJ, 0, &A); break;
        case 3: case 5: force_all(S, p, qi, t->eps, t->sig, 1, 1, 0, &A); break;
        case 4: case 6: inside = force_lc(S, p, qi, t->eps, t->sig, LC_LJ | LC_COUL, 0, &A); break;
      }
    }
  } else { /* CO2: carbon (iatom 1) uses the central-site parameters */
    const double *e = iatom == 1 ? t->eps_c : t->eps, *s = iatom == 1 ? t->sig_c : t->sig;
    switch (ft) {
      case 1: force_all(S, p, qi, e, s, 1, 0, 0, &A); break;
      case 2: inside = force_lc(S, p, qi, e, s, LC_LJ, 0, &A); break;
      case 3: force_all(S, p, qi, e, s, 1, 1, 0, &A); break;
      case 4: inside = force_lc(S, p, qi, e, s, LC_LJ | LC_COUL, 0, &A); break;
      case 5:
        if (iatom == 1) { force_all(S, p, qi, e, s, 1, 1, 1, &A); dip = 1; }
        else force_all(S, p, qi, e, s, 1, 1, 0, &A);
        break;
      case 6:
        if (iatom == 1) { inside = force_lc(S, p, qi, e, s, LC_LJ | LC_COUL | LC_DIP, 1, &A); dip = 1; }
        else inside = force_lc(S, p, qi, e, s, LC_LJ | LC_COUL, 0, &A);
        break;
    }
  }
  if (!inside) { f[0] = f[1] = f[2] = 0.0; *U = 0.0; }
  else finish(&A, S->alpha, dip, f, U);
  if (visits) *visits += A.visits;
}

int orc_site_force(const orc_system *S, int iatom, const double pos[3], double f[3], double *U,
                   uint64_t *visits) {
  if (iatom < 0 || iatom >= S->gas.natoms) return -1;
  if (visits) *visits = 0;
  site_force(S, iatom, pos, f, U, visits);
  return 0;
}

/* ---- trajectories (System.cpp) --------------------------------------------- */
/* velDistr / velGenerator (System.cpp:1523-1555) */
static double vel_distr(double v, double m, double temperature) {
  m = m * AMU_TO_KG;
  v = v * ANG_TO_M / FS_TO_S;
  return pow(v, 5.0) * pow((m / (2.0 * BOLTZMANN_K * temperature)), 3.0) *
         exp(-(m * pow(v, 2.0)) / (2.0 * BOLTZMANN_K * temperature));
}
static double vel_generator(double m, double temperature, double sd) {
  double v = 0.0, dv = 1.0E-5;
  double sum = vel_distr(v, m, temperature);
  /* The reference loops without bound; the CDF saturates just below 1 for
   * some masses, so a draw of exactly 1.0 would never end.  Stop at 1e7 steps
   * (1e7 m/s), far beyond any thermal speed. */
  long guard = 0;
  while (sum < sd && guard++ < 10000000L) {
    v += dv;
    sum += vel_distr(v, m, temperature);
  }
  return v;
}
double orc_vel_generator(const orc_system *S, double u) {
  return vel_generator(S->mu, S->in.temp, u);
}

static double kinetic(double m, const double v[3]) { /* System.cpp:1560-1564 */
  return 0.5 * m * dot3(v, v) * AMUANGFS2_TO_KCAL_MOL;
}
static double anglevec(const double vi[3], const double vf[3]) { /* System.cpp:1566-1579 */
  double t1 = dot3(vi, vf), t2 = mod3(vi), t3 = mod3(vf);
  double arg = t1 / (t2 * t3);
  if (fabs(arg) > 1.0) return 0.0;
  return acos(arg);
}
/* rotate (System.cpp:1583-1619): Rz(gamma) Ry(phi) Rz(theta), applied in that order */
static void rotate(double r[3], double v[3], const double ang[3]) {
  double ri[3], vi[3];
  memcpy(ri, r, sizeof ri); memcpy(vi, v, sizeof vi);
  r[0] = ri[0] * cos(ang[0]) - ri[1] * sin(ang[0]);
  r[1] = ri[0] * sin(ang[0]) + ri[1] * cos(ang[0]);
  r[2] = ri[2];
  v[0] = vi[0] * cos(ang[0]) - vi[1] * sin(ang[0]);
  v[1] = vi[0] * sin(ang[0]) + vi[1] * cos(ang[0]);
  v[2] = vi[2];
  memcpy(ri, r, sizeof ri); memcpy(vi, v, sizeof vi);
  r[0] = ri[0] * cos(ang[1]) + ri[2] * sin(ang[1]);
  r[1] = ri[1];
  r[2] = ri[0] * -sin(ang[1]) + ri[2] * cos(ang[1]);
  v[0] = vi[0] * cos(ang[1]) + vi[2] * sin(ang[1]);
  v[1] = vi[1];
  v[2] = vi[0] * -sin(ang[1]) + vi[2] * cos(ang[1]);
  memcpy(ri, r, sizeof ri); memcpy(vi, v, sizeof vi);
  r[0] = ri[0] * cos(ang[2]) - ri[1] * sin(ang[2]);
  r[1] = ri[0] * sin(ang[2]) + ri[1] * cos(ang[2]);
  r[2] = ri[2];
  v[0] = vi[0] * cos(ang[2]) - vi[1] * sin(ang[2]);
  v[1] = vi[0] * sin(ang[2]) + vi[1] * cos(ang[2]);
  v[2] = vi[2];
}
static void rotate_gas(double v[3], double theta, double phi) { /* System.cpp:1624-1638 */
  double vi[3];
  memcpy(vi, v, sizeof vi);
  v[0] = vi[0] * cos(theta) + vi[2] * sin(theta);
  v[1] = vi[1];
  v[2] = vi[0] * -sin(theta) + vi[2] * cos(theta);
  memcpy(vi, v, sizeof vi);
  v[0] = vi[0] * cos(phi) - vi[1] * sin(phi);
  v[1] = vi[0] * sin(phi) + vi[1] * cos(phi);
  v[2] = vi[2];
}

typedef struct {
  double x[3], y[3], z[3], vx[3], vy[3], vz[3];
  double rcm[3], vcm[3];
} probe_t;

/* System::setup (System.cpp:1397-1518). Returns hit. */
static int setup(const orc_system *S, probe_t *P, const double u[9]) {
  const orc_gas *g = &S->gas;
  memset(P, 0, sizeof(*P));
  for (int i = 0; i < g->natoms; i++) { P->x[i] = g->x[i]; P->y[i] = g->y[i]; P->z[i] = g->z[i]; }
  double rcm[3] = {u[0], 0.0, S->bmax};
  double vi = vel_generator(S->mu, S->in.temp, u[1]);
  double vcm[3] = {0.0, 0.0, -vi};
  double ang[3] = {2.0 * PI_D * u[2], asin(2.0 * u[3] - 1.0) + 0.5 * PI_D, 2.0 * PI_D * u[4]};
  rotate(rcm, vcm, ang);
  double ur[3] = {rcm[0] / S->a, rcm[1] / S->b, rcm[2] / S->c};
  double uv[3] = {vcm[0] / S->a, vcm[1] / S->b, vcm[2] / S->c};
  double cr[3];
  cross3(ur, uv, cr);
  double delta = -dot3(cr, cr) + dot3(uv, uv);
  if (delta < 0) return 0;
  double lambda = -dot3(ur, uv) / dot3(uv, uv) - sqrt(delta) / dot3(uv, uv);
  for (int k = 0; k < 3; k++) rcm[k] = rcm[k] + lambda * vcm[k];
  memcpy(P->rcm, rcm, sizeof rcm);
  memcpy(P->vcm, vcm, sizeof vcm);
  int gf = S->in.gas_flag;
  if (gf == 1 || gf == 4 || gf == 5) {
    P->x[0] = rcm[0]; P->y[0] = rcm[1]; P->z[0] = rcm[2];
    P->vx[0] = vcm[0]; P->vy[0] = vcm[1]; P->vz[0] = vcm[2];
  } else {
    double theta = asin(2.0 * u[5] - 1.0) + 0.5 * PI_D;
    double phi = 2.0 * PI_D * u[6];
    double psi = 2.0 * PI_D * u[7];
    double omega = sqrt(2.0 * BOLTZMANN_K * S->in.temp / S->inertia_gas * log(1. / (1. - u[8]))) *
                   OMEGA_TO_FS_INV;
    double w[3] = {omega * cos(psi), omega * sin(psi), 0.0};
    rotate_gas(w, theta, phi);
    for (int i = 0; i < g->natoms; i++) {
      double r[3] = {P->x[i], P->y[i], P->z[i]}, v[3];
      rotate_gas(r, theta, phi);
      P->x[i] = r[0]; P->y[i] = r[1]; P->z[i] = r[2];
      cross3(w, r, v);
      P->vx[i] = v[0]; P->vy[i] = v[1]; P->vz[i] = v[2];
    }
    for (int i = 0; i < g->natoms; i++) {
      P->x[i] += rcm[0]; P->y[i] += rcm[1]; P->z[i] += rcm[2];
      P->vx[i] += vcm[0]; P->vy[i] += vcm[1]; P->vz[i] += vcm[2];
    }
  }
  return 1;
}

int orc_setup_one(const orc_system *S, const double rnd9[9], double pos[9], double vel[9],
                  double rcm[3], double vcm[3]) {
  probe_t P;
  int hit = setup(S, &P, rnd9);
  for (int i = 0; i < 3; i++) {
    pos[3 * i] = P.x[i]; pos[3 * i + 1] = P.y[i]; pos[3 * i + 2] = P.z[i];
    vel[3 * i] = P.vx[i]; vel[3 * i + 1] = P.vy[i]; vel[3 * i + 2] = P.vz[i];
  }
  memcpy(rcm, P.rcm, 3 * sizeof(double));
  memcpy(vcm, P.vcm, 3 * sizeof(double));
  return hit;
}

/* Cap on integration steps per try.  The reference has none (a probe that
 * neither leaves nor winds past 1.5 pi would integrate forever); such a
 * trajectory is reported lost here. */
#define ORC_MAX_STEPS_PER_TRY 2000000L

static int outside(const orc_system *S, const double r[3]) { /* box or ellipsoid exit */
  if (fabs(r[0]) >= S->lx || fabs(r[1]) >= S->ly || fabs(r[2]) >= S->lz) return 1;
  double ur[3] = {r[0] / S->a, r[1] / S->b, r[2] / S->c};
  return dot3(ur, ur) > 1.0;
}

/* run_He (System.cpp:338-511) for He, Ar and the one-site "co2" */
static int run_atom(const orc_system *S, probe_t *P, double *chi, uint32_t *steps, uint64_t *visits) {
  const double time_step = S->in.dt, mu = S->mu, theta_max = 1.5 * PI_D;
  double dt = time_step;
  int maxTries = 8, trajTries = 0;
  double rcm_i[3] = {P->x[0], P->y[0], P->z[0]}, vcm_i[3] = {P->vx[0], P->vy[0], P->vz[0]};
  double rcm[3], vcm[3], rcm_old[3], f[3], fi[3], Up;
  memcpy(rcm, rcm_i, sizeof rcm); memcpy(vcm, vcm_i, sizeof vcm);
  site_force(S, 0, rcm, f, &Up, visits);
  memcpy(fi, f, sizeof f);
  double Ei = Up + kinetic(mu, vcm);
  double dtheta = 0.0;
  long stepcount = 0;
  while (trajTries < maxTries && maxTries < 10) {
    if (stepcount == 0) {
      memcpy(vcm, vcm_i, sizeof vcm); memcpy(rcm, rcm_i, sizeof rcm);
      memcpy(rcm_old, rcm_i, sizeof rcm_old); memcpy(f, fi, sizeof f);
      dtheta = 0.0;
    }
    for (int i = 0; i < 3; i++) {
      vcm[i] += 0.5 * dt / mu * f[i] * KCALMOLANGAMU_TO_ANGFS2;
      rcm[i] += dt * vcm[i];
    }
    dtheta += anglevec(rcm, rcm_old);
    memcpy(rcm_old, rcm, sizeof rcm);
    site_force(S, 0, rcm, f, &Up, visits);
    for (int i = 0; i < 3; i++) vcm[i] += 0.5 * dt / mu * f[i] * KCALMOLANGAMU_TO_ANGFS2;
    stepcount++;
    (*steps)++;
    if (dtheta > theta_max) {
      trajTries++;
      dt = time_step / (trajTries + 1);
      stepcount = 0;
      continue;
    }
    if (outside(S, rcm)) {
      double E = Up + kinetic(mu, vcm);
      double dE = fabs(E - Ei) / Ei * 100.0;
      if (dE > 0.5) {
        trajTries++;
        maxTries++;
        dt = time_step / (trajTries + 1);
        stepcount = 0;
        continue;
      }
      *chi = anglevec(vcm_i, vcm);
      return 1;
    }
    if (stepcount >= ORC_MAX_STEPS_PER_TRY) return 0;
  }
  return 0;
}

/* first/second_half_verlet_constrained (System.cpp:1700-1767) */
static void verlet_c1(double ri[3], double rj[3], double vi[3], double vj[3], const double fi[3],
                      const double fj[3], double mi, double mj, double dt, double d2ij) {
  double muij = mi * mj / (mi + mj);
  double rci[3], rcj[3], vci[3], vcj[3], rcij[3], rij[3];
  for (int i = 0; i < 3; i++) {
    vci[i] = vi[i] + 0.5 * dt / mi * fi[i] * KCALMOLANGAMU_TO_ANGFS2;
    vcj[i] = vj[i] + 0.5 * dt / mj * fj[i] * KCALMOLANGAMU_TO_ANGFS2;
    rci[i] = ri[i] + dt * vci[i];
    rcj[i] = rj[i] + dt * vcj[i];
    rij[i] = ri[i] - rj[i];
    rcij[i] = rci[i] - rcj[i];
  }
  double r2ij = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
  double rc2ij = rcij[0] * rcij[0] + rcij[1] * rcij[1] + rcij[2] * rcij[2];
  double rcijrij = rcij[0] * rij[0] + rcij[1] * rij[1] + rcij[2] * rij[2];
  double determ = rcijrij * rcijrij - r2ij * (rc2ij - d2ij);
  if (determ < 0.0) determ = 0.0;
  double lambda = (rcijrij - sqrt(determ)) / r2ij;
  for (int i = 0; i < 3; i++) {
    vi[i] = vci[i] - muij / (mi * dt) * lambda * rij[i];
    vj[i] = vcj[i] + muij / (mj * dt) * lambda * rij[i];
    ri[i] = rci[i] - muij / mi * lambda * rij[i];
    rj[i] = rcj[i] + muij / mi * lambda * rij[i]; /* the reference uses mi here (:1736) */
  }
}
static void verlet_c2(const double ri[3], const double rj[3], double vi[3], double vj[3],
                      const double fi[3], const double fj[3], double mi, double mj, double dt) {
  double muij = mi * mj / (mi + mj);
  double rij[3], vcij[3], vci[3], vcj[3];
  for (int i = 0; i < 3; i++) {
    vci[i] = vi[i] + 0.5 * dt / mi * fi[i] * KCALMOLANGAMU_TO_ANGFS2;
    vcj[i] = vj[i] + 0.5 * dt / mj * fj[i] * KCALMOLANGAMU_TO_ANGFS2;
    rij[i] = ri[i] - rj[i];
    vcij[i] = vci[i] - vcj[i];
  }
  double rijvcij = rij[0] * vcij[0] + rij[1] * vcij[1] + rij[2] * vcij[2];
  double r2ij = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
  double lambda = muij * rijvcij / r2ij;
  for (int i = 0; i < 3; i++) {
    vi[i] = vci[i] - lambda / mi * rij[i];
    vj[i] = vcj[i] + lambda / mj * rij[i];
  }
}

/* run_N2 (System.cpp:514-945) and run_CO2 (System.cpp:948-1392).
 * N2: constrained pair = sites 0,1; massless dummy charge (site 2) at the COM,
 *     its force split half/half (:736-739); 1 % energy test over sites 0,1.
 * CO2: constrained pair = O sites 0,2; carbon (site 1) at the COM with the
 *     Ciccotti force redistribution (:1154-1158); 20 % energy test over all sites. */
static int run_molecule(const orc_system *S, probe_t *P, int quirks, double *chi, uint32_t *steps,
                        uint64_t *visits) {
  const int co2 = S->in.gas_flag == 3;
  const int na = S->gas.natoms;
  const int pa = 0, pb = co2 ? 2 : 1, pc = co2 ? 1 : 2; /* pair atoms and the centre site */
  const double time_step = S->in.dt, theta_max = 1.5 * PI_D;
  const double *m = S->gas.m, M = S->gas.mass;
  const double tol = co2 ? 20.0 : 1.0;
  const int nke = co2 ? na : na - 1;
  double dt = time_step;
  int maxTries = 8, trajTries = 0;
  double x[3], y[3], z[3], vx[3], vy[3], vz[3], xi[3], yi[3], zi[3], vxi[3], vyi[3], vzi[3];
  for (int i = 0; i < na; i++) {
    x[i] = xi[i] = P->x[i]; y[i] = yi[i] = P->y[i]; z[i] = zi[i] = P->z[i];
    vx[i] = vxi[i] = P->vx[i]; vy[i] = vyi[i] = P->vy[i]; vz[i] = vzi[i] = P->vz[i];
  }
  double rcm_i[3] = {P->rcm[0], P->rcm[1], P->rcm[2]};
  double vcm_i[3] = {P->vcm[0], P->vcm[1], P->vcm[2]};
  if (co2 && (quirks & ORC_QUIRK_CO2_VCM)) vcm_i[0] = P->vcm[1]; /* System.cpp:1012 */
  double rcm[3], vcm[3], rcm_old[3];
  double f_gas[3][3], fi_gas[3][3], Up, Up_gas = 0.0;
  for (int i = 0; i < na; i++) {
    double p[3] = {x[i], y[i], z[i]}, f[3];
    site_force(S, i, p, f, &Up, visits);
    Up_gas += Up;
    for (int k = 0; k < 3; k++) f_gas[i][k] = fi_gas[i][k] = f[k];
  }
  double Ek = 0.0;
  for (int i = 0; i < na; i++) { /* initial KE sums every site (:650-655, :1078-1083) */
    double v[3] = {vx[i], vy[i], vz[i]};
    Ek += kinetic(m[i], v);
  }
  double Ei = Up_gas + Ek;
  double d2ij = S->d_bond * S->d_bond;
  double dtheta = 0.0;
  long stepcount = 0;
  while (trajTries < maxTries && maxTries < 10) {
    if (stepcount == 0) {
      memcpy(vcm, vcm_i, sizeof vcm); memcpy(rcm, rcm_i, sizeof rcm); memcpy(rcm_old, rcm_i, sizeof rcm);
      for (int i = 0; i < na; i++) {
        x[i] = xi[i]; y[i] = yi[i]; z[i] = zi[i]; vx[i] = vxi[i]; vy[i] = vyi[i]; vz[i] = vzi[i];
        for (int k = 0; k < 3; k++) f_gas[i][k] = fi_gas[i][k];
      }
      dtheta = 0.0;
    }
    double ri[3] = {x[pa], y[pa], z[pa]}, vi[3] = {vx[pa], vy[pa], vz[pa]};
    double rj[3] = {x[pb], y[pb], z[pb]}, vj[3] = {vx[pb], vy[pb], vz[pb]};
    double fi[3], fj[3];
    if (co2) {
      double m2M = m[1] / M;
      for (int i = 0; i < 3; i++) {
        fi[i] = (1.0 - 0.5 * m2M) * f_gas[0][i] + m[0] / M * f_gas[1][i] - 0.5 * m2M * f_gas[2][i];
        fj[i] = (1.0 - 0.5 * m2M) * f_gas[2][i] + m[0] / M * f_gas[1][i] - 0.5 * m2M * f_gas[0][i];
      }
    } else {
      for (int i = 0; i < 3; i++) {
        fi[i] = f_gas[0][i] + 0.5 * f_gas[2][i];
        fj[i] = f_gas[1][i] + 0.5 * f_gas[2][i];
      }
    }
    verlet_c1(ri, rj, vi, vj, fi, fj, m[pa], m[pb], dt, d2ij);
    x[pa] = ri[0]; y[pa] = ri[1]; z[pa] = ri[2]; vx[pa] = vi[0]; vy[pa] = vi[1]; vz[pa] = vi[2];
    x[pb] = rj[0]; y[pb] = rj[1]; z[pb] = rj[2]; vx[pb] = vj[0]; vy[pb] = vj[1]; vz[pb] = vj[2];
    for (int i = 0; i < 3; i++) {
      rcm[i] = 0.5 * (ri[i] + rj[i]);
      vcm[i] = 0.5 * (vi[i] + vj[i]);
    }
    x[pc] = rcm[0]; y[pc] = rcm[1]; z[pc] = rcm[2];
    if (co2) { vx[pc] = vcm[0]; vy[pc] = vcm[1]; vz[pc] = vcm[2]; }
    dtheta += anglevec(rcm, rcm_old);
    memcpy(rcm_old, rcm, sizeof rcm);
    Up_gas = 0.0;
    for (int i = 0; i < na; i++) {
      double p[3] = {x[i], y[i], z[i]}, f[3];
      site_force(S, i, p, f, &Up, visits);
      Up_gas += Up;
      for (int k = 0; k < 3; k++) f_gas[i][k] = f[k];
    }
    double ri2[3] = {x[pa], y[pa], z[pa]}, rj2[3] = {x[pb], y[pb], z[pb]};
    double vi2[3] = {vx[pa], vy[pa], vz[pa]}, vj2[3] = {vx[pb], vy[pb], vz[pb]};
    if (co2) {
      double m2M = m[1] / M;
      for (int i = 0; i < 3; i++) {
        fi[i] = (1.0 - 0.5 * m2M) * f_gas[0][i] + m[0] / M * f_gas[1][i] - 0.5 * m2M * f_gas[2][i];
        fj[i] = (1.0 - 0.5 * m2M) * f_gas[2][i] + m[0] / M * f_gas[1][i] - 0.5 * m2M * f_gas[0][i];
      }
    } else {
      for (int i = 0; i < 3; i++) {
        fi[i] = f_gas[0][i] + 0.5 * f_gas[2][i];
        fj[i] = f_gas[1][i] + 0.5 * f_gas[2][i];
      }
    }
    verlet_c2(ri2, rj2, vi2, vj2, fi, fj, m[pa], m[pb], dt);
    vx[pa] = vi2[0]; vy[pa] = vi2[1]; vz[pa] = vi2[2];
    vx[pb] = vj2[0]; vy[pb] = vj2[1]; vz[pb] = vj2[2];
    for (int i = 0; i < 3; i++) vcm[i] = 0.5 * (vi2[i] + vj2[i]);
    if (co2) { vx[pc] = vcm[0]; vy[pc] = vcm[1]; vz[pc] = vcm[2]; }
    stepcount++;
    (*steps)++;
    if (dtheta > theta_max) {
      trajTries++;
      dt = time_step / (trajTries + 1);
      stepcount = 0;
      continue;
    }
    if (outside(S, rcm)) {
      Ek = 0.0;
      for (int i = 0; i < nke; i++) {
        double v[3] = {vx[i], vy[i], vz[i]};
        Ek += kinetic(m[i], v);
      }
      double E = Up_gas + Ek;
      double dE = fabs((E - Ei) / Ei) * 100.0;
      if (dE > tol) {
        trajTries++;
        maxTries++;
        dt = time_step / (trajTries + 1);
        stepcount = 0;
        continue;
      }
      *chi = anglevec(vcm_i, vcm);
      return 1;
    }
    if (stepcount >= ORC_MAX_STEPS_PER_TRY) return 0;
  }
  return 0;
}

void orc_run(const orc_system *S, size_t n, const double *rnd, size_t stride, int quirks,
             int nthreads, int8_t *status, double *one_minus_cos, uint32_t *steps, uint64_t *visits) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  const int atomic = S->gas.natoms == 1;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
  for (long j = 0; j < (long)n; j++) {
    double u[9];
    for (int k = 0; k < 9; k++) u[k] = rnd[(size_t)k * stride + (size_t)j];
    probe_t P;
    double chi = 0.0;
    uint32_t st = 0;
    uint64_t vis = 0;
    int8_t s;
    double omc = 0.0;
    if (!setup(S, &P, u)) s = 0;
    else {
      int ok = atomic ? run_atom(S, &P, &chi, &st, &vis) : run_molecule(S, &P, quirks, &chi, &st, &vis);
      if (ok) { s = 1; omc = 1.0 - cos(chi); }
      else s = 2;
    }
    if (status) status[j] = s;
    if (one_minus_cos) one_minus_cos[j] = omc;
    if (steps) steps[j] = st;
    if (visits) visits[j] = vis;
  }
}

void orc_predraw(const orc_system *S, unsigned seed, size_t ntraj, double *rnd) {
  mt_t m;
  mt_seed(&m, seed);
  const int mol = S->in.gas_flag == 2 || S->in.gas_flag == 3;
  memset(rnd, 0, sizeof(double) * 9 * ntraj);
  for (size_t j = 0; j < ntraj; j++) { /* System.cpp:184-197 */
    rnd[j] = sqrt(S->bmax * S->bmax * mt_uniform(&m));
    for (int k = 1; k < 5; k++) rnd[(size_t)k * ntraj + j] = mt_uniform(&m);
    if (mol)
      for (int k = 5; k < 9; k++) rnd[(size_t)k * ntraj + j] = mt_uniform(&m);
  }
}

void orc_reduce(size_t niter, size_t nprobe, const int8_t *status, const double *omc, double bmax,
                double *omega, int *nfree, int *nscatter, int *nlost, double *ccs, double *err) {
  double Om = 0.0, Om2 = 0.0;
  size_t count = 0;
  for (size_t i = 0; i < niter; i++) {
    double dOmega = 0.0;
    int ns = 0, nf = 0, nl = 0;
    for (size_t j = 0; j < nprobe; j++, count++) {
      if (status[count] == 1) dOmega += PI_D * omc[count] * pow(bmax, 2.0);
      else dOmega += 0.0;
      ns += status[count] == 1;
      nf += status[count] == 0;
      nl += status[count] == 2;
    }
    double w = 1.0 / ((double)(float)(ns + nf)) * dOmega; /* float() as System.cpp:301 */
    Om += w;
    Om2 += pow(w, 2.0);
    if (omega) omega[i] = w;
    if (nfree) nfree[i] = nf;
    if (nscatter) nscatter[i] = ns;
    if (nlost) nlost[i] = nl;
  }
  double ave = Om / niter;
  double sig2 = Om2 / niter - pow(ave, 2.0);
  if (ccs) *ccs = ave;
  if (err) *err = sqrt(sig2 / (double)(float)niter);
}

int orc_run_system(orc_system *S, int nthreads, int quirks, int print, double *ccs_out, double *err_out) {
  size_t niter = S->in.niter, nprobe = S->in.nprobe, n = niter * nprobe;
  double t0 = wall_s();
  double *rnd = malloc(sizeof(double) * 9 * (n > 0 ? n : 1));
  int8_t *st = malloc(n > 0 ? n : 1);
  double *omc = malloc(sizeof(double) * (n > 0 ? n : 1));
  if (!rnd || !st || !omc) { free(rnd); free(st); free(omc); return -1; }
  orc_predraw(S, S->in.seed, n, rnd);
  if (print) {
    printf("*********************************************************\n");
    printf("Trajectory calculations \n");
    printf("*********************************************************\n");
  }
  orc_run(S, n, rnd, n, quirks, nthreads, st, omc, NULL, NULL);
  double *omega = malloc(sizeof(double) * (niter > 0 ? niter : 1));
  int *nf = malloc(sizeof(int) * (niter > 0 ? niter : 1)), *ns = malloc(sizeof(int) * (niter > 0 ? niter : 1)),
      *nl = malloc(sizeof(int) * (niter > 0 ? niter : 1));
  double ccs, err;
  orc_reduce(niter, nprobe, st, omc, S->bmax, omega, nf, ns, nl, &ccs, &err);
  if (print) {
    for (size_t i = 0; i < niter; i++) {
      printf("Ntraj: %i\n", (int)nprobe);
      printf("Nfree: %i\n", nf[i]);
      printf("Nscatter: %i\n", ns[i]);
      printf("Nlost: %i\n", nl[i]);
      printf("omega: %g\n", omega[i]);
    }
    printf("CCS time: %g s\n", wall_s() - t0);
    printf("*********************************************************\n");
    printf("average value of CCS = %g Ang^2\n", ccs);
    printf("error value of CCS = %g Ang^2\n", err);
  }
  if (ccs_out) *ccs_out = ccs;
  if (err_out) *err_out = err;
  free(rnd); free(st); free(omc); free(omega); free(nf); free(ns); free(nl);
  return 0;
}
