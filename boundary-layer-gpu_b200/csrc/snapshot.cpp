// snapshot.cpp -- the reference's files at the C ABI (host code only):
//   .turbb run parameters  params.f90:119-207 through getvar/get_* (miscel.f90:13-262)
//   flow snapshots         read_input_data (input_output.f90:288-487),
//                          output_data (input_output.f90:496-680)
//   Lund restart means     <snapshot>.mean.rescaling (input_output.f90:440-458, 668-676)
// The context-level calls go through the public entry points only.
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <strings.h>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

#include "../../include/blgpu.h"

namespace {

thread_local std::string g_io_error;

int io_err(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_io_error = buf;
  return code;
}

// ---------------------------------------------------------------------------
// .turbb: a key matches a line when the text before the line's first '=',
// without surrounding blanks, equals it; the value is the rest of the line up
// to a '!'; the first matching line wins; lines are read as 256 characters.
// ---------------------------------------------------------------------------
std::string strip(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && s[a] == ' ') ++a;
  while (b > a && s[b - 1] == ' ') --b;
  return s.substr(a, b - a);
}

struct ParamFile {
  std::vector<std::string> lines;
  bool value(const char *key, std::string &out) const {
    for (const std::string &full : lines) {
      const std::string line = full.substr(0, 256);
      const size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      if (strip(line.substr(0, eq)) != key) continue;
      std::string v = line.substr(eq + 1);
      const size_t bang = v.find('!');
      if (bang != std::string::npos) v = v.substr(0, bang);
      out = strip(v);
      return !out.empty();  // a blank value counts as absent, as in getvar's callers
    }
    return false;
  }
};

// list-directed items: separated by blanks or commas, '/' ends the list,
// r*c repeats c r times
bool items(const std::string &s, std::vector<std::string> &out) {
  out.clear();
  size_t i = 0;
  while (i < s.size()) {
    while (i < s.size() && (s[i] == ' ' || s[i] == ',' || s[i] == '\t')) ++i;
    if (i >= s.size() || s[i] == '/') break;
    size_t j = i;
    while (j < s.size() && s[j] != ' ' && s[j] != ',' && s[j] != '\t' && s[j] != '/') ++j;
    std::string tok = s.substr(i, j - i);
    const size_t star = tok.find('*');
    if (star != std::string::npos) {
      char *end = nullptr;
      const long r = strtol(tok.c_str(), &end, 10);
      if (end != tok.c_str() + star || r < 1 || r > 1000000) return false;
      const std::string c = tok.substr(star + 1);
      for (long q = 0; q < r; ++q) out.push_back(c);
    } else {
      out.push_back(tok);
    }
    i = j;
  }
  return true;
}

bool to_double(std::string t, double &v) {
  for (char &c : t)
    if (c == 'd' || c == 'D') c = 'e';
  if (t.empty()) return false;
  char *end = nullptr;
  errno = 0;
  v = strtod(t.c_str(), &end);
  return end == t.c_str() + t.size() && errno == 0;
}

bool to_int(const std::string &t, int &v) {
  if (t.empty()) return false;
  char *end = nullptr;
  errno = 0;
  const long x = strtol(t.c_str(), &end, 10);
  if (end != t.c_str() + t.size() || errno != 0 || x < INT32_MIN || x > INT32_MAX) return false;
  v = (int)x;
  return true;
}

struct Reader {
  const ParamFile &f;
  blgpu_params *p;
  int bit = 0;
  int rc = BLGPU_OK;
  void mark(bool found) {
    if (found) p->found |= 1ull << bit;
    ++bit;
  }
  void dbl(const char *key, double *v, int n = 1) {
    std::string s;
    std::vector<std::string> it;
    const bool f0 = f.value(key, s);
    if (f0 && !rc) {
      if (!items(s, it) || (int)it.size() < n) {
        rc = io_err(BLGPU_EINVAL, ".turbb: %s = '%s': expected %d real value(s)", key, s.c_str(), n);
      } else {
        for (int q = 0; q < n && !rc; ++q)
          if (!to_double(it[q], v[q])) rc = io_err(BLGPU_EINVAL, ".turbb: %s: '%s' is not a real", key, it[q].c_str());
      }
    }
    mark(f0);
  }
  void integer(const char *key, int *v, int n = 1) {
    std::string s;
    std::vector<std::string> it;
    const bool f0 = f.value(key, s);
    if (f0 && !rc) {
      if (!items(s, it) || (int)it.size() < n) {
        rc = io_err(BLGPU_EINVAL, ".turbb: %s = '%s': expected %d integer(s)", key, s.c_str(), n);
      } else {
        for (int q = 0; q < n && !rc; ++q)
          if (!to_int(it[q], v[q])) rc = io_err(BLGPU_EINVAL, ".turbb: %s: '%s' is not an integer", key, it[q].c_str());
      }
    }
    mark(f0);
  }
  void str(const char *key, char *v, size_t cap) {
    std::string s;
    const bool f0 = f.value(key, s);
    if (f0) {
      strncpy(v, s.c_str(), cap - 1);
      v[cap - 1] = '\0';
    }
    mark(f0);
  }
};

// ---------------------------------------------------------------------------
// binary helpers (stream access, as the reference's unformatted stream
// files: native little-endian on x86, or big-endian, below)
// ---------------------------------------------------------------------------
struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

bool rd(FILE *f, void *p, size_t bytes) { return fread(p, 1, bytes, f) == bytes; }
bool wr(FILE *f, const void *p, size_t bytes) { return fwrite(p, 1, bytes, f) == bytes; }

int32_t bswap32(int32_t v) {
  uint32_t u = (uint32_t)v;
  u = (u >> 24) | ((u >> 8) & 0xff00u) | ((u << 8) & 0xff0000u) | (u << 24);
  return (int32_t)u;
}
double bswapd(double v) {
  uint64_t u;
  memcpy(&u, &v, 8);
  u = __builtin_bswap64(u);
  memcpy(&v, &u, 8);
  return v;
}

// Byte order of the unformatted files.  The reference's GPU build runs with
// F_UFMTENDIAN=big (its Makefile exports it), so its snapshots, Lund means
// and inflow profiles are big-endian there and native (little-endian) in
// the CPU build; readers here take either order, writers follow the same
// variable: "big" makes every file big-endian (a unit list after ':' is
// not modelled and leaves the native order).
bool out_swapped() {
  const char *e = getenv("F_UFMTENDIAN");
  return e && strncasecmp(e, "big", 3) == 0 && e[3] == '\0';
}
void swap_n(int32_t *v, size_t n) {
  for (size_t i = 0; i < n; ++i) v[i] = bswap32(v[i]);
}
void swap_n(double *v, size_t n) {
  for (size_t i = 0; i < n; ++i) v[i] = bswapd(v[i]);
}
bool rd_i(FILE *f, int32_t *v, size_t n, bool sw) {
  if (!rd(f, v, n * 4)) return false;
  if (sw) swap_n(v, n);
  return true;
}
bool rd_d(FILE *f, double *v, size_t n, bool sw) {
  if (!rd(f, v, n * 8)) return false;
  if (sw) swap_n(v, n);
  return true;
}
bool wr_i(FILE *f, const int32_t *v, size_t n, bool sw) {
  if (!sw) return wr(f, v, n * 4);
  std::vector<int32_t> t(v, v + n);
  swap_n(t.data(), n);
  return wr(f, t.data(), n * 4);
}
bool wr_d(FILE *f, const double *v, size_t n, bool sw) {
  if (!sw) return wr(f, v, n * 8);
  const size_t chunk = 1 << 16;
  std::vector<double> t(n < chunk ? n : chunk);
  for (size_t i = 0; i < n; i += chunk) {
    const size_t m = n - i < chunk ? n - i : chunk;
    memcpy(t.data(), v + i, m * 8);
    swap_n(t.data(), m);
    if (!wr(f, t.data(), m * 8)) return false;
  }
  return true;
}

struct Layout {
  long long header = 0;                // bytes before the U size record
  int n[3][3] = {};                    // U, V, W dims from their size records
  int planes[5] = {};                  // planes stored of U, V, W, nu_t, P
  bool has_tail = false;               // nu_t and P present
  bool swap = false;                   // big-endian file
};

// the snapshot's header (metadata and mesh) into h and, if non-null, x/y/z
int read_header(FILE *f, bool sw, blgpu_snapshot_info *h, double *x, double *y, double *z, long long *pos) {
  double tn[2];
  int32_t a;
  if (fseek(f, 0, SEEK_SET) != 0 || !rd_d(f, tn, 2, sw) || !rd_i(f, &a, 1, sw))
    return io_err(BLGPU_EINVAL, "snapshot: truncated header");
  h->t = tn[0];
  h->nu = tn[1];
  h->step = -1;
  if (a == -73) {  // magic number, then the step, then nx
    int32_t st;
    if (!rd_i(f, &st, 1, sw) || !rd_i(f, &a, 1, sw)) return io_err(BLGPU_EINVAL, "snapshot: truncated header");
    h->step = st;
  }
  int32_t n[6];
  n[0] = a;
  double *dst[6] = {x, y, z, nullptr, nullptr, nullptr};
  for (int q = 0; q < 6; ++q) {
    if (q > 0 && !rd_i(f, &n[q], 1, sw)) return io_err(BLGPU_EINVAL, "snapshot: truncated mesh record %d", q);
    if (n[q] < 2 || n[q] > (1 << 24)) return io_err(BLGPU_EINVAL, "snapshot: mesh record %d has size %d", q, n[q]);
    const size_t bytes = (size_t)n[q] * 8;
    if (dst[q]) {
      if (!rd_d(f, dst[q], (size_t)n[q], sw)) return io_err(BLGPU_EINVAL, "snapshot: truncated mesh record %d", q);
    } else if (fseek(f, (long)bytes, SEEK_CUR) != 0) {
      return io_err(BLGPU_EINVAL, "snapshot: truncated mesh record %d", q);
    }
  }
  h->nx = n[0];
  h->ny = n[1];
  h->nz = n[2];
  if (n[3] != n[0] - 1 || n[4] != n[1] - 1 || n[5] != n[2] - 1)
    return io_err(BLGPU_EINVAL, "snapshot: centre meshes %d %d %d do not match faces %d %d %d", n[3], n[4], n[5],
                  n[0], n[1], n[2]);
  *pos = ftell(f);
  return BLGPU_OK;
}

// which plane counts the file holds: output_data of one process writes
// n3-1 planes of U, V, W and nu_t (their last z ghost is left out) and all
// planes of P; a file assembled from several processes holds every plane.
int layout(FILE *f, const blgpu_snapshot_info &h, long long pos, Layout &L) {
  const long long nx = h.nx, ny = h.ny, nz = h.nz, nxg = nx + 1, nyg = ny + 1, nzg = nz + 1;
  L.header = pos;
  const long long dims[5][3] = {{nx, nyg, nzg}, {nxg, ny, nzg}, {nxg, nyg, nz}, {nxg, nyg, nzg}, {nxg, nyg, nzg}};
  if (fseek(f, 0, SEEK_END) != 0) return io_err(BLGPU_EINVAL, "snapshot: cannot seek");
  const long long size = ftell(f);
  auto total = [&](int short_planes, int nfields) {
    long long s = pos;
    for (int q = 0; q < nfields; ++q) {
      const long long pl = dims[q][2] - ((short_planes && q < 4) ? 1 : 0);
      s += 12 + dims[q][0] * dims[q][1] * pl * 8;
    }
    return s;
  };
  int sh = -1;
  for (int s = 0; s < 2 && sh < 0; ++s)
    for (int nf : {5, 3})
      if (size == total(s == 0, nf)) {
        sh = (s == 0);
        L.has_tail = (nf == 5);
        break;
      }
  if (sh < 0)
    return io_err(BLGPU_EINVAL, "snapshot: %lld bytes fit neither the one-process (n3-1 planes) nor the full layout "
                  "of a %d x %d x %d box", size, h.nx, h.ny, h.nz);
  for (int q = 0; q < 5; ++q) L.planes[q] = (int)(dims[q][2] - ((sh && q < 4) ? 1 : 0));
  // check the three size records
  long long at = pos;
  for (int q = 0; q < 3; ++q) {
    int32_t r[3];
    if (fseek(f, (long)at, SEEK_SET) != 0 || !rd_i(f, r, 3, L.swap)) return io_err(BLGPU_EINVAL, "snapshot: truncated");
    if (r[0] != dims[q][0] || r[1] != dims[q][1] || r[2] != dims[q][2])
      return io_err(BLGPU_EINVAL, "snapshot: field %d size record %d %d %d, expected %lld %lld %lld", q, r[0], r[1],
                    r[2], dims[q][0], dims[q][1], dims[q][2]);
    for (int e = 0; e < 3; ++e) L.n[q][e] = r[e];
    at += 12 + dims[q][0] * dims[q][1] * (long long)L.planes[q] * 8;
  }
  return BLGPU_OK;
}

// the header and the layout in the byte order that fits the file: native
// first, then swapped (a wrong order gives implausible sizes)
int header_and_layout(FILE *f, blgpu_snapshot_info *h, double *x, double *y, double *z, long long *pos, Layout &L) {
  std::string native_err;
  for (int sw = 0; sw < 2; ++sw) {
    // sizes first (the mesh skipped): the caller's arrays are filled only
    // once the order is known
    blgpu_snapshot_info hh = *h;
    long long p = 0;
    int rc = read_header(f, sw != 0, &hh, nullptr, nullptr, nullptr, &p);
    if (!rc) {
      Layout LL;
      LL.swap = sw != 0;
      rc = layout(f, hh, p, LL);
      if (!rc && (x || y || z)) rc = read_header(f, sw != 0, &hh, x, y, z, &p);
      if (!rc) {
        *h = hh;
        *pos = p;
        L = LL;
        return BLGPU_OK;
      }
    }
    if (!sw) native_err = g_io_error;
  }
  return io_err(BLGPU_EINVAL, "%s", native_err.c_str());
}

// one field: size record then `planes` planes of n1 x n2; a plane left out
// (k = n3) is filled as the z-periodic boundary pass fills it
// (boundary_conditions.f90:204-216): plane 3 for centred fields, 2 for W.
int read_field(FILE *f, long long n1, long long n2, long long n3, long long planes, bool w_face, bool sw, double *dst) {
  if (fseek(f, 12, SEEK_CUR) != 0) return io_err(BLGPU_EINVAL, "snapshot: truncated field");
  const size_t pl = (size_t)(n1 * n2);
  if (!dst) {
    if (fseek(f, (long)(pl * planes * 8), SEEK_CUR) != 0) return io_err(BLGPU_EINVAL, "snapshot: truncated field");
    return BLGPU_OK;
  }
  if (!rd_d(f, dst, pl * planes, sw)) return io_err(BLGPU_EINVAL, "snapshot: truncated field data");
  if (planes < n3) memcpy(dst + pl * (n3 - 1), dst + pl * (w_face ? 1 : 2), pl * 8);
  return BLGPU_OK;
}

int write_field(FILE *f, int n1, int n2, int n3, int planes, bool sw, const double *src) {
  const int32_t r[3] = {n1, n2, n3};
  if (!wr_i(f, r, 3, sw)) return io_err(BLGPU_EINVAL, "snapshot: write failed (%s)", strerror(errno));
  if (src) {
    if (!wr_d(f, src, (size_t)n1 * n2 * planes, sw))
      return io_err(BLGPU_EINVAL, "snapshot: write failed (%s)", strerror(errno));
  } else {
    std::vector<double> zero((size_t)n1 * n2, 0.0);
    for (int k = 0; k < planes; ++k)
      if (!wr(f, zero.data(), zero.size() * 8)) return io_err(BLGPU_EINVAL, "snapshot: write failed (%s)", strerror(errno));
  }
  return BLGPU_OK;
}

// mkdir -p of the directory part of a path (initparams creates the
// parent directory of fileout, params.f90:177-191)
void make_parent(const std::string &path) {
  const size_t slash = path.rfind('/');
  if (slash == std::string::npos || slash == 0) return;
  std::string dir = path.substr(0, slash);
  for (size_t i = 1; i <= dir.size(); ++i) {
    if (i == dir.size() || dir[i] == '/') {
      const std::string part = dir.substr(0, i);
      mkdir(part.c_str(), 0755);
    }
  }
}

}  // namespace

extern "C" {

const char *blgpu_io_last_error(void) { return g_io_error.c_str(); }

int blgpu_read_params(const char *path, blgpu_params *p) {
  if (!path || !p) return io_err(BLGPU_EINVAL, "blgpu_read_params: null argument");
  memset(p, 0, sizeof *p);
  p->init_step = -45;  // input_output.f90:33: "not given"
  FILE *f = fopen(path, "r");
  if (!f) return io_err(BLGPU_EINVAL, "input file: %s does not exist", path);
  ParamFile pf;
  char buf[65536];
  std::string cur;
  while (fgets(buf, sizeof buf, f)) {
    cur += buf;
    if (!cur.empty() && cur.back() == '\n') {
      cur.pop_back();
      if (!cur.empty() && cur.back() == '\r') cur.pop_back();
      pf.lines.push_back(cur);
      cur.clear();
    }
  }
  if (!cur.empty()) pf.lines.push_back(cur);
  fclose(f);
  Reader r{pf, p};
  // in the order of initparams (params.f90:119-197); bit q of p->found is
  // set when the q-th key below was given
  r.dbl("nu", &p->nu);
  r.dbl("CFL", &p->cfl);
  r.dbl("Vmax", &p->vmax);
  r.dbl("x0", &p->x0);
  r.dbl("sigma", &p->sigma);
  r.dbl("phi", &p->phi);
  r.integer("nsteps", &p->nsteps);
  r.integer("nsave", &p->nsave);
  r.integer("nstats", &p->nstats);
  r.integer("nmonitor", &p->nmonitor);
  r.integer("nxyz", p->nxyz, 3);
  r.dbl("boxsize", p->boxsize, 4);
  r.integer("inflow_flag", &p->inflow_flag);
  r.integer("top_flag", &p->top_flag);
  r.str("inflow_file", p->inflow_file, sizeof p->inflow_file);
  r.integer("Lund_ix", &p->lund_ix);
  r.dbl("Lund_deltai", &p->lund_deltai);
  r.dbl("Lund_T", &p->lund_T);
  r.dbl("dPdx", &p->dpdx);
  r.dbl("dPdz", &p->dpdz);
  r.integer("LES", &p->les);
  r.integer("WM", &p->wm);
  r.integer("TauwModel", &p->tauw_model);
  r.integer("nutBC", &p->nut_bc);
  r.integer("WMnutflag", &p->wm_nut_flag);
  r.dbl("WMnut", &p->wm_nut);
  r.dbl("Amplitude", &p->amplitude);
  r.integer("init_step", &p->init_step);
  r.integer("init_rand", &p->init_rand);
  r.str("filein", p->filein, sizeof p->filein);
  r.str("fileout", p->fileout, sizeof p->fileout);
  r.str("timeinflow_file", p->timeinflow_file, sizeof p->timeinflow_file);
  r.integer("RKscheme", &p->rk_scheme);
  r.dbl("alphas", p->alphas, 5);
  if (r.rc) return r.rc;
  // the checks initparams stops on (params.f90:136-139, 166-169)
  if (!(p->found & (1ull << BLGPU_PARAM_INFLOW_FILE)))
    return io_err(BLGPU_EINVAL, "ERROR: you must specify a BL profile in inflow_file");
  if (p->init_rand == 1 && (p->found & (1ull << BLGPU_PARAM_FILEIN)))
    return io_err(BLGPU_EINVAL, "ERROR: init_rand = 1, but filein exists");
  return BLGPU_OK;
}

int blgpu_params_config(const blgpu_params *p, blgpu_config *cfg) {
  if (!p || !cfg) return io_err(BLGPU_EINVAL, "blgpu_params_config: null argument");
  cfg->nx = p->nxyz[0];
  cfg->ny = p->nxyz[1];
  cfg->nz = p->nxyz[2];
  cfg->nu = p->nu;
  cfg->cfl = p->cfl;
  cfg->dpdx = p->dpdx;
  cfg->dpdz = p->dpdz;
  cfg->rk_scheme = p->rk_scheme;
  cfg->les_model = p->les;
  return BLGPU_OK;
}

int blgpu_snapshot_info_read(const char *path, blgpu_snapshot_info *h) {
  if (!path || !h) return io_err(BLGPU_EINVAL, "blgpu_snapshot_info_read: null argument");
  File F;
  F.f = fopen(path, "rb");
  if (!F.f) return io_err(BLGPU_EINVAL, "snapshot %s: cannot open (%s)", path, strerror(errno));
  long long pos = 0;
  Layout L;
  int rc = header_and_layout(F.f, h, nullptr, nullptr, nullptr, &pos, L);
  if (rc) return rc;
  h->full_planes = (L.planes[0] == h->nz + 1) ? 1 : 0;
  h->has_nu_t_p = L.has_tail ? 1 : 0;
  return BLGPU_OK;
}

int blgpu_read_snapshot(const char *path, blgpu_snapshot_info *h, double *x, double *y, double *z, double *U,
                        double *V, double *W, double *nu_t, double *P) {
  if (!path || !h) return io_err(BLGPU_EINVAL, "blgpu_read_snapshot: null argument");
  File F;
  F.f = fopen(path, "rb");
  if (!F.f) return io_err(BLGPU_EINVAL, "snapshot %s: cannot open (%s)", path, strerror(errno));
  long long pos = 0;
  Layout L;
  int rc = header_and_layout(F.f, h, x, y, z, &pos, L);
  if (rc) return rc;
  h->full_planes = (L.planes[0] == h->nz + 1) ? 1 : 0;
  h->has_nu_t_p = L.has_tail ? 1 : 0;
  const long long nx = h->nx, ny = h->ny, nz = h->nz, nxg = nx + 1, nyg = ny + 1, nzg = nz + 1;
  if (fseek(F.f, (long)pos, SEEK_SET) != 0) return io_err(BLGPU_EINVAL, "snapshot: cannot seek");
  if ((rc = read_field(F.f, nx, nyg, nzg, L.planes[0], false, L.swap, U))) return rc;
  if ((rc = read_field(F.f, nxg, ny, nzg, L.planes[1], false, L.swap, V))) return rc;
  if ((rc = read_field(F.f, nxg, nyg, nz, L.planes[2], true, L.swap, W))) return rc;
  if (L.has_tail) {
    if ((rc = read_field(F.f, nxg, nyg, nzg, L.planes[3], false, L.swap, nu_t))) return rc;
    if ((rc = read_field(F.f, nxg, nyg, nzg, L.planes[4], false, L.swap, P))) return rc;
  } else {
    if (nu_t) memset(nu_t, 0, (size_t)(nxg * nyg * nzg) * 8);
    if (P) memset(P, 0, (size_t)(nxg * nyg * nzg) * 8);
  }
  return BLGPU_OK;
}

int blgpu_write_snapshot(const char *path, int nx, int ny, int nz, double t, double nu, int step, const double *x,
                         const double *y, const double *z, const double *U, const double *V, const double *W,
                         const double *nu_t, const double *P) {
  if (!path || !x || !y || !z || !U || !V || !W) return io_err(BLGPU_EINVAL, "blgpu_write_snapshot: null argument");
  if (nx < 3 || ny < 3 || nz < 3) return io_err(BLGPU_EINVAL, "blgpu_write_snapshot: box %d x %d x %d", nx, ny, nz);
  File F;
  F.f = fopen(path, "wb");
  if (!F.f) return io_err(BLGPU_EINVAL, "snapshot %s: cannot create (%s)", path, strerror(errno));
  FILE *f = F.f;
  const bool sw = out_swapped();
  const int nxg = nx + 1, nyg = ny + 1, nzg = nz + 1;
  const double tn[2] = {t, nu};
  const int32_t magic[2] = {-73, step};
  if (!wr_d(f, tn, 2, sw) || !wr_i(f, magic, 2, sw))
    return io_err(BLGPU_EINVAL, "snapshot: write failed (%s)", strerror(errno));
  // faces, then centres xm(i) = (x(i)+x(i+1))/2 (initialization.f90:181-189)
  const double *fc[3] = {x, y, z};
  const int nf[3] = {nx, ny, nz};
  for (int q = 0; q < 3; ++q) {
    const int32_t n = nf[q];
    if (!wr_i(f, &n, 1, sw) || !wr_d(f, fc[q], (size_t)n, sw)) return io_err(BLGPU_EINVAL, "snapshot: write failed");
  }
  for (int q = 0; q < 3; ++q) {
    const int32_t n = nf[q] - 1;
    std::vector<double> m((size_t)n);
    for (int i = 0; i < n; ++i) m[i] = 0.5 * (fc[q][i] + fc[q][i + 1]);
    if (!wr_i(f, &n, 1, sw) || !wr_d(f, m.data(), (size_t)n, sw)) return io_err(BLGPU_EINVAL, "snapshot: write failed");
  }
  int rc;
  if ((rc = write_field(f, nx, nyg, nzg, nzg - 1, sw, U))) return rc;
  if ((rc = write_field(f, nxg, ny, nzg, nzg - 1, sw, V))) return rc;
  if ((rc = write_field(f, nxg, nyg, nz, nz - 1, sw, W))) return rc;
  if ((rc = write_field(f, nxg, nyg, nzg, nzg - 1, sw, nu_t))) return rc;
  if ((rc = write_field(f, nxg, nyg, nzg, nzg, sw, P))) return rc;
  if (fflush(f) != 0) return io_err(BLGPU_EINVAL, "snapshot: write failed (%s)", strerror(errno));
  return BLGPU_OK;
}

int blgpu_read_rescaling(const char *path, int nyg, int ny, double *Umean, double *Vmean) {
  if (!path || !Umean || !Vmean) return io_err(BLGPU_EINVAL, "blgpu_read_rescaling: null argument");
  File F;
  F.f = fopen(path, "rb");
  if (!F.f) return io_err(BLGPU_EINVAL, "%s: cannot open (%s)", path, strerror(errno));
  int32_t n;
  if (!rd(F.f, &n, 4)) return io_err(BLGPU_EINVAL, "%s: truncated", path);
  // written in native order (input_output.f90:671-675), read as big-endian
  // (:445): accept either, told apart by the size record
  bool swap = false;
  if (n != nyg) {
    if (bswap32(n) != nyg) return io_err(BLGPU_EINVAL, "Error! nyg_resc/=nyg_global (%d, %d)", n, nyg);
    swap = true;
  }
  if (!rd(F.f, Umean, (size_t)nyg * 8) || !rd(F.f, Vmean, (size_t)ny * 8))
    return io_err(BLGPU_EINVAL, "%s: truncated", path);
  if (swap) {
    for (int j = 0; j < nyg; ++j) Umean[j] = bswapd(Umean[j]);
    for (int j = 0; j < ny; ++j) Vmean[j] = bswapd(Vmean[j]);
  }
  return BLGPU_OK;
}

// Inflow profile of inflow flags 2 and 5 (boundary_conditions.f90:1405-1413,
// 1550-1558): a stream file holding ny (int32), U_inlet (ny+1 doubles, at
// the centres yg) and V_inlet (ny doubles, at the faces y).  The reference
// reads it in the byte order its runtime is set to (the GPU build exports
// F_UFMTENDIAN=big); the files it ships are of both orders, so the size
// record tells them apart.  The file's ny must equal the grid's, as there.
static int inflow_open(const char *path, File &F, int32_t *n, bool *swap) {
  F.f = fopen(path, "rb");
  if (!F.f) return io_err(BLGPU_EINVAL, "%s: cannot open (%s)", path, strerror(errno));
  if (!rd(F.f, n, 4)) return io_err(BLGPU_EINVAL, "%s: truncated", path);
  if (fseek(F.f, 0, SEEK_END) != 0) return io_err(BLGPU_EINVAL, "%s: cannot seek", path);
  const long size = ftell(F.f);
  if (fseek(F.f, 4, SEEK_SET) != 0) return io_err(BLGPU_EINVAL, "%s: cannot seek", path);
  // the order whose ny makes the file 4 + 8 (2 ny + 1) bytes long
  const auto fits = [size](int32_t v) { return v > 0 && v < (1 << 24) && size == 4 + 8 * (2L * v + 1); };
  *swap = false;
  if (!fits(*n)) {
    if (!fits(bswap32(*n))) return io_err(BLGPU_EINVAL, "%s: not an inflow profile (%ld bytes)", path, size);
    *n = bswap32(*n);
    *swap = true;
  }
  return BLGPU_OK;
}

int blgpu_read_inflow_profile_info(const char *path, int *ny) {
  if (!path || !ny) return io_err(BLGPU_EINVAL, "blgpu_read_inflow_profile_info: null argument");
  File F;
  int32_t n;
  bool swap;
  int rc = inflow_open(path, F, &n, &swap);
  if (rc) return rc;
  *ny = n;
  return BLGPU_OK;
}

int blgpu_read_inflow_profile(const char *path, int ny, double *U_inlet, double *V_inlet) {
  if (!path || !U_inlet || !V_inlet) return io_err(BLGPU_EINVAL, "blgpu_read_inflow_profile: null argument");
  File F;
  int32_t n;
  bool swap;
  int rc = inflow_open(path, F, &n, &swap);
  if (rc) return rc;
  if (n != ny) return io_err(BLGPU_EINVAL, "Profile doesnt match dimensions %d %d", n, ny);
  if (!rd(F.f, U_inlet, (size_t)(ny + 1) * 8) || !rd(F.f, V_inlet, (size_t)ny * 8))
    return io_err(BLGPU_EINVAL, "%s: truncated", path);
  if (swap) {
    for (int j = 0; j <= ny; ++j) U_inlet[j] = bswapd(U_inlet[j]);
    for (int j = 0; j < ny; ++j) V_inlet[j] = bswapd(V_inlet[j]);
  }
  return BLGPU_OK;
}

int blgpu_write_rescaling(const char *path, int nyg, int ny, const double *Umean, const double *Vmean) {
  if (!path || !Umean || !Vmean) return io_err(BLGPU_EINVAL, "blgpu_write_rescaling: null argument");
  File F;
  F.f = fopen(path, "wb");
  if (!F.f) return io_err(BLGPU_EINVAL, "%s: cannot create (%s)", path, strerror(errno));
  const int32_t n = nyg;
  const bool sw = out_swapped();
  if (!wr_i(F.f, &n, 1, sw) || !wr_d(F.f, Umean, (size_t)nyg, sw) || !wr_d(F.f, Vmean, (size_t)ny, sw))
    return io_err(BLGPU_EINVAL, "%s: write failed (%s)", path, strerror(errno));
  return BLGPU_OK;
}

int blgpu_snapshot_name(const char *fileout, int step, char *name, int cap) {
  if (!fileout || !name || cap < 1) return io_err(BLGPU_EINVAL, "blgpu_snapshot_name: null argument");
  // Write(ext,'(I0.8)') istep + nstep_init (input_output.f90:516-518)
  char ext[32];
  snprintf(ext, sizeof ext, "%08d", step);
  const std::string s = strip(fileout) + "." + ext;
  if ((int)s.size() >= cap) return io_err(BLGPU_EINVAL, "blgpu_snapshot_name: buffer of %d too small", cap);
  memcpy(name, s.c_str(), s.size() + 1);
  return BLGPU_OK;
}

int blgpu_output_data(blgpu_ctx *ctx, const char *fileout, int step, int rescaling) {
  if (!ctx || !fileout) return io_err(BLGPU_EINVAL, "blgpu_output_data: null argument");
  int nx, ny, nz;
  double nu;
  if (blgpu_box(ctx, &nx, &ny, &nz, &nu)) return io_err(BLGPU_ESTATE, "%s", blgpu_last_error(ctx));
  const long long nxg = nx + 1, nyg = ny + 1, nzg = nz + 1;
  std::vector<double> x(nx), y(ny), z(nz);
  std::vector<double> U((size_t)(nx * nyg * nzg)), V((size_t)(nxg * ny * nzg)), W((size_t)(nxg * nyg * nz));
  std::vector<double> P((size_t)(nxg * nyg * nzg)), nt((size_t)(nxg * nyg * nzg));
  double t = 0;
  int rc = blgpu_get_grid(ctx, x.data(), y.data(), z.data());
  if (!rc) rc = blgpu_download_state(ctx, U.data(), V.data(), W.data(), P.data(), &t);
  if (!rc) rc = blgpu_get_nu_t(ctx, nt.data());
  if (rc) return io_err(rc, "%s", blgpu_last_error(ctx));
  char name[4096];
  if ((rc = blgpu_snapshot_name(fileout, step, name, sizeof name))) return rc;
  make_parent(name);
  rc = blgpu_write_snapshot(name, nx, ny, nz, t, nu, step, x.data(), y.data(), z.data(), U.data(), V.data(),
                            W.data(), nt.data(), P.data());
  if (rc) return rc;
  // fileout.restart -> the new snapshot (input_output.f90:640-655)
  const std::string link = strip(fileout) + ".restart";
  unlink(link.c_str());
  if (symlink(name, link.c_str()) != 0)
    return io_err(BLGPU_EINVAL, "%s: cannot link to %s (%s)", link.c_str(), name, strerror(errno));
  if (rescaling) {
    std::vector<double> um((size_t)nyg), vm((size_t)ny);
    if ((rc = blgpu_get_rescaling(ctx, um.data(), vm.data(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                  nullptr)))
      return io_err(rc, "%s", blgpu_last_error(ctx));
    const std::string rn = std::string(name) + ".mean.rescaling";
    if ((rc = blgpu_write_rescaling(rn.c_str(), (int)nyg, ny, um.data(), vm.data()))) return rc;
  }
  return BLGPU_OK;
}

// ---------------------------------------------------------------------------
// output_statistics (input_output.f90:685-746): the text file
// <fileout>.<istep+nstep_init, 8 digits>.stats.txt holding, in Fortran list
// formats, '%', t, nu (F15.8), nx, ny, nz, istep (I8); Cf and x (nx values,
// F15.8, one record each); y (ny values); then Umean, Vmean, Wmean, U2mean,
// V2mean, W2mean, Pmean, P2mean as nx records of ny values.
// ---------------------------------------------------------------------------
namespace {
// Fortran Fw.d: right-justified in w columns, w asterisks when it does not
// fit; NaN and infinities as the gfortran runtime spells them
void put_f(std::string &out, double v, int w = 15, int d = 8) {
  char b[64];
  int n;
  if (v != v) n = snprintf(b, sizeof b, "%*s", w, "NaN");
  else if (v == INFINITY || v == -INFINITY) n = snprintf(b, sizeof b, "%*s", w, v > 0 ? "Infinity" : "-Infinity");
  else n = snprintf(b, sizeof b, "%*.*f", w, d, v);
  if (n > w) out.append((size_t)w, '*');
  else out.append(b, (size_t)n);
}
void put_i(std::string &out, long long v, int w = 8) {
  char b[64];
  const int n = snprintf(b, sizeof b, "%*lld", w, v);
  if (n > w) out.append((size_t)w, '*');
  else out.append(b, (size_t)n);
}
}  // namespace

int blgpu_write_statistics(const char *path, double t, double nu, int nx, int ny, int nz, int istep,
                           const double *Cf, const double *x, const double *y, const double *means) {
  if (!path || !Cf || !x || !y || !means) return io_err(BLGPU_EINVAL, "blgpu_write_statistics: null argument");
  if (nx < 1 || ny < 1) return io_err(BLGPU_EINVAL, "blgpu_write_statistics: box %d x %d", nx, ny);
  std::string out;
  out.reserve((size_t)(nx + 2) * (ny + 2) * 15 * 8 / 7);
  out += '%';
  put_f(out, t);
  put_f(out, nu);
  put_i(out, nx);
  put_i(out, ny);
  put_i(out, nz);
  put_i(out, istep);
  out += '\n';
  for (int i = 0; i < nx; ++i) put_f(out, Cf[i]);
  out += '\n';
  for (int i = 0; i < nx; ++i) put_f(out, x[i]);
  out += '\n';
  for (int j = 0; j < ny; ++j) put_f(out, y[j]);
  out += '\n';
  // means: Umean, Vmean, Wmean, U2mean, V2mean, W2mean, UVmean, Pmean, P2mean,
  // each (nx, ny) in Fortran order; the file leaves UVmean out
  const long long plane = (long long)nx * ny;
  for (int q : {0, 1, 2, 3, 4, 5, 7, 8}) {
    const double *a = means + q * plane;
    for (int i = 0; i < nx; ++i) {
      for (int j = 0; j < ny; ++j) put_f(out, a[i + (long long)nx * j]);
      out += '\n';
    }
  }
  File F;
  F.f = fopen(path, "w");
  if (!F.f) return io_err(BLGPU_EINVAL, "%s: cannot create (%s)", path, strerror(errno));
  if (!wr(F.f, out.data(), out.size()) || fflush(F.f) != 0)
    return io_err(BLGPU_EINVAL, "%s: write failed (%s)", path, strerror(errno));
  return BLGPU_OK;
}

int blgpu_output_statistics(blgpu_ctx *ctx, const char *fileout, int istep, int nstep_init) {
  if (!ctx || !fileout) return io_err(BLGPU_EINVAL, "blgpu_output_statistics: null argument");
  int nx, ny, nz;
  double nu, t, dt;
  if (blgpu_box(ctx, &nx, &ny, &nz, &nu) || blgpu_get_time(ctx, &t, &dt))
    return io_err(BLGPU_ESTATE, "%s", blgpu_last_error(ctx));
  std::vector<double> means((size_t)9 * nx * ny), Cf((size_t)nx), x((size_t)nx), y((size_t)ny), z((size_t)nz);
  int rc = blgpu_statistics(ctx, means.data(), nullptr, Cf.data(), nullptr, nullptr);
  if (!rc) rc = blgpu_get_grid(ctx, x.data(), y.data(), z.data());
  if (rc) return io_err(rc, "%s", blgpu_last_error(ctx));
  char name[4096];
  if ((rc = blgpu_snapshot_name(fileout, istep + nstep_init, name, sizeof name))) return rc;
  const std::string fn = std::string(name) + ".stats.txt";
  make_parent(fn);
  return blgpu_write_statistics(fn.c_str(), t, nu, nx, ny, nz, istep, Cf.data(), x.data(), y.data(), means.data());
}

int blgpu_read_input_data(blgpu_ctx *ctx, const char *filein, int *step) {
  if (!ctx || !filein) return io_err(BLGPU_EINVAL, "blgpu_read_input_data: null argument");
  int nx, ny, nz;
  double nu;
  if (blgpu_box(ctx, &nx, &ny, &nz, &nu)) return io_err(BLGPU_ESTATE, "%s", blgpu_last_error(ctx));
  const std::string path = strip(filein);
  blgpu_snapshot_info h{};
  int rc = blgpu_snapshot_info_read(path.c_str(), &h);
  if (rc) return rc;
  // size checks of read_input_data (input_output.f90:321-348)
  if (h.nx != nx) return io_err(BLGPU_EINVAL, "nx_f(%5d)/=nx(%5d)", h.nx, nx);
  if (h.ny != ny) return io_err(BLGPU_EINVAL, "ny_f(%5d)/=ny(%5d)", h.ny, ny);
  if (h.nz != nz) return io_err(BLGPU_EINVAL, "nz_f(%5d)/=nz(%5d)", h.nz, nz);
  const long long nxg = nx + 1, nyg = ny + 1, nzg = nz + 1;
  std::vector<double> x(nx), y(ny), z(nz);
  std::vector<double> U((size_t)(nx * nyg * nzg)), V((size_t)(nxg * ny * nzg)), W((size_t)(nxg * nyg * nz));
  if ((rc = blgpu_read_snapshot(path.c_str(), &h, x.data(), y.data(), z.data(), U.data(), V.data(), W.data(),
                                nullptr, nullptr)))
    return rc;
  // the NaN check of read_input_data (input_output.f90:480-484)
  for (const std::vector<double> *a : {&U, &V, &W})
    for (double v : *a)
      if (v != v) return io_err(BLGPU_EINVAL, "Error %c NaNs!", a == &U ? 'U' : a == &V ? 'V' : 'W');
  // the grid of the file replaces the context's (initialization.f90:171-190)
  rc = blgpu_set_grid(ctx, x.data(), y.data(), z.data());
  if (!rc) rc = blgpu_upload_state(ctx, U.data(), V.data(), W.data(), h.t);
  if (rc) return io_err(rc, "%s", blgpu_last_error(ctx));
  if (step) *step = h.step;
  return BLGPU_OK;
}

// ---------------------------------------------------------------------------
// Temporal inflow modes (the inflow_flag = 1 branch of
// compute_blasius_solution_for_bc, boundary_conditions.f90:1652-1797).  The
// file is a stream (native order, or big-endian as the GPU build's runtime
// reads it, told apart by the sizes): ny_inlet, n, m (int32), beta, omega (f64),
// ymesh(ny_inlet), zmode(n), tmode(m), then qu_r, qu_i, qv_r, qv_i, qw_r,
// qw_i, each (ny_inlet, n, m) in Fortran order.
// ---------------------------------------------------------------------------
// the header in the byte order whose sizes fit the file (native first)
static int modes_header(const char *path, blgpu_modes_info *h, bool *swap) {
  FILE *f = fopen(path, "rb");
  if (!f) return io_err(BLGPU_EINVAL, "cannot open %s: %s", path, strerror(errno));
  int32_t iv0[3];
  double dv0[2];
  const bool ok = rd(f, iv0, sizeof iv0) && rd(f, dv0, sizeof dv0);
  fseek(f, 0, SEEK_END);
  const long long size = ftell(f);
  fclose(f);
  if (!ok) return io_err(BLGPU_EINVAL, "%s: short header", path);
  for (int sw = 0; sw < 2; ++sw) {
    int32_t iv[3] = {iv0[0], iv0[1], iv0[2]};
    double dv[2] = {dv0[0], dv0[1]};
    if (sw) {
      swap_n(iv, 3);
      swap_n(dv, 2);
    }
    if (iv[0] < 2 || iv[1] < 1 || iv[2] < 1 || iv[0] > (1 << 24) || iv[1] > 4096 || iv[2] > 4096) {
      if (!sw) io_err(BLGPU_EINVAL, "%s: implausible sizes ny_inlet %d, n %d, m %d", path, iv[0], iv[1], iv[2]);
      continue;
    }
    const long long nq = (long long)iv[0] * iv[1] * iv[2];
    const long long want = 12 + 16 + 8LL * (iv[0] + iv[1] + iv[2]) + 6 * 8 * nq;
    if (size != want) {
      if (!sw) io_err(BLGPU_EINVAL, "%s: %lld bytes, the header's sizes need %lld", path, size, want);
      continue;
    }
    h->ny_inlet = iv[0];
    h->n_modes = iv[1];
    h->m_modes = iv[2];
    h->beta = dv[0];
    h->omega = dv[1];
    *swap = sw != 0;
    return BLGPU_OK;
  }
  return BLGPU_EINVAL;  // the native order's message stands
}

int blgpu_read_temporal_modes_info(const char *path, blgpu_modes_info *h) {
  if (!path || !h) return io_err(BLGPU_EINVAL, "blgpu_read_temporal_modes_info: null argument");
  bool swap = false;
  return modes_header(path, h, &swap);
}

int blgpu_read_temporal_modes(const char *path, int ny, const double *y, double *zmode, double *tmode, double *qu,
                              double *qv, double *qw, double *ymesh) {
  if (!path) return io_err(BLGPU_EINVAL, "blgpu_read_temporal_modes: null argument");
  blgpu_modes_info h{};
  bool swap = false;
  int rc = modes_header(path, &h, &swap);
  if (rc) return rc;
  if (!y || ny < 3 || !zmode || !tmode || !qu || !qv || !qw)
    return io_err(BLGPU_EINVAL, "blgpu_read_temporal_modes: bad argument");
  for (int j = 1; j < ny; ++j)
    if (!(y[j] > y[j - 1])) return io_err(BLGPU_EINVAL, "blgpu_read_temporal_modes: y not increasing at %d", j + 1);
  const int nyi = h.ny_inlet, n = h.n_modes, m = h.m_modes;
  const long long nq = (long long)nyi * n * m;
  std::vector<double> ym(nyi), zm(n), tm(m), q(6 * nq);
  FILE *f = fopen(path, "rb");
  if (!f) return io_err(BLGPU_EINVAL, "cannot open %s: %s", path, strerror(errno));
  fseek(f, 28, SEEK_SET);
  const bool ok = rd_d(f, ym.data(), nyi, swap) && rd_d(f, zm.data(), n, swap) && rd_d(f, tm.data(), m, swap) &&
                  rd_d(f, q.data(), 6 * nq, swap);
  fclose(f);
  if (!ok) return io_err(BLGPU_EINVAL, "%s: short read", path);
  for (int a = 0; a < n; ++a) zmode[a] = h.beta * zm[a];   // zmode_inlet = beta_inlet*zmode_inlet
  for (int b = 0; b < m; ++b) tmode[b] = h.omega * tm[b];  // tmode_inlet = omega_inlet*tmode_inlet
  if (ymesh)
    for (int j = 0; j < nyi; ++j) ymesh[j] = ym[j];
  // centres with mirrored ghosts (initialization.f90:174-222): yg(1..ny+1)
  const int nyg = ny + 1;
  std::vector<double> yc(ny - 1), yg(nyg);
  for (int j = 0; j < ny - 1; ++j) yc[j] = 0.5 * (y[j] + y[j + 1]);
  for (int j = 0; j < ny - 1; ++j) yg[j + 1] = yc[j];
  yg[0] = yc[0] - 2.0 * (yc[0] - y[0]);
  yg[ny] = yc[ny - 2] + 2.0 * (y[ny - 1] - yc[ny - 2]);
  // linear interpolation of the modes onto target rows (boundary_conditions.f90:1730-1774):
  // j1 = first jj >= 2 with ymesh(jj) >= target, else ny_inlet; rows at or past the
  // mesh end are zero
  auto interp = [&](const double *re, const double *im, const std::vector<double> &tgt, double *out) {
    const int nt = (int)tgt.size();
    for (int j = 0; j < nt; ++j) {
      int j1 = nyi;  // 1-based
      for (int jj = 2; jj <= nyi; ++jj)
        if (ym[jj - 1] >= tgt[j]) {
          j1 = jj;
          break;
        }
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < m; ++b) {
          double *o = out + 2 * ((long long)j + (long long)nt * (a + (long long)n * b));
          if (j1 == nyi) {
            o[0] = o[1] = 0.0;
            continue;
          }
          const int j0 = j1 - 1;
          const long long i0 = (j0 - 1) + (long long)nyi * (a + (long long)n * b), i1 = i0 + 1;
          // q(j0) + (y - ymesh(j0)) (q(j1) - q(j0)) / (ymesh(j1) - ymesh(j0)), per component
          const double dy = tgt[j] - ym[j0 - 1], span = ym[j1 - 1] - ym[j0 - 1];
          o[0] = re[i0] + dy * (re[i1] - re[i0]) / span;
          o[1] = im[i0] + dy * (im[i1] - im[i0]) / span;
        }
    }
  };
  std::vector<double> yv(y, y + ny);
  interp(q.data(), q.data() + nq, yg, qu);
  interp(q.data() + 2 * nq, q.data() + 3 * nq, yv, qv);
  interp(q.data() + 4 * nq, q.data() + 5 * nq, yg, qw);
  return BLGPU_OK;
}

}  // extern "C"
