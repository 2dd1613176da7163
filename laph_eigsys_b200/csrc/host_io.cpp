// host_io.cpp -- host-side parts of liblaph_gpu.so that need no device:
// synthetic gauge fields, LIME/ILDG gauge I/O, eigensystem files, the
// parameters.txt parser, check_trace / fix_phase / recover_spectrum.
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <errno.h>
#include <sys/stat.h>
#include <omp.h>
#include <unistd.h>
#endif

#include "../../include/laph_gpu.h"

namespace laph {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

namespace {

typedef std::complex<double> cd;

// ---------------------------------------------------------- SU(3) (host) ---
struct HM3 {
  cd e[9];
};
HM3 hmul(const HM3& a, const HM3& b) {
  HM3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.e[3 * i + j] = a.e[3 * i] * b.e[j] + a.e[3 * i + 1] * b.e[3 + j] + a.e[3 * i + 2] * b.e[6 + j];
  return r;
}
HM3 hadj(const HM3& a) {
  HM3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.e[3 * i + j] = std::conj(a.e[3 * j + i]);
  return r;
}
HM3 hid() {
  HM3 r;
  for (int i = 0; i < 9; ++i) r.e[i] = 0.0;
  r.e[0] = r.e[4] = r.e[8] = 1.0;
  return r;
}
// Hermitian 3x3 Jacobi eigendecomposition (same rotation as the device code).
void heig3(HM3 A, double d[3], HM3& Q) {
  Q = hid();
  const int P[3] = {0, 0, 1}, QQ[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 12; ++sweep) {
    double off = std::norm(A.e[1]) + std::norm(A.e[2]) + std::norm(A.e[5]);
    double dg = std::norm(A.e[0]) + std::norm(A.e[4]) + std::norm(A.e[8]);
    if (off <= 1e-34 * dg || off == 0.0) break;
    for (int k = 0; k < 3; ++k) {
      const int p = P[k], q = QQ[k];
      const cd g = A.e[3 * p + q];
      const double r = std::abs(g);
      if (r == 0.0) continue;
      const cd emph = std::conj(g / r);
      const double tau = (A.e[4 * q].real() - A.e[4 * p].real()) / (2.0 * r);
      const double t = (tau >= 0.0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
      const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
      HM3 J = hid();
      J.e[3 * p + p] = c;
      J.e[3 * p + q] = s;
      J.e[3 * q + p] = -s * emph;
      J.e[3 * q + q] = c * emph;
      A = hmul(hadj(J), hmul(A, J));
      A.e[3 * p + q] = A.e[3 * q + p] = 0.0;
      Q = hmul(Q, J);
    }
  }
  for (int i = 0; i < 3; ++i) d[i] = A.e[4 * i].real();
}

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

void put_be64(unsigned char* p, uint64_t v) {
  for (int i = 7; i >= 0; --i) {
    p[i] = (unsigned char)(v & 0xff);
    v >>= 8;
  }
}
uint64_t get_be64(const unsigned char* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; ++i) v = v << 8 | p[i];
  return v;
}

// LIME record header: magic 0x456789ab, version 1, MB/ME bits, 64-bit
// length, 128-byte type string; all big-endian; payload padded to 8 bytes.
void lime_header(unsigned char h[144], bool mb, bool me, uint64_t len, const char* type) {
  std::memset(h, 0, 144);
  h[0] = 0x45; h[1] = 0x67; h[2] = 0x89; h[3] = 0xab;
  h[4] = 0; h[5] = 1;
  uint16_t flags = (mb ? 0x8000 : 0) | (me ? 0x4000 : 0);
  h[6] = (unsigned char)(flags >> 8);
  h[7] = (unsigned char)(flags & 0xff);
  put_be64(h + 8, len);
  std::strncpy(reinterpret_cast<char*>(h + 16), type, 127);
}

}  // namespace
}  // namespace laph

using namespace laph;

extern "C" {

const char* laph_last_error(void) { return g_err; }

const char* laph_strerror(int s) {
  switch (s) {
    case LAPH_OK: return "ok";
    case LAPH_EINVAL: return "invalid argument";
    case LAPH_ECUDA: return "CUDA error";
    case LAPH_ENOMEM: return "out of memory";
    case LAPH_EIO: return "I/O error";
    case LAPH_ENORECORD: return "no ildg-binary-data record";
    case LAPH_ESIZE: return "record size does not match the lattice";
    case LAPH_ESINGLE: return "single-precision ILDG data not implemented";
    case LAPH_ENOTCONV: return "eigensolver did not converge";
    case LAPH_ETIMEOUT: return "device wait timed out";
    case LAPH_ETRACE: return "tr(V^dag V) check failed";
    case LAPH_EPARSE: return "parse error (parameters.txt or ildg-format record)";
    case LAPH_ENODEV: return "no CUDA device";
    default: return "unknown status";
  }
}

int laph_version(void) { return 100; }

int laph_gauge_random(double* conf, int L, int nt, double eps, uint64_t seed) {
  if (!conf || L < 1 || nt < 1) {
    set_error("laph_gauge_random: bad argument");
    return LAPH_EINVAL;
  }
  const long long V3 = (long long)L * L * L;
  const long long nlinks = V3 * nt * 4;
  const double is3 = 1.0 / std::sqrt(3.0);
#pragma omp parallel for schedule(static)
  for (long long n = 0; n < nlinks; ++n) {
    // counter-based stream: link n draws 8 normals (4 Box-Muller pairs)
    uint64_t st = seed * 0x9E3779B97F4A7C15ULL + (uint64_t)n * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL;
    double c[8];
    for (int k = 0; k < 4; ++k) {
      st += 0x9E3779B97F4A7C15ULL;
      const double u1 = ((mix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      st += 0x9E3779B97F4A7C15ULL;
      const double u2 = ((mix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      const double r = std::sqrt(-2.0 * std::log(u1));
      c[2 * k] = r * std::cos(2.0 * M_PI * u2);
      c[2 * k + 1] = r * std::sin(2.0 * M_PI * u2);
    }
    // H = sum_a c_a lambda_a (Gell-Mann)
    HM3 H;
    H.e[0] = c[2] + c[7] * is3;
    H.e[4] = -c[2] + c[7] * is3;
    H.e[8] = -2.0 * c[7] * is3;
    H.e[1] = cd(c[0], -c[1]);
    H.e[3] = cd(c[0], c[1]);
    H.e[2] = cd(c[3], -c[4]);
    H.e[6] = cd(c[3], c[4]);
    H.e[5] = cd(c[5], -c[6]);
    H.e[7] = cd(c[5], c[6]);
    double d[3];
    HM3 Q;
    heig3(H, d, Q);
    // U = Q diag(e^{i eps d}) Q^dag
    cd f[3];
    for (int i = 0; i < 3; ++i) f[i] = cd(std::cos(eps * d[i]), std::sin(eps * d[i]));
    double* out = conf + n * 18;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        cd s = 0.0;
        for (int k = 0; k < 3; ++k) s += Q.e[3 * i + k] * f[k] * std::conj(Q.e[3 * j + k]);
        out[2 * (3 * i + j)] = s.real();
        out[2 * (3 * i + j) + 1] = s.imag();
      }
  }
  return LAPH_OK;
}

int laph_lime_write_gauge_prec(const char* path, const double* conf, int L, int T, int precision) {
  if (!path || !conf || L < 1 || T < 1 || (precision != 32 && precision != 64)) {
    set_error("laph_lime_write_gauge_prec: bad argument (precision must be 32 or 64)");
    return LAPH_EINVAL;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("cannot open %s for writing", path);
    return LAPH_EIO;
  }
  char xml[1024];
  std::snprintf(xml, sizeof xml,
                "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n<ildgFormat xmlns=\"http://www.lqcd.org/ildg\" "
                "xmlns:xsi=\"http://www.w3.org/2001/XMLSchema-instance\" "
                "xsi:schemaLocation=\"http://www.lqcd.org/ildg http://www.lqcd.org/ildg/filefmt.xsd\">\n"
                "  <version>1.0</version>\n  <field>su3gauge</field>\n  <precision>%d</precision>\n"
                "  <lx>%d</lx>\n  <ly>%d</ly>\n  <lz>%d</lz>\n  <lt>%d</lt>\n</ildgFormat>\n",
                precision, L, L, L, T);
  const uint64_t xl = std::strlen(xml);
  unsigned char h[144];
  static const unsigned char pad[8] = {0};
  lime_header(h, true, false, xl, "ildg-format");
  bool ok = std::fwrite(h, 1, 144, f) == 144 && std::fwrite(xml, 1, xl, f) == xl;
  if (ok && xl % 8) ok = std::fwrite(pad, 1, 8 - xl % 8, f) == 8 - xl % 8;
  const long long V3 = (long long)L * L * L;
  const int es = precision / 8;
  const uint64_t dl = (uint64_t)V3 * T * 72ull * es;
  lime_header(h, false, true, dl, "ildg-binary-data");
  ok = ok && std::fwrite(h, 1, 144, f) == 144;
  std::vector<unsigned char> buf((size_t)L * 72 * es);
  static const int slot_of_mu[4] = {1, 2, 3, 0};  // ILDG mu order x,y,z,t
  for (int t = 0; ok && t < T; ++t)
    for (int z = 0; ok && z < L; ++z)
      for (int y = 0; ok && y < L; ++y) {
        for (int x = 0; x < L; ++x) {
          const double* site = conf + ((long long)t * V3 + (long long)x * L * L + (long long)y * L + z) * 72;
          for (int mu = 0; mu < 4; ++mu)
            for (int k = 0; k < 18; ++k) {
              unsigned char* o = &buf[((size_t)x * 72 + mu * 18 + k) * es];
              if (es == 8) {
                uint64_t v;
                std::memcpy(&v, &site[slot_of_mu[mu] * 18 + k], 8);
                put_be64(o, v);
              } else {
                const float fv = (float)site[slot_of_mu[mu] * 18 + k];
                uint32_t v;
                std::memcpy(&v, &fv, 4);
                for (int b = 3; b >= 0; --b, v >>= 8) o[b] = (unsigned char)(v & 0xff);
              }
            }
        }
        ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
      }
  if (std::fclose(f) != 0) ok = false;
  if (!ok) {
    set_error("write error on %s", path);
    return LAPH_EIO;
  }
  return LAPH_OK;
}

int laph_lime_write_gauge(const char* path, const double* conf, int L, int T) {
  return laph_lime_write_gauge_prec(path, conf, L, T, 64);
}

}  // extern "C"

namespace {

// Integer content of <tag>...</tag> in an XML text, 0 when absent.
int xml_int(const std::string& xml, const char* tag) {
  const std::string open = std::string("<") + tag + ">";
  const size_t a = xml.find(open);
  if (a == std::string::npos) return 0;
  return std::atoi(xml.c_str() + a + open.size());
}

// Walk the LIME records of an open file: keeps the ildg-format payload (if any
// precedes the binary data) and stops at the ildg-binary-data header, leaving
// the file positioned at its payload.
int lime_find_binary(FILE* f, const char* path, uint64_t* len, std::string* xml) {
  unsigned char h[144];
  for (;;) {
    if (std::fread(h, 1, 144, f) != 144) break;
    if (!(h[0] == 0x45 && h[1] == 0x67 && h[2] == 0x89 && h[3] == 0xab)) {
      set_error("%s: bad LIME magic number", path);
      return LAPH_EIO;
    }
    const uint64_t n = get_be64(h + 8);
    char type[129];
    std::memcpy(type, h + 16, 128);
    type[128] = 0;
    if (std::strcmp(type, "ildg-binary-data") == 0) {
      *len = n;
      return LAPH_OK;
    }
    if (xml && std::strcmp(type, "ildg-format") == 0 && n < (1u << 20)) {
      std::string s(n, '\0');
      if (std::fread(&s[0], 1, n, f) != n) break;
      *xml = s;
      if (n % 8 && fseeko(f, (off_t)(8 - n % 8), SEEK_CUR) != 0) break;
      continue;
    }
    if (fseeko(f, (off_t)((n + 7) / 8 * 8), SEEK_CUR) != 0) break;
  }
  set_error("no ildg-binary-data record found in file %s", path);
  return LAPH_ENORECORD;
}

// Timeslices [t_i, t_f] of an ILDG payload of len bytes with es-byte big-endian
// reals at the file position, into conf in the LAPH_LAYOUT_CONF order (FP32
// widened).
// The file order is t, z, y, x (x fastest), so every (t, z) plane is one
// contiguous run of L^2 sites; the planes are independent units of work: each
// OpenMP thread reads whole planes with pread (the FILE position is left as it
// is) and byte-swaps them into their sites, so the read and the reorder both
// run on every core and many reads are in flight for a cold file.
int lime_read_payload(FILE* f, const char* path, uint64_t len, int L, int t_i, int t_f, int es, double* conf) {
  const long long V3 = (long long)L * L * L;
  const off_t base = ftello(f);
  if (base < 0) {
    set_error("%s: cannot locate the binary record", path);
    return LAPH_EIO;
  }
  const int fd = fileno(f);
  // the whole record must be present, as the reference (which reads all of it)
  // requires, although only [t_i, t_f] is read
  struct stat sb;
  if (fstat(fd, &sb) != 0 || (uint64_t)sb.st_size < (uint64_t)base + len) {
    set_error("LIME read error while reading file %s (binary record truncated)", path);
    return LAPH_EIO;
  }
  const size_t plane = (size_t)L * L * 72 * es;
  const off_t start = base + (off_t)((uint64_t)t_i * V3 * 72 * es);
  const long long nplanes = (long long)(t_f - t_i + 1) * L;
  int failed = 0;
#pragma omp parallel
  {
    std::vector<unsigned char> buf(plane);
#pragma omp for schedule(dynamic, 1)
    for (long long pz = 0; pz < nplanes; ++pz) {
      if (__atomic_load_n(&failed, __ATOMIC_RELAXED)) continue;
      const off_t off = start + (off_t)(pz * (long long)plane);
      size_t got = 0;
      while (got < plane) {
        const ssize_t r = pread(fd, buf.data() + got, plane - got, off + (off_t)got);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) break;
        got += (size_t)r;
      }
      if (got != plane) {
        __atomic_store_n(&failed, 1, __ATOMIC_RELAXED);
        continue;
      }
      const long long t = pz / L;
      const int z = (int)(pz % L);
      for (int y = 0; y < L; ++y)
        for (int x = 0; x < L; ++x) {
          double* site = conf + (t * V3 + (long long)x * L * L + (long long)y * L + z) * 72;
          const unsigned char* src = &buf[((size_t)y * L + x) * 72 * es];
          for (int mu = 0; mu < 4; ++mu) {
            const int slot = (mu == 3) ? 0 : mu + 1;
            for (int k = 0; k < 18; ++k) {
              const unsigned char* q = src + (size_t)(mu * 18 + k) * es;
              if (es == 8) {
                uint64_t v;
                std::memcpy(&v, q, 8);
                v = __builtin_bswap64(v);
                std::memcpy(&site[slot * 18 + k], &v, 8);
              } else {
                uint32_t v;
                std::memcpy(&v, q, 4);
                v = __builtin_bswap32(v);
                float fv;
                std::memcpy(&fv, &v, 4);
                site[slot * 18 + k] = fv;
              }
            }
          }
        }
    }
  }
  if (failed) {
    set_error("LIME read error while reading file %s", path);
    return LAPH_EIO;
  }
  return LAPH_OK;
}

}  // namespace

extern "C" {

// read_lime_gauge_field_doubleprec_timeslices (modules/io.cpp:22-146), but
// seeking straight to timeslice t_i instead of reading the whole file.
int laph_lime_read_gauge(const char* path, int T, int L, int t_i, int t_f, double* conf) {
  if (!path || !conf || T < 1 || L < 1 || t_i < 0 || t_f < t_i || t_f >= T) {
    set_error("laph_lime_read_gauge: bad argument");
    return LAPH_EINVAL;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("Could not open file %s", path);
    return LAPH_EIO;
  }
  uint64_t len = 0;
  int st = lime_find_binary(f, path, &len, nullptr);
  if (st != LAPH_OK) {
    std::fclose(f);
    return st;
  }
  const long long V3 = (long long)L * L * L;
  const uint64_t want = (uint64_t)V3 * T * 72ull * 8ull;
  if (len != want) {
    std::fclose(f);
    if (len == want / 2) {
      set_error("%s: single precision read! Not implemented", path);
      return LAPH_ESINGLE;
    }
    set_error("Probably wrong lattice size or precision (bytes=%llu) in file %s expected %llu",
              (unsigned long long)len, path, (unsigned long long)want);
    return LAPH_ESIZE;
  }
  st = lime_read_payload(f, path, len, L, t_i, t_f, 8, conf);
  std::fclose(f);
  return st;
}

int laph_lime_read_gauge_any(const char* path, int T, int L, int t_i, int t_f, double* conf, int* precision) {
  if (!path || !conf || T < 1 || L < 1 || t_i < 0 || t_f < t_i || t_f >= T) {
    set_error("laph_lime_read_gauge_any: bad argument");
    return LAPH_EINVAL;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("Could not open file %s", path);
    return LAPH_EIO;
  }
  uint64_t len = 0;
  std::string xml;
  int st = lime_find_binary(f, path, &len, &xml);
  if (st != LAPH_OK) {
    std::fclose(f);
    return st;
  }
  const uint64_t want = (uint64_t)L * L * L * T * 72ull * 8ull;
  const int es = len == want ? 8 : (len == want / 2 ? 4 : 0);
  const int declared = xml.empty() ? 0 : xml_int(xml, "precision");
  if (es == 0 || (declared && declared != 8 * es)) {
    std::fclose(f);
    if (es == 0)
      set_error("%s: %llu bytes of binary data fit neither FP64 nor FP32 links of %d^3 x %d", path,
                (unsigned long long)len, L, T);
    else
      set_error("%s: ildg-format declares precision %d but the binary data holds %d-bit reals", path, declared,
                8 * es);
    return LAPH_ESIZE;
  }
  st = lime_read_payload(f, path, len, L, t_i, t_f, es, conf);
  std::fclose(f);
  if (st == LAPH_OK && precision) *precision = 8 * es;
  return st;
}

int laph_lime_info(const char* path, int* lx, int* ly, int* lz, int* lt, int* precision) {
  if (!path || !lx || !ly || !lz || !lt || !precision) {
    set_error("laph_lime_info: bad argument");
    return LAPH_EINVAL;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("Could not open file %s", path);
    return LAPH_EIO;
  }
  uint64_t len = 0;
  std::string xml;
  const int st = lime_find_binary(f, path, &len, &xml);
  std::fclose(f);
  if (st != LAPH_OK) return st;
  if (xml.empty()) {
    set_error("%s: no ildg-format record before the binary data", path);
    return LAPH_ENORECORD;
  }
  *lx = xml_int(xml, "lx");
  *ly = xml_int(xml, "ly");
  *lz = xml_int(xml, "lz");
  *lt = xml_int(xml, "lt");
  *precision = xml_int(xml, "precision");
  if (*lx <= 0 || *ly <= 0 || *lz <= 0 || *lt <= 0 || (*precision != 32 && *precision != 64)) {
    set_error("%s: ildg-format record without valid lx/ly/lz/lt/precision", path);
    return LAPH_EPARSE;
  }
  const uint64_t want = (uint64_t)*lx * *ly * *lz * *lt * 72ull * (*precision / 8);
  if (len != want) {
    set_error("%s: ildg-format describes %llu bytes of links, the binary record holds %llu", path,
              (unsigned long long)want, (unsigned long long)len);
    return LAPH_ESIZE;
  }
  return LAPH_OK;
}

int laph_check_trace(int dim, int nev, const double* Vd, double* trace, double* sum) {
  // tr(V^dag V) = sum_n |v_n|^2 and sum(V^dag V) = |sum_n v_n|^2 (read_write.cpp:20-35)
  const cd* V = reinterpret_cast<const cd*>(Vd);
  double tr = 0.0, sre = 0.0;
#pragma omp parallel for reduction(+ : tr, sre) schedule(static)
  for (long long i = 0; i < dim; ++i) {
    cd acc = 0.0;
    for (int n = 0; n < nev; ++n) {
      const cd v = V[(size_t)n * dim + i];
      tr += std::norm(v);
      acc += v;
    }
    sre += std::norm(acc);
  }
  if (trace) *trace = tr;
  if (sum) *sum = sre;
  const double eps = 10e-10;
  return !(std::fabs(tr) - nev > eps || std::fabs(sre) - nev > eps);
}

static void eig_name(char* out, size_t n, const char* dir, const char* prefix, int config, int t) {
  std::snprintf(out, n, "%s/%s.%04d.%03d", dir, prefix, config, t);
}

int laph_write_eigsys_bin(const char* dir, const char* prefix, int config, int t, int dim, int nev, const double* V) {
  if (!laph_check_trace(dim, nev, V, nullptr, nullptr)) {
    set_error("Timeslice: %d: Eigenvectors damaged, abort writing", t);
    return LAPH_ETRACE;
  }
  char name[1024];
  eig_name(name, sizeof name, dir, prefix, config, t);
  FILE* f = std::fopen(name, "wb");
  if (!f) {
    set_error("cannot open %s", name);
    return LAPH_EIO;
  }
  const size_t n = (size_t)2 * dim * nev;
  const bool ok = std::fwrite(V, sizeof(double), n, f) == n;
  if (std::fclose(f) != 0 || !ok) {
    set_error("Timeslice: %d Error: write incomplete", t);
    return LAPH_EIO;
  }
  return LAPH_OK;
}

int laph_write_eigenvalues_bin(const char* dir, const char* prefix, int config, int t, int nev, const double* ev) {
  char name[1024];
  eig_name(name, sizeof name, dir, prefix, config, t);
  FILE* f = std::fopen(name, "wb");
  if (!f) {
    set_error("cannot open %s", name);
    return LAPH_EIO;
  }
  const bool ok = std::fwrite(ev, sizeof(double), nev, f) == (size_t)nev;
  if (std::fclose(f) != 0 || !ok) {
    set_error("write error on %s", name);
    return LAPH_EIO;
  }
  return LAPH_OK;
}

int laph_read_eigsys_bin(const char* dir, const char* prefix, int config, int t, int dim, int nev, double* V) {
  char name[1024];
  eig_name(name, sizeof name, dir, prefix, config, t);
  FILE* f = std::fopen(name, "rb");
  if (!f) {
    set_error("cannot open %s", name);
    return LAPH_EIO;
  }
  const size_t n = (size_t)2 * dim * nev;
  const size_t got = std::fread(V, sizeof(double), n, f);
  std::fclose(f);
  if (got != n) {
    set_error("Timeslice: %d: wrong number of eigenvectors read", t);
    return LAPH_EIO;
  }
  if (!laph_check_trace(dim, nev, V, nullptr, nullptr)) {
    set_error("Timeslice: %d: Eigenvectors damaged", t);
    return LAPH_ETRACE;
  }
  return LAPH_OK;
}

int laph_read_eigenvalues_bin(const char* dir, const char* prefix, int config, int t, int nev, double* ev) {
  char name[1024];
  eig_name(name, sizeof name, dir, prefix, config, t);
  FILE* f = std::fopen(name, "rb");
  if (!f) {
    set_error("cannot open %s", name);
    return LAPH_EIO;
  }
  const size_t got = std::fread(ev, sizeof(double), nev, f);
  std::fclose(f);
  if (got != (size_t)nev) {
    set_error("%s: short read", name);
    return LAPH_EIO;
  }
  return LAPH_OK;
}

int laph_sourceshape_avg(int L, const double* psi, double* r_out, double* psi_out, int* n_out) {
  if (L < 2 || (L & 1) || !psi || !r_out || !psi_out || !n_out) {
    set_error("laph_sourceshape_avg: bad argument (even L >= 2 and all arrays needed)");
    return LAPH_EINVAL;
  }
  std::vector<long long> cnt;
  std::vector<double> rad, sum;
  int idx = 0;
  for (int r1 = 0; r1 < L; r1 += 2)
    for (int r2 = 0; r2 < L; r2 += 2)
      for (int r3 = 0; r3 < L; r3 += 2, ++idx) {
        const double len = std::sqrt((double)r1 * r1 + (double)r2 * r2 + (double)r3 * r3);
        size_t t = 0;
        while (t < rad.size() && !(std::fabs(len - rad[t]) < 1e-11)) ++t;
        if (t == rad.size()) {
          rad.push_back(len);
          cnt.push_back(0);
          sum.push_back(0.0);
        }
        ++cnt[t];
        sum[t] += psi[idx];
      }
  for (size_t t = 0; t < rad.size(); ++t) {
    r_out[t] = rad[t];
    psi_out[t] = sum[t] / (double)cnt[t];
  }
  *n_out = (int)rad.size();
  return LAPH_OK;
}

int laph_write_sourceshape(const char* dir, int config, int t, int nev, int n, const double* r, const double* psi) {
  if (n < 0 || (n > 0 && (!r || !psi))) {
    set_error("laph_write_sourceshape: bad argument");
    return LAPH_EINVAL;
  }
  const std::string pre = (dir && *dir) ? std::string(dir) + "/" : std::string();
  char name[1200];
  std::snprintf(name, sizeof name, "%ssourceshape_nev%d.%d.%d", pre.c_str(), nev, config, t);
  FILE* f = std::fopen(name, "w");
  if (!f) {
    set_error("cannot open %s for writing", name);
    return LAPH_EIO;
  }
  bool ok = std::fprintf(f, "#r\tpsi(r)\n") > 0;
  for (int i = 0; ok && i < n; ++i) ok = std::fprintf(f, "%.12g %.12g\n", r[i], psi[i]) > 0;
  if (std::fclose(f) != 0) ok = false;
  std::snprintf(name, sizeof name, "%ssourceshape_nev%d.%04d.%03d.bin", pre.c_str(), nev, config, t);
  f = ok ? std::fopen(name, "wb") : nullptr;
  if (f) {
    for (int i = 0; ok && i < n; ++i) {
      const double pair[2] = {r[i], psi[i]};
      ok = std::fwrite(pair, sizeof(double), 2, f) == 2;
    }
    if (std::fclose(f) != 0) ok = false;
  } else {
    ok = false;
  }
  if (!ok) {
    set_error("write error on %s", name);
    return LAPH_EIO;
  }
  return LAPH_OK;
}

int laph_fix_phase_host(int dim, int nev, const double* Vd, double* Vfd, double* phase) {
  const cd* V = reinterpret_cast<const cd*>(Vd);
  cd* Vf = reinterpret_cast<cd*>(Vfd);
  for (int n = 0; n < nev; ++n) {
    const double ph = std::arg(V[(size_t)n * dim]);
    if (phase) phase[n] = ph;
    const cd fac = std::exp(cd(0.0, -ph));
    for (long long i = 0; i < dim; ++i) Vf[(size_t)n * dim + i] = fac * V[(size_t)n * dim + i];
  }
  return LAPH_OK;
}

int laph_reset_phase_host(int dim, int nev, const double* Vd, const double* phase_want, double* Vrd) {
  if (dim < 1 || nev < 0 || (nev > 0 && (!Vd || !phase_want || !Vrd))) {
    set_error("laph_reset_phase_host: bad argument");
    return LAPH_EINVAL;
  }
  // reset_phase (modules/eigensystem.cpp:32-57): rotate column n so that its
  // first entry has the phase phase_want[n]
  const cd* V = reinterpret_cast<const cd*>(Vd);
  cd* Vr = reinterpret_cast<cd*>(Vrd);
  for (int n = 0; n < nev; ++n) {
    const cd fac = std::exp(cd(0.0, -(std::arg(V[(size_t)n * dim]) - phase_want[n])));
    for (long long i = 0; i < dim; ++i) Vr[(size_t)n * dim + i] = fac * V[(size_t)n * dim + i];
  }
  return LAPH_OK;
}

int laph_read_eigenvalues_ascii(const char* prefix, int config, int t, int nev, double* ev) {
  if (!prefix || nev < 0 || (nev > 0 && !ev)) {
    set_error("laph_read_eigenvalues_ascii: bad argument");
    return LAPH_EINVAL;
  }
  // read_eigenvalues_ascii (modules/read_write.cpp:99-115): "<prefix>.%03d.%04d"
  // (timeslice first, then configuration), whitespace-separated values.  The
  // reference skips a missing file silently and leaves unread values as they
  // were; here both are errors.
  char name[1100];
  std::snprintf(name, sizeof name, "%s.%03d.%04d", prefix, t, config);
  FILE* f = std::fopen(name, "r");
  if (!f) {
    set_error("cannot open %s", name);
    return LAPH_EIO;
  }
  int got = 0;
  while (got < nev && std::fscanf(f, "%lf", ev + got) == 1) ++got;
  std::fclose(f);
  if (got != nev) {
    set_error("%s: %d of %d values", name, got, nev);
    return LAPH_ESIZE;
  }
  return LAPH_OK;
}

int laph_write_gauge_matrices(const char* path, int V3, const double* G) {
  if (!path || V3 < 1 || !G) {
    set_error("laph_write_gauge_matrices: bad argument");
    return LAPH_EINVAL;
  }
  // write_gauge_matrices (modules/read_write.cpp:253-261): V3 raw Matrix3cd
  // (column-major complex128, 144 bytes each), no header
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("cannot create %s", path);
    return LAPH_EIO;
  }
  const size_t n = (size_t)V3 * 18;
  const bool ok = std::fwrite(G, sizeof(double), n, f) == n;
  if (std::fclose(f) != 0 || !ok) {
    set_error("%s: write failed", path);
    return LAPH_EIO;
  }
  return LAPH_OK;
}

int laph_read_gauge_matrices(const char* path, int V3, double* G) {
  if (!path || V3 < 1 || !G) {
    set_error("laph_read_gauge_matrices: bad argument");
    return LAPH_EINVAL;
  }
  // read_gauge_matrices (modules/read_write.cpp:117-132); a short file is an
  // error here (the reference keeps whatever the failed reads left)
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("cannot open %s", path);
    return LAPH_EIO;
  }
  const size_t n = (size_t)V3 * 18;
  const size_t got = std::fread(G, sizeof(double), n, f);
  std::fclose(f);
  if (got != n) {
    set_error("%s: %zu of %zu bytes", path, got * sizeof(double), n * sizeof(double));
    return LAPH_ESIZE;
  }
  return LAPH_OK;
}

int laph_timeslice_split(int LT, int size, int rank, int* t0, int* count) {
  if (LT < 0 || size < 1 || rank < 0 || rank >= size || !t0 || !count) {
    set_error("laph_timeslice_split: bad argument");
    return LAPH_EINVAL;
  }
  // rank 0 of the reference fills todos = LT/size, adds one to the first
  // LT % size, and chains tstart/tend (src/ev_ts.cpp:103-119)
  const int base = LT / size, extra = LT % size;
  *count = base + (rank < extra ? 1 : 0);
  *t0 = rank * base + (rank < extra ? rank : extra);
  return LAPH_OK;
}

int laph_recover_spectrum(int nev, const double* theta, int deg, double lam_l, double lam_c, double* out) {
  for (int i = 0; i < nev; ++i) {
    const double b = std::cosh(1.0 / deg * std::acosh(theta[i]));
    out[i] = (lam_l - lam_c) * (b - 1) * 0.5 - lam_c;
  }
  return LAPH_OK;
}

// IO::set_values (modules/par_io.cpp:8-136): "key = value" with exactly one
// space either side of '=', '#' lines skipped, and -- like
// while(!getline().eof()) -- a last line without trailing newline ignored.
// An empty line (or one ending right after '=') makes the reference throw
// std::out_of_range; here it returns LAPH_EPARSE.  Missing keys read as
// 0 / 0.0 / "".
int laph_parse_parameters(const char* path, laph_config* cfg) {
  std::memset(cfg, 0, sizeof *cfg);
  cfg->smear = LAPH_SMEAR_HYP;
  cfg->tol = 1e-9;
  cfg->guard = 16;
  std::ifstream in(path);
  if (!in) {
    set_error("cannot open %s", path);
    return LAPH_EIO;
  }
  std::string content((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  std::vector<std::string> lines;
  size_t pos = 0;
  for (;;) {
    size_t nl = content.find('\n', pos);
    if (nl == std::string::npos) break;  // unterminated last line is dropped
    lines.push_back(content.substr(pos, nl - pos));
    pos = nl + 1;
  }
  std::map<std::string, std::string> kv;
  int lineno = 0;
  for (const std::string& line : lines) {
    ++lineno;
    if (!line.empty() && line[0] == '#') continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) {
      // the reference takes the whole line as an (unknown) key and value
      // substr(1); only an empty line makes substr throw
      if (line.empty()) {
        set_error("%s:%d: empty line (the reference parser throws std::out_of_range here)", path, lineno);
        return LAPH_EPARSE;
      }
      continue;
    }
    if (eq + 2 > line.size()) {
      set_error("%s:%d: nothing after '=' (the reference parser throws std::out_of_range here)", path, lineno);
      return LAPH_EPARSE;
    }
    const std::string key = eq >= 1 ? line.substr(0, eq - 1) : std::string();
    kv[key] = line.substr(eq + 2);
  }
  auto S = [&](const char* k, char* dst) {
    auto it = kv.find(k);
    std::snprintf(dst, 512, "%s", it == kv.end() ? "" : it->second.c_str());
  };
  auto I = [&](const char* k, int def) {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::atoi(it->second.c_str());
  };
  auto F = [&](const char* k, double def) {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::atof(it->second.c_str());
  };
  S("config_path", cfg->config_path);
  S("result_path", cfg->result_path);
  S("in_path", cfg->in_path);
  S("phase_path", cfg->phase_path);
  cfg->LT = I("LT", 0);
  cfg->LX = I("LX", 0);
  cfg->NEV = I("NEV", 0);
  cfg->iter = I("iter", 0);
  cfg->DEG = I("DEG", 0);
  cfg->OMP_THRDS = I("OMP_THRDS", 0);
  cfg->alpha_1 = F("alpha_1", 0.0);
  cfg->alpha_2 = F("alpha_2", 0.0);
  cfg->LAM_L = F("LAM_L", 0.0);
  cfg->LAM_C = F("LAM_C", 0.0);
  auto sm = kv.find("smear");
  if (sm != kv.end()) {
    const std::string v = sm->second;
    if (v.rfind("hyp", 0) == 0) cfg->smear = LAPH_SMEAR_HYP;
    else if (v.rfind("stout", 0) == 0) cfg->smear = LAPH_SMEAR_STOUT;
    else if (v.rfind("ape", 0) == 0) cfg->smear = LAPH_SMEAR_APE;
    else if (v.rfind("none", 0) == 0) cfg->smear = LAPH_SMEAR_NONE;
    else {
      set_error("%s: unknown smear '%s'", path, v.c_str());
      return LAPH_EPARSE;
    }
  }
  cfg->rho = F("rho", 0.1);
  cfg->alpha = F("alpha", 0.5);
  cfg->tol = F("tol", 1e-9);
  cfg->guard = I("guard", 16);
  cfg->block = I("block", 0);
  auto wi = kv.find("window");
  cfg->window = LAPH_WINDOW_LANCZOS;
  if (wi != kv.end()) {
    const std::string v = wi->second;
    if (v.rfind("fixed", 0) == 0) cfg->window = LAPH_WINDOW_FIXED;
    else if (v.rfind("lanczos", 0) == 0) cfg->window = LAPH_WINDOW_LANCZOS;
    else if (v.rfind("mlp", 0) == 0) cfg->window = LAPH_WINDOW_MLP;
  }
  auto so = kv.find("solver");
  cfg->solver = (so != kv.end() && so->second.rfind("plain", 0) == 0) ? 1 : 0;
  cfg->V3 = cfg->LX * cfg->LX * cfg->LX;
  cfg->MAT_ENTRIES = 3 * cfg->V3;
  cfg->V_TS = cfg->V3 * 72;
  cfg->alpha_1_i = F("alpha_1_i", 0.0);
  cfg->alpha_1_f = F("alpha_1_f", 0.0);
  cfg->alpha_2_i = F("alpha_2_i", 0.0);
  cfg->alpha_2_f = F("alpha_2_f", 0.0);
  cfg->autotune = I("autotune", 0);
  cfg->filter_deg = I("filter_deg", 0);
  return LAPH_OK;
}

}  // extern "C"
