/*
 * laph_oracle.cpp -- CPU FP64 oracle (TEST INFRASTRUCTURE, see laph_oracle.h).
 *
 * Parity status: arithmetic unpinned against reference outputs (the reference
 * cannot be built here as a whole and has no golden vectors); site indexing and
 * formulas checked on the reference's compiled lookup tables, and pinned by
 * analytic known answers (laph_oracle.h).
 * Each function cites the reference file:line it restates.  Third-party
 * arithmetic the reference delegates to libraries is restated from the
 * mathematics:
 *   - Eigen 3.2/3.3 Matrix3cd::sqrt()/inverse()/exp(): replaced by a
 *     Hermitian 3x3 Jacobi eigendecomposition (principal square root of the
 *     positive-definite M^dag M, and exp(iH) of a Hermitian H).
 *   - SLEPc 3.12 EPS Krylov-Schur (HEP, largest magnitude): restated as a
 *     thick-restart Lanczos with full (classical, twice) reorthogonalisation
 *     and SLEPc's defaults (ncv = max(2 nev, nev+15), keep = 1/2, relative
 *     convergence test).
 *   - c-lime 1.3.2 record parsing: restated from the public LIME record
 *     layout (144-byte big-endian header, 8-byte padded payload).
 */
#include "laph_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

namespace {

struct M3 {
  cd m[9];
};

inline M3 m3_zero() {
  M3 r;
  for (int i = 0; i < 9; ++i) r.m[i] = 0.0;
  return r;
}
inline M3 m3_id() {
  M3 r = m3_zero();
  r.m[0] = r.m[4] = r.m[8] = 1.0;
  return r;
}
inline M3 mul(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      r.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
  return r;
}
inline M3 adj(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[3 * i + j] = std::conj(a.m[3 * j + i]);
  return r;
}
inline M3 add(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 9; ++i) r.m[i] = a.m[i] + b.m[i];
  return r;
}
inline M3 scal(const M3& a, cd s) {
  M3 r;
  for (int i = 0; i < 9; ++i) r.m[i] = a.m[i] * s;
  return r;
}
inline cd det3(const M3& a) {
  const cd* m = a.m;
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}
inline M3 load(const double* p) {
  M3 r;
  for (int i = 0; i < 9; ++i) r.m[i] = cd(p[2 * i], p[2 * i + 1]);
  return r;
}
inline void store(double* p, const M3& a) {
  for (int i = 0; i < 9; ++i) {
    p[2 * i] = a.m[i].real();
    p[2 * i + 1] = a.m[i].imag();
  }
}

/* Cyclic Jacobi eigendecomposition of a Hermitian 3x3: A = Q diag(d) Q^dag.
 * For the pair (p,q) with A_pq = r e^{i phi}, the unitary J = P R with
 * P = diag(1, e^{-i phi}) on (p,q) and R the real Jacobi rotation of the
 * symmetric 2x2 [[a_pp, r], [r, a_qq]] annihilates A_pq. */
void herm3_eig(const M3& Ain, double d[3], M3& Q) {
  M3 A = Ain;
  Q = m3_id();
  static const int P[3] = {0, 0, 1}, Qi[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 12; ++sweep) {
    double off = std::norm(A.m[1]) + std::norm(A.m[2]) + std::norm(A.m[5]);
    double dg = std::norm(A.m[0]) + std::norm(A.m[4]) + std::norm(A.m[8]);
    if (off <= 1e-34 * dg || off == 0.0) break;
    for (int k = 0; k < 3; ++k) {
      const int p = P[k], q = Qi[k];
      const cd g = A.m[3 * p + q];
      const double r = std::abs(g);
      if (r == 0.0) continue;
      const cd eph = g / r;  // e^{i phi}
      const double app = A.m[3 * p + p].real(), aqq = A.m[3 * q + q].real();
      const double tau = (aqq - app) / (2.0 * r);
      const double t = (tau >= 0.0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
      const double c = 1.0 / std::sqrt(1.0 + t * t);
      const double s = t * c;
      // J (3x3 unitary): identity outside (p,q); block [[c, s], [-s e^{-i phi}, c e^{-i phi}]]
      M3 J = m3_id();
      const cd emph = std::conj(eph);
      J.m[3 * p + p] = c;
      J.m[3 * p + q] = s;
      J.m[3 * q + p] = -s * emph;
      J.m[3 * q + q] = c * emph;
      A = mul(adj(J), mul(A, J));
      A.m[3 * p + q] = 0.0;
      A.m[3 * q + p] = 0.0;
      Q = mul(Q, J);
    }
  }
  for (int i = 0; i < 3; ++i) d[i] = A.m[4 * i].real();
}

/* Q diag(f) Q^dag */
inline M3 qfq(const M3& Q, const cd f[3]) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      cd s = 0.0;
      for (int k = 0; k < 3; ++k) s += Q.m[3 * i + k] * f[k] * std::conj(Q.m[3 * j + k]);
      r.m[3 * i + j] = s;
    }
  return r;
}

/* proj_to_su3_imp, modules/timeslice.cpp:90-104 */
M3 proj_su3(const M3& in) {
  M3 A = mul(adj(in), in);
  double d[3];
  M3 Q;
  herm3_eig(A, d, Q);
  cd f[3];
  for (int i = 0; i < 3; ++i) f[i] = 1.0 / std::sqrt(d[i]);
  M3 W = mul(in, qfq(Q, f));
  cd det = det3(W);
  cd fac = 1.0 / std::pow(det, 1.0 / 3.0);  // principal branch, as std::pow in the reference
  return scal(W, fac);
}

/* exp(i H), H Hermitian */
M3 expiH(const M3& H) {
  double d[3];
  M3 Q;
  herm3_eig(H, d, Q);
  cd f[3];
  for (int i = 0; i < 3; ++i) f[i] = cd(std::cos(d[i]), std::sin(d[i]));
  return qfq(Q, f);
}

/* Periodic neighbours, modules/navigation.cpp:27-88 */
struct Geo {
  int L, L2, V3;
  explicit Geo(int l) : L(l), L2(l * l), V3(l * l * l) {}
  inline int up(int i, int dir) const {
    int x = i / L2, y = (i / L) % L, z = i % L;
    if (dir == 0) x = (x + 1 == L) ? 0 : x + 1;
    else if (dir == 1) y = (y + 1 == L) ? 0 : y + 1;
    else z = (z + 1 == L) ? 0 : z + 1;
    return x * L2 + y * L + z;
  }
  inline int dn(int i, int dir) const {
    int x = i / L2, y = (i / L) % L, z = i % L;
    if (dir == 0) x = (x == 0) ? L - 1 : x - 1;
    else if (dir == 1) y = (y == 0) ? L - 1 : y - 1;
    else z = (z == 0) ? L - 1 : z - 1;
    return x * L2 + y * L + z;
  }
};

inline M3 link(const double* U, int site, int dir) { return load(U + (size_t)(site * 3 + dir) * 18); }

/* get_dirs, modules/timeslice.cpp:106-122 */
inline void perp_dirs(int mu, int out[2]) {
  if (mu == 0) { out[0] = 1; out[1] = 2; }
  else if (mu == 1) { out[0] = 0; out[1] = 2; }
  else { out[0] = 0; out[1] = 1; }
}
/* decor, modules/timeslice.cpp:125-140 */
inline int decor(int dir, int plane) {
  if (dir == 0) return plane == 1 ? 0 : 3;
  if (dir == 1) return plane == 0 ? 1 : 4;
  return plane == 0 ? 2 : 5;
}

/* staple sum of smearing_stout / smearing_ape, modules/timeslice.cpp:159-174 */
M3 staple_sum(const double* U, const Geo& g, int i, int dir, int compat) {
  M3 st = m3_zero();
  for (int nd = 0; nd < 3; ++nd) {
    if (nd == dir) continue;
    int mu = g.up(i, nd);
    int nu = g.up(mu, dir);
    int eta = g.dn(nu, nd);
    st = add(st, mul(link(U, i, nd), mul(link(U, mu, dir), adj(link(U, eta, nd)))));
    mu = g.dn(i, nd);
    nu = g.up(mu, dir);
    // reference quirk (timeslice.cpp:171-172): third factor is U[nu][dir]
    const M3 third = compat ? link(U, nu, dir) : link(U, nu, nd);
    st = add(st, mul(adj(link(U, mu, nd)), mul(link(U, mu, dir), third)));
  }
  return st;
}

inline void zaxpy_region(long n, cd a, const cd* x, cd* y) {
  for (long i = 0; i < n; ++i) y[i] += a * x[i];
}

/* Cyclic Jacobi for a real symmetric n x n (row-major), eigenvectors in Z. */
void sym_jacobi(int n, std::vector<double>& A, std::vector<double>& d, std::vector<double>& Z) {
  Z.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Z[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int i = 0; i < n; ++i) {
      dg += A[(size_t)i * n + i] * A[(size_t)i * n + i];
      for (int j = i + 1; j < n; ++j) off += A[(size_t)i * n + j] * A[(size_t)i * n + j];
    }
    if (off <= 1e-32 * dg || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
        if (std::fabs(apq) < 1e-300) { A[(size_t)p * n + q] = A[(size_t)q * n + p] = 0.0; continue; }
        const double tau = (aqq - app) / (2.0 * apq);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p,q
          const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * akp - s * akq;
          A[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p,q
          const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * apk - s * aqk;
          A[(size_t)q * n + k] = s * apk + c * aqk;
        }
        A[(size_t)p * n + q] = A[(size_t)q * n + p] = 0.0;
        for (int k = 0; k < n; ++k) {
          const double zkp = Z[(size_t)k * n + p], zkq = Z[(size_t)k * n + q];
          Z[(size_t)k * n + p] = c * zkp - s * zkq;
          Z[(size_t)k * n + q] = s * zkp + c * zkq;
        }
      }
    }
  }
  d.resize(n);
  for (int i = 0; i < n; ++i) d[i] = A[(size_t)i * n + i];
}

/* SplitMix64 stream, used only for the Krylov start vector. */
struct SplitMix {
  uint64_t s;
  explicit SplitMix(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
};

uint32_t be32(const unsigned char* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }
uint64_t be64(const unsigned char* p) {
  uint64_t v = 0;
  for (int i = 0; i < 8; ++i) v = v << 8 | p[i];
  return v;
}

}  // namespace

extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* modules/io.cpp:22-146 */
int orc_lime_read_gauge(const char* path, int T, int L, int t_i, int t_f, double* conf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return 500;
  unsigned char hdr[144];
  long long data_off = -1;
  uint64_t nbytes = 0;
  for (;;) {
    if (std::fread(hdr, 1, 144, f) != 144) break;
    if (be32(hdr) != 0x456789abu) { std::fclose(f); return 500; }
    uint64_t len = be64(hdr + 8);
    char type[129];
    std::memcpy(type, hdr + 16, 128);
    type[128] = 0;
    long long here = std::ftell(f);
    if (std::strcmp(type, "ildg-binary-data") == 0) { data_off = here; nbytes = len; break; }
    uint64_t padded = (len + 7) / 8 * 8;
    if (std::fseek(f, (long)padded, SEEK_CUR) != 0) break;
  }
  if (data_off < 0) { std::fclose(f); return -2; }
  const uint64_t V = (uint64_t)L * L * L;
  const uint64_t want = V * (uint64_t)T * 72ull * 8ull;
  if (nbytes != want) { std::fclose(f); return nbytes == want / 2 ? 502 : 501; }
  std::vector<unsigned char> buf(72 * 8);
  for (int t = 0; t < T; ++t)
    for (int z = 0; z < L; ++z)
      for (int y = 0; y < L; ++y)
        for (int x = 0; x < L; ++x) {
          if (std::fread(buf.data(), 1, 72 * 8, f) != 72 * 8) { std::fclose(f); return 500; }
          if (t < t_i || t > t_f) continue;
          double tmp2[72];
          for (int k = 0; k < 72; ++k) {
            uint64_t v = be64(buf.data() + 8 * k);
            std::memcpy(&tmp2[k], &v, 8);
          }
          const size_t p = ((size_t)(t - t_i) * V + (size_t)x * L * L + (size_t)y * L + z) * 72;
          size_t k = 0;
          for (int mu = 1; mu <= 4; ++mu) {  // ILDG mu order x,y,z,t -> slots 1,2,3,0
            const size_t index = (mu != 4) ? p + mu * 18 : p;
            for (int i = 0; i < 3; ++i)
              for (int j = 0; j < 3; ++j) {
                conf[index + 6 * i + 2 * j] = tmp2[2 * k];
                conf[index + 6 * i + 2 * j + 1] = tmp2[2 * k + 1];
                ++k;
              }
          }
        }
  std::fclose(f);
  return 0;
}

/* modules/timeslice.cpp:34-79: U[site][mu-1](a,b) = conf[site*72 + mu*18 + 6a + 2b] */
void orc_map_timeslice(const double* conf_ts, int L, double* links3) {
  const long V3 = (long)L * L * L;
  for (long s = 0; s < V3; ++s)
    for (int mu = 1; mu < 4; ++mu)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const double* src = conf_ts + s * 72 + mu * 18 + 6 * a + 2 * b;
          double* dst = links3 + ((s * 3 + (mu - 1)) * 9 + 3 * a + b) * 2;
          dst[0] = src[0];
          dst[1] = src[1];
        }
}

void orc_proj_su3(double* m18) { store(m18, proj_su3(load(m18))); }

void orc_expiH(const double* h18, double* out18) { store(out18, expiH(load(h18))); }

/* The seeded synthetic gauge field of the benchmark configurations (no
 * reference function: the reference reads its fields from ILDG files):
 * U = exp(i eps H), H = sum_a c_a lambda_a over the Gell-Mann matrices, c_a
 * i.i.d. N(0, 1), for all 4 links of every site of nt timeslices, conf laid
 * out [t][site][mu][3][3] complex128 as the ILDG slice (slot 0 = U_t).  The
 * normals come from the same counter-based SplitMix64 stream as the
 * library's laph_gauge_random (link n: 4 Box-Muller pairs), so the two agree
 * to rounding; exp(i eps H) goes through this oracle's own Hermitian
 * eigensolver.  Lets CPU-only runs build their inputs without the library. */
static inline uint64_t orc_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

void orc_gauge_random(double* conf, int L, int nt, double eps, uint64_t seed) {
  const long long nlinks = (long long)L * L * L * nt * 4;
  const double is3 = 1.0 / std::sqrt(3.0);
#pragma omp parallel for schedule(static)
  for (long long n = 0; n < nlinks; ++n) {
    uint64_t st = seed * 0x9E3779B97F4A7C15ULL + (uint64_t)n * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL;
    double c[8];
    for (int k = 0; k < 4; ++k) {
      st += 0x9E3779B97F4A7C15ULL;
      const double u1 = ((orc_mix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      st += 0x9E3779B97F4A7C15ULL;
      const double u2 = ((orc_mix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      const double r = std::sqrt(-2.0 * std::log(u1));
      c[2 * k] = r * std::cos(2.0 * M_PI * u2);
      c[2 * k + 1] = r * std::sin(2.0 * M_PI * u2);
    }
    M3 H = m3_zero();
    H.m[0] = eps * (c[2] + c[7] * is3);
    H.m[4] = eps * (-c[2] + c[7] * is3);
    H.m[8] = eps * (-2.0 * c[7] * is3);
    H.m[1] = eps * cd(c[0], -c[1]);
    H.m[3] = eps * cd(c[0], c[1]);
    H.m[2] = eps * cd(c[3], -c[4]);
    H.m[6] = eps * cd(c[3], c[4]);
    H.m[5] = eps * cd(c[5], -c[6]);
    H.m[7] = eps * cd(c[5], c[6]);
    store(conf + n * 18, expiH(H));
  }
}

/* Tslice::smearing_stout, modules/timeslice.cpp:145-193 */
void orc_smear_stout(double* U, int L, double rho, int iter, int compat) {
  Geo g(L);
  std::vector<double> tmp((size_t)g.V3 * 3 * 18);
  for (int it = 0; it < iter; ++it) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g.V3; ++i)
      for (int dir = 0; dir < 3; ++dir) {
        M3 st = staple_sum(U, g, i, dir, compat);
        M3 u = link(U, i, dir);
        M3 omega = mul(scal(st, rho / 4.0), adj(u));
        M3 d = add(adj(omega), scal(omega, -1.0));  // Omega^dag - Omega
        cd tr = d.m[0] + d.m[4] + d.m[8];
        M3 q = add(scal(d, 0.5), scal(m3_id(), -tr / 6.0));
        // exp(-q) with -q = iH, H = i q (Hermitian)
        M3 H = scal(q, cd(0.0, 1.0));
        store(&tmp[(size_t)(i * 3 + dir) * 18], mul(expiH(H), u));
      }
    std::memcpy(U, tmp.data(), tmp.size() * sizeof(double));
  }
}

/* Tslice::smearing_ape, modules/timeslice.cpp:196-239 */
void orc_smear_ape(double* U, int L, double alpha, int iter, int compat) {
  Geo g(L);
  std::vector<double> tmp((size_t)g.V3 * 3 * 18);
  for (int it = 0; it < iter; ++it) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g.V3; ++i)
      for (int dir = 0; dir < 3; ++dir) {
        M3 st = staple_sum(U, g, i, dir, compat);
        M3 m = add(scal(link(U, i, dir), 1.0 - alpha), scal(st, alpha / 4.0));
        store(&tmp[(size_t)(i * 3 + dir) * 18], proj_su3(m));
      }
    std::memcpy(U, tmp.data(), tmp.size() * sizeof(double));
  }
}

/* Tslice::smearing_hyp, modules/timeslice.cpp:243-369 */
void orc_smear_hyp(double* U, int L, double a1, double a2, int iter) {
  Geo g(L);
  std::vector<double> dec((size_t)g.V3 * 6 * 18);
  std::vector<double> tmp((size_t)g.V3 * 3 * 18);
  for (int run = 0; run < iter; ++run) {
    // level 1: decorated links, :263-306
#pragma omp parallel for schedule(static)
    for (int v = 0; v < g.V3; ++v)
      for (int dir = 0; dir < 3; ++dir) {
        int pd[2];
        perp_dirs(dir, pd);
        M3 res[2];
        for (int n = 0; n < 2; ++n) {
          const int p = pd[n];
          int mu = g.up(v, p);
          int eta = g.up(v, dir);
          M3 inner = mul(link(U, v, p), mul(link(U, mu, dir), adj(link(U, eta, p))));
          mu = g.dn(v, p);
          int nu = g.up(mu, dir);
          inner = add(inner, mul(adj(link(U, mu, p)), mul(link(U, mu, dir), link(U, nu, p))));
          M3 stac = add(scal(link(U, v, dir), 1.0 - a2), scal(inner, a2 / 2.0));
          res[n] = proj_su3(stac);
        }
        store(&dec[((size_t)v * 6 + dir) * 18], res[0]);
        store(&dec[((size_t)v * 6 + dir + 3) * 18], res[1]);
      }
    // level 2: :311-357
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g.V3; ++i)
      for (int dir = 0; dir < 3; ++dir) {
        M3 outer = m3_zero();
        for (int nd = 0; nd < 3; ++nd) {
          if (nd == dir) continue;
          const int plane = ((dir + 1) ^ (nd + 1)) - 1;
          int mu = g.up(i, nd);
          int nu = g.up(mu, dir);
          int eta = g.dn(nu, nd);
          const int a = decor(nd, plane), b = decor(dir, plane);
          auto D = [&](int s, int k) { return load(&dec[((size_t)s * 6 + k) * 18]); };
          outer = add(outer, mul(D(i, a), mul(D(mu, b), adj(D(eta, a)))));
          mu = g.dn(i, nd);
          nu = g.up(mu, dir);
          outer = add(outer, mul(adj(D(mu, a)), mul(D(mu, b), D(nu, a))));
        }
        M3 m = add(scal(link(U, i, dir), 1.0 - a1), scal(outer, a1 / 4.0));
        store(&tmp[(size_t)(i * 3 + dir) * 18], m);
      }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g.V3; ++i)
      for (int dir = 0; dir < 3; ++dir) {
        double* p = &tmp[(size_t)(i * 3 + dir) * 18];
        store(U + (size_t)(i * 3 + dir) * 18, proj_su3(load(p)));
      }
  }
}

static void hop_apply(const double* U, const Geo& g, const cd* x, cd* y, double c_hop, double c_diag) {
  // y = c_hop * hop(x) + c_diag * x
#pragma omp parallel for schedule(static)
  for (int k = 0; k < g.V3; ++k) {
    cd acc[3] = {0.0, 0.0, 0.0};
    for (int mu = 0; mu < 3; ++mu) {
      const int up = g.up(k, mu), dn = g.dn(k, mu);
      const double* uf = U + (size_t)(k * 3 + mu) * 18;
      const double* ub = U + (size_t)(dn * 3 + mu) * 18;
      for (int a = 0; a < 3; ++a) {
        cd s = 0.0;
        for (int b = 0; b < 3; ++b) {
          s += cd(uf[2 * (3 * a + b)], uf[2 * (3 * a + b) + 1]) * x[3 * up + b];
          s += std::conj(cd(ub[2 * (3 * b + a)], ub[2 * (3 * b + a) + 1])) * x[3 * dn + b];
        }
        acc[a] += s;
      }
    }
    for (int a = 0; a < 3; ++a) y[3 * k + a] = c_hop * acc[a] + c_diag * x[3 * k + a];
  }
}

/* tv2, modules/shell_matop.cpp:16-103: y = c(hop(x) - 6x) + a x */
void orc_tv2(const double* U, int L, double lam_l, double lam_c, const double* x, double* y) {
  Geo g(L);
  const double c = 2.0 / (lam_l - lam_c);
  const double a = 1.0 + c * lam_c;
  hop_apply(U, g, reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y), c, a - 6.0 * c);
}

/* tv_iter, modules/shell_matop.cpp:136-168 */
void orc_tv_iter(const double* U, int L, double lam_l, double lam_c, int deg, const double* x, double* y) {
  const long n = 3L * L * L * L;
  std::vector<cd> Told(n), Tcur(n), tmp(n);
  orc_tv2(U, L, lam_l, lam_c, x, reinterpret_cast<double*>(Tcur.data()));
  std::memcpy(static_cast<void*>(Told.data()), x, n * sizeof(cd));
  cd* yc = reinterpret_cast<cd*>(y);
  for (int k = 2; k <= deg; ++k) {
    orc_tv2(U, L, lam_l, lam_c, reinterpret_cast<const double*>(Tcur.data()), reinterpret_cast<double*>(tmp.data()));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
      yc[i] = 2.0 * tmp[i] - Told[i];
      Told[i] = Tcur[i];
      Tcur[i] = yc[i];
    }
  }
}

void orc_neglap(const double* U, int L, const double* x, double* y) {
  Geo g(L);
  hop_apply(U, g, reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y), -1.0, 6.0);
}

/* plaque_timeslice, modules/config_utils.cpp:388-426 */
double orc_plaquette(const double* U, int L) {
  Geo g(L);
  double p = 0.0;
  long cnt = 0;
  for (int i = 0; i < g.V3; ++i)
    for (int d1 = 0; d1 < 3; ++d1)
      for (int d2 = 0; d2 < 3; ++d2) {
        if (d1 == d2) continue;
        int j = g.up(i, d1), k = g.up(j, d2), l = g.dn(k, d1);
        M3 pl = mul(link(U, i, d1), mul(link(U, j, d2), mul(adj(link(U, l, d1)), adj(link(U, i, d2)))));
        p += (pl.m[0] + pl.m[4] + pl.m[8]).real() / 3.0;
        ++cnt;
      }
  return p / (double)cnt;
}

/* SLEPc EPS Krylov-Schur on T_deg(B) (src/ev_ts.cpp:231-263), restated. */
int orc_eps_solve(const double* U, int L, double lam_l, double lam_c, int deg, int nev, int ncv, double tol,
                  int max_it, uint64_t seed, double* theta_out, double* V_out, int* nconv_out, int* its_out,
                  long long* nmatvec_out) {
  const long dim = 3L * L * L * L;
  if (ncv <= 0) ncv = std::max(2 * nev, nev + 15);
  if (ncv > dim) ncv = (int)dim;
  const int m = ncv;
  std::vector<cd> V((size_t)dim * (m + 1)), w(dim), h(m + 1), h2(m + 1);
  std::vector<double> T((size_t)m * m, 0.0);
  long long nmv = 0;
  auto op = [&](const cd* x, cd* y) {
    ++nmv;
    if (deg >= 2) orc_tv_iter(U, L, lam_l, lam_c, deg, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y));
    else orc_tv2(U, L, lam_l, lam_c, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y));
  };
  auto col = [&](int j) { return V.data() + (size_t)j * dim; };
  // start vector
  {
    SplitMix rng(seed);
    double nrm = 0.0;
    for (long i = 0; i < dim; ++i) {
      double u1 = rng.uniform(), u2 = rng.uniform();
      double r = std::sqrt(-2.0 * std::log(u1));
      col(0)[i] = cd(r * std::cos(2 * M_PI * u2), r * std::sin(2 * M_PI * u2));
      nrm += std::norm(col(0)[i]);
    }
    nrm = 1.0 / std::sqrt(nrm);
    for (long i = 0; i < dim; ++i) col(0)[i] *= nrm;
  }
  int k = 0;  // kept vectors (arrow) before v_k
  std::vector<double> arrow;
  std::vector<double> d, Z;
  std::vector<int> ord(m);
  int nconv = 0, it = 0, info = 1;
  double beta_m = 0.0;
  std::vector<cd> Vnew;
  for (it = 1; it <= max_it; ++it) {
    // expand
    for (int j = k; j < m; ++j) {
      op(col(j), w.data());
      // classical Gram-Schmidt, applied twice
      for (int pass = 0; pass < 2; ++pass) {
        cd* hh = pass == 0 ? h.data() : h2.data();
#pragma omp parallel for schedule(static)
        for (int c = 0; c <= j; ++c) {
          cd s = 0.0;
          const cd* vc = col(c);
          for (long i = 0; i < dim; ++i) s += std::conj(vc[i]) * w[i];
          hh[c] = s;
        }
#pragma omp parallel for schedule(static)
        for (long i0 = 0; i0 < dim; i0 += 512) {
          const long i1 = std::min(dim, i0 + 512);
          for (int c = 0; c <= j; ++c) {
            const cd a = hh[c];
            const cd* vc = col(c);
            for (long i = i0; i < i1; ++i) w[i] -= vc[i] * a;
          }
        }
      }
      for (int c = 0; c <= j; ++c) h[c] += h2[c];
      double beta = 0.0;
#pragma omp parallel for reduction(+ : beta)
      for (long i = 0; i < dim; ++i) beta += std::norm(w[i]);
      beta = std::sqrt(beta);
      T[(size_t)j * m + j] = h[j].real();
      if (j + 1 < m) T[(size_t)j * m + j + 1] = T[(size_t)(j + 1) * m + j] = beta;
      beta_m = beta;
      const double ib = 1.0 / beta;
      cd* vn = col(j + 1);
#pragma omp parallel for schedule(static)
      for (long i = 0; i < dim; ++i) vn[i] = w[i] * ib;
    }
    // projected problem
    std::vector<double> A = T;
    sym_jacobi(m, A, d, Z);
    for (int i = 0; i < m; ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return std::fabs(d[a]) > std::fabs(d[b]); });
    int nc = 0;
    for (int i = 0; i < m; ++i) {
      const int o = ord[i];
      const double res = std::fabs(beta_m * Z[(size_t)(m - 1) * m + o]);
      if (res <= tol * std::fabs(d[o])) ++nc;
      else break;
    }
    nconv = nc;
    const bool done = nconv >= nev || it == max_it;
    int keep = done ? std::max(nev, 1) : nconv + std::max(1, (m - nconv) / 2);
    if (keep > m - 1 && !done) keep = m - 1;
    // V[:, 0:keep] = V[:, 0:m] Z[:, ord[0:keep]]
    Vnew.assign((size_t)dim * keep, 0.0);
#pragma omp parallel for schedule(static)
    for (long i0 = 0; i0 < dim; i0 += 256) {
      const long i1 = std::min(dim, i0 + 256);
      for (int c = 0; c < keep; ++c) {
        const int o = ord[c];
        cd* dst = &Vnew[(size_t)c * dim];
        for (int r = 0; r < m; ++r) {
          const double z = Z[(size_t)r * m + o];
          const cd* vr = col(r);
          for (long i = i0; i < i1; ++i) dst[i] += vr[i] * z;
        }
      }
    }
    if (done) {
      for (int c = 0; c < nev; ++c) theta_out[c] = d[ord[c]];
      std::memcpy(V_out, Vnew.data(), (size_t)dim * nev * sizeof(cd));
      info = nconv >= nev ? 0 : 1;
      break;
    }
    std::memcpy(col(keep), col(m), dim * sizeof(cd));
    std::memcpy(V.data(), Vnew.data(), (size_t)dim * keep * sizeof(cd));
    std::fill(T.begin(), T.end(), 0.0);
    for (int c = 0; c < keep; ++c) {
      T[(size_t)c * m + c] = d[ord[c]];
      const double b = beta_m * Z[(size_t)(m - 1) * m + ord[c]];
      T[(size_t)c * m + keep] = T[(size_t)keep * m + c] = b;
    }
    k = keep;
  }
  if (it > max_it) it = max_it;
  if (nconv_out) *nconv_out = nconv;
  if (its_out) *its_out = it;
  if (nmatvec_out) *nmatvec_out = nmv;
  return info;
}

/* recover_spectrum / invert_Tn / invert_B, modules/recover_spec.cpp:13-54 */
void orc_recover_spectrum(int nev, const double* theta, int deg, double lam_l, double lam_c, double* out) {
  for (int i = 0; i < nev; ++i) {
    double b = std::cosh(1.0 / deg * std::acosh(theta[i]));
    out[i] = (lam_l - lam_c) * (b - 1) * 0.5 - lam_c;
  }
}

/* fix_phase, modules/eigensystem.cpp:4-30 */
void orc_fix_phase(int dim, int nev, const double* V, double* Vfix, double* phase) {
  const cd* v = reinterpret_cast<const cd*>(V);
  cd* vf = reinterpret_cast<cd*>(Vfix);
  for (int n = 0; n < nev; ++n) {
    const double ph = std::arg(v[(size_t)n * dim]);
    phase[n] = ph;
    const cd fac = std::exp(cd(0.0, -1.0) * ph);
    for (long i = 0; i < dim; ++i) vf[(size_t)n * dim + i] = fac * v[(size_t)n * dim + i];
  }
}

/* reset_phase, modules/eigensystem.cpp:32-57: V_reset(:, n) = exp(-i (arg V(0, n) - want_n)) V(:, n) */
void orc_reset_phase(int dim, int nev, const double* V, const double* phase_want, double* Vreset) {
  const cd* v = reinterpret_cast<const cd*>(V);
  cd* vr = reinterpret_cast<cd*>(Vreset);
  for (int n = 0; n < nev; ++n) {
    const cd fac = std::exp(cd(0.0, -1.0) * (std::arg(v[(size_t)n * dim]) - phase_want[n]));
    for (long i = 0; i < dim; ++i) vr[(size_t)n * dim + i] = fac * v[(size_t)n * dim + i];
  }
}

/* BuildLaplacian analogue (modules/config_utils.cpp:18-58): 6 on the diagonal,
 * -U_mu(i)(a,b) at (3i+a, 3up+b), -U_mu(dn)^dag(a,b) at (3i+a, 3dn+b). */
void orc_build_neglap_dense(const double* U, int L, double* Aout) {
  Geo g(L);
  const long dim = 3L * g.V3;
  cd* A = reinterpret_cast<cd*>(Aout);
  std::fill(A, A + dim * dim, cd(0.0));
  for (int i = 0; i < g.V3; ++i) {
    for (int a = 0; a < 3; ++a) A[(3L * i + a) * dim + 3L * i + a] += 6.0;
    for (int mu = 0; mu < 3; ++mu) {
      const int up = g.up(i, mu), dn = g.dn(i, mu);
      M3 uf = link(U, i, mu), ub = adj(link(U, dn, mu));
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          A[(3L * i + a) * dim + 3L * up + b] -= uf.m[3 * a + b];
          A[(3L * i + a) * dim + 3L * dn + b] -= ub.m[3 * a + b];
        }
    }
  }
}

/* Loss and gradient of the window MLP (16 -> 64 -> 64 -> 3, tanh) in FP64:
 * L = mean_{i,k} (O_ik - Y_ik)^2, parameters W1[64][16] b1 W2[64][64] b2
 * W3[3][64] b3.  The CPU check for the device training kernels (this part
 * has no counterpart in the reference). */
double orc_mlp_loss_grad(const double* P, const double* X, const double* Y, int n, double* grad) {
  const int I = 16, H = 64, O = 3;
  const int oW1 = 0, ob1 = H * I, oW2 = ob1 + H, ob2 = oW2 + H * H, oW3 = ob2 + H, ob3 = oW3 + O * H, np_ = ob3 + O;
  std::fill(grad, grad + np_, 0.0);
  double loss = 0.0;
  std::vector<double> h1(H), h2(H), d1(H), d2(H);
  const double sc = 2.0 / (n * O);
  for (int i = 0; i < n; ++i) {
    const double* x = X + (size_t)i * I;
    for (int j = 0; j < H; ++j) {
      double z = P[ob1 + j];
      for (int q = 0; q < I; ++q) z += P[oW1 + j * I + q] * x[q];
      h1[j] = std::tanh(z);
    }
    for (int j = 0; j < H; ++j) {
      double z = P[ob2 + j];
      for (int q = 0; q < H; ++q) z += P[oW2 + j * H + q] * h1[q];
      h2[j] = std::tanh(z);
    }
    double dout[3];
    for (int k = 0; k < O; ++k) {
      double o = P[ob3 + k];
      for (int q = 0; q < H; ++q) o += P[oW3 + k * H + q] * h2[q];
      const double d = o - Y[(size_t)i * O + k];
      loss += d * d;
      dout[k] = sc * d;
    }
    for (int j = 0; j < H; ++j) {
      double dh = 0.0;
      for (int k = 0; k < O; ++k) {
        grad[oW3 + k * H + j] += dout[k] * h2[j];
        dh += P[oW3 + k * H + j] * dout[k];
      }
      d2[j] = dh * (1.0 - h2[j] * h2[j]);
    }
    for (int k = 0; k < O; ++k) grad[ob3 + k] += dout[k];
    for (int j = 0; j < H; ++j) {
      for (int q = 0; q < H; ++q) grad[oW2 + j * H + q] += d2[j] * h1[q];
      grad[ob2 + j] += d2[j];
      double dh = 0.0;
      for (int r = 0; r < H; ++r) dh += P[oW2 + r * H + j] * d2[r];
      d1[j] = dh * (1.0 - h1[j] * h1[j]);
    }
    for (int j = 0; j < H; ++j) {
      for (int q = 0; q < I; ++q) grad[oW1 + j * I + q] += d1[j] * x[q];
      grad[ob1 + j] += d1[j];
    }
  }
  return loss / (n * O);
}

// right_displacement_one_dir (modules/config_utils.cpp:344-382):
// W_i(x) = 1/2 (U_dir(x) V_i(x+dir) - U_dir(x-dir)^dag V_i(x-dir)).
void orc_displace(const double* links3, int L, int dir, const double* Vd, int nev, double* Wd) {
  const cd* V = reinterpret_cast<const cd*>(Vd);
  cd* W = reinterpret_cast<cd*>(Wd);
  const long long V3 = (long long)L * L * L, dim = 3 * V3;
  const Geo nav(L);
#pragma omp parallel for schedule(static)
  for (long long s = 0; s < V3; ++s) {
    const int up = nav.up((int)s, dir), dn = nav.dn((int)s, dir);
    const M3 U = load(links3 + ((size_t)s * 3 + dir) * 18);
    const M3 Ud = adj(load(links3 + ((size_t)dn * 3 + dir) * 18));
    for (int n = 0; n < nev; ++n)
      for (int a = 0; a < 3; ++a) {
        cd f = 0.0, b = 0.0;
        for (int c = 0; c < 3; ++c) {
          f += U.m[3 * a + c] * V[3 * up + c + n * dim];
          b += Ud.m[3 * a + c] * V[3 * dn + c + n * dim];
        }
        W[3 * s + a + n * dim] = 0.5 * (f - b);
      }
  }
}

// source_shape_complete (modules/sourceshape_funcs.cpp:58-81) with dll_op
// (:30-55) and get_vectorial_dst_ind (:11-27): for r = (r1, r2, r3) on the grid
// r_i = 0, 2, ... < L (r1 outer, r3 inner), psi(r) = sum over sites x of
// sqrt(tr(M M^dag)), M = V_{x+r} V_x^dag with V_y the 3 x nev block of rows
// 3y .. 3y+2 of the column-major eigensystem; x+r steps r_i times up in
// direction i with the periodic neighbours of modules/navigation.cpp.
void orc_sourceshape(const double* Vd, int L, int nev, double* psi) {
  const cd* V = reinterpret_cast<const cd*>(Vd);
  const long long V3 = (long long)L * L * L, dim = 3 * V3;
  int idx = 0;
  std::vector<std::array<int, 3>> grid;
  for (int r1 = 0; r1 < L; r1 += 2)
    for (int r2 = 0; r2 < L; r2 += 2)
      for (int r3 = 0; r3 < L; r3 += 2) grid.push_back({r1, r2, r3});
  for (const auto& r : grid) {
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (long long s = 0; s < V3; ++s) {
      const int x = (int)(s / (L * L)), y = (int)((s / L) % L), z = (int)(s % L);
      const long long dst = (long long)((x + r[0]) % L) * L * L + ((y + r[1]) % L) * L + (z + r[2]) % L;
      double fro = 0.0;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          cd m = 0.0;
          for (int n = 0; n < nev; ++n) m += V[3 * dst + a + n * dim] * std::conj(V[3 * s + b + n * dim]);
          fro += std::norm(m);
        }
      acc += std::sqrt(fro);
    }
    psi[idx++] = acc;
  }
}

// avg_radii (modules/sourceshape_funcs.cpp:100-135): psi averaged over grid
// points of equal |r| (within 1e-11), radii in order of first appearance.
int orc_sourceshape_avg(int L, const double* psi, double* r_out, double* psi_out) {
  std::vector<int> cnt;
  std::vector<double> rad, sum;
  int idx = 0;
  for (int r1 = 0; r1 < L; r1 += 2)
    for (int r2 = 0; r2 < L; r2 += 2)
      for (int r3 = 0; r3 < L; r3 += 2) {
        const double len = std::sqrt((double)(r1 * r1 + r2 * r2 + r3 * r3));
        bool found = false;
        for (size_t t = 0; t < rad.size(); ++t)
          if (std::fabs(len - rad[t]) < 1e-11) {
            ++cnt[t];
            sum[t] += psi[idx];
            found = true;
          }
        if (!found) {
          cnt.push_back(1);
          rad.push_back(len);
          sum.push_back(psi[idx]);
        }
        ++idx;
      }
  for (size_t t = 0; t < rad.size(); ++t) {
    r_out[t] = rad[t];
    psi_out[t] = sum[t] / cnt[t];
  }
  return (int)rad.size();
}

}  // extern "C"
