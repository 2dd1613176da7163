// su3.cuh -- FP64 3x3 complex algebra on the device: products, adjoint,
// Hermitian Jacobi eigendecomposition, the SU(3) projection of the reference's
// proj_to_su3_imp (modules/timeslice.cpp:90-104) and exp(iH) for stout.
//
// Eigen's Matrix3cd::sqrt()/inverse()/exp() (which the reference calls) are
// replaced by one primitive: a cyclic Jacobi eigendecomposition A = Q D Q^dag
// of a Hermitian 3x3, giving (M^dag M)^{-1/2} = Q D^{-1/2} Q^dag and
// exp(iH) = Q e^{iD} Q^dag.  Both are the unique principal functions, so the
// results agree with the reference's to rounding.
#pragma once
#include "common.cuh"

namespace laph {

struct M3 {
  double2 e[9];  // row-major (a,b) -> e[3a+b]
};

// Links of one timeslice live in "site-minor" order: element e (0..8) of the
// link in direction dir at site s is U[(dir*9 + e)*V3 + s], so a warp of
// consecutive sites reads each element with one coalesced 512-byte access.
__device__ __forceinline__ M3 ld_link(const double2* __restrict__ U, int V3, int s, int dir) {
  M3 m;
#pragma unroll
  for (int e = 0; e < 9; ++e) m.e[e] = __ldg(U + (size_t)(dir * 9 + e) * V3 + s);
  return m;
}
__device__ __forceinline__ void st_link(double2* __restrict__ U, int V3, int s, int dir, const M3& m) {
#pragma unroll
  for (int e = 0; e < 9; ++e) U[(size_t)(dir * 9 + e) * V3 + s] = m.e[e];
}

__device__ __forceinline__ M3 m3_zero() {
  M3 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r.e[i] = make_double2(0.0, 0.0);
  return r;
}
__device__ __forceinline__ M3 m3_id() {
  M3 r = m3_zero();
  r.e[0].x = r.e[4].x = r.e[8].x = 1.0;
  return r;
}
__device__ __forceinline__ M3 m3_mul(const M3& a, const M3& b) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double2 s = cmul(a.e[3 * i], b.e[j]);
      cfma(s, a.e[3 * i + 1], b.e[3 + j]);
      cfma(s, a.e[3 * i + 2], b.e[6 + j]);
      r.e[3 * i + j] = s;
    }
  return r;
}
// a^dag * b
__device__ __forceinline__ M3 m3_adj_mul(const M3& a, const M3& b) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double2 s = cmulc(a.e[i], b.e[j]);
      cfmac(s, a.e[3 + i], b.e[3 + j]);
      cfmac(s, a.e[6 + i], b.e[6 + j]);
      r.e[3 * i + j] = s;
    }
  return r;
}
// a * b^dag
__device__ __forceinline__ M3 m3_mul_adj(const M3& a, const M3& b) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double2 s = cmul(a.e[3 * i], cconj(b.e[3 * j]));
      cfma(s, a.e[3 * i + 1], cconj(b.e[3 * j + 1]));
      cfma(s, a.e[3 * i + 2], cconj(b.e[3 * j + 2]));
      r.e[3 * i + j] = s;
    }
  return r;
}
__device__ __forceinline__ M3 m3_adj(const M3& a) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.e[3 * i + j] = cconj(a.e[3 * j + i]);
  return r;
}
__device__ __forceinline__ void m3_acc(M3& a, const M3& b) {
#pragma unroll
  for (int i = 0; i < 9; ++i) a.e[i] = cadd(a.e[i], b.e[i]);
}
// a*s + b*t (real s, t)
__device__ __forceinline__ M3 m3_lin(const M3& a, double s, const M3& b, double t) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 9; ++i) r.e[i] = make_double2(a.e[i].x * s + b.e[i].x * t, a.e[i].y * s + b.e[i].y * t);
  return r;
}
__device__ __forceinline__ double2 m3_det(const M3& a) {
  const double2* m = a.e;
  double2 t0 = csub(cmul(m[4], m[8]), cmul(m[5], m[7]));
  double2 t1 = csub(cmul(m[3], m[8]), cmul(m[5], m[6]));
  double2 t2 = csub(cmul(m[3], m[7]), cmul(m[4], m[6]));
  return cadd(csub(cmul(m[0], t0), cmul(m[1], t1)), cmul(m[2], t2));
}

// Cyclic Jacobi on a Hermitian 3x3: A = Q diag(d) Q^dag.  For the pair (p,q)
// with A_pq = r e^{i phi} the unitary J = P R, P = diag(1, e^{-i phi}) on
// (p,q) and R the real Jacobi rotation of [[a_pp, r], [r, a_qq]], zeroes A_pq.
__device__ __forceinline__ void herm3_eig(M3 A, double d[3], M3& Q) {
  Q = m3_id();
  const int P[3] = {0, 0, 1}, QQ[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 12; ++sweep) {
    const double off = A.e[1].x * A.e[1].x + A.e[1].y * A.e[1].y + A.e[2].x * A.e[2].x + A.e[2].y * A.e[2].y +
                       A.e[5].x * A.e[5].x + A.e[5].y * A.e[5].y;
    const double dg = A.e[0].x * A.e[0].x + A.e[4].x * A.e[4].x + A.e[8].x * A.e[8].x;
    if (off <= 1e-34 * dg || off == 0.0) break;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int p = P[k], q = QQ[k];
      const double2 g = A.e[3 * p + q];
      const double r = hypot(g.x, g.y);
      if (r == 0.0) continue;
      const double2 emph = make_double2(g.x / r, -g.y / r);  // e^{-i phi}
      const double app = A.e[4 * p].x, aqq = A.e[4 * q].x;
      const double tau = (aqq - app) / (2.0 * r);
      const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
      const double c = 1.0 / sqrt(1.0 + t * t);
      const double s = t * c;
      M3 J = m3_id();
      J.e[3 * p + p] = make_double2(c, 0.0);
      J.e[3 * p + q] = make_double2(s, 0.0);
      J.e[3 * q + p] = cscal(emph, -s);
      J.e[3 * q + q] = cscal(emph, c);
      A = m3_adj_mul(J, m3_mul(A, J));
      A.e[3 * p + q] = make_double2(0.0, 0.0);
      A.e[3 * q + p] = make_double2(0.0, 0.0);
      Q = m3_mul(Q, J);
    }
  }
  d[0] = A.e[0].x;
  d[1] = A.e[4].x;
  d[2] = A.e[8].x;
}

// Q diag(f) Q^dag
__device__ __forceinline__ M3 m3_qfq(const M3& Q, const double2 f[3]) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 3; ++k) cfma(s, cmul(Q.e[3 * i + k], f[k]), cconj(Q.e[3 * j + k]));
      r.e[3 * i + j] = s;
    }
  return r;
}

// proj_to_su3_imp (modules/timeslice.cpp:90-104): W = M (M^dag M)^{-1/2};
// W <- W / det(W)^{1/3} with the principal complex cube root (std::pow).
__device__ __forceinline__ M3 proj_su3(const M3& M) {
  const M3 A = m3_adj_mul(M, M);
  double d[3];
  M3 Q;
  herm3_eig(A, d, Q);
  double2 f[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) f[i] = make_double2(1.0 / sqrt(d[i]), 0.0);
  M3 W = m3_mul(M, m3_qfq(Q, f));
  const double2 det = m3_det(W);
  double2 fac;
  if (det.y == 0.0 && det.x > 0.0) {
    fac = make_double2(1.0 / pow(det.x, 1.0 / 3.0), 0.0);
  } else {
    const double mag = exp(log(hypot(det.x, det.y)) / 3.0);
    const double ph = atan2(det.y, det.x) / 3.0;
    double sn, cs;
    sincos(ph, &sn, &cs);
    // 1 / (mag e^{i ph}) = e^{-i ph} / mag
    fac = make_double2(cs / mag, -sn / mag);
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) W.e[i] = cmul(W.e[i], fac);
  return W;
}

// exp(i H) for Hermitian H.
__device__ __forceinline__ M3 expiH(const M3& H) {
  double d[3];
  M3 Q;
  herm3_eig(H, d, Q);
  double2 f[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double sn, cs;
    sincos(d[i], &sn, &cs);
    f[i] = make_double2(cs, sn);
  }
  return m3_qfq(Q, f);
}

}  // namespace laph
