// ORACLE — test infrastructure, not product code.
//
// f64 CPU restatement of the reference's dynamic-relaxation solver (uwenji/weave-sim, web/js/solver_cpu.js with
// web/js/rod_cosserat.js, web/js/model.js and web/js/quat.js).  It is the checker of the CUDA path: only the tests,
// the smoke check and the CPU-baseline leg of the benchmark load it.  It follows the JavaScript line by line and keeps
// its order of operations, including the numpy-order pairwise sums that steer kinetic damping:
//   quat helpers              web/js/quat.js:4-57
//   relRotation, CosseratRod  web/js/rod_cosserat.js:33-209
//   nodeQuats, Anchors        web/js/model.js:89-105, 162-189
//   pairwiseSum               web/js/solver_cpu.js:42-54
//   PolylineContact (core)    web/js/solver_cpu.js:99-228, 274-282, 381-478
//   CpuSolver goals / step    web/js/solver_cpu.js:670-710, 719-732, 737-853, 868
//   buildResults (segment)    web/js/solver_cpu.js:878-898
// Not restated (not on this path's configurations): the W2 rotational friction, the W3 seat law, the augmented
// Lagrangian, the Floor goal and the rigid-body freedoms.  Math.* differs from libm in the last ulp, so this oracle is
// the reference's semantics, not a bit-copy of V8's arithmetic; it is pinned by the reference's own known-answer
// tests (finite-difference gradient, closed-form beams, crossing cases) in tests/test_oracle_known_answers.py.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

#include "../include/weavesim.h"

namespace orc {

static const double SUPPORT_SMOOTH = 0.03;
static const double TWIST_RATE_MAX = 0.5 * SUPPORT_SMOOTH;
static const double ROLL_DAMP = 0.5;
static const double INF = std::numeric_limits<double>::infinity();
static const double AL_FREE_MIN = 0.25;               // solver_cpu.js:33
// the rigid-body freedoms of a model that only the ground holds (solver_cpu.js:35-39)
static const double RB_MASS = 2.0, RB_VMAX = 0.05, RB_LEVER = 0.05;
static const double PI = 3.141592653589793;           // Math.PI
// Math.sign: −1, 0 or +1 (0 for ±0)
static double jsSign(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); }

// ------------------------------------------------------------------------------------------------ quat.js
static void qnormalize(double *q) {
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (n == 0) n = 1.0;
  q[0] /= n; q[1] /= n; q[2] /= n; q[3] /= n;
}
static void qmul(const double *a, const double *b, double *out) {
  double aw = a[0], ax = a[1], ay = a[2], az = a[3], bw = b[0], bx = b[1], by = b[2], bz = b[3];
  out[0] = aw * bw - ax * bx - ay * by - az * bz;
  out[1] = aw * bx + ax * bw + ay * bz - az * by;
  out[2] = aw * by - ax * bz + ay * bw + az * bx;
  out[3] = aw * bz + ax * by - ay * bx + az * bw;
}
static void toFrame(const double *Q, double *R) {
  double w = Q[0], x = Q[1], y = Q[2], z = Q[3];
  double n = std::sqrt(w * w + x * x + y * y + z * z);
  if (n == 0) n = 1.0;
  w /= n; x /= n; y /= n; z /= n;
  R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y + z * w); R[2] = 2 * (x * z - y * w);
  R[3] = 2 * (x * y - z * w); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z + x * w);
  R[6] = 2 * (x * z + y * w); R[7] = 2 * (y * z - x * w); R[8] = 1 - 2 * (x * x + y * y);
}
static void qexp(double tx, double ty, double tz, double *out) {
  double a = std::sqrt(tx * tx + ty * ty + tz * tz), half = 0.5 * a;
  double s = a > 1e-12 ? std::sin(half) / a : 0.5;
  out[0] = std::cos(half); out[1] = tx * s; out[2] = ty * s; out[3] = tz * s;
}

// rod_cosserat.js:33-45: Ψ = log(q_a* ⊗ q_b), returns θ
static double relRotation(const double *qa, const double *qb, double *out) {
  double aw = qa[0], ax = -qa[1], ay = -qa[2], az = -qa[3];
  double bw = qb[0], bx = qb[1], by = qb[2], bz = qb[3];
  double w = aw * bw - ax * bx - ay * by - az * bz;
  double x = aw * bx + ax * bw + ay * bz - az * by;
  double y = aw * by - ax * bz + ay * bw + az * bx;
  double z = aw * bz + ax * by - ay * bx + az * bw;
  if (w < 0) { w = -w; x = -x; y = -y; z = -z; }
  double s = std::sqrt(x * x + y * y + z * z), th = 2 * std::atan2(s, w);
  double f = s > 1e-12 ? th / s : 2 / std::max(w, 1e-12);
  out[0] = f * x; out[1] = f * y; out[2] = f * z;
  return th;
}

// solver_cpu.js:42-54
static double pairwiseSum(const double *a, size_t lo, size_t n) {
  if (n < 8) { double r = 0; for (size_t i = 0; i < n; i++) r += a[lo + i]; return r; }
  if (n <= 128) {
    double r[8];
    for (int k = 0; k < 8; k++) r[k] = a[lo + k];
    size_t i = 8;
    for (; i < n - (n % 8); i += 8) for (int k = 0; k < 8; k++) r[k] += a[lo + i + k];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; i++) res += a[lo + i];
    return res;
  }
  size_t n2 = n >> 1;
  n2 -= n2 % 8;
  return pairwiseSum(a, lo, n2) + pairwiseSum(a, lo + n2, n - n2);
}
static double pairwiseSum(const std::vector<double> &a) { return pairwiseSum(a.data(), 0, a.size()); }

// ------------------------------------------------------------------------------------------------ state
struct St {
  int n = 0, m = 0, p = 0, K = 0, S = 0;
  std::vector<double> X, X0, V, Q, Q0, Wr, l0, jLen, Omega0, u, nPrev, slip;
  std::vector<int> segI0, segI1, segOffset, jSeg0, jSeg1;
  std::vector<uint8_t> stuck;
  int iteration = 0;
  double residual = INF;
};

// model.js:89-105
static void nodeQuats(const St &st, std::vector<double> &out) {
  std::vector<int> ref(st.n, -1);
  for (int j = 0; j < st.m; j++) ref[st.segI1[j]] = j;
  for (int j = 0; j < st.m; j++) ref[st.segI0[j]] = j;
  out.assign(4 * size_t(st.n), 0.0);
  const double *Q = st.Q.data();
  for (const std::vector<int> *idx : {&st.segI0, &st.segI1})
    for (int j = 0; j < st.m; j++) {
      int i = (*idx)[j], r = ref[i];
      double dot = Q[4 * j] * Q[4 * r] + Q[4 * j + 1] * Q[4 * r + 1] + Q[4 * j + 2] * Q[4 * r + 2] + Q[4 * j + 3] * Q[4 * r + 3];
      double sg = dot < 0 ? -1 : 1;
      for (int c = 0; c < 4; c++) out[4 * size_t(i) + c] += sg * Q[4 * j + c];
    }
  for (int i = 0; i < st.n; i++) qnormalize(&out[4 * size_t(i)]);
}

// ------------------------------------------------------------------------------------------------ CosseratRod
struct Clamp { int node, seg; bool mk[3]; };

struct Rod {
  std::vector<double> segEA, segEIx, segEIy, segGJ, segGA, EIx, EIy, GJ;
  std::vector<double> N, Vs, M, R, kDyn;
  std::vector<int> cNode, cSeg;
  std::vector<double> cLen, cB, cQ, cM;
  double energy = 0, eBend = 0, eTwist = 0, eStretch = 0, eShear = 0;

  void init(const St &st, const ws_model &md) {
    const int m = st.m, p = st.p;
    segEA.assign(md.EA, md.EA + m); segEIx.assign(md.EIx, md.EIx + m); segEIy.assign(md.EIy, md.EIy + m);
    segGJ.assign(md.GJ, md.GJ + m); segGA.assign(md.GA, md.GA + m);
    EIx.resize(p); EIy.resize(p); GJ.resize(p);
    for (int j = 0; j < p; j++) { int s0 = st.jSeg0[j]; EIx[j] = segEIx[s0]; EIy[j] = segEIy[s0]; GJ[j] = segGJ[s0]; }
    N.assign(m, 0.0); Vs.assign(2 * size_t(m), 0.0); M.assign(3 * size_t(p), 0.0);
    R.assign(9 * size_t(m), 0.0); kDyn.assign(3 * size_t(m), 0.0);
  }
  // rod_cosserat.js:92-100
  void setClamps(const St &st, const std::vector<Clamp> &rc) {
    const size_t nc = rc.size();
    cNode.clear(); cSeg.clear(); cLen.clear(); cB.clear();
    for (const Clamp &c : rc) {
      cNode.push_back(c.node); cSeg.push_back(c.seg); cLen.push_back(0.5 * st.l0[c.seg]);
      cB.push_back(c.mk[0] ? segEIx[c.seg] : 0); cB.push_back(c.mk[1] ? segEIy[c.seg] : 0); cB.push_back(c.mk[2] ? segGJ[c.seg] : 0);
    }
    cQ.assign(4 * nc, 0.0);
    for (size_t c = 0; c < nc; c++) for (int k = 0; k < 4; k++) cQ[4 * c + k] = st.Q[4 * size_t(cSeg[c]) + k];
    cM.assign(2 * nc, 0.0);
  }
  // rod_cosserat.js:114-183
  void apply(const St &st, double *F, double *T) {
    const double *X = st.X.data(), *Q = st.Q.data();
    const int m = st.m, p = st.p;
    for (int j = 0; j < m; j++) toFrame(Q + 4 * size_t(j), &R[9 * size_t(j)]);
    double es = 0, esh = 0, eb = 0, et = 0;
    for (int j = 0; j < m; j++) {
      const int a = st.segI0[j], b = st.segI1[j];
      const size_t o = 9 * size_t(j);
      const double l0 = st.l0[j];
      const double ex = X[3 * size_t(b)] - X[3 * size_t(a)];
      const double ey = X[3 * size_t(b) + 1] - X[3 * size_t(a) + 1], ez = X[3 * size_t(b) + 2] - X[3 * size_t(a) + 2];
      const double s1 = (R[o] * ex + R[o + 1] * ey + R[o + 2] * ez) / l0;
      const double s2 = (R[o + 3] * ex + R[o + 4] * ey + R[o + 5] * ez) / l0;
      const double s3 = (R[o + 6] * ex + R[o + 7] * ey + R[o + 8] * ez) / l0 - 1.0;
      const double n1 = segGA[j] * s1, n2 = segGA[j] * s2, n3 = segEA[j] * s3;
      const double nx = n1 * R[o] + n2 * R[o + 3] + n3 * R[o + 6];
      const double ny = n1 * R[o + 1] + n2 * R[o + 4] + n3 * R[o + 7];
      const double nz = n1 * R[o + 2] + n2 * R[o + 5] + n3 * R[o + 8];
      F[3 * size_t(a)] += nx; F[3 * size_t(a) + 1] += ny; F[3 * size_t(a) + 2] += nz;
      F[3 * size_t(b)] -= nx; F[3 * size_t(b) + 1] -= ny; F[3 * size_t(b) + 2] -= nz;
      T[3 * size_t(j)] += ey * nz - ez * ny; T[3 * size_t(j) + 1] += ez * nx - ex * nz; T[3 * size_t(j) + 2] += ex * ny - ey * nx;
      N[j] = n3; Vs[2 * size_t(j)] = n1; Vs[2 * size_t(j) + 1] = n2;
      es += 0.5 * l0 * n3 * s3; esh += 0.5 * l0 * (n1 * s1 + n2 * s2);
    }
    double psi[3];
    std::fill(kDyn.begin(), kDyn.end(), 0.0);
    for (int j = 0; j < p; j++) {
      const int sa = st.jSeg0[j], sb = st.jSeg1[j];
      const double lb = st.jLen[j];
      const size_t o = 9 * size_t(sa);
      const double th = relRotation(Q + 4 * size_t(sa), Q + 4 * size_t(sb), psi);
      const double d0 = psi[0] / lb - st.Omega0[3 * size_t(j)], d1 = psi[1] / lb - st.Omega0[3 * size_t(j) + 1], d2 = psi[2] / lb - st.Omega0[3 * size_t(j) + 2];
      const double m0 = EIx[j] * d0, m1 = EIy[j] * d1, m2 = GJ[j] * d2;
      {
        const double q0 = psi[0] * psi[0], q1 = psi[1] * psi[1], q2 = psi[2] * psi[2], f = 0.25 / lb;
        const double k0 = f * (EIy[j] * q2 + GJ[j] * q1), k1 = f * (EIx[j] * q2 + GJ[j] * q0), k2 = f * (EIx[j] * q1 + EIy[j] * q0);
        kDyn[3 * size_t(sa)] += k0; kDyn[3 * size_t(sa) + 1] += k1; kDyn[3 * size_t(sa) + 2] += k2;
        kDyn[3 * size_t(sb)] += k0; kDyn[3 * size_t(sb) + 1] += k1; kDyn[3 * size_t(sb) + 2] += k2;
      }
      const double beta = th < 1e-3 ? 1.0 / 12 + th * th / 720 : 1 / (th * th) - (1 + std::cos(th)) / (2 * th * std::sin(th));
      const double c0 = psi[1] * m2 - psi[2] * m1, c1 = psi[2] * m0 - psi[0] * m2, c2 = psi[0] * m1 - psi[1] * m0;
      const double e0 = psi[1] * c2 - psi[2] * c1, e1 = psi[2] * c0 - psi[0] * c2, e2 = psi[0] * c1 - psi[1] * c0;
      const double j0 = m0 + 0.5 * c0 + beta * e0, j1 = m1 + 0.5 * c1 + beta * e1, j2 = m2 + 0.5 * c2 + beta * e2;
      const double tx = j0 * R[o] + j1 * R[o + 3] + j2 * R[o + 6];
      const double ty = j0 * R[o + 1] + j1 * R[o + 4] + j2 * R[o + 7];
      const double tz = j0 * R[o + 2] + j1 * R[o + 5] + j2 * R[o + 8];
      T[3 * size_t(sa)] += tx; T[3 * size_t(sa) + 1] += ty; T[3 * size_t(sa) + 2] += tz;
      T[3 * size_t(sb)] -= tx; T[3 * size_t(sb) + 1] -= ty; T[3 * size_t(sb) + 2] -= tz;
      M[3 * size_t(j)] = m0; M[3 * size_t(j) + 1] = m1; M[3 * size_t(j) + 2] = m2;
      eb += 0.5 * lb * (m0 * d0 + m1 * d1); et += 0.5 * lb * m2 * d2;
    }
    for (size_t c = 0; c < cSeg.size(); c++) {
      const int j = cSeg[c];
      const double lc = cLen[c], *B = &cB[3 * c];
      double Rc[9];
      const double th = relRotation(&cQ[4 * c], Q + 4 * size_t(j), psi);
      toFrame(&cQ[4 * c], Rc);
      const double d0 = psi[0] / lc, d1 = psi[1] / lc, d2 = psi[2] / lc;
      const double m0 = B[0] * d0, m1 = B[1] * d1, m2 = B[2] * d2;
      const double beta = th < 1e-3 ? 1.0 / 12 + th * th / 720 : 1 / (th * th) - (1 + std::cos(th)) / (2 * th * std::sin(th));
      const double c0 = psi[1] * m2 - psi[2] * m1, c1 = psi[2] * m0 - psi[0] * m2, c2 = psi[0] * m1 - psi[1] * m0;
      const double e0 = psi[1] * c2 - psi[2] * c1, e1 = psi[2] * c0 - psi[0] * c2, e2 = psi[0] * c1 - psi[1] * c0;
      const double j0 = m0 + 0.5 * c0 + beta * e0, j1 = m1 + 0.5 * c1 + beta * e1, j2 = m2 + 0.5 * c2 + beta * e2;
      T[3 * size_t(j)] -= j0 * Rc[0] + j1 * Rc[3] + j2 * Rc[6];
      T[3 * size_t(j) + 1] -= j0 * Rc[1] + j1 * Rc[4] + j2 * Rc[7];
      T[3 * size_t(j) + 2] -= j0 * Rc[2] + j1 * Rc[5] + j2 * Rc[8];
      cM[2 * c] = m0; cM[2 * c + 1] = m1;
      eb += 0.5 * lc * (m0 * d0 + m1 * d1); et += 0.5 * lc * m2 * d2;
    }
    eBend = eb; eTwist = et; eStretch = es; eShear = esh;
    energy = es + esh + eb + et;
  }
  // rod_cosserat.js:186-191
  void addStiffness(const St &st, std::vector<double> &kNode) const {
    for (int j = 0; j < st.m; j++) {
      const double k = (segEA[j] + segGA[j]) / st.l0[j];
      kNode[st.segI0[j]] += k; kNode[st.segI1[j]] += k;
    }
  }
  // rod_cosserat.js:196-209
  void addRotStiffness(const St &st, std::vector<double> &kRot) const {
    const double *X = st.X.data();
    for (int j = 0; j < st.p; j++) {
      const double lb = std::max(st.jLen[j], 1e-12), B[3] = {EIx[j], EIy[j], GJ[j]};
      for (int s : {st.jSeg0[j], st.jSeg1[j]}) for (int k = 0; k < 3; k++) kRot[3 * size_t(s) + k] += B[k] / lb;
    }
    for (size_t c = 0; c < cSeg.size(); c++)
      for (int k = 0; k < 3; k++) kRot[3 * size_t(cSeg[c]) + k] += cB[3 * c + k] / std::max(cLen[c], 1e-12);
    for (int j = 0; j < st.m; j++) {
      const int a = st.segI0[j], b = st.segI1[j];
      const double L = std::hypot(X[3 * size_t(b)] - X[3 * size_t(a)], X[3 * size_t(b) + 1] - X[3 * size_t(a) + 1], X[3 * size_t(b) + 2] - X[3 * size_t(a) + 2]);
      const double k = segGA[j] * L * L / st.l0[j];
      kRot[3 * size_t(j)] += k; kRot[3 * size_t(j) + 1] += k;
    }
  }
};

// ------------------------------------------------------------------------------------------------ PolylineContact
struct Side {
  std::vector<double> P, t, R, L, tp;
  std::vector<int> seg, a, b;
  void resize(int K) { P.assign(3 * size_t(K), 0); t.assign(3 * size_t(K), 0); R.assign(9 * size_t(K), 0); L.assign(K, 0); tp.assign(K, 0); seg.assign(K, 0); a.assign(K, 0); b.assign(K, 0); }
};

struct Contact {
  int K = 0;
  ws_params p{};
  std::vector<int> segOff, nseg;
  std::vector<double> wk, hk, w, h, mu;
  std::vector<uint8_t> locked, enabled;
  std::vector<double> Fn, Ft, state, gap, mid, Tn, Qn;
  std::vector<double> fc90, E90, Hs;                     // [2K] timber across the grain (solver_cpu.js:71-76)
  std::vector<int> ctype, faceSide;                      // W1 outputs (solver_cpu.js:87-88)
  std::vector<double> phi, theta, Anom, pressure, util;
  std::vector<double> cFace;                             // [2K] contact face width of each side (the _classify result)
  // contact extensions (solver_cpu.js:84-92): the multiplier λ (st.lam, model.js:10-75) and the penetration summed
  // since its last update; W3 seat depths, climbs and wall slopes per side, edge-on-face embedment per crossing; W2
  // reference angle, rotational slip and moment
  std::vector<double> lam, penAcc;
  int penN = 0;
  std::vector<double> dent, climb, tanpsi, dentE, theta0, rotSlip, Mrot;
  std::vector<uint8_t> nodeFixed;
  std::vector<double> dentSum;                           // [K] the seat depth buildResults reports (solver_cpu.js:906)
  double rotEnergy = 0;
  int dentAfterDefault = 1500;
  double energy = 0, ramp = 1.0;
  Side ev[2];

  // solver_cpu.js:62-96 (sections and flags from the model)
  void init(St &st, const ws_model &md) {
    K = st.K; p = md.params;
    segOff.resize(2 * size_t(K)); nseg.resize(2 * size_t(K));
    wk.assign(md.cross_wk, md.cross_wk + 2 * K); hk.assign(md.cross_hk, md.cross_hk + 2 * K);
    w.resize(K); h.resize(K);
    for (int c = 0; c < K; c++) { w[c] = 0.5 * (wk[2 * c] + wk[2 * c + 1]); h[c] = 0.5 * (hk[2 * c] + hk[2 * c + 1]); }
    for (int i = 0; i < 2 * K; i++) { int s = md.cross_strand[i]; segOff[i] = st.segOffset[s]; nseg[i] = st.segOffset[s + 1] - st.segOffset[s]; }
    locked.assign(md.cross_locked, md.cross_locked + K);
    enabled.assign(md.cross_enabled, md.cross_enabled + K);
    mu.assign(md.cross_mu, md.cross_mu + K);
    auto side = [&](const double *a, double dflt) { return a ? std::vector<double>(a, a + 2 * K) : std::vector<double>(2 * size_t(K), dflt); };
    fc90 = side(md.cross_fc90, 8.0); E90 = side(md.cross_E90, 800.0); Hs = side(md.cross_H, 30.0);
    ctype.assign(K, 0); faceSide.assign(K, -1); phi.assign(2 * size_t(K), 0); theta.assign(K, 0);
    Anom.assign(K, 0); pressure.assign(K, 0); util.assign(K, 0); cFace.assign(2 * size_t(K), 0);
    lam.assign(K, 0); penAcc.assign(K, 0); penN = 0;
    dent.assign(2 * size_t(K), 0); climb.assign(2 * size_t(K), 0); tanpsi.assign(2 * size_t(K), 1.0); dentE.assign(K, 0);
    theta0.assign(K, std::numeric_limits<double>::quiet_NaN()); rotSlip.assign(K, 0); Mrot.assign(K, 0); rotEnergy = 0;
    dentAfterDefault = md.params.warmup_iter + md.params.ramp_iter;      // solver_cpu.js:686
    Fn.assign(K, 0); Ft.assign(K, 0); state.assign(K, 0); gap.assign(K, 0); mid.assign(3 * size_t(K), 0);
    energy = 0; ramp = 1.0;
    ev[0].resize(K); ev[1].resize(K);
    initialize(st);
  }
  // solver_cpu.js:144-149
  void segmentOf(const St &st, int side, int c, int &seg, double &t) const {
    const double u = st.u[2 * size_t(c) + side];
    const int n = nseg[2 * c + side];
    const int i = int(std::min(std::max(std::floor(u), 0.0), double(std::max(n - 1, 0))));
    t = std::min(std::max(u - i, 0.0), 1.0);
    seg = segOff[2 * c + side] + i;
  }
  // solver_cpu.js:179-193
  void prepare(const St &st) {
    const double *X = st.X.data();
    const int n = st.n;
    Tn.assign(3 * size_t(n), 0.0);
    std::vector<double> eh(3 * size_t(st.m));
    for (int j = 0; j < st.m; j++) {
      const int a = st.segI0[j], b = st.segI1[j];
      const double ex = X[3 * size_t(b)] - X[3 * size_t(a)], ey = X[3 * size_t(b) + 1] - X[3 * size_t(a) + 1], ez = X[3 * size_t(b) + 2] - X[3 * size_t(a) + 2];
      const double l = std::max(std::sqrt(ex * ex + ey * ey + ez * ez), 1e-12);
      eh[3 * size_t(j)] = ex / l; eh[3 * size_t(j) + 1] = ey / l; eh[3 * size_t(j) + 2] = ez / l;
    }
    for (int j = 0; j < st.m; j++) { const size_t a = st.segI0[j]; for (int k = 0; k < 3; k++) Tn[3 * a + k] += eh[3 * size_t(j) + k]; }
    for (int j = 0; j < st.m; j++) { const size_t b = st.segI1[j]; for (int k = 0; k < 3; k++) Tn[3 * b + k] += eh[3 * size_t(j) + k]; }
    for (int i = 0; i < n; i++) {
      double *T = &Tn[3 * size_t(i)];
      const double l = std::max(std::sqrt(T[0] * T[0] + T[1] * T[1] + T[2] * T[2]), 1e-12);
      T[0] /= l; T[1] /= l; T[2] /= l;
    }
    nodeQuats(st, Qn);
  }
  // solver_cpu.js:197-228
  void eval(const St &st, int side) {
    Side &e = ev[side];
    const double *X = st.X.data();
    double Rn[9], q[4];
    for (int c = 0; c < K; c++) {
      int seg; double t;
      segmentOf(st, side, c, seg, t);
      const size_t a = st.segI0[seg], b = st.segI1[seg];
      const double dx = X[3 * b] - X[3 * a], dy = X[3 * b + 1] - X[3 * a + 1], dz = X[3 * b + 2] - X[3 * a + 2];
      const double L = std::sqrt(dx * dx + dy * dy + dz * dz);
      const double t2 = t * t, t3 = t * t * t;
      const double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + t, h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
      const double d00 = 6 * t2 - 6 * t, d10 = 3 * t2 - 4 * t + 1, d01 = -6 * t2 + 6 * t, d11 = 3 * t2 - 2 * t;
      double tg[3];
      for (int k = 0; k < 3; k++) {
        e.P[3 * size_t(c) + k] = h00 * X[3 * a + k] + (h10 * L) * Tn[3 * a + k] + h01 * X[3 * b + k] + (h11 * L) * Tn[3 * b + k];
        tg[k] = d00 * X[3 * a + k] + (d10 * L) * Tn[3 * a + k] + d01 * X[3 * b + k] + (d11 * L) * Tn[3 * b + k];
      }
      const double tl = std::max(std::sqrt(tg[0] * tg[0] + tg[1] * tg[1] + tg[2] * tg[2]), 1e-12);
      tg[0] /= tl; tg[1] /= tl; tg[2] /= tl;
      const double *Qa = &Qn[4 * a], *Qb = &Qn[4 * b];
      const double sgn = (Qa[0] * Qb[0] + Qa[1] * Qb[1] + Qa[2] * Qb[2] + Qa[3] * Qb[3]) < 0 ? -1 : 1;
      for (int k = 0; k < 4; k++) q[k] = (1 - t) * Qa[k] + t * sgn * Qb[k];
      qnormalize(q);
      toFrame(q, Rn);
      double y[3] = {Rn[3], Rn[4], Rn[5]};
      const double yt = y[0] * tg[0] + y[1] * tg[1] + y[2] * tg[2];
      y[0] -= yt * tg[0]; y[1] -= yt * tg[1]; y[2] -= yt * tg[2];
      const double yl = std::max(std::sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]), 1e-12);
      y[0] /= yl; y[1] /= yl; y[2] /= yl;
      const double x[3] = {y[1] * tg[2] - y[2] * tg[1], y[2] * tg[0] - y[0] * tg[2], y[0] * tg[1] - y[1] * tg[0]};
      double *R = &e.R[9 * size_t(c)];
      R[0] = x[0]; R[1] = x[1]; R[2] = x[2]; R[3] = y[0]; R[4] = y[1]; R[5] = y[2]; R[6] = tg[0]; R[7] = tg[1]; R[8] = tg[2];
      e.t[3 * size_t(c)] = tg[0]; e.t[3 * size_t(c) + 1] = tg[1]; e.t[3 * size_t(c) + 2] = tg[2];
      e.L[c] = L; e.seg[c] = seg; e.tp[c] = t; e.a[c] = int(a); e.b[c] = int(b);
    }
  }
  // solver_cpu.js:99-139
  void initialize(St &st, int sweeps = 3) {
    std::vector<double> St_(3 * size_t(K)), nv(3 * size_t(K));
    auto offsets = [&]() {
      prepare(st); eval(st, 0); eval(st, 1);
      const Side &A = ev[0], &B = ev[1];
      for (int c = 0; c < K; c++) {
        const double *tA = &A.t[3 * size_t(c)], *tB = &B.t[3 * size_t(c)];
        double nx = tA[1] * tB[2] - tA[2] * tB[1], ny = tA[2] * tB[0] - tA[0] * tB[2], nz = tA[0] * tB[1] - tA[1] * tB[0];
        const double nn = std::sqrt(nx * nx + ny * ny + nz * nz);
        const double *np = &st.nPrev[3 * size_t(c)];
        if (nn < 1e-6) { nx = np[0]; ny = np[1]; nz = np[2]; }
        else { const double d = std::max(nn, 1e-12); nx /= d; ny /= d; nz /= d; }
        if (nx * np[0] + ny * np[1] + nz * np[2] < 0) { nx = -nx; ny = -ny; nz = -nz; }
        const double S[3] = {B.P[3 * size_t(c)] - A.P[3 * size_t(c)], B.P[3 * size_t(c) + 1] - A.P[3 * size_t(c) + 1], B.P[3 * size_t(c) + 2] - A.P[3 * size_t(c) + 2]};
        const double g = S[0] * nx + S[1] * ny + S[2] * nz;
        St_[3 * size_t(c)] = S[0] - g * nx; St_[3 * size_t(c) + 1] = S[1] - g * ny; St_[3 * size_t(c) + 2] = S[2] - g * nz;
        nv[3 * size_t(c)] = nx; nv[3 * size_t(c) + 1] = ny; nv[3 * size_t(c) + 2] = nz;
      }
    };
    auto nrm = [&](int c) { return std::sqrt(St_[3 * size_t(c)] * St_[3 * size_t(c)] + St_[3 * size_t(c) + 1] * St_[3 * size_t(c) + 1] + St_[3 * size_t(c) + 2] * St_[3 * size_t(c) + 2]); };
    for (int it = 0; it < sweeps; it++) {
      offsets();
      const Side &A = ev[0], &B = ev[1];
      std::vector<double> uOld = st.u, before(K);
      for (int c = 0; c < K; c++) {
        const double *tA = &A.t[3 * size_t(c)], *tB = &B.t[3 * size_t(c)], *S = &St_[3 * size_t(c)];
        const double taa = tA[0] * tA[0] + tA[1] * tA[1] + tA[2] * tA[2], tbb = tB[0] * tB[0] + tB[1] * tB[1] + tB[2] * tB[2], tab = tA[0] * tB[0] + tA[1] * tB[1] + tA[2] * tB[2];
        const double sa = S[0] * tA[0] + S[1] * tA[1] + S[2] * tA[2], sb = S[0] * tB[0] + S[1] * tB[1] + S[2] * tB[2];
        const double det = taa * tbb - tab * tab;
        const bool ok = det > 1e-3 && enabled[c];
        const double ca = ok ? (sa * tbb - sb * tab) / det : 0, cb = ok ? (sb * taa - sa * tab) / det : 0;
        before[c] = nrm(c);
        st.u[2 * size_t(c)] = std::min(std::max(st.u[2 * size_t(c)] + ca / std::max(A.L[c], 1e-12), 0.0), double(nseg[2 * c]));
        st.u[2 * size_t(c) + 1] = std::min(std::max(st.u[2 * size_t(c) + 1] - cb / std::max(B.L[c], 1e-12), 0.0), double(nseg[2 * c + 1]));
      }
      offsets();
      for (int c = 0; c < K; c++) if (nrm(c) >= before[c]) { st.u[2 * size_t(c)] = uOld[2 * size_t(c)]; st.u[2 * size_t(c) + 1] = uOld[2 * size_t(c) + 1]; }
    }
    offsets();
    st.nPrev = nv;
  }
  // solver_cpu.js:151-167
  void addStiffness(const St &st, std::vector<double> &kNode, std::vector<double> &kSeg) const {
    const double k = p.strength + p.stick_strength;
    for (int side = 0; side < 2; side++) {
      for (int c = 0; c < K; c++) { int seg; double t; segmentOf(st, side, c, seg, t); kNode[st.segI0[seg]] += k; }
      for (int c = 0; c < K; c++) { int seg; double t; segmentOf(st, side, c, seg, t); kNode[st.segI1[seg]] += k; }
    }
    if (p.rot_friction) {
      for (int side = 0; side < 2; side++)
        for (int pass = 0; pass < 2; pass++)
          for (int c = 0; c < K; c++) {
            int seg; double t;
            segmentOf(st, side, c, seg, t);
            const double kr = p.stick_strength * (0.38 * 0.38) * wk[2 * size_t(c)] * wk[2 * size_t(c) + 1] / 0.5;
            const double l = std::max(st.l0[seg], 1e-12);
            kNode[pass ? st.segI1[seg] : st.segI0[seg]] += kr / (l * l);
          }
    }
    addTwistStiffness(st, kSeg);
  }
  // fixed-node mask from the anchors (setFixed, solver_cpu.js:481)
  void setFixed(const std::vector<uint8_t> &nodeFree) {
    nodeFixed.assign(nodeFree.size() / 3, 0);
    for (size_t i = 0; i < nodeFixed.size(); i++) nodeFixed[i] = (nodeFree[3 * i] || nodeFree[3 * i + 1] || nodeFree[3 * i + 2]) ? 0 : 1;
  }
  // free weight of the contact point on `side` (freeWeight, solver_cpu.js:483-487)
  double freeWeight(const St &st, int side, int c) const {
    int seg; double t;
    segmentOf(st, side, c, seg, t);
    const int a = st.segI0[seg], b = st.segI1[seg];
    return (nodeFixed[a] ? 0.0 : (1 - t) * (1 - t)) + (nodeFixed[b] ? 0.0 : t * t);
  }
  // crushing capacity of the face overlap (capForce, solver_cpu.js:489)
  double capForce(int c) const {
    return std::min(fc90[2 * size_t(c)], fc90[2 * size_t(c) + 1]) * wk[2 * size_t(c)] * wk[2 * size_t(c) + 1] / std::max(std::sin(theta[c]), 1e-6);
  }
  // safeguarded Uzawa value (alValue, solver_cpu.js:492-497)
  static double alValue(double l, double penMean, double kn, bool lockedC, bool enabledC, bool pinned, double cap) {
    if (!enabledC || pinned) return 0;
    double v = l + kn * penMean;
    if (!lockedC) v = std::max(v, 0.0);
    return std::min(std::max(v, -cap), cap);
  }
  // Uzawa step on the window-mean penetration (updateMultipliers, solver_cpu.js:499-506)
  void updateMultipliers(const St &st) {
    const double kn = ramp * p.strength, nw = std::max(penN, 1);
    for (int c = 0; c < K; c++) {
      const bool pinned = freeWeight(st, 0, c) < AL_FREE_MIN || freeWeight(st, 1, c) < AL_FREE_MIN;
      lam[c] = alValue(lam[c], penAcc[c] / nw, kn, locked[c], enabled[c], pinned, capForce(c));
    }
    std::fill(penAcc.begin(), penAcc.end(), 0.0);
    penN = 0;
  }
  // W3: slope of the wall a sliding side climbs (_walls, solver_cpu.js:284-292)
  static double walls(int sideCut, const double *R, const double *n, const double *m) {
    const double sg = sideCut == 0 ? 1.0 : -1.0;
    const double *X = R, *Y = R + 3;
    const double nx = (n[0] * X[0] + n[1] * X[1] + n[2] * X[2]) * sg, ny = (n[0] * Y[0] + n[1] * Y[1] + n[2] * Y[2]) * sg;
    double fx[3], fy[3];
    for (int k = 0; k < 3; k++) { fx[k] = jsSign(nx) * X[k]; fy[k] = jsSign(ny) * Y[k]; }
    const double *f = (fx[0] * m[0] + fx[1] * m[1] + fx[2] * m[2]) > 0 ? fx : fy;
    const double cosPsi = std::min(std::max(std::fabs(f[0] * n[0] + f[1] * n[1] + f[2] * n[2]), 1e-6), 1.0);
    return std::tan(std::acos(cosPsi));
  }
  // n × t, normalised (the wall direction across the cutting side)
  static void wallAxis(const double *n, const double *tCut, double *m) {
    m[0] = n[1] * tCut[2] - n[2] * tCut[1]; m[1] = n[2] * tCut[0] - n[0] * tCut[2]; m[2] = n[0] * tCut[1] - n[1] * tCut[0];
    const double ml = std::max(std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]), 1e-12);
    m[0] /= ml; m[1] /= ml; m[2] /= ml;
  }
  // W3: friction coefficient against the slide direction with the seats' walls (_seatFriction, solver_cpu.js:294-313)
  double seatFriction(int c, const double *St_, const double *n, const double *tA, const double *tB) {
    const double mu0 = mu[c];
    double muD = mu0;
    const double norm = std::sqrt(St_[0] * St_[0] + St_[1] * St_[1] + St_[2] * St_[2]);
    const double dn = std::max(norm, 1e-12), dhat[3] = {St_[0] / dn, St_[1] / dn, St_[2] / dn};
    const bool has = norm > 1e-12;
    for (int j = 0; j < 2; j++) {
      if (!(dent[2 * size_t(c) + j] > 0 && has)) continue;
      const double *tCut = j == 0 ? tB : tA;
      const double *Rcut = j == 0 ? &ev[1].R[9 * size_t(c)] : &ev[0].R[9 * size_t(c)];
      double m[3];
      wallAxis(n, tCut, m);
      const double sgn = j == 0 ? 1.0 : -1.0;
      const double dj = (dhat[0] * m[0] + dhat[1] * m[1] + dhat[2] * m[2]) * sgn;
      const double wallDir[3] = {jsSign(dj) * m[0] * sgn, jsSign(dj) * m[1] * sgn, jsSign(dj) * m[2] * sgn};
      const double tp = walls(1 - j, Rcut, n, wallDir);
      tanpsi[2 * size_t(c) + j] = tp;
      const double add = std::fabs(dj) * (mu0 * tp < 1.0 ? (mu0 + tp) / std::max(1.0 - mu0 * tp, 1e-6) - mu0 : 9.0 * mu0);
      muD += std::min(add, 9.0 * mu0);
    }
    return muD;
  }
  // W3: climb out of the seats, seat growth under an edge (_seatUpdate, solver_cpu.js:315-344)
  void seatUpdate(const St &st, int c, bool slip, double da, double db, const double *tA, const double *tB, const double *n,
                  double fn, bool active) {
    const double inc[3] = {da * tA[0] - db * tB[0], da * tA[1] - db * tB[1], da * tA[2] - db * tB[2]};
    for (int j = 0; j < 2; j++) {
      double m[3];
      wallAxis(n, j == 0 ? tB : tA, m);
      const double step = (inc[0] * m[0] + inc[1] * m[1] + inc[2] * m[2]) * (j == 0 ? 1.0 : -1.0);
      const size_t i = 2 * size_t(c) + j;
      const bool has = dent[i] > 0;
      if (has && slip) climb[i] += step;
      if (has && std::fabs(climb[i]) >= dent[i] / std::max(tanpsi[i], 1e-6)) { dent[i] = 0; climb[i] = 0; }
    }
    const int after = p.dent_after_iter >= 0 ? p.dent_after_iter : dentAfterDefault;
    if (st.iteration < after) return;
    const double sinp0 = std::sin(phi[2 * size_t(c)]) * std::cos(phi[2 * size_t(c)]);
    const double sinp1 = std::sin(phi[2 * size_t(c) + 1]) * std::cos(phi[2 * size_t(c) + 1]);
    const double sinT = std::sin(theta[c]);
    if (ctype[c] == 2 && active && !locked[c]) {
      const double fc = std::min(fc90[2 * size_t(c)], fc90[2 * size_t(c) + 1]);
      const double dEst = std::sqrt(std::fabs(fn) / std::max(fc, 1e-12) * sinT * sinp0 * sinp1);
      for (int j = 0; j < 2; j++) { const double cur = dent[2 * size_t(c) + j]; dent[2 * size_t(c) + j] = std::max(cur, std::min(cur + p.dent_rate * dEst, dEst)); }
    }
    if (ctype[c] == 1 && active && !locked[c]) {
      const int fs = faceSide[c], es = 1 - fs;
      const double ell = cFace[2 * size_t(c) + fs] / std::max(sinT, 1e-6);
      const double dE = std::fabs(fn) / std::max(fc90[2 * size_t(c) + es] * ell, 1e-12) * (es == 0 ? sinp0 : sinp1);
      dentE[c] = std::max(dentE[c], dE);
    }
  }
  // W2: rotational friction about the contact normal (_rotationalFriction, solver_cpu.js:347-379)
  void rotationalFriction(double *T, const std::vector<double> &n, const std::vector<uint8_t> &active, double kt) {
    const Side &A = ev[0], &B = ev[1];
    std::vector<double> e(K);
    for (int c = 0; c < K; c++) {
      const double *tA = &A.t[3 * size_t(c)], *tB = &B.t[3 * size_t(c)], *nc = &n[3 * size_t(c)];
      const double cr[3] = {tA[1] * tB[2] - tA[2] * tB[1], tA[2] * tB[0] - tA[0] * tB[2], tA[0] * tB[1] - tA[1] * tB[0]};
      const double th = std::atan2(cr[0] * nc[0] + cr[1] * nc[1] + cr[2] * nc[2], tA[0] * tB[0] + tA[1] * tB[1] + tA[2] * tB[2]);
      if (std::isnan(theta0[c]) && active[c]) theta0[c] = th;
      const bool ok = active[c] && !std::isnan(theta0[c]);
      const double sinT = std::max(std::sin(theta[c]), 1e-6);
      double req = 0.38 * std::sqrt(wk[2 * size_t(c)] * wk[2 * size_t(c) + 1] / sinT);
      if (ctype[c] == 1) { const double cw = faceSide[c] == 0 ? wk[2 * size_t(c)] : wk[2 * size_t(c) + 1]; req = 0.25 * cw / sinT; }
      else if (ctype[c] == 2) req = 0.38 * std::sqrt(std::max(Anom[c], 1e-12));
      const double kr = kt * req * req;
      double dth = ok ? th - theta0[c] : 0.0;
      dth = std::fmod(std::fmod(dth + PI, 2 * PI) + 2 * PI, 2 * PI) - PI;
      double Mc = kr * dth;
      const double Mlim = locked[c] ? INF : p.rot_factor * mu[c] * std::fabs(Fn[c]) * req;
      if (ok && std::fabs(Mc) > Mlim) {
        const double rate = std::min(std::max(p.slip_rate, 1e-3), 1.0);
        double adv = rate * (1.0 - Mlim / std::max(std::fabs(Mc), 1e-12)) * dth;
        adv = std::min(std::max(adv, -0.05), 0.05);
        theta0[c] += adv; rotSlip[c] += std::fabs(adv); dth -= adv;
        Mc = kr * dth;
      }
      Mrot[c] = ok ? Mc : 0.0;
      e[c] = kr * dth * dth;
    }
    for (int c = 0; c < K; c++) { const size_t s = A.seg[c]; for (int k = 0; k < 3; k++) T[3 * s + k] += Mrot[c] * n[3 * size_t(c) + k]; }
    for (int c = 0; c < K; c++) { const size_t s = B.seg[c]; for (int k = 0; k < 3; k++) T[3 * s + k] -= Mrot[c] * n[3 * size_t(c) + k]; }
    rotEnergy = 0.5 * pairwiseSum(e);
  }
  // solver_cpu.js:170-176
  void addTwistStiffness(const St &st, std::vector<double> &kSeg) const {
    const double kn = ramp * p.strength, kt = ramp * p.stick_strength, tf = std::max(p.torsion_factor, 1e-3);
    for (int side = 0; side < 2; side++)
      for (int c = 0; c < K; c++) {
        const double kth = tf * ((Fn[c] + kn * 0.25 * h[c]) * (0.5 * w[c]) / SUPPORT_SMOOTH + kt * (0.5 * h[c]) * (0.5 * h[c]));
        int seg; double t;
        segmentOf(st, side, c, seg, t);
        kSeg[seg] += kth;
      }
  }
  // solver_cpu.js:274-282
  double support(const double *R, const double *n, int c, double sign, int side, double *r) const {
    const double *Xa = R, *Ya = R + 3;
    const double wv = wk[2 * c + side], hv = hk[2 * c + side];
    const double nx = (n[0] * Xa[0] + n[1] * Xa[1] + n[2] * Xa[2]) * sign, ny = (n[0] * Ya[0] + n[1] * Ya[1] + n[2] * Ya[2]) * sign;
    const double hh = 0.5 * wv * std::fabs(nx) + 0.5 * hv * std::fabs(ny);
    const double ax = 0.5 * wv * std::tanh(nx / SUPPORT_SMOOTH), ay = 0.5 * hv * std::tanh(ny / SUPPORT_SMOOTH);
    for (int k = 0; k < 3; k++) r[k] = ax * Xa[k] + ay * Ya[k];
    return hh;
  }
  // W1: contact type per crossing from the roll of each section against the contact plane n (solver_cpu.js:231-271)
  void classify(const std::vector<double> &n) {
    const Side &A = ev[0], &B = ev[1];
    std::vector<double> Z0(2 * size_t(K));
    std::vector<uint8_t> edge(2 * size_t(K));
    for (int c = 0; c < K; c++) {
      for (int side = 0; side < 2; side++) {
        const double *R = side == 0 ? &A.R[9 * size_t(c)] : &B.R[9 * size_t(c)];
        const double sg = side == 0 ? 1.0 : -1.0;
        const size_t i = 2 * size_t(c) + side;
        const double *nc = &n[3 * size_t(c)];
        const double nx = (nc[0] * R[0] + nc[1] * R[1] + nc[2] * R[2]) * sg;
        const double ny = (nc[0] * R[3] + nc[1] * R[4] + nc[2] * R[5]) * sg;
        const double sx = std::fabs(std::tanh(nx / SUPPORT_SMOOTH)), sy = std::fabs(std::tanh(ny / SUPPORT_SMOOTH));
        edge[i] = sx * sy > p.edge_threshold ? 1 : 0;
        const bool yFace = std::fabs(ny) >= std::fabs(nx);
        cFace[i] = yFace ? wk[i] : hk[i];
        Z0[i] = yFace ? hk[i] : wk[i];
        phi[i] = std::atan(std::min(std::fabs(nx), std::fabs(ny)) / std::max(std::max(std::fabs(nx), std::fabs(ny)), 1e-12));
      }
      const double *tA = &A.t[3 * size_t(c)], *tB = &B.t[3 * size_t(c)];
      const double cr[3] = {tA[1] * tB[2] - tA[2] * tB[1], tA[2] * tB[0] - tA[0] * tB[2], tA[0] * tB[1] - tA[1] * tB[0]};
      const double sinT = std::min(std::max(std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]), 1e-6), 1.0);
      theta[c] = std::asin(sinT);
      const int nEdge = edge[2 * size_t(c)] + edge[2 * size_t(c) + 1];
      ctype[c] = nEdge;
      faceSide[c] = nEdge == 1 ? (edge[2 * size_t(c) + 1] ? 0 : 1) : -1;
      const double fn = std::fabs(Fn[c]);
      double Aa = cFace[2 * size_t(c)] * cFace[2 * size_t(c) + 1] / sinT, pres = fn / std::max(Aa, 1e-12);
      double ut = pres / std::max(std::min(Hs[2 * size_t(c)], Hs[2 * size_t(c) + 1]), 1e-12);
      if (nEdge == 1) {
        const int fs = faceSide[c], es = 1 - fs;
        const double ell = cFace[2 * size_t(c) + fs] / sinT, kap = E90[2 * size_t(c) + fs] / std::max(Z0[2 * size_t(c) + fs], 1e-12);
        const double phiE = std::max(phi[2 * size_t(c) + es], 1e-4);
        const double b = std::sqrt(2.0 * fn / std::max(ell * kap * phiE, 1e-12));
        const bool full = b >= cFace[2 * size_t(c) + es];
        const double Afe = full ? cFace[2 * size_t(c)] * cFace[2 * size_t(c) + 1] / sinT : b * ell;
        const double pfe = full ? fn / std::max(Afe, 1e-12) : kap * phiE * b;
        Aa = Afe; pres = pfe; ut = pfe / std::max(fc90[2 * size_t(c) + es], 1e-12);
      } else if (nEdge == 2) {
        const double fc = std::min(fc90[2 * size_t(c)], fc90[2 * size_t(c) + 1]);
        Aa = fn / std::max(fc, 1e-12); pres = fc * (fn > 0 ? 1 : 0); ut = fn > 0 ? 1.0 : 0.0;
      }
      Anom[c] = Aa; pressure[c] = pres; util[c] = ut;
    }
  }
  // solver_cpu.js:381-478
  void apply(St &st, double *F, double *T) {
    if (!K) return;
    prepare(st); eval(st, 0); eval(st, 1);
    const Side &A = ev[0], &B = ev[1];
    const double kn = ramp * p.strength, kt = ramp * p.stick_strength;
    const bool seat = p.seat_law != 0, aug = p.augmented != 0;
    const bool accum = st.iteration >= std::max(p.ramp_iter, 0);       // the multiplier's penetration window: after the ramp
    std::vector<double> nA(3 * size_t(K)), FA(3 * size_t(K)), FB(3 * size_t(K)), rAx(3 * size_t(K)), rBx(3 * size_t(K)), ePen(K), eTan(K);
    std::vector<uint8_t> slipA(K), activeA(K);
    std::vector<double> daA(K), dbA(K);
    double rA[3], rB[3];
    for (int c = 0; c < K; c++) {
      const double *tA = &A.t[3 * size_t(c)], *tB = &B.t[3 * size_t(c)];
      double *np = &st.nPrev[3 * size_t(c)];
      double nx = tA[1] * tB[2] - tA[2] * tB[1], ny = tA[2] * tB[0] - tA[0] * tB[2], nz = tA[0] * tB[1] - tA[1] * tB[0];
      const double nn = std::sqrt(nx * nx + ny * ny + nz * nz);
      if (nn < 1e-6) { nx = np[0]; ny = np[1]; nz = np[2]; }
      else { const double d = std::max(nn, 1e-12); nx /= d; ny /= d; nz /= d; }
      if (nx * np[0] + ny * np[1] + nz * np[2] < 0) { nx = -nx; ny = -ny; nz = -nz; }
      np[0] = nx; np[1] = ny; np[2] = nz;
      nA[3 * size_t(c)] = nx; nA[3 * size_t(c) + 1] = ny; nA[3 * size_t(c) + 2] = nz;
      const double nv[3] = {nx, ny, nz};
      const double S[3] = {B.P[3 * size_t(c)] - A.P[3 * size_t(c)], B.P[3 * size_t(c) + 1] - A.P[3 * size_t(c) + 1], B.P[3 * size_t(c) + 2] - A.P[3 * size_t(c) + 2]};
      for (int k = 0; k < 3; k++) mid[3 * size_t(c) + k] = 0.5 * (A.P[3 * size_t(c) + k] + B.P[3 * size_t(c) + k]);
      const double g = S[0] * nx + S[1] * ny + S[2] * nz;
      const double hA = support(&A.R[9 * size_t(c)], nv, c, +1.0, 0, rA);
      const double hB = support(&B.R[9 * size_t(c)], nv, c, -1.0, 1, rB);
      double D = hA + hB;
      if (seat && p.seat_gap) D -= dent[2 * size_t(c)] + dent[2 * size_t(c) + 1] + dentE[c];
      const double pen = D - g;
      if (accum) penAcc[c] += pen;
      bool active;
      double fn;
      if (aug) {
        const double trial = lam[c] + kn * pen;
        active = (trial > 0 || locked[c]) && enabled[c];
        fn = active ? (locked[c] ? trial : std::max(trial, 0.0)) : 0.0;
      } else {
        active = (pen > 0 || locked[c]) && enabled[c];
        fn = active ? kn * pen : 0.0;
      }
      activeA[c] = active ? 1 : 0;
      const double Stv[3] = {S[0] - g * nx, S[1] - g * ny, S[2] - g * nz};
      const double taa = tA[0] * tA[0] + tA[1] * tA[1] + tA[2] * tA[2], tbb = tB[0] * tB[0] + tB[1] * tB[1] + tB[2] * tB[2], tab = tA[0] * tB[0] + tA[1] * tB[1] + tA[2] * tB[2];
      const double sa = Stv[0] * tA[0] + Stv[1] * tA[1] + Stv[2] * tA[2], sb = Stv[0] * tB[0] + Stv[1] * tB[1] + Stv[2] * tB[2];
      const double det = taa * tbb - tab * tab;
      const bool ok = det > 1e-8;
      const double ca = ok ? (sa * tbb - sb * tab) / det : 0.0, cb = ok ? (sb * taa - sa * tab) / det : 0.0;
      const double Ftv = std::sqrt((kt * Stv[0]) * (kt * Stv[0]) + (kt * Stv[1]) * (kt * Stv[1]) + (kt * Stv[2]) * (kt * Stv[2]));
      const double muDir = seat ? seatFriction(c, Stv, nv, tA, tB) : mu[c];
      const double limit = locked[c] ? INF : muDir * std::fabs(fn);
      const bool inContact = active && ok;
      const bool slip = inContact && Ftv > limit;
      const bool free_ = !active && ok && enabled[c];
      double scale = 0;
      if (slip) scale = std::min(std::max(p.slip_rate, 1e-3), 1.0) * (1.0 - limit / std::max(Ftv, 1e-12));
      if (free_) scale = 1.0;
      const double eps = std::max(p.epsilon, 1e-9);
      const double da = std::min(std::max(ca * scale, -eps), eps), db = std::min(std::max(cb * scale, -eps), eps);
      const bool moved = slip || free_;
      if (moved) { st.u[2 * size_t(c)] += da / std::max(A.L[c], 1e-12); st.u[2 * size_t(c) + 1] -= db / std::max(B.L[c], 1e-12); }
      st.u[2 * size_t(c)] = std::min(std::max(st.u[2 * size_t(c)], 0.0), double(nseg[2 * c]));
      st.u[2 * size_t(c) + 1] = std::min(std::max(st.u[2 * size_t(c) + 1], 0.0), double(nseg[2 * c + 1]));
      if (slip) {
        const double sx = da * tA[0] + db * tB[0], sy = da * tA[1] + db * tB[1], sz = da * tA[2] + db * tB[2];
        st.slip[c] += std::sqrt(sx * sx + sy * sy + sz * sz);
      }
      st.stuck[c] = moved ? 0 : 1;
      double Se[3] = {0, 0, 0};
      if (active) for (int k = 0; k < 3; k++) Se[k] = Stv[k] - da * tA[k] - db * tB[k];
      const double fT[3] = {kt * Se[0], kt * Se[1], kt * Se[2]};
      for (int k = 0; k < 3; k++) { FA[3 * size_t(c) + k] = -fn * nv[k] + fT[k]; FB[3 * size_t(c) + k] = fn * nv[k] - fT[k]; }
      Fn[c] = fn;
      Ft[c] = std::sqrt(fT[0] * fT[0] + fT[1] * fT[1] + fT[2] * fT[2]);
      state[c] = slip ? 1 : 0; gap[c] = g;
      for (int k = 0; k < 3; k++) { rAx[3 * size_t(c) + k] = rA[k]; rBx[3 * size_t(c) + k] = rB[k]; }
      slipA[c] = slip ? 1 : 0; daA[c] = da; dbA[c] = db;
      ePen[c] = active ? (aug ? fn * fn / std::max(kn, 1e-300) : kn * pen * pen) : 0.0;
      eTan[c] = Se[0] * Se[0] + Se[1] * Se[1] + Se[2] * Se[2];
    }
    if (accum) penN += 1;
    classify(nA);                                        // solver_cpu.js:460
    if (seat)
      for (int c = 0; c < K; c++)
        seatUpdate(st, c, slipA[c], daA[c], dbA[c], &A.t[3 * size_t(c)], &B.t[3 * size_t(c)], &nA[3 * size_t(c)], Fn[c], activeA[c]);
    for (int c = 0; c < K; c++) { const size_t i = A.a[c]; const double wt = 1 - A.tp[c]; for (int k = 0; k < 3; k++) F[3 * i + k] += wt * FA[3 * size_t(c) + k]; }
    for (int c = 0; c < K; c++) { const size_t i = A.b[c]; const double wt = A.tp[c]; for (int k = 0; k < 3; k++) F[3 * i + k] += wt * FA[3 * size_t(c) + k]; }
    for (int c = 0; c < K; c++) { const size_t i = B.a[c]; const double wt = 1 - B.tp[c]; for (int k = 0; k < 3; k++) F[3 * i + k] += wt * FB[3 * size_t(c) + k]; }
    for (int c = 0; c < K; c++) { const size_t i = B.b[c]; const double wt = B.tp[c]; for (int k = 0; k < 3; k++) F[3 * i + k] += wt * FB[3 * size_t(c) + k]; }
    const double tf = p.torsion_factor;
    for (int c = 0; c < K; c++) {
      const size_t s = A.seg[c];
      const double *r = &rAx[3 * size_t(c)], *f = &FA[3 * size_t(c)];
      T[3 * s] += tf * (r[1] * f[2] - r[2] * f[1]); T[3 * s + 1] += tf * (r[2] * f[0] - r[0] * f[2]); T[3 * s + 2] += tf * (r[0] * f[1] - r[1] * f[0]);
    }
    for (int c = 0; c < K; c++) {
      const size_t s = B.seg[c];
      const double *r = &rBx[3 * size_t(c)], *f = &FB[3 * size_t(c)];
      T[3 * s] += tf * (r[1] * f[2] - r[2] * f[1]); T[3 * s + 1] += tf * (r[2] * f[0] - r[0] * f[2]); T[3 * s + 2] += tf * (r[0] * f[1] - r[1] * f[0]);
    }
    if (p.rot_friction) rotationalFriction(T, nA, activeA, kt);
    energy = 0.5 * pairwiseSum(ePen) + 0.5 * kt * pairwiseSum(eTan) + (p.rot_friction ? rotEnergy : 0.0);
  }
};

// ------------------------------------------------------------------------------------------------ CpuSolver
struct Solver {
  St st;
  ws_params sp{};
  Rod rod;
  bool hasContact = false;
  Contact contact;
  std::vector<double> loadConst, total, localF;
  std::vector<int> localNode;
  std::vector<uint8_t> nodeFree, fixedAny;
  std::vector<int> fixedNodes;
  std::vector<Clamp> rotClamps;
  std::vector<double> reactions, mass, kRotStatic, inertia3, F, T, tm, kTw;
  double lRef = 1.0, kePrev = 0.0, ke = 0.0, fref = 0.0, resF = 0.0, resT = 0.0, resRigid = 0.0;
  bool converged = false;
  int rollbacks = 0;
  // prescribed support motion (an extension of the reference's anchors): fixed translations move linearly from
  // ancStart to ancStart + ancDelta over params.disp_ramp_iter iterations counted from dispIt0, or from the end of
  // the warm-up when that is later
  std::vector<double> ancStart, ancDelta;
  std::vector<uint8_t> hasTarget;
  int dispIt0 = 0;

  void setTargets(const ws_model &md) {
    const int n = st.n;
    ancStart.assign(3 * size_t(n), 0.0); ancDelta.assign(3 * size_t(n), 0.0); hasTarget.assign(n, 0);
    dispIt0 = st.iteration;
    if (!md.anchor_target) return;
    for (int a = 0; a < md.n_anchors; a++) {
      const size_t nid = md.anchor_node[a];
      if (!(md.anchor_mask[a] & 7)) continue;
      hasTarget[nid] = 1;
      for (int c = 0; c < 3; c++) {
        ancStart[3 * nid + c] = st.X[3 * nid + c];
        if (md.anchor_mask[a] & (1 << c)) ancDelta[3 * nid + c] = md.anchor_target[3 * size_t(a) + c] - st.X[3 * nid + c];
      }
    }
  }

  void load(const ws_model &md) {
    st.n = md.n; st.m = md.m; st.p = md.p; st.K = md.K; st.S = md.n_strands;
    st.X.assign(md.X, md.X + 3 * size_t(md.n)); st.X0.assign(md.X0, md.X0 + 3 * size_t(md.n));
    st.V.assign(3 * size_t(md.n), 0.0);
    st.Q.assign(md.Q, md.Q + 4 * size_t(md.m)); st.Q0 = st.Q; st.Wr.assign(3 * size_t(md.m), 0.0);
    st.l0.assign(md.l0, md.l0 + md.m);
    st.segI0.assign(md.seg_i0, md.seg_i0 + md.m); st.segI1.assign(md.seg_i1, md.seg_i1 + md.m);
    st.segOffset.assign(md.seg_offset, md.seg_offset + md.n_strands + 1);
    st.jSeg0.assign(md.joint_seg0, md.joint_seg0 + md.p); st.jSeg1.assign(md.joint_seg1, md.joint_seg1 + md.p);
    st.jLen.assign(md.joint_len, md.joint_len + md.p);
    if (md.omega0) st.Omega0.assign(md.omega0, md.omega0 + 3 * size_t(md.p)); else st.Omega0.assign(3 * size_t(md.p), 0.0);
    st.u.assign(md.cross_u, md.cross_u + 2 * size_t(md.K)); st.nPrev.assign(md.cross_nprev, md.cross_nprev + 3 * size_t(md.K));
    st.slip.assign(md.K, 0.0); st.stuck.assign(md.K, 1);
    st.iteration = 0; st.residual = INF;
    sp = md.params;
    proto = ws_protocol{};
    if (md.protocol && md.protocol->mode) proto = *md.protocol;
    buildGoals(md, false);
    setTargets(md);
    startProtocol();
  }

  // ---------------------------------------------------------------------------------------------- the ground
  // Floor (solver_cpu.js:509-634), with the rigid-body freedoms of a model that only the ground holds
  bool hasFloor = false;
  double floorFnMax = 0, floorEnergy = 0, floorRamp = 1.0;
  std::vector<double> flW, flH, flAx, flAy, flF;
  std::vector<uint8_t> flState;
  // rigid-body freedoms (Floor constructor, solver_cpu.js:546-553): the reference point c (the centroid of the nodes,
  // followed at every evaluation), the model radius about it at construction, the rigid velocities, and the sums of the
  // last evaluation
  double rbC[3] = {0, 0, 0}, rbR = 1e-9, rbV[3] = {0, 0, 0}, rbW[3] = {0, 0, 0}, rbQt[3] = {0, 0, 0}, rbQr[3] = {0, 0, 0};
  double rbD2[3] = {0, 0, 0}, rbVmax = 0, rbWmax = 0;
  int rbNc = 0;
  // the Floor constructor / bind (solver_cpu.js:531-562): sections from the model; stick points, the reference point and
  // the model radius at the nodes when new
  void floorBind(const ws_model &md) {
    const int n = st.n;
    if (!md.params.floor) { hasFloor = false; return; }
    if (!md.node_w || !md.node_h) throw std::invalid_argument("oracle: a ground needs the node sections");
    flW.assign(md.node_w, md.node_w + n); flH.assign(md.node_h, md.node_h + n);
    if (!hasFloor || flAx.size() != size_t(n)) {
      flAx.resize(n); flAy.resize(n);
      for (int i = 0; i < n; i++) { flAx[i] = st.X[3 * size_t(i)]; flAy[i] = st.X[3 * size_t(i) + 1]; }
      flF.assign(3 * size_t(n), 0.0); flState.assign(n, 0); floorFnMax = floorEnergy = 0;
      double c[3] = {0, 0, 0};
      for (int i = 0; i < n; i++) for (int k = 0; k < 3; k++) c[k] += st.X[3 * size_t(i) + k] / std::max(n, 1);
      double R2 = 0;
      for (int i = 0; i < n; i++) {
        const double *x = &st.X[3 * size_t(i)];
        R2 = std::max(R2, (x[0] - c[0]) * (x[0] - c[0]) + (x[1] - c[1]) * (x[1] - c[1]) + (x[2] - c[2]) * (x[2] - c[2]));
      }
      for (int k = 0; k < 3; k++) { rbC[k] = c[k]; rbV[k] = rbW[k] = rbQt[k] = rbQr[k] = rbD2[k] = 0; }
      rbR = std::max(std::sqrt(R2), 1e-9);
      rbNc = 0;
    }
    double hmin = INF;
    for (int i = 0; i < n; i++) hmin = std::min(hmin, std::min(flH[i], flW[i]));
    rbVmax = RB_VMAX * (std::isfinite(hmin) && hmin > 0 ? hmin : 1.0);
    rbWmax = rbVmax / rbR;
    hasFloor = true;
  }
  // Floor.rigidMasses (solver_cpu.js:564-572): fictitious masses of the rigid translations and rotations
  void rigidMasses(double ms, double out[6]) const {
    const double kn = floorRamp * sp.strength, kt = floorRamp * sp.stick_strength, f = ms * RB_MASS;
    const double nc = std::max(rbNc, 1), rmin = (RB_LEVER * rbR) * (RB_LEVER * rbR) * kn;
    out[0] = std::max(f * nc * kt, 1e-30); out[1] = out[0]; out[2] = std::max(f * nc * kn, 1e-30);
    out[3] = std::max(f * std::max(kn * rbD2[1] + kt * rbD2[2], rmin), 1e-30);
    out[4] = std::max(f * std::max(kn * rbD2[0] + kt * rbD2[2], rmin), 1e-30);
    out[5] = std::max(f * std::max(kt * (rbD2[0] + rbD2[1]), rmin), 1e-30);
  }
  // Floor.rigidResidual (solver_cpu.js:574)
  double rigidResidual(double fr) const {
    return std::max(std::hypot(rbQt[0], rbQt[1], rbQt[2]) / fr, std::hypot(rbQr[0], rbQr[1], rbQr[2]) / (fr * rbR));
  }
  // Floor.apply with the rigid-body sums of the external forces `loads` + the ground (solver_cpu.js:583-631)
  void floorApply(double ramp, const std::vector<double> &loads) {
    const int n = st.n;
    const double z0 = sp.floor_z, mu = std::max(sp.floor_mu, 0.0), kn = ramp * sp.strength, kt = ramp * sp.stick_strength;
    floorRamp = ramp;
    double q0 = 0, q1 = 0, q2 = 0, q3 = 0, q4 = 0, q5 = 0, dxx = 0, dyy = 0, dzz = 0;
    int nc = 0;
    double *c = rbC;
    if (n) {
      double cx = 0, cy = 0, cz = 0;
      for (int i = 0; i < n; i++) { cx += st.X[3 * size_t(i)]; cy += st.X[3 * size_t(i) + 1]; cz += st.X[3 * size_t(i) + 2]; }
      c[0] = cx / n; c[1] = cy / n; c[2] = cz / n;
    }
    std::vector<double> qn;
    nodeQuats(st, qn);
    double e = 0, fmax = 0, R[9];
    for (int i = 0; i < n; i++) {
      toFrame(&qn[4 * size_t(i)], R);
      const double *x = &st.X[3 * size_t(i)];
      const double pen = (z0 - x[2]) + (0.5 * flW[i] * std::fabs(R[2]) + 0.5 * flH[i] * std::fabs(R[5]));
      double *f = &flF[3 * size_t(i)];
      if (pen > 0) {
        const double fn = kn * pen;
        const double sx = x[0] - flAx[i], sy = x[1] - flAy[i];
        const double Ftv = kt * std::sqrt(sx * sx + sy * sy), limit = mu * fn;
        const double scale = Ftv > limit ? 1.0 - limit / std::max(Ftv, 1e-12) : 0.0;
        const double dax = sx * scale, day = sy * scale;
        if (scale > 0) { flAx[i] += dax; flAy[i] += day; }
        const double ex = sx - dax, ey = sy - day;
        f[0] = -kt * ex; f[1] = -kt * ey; f[2] = fn;
        flState[i] = scale > 0 ? 2 : 1;
        e += 0.5 * kn * pen * pen + 0.5 * kt * (ex * ex + ey * ey);
        if (fn > fmax) fmax = fn;
        const double dx = x[0] - c[0], dy = x[1] - c[1], dz = x[2] - c[2];
        dxx += dx * dx; dyy += dy * dy; dzz += dz * dz; nc++;
      } else {
        flAx[i] = x[0]; flAy[i] = x[1];
        f[0] = f[1] = f[2] = 0; flState[i] = 0;
      }
      for (int k = 0; k < 3; k++) F[3 * size_t(i) + k] += f[k];
      const double gx = loads[3 * size_t(i)] + f[0], gy = loads[3 * size_t(i) + 1] + f[1], gz = loads[3 * size_t(i) + 2] + f[2];
      const double dx = x[0] - c[0], dy = x[1] - c[1], dz = x[2] - c[2];
      q0 += gx; q1 += gy; q2 += gz; q3 += dy * gz - dz * gy; q4 += dz * gx - dx * gz; q5 += dx * gy - dy * gx;
    }
    floorEnergy = e; floorFnMax = fmax;
    rbQt[0] = q0; rbQt[1] = q1; rbQt[2] = q2; rbQr[0] = q3; rbQr[1] = q4; rbQr[2] = q5;
    rbD2[0] = dxx; rbD2[1] = dyy; rbD2[2] = dzz; rbNc = nc;
  }

  // ---------------------------------------------------------------------------------------------- load protocol
  // The UTM replay of the reference's GPU form (web/js/wgsl.js:1048-1093, set up by solver_gpu.js:215,286,296-318),
  // restated over this CPU iteration: the reference's CPU solver has no protocol of its own.
  ws_protocol proto{};
  double probe0[3] = {0, 0, 0}, utmPf[3] = {0, 0, 0}, utmCurF = 0, utmSum[4] = {0, 0, 0, 0};
  int utmPhase = 0, utmIt = 0, utmInc = 0, utmAccN = 0;
  bool utmDone = false;
  std::vector<double> utmOut = std::vector<double>(4 * WS_PROTOCOL_MAX_INC, 0.0);

  // P0 = the probe's position now; the first value applied (the probe placed there under displacement control)
  void startProtocol() {
    utmPhase = utmIt = utmInc = utmAccN = 0; utmDone = false;
    for (double &v : utmSum) v = 0;
    std::fill(utmOut.begin(), utmOut.end(), 0.0);
    if (!proto.mode) return;
    const size_t pb = 3 * size_t(proto.probe);
    for (int k = 0; k < 3; k++) probe0[k] = st.X[pb + k];
    utmCurF = proto.sched[0];
    for (int k = 0; k < 3; k++) utmPf[k] = proto.mode == 1 ? proto.axis[k] * proto.sched[0] : 0.0;
    if (proto.mode == 2)
      for (int k = 0; k < 3; k++) { st.X[pb + k] = probe0[k] + proto.axis[k] * proto.sched[0]; st.V[pb + k] = 0; }
  }
  // after an iteration: settle, average the read-out, record, next increment (wgsl.js:1048-1093)
  void protocolStep() {
    if (!proto.mode || utmDone) return;
    const bool conv = st.residual <= sp.tol;
    const size_t pb = 3 * size_t(proto.probe);
    utmIt += 1;
    if (utmPhase == 0) {
      if (conv || utmIt >= proto.settle) {
        utmPhase = 1; utmIt = 0; utmAccN = 0;
        for (double &v : utmSum) v = 0;
      }
    } else if (utmPhase == 1) {
      double r = 0;
      for (int k = 0; k < 3; k++) {
        utmSum[k] += st.X[pb + k] - probe0[k];
        r += reactions[pb + k] * proto.axis[k];
      }
      utmSum[3] += r;
      utmAccN += 1;
      if (utmIt >= proto.avg) {
        double *o = &utmOut[4 * size_t(utmInc)];
        const double nn = utmAccN;
        o[0] = (utmSum[0] * proto.axis[0] + utmSum[1] * proto.axis[1] + utmSum[2] * proto.axis[2]) / nn;
        o[1] = utmSum[3] / nn;
        o[2] = utmCurF;
        o[3] = st.iteration;
        utmInc += 1; utmIt = 0; utmPhase = 0;
        if (utmInc >= proto.n_inc) { utmPhase = 2; utmDone = true; }
        else {
          const double v = proto.sched[std::min(utmInc, WS_PROTOCOL_MAX_INC - 1)];
          utmCurF = v;
          if (proto.mode == 1) for (int k = 0; k < 3; k++) utmPf[k] = proto.axis[k] * v;
          else for (int k = 0; k < 3; k++) { st.X[pb + k] = probe0[k] + proto.axis[k] * v; st.V[pb + k] = 0; }
        }
      }
    }
  }

  // solver_cpu.js:670-710; rebuild = true keeps the contact and its state (rebuildGoals, :719-732)
  void buildGoals(const ws_model &md, bool rebuild) {
    const int n = st.n, m = st.m;
    rod.init(st, md);
    loadConst.assign(md.load_const, md.load_const + 3 * size_t(n));
    localNode.assign(md.local_load_node, md.local_load_node + md.n_local_loads);
    localF.assign(md.local_load_F, md.local_load_F + 3 * size_t(md.n_local_loads));
    total.assign(3 * size_t(n), 0.0);
    // Anchors (model.js:162-189)
    nodeFree.assign(3 * size_t(n), 1); fixedNodes.clear(); rotClamps.clear();
    std::vector<std::vector<int>> adj(n);
    for (int j = 0; j < m; j++) { adj[st.segI0[j]].push_back(j); adj[st.segI1[j]].push_back(j); }
    for (int i = 0; i < md.n_anchors; i++) {
      const int nid = md.anchor_node[i];
      const uint8_t mk = md.anchor_mask[i];
      for (int c = 0; c < 3; c++) if (mk & (1 << c)) nodeFree[3 * size_t(nid) + c] = 0;
      if ((mk & 7) && std::find(fixedNodes.begin(), fixedNodes.end(), nid) == fixedNodes.end()) fixedNodes.push_back(nid);
      for (int j : adj[nid]) if (mk & 0x38) rotClamps.push_back({nid, j, {bool(mk & 8), bool(mk & 16), bool(mk & 32)}});
    }
    if (proto.mode == 2) {                               // displacement control holds the probe (solver_gpu.js:215)
      const int pn = proto.probe;
      for (int c = 0; c < 3; c++) nodeFree[3 * size_t(pn) + c] = 0;
      if (std::find(fixedNodes.begin(), fixedNodes.end(), pn) == fixedNodes.end()) fixedNodes.push_back(pn);
    }
    reactions.assign(3 * size_t(n), 0.0); fixedAny.assign(n, 0);
    for (int i = 0; i < n; i++) fixedAny[i] = (nodeFree[3 * size_t(i)] && nodeFree[3 * size_t(i) + 1] && nodeFree[3 * size_t(i) + 2]) ? 0 : 1;
    rod.setClamps(st, rotClamps);
    if (!rebuild) {
      hasContact = md.params.contacts && st.K > 0;
      if (hasContact) contact.init(st, md);
    } else if (hasContact) {
      contact.p = md.params;
      contact.mu.assign(md.cross_mu, md.cross_mu + st.K);
      contact.locked.assign(md.cross_locked, md.cross_locked + st.K);
    }
    if (hasContact) {                                     // solver_cpu.js:688
      contact.setFixed(nodeFree);
      std::fill(contact.penAcc.begin(), contact.penAcc.end(), 0.0);
      contact.penN = 0;
    }
    std::vector<double> kNode(n, 0.0), kSeg(m, 0.0);
    rod.addStiffness(st, kNode);
    if (hasContact) contact.addStiffness(st, kNode, kSeg);
    floorBind(md);
    if (hasFloor) for (int i = 0; i < n; i++) kNode[i] += sp.strength + sp.stick_strength;   // Floor.addStiffness
    const double ms = sp.mass_scale;
    mass.resize(n);
    for (int i = 0; i < n; i++) mass[i] = ms * std::max(kNode[i], 1e-12);
    kRotStatic.assign(3 * size_t(m), 0.0);
    rod.addRotStiffness(st, kRotStatic);
    inertia3.resize(3 * size_t(m));
    for (int j = 0; j < m; j++) for (int k = 0; k < 3; k++) inertia3[3 * size_t(j) + k] = ms * std::max(kRotStatic[3 * size_t(j) + k] + kSeg[j], 1e-12);
    double lmin = INF;
    for (double v : st.jLen) lmin = std::min(lmin, v);
    for (double v : st.l0) lmin = std::min(lmin, v);
    lRef = std::isfinite(lmin) ? lmin : 1.0;
    F.assign(3 * size_t(n), 0.0); T.assign(3 * size_t(m), 0.0); tm.assign(3 * size_t(m), 0.0); kTw.assign(m, 0.0);
  }

  // solver_cpu.js:843-853 (no floor)
  double forceRef() const {
    double a = 0; for (double v : total) a = std::max(a, std::fabs(v));
    double b = 0; for (double v : rod.N) b = std::max(b, std::fabs(v));
    double c = 0; for (double v : rod.M) c = std::max(c, std::fabs(v));
    double lmin = INF; for (double v : st.jLen) lmin = std::min(lmin, v);
    c = st.p ? c / std::max(lmin, 1e-12) : 0;
    double d = 0;
    if (hasContact) { d = -INF; for (double v : contact.Fn) d = std::max(d, v); }
    const double e = hasFloor ? floorFnMax : 0.0;
    return std::max(std::max(std::max(a, b), std::max(c, d)), std::max(e, 1e-12));
  }

  // solver_cpu.js:737-841
  bool step(int nIter) {
    const int n = st.n, m = st.m;
    const int rampN = std::max(sp.ramp_iter, 0);
    double R[9], dq[4], qq[4], q0[4], Mrb[6], qw[4];
    std::vector<double> Xprev(3 * size_t(n)), Qprev(4 * size_t(m)), kin(3 * size_t(n)), kinR(3 * size_t(m)), nq;
    std::fill(kTw.begin(), kTw.end(), 0.0);
    double *W = st.Wr.data();
    // the rigid-body freedoms of a model that only the ground holds: off as soon as an anchor exists
    const bool rb = hasFloor && fixedNodes.empty() && rotClamps.empty();
    if (hasFloor && !rb) for (int k = 0; k < 3; k++) rbV[k] = rbW[k] = 0;
    bool broke = false;
    for (int it = 0; it < nIter; it++) {
      if (hasContact) contact.ramp = rampN == 0 ? 1.0 : std::min(1.0, 0.01 + 0.99 * st.iteration / rampN);
      std::fill(F.begin(), F.end(), 0.0); std::fill(T.begin(), T.end(), 0.0);
      rod.apply(st, F.data(), T.data());
      total = loadConst;
      if (!localNode.empty()) {
        nodeQuats(st, nq);
        double Rl[9];
        for (size_t l = 0; l < localNode.size(); l++) {
          const size_t nid = localNode[l];
          const double *Fv = &localF[3 * l];
          toFrame(&nq[4 * nid], Rl);
          for (int k = 0; k < 3; k++) total[3 * nid + k] += Rl[k] * Fv[0] + Rl[3 + k] * Fv[1] + Rl[6 + k] * Fv[2];
        }
      }
      if (proto.mode == 1)                               // the protocol's probe force (wgsl.js:914)
        for (int k = 0; k < 3; k++) total[3 * size_t(proto.probe) + k] += utmPf[k];
      for (size_t i = 0; i < 3 * size_t(n); i++) F[i] += total[i];
      if (hasContact) contact.apply(st, F.data(), T.data());
      if (hasFloor) floorApply(rampN <= 0 ? 1.0 : std::min(1.0, 0.01 + 0.99 * st.iteration / rampN), total);
      std::fill(reactions.begin(), reactions.end(), 0.0);
      for (int i = 0; i < n; i++) if (fixedAny[i]) for (int k = 0; k < 3; k++) reactions[3 * size_t(i) + k] = -F[3 * size_t(i) + k];
      for (size_t i = 0; i < 3 * size_t(n); i++) if (!nodeFree[i]) F[i] = 0;
      for (int j = 0; j < m; j++) {
        toFrame(&st.Q[4 * size_t(j)], R);
        for (int k = 0; k < 3; k++) tm[3 * size_t(j) + k] = R[3 * k] * T[3 * size_t(j)] + R[3 * k + 1] * T[3 * size_t(j) + 1] + R[3 * k + 2] * T[3 * size_t(j) + 2];
      }
      if (hasContact) { std::fill(kTw.begin(), kTw.end(), 0.0); contact.addTwistStiffness(st, kTw); }
      for (int j = 0; j < m; j++)
        for (int k = 0; k < 3; k++)
          inertia3[3 * size_t(j) + k] = sp.mass_scale * std::max(kRotStatic[3 * size_t(j) + k] + kTw[j] + rod.kDyn[3 * size_t(j) + k], 1e-12);
      Xprev = st.X; Qprev = st.Q;
      const bool warm = st.iteration < sp.warmup_iter && hasContact;
      if (warm) {
        std::fill(F.begin(), F.end(), 0.0); std::fill(st.V.begin(), st.V.end(), 0.0);
        if (rb) for (int k = 0; k < 3; k++) rbV[k] = rbW[k] = 0;
      }
      for (int i = 0; i < n; i++) for (int k = 0; k < 3; k++) st.V[3 * size_t(i) + k] += F[3 * size_t(i) + k] / mass[i];
      for (size_t j = 0; j < 3 * size_t(m); j++) W[j] += tm[j] / inertia3[j];
      for (int j = 0; j < m; j++) {
        W[3 * size_t(j) + 2] = std::min(std::max(W[3 * size_t(j) + 2], -TWIST_RATE_MAX), TWIST_RATE_MAX);
        if (kTw[j] > 0) W[3 * size_t(j) + 2] *= ROLL_DAMP;
      }
      if (sp.damping != 1.0) {
        for (size_t i = 0; i < 3 * size_t(n); i++) st.V[i] *= sp.damping;
        for (size_t j = 0; j < 3 * size_t(m); j++) W[j] *= sp.damping;
      }
      for (size_t i = 0; i < 3 * size_t(n); i++) if (!nodeFree[i]) st.V[i] = 0;
      for (size_t i = 0; i < 3 * size_t(n); i++) st.X[i] += st.V[i];
      {
        // the motion starts once the warm-up (which holds every node) is over
        const int N = sp.disp_ramp_iter, start = std::max(dispIt0, hasContact ? sp.warmup_iter : 0);
        const double r = N > 0 ? std::min(1.0, std::max(0.0, double(st.iteration - start + 1) / N)) : 1.0;
        for (int i = 0; i < n; i++)
          if (hasTarget[i])
            for (int c = 0; c < 3; c++)
              if (!nodeFree[3 * size_t(i) + c]) st.X[3 * size_t(i) + c] = ancStart[3 * size_t(i) + c] + r * ancDelta[3 * size_t(i) + c];
      }
      // rigid-body freedoms, integrated like the nodes: velocity from this iteration's resultant (v += Q / M, speed
      // limit), then the step x += v + w x (x - c) from the position before the node step, frames turned by w
      // (solver_cpu.js:785-800)
      if (rb) {
        rigidMasses(sp.mass_scale, Mrb);
        if (!warm)
          for (int k = 0; k < 3; k++) {
            rbV[k] = std::min(std::max((rbV[k] + rbQt[k] / Mrb[k]) * sp.damping, -rbVmax), rbVmax);
            rbW[k] = std::min(std::max((rbW[k] + rbQr[k] / Mrb[3 + k]) * sp.damping, -rbWmax), rbWmax);
          }
      }
      const bool rbMove = rb && (rbV[0] != 0 || rbV[1] != 0 || rbV[2] != 0 || rbW[0] != 0 || rbW[1] != 0 || rbW[2] != 0);
      if (rbMove) {
        const double *v = rbV, *w = rbW, *c = rbC;
        for (int i = 0; i < n; i++) {
          const double dx = Xprev[3 * size_t(i)] - c[0], dy = Xprev[3 * size_t(i) + 1] - c[1], dz = Xprev[3 * size_t(i) + 2] - c[2];
          st.X[3 * size_t(i)] += v[0] + w[1] * dz - w[2] * dy;
          st.X[3 * size_t(i) + 1] += v[1] + w[2] * dx - w[0] * dz;
          st.X[3 * size_t(i) + 2] += v[2] + w[0] * dy - w[1] * dx;
        }
        qexp(w[0], w[1], w[2], qw);
      }
      for (int j = 0; j < m; j++) {
        qexp(W[3 * size_t(j)], W[3 * size_t(j) + 1], W[3 * size_t(j) + 2], dq);
        for (int k = 0; k < 4; k++) q0[k] = st.Q[4 * size_t(j) + k];
        qmul(q0, dq, qq);
        if (rbMove) { for (int k = 0; k < 4; k++) q0[k] = qq[k]; qmul(qw, q0, qq); }   // the rigid step's world rotation
        qnormalize(qq);
        for (int k = 0; k < 4; k++) st.Q[4 * size_t(j) + k] = qq[k];
      }
      for (int i = 0; i < n; i++) for (int k = 0; k < 3; k++) kin[3 * size_t(i) + k] = mass[i] * st.V[3 * size_t(i) + k] * st.V[3 * size_t(i) + k];
      for (size_t j = 0; j < 3 * size_t(m); j++) kinR[j] = inertia3[j] * W[j] * W[j];
      ke = 0.5 * (pairwiseSum(kin) + pairwiseSum(kinR));
      if (rb) for (int k = 0; k < 3; k++) ke += 0.5 * (Mrb[k] * rbV[k] * rbV[k] + Mrb[3 + k] * rbW[k] * rbW[k]);
      if (sp.kinetic_damping && ke < kePrev) {
        st.X = Xprev; st.Q = Qprev;
        std::fill(st.V.begin(), st.V.end(), 0.0); std::fill(st.Wr.begin(), st.Wr.end(), 0.0);
        if (rb) for (int k = 0; k < 3; k++) rbV[k] = rbW[k] = 0;
        ke = 0.0; rollbacks++;
      }
      kePrev = ke;
      st.iteration += 1;
      // augmented Lagrangian: Uzawa update every al_every iterations once the ramp is over (solver_cpu.js:819-821)
      if (hasContact && contact.p.augmented && contact.p.al_every > 0 && st.iteration > rampN &&
          (st.iteration - rampN) % contact.p.al_every == 0)
        contact.updateMultipliers(st);
      double fmax = 0, tmax = 0;
      for (int i = 0; i < n; i++) {
        const double f = std::sqrt(F[3 * size_t(i)] * F[3 * size_t(i)] + F[3 * size_t(i) + 1] * F[3 * size_t(i) + 1] + F[3 * size_t(i) + 2] * F[3 * size_t(i) + 2]);
        if (f > fmax) fmax = f;
      }
      for (int j = 0; j < m; j++) {
        const double t = std::sqrt(tm[3 * size_t(j)] * tm[3 * size_t(j)] + tm[3 * size_t(j) + 1] * tm[3 * size_t(j) + 1] + tm[3 * size_t(j) + 2] * tm[3 * size_t(j) + 2]);
        if (t > tmax) tmax = t;
      }
      fref = forceRef();
      resF = n ? fmax / fref : 0; resT = m ? tmax / (fref * lRef) : 0;
      resRigid = rb ? rigidResidual(fref) : 0;
      const double resid = std::max(std::max(resF, resT), resRigid);
      st.residual = st.iteration > sp.warmup_iter ? resid : INF;
      if (proto.mode) {                                  // a load protocol runs on past convergence
        protocolStep();
        if (utmDone) break;
        continue;
      }
      if (st.residual <= sp.tol) { converged = true; broke = true; break; }
    }
    if (proto.mode) return utmDone;
    if (!broke) converged = st.residual <= sp.tol;
    return converged;
  }

  // rebuildGoals with new parameters: state kept; anchored translations move to the model's targets from where they are
  void rebuild(const ws_model &md) {
    sp = md.params;
    buildGoals(md, true);
    setTargets(md);
    converged = false; kePrev = 0.0;
  }
};

}  // namespace orc

// ------------------------------------------------------------------------------------------------ C entry points
extern "C" {

struct orc_view {
  int32_t n, m, p, K, iteration, converged, rollbacks, has_contact;
  double residual, ke_prev, ke, fref, res_force, res_torque, l_ref;
  double e_stretch, e_shear, e_bend, e_twist, e_contact;
  double *X, *X0, *V, *Q, *W, *u, *nprev, *slip, *Fn, *Ft, *gap, *state, *N, *Vsh, *M, *reactions, *mass, *inertia3, *k_rot_static, *F, *T, *tm;
  uint8_t *stuck;
  int32_t *ctype;
  double *theta, *phi, *area, *pressure, *util;
  double *lambda, *dent, *M_rot, *rot_slip;     // contact extensions (buildResults, solver_cpu.js:906-908)
  double *utm;                                  // load protocol read-out [4 WS_PROTOCOL_MAX_INC]
  int32_t utm_inc, utm_phase, utm_done, has_floor;
  double *floor_F, e_floor;                     // the ground
  uint8_t *floor_state;
  double res_rigid, rb_v[3], rb_w[3];           // the rigid-body freedoms: residual part, velocities
};

void *orc_create(const ws_model *md) {
  try {
    auto *s = new orc::Solver();
    s->load(*md);
    return s;
  } catch (...) { return nullptr; }
}
void orc_free(void *h) { delete static_cast<orc::Solver *>(h); }
int orc_step(void *h, int32_t n) { return static_cast<orc::Solver *>(h)->step(n) ? 1 : 0; }
void orc_rebuild(void *h, const ws_model *md) { static_cast<orc::Solver *>(h)->rebuild(*md); }
void orc_internalize(void *h) {
  auto *s = static_cast<orc::Solver *>(h);
  s->st.X0 = s->st.X; s->st.Q0 = s->st.Q; std::fill(s->st.slip.begin(), s->st.slip.end(), 0.0);
}
void orc_view_get(void *h, orc_view *v) {
  auto *s = static_cast<orc::Solver *>(h);
  orc::St &st = s->st;
  v->n = st.n; v->m = st.m; v->p = st.p; v->K = st.K; v->iteration = st.iteration; v->converged = s->converged;
  v->rollbacks = s->rollbacks; v->has_contact = s->hasContact;
  v->residual = st.residual; v->ke_prev = s->kePrev; v->ke = s->ke; v->fref = s->fref; v->res_force = s->resF; v->res_torque = s->resT; v->l_ref = s->lRef;
  v->res_rigid = s->resRigid;
  for (int k = 0; k < 3; k++) { v->rb_v[k] = s->rbV[k]; v->rb_w[k] = s->rbW[k]; }
  v->e_stretch = s->rod.eStretch; v->e_shear = s->rod.eShear; v->e_bend = s->rod.eBend; v->e_twist = s->rod.eTwist;
  v->e_contact = s->hasContact ? s->contact.energy : 0.0;
  v->X = st.X.data(); v->X0 = st.X0.data(); v->V = st.V.data(); v->Q = st.Q.data(); v->W = st.Wr.data();
  v->u = st.u.data(); v->nprev = st.nPrev.data(); v->slip = st.slip.data(); v->stuck = st.stuck.data();
  v->Fn = s->hasContact ? s->contact.Fn.data() : nullptr; v->Ft = s->hasContact ? s->contact.Ft.data() : nullptr;
  v->gap = s->hasContact ? s->contact.gap.data() : nullptr; v->state = s->hasContact ? s->contact.state.data() : nullptr;
  v->ctype = s->hasContact ? s->contact.ctype.data() : nullptr; v->theta = s->hasContact ? s->contact.theta.data() : nullptr;
  v->phi = s->hasContact ? s->contact.phi.data() : nullptr; v->area = s->hasContact ? s->contact.Anom.data() : nullptr;
  v->pressure = s->hasContact ? s->contact.pressure.data() : nullptr; v->util = s->hasContact ? s->contact.util.data() : nullptr;
  if (s->hasContact) {
    orc::Contact &ct = s->contact;
    ct.dentSum.resize(ct.K);
    for (int k = 0; k < ct.K; k++) ct.dentSum[k] = ct.dent[2 * size_t(k)] + ct.dent[2 * size_t(k) + 1] + ct.dentE[k];
  }
  v->lambda = s->hasContact ? s->contact.lam.data() : nullptr; v->dent = s->hasContact ? s->contact.dentSum.data() : nullptr;
  v->M_rot = s->hasContact ? s->contact.Mrot.data() : nullptr; v->rot_slip = s->hasContact ? s->contact.rotSlip.data() : nullptr;
  v->utm = s->utmOut.data(); v->utm_inc = s->utmInc; v->utm_phase = s->utmPhase; v->utm_done = s->utmDone ? 1 : 0;
  v->has_floor = s->hasFloor; v->floor_F = s->hasFloor ? s->flF.data() : nullptr; v->e_floor = s->floorEnergy;
  v->floor_state = s->hasFloor ? s->flState.data() : nullptr;
  v->N = s->rod.N.data(); v->Vsh = s->rod.Vs.data(); v->M = s->rod.M.data(); v->reactions = s->reactions.data();
  v->mass = s->mass.data(); v->inertia3 = s->inertia3.data(); v->k_rot_static = s->kRotStatic.data();
  v->F = s->F.data(); v->T = s->T.data(); v->tm = s->tm.data();
}
// rod forces and energy at positions X [3n] and frames Q [4m] (the state is left as it was); F [3n], T [3m] are
// overwritten.  rod_check.mjs differentiates this energy.
double orc_rod_eval(void *h, const double *X, const double *Q, double *F, double *T) {
  auto *s = static_cast<orc::Solver *>(h);
  orc::St &st = s->st;
  std::vector<double> X0 = st.X, Q0 = st.Q;
  std::copy(X, X + 3 * size_t(st.n), st.X.begin());
  std::copy(Q, Q + 4 * size_t(st.m), st.Q.begin());
  std::fill(F, F + 3 * size_t(st.n), 0.0);
  std::fill(T, T + 3 * size_t(st.m), 0.0);
  s->rod.apply(st, F, T);
  st.X = X0; st.Q = Q0;
  return s->rod.energy;
}
// rod clamps from (node, segment, mask) triples, re-frozen at the current frames (setClamps)
void orc_set_clamps(void *h, int32_t nc, const int32_t *node, const int32_t *seg, const uint8_t *mask) {
  auto *s = static_cast<orc::Solver *>(h);
  std::vector<orc::Clamp> rc;
  for (int i = 0; i < nc; i++) rc.push_back({node[i], seg[i], {bool(mask[i] & 1), bool(mask[i] & 2), bool(mask[i] & 4)}});
  s->rod.setClamps(s->st, rc);
}
// overwrite positions / frames / rest curvature of the state
void orc_set_state(void *h, const double *X, const double *Q, const double *omega0) {
  auto *s = static_cast<orc::Solver *>(h);
  if (X) std::copy(X, X + 3 * size_t(s->st.n), s->st.X.begin());
  if (Q) std::copy(Q, Q + 4 * size_t(s->st.m), s->st.Q.begin());
  if (omega0) std::copy(omega0, omega0 + 3 * size_t(s->st.p), s->st.Omega0.begin());
}
// results: segment moments Mx My T from the joint moments (buildResults, solver_cpu.js:878-898); seg_m [3m]
void orc_segment_moments(void *h, double *seg_m) {
  auto *s = static_cast<orc::Solver *>(h);
  const orc::St &st = s->st;
  const int n = st.n, m = st.m;
  std::vector<double> nodeM(3 * size_t(n), 0.0);
  std::vector<uint8_t> has0(n, 0);
  // joint node of joint j: the node shared by its two segments
  for (int j = 0; j < st.p; j++) {
    const int sa = st.jSeg0[j];
    const size_t i = st.segI1[sa];
    for (int k = 0; k < 3; k++) nodeM[3 * i + k] = s->rod.M[3 * size_t(j) + k];
    has0[i] = 1;
  }
  std::vector<uint8_t> hasB = has0;
  for (size_t c = 0; c < s->rod.cNode.size(); c++) {
    const size_t i = s->rod.cNode[c];
    nodeM[3 * i] = s->rod.cM[2 * c]; nodeM[3 * i + 1] = s->rod.cM[2 * c + 1]; hasB[i] = 1;
  }
  for (int j = 0; j < m; j++) for (int k = 0; k < 3; k++) seg_m[3 * size_t(j) + k] = 0.5 * (nodeM[3 * size_t(st.segI0[j]) + k] + nodeM[3 * size_t(st.segI1[j]) + k]);
  const int colsB[2] = {0, 1}, cols0[1] = {2};
  for (int pass = 0; pass < 2; pass++) {
    const int *cols = pass == 0 ? colsB : cols0;
    const int nc = pass == 0 ? 2 : 1;
    const std::vector<uint8_t> &has = pass == 0 ? hasB : has0;
    for (int j = 0; j < m; j++) { const int a = st.segI0[j], b = st.segI1[j]; for (int q = 0; q < nc; q++) if (!has[a]) seg_m[3 * size_t(j) + cols[q]] = nodeM[3 * size_t(b) + cols[q]]; }
    for (int j = 0; j < m; j++) { const int a = st.segI0[j], b = st.segI1[j]; for (int q = 0; q < nc; q++) if (!has[b]) seg_m[3 * size_t(j) + cols[q]] = nodeM[3 * size_t(a) + cols[q]]; }
  }
}
// results: the segment layers Mx My T N at the nodes (fields.js nodeValues without shear): the mean of a node's two
// segments along its strand, the one segment at a strand's end, closed strands wrapping; out [4n] layer-major
void orc_node_layers(void *h, double *out) {
  auto *s = static_cast<orc::Solver *>(h);
  const orc::St &st = s->st;
  const int n = st.n, m = st.m;
  std::vector<double> seg(3 * size_t(m));
  orc_segment_moments(h, seg.data());
  std::fill(out, out + 4 * size_t(n), 0.0);
  for (int S = 0; S < int(st.segOffset.size()) - 1; S++) {
    const int j0 = st.segOffset[S], ms = st.segOffset[S + 1] - j0;
    if (ms < 1) continue;
    const bool closed = ms > 2 && st.segI1[j0 + ms - 1] == st.segI0[j0];
    for (int L = 0; L < 4; L++) {
      auto A = [&](int j) { return L < 3 ? seg[3 * size_t(j0 + j) + L] : s->rod.N[j0 + j]; };
      double *o = out + size_t(L) * n;
      if (closed) {
        for (int i = 0; i < ms; i++) o[st.segI0[j0 + i]] = 0.5 * (A((i - 1 + ms) % ms) + A(i));
      } else {
        for (int j = 0; j < ms; j++) { o[st.segI0[j0 + j]] += A(j); o[st.segI1[j0 + j]] += A(j); }
        for (int j = 1; j < ms; j++) o[st.segI0[j0 + j]] *= 0.5;
      }
    }
  }
}

}  // extern "C"
