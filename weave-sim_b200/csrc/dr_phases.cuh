// The phases of one dynamic-relaxation iteration (CpuSolver.step, web/js/solver_cpu.js:737-841) as device functions
// over element ranges.  Every phase writes disjoint outputs; the force gather is conflict-free (no atomics):
//   A  elements:  segments (stretch/shear force n, e × n)          rod_cosserat.js:118-133
//                 joints (bend/twist torque, kDyn share)           rod_cosserat.js:136-159
//                 clamps (joints against frozen frames)            rod_cosserat.js:161-180
//                 crossings (Hermite evaluation, normal, gap, penalty, Coulomb return mapping, slide of u on both
//                 laths, force and lever torque per side)          solver_cpu.js:179-228, 274-282, 381-478
//   BC sides:     new sorted order of the crossing sides along each strand, by rank (each side counts the sides
//                 before it); segments: their slice of that order, by counting the keys below and equal
//                 (both read only the keys of phase A, so they share one phase)
//   D  nodes:     F = n_out − n_in + loads + Σ sides on the two adjacent segments (weights 1 − t, t, the slices of
//                 the previous sort); reactions, fixed DOFs, warm-up, v += F/m, x += v, prescribed support motion
//                 segments: T = e × n ± joint torques − clamp torques + lever torques; tm = Rᵀ T; frame inertia
//                 with the righting share of the crossings on the segment now (the new slices) and kDyn;
//                 ω += tm / I, roll limit and roll damping, q ← q ⊗ exp(ω)
//   E  instance:  kinetic energy, kinetic-damping roll-back, residual, convergence (one thread)
#pragma once
#include <cfloat>

#include "../../include/weavesim.h"
#include "dr_common.cuh"

namespace wsb {

static constexpr double SUPPORT_SMOOTH = 0.03;                // solver_cpu.js:16
static constexpr double TWIST_RATE_MAX = 0.5 * SUPPORT_SMOOTH;  // solver_cpu.js:21
static constexpr double ROLL_DAMP = 0.5;                      // solver_cpu.js:28
static constexpr double AL_FREE_MIN = 0.25;                   // solver_cpu.js:33
static constexpr double PI_D = 3.141592653589793;             // Math.PI

// ------------------------------------------------------------------------------------------------ math helpers
__device__ __forceinline__ float msqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double msqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float matan2(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double matan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float mtanh(float x) { return tanhf(x); }
__device__ __forceinline__ float masin(float x) { return asinf(x); }
__device__ __forceinline__ double masin(double x) { return asin(x); }
__device__ __forceinline__ double mtanh(double x) { return tanh(x); }
__device__ __forceinline__ void msincos(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void msincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ float mfloor(float x) { return floorf(x); }
__device__ __forceinline__ double mfloor(double x) { return floor(x); }
__device__ __forceinline__ float msin(float x) { return sinf(x); }
__device__ __forceinline__ double msin(double x) { return sin(x); }
__device__ __forceinline__ float mcos(float x) { return cosf(x); }
__device__ __forceinline__ double mcos(double x) { return cos(x); }
__device__ __forceinline__ float mtan(float x) { return tanf(x); }
__device__ __forceinline__ double mtan(double x) { return tan(x); }
__device__ __forceinline__ float macos(float x) { return acosf(x); }
__device__ __forceinline__ double macos(double x) { return acos(x); }
__device__ __forceinline__ float mfmod(float x, float y) { return fmodf(x, y); }
__device__ __forceinline__ double mfmod(double x, double y) { return fmod(x, y); }
// Math.sign: −1, 0 or +1
template <class T> __device__ __forceinline__ T msign(T v) { return v > T(0) ? T(1) : (v < T(0) ? T(-1) : T(0)); }
template <class T> __device__ __forceinline__ T mmin(T a, T b) { return a < b ? a : b; }
template <class T> __device__ __forceinline__ T mmax(T a, T b) { return a > b ? a : b; }
template <class T> __device__ __forceinline__ T mabs(T a) { return a < T(0) ? -a : a; }
template <class T> __device__ __forceinline__ T mclamp(T v, T lo, T hi) { return mmin(mmax(v, lo), hi); }

// Scale that takes a near-unit quaternion of squared norm n2 = 1 + δ to unit length: 1/√(1 + δ) = 1 − δ/2 + 3δ²/8
// + O(δ³), the binomial series.  Used on frames stored as two floats and renormalised every iteration (|δ| below
// ~1e-7), where the remainder is under the double rounding of the result; the exact form is kept everywhere else.
template <class T>
__device__ __forceinline__ T nearUnitScale(T n2) {
  const T dl = n2 - T(1);
  return T(1) + dl * (T(-0.5) + T(0.375) * dl);
}

// frame [X | Y | Z] of a quaternion (normalised first): quat.js:19-27; NU: q is near unit (see nearUnitScale)
template <class T, bool NU = false>
__device__ __forceinline__ void qframe(const T q[4], T R[9]) {
  T w = q[0], x = q[1], y = q[2], z = q[3];
  const T n2 = w * w + x * x + y * y + z * z;
  T in;
  if constexpr (NU) {
    in = nearUnitScale(n2);
  } else {
    T n = msqrt(n2);
    if (n == T(0)) n = T(1);
    in = T(1) / n;
  }
  w *= in; x *= in; y *= in; z *= in;
  R[0] = T(1) - T(2) * (y * y + z * z); R[1] = T(2) * (x * y + z * w); R[2] = T(2) * (x * z - y * w);
  R[3] = T(2) * (x * y - z * w); R[4] = T(1) - T(2) * (x * x + z * z); R[5] = T(2) * (y * z + x * w);
  R[6] = T(2) * (x * z + y * w); R[7] = T(2) * (y * z - x * w); R[8] = T(1) - T(2) * (x * x + y * y);
}
template <class T>
__device__ __forceinline__ void qmul(const T a[4], const T b[4], T o[4]) {
  o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  o[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  o[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  o[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}
template <class T, bool NU = false>
__device__ __forceinline__ void qnormalize(T q[4]) {
  const T n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if constexpr (NU) {
    const T f = nearUnitScale(n2);
    q[0] *= f; q[1] *= f; q[2] *= f; q[3] *= f;
  } else {
    T n = msqrt(n2);
    if (n == T(0)) n = T(1);
    q[0] /= n; q[1] /= n; q[2] /= n; q[3] /= n;
  }
}
template <class T>
__device__ __forceinline__ void cross3(const T a[3], const T b[3], T o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; o[2] = a[0] * b[1] - a[1] * b[0];
}
template <class T> __device__ __forceinline__ T dot3(const T a[3], const T b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// β of J_l⁻ᵀ(Ψ) = 1 + ½[Ψ]× + β[Ψ]×²: 1/θ² − (1 + cos θ)/(2θ sin θ), series 1/12 + θ²/720 + θ⁴/30240 near 0
// (rod_cosserat.js:147-148 switches at 1e-3; in float the closed form cancels below ~0.3 rad, so float switches there)
template <class T>
__device__ __forceinline__ T jbeta(T th) {
  const T thr = sizeof(T) == 8 ? T(1e-3) : T(0.3);
  if (th < thr) {
    const T t2 = th * th;
    return sizeof(T) == 8 ? T(1.0 / 12) + t2 / T(720) : T(1.0 / 12) + t2 * (T(1.0 / 720) + t2 * T(1.0 / 30240));
  }
  T s, c;
  msincos(th, &s, &c);
  return T(1) / (th * th) - (T(1) + c) / (T(2) * th * s);
}

// ------------------------------------------------------------------------------------------------ state access
template <int P> struct Acc {
  using D = Dev<P>;
  using R = typename D::R; using W = typename D::W; using S = typename D::S;
  __device__ static __forceinline__ W xw(const D &d, int buf, int k, int i) {
    const size_t o = size_t(buf) * d.xB + size_t(k) * d.nS + i;
    if constexpr (PrecT<P>::TWO) return W(d.X[o]) + W(d.Xlo[o]); else return W(d.X[o]);
  }
  __device__ static __forceinline__ R xr(const D &d, int buf, int k, int i) { return R(d.X[size_t(buf) * d.xB + size_t(k) * d.nS + i]); }
  __device__ static __forceinline__ void xs(const D &d, int buf, int k, int i, W v) {
    const size_t o = size_t(buf) * d.xB + size_t(k) * d.nS + i;
    if constexpr (PrecT<P>::TWO) { const S hi = S(v); d.X[o] = hi; d.Xlo[o] = S(v - W(hi)); } else d.X[o] = S(v);
  }
  __device__ static __forceinline__ W qw(const D &d, int buf, int k, int j) {
    const size_t o = size_t(buf) * d.qB + size_t(k) * d.mS + j;
    if constexpr (PrecT<P>::TWO) return W(d.Q[o]) + W(d.Qlo[o]); else return W(d.Q[o]);
  }
  __device__ static __forceinline__ R qr(const D &d, int buf, int k, int j) { return R(d.Q[size_t(buf) * d.qB + size_t(k) * d.mS + j]); }
  __device__ static __forceinline__ void qs(const D &d, int buf, int k, int j, W v) {
    const size_t o = size_t(buf) * d.qB + size_t(k) * d.mS + j;
    if constexpr (PrecT<P>::TWO) { const S hi = S(v); d.Q[o] = hi; d.Qlo[o] = S(v - W(hi)); } else d.Q[o] = S(v);
  }
  // edge vector x_b − x_a formed in the wide type, returned in R
  __device__ static __forceinline__ void edge(const D &d, int buf, int a, int b, R e[3]) {
    for (int k = 0; k < 3; k++) e[k] = R(xw(d, buf, k, b) - xw(d, buf, k, a));
  }
};

// reduction partials of one thread
template <class A>
struct Part {
  A s[RS_NSUM];
  A x[RX_NMAX];
  __device__ void init() {
    for (int i = 0; i < RS_NSUM; i++) s[i] = A(0);
    for (int i = 0; i < RX_NMAX; i++) x[i] = A(0);
    x[RX_FN] = -A(INFINITY);
  }
};

// Arrays that never change during a step (topology, masses, loads, stiffness, crossing constants) are read through the
// read-only path; they live in global memory in every form.
template <class T> __device__ __forceinline__ T ro(const T *p) { return __ldg(p); }

// ------------------------------------------------------------------------------------------------ node helpers
// node tangent: normalised sum of the unit chords of the adjacent segments (PolylineContact._prepare), from its
// outgoing chord (o0 → o1) and incoming chord (i0 → i1) given by their end nodes; a chord whose first node is negative
// is absent
template <int P>
__device__ __forceinline__ void chordTangent(const Dev<P> &d, int buf, int o0, int o1, int i0, int i1, typename Dev<P>::R T[3]) {
  using R = typename Dev<P>::R;
  T[0] = T[1] = T[2] = R(0);
  auto chord = [&](int a, int b) {
    R e[3];
    Acc<P>::edge(d, buf, a, b, e);
    const R l = mmax(msqrt(dot3(e, e)), R(1e-12));
    for (int k = 0; k < 3; k++) T[k] += e[k] / l;
  };
  if (o0 >= 0) chord(o0, o1);
  if (i0 >= 0) chord(i0, i1);
  const R l = mmax(msqrt(dot3(T, T)), R(1e-12));
  for (int k = 0; k < 3; k++) T[k] /= l;
}
// the same for node i, from its outgoing and incoming segments
template <int P>
__device__ __forceinline__ void nodeTangent(const Dev<P> &d, int buf, int i, typename Dev<P>::R T[3]) {
  const int so = ro(d.nsOut + i), si = ro(d.nsIn + i);
  chordTangent<P>(d, buf, so >= 0 ? ro(d.segI0 + so) : -1, so >= 0 ? ro(d.segI1 + so) : -1,
                  si >= 0 ? ro(d.segI0 + si) : -1, si >= 0 ? ro(d.segI1 + si) : -1, T);
}
// hemisphere-consistent mean of the adjacent segment frames (nodeQuats, model.js:89-105)
// WIDE: from the frames in the wide type (the two-float frames of the mixed policy in double), in that type
template <int P, bool WIDE = false>
__device__ __forceinline__ void segsQuat(const Dev<P> &d, int buf, int so, int si,
                                         std::conditional_t<WIDE, typename Dev<P>::W, typename Dev<P>::R> q[4]) {
  using R = std::conditional_t<WIDE, typename Dev<P>::W, typename Dev<P>::R>;
  auto rd = [&](int k, int j) -> R {
    if constexpr (WIDE) return Acc<P>::qw(d, buf, k, j);
    else return Acc<P>::qr(d, buf, k, j);
  };
  const int ref = so >= 0 ? so : si;
  q[0] = q[1] = q[2] = q[3] = R(0);
  if (ref < 0) return;
  R qr[4];
  for (int k = 0; k < 4; k++) qr[k] = rd(k, ref);
  auto add = [&](int j) {
    R qj[4];
    for (int k = 0; k < 4; k++) qj[k] = rd(k, j);
    const R dd = qj[0] * qr[0] + qj[1] * qr[1] + qj[2] * qr[2] + qj[3] * qr[3];
    const R sg = dd < R(0) ? R(-1) : R(1);
    for (int k = 0; k < 4; k++) q[k] += sg * qj[k];
  };
  if (so >= 0) add(so);
  if (si >= 0) add(si);
  qnormalize(q);
}
// the same for node i, from its outgoing and incoming segments
template <int P>
__device__ __forceinline__ void nodeQuat(const Dev<P> &d, int buf, int i, typename Dev<P>::R q[4]) {
  segsQuat<P>(d, buf, ro(d.nsOut + i), ro(d.nsIn + i), q);
}

// ------------------------------------------------------------------------------------------------ phase A
// segment j: σ = Rᵀe/l0 − e3, n = R·diag(κGA, κGA, EA)·σ (rod_cosserat.js:118-133)
template <int P>
__device__ __forceinline__ void segForce(const Dev<P> &d, int buf, int j, Part<typename Dev<P>::A> &pt) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A;
  const int a = ro(d.segI0 + j), b = ro(d.segI1 + j);
  W ew[3], qw[4], Rw[9];
  for (int k = 0; k < 3; k++) ew[k] = Acc<P>::xw(d, buf, k, b) - Acc<P>::xw(d, buf, k, a);
  for (int k = 0; k < 4; k++) qw[k] = Acc<P>::qw(d, buf, k, j);
  R s1, s2, s3;
  if constexpr (P == PREC_MIXED) {      // two-float frames are near unit; the inverse rest length is kept in f64
    qframe<W, true>(qw, Rw);
    const W il = ro(d.il0 + j);
    s1 = R((Rw[0] * ew[0] + Rw[1] * ew[1] + Rw[2] * ew[2]) * il);
    s2 = R((Rw[3] * ew[0] + Rw[4] * ew[1] + Rw[5] * ew[2]) * il);
    s3 = R((Rw[6] * ew[0] + Rw[7] * ew[1] + Rw[8] * ew[2]) * il - W(1));
  } else {
    qframe(qw, Rw);
    const W l0 = W(ro(d.l0 + j));
    s1 = R((Rw[0] * ew[0] + Rw[1] * ew[1] + Rw[2] * ew[2]) / l0);
    s2 = R((Rw[3] * ew[0] + Rw[4] * ew[1] + Rw[5] * ew[2]) / l0);
    s3 = R((Rw[6] * ew[0] + Rw[7] * ew[1] + Rw[8] * ew[2]) / l0 - W(1));
  }
  const R GA = ro(d.GA + j), EA = ro(d.EA + j);
  const R n1 = GA * s1, n2 = GA * s2, n3 = EA * s3;
  R Rr[9];
  for (int k = 0; k < 9; k++) Rr[k] = R(Rw[k]);
  const R nv[3] = {n1 * Rr[0] + n2 * Rr[3] + n3 * Rr[6], n1 * Rr[1] + n2 * Rr[4] + n3 * Rr[7], n1 * Rr[2] + n2 * Rr[5] + n3 * Rr[8]};
  const R e[3] = {R(ew[0]), R(ew[1]), R(ew[2])};
  R en[3];
  cross3(e, nv, en);
  const int ms = d.mS;
  for (int k = 0; k < 3; k++) { d.nF[k * ms + j] = nv[k]; d.en[k * ms + j] = en[k]; }
  d.Nax[j] = n3; d.Vsh[j] = n1; d.Vsh[d.mtot + j] = n2;
  const R l0r = ro(d.l0 + j);
  pt.s[RS_STRETCH] += A(R(0.5) * l0r * n3 * s3);
  pt.s[RS_SHEAR] += A(R(0.5) * l0r * (n1 * s1 + n2 * s2));
  pt.x[RX_N] = mmax(pt.x[RX_N], A(mabs(n3)));
}

// relative rotation Ψ = log(q_a* ⊗ q_b) (rod_cosserat.js:33-45); the product in the wide type, the log in R
template <int P>
__device__ __forceinline__ typename Dev<P>::R relRot(const typename Dev<P>::W qa[4], const typename Dev<P>::W qb[4], typename Dev<P>::R psi[3]) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W;
  const W ac[4] = {qa[0], -qa[1], -qa[2], -qa[3]};
  W pw[4];
  qmul(ac, qb, pw);
  R w = R(pw[0]), x = R(pw[1]), y = R(pw[2]), z = R(pw[3]);
  if (w < R(0)) { w = -w; x = -x; y = -y; z = -z; }
  const R s = msqrt(x * x + y * y + z * z), th = R(2) * matan2(s, w);
  const R f = s > R(1e-12) ? th / s : R(2) / mmax(w, R(1e-12));
  psi[0] = f * x; psi[1] = f * y; psi[2] = f * z;
  return th;
}

// J_l⁻ᵀ(Ψ) m = m + ½ Ψ × m + β Ψ × (Ψ × m)
template <class R>
__device__ __forceinline__ void jlinvT(const R psi[3], const R m[3], R th, R j[3]) {
  const R beta = jbeta(th);
  R c[3], e[3];
  cross3(psi, m, c);
  cross3(psi, c, e);
  for (int k = 0; k < 3; k++) j[k] = m[k] + R(0.5) * c[k] + beta * e[k];
}

// joint jt between segments sa -> sb (rod_cosserat.js:136-159)
template <int P>
__device__ __forceinline__ void jointTorque(const Dev<P> &d, int buf, int jt, Part<typename Dev<P>::A> &pt) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A;
  const int sa = ro(d.jS0 + jt), sb = ro(d.jS1 + jt), pt_ = d.ptot;
  W qa[4], qb[4];
  for (int k = 0; k < 4; k++) { qa[k] = Acc<P>::qw(d, buf, k, sa); qb[k] = Acc<P>::qw(d, buf, k, sb); }
  R psi[3];
  const R th = relRot<P>(qa, qb, psi);
  const R lb = ro(d.jLen + jt);
  const R dd[3] = {psi[0] / lb - ro(d.om + jt), psi[1] / lb - ro(d.om + pt_ + jt), psi[2] / lb - ro(d.om + 2 * pt_ + jt)};
  const R EIx = ro(d.EIx + jt), EIy = ro(d.EIy + jt), GJ = ro(d.GJ + jt);
  const R mm[3] = {EIx * dd[0], EIy * dd[1], GJ * dd[2]};
  {
    const R q0 = psi[0] * psi[0], q1 = psi[1] * psi[1], q2 = psi[2] * psi[2], f = R(0.25) / lb;
    d.kd[jt] = f * (EIy * q2 + GJ * q1);
    d.kd[d.pS + jt] = f * (EIx * q2 + GJ * q0);
    d.kd[2 * d.pS + jt] = f * (EIx * q1 + EIy * q0);
  }
  R jv[3];
  jlinvT(psi, mm, th, jv);
  R qr[4], Ra[9];
  for (int k = 0; k < 4; k++) qr[k] = R(qa[k]);
  qframe(qr, Ra);
  for (int k = 0; k < 3; k++) {
    d.tau[k * d.pS + jt] = jv[0] * Ra[k] + jv[1] * Ra[3 + k] + jv[2] * Ra[6 + k];
    d.Mj[k * pt_ + jt] = mm[k];
  }
  pt.s[RS_BEND] += A(R(0.5) * lb * (mm[0] * dd[0] + mm[1] * dd[1]));
  pt.s[RS_TWIST] += A(R(0.5) * lb * mm[2] * dd[2]);
  pt.x[RX_M] = mmax(pt.x[RX_M], A(mmax(mabs(mm[0]), mmax(mabs(mm[1]), mabs(mm[2])))));
}

// clamp joint cc: frozen frame (side a) -> segment frame j (side b) (rod_cosserat.js:161-180)
template <int P>
__device__ __forceinline__ void clampTorque(const Dev<P> &d, int buf, int cc, Part<typename Dev<P>::A> &pt) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A;
  const int j = ro(d.cSeg + cc), ct = d.ctot;
  W qa[4], qb[4];
  for (int k = 0; k < 4; k++) { qa[k] = ro(d.cQ + k * ct + cc); qb[k] = Acc<P>::qw(d, buf, k, j); }
  R psi[3];
  const R th = relRot<P>(qa, qb, psi);
  const R lc = ro(d.cLen + cc);
  const R dd[3] = {psi[0] / lc, psi[1] / lc, psi[2] / lc};
  const R mm[3] = {ro(d.cB + cc) * dd[0], ro(d.cB + ct + cc) * dd[1], ro(d.cB + 2 * ct + cc) * dd[2]};
  R jv[3];
  jlinvT(psi, mm, th, jv);
  R qr[4], Rc[9];
  for (int k = 0; k < 4; k++) qr[k] = R(qa[k]);
  qframe(qr, Rc);
  for (int k = 0; k < 3; k++) d.tauC[k * d.cS + cc] = jv[0] * Rc[k] + jv[1] * Rc[3 + k] + jv[2] * Rc[6 + k];
  d.cM[cc] = mm[0]; d.cM[ct + cc] = mm[1];
  pt.s[RS_BEND] += A(R(0.5) * lc * (mm[0] * dd[0] + mm[1] * dd[1]));
  pt.s[RS_TWIST] += A(R(0.5) * lc * mm[2] * dd[2]);
}

// half-extent h(n) and smoothed support point r of a section (PolylineContact._support, solver_cpu.js:274-282)
template <class R>
__device__ __forceinline__ R support(const R Rf[9], const R n[3], R sign, R w, R h, R r[3]) {
  const R nx = (n[0] * Rf[0] + n[1] * Rf[1] + n[2] * Rf[2]) * sign, ny = (n[0] * Rf[3] + n[1] * Rf[4] + n[2] * Rf[5]) * sign;
  const R hh = R(0.5) * w * mabs(nx) + R(0.5) * h * mabs(ny);
  const R ax = R(0.5) * w * mtanh(nx / R(SUPPORT_SMOOTH)), ay = R(0.5) * h * mtanh(ny / R(SUPPORT_SMOOTH));
  for (int k = 0; k < 3; k++) r[k] = ax * Rf[k] + ay * Rf[3 + k];
  return hh;
}

// ------------------------------------------------------------------------------------------------ W1 / W2 / W3 / AL
// W1 per side (PolylineContact._classify, solver_cpu.js:234-244): does the side bear on an edge, the width of its
// contact face, the depth behind it, and the roll of its section against the contact plane, from the contact normal in
// the side's section frame (nx, ny)
template <class R>
__device__ __forceinline__ void sideClass(R nx, R ny, R wk, R hk, double thr, int &edge, R &cFace, R &Z0, R &phi) {
  const R sx = mabs(mtanh(nx / R(SUPPORT_SMOOTH))), sy = mabs(mtanh(ny / R(SUPPORT_SMOOTH)));
  edge = sx * sy > R(thr) ? 1 : 0;
  const bool yFace = mabs(ny) >= mabs(nx);
  cFace = yFace ? wk : hk;
  Z0 = yFace ? hk : wk;
  phi = matan2(mmin(mabs(nx), mabs(ny)), mmax(mmax(mabs(nx), mabs(ny)), R(1e-12)));
}
// W1 per crossing (solver_cpu.js:245-269): type (edges bearing), face side of an edge-on-face contact, nominal area,
// pressure and utilisation from both sides' terms, the crossing angle's sine and |Fn|
template <class R>
struct ClassOut { int ctype, faceSide; R area, pres, util; };
template <class R>
__device__ __forceinline__ ClassOut<R> classCore(int e0, int e1, R cf0, R cf1, R z0, R z1, R ph0, R ph1, R sinT, R fn,
                                                 R fc0, R fc1, R E0, R E1, R H0, R H1) {
  ClassOut<R> o;
  const int nEdge = e0 + e1;
  o.ctype = nEdge;
  o.faceSide = nEdge == 1 ? (e1 ? 0 : 1) : -1;
  R Aa = cf0 * cf1 / sinT, pres = fn / mmax(Aa, R(1e-12));
  R ut = pres / mmax(mmin(H0, H1), R(1e-12));
  if (nEdge == 1) {
    const bool f1 = e1 == 0;          // face side 1 (side 0 bears the edge)
    const R cfF = f1 ? cf1 : cf0, cfE = f1 ? cf0 : cf1, zF = f1 ? z1 : z0, EF = f1 ? E1 : E0;
    const R phE = f1 ? ph0 : ph1, fcE = f1 ? fc0 : fc1;
    const R ell = cfF / sinT, kap = EF / mmax(zF, R(1e-12));
    const R phiE = mmax(phE, R(1e-4));
    const R b = msqrt(R(2) * fn / mmax(ell * kap * phiE, R(1e-12)));
    const bool full = b >= cfE;
    const R Afe = full ? cf0 * cf1 / sinT : b * ell;
    const R pfe = full ? fn / mmax(Afe, R(1e-12)) : kap * phiE * b;
    Aa = Afe; pres = pfe; ut = pfe / mmax(fcE, R(1e-12));
  } else if (nEdge == 2) {
    const R fc = mmin(fc0, fc1);
    Aa = fn / mmax(fc, R(1e-12)); pres = fn > R(0) ? fc : R(0); ut = fn > R(0) ? R(1) : R(0);
  }
  o.area = Aa; o.pres = pres; o.util = ut;
  return o;
}
// W3: n × t of the cutting side, normalised: the direction across that side's seat (solver_cpu.js:302-303, 320-321)
template <class R>
__device__ __forceinline__ void wallAxis(const R n[3], const R t[3], R m[3]) {
  cross3(n, t, m);
  const R ml = mmax(msqrt(dot3(m, m)), R(1e-12));
  m[0] /= ml; m[1] /= ml; m[2] /= ml;
}
// W3: slope tan ψ of the seat wall that sliding along m climbs, from the cutting side's section axes X, Y with sign sg
// (_walls, solver_cpu.js:284-292)
template <class R>
__device__ __forceinline__ R wallSlope(R sg, const R X[3], const R Y[3], const R n[3], const R m[3]) {
  const R nx = (n[0] * X[0] + n[1] * X[1] + n[2] * X[2]) * sg, ny = (n[0] * Y[0] + n[1] * Y[1] + n[2] * Y[2]) * sg;
  const R sx = msign(nx), sy = msign(ny);
  const R fx[3] = {sx * X[0], sx * X[1], sx * X[2]}, fy[3] = {sy * Y[0], sy * Y[1], sy * Y[2]};
  const bool useX = (fx[0] * m[0] + fx[1] * m[1] + fx[2] * m[2]) > R(0);
  R f[3];
  for (int k = 0; k < 3; k++) f[k] = useX ? fx[k] : fy[k];
  const R cosPsi = mmin(mmax(mabs(f[0] * n[0] + f[1] * n[1] + f[2] * n[2]), R(1e-6)), R(1));
  return mtan(macos(cosPsi));
}
// augmented Lagrangian: crossing c's multiplier after the Uzawa step on its window-mean penetration, with the
// safeguards (alValue / updateMultipliers, solver_cpu.js:483-506): none on a disabled crossing or on one whose contact
// point sits on supported nodes (free weight of either side under AL_FREE_MIN, from the current slide coordinates),
// and |λ| at most the crushing capacity min fc90 · wA wB / sin θ with θ of the last evaluation.  `iter` is the
// iteration about to run: the update belongs to the end of the one before, at that iteration's ramp.
template <int P>
__device__ __forceinline__ typename Dev<P>::A alUpdated(const Dev<P> &d, const InstDesc &I, int c, int iter, int penN,
                                                        typename Dev<P>::A lam, typename Dev<P>::A pacc, uint8_t fl) {
  using A = typename Dev<P>::A; using U = typename Dev<P>::U;
  const bool enabled = fl & 1, locked = fl & 2;
  bool pinned = false;
  for (int side = 0; side < 2; side++) {
    const int o = side * d.ktot + c;
    const U uu = d.u[side * d.kS + c];
    const int nseg = ro(d.cxNseg + o);
    const int li = int(mmin(mmax(mfloor(uu), U(0)), U(mmax(nseg - 1, 0))));
    const double t = double(mmin(mmax(uu - U(li), U(0)), U(1)));
    const int sg = ro(d.cxSegOff + o) + li;
    const int a = ro(d.segI0 + sg), b = ro(d.segI1 + sg);
    const bool fa = (ro(d.nflag + a) & 7) == 0, fb = (ro(d.nflag + b) & 7) == 0;
    const double w = (fa ? 0.0 : (1 - t) * (1 - t)) + (fb ? 0.0 : t * t);
    pinned = pinned || w < AL_FREE_MIN;
  }
  if (!enabled || pinned) return A(0);
  const double cap = fmin(double(d.fc90[c]), double(d.fc90[d.ktot + c])) * double(d.wk[c]) * double(d.wk[d.ktot + c]) /
                     fmax(sin(asin(double(d.sinT[c]))), 1e-6);
  const double rampPrev = I.ramp_iter <= 0 ? 1.0 : fmin(1.0, 0.01 + 0.99 * double(iter - 1) / I.ramp_iter);
  const double kn = rampPrev * I.strength;
  double v = double(lam) + kn * (double(pacc) / double(max(penN, 1)));
  if (!locked) v = fmax(v, 0.0);
  return A(fmin(fmax(v, -cap), cap));
}

// crossing c: one evaluation of PolylineContact.apply (solver_cpu.js:381-478) by two adjacent lanes of a warp, one a
// side.  Each lane evaluates its side
// (Hermite point and tangent with node tangents and frames from the neighbours, the nlerp frame); the lanes swap those
// results with pair shuffles and both run the contact law on the same values (the same instructions on the same inputs,
// so the same results).  Each lane writes its side's records and key; the side-0 lane writes the crossing's own
// outputs and adds to the reductions.  Side records go to the side's strand position (general order) or, with SHORT,
// straight to its position in this iteration's sorted order, so the gathers read them without an indirection.
// kb: the buffer that receives the keys after the slide (the next sorted order's); ob: this iteration's sorted order.
// The contact extensions run when the instance has them: the augmented-Lagrangian gap (with the multiplier update that
// fell due at the end of the last iteration, alPend, over a window of penN iterations), the W3 seat law and the W2
// rotational friction, which both classify the contact (W1) within the iteration.
template <int P, bool SHORT, bool EXT>
__device__ __forceinline__ void crossing(const Dev<P> &d, const InstDesc &I, int buf, int iter, int kb, int ob, int c, int side,
                                         int alPend, int penN, Part<typename Dev<P>::A> &pt) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A; using U = typename Dev<P>::U;
  const int kt_ = d.ktot, ks = d.kS, K2 = d.sS;
  const unsigned pair = 3u << ((threadIdx.x & 31) & 30);
  // everything the crossing reads, before anything it writes
  const int pos = ro(d.sPos + 2 * c + side);
  const int rec = SHORT ? d.sInv[size_t(ob) * d.kB + pos] : pos;
  const R np[3] = {d.nPrev[c], d.nPrev[ks + c], d.nPrev[2 * ks + c]};
  const uint8_t fl = ro(d.cflag + c);
  const R muc = ro(d.mu + c), wkA = ro(d.wk + c), hkA = ro(d.hk + c), wkB = ro(d.wk + kt_ + c), hkB = ro(d.hk + kt_ + c);
  const R hc = ro(d.ch + c), wc = ro(d.cw + c);
  const A slip0 = d.slip[c];
  // contact-extension state (this lane's side for the per-side arrays)
  R dentMe = R(0), dentO = R(0), climbMe = R(0), tanpsiMe = R(1), dentE0 = R(0), th0 = R(0);
  A lamc = A(0), pacc = A(0), rslip = A(0);
  if constexpr (EXT) {
    if (EXT && I.seat) {
      dentMe = d.dent[2 * c + side]; dentO = d.dent[2 * c + 1 - side]; climbMe = d.climb[2 * c + side];
      tanpsiMe = d.tanpsi[2 * c + side]; dentE0 = d.dentE[c];
    }
    if (EXT && I.aug) { lamc = d.lam[c]; pacc = d.penAcc[c]; }
    if (EXT && I.rotFric) { th0 = d.theta0[c]; rslip = d.rotSlip[c]; }
  }
  const double rampN = I.ramp_iter;
  const double rampd = rampN <= 0 ? 1.0 : fmin(1.0, 0.01 + 0.99 * double(iter) / rampN);
  const R kn = R(rampd * I.strength), kt = R(rampd * I.stick);
  // this lane's side
  const int o = side * kt_ + c;
  U uu = d.u[side * ks + c];
  const int nseg = ro(d.cxNseg + o);
  R Pm[3], Tm[3], Xm[3], Ym[3], Lm, tpm;
  W xm[3];                              // base node of the side's segment, for the gap in the wide type
  {
    const int li = int(mmin(mmax(mfloor(uu), U(0)), U(mmax(nseg - 1, 0))));
    const R t = R(mmin(mmax(uu - U(li), U(0)), U(1)));
    const int sg = ro(d.cxSegOff + o) + li;
    // the segment's nodes a → b, the segment ending at a (sIn, from aPrev) and the one starting at b (sOut, to bNext):
    // by arithmetic on a linear strand, else gathered (the same indices either way)
    int a, b, sIn, sOut, aPrev, bNext;
    if (I.cxLin) {
      a = ro(d.cxNodeOff + o) + li; b = a + 1;
      sIn = li > 0 ? sg - 1 : -1; sOut = li < nseg - 1 ? sg + 1 : -1;
      aPrev = a - 1; bNext = b + 1;
    } else {
      a = ro(d.segI0 + sg); b = ro(d.segI1 + sg);
      sIn = ro(d.nsIn + a); sOut = ro(d.nsOut + b);
      aPrev = sIn >= 0 ? ro(d.segI0 + sIn) : -1; bNext = sOut >= 0 ? ro(d.segI1 + sOut) : -1;
    }
    for (int k = 0; k < 3; k++) xm[k] = Acc<P>::xw(d, buf, k, a);
    R e[3], Ta[3], Tb[3];
    Acc<P>::edge(d, buf, a, b, e);
    const R Ls = msqrt(dot3(e, e));
    chordTangent<P>(d, buf, a, b, sIn >= 0 ? aPrev : -1, a, Ta);
    chordTangent<P>(d, buf, sOut >= 0 ? b : -1, bNext, a, b, Tb);
    const R t2 = t * t, t3 = t2 * t;
    const R h10 = t3 - R(2) * t2 + t, h01 = R(-2) * t3 + R(3) * t2, h11 = t3 - t2;
    const R d10 = R(3) * t2 - R(4) * t + R(1), d01 = R(-6) * t2 + R(6) * t, d11 = R(3) * t2 - R(2) * t;
    for (int k = 0; k < 3; k++) {
      Pm[k] = h01 * e[k] + (h10 * Ls) * Ta[k] + (h11 * Ls) * Tb[k];
      Tm[k] = d01 * e[k] + (d10 * Ls) * Ta[k] + (d11 * Ls) * Tb[k];
    }
    const R tl = mmax(msqrt(dot3(Tm, Tm)), R(1e-12));
    for (int k = 0; k < 3; k++) Tm[k] /= tl;
    R qa[4], qb[4], q[4], Rn[9];
    segsQuat<P>(d, buf, sg, sIn, qa);
    segsQuat<P>(d, buf, sOut, sg, qb);
    const R sgn = (qa[0] * qb[0] + qa[1] * qb[1] + qa[2] * qb[2] + qa[3] * qb[3]) < R(0) ? R(-1) : R(1);
    for (int k = 0; k < 4; k++) q[k] = (R(1) - t) * qa[k] + t * sgn * qb[k];
    qnormalize(q);
    qframe(q, Rn);
    R y[3] = {Rn[3], Rn[4], Rn[5]};
    const R yt = dot3(y, Tm);
    for (int k = 0; k < 3; k++) y[k] -= yt * Tm[k];
    const R yl = mmax(msqrt(dot3(y, y)), R(1e-12));
    for (int k = 0; k < 3; k++) y[k] /= yl;
    cross3(y, Tm, Xm);
    for (int k = 0; k < 3; k++) Ym[k] = y[k];
    Lm = Ls; tpm = t;
  }
  // the partner's side, and both sides in order (selects, so every array index stays a constant)
  R Pl[2][3], tg[2][3], Rf[2][9], L[2];
  W xa[2][3];
  const bool s1 = side != 0;
  for (int k = 0; k < 3; k++) {
    const R po = __shfl_xor_sync(pair, Pm[k], 1), to = __shfl_xor_sync(pair, Tm[k], 1);
    const R xo = __shfl_xor_sync(pair, Xm[k], 1), yo = __shfl_xor_sync(pair, Ym[k], 1);
    const W wo = __shfl_xor_sync(pair, xm[k], 1);
    Pl[0][k] = s1 ? po : Pm[k]; Pl[1][k] = s1 ? Pm[k] : po;
    tg[0][k] = s1 ? to : Tm[k]; tg[1][k] = s1 ? Tm[k] : to;
    xa[0][k] = s1 ? wo : xm[k]; xa[1][k] = s1 ? xm[k] : wo;
    Rf[0][k] = s1 ? xo : Xm[k]; Rf[1][k] = s1 ? Xm[k] : xo;
    Rf[0][3 + k] = s1 ? yo : Ym[k]; Rf[1][3 + k] = s1 ? Ym[k] : yo;
    Rf[0][6 + k] = tg[0][k]; Rf[1][6 + k] = tg[1][k];
  }
  {
    const R lo = __shfl_xor_sync(pair, Lm, 1);
    L[0] = s1 ? lo : Lm; L[1] = s1 ? Lm : lo;
  }
  const R *tA = tg[0], *tB = tg[1];
  // contact normal with side persistence (solver_cpu.js:396-402)
  R nv[3];
  cross3(tA, tB, nv);
  const R crw[3] = {nv[0], nv[1], nv[2]};    // tA × tB before normalisation (W2 angle)
  const R nn = msqrt(dot3(nv, nv));
  if (nn < R(1e-6)) { nv[0] = np[0]; nv[1] = np[1]; nv[2] = np[2]; }
  else { const R dn = mmax(nn, R(1e-12)); nv[0] /= dn; nv[1] /= dn; nv[2] /= dn; }
  if (dot3(nv, np) < R(0)) { nv[0] = -nv[0]; nv[1] = -nv[1]; nv[2] = -nv[2]; }
  // gap vector P_B − P_A: the base-node difference in the wide type
  R S[3];
  for (int k = 0; k < 3; k++) S[k] = R(xa[1][k] - xa[0][k]) + (Pl[1][k] - Pl[0][k]);
  const R g = dot3(S, nv);
  R rA[3], rB[3];
  const R hA = support(Rf[0], nv, R(1), wkA, hkA, rA);
  const R hB = support(Rf[1], nv, R(-1), wkB, hkB, rB);
  R D = hA + hB;
  if (EXT && I.seat && I.seatGap) D -= (s1 ? dentO + dentMe : dentMe + dentO) + dentE0;     // W3 (solver_cpu.js:410)
  const R pen = D - g;
  const bool enabled = fl & 1, locked = fl & 2;
  bool active;
  R Fn;
  if (EXT && I.aug) {
    // the Uzawa step that fell due after the last iteration, then the penetration window (solver_cpu.js:412-418)
    if (alPend) { lamc = alUpdated<P>(d, I, c, iter, penN, lamc, pacc, fl); pacc = A(0); }
    if (iter >= I.ramp_iter) pacc += A(pen);
    const R trial = R(lamc) + kn * pen;
    active = (trial > R(0) || locked) && enabled;
    Fn = active ? (locked ? trial : mmax(trial, R(0))) : R(0);
  } else {
    active = (pen > R(0) || locked) && enabled;
    Fn = active ? kn * pen : R(0);
  }
  // tangential spring / stick-slip: S_t = a tA + b tB
  const R St[3] = {S[0] - g * nv[0], S[1] - g * nv[1], S[2] - g * nv[2]};
  const R taa = dot3(tA, tA), tbb = dot3(tB, tB), tab = dot3(tA, tB);
  const R sa = dot3(St, tA), sb = dot3(St, tB);
  const R det = taa * tbb - tab * tab;
  const bool ok = det > R(1e-8);
  const R ca = ok ? (sa * tbb - sb * tab) / det : R(0), cb = ok ? (sb * taa - sa * tab) / det : R(0);
  const R Ftv = msqrt((kt * St[0]) * (kt * St[0]) + (kt * St[1]) * (kt * St[1]) + (kt * St[2]) * (kt * St[2]));
  // W3: the seats' walls raise the friction against the slide direction (_seatFriction, solver_cpu.js:294-313); this
  // lane takes the term of its own side's seat, cut by the other side
  R muDir = muc;
  R wm[3] = {R(0), R(0), R(0)};       // wall axis of this side's seat: n × the other side's tangent, normalised
  if (EXT && I.seat) {
    R tc[3], Xo[3], Yo[3];
    for (int k = 0; k < 3; k++) { tc[k] = s1 ? tg[0][k] : tg[1][k]; Xo[k] = s1 ? Rf[0][k] : Rf[1][k]; Yo[k] = s1 ? Rf[0][3 + k] : Rf[1][3 + k]; }
    wallAxis(nv, tc, wm);
    const R nrm = msqrt(dot3(St, St));
    R addMe = R(0);
    if (dentMe > R(0) && nrm > R(1e-12)) {
      const R dn = mmax(nrm, R(1e-12)), sgn = s1 ? R(-1) : R(1);
      const R dhat[3] = {St[0] / dn, St[1] / dn, St[2] / dn};
      const R dj = dot3(dhat, wm) * sgn;
      const R wd[3] = {msign(dj) * wm[0] * sgn, msign(dj) * wm[1] * sgn, msign(dj) * wm[2] * sgn};
      tanpsiMe = wallSlope(s1 ? R(1) : R(-1), Xo, Yo, nv, wd);
      const R add = mabs(dj) * (muc * tanpsiMe < R(1) ? (muc + tanpsiMe) / mmax(R(1) - muc * tanpsiMe, R(1e-6)) - muc : R(9) * muc);
      addMe = mmin(add, R(9) * muc);
    }
    const R addO = __shfl_xor_sync(pair, addMe, 1);
    muDir = (muc + (s1 ? addO : addMe)) + (s1 ? addMe : addO);
  }
  const R limit = muDir * mabs(Fn);
  const bool slip = active && ok && !locked && Ftv > limit;
  const bool freeS = !active && ok && enabled;
  R scale = R(0);
  if (slip) scale = R(mclamp(I.slip_rate, 1e-3, 1.0)) * (R(1) - limit / mmax(Ftv, R(1e-12)));
  if (freeS) scale = R(1);
  const R eps = R(fmax(I.eps, 1e-9));
  const R da = mclamp(ca * scale, -eps, eps), db = mclamp(cb * scale, -eps, eps);
  const bool moved = slip || freeS;
  if (moved) uu += side ? -U(db) / U(mmax(L[1], R(1e-12))) : U(da) / U(mmax(L[0], R(1e-12)));
  const U un = mclamp(uu, U(0), U(nseg));
  A slipNew = slip0;
  if (slip) {
    const R sx = da * tA[0] + db * tB[0], sy = da * tA[1] + db * tB[1], sz = da * tA[2] + db * tB[2];
    slipNew += A(msqrt(sx * sx + sy * sy + sz * sz));
  }
  R Se[3] = {R(0), R(0), R(0)};
  if (active) for (int k = 0; k < 3; k++) Se[k] = St[k] - da * tA[k] - db * tB[k];
  const R fT[3] = {kt * Se[0], kt * Se[1], kt * Se[2]};
  R FA[3];
  for (int k = 0; k < 3; k++) FA[k] = -Fn * nv[k] + fT[k];
  const R sgS = side ? R(-1) : R(1);
  const R nxMe = dot3(nv, Xm) * sgS, nyMe = dot3(nv, Ym) * sgS;    // the normal in this side's section frame
  const R sinTc = mmin(mmax(nn, R(1e-6)), R(1));
  R Mrot = R(0), eRot = R(0);
  if (EXT && (I.seat || I.rotFric)) {
    // W1 within the iteration (solver_cpu.js:460): each lane its side's terms, swapped, both lanes the crossing's
    int eMe;
    R cfMe, zMe, phMe;
    sideClass(nxMe, nyMe, side ? wkB : wkA, side ? hkB : hkA, I.edgeThr, eMe, cfMe, zMe, phMe);
    const int eO = __shfl_xor_sync(pair, eMe, 1);
    const R cfO = __shfl_xor_sync(pair, cfMe, 1), zO = __shfl_xor_sync(pair, zMe, 1), phO = __shfl_xor_sync(pair, phMe, 1);
    const int e0 = s1 ? eO : eMe, e1 = s1 ? eMe : eO;
    const R cf0 = s1 ? cfO : cfMe, cf1 = s1 ? cfMe : cfO, z0 = s1 ? zO : zMe, z1 = s1 ? zMe : zO;
    const R ph0 = s1 ? phO : phMe, ph1 = s1 ? phMe : phO;
    const R fc0 = ro(d.fc90 + c), fc1 = ro(d.fc90 + kt_ + c);
    const ClassOut<R> co = classCore(e0, e1, cf0, cf1, z0, z1, ph0, ph1, sinTc, mabs(Fn), fc0, fc1, ro(d.E90 + c),
                                     ro(d.E90 + kt_ + c), ro(d.Hs + c), ro(d.Hs + kt_ + c));
    const R thetaC = masin(sinTc);
    if (EXT && I.seat) {
      // W3: climbing out of this side's seat, seat growth under an edge (_seatUpdate, solver_cpu.js:315-344)
      R inc[3];
      for (int k = 0; k < 3; k++) inc[k] = da * tA[k] - db * tB[k];
      const R step = dot3(inc, wm) * sgS;
      R dn = dentMe, cl = climbMe, dE = dentE0;
      const bool has = dn > R(0);
      if (has && slip) cl += step;
      if (has && mabs(cl) >= dn / mmax(tanpsiMe, R(1e-6))) { dn = R(0); cl = R(0); }
      if (iter >= I.dentAfter) {
        const R sinp0 = msin(ph0) * mcos(ph0), sinp1 = msin(ph1) * mcos(ph1);
        const R sT = msin(thetaC);
        if (co.ctype == 2 && active && !locked) {
          const R fc = mmin(fc0, fc1);
          const R dEst = msqrt(mabs(Fn) / mmax(fc, R(1e-12)) * sT * sinp0 * sinp1);
          dn = mmax(dn, mmin(dn + R(I.dentRate) * dEst, dEst));
        }
        if (co.ctype == 1 && active && !locked) {
          const bool f1 = co.faceSide == 1;
          const R ell = (f1 ? cf1 : cf0) / mmax(sT, R(1e-6));
          dE = mmax(dE, mabs(Fn) / mmax((f1 ? fc0 : fc1) * ell, R(1e-12)) * (f1 ? sinp0 : sinp1));
        }
      }
      d.dent[2 * c + side] = dn; d.climb[2 * c + side] = cl; d.tanpsi[2 * c + side] = tanpsiMe;
      if (side == 0) d.dentE[c] = dE;
    }
    if (EXT && I.rotFric) {
      // W2: the scissor moment about n with Coulomb's limit on it (_rotationalFriction, solver_cpu.js:347-379)
      const R th = matan2(dot3(crw, nv), dot3(tA, tB));
      if (isnan(th0) && active) th0 = th;
      const bool ok = active && !isnan(th0);
      const R sTc = mmax(msin(thetaC), R(1e-6));
      R req = R(0.38) * msqrt(wkA * wkB / sTc);
      if (co.ctype == 1) req = R(0.25) * (co.faceSide == 0 ? wkA : wkB) / sTc;
      else if (co.ctype == 2) req = R(0.38) * msqrt(mmax(co.area, R(1e-12)));
      const R kr = kt * req * req;
      const R PI = R(PI_D);
      R dth = ok ? th - th0 : R(0);
      dth = mfmod(mfmod(dth + PI, R(2) * PI) + R(2) * PI, R(2) * PI) - PI;
      R Mc = kr * dth;
      if (ok && !locked) {
        const R Mlim = R(I.rotFactor) * muc * mabs(Fn) * req;
        if (mabs(Mc) > Mlim) {
          const R rate = R(mclamp(I.slip_rate, 1e-3, 1.0));
          R adv = rate * (R(1) - Mlim / mmax(mabs(Mc), R(1e-12))) * dth;
          adv = mclamp(adv, R(-0.05), R(0.05));
          th0 += adv; rslip += A(mabs(adv)); dth -= adv;
          Mc = kr * dth;
        }
      }
      Mrot = ok ? Mc : R(0);
      eRot = kr * dth * dth;
      if (side == 0) { d.theta0[c] = th0; d.rotSlip[c] = rslip; d.Mrot[c] = Mrot; }
    }
  }
  // side records for the gathers: t before the slide, force on the side, lever torque tf (r × F); the righting
  // stiffness of the support point (addTwistStiffness, solver_cpu.js:170-176) goes to the segments the sides sit on
  // after the slide
  const R tf = R(I.tf);
  const R tfc = R(fmax(I.tf, 1e-3));
  const R kth = tfc * ((Fn + kn * R(0.25) * hc) * (R(0.5) * wc) / R(SUPPORT_SMOOTH) + kt * (R(0.5) * hc) * (R(0.5) * hc));
  // stores: the crossing's own outputs from the side-0 lane, each side's slide coordinate, key and records from its lane
  if (side == 0) {
    for (int k = 0; k < 3; k++) d.nPrev[k * ks + c] = nv[k];
    d.slip[c] = slipNew;
    d.stuck[c] = moved ? 0 : 1;
    d.Fn[c] = Fn;
    d.Ft[c] = msqrt(dot3(fT, fT));
    d.cstate[c] = slip ? 1 : 0;
    d.gap[c] = g;
    // penalty energy (k_n pen², or Fn²/k_n with the multiplier) and the W2 spring's k_r Δθ² (solver_cpu.js:469,378)
    pt.s[RS_PEN] += A(active ? (EXT && I.aug ? Fn * Fn / mmax(kn, R(PrecT<P>::TINY)) : kn * pen * pen) : R(0)) + A(eRot);
    if (EXT && I.aug) { d.lam[c] = lamc; d.penAcc[c] = pacc; }
    pt.s[RS_TAN] += A(dot3(Se, Se));
    pt.x[RX_FN] = mmax(pt.x[RX_FN], A(Fn));
  }
  d.u[side * ks + c] = un;
  {
    // what the W1 classification needs of this evaluation: the normal in the side's section frame, the crossing angle
    d.sProj[2 * c + side] = nxMe;
    d.sProj[2 * size_t(kt_) + 2 * c + side] = nyMe;
    if (side == 0) d.sinT[c] = sinTc;
  }
  // the side's segment after the slide (solver_cpu.js:144-149): the key of the next sort, into key buffer kb
  const int key = int(mmin(mmax(mfloor(un), U(0)), U(mmax(nseg - 1, 0))));
  d.sKey[size_t(kb) * d.kB + pos] = key;
  if constexpr (SHORT) { d.sKeyS[rec] = key; d.sSideAt[rec] = pos; }
  {
    const R sgn = side ? R(-1) : R(1);
    const R F[3] = {sgn * FA[0], sgn * FA[1], sgn * FA[2]};
    R tq[3];
    cross3(side ? rB : rA, F, tq);
    d.sT[rec] = tpm;
    d.kth[rec] = kth;
    // lever torque, and the W2 moment about n: +M on side A's segment, −M on side B's
    const R Ms = sgn * Mrot;
    for (int k = 0; k < 3; k++) { d.sF[k * K2 + rec] = F[k]; d.sTq[k * K2 + rec] = tf * tq[k] + Ms * nv[k]; }
  }
}

// W1: the contact type of crossing c from the roll of each section against the contact plane, from the normal in each
// side's section frame, the crossing angle and the normal force of its last evaluation (PolylineContact._classify,
// solver_cpu.js:231-271; outputs only, nothing of the iteration reads them)
template <int P>
__device__ __forceinline__ void classify(const Dev<P> &d, const InstDesc &I, int c) {
  using R = typename Dev<P>::R;
  const int kt_ = d.ktot, K2 = 2 * kt_;
  int e0, e1;
  R cf0, cf1, z0, z1, ph0, ph1;
  sideClass(d.sProj[2 * c], d.sProj[K2 + 2 * c], d.wk[c], d.hk[c], I.edgeThr, e0, cf0, z0, ph0);
  sideClass(d.sProj[2 * c + 1], d.sProj[K2 + 2 * c + 1], d.wk[kt_ + c], d.hk[kt_ + c], I.edgeThr, e1, cf1, z1, ph1);
  const R sinT = d.sinT[c];
  const ClassOut<R> o = classCore(e0, e1, cf0, cf1, z0, z1, ph0, ph1, sinT, mabs(d.Fn[c]), d.fc90[c], d.fc90[kt_ + c],
                                  d.E90[c], d.E90[kt_ + c], d.Hs[c], d.Hs[kt_ + c]);
  d.phiS[2 * c] = ph0; d.phiS[2 * c + 1] = ph1;
  d.ctype[c] = uint8_t(o.ctype);
  d.theta[c] = masin(sinT);
  d.area[c] = o.area; d.pres[c] = o.pres; d.util[c] = o.util;
}

// ------------------------------------------------------------------------------------------------ phase B / C
// The order of the crossing sides along each strand, sorted by (local segment, side), built by rank: the side at
// position p counts the sides of its strand that sort before it (no serial sort, no atomics).  Keys are read by
// position, so a strand's keys are one contiguous run every thread of the strand reads alike.
struct SideRank { int pos, below, equal; };
__device__ __forceinline__ SideRank sideRank(const int *key, int p, int off, int cnt) {
  const int k = key[p];
  int below = 0, equal = 0, before = 0;
  for (int q = off; q < off + cnt; q++) {
    const int kq = key[q];
    below += kq < k ? 1 : 0;
    equal += kq == k ? 1 : 0;
    before += (kq == k && q < p) ? 1 : 0;
  }
  return SideRank{off + below + before, below, equal};
}
// general order (any slide length): side p takes its place in sorted-side buffer dst by the keys of buffer kb (after
// this iteration's slide); every segment's slice is then counted by segCount
template <int P>
__device__ __forceinline__ void rankSide(const Dev<P> &d, int p, int kb, int dst) {
  const int s = d.sStrand[p];
  const int *key = d.sKey + size_t(kb) * d.kB;
  const SideRank r = sideRank(key, p, d.stSideOff[s], d.stSideCnt[s]);
  d.ord[size_t(dst) * d.oB + r.pos] = p;
  d.ordSeg[size_t(dst) * d.oB + r.pos] = key[p];
}
// segment j: its slice of the new order = [off + #keys below, off + #keys below + #keys equal) among its strand's sides
template <int P>
__device__ __forceinline__ void segCount(const Dev<P> &d, int j, int kb, int dst) {
  const int *key = d.sKey + size_t(kb) * d.kB;
  const int s = d.segStrand[j], lj = d.segLocal[j];
  const int off = d.stSideOff[s], cnt = d.stSideCnt[s];
  int lo = 0, eq = 0;
  for (int q = off; q < off + cnt; q++) {
    const int kq = key[q];
    lo += kq < lj ? 1 : 0;
    eq += kq == lj ? 1 : 0;
  }
  d.rngLo[size_t(dst) * d.rB + j] = off + lo;
  d.rngHi[size_t(dst) * d.rB + j] = off + lo + eq;
}
// short-slide order (the slide limit is under half the shortest segment, so a side moves at most one segment per
// iteration): built in the update phase from the keys this iteration's slide produced, into buffer kb, the order the
// next iteration's crossings write their side records into and its gathers read.  Side p's sorted position goes to
// sInv, its key to ordSeg; the first side of each segment writes that segment's slice.  A segment without sides
// keeps a slice of an earlier iteration, whose entries carry other keys, and the gathers skip entries whose key is
// not the segment's.
template <int P>
__device__ __forceinline__ void rankSideShort(const Dev<P> &d, int p, int kb) {
  const int s = d.sStrand[p], off = d.stSideOff[s];
  const int *key = d.sKey + size_t(kb) * d.kB;
  const SideRank r = sideRank(key, p, off, d.stSideCnt[s]);
  const int k = key[p];
  d.sInv[size_t(kb) * d.kB + p] = r.pos;
  d.ordSeg[size_t(kb) * d.oB + r.pos] = k;
  if (r.pos == off + r.below) {
    const int j = d.stSegOff[s] + k;
    d.rngLo[size_t(kb) * d.rB + j] = off + r.below;
    d.rngHi[size_t(kb) * d.rB + j] = off + r.below + r.equal;
  }
}

// The same order, built each iteration from the previous one (buffer ob) instead of by counting every side of the
// strand: a side moves at most one segment an iteration, so every side whose previous key is at most k − 2 (k: side
// p's key after this iteration's slide) sorts before p, and every side whose previous key is at least k + 2 after it.
// The others sit next to p's previous sorted position and are the only ones compared, by their new keys and strand
// positions, which this iteration's crossings wrote at their previous sorted positions (sKeyS, sSideAt).  The result
// is the full count's (sideRank's) position, slice and key, from a few neighbours instead of the whole strand.
template <int P>
__device__ __forceinline__ void rankSideWindow(const Dev<P> &d, int p, int ob, int kb) {
  const int s = d.sStrand[p], off = d.stSideOff[s], end = off + d.stSideCnt[s];
  const int k = d.sKey[size_t(kb) * d.kB + p];
  const int sp = d.sInv[size_t(ob) * d.kB + p];
  const int *prevKey = d.ordSeg + size_t(ob) * d.oB;
  int below = 0, equal = 1, before = 0;           // p itself counts among the equal keys
  auto visit = [&](int q) {
    const int kq = d.sKeyS[q], pq = d.sSideAt[q];
    below += kq < k ? 1 : 0;
    equal += kq == k ? 1 : 0;
    before += (kq == k && pq < p) ? 1 : 0;
  };
  int lo = sp;
  while (lo > off && prevKey[lo - 1] >= k - 1) visit(--lo);
  for (int q = sp + 1; q < end && prevKey[q] <= k + 1; q++) visit(q);
  below += lo - off;
  const int pos = off + below + before;
  d.sInv[size_t(kb) * d.kB + p] = pos;
  d.ordSeg[size_t(kb) * d.oB + pos] = k;
  if (before == 0) {
    const int j = d.stSegOff[s] + k;
    d.rngLo[size_t(kb) * d.rB + j] = off + below;
    d.rngHi[size_t(kb) * d.rB + j] = off + below + equal;
  }
}

// ------------------------------------------------------------------------------------------------ phase D
struct StepCtx {
  int cur, nxt, obuf, onxt, pending, iter, warm;
  int alPend, penN;  // augmented Lagrangian: the multiplier update is due before this iteration's evaluation
  const double *utmPf;  // load protocol: the force on the probe (mode 1)
  double dispR;      // prescribed-motion fraction of this iteration
};

// a key no side carries (an empty slice's placeholder)
constexpr int NO_KEY = -0x40000000;

// the side records in the slice of segment j (strand-local index lj) of sorted-side buffer ob, in sorted order: with
// SHORT the records sit at the sorted positions, and an entry counts only if it carries the segment's key (a slice left
// over from an earlier iteration carries other keys); in the general order the entries name the records' positions
template <bool SHORT, int P, class F>
__device__ __forceinline__ void sidesOn(const Dev<P> &d, int ob, int j, int lj, F &&f) {
  const int lo = d.rngLo[size_t(ob) * d.rB + j], hi = d.rngHi[size_t(ob) * d.rB + j];
  for (int e = lo; e < hi; e++) {
    if constexpr (SHORT) {
      if (d.ordSeg[size_t(ob) * d.oB + e] == lj) f(e);
    } else {
      f(d.ord[size_t(ob) * d.oB + e]);
    }
  }
}

// Both updates read everything first and store at the end, so no store stands between a load and the loads after it
// (the compiler must assume they alias) and the loads of one element go out together.

// the ground on node i (Floor.apply, solver_cpu.js:572-620): a penalty under the lowest point of the section in the
// node's frame, a stick point on the plane dragged after the node by Coulomb's return mapping; adds to F.
template <int P>
__device__ __forceinline__ void floorForce(const Dev<P> &d, const InstDesc &I, const StepCtx &sc, int i,
                                        const typename Dev<P>::W x[3], typename Dev<P>::R F[3], Part<typename Dev<P>::A> &pt) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A;
  const int nt = d.ntot;
  const double rampN = I.ramp_iter;
  const double ramp = rampN <= 0 ? 1.0 : fmin(1.0, 0.01 + 0.99 * double(sc.iter) / rampN);
  const R kn = R(ramp * I.strength), kt = R(ramp * I.stick);
  // the gap from the plane and the section's depth below the node cancel (a penetration of ~1e-3 of the depth): both
  // are formed in the wide type, the depth from the node frame of the wide-type segment frames (a frame in float
  // leaves ~1e-7 of the depth, which the mixed policy's ground forces would carry as noise of ~1e-4 of their size)
  W q[4], Rn[9];
  segsQuat<P, true>(d, sc.cur, ro(d.nsOut + i), ro(d.nsIn + i), q);
  qframe(q, Rn);
  const R pen = R((W(I.floorZ) - x[2]) + (W(0.5) * W(ro(d.flW + i)) * mabs(Rn[2]) + W(0.5) * W(ro(d.flH + i)) * mabs(Rn[5])));
  const W ax = d.flAx[i], ay = d.flAy[i];
  R ff[3] = {R(0), R(0), R(0)};
  if (pen > R(0)) {
    const R fn = kn * pen;
    const R sx = R(x[0] - ax), sy = R(x[1] - ay);
    const R Ftv = kt * msqrt(sx * sx + sy * sy), limit = R(fmax(I.floorMu, 0.0)) * fn;
    const R scale = Ftv > limit ? R(1) - limit / mmax(Ftv, R(1e-12)) : R(0);
    const R dax = sx * scale, day = sy * scale;
    if (scale > R(0)) { d.flAx[i] = ax + W(dax); d.flAy[i] = ay + W(day); }
    const R ex = sx - dax, ey = sy - day;
    ff[0] = -kt * ex; ff[1] = -kt * ey; ff[2] = fn;
    d.flState[i] = scale > R(0) ? 2 : 1;
    pt.s[RS_FLOOR] += A(R(0.5) * kn * pen * pen + R(0.5) * kt * (ex * ex + ey * ey));
    pt.x[RX_FN] = mmax(pt.x[RX_FN], A(fn));
  } else {
    d.flAx[i] = x[0]; d.flAy[i] = x[1];
    d.flState[i] = 0;
  }
  for (int k = 0; k < 3; k++) { d.flF[size_t(k) * nt + i] = ff[k]; F[k] += ff[k]; }
}

template <int P, bool SHORT, bool EXT>
__device__ __forceinline__ void nodeUpdate(const Dev<P> &d, const InstDesc &I, const StepCtx &sc, int i, Part<typename Dev<P>::A> &pt) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A;
  const int nt = d.ntot, ns = d.nS, ms = d.mS, K2 = d.sS;
  const int so = ro(d.nsOut + i), si = ro(d.nsIn + i);
  const uint8_t fl = ro(d.nflag + i);
  const R m = ro(d.mass + i);
  R tot[3] = {ro(d.lc + i), ro(d.lc + nt + i), ro(d.lc + 2 * nt + i)};
  const int ai = (fl & 32) ? ro(d.anc + i) : -1;
  W x[3], v0[3] = {W(0), W(0), W(0)};
  for (int k = 0; k < 3; k++) x[k] = Acc<P>::xw(d, sc.cur, k, i);
  if (!(sc.pending || sc.warm)) for (int k = 0; k < 3; k++) v0[k] = W(d.V[k * ns + i]);
  R F[3] = {R(0), R(0), R(0)};
  if (so >= 0) for (int k = 0; k < 3; k++) F[k] += d.nF[k * ms + so];
  if (si >= 0) for (int k = 0; k < 3; k++) F[k] -= d.nF[k * ms + si];
  if (fl & 16) {                          // load in the node frame (solver_cpu.js:755-758)
    R q[4], Rn[9];
    nodeQuat<P>(d, sc.cur, i, q);
    qframe(q, Rn);
    const R f0 = ro(d.ll + i), f1 = ro(d.ll + nt + i), f2 = ro(d.ll + 2 * nt + i);
    for (int k = 0; k < 3; k++) tot[k] += Rn[k] * f0 + Rn[3 + k] * f1 + Rn[6 + k] * f2;
  }
  if constexpr (EXT)
    if (I.utmMode == 1 && i == I.utmProbe)   // the load protocol's force on its probe (wgsl.js:914)
      for (int k = 0; k < 3; k++) tot[k] += R(sc.utmPf[k]);
  for (int k = 0; k < 3; k++) F[k] += tot[k];
  pt.x[RX_LOAD] = mmax(pt.x[RX_LOAD], A(mmax(mabs(tot[0]), mmax(mabs(tot[1]), mabs(tot[2])))));
  // crossing sides on the adjacent segments, as distributed by the last evaluation (weights 1 − t at a, t at b)
  const bool cx = I.contacts && I.K;
  if constexpr (EXT)
    if (I.floorOn) {
      for (int k = 0; k < 3; k++) d.ldTot[k * nt + i] = tot[k];     // the external loads, for the rigid-body sums
      floorForce<P>(d, I, sc, i, x, F, pt);
    }
  if constexpr (SHORT) {
    if (cx) {
      // the slices of both segments (bounds and keys together), then the first entry of each, then any further
      // entries in order: two levels of dependent loads after the segment indices
      const int ob = sc.obuf;
      const int *oseg = d.ordSeg + size_t(ob) * d.oB;
      const int sg[2] = {so, si};
      int lo[2], hi[2], lk[2];
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int jc = sg[t] >= 0 ? sg[t] : I.m0;      // (a segment of this instance: its slice is read, not used)
        lk[t] = ro(d.segLocal + jc);
        lo[t] = d.rngLo[size_t(ob) * d.rB + jc];
        const int h = d.rngHi[size_t(ob) * d.rB + jc];
        hi[t] = sg[t] >= 0 ? h : lo[t];
      }
      int key0[2];
      R t0[2], f0[2][3];
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const bool ok = lo[t] < hi[t];
        const int e = lo[t];
        key0[t] = ok ? oseg[e] : NO_KEY;
        t0[t] = ok ? d.sT[e] : R(0);
#pragma unroll
        for (int k = 0; k < 3; k++) f0[t][k] = ok ? d.sF[k * K2 + e] : R(0);
      }
#pragma unroll
      for (int t = 0; t < 2; t++) {
        // weights 1 − t on the outgoing segment (the node is its start), t on the incoming one
        if (key0[t] == lk[t]) {
          const R wgt = t == 0 ? R(1) - t0[t] : t0[t];
          for (int k = 0; k < 3; k++) F[k] += wgt * f0[t][k];
        }
        for (int e = lo[t] + 1; e < hi[t]; e++)
          if (oseg[e] == lk[t]) {
            const R wgt = t == 0 ? R(1) - d.sT[e] : d.sT[e];
            for (int k = 0; k < 3; k++) F[k] += wgt * d.sF[k * K2 + e];
          }
      }
    }
  } else {
    if (cx && so >= 0)
      sidesOn<SHORT>(d, sc.obuf, so, 0, [&](int q) {
        const R wgt = R(1) - d.sT[q];
        for (int k = 0; k < 3; k++) F[k] += wgt * d.sF[k * K2 + q];
      });
    if (cx && si >= 0)
      sidesOn<SHORT>(d, sc.obuf, si, 0, [&](int q) {
        const R wgt = d.sT[q];
        for (int k = 0; k < 3; k++) F[k] += wgt * d.sF[k * K2 + q];
      });
  }
  const R react[3] = {-F[0], -F[1], -F[2]};
  for (int k = 0; k < 3; k++) if (!(fl & (1 << k))) F[k] = R(0);
  pt.x[RX_F] = mmax(pt.x[RX_F], A(msqrt(dot3(F, F))));
  R v[3];
  for (int k = 0; k < 3; k++) v[k] = R(v0[k]);
  if (!sc.warm) for (int k = 0; k < 3; k++) v[k] += F[k] / m;
  if (I.damping != 1.0) for (int k = 0; k < 3; k++) v[k] *= R(I.damping);
  for (int k = 0; k < 3; k++) if (!(fl & (1 << k))) v[k] = R(0);
  for (int k = 0; k < 3; k++) {
    x[k] += W(v[k]);
    if (ai >= 0 && !(fl & (1 << k))) x[k] = ro(d.ancStart + size_t(k) * nt + ai) + W(sc.dispR) * ro(d.ancDelta + size_t(k) * nt + ai);
  }
  if (fl & 8) for (int k = 0; k < 3; k++) d.react[k * nt + i] = react[k];
  for (int k = 0; k < 3; k++) {
    d.V[k * ns + i] = v[k];
    Acc<P>::xs(d, sc.nxt, k, i, x[k]);
  }
  pt.s[RS_KE] += A(m) * (A(v[0]) * A(v[0]) + A(v[1]) * A(v[1]) + A(v[2]) * A(v[2]));
}

template <int P, bool SHORT>
__device__ __forceinline__ void segUpdate(const Dev<P> &d, const InstDesc &I, const StepCtx &sc, int j, Part<typename Dev<P>::A> &pt) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using A = typename Dev<P>::A;
  const int mt = d.mtot, sm = d.mS, ps = d.pS, cs = d.cS, K2 = d.sS;
  const int ja = ro(d.jA + j), jb = ro(d.jB + j), c0 = ro(d.cl0 + j), c1 = ro(d.cl1 + j);
  const R krs[3] = {ro(d.krs + j), ro(d.krs + mt + j), ro(d.krs + 2 * mt + j)};
  W qw[4];
  for (int k = 0; k < 4; k++) qw[k] = Acc<P>::qw(d, sc.cur, k, j);
  R w0[3] = {R(0), R(0), R(0)};
  if (!sc.pending) for (int k = 0; k < 3; k++) w0[k] = d.Wr[k * sm + j];
  R T[3] = {d.en[j], d.en[sm + j], d.en[2 * sm + j]};
  R kD[3] = {R(0), R(0), R(0)};
  if (ja >= 0) for (int k = 0; k < 3; k++) { T[k] += d.tau[k * ps + ja]; kD[k] += d.kd[k * ps + ja]; }
  if (jb >= 0) for (int k = 0; k < 3; k++) { T[k] -= d.tau[k * ps + jb]; kD[k] += d.kd[k * ps + jb]; }
  if (c0 >= 0) for (int k = 0; k < 3; k++) T[k] -= d.tauC[k * cs + c0];
  if (c1 >= 0) for (int k = 0; k < 3; k++) T[k] -= d.tauC[k * cs + c1];
  R kTw = R(0);
  if (I.contacts && I.K) {
    const int lj = SHORT ? ro(d.segLocal + j) : 0;
    if constexpr (SHORT) {
      // The lever torques of the sides on j (its slice, entries keyed lj) and the twist stiffness of the sides on j
      // after the slide, which before it were on j − 1, j or j + 1 of the same strand (those slices, entries keyed
      // lj − 1, lj, lj + 1 whose key after the slide is lj).  The three slices' bounds load together, then the first
      // entry of each, so the gathers take two levels of dependent loads; further entries follow in order.
      const int ob = sc.obuf;
      const int *oseg = d.ordSeg + size_t(ob) * d.oB;
      const int s = ro(d.segStrand + j);
      int lo[3], hi[3];
#pragma unroll
      for (int t = 0; t < 3; t++) {
        // a neighbour outside the instance is never on j's strand; it is not read either (in the resident form the
        // slice arrays hold this instance's segments only)
        const int jj = j + t - 1;
        const bool inr = jj >= I.m0 && jj < I.m0 + I.m;
        const int jc = inr ? jj : j;
        const bool same = inr && ro(d.segStrand + jc) == s;
        lo[t] = d.rngLo[size_t(ob) * d.rB + jc];
        const int h = d.rngHi[size_t(ob) * d.rB + jc];
        hi[t] = same ? h : lo[t];
      }
      int key0[3], ks0[3];
      R kv0[3], tq0[3];
#pragma unroll
      for (int t = 0; t < 3; t++) {
        const bool ok = lo[t] < hi[t];
        const int e = lo[t];
        key0[t] = ok ? oseg[e] : NO_KEY;
        ks0[t] = ok ? d.sKeyS[e] : NO_KEY;
        kv0[t] = ok ? d.kth[e] : R(0);
      }
#pragma unroll
      for (int k = 0; k < 3; k++) tq0[k] = lo[1] < hi[1] ? d.sTq[k * K2 + lo[1]] : R(0);
      if (key0[1] == lj) for (int k = 0; k < 3; k++) T[k] += tq0[k];
      for (int e = lo[1] + 1; e < hi[1]; e++)
        if (oseg[e] == lj) for (int k = 0; k < 3; k++) T[k] += d.sTq[k * K2 + e];
#pragma unroll
      for (int t = 0; t < 3; t++) {
        const int want = lj + t - 1;
        if (key0[t] == want && ks0[t] == lj) kTw += kv0[t];
        for (int e = lo[t] + 1; e < hi[t]; e++)
          if (oseg[e] == want && d.sKeyS[e] == lj) kTw += d.kth[e];
      }
    } else {
      sidesOn<SHORT>(d, sc.obuf, j, lj, [&](int q) { for (int k = 0; k < 3; k++) T[k] += d.sTq[k * K2 + q]; });
      sidesOn<false>(d, sc.onxt, j, 0, [&](int q) { kTw += d.kth[q]; });
    }
  }
  R q[4], Rm[9];
  for (int k = 0; k < 4; k++) q[k] = R(qw[k]);
  qframe(q, Rm);
  R tm[3];
  for (int k = 0; k < 3; k++) tm[k] = Rm[3 * k] * T[0] + Rm[3 * k + 1] * T[1] + Rm[3 * k + 2] * T[2];
  pt.x[RX_T] = mmax(pt.x[RX_T], A(msqrt(dot3(tm, tm))));
  const R ms = R(I.ms);
  R w[3], I3[3];
  for (int k = 0; k < 3; k++) {
    I3[k] = ms * mmax(krs[k] + kTw + kD[k], R(1e-12));
    w[k] = w0[k] + tm[k] / I3[k];
  }
  w[2] = mclamp(w[2], R(-TWIST_RATE_MAX), R(TWIST_RATE_MAX));
  if (kTw > R(0)) w[2] *= R(ROLL_DAMP);
  if (I.damping != 1.0) for (int k = 0; k < 3; k++) w[k] *= R(I.damping);
  // q ← normalize(q ⊗ exp(ω)) in the wide type; the increment q ⊗ (exp(ω) − 1) is small, formed in R
  const R a = msqrt(dot3(w, w)), half = R(0.5) * a;
  R sh, ch;
  msincos(half, &sh, &ch);
  const R s = a > R(1e-12) ? sh / a : R(0.5);
  W qn[4];
  if constexpr (P != PREC_MIXED) {
    const W dq[4] = {ch, w[0] * s, w[1] * s, w[2] * s};
    qmul(qw, dq, qn);
  } else {
    R sq, cq;
    msincos(R(0.5) * half, &sq, &cq);
    const R dm1[4] = {R(-2) * sq * sq, w[0] * s, w[1] * s, w[2] * s};
    R inc[4];
    qmul(q, dm1, inc);
    for (int k = 0; k < 4; k++) qn[k] = qw[k] + W(inc[k]);
  }
  qnormalize<W, P == PREC_MIXED>(qn);
  for (int k = 0; k < 3; k++) d.Wr[k * sm + j] = w[k];
  for (int k = 0; k < 4; k++) Acc<P>::qs(d, sc.nxt, k, j, qn[k]);
  pt.s[RS_KE] += A(I3[0]) * A(w[0]) * A(w[0]) + A(I3[1]) * A(w[1]) * A(w[1]) + A(I3[2]) * A(w[2]) * A(w[2]);
}

// ------------------------------------------------------------------------------------------------ reductions
// Slot sets: a kernel that feeds only some slots reduces only those (SM: sum slots, XM: max slots, bit i for slot i);
// the others keep their identity values (0, or −∞ for RX_FN), so the result is the same as reducing every slot.
constexpr unsigned SUMS_ALL = (1u << RS_NSUM) - 1, MAXS_ALL = (1u << RX_NMAX) - 1;
constexpr unsigned SUMS_UPDATE = 1u << RS_KE, MAXS_UPDATE = (1u << RX_F) | (1u << RX_T) | (1u << RX_LOAD);
constexpr unsigned SUMS_FLOOR = 1u << RS_FLOOR, MAXS_FLOOR = 1u << RX_FN;     // the ground's, in the node update
constexpr unsigned SUMS_CROSS = (1u << RS_PEN) | (1u << RS_TAN), MAXS_CROSS = 1u << RX_FN;
constexpr unsigned SUMS_ROD = (1u << RS_STRETCH) | (1u << RS_SHEAR) | (1u << RS_BEND) | (1u << RS_TWIST),
                   MAXS_ROD = (1u << RX_N) | (1u << RX_M);

template <unsigned SM = SUMS_ALL, unsigned XM = MAXS_ALL, class A>
__device__ __forceinline__ void warpReduce(Part<A> &p) {
  // every slot's shuffle of a level goes out before the first add of that level, so the slots' latencies overlap
  // (one shuffle after another, each waited for by its add, cost a full shuffle latency per slot and level)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    A ts[RS_NSUM], tx[RX_NMAX];
#pragma unroll
    for (int i = 0; i < RS_NSUM; i++)
      if (SM & (1u << i)) ts[i] = __shfl_xor_sync(0xffffffffu, p.s[i], o);
#pragma unroll
    for (int i = 0; i < RX_NMAX; i++)
      if (XM & (1u << i)) tx[i] = __shfl_xor_sync(0xffffffffu, p.x[i], o);
#pragma unroll
    for (int i = 0; i < RS_NSUM; i++)
      if (SM & (1u << i)) p.s[i] += ts[i];
#pragma unroll
    for (int i = 0; i < RX_NMAX; i++)
      if (XM & (1u << i)) p.x[i] = mmax(p.x[i], tx[i]);
  }
}
// block-wide reduction in a fixed order; the result is valid in thread 0 (smem: >= 32 * (RS_NSUM + RX_NMAX) values)
template <unsigned SM = SUMS_ALL, unsigned XM = MAXS_ALL, class A>
__device__ __forceinline__ void blockReduce(Part<A> &p, A *smem) {
  warpReduce<SM, XM>(p);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  constexpr int NV = RS_NSUM + RX_NMAX;
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < RS_NSUM; i++)
      if (SM & (1u << i)) smem[wid * NV + i] = p.s[i];
#pragma unroll
    for (int i = 0; i < RX_NMAX; i++)
      if (XM & (1u << i)) smem[wid * NV + RS_NSUM + i] = p.x[i];
  }
  __syncthreads();
  if (wid == 0) {
    Part<A> q;
    q.init();
    if (lane < nw) {
#pragma unroll
      for (int i = 0; i < RS_NSUM; i++)
        if (SM & (1u << i)) q.s[i] = smem[lane * NV + i];
#pragma unroll
      for (int i = 0; i < RX_NMAX; i++)
        if (XM & (1u << i)) q.x[i] = smem[lane * NV + RS_NSUM + i];
    }
    warpReduce<SM, XM>(q);
    if (lane == 0) p = q;
  }
  __syncthreads();
}

// ------------------------------------------------------------------------------------------------ phase E
// kinetic-damping decision, residual and convergence of one instance from its reduced partials (solver_cpu.js:809-837);
// EXT: the kernel variant that has the extensions (the ground, a load protocol)
template <bool EXT, class A>
__device__ __forceinline__ void decide(const InstDesc &I, InstCtl &c, const Part<A> &p, int n_iter_stop,
                                       const double *rbq = nullptr) {
  double ke = 0.5 * double(p.s[RS_KE]);
  const bool rollback = I.kd && ke < c.ke_prev;
  if (!isfinite(ke)) { c.status = WS_NONFINITE; }
  if (rollback) { ke = 0.0; c.pending = 1; c.rollbacks++; }
  else { c.pending = 0; c.cur ^= 1; }
  c.obuf ^= 1;
  c.ke = ke; c.ke_prev = ke;
  c.iter += 1;
  if (I.aug && I.contacts && I.K) {
    // the penetration window of the multiplier: this iteration counts when it ran after the ramp; an update that was
    // due before it (applied by its crossings) restarted the window; the next is due every al_every iterations after
    // the ramp (solver_cpu.js:387,470,819-821)
    c.penN = (c.alPend ? 0 : c.penN) + (c.iter - 1 >= I.ramp_iter ? 1 : 0);
    c.alPend = (I.alEvery > 0 && c.iter > I.ramp_iter && (c.iter - I.ramp_iter) % I.alEvery == 0) ? 1 : 0;
  }
  const double maxM = I.p ? double(p.x[RX_M]) / fmax(I.jLenMin, 1e-12) : 0.0;
  const double maxFn = ((I.contacts && I.K) || (EXT && I.floorOn)) ? double(p.x[RX_FN]) : 0.0;
  const double fref = fmax(fmax(fmax(double(p.x[RX_LOAD]), double(p.x[RX_N])), fmax(maxM, maxFn)), 1e-12);
  c.fref = fref;
  c.res_f = I.n ? double(p.x[RX_F]) / fref : 0.0;
  c.res_t = I.m ? double(p.x[RX_T]) / (fref * I.lRef) : 0.0;
  // rbq: the rigid-body freedoms' unbalanced resultants |Q_t|, |Q_r| (Floor.rigidResidual, solver_cpu.js:574)
  const double resRb = rbq ? fmax(rbq[0] / fref, rbq[1] / (fref * I.rbR)) : 0.0;
  const double resid = fmax(fmax(c.res_f, c.res_t), resRb);
  c.residual = c.iter > I.warmup ? resid : INFINITY;
  c.e_stretch = double(p.s[RS_STRETCH]); c.e_shear = double(p.s[RS_SHEAR]);
  c.e_bend = double(p.s[RS_BEND]); c.e_twist = double(p.s[RS_TWIST]);
  // contact energy of the iteration: ½ Σ k_n pen² + ½ k_t Σ |S_e|² with the ramp of that iteration
  const double rampd = I.ramp_iter <= 0 ? 1.0 : fmin(1.0, 0.01 + 0.99 * double(c.iter - 1) / I.ramp_iter);
  c.e_contact = 0.5 * double(p.s[RS_PEN]) + 0.5 * rampd * I.stick * double(p.s[RS_TAN]);
  if (c.status == WS_RUNNING && !(EXT && I.utmMode)) {   // a load protocol runs on past convergence (protocolStep)
    if (c.residual <= I.tol) c.status = WS_CONVERGED;
    else if (c.iter >= I.max_iter) c.status = WS_MAX_ITER;
  }
  (void)n_iter_stop;
}

// The load protocol of one instance after its iteration (the UTM replay of web/js/wgsl.js:1048-1093): settle until
// convergence or `settle` iterations, average the probe's travel from P0 and its reaction along the axis over `avg`
// iterations, record them, then apply the next value of the schedule: the probe force (mode 1) or the probe's
// position P0 + value·axis, at rest (mode 2).  d is the view whose buffer `buf` holds the positions the instance
// continues from (after a roll-back, the restored ones).  One thread, in the kernel variants that have the extensions;
// it also records the ground's energy of the iteration (p: the reduced partials).
template <int P, class A>
__device__ __forceinline__ void protocolStep(const Dev<P> &d, int buf, const InstDesc &I, InstCtl &c, const Part<A> &p) {
  using W = typename Dev<P>::W;
  d.ext[I.utmIdx].eFloor = double(p.s[RS_FLOOR]);     // the ground's energy of the iteration, beside the protocol
  if (!I.utmMode || c.status != WS_RUNNING) return;
  const bool conv = c.residual <= I.tol;
  const int pi = I.utmProbe;
  InstExt &u = d.ext[I.utmIdx];
  u.it += 1;
  if (u.phase == 0) {
    if (conv || u.it >= I.utmSettle) {
      u.phase = 1; u.it = 0; u.accN = 0;
      for (int k = 0; k < 4; k++) u.sum[k] = 0.0;
    }
  } else if (u.phase == 1) {
    double r = 0.0;
    for (int k = 0; k < 3; k++) {
      u.sum[k] += double(Acc<P>::xw(d, buf, k, pi)) - u.p0[k];
      r += double(d.react[size_t(k) * d.ntot + pi]) * I.utmAxis[k];
    }
    u.sum[3] += r;
    u.accN += 1;
    if (u.it >= I.utmAvg) {
      double *o = d.utmOut + (size_t(I.utmIdx) * WS_PROTOCOL_MAX_INC + u.inc) * 4;
      const double n = double(u.accN);
      o[0] = (u.sum[0] * I.utmAxis[0] + u.sum[1] * I.utmAxis[1] + u.sum[2] * I.utmAxis[2]) / n;
      o[1] = u.sum[3] / n;
      o[2] = u.curF;
      o[3] = double(c.iter);
      u.inc += 1; u.it = 0; u.phase = 0;
      if (u.inc >= I.utmNInc) {
        u.phase = 2;
        c.status = WS_DONE;
      } else {
        const double v = d.utmSched[size_t(I.utmIdx) * WS_PROTOCOL_MAX_INC + min(u.inc, WS_PROTOCOL_MAX_INC - 1)];
        u.curF = v;
        if (I.utmMode == 1) {
          for (int k = 0; k < 3; k++) u.pf[k] = I.utmAxis[k] * v;
        } else {
          for (int k = 0; k < 3; k++) {
            Acc<P>::xs(d, buf, k, pi, W(u.p0[k] + I.utmAxis[k] * v));
            d.V[size_t(k) * d.nS + pi] = 0;
          }
        }
      }
    }
  }
  if (c.status == WS_RUNNING && c.iter >= I.max_iter) c.status = WS_MAX_ITER;
}

// ------------------------------------------------------------------------------------------------ rigid-body freedoms
// A model that only the ground holds carries six more freedoms: a translation v and a rotation w of the whole model
// about the centroid c of its nodes, driven by the resultant of the external forces (loads + ground) with fictitious
// masses from the ground springs in contact (Floor, solver_cpu.js:520-533,564-631; the step, solver_cpu.js:785-800).
// Sums of one iteration: [0..2] Q_t = sum (L + G), [3..5] Q_r = sum (x - c) x (L + G), [6..8] sum over the nodes in
// contact of (x - c)^2 per axis, [9] how many nodes are in contact.
enum { RB_NSUM = 10 };
constexpr double RB_MASS = 2.0, RB_LEVER = 0.05;    // solver_cpu.js:37,39 (RB_VMAX is in the host's speed limits)

// node i's share of the sums, at its position `x` at the start of the iteration (buffer `buf`) about c
template <int P>
__device__ __forceinline__ void rigidNode(const Dev<P> &d, int buf, int i, const double c[3], double s[RB_NSUM]) {
  const int nt = d.ntot;
  double dx[3], g[3];
  for (int k = 0; k < 3; k++) {
    dx[k] = double(Acc<P>::xw(d, buf, k, i)) - c[k];
    g[k] = double(d.ldTot[k * nt + i]) + double(d.flF[k * nt + i]);
  }
  s[0] += g[0]; s[1] += g[1]; s[2] += g[2];
  s[3] += dx[1] * g[2] - dx[2] * g[1]; s[4] += dx[2] * g[0] - dx[0] * g[2]; s[5] += dx[0] * g[1] - dx[1] * g[0];
  if (d.flState[i]) { s[6] += dx[0] * dx[0]; s[7] += dx[1] * dx[1]; s[8] += dx[2] * dx[2]; s[9] += 1.0; }
}
// one thread: the fictitious masses (Floor.rigidMasses), the velocity update (v += Q / M, damping, speed limit; not in
// the warm-up, which zeroes them), the kinetic energy the rigid step adds (sum M v^2, to be halved with the rest), and
// |Q_t|, |Q_r| for the residual
__device__ __forceinline__ double rigidUpdate(const InstDesc &I, int iter, bool warm, const double s[RB_NSUM], InstExt &u,
                                             double rbq[2]) {
  const double rampN = I.ramp_iter;
  const double ramp = rampN <= 0 ? 1.0 : fmin(1.0, 0.01 + 0.99 * double(iter) / rampN);
  const double kn = ramp * I.strength, kt = ramp * I.stick, f = I.ms * RB_MASS;
  const double nc = fmax(s[9], 1.0), rmin = (RB_LEVER * I.rbR) * (RB_LEVER * I.rbR) * kn;
  double M[6];
  M[0] = fmax(f * nc * kt, 1e-30); M[1] = M[0]; M[2] = fmax(f * nc * kn, 1e-30);
  M[3] = fmax(f * fmax(kn * s[7] + kt * s[8], rmin), 1e-30); M[4] = fmax(f * fmax(kn * s[6] + kt * s[8], rmin), 1e-30);
  M[5] = fmax(f * fmax(kt * (s[6] + s[7]), rmin), 1e-30);
  if (warm) {
    for (int k = 0; k < 3; k++) u.rbV[k] = u.rbW[k] = 0.0;
  } else {
    for (int k = 0; k < 3; k++) {
      u.rbV[k] = fmin(fmax((u.rbV[k] + s[k] / M[k]) * I.damping, -I.rbVmax), I.rbVmax);
      u.rbW[k] = fmin(fmax((u.rbW[k] + s[3 + k] / M[3 + k]) * I.damping, -I.rbWmax), I.rbWmax);
    }
  }
  rbq[0] = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
  rbq[1] = sqrt(s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
  double ke = 0.0;
  for (int k = 0; k < 3; k++) ke += M[k] * u.rbV[k] * u.rbV[k] + M[3 + k] * u.rbW[k] * u.rbW[k];
  return ke;
}
__device__ __forceinline__ bool rigidMoves(const InstExt &u) {
  return u.rbV[0] != 0.0 || u.rbV[1] != 0.0 || u.rbV[2] != 0.0 || u.rbW[0] != 0.0 || u.rbW[1] != 0.0 || u.rbW[2] != 0.0;
}
// the rigid step of node i: x (buffer nxt) += v + w x (x_prev - c), x_prev in buffer cur
template <int P>
__device__ __forceinline__ void rigidMoveNode(const Dev<P> &d, int cur, int nxt, int i, const double c[3], const double v[3],
                                              const double w[3]) {
  using W = typename Dev<P>::W;
  double dx[3];
  for (int k = 0; k < 3; k++) dx[k] = double(Acc<P>::xw(d, cur, k, i)) - c[k];
  const double m[3] = {v[0] + w[1] * dx[2] - w[2] * dx[1], v[1] + w[2] * dx[0] - w[0] * dx[2], v[2] + w[0] * dx[1] - w[1] * dx[0]};
  for (int k = 0; k < 3; k++) Acc<P>::xs(d, nxt, k, i, W(double(Acc<P>::xw(d, nxt, k, i)) + m[k]));
}
// the rigid step of segment j's frame (buffer nxt): q <- normalize(exp(w) ⊗ q)
template <int P>
__device__ __forceinline__ void rigidMoveSeg(const Dev<P> &d, int nxt, int j, const double qw[4]) {
  using W = typename Dev<P>::W;
  W q[4], qr[4];
  for (int k = 0; k < 4; k++) q[k] = Acc<P>::qw(d, nxt, k, j);
  const W a[4] = {W(qw[0]), W(qw[1]), W(qw[2]), W(qw[3])};
  qmul(a, q, qr);
  qnormalize<W, P == PREC_MIXED>(qr);
  for (int k = 0; k < 4; k++) Acc<P>::qs(d, nxt, k, j, qr[k]);
}

template <class A>
__device__ __forceinline__ StepCtx makeCtx(const InstDesc &I, const InstCtl &c, const double *utmPf = nullptr) {
  StepCtx sc;
  sc.utmPf = utmPf;
  sc.cur = c.cur; sc.nxt = c.cur ^ 1; sc.obuf = c.obuf; sc.onxt = c.obuf ^ 1; sc.pending = c.pending; sc.iter = c.iter;
  sc.warm = (c.iter < I.warmup && I.contacts && I.K) ? 1 : 0;
  sc.alPend = c.alPend; sc.penN = c.penN;
  const int start = max(c.disp_it0, (I.contacts && I.K) ? I.warmup : 0);
  sc.dispR = I.disp_ramp > 0 ? fmin(1.0, fmax(0.0, double(c.iter - start + 1) / I.disp_ramp)) : 1.0;
  return sc;
}

}  // namespace wsb
