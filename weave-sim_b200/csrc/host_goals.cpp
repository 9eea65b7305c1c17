// Host-side goal assembly (f64) — see host_goals.hpp.
#include "host_goals.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>

namespace wsb {

// ------------------------------------------------------------------------------------------------ small helpers
static void qnorm4(double *q) {
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (n == 0) n = 1.0;
  for (int k = 0; k < 4; k++) q[k] /= n;
}
template <class T>
static std::vector<T> copyOf(const T *p, size_t n) { return p ? std::vector<T>(p, p + n) : std::vector<T>(n, T(0)); }

// ------------------------------------------------------------------------------------------------ model
void HostGoals::loadModel(const ws_model &md, bool keepState) {
  if (md.n <= 0 || md.m < 0 || md.p < 0 || md.K < 0 || md.n_strands <= 0) throw std::invalid_argument("model: bad sizes");
  if (!md.X || !md.Q || !md.l0 || !md.seg_i0 || !md.seg_i1 || !md.seg_offset || !md.EA || !md.EIx || !md.EIy || !md.GJ || !md.GA || !md.load_const)
    throw std::invalid_argument("model: a required array is missing");
  if (md.K && (!md.cross_strand || !md.cross_wk || !md.cross_hk || !md.cross_u || !md.cross_nprev || !md.cross_enabled || !md.cross_locked || !md.cross_mu))
    throw std::invalid_argument("model: crossing arrays are missing");
  if (keepState && (md.n != n || md.m != m || md.p != p || md.K != K || md.n_strands != S))
    throw std::invalid_argument("model: the topology differs from the instance's");
  n = md.n; m = md.m; p = md.p; S = md.n_strands; K = md.K;
  prm = md.params;
  if (!keepState) {
    X = copyOf(md.X, 3 * size_t(n));
    X0 = md.X0 ? copyOf(md.X0, 3 * size_t(n)) : X;
    Q = copyOf(md.Q, 4 * size_t(m));
    u = copyOf(md.cross_u, 2 * size_t(K));
    nPrev = copyOf(md.cross_nprev, 3 * size_t(K));
    segI0 = copyOf(md.seg_i0, m); segI1 = copyOf(md.seg_i1, m);
    segOffset = copyOf(md.seg_offset, S + 1);
    jSeg0 = copyOf(md.joint_seg0, p); jSeg1 = copyOf(md.joint_seg1, p);
    l0 = copyOf(md.l0, m); jLen = copyOf(md.joint_len, p);
    for (int j = 0; j < m; j++) {
      if (segI0[j] < 0 || segI0[j] >= n || segI1[j] < 0 || segI1[j] >= n) throw std::invalid_argument("model: segment node out of range");
      if (!(l0[j] > 0)) throw std::invalid_argument("model: rest length must be positive");
    }
    for (int j = 0; j < p; j++)
      if (jSeg0[j] < 0 || jSeg0[j] >= m || jSeg1[j] < 0 || jSeg1[j] >= m) throw std::invalid_argument("model: joint segment out of range");
    if (segOffset[0] != 0 || segOffset[S] != m) throw std::invalid_argument("model: seg_offset must run from 0 to m");
    for (int s = 0; s < S; s++) if (segOffset[s + 1] < segOffset[s]) throw std::invalid_argument("model: seg_offset must not decrease");
    for (int i = 0; i < 2 * K; i++) if (md.cross_strand[i] < 0 || md.cross_strand[i] >= S) throw std::invalid_argument("model: crossing strand out of range");
    proto = ws_protocol{};
    if (md.protocol && md.protocol->mode) {
      const ws_protocol &pr = *md.protocol;
      if (pr.mode < 0 || pr.mode > 2) throw std::invalid_argument("model: protocol mode must be 0, 1 or 2");
      if (pr.probe < 0 || pr.probe >= n) throw std::invalid_argument("model: protocol probe node out of range");
      if (pr.n_inc < 1 || pr.n_inc > WS_PROTOCOL_MAX_INC) throw std::invalid_argument("model: protocol needs 1..64 increments");
      if (pr.settle < 0 || pr.avg < 1) throw std::invalid_argument("model: protocol settle must be >= 0 and avg >= 1");
      proto = pr;
    }
  }
  omega0 = md.omega0 ? copyOf(md.omega0, 3 * size_t(p)) : std::vector<double>(3 * size_t(p), 0.0);
  EA = copyOf(md.EA, m); GA = copyOf(md.GA, m);
  EIx.resize(p); EIy.resize(p); GJ.resize(p);
  for (int j = 0; j < p; j++) { const int s0 = jSeg0[j]; EIx[j] = md.EIx[s0]; EIy[j] = md.EIy[s0]; GJ[j] = md.GJ[s0]; }
  loadConst = copyOf(md.load_const, 3 * size_t(n));
  loadLocal.assign(3 * size_t(n), 0.0); hasLocal.assign(n, 0);
  for (int l = 0; l < md.n_local_loads; l++) {
    const int nid = md.local_load_node[l];
    if (nid < 0 || nid >= n) throw std::invalid_argument("model: local load node out of range");
    for (int c = 0; c < 3; c++) loadLocal[3 * size_t(nid) + c] += md.local_load_F[3 * size_t(l) + c];
    hasLocal[nid] = 1;
  }
  loadMaxConst = 0;
  for (double v : loadConst) loadMaxConst = std::max(loadMaxConst, std::fabs(v));
  // crossings
  cxSegOff.resize(2 * size_t(K)); cxNseg.resize(2 * size_t(K)); cxStrand.resize(2 * size_t(K));
  for (int i = 0; i < 2 * K; i++) {
    const int s = md.cross_strand[i];
    cxStrand[i] = s; cxSegOff[i] = segOffset[s]; cxNseg[i] = segOffset[s + 1] - segOffset[s];
    if (cxNseg[i] < 1) throw std::invalid_argument("model: a crossing lies on a strand without segments");
  }
  wk = copyOf(md.cross_wk, 2 * size_t(K)); hk = copyOf(md.cross_hk, 2 * size_t(K));
  w.resize(K); h.resize(K);
  for (int c = 0; c < K; c++) { w[c] = 0.5 * (wk[2 * c] + wk[2 * c + 1]); h[c] = 0.5 * (hk[2 * c] + hk[2 * c + 1]); }
  mu = copyOf(md.cross_mu, K);
  // N/mm² defaults of the classification (solver_cpu.js:231-271)
  auto orDefault = [&](const double *p, double v) { return p ? copyOf(p, 2 * size_t(K)) : std::vector<double>(2 * size_t(K), v); };
  fc90 = orDefault(md.cross_fc90, 8.0); E90 = orDefault(md.cross_E90, 800.0); Hs = orDefault(md.cross_H, 30.0);
  enabled = copyOf(md.cross_enabled, K); locked = copyOf(md.cross_locked, K);
}

// node -> segments, segment -> joints, strand of every segment (static gather tables)
static void buildTables(HostGoals &g) {
  g.nodeSegOut.assign(g.n, -1); g.nodeSegIn.assign(g.n, -1);
  for (int j = 0; j < g.m; j++) {
    if (g.nodeSegOut[g.segI0[j]] >= 0 || g.nodeSegIn[g.segI1[j]] >= 0)
      throw std::invalid_argument("model: a node starts or ends more than one segment (strands must be simple polylines)");
    g.nodeSegOut[g.segI0[j]] = j; g.nodeSegIn[g.segI1[j]] = j;
  }
  g.segJointA.assign(g.m, -1); g.segJointB.assign(g.m, -1);
  for (int j = 0; j < g.p; j++) {
    if (g.segJointA[g.jSeg0[j]] >= 0 || g.segJointB[g.jSeg1[j]] >= 0) throw std::invalid_argument("model: a segment is in two joints on one side");
    g.segJointA[g.jSeg0[j]] = j; g.segJointB[g.jSeg1[j]] = j;
  }
  g.segStrand.resize(g.m); g.segLocal.resize(g.m);
  for (int s = 0; s < g.S; s++)
    for (int j = g.segOffset[s]; j < g.segOffset[s + 1]; j++) { g.segStrand[j] = s; g.segLocal[j] = j - g.segOffset[s]; }
  // linear crossing strands: segment k of the strand joins nodes N0 + k and N0 + k + 1, and its end nodes start or end
  // no other segment (the layout buildState gives, model.js:10-75), so a crossing side's nodes and neighbouring
  // segments are the strand's first node and segment plus the side's segment index
  auto linear = [&](int s) {
    const int j0 = g.segOffset[s], j1 = g.segOffset[s + 1];
    if (j1 <= j0) return false;
    const int n0 = g.segI0[j0];
    for (int j = j0; j < j1; j++)
      if (g.segI0[j] != n0 + (j - j0) || g.segI1[j] != n0 + (j - j0) + 1) return false;
    return g.nodeSegIn[n0] < 0 && g.nodeSegOut[n0 + (j1 - j0)] < 0;
  };
  std::vector<signed char> lin(g.S, -1);
  g.cxNodeOff.assign(2 * size_t(g.K), 0);
  g.cxLinear = true;
  for (int i = 0; i < 2 * g.K; i++) {
    const int s = g.cxStrand[i];
    if (lin[s] < 0) lin[s] = linear(s) ? 1 : 0;
    g.cxLinear = g.cxLinear && lin[s] == 1;
    g.cxNodeOff[i] = g.segI0[g.segOffset[s]];
  }
}

// Anchors (model.js:162-189) and the clamp joints of the rotation anchors (rod_cosserat.js:92-100), frozen at Q
void HostGoals::buildAnchors(const ws_model &md) {
  nodeFree.assign(3 * size_t(n), 1);
  std::vector<std::vector<int>> adj(n);
  for (int j = 0; j < m; j++) { adj[segI0[j]].push_back(j); adj[segI1[j]].push_back(j); }
  cSeg.clear(); cNode.clear(); cLen.clear(); cB.clear(); cQ.clear();
  for (int a = 0; a < md.n_anchors; a++) {
    const int nid = md.anchor_node[a];
    if (nid < 0 || nid >= n) throw std::invalid_argument("model: anchor node out of range");
    const uint8_t mk = md.anchor_mask[a];
    for (int c = 0; c < 3; c++) if (mk & (1 << c)) nodeFree[3 * size_t(nid) + c] = 0;
    if (mk & 0x38)
      for (int j : adj[nid]) {
        cSeg.push_back(j); cNode.push_back(nid); cLen.push_back(0.5 * l0[j]);
        cB.push_back((mk & 8) ? md.EIx[j] : 0.0); cB.push_back((mk & 16) ? md.EIy[j] : 0.0); cB.push_back((mk & 32) ? md.GJ[j] : 0.0);
        for (int k = 0; k < 4; k++) cQ.push_back(Q[4 * size_t(j) + k]);
      }
  }
  C = int(cSeg.size());
  if (proto.mode == 2)   // displacement control holds the probe (solver_gpu.js:215)
    for (int c = 0; c < 3; c++) nodeFree[3 * size_t(proto.probe) + c] = 0;
  if (prm.floor) {
    if (!md.node_w || !md.node_h) throw std::invalid_argument("model: a ground needs node_w and node_h");
    bool held = C > 0;
    for (uint8_t f : nodeFree) held = held || !f;
    nodeW.assign(md.node_w, md.node_w + n); nodeH.assign(md.node_h, md.node_h + n);
    // a model that only the ground holds gets the rigid-body freedoms (Floor, solver_cpu.js:520-533,546-562): the
    // model radius about the centroid of the nodes, the speed limits from the thinnest section
    rigid = !held;
    if (rigid && proto.mode) throw std::invalid_argument("model: a load protocol on a model that only the ground holds");
    double c[3] = {0, 0, 0}, R2 = 0, hmin = std::numeric_limits<double>::infinity();
    for (int i = 0; i < n; i++) for (int k = 0; k < 3; k++) c[k] += X[3 * size_t(i) + k] / std::max(n, 1);
    for (int i = 0; i < n; i++) {
      double r2 = 0;
      for (int k = 0; k < 3; k++) r2 += (X[3 * size_t(i) + k] - c[k]) * (X[3 * size_t(i) + k] - c[k]);
      R2 = std::max(R2, r2);
      hmin = std::min(hmin, std::min(nodeH[i], nodeW[i]));
    }
    rbR = std::max(std::sqrt(R2), 1e-9);
    rbVmax = 0.05 * (std::isfinite(hmin) && hmin > 0 ? hmin : 1.0);      // RB_VMAX, solver_cpu.js:38
    rbWmax = rbVmax / rbR;
  }
  fixedAny.assign(n, 0);
  for (int i = 0; i < n; i++) fixedAny[i] = (nodeFree[3 * size_t(i)] && nodeFree[3 * size_t(i) + 1] && nodeFree[3 * size_t(i) + 2]) ? 0 : 1;
  segClamp0.assign(m, -1); segClamp1.assign(m, -1);
  for (int c = 0; c < C; c++) {
    const int j = cSeg[c];
    if (segClamp0[j] < 0) segClamp0[j] = c;
    else if (segClamp1[j] < 0) segClamp1[j] = c;
    else throw std::invalid_argument("model: more than two clamp joints on one segment");
  }
}

// prescribed support motion: from where the anchored nodes are now to the model's targets
void HostGoals::buildTargets(const ws_model &md) {
  ancIndex.assign(n, -1); ancStart.clear(); ancDelta.clear();
  if (!md.anchor_target) return;
  for (int a = 0; a < md.n_anchors; a++) {
    const int nid = md.anchor_node[a];
    if (!(md.anchor_mask[a] & 7) || ancIndex[nid] >= 0) continue;
    ancIndex[nid] = int(ancStart.size() / 3);
    for (int c = 0; c < 3; c++) {
      ancStart.push_back(X[3 * size_t(nid) + c]);
      ancDelta.push_back((md.anchor_mask[a] & (1 << c)) ? md.anchor_target[3 * size_t(a) + c] - X[3 * size_t(nid) + c] : 0.0);
    }
  }
}

int HostGoals::sideSegLocal(int sd) const {
  const double uu = u[sd];
  const int ns = cxNseg[sd];
  return int(std::min(std::max(std::floor(uu), 0.0), double(std::max(ns - 1, 0))));
}

double HostGoals::sideSegMin() const {
  double mn = INFINITY;
  std::vector<char> seen(S, 0);
  for (int sd = 0; sd < 2 * K; sd++) {
    if (seen[cxStrand[sd]]) continue;
    seen[cxStrand[sd]] = 1;
    for (int j = cxSegOff[sd]; j < cxSegOff[sd] + cxNseg[sd]; j++) mn = std::min(mn, l0[j]);
  }
  return mn;
}

void HostGoals::sortSides() {
  strandSideOff.assign(S, 0); strandSideCnt.assign(S, 0);
  std::vector<std::vector<int>> per(S);
  for (int sd = 0; sd < 2 * K; sd++) per[cxStrand[sd]].push_back(sd);
  sideList.clear(); sidePos.assign(2 * K, 0);
  for (int s = 0; s < S; s++)
    for (int sd : per[s]) { sidePos[sd] = int(sideList.size()); sideList.push_back(sd); }
  ord.clear(); ordSeg.clear();
  for (int s = 0; s < S; s++) {
    std::vector<int> &L = per[s];
    std::stable_sort(L.begin(), L.end(), [&](int a, int b) {
      const int sa = sideSegLocal(a), sb = sideSegLocal(b);
      return sa != sb ? sa < sb : a < b;
    });
    strandSideOff[s] = int(ord.size()); strandSideCnt[s] = int(L.size());
    for (int sd : L) { ord.push_back(sd); ordSeg.push_back(sideSegLocal(sd)); }
  }
  rngLo.assign(m, 0); rngHi.assign(m, 0);
  for (int j = 0; j < m; j++) {
    const int s = segStrand[j], lj = segLocal[j];
    const int *b = ordSeg.data() + strandSideOff[s], *e = b + strandSideCnt[s];
    rngLo[j] = int(std::lower_bound(b, e, lj) - ordSeg.data());
    rngHi[j] = int(std::upper_bound(b, e, lj) - ordSeg.data());
  }
}

// ------------------------------------------------------------------------------------------------ contact set-up
// node tangents and node frames of the current state (PolylineContact._prepare, solver_cpu.js:179-193, with
// nodeQuats, model.js:89-105), the Hermite evaluation of one side (solver_cpu.js:197-228)
struct SideEval { double P[3], t[3], L; };

static void nodeTangentsAndQuats(const HostGoals &g, std::vector<double> &Tn, std::vector<double> &Qn) {
  Tn.assign(3 * size_t(g.n), 0.0); Qn.assign(4 * size_t(g.n), 0.0);
  std::vector<double> eh(3 * size_t(g.m));
  for (int j = 0; j < g.m; j++) {
    const size_t a = g.segI0[j], b = g.segI1[j];
    double e[3] = {g.X[3 * b] - g.X[3 * a], g.X[3 * b + 1] - g.X[3 * a + 1], g.X[3 * b + 2] - g.X[3 * a + 2]};
    const double l = std::max(std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]), 1e-12);
    for (int k = 0; k < 3; k++) eh[3 * size_t(j) + k] = e[k] / l;
  }
  for (int i = 0; i < g.n; i++) {
    const int so = g.nodeSegOut[i], si = g.nodeSegIn[i];
    double T[3] = {0, 0, 0};
    if (so >= 0) for (int k = 0; k < 3; k++) T[k] += eh[3 * size_t(so) + k];
    if (si >= 0) for (int k = 0; k < 3; k++) T[k] += eh[3 * size_t(si) + k];
    const double l = std::max(std::sqrt(T[0] * T[0] + T[1] * T[1] + T[2] * T[2]), 1e-12);
    for (int k = 0; k < 3; k++) Tn[3 * size_t(i) + k] = T[k] / l;
    const int ref = so >= 0 ? so : si;
    double q[4] = {0, 0, 0, 0};
    for (int j : {so, si}) {
      if (j < 0) continue;
      const double *Qj = &g.Q[4 * size_t(j)], *Qr = &g.Q[4 * size_t(ref)];
      const double d = Qj[0] * Qr[0] + Qj[1] * Qr[1] + Qj[2] * Qr[2] + Qj[3] * Qr[3];
      const double sg = d < 0 ? -1 : 1;
      for (int k = 0; k < 4; k++) q[k] += sg * Qj[k];
    }
    qnorm4(q);
    for (int k = 0; k < 4; k++) Qn[4 * size_t(i) + k] = q[k];
  }
}

static SideEval evalSide(const HostGoals &g, const std::vector<double> &Tn, int sd) {
  const int ls = g.sideSegLocal(sd);
  const double t = std::min(std::max(g.u[sd] - ls, 0.0), 1.0);
  const int seg = g.cxSegOff[sd] + ls;
  const size_t a = g.segI0[seg], b = g.segI1[seg];
  const double *Xa = &g.X[3 * a], *Xb = &g.X[3 * b];
  const double d[3] = {Xb[0] - Xa[0], Xb[1] - Xa[1], Xb[2] - Xa[2]};
  SideEval e;
  e.L = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double t2 = t * t, t3 = t * t * t;
  const double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + t, h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
  const double d00 = 6 * t2 - 6 * t, d10 = 3 * t2 - 4 * t + 1, d01 = -6 * t2 + 6 * t, d11 = 3 * t2 - 2 * t;
  for (int k = 0; k < 3; k++) {
    e.P[k] = h00 * Xa[k] + (h10 * e.L) * Tn[3 * a + k] + h01 * Xb[k] + (h11 * e.L) * Tn[3 * b + k];
    e.t[k] = d00 * Xa[k] + (d10 * e.L) * Tn[3 * a + k] + d01 * Xb[k] + (d11 * e.L) * Tn[3 * b + k];
  }
  const double tl = std::max(std::sqrt(e.t[0] * e.t[0] + e.t[1] * e.t[1] + e.t[2] * e.t[2]), 1e-12);
  for (int k = 0; k < 3; k++) e.t[k] /= tl;
  return e;
}

// closest-point pairing of the material points by three guarded Gauss-Newton sweeps; persistent normals
void HostGoals::contactInitialize(int sweeps) {
  if (!K) return;
  std::vector<double> Tn, Qn;
  nodeTangentsAndQuats(*this, Tn, Qn);       // positions do not change during the sweeps
  std::vector<SideEval> A(K), B(K);
  std::vector<double> St(3 * size_t(K)), nrmv(3 * size_t(K)), before(K);
  auto offsets = [&]() {
    for (int c = 0; c < K; c++) {
      A[c] = evalSide(*this, Tn, 2 * c); B[c] = evalSide(*this, Tn, 2 * c + 1);
      const double *tA = A[c].t, *tB = B[c].t, *np = &nPrev[3 * size_t(c)];
      double nx = tA[1] * tB[2] - tA[2] * tB[1], ny = tA[2] * tB[0] - tA[0] * tB[2], nz = tA[0] * tB[1] - tA[1] * tB[0];
      const double nn = std::sqrt(nx * nx + ny * ny + nz * nz);
      if (nn < 1e-6) { nx = np[0]; ny = np[1]; nz = np[2]; }
      else { const double d = std::max(nn, 1e-12); nx /= d; ny /= d; nz /= d; }
      if (nx * np[0] + ny * np[1] + nz * np[2] < 0) { nx = -nx; ny = -ny; nz = -nz; }
      const double S_[3] = {B[c].P[0] - A[c].P[0], B[c].P[1] - A[c].P[1], B[c].P[2] - A[c].P[2]};
      const double gg = S_[0] * nx + S_[1] * ny + S_[2] * nz;
      St[3 * size_t(c)] = S_[0] - gg * nx; St[3 * size_t(c) + 1] = S_[1] - gg * ny; St[3 * size_t(c) + 2] = S_[2] - gg * nz;
      nrmv[3 * size_t(c)] = nx; nrmv[3 * size_t(c) + 1] = ny; nrmv[3 * size_t(c) + 2] = nz;
    }
  };
  auto len = [&](int c) { const double *s = &St[3 * size_t(c)]; return std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]); };
  for (int it = 0; it < sweeps; it++) {
    offsets();
    std::vector<double> uOld = u;
    for (int c = 0; c < K; c++) {
      const double *tA = A[c].t, *tB = B[c].t, *s = &St[3 * size_t(c)];
      const double taa = tA[0] * tA[0] + tA[1] * tA[1] + tA[2] * tA[2], tbb = tB[0] * tB[0] + tB[1] * tB[1] + tB[2] * tB[2], tab = tA[0] * tB[0] + tA[1] * tB[1] + tA[2] * tB[2];
      const double sa = s[0] * tA[0] + s[1] * tA[1] + s[2] * tA[2], sb = s[0] * tB[0] + s[1] * tB[1] + s[2] * tB[2];
      const double det = taa * tbb - tab * tab;
      const bool ok = det > 1e-3 && enabled[c];
      const double ca = ok ? (sa * tbb - sb * tab) / det : 0, cb = ok ? (sb * taa - sa * tab) / det : 0;
      before[c] = len(c);
      u[2 * size_t(c)] = std::min(std::max(u[2 * size_t(c)] + ca / std::max(A[c].L, 1e-12), 0.0), double(cxNseg[2 * c]));
      u[2 * size_t(c) + 1] = std::min(std::max(u[2 * size_t(c) + 1] - cb / std::max(B[c].L, 1e-12), 0.0), double(cxNseg[2 * c + 1]));
    }
    offsets();
    for (int c = 0; c < K; c++) if (len(c) >= before[c]) { u[2 * size_t(c)] = uOld[2 * size_t(c)]; u[2 * size_t(c) + 1] = uOld[2 * size_t(c) + 1]; }
  }
  offsets();
  nPrev = nrmv;
}

// node masses ms·Σk (rod: (EA + GA)/l0 per end node; contact: strength + stick on the nodes of each side's segment, and
// with W2 the rotational spring k_t·0.38²·wA·wB/0.5 / l0² of each crossing) and
// static frame stiffness per body axis (joints B/l̄, clamps B/l_c, shear lever κGA L²/l0): rod_cosserat.js:186-209,
// solver_cpu.js:151-167, 694-705
void HostGoals::buildMasses(double ramp, const std::vector<double> &Fn) {
  (void)ramp; (void)Fn;   // the contact twist share of the inertia is rebuilt by the device every iteration
  std::vector<double> kNode(n, 0.0);
  for (int j = 0; j < m; j++) {
    const double k = (EA[j] + GA[j]) / l0[j];
    kNode[segI0[j]] += k; kNode[segI1[j]] += k;
  }
  if (prm.contacts && K) {
    const double k = prm.strength + prm.stick_strength;
    for (int side = 0; side < 2; side++) {
      for (int c = 0; c < K; c++) kNode[segI0[cxSegOff[2 * c + side] + sideSegLocal(2 * c + side)]] += k;
      for (int c = 0; c < K; c++) kNode[segI1[cxSegOff[2 * c + side] + sideSegLocal(2 * c + side)]] += k;
    }
    // W2: the rotational spring of each crossing on the nodes of both sides' segments
    if (prm.rot_friction)
      for (int side = 0; side < 2; side++)
        for (int pass = 0; pass < 2; pass++)
          for (int c = 0; c < K; c++) {
            const int seg = cxSegOff[2 * c + side] + sideSegLocal(2 * c + side);
            const double kr = prm.stick_strength * (0.38 * 0.38) * wk[2 * size_t(c)] * wk[2 * size_t(c) + 1] / 0.5;
            const double l = std::max(l0[seg], 1e-12);
            kNode[pass ? segI1[seg] : segI0[seg]] += kr / (l * l);
          }
  }
  if (prm.floor)                                      // Floor.addStiffness (solver_cpu.js:565)
    for (int i = 0; i < n; i++) kNode[i] += prm.strength + prm.stick_strength;
  const double ms = prm.mass_scale;
  mass.resize(n);
  for (int i = 0; i < n; i++) mass[i] = ms * std::max(kNode[i], 1e-12);
  kRotStatic.assign(3 * size_t(m), 0.0);
  for (int j = 0; j < p; j++) {
    const double lb = std::max(jLen[j], 1e-12), B[3] = {EIx[j], EIy[j], GJ[j]};
    for (int s : {jSeg0[j], jSeg1[j]}) for (int k = 0; k < 3; k++) kRotStatic[3 * size_t(s) + k] += B[k] / lb;
  }
  for (int c = 0; c < C; c++) for (int k = 0; k < 3; k++) kRotStatic[3 * size_t(cSeg[c]) + k] += cB[3 * size_t(c) + k] / std::max(cLen[c], 1e-12);
  for (int j = 0; j < m; j++) {
    const size_t a = segI0[j], b = segI1[j];
    const double L = std::hypot(X[3 * b] - X[3 * a], X[3 * b + 1] - X[3 * a + 1], X[3 * b + 2] - X[3 * a + 2]);
    const double k = GA[j] * L * L / l0[j];
    kRotStatic[3 * size_t(j)] += k; kRotStatic[3 * size_t(j) + 1] += k;
  }
  double lmin = 1e300;
  for (double v : jLen) lmin = std::min(lmin, v);
  jLenMin = p ? lmin : 1.0;
  for (double v : l0) lmin = std::min(lmin, v);
  lRef = lmin < 1e300 ? lmin : 1.0;
}

// the load protocol starts: P0 is the probe's position now; displacement control places the probe at the first value
void HostGoals::startProtocol() {
  if (!proto.mode) return;
  for (int c = 0; c < 3; c++) probe0[c] = X[3 * size_t(proto.probe) + c];
  if (proto.mode == 2)
    for (int c = 0; c < 3; c++) X[3 * size_t(proto.probe) + c] = probe0[c] + proto.axis[c] * proto.sched[0];
}

void HostGoals::build(const ws_model &md) {
  loadModel(md, false);
  dentAfterDefault = md.params.warmup_iter + md.params.ramp_iter;
  buildTables(*this);
  buildAnchors(md);
  if (prm.contacts && K) contactInitialize();
  buildMasses(1.0, std::vector<double>(K, 0.0));
  buildTargets(md);
  sortSides();
  startProtocol();          // after the goals: they are the model's, as GpuSolver uploads it (solver_gpu.js:286,311)
}

// warm start (rebuildGoals): the caller has put the current X, Q, u, nPrev into this object first
void HostGoals::rebuild(const ws_model &md) {
  loadModel(md, true);
  buildAnchors(md);
  buildMasses(1.0, std::vector<double>(K, 0.0));
  buildTargets(md);
  sortSides();
}

}  // namespace wsb
