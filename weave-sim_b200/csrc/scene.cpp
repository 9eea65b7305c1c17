// Scene builder: triangle mesh -> Kagome laths -> flat solver model (ws_model).
//
// Host-side set-up, f64.  It follows the reference's input chain step by step so that a mesh gives the same strands,
// knots, polylines, frames and state as the web solver's:
//   Mesh.fromArrays / edgeTopology / normals            web/js/mesh.js:8-21, 137-187
//   buildTopology: traceStrands, assignParity, applyFlips, buildPolylines, consistentFrames
//                                                       web/js/topology.js:78-345
//   topologyFromPolylines (stand-alone laths)           web/js/topology.js:348-363
//   buildState                                          web/js/model.js:10-75
//   anchorMasks / Anchors selection, Loads              web/js/model.js:150-231
//   section stiffness                                   web/js/params.js:33-45
//   seeded numbers (xoshiro128** + splitmix32)          web/js/rng.js:4-27
// The family colouring (topology.js:152-174) is display-only and is not built.
#include "scene.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>
#include <unordered_map>
#include <unordered_set>

namespace wsb {

// ------------------------------------------------------------------------------------------------ seeded numbers
Rng::Rng(uint32_t seed) {
  uint32_t a = seed;
  auto sm = [&a]() {
    a = a + 0x9e3779b9u;
    uint32_t t = a ^ (a >> 16);
    t = t * 0x21f0aaadu;
    t ^= t >> 15;
    t = t * 0x735a2d97u;
    return t ^ (t >> 15);
  };
  s[0] = sm(); s[1] = sm(); s[2] = sm(); s[3] = sm();
}
static inline uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
uint32_t Rng::u32() {
  uint32_t r = rotl32(s[1] * 5u, 7) * 9u, t = s[1] << 9;
  s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl32(s[3], 11);
  return r;
}
double Rng::uniform() {
  double hi = double(u32() >> 5);
  double lo = double(u32() >> 6);
  return (hi * 67108864.0 + lo) / 9007199254740992.0;
}
double Rng::normal() {
  if (has_spare) { has_spare = false; return spare; }
  double u = 0;
  while (u == 0) u = uniform();
  double v = uniform(), r = std::sqrt(-2.0 * std::log(u));
  spare = r * std::sin(2 * M_PI * v); has_spare = true;
  return r * std::cos(2 * M_PI * v);
}

// ------------------------------------------------------------------------------------------------ small vectors
static inline V3 sub3(const V3 &a, const V3 &b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static inline V3 add3(const V3 &a, const V3 &b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
static inline V3 scl3(const V3 &a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
static inline double dot3(const V3 &a, const V3 &b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline V3 cross3(const V3 &a, const V3 &b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static inline double norm3(const V3 &a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
static inline V3 normalize3(const V3 &v, double eps = 1e-12) {
  double n = norm3(v);
  if (n < eps) n = 1.0;
  return {v[0] / n, v[1] / n, v[2] / n};
}

// ------------------------------------------------------------------------------------------------ mesh
// edge i of a face is opposite local vertex i; E = sorted unique vertex pairs; EF in the fill order of mesh.js:137-163
Mesh Mesh::fromArrays(const std::vector<double> &V, const std::vector<int> &F) {
  Mesh m;
  m.V = V; m.F = F; m.nV = int(V.size() / 3); m.nF = int(F.size() / 3);
  const int nF = m.nF;
  std::vector<std::pair<int, int>> rows(3 * size_t(nF));
  for (int i = 0; i < 3; i++)
    for (int f = 0; f < nF; f++) {
      int a = F[3 * f + (i + 1) % 3], b = F[3 * f + (i + 2) % 3];
      rows[size_t(i) * nF + f] = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
    }
  std::vector<int> order(rows.size());
  for (size_t r = 0; r < order.size(); r++) order[r] = int(r);
  std::sort(order.begin(), order.end(), [&](int r, int s) {
    if (rows[r].first != rows[s].first) return rows[r].first < rows[s].first;
    if (rows[r].second != rows[s].second) return rows[r].second < rows[s].second;
    return r < s;
  });
  std::vector<int> inv(rows.size());
  int u = -1;
  for (size_t k = 0; k < order.size(); k++) {
    int r = order[k];
    if (k == 0 || rows[r] != rows[order[k - 1]]) { u++; m.E.push_back(rows[r].first); m.E.push_back(rows[r].second); }
    inv[r] = u;
  }
  m.nE = int(m.E.size() / 2);
  m.FE.assign(3 * size_t(nF), 0);
  for (int i = 0; i < 3; i++)
    for (int f = 0; f < nF; f++) m.FE[3 * f + i] = inv[size_t(i) * nF + f];
  m.EF.assign(2 * size_t(m.nE), -1);
  for (size_t r = 0; r < rows.size(); r++) {
    int e = inv[r], f = int(r % nF);
    if (m.EF[2 * e] < 0) m.EF[2 * e] = f;
    else if (m.EF[2 * e + 1] < 0) m.EF[2 * e + 1] = f;
    else throw std::runtime_error("non-manifold edge shared by more than two faces");
  }
  // face normals, edge normals (sum of the adjacent face normals, normalised), boundary flags, midpoints
  m.faceN.assign(3 * size_t(nF), 0.0);
  for (int f = 0; f < nF; f++) {
    int i = 3 * F[3 * f], j = 3 * F[3 * f + 1], k = 3 * F[3 * f + 2];
    double ux = V[j] - V[i], uy = V[j + 1] - V[i + 1], uz = V[j + 2] - V[i + 2];
    double vx = V[k] - V[i], vy = V[k + 1] - V[i + 1], vz = V[k + 2] - V[i + 2];
    double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
    double l = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (l == 0) l = 1;
    m.faceN[3 * f] = nx / l; m.faceN[3 * f + 1] = ny / l; m.faceN[3 * f + 2] = nz / l;
  }
  m.edgeN.assign(3 * size_t(m.nE), 0.0);
  for (int side = 0; side < 2; side++)
    for (int e = 0; e < m.nE; e++) {
      int f = m.EF[2 * e + side];
      if (f >= 0) for (int c = 0; c < 3; c++) m.edgeN[3 * e + c] += m.faceN[3 * f + c];
    }
  for (int e = 0; e < m.nE; e++) {
    double *n = &m.edgeN[3 * e];
    double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (l == 0) l = 1;
    for (int c = 0; c < 3; c++) n[c] /= l;
  }
  m.isB.assign(m.nE, 0);
  for (int e = 0; e < m.nE; e++) m.isB[e] = (m.EF[2 * e] < 0 || m.EF[2 * e + 1] < 0) ? 1 : 0;
  m.edgeMid.assign(3 * size_t(m.nE), 0.0);
  for (int e = 0; e < m.nE; e++)
    for (int c = 0; c < 3; c++) m.edgeMid[3 * e + c] = 0.5 * (V[3 * m.E[2 * e] + c] + V[3 * m.E[2 * e + 1] + c]);
  return m;
}

int Mesh::faceEdgeContaining(int face, int vertex, int exclude) const {
  for (int i = 0; i < 3; i++) {
    int e = FE[3 * face + i];
    if (e == exclude) continue;
    if (edgeHas(e, vertex)) return e;
  }
  throw std::runtime_error("face has no edge containing the vertex");
}

// ------------------------------------------------------------------------------------------------ topology
static inline int64_t fkey(int s, int k) { return int64_t(s) * 1048576 + k; }

const Frame &Knot::overFrame() const { return overSide ? b : a; }

static bool isOverFrame(const Knot &kn, int s, int k) {
  const Frame &f = kn.overFrame();
  return f.s == s && f.k == k;
}

// topology.js:90-149
static void traceStrands(Topology &topo) {
  const Mesh &mesh = *topo.mesh;
  const std::vector<int> &E = mesh.E;
  std::unordered_set<int64_t> visited;
  auto vkey = [](int f, int v) { return int64_t(f) * 2097152 + v; };
  std::vector<Strand> &strands = topo.strands;
  auto finish = [&](std::vector<int> edges, const std::vector<std::pair<int, int>> &segments, bool closed) {
    if (closed && edges.size() > segments.size()) edges.resize(segments.size());
    Strand st;
    st.index = int(strands.size()); st.edges = std::move(edges); st.nsegments = int(segments.size()); st.closed = closed;
    return st;
  };
  auto trace = [&](int face, int entry, int pivot, Strand &out) -> bool {
    std::vector<int> edges{entry};
    std::vector<std::pair<int, int>> segments;
    const int f0 = face, e0 = entry, p0 = pivot;
    for (;;) {
      int q = pivot;
      int p = E[2 * entry] == q ? E[2 * entry + 1] : E[2 * entry];
      int64_t key = vkey(face, p);
      if (visited.count(key)) {
        bool closed = !segments.empty() && face == f0 && entry == e0 && pivot == p0;
        if (segments.empty()) return false;
        out = finish(edges, segments, closed);
        return true;
      }
      visited.insert(key);
      segments.push_back({face, p});
      int g = mesh.faceEdgeContaining(face, p, entry);
      int nxt = mesh.otherFace(g, face);
      pivot = p; entry = g;
      if (nxt < 0) { edges.push_back(g); out = finish(edges, segments, false); return true; }
      face = nxt;
      if (face == f0 && entry == e0 && pivot == p0) { out = finish(edges, segments, true); return true; }
      edges.push_back(g);
    }
  };
  for (int e = 0; e < mesh.nE; e++) {
    if (!mesh.isB[e]) continue;
    int f = mesh.EF[2 * e] >= 0 ? mesh.EF[2 * e] : mesh.EF[2 * e + 1];
    for (int pivot : {E[2 * e], E[2 * e + 1]}) {
      Strand st;
      if (trace(f, e, pivot, st)) strands.push_back(std::move(st));
    }
  }
  for (int f = 0; f < mesh.nF; f++)
    for (int c = 0; c < 3; c++) {
      int corner = mesh.F[3 * f + c];
      if (visited.count(vkey(f, corner))) continue;
      int entry = -1;
      for (int i = 0; i < 3; i++) {
        int e = mesh.FE[3 * f + i];
        if (mesh.edgeHas(e, corner)) { entry = e; break; }
      }
      int otherV = E[2 * entry] == corner ? E[2 * entry + 1] : E[2 * entry];
      Strand st;
      if (trace(f, entry, otherV, st)) strands.push_back(std::move(st));
    }
  // knots in first-pass order (a Map keyed by edge id in the reference)
  std::unordered_map<int, std::vector<Frame>> passes;
  std::vector<int> order;
  for (const Strand &s : strands)
    for (size_t k = 0; k < s.edges.size(); k++) {
      int e = s.edges[k];
      auto it = passes.find(e);
      if (it == passes.end()) { order.push_back(e); passes[e] = {}; }
      passes[e].push_back({s.index, int(k)});
    }
  for (int e : order) {
    const std::vector<Frame> &fids = passes[e];
    if (fids.size() != 2) throw std::runtime_error("tracing invariant broken: an edge is not visited twice");
    Knot kn;
    kn.edge = e; kn.a = fids[0]; kn.b = fids[1]; kn.overSide = 0; kn.isBoundary = mesh.isB[e] != 0;
    topo.knotIndex[e] = int(topo.knots.size());
    topo.knots.push_back(kn);
    topo.frameToKnot[fkey(kn.a.s, kn.a.k)] = e;
    topo.frameToKnot[fkey(kn.b.s, kn.b.k)] = e;
  }
}

// topology.js:177-201: over_s(k) = (k + φ_s) % 2 == 0; a knot (s,i)-(t,j) needs φ_s + φ_t = i + j + 1 (mod 2)
static void assignParity(Topology &topo, int seedPhase) {
  const int n = int(topo.strands.size());
  auto mod2 = [](int x) { return ((x % 2) + 2) % 2; };
  std::vector<int> phi(n, -1);
  std::vector<std::vector<std::pair<int, int>>> adj(n);
  for (const Knot &kn : topo.knots) {
    int req = mod2(kn.a.k + kn.b.k + 1);
    adj[kn.a.s].push_back({kn.b.s, req});
    adj[kn.b.s].push_back({kn.a.s, req});
  }
  for (int root = 0; root < n; root++) {
    if (phi[root] >= 0) continue;
    phi[root] = root == 0 ? mod2(seedPhase) : 0;
    std::vector<int> dq{root};
    for (size_t head = 0; head < dq.size(); head++) {
      int s = dq[head];
      for (auto &tr : adj[s]) {
        int want = mod2(tr.second - phi[s]);
        if (phi[tr.first] < 0) { phi[tr.first] = want; dq.push_back(tr.first); }
      }
    }
  }
  topo.parityConflicts = 0;
  for (Knot &kn : topo.knots) {
    bool overS = mod2(kn.a.k + phi[kn.a.s]) == 0, overT = mod2(kn.b.k + phi[kn.b.s]) == 0;
    if (overS == overT) { kn.conflict = true; topo.parityConflicts++; kn.overSide = 0; }
    else kn.overSide = overS ? 0 : 1;
  }
}

// centripetal Catmull-Rom point between K[i1] and K[i2]; i0 / i3 may be -1 (end spans): topology.js:269-280
static V3 catmullRom(const std::vector<V3> &K, int i0, int i1, int i2, int i3, double t) {
  const V3 &P1 = K[i1], &P2 = K[i2];
  V3 P0 = i0 >= 0 ? K[i0] : sub3(scl3(P1, 2), P2);
  V3 P3 = i3 >= 0 ? K[i3] : sub3(scl3(P2, 2), P1);
  auto tj = [](double ti, const V3 &a, const V3 &b) { return ti + std::sqrt(std::max(norm3(sub3(b, a)), 1e-12)); };
  double t0 = 0.0, t1 = tj(t0, P0, P1), t2 = tj(t1, P1, P2), t3 = tj(t2, P2, P3);
  double tt = t1 + t * (t2 - t1);
  auto lerp = [tt](const V3 &a, const V3 &b, double ta, double tb) -> V3 {
    if (tb - ta < 1e-12) return a;
    return scl3(add3(scl3(a, tb - tt), scl3(b, tt - ta)), 1 / (tb - ta));
  };
  V3 A1 = lerp(P0, P1, t0, t1), A2 = lerp(P1, P2, t1, t2), A3 = lerp(P2, P3, t2, t3);
  V3 B1 = lerp(A1, A2, t0, t2), B2 = lerp(A2, A3, t1, t3);
  return lerp(B1, B2, t1, t2);
}

// topology.js:283-292
static std::vector<V3> nodeTangents(const std::vector<double> &P, bool closed) {
  const int n = int(P.size() / 3);
  auto pt = [&](int i) { return V3{P[3 * i], P[3 * i + 1], P[3 * i + 2]}; };
  std::vector<V3> T;
  if (n == 1) return {V3{0, 0, 1}};
  if (closed) {
    for (int i = 0; i < n; i++) T.push_back(normalize3(sub3(pt((i + 1) % n), pt((i - 1 + n) % n))));
    return T;
  }
  T.push_back(sub3(pt(1), pt(0)));
  for (int i = 1; i < n - 1; i++) T.push_back(add3(normalize3(sub3(pt(i + 1), pt(i))), normalize3(sub3(pt(i), pt(i - 1)))));
  T.push_back(sub3(pt(n - 1), pt(n - 2)));
  for (V3 &t : T) t = normalize3(t);
  return T;
}

// R with Z = tangent, Y = hint made orthogonal to Z, X = Y × Z, as 9 numbers [X | Y | Z]: topology.js:37-44
std::array<double, 9> frameFromTangentNormal(const V3 &t, const V3 &hint) {
  V3 z = normalize3(t);
  V3 y = sub3(hint, scl3(z, dot3(hint, z)));
  if (norm3(y) < 1e-9) {
    V3 a = std::fabs(z[0]) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0};
    y = sub3(a, scl3(z, dot3(a, z)));
  }
  y = normalize3(y);
  V3 x = cross3(y, z);
  return {x[0], x[1], x[2], y[0], y[1], y[2], z[0], z[1], z[2]};
}

static std::vector<double> nodeFrames(const std::vector<double> &P, const std::vector<V3> &hints, bool closed) {
  const int n = int(P.size() / 3);
  std::vector<double> out(9 * size_t(n));
  if (n == 1) { double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}; std::copy(I, I + 9, out.begin()); return out; }
  std::vector<V3> T = nodeTangents(P, closed);
  for (int i = 0; i < n; i++) {
    auto R = frameFromTangentNormal(T[i], hints[i]);
    std::copy(R.begin(), R.end(), out.begin() + 9 * size_t(i));
  }
  return out;
}

// topology.js:214-266
static void buildPolylines(Topology &topo, const WeaveParams &p) {
  const Mesh &mesh = *topo.mesh;
  auto mid = [&](int e) { return V3{mesh.edgeMid[3 * e], mesh.edgeMid[3 * e + 1], mesh.edgeMid[3 * e + 2]}; };
  auto en = [&](int e) { return V3{mesh.edgeN[3 * e], mesh.edgeN[3 * e + 1], mesh.edgeN[3 * e + 2]}; };
  const double h = p.half_height ? topo.thickness : 0.0;
  const int sub = std::max(1, p.subdivisions);
  auto roundHalfEven = [](double x) {
    double r = std::floor(x + 0.5);
    return std::fabs(std::fmod(x, 1.0)) == 0.5 ? 2 * std::floor(x / 2 + 0.5) : r;
  };
  for (const Strand &s : topo.strands) {
    const int nk = int(s.edges.size());
    std::vector<V3> Nn(nk), K(nk), K0(nk);
    std::vector<double> sign(nk), off(nk);
    for (int k = 0; k < nk; k++) {
      int e = s.edges[k];
      Nn[k] = en(e);
      const Knot &kn = topo.knots[topo.knotIndex.at(e)];
      sign[k] = isOverFrame(kn, s.index, k) ? 1.0 : -1.0;
      // with lath groups the knot's offset is the mean height of its two strands (topology.js:225)
      const double he = (!topo.strandThickness.empty() && p.half_height)
                            ? 0.5 * (topo.strandThickness[kn.a.s] + topo.strandThickness[kn.b.s]) : h;
      K[k] = add3(mid(e), scl3(Nn[k], 0.5 * he * sign[k]));
      K0[k] = mid(e);
      off[k] = (0.5 * h) * sign[k];
    }
    std::vector<V3> nodes, normals;
    std::vector<int> knotRows;
    if (!s.closed && p.overhang > 0 && nk > 1) {
      V3 t0 = normalize3(sub3(K[1], K[0]));
      double seg = norm3(sub3(K[1], K[0])) / sub;
      int m = std::max(1, int(roundHalfEven(p.overhang / std::max(seg, 1e-9))));
      for (int i = 0; i < m; i++) {
        double d = p.overhang * (1 - double(i) / m);
        nodes.push_back(sub3(K[0], scl3(t0, d)));
        normals.push_back(Nn[0]);
      }
    }
    const double step = 1.0 / sub;
    for (int k = 0; k < nk; k++) {
      knotRows.push_back(int(nodes.size()));
      nodes.push_back(K[k]); normals.push_back(Nn[k]);
      int nxt = k + 1 < nk ? k + 1 : (s.closed ? 0 : -1);
      if (nxt >= 0) {
        int prv = (s.closed || k > 0) ? ((k - 1) % nk + nk) % nk : -1;
        int nx2 = (s.closed || nxt + 1 < nk) ? (nxt + 1) % nk : -1;
        for (int i = 1; i < sub; i++) {
          double t = i * step;
          V3 base = catmullRom(K0, prv, k, nxt, nx2, t);
          V3 nrm = normalize3(add3(scl3(Nn[k], 1 - t), scl3(Nn[nxt], t)));
          double w = 0.5 * (1.0 + std::cos(M_PI * t));
          double o = w * off[k] + (1 - w) * off[nxt];
          nodes.push_back(add3(base, scl3(nrm, o)));
          normals.push_back(nrm);
        }
      }
    }
    if (!s.closed && p.overhang > 0 && nk > 1) {
      V3 t1 = normalize3(sub3(K[nk - 1], K[nk - 2]));
      double seg = norm3(sub3(K[nk - 1], K[nk - 2])) / sub;
      int m = std::max(1, int(roundHalfEven(p.overhang / std::max(seg, 1e-9))));
      for (int i = 1; i <= m; i++) { nodes.push_back(add3(K[nk - 1], scl3(t1, p.overhang * i / m))); normals.push_back(Nn[nk - 1]); }
    }
    std::vector<double> P(3 * nodes.size());
    for (size_t i = 0; i < nodes.size(); i++) for (int c = 0; c < 3; c++) P[3 * i + c] = nodes[i][c];
    topo.nodeFrames.push_back(nodeFrames(P, normals, s.closed));
    topo.polylines.push_back(std::move(P));
    for (int k = 0; k < nk; k++) topo.knotNode[fkey(s.index, k)] = knotRows[k];
  }
}

// np.interp on increasing integer abscissae: topology.js:302-310
static double interp(double x, const std::vector<int> &xp, const std::vector<double> &fp) {
  if (x <= xp[0]) return fp[0];
  const int last = int(xp.size()) - 1;
  if (x >= xp[last]) return fp[last];
  int lo = 0, hi = last;
  while (hi - lo > 1) { int m = (lo + hi) >> 1; if (xp[m] <= x) lo = m; else hi = m; }
  double slope = (fp[lo + 1] - fp[lo]) / double(xp[lo + 1] - xp[lo]);
  return slope * (x - xp[lo]) + fp[lo];
}

// topology.js:314-345
static void consistentFrames(Topology &topo) {
  if (!topo.mesh || topo.knots.empty()) return;
  const Mesh &mesh = *topo.mesh;
  const int S = int(topo.strands.size());
  std::vector<std::vector<V3>> tang(S);
  std::vector<std::vector<V3>> hints(S);
  std::vector<std::vector<uint8_t>> has(S);
  for (int s = 0; s < S; s++) {
    tang[s] = nodeTangents(topo.polylines[s], topo.strands[s].closed);
    hints[s].assign(topo.polylines[s].size() / 3, V3{0, 0, 0});
    has[s].assign(topo.polylines[s].size() / 3, 0);
  }
  for (const Knot &kn : topo.knots) {
    int sA = kn.a.s, sB = kn.b.s;
    int rA = topo.knotNode.at(fkey(kn.a.s, kn.a.k)), rB = topo.knotNode.at(fkey(kn.b.s, kn.b.k));
    V3 n = cross3(tang[sA][rA], tang[sB][rB]);
    double nn = norm3(n);
    V3 ref{mesh.edgeN[3 * kn.edge], mesh.edgeN[3 * kn.edge + 1], mesh.edgeN[3 * kn.edge + 2]};
    n = nn < 1e-9 ? ref : scl3(n, 1 / nn);
    if (dot3(n, ref) < 0) n = scl3(n, -1);
    hints[sA][rA] = n; has[sA][rA] = 1;
    hints[sB][rB] = n; has[sB][rB] = 1;
  }
  for (int s = 0; s < S; s++) {
    const std::vector<V3> &H = hints[s];
    std::vector<int> known;
    for (size_t i = 0; i < H.size(); i++) if (has[s][i]) known.push_back(int(i));
    if (known.empty()) continue;
    std::vector<V3> Hf(H.size());
    if (known.size() == 1) { for (auto &v : Hf) v = H[known[0]]; }
    else {
      std::vector<double> comp[3];
      for (int c = 0; c < 3; c++) for (int i : known) comp[c].push_back(H[i][c]);
      for (size_t i = 0; i < H.size(); i++) {
        if (int(i) < known[0]) Hf[i] = H[known[0]];
        else if (int(i) > known.back()) Hf[i] = H[known.back()];
        else for (int c = 0; c < 3; c++) Hf[i][c] = interp(double(i), known, comp[c]);
      }
    }
    for (auto &v : Hf) { double l = std::max(norm3(v), 1e-12); v = {v[0] / l, v[1] / l, v[2] / l}; }
    topo.nodeFrames[s] = nodeFrames(topo.polylines[s], Hf, topo.strands[s].closed);
  }
}

double Mesh::area() const {
  double a = 0;
  for (int f = 0; f < nF; f++) {
    const double *p = &V[3 * size_t(F[3 * f])], *q = &V[3 * size_t(F[3 * f + 1])], *r = &V[3 * size_t(F[3 * f + 2])];
    const double ux = q[0] - p[0], uy = q[1] - p[1], uz = q[2] - p[2], vx = r[0] - p[0], vy = r[1] - p[1], vz = r[2] - p[2];
    a += 0.5 * std::hypot(uy * vz - uz * vy, uz * vx - ux * vz, ux * vy - uy * vx);
  }
  return a;
}

Topology buildTopology(const Mesh &mesh, const WeaveParams &p, double thickness, const std::vector<double> *strandThickness) {
  Topology topo;
  topo.mesh = &mesh; topo.thickness = thickness; topo.overhang = p.overhang;
  traceStrands(topo);
  if (strandThickness) {
    // a strand the caller's table does not reach keeps the base thickness
    topo.strandThickness.assign(topo.strands.size(), thickness);
    for (size_t s = 0; s < topo.strands.size() && s < strandThickness->size(); s++) topo.strandThickness[s] = (*strandThickness)[s];
  }
  assignParity(topo, p.seed_strand_phase);
  for (auto &fk : p.flip_knots) {                           // applyFlips: topology.js:203-211
    auto it = topo.frameToKnot.find(fkey(fk.first, fk.second));
    if (it == topo.frameToKnot.end()) continue;
    Knot &kn = topo.knots[topo.knotIndex.at(it->second)];
    kn.overSide = kn.overSide ? 0 : 1;
    kn.flipped = !kn.flipped;
  }
  buildPolylines(topo, p);
  consistentFrames(topo);
  return topo;
}

// topology.js:348-363: no mesh, knots given by the caller
Topology topologyFromPolylines(const std::vector<std::vector<double>> &polylines, const std::vector<std::vector<V3>> *normals,
                               double thickness, const std::vector<std::vector<int>> *knotRows) {
  Topology topo;
  topo.mesh = nullptr; topo.thickness = thickness; topo.overhang = 0;
  for (size_t s = 0; s < polylines.size(); s++) {
    const std::vector<double> &P = polylines[s];
    const int n = int(P.size() / 3);
    std::vector<int> rows = knotRows ? (*knotRows)[s] : std::vector<int>{0, n - 1};
    std::vector<V3> nh = normals ? (*normals)[s] : std::vector<V3>(n, V3{0, 0, 1});
    Strand st;
    st.index = int(s); st.closed = false; st.nsegments = 0;
    for (size_t k = 0; k < rows.size(); k++) st.edges.push_back(-(int(s) * 1000 + int(k) + 1));
    topo.strands.push_back(st);
    topo.polylines.push_back(P);
    topo.nodeFrames.push_back(nodeFrames(P, nh, false));
    for (size_t k = 0; k < rows.size(); k++) {
      topo.knotNode[fkey(int(s), int(k))] = rows[k];
      topo.frameToKnot[fkey(int(s), int(k))] = -(int(s) * 1000 + int(k) + 1);
    }
  }
  return topo;
}

// ------------------------------------------------------------------------------------------------ state
// Shepperd with strict comparisons (the set-up version): quat.js:29-39
static void fromFrame(const std::array<double, 9> &F, double out[4]) {
  double m00 = F[0], m10 = F[1], m20 = F[2], m01 = F[3], m11 = F[4], m21 = F[5], m02 = F[6], m12 = F[7], m22 = F[8];
  double t = m00 + m11 + m22;
  if (t > 0) { double s = std::sqrt(t + 1.0) * 2; out[0] = 0.25 * s; out[1] = (m21 - m12) / s; out[2] = (m02 - m20) / s; out[3] = (m10 - m01) / s; }
  else if (m00 > m11 && m00 > m22) { double s = std::sqrt(1.0 + m00 - m11 - m22) * 2; out[0] = (m21 - m12) / s; out[1] = 0.25 * s; out[2] = (m01 + m10) / s; out[3] = (m02 + m20) / s; }
  else if (m11 > m22) { double s = std::sqrt(1.0 + m11 - m00 - m22) * 2; out[0] = (m02 - m20) / s; out[1] = (m01 + m10) / s; out[2] = 0.25 * s; out[3] = (m12 + m21) / s; }
  else { double s = std::sqrt(1.0 + m22 - m00 - m11) * 2; out[0] = (m10 - m01) / s; out[1] = (m02 + m20) / s; out[2] = (m12 + m21) / s; out[3] = 0.25 * s; }
  double n = std::sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2] + out[3] * out[3]);
  if (n == 0) n = 1.0;
  for (int k = 0; k < 4; k++) out[k] /= n;
}

// model.js:10-75
State buildState(const Topology &topo) {
  State st;
  const int S = int(topo.strands.size());
  st.S = S;
  st.nodeOffset.assign(S + 1, 0);
  for (int s = 0; s < S; s++) st.nodeOffset[s + 1] = st.nodeOffset[s] + int(topo.polylines[s].size() / 3);
  st.n = st.nodeOffset[S];
  st.X.reserve(3 * size_t(st.n));
  for (int s = 0; s < S; s++) st.X.insert(st.X.end(), topo.polylines[s].begin(), topo.polylines[s].end());
  st.nodeStrand.assign(st.n, 0);
  for (int s = 0; s < S; s++) std::fill(st.nodeStrand.begin() + st.nodeOffset[s], st.nodeStrand.begin() + st.nodeOffset[s + 1], s);
  std::vector<int> segCounts;
  int base = 0;
  for (int s = 0; s < S; s++) {
    const Strand &strand = topo.strands[s];
    const int off = st.nodeOffset[s], nn = int(topo.polylines[s].size() / 3);
    const int nseg = strand.closed ? nn : nn - 1;
    segCounts.push_back(nseg);
    const std::vector<double> &P = topo.polylines[s], &R = topo.nodeFrames[s];
    for (int k = 0; k < nseg; k++) {
      int a = k, b = (k + 1) % nn;
      st.segI0.push_back(off + a); st.segI1.push_back(off + b); st.segStrand.push_back(s);
      V3 d{P[3 * b] - P[3 * a], P[3 * b + 1] - P[3 * a + 1], P[3 * b + 2] - P[3 * a + 2]};
      st.l0.push_back(std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
      V3 hint{R[9 * a + 3] + R[9 * b + 3], R[9 * a + 4] + R[9 * b + 4], R[9 * a + 5] + R[9 * b + 5]};
      double q[4];
      fromFrame(frameFromTangentNormal(d, hint), q);
      st.Q.insert(st.Q.end(), q, q + 4);
    }
    if (strand.closed)
      for (int k = 0; k < nseg; k++) { st.jSeg0.push_back(base + k); st.jSeg1.push_back(base + (k + 1) % nseg); st.jNode.push_back(off + (k + 1) % nn); }
    else
      for (int k = 0; k < std::max(nseg - 1, 0); k++) { st.jSeg0.push_back(base + k); st.jSeg1.push_back(base + k + 1); st.jNode.push_back(off + 1 + k); }
    base += nseg;
  }
  st.segOffset.assign(S + 1, 0);
  for (int s = 0; s < S; s++) st.segOffset[s + 1] = st.segOffset[s] + segCounts[s];
  st.m = st.segOffset[S]; st.p = int(st.jSeg0.size());
  st.jLen.resize(st.p);
  for (int j = 0; j < st.p; j++) st.jLen[j] = 0.5 * (st.l0[st.jSeg0[j]] + st.l0[st.jSeg1[j]]);
  // contacts: knots in sorted edge order, u = node row of the knot, n_prev = A -> B
  for (const Knot &kn : topo.knots) st.knotEdges.push_back(kn.edge);
  std::sort(st.knotEdges.begin(), st.knotEdges.end());
  st.K = int(st.knotEdges.size());
  for (auto &kv : topo.knotNode) {
    int s = int(kv.first / 1048576);
    st.nodeFrameIds[kv.first] = st.nodeOffset[s] + kv.second;
  }
  st.u.assign(2 * size_t(st.K), 0.0); st.nPrev.assign(3 * size_t(st.K), 0.0);
  st.crossStrand.assign(2 * size_t(st.K), 0);
  for (int c = 0; c < st.K; c++) {
    const Knot &kn = topo.knots[topo.knotIndex.at(st.knotEdges[c])];
    const Frame fr[2] = {kn.a, kn.b};
    for (int side = 0; side < 2; side++) {
      int s = fr[side].s, row = topo.knotNode.at(fkey(fr[side].s, fr[side].k));
      int nseg = st.segOffset[s + 1] - st.segOffset[s];
      st.u[2 * c + side] = std::min(row, nseg);
      st.crossStrand[2 * c + side] = s;
    }
    int ia = st.nodeFrameIds.at(fkey(kn.a.s, kn.a.k)), ib = st.nodeFrameIds.at(fkey(kn.b.s, kn.b.k));
    V3 d{st.X[3 * ib] - st.X[3 * ia], st.X[3 * ib + 1] - st.X[3 * ia + 1], st.X[3 * ib + 2] - st.X[3 * ia + 2]};
    double nd = norm3(d);
    for (int k = 0; k < 3; k++)
      st.nPrev[3 * c + k] = nd > 1e-12 ? d[k] / nd : (topo.mesh ? topo.mesh->edgeN[3 * kn.edge + k] : 0.0);
    st.crossBoundary.push_back(kn.isBoundary ? 1 : 0);
  }
  st.X0 = st.X;
  return st;
}

// ------------------------------------------------------------------------------------------------ sections
// params.js:33-45 (section axes: X = width, Y = normal, Z = tangent)
double rectTorsionConstant(double a, double b) {
  if (a < b) std::swap(a, b);
  double r = b / a;
  return a * b * b * b * (1.0 / 3.0 - 0.21 * r * (1.0 - r * r * r * r / 12.0));
}
Section sectionStiffness(double w, double h, double E, double G) {
  Section s;
  double A = w * h;
  s.EA = E * A; s.EIx = E * w * h * h * h / 12.0; s.EIy = E * h * w * w * w / 12.0;
  s.GJ = G * rectTorsionConstant(w, h); s.GA = (5.0 / 6.0) * G * A;
  return s;
}
static const double G_SI = 9.80665;

// ------------------------------------------------------------------------------------------------ scene assembly
void Scene::fillModel() {
  ws_model &m = model;
  std::memset(&m, 0, sizeof(m));
  m.n = st.n; m.m = st.m; m.p = st.p; m.n_strands = st.S; m.K = st.K;
  m.X = st.X.data(); m.X0 = st.X0.data(); m.Q = st.Q.data(); m.l0 = st.l0.data();
  m.seg_i0 = st.segI0.data(); m.seg_i1 = st.segI1.data(); m.seg_offset = st.segOffset.data();
  m.joint_seg0 = st.jSeg0.data(); m.joint_seg1 = st.jSeg1.data(); m.joint_len = st.jLen.data();
  m.omega0 = omega0.empty() ? nullptr : omega0.data();
  m.EA = EA.data(); m.EIx = EIx.data(); m.EIy = EIy.data(); m.GJ = GJ.data(); m.GA = GA.data();
  m.load_const = loadConst.data();
  m.n_local_loads = int(localNode.size()); m.local_load_node = localNode.data(); m.local_load_F = localF.data();
  m.n_anchors = int(anchorNode.size()); m.anchor_node = anchorNode.data(); m.anchor_mask = anchorMask.data();
  m.anchor_target = anchorTarget.size() == 3 * anchorNode.size() && !anchorTarget.empty() ? anchorTarget.data() : nullptr;
  m.cross_strand = st.crossStrand.data(); m.cross_wk = wk.data(); m.cross_hk = hk.data();
  m.cross_u = st.u.data(); m.cross_nprev = st.nPrev.data();
  m.cross_enabled = enabled.data(); m.cross_locked = locked.data(); m.cross_mu = mu.data();
  m.cross_fc90 = fc90.size() == 2 * size_t(st.K) && st.K ? fc90.data() : nullptr;
  m.cross_E90 = E90.size() == 2 * size_t(st.K) && st.K ? E90.data() : nullptr;
  m.cross_H = H.size() == 2 * size_t(st.K) && st.K ? H.data() : nullptr;
  m.node_w = nodeW.size() == size_t(st.n) ? nodeW.data() : nullptr;
  m.node_h = nodeH.size() == size_t(st.n) ? nodeH.data() : nullptr;
  m.params = params;
}

// uniform section and material for every segment and crossing side; self-weight half to each end node (model.js:200-212)
void Scene::setUniformSection(double w, double h, double E, double G, double density, bool gravity) {
  Section s = sectionStiffness(w, h, E, G);
  EA.assign(st.m, s.EA); EIx.assign(st.m, s.EIx); EIy.assign(st.m, s.EIy); GJ.assign(st.m, s.GJ); GA.assign(st.m, s.GA);
  wk.assign(2 * size_t(st.K), w); hk.assign(2 * size_t(st.K), h);
  // across the grain, in the proportions of the reference's default timber (params.js:6: E 10000, fc90 8, E90 800,
  // H 30), so that any unit system of E carries over
  fc90.assign(2 * size_t(st.K), 8e-4 * E); E90.assign(2 * size_t(st.K), 0.08 * E); H.assign(2 * size_t(st.K), 3e-3 * E);
  nodeW.assign(st.n, w); nodeH.assign(st.n, h);
  loadConst.assign(3 * size_t(st.n), 0.0);
  if (gravity) {
    const double g[3] = {0.0, 0.0, -1.0};
    const double qline = density * (w * h) * G_SI;         // UnitSystem.selfWeightLineLoad in m, N (units.js:21-25)
    for (int j = 0; j < st.m; j++) {
      double q = 0.5 * st.l0[j] * qline;
      for (int i : {st.segI0[j], st.segI1[j]})
        for (int c = 0; c < 3; c++) loadConst[3 * size_t(i) + c] += q * g[c];
    }
  }
}

// anchorMasks: union of the masks per frame, in resolution order (model.js:150-159), then frame -> node
void Scene::addAnchorFrames(const std::vector<std::pair<int, int>> &frames, uint8_t mask) {
  for (auto &fr : frames) {
    auto it = st.nodeFrameIds.find(fkey(fr.first, fr.second));
    if (it == st.nodeFrameIds.end()) continue;
    int nid = it->second;
    auto pos = std::find(anchorNode.begin(), anchorNode.end(), nid);
    if (pos == anchorNode.end()) { anchorNode.push_back(nid); anchorMask.push_back(mask); }
    else anchorMask[pos - anchorNode.begin()] |= mask;
  }
}

void Scene::addPointLoad(int s, int k, const double F[3], bool local) {
  auto it = st.nodeFrameIds.find(fkey(s, k));
  if (it == st.nodeFrameIds.end()) return;
  int nid = it->second;
  if (local) { localNode.push_back(nid); localF.insert(localF.end(), F, F + 3); }
  else for (int c = 0; c < 3; c++) loadConst[3 * size_t(nid) + c] += F[c];
}

double Scene::span() const {
  double lo[2] = {1e300, 1e300}, hi[2] = {-1e300, -1e300};
  for (int i = 0; i < st.n; i++)
    for (int c = 0; c < 2; c++) { lo[c] = std::min(lo[c], st.X0[3 * size_t(i) + c]); hi[c] = std::max(hi[c], st.X0[3 * size_t(i) + c]); }
  return st.n ? std::max(hi[0] - lo[0], hi[1] - lo[1]) : 0.0;
}

// hexagonal patch of the triangular lattice with basis e1 = (a, 0), e2 = (a/2, a√3/2): vertices with
// |i|, |j|, |i + j| <= side; counter-clockwise up and down triangles (the tri_lattice pattern, make_meshes.py:13-29)
Mesh hexLatticeMesh(int side, double a) {
  std::vector<double> V;
  std::map<std::pair<int, int>, int> id;
  for (int j = -side; j <= side; j++)
    for (int i = -side; i <= side; i++) {
      if (std::abs(i + j) > side) continue;
      id[{i, j}] = int(V.size() / 3);
      V.push_back(a * (i + 0.5 * j)); V.push_back(a * j * std::sqrt(3.0) / 2); V.push_back(0.0);
    }
  std::vector<int> F;
  auto has = [&](int i, int j) { return id.count({i, j}) > 0; };
  for (int j = -side; j <= side; j++)
    for (int i = -side; i <= side; i++) {
      if (has(i, j) && has(i + 1, j) && has(i, j + 1)) { F.push_back(id[{i, j}]); F.push_back(id[{i + 1, j}]); F.push_back(id[{i, j + 1}]); }
      if (has(i + 1, j) && has(i + 1, j + 1) && has(i, j + 1)) { F.push_back(id[{i + 1, j}]); F.push_back(id[{i + 1, j + 1}]); F.push_back(id[{i, j + 1}]); }
    }
  return Mesh::fromArrays(V, F);
}

Scene *buildKagome(const ws_kagome_cfg &cfg) {
  if (cfg.side < 1 || cfg.subdivisions < 1 || !(cfg.edge > 0) || !(cfg.width > 0) || !(cfg.height > 0))
    throw std::invalid_argument("kagome: side, subdivisions, edge, width and height must be positive");
  auto sc = std::make_unique<Scene>();
  sc->mesh = hexLatticeMesh(cfg.side, cfg.edge);
  WeaveParams wp;
  wp.subdivisions = cfg.subdivisions; wp.overhang = 0.0; wp.half_height = true; wp.seed_strand_phase = 0;
  sc->topo = buildTopology(sc->mesh, wp, cfg.height);
  sc->st = buildState(sc->topo);
  State &st = sc->st;
  sc->params = cfg.params;
  sc->setUniformSection(cfg.width, cfg.height, cfg.E, cfg.G, cfg.density, cfg.gravity != 0);
  // anchors: all_start + all_end, translations fixed (dome_basic.json anchors)
  std::vector<std::pair<int, int>> starts, ends;
  for (const Strand &s : sc->topo.strands)
    if (!s.closed) { starts.push_back({s.index, 0}); ends.push_back({s.index, int(s.edges.size()) - 1}); }
  sc->addAnchorFrames(starts, 0x7);
  sc->addAnchorFrames(ends, 0x7);
  // crossings: boundary knots carry no contact without overhang (solver_cpu.js:83)
  sc->enabled.assign(st.K, 1);
  for (int c = 0; c < st.K; c++) if (st.crossBoundary[c]) sc->enabled[c] = 0;
  sc->locked.assign(st.K, 0);
  Rng rng(cfg.seed);
  // 1) z-noise of every node
  if (cfg.z_noise > 0) for (int i = 0; i < st.n; i++) st.X[3 * size_t(i) + 2] += cfg.z_noise * rng.normal();
  // 2) friction per crossing
  sc->mu.assign(st.K, cfg.mu);
  if (cfg.mu_hi > cfg.mu_lo) for (int c = 0; c < st.K; c++) sc->mu[c] = cfg.mu_lo + (cfg.mu_hi - cfg.mu_lo) * rng.uniform();
  // anchor targets start at the anchored nodes (they stay unless a prescribed motion is set below)
  sc->anchorTarget.resize(3 * sc->anchorNode.size());
  for (size_t a = 0; a < sc->anchorNode.size(); a++)
    for (int c = 0; c < 3; c++) sc->anchorTarget[3 * a + c] = st.X[3 * size_t(sc->anchorNode[a]) + c];
  // 3) prescribed inward motion of the perimeter ends: the targets are the anchored nodes scaled in plan about the
  //    centre so that the ends move `inward` on average; the laths start flat and buckle as the supports move in
  //    (params.disp_ramp_iter)
  if (cfg.inward != 0 && !sc->anchorNode.empty()) {
    double R = 0;
    for (int nid : sc->anchorNode) R += std::hypot(st.X[3 * size_t(nid)], st.X[3 * size_t(nid) + 1]);
    R /= sc->anchorNode.size();
    double lam = 1.0 - cfg.inward / R;
    for (size_t a = 0; a < sc->anchorNode.size(); a++) { sc->anchorTarget[3 * a] *= lam; sc->anchorTarget[3 * a + 1] *= lam; }
  }
  // 4) supports lifted 0..lift by a smooth seeded field (a few long waves)
  if (cfg.lift > 0 && !sc->anchorNode.empty()) {
    double span = sc->span();
    const int NW = 4;
    double kx[NW], ky[NW], ph[NW], am[NW];
    for (int w = 0; w < NW; w++) {
      double ang = 2 * M_PI * rng.uniform(), lam = span * (0.75 + 1.25 * rng.uniform());
      kx[w] = 2 * M_PI / lam * std::cos(ang); ky[w] = 2 * M_PI / lam * std::sin(ang);
      ph[w] = 2 * M_PI * rng.uniform(); am[w] = 0.5 + rng.uniform();
    }
    auto field = [&](double x, double y) { double f = 0; for (int w = 0; w < NW; w++) f += am[w] * std::cos(kx[w] * x + ky[w] * y + ph[w]); return f; };
    double fmin = 1e300, fmax = -1e300;
    for (int nid : sc->anchorNode) { double f = field(st.X[3 * size_t(nid)], st.X[3 * size_t(nid) + 1]); fmin = std::min(fmin, f); fmax = std::max(fmax, f); }
    double sc_ = fmax > fmin ? cfg.lift / (fmax - fmin) : 0.0;
    for (size_t a = 0; a < sc->anchorNode.size(); a++) {
      const int nid = sc->anchorNode[a];
      sc->anchorTarget[3 * a + 2] += sc_ * (field(st.X[3 * size_t(nid)], st.X[3 * size_t(nid) + 1]) - fmin);
    }
  }
  sc->fillModel();
  return sc.release();
}

// rotation vector log(q_a* ⊗ q_b) of two unit quaternions, the short way round (relRotation, rod_cosserat.js:33-45)
static void relRotationVec(const double *qa, const double *qb, double out[3]) {
  const double aw = qa[0], ax = -qa[1], ay = -qa[2], az = -qa[3];
  const double bw = qb[0], bx = qb[1], by = qb[2], bz = qb[3];
  double w = aw * bw - ax * bx - ay * by - az * bz, x = aw * bx + ax * bw + ay * bz - az * by;
  double y = aw * by - ax * bz + ay * bw + az * bx, z = aw * bz + ax * by - ay * bx + az * bw;
  if (w < 0) { w = -w; x = -x; y = -y; z = -z; }
  const double s = std::sqrt(x * x + y * y + z * z), th = 2 * std::atan2(s, w);
  const double f = s > 1e-12 ? th / s : 2 / std::max(w, 1e-12);
  out[0] = f * x; out[1] = f * y; out[2] = f * z;
}

// a scene from a triangle mesh and the parameters of a scene.json (Scene.fromJSON + CpuSolver set-up, scene.js:142-190,
// model.js:112-252): the topology of the mesh, uniform section and material, selectors resolved to frames, loads
Scene *buildMeshScene(const ws_mesh_cfg &cfg) {
  if (cfg.n_vertices < 3 || cfg.n_faces < 1 || !cfg.vertices || !cfg.faces) throw std::invalid_argument("mesh: no triangles");
  if (cfg.subdivisions < 1 || !(cfg.width > 0) || !(cfg.height > 0)) throw std::invalid_argument("mesh: subdivisions and section must be positive");
  for (int i = 0; i < 3 * cfg.n_faces; i++)
    if (cfg.faces[i] < 0 || cfg.faces[i] >= cfg.n_vertices) throw std::invalid_argument("mesh: face vertex out of range");
  auto sc = std::make_unique<Scene>();
  sc->mesh = Mesh::fromArrays(std::vector<double>(cfg.vertices, cfg.vertices + 3 * size_t(cfg.n_vertices)),
                              std::vector<int>(cfg.faces, cfg.faces + 3 * size_t(cfg.n_faces)));
  WeaveParams wp;
  wp.subdivisions = cfg.subdivisions; wp.overhang = cfg.overhang; wp.half_height = cfg.half_height != 0;
  wp.seed_strand_phase = cfg.seed_strand_phase;
  for (int f = 0; f < cfg.n_flips; f++) wp.flip_knots.push_back({cfg.flips[2 * f], cfg.flips[2 * f + 1]});
  // lath groups: group 0 is the cfg's own section and material, group g >= 1 is cfg.groups[g - 1] (the scene's group
  // g + 1); the strands' groups from the assignments (an assignment out of range leaves the strand in group 0)
  ws_lath_group base{};
  base.width = cfg.width; base.height = cfg.height;
  base.EA = cfg.EA; base.EIx = cfg.EIx; base.EIy = cfg.EIy; base.GJ = cfg.GJ; base.GA = cfg.GA;
  for (int k = 0; k < 3; k++) base.activation[k] = cfg.activation[k];
  base.line_weight = cfg.line_weight; base.fc90 = cfg.fc90; base.E90 = cfg.E90; base.H = cfg.H;
  std::vector<ws_lath_group> groups{base};
  if (cfg.n_groups > 0) {
    if (!cfg.groups) throw std::invalid_argument("mesh: lath groups without their table");
    for (int g = 0; g < cfg.n_groups; g++) {
      const ws_lath_group &G = cfg.groups[g];
      if (!(G.width > 0) || !(G.height > 0)) throw std::invalid_argument("mesh: a lath group's section must be positive");
      groups.push_back(G);
    }
  }
  std::vector<int> strandAssign;         // by strand index: group (0 = base)
  int maxStrand = -1;
  for (int i = 0; i < cfg.n_assign; i++) maxStrand = std::max(maxStrand, cfg.assign_strand[i]);
  strandAssign.assign(size_t(maxStrand + 1), 0);
  for (int i = 0; i < cfg.n_assign; i++) {
    const int s = cfg.assign_strand[i], g = cfg.assign_group[i];
    if (s >= 0 && g >= 2 && g - 1 < int(groups.size())) strandAssign[s] = g - 1;
  }
  std::vector<double> thick;
  if (groups.size() > 1)
    for (size_t s = 0; s < strandAssign.size(); s++) thick.push_back(groups[strandAssign[s]].height);
  sc->topo = buildTopology(sc->mesh, wp, cfg.height, groups.size() > 1 ? &thick : nullptr);
  sc->st = buildState(sc->topo);
  State &st = sc->st;
  sc->params = cfg.params;
  auto grpOf = [&](int strand) -> const ws_lath_group & {
    return groups[strand >= 0 && strand < int(strandAssign.size()) ? strandAssign[strand] : 0];
  };
  // section and material per segment, crossing side and node (strandStiffness, model.js:236-252; the contact's secOf
  // and matOf, solver_cpu.js:682-684; the ground's node sections, solver_cpu.js:560)
  sc->EA.resize(st.m); sc->EIx.resize(st.m); sc->EIy.resize(st.m); sc->GJ.resize(st.m); sc->GA.resize(st.m);
  for (int j = 0; j < st.m; j++) {
    const ws_lath_group &G = grpOf(st.segStrand[j]);
    sc->EA[j] = G.EA; sc->EIx[j] = G.EIx; sc->EIy[j] = G.EIy; sc->GJ[j] = G.GJ; sc->GA[j] = G.GA;
  }
  sc->wk.resize(2 * size_t(st.K)); sc->hk.resize(2 * size_t(st.K));
  sc->fc90.resize(2 * size_t(st.K)); sc->E90.resize(2 * size_t(st.K)); sc->H.resize(2 * size_t(st.K));
  for (size_t q = 0; q < 2 * size_t(st.K); q++) {
    const ws_lath_group &G = grpOf(st.crossStrand[q]);
    sc->wk[q] = G.width; sc->hk[q] = G.height; sc->fc90[q] = G.fc90; sc->E90[q] = G.E90; sc->H[q] = G.H;
  }
  sc->nodeW.resize(st.n); sc->nodeH.resize(st.n);
  for (int i = 0; i < st.n; i++) { sc->nodeW[i] = grpOf(st.nodeStrand[i]).width; sc->nodeH[i] = grpOf(st.nodeStrand[i]).height; }
  // rest curvature: the unprestressed share of the as-built curvature (CosseratRod constructor, rod_cosserat.js:58-66),
  // each joint with the activation of its first segment's group
  bool prestress = false;
  for (const ws_lath_group &G : groups) prestress = prestress || G.activation[0] < 1 || G.activation[1] < 1 || G.activation[2] < 1;
  if (prestress) {
    sc->omega0.assign(3 * size_t(st.p), 0.0);
    for (int j = 0; j < st.p; j++) {
      double psi[3];
      relRotationVec(&st.Q[4 * size_t(st.jSeg0[j])], &st.Q[4 * size_t(st.jSeg1[j])], psi);
      const ws_lath_group &G = grpOf(st.segStrand[st.jSeg0[j]]);
      for (int k = 0; k < 3; k++) {
        const double a = std::min(std::max(G.activation[k], 0.0), 1.0);
        sc->omega0[3 * size_t(j) + k] = (1.0 - a) * (psi[k] / st.jLen[j]);
      }
    }
  }
  // loads (Loads, model.js:191-231): self-weight per segment (its group's) half to each end node, udl on the
  // tributary lengths (per length) or the mesh's area shared in proportion to them (per area), point loads at frames
  sc->loadConst.assign(3 * size_t(st.n), 0.0);
  bool weight = false;
  for (const ws_lath_group &G : groups) weight = weight || G.line_weight != 0;
  if (weight) {
    double g[3] = {cfg.gravity_dir[0], cfg.gravity_dir[1], cfg.gravity_dir[2]};
    const double gl = std::max(std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]), 1e-12);
    for (double &v : g) v /= gl;
    for (int j = 0; j < st.m; j++) {
      const double q = 0.5 * st.l0[j] * grpOf(st.segStrand[j]).line_weight;
      for (int i : {st.segI0[j], st.segI1[j]})
        for (int c = 0; c < 3; c++) sc->loadConst[3 * size_t(i) + c] += q * g[c];
    }
  }
  if (cfg.udl_on) {
    std::vector<double> trib(st.n, 0.0);
    for (int j = 0; j < st.m; j++) trib[st.segI0[j]] += 0.5 * st.l0[j];
    for (int j = 0; j < st.m; j++) trib[st.segI1[j]] += 0.5 * st.l0[j];
    if (cfg.udl_on == 1) {
      for (int i = 0; i < st.n; i++) for (int c = 0; c < 3; c++) sc->loadConst[3 * size_t(i) + c] += trib[i] * cfg.udl[c];
    } else {
      const double area = sc->mesh.area();
      double total = 0;
      for (int i = 0; i < st.n; i++) total += trib[i];
      for (int i = 0; i < st.n; i++) {
        const double w = trib[i] / std::max(total, 1e-12) * area;
        for (int c = 0; c < 3; c++) sc->loadConst[3 * size_t(i) + c] += w * cfg.udl[c];
      }
    }
  }
  for (int l = 0; l < cfg.n_loads; l++)
    sc->addPointLoad(cfg.load_frames[2 * l], cfg.load_frames[2 * l + 1], &cfg.load_F[3 * l], cfg.load_local && cfg.load_local[l]);
  // anchors: selectors to frames (resolveSelector / anchorMasks, model.js:114-159)
  for (int a = 0; a < cfg.n_anchors; a++) {
    std::vector<std::pair<int, int>> fr;
    const int kind = cfg.anchor_kind[a], s = cfg.anchor_id[2 * a], k = cfg.anchor_id[2 * a + 1];
    switch (kind) {
      case WS_SEL_FRAME: fr.push_back({s, k}); break;
      case WS_SEL_ALL_START: case WS_SEL_ALL_END: case WS_SEL_ALL_ENDS:
        if (kind != WS_SEL_ALL_END) for (const Strand &t : sc->topo.strands) if (!t.closed) fr.push_back({t.index, 0});
        if (kind != WS_SEL_ALL_START) for (const Strand &t : sc->topo.strands) if (!t.closed) fr.push_back({t.index, int(t.edges.size()) - 1});
        break;
      case WS_SEL_STRAND:
        if (s < 0 || s >= int(sc->topo.strands.size())) throw std::invalid_argument("mesh: anchor strand out of range");
        for (size_t q = 0; q < sc->topo.strands[s].edges.size(); q++) fr.push_back({s, int(q)});
        break;
      case WS_SEL_BOUNDARY:
        for (const Knot &kn : sc->topo.knots) if (kn.isBoundary) { fr.push_back({kn.a.s, kn.a.k}); fr.push_back({kn.b.s, kn.b.k}); }
        break;
      default: throw std::invalid_argument("mesh: unknown anchor selector");
    }
    sc->addAnchorFrames(fr, cfg.anchor_mask[a]);
  }
  // crossings: without overhang the boundary knots carry no contact (solver_cpu.js:83); one μ
  sc->enabled.assign(st.K, 1);
  if (cfg.overhang <= 0) for (int c = 0; c < st.K; c++) if (st.crossBoundary[c]) sc->enabled[c] = 0;
  sc->locked.assign(st.K, 0);            // contact.locked: the caller sets cross_locked
  sc->mu.assign(st.K, cfg.mu);
  sc->fillModel();
  return sc.release();
}

Scene *buildPolylineScene(const ws_polyline_cfg &cfg) {
  if (cfg.n_strands < 1 || !cfg.node_count || !cfg.points) throw std::invalid_argument("polylines: no strands");
  auto sc = std::make_unique<Scene>();
  std::vector<std::vector<double>> P(cfg.n_strands);
  std::vector<std::vector<V3>> N(cfg.n_strands);
  std::vector<std::vector<int>> rows(cfg.n_strands);
  size_t o = 0, ko = 0;
  for (int s = 0; s < cfg.n_strands; s++) {
    int nn = cfg.node_count[s];
    if (nn < 2) throw std::invalid_argument("polylines: a strand needs two nodes");
    P[s].assign(cfg.points + 3 * o, cfg.points + 3 * (o + nn));
    for (int i = 0; i < nn; i++)
      N[s].push_back(cfg.normals ? V3{cfg.normals[3 * (o + i)], cfg.normals[3 * (o + i) + 1], cfg.normals[3 * (o + i) + 2]} : V3{0, 0, 1});
    if (cfg.knot_count) {
      for (int k = 0; k < cfg.knot_count[s]; k++) {
        int r = cfg.knot_rows[ko + k];
        if (r < 0 || r >= nn) throw std::invalid_argument("polylines: knot row outside the strand");
        rows[s].push_back(r);
      }
      ko += cfg.knot_count[s];
    } else rows[s] = {0, nn - 1};
    o += nn;
  }
  sc->topo = topologyFromPolylines(P, &N, cfg.thickness, &rows);
  for (int i = 0; i < cfg.n_knots; i++) {
    Knot kn;
    kn.edge = i; kn.a = {cfg.knots[4 * i], cfg.knots[4 * i + 1]}; kn.b = {cfg.knots[4 * i + 2], cfg.knots[4 * i + 3]};
    kn.overSide = 1; kn.isBoundary = false;
    if (!sc->topo.frameToKnot.count(fkey(kn.a.s, kn.a.k)) || !sc->topo.frameToKnot.count(fkey(kn.b.s, kn.b.k)))
      throw std::invalid_argument("polylines: a knot names a frame that does not exist");
    sc->topo.knotIndex[i] = int(sc->topo.knots.size());
    sc->topo.knots.push_back(kn);
    sc->topo.frameToKnot[fkey(kn.a.s, kn.a.k)] = i;
    sc->topo.frameToKnot[fkey(kn.b.s, kn.b.k)] = i;
  }
  sc->st = buildState(sc->topo);
  sc->params = cfg.params;
  sc->setUniformSection(cfg.width, cfg.height, cfg.E, cfg.G, cfg.density, cfg.gravity != 0);
  for (int i = 0; i < cfg.n_anchors; i++)
    sc->addAnchorFrames({{cfg.anchor_frames[2 * i], cfg.anchor_frames[2 * i + 1]}}, cfg.anchor_masks[i]);
  for (int i = 0; i < cfg.n_loads; i++)
    sc->addPointLoad(cfg.load_frames[2 * i], cfg.load_frames[2 * i + 1], cfg.load_F + 3 * i, cfg.load_local && cfg.load_local[i]);
  sc->enabled.assign(sc->st.K, 1);
  sc->locked.assign(sc->st.K, 0);
  sc->mu.assign(sc->st.K, cfg.mu);
  sc->fillModel();
  return sc.release();
}

}  // namespace wsb
