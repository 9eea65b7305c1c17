// Internal types of the scene builder (scene.cpp).
#pragma once
#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <unordered_map>
#include <vector>

#include "../../include/weavesim.h"

namespace wsb {

using V3 = std::array<double, 3>;

// xoshiro128** seeded by splitmix32 (web/js/rng.js:4-27)
struct Rng {
  uint32_t s[4];
  bool has_spare = false;
  double spare = 0;
  explicit Rng(uint32_t seed);
  uint32_t u32();
  double uniform();
  double normal();
};

struct Mesh {
  int nV = 0, nF = 0, nE = 0;
  std::vector<double> V, faceN, edgeN, edgeMid;
  std::vector<int> F, E, FE, EF;
  std::vector<uint8_t> isB;
  static Mesh fromArrays(const std::vector<double> &V, const std::vector<int> &F);
  int otherFace(int edge, int face) const { int a = EF[2 * edge], b = EF[2 * edge + 1]; return a == face ? b : a; }
  bool edgeHas(int e, int v) const { return E[2 * e] == v || E[2 * e + 1] == v; }
  int faceEdgeContaining(int face, int vertex, int exclude) const;
  double area() const;                         // sum of the triangles' areas (Mesh.area, mesh.js:50-58)
};

struct Frame { int s = 0, k = 0; };
struct Knot {
  int edge = 0;
  Frame a, b;
  int overSide = 0;
  bool conflict = false, flipped = false, isBoundary = false;
  const Frame &overFrame() const;
};
struct Strand {
  int index = 0;
  std::vector<int> edges;
  int nsegments = 0;
  bool closed = false;
};
struct WeaveParams {
  int subdivisions = 4;
  double overhang = 0.0;
  bool half_height = true;
  int seed_strand_phase = 0;
  std::vector<std::pair<int, int>> flip_knots;
};
struct Topology {
  const Mesh *mesh = nullptr;
  double thickness = 0, overhang = 0;
  std::vector<double> strandThickness;         // per strand (lath groups); empty: `thickness` for every strand
  std::vector<Strand> strands;
  std::vector<Knot> knots;                     // first-pass (Map insertion) order
  std::unordered_map<int, int> knotIndex;      // edge -> index in knots
  std::unordered_map<int64_t, int> frameToKnot;
  std::vector<std::vector<double>> polylines, nodeFrames;
  std::map<int64_t, int> knotNode;             // fkey -> node row
  int parityConflicts = 0;
};
struct State {
  int S = 0, n = 0, m = 0, p = 0, K = 0;
  std::vector<double> X, X0, Q, l0, jLen, u, nPrev;
  std::vector<int> nodeOffset, nodeStrand, segI0, segI1, segStrand, segOffset, jSeg0, jSeg1, jNode, knotEdges, crossStrand;
  std::vector<uint8_t> crossBoundary;
  std::map<int64_t, int> nodeFrameIds;
};
struct Section { double EA, EIx, EIy, GJ, GA; };

Mesh hexLatticeMesh(int side, double a);
Topology buildTopology(const Mesh &mesh, const WeaveParams &p, double thickness,
                       const std::vector<double> *strandThickness = nullptr);
Topology topologyFromPolylines(const std::vector<std::vector<double>> &polylines, const std::vector<std::vector<V3>> *normals,
                               double thickness, const std::vector<std::vector<int>> *knotRows);
State buildState(const Topology &topo);
std::array<double, 9> frameFromTangentNormal(const V3 &t, const V3 &hint);
double rectTorsionConstant(double a, double b);
Section sectionStiffness(double w, double h, double E, double G);

// a scene owns the arrays that its ws_model view points into
struct Scene {
  Mesh mesh;
  Topology topo;
  State st;
  std::vector<double> EA, EIx, EIy, GJ, GA, omega0, loadConst, localF, wk, hk, mu, anchorTarget;
  std::vector<double> fc90, E90, H;          // [2K] timber of each crossing side across the grain
  std::vector<double> nodeW, nodeH;          // [n] section at every node (the ground's clearance)
  std::vector<int> localNode, anchorNode;
  std::vector<uint8_t> anchorMask, enabled, locked;
  ws_params params{};
  ws_model model{};
  void fillModel();
  void setUniformSection(double w, double h, double E, double G, double density, bool gravity);
  void addAnchorFrames(const std::vector<std::pair<int, int>> &frames, uint8_t mask);
  void addPointLoad(int s, int k, const double F[3], bool local);
  double span() const;
};

Scene *buildKagome(const ws_kagome_cfg &cfg);
Scene *buildPolylineScene(const ws_polyline_cfg &cfg);
Scene *buildMeshScene(const ws_mesh_cfg &cfg);

}  // namespace wsb

struct ws_scene { wsb::Scene *sc; };
