// Host-side goal assembly of one instance (f64): everything the device step needs that is built once per model or per
// warm start — node masses and static frame inertias (CpuSolver._buildGoals, web/js/solver_cpu.js:670-710), clamp
// joints (CosseratRod.setClamps, web/js/rod_cosserat.js:92-100), anchors (Anchors, web/js/model.js:162-189), the
// contact initialisation (PolylineContact.initialize, web/js/solver_cpu.js:99-139) and the static gather tables
// (segment -> joints / clamps, node -> segments, crossing sides sorted along their strand).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/weavesim.h"

namespace wsb {

struct HostGoals {
  // sizes
  int n = 0, m = 0, p = 0, S = 0, K = 0, C = 0;
  ws_params prm{};
  // state (f64)
  std::vector<double> X, X0, Q, u, nPrev;
  // rod
  std::vector<double> l0, jLen, omega0, EA, GA, EIx, EIy, GJ;   // EIx/EIy/GJ per joint (joint's first segment)
  std::vector<int> segI0, segI1, jSeg0, jSeg1, segOffset;
  // clamps (rotation anchors): segment, half length, per-axis stiffness, frozen frame, node
  std::vector<int> cSeg, cNode;
  std::vector<double> cLen, cB, cQ;
  // loads
  std::vector<double> loadConst, loadLocal;          // loadLocal [3n]: node-frame force (zero where none)
  std::vector<uint8_t> hasLocal;
  // anchors
  std::vector<uint8_t> nodeFree;                     // [3n] 1 = free
  std::vector<uint8_t> fixedAny;                     // [n]
  std::vector<int> ancIndex;                         // [n] -> prescribed-motion slot or -1
  std::vector<double> ancStart, ancDelta;            // [3 * slots]
  // contact
  std::vector<int> cxSegOff, cxNseg, cxStrand;       // [2K] first segment, segment count and strand of each side
  std::vector<int> cxNodeOff;                        // [2K] first node of each side's strand
  bool cxLinear = false;                             // every crossing strand is linear (InstDesc::cxLin)
  std::vector<double> wk, hk, w, h, mu;
  std::vector<double> fc90, E90, Hs;                 // [2K] timber across the grain, each side (W1 classification)
  ws_protocol proto{};                               // load protocol (mode 0: none), kept over warm starts
  std::vector<double> nodeW, nodeH;                  // [n] section at every node, for the ground (params.floor)
  bool rigid = false;                                // only the ground holds the model: the rigid-body freedoms
  double rbR = 1e-9, rbVmax = 0, rbWmax = 0;         // model radius about the centroid; rigid speed limits
  double probe0[3] = {0, 0, 0};                      // the probe's position when the protocol started (P0)
  int dentAfterDefault = 1500;                       // first seat iteration when dent_after_iter < 0: warm-up + ramp of
                                                     // the model the instance was built from (solver_cpu.js:686)
  std::vector<uint8_t> enabled, locked;
  // goals
  std::vector<double> mass, kRotStatic;              // [n], [3m]
  double lRef = 1.0, jLenMin = 1.0, loadMaxConst = 0.0;
  // gather tables
  std::vector<int> nodeSegOut, nodeSegIn;            // [n] segment with seg_i0 = i / seg_i1 = i (-1 none)
  std::vector<int> segJointA, segJointB;             // [m] joint whose first / second segment this is (-1 none)
  std::vector<int> segClamp0, segClamp1;             // [m] clamps acting on the segment (-1 none)
  std::vector<int> segStrand, segLocal;              // [m]
  std::vector<int> strandSideOff, strandSideCnt;     // [S] slice of the sorted side list
  std::vector<int> sideList, sidePos;                // [2K] side at each position (strand-grouped, ascending id); position of each side
  std::vector<int> ord, ordSeg;                      // [2K] side ids (2c + side) sorted by (local segment, id) per strand
  std::vector<int> rngLo, rngHi;                     // [m] slice of ord on the segment

  void build(const ws_model &md);                    // everything, including the contact initialisation
  void rebuild(const ws_model &md);                  // warm start: new stiffness / loads / parameters, state kept
  void sortSides();                                  // ord / ordSeg / rngLo / rngHi from u
  void startProtocol();                              // P0 from the probe's position, the probe placed at the first value
  int sideSegLocal(int sd) const;                    // local segment of side sd from u (solver_cpu.js:144-149)
  double sideSegMin() const;                         // shortest rest length among the segments of strands with sides

 private:
  void loadModel(const ws_model &md, bool keepState);
  void buildAnchors(const ws_model &md);
  void buildTargets(const ws_model &md);
  void buildMasses(double ramp, const std::vector<double> &Fn);
  void contactInitialize(int sweeps = 3);
};

}  // namespace wsb
