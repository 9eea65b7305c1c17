// Device data layout and precision policies of the DR step (sm_100a).
//
// Layout in HBM: structure of arrays, one plane per vector component, all instances of a batch concatenated (every
// topology index is global).  Positions and frames are double-buffered (the kinetic-damping roll-back keeps the
// previous buffer instead of copying it back).
//
// Precision policies (ws_opts.precision):
//   F64    every quantity in double.
//   MIXED  element forces and torques in float; positions and frames stored as two floats (hi + lo) and updated in
//          double; the quantities that cancel — edge vectors against the frame (strain), the relative rotation of
//          joints, the crossing gap vector — are formed in double before the float arithmetic; slide coordinates,
//          slips and every reduction (kinetic energy, residual, force reference) in double.
//   F32    every quantity in float (the naive form).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <type_traits>

namespace wsb {

enum { PREC_F64 = 0, PREC_MIXED = 1, PREC_F32 = 2 };

template <int P> struct PrecT;
// TINY: a floor for divisors in R that stays a normal number of R
template <> struct PrecT<PREC_F64> { using R = double; using W = double; using A = double; using U = double; using S = double; static constexpr bool TWO = false; static constexpr double TINY = 1e-300; };
template <> struct PrecT<PREC_MIXED> { using R = float; using W = double; using A = double; using U = double; using S = float; static constexpr bool TWO = true; static constexpr double TINY = 1e-30; };
template <> struct PrecT<PREC_F32> { using R = float; using W = float; using A = float; using U = float; using S = float; static constexpr bool TWO = false; static constexpr double TINY = 1e-30; };

// per-instance description (host-written, read-only on the device)
struct InstDesc {
  int n0, n, m0, m, p0, p, c0, C, k0, K, s0, S;   // first global element and count: nodes, segments, joints, clamps, crossings, strands
  int warmup, ramp_iter, disp_ramp, kd, contacts, max_iter, localLoads;   // localLoads: some node carries a node-frame load
  double ms, damping, tol, strength, stick, tf, eps, slip_rate, lRef, jLenMin, edgeThr;
  // contact extensions: augmented Lagrangian, W2 rotational friction, W3 seat law (ext: any of them)
  int ext, aug, alEvery, rotFric, seat, seatGap, dentAfter;
  double rotFactor, dentRate;
  // load protocol (ws_protocol): mode (0 none), probe node (global index), increments, settle / average lengths, the
  // instance's slot in the schedule and read-out arrays, probe axis
  int utmMode, utmProbe, utmNInc, utmSettle, utmAvg, utmIdx;
  double utmAxis[3];
  // the ground: on / off, height, friction coefficient
  int floorOn;
  // every strand that carries a crossing side is linear: its segment k joins its nodes N0 + k and N0 + k + 1, and no
  // other segment starts or ends on those nodes; a side's nodes and neighbouring segments then follow by arithmetic
  int cxLin;
  double floorZ, floorMu;
  // rigid-body freedoms of a model that only the ground holds (Floor, solver_cpu.js:520-533): on / off, the model
  // radius about its centroid at set-up, the speed limits per iteration of the rigid translation and rotation
  int rbOn;
  double rbR, rbVmax, rbWmax;
};

// per-instance control (device-written every iteration)
struct InstCtl {
  int iter, status, rollbacks, pending;      // pending: the last iteration rolled back (velocities read as zero)
  int cur, obuf, disp_it0, stop_at;          // cur: position / frame buffer; obuf: sorted-side buffer
  double ke, ke_prev, residual, res_f, res_t, fref;
  double e_stretch, e_shear, e_bend, e_twist, e_contact;
  int penN, alPend;    // augmented Lagrangian: iterations in the penetration window; the multiplier update is due
  // batched forms: global timer (ns) when the instance's block (or cluster) took it up in the last launch, and when it
  // left it; 0 in the other forms
  unsigned long long tBeg, tEnd;
};

// per-instance state of the extensions, apart from the control block that every iteration carries (kernel variants
// without extensions never touch it): the load protocol's phase (0 settle, 1 average, 2 finished), iterations in the
// phase, increments recorded, samples averaged; probe force (mode 1), applied value, probe origin P0, sums of the
// probe travel (x, y, z) and reaction; the ground's spring energy
struct InstExt {
  int phase, it, inc, accN;
  double pf[3], curF, p0[3], sum[4];
  double eFloor;
  // the rigid-body freedoms: translation and rotation velocities, and the rigid part of the last residual
  double rbV[3], rbW[3], rbRes;
};

// reduction slots
enum { RS_KE = 0, RS_STRETCH, RS_SHEAR, RS_BEND, RS_TWIST, RS_PEN, RS_TAN, RS_FLOOR, RS_NSUM };
enum { RX_F = 0, RX_T, RX_N, RX_M, RX_FN, RX_LOAD, RX_NMAX };

template <int P>
struct Dev {
  using T = PrecT<P>;
  using R = typename T::R; using W = typename T::W; using A = typename T::A; using U = typename T::U; using S = typename T::S;
  int ntot, mtot, ptot, ctot, ktot, stot;
  // Plane and buffer strides of the arrays that change every iteration.  In the global layout they follow the totals
  // (nS = ntot, xB = 3 ntot, mS = mtot, qB = 4 mtot, pS = ptot, cS = ctot, kS = ktot, sS = kB = oB = 2 ktot,
  // rB = mtot); the resident form points those arrays into shared memory with one instance's counts as strides (and
  // buffer strides of 0 where it works in place).
  int nS, xB, mS, qB, pS, cS, kS, sS, kB, oB, rB;
  // nodes: planes [buf][3][ntot] (lo planes only for MIXED)
  S *X, *Xlo;
  R *V;            // [3][ntot]
  R *mass;         // [ntot]
  R *lc, *ll;      // [3][ntot] constant loads, node-frame loads
  uint8_t *nflag;  // bits 0-2 free X Y Z, 3 fixed (any), 4 local load, 5 prescribed motion
  int *nsOut, *nsIn, *anc;   // [ntot]
  W *ancStart;     // [3][ntot slots]
  W *ancDelta;
  R *react;        // [3][ntot]
  // segments
  S *Q, *Qlo;      // [buf][4][mtot]
  R *Wr;           // [3][mtot]
  int *segI0, *segI1, *jA, *jB, *cl0, *cl1, *segStrand, *segLocal;
  R *l0, *EA, *GA, *krs;    // krs [3][mtot]
  W *il0;                   // 1 / l0 in the wide type (the mixed policy's strain)
  R *nF, *en;      // [3][mtot] segment force n and e × n
  R *Nax, *Vsh;    // [mtot], [2][mtot]
  int *rngLo, *rngHi;       // [2][mtot]
  // joints
  int *jS0, *jS1;
  R *jLen, *EIx, *EIy, *GJ, *om;   // om [3][ptot]
  R *tau, *kd, *Mj;                // [3][ptot]
  // clamps
  int *cSeg;
  R *cLen, *cB;    // cB [3][ctot]
  W *cQ;           // [4][ctot]
  R *tauC, *cM;    // [3][ctot], [2][ctot]
  // crossings
  int *cxSegOff, *cxNseg;   // [2][ktot]
  int *cxNodeOff;           // [2][ktot] first node of the side's strand (read when the instance's strands are linear)
  R *wk, *hk;               // [2][ktot]
  R *cw, *ch, *mu;          // [ktot]
  uint8_t *cflag;           // bit 0 enabled, bit 1 locked
  U *u;                     // [2][ktot]
  R *nPrev;                 // [3][ktot]
  A *slip;                  // [ktot]
  uint8_t *stuck, *cstate;  // [ktot]
  R *Fn, *Ft, *gap;         // [ktot]
  R *fc90, *E90, *Hs;       // [2][ktot] timber of each side across the grain (W1 classification)
  R *sProj;                 // [2][2 ktot] contact normal in each side's section frame (x, y; sd = 2c + side), last evaluation
  R *sinT;                  // [ktot] |tA × tB| clipped to [1e-6, 1] at the last evaluation
  uint8_t *ctype;           // [ktot] W1 outputs, filled when a download asks for them
  R *theta, *area, *pres, *util;   // [ktot]
  R *phiS;
  // contact extensions (state): multiplier and the penetration summed since its update; seat depth, climb and wall
  // slope per side (sd = 2c + side), edge-on-face embedment; W2 reference angle, rotational slip and moment
  A *lam, *penAcc;          // [ktot]
  R *dent, *climb, *tanpsi; // [2 ktot]
  R *dentE, *theta0, *Mrot; // [ktot]
  A *rotSlip;               // [ktot]
  // load protocol: schedule [instances][WS_PROTOCOL_MAX_INC], read-out [instances][WS_PROTOCOL_MAX_INC][4]
  double *utmSched, *utmOut;
  InstExt *ext;             // [instances]
  // the ground: section at every node [ntot], stick points (state) [ntot], force [3][ntot] and contact state [ntot]
  R *flW, *flH;
  W *flAx, *flAy;
  R *flF;
  uint8_t *flState;
  R *ldTot;        // [3][ntot] the external loads of a node on the ground in the last evaluation (rigid-body sums)
  // results post-processing: the joint and the clamp at every node [ntot] (−1 none), the displacement origin [3][ntot],
  // segment moments [3][mtot] and node layers [4][ntot] (outputs)
  int *nodeJoint, *nodeClamp;
  W *X0;
  R *segM, *nodeLay;                  // [2 ktot]
  // side records, indexed by side position p: the sides (sd = 2c + side) grouped by strand, ascending sd within a
  // strand (the strand's range is [stSideOff, stSideOff + stSideCnt))
  int *sPos;                // [2 ktot] position of side sd
  int *sKey;                // [2][2 ktot] local segment of the side after the slide, by sorted-side buffer
  int *sInv;                // [2][2 ktot] short order: the side's position in the sorted order of that buffer
  int *sKeyS;               // [2 ktot] short order: the key after the slide, at the side's sorted position
  int *sSideAt;             // [2 ktot] short order: the side's strand position, at its sorted position
  int *sStrand;             // [2 ktot] strand of the side
  R *sT, *kth;              // [2 ktot] Hermite parameter before the slide; righting stiffness of the side's crossing
  R *sF, *sTq;              // [3][2 ktot] force on the side; lever torque
                            // (side records: at the strand position, or with the short order at the sorted position)
  // strands
  int *stSideOff, *stSideCnt;   // [stot]
  int *stSegOff;                // [stot] first (global) segment of the strand
  int *ord, *ordSeg;            // [2][2 ktot] side positions sorted by (local segment, position) per strand; their keys
};

// Shared-memory layout of one instance in the resident form: byte offsets of the arrays that change every iteration
// (one buffer of positions and frames, updated in place), from the instance's element counts.  The host sizes the
// launch with the same function.  The side order keeps two buffers (this iteration's and the next's); the short-slide
// variant keeps sorted positions and the keys at them, the general one the sorted list of side positions.
struct ResLayout {
  unsigned X, Xlo, V, Q, Qlo, Wr, nF, en, tau, kd, tauC, u, nPrev, sKey, sInv, sKeyS, sSideAt, sT, kth, sF, sTq, ord, ordSeg, rngLo,
      rngHi, bytes;
};
__host__ __device__ inline unsigned resTake(unsigned &o, size_t bytes) {
  const unsigned r = o;
  o += unsigned((bytes + 15) & ~size_t(15));
  return r;
}
template <int P>
__host__ __device__ inline ResLayout residentLayout(int n, int m, int p, int C, int K, bool shortSides) {
  using R = typename PrecT<P>::R; using S = typename PrecT<P>::S; using U = typename PrecT<P>::U;
  const bool two = PrecT<P>::TWO;
  const size_t N = n, M = m, J = p, CC = C, K2 = 2 * size_t(K);
  ResLayout L{};
  unsigned o = 0;
  L.X = resTake(o, 3 * N * sizeof(S)); L.Xlo = two ? resTake(o, 3 * N * sizeof(S)) : 0; L.V = resTake(o, 3 * N * sizeof(R));
  L.Q = resTake(o, 4 * M * sizeof(S)); L.Qlo = two ? resTake(o, 4 * M * sizeof(S)) : 0; L.Wr = resTake(o, 3 * M * sizeof(R));
  L.nF = resTake(o, 3 * M * sizeof(R)); L.en = resTake(o, 3 * M * sizeof(R));
  L.tau = resTake(o, 3 * J * sizeof(R)); L.kd = resTake(o, 3 * J * sizeof(R)); L.tauC = resTake(o, 3 * CC * sizeof(R));
  L.u = resTake(o, K2 * sizeof(U)); L.nPrev = resTake(o, 3 * size_t(K) * sizeof(R));
  L.sKey = resTake(o, 2 * K2 * sizeof(int));
  L.sInv = resTake(o, (shortSides ? 2 : 0) * K2 * sizeof(int)); L.sKeyS = resTake(o, (shortSides ? 1 : 0) * K2 * sizeof(int));
  L.sSideAt = resTake(o, (shortSides ? 1 : 0) * K2 * sizeof(int));
  L.sT = resTake(o, K2 * sizeof(R)); L.kth = resTake(o, K2 * sizeof(R));
  L.sF = resTake(o, 3 * K2 * sizeof(R)); L.sTq = resTake(o, 3 * K2 * sizeof(R));
  L.ord = resTake(o, (shortSides ? 0 : 2) * K2 * sizeof(int)); L.ordSeg = resTake(o, 2 * K2 * sizeof(int));
  L.rngLo = resTake(o, 2 * M * sizeof(int)); L.rngHi = resTake(o, 2 * M * sizeof(int));
  L.bytes = o;
  return L;
}

}  // namespace wsb
