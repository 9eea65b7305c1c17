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
template <> struct PrecT<PREC_F64> { using R = double; using W = double; using A = double; using U = double; using S = double; static constexpr bool TWO = false; };
template <> struct PrecT<PREC_MIXED> { using R = float; using W = double; using A = double; using U = double; using S = float; static constexpr bool TWO = true; };
template <> struct PrecT<PREC_F32> { using R = float; using W = float; using A = float; using U = float; using S = float; static constexpr bool TWO = false; };

// per-instance description (host-written, read-only on the device)
struct InstDesc {
  int n0, n, m0, m, p0, p, c0, C, k0, K, s0, S;   // first global element and count: nodes, segments, joints, clamps, crossings, strands
  int warmup, ramp_iter, disp_ramp, kd, contacts, max_iter;
  double ms, damping, tol, strength, stick, tf, eps, slip_rate, lRef, jLenMin;
};

// per-instance control (device-written every iteration)
struct InstCtl {
  int iter, status, rollbacks, pending;      // pending: the last iteration rolled back (velocities read as zero)
  int cur, obuf, disp_it0, stop_at;          // cur: position / frame buffer; obuf: sorted-side buffer
  double ke, ke_prev, residual, res_f, res_t, fref;
  double e_stretch, e_shear, e_bend, e_twist, e_contact;
};

// reduction slots
enum { RS_KE = 0, RS_STRETCH, RS_SHEAR, RS_BEND, RS_TWIST, RS_PEN, RS_TAN, RS_NSUM };
enum { RX_F = 0, RX_T, RX_N, RX_M, RX_FN, RX_LOAD, RX_NMAX };

template <int P>
struct Dev {
  using T = PrecT<P>;
  using R = typename T::R; using W = typename T::W; using A = typename T::A; using U = typename T::U; using S = typename T::S;
  int ntot, mtot, ptot, ctot, ktot, stot;
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
  R *wk, *hk;               // [2][ktot]
  R *cw, *ch, *mu;          // [ktot]
  uint8_t *cflag;           // bit 0 enabled, bit 1 locked
  U *u;                     // [2][ktot]
  R *nPrev;                 // [3][ktot]
  A *slip;                  // [ktot]
  uint8_t *stuck, *cstate;  // [ktot]
  R *Fn, *Ft, *gap;         // [ktot]
  // side records, indexed by side position p: the sides (sd = 2c + side) grouped by strand, ascending sd within a
  // strand (the strand's range is [stSideOff, stSideOff + stSideCnt))
  int *sPos;                // [2 ktot] position of side sd
  int *sKey;                // [2][2 ktot] local segment of the side after the slide, by sorted-side buffer
  int *sStrand;             // [2 ktot] strand of the side
  R *sT, *kth;              // [2 ktot] Hermite parameter before the slide; righting stiffness of the side's crossing
  R *sF, *sTq;              // [3][2 ktot] force on the side; lever torque
  // strands
  int *stSideOff, *stSideCnt;   // [stot]
  int *stSegOff;                // [stot] first (global) segment of the strand
  int *ord, *ordSeg;            // [2][2 ktot] side positions sorted by (local segment, position) per strand; their keys
};

}  // namespace wsb
