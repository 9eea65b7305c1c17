// sm_100a kernels of the DR step: the persistent batched form (one thread block per instance, every phase of every
// iteration inside one launch) and the plain form (one kernel per phase, one instance, captured as a CUDA graph).
#include <mutex>
#include <algorithm>

#include "dr_kernels.hpp"
#include "dr_phases.cuh"

// Minimum resident blocks of 256 threads per SM asked of the large-instance kernels, i.e. their register budget
// (65536 / (256 × blocks) registers a thread), each chosen by measurement on the 20 m shell: the whole element kernel
// unbounded (the crossing code is heavy in live values), its rod half (Y) at 4 (64 registers; 3 in FP64, where 64
// registers spill), the element launch with block roles at 2, the whole update kernel at 4 (64 registers, a few
// spills), its node and segment halves (DN, DM) at 3, the grid form at 2.
#ifndef WSB_MINB_A
#define WSB_MINB_A 1
#endif
#ifndef WSB_MINB_D
#define WSB_MINB_D 4
#endif
// The rod kernel's block: 512 threads at 2 blocks per SM (64 registers) in the mixed and FP32 policies, which halves
// its block partials against 256 × 4 at the same occupancy; 256 threads at 3 blocks per SM in FP64.
#ifndef WSB_Y_T_MIXED
#define WSB_Y_T_MIXED 512
#endif
#define WSB_Y_THREADS(P) ((P) == PREC_F64 ? 256 : WSB_Y_T_MIXED)
#ifndef WSB_MINB_Y
#ifndef WSB_MINB_YM
#define WSB_MINB_YM 2
#endif
#define WSB_MINB_Y(P) ((P) == PREC_F64 ? 3 : WSB_MINB_YM)
#endif
#ifndef WSB_MINB_XY
#define WSB_MINB_XY 2
#endif
// The split update kernels (nodes, segments) without the extensions run five blocks of 256 threads per SM in the
// mixed and FP32 policies (48 registers, a few dozen bytes of spill): with the crossing and rod kernels' results in
// L2, both kernels' blocks are then resident at once, measured 0.8 us an iteration faster on the 20 m shell than three
// blocks at 80 registers.  FP64 and the extension variants need more registers and keep three.
#ifndef WSB_MINB_DN
#define WSB_MINB_DN(P, EXT) (((P) == PREC_F64 || (EXT)) ? 3 : 5)
#endif
#ifndef WSB_MINB_DM
#define WSB_MINB_DM(P, EXT) (((P) == PREC_F64 || (EXT)) ? 3 : 5)
#endif
#ifndef WSB_MINB_G
#define WSB_MINB_G 2
#endif

namespace wsb {

// Programmatic dependent launch: a kernel of the plain form lets the next one be launched as soon as all its blocks
// have started, and waits for the previous one (completion and memory) before it reads anything.  Launched without the
// attribute, both instructions do nothing.
__device__ __forceinline__ void waitPrevGrid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allowNextGrid() { asm volatile("griddepcontrol.launch_dependents;" :::); }
// the GPU's global nanosecond timer (per-instance device times of the batched forms)
__device__ __forceinline__ unsigned long long globalTimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Block partials, value-major: slot i of block b at part[i * stride + b], so the finishing block reads them coalesced.
template <class A>
__device__ __forceinline__ void putPart(const Part<A> &p, A *part, int b, int stride) {
  for (int i = 0; i < RS_NSUM; i++) part[size_t(i) * stride + b] = p.s[i];
  for (int i = 0; i < RX_NMAX; i++) part[size_t(RS_NSUM + i) * stride + b] = p.x[i];
}
// the same, writing only the slots in SM / XM (the plain form: the close reads only those)
template <unsigned SM, unsigned XM, class A>
__device__ __forceinline__ void putPartSlots(const Part<A> &p, A *part, int b, int stride) {
#pragma unroll
  for (int i = 0; i < RS_NSUM; i++)
    if (SM & (1u << i)) part[size_t(i) * stride + b] = p.s[i];
#pragma unroll
  for (int i = 0; i < RX_NMAX; i++)
    if (XM & (1u << i)) part[size_t(RS_NSUM + i) * stride + b] = p.x[i];
}
// row b of the partial range [lo, hi) added into q, only the slots in SM / XM.  A row past the range is read at hi − 1
// instead (every range holds at least one row: each kernel launches a block or more): a repeated row leaves a maximum
// unchanged, and its sums are not added.  The loads do not depend on b being in the range, so the rows of several
// ranges go out together.
template <unsigned SM, unsigned XM, class A>
__device__ __forceinline__ void addRangeRow(Part<A> &q, const A *part, int b, int hi, int stride) {
  const bool in = b < hi;
  const int bc = in ? b : hi - 1;
#pragma unroll
  for (int i = 0; i < RS_NSUM; i++)
    if (SM & (1u << i)) {
      const A v = __ldcg(part + size_t(i) * stride + bc);
      q.s[i] += in ? v : A(0);
    }
#pragma unroll
  for (int i = 0; i < RX_NMAX; i++)
    if (XM & (1u << i)) q.x[i] = mmax(q.x[i], __ldcg(part + size_t(RS_NSUM + i) * stride + bc));
}
// the same in two steps, so that the loads of several rows go out before the first of their adds
template <unsigned SM, unsigned XM, class A>
struct RangeRow {
  A v[RS_NSUM + RX_NMAX];
  bool in;
  __device__ __forceinline__ void load(const A *part, int b, int hi, int stride) {
    in = b < hi;
    const int bc = in ? b : hi - 1;
#pragma unroll
    for (int i = 0; i < RS_NSUM; i++)
      if (SM & (1u << i)) v[i] = __ldcg(part + size_t(i) * stride + bc);
#pragma unroll
    for (int i = 0; i < RX_NMAX; i++)
      if (XM & (1u << i)) v[RS_NSUM + i] = __ldcg(part + size_t(RS_NSUM + i) * stride + bc);
  }
  __device__ __forceinline__ void add(Part<A> &q) const {
#pragma unroll
    for (int i = 0; i < RS_NSUM; i++)
      if (SM & (1u << i)) q.s[i] += in ? v[i] : A(0);
#pragma unroll
    for (int i = 0; i < RX_NMAX; i++)
      if (XM & (1u << i)) q.x[i] = mmax(q.x[i], v[RS_NSUM + i]);
  }
};
template <class A>
__device__ __forceinline__ void addPart(Part<A> &q, const A *part, int b, int stride) {
  for (int i = 0; i < RS_NSUM; i++) q.s[i] += __ldcg(part + size_t(i) * stride + b);
  for (int i = 0; i < RX_NMAX; i++) q.x[i] = mmax(q.x[i], __ldcg(part + size_t(RS_NSUM + i) * stride + b));
}

// rod element e of phase A: segments, joints, clamps
template <int P>
__device__ __forceinline__ void rodElement(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, int e, Part<typename Dev<P>::A> &pt) {
  if (e < I.m) segForce<P>(d, sx.cur, I.m0 + e, pt);
  else if ((e -= I.m) < I.p) jointTorque<P>(d, sx.cur, I.p0 + e, pt);
  else clampTorque<P>(d, sx.cur, I.c0 + (e - I.p), pt);
}
// rod element pair e of the plain form's rod kernel: segment e and joint e (or, past the joints, clamp e − p) in one
// thread, so the kernel runs half as many threads as rod elements and all of its blocks are resident beside the
// crossing kernel's (its per-thread chain is two elements long, still shorter than a crossing side's)
template <int P>
__device__ __forceinline__ void rodPair(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, int e, Part<typename Dev<P>::A> &pt) {
  if (e < I.m) segForce<P>(d, sx.cur, I.m0 + e, pt);
  if (e < I.p) jointTorque<P>(d, sx.cur, I.p0 + e, pt);
  else if (e - I.p < I.C) clampTorque<P>(d, sx.cur, I.c0 + (e - I.p), pt);
}
// crossing element e of phase A: two adjacent elements, one a side, per crossing
template <int P, bool SHORT, bool EXT>
__device__ __forceinline__ void crossElement(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, int e, Part<typename Dev<P>::A> &pt) {
  crossing<P, SHORT, EXT>(d, I, sx.cur, sx.iter, sx.onxt, sx.obuf, I.k0 + (e >> 1), e & 1, sx.alPend, sx.penN, pt);
}
// element e of phase A: the crossings come first (the heaviest elements start earliest), then the rods
template <int P, bool SHORT, bool EXT>
__device__ __forceinline__ void phaseA(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, int e, int nK, Part<typename Dev<P>::A> &pt) {
  if (e < 2 * nK) crossElement<P, SHORT, EXT>(d, I, sx, e, pt);
  else rodElement<P>(d, I, sx, e - 2 * nK, pt);
}
__device__ __forceinline__ int countA(const InstDesc &I) {
  const int nK = (I.contacts && I.K) ? I.K : 0;
  return I.m + I.p + I.C + 2 * nK;
}
// elements of phase D: nodes, segments and, with the short order, the ranks of the sides (the next iteration's order)
template <bool SHORT>
__device__ __forceinline__ int countD(const InstDesc &I) {
  return I.n + I.m + ((SHORT && I.contacts && I.K) ? 2 * I.K : 0);
}
// phase B / C of the general order: the ranks of the sides and the slices of the segments in the new order
template <int P>
__device__ __forceinline__ void phaseBC(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, int e) {
  const int n2 = 2 * I.K;
  if (e < n2) rankSide<P>(d, 2 * I.k0 + e, sx.onxt, sx.onxt);
  else segCount<P>(d, I.m0 + (e - n2), sx.onxt, sx.onxt);
}
template <int P, bool SHORT, bool EXT>
__device__ __forceinline__ void phaseD(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, int e, Part<typename Dev<P>::A> &pt) {
  if (e < I.n) nodeUpdate<P, SHORT, EXT>(d, I, sx, I.n0 + e, pt);
  else if ((e -= I.n) < I.m) segUpdate<P, SHORT>(d, I, sx, I.m0 + e, pt);
  else rankSideWindow<P>(d, 2 * I.k0 + (e - I.m), sx.obuf, sx.onxt);
}

// ------------------------------------------------------------------------------------------------ balanced warps
// Inside one block, a phase's elements are split over the warps by cost: the elements come in runs of one kind
// (crossings, side ranks, segments, ...), each run cut into chunks of 32 (one element a lane, so a chunk never mixes
// kinds), and warp w takes the chunks whose cost midpoint falls in its equal share of the phase's total cost.  Every
// warp's range is contiguous.  The split is a function of the element counts and the block size only, so the
// per-thread partial sums, and with them every reduction, are the same from run to run.  Relative costs are rough
// instruction counts of one element.
struct PhaseRun { int count, cost; };
enum { COST_CROSSING = 24, COST_RANK = 3, COST_SEGMENT = 5, COST_JOINT = 8, COST_CLAMP = 8, COST_NODE_UPD = 3,
       COST_SEG_UPD = 5, COST_SLICE = 3 };

// chunks i in [0, nc) of a run starting at cumulative cost cb whose midpoint, doubled and scaled by the warp count,
// nw·(2·cb + (2i + 1)·cost), lies below x
__device__ __forceinline__ int chunksBelow(long long x, long long cb, int cost, int nw, int nc) {
  const long long num = x - 2LL * nw * cb - (long long)nw * cost;
  if (num <= 0) return 0;
  const long long den = 2LL * nw * cost;
  const long long c = (num + den - 1) / den;
  return int(c < nc ? c : nc);
}
// over nw warps of which this thread's is w (a block's warps, or a cluster's)
template <int NR, class F>
__device__ __forceinline__ void forBalancedOver(const PhaseRun (&runs)[NR], int nw, int w, F &&f) {
  const int lane = threadIdx.x & 31;
  long long total = 0;
  for (int r = 0; r < NR; r++) total += (long long)((runs[r].count + 31) >> 5) * runs[r].cost;
  long long cb = 0;
  for (int r = 0; r < NR; r++) {
    const int nc = (runs[r].count + 31) >> 5, cost = runs[r].cost;
    if (nc > 0) {
      const int i0 = chunksBelow(2LL * w * total, cb, cost, nw, nc), i1 = chunksBelow(2LL * (w + 1) * total, cb, cost, nw, nc);
      for (int i = i0; i < i1; i++) {
        const int e = i * 32 + lane;
        if (e < runs[r].count) f(r, e);
      }
    }
    cb += (long long)nc * cost;
  }
}
template <int NR, class F>
__device__ __forceinline__ void forBalanced(const PhaseRun (&runs)[NR], F &&f) {
  forBalancedOver(runs, int(blockDim.x >> 5), int(threadIdx.x >> 5), f);
}

// phase A of one instance over the block: crossings, segments, joints, clamps
template <int P, bool SHORT, bool EXT>
__device__ __forceinline__ void blockPhaseA(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, Part<typename Dev<P>::A> &pt,
                                            int nw, int w) {
  const int nK = (I.contacts && I.K) ? I.K : 0;
  const PhaseRun runs[4] = {{2 * nK, COST_CROSSING}, {I.m, COST_SEGMENT}, {I.p, COST_JOINT}, {I.C, COST_CLAMP}};
  forBalancedOver(runs, nw, w, [&](int r, int e) {
    switch (r) {
      case 0: crossing<P, SHORT, EXT>(d, I, sx.cur, sx.iter, sx.onxt, sx.obuf, I.k0 + (e >> 1), e & 1, sx.alPend, sx.penN, pt); break;
      case 1: segForce<P>(d, sx.cur, I.m0 + e, pt); break;
      case 2: jointTorque<P>(d, sx.cur, I.p0 + e, pt); break;
      default: clampTorque<P>(d, sx.cur, I.c0 + e, pt); break;
    }
  });
}
// phase B / C (general order) of one instance over the block
template <int P>
__device__ __forceinline__ void blockPhaseBC(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, int nw, int w) {
  const PhaseRun runs[2] = {{2 * I.K, COST_RANK}, {I.m, COST_SLICE}};
  forBalancedOver(runs, nw, w, [&](int r, int e) {
    if (r == 0) rankSide<P>(d, 2 * I.k0 + e, sx.onxt, sx.onxt);
    else segCount<P>(d, I.m0 + e, sx.onxt, sx.onxt);
  });
}

// ------------------------------------------------------------------------------------------------ rigid-body freedoms
// K doubles summed over the block in a fixed order (warp shuffles, then the warps' results in order); the result is
// valid in thread 0.  smem: >= 32 K doubles.
template <int K>
__device__ __forceinline__ void blockSumD(double (&v)[K], double *smem) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < K; k++) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  __syncthreads();
  if (lane == 0)
    for (int k = 0; k < K; k++) smem[wid * K + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < K; k++) v[k] = 0.0;
    for (int w = 0; w < nw; w++)
      for (int k = 0; k < K; k++) v[k] += smem[w * K + k];
  }
  __syncthreads();
}
// The rigid-body freedoms of instance I over one block, after its update phase and its block reduction `pt` (valid in
// thread 0): the centroid of the positions at the iteration's start (buffer sx.cur), the sums about it, then in thread 0
// the velocity update and the kinetic-damping decision with the rigid kinetic energy and residual, then, unless the
// iteration rolls back, the rigid step of every node and frame of the new buffer (sx.nxt).  sc: the block's control
// block; ux: the instance's extension state.
template <int P, bool EXT>
__device__ void rigidBlockStep(const Dev<P> &d, const InstDesc &I, const StepCtx &sx, InstCtl &sc, InstExt &ux,
                               Part<typename Dev<P>::A> &pt, int nIter) {
  using A = typename Dev<P>::A;
  __shared__ double rsm[32 * RB_NSUM];
  __shared__ double rc[3], rv[3], rw[3], rq[4];
  __shared__ int rmove;
  double cs[3] = {0.0, 0.0, 0.0};
  for (int e = threadIdx.x; e < I.n; e += blockDim.x)
    for (int k = 0; k < 3; k++) cs[k] += double(Acc<P>::xw(d, sx.cur, k, I.n0 + e));
  blockSumD<3>(cs, rsm);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) rc[k] = cs[k] / double(max(I.n, 1));
  __syncthreads();
  double s[RB_NSUM] = {0.0};
  const double c[3] = {rc[0], rc[1], rc[2]};
  for (int e = threadIdx.x; e < I.n; e += blockDim.x) rigidNode<P>(d, sx.cur, I.n0 + e, c, s);
  blockSumD<RB_NSUM>(s, rsm);
  if (threadIdx.x == 0) {
    double rbq[2];
    const double ke2 = rigidUpdate(I, sx.iter, sx.warm != 0, s, ux, rbq);
    pt.s[RS_KE] += A(ke2);
    decide<EXT>(I, sc, pt, nIter, rbq);
    if (sc.pending) for (int k = 0; k < 3; k++) ux.rbV[k] = ux.rbW[k] = 0.0;
    ux.rbRes = fmax(rbq[0] / sc.fref, rbq[1] / (sc.fref * I.rbR));
    rmove = !sc.pending && rigidMoves(ux);
    for (int k = 0; k < 3; k++) { rv[k] = ux.rbV[k]; rw[k] = ux.rbW[k]; }
    const double a = sqrt(rw[0] * rw[0] + rw[1] * rw[1] + rw[2] * rw[2]), half = 0.5 * a;
    const double sn = a > 1e-12 ? sin(half) / a : 0.5;
    rq[0] = cos(half); rq[1] = rw[0] * sn; rq[2] = rw[1] * sn; rq[3] = rw[2] * sn;
  }
  __syncthreads();
  if (rmove) {
    const double v[3] = {rv[0], rv[1], rv[2]}, w[3] = {rw[0], rw[1], rw[2]}, q[4] = {rq[0], rq[1], rq[2], rq[3]};
    for (int e = threadIdx.x; e < I.n + I.m; e += blockDim.x) {
      if (e < I.n) rigidMoveNode<P>(d, sx.cur, sx.nxt, I.n0 + e, c, v, w);
      else rigidMoveSeg<P>(d, sx.nxt, I.m0 + (e - I.n), q);
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------------------------------------ batched form
// Block b relaxes instance order[b] (and further instances grid-strided) for up to nIter iterations, stopping at its
// own convergence.  Instance state lives in HBM / L2; the block's barriers separate the phases, so an instance never
// waits on another and no kernel spins.
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(512) k_batched(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                  const int *__restrict__ order, int nInst, int nIter, const uint8_t *__restrict__ mask) {
  using A = typename Dev<P>::A;
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  const int nwB = blockDim.x >> 5, wB = threadIdx.x >> 5;
  for (int bi = blockIdx.x; bi < nInst; bi += gridDim.x) {
    const int b = order ? order[bi] : bi;
    if (mask && !mask[b]) continue;
    if (threadIdx.x == 0) { sc = ctl[b]; si = insts[b]; sc.tBeg = globalTimer(); }
    __syncthreads();
    const InstDesc &I = si;
    const bool cx = I.contacts && I.K;
    for (int it = 0; it < nIter; it++) {
      if (sc.status != WS_RUNNING) break;
      const StepCtx sx = makeCtx<A>(I, sc, EXT ? d.ext[I.utmIdx].pf : nullptr);
      Part<A> pt;
      pt.init();
      blockPhaseA<P, SHORT, EXT>(d, I, sx, pt, nwB, wB);
      __syncthreads();
      if (!SHORT && cx) {
        blockPhaseBC<P>(d, I, sx, nwB, wB);
        __syncthreads();
      }
      {
        const PhaseRun runs[3] = {{I.n, COST_NODE_UPD}, {I.m, COST_SEG_UPD}, {(SHORT && cx) ? 2 * I.K : 0, COST_RANK}};
        forBalanced(runs, [&](int r, int e) {
          if (r == 0) nodeUpdate<P, SHORT, EXT>(d, I, sx, I.n0 + e, pt);
          else if (r == 1) segUpdate<P, SHORT>(d, I, sx, I.m0 + e, pt);
          else rankSideWindow<P>(d, 2 * I.k0 + e, sx.obuf, sx.onxt);
        });
      }
      __syncthreads();
      blockReduce(pt, red);
      if constexpr (EXT) {
        if (I.rbOn) {                   // a model only the ground holds: its rigid-body freedoms decide with it
          rigidBlockStep<P, EXT>(d, I, sx, sc, d.ext[I.utmIdx], pt, nIter);
          if (threadIdx.x == 0) d.ext[I.utmIdx].eFloor = double(pt.s[RS_FLOOR]);
          __syncthreads();
          continue;
        }
      }
      if (threadIdx.x == 0) decide<EXT>(I, sc, pt, nIter);
      __syncthreads();
      if constexpr (EXT) {
        if (threadIdx.x == 0) protocolStep<P>(d, sc.cur, I, sc, pt);
        __syncthreads();
      }
    }
    if (threadIdx.x == 0) { sc.tEnd = globalTimer(); ctl[b] = sc; }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------ wide instances
// The batched form for an instance too large for one block to keep pace with the rest of the batch: a thread-block
// cluster (its blocks on SMs of one GPC, launched together) relaxes it.  Every phase's elements are split by cost over
// all the cluster's warps (the split depends only on the counts, the block size and the cluster size); the phases are
// separated by the cluster's hardware barrier, whose arrive has release and whose wait has acquire semantics at cluster
// scope, so a phase reads in global memory what the other blocks wrote in the one before, and nothing spins.  Each
// block reduces its partials, and every block then adds the cluster's block partials from distributed shared memory in
// rank order and takes the same kinetic-damping decision on its own copy of the control block, so no broadcast is
// needed.  The state stays in global memory (double-buffered, as in k_batched).  A load protocol is not run here (the
// host keeps such instances in the one-block kernels).
__device__ __forceinline__ void clusterSync() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
__device__ __forceinline__ unsigned clusterRank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned clusterSize() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
// a value of block `rank`'s shared memory: the address of `p` in that block (mapa), read through the cluster window
template <class A>
__device__ __forceinline__ A remoteLoad(const A *p, unsigned rank) {
  const unsigned local = static_cast<unsigned>(__cvta_generic_to_shared(p));
  unsigned remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
  if constexpr (sizeof(A) == 8) {
    unsigned long long v;
    asm volatile("ld.shared::cluster.u64 %0, [%1];" : "=l"(v) : "r"(remote) : "memory");
    return __longlong_as_double(static_cast<long long>(v));
  } else {
    unsigned v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(remote) : "memory");
    return __uint_as_float(v);
  }
}

template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(512) k_wide(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                               const int *__restrict__ wide, int nWide, int nIter, const uint8_t *__restrict__ mask) {
  using A = typename Dev<P>::A;
  static_assert(sizeof(A) == 4 || sizeof(A) == 8, "reduction type");
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  __shared__ A cpart[RS_NSUM + RX_NMAX];     // this block's partials, read by every block of the cluster
  const unsigned rank = clusterRank(), ncl = clusterSize();
  const int nwB = blockDim.x >> 5;
  const int nw = nwB * int(ncl), w = int(rank) * nwB + int(threadIdx.x >> 5);
  const int nClusters = int(gridDim.x / ncl), cid = int(blockIdx.x / ncl);
  for (int wi = cid; wi < nWide; wi += nClusters) {
    const int b = wide[wi];
    if (mask && !mask[b]) continue;                 // the same answer in every block of the cluster
    if (threadIdx.x == 0) { sc = ctl[b]; si = insts[b]; sc.tBeg = globalTimer(); }
    __syncthreads();
    const InstDesc &I = si;
    const bool cx = I.contacts && I.K;
    for (int it = 0; it < nIter; it++) {
      if (sc.status != WS_RUNNING) break;           // every block holds the same control block
      const StepCtx sx = makeCtx<A>(I, sc, EXT ? d.ext[I.utmIdx].pf : nullptr);
      Part<A> pt;
      pt.init();
      blockPhaseA<P, SHORT, EXT>(d, I, sx, pt, nw, w);
      clusterSync();
      if (!SHORT && cx) {
        blockPhaseBC<P>(d, I, sx, nw, w);
        clusterSync();
      }
      {
        const PhaseRun runs[3] = {{I.n, COST_NODE_UPD}, {I.m, COST_SEG_UPD}, {(SHORT && cx) ? 2 * I.K : 0, COST_RANK}};
        forBalancedOver(runs, nw, w, [&](int r, int e) {
          if (r == 0) nodeUpdate<P, SHORT, EXT>(d, I, sx, I.n0 + e, pt);
          else if (r == 1) segUpdate<P, SHORT>(d, I, sx, I.m0 + e, pt);
          else rankSideWindow<P>(d, 2 * I.k0 + e, sx.obuf, sx.onxt);
        });
      }
      blockReduce(pt, red);
      if (threadIdx.x == 0) {
        for (int i = 0; i < RS_NSUM; i++) cpart[i] = pt.s[i];
        for (int i = 0; i < RX_NMAX; i++) cpart[RS_NSUM + i] = pt.x[i];
      }
      // the phase-D writes of every block, and every block's partials, visible cluster-wide
      clusterSync();
      if (threadIdx.x == 0) {
        Part<A> q;
        q.init();
        for (unsigned r = 0; r < ncl; r++) {
          for (int i = 0; i < RS_NSUM; i++) q.s[i] += remoteLoad(cpart + i, r);
          for (int i = 0; i < RX_NMAX; i++) q.x[i] = mmax(q.x[i], remoteLoad(cpart + RS_NSUM + i, r));
        }
        decide<EXT>(I, sc, q, nIter);
        if constexpr (EXT)     // the ground's energy of the iteration
          if (rank == 0) d.ext[I.utmIdx].eFloor = double(q.s[RS_FLOOR]);
      }
      // the next write of cpart (after the next iteration's first cluster barrier) cannot overtake these reads
      __syncthreads();
    }
    if (threadIdx.x == 0 && rank == 0) { sc.tEnd = globalTimer(); ctl[b] = sc; }
    // no block leaves, or takes up the next instance, while another still reads its partials
    clusterSync();
  }
}

// ------------------------------------------------------------------------------------------------ resident form
// The batched form with each instance's changing state held in shared memory for the whole launch: positions,
// frames, velocities, the element results of phase A, the side records, the order and the slide coordinates.  Static
// data (topology, stiffness, loads) is read from global memory through L1; outputs that only a download reads (axial
// and shear forces, moments, contact forces, reactions, slip) are written to global memory as they are produced.
// Positions and frames are updated in place; the values they had at the start of the iteration go to a global backup
// buffer, and a kinetic-damping roll-back copies them back.

// the instance's shared-memory view: the changing arrays point into `sm`, offset so that the global element indices
// of the phase code land on the instance's local rows
template <int P>
__device__ __forceinline__ Dev<P> residentView(const Dev<P> &d, const InstDesc &I, unsigned char *sm, const ResLayout &L, bool shortSides) {
  using R = typename Dev<P>::R; using S = typename Dev<P>::S; using U = typename Dev<P>::U;
  Dev<P> v = d;
  const int k2 = 2 * I.k0;
  v.X = reinterpret_cast<S *>(sm + L.X) - I.n0;
  v.Xlo = PrecT<P>::TWO ? reinterpret_cast<S *>(sm + L.Xlo) - I.n0 : nullptr;
  v.V = reinterpret_cast<R *>(sm + L.V) - I.n0;
  v.Q = reinterpret_cast<S *>(sm + L.Q) - I.m0;
  v.Qlo = PrecT<P>::TWO ? reinterpret_cast<S *>(sm + L.Qlo) - I.m0 : nullptr;
  v.Wr = reinterpret_cast<R *>(sm + L.Wr) - I.m0;
  v.nF = reinterpret_cast<R *>(sm + L.nF) - I.m0;
  v.en = reinterpret_cast<R *>(sm + L.en) - I.m0;
  v.tau = reinterpret_cast<R *>(sm + L.tau) - I.p0;
  v.kd = reinterpret_cast<R *>(sm + L.kd) - I.p0;
  v.tauC = reinterpret_cast<R *>(sm + L.tauC) - I.c0;
  v.u = reinterpret_cast<U *>(sm + L.u) - I.k0;
  v.nPrev = reinterpret_cast<R *>(sm + L.nPrev) - I.k0;
  v.sKey = reinterpret_cast<int *>(sm + L.sKey) - k2;
  v.sInv = reinterpret_cast<int *>(sm + L.sInv) - k2;
  v.sKeyS = reinterpret_cast<int *>(sm + L.sKeyS) - k2;
  v.sSideAt = reinterpret_cast<int *>(sm + L.sSideAt) - k2;
  v.sT = reinterpret_cast<R *>(sm + L.sT) - k2;
  v.kth = reinterpret_cast<R *>(sm + L.kth) - k2;
  v.sF = reinterpret_cast<R *>(sm + L.sF) - k2;
  v.sTq = reinterpret_cast<R *>(sm + L.sTq) - k2;
  v.ord = reinterpret_cast<int *>(sm + L.ord) - k2;
  v.ordSeg = reinterpret_cast<int *>(sm + L.ordSeg) - k2;
  v.rngLo = reinterpret_cast<int *>(sm + L.rngLo) - I.m0;
  v.rngHi = reinterpret_cast<int *>(sm + L.rngHi) - I.m0;
  v.nS = I.n; v.xB = 0; v.mS = I.m; v.qB = 0; v.pS = I.p; v.cS = I.C; v.kS = I.K;
  v.sS = v.kB = v.oB = 2 * I.K;
  v.rB = I.m;
  (void)shortSides;
  return v;
}

// copy `planes` planes of `count` elements from array a (plane stride as, first element a0) to array b (bs, b0)
template <class T>
__device__ __forceinline__ void copyPlanes(T *b, int bs, const T *a, int as, int first, int count, int planes) {
  for (int e = threadIdx.x; e < planes * count; e += blockDim.x) {
    const int k = e / count, i = first + e % count;
    b[size_t(k) * bs + i] = a[size_t(k) * as + i];
  }
}

// global -> shared at the start of a launch (g: the global view, v: the instance's shared view); positions and
// frames from buffer `home`
template <int P, bool SHORT>
__device__ void residentLoad(const Dev<P> &g, const Dev<P> &v, const InstDesc &I, const InstCtl &c, int home) {
  copyPlanes(v.X, v.nS, g.X + size_t(home) * g.xB, g.nS, I.n0, I.n, 3);
  if constexpr (PrecT<P>::TWO) copyPlanes(v.Xlo, v.nS, g.Xlo + size_t(home) * g.xB, g.nS, I.n0, I.n, 3);
  copyPlanes(v.V, v.nS, g.V, g.nS, I.n0, I.n, 3);
  copyPlanes(v.Q, v.mS, g.Q + size_t(home) * g.qB, g.mS, I.m0, I.m, 4);
  if constexpr (PrecT<P>::TWO) copyPlanes(v.Qlo, v.mS, g.Qlo + size_t(home) * g.qB, g.mS, I.m0, I.m, 4);
  copyPlanes(v.Wr, v.mS, g.Wr, g.mS, I.m0, I.m, 3);
  if (!I.K) return;
  copyPlanes(v.u, v.kS, g.u, g.kS, I.k0, I.K, 2);
  copyPlanes(v.nPrev, v.kS, g.nPrev, g.kS, I.k0, I.K, 3);
  const int k2 = 2 * I.k0, K2 = 2 * I.K, ob = c.obuf;
  // the side order the next iteration reads: keys at the sorted positions, the segments' slices (with the short order
  // some slices are an earlier iteration's, which the keys mark), and the sorted positions (short) or the sorted list
  // of side positions (general)
  // both slice buffers: the short order rewrites only the slices of segments with sides, and the rest must stay the
  // (valid, older) slices of the global buffers
  copyPlanes(v.ordSeg + size_t(ob) * v.oB, 0, g.ordSeg + size_t(ob) * g.oB, 0, k2, K2, 1);
  copyPlanes(v.rngLo, v.rB, g.rngLo, g.rB, I.m0, I.m, 2);
  copyPlanes(v.rngHi, v.rB, g.rngHi, g.rB, I.m0, I.m, 2);
  if constexpr (SHORT) copyPlanes(v.sInv + size_t(ob) * v.kB, 0, g.sInv + size_t(ob) * g.kB, 0, k2, K2, 1);
  else copyPlanes(v.ord + size_t(ob) * v.oB, 0, g.ord + size_t(ob) * g.oB, 0, k2, K2, 1);
}

// shared -> global at the end of a launch, into the buffers the control block names
template <int P, bool SHORT>
__device__ void residentStore(const Dev<P> &g, const Dev<P> &v, const InstDesc &I, const InstCtl &c) {
  copyPlanes(g.X + size_t(c.cur) * g.xB, g.nS, v.X, v.nS, I.n0, I.n, 3);
  if constexpr (PrecT<P>::TWO) copyPlanes(g.Xlo + size_t(c.cur) * g.xB, g.nS, v.Xlo, v.nS, I.n0, I.n, 3);
  copyPlanes(g.V, g.nS, v.V, v.nS, I.n0, I.n, 3);
  copyPlanes(g.Q + size_t(c.cur) * g.qB, g.mS, v.Q, v.mS, I.m0, I.m, 4);
  if constexpr (PrecT<P>::TWO) copyPlanes(g.Qlo + size_t(c.cur) * g.qB, g.mS, v.Qlo, v.mS, I.m0, I.m, 4);
  copyPlanes(g.Wr, g.mS, v.Wr, v.mS, I.m0, I.m, 3);
  if (!I.K) return;
  copyPlanes(g.u, g.kS, v.u, v.kS, I.k0, I.K, 2);
  copyPlanes(g.nPrev, g.kS, v.nPrev, v.kS, I.k0, I.K, 3);
  const int k2 = 2 * I.k0, K2 = 2 * I.K, ob = c.obuf;
  copyPlanes(g.ordSeg + size_t(ob) * g.oB, 0, v.ordSeg + size_t(ob) * v.oB, 0, k2, K2, 1);
  copyPlanes(g.rngLo, g.rB, v.rngLo, v.rB, I.m0, I.m, 2);
  copyPlanes(g.rngHi, g.rB, v.rngHi, v.rB, I.m0, I.m, 2);
  if constexpr (SHORT) copyPlanes(g.sInv + size_t(ob) * g.kB, 0, v.sInv + size_t(ob) * v.kB, 0, k2, K2, 1);
  else copyPlanes(g.ord + size_t(ob) * g.oB, 0, v.ord + size_t(ob) * v.oB, 0, k2, K2, 1);
}

// positions / frames of node i or segment j between the shared view and global buffer bk (backup or restore)
template <int P>
__device__ __forceinline__ void backupNode(const Dev<P> &g, const Dev<P> &v, int bk, int i, bool restore) {
  for (int k = 0; k < 3; k++) {
    const size_t go = size_t(bk) * g.xB + size_t(k) * g.nS + i, so = size_t(k) * v.nS + i;
    if (restore) { v.X[so] = g.X[go]; if constexpr (PrecT<P>::TWO) v.Xlo[so] = g.Xlo[go]; }
    else { g.X[go] = v.X[so]; if constexpr (PrecT<P>::TWO) g.Xlo[go] = v.Xlo[so]; }
  }
}
template <int P>
__device__ __forceinline__ void backupSeg(const Dev<P> &g, const Dev<P> &v, int bk, int j, bool restore) {
  for (int k = 0; k < 4; k++) {
    const size_t go = size_t(bk) * g.qB + size_t(k) * g.mS + j, so = size_t(k) * v.mS + j;
    if (restore) { v.Q[so] = g.Q[go]; if constexpr (PrecT<P>::TWO) v.Qlo[so] = g.Qlo[go]; }
    else { g.Q[go] = v.Q[so]; if constexpr (PrecT<P>::TWO) g.Qlo[go] = v.Qlo[so]; }
  }
}

template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(512, 1) k_resident(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                      const int *__restrict__ order, int nInst, int nIter, const uint8_t *__restrict__ mask) {
  using A = typename Dev<P>::A;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  const int nwB = blockDim.x >> 5, wB = threadIdx.x >> 5;
  for (int bi = blockIdx.x; bi < nInst; bi += gridDim.x) {
    const int b = order ? order[bi] : bi;
    if (mask && !mask[b]) continue;
    if (threadIdx.x == 0) { sc = ctl[b]; si = insts[b]; sc.tBeg = globalTimer(); }
    __syncthreads();
    const InstDesc &I = si;
    const ResLayout L = residentLayout<P>(I.n, I.m, I.p, I.C, I.K, SHORT);
    const Dev<P> v = residentView<P>(d, I, smem, L, SHORT);
    const int bk = sc.cur ^ 1;          // global buffer that holds the start of each iteration (roll-back)
    residentLoad<P, SHORT>(d, v, I, sc, sc.cur);
    __syncthreads();
    const bool cx = I.contacts && I.K;
    for (int it = 0; it < nIter; it++) {
      if (sc.status != WS_RUNNING) break;
      StepCtx sx = makeCtx<A>(I, sc, EXT ? d.ext[I.utmIdx].pf : nullptr);
      sx.cur = sx.nxt = 0;              // in place
      Part<A> pt;
      pt.init();
      blockPhaseA<P, SHORT, EXT>(v, I, sx, pt, nwB, wB);
      __syncthreads();
      if (!SHORT && cx) {
        blockPhaseBC<P>(v, I, sx, nwB, wB);
        __syncthreads();
      }
      auto upd = [&](int r, int e) {
        if (r == 0) {
          if (I.kd) backupNode<P>(d, v, bk, I.n0 + e, false);
          nodeUpdate<P, SHORT, EXT>(v, I, sx, I.n0 + e, pt);
        } else if (r == 1) {
          if (I.kd) backupSeg<P>(d, v, bk, I.m0 + e, false);
          segUpdate<P, SHORT>(v, I, sx, I.m0 + e, pt);
        } else {
          rankSideWindow<P>(v, 2 * I.k0 + e, sx.obuf, sx.onxt);
        }
      };
      const int nR = (SHORT && cx) ? 2 * I.K : 0;
      if (I.localLoads) {               // node-frame loads read the frames before the segments update them
        const PhaseRun nodes[3] = {{I.n, COST_NODE_UPD}, {0, COST_SEG_UPD}, {nR, COST_RANK}};
        const PhaseRun segs[3] = {{0, COST_NODE_UPD}, {I.m, COST_SEG_UPD}, {0, COST_RANK}};
        forBalanced(nodes, upd);
        __syncthreads();
        forBalanced(segs, upd);
      } else {
        const PhaseRun runs[3] = {{I.n, COST_NODE_UPD}, {I.m, COST_SEG_UPD}, {nR, COST_RANK}};
        forBalanced(runs, upd);
      }
      __syncthreads();
      blockReduce(pt, red);
      if (threadIdx.x == 0) decide<EXT>(I, sc, pt, nIter);
      __syncthreads();
      if (sc.pending) {                 // roll-back: the positions and frames of the iteration's start
        for (int e = threadIdx.x; e < I.n + I.m; e += blockDim.x) {
          if (e < I.n) backupNode<P>(d, v, bk, I.n0 + e, true);
          else backupSeg<P>(d, v, bk, I.m0 + (e - I.n), true);
        }
        __syncthreads();
      }
      if constexpr (EXT) {
        if (threadIdx.x == 0) protocolStep<P>(v, 0, I, sc, pt);
        __syncthreads();
      }
    }
    residentStore<P, SHORT>(d, v, I, sc);
    if (threadIdx.x == 0) { sc.tEnd = globalTimer(); ctl[b] = sc; }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------ plain form
// the sum and max slots each part of a phase feeds: element phase whole (0), crossings (1), rods (2); update phase
// whole (0), nodes with the side ranks (1), segments (2)
constexpr unsigned elemSums(int part) { return part == 1 ? SUMS_CROSS : part == 2 ? SUMS_ROD : (SUMS_CROSS | SUMS_ROD); }
constexpr unsigned elemMaxs(int part) { return part == 1 ? MAXS_CROSS : part == 2 ? MAXS_ROD : (MAXS_CROSS | MAXS_ROD); }
constexpr unsigned updateSums(int part, bool ext) { return SUMS_UPDATE | (ext && part != 2 ? SUMS_FLOOR : 0u); }
constexpr unsigned updateMaxs(int part, bool ext) {
  return (part == 1 ? ((1u << RX_F) | (1u << RX_LOAD)) : part == 2 ? (1u << RX_T) : MAXS_UPDATE) |
         (ext && part != 2 ? MAXS_FLOOR : 0u);
}
// every block partial of one iteration, in ranges of fixed order, each read only in the slots its kernel feeds (the
// others hold nothing): SPLIT, the four kernels of the split phases; else the two whole phases.  In round o thread t
// reads row o + t of every range at once, so the close takes as many rounds of loads as the longest range has rows
// per thread (one for a small instance), not the sum over the ranges.
template <bool SPLIT, bool EXT, class A>
__device__ __forceinline__ void reduceIteration(Part<A> &q, const A *part, int ex, int ey, int en, int em, int stride) {
  if constexpr (SPLIT) {
    const int len = max(max(ex, ey - ex), max(en - ey, em - en)), bd = blockDim.x;
    int o0 = threadIdx.x;
    // two rounds at a time: the rows of both go out in one batch of loads, then they are added in round order
    for (; o0 + bd < len; o0 += 2 * bd) {
      RangeRow<elemSums(1), elemMaxs(1), A> x0, x1;
      RangeRow<elemSums(2), elemMaxs(2), A> y0, y1;
      RangeRow<updateSums(1, EXT), updateMaxs(1, EXT), A> n0, n1;
      RangeRow<updateSums(2, EXT), updateMaxs(2, EXT), A> m0, m1;
      x0.load(part, o0, ex, stride); y0.load(part, ex + o0, ey, stride);
      n0.load(part, ey + o0, en, stride); m0.load(part, en + o0, em, stride);
      const int o1 = o0 + bd;
      x1.load(part, o1, ex, stride); y1.load(part, ex + o1, ey, stride);
      n1.load(part, ey + o1, en, stride); m1.load(part, en + o1, em, stride);
      x0.add(q); y0.add(q); n0.add(q); m0.add(q);
      x1.add(q); y1.add(q); n1.add(q); m1.add(q);
    }
    for (int o = o0; o < len; o += bd) {
      addRangeRow<elemSums(1), elemMaxs(1)>(q, part, o, ex, stride);
      addRangeRow<elemSums(2), elemMaxs(2)>(q, part, ex + o, ey, stride);
      addRangeRow<updateSums(1, EXT), updateMaxs(1, EXT)>(q, part, ey + o, en, stride);
      addRangeRow<updateSums(2, EXT), updateMaxs(2, EXT)>(q, part, en + o, em, stride);
    }
  } else {
    const int len = max(ex, em - ex);
    for (int o = threadIdx.x; o < len; o += blockDim.x) {
      addRangeRow<elemSums(0), elemMaxs(0)>(q, part, o, ex, stride);
      addRangeRow<updateSums(0, EXT), updateMaxs(0, EXT)>(q, part, ex + o, em, stride);
    }
  }
}
// One kernel per phase over the elements of instance 0; block partials go to part[block] and the last block of the
// update kernel reduces them in a fixed order.  Every kernel returns at once when the instance has stopped.
// The element phase, whole (PART 0) or split in two kernels that run side by side on forked branches of the graph:
// the crossings (PART 1), whose long per-element code needs many registers, and the segments, joints and clamps
// (PART 2), which then run at the occupancy of their own, smaller register budget.
template <int P, bool SHORT, bool EXT, int PART>
__device__ __forceinline__ void plainA(const Dev<P> &d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl,
                                       typename Dev<P>::A *part, int partStride, int blk, int nblk) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  const InstDesc &I = insts[0];
  const InstCtl c = ctl[0];
  if (c.status != WS_RUNNING) return;
  const int nK = (I.contacts && I.K) ? I.K : 0;
  const int nA = PART == 1 ? 2 * nK : PART == 2 ? max(I.m, I.p + I.C) : countA(I);
  const StepCtx sx = makeCtx<A>(I, c);
  Part<A> pt;
  pt.init();
  // each part compiles only its own element code (a branch the part never takes still costs registers)
  for (int e = blk * blockDim.x + threadIdx.x; e < nA; e += nblk * blockDim.x) {
    if (PART == 1) crossElement<P, SHORT, EXT>(d, I, sx, e, pt);
    else if (PART == 2) rodPair<P>(d, I, sx, e, pt);
    else phaseA<P, SHORT, EXT>(d, I, sx, e, nK, pt);
  }
  constexpr unsigned SM = elemSums(PART), XM = elemMaxs(PART);
  blockReduce<SM, XM>(pt, red);
  if (threadIdx.x == 0) putPartSlots<SM, XM>(pt, part, blk, partStride);
}
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(256, WSB_MINB_A) k_plainA(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl,
                                                typename Dev<P>::A *part, int partStride) {
  waitPrevGrid();
  allowNextGrid();
  plainA<P, SHORT, EXT, 0>(d, insts, ctl, part, partStride, blockIdx.x, gridDim.x);
}
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(128) k_plainX(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl,
                                                typename Dev<P>::A *part, int partStride) {
  plainA<P, SHORT, EXT, 1>(d, insts, ctl, part, partStride, blockIdx.x, gridDim.x);
}
template <int P, bool SHORT>
__global__ void __launch_bounds__(WSB_Y_THREADS(P), WSB_MINB_Y(P)) k_plainY(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl,
                                                typename Dev<P>::A *part, int partStride) {
  plainA<P, SHORT, false, 2>(d, insts, ctl, part, partStride, blockIdx.x, gridDim.x);
}
// The element phase as one launch whose blocks take roles: the first nbX blocks the crossings, the others the segments,
// joints and clamps, so both run side by side without a fork in the graph; partials at part[block] in that order.
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(256, WSB_MINB_XY) k_plainXY(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl,
                                                 typename Dev<P>::A *part, int partStride, int nbX) {
  waitPrevGrid();
  allowNextGrid();
  if (int(blockIdx.x) < nbX) plainA<P, SHORT, EXT, 1>(d, insts, ctl, part, partStride, blockIdx.x, nbX);
  else plainA<P, SHORT, false, 2>(d, insts, ctl, part + nbX, partStride, blockIdx.x - nbX, gridDim.x - nbX);
}
template <int P>
__global__ void __launch_bounds__(256) k_plainBC(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl) {
  using A = typename Dev<P>::A;
  waitPrevGrid();
  allowNextGrid();
  const InstDesc &I = insts[0];
  const InstCtl c = ctl[0];
  if (c.status != WS_RUNNING) return;
  const StepCtx sx = makeCtx<A>(I, c);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * I.K + I.m; e += gridDim.x * blockDim.x) phaseBC<P>(d, I, sx, e);
}
// The end of an iteration without the extensions, run by the update phase's last block: every block partial reduced in
// a fixed order, then the kinetic-damping decision.  Out of line, so that its registers do not count against the
// element loop's budget.  The control block is read again here: no block writes it before this one.
// ---- the split close: one slot of one range of partials a warp
// One slot of a range of block partials (rows [lo, hi)), a sum or a maximum, reduced by one warp: lane l takes rows
// lo + l, lo + l + 32, ... in row order, the loads of a pass issued together, then a butterfly over the lanes leaves
// the same value in every lane.
template <class A>
__device__ __forceinline__ A warpSlot(const A *part, int stride, int slot, bool mx, A ident, int lo, int hi) {
  const int lane = threadIdx.x & 31;
  const A *p = part + size_t(slot) * stride;
  A acc = ident;
  constexpr int U = 12;
  for (int b0 = lo; b0 < hi; b0 += 32 * U) {
    A v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int b = b0 + lane + 32 * u;
      v[u] = b < hi ? __ldcg(p + b) : ident;
    }
#pragma unroll
    for (int u = 0; u < U; u++) acc = mx ? mmax(acc, v[u]) : acc + v[u];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const A w = __shfl_xor_sync(0xffffffffu, acc, o);
    acc = mx ? mmax(acc, w) : acc + w;
  }
  return acc;
}
// a range of partial rows and the slots its kernel feeds
struct SlotRange { int lo, hi; unsigned sums, maxs; };
// the k-th (range, slot) item of ranges r[0..nr), sum slots before maximum slots within a range; false past the end
__device__ __forceinline__ bool slotItem(const SlotRange *r, int nr, int k, int &ri, int &slot, bool &mx) {
  for (int i = 0; i < nr; i++) {
    for (int b = 0; b < RS_NSUM + RX_NMAX; b++) {
      const bool isMax = b >= RS_NSUM;
      const unsigned m = isMax ? r[i].maxs : r[i].sums;
      if (!(m & (1u << (isMax ? b - RS_NSUM : b)))) continue;
      if (k == 0) { ri = i; slot = b; mx = isMax; return true; }
      k--;
    }
  }
  return false;
}
__device__ __forceinline__ int slotItems(const SlotRange *r, int nr) {
  int n = 0;
  for (int i = 0; i < nr; i++) n += __popc(r[i].sums) + __popc(r[i].maxs);
  return n;
}
// identity of a slot: 0, or -inf for the largest normal force
template <class A> __device__ __forceinline__ A slotIdent(int slot) { return slot == RS_NSUM + RX_FN ? -A(INFINITY) : A(0); }
// every item of the ranges, one a warp (warp w: items w, w + warps, ...), values into vals[item] (shared); then
// thread 0 folds them into q in item order (ranges in order), so the result does not depend on timing
template <class A>
__device__ __forceinline__ void slotsToVals(const SlotRange *r, int nr, const A *part, int stride, A *vals) {
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
  const int n = slotItems(r, nr);
  for (int k = warp; k < n; k += nw) {
    int ri, slot;
    bool mx;
    slotItem(r, nr, k, ri, slot, mx);
    const A v = warpSlot(part, stride, slot, mx, slotIdent<A>(slot), r[ri].lo, r[ri].hi);
    if (lane == 0) vals[k] = v;
  }
}
// thread 0, after a barrier: the items' values folded into q in item order
template <class A>
__device__ __forceinline__ void foldVals(const SlotRange *r, int nr, const A *vals, Part<A> &q) {
  const int n = slotItems(r, nr);
  for (int k = 0; k < n; k++) {
    int ri, slot;
    bool mx;
    slotItem(r, nr, k, ri, slot, mx);
    if (mx) q.x[slot - RS_NSUM] = mmax(q.x[slot - RS_NSUM], vals[k]);
    else q.s[slot] += vals[k];
  }
}
template <class A>
__device__ __forceinline__ void reduceSlots(const SlotRange *r, int nr, const A *part, int stride, A *vals, Part<A> &q) {
  const int n = slotItems(r, nr);
  slotsToVals(r, nr, part, stride, vals);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < n; k++) {
      int ri, slot;
      bool mx;
      slotItem(r, nr, k, ri, slot, mx);
      if (mx) q.x[slot - RS_NSUM] = mmax(q.x[slot - RS_NSUM], vals[k]);
      else q.s[slot] += vals[k];
    }
  }
}

// fetch-and-add on a GPU-scope counter with acquire-release semantics: the calling thread's earlier writes become
// visible to any thread that later acquires the counter, and the caller sees the writes released by the earlier adds
__device__ __forceinline__ unsigned long long ticketAdd(unsigned long long *p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
// The node kernel's last block (split update phase without the extensions): the partials of the crossings, the rods and
// the nodes reduced into the summary row S (slot i at S[i]), which the iteration's close reads instead of their rows.
template <class A>
__device__ __noinline__ void summariseNodes(const A *partAll, int ex, int ey, int en, int stride, A *S) {
  __shared__ A vals[32];
  const SlotRange r[3] = {{0, ex, elemSums(1), elemMaxs(1)}, {ex, ey, elemSums(2), elemMaxs(2)},
                          {ey, en, updateSums(1, false), updateMaxs(1, false)}};
  Part<A> q;
  q.init();
  reduceSlots(r, 3, partAll, stride, vals, q);
  if (threadIdx.x == 0) {
    for (int i = 0; i < RS_NSUM; i++) S[i] = q.s[i];
    for (int i = 0; i < RX_NMAX; i++) S[RS_NSUM + i] = q.x[i];
  }
}
// The element summary block of the node kernel (fork launch without the extensions): the crossing and rod partials,
// complete before the update phase starts, reduced into the summary row S by one extra block of the node kernel while
// the other blocks update the nodes, so that the close that follows the update blocks reads only the summary and the
// update kernels' own partials.
template <class A>
__device__ __noinline__ void summariseElements(const A *partAll, int ex, int ey, int stride, A *S) {
  __shared__ A vals[32];
  const SlotRange r[2] = {{0, ex, elemSums(1), elemMaxs(1)}, {ex, ey, elemSums(2), elemMaxs(2)}};
  Part<A> q;
  q.init();
  reduceSlots(r, 2, partAll, stride, vals, q);
  if (threadIdx.x == 0) {
    for (int i = 0; i < RS_NSUM; i++) S[i] = q.s[i];
    for (int i = 0; i < RX_NMAX; i++) S[RS_NSUM + i] = q.x[i];
  }
}
// The close of a split iteration without the extensions: the summary row and the segment kernel's partials (rows
// [en, em)) and, with NODES, the node kernel's partials (rows [ey, en)), one item a warp, then the kinetic-damping
// decision.  The control block, the descriptor and the summary row
// are copied to shared memory a word a thread, their loads in flight beside the partials'.
template <class A, bool NODES>
__device__ __noinline__ void closeSplit(const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl, const A *partAll,
                                        int ey, int en, int em, int stride, const A *S, unsigned long long *counter) {
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  __shared__ A vals[8], sS[RS_NSUM + RX_NMAX];
  constexpr int NC = sizeof(InstCtl) / 4, ND = sizeof(InstDesc) / 4, NV = RS_NSUM + RX_NMAX;
  static_assert(NC <= 64 && 64 + ND <= 224 && NV <= 32, "the copies take one word a thread of a 256-thread block");
  // the items the close reduces, fixed at compile time (a warp each): the node rows [ey, en) feed the kinetic energy
  // and the largest force and load, the segment rows [en, em) the kinetic energy and the largest torque
  static_assert(updateSums(1, false) == (1u << RS_KE) && updateMaxs(1, false) == ((1u << RX_F) | (1u << RX_LOAD)) &&
                updateSums(2, false) == (1u << RS_KE) && updateMaxs(2, false) == (1u << RX_T), "the close's items");
  constexpr int NI = NODES ? 5 : 2;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  int wc = 0, wd = 0;
  A ws = A(0);
  if (t < NC) wc = __ldcg(reinterpret_cast<const int *>(ctl) + t);
  if (t >= 64 && t < 64 + ND) wd = __ldg(reinterpret_cast<const int *>(insts) + (t - 64));
  if (t >= 224 && t < 224 + NV) ws = __ldcg(S + (t - 224));
  if (warp < NI) {
    const int k = NODES ? warp : warp + 3;          // 0-2 node items, 3-4 segment items
    const bool seg = k >= 3, mx = k == 1 || k == 2 || k == 4;
    const int slot = k == 1 ? RS_NSUM + RX_F : k == 2 ? RS_NSUM + RX_LOAD : k == 4 ? RS_NSUM + RX_T : RS_KE;
    const A v = warpSlot(partAll, stride, slot, mx, A(0), seg ? en : ey, seg ? em : en);
    if (lane == 0) vals[warp] = v;
  }
  if (t < NC) reinterpret_cast<int *>(&sc)[t] = wc;
  if (t >= 64 && t < 64 + ND) reinterpret_cast<int *>(&si)[t - 64] = wd;
  if (t >= 224 && t < 224 + NV) sS[t - 224] = ws;
  __syncthreads();
  if (t == 0) {
    Part<A> q;
    for (int i = 0; i < RS_NSUM; i++) q.s[i] = sS[i];
    for (int i = 0; i < RX_NMAX; i++) q.x[i] = sS[RS_NSUM + i];
    if constexpr (NODES) {
      q.s[RS_KE] += vals[0];
      q.x[RX_F] = mmax(q.x[RX_F], vals[1]);
      q.x[RX_LOAD] = mmax(q.x[RX_LOAD], vals[2]);
      q.s[RS_KE] += vals[3];
      q.x[RX_T] = mmax(q.x[RX_T], vals[4]);
    } else {
      q.s[RS_KE] += vals[0];
      q.x[RX_T] = mmax(q.x[RX_T], vals[1]);
    }
    InstCtl cc = sc;
    decide<false>(si, cc, q, 0);
    ctl[0] = cc;
    *counter = 0ull;
  }
}
template <bool SPLIT, class A>
__device__ __noinline__ void closeIteration(const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl, const A *partAll,
                                            int ex, int ey, int en, int em, int partStride, unsigned *counter, A *red) {
  // the control block and the descriptor go to shared memory a word a thread, their loads in flight beside the
  // partials' (the decision then reads them there instead of waiting on one global load after another)
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  constexpr int NC = sizeof(InstCtl) / 4, ND = sizeof(InstDesc) / 4;
  static_assert(NC <= 64 && 64 + ND <= 256, "the copy takes one word a thread of a 256-thread block");
  const int t = threadIdx.x;
  int wc = 0, wd = 0;
  if (t < NC) wc = __ldcg(reinterpret_cast<const int *>(ctl) + t);
  if (t >= 64 && t < 64 + ND) wd = __ldg(reinterpret_cast<const int *>(insts) + (t - 64));
  Part<A> q;
  q.init();
  reduceIteration<SPLIT, false>(q, partAll, ex, ey, en, em, partStride);
  if (t < NC) reinterpret_cast<int *>(&sc)[t] = wc;
  if (t >= 64 && t < 64 + ND) reinterpret_cast<int *>(&si)[t - 64] = wd;
  blockReduce<SUMS_ALL & ~SUMS_FLOOR, MAXS_ALL>(q, red);      // (its barriers also publish the copies)
  if (t == 0) {
    InstCtl cc = sc;
    decide<false>(si, cc, q, 0);
    ctl[0] = cc;
    *counter = 0;
  }
}
// The update kernel also closes the iteration: every block publishes its partials, and the last block to finish
// (counted on `counter` over all `nBlocks` blocks of the update phase) reduces the partials of phases A and D in a
// fixed order and takes the kinetic-damping decision.  Every block reads the control block before it counts itself,
// so the last block's write cannot race a reader.  The phase runs whole (PART 0) or split in two kernels on forked
// branches: the nodes with the side ranks (PART 1) and the segments (PART 2), each at its own register budget.
// XYS (the fork launch without the extensions): the node kernel has one block more than its node blocks (blk == nblk),
// which summarises the crossing and rod partials while the others update the nodes; every block of the pair then takes
// one ticket, and the last closes the iteration from that summary and the node and segment partials.
template <int P, bool SHORT, bool EXT, int PART, bool XYS = false>
__device__ __forceinline__ void plainD(const Dev<P> &d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                       typename Dev<P>::A *part, typename Dev<P>::A *partAll, const PartEnds &pe,
                                       int partStride, unsigned *counter, unsigned nBlocks, int blk, int nblk) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  __shared__ bool last;
  const InstDesc &I = insts[0];
  const InstCtl c = ctl[0];
  if (c.status != WS_RUNNING) return;
  if constexpr (XYS && !EXT && PART == 1)
    if (blk == nblk) {
      unsigned long long *cnt = reinterpret_cast<unsigned long long *>(counter);
      A *S = partAll + size_t(RS_NSUM + RX_NMAX) * partStride;
      summariseElements<A>(partAll, pe.x, pe.y, partStride, S);
      if (threadIdx.x == 0) last = unsigned(ticketAdd(cnt, 1ull)) + 1u == nBlocks;
      __syncthreads();
      if (last) closeSplit<A, true>(insts, ctl, partAll, pe.y, pe.n, pe.m, partStride, S, cnt);
      return;
    }
  const StepCtx sx = makeCtx<A>(I, c, EXT ? d.ext[I.utmIdx].pf : nullptr);
  Part<A> pt;
  pt.init();
  const int nR = countD<SHORT>(I) - I.n - I.m;
  const int nD = PART == 1 ? I.n + nR : PART == 2 ? I.m : countD<SHORT>(I);
  for (int e = blk * blockDim.x + threadIdx.x; e < nD; e += nblk * blockDim.x) {
    if (PART == 0) phaseD<P, SHORT, EXT>(d, I, sx, e, pt);
    else if (PART == 2) segUpdate<P, SHORT>(d, I, sx, I.m0 + e, pt);
    else if (e < I.n) nodeUpdate<P, SHORT, EXT>(d, I, sx, I.n0 + e, pt);
    else rankSideWindow<P>(d, 2 * I.k0 + (e - I.n), sx.obuf, sx.onxt);
  }
  constexpr unsigned SM = updateSums(PART, EXT), XM = updateMaxs(PART, EXT);
  blockReduce<SM, XM>(pt, red);
  if constexpr (XYS && !EXT && PART != 0) {
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(counter);
    const A *S = partAll + size_t(RS_NSUM + RX_NMAX) * partStride;
    if (threadIdx.x == 0) {
      putPartSlots<SM, XM>(pt, part, blk, partStride);
      last = unsigned(ticketAdd(cnt, 1ull)) + 1u == nBlocks;
    }
    __syncthreads();
    if (!last) return;
    closeSplit<A, true>(insts, ctl, partAll, pe.y, pe.n, pe.m, partStride, S, cnt);
    return;
  }
  if constexpr (!EXT && PART != 0) {
    // The split update phase counts its blocks on one 64-bit counter: node blocks in the high word, segment blocks
    // in the low word.  The node kernel's last block summarises the partials of the crossings, the rods and the nodes
    // (summariseNodes), then adds all node blocks to the low word at once; the block that brings the low word to the
    // total closes the iteration from the summary and the segment partials (closeSplit).
    __shared__ int role;                       // 0 done, 1 summarise, 2 close
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(counter);
    A *S = partAll + size_t(RS_NSUM + RX_NMAX) * partStride;
    // The tickets are acquire-release fetch-and-adds by thread 0, which also wrote the block's partials (and the
    // summary): its writes are released with its ticket, and the block that takes the last ticket acquires every
    // earlier one before its barrier, after which its threads read the partials from L2 (no separate fences).
    if (threadIdx.x == 0) {
      putPartSlots<SM, XM>(pt, part, blk, partStride);
      const unsigned long long old = ticketAdd(cnt, PART == 1 ? (1ull << 32) : 1ull);
      role = (PART == 1 && unsigned(old >> 32) == unsigned(nblk) - 1u) ? 1
             : (PART == 2 && unsigned(old) + 1u == nBlocks) ? 2 : 0;
    }
    __syncthreads();
    const int rl = role;
    if (rl == 0) return;
    if (rl == 1) {
      summariseNodes<A>(partAll, pe.x, pe.y, pe.n, partStride, S);
      if (threadIdx.x == 0) {
        const unsigned long long old = ticketAdd(cnt, (unsigned long long)unsigned(nblk));
        role = unsigned(old) + unsigned(nblk) == nBlocks ? 2 : 0;
      }
      __syncthreads();
      if (role != 2) return;
    }
    closeSplit<A, false>(insts, ctl, partAll, 0, pe.n, pe.m, partStride, S, cnt);
    return;
  }
  if (threadIdx.x == 0) {
    putPartSlots<SM, XM>(pt, part, blk, partStride);
    __threadfence();
    last = atomicAdd(counter, 1u) == nBlocks - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if constexpr (!EXT) {
    closeIteration<PART != 0, A>(insts, ctl, partAll, pe.x, pe.y, pe.n, pe.m, partStride, counter, red);
    return;
  }
  if (I.rbOn) return;             // a model only the ground holds: k_rigidClose closes the iteration after this kernel
  Part<A> q;
  q.init();
  reduceIteration<PART != 0, EXT>(q, partAll, pe.x, pe.y, pe.n, pe.m, partStride);
  blockReduce(q, red);
  if (threadIdx.x == 0) {
    InstCtl cc = c;
    decide<EXT>(I, cc, q, 0);
    if constexpr (EXT) protocolStep<P>(d, cc.cur, I, cc, q);
    ctl[0] = cc;
    *counter = 0;
  }
}
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(256, WSB_MINB_D) k_plainD(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                typename Dev<P>::A *part, typename Dev<P>::A *partAll, PartEnds pe,
                                                int partStride, unsigned *counter) {
  waitPrevGrid();
  allowNextGrid();
  plainD<P, SHORT, EXT, 0>(d, insts, ctl, part, partAll, pe, partStride, counter, gridDim.x, blockIdx.x, gridDim.x);
}
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(256, WSB_MINB_DN(P, EXT)) k_plainDN(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                  typename Dev<P>::A *part, typename Dev<P>::A *partAll, PartEnds pe,
                                                  int partStride, unsigned *counter, unsigned nBlocks) {
  plainD<P, SHORT, EXT, 1, !EXT>(d, insts, ctl, part, partAll, pe, partStride, counter, nBlocks, blockIdx.x,
                                  EXT ? gridDim.x : gridDim.x - 1);
}
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(256, WSB_MINB_DM(P, EXT)) k_plainDM(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                  typename Dev<P>::A *part, typename Dev<P>::A *partAll, PartEnds pe,
                                                  int partStride, unsigned *counter, unsigned nBlocks) {
  plainD<P, SHORT, EXT, 2, !EXT>(d, insts, ctl, part, partAll, pe, partStride, counter, nBlocks, blockIdx.x, gridDim.x);
}
// The update phase as one launch with roles: the first nbN blocks the nodes (with the side ranks of the short order),
// the others the segments; the last of all its blocks closes the iteration.
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(256, WSB_MINB_DN(P, EXT)) k_plainDNM(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                   typename Dev<P>::A *part, typename Dev<P>::A *partAll, PartEnds pe,
                                                   int partStride, unsigned *counter, int nbN) {
  waitPrevGrid();
  allowNextGrid();
  if (int(blockIdx.x) < nbN)
    plainD<P, SHORT, EXT, 1>(d, insts, ctl, part, partAll, pe, partStride, counter, gridDim.x, blockIdx.x, nbN);
  else
    plainD<P, SHORT, EXT, 2>(d, insts, ctl, part + nbN, partAll, pe, partStride, counter, gridDim.x, blockIdx.x - nbN,
                             gridDim.x - nbN);
}

// The close of a plain-form iteration of a model that only the ground holds (one block, launched after the update
// kernels): every block partial reduced as the update kernel's last block would, then the rigid-body freedoms (their
// sums need the ground's forces of every node) with the kinetic-damping decision, and the rigid step of the new buffer.
template <int P, bool SPLIT>
__global__ void __launch_bounds__(1024) k_rigidClose(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                     const typename Dev<P>::A *partAll, PartEnds pe, int partStride,
                                                     unsigned *counter) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  __shared__ InstCtl sc;
  const InstDesc &I = insts[0];
  if (threadIdx.x == 0) sc = ctl[0];
  __syncthreads();
  if (sc.status != WS_RUNNING) return;
  const StepCtx sx = makeCtx<A>(I, sc);
  Part<A> q;
  q.init();
  reduceIteration<SPLIT, true>(q, partAll, pe.x, pe.y, pe.n, pe.m, partStride);
  blockReduce(q, red);
  rigidBlockStep<P, true>(d, I, sx, sc, d.ext[I.utmIdx], q, 0);
  if (threadIdx.x == 0) {
    d.ext[I.utmIdx].eFloor = double(q.s[RS_FLOOR]);
    ctl[0] = sc;
    *counter = 0;
  }
}

// ------------------------------------------------------------------------------------------------ grid form
// Grid-wide barrier for a cooperative launch (every block resident).  The wait is bounded: past ~2^24 polls (about a
// second) it raises *err and every block leaves its iteration loop, so a kernel never hangs the device.
__device__ __forceinline__ bool gridSync(unsigned *bar, unsigned nb, int *err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = atomicAdd(bar + 1, 0u);
    __threadfence();
    if (atomicAdd(bar, 1u) == nb - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned long long spins = 0;
      while (atomicAdd(bar + 1, 0u) == g) {
        if (++spins > (1ull << 24) || atomicAdd(err, 0) != 0) { atomicExch(err, 1); break; }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *reinterpret_cast<volatile int *>(err) == 0;
}

// One instance over the whole (co-resident) grid, every phase of up to nIter iterations in one launch: two grid
// barriers per iteration with the short-slide order, three with the general one.  Block partials go to part[block];
// after the barrier every block reduces all of them in the same order and takes the same kinetic-damping decision, so
// no further broadcast is needed.
template <int P, bool SHORT, bool EXT>
__global__ void __launch_bounds__(256, WSB_MINB_G) k_grid(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                              typename Dev<P>::A *part, unsigned *bar, int *err, int nIter) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  if (threadIdx.x == 0) { sc = ctl[0]; si = insts[0]; }
  __syncthreads();
  const InstDesc &I = si;
  const bool cx = I.contacts && I.K;
  const int nA = countA(I), nD = countD<SHORT>(I);
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const unsigned nb = gridDim.x;
  for (int it = 0; it < nIter; it++) {
    if (sc.status != WS_RUNNING) break;
    const StepCtx sx = makeCtx<A>(I, sc);
    Part<A> pt;
    pt.init();
    for (int e = gt; e < nA; e += gs) phaseA<P, SHORT, EXT>(d, I, sx, e, cx ? I.K : 0, pt);
    if (!gridSync(bar, nb, err)) break;
    if (!SHORT && cx) {
      for (int e = gt; e < 2 * I.K + I.m; e += gs) phaseBC<P>(d, I, sx, e);
      if (!gridSync(bar, nb, err)) break;
    }
    for (int e = gt; e < nD; e += gs) phaseD<P, SHORT, EXT>(d, I, sx, e, pt);
    blockReduce(pt, red);
    if (threadIdx.x == 0) putPart(pt, part, blockIdx.x, int(nb));
    if (!gridSync(bar, nb, err)) break;
    Part<A> q;
    q.init();
    for (int b = threadIdx.x; b < int(nb); b += blockDim.x) addPart(q, part, b, int(nb));
    blockReduce(q, red);
    if (threadIdx.x == 0) decide<EXT>(I, sc, q, nIter);
    if constexpr (EXT)      // the ground's energy (a load protocol is not run in this form)
      if (blockIdx.x == 0 && threadIdx.x == 0) d.ext[I.utmIdx].eFloor = double(q.s[RS_FLOOR]);
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl[0] = sc;
}

// ------------------------------------------------------------------------------------------------ transfers
// Upload: the caller's interleaved f64 state of instance b (X [3n], Q [4m], then u [2K] when given) goes to the device
// as it is; this kernel splits it into the planes (two-float in the mixed policy) of the position / frame buffer the
// control block names, clears the velocities and restarts the kinetic-damping peak.  The order of the sides is
// rebuilt from the new slide coordinates by k_keysFromU and the ranking kernels that follow.
template <int P>
__global__ void __launch_bounds__(256) k_unpack(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl, int b,
                                                const double *__restrict__ in, int withU) {
  using R = typename Dev<P>::R; using W = typename Dev<P>::W; using U = typename Dev<P>::U;
  const InstDesc &I = insts[b];
  const int cur = ctl[b].cur;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const int nX = 3 * I.n, nQ = 4 * I.m, nU = withU ? 2 * I.K : 0;
  // an upload restarts the load protocol from the uploaded probe: P0 = its position, placed at the first value under
  // displacement control (solver_gpu.js:286,296-311)
  const double v0 = I.utmMode ? d.utmSched[size_t(I.utmIdx) * WS_PROTOCOL_MAX_INC] : 0.0;
  for (int e = gt; e < nX; e += gs) {
    const int i = I.n0 + e / 3, k = e % 3;
    const double x = (I.utmMode == 2 && i == I.utmProbe) ? in[e] + I.utmAxis[k] * v0 : in[e];
    Acc<P>::xs(d, cur, k, i, W(x));
    d.V[size_t(k) * d.nS + i] = R(0);
    if (I.floorOn && k < 2) (k == 0 ? d.flAx : d.flAy)[i] = W(x);   // the ground's stick points start under the nodes
  }
  for (int e = gt; e < nQ; e += gs) {
    const int j = I.m0 + e / 4, k = e % 4;
    Acc<P>::qs(d, cur, k, j, W(in[nX + e]));
    if (k < 3) d.Wr[size_t(k) * d.mS + j] = R(0);
  }
  for (int e = gt; e < nU; e += gs) d.u[size_t(e % 2) * d.kS + I.k0 + e / 2] = U(in[nX + nQ + e]);
  if (gt == 0) {
    InstCtl &c = ctl[b];
    c.pending = 0;
    c.ke_prev = 0.0;
    c.status = WS_RUNNING;
    if (I.rbOn)                         // the rigid-body freedoms restart at rest, as the nodes do
      for (int k = 0; k < 3; k++) d.ext[I.utmIdx].rbV[k] = d.ext[I.utmIdx].rbW[k] = 0.0;
    if (I.utmMode) {
      InstExt &u = d.ext[I.utmIdx];
      u.phase = 0; u.it = 0; u.inc = 0; u.accN = 0; u.curF = v0;
      for (int k = 0; k < 4; k++) u.sum[k] = 0.0;
      for (int k = 0; k < 3; k++) {
        u.p0[k] = in[3 * (I.utmProbe - I.n0) + k];
        u.pf[k] = I.utmMode == 1 ? I.utmAxis[k] * v0 : 0.0;
      }
    }
  }
}
// the segment each side sits on now (solver_cpu.js:144-149), from the slide coordinates, into key buffer obuf
template <int P>
__global__ void __launch_bounds__(256) k_keysFromU(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl, int b) {
  using U = typename Dev<P>::U;
  const InstDesc &I = insts[b];
  const int ob = ctl[b].obuf;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * I.K; e += gridDim.x * blockDim.x) {
    const int c = I.k0 + e / 2, side = e % 2;
    const U un = d.u[size_t(side) * d.kS + c];
    const int ns = d.cxNseg[side * d.ktot + c];
    d.sKey[size_t(ob) * d.kB + d.sPos[2 * c + side]] = int(mmin(mmax(mfloor(un), U(0)), U(mmax(ns - 1, 0))));
  }
}
// the order of buffer obuf from its keys: sorted positions / keys / slices (short order) or the sorted list and every
// segment's slice (general order)
template <int P, bool SHORT>
__global__ void __launch_bounds__(256) k_rankOrder(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl, int b) {
  const InstDesc &I = insts[b];
  const int ob = ctl[b].obuf;
  const int n2 = 2 * I.K, nE = SHORT ? n2 : n2 + I.m;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nE; e += gridDim.x * blockDim.x) {
    if (SHORT) rankSideShort<P>(d, 2 * I.k0 + e, ob);
    else if (e < n2) rankSide<P>(d, 2 * I.k0 + e, ob, ob);
    else segCount<P>(d, I.m0 + (e - n2), ob, ob);
  }
}

// the W1 classification of every crossing of instance b from its last evaluation (outputs of a download)
template <int P>
__global__ void __launch_bounds__(256) k_classify(Dev<P> d, const InstDesc *__restrict__ insts, int b) {
  const InstDesc &I = insts[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < I.K; e += gridDim.x * blockDim.x) classify<P>(d, I, I.k0 + e);
}

// the augmented-Lagrangian update of instance b that fell due at the end of its last iteration, applied now (before a
// download reads the multipliers, a warm start resets their window or new slide coordinates arrive); one block
template <int P>
__global__ void __launch_bounds__(256) k_alFlush(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl, int b) {
  const InstDesc &I = insts[b];
  const int pend = ctl[b].alPend, penN = ctl[b].penN, iter = ctl[b].iter;
  __syncthreads();
  if (!pend) return;
  for (int e = threadIdx.x; e < I.K; e += blockDim.x) {
    const int c = I.k0 + e;
    d.lam[c] = alUpdated<P>(d, I, c, iter, penN, d.lam[c], d.penAcc[c], ro(d.cflag + c));
    d.penAcc[c] = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) { ctl[b].alPend = 0; ctl[b].penN = 0; }
}

// Results post-processing (buildResults, solver_cpu.js:878-898): the moment at a node is its joint's (M of the two
// segments' joint), replaced in Mx, My by its clamp's where it has one; a segment takes the mean of its end nodes, and
// the value of the other end where one end has no joint (Mx, My: no joint or clamp)
template <int P>
__device__ __forceinline__ typename Dev<P>::R nodeMoment(const Dev<P> &d, int i, int k) {
  using R = typename Dev<P>::R;
  const int jn = d.nodeJoint[i], cl = d.nodeClamp[i];
  if (k < 2 && cl >= 0) return d.cM[size_t(k) * d.ctot + cl];
  return jn >= 0 ? d.Mj[size_t(k) * d.ptot + jn] : R(0);
}
template <int P>
__global__ void __launch_bounds__(256) k_segResults(Dev<P> d, const InstDesc *__restrict__ insts, int b) {
  const InstDesc &I = insts[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < I.m; e += gridDim.x * blockDim.x) {
    const int j = I.m0 + e, a = d.segI0[j], c = d.segI1[j];
    const bool a0 = d.nodeJoint[a] >= 0, c0 = d.nodeJoint[c] >= 0;
    const bool aB = a0 || d.nodeClamp[a] >= 0, cB = c0 || d.nodeClamp[c] >= 0;
    for (int k = 0; k < 3; k++) {
      const bool ha = k < 2 ? aB : a0, hc = k < 2 ? cB : c0;
      const auto ma = nodeMoment<P>(d, a, k), mc = nodeMoment<P>(d, c, k);
      auto v = decltype(ma)(0.5) * (ma + mc);
      if (!ha) v = mc;
      if (!hc) v = ma;
      d.segM[size_t(k) * d.mtot + j] = v;
    }
  }
}
// the segment layers Mx My T N at the nodes (fields.js nodeValues): the mean of a node's two segments along its strand
// (a closed strand wraps), the one segment at a strand's end
template <int P>
__global__ void __launch_bounds__(256) k_nodeResults(Dev<P> d, const InstDesc *__restrict__ insts, int b) {
  using R = typename Dev<P>::R;
  const InstDesc &I = insts[b];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < I.n; e += gridDim.x * blockDim.x) {
    const int i = I.n0 + e, si = d.nsIn[i], so = d.nsOut[i];
    for (int L = 0; L < 4; L++) {
      auto A = [&](int j) { return L < 3 ? d.segM[size_t(L) * d.mtot + j] : d.Nax[j]; };
      R v = R(0);
      if (si >= 0 && so >= 0) v = R(0.5) * (A(si) + A(so));
      else if (si >= 0) v = A(si);
      else if (so >= 0) v = A(so);
      d.nodeLay[size_t(L) * d.ntot + i] = v;
    }
  }
}

// Download: the requested fields of instance b, interleaved per element as the caller's arrays are (f64, or bytes for
// the stick / slip flags), packed one after another into `out` for a single copy to the host.
template <int P>
__global__ void __launch_bounds__(256) k_pack(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl, int b,
                                              PackList L, unsigned char *__restrict__ out) {
  const InstDesc &I = insts[b];
  const InstCtl c = ctl[b];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  for (int f = 0; f < L.nf; f++) {
    const PackField F = L.f[f];
    const int total = F.count * F.ncomp;
    double *od = reinterpret_cast<double *>(out + F.off);
    unsigned char *ob = out + F.off;
    for (int e = gt; e < total; e += gs) {
      const int i = e / F.ncomp, k = e % F.ncomp;
      switch (F.kind) {
        case PF_X: od[e] = double(Acc<P>::xw(d, c.cur, k, I.n0 + i)); break;
        case PF_Q: od[e] = double(Acc<P>::qw(d, c.cur, k, I.m0 + i)); break;
        case PF_V: od[e] = c.pending ? 0.0 : double(d.V[size_t(k) * d.nS + I.n0 + i]); break;
        case PF_W: od[e] = c.pending ? 0.0 : double(d.Wr[size_t(k) * d.mS + I.m0 + i]); break;
        case PF_U: od[e] = double(d.u[size_t(k) * d.kS + I.k0 + i]); break;
        case PF_NPREV: od[e] = double(d.nPrev[size_t(k) * d.kS + I.k0 + i]); break;
        case PF_SLIP: od[e] = double(d.slip[I.k0 + i]); break;
        case PF_FN: od[e] = double(d.Fn[I.k0 + i]); break;
        case PF_FT: od[e] = double(d.Ft[I.k0 + i]); break;
        case PF_GAP: od[e] = double(d.gap[I.k0 + i]); break;
        case PF_N: od[e] = double(d.Nax[I.m0 + i]); break;
        case PF_VSH: od[e] = double(d.Vsh[size_t(k) * d.mtot + I.m0 + i]); break;
        case PF_M: od[e] = double(d.Mj[size_t(k) * d.ptot + I.p0 + i]); break;
        case PF_REACT: od[e] = double(d.react[size_t(k) * d.ntot + I.n0 + i]); break;
        case PF_STUCK: ob[e] = d.stuck[I.k0 + i]; break;
        case PF_STATE: ob[e] = d.cstate[I.k0 + i]; break;
        case PF_CTYPE: ob[e] = d.ctype[I.k0 + i]; break;
        case PF_THETA: od[e] = double(d.theta[I.k0 + i]); break;
        case PF_PHI: od[e] = double(d.phiS[2 * (I.k0 + i) + k]); break;
        case PF_AREA: od[e] = double(d.area[I.k0 + i]); break;
        case PF_PRES: od[e] = double(d.pres[I.k0 + i]); break;
        case PF_UTIL: od[e] = double(d.util[I.k0 + i]); break;
        case PF_LAM: od[e] = double(d.lam[I.k0 + i]); break;
        case PF_DENT: od[e] = double(d.dent[2 * (I.k0 + i)]) + double(d.dent[2 * (I.k0 + i) + 1]) + double(d.dentE[I.k0 + i]); break;
        case PF_MROT: od[e] = double(d.Mrot[I.k0 + i]); break;
        case PF_RSLIP: od[e] = double(d.rotSlip[I.k0 + i]); break;
        case PF_UTM: od[e] = d.utmOut[size_t(I.utmIdx) * 4 * WS_PROTOCOL_MAX_INC + e]; break;
        case PF_FLF: od[e] = double(d.flF[size_t(k) * d.ntot + I.n0 + i]); break;
        case PF_FLS: ob[e] = d.flState[I.n0 + i]; break;
        case PF_SEGM: od[e] = double(d.segM[size_t(k) * d.mtot + I.m0 + i]); break;
        case PF_NODEM: od[e] = double(d.nodeLay[size_t(k) * d.ntot + I.n0 + i]); break;
        default: od[e] = double(Acc<P>::xw(d, c.cur, k, I.n0 + i)) - double(d.X0[size_t(k) * d.ntot + I.n0 + i]); break;
      }
    }
  }
}

template <int P>
cudaError_t launchUnpack(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, int b, const double *in, int n, int m, int K,
                         bool withU, bool rebuildOrder, bool shortSides, cudaStream_t st) {
  const int work = std::max(3 * n, std::max(4 * m, 2 * K));
  const int blocks = std::max(1, std::min((work + 255) / 256, 148 * 8));
  k_unpack<P><<<blocks, 256, 0, st>>>(d, insts, ctl, b, in, withU ? 1 : 0);
  if (withU && rebuildOrder && K) {
    const int kb = std::max(1, std::min((2 * K + 255) / 256, 148 * 8));
    k_keysFromU<P><<<kb, 256, 0, st>>>(d, insts, ctl, b);
    const int rb = std::max(1, std::min((2 * K + (shortSides ? 0 : m) + 255) / 256, 148 * 8));
    if (shortSides) k_rankOrder<P, true><<<rb, 256, 0, st>>>(d, insts, ctl, b);
    else k_rankOrder<P, false><<<rb, 256, 0, st>>>(d, insts, ctl, b);
  }
  return cudaGetLastError();
}
template <int P>
cudaError_t launchResults(const Dev<P> &d, const InstDesc *insts, int b, int n, int m, cudaStream_t st) {
  if (m > 0) k_segResults<P><<<std::max(1, std::min((m + 255) / 256, 148 * 8)), 256, 0, st>>>(d, insts, b);
  if (n > 0) k_nodeResults<P><<<std::max(1, std::min((n + 255) / 256, 148 * 8)), 256, 0, st>>>(d, insts, b);
  return cudaGetLastError();
}
template <int P>
cudaError_t launchAlFlush(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, int b, cudaStream_t st) {
  k_alFlush<P><<<1, 256, 0, st>>>(d, insts, ctl, b);
  return cudaGetLastError();
}
template <int P>
cudaError_t launchClassify(const Dev<P> &d, const InstDesc *insts, int b, int K, cudaStream_t st) {
  if (K <= 0) return cudaSuccess;
  k_classify<P><<<std::max(1, std::min((K + 255) / 256, 148 * 8)), 256, 0, st>>>(d, insts, b);
  return cudaGetLastError();
}
template <int P>
cudaError_t launchPack(const Dev<P> &d, const InstDesc *insts, const InstCtl *ctl, int b, const PackList &L, size_t elems,
                       unsigned char *out, cudaStream_t st) {
  const int blocks = int(std::max<size_t>(1, std::min<size_t>((elems + 255) / 256, 148 * 8)));
  k_pack<P><<<blocks, 256, 0, st>>>(d, insts, ctl, b, L, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------ launchers
// the variant of kernel K for the side order (sh) and the contact extensions (ex)
#define WSB_PICK(K, P, sh, ex) ((sh) ? ((ex) ? K<P, true, true> : K<P, true, false>) : ((ex) ? K<P, false, true> : K<P, false, false>))

template <int P>
cudaError_t launchBatched(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *order, int nInst, int nIter,
                          const uint8_t *mask, int threads, int blocks, bool shortSides, bool ext, cudaStream_t st) {
  const auto k = WSB_PICK(k_batched, P, shortSides, ext);
  k<<<blocks, threads, 0, st>>>(d, insts, ctl, order, nInst, nIter, mask);
  return cudaGetLastError();
}

template <int P>
cudaError_t launchWide(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *wide, int nWide, int nIter,
                       const uint8_t *mask, int threads, int cluster, bool shortSides, bool ext, cudaStream_t st) {
  if (nWide <= 0) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(nWide * cluster));
  cfg.blockDim = dim3(unsigned(threads));
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(cluster);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, WSB_PICK(k_wide, P, shortSides, ext), d, insts, ctl, wide, nWide, nIter, mask);
}
// clusters of `cluster` blocks of `threads` threads that can be resident at once (0: the shape cannot launch)
template <int P>
int wideClusters(int threads, int cluster, bool shortSides, bool ext) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(cluster));
  cfg.blockDim = dim3(unsigned(threads));
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(cluster);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, WSB_PICK(k_wide, P, shortSides, ext), &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// dynamic shared memory of the resident form for a batch whose largest instance needs `bytes` (0 when it does not fit
// on this device); sets the kernel's limit to it
// (both variants of the side order, with and without the contact extensions)
template <int P>
cudaError_t residentPrepare(size_t bytes, bool shortSides, size_t *granted) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  *granted = 0;
  for (int ex = 0; ex < 2; ex++) {
    const auto k = WSB_PICK(k_resident, P, shortSides, ex != 0);
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, k);
    if (e != cudaSuccess) return e;
    if (bytes + fa.sharedSizeBytes > size_t(optin)) return cudaSuccess;
  }
  // The attribute belongs to the kernel, not to a context: every context of the process launches the same kernel, so
  // it is only ever raised (to the largest instance any context holds), under a lock; lowering it for a context of
  // small instances would make another context's launches fail.
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  for (int ex = 0; ex < 2; ex++) {
    const auto k = WSB_PICK(k_resident, P, shortSides, ex != 0);
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, k);
    if (e != cudaSuccess) return e;
    if (fa.maxDynamicSharedSizeBytes >= int(bytes)) continue;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e != cudaSuccess) return e;
  }
  *granted = bytes;
  return cudaSuccess;
}
template <int P>
cudaError_t launchResident(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *order, int nInst, int nIter,
                           const uint8_t *mask, int threads, size_t smemBytes, bool shortSides, bool ext, cudaStream_t st) {
  const auto k = WSB_PICK(k_resident, P, shortSides, ext);
  k<<<nInst, threads, smemBytes, st>>>(d, insts, ctl, order, nInst, nIter, mask);
  return cudaGetLastError();
}

// a launch of the plain form with programmatic stream serialisation (the kernel may start while its predecessor ends)
template <class... KArgs, class... Args>
static cudaError_t launchPDL(void (*k)(KArgs...), int blocks, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

template <int P>
cudaError_t launchPlainIter(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, const PlainShape &sh, bool contacts,
                            bool shortSides, bool ext, cudaStream_t st, int *launches, unsigned *counter, const PlainFork *fork,
                            bool roles, bool rigid) {
  using A = typename Dev<P>::A;
  const bool sh2 = shortSides && contacts;
  // a model that only the ground holds: its iteration closes in one more launch (k_rigidClose)
  auto rigidClose = [&](bool split, const PartEnds &pe, int nParts) -> cudaError_t {
    if (!rigid) return cudaSuccess;
    const A *pa = static_cast<const A *>(part);
    if (split) k_rigidClose<P, true><<<1, 1024, 0, st>>>(d, insts, ctl, pa, pe, nParts, counter);
    else k_rigidClose<P, false><<<1, 1024, 0, st>>>(d, insts, ctl, pa, pe, nParts, counter);
    if (launches) *launches += 1;
    return cudaGetLastError();
  };
  if (roles && contacts) {
    // two launches with block roles, each scheduled while its predecessor drains (the general order's ranking kernel
    // between them)
    const int nbX = sh.blocksXR, nDN = sh2 ? sh.blocksDNS : sh.blocksDN;
    const int nXY = nbX + sh.blocksY, nParts = nXY + nDN + sh.blocksDM;
    A *px = static_cast<A *>(part), *pn = px + nXY;
    cudaError_t e = launchPDL(WSB_PICK(k_plainXY, P, sh2, ext), nXY, st, d, insts, ctl, px, nParts, nbX);
    if (e != cudaSuccess) return e;
    int nl = 1;
    if (!sh2) {
      if ((e = launchPDL(k_plainBC<P>, sh.blocksR, st, d, insts, ctl)) != cudaSuccess) return e;
      nl += 1;
    }
    const PartEnds pe{nbX, nXY, nXY + nDN, nParts};
    e = launchPDL(WSB_PICK(k_plainDNM, P, sh2, ext), nDN + sh.blocksDM, st, d, insts, ctl, pn, px, pe, nParts, counter,
                  nDN);
    if (e != cudaSuccess) return e;
    nl += 1;
    if (launches) *launches += nl;
    if ((e = rigidClose(true, pe, nParts)) != cudaSuccess) return e;
    return cudaGetLastError();
  }
  if (fork && contacts) {
    // crossings on a forked branch, segments / joints / clamps on the main one, joined before the update; the update
    // forks again: nodes on the side branch, segments and side ranks on the main one
    // rod blocks of WSB_Y_THREADS(P) threads over the rod pairs, one pair a thread
    const int nbY = std::min((sh.pairsY + WSB_Y_THREADS(P) - 1) / WSB_Y_THREADS(P), 148 * 8);
    const int nDN = sh2 ? sh.blocksDNS : sh.blocksDN, nParts = sh.blocksX + nbY + nDN + sh.blocksDM;
    A *px = static_cast<A *>(part), *py = px + sh.blocksX, *pn = py + nbY, *pm = pn + nDN;
    // without the extensions the node kernel runs one more block, which summarises the element partials
    const int xys = ext ? 0 : 1;
    const unsigned nB = unsigned(nDN + xys + sh.blocksDM);
    const PartEnds pe{sh.blocksX, sh.blocksX + nbY, sh.blocksX + nbY + nDN, nParts};
    cudaError_t e;
    if ((e = cudaEventRecord(fork->fork, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(fork->side, fork->fork, 0)) != cudaSuccess) return e;
    const auto kx = WSB_PICK(k_plainX, P, sh2, ext);
    kx<<<sh.blocksX, 128, 0, fork->side>>>(d, insts, ctl, px, nParts);
    if ((e = cudaEventRecord(fork->join, fork->side)) != cudaSuccess) return e;
    if (sh2) k_plainY<P, true><<<nbY, WSB_Y_THREADS(P), 0, st>>>(d, insts, ctl, py, nParts);
    else k_plainY<P, false><<<nbY, WSB_Y_THREADS(P), 0, st>>>(d, insts, ctl, py, nParts);
    if ((e = cudaStreamWaitEvent(st, fork->join, 0)) != cudaSuccess) return e;
    int nl = 2;
    if (!sh2) {
      k_plainBC<P><<<sh.blocksR, 256, 0, st>>>(d, insts, ctl);
      nl += 1;
    }
    if ((e = cudaEventRecord(fork->fork2, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(fork->side, fork->fork2, 0)) != cudaSuccess) return e;
    const auto kdn = WSB_PICK(k_plainDN, P, sh2, ext);
    kdn<<<(sh2 ? sh.blocksDNS : sh.blocksDN) + xys, 256, 0, fork->side>>>(d, insts, ctl, pn, px, pe, nParts, counter, nB);
    if ((e = cudaEventRecord(fork->join2, fork->side)) != cudaSuccess) return e;
    const auto kdm = WSB_PICK(k_plainDM, P, sh2, ext);
    kdm<<<sh.blocksDM, 256, 0, st>>>(d, insts, ctl, pm, px, pe, nParts, counter, nB);
    if ((e = cudaStreamWaitEvent(st, fork->join2, 0)) != cudaSuccess) return e;
    nl += 2;
    if (launches) *launches += nl;
    if ((e = rigidClose(true, pe, nParts)) != cudaSuccess) return e;
    return cudaGetLastError();
  }
  const int nD = sh2 ? sh.blocksDS : sh.blocksD, nParts = sh.blocksA + nD;
  A *pa = static_cast<A *>(part), *pd = pa + sh.blocksA;      // value-major rows of nParts: A's blocks, then D's
  cudaError_t e = launchPDL(WSB_PICK(k_plainA, P, sh2, ext), sh.blocksA, st, d, insts, ctl, pa, nParts);
  if (e != cudaSuccess) return e;
  int nl = 1;
  if (contacts && !sh2) {
    if ((e = launchPDL(k_plainBC<P>, sh.blocksR, st, d, insts, ctl)) != cudaSuccess) return e;
    nl += 1;
  }
  const PartEnds pe{sh.blocksA, sh.blocksA, sh.blocksA, nParts};
  e = launchPDL(WSB_PICK(k_plainD, P, sh2, ext), sh2 ? sh.blocksDS : sh.blocksD, st, d, insts, ctl, pd, pa, pe, nParts,
                counter);
  if (e != cudaSuccess) return e;
  nl += 1;
  if (launches) *launches += nl;
  if ((e = rigidClose(false, pe, nParts)) != cudaSuccess) return e;
  return cudaGetLastError();
}

template <int P>
cudaError_t launchGrid(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, unsigned *bar, int *err, int nIter,
                       int blocks, bool shortSides, bool ext, cudaStream_t st) {
  using A = typename Dev<P>::A;
  A *pa = static_cast<A *>(part);
  void *args[] = {(void *)&d, (void *)&insts, (void *)&ctl, (void *)&pa, (void *)&bar, (void *)&err, (void *)&nIter};
  const void *k = (const void *)WSB_PICK(k_grid, P, shortSides, ext);
  return cudaLaunchCooperativeKernel(k, dim3(blocks), dim3(256), args, 0, st);
}
// co-resident blocks of the grid form: SMs × resident blocks per SM of the kernel variant that runs
template <int P>
int gridBlocks(bool shortSides, bool ext) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, WSB_PICK(k_grid, P, shortSides, ext), 256, 0);
  return sms * (per > 0 ? per : 1);
}

#define WSB_INST(P)                                                                                                  \
  template cudaError_t launchBatched<P>(const Dev<P> &, const InstDesc *, InstCtl *, const int *, int, int, const uint8_t *, \
                                        int, int, bool, bool, cudaStream_t);                                         \
  template cudaError_t launchPlainIter<P>(const Dev<P> &, const InstDesc *, InstCtl *, void *, const PlainShape &, bool,    \
                                          bool, bool, cudaStream_t, int *, unsigned *, const PlainFork *, bool, bool); \
  template cudaError_t launchGrid<P>(const Dev<P> &, const InstDesc *, InstCtl *, void *, unsigned *, int *, int, int, bool, \
                                     bool, cudaStream_t);                                                            \
  template int gridBlocks<P>(bool, bool);                                                                           \
  template cudaError_t launchWide<P>(const Dev<P> &, const InstDesc *, InstCtl *, const int *, int, int, const uint8_t *, \
                                     int, int, bool, bool, cudaStream_t);                                            \
  template int wideClusters<P>(int, int, bool, bool);                                                              \
  template cudaError_t launchUnpack<P>(const Dev<P> &, const InstDesc *, InstCtl *, int, const double *, int, int, int, bool, \
                                       bool, bool, cudaStream_t);                                                    \
  template cudaError_t launchPack<P>(const Dev<P> &, const InstDesc *, const InstCtl *, int, const PackList &, size_t,      \
                                     unsigned char *, cudaStream_t);                                                 \
  template cudaError_t launchClassify<P>(const Dev<P> &, const InstDesc *, int, int, cudaStream_t);                \
  template cudaError_t launchAlFlush<P>(const Dev<P> &, const InstDesc *, InstCtl *, int, cudaStream_t);           \
  template cudaError_t launchResults<P>(const Dev<P> &, const InstDesc *, int, int, int, cudaStream_t);             \
  template cudaError_t residentPrepare<P>(size_t, bool, size_t *);                                                   \
  template cudaError_t launchResident<P>(const Dev<P> &, const InstDesc *, InstCtl *, const int *, int, int, const uint8_t *, \
                                         int, size_t, bool, bool, cudaStream_t);
WSB_INST(PREC_F64)
WSB_INST(PREC_MIXED)
WSB_INST(PREC_F32)

}  // namespace wsb
