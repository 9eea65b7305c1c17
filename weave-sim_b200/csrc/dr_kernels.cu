// sm_100a kernels of the DR step: the persistent batched form (one thread block per instance, every phase of every
// iteration inside one launch) and the plain form (one kernel per phase, one instance, captured as a CUDA graph).
#include "dr_kernels.hpp"
#include "dr_phases.cuh"

#ifndef WSB_MINB
#define WSB_MINB 1          // minimum resident blocks per SM asked of the large-instance kernels (register budget)
#endif

namespace wsb {

// element e of phase A: the crossings come first (the heaviest elements start earliest), then segments, joints, clamps
template <int P>
__device__ __forceinline__ void phaseA(const Dev<P> &d, const InstDesc &I, int cur, int iter, int e, int nK, Part<typename Dev<P>::A> &pt) {
  if (e < nK) crossing<P>(d, I, cur, iter, I.k0 + e, pt);
  else if ((e -= nK) < I.m) segForce<P>(d, cur, I.m0 + e, pt);
  else if ((e -= I.m) < I.p) jointTorque<P>(d, cur, I.p0 + e, pt);
  else clampTorque<P>(d, cur, I.c0 + (e - I.p), pt);
}

// ------------------------------------------------------------------------------------------------ batched form
// Block b relaxes instance order[b] (and further instances grid-strided) for up to nIter iterations, stopping at its
// own convergence.  Instance state lives in HBM / L2; the block's barriers separate the phases, so an instance never
// waits on another and no kernel spins.
template <int P>
__global__ void __launch_bounds__(512) k_batched(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                  const int *__restrict__ order, int nInst, int nIter, const uint8_t *__restrict__ mask) {
  using A = typename Dev<P>::A;
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  for (int bi = blockIdx.x; bi < nInst; bi += gridDim.x) {
    const int b = order ? order[bi] : bi;
    if (mask && !mask[b]) continue;
    if (threadIdx.x == 0) { sc = ctl[b]; si = insts[b]; }
    __syncthreads();
    const InstDesc &I = si;
    const bool cx = I.contacts && I.K;
    const int nA = I.m + I.p + I.C + (cx ? I.K : 0);
    for (int it = 0; it < nIter; it++) {
      if (sc.status != WS_RUNNING) break;
      const StepCtx sx = makeCtx<A>(I, sc);
      Part<A> pt;
      pt.init();
      for (int e = threadIdx.x; e < nA; e += blockDim.x) phaseA<P>(d, I, sx.cur, sx.iter, e, cx ? I.K : 0, pt);
      __syncthreads();
      if (cx) {
        const int n2 = 2 * I.K;
        for (int e = threadIdx.x; e < n2 + I.m; e += blockDim.x) {
          if (e < n2) rankSide<P>(d, 2 * I.k0 + e, sx.obuf, sx.onxt);
          else segCount<P>(d, I.m0 + (e - n2), sx.obuf, sx.onxt);
        }
        __syncthreads();
      }
      for (int e = threadIdx.x; e < I.n + I.m; e += blockDim.x) {
        if (e < I.n) nodeUpdate<P>(d, I, sx, I.n0 + e, pt);
        else segUpdate<P>(d, I, sx, I.m0 + (e - I.n), pt);
      }
      __syncthreads();
      blockReduce(pt, red);
      if (threadIdx.x == 0) decide(I, sc, pt, nIter);
      __syncthreads();
    }
    if (threadIdx.x == 0) ctl[b] = sc;
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------ plain form
// One kernel per phase over the elements of instance 0; block partials go to part[phase][block] and k_decide reduces
// them in a fixed order.  Every kernel returns at once when the instance has stopped.
template <int P>
__global__ void __launch_bounds__(256, WSB_MINB) k_plainA(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl,
                                                typename Dev<P>::A *part) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  const InstDesc I = insts[0];
  const InstCtl c = ctl[0];
  if (c.status != WS_RUNNING) return;
  const bool cx = I.contacts && I.K;
  const int nA = I.m + I.p + I.C + (cx ? I.K : 0);
  Part<A> pt;
  pt.init();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nA; e += gridDim.x * blockDim.x) phaseA<P>(d, I, c.cur, c.iter, e, cx ? I.K : 0, pt);
  blockReduce(pt, red);
  constexpr int NV = RS_NSUM + RX_NMAX;
  if (threadIdx.x == 0) {
    for (int i = 0; i < RS_NSUM; i++) part[blockIdx.x * NV + i] = pt.s[i];
    for (int i = 0; i < RX_NMAX; i++) part[blockIdx.x * NV + RS_NSUM + i] = pt.x[i];
  }
}
template <int P>
__global__ void __launch_bounds__(256) k_plainBC(Dev<P> d, const InstDesc *__restrict__ insts, const InstCtl *__restrict__ ctl) {
  const InstDesc I = insts[0];
  const InstCtl c = ctl[0];
  if (c.status != WS_RUNNING) return;
  const int n2 = 2 * I.K;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n2 + I.m; e += gridDim.x * blockDim.x) {
    if (e < n2) rankSide<P>(d, 2 * I.k0 + e, c.obuf, c.obuf ^ 1);
    else segCount<P>(d, I.m0 + (e - n2), c.obuf, c.obuf ^ 1);
  }
}
// The update kernel also closes the iteration: every block publishes its partials, and the last block to finish
// (counted on `counter`) reduces the partials of phases A and D in a fixed order and takes the kinetic-damping decision.
template <int P>
__global__ void __launch_bounds__(256, WSB_MINB) k_plainD(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                                typename Dev<P>::A *part, typename Dev<P>::A *partAll, int nParts,
                                                unsigned *counter) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  __shared__ bool last;
  const InstDesc I = insts[0];
  const InstCtl c = ctl[0];
  if (c.status != WS_RUNNING) return;
  const StepCtx sx = makeCtx<A>(I, c);
  Part<A> pt;
  pt.init();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < I.n + I.m; e += gridDim.x * blockDim.x) {
    if (e < I.n) nodeUpdate<P>(d, I, sx, I.n0 + e, pt);
    else segUpdate<P>(d, I, sx, I.m0 + (e - I.n), pt);
  }
  blockReduce(pt, red);
  constexpr int NV = RS_NSUM + RX_NMAX;
  if (threadIdx.x == 0) {
    for (int i = 0; i < RS_NSUM; i++) part[blockIdx.x * NV + i] = pt.s[i];
    for (int i = 0; i < RX_NMAX; i++) part[blockIdx.x * NV + RS_NSUM + i] = pt.x[i];
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  Part<A> q;
  q.init();
  for (int b = threadIdx.x; b < nParts; b += blockDim.x) {
    for (int i = 0; i < RS_NSUM; i++) q.s[i] += __ldcg(partAll + b * NV + i);
    for (int i = 0; i < RX_NMAX; i++) q.x[i] = mmax(q.x[i], __ldcg(partAll + b * NV + RS_NSUM + i));
  }
  blockReduce(q, red);
  if (threadIdx.x == 0) {
    InstCtl cc = c;
    decide(I, cc, q, 0);
    ctl[0] = cc;
    *counter = 0;
  }
}
template <int P>
__global__ void __launch_bounds__(256) k_plainDecide(const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl, const typename Dev<P>::A *part, int nParts) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  if (ctl[0].status != WS_RUNNING) return;
  constexpr int NV = RS_NSUM + RX_NMAX;
  Part<A> pt;
  pt.init();
  for (int b = threadIdx.x; b < nParts; b += blockDim.x) {
    for (int i = 0; i < RS_NSUM; i++) pt.s[i] += part[b * NV + i];
    for (int i = 0; i < RX_NMAX; i++) pt.x[i] = mmax(pt.x[i], part[b * NV + RS_NSUM + i]);
  }
  blockReduce(pt, red);
  if (threadIdx.x == 0) {
    InstCtl c = ctl[0];
    decide(insts[0], c, pt, 0);
    ctl[0] = c;
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

// One instance over the whole (co-resident) grid, every phase of up to nIter iterations in one launch: three grid
// barriers per iteration.  Block partials go to part[block]; after the barrier every block reduces all of them in the
// same order and takes the same kinetic-damping decision, so no further broadcast is needed.
template <int P>
__global__ void __launch_bounds__(256, WSB_MINB) k_grid(Dev<P> d, const InstDesc *__restrict__ insts, InstCtl *__restrict__ ctl,
                                              typename Dev<P>::A *part, unsigned *bar, int *err, int nIter) {
  using A = typename Dev<P>::A;
  __shared__ A red[32 * (RS_NSUM + RX_NMAX)];
  __shared__ InstCtl sc;
  __shared__ InstDesc si;
  constexpr int NV = RS_NSUM + RX_NMAX;
  if (threadIdx.x == 0) { sc = ctl[0]; si = insts[0]; }
  __syncthreads();
  const InstDesc &I = si;
  const bool cx = I.contacts && I.K;
  const int nA = I.m + I.p + I.C + (cx ? I.K : 0);
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const unsigned nb = gridDim.x;
  for (int it = 0; it < nIter; it++) {
    if (sc.status != WS_RUNNING) break;
    const StepCtx sx = makeCtx<A>(I, sc);
    Part<A> pt;
    pt.init();
    for (int e = gt; e < nA; e += gs) phaseA<P>(d, I, sx.cur, sx.iter, e, cx ? I.K : 0, pt);
    if (!gridSync(bar, nb, err)) break;
    if (cx) {
      const int n2 = 2 * I.K;
      for (int e = gt; e < n2 + I.m; e += gs) {
        if (e < n2) rankSide<P>(d, 2 * I.k0 + e, sx.obuf, sx.onxt);
        else segCount<P>(d, I.m0 + (e - n2), sx.obuf, sx.onxt);
      }
      if (!gridSync(bar, nb, err)) break;
    }
    for (int e = gt; e < I.n + I.m; e += gs) {
      if (e < I.n) nodeUpdate<P>(d, I, sx, I.n0 + e, pt);
      else segUpdate<P>(d, I, sx, I.m0 + (e - I.n), pt);
    }
    blockReduce(pt, red);
    if (threadIdx.x == 0) {
      for (int i = 0; i < RS_NSUM; i++) part[blockIdx.x * NV + i] = pt.s[i];
      for (int i = 0; i < RX_NMAX; i++) part[blockIdx.x * NV + RS_NSUM + i] = pt.x[i];
    }
    if (!gridSync(bar, nb, err)) break;
    Part<A> q;
    q.init();
    for (int b = threadIdx.x; b < int(nb); b += blockDim.x) {
      for (int i = 0; i < RS_NSUM; i++) q.s[i] += part[b * NV + i];
      for (int i = 0; i < RX_NMAX; i++) q.x[i] = mmax(q.x[i], part[b * NV + RS_NSUM + i]);
    }
    blockReduce(q, red);
    if (threadIdx.x == 0) decide(I, sc, q, nIter);
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl[0] = sc;
}

// ------------------------------------------------------------------------------------------------ launchers
template <int P>
cudaError_t launchBatched(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *order, int nInst, int nIter,
                          const uint8_t *mask, int threads, int blocks, cudaStream_t st) {
  k_batched<P><<<blocks, threads, 0, st>>>(d, insts, ctl, order, nInst, nIter, mask);
  return cudaGetLastError();
}

template <int P>
cudaError_t launchPlainIter(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, const PlainShape &sh, bool contacts,
                            cudaStream_t st, int *launches, unsigned *counter) {
  using A = typename Dev<P>::A;
  A *pa = static_cast<A *>(part), *pd = pa + size_t(sh.blocksA) * (RS_NSUM + RX_NMAX);
  k_plainA<P><<<sh.blocksA, 256, 0, st>>>(d, insts, ctl, pa);
  int nl = 1;
  if (contacts) {
    k_plainBC<P><<<sh.blocksR, 256, 0, st>>>(d, insts, ctl);
    nl += 1;
  }
  k_plainD<P><<<sh.blocksD, 256, 0, st>>>(d, insts, ctl, pd, pa, sh.blocksA + sh.blocksD, counter);
  nl += 1;
  if (launches) *launches += nl;
  return cudaGetLastError();
}

template <int P>
cudaError_t launchGrid(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, unsigned *bar, int *err, int nIter,
                       int blocks, cudaStream_t st) {
  using A = typename Dev<P>::A;
  A *pa = static_cast<A *>(part);
  void *args[] = {(void *)&d, (void *)&insts, (void *)&ctl, (void *)&pa, (void *)&bar, (void *)&err, (void *)&nIter};
  return cudaLaunchCooperativeKernel((const void *)k_grid<P>, dim3(blocks), dim3(256), args, 0, st);
}
template <int P>
int gridBlocks() {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_grid<P>, 256, 0);
  return sms * (per > 0 ? per : 1);
}

#define WSB_INST(P)                                                                                                  \
  template cudaError_t launchBatched<P>(const Dev<P> &, const InstDesc *, InstCtl *, const int *, int, int, const uint8_t *, \
                                        int, int, cudaStream_t);                                                     \
  template cudaError_t launchPlainIter<P>(const Dev<P> &, const InstDesc *, InstCtl *, void *, const PlainShape &, bool,    \
                                          cudaStream_t, int *, unsigned *);                                                        \
  template cudaError_t launchGrid<P>(const Dev<P> &, const InstDesc *, InstCtl *, void *, unsigned *, int *, int, int, cudaStream_t); \
  template int gridBlocks<P>();
WSB_INST(PREC_F64)
WSB_INST(PREC_MIXED)
WSB_INST(PREC_F32)

}  // namespace wsb
