// Host-visible launchers of the DR kernels (dr_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "dr_common.cuh"

namespace wsb {

// blocks of the plain form's kernels: element phase, general side order, update phase (general order; with the side
// ranks of the short-slide order); crossings, rods, nodes (with the side ranks) and segments of the split phases;
// the crossing blocks of 256 threads in the launch with block roles
// pairsY: the rod kernel's pairs (segment e with joint or clamp e), one a thread
struct PlainShape { int blocksA, blocksR, blocksD, blocksDS, blocksX, blocksY, blocksDN, blocksDNS, blocksDM, blocksXR, pairsY; };
// a second stream and events: the element phase forks into a crossing kernel on `side` and a rod kernel on the main
// stream, joined before the update, which forks again into a node kernel on `side` and a segment kernel on the main
// stream, joined at the end of the iteration
struct PlainFork { cudaStream_t side; cudaEvent_t fork, join, fork2, join2; };
// where each kernel's block partials end in one plain-form iteration: split phases (crossings, rods, nodes, segments:
// x, y, n, m) or whole phases (element phase x, update phase m; y = n = x)
struct PartEnds { int x, y, n, m; };

template <int P>
cudaError_t launchBatched(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *order, int nInst, int nIter,
                          const uint8_t *mask, int threads, int blocks, bool shortSides, bool ext, cudaStream_t st);
// the wide instances wide[0, nWide) of the batched form, each on a thread-block cluster of `cluster` blocks of `threads`
template <int P>
cudaError_t launchWide(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *wide, int nWide, int nIter,
                       const uint8_t *mask, int threads, int cluster, bool shortSides, bool ext, cudaStream_t st);
template <int P>
int wideClusters(int threads, int cluster, bool shortSides, bool ext);
// ext: some instance runs an extension (contact extensions, the ground, a load protocol): the kernels' variants that
// have them.  rigid: the instance is a model that only the ground holds (one more launch closes its iteration).  roles: each split phase as one launch whose blocks take the two parts' roles (no fork); else `fork`
// (when given) runs the parts on forked branches, else each phase is one kernel.
template <int P>
cudaError_t launchPlainIter(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, const PlainShape &sh, bool contacts,
                            bool shortSides, bool ext, cudaStream_t st, int *launches, unsigned *counter, const PlainFork *fork,
                            bool roles, bool rigid);

template <int P>
cudaError_t launchGrid(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, unsigned *bar, int *err, int nIter,
                       int blocks, bool shortSides, bool ext, cudaStream_t st);
template <int P>
int gridBlocks(bool shortSides, bool ext);
// resident form: checks that `bytes` of dynamic shared memory fit a block on this device and opts the kernel in, with
// and without the contact extensions (*granted = bytes), else *granted = 0
template <int P>
cudaError_t residentPrepare(size_t bytes, bool shortSides, size_t *granted);
// host <-> device transfers of one instance's state (interleaved per element, as the C ABI's arrays are)
enum { PF_X, PF_Q, PF_V, PF_W, PF_U, PF_NPREV, PF_SLIP, PF_FN, PF_FT, PF_GAP, PF_N, PF_VSH, PF_M, PF_REACT, PF_STUCK, PF_STATE,
       PF_CTYPE, PF_THETA, PF_PHI, PF_AREA, PF_PRES, PF_UTIL, PF_LAM, PF_DENT, PF_MROT, PF_RSLIP, PF_UTM,
       PF_FLF, PF_FLS, PF_SEGM, PF_NODEM, PF_DISP };
struct PackField { int kind, count, ncomp; long long off; };   // off: byte offset in the packed buffer
struct PackList { PackField f[36]; int nf; };
// the results post-processing of instance b into the device output arrays: segment moments, then the node layers
template <int P>
cudaError_t launchResults(const Dev<P> &d, const InstDesc *insts, int b, int n, int m, cudaStream_t st);
// the multiplier update of instance b that fell due at the end of its last iteration, applied now
template <int P>
cudaError_t launchAlFlush(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, int b, cudaStream_t st);
// the W1 classification of instance b's crossings into the device output arrays
template <int P>
cudaError_t launchClassify(const Dev<P> &d, const InstDesc *insts, int b, int K, cudaStream_t st);
template <int P>
cudaError_t launchUnpack(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, int b, const double *in, int n, int m, int K,
                         bool withU, bool rebuildOrder, bool shortSides, cudaStream_t st);
template <int P>
cudaError_t launchPack(const Dev<P> &d, const InstDesc *insts, const InstCtl *ctl, int b, const PackList &L, size_t elems,
                       unsigned char *out, cudaStream_t st);
template <int P>
cudaError_t launchResident(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *order, int nInst, int nIter,
                           const uint8_t *mask, int threads, size_t smemBytes, bool shortSides, bool ext, cudaStream_t st);

}  // namespace wsb
