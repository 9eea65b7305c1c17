// Host-visible launchers of the DR kernels (dr_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "dr_common.cuh"

namespace wsb {

struct PlainShape { int blocksA, blocksS, blocksR, blocksD; };

template <int P>
cudaError_t launchBatched(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, const int *order, int nInst, int nIter,
                          const uint8_t *mask, int threads, int blocks, cudaStream_t st);
template <int P>
cudaError_t launchPlainIter(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, const PlainShape &sh, bool contacts,
                            cudaStream_t st, int *launches, unsigned *counter);

template <int P>
cudaError_t launchGrid(const Dev<P> &d, const InstDesc *insts, InstCtl *ctl, void *part, unsigned *bar, int *err, int nIter,
                       int blocks, cudaStream_t st);
template <int P>
int gridBlocks();

}  // namespace wsb
