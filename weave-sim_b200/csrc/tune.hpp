// The autotuner's host side: the candidate launch shapes of a batch, the key of its size bucket, and the cache of the
// shapes it picked (tune.cpp).  The timing of the candidates on the device is in capi_solver.cu.
#pragma once
#include <string>
#include <vector>

#include "../../include/weavesim.h"

namespace wsb {

// what the choice of shape depends on
struct TuneInfo {
  int form = 0, prec = 0, nInst = 0, shortSides = 1, ext = 0;
  long long maxElems = 0, totalElems = 0;    // nodes + segments: the largest instance, the whole batch
};

// the size bucket of a batch on a device: the form, precision and variants, and the instance count, largest instance
// and total work in half-octave steps
std::string tuneKey(const std::string &device, const TuneInfo &t);
// stage 1 of the batched form's search: block size and state placement, no wide instances; stage 2: cluster shapes
// and thresholds for the wide instances at the best stage-1 shape; the plain form: its three launch modes
std::vector<ws_shape> tuneStage1(const TuneInfo &t);
std::vector<ws_shape> tuneStage2(const TuneInfo &t, const ws_shape &best1);
// the cache: process-wide, loaded from and appended to the file WEAVESIM_TUNE_CACHE names, when it is set
bool tuneLookup(const std::string &key, ws_shape *out);
void tuneStore(const std::string &key, const ws_shape &s);
void tuneClear();

}  // namespace wsb
