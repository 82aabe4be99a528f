// Autotuner for launch parameters that do not change results.
//
// A tuned parameter (the local operator's bands per chunk, the tensor-core
// GEMM's tile width) is chosen per shape signature by measurement on the
// caller's own work: successive calls with the same signature try the
// candidates in turn, each timed with a pair of CUDA events on the call's
// stream, and once every candidate has a completed timing the fastest per
// unit of work is used from then on.  Events are read without waiting (a
// timing whose events have not completed yet is picked up by a later call),
// so tuning adds no synchronisation.  Every candidate produces bit-identical
// results: chunking only regroups independent bands, and the GEMM tile width
// changes neither the k order of any output element nor the split-K
// boundaries, so tuning never changes a solve's iterates.
//
// Environment HALF_TUNE=0 disables tuning (the first candidate is always
// used); HALF_TUNE_LOG=1 prints each decision to stderr.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace hb {

class Tuner {
 public:
  // Index into `candidates` to use for the next call with this signature.
  static int pick(const std::string& key, const std::vector<int>& candidates);
  // Starts timing a call made with candidate `index`; returns a token for finish.
  static int begin(const std::string& key, int index, cudaStream_t s);
  // Ends the timing started with `token`; `units` = work of the call (bands, 1 per GEMM).
  static void finish(int token, cudaStream_t s, double units);
  // Decision recorded for a signature (-1 while still measuring).
  static int decided(const std::string& key);
};

}  // namespace hb
