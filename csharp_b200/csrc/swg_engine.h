// Whole-job engine: length-binned persistent kernels over all pairs of a job.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>

namespace swg {

struct EngineParams {
  const uint8_t* seq;      // device residues
  const int64_t* off;      // device offsets
  const int64_t* h_off;    // host offsets
  const uint8_t* h_seq;    // host residues
  int nseq, maxlen;
  const int16_t* scores;   // device [128*128]
  const uint8_t* flags;    // device [128*128]
  const int16_t* h_scores; // host [128*128]
  const uint8_t* h_flags;  // host [128*128]
  int max_score, max_abs_score;
  int o, e;
  int mode, protein, lanes;
  int ranks;
  int row_lo = 0, row_hi = -1;  // queries (s1 indices) aligned; row_hi < 0: all
  int16_t* out;
  long long ld;
  int sms;
  cudaStream_t stream;
};

struct EngineOptions {
  long long int16_threshold = -1;  // < 0: derived from the lane range; else forced trip level
  int use_graph = 1;
  int chunk = 512;                 // database entries per work item
  int k_override = 0;              // 0: per-query choice; else rows per lane
  int plan_only = 0;               // build plans and graphs, launch nothing
};

class Engine {
 public:
  static Engine* create();
  virtual ~Engine() {}
  virtual void invalidate() = 0;
  virtual EngineOptions& options() = 0;
  virtual void set_plan_only(int v) = 0;  // keeps the plans (options() drops them)
  // Returns an SW_* status.
  virtual int run(const EngineParams& p, int64_t* pairs, int64_t* cells, int64_t* reruns,
                  std::string* msg) = 0;
  // Counters of the last run: launches, bins, alphabet.
  virtual int64_t stat(const char* key) const = 0;
  // Pairs the last run gave to 32-bit lanes (static guard plus tripped lanes); waits on st.
  virtual int rerun_count(cudaStream_t st, int64_t* count, std::string* msg) = 0;
};

}  // namespace swg
