// Host build of the two-pass box step (csharp_b200/csrc/swg_box_lane.cuh) for the CPU tests: the
// same source the box_lane_kernel runs, driven for a list of pairs as `threads` emulated lanes
// (lane t takes pairs t, t + threads, ...), with a bounds check on every scratch word.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static void swg_lane_check_failed(int k) {
  fprintf(stderr, "box step scratch index %d out of range\n", k);
  abort();
}
#define SWG_LANE_CHECK 1
#include "../csharp_b200/csrc/swg_box_lane.cuh"

// Pair p: s1 = sequence q[p], s2 = sequence d[p], best score S[p] at (ie[p], je[p]).  Writes the
// outcome (0 = solved, else the reason it was given up) and the counters
// (aligned << 8 | counted) of every pair.  Returns 0, or 1 if a pair's outcome came twice.
extern "C" int box_step_run(const uint8_t* seqs, const int64_t* off, const int32_t* q, const int32_t* d,
                            const int32_t* S, const int32_t* ie, const int32_t* je, long np,
                            const int32_t* scores, const uint32_t* flags, int A1, int o, int e,
                            int max_score, int threads, int32_t* outcome, uint32_t* counters) {
  std::vector<int16_t> sc((size_t)A1 * A1);
  std::vector<uint8_t> fl((size_t)A1 * A1);
  for (int k = 0; k < A1 * A1; k++) {
    sc[k] = (int16_t)scores[k];
    fl[k] = (uint8_t)flags[k];
  }
  std::vector<int4> list((size_t)(np > 0 ? np : 1));
  for (long p = 0; p < np; p++) {
    list[p].x = q[p];
    list[p].y = d[p];
    list[p].z = S[p];
    list[p].w = (int)(((uint32_t)ie[p] << 16) | (uint32_t)je[p]);
    outcome[p] = -1;
  }
  uint32_t scratch[swg::kLaneWords];
  int bad = 0;
  for (int t = 0; t < threads; t++) {
    for (int k = 0; k < swg::kLaneWords; k++) scratch[k] = 0xA5A5A5A5u * (uint32_t)(k + t + 1);
    const swg::LaneMem mem{scratch, 1};
    long cur = t;
    auto emit = [&](const int4&, int rc, uint32_t c) {
      if (cur >= np || outcome[cur] != -1) {
        bad = 1;
        return;
      }
      outcome[cur] = rc;
      counters[cur] = c;
      cur += threads;
    };
    swg::lane_box_run(list.data(), (long long)t, (long long)np, (long long)threads, seqs, off, sc.data(),
                      fl.data(), A1, o, e, max_score, mem, emit);
  }
  return bad;
}
