// Whole-job engine: length-binned persistent kernels over all pairs of a job.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

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
  int dist_fn = 0;         // SW_DIST_*: Kimura2 / JukesCantor run on 32-bit lanes
  int two_pass = 1;        // serving: the engine's two_pass option (0 never, 1 where it suits, 2 always)
  int third_pass = 1;      // serving: the engine's third_pass option
  int* throws = nullptr;   // device flag: SWG-MPI JukesCantor met log(0)
  int ranks;
  int row_lo = 0, row_hi = -1;  // queries (s1 indices) aligned; row_hi < 0: all
  int block = 0;                // 1 / 2: only the diagonal / off-diagonal block of rows row_lo..row_hi
  int col_lo = 0, col_hi = -1;  // and columns col_lo..col_hi (out points at element (0, 0))
  int16_t* out;
  long long ld;
  int sms;
  cudaStream_t stream;
};

struct EngineOptions {
  long long int16_threshold = -1;  // < 0: derived from the lane range; else forced trip level
  int use_graph = 1;
  int chunk = 0;                   // database entries per work item (0: 1024 for 8,192 sequences or more, else 512)
  int k_override = 0;              // 0: per-query choice; else rows per lane
  int plan_only = 0;               // build plans and graphs, launch nothing
  int two_pass = 1;                // SW: score-only pass, then counters from boxes (box step):
                                   // 1 where the gap costs suit it, 2 whenever min(o, e) >= 2, 0 never
  int box_reg = 1;                 // two-pass: register box step first (0: the warp box kernel alone)
  int third_pass = 1;              // two-pass: the box step's give-ups on 16-bit lanes (0: 32-bit lanes)
  int m_lo = 0, m_hi = 0;          // autotuner: only queries with m_lo < length <= m_hi (0: all)
  int k_weights[7] = {0, 0, 0, 0, 0, 0, 0};  // cost per row at 4, 6, ..., 16 rows per lane
                                             // (0: built-in table; set by autotune)
};

class Engine {
 public:
  static Engine* create();
  virtual ~Engine() {}
  virtual void invalidate() = 0;
  // The set's residues changed but not its lengths or letters: the plans and graphs stay valid;
  // the dense residue codes are rebuilt on the device from d_seq (ordered on st).
  virtual int refresh_codes(const uint8_t* d_seq, int64_t total, cudaStream_t st, std::string* msg) = 0;
  virtual EngineOptions& options() = 0;                 // for changing them: drops the plans
  virtual const EngineOptions& current_options() const = 0;  // reading them keeps the plans
  virtual void set_plan_only(int v) = 0;  // keeps the plans (options() drops them)
  // Returns an SW_* status.
  virtual int run(const EngineParams& p, int64_t* pairs, int64_t* cells, int64_t* reruns,
                  std::string* msg) = 0;
  // Counters of the last run: launches, bins, alphabet.
  virtual int64_t stat(const char* key) const = 0;
  // Pairs the last run gave to 32-bit lanes (static guard plus tripped lanes); waits on st.
  virtual int rerun_count(cudaStream_t st, int64_t* count, std::string* msg) = 0;
  // Times every rows-per-lane choice forced on a sample of the job's queries (writing their
  // distances to p.out) and installs the measured per-row costs for later plans; weights gets
  // them (100 = the cheapest, 0 = not measured).  Waits on p.stream.
  virtual int autotune(const EngineParams& p, int weights[7], std::string* msg) = 0;
};

// ---- query mode (serving) ---------------------------------------------------------------------
// A query batch is aligned (query = s1) against every sequence of the set, which serves as the
// database.  Work is cut into items (query slot, chunk of the database in length order) that
// waves of the same persistent kernels execute; the caller (the server) decides which items go
// into which wave.

struct QueryItem {
  int slot;       // query slot (row of the device query tables)
  int c0, c1;     // database chunk: positions [c0, c1) of the length order
  int K, passes;  // rows per lane and passes (16-bit lanes); K = 0: 32-bit lanes
  double cost;    // estimated GPU seconds
};

struct QueryTables {   // device, indexed by slot
  const uint8_t* qseq;
  const int64_t* qoff;
  const int32_t* qlen;
  int16_t* const* qout;  // each a row of database-count distances
};

class QueryRunner {
 public:
  // db describes the database (the context's uploaded sequences, scores and penalties).
  static QueryRunner* create(const EngineParams& db, std::string* msg, int* rc);
  virtual ~QueryRunner() {}
  virtual int db_count() const = 0;
  // Appends the items of one query of m residues held in `slot`.
  virtual void plan_query(int slot, int m, std::vector<QueryItem>* items) const = 0;
  // Useful cells of one query of m residues against the whole database.
  virtual int64_t query_cells(int m) const = 0;
  // Enqueues one wave on st (wave buffer `buf`, 0 or 1, reused once its earlier wave is done).
  // Waves of the two buffers may be enqueued on different streams and overlap on the GPU.
  virtual int enqueue(int buf, const std::vector<QueryItem>& items, const QueryTables& T,
                      cudaStream_t st, std::string* msg) = 0;
};

}  // namespace swg
