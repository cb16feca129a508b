// Serving scheduler: query batches against the context's sequences, continuous batching.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/swgb200.h"
#include "swg_engine.h"

namespace swg {

struct ServeOptions {
  size_t memory_bytes = 0;          // device bytes for admitted jobs' results (0: half the free memory)
  size_t arena_bytes = 64u << 20;   // device bytes for admitted jobs' query residues
  int slots = 8192;                 // queries admitted at once
  double wave_seconds = 0.1;        // estimated GPU time of one wave
};

class Server {
 public:
  static Server* create(const EngineParams& db, int device, const ServeOptions& opt,
                        std::string* msg, int* rc);
  virtual ~Server() {}  // ends the threads; unfinished jobs end with SW_E_STATE
  virtual int submit(const uint8_t* q, const int64_t* off, int nq, int16_t* out, int64_t ld,
                     int64_t* ticket, std::string* msg) = 0;
  virtual int poll(int64_t ticket, int timeout_ms, int* done, sw_job_info* info) = 0;
  virtual void stats(sw_serve_counters* s) = 0;
  virtual void drain() = 0;  // waits until every submitted job is done
};

}  // namespace swg
