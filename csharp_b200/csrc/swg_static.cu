// Block handler that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application that hands the GPU's memory to its
// own pool allocator at start-up and forbids other allocations, or a plug-in loaded into a
// process whose device memory budget is fixed and already spent by its host.
// sw_compute_block_static serves them: it is the plain block kernel of sw_compute_block_device,
// with the kernel's scratch (the substitution and flag tables, and each thread's carry row
// between strips of the DP) taken from the file-scope array below instead of from cudaMalloc.  The caller passes the residues, the
// offsets and the output in device memory it owns.
//
// The array is 64 MiB and lives in every GPU that loads this library until the process exits.
// Calls share it and leave the last call's contents in it; only the input check's two status
// words have to start at zero, and every call clears them (the tables are rewritten by every call
// and each carry row is written before it is read).  Calls whose kernels overlap on the GPU
// (different streams, or different host threads) race on it: the caller must order them.  The
// first call on a device looks up the array's device address (cudaGetSymbolAddress, with that
// device current) and keeps it; make that first call before any stream capture.  A call runs
// on cfg->device (made current for the call, the caller's current device restored before it
// returns) and refuses buffers that are not that device's memory.
#include <cuda_runtime.h>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/swgb200.h"
#include "swg_device.cuh"
#include "swg_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr size_t kTableRegion = size_t(64) << 10;  // scores (32 KiB) + flags (16 KiB), padded
constexpr int kBlockThreads = 128;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_block_scratch[kScratchBytes];

// The array's device address per device ordinal (looked up once, with that device current).
void* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return SW_E_ARG;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_block_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return SW_E_CUDA;
    }
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return SW_OK;
}

// Status words of the input check, in the table region past the scores and flags.
constexpr size_t kStatusOffset = size_t(48) << 10;
enum { kBadLength = 1, kTooLong = 2, kBadResidue = 4 };

// One warp per sequence of the block's row and column ranges: its length (non-negative, at most
// 16,383 residues) and residues (inside the 127-entry scoring table); status[0] collects the
// problems found, status[1] the longest length.
__global__ void static_check_kernel(const uint8_t* seq, const int64_t* off, int rs, int re, int cs, int ce,
                                    int* status) {
  const int lane = threadIdx.x & 31;
  const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
  const long nr = (long)re - rs + 1, total = nr + ((long)ce - cs + 1);
  for (long w = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < total; w += nwarps) {
    const long k = w < nr ? rs + w : cs + (w - nr);
    const int64_t lo = off[k], len = off[k + 1] - lo;
    if (len < 0 || len > 16383) {
      if (lane == 0) atomicOr(status, len < 0 ? kBadLength : kTooLong);
      continue;
    }
    bool bad = false;
    for (int64_t x = lane; x < len; x += 32) bad |= seq[lo + x] >= 127;
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status, kBadResidue);
    if (lane == 0) atomicMax(status + 1, (int)len);
  }
}

// The caller's buffers must be memory this device can address as its own.
bool on_device(const void* p, int device) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == device;
}

// Makes `device` current for the call and puts the caller's device back when the call returns.
struct DeviceScope {
  int prev = -1;
  bool ok = false;
  explicit DeviceScope(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) return;
    ok = prev == device || cudaSetDevice(device) == cudaSuccess;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int sw_compute_block_static(const sw_config* cfg, const uint8_t* d_residues,
                                       const int64_t* d_offsets, int32_t count, int32_t rs,
                                       int32_t re, int32_t cs, int32_t ce, int32_t is_diagonal,
                                       int16_t* d_out, int64_t ld_out, int64_t* pairs_computed,
                                       void* stream) {
  if (!cfg || !d_residues || !d_offsets || !d_out || count < 1) return SW_E_ARG;
  if (cfg->mode < 0 || cfg->mode > 2) return SW_E_ARG;
  if (cfg->alignment_type != SW_PROTEIN && cfg->alignment_type != SW_NUCLEIC) return SW_E_ARG;
  if (cfg->distance_fn < 0 || cfg->distance_fn > 3) return SW_E_ARG;
  // Kimura2 / JukesCantor / MinMaxNormScore (nucleic) are the allocating entry points' work
  if (cfg->distance_fn != SW_DIST_PERCENT_IDENTITY && cfg->alignment_type == SW_NUCLEIC) return SW_E_UNSUPPORTED;
  const float o = cfg->gap_open, e = cfg->gap_extension;
  if (!(o == o && e == e) || o != (float)(int)o || e != (float)(int)e) return SW_E_UNSUPPORTED;
  if (o < 1 || e < 0 || o > 10000 || e > 10000) return SW_E_UNSUPPORTED;
  if (cfg->mode == SW_MODE_NW && !(o > e)) return SW_E_UNSUPPORTED;
  if (rs < 0 || cs < 0 || re >= count || ce >= count || rs > re || cs > ce) return SW_E_ARG;
  const bool tri = is_diagonal && cfg->mode != SW_MODE_SWG_MS;
  if (tri && (rs != cs || re != ce)) return SW_E_ARG;
  if (ld_out < (int64_t)(ce - cs + 1)) return SW_E_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int device = cfg->device;
  const DeviceScope scope(device);
  if (!scope.ok) {
    cudaGetLastError();
    return SW_E_ARG;
  }
  if (!on_device(d_residues, device) || !on_device(d_offsets, device) || !on_device(d_out, device)) return SW_E_ARG;
  void* base = nullptr;
  int rc = scratch_address(device, &base);
  if (rc) return rc;

  // tables as sw_create builds them: scores (pad code 127 scores -16384) and column flags
  int16_t scores[128 * 128];
  uint8_t flags[128 * 128];
  int maxabs = 0;
  for (int a = 0; a < 128; a++)
    for (int b = 0; b < 128; b++) {
      const int s = cfg->scores[a][b];
      if (s < -16383 || s > 16383) return SW_E_UNSUPPORTED;
      const bool pad = a == swg::kPadCode || b == swg::kPadCode;
      scores[a * 128 + b] = pad ? (int16_t)swg::kPadScore : (int16_t)s;
      if (!pad && (s < 0 ? -s : s) > maxabs) maxabs = s < 0 ? -s : s;
      uint32_t f = 0;
      if (a == b) f |= swg::kFlagIdent;
      if (a == b || s > 0) f |= swg::kFlagSimNA;
      bool counted;
      if (cfg->alignment_type == SW_NUCLEIC) counted = a == b;
      else if (cfg->mode == SW_MODE_SWG_MPI) counted = a == b || s > 0;
      else counted = s > 0;
      if (counted) f |= swg::kFlagCount;
      flags[a * 128 + b] = pad ? 0 : (uint8_t)f;
    }

  // inputs: lengths and residues of the block's sequences, checked by one kernel whose status
  // words come back in one small copy
  unsigned char* p = static_cast<unsigned char*>(base);
  int* d_status = reinterpret_cast<int*>(p + kStatusOffset);
  int status[2] = {0, 0};
  if (cudaMemsetAsync(d_status, 0, sizeof(status), st) != cudaSuccess) {
    cudaGetLastError();
    return SW_E_CUDA;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  static_check_kernel<<<std::max(sms, 1) * 4, 256, 0, st>>>(d_residues, d_offsets, rs, re, cs, ce, d_status);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(status, d_status, sizeof(status), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return SW_E_CUDA;
  }
  if (status[0] & kBadLength) return SW_E_ARG;
  if (status[0] & kTooLong) return SW_E_UNSUPPORTED;
  if (status[0] & kBadResidue) return SW_E_ARG;
  const int maxlen = status[1];
  if ((double)(maxabs + (int)e) * 2.0 * maxlen + o >= 16777216.0) return SW_E_UNSUPPORTED;

  const long long R = re - rs + 1, C = ce - cs + 1;
  const long long npairs = tri ? R * (R - 1) / 2 : R * C;
  if (pairs_computed) *pairs_computed = npairs;
  if (npairs == 0) return SW_OK;
  // threads whose carry rows fit in the array beyond the tables
  const size_t per_thread = swg::plain_carry_bytes(cfg->mode == SW_MODE_NW ? swg::kModeNw : swg::kModeSwgMpi, 1, maxlen);
  long threads = (long)((kScratchBytes - kTableRegion) / per_thread) / kBlockThreads * kBlockThreads;
  if (threads < kBlockThreads) return SW_E_UNSUPPORTED;
  threads = std::min<long>(threads, (long)std::max(sms, 1) * 8 * kBlockThreads);
  threads = std::min<long>(threads, (long)((npairs + kBlockThreads - 1) / kBlockThreads) * kBlockThreads);

  if (cudaMemcpyAsync(p, scores, sizeof(scores), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(p + sizeof(scores), flags, sizeof(flags), cudaMemcpyHostToDevice, st) != cudaSuccess) {
    cudaGetLastError();
    return SW_E_CUDA;
  }
  swg::PlainJob J;
  std::memset(&J, 0, sizeof(J));
  J.seq = d_residues;
  J.off = d_offsets;
  J.rs = rs; J.re = re; J.cs = cs; J.ce = ce;
  J.tri = tri ? 1 : 0;
  J.npairs = npairs;
  J.out = d_out;
  J.ld = ld_out;
  J.out_r0 = rs;
  J.out_c0 = cs;
  J.mirror = tri ? 1 : 0;
  J.scores = reinterpret_cast<const int16_t*>(p);
  J.flags = p + sizeof(scores);
  J.o = (int)o;
  J.e = (int)e;
  J.mode = cfg->mode;
  J.protein = cfg->alignment_type == SW_PROTEIN;
  J.carry = p + kTableRegion;
  if (swg::launch_plain_block(J, (int)(threads / kBlockThreads), kBlockThreads, st) != cudaSuccess) {
    cudaGetLastError();
    return SW_E_CUDA;
  }
  return SW_OK;
}
