// vp8a_internal.cuh — shared internals of libvp8a (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/vp8a.h"

#define VP8A_ABI_VERSION ((1u << 16) | 1u)  /* 1.1: the bitstream writer */

// ----------------------------------------------------------------- context
struct vp8a_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  uint64_t launches = 0;
  // Device-resident status word shared by kernels with bounded waits.
  uint32_t* d_status = nullptr;
  // Poll budget of the analysis wavefront waits (vp8a_ctx_set_wait_limit).
  uint64_t wait_limit = 1ull << 24;
  // Device copy of the 256-entry -log2(p/256) bit-cost table (f64).
  double* d_bit_cost = nullptr;
  // Pinned host ring for the small tables a call builds on the host
  // (schedules, job tables, candidate lists): a table is copied into slot k
  // and uploaded asynchronously, so the call never waits for the GPU to
  // take it; slot k is reused only once the event recorded behind its last
  // upload has completed.
  static constexpr int UP_SLOTS = 16;
  static constexpr size_t UP_SLOT_BYTES = 256 << 10;
  uint8_t* up_host = nullptr;
  cudaEvent_t up_ev[UP_SLOTS] = {};
  unsigned up_next = 0;
  // Launch-shape choice of the loop-filter sweep: measured on first use
  // per picture shape (autotune) or by the cost model; a forced layout
  // (tests) overrides both. Cache: shape key -> (passes per CTA, threads,
  // prefetch). last_layout: the last sweep's (passes, threads, prefetch,
  // CTAs per SM).
  bool autotune = true;
  // The analysis reads its half- and quarter-pel predictions from planes
  // precomputed per call (vp8a_ctx_set_subpel_planes; off by default: the
  // SPLITMV warps, not the refinements, bound each MB's latency).
  bool subpel_planes = false;
  // TrellisStrength of the reconstructions (vp8a_ctx_set_trellis_strength;
  // 0 = plain rounding).
  double trellis_strength = 0.0;
  int force_layout[3] = {0, 0, 0};
  std::map<std::array<int64_t, 6>, std::array<int, 3>> lf_tuned;
  std::map<std::vector<int64_t>, std::array<int, 3>> lf_tuned_batch;  // batched sweeps: job shapes -> layout
  int last_layout[4] = {0, 0, 0, 0};
};

namespace vp8a {

void set_error(const std::string& msg);
vp8a_status cuda_fail(cudaError_t e, const char* what);
inline vp8a_status cuda_ok(cudaError_t e, const char* what) { return e == cudaSuccess ? VP8A_OK : cuda_fail(e, what); }

#define VP8A_CUDA(call)                                        \
  do {                                                         \
    cudaError_t _e = (call);                                   \
    if (_e != cudaSuccess) return ::vp8a::cuda_fail(_e, #call); \
  } while (0)

// Device status codes written by kernels (host maps them to vp8a_status).
enum : uint32_t { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_BAD_INPUT = 2 };

// Host/device staging of ABI buffers. Each buffer passed through the ABI may
// be host or device memory; host buffers get a stream-ordered device copy.
class Stager {
 public:
  explicit Stager(vp8a_ctx* ctx) : ctx_(ctx) {}
  ~Stager();
  // Device view of a read-only input of `bytes` bytes.
  vp8a_status in(const void* p, size_t bytes, const void** dev);
  // Device view of an output; host outputs are copied back in finish().
  vp8a_status out(void* p, size_t bytes, void** dev);
  // Device view of an in/out buffer.
  vp8a_status inout(void* p, size_t bytes, void** dev);
  // Scratch device memory owned by this call.
  vp8a_status scratch(size_t bytes, void** dev);
  // Scratch device memory holding a copy of `bytes` host bytes (a table the
  // call built). The host buffer may go away once this returns; the copy
  // is stream-ordered and the call does not wait for it.
  vp8a_status upload(const void* host, size_t bytes, void** dev);
  // Host copy of a small buffer that may be host or device memory (for
  // metadata the host logic itself reads, e.g. reference ids).
  vp8a_status read_to_host(const void* p, size_t bytes, void* host_dst);
  // Store a small host value into an output that may be host or device
  // memory.
  vp8a_status write_from_host(void* dst, const void* host_src, size_t bytes);
  // Copies host outputs back and synchronises when any host buffer was
  // involved (otherwise the call stays asynchronous on the stream).
  vp8a_status finish();
  bool touched_host() const { return host_; }
  void force_sync() { host_ = true; }

 private:
  vp8a_status classify(const void* p, bool* is_device);
  vp8a_ctx* ctx_;
  bool host_ = false;
  struct Back {
    void* host;
    void* dev;
    size_t bytes;
  };
  std::vector<Back> backs_;
  std::vector<void*> owned_;
};

inline unsigned grid_for(size_t n, unsigned block) {
  return (unsigned)((n + block - 1) / block);
}

// Reads the device status word after the call's kernels and maps it.
vp8a_status check_device_status(vp8a_ctx* ctx);

// Device views left by predict_frame: the staged decisions and the output
// planes (device pointers) now holding the prediction, plus the host copy of
// the reference ids.
struct FramePrediction {
  const vp8a_mb_decision* dec = nullptr;
  vp8a_planes planes{};
  uint8_t ref_ids[3] = {0, 0, 0};
  uint32_t n_refs = 0;
  alignas(16) unsigned char args[320];  // the prediction kernel's arguments
};

// Validates and stages the arguments of vp8a_predict_inter_frame through
// `st` and queues the per-MB §18 prediction into `out` (predict.cu); with
// `defer` it only prepares the launch, which predict_frames then makes for
// many frames at once.
vp8a_status predict_frame(vp8a_ctx* ctx, Stager& st, const vp8a_planes* refs, const uint8_t* ref_ids,
                          uint32_t n_refs, const vp8a_mb_decision* decisions, uint32_t full_pixel,
                          uint32_t filter_set, const vp8a_planes* out, FramePrediction* fp, bool defer = false);

// One launch predicting every deferred frame of `fps`.
vp8a_status predict_frames(vp8a_ctx* ctx, Stager& st, const FramePrediction* fps, uint32_t n);

}  // namespace vp8a

// ------------------------------------------------------------ device helpers
namespace vp8a_dev {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// §18.3 six-tap filter table (SIXTAP_FILTERS, src/motion_comp.rs:294;
// RFC 6386 §18.3 filters[8][6]). One copy per translation unit.
static __constant__ int c_sixtap[8][6] = {
    {0, 0, 128, 0, 0, 0},     {0, -6, 123, 12, -1, 0}, {2, -11, 108, 36, -8, 1},
    {0, -9, 93, 50, -6, 0},   {3, -16, 77, 77, -16, 3}, {0, -6, 50, 93, -9, 0},
    {1, -8, 36, 108, -11, 2}, {0, -1, 12, 123, -6, 0},
};

// A batched launch's CTA finds its job: thread 0 searches the CTA offsets
// (cta_start[j] <= blockIdx.x < cta_start[j + 1], n_jobs + 1 entries),
// copies the job's arguments into shared `*sa` and its first CTA and CTA
// count into `first[0..1]`; the block then synchronises.
template <typename Args>
__device__ __forceinline__ void find_job(const Args* jobs, const uint32_t* cta_start, int n_jobs, Args* sa,
                                         uint32_t* first) {
  if (threadIdx.x == 0) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cta_start[mid] <= blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    *sa = jobs[lo];
    first[0] = cta_start[lo];
    first[1] = cta_start[lo + 1] - cta_start[lo];
  }
  __syncthreads();
}

// interp (src/motion_comp.rs:396): dot product, (a + 64) >> 7, clamp255.
__device__ __forceinline__ int interp6(const int* f, int s0, int s1, int s2, int s3, int s4, int s5) {
  int a = s0 * f[0] + s1 * f[1] + s2 * f[2] + s3 * f[3] + s4 * f[4] + s5 * f[5];
  return clampi((a + 64) >> 7, 0, 255);
}

// interp with the half-pel taps (row 4: 3, -16, 77, 77, -16, 3) as
// literals; the integer dot product is the same.
__device__ __forceinline__ int interp6_half(int s0, int s1, int s2, int s3, int s4, int s5) {
  const int a = 3 * (s0 + s5) - 16 * (s1 + s4) + 77 * (s2 + s3);
  return clampi((a + 64) >> 7, 0, 255);
}

}  // namespace vp8a_dev
