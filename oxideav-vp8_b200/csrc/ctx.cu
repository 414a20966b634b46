// ctx.cu — context lifetime, host/device staging and error reporting of the
// vp8a C ABI. No compute happens here; every compute entry point launches
// its own CUDA kernels on the context stream. There is no CPU fallback: a
// process without a visible GPU gets VP8A_E_NO_DEVICE from vp8a_ctx_create.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "vp8a_internal.cuh"


namespace vp8a {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

vp8a_status cuda_fail(cudaError_t e, const char* what) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  set_error(buf);
  if (e == cudaErrorMemoryAllocation) return VP8A_E_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return VP8A_E_NO_DEVICE;
  return VP8A_E_CUDA;
}

Stager::~Stager() {
  for (void* p : owned_) cudaFreeAsync(p, ctx_->stream);
}

vp8a_status Stager::classify(const void* p, bool* is_device) {
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *is_device = false;
    return VP8A_OK;
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) {
    if (a.type == cudaMemoryTypeDevice && a.device != ctx_->device) {
      set_error("buffer lives on a different GPU than the context");
      return VP8A_E_INVALID_ARGUMENT;
    }
    *is_device = true;
  } else {
    *is_device = false;
  }
  return VP8A_OK;
}

vp8a_status Stager::scratch(size_t bytes, void** dev) {
  void* d = nullptr;
  VP8A_CUDA(cudaMallocAsync(&d, bytes ? bytes : 16, ctx_->stream));
  owned_.push_back(d);
  *dev = d;
  return VP8A_OK;
}

vp8a_status Stager::upload(const void* host, size_t bytes, void** dev) {
  vp8a_status st = scratch(bytes, dev);
  if (st != VP8A_OK || bytes == 0) return st;
  if (!ctx_->up_host || bytes > vp8a_ctx::UP_SLOT_BYTES) {
    // Pageable source: the call waits for the copy before it returns.
    VP8A_CUDA(cudaMemcpyAsync(*dev, host, bytes, cudaMemcpyHostToDevice, ctx_->stream));
    VP8A_CUDA(cudaStreamSynchronize(ctx_->stream));
    return VP8A_OK;
  }
  const unsigned k = ctx_->up_next++ % vp8a_ctx::UP_SLOTS;
  VP8A_CUDA(cudaEventSynchronize(ctx_->up_ev[k]));  // that slot's previous upload is done
  uint8_t* slot = ctx_->up_host + (size_t)k * vp8a_ctx::UP_SLOT_BYTES;
  memcpy(slot, host, bytes);
  VP8A_CUDA(cudaMemcpyAsync(*dev, slot, bytes, cudaMemcpyHostToDevice, ctx_->stream));
  VP8A_CUDA(cudaEventRecord(ctx_->up_ev[k], ctx_->stream));
  return VP8A_OK;
}

vp8a_status Stager::read_to_host(const void* p, size_t bytes, void* host_dst) {
  if (!p) {
    set_error("null input buffer");
    return VP8A_E_INVALID_ARGUMENT;
  }
  bool is_dev = false;
  vp8a_status st = classify(p, &is_dev);
  if (st != VP8A_OK) return st;
  if (!is_dev) {
    memcpy(host_dst, p, bytes);
    return VP8A_OK;
  }
  VP8A_CUDA(cudaMemcpyAsync(host_dst, p, bytes, cudaMemcpyDeviceToHost, ctx_->stream));
  VP8A_CUDA(cudaStreamSynchronize(ctx_->stream));
  return VP8A_OK;
}

vp8a_status Stager::write_from_host(void* dst, const void* host_src, size_t bytes) {
  if (!dst) {
    set_error("null output buffer");
    return VP8A_E_INVALID_ARGUMENT;
  }
  bool is_dev = false;
  vp8a_status st = classify(dst, &is_dev);
  if (st != VP8A_OK) return st;
  if (!is_dev) {
    memcpy(dst, host_src, bytes);
    return VP8A_OK;
  }
  VP8A_CUDA(cudaMemcpyAsync(dst, host_src, bytes, cudaMemcpyHostToDevice, ctx_->stream));
  VP8A_CUDA(cudaStreamSynchronize(ctx_->stream));
  return VP8A_OK;
}

vp8a_status Stager::in(const void* p, size_t bytes, const void** dev) {
  if (!p) {
    set_error("null input buffer");
    return VP8A_E_INVALID_ARGUMENT;
  }
  bool is_dev = false;
  vp8a_status st = classify(p, &is_dev);
  if (st != VP8A_OK) return st;
  if (is_dev) {
    *dev = p;
    return VP8A_OK;
  }
  host_ = true;
  void* d = nullptr;
  st = scratch(bytes, &d);
  if (st != VP8A_OK) return st;
  if (bytes) VP8A_CUDA(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, ctx_->stream));
  *dev = d;
  return VP8A_OK;
}

vp8a_status Stager::out(void* p, size_t bytes, void** dev) {
  if (!p) {
    set_error("null output buffer");
    return VP8A_E_INVALID_ARGUMENT;
  }
  bool is_dev = false;
  vp8a_status st = classify(p, &is_dev);
  if (st != VP8A_OK) return st;
  if (is_dev) {
    *dev = p;
    return VP8A_OK;
  }
  host_ = true;
  void* d = nullptr;
  st = scratch(bytes, &d);
  if (st != VP8A_OK) return st;
  backs_.push_back({p, d, bytes});
  *dev = d;
  return VP8A_OK;
}

vp8a_status Stager::inout(void* p, size_t bytes, void** dev) {
  const void* d = nullptr;
  bool is_dev = false;
  if (!p) {
    set_error("null in/out buffer");
    return VP8A_E_INVALID_ARGUMENT;
  }
  vp8a_status st = classify(p, &is_dev);
  if (st != VP8A_OK) return st;
  st = in(p, bytes, &d);
  if (st != VP8A_OK) return st;
  if (!is_dev) backs_.push_back({p, const_cast<void*>(d), bytes});
  *dev = const_cast<void*>(d);
  return VP8A_OK;
}

vp8a_status Stager::finish() {
  for (const Back& b : backs_)
    if (b.bytes)
      VP8A_CUDA(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, ctx_->stream));
  if (host_) VP8A_CUDA(cudaStreamSynchronize(ctx_->stream));
  return VP8A_OK;
}

vp8a_status check_device_status(vp8a_ctx* ctx) {
  uint32_t st = 0;
  VP8A_CUDA(cudaMemcpyAsync(&st, ctx->d_status, sizeof st, cudaMemcpyDeviceToHost, ctx->stream));
  VP8A_CUDA(cudaStreamSynchronize(ctx->stream));
  if (st == DEV_OK) return VP8A_OK;
  VP8A_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream));
  if (st == DEV_TIMEOUT) {
    set_error("device wavefront wait exceeded its iteration budget");
    return VP8A_E_DEVICE_TIMEOUT;
  }
  set_error("device kernel rejected its input");
  return VP8A_E_INVALID_ARGUMENT;
}

}  // namespace vp8a

using namespace vp8a;

extern "C" {

vp8a_status vp8a_ctx_create(int device, vp8a_ctx** out) {
  if (!out) {
    set_error("null output pointer");
    return VP8A_E_INVALID_ARGUMENT;
  }
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device is visible; libvp8a has no CPU fallback");
    return VP8A_E_NO_DEVICE;
  }
  if (device < 0 || device >= n) {
    set_error("device index out of range");
    return VP8A_E_INVALID_ARGUMENT;
  }
  VP8A_CUDA(cudaSetDevice(device));
  vp8a_ctx* c = new vp8a_ctx();
  c->device = device;
  cudaDeviceProp prop;
  cudaError_t pe = cudaGetDeviceProperties(&prop, device);
  if (pe != cudaSuccess) {
    delete c;
    return cuda_fail(pe, "cudaGetDeviceProperties");
  }
  c->sm_count = prop.multiProcessorCount;
  // Keep freed stream-ordered staging memory in the device pool instead of
  // returning it to the driver at every synchronisation, so per-call
  // staging allocations stay cheap.
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  cudaError_t se = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (se != cudaSuccess) {
    delete c;
    return cuda_fail(se, "cudaStreamCreateWithFlags");
  }
  // The bit-cost table of bool_bits (src/encoder.rs:2243-2260), built on
  // the host so device and host RD costs use identical doubles.
  double t[256];
  t[0] = -std::log2(1.0 / 256.0);
  for (int p = 1; p < 256; p++) t[p] = -std::log2((double)p / 256.0);
  if ((se = cudaMalloc(&c->d_status, sizeof(uint32_t))) != cudaSuccess ||
      (se = cudaMalloc(&c->d_bit_cost, sizeof t)) != cudaSuccess ||
      (se = cudaMemcpy(c->d_bit_cost, t, sizeof t, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (se = cudaMemset(c->d_status, 0, sizeof(uint32_t))) != cudaSuccess) {
    vp8a_ctx_destroy(c);
    return cuda_fail(se, "context buffers");
  }
  if ((se = cudaHostAlloc((void**)&c->up_host, vp8a_ctx::UP_SLOTS * vp8a_ctx::UP_SLOT_BYTES,
                          cudaHostAllocDefault)) != cudaSuccess) {
    c->up_host = nullptr;
    vp8a_ctx_destroy(c);
    return cuda_fail(se, "pinned upload ring");
  }
  for (int k = 0; k < vp8a_ctx::UP_SLOTS; k++)
    if ((se = cudaEventCreateWithFlags(&c->up_ev[k], cudaEventDisableTiming)) != cudaSuccess) {
      vp8a_ctx_destroy(c);
      return cuda_fail(se, "upload events");
    }
  *out = c;
  return VP8A_OK;
}

vp8a_status vp8a_ctx_destroy(vp8a_ctx* ctx) {
  if (!ctx) return VP8A_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->d_bit_cost) cudaFree(ctx->d_bit_cost);
  for (int k = 0; k < vp8a_ctx::UP_SLOTS; k++)
    if (ctx->up_ev[k]) cudaEventDestroy(ctx->up_ev[k]);
  if (ctx->up_host) cudaFreeHost(ctx->up_host);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return VP8A_OK;
}

void* vp8a_ctx_stream(vp8a_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

vp8a_status vp8a_ctx_synchronize(vp8a_ctx* ctx) {
  if (!ctx) return VP8A_E_INVALID_ARGUMENT;
  // Waits for the stream and reports a bounded device wait that ran out in
  // an asynchronous call since the last check.
  return check_device_status(ctx);
}

uint64_t vp8a_ctx_launch_count(const vp8a_ctx* ctx) { return ctx ? ctx->launches : 0; }

vp8a_status vp8a_ctx_set_wait_limit(vp8a_ctx* ctx, uint64_t polls) {
  if (!ctx) return VP8A_E_INVALID_ARGUMENT;
  ctx->wait_limit = polls;
  return VP8A_OK;
}

vp8a_status vp8a_ctx_set_trellis_strength(vp8a_ctx* ctx, double strength) {
  if (!ctx) return VP8A_E_INVALID_ARGUMENT;
  // TrellisStrength::new (src/encoder.rs:2686-2692): NaN is the default,
  // the rest is clamped to 0..=8.
  ctx->trellis_strength = strength != strength ? 1.0 : (strength < 0.0 ? 0.0 : (strength > 8.0 ? 8.0 : strength));
  return VP8A_OK;
}

vp8a_status vp8a_ctx_set_subpel_planes(vp8a_ctx* ctx, uint32_t on) {
  if (!ctx) return VP8A_E_INVALID_ARGUMENT;
  ctx->subpel_planes = on != 0;
  return VP8A_OK;
}

vp8a_status vp8a_ctx_set_autotune(vp8a_ctx* ctx, uint32_t on) {
  if (!ctx) return VP8A_E_INVALID_ARGUMENT;
  ctx->autotune = on != 0;
  return VP8A_OK;
}

vp8a_status vp8a_ctx_force_sweep_layout(vp8a_ctx* ctx, uint32_t passes, uint32_t threads, uint32_t prefetch) {
  if (!ctx || passes > 3 || (passes && (threads < 32 || threads > 1024 || threads % 32 != 0))) {
    set_error("passes must be 0-3 and threads a multiple of 32 in 32..1024");
    return VP8A_E_INVALID_ARGUMENT;
  }
  ctx->force_layout[0] = (int)passes;
  ctx->force_layout[1] = (int)threads;
  ctx->force_layout[2] = prefetch != 0;
  return VP8A_OK;
}

vp8a_status vp8a_ctx_last_sweep_layout(const vp8a_ctx* ctx, uint32_t out[4]) {
  if (!ctx || !out) return VP8A_E_INVALID_ARGUMENT;
  for (int i = 0; i < 4; i++) out[i] = (uint32_t)ctx->last_layout[i];
  return VP8A_OK;
}

const char* vp8a_last_error(void) { return g_last_error.c_str(); }

uint32_t vp8a_abi_version(void) { return VP8A_ABI_VERSION; }

double vp8a_rd_lambda(uint32_t qi) {
  // AC_QLOOKUP (src/inverse_transform.rs:87; RFC 6386 §14.1 ac_qlookup).
  static const int16_t ac[128] = {
      4,   5,   6,   7,   8,   9,   10,  11,  12,  13,  14,  15,  16,  17,  18,  19,
      20,  21,  22,  23,  24,  25,  26,  27,  28,  29,  30,  31,  32,  33,  34,  35,
      36,  37,  38,  39,  40,  41,  42,  43,  44,  45,  46,  47,  48,  49,  50,  51,
      52,  53,  54,  55,  56,  57,  58,  60,  62,  64,  66,  68,  70,  72,  74,  76,
      78,  80,  82,  84,  86,  88,  90,  92,  94,  96,  98,  100, 102, 104, 106, 108,
      110, 112, 114, 116, 119, 122, 125, 128, 131, 134, 137, 140, 143, 146, 149, 152,
      155, 158, 161, 164, 167, 170, 173, 177, 181, 185, 189, 193, 197, 201, 205, 209,
      213, 217, 221, 225, 229, 234, 239, 245, 249, 254, 259, 264, 269, 274, 279, 284};
  double q = (double)ac[qi > 127 ? 127 : qi];
  return q * q / 32.0;
}

}  // extern "C"
