// noalloc.cu — sg_search_noalloc: one query through the whole search path with every scratch
// buffer taken from a fixed array in device memory, so the call itself allocates nothing.
//
// Who needs it: callers that must not allocate device memory while they serve queries — a
// latency-critical serving thread (cudaFree synchronises the whole device and cudaMalloc can
// wait behind kernels already in flight), or a host whose device-memory budget is fixed up
// front (another framework's caching allocator owns the rest of HBM, so a fresh cudaMalloc can
// fail mid-request). sg_search grows its workspace with cudaMalloc; this entry point does not.
//
// The scratch is g_scratch, a file-scope __device__ array of kScratchBytes (32 MiB). Every GPU
// that loads this library holds it until the process exits. In host code the name g_scratch is
// only a host-side stand-in: a kernel given it would fault, or silently use the wrong memory
// where the GPU can reach host memory. So, once per device and with that device current, the
// first call on the device asks cudaGetSymbolAddress for the real device address and keeps it;
// that first call should therefore come before any stream capture begins on the caller's side.
//
// Failures on the device (a bounded tensor-core wait that ran out, a work queue or candidate
// buffer that overflowed) cannot be returned from an asynchronous call: a last one-thread kernel
// turns them into the count SG_COUNT_FAILED in *d_out_count, which the caller checks with its
// results.
#include <mutex>
#include <string>

#include "internal.hpp"

namespace {

constexpr size_t kScratchBytes = 32u << 20;
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
unsigned char* g_addr[kMaxDevices] = {};

// Device address of g_scratch on `device` (which must be current), looked up once.
int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return sg::fail(SG_ERR_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> g(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess)
      return sg::fail(SG_ERR_DEVICE, std::string("cudaGetSymbolAddress(g_scratch): ") + cudaGetErrorString(e));
    g_addr[device] = static_cast<unsigned char*>(p);
  }
  *out = g_addr[device];
  return SG_OK;
}

// Bump allocator over the scratch array (256-byte aligned pieces); sizes only when base is null.
struct Carve {
  unsigned char* base;
  size_t used = 0;
  template <typename T>
  T* take(size_t n) {
    size_t off = (used + 255) & ~size_t(255);
    used = off + (n ? n : 1) * sizeof(T);
    return base ? reinterpret_cast<T*>(base + off) : nullptr;
  }
};

void carve_workspace(Carve& c, sg::Workspace& w, const sg::DevIndex& x, uint32_t P, uint32_t cand,
                     uint64_t items, uint32_t cbuf, bool need_q256) {
  if (need_q256) w.q256 = c.take<float>(SG_PDIM);
  w.q16 = c.take<__nv_bfloat16>(SG_PDIM);
  w.tables = c.take<uint8_t>(SG_GROUPS * 16);
  w.qp = c.take<float4>(1);
  w.qnorm = c.take<float>(1);
  w.wq = c.take<int8_t>(SG_DIM);
  w.winv = c.take<float>(1);
  w.wq256 = c.take<int8_t>(SG_PDIM);
  w.winv256 = c.take<float>(1);
  w.scores = c.take<float>(x.kc);
  w.probe_sc = c.take<float>(P);
  w.probe_cl = c.take<uint32_t>(P);
  w.probe_off = c.take<uint32_t>(P);
  w.probe_n = c.take<uint32_t>(1);
  w.scanned = c.take<uint64_t>(1);
  w.items = c.take<uint4>(items);
  w.seed_items = c.take<uint4>(1);
  w.counters = c.take<uint32_t>(8);
  w.thr = c.take<uint32_t>(1);
  w.ccount = c.take<uint32_t>(1);
  w.cbuf_est = c.take<uint32_t>(cbuf);
  w.cbuf_info = c.take<uint2>(cbuf);
  w.overflow = c.take<uint8_t>(1);
  w.cest = c.take<float>(cand);
  w.cid = c.take<uint32_t>(cand);
  w.cerr = c.take<float>(cand);
  w.cn = c.take<uint32_t>(1);
  w.lid = c.take<uint32_t>(cand);
  w.lsc = c.take<float>(cand);
  w.ln = c.take<uint32_t>(1);
}

// Runs after the rerank on the call's stream: a device-side failure of any earlier stage (the
// status word's overflow or timeout bit, or the candidate buffer's overflow flag) replaces the
// result count with SG_COUNT_FAILED.
__global__ void k_noalloc_status(const uint32_t* __restrict__ counters, const uint8_t* __restrict__ overflow,
                                 uint32_t* __restrict__ out_n) {
  if (threadIdx.x == 0 && ((counters[2] & (sg::kStatusOverflow | sg::kStatusTimeout)) || overflow[0]))
    out_n[0] = SG_COUNT_FAILED;
}

}  // namespace

extern "C" int sg_search_noalloc(sg_index* h, const float* d_q768, const float* d_q256,
                                 const sg_params* params, const uint64_t* d_allow_bits,
                                 uint64_t allow_words, float* d_out_scores, uint32_t* d_out_ids,
                                 uint32_t* d_out_count, void* stream) {
  if (!h || !params || !d_q768 || !d_out_count || (params->k && (!d_out_scores || !d_out_ids)))
    return sg::fail(SG_ERR_INVALID, "null argument");
  int rc = sg::index_check_params(h, params);
  if (rc) return rc;
  const sg::DevIndex& x = *sg::index_arrays(h);
  const sg::Config cfg = sg::index_config(h);  // one snapshot: sg_set_tuning may run concurrently
  const sg_params& p = *params;
  cudaError_t e = cudaSetDevice(x.device);
  if (e != cudaSuccess) return sg::fail(SG_ERR_DEVICE, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  unsigned char* base = nullptr;
  if ((rc = scratch_address(x.device, &base))) return rc;

  // Sizes of one query's buffers: the exact work-item and candidate-buffer bounds sg_search uses
  // for one query. A slot is appended at most once, so the probed clusters' slots bound the
  // candidate buffer; the chunk scan keeps at most cand per chunk, so chunks x cand does too.
  const uint32_t P = sg::probe_stride(x, p.nprobe);
  const uint32_t cand = p.cand > 0 ? p.cand : 1;
  const uint64_t items = x.h_chunks_desc_prefix[P];
  const uint64_t slots = x.h_slots_desc_prefix[P];
  const uint64_t cbuf = ((items * cand < slots ? items * cand : slots) + 3) & ~3ull;
  Carve sizing{nullptr};
  sg::Workspace w;
  carve_workspace(sizing, w, x, P, cand, items, (uint32_t)cbuf, d_q256 == nullptr);
  if (sizing.used > kScratchBytes || cbuf > 0x7FFFFFFFull)
    return sg::fail(SG_ERR_INVALID,
                    "sg_search_noalloc: these params need " + std::to_string(sizing.used) +
                        " bytes of scratch; the fixed device array holds " +
                        std::to_string(kScratchBytes) + " (lower nprobe or cand, or use sg_search)");
  Carve c{base};
  w = sg::Workspace();
  carve_workspace(c, w, x, P, cand, items, (uint32_t)cbuf, d_q256 == nullptr);
  w.q768 = const_cast<float*>(d_q768);
  if (d_q256) w.q256 = const_cast<float*>(d_q256);
  w.item_cap = items;
  w.cbuf_per_q = (uint32_t)cbuf;
  w.out_sc = d_out_scores;
  w.out_id = d_out_ids;
  w.out_n = d_out_count;

  // The array keeps the previous call's contents: clear everything that must start at zero.
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((e = cudaMemsetAsync(w.counters, 0, 8 * sizeof(uint32_t), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(w.thr, 0, sizeof(uint32_t), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(w.ccount, 0, sizeof(uint32_t), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(w.overflow, 0, 1, st)) != cudaSuccess)
    return sg::fail(SG_ERR_DEVICE, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  if (!d_q256) sg::launch_prefix(w, 1, st);
  sg::launch_prep(x, w, 1, st);
  if ((e = sg::launch_route_scores(x, w, 1, cfg.route_precision, st)) != cudaSuccess)
    return sg::fail(SG_ERR_DEVICE, std::string("sg_search_noalloc routing: ") + cudaGetErrorString(e));
  // one query runs with the small-batch shapes, as sg_search runs it
  sg::launch_route_select(x, w, 1, p, cfg.route_precision, cfg.small_chunk_blocks, cfg.small_seed_blocks,
                          true, st);
  if (p.cand > 0) {
    sg::launch_scan(x, w, 1, p, d_allow_bits, allow_words, sg::index_sms(h), cfg.small_chunk_blocks,
                    cfg.small_seed_blocks, cfg.scan_ctas_per_sm, st);
    sg::launch_cut(x, w, 1, p, st);
  } else if ((e = cudaMemsetAsync(w.cn, 0, sizeof(uint32_t), st)) != cudaSuccess) {
    return sg::fail(SG_ERR_DEVICE, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  }
  sg::launch_rerank(x, w, 1, p, st, nullptr, nullptr);
  k_noalloc_status<<<1, 32, 0, st>>>(w.counters, w.overflow, w.out_n);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return sg::fail(SG_ERR_DEVICE, std::string("sg_search_noalloc launch: ") + cudaGetErrorString(e));
  return SG_OK;
}
