// Device -> pageable host copies of the large results (Mat_el and its y2) of the one-shot
// entry points that take host buffers.  One cudaMemcpy into fresh pageable memory runs at
// the speed of the driver's single staging copy plus the first-touch page faults of the
// destination: 15-20 ms for a 77 MB matrix on a B200 host, against 1.4 ms device -> pinned.
// Here kSlots threads each own one pinned staging slot and one stream; a thread copies its
// chunks from the device into its slot, waits for that copy and copies the slot into the
// destination on the CPU, so the device copies of one thread overlap the host copies and
// page faults of the others.  The slots are pinned once per process; concurrent calls take
// turns on them.  A copy below two chunks, or into a destination that is itself pinned
// (cudaHostAlloc'd or registered), goes through one cudaMemcpyAsync on the caller's
// stream, which is then synchronised: either way the copy is complete on return.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"

namespace mqct {
namespace {

constexpr int kSlots = 4;
constexpr size_t kChunk = (size_t)8 << 20;
std::mutex g_mu;
void* g_slot[kSlots] = {nullptr, nullptr, nullptr, nullptr};
bool g_failed = false;

bool slots_ready() {  // with g_mu held
  if (g_slot[kSlots - 1]) return true;
  if (g_failed) return false;
  for (int w = 0; w < kSlots; ++w)
    if (!g_slot[w] && cudaHostAlloc(&g_slot[w], kChunk, cudaHostAllocPortable) != cudaSuccess) {
      g_slot[w] = nullptr;
      cudaGetLastError();
      g_failed = true;  // pinned memory refused: every copy takes the plain path
      return false;
    }
  return true;
}

}  // namespace

int copy_d2h_host(void* dst, const void* src, size_t bytes, cudaStream_t after) {
  if (bytes == 0) return MQCT_OK;
  {
    // a pinned (page-locked or registered) destination takes the copy engine directly
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeHost) {
      MQCT_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, after));
      MQCT_CUDA_TRY(cudaStreamSynchronize(after));
      return MQCT_OK;
    }
    cudaGetLastError();  // an unregistered pointer may leave an error code on older drivers
  }
  std::unique_lock<std::mutex> lk(g_mu);
  if (bytes < 2 * kChunk || !slots_ready()) {  // one copy on `after`, complete on return
    lk.unlock();
    MQCT_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, after));
    MQCT_CUDA_TRY(cudaStreamSynchronize(after));
    return MQCT_OK;
  }
  int dev = 0;
  MQCT_CUDA_TRY(cudaGetDevice(&dev));
  cudaEvent_t ready = nullptr;
  MQCT_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  cudaError_t e0 = cudaEventRecord(ready, after);
  if (e0 != cudaSuccess) {
    cudaEventDestroy(ready);
    set_error("copy_d2h_host: %s", cudaGetErrorString(e0));
    return MQCT_E_CUDA;
  }
  const size_t n_chunks = (bytes + kChunk - 1) / kChunk;
  std::vector<cudaError_t> err(kSlots, cudaSuccess);
  auto work = [&](int w) {
    cudaError_t e = cudaSetDevice(dev);
    cudaStream_t s = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ready, 0);
    for (size_t c = (size_t)w; c < n_chunks && e == cudaSuccess; c += kSlots) {
      const size_t off = c * kChunk, len = bytes - off < kChunk ? bytes - off : kChunk;
      e = cudaMemcpyAsync(g_slot[w], static_cast<const char*>(src) + off, len,
                          cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e == cudaSuccess) memcpy(static_cast<char*>(dst) + off, g_slot[w], len);
    }
    if (s) cudaStreamDestroy(s);
    err[w] = e;
  };
  std::vector<std::thread> th;
  std::vector<int> inline_w;  // workers whose thread could not start run here, in turn
  for (int w = 1; w < kSlots; ++w) {
    try {
      th.emplace_back(work, w);
    } catch (...) {
      inline_w.push_back(w);
    }
  }
  work(0);
  for (int w : inline_w) work(w);
  for (auto& t : th) t.join();
  cudaEventDestroy(ready);
  for (int w = 0; w < kSlots; ++w)
    if (err[w] != cudaSuccess) {
      set_error("copy_d2h_host: %s", cudaGetErrorString(err[w]));
      return MQCT_E_CUDA;
    }
  return MQCT_OK;
}

}  // namespace mqct
