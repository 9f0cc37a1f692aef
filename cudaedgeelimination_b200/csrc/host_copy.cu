// Copies between device memory and caller host memory that is not page-locked.
//
// The runtime moves a pageable buffer through its own small staging area at a few GB/s; a large
// k-opt cost matrix (126 MB for 200,000 rows) then takes tens of milliseconds to reach the
// caller. Here a large copy goes through the context's pinned staging buffers instead: the DMA of
// one 16 MB chunk overlaps host threads copying the previous chunk between the staging buffer and
// the caller's memory (which also spreads the first-touch page faults of a fresh destination over
// the threads). Page-locked destinations and small copies take one cudaMemcpyAsync.
#include "cee_internal.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

namespace cee {
namespace {

constexpr size_t kStageChunk = size_t{16} << 20;
constexpr size_t kStageMinBytes = size_t{4} << 20;   // smaller copies: one cudaMemcpyAsync
constexpr size_t kBytesPerThread = size_t{2} << 20;  // host threads per chunk: at most chunk / 2 MB
constexpr int kMaxThreads = 8;

bool PageLocked(const void* p) {
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeHost;
}

cudaError_t EnsureStage(HostStage& h) {
  if (h.ready) return cudaSuccess;
  cudaError_t status = cudaSuccess;
  for (int b = 0; b < kStageBuffers && status == cudaSuccess; ++b) {
    status = cudaHostAlloc(reinterpret_cast<void**>(&h.buf[b]), kStageChunk, cudaHostAllocDefault);
    if (status == cudaSuccess) status = cudaEventCreateWithFlags(&h.ev[b], cudaEventDisableTiming);
  }
  if (status != cudaSuccess) {
    h.Release();
    return status;
  }
  h.ready = true;
  return cudaSuccess;
}

int ThreadsFor(size_t bytes) {
  const size_t per_chunk = std::min(bytes, kStageChunk);
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  return static_cast<int>(std::max<size_t>(1, std::min<size_t>({static_cast<size_t>(kMaxThreads), hw,
                                                                 per_chunk / kBytesPerThread})));
}

// Runs worker(t) for t = 0 .. threads - 1 on new threads (each with the context's device current)
// while the calling thread runs `main`, then joins them.
template <typename Worker, typename Main>
void Team(int device, int threads, Worker worker, Main main) {
  std::vector<std::thread> team;
  team.reserve(static_cast<size_t>(threads));
  for (int t = 0; t < threads; ++t) {
    team.emplace_back([&worker, device, t] {
      cudaSetDevice(device);
      worker(t);
    });
  }
  main();
  for (std::thread& th : team) th.join();
}

}  // namespace

void HostStage::Release() {
  for (int b = 0; b < kStageBuffers; ++b) {
    if (ev[b] != nullptr) cudaEventSynchronize(ev[b]);
    if (buf[b] != nullptr) cudaFreeHost(buf[b]);
    if (ev[b] != nullptr) cudaEventDestroy(ev[b]);
    buf[b] = nullptr;
    ev[b] = nullptr;
  }
  ready = false;
}

cudaError_t CopyToHost(cee_ctx* ctx, void* dst, const void* src, size_t bytes) {
  cudaStream_t st = ctx->stream;
  if (bytes == 0) return cudaStreamSynchronize(st);
  if (bytes < kStageMinBytes || PageLocked(dst)) {
    cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
    return cudaStreamSynchronize(st);
  }
  HostStage& h = ctx->stage;
  cudaError_t status = EnsureStage(h);
  if (status != cudaSuccess) return status;
  const size_t chunks = (bytes + kStageChunk - 1) / kStageChunk;
  auto length = [&](size_t i) { return std::min(kStageChunk, bytes - i * kStageChunk); };
  const int threads = ThreadsFor(bytes);
  std::vector<std::atomic<int>> issued(chunks), copied(chunks);
  for (size_t i = 0; i < chunks; ++i) {
    issued[i].store(0, std::memory_order_relaxed);
    copied[i].store(0, std::memory_order_relaxed);
  }
  std::atomic<bool> failed{false};
  const uint8_t* from = static_cast<const uint8_t*>(src);
  uint8_t* to = static_cast<uint8_t*>(dst);
  auto issue = [&](size_t i) {
    const int b = static_cast<int>(i % kStageBuffers);
    cudaMemcpyAsync(h.buf[b], from + i * kStageChunk, length(i), cudaMemcpyDeviceToHost, st);
    cudaEventRecord(h.ev[b], st);
    issued[i].store(1, std::memory_order_release);
  };
  // chunk i lands in buffer i mod kStageBuffers; the buffer is refilled with chunk i + kStageBuffers
  // once every thread has copied its slice of chunk i out of it
  auto worker = [&](int t) {
    for (size_t i = 0; i < chunks; ++i) {
      while (issued[i].load(std::memory_order_acquire) == 0) std::this_thread::yield();
      const int b = static_cast<int>(i % kStageBuffers);
      if (cudaEventSynchronize(h.ev[b]) != cudaSuccess) failed.store(true);
      const size_t len = length(i), lo = len * t / threads, hi = len * (t + 1) / threads;
      if (!failed.load()) std::memcpy(to + i * kStageChunk + lo, h.buf[b] + lo, hi - lo);
      copied[i].fetch_add(1, std::memory_order_release);
    }
  };
  Team(ctx->device, threads, worker, [&] {
    for (size_t i = 0; i < chunks; ++i) {
      if (i >= kStageBuffers) {
        while (copied[i - kStageBuffers].load(std::memory_order_acquire) < threads) std::this_thread::yield();
      }
      issue(i);
    }
  });
  status = cudaStreamSynchronize(st);
  if (status == cudaSuccess && failed.load()) status = cudaErrorUnknown;
  return status;
}

cudaError_t CopyFromHost(cee_ctx* ctx, void* dst, const void* src, size_t bytes) {
  cudaStream_t st = ctx->stream;
  if (bytes == 0) return cudaSuccess;
  if (bytes < kStageMinBytes || PageLocked(src)) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  }
  HostStage& h = ctx->stage;
  cudaError_t status = EnsureStage(h);
  if (status != cudaSuccess) return status;
  const size_t chunks = (bytes + kStageChunk - 1) / kStageChunk;
  auto length = [&](size_t i) { return std::min(kStageChunk, bytes - i * kStageChunk); };
  const int threads = ThreadsFor(bytes);
  std::vector<std::atomic<int>> issued(chunks), copied(chunks);
  for (size_t i = 0; i < chunks; ++i) {
    issued[i].store(0, std::memory_order_relaxed);
    copied[i].store(0, std::memory_order_relaxed);
  }
  std::atomic<bool> failed{false};
  const uint8_t* from = static_cast<const uint8_t*>(src);
  uint8_t* to = static_cast<uint8_t*>(dst);
  // chunk i is staged in buffer i mod kStageBuffers once the DMA that last read that buffer (an
  // earlier chunk, or an earlier call's) has completed; its DMA goes out once every thread staged
  // its slice
  auto worker = [&](int t) {
    for (size_t i = 0; i < chunks; ++i) {
      const int b = static_cast<int>(i % kStageBuffers);
      if (i >= kStageBuffers) {
        while (issued[i - kStageBuffers].load(std::memory_order_acquire) == 0) std::this_thread::yield();
      }
      if (cudaEventSynchronize(h.ev[b]) != cudaSuccess) failed.store(true);
      const size_t len = length(i), lo = len * t / threads, hi = len * (t + 1) / threads;
      if (!failed.load()) std::memcpy(h.buf[b] + lo, from + i * kStageChunk + lo, hi - lo);
      copied[i].fetch_add(1, std::memory_order_release);
    }
  };
  Team(ctx->device, threads, worker, [&] {
    for (size_t i = 0; i < chunks; ++i) {
      while (copied[i].load(std::memory_order_acquire) < threads) std::this_thread::yield();
      const int b = static_cast<int>(i % kStageBuffers);
      cudaMemcpyAsync(to + i * kStageChunk, h.buf[b], length(i), cudaMemcpyHostToDevice, st);
      cudaEventRecord(h.ev[b], st);
      issued[i].store(1, std::memory_order_release);
    }
  });
  status = cudaGetLastError();
  if (status == cudaSuccess && failed.load()) status = cudaErrorUnknown;
  return status;
}

}  // namespace cee
