// Host side of the serving loop (serve_screen.cuh): HBM-budget admission into a device arena,
// device-resident snapshots kept across jobs until released, job posting through a host-mapped
// mailbox that the persistent kernel's dispatcher warp reads, completion polling and result download.
#include "cee.h"
#include "cee_internal.h"

#include "serve_screen.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

namespace cee {
namespace {

constexpr size_t kArenaAlign = 256;

int TemplateCount(int k) { return k == 3 ? 4 : (k == 4 ? 25 : 208); }

// First-fit allocator over [0, capacity) with coalescing frees.
class Arena {
 public:
  void Reset(size_t capacity) {
    free_.clear();
    if (capacity > 0) free_[0] = capacity;
    used_ = 0;
  }
  bool Allocate(size_t bytes, size_t* offset) {
    bytes = (std::max<size_t>(bytes, 1) + kArenaAlign - 1) & ~(kArenaAlign - 1);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *offset = it->first;
        const size_t rest = it->second - bytes;
        const size_t start = it->first + bytes;
        free_.erase(it);
        if (rest > 0) free_[start] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void Free(size_t offset, size_t bytes) {
    bytes = (std::max<size_t>(bytes, 1) + kArenaAlign - 1) & ~(kArenaAlign - 1);
    used_ -= bytes;
    auto next = free_.lower_bound(offset);
    size_t start = offset, size = bytes;
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == offset) {
        start = prev->first;
        size += prev->second;
        free_.erase(prev);
      }
    }
    if (next != free_.end() && start + size == next->first) {
      size += next->second;
      free_.erase(next);
    }
    free_[start] = size;
  }
  size_t used() const { return used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t used_ = 0;
};

struct ServeSnapshotHost {
  bool live = false;
  bool released = false;
  size_t offset = 0, bytes = 0;
  int32_t n = 0, dist_type = 0;
  int64_t m = 0, adj = 0;
  int span = kSpanSmall;
  JvGraph g{};
  int refs = 0;
};

struct Download {
  void* host;
  size_t device_offset;
  size_t bytes;
};

struct ServeJobHost {
  bool live = false;
  int slot = -1;
  uint32_t generation = 0;
  int snapshot = -1;
  uint64_t tag = 0;
  int phase = 0;  // 0: on the GPU, 1: downloading, 2: done (no device work)
  bool direct = false;  // the kernel writes the outputs straight into page-locked host memory
  int status = CEE_OK;
  std::vector<std::pair<size_t, size_t>> regions;  // arena (offset, bytes) to free
  std::vector<Download> downloads;
};

// The downloads of a slot's current job, shared by the API thread (which fills the ticket at
// submission, before publishing the job) and the downloader thread (which issues the copies the
// moment it sees the job's finished word). Whichever thread first moves state from kArmed to
// kIssuing issues them; the job is reported once `event` has completed.
constexpr int kTicketIdle = 0, kTicketArmed = 1, kTicketIssuing = 2, kTicketIssued = 3;
constexpr int kMaxDownloads = 9;  // three segments x (costs, masks, first)
constexpr size_t kServeSmallDownload = size_t{4} << 20;
struct SlotTicket {
  std::atomic<int> state{kTicketIdle};
  uint32_t generation = 0;
  int count = 0;
  Download downloads[kMaxDownloads];
  cudaEvent_t event = nullptr;  // recorded on the download stream after the copies
};

}  // namespace

struct ServeState {
  cee_serve_config cfg{};
  DevBuf arena_buf, control, templates;
  Arena arena;
  // mapped: [slot] generation done, [kServeMaxSlots + slot] error word, [kServeLostWord] lost item
  uint32_t* finished_host = nullptr;
  uint32_t* finished_dev = nullptr;
  ServeMailbox* mailbox_host = nullptr;  // mapped: posted jobs (serve_screen.cuh)
  ServeMailbox* mailbox_dev = nullptr;
  uint32_t* words_host = nullptr;     // pinned: [0] = 0, [1] = 1, [2 + s] = generation of slot s
  uint8_t* pinned_stage = nullptr;    // snapshot packing
  size_t pinned_stage_bytes = 0;
  cee_serve_stats stats{};
  // downloads: jobs whose outputs total under kServeSmallDownload on d2h_small, larger ones on d2h, so a
  // witness array never queues behind a large k-opt matrix
  cudaStream_t server = nullptr, copy = nullptr, d2h = nullptr, d2h_small = nullptr;
  SlotTicket tickets[kServeMaxSlots];
  // the downloader thread: issues a job's copies as soon as its finished word lands, whether or not
  // the caller is polling (it sleeps while no job is armed)
  std::thread downloader;
  std::atomic<bool> downloader_stop{false};
  std::atomic<int> armed{0};
  std::mutex wake_mutex;
  std::condition_variable wake;
  cudaEvent_t kernel_done = nullptr;
  bool launched = false;
  int grid = 1;
  long long idle_limit = 1;
  bool slot_busy[kServeMaxSlots] = {};
  int next_slot = 0;
  uint32_t next_generation = 1;
  std::vector<ServeSnapshotHost> snapshots;
  std::vector<ServeJobHost> jobs;
  std::vector<int> finished_jobs;  // completed without device work, reported at the next poll
  int pending = 0;
  bool broken = false;  // an item was lost (see cee_serve_poll)
};

namespace {

ServeState* Serving(cee_ctx* ctx) { return ctx->serve; }

int ServeFail(cee_ctx* ctx, int code, const std::string& m) { return Fail(ctx, code, "serve: " + m); }

int EnsurePinned(cee_ctx* ctx, ServeState& s, size_t bytes) {
  if (bytes <= s.pinned_stage_bytes) return CEE_OK;
  if (s.pinned_stage != nullptr) cudaFreeHost(s.pinned_stage);
  s.pinned_stage = nullptr;
  const size_t want = std::max(bytes, s.pinned_stage_bytes * 2);
  const cudaError_t status = cudaHostAlloc(reinterpret_cast<void**>(&s.pinned_stage), want, cudaHostAllocDefault);
  if (status != cudaSuccess) {
    s.pinned_stage_bytes = 0;
    return CudaFail(ctx, status, "serve staging allocation");
  }
  s.pinned_stage_bytes = want;
  return CEE_OK;
}

// Stops a running kernel (stop word, then wait for it to end) so that the host may write
// snapshot memory, which the kernel reads through L1; the next launch clears the stop word.
int QuiesceServer(cee_ctx* ctx, ServeState& s) {
  if (!s.launched || cudaEventQuery(s.kernel_done) == cudaSuccess) return CEE_OK;
  ServeControl* ctl = static_cast<ServeControl*>(s.control.ptr);
  cudaMemcpyAsync(&ctl->stop, &s.words_host[1], sizeof(uint32_t), cudaMemcpyHostToDevice, s.copy);
  const cudaError_t status = cudaEventSynchronize(s.kernel_done);
  if (status != cudaSuccess) return CudaFail(ctx, status, "serve kernel stop");
  return CEE_OK;
}

int LaunchServer(cee_ctx* ctx, ServeState& s) {
  if (s.launched) {
    const cudaError_t q = cudaEventQuery(s.kernel_done);
    if (q == cudaErrorNotReady) return CEE_OK;  // still running
    if (q != cudaSuccess) return CudaFail(ctx, q, "serve kernel");
  }
  ServeControl* ctl = static_cast<ServeControl*>(s.control.ptr);
  cudaMemsetAsync(&ctl->stop, 0, sizeof(uint32_t), s.server);
  serve_kernel<<<s.grid, kServeWarps * 32, 0, s.server>>>(
      static_cast<ServeControl*>(s.control.ptr), s.mailbox_dev, s.finished_dev,
      static_cast<const uint8_t*>(s.templates.ptr), s.cfg.slots, s.idle_limit);
  cudaError_t status = cudaGetLastError();
  if (status == cudaSuccess) status = cudaEventRecord(s.kernel_done, s.server);
  if (status != cudaSuccess) return CudaFail(ctx, status, "serve kernel launch");
  s.launched = true;
  return CEE_OK;
}

int FreeSlot(const ServeState& s) {
  for (int i = 0; i < s.cfg.slots; ++i) {
    const int slot = (s.next_slot + i) % s.cfg.slots;
    if (!s.slot_busy[slot]) return slot;
  }
  return -1;
}

// cuPointerGetAttribute, from the driver through the runtime (the library links only cudart).
using PointerAttributeFn = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
PointerAttributeFn PointerAttribute() {
  static const PointerAttributeFn fn = [] {
    void* entry = nullptr;
    cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuPointerGetAttribute", &entry, 12000, cudaEnableDefault, &found) !=
            cudaSuccess ||
        found != cudaDriverEntryPointSuccess) {
      return static_cast<PointerAttributeFn>(nullptr);
    }
    return reinterpret_cast<PointerAttributeFn>(entry);
  }();
  return fn;
}

// The device address of the `bytes` bytes at `p` when all of them lie in one page-locked,
// device-mapped host allocation and `p` is `align`-byte aligned (the kernel may then write them in
// place), else null.
void* MappedRange(void* p, size_t bytes, size_t align) {
  if (p == nullptr || bytes == 0 || reinterpret_cast<uintptr_t>(p) % align != 0) return nullptr;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || a.devicePointer == nullptr) return nullptr;
  const PointerAttributeFn get = PointerAttribute();
  if (get == nullptr) return nullptr;
  const CUdeviceptr d = reinterpret_cast<CUdeviceptr>(a.devicePointer);
  CUdeviceptr start = 0;
  size_t size = 0;
  if (get(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, d) != CUDA_SUCCESS ||
      get(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, d) != CUDA_SUCCESS) {
    return nullptr;
  }
  if (d % align != 0 || d < start || d - start > size || bytes > size - (d - start)) return nullptr;
  return a.devicePointer;
}

// Posts `desc` in `slot`: the descriptor, then (release) its generation, into the mapped mailbox,
// which the kernel's dispatcher warp installs in the slot table. A slot's mailbox entry is rewritten
// only after its previous job was reported, so the dispatcher installed that one long before.
int Publish(cee_ctx* ctx, ServeState& s, int slot, const ServeJob& desc) {
  s.mailbox_host->desc[slot] = desc;
  std::atomic_thread_fence(std::memory_order_release);
  reinterpret_cast<volatile uint32_t*>(s.mailbox_host->posted)[slot] = desc.generation;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  ++s.stats.jobs;
  return LaunchServer(ctx, s);
}

// Clears a job record.
void ResetJob(ServeJobHost& job) { job = ServeJobHost{}; }

int NewJob(ServeState& s) {
  for (int i = 0; i < static_cast<int>(s.jobs.size()); ++i) {
    if (!s.jobs[i].live) return i;
  }
  s.jobs.emplace_back();
  return static_cast<int>(s.jobs.size()) - 1;
}

void ReleaseJob(ServeState& s, ServeJobHost& job) {
  for (const auto& [offset, bytes] : job.regions) s.arena.Free(offset, bytes);
  job.regions.clear();
  job.downloads.clear();
  if (job.slot >= 0) {
    s.tickets[job.slot].state.store(kTicketIdle, std::memory_order_release);
    s.slot_busy[job.slot] = false;
  }
  if (job.snapshot >= 0) {
    ServeSnapshotHost& snap = s.snapshots[job.snapshot];
    --snap.refs;
    if (snap.refs == 0 && snap.released && snap.live) {
      s.arena.Free(snap.offset, snap.bytes);
      snap.live = false;
    }
  }
  job.live = false;
  --s.pending;
}

// Fills the slot's ticket with the job's downloads and arms it (before the job is published, so the
// finished word of this generation cannot land before the ticket is armed).
int ArmDownloads(cee_ctx* ctx, ServeState& s, ServeJobHost& job) {
  SlotTicket& t = s.tickets[job.slot];
  if (static_cast<int>(job.downloads.size()) > kMaxDownloads) return ServeFail(ctx, CEE_ERR_INVALID, "too many outputs");
  if (t.event == nullptr) {
    const cudaError_t status = cudaEventCreateWithFlags(&t.event, cudaEventDisableTiming);
    if (status != cudaSuccess) return CudaFail(ctx, status, "serve download event");
  }
  t.generation = job.generation;
  t.count = static_cast<int>(job.downloads.size());
  for (int i = 0; i < t.count; ++i) {
    t.downloads[i] = job.downloads[static_cast<size_t>(i)];
    s.stats.download_bytes += t.downloads[i].bytes;
  }
  t.state.store(kTicketArmed, std::memory_order_release);
  {
    std::lock_guard<std::mutex> lock(s.wake_mutex);
    s.armed.fetch_add(1);
  }
  s.wake.notify_one();
  return CEE_OK;
}

// Issues the slot's downloads if its ticket is armed and no other thread got there first.
void IssueDownloads(ServeState& s, int slot) {
  SlotTicket& t = s.tickets[slot];
  int expected = kTicketArmed;
  if (!t.state.compare_exchange_strong(expected, kTicketIssuing, std::memory_order_acq_rel)) return;
  const uint8_t* arena = static_cast<const uint8_t*>(s.arena_buf.ptr);
  size_t bytes = 0;
  for (int i = 0; i < t.count; ++i) bytes += t.downloads[i].bytes;
  cudaStream_t st = bytes < kServeSmallDownload ? s.d2h_small : s.d2h;
  for (int i = 0; i < t.count; ++i) {
    cudaMemcpyAsync(t.downloads[i].host, arena + t.downloads[i].device_offset, t.downloads[i].bytes,
                    cudaMemcpyDeviceToHost, st);
  }
  cudaEventRecord(t.event, st);
  s.armed.fetch_sub(1);
  t.state.store(kTicketIssued, std::memory_order_release);
}

bool Finished(const ServeState& s, int slot, uint32_t generation) {
  return reinterpret_cast<const volatile uint32_t*>(s.finished_host)[slot] == generation;
}

void DownloaderLoop(ServeState* s, int device) {
  cudaSetDevice(device);
  while (!s->downloader_stop.load()) {
    if (s->armed.load() == 0) {
      std::unique_lock<std::mutex> lock(s->wake_mutex);
      s->wake.wait_for(lock, std::chrono::milliseconds(50),
                       [s] { return s->downloader_stop.load() || s->armed.load() > 0; });
      continue;
    }
    for (int slot = 0; slot < s->cfg.slots; ++slot) {
      SlotTicket& t = s->tickets[slot];
      if (t.state.load(std::memory_order_acquire) == kTicketArmed && Finished(*s, slot, t.generation)) {
        IssueDownloads(*s, slot);
      }
    }
    std::this_thread::yield();
  }
}

// The ticket of a job that will not finish (the loop broke): nothing is issued for it any more.
void DropTicket(ServeState& s, int slot) {
  SlotTicket& t = s.tickets[slot];
  int expected = kTicketArmed;
  if (t.state.compare_exchange_strong(expected, kTicketIdle, std::memory_order_acq_rel)) s.armed.fetch_sub(1);
  while (t.state.load(std::memory_order_acquire) == kTicketIssuing) std::this_thread::yield();
}

void StopDownloader(ServeState& s) {
  if (!s.downloader.joinable()) return;
  {
    std::lock_guard<std::mutex> lock(s.wake_mutex);
    s.downloader_stop.store(true);
  }
  s.wake.notify_one();
  s.downloader.join();
}

}  // namespace

void ReleaseServe(cee_ctx* ctx, int32_t* error_word) {
  if (error_word != nullptr) *error_word = 0;
  ServeState* s = ctx->serve;
  if (s == nullptr) return;
  if (s->control.ptr != nullptr) {
    const uint32_t one = 1;
    cudaMemcpy(&static_cast<ServeControl*>(s->control.ptr)->stop, &one, sizeof(one), cudaMemcpyHostToDevice);
  }
  StopDownloader(*s);
  if (s->server != nullptr) cudaStreamSynchronize(s->server);
  if (s->copy != nullptr) cudaStreamSynchronize(s->copy);
  if (s->d2h != nullptr) cudaStreamSynchronize(s->d2h);
  if (s->d2h_small != nullptr) cudaStreamSynchronize(s->d2h_small);
  if (error_word != nullptr && s->control.ptr != nullptr) {
    cudaMemcpy(error_word, &static_cast<ServeControl*>(s->control.ptr)->error, sizeof(int32_t), cudaMemcpyDeviceToHost);
  }
  for (SlotTicket& t : s->tickets) {
    if (t.event != nullptr) cudaEventDestroy(t.event);
  }
  s->arena_buf.Release();
  s->control.Release();
  s->templates.Release();
  if (s->finished_host != nullptr) cudaFreeHost(s->finished_host);
  if (s->mailbox_host != nullptr) cudaFreeHost(s->mailbox_host);
  if (s->words_host != nullptr) cudaFreeHost(s->words_host);
  if (s->pinned_stage != nullptr) cudaFreeHost(s->pinned_stage);
  for (cudaStream_t st : {s->server, s->copy, s->d2h, s->d2h_small}) {
    if (st != nullptr) cudaStreamDestroy(st);
  }
  if (s->kernel_done != nullptr) cudaEventDestroy(s->kernel_done);
  cudaGetLastError();
  delete s;
  ctx->serve = nullptr;
}

uint64_t ServeResident(const cee_ctx* ctx) {
  const ServeState* s = ctx->serve;
  return s == nullptr ? 0 : s->arena_buf.capacity + s->control.capacity + s->templates.capacity;
}

}  // namespace cee

using namespace cee;

extern "C" {

int cee_serve_start(cee_ctx* ctx, const cee_serve_config* config) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (config == nullptr || config->hbm_budget_bytes < (1 << 20) || config->slots < 1 ||
      config->slots > kServeMaxSlots || config->blocks_per_sm < 0 || config->idle_ms < 1) {
    return ServeFail(ctx, CEE_ERR_INVALID, "bad configuration");
  }
  if (ctx->serve != nullptr) ReleaseServe(ctx);
  ctx->serve = new ServeState();
  ServeState& s = *ctx->serve;
  s.cfg = *config;
  cudaError_t status = s.arena_buf.Reserve(static_cast<size_t>(config->hbm_budget_bytes), nullptr);
  if (status == cudaSuccess) status = s.control.Reserve(sizeof(ServeControl), nullptr);
  if (status == cudaSuccess) status = cudaMemset(s.control.ptr, 0, sizeof(ServeControl));
  if (status == cudaSuccess) status = s.templates.Reserve(kServeTemplateBytes + kServeValidityWords * 4, nullptr);
  if (status == cudaSuccess) {
    status = cudaHostAlloc(reinterpret_cast<void**>(&s.finished_host), (kServeLostWord + 1) * sizeof(uint32_t),
                           cudaHostAllocMapped);
  }
  if (status == cudaSuccess) status = cudaHostGetDevicePointer(reinterpret_cast<void**>(&s.finished_dev), s.finished_host, 0);
  if (status == cudaSuccess) {
    status = cudaHostAlloc(reinterpret_cast<void**>(&s.mailbox_host), sizeof(ServeMailbox), cudaHostAllocMapped);
  }
  if (status == cudaSuccess) status = cudaHostGetDevicePointer(reinterpret_cast<void**>(&s.mailbox_dev), s.mailbox_host, 0);
  if (status == cudaSuccess) {
    status = cudaHostAlloc(reinterpret_cast<void**>(&s.words_host), (kServeMaxSlots + 2) * sizeof(uint32_t),
                           cudaHostAllocDefault);
  }
  for (cudaStream_t* st : {&s.server, &s.copy, &s.d2h, &s.d2h_small}) {
    if (status == cudaSuccess) status = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking);
  }
  if (status == cudaSuccess) status = cudaEventCreateWithFlags(&s.kernel_done, cudaEventDisableTiming);
  int per_sm = 0;
  if (status == cudaSuccess) {
    status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_kernel, kServeWarps * 32, 0);
  }
  if (status != cudaSuccess) {
    const int code = CudaFail(ctx, status, "serve start");
    ReleaseServe(ctx);
    return code;
  }
  std::memset(s.finished_host, 0, (kServeLostWord + 1) * sizeof(uint32_t));
  std::memset(static_cast<void*>(s.mailbox_host), 0, sizeof(ServeMailbox));
  s.words_host[0] = 0;
  s.words_host[1] = 1;
  per_sm = std::max(1, config->blocks_per_sm > 0 ? std::min(per_sm, config->blocks_per_sm) : per_sm);
  s.grid = ctx->sm_count * per_sm;
  s.idle_limit = static_cast<long long>(config->idle_ms) * 500;  // ~2 us per idle scan
  s.arena.Reset(static_cast<size_t>(config->hbm_budget_bytes));
  // canonical template pair tables, k = 3, 4, 5 back to back
  std::vector<uint8_t> table(kServeTemplateBytes);
  for (uint32_t k = 3; k <= 5; ++k) {
    std::vector<uint8_t> mates(14 * 208, 0xff);
    const int count = cee_kopt_templates(k, mates.data(), nullptr);
    int at = serve_template_offset(static_cast<int>(k));
    for (int t = 0; t < count; ++t) {
      for (uint32_t p = 0; p < 2 * k; ++p) {
        const uint32_t q = mates[14 * t + p];
        if (p < q) table[at++] = static_cast<uint8_t>(kopt_pair_index(static_cast<int>(p), static_cast<int>(q), 2 * k));
      }
    }
  }
  // then the validity words of the proper templates by gap pattern, from the compile-time tables
  std::vector<uint32_t> valid(kServeValidityWords, 0);
  auto fill = [&](const auto& tab, int k) {
    const int words = (tab.count + 31) / 32;
    for (int g = 0; g < 32; ++g) {
      for (int t = 0; t < tab.count; ++t) {
        valid[serve_validity_offset(k) + g * words + t / 32] |= ((tab.invalid_on[t] >> g) & 1u) << (t % 32);
      }
    }
  };
  fill(KoptCanon<3>::value, 3);
  fill(KoptCanon<4>::value, 4);
  fill(KoptCanon<5>::value, 5);
  table.resize(kServeTemplateBytes + kServeValidityWords * 4);
  std::memcpy(table.data() + kServeTemplateBytes, valid.data(), valid.size() * 4);
  status = cudaMemcpy(s.templates.ptr, table.data(), table.size(), cudaMemcpyHostToDevice);
  if (status != cudaSuccess) {
    const int code = CudaFail(ctx, status, "serve templates");
    ReleaseServe(ctx);
    return code;
  }
  s.downloader = std::thread(DownloaderLoop, &s, ctx->device);
  return CEE_OK;
}

int cee_serve_add_snapshot(cee_ctx* ctx, const cee_graph_view* g, int32_t* snapshot) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  ServeState* sp = Serving(ctx);
  if (sp == nullptr) return ServeFail(ctx, CEE_ERR_STATE, "not started");
  ServeState& s = *sp;
  if (g == nullptr || snapshot == nullptr) return ServeFail(ctx, CEE_ERR_INVALID, "null argument");
  if (g->n <= 0 || g->m < 0 || g->m > INT32_MAX || (g->dist_type != CEE_EUC_2D && g->dist_type != CEE_CEIL_2D)) {
    return ServeFail(ctx, CEE_ERR_INVALID, "bad snapshot");
  }
  if (g->m > 0) {
    if (g->adjacency < 0 || g->adjacency > INT32_MAX || g->row_offsets == nullptr || g->row_offsets[0] != 0 ||
        g->row_offsets[g->n] != g->adjacency) {
      return ServeFail(ctx, CEE_ERR_INVALID, "bad CSR");
    }
    for (int32_t v = 0; v < g->n; ++v) {
      if (g->row_offsets[v + 1] < g->row_offsets[v]) return ServeFail(ctx, CEE_ERR_INVALID, "bad CSR row offsets");
    }
    for (int64_t i = 0; i < g->adjacency; ++i) {
      if (g->neighbors[i] < 0 || g->neighbors[i] >= g->n || g->csr_edge_ids[i] < 0 || g->csr_edge_ids[i] >= g->m) {
        return ServeFail(ctx, CEE_ERR_INVALID, "CSR index out of range");
      }
    }
  }
  std::vector<int2> xy;
  int span = kSpanSmall;
  rc = PackCoordinates(ctx, g->n, g->x, g->y, &xy, &span);
  if (rc != CEE_OK) return rc;
  const size_t n = static_cast<size_t>(g->n), m = static_cast<size_t>(g->m);
  const size_t adj = g->m > 0 ? static_cast<size_t>(g->adjacency) : 0;
  auto up = [](size_t b) { return (b + 15) & ~size_t{15}; };
  const size_t o_xy = 0, o_uv = up(o_xy + 8 * n), o_w = up(o_uv + 8 * m), o_act = up(o_w + 4 * m);
  // CSR slots twice: neighbours alone (binary searches of a row) and 16-byte records {neighbour,
  // slot weight, neighbour x, neighbour y} (one load per slot in the JV screen)
  const size_t o_ro = up(o_act + m), o_nbr = up(o_ro + 4 * (n + 1)), o_slot4 = up(o_nbr + 4 * adj);
  const size_t bytes = up(o_slot4 + 16 * adj);
  size_t offset = 0;
  if (!s.arena.Allocate(bytes, &offset)) return CEE_BUSY;  // over the HBM budget now
  rc = EnsurePinned(ctx, s, bytes);
  if (rc != CEE_OK) {
    s.arena.Free(offset, bytes);
    return rc;
  }
  uint8_t* st = s.pinned_stage;
  std::memcpy(st + o_xy, xy.data(), 8 * n);
  int2* uv = reinterpret_cast<int2*>(st + o_uv);
  int32_t* w32 = reinterpret_cast<int32_t*>(st + o_w);
  for (size_t e = 0; e < m; ++e) {
    if (g->edge_u[e] < 0 || g->edge_u[e] >= g->n || g->edge_v[e] < 0 || g->edge_v[e] >= g->n) {
      s.arena.Free(offset, bytes);
      return ServeFail(ctx, CEE_ERR_INVALID, "edge endpoint out of range");
    }
    if (g->edge_w[e] < 0 || g->edge_w[e] > INT32_MAX) {
      s.arena.Free(offset, bytes);
      return ServeFail(ctx, CEE_ERR_RANGE, "edge weight outside [0, 2^31)");
    }
    uv[e] = make_int2(g->edge_u[e], g->edge_v[e]);
    w32[e] = static_cast<int32_t>(g->edge_w[e]);
  }
  if (m > 0) std::memcpy(st + o_act, g->active, m);
  int32_t* ro = reinterpret_cast<int32_t*>(st + o_ro);
  if (g->m > 0) {
    std::memcpy(ro, g->row_offsets, 4 * (n + 1));
  } else {
    std::memset(ro, 0, 4 * (n + 1));
  }
  if (adj > 0) {
    std::memcpy(st + o_nbr, g->neighbors, 4 * adj);
    int4* slot4 = reinterpret_cast<int4*>(st + o_slot4);
    for (size_t i = 0; i < adj; ++i) {
      const int32_t c = g->neighbors[i];
      slot4[i] = make_int4(c, w32[g->csr_edge_ids[i]], xy[static_cast<size_t>(c)].x, xy[static_cast<size_t>(c)].y);
    }
  }
  uint8_t* base = static_cast<uint8_t*>(s.arena_buf.ptr) + offset;
  rc = QuiesceServer(ctx, s);
  if (rc != CEE_OK) {
    s.arena.Free(offset, bytes);
    return rc;
  }
  cudaMemcpyAsync(base, st, bytes, cudaMemcpyHostToDevice, s.copy);
  const cudaError_t status = cudaStreamSynchronize(s.copy);  // the staging buffer is reused
  if (status != cudaSuccess) {
    s.arena.Free(offset, bytes);
    return CudaFail(ctx, status, "serve snapshot upload");
  }
  int id = -1;
  for (int i = 0; i < static_cast<int>(s.snapshots.size()); ++i) {
    if (!s.snapshots[i].live && s.snapshots[i].refs == 0) {
      id = i;
      break;
    }
  }
  if (id < 0) {
    s.snapshots.emplace_back();
    id = static_cast<int>(s.snapshots.size()) - 1;
  }
  ServeSnapshotHost& snap = s.snapshots[id];
  snap = ServeSnapshotHost{};
  snap.live = true;
  snap.offset = offset;
  snap.bytes = bytes;
  snap.n = g->n;
  snap.m = g->m;
  snap.adj = static_cast<int64_t>(adj);
  snap.dist_type = g->dist_type;
  snap.span = span;
  snap.g.n = g->n;
  snap.g.dist_type = g->dist_type;
  snap.g.m = g->m;
  snap.g.xy = reinterpret_cast<const int2*>(base + o_xy);
  snap.g.edge_uv = reinterpret_cast<const int2*>(base + o_uv);
  snap.g.edge_w = reinterpret_cast<const int32_t*>(base + o_w);
  snap.g.active = base + o_act;
  snap.g.row_offsets = reinterpret_cast<const int32_t*>(base + o_ro);
  snap.g.nbr = reinterpret_cast<const int32_t*>(base + o_nbr);
  snap.g.slot_w = nullptr;
  snap.g.slot4 = reinterpret_cast<const int4*>(base + o_slot4);
  *snapshot = id;
  return CEE_OK;
}

int cee_serve_release_snapshot(cee_ctx* ctx, int32_t snapshot) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  ServeState* s = Serving(ctx);
  if (s == nullptr) return ServeFail(ctx, CEE_ERR_STATE, "not started");
  if (snapshot < 0 || snapshot >= static_cast<int>(s->snapshots.size()) || !s->snapshots[snapshot].live) {
    return ServeFail(ctx, CEE_ERR_INVALID, "unknown snapshot");
  }
  ServeSnapshotHost& snap = s->snapshots[snapshot];
  snap.released = true;
  if (snap.refs == 0) {
    s->arena.Free(snap.offset, snap.bytes);
    snap.live = false;
  }
  return CEE_OK;
}

int cee_serve_submit_jv(cee_ctx* ctx, int32_t snapshot, int32_t* witness_out, uint64_t tag, int32_t* job_out) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  ServeState* sp = Serving(ctx);
  if (sp == nullptr) return ServeFail(ctx, CEE_ERR_STATE, "not started");
  ServeState& s = *sp;
  if (s.broken) return ServeFail(ctx, CEE_ERR_TIMEOUT, "loop lost a work item; restart it");
  if (snapshot < 0 || snapshot >= static_cast<int>(s.snapshots.size()) || !s.snapshots[snapshot].live || job_out == nullptr ||
      (s.snapshots[snapshot].m > 0 && witness_out == nullptr)) {
    return ServeFail(ctx, CEE_ERR_INVALID, "bad JV job");
  }
  ServeSnapshotHost& snap = s.snapshots[snapshot];
  const int id = NewJob(s);
  ServeJobHost& job = s.jobs[id];
  ResetJob(job);
  job.tag = tag;
  if (snap.m == 0) {  // nothing to screen
    job.live = true;
    job.phase = 2;
    job.snapshot = snapshot;
    ++snap.refs;
    ++s.pending;
    s.finished_jobs.push_back(id);
    *job_out = id;
    return CEE_OK;
  }
  const int slot = FreeSlot(s);
  if (slot < 0) return CEE_BUSY;  // every slot holds a job
  size_t out = 0;
  const size_t out_bytes = static_cast<size_t>(snap.m) * 4;
  // a page-locked witness array is written by the kernel in place: no arena room, no download
  void* direct = MappedRange(witness_out, out_bytes, 4);
  if (direct == nullptr && !s.arena.Allocate(out_bytes, &out)) return CEE_BUSY;
  ServeJob desc{};
  desc.generation = s.next_generation++;
  desc.type = kServeJv;
  desc.span = snap.span;
  desc.g = snap.g;
  desc.witness = direct != nullptr ? static_cast<int32_t*>(direct)
                                   : reinterpret_cast<int32_t*>(static_cast<uint8_t*>(s.arena_buf.ptr) + out);
  desc.host_outputs = direct != nullptr ? 1u : 0u;
  desc.items = static_cast<uint32_t>((snap.m + kServeJvTile - 1) / kServeJvTile);
  s.slot_busy[slot] = true;
  s.next_slot = (slot + 1) % s.cfg.slots;
  job.live = true;
  job.slot = slot;
  job.generation = desc.generation;
  job.snapshot = snapshot;
  job.direct = direct != nullptr;
  ++snap.refs;
  ++s.pending;
  *job_out = id;
  if (job.direct) {
    s.stats.direct_bytes += out_bytes;
  } else {
    job.regions.push_back({out, out_bytes});
    job.downloads.push_back({witness_out, out, out_bytes});
    rc = ArmDownloads(ctx, s, job);
    if (rc != CEE_OK) {
      ReleaseJob(s, job);
      return rc;
    }
  }
  return Publish(ctx, s, slot, desc);
}

}  // extern "C"

namespace cee {
namespace {

// A k-opt job of 1..3 segments: the cost matrices (costs_out, or null for none), and with
// masks_out / first_out the improving-template sets (cee_kopt_improving_multi's outputs).
int SubmitKopt(cee_ctx* ctx, int32_t snapshot, int32_t segments, const uint32_t* ks, const cee_kopt_task* const* tasks,
               const int64_t* rows, int64_t* const* costs_out, uint32_t* const* masks_out, int32_t* const* first_out,
               uint64_t tag, int32_t* job_out) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  ServeState* sp = Serving(ctx);
  if (sp == nullptr) return ServeFail(ctx, CEE_ERR_STATE, "not started");
  ServeState& s = *sp;
  if (s.broken) return ServeFail(ctx, CEE_ERR_TIMEOUT, "loop lost a work item; restart it");
  const bool sets = masks_out != nullptr;
  if (snapshot < 0 || snapshot >= static_cast<int>(s.snapshots.size()) || !s.snapshots[snapshot].live ||
      segments < 1 || segments > 3 || ks == nullptr || tasks == nullptr || rows == nullptr ||
      (costs_out == nullptr && !sets) || (sets && first_out == nullptr) || job_out == nullptr) {
    return ServeFail(ctx, CEE_ERR_INVALID, "bad k-opt job");
  }
  ServeSnapshotHost& snap = s.snapshots[snapshot];
  auto words = [](uint32_t k) { return (TemplateCount(static_cast<int>(k)) + 31) / 32; };
  auto rounded = [](size_t bytes) { return (bytes + 255) & ~size_t{255}; };
  size_t in_bytes = 0, out_bytes = 0;
  int64_t items = 0;
  for (int i = 0; i < segments; ++i) {
    if (ks[i] < 3 || ks[i] > 5 || rows[i] < 0 ||
        (rows[i] > 0 && (tasks[i] == nullptr || (costs_out != nullptr && costs_out[i] == nullptr) ||
                         (sets && (masks_out[i] == nullptr || first_out[i] == nullptr))))) {
      return ServeFail(ctx, CEE_ERR_INVALID, "bad k-opt segment");
    }
    const size_t r = static_cast<size_t>(rows[i]);
    in_bytes += rounded(r * sizeof(cee_kopt_task));
    if (costs_out != nullptr) out_bytes += rounded(r * TemplateCount(ks[i]) * 8);
    if (sets) out_bytes += rounded(r * words(ks[i]) * 4) + rounded(r * 4);
    items += (rows[i] + kServeKoptRowsPerItem - 1) / kServeKoptRowsPerItem;
  }
  const int id = NewJob(s);
  ServeJobHost& job = s.jobs[id];
  ResetJob(job);
  job.tag = tag;
  if (items == 0) {
    job.live = true;
    job.phase = 2;
    job.snapshot = snapshot;
    ++snap.refs;
    ++s.pending;
    s.finished_jobs.push_back(id);
    *job_out = id;
    return CEE_OK;
  }
  const int slot = FreeSlot(s);
  if (slot < 0) return CEE_BUSY;
  size_t in = 0, out = 0;
  if (!s.arena.Allocate(in_bytes, &in)) return CEE_BUSY;
  if (!s.arena.Allocate(out_bytes, &out)) {
    s.arena.Free(in, in_bytes);
    return CEE_BUSY;
  }
  ServeJob desc{};
  desc.generation = s.next_generation++;
  desc.type = kServeKopt;
  desc.span = snap.span;
  desc.g = snap.g;
  desc.segments = segments;
  uint8_t* arena = static_cast<uint8_t*>(s.arena_buf.ptr);
  size_t in_at = in, out_at = out;
  int64_t item_at = 0;
  for (int i = 0; i < segments; ++i) {
    ServeSegment& seg = desc.seg[i];
    const size_t r = static_cast<size_t>(rows[i]);
    seg.rows = rows[i];
    seg.k = static_cast<int32_t>(ks[i]);
    seg.T = TemplateCount(seg.k);
    seg.item_begin = item_at;
    seg.tasks = reinterpret_cast<const int32_t*>(arena + in_at);
    if (rows[i] > 0) {
      cudaMemcpyAsync(arena + in_at, tasks[i], r * sizeof(cee_kopt_task), cudaMemcpyHostToDevice, s.copy);
      s.stats.rows_bytes += r * sizeof(cee_kopt_task);
    }
    in_at += rounded(r * sizeof(cee_kopt_task));
    if (costs_out != nullptr) {
      seg.costs = reinterpret_cast<int64_t*>(arena + out_at);
      if (rows[i] > 0) job.downloads.push_back({costs_out[i], out_at, r * seg.T * 8});
      out_at += rounded(r * seg.T * 8);
    }
    if (sets) {
      seg.improving = reinterpret_cast<uint32_t*>(arena + out_at);
      if (rows[i] > 0) job.downloads.push_back({masks_out[i], out_at, r * words(ks[i]) * 4});
      out_at += rounded(r * words(ks[i]) * 4);
      seg.first = reinterpret_cast<int32_t*>(arena + out_at);
      if (rows[i] > 0) job.downloads.push_back({first_out[i], out_at, r * 4});
      out_at += rounded(r * 4);
    }
    item_at += (rows[i] + kServeKoptRowsPerItem - 1) / kServeKoptRowsPerItem;
  }
  desc.items = static_cast<uint32_t>(items);
  desc.rows_gate = 1;
  // after the rows: the slot's rows-ready word = generation (the dispatcher installs the job then)
  s.words_host[2 + slot] = desc.generation;
  cudaMemcpyAsync(&static_cast<ServeControl*>(s.control.ptr)->rows_ready[slot], &s.words_host[2 + slot],
                  sizeof(uint32_t), cudaMemcpyHostToDevice, s.copy);
  s.slot_busy[slot] = true;
  s.next_slot = (slot + 1) % s.cfg.slots;
  job.live = true;
  job.slot = slot;
  job.generation = desc.generation;
  job.snapshot = snapshot;
  job.regions.push_back({in, in_bytes});
  job.regions.push_back({out, out_bytes});
  ++snap.refs;
  ++s.pending;
  *job_out = id;
  rc = ArmDownloads(ctx, s, job);
  if (rc != CEE_OK) {
    ReleaseJob(s, job);
    return rc;
  }
  return Publish(ctx, s, slot, desc);
}

}  // namespace
}  // namespace cee

extern "C" {

int cee_serve_submit_kopt(cee_ctx* ctx, int32_t snapshot, int32_t segments, const uint32_t* ks,
                          const cee_kopt_task* const* tasks, const int64_t* rows, int64_t* const* costs_out,
                          uint64_t tag, int32_t* job_out) {
  if (costs_out == nullptr) return ServeFail(ctx, CEE_ERR_INVALID, "bad k-opt job");
  return SubmitKopt(ctx, snapshot, segments, ks, tasks, rows, costs_out, nullptr, nullptr, tag, job_out);
}

int cee_serve_submit_kopt_improving(cee_ctx* ctx, int32_t snapshot, int32_t segments, const uint32_t* ks,
                                    const cee_kopt_task* const* tasks, const int64_t* rows,
                                    uint32_t* const* masks_out, int32_t* const* first_out, int64_t* const* costs_out,
                                    uint64_t tag, int32_t* job_out) {
  if (masks_out == nullptr || first_out == nullptr) return ServeFail(ctx, CEE_ERR_INVALID, "null improving-set outputs");
  return SubmitKopt(ctx, snapshot, segments, ks, tasks, rows, costs_out, masks_out, first_out, tag, job_out);
}

int cee_serve_poll(cee_ctx* ctx, cee_serve_event* events, int32_t capacity, int32_t* count) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  ServeState* sp = Serving(ctx);
  if (sp == nullptr || count == nullptr) return ServeFail(ctx, CEE_ERR_STATE, "not started");
  ServeState& s = *sp;
  *count = 0;
  auto report = [&](int id, ServeJobHost& job) {
    if (*count < capacity && events != nullptr) {
      events[*count].job = id;
      events[*count].status = job.status;
      events[*count].tag = job.tag;
      ++*count;
      ReleaseJob(s, job);
      return true;
    }
    return false;
  };
  while (!s.finished_jobs.empty() && *count < capacity) {
    const int id = s.finished_jobs.back();
    s.finished_jobs.pop_back();
    report(id, s.jobs[id]);
  }
  if (!s.broken && reinterpret_cast<volatile uint32_t*>(s.finished_host)[kServeLostWord] != 0) {
    // a claimed item's descriptor never became visible: that job cannot finish. Stop the kernel
    // and fail every job still on the GPU; the loop must be restarted.
    rc = QuiesceServer(ctx, s);
    if (rc != CEE_OK) return rc;
    s.broken = true;
  }
  bool on_gpu = false;
  for (int id = 0; id < static_cast<int>(s.jobs.size()); ++id) {
    ServeJobHost& job = s.jobs[id];
    if (!job.live || job.phase == 2) continue;
    if (job.phase == 0 && s.broken &&
        *reinterpret_cast<volatile uint32_t*>(s.finished_host + job.slot) != job.generation) {
      DropTicket(s, job.slot);
      job.status = Fail(ctx, CEE_ERR_TIMEOUT, "serving loop lost a work item; restart it with cee_serve_start");
      if (!report(id, job)) break;
      continue;
    }
    if (job.phase == 0) {
      if (*reinterpret_cast<volatile uint32_t*>(s.finished_host + job.slot) != job.generation) {
        on_gpu = true;
        continue;
      }
      if (reinterpret_cast<volatile uint32_t*>(s.finished_host)[kServeMaxSlots + job.slot] != 0) {
        job.status = Fail(ctx, CEE_ERR_INVALID, "serving loop: device bounds check rejected an out-of-range index");
      }
      if (job.direct) {  // the outputs are in place (the kernel fenced them before the finished word)
        std::atomic_thread_fence(std::memory_order_acquire);
        if (!report(id, job)) break;
        continue;
      }
      IssueDownloads(s, job.slot);  // unless the downloader thread already has
      int state = kTicketIssuing;
      while ((state = s.tickets[job.slot].state.load(std::memory_order_acquire)) == kTicketIssuing) {
        std::this_thread::yield();
      }
      if (state != kTicketIssued) return ServeFail(ctx, CEE_ERR_STATE, "a finished job's downloads were not queued");
      job.phase = 1;
    }
    const cudaError_t q = cudaEventQuery(s.tickets[job.slot].event);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return CudaFail(ctx, q, "serve download");
    if (!report(id, job)) break;
  }
  if (on_gpu && !s.broken) {  // the kernel may have gone idle before a late publication: relaunch if it ended
    rc = LaunchServer(ctx, s);
    if (rc != CEE_OK) return rc;
  }
  return CEE_OK;
}

int cee_serve_stop(cee_ctx* ctx) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (ctx->serve == nullptr) return CEE_OK;
  int32_t error_word = 0;
  ReleaseServe(ctx, &error_word);
  if (error_word != 0) {
    return Fail(ctx, CEE_ERR_INVALID, "serving loop: a claimed work item's job never became visible (code " +
                                          std::to_string(error_word) + ")");
  }
  return CEE_OK;
}

int cee_serve_get_stats(const cee_ctx* ctx, cee_serve_stats* stats) {
  if (ctx == nullptr || stats == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null argument");
  *stats = ctx->serve == nullptr ? cee_serve_stats{} : ctx->serve->stats;
  return CEE_OK;
}

int cee_serve_pending(const cee_ctx* ctx, int32_t* jobs, uint64_t* arena_used) {
  if (ctx == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null context");
  const ServeState* s = ctx->serve;
  if (jobs != nullptr) *jobs = s == nullptr ? 0 : s->pending;
  if (arena_used != nullptr) *arena_used = s == nullptr ? 0 : s->arena.used();
  return CEE_OK;
}

}  // extern "C"
