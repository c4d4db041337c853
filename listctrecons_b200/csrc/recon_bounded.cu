// Whole-scan runs with a bounded device footprint, and runs straight from the reference's raw
// files.
//
// The reference bounds device memory per 32-slice block: it reads each block's window of fan
// views from the raw file (Src/DataReader.cpp:8-19, an `int`-sized offset), rebins, filters and
// backprojects it, and moves on (Src/Reconstructor.cpp:33-48) -- every view is read, rebinned and
// filtered about three times, once per block whose window holds it.  A bounded recon keeps the
// scan-mode property (each view uploaded, rebinned and filtered once) with memory that does not
// grow with the scan:
//   fan    a ring of fan views: the upload of a piece overwrites only views whose rebins are done
//   par    one piece of rebinned, filtered views (the backprojector reads the quads)
//   quads  a ring holding the windows of the slabs in flight (quad views, or the slots of the
//          3-D texture the TEX8 backprojector samples): a piece is packed only after every slab
//          whose window held the slots it overwrites is backprojected
//   img    a ring of four slabs for volumes written to host memory or a file (a device volume is
//          written in place)
// Slabs are taken in the order their windows end and backprojected on two alternating streams,
// the first in parts while its window arrives, exactly as the streamed unbounded run does; the
// kernels and their order per view are the same, so the volume is bit-identical to it.
//
// lct_recon_run_file reads the fan from the reference's raw file with 64-bit offsets on reader
// threads into small pinned chunks that are uploaded as the pipeline needs them, and writes the
// volume through slab writer threads (64-bit offsets) -- RawDataReader::readData and RawImageWriter
// (Src/ImageWriter.cpp:9-43) for whole scans.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstring>
#include <condition_variable>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "lct_internal.h"

namespace lct {
const float* plan_angles(const lct_plan* p);
}  // namespace lct

#include "recon_internal.h"

namespace lct {

int pinned_alloc(size_t bytes, PinnedBuf& b) {
  constexpr size_t kHuge = 2u << 20;
  const size_t len = (bytes + kHuge - 1) / kHuge * kHuge;
  void* m = ::mmap(nullptr, len + kHuge, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
  if (m != MAP_FAILED) {
    char* p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(m) + kHuge - 1) & ~(uintptr_t)(kHuge - 1));
    ::madvise(p, len, MADV_HUGEPAGE);  // a request: 4 KiB pages if refused
    for (size_t o = 0; o < len; o += kHuge) p[o] = 0;
    if (cudaHostRegister(p, len, cudaHostRegisterDefault) == cudaSuccess) {
      b.p = reinterpret_cast<float*>(p);
      b.map = m;
      b.map_bytes = len + kHuge;
      return LCT_OK;
    }
    cudaGetLastError();
    ::munmap(m, len + kHuge);
  }
  void* h = nullptr;
  if (cudaHostAlloc(&h, bytes, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return LCT_ERR_ALLOC;
  }
  b.p = static_cast<float*>(h);
  b.map = nullptr;
  b.map_bytes = 0;
  return LCT_OK;
}

void pinned_free(PinnedBuf& b) {
  if (!b.p) return;
  if (b.map) {
    cudaHostUnregister(b.p);
    ::munmap(b.map, b.map_bytes);
  } else {
    cudaFreeHost(b.p);
  }
  b = PinnedBuf{};
}

static double wall_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr long long kDefaultPiece = 512;  // views per rebin / filter / pack step
constexpr int kImgRing = 4;               // slabs in the volume ring (host / file output)
constexpr int kFanStage = 8;              // pinned fan chunks of lct_recon_run_file
constexpr long long kFanChunkBytes = 16LL << 20;  // a chunk: whole views, at most 16 MiB (>= 1 view)
constexpr int kFanReaders = 4;            // reader threads (chunk c on thread c mod 4)
static_assert(kFanStage % kFanReaders == 0, "slot s must belong to reader s mod kFanReaders");
constexpr int kImgStage = 4;              // pinned slabs of the slab writer
constexpr int kSinkThreads = 4;           // slab writer threads (file writes, pageable copies:
                                          // first-touch page faults of a fresh host volume
                                          // spread over the threads)

// Fan views a global parallel view g reads lie in [g + lo, g + hi] (scan rebin shifts, FP64).
static void rebin_reach(const lct_geom& g, long long& lo, long long& hi) {
  const double s0 = ((0.0 - (double)g.ws) * (double)g.ds / (double)g.dso) / (double)g.orbit;
  const double s1 = (((double)(g.ns - 1) - (double)g.ws) * (double)g.ds / (double)g.dso) /
                    (double)g.orbit;
  lo = (long long)std::floor(std::min(s0, s1));
  hi = (long long)std::floor(std::max(s0, s1)) + 1;
}

// ----------------------------------------------------------------------------------------------
// reader: file views -> pinned chunks (kFanReaders threads), chunks -> device (the issuing thread)
// ----------------------------------------------------------------------------------------------
class FanReader {
 public:
  // views [0, nviews) of the run lie at byte0 + v * view_bytes of the file; slots: one pinned
  // buffer of `chunk` views per slot (null ones are pinned by their reader thread before its
  // first read into them; slot s is filled only by thread s mod kFanReaders); device: the
  // caller's CUDA device
  int start(const char* path, long long byte0, long long view_bytes, long long nviews,
            long long chunk, std::vector<PinnedBuf>* slots, int device) {
    fd_ = ::open(path, O_RDONLY);
    if (fd_ < 0) return LCT_ERR_IO;
    struct stat sb;
    if (fstat(fd_, &sb) != 0 || (long long)sb.st_size < byte0 + nviews * view_bytes) {
      ::close(fd_);
      fd_ = -1;
      return LCT_ERR_IO;  // the file ends before the run's last view
    }
    byte0_ = byte0;
    view_bytes_ = view_bytes;
    nviews_ = nviews;
    chunk_ = chunk;
    stage_ = slots;
    slots_ = (int)slots->size();
    device_ = device;
    state_.assign(slots_, kFree);
    held_.resize(slots_);
    for (int i = 0; i < slots_; ++i) held_[i] = i - slots_;  // "chunk i - slots" done: free for chunk i
    rel_.resize(slots_);
    for (int i = 0; i < slots_; ++i) rel_[i] = {this, i};
    for (int t = 0; t < kFanReaders; ++t) th_.emplace_back([this, t] { loop(t); });
    return LCT_OK;
  }
  long long chunks() const { return (nviews_ + chunk_ - 1) / chunk_; }
  long long chunk() const { return chunk_; }
  double read_seconds() const { return (double)read_ns_.load() * 1e-9; }
  double wait_seconds() const { return wait_s_; }
  // blocks until chunk c is in its pinned slot
  int acquire(long long c, const float** data, long long* nv) {
    const int slot = (int)(c % slots_);
    const double t0 = wall_seconds();
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return err_ || (state_[slot] == kReady && held_[slot] == c); });
    wait_s_ += wall_seconds() - t0;
    if (err_) return err_;
    *data = (*stage_)[slot].p;  // written by its reader before the slot was marked ready
    *nv = std::min(chunk_, nviews_ - c * chunk_);
    return LCT_OK;
  }
  // the slot of chunk c is free again once the work queued on s so far (its upload) is done
  int release_after(cudaStream_t s, long long c) {
    const int slot = (int)(c % slots_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      state_[slot] = kUploading;
    }
    return cuda_status(cudaLaunchHostFunc(s, &FanReader::on_uploaded, &rel_[slot]));
  }
  // stops the thread (every queued upload must have completed); the first error, if any
  int finish() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_)
      if (t.joinable()) t.join();
    th_.clear();
    if (fd_ >= 0) ::close(fd_);
    fd_ = -1;
    return err_;
  }

 private:
  enum { kFree = 0, kReading = 1, kReady = 2, kUploading = 3 };
  struct Rel {
    FanReader* self;
    int slot;
  };
  static void CUDART_CB on_uploaded(void* p) {  // a CUDA host function: no CUDA calls here
    Rel* r = static_cast<Rel*>(p);
    {
      std::lock_guard<std::mutex> lk(r->self->mu_);
      r->self->state_[r->slot] = kFree;
    }
    r->self->cv_.notify_all();
  }
  // reader thread t: chunks t, t + kFanReaders, ...; chunk c waits for its slot (c mod slots)
  // to be free, i.e. for chunk c - slots to be uploaded
  void loop(int t) {
    if (cudaSetDevice(device_) != cudaSuccess) {
      fail(LCT_ERR_CUDA);
      return;
    }
    for (long long c = t; c < chunks(); c += kFanReaders) {
      const int slot = (int)(c % slots_);
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] {
          return stop_ || err_ || (state_[slot] == kFree && held_[slot] == c - slots_);
        });
        if (stop_ || err_) return;
        state_[slot] = kReading;
      }
      PinnedBuf& buf = (*stage_)[slot];  // this thread's slot: no other thread writes it
      if (!buf.p && pinned_alloc((size_t)(chunk_ * view_bytes_), buf) != LCT_OK) {
        fail(LCT_ERR_ALLOC);
        return;
      }
      const double t0 = wall_seconds();
      const long long nv = std::min(chunk_, nviews_ - c * chunk_);
      char* dst = reinterpret_cast<char*>(buf.p);
      long long left = nv * view_bytes_, off = byte0_ + c * chunk_ * view_bytes_;
      int e = LCT_OK;
      while (left > 0) {
        const ssize_t n = ::pread(fd_, dst, (size_t)std::min<long long>(left, 1LL << 30), (off_t)off);
        if (n < 0 && errno == EINTR) continue;
        if (n <= 0) {
          e = LCT_ERR_IO;
          break;
        }
        dst += n;
        off += n;
        left -= n;
      }
      read_ns_ += (long long)((wall_seconds() - t0) * 1e9);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (e) err_ = e;
        held_[slot] = c;
        state_[slot] = kReady;
      }
      cv_.notify_all();
      if (e) return;
    }
  }
  void fail(int e) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (!err_) err_ = e;
    }
    cv_.notify_all();
  }
  int fd_ = -1;
  long long byte0_ = 0, view_bytes_ = 0, nviews_ = 0, chunk_ = 1;
  std::atomic<long long> read_ns_{0};  // time in reads, summed over the threads
  double wait_s_ = 0.0;                // the pipeline's waits in acquire (its thread only)
  std::vector<PinnedBuf>* stage_ = nullptr;
  int slots_ = 0, device_ = 0;
  std::vector<int> state_;
  std::vector<long long> held_;
  std::vector<Rel> rel_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool stop_ = false;
  int err_ = LCT_OK;
};

// ----------------------------------------------------------------------------------------------
// writer: device slab -> pinned slot (D2H on the download stream) -> file and/or pageable host
// volume (four threads)
// ----------------------------------------------------------------------------------------------
class SlabWriter {
 public:
  // path (or null): the volume file, sized and written slab by slab; host (or null): a pageable
  // host volume the slabs are copied into (a download straight into pageable memory would hold
  // the issuing thread until the slab is backprojected, stalling the whole pipeline)
  // slots: one pinned buffer of a slab per slot; null ones are pinned in order by the first
  // writer thread while the first slabs are computed.  device: the caller's CUDA device.
  int start(const char* path, float* host, long long slab_bytes, int nslabs,
            std::vector<PinnedBuf>* slots, int device) {
    if (path) {
      fd_ = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
      if (fd_ < 0) return LCT_ERR_IO;
      if (::ftruncate(fd_, (off_t)(slab_bytes * nslabs)) != 0) {
        ::close(fd_);
        fd_ = -1;
        return LCT_ERR_IO;
      }
    }
    host_ = reinterpret_cast<char*>(host);
    slab_bytes_ = slab_bytes;
    stage_ = slots;
    slots_ = (int)slots->size();
    device_ = device;
    busy_.assign(slots_, 0);
    dest_.assign(slots_, -1);
    have_.assign(slots_, 0);
    for (int i = 0; i < slots_; ++i) have_[i] = (*slots)[i].p != nullptr;
    sub_.resize(slots_);
    for (int i = 0; i < slots_; ++i) sub_[i] = {this, i};
    for (int t = 0; t < kSinkThreads; ++t) th_.emplace_back([this, t] { loop(t); });
    return LCT_OK;
  }
  // pinned slot for the k-th slab written (blocks while its previous slab is being written)
  int slot_for(int k, float** p) {
    const int slot = k % slots_;
    const double t0 = wall_seconds();
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return err_ || (have_[slot] && !busy_[slot]); });
    wait_s_ += wall_seconds() - t0;
    if (err_) return err_;
    busy_[slot] = 1;
    *p = (*stage_)[slot].p;
    return LCT_OK;
  }
  // once the work queued on s (the slab's download into slot k % slots) is done, write it as
  // slab `dest` of the file
  int submit_after(cudaStream_t s, int k, int dest) {
    const int slot = k % slots_;
    {
      std::lock_guard<std::mutex> lk(mu_);
      dest_[slot] = dest;
    }
    return cuda_status(cudaLaunchHostFunc(s, &SlabWriter::on_downloaded, &sub_[slot]));
  }
  double wait_seconds() const { return wait_s_; }
  int finish() {
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] {
        if (err_) return true;
        for (int b : busy_)
          if (b) return false;
        return true;
      });
      stop_ = true;
    }
    cv_.notify_all();
    for (std::thread& t : th_)
      if (t.joinable()) t.join();
    th_.clear();
    if (fd_ >= 0 && ::close(fd_) != 0 && !err_) err_ = LCT_ERR_IO;
    fd_ = -1;
    return err_;
  }

 private:
  struct Sub {
    SlabWriter* self;
    int slot;
  };
  static void CUDART_CB on_downloaded(void* p) {  // a CUDA host function: no CUDA calls here
    Sub* s = static_cast<Sub*>(p);
    {
      std::lock_guard<std::mutex> lk(s->self->mu_);
      s->self->ready_.push_back(s->slot);
    }
    s->self->cv_.notify_all();
  }
  void loop(int t) {
    if (cudaSetDevice(device_) != cudaSuccess) return fail(LCT_ERR_CUDA);
    if (t == 0) {
      for (int i = 0; i < slots_; ++i) {
        PinnedBuf b;
        {
          std::lock_guard<std::mutex> lk(mu_);
          if (have_[i]) continue;
        }
        if (pinned_alloc((size_t)slab_bytes_, b) != LCT_OK) return fail(LCT_ERR_ALLOC);
        {
          std::lock_guard<std::mutex> lk(mu_);
          (*stage_)[i] = b;
          have_[i] = 1;
        }
        cv_.notify_all();
      }
    }
    for (;;) {
      int slot;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || !ready_.empty(); });
        if (ready_.empty()) return;
        slot = ready_.front();
        ready_.erase(ready_.begin());
      }
      const char* src;
      long long off0;
      {
        std::lock_guard<std::mutex> lk(mu_);
        src = reinterpret_cast<const char*>((*stage_)[slot].p);
        off0 = (long long)dest_[slot] * slab_bytes_;
      }
      if (host_) std::memcpy(host_ + off0, src, (size_t)slab_bytes_);
      long long left = fd_ >= 0 ? slab_bytes_ : 0, off = off0;
      int e = LCT_OK;
      while (left > 0) {
        const ssize_t n = ::pwrite(fd_, src, (size_t)std::min<long long>(left, 1LL << 30), (off_t)off);
        if (n < 0 && errno == EINTR) continue;
        if (n <= 0) {
          e = LCT_ERR_IO;
          break;
        }
        src += n;
        off += n;
        left -= n;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (e && !err_) err_ = e;
        busy_[slot] = 0;
      }
      cv_.notify_all();
    }
  }
  void fail(int e) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (!err_) err_ = e;
    }
    cv_.notify_all();
  }
  double wait_s_ = 0.0;  // the pipeline's waits for a free slot (its thread only)
  int fd_ = -1;
  char* host_ = nullptr;
  long long slab_bytes_ = 0;
  std::vector<PinnedBuf>* stage_ = nullptr;
  int slots_ = 0, device_ = 0;
  std::vector<int> busy_, dest_, ready_, have_;
  std::vector<Sub> sub_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool stop_ = false;
  int err_ = LCT_OK;
};

// ----------------------------------------------------------------------------------------------
// the pipeline
// ----------------------------------------------------------------------------------------------
struct FanFeed {
  const float* dev = nullptr;   // device fan, the run's view 0 (read in place)
  const float* host = nullptr;  // host fan, the run's view 0
  FanReader* reader = nullptr;  // file
};
struct ImageSink {
  float* dev = nullptr;         // the caller's device volume (written in place)
  float* host = nullptr;        // the caller's host volume
  SlabWriter* writer = nullptr;  // a file
};

// Events of one run: kForkJoinEvents for the fork and join, per slab: views ready, backprojected, downloaded;
// per piece: uploaded, packed.
static int run_events(lct_recon* r, long long n_pieces, cudaEvent_t** base) {
  const int nb = r->info.n_blocks_run;
  const size_t n_ev = kForkJoinEvents + 3 * (size_t)nb + 2 * (size_t)n_pieces;
  while (r->sev.size() < n_ev) {
    cudaEvent_t e;
    int st = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    if (st) return st;
    r->sev.push_back(e);
  }
  *base = r->sev.data();
  return LCT_OK;
}

static int run_pipeline(lct_recon* r, const FanFeed& feed, const ImageSink& sink,
                        cudaStream_t caller, const StreamSet& ss) {
  (void)caller;                    // the caller forks the set from it and joins it back
  const cudaStream_t s = ss.prep;  // per-piece rebin / filter / pack
  const lct_geom& g = r->info.ctg;
  const lct_img& ig = r->info.ig;
  const int nb = r->info.n_blocks_run;
  const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;
  const long long plane = r->plane;
  const long long P = r->piece > 0 ? r->piece : kDefaultPiece;
  int st;
  // + the first slab's short pieces (the pivot and at most 64 doublings up to a full piece)
  const long long n_pieces = r->g_count / P + nb + 2 + 64;
  cudaEvent_t* ev = nullptr;
  if ((st = run_events(r, n_pieces, &ev))) return st;
  cudaEvent_t* ev_views = ev + kForkJoinEvents;
  cudaEvent_t* ev_bp = ev_views + nb;
  cudaEvent_t* ev_dl = ev_bp + nb;
  cudaEvent_t* ev_up = ev_dl + nb;
  cudaEvent_t* ev_packed = ev_up + n_pieces;
  long long piece = 0;

  long long reach_lo, reach_hi;
  rebin_reach(g, reach_lo, reach_hi);
  std::vector<int> order(nb);
  std::vector<long long> gfirst(nb), gend(nb);
  for (int b = 0; b < nb; ++b) {
    order[b] = b;
    gfirst[b] = r->blocks[b].block_proj_start + g.add_projections;
    gend[b] = gfirst[b] + g.n_angle;
  }
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return gend[x] < gend[y]; });
  const int packed = r->o.addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER;
  const long long fan_ring = feed.dev ? 0 : r->fan_ring;
  long long done = r->g_first, up = 0;  // global views packed so far; fan views uploaded
  int waited = 0;                       // slabs (in processing order) the packs have waited for
  const bool ring_img = !sink.dev && r->img_ring > 0;
  float* const img_base = sink.dev ? sink.dev : r->d_img;

  // fan views [a, b) of the run into the fan buffer (a ring: split at its end)
  auto upload = [&](long long a, long long b, const float* src) -> int {
    while (a < b) {
      const long long slot = fan_ring > 0 ? a % fan_ring : a;
      const long long n = fan_ring > 0 ? std::min(b - a, fan_ring - slot) : b - a;
      int e = cuda_status(cudaMemcpyAsync(r->d_fan + slot * plane, src, sizeof(float) * n * plane,
                                          cudaMemcpyHostToDevice, ss.up));
      if (e) return e;
      a += n;
      src += n * plane;
    }
    return LCT_OK;
  };
  auto bp = [&](int k, int b, int lo, int hi, int part, cudaStream_t sb) -> int {
    BpLaunch L;
    recon_bp_launch(r, b, b + 1, img_base, L);
    if (ring_img) {
      L.img = r->d_img + (long long)(k % r->img_ring) * slab;
      L.slab_z0[0] = 0;
    }
    L.view_lo = lo;
    L.view_hi = hi;
    L.part = part;
    const int e = recon_bp_pairs(r, L, sb);
    if (!e) r->launches++;
    return e;
  };
  for (int k = 0; k < nb; ++k) {
    const int b = order[k];
    cudaStream_t sb = ss.bp[k & 1];
    const bool split = k == 0;  // the first slab in parts as its views arrive
    const long long slab_end = std::min(gend[b], r->g_first + r->g_count);
    int bp_lo = 0, parts = 0;
    while (slab_end > done) {
      long long target = std::min(slab_end, done + P);
      if (split) target = first_part_target(done, target, gfirst[b], g.n_proj_turn / 2);
      const long long need = std::min(r->fan_count, target + reach_hi + 1 - r->fan_first);
      if (piece >= n_pieces) return LCT_ERR_ARG;  // cannot happen: pieces are counted above
      if (!feed.dev && need > up) {
        // the upload overwrites ring slots of views only the rebins up to piece - 2 read
        if (fan_ring > 0 && piece >= 2 &&
            (st = cuda_status(cudaStreamWaitEvent(ss.up, ev_packed[piece - 2], 0))))
          return st;
        if (feed.reader) {
          while (up < need) {  // whole chunks, in order
            const float* h = nullptr;
            long long nv = 0;
            const long long c = up / feed.reader->chunk();
            if ((st = feed.reader->acquire(c, &h, &nv))) return st;
            if ((st = upload(up, up + nv, h))) return st;
            if ((st = feed.reader->release_after(ss.up, c))) return st;
            up += nv;
          }
        } else {
          if ((st = upload(up, need, feed.host + up * plane))) return st;
          up = need;
        }
      }
      if ((st = cuda_status(cudaEventRecord(ev_up[piece], ss.up)))) return st;
      if ((st = cuda_status(cudaStreamWaitEvent(s, ev_up[piece], 0)))) return st;
      // the pack overwrites quad-ring slots of views [target - ring - (target - done), target -
      // ring): wait for every slab whose window holds one of them
      if (r->quad_ring > 0) {
        while (waited < k && gfirst[order[waited]] < target - r->quad_ring) {
          if ((st = cuda_status(cudaStreamWaitEvent(s, ev_bp[waited], 0)))) return st;
          ++waited;
        }
        if (waited < nb && waited >= k && k < nb && gfirst[order[waited]] < target - r->quad_ring)
          return LCT_ERR_UNSUPPORTED;  // a slab not yet backprojected would lose views (ring too small)
      }
      const long long v0 = done - r->g_first, nv = target - done;
      float* par = r->bounded ? r->d_par : r->d_par + v0 * plane;
      if ((st = launch_rebin_fan2par_scan(g, feed.dev ? feed.dev : r->d_fan, r->fan_first,
                                          r->fan_count, par, done, nv, r->o.interp, packed, s,
                                          fan_ring)))
        return st;
      r->launches++;
      if (r->o.filter_mode != LCT_FILTER_FP32)
        st = tc_filter(g.ns, par, nv * g.nt, r->d_tc, r->tc_rows, r->o.filter_mode, s);
      else
        st = launch_filter_rows(g.ns, r->d_h, par, nv * g.nt, LCT_FILTER_FP32, s);
      if (st) return st;
      r->launches += filter_launches(r->o.filter_mode);
      if ((st = recon_pack(r, par, nv, v0, packed, s))) return st;
      r->launches++;
      done = target;
      if ((st = cuda_status(cudaEventRecord(ev_packed[piece], s)))) return st;
      ++piece;
      // a pair starting at local view ia also reads its conjugate ia + half: a part takes the
      // pair starts whose conjugates are packed too
      const long long local = std::min<long long>(done - gfirst[b], g.n_angle);
      const int avail = (int)std::max<long long>(local - g.n_proj_turn / 2, 0);
      if (split && done < slab_end && avail > bp_lo) {
        if ((st = cuda_status(cudaStreamWaitEvent(sb, ev_packed[piece - 1], 0)))) return st;
        if ((st = bp(k, b, bp_lo, avail, parts ? kBpMiddle : kBpFirst, sb))) return st;
        bp_lo = avail;
        ++parts;
      }
    }
    if ((st = cuda_status(cudaEventRecord(ev_views[k], s)))) return st;
    if ((st = cuda_status(cudaStreamWaitEvent(sb, ev_views[k], 0)))) return st;
    // the volume slot is free once the slab that used it before is downloaded
    if (ring_img && k >= r->img_ring &&
        (st = cuda_status(cudaStreamWaitEvent(sb, ev_dl[k - r->img_ring], 0))))
      return st;
    if ((st = parts ? bp(k, b, bp_lo, g.n_angle, kBpLast, sb) : bp(k, b, 0, 1 << 30, kBpWhole, sb)))
      return st;
    if ((st = cuda_status(cudaEventRecord(ev_bp[k], sb)))) return st;
    const float* src = ring_img ? r->d_img + (long long)(k % r->img_ring) * slab
                                : img_base + (long long)b * slab;
    if (sink.host || sink.writer) {
      if ((st = cuda_status(cudaStreamWaitEvent(ss.down, ev_bp[k], 0)))) return st;
      float* dst = sink.host ? sink.host + (long long)b * slab : nullptr;
      if (sink.writer && (st = sink.writer->slot_for(k, &dst))) return st;
      if ((st = cuda_status(cudaMemcpyAsync(dst, src, sizeof(float) * slab, cudaMemcpyDeviceToHost,
                                            ss.down))))
        return st;
      if (sink.writer && (st = sink.writer->submit_after(ss.down, k, b))) return st;
    }
    if ((st = cuda_status(cudaEventRecord(ev_dl[k], sink.host || sink.writer ? ss.down : sb))))
      return st;
  }
  return LCT_OK;
}

// Fork the streams from s, run, join them back and time the span; on an error every stream is
// drained before returning (host functions of the reader and writer may still be queued).
template <class F>
static int run_forked(lct_recon* r, cudaStream_t s, F body) {
  int st;
  r->launches = 0;
  r->streamed = true;
  if ((st = cuda_status(cudaEventRecord(r->ev[0], s)))) return st;
  for (int i = 1; i < 4; ++i)
    if ((st = cuda_status(cudaEventRecord(r->ev[i], s)))) return st;
  if ((st = streams_create(r->ss))) return st;
  cudaEvent_t* ev = nullptr;
  if ((st = run_events(r, 0, &ev))) return st;
  if ((st = streams_fork(r->ss, s, r->sev[0]))) return st;
  st = body();
  int st2 = streams_join(r->ss, s, r->sev.data() + 1);
  if (st) {
    cudaStream_t all[7] = {r->ss.up, r->ss.down, r->ss.bp[0], r->ss.bp[1], r->ss.cnn, r->ss.prep, s};
    for (cudaStream_t x : all) cudaStreamSynchronize(x);
    return st;
  }
  if (st2) return st2;
  if ((st = cuda_status(cudaEventRecord(r->ev[4], s)))) return st;
  if ((st = cuda_status(cudaEventRecord(r->ev[5], s)))) return st;
  if ((st = cuda_status(cudaEventSynchronize(r->ev[5])))) return st;
  for (int i = 0; i < 5; ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r->ev[i], r->ev[i + 1]);
    r->times[i] = ms;
  }
  r->cnn_ms = 0.f;
  return LCT_OK;
}

bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// the slab writer's pinned slots (pinned by the writer on first use, kept with the recon)
static std::vector<PinnedBuf>* img_slots(lct_recon* r) {
  if (r->h_img_slots.empty()) r->h_img_slots.assign(kImgStage, PinnedBuf{});
  return &r->h_img_slots;
}

int recon_run_bounded_ptr(lct_recon* r, const float* fan, bool fan_on_device, float* image,
                          bool image_on_device, cudaStream_t s) {
  FanFeed feed;
  ImageSink sink;
  if (fan_on_device)
    feed.dev = fan;
  else
    feed.host = fan;
  if (image_on_device) {
    sink.dev = image;
  } else if (host_pinned(image)) {
    sink.host = image;
  } else {
    // pageable volume: slabs go through the pinned slots and are copied on the writer's threads
    const lct_img& ig = r->info.ig;
    const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;
    int dev = 0, st = cuda_status(cudaGetDevice(&dev));
    if (st) return st;
    SlabWriter writer;
    if ((st = writer.start(nullptr, image, (long long)sizeof(float) * slab, r->info.n_blocks_run,
                           img_slots(r), dev)))
      return st;
    sink.writer = &writer;
    st = run_forked(r, s, [&] { return run_pipeline(r, feed, sink, s, r->ss); });
    const int st_w = writer.finish();
    return st ? st : st_w;
  }
  return run_forked(r, s, [&] { return run_pipeline(r, feed, sink, s, r->ss); });
}

void recon_free_bounded(lct_recon* r) {
  for (PinnedBuf& b : r->h_fan_slots) pinned_free(b);
  for (PinnedBuf& b : r->h_img_slots) pinned_free(b);
  r->h_fan_slots.clear();
  r->h_img_slots.clear();
}

}  // namespace lct

using namespace lct;

LCT_API int lct_recon_create_bounded(const lct_plan* plan, const lct_recon_opts* opts,
                                     int piece_views, lct_recon** out) {
  if (piece_views < 0) return LCT_ERR_ARG;
  lct_recon* r = nullptr;
  int st = recon_setup(plan, opts, &r);
  if (st) return st;
  const lct_geom& g = r->info.ctg;
  const lct_img& ig = r->info.ig;
  const int nb = r->info.n_blocks_run;
  if (!recon_streamable(r) || !r->quads || r->o.addr == LCT_ADDR_LEGACY) {
    lct_recon_destroy(r);
    return LCT_ERR_UNSUPPORTED;
  }
  if (r->o.bp_nz == -1) r->o.bp_nz = 0;  // no whole-scan buffers to tune on: the default shape
  r->bounded = true;
  r->piece = piece_views > 0 ? piece_views : kDefaultPiece;
  const long long P = r->piece;
  long long reach_lo, reach_hi;
  rebin_reach(g, reach_lo, reach_hi);
  // fan ring: the views the rebins of two consecutive pieces read, plus a chunk of read-ahead
  const long long fr = 3 * P + (reach_hi - reach_lo) + 16;
  r->fan_ring = fr < r->fan_count ? fr : 0;
  // quad ring: a window, a piece and the two slab strides the alternating streams keep in flight
  long long stride = 0;
  for (int b = 1; b < nb; ++b)
    stride = std::max<long long>(stride, std::llabs((long long)r->blocks[b].block_proj_start -
                                                   r->blocks[b - 1].block_proj_start));
  const long long qr = g.n_angle + P + 2 * stride + 16;
  r->quad_ring = qr < r->g_count ? qr : 0;
  r->img_ring = nb > kImgRing ? kImgRing : 0;
  const long long fan_views = r->fan_ring > 0 ? r->fan_ring : r->fan_count;
  const long long quad_views = r->quad_ring > 0 ? r->quad_ring : r->g_count;
  const long long img_slabs = r->img_ring > 0 ? r->img_ring : nb;
  const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;
  auto alloc = [&](void** p, size_t bytes) {
    int e = cuda_status(cudaMalloc(p, bytes));
    if (!e) r->device_bytes += (long long)bytes;
    return e;
  };
  do {
    if ((st = alloc((void**)&r->d_fan, sizeof(float) * fan_views * r->plane))) break;
    if ((st = alloc((void**)&r->d_par, sizeof(float) * P * r->plane))) break;
    if ((st = alloc((void**)&r->d_img, sizeof(float) * img_slabs * slab))) break;
    if (r->tex_bp) {
      if ((st = view_texture_create(r->vtex, g.ns, g.nt, quad_views,
                                    r->o.addr == LCT_ADDR_CLAMP ? LCT_ADDR_CLAMP : LCT_ADDR_BORDER))) {
        if (st != LCT_ERR_UNSUPPORTED) break;
        r->tex_bp = false;  // deeper than the device's 3-D texture limit: quads
        st = LCT_OK;
      } else {
        r->device_bytes += (long long)sizeof(float) * quad_views * r->plane;
      }
    }
    if (!r->tex_bp &&
        (st = alloc((void**)&r->d_quad, sizeof(float4) * quad_views * quad_view_elems(g.ns, g.nt))))
      break;
    if (r->tma_bp && bp_tma_map(&r->tma_map, r->d_quad, g.ns, g.nt, quad_views) != LCT_OK)
      r->tma_bp = false;
    if (r->o.filter_mode != LCT_FILTER_FP32) r->tc_rows = P * g.nt;
    st = recon_alloc_common(r, plan);
  } while (0);
  if (st) {
    lct_recon_destroy(r);
    return recon_alloc_status(st);
  }
  *out = r;
  return LCT_OK;
}

LCT_API int lct_recon_device_bytes(const lct_recon* r, int64_t* bytes) {
  if (!r || !bytes) return LCT_ERR_ARG;
  *bytes = r->device_bytes;
  return LCT_OK;
}

LCT_API int lct_recon_run_file(lct_recon* r, const char* fan_path, const char* image_path,
                               float* image, lct_stream stream) {
  if (!r || !fan_path || (!image_path && !image)) return LCT_ERR_ARG;
  if (!recon_streamable(r) || !r->quads || r->o.addr == LCT_ADDR_LEGACY) return LCT_ERR_UNSUPPORTED;
  if (r->cnn) return LCT_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
  const lct_img& ig = r->info.ig;
  const int nb = r->info.n_blocks_run;
  const long long P = r->piece > 0 ? r->piece : kDefaultPiece;
  const long long slab = (long long)kBlockSlices * ig.nx * ig.ny;
  int st;
  // pinned staging, kept with the recon: chunks of whole views (pinning costs time in
  // proportion to the bytes, so the chunks are small and many, and each is pinned by its reader
  // thread just before its first read)
  const long long view_bytes = (long long)sizeof(float) * r->plane;
  const long long chunk = std::max<long long>(1, std::min<long long>(P, kFanChunkBytes / view_bytes));
  if (r->h_fan_slots.empty()) {
    r->h_fan_slots.assign(kFanStage, PinnedBuf{});
    r->fan_chunk_views = chunk;
  }
  if (r->fan_chunk_views != chunk) return LCT_ERR_ARG;  // cannot happen: fixed per recon
  int dev = 0;
  if ((st = cuda_status(cudaGetDevice(&dev)))) return st;
  // a file, or a pageable volume, is written from pinned slots by the writer's threads (both at
  // once when both are asked for); a pinned volume is downloaded into directly
  const bool use_writer = image_path || !host_pinned(image);
  FanReader reader;
  SlabWriter writer;
  // file view v of the run's fan views lies at (fan_first + DataOffset + v) views into the file
  // (Src/DataReader.cpp:14, in 64 bits)
  const long long byte0 = (r->fan_first + r->info.data_offset) * view_bytes;
  if ((st = reader.start(fan_path, byte0, view_bytes, r->fan_count, chunk, &r->h_fan_slots, dev)))
    return st;
  if (use_writer && (st = writer.start(image_path, image, (long long)sizeof(float) * slab, nb,
                                       img_slots(r), dev))) {
    reader.finish();
    return st;
  }
  FanFeed feed;
  feed.reader = &reader;
  ImageSink sink;
  if (use_writer)
    sink.writer = &writer;
  else
    sink.host = image;
  st = run_forked(r, s, [&] { return run_pipeline(r, feed, sink, s, r->ss); });
  const int st_r = reader.finish();
  const int st_w = use_writer ? writer.finish() : LCT_OK;
  r->io_times[0] = (float)reader.read_seconds();
  r->io_times[1] = (float)reader.wait_seconds();
  r->io_times[2] = (float)writer.wait_seconds();
  return st ? st : (st_r ? st_r : st_w);
}

LCT_API int lct_recon_io_times(const lct_recon* r, float* s3) {
  if (!r || !s3) return LCT_ERR_ARG;
  for (int i = 0; i < 3; ++i) s3[i] = r->io_times[i];
  return LCT_OK;
}
