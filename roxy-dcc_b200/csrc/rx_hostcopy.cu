// Host <-> device copies of pageable arrays through one pinned buffer per
// context.  A cudaMemcpyAsync from or to pageable memory is staged by the
// driver through its own small pinned buffers, one chunk at a time on the
// calling thread.  Here worker threads move the bytes between the pageable
// arrays and the context's pinned buffer, a piece at a time, while the
// calling thread hands each finished piece to the copy engine, so that the
// host copies of later pieces overlap the DMA of earlier ones.
//
// Uploads fill the buffer with non-temporal stores.  Lines written by
// ordinary stores on several cores stay dirty in those cores' caches, and a
// DMA that reads them right after runs at a third of its rate (measured on
// the benchmark host: 17 MB in 1.0-1.6 ms after an 8-thread memcpy, 0.33 ms
// after an 8-thread streaming-store fill).
//
// All copies go on the context's stream and every caller holds the context
// lock, so one buffer serves uploads and reads alike.  Host writes into the
// buffer wait for `stage_done`: the last DMA that read it.
#include <algorithm>
#include <memory>
#include <thread>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "rx_runtime.h"

namespace rx {

namespace {

constexpr size_t kPiece = 2u << 20;        // bytes per staged piece
constexpr size_t kMinStaged = 1u << 20;    // smaller transfers go to the driver as they are
constexpr int kMaxWorkers = 8;
constexpr size_t kPieceEvents = Ctx::kPieceEvents;

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int worker_count(size_t pieces) {
  unsigned hw = std::thread::hardware_concurrency();
  size_t t = std::min<size_t>(kMaxWorkers, pieces);
  if (hw) t = std::min<size_t>(t, hw);
  return (int)std::max<size_t>(t, 1);
}

// Copy into the pinned buffer around the CPU caches; `dst` is 16-byte
// aligned.  The fence makes the stores visible before the piece is handed to
// the copy engine.
void stream_copy(char* dst, const char* src, size_t n) {
#if defined(__SSE2__)
  size_t i = 0;
  for (; i + 64 <= n; i += 64) {
    const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i));
    const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 16));
    const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 32));
    const __m128i d = _mm_loadu_si128(reinterpret_cast<const __m128i*>(src + i + 48));
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i), a);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 16), b);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 32), c);
    _mm_stream_si128(reinterpret_cast<__m128i*>(dst + i + 48), d);
  }
  if (i < n) std::memcpy(dst + i, src + i, n - i);
  _mm_sfence();
#else
  std::memcpy(dst, src, n);
#endif
}

// One piece: `bytes` at `host_off` of host array `array`, at `stage_off` of
// the pinned buffer.
struct Piece {
  int array;
  size_t host_off, stage_off, bytes;
};

}  // namespace

bool host_stage_reserve(Ctx* c, size_t bytes) {
  if (!c->stage_done && cudaEventCreateWithFlags(&c->stage_done, cudaEventDisableTiming) != cudaSuccess) {
    (void)cudaGetLastError();
    c->stage_done = nullptr;
    return false;
  }
  if (c->stage_bytes >= bytes) return true;
  if (c->stage) {
    cudaEventSynchronize(c->stage_done);  // the old buffer may still feed a copy
    cudaFreeHost(c->stage);
  }
  c->stage = nullptr;
  c->stage_bytes = 0;
  const size_t want = align_up(std::max(bytes, (size_t)16 << 20), kPiece);
  if (cudaHostAlloc(&c->stage, want, cudaHostAllocDefault) != cudaSuccess) {
    (void)cudaGetLastError();  // no pinned memory to be had: callers use the driver's path
    c->stage = nullptr;
    return false;
  }
  c->stage_bytes = want;
  return true;
}

void host_stage_free(Ctx* c) {
  if (c->stage) {
    if (c->stage_done) cudaEventSynchronize(c->stage_done);
    cudaFreeHost(c->stage);
  }
  if (c->stage_done) cudaEventDestroy(c->stage_done);
  for (auto& e : c->piece_ev)
    if (e) cudaEventDestroy(e);
  c->stage = nullptr;
  c->stage_bytes = 0;
  c->stage_done = nullptr;
  for (auto& e : c->piece_ev) e = nullptr;
}

int upload_staged(Ctx* c, const HostPiece* arrays, int n) {
  size_t total = 0;
  for (int i = 0; i < n; ++i) total += align_up(arrays[i].bytes, 256);
  if (total < kMinStaged || !host_stage_reserve(c, total)) {
    for (int i = 0; i < n; ++i)
      if (arrays[i].bytes)
        CUDA_TRY(c, cudaMemcpyAsync(arrays[i].dev, arrays[i].host, arrays[i].bytes, cudaMemcpyHostToDevice,
                                    c->stream));
    return RX_OK;
  }
  std::vector<Piece> pieces;
  size_t at = 0;
  for (int i = 0; i < n; ++i) {
    for (size_t off = 0; off < arrays[i].bytes; off += kPiece)
      pieces.push_back({i, off, at + off, std::min(kPiece, arrays[i].bytes - off)});
    at += align_up(arrays[i].bytes, 256);
  }
  CUDA_TRY(c, cudaEventSynchronize(c->stage_done));  // the last DMA out of the buffer has finished
  const size_t P = pieces.size();
  std::unique_ptr<std::atomic<int>[]> ready(new std::atomic<int>[P]);
  for (size_t k = 0; k < P; ++k) ready[k].store(0, std::memory_order_relaxed);
  char* stage = static_cast<char*>(c->stage);
  const int T = worker_count(P);
  std::vector<std::thread> th;
  th.reserve(T);
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t] {
      for (size_t k = t; k < P; k += T) {
        const Piece& p = pieces[k];
        stream_copy(stage + p.stage_off, static_cast<const char*>(arrays[p.array].host) + p.host_off, p.bytes);
        ready[k].store(1, std::memory_order_release);
      }
    });
  cudaError_t err = cudaSuccess;
  for (size_t k = 0; k < P; ++k) {
    while (!ready[k].load(std::memory_order_acquire)) std::this_thread::yield();
    const Piece& p = pieces[k];
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(static_cast<char*>(arrays[p.array].dev) + p.host_off, stage + p.stage_off, p.bytes,
                            cudaMemcpyHostToDevice, c->stream);
  }
  for (auto& x : th) x.join();
  if (err == cudaSuccess) err = cudaEventRecord(c->stage_done, c->stream);
  if (err != cudaSuccess) cudaStreamSynchronize(c->stream);  // no copy may still read the buffer
  CUDA_TRY(c, err);
  return RX_OK;
}

int download_staged(Ctx* c, void* host, const void* dev, size_t bytes) {
  if (bytes == 0) return RX_OK;
  if (bytes < kMinStaged || !host_stage_reserve(c, bytes)) {
    CUDA_TRY(c, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return RX_OK;
  }
  // pieces of at least kPiece bytes, at most one event each
  const size_t piece = align_up(std::max(kPiece, (bytes + kPieceEvents - 1) / kPieceEvents), 4096);
  const size_t P = (bytes + piece - 1) / piece;
  for (size_t k = 0; k < P; ++k)
    if (!c->piece_ev[k] && cudaEventCreateWithFlags(&c->piece_ev[k], cudaEventDisableTiming) != cudaSuccess) {
      (void)cudaGetLastError();
      c->piece_ev[k] = nullptr;
      CUDA_TRY(c, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
      CUDA_TRY(c, cudaStreamSynchronize(c->stream));
      return RX_OK;
    }
  char* stage = static_cast<char*>(c->stage);
  cudaError_t err = cudaSuccess;
  size_t issued = 0;
  for (; issued < P && err == cudaSuccess; ++issued) {
    const size_t off = issued * piece, n = std::min(piece, bytes - off);
    err = cudaMemcpyAsync(stage + off, static_cast<const char*>(dev) + off, n, cudaMemcpyDeviceToHost, c->stream);
    if (err == cudaSuccess) err = cudaEventRecord(c->piece_ev[issued], c->stream);
  }
  if (err != cudaSuccess) {
    cudaStreamSynchronize(c->stream);
    CUDA_TRY(c, err);
  }
  // the calling thread waits for each piece in order; workers copy it out
  std::unique_ptr<std::atomic<int>[]> ready(new std::atomic<int>[P]);
  for (size_t k = 0; k < P; ++k) ready[k].store(0, std::memory_order_relaxed);
  const int T = worker_count(P);
  std::vector<std::thread> th;
  th.reserve(T);
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t] {
      for (size_t k = t; k < P; k += T) {
        int r;
        while ((r = ready[k].load(std::memory_order_acquire)) == 0) std::this_thread::yield();
        if (r < 0) continue;  // the copy failed: nothing to move
        const size_t off = k * piece;
        std::memcpy(static_cast<char*>(host) + off, stage + off, std::min(piece, bytes - off));
      }
    });
  for (size_t k = 0; k < P; ++k) {
    if (err == cudaSuccess) err = cudaEventSynchronize(c->piece_ev[k]);
    ready[k].store(err == cudaSuccess ? 1 : -1, std::memory_order_release);
  }
  for (auto& x : th) x.join();
  CUDA_TRY(c, err);
  return RX_OK;
}

}  // namespace rx
