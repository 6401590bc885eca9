// Host <-> device transfers of large pageable arrays through a few pinned
// staging buffers per device: the host copies a piece into a pinned buffer
// with all threads (OpenMP) while the DMA engine moves the previous piece, so
// a transfer runs at the pinned rate instead of the driver's single-threaded
// pageable path. One transfer at a time per device (a mutex); the buffers are
// allocated on first use and kept until exit.
#pragma once
#include <cuda_runtime.h>
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <mutex>

namespace fe {

class Staging {
 public:
  static constexpr int NB = 4;                    // buffers in flight
  static constexpr size_t PIECE = size_t(32) << 20;  // bytes per buffer

  // The staging area of the current device (nullptr if it cannot be made).
  static Staging* get() {
    static std::mutex mu;
    static Staging* per_dev[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (!per_dev[dev]) {
      Staging* s = new Staging();
      if (!s->init()) {
        delete s;
        return nullptr;
      }
      per_dev[dev] = s;
    }
    return per_dev[dev];
  }

  // bytes from pageable src to device dst on stream st (after the work
  // queued on it); returns when every piece has reached the device.
  cudaError_t to_device(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    std::lock_guard<std::mutex> g(mu_);
    cudaError_t e = cudaSuccess;
    for (size_t off = 0, k = 0; off < bytes && e == cudaSuccess; off += PIECE, ++k) {
      const int b = (int)(k % NB);
      const size_t len = bytes - off < PIECE ? bytes - off : PIECE;
      if ((e = cudaEventSynchronize(ev_[b])) != cudaSuccess) break;
      par_copy(buf_[b], static_cast<const char*>(src) + off, len);
      if ((e = cudaMemcpyAsync(static_cast<char*>(dst) + off, buf_[b], len, cudaMemcpyHostToDevice, st)) !=
          cudaSuccess)
        break;
      e = cudaEventRecord(ev_[b], st);
    }
    // src is no longer needed, but the buffers are: finish before releasing them
    for (int b = 0; b < NB && e == cudaSuccess; ++b) e = cudaEventSynchronize(ev_[b]);
    return e;
  }

  // bytes from device src to pageable dst, after the work queued on st.
  cudaError_t to_host(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    std::lock_guard<std::mutex> g(mu_);
    const size_t n = (bytes + PIECE - 1) / PIECE;
    cudaError_t e = cudaSuccess;
    auto issue = [&](size_t k) {
      const size_t off = k * PIECE, len = bytes - off < PIECE ? bytes - off : PIECE;
      const int b = (int)(k % NB);
      cudaError_t r = cudaMemcpyAsync(buf_[b], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, st);
      return r == cudaSuccess ? cudaEventRecord(ev_[b], st) : r;
    };
    for (size_t k = 0; k < n && k < (size_t)NB && e == cudaSuccess; ++k) e = issue(k);
    for (size_t k = 0; k < n && e == cudaSuccess; ++k) {
      const int b = (int)(k % NB);
      const size_t off = k * PIECE, len = bytes - off < PIECE ? bytes - off : PIECE;
      if ((e = cudaEventSynchronize(ev_[b])) != cudaSuccess) break;
      par_copy(static_cast<char*>(dst) + off, buf_[b], len);
      if (k + NB < n) e = issue(k + NB);
    }
    if (e != cudaSuccess)  // no copy may still target the buffers
      for (int b = 0; b < NB; ++b) cudaEventSynchronize(ev_[b]);
    return e;
  }

  // count doubles from pageable src to floats at device dst: each piece is
  // narrowed (round to nearest, as the device's conversion) into a pinned
  // buffer by all threads, so the host moves 12 bytes an entry instead of 16
  // and the link 4 instead of 8.
  cudaError_t to_device_narrow(float* dst, const double* src, size_t count, cudaStream_t st) {
    std::lock_guard<std::mutex> g(mu_);
    constexpr size_t PE = PIECE / sizeof(float);
    cudaError_t e = cudaSuccess;
    for (size_t off = 0, k = 0; off < count && e == cudaSuccess; off += PE, ++k) {
      const int b = (int)(k % NB);
      const size_t len = count - off < PE ? count - off : PE;
      if ((e = cudaEventSynchronize(ev_[b])) != cudaSuccess) break;
      float* pb = static_cast<float*>(buf_[b]);
      const double* ps = src + off;
#pragma omp parallel for schedule(static)
      for (int64_t j = 0; j < (int64_t)len; ++j) pb[j] = (float)ps[j];
      if ((e = cudaMemcpyAsync(dst + off, pb, len * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess) break;
      e = cudaEventRecord(ev_[b], st);
    }
    for (int b = 0; b < NB && e == cudaSuccess; ++b) e = cudaEventSynchronize(ev_[b]);
    return e;
  }

  // count floats from device src to doubles at pageable dst (exact), after
  // the work queued on st.
  cudaError_t to_host_widen(double* dst, const float* src, size_t count, cudaStream_t st) {
    std::lock_guard<std::mutex> g(mu_);
    constexpr size_t PE = PIECE / sizeof(float);
    const size_t n = (count + PE - 1) / PE;
    cudaError_t e = cudaSuccess;
    auto issue = [&](size_t k) {
      const size_t off = k * PE, len = count - off < PE ? count - off : PE;
      const int b = (int)(k % NB);
      cudaError_t r = cudaMemcpyAsync(buf_[b], src + off, len * sizeof(float), cudaMemcpyDeviceToHost, st);
      return r == cudaSuccess ? cudaEventRecord(ev_[b], st) : r;
    };
    for (size_t k = 0; k < n && k < (size_t)NB && e == cudaSuccess; ++k) e = issue(k);
    for (size_t k = 0; k < n && e == cudaSuccess; ++k) {
      const int b = (int)(k % NB);
      const size_t off = k * PE, len = count - off < PE ? count - off : PE;
      if ((e = cudaEventSynchronize(ev_[b])) != cudaSuccess) break;
      const float* pb = static_cast<const float*>(buf_[b]);
      double* pd = dst + off;
#pragma omp parallel for schedule(static)
      for (int64_t j = 0; j < (int64_t)len; ++j) pd[j] = (double)pb[j];
      if (k + NB < n) e = issue(k + NB);
    }
    if (e != cudaSuccess)
      for (int b = 0; b < NB; ++b) cudaEventSynchronize(ev_[b]);
    return e;
  }

 private:
  std::mutex mu_;
  void* buf_[NB] = {};
  cudaEvent_t ev_[NB] = {};

  bool init() {
    for (int b = 0; b < NB; ++b) {
      if (cudaMallocHost(&buf_[b], PIECE) != cudaSuccess ||
          cudaEventCreateWithFlags(&ev_[b], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
    }
    return true;
  }
  static void par_copy(void* dst, const void* src, size_t len) {
    const int nt = omp_get_max_threads();
    const size_t part = ((len / (size_t)nt) + 4095) & ~size_t(4095);
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nt; ++t) {
      const size_t a = (size_t)t * part;
      if (a < len)
        std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, len - a < part ? len - a : part);
    }
  }
};

}  // namespace fe
