// Shared definitions of the B200 H-matrix engine: status codes, error
// plumbing, device buffers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dmhm_b200.h"

namespace hmb {

// Thrown inside the library, turned into an HM_* status at the C-ABI.
struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

void set_last_error(const std::string& msg);

#define HMB_CUDA(call)                                                        \
    do {                                                                      \
        cudaError_t err__ = (call);                                           \
        if (err__ != cudaSuccess)                                             \
            throw ::hmb::Error(HM_ERR_CUDA, std::string(#call) + ": " +       \
                               cudaGetErrorString(err__));                    \
    } while (0)

#define HMB_CHECK_LAUNCH() HMB_CUDA(cudaGetLastError())

#define HMB_REQUIRE(cond, code, msg)                                          \
    do {                                                                      \
        if (!(cond)) throw ::hmb::Error((code), (msg));                       \
    } while (0)

// Host-to-device copy of `bytes` from pageable `src` that does not block the
// host behind the stream's earlier work: the data go through a pinned staging
// ring owned per stream (the ring is reused after the stream has passed the
// copies that read it).  Falls back to a plain copy when the data do not fit.
void staged_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);
void release_staging(cudaStream_t s);

// Owning device allocation (cudaMallocAsync on the engine stream).
template <typename T>
class DeviceBuffer {
  public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept { swap(o); }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) { reset(); swap(o); }
        return *this;
    }
    ~DeviceBuffer() { reset(); }

    void allocate(size_t n, cudaStream_t s) {
        reset();
        stream_ = s;
        n_ = n;
        if (n) {
            cudaError_t e = cudaMallocAsync((void**)&p_, n * sizeof(T), s);
            if (e != cudaSuccess) {
                p_ = nullptr;
                n_ = 0;
                throw Error(HM_ERR_OOM, std::string("device allocation of ") +
                                            std::to_string(n * sizeof(T)) +
                                            " bytes failed: " + cudaGetErrorString(e));
            }
        }
    }
    void reset() {
        if (p_) cudaFreeAsync(p_, stream_);
        p_ = nullptr;
        n_ = 0;
    }
    void upload(const std::vector<T>& h, cudaStream_t s) {
        allocate(h.size(), s);
        if (!h.empty()) staged_h2d(p_, h.data(), h.size() * sizeof(T), s);
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }

  private:
    void swap(DeviceBuffer& o) {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        std::swap(stream_, o.stream_);
    }
    T* p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t stream_ = 0;
};

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace hmb
