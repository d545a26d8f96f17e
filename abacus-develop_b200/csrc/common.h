// Shared host-side helpers: status codes, error capture, device buffers.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace b200 {

enum Status : int {
    kOk = 0,
    kInvalidArgument = 1,
    kCudaError = 2,
    kCublasError = 3,
    kCusolverError = 4,
    kNumericalError = 5,
    kCapacityError = 6,
    kNotConverged = 7,
    kCallbackError = 8,
    kShed = 9,
};

// A failure raised inside the library; the C-ABI turns it into a status code
// plus a message readable through b200_last_error().
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);
const char* last_error();

// Number of kernels this library has launched (all devices, all threads).
void note_launch(unsigned n = 1);
unsigned long long launches();

#define B200_CUDA(call)                                                                                    \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            throw ::b200::Error(::b200::kCudaError, std::string(#call) + ": " + cudaGetErrorString(e_) +   \
                                                        " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
    } while (0)

#define B200_CHECK(cond, code, msg)                      \
    do {                                                 \
        if (!(cond)) throw ::b200::Error((code), (msg)); \
    } while (0)

// Owning device allocation (cudaMalloc / cudaFree).
template <typename T> struct DeviceArray {
    T* ptr = nullptr;
    size_t n = 0;
    DeviceArray() = default;
    explicit DeviceArray(size_t count) { resize(count); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : ptr(o.ptr), n(o.n) {
        o.ptr = nullptr;
        o.n = 0;
    }
    DeviceArray& operator=(DeviceArray&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            n = o.n;
            o.ptr = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DeviceArray() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        n = 0;
    }
    void resize(size_t count) {
        if (count <= n && ptr) return;
        release();
        if (count == 0) return;
        B200_CUDA(cudaMalloc(&ptr, count * sizeof(T)));
        n = count;
    }
    void upload(const T* host, size_t count, cudaStream_t s = 0) {
        resize(count);
        if (count) B200_CUDA(cudaMemcpyAsync(ptr, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

inline int ceil_div(long a, long b) { return int((a + b - 1) / b); }

}  // namespace b200
