// Shared host/device definitions of the spider_b200 library.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace spi {

// Status codes (IRTFLG-style, see include/spider_b200.h)
enum : int {
  kOk = 0,
  kAlloc = 46,
  kInvalid = 101,
  kMissing = 102,
  kCuda = 200,
  kCufft = 201,
  kDevice = 202,
};

void set_error(const char* fmt, ...);
const char* last_error_cstr();
int fail(int code, const char* fmt, ...);

#define SPI_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return ::spi::fail(::spi::kCuda, "%s:%d %s: %s", __FILE__, __LINE__, #call,   \
                         cudaGetErrorString(e_));                                   \
  } while (0)

#define SPI_CUFFT(call)                                                             \
  do {                                                                              \
    cufftResult r_ = (call);                                                        \
    if (r_ != CUFFT_SUCCESS)                                                        \
      return ::spi::fail(::spi::kCufft, "%s:%d %s: cufft error %d", __FILE__,       \
                         __LINE__, #call, (int)r_);                                 \
  } while (0)

#define SPI_TRY(expr)            \
  do {                           \
    int s_ = (expr);             \
    if (s_ != 0) return s_;      \
  } while (0)

// Device buffer owned by a context (cudaMalloc / cudaFree).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t want);   // grows (never shrinks) and keeps nothing
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// Pinned host buffer.
struct HostBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t want);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// Host-side tables shared by the kernels (computed in host_math.cpp with
// IEEE single/double semantics, no contraction).
struct KBTab {
  float tab[5000];
  float fltb, alpha, aaaa;
  int ln2;
};
void fill_kb(int n2, KBTab& t);
void windkb_table(int nx, const KBTab& kb, std::vector<float>& wkb);
void cang(float phi, float theta, float psi, float* dm9);
void matmul33(const float* sm, const float* dm, float* out);
void cang_pj(float phi, float theta, float psi, float* dm9);  // WPRO_N's own copy

}  // namespace spi
