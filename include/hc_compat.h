/*
 * hc_compat.h -- the HCC runtime types that hcBLAS's public headers expose,
 * re-expressed for CUDA so that existing hcBLAS callers compile unchanged.
 *
 * The reference's API is written against HCC (hc.hpp / hc_am.hpp):
 *   hc::accelerator, hc::accelerator_view      (lib/include/hcblas.h:42-45)
 *   hc::half                                   (lib/include/hcblas.h:685-689)
 *   hc::short_vector::float_2 / double_2       (lib/include/hcblaslib.h:269-315)
 *   hc::am_alloc / hc::am_free                  (used by every reference test,
 *                                               e.g. test/unit/hcblas_sgemm.cpp:56)
 * Here an accelerator is a CUDA device ordinal and an accelerator_view is a
 * (device, cudaStream_t) pair -- the view *is* the stream, exactly as in HCC,
 * where kernels are enqueued on a view's queue.
 *
 * The C part (hcblas_accl_view_t, hcblas_half_t) is what crosses the C ABI;
 * the C++ part wraps it with the HCC method names the reference tests call
 * (accelerator::get_default_view, accelerator_view::copy / wait, ...).
 */
#ifndef HCBLAS_B200_HC_COMPAT_H_
#define HCBLAS_B200_HC_COMPAT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* An accelerator view: a CUDA device ordinal and a stream on it (NULL = the
 * legacy default stream of that device). */
typedef struct hcblas_accl_view {
  int device_id;
  void *stream; /* cudaStream_t */
} hcblas_accl_view_t;

/* IEEE binary16 storage (the bits of an hc::half). */
typedef struct hcblas_half {
  uint16_t bits;
} hcblas_half_t;

/* Device memory and copies behind hc::am_alloc / am_free / copy. */
void *hcblas_am_alloc(size_t bytes, int device_id, unsigned flags);
int hcblas_am_free(void *ptr);
int hcblas_am_copy(hcblas_accl_view_t view, const void *src, void *dst, size_t bytes);
int hcblas_view_wait(hcblas_accl_view_t view);
int hcblas_device_count(void);
int hcblas_current_device(void);

#ifdef __cplusplus
} /* extern "C" */

#include <vector>

namespace hc {

class accelerator_view;

/* A CUDA device. */
class accelerator {
 public:
  accelerator() : device_id_(hcblas_current_device()) {}
  explicit accelerator(int device_id) : device_id_(device_id) {}
  int get_device_id() const { return device_id_; }
  inline accelerator_view get_default_view() const;
  bool operator==(const accelerator &o) const { return device_id_ == o.device_id_; }
  bool operator!=(const accelerator &o) const { return device_id_ != o.device_id_; }
  static std::vector<accelerator> get_all() {
    std::vector<accelerator> v;
    int n = hcblas_device_count();
    for (int i = 0; i < n; ++i) v.push_back(accelerator(i));
    return v;
  }

 private:
  int device_id_;
};

/* A stream on a device; layout-compatible with hcblas_accl_view_t. */
class accelerator_view : public hcblas_accl_view_t {
 public:
  accelerator_view() {
    device_id = hcblas_current_device();
    stream = nullptr;
  }
  accelerator_view(int dev, void *s) {
    device_id = dev;
    stream = s;
  }
  accelerator get_accelerator() const { return accelerator(device_id); }
  /* Enqueue a copy (host<->device or device<->device) on this view, then
   * wait for it, as HCC's accelerator_view::copy does. */
  void copy(const void *src, void *dst, size_t bytes) const {
    hcblas_am_copy(*this, src, dst, bytes);
  }
  void wait() const { hcblas_view_wait(*this); }
};

inline accelerator_view accelerator::get_default_view() const {
  return accelerator_view(device_id_, nullptr);
}

/* Device allocation in the style of hc::am_alloc: the result converts to any
 * pointer type. */
struct am_voidp {
  void *p;
  template <typename T> operator T *() const { return static_cast<T *>(p); }
};
inline am_voidp am_alloc(size_t bytes, const accelerator &acc, unsigned flags) {
  return am_voidp{hcblas_am_alloc(bytes, acc.get_device_id(), flags)};
}
inline int am_free(void *p) { return hcblas_am_free(p); }

/* IEEE binary16 value (round-to-nearest-even conversions written from the
 * IEEE 754 encoding). */
struct half : public hcblas_half_t {
  half() { bits = 0; }
  half(float f) { bits = from_float(f); }
  half(double d) { bits = from_float(static_cast<float>(d)); }
  half(int i) { bits = from_float(static_cast<float>(i)); }
  operator float() const { return to_float(bits); }
  static half from_bits(uint16_t b) {
    half h;
    h.bits = b;
    return h;
  }

  static float to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t out;
    if (exp == 0) {
      if (man == 0) {
        out = sign;
      } else { /* subnormal: normalise */
        int e = -1;
        do {
          ++e;
          man <<= 1;
        } while ((man & 0x400u) == 0);
        man &= 0x3ffu;
        out = sign | ((uint32_t)(127 - 15 - e) << 23) | (man << 13);
      }
    } else if (exp == 31) {
      out = sign | 0x7f800000u | (man << 13);
    } else {
      out = sign | ((exp + 112u) << 23) | (man << 13);
    }
    float f;
    __builtin_memcpy(&f, &out, 4);
    return f;
  }

  static uint16_t from_float(float f) {
    uint32_t x;
    __builtin_memcpy(&x, &f, 4);
    const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
    const uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) /* inf or nan */
      return sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u);
    if (ax >= 0x477ff000u) return sign | 0x7c00u; /* rounds to >= 65520 -> inf */
    if (ax < 0x33000001u) return sign;            /* < 2^-25 (ties to 0) */
    int e = (int)(ax >> 23) - 127;
    uint32_t man = (ax & 0x7fffffu) | 0x800000u; /* 24-bit significand */
    int shift;                                    /* bits to drop */
    uint16_t base;
    if (e < -14) { /* half subnormal */
      shift = 13 + (-14 - e);
      base = 0;
    } else {
      shift = 13;
      base = (uint16_t)((e + 15) << 10);
      man &= 0x7fffffu; /* implicit bit handled by exponent field */
    }
    uint32_t q = man >> shift;
    const uint32_t rem = man & ((1u << shift) - 1u);
    const uint32_t halfway = 1u << (shift - 1);
    if (rem > halfway || (rem == halfway && (q & 1u))) ++q;
    /* carry from the significand into the exponent is the correct result */
    return sign | (uint16_t)(base + q);
  }
};

namespace short_vector {
struct float_2 {
  float x, y;
  float_2() : x(0), y(0) {}
  float_2(float a, float b) : x(a), y(b) {}
};
struct double_2 {
  double x, y;
  double_2() : x(0), y(0) {}
  double_2(double a, double b) : x(a), y(b) {}
};
typedef float_2 float2;
typedef double_2 double2;
}  // namespace short_vector

}  // namespace hc

#endif /* __cplusplus */

#endif /* HCBLAS_B200_HC_COMPAT_H_ */
