// f16.h -- float <-> half conversion of the scene packer, usable in host and
// device code: round to nearest with ties away from zero on the magnitude
// bits, as the reference's host conversion does (Utils/Math/Float16.cpp:56-169),
// so that materials packed on the device equal those packed on the host.
#pragma once

#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define F16_HD __host__ __device__ __forceinline__
#else
#define F16_HD inline
#endif

namespace fpt {

F16_HD uint16_t f32_to_f16_bits(float value) {
    uint32_t bits;
#if defined(__CUDA_ARCH__)
    bits = __float_as_uint(value);
#else
    std::memcpy(&bits, &value, 4);
#endif
    const int32_t sign = int32_t((bits >> 16) & 0x8000u);
    int32_t exp = int32_t((bits >> 23) & 0xffu) - (127 - 15);
    int32_t man = int32_t(bits & 0x007fffffu);
    if (exp <= 0) {
        if (exp < -10) return uint16_t(sign);
        man = (man | 0x00800000) >> (1 - exp);
        if (man & 0x00001000) man += 0x00002000;
        return uint16_t(sign | (man >> 13));
    }
    if (exp == 0xff - (127 - 15)) {
        if (man == 0) return uint16_t(sign | 0x7c00);
        man >>= 13;
        return uint16_t(sign | 0x7c00 | man | (man == 0));
    }
    if (man & 0x00001000) {
        man += 0x00002000;
        if (man & 0x00800000) {
            man = 0;
            exp += 1;
        }
    }
    if (exp > 30) return uint16_t(sign | 0x7c00);
    return uint16_t(sign | (exp << 10) | (man >> 13));
}

}  // namespace fpt
