// tracker_common.cuh -- register-level pieces of the streaming trackers
// (tracker_stream.cu, and the served batch in serve_kernels.cu): the int4 ->
// fp16 decode, the m16n8k16 MMA, and the FP64-phase steering weight.
#pragma once

#include <cuda_fp16.h>

#include "bf_internal.cuh"

namespace bf {
namespace trk {

__device__ __forceinline__ uint32_t lop3_and_xor(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm("lop3.b32 %0, %1, %2, %3, 0x6A;" : "=r"(r) : "r"(a), "r"(b), "r"(c));  // (a & b) ^ c
    return r;
}

__device__ __forceinline__ uint32_t h2_bits(__half2 h) {
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ __half2 bits_h2(uint32_t u) {
    return *reinterpret_cast<__half2*>(&u);
}

// Decode one 32-bit word (bytes b0..b3) into four fp16 pairs:
//   re02 = (re b0, re b2), im02 = (im b0, im b2), re13, im13.
__device__ __forceinline__ void decode_word(uint32_t w, uint32_t& re02, uint32_t& im02,
                                            uint32_t& re13, uint32_t& im13) {
    const __half2 bias_lo = __floats2half2_rn(1032.0f, 1032.0f);
    const __half2 sixteenth = __floats2half2_rn(0.0625f, 0.0625f);
    const __half2 bias_hi = __floats2half2_rn(-72.0f, -72.0f);
    const uint32_t w1 = w >> 8;
    re02 = h2_bits(__hsub2(bits_h2(lop3_and_xor(w, 0x000F000Fu, 0x64086408u)), bias_lo));
    im02 = h2_bits(__hfma2(bits_h2(lop3_and_xor(w, 0x00F000F0u, 0x64806480u)), sixteenth, bias_hi));
    re13 = h2_bits(__hsub2(bits_h2(lop3_and_xor(w1, 0x000F000Fu, 0x64086408u)), bias_lo));
    im13 = h2_bits(__hfma2(bits_h2(lop3_and_xor(w1, 0x00F000F0u, 0x64806480u)), sixteenth, bias_hi));
}

__device__ __forceinline__ void mma_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                          uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Steering weight w = exp(i * k * (p . d)) in two steps: the FP64 delay
// p . d (shared by all channels of a direction), then the FP64 phase
// k * delay reduced to a quadrant n and r = phase - n pi / 2 in [-pi/4, pi/4]
// (one fused multiply-add), and sin r, cos r from their Taylor series
// through r^11 and r^12 (truncation error below 3e-11 on the interval)
// evaluated in FP32 by Horner's rule.  Every operation is an explicitly
// rounded intrinsic, so any kernel that composes these two gets
// bit-identical weights.
__device__ __forceinline__ float2 sincos_quadrant(float r, int quad) {
    const float r2 = __fmul_rn(r, r);
    float ps = -2.5052108385441718775e-8f;               // -1/11!
    ps = __fmaf_rn(ps, r2, 2.7557319223985890653e-6f);   //  1/9!
    ps = __fmaf_rn(ps, r2, -1.9841269841269841270e-4f);  // -1/7!
    ps = __fmaf_rn(ps, r2, 8.3333333333333333333e-3f);   //  1/5!
    ps = __fmaf_rn(ps, r2, -1.6666666666666666667e-1f);  // -1/3!
    const float sn = __fmaf_rn(__fmul_rn(ps, r2), r, r);
    float pc = 2.0876756987868098979e-9f;                //  1/12!
    pc = __fmaf_rn(pc, r2, -2.7557319223985890653e-7f);  // -1/10!
    pc = __fmaf_rn(pc, r2, 2.4801587301587301587e-5f);   //  1/8!
    pc = __fmaf_rn(pc, r2, -1.3888888888888888889e-3f);  // -1/6!
    pc = __fmaf_rn(pc, r2, 4.1666666666666666667e-2f);   //  1/4!
    pc = __fmaf_rn(pc, r2, -0.5f);
    const float cs = __fmaf_rn(pc, r2, 1.0f);
    // (cos, sin) of n pi / 2 + r: quadrants 1 and 3 swap, 1 and 2 negate
    // cos, 2 and 3 negate sin
    const float c1 = (quad & 1) != 0 ? sn : cs;
    const float s1 = (quad & 1) != 0 ? cs : sn;
    return make_float2(quad == 1 || quad == 2 ? -c1 : c1, (quad & 2) != 0 ? -s1 : s1);
}
__device__ __forceinline__ double steering_delay(const float* pos, int a, double dx, double dy, double dz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(static_cast<double>(pos[3 * a]), dx),
                               __dmul_rn(static_cast<double>(pos[3 * a + 1]), dy)),
                     __dmul_rn(static_cast<double>(pos[3 * a + 2]), dz));
}
// n = rint(x) and n mod 4.  Below 2^51 in magnitude, x + 1.5 * 2^52 lands
// where the ulp is 1, so the addition rounds x to an integer exactly as rint
// does (to nearest, ties to even) and the low bits of the sum hold n mod 4
// (1.5 * 2^52 is a multiple of 4): two additions instead of a rounding and a
// 64-bit conversion.  Larger |x| takes rint.
__device__ __forceinline__ double round_quadrant(double x, int& quad) {
    constexpr double kShift = 6755399441055744.0;  // 1.5 * 2^52
    if (fabs(x) < 0x1p51) {
        const double s = __dadd_rn(x, kShift);
        quad = __double2loint(s) & 3;
        return __dsub_rn(s, kShift);
    }
    const double n = rint(x);
    quad = static_cast<int>(static_cast<long long>(n) & 3);
    return n;
}
__device__ __forceinline__ float2 steering_from_delay(double k, double delay) {
    constexpr double kHalfPi = 1.5707963267948966192313216916398;
    constexpr double kTwoOverPi = 0.63661977236758134307553505349006;
    const double phase = __dmul_rn(k, delay);
    int quad;
    const double n = round_quadrant(__dmul_rn(phase, kTwoOverPi), quad);
    const float r = __double2float_rn(__fma_rn(-kHalfPi, n, phase));
    return sincos_quadrant(r, quad);
}
__device__ __forceinline__ float2 steering_weight(const float* pos, int a, double k, double dx,
                                                  double dy, double dz) {
    return steering_from_delay(k, steering_delay(pos, a, dx, dy, dz));
}

__device__ __forceinline__ uint16_t split_part(float c, bool lo) {
    const __half h = __float2half_rn(c);
    if (!lo) return __half_as_ushort(h);
    return __half_as_ushort(__float2half_rn(c - __half2float(h)));
}

}  // namespace trk
}  // namespace bf
