// Shared scalar helpers of the CPU oracle (test infrastructure only).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace orc {

// MACHINE_EPSILON = f32::EPSILON * 0.5 (core/pbrt.rs:23)
static const float kMachineEps = std::numeric_limits<float>::epsilon() * 0.5f;
static const float kPi = 3.14159265358979323846f;

// gamma(n) (core/pbrt.rs:172-174)
static inline float gamma(int n) {
    return ((float)n * kMachineEps) / (1.0f - (float)n * kMachineEps);
}

static inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// next_float_up (core/pbrt.rs:129-147)
static inline float next_float_up(float v) {
    if (std::isinf(v) && v > 0.0f) return v;
    float nv = (v == -0.0f) ? 0.0f : v;   // -0.0 == 0.0, so both zeros map to +0
    uint32_t ui = f2u(nv);
    if (nv >= 0.0f) ++ui; else --ui;
    return u2f(ui);
}
// next_float_down (core/pbrt.rs:151-169)
static inline float next_float_down(float v) {
    if (std::isinf(v) && v < 0.0f) return v;
    float nv = (v == 0.0f) ? -0.0f : v;
    uint32_t ui = f2u(nv);
    if (nv > 0.0f) --ui; else ++ui;
    return u2f(ui);
}

// PCG32 (core/rng.rs:9-63); advance() with D18 repaired (loop while delta>0,
// wrapping arithmetic).
struct Rng {
    uint64_t state = 0x853c49e6748fea9bULL, inc = 0xda3e39cb94b95bdbULL;
    static constexpr uint64_t kMult = 0x5851f42d4c957f2dULL;
    explicit Rng(uint64_t seq) { set_sequence(seq); }
    void set_sequence(uint64_t initseq) {          // rng.rs:30-36
        state = 0;
        inc = (initseq << 1) | 1;
        uniform_u32();
        state += 0x853c49e6748fea9bULL;
        uniform_u32();
    }
    uint32_t uniform_u32() {                       // rng.rs:38-49
        uint64_t old = state;
        state = old * kMult + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
    }
    float uniform_float() {                        // rng.rs:60-63
        float f = (float)uniform_u32() * 0x1p-32f;
        const float one_minus_eps = 0x1.fffffep-1f;
        return f < one_minus_eps ? f : one_minus_eps;
    }
    void advance(int64_t idelta) {                 // rng.rs:65-82, D18
        uint64_t cur_mult = kMult, cur_plus = inc, acc_mult = 1, acc_plus = 0;
        uint64_t delta = (uint64_t)idelta;
        while (delta > 0) {
            if (delta & 1) { acc_mult *= cur_mult; acc_plus = acc_plus * cur_mult + cur_plus; }
            cur_plus = (cur_mult + 1) * cur_plus;
            cur_mult *= cur_mult;
            delta /= 2;
        }
        state = acc_mult * state + acc_plus;
    }
};

}  // namespace orc
