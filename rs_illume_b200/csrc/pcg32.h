// PCG32 with the constants, seeding and float mapping of rs_illume's Rng
// (src/core/rng.rs:9-82): set_sequence (30-36), uniform_uint32 (38-49),
// uniform_float = min(u32 * 2^-32, 1 - 2^-24) (60-63).  advance() uses the
// standard LCG jump-ahead with wrapping arithmetic (the reference's loop bound
// `delta > 1` and non-wrapping multiplies are a bug; this is the repaired
// form).  Usable from host and device code.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define ILM_HD __host__ __device__ __forceinline__
#else
#define ILM_HD inline
#endif

namespace ilm {

struct Pcg32 {
    uint64_t state, inc;
    static constexpr uint64_t kMult = 0x5851f42d4c957f2dULL;
    static constexpr uint64_t kDefaultState = 0x853c49e6748fea9bULL;

    ILM_HD Pcg32() : state(kDefaultState), inc(0xda3e39cb94b95bdbULL) {}
    ILM_HD explicit Pcg32(uint64_t seq) { set_sequence(seq); }

    ILM_HD void set_sequence(uint64_t initseq) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        uniform_u32();
        state += kDefaultState;
        uniform_u32();
    }
    ILM_HD uint32_t uniform_u32() {
        uint64_t old = state;
        state = old * kMult + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((~rot + 1u) & 31u));
    }
    ILM_HD float uniform_float() {
        float f = (float)uniform_u32() * 0x1p-32f;
        const float kOneMinusEps = 0x1.fffffep-1f;
        return f < kOneMinusEps ? f : kOneMinusEps;
    }
    ILM_HD void advance(uint64_t delta) {
        uint64_t cur_mult = kMult, cur_plus = inc, acc_mult = 1u, acc_plus = 0u;
        while (delta > 0) {
            if (delta & 1u) {
                acc_mult *= cur_mult;
                acc_plus = acc_plus * cur_mult + cur_plus;
            }
            cur_plus = (cur_mult + 1u) * cur_plus;
            cur_mult *= cur_mult;
            delta >>= 1u;
        }
        state = acc_mult * state + acc_plus;
    }
};

}  // namespace ilm
