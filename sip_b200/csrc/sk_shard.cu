// Instantiations of the size-specialized kernels of one shard of
// sk_configs.h (the build compiles this file once per shard with
// -DSIP_SK_SHARD=<i>).
#include "sk_configs.h"
#include "sk_kernel.cuh"
#include "sk_registry.h"

#ifndef SIP_SK_SHARD
#error "SIP_SK_SHARD must be defined"
#endif

namespace sipfft {

namespace {

template <class K, int STAGES>
SkEntry make_entry(std::vector<int> radices) {
    SkEntry e;
    e.n = K::N;
    e.P = K::P;
    e.T = K::T;
    e.op = K::OP;
    e.mode = K::MODE;
    e.sign = K::SIGN;
    e.tw4 = K::TW4;
    e.twb = K::TWB;
    e.flags = K::FLAGS;
    e.stages = STAGES;
    e.radices = std::move(radices);
    e.LD = K::LD;
    e.smem = (STAGES == 2 ? 2 : 1) * K::BUF * 8 + K::TWSM * 8;
    e.fn = reinterpret_cast<const void*>(&sk_fft_kernel<K, STAGES>);
    e.minb = K::MINB;
    return e;
}

// Registers this shard's entries, each with its position in the
// SIP_SK_CONFIGS list (the registry is ordered by it).
template <int SHARD>
void register_shard(std::vector<SkEntry>& out) {
    int order = 0;
#define SIP_SK_ENTRY(S, N, P, T, OP, MODE, SIGN, TW4, STAGES, MINB, TWB, ...)                                  \
    if constexpr (S == SHARD) {                                                                                   \
        out.push_back(make_entry<SkCfg<N, P, T, OP, MODE, SIGN, TW4, MINB, TWB, __VA_ARGS__>, STAGES>({__VA_ARGS__})); \
        out.back().order = order;                                                                                 \
    }                                                                                                             \
    ++order;
    SIP_SK_CONFIGS(SIP_SK_ENTRY)
#undef SIP_SK_ENTRY
}

}  // namespace

#define SIP_CAT2(a, b) a##b
#define SIP_CAT(a, b) SIP_CAT2(a, b)

void SIP_CAT(sk_register_shard_, SIP_SK_SHARD)(std::vector<SkEntry>& out) { register_shard<SIP_SK_SHARD>(out); }

}  // namespace sipfft
