// CPU harness for the FFT kernels (test infrastructure only).
//
// Builds a plan with the library's own planner (sip_b200/csrc/plan.cpp)
// and runs every step on the host by calling the kernels' own
// __host__ __device__ phase functions (tile_io.cuh loads/stores,
// fft_core.cuh pass_read / pass_write, real_math.cuh) for every thread
// index of every tile, with a barrier between phases emulated by running
// each phase for all threads before the next.  This checks the planner,
// the index arithmetic and the butterflies against numpy without a GPU.
// Shared memory is filled with NaN before each tile so a read of a slot no
// phase wrote shows up in the result.  Twiddles are computed on the host
// in long double and rounded once to float.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "plan.h"
#include "real_math.cuh"
#include "sk_configs.h"
#include "sk_kernel.cuh"
#include "cluster_configs.h"
#include "tc_core.cuh"

using namespace sipfft;

namespace {

float2 root_host(long long m, long long n) {
    m %= n;
    if (m < 0) m += n;
    const long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
    return make_float2((float)std::cos(a), (float)(-std::sin(a)));
}

std::vector<float2> stockham_host(const PlanDev& pd) {
    int entries = 0;
    for (int i = 0; i < pd.npass; ++i)
        if (pd.pass[i].L > 1) entries = pd.pass[i].tw + pd.pass[i].L * (pd.pass[i].R - 1);
    std::vector<float2> t(std::max(entries, 1));
    for (int i = 0; i < pd.npass; ++i) {
        const PassDesc& p = pd.pass[i];
        if (p.L <= 1) continue;
        for (int k = 0; k < p.L; ++k)
            for (int r = 1; r < p.R; ++r) t[p.tw + (r - 1) * p.L + k] = root_host((long long)r * k, (long long)p.L * p.R);
    }
    return t;
}

// Bluestein chirp c_j = exp(s i pi (j^2 mod 2n) / n), j < n (bluestein.cuh).
std::vector<float2> chirp_host(long long n, int sign) {
    std::vector<float2> chirp(n);
    for (long long j = 0; j < n; ++j) {
        const long long q = (j * j) % (2 * n);
        const long double a = 3.141592653589793238462643383279502884L * (long double)q / (long double)n;
        chirp[j] = make_float2((float)std::cos(a), (float)(sign * std::sin(a)));
    }
    return chirp;
}

// Second table of a step: roots W_n^k (kind 1), the split cross-twiddle
// table of four-step passes (kind 2, tile_io.cuh cross_tw) or the Bluestein
// chirp of a fused Bluestein tile (kind 3).
std::vector<float2> tw2_host(const Step& st) {
    std::vector<float2> t;
    if (st.tw2_kind == 3) return chirp_host(st.blue_n, st.blue_sign);
    if (st.tw2_kind == 1) {
        for (long long k = 0; k < st.tw2_count; ++k) t.push_back(root_host(k, st.tw2_n));
    } else if (st.tw2_kind == 2) {
        const long long B = 1LL << st.L.args.tw4_shift;
        for (long long k = 0; k < st.tw2_count; ++k) t.push_back(root_host(k < B ? k : (k - B) * B, st.tw2_n));
    }
    return t;
}

// Basis twiddle table of the size-specialized kernels (fft_core.cuh basis_split).
std::vector<float2> basis_host(const std::vector<int>& radices) {
    std::vector<float2> t;
    int L = 1;
    for (int R : radices) {
        if (L > 1) {
            const int a = basis_split(R);
            for (int r = 1; r < a; ++r)
                for (int k = 0; k < L; ++k) t.push_back(root_host((long long)r * k, (long long)L * R));
            for (int h = 1; h < R / a; ++h)
                for (int k = 0; k < L; ++k) t.push_back(root_host((long long)a * h * k, (long long)L * R));
        }
        L *= R;
    }
    if (t.empty()) t.push_back(make_float2(1.f, 0.f));
    return t;
}

template <int R, int SIGN, int S>
void emu_pass(int T, const TileArgs& a, float2* sm, const PassDesc& pd) {
    std::vector<PassRegs<R, S>> regs(T);
    for (int tid = 0; tid < T; ++tid) pass_read<R, SIGN, S>(tid, T, a.P, a.N, sm, a.LD, pd, a.tw, regs[tid]);
    for (int tid = 0; tid < T; ++tid) pass_write<R, S>(tid, T, a.P, sm, a.LD, pd, regs[tid]);
}

template <int SIGN, int E>
void emu_passes(int T, const TileArgs& a, float2* sm) {
    for (int i = 0; i < a.plan->npass; ++i) {
        const PassDesc& pd = a.plan->pass[i];
        switch (pd.R) {
#define SIP_EMU_CASE(R)                               \
    case R:                                           \
        emu_pass<R, SIGN, cdiv(E, R)>(T, a, sm, pd);  \
        break;
            SIP_FFT_FOR_EACH_RADIX(SIP_EMU_CASE)
#undef SIP_EMU_CASE
            default:
                throw std::runtime_error("radix without a pass");
        }
    }
}

// ---- size-specialized kernels: the same SkPass phase functions per thread
template <class K, int PASS>
void emu_sk_passes(const TileArgs& a, const TileCtx& c, float2* buf) {
    using SP = SkPass<K, PASS>;
    if constexpr (K::MPAIR && K::OP == OP_R2C_HALF && SP::LAST) {
        for (int tid = 0; tid < K::T; ++tid) sk_pair_last_r2c<K>(tid, a, c, buf);
    } else if constexpr (K::MPAIR && K::OP == OP_R2C_PAIR && SP::LAST) {
        for (int tid = 0; tid < K::T; ++tid) sk_pair_last_r2c_rows<K>(tid, a, c, buf);
    } else if constexpr (K::MPAIR && K::OP == OP_R2C_4B && SP::LAST) {
        for (int tid = 0; tid < K::T; ++tid) sk_pair_last_r2c_4b<K>(tid, a, c, buf);
    } else if constexpr (K::MPAIR && K::OP == OP_C2R_4A && PASS == 0) {
        using PP = SkPairFirstC2R4A<K>;
        std::vector<typename PP::Regs> regs(K::T);
        for (int tid = 0; tid < K::T; ++tid) PP::read(tid, a, c, buf, regs[tid]);
        for (int tid = 0; tid < K::T; ++tid) PP::write_smem(tid, a, c, buf, regs[tid]);
        emu_sk_passes<K, 1>(a, c, buf);
    } else if constexpr (K::MPAIR && (K::OP == OP_C2R_HALF || K::OP == OP_C2R_PAIR) && PASS == 0) {
        using PP = typename SkPick<K::OP == OP_C2R_HALF, SkPairFirstC2R<K>, SkPairFirstC2RRows<K>>::type;
        std::vector<typename PP::Regs> regs(K::T);
        for (int tid = 0; tid < K::T; ++tid) PP::read(tid, a, c, buf, regs[tid]);
        for (int tid = 0; tid < K::T; ++tid) PP::write_smem(tid, buf, regs[tid]);
        emu_sk_passes<K, 1>(a, c, buf);
    } else {
        std::vector<typename SP::Regs> regs(K::T);
        for (int tid = 0; tid < K::T; ++tid) SP::read(tid, a, c, buf, regs[tid]);
        if constexpr (SP::LAST && !sk_last_to_smem<K>()) {
            for (int tid = 0; tid < K::T; ++tid) SP::write_global(tid, a, c, regs[tid]);
        } else {
            for (int tid = 0; tid < K::T; ++tid) SP::write_smem(tid, buf, regs[tid]);
            if constexpr (!SP::LAST) emu_sk_passes<K, PASS + 1>(a, c, buf);
        }
    }
}

template <class K>
void emu_sk_run(const TileArgs& a) {
    const float nan = std::numeric_limits<float>::quiet_NaN();
    std::vector<float2> buf(K::BUF);
    // staged twiddles (SK_TW_SMEM), NaN where the copy does not write
    std::vector<float2> tws(K::TWSM + 1, make_float2(nan, nan));
    for (int tid = 0; tid < K::T; ++tid) sk_load_tws<K>(tid, a, tws.data());
    for (int tile = 0; tile < a.ntiles; ++tile) {
        TileCtx c = decode_tile(a, tile);
        if constexpr (K::TWS) c.tws = tws.data();
        for (auto& v : buf) v = make_float2(nan, nan);
        for (int tid = 0; tid < K::T; ++tid) sk_stage<K>(tid, a, c, buf.data());
        for (int tid = 0; tid < K::T; ++tid) sk_zero_missing<K>(tid, a, c, buf.data());
        if constexpr (K::SPLIT) {  // pass 0 from the staging buffer into a separate work buffer
            std::vector<float2> work(K::BUF, make_float2(nan, nan));
            for (int tid = 0; tid < K::T; ++tid) sk_pass0_split<K>(tid, a, c, buf.data(), work.data());
            emu_sk_passes<K, 1>(a, c, work.data());
            if constexpr (sk_last_to_smem<K>())
                for (int tid = 0; tid < K::T; ++tid) sk_post<K>(tid, a, c, work.data());
            continue;
        }
        if constexpr (K::OP == OP_PC) {
            emu_sk_passes<SkView<K, OP_PC, -1, false>, 0>(a, c, buf.data());
            for (int tid = 0; tid < K::T; ++tid) sk_mul<K>(tid, a, c, buf.data());
            emu_sk_passes<SkView<K, OP_C2C, 1, true>, 0>(a, c, buf.data());
            continue;
        }
        emu_sk_passes<K, 0>(a, c, buf.data());
        if constexpr (sk_last_to_smem<K>())
            for (int tid = 0; tid < K::T; ++tid) sk_post<K>(tid, a, c, buf.data());
    }
}

using EmuSkFn = void (*)(const TileArgs&);

// ---- cluster four-step: the kernel's phases rank by rank, the cluster's
// shared memories as host vectors
template <class CC, int PASS>
void emu_cl_passes_a(const TileArgs& a, const TileCtx& c, float2* buf, float2* rows) {
    using SP = SkPass<typename CC::KA, PASS>;
    std::vector<typename SP::Regs> regs(CC::T);
    for (int tid = 0; tid < CC::T; ++tid) SP::read(tid, a, c, buf, regs[tid]);
    if constexpr (SP::LAST) {
        for (int tid = 0; tid < CC::T; ++tid) cl_pass_a_write_rows<CC, PASS>(tid, rows, regs[tid]);
    } else {
        for (int tid = 0; tid < CC::T; ++tid) SP::write_smem(tid, buf, regs[tid]);
        emu_cl_passes_a<CC, PASS + 1>(a, c, buf, rows);
    }
}

template <class CC>
void emu_cluster_run(const TileArgs& a, const TileArgs& b, long long transforms) {
    const float nan = std::numeric_limits<float>::quiet_NaN();
    for (long long tr = 0; tr < transforms; ++tr) {
        std::vector<std::vector<float2>> rows(CC::C, std::vector<float2>(CC::N1 * CC::PA, make_float2(nan, nan)));
        for (int r = 0; r < CC::C; ++r) {
            std::vector<float2> abuf(CC::KA::BUF, make_float2(nan, nan));
            TileCtx ca;
            ca.i0 = r * CC::PA;
            ca.cnt = CC::PA;
            ca.in_base = tr * CC::N + ca.i0;
            ca.out_base = 0;
            for (int tid = 0; tid < CC::T; ++tid) sk_stage<typename CC::KA>(tid, a, ca, abuf.data());
            emu_cl_passes_a<CC, 0>(a, ca, abuf.data(), rows[r].data());
        }
        for (int r = 0; r < CC::C; ++r) {
            std::vector<float2> bbuf(CC::KB::BUF, make_float2(nan, nan));
            for (int tid = 0; tid < CC::T; ++tid)
                cl_gather<CC>(tid, b, r, [&](int p) -> const float2* { return rows[p].data(); }, bbuf.data());
            TileCtx cb;
            cb.i0 = r * CC::PB;
            cb.cnt = CC::PB;
            cb.in_base = 0;
            cb.out_base = tr * CC::N + cb.i0;
            emu_sk_passes<typename CC::KB, 0>(b, cb, bbuf.data());
        }
    }
}

using EmuClFn = void (*)(const TileArgs&, const TileArgs&, long long);

template <class K>
std::vector<int> emu_radices_of() {
    std::vector<int> r;
    for (int p = 0; p < K::NP; ++p) r.push_back(K::radix(p));
    return r;
}

template <class CC>
ClEntry emu_cl_entry() {
    ClEntry e;
    e.n = CC::N;
    e.n1 = CC::N1;
    e.n2 = CC::N2;
    e.C = CC::C;
    e.T = CC::T;
    e.sign = CC::SIGN;
    e.pa = CC::PA;
    e.pb = CC::PB;
    e.ra = emu_radices_of<typename CC::KA>();
    e.rb = emu_radices_of<typename CC::KB>();
    e.smem = CC::SMEM_VALUES * 8;
    e.fn = reinterpret_cast<const void*>(&emu_cluster_run<CC>);
    return e;
}

template <class K, int STAGES>
SkEntry emu_entry(std::vector<int> radices) {
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
    e.fn = reinterpret_cast<const void*>(&emu_sk_run<K>);
    return e;
}

}  // namespace

namespace sipfft {
const std::vector<SkEntry>& sk_registry() {
    static const std::vector<SkEntry> reg = [] {
        std::vector<SkEntry> v;
#define SIP_EMU_SK(S, N, P, T, OP, MODE, SIGN, TW4, STAGES, MINB, TWB, ...) \
    v.push_back(emu_entry<SkCfg<N, P, T, OP, MODE, SIGN, TW4, MINB, TWB, __VA_ARGS__>, STAGES>({__VA_ARGS__}));
        SIP_SK_CONFIGS(SIP_EMU_SK)
        // Pulse-compression tiles (the library compiles these at run time,
        // csrc/jit.cpp): rows of 1000, Bluestein's 2025 for n = 1009, and the
        // four-step pass P (cross twiddles) of 2^18 = 512 x 512 and of
        // Bluestein's 40500 = 180 x 225 for n = 20011.
        SIP_EMU_SK(0, 1000, 4, 128, OP_PC, SK_ROWS, 1, false, 2, 4, 1, 10, 10, 10)
        SIP_EMU_SK(0, 2025, 2, 192, OP_PC, SK_ROWS, 1, false, 2, 2, 1, 15, 15, 9)
        SIP_EMU_SK(0, 512, 8, 256, OP_PC, SK_ROWS, 1, true, 2, 2, 1, 32, 16)
        SIP_EMU_SK(0, 225, 16, 256, OP_PC, SK_ROWS, 1, true, 2, 2, 1, 15, 15)
#undef SIP_EMU_SK
        return v;
    }();
    return reg;
}
const SkEntry* sk_find(int op, int mode, int sign, bool tw4, int n, int variant) {
    if (std::getenv("SIP_EMU_GENERIC_ONLY")) return nullptr;
    if (variant < 0) variant = 0;
    const SkEntry* first = nullptr;
    for (const SkEntry& e : sk_registry()) {
        if (e.op != op || e.mode != mode || e.sign != sign || e.tw4 != tw4 || e.n != n) continue;
        if (first == nullptr) first = &e;
        if (variant-- == 0) return &e;
    }
    return first;
}
const SkEntry* sk_find_flags(int op, int mode, int sign, bool tw4, int n, int flags) {
    for (const SkEntry& x : sk_registry())
        if (x.op == op && x.mode == mode && x.sign == sign && x.tw4 == tw4 && x.n == n && (x.flags & flags) == flags)
            return &x;
    return nullptr;
}
const SkEntry* sk_find_wider(const SkEntry* e) {
    for (const SkEntry& x : sk_registry())
        if (x.op == e->op && x.mode == e->mode && x.sign == e->sign && x.tw4 == e->tw4 && x.n == e->n &&
            x.P == e->P && x.T > e->T)
            return &x;
    return nullptr;
}
const ClEntry* cluster_find(int n, int sign) {
    static const std::vector<ClEntry> reg = [] {
        std::vector<ClEntry> v;
#define SIP_EMU_CL(CC) v.push_back(emu_cl_entry<CC>());
        SIP_CL_CONFIGS(SIP_EMU_CL)
#undef SIP_EMU_CL
        return v;
    }();
    for (const ClEntry& e : reg)
        if (e.n == n && e.sign == sign) return &e;
    return nullptr;
}
// The harness runs only the kernels it instantiates: no run-time compiled ones.
const SkEntry* sk_jit_entry(int, int, int, bool, int, long long, bool) { return nullptr; }
bool sk_jit_available() { return false; }
bool sk_jit_wait(long long) { return true; }
}  // namespace sipfft

namespace {

void emu_tile_step(const Step& st, const void* src, void* dst) {
    TileArgs a = st.L.args;
    a.src = src;
    a.dst = dst;
    a.plan = &st.host_plan;
    std::vector<float2> tw = (st.sk && st.sk->twb) ? basis_host(st.radices) : stockham_host(st.host_plan);
    std::vector<float2> tw2 = tw2_host(st);
    a.tw = tw.data();
    a.tw2 = tw2.empty() ? nullptr : tw2.data();
    if (st.sk != nullptr) {
        reinterpret_cast<EmuSkFn>(const_cast<void*>(st.sk->fn))(a);
        return;
    }
    const int T = st.L.block;
    const float nan = std::numeric_limits<float>::quiet_NaN();
    std::vector<float2> smv((size_t)a.P * a.LD);
    float2* sm = smv.data();
    for (int tile = 0; tile < a.ntiles; ++tile) {
        const TileCtx c = decode_tile(a, tile);
        for (auto& v : smv) v = make_float2(nan, nan);
        for (int tid = 0; tid < T; ++tid) {
            switch (st.L.op) {
                case OP_C2C:
                case OP_PC: load_c2c(tid, T, a, c, sm); break;
                case OP_R2C_HALF: load_r2c_half(tid, T, a, c, sm); break;
                case OP_C2R_HALF: load_c2r_half(tid, T, a, c, sm); break;
                case OP_R2C_PAIR: load_r2c_pair(tid, T, a, c, sm); break;
                case OP_C2R_PAIR: load_c2r_pair(tid, T, a, c, sm); break;
            }
        }
        if (st.L.op == OP_C2R_HALF)
            for (int tid = 0; tid < T; ++tid) prep_c2r_half(tid, T, a, c, sm);
        if (st.L.op == OP_PC) {
            if (st.L.e == 16) emu_passes<-1, 16>(T, a, sm); else emu_passes<-1, 32>(T, a, sm);
            for (int tid = 0; tid < T; ++tid) mul_tile(tid, T, a, c, sm);
            if (st.L.e == 16) emu_passes<1, 16>(T, a, sm); else emu_passes<1, 32>(T, a, sm);
        } else if (st.L.sign < 0) {
            if (st.L.e == 16) emu_passes<-1, 16>(T, a, sm); else emu_passes<-1, 32>(T, a, sm);
        } else {
            if (st.L.e == 16) emu_passes<1, 16>(T, a, sm); else emu_passes<1, 32>(T, a, sm);
        }
        for (int tid = 0; tid < T; ++tid) {
            switch (st.L.op) {
                case OP_PC:
                case OP_C2C:
                    if (st.L.sign < 0) {
                        if (st.L.tw4) store_c2c<-1, true>(tid, T, a, c, sm); else store_c2c<-1, false>(tid, T, a, c, sm);
                    } else {
                        if (st.L.tw4) store_c2c<1, true>(tid, T, a, c, sm); else store_c2c<1, false>(tid, T, a, c, sm);
                    }
                    break;
                case OP_R2C_HALF: store_r2c_half(tid, T, a, c, sm); break;
                case OP_C2R_HALF: store_c2r_half(tid, T, a, c, sm); break;
                case OP_R2C_PAIR: store_r2c_pair(tid, T, a, c, sm); break;
                case OP_C2R_PAIR: store_c2r_pair(tid, T, a, c, sm); break;
            }
        }
    }
}

// Tensor-core step: the kernel's phase functions (tc_core.cuh) per thread,
// with a host GEMM over the same split operand layouts in place of tcgen05.
template <int SIGN, bool TW4, bool CI, bool CO>
void emu_tc_tiles(const TileArgs& a) {
    std::vector<uint16_t> b(3 * kTcK * kTcK);
    tc_make_b(SIGN, b.data());
    std::vector<float2> tw256(256);
    for (int m = 0; m < 256; ++m) tw256[m] = root_host(m, 256);
    std::vector<float2> tile(kTcP * kTcLD);
    std::vector<unsigned char> abuf(3 * kTcTermBytes);
    std::vector<float> d(kTcRows * kTcK);
    for (int t = 0; t < a.ntiles; ++t) {
        const TileCtx c = decode_tile(a, t);
        for (int tid = 0; tid < kTcThreads; ++tid) tc_load_tile<CI>(tid, a, c, tile.data());
        for (int stage = 0; stage < 2; ++stage) {
            for (int tid = 0; tid < kTcThreads; ++tid) {
                float2 x[16];
                if (stage == 0) tc_gather1(tile.data(), tid, x); else tc_gather2(tile.data(), tid, x);
                tc_put_row(abuf.data(), tid, x);
            }
            tc_gemm_host(abuf.data(), b.data(), d.data());
            for (int tid = 0; tid < kTcThreads; ++tid) {
                float r[32];
                for (int i = 0; i < 32; ++i) r[i] = d[tid * kTcK + i];
                if (stage == 0) tc_scatter1<SIGN>(tile.data(), tid, r, tw256.data()); else tc_scatter2(tile.data(), tid, r);
            }
        }
        for (int tid = 0; tid < kTcThreads; ++tid) tc_store_tile<SIGN, TW4, CO>(tid, a, c, tile.data());
    }
}

void emu_tc_step(const Step& st, const void* src, void* dst) {
    TileArgs a = st.L.args;
    a.src = src;
    a.dst = dst;
    std::vector<float2> tw2 = tw2_host(st);
    a.tw2 = tw2.empty() ? nullptr : tw2.data();
    const bool ci = st.tc_cols_in, co = st.tc_cols_out, t4 = st.L.tw4;
#define SIP_EMU_TC(S)                                                   \
    if (t4) emu_tc_tiles<S, true, true, true>(a);                     \
    else if (ci && co) emu_tc_tiles<S, false, true, true>(a);         \
    else if (!ci && co) emu_tc_tiles<S, false, false, true>(a);       \
    else emu_tc_tiles<S, false, false, false>(a);
    if (st.L.sign < 0) { SIP_EMU_TC(-1) } else { SIP_EMU_TC(1) }
#undef SIP_EMU_TC
}

// Bluestein pre / post pass on the CPU (bluestein.cuh element functions)
// with the chirp computed on the host.
void emu_blue_step(const Step& st, const void* src, void* dst) {
    std::vector<float2> chirp = chirp_host(st.blue_n, st.blue_sign);
    BluesteinArgs a = st.blue;
    a.src = src;
    a.dst = dst;
    a.chirp = chirp.data();
    if (!st.blue_post) {
        float2* out = static_cast<float2*>(dst);
        for (long long row = 0; row < a.rows; ++row)
            for (long long j = 0; j < a.m; ++j) out[row * a.m + j] = blue_pre_elem(a, row, j);
    } else {
        const long long cnt = blue_out_count(a);
        for (long long row = 0; row < a.rows; ++row)
            for (long long k = 0; k < cnt; ++k) blue_post_elem(a, row, k);
    }
}

// Cluster four-step step: the harness's runner of the step's configuration.
void emu_cluster_step(const Step& st, const void* src, void* dst) {
    TileArgs a = st.L.args, b = st.cl_b;
    std::vector<float2> twa = basis_host(st.radices), twb = basis_host(st.cl_radices_b), tw2 = tw2_host(st);
    a.src = src;
    a.tw = twa.data();
    b.dst = dst;
    b.tw = twb.data();
    b.tw2 = tw2.data();
    reinterpret_cast<EmuClFn>(const_cast<void*>(st.cl->fn))(a, b, st.cl_transforms);
}

// Element-wise passes of odd real lengths above one tile (real_kernels.cu).
void emu_pair_step(const Step& st, const void* src, void* dst) {
    const PairPassArgs& a = st.pair;
    const long long pairs = (a.rows + 1) / 2;
    for (long long p = 0; p < pairs; ++p) {
        const bool second = 2 * p + 1 < a.rows;
        if (st.kind == StepKind::PairPack) {
            const float* xa = static_cast<const float*>(src) + 2 * p * a.in_pitch;
            float2* z = static_cast<float2*>(dst) + p * a.out_pitch;
            for (long long j = 0; j < a.n; ++j) z[j] = make_float2(xa[j], second ? xa[a.in_pitch + j] : 0.f);
        } else if (st.kind == StepKind::PairSeparate) {
            const float2* z = static_cast<const float2*>(src) + p * a.in_pitch;
            float2* outa = static_cast<float2*>(dst) + 2 * p * a.out_pitch;
            for (long long k = 0; 2 * k <= a.n; ++k) {
                float2 xa, xb;
                pair_separate_elem(z, k, a.n, a.conj != 0, &xa, &xb);
                outa[k] = xa;
                if (second) outa[a.out_pitch + k] = xb;
            }
        } else if (st.kind == StepKind::PairCombine) {
            const float2* xa = static_cast<const float2*>(src) + 2 * p * a.in_pitch;
            float2* z = static_cast<float2*>(dst) + p * a.out_pitch;
            for (long long k = 0; k < a.n; ++k)
                z[k] = pair_combine_elem(xa, second ? xa + a.in_pitch : nullptr, k, a.n, a.conj != 0);
        } else {
            const float2* z = static_cast<const float2*>(src) + p * a.in_pitch;
            float* outa = static_cast<float*>(dst) + 2 * p * a.out_pitch;
            for (long long j = 0; j < a.n; ++j) {
                outa[j] = z[j].x;
                if (second) outa[a.out_pitch + j] = z[j].y;
            }
        }
    }
}

void emu_real_step(const Step& st, const void* src, void* dst) {
    std::vector<float2> tw = tw2_host(st);
    const RealPassArgs& r = st.real;
    const float2* s = static_cast<const float2*>(src);
    float2* d = static_cast<float2*>(dst);
    // the kernels' pairing (real_kernels.cu): pair functions for 0 < k < m - k
    const bool cj = r.conj != 0;
    for (long long row = 0; row < r.rows; ++row) {
        const float2* in = s + row * r.in_pitch;
        float2* out = d + row * r.out_pitch;
        for (long long k = 0; k <= r.m / 2; ++k) {
            const long long km = r.m - k;
            if (st.kind == StepKind::RealPost) {
                if (k > 0 && k < km) {
                    real_post_pair(in, k, r.m, tw.data(), cj, out + k, out + km);
                } else {
                    out[k] = real_post_elem(in, k, r.m, tw.data(), cj);
                    if (km != k) out[km] = real_post_elem(in, km, r.m, tw.data(), cj);
                }
            } else {
                if (k > 0 && k < km) {
                    real_pre_pair(in, k, r.m, tw.data(), cj, out + k, out + km);
                } else {
                    out[k] = real_pre_elem(in, k, r.m, tw.data(), cj);
                    if (km != k && km < r.m) out[km] = real_pre_elem(in, km, r.m, tw.data(), cj);
                }
            }
        }
    }
}

}  // namespace

extern "C" {

// Plans (type, direction, sizes, batch) with the library planner and runs
// it on host buffers.  Returns 0 on success, the planner's status code on
// a planning failure, -1 on an emulation failure.  `desc` receives the
// plan description (JSON) when non-null.
int emu_exec_mode(int type, int direction, int ndim, const long long* sizes, long long batch, const void* in,
                  void* out, char* desc, size_t desc_cap, int mode);

int emu_run_plan(FftPlan& p, const void* in, void* out, char* desc, size_t desc_cap);

// Planner real-fused hint applied to the plans emu_exec builds (0 default).
static int g_emu_real_fused = 0;
void emu_set_real_fused(int v) { g_emu_real_fused = v; }
// Planner sk-variant hint applied likewise.
static int g_emu_sk_variant = -1;
void emu_set_sk_variant(int v) { g_emu_sk_variant = v; }
// Output shift (mode, scale) applied likewise.
static int g_emu_shift = 0;
static double g_emu_shift_scale = 1.0;
void emu_set_out_shift(int mode, double scale) {
    g_emu_shift = mode;
    g_emu_shift_scale = scale;
}

// Pulse-compression plan of length n over batch rows with the host filter
// spectrum `filter` (n complex values) and flags (1 conj, 2 scale 1/n).
int emu_exec_pulse(long long n, long long batch, const void* filter, int flags, const void* in, void* out,
                   char* desc, size_t desc_cap) {
    FftPlan p;
    p.type = AsdSip::ASCEND_FFT_C2C;
    p.direction = AsdSip::ASCEND_FFT_FORWARD;
    p.sizes = {n};
    p.batch = batch;
    p.pulse = true;
    p.pulse_filter = filter;
    p.pulse_flags = flags;
    return emu_run_plan(p, in, out, desc, desc_cap);
}

int emu_exec(int type, int direction, int ndim, const long long* sizes, long long batch, const void* in, void* out,
             char* desc, size_t desc_cap) {
    return emu_exec_mode(type, direction, ndim, sizes, batch, in, out, desc, desc_cap, 0);
}

// As emu_exec with a compute mode (0 FP32, 1 tensor-core split).
int emu_exec_mode(int type, int direction, int ndim, const long long* sizes, long long batch, const void* in,
                  void* out, char* desc, size_t desc_cap, int mode) {
    FftPlan p;
    p.compute_mode = mode;
    p.type = static_cast<AsdSip::asdFftType>(type);
    p.direction = static_cast<AsdSip::asdFftDirection>(direction);
    p.sizes.assign(sizes, sizes + ndim);
    p.batch = batch;
    p.hint_real_fused = g_emu_real_fused;
    p.hint_sk_variant = g_emu_sk_variant;
    p.out_shift = g_emu_shift;
    p.out_scale = g_emu_shift_scale;
    return emu_run_plan(p, in, out, desc, desc_cap);
}

// Builds the plan's steps and runs them on host buffers.
int emu_run_plan(FftPlan& p, const void* in, void* out, char* desc, size_t desc_cap) {
    try {
        build_steps(p);
    } catch (const PlanError& e) {
        if (desc && desc_cap) std::snprintf(desc, desc_cap, "%s", e.what());
        return e.code;
    }
    if (desc && desc_cap) std::snprintf(desc, desc_cap, "%s", describe(p).c_str());
    try {
        // NaN-filled workspace: a chunk that read what no step of it wrote
        // would show up in the result
        std::vector<float> wsf((p.workspace_need + 16) / 4 + 1, std::numeric_limits<float>::quiet_NaN());
        char* ws = reinterpret_cast<char*>(wsf.data());
        // one step, restricted to chunk units [u0, u0 + cnt) of its group
        // when cnt >= 0 (the launch_steps order of the library)
        auto run_step = [&](const Step& st, long long u0, long long cnt, int lane, long long cu) {
            auto resolve = [&](Loc l, size_t off) -> char* {
                char* base = l == Loc::In ? const_cast<char*>(static_cast<const char*>(in))
                           : l == Loc::Out ? static_cast<char*>(out) : ws;
                return base + off;
            };
            char* s = resolve(st.src, st.src_off);
            char* d = resolve(st.dst, st.dst_off);
            std::vector<float2> filt;
            Step stc = st;
            if (cnt >= 0) {
                s += chunk_offset(st, true, u0, lane, cu);
                d += chunk_offset(st, false, u0, lane, cu);
                if (st.kind == StepKind::Tile) stc.L = chunk_tile_launch(st, cnt);
                else stc.real.rows = cnt * st.chunk_per;
            }
            if (st.mul_table == 1) {  // the Bluestein filter the device preparation would make
                filt = bluestein_filter(st.blue_n, st.blue_m, st.blue_sign);
                stc.L.args.mul = filt.data();
            }
            if (st.kind == StepKind::Blue) emu_blue_step(st, s, d);
            else if (is_pair_kind(st.kind)) emu_pair_step(st, s, d);
            else if (st.kind == StepKind::Cluster) emu_cluster_step(st, s, d);
            else if (st.kind == StepKind::Tile) emu_tile_step(stc, s, d);
            else if (st.kind == StepKind::Tc) emu_tc_step(st, s, d);
            else emu_real_step(stc, s, d);
        };
        for (size_t i = 0; i < p.steps.size();) {
            const int gi = p.steps[i].chunk_group;
            if (gi >= 0) {
                const ChunkGroup& g = p.chunk_groups[gi];
                const long long cu = chunk_units(g);
                if (cu < g.units) {
                    // the library's lanes: chunk k on lane k % 2 (workspace
                    // regions per lane); run in order here
                    int k = 0;
                    for (long long u0 = 0; u0 < g.units; u0 += cu, ++k)
                        for (size_t j = g.first; j < g.last; ++j)
                            run_step(p.steps[j], u0, std::min(cu, g.units - u0), chunk_lanes() == 2 ? (k & 1) : 0, cu);
                    i = g.last;
                    continue;
                }
            }
            run_step(p.steps[i], 0, -1, 0, 0);
            ++i;
        }
    } catch (const std::exception&) {
        return -1;
    }
    return 0;
}

// Chunk size of the L2-resident chunks for plans made afterwards (bytes;
// 0 off, negative: the library default).
void emu_set_chunk_bytes(long long bytes) { set_l2_chunk_bytes(bytes); }

// Fast-division check: returns the number of mismatches of fd_div against
// exact division over `count` (divisor, dividend) pairs.
long long emu_fastdiv_check(const unsigned* d, const unsigned* n, long long count) {
    long long bad = 0;
    for (long long i = 0; i < count; ++i) {
        const FastDiv f = make_fastdiv(d[i]);
        if (fd_div(f, n[i]) != n[i] / d[i]) ++bad;
    }
    return bad;
}

// Radix plan chosen for length n (elements per thread e); writes up to cap
// radices, returns the count (-1: not factorizable).
int emu_radices(int n, int e, int* out, int cap) {
    std::vector<int> r = choose_radices(n, e);
    if (r.size() == 1 && r[0] == -1) return -1;
    for (int i = 0; i < (int)r.size() && i < cap; ++i) out[i] = r[i];
    return (int)r.size();
}

// One in-register butterfly on host data (checks dft<R, SIGN>).
int emu_dft(int r, int sign, float* data) {
    float2* v = reinterpret_cast<float2*>(data);
    bool ok = true;
    auto run = [&](auto rc) {
        constexpr int R = decltype(rc)::value;
        float2 t[R];
        for (int i = 0; i < R; ++i) t[i] = v[i];
        if (sign < 0) dft<R, -1>(t); else dft<R, 1>(t);
        for (int i = 0; i < R; ++i) v[i] = t[i];
    };
    switch (r) {
#define SIP_EMU_DFT(R) case R: run(std::integral_constant<int, R>{}); break;
        SIP_FFT_FOR_EACH_RADIX(SIP_EMU_DFT)
#undef SIP_EMU_DFT
        default: ok = false;
    }
    return ok ? 0 : -1;
}

}  // extern "C"

extern "C" {
// Lists the compiled size-specialized configurations: 7 ints per entry
// (op, mode, sign, tw4, n, P, T); returns the entry count.
int emu_sk_list(int* out, int cap) {
    const auto& reg = sipfft::sk_registry();
    int i = 0;
    for (const auto& e : reg) {
        if (i < cap) {
            int* o = out + 7 * i;
            o[0] = e.op; o[1] = e.mode; o[2] = e.sign; o[3] = e.tw4 ? 1 : 0; o[4] = e.n; o[5] = e.P; o[6] = e.T;
        }
        ++i;
    }
    return i;
}
}
