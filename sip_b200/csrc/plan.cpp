// Planner of the B200 FFT library.
//
// Replaces the reference's plan builder (core/fft/fft_api.cpp:662-992:
// addFFTSteps / init2DSteps / init3DSteps with their per-axis core
// routing and explicit last-two-axis transposes).  Here every axis pass is
// one tile-kernel launch that reads its transforms in place through
// strides, so a 2D transform is two HBM round trips and a 3D transform
// three, with no transpose steps.  Lengths above one tile (16384 complex
// points) use a two-pass four-step split N = N1 * N2.
#include "plan.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <sstream>
#include <tuple>

#include "real_kernels.h"
#include "sk_registry.h"

namespace sipfft {

using namespace AsdSip;

DeviceBuf::~DeviceBuf() {
    if (ptr == nullptr) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (device >= 0 && device != cur) cudaSetDevice(device);
    cudaFree(ptr);
    if (device >= 0 && device != cur && cur >= 0) cudaSetDevice(cur);
}

int64_t FftPlan::elements() const {
    int64_t e = batch;
    for (int64_t s : sizes) e *= s;
    return e;
}

// Compute mode and hints of the plan being built, set by build_steps for the
// helpers below (per thread, so concurrent planners do not interfere; the C
// ABI also plans under its global lock).
namespace {
thread_local int g_compute_mode = kComputeFp32;
thread_local int g_hint_p = 0, g_hint_e = 0, g_hint_generic = 0, g_hint_order = 0, g_hint_real_fused = 0,
                 g_hint_variant = -1, g_hint_jit = 0;
// Column length the next four-step split must use (0: the balanced split);
// set by a caller that needs the passes of a particular split.
thread_local int g_split_n1 = 0;
}  // namespace

// ------------------------------------------------------------ radices
namespace {

struct RadixCost {
    int r;
    double cost;
};

// Cost of one pass: dominated by the shared-memory round trip (1.0); larger
// radices pay a little for register pressure and prime radices for their
// O(R^2) butterfly.
double radix_cost(int r) {
    double c = 1.0 + 0.002 * r;
    if (r == 11 || r == 13 || r == 17 || r == 19) c += 0.2;
    if (r == 23 || r == 29 || r == 31) c += 0.5;
    return c;
}

const int kRadixList[] = {32, 31, 29, 27, 25, 23, 19, 17, 16, 15, 13, 11, 10, 9, 8, 7, 5, 4, 3, 2};

}  // namespace

std::vector<int> choose_radices(int n, int e) {
    if (n == 1) return {};
    const int maxr = e >= 32 ? 32 : 31;  // a pass needs R < 2E
    std::map<int, std::pair<double, std::vector<int>>> memo;
    std::function<std::pair<double, std::vector<int>>(int)> best = [&](int m) -> std::pair<double, std::vector<int>> {
        if (m == 1) return {0.0, {}};
        auto it = memo.find(m);
        if (it != memo.end()) return it->second;
        std::pair<double, std::vector<int>> res{1e30, {}};
        for (int r : kRadixList) {
            if (r > maxr || m % r != 0 || !radix_supported(r)) continue;
            auto sub = best(m / r);
            if (sub.first >= 1e29) continue;
            const double c = sub.first + radix_cost(r);
            if (c < res.first) {
                res.first = c;
                res.second = sub.second;
                res.second.push_back(r);
            }
        }
        memo[m] = res;
        return res;
    };
    auto r = best(n);
    if (r.first >= 1e29) return {-1};
    if (g_hint_order == 1) std::sort(r.second.begin(), r.second.end());
    else std::sort(r.second.begin(), r.second.end(), std::greater<int>());
    return r.second;
}

namespace {

bool factorizable(int n, int e) {
    if (n == 1) return true;
    auto r = choose_radices(n, e);
    return !(r.size() == 1 && r[0] == -1);
}

PlanDev make_plandev(int n, const std::vector<int>& radices, int* tw_entries) {
    PlanDev pd{};
    pd.N = n;
    pd.npass = (int)radices.size();
    if (pd.npass > kMaxPasses) throw PlanError(ACL_ERROR_INTERNAL_ERROR, "too many passes");
    int L = 1, off = 0;
    for (int i = 0; i < pd.npass; ++i) {
        PassDesc& p = pd.pass[i];
        p.R = radices[i];
        p.L = L;
        p.tw = off;
        p.nr = make_fastdiv((uint32_t)(n / p.R));
        p.l = make_fastdiv((uint32_t)L);
        if (L > 1) off += L * (p.R - 1);
        L *= p.R;
    }
    *tw_entries = off;
    return pd;
}

int even_ld(int rowlen) {
    int ld = sidx(rowlen - 1) + 1;
    if ((ld & 1) == 0) ++ld;
    return ld;
}

constexpr int kSmemLimit = kMaxTileSmem;
constexpr int kRowTileBytes = 64 * 1024;
// Row tiles of the generic kernel hold about this many values: small CTAs
// (32-256 threads at 32 values per thread), several per SM, so that one
// CTA's loads overlap another's passes (the generic kernel does not stage
// the next tile itself).  Measured against 16 values per thread and 64 KB
// tiles: 11-31 % faster on C2C 544 to 6720, R2C 6688, C2R 3000.  Plans made
// with the generic-only hint keep 64 KB tiles (still at 32 values per
// thread): the batch work queue (queue.cu), which runs those plans, gives
// every tile a 512-thread CTA and claims tiles one by one, and lost 20 % of
// its serving capacity with the small tiles.
constexpr int kRowTileValues = 2048;

struct TileShape {
    int e, P, T, LD, smem;
};

// `column`: the tile's transforms are adjacent in memory on the load or
// store side, so P sets the contiguous run length (8-16 values wanted).
TileShape pick_shape(int n, int rowlen, bool column, long long transforms) {
    TileShape s{};
    const bool queue_shape = g_hint_generic != 0;
    s.e = 32;
    if (g_hint_e == 16 && n <= 8192) s.e = 16;
    if (g_hint_e == 32) s.e = 32;
    s.LD = even_ld(std::max(rowlen, 1));
    const long long row_bytes = (long long)s.LD * 8;
    long long maxp_thr = std::max<long long>(1, (long long)kMaxTileThreads * s.e / std::max(n, 1));
    long long p;
    if (column) {
        p = std::min<long long>({16, maxp_thr, std::max<long long>(1, kSmemLimit / row_bytes)});
    } else {
        p = std::min<long long>(maxp_thr, std::max<long long>(1, kRowTileBytes / row_bytes));
        if (!queue_shape) p = std::min<long long>(p, std::max<long long>(1, kRowTileValues / std::max(n, 1)));
    }
    if (g_hint_p > 0)
        p = std::min<long long>({(long long)g_hint_p, maxp_thr, std::max<long long>(1, kSmemLimit / row_bytes)});
    p = std::max<long long>(1, std::min<long long>(p, transforms));
    s.P = (int)p;
    long long t = ((long long)s.P * n + s.e - 1) / s.e;
    t = std::max<long long>(32, (t + 31) / 32 * 32);
    s.T = (int)std::min<long long>(t, kMaxTileThreads);
    s.smem = (int)(s.P * row_bytes);
    if (s.smem > kSmemLimit) throw PlanError(ACL_ERROR_INTERNAL_ERROR, "tile does not fit shared memory");
    return s;
}

struct AxisIO {
    long long inner = 1, outer = 1;
    long long in_odist = 0, in_idist = 0, in_stride = 1;
    long long out_odist = 0, out_idist = 0, out_stride = 1;
};

// One tile launch.  n = FFT length of each tile transform; rowlen = values
// a shared-memory row must hold; transforms = inner * outer.
// Layout mode of a step for the size-specialized kernels, or -1.
int sk_mode_of(int op, int n, const AxisIO& io, int blue_n = 0) {
    long long in_row = n, out_row = n;
    if (blue_n > 0) in_row = out_row = blue_n;  // fused Bluestein rows (TF_BLUE)
    switch (op) {
        case OP_R2C_HALF: out_row = n + 1; break;
        case OP_C2R_HALF: in_row = n + 1; break;
        case OP_R2C_PAIR: out_row = n / 2 + 1; break;
        case OP_C2R_PAIR: in_row = n / 2 + 1; break;
        default: break;
    }
    // rows: contiguous within a tile; successive outer indices continue the
    // same row pitch (the tile decode keeps a tile inside one outer index)
    if (io.in_stride == 1 && io.out_stride == 1 && io.in_idist == in_row && io.out_idist == out_row &&
        (io.outer == 1 || (io.in_odist == io.inner * in_row && io.out_odist == io.inner * out_row)))
        return SK_ROWS;
    if (op != OP_C2C) return -1;
    if (io.in_idist == 1 && io.out_idist == 1) return SK_COLS;
    if (io.in_stride == 1 && io.in_idist == n && io.in_odist == io.inner * n && io.out_idist == 1) return SK_ROWS_T;
    return -1;
}

// Switches a generic tile step to a size-specialized kernel when one is
// compiled for it (its radix order, tile size and threads then apply).
void try_specialize(Step& st, const AxisIO& io) {
    TileLaunch& L = st.L;
    TileArgs& a = L.args;
    const int mode = sk_mode_of(L.op, a.N, io, (a.flags & TF_BLUE) ? a.n_other : 0);
    if (mode < 0) return;
    // SIP_FFT_JIT_PREFER=1 (tuning sweeps) skips the compiled kernels so that
    // run-time configurations can be timed against them; =<length> does so
    // for steps of that length only
    const char* prefer = std::getenv("SIP_FFT_JIT_PREFER");
    const int prefer_n = prefer != nullptr ? std::atoi(prefer) : 0;
    const bool prefer_jit = prefer_n == 1 || (prefer_n > 1 && prefer_n == a.N);
    const SkEntry* e = prefer_jit ? nullptr : sk_find(L.op, mode, L.sign, L.tw4, a.N, g_hint_variant);
    // No compiled kernel for this length: a run-time compiled one (jit.cpp)
    // for steps large enough to repay the compilation, or on request.
    const long long values = io.inner * io.outer * (long long)a.N;
    if (e == nullptr && (g_hint_jit == 1 || (g_hint_jit == 0 && values >= (1LL << 18)))) {
        // hint 1 (or SIP_FFT_JIT_SYNC=1) compiles now; the default compiles
        // a new configuration in the background and plans later shapes with it
        const char* sync_env = std::getenv("SIP_FFT_JIT_SYNC");
        const bool sync = g_hint_jit == 1 || (sync_env != nullptr && std::strcmp(sync_env, "1") == 0);
        e = sk_jit_entry(L.op, mode, L.sign, L.tw4, a.N, io.inner, sync);
    }
    if (e == nullptr) return;
    // A row step of less than one wave of tiles (two per SM) takes the
    // compiled variant with more threads per tile when there is one: each
    // transform's loads, passes and stores spread over more warps (C2C 4096
    // x 256: 7.2 us with 256 threads per transform, 8.7 us with 128).
    if (g_hint_variant < 0 && mode == SK_ROWS && !e->jit) {
        const long long tiles = (io.inner + e->P - 1) / e->P * io.outer;
        if (tiles <= kOneWaveTiles)
            if (const SkEntry* w = sk_find_wider(e)) e = w;
    }
    st.sk = e;
    st.radices = e->radices;
    int tw_entries = 0;
    st.host_plan = make_plandev(a.N, st.radices, &tw_entries);
    L.block = e->T;
    L.smem_bytes = e->smem;
    a.P = e->P;
    a.LD = e->LD;
    a.tiles_per_outer = (int)((io.inner + e->P - 1) / e->P);
    a.ntiles = (int)((long long)a.tiles_per_outer * io.outer);
    a.div_p = make_fastdiv((uint32_t)e->P);
    a.div_tpo = make_fastdiv((uint32_t)a.tiles_per_outer);
    L.grid = a.ntiles;  // capped to the resident CTAs at device preparation
    st.what += std::string(e->jit ? " [sk jit P=" : " [sk P=") + std::to_string(e->P) + "]";
}



// Tensor-core form: a C2C step of length 256 runs as two BF16x3 split
// DFT-16 GEMM stages on tcgen05 (tc_kernel.cu) instead of Stockham passes.
void try_tensor_core(Step& st, const AxisIO& io) {
    TileLaunch& L = st.L;
    TileArgs& a = L.args;
    if (g_compute_mode != kComputeTcSplit || g_hint_generic || L.op != OP_C2C || a.N != 256) return;
    st.kind = StepKind::Tc;
    st.sk = nullptr;
    st.tc_cols_in = io.in_idist == 1;
    st.tc_cols_out = io.out_idist == 1;
    a.P = 8;
    a.tiles_per_outer = (int)((io.inner + 7) / 8);
    a.ntiles = (int)((long long)a.tiles_per_outer * io.outer);
    a.div_p = make_fastdiv(8);
    a.div_tpo = make_fastdiv((uint32_t)a.tiles_per_outer);
    L.block = 128;
    L.grid = a.ntiles;
    st.what += " [tensor-core bf16x3]";
}

Step make_tile_step(int op, int sign, int n, int rowlen, bool column, const AxisIO& io, int flags, int rows,
                    const std::string& what, bool tw4 = false, int blue_n = 0) {
    Step st;
    const long long transforms = io.inner;
    TileShape sh = pick_shape(n, rowlen, column, transforms);
    st.radices = choose_radices(n, sh.e);
    if (st.radices.size() == 1 && st.radices[0] == -1)
        throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "length " + std::to_string(n) + " has no supported radix plan");
    int tw_entries = 0;
    st.host_plan = make_plandev(n, st.radices, &tw_entries);
    TileLaunch& L = st.L;
    L.sign = sign;
    L.e = sh.e;
    L.op = op;
    L.block = sh.T;
    L.smem_bytes = sh.smem;
    TileArgs& a = L.args;
    a.N = n;
    a.P = sh.P;
    a.LD = sh.LD;
    a.inner = (int)io.inner;
    a.tiles_per_outer = (int)((io.inner + sh.P - 1) / sh.P);
    const long long ntiles = (long long)a.tiles_per_outer * io.outer;
    if (ntiles > 0x7fffffffLL || io.inner > 0x7fffffffLL)
        throw PlanError(ACL_ERROR_INVALID_PARAM, "too many transforms");
    a.ntiles = (int)ntiles;
    a.in_odist = io.in_odist;
    a.in_idist = io.in_idist;
    a.in_stride = io.in_stride;
    a.out_odist = io.out_odist;
    a.out_idist = io.out_idist;
    a.out_stride = io.out_stride;
    a.rows = rows;
    a.flags = flags;
    a.n_other = blue_n;
    a.scale = 1.0f;
    a.div_n = make_fastdiv((uint32_t)std::max(n, 1));
    a.div_p = make_fastdiv((uint32_t)sh.P);
    const int h = (op == OP_R2C_HALF || op == OP_C2R_HALF) ? n + 1 : n / 2 + 1;
    a.div_h = make_fastdiv((uint32_t)h);
    a.div_tpo = make_fastdiv((uint32_t)a.tiles_per_outer);
    L.grid = a.ntiles;
    L.tw4 = tw4;
    st.what = what;
    (void)tw_entries;
    if (!std::getenv("SIP_FFT_GENERIC_ONLY") && !g_hint_generic) try_specialize(st, io);
    try_tensor_core(st, io);
    return st;
}

int c2c_sign(const FftPlan& plan) { return plan.forward() ? -1 : 1; }

// Splits n > kMaxTileN into n1 (column pass) * n2 (row pass), both one
// tile long and factorizable, n1 <= n2 and as balanced as possible.
bool four_step_split(long long n, int* n1, int* n2) {
    int best1 = 0;
    for (long long a = 2; a * a <= n; ++a) {
        if (n % a) continue;
        const long long b = n / a;
        if (b > kMaxTileN || a > kMaxTileN) continue;
        if (!factorizable((int)a, 32) || !factorizable((int)b, 32)) continue;
        best1 = (int)a;  // ascending a: the last hit is the most balanced
    }
    if (best1 == 0) return false;
    // SIP_FFT_SPLIT_N1 (tuning sweeps) or a caller's choice: the column
    // length, when it divides n into two lengths that fit a tile
    const char* env = std::getenv("SIP_FFT_SPLIT_N1");
    if (g_split_n1 > 0 || env != nullptr) {
        const long long a = g_split_n1 > 0 ? g_split_n1 : std::atoll(env);
        if (a >= 2 && n % a == 0 && a <= kMaxTileN && n / a <= kMaxTileN && factorizable((int)a, 32) &&
            factorizable((int)(n / a), 32))
            best1 = (int)a;
    }
    *n1 = best1;
    *n2 = (int)(n / best1);
    return true;
}

struct C2COpts {
    int sign = 0;        // 0: the plan's direction
    int last_flags = 0;  // flags of the final pass (scaling)
    float last_scale = 1.0f;
    Loc src = Loc::In, dst = Loc::Out;
    size_t src_off = 0, dst_off = 0;
    size_t scratch_off = 0;  // four-step scratch region in the workspace
};

// The cluster four-step (cluster.h) for a plain C2C of few transforms: one
// cluster of CTAs per transform (C2C 4096 x 256: 1024 CTAs instead of 256).
// Opt-in (SIP_FFT_CLUSTER=1) for the lengths with a compiled configuration:
// on B200 it was 15-80 % slower than one CTA per transform at every batch
// measured (4096 x 64 .. 512, 1024 x 1024 / 2048, 8192 x 128 / 256), the
// cluster launch, the two cluster barriers and the DSMEM gather costing more
// than the wider spread of the loads gains.
const ClEntry* pick_cluster(long long n, long long batch, int sign, const C2COpts& o) {
    (void)batch;
    if (o.src != Loc::In || o.dst != Loc::Out || o.src_off || o.dst_off || o.last_flags) return nullptr;
    if (g_hint_generic || std::getenv("SIP_FFT_GENERIC_ONLY")) return nullptr;
    const char* e = std::getenv("SIP_FFT_CLUSTER");
    if (e == nullptr || std::atoi(e) != 1) return nullptr;
    return cluster_find((int)n, sign);
}

void add_cluster_c2c(FftPlan& plan, const ClEntry* ce, long long n, long long batch) {
    Step st;
    st.kind = StepKind::Cluster;
    st.cl = ce;
    st.cl_transforms = batch;
    int tw_entries = 0;
    st.radices = ce->ra;
    st.host_plan = make_plandev(ce->n1, ce->ra, &tw_entries);
    st.cl_radices_b = ce->rb;
    st.cl_plan_b = make_plandev(ce->n2, ce->rb, &tw_entries);
    int shift = 0;
    while ((1LL << (2 * shift)) < n) ++shift;
    TileArgs& a = st.L.args;  // columns i2 of x viewed as [n1][n2]
    a.N = ce->n1;
    a.P = ce->pa;
    a.inner = ce->n2;
    a.in_odist = n;
    a.in_idist = 1;
    a.in_stride = ce->n2;
    a.scale = 1.0f;
    a.tw4_shift = shift;
    TileArgs& b = st.cl_b;  // rows k1 of Y, X[k1 + n1 k2] out
    b.N = ce->n2;
    b.P = ce->pb;
    b.inner = ce->n1;
    b.out_odist = n;
    b.out_idist = 1;
    b.out_stride = ce->n1;
    b.scale = 1.0f;
    b.tw4_shift = shift;
    st.tw2_kind = 2;  // the cross twiddles W_n^m, pass B's gather
    st.tw2_n = n;
    st.tw2_count = (1LL << shift) + (n + (1LL << shift) - 1) / (1LL << shift);
    st.L.sign = ce->sign;
    st.L.block = ce->T;
    st.L.smem_bytes = ce->smem;
    st.L.grid = (int)(batch * ce->C);
    st.src = Loc::In;
    st.dst = Loc::Out;
    st.what = "c2c cluster n=" + std::to_string(n) + " [" + std::to_string(ce->C) + " CTAs per transform]";
    plan.steps.push_back(st);
}

void add_c2c_1d(FftPlan& plan, long long n, long long batch, const C2COpts& o) {
    const int sign = o.sign != 0 ? o.sign : c2c_sign(plan);
    if (const ClEntry* ce = n <= kMaxTileN ? pick_cluster(n, batch, sign, o) : nullptr) {
        add_cluster_c2c(plan, ce, n, batch);
        return;
    }
    if (n <= kMaxTileN) {
        AxisIO io;
        io.inner = batch;
        io.in_idist = n;
        io.out_idist = n;
        Step st = make_tile_step(OP_C2C, sign, (int)n, (int)n, false, io, o.last_flags, 0,
                                 "c2c rows n=" + std::to_string(n));
        st.batch_dim = 1;
        st.L.args.scale = o.last_scale;
        st.src = o.src;
        st.dst = o.dst;
        st.src_off = o.src_off;
        st.dst_off = o.dst_off;
        plan.steps.push_back(st);
        return;
    }
    int n1 = 0, n2 = 0;
    if (!four_step_split(n, &n1, &n2))
        throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "length " + std::to_string(n) + " has no four-step split");
    // Pass A: n1-point FFTs down the n2 columns of x viewed as [n1][n2],
    // times W_n^{n2 k1}, into the workspace as Y[k1][n2]
    // (reference: phase A of core/fft/fftcore/fft_c2c_large.cpp:199-204).
    AxisIO a;
    a.inner = n2;
    a.outer = batch;
    a.in_odist = n;
    a.in_idist = 1;
    a.in_stride = n2;
    a.out_odist = n;
    a.out_idist = 1;
    a.out_stride = n2;
    Step sa = make_tile_step(OP_C2C, sign, n1, n1, true, a, 0, 0,
                             "four-step A n=" + std::to_string(n) + " n1=" + std::to_string(n1), true);
    {
        int shift = 0;
        while ((1LL << (2 * shift)) < n) ++shift;  // B = 2^shift >= sqrt(n)
        sa.L.args.tw4_shift = shift;
        sa.tw2_kind = 2;
        sa.tw2_n = n;
        sa.tw2_count = (1LL << shift) + (n + (1LL << shift) - 1) / (1LL << shift);
    }
    sa.src = o.src;
    sa.src_off = o.src_off;
    sa.dst = Loc::Ws;
    sa.dst_off = o.scratch_off;
    // Pass B: n2-point FFTs along the rows of Y; X[k1 + n1 k2] is stored
    // with stride n1, so adjacent rows of a tile are adjacent outputs.
    AxisIO b;
    b.inner = n1;
    b.outer = batch;
    b.in_odist = n;
    b.in_idist = n2;
    b.in_stride = 1;
    b.out_odist = n;
    b.out_idist = 1;
    b.out_stride = n1;
    Step sb = make_tile_step(OP_C2C, sign, n2, n2, true, b, o.last_flags, 0,
                             "four-step B n=" + std::to_string(n) + " n2=" + std::to_string(n2));
    sb.L.args.scale = o.last_scale;
    sa.batch_dim = 2;
    sb.batch_dim = 2;
    sb.src = Loc::Ws;
    sb.src_off = o.scratch_off;
    sb.dst = o.dst;
    sb.dst_off = o.dst_off;
    plan.steps.push_back(sa);
    plan.steps.push_back(sb);
    plan.workspace_need = std::max(plan.workspace_need, o.scratch_off + (size_t)(batch * n * 8));
}

// Pulse compression y = IFFT(FFT(x) * F) of every row (length n, batch
// rows), F the filter spectrum (conjugated with kPulseConj), optionally
// scaled by 1/n.  Up to one tile the chain is one kernel (OP_PC: load, forward
// passes, multiply, inverse passes, store).  Above it the four-step
// factorisation n = n1 n2 is kept open in the middle:
//   pass A (existing): n1-point FFTs down the columns, times W_n^{n2 k1},
//          into Y[k1][n2] in the workspace;
//   pass P (OP_PC, rows of Y in place): n2-point forward FFT giving
//          X[k1 + n1 k2], times F[k1 + n1 k2], n2-point inverse FFT over k2,
//          times W_n^{-k1 m2};
//   pass C: n1-point inverse FFTs down the columns into y[m2 + n2 m1].
// Three HBM round trips instead of five (forward four-step, multiply,
// inverse four-step), and no transposed store.
// Operand placement of a pulse chain: input, output, and the four-step
// intermediate (workspace offset), so the chain also runs on workspace
// buffers (Bluestein's convolution).
struct PulseIO {
    Loc src = Loc::In, dst = Loc::Out;
    size_t src_off = 0, dst_off = 0, scratch_off = 0;
    int mul_table = 0;  // 1: the filter is the plan's Bluestein table (set at device preparation)
};

void add_pulse_steps(FftPlan& plan, long long n, long long batch, const float2* filt, int flags, const PulseIO& pio) {
    const bool cj = (flags & kPulseConj) != 0;
    const bool sc = (flags & kPulseScale) != 0;
    const int mul_flags = cj ? TF_MUL_CONJ : 0;
    const int out_flags = sc ? TF_SCALE : 0;
    const float scale = 1.0f / (float)n;
    if (n <= kMaxTileN) {
        AxisIO io;
        io.inner = batch;
        io.in_idist = n;
        io.out_idist = n;
        Step st = make_tile_step(OP_PC, 1, (int)n, (int)n, false, io, mul_flags | out_flags, 0,
                                 "pulse rows n=" + std::to_string(n));
        st.L.args.mul = filt;
        st.L.args.mul_pitch_p = 0;
        st.L.args.mul_pitch_k = 1;
        st.L.args.scale = scale;
        st.batch_dim = 1;
        st.src = pio.src;
        st.dst = pio.dst;
        st.src_off = pio.src_off;
        st.dst_off = pio.dst_off;
        st.mul_table = pio.mul_table;
        plan.steps.push_back(st);
        return;
    }
    int n1 = 0, n2 = 0;
    if (!four_step_split(n, &n1, &n2))
        throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "length " + std::to_string(n) + " has no four-step split");
    int shift = 0;
    while ((1LL << (2 * shift)) < n) ++shift;
    const long long split_count = (1LL << shift) + (n + (1LL << shift) - 1) / (1LL << shift);
    AxisIO a;  // columns of x viewed as [n1][n2]
    a.inner = n2;
    a.outer = batch;
    a.in_odist = n;
    a.in_idist = 1;
    a.in_stride = n2;
    a.out_odist = n;
    a.out_idist = 1;
    a.out_stride = n2;
    Step sa = make_tile_step(OP_C2C, -1, n1, n1, true, a, 0, 0,
                             "four-step A n=" + std::to_string(n) + " n1=" + std::to_string(n1), true);
    sa.L.args.tw4_shift = shift;
    sa.tw2_kind = 2;
    sa.tw2_n = n;
    sa.tw2_count = split_count;
    sa.src = pio.src;
    sa.src_off = pio.src_off;
    sa.dst = Loc::Ws;
    sa.dst_off = pio.scratch_off;
    AxisIO r;  // rows of Y, in place
    r.inner = n1;
    r.outer = batch;
    r.in_odist = n;
    r.in_idist = n2;
    r.out_odist = n;
    r.out_idist = n2;
    Step sp = make_tile_step(OP_PC, 1, n2, n2, false, r, mul_flags, 0,
                             "pulse rows n=" + std::to_string(n) + " n2=" + std::to_string(n2), true);
    sp.L.args.tw4_shift = shift;
    sp.tw2_kind = 2;
    sp.tw2_n = n;
    sp.tw2_count = split_count;
    sp.L.args.mul = filt;
    sp.L.args.mul_pitch_p = 1;
    sp.L.args.mul_pitch_k = n1;
    sp.src = Loc::Ws;
    sp.dst = Loc::Ws;
    sp.src_off = sp.dst_off = pio.scratch_off;
    sp.mul_table = pio.mul_table;
    Step sc3 = make_tile_step(OP_C2C, 1, n1, n1, true, a, out_flags, 0,
                              "pulse inverse columns n=" + std::to_string(n) + " n1=" + std::to_string(n1));
    sc3.L.args.scale = scale;
    sc3.src = Loc::Ws;
    sc3.src_off = pio.scratch_off;
    sc3.dst = pio.dst;
    sc3.dst_off = pio.dst_off;
    sa.batch_dim = sp.batch_dim = sc3.batch_dim = 2;
    plan.steps.push_back(sa);
    plan.steps.push_back(sp);
    plan.steps.push_back(sc3);
    plan.workspace_need = std::max(plan.workspace_need, pio.scratch_off + (size_t)(batch * n * 8));
}

void add_pulse(FftPlan& plan) {
    add_pulse_steps(plan, plan.sizes[0], plan.batch, static_cast<const float2*>(plan.pulse_filter),
                    plan.pulse_flags, PulseIO{});
}

// Sets the fftshift epilogue on the step that writes the output: each
// output slice of rows x cols is rotated as asdFftShift (mode 1) or
// asdIfftShift (mode 2) would, and scaled.
void set_out_shift(Step& st, const FftPlan& plan, long long rows, long long cols) {
    TileArgs& a = st.L.args;
    a.flags |= TF_SHIFT_OUT;
    a.sh_rows = (int)rows;
    a.sh_cols = (int)cols;
    a.sh_slice = rows * cols;
    a.sh_r = (int)(plan.out_shift == 1 ? (rows + 1) / 2 : rows / 2);
    a.sh_c = (int)(plan.out_shift == 1 ? (cols + 1) / 2 : cols / 2);
    a.div_sh_cols = make_fastdiv((uint32_t)cols);
    if (plan.out_scale != 1.0) {
        a.flags |= TF_SCALE;
        a.scale = (float)plan.out_scale;
    }
    st.what += " + shift";
}

// C2C with the fftshift epilogue (1-D: slices of 1 x N; 2-D: slices of
// X x Y).  The rotation moves values across tiles, so the step that writes
// the output reads from another buffer: 1-D rows and the four-step pass B
// already do; 2-D runs its row pass into the workspace and the column pass
// from there into the output.  Generic tile kernels only.
void add_shifted_c2c(FftPlan& plan) {
    if (plan.type != ASCEND_FFT_C2C || plan.sizes.size() > 2)
        throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "output shift is for 1-D and 2-D C2C plans");
    g_hint_generic = 1;
    const long long b = plan.batch;
    if (plan.sizes.size() == 1) {
        const long long n = plan.sizes[0];
        add_c2c_1d(plan, n, b, C2COpts{});
        set_out_shift(plan.steps.back(), plan, 1, n);
        return;
    }
    const long long X = plan.sizes[0], Y = plan.sizes[1];
    if (X > kMaxTileN || Y > kMaxTileN || X * Y > 0x7fffffffLL)
        throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "multi-dimensional axis above one tile is not supported");
    AxisIO r;
    r.inner = b * X;
    r.in_idist = Y;
    r.out_idist = Y;
    Step rows = make_tile_step(OP_C2C, c2c_sign(plan), (int)Y, (int)Y, false, r, 0, 0,
                               "c2c axis 1 n=" + std::to_string(Y));
    rows.src = Loc::In;
    rows.dst = Loc::Ws;
    rows.chunk_dim = 1;
    rows.chunk_per = X;
    plan.steps.push_back(rows);
    AxisIO c;
    c.inner = Y;
    c.outer = b;
    c.in_odist = X * Y;
    c.in_idist = 1;
    c.in_stride = Y;
    c.out_odist = X * Y;
    c.out_idist = 1;
    c.out_stride = Y;
    Step cols = make_tile_step(OP_C2C, c2c_sign(plan), (int)X, (int)X, true, c, 0, 0,
                               "c2c axis 0 n=" + std::to_string(X));
    cols.src = Loc::Ws;
    cols.dst = Loc::Out;
    cols.chunk_dim = 2;
    cols.chunk_per = 1;
    set_out_shift(cols, plan, X, Y);
    plan.steps.push_back(cols);
    plan.workspace_need = (size_t)(b * X * Y * 8);
}

// Lengths the radix passes handle directly (the rest take Bluestein).
bool c2c_direct(long long n) {
    if (n <= kMaxTileN) return factorizable((int)n, 32);
    int n1 = 0, n2 = 0;
    return four_step_split(n, &n1, &n2);
}

bool real_direct(long long n) {
    if (n % 2 == 0) return c2c_direct(n / 2);
    return n <= kMaxTileN && factorizable((int)n, 32);
}

// Bluestein up to the reference's largest length (fft_api.cpp:82): the
// convolution length m <= 2^28 splits into two passes of at most 16384.
constexpr long long kMaxBluesteinN = 1LL << 27;

// Bluestein's algorithm (bluestein.cuh): pre pass into the workspace, the
// fused pulse chain of length m in place there (filter = the plan's
// Bluestein table, scale 1/m), post pass into the destination.  Workspace
// from ws_off: the convolution rows, then the four-step intermediate of m.
struct BlueIO {
    Loc src = Loc::In, dst = Loc::Out;
    size_t src_off = 0, dst_off = 0;
    size_t ws_off = 0;   // start of the Bluestein's own workspace
    int sign = 0;        // 0: the plan's direction
    float scale = 1.0f;  // on the post pass's outputs
};

void add_bluestein(FftPlan& plan, int kind, long long n, long long batch, const BlueIO& io = BlueIO{}) {
    if (n > kMaxBluesteinN)
        throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "length " + std::to_string(n) + " needs Bluestein above 2^27");
    const long long m = bluestein_length(n);
    const int sign = io.sign != 0 ? io.sign : (plan.forward() ? -1 : 1);
    if (kind == BLUE_C2C && m <= kMaxTileN) {
        // One size-specialized pulse tile per row does the whole transform:
        // chirp on load (zero padded to m), convolution, chirp on store
        // (TF_BLUE); the generic tile kernel has no such form, so without a
        // specialized kernel the three passes below run instead.
        AxisIO fio;
        fio.inner = batch;
        fio.in_idist = n;
        fio.out_idist = n;
        Step st = make_tile_step(OP_PC, 1, (int)m, (int)m, false, fio, TF_BLUE | TF_SCALE, 0,
                                 "bluestein n=" + std::to_string(n) + " m=" + std::to_string(m), false, (int)n);
        if (st.sk != nullptr) {
            st.L.args.mul_pitch_p = 0;
            st.L.args.mul_pitch_k = 1;
            st.L.args.scale = io.scale / (float)m;
            st.batch_dim = 1;
            st.mul_table = 1;
            st.tw2_kind = 3;  // the chirp c_j, j < n
            st.blue_n = n;
            st.blue_m = m;
            st.blue_sign = sign;
            st.src = io.src;
            st.src_off = io.src_off;
            st.dst = io.dst;
            st.dst_off = io.dst_off;
            plan.steps.push_back(st);
            return;
        }
    }
    const size_t conv = ((size_t)(batch * m * 8) + 255) / 256 * 256;
    Step pre;
    pre.kind = StepKind::Blue;
    pre.blue.n = n;
    pre.blue.m = m;
    pre.blue.rows = batch;
    pre.blue.kind = kind;
    pre.blue.in_pitch = kind == BLUE_C2R ? n / 2 + 1 : n;
    pre.blue.out_pitch = m;
    pre.blue_n = n;
    pre.blue_m = m;
    pre.blue_sign = sign;
    pre.src = io.src;
    pre.src_off = io.src_off;
    pre.dst = Loc::Ws;
    pre.dst_off = io.ws_off;
    pre.what = "bluestein pre n=" + std::to_string(n) + " m=" + std::to_string(m);
    plan.steps.push_back(pre);
    const size_t first = plan.steps.size();
    PulseIO pio;
    pio.src = pio.dst = Loc::Ws;
    pio.src_off = pio.dst_off = io.ws_off;
    pio.scratch_off = io.ws_off + conv;
    pio.mul_table = 1;
    add_pulse_steps(plan, m, batch, nullptr, kPulseScale, pio);
    for (size_t i = first; i < plan.steps.size(); ++i) {
        plan.steps[i].blue_n = n;
        plan.steps[i].blue_m = m;
        plan.steps[i].blue_sign = sign;
    }
    Step post = pre;
    post.blue_post = true;
    post.blue.in_pitch = m;
    post.blue.out_pitch = kind == BLUE_R2C ? n / 2 + 1 : n;
    post.blue.scale = io.scale;
    post.src = Loc::Ws;
    post.src_off = io.ws_off;
    post.dst = io.dst;
    post.dst_off = io.dst_off;
    post.what = "bluestein post n=" + std::to_string(n);
    plan.steps.push_back(post);
    plan.workspace_need =
        std::max(plan.workspace_need, io.ws_off + conv + (m > kMaxTileN ? (size_t)(batch * m * 8) : 0));
}

// Even real length n whose half length m = n/2 needs Bluestein: the
// half-length complex transform (real rows read as m complex values) runs
// through Bluestein, with the real post-process (R2C) after it or the real
// pre-process (C2R) before it, as the large-real path does around a
// four-step C2C.  The convolution is half as long as the full-length
// complex Bluestein's.  Workspace: [0, z) the m-point rows, then the
// Bluestein's own.
// C2R in a multi-D plan reads its half spectra from `c2r_src` (the column
// passes' output in the workspace) and puts its own workspace from ws_base.
void add_real_bluestein_half(FftPlan& plan, bool r2c, long long n, long long rows, Loc c2r_src = Loc::In,
                             size_t ws_base = 0) {
    if (r2c && (c2r_src != Loc::In || ws_base != 0))
        throw PlanError(ACL_ERROR_INTERNAL_ERROR, "real Bluestein R2C reads the input");
    const long long m = n / 2;
    const size_t zbytes = (size_t)(rows * m * 8);
    const size_t zoff = ws_base + (zbytes + 255) / 256 * 256;
    Step pp;
    pp.kind = r2c ? StepKind::RealPost : StepKind::RealPre;
    pp.real.m = m;
    pp.real.rows = rows;
    pp.real.conj = r2c ? (plan.forward() ? 0 : 1) : (plan.forward() ? 1 : 0);
    pp.tw2_kind = 1;
    pp.tw2_n = n;
    pp.tw2_count = m + 1;
    BlueIO io;
    io.ws_off = zoff;
    if (r2c) {
        io.sign = -1;
        io.src = Loc::In;
        io.dst = Loc::Ws;
        io.dst_off = 0;
        add_bluestein(plan, BLUE_C2C, m, rows, io);
        pp.real.in_pitch = m;
        pp.real.out_pitch = m + 1;
        pp.src = Loc::Ws;
        pp.src_off = 0;
        pp.dst = Loc::Out;
        pp.what = "r2c post n=" + std::to_string(n);
        plan.steps.push_back(pp);
    } else {
        pp.real.in_pitch = m + 1;
        pp.real.out_pitch = m;
        pp.src = c2r_src;
        pp.dst = Loc::Ws;
        pp.dst_off = ws_base;
        pp.what = "c2r pre n=" + std::to_string(n);
        plan.steps.push_back(pp);
        io.sign = 1;
        io.src = Loc::Ws;
        io.src_off = ws_base;
        io.dst = Loc::Out;
        io.scale = 2.0f;
        add_bluestein(plan, BLUE_C2C, m, rows, io);
    }
    plan.workspace_need = std::max(plan.workspace_need, zoff);
}

// Real transform along contiguous rows of length n (rows rows), one tile.
void add_real_rows(FftPlan& plan, bool r2c, long long n, long long rows, Loc src, Loc dst) {
    const long long h = n / 2 + 1;
    const int flags = r2c ? (plan.forward() ? 0 : TF_CONJ_OUT) : (plan.forward() ? TF_CONJ_IN : 0);
    if (n % 2 == 0) {
        const int m = (int)(n / 2);
        AxisIO io;
        io.inner = rows;
        io.in_idist = r2c ? m : h;
        io.out_idist = r2c ? h : m;
        Step st = make_tile_step(r2c ? OP_R2C_HALF : OP_C2R_HALF, r2c ? -1 : 1, m, r2c ? m : m + 1, false, io, flags,
                                 (int)rows, std::string(r2c ? "r2c" : "c2r") + " half n=" + std::to_string(n));
        st.tw2_kind = 1;
        st.tw2_n = n;
        st.tw2_count = m + 1;
        st.batch_dim = 1;
        st.src = src;
        st.dst = dst;
        plan.steps.push_back(st);
        return;
    }
    AxisIO io;
    io.inner = (rows + 1) / 2;
    io.in_idist = r2c ? n : h;
    io.out_idist = r2c ? h : n;
    Step st = make_tile_step(r2c ? OP_R2C_PAIR : OP_C2R_PAIR, r2c ? -1 : 1, (int)n, (int)n, false, io, flags,
                             (int)rows, std::string(r2c ? "r2c" : "c2r") + " pair n=" + std::to_string(n));
    st.src = src;
    st.dst = dst;
    plan.steps.push_back(st);
}

bool real_fits_tile(long long n) { return (n % 2 == 0) ? n / 2 <= kMaxTileN : n <= kMaxTileN; }

// Step of a mirrored four-step kernel (OP_R2C_4B / OP_C2R_4A), which only
// exist size-specialized: `e` is its registry entry.
Step mirrored_step(const SkEntry* e, int n, int n_other, long long rows, const AxisIO& io, int flags,
                   long long tw_n, const std::string& what) {
    Step st;
    st.sk = e;
    st.radices = e->radices;
    int tw_entries = 0;
    st.host_plan = make_plandev(n, st.radices, &tw_entries);
    TileLaunch& L = st.L;
    L.sign = e->sign;
    L.op = e->op;
    L.block = e->T;
    L.smem_bytes = e->smem;
    TileArgs& a = L.args;
    a.N = n;
    a.P = e->P / 2;  // first-half rows / columns per tile; the mirrors fill the other half
    a.LD = e->LD;
    a.n_other = n_other;
    a.inner = n_other / 2 + 1;
    a.tiles_per_outer = (a.inner + a.P - 1) / a.P;
    a.ntiles = (int)((long long)a.tiles_per_outer * rows);
    a.in_odist = io.in_odist;
    a.in_idist = io.in_idist;
    a.in_stride = io.in_stride;
    a.out_odist = io.out_odist;
    a.out_idist = io.out_idist;
    a.out_stride = io.out_stride;
    a.flags = flags;
    a.scale = 1.0f;
    a.div_n = make_fastdiv((uint32_t)n);
    a.div_p = make_fastdiv((uint32_t)a.P);
    a.div_h = make_fastdiv((uint32_t)(n / 2 + 1));
    a.div_tpo = make_fastdiv((uint32_t)a.tiles_per_outer);
    int shift = 0;
    while ((1LL << (2 * shift)) < tw_n) ++shift;
    a.tw4_shift = shift;
    st.tw2_kind = 2;
    st.tw2_n = tw_n;
    st.tw2_count = (1LL << shift) + (tw_n + (1LL << shift) - 1) / (1LL << shift);
    L.grid = a.ntiles;
    st.batch_dim = 2;
    st.what = what + " [sk mirrored P=" + std::to_string(e->P) + "]";
    return st;
}

// Odd real length above one tile whose complex FFT has a four-step split:
// real rows 2p and 2p + 1 travel as complex row p (x_a + i x_b) through the
// complex four-step of length n, between element-wise passes (R2C: pack, then
// separate the two rows' bins from Z[k] and Z[n-k]; C2R: combine the two half
// spectra into one complex spectrum, then split the real and imaginary
// parts).  Four HBM round trips of the packed data instead of Bluestein's
// convolution of twice the length.  Workspace: [0, zb) the packed rows
// (pass B of the four-step writes back there), then the four-step scratch.
// The reference takes such lengths whole into its arch35 real core
// (core/fft/fftcore/fft_r2c_arch35.cpp:121-148).
// C2R in a multi-D plan reads its half spectra from `c2r_src` (the column
// passes' output in the workspace) and puts its own workspace from ws_base.
void add_real_odd_large(FftPlan& plan, bool r2c, long long n, long long rows, Loc c2r_src = Loc::In,
                        size_t ws_base = 0) {
    if (r2c && (c2r_src != Loc::In || ws_base != 0))
        throw PlanError(ACL_ERROR_INTERNAL_ERROR, "large R2C reads the input");
    const long long pairs = (rows + 1) / 2;
    const size_t zb = ((size_t)(pairs * n * 8) + 255) / 256 * 256;
    const long long h = n / 2 + 1;
    Step first;
    first.kind = r2c ? StepKind::PairPack : StepKind::PairCombine;
    first.pair.n = n;
    first.pair.rows = rows;
    first.pair.in_pitch = r2c ? n : h;
    first.pair.out_pitch = n;
    first.pair.conj = (!r2c && plan.forward()) ? 1 : 0;
    first.src = c2r_src;
    first.dst = Loc::Ws;
    first.dst_off = ws_base;
    first.what = std::string(r2c ? "r2c pair pack" : "c2r pair combine") + " n=" + std::to_string(n);
    plan.steps.push_back(first);
    C2COpts o;
    o.sign = r2c ? -1 : 1;
    o.src = Loc::Ws;
    o.src_off = ws_base;
    o.dst = Loc::Ws;
    o.dst_off = ws_base;
    o.scratch_off = ws_base + zb;
    add_c2c_1d(plan, n, pairs, o);
    Step last;
    last.kind = r2c ? StepKind::PairSeparate : StepKind::PairSplit;
    last.pair.n = n;
    last.pair.rows = rows;
    last.pair.in_pitch = n;
    last.pair.out_pitch = r2c ? h : n;
    last.pair.conj = (r2c && !plan.forward()) ? 1 : 0;
    last.src = Loc::Ws;
    last.src_off = ws_base;
    last.dst = Loc::Out;
    last.what = std::string(r2c ? "r2c pair separate" : "c2r pair split") + " n=" + std::to_string(n);
    plan.steps.push_back(last);
    plan.workspace_need = std::max(plan.workspace_need, ws_base + zb + (size_t)(pairs * n * 8));
}

// Even real length whose half-length FFT M needs the four-step split.
// Fused form (both mirrored kernels compiled for the split): R2C = column
// pass A + row pass B with the post-process on mirrored row pairs; C2R =
// column pass A with the pre-process on mirrored column pairs + row pass B.
// Otherwise: the complex four-step over the workspace plus an element-wise
// pre/post pass.  Workspace: [0, zbytes) four-step scratch, then Z.
// By default R2C is fused and C2R is not: on B200 the fused C2R column pass
// (each element's mirror and pre-process twiddle read before the column FFT)
// is slower than a separate pre-process pass plus the plain four-step
// (2^20 x 256 rows: 2.12 ms fused, 1.74 ms unfused).  The real-fused planner
// hint selects either form for both directions.
// C2R in a multi-D plan reads its half spectra from `c2r_src` (the column
// passes' output in the workspace) and puts its own workspace from ws_base.
void add_real_large(FftPlan& plan, bool r2c, long long n, long long rows, Loc c2r_src = Loc::In,
                    size_t ws_base = 0) {
    if (r2c && (c2r_src != Loc::In || ws_base != 0))
        throw PlanError(ACL_ERROR_INTERNAL_ERROR, "large R2C reads the input");
    if (n % 2 != 0)
        throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "odd real length " + std::to_string(n) + " above one tile");
    const long long m = n / 2;
    const size_t zbytes = (size_t)(rows * m * 8);
    int n1 = 0, n2 = 0;
    const bool split = four_step_split(m, &n1, &n2);
    const bool generic_only = std::getenv("SIP_FFT_GENERIC_ONLY") != nullptr || g_hint_generic;
    // C2R stays unfused by default: its fused pass A, with the pre-process on
    // mirrored butterfly pairs too, measured slower (1.38 ms against 0.45 +
    // 0.60 ms for 2^20 x 256); the real-fused and variant hints select it.
    const bool fuse = g_hint_real_fused == 1 || (g_hint_real_fused == 0 && r2c);
    // R2C without a variant hint: the split whose pass B has the post-process
    // on mirrored butterfly pairs (rows of 512 for m = 2^19: 1.36 ms for
    // 2^20 x 256 against 1.46 with the 512 x 1024 split's pass B, which
    // holds 16 rows of 1024 in one CTA per SM)
    const SkEntry* pair_b = nullptr;
    if (split && !generic_only && fuse && r2c && g_hint_variant < 0 && !std::getenv("SIP_FFT_SPLIT_N1")) {
        for (const int b : {n1, n2}) {  // shorter rows first: smaller tiles, more CTAs per SM
            const SkEntry* e = sk_find_flags(OP_R2C_4B, SK_ROWS_T, -1, false, b, SK_MIRROR_PAIR);
            if (e != nullptr && sk_find(OP_C2C, SK_COLS, -1, true, (int)(m / b)) != nullptr) {
                pair_b = e;
                n1 = (int)(m / b);
                n2 = b;
                break;
            }
        }
    }
    if (split && !generic_only && fuse) {
        const SkEntry* ea = r2c ? sk_find(OP_C2C, SK_COLS, -1, true, n1)
                                : sk_find(OP_C2R_4A, SK_COLS, 1, false, n1, g_hint_variant);
        const SkEntry* eb = r2c ? (pair_b != nullptr ? pair_b : sk_find(OP_R2C_4B, SK_ROWS_T, -1, false, n2, g_hint_variant))
                                : sk_find(OP_C2C, SK_ROWS_T, 1, false, n2);
        if (ea != nullptr && eb != nullptr) {
            if (r2c) {
                C2COpts o;
                o.sign = -1;
                o.src = Loc::In;
                o.dst = Loc::Out;  // replaced: pass B below
                g_split_n1 = n1;   // pass A of this split
                try {
                    add_c2c_1d(plan, m, rows, o);
                } catch (...) {
                    g_split_n1 = 0;
                    throw;
                }
                g_split_n1 = 0;
                plan.steps.pop_back();  // keep pass A (column FFTs + cross twiddles) only
                AxisIO io;
                io.in_odist = m;
                io.in_idist = n2;
                io.in_stride = 1;
                io.out_odist = m + 1;
                io.out_idist = 1;
                io.out_stride = n1;
                Step sb = mirrored_step(eb, n2, n1, rows, io, plan.forward() ? 0 : TF_CONJ_OUT, 2 * m,
                                        "r2c four-step B + post n=" + std::to_string(n));
                sb.src = Loc::Ws;
                sb.dst = Loc::Out;
                plan.steps.push_back(sb);
            } else {
                AxisIO io;
                io.in_odist = m + 1;
                io.in_idist = 1;
                io.in_stride = n2;
                io.out_odist = m;
                io.out_idist = 1;
                io.out_stride = n2;
                Step sa = mirrored_step(ea, n1, n2, rows, io, plan.forward() ? TF_CONJ_IN : 0, 2 * m,
                                        "c2r pre + four-step A n=" + std::to_string(n));
                sa.src = c2r_src;
                sa.dst = Loc::Ws;
                sa.dst_off = ws_base;
                plan.steps.push_back(sa);
                AxisIO b;
                b.inner = n1;
                b.outer = rows;
                b.in_odist = m;
                b.in_idist = n2;
                b.in_stride = 1;
                b.out_odist = m;
                b.out_idist = 1;
                b.out_stride = n1;
                Step sb = make_tile_step(OP_C2C, 1, n2, n2, true, b, TF_SCALE, 0,
                                         "four-step B n=" + std::to_string(m) + " n2=" + std::to_string(n2));
                sb.L.args.scale = 2.0f;
                sb.batch_dim = 2;  // the batch rows are the outer index
                sb.src = Loc::Ws;
                sb.src_off = ws_base;
                sb.dst = Loc::Out;
                plan.steps.push_back(sb);
            }
            plan.workspace_need = std::max(plan.workspace_need, ws_base + zbytes);
            return;
        }
    }
    const size_t zoff = (zbytes + 255) / 256 * 256;
    Step pp;
    pp.kind = r2c ? StepKind::RealPost : StepKind::RealPre;
    pp.real.m = m;
    pp.real.rows = rows;
    pp.real.conj = r2c ? (plan.forward() ? 0 : 1) : (plan.forward() ? 1 : 0);
    pp.tw2_kind = 1;
    pp.tw2_n = n;
    pp.tw2_count = m + 1;
    C2COpts o;
    o.scratch_off = ws_base;
    if (r2c) {
        pp.real.in_pitch = m;
        pp.real.out_pitch = m + 1;
        pp.src = Loc::Ws;
        pp.src_off = zoff;
        pp.dst = Loc::Out;
        pp.what = "r2c post n=" + std::to_string(n);
        o.sign = -1;
        o.src = Loc::In;
        o.dst = Loc::Ws;
        o.dst_off = zoff;
        add_c2c_1d(plan, m, rows, o);
        plan.steps.push_back(pp);
    } else {
        pp.real.in_pitch = m + 1;
        pp.real.out_pitch = m;
        pp.src = c2r_src;
        pp.dst = Loc::Ws;
        pp.dst_off = ws_base + zoff;
        pp.what = "c2r pre n=" + std::to_string(n);
        plan.steps.push_back(pp);
        o.sign = 1;
        o.src = Loc::Ws;
        o.src_off = ws_base + zoff;
        o.dst = Loc::Out;
        o.last_flags = TF_SCALE;
        o.last_scale = 2.0f;
        add_c2c_1d(plan, m, rows, o);
    }
    plan.workspace_need = std::max(plan.workspace_need, ws_base + zoff + zbytes);
}

}  // namespace

bool apply_tune_cache(FftPlan& plan) {
    const char* path = std::getenv("SIP_FFT_TUNE_CACHE");
    if (path == nullptr) return false;
    FILE* f = std::fopen(path, "r");
    if (f == nullptr) return false;
    std::string dims;
    for (size_t i = 0; i < plan.sizes.size(); ++i) dims += (i ? "x" : "") + std::to_string(plan.sizes[i]);
    char line[512];
    bool hit = false;
    while (std::fgets(line, sizeof(line), f)) {
        int type = 0, dir = 0, p = 0, e = 0, gen = 0, order = 0, fused = 0, variant = 0, jit = 0;
        long long batch = 0;
        char d[256] = {0};
        const int got = std::sscanf(line, "%d %d %255s %lld %d %d %d %d %d %d %d", &type, &dir, d, &batch, &p, &e,
                                    &gen, &order, &fused, &variant, &jit);
        if (got < 8) continue;
        if (type == (int)plan.type && dir == (int)plan.direction && dims == d && batch == plan.batch) {
            plan.hint_p = p;
            plan.hint_e = e;
            plan.hint_generic = gen;
            plan.hint_order = order;
            plan.hint_real_fused = got >= 9 ? fused : 0;
            plan.hint_sk_variant = got >= 10 ? variant : -1;
            plan.hint_jit = got >= 11 ? jit : 0;
            hit = true;  // the last matching line wins
        }
    }
    std::fclose(f);
    return hit;
}

namespace {

std::atomic<long long> g_chunk_override{-1};

long long chunk_target_bytes() {
    const long long o = g_chunk_override.load();
    if (o >= 0) return o;
    static const long long target = [] {
        const char* e = std::getenv("SIP_FFT_L2_CHUNK_MB");
        if (e == nullptr || *e == '\0') return kL2ChunkBytes;
        const long long mb = std::atoll(e);
        return mb <= 0 ? 0LL : mb << 20;
    }();
    return target;
}

// Operand bytes one chunk unit spans on the input and output side of a step.
void chunk_slices(const Step& st, long long* in_b, long long* out_b) {
    if (st.kind == StepKind::Tile) {
        const TileArgs& a = st.L.args;
        *in_b = (st.chunk_dim == 2 ? a.in_odist : a.in_idist) * st.chunk_per * 8;
        *out_b = (st.chunk_dim == 2 ? a.out_odist : a.out_idist) * st.chunk_per * 8;
    } else {
        *in_b = st.real.in_pitch * 8 * st.chunk_per;
        *out_b = st.real.out_pitch * 8 * st.chunk_per;
    }
}

// Makes steps [first, last) one chunk group of `units` units when every
// step can run on a slice of the units: tile steps with a chunk dimension
// (not the two-rows-per-transform real ops) and the real pre/post passes.
// Input and output operands move by one slice per unit; workspace regions
// are reused by every chunk (a group holds every step that writes or reads
// them, so each chunk's intermediate is its own).
bool make_chunk_group(FftPlan& plan, size_t first, size_t last, long long units) {
    if (last - first < 2 || units < 2) return false;
    ChunkGroup g;
    g.first = first;
    g.last = last;
    g.units = units;
    for (size_t i = first; i < last; ++i) {
        const Step& st = plan.steps[i];
        if (st.chunk_group >= 0) return false;
        if (st.kind == StepKind::Tile) {
            if (st.chunk_dim != 1 && st.chunk_dim != 2) return false;
            if (st.L.op == OP_R2C_PAIR || st.L.op == OP_C2R_PAIR) return false;
        } else if (st.kind != StepKind::RealPre && st.kind != StepKind::RealPost) {
            return false;
        }
        long long ib = 0, ob = 0;
        chunk_slices(st, &ib, &ob);
        g.unit_bytes = std::max(g.unit_bytes, std::max(ib, ob));
    }
    for (size_t i = first; i < last; ++i) {
        Step& st = plan.steps[i];
        long long ib = 0, ob = 0;
        chunk_slices(st, &ib, &ob);
        st.chunk_group = (int)plan.chunk_groups.size();
        st.chunk_src = ib;
        st.chunk_dst = ob;
    }
    plan.chunk_groups.push_back(g);
    return true;
}

// Chunk groups of a built plan.  1-D plans (and pulse plans): every step
// carries the batch rows, so the whole chain runs row chunk by row chunk.
// Multi-D plans: whole batch items per chunk when an item fits the chunk
// size; otherwise, for 3-D, slabs of the outermost axis through the last-axis
// pass and the pass along the middle axis (the outermost-axis pass then runs
// over the whole volume).  Plans with other step kinds run unchunked.
void form_chunk_groups(FftPlan& plan) {
    plan.chunk_groups.clear();
    for (Step& st : plan.steps) st.chunk_group = -1;
    const size_t ns = plan.steps.size();
    // 1-D and pulse plans: a chunk unit is one batch row in every step (also
    // what a row-limited exec, launch_rows, runs on)
    if (plan.sizes.size() == 1 || plan.pulse)
        for (Step& st : plan.steps)
            if (st.kind == StepKind::Tile) {
                st.chunk_dim = st.batch_dim;
                st.chunk_per = 1;
            }
    if (ns < 2) return;
    if (plan.sizes.size() == 1 || plan.pulse) {
        make_chunk_group(plan, 0, ns, plan.batch);
        return;
    }
    // Multi-D chunks only on request (SIP_FFT_L2_CHUNK_MB or the test hook):
    // measured slower than the unchunked axis passes on B200 (2048^2 x 8:
    // 0.34 ms unchunked, 0.38-0.40 ms in chunks of one or two items).
    const char* req = std::getenv("SIP_FFT_L2_CHUNK_MB");
    if (g_chunk_override.load() < 0 && (req == nullptr || *req == '\0')) return;
    long long item = 8;
    for (int64_t s : plan.sizes) item *= s;
    const long long target = chunk_target_bytes();
    if (target > 0 && item <= target) {
        make_chunk_group(plan, 0, ns, plan.batch);
        return;
    }
    if (plan.sizes.size() == 3 && ns == 3 && plan.type != ASCEND_FFT_C2R) {
        const long long X = plan.sizes[0];
        Step& s0 = plan.steps[0];
        Step& s1 = plan.steps[1];
        if (s0.chunk_dim != 1 || s1.chunk_dim != 2 || s0.chunk_per % X != 0 || s1.chunk_per % X != 0) return;
        const long long p0 = s0.chunk_per, p1 = s1.chunk_per;
        s0.chunk_per /= X;
        s1.chunk_per /= X;
        if (!make_chunk_group(plan, 0, 2, plan.batch * X)) {
            s0.chunk_per = p0;
            s1.chunk_per = p1;
        }
    }
}

void build_steps_inner(FftPlan& plan);

}  // namespace

void set_l2_chunk_bytes(long long bytes) { g_chunk_override.store(bytes < 0 ? -1 : bytes); }

int chunk_lanes() {
    static const int v = [] {
        const char* e = std::getenv("SIP_FFT_L2_CHUNK_LANES");
        return (e != nullptr && std::atoi(e) == 1) ? 1 : 2;
    }();
    return v;
}

long long chunk_offset(const Step& st, bool src, long long u0, int lane, long long cu) {
    const Loc l = src ? st.src : st.dst;
    const long long slice = src ? st.chunk_src : st.chunk_dst;
    return l == Loc::Ws ? (long long)lane * cu * slice : u0 * slice;
}

// Smallest chunk unit that is chunked: on B200, running the passes chunk by
// chunk (one launch per step and chunk) costs more in launch gaps and
// partial waves than the L2 reuse saves for units of a few MB (2^20-point
// real rows, 65536-point rows, 2048^2 items: 1.2-1.7x slower), and pays for
// transforms of 2^21 points and more, whose strided column pass is slow
// from HBM (c2c 2^21 x 64: 4.1 ms unchunked, 1.8 ms in chunks of two rows).
// SIP_FFT_L2_CHUNK_MIN_MB overrides it (measurements).
long long chunk_min_unit_bytes() {
    if (g_chunk_override.load() >= 0) return 0;  // the test hook chunks every group
    static const long long v = [] {
        const char* e = std::getenv("SIP_FFT_L2_CHUNK_MIN_MB");
        return (e != nullptr && *e != '\0') ? std::max(0LL, (long long)std::atoll(e)) << 20 : kL2ChunkMinUnit;
    }();
    return v;
}

long long chunk_units(const ChunkGroup& g) {
    const long long target = chunk_target_bytes();
    if (target <= 0 || g.unit_bytes <= 0 || g.unit_bytes < chunk_min_unit_bytes()) return g.units;
    return std::max(1LL, std::min(g.units, target / g.unit_bytes));
}

long long exec_launches(const FftPlan& plan) {
    long long n = 0;
    for (size_t i = 0; i < plan.steps.size();) {
        const int gi = plan.steps[i].chunk_group;
        if (gi >= 0) {
            const ChunkGroup& g = plan.chunk_groups[gi];
            const long long cu = chunk_units(g);
            n += (long long)(g.last - g.first) * ((g.units + cu - 1) / cu);
            i = g.last;
        } else {
            ++n;
            ++i;
        }
    }
    return n;
}

bool rows_exec_supported(const FftPlan& plan) {
    if (plan.sizes.size() != 1 && !plan.pulse) return false;
    for (const Step& st : plan.steps) {
        if (st.kind == StepKind::Tile) {
            if (st.chunk_dim != 1 && st.chunk_dim != 2) return false;
            if (st.L.op == OP_R2C_PAIR || st.L.op == OP_C2R_PAIR) return false;
        } else if (st.kind != StepKind::RealPre && st.kind != StepKind::RealPost) {
            return false;
        }
    }
    return true;
}

TileLaunch chunk_tile_launch(const Step& st, long long cnt) {
    TileLaunch L = st.L;
    TileArgs& a = L.args;
    const long long n = cnt * st.chunk_per;
    if (st.chunk_dim == 1) {
        const long long outer = st.L.args.ntiles / st.L.args.tiles_per_outer;
        a.inner = (int)n;
        a.tiles_per_outer = (int)((n + a.P - 1) / a.P);
        a.div_tpo = make_fastdiv((uint32_t)a.tiles_per_outer);
        a.ntiles = (int)(a.tiles_per_outer * outer);
    } else {
        a.ntiles = (int)(a.tiles_per_outer * n);
    }
    L.grid = st.max_grid > 0 ? std::min(a.ntiles, st.max_grid) : a.ntiles;
    return L;
}

void build_steps(FftPlan& plan) {
    build_steps_inner(plan);
    form_chunk_groups(plan);
}

namespace {

void build_steps_inner(FftPlan& plan) {
    g_compute_mode = plan.compute_mode;
    g_hint_p = plan.hint_p;
    g_hint_e = plan.hint_e;
    g_hint_generic = plan.hint_generic;
    g_hint_order = plan.hint_order;
    g_hint_real_fused = plan.hint_real_fused;
    g_hint_variant = plan.hint_sk_variant;
    g_hint_jit = plan.hint_jit;
    plan.steps.clear();
    plan.workspace_need = 0;
    if (plan.pulse) {
        add_pulse(plan);
        return;
    }
    if (plan.out_shift != 0) {
        add_shifted_c2c(plan);
        return;
    }
    if (plan.type == ASCEND_FFT_C2C_SEP) {
        // separated planes: one generic tile pass per transform (the planar
        // load / store of tile_io.cuh); the reference limits the length to
        // 2..256, here any one-tile length works
        if (plan.sizes.size() != 1 || plan.sizes[0] > kMaxTileN)
            throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "separated C2C supports 1-D lengths up to one tile");
        g_hint_generic = 1;
        add_c2c_1d(plan, plan.sizes[0], plan.batch, C2COpts{});
        return;
    }
    const long long b = plan.batch;
    const auto& sz = plan.sizes;
    const bool c2c = plan.type == ASCEND_FFT_C2C || plan.type == ASCEND_FFT_C2C_SEP;
    const bool r2c = plan.type == ASCEND_FFT_R2C;
    if (sz.size() == 1) {
        const long long n = sz[0];
        if (plan.type == ASCEND_FFT_C2C && !c2c_direct(n)) {
            add_bluestein(plan, BLUE_C2C, n, b);
            return;
        }
        if (!c2c && n % 2 == 1 && n > kMaxTileN && c2c_direct(n)) {
            add_real_odd_large(plan, r2c, n, b);
            return;
        }
        if (!c2c && !real_direct(n)) {
            if (n % 2 == 0 && n / 2 <= kMaxBluesteinN)
                add_real_bluestein_half(plan, r2c, n, b);
            else
                add_bluestein(plan, r2c ? BLUE_R2C : BLUE_C2R, n, b);
            return;
        }
        if (c2c) {
            add_c2c_1d(plan, n, b, C2COpts{});
        } else if (real_fits_tile(n)) {
            add_real_rows(plan, r2c, n, b, Loc::In, Loc::Out);
        } else {
            add_real_large(plan, r2c, n, b);
        }
        return;
    }
    // Multi-dimensional: the last axis is contiguous, the others are
    // strided column passes done in place on the destination.
    const int nd = (int)sz.size();
    for (int i = 0; i < nd - 1; ++i)
        if (sz[i] > kMaxTileN)
            throw PlanError(ACL_ERROR_API_NOT_SUPPORT, "multi-dimensional axis above one tile is not supported");
    const long long last = sz[nd - 1];
    // A last axis above one tile, or one that needs Bluestein, runs as the
    // batched 1-D transform of the rows, routed as a 1-D plan of that
    // length would be: C2C four-step or Bluestein; real: one tile, the
    // half-length four-step (even), row pairs through the complex four-step
    // (odd), or Bluestein (half length when even)
    enum { kRows, kLarge, kOddLarge, kBlueHalf, kBlue };
    const int real_route = c2c ? kRows
                         : (real_fits_tile(last) && real_direct(last)) ? kRows
                         : (last % 2 == 0 && real_direct(last)) ? kLarge
                         : (last % 2 == 1 && last > kMaxTileN && c2c_direct(last)) ? kOddLarge
                         : (last % 2 == 0 && last / 2 <= kMaxBluesteinN) ? kBlueHalf
                                                                           : kBlue;
    const long long lastc = c2c ? last : last / 2 + 1;  // complex extent of the last axis
    long long rows = b;
    for (int i = 0; i < nd - 1; ++i) rows *= sz[i];
    // Column pass along axis `ax` of the complex array [b][sz0]..[lastc].
    auto column_pass = [&](int ax, Loc src, Loc dst) {
        long long inner = lastc;
        for (int i = ax + 1; i < nd - 1; ++i) inner *= sz[i];
        long long outer = b;
        for (int i = 0; i < ax; ++i) outer *= sz[i];
        const long long n = sz[ax];
        AxisIO io;
        io.inner = inner;
        io.outer = outer;
        io.in_odist = n * inner;
        io.in_idist = 1;
        io.in_stride = inner;
        io.out_odist = n * inner;
        io.out_idist = 1;
        io.out_stride = inner;
        Step st = make_tile_step(OP_C2C, c2c_sign(plan), (int)n, (int)n, true, io, 0, 0,
                                 "c2c axis " + std::to_string(ax) + " n=" + std::to_string(n));
        st.src = src;
        st.dst = dst;
        st.chunk_dim = 2;  // outer index: the batch item, then the axes before ax
        st.chunk_per = outer / b;
        plan.steps.push_back(st);
    };
    // the contiguous last-axis pass: rows / b rows per batch item
    auto rows_chunks = [&]() {
        Step& st = plan.steps.back();
        if (st.L.op == OP_R2C_PAIR || st.L.op == OP_C2R_PAIR) return;  // two rows per transform
        st.chunk_dim = 1;
        st.chunk_per = rows / b;
    };
    if (c2c) {
        if (last <= kMaxTileN && factorizable((int)last, 32)) {
            AxisIO io;
            io.inner = rows;
            io.in_idist = last;
            io.out_idist = last;
            Step st = make_tile_step(OP_C2C, c2c_sign(plan), (int)last, (int)last, false, io, 0, 0,
                                     "c2c axis " + std::to_string(nd - 1) + " n=" + std::to_string(last));
            st.src = Loc::In;
            st.dst = Loc::Out;
            plan.steps.push_back(st);
            rows_chunks();
        } else if (c2c_direct(last)) {
            // the steps of the 1-D plan of `rows` rows (their chunk fields
            // stay unset, so no multi-D chunk group takes them)
            C2COpts o;
            o.src = Loc::In;
            o.dst = Loc::Out;
            add_c2c_1d(plan, last, rows, o);
        } else {
            add_bluestein(plan, BLUE_C2C, last, rows);
        }
        for (int ax = nd - 2; ax >= 0; --ax) column_pass(ax, Loc::Out, Loc::Out);
    } else if (r2c) {
        if (real_route == kRows) {
            add_real_rows(plan, true, last, rows, Loc::In, Loc::Out);
            rows_chunks();
        } else if (real_route == kLarge) {
            add_real_large(plan, true, last, rows);
        } else if (real_route == kOddLarge) {
            add_real_odd_large(plan, true, last, rows);
        } else if (real_route == kBlueHalf) {
            add_real_bluestein_half(plan, true, last, rows);
        } else {
            add_bluestein(plan, BLUE_R2C, last, rows);
        }
        for (int ax = nd - 2; ax >= 0; --ax) column_pass(ax, Loc::Out, Loc::Out);
    } else {
        column_pass(nd - 2, Loc::In, Loc::Ws);
        for (int ax = nd - 3; ax >= 0; --ax) column_pass(ax, Loc::Ws, Loc::Ws);
        plan.workspace_need = (size_t)(rows * lastc * 8);
        const size_t base = (plan.workspace_need + 255) / 256 * 256;
        if (real_route == kRows) {
            add_real_rows(plan, false, last, rows, Loc::Ws, Loc::Out);
            rows_chunks();
        } else if (real_route == kLarge) {
            add_real_large(plan, false, last, rows, Loc::Ws, base);
        } else if (real_route == kOddLarge) {
            add_real_odd_large(plan, false, last, rows, Loc::Ws, base);
        } else if (real_route == kBlueHalf) {
            add_real_bluestein_half(plan, false, last, rows, Loc::Ws, base);
        } else {
            BlueIO io;
            io.src = Loc::Ws;
            io.ws_off = base;
            add_bluestein(plan, BLUE_C2R, last, rows, io);
        }
    }
}

}  // namespace

std::string describe(const FftPlan& plan) {
    static const char* locs[] = {"in", "out", "ws"};
    std::ostringstream os;
    os << "{\"type\":" << (int)plan.type << ",\"forward\":" << (plan.forward() ? "true" : "false")
       << ",\"batch\":" << plan.batch << ",\"sizes\":[";
    for (size_t i = 0; i < plan.sizes.size(); ++i) os << (i ? "," : "") << plan.sizes[i];
    os << "],\"workspace\":" << plan.workspace_need << ",\"launches\":" << exec_launches(plan)
       << ",\"chunk_groups\":[";
    for (size_t i = 0; i < plan.chunk_groups.size(); ++i) {
        const ChunkGroup& g = plan.chunk_groups[i];
        os << (i ? "," : "") << "{\"first\":" << g.first << ",\"last\":" << g.last << ",\"units\":" << g.units
           << ",\"unit_bytes\":" << g.unit_bytes << ",\"chunk_units\":" << chunk_units(g) << "}";
    }
    os << "],\"steps\":[";
    for (size_t i = 0; i < plan.steps.size(); ++i) {
        const Step& st = plan.steps[i];
        os << (i ? "," : "") << "{\"what\":\"" << st.what << "\",\"kind\":" << (int)st.kind << ",\"src\":\""
           << locs[(int)st.src] << "\",\"dst\":\"" << locs[(int)st.dst] << "\",\"src_off\":" << st.src_off
           << ",\"dst_off\":" << st.dst_off << ",\"chunk_group\":" << st.chunk_group;
        if (st.kind == StepKind::Tile || st.kind == StepKind::Tc) {
            const TileArgs& a = st.L.args;
            os << ",\"op\":" << st.L.op << ",\"sign\":" << st.L.sign << ",\"e\":" << st.L.e << ",\"n\":" << a.N
               << ",\"P\":" << a.P << ",\"LD\":" << a.LD << ",\"threads\":" << st.L.block << ",\"grid\":" << st.L.grid
               << ",\"smem\":" << st.L.smem_bytes << ",\"tw4\":" << (st.L.tw4 ? "true" : "false")
               << ",\"flags\":" << a.flags << ",\"inner\":" << a.inner << ",\"tiles_per_outer\":" << a.tiles_per_outer
               << ",\"in\":[" << a.in_odist << "," << a.in_idist << "," << a.in_stride << "],\"out\":["
               << a.out_odist << "," << a.out_idist << "," << a.out_stride << "],\"sk\":" << (st.sk ? "true" : "false")
               << ",\"jit\":" << (st.sk && st.sk->jit ? "true" : "false");
            if (st.sk)  // the compiled configuration (SkCfg<N, P, T, OP, MODE, SIGN, TW4, MINB, TWB, radices>)
                os << ",\"sk_cfg\":[" << st.sk->n << "," << st.sk->P << "," << st.sk->T << "," << st.sk->op << ","
                   << st.sk->mode << "," << st.sk->sign << "," << (st.sk->tw4 ? 1 : 0) << "," << st.sk->minb << ","
                   << st.sk->flags << "]";
            os << ",\"radices\":[";
            for (size_t r = 0; r < st.radices.size(); ++r) os << (r ? "," : "") << st.radices[r];
            os << "]";
        } else if (st.kind == StepKind::Blue) {
            os << ",\"n\":" << st.blue.n << ",\"m\":" << st.blue.m << ",\"rows\":" << st.blue.rows
               << ",\"post\":" << (st.blue_post ? "true" : "false");
        } else if (is_pair_kind(st.kind)) {
            os << ",\"n\":" << st.pair.n << ",\"rows\":" << st.pair.rows << ",\"conj\":" << st.pair.conj;
        } else if (st.kind == StepKind::Cluster) {
            os << ",\"n\":" << st.cl->n << ",\"cluster\":" << st.cl->C << ",\"threads\":" << st.cl->T
               << ",\"transforms\":" << st.cl_transforms << ",\"sign\":" << st.cl->sign;
        } else {
            os << ",\"m\":" << st.real.m << ",\"rows\":" << st.real.rows << ",\"conj\":" << st.real.conj;
        }
        os << "}";
    }
    os << "]}";
    return os.str();
}

}  // namespace sipfft
