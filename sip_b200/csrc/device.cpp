// Device resources of plans and step launching.
//
// Twiddle tables are cached per (device, kind, parameters) through
// weak_ptr, so plans of the same length share one device copy and the
// copy is freed with its last plan (the reference's FFTensorCache,
// core/fft/utils/fftensor_cache.cpp:82-101).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>

#include "jit.h"
#include "noalloc.h"
#include "plan.h"
#include "tc_core.cuh"
#include "tc_launch.h"

namespace sipfft {

namespace {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw PlanError(AsdSip::ACL_ERROR_INTERNAL_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

struct TableKey {
    int device;
    int kind;  // 0 stockham, 1 roots, 2 basis, 3 split cross twiddles, 4 tensor-core B operand,
               // 5 Bluestein chirp, 6 Bluestein filter
    long long a, b;
    std::vector<int> radices;
    bool operator<(const TableKey& o) const {
        return std::tie(device, kind, a, b, radices) < std::tie(o.device, o.kind, o.a, o.b, o.radices);
    }
};

std::mutex g_table_mu;
std::map<TableKey, std::weak_ptr<DeviceBuf>> g_tables;

BufPtr alloc_buf(size_t bytes, int device) {
    auto b = std::make_shared<DeviceBuf>();
    b->device = device;
    b->bytes = bytes;
    if (bytes > 0) check(cudaMalloc(&b->ptr, bytes), "cudaMalloc");
    return b;
}

// Runs `gen` on a private non-blocking stream and waits for it.
template <class F>
void run_sync(F gen) {
    cudaStream_t s = nullptr;
    check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaError_t e = gen(s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    check(e, "table generation");
}

BufPtr stockham_table(int device, const PlanDev& pd, const std::vector<int>& radices) {
    int entries = 0;
    for (int i = 0; i < pd.npass; ++i)
        if (pd.pass[i].L > 1) entries = pd.pass[i].tw + pd.pass[i].L * (pd.pass[i].R - 1);
    TableKey key{device, 0, pd.N, 0, radices};
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_tables.find(key);
    if (it != g_tables.end())
        if (auto sp = it->second.lock()) return sp;
    BufPtr b = alloc_buf((size_t)std::max(entries, 1) * sizeof(float2), device);
    run_sync([&](cudaStream_t s) { return gen_stockham_twiddles(static_cast<float2*>(b->ptr), pd, entries, s); });
    g_tables[key] = b;
    return b;
}

BufPtr basis_table(int device, const PlanDev& pd, const std::vector<int>& radices) {
    const int entries = basis_entries(pd);
    TableKey key{device, 2, pd.N, 0, radices};
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_tables.find(key);
    if (it != g_tables.end())
        if (auto sp = it->second.lock()) return sp;
    BufPtr b = alloc_buf((size_t)std::max(entries, 1) * sizeof(float2), device);
    run_sync([&](cudaStream_t s) { return gen_basis_twiddles(static_cast<float2*>(b->ptr), pd, s); });
    g_tables[key] = b;
    return b;
}

// Split B operand (3 x 2 KB, core-matrix layout) of the DFT-16 stage.
BufPtr tc_bmat_table(int device, int sign) {
    TableKey key{device, 4, sign, 0, {}};
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_tables.find(key);
    if (it != g_tables.end())
        if (auto sp = it->second.lock()) return sp;
    std::vector<uint16_t> host(3 * kTcK * kTcK);
    tc_make_b(sign, host.data());
    BufPtr b = alloc_buf(host.size() * sizeof(uint16_t), device);
    check(cudaMemcpy(b->ptr, host.data(), host.size() * sizeof(uint16_t), cudaMemcpyHostToDevice), "cudaMemcpy");
    g_tables[key] = b;
    return b;
}

BufPtr root_table(int device, long long n, long long count) {
    TableKey key{device, 1, n, count, {}};
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_tables.find(key);
    if (it != g_tables.end())
        if (auto sp = it->second.lock()) return sp;
    BufPtr b = alloc_buf((size_t)count * sizeof(float2), device);
    run_sync([&](cudaStream_t s) { return gen_root_twiddles(static_cast<float2*>(b->ptr), n, count, s); });
    g_tables[key] = b;
    return b;
}

BufPtr split_table(int device, long long n, int shift) {
    const long long B = 1LL << shift;
    const long long count = B + (n + B - 1) / B;
    TableKey key{device, 3, n, shift, {}};
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_tables.find(key);
    if (it != g_tables.end())
        if (auto sp = it->second.lock()) return sp;
    BufPtr b = alloc_buf((size_t)count * sizeof(float2), device);
    run_sync([&](cudaStream_t s) { return gen_split_twiddles(static_cast<float2*>(b->ptr), n, shift, s); });
    g_tables[key] = b;
    return b;
}

BufPtr chirp_table(int device, long long n, int sign) {
    TableKey key{device, 5, n, sign, {}};
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_tables.find(key);
    if (it != g_tables.end())
        if (auto sp = it->second.lock()) return sp;
    BufPtr b = alloc_buf((size_t)n * sizeof(float2), device);
    run_sync([&](cudaStream_t s) { return gen_chirp(static_cast<float2*>(b->ptr), n, sign, s); });
    g_tables[key] = b;
    return b;
}

// Filter of a long Bluestein convolution made on the GPU: the sequence b in
// FP64 (rounded once), then the library's own forward C2C plan of length m
// (2,3,5-smooth, so it never needs Bluestein itself) in FP32.
BufPtr blue_filter_gpu(int device, long long n, long long m, int sign) {
    BufPtr seq = alloc_buf((size_t)m * sizeof(float2), device);
    BufPtr out = alloc_buf((size_t)m * sizeof(float2), device);
    run_sync([&](cudaStream_t s) { return gen_blue_b(static_cast<float2*>(seq->ptr), n, m, sign, s); });
    FftPlan p;
    p.type = AsdSip::ASCEND_FFT_C2C;
    p.direction = AsdSip::ASCEND_FFT_FORWARD;
    p.sizes = {m};
    p.batch = 1;
    build_steps(p);
    prepare_device(p);
    BufPtr ws = alloc_buf(p.workspace_need, device);
    run_sync([&](cudaStream_t s) {
        p.stream = s;
        launch_steps(p, seq->ptr, out->ptr, ws->ptr);
        return cudaGetLastError();
    });
    return out;
}

BufPtr blue_filter_table(int device, long long n, long long m, int sign) {
    TableKey key{device, 6, n, m * 2 + (sign > 0 ? 1 : 0), {}};
    {
        std::lock_guard<std::mutex> lk(g_table_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end())
            if (auto sp = it->second.lock()) return sp;
    }
    // made without the table lock: the GPU form prepares a plan of its own,
    // whose twiddle tables go through the same cache
    BufPtr b;
    if (m > kHostBlueFilterMax) {
        b = blue_filter_gpu(device, n, m, sign);
    } else {
        const std::vector<float2> host = bluestein_filter(n, m, sign);
        b = alloc_buf(host.size() * sizeof(float2), device);
        check(cudaMemcpy(b->ptr, host.data(), host.size() * sizeof(float2), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    std::lock_guard<std::mutex> lk(g_table_mu);
    auto it = g_tables.find(key);
    if (it != g_tables.end())
        if (auto sp = it->second.lock()) return sp;  // made by another thread meanwhile
    g_tables[key] = b;
    return b;
}

}  // namespace

ChunkLanes::~ChunkLanes() {
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (side) cudaStreamDestroy(side);
}

void prepare_device(FftPlan& plan) {
    int device = -1;
    check(cudaGetDevice(&device), "cudaGetDevice");
    // The second lane (a stream and two events) only for plans that run in
    // chunks under the current settings: creating and destroying a stream
    // costs a few hundred microseconds, which plans made per request (a
    // serving loop's plain path) would pay every time.  A plan without it
    // runs its chunks on one lane.
    bool chunked = false;
    for (const ChunkGroup& g : plan.chunk_groups) chunked = chunked || chunk_units(g) < g.units;
    if (chunked) {
        auto l = std::make_shared<ChunkLanes>();
        check(cudaStreamCreateWithFlags(&l->side, cudaStreamNonBlocking), "cudaStreamCreate");
        check(cudaEventCreateWithFlags(&l->fork, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaEventCreateWithFlags(&l->join, cudaEventDisableTiming), "cudaEventCreate");
        plan.lanes = l;
    }
    for (Step& st : plan.steps) {
        if (is_pair_kind(st.kind)) continue;  // no tables
        if (st.kind == StepKind::Cluster) {
            st.tw = basis_table(device, st.host_plan, st.radices);
            st.tw_b = basis_table(device, st.cl_plan_b, st.cl_radices_b);
            st.tw2 = split_table(device, st.tw2_n, st.cl_b.tw4_shift);
            st.L.args.tw = static_cast<const float2*>(st.tw->ptr);
            st.cl_b.tw = static_cast<const float2*>(st.tw_b->ptr);
            st.cl_b.tw2 = static_cast<const float2*>(st.tw2->ptr);
            check(cluster_prepare(st.cl), "cluster_prepare");
            continue;
        }
        if (st.kind == StepKind::Blue) {
            st.chirp_buf = chirp_table(device, st.blue_n, st.blue_sign);
            st.blue.chirp = static_cast<const float2*>(st.chirp_buf->ptr);
            check(bluestein_prepare(), "bluestein_prepare");
            continue;
        }
        if (st.mul_table == 1) {
            st.mul_buf = blue_filter_table(device, st.blue_n, st.blue_m, st.blue_sign);
            st.L.args.mul = static_cast<const float2*>(st.mul_buf->ptr);
        }
        if (st.tw2_kind == 1) st.tw2 = root_table(device, st.tw2_n, st.tw2_count);
        if (st.tw2_kind == 2) st.tw2 = split_table(device, st.tw2_n, st.L.args.tw4_shift);
        if (st.tw2_kind == 3) st.tw2 = chirp_table(device, st.blue_n, st.blue_sign);
        if (st.kind == StepKind::RealPost || st.kind == StepKind::RealPre) {
            st.real.tw = static_cast<const float2*>(st.tw2->ptr);
            continue;
        }
        if (st.kind == StepKind::Tc) {
            st.tc_bmat = tc_bmat_table(device, st.L.sign);
            st.tw = root_table(device, 256, 256);
            st.L.args.tw = static_cast<const float2*>(st.tw->ptr);
            st.L.args.tw2 = st.tw2 ? static_cast<const float2*>(st.tw2->ptr) : nullptr;
            st.tc_fn = tc_kernel(st.L.sign, st.L.tw4, st.tc_cols_in, st.tc_cols_out);
            int per_sm = 1, sms = 1;
            check(tc_prepare(st.tc_fn, &per_sm), "tc_prepare");
            check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
            st.L.grid = (int)std::min<long long>(st.L.args.ntiles, (long long)sms * (per_sm > 0 ? per_sm : 1));
            continue;
        }
        st.tw = (st.sk && st.sk->twb) ? basis_table(device, st.host_plan, st.radices)
                                      : stockham_table(device, st.host_plan, st.radices);
        st.plan_dev = alloc_buf(sizeof(PlanDev), device);
        check(cudaMemcpy(st.plan_dev->ptr, &st.host_plan, sizeof(PlanDev), cudaMemcpyHostToDevice), "cudaMemcpy");
        st.L.args.plan = static_cast<const PlanDev*>(st.plan_dev->ptr);
        st.L.args.tw = static_cast<const float2*>(st.tw->ptr);
        st.L.args.tw2 = st.tw2 ? static_cast<const float2*>(st.tw2->ptr) : nullptr;
        if (st.sk != nullptr) {
            int per_sm = 1, sms = 1;
            // run-time specialized kernels are compiled (or fetched from the
            // cache) on first use
            const void* fn = st.sk->jit ? sk_jit_load(st.sk) : st.sk->fn;
            check(sk_prepare(fn, st.L.smem_bytes, st.L.block, &per_sm), "sk_prepare");
            check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "cudaDeviceGetAttribute");
            const long long resident = (long long)sms * (per_sm > 0 ? per_sm : 1);
            st.L.grid = (int)std::min<long long>(st.L.args.ntiles, resident);
            st.max_grid = (int)std::min<long long>(resident, 0x7fffffffLL);
            st.L.sk_fn = fn;
        } else {
            check(tile_prepare(st.L.sign, st.L.e, st.L.op, st.L.tw4, st.L.smem_bytes), "cudaFuncSetAttribute");
        }
    }
    plan.device = device;
    // the static scratch of the no-alloc exec is looked up (and, under lazy
    // module loading, reserved) here rather than in that exec call
    noalloc_resolve(plan);
    plan.resources_ready = true;
}

void launch_separated(const FftPlan& plan, const float* in_re, const float* in_im, float* out_re, float* out_im) {
    if (plan.steps.size() != 1 || plan.steps[0].kind != StepKind::Tile || plan.steps[0].sk != nullptr)
        throw PlanError(AsdSip::ACL_ERROR_INTERNAL_ERROR, "separated plan must be one generic tile step");
    TileLaunch L = plan.steps[0].L;
    L.args.flags |= TF_PLANAR_IN | TF_PLANAR_OUT;
    L.args.src_im = in_im;
    L.args.dst_im = out_im;
    check(tile_launch(L, in_re, out_re, static_cast<cudaStream_t>(plan.stream)), "tile kernel launch");
}

namespace {

// Launches one step, restricted to chunk units [u0, u0 + cnt) of its chunk
// group on lane `lane` (cu units per chunk) when cnt >= 0 (cnt < 0: the whole
// step as planned).
void launch_one(const Step& st, cudaStream_t stream, const void* in, void* out, void* ws, long long u0,
                long long cnt, int lane = 0, long long cu = 0) {
    auto resolve = [&](Loc l, size_t off) -> char* {
        char* base = nullptr;
        switch (l) {
            case Loc::In: base = const_cast<char*>(static_cast<const char*>(in)); break;
            case Loc::Out: base = static_cast<char*>(out); break;
            case Loc::Ws: base = static_cast<char*>(ws); break;
        }
        return base + off;
    };
    char* src = resolve(st.src, st.src_off);
    char* dst = resolve(st.dst, st.dst_off);
    if (cnt >= 0) {
        src += chunk_offset(st, true, u0, lane, cu);
        dst += chunk_offset(st, false, u0, lane, cu);
    }
    if (st.kind == StepKind::Tile) {
        if (cnt < 0) {
            check(tile_launch(st.L, src, dst, stream), "tile kernel launch");
            return;
        }
        check(tile_launch(chunk_tile_launch(st, cnt), src, dst, stream), "tile kernel launch");
    } else if (st.kind == StepKind::Blue) {
        BluesteinArgs a = st.blue;
        a.src = src;
        a.dst = dst;
        check(st.blue_post ? bluestein_post(a, stream) : bluestein_pre(a, stream), "bluestein pass launch");
    } else if (st.kind == StepKind::Tc) {
        check(tc_launch(st.tc_fn, st.L.grid, st.L.args, src, dst, static_cast<const uint16_t*>(st.tc_bmat->ptr),
                        st.L.args.tw, stream),
              "tensor-core kernel launch");
    } else if (st.kind == StepKind::Cluster) {
        TileArgs a = st.L.args, b = st.cl_b;
        a.src = src;
        b.dst = dst;
        check(cluster_launch(st.cl, st.cl_transforms, a, b, stream), "cluster kernel launch");
    } else if (is_pair_kind(st.kind)) {
        PairPassArgs a = st.pair;
        a.src = src;
        a.dst = dst;
        cudaError_t e = cudaSuccess;
        switch (st.kind) {
            case StepKind::PairPack: e = pair_pack(a, stream); break;
            case StepKind::PairSeparate: e = pair_separate(a, stream); break;
            case StepKind::PairCombine: e = pair_combine(a, stream); break;
            default: e = pair_split(a, stream); break;
        }
        check(e, "pair pass launch");
    } else {
        RealPassArgs a = st.real;
        a.src = reinterpret_cast<const float2*>(src);
        a.dst = reinterpret_cast<float2*>(dst);
        if (cnt >= 0) a.rows = cnt * st.chunk_per;
        check(st.kind == StepKind::RealPost ? real_post(a, stream) : real_pre(a, stream), "real pass launch");
    }
}

}  // namespace

// A row-limited exec: every step as chunk units [0, rows) (a unit is one
// batch row in 1-D and pulse plans), workspace regions at their start.
void launch_rows(const FftPlan& plan, long long rows, const void* in, void* out, void* ws) {
    cudaStream_t stream = static_cast<cudaStream_t>(plan.stream);
    for (const Step& st : plan.steps) launch_one(st, stream, in, out, ws, 0, rows);
}

// Steps of a chunk group run chunk by chunk: every step of the group on
// units [u0, u0 + cu), then the next chunk.  The workspace regions of the
// group are reused by every chunk, so the intermediate one step writes and
// the next reads stays in L2 and the chain costs about one HBM round trip
// of its input and output instead of one per step.
void launch_steps(const FftPlan& plan, const void* in, void* out, void* ws) {
    cudaStream_t stream = static_cast<cudaStream_t>(plan.stream);
    for (size_t i = 0; i < plan.steps.size();) {
        const int gi = plan.steps[i].chunk_group;
        if (gi >= 0) {
            const ChunkGroup& g = plan.chunk_groups[gi];
            const long long cu = chunk_units(g);
            if (cu < g.units) {
                // lane 0 is the plan's stream; lane 1 forks from it and joins
                // it again after the group
                const bool two = plan.lanes != nullptr && chunk_lanes() == 2;
                cudaStream_t side = two ? plan.lanes->side : nullptr;
                if (two) {
                    check(cudaEventRecord(plan.lanes->fork, stream), "cudaEventRecord");
                    check(cudaStreamWaitEvent(side, plan.lanes->fork, 0), "cudaStreamWaitEvent");
                }
                int k = 0;
                for (long long u0 = 0; u0 < g.units; u0 += cu, ++k) {
                    const long long cnt = std::min(cu, g.units - u0);
                    const int lane = two ? (k & 1) : 0;
                    for (size_t j = g.first; j < g.last; ++j)
                        launch_one(plan.steps[j], lane ? side : stream, in, out, ws, u0, cnt, lane, cu);
                }
                if (two) {
                    check(cudaEventRecord(plan.lanes->join, side), "cudaEventRecord");
                    check(cudaStreamWaitEvent(stream, plan.lanes->join, 0), "cudaStreamWaitEvent");
                }
                i = g.last;
                continue;
            }
        }
        launch_one(plan.steps[i], stream, in, out, ws, 0, -1);
        ++i;
    }
}

}  // namespace sipfft
