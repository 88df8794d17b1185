// Batched execution of many planned handles in one persistent queue launch
// per wave (queue.cu), replayed from captured CUDA graphs.
//
// Descriptors are written to a pinned host buffer and copied to the device
// by the first node of the launch sequence, so a captured graph stays valid
// for any batch with the same wave count, shared-memory size and buffer
// capacity: the per-wave item and tile counts travel in the copied header.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "plan.h"
#include "queue.h"

namespace sipfft {

namespace {

void chk(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw PlanError(AsdSip::ACL_ERROR_INTERNAL_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

bool queueable(const Step& st) {
    return st.kind == StepKind::Tile && st.sk == nullptr && st.L.smem_bytes <= kQueueMaxSmem &&
           (st.L.op == OP_C2C || st.L.op == OP_R2C_HALF || st.L.op == OP_C2R_HALF || st.L.op == OP_R2C_PAIR ||
            st.L.op == OP_C2R_PAIR || st.L.op == OP_PC);
}

}  // namespace

Batch* batch_create() {
    auto b = std::make_unique<Batch>();
    chk(cudaGetDevice(&b->device), "cudaGetDevice");
    chk(cudaEventCreateWithFlags(&b->upload_done, cudaEventDisableTiming), "cudaEventCreate");
    chk(cudaMalloc(&b->status, sizeof(unsigned)), "cudaMalloc");
    chk(cudaMemset(b->status, 0, sizeof(unsigned)), "cudaMemset");
    return b.release();
}

void batch_destroy(Batch* b) { delete b; }

void batch_clear(Batch* b) { b->waves.clear(); }

// Adds every pass of a planned handle; all passes must be generic tile
// passes (the planner's generic-only hint gives such plans).
bool batch_add(Batch* b, const FftPlan& p, const void* in, void* out) {
    return batch_add_rows(b, p, in, out, p.batch, p.workspace);
}

bool batch_add_rows(Batch* b, const FftPlan& p, const void* in, void* out, long long rows, void* ws) {
    if (rows < 1 || rows > p.batch) return false;
    for (const Step& st : p.steps) {
        if (!queueable(st)) return false;
        if (rows != p.batch && st.batch_dim == 0) return false;
    }
    if ((int)b->waves.size() < (int)p.steps.size()) b->waves.resize(p.steps.size());
    for (size_t k = 0; k < p.steps.size(); ++k) {
        const Step& st = p.steps[k];
        auto loc = [&](Loc l, size_t off) -> char* {
            char* base = l == Loc::In ? const_cast<char*>(static_cast<const char*>(in))
                       : l == Loc::Out ? static_cast<char*>(out) : static_cast<char*>(ws);
            return base + off;
        };
        QueueItem it{};
        it.args = st.L.args;
        if (rows != p.batch) {
            TileArgs& a = it.args;
            if (st.batch_dim == 1) {
                a.inner = (int)rows;
                a.tiles_per_outer = (int)((rows + a.P - 1) / a.P);
                a.ntiles = a.tiles_per_outer;
                a.div_tpo = make_fastdiv((uint32_t)a.tiles_per_outer);
            } else {
                a.ntiles = (int)(a.tiles_per_outer * rows);
            }
        }
        it.args.src = loc(st.src, st.src_off);
        it.args.dst = loc(st.dst, st.dst_off);
        it.sign = st.L.sign;
        it.e = st.L.e;
        it.op = st.L.op;
        it.tw4 = st.L.tw4 ? 1 : 0;
        it.smem = st.L.smem_bytes;
        b->waves[k].push_back(it);
    }
    return true;
}

void batch_set_gate(Batch* b, const unsigned* gate, long long limit) {
    b->gate = gate;
    b->gate_limit = limit;
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

void batch_use_graphs(Batch* b, bool on) { b->use_graphs = on; }

unsigned batch_take_status(Batch* b) {
    unsigned s = 0, z = 0;
    chk(cudaMemcpy(&s, b->status, sizeof(unsigned), cudaMemcpyDeviceToHost), "cudaMemcpy");
    chk(cudaMemcpy(b->status, &z, sizeof(unsigned), cudaMemcpyHostToDevice), "cudaMemcpy");
    return s;
}

int batch_last_launches(const Batch* b) { return b->launches; }

void batch_exec(Batch* b, cudaStream_t stream) {
    const int nw = (int)b->waves.size();
    b->launches = 0;
    if (nw == 0) return;
    // layout: [nw headers][wave 0 items][wave 1 items]...; kernel arguments
    // depend only on nw, the item offsets travel in the headers
    const size_t items_off = sizeof(QueueWave) * nw;
    size_t bytes = items_off;
    std::vector<int> first(nw);
    int smem = 0;
    int nitems = 0;
    for (int w = 0; w < nw; ++w) {
        first[w] = nitems;
        nitems += (int)b->waves[w].size();
        for (const QueueItem& it : b->waves[w]) smem = std::max(smem, it.smem);
    }
    bytes += sizeof(QueueItem) * (size_t)std::max(nitems, 1);
    smem = (smem + 32767) / 32768 * 32768;  // bucket so graphs are reused
    smem = std::min(smem, kQueueMaxSmem);
    size_t copy = 4096;  // upload size, bucketed to a power of two for the same reason
    while (copy < bytes) copy *= 2;
    if (copy > b->cap) {
        chk(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        size_t cap = std::max<size_t>(copy * 2, 1 << 16);
        if (b->dev_buf) cudaFree(b->dev_buf);
        if (b->host_buf) cudaFreeHost(b->host_buf);
        b->dev_buf = nullptr;
        b->host_buf = nullptr;
        chk(cudaMalloc(&b->dev_buf, cap), "cudaMalloc");
        chk(cudaMallocHost(&b->host_buf, cap), "cudaMallocHost");
        b->cap = cap;
        for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
        b->graphs.clear();
    }
    if (b->counters < nw) {
        chk(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        if (b->counter) cudaFree(b->counter);
        chk(cudaMalloc(&b->counter, sizeof(unsigned) * nw), "cudaMalloc");
        b->counters = nw;
        for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
        b->graphs.clear();
    }
    // the previous upload must have consumed the staging buffer
    chk(cudaEventSynchronize(b->upload_done), "cudaEventSynchronize");
    char* h = static_cast<char*>(b->host_buf);
    for (int w = 0; w < nw; ++w) {
        QueueWave hd{};
        int tiles = 0;
        for (QueueItem& it : b->waves[w]) {
            it.tile_begin = tiles;
            tiles += it.args.ntiles;
        }
        hd.items = (int)b->waves[w].size();
        hd.tiles = tiles;
        hd.first = first[w];
        std::memcpy(h + sizeof(QueueWave) * w, &hd, sizeof(hd));
        if (!b->waves[w].empty())
            std::memcpy(h + items_off + sizeof(QueueItem) * (size_t)first[w], b->waves[w].data(),
                        sizeof(QueueItem) * b->waves[w].size());
    }
    int per_sm = 1, sms = 1;
    chk(queue_prepare(smem, &per_sm), "queue_prepare");
    chk(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "cudaDeviceGetAttribute");
    const int grid = sms * std::max(per_sm, 1);
    char* d = static_cast<char*>(b->dev_buf);
    auto issue = [&](cudaStream_t s) {
        chk(cudaMemcpyAsync(d, h, copy, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        for (int w = 0; w < nw; ++w)
            chk(queue_launch(reinterpret_cast<const QueueWave*>(d + sizeof(QueueWave) * w),
                             reinterpret_cast<const QueueItem*>(d + items_off), b->counter + w, b->gate,
                             b->gate_limit, b->status, grid, smem, s),
                "queue_launch");
    };
    if (b->use_graphs) {
        const auto key = std::make_tuple(nw, smem, grid, copy);
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ge = nullptr;
            chk(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            issue(stream);
            chk(cudaStreamEndCapture(stream, &g), "cudaStreamEndCapture");
            chk(cudaGraphInstantiate(&ge, g, 0), "cudaGraphInstantiate");
            cudaGraphDestroy(g);
            it = b->graphs.emplace(key, ge).first;
        }
        chk(cudaGraphLaunch(it->second, stream), "cudaGraphLaunch");
    } else {
        issue(stream);
    }
    chk(cudaEventRecord(b->upload_done, stream), "cudaEventRecord");
    b->launches = nw;
}

}  // namespace sipfft
