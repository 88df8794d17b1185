// Batch work queue (queue.cu) descriptors and launch entry points.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <tuple>
#include <vector>

#include "tile_io.cuh"
#include "tile_launch.h"

namespace sipfft {

// One transform pass of a batch: the tile arguments of the plan step with
// its operands bound, the kernel variant, the first tile index of the item
// within its wave and the dynamic shared memory its tiles need.
struct QueueItem {
    TileArgs args;
    int sign, e, op, tw4;
    int tile_begin;
    int smem;
    int pad_[2];
};

// Per-wave header: its items are items_base[first .. first + items).  The
// offsets travel in the uploaded header rather than in kernel arguments, so
// a captured launch sequence stays valid when the item counts change.
struct QueueWave {
    int items;
    int tiles;
    int first;
    int pad_;
};

// Host state of a batch (batch.cpp).
struct Batch {
    int device = -1;
    std::vector<std::vector<QueueItem>> waves;
    void* dev_buf = nullptr;
    void* host_buf = nullptr;
    size_t cap = 0;
    unsigned* counter = nullptr;  // one per wave
    unsigned* status = nullptr;
    int counters = 0;
    const unsigned* gate = nullptr;
    long long gate_limit = 0;
    bool use_graphs = true;
    cudaEvent_t upload_done = nullptr;
    std::map<std::tuple<int, int, int, size_t>, cudaGraphExec_t> graphs;
    int launches = 0;  // queue launches issued by the last exec

    ~Batch() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        if (upload_done) cudaEventDestroy(upload_done);
        if (dev_buf) cudaFree(dev_buf);
        if (host_buf) cudaFreeHost(host_buf);
        if (counter) cudaFree(counter);
        if (status) cudaFree(status);
    }
};


// Dynamic shared memory a queue launch may use (the kernel also holds a few
// bytes of static shared memory).
constexpr int kQueueMaxSmem = kMaxTileSmem - 1024;

// Status word bits.
constexpr unsigned kQueueGateTimeout = 2u;

cudaError_t queue_prepare(int smem_bytes, int* ctas_per_sm);

// Resets the tile counter and launches one wave (header `wave`, items at
// `items_base` + wave->first, both in device memory).  `gate` may be null;
// otherwise CTAs wait (at most gate_limit polls) for *gate != 0.
cudaError_t queue_launch(const QueueWave* wave, const QueueItem* items_base, unsigned* counter, const unsigned* gate,
                         long long gate_limit, unsigned* status, int grid, int smem_bytes, cudaStream_t stream);

}  // namespace sipfft
