// Batch work queue: one persistent launch processes the tiles of many
// transforms of different lengths, batch counts and directions.
//
// The host uploads one header {items, tiles, first item} per wave followed
// by every wave's QueueItem descriptors (tile arguments + variant + first
// tile).
// Every CTA repeatedly claims the next tile index with an atomic counter,
// finds its item by binary search over the items' first tiles and runs the
// generic tile body (tile_kernel_impl.cuh) of that item's variant.  Items
// of multi-pass plans are split into waves (pass k of every plan in wave
// k), one launch per wave.  An optional gate makes the CTAs wait for a
// device flag before they start; the wait is bounded and, when it runs
// out, the kernel sets bit 1 of the status word and returns, leaving the
// context usable.
#include <cuda_runtime.h>

#include "queue.h"
#include "tile_kernel_impl.cuh"

namespace sipfft {

namespace {

template <int SIGN, int E, int OP, bool TW4>
__device__ __noinline__ void q_tile(const TileArgs* a, int tile) {
    tile_body<SIGN, E, OP, TW4>(*a, tile, threadIdx.x, blockDim.x);
}

__device__ void q_dispatch(const QueueItem* it, int tile) {
    const TileArgs* a = &it->args;
    const int e32 = it->e == 32;
    switch (it->op) {
        case OP_C2C:
            if (it->sign < 0) {
                if (it->tw4) {
                    if (e32) q_tile<-1, 32, OP_C2C, true>(a, tile); else q_tile<-1, 16, OP_C2C, true>(a, tile);
                } else {
                    if (e32) q_tile<-1, 32, OP_C2C, false>(a, tile); else q_tile<-1, 16, OP_C2C, false>(a, tile);
                }
            } else {
                if (it->tw4) {
                    if (e32) q_tile<1, 32, OP_C2C, true>(a, tile); else q_tile<1, 16, OP_C2C, true>(a, tile);
                } else {
                    if (e32) q_tile<1, 32, OP_C2C, false>(a, tile); else q_tile<1, 16, OP_C2C, false>(a, tile);
                }
            }
            break;
        case OP_R2C_HALF:
            if (e32) q_tile<-1, 32, OP_R2C_HALF, false>(a, tile); else q_tile<-1, 16, OP_R2C_HALF, false>(a, tile);
            break;
        case OP_C2R_HALF:
            if (e32) q_tile<1, 32, OP_C2R_HALF, false>(a, tile); else q_tile<1, 16, OP_C2R_HALF, false>(a, tile);
            break;
        case OP_R2C_PAIR:
            if (e32) q_tile<-1, 32, OP_R2C_PAIR, false>(a, tile); else q_tile<-1, 16, OP_R2C_PAIR, false>(a, tile);
            break;
        case OP_C2R_PAIR:
            if (e32) q_tile<1, 32, OP_C2R_PAIR, false>(a, tile); else q_tile<1, 16, OP_C2R_PAIR, false>(a, tile);
            break;
        case OP_PC:
            if (it->tw4) {
                if (e32) q_tile<1, 32, OP_PC, true>(a, tile); else q_tile<1, 16, OP_PC, true>(a, tile);
            } else {
                if (e32) q_tile<1, 32, OP_PC, false>(a, tile); else q_tile<1, 16, OP_PC, false>(a, tile);
            }
            break;
        default:
            break;
    }
}

__global__ void __launch_bounds__(kMaxTileThreads, 1)
    queue_kernel(const QueueWave* wave, const QueueItem* items_base, unsigned* counter, const volatile unsigned* gate,
                 long long gate_limit, unsigned* status) {
    __shared__ int s_tile;
    __shared__ int s_stop;
    if (gate != nullptr) {
        if (threadIdx.x == 0) {
            long long i = 0;
            while (*gate == 0u && i < gate_limit) ++i;
            s_stop = *gate == 0u;
            if (s_stop) atomicOr(status, kQueueGateTimeout);
        }
        __syncthreads();
        if (s_stop) return;
    }
    const int nitems = wave->items;
    const int total = wave->tiles;
    const QueueItem* items = items_base + wave->first;
    // The descriptor of the item being worked on is kept in shared memory
    // (the tile body reads its arguments many times), re-copied only when a
    // claimed tile belongs to another item; the next tile is claimed while
    // the current one is transformed.
    __shared__ QueueItem s_item;
    __shared__ int s_next, s_item_idx, s_copy;
    if (threadIdx.x == 0) {
        s_tile = (int)atomicAdd(counter, 1u);
        s_item_idx = -1;
    }
    constexpr int kWords = (int)(sizeof(QueueItem) / sizeof(int));
    static_assert(sizeof(QueueItem) % sizeof(int) == 0, "QueueItem copies as words");
    for (;;) {
        __syncthreads();
        const int t = s_tile;
        if (t >= total) break;
        if (threadIdx.x == 0) {
            int cur = s_item_idx;
            const bool inside = cur >= 0 && t >= s_item.tile_begin && t < s_item.tile_begin + s_item.args.ntiles;
            if (!inside) {
                int lo = 0, hi = nitems - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (items[mid].tile_begin <= t) lo = mid;
                    else hi = mid - 1;
                }
                cur = lo;
            }
            s_copy = inside ? -1 : cur;
            s_item_idx = cur;
            s_next = (int)atomicAdd(counter, 1u);
        }
        __syncthreads();
        const int copy = s_copy;
        if (copy >= 0) {
            const int* src = reinterpret_cast<const int*>(items + copy);
            int* dst = reinterpret_cast<int*>(&s_item);
            for (int w = threadIdx.x; w < kWords; w += blockDim.x) dst[w] = src[w];
            __syncthreads();
        }
        q_dispatch(&s_item, t - s_item.tile_begin);  // ends with a barrier
        if (threadIdx.x == 0) s_tile = s_next;
    }
}

}  // namespace

cudaError_t queue_prepare(int smem_bytes, int* ctas_per_sm) {
    const void* fn = reinterpret_cast<const void*>(&queue_kernel);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kQueueMaxSmem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, kMaxTileThreads, (size_t)smem_bytes);
}

cudaError_t queue_launch(const QueueWave* wave, const QueueItem* items_base, unsigned* counter, const unsigned* gate,
                         long long gate_limit, unsigned* status, int grid, int smem_bytes, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    queue_kernel<<<grid, kMaxTileThreads, smem_bytes, stream>>>(wave, items_base, counter, gate, gate_limit, status);
    return cudaGetLastError();
}

}  // namespace sipfft
