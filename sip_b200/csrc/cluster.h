// Registry and launch of the cluster four-step kernels (cluster_fft.cuh).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "tile_io.cuh"

namespace sipfft {

struct ClEntry {
    int n, n1, n2;  // transform length N = n1 x n2
    int C;          // CTAs per cluster (one transform per cluster)
    int T;          // threads per CTA
    int sign;
    int pa, pb;     // columns of pass A, rows of pass B per CTA
    std::vector<int> ra, rb;  // radices of the n1- and n2-point passes
    int smem;       // dynamic shared memory per CTA (bytes)
    const void* fn; // kernel (library) or CPU runner (test harness)
};

// The cluster kernel for a C2C length and direction; nullptr when none is
// compiled.
const ClEntry* cluster_find(int n, int sign);

// Raises the kernel's shared-memory limit.
cudaError_t cluster_prepare(const ClEntry* e);

// One launch over `transforms` transforms (a: pass A arguments, b: pass B).
cudaError_t cluster_launch(const ClEntry* e, long long transforms, const TileArgs& a, const TileArgs& b,
                           cudaStream_t stream);

}  // namespace sipfft
