// Cluster four-step kernels (cluster_fft.cuh): instantiations, registry,
// launch with the cluster dimension.
#include "cluster.h"
#include "cluster_configs.h"

namespace sipfft {

namespace {

template <class K>
std::vector<int> radices_of() {
    std::vector<int> r;
    for (int p = 0; p < K::NP; ++p) r.push_back(K::radix(p));
    return r;
}

template <class CC>
ClEntry entry() {
    ClEntry e;
    e.n = CC::N;
    e.n1 = CC::N1;
    e.n2 = CC::N2;
    e.C = CC::C;
    e.T = CC::T;
    e.sign = CC::SIGN;
    e.pa = CC::PA;
    e.pb = CC::PB;
    e.ra = radices_of<typename CC::KA>();
    e.rb = radices_of<typename CC::KB>();
    e.smem = CC::SMEM_VALUES * 8;
    e.fn = reinterpret_cast<const void*>(&cluster_fft_kernel<CC>);
    return e;
}

const std::vector<ClEntry>& registry() {
    static const std::vector<ClEntry> reg = [] {
        std::vector<ClEntry> v;
#define SIP_CL_ENTRY(CC) v.push_back(entry<CC>());
        SIP_CL_CONFIGS(SIP_CL_ENTRY)
#undef SIP_CL_ENTRY
        return v;
    }();
    return reg;
}

}  // namespace

const ClEntry* cluster_find(int n, int sign) {
    for (const ClEntry& e : registry())
        if (e.n == n && e.sign == sign) return &e;
    return nullptr;
}

cudaError_t cluster_prepare(const ClEntry* e) {
    return cudaFuncSetAttribute(e->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem);
}

cudaError_t cluster_launch(const ClEntry* e, long long transforms, const TileArgs& a, const TileArgs& b,
                           cudaStream_t stream) {
    if (transforms <= 0 || transforms * e->C > 0x7fffffffLL) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(transforms * e->C), 1, 1);
    cfg.blockDim = dim3((unsigned)e->T, 1, 1);
    cfg.dynamicSmemBytes = (size_t)e->smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)e->C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TileArgs aa = a, bb = b;
    void* params[] = {&aa, &bb};
    return cudaLaunchKernelExC(&cfg, e->fn, params);
}

}  // namespace sipfft
