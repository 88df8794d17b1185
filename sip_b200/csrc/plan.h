// Plan model of the B200 FFT library: a plan is an ordered list of tile
// kernel launches ("steps") whose operands are the exec's input, output or
// a region of the caller's workspace.  It replaces the reference's
// FFTPlan{steps[]} of FftOperation cores (core/fft/fftplan/include/fftplan/
// fft_plan.h:43-71) with direct CUDA launches.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "fft_api.h"
#include "bluestein.h"
#include "cluster.h"
#include "real_kernels.h"
#include "sk_registry.h"
#include "tile_launch.h"

namespace sipfft {

// Error carrying the status code the C ABI returns.
struct PlanError : std::runtime_error {
    int code;
    PlanError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Device allocation owned by plans through shared_ptr (tables are shared
// between plans through TableCache).
struct DeviceBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    int device = -1;
    ~DeviceBuf();
};
using BufPtr = std::shared_ptr<DeviceBuf>;

// Operand of a step.
enum class Loc : int { In = 0, Out = 1, Ws = 2 };

enum class StepKind : int {
    Tile = 0,
    RealPost = 1,
    RealPre = 2,
    Tc = 3,
    Blue = 4,
    // element-wise passes of odd real lengths above one tile (real_kernels.h)
    PairPack = 5,
    PairSeparate = 6,
    PairCombine = 7,
    PairSplit = 8,
    // one C2C transform per thread-block cluster (cluster.h)
    Cluster = 9,
};

inline bool is_pair_kind(StepKind k) { return k >= StepKind::PairPack && k <= StepKind::PairSplit; }

struct Step {
    StepKind kind = StepKind::Tile;
    TileLaunch L;
    RealPassArgs real{};  // RealPost / RealPre
    PairPassArgs pair{};  // PairPack / PairSeparate / PairCombine / PairSplit
    // Cluster: L.args drives pass A (n1-point columns), cl_b pass B (n2-point
    // rows, the cross twiddle table in its tw2); cl_plan_b / cl_radices_b
    // describe pass B's radix passes; cl_transforms transforms per exec.
    const ClEntry* cl = nullptr;
    TileArgs cl_b{};
    PlanDev cl_plan_b{};
    std::vector<int> cl_radices_b;
    long long cl_transforms = 0;
    BufPtr tw_b;
    Loc src = Loc::In, dst = Loc::Out;
    size_t src_off = 0, dst_off = 0;  // byte offsets into the operand
    // Which tile index the plan's batch runs along (for executing fewer rows
    // than planned through the batch queue): 0 neither, 1 inner, 2 outer.
    int batch_dim = 0;
    // Bluestein: pre / post pass arguments (kind Blue), and on the pulse
    // steps of the convolution mul_table = 1 (filter FFT_m(b) of length blue_m
    // for transform length blue_n and sign blue_sign, made at device preparation).
    BluesteinArgs blue{};
    bool blue_post = false;
    int mul_table = 0;
    long long blue_n = 0, blue_m = 0;
    int blue_sign = 0;
    BufPtr mul_buf, chirp_buf;
    PlanDev host_plan{};              // pass list (uploaded to plan_dev)
    std::vector<int> radices;
    int tw2_kind = 0;                 // 0 none, 1 roots W_n^k for k < count, 2 split cross twiddles,
                                      // 3 the Bluestein chirp of (blue_n, blue_sign)
    long long tw2_n = 0, tw2_count = 0;
    const SkEntry* sk = nullptr;      // size-specialized kernel, when compiled for this step
    bool tc_cols_in = false, tc_cols_out = false;  // tensor-core step operand layouts
    const void* tc_fn = nullptr;
    BufPtr tc_bmat;
    BufPtr plan_dev, tw, tw2;
    std::string what;                 // human-readable description
    // L2-resident chunks (launch_steps): the steps of one chunk group run
    // back to back on a slice of `units` chunk units at a time, so that what
    // one step writes for the next is still in L2.  chunk_dim is the tile
    // index that carries the units (1 inner, 2 outer; RealPre/RealPost steps
    // use their rows), chunk_per its count per unit, chunk_src / chunk_dst the
    // bytes one unit spans in the source / destination operand.  Input and
    // output operands move by one slice per unit; a workspace operand does
    // not: every chunk of a lane reuses the same region (lane l at l chunks'
    // worth of slices), which stays in L2.
    int chunk_group = -1;
    int chunk_dim = 0;
    long long chunk_per = 1;
    long long chunk_src = 0, chunk_dst = 0;
    int max_grid = 0;  // resident CTAs of a persistent (sk) kernel; 0: one CTA per tile
};

// The second stream and the fork / join events of a plan's chunk lanes.
struct ChunkLanes {
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    ~ChunkLanes();
};

// Steps [first, last) of a plan that run chunk by chunk; `units` chunk units
// in all, `unit_bytes` the largest operand slice of one unit.  Consecutive
// chunks alternate between the plan's stream and a second stream (two
// lanes), so that one chunk's passes overlap the next one's.
struct ChunkGroup {
    size_t first = 0, last = 0;
    long long units = 0;
    long long unit_bytes = 0;
};

struct FftPlan {
    AsdSip::asdFftType type = AsdSip::ASCEND_FFT_C2C;
    AsdSip::asdFftDirection direction = AsdSip::ASCEND_FFT_FORWARD;
    std::vector<int64_t> sizes;  // transform dims, outermost first
    int64_t batch = 1;
    bool vertical = false;
    int compute_mode = 0;  // 0: FP32 Stockham, 1: tensor-core BF16x3 split for length-256 passes
    // Planner hints (sipFftSetPlanHint / the tune cache); 0 = planner default.
    int hint_p = 0;        // transforms per tile
    int hint_e = 0;        // elements per thread (16 or 32)
    int hint_generic = 0;  // 1: generic tile kernels only (no size-specialized / tensor-core)
    int hint_order = 0;    // radix order: 0 descending, 1 ascending
    int hint_real_fused = 0;  // real lengths above one tile: 0 default, 1 fuse both, 2 fuse neither
    int hint_sk_variant = -1;  // compiled size-specialized variant (sk_configs.h order); -1 automatic
    int hint_jit = 0;  // run-time compiled sk kernels: 0 default (large steps), 1 always, 2 never
    bool hints_explicit = false;
    // Pulse-compression plan (sipFftMakePlanPulse1D): x -> IFFT(FFT(x) * F)
    // per row, F a device spectrum of length sizes[0] owned by the caller.
    // Output rotation (sipFftSetOutputShift): 0 none, 1 fftshift, 2 ifftshift
    // of every (1 x N) or (X x Y) output slice, times out_scale.
    int out_shift = 0;
    double out_scale = 1.0;
    bool pulse = false;
    const void* pulse_filter = nullptr;
    int pulse_flags = 0;  // SIP_FFT_PULSE_CONJ_FILTER | SIP_FFT_PULSE_SCALE
    bool initialized = false;
    bool resources_ready = false;
    int device = -1;
    void* stream = nullptr;
    void* workspace = nullptr;
    size_t workspace_recorded = 0;  // value recorded by GetWorkspaceSize
    size_t workspace_need = 0;
    // Device address of the static scratch array of sipFftExecC2CNoAlloc
    // (noalloc.cu), resolved while the plan is prepared on its device for
    // FP32 C2C plans whose workspace fits the array; null otherwise.
    void* noalloc_scratch = nullptr;
    std::vector<Step> steps;
    std::vector<ChunkGroup> chunk_groups;
    // Second stream and fork / join events of the two chunk lanes (made at
    // device preparation when the plan has chunk groups).
    std::shared_ptr<ChunkLanes> lanes;

    bool forward() const { return direction == AsdSip::ASCEND_FFT_FORWARD; }
    int64_t elements() const;  // batch * prod(sizes)
};

// Radix sequence for a length that fits one tile; empty if the length has
// a prime factor without a compiled butterfly.
std::vector<int> choose_radices(int n, int e);

// Largest complex length one tile kernel transforms (shared memory bound).
constexpr int kMaxTileN = 16384;
// Tiles of one wave on B200 at two CTAs per SM (148 SMs).
constexpr long long kOneWaveTiles = 2 * 148;

constexpr int kComputeFp32 = 0;
constexpr int kPulseConj = 1;   // multiply by conj(F)
constexpr int kPulseScale = 2;  // scale the output by 1/n
constexpr int kComputeTcSplit = 1;

// Builds the steps of a validated plan (host side only).
void build_steps(FftPlan& plan);

// Allocates the plan's device tables on the current device.
void prepare_device(FftPlan& plan);

// Applies the tune-cache entry for the plan (file named by SIP_FFT_TUNE_CACHE,
// lines "type direction n0[xn1[xn2]] batch P E generic order [real_fused
// [sk_variant]]");
// returns true
// when an entry matched.
bool apply_tune_cache(FftPlan& plan);

// Batched queue execution (batch.cpp).
struct Batch;
Batch* batch_create();
void batch_destroy(Batch* b);
void batch_clear(Batch* b);
bool batch_add(Batch* b, const FftPlan& p, const void* in, void* out);
// As batch_add for the first `rows` rows of the plan's batch (rows <= the
// plan's batch; every step must declare its batch dimension), with the
// workspace at `ws` (rows * the plan's per-row workspace; null when none).
bool batch_add_rows(Batch* b, const FftPlan& p, const void* in, void* out, long long rows, void* ws);
void batch_exec(Batch* b, cudaStream_t stream);
void batch_set_gate(Batch* b, const unsigned* gate, long long limit);
void batch_use_graphs(Batch* b, bool on);
unsigned batch_take_status(Batch* b);
int batch_last_launches(const Batch* b);

// Runs a separated-plane C2C plan (one tile step) with real / imaginary
// float planes.
void launch_separated(const FftPlan& plan, const float* in_re, const float* in_im, float* out_re, float* out_im);

// Launches every step on the plan's stream (chunk groups chunk by chunk).
void launch_steps(const FftPlan& plan, const void* in, void* out, void* ws);

// True when every step of the plan can run on the first rows of its batch
// alone (1-D and pulse plans of tile and real pre/post steps).
bool rows_exec_supported(const FftPlan& plan);
// Every step of the plan over the first `rows` transforms of its batch,
// 1 <= rows <= plan.batch, with workspace `ws`.
void launch_rows(const FftPlan& plan, long long rows, const void* in, void* out, void* ws);

// Chunk units per chunk of a group for the current L2 chunk size
// (SIP_FFT_L2_CHUNK_MB, default kL2ChunkBytes; 0 turns chunking off); the
// group's `units` when it runs as one launch per step.
long long chunk_units(const ChunkGroup& g);
constexpr long long kL2ChunkBytes = 32LL << 20;
// Units smaller than this run unchunked (plan.cpp chunk_min_unit_bytes).
constexpr long long kL2ChunkMinUnit = 16LL << 20;
// Overrides the chunk size for plans made and execs run afterwards (0 turns
// chunking off; a negative value restores the default).
void set_l2_chunk_bytes(long long bytes);
// Chunk lanes (1 or 2; SIP_FFT_L2_CHUNK_LANES, default 2).
int chunk_lanes();
// Byte offset of a step operand for chunk units [u0, ...) on lane `lane`
// with `cu` units per chunk.
long long chunk_offset(const Step& st, bool src, long long u0, int lane, long long cu);

// Kernel launches one exec of the plan makes (chunking included).
long long exec_launches(const FftPlan& plan);

// The launch of a tile step restricted to `cnt` chunk units of its group
// (tile counts and the persistent grid recomputed).
TileLaunch chunk_tile_launch(const Step& st, long long cnt);

// JSON description of the steps (tests, ASDSIP_FFT_PLAN_TRACE).
std::string describe(const FftPlan& plan);

}  // namespace sipfft
