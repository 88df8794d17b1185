// Run-time specialization of the sk tile kernels (jit.h).
#include "jit.h"

#include <dlfcn.h>
#include <pthread.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <functional>
#include <map>
#include <mutex>
#include <new>
#include <sstream>
#include <thread>
#include <condition_variable>
#include <chrono>
#include <set>

#include "plan.h"
#include "sk_kernel.cuh"

namespace sipfft {

// Kernel headers embedded by the build (generated jit_headers.cpp).
extern const int kJitHeaderCount;
extern const char* const kJitHeaderNames[];
extern const char* const kJitHeaderTexts[];

namespace {

// ------------------------------------------------------------ NVRTC (dlopen)
struct Nvrtc {
    bool ok = false;
    int major = 0, minor = 0;
    nvrtcResult (*version)(int*, int*) = nullptr;
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*,
                          const char* const*) = nullptr;
    nvrtcResult (*destroy)(nvrtcProgram*) = nullptr;
    nvrtcResult (*add_name)(nvrtcProgram, const char*) = nullptr;
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*) = nullptr;
    nvrtcResult (*log_size)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*log)(nvrtcProgram, char*) = nullptr;
    nvrtcResult (*lowered)(nvrtcProgram, const char*, const char**) = nullptr;
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*cubin)(nvrtcProgram, char*) = nullptr;
};

const Nvrtc& nvrtc() {
    static const Nvrtc api = [] {
        Nvrtc a;
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void* h = nullptr;
        for (const char* n : names)
            if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL)) != nullptr) break;
        if (h == nullptr) return a;
        auto sym = [&](auto& fp, const char* name) {
            fp = reinterpret_cast<std::remove_reference_t<decltype(fp)>>(dlsym(h, name));
            return fp != nullptr;
        };
        a.ok = sym(a.version, "nvrtcVersion") && sym(a.create, "nvrtcCreateProgram") &&
               sym(a.destroy, "nvrtcDestroyProgram") && sym(a.add_name, "nvrtcAddNameExpression") &&
               sym(a.compile, "nvrtcCompileProgram") && sym(a.log_size, "nvrtcGetProgramLogSize") &&
               sym(a.log, "nvrtcGetProgramLog") && sym(a.lowered, "nvrtcGetLoweredName") &&
               sym(a.cubin_size, "nvrtcGetCUBINSize") && sym(a.cubin, "nvrtcGetCUBIN");
        if (a.ok && a.version(&a.major, &a.minor) != NVRTC_SUCCESS) a.ok = false;
        return a;
    }();
    return api;
}

// -default-device: the headers' unannotated constexpr helpers (evaluated at
// compile time) are device functions here, as --expt-relaxed-constexpr
// makes them usable for the library's nvcc build.
const char* const kOptions[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-default-device"};

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return v != nullptr && *v ? std::atoi(v) : dflt;
}

// ------------------------------------------------------------ configuration
// Cost of one pass of radix r in the run-time radix choice: passes
// dominate (each is a shared-memory round trip), then larger radices and
// the odd butterflies of the primes from 11 up.
double jit_radix_cost(int r) {
    int big = 1;
    for (int p = 2, m = r; p <= m; ++p)
        while (m % p == 0) {
            big = p;
            m /= p;
        }
    double c = 1.0 + 0.002 * r;
    if (big >= 11) c += 0.2;
    if (big >= 23) c += 0.3;
    return c;
}

// Fewest, cheapest passes of radices 2..32 (any radix: the sk passes
// build composite butterflies at compile time), largest first.
std::vector<int> jit_radices(int n) {
    std::map<int, std::pair<double, std::vector<int>>> memo;
    std::function<std::pair<double, std::vector<int>>(int)> best = [&](int m) -> std::pair<double, std::vector<int>> {
        if (m == 1) return {0.0, {}};
        auto it = memo.find(m);
        if (it != memo.end()) return it->second;
        std::pair<double, std::vector<int>> res{1e30, {}};
        for (int r = 32; r >= 2; --r) {
            if (m % r != 0) continue;
            auto sub = best(m / r);
            if (sub.first >= 1e29) continue;
            const double c = sub.first + jit_radix_cost(r);
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
    if (r.first >= 1e29 || r.second.size() > (size_t)kMaxPasses) return {};
    std::sort(r.second.begin(), r.second.end(), std::greater<int>());
    return r.second;
}

// Threads so that no pass holds more than `e` values per thread (one
// butterfly per thread for radices above e).
int jit_threads(int P, int n, const std::vector<int>& radices, int e) {
    long long t = 32;
    for (int r : radices) {
        const long long b = (long long)P * (n / r);
        const long long per = std::max(1, e / r);
        t = std::max(t, (b + per - 1) / per);
    }
    return (int)((t + 31) / 32 * 32);
}

// ------------------------------------------------------------ registry
// Registry state lives on the heap and is never destroyed: background
// compilations may still run while the process exits.
std::mutex& g_jit_mu = *new std::mutex;
std::deque<SkEntry>& g_jit_entries = *new std::deque<SkEntry>;  // stable addresses
std::map<std::string, SkEntry*>& g_jit_index = *new std::map<std::string, SkEntry*>;
std::map<std::string, const void*>& g_jit_kernels = *new std::map<std::string, const void*>;  // name -> kernel
struct JitBinary {
    std::vector<char> cubin;
    std::string lowered;
    int spill = 0;
};
std::map<std::string, JitBinary>& g_jit_cubins = *new std::map<std::string, JitBinary>;  // key -> compiled here

JitCfg cfg_of(const SkEntry& e) {
    JitCfg c;
    c.op = e.op;
    c.mode = e.mode;
    c.sign = e.sign;
    c.tw4 = e.tw4;
    c.n = e.n;
    c.P = e.P;
    c.T = e.T;
    c.stages = e.stages;
    c.minb = e.minb;
    c.radices = e.radices;
    c.LD = e.LD;
    c.smem = e.smem;
    c.twb = e.flags;
    return c;
}

uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

std::string cache_dir() {
    const char* env = std::getenv("SIP_FFT_JIT_CACHE");
    std::string d;
    if (env != nullptr) {
        d = env;
    } else {
        const char* home = std::getenv("HOME");
        if (home == nullptr || *home == 0) return "";
        d = std::string(home) + "/.cache/sip_fft_jit";
    }
    // mkdir -p
    for (size_t i = 1; i <= d.size(); ++i)
        if (i == d.size() || d[i] == '/') mkdir(d.substr(0, i).c_str(), 0755);
    struct stat st {};
    if (stat(d.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) return "";
    return d;
}

// Cache file: "SIPJIT2\n<lowered name>\n<spill bytes>\n<cubin bytes>".
bool cache_read(const std::string& path, std::vector<char>* cubin, std::string* lowered, int* spill) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::string magic, sp;
    if (!std::getline(f, magic) || magic != "SIPJIT2") return false;
    if (!std::getline(f, *lowered) || lowered->empty()) return false;
    if (!std::getline(f, sp) || sp.empty()) return false;
    *spill = std::atoi(sp.c_str());
    cubin->assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return !cubin->empty();
}

void cache_write(const std::string& path, const std::vector<char>& cubin, const std::string& lowered, int spill) {
    const std::string tmp = path + ".tmp." + std::to_string((long long)getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        f << "SIPJIT2\n" << lowered << "\n" << spill << "\n";
        f.write(cubin.data(), (std::streamsize)cubin.size());
        if (!f) {
            std::remove(tmp.c_str());
            return;
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

}  // namespace

// Set in a child process forked from one that had started the compiler's
// worker threads: the compiler's state may have been copied in the middle
// of a compilation by another thread, so the child does not compile (its
// plans run the generic or compiled kernels).
static bool g_forked_child = false;

bool sk_jit_available() {
    if (g_forked_child) return false;
    const char* env = std::getenv("SIP_FFT_JIT");
    if (env != nullptr && std::strcmp(env, "0") == 0) return false;
    return nvrtc().ok;
}

bool sk_jit_choose(int op, int mode, int sign, bool tw4, int n, long long transforms, JitCfg* out, int values,
                   const std::vector<int>* order) {
    const bool real_op = op == OP_R2C_HALF || op == OP_C2R_HALF || op == OP_R2C_PAIR || op == OP_C2R_PAIR;
    if (op != OP_C2C && op != OP_PC && !real_op) return false;
    if (real_op && (mode != SK_ROWS || tw4)) return false;
    if (op == OP_PC && mode != SK_ROWS) return false;
    if ((op == OP_R2C_PAIR || op == OP_C2R_PAIR) && n % 2 == 0) return false;
    if (n < 8 || n > kMaxTileN) return false;
    JitCfg c;
    c.op = op;
    c.mode = mode;
    c.sign = sign;
    c.tw4 = tw4;
    c.n = n;
    c.radices = order != nullptr ? *order : jit_radices(n);
    // Tuning overrides (sweeps; unset in normal use): SIP_FFT_JIT_RADICES
    // ("25,15,8", must multiply to n), SIP_FFT_JIT_P, SIP_FFT_JIT_T,
    // SIP_FFT_JIT_MINB, SIP_FFT_JIT_STAGES, SIP_FFT_JIT_TWB (the SK_TW_* bits
    // of sk_kernel.cuh: basis table, twiddles in shared memory, mirrored pairs).
    // With SIP_FFT_JIT_PREFER=<length> they apply to steps of that length only.
    const int only_n = env_int("SIP_FFT_JIT_PREFER", 0);
    const bool ovr = only_n <= 1 || only_n == n;
    auto ovr_int = [&](const char* name, int dflt) { return ovr ? env_int(name, dflt) : dflt; };
    if (const char* rs = ovr ? std::getenv("SIP_FFT_JIT_RADICES") : nullptr) {
        std::vector<int> r;
        long long prod = 1;
        for (const char* q = rs; *q;) {
            const int v = std::atoi(q);
            if (v < 2 || v > 32) return false;
            r.push_back(v);
            prod *= v;
            while (*q && *q != ',') ++q;
            if (*q == ',') ++q;
        }
        if (prod != n || r.empty() || r.size() > (size_t)kMaxPasses) return false;
        c.radices = r;
    }
    if (c.radices.empty()) return false;
    transforms = std::max<long long>(1, transforms);
    // transforms per tile: about SIP_FFT_JIT_TILE (4096) values for rows,
    // runs of 16 adjacent transforms (128-byte segments) for the column
    // modes; at most SIP_FFT_JIT_E (32) values per thread and pass
    const int tile_values = std::max(64, env_int("SIP_FFT_JIT_TILE", 4096));
    const int per_thread = std::max(8, values > 0 ? values : env_int("SIP_FFT_JIT_E", 32));
    long long P = mode == SK_ROWS ? std::max(1, tile_values / n) : 16;
    P = std::min<long long>(P, transforms);
    int T = 0;
    for (;;) {
        T = jit_threads((int)P, n, c.radices, per_thread);
        if (T > kMaxTileThreads && P == 1) T = jit_threads(1, n, c.radices, 2 * per_thread);
        if (T <= kMaxTileThreads || P == 1) break;
        P = std::max<long long>(1, P / 2);
    }
    if (T > kMaxTileThreads) return false;
    if (ovr_int("SIP_FFT_JIT_P", 0) > 0) P = std::min<long long>(ovr_int("SIP_FFT_JIT_P", 0), transforms);
    if (ovr_int("SIP_FFT_JIT_T", 0) > 0) T = ovr_int("SIP_FFT_JIT_T", 0);
    if (T % 32 != 0 || T > kMaxTileThreads) return false;
    c.P = (int)P;
    c.T = T;
    const int r0 = c.radices[0];
    c.LD = sk_pitch(n, r0);
    // twiddle options (SK_TW_* bits; SIP_FFT_JIT_TWB overrides them).  By
    // default the basis table staged in shared memory and a split pass 0
    // (dropped below where they do not apply): 3-23 % faster on B200 than
    // the basis table through L1 over run-time compiled C2C rows of 544 to
    // 8160 points.  Mirrored butterfly pairs (on request) apply to real
    // half-length tiles of two or more passes.
    c.twb = ovr_int("SIP_FFT_JIT_TWB", SK_TW_BASIS | SK_TW_SMEM | SK_SPLIT_PASS0);
    if (c.twb < 0 || c.twb > 15) return false;
    if ((c.twb & SK_MIRROR_PAIR) && (!real_op || c.radices.size() < 2)) c.twb &= ~SK_MIRROR_PAIR;
    if ((c.twb & SK_SPLIT_PASS0) && (c.radices.size() < 2 || op == OP_PC)) c.twb &= ~SK_SPLIT_PASS0;
    const long long buf = (long long)sk_buffer_values(op, c.P, n, r0) * 8;
    long long tws = (long long)sk_tws_values(op, n, c.radices.data(), (int)c.radices.size(), c.twb) * 8;
    if (buf + tws > kMaxTileSmem && (c.twb & SK_TW_SMEM)) {  // no room for the staged twiddles
        c.twb &= ~SK_TW_SMEM;
        tws = 0;
    }
    if (2 * buf + tws <= kMaxTileSmem) c.stages = 2;
    else if (buf + tws <= kMaxTileSmem) c.stages = 1;
    else return false;
    if (ovr_int("SIP_FFT_JIT_STAGES", 0) == 1) c.stages = 1;
    if (c.stages != 2) c.twb &= ~SK_SPLIT_PASS0;  // a split pass 0 uses the second buffer as its work layout
    c.smem = (int)(c.stages * buf + tws);
    const int smem_ctas = std::max<int>(1, (228 * 1024) / (c.smem + 1024));
    c.minb = std::max(1, std::min(65536 / (T * 128), smem_ctas));
    if (ovr_int("SIP_FFT_JIT_MINB", 0) > 0) c.minb = ovr_int("SIP_FFT_JIT_MINB", 0);
    *out = c;
    return true;
}

std::string sk_jit_source() { return "#include \"sk_kernel.cuh\"\n"; }

std::string sk_jit_name_expr(const JitCfg& c) {
    std::ostringstream s;
    s << "&sipfft::sk_fft_kernel<sipfft::SkCfg<" << c.n << ", " << c.P << ", " << c.T << ", " << c.op << ", "
      << c.mode << ", " << c.sign << ", " << (c.tw4 ? "true" : "false") << ", " << c.minb << ", " << c.twb;
    for (int r : c.radices) s << ", " << r;
    s << ">, " << c.stages << ">";
    return s.str();
}

// Spill stores the compiler's resource report (--ptxas-options=-v) states.
int spill_bytes(const std::string& log) {
    int total = 0;
    const std::string key = " bytes spill stores";
    for (size_t pos = log.find(key); pos != std::string::npos; pos = log.find(key, pos + 1)) {
        size_t b = pos;
        while (b > 0 && std::isdigit((unsigned char)log[b - 1])) --b;
        if (b < pos) total += std::atoi(log.substr(b, pos - b).c_str());
    }
    return total;
}

namespace {

// Options, cache key (hash) and cache file of a configuration.
struct JitKey {
    std::vector<const char*> opts;
    std::string hex, path;
};

JitKey jit_key(const JitCfg& c) {
    const Nvrtc& api = nvrtc();
    JitKey k;
    const std::string src = sk_jit_source();
    const std::string expr = sk_jit_name_expr(c);
    // SIP_FFT_JIT_PC_SPLIT=1: pulse tiles with out-of-line halves (sk_kernel.cuh)
    k.opts.assign(std::begin(kOptions), std::end(kOptions));
    k.opts.push_back("--ptxas-options=-v");
    if (env_int("SIP_FFT_JIT_PC_SPLIT", 0) != 0) k.opts.push_back("-DSIP_SK_PC_SPLIT=1");
    uint64_t h = 1469598103934665603ull;
    const int ver[2] = {api.major, api.minor};
    h = fnv1a(h, ver, sizeof(ver));
    for (const char* o : k.opts) h = fnv1a(h, o, std::strlen(o) + 1);
    h = fnv1a(h, src.data(), src.size());
    h = fnv1a(h, expr.data(), expr.size());
    for (int i = 0; i < kJitHeaderCount; ++i) {
        h = fnv1a(h, kJitHeaderNames[i], std::strlen(kJitHeaderNames[i]) + 1);
        h = fnv1a(h, kJitHeaderTexts[i], std::strlen(kJitHeaderTexts[i]) + 1);
    }
    char hex[17];
    std::snprintf(hex, sizeof(hex), "%016llx", (unsigned long long)h);
    k.hex = hex;
    const std::string dir = cache_dir();
    k.path = dir.empty() ? "" : dir + "/sk_" + k.hex + ".cubin";
    return k;
}

// A compiled configuration from the process or disk cache, without compiling.
bool jit_cached(const JitCfg& c, std::vector<char>* cubin, std::string* lowered, int* spill) {
    const JitKey k = jit_key(c);
    {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        auto it = g_jit_cubins.find(k.hex);
        if (it != g_jit_cubins.end()) {
            *cubin = it->second.cubin;
            *lowered = it->second.lowered;
            *spill = it->second.spill;
            return true;
        }
    }
    if (!k.path.empty() && env_int("SIP_FFT_JIT_VERBOSE", 0) == 0 && cache_read(k.path, cubin, lowered, spill)) {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        g_jit_cubins[k.hex] = {*cubin, *lowered, *spill};
        return true;
    }
    return false;
}

}  // namespace

bool sk_jit_compile(const JitCfg& c, std::vector<char>* cubin, std::string* lowered, std::string* err, int* spill) {
    const Nvrtc& api = nvrtc();
    if (!api.ok) {
        *err = "NVRTC is not available";
        return false;
    }
    if (jit_cached(c, cubin, lowered, spill)) return true;
    const std::string src = sk_jit_source();
    const std::string expr = sk_jit_name_expr(c);
    const JitKey key = jit_key(c);
    const std::vector<const char*>& opts = key.opts;
    const std::string& hex = key.hex;
    const std::string& path = key.path;

    nvrtcProgram prog = nullptr;
    if (api.create(&prog, src.c_str(), "sip_fft_jit.cu", kJitHeaderCount, kJitHeaderTexts, kJitHeaderNames) !=
        NVRTC_SUCCESS) {
        *err = "nvrtcCreateProgram failed";
        return false;
    }
    // the compiler's resource report (registers, spills) steers the choice
    // between configurations; SIP_FFT_JIT_VERBOSE=1 prints it
    const bool verbose = env_int("SIP_FFT_JIT_VERBOSE", 0) != 0;
    bool ok = api.add_name(prog, expr.c_str()) == NVRTC_SUCCESS;
    const nvrtcResult rc = ok ? api.compile(prog, (int)opts.size(), opts.data()) : NVRTC_ERROR_INVALID_INPUT;
    size_t ls = 0;
    std::string log;
    if (api.log_size(prog, &ls) == NVRTC_SUCCESS && ls > 1) {
        log.resize(ls);
        api.log(prog, &log[0]);
    }
    if (verbose) std::fprintf(stderr, "sip_fft jit %s\n%s\n", expr.c_str(), log.c_str());
    if (rc != NVRTC_SUCCESS) {
        *err = "NVRTC failed for " + expr + ": " + log.substr(0, 2000);
        api.destroy(&prog);
        return false;
    }
    const char* low = nullptr;
    size_t cs = 0;
    ok = api.lowered(prog, expr.c_str(), &low) == NVRTC_SUCCESS && low != nullptr &&
         api.cubin_size(prog, &cs) == NVRTC_SUCCESS && cs > 0;
    if (ok) {
        *lowered = low;
        cubin->resize(cs);
        ok = api.cubin(prog, cubin->data()) == NVRTC_SUCCESS;
    }
    api.destroy(&prog);
    if (!ok) {
        *err = "NVRTC produced no kernel for " + expr;
        return false;
    }
    *spill = spill_bytes(log);
    if (!path.empty()) cache_write(path, *cubin, *lowered, *spill);
    std::lock_guard<std::mutex> lk(g_jit_mu);
    g_jit_cubins[hex] = {*cubin, *lowered, *spill};
    return true;
}

namespace {

// Candidate configurations of a step, in order of preference: at most 32
// values per thread and pass (the default), then 16 and 48.
// SIP_FFT_JIT_E pins one.
std::vector<JitCfg> jit_candidates(int op, int mode, int sign, bool tw4, int n, long long transforms,
                                   size_t* n_first = nullptr) {
    std::vector<int> tries = {32, 16, 48};
    if (env_int("SIP_FFT_JIT_E", 0) > 0) tries = {env_int("SIP_FFT_JIT_E", 0)};
    std::vector<JitCfg> cands;
    std::vector<std::string> seen;
    auto add = [&](const JitCfg& c) {
        const std::string expr = sk_jit_name_expr(c);
        if (std::find(seen.begin(), seen.end(), expr) != seen.end()) return;
        seen.push_back(expr);
        cands.push_back(c);
    };
    // each try with the cheapest factorization largest radix first, then
    // (when its radices differ) smallest first: which order the compiler
    // fits in the registers without spills varies (a pulse tile of 4320
    // points as 18 x 16 x 15 on 288 threads spills 240 bytes per thread,
    // as 15 x 16 x 18 none)
    std::vector<std::vector<int>> orders = {jit_radices(n)};
    if (!orders[0].empty() && orders[0].front() != orders[0].back())
        orders.push_back(std::vector<int>(orders[0].rbegin(), orders[0].rend()));
    for (size_t oi = 0; oi < orders.size(); ++oi)
    for (int v : tries) {
        if (oi == 1 && n_first != nullptr && *n_first == 0) *n_first = cands.size();
        JitCfg c;
        if (!sk_jit_choose(op, mode, sign, tw4, n, transforms, &c, v, oi == 0 ? nullptr : &orders[oi])) continue;
        add(c);
        // The register file is split over the SM's four schedulers: with one
        // CTA per SM a block of 9-12 warps gets at most 168 registers per
        // thread, one of 8 warps 255.  So each candidate is also tried with
        // its threads rounded down to a multiple of 128 (more values per
        // thread) and the register target left to the compiler.
        if (c.T % 128 != 0 && c.T > 128) {
            JitCfg r = c;
            r.T = c.T / 128 * 128;
            bool ok = true;
            for (int rad : r.radices) {
                const long long b = (long long)r.P * (n / rad);
                if ((b + r.T - 1) / r.T * rad > 96) ok = false;  // values per thread and pass
            }
            r.minb = 1;
            if (ok) add(r);
        }
    }
    if (n_first != nullptr && *n_first == 0) *n_first = cands.size();
    return cands;
}

}  // namespace

bool sk_jit_select(int op, int mode, int sign, bool tw4, int n, long long transforms, JitCfg* out,
                   std::string* err) {
    // The first candidate in order without register spills wins, else the
    // one with the fewest spilled bytes.  The first is compiled alone (it
    // wins whenever it does not spill, which saves the others' compilation
    // time); only when it spills are the others of its radix order
    // compiled, concurrently, and only when they all spill those of the
    // reversed order (its first alone, then the rest).
    size_t n_first = 0;
    const std::vector<JitCfg> cands = jit_candidates(op, mode, sign, tw4, n, transforms, &n_first);
    if (cands.empty()) {
        *err = "no run-time configuration for this step";
        return false;
    }
    struct Result {
        bool ok = false;
        int spill = 0;
        std::string err;
    };
    std::vector<Result> res(cands.size());
    auto compile = [&](size_t i) {
        std::vector<char> cubin;
        std::string lowered;
        res[i].ok = sk_jit_compile(cands[i], &cubin, &lowered, &res[i].err, &res[i].spill);
    };
    compile(0);
    if (res[0].ok && res[0].spill == 0) {
        *out = cands[0];
        return true;
    }
    auto compile_range = [&](size_t lo, size_t hi) {
        std::vector<std::thread> workers;
        for (size_t i = lo; i < hi; ++i) workers.emplace_back(compile, i);
        for (auto& w : workers) w.join();
    };
    compile_range(1, n_first);
    bool clean = false;
    for (size_t i = 0; i < n_first; ++i) clean = clean || (res[i].ok && res[i].spill == 0);
    if (!clean && n_first < cands.size()) {
        // the reversed order's first candidate alone, then its others
        compile(n_first);
        if (!(res[n_first].ok && res[n_first].spill == 0)) compile_range(n_first + 1, cands.size());
    }
    int best = -1;
    const size_t done = clean ? n_first
                      : (n_first < cands.size() && res[n_first].ok && res[n_first].spill == 0) ? n_first + 1
                                                                                           : cands.size();
    for (size_t i = 0; i < done; ++i) {
        if (!res[i].ok) {
            *err = res[i].err;
            continue;
        }
        if (best < 0 || res[i].spill < res[best].spill) best = (int)i;
        if (res[i].spill == 0) break;
    }
    if (best < 0) return false;
    *out = cands[best];
    return true;
}

namespace {

// Entry (stable address) of a selected configuration.
const SkEntry* entry_of(const JitCfg& c) {
    const std::string key = sk_jit_name_expr(c);
    std::lock_guard<std::mutex> lk(g_jit_mu);
    auto it = g_jit_index.find(key);
    if (it != g_jit_index.end()) return it->second;
    SkEntry e;
    e.n = c.n;
    e.P = c.P;
    e.T = c.T;
    e.op = c.op;
    e.mode = c.mode;
    e.sign = c.sign;
    e.tw4 = c.tw4;
    e.twb = (c.twb & SK_TW_BASIS) != 0;
    e.flags = c.twb;
    e.stages = c.stages;
    e.radices = c.radices;
    e.LD = c.LD;
    e.smem = c.smem;
    e.fn = nullptr;
    e.minb = c.minb;
    e.jit = true;
    auto kit = g_jit_kernels.find(key);
    if (kit != g_jit_kernels.end()) e.fn = kit->second;
    g_jit_entries.push_back(e);
    g_jit_index[key] = &g_jit_entries.back();
    return &g_jit_entries.back();
}

// Selections by step (the joined candidate names): found + configuration.
std::map<std::string, std::pair<bool, JitCfg>>& g_jit_selected = *new std::map<std::string, std::pair<bool, JitCfg>>;

// The selection from cached binaries alone, when they decide it: the first
// candidate without spills whose predecessors are all cached, or the
// fewest spills when every candidate is cached.
bool select_cached(const std::vector<JitCfg>& cands, JitCfg* out) {
    int best = -1, best_spill = 0;
    for (size_t i = 0; i < cands.size(); ++i) {
        std::vector<char> cubin;
        std::string lowered;
        int spill = 0;
        if (!jit_cached(cands[i], &cubin, &lowered, &spill)) return false;
        if (best < 0 || spill < best_spill) {
            best = (int)i;
            best_spill = spill;
        }
        if (spill == 0) break;
    }
    if (best < 0) return false;
    *out = cands[best];
    return true;
}

// Background compilation: a FIFO of steps served by detached worker threads
// (2, or SIP_FFT_JIT_THREADS, at most 64).  The state is never destroyed, so a worker still compiling while
// the process exits touches no destroyed object; an exit handler (registered
// after NVRTC is loaded, so it runs before NVRTC's own teardown) stops the
// queue and waits up to 30 s for the jobs already running.  A fork waits
// (up to 60 s) until no compilation is running, so that no compiler state
// is copied mid-compilation; the child starts with an empty queue and no
// workers (its parent's threads do not exist there), re-creates its locks
// and compiles nothing (g_forked_child).
void register_drain();

struct JitWorkers {
    std::mutex mu;
    std::condition_variable cv, idle;
    std::deque<std::function<void()>> jobs;
    std::set<std::string> pending;  // step keys queued or running
    int running = 0;                // jobs being run
    bool started = false, stop = false;

    void start() {  // with mu held
        if (started) return;
        started = true;
        const int nthreads = std::max(1, std::min(64, env_int("SIP_FFT_JIT_THREADS", 2)));
        for (int i = 0; i < nthreads; ++i)
            std::thread([this] {
                for (;;) {
                    std::function<void()> job;
                    {
                        std::unique_lock<std::mutex> lk(mu);
                        cv.wait(lk, [this] { return stop || !jobs.empty(); });
                        if (stop) return;
                        job = std::move(jobs.front());
                        jobs.pop_front();
                        ++running;
                    }
                    // exit handlers run last-registered first: registering the
                    // drain again here puts it ahead of any handler the
                    // compiler registered during earlier compilations
                    register_drain();
                    job();
                    job = nullptr;
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        --running;
                    }
                    idle.notify_all();
                }
            }).detach();
    }
};

JitWorkers& workers();
void drain_at_exit();

void register_drain() { std::atexit(&drain_at_exit); }

void drain_at_exit() {
    JitWorkers& w = workers();
    std::unique_lock<std::mutex> lk(w.mu);
    w.stop = true;
    w.jobs.clear();
    w.cv.notify_all();
    w.idle.wait_for(lk, std::chrono::seconds(30), [&w] { return w.running == 0; });
}

// Fork: no compilation may be in flight; the lock is held across the fork.
void before_fork() {
    JitWorkers& w = workers();
    w.mu.lock();
    for (int i = 0; i < 600 && w.running > 0; ++i) {
        w.mu.unlock();
        std::this_thread::sleep_for(std::chrono::milliseconds(100));
        w.mu.lock();
    }
}

void after_fork_parent() {
    workers().mu.unlock();
    register_drain();
}

void after_fork_child() {
    JitWorkers& w = workers();
    new (&w.mu) std::mutex;
    new (&w.cv) std::condition_variable;
    new (&w.idle) std::condition_variable;
    w.jobs.clear();
    w.pending.clear();
    w.running = 0;
    w.started = false;
    w.stop = false;
    new (&g_jit_mu) std::mutex;
    g_forked_child = true;
}

// One small compilation on the calling thread before the first background
// job.  The compiler sets up much of its internal state (and registers the
// exit-time teardown of it) on its first compilation; doing that here, ahead
// of the drain handler's registration, puts the drain before that teardown
// at exit, so that a compilation still running when the process exits does
// not meet a compiler whose state is being destroyed (a crash observed when a
// process exited a fraction of a second after starting background jobs).
void nvrtc_warmup() {
    const Nvrtc& api = nvrtc();
    if (!api.ok) return;
    nvrtcProgram prog = nullptr;
    const char* src = "extern \"C\" __global__ void sip_fft_warmup(float* p) { p[threadIdx.x] *= 2.0f; }\n";
    if (api.create(&prog, src, "sip_fft_warmup.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) return;
    std::vector<const char*> opts(std::begin(kOptions), std::end(kOptions));
    opts.push_back("--ptxas-options=-v");
    (void)api.compile(prog, (int)opts.size(), opts.data());
    size_t cs = 0;
    (void)api.cubin_size(prog, &cs);
    api.destroy(&prog);
}

JitWorkers& workers() {
    static JitWorkers* w = [] {
        JitWorkers* p = new JitWorkers;
        pthread_atfork(&before_fork, &after_fork_parent, &after_fork_child);
        nvrtc_warmup();
        register_drain();
        return p;
    }();
    return *w;
}

}  // namespace

const SkEntry* sk_jit_entry(int op, int mode, int sign, bool tw4, int n, long long transforms, bool sync) {
    if (!sk_jit_available()) return nullptr;
    const std::vector<JitCfg> cands = jit_candidates(op, mode, sign, tw4, n, transforms);
    if (cands.empty()) return nullptr;
    std::string step;
    for (const JitCfg& c : cands) step += sk_jit_name_expr(c) + ";";
    bool known = false, found = false;
    JitCfg sel;
    {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        auto it = g_jit_selected.find(step);
        if (it != g_jit_selected.end()) {
            known = true;
            found = it->second.first;
            sel = it->second.second;
        }
    }
    if (known) return found ? entry_of(sel) : nullptr;
    if (select_cached(cands, &sel)) {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        g_jit_selected[step] = {true, sel};
    } else if (sync) {
        std::string err;
        const bool ok = sk_jit_select(op, mode, sign, tw4, n, transforms, &sel, &err);
        if (!ok && env_int("SIP_FFT_JIT_VERBOSE", 0) != 0) std::fprintf(stderr, "sip_fft jit: %s\n", err.c_str());
        {
            std::lock_guard<std::mutex> lk(g_jit_mu);
            g_jit_selected[step] = {ok, sel};
        }
        if (!ok) return nullptr;  // the generic tile kernel runs the step
    } else {
        // compile in the background; this plan runs the generic kernel, plans
        // made after the compilation finished use the specialized one
        JitWorkers& w = workers();
        std::lock_guard<std::mutex> lk(w.mu);
        if (!w.stop && w.pending.insert(step).second) {
            w.jobs.push_back([=] {
                JitCfg c;
                std::string err;
                const bool ok = sk_jit_select(op, mode, sign, tw4, n, transforms, &c, &err);
                {
                    std::lock_guard<std::mutex> l2(g_jit_mu);
                    g_jit_selected[step] = {ok, c};
                }
                {
                    std::lock_guard<std::mutex> l3(workers().mu);
                    workers().pending.erase(step);
                }
                workers().idle.notify_all();
            });
            w.start();
            w.cv.notify_one();
        }
        return nullptr;
    }
    return entry_of(sel);
}

bool sk_jit_wait(long long timeout_ms) {
    JitWorkers& w = workers();
    std::unique_lock<std::mutex> lk(w.mu);
    return w.idle.wait_for(lk, std::chrono::milliseconds(std::max(0LL, timeout_ms)),
                           [&w] { return w.pending.empty(); });
}

const void* sk_jit_load(const SkEntry* entry) {
    const JitCfg c = cfg_of(*entry);
    const std::string key = sk_jit_name_expr(c);
    {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        auto kit = g_jit_kernels.find(key);
        if (kit != g_jit_kernels.end()) return kit->second;
    }
    std::vector<char> cubin;
    std::string lowered, err;
    int spill = 0;
    if (!sk_jit_compile(c, &cubin, &lowered, &err, &spill)) throw PlanError(AsdSip::ACL_ERROR_INTERNAL_ERROR, err);
    cudaLibrary_t lib = nullptr;
    cudaError_t e = cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess)
        throw PlanError(AsdSip::ACL_ERROR_INTERNAL_ERROR, std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e));
    cudaKernel_t k = nullptr;
    e = cudaLibraryGetKernel(&k, lib, lowered.c_str());
    if (e != cudaSuccess)
        throw PlanError(AsdSip::ACL_ERROR_INTERNAL_ERROR, std::string("cudaLibraryGetKernel: ") + cudaGetErrorString(e));
    const void* fn = reinterpret_cast<const void*>(k);
    std::lock_guard<std::mutex> lk(g_jit_mu);
    auto kit = g_jit_kernels.find(key);
    if (kit != g_jit_kernels.end()) return kit->second;  // another thread loaded it first; lib stays loaded
    g_jit_kernels[key] = fn;
    auto it = g_jit_index.find(key);
    if (it != g_jit_index.end()) it->second->fn = fn;
    return fn;
}

}  // namespace sipfft
