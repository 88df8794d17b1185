// Lookup of the size-specialized kernels compiled by the sk_shard units.
#include <algorithm>

#include "sk_configs.h"
#include "sk_registry.h"

namespace sipfft {

void sk_register_shard_0(std::vector<SkEntry>&);
void sk_register_shard_1(std::vector<SkEntry>&);
void sk_register_shard_2(std::vector<SkEntry>&);
void sk_register_shard_3(std::vector<SkEntry>&);
void sk_register_shard_4(std::vector<SkEntry>&);
void sk_register_shard_5(std::vector<SkEntry>&);
void sk_register_shard_6(std::vector<SkEntry>&);
void sk_register_shard_7(std::vector<SkEntry>&);

const std::vector<SkEntry>& sk_registry() {
    static const std::vector<SkEntry> reg = [] {
        std::vector<SkEntry> v;
        sk_register_shard_0(v);
        sk_register_shard_1(v);
        sk_register_shard_2(v);
        sk_register_shard_3(v);
        sk_register_shard_4(v);
        sk_register_shard_5(v);
        sk_register_shard_6(v);
        sk_register_shard_7(v);
        std::stable_sort(v.begin(), v.end(), [](const SkEntry& a, const SkEntry& b) { return a.order < b.order; });
        return v;
    }();
    return reg;
}

const SkEntry* sk_find(int op, int mode, int sign, bool tw4, int n, int variant) {
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

}  // namespace sipfft
