// Host-only check of the batched kernel's work-queue order (redzone_b200/csrc/rz_batch_order.h):
// for random mixes of lists and every lag, the queue is a permutation of the items, and each
// item comes after everything it waits for -- all MARK items of its list before its first
// CLASSIFY item, all CLASSIFY items before its first PAIR item -- which is what makes the
// kernel's bounded waits always end. Prints "ok" or the first violation.
#include <cstdio>
#include <map>
#include <random>
#include <set>

#include "rz_batch_order.h"

enum : uint32_t { K_MARK = 0, K_SINGLE = 1, K_CLASSIFY = 2, K_PAIR = 3 };

static uint2 item(uint32_t list, uint32_t word) {
    uint2 v;
    v.x = list;
    v.y = word;
    return v;
}

int main() {
    std::mt19937 rng(7);
    for (int trial = 0; trial < 300; ++trial) {
        const int nlists = 1 + int(rng() % 200);
        std::vector<uint2> mark, single, classify, pair;
        std::vector<uint32_t> groups;
        for (int l = 0; l < nlists; ++l) {
            if (rng() % 3 == 0) {
                single.push_back(item(uint32_t(l), K_SINGLE << 28));
                continue;
            }
            const uint32_t g = 1 + rng() % (rng() % 4 == 0 ? 200 : 6);
            groups.push_back(g);
            for (uint32_t q = 0; q < g; ++q) {
                mark.push_back(item(uint32_t(l), (K_MARK << 28) | q));
                classify.push_back(item(uint32_t(l), (K_CLASSIFY << 28) | q));
                pair.push_back(item(uint32_t(l), (K_PAIR << 28) | q));
            }
        }
        for (size_t lag : {size_t(0), size_t(1), size_t(7), size_t(148), size_t(888)}) {
            std::vector<uint2> out;
            rz::order_queue(mark, single, classify, pair, groups, lag, out);
            if (out.size() != mark.size() + single.size() + classify.size() + pair.size()) {
                std::printf("trial %d lag %zu: %zu items, expected %zu\n", trial, lag, out.size(),
                            mark.size() + single.size() + classify.size() + pair.size());
                return 1;
            }
            std::set<std::pair<uint32_t, uint32_t>> seen;
            std::map<uint32_t, size_t> last_mark, last_classify, first_classify, first_pair;
            for (size_t t = 0; t < out.size(); ++t) {
                const uint32_t l = out[t].x, kind = out[t].y >> 28;
                if (!seen.insert({out[t].x, out[t].y}).second) {
                    std::printf("trial %d lag %zu: item repeated at %zu\n", trial, lag, t);
                    return 1;
                }
                if (kind == K_MARK) last_mark[l] = t;
                if (kind == K_CLASSIFY) {
                    last_classify[l] = t;
                    if (!first_classify.count(l)) first_classify[l] = t;
                }
                if (kind == K_PAIR && !first_pair.count(l)) first_pair[l] = t;
            }
            for (auto& kv : first_classify)
                if (last_mark.at(kv.first) > kv.second) {
                    std::printf("trial %d lag %zu: list %u classifies before its marks\n", trial, lag, kv.first);
                    return 1;
                }
            for (auto& kv : first_pair)
                if (last_classify.at(kv.first) > kv.second) {
                    std::printf("trial %d lag %zu: list %u pairs before it is classified\n", trial, lag, kv.first);
                    return 1;
                }
        }
    }
    std::printf("ok\n");
    return 0;
}
