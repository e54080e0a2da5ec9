// rz_batch_order.h -- the work-queue order of the batched kernel (host only; rz_batched.cu).
// Items are uint2 {list, kind << 28 | group}; kept in its own header so that a host-only test
// can check the order's invariants (every item after everything it waits for) without a GPU.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include <vector_types.h>

namespace rz {

// Queue order. With lag == 0, phase by phase over all lists. Otherwise the multi-tile lists run
// as a wavefront, list after list: a list's CLASSIFY items follow its MARK items, and its PAIR
// items its CLASSIFY items, by about `lag` tickets (a grid or more, so what an item waits for was
// taken a full round of the grid earlier and has normally finished). A list's phases thus run
// close together in time: the index list is read again while still in L2, and its hole writes
// -- classified and orphan ones alike -- land while the lines of its prefix are still in L2,
// where writes to the same 32-byte sector merge before one write-back. MARK items run ahead of the wavefront by at most 2 lag; SINGLE items fill
// the gaps the lags leave. Every item still follows everything it waits for (MARK before
// CLASSIFY before PAIR of the same list), so no wait can deadlock.
// mark / classify / pair hold the groups of each multi-tile list in list order; `groups` holds
// each such list's group count, in the same order.
inline void order_queue(const std::vector<uint2>& mark, const std::vector<uint2>& single,
                        const std::vector<uint2>& classify, const std::vector<uint2>& pair,
                        const std::vector<uint32_t>& groups, size_t lag, std::vector<uint2>& out) {
    out.clear();
    if (lag == 0) {
        // Phase by phase: every MARK item, the SINGLE items (largest first, while the marks land),
        // every CLASSIFY item, every PAIR item.
        out.reserve(mark.size() + single.size() + classify.size() + pair.size());
        out.insert(out.end(), mark.begin(), mark.end());
        out.insert(out.end(), single.begin(), single.end());
        out.insert(out.end(), classify.begin(), classify.end());
        out.insert(out.end(), pair.begin(), pair.end());
        return;
    }
    const size_t nb = groups.size();
    std::vector<size_t> first(nb + 1, 0);  // first item of block b in mark / classify / pair
    for (size_t b = 0; b < nb; ++b) first[b + 1] = first[b] + groups[b];
    std::vector<size_t> last_m(nb, 0), last_c(nb, 0);
    size_t im = 0, ic = 0, ip = 0, is = 0;  // items emitted from each stream
    size_t bm = 0, bc = 0, bp = 0;          // block of the next item of each stream
    const size_t total = mark.size() + single.size() + classify.size() + pair.size();
    out.clear();
    out.reserve(total);
    auto pos = [&]() { return out.size(); };
    auto emit_m = [&]() {
        out.push_back(mark[im++]);
        if (im == first[bm + 1]) last_m[bm++] = pos();
    };
    auto emit_c = [&]() {
        out.push_back(classify[ic++]);
        if (ic == first[bc + 1]) last_c[bc++] = pos();
    };
    auto emit_p = [&]() {
        out.push_back(pair[ip++]);
        if (ip == first[bp + 1]) ++bp;
    };
    while (out.size() < total) {
        const bool p_ready = ip < pair.size() && bp < bc;            // its CLASSIFY items are all queued
        const bool c_ready = ic < classify.size() && bc < bm;        // its MARK items are all queued
        if (p_ready && last_c[bp] + lag <= pos()) emit_p();
        else if (c_ready && last_m[bc] + lag <= pos()) emit_c();
        else if (im < mark.size() && im < ic + 2 * lag) emit_m();
        else if (is < single.size()) out.push_back(single[is++]);
        else if (c_ready) emit_c();
        else if (p_ready) emit_p();
        else emit_m();
    }
}

}  // namespace rz
