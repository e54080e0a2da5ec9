/*
 * canonical.c -- CPU oracle for Redzone O(k) removal. TEST INFRASTRUCTURE ONLY: tests/, the
 * smoke check and bench.py's CPU-baseline leg may call it; the library never does.
 *
 * It restates, sequentially and payload-agnostically, the result every correct implementation
 * in the reference produces on the surviving prefix:
 *   - phase 1 marks the red-zone sources that are themselves removed
 *     (Redzone_CPU.hxx:12-24, redzone.hxx:698-706);
 *   - phase 2 walks i in [0,k): dest = R[i], src = cut+i, with the four cases of the paper's
 *     Table 1: move when both are valid, otherwise record a destination orphan or a source
 *     orphan in i order (Redzone_CPU.hxx:26-59, redzone.hxx:752-822);
 *   - phase 3 pairs the j-th destination orphan with the j-th source orphan
 *     (Redzone_CPU.hxx:104-129, redzone.hxx:913-934). The reference concatenates per-chunk
 *     orphan lists in chunk order (Redzone_CPU.hxx:209-219, redzone.hxx:852-900), which is the
 *     global i order used here.
 * Pinned against the reference's own redzone_CPU (compiled from its sources by oracle/Makefile)
 * by tests/test_oracle.py and by the golden vectors under tests/golden/.
 *
 * Also here: the stable O(n) removal (std::remove / thrust::remove semantics,
 * std_parallel_remove.hxx:13-36, Thrust_remove.hxx:15-17) and a duplicate/range validator.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Return codes mirror rz_status: 0 ok, 1 invalid argument, 2 duplicate, 3 out of range, 4 oom. */

int rz_oracle_validate(uint64_t n, const uint32_t* idx, uint64_t k) {
    uint64_t words = (n + 63) / 64;
    uint64_t* seen = (uint64_t*)calloc(words ? words : 1, 8);
    if (!seen) return 4;
    int rc = 0;
    for (uint64_t i = 0; i < k && rc == 0; ++i) {
        uint64_t r = idx[i];
        if (r >= n) { rc = 3; break; }
        uint64_t bit = 1ull << (r & 63);
        if (seen[r >> 6] & bit) rc = 2;
        seen[r >> 6] |= bit;
    }
    free(seen);
    return rc;
}

/* Redzone removal, in place on data[0..n) of w-byte items. Leaves the tail [n-k, n) as is. */
int rz_oracle_remove(void* data, uint64_t n, uint32_t w, const uint32_t* idx, uint64_t k) {
    if (k > n || w == 0) return 1;
    if (k == 0 || k == n) return 0; /* nothing moves (redzone.hxx:651) */
    uint8_t* A = (uint8_t*)data;
    const uint64_t cut = n - k;
    uint8_t* red = (uint8_t*)calloc(k, 1);
    uint32_t* dorph = (uint32_t*)malloc(k * sizeof(uint32_t));
    uint64_t* sorph = (uint64_t*)malloc(k * sizeof(uint64_t));
    if (!red || !dorph || !sorph) { free(red); free(dorph); free(sorph); return 4; }
    int rc = 0;
    /* phase 1: which red-zone sources are removed */
    for (uint64_t i = 0; i < k; ++i) {
        uint64_t r = idx[i];
        if (r >= n) { rc = 3; goto done; }
        if (r >= cut) red[r - cut] = 1;
    }
    /* phase 2: four cases, orphans recorded in i order */
    uint64_t nd = 0, ns = 0;
    for (uint64_t i = 0; i < k; ++i) {
        const uint64_t dest = idx[i];
        const int dest_valid = dest < cut;
        const int src_valid = !red[i];
        if (dest_valid && src_valid) memcpy(A + dest * w, A + (cut + i) * w, w);
        else if (dest_valid) dorph[nd++] = (uint32_t)dest;
        else if (src_valid) sorph[ns++] = cut + i;
    }
    if (nd != ns) { rc = 2; goto done; } /* only possible with duplicate indices */
    /* phase 3: pair orphans by rank */
    for (uint64_t j = 0; j < nd; ++j) memcpy(A + (uint64_t)dorph[j] * w, A + sorph[j] * w, w);
done:
    free(red); free(dorph); free(sorph);
    return rc;
}

/* Stable removal (survivors keep their order), in place. */
int rz_oracle_stable_remove(void* data, uint64_t n, uint32_t w, const uint32_t* idx, uint64_t k) {
    if (k > n || w == 0) return 1;
    uint8_t* A = (uint8_t*)data;
    uint64_t words = (n + 63) / 64;
    uint64_t* rm = (uint64_t*)calloc(words ? words : 1, 8);
    if (!rm) return 4;
    for (uint64_t i = 0; i < k; ++i) {
        uint64_t r = idx[i];
        if (r >= n) { free(rm); return 3; }
        rm[r >> 6] |= 1ull << (r & 63);
    }
    uint64_t o = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (rm[i >> 6] & (1ull << (i & 63))) continue;
        if (o != i) memcpy(A + o * w, A + i * w, w);
        ++o;
    }
    free(rm);
    return 0;
}

/* Batched form: lists are independent; offsets are element offsets into one data buffer and one
 * index buffer (the layout of the batched kernel's descriptor table). */
int rz_oracle_remove_batched(void* data, uint32_t w, const uint32_t* idx, int64_t nlists,
                             const uint64_t* data_off, const uint64_t* n, const uint64_t* idx_off,
                             const uint64_t* k) {
    for (int64_t l = 0; l < nlists; ++l) {
        int rc = rz_oracle_remove((uint8_t*)data + data_off[l] * w, n[l], w, idx + idx_off[l], k[l]);
        if (rc) return rc;
    }
    return 0;
}
