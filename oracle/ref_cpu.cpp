// oracle/ref_cpu.cpp -- C entry points over the reference's own CPU implementations, compiled
// from the reference sources where they lie (see oracle/Makefile). TEST INFRASTRUCTURE ONLY:
// used to pin the oracle, to make golden vectors, and as bench.py's timed CPU baseline.
#include "Redzone_CPU.hxx"          // reference: redzone_CPU, Redzone_CPU.hxx:150-248
#include "std_parallel_remove.hxx"  // reference: par_remove_phase1/2, std_parallel_remove.hxx:13-36

extern "C" {

// Redzone on the CPU, in place; clobbers `removals` exactly as the reference does.
void ref_redzone_cpu(int* list, int listsize, int* removals, int removecount) {
    int times[4] = {0, 0, 0, 0};
    redzone_CPU(list, listsize, removals, removecount, times);
}

// Mark with -1, then std::remove(par_unseq): the reference's CPU O(n) comparator.
void ref_par_remove(int* list, int listsize, const int* removals, int removecount) {
    par_remove_phase1(list, removals, removecount);
    par_remove_phase2(list, listsize);
}

// Worker count redzone_CPU splits its work into (hardware_concurrency - 1, Redzone_CPU.hxx:153).
int ref_redzone_threads() { return int(std::thread::hardware_concurrency() - 1); }

// Threads the TBB-API shim runs the reference's parallel_for bodies on.
int ref_pool_threads() { return int(tbb::shim::pool::get().workers()); }

// 1 when libstdc++'s parallel algorithms have a parallel backend (they do only with oneTBB).
int ref_pstl_parallel() {
#if defined(_PSTL_PAR_BACKEND_TBB) || defined(__PSTL_PAR_BACKEND_TBB)
    return 1;
#else
    return 0;
#endif
}

}  // extern "C"
