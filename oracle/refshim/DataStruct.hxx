// oracle/refshim/DataStruct.hxx -- project-written stand-in for the reference's fixture header
// (DataStruct.hxx, which pulls in Macros.hxx). TEST INFRASTRUCTURE ONLY.
//
// The reference's CPU algorithm files (Redzone_CPU.hxx, std_parallel_remove.hxx) are compiled
// unmodified where they lie. They need only a handful of names from their fixture/utility
// headers, and those headers do not compile with g++ 13 as shipped (Macros.hxx:451 redeclares a
// template parameter; its CUDA-only parts need nvcc). oracle/Makefile puts this directory first
// on the quoted-include path, so the reference's `#include "DataStruct.hxx"` resolves here.
// Provided names and their meaning in the reference:
//   divup(n, d)      ceiling division                                (Macros.hxx:131-133)
//   bs::timer        phase timer; current_us() is always 0 there,   (Macros.hxx:34-64)
//                    because stop() is never called -- kept as 0
//   removeme         the -1 mark of the O(n) baselines               (DataStruct.hxx:9)
//   TestLists_t      the benchmark fixture, referenced only by the reference's own test driver
//                    functions (never called through this build), so an inert placeholder
#pragma once

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <thread>
#include <vector>

#ifndef __host__
#define __host__
#endif

template <typename A, typename B>
constexpr auto divup(A n, B d) {
    return (n + d - 1) / d;
}

namespace bs {
struct timer {
    long long current_us() const { return 0; }
};
}  // namespace bs

static constexpr int removeme = -1;

struct TestLists_t {
    TestLists_t(int, int) {}
    void Update(int, int, int) {}
    bool isOK_CPU() const { return true; }
    int* host_A = nullptr;
    int* host_R = nullptr;
    int Asize = 0;
    int Rsize = 0;
};
