// cl_as_cpp.hpp -- lets the reference's OpenCL C kernel file compile as C++ so its kernels can be
// run serially on the host as the oracle.  TEST INFRASTRUCTURE ONLY (see oracle/be_oracle.c).
//
// The OpenCL built-ins the kernels use are: the __kernel/__global qualifiers, the uchar/uint/ulong
// scalar types, get_global_id/get_global_size and the integer min/max.  An NDRange launch becomes
// nested loops that set the current work-item id (ref_ndrange below).  A serial sweep is one legal
// schedule of the reference's racy Scan kernels; the BE fixpoint does not depend on the schedule.
#pragma once
#include <cmath>
#include <climits>
#include <cstddef>
#include <cstdint>

#define __kernel
#define __global
typedef unsigned char uchar;
typedef unsigned int uint;
typedef unsigned long ulong;

namespace refcl {
extern thread_local size_t gid[3];
extern thread_local size_t gsz[3];
extern int nthreads;   // work-item threads of ref_ndrange (1 = serial)
}  // namespace refcl

static inline size_t get_global_id(int d) { return refcl::gid[d]; }
static inline size_t get_global_size(int d) { return refcl::gsz[d]; }
template <class T> static inline T min(T a, T b) { return b < a ? b : a; }
template <class T> static inline T max(T a, T b) { return a < b ? b : a; }

// Runs `body()` once per work-item of a 1-, 2- or 3-dimensional NDRange, dimension 0 fastest.
// With refcl::nthreads > 1 the work-items are spread over OpenMP threads (rows of dimension 0,
// or chunks of it for a 1-D range); the kernels' unsynchronised stores then race exactly as
// they do between GPU work-items, which the BE fixpoint tolerates.
template <class F> static void ref_ndrange(int dims, const size_t *sz, F body)
{
    const size_t s0 = sz[0], s1 = dims > 1 ? sz[1] : 1, s2 = dims > 2 ? sz[2] : 1;
    if (refcl::nthreads <= 1) {
        refcl::gsz[0] = s0; refcl::gsz[1] = s1; refcl::gsz[2] = s2;
        for (size_t k = 0; k < s2; ++k)
            for (size_t j = 0; j < s1; ++j)
                for (size_t i = 0; i < s0; ++i) {
                    refcl::gid[0] = i; refcl::gid[1] = j; refcl::gid[2] = k;
                    body();
                }
        return;
    }
    const size_t chunk = dims == 1 ? 4096 : s0;
    const long long nchunks = dims == 1 ? (long long)((s0 + chunk - 1) / chunk) : (long long)(s1 * s2);
#pragma omp parallel for schedule(static) num_threads(refcl::nthreads)
    for (long long c = 0; c < nchunks; ++c) {
        refcl::gsz[0] = s0; refcl::gsz[1] = s1; refcl::gsz[2] = s2;
        size_t i0 = 0, i1 = s0, j = 0, k = 0;
        if (dims == 1) {
            i0 = (size_t)c * chunk;
            i1 = i0 + chunk < s0 ? i0 + chunk : s0;
        } else {
            j = (size_t)c % s1;
            k = (size_t)c / s1;
        }
        for (size_t i = i0; i < i1; ++i) {
            refcl::gid[0] = i; refcl::gid[1] = j; refcl::gid[2] = k;
            body();
        }
    }
}
