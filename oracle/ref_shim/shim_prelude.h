// Force-included before the reference's device sources when they are compiled
// as host C++ for the oracle.  Supplies the CUDA device built-ins those sources
// call (atomics, bit casts) with host equivalents.  Test infrastructure only.
#ifndef UPBP_ORACLE_SHIM_PRELUDE_H
#define UPBP_ORACLE_SHIM_PRELUDE_H

#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

using std::isinf;
using std::isnan;

inline int __float_as_int(float f)
{
    int i;
    std::memcpy(&i, &f, sizeof(i));
    return i;
}

inline float __int_as_float(int i)
{
    float f;
    std::memcpy(&f, &i, sizeof(f));
    return f;
}

inline unsigned int atomicAdd(unsigned int* addr, unsigned int val)
{
    return __atomic_fetch_add(addr, val, __ATOMIC_RELAXED);
}

inline float atomicAdd(float* addr, float val)
{
    float old;
    __atomic_load(addr, &old, __ATOMIC_RELAXED);
    float desired;
    do {
        desired = old + val;
    } while (!__atomic_compare_exchange(addr, &old, &desired, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
    return old;
}

#endif
