// Minimal stand-in for <windows.h>: the reference's stopwatch_win.h needs LARGE_INTEGER and the
// performance-counter calls.  Backed by std::chrono.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <chrono>
typedef union _LARGE_INTEGER { long long QuadPart; } LARGE_INTEGER;
typedef int BOOL;
static inline BOOL QueryPerformanceFrequency(LARGE_INTEGER *f) { f->QuadPart = 1000000000LL; return 1; }
static inline BOOL QueryPerformanceCounter(LARGE_INTEGER *c)
{
    c->QuadPart = std::chrono::duration_cast<std::chrono::nanoseconds>(
                      std::chrono::steady_clock::now().time_since_epoch()).count();
    return 1;
}
