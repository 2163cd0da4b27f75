/*
 * win32_compat.h - force-included when the reference CPU backend is compiled
 * on Linux. src/core/engine.cpp of the reference times itself with the Win32
 * high resolution counter unconditionally (engine.cpp:98, 542-545); these
 * stand-ins give it a monotonic nanosecond clock. Test infrastructure only.
 */
#ifndef AV1B_ORACLE_WIN32_COMPAT_H
#define AV1B_ORACLE_WIN32_COMPAT_H
#ifndef _WIN32
#include <time.h>
typedef union {
  long long QuadPart;
} LARGE_INTEGER;
static inline int QueryPerformanceCounter(LARGE_INTEGER* v) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  v->QuadPart = (long long)ts.tv_sec * 1000000000LL + ts.tv_nsec;
  return 1;
}
static inline int QueryPerformanceFrequency(LARGE_INTEGER* v) {
  v->QuadPart = 1000000000LL;
  return 1;
}
#endif
#endif
