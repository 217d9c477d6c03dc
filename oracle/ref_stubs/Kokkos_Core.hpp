/* Host-only stand-in for the few Kokkos names the reference's hydro headers
 * use: inline-function markers and serial atomics. The pair bodies compiled
 * against it run on the CPU, one target per OpenMP thread; j-side writes
 * go through OpenMP atomics. */
#ifndef ORACLE_STUB_KOKKOS_CORE_HPP
#define ORACLE_STUB_KOKKOS_CORE_HPP
#include <cstddef>
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_LAMBDA [=]
#define KOKKOS_IF_ON_HOST(x) { _ORACLE_UNPAREN x }
#define _ORACLE_UNPAREN(...) __VA_ARGS__
#define KOKKOS_IF_ON_DEVICE(x) {}
namespace Kokkos {
template <class T, class U> inline void atomic_add(T* p, U v)
{
    const T add = (T)v;
#pragma omp atomic update
    *p += add;
}
template <class T, class U> inline void atomic_max(T* p, U v)
{
#pragma omp critical(oracle_stub_atomic_max)
    { if (*p < v) *p = v; }
}
template <class T, class U> inline void atomic_min(T* p, U v)
{
#pragma omp critical(oracle_stub_atomic_min)
    { if (*p > v) *p = v; }
}
template <class T, class U> inline void atomic_store(T* p, U v)
{
    const T val = (T)v;
#pragma omp atomic write
    *p = val;
}
template <class T> inline T atomic_load(T* p) { return *p; }
}
#endif
