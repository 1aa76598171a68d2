// Minimal host-only stand-in for the parts of RAJA that the Devil Ray
// hot-path sources use (forall over a range, min/max/sum reducers, atomics,
// exclusive scans).  It exists only so that the reference's own C++ sources
// can be compiled on the host as a test oracle; it is not product code.
//
// Semantics follow RAJA's documented behaviour:
//   forall<seq_exec>              -> sequential loop
//   forall<omp_parallel_for_exec> -> `#pragma omp parallel for`
//   Reduce{Min,Max,Sum}           -> copies made by lambda capture share one
//                                    accumulator; get() returns the result
//   atomicAdd / atomicCAS         -> return the old value
//   exclusive_scan(_inplace)      -> sequential prefix sum
#ifndef ORACLE_SHIM_RAJA_HPP
#define ORACLE_SHIM_RAJA_HPP

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <iostream>
#include <limits>
#include <memory>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define RAJA_INLINE inline
#define RAJA_HOST_DEVICE
#define RAJA_DEVICE
#define RAJA_HOST

namespace RAJA
{
struct seq_exec {};
struct omp_parallel_for_exec {};
template <int N> struct cuda_exec {};
template <int N> struct hip_exec {};
struct seq_reduce {};
struct omp_reduce {};
struct cuda_reduce {};
struct hip_reduce {};
struct seq_atomic {};
struct omp_atomic {};
struct cuda_atomic {};
struct hip_atomic {};
struct auto_atomic {};

template <typename T> struct TypedRangeSegment
{
  T m_begin, m_end;
  TypedRangeSegment (T b, T e) : m_begin (b), m_end (e) {}
  T begin () const { return m_begin; }
  T end () const { return m_end; }
  T size () const { return m_end > m_begin ? m_end - m_begin : 0; }
};
using RangeSegment = TypedRangeSegment<long long>;

namespace shim_detail
{
template <typename Seg, typename Body> void run_seq (const Seg &seg, Body &&body)
{
  for (auto i = seg.begin (); i < seg.end (); ++i)
    body (i);
}
template <typename Seg, typename Body> void run_omp (const Seg &seg, Body &&body)
{
  const long long b = (long long)seg.begin ();
  const long long e = (long long)seg.end ();
#pragma omp parallel for schedule(static)
  for (long long i = b; i < e; ++i)
    body (i);
}
} // namespace shim_detail

template <typename Policy, typename Seg, typename Body>
void forall (const Seg &seg, Body &&body)
{
  if (std::is_same<Policy, omp_parallel_for_exec>::value)
    shim_detail::run_omp (seg, body);
  else
    shim_detail::run_seq (seg, body);
}

// Reducers: every copy refers to the same shared state, so a lambda that
// captures the reducer by value still contributes to the original.
template <typename T> struct ReduceState
{
  std::mutex m;
  T value;
  explicit ReduceState (T v) : value (v) {}
};

template <typename Policy, typename T> class ReduceMin
{
  std::shared_ptr<ReduceState<T>> s;
  public:
  explicit ReduceMin (T init) : s (std::make_shared<ReduceState<T>> (init)) {}
  const ReduceMin &min (T v) const
  {
    std::lock_guard<std::mutex> g (s->m);
    if (v < s->value) s->value = v;
    return *this;
  }
  T get () const { return s->value; }
  operator T () const { return s->value; }
};

template <typename Policy, typename T> class ReduceMax
{
  std::shared_ptr<ReduceState<T>> s;
  public:
  explicit ReduceMax (T init) : s (std::make_shared<ReduceState<T>> (init)) {}
  const ReduceMax &max (T v) const
  {
    std::lock_guard<std::mutex> g (s->m);
    if (v > s->value) s->value = v;
    return *this;
  }
  T get () const { return s->value; }
  operator T () const { return s->value; }
};

template <typename Policy, typename T> class ReduceSum
{
  std::shared_ptr<ReduceState<T>> s;
  public:
  explicit ReduceSum (T init) : s (std::make_shared<ReduceState<T>> (init)) {}
  const ReduceSum &operator+= (T v) const
  {
    std::lock_guard<std::mutex> g (s->m);
    s->value += v;
    return *this;
  }
  T get () const { return s->value; }
  operator T () const { return s->value; }
};

template <typename Policy, typename T> T atomicAdd (T *addr, T val)
{
  return __atomic_fetch_add (addr, val, __ATOMIC_SEQ_CST);
}
template <typename T> T atomicAdd (T *addr, T val)
{
  return __atomic_fetch_add (addr, val, __ATOMIC_SEQ_CST);
}
template <typename Policy, typename T> T atomicCAS (T *addr, T compare, T val)
{
  T expected = compare;
  __atomic_compare_exchange_n (addr, &expected, val, false, __ATOMIC_SEQ_CST,
                               __ATOMIC_SEQ_CST);
  return expected;
}
template <typename Policy, typename T> T atomicMin (T *addr, T val)
{
  T old = *addr;
  while (val < old &&
         !__atomic_compare_exchange_n (addr, &old, val, false, __ATOMIC_SEQ_CST,
                                       __ATOMIC_SEQ_CST))
  {
  }
  return old;
}
template <typename Policy, typename T> T atomicMax (T *addr, T val)
{
  T old = *addr;
  while (val > old &&
         !__atomic_compare_exchange_n (addr, &old, val, false, __ATOMIC_SEQ_CST,
                                       __ATOMIC_SEQ_CST))
  {
  }
  return old;
}

template <typename T> struct Span
{
  T *ptr;
  std::size_t n;
  T *begin () const { return ptr; }
  T *end () const { return ptr + n; }
  std::size_t size () const { return n; }
};
template <typename T, typename N> Span<T> make_span (T *p, N n)
{
  return Span<T>{ p, (std::size_t)n };
}

namespace operators
{
template <typename T> struct plus
{
  T operator() (const T &a, const T &b) const { return a + b; }
  static T identity () { return T (0); }
};
template <typename T> struct safe_plus
{
  T operator() (const T &a, const T &b) const { return a + b; }
  static T identity () { return T (0); }
};
} // namespace operators

template <typename Policy, typename InT, typename OutT, typename Op>
void exclusive_scan (Span<InT> in, Span<OutT> out, Op op)
{
  typename std::remove_const<OutT>::type acc = Op::identity ();
  for (std::size_t i = 0; i < in.size (); ++i)
  {
    typename std::remove_const<OutT>::type v = in.ptr[i];
    out.ptr[i] = acc;
    acc = op (acc, v);
  }
}
template <typename Policy, typename T, typename Op>
void exclusive_scan_inplace (Span<T> io, Op op)
{
  T acc = Op::identity ();
  for (std::size_t i = 0; i < io.size (); ++i)
  {
    T v = io.ptr[i];
    io.ptr[i] = acc;
    acc = op (acc, v);
  }
}

using std::make_tuple;
} // namespace RAJA

#endif
