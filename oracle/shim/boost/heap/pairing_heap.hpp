// Test infrastructure only: std-only stand-in for boost::heap::pairing_heap,
// sharing the indexed binary heap of fibonacci_heap.hpp (same API surface).
#pragma once
#include <boost/heap/fibonacci_heap.hpp>

namespace boost {
namespace heap {
template <class T>
class pairing_heap : public shim_detail::indexed_heap<T> {};
}  // namespace heap
}  // namespace boost
