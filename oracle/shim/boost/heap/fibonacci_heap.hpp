// Test infrastructure only: a std-only stand-in for the two Boost.Heap
// containers that the reference CPU oracles include (PrunedDP++ and
// D-PrunedDP++, see oracle/Makefile).  It is never linked into the engine.
//
// The reference uses exactly this surface of boost::heap::fibonacci_heap and
// boost::heap::pairing_heap (Boost 1.75 documented API):
//   handle_type            copyable, default-constructible
//   handle_type push(const T&)
//   const T& top() const    -- the element that is *largest* under operator<
//   void pop()
//   void update(handle_type, const T&)   -- key may go up or down
//   size_type size() const
//
// Implemented as an indexed binary max-heap (O(log n) for every operation;
// Fibonacci heaps only change the asymptotics of decrease-key, not results:
// the costs the oracles return do not depend on the order of ties).
#pragma once
#include <cstddef>
#include <deque>
#include <vector>

namespace boost {
namespace heap {
namespace shim_detail {

template <class T>
class indexed_heap {
  struct cell {
    T value;
    std::size_t pos;  // index into heap_ while live
  };

 public:
  using value_type = T;
  using size_type = std::size_t;

  class handle_type {
   public:
    handle_type() : c_(nullptr) {}
    explicit handle_type(cell* c) : c_(c) {}
    const T& operator*() const { return c_->value; }
    cell* c_;
  };

  indexed_heap() = default;
  indexed_heap(const indexed_heap&) = delete;
  indexed_heap& operator=(const indexed_heap&) = delete;

  handle_type push(const T& v) {
    cell* c;
    if (!free_.empty()) {
      c = free_.back();
      free_.pop_back();
      c->value = v;
    } else {
      store_.push_back(cell{v, 0});
      c = &store_.back();
    }
    c->pos = heap_.size();
    heap_.push_back(c);
    sift_up(c->pos);
    return handle_type(c);
  }

  const T& top() const { return heap_.front()->value; }

  void pop() {
    cell* root = heap_.front();
    cell* last = heap_.back();
    heap_.pop_back();
    if (root != last) {
      heap_[0] = last;
      last->pos = 0;
      sift_down(0);
    }
    free_.push_back(root);
  }

  void update(handle_type h, const T& v) {
    h.c_->value = v;
    std::size_t p = h.c_->pos;
    sift_up(p);
    sift_down(h.c_->pos);
  }

  void increase(handle_type h, const T& v) { update(h, v); }
  void decrease(handle_type h, const T& v) { update(h, v); }

  size_type size() const { return heap_.size(); }
  bool empty() const { return heap_.empty(); }

 private:
  // max-heap on operator< : parent is not less than its children
  void sift_up(std::size_t i) {
    while (i > 0) {
      std::size_t p = (i - 1) / 2;
      if (heap_[p]->value < heap_[i]->value) {
        swap_cells(p, i);
        i = p;
      } else {
        break;
      }
    }
  }
  void sift_down(std::size_t i) {
    const std::size_t n = heap_.size();
    for (;;) {
      std::size_t l = 2 * i + 1, r = l + 1, m = i;
      if (l < n && heap_[m]->value < heap_[l]->value) m = l;
      if (r < n && heap_[m]->value < heap_[r]->value) m = r;
      if (m == i) break;
      swap_cells(i, m);
      i = m;
    }
  }
  void swap_cells(std::size_t a, std::size_t b) {
    cell* t = heap_[a];
    heap_[a] = heap_[b];
    heap_[b] = t;
    heap_[a]->pos = a;
    heap_[b]->pos = b;
  }

  std::deque<cell> store_;  // stable addresses for handles
  std::vector<cell*> free_;
  std::vector<cell*> heap_;
};

}  // namespace shim_detail

template <class T>
class fibonacci_heap : public shim_detail::indexed_heap<T> {};

}  // namespace heap
}  // namespace boost
