// thx_ring.h -- internal: space bookkeeping of a FIFO ring of byte spans
// (pure C++, no CUDA), used by the pinned host staging ring of the uploads.
//
// Spans are placed at the head and retired oldest first.  The live spans
// occupy [tail, head) when head > tail, and [tail, end of the last span before
// the wrap) plus [0, head) when head <= tail; with live spans, head == tail
// means the ring is full.
#pragma once
#include <cstddef>
#include <deque>

namespace thx {

class RingSpace {
 public:
  explicit RingSpace(size_t cap = 0) : cap_(cap) {}
  void reset(size_t cap) {
    cap_ = cap;
    head_ = 0;
    spans_.clear();
  }
  size_t capacity() const { return cap_; }
  bool empty() const { return spans_.empty(); }
  size_t live() const { return spans_.size(); }

  // Offset of `need` contiguous free bytes; false when the oldest span has
  // to be retired first (or need exceeds the capacity).
  bool place(size_t need, size_t *off) const {
    if (need > cap_) return false;
    if (spans_.empty()) {
      *off = 0;
      return true;
    }
    const size_t tail = spans_.front().off;
    if (head_ > tail) {
      if (cap_ - head_ >= need) {
        *off = head_;
        return true;
      }
      if (tail >= need) {
        *off = 0;
        return true;
      }
      return false;
    }
    if (tail - head_ >= need) {  // wrapped; head == tail is full
      *off = head_;
      return true;
    }
    return false;
  }
  // record a span at an offset that place() returned
  void push(size_t off, size_t size) {
    spans_.push_back({off, size});
    head_ = off + size;
  }
  // retire the oldest span
  void pop() {
    spans_.pop_front();
    if (spans_.empty()) head_ = 0;
  }

 private:
  struct Span {
    size_t off, size;
  };
  size_t cap_ = 0, head_ = 0;
  std::deque<Span> spans_;
};

}  // namespace thx
