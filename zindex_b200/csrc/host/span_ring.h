// Spans of a ring buffer: variable-size byte ranges taken in order and freed
// in any order (the request server's page-locked staging of request bases).
//
// Spans are placed after the newest live span, or at the start of the ring
// when the end has no room (the tail of the ring is then skipped); space
// comes back as the oldest spans are freed, so a span freed early waits for
// the older ones. Only offsets are managed here, no memory.
#pragma once
#include <stdint.h>

#include <deque>

namespace zx {

class SpanRing {
 public:
  explicit SpanRing(uint64_t capacity = 0) : cap_(capacity) {}

  uint64_t capacity() const { return cap_; }
  bool empty() const { return spans_.empty(); }
  uint64_t live() const { return spans_.size(); }

  // Offset of n contiguous free bytes (0 < n <= capacity) and the span's id;
  // false when they are not free yet.
  bool reserve(uint64_t n, uint64_t* off, uint64_t* id) {
    if (n == 0 || n > cap_) return false;
    uint64_t at = UINT64_MAX;
    if (spans_.empty()) {
      head_ = tail_ = 0;
      at = 0;
    } else if (tail_ > head_) {  // live spans in [head, tail)
      if (cap_ - tail_ >= n) at = tail_;
      else if (head_ >= n) at = 0;
    } else if (head_ - tail_ >= n) {  // wrapped: live in [head, cap) and [0, tail)
      at = tail_;
    }
    if (at == UINT64_MAX) return false;
    *off = at;
    *id = next_id_++;
    spans_.push_back(Span{at, false});
    tail_ = at + n;
    return true;
  }

  // Frees span `id` (ids of live spans only; others are ignored).
  void release(uint64_t id) {
    if (spans_.empty() || id < first_id_ || id - first_id_ >= spans_.size()) return;
    spans_[id - first_id_].released = true;
    while (!spans_.empty() && spans_.front().released) {
      spans_.pop_front();
      ++first_id_;
    }
    if (spans_.empty()) head_ = tail_ = 0;
    else head_ = spans_.front().off;
  }

 private:
  struct Span {
    uint64_t off;
    bool released;
  };
  uint64_t cap_ = 0, head_ = 0, tail_ = 0;
  uint64_t next_id_ = 1, first_id_ = 1;  // ids of the spans are consecutive
  std::deque<Span> spans_;
};

}  // namespace zx
