// Minimal stand-in for boost::queue (boost/pending/queue.hpp).
#ifndef XPIR_REF_SHIM_PENDING_QUEUE_HPP
#define XPIR_REF_SHIM_PENDING_QUEUE_HPP

#include <deque>

namespace boost {

template <class T>
class queue {
 public:
  void push(const T &v) { d_.push_back(v); }
  T &front() { return d_.front(); }
  void pop() { d_.pop_front(); }
  bool empty() const { return d_.empty(); }
  size_t size() const { return d_.size(); }

 private:
  std::deque<T> d_;
};

}  // namespace boost

#endif
