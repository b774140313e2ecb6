// Minimal stand-in for boost::signals2: a signal calls its connected slots in connection
// order; a connection can disconnect its slot.  (XPIR's client wires its view, its reply
// writer and its catalog menu to the client through these signals.)
#ifndef XPIR_COMPAT_BOOST_SIGNALS2_HPP
#define XPIR_COMPAT_BOOST_SIGNALS2_HPP

#include <functional>
#include <memory>
#include <vector>

namespace boost {
namespace signals2 {

class connection {
 public:
  connection() {}
  explicit connection(std::shared_ptr<bool> alive) : alive_(alive) {}
  void disconnect() {
    if (alive_) *alive_ = false;
  }
  bool connected() const { return alive_ && *alive_; }

 private:
  std::shared_ptr<bool> alive_;
};

template <class Signature>
class signal;

template <class R, class... Args>
class signal<R(Args...)> {
 public:
  typedef std::function<R(Args...)> slot_function_type;
  signal() {}
  signal(const signal &) = delete;
  signal &operator=(const signal &) = delete;
  connection connect(const slot_function_type &f) {
    slots_.push_back(Slot{f, std::make_shared<bool>(true)});
    return connection(slots_.back().alive);
  }
  void operator()(Args... args) {
    for (size_t i = 0; i < slots_.size(); i++)
      if (*slots_[i].alive) slots_[i].fn(args...);
  }

 private:
  struct Slot {
    slot_function_type fn;
    std::shared_ptr<bool> alive;
  };
  std::vector<Slot> slots_;
};

}  // namespace signals2
}  // namespace boost

#endif
