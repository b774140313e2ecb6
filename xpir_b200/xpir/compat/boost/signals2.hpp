// Type-only stand-in for boost::signals2: the XPIR client headers included by the
// reference's query generator and reply extraction declare listener typedefs and
// connection members but the compiled reference files never fire a signal.
#ifndef XPIR_REF_SHIM_SIGNALS2_HPP
#define XPIR_REF_SHIM_SIGNALS2_HPP

#include <functional>

namespace boost {
namespace signals2 {

class connection {
 public:
  void disconnect() {}
};

template <class Signature>
class signal {
 public:
  typedef std::function<Signature> slot_function_type;
  connection connect(const slot_function_type &) { return connection(); }
  template <class... Args>
  void operator()(Args &&...) {}
};

}  // namespace signals2
}  // namespace boost

#endif
