// boost::shared_ptr and enable_shared_from_this as the std ones (using-declarations, so
// that unqualified names under "using namespace std; using namespace boost;" agree).
#ifndef XPIR_COMPAT_BOOST_SHARED_PTR_HPP
#define XPIR_COMPAT_BOOST_SHARED_PTR_HPP

#include <memory>

namespace boost {
using std::enable_shared_from_this;
using std::shared_ptr;
}  // namespace boost

#endif
