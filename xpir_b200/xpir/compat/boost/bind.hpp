// boost::bind as std::bind (a using-declaration, so that an unqualified `bind` under
// "using namespace std; using namespace boost;" names one entity).
#ifndef XPIR_COMPAT_BOOST_BIND_HPP
#define XPIR_COMPAT_BOOST_BIND_HPP

#include <functional>

namespace boost {
using std::bind;
}  // namespace boost

// Boost.Bind's placeholders are visible at global scope (XPIR writes `_1` unqualified).
using std::placeholders::_1;
using std::placeholders::_2;
using std::placeholders::_3;

#endif
